"""CPU oracle of the frame renderer (TEST INFRASTRUCTURE ONLY): a numpy restatement of
src/microcosmos/rendering.py:20-80 -- grey steric texture, node and debug pixels written in
the reference's scatter order (later writes win), uint8 conversion, nearest resize with
output index o reading floor((o + 0.5) * m / n) (float32).  Pinned against golden frames
that ran the reference's render() on numpy (tests/golden/render_*.npz)."""
from __future__ import annotations

import numpy as np

BASE = np.array([0.3, 0.6, 0.9], np.float32)
VAR = np.array([0.3, 0.2, 0.0], np.float32)


def render(position, debug_vector, color_bend, steric, sz, render_particles=True, uniform_color=False):
    steric = np.asarray(steric, np.float32)
    T, H, W = steric.shape
    tex = np.float32(1.0) - np.clip(steric, np.float32(0.0), np.float32(1.0))
    tex = np.stack([tex] * 3, axis=-1)
    if render_particles:
        pos = np.asarray(position, np.float32).reshape(T, -1, 2)
        N = pos.shape[1]
        col = np.broadcast_to(BASE, (N, 3)) if uniform_color else BASE + VAR * np.asarray(color_bend, np.float32)[:, None]
        for t in range(T):
            for i in range(N):
                x = min(max(int(np.floor(pos[t, i, 0])), 0), W - 1)
                y = min(max(int(np.floor(pos[t, i, 1])), 0), H - 1)
                tex[t, y, x] = col[i]
        d = pos if debug_vector is None else pos + np.asarray(debug_vector, np.float32).reshape(T, N, 2)
        for t in range(T):
            for i in range(N):
                x = min(max(int(np.floor(d[t, i, 0])), 0), W - 1)
                y = min(max(int(np.floor(d[t, i, 1])), 0), H - 1)
                tex[t, y, x] = (1.0, 0.0, 0.0)
    img = np.clip(tex * np.float32(255.0), 0, 255).astype(np.uint8)
    m = max(H, W)
    out = (sz * H // m, sz * W // m)
    for axis, (a, b) in ((1, (H, out[0])), (2, (W, out[1]))):
        if a != b:
            o = ((np.arange(b, dtype=np.float32) + np.float32(0.5)) * np.float32(a)) / np.float32(b)
            img = np.take(img, np.floor(o).astype(np.int64), axis=axis)
    return img
