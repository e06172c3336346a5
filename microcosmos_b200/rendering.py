"""Frames of a recorded rollout on the device: the reference's ``render``
(src/microcosmos/rendering.py:20-80) as the ``mc_render_frames`` kernels, writing uint8
RGB frames into a device tensor (no display, window or graphics API; save them with any
image writer)."""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .engine import _require_cuda


def _dev(x, dtype):
    return torch.as_tensor(np.asarray(x) if not isinstance(x, torch.Tensor) else x, dtype=dtype,
                           device="cuda").contiguous()


def render(node_timeseries, field_timeseries, sz, render_particles=True, uniform_color=False):
    """(T, sz*H//max(H,W), sz*W//max(H,W), 3) uint8 CUDA tensor: the steric field as a grey
    texture, nodes in BASE_COLOR + COLOR_VARIATION * color_bend (of the first frame),
    debug pixels (position + debug_vector) in red, nearest-neighbour resized."""
    _require_cuda()
    H, W = (int(v) for v in field_timeseries.grid_shape)
    steric = _dev(field_timeseries.steric, torch.float32).reshape(-1, H, W)
    T = int(steric.shape[0])
    pos = _dev(node_timeseries.position, torch.float32).reshape(T, -1, 2)
    N = int(pos.shape[1])
    dbg = getattr(node_timeseries, "debug_vector", None)
    dbg = _dev(dbg, torch.float32).reshape(T, N, 2) if dbg is not None else None
    col = getattr(node_timeseries, "color_bend", None)
    if col is not None:
        col = _dev(col, torch.float32)
        col = (col[0] if col.dim() == 2 else col).reshape(N).contiguous()
    m = max(H, W)
    oh, ow = sz * H // m, sz * W // m
    frames = torch.empty((T, oh, ow, 3), dtype=torch.uint8, device="cuda")
    lib = _lib.load()
    scratch = torch.empty(max(1, lib.mc_render_scratch_bytes(T, H, W) // 4), dtype=torch.int32, device="cuda")
    ptr = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
    _lib.check(lib.mc_render_frames(ptr(pos), ptr(dbg), ptr(col), ptr(steric), T, N, H, W, int(sz),
                                    int(bool(render_particles)), int(bool(uniform_color)), ptr(scratch),
                                    ptr(frames), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    return frames
