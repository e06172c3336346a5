"""The allocation-free steric-potential entry point (mc_steric_potential_noalloc).

It exists for callers that cannot call cudaMalloc (a framework that owns all device
memory and hands a custom call no workspace, a host loop that must not allocate while it
runs).  Its scratch is a fixed file-scope device array, so this test checks, through the
C ABI, that two calls in a row reproduce the steric field the regular rollout entry point
(mc_rollout, one step, zero velocity) writes to fields.steric, within the tolerance the
parity tests use.  It lives in its own file so it is collected after every other test.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from microcosmos_b200 import _lib, baseline_config, scenarios  # noqa: E402
from microcosmos_b200.engine import DeviceState, Plan  # noqa: E402
from oracle import ref_numpy as O  # noqa: E402

TOL = 1e-5


def steric_via_rollout(sc, cfg):
    """fields.steric after one regular step from the scenario's positions with zero velocity."""
    st = DeviceState.from_scenario(sc)
    st.velocity.zero_()
    plan = Plan.for_states([st], [cfg], [0.01])
    plan.rollout([st], 1)
    torch.cuda.synchronize()
    return st.steric.cpu().numpy()


def steric_noalloc(pos, H, W, cfg):
    lib = _lib.load()
    out = torch.full((H, W), float("nan"), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    status = lib.mc_steric_potential_noalloc(ctypes.c_void_p(pos.data_ptr()), pos.shape[0], H, W,
                                             float(cfg.steric_sigma), float(cfg.steric_scatter_value),
                                             ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
    _lib.check(status)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_steric_matches_rollout_twice():
    cfg = baseline_config()
    cases = [scenarios.make_scenario(96, 128, 5, 30, seed=41), scenarios.make_scenario(64, 64, 3, 20, seed=42),
             scenarios.make_scenario(60, 90, 3, 16, seed=43)]  # 60 x 90: the mixed-radix FFT path
    refs = [steric_via_rollout(sc, cfg) for sc in cases]
    # calls in a row on the shared scratch (different sizes, so leftovers would show)
    for sc, ref in zip(cases + cases[:1], refs + refs[:1]):
        pos = torch.as_tensor(sc.position, device="cuda").contiguous()
        got = steric_noalloc(pos, sc.H, sc.W, cfg)
        assert np.isfinite(got).all()
        assert O.rel_l2(got, ref) <= TOL
        # and against the oracle's update_steric_potential of the same positions
        oref = O.update_steric_potential(sc.H, sc.W, sc.position, cfg.steric_sigma, cfg.steric_scatter_value)
        assert O.rel_l2(got, oref) <= TOL


def _crowded_positions(H, W, N, crowd, seed):
    """N positions on an H x W grid, `crowd` of them inside one 16 x 16 tile (more than the
    per-tile bin holds, so that tile spills into the overflow list and the arena)."""
    rng = np.random.default_rng(seed)
    pos = np.stack([rng.uniform(0, W, N), rng.uniform(0, H, N)], axis=1).astype(np.float32)
    pos[:crowd] = np.stack([rng.uniform(32, 48, crowd), rng.uniform(48, 64, crowd)], axis=1).astype(np.float32)
    return pos


def test_noalloc_at_its_limits_and_after_smaller_calls():
    """512 x 512 with 16,384 nodes (the limits), 600 of them in one tile (2,400 deposit
    entries against a bin of 512); then a small call, then the large one again, and the
    small one first in a fresh order: each matches the oracle."""
    cfg = baseline_config()
    big = (512, 512, _crowded_positions(512, 512, 16384, 600, seed=7))
    small = (64, 96, _crowded_positions(64, 96, 300, 200, seed=8))
    for H, W, p in (small, big, small, big, big):
        got = steric_noalloc(torch.as_tensor(p, device="cuda").contiguous(), H, W, cfg)
        oref = O.update_steric_potential(H, W, p, cfg.steric_sigma, cfg.steric_scatter_value)
        assert np.isfinite(got).all()
        assert O.rel_l2(got, oref) <= TOL, (H, W)


def test_noalloc_rejects_sizes_beyond_its_limit():
    lib = _lib.load()
    pos = torch.zeros((4, 2), dtype=torch.float32, device="cuda")
    out = torch.zeros((1024, 1024), dtype=torch.float32, device="cuda")
    status = lib.mc_steric_potential_noalloc(ctypes.c_void_p(pos.data_ptr()), 4, 1024, 1024, 1.5, 1.0,
                                             ctypes.c_void_p(out.data_ptr()), None)
    assert status == _lib.MC_ERR_INVALID
    assert b"512" in lib.mc_last_error()
