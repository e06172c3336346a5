"""Edge cases of the device path against the oracle: no nodes at all (fluid only), isolated
nodes (no edges), two-node rods (no bending pairs), a 2048^2 grid, the largest FFT side
(4096) on a thin domain, and nodes far outside the domain (the final wrap)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from microcosmos_b200 import baseline_config, scenarios  # noqa: E402
from test_gpu_rows_next import check, gpu_run, oracle_run  # noqa: E402


@pytest.mark.parametrize("F,n", [(0, 0), (5, 1), (6, 2)])
def test_degenerate_topologies(F, n):
    sc = scenarios.make_scenario(64, 48, F, n, seed=F * 10 + n, amp=0.2)
    if F:
        sc.velocity = np.random.default_rng(F).normal(0, 3.0, sc.velocity.shape).astype(np.float32)
    cfg = baseline_config()
    out, = gpu_run([sc], [cfg], 10, act=sc.act_amp is not None)
    ref = oracle_run(sc, cfg, 10, act=sc.act_amp is not None)
    check(out, ref)
    if F == 0:
        assert not np.any(out["steric"])
        m0 = sc.f_grid.astype(np.float64).sum()
        assert abs(out["f_grid"].astype(np.float64).sum() - m0) / m0 < 1e-6


@pytest.mark.parametrize("H,W,F,n,steps", [(2048, 2048, 8, 64, 3), (64, 4096, 4, 40, 2)])
def test_large_and_thin_grids(H, W, F, n, steps):
    sc = scenarios.make_scenario(H, W, F, n, seed=H + W, amp=0.2)
    cfg = baseline_config()
    out, = gpu_run([sc], [cfg], steps)
    check(out, oracle_run(sc, cfg, steps))


def test_positions_far_outside_the_domain_wrap_like_the_reference():
    """Nodes several periods outside the grid: the first step's prediction, deposit and
    stencils wrap them, and the final wrap returns them to [0, W) x [0, H)."""
    sc = scenarios.make_scenario(48, 64, 3, 12, seed=5)
    sc.position = (sc.position + np.array([3 * 64, -2 * 48], np.float32)).astype(np.float32)
    cfg = baseline_config()
    out, = gpu_run([sc], [cfg], 5)
    assert np.all((out["position"] >= 0) & (out["position"] < np.array([64, 48], np.float32)))
    check(out, oracle_run(sc, cfg, 5))
