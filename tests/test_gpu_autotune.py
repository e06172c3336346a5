"""Dense-pass tile shapes: every shape gives bit-identical results, and the autotuner
returns one of its candidates with a timing for each."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from microcosmos_b200 import autotune, baseline_config, scenarios  # noqa: E402
from microcosmos_b200.engine import Actuation, DeviceState, Plan  # noqa: E402


def _batch():
    sizes = [(64, 128, 3, 20), (96, 64, 2, 30), (128, 128, 5, 16)]
    return [scenarios.make_scenario(H, W, F, n, seed=10 + i) for i, (H, W, F, n) in enumerate(sizes)]


def _run(scs, shape, steps=12):
    sts = [DeviceState.from_scenario(s) for s in scs]
    acts = [Actuation.from_scenario(s) for s in scs]
    cfg = baseline_config()
    plan = Plan.for_states(sts, [cfg] * len(sts), [0.01] * len(sts), lbm_shape=shape)
    assert plan.lbm_shape() == shape
    plan.rollout(sts, steps, actuations=acts)
    torch.cuda.synchronize()
    return [s.host() for s in sts]


def test_every_tile_shape_gives_identical_results():
    scs = _batch()
    ref = _run(scs, (2, 8))
    for shape in [(1, 2), (1, 8), (2, 2), (2, 4), (4, 4), (4, 8)]:
        got = _run(scs, shape)
        for a, b in zip(got, ref):
            for k in ("f_grid", "position", "velocity", "fluid_velocity"):
                assert np.array_equal(a[k], b[k]), (shape, k)


def test_autotuner_picks_a_timed_candidate():
    scs = _batch()
    sts = [DeviceState.from_scenario(s) for s in scs]
    before = [s.f_grid.clone() for s in sts]
    cfg = baseline_config()
    best, timings = autotune.tune(sts, [cfg] * 3, [0.01] * 3, steps=4, warmup=2, use_cache=False)
    assert f"lbm{best['lbm_shape'][0]}x{best['lbm_shape'][1]}" in timings
    assert f"fft{best['fft_values']}" in timings
    assert len(timings) == len(autotune.candidates(sts)) + 3 + len(autotune.BIN_SHAPES) + len(autotune.IB_CLUSTER)
    assert all(t > 0 for t in timings.values())
    assert all(torch.equal(a, b.f_grid) for a, b in zip(before, sts))  # caller's states untouched
    plan = autotune.tuned_plan(sts, [cfg] * 3, [0.01] * 3)
    assert plan.lbm_shape() == best["lbm_shape"] and plan.fft_values() == best["fft_values"]
    assert plan.bin_threads() == best["bin_threads"] and plan.ib_cluster() == best["ib_cluster"]


def test_fft_values_per_thread_agree():
    from oracle import ref_numpy as O
    scs = [scenarios.make_scenario(H, W, 5, 20, seed=30 + i) for i, (H, W) in
           enumerate([(64, 128), (256, 256), (1024, 64), (96, 128)])]
    cfg = baseline_config()
    ref = None
    for e in (4, 8, 16):
        sts = [DeviceState.from_scenario(s) for s in scs]
        for s in sts:
            s.velocity.zero_()
        plan = Plan.for_states(sts, [cfg] * 4, [0.01] * 4, fft_values=e)
        assert plan.fft_values() == e
        plan.rollout(sts, 1)
        torch.cuda.synchronize()
        got = [s.steric.cpu().numpy() for s in sts]
        for sc, g in zip(scs, got):
            want = O.update_steric_potential(sc.H, sc.W, sc.position, cfg.steric_sigma, cfg.steric_scatter_value)
            assert O.rel_l2(g, want) <= 1e-5, (e, sc.H, sc.W)
        if ref is not None:
            assert all(O.rel_l2(a, b) <= 1e-6 for a, b in zip(got, ref))
        ref = got
