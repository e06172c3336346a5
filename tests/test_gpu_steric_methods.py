"""The two forms of the steric filter: FFT (default) and direct convolution with the
filter's periodic kernel kept to radius 24.  The direct form drops the kernel's ~1e-6
tail beyond that radius (the spectral Gaussian is cut off at the Nyquist frequency), so
it is held to DIRECT_TOL against the oracle's FFT filter."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from microcosmos_b200 import baseline_config, scenarios  # noqa: E402
from microcosmos_b200.engine import Actuation, DeviceState, Plan  # noqa: E402
from oracle import ref_numpy as O  # noqa: E402

DIRECT_TOL = 2e-6


def _steric(sc, method):
    st = DeviceState.from_scenario(sc)
    st.velocity.zero_()
    plan = Plan.for_states([st], [baseline_config()], [0.01], steric_method=method)
    assert plan.steric_method() == method
    plan.rollout([st], 1)
    torch.cuda.synchronize()
    return st.steric.cpu().numpy()


@pytest.mark.parametrize("H,W", [(64, 96), (128, 128), (51, 75)])
def test_direct_filter_matches_the_spectral_filter(H, W):
    sc = scenarios.make_scenario(H, W, 6, 24, seed=3)
    cfg = baseline_config()
    ref = O.update_steric_potential(H, W, sc.position, cfg.steric_sigma, cfg.steric_scatter_value)
    direct = _steric(sc, 2)
    assert O.rel_l2(direct, ref) <= DIRECT_TOL
    if H != 51:
        assert O.rel_l2(_steric(sc, 1), ref) <= 1e-5


def test_direct_filter_rollout_against_the_oracle():
    sc = scenarios.make_scenario(64, 64, 4, 20, seed=8)
    cfg = baseline_config()
    st = DeviceState.from_scenario(sc)
    plan = Plan.for_states([st], [cfg], [0.01], steric_method=2)
    plan.rollout([st], 20, actuations=[Actuation.from_scenario(sc)])
    torch.cuda.synchronize()
    s = O.state_from_scenario(sc)
    act = (sc.act_c, sc.act_amp, sc.act_omega, sc.act_phase)
    s, _ = O.simulate(s, O.Config(), 0.01, 20, act=act)
    assert O.rel_l2(st.position.cpu().numpy(), s.position) <= 1e-5
    assert O.rel_l2(st.f_grid.cpu().numpy(), s.f_grid) <= 1e-5
    # the field of the final positions, which carry 20 steps of drift: the parity bar
    assert O.rel_l2(st.steric.cpu().numpy(), s.steric) <= 1e-5


@pytest.mark.parametrize("H,W", [(96, 192), (384, 48), (24, 1536), (12, 12), (192, 128)])
def test_three_times_power_of_two_sides(H, W):
    # sides 3 * 2^a take the twelve-values-per-thread register FFT (radix-4 passes + radix 3)
    sc = scenarios.make_scenario(H, W, 3, 6 if min(H, W) < 24 else 16, seed=7)
    cfg = baseline_config()
    ref = O.update_steric_potential(H, W, sc.position, cfg.steric_sigma, cfg.steric_scatter_value)
    got = _steric(sc, 1)
    assert O.rel_l2(got, ref) <= 1e-5, (H, W, O.rel_l2(got, ref))
