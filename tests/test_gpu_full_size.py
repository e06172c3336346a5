"""Size-independent properties at the benchmark configurations' full sizes (the oracle
is too slow there): the plain configuration at scale (1024^2, 256 x 64 nodes) and the
batching configuration (256 uneven rollouts, 25 M cells).  Mass (the sum of the
populations, in float64) is conserved while the EPSIL / density clamps are inactive,
positions stay in the domain, no non-finite flag is raised, and reruns are bitwise equal."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from microcosmos_b200 import baseline_config, scenarios  # noqa: E402
from microcosmos_b200.engine import Actuation, DeviceState, Plan  # noqa: E402


def _run(scs, steps, **plan_kw):
    sts = [DeviceState.from_scenario(s) for s in scs]
    plan = Plan.for_states(sts, [baseline_config()] * len(scs), [0.01] * len(scs), **plan_kw)
    plan.rollout(sts, steps, actuations=[Actuation.from_scenario(s) for s in scs])
    torch.cuda.synchronize()
    return sts, plan.read_flags()


def _mass(f):
    return float(f.double().sum().item())


def test_scale_configuration_properties():
    sc = scenarios.config_scale(seed=0)
    m0 = float(sc.f_grid.astype(np.float64).sum())
    (st,), flags = _run([sc], 20)
    assert flags == [0]
    assert abs(_mass(st.f_grid) - m0) / m0 < 1e-6
    p = st.position.cpu().numpy()
    assert np.all((p >= 0) & (p < np.array([sc.W, sc.H], np.float32)))
    assert torch.isfinite(st.fluid_velocity).all() and torch.isfinite(st.steric).all()
    (st2,), _ = _run([sc], 20)
    assert torch.equal(st.f_grid, st2.f_grid) and torch.equal(st.position, st2.position)


def test_batch_configuration_properties():
    scs = scenarios.config_batch(256, seed=0)
    m0 = [float(s.f_grid.astype(np.float64).sum()) for s in scs]
    sts, flags = _run(scs, 10, lbm_shape=(2, 2), bin_threads=128)
    assert flags == [0] * len(scs)
    for s, st, m in zip(scs, sts, m0):
        assert abs(_mass(st.f_grid) - m) / m < 1e-6
        p = st.position.cpu().numpy()
        assert np.all((p >= 0) & (p < np.array([s.W, s.H], np.float32)))
    sts2, _ = _run(scs, 10, lbm_shape=(1, 4), bin_threads=256)
    for i in (0, 17, 128, 255):
        assert torch.equal(sts[i].f_grid, sts2[i].f_grid) and torch.equal(sts[i].position, sts2[i].position)
