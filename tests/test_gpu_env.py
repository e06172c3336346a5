"""MicrocosmosEnv (src/microcosmos/env.py) on the device against the reference's own
rollout and step of the same structures (golden fixtures env_*.npz): the env defaults
(PBD_SCHEME with the fluid on, dt 0.05) and the fluid-free preset.

Tolerances as for the other golden runs: positions, theta, steric and populations rel-L2
1e-5, velocities 1e-3 (difference quotients of nearly equal positions), u* 1e-4."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from test_env_cpu import build  # noqa: E402
from oracle import ref_numpy as O  # noqa: E402

TOL = 1e-5
VEL_TOL = 1e-3


def rel(a, b):
    a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
    return O.rel_l2(a, np.asarray(b))


@pytest.mark.parametrize("name", ["env_chain_32x40", "env_loop_48x48"])
def test_env_rollout_matches_reference(golden_dir, name):
    z = dict(np.load(f"{golden_dir}/{name}.npz"))
    z["name"] = name
    env, nodes, edges = build(z)
    nts, fts = env.rollout(nodes, edges)
    assert tuple(nts.position.shape) == z["ts_position"].shape
    assert rel(nts.position, z["ts_position"]) < TOL
    assert rel(nts.velocity, z["ts_velocity"]) < VEL_TOL
    assert rel(fts.steric, z["ts_steric"]) < TOL
    assert rel(fts.fluid_velocity, z["ts_fluid_velocity"]) < 1e-4


def test_env_step_of_the_fluid_free_preset_matches_reference(golden_dir):
    name = "env_loop_nofluid_24x24"
    z = dict(np.load(f"{golden_dir}/{name}.npz"))
    z["name"] = name
    env, nodes, edges = build(z)
    n1, e1, f1 = env.step(nodes, edges)
    assert rel(n1.position, z["out_position"]) < TOL
    assert rel(n1.velocity, z["out_velocity"]) < VEL_TOL
    assert rel(e1.theta, z["out_theta"]) < TOL
    assert rel(f1.f_grid, z["out_f_grid"]) < TOL
    # the stored fields are not modified by a step
    np.testing.assert_array_equal(env.fields.f_grid, z["in_f_grid"])
