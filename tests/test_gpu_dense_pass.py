"""The dense stream + collide pass against the float32 oracle, bit for bit.

Without nodes the step is the lattice-Boltzmann update alone (solver/fluid.py:268-357 with
F = 0): every operation is an elementwise IEEE float32 operation (sums, products, the
division by the density, the square root of the clamp) in the reference's order, so the
device must reproduce the oracle's populations and u* exactly, on the fast path (force-free
cells with |u| <= vmax / 2, whose terms are shared between opposite directions by exact
identities) and on the clamp path (|u| > vmax / 2, where the velocity clamp is evaluated).
Every dense-pass tile shape must give the same bits."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from microcosmos_b200 import baseline_config, scenarios  # noqa: E402
from microcosmos_b200.engine import DeviceState, Plan  # noqa: E402
from oracle import ref_numpy as O  # noqa: E402


def fluid_only(H, W, seed, u_std):
    """No nodes; populations of a random velocity field, perturbed so that densities differ."""
    sc = scenarios.make_scenario(H, W, 0, 0, seed=seed, u0_std=u_std)
    rng = np.random.default_rng(seed + 1)
    sc.f_grid = (sc.f_grid * rng.uniform(0.9, 1.1, sc.f_grid.shape)).astype(np.float32)
    return sc


def run(sc, steps, shape=None, stages=None):
    st = DeviceState.from_scenario(sc)
    plan = Plan.for_states([st], [baseline_config()], [0.01], lbm_shape=shape, lbm_stages=stages)
    if stages is not None:
        assert plan.lbm_stages() == stages
    plan.rollout([st], steps)
    torch.cuda.synchronize()
    assert plan.read_flags() == [0]
    return st.host()


def oracle(sc, steps):
    s, _ = O.simulate(O.state_from_scenario(sc), O.Config(), 0.01, steps)
    return s


@pytest.mark.parametrize("H,W,u_std,stages", [(96, 160, 0.04, None), (100, 130, 0.09, None), (33, 61, 0.12, None),
                                               (96, 160, 0.04, 3), (37, 1024, 0.09, 2), (70, 92, 0.12, 4)])
def test_dense_pass_is_bit_exact(H, W, u_std, stages):
    sc = fluid_only(H, W, seed=H + W, u_std=u_std)
    out = run(sc, 3, stages=stages)
    ref = oracle(sc, 3)
    # both paths are exercised: some cells above vmax / 2 (clamp path), most below
    rho, ux, uy = O.macroscopic(np.maximum(sc.f_grid, np.float32(O.EPSIL32)))
    speed = np.sqrt(ux * ux + uy * uy)
    assert (speed > 0.1).any() and (speed <= 0.1).any()
    np.testing.assert_array_equal(out["f_grid"], ref.f_grid)
    np.testing.assert_array_equal(out["fluid_velocity"], ref.fluid_velocity)


@pytest.mark.parametrize("vec", [1, 2, 4])
def test_dense_pass_shapes_agree(vec):
    sc = fluid_only(64, 256, seed=5, u_std=0.08)
    base = run(sc, 4, shape=(1, 2))
    for rows in (2, 4, 8, 16, 32):
        got = run(sc, 4, shape=(vec, rows))
        np.testing.assert_array_equal(got["f_grid"], base["f_grid"])
        np.testing.assert_array_equal(got["fluid_velocity"], base["fluid_velocity"])


def test_dense_pass_with_nodes_all_shapes_agree():
    """With IB forcing (the force overlay in some tiles) every tile shape gives the same bits."""
    sc = scenarios.make_scenario(128, 192, 4, 30, seed=9)
    outs = [run(sc, 6, shape=s) for s in ((1, 2), (2, 8), (4, 4), (4, 8), (4, 32))]
    for o in outs[1:]:
        for k in ("f_grid", "position", "velocity", "fluid_velocity"):
            np.testing.assert_array_equal(o[k], outs[0][k])


@pytest.mark.parametrize("H,W", [(64, 256), (5, 1024), (4, 8), (5, 4), (39, 12), (130, 100), (9, 1008)])
def test_staged_dense_pass_matches_tiled(H, W):
    """The staged kernel (row bands copied into shared memory) gives the tiled kernel's bits:
    bands of one row (W = 1024), of many rows (W = 4, 8, 12), a last band shorter than the
    others, lattices shorter than one band (H = 4, 5), and every stage count."""
    sc = fluid_only(H, W, seed=3 * H + W, u_std=0.08)
    base = run(sc, 4, shape=(1, 2))
    for stages in (2, 3, 4, 6):
        got = run(sc, 4, stages=stages)
        np.testing.assert_array_equal(got["f_grid"], base["f_grid"])
        np.testing.assert_array_equal(got["fluid_velocity"], base["fluid_velocity"])


def test_staged_dense_pass_batch_and_nodes():
    """A batch of uneven rollouts with IB nodes: staged and tiled dense passes agree bit for bit."""
    scs = [scenarios.make_scenario(h, w, f, nn, seed=s) for (h, w, f, nn, s) in
           ((128, 192, 4, 30, 1), (96, 64, 2, 20, 2), (200, 256, 3, 40, 3), (48, 1024, 1, 16, 4))]

    def go(**kw):
        sts = [DeviceState.from_scenario(sc) for sc in scs]
        plan = Plan.for_states(sts, [baseline_config()] * len(sts), [0.01] * len(sts), **kw)
        plan.rollout(sts, 5)
        torch.cuda.synchronize()
        assert plan.read_flags() == [0] * len(sts)
        return [st.host() for st in sts]

    base = go(lbm_shape=(1, 4))
    for stages in (2, 3):
        for a, b in zip(go(lbm_stages=stages), base):
            for k in ("f_grid", "position", "velocity", "fluid_velocity"):
                np.testing.assert_array_equal(a[k], b[k])


def test_staged_dense_pass_rejects_unsupported_widths():
    from microcosmos_b200 import _lib
    for H, W in ((64, 66), (16, 1040)):
        sc = fluid_only(H, W, seed=1, u_std=0.01)
        st = DeviceState.from_scenario(sc)
        with pytest.raises(_lib.McError, match="multiples of 4"):
            Plan.for_states([st], [baseline_config()], [0.01], lbm_stages=2)
