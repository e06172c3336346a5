"""Oracle parity at the benchmarked configurations' full sizes, and the momentum balance.

* Plain method at scale (1024^2 periodic, 256 filaments x 64 nodes, Poisson-disk centres):
  20 steps on the device against 20 steps of the float32 oracle.
* Batching configuration (256 uneven rollouts in one plan): a seeded sample of 8 rollouts,
  each compared after 10 steps taken inside the 256-rollout plan.
* Bars: positions and edge angles rel-L2 <= 1e-5 after the multi-step rollout.  One step
  from the same state (the device's state after the rollout, stepped once more by the
  device and by the oracle) matches to <= 1e-5 in positions, populations, edge angles and
  the steric field (node velocity: VEL_TOL; u*: 1e-4).
  After the multi-step rollout the populations must be within 1e-5 of the float32 oracle
  or within the float32 oracle's own distance from the float64 oracle, whichever is
  larger: node velocities are (x - x_prev) / dt, so position differences of one ulp become
  ~1e-3 relative velocity differences, the IB force at a node follows its velocity, and in
  rollouts with many nodes per cell the populations of the forced cells take that
  difference (measured: a 192^2 rollout with 1,932 nodes, the densest of the sample, has
  populations 1.04e-5 from the float32 oracle after 10 steps while float32 arithmetic
  itself, the float32 oracle against the float64 one, is 2.3e-5 off).  Every result's
  distance from the float64 oracle is recorded beside the float32 oracle's own.
* Momentum, FP64 accumulation on the host: in the clamp-free regime the fluid's momentum
  change over one step equals the body force summed over the lattice, and the nodes'
  reaction equals the force summed with each cell's stencil coverage as its weight
  (src/microcosmos/solver/fluid.py:331, 362-380: the reaction interpolates the force field
  with the same stencils).  The ratio of the nodes' reaction to the fluid's gain is
  recorded: it is not 1, because the coverage of a cell is not 1.

The node velocity is (x - x_prev) / dt: position differences of a few ulp appear in it
amplified by |x| / |x - x_prev|, so it is held to VEL_TOL as in test_gpu_parity.py.
"""
import dataclasses

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from microcosmos_b200 import baseline_config, scenarios  # noqa: E402
from microcosmos_b200.engine import Actuation, DeviceState, Plan  # noqa: E402
from oracle import ref_numpy as O  # noqa: E402

TOL = 1e-5
VEL_TOL = 1e-3
KEYS = ("position", "f_grid", "theta")


def _acts(sc):
    return (sc.act_c, sc.act_amp, sc.act_omega, sc.act_phase)


def _oracle(sc, steps, dtype):
    s, _ = O.simulate(O.state_from_scenario(sc, dtype), O.Config(), 0.01, steps, act=_acts(sc))
    return s


def _errors(out, r32, r64):
    """rel-L2 of the device result vs the float32 and float64 oracles, and of the float32
    oracle vs the float64 one, per output."""
    e = {}
    for k in KEYS + ("velocity", "steric", "fluid_velocity"):
        e[f"{k}_vs_f32"] = O.rel_l2(out[k], getattr(r32, k))
        e[f"{k}_vs_f64"] = O.rel_l2(out[k], getattr(r64, k))
        e[f"{k}_oracle32_vs_f64"] = O.rel_l2(getattr(r32, k), getattr(r64, k))
    return e


def _check(e):
    for k in ("position", "theta"):
        assert e[f"{k}_vs_f32"] <= TOL, (k, e[f"{k}_vs_f32"])
    assert e["f_grid_vs_f32"] <= max(TOL, e["f_grid_oracle32_vs_f64"]), e["f_grid_vs_f32"]
    assert e["velocity_vs_f32"] <= VEL_TOL, e["velocity_vs_f32"]


def _one_more_step(sc, out, t0, parity_log, name):
    """The device's state `out` (after t0 steps) stepped once by the device and by both
    oracles: positions, populations, edge angles and the steric field within 1e-5 of the
    float32 oracle, node velocity within VEL_TOL, u* within 1e-4 (as in test_gpu_parity)."""
    st = DeviceState.from_arrays(sc.H, sc.W, out["position"], out["velocity"], sc.pairs, out["theta"],
                                 sc.rest_lengths, sc.bending_pairs, out["bending_rest_angles"], sc.bending_stiffness,
                                 out["f_grid"], out["steric"], out["fluid_velocity"])
    plan = Plan.for_states([st], [baseline_config()], [0.01])
    plan.rollout([st], 1, actuations=[Actuation.from_scenario(sc, t0=t0)])
    torch.cuda.synchronize()
    assert plan.read_flags() == [0]
    got = st.host()
    refs = []
    for dtype in (np.float32, np.float64):
        s0 = O.State(H=sc.H, W=sc.W, position=out["position"], velocity=out["velocity"], pairs=sc.pairs,
                     theta=out["theta"], rest_lengths=sc.rest_lengths, bending_pairs=sc.bending_pairs,
                     bending_rest_angles=out["bending_rest_angles"], bending_stiffness=sc.bending_stiffness,
                     f_grid=out["f_grid"], steric=out["steric"], fluid_velocity=out["fluid_velocity"]).astype(dtype)
        r, _ = O.simulate(s0, O.Config(), 0.01, 1, act=_acts(sc), t0=t0)
        refs.append(r)
    e = _errors(got, *refs)
    parity_log(name + "_one_more_step", **e)
    for k in KEYS + ("steric",):
        assert e[f"{k}_vs_f32"] <= TOL, (k, e[f"{k}_vs_f32"])
    assert e["velocity_vs_f32"] <= VEL_TOL, e["velocity_vs_f32"]
    # u* = u + F / (2 rho) carries the node-velocity difference in the forced cells
    assert e["fluid_velocity_vs_f32"] <= 1e-4, e["fluid_velocity_vs_f32"]


def test_scale_configuration_matches_oracle_20_steps(parity_log):
    """1024^2, 256 x 64 nodes, 20 steps (simulate.py:37-100 applied 20 times)."""
    sc = scenarios.config_scale(seed=0)
    steps = 20
    st = DeviceState.from_scenario(sc)
    plan = Plan.for_states([st], [baseline_config()], [0.01])
    plan.rollout([st], steps, actuations=[Actuation.from_scenario(sc)])
    torch.cuda.synchronize()
    assert plan.read_flags() == [0]
    out = st.host()
    e = _errors(out, _oracle(sc, steps, np.float32), _oracle(sc, steps, np.float64))
    parity_log("scale_1024_256x64_20_steps", **e)
    _check(e)
    _one_more_step(sc, out, steps, parity_log, "scale_1024_256x64_20_steps")


def test_batch_configuration_sample_matches_oracle_10_steps(parity_log):
    """8 rollouts drawn (seeded) from the 256-rollout batch, stepped inside the full plan."""
    scs = scenarios.config_batch(256, seed=0)
    steps = 10
    sts = [DeviceState.from_scenario(s) for s in scs]
    plan = Plan.for_states(sts, [baseline_config()] * len(scs), [0.01] * len(scs))
    plan.rollout(sts, steps, actuations=[Actuation.from_scenario(s) for s in scs])
    torch.cuda.synchronize()
    assert plan.read_flags() == [0] * len(scs)
    pick = sorted(np.random.default_rng(2024).choice(len(scs), size=8, replace=False).tolist())
    worst = {}
    for i in pick:
        sc = scs[i]
        out = sts[i].host()
        e = _errors(out, _oracle(sc, steps, np.float32), _oracle(sc, steps, np.float64))
        name = f"batch256_rollout{i}_{sc.H}x{sc.W}_N{sc.position.shape[0]}_10_steps"
        parity_log(name, **e)
        _check(e)
        _one_more_step(sc, out, steps, parity_log, name)
        for k, v in e.items():
            worst[k] = max(worst.get(k, 0.0), v)
    parity_log("batch256_sample8_10_steps_worst", rollouts=pick, **worst)


def _momentum(f):
    f = np.asarray(f, np.float64)
    return np.array([np.tensordot(O.E[:, 0].astype(np.float64), f, axes=(0, 0)).sum(),
                     np.tensordot(O.E[:, 1].astype(np.float64), f, axes=(0, 0)).sum()])


def _one_step(S, sc, cfg):
    st = DeviceState.from_arrays(sc.H, sc.W, S["position"], S["velocity"], sc.pairs, S["theta"], sc.rest_lengths,
                                 sc.bending_pairs, S["bending_rest_angles"], sc.bending_stiffness, S["f_grid"],
                                 S["steric"], S["fluid_velocity"])
    plan = Plan.for_states([st], [cfg], [0.01])
    plan.rollout([st], 1)
    torch.cuda.synchronize()
    assert plan.read_flags() == [0]
    return st.host()


@pytest.mark.parametrize("which", ["small", "scale"])
def test_momentum_balance_fp64(which, parity_log):
    """One step after 10 actuated steps, clamps inactive (checked):
      fluid momentum change == sum over the lattice of F          (<= 1e-6 of sum |F|)
      node reaction summed  == sum over the lattice of cov * F    (<= 1e-6 of sum |F|)
    F is recovered from the step's u* = u + F / (2 rho) (fluid.py:346) and the density and
    velocity of the populations the step started from; the node reaction from the node
    velocity with and without the fluid coupling (everything before the coupling is the
    same, which the test checks bit for bit)."""
    sc = scenarios.config_small(seed=0) if which == "small" else scenarios.config_scale(seed=0)
    cfg = baseline_config()
    st = DeviceState.from_scenario(sc)
    plan = Plan.for_states([st], [cfg], [0.01])
    plan.rollout([st], 10, actuations=[Actuation.from_scenario(sc)])
    torch.cuda.synchronize()
    S = st.host()
    on = _one_step(S, sc, cfg)
    off = _one_step(S, sc, dataclasses.replace(cfg, enable_fluid=False))
    np.testing.assert_array_equal(on["position"], off["position"])

    f0 = S["f_grid"].astype(np.float64)
    f1 = on["f_grid"].astype(np.float64)
    rho, ux, uy = O.macroscopic(f0)
    vmax = cfg.max_fluid_velocity
    # clamp-free regime: EPSIL floors, density floor and the entry velocity clamp inactive
    assert f0.min() > 2 * O.EPSIL32 and f1.min() > 2 * O.EPSIL32
    assert rho.min() > 0.1
    assert np.sqrt(ux * ux + uy * uy).max() < 0.99 * vmax
    F = 2.0 * rho * (on["fluid_velocity"].astype(np.float64) - np.stack([ux, uy]))
    sumF = F.reshape(2, -1).sum(axis=1)
    l1 = float(np.abs(F).sum())
    dP = _momentum(f1) - _momentum(f0)
    mass_rel = abs(f1.sum() - f0.sum()) / f0.sum()

    # node reaction: v_on = v_off - F_I / (m * scale * dt), scale = 1 here
    Fn = (off["velocity"].astype(np.float64) - on["velocity"].astype(np.float64)) * cfg.node_mass * 0.01
    sumFn = Fn.sum(axis=0)
    idx, w = O.peskin_weights(sc.H, sc.W, on["position"].astype(np.float64), cfg.ibm_kernel_size)
    cov = np.zeros(sc.H * sc.W)
    np.add.at(cov, idx.reshape(-1), w.reshape(-1))
    sum_covF = (F.reshape(2, -1) * cov).sum(axis=1)

    e_fluid = float(np.linalg.norm(dP - sumF)) / l1
    e_nodes = float(np.linalg.norm(sumFn - sum_covF)) / l1
    parity_log(f"momentum_{which}", fluid_change_minus_sumF_rel=e_fluid, nodes_minus_sum_covF_rel=e_nodes,
               sumF_x=sumF[0], sumF_y=sumF[1], sum_abs_F=l1, node_reaction_x=sumFn[0], node_reaction_y=sumFn[1],
               reaction_over_injection=float(np.dot(sumFn, sumF) / np.dot(sumF, sumF)), mass_rel=mass_rel)
    assert e_fluid <= 1e-6, e_fluid
    assert e_nodes <= 1e-6, e_nodes
    assert mass_rel <= 1e-6
