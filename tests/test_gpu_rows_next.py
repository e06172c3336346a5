"""Parity of the plugin and IB variants beyond the benchmark configuration, through the C ABI:
the stable-Cosserat rod solver (src/microcosmos/solver/stable_cosserat.py:13-119, selected by
``solver_type="cosserat"``) and synthetic IB node pairs (``synthetic_node_width > 0``,
src/microcosmos/solver/fluid.py:241-263, 371-374).

Tolerances as in test_gpu_parity.py: rel-L2 <= 1e-5 for positions, angles, populations
and the steric field after a few to 20 steps; VEL_TOL = 1e-3 for node velocities (a
difference quotient of nearly equal positions); 1e-4 for u*.  The Cosserat theta pull uses
atan2, whose float32 result may differ from numpy's by an ulp.
"""
import dataclasses

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from microcosmos_b200 import COSSERAT_SCHEME, baseline_config, scenarios  # noqa: E402
from microcosmos_b200.engine import Actuation, DeviceState, Plan  # noqa: E402
from microcosmos_b200.simulate import run, step  # noqa: E402
from oracle import ref_numpy as O  # noqa: E402
from test_gpu_parity import TOL, VEL_TOL, cfg_from, containers, rel  # noqa: E402

GOLDEN_RUNS = ["sim_cosserat_nofluid_24x32", "sim_cosserat_fluid_32x32", "sim_syn_32x32"]


def cosserat_cfg(**over):
    """COSSERAT_SCHEME at dt = 0.01 with the benchmark's fluid/steric overrides and the
    stiffness scaled to the inertia weight (k_s / l^2 = 1 / dt^2 for unit rest lengths)."""
    kw = dict(dt=0.01, stiffness_stretch=10000.0, stiffness_shear=10000.0, viscosity=0.1, ibm_kernel_size=4,
              enable_steric=True)
    kw.update(over)
    return dataclasses.replace(COSSERAT_SCHEME, **kw)


def oracle_cfg(cfg):
    return O.Config(**{f.name: getattr(cfg, f.name) for f in dataclasses.fields(O.Config)})


def gpu_run(scs, cfgs, steps, act=True):
    sts = [DeviceState.from_scenario(s) for s in scs]
    plan = Plan.for_states(sts, cfgs, [0.01] * len(scs))
    plan.rollout(sts, steps, actuations=[Actuation.from_scenario(s) if act else None for s in scs])
    torch.cuda.synchronize()
    assert plan.read_flags() == [0] * len(scs)
    return [st.host() for st in sts]


def oracle_run(sc, cfg, steps, act=True, dtype=np.float32):
    a = (sc.act_c, sc.act_amp, sc.act_omega, sc.act_phase) if act else None
    s, _ = O.simulate(O.state_from_scenario(sc, dtype), oracle_cfg(cfg), 0.01, steps, act=a)
    return s


def check(out, ref, ref64=None, **over):
    """Each output against the float32 oracle within its tolerance; with ``ref64`` (the
    float64 oracle) within max(tolerance, twice the float32 oracle's own distance from
    float64).  Dense, stiff cases (100-node chains on 64x48) amplify rounding: there the
    float32 oracle's u* is ~2e-4 from the float64 value after 20 steps."""
    tols = {"position": TOL, "theta": TOL, "steric": TOL, "f_grid": TOL, "velocity": VEL_TOL,
            "fluid_velocity": 1e-4}
    tols.update(over)
    for k, tol in tols.items():
        if ref64 is not None:
            tol = max(tol, 2.0 * O.rel_l2(getattr(ref, k), getattr(ref64, k)))
        assert rel(out[k], getattr(ref, k)) < tol, (k, rel(out[k], getattr(ref, k)), tol)


@pytest.mark.parametrize("name", GOLDEN_RUNS)
def test_actuated_rollout_matches_reference_golden(golden_dir, name):
    z = np.load(f"{golden_dir}/{name}.npz")
    oc = O.config_from_npz(z)
    cfg = cfg_from(z, base=COSSERAT_SCHEME if oc.solver_type == "cosserat" else baseline_config())
    assert cfg.solver_type == oc.solver_type and cfg.synthetic_node_width == oc.synthetic_node_width
    nodes, edges, fields = containers(z)
    act = (z["act_c"], z["act_amp"], z["act_omega"], z["act_phase"])
    n, e, f = run(nodes, edges, fields, float(z["dt"]), int(z["steps"]), cfg, actuation=act)
    assert rel(n.position, z["act_position"][-1]) < TOL
    assert rel(n.velocity, z["act_velocity"]) < VEL_TOL
    assert rel(e.theta, z["act_theta"]) < TOL
    assert rel(f.f_grid, z["act_f_grid"]) < TOL
    assert rel(f.steric, z["act_steric"]) < TOL
    assert rel(f.fluid_velocity, z["act_fluid_velocity"]) < 1e-4


@pytest.mark.parametrize("H,W,F,n", [(32, 32, 2, 12), (20, 30, 2, 9), (64, 48, 2, 100), (24, 36, 1, 30)])
def test_cosserat_chains_match_oracle(H, W, F, n):
    """Chains of 9 to 100 nodes (one to four nodes per lane of the chain kernel), non-square grids."""
    sc = scenarios.make_scenario(H, W, F, n, seed=H * 5 + W, amp=0.25, period=30.0)
    cfg = cosserat_cfg()
    out, = gpu_run([sc], [cfg], 20)
    check(out, oracle_run(sc, cfg, 20), ref64=oracle_run(sc, cfg, 20, dtype=np.float64))


def test_cosserat_without_fluid_matches_oracle():
    sc = scenarios.make_scenario(40, 40, 3, 14, seed=3, amp=0.3, period=25.0)
    cfg = dataclasses.replace(COSSERAT_SCHEME, enable_fluid=False, damping=0.0)
    out, = gpu_run([sc], [cfg], 20)
    ref = oracle_run(sc, cfg, 20)
    for k in ("position", "theta"):
        assert rel(out[k], getattr(ref, k)) < TOL, k


def test_cosserat_loop_topology_matches_oracle(golden_dir):
    """The reference's conftest loop (not a chain: the one-CTA-per-rod kernel) with the
    Cosserat solver, four steps against the oracle."""
    z = np.load(f"{golden_dir}/loop_32x32.npz")
    nodes, edges, fields = containers(z)
    cfg = cosserat_cfg(stiffness_stretch=900.0, ibm_kernel_size=2, enable_steric=False)
    n, e, f = nodes, edges, fields
    for _ in range(4):
        n, e, f = step(n, e, f, 0.01, cfg)
    s = O.State(H=32, W=32, **{k[3:]: z[k] for k in z.files if k.startswith("in_")})
    for _ in range(4):
        s = O.step(s, oracle_cfg(cfg), 0.01)
    assert rel(n.position, s.position) < TOL
    assert rel(e.theta, s.theta) < TOL
    assert rel(f.f_grid, s.f_grid) < TOL
    assert rel(n.velocity, s.velocity) < VEL_TOL


def test_cosserat_100_steps():
    """The small configuration's shape (128x128, 4 x 32 nodes) with the Cosserat solver,
    100 steps: positions and populations rel-L2 <= 1e-5.  The rod angles are the most
    rounding-sensitive output (the float32 oracle is ~2e-5 from the float64 one after 100
    steps), so they are held to max(1e-5, twice that distance)."""
    sc = scenarios.config_small(seed=0)
    cfg = cosserat_cfg()
    out, = gpu_run([sc], [cfg], 100)
    ref = oracle_run(sc, cfg, 100)
    a = (sc.act_c, sc.act_amp, sc.act_omega, sc.act_phase)
    ref64, _ = O.simulate(O.state_from_scenario(sc, np.float64), oracle_cfg(cfg), 0.01, 100, act=a)
    for k in ("position", "f_grid"):
        assert rel(out[k], getattr(ref, k)) < TOL, k
    e_ref = O.rel_l2(ref.theta, ref64.theta)
    assert rel(out["theta"], ref.theta) <= max(TOL, 2.0 * e_ref), (rel(out["theta"], ref.theta), e_ref)


@pytest.mark.parametrize("H,W,F,n,K,width", [(32, 32, 2, 12, 4, 1.0), (20, 30, 2, 9, 2, 0.5),
                                               (24, 36, 1, 30, 3, 1.5), (40, 40, 2, 10, 6, 1.0)])
def test_synthetic_ib_pairs_match_oracle(H, W, F, n, K, width):
    """Synthetic IB node pairs with 2- to 4-point kernels (the 16-lane stencil kernel) and a
    6-point kernel (the per-point stencil kernel), non-square grids, 20 free-running steps."""
    sc = scenarios.make_scenario(H, W, F, n, seed=H * 3 + W, amp=0.25, period=30.0)
    cfg = baseline_config(ibm_kernel_size=K, synthetic_node_width=width)
    out, = gpu_run([sc], [cfg], 20)
    check(out, oracle_run(sc, cfg, 20), ref64=oracle_run(sc, cfg, 20, dtype=np.float64))


def stepwise_errors(sc, cfg, steps):
    """Every step started from the oracle's own state: the largest per-step rel-L2 of each
    output over ``steps`` steps."""
    oc = oracle_cfg(cfg)
    act = (sc.act_c, sc.act_amp, sc.act_omega, sc.act_phase)
    s = O.state_from_scenario(sc)
    worst = {}
    for t in range(steps):
        st = DeviceState.from_arrays(s.H, s.W, s.position, s.velocity, s.pairs, s.theta, s.rest_lengths,
                                     s.bending_pairs, s.bending_rest_angles, s.bending_stiffness, s.f_grid)
        plan = Plan.for_states([st], [cfg], [0.01])
        a = Actuation(*[torch.as_tensor(x, device="cuda") for x in act], t)
        plan.rollout([st], 1, actuations=[a])
        torch.cuda.synchronize()
        out = st.host()
        s = O.step(s, oc, 0.01, O.actuation(act, t))
        for k in ("position", "theta", "f_grid", "steric", "velocity", "fluid_velocity"):
            worst[k] = max(worst.get(k, 0.0), rel(out[k], getattr(s, k)))
    return worst


def test_synthetic_pairs_dense_stepwise():
    """120 nodes as 240 synthetic IB points on 48x40 (tiles of up to 1,200 contributions).
    The renormalised 4-point stencil is discontinuous where a point crosses a cell edge
    (its edge cells carry weight >= 1/4 of the peak), and this trajectory passes points
    within an ulp of cell edges: the oracle and the reference (run on numpy) part by 2e-5
    in node velocity in one step at step 7, the kernels and the oracle by 5e-3 at step 17
    (measured; 1e-6 before it).  A free-running comparison then measures the crossing,
    not the kernels, so each step is started from the oracle's state and held to the
    single-step tolerances."""
    sc = scenarios.make_scenario(48, 40, 3, 40, seed=48 * 3 + 40, amp=0.25, period=30.0)
    cfg = baseline_config(ibm_kernel_size=4, synthetic_node_width=0.75)
    worst = stepwise_errors(sc, cfg, 20)
    print(worst)
    for k in ("position", "theta", "f_grid", "steric"):
        assert worst[k] < TOL, (k, worst[k])
    assert worst["velocity"] < VEL_TOL
    assert worst["fluid_velocity"] < 1e-4


def test_cosserat_with_synthetic_pairs_matches_oracle():
    sc = scenarios.make_scenario(48, 48, 3, 16, seed=8, amp=0.25, period=30.0)
    cfg = cosserat_cfg(synthetic_node_width=1.0)
    out, = gpu_run([sc], [cfg], 20)
    check(out, oracle_run(sc, cfg, 20), ref64=oracle_run(sc, cfg, 20, dtype=np.float64))


def test_synthetic_pairs_in_one_batch_equal_alone():
    scs = [scenarios.make_scenario(64, 64, 2, 16, seed=4), scenarios.make_scenario(48, 96, 3, 20, seed=5),
           scenarios.make_scenario(32, 32, 1, 12, seed=6)]
    cfgs = [baseline_config(synthetic_node_width=1.0), baseline_config(),
            cosserat_cfg(synthetic_node_width=0.5, ibm_kernel_size=2)]
    both = gpu_run(scs, cfgs, 10)
    for sc, cfg, b in zip(scs, cfgs, both):
        alone, = gpu_run([sc], [cfg], 10)
        for k in alone:
            np.testing.assert_array_equal(b[k], alone[k])


def test_mixed_solvers_in_one_batch_equal_alone():
    """PBD and Cosserat rollouts stepped in one plan give bitwise their results alone."""
    scs = [scenarios.make_scenario(64, 64, 2, 16, seed=1), scenarios.make_scenario(48, 96, 3, 20, seed=2),
           scenarios.make_scenario(32, 32, 1, 12, seed=3)]
    cfgs = [baseline_config(), cosserat_cfg(), cosserat_cfg(enable_fluid=False)]
    both = gpu_run(scs, cfgs, 10)
    for sc, cfg, b in zip(scs, cfgs, both):
        alone, = gpu_run([sc], [cfg], 10)
        for k in alone:
            np.testing.assert_array_equal(b[k], alone[k])


def test_solver_plugin_mismatch_is_rejected():
    from microcosmos_b200 import PBD_SCHEME
    sc = scenarios.make_scenario(32, 32, 1, 8, seed=1)
    bad = dataclasses.replace(PBD_SCHEME, solver_type="cosserat")
    with pytest.raises(ValueError, match="solver_type"):
        gpu_run([sc], [bad], 1)


# ---------------------------------------------------------------- fluid lattice != domain grid
LATTICE_GOLDEN = ["sim_lat_32_on_64", "sim_lat_40_on_30"]


def on_lattice(sc, h, w, seed):
    """The scenario's fluid on an h x w lattice: feq(1, u0) with u0 ~ N(0, 1e-3)."""
    rng = np.random.default_rng(seed)
    ux = rng.normal(0, 1e-3, (h, w)).astype(np.float32)
    uy = rng.normal(0, 1e-3, (h, w)).astype(np.float32)
    sc.f_grid = scenarios.equilibrium(np.ones((h, w), np.float32), ux, uy)
    sc.fluid_velocity = np.zeros((2, h, w), np.float32)
    return sc


@pytest.mark.parametrize("name", LATTICE_GOLDEN)
def test_lattice_rollout_matches_reference_golden(golden_dir, name):
    """f_grid on its own lattice (2x finer, 0.75x coarser than grid_shape): the final state of
    actuated steps and simulate()'s timeseries, whose u* the reference resizes to the domain
    grid (simulate.py:24-29)."""
    from microcosmos_b200.simulate import simulate
    z = np.load(f"{golden_dir}/{name}.npz")
    cfg = cfg_from(z, base=baseline_config())
    nodes, edges, fields = containers(z)
    act = (z["act_c"], z["act_amp"], z["act_omega"], z["act_phase"])
    n, e, f = run(nodes, edges, fields, float(z["dt"]), int(z["steps"]), cfg, actuation=act)
    assert tuple(f.f_grid.shape) == z["act_f_grid"].shape
    assert rel(n.position, z["act_position"][-1]) < TOL
    assert rel(n.velocity, z["act_velocity"]) < VEL_TOL
    assert rel(e.theta, z["act_theta"]) < TOL
    assert rel(f.f_grid, z["act_f_grid"]) < TOL
    assert rel(f.steric, z["act_steric"]) < TOL
    assert rel(f.fluid_velocity, z["act_fluid_velocity"]) < 1e-4
    nts, fts = simulate(nodes, edges, fields, float(z["dt"]), int(z["steps"]), cfg)
    assert tuple(fts.fluid_velocity.shape[1:]) == (2, int(z["H"]), int(z["W"]))
    assert rel(nts.position, z["ts_position"]) < TOL
    assert rel(fts.steric, z["ts_steric"]) < TOL
    assert rel(fts.fluid_velocity, z["ts_fluid_velocity"]) < 1e-4


@pytest.mark.parametrize("H,W,h,w,K", [(32, 32, 48, 48, 4), (24, 40, 36, 60, 2), (48, 40, 24, 20, 4),
                                       (32, 48, 32, 72, 3)])
def test_lattice_rollouts_match_oracle(H, W, h, w, K):
    """Finer, coarser and anisotropic lattices over 20 free-running steps."""
    sc = on_lattice(scenarios.make_scenario(H, W, 2, 12, seed=H + w, amp=0.25, period=30.0), h, w, seed=H * w)
    cfg = baseline_config(ibm_kernel_size=K)
    out, = gpu_run([sc], [cfg], 20)
    check(out, oracle_run(sc, cfg, 20), ref64=oracle_run(sc, cfg, 20, dtype=np.float64))


def test_lattice_recording_matches_the_oracle_resize():
    """Recorded u* on the domain grid: the kernels' linear resize against the oracle's."""
    from microcosmos_b200.engine import Record
    sc = on_lattice(scenarios.make_scenario(40, 40, 2, 12, seed=9), 100, 70, seed=9)
    cfg = baseline_config()
    st = DeviceState.from_scenario(sc)
    plan = Plan.for_states([st], [cfg], [0.01])
    rec = Record.allocate(st, 4, every=1)
    plan.rollout([st], 4, actuations=[Actuation.from_scenario(sc)], records=[rec])
    torch.cuda.synchronize()
    assert tuple(rec.fluid_velocity.shape) == (4, 2, 40, 40)
    want = O.resize_linear(st.fluid_velocity.cpu().numpy(), (2, 40, 40))
    assert rel(rec.fluid_velocity[-1], want) < 1e-6
    ref = oracle_run(sc, cfg, 4)
    assert rel(st.f_grid, ref.f_grid) < TOL


def test_lattices_in_one_batch_equal_alone():
    scs = [on_lattice(scenarios.make_scenario(32, 32, 2, 12, seed=1), 64, 64, seed=1),
           scenarios.make_scenario(48, 40, 2, 16, seed=2),
           on_lattice(scenarios.make_scenario(40, 40, 1, 12, seed=3), 30, 30, seed=3)]
    cfgs = [baseline_config()] * 3
    both = gpu_run(scs, cfgs, 8)
    for sc, cfg, b in zip(scs, cfgs, both):
        alone, = gpu_run([sc], [cfg], 8)
        for k in alone:
            np.testing.assert_array_equal(b[k], alone[k])


def test_lattice_with_synthetic_pairs_and_cosserat_matches_oracle():
    """All three variants at once: the Cosserat solver, synthetic pairs (their offset scaled
    by the mean lattice/domain ratio) and a 1.5x lattice."""
    sc = on_lattice(scenarios.make_scenario(32, 32, 2, 14, seed=21, amp=0.25, period=30.0), 48, 48, seed=21)
    cfg = cosserat_cfg(synthetic_node_width=0.75)
    out, = gpu_run([sc], [cfg], 20)
    check(out, oracle_run(sc, cfg, 20), ref64=oracle_run(sc, cfg, 20, dtype=np.float64))
