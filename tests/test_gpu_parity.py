"""Parity of the CUDA path (through the C ABI) with the reference's golden vectors and
the CPU oracle.

Tolerances (float32 everywhere):
  * golden vectors / oracle after <= 20 steps: rel-L2 <= 1e-5 (the kernels round every
    elementwise op like the reference; remaining differences are the transcendental
    implementations, the FFT, and the reference's own summation order);
  * the small benchmark configuration (128^2, 4 x 32 nodes): rel-L2 <= 1e-5 after 100 steps,
    <= 1e-3 after 1000 steps (chaotic growth of ulp-level differences);
  * node velocity = (x - x_prev) / dt is a difference of nearly equal positions (|x| ~ grid
    size, |x - x_prev| ~ 1e-2), so position differences of a few ulp appear amplified by
    |x| / |x - x_prev| ~ 1e3 in it: VEL_TOL = 1e-3.
"""
import dataclasses

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from microcosmos_b200 import PBD_SCHEME, baseline_config, scenarios  # noqa: E402
from microcosmos_b200.engine import Actuation, DeviceState, Plan, Record  # noqa: E402
from microcosmos_b200.simulate import run, simulate, step  # noqa: E402
from microcosmos_b200.structs import Edges, Fields, Nodes  # noqa: E402
from oracle import ref_numpy as O  # noqa: E402

TOL = 1e-5
VEL_TOL = 1e-3


def rel(a, b):
    if isinstance(a, torch.Tensor):
        a = a.detach().cpu().numpy()
    return O.rel_l2(a, b)


def containers(z, prefix="in_"):
    H, W = int(z["H"]), int(z["W"])
    N = z[prefix + "position"].shape[0]
    nodes = Nodes(position=z[prefix + "position"], velocity=z[prefix + "velocity"],
                  color_bend=np.zeros(N, np.float32), debug_vector=np.zeros((N, 2), np.float32))
    edges = Edges(pairs=z[prefix + "pairs"], theta=z[prefix + "theta"], rest_lengths=z[prefix + "rest_lengths"],
                  bending_pairs=z[prefix + "bending_pairs"], bending_rest_angles=z[prefix + "bending_rest_angles"],
                  bending_stiffness=z[prefix + "bending_stiffness"])
    fields = Fields(grid_shape=(H, W), steric=z[prefix + "steric"], fluid_velocity=z[prefix + "fluid_velocity"],
                    f_grid=z[prefix + "f_grid"])
    return nodes, edges, fields


def cfg_from(z, base=PBD_SCHEME):
    oc = O.config_from_npz(z)
    return dataclasses.replace(base, **{f.name: getattr(oc, f.name) for f in dataclasses.fields(O.Config)})


@pytest.mark.parametrize("name", ["sim_24x32", "sim_32x32"])
def test_simulate_timeseries_matches_reference_golden(golden_dir, name):
    z = np.load(f"{golden_dir}/{name}.npz")
    nodes, edges, fields = containers(z)
    nts, fts = simulate(nodes, edges, fields, float(z["dt"]), int(z["steps"]), cfg_from(z))
    assert rel(nts.position, z["ts_position"]) < TOL
    assert rel(nts.velocity, z["ts_velocity"]) < VEL_TOL
    assert rel(fts.steric, z["ts_steric"]) < TOL
    assert rel(fts.fluid_velocity, z["ts_fluid_velocity"]) < 1e-4
    assert fts.f_grid is None


@pytest.mark.parametrize("name", ["sim_24x32", "sim_32x32"])
def test_actuated_rollout_matches_reference_golden(golden_dir, name):
    z = np.load(f"{golden_dir}/{name}.npz")
    nodes, edges, fields = containers(z)
    act = (z["act_c"], z["act_amp"], z["act_omega"], z["act_phase"])
    n, e, f = run(nodes, edges, fields, float(z["dt"]), int(z["steps"]), cfg_from(z), actuation=act)
    assert rel(n.position, z["act_position"][-1]) < TOL
    assert rel(n.velocity, z["act_velocity"]) < VEL_TOL
    assert rel(e.theta, z["act_theta"]) < TOL
    assert rel(f.f_grid, z["act_f_grid"]) < TOL
    assert rel(f.steric, z["act_steric"]) < TOL
    assert rel(f.fluid_velocity, z["act_fluid_velocity"]) < 1e-4


def test_reference_loop_two_steps(golden_dir):
    """The reference's conftest loop under PBD_SCHEME defaults (2-point kernel, no steric)."""
    z = np.load(f"{golden_dir}/loop_32x32.npz")
    nodes, edges, fields = containers(z)
    cfg = cfg_from(z)
    n, e, f = step(nodes, edges, fields, 0.01, cfg)
    n, e, f = step(n, e, f, 0.01, cfg)
    assert rel(n.position, z["out_position"]) < TOL
    assert rel(e.theta, z["out_theta"]) < TOL
    assert rel(f.f_grid, z["out_f_grid"]) < TOL
    assert rel(n.velocity, z["out_velocity"]) < VEL_TOL


def _oracle_run(sc, steps, cfg=O.Config(), act=True):
    a = (sc.act_c, sc.act_amp, sc.act_omega, sc.act_phase) if act and sc.act_amp is not None else None
    s, _ = O.simulate(O.state_from_scenario(sc), cfg, 0.01, steps, act=a)
    return s


def _gpu_run(sc, steps, cfg=None, use_graph=True, act=True):
    cfg = cfg or baseline_config()
    st = DeviceState.from_scenario(sc)
    plan = Plan.for_states([st], [cfg], [0.01])
    plan.rollout([st], steps, actuations=[Actuation.from_scenario(sc) if act else None], use_graph=use_graph)
    torch.cuda.synchronize()
    assert plan.read_flags() == [0]
    return st.host()


@pytest.mark.parametrize("H,W,F,n", [(32, 32, 2, 12), (20, 30, 2, 9), (48, 40, 3, 16), (24, 36, 1, 30)])
def test_oracle_parity_small_grids(H, W, F, n):
    """Non-square grids, widths that are not multiples of 4 (scalar LBM path), wrap-around."""
    sc = scenarios.make_scenario(H, W, F, n, seed=H * 7 + W, amp=0.25, period=30.0)
    out = _gpu_run(sc, 20)
    ref = _oracle_run(sc, 20)
    for k in ("position", "theta", "f_grid", "steric"):
        assert rel(out[k], getattr(ref, k)) < TOL, k
    assert rel(out["velocity"], ref.velocity) < VEL_TOL
    assert rel(out["fluid_velocity"], ref.fluid_velocity) < 1e-4


def _errors_vs_oracles(out, sc, steps):
    """rel-L2 of every output vs the float32 and the float64 oracle, and of the float32
    oracle vs the float64 one (the distance float32 arithmetic alone accounts for)."""
    r32 = _oracle_run(sc, steps)
    s64, _ = O.simulate(O.state_from_scenario(sc, np.float64), O.Config(), 0.01, steps,
                        act=(sc.act_c, sc.act_amp, sc.act_omega, sc.act_phase))
    e = {}
    for k in ("position", "f_grid", "theta", "velocity", "steric", "fluid_velocity"):
        e[f"{k}_vs_f32"] = rel(out[k], getattr(r32, k))
        e[f"{k}_vs_f64"] = rel(out[k], getattr(s64, k))
        e[f"{k}_oracle32_vs_f64"] = rel(getattr(r32, k), getattr(s64, k))
    return e


def test_small_config_100_steps(parity_log):
    """Plain method, small: 128x128, 4 filaments x 32 nodes, 100 steps: rel-L2 <= 1e-5."""
    sc = scenarios.config_small(seed=0)
    out = _gpu_run(sc, 100)
    e = _errors_vs_oracles(out, sc, 100)
    parity_log("small_128_4x32_100_steps", **e)
    for k in ("position", "f_grid", "theta"):
        assert e[f"{k}_vs_f32"] < TOL, k
    assert e["velocity_vs_f32"] < VEL_TOL
    # the steric field is a sigma = 1.5 Gaussian sum around positions ~1e2: a position
    # difference of rel-L2 1e-6 (~1e-4 absolute) moves it by ~1e-4 relative
    assert e["steric_vs_f32"] < 1e-3


def test_small_config_1000_steps(parity_log):
    """Same configuration, 1000 steps: rel-L2 <= 1e-3 (positions and populations)."""
    sc = scenarios.config_small(seed=0)
    out = _gpu_run(sc, 1000)
    e = _errors_vs_oracles(out, sc, 1000)
    parity_log("small_128_4x32_1000_steps", **e)
    for k in ("position", "f_grid"):
        assert e[f"{k}_vs_f32"] < 1e-3, k


def test_graph_and_direct_launches_agree():
    sc = scenarios.make_scenario(64, 64, 3, 20, seed=11)
    a = _gpu_run(sc, 9, use_graph=True)
    b = _gpu_run(sc, 9, use_graph=False)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])


def test_deterministic_reruns():
    sc = scenarios.make_scenario(96, 64, 6, 24, seed=5)
    a = _gpu_run(sc, 15)
    b = _gpu_run(sc, 15)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])


def test_batch_equals_single_rollouts():
    """Rollouts of different sizes stepped together give bitwise the results they give alone."""
    scs = [scenarios.make_scenario(64, 64, 2, 16, seed=1), scenarios.make_scenario(48, 96, 3, 20, seed=2),
           scenarios.make_scenario(128, 128, 1, 40, seed=3)]
    cfg = baseline_config()
    sts = [DeviceState.from_scenario(s) for s in scs]
    plan = Plan.for_states(sts, [cfg] * 3, [0.01] * 3)
    plan.rollout(sts, 12, actuations=[Actuation.from_scenario(s) for s in scs])
    torch.cuda.synchronize()
    for sc, st in zip(scs, sts):
        alone = _gpu_run(sc, 12)
        both = st.host()
        for k in alone:
            np.testing.assert_array_equal(both[k], alone[k])


def test_batch_with_different_ib_rounds_equals_single_rollouts():
    """A plan whose rollouts run different numbers of multi-direct forcing rounds computes the
    body force in its own pass after the rounds; a rollout alone computes it in its last
    round.  Both give the same bits."""
    scs = [scenarios.make_scenario(64, 64, 2, 16, seed=11), scenarios.make_scenario(48, 80, 3, 12, seed=12),
           scenarios.make_scenario(64, 48, 2, 20, seed=13)]
    cfgs = [baseline_config(ibm_iterations=5), baseline_config(ibm_iterations=2),
            baseline_config(ibm_iterations=1)]
    sts = [DeviceState.from_scenario(s) for s in scs]
    acts = [Actuation.from_scenario(s) for s in scs]
    plan = Plan.for_states(sts, cfgs, [0.01] * 3)
    plan.rollout(sts, 10, actuations=acts)
    torch.cuda.synchronize()
    for sc, cfg, st, act in zip(scs, cfgs, sts, acts):
        one = DeviceState.from_scenario(sc)
        p1 = Plan.for_states([one], [cfg], [0.01])
        p1.rollout([one], 10, actuations=[act])
        torch.cuda.synchronize()
        alone, both = one.host(), st.host()
        for k in alone:
            np.testing.assert_array_equal(both[k], alone[k])


def test_recording_matches_final_state():
    sc = scenarios.make_scenario(32, 48, 2, 10, seed=4)
    cfg = baseline_config()
    st = DeviceState.from_scenario(sc)
    plan = Plan.for_states([st], [cfg], [0.01])
    rec = Record.allocate(st, 8, every=2)
    plan.rollout([st], 8, actuations=[Actuation.from_scenario(sc)], records=[rec])
    torch.cuda.synchronize()
    assert rec.position.shape[0] == 4
    np.testing.assert_array_equal(rec.position[-1].cpu().numpy(), st.position.cpu().numpy())
    np.testing.assert_array_equal(rec.steric[-1].cpu().numpy(), st.steric.cpu().numpy())
    np.testing.assert_array_equal(rec.fluid_velocity[-1].cpu().numpy(), st.fluid_velocity.cpu().numpy())
    ref4 = _oracle_run(sc, 4)
    assert rel(rec.position[1], ref4.position) < TOL


def test_mass_conservation_fp64():
    """Sum of populations is conserved while the EPSIL / density clamps are inactive."""
    sc = scenarios.make_scenario(64, 64, 3, 16, seed=9)
    m0 = sc.f_grid.astype(np.float64).sum()
    out = _gpu_run(sc, 50)
    m1 = out["f_grid"].astype(np.float64).sum()
    assert abs(m1 - m0) / m0 < 1e-6


def test_non_finite_state_is_flagged():
    sc = scenarios.make_scenario(32, 32, 1, 10, seed=2)
    sc.velocity[3, 0] = np.inf
    cfg = baseline_config()
    st = DeviceState.from_scenario(sc)
    plan = Plan.for_states([st], [cfg], [0.01])
    plan.rollout([st], 2, actuations=[Actuation.from_scenario(sc)])
    torch.cuda.synchronize()
    assert plan.read_flags(clear=True) == [1]
    assert plan.read_flags() == [0]


def test_pipelined_and_sequential_schedules_agree():
    """Without field recording the next step's node pipeline overlaps the dense pass on a
    second stream; with it the step runs sequentially.  Both give the same bits."""
    sc = scenarios.make_scenario(96, 128, 5, 30, seed=21)
    cfg = baseline_config()
    outs = []
    for record in (False, True):
        st = DeviceState.from_scenario(sc)
        plan = Plan.for_states([st], [cfg], [0.01])
        rec = Record.allocate(st, 11, every=1) if record else None
        plan.rollout([st], 11, actuations=[Actuation.from_scenario(sc)], records=[rec])
        torch.cuda.synchronize()
        outs.append(st.host())
    for k in outs[0]:
        np.testing.assert_array_equal(outs[0][k], outs[1][k])


def test_zero_steps_leave_state_unchanged():
    sc = scenarios.make_scenario(32, 32, 2, 10, seed=8)
    st = DeviceState.from_scenario(sc)
    plan = Plan.for_states([st], [baseline_config()], [0.01])
    plan.rollout([st], 0, actuations=[Actuation.from_scenario(sc)])
    torch.cuda.synchronize()
    out = st.host()
    np.testing.assert_array_equal(out["position"], sc.position)
    np.testing.assert_array_equal(out["f_grid"], sc.f_grid)


def test_fused_and_separate_ib_kernels_agree():
    """The cooperative fused IB kernel and the separate interpolate/spread launches give the
    same bits, for a single rollout and a batch."""
    scs = [scenarios.make_scenario(128, 128, 6, 40, seed=31), scenarios.make_scenario(64, 96, 2, 20, seed=32)]
    cfg = baseline_config()
    results = []
    for fused in (True, False):
        sts = [DeviceState.from_scenario(s) for s in scs]
        plan = Plan.for_states(sts, [cfg] * 2, [0.01] * 2)
        plan.set_fused_ib(fused)
        assert plan.uses_fused_ib() == fused
        plan.rollout(sts, 13, actuations=[Actuation.from_scenario(s) for s in scs])
        torch.cuda.synchronize()
        assert plan.read_flags() == [0, 0]
        results.append([st.host() for st in sts])
    for a, b in zip(*results):
        for k in a:
            np.testing.assert_array_equal(a[k], b[k])


def test_plans_of_different_sizes_coexist():
    """Binding a plan with a small grid must not break a plan with a larger one."""
    big = scenarios.make_scenario(256, 256, 2, 20, seed=51)
    small = scenarios.make_scenario(32, 32, 1, 10, seed=52)
    cfg = baseline_config()
    st_big = DeviceState.from_scenario(big)
    plan_big = Plan.for_states([st_big], [cfg], [0.01])
    st_small = DeviceState.from_scenario(small)
    Plan.for_states([st_small], [cfg], [0.01]).rollout([st_small], 2)
    plan_big.rollout([st_big], 3, actuations=[Actuation.from_scenario(big)])
    torch.cuda.synchronize()
    ref = _oracle_run(big, 3)
    assert rel(st_big.position, ref.position) < TOL


@pytest.mark.parametrize("ctas", [1, 3, 8, 16])
def test_cluster_and_separate_ib_kernels_agree(ctas):
    """The IB iterations in one thread-block cluster per rollout (hardware cluster barriers
    between the phases) give the same bits as the separate launches, for a batch of rollouts
    of different sizes (one without nodes) and for a single 1024^2 rollout."""
    scs = [scenarios.make_scenario(128, 128, 6, 40, seed=31), scenarios.make_scenario(64, 96, 2, 20, seed=32),
           scenarios.make_scenario(48, 48, 0, 0, seed=33), scenarios.make_scenario(256, 192, 12, 64, seed=34)]
    cfg = baseline_config()
    results = []
    for cl in (0, ctas):
        sts = [DeviceState.from_scenario(s) for s in scs]
        plan = Plan.for_states(sts, [cfg] * len(scs), [0.01] * len(scs), ib_cluster=cl)
        assert plan.ib_cluster() == cl
        plan.rollout(sts, 13, actuations=[Actuation.from_scenario(s) for s in scs])
        torch.cuda.synchronize()
        assert plan.read_flags() == [0] * len(scs)
        results.append([st.host() for st in sts])
    for a, b in zip(*results):
        for k in a:
            np.testing.assert_array_equal(a[k], b[k])
    if ctas == 16:
        sc = scenarios.config_scale(seed=1)
        outs = []
        for cl in (0, 16):
            st = DeviceState.from_scenario(sc)
            plan = Plan.for_states([st], [cfg], [0.01], ib_cluster=cl)
            plan.rollout([st], 4, actuations=[Actuation.from_scenario(sc)])
            torch.cuda.synchronize()
            outs.append(st.host())
        for k in outs[0]:
            np.testing.assert_array_equal(outs[0][k], outs[1][k])
