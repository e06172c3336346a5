"""The CPU oracle against golden vectors produced by executing the reference's own
source (tests/golden/make_golden.py).  Exact where the reference's arithmetic is
elementwise; within 1e-6 relative where the reference reduces with numpy's
pairwise sum or a BLAS dot (IB weight normalisation, momentum tensordot)."""
import numpy as np
import pytest

from oracle import ref_numpy as O


def load(golden_dir, name):
    return np.load(f"{golden_dir}/{name}.npz")


@pytest.mark.parametrize("name", ["utils_16x16", "utils_12x20"])
def test_utils(golden_dir, name):
    z = load(golden_dir, name)
    H, W = int(z["H"]), int(z["W"])
    np.testing.assert_array_equal(O.displacement(H, W, z["x"], z["y"]), z["displacement"])
    np.testing.assert_array_equal(O.periodic_boundary(H, W, z["x"]), z["periodic_boundary"])
    np.testing.assert_array_equal(O.gaussian_filter(z["data"], 1.5), z["gaussian_filter"])


@pytest.mark.parametrize("name", ["steric_20x28", "steric_32x32"])
def test_steric(golden_dir, name):
    z = load(golden_dir, name)
    V, f = O.steric_force(int(z["H"]), int(z["W"]), z["position"], O.Config())
    np.testing.assert_array_equal(V, z["steric"])
    np.testing.assert_array_equal(f, z["force"])


@pytest.mark.parametrize("name", ["pbd_20x28", "pbd_64x64"])
def test_pbd(golden_dir, name):
    z = load(golden_dir, name)
    H, W = int(z["H"]), int(z["W"])
    cfg = O.config_from_npz(z)
    args = (z["in_pairs"], z["in_bending_pairs"], z["in_rest_lengths"], z["in_bending_rest_angles"],
            z["in_bending_stiffness"], cfg)
    p, t = O.pbd_iteration(H, W, z["in_position"], z["in_theta"], *args)
    np.testing.assert_array_equal(p, z["pos_1"])
    np.testing.assert_array_equal(t, z["theta_1"])
    p, t = z["in_position"], z["in_theta"]
    for _ in range(cfg.cycles_per_step):
        p, t = O.pbd_iteration(H, W, p, t, *args)
    np.testing.assert_array_equal(p, z["pos_20"])
    np.testing.assert_array_equal(t, z["theta_20"])


@pytest.mark.parametrize("name", ["cosserat_20x28", "cosserat_64x64"])
def test_stable_cosserat(golden_dir, name):
    """stable_cosserat_constraint (solver/stable_cosserat.py:13-119): one iteration and the
    preset's cycles_per_step iterations, bit for bit."""
    z = load(golden_dir, name)
    H, W = int(z["H"]), int(z["W"])
    cfg = O.config_from_npz(z)
    assert cfg.solver_type == "cosserat" and cfg.dt == 0.05
    args = (z["in_pairs"], z["in_bending_pairs"], z["in_rest_lengths"], z["in_bending_rest_angles"],
            z["in_bending_stiffness"], cfg)
    p, t = O.cosserat_iteration(H, W, z["in_position"], z["in_y"], z["in_theta"], *args)
    np.testing.assert_array_equal(p, z["pos_1"])
    np.testing.assert_array_equal(t, z["theta_1"])
    p, t = z["in_position"], z["in_theta"]
    for _ in range(cfg.cycles_per_step):
        p, t = O.cosserat_iteration(H, W, p, z["in_y"], t, *args)
    np.testing.assert_array_equal(p, z["pos_20"])
    np.testing.assert_array_equal(t, z["theta_20"])


@pytest.mark.parametrize("name", ["ib_24x24_k4", "ib_24x24_k2", "ib_20x28_k4", "ib_16x16_k4_clamp",
                                  "ib_syn_24x24_k4", "ib_syn_20x28_k2", "ib_lat_24x24_on_48x48",
                                  "ib_lat_32x32_on_24x24", "ib_lat_20x28_on_30x42"])
def test_ib_lbm(golden_dir, name):
    z = load(golden_dir, name)
    H, W = int(z["H"]), int(z["W"])
    cfg = O.config_from_npz(z)
    assert (cfg.synthetic_node_width > 0) == name.startswith("ib_syn")
    r = O.ib_lbm(H, W, (H, W), z["in_position"], z["in_velocity"], z["in_f_grid"], cfg,
                 float(z["dt"]), pairs=z["in_pairs"])
    assert O.rel_l2(r.velocity, z["velocity_out"]) < 1e-6
    assert O.rel_l2(r.fluid_velocity, z["fluid_velocity_out"]) < 1e-6
    assert O.rel_l2(r.f_grid, z["f_grid_out"]) < 1e-7


def _state(z):
    return O.State(H=int(z["H"]), W=int(z["W"]), **{k[3:]: z[k] for k in z.files if k.startswith("in_")})


@pytest.mark.parametrize("name", ["sim_24x32", "sim_32x32", "sim_lat_32_on_64", "sim_lat_40_on_30"])
def test_simulate_timeseries(golden_dir, name):
    z = load(golden_dir, name)
    cfg = O.config_from_npz(z)
    _, ts = O.simulate(_state(z), cfg, float(z["dt"]), int(z["steps"]), record=True)
    assert O.rel_l2(ts["position"], z["ts_position"]) < 1e-7
    assert O.rel_l2(ts["velocity"], z["ts_velocity"]) < 1e-6
    assert O.rel_l2(ts["steric"], z["ts_steric"]) < 1e-7
    assert O.rel_l2(ts["fluid_velocity"], z["ts_fluid_velocity"]) < 1e-5


@pytest.mark.parametrize("name", ["sim_24x32", "sim_32x32", "sim_cosserat_nofluid_24x32",
                                  "sim_cosserat_fluid_32x32", "sim_syn_32x32", "sim_lat_32_on_64", "sim_lat_40_on_30"])
def test_actuated_steps(golden_dir, name):
    z = load(golden_dir, name)
    cfg = O.config_from_npz(z)
    act = (z["act_c"], z["act_amp"], z["act_omega"], z["act_phase"])
    s, _ = O.simulate(_state(z), cfg, float(z["dt"]), int(z["steps"]), act=act)
    assert O.rel_l2(s.position, z["act_position"][-1]) < 1e-7
    assert O.rel_l2(s.velocity, z["act_velocity"]) < 1e-6
    assert O.rel_l2(s.theta, z["act_theta"]) < 1e-7
    assert O.rel_l2(s.f_grid, z["act_f_grid"]) < 1e-7
    assert O.rel_l2(s.steric, z["act_steric"]) < 1e-7


def test_reference_loop_scenario(golden_dir):
    """The reference's conftest loop (10 nodes, rest length 3) under PBD_SCHEME defaults."""
    z = load(golden_dir, "loop_32x32")
    cfg = O.config_from_npz(z)
    assert cfg.ibm_kernel_size == 2 and not cfg.enable_steric
    s = O.step(O.step(_state(z), cfg, 0.01), cfg, 0.01)
    np.testing.assert_array_equal(s.position, z["out_position"])
    np.testing.assert_array_equal(s.theta, z["out_theta"])
    assert O.rel_l2(s.f_grid, z["out_f_grid"]) < 1e-7


def test_reference_property_displacement():
    """tests/test_utils.py:25-56 of the reference: wrap gives +2, plain gives +1, wrap(-1, 11) = (9, 1)."""
    d = O.displacement(10, 10, np.array([1.0, 1.0], np.float32), np.array([9.0, 9.0], np.float32))
    np.testing.assert_allclose(d, [2.0, 2.0])
    d = O.displacement(10, 10, np.array([5.0, 5.0], np.float32), np.array([4.0, 4.0], np.float32))
    np.testing.assert_allclose(d, [1.0, 1.0])
    np.testing.assert_allclose(O.periodic_boundary(10, 10, np.array([-1.0, 11.0], np.float32)), [9.0, 1.0])


def test_reference_property_gaussian_filter():
    """tests/test_utils.py:59-68: the filtered delta keeps its peak and is symmetric."""
    d = np.zeros((10, 10), np.float32)
    d[5, 5] = 1.0
    g = O.gaussian_filter(d, 1.0)
    assert np.argmax(g) == 55
    np.testing.assert_allclose(g[5, 4], g[5, 6], rtol=1e-6)
    np.testing.assert_allclose(g[4, 5], g[6, 5], rtol=1e-6)


def test_reference_worm_run(golden_dir):
    """The reference's end-to-end swimmer (its tests/test_worm.py scenario): 200 steps with
    the rest angles rewritten before each step; the reference asserts a centre-of-mass
    displacement in (0.2, 50)."""
    z = load(golden_dir, "worm_50x50")
    from microcosmos_b200 import PBD_SCHEME
    import dataclasses
    cfg = O.Config(**{f.name: getattr(PBD_SCHEME, f.name) for f in dataclasses.fields(O.Config)})
    s = _state(z)
    for t in range(200):
        s = O.step(s, cfg, 0.01, rest_angles=z["rest_angles"][t])
        if t == 49:
            np.testing.assert_array_equal(s.position, z["pos_50"])
    assert O.rel_l2(s.position, z["pos_200"]) < 1e-6
    d = abs(float(z["in_position"][:, 0].mean()) - float(s.position[:, 0].mean()))
    assert 0.2 < d < 50
