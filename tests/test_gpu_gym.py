"""The gym environments on the device (mc_env_act / rollout / mc_env_observe) against the
reference's golden episodes and the gym oracle, and the batched environment against
environments stepped one by one.

Tolerances: observed positions, energies and the reward rel 1e-5 (the physics step's
float32 parity; the centre of mass and the reward are sums whose order differs from numpy's
pairwise one), node velocities VEL_TOL = 1e-3 (difference quotients), positions 1e-5."""
import dataclasses

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from microcosmos_b200.gym import BatchedEnv, RingEnv, TadpoleEnv, make, topology  # noqa: E402
from oracle import gym_numpy as G  # noqa: E402
from oracle import ref_numpy as O  # noqa: E402
from test_gym_cpu import SPECS, make_env  # noqa: E402

TOL = 1e-5
VEL_TOL = 1e-3


def np_(t):
    return t.detach().cpu().numpy()


def assert_obs_close(got, want, N, what):
    """Observation parts: centred positions and node energies to TOL, velocities (difference
    quotients of positions) to VEL_TOL."""
    got = np.asarray(got)
    assert O.rel_l2(got[:2 * N], want[:2 * N]) < TOL, (what, "positions")
    assert O.rel_l2(got[2 * N:4 * N], want[2 * N:4 * N]) < VEL_TOL, (what, "velocities")
    assert O.rel_l2(got[4 * N:], want[4 * N:]) < TOL, (what, "energy")


@pytest.mark.parametrize("name", list(SPECS))
def test_episode_matches_reference_golden(golden_dir, name):
    z = np.load(f"{golden_dir}/{name}.npz")
    env = make_env(name)
    obs0, st = env.reset(0)
    assert O.rel_l2(np_(obs0), z["obs0"]) < 1e-6
    for t in range(3):
        a = {"d_rest_length": z["act_rest"][t], "d_bending_angle": z["act_bend"][t]}
        obs, st, r, done, info = env.step(t, st, a)
        assert_obs_close(np_(obs), z["obs"][t], st.device.N, t)
        assert abs(float(r) - float(z["reward"][t])) <= TOL * max(1.0, abs(float(z["reward"][t]))), t
        assert bool(done) == bool(z["done"][t])
    assert O.rel_l2(np_(st.nodes.position), z["out_position"]) < TOL
    assert O.rel_l2(np_(st.nodes.velocity), z["out_velocity"]) < VEL_TOL
    assert O.rel_l2(np_(st.fields.f_grid), z["out_f_grid"]) < TOL
    np.testing.assert_array_equal(np_(st.edges.bending_rest_angles), z["out_bending_rest_angles"])
    np.testing.assert_array_equal(np_(st.energy_center), z["center"])
    assert int(st.time) == int(z["time"])
    if "fitness" in z.files:
        assert O.rel_l2(np_(env.fitness_per_creature(st)), z["fitness"]) < TOL


def test_step_does_not_modify_its_input_state():
    env = RingEnv(num_nodes=10, grid_shape=(32, 32), energy_amplitude=1.0)
    _, st = env.reset(0)
    before = {k: np_(getattr(st.device, k)).copy() for k in ("position", "velocity", "f_grid", "rest_lengths")}
    a = {"d_rest_length": np.full(env.num_edges, 0.3, np.float32), "d_bending_angle": None}
    _, st2, _, _, _ = env.step(0, st, a)
    for k, v in before.items():
        np.testing.assert_array_equal(np_(getattr(st.device, k)), v)
    assert not np.array_equal(np_(st2.device.position), before["position"])
    np.testing.assert_array_equal(np_(st2.device.rest_lengths), before["rest_lengths"] + np.float32(0.3))


def _oracle_episode(env, actions, steps, noise=None):
    h0 = env._init_state(np.random.default_rng(0))
    H, W = env.grid_shape
    steric, u, f = topology.make_fields(env.grid_shape)
    s = O.State(H=H, W=W, position=h0.position, velocity=np.zeros_like(h0.position), pairs=h0.pairs, theta=h0.theta,
                rest_lengths=h0.rest_lengths, bending_pairs=h0.bending_pairs,
                bending_rest_angles=h0.bending_rest_angles, bending_stiffness=h0.bending_stiffness, f_grid=f,
                steric=steric, fluid_velocity=u)
    cfg = O.Config(**{f_.name: getattr(env.solver_config, f_.name) for f_ in dataclasses.fields(O.Config)})
    center, time = env._sample_energy_center(None), 0
    base_r, base_b = s.rest_lengths.copy(), s.bending_rest_angles.copy()
    seg = env._segments()
    out = []
    for t in range(steps):
        obs, s, r, done, center, time, _ = G.env_step(
            s, cfg, env.dt, base_r, base_b, actions[t], center, time, env.max_steps, env.energy_amplitude,
            env.energy_size, env.energy_walk_std, None if noise is None else noise[t], seg)
        out.append((obs, r, done))
    return out, s, center


def test_tadpole_episode_against_the_oracle():
    """A branched body (one CTA per rod kernel) over 25 steps with random actions."""
    env = TadpoleEnv(head_nodes=10, tail_nodes=8, grid_shape=(64, 64), energy_amplitude=1.0, max_steps=25)
    rng = np.random.default_rng(1)
    acts = [{"d_rest_length": rng.normal(0, 0.2, env.num_edges).astype(np.float32),
             "d_bending_angle": rng.normal(0, 0.3, env.num_bending_pairs).astype(np.float32)} for _ in range(25)]
    ref, s_ref, _ = _oracle_episode(env, acts, 25)
    _, st = env.reset(0)
    for t in range(25):
        obs, st, r, done, _ = env.step(t, st, acts[t])
        assert_obs_close(np_(obs), ref[t][0], env.num_nodes, t)
        assert abs(float(r) - float(ref[t][1])) <= TOL * max(1.0, abs(float(ref[t][1])))
        assert bool(done) == bool(ref[t][2])
    assert O.rel_l2(np_(st.nodes.position), s_ref.position) < TOL


def test_energy_walk_uses_the_step_noise():
    env = make("line", num_nodes=8, grid_shape=(40, 40), energy_amplitude=1.0, energy_walk_std=3.0)
    _, st = env.reset(0)
    c0 = np_(st.energy_center).copy()
    _, st, _, _, info = env.step(7, st, None)
    noise = np.random.default_rng(7).standard_normal(2).astype(np.float32)
    want = np.mod(c0 + noise * np.float32(3.0), np.array([40, 40], np.float32))
    np.testing.assert_array_equal(np_(info["energy_center"]), want)


@pytest.mark.parametrize("name", ["gym_ring", "gym_multi"])
def test_batched_env_equals_environments_stepped_alone(name):
    env = make_env(name)
    env.max_steps = 6
    B = 5
    rng = np.random.default_rng(3)
    acts = [[{"d_rest_length": rng.normal(0, 0.2, env.num_edges).astype(np.float32),
              "d_bending_angle": rng.normal(0, 0.3, env.num_bending_pairs).astype(np.float32)} for _ in range(B)]
            for _ in range(6)]
    benv = BatchedEnv(env, B)
    obs_b, bst = benv.reset([0] * B)
    singles = [env.reset(0) for _ in range(B)]
    for i in range(B):
        assert torch.equal(obs_b[i], singles[i][0])
    states = [s for _, s in singles]
    for t in range(6):
        batch_act = {k: np.stack([acts[t][i][k] for i in range(B)]) for k in ("d_rest_length", "d_bending_angle")}
        obs_b, bst, r_b, d_b, _ = benv.step(None, bst, batch_act)
        for i in range(B):
            o, states[i], r, d, _ = env.step(None, states[i], acts[t][i])
            assert torch.equal(obs_b[i], o), (t, i)
            assert torch.equal(r_b[i], r) and bool(d_b[i]) == bool(d)
    for i in range(B):
        e = bst.env_state(i)
        assert torch.equal(e.device.f_grid, states[i].device.f_grid)
        assert torch.equal(e.device.position, states[i].device.position)


def test_environment_with_the_cosserat_solver_and_synthetic_pairs_matches_the_oracle():
    """The environment's solver_config passes through to the rollout: a ring under the
    stable-Cosserat scheme with synthetic IB pairs, 10 steps with random actions."""
    import dataclasses as dc
    from microcosmos_b200 import COSSERAT_SCHEME
    cfg = dc.replace(COSSERAT_SCHEME, dt=0.01, stiffness_stretch=2500.0, stiffness_shear=2500.0,
                     synthetic_node_width=0.5)
    env = RingEnv(num_nodes=12, grid_shape=(48, 48), energy_amplitude=1.0, solver_config=cfg, max_steps=10)
    rng = np.random.default_rng(4)
    acts = [{"d_rest_length": rng.normal(0, 0.2, env.num_edges).astype(np.float32),
             "d_bending_angle": rng.normal(0, 0.3, env.num_bending_pairs).astype(np.float32)} for _ in range(10)]
    ref, s_ref, _ = _oracle_episode(env, acts, 10)
    _, st = env.reset(0)
    for t in range(10):
        obs, st, r, done, _ = env.step(t, st, acts[t])
        assert_obs_close(np_(obs), ref[t][0], env.num_nodes, t)
        assert bool(done) == bool(ref[t][2])
    assert O.rel_l2(np_(st.nodes.position), s_ref.position) < TOL
