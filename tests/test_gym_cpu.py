"""The gym environments' host side and the gym oracle, against golden vectors that ran the
reference's own environments (src/microcosmos/gym/*.py) on numpy: initial layouts and
topologies bit for bit, the oracle's three-step episodes within float32 reduction-order
tolerance."""
import dataclasses

import numpy as np
import pytest

from microcosmos_b200 import PBD_SCHEME
from microcosmos_b200.gym import envs as E
from microcosmos_b200.gym import registry, topology
from oracle import gym_numpy as G
from oracle import ref_numpy as O

SPECS = {
    "gym_line": (E.LineEnv, dict(num_nodes=12, grid_shape=(48, 48), energy_size=6.0)),
    "gym_ring": (E.RingEnv, dict(num_nodes=12, grid_shape=(48, 48), energy_size=6.0)),
    "gym_tadpole": (E.TadpoleEnv, dict(head_nodes=8, tail_nodes=6, grid_shape=(48, 64))),
    "gym_multi": (E.MultiAgentEnv, dict(creatures=(E.LineTopology(num_nodes=10), E.RingTopology(num_nodes=12)),
                                        grid_shape=(64, 64), energy_size=8.0)),
    "gym_line_ring": (E.LineRingEnv, dict(line_nodes=10, ring_nodes=12, centered_line=True, grid_shape=(64, 64),
                                          energy_size=8.0)),
}


def make_env(name):
    cls, kw = SPECS[name]
    return cls(**kw, energy_amplitude=1.0, max_steps=3)


def oracle_cfg():
    return O.Config(**{f.name: getattr(PBD_SCHEME, f.name) for f in dataclasses.fields(O.Config)})


@pytest.mark.parametrize("name", list(SPECS))
def test_initial_state_matches_reference(golden_dir, name):
    z = np.load(f"{golden_dir}/{name}.npz")
    env = make_env(name)
    init = env._init_state(np.random.default_rng(0))
    np.testing.assert_array_equal(init.pairs, z["in_pairs"])
    np.testing.assert_array_equal(init.bending_pairs, z["in_bending_pairs"])
    np.testing.assert_array_equal(init.position, z["in_position"])
    np.testing.assert_array_equal(init.theta, z["in_theta"])
    np.testing.assert_array_equal(init.rest_lengths, z["in_rest_lengths"])
    np.testing.assert_array_equal(init.bending_rest_angles, z["in_bending_rest_angles"])
    np.testing.assert_array_equal(init.bending_stiffness, z["in_bending_stiffness"])
    np.testing.assert_array_equal(env._sample_energy_center(None), z["center0"])
    steric, u, f = topology.make_fields(env.grid_shape)
    np.testing.assert_array_equal(f, z["in_f_grid"])
    np.testing.assert_array_equal(steric, z["in_steric"])
    assert env.action_spec() == {"d_rest_length": (z["in_pairs"].shape[0],),
                                 "d_bending_angle": (z["in_bending_pairs"].shape[0],)}


def golden_state(z):
    return O.State(H=int(z["H"]), W=int(z["W"]), **{k[3:]: z[k] for k in z.files if k.startswith("in_")})


@pytest.mark.parametrize("name", list(SPECS))
def test_oracle_episode_matches_reference(golden_dir, name):
    z = np.load(f"{golden_dir}/{name}.npz")
    s = golden_state(z)
    H, W = s.H, s.W
    obs0 = G.observation(H, W, s.position, s.velocity, z["center0"], float(z["energy_amplitude"]),
                         float(z["energy_size"]))
    assert O.rel_l2(obs0, z["obs0"]) < 1e-6
    segs = z["segments"] if "segments" in z.files else None
    center, time = z["center0"], 0
    base_r, base_b = s.rest_lengths.copy(), s.bending_rest_angles.copy()
    for t in range(3):
        a = {"d_rest_length": z["act_rest"][t], "d_bending_angle": z["act_bend"][t]}
        obs, s, r, done, center, time, fit = G.env_step(s, oracle_cfg(), float(z["dt"]), base_r, base_b, a, center,
                                                        time, int(z["max_steps"]), float(z["energy_amplitude"]),
                                                        float(z["energy_size"]), segments=segs)
        assert O.rel_l2(obs, z["obs"][t]) < 1e-6, t
        assert abs(r - z["reward"][t]) <= 1e-6 * max(1.0, abs(z["reward"][t]))
        assert done == z["done"][t]
    np.testing.assert_array_equal(s.position, z["out_position"])
    assert O.rel_l2(s.f_grid, z["out_f_grid"]) < 1e-7
    np.testing.assert_array_equal(s.bending_rest_angles, z["out_bending_rest_angles"])
    np.testing.assert_array_equal(center, z["center"])
    assert time == int(z["time"])
    if segs is not None:
        assert O.rel_l2(fit, z["fitness"]) < 1e-6


def test_registry_and_reference_constructor_behaviour():
    assert registry.registered_envs() == ["line", "line-random-food", "line-ring", "multi-agent", "ring", "tadpole"]
    assert isinstance(registry.make("ring", num_nodes=8), E.RingEnv)
    with pytest.raises(ValueError, match="unknown env"):
        registry.make("nope")
    # as in the reference, the creature topologies need a node count
    with pytest.raises(TypeError):
        E.MultiAgentEnv()


def test_multi_agent_action_split_and_merge():
    env = make_env("gym_multi")
    a = {"d_rest_length": np.arange(env.num_edges, dtype=np.float32),
         "d_bending_angle": np.arange(env.num_bending_pairs, dtype=np.float32)}
    parts = env.split_action(a)
    assert [p["d_rest_length"].shape[0] for p in parts] == [9, 12]
    back = env.merge_action(parts)
    np.testing.assert_array_equal(back["d_rest_length"], a["d_rest_length"])
    np.testing.assert_array_equal(back["d_bending_angle"], a["d_bending_angle"])


def test_random_food_center_is_inside_the_margins():
    env = E.RandomFoodLineEnv(num_nodes=8, grid_shape=(40, 60))
    for seed in range(20):
        c = env._sample_energy_center(np.random.default_rng(seed))
        m = np.minimum(np.float32(30.0), np.float32(0.45) * np.array([60, 40], np.float32))
        assert np.all(c >= m) and np.all(c <= np.array([60, 40], np.float32) - m)


def test_graph_builder_lists_edges_like_a_digraph():
    b = topology.GraphBuilder()
    head = b.add_loop(4)
    b.add_branch(from_node=head[0], length=3)
    b.add_branch(from_node=head[2], length=2)
    e, d = b.build()
    # node 0's successors (1, then the first branch) come before node 1's edge
    assert e[:2].tolist() == [[0, 1], [0, 4]]
    assert d[1] == np.float32(np.pi / 2) and d[e.tolist().index([2, 7])] == np.float32(np.pi / 2)
