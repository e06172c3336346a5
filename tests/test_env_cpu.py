"""MicrocosmosEnv's structure factories (src/microcosmos/env.py) against the reference's
own output (golden fixtures env_*.npz): positions, edges, angles, rest lengths, bending
pairs and rest angles, stiffness, colours and the initial fields."""
import numpy as np
import pytest

from microcosmos_b200.env import MicrocosmosEnv

CASES = ["env_chain_32x40", "env_loop_48x48", "env_loop_nofluid_24x24"]


def build(z):
    H, W = int(z["H"]), int(z["W"])
    if bool(z["no_fluid"]):
        env = MicrocosmosEnv.no_fluid(grid_shape=(H, W), num_steps=int(z["num_steps"]))
    else:
        env = MicrocosmosEnv(grid_shape=(H, W), num_steps=int(z["num_steps"]))
    kind = "chain" if "chain" in str(z["name"]) else "loop"
    make = env.make_chain if kind == "chain" else env.make_loop
    nodes, edges = make(int(z["num_nodes"]), spacing=float(z["spacing"]))
    return env, nodes, edges


@pytest.mark.parametrize("name", CASES)
def test_factories_match_the_reference(golden_dir, name):
    z = dict(np.load(f"{golden_dir}/{name}.npz"))
    z["name"] = name
    env, nodes, edges = build(z)
    assert np.float32(env.dt) == z["dt"]
    np.testing.assert_array_equal(nodes.position, z["in_position"])
    np.testing.assert_array_equal(nodes.velocity, z["in_velocity"])
    np.testing.assert_array_equal(nodes.color_bend, z["in_color_bend"])
    np.testing.assert_array_equal(edges.pairs, z["in_pairs"])
    np.testing.assert_array_equal(edges.theta, z["in_theta"])
    np.testing.assert_array_equal(edges.rest_lengths, z["in_rest_lengths"])
    np.testing.assert_array_equal(edges.bending_pairs, z["in_bending_pairs"])
    np.testing.assert_array_equal(edges.bending_rest_angles, z["in_bending_rest_angles"])
    np.testing.assert_array_equal(edges.bending_stiffness, z["in_bending_stiffness"])
    np.testing.assert_array_equal(env.fields.steric, z["in_steric"])
    np.testing.assert_array_equal(env.fields.fluid_velocity, z["in_fluid_velocity"])
    np.testing.assert_array_equal(env.fields.f_grid, z["in_f_grid"])
