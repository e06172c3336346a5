"""The frame renderer (rendering.render, src/microcosmos/rendering.py:20-80): the oracle
against golden frames produced by the reference's render() (CPU), and the device kernels
(mc_render_frames) against both, bit for bit (GPU)."""
import numpy as np
import pytest

from oracle import render_numpy as R

CASES = [("render_32x32", [(64, 1, 0), (16, 1, 0), (32, 1, 1), (48, 0, 0)]),
         ("render_24x40", [(50, 1, 0), (20, 1, 0)])]


def _variants():
    for name, vs in CASES:
        for v in vs:
            yield name, v


@pytest.mark.parametrize("name,variant", list(_variants()))
def test_oracle_matches_reference_frames(golden_dir, name, variant):
    z = np.load(f"{golden_dir}/{name}.npz")
    sz, particles, uniform = variant
    img = R.render(z["position"], z["debug_vector"], z["color_bend"], z["steric"], sz, bool(particles), bool(uniform))
    np.testing.assert_array_equal(img, z[f"frames_{sz}_{particles}{uniform}"])


@pytest.mark.gpu
@pytest.mark.parametrize("name,variant", list(_variants()))
def test_device_frames_match_reference(golden_dir, name, variant):
    torch = pytest.importorskip("torch")
    from microcosmos_b200.rendering import render
    from microcosmos_b200.structs import Fields, Nodes
    z = np.load(f"{golden_dir}/{name}.npz")
    sz, particles, uniform = variant
    T = z["steric"].shape[0]
    nodes = Nodes(position=z["position"], velocity=None, color_bend=z["color_bend"], debug_vector=z["debug_vector"])
    fields = Fields(grid_shape=(int(z["H"]), int(z["W"])), steric=z["steric"], fluid_velocity=None, f_grid=None)
    img = render(nodes, fields, sz, render_particles=bool(particles), uniform_color=bool(uniform))
    torch.cuda.synchronize()
    assert img.dtype == torch.uint8 and img.shape[0] == T
    np.testing.assert_array_equal(img.cpu().numpy(), z[f"frames_{sz}_{particles}{uniform}"])


@pytest.mark.gpu
def test_device_frames_of_a_rollout_match_the_oracle():
    """A recorded 128x96 rollout (steric field on), rendered at 256 and at 50 pixels."""
    torch = pytest.importorskip("torch")
    from microcosmos_b200 import baseline_config, scenarios
    from microcosmos_b200.rendering import render
    from microcosmos_b200.simulate import simulate
    from microcosmos_b200.structs import Edges, Fields, Nodes
    sc = scenarios.make_scenario(128, 96, 6, 30, seed=3)
    nodes = Nodes(position=sc.position, velocity=sc.velocity, color_bend=np.arange(sc.N) % 3,
                  debug_vector=np.zeros_like(sc.position))
    edges = Edges(pairs=sc.pairs, theta=sc.theta, rest_lengths=sc.rest_lengths, bending_pairs=sc.bending_pairs,
                  bending_rest_angles=sc.bending_rest_angles, bending_stiffness=sc.bending_stiffness)
    fields = Fields(grid_shape=(128, 96), steric=sc.steric, fluid_velocity=sc.fluid_velocity, f_grid=sc.f_grid)
    nts, fts = simulate(nodes, edges, fields, 0.01, 8, baseline_config())
    for sz in (256, 50):
        img = render(nts, fts, sz)
        torch.cuda.synchronize()
        want = R.render(nts.position.cpu().numpy(), None, np.arange(sc.N) % 3, fts.steric.cpu().numpy(), sz)
        np.testing.assert_array_equal(img.cpu().numpy(), want)
