"""The reference's end-to-end swimmer test (tests/test_worm.py:15-152 of the reference): a
20-node sine-wave worm on a 50x50 periodic grid under PBD_SCHEME, its bending rest angles
rewritten before every step from a phase advancing 0.1 rad per step, 200 steps through
``step``.  The reference asserts finite state and a centre-of-mass x displacement in
(0.2, grid width).  Here the same run from the fixture the reference's own code produced
(tests/golden/worm_50x50.npz), its frames rendered into a device buffer (the reference
writes a GIF), and the state held to the reference's run after 50 steps and to the
float64 oracle after 200.  Past step ~190 the reference's own float32 trajectory crosses a
stencil discontinuity that its neighbours do not: runs started one ulp away (float32) and
the float64 run end within 2e-6 of each other, the reference's 6e-4 away (centre-of-mass
displacement 0.8631 against 0.8562), so the long run is compared with the float64 oracle."""
import dataclasses

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from microcosmos_b200 import PBD_SCHEME  # noqa: E402
from microcosmos_b200.rendering import render  # noqa: E402
from microcosmos_b200.simulate import step  # noqa: E402
from microcosmos_b200.structs import Fields, Nodes  # noqa: E402
from oracle import ref_numpy as O  # noqa: E402
from test_gpu_parity import containers  # noqa: E402


def wrapped_rel(a, b, H, W):
    """rel-L2 of the min-image position differences (positions wrap at the borders)."""
    d = O.displacement(H, W, np.asarray(a, np.float32), np.asarray(b, np.float32))
    return float(np.sqrt((d.astype(np.float64) ** 2).sum()) / np.sqrt((np.asarray(b, np.float64) ** 2).sum()))


def test_worm_swims_like_the_reference(golden_dir):
    z = np.load(f"{golden_dir}/worm_50x50.npz")
    H, W = int(z["H"]), int(z["W"])
    nodes, edges, fields = containers(z)
    traj, sterics = [], []
    for t in range(200):
        edges = edges.__replace__(bending_rest_angles=z["rest_angles"][t])
        nodes, edges, fields = step(nodes, edges, fields, 0.01, PBD_SCHEME)
        traj.append(nodes.position)
        sterics.append(fields.steric)
        if t == 49:
            assert wrapped_rel(nodes.position.cpu().numpy(), z["pos_50"], H, W) < 1e-5
    pos = nodes.position.cpu().numpy()
    assert np.isfinite(pos).all() and np.isfinite(nodes.velocity.cpu().numpy()).all()
    x0 = float(z["in_position"][:, 0].mean())
    d = abs(x0 - float(pos[:, 0].mean()))
    assert 0.2 < d < W, d
    cfg = O.Config(**{f.name: getattr(PBD_SCHEME, f.name) for f in dataclasses.fields(O.Config)})
    s64 = O.State(H=H, W=W, **{k[3:]: z[k] for k in z.files if k.startswith("in_")}).astype(np.float64)
    for t in range(200):
        s64 = O.step(s64, cfg, 0.01, rest_angles=z["rest_angles"][t].astype(np.float64))
    d64 = abs(x0 - float(s64.position[:, 0].mean()))
    assert abs(d - d64) < 1e-3 * d64, (d, d64)
    assert wrapped_rel(pos, s64.position, H, W) < 1e-4
    assert O.rel_l2(fields.f_grid.cpu().numpy(), s64.f_grid) < 1e-4
    ts = Nodes(position=torch.stack(traj), velocity=None, color_bend=np.arange(20) % 3, debug_vector=None)
    fr = render(ts, Fields(grid_shape=(H, W), steric=torch.stack(sterics), fluid_velocity=None, f_grid=None), 200)
    torch.cuda.synchronize()
    assert tuple(fr.shape) == (200, 200, 200, 3) and fr.dtype == torch.uint8
