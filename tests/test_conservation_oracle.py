"""Momentum and mass balance of the reference's IB + LBM step, on the float64 oracle.

In exact arithmetic, with the EPSIL / density floors and the entry velocity clamp
inactive, one call of immersed_boundary_interaction (src/microcosmos/solver/fluid.py:202-386)
* conserves mass;
* changes the fluid's momentum by the body force summed over the lattice (TRT collision
  with u* = u + F / (2 rho) and the Guo source, whose first moment is F);
* gives the nodes a reaction equal to the force summed over the lattice with each
  cell's stencil coverage as its weight, since the reaction interpolates F with the
  same normalised stencils (fluid.py:362-368).
The float64 oracle must show all three to round-off.  The reaction equals the fluid's
gain only where every touched cell's coverage is 1; for rods of unit node spacing under
the 4-point kernel the coverage is well below 1 in most touched cells, and the test
records that the reaction is then a fraction of the injection (the reference's comment
at fluid.py:359-361 calls the reaction exactly momentum-conserving)."""
import numpy as np

from microcosmos_b200 import scenarios
from oracle import ref_numpy as O


def _mom(f):
    return np.array([np.tensordot(O.E[:, k].astype(np.float64), f, axes=(0, 0)).sum() for k in (0, 1)])


def test_ib_lbm_balances_float64():
    sc = scenarios.make_scenario(48, 48, 2, 16, seed=4, amp=0.25, period=40.0)
    cfg = O.Config()
    s = O.state_from_scenario(sc, np.float64)
    s, _ = O.simulate(s, cfg, 0.01, 4, act=(sc.act_c, sc.act_amp, sc.act_omega, sc.act_phase))
    # the step up to the coupling, then the coupling itself
    pos = s.position + s.velocity * 0.01
    V, fst = O.steric_force(s.H, s.W, pos, cfg)
    pos = pos + fst * 0.01
    prev = s.position
    th = s.theta
    for _ in range(cfg.cycles_per_step):
        pos, th = O.pbd_iteration(s.H, s.W, pos, th, s.pairs, s.bending_pairs, s.rest_lengths,
                                  s.bending_rest_angles, s.bending_stiffness, cfg)
    vel = (pos - prev) / 0.01
    r = O.ib_lbm(s.H, s.W, (s.H, s.W), pos, vel, s.f_grid, cfg, 0.01)
    f0 = np.maximum(s.f_grid, O.EPSIL32)
    assert f0.min() > 2 * O.EPSIL32 and r.f_grid.min() > 2 * O.EPSIL32
    rho, ux, uy = O.macroscopic(f0)
    assert rho.min() > 0.1 and np.sqrt(ux * ux + uy * uy).max() < 0.99 * cfg.max_fluid_velocity

    F = r.force_field
    sumF = F.reshape(2, -1).sum(axis=1)
    l1 = np.abs(F).sum()
    assert l1 > 0
    assert abs(r.f_grid.sum() - f0.sum()) / f0.sum() < 1e-13
    assert np.linalg.norm(_mom(r.f_grid) - _mom(f0) - sumF) / l1 < 1e-10

    idx, w = O.peskin_weights(s.H, s.W, pos, cfg.ibm_kernel_size)
    cov = np.zeros(s.H * s.W)
    np.add.at(cov, idx.reshape(-1), w.reshape(-1))
    reaction = (vel - r.velocity) * cfg.node_mass * 0.01
    assert np.linalg.norm(reaction.sum(axis=0) - (F.reshape(2, -1) * cov).sum(axis=1)) / l1 < 1e-10
    # the reaction is the coverage-weighted sum, not the plain sum
    touched = cov > 0
    assert cov[touched].mean() < 1.0
    ratio = float(np.dot(reaction.sum(axis=0), sumF) / np.dot(sumF, sumF))
    assert 0.0 < ratio < 1.0
