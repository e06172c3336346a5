"""The gradient oracle (oracle/adjoint_numpy.py) against central finite differences of
the numpy step in float64, with the Peskin stencil positions held at the unperturbed
trajectory's values (the reference's stop_gradient, solver/fluid.py:239)."""
import dataclasses

import numpy as np
import pytest

from microcosmos_b200 import scenarios
from oracle import adjoint_numpy as A
from oracle import ref_numpy as O


def _state(H, W, F, n, seed, u0_std=2e-2):
    sc = scenarios.make_scenario(H, W, F, n, seed=seed, u0_std=u0_std)
    s = O.state_from_scenario(sc, np.float64)
    rng = np.random.default_rng(seed + 100)
    # a moving, bent start so every term is active
    s.velocity = rng.normal(0, 0.5, s.velocity.shape)
    s.theta = s.theta + rng.normal(0, 0.1, s.theta.shape)
    act = tuple(np.asarray(a, np.float64) for a in (sc.act_c, sc.act_amp, sc.act_omega, sc.act_phase))
    return s, act


def _loss(s, cot):
    return (np.sum(s.position * cot["position"]) + np.sum(s.velocity * cot["velocity"])
            + np.sum(s.theta * cot["theta"]) + np.sum(s.f_grid * cot["f_grid"]))


def _check(cfg, H=16, W=20, F=2, n=7, steps=3, seed=0, h=1e-6, tol=2e-6, ndir=3, lattice=None):
    s0, act = _state(H, W, F, n, seed)
    if lattice is not None:
        # the fluid on its own (h, w) lattice (Fields.grid_shape stays (H, W))
        rng = np.random.default_rng(seed + 200)
        u = rng.normal(0, 2e-2, (2,) + lattice)
        s0.f_grid = O.equilibrium(np.ones(lattice), u[0], u[1])
        s0.fluid_velocity = np.zeros((2,) + lattice)
    dt = 0.01
    sT, tapes = A.rollout(s0, cfg, dt, steps, act)
    ibp = A.ib_positions_of(tapes)
    rng = np.random.default_rng(seed + 7)
    cot = {k: rng.normal(size=getattr(sT, k).shape) for k in ("position", "velocity", "theta", "f_grid")}
    g = A.rollout_vjp(cfg, dt, tapes, A.StepCot(cot["position"], cot["velocity"], cot["theta"], cot["f_grid"]),
                      act)
    names = ["position", "velocity", "theta", "f_grid", "act_c", "act_amp", "act_omega", "act_phase",
             "rest_lengths", "bending_stiffness"]
    for _ in range(ndir):
        d = {k: rng.normal(size=(s0.f_grid.shape if k == "f_grid" else
                                 getattr(s0, k).shape if hasattr(s0, k) else act[0].shape)) for k in names}
        d["f_grid"] *= 1e-2

        def run(eps):
            s = s0.copy()
            for k in ("position", "velocity", "theta", "f_grid", "rest_lengths", "bending_stiffness"):
                setattr(s, k, getattr(s0, k) + eps * d[k])
            a = (act[0] + eps * d["act_c"], act[1] + eps * d["act_amp"], act[2] + eps * d["act_omega"],
                 act[3] + eps * d["act_phase"])
            out, _ = A.rollout(s, cfg, dt, steps, a, ib_positions=ibp)
            return _loss(out, cot)

        fd = (run(h) - run(-h)) / (2 * h)
        ad = sum(np.sum(g[k] * d[k]) for k in names)
        assert abs(fd - ad) <= tol * max(abs(fd), 1e-3), (fd, ad)


def test_vjp_pbd_only():
    _check(O.Config(enable_fluid=False, enable_steric=False))


def test_vjp_pbd_and_steric():
    _check(O.Config(enable_fluid=False))


def test_vjp_pbd_and_fluid():
    _check(O.Config(enable_steric=False))


def test_vjp_full_step():
    _check(O.Config(), steps=4, seed=3)


def test_vjp_full_step_with_active_velocity_clamp():
    # a fast start drives the fluid and correction clamps into their active branch
    _check(dataclasses.replace(O.Config(), max_fluid_velocity=0.02), steps=3, seed=5)


def test_vjp_cosserat_only():
    _check(O.Config(enable_fluid=False, enable_steric=False, solver_type="cosserat", dt=0.05))


def test_vjp_cosserat_full_step():
    # the stable-Cosserat rods inside the full step (steric prediction, IB, lattice)
    _check(O.Config(solver_type="cosserat", dt=0.05, stiffness_stretch=50.0), steps=3, seed=2)


def test_vjp_force_clamp():
    # enable_force_clamp: |F| <= 2 vmax rho, so the clamp needs a low cap and full
    # relaxation to act (here at 2-4 cells per step)
    _check(dataclasses.replace(O.Config(), enable_force_clamp=True, max_fluid_velocity=0.004, ibm_relaxation=1.0),
           steps=3, seed=6)


def test_vjp_fluid_lattice_finer_and_coarser():
    # f_grid on a lattice other than the domain grid: scale = (w / H, h / W) into the
    # lattice, the velocity cap and synthetic offsets by the mean scale
    _check(O.Config(), lattice=(24, 30), steps=3, seed=7)
    _check(O.Config(synthetic_node_width=0.5), lattice=(12, 14), steps=3, seed=8)


def test_vjp_synthetic_ib_pairs():
    # two IB points per node off the chain tangent; their positions are stencil positions
    # (held fixed), the node velocity feeds both and the reaction is their mean
    _check(O.Config(synthetic_node_width=0.5), steps=3, seed=4)


def test_vjp_nonsquare_grid_scale():
    _check(O.Config(), H=12, W=24, steps=2, seed=9)


def test_frozen_ib_positions_change_nothing_at_the_base_point():
    s0, act = _state(16, 16, 2, 6, 1)
    a, tapes = A.rollout(s0, O.Config(), 0.01, 3, act)
    b, _ = A.rollout(s0, O.Config(), 0.01, 3, act, ib_positions=A.ib_positions_of(tapes))
    for k in ("position", "velocity", "theta", "f_grid"):
        assert np.array_equal(getattr(a, k), getattr(b, k))


def test_tape_step_matches_the_oracle_step():
    s0, act = _state(16, 16, 2, 6, 2)
    ra = A.actuation(act, 0, np.float64)
    a, _ = A.step_tape(s0, O.Config(), 0.01, ra)
    b = O.step(s0, O.Config(), 0.01, ra)
    for k in ("position", "velocity", "theta", "f_grid", "steric", "fluid_velocity"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
