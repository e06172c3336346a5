"""Solver configuration, mirroring ``ConstraintSolverConfig`` and its presets
(src/microcosmos/solver/config.py:9-171).

``bending_constraint`` keeps the reference's plugin slot.  The device implements both of
the reference's rod constraints: the PBD rod constraint (src/microcosmos/solver/pbd.py:14-91)
and the stable-Cosserat projective-dynamics constraint
(src/microcosmos/solver/stable_cosserat.py:13-119); any other callable raises
``NotImplementedError`` when a plan is built.
"""
from __future__ import annotations

import dataclasses
from typing import Callable


def pbd_rod_constraint(*args, **kwargs):
    """Marker for the PBD rod constraint plugin.  It runs on the device inside
    ``simulate``/``step``; it is not callable on host arrays."""
    raise NotImplementedError("pbd_rod_constraint runs on the device inside simulate()/step()")


def stable_cosserat_constraint(*args, **kwargs):
    """Marker for the stable-Cosserat plugin (src/microcosmos/solver/stable_cosserat.py:13).
    It runs on the device inside ``simulate``/``step`` (with ``solver_type="cosserat"``);
    it is not callable on host arrays."""
    raise NotImplementedError("stable_cosserat_constraint runs on the device inside simulate()/step()")


@dataclasses.dataclass(frozen=True)
class ConstraintSolverConfig:
    bending_constraint: Callable
    name: str
    cycles_per_constraint: int
    cycles_per_step: int
    stiffness_stretch: float
    stiffness_shear: float
    damping: float
    enable_fluid: bool
    viscosity: float
    max_fluid_velocity: float
    solver_type: str = "pbd"
    dt: float = 0.05
    ibm_iterations: int = 5
    synthetic_node_width: float = 0.0
    ibm_kernel_size: int = 3
    ibm_relaxation: float = 0.3
    node_mass: float = 1.0
    lambda_trt: float = 0.25
    enable_force_clamp: bool = False
    enable_steric: bool = False
    steric_strength: float = 1.0
    steric_sigma: float = 1.5
    steric_neighbor_skip: int = 5
    steric_scatter_value: float = 1.0


PBD_SCHEME = ConstraintSolverConfig(
    bending_constraint=pbd_rod_constraint, name="cosserat rods", cycles_per_constraint=2,
    cycles_per_step=20, stiffness_stretch=0.6, stiffness_shear=1.0, damping=1.0, enable_fluid=True,
    viscosity=0.01, max_fluid_velocity=0.2, synthetic_node_width=0.0, ibm_iterations=5,
    ibm_kernel_size=2)

PBD_SCHEME_NO_FLUID = ConstraintSolverConfig(
    bending_constraint=pbd_rod_constraint, name="cosserat rods (no fluid)", cycles_per_constraint=2,
    cycles_per_step=10, stiffness_stretch=0.7, stiffness_shear=0.7, damping=0.0, enable_fluid=False,
    viscosity=0.1, max_fluid_velocity=0.1, enable_steric=False)

COSSERAT_SCHEME_NO_FLUID = ConstraintSolverConfig(
    bending_constraint=stable_cosserat_constraint, solver_type="cosserat",
    name="stable cosserat (no fluid)", cycles_per_constraint=2, cycles_per_step=20,
    stiffness_stretch=50.0, stiffness_shear=50.0, damping=0.0, dt=0.05, enable_fluid=False,
    viscosity=0.1, max_fluid_velocity=0.1, enable_steric=False, steric_strength=100.0)

COSSERAT_SCHEME = ConstraintSolverConfig(
    bending_constraint=stable_cosserat_constraint, solver_type="cosserat",
    name="stable cosserat with fluid", cycles_per_constraint=2, cycles_per_step=20,
    stiffness_stretch=50.0, stiffness_shear=50.0, damping=1.0, dt=0.05, enable_fluid=True,
    viscosity=0.01, max_fluid_velocity=0.2, synthetic_node_width=0.0, ibm_iterations=5,
    ibm_kernel_size=2)


def baseline_config(**over) -> ConstraintSolverConfig:
    """PBD_SCHEME with the benchmark overrides: viscosity 0.1 (tau+ = 0.8), Lambda = 1/4,
    4-point IB kernel, steric field on, stretch 1.0 and shear ("twist" in 2-D) 0.1."""
    kw = dict(viscosity=0.1, lambda_trt=0.25, ibm_kernel_size=4, enable_steric=True,
              stiffness_stretch=1.0, stiffness_shear=0.1)
    kw.update(over)
    return dataclasses.replace(PBD_SCHEME, **kw)
