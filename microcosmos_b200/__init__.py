"""microcosmos_b200: the per-step physics hot path of microcosmos (D2Q9 TRT
lattice-Boltzmann + immersed boundary + PBD Cosserat rods + FFT steric field) as
sm_100a CUDA kernels behind a C ABI, with the reference's ``simulate``/``step`` API.
"""
from .config import (COSSERAT_SCHEME, COSSERAT_SCHEME_NO_FLUID, PBD_SCHEME, PBD_SCHEME_NO_FLUID,
                     ConstraintSolverConfig, baseline_config, pbd_rod_constraint, stable_cosserat_constraint)
from .structs import Edges, Fields, Nodes

__all__ = ["ConstraintSolverConfig", "PBD_SCHEME", "PBD_SCHEME_NO_FLUID", "COSSERAT_SCHEME",
           "COSSERAT_SCHEME_NO_FLUID", "baseline_config", "pbd_rod_constraint", "stable_cosserat_constraint",
           "Nodes", "Edges", "Fields", "simulate", "step", "run", "MicrocosmosEnv"]


def __getattr__(name):
    # the device entry points import torch lazily
    if name in ("simulate", "step", "run"):
        from . import simulate as _s
        return getattr(_s, name)
    if name == "MicrocosmosEnv":
        from .env import MicrocosmosEnv
        return MicrocosmosEnv
    raise AttributeError(name)
