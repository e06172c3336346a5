"""``MicrocosmosEnv``: the reference's thin wrapper around the simulator with default
settings and chain / loop factories (src/microcosmos/env.py), here over this package's
device ``simulate`` / ``step``.

The factories build the same arrays as the reference's: positions from the float32
rounding of ``linspace`` (a centred horizontal chain) or of the circle ``w/2 + r cos a``,
``h/2 + r sin a`` with r = n * spacing / (2 pi); edges and bending pairs from the graph
helpers; theta = atan2 of each edge's min-image vector; rest lengths = spacing; bending
stiffness 0.5; ``color_bend`` = node index mod 3.
"""
from __future__ import annotations

import math

import numpy as np

from .config import PBD_SCHEME, PBD_SCHEME_NO_FLUID, ConstraintSolverConfig
from .gym import topology
from .structs import Edges, Fields, Nodes

DEFAULT_GRID_SHAPE = (64, 64)
DEFAULT_DT = 0.05
DEFAULT_NUM_STEPS = 200
DEFAULT_SPACING = 2.0
DEFAULT_BENDING_STIFFNESS = 0.5

_F32 = np.float32


def make_fields(grid_shape) -> Fields:
    """Zero steric and velocity fields and the populations at rest (graph.py:586-596)."""
    steric, u, f = topology.make_fields(grid_shape)
    return Fields(grid_shape=tuple(grid_shape), steric=steric, fluid_velocity=u, f_grid=f)


class MicrocosmosEnv:
    """Simulator defaults plus structure factories (src/microcosmos/env.py:18-120):
    build a chain or a loop with ``make_chain`` / ``make_loop``, then drive it with
    ``step`` (one step) or ``rollout`` (``num_steps`` steps with per-step recording)."""

    def __init__(self, grid_shape=DEFAULT_GRID_SHAPE, dt: float = DEFAULT_DT, num_steps: int = DEFAULT_NUM_STEPS,
                 solver_config: ConstraintSolverConfig = PBD_SCHEME):
        self.grid_shape = tuple(grid_shape)
        self.dt = dt
        self.num_steps = num_steps
        self.solver_config = solver_config
        self.fields = make_fields(self.grid_shape)

    # --- simulation ---
    def step(self, nodes: Nodes, edges: Edges, fields: Fields | None = None):
        """One physics step; the stored fields when none are given."""
        from .simulate import step
        return step(nodes, edges, fields or self.fields, self.dt, self.solver_config)

    def rollout(self, nodes: Nodes, edges: Edges, fields: Fields | None = None):
        """A full episode: (nodes_timeseries, fields_timeseries)."""
        from .simulate import simulate
        return simulate(nodes, edges, fields or self.fields, self.dt, self.num_steps, self.solver_config)

    # --- structure factories ---
    def make_chain(self, num_nodes: int, spacing: float = DEFAULT_SPACING):
        """A horizontal chain of nodes centred in the grid."""
        h, w = self.grid_shape
        edge_pairs, departure = topology.make_edges(num_nodes, "line")
        bending_pairs, rest_angles = topology.compute_bending_pairs(edge_pairs, departure, num_nodes)
        total = (num_nodes - 1) * spacing
        xs = np.linspace(w / 2 - total / 2, w / 2 + total / 2, num_nodes).astype(_F32)
        positions = np.stack([xs, np.full(num_nodes, h / 2.0, _F32)], axis=1)
        return self._build(positions, edge_pairs, spacing, bending_pairs, rest_angles)

    def make_loop(self, num_nodes: int, spacing: float = DEFAULT_SPACING):
        """A closed circular loop of nodes centred in the grid."""
        h, w = self.grid_shape
        edge_pairs, departure = topology.make_edges(num_nodes, "loop")
        bending_pairs, rest_angles = topology.compute_bending_pairs(edge_pairs, departure, num_nodes)
        radius = num_nodes * spacing / (2 * math.pi)
        angles = np.linspace(0, 2 * math.pi, num_nodes, endpoint=False).astype(_F32)
        # float32 arrays with Python-float scalars stay float32 (JAX's weak types)
        positions = np.stack([w / 2 + radius * np.cos(angles), h / 2 + radius * np.sin(angles)], axis=1).astype(_F32)
        return self._build(positions, edge_pairs, spacing, bending_pairs, rest_angles)

    def _build(self, positions, edge_pairs, spacing, bending_pairs, rest_angles):
        n = positions.shape[0]
        nodes = Nodes(position=positions, velocity=np.zeros_like(positions), color_bend=np.arange(n, dtype=np.int32) % 3,
                      debug_vector=np.zeros_like(positions))
        edges = Edges(pairs=edge_pairs, theta=topology.edge_angles(self.grid_shape, positions, edge_pairs),
                      rest_lengths=np.full(edge_pairs.shape[0], spacing, _F32), bending_pairs=bending_pairs,
                      bending_rest_angles=rest_angles,
                      bending_stiffness=np.full(bending_pairs.shape[0], DEFAULT_BENDING_STIFFNESS, _F32))
        return nodes, edges

    # --- presets ---
    @classmethod
    def no_fluid(cls, grid_shape=DEFAULT_GRID_SHAPE, dt: float = DEFAULT_DT, num_steps: int = DEFAULT_NUM_STEPS):
        return cls(grid_shape=grid_shape, dt=dt, num_steps=num_steps, solver_config=PBD_SCHEME_NO_FLUID)
