"""The reference's predefined environments (src/microcosmos/gym/line.py, ring.py,
random_food.py, tadpole.py, multi_agent.py, line_ring.py): their topologies and initial
layouts, built on the host once per reset, then stepped on the device by
``Environment``.  Layout arithmetic is float32 with the reference's operation order
(linspace evaluated in float64 and rounded once, as numpy does)."""
from __future__ import annotations

import dataclasses
import math
from typing import Sequence

import numpy as np

from . import topology
from .base import Environment, HostInit

_F = np.float32


def _linspace(a, b, n, endpoint=True):
    return np.linspace(a, b, n, endpoint=endpoint).astype(_F)


def _init(grid_shape, positions, pairs, rest_lengths, bpairs, rest_angles, stiffness):
    theta = topology.edge_angles(grid_shape, positions, pairs)
    return HostInit(position=np.asarray(positions, _F), pairs=np.asarray(pairs, np.int32).reshape(-1, 2),
                    theta=theta, rest_lengths=np.asarray(rest_lengths, _F),
                    bending_pairs=np.asarray(bpairs, np.int32).reshape(-1, 2),
                    bending_rest_angles=np.asarray(rest_angles, _F), bending_stiffness=np.asarray(stiffness, _F))


class LineEnv(Environment):
    """Open chain of nodes laid out horizontally through the grid centre (line.py:12-89)."""

    def __init__(self, num_nodes=16, spacing=2.0, bending_stiffness=0.5, **kwargs):
        super().__init__(**kwargs)
        self._num_nodes = num_nodes
        self._spacing = spacing
        self._bending_stiffness = bending_stiffness
        self._edge_pairs, dep = topology.make_edges(num_nodes, "line")
        self._bending_pairs, self._bending_rest_angles = topology.compute_bending_pairs(
            self._edge_pairs, dep, num_nodes)

    @property
    def num_nodes(self):
        return self._num_nodes

    @property
    def num_edges(self):
        return int(self._edge_pairs.shape[0])

    @property
    def num_bending_pairs(self):
        return int(self._bending_pairs.shape[0])

    def _init_state(self, key):
        h, w = self.grid_shape
        n, sp = self._num_nodes, self._spacing
        total = (n - 1) * sp
        xs = _linspace(w / 2 - total / 2, w / 2 + total / 2, n)
        pos = np.stack([xs, np.full(n, h / 2.0, _F)], axis=1)
        return _init(self.grid_shape, pos, self._edge_pairs, np.full(self.num_edges, sp, _F), self._bending_pairs,
                     self._bending_rest_angles, np.full(self.num_bending_pairs, self._bending_stiffness, _F))


class RingEnv(Environment):
    """Closed circular loop of nodes around the grid centre (ring.py:16-86)."""

    def __init__(self, num_nodes=16, spacing=2.0, **kwargs):
        super().__init__(**kwargs)
        self._num_nodes = num_nodes
        self._spacing = spacing
        self._edge_pairs, dep = topology.make_edges(num_nodes, "loop")
        self._bending_pairs, self._bending_rest_angles = topology.compute_bending_pairs(
            self._edge_pairs, dep, num_nodes)

    @property
    def num_nodes(self):
        return self._num_nodes

    @property
    def num_edges(self):
        return int(self._edge_pairs.shape[0])

    @property
    def num_bending_pairs(self):
        return int(self._bending_pairs.shape[0])

    def _init_state(self, key):
        h, w = self.grid_shape
        n, sp = self._num_nodes, self._spacing
        radius = n * sp / (2 * math.pi)
        ang = _linspace(0, 2 * math.pi, n, endpoint=False)
        pos = np.stack([_F(w / 2) + _F(radius) * np.cos(ang), _F(h / 2) + _F(radius) * np.sin(ang)], axis=1)
        return _init(self.grid_shape, pos, self._edge_pairs, np.full(self.num_edges, sp, _F), self._bending_pairs,
                     self._bending_rest_angles, np.full(self.num_bending_pairs, 0.5, _F))


class RandomFoodLineEnv(LineEnv):
    """Line environment whose energy source is placed uniformly at random on every reset,
    at least min(2 * energy_size, 0.45 * side) from the borders (random_food.py:7-23)."""

    def __init__(self, *args, energy_amplitude=1.0, **kwargs):
        super().__init__(*args, energy_amplitude=energy_amplitude, **kwargs)

    def _sample_energy_center(self, key):
        h, w = self.grid_shape
        world = np.array([w, h], _F)
        margin = np.minimum(_F(2.0 * self.energy_size), _F(0.45) * world)
        low, high = margin, world - margin
        u = key.random(2).astype(_F)
        return (low + u * (high - low)).astype(_F)


class TadpoleEnv(Environment):
    """A circular head loop with a straight tail from head node 0 (tadpole.py:20-124)."""

    def __init__(self, head_nodes=8, tail_nodes=10, spacing=2.0, **kwargs):
        super().__init__(**kwargs)
        self._head_nodes = head_nodes
        self._tail_nodes = tail_nodes
        self._spacing = spacing
        b = topology.GraphBuilder()
        head = b.add_loop(head_nodes)
        b.add_branch(from_node=head[0], length=tail_nodes)
        self._edge_pairs, dep = b.build()
        self._bending_pairs, self._bending_rest_angles = topology.compute_bending_pairs(
            self._edge_pairs, dep, head_nodes + tail_nodes)

    @property
    def num_nodes(self):
        return self._head_nodes + self._tail_nodes

    @property
    def num_edges(self):
        return int(self._edge_pairs.shape[0])

    @property
    def num_bending_pairs(self):
        return int(self._bending_pairs.shape[0])

    def _init_state(self, key):
        h, w = self.grid_shape
        hn, tn, sp = self._head_nodes, self._tail_nodes, self._spacing
        radius = hn * sp / (2 * math.pi)
        cx = w / 2 - (tn * sp) / 2
        cy = h / 2
        ang = _linspace(0.0, 2 * math.pi, hn, endpoint=False)
        head = np.stack([_F(cx) + _F(radius) * np.cos(ang), _F(cy) + _F(radius) * np.sin(ang)], axis=1)
        tail_x = _linspace(cx + radius + sp, cx + radius + tn * sp, tn)
        tail = np.stack([tail_x, np.full(tn, cy, _F)], axis=1)
        pos = np.concatenate([head, tail], axis=0)
        theta = topology.edge_angles(self.grid_shape, pos, self._edge_pairs)
        rest = topology.set_orthogonal_rest_angles(self._edge_pairs, theta, self._bending_pairs,
                                                   self._bending_rest_angles, self.num_nodes)
        return _init(self.grid_shape, pos, self._edge_pairs, np.full(self.num_edges, sp, _F), self._bending_pairs,
                     rest, np.full(self.num_bending_pairs, 0.5, _F))


@dataclasses.dataclass(frozen=True)
class CreatureTopology:
    """Local creature topology and rest geometry (multi_agent.py:15-27)."""
    num_nodes: int
    spacing: float = 2.0
    bending_stiffness: float = 0.5

    def edges(self):
        raise NotImplementedError

    def local_positions(self):
        raise NotImplementedError


@dataclasses.dataclass(frozen=True)
class LineTopology(CreatureTopology):
    """Open chain centred on the local origin (multi_agent.py:30-40)."""

    def edges(self):
        return topology.make_edges(self.num_nodes, "line")

    def local_positions(self):
        total = (self.num_nodes - 1) * self.spacing
        xs = _linspace(-total / 2.0, total / 2.0, self.num_nodes)
        return np.stack([xs, np.zeros(self.num_nodes, _F)], axis=1)


@dataclasses.dataclass(frozen=True)
class RingTopology(CreatureTopology):
    """Closed loop centred on the local origin (multi_agent.py:43-53)."""

    def edges(self):
        return topology.make_edges(self.num_nodes, "loop")

    def local_positions(self):
        radius = self.num_nodes * self.spacing / (2 * math.pi)
        ang = _linspace(0, 2 * math.pi, self.num_nodes, endpoint=False)
        return np.stack([_F(radius) * np.cos(ang), _F(radius) * np.sin(ang)], axis=1)


class MultiAgentEnv(Environment):
    """Several independent creatures in one domain (multi_agent.py:56-262): one rollout
    whose nodes, edges and bending pairs are the creatures' concatenated; the reward is the
    sum of the per-creature energy sums."""

    def __init__(self, creatures: Sequence[CreatureTopology] | None = None, random_initial_positions=False,
                 position_margin=0.0, **kwargs):
        super().__init__(**kwargs)
        if creatures is None:
            # as in the reference, the topologies have no default node count, so the
            # default creature pair cannot be built (TypeError) unless creatures are given
            creatures = (LineTopology(), RingTopology())
        if not creatures:
            raise ValueError("MultiAgentEnv requires at least one creature topology")
        self._creatures = tuple(creatures)
        self._random_initial_positions = random_initial_positions
        self._position_margin = position_margin
        edges, rest_l, bps, bra, bst, local, margins = [], [], [], [], [], [], []
        node_slices, edge_slices, bend_slices = [], [], []
        n0 = e0 = b0 = 0
        for c in self._creatures:
            ep, dep = c.edges()
            lp = c.local_positions()
            ne = int(ep.shape[0])
            bp, ra = topology.compute_bending_pairs(ep, dep, c.num_nodes)
            nb = int(bp.shape[0])
            edges.append(ep + n0)
            rest_l.append(np.full(ne, c.spacing, _F))
            bps.append(bp + e0)
            bra.append(ra)
            bst.append(np.full(nb, c.bending_stiffness, _F))
            local.append(lp)
            margins.append(np.max(np.abs(lp), axis=0) + _F(position_margin))
            node_slices.append(slice(n0, n0 + c.num_nodes))
            edge_slices.append(slice(e0, e0 + ne))
            bend_slices.append(slice(b0, b0 + nb))
            n0 += c.num_nodes
            e0 += ne
            b0 += nb
        self._node_slices, self._edge_slices, self._bending_slices = (tuple(node_slices), tuple(edge_slices),
                                                                      tuple(bend_slices))
        self._local_positions = tuple(local)
        self._center_margins = np.stack(margins).astype(_F)
        self._edge_pairs = np.concatenate(edges).astype(np.int32)
        self._rest_lengths = np.concatenate(rest_l)
        self._bending_pairs = np.concatenate(bps).astype(np.int32).reshape(-1, 2)
        self._bending_rest_angles = np.concatenate(bra).astype(_F)
        self._bending_stiffness = np.concatenate(bst)
        self._num_nodes = n0

    @property
    def creatures(self):
        return self._creatures

    @property
    def node_slices(self):
        return self._node_slices

    @property
    def edge_slices(self):
        return self._edge_slices

    @property
    def bending_slices(self):
        return self._bending_slices

    @property
    def num_nodes(self):
        return self._num_nodes

    @property
    def num_edges(self):
        return int(self._edge_pairs.shape[0])

    @property
    def num_bending_pairs(self):
        return int(self._bending_pairs.shape[0])

    def _segments(self):
        return [s.start for s in self._node_slices] + [self._node_slices[-1].stop]

    def split_action(self, action):
        """The flat action as one action dict per creature (multi_agent.py:170-181)."""
        return tuple({"d_rest_length": action["d_rest_length"][es], "d_bending_angle": action["d_bending_angle"][bs]}
                     for es, bs in zip(self._edge_slices, self._bending_slices, strict=True))

    def merge_action(self, creature_actions):
        """Per-creature action dicts concatenated into the flat action (multi_agent.py:183-198)."""
        if len(creature_actions) != len(self._creatures):
            raise ValueError(f"Expected {len(self._creatures)} creature actions, got {len(creature_actions)}")
        import torch
        cat = (lambda xs: torch.cat([torch.as_tensor(x) for x in xs])) if any(
            isinstance(a["d_rest_length"], torch.Tensor) for a in creature_actions) else np.concatenate
        return {"d_rest_length": cat([a["d_rest_length"] for a in creature_actions]),
                "d_bending_angle": cat([a["d_bending_angle"] for a in creature_actions])}

    def _agent_centers(self, key):
        h, w = self.grid_shape
        k = len(self._creatures)
        if self._random_initial_positions:
            world = np.array([w, h], _F)
            margins = np.minimum(self._center_margins, world / _F(2.0))
            span = world - _F(2.0) * margins
            return (margins + key.random((k, 2)).astype(_F) * span).astype(_F)
        if k == 1:
            xs = np.array([w / 2.0], _F)
        elif k == 2:
            xs = np.array([w / 4.0, 3.0 * w / 4.0], _F)
        else:
            xs = _linspace(w / (k + 1), w * k / (k + 1), k)
        return np.stack([xs, np.full(k, h / 2.0, _F)], axis=1)

    def _init_state(self, key):
        centers = self._agent_centers(key)
        pos = np.concatenate([lp + centers[i] for i, lp in enumerate(self._local_positions)], axis=0).astype(_F)
        return _init(self.grid_shape, pos, self._edge_pairs, self._rest_lengths, self._bending_pairs,
                     self._bending_rest_angles, self._bending_stiffness)


class LineRingEnv(MultiAgentEnv):
    """The default line + ring pair (line_ring.py:7-58); ``centered_line`` puts the line at
    the centre and the ring at ``ring_spawn_radius`` (default w/4) from it."""

    def __init__(self, line_topology=None, ring_topology=None, line_nodes=16, ring_nodes=16, spacing=2.0,
                 bending_stiffness=0.5, centered_line=False, ring_spawn_radius=None, random_ring_angle=False,
                 **kwargs):
        line = line_topology or LineTopology(num_nodes=line_nodes, spacing=spacing,
                                             bending_stiffness=bending_stiffness)
        ring = ring_topology or RingTopology(num_nodes=ring_nodes, spacing=spacing,
                                             bending_stiffness=bending_stiffness)
        self._centered_line = centered_line
        self._ring_spawn_radius = ring_spawn_radius
        self._random_ring_angle = random_ring_angle
        super().__init__(creatures=(line, ring), **kwargs)

    def _agent_centers(self, key):
        if not self._centered_line:
            return super()._agent_centers(key)
        h, w = self.grid_shape
        r = self._ring_spawn_radius if self._ring_spawn_radius is not None else w / 4.0
        a = _F(key.random() * 2 * math.pi) if self._random_ring_angle else _F(0.0)
        line_c = np.array([w / 2.0, h / 2.0], _F)
        ring_c = np.array([_F(w / 2.0) + _F(r) * np.cos(a), _F(h / 2.0) + _F(r) * np.sin(a)], _F)
        return np.stack([line_c, ring_c], axis=0)
