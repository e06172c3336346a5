"""Host-side construction of the environments' rod topologies and fields: the parts of the
reference's graph utilities the gym environments use (src/microcosmos/graph.py,
src/microcosmos/graph_builder.py).  One-time set-up in numpy; the device never sees it.

* ``make_edges`` (graph.py:156-260): forward-only directed edges of "loop", "line" and
  "tree" instances laid out one after another, with per-edge departure angles;
* ``compute_bending_pairs`` (graph.py:347-401): (incoming edge, outgoing edge) pairs per
  node in node order, rest angle = departure[out] - departure[in];
* ``set_orthogonal_rest_angles`` (graph.py:404-520): at junctions, the most aligned pair
  stays straight and the others get +-pi/2 by the layout's turning direction;
* ``GraphBuilder`` (graph_builder.py:30-157): loops, lines and branches; edges listed the
  way a networkx DiGraph lists them (nodes in first-insertion order, each node's
  successors in insertion order);
* ``make_fields`` (graph.py:586-596): zero steric and velocity, populations at rest.
"""
from __future__ import annotations

import math

import numpy as np

from .. import scenarios


def _single_edges(n, graph, offset):
    if graph == "loop":
        src = np.arange(n) + offset
        return np.stack([src, np.roll(src, -1)], axis=1), np.zeros(n, np.float32)
    if graph == "line":
        src = np.arange(n - 1) + offset
        return np.stack([src, src + 1], axis=1), np.zeros(n - 1, np.float32)
    if graph == "tree":
        trunk = int(n * 0.6)
        rest = n - trunk
        b1 = rest // 2
        b2 = rest - b1
        b1_start, b2_start = offset + trunk, offset + trunk + b1
        junction = offset + trunk // 2
        edges, dep = [], []
        for i in range(trunk - 1):
            edges.append((offset + i, offset + i + 1))
            dep.append(0.0)
        edges.append((junction, b1_start))
        dep.append(math.pi / 2.0)
        for i in range(b1 - 1):
            edges.append((b1_start + i, b1_start + i + 1))
            dep.append(math.pi / 2.0)
        edges.append((junction, b2_start))
        dep.append(-math.pi / 2.0)
        for i in range(b2 - 1):
            edges.append((b2_start + i, b2_start + i + 1))
            dep.append(-math.pi / 2.0)
        return np.array(edges, np.int32), np.array(dep, np.float32)
    raise ValueError(f"Unknown graph type: {graph}")


def make_edges(num_nodes, graph="loop", num_instances=1):
    """(E, 2) int32 edges and (E,) float32 departure angles of ``num_instances`` instances
    of ``graph`` with ``num_nodes`` nodes in total (the first ``num_nodes % num_instances``
    instances get one node more)."""
    per, rem = divmod(num_nodes, num_instances)
    if per < 1:
        raise ValueError(f"num_nodes ({num_nodes}) must be at least {num_instances} to create "
                         f"{num_instances} instances.")
    edges, deps = [], []
    start = 0
    for i in range(num_instances):
        size = per + (1 if i < rem else 0)
        e, d = _single_edges(size, graph, start)
        edges.append(np.asarray(e).reshape(-1, 2))
        deps.append(np.asarray(d, np.float32))
        start += size
    return np.concatenate(edges).astype(np.int32), np.concatenate(deps).astype(np.float32)


def _incidence(edge_pairs, num_nodes):
    incoming = [[] for _ in range(num_nodes)]
    outgoing = [[] for _ in range(num_nodes)]
    for e, (s, t) in enumerate(np.asarray(edge_pairs).reshape(-1, 2)):
        outgoing[int(s)].append(e)
        incoming[int(t)].append(e)
    return incoming, outgoing


def compute_bending_pairs(edge_pairs, departure_angles, num_nodes):
    """(B, 2) int32 (edge_in, edge_out) pairs and (B,) float32 rest angles."""
    dep = np.asarray(departure_angles, np.float32)
    incoming, outgoing = _incidence(edge_pairs, num_nodes)
    pairs, rest = [], []
    for node in range(num_nodes):
        for ei in incoming[node]:
            for eo in outgoing[node]:
                pairs.append((ei, eo))
                rest.append(float(dep[eo] - dep[ei]))
    return (np.array(pairs, np.int32).reshape(-1, 2), np.array(rest, np.float32))


def set_orthogonal_rest_angles(edge_pairs, edge_theta, bending_pairs, bending_rest_angles, num_nodes):
    """Junction rest angles from the layout: per junction node (more than two incident
    edges) the pair with the smallest |wrap(theta_out - theta_in)| is the continuation
    (rest 0), every other pair gets sign(wrap(...)) * pi/2 (0 counts as +)."""
    edges = np.asarray(edge_pairs).reshape(-1, 2)
    theta = np.asarray(edge_theta, np.float32)
    bp = np.asarray(bending_pairs).reshape(-1, 2)
    rest = np.array(bending_rest_angles, np.float32, copy=True)
    if bp.shape[0] == 0:
        return rest
    incoming, outgoing = _incidence(edges, num_nodes)
    junctions = [n for n in range(num_nodes) if len(incoming[n]) + len(outgoing[n]) > 2]

    def turn(b):
        ti, to = float(theta[bp[b, 0]]), float(theta[bp[b, 1]])
        return float(np.arctan2(np.sin(to - ti), np.cos(to - ti)))

    # the reference walks its junction set; each junction's update touches only its own pairs
    for node in junctions:
        at = [b for b in range(bp.shape[0]) if int(edges[bp[b, 0], 1]) == node]
        if not at:
            continue
        cont = int(np.argmin([abs(turn(b)) for b in at]))
        for i, b in enumerate(at):
            rest[b] = 0.0 if i == cont else (1.0 if turn(b) >= 0 else -1.0) * (np.pi / 2)
    return rest.astype(np.float32)


class GraphBuilder:
    """Loops, lines and branches into a forward-only edge list (graph_builder.py:30-157)."""

    def __init__(self):
        self._succ = {}   # node -> {successor: departure angle}, both in insertion order
        self.next_id = 0

    def _add_edge(self, u, v, angle):
        self._succ.setdefault(u, {})
        self._succ.setdefault(v, {})
        self._succ[u][v] = angle

    def add_loop(self, length):
        nodes = list(range(self.next_id, self.next_id + length))
        for i, u in enumerate(nodes):
            self._add_edge(u, nodes[(i + 1) % len(nodes)], 0.0)
        self.next_id += length
        return nodes

    def add_line(self, length):
        nodes = list(range(self.next_id, self.next_id + length))
        for u, v in zip(nodes[:-1], nodes[1:]):
            self._add_edge(u, v, 0.0)
        self.next_id += length
        return nodes

    def add_branch(self, from_node, length, departure_angle=None):
        nodes = list(range(self.next_id, self.next_id + length))
        self.next_id += length
        for u, v in zip(nodes[:-1], nodes[1:]):
            self._add_edge(u, v, 0.0)
        if departure_angle is None:
            existing = sum(1 for a in self._succ.get(from_node, {}).values() if abs(a) > 0.1)
            departure_angle = math.pi / 2.0 if existing == 0 else -math.pi / 2.0
        self._add_edge(from_node, nodes[0], departure_angle)
        for u, v in zip(nodes[:-1], nodes[1:]):
            self._succ[u][v] = departure_angle
        return nodes

    def build(self):
        n = len(self._succ)
        if set(self._succ) != set(range(n)):
            raise ValueError(f"Graph nodes must be contiguous integers from 0 to {n - 1}. "
                             f"Got nodes: {sorted(self._succ)}")
        edges, dep = [], []
        for u, succ in self._succ.items():
            for v, a in succ.items():
                edges.append((u, v))
                dep.append(a)
        return np.array(edges, np.int32).reshape(-1, 2), np.array(dep, np.float32)


def edge_angles(grid_shape, positions, edge_pairs):
    """arctan2 of each edge's min-image vector (the environments' initial theta)."""
    H, W = grid_shape
    p = np.asarray(positions, np.float32)
    e = np.asarray(edge_pairs).reshape(-1, 2)
    L = np.array([W, H], np.float32)
    half = L / np.float32(2.0)
    d = np.mod(p[e[:, 1]] - p[e[:, 0]] + half, L) - half
    return np.arctan2(d[:, 1], d[:, 0]).astype(np.float32)


def make_fields(grid_shape):
    """(steric, fluid_velocity, f_grid) of a fluid at rest: zeros and feq(1, 0)."""
    H, W = grid_shape
    z = np.zeros((H, W), np.float32)
    return z, np.zeros((2, H, W), np.float32), scenarios.equilibrium(np.ones((H, W), np.float32), z, z)
