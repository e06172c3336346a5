"""Seeded synthetic workloads (filament swimmers in a periodic D2Q9 fluid).

The reference repository ships no datasets for this path; its benchmark
configurations are synthetic.  This module builds them with
``numpy.random.default_rng(seed)`` so that the CUDA path, the tests and the
benchmark all see identical inputs.

Topology follows the reference's builders:

* edges: ``make_edges(N_total, "line", num_instances=F)`` (graph.py:156-192) — F
  independent chains, edge e = (i, i+1) inside each chain, chains laid out one
  after another;
* bending pairs: ``compute_bending_pairs`` (graph.py:347-401) — for every node,
  (incoming edge, outgoing edge) pairs, i.e. (e, e+1) inside a chain;
* edge angle: ``arctan2`` of the minimum-image edge vector (env.py:61-62);
* populations: ``feq(rho=1, u0)`` as ``graph._initialize_f_from_velocity``
  (graph.py:533-540).

Curvature actuation is a caller-side control in the reference (it rewrites
``edges.bending_rest_angles`` before each ``step``: experiments/swim_sweep/
swimmers/worm.py:60-74, tests/test_worm.py:100-116).  This build fixes one closed
form, used identically by the kernels and the oracle::

    rest[b](t) = c[b] + A_f * sin(2*pi*t/P_f + phi_f - 2*pi*j_b/n_f)

with t the step index (0 for the first step), f the filament of pair b, j_b the
pair's index inside its filament and n_f the filament's pair count.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

LBM_E = np.array([[0, 0], [1, 0], [0, 1], [-1, 0], [0, -1],
                  [1, 1], [-1, 1], [-1, -1], [1, -1]], dtype=np.int32)
LBM_W = np.array([4 / 9, 1 / 9, 1 / 9, 1 / 9, 1 / 9, 1 / 36, 1 / 36, 1 / 36, 1 / 36])


@dataclasses.dataclass
class Scenario:
    """One rollout's initial state, topology and actuation (numpy, host)."""
    H: int
    W: int
    position: np.ndarray          # (N, 2) f32, (x, y)
    velocity: np.ndarray          # (N, 2) f32
    pairs: np.ndarray             # (E, 2) i32
    theta: np.ndarray             # (E,) f32
    rest_lengths: np.ndarray      # (E,) f32
    bending_pairs: np.ndarray     # (B, 2) i32
    bending_rest_angles: np.ndarray  # (B,) f32
    bending_stiffness: np.ndarray    # (B,) f32
    f_grid: np.ndarray            # (9, H, W) f32
    steric: np.ndarray            # (H, W) f32
    fluid_velocity: np.ndarray    # (2, H, W) f32
    # actuation (None = no actuation)
    act_c: np.ndarray | None = None      # (B,) f32 rest-curvature offsets
    act_amp: np.ndarray | None = None    # (B,) f32 amplitude of the pair's filament
    act_omega: np.ndarray | None = None  # (B,) f32  2*pi/P_f
    act_phase: np.ndarray | None = None  # (B,) f32  phi_f - 2*pi*j_b/n_f

    @property
    def N(self):
        return self.position.shape[0]

    @property
    def E(self):
        return self.pairs.shape[0]

    @property
    def B(self):
        return self.bending_pairs.shape[0]


def line_topology(sizes):
    """Edges and bending pairs of independent chains with the given node counts
    (make_edges(..., "line", F) + compute_bending_pairs)."""
    pairs = []
    bpairs = []
    start = 0
    e0 = 0
    for n in sizes:
        for i in range(n - 1):
            pairs.append((start + i, start + i + 1))
        for i in range(n - 2):
            bpairs.append((e0 + i, e0 + i + 1))
        start += n
        e0 += n - 1
    return (np.array(pairs, dtype=np.int32).reshape(-1, 2),
            np.array(bpairs, dtype=np.int32).reshape(-1, 2))


def equilibrium(rho, ux, uy):
    """feq(rho, u) in float32 with the reference's operation order
    (graph.py:533-540, solver/fluid.py:145-151)."""
    rho = np.asarray(rho, np.float32)
    ux = np.asarray(ux, np.float32)
    uy = np.asarray(uy, np.float32)
    usq = ux * ux + uy * uy
    out = np.empty((9,) + ux.shape, np.float32)
    for i in range(9):
        eu = np.float32(LBM_E[i, 0]) * ux + np.float32(LBM_E[i, 1]) * uy
        out[i] = rho * np.float32(LBM_W[i]) * (np.float32(1.0) + np.float32(3.0) * eu
                                               + np.float32(4.5) * (eu * eu) - np.float32(1.5) * usq)
    return out


def _wrap_mod(x, L):
    return np.mod(x, np.float32(L)).astype(np.float32)


def _poisson_centres(rng, n, H, W, min_sep, max_tries=200000):
    pts = []
    tries = 0
    while len(pts) < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError(f"Poisson-disk placement of {n} centres with min sep {min_sep} failed")
        p = np.array([rng.uniform(0, W), rng.uniform(0, H)])
        ok = True
        for q in pts:
            d = p - q
            d[0] -= W * np.round(d[0] / W)
            d[1] -= H * np.round(d[1] / H)
            if d[0] * d[0] + d[1] * d[1] < min_sep * min_sep:
                ok = False
                break
        if ok:
            pts.append(p)
    return np.array(pts)


def make_scenario(H, W, num_filaments, nodes_per_filament, *, seed=0, rng=None,
                  placement="uniform", min_sep=8.0, spacing=1.0, u0_std=1e-3,
                  bending_stiffness=0.1, amp=0.2, period=200.0, amp_dist=None,
                  period_dist=None, phase_dist=None, actuate=True):
    """Build a seeded filament-swimmer scenario.

    ``amp_dist``/``period_dist``/``phase_dist`` are callables ``rng -> value`` drawn per
    filament; otherwise the scalar ``amp``/``period`` and phase 0 are used.
    """
    rng = np.random.default_rng(seed) if rng is None else rng
    F = int(num_filaments)
    n = int(nodes_per_filament)
    sizes = [n] * F
    pairs, bpairs = line_topology(sizes)
    if placement == "poisson":
        centres = _poisson_centres(rng, F, H, W, min_sep)
    else:
        centres = np.stack([rng.uniform(0, W, F), rng.uniform(0, H, F)], axis=1)
    angles = rng.uniform(0, 2 * np.pi, F)
    pos = np.zeros((F * n, 2), np.float64)
    offs = (np.arange(n) - (n - 1) / 2.0) * spacing
    for f in range(F):
        pos[f * n:(f + 1) * n, 0] = centres[f, 0] + offs * np.cos(angles[f])
        pos[f * n:(f + 1) * n, 1] = centres[f, 1] + offs * np.sin(angles[f])
    pos = pos.astype(np.float32)
    pos[:, 0] = _wrap_mod(pos[:, 0], W)
    pos[:, 1] = _wrap_mod(pos[:, 1], H)
    # edge angle from the minimum-image edge vector (utils.displacement, size=(H, W))
    L = np.array([W, H], np.float32)
    d = pos[pairs[:, 1]] - pos[pairs[:, 0]]
    d = (np.mod(d + L / np.float32(2.0), L) - L / np.float32(2.0)).astype(np.float32)
    theta = np.arctan2(d[:, 1], d[:, 0]).astype(np.float32)
    E = pairs.shape[0]
    B = bpairs.shape[0]
    u0 = rng.normal(0.0, u0_std, size=(2, H, W)).astype(np.float32)
    f_grid = equilibrium(np.ones((H, W), np.float32), u0[0], u0[1])
    sc = Scenario(
        H=H, W=W, position=pos, velocity=np.zeros_like(pos), pairs=pairs, theta=theta,
        rest_lengths=np.full(E, spacing, np.float32), bending_pairs=bpairs,
        bending_rest_angles=np.zeros(B, np.float32),
        bending_stiffness=np.full(B, bending_stiffness, np.float32),
        f_grid=f_grid, steric=np.zeros((H, W), np.float32),
        fluid_velocity=np.zeros((2, H, W), np.float32))
    if actuate and B > 0:
        amps = np.array([amp_dist(rng) if amp_dist else amp for _ in range(F)], np.float64)
        periods = np.array([period_dist(rng) if period_dist else period for _ in range(F)], np.float64)
        phases = np.array([phase_dist(rng) if phase_dist else 0.0 for _ in range(F)], np.float64)
        nb = n - 2
        fil = np.repeat(np.arange(F), nb)
        j = np.tile(np.arange(nb), F)
        sc.act_c = np.zeros(B, np.float32)
        sc.act_amp = amps[fil].astype(np.float32)
        sc.act_omega = (2 * np.pi / periods[fil]).astype(np.float32)
        sc.act_phase = (phases[fil] - 2 * np.pi * j / max(nb, 1)).astype(np.float32)
        sc.bending_rest_angles = actuation_rest_angles(sc, 0)
    return sc


def actuation_rest_angles(sc, t):
    """rest[b](t) = c[b] + A*sin(omega*t + phase) in float32 (same op order as the kernel)."""
    arg = sc.act_omega * np.float32(t) + sc.act_phase
    return (sc.act_c + sc.act_amp * np.sin(arg.astype(np.float32))).astype(np.float32)


# ------------------------------------------------------------------ benchmark configurations
def config_small(seed=0):
    """128x128 periodic, 4 filaments x 32 nodes, uniform placement, amp 0.2, period 200."""
    return make_scenario(128, 128, 4, 32, seed=seed, placement="uniform", amp=0.2, period=200.0)


def config_scale(seed=0):
    """1024x1024 periodic, 256 filaments x 64 nodes, Poisson-disk centres (min sep 8),
    amp ~ U(0.1, 0.3), period ~ U(100, 400)."""
    return make_scenario(1024, 1024, 256, 64, seed=seed, placement="poisson", min_sep=8.0,
                         amp_dist=lambda r: r.uniform(0.1, 0.3),
                         period_dist=lambda r: r.uniform(100.0, 400.0))


def config_batch(num_rollouts=256, seed=0):
    """Evolutionary-search population of uneven rollouts: side ~ U{128,192,256,384,512},
    filaments ~ U{1..32}, nodes/filament ~ U{16..128}, amplitude ~ N(0.2, 0.05)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(num_rollouts):
        side = int(rng.choice([128, 192, 256, 384, 512]))
        F = int(rng.integers(1, 33))
        n = int(rng.integers(16, 129))
        a = float(rng.normal(0.2, 0.05))
        out.append(make_scenario(side, side, F, n, rng=rng, amp=a, period=200.0))
    return out
