"""CPU oracle of the gym environment step (TEST INFRASTRUCTURE ONLY; the product never
imports it): a numpy restatement of src/microcosmos/gym/base.py:89-196 and
multi_agent.py:201-212 around ``ref_numpy.step``.  Pinned against golden vectors that
executed the reference's gym environments on numpy (tests/golden/make_golden.py, group
"gym")."""
from __future__ import annotations

import numpy as np

from . import ref_numpy as O


def energy_at(H, W, positions, center, amplitude, size):
    """amplitude * exp(-|min-image(x - center)|^2 / (2 size^2)) (base.py:89-94)."""
    t = positions.dtype.type
    d = O.displacement(H, W, positions, np.asarray(center, positions.dtype))
    dist_sq = d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]
    return t(amplitude) * np.exp(-dist_sq / t(2.0 * size ** 2))


def observation(H, W, positions, velocity, center, amplitude, size):
    """[positions - mean, velocities, energy at the nodes] (base.py:112-121)."""
    centered = positions - positions.mean(axis=0)
    e = energy_at(H, W, positions, center, amplitude, size)
    return np.concatenate([centered.reshape(-1), velocity.reshape(-1), e])


def env_step(s: O.State, cfg: O.Config, dt, base_rest, base_angles, action, center, time, max_steps, amplitude,
             size, walk_std=0.0, noise=None, segments=None):
    """One Environment.step (base.py:163-196): rest geometry = base + action, the physics
    step, the energy source's walk, then observation, reward (per-creature sums added,
    multi_agent.py:201-212), time + 1 and done.  Returns (obs, state, reward, done,
    center, time, fitness)."""
    t = s.position.dtype.type
    s = s.copy()
    s.rest_lengths = (base_rest + action["d_rest_length"]).astype(s.position.dtype)
    s.bending_rest_angles = (base_angles + action["d_bending_angle"]).astype(s.position.dtype)
    s = O.step(s, cfg, dt)
    step_noise = (np.zeros(2, s.position.dtype) if noise is None else np.asarray(noise, s.position.dtype)) * t(walk_std)
    center = np.mod(np.asarray(center, s.position.dtype) + step_noise,
                    np.array([s.W, s.H], s.position.dtype))
    obs = observation(s.H, s.W, s.position, s.velocity, center, amplitude, size)
    e = energy_at(s.H, s.W, s.position, center, amplitude, size)
    segs = [0, s.position.shape[0]] if segments is None else list(segments)
    fitness = np.array([e[a:b].sum() for a, b in zip(segs[:-1], segs[1:])], s.position.dtype)
    reward = fitness.sum() if segments is not None else e.sum()
    time = time + 1
    return obs, s, reward, time >= max_steps, center, time, fitness
