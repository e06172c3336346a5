"""The gymnax-style environment interface of the reference (src/microcosmos/gym/base.py:15-196)
over the device rollout.

``Environment.reset(key)`` / ``step(key, state, action)`` keep the reference's signatures,
return values and pure-functional contract (the input state is never modified; ``step``
returns a new state).  One step is: ``mc_env_act`` (rest lengths / rest angles = the
episode's base values + the action), the physics step through the rollout plan (the same
kernels as ``simulate``), and ``mc_env_observe`` (energy-source walk, observation, reward,
step counter, done flag) -- all on the device, the state never leaves it.

``key`` is an integer seed, a ``numpy.random.Generator`` or ``None``.  It is used where the
reference draws from ``jax.random`` (the energy source's walk noise, randomised energy or
creature placement); JAX's PRNG stream is not reproduced, so those draws follow the same
distributions with different values.  With the defaults (``energy_walk_std = 0``,
deterministic placement) no draw affects the result.
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np
import torch

from .. import _lib
from ..config import PBD_SCHEME, ConstraintSolverConfig
from ..engine import DeviceState, Plan, _require_cuda
from ..structs import Edges, Fields, Nodes
from . import topology

_F32 = torch.float32


def _rng(key):
    if isinstance(key, np.random.Generator):
        return key
    return np.random.default_rng(None if key is None else int(np.asarray(key).ravel()[-1]))


@dataclasses.dataclass
class EnvState:
    """The reference's EnvState (base.py:16-37) on the device: ``device`` holds the
    nodes/edges/fields arrays the rollout reads and writes; ``time`` () int32,
    ``energy_center`` (2,) float32, and the episode's base rest geometry."""
    device: DeviceState
    time: torch.Tensor
    energy_center: torch.Tensor
    base_rest_lengths: torch.Tensor
    base_bending_rest_angles: torch.Tensor
    color_bend: np.ndarray

    @property
    def nodes(self):
        s = self.device
        return Nodes(position=s.position, velocity=s.velocity, color_bend=self.color_bend,
                     debug_vector=torch.zeros_like(s.position))

    @property
    def edges(self):
        s = self.device
        return Edges(pairs=s.pairs, theta=s.theta, rest_lengths=s.rest_lengths, bending_pairs=s.bending_pairs,
                     bending_rest_angles=s.bending_rest_angles, bending_stiffness=s.bending_stiffness)

    @property
    def fields(self):
        s = self.device
        return Fields(grid_shape=(s.H, s.W), steric=s.steric, fluid_velocity=s.fluid_velocity, f_grid=s.f_grid)

    def clone(self):
        s = self.device
        dev = dataclasses.replace(s, **{f.name: getattr(s, f.name).clone() for f in dataclasses.fields(s)
                                        if isinstance(getattr(s, f.name), torch.Tensor)})
        return EnvState(dev, self.time.clone(), self.energy_center.clone(), self.base_rest_lengths,
                        self.base_bending_rest_angles, self.color_bend)


@dataclasses.dataclass
class HostInit:
    """An environment's initial state on the host (what ``_init_state`` builds)."""
    position: np.ndarray
    pairs: np.ndarray
    theta: np.ndarray
    rest_lengths: np.ndarray
    bending_pairs: np.ndarray
    bending_rest_angles: np.ndarray
    bending_stiffness: np.ndarray


class Environment:
    """Pure-functional environment with a Gaussian energy source (base.py:40-196).
    Subclasses implement ``_init_state(key) -> HostInit`` and the ``num_edges`` /
    ``num_bending_pairs`` properties; ``_segments`` (node offsets per creature) lets a
    subclass split the reward into per-creature sums."""

    def __init__(self, grid_shape=(128, 128), dt=0.01, max_steps=1000,
                 solver_config: ConstraintSolverConfig = PBD_SCHEME, energy_size=15.0, energy_amplitude=0.0,
                 energy_walk_std=0.0):
        self.grid_shape = tuple(int(v) for v in grid_shape)
        self.dt = dt
        self.max_steps = max_steps
        self.solver_config = solver_config
        self.energy_size = energy_size
        self.energy_amplitude = energy_amplitude
        self.energy_walk_std = energy_walk_std
        self._plan = None
        self._seg_dev = None

    # ----- subclass hooks -----
    def _init_state(self, key) -> HostInit:
        raise NotImplementedError

    @property
    def num_edges(self) -> int:
        raise NotImplementedError

    @property
    def num_bending_pairs(self) -> int:
        raise NotImplementedError

    def _segments(self):
        """Node offsets of the creatures (None: one)."""
        return None

    # ----- energy helpers -----
    def _sample_energy_center(self, key):
        """Fixed at (2 * energy_size, 2 * energy_size) (base.py:96-101)."""
        m = 2.0 * self.energy_size
        return np.array([m, m], np.float32)

    # ----- public API -----
    def action_spec(self) -> dict:
        return {"d_rest_length": (self.num_edges,), "d_bending_angle": (self.num_bending_pairs,)}

    def zero_action(self, device="cuda") -> dict:
        return {"d_rest_length": torch.zeros(self.num_edges, dtype=_F32, device=device),
                "d_bending_angle": torch.zeros(self.num_bending_pairs, dtype=_F32, device=device)}

    def _device_state(self, init: HostInit, device="cuda") -> DeviceState:
        H, W = self.grid_shape
        steric, fluid_velocity, f_grid = topology.make_fields(self.grid_shape)
        return DeviceState.from_arrays(H, W, init.position, np.zeros_like(init.position), init.pairs, init.theta,
                                       init.rest_lengths, init.bending_pairs, init.bending_rest_angles,
                                       init.bending_stiffness, f_grid, steric, fluid_velocity, device=device)

    def reset(self, key=None, device="cuda"):
        """(observation, state) of a new episode (base.py:140-149)."""
        _require_cuda()
        rng = _rng(key)
        init = self._init_state(rng)
        dev = self._device_state(init, device)
        state = EnvState(dev, torch.zeros((), dtype=torch.int32, device=device),
                         torch.as_tensor(self._sample_energy_center(rng), dtype=_F32, device=device),
                         dev.rest_lengths.clone(), dev.bending_rest_angles.clone(),
                         np.arange(dev.N) % 3)
        obs, _, _, _ = self._observe([state], advance=False)
        return obs[0], state

    def step(self, key, state: EnvState, action: dict):
        """(obs, new_state, reward, done, info) (base.py:163-196); ``state`` is not modified."""
        new = state.clone()
        plan = self._get_plan(new.device)
        acts = [_action_tensors(action, new.device)]
        noise = [self._noise(key, new.device)]
        table = self._table([new], acts, noise)
        stream = torch.cuda.current_stream().cuda_stream
        lib = _lib.load()
        _lib.check(lib.mc_env_act(ctypes.c_void_p(table["ptr"]), 1, ctypes.c_void_p(stream)))
        plan.rollout([new.device], 1)
        _lib.check(lib.mc_env_observe(ctypes.c_void_p(table["ptr"]), 1, 1, ctypes.c_void_p(stream)))
        out = table["out"]
        info = {"steps": new.time, "energy_center": new.energy_center}
        return out["obs"][0], new, out["reward"][0], out["done"][0].bool(), info

    def fitness_per_creature(self, state: EnvState):
        """Sum of the energy over each creature's nodes (multi_agent.py:201-208)."""
        _, _, _, fit = self._observe([state], advance=False)
        return fit[0]

    # ----- device plumbing -----
    def _get_plan(self, dev: DeviceState):
        if self._plan is None:
            self._plan = Plan.for_states([dev], [self.solver_config], [self.dt])
        return self._plan

    def _noise(self, key, dev):
        if self.energy_walk_std == 0.0 and key is None:
            return None
        return torch.as_tensor(_rng(key).standard_normal(2).astype(np.float32), device=dev.position.device)

    def _segment_offsets(self, device):
        seg = self._segments()
        if seg is None:
            return None
        if self._seg_dev is None:
            self._seg_dev = torch.as_tensor(np.asarray(seg, np.int32), device=device)
        return self._seg_dev

    def _table(self, states, actions, noises):
        """mc_env structs for ``states`` uploaded into a fresh device table; the output
        tensors live in the returned dict (and keep the table's pointers valid)."""
        n = len(states)
        dev0 = states[0].device
        device = dev0.position.device
        N = dev0.N
        seg = self._segment_offsets(device)
        nseg = 1 if seg is None else int(seg.numel()) - 1
        out = {"obs": torch.empty((n, 5 * N), dtype=_F32, device=device),
               "reward": torch.empty(n, dtype=_F32, device=device),
               "done": torch.zeros(n, dtype=torch.int32, device=device),
               "fitness": torch.empty((n, nseg), dtype=_F32, device=device)}
        lib = _lib.load()
        envs = (_lib.McEnv * n)()
        keep = [out]
        for i, (st, act, nz) in enumerate(zip(states, actions, noises)):
            d = st.device
            e = envs[i]
            e.N, e.E, e.B, e.H, e.W = d.N, d.E, d.B, d.H, d.W
            e.base_rest_lengths = st.base_rest_lengths.data_ptr()
            e.base_bending_rest_angles = st.base_bending_rest_angles.data_ptr()
            if act is not None:
                keep.append(act)
                e.d_rest_length = act[0].data_ptr() if act[0] is not None else None
                e.d_bending_angle = act[1].data_ptr() if act[1] is not None else None
            e.rest_lengths = d.rest_lengths.data_ptr()
            e.bending_rest_angles = d.bending_rest_angles.data_ptr()
            e.position = d.position.data_ptr()
            e.velocity = d.velocity.data_ptr()
            e.energy_center = st.energy_center.data_ptr()
            e.noise = nz.data_ptr() if nz is not None else None
            keep.append(nz)
            e.energy_walk_std = float(self.energy_walk_std)
            e.energy_amplitude = float(self.energy_amplitude)
            e.energy_two_size_sq = float(2.0 * self.energy_size ** 2)
            e.max_steps = int(self.max_steps)
            e.time = st.time.data_ptr()
            e.done = out["done"][i:].data_ptr()
            e.observation = out["obs"][i].data_ptr()
            e.reward = out["reward"][i:].data_ptr()
            e.num_segments = nseg
            e.segment_offsets = seg.data_ptr() if seg is not None else None
            e.segment_fitness = out["fitness"][i].data_ptr()
        nbytes = lib.mc_env_table_bytes(n)
        buf = torch.empty(nbytes + 64, dtype=torch.uint8, device=device)
        ptr = (buf.data_ptr() + 63) // 64 * 64
        stream = torch.cuda.current_stream().cuda_stream
        _lib.check(lib.mc_env_table_upload(envs, n, ctypes.c_void_p(ptr), ctypes.c_void_p(stream)))
        return {"ptr": ptr, "buf": buf, "out": out, "keep": keep}

    def _observe(self, states, advance):
        """Observation / reward / done / per-creature fitness of ``states`` without a step;
        with ``advance`` the energy source walks and the step counter advances."""
        t = self._table(states, [None] * len(states), [None] * len(states))
        stream = torch.cuda.current_stream().cuda_stream
        _lib.check(_lib.load().mc_env_observe(ctypes.c_void_p(t["ptr"]), len(states), int(bool(advance)),
                                              ctypes.c_void_p(stream)))
        o = t["out"]
        return o["obs"], o["reward"], o["done"], o["fitness"]


def _action_tensors(action, dev: DeviceState):
    if action is None:
        return None
    device = dev.position.device

    def conv(x, n):
        if x is None:
            return None
        t = torch.as_tensor(x, dtype=_F32, device=device).reshape(-1).contiguous()
        if t.numel() != n:
            raise ValueError(f"action of {t.numel()} values, expected {n}")
        return t
    return (conv(action.get("d_rest_length"), dev.E), conv(action.get("d_bending_angle"), dev.B))
