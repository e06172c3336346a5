"""Many environments stepped together: the reference batches ``Environment.step`` with
``jax.vmap`` (the ES notebook evaluates a population that way); here B environments of
one ``Environment`` share one rollout plan, one action launch and one observation launch
per step, and their physics steps run in one launch sequence (every kernel takes the
batch's table of rollouts).

The batch owns its states: ``step`` advances them in place and returns the same
``BatchedState`` (like a donated argument under ``jax.jit``); ``state.env_state(i)`` gives
one environment's ``EnvState`` (the populations are brought back up to date first).
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np
import torch

from .. import _lib
from ..engine import Plan, _require_cuda
from .base import Environment, EnvState, _rng

_F32 = torch.float32


@dataclasses.dataclass
class BatchedState:
    states: list
    _owner: "BatchedEnv"

    def env_state(self, i) -> EnvState:
        self._owner._close()
        return self.states[i]

    @property
    def time(self):
        return self._owner._time

    @property
    def energy_center(self):
        return self._owner._centers


class BatchedEnv:
    def __init__(self, env: Environment, batch_size: int, device="cuda"):
        if batch_size < 1:
            raise ValueError("batch_size must be >= 1")
        self.env = env
        self.batch_size = int(batch_size)
        self.device = device
        self._plan = None
        self._open = False
        self._state = None

    def reset(self, keys=None):
        """(observations (B, 5N), state).  ``keys``: one key per environment, or None."""
        _require_cuda()
        self._close()
        B = self.batch_size
        keys = [None] * B if keys is None else list(keys)
        if len(keys) != B:
            raise ValueError(f"{len(keys)} keys for a batch of {B}")
        env = self.env
        inits, centers = [], []
        for k in keys:
            rng = _rng(k)
            inits.append(env._init_state(rng))
            centers.append(env._sample_energy_center(rng))
        # one counter array and one centre array for the batch; each state holds views of them
        self._time = torch.zeros(B, dtype=torch.int32, device=self.device)
        self._centers = torch.as_tensor(np.stack(centers).astype(np.float32), device=self.device)
        states = []
        for i, init in enumerate(inits):
            dev = env._device_state(init, self.device)
            states.append(EnvState(dev, self._time[i], self._centers[i], dev.rest_lengths.clone(),
                                   dev.bending_rest_angles.clone(), np.arange(dev.N) % 3))
        d0 = states[0].device
        if self._plan is None:
            self._plan = Plan.for_states([s.device for s in states], [env.solver_config] * B, [env.dt] * B)
        self._d_rest = torch.zeros((B, d0.E), dtype=_F32, device=self.device)
        self._d_ang = torch.zeros((B, d0.B), dtype=_F32, device=self.device)
        self._noise = torch.zeros((B, 2), dtype=_F32, device=self.device) if env.energy_walk_std != 0.0 else None
        acts = [(self._d_rest[i], self._d_ang[i]) for i in range(B)]
        noises = [self._noise[i] if self._noise is not None else None for i in range(B)]
        self._table = env._table(states, acts, noises)
        self._state = BatchedState(states, self)
        self._observe(advance=False)
        return self._table["out"]["obs"].clone(), self._state

    def step(self, keys, state: BatchedState, actions: dict):
        """(observations (B, 5N), state, rewards (B,), dones (B,), info) for one step of
        every environment.  ``actions``: {"d_rest_length": (B, E), "d_bending_angle": (B, B_pairs)}."""
        if state is not self._state:
            raise ValueError("step() takes the state returned by this batch's reset()/step()")
        B = self.batch_size
        if actions is not None:
            for name, buf in (("d_rest_length", self._d_rest), ("d_bending_angle", self._d_ang)):
                a = actions.get(name)
                if a is None:
                    buf.zero_()
                else:
                    buf.copy_(torch.as_tensor(a, dtype=_F32).reshape(buf.shape))
        else:
            self._d_rest.zero_()
            self._d_ang.zero_()
        if self._noise is not None:
            g = np.random.default_rng(None if keys is None else [int(np.asarray(k).ravel()[-1]) for k in keys])
            self._noise.copy_(torch.as_tensor(g.standard_normal((B, 2)).astype(np.float32)))
        lib = _lib.load()
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        ptr = ctypes.c_void_p(self._table["ptr"])
        _lib.check(lib.mc_env_act(ptr, B, stream))
        if not self._open:
            self._plan.begin([s.device for s in state.states])
            self._open = True
        self._plan.advance(1, last=True)
        self._observe(advance=True)
        out = self._table["out"]
        info = {"steps": state.time.clone(), "energy_center": state.energy_center.clone()}
        return out["obs"].clone(), state, out["reward"].clone(), out["done"].bool(), info

    def fitness_per_creature(self, state: BatchedState):
        self._observe(advance=False)
        return self._table["out"]["fitness"].clone()

    def _observe(self, advance):
        lib = _lib.load()
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        _lib.check(lib.mc_env_observe(ctypes.c_void_p(self._table["ptr"]), self.batch_size, int(bool(advance)),
                                      stream))

    def _close(self):
        """Write the populations back to the states' f_grid (mc_rollout_end)."""
        if self._open:
            self._plan.end()
            self._open = False
