"""Drop-in rollout API: ``simulate`` and ``step`` with the reference's signatures
(src/microcosmos/simulate.py:15-16, 37-38), computed by the sm_100a kernels.

Semantics follow the reference: inputs are not modified and new containers are
returned; ``simulate`` returns per-step timeseries of nodes and render fields (steric,
fluid_velocity, ``f_grid=None``).  Two keyword extensions:

* ``actuation=(c, amp, omega, phase)``: the caller-side curvature control evaluated on
  the device before each step, rest[b](t) = c + amp sin(omega t + phase);
* ``record_every``: keep every k-th step of the timeseries (1 = the reference's shape).

Plans (topology tables, workspace, CUDA graphs) are cached per (sizes, topology,
config, dt), as the reference's ``jax.jit`` caches per static arguments.
"""
from __future__ import annotations

import collections
import hashlib

import numpy as np
import torch

from .config import ConstraintSolverConfig
from .engine import Actuation, DeviceState, Plan, Record
from .structs import Edges, Fields, Nodes

_PLAN_CACHE: "collections.OrderedDict[tuple, Plan]" = collections.OrderedDict()
_PLAN_CACHE_MAX = 8


def _np(x, dtype):
    if isinstance(x, torch.Tensor):
        x = x.detach().cpu().numpy()
    return np.ascontiguousarray(x, dtype=dtype)


def _plan_for(state: DeviceState, cfg: ConstraintSolverConfig, dt: float) -> Plan:
    h = hashlib.sha1()
    h.update(state.pairs.tobytes())
    h.update(b"|")
    h.update(state.bending_pairs.tobytes())
    key = (state.H, state.W, state.lH, state.lW, state.N, h.hexdigest(), cfg, float(dt), torch.cuda.current_device())
    p = _PLAN_CACHE.get(key)
    if p is None:
        p = Plan.for_states([state], [cfg], [dt])
        _PLAN_CACHE[key] = p
        while len(_PLAN_CACHE) > _PLAN_CACHE_MAX:
            _PLAN_CACHE.popitem(last=False)
    else:
        _PLAN_CACHE.move_to_end(key)
    return p


def _state(nodes: Nodes, edges: Edges, fields: Fields) -> DeviceState:
    H, W = (int(v) for v in fields.grid_shape)
    f = fields.f_grid
    if len(tuple(f.shape)) != 3 or f.shape[0] != 9:
        raise ValueError("f_grid must be (9, h, w): the fluid lattice, grid_shape or its own (fluid.py:221-235)")
    return DeviceState.from_arrays(H, W, nodes.position, nodes.velocity, _np(edges.pairs, np.int32), edges.theta,
                                   edges.rest_lengths, _np(edges.bending_pairs, np.int32),
                                   edges.bending_rest_angles, edges.bending_stiffness, f, fields.steric,
                                   fields.fluid_velocity)


def _actuation(actuation):
    if actuation is None:
        return None
    if isinstance(actuation, Actuation):
        return actuation
    c, amp, omega, phase = actuation[:4]
    t0 = int(actuation[4]) if len(actuation) > 4 else 0
    dev = lambda a: torch.as_tensor(np.asarray(a, np.float32) if not isinstance(a, torch.Tensor) else a,
                                    dtype=torch.float32, device="cuda").contiguous()
    return Actuation(dev(c), dev(amp), dev(omega), dev(phase), t0)


def _like(x, device):
    return x if isinstance(x, torch.Tensor) else torch.as_tensor(np.asarray(x), device=device)


def run(nodes: Nodes, edges: Edges, fields: Fields, dt: float, num_steps: int,
        solver_config: ConstraintSolverConfig, *, actuation=None, use_graph: bool = True):
    """``num_steps`` steps returning only the final (nodes, edges, fields)."""
    st = _state(nodes, edges, fields)
    plan = _plan_for(st, solver_config, dt)
    act = _actuation(actuation)
    plan.rollout([st], num_steps, actuations=[act], use_graph=use_graph)
    return _outputs(st, nodes, edges, fields)


def _outputs(st: DeviceState, nodes: Nodes, edges: Edges, fields: Fields):
    dev = st.position.device
    n = Nodes(position=st.position, velocity=st.velocity, color_bend=_like(nodes.color_bend, dev),
              debug_vector=torch.zeros_like(st.position))
    e = Edges(pairs=_like(edges.pairs, dev), theta=st.theta, rest_lengths=st.rest_lengths,
              bending_pairs=_like(edges.bending_pairs, dev), bending_rest_angles=st.bending_rest_angles,
              bending_stiffness=st.bending_stiffness)
    f = Fields(grid_shape=tuple(fields.grid_shape), steric=st.steric, fluid_velocity=st.fluid_velocity,
               f_grid=st.f_grid, energy=fields.energy)
    return n, e, f


def step(nodes: Nodes, edges: Edges, fields: Fields, dt: float, solver_config: ConstraintSolverConfig):
    """One physics step (src/microcosmos/simulate.py:37-100)."""
    return run(nodes, edges, fields, dt, 1, solver_config, use_graph=False)


def simulate(nodes: Nodes, edges: Edges, fields: Fields, dt: float, num_steps: int,
             solver_config: ConstraintSolverConfig, *, actuation=None, record_every: int = 1,
             use_graph: bool = True):
    """Rollout with per-step recording (src/microcosmos/simulate.py:15-35).

    Returns (nodes_timeseries, fields_timeseries) with leading time axis of length
    ``num_steps // record_every``."""
    st = _state(nodes, edges, fields)
    plan = _plan_for(st, solver_config, dt)
    act = _actuation(actuation)
    rec = Record.allocate(st, num_steps, every=record_every, fields=True)
    plan.rollout([st], num_steps, actuations=[act], records=[rec], use_graph=use_graph)
    T = rec.position.shape[0]
    dev = st.position.device
    cb = _like(nodes.color_bend, dev)
    nodes_ts = Nodes(position=rec.position, velocity=rec.velocity,
                     color_bend=cb.unsqueeze(0).expand(T, *cb.shape).clone(),
                     debug_vector=torch.zeros_like(rec.position))
    fields_ts = Fields(grid_shape=tuple(fields.grid_shape), steric=rec.steric, fluid_velocity=rec.fluid_velocity,
                       f_grid=None, energy=None)
    return nodes_ts, fields_ts
