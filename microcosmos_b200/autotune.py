"""Autotuner for the tile shape of the dense stream+collide pass.

The dense pass is the one kernel whose CTA shape is a free choice: each CTA covers
32 x cells_per_lane columns (1, 2 or 4 cells per thread, vector loads/stores) by
rows_per_cta rows (2, 4 or 8).  Which shape is fastest depends on the rollout sizes of
a plan (grid widths, how many CTAs a step launches, how many tiles carry IB forcing),
so the tuner times whole graph-replayed steps of the actual plan for every candidate
on scratch copies of the states and keeps the fastest.  Results are cached per plan
signature (sizes, configs, dt) for the life of the process.  The shape changes no
result, only the time.
"""
from __future__ import annotations

import dataclasses
import hashlib

import torch

from .engine import DeviceState, Plan

CELLS_PER_LANE = (1, 2, 4)
ROWS_PER_CTA = (2, 4, 8)

_cache: dict[str, tuple[tuple[int, int], dict]] = {}


def signature(states, cfgs, dts) -> str:
    h = hashlib.sha1()
    for s, c, d in zip(states, cfgs, dts):
        h.update(repr((s.H, s.W, s.N, s.pairs.shape[0], s.bending_pairs.shape[0], float(d))).encode())
        h.update(repr(sorted(dataclasses.asdict(c).items()) if dataclasses.is_dataclass(c) else c).encode())
    return h.hexdigest()


def candidates(states):
    out = []
    for v in CELLS_PER_LANE:
        if all(s.W % v == 0 and s.W >= v for s in states):
            for r in ROWS_PER_CTA:
                out.append((v, r))
    return out


def _clone(s: DeviceState) -> DeviceState:
    return dataclasses.replace(s, **{f.name: getattr(s, f.name).clone() for f in dataclasses.fields(s)
                                     if isinstance(getattr(s, f.name), torch.Tensor)})


def tune(states, cfgs, dts, actuations=None, steps=10, warmup=4, shapes=None, use_cache=True):
    """Time ``steps`` graph-replayed steps of the plan for every candidate shape and return
    ``(best_shape, {shape: ms_per_step})``.  The caller's states are not modified."""
    key = signature(states, cfgs, dts)
    if use_cache and key in _cache:
        return _cache[key]
    scratch = [_clone(s) for s in states]
    timings = {}
    for shape in (shapes or candidates(states)):
        plan = Plan.for_states(scratch, cfgs, dts, lbm_shape=shape)
        plan.begin(scratch, actuations=actuations)
        plan.advance(warmup, use_graph=True)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        plan.advance(steps, use_graph=True, last=True)
        b.record()
        plan.end()
        torch.cuda.synchronize()
        timings[shape] = a.elapsed_time(b) / steps
        plan.close()
        del plan
    best = min(timings, key=timings.get)
    _cache[key] = (best, timings)
    return best, timings


def tuned_plan(states, cfgs, dts, actuations=None, **kw) -> Plan:
    """A plan for these rollouts with the autotuned dense-pass tile shape."""
    best, _ = tune(states, cfgs, dts, actuations=actuations, **kw)
    return Plan.for_states(states, cfgs, dts, lbm_shape=best)
