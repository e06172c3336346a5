"""Autotuner for the launch shapes of a plan.

Three kernels have a free shape:
  * the dense stream+collide pass: each CTA covers 32 x cells_per_lane columns (1, 2 or 4
    cells per thread, vector loads/stores) by rows_per_cta rows (4, 8, 16 or 32 tried;
    up to 4 warps per CTA, each looping over rows_per_cta / 4 rows);
  * the power-of-two FFT kernels of the steric filter: each thread holds 4, 8 or 16
    values in registers (more values: fewer instructions per value; fewer: more threads);
  * the tile kernel that sorts the IB and cloud-in-cell contributions: 128 or 256 threads
    per CTA, and 512 or 1024 contributions per tile sorted in shared memory;
  * the IB iterations: separate launches per phase, or (when asked for) one thread-block
    cluster of CTAs per rollout with hardware cluster barriers between the phases.
Which shape is fastest depends on the rollout sizes of a plan (grid widths, how many CTAs
a step launches, how many tiles carry IB forcing), so the tuner times whole
graph-replayed steps of the actual plan on scratch copies of the states: first the FFT
shape, then the dense-pass shapes with the chosen FFT shape, then the tile-kernel CTA
size with both, then the IB iteration layout.  Results are cached per plan signature (sizes, configs, dt) for the life of the
process.  The dense-pass shape changes no result; the FFT shape changes the float32
rounding of the transform only.
"""
from __future__ import annotations

import dataclasses
import hashlib

import torch

from .engine import DeviceState, Plan

CELLS_PER_LANE = (1, 2, 4)
ROWS_PER_CTA = (4, 8, 16, 32)
FFT_VALUES = (4, 8, 16)
BIN_SHAPES = ((128, 2048), (256, 2048), (128, 1024), (256, 1024), (128, 512))  # (threads per CTA, shared sort capacity)
# CTAs per rollout cluster of the IB iterations tried besides the separate launches: none by
# default (measured slower everywhere: 1.886 vs 1.852 ms per 256-rollout batch step with 8
# CTAs, 0.228 vs 0.168 ms per 1024^2 step with 16); tune(ib_cluster=(...)) tries some
IB_CLUSTER = ()

_cache: dict[str, tuple[dict, dict]] = {}


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


def _time(scratch, cfgs, dts, actuations, steps, warmup, **shape):
    plan = Plan.for_states(scratch, cfgs, dts, **shape)
    plan.begin(scratch, actuations=actuations)
    plan.advance(warmup, use_graph=True)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    plan.advance(steps, use_graph=True, last=True)
    b.record()
    plan.end()
    torch.cuda.synchronize()
    plan.close()
    return a.elapsed_time(b) / steps


def tune(states, cfgs, dts, actuations=None, steps=10, warmup=4, shapes=None, fft_values=None, use_cache=True,
         ib_cluster=IB_CLUSTER):
    """Time ``steps`` graph-replayed steps of the plan for the candidate shapes and return
    ``(best, timings)``: best = {"lbm_shape": (cells_per_lane, rows_per_cta),
    "fft_values": 4 | 8 | 16, "bin_threads": 128 | 256, "bin_sort_capacity": 512 | 1024 | 2048},
    timings = {label: ms per step}.  The caller's states are
    not modified."""
    key = signature(states, cfgs, dts)
    if use_cache and key in _cache:
        return _cache[key]
    scratch = [_clone(s) for s in states]
    timings = {}
    steric = any(getattr(c, "enable_steric", True) for c in cfgs)
    fft_best = 0
    if steric:
        ft = {}
        for e in (fft_values or FFT_VALUES):
            ft[e] = _time(scratch, cfgs, dts, actuations, steps, warmup, fft_values=e)
            timings[f"fft{e}"] = ft[e]
        fft_best = min(ft, key=ft.get)
    lt = {}
    for shape in (shapes or candidates(states)):
        lt[shape] = _time(scratch, cfgs, dts, actuations, steps, warmup, lbm_shape=shape, fft_values=fft_best)
        timings[f"lbm{shape[0]}x{shape[1]}"] = lt[shape]
    lbm_best = min(lt, key=lt.get)
    # the shape candidates ran with the library's default tile kernel (128 threads, 1024 sorted in shared memory)
    bt = {(128, 1024): lt[lbm_best]}
    for t, cap in BIN_SHAPES:
        if (t, cap) not in bt:
            bt[(t, cap)] = _time(scratch, cfgs, dts, actuations, steps, warmup, lbm_shape=lbm_best,
                                 fft_values=fft_best, bin_threads=t, bin_sort_capacity=cap)
        timings[f"bins{t}x{cap}"] = bt[(t, cap)]
    bins_best = min(bt, key=bt.get)
    # the IB iterations: separate launches, or one cluster of CTAs per rollout
    ct = {0: bt[bins_best]}
    if any(getattr(c, "enable_fluid", True) for c in cfgs):
        for c in ib_cluster:
            ct[c] = _time(scratch, cfgs, dts, actuations, steps, warmup, lbm_shape=lbm_best, fft_values=fft_best,
                          bin_threads=bins_best[0], bin_sort_capacity=bins_best[1], ib_cluster=c)
            timings[f"ib_cluster{c}"] = ct[c]
    cl_best = min(ct, key=ct.get)
    best = {"lbm_shape": lbm_best, "fft_values": fft_best, "bin_threads": bins_best[0], "ib_cluster": cl_best,
            "bin_sort_capacity": bins_best[1]}
    _cache[key] = (best, timings)
    return best, timings


def tuned_plan(states, cfgs, dts, actuations=None, **kw) -> Plan:
    """A plan for these rollouts with the autotuned launch shapes."""
    best, _ = tune(states, cfgs, dts, actuations=actuations, **kw)
    return Plan.for_states(states, cfgs, dts, lbm_shape=best["lbm_shape"], fft_values=best["fft_values"],
                           bin_threads=best["bin_threads"], bin_sort_capacity=best["bin_sort_capacity"],
                           ib_cluster=best["ib_cluster"])
