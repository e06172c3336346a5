"""Continuous-batching rollout server.

Requests (a rollout of any grid and filament size, a step count) arrive over time.  The
server admits a request as soon as a slot is free and its device memory fits in the HBM
budget, keeps its lattice and rod state resident on the device, and advances every
admitted rollout in chunks of steps (CUDA-graph replays) on its own CUDA stream, so the
work of rollouts that arrive while others run overlaps with theirs on the device.  A
finished rollout's state is copied back, its memory returns to the budget, and waiting
requests take its place.

Each rollout owns its plan, workspace and stream, and every kernel is deterministic (no
float atomics), so a rollout's result is bit-for-bit the same whatever else is in flight.

More hardware queues than CUDA's default of 8 let more rollouts overlap: set
``CUDA_DEVICE_MAX_CONNECTIONS`` (e.g. 32) before the process first touches the GPU.

Requests that ask for gradients get the gradient of the mean centre-of-mass x
displacement of their final state with respect to the actuation (c, amplitude, phase of
every bending pair) and the initial positions: the forward rollout with checkpoints and
the adjoint run as one job on a worker thread (own stream, own gradient plan, see
``microcosmos_b200.autodiff``), overlapping with the chunked forward rollouts.

The scheduler is written against a small backend interface (``bytes_needed``, ``start``,
``advance``, ``inflight``, ``finish``) so that its admission and ordering logic is tested
without a GPU; ``CudaBackend`` is the device implementation over
``microcosmos_b200.engine`` and ``microcosmos_b200.autodiff``.
"""
from __future__ import annotations

import collections
import concurrent.futures
import ctypes
import dataclasses
import time
from typing import Any, Callable

import numpy as np


@dataclasses.dataclass
class Request:
    rid: int
    arrival: float            # seconds after the start of the run
    scenario: Any             # microcosmos_b200.scenarios.Scenario
    steps: int
    want_grad: bool = False


@dataclasses.dataclass
class Result:
    rid: int
    arrival: float
    admitted: float
    done: float
    steps: int
    cells: int
    state: dict | None = None
    flags: int = 0

    @property
    def latency(self):
        return self.done - self.arrival


class CudaBackend:
    """Device backend: one bound plan + workspace + CUDA stream per admitted rollout;
    gradient requests run as one job each on a thread pool.  A gradient job's reverse steps
    are chains of small dependent kernels that leave most of the GPU idle, so several jobs
    in flight overlap well: on the serving workload 8 workers finished the stream in 32 s
    against 45 s with 2 (4: 34 s, 16: 35 s)."""

    def __init__(self, cfg, dt=0.01, device="cuda", grad_workers=8):
        self.cfg = cfg
        self.dt = float(dt)
        self.device = device
        self.pool = concurrent.futures.ThreadPoolExecutor(max_workers=max(1, int(grad_workers)))

    def bytes_needed(self, req: Request) -> int:
        """Device bytes of the rollout: its plan workspace (mc_plan_workspace_bytes, or
        mc_grad_plan_workspace_bytes for a gradient request) plus state."""
        from . import _lib
        from .engine import mc_config
        sc = req.scenario
        lib = _lib.load()
        pairs = np.ascontiguousarray(sc.pairs, np.int32).reshape(-1, 2)
        bp = np.ascontiguousarray(sc.bending_pairs, np.int32).reshape(-1, 2)
        fh, fw = (int(v) for v in np.shape(sc.f_grid)[-2:])  # the fluid lattice (may differ from H, W)
        dims = _lib.McDims(sc.H, sc.W, sc.position.shape[0], pairs.shape[0], bp.shape[0], fh, fw)
        cfg = mc_config(self.cfg)
        h = ctypes.c_void_p()
        if req.want_grad:
            _lib.check(lib.mc_grad_plan_create(ctypes.byref(dims), ctypes.byref(cfg), self.dt,
                                               pairs.ctypes.data_as(_lib.c_int_p), bp.ctypes.data_as(_lib.c_int_p),
                                               int(req.steps), 0, ctypes.byref(h)))
            try:
                ws = int(lib.mc_grad_plan_workspace_bytes(h))
            finally:
                lib.mc_grad_plan_destroy(h)
        else:
            dt = ctypes.c_float(self.dt)
            pp = (_lib.c_int_p * 1)(pairs.ctypes.data_as(_lib.c_int_p))
            bb = (_lib.c_int_p * 1)(bp.ctypes.data_as(_lib.c_int_p))
            _lib.check(lib.mc_plan_create(1, ctypes.byref(dims), ctypes.byref(cfg), ctypes.byref(dt), pp, bb,
                                          ctypes.byref(h)))
            try:
                ws = int(lib.mc_plan_workspace_bytes(h))
            finally:
                lib.mc_plan_destroy(h)
        N = sc.position.shape[0]
        state = 4 * (11 * fh * fw + sc.H * sc.W + 8 * N + 4 * bp.shape[0]) + 256
        return ws + state

    def _grad_job(self, req: Request):
        import torch
        from .autodiff import GradPlan
        from .engine import Actuation, DeviceState
        stream = torch.cuda.Stream(device=self.device)
        with torch.cuda.stream(stream):
            sc = req.scenario
            st = DeviceState.from_scenario(sc, device=self.device)
            act = Actuation.from_scenario(sc, device=self.device)
            plan = GradPlan(sc.H, sc.W, st.N, sc.pairs, sc.bending_pairs, self.cfg, self.dt, req.steps,
                            device=self.device)
            plan.forward(st, act)
            seed = torch.zeros((st.N, 2), dtype=torch.float32, device=self.device)
            seed[:, 0] = 1.0 / st.N  # d(mean x of the final positions)
            g = plan.backward(seed)
            g["position"][:, 0] -= 1.0 / st.N  # the loss subtracts the initial mean x
            state = st.host()
            state["grad"] = {k: v.cpu().numpy() for k, v in g.items()}
            stream.synchronize()
            plan.close()
        return state, 0

    def start(self, req: Request):
        import torch
        from .engine import Actuation, DeviceState, Plan
        if req.want_grad:
            return {"future": self.pool.submit(self._grad_job, req)}
        stream = torch.cuda.Stream(device=self.device)
        with torch.cuda.stream(stream):
            st = DeviceState.from_scenario(req.scenario, device=self.device)
            act = Actuation.from_scenario(req.scenario, device=self.device)
            plan = Plan.for_states([st], [self.cfg], [self.dt], device=self.device)
            plan.begin([st], actuations=[act], stream=stream.cuda_stream)
        return {"stream": stream, "state": st, "act": act, "plan": plan, "events": collections.deque()}

    def advance(self, h, steps: int, last: bool):
        import torch
        if "future" in h:
            return  # the gradient job runs all its steps at once
        h["plan"].advance(steps, use_graph=True, last=last, stream=h["stream"].cuda_stream)
        ev = torch.cuda.Event()
        ev.record(h["stream"])
        h["events"].append(ev)

    def inflight(self, h) -> int:
        """Chunks issued and not finished yet."""
        if "future" in h:
            return 0 if h["future"].done() else 1
        q = h["events"]
        while q and q[0].query():
            q.popleft()
        return len(q)

    def finish(self, h):
        import torch
        if "future" in h:
            return h["future"].result()
        with torch.cuda.stream(h["stream"]):
            h["plan"].end(stream=h["stream"].cuda_stream)
            flags = h["plan"].read_flags()[0]
            state = h["state"].host()
        h["stream"].synchronize()
        h["plan"].close()
        return state, flags


class Server:
    """Admission by memory budget and slot count, chunked stepping, overlap across rollouts.

    ``depth`` chunks per rollout are kept queued on its stream, so a stream never drains
    while the host services the others.
    """

    def __init__(self, backend, hbm_budget_bytes: float = 180e9, max_active: int = 16, chunk: int = 200,
                 depth: int = 2, clock: Callable[[], float] | None = None, sleep: Callable[[float], None] | None = None,
                 keep_state: bool = True):
        if chunk < 1 or depth < 1 or max_active < 1:
            raise ValueError("chunk, depth and max_active must be >= 1")
        self.backend = backend
        self.budget = float(hbm_budget_bytes)
        self.max_active = int(max_active)
        self.chunk = int(chunk)
        self.depth = int(depth)
        self.clock = clock or time.perf_counter
        self.sleep = sleep or time.sleep
        self.keep_state = keep_state
        self.peak_active = 0
        self.peak_bytes = 0

    def run(self, requests: list[Request], realtime: bool = True) -> list[Result]:
        """Serve ``requests``: arrival times are seconds from the call when ``realtime``,
        otherwise every request is present at the start.  Returns results ordered by id."""
        need = {r.rid: int(self.backend.bytes_needed(r)) for r in requests}
        for r in requests:
            if need[r.rid] > self.budget:
                raise ValueError(f"request {r.rid} needs {need[r.rid]} bytes of device memory, more than the "
                                 f"whole budget of {int(self.budget)}")
            if r.steps < 0:
                raise ValueError(f"request {r.rid} asks for a negative step count")
        pending = collections.deque(sorted(requests, key=lambda r: (r.arrival, r.rid)))
        active = {}   # rid -> [request, handle, steps issued, admitted at]
        used = 0
        results = []
        t0 = self.clock()

        def now():
            return self.clock() - t0

        while pending or active:
            # admit, in arrival order, every request that has arrived and fits
            while pending and (not realtime or pending[0].arrival <= now()):
                r = pending[0]
                if len(active) >= self.max_active or used + need[r.rid] > self.budget:
                    break
                pending.popleft()
                used += need[r.rid]
                active[r.rid] = [r, self.backend.start(r), 0, now()]
                self.peak_active = max(self.peak_active, len(active))
                self.peak_bytes = max(self.peak_bytes, used)
            busy = False
            for rid in list(active):
                r, h, issued, adm = active[rid]
                q = self.backend.inflight(h)
                if issued >= r.steps:
                    if q:
                        busy = True
                        continue
                    state, flags = self.backend.finish(h)
                    used -= need[rid]
                    results.append(Result(rid=rid, arrival=r.arrival, admitted=adm, done=now(), steps=r.steps,
                                          cells=r.scenario.H * r.scenario.W,
                                          state=state if self.keep_state else None, flags=flags))
                    del active[rid]
                    continue
                busy = busy or q > 0
                while q < self.depth and issued < r.steps:
                    n = min(self.chunk, r.steps - issued)
                    issued += n
                    self.backend.advance(h, n, last=issued >= r.steps)
                    q += 1
                active[rid][2] = issued
            if not active and pending and realtime:
                wait = pending[0].arrival - now()
                if wait > 0:
                    self.sleep(min(wait, 1e-3))
            elif busy:
                self.sleep(0)
        return sorted(results, key=lambda x: x.rid)


def run_plain(backend, requests: list[Request]):
    """The plain path for comparison: each request alone, one after another, on one stream."""
    out = []
    for r in requests:
        h = backend.start(r)
        if r.steps:
            backend.advance(h, r.steps, last=True)
        state, flags = backend.finish(h)
        out.append((r.rid, state, flags))
    return out


def summarize(results: list[Result], wall_s: float, grad_ids=()) -> dict:
    """Throughput and latency; MLUPS counts forward cell updates of every request (a
    gradient request's adjoint work is not counted)."""
    lat = np.array([r.latency for r in results]) if results else np.zeros(1)
    cell_steps = sum(r.cells * r.steps for r in results)
    out = {"requests": len(results), "wall_s": wall_s, "rollouts_per_s": len(results) / wall_s,
           "mlups": cell_steps / wall_s / 1e6, "p50_latency_s": float(np.percentile(lat, 50)),
           "p99_latency_s": float(np.percentile(lat, 99)), "mean_latency_s": float(lat.mean())}
    g = set(grad_ids)
    if g:
        gl = np.array([r.latency for r in results if r.rid in g])
        fl = np.array([r.latency for r in results if r.rid not in g])
        out["grad_requests"] = len(gl)
        if len(gl):
            out["grad_p50_latency_s"] = float(np.percentile(gl, 50))
        if len(fl):
            out["forward_p50_latency_s"] = float(np.percentile(fl, 50))
    return out


def poisson_requests(n, rate_per_s, seed=0, sides=None, filaments=(1, 128), nodes=(16, 128), steps=(500, 5000),
                     grad_fraction=0.2, actuation_mean=0.2, actuation_std=0.05):
    """A seeded Poisson request stream: exponential inter-arrival times at ``rate_per_s``,
    grid side uniform over ``sides`` (default 64..1024 in steps of 64), filaments and
    nodes per filament uniform over the given inclusive ranges, step count uniform over
    ``steps``, actuation amplitude ~ N(actuation_mean, actuation_std), and a fraction of
    requests marked as asking for gradients."""
    from . import scenarios
    rng = np.random.default_rng(seed)
    sides = list(sides) if sides is not None else list(range(64, 1025, 64))
    t = 0.0
    out = []
    for i in range(n):
        t += float(rng.exponential(1.0 / rate_per_s))
        side = int(rng.choice(sides))
        F = int(rng.integers(filaments[0], filaments[1] + 1))
        nn = int(rng.integers(nodes[0], nodes[1] + 1))
        amp = float(rng.normal(actuation_mean, actuation_std))
        sc = scenarios.make_scenario(side, side, F, nn, rng=rng, amp=amp,
                                     period=float(rng.uniform(100.0, 400.0)))
        out.append(Request(rid=i, arrival=t, scenario=sc, steps=int(rng.integers(steps[0], steps[1] + 1)),
                           want_grad=bool(rng.uniform() < grad_fraction)))
    return out
