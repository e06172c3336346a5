"""Continuous-batching rollout server.

Requests (a rollout of any grid and filament size, a step count) arrive over time.  The
server admits a request as soon as a slot is free and its device memory fits in the HBM
budget and keeps its lattice and rod state resident on the device.  All admitted forward
rollouts then advance TOGETHER: the server runs "epochs", each one ragged plan over the
current set of rollouts (every kernel launched once per step for the whole set, the steps
replayed from CUDA graphs), for as many steps as the set's nearest finish allows (at most
``chunk``).  At every epoch boundary finished rollouts leave (their state is copied back and
their memory returns to the budget) and newly admitted ones join, so requests that arrive
while others run share the device's launches with them.  Up to ``depth`` epochs are queued
on the serving stream, so the device does not wait for the host between epochs.

Every kernel is deterministic (no float atomics), a rollout's result does not depend on
the other rollouts of a plan, and splitting a rollout into epochs (begin / advance / end
with the actuation clock continued) gives the same bits as one call, so a rollout's result
is bit-for-bit the same alone and in the mix.

Requests that ask for gradients get the gradient of the mean centre-of-mass x
displacement of their final state with respect to the actuation (c, amplitude, phase of
every bending pair) and the initial positions: the forward rollout with checkpoints and
the adjoint run as one job on a worker thread (own stream, own gradient plan, see
``microcosmos_b200.autodiff``), overlapping with the batched forward epochs.

The scheduler is written against a small backend interface (``bytes_needed``, ``load``,
``launch_epoch``, ``epoch_done``, ``collect``, ``release_epoch``, ``start_grad``,
``grad_done``, ``grad_result``) so that its admission and ordering logic is tested without
a GPU; ``CudaBackend`` is the device implementation over ``microcosmos_b200.engine`` and
``microcosmos_b200.autodiff``.
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
    """Device backend.  Forward rollouts: device-resident state per request, one ragged
    plan per epoch over the epoch's rollouts, all on one serving stream.  Gradient requests
    run as one job each on a thread pool (own stream, own gradient plan): a gradient job's
    reverse steps are chains of small dependent kernels that leave most of the GPU idle, so
    several jobs in flight overlap well (beside the epochs, 16 workers measured better than
    8: 32.2 vs 34.6 s for the 96-request serving stream)."""

    def __init__(self, cfg, dt=0.01, device="cuda", grad_workers=16):
        import torch
        self.cfg = cfg
        self.dt = float(dt)
        self.device = device
        self.pool = concurrent.futures.ThreadPoolExecutor(max_workers=max(1, int(grad_workers)))
        # epochs on the highest stream priority, gradient jobs on the default (lowest): when
        # both have work ready the forward rollouts' CTAs are scheduled first (the values
        # outside the device's range are clamped to it)
        self.stream = torch.cuda.Stream(device=device, priority=-100)
        self.copy_stream = torch.cuda.Stream(device=device)  # results back to the host

    # a forward rollout's workspace exists once per epoch plan alive at a time: up to two
    # queued (Server.depth) and one completed but not yet released
    EPOCH_PLANS = 3

    def bytes_needed(self, req: Request) -> int:
        """Device bytes of the rollout: its state plus its plan workspace
        (mc_plan_workspace_bytes, counted EPOCH_PLANS times for a forward rollout; or
        mc_grad_plan_workspace_bytes for a gradient request)."""
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
        return (ws if req.want_grad else self.EPOCH_PLANS * ws) + state

    # ---------------------------------------------------------------- forward rollouts
    def load(self, req: Request):
        """Upload the request's state; it stays resident until collected."""
        import torch
        from .engine import Actuation, DeviceState
        with torch.cuda.stream(self.stream):
            st = DeviceState.from_scenario(req.scenario, device=self.device)
            sc = req.scenario
            act = Actuation.from_scenario(sc, device=self.device)
        return {"state": st, "act": act, "flags": 0}

    def launch_epoch(self, handles, steps: int, t0s):
        """Enqueue `steps` steps of every rollout in `handles` as one plan (rollout i continues
        its actuation clock at t0s[i]) on the serving stream; returns the epoch handle."""
        import torch
        from .engine import Actuation, Plan
        stream = self.stream
        with torch.cuda.stream(stream):
            sts = [h["state"] for h in handles]
            acts = [None if h["act"] is None else dataclasses.replace(h["act"], t0=int(t)) for h, t in zip(handles, t0s)]
            plan = Plan.for_states(sts, [self.cfg] * len(sts), [self.dt] * len(sts), device=self.device)
            plan.begin(sts, actuations=acts, stream=stream.cuda_stream)
            plan.advance(int(steps), use_graph=True, last=True, stream=stream.cuda_stream)
            plan.end(stream=stream.cuda_stream)
            ev = torch.cuda.Event()
            ev.record(stream)
        return {"plan": plan, "event": ev, "handles": handles, "flags_read": False}

    def epoch_done(self, e) -> bool:
        return e["event"].query()

    def _read_epoch_flags(self, e):
        if not e["flags_read"]:
            import torch
            with torch.cuda.stream(self.copy_stream):
                fl = e["plan"].read_flags()
            for h, f in zip(e["handles"], fl):
                h["flags"] |= int(f)
            e["flags_read"] = True

    def collect(self, h, e=None):
        """State and flags of a finished rollout (after its last epoch `e` completed)."""
        import torch
        if e is not None:
            self._read_epoch_flags(e)
        with torch.cuda.stream(self.copy_stream):
            state = h["state"].host()
        return state, h["flags"]

    def release_epoch(self, e):
        self._read_epoch_flags(e)
        e["plan"].close()

    # ---------------------------------------------------------------- gradient requests
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

    def start_grad(self, req: Request):
        return self.pool.submit(self._grad_job, req)

    def grad_done(self, h) -> bool:
        return h.done()

    def grad_result(self, h):
        return h.result()


@dataclasses.dataclass
class _Epoch:
    handle: Any
    members: list
    finishing: list


class Server:
    """Admission by memory budget and slot count; forward rollouts advance together in
    epochs (one ragged plan each), at most ``chunk`` steps per epoch and ``depth`` epochs
    queued; gradient requests run beside them."""

    def __init__(self, backend, hbm_budget_bytes: float = 180e9, max_active: int = 256, chunk: int = 200,
                 depth: int = 2, clock: Callable[[], float] | None = None, sleep: Callable[[float], None] | None = None,
                 keep_state: bool = True, epoch_cells: int | None = None):
        """``epoch_cells``: None advances every admitted forward rollout in each epoch; a
        number makes each epoch take the rollouts with the least remaining work (remaining
        steps x lattice cells) first, up to that many lattice cells in total (at least one
        rollout), so that short requests finish early while long ones wait for room."""
        if chunk < 1 or depth < 1 or max_active < 1:
            raise ValueError("chunk, depth and max_active must be >= 1")
        if epoch_cells is not None and epoch_cells < 1:
            raise ValueError("epoch_cells must be >= 1")
        self.epoch_cells = epoch_cells
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
        self.epochs = 0

    def run(self, requests: list[Request], realtime: bool = True) -> list[Result]:
        """Serve ``requests``: arrival times are seconds from the call when ``realtime``,
        otherwise every request is present at the start.  Returns results ordered by id."""
        be = self.backend
        need = {r.rid: int(be.bytes_needed(r)) for r in requests}
        for r in requests:
            if need[r.rid] > self.budget:
                raise ValueError(f"request {r.rid} needs {need[r.rid]} bytes of device memory, more than the "
                                 f"whole budget of {int(self.budget)}")
            if r.steps < 0:
                raise ValueError(f"request {r.rid} asks for a negative step count")
        pending = collections.deque(sorted(requests, key=lambda r: (r.arrival, r.rid)))
        fwd = {}      # rid -> [request, handle, steps issued, admitted at]
        grads = {}    # rid -> [request, job, admitted at]
        queued = collections.deque()  # epochs in flight, oldest first
        used = 0
        results = []
        t0 = self.clock()

        def now():
            return self.clock() - t0

        def done(r, adm, state, flags):
            nonlocal used
            used -= need[r.rid]
            results.append(Result(rid=r.rid, arrival=r.arrival, admitted=adm, done=now(), steps=r.steps,
                                  cells=r.scenario.H * r.scenario.W,
                                  state=state if self.keep_state else None, flags=flags))

        while pending or fwd or grads or queued:
            # admit, in arrival order, every request that has arrived and fits
            while pending and (not realtime or pending[0].arrival <= now()):
                r = pending[0]
                if len(fwd) + len(grads) >= self.max_active or used + need[r.rid] > self.budget:
                    break
                pending.popleft()
                used += need[r.rid]
                if r.want_grad:
                    grads[r.rid] = [r, be.start_grad(r), now()]
                else:
                    fwd[r.rid] = [r, be.load(r), 0, now()]
                    if r.steps == 0:
                        state, flags = be.collect(fwd[r.rid][1])
                        done(r, fwd[r.rid][3], state, flags)
                        del fwd[r.rid]
                self.peak_active = max(self.peak_active, len(fwd) + len(grads))
                self.peak_bytes = max(self.peak_bytes, used)
            progressed = False
            # retire completed epochs, oldest first: their finished rollouts leave
            while queued and be.epoch_done(queued[0].handle):
                e = queued.popleft()
                for rid in e.finishing:
                    r, h, _, adm = fwd.pop(rid)
                    state, flags = be.collect(h, e.handle)
                    done(r, adm, state, flags)
                be.release_epoch(e.handle)
                progressed = True
            for rid in list(grads):
                r, job, adm = grads[rid]
                if be.grad_done(job):
                    state, flags = be.grad_result(job)
                    done(r, adm, state, flags)
                    del grads[rid]
                    progressed = True
            # queue the next epoch over every admitted rollout with steps left
            if len(queued) < self.depth:
                members = self._epoch_members(fwd)
                if members:
                    n = min([self.chunk] + [fwd[rid][0].steps - fwd[rid][2] for rid in members])
                    eh = be.launch_epoch([fwd[rid][1] for rid in members], n, [fwd[rid][2] for rid in members])
                    for rid in members:
                        fwd[rid][2] += n
                    finishing = [rid for rid in members if fwd[rid][2] >= fwd[rid][0].steps]
                    queued.append(_Epoch(eh, members, finishing))
                    self.epochs += 1
                    progressed = True
            if progressed:
                continue
            if not fwd and not grads and not queued and pending and realtime:
                wait = pending[0].arrival - now()
                if wait > 0:
                    self.sleep(min(wait, 1e-3))
            else:
                self.sleep(0)
        return sorted(results, key=lambda x: x.rid)


    def _epoch_members(self, fwd):
        """The admitted forward rollouts with steps left that the next epoch advances."""
        cand = [rid for rid, (r, h, issued, _) in fwd.items() if issued < r.steps]
        if self.epoch_cells is None:
            return cand

        def cells(rid):
            sc = fwd[rid][0].scenario
            return sc.H * sc.W

        cand.sort(key=lambda rid: ((fwd[rid][0].steps - fwd[rid][2]) * cells(rid), rid))
        members, total = [], 0
        for rid in cand:
            if members and total + cells(rid) > self.epoch_cells:
                continue
            members.append(rid)
            total += cells(rid)
        return members


def run_plain(backend, requests: list[Request]):
    """The plain path for comparison: each request alone, one after another (a forward
    request as one single-rollout epoch, a gradient request as its gradient job)."""
    out = []
    for r in requests:
        if r.want_grad:
            state, flags = backend.grad_result(backend.start_grad(r))
        else:
            h = backend.load(r)
            e = backend.launch_epoch([h], r.steps, [0]) if r.steps else None
            if e is not None:
                while not backend.epoch_done(e):
                    time.sleep(0)
            state, flags = backend.collect(h, e)
            if e is not None:
                backend.release_epoch(e)
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
