"""Benchmark: lattice MLUPS of the microcosmos per-step physics hot path on B200.

Workload (default): the plain method at scale — one 1024x1024 periodic D2Q9 TRT fp32
lattice, 256 filaments x 64 nodes (Poisson-disk centres, min sep 8), steric FFT on the
same grid, 4-point IB, 20 PBD iterations, curvature actuation amp ~U(0.1,0.3),
period ~U(100,400), dt = 0.01.  A "step" is one simulate.step of that instance.

  value      MLUPS = cells x steps / device time, state resident in HBM, L2 flushed
             (256 MiB written, then 256 MiB read) between timed steps, each step timed
             with CUDA events
  e2e        MLUPS through the reference-facing run() API with pinned host inputs and
             host outputs (H2D of the state, the rollout, D2H of the final state)
  roofline   the dense stream+collide kernel: 72 B/cell algorithmic traffic per launch
             / its CUDA-event duration (L2 flushed before every step)
  cpu_baseline  the numpy restatement (oracle) on a bounded sample of the same workload

--impl reference times the reference's CPU path (its numpy restatement, since JAX is not
installed) on the same workload, metric and unit.

Multi-GPU: rollouts do not exchange data, so N GPUs run N independent replicas
("scaling": "weak"); value = total cells x steps / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

# more hardware work queues, so that the served rollouts' streams overlap (set before CUDA starts)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "lattice MLUPS & rollouts/s batched vs plain on 1 B200; p50/p99 latency"
BYTES_PER_CELL = 72  # 9 fp32 populations read + 9 written per cell per step
QUEUE_SPIN_CYCLES = 1_000_000  # device spin after each L2 flush (about 0.5 ms at 1.965 GHz)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="scale", choices=["scale", "small"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-steps", type=int, default=100)
    ap.add_argument("--batch-rollouts", type=int, default=256)
    ap.add_argument("--batch-steps", type=int, default=100)
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--serve-requests", type=int, default=96)
    ap.add_argument("--serve-rate", type=float, default=200.0)
    ap.add_argument("--serve-plain-sample", type=int, default=12)
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--grad-steps", type=int, default=2000)
    ap.add_argument("--no-grad", action="store_true")
    ap.add_argument("--gym-envs", type=int, default=256)
    ap.add_argument("--gym-steps", type=int, default=50)
    ap.add_argument("--no-gym", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=0,
                    help="steps of the end-to-end run() call (0: the workload's own rollout length)")
    return ap.parse_args()


def workload(name, seed):
    from microcosmos_b200 import scenarios
    if name == "scale":
        return scenarios.config_scale(seed=seed), {
            "workload": "plain method at scale: 1024x1024 periodic D2Q9 TRT fp32, 256 filaments x 64 nodes "
                        "(Poisson-disk, min sep 8), steric FFT 1024^2, 4-pt IB, 20 PBD iterations, dt 0.01",
            "grid": [1024, 1024], "filaments": 256, "nodes_per_filament": 64, "rollout_steps": 10000}
    return scenarios.config_small(seed=seed), {
        "workload": "plain method small: 128x128 periodic D2Q9 TRT fp32, 4 filaments x 32 nodes, dt 0.01",
        "grid": [128, 128], "filaments": 4, "nodes_per_filament": 32, "rollout_steps": 1000}


def measured_peaks():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def committed_traffic(kernel, H, W):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, scaled to H*W."""
    p = os.path.join(HERE, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    e = d.get(kernel)
    if not e:
        return None
    return float(e["dram_bytes_per_launch"]) * (H * W) / float(e["cells"])


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled DURING a timed region.

    NVML is polled from a thread every ~2 ms (the timed regions here last milliseconds to
    seconds; nvidia-smi's loop mode samples every 100 ms at best); without NVML it falls
    back to ``nvidia-smi --query-gpu=... -lms 100``.  Read-only: no clock or GPU setting
    is changed."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))

    def __init__(self, gpu_index, period_s=0.0002):
        self.gpu = gpu_index
        self.period = period_s
        self.proc = None
        self.samples = []  # (sm_mhz, max_mhz, reason bits)
        self.lines = []
        self._stop = threading.Event()
        self._nvml = None

    def _handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            p = torch.cuda.get_device_properties(self.gpu)
            bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.gpu)

    def start(self):
        try:
            self._nvml = self._handle()
        except Exception:
            self._nvml = None
        if self._nvml is not None:
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _poll(self):
        nv, h = self._nvml
        mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        while not self._stop.is_set():
            try:
                t = time.perf_counter()
                self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)), mx,
                                     int(nv.nvmlDeviceGetCurrentClocksEventReasons(h)), t))
            except Exception:
                break
            time.sleep(self.period)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self, window=None):
        """Summary of the samples; with window = (t0, t1) (time.perf_counter values) only the
        samples taken inside it."""
        self._stop.set()
        if self._nvml is not None:
            self.t.join(timeout=5)
            smp = [x for x in self.samples if window is None or window[0] <= x[3] <= window[1]]
            sm = [x[0] for x in smp]
            reasons = sorted({n for x in smp for n, b in self.REASONS if x[2] & b})
            return {"sm_mhz": float(np.median(sm)) if sm else None,
                    "sm_max_mhz": self.samples[0][1] if self.samples else None,
                    "reasons": reasons, "samples": len(sm),
                    "source": f"NVML, polled every {self.period * 1e3:g} ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi -lms 100"}


def cpu_baseline(sc, cfg_steps_budget_s=15.0):
    """Oracle (numpy restatement, single process) on a bounded sample of the workload."""
    from oracle import ref_numpy as O
    s = O.state_from_scenario(sc)
    act = (sc.act_c, sc.act_amp, sc.act_omega, sc.act_phase)
    cfg = O.Config()
    t0 = time.perf_counter()
    s, _ = O.simulate(s, cfg, 0.01, 1, act=act, t0=0)
    t1 = time.perf_counter() - t0
    n = int(max(1, min(50, cfg_steps_budget_s / max(t1, 1e-6))))
    t0 = time.perf_counter()
    s, _ = O.simulate(s, cfg, 0.01, n, act=act, t0=1)
    dt = time.perf_counter() - t0
    cells = sc.H * sc.W
    return {"value": cells * n / dt / 1e6, "unit": "MLUPS", "cores": 1, "kind": "port",
            "sample": f"{n} steps of the {sc.H}x{sc.W} workload after 1 warm-up step (numpy restatement, not JAX; "
                      f"{dt:.1f} s)", "seconds_per_step": dt / n}


def batch_section(args, flush):
    """Batching configuration: an evolutionary-search population of uneven rollouts (side
    ~U{128,192,256,384,512}, filaments ~U{1..32}, nodes/filament ~U{16..128}, amplitude
    ~N(0.2, 0.05), 2000-step rollouts) stepped together as one plan (every kernel launched
    once per step for the whole population, steps replayed from CUDA graphs), against the
    plain path: the same rollouts as one plan each, run one after another.  Rollouts/s are
    for 2000-step rollouts, from the per-step device time of a bounded number of steps."""
    import torch
    from microcosmos_b200 import baseline_config, scenarios
    from microcosmos_b200.engine import Actuation, DeviceState, Plan
    cfg = baseline_config()
    scs = scenarios.config_batch(args.batch_rollouts, seed=0)
    cells = sum(s.H * s.W for s in scs)
    nodes = sum(s.N for s in scs)
    sts = [DeviceState.from_scenario(s) for s in scs]
    acts = [Actuation.from_scenario(s) for s in scs]
    from microcosmos_b200 import autotune
    tuned, tune_ms = autotune.tune(sts, [cfg] * len(scs), [0.01] * len(scs), actuations=acts, steps=10, warmup=4)
    shape = tuned["lbm_shape"]
    plan = Plan.for_states(sts, [cfg] * len(scs), [0.01] * len(scs), lbm_shape=shape,
                           fft_values=tuned["fft_values"], bin_threads=tuned["bin_threads"],
                           bin_sort_capacity=tuned["bin_sort_capacity"], ib_cluster=tuned["ib_cluster"])
    stream = torch.cuda.current_stream()
    plan.begin(sts, actuations=acts)
    plan.advance(6, use_graph=True)
    K = args.batch_steps
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    torch.cuda.synchronize()
    for i in range(K):
        flush()
        ev[i][0].record(stream)
        plan.advance(1, use_graph=True, last=(i == K - 1))
        ev[i][1].record(stream)
    plan.end()
    torch.cuda.synchronize()
    t_batch = sum(a.elapsed_time(b) for a, b in ev) / K  # ms per step, whole population
    flags = plan.read_flags()
    # dense-pass share of a batched step (per-kernel events, sequential schedule)
    plan.profile(True)
    plan.begin(sts, actuations=acts)
    plan.advance(1, use_graph=False)
    plan.profile_reset()
    for i in range(10):
        flush()
        plan.advance(1, use_graph=False, last=(i == 9))
    plan.end()
    torch.cuda.synchronize()
    prof = plan.profile_read()
    plan.profile(False)
    lbm_ms = prof["lbm"][0] / max(prof["lbm"][1], 1)
    del plan
    # the same population with the direct-convolution steric filter (opt-in: ~6e-7 rel-L2 from the FFT's)
    plan = Plan.for_states(sts, [cfg] * len(scs), [0.01] * len(scs), lbm_shape=shape, steric_method=2,
                           fft_values=tuned["fft_values"])
    plan.begin(sts, actuations=acts)
    plan.advance(4, use_graph=True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    plan.advance(K, use_graph=True, last=True)
    e1.record(stream)
    plan.end()
    torch.cuda.synchronize()
    t_direct = e0.elapsed_time(e1) / K
    del plan
    # plain: one plan per rollout, run sequentially (a bounded subset of the population)
    nplain = min(len(scs), 32)
    t_plain = 0.0
    for s, st, a in zip(scs[:nplain], sts[:nplain], acts[:nplain]):
        p1 = Plan.for_states([st], [cfg], [0.01])
        p1.begin([st], actuations=[a])
        p1.advance(4, use_graph=True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        p1.advance(K, use_graph=True, last=True)
        e1.record(stream)
        p1.end()
        torch.cuda.synchronize()
        t_plain += e0.elapsed_time(e1) / K  # ms per step of this rollout
        del p1
    t_plain_pop = t_plain / nplain * len(scs)  # ms per step, population run sequentially
    steps = 2000
    return {
        "workload": f"{len(scs)} uneven rollouts (side U{{128..512}}, 1-32 filaments x 16-128 nodes), "
                    f"{cells} cells, {nodes} nodes in total; rollouts/s for 2000-step rollouts",
        "steps_timed": K, "ms_per_step": t_batch, "mlups": cells / (t_batch / 1e3) / 1e6,
        "node_steps_per_s": nodes / (t_batch / 1e3),
        "rollouts_per_s": len(scs) / (t_batch / 1e3 * steps),
        "plain_rollouts_per_s": len(scs) / (t_plain_pop / 1e3 * steps),
        "plain_sample": f"{nplain} rollouts, one plan each, {K} graph-launched steps each",
        "speedup_vs_plain": t_plain_pop / t_batch,
        "direct_steric_filter": {"ms_per_step": t_direct, "mlups": cells / (t_direct / 1e3) / 1e6,
                                 "note": "opt-in steric_method=2, no L2 flush between steps"},
        "autotune": {"dense_pass_shape": {"cells_per_lane": shape[0], "rows_per_cta": shape[1]},
                     "fft_values_per_thread": tuned["fft_values"], "bin_threads": tuned["bin_threads"],
                     "bin_sort_capacity": tuned["bin_sort_capacity"], "ib_cluster_ctas": tuned["ib_cluster"],
                     "ms_per_step_by_candidate": tune_ms},
        "lbm_ms_per_launch": lbm_ms,
        "kernels_ms_per_step": {k: ms / 10 for k, (ms, n) in prof.items() if n},
        "lbm_frac_of_peak": BYTES_PER_CELL * cells / (lbm_ms / 1e3) / 1e9 / measured_peaks()[0],
        "roofline_frac_mlups": cells / (t_batch / 1e3) / 1e6 / (measured_peaks()[0] * 1e9 / BYTES_PER_CELL / 1e6),
        "flags_nonzero": int(sum(1 for f in flags if f)),
        "l2": "flushed before every timed step (256 MiB written, then 256 MiB read)"}


def serve_section(args):
    """Serving configuration: a seeded Poisson stream (mean ``--serve-rate`` requests/s) of
    rollouts with grid side ~U{64..1024} step 64, filaments ~U{1..128}, nodes/filament
    ~U{16..128}, steps ~U{500..5000}, 20% marked as asking for gradients, served by the
    continuous-batching server (admission by a 180 GB budget; every admitted forward
    rollout advances in shared epochs, one ragged plan per epoch of at most 200
    graph-replayed steps, ending where the nearest rollout finishes, over the rollouts with
    the least remaining work up to 8 M lattice cells; up to 16 gradient
    jobs at once beside them).  Latency = completion (state back on the host) minus
    arrival, wall clock.  The plain path runs a sample of the same requests one after
    another, one plan each."""
    import torch
    from microcosmos_b200 import baseline_config, serve
    cfg = baseline_config()
    reqs = serve.poisson_requests(args.serve_requests, args.serve_rate, seed=0)
    be = serve.CudaBackend(cfg, dt=0.01, grad_workers=16)
    # warm the allocator and the module (one tiny request); not part of the measurement
    serve.run_plain(be, serve.poisson_requests(1, 1.0, seed=99, sides=(64,), filaments=(1, 1), nodes=(16, 16),
                                               steps=(8, 8)))
    torch.cuda.synchronize()
    # epochs take the rollouts with the least remaining work first, up to 8 M lattice cells
    # (measured on this stream: p50 23.5-24.3 s against 26.9-29.8 s when every rollout joins
    # every epoch, at the same throughput)
    srv = serve.Server(be, hbm_budget_bytes=180e9, max_active=256, chunk=200, keep_state=False,
                       epoch_cells=8 << 20)
    t0 = time.perf_counter()
    res = srv.run(reqs, realtime=True)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    summ = serve.summarize(res, wall, grad_ids=[r.rid for r in reqs if r.want_grad])
    # the plain path: requests one after another, each alone (forward, or forward + adjoint for a
    # gradient request); timed on a sample of each kind and scaled by cell-steps to the stream
    def plain_rate(sample):
        if not sample:
            return None, 0.0
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        serve.run_plain(be, sample)
        torch.cuda.synchronize()
        dt_ = time.perf_counter() - t1
        return sum(r.scenario.H * r.scenario.W * r.steps for r in sample) / dt_, dt_
    fwd_reqs = [r for r in reqs if not r.want_grad]
    grad_reqs = [r for r in reqs if r.want_grad]
    k = min(args.serve_plain_sample, len(fwd_reqs))
    kg = min(max(1, args.serve_plain_sample // 4), len(grad_reqs))
    rate_f, t_f = plain_rate(fwd_reqs[:k])
    rate_g, t_g = plain_rate(grad_reqs[:kg])
    t_plain_all = sum(r.scenario.H * r.scenario.W * r.steps for r in fwd_reqs) / rate_f
    if grad_reqs:
        t_plain_all += sum(r.scenario.H * r.scenario.W * r.steps for r in grad_reqs) / rate_g
    cs_all = sum(r.scenario.H * r.scenario.W * r.steps for r in reqs)
    plain_rps = len(reqs) / t_plain_all
    return dict(summ, workload=f"{len(reqs)} Poisson requests at {args.serve_rate:g}/s (side U{{64..1024}} step 64, "
                                f"1-128 filaments x 16-128 nodes, 500-5000 steps); {cs_all} cell-steps",
                grad_note="gradient requests: forward with checkpoints + adjoint of the mean centre-of-mass x "
                          "displacement w.r.t. actuation and initial positions, on worker threads",
                flags_nonzero=int(sum(1 for r in res if r.flags)),
                peak_active=srv.peak_active, peak_bytes=srv.peak_bytes, epochs=srv.epochs,
                plain_mlups=cs_all / t_plain_all / 1e6, plain_rollouts_per_s=plain_rps,
                plain_sample=f"first {k} forward requests ({t_f:.2f} s) and first {kg} gradient requests "
                             f"({t_g:.2f} s), each alone and in turn, scaled by cell-steps to the stream",
                speedup_vs_plain=summ["rollouts_per_s"] / plain_rps,
                roofline_frac_mlups=summ["mlups"] / (measured_peaks()[0] * 1e9 / BYTES_PER_CELL / 1e6),
                timing="wall clock from the first arrival to the last completion")


def grad_section(args):
    """Differentiation configuration: 256x256 lattice, 8 filaments x 48 nodes, actuation amp
    0.2 and period 200 steps; loss = mean centre-of-mass x displacement after
    ``--grad-steps`` steps; gradients w.r.t. the per-bending-pair rest curvature offsets
    (act_c, 46 x 8), actuation amplitude and phase, through the torch autograd binding
    (forward with ceil(sqrt(T)) checkpoints, backward = segment recompute + adjoint
    kernels).  Timed with CUDA events around the forward call and around backward()."""
    import torch
    from microcosmos_b200 import baseline_config, scenarios
    from microcosmos_b200.autodiff import rollout
    cfg = baseline_config()
    sc = scenarios.make_scenario(256, 256, 8, 48, seed=0, amp=0.2, period=200.0)
    dev = "cuda"

    def leaf(a, grad=True):
        t = torch.as_tensor(np.asarray(a), device=dev).clone()
        return t.requires_grad_(grad)

    def once(T):
        pos, vel, th, f = leaf(sc.position), leaf(sc.velocity), leaf(sc.theta), leaf(sc.f_grid)
        L0, kb, ra = leaf(sc.rest_lengths, False), leaf(sc.bending_stiffness, False), leaf(sc.bending_rest_angles, False)
        c, amp, ph = leaf(sc.act_c), leaf(sc.act_amp), leaf(sc.act_phase)
        om = leaf(sc.act_omega, False)
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        torch.cuda.synchronize()
        e[0].record()
        out = rollout(pos, vel, th, f, L0, kb, ra, sc.pairs, sc.bending_pairs, cfg, 0.01, T, actuation=(c, amp, om, ph))
        loss = out[0][:, 0].mean() - pos[:, 0].mean()
        e[1].record()
        loss.backward()
        e[2].record()
        torch.cuda.synchronize()
        grads = {"act_c": c.grad, "act_amp": amp.grad, "act_phase": ph.grad, "position": pos.grad, "f_grid": f.grad}
        return float(loss.item()), e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2]), grads

    once(8)  # module load and allocator warm-up
    T = args.grad_steps
    loss, fwd_ms, bwd_ms, grads = once(T)
    cells = 256 * 256
    S = int(np.ceil(np.sqrt(T)))
    return {"workload": f"256x256, 8 filaments x 48 nodes, {T} steps, loss = mean COM x displacement; "
                        f"grads w.r.t. act_c/amp/phase ({sc.bending_pairs.shape[0]} bending pairs), initial state",
            "steps": T, "checkpoint_every": S, "loss": loss, "forward_ms": fwd_ms, "backward_ms": bwd_ms,
            "gradient_ms": fwd_ms + bwd_ms, "forward_mlups": cells * T / (fwd_ms / 1e3) / 1e6,
            "gradient_mlups": cells * T / ((fwd_ms + bwd_ms) / 1e3) / 1e6,
            "grad_norms": {k: float(v.norm().item()) for k, v in grads.items()},
            "all_finite": bool(all(torch.isfinite(v).all().item() for v in grads.values())),
            "reference_jax_grad": "unavailable (JAX is not installed); gradients are checked against the numpy "
                                  "VJP oracle and float64 central differences in the tests"}


def gym_section(args):
    """Gym caller of the step (gym/base.py:163-196): ``--gym-envs`` LineEnv environments
    (the reference's defaults: 128x128, 16 nodes, PBD_SCHEME; energy source on) stepped
    together by BatchedEnv (action kernel, one batched physics step, observation/reward
    kernel), against one Environment stepped alone (functional step: state copy, action,
    rollout call, observation).  Random actions, resident on the device."""
    import torch
    from microcosmos_b200.gym import BatchedEnv, LineEnv
    env = LineEnv(energy_amplitude=1.0, max_steps=10 ** 9)
    B, K = args.gym_envs, args.gym_steps
    g = torch.Generator(device="cuda").manual_seed(0)
    acts = [{"d_rest_length": 0.1 * torch.randn((B, env.num_edges), generator=g, device="cuda"),
             "d_bending_angle": 0.2 * torch.randn((B, env.num_bending_pairs), generator=g, device="cuda")}
            for _ in range(K)]
    benv = BatchedEnv(env, B)
    _, st = benv.reset(list(range(B)))
    for t in range(3):
        benv.step(None, st, acts[t])
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for t in range(K):
        obs, st, rew, done, _ = benv.step(None, st, acts[t])
    e1.record()
    torch.cuda.synchronize()
    batch_ms = e0.elapsed_time(e1)
    mean_reward = float(rew.mean().item())
    _, s1 = env.reset(0)
    one = [{k: v[0] for k, v in a.items()} for a in acts]
    for t in range(3):
        _, s1, _, _, _ = env.step(None, s1, one[t])
    torch.cuda.synchronize()
    e0.record()
    for t in range(K):
        _, s1, _, _, _ = env.step(None, s1, one[t])
    e1.record()
    torch.cuda.synchronize()
    single_ms = e0.elapsed_time(e1)
    H, W = env.grid_shape
    return {"workload": f"{B} x LineEnv (128x128, 16 nodes, PBD_SCHEME, energy source on), {K} steps, random actions",
            "batched_env_steps_per_s": B * K / (batch_ms / 1e3), "batched_ms_per_step": batch_ms / K,
            "batched_mlups": B * H * W * K / (batch_ms / 1e3) / 1e6,
            "single_env_steps_per_s": K / (single_ms / 1e3), "single_ms_per_step": single_ms / K,
            "speedup_vs_single": (B * K / batch_ms) / (K / single_ms), "mean_reward_last_step": mean_reward}


def config_json(cfgj, ws):
    """The ``config`` object of both arms' JSON lines."""
    return dict(cfgj, l2="flushed before every timed step (256 MiB written, then 256 MiB read); each step timed "
                         "alone with CUDA events",
                parallelism=f"replicas x{ws}", dt=0.01,
                timed="device-resident: one graph-launched simulate.step per event pair")


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _ref_replica(job):
    """One CPU process: warm-up, then timed steps of its own copy of the workload for about
    `budget_s` seconds (numpy restatement of the reference step, one thread)."""
    name, steps_max, warmup, budget_s = job
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    sys.path.insert(0, HERE)
    from oracle import ref_numpy as O
    sc, _ = workload(name, 0)
    s = O.state_from_scenario(sc)
    act = (sc.act_c, sc.act_amp, sc.act_omega, sc.act_phase)
    cfg = O.Config()
    s, _ = O.simulate(s, cfg, 0.01, warmup, act=act)
    t0 = time.perf_counter()
    k = 0
    while k < steps_max and (k == 0 or time.perf_counter() - t0 < budget_s):
        s, _ = O.simulate(s, cfg, 0.01, 1, act=act, t0=warmup + k)
        k += 1
    return k, time.perf_counter() - t0, sc.H * sc.W


def run_reference(args):
    """The reference's CPU path on the host cores: JAX is not installed, so the numpy
    restatement of the reference step runs instead, as independent replicas of the
    workload on all usable cores (one single-threaded process each, bounded by memory),
    each for about 45 s; value = all replicas' cell updates / the slowest replica's time."""
    ws, rank, _ = dist_setup()
    if rank != 0:
        return
    import multiprocessing as mp
    sc, cfgj = workload(args.config, 0)
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    per_replica = 48 * sc.H * sc.W * 4 + (256 << 20)  # state, tapes of the numpy step and interpreter
    try:
        import psutil
        avail = psutil.virtual_memory().available
        procs = max(1, min(cores, int(0.6 * avail // per_replica)))
    except Exception:
        procs = max(1, min(cores, 8))
    w = max(1, min(args.warmup, 2))
    jobs = [(args.config, max(1, args.steps), w, 45.0)] * procs
    with mp.get_context("spawn").Pool(procs) as pool:
        res = pool.map(_ref_replica, jobs)
    k_tot = sum(k for k, _, _ in res)
    dt = max(t for _, t, _ in res)
    cells = res[0][2]
    v = cells * k_tot / dt / 1e6
    sample = (f"{procs} single-threaded replicas x {min(k for k, _, _ in res)}-{max(k for k, _, _ in res)} steps of "
              f"the {sc.H}x{sc.W} workload ({dt:.0f} s; numpy restatement of the reference step: JAX is not "
              f"installed, so the reference itself cannot run)")
    k_min = min(k for k, _, _ in res)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "MLUPS", "n_gpus": args.gpus,
        # every replica runs the same K steps (up to its time budget); steps and ms_per_step
        # describe one replica, value sums all replicas' cell updates over the slowest one's time
        "steps": k_min, "warmup": w, "ms_per_step": dt / k_min * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded numpy.random, the benchmark configurations' shapes)",
        "config": config_json(cfgj, args.gpus), "replicas": procs, "replica_steps_total": k_tot,
        "node_steps_per_s": k_tot * sc.N / dt,
        "cpu_baseline": {"value": v, "unit": "MLUPS", "cores": procs, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    import torch.distributed as dist
    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if ws > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    from microcosmos_b200 import baseline_config
    from microcosmos_b200.engine import Actuation, DeviceState, Plan
    from microcosmos_b200.simulate import run as api_run
    from microcosmos_b200.structs import Edges, Fields, Nodes

    from microcosmos_b200.replicas import job_totals, replica_seed
    sc, cfgj = workload(args.config, replica_seed(0, rank))
    cfg = baseline_config()
    H, W = sc.H, sc.W
    cells = H * W
    st = DeviceState.from_scenario(sc)
    act = Actuation.from_scenario(sc)
    plan = Plan.for_states([st], [cfg], [0.01])
    # L2 flush between timed steps: write a 256 MiB buffer (evicts the rollout's data), then
    # read another 256 MiB buffer, so that the write's dirty lines are written back here and
    # not during the next timed step.  Then a spin kernel that touches no memory holds the
    # stream for about 0.5 ms while the host enqueues the step behind it, so the step's
    # events and kernels run back to back on the device instead of waiting for the host's
    # launch calls.
    flush_w = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    flush_r = torch.zeros(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def flush():
        flush_w.zero_()
        flush_r.sum()
        torch.cuda._sleep(QUEUE_SPIN_CYCLES)
    stream = torch.cuda.current_stream()

    # ---------------- device-resident timed region
    clocks = ClockSampler(local)
    clocks.start()
    plan.begin([st], actuations=[act])
    plan.advance(args.warmup, use_graph=True)
    K = args.steps
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    # last_launch_count accumulates over the begin/advance calls of one rollout
    launches0 = plan.last_launch_count()
    tw0 = time.perf_counter()
    for i in range(K):
        flush()
        ev[i][0].record(stream)
        plan.advance(1, use_graph=True, last=(i == K - 1))
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop(window=(tw0, time.perf_counter()))
    if ws > 1:
        dist.barrier()
    launches = plan.last_launch_count() - launches0
    plan.end()
    torch.cuda.synchronize()
    t_ms = sum(a.elapsed_time(b) for a, b in ev)
    # job time = max over ranks, job work = sum over ranks (replicas: no data exchange)
    t_ms, job_cell_steps = job_totals(t_ms, cells * K, device="cuda")
    flags = plan.read_flags()

    # ---------------- per-kernel event pass (roofline), L2 flushed before each step
    st2 = DeviceState.from_scenario(sc)
    plan.profile(True)
    plan.begin([st2], actuations=[act])
    plan.advance(2, use_graph=False)
    plan.profile_reset()
    P = args.profile_steps
    for i in range(P):
        flush()
        plan.advance(1, use_graph=False, last=(i == P - 1))
    plan.end()
    torch.cuda.synchronize()
    prof = plan.profile_read()
    plan.profile(False)
    step_kernel_ms = sum(ms for ms, n in prof.values())
    per_step = {k: {"ms_per_launch": ms / n, "launches_per_step": n / P, "share": ms / step_kernel_ms}
                for k, (ms, n) in prof.items() if n}
    lbm_ms, lbm_n = prof["lbm"]
    lbm_s = lbm_ms / lbm_n / 1e3
    achieved = BYTES_PER_CELL * cells / lbm_s / 1e9
    peak, peak_kind = measured_peaks()
    traffic = committed_traffic("lbm", H, W)

    # ---------------- end to end through the reference-facing API (host buffers)
    def pinned(a):
        return torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    hn = Nodes(position=pinned(sc.position), velocity=pinned(sc.velocity), color_bend=pinned(np.zeros(sc.N, np.float32)),
               debug_vector=pinned(np.zeros((sc.N, 2), np.float32)))
    he = Edges(pairs=sc.pairs, theta=pinned(sc.theta), rest_lengths=pinned(sc.rest_lengths),
               bending_pairs=sc.bending_pairs, bending_rest_angles=pinned(sc.bending_rest_angles),
               bending_stiffness=pinned(sc.bending_stiffness))
    hf = Fields(grid_shape=(H, W), steric=pinned(sc.steric), fluid_velocity=pinned(sc.fluid_velocity),
                f_grid=pinned(sc.f_grid))
    actn = (sc.act_c, sc.act_amp, sc.act_omega, sc.act_phase)
    outs = {k: torch.empty(s, dtype=torch.float32).pin_memory() for k, s in
            (("position", (sc.N, 2)), ("velocity", (sc.N, 2)), ("theta", (sc.E,)), ("f_grid", (9, H, W)),
             ("steric", (H, W)), ("fluid_velocity", (2, H, W)))}
    api_run(hn, he, hf, 0.01, 4, cfg, actuation=actn)  # plan/graph warm-up
    torch.cuda.synchronize()
    # one call of the workload's own rollout length (10,000 steps at scale): the state goes
    # in from pinned host memory once and the final state comes back once, as a caller of
    # simulate/run with that rollout pays it
    Ke = args.e2e_steps or cfgj["rollout_steps"]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks_e = ClockSampler(local, period_s=0.01)
    clocks_e.start()
    e0.record(stream)
    n_, e_, f_ = api_run(hn, he, hf, 0.01, Ke, cfg, actuation=actn)
    outs["position"].copy_(n_.position)
    outs["velocity"].copy_(n_.velocity)
    outs["theta"].copy_(e_.theta)
    outs["f_grid"].copy_(f_.f_grid)
    outs["steric"].copy_(f_.steric)
    outs["fluid_velocity"].copy_(f_.fluid_velocity)
    e1.record(stream)
    torch.cuda.synchronize()
    clk_e = clocks_e.stop()
    te = e0.elapsed_time(e1)
    h2d = sum(int(np.asarray(a).nbytes) for a in (sc.position, sc.velocity, sc.theta, sc.rest_lengths,
                                                   sc.bending_rest_angles, sc.bending_stiffness, sc.f_grid,
                                                   sc.steric, sc.fluid_velocity))
    d2h = sum(int(v.numel() * 4) for v in outs.values())
    te, job_cell_steps_e = job_totals(te, cells * Ke, device="cuda")

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(sc)
    batch = None
    if ws == 1 and not args.no_batch:
        batch = batch_section(args, flush)
    graded = None
    if ws == 1 and not args.no_grad:
        graded = grad_section(args)
    served = None
    if ws == 1 and not args.no_serve:
        served = serve_section(args)
    gym = None
    if ws == 1 and not args.no_gym:
        gym = gym_section(args)

    if rank == 0:
        value = job_cell_steps / (t_ms / 1e3) / 1e6
        out = {
            "metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": ws, "steps": K, "warmup": args.warmup,
            "ms_per_step": t_ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded numpy.random, the benchmark configurations' shapes)",
            "config": config_json(cfgj, ws),
            "node_steps_per_s": job_cell_steps / cells * sc.N / (t_ms / 1e3),
            "e2e": {"value": job_cell_steps_e / (te / 1e3) / 1e6, "unit": "MLUPS",
                    "h2d_bytes_per_step": h2d / Ke, "d2h_bytes_per_step": d2h / Ke, "steps_per_call": Ke,
                    "h2d_bytes_per_call": h2d, "d2h_bytes_per_call": d2h, "ms": te,
                    "node_steps_per_s": job_cell_steps_e / cells * sc.N / (te / 1e3),
                    "clocks": clk_e,
                    "api": "microcosmos_b200.simulate.run, one call of the workload's rollout length "
                           "(pinned host inputs -> host outputs)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "k_lbm (fused pull stream + TRT/Guo collide), %d cells per lane x %d rows per CTA"
                                   % plan.lbm_shape(),
                         "algorithmic_bytes_per_launch": BYTES_PER_CELL * cells,
                         "ms_per_launch": lbm_s * 1e3},
            "cpu_baseline": cpu,
            "clocks": clk,
            "gpu_launches": int(launches),
            "kernels": per_step,
            "flags": flags,
            "batch": batch,
            "serve": served,
            "grad": graded,
            "gym": gym,
            "step_kernel_ms": step_kernel_ms / P,
        }
        print(json.dumps(out))
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
