"""Benchmark driver (not part of the library): run a named workload for a fixed number of
steps, untimed, for external profilers (ncu launch lists and captures).

    python benchmarks/workload.py --workload scale --steps 5
    python benchmarks/workload.py --workload scale --side 2048 --steps 3
    python benchmarks/workload.py --workload batch --rollouts 64 --steps 10
    python benchmarks/workload.py --workload grad --steps 20

Workloads (seeded synthetic inputs):
  scale  one 1024x1024 lattice, 256 filaments x 64 nodes (Poisson-disk placement);
         --side picks another lattice side with the same nodes (2048: populations larger
         than the L2 cache, for DRAM counters of the dense pass)
  small  one 128x128 lattice, 4 filaments x 32 nodes
  batch  a population of uneven rollouts (side U{128..512}, 1-32 filaments x 16-128 nodes)
         as one plan with the library's default launch shapes
  grad   the 256x256, 8 x 48 differentiation workload (--grad-size picks another): forward with
         checkpoints + backward
  gym    --rollouts LineEnv environments (128x128, 16 nodes) stepped together by BatchedEnv
Steps are launched directly (no CUDA graph) unless --graph is given, so that every kernel
launch is visible to a profiler.
"""
from __future__ import annotations

import argparse
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="scale", choices=["scale", "small", "batch", "grad", "gym"])
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--rollouts", type=int, default=64)
    ap.add_argument("--graph", action="store_true")
    ap.add_argument("--side", type=int, default=1024, help="lattice side of the scale workload")
    ap.add_argument("--grad-size", type=int, nargs=3, default=(256, 8, 48), metavar=("SIDE", "FILAMENTS", "NODES"),
                    help="lattice side, filaments and nodes per filament of the grad workload")
    ap.add_argument("--lbm-shape", type=int, nargs=2, default=None, metavar=("CELLS_PER_LANE", "ROWS"),
                    help="dense-pass tile shape (default: the library's)")
    ap.add_argument("--lbm-stages", type=int, default=None,
                    help="staged dense pass with this many row bands in flight per CTA (0: tiled)")
    a = ap.parse_args(argv)
    import numpy as np
    import torch

    from microcosmos_b200 import baseline_config, scenarios
    from microcosmos_b200.engine import Actuation, DeviceState, Plan
    cfg = baseline_config()
    if a.workload == "grad":
        from microcosmos_b200.autodiff import GradPlan
        side, nf, nn = a.grad_size
        sc = scenarios.make_scenario(side, side, nf, nn, seed=0, amp=0.2, period=200.0)
        st = DeviceState.from_scenario(sc)
        plan = GradPlan(sc.H, sc.W, st.N, sc.pairs, sc.bending_pairs, cfg, 0.01, a.steps)
        plan.forward(st, Actuation.from_scenario(sc))
        seed = torch.zeros((st.N, 2), dtype=torch.float32, device="cuda")
        seed[:, 0] = 1.0 / st.N
        g = plan.backward(seed)
        torch.cuda.synchronize()
        print("grad ok", float(g["act_amp"].norm()))
        return
    if a.workload == "gym":
        from microcosmos_b200.gym import BatchedEnv, LineEnv
        env = LineEnv(energy_amplitude=1.0, max_steps=10 ** 9)
        benv = BatchedEnv(env, a.rollouts)
        _, st = benv.reset(list(range(a.rollouts)))
        g = torch.Generator(device="cuda").manual_seed(0)
        for _ in range(a.warmup + a.steps):
            act = {"d_rest_length": 0.1 * torch.randn((a.rollouts, env.num_edges), generator=g, device="cuda"),
                   "d_bending_angle": 0.2 * torch.randn((a.rollouts, env.num_bending_pairs), generator=g,
                                                        device="cuda")}
            obs, st, rew, done, _ = benv.step(None, st, act)
        torch.cuda.synchronize()
        print("gym ok", a.rollouts, "environments, mean reward", float(rew.mean()))
        return
    if a.workload == "batch":
        scs = scenarios.config_batch(a.rollouts, seed=0)
    elif a.workload == "small":
        scs = [scenarios.config_small(seed=0)]
    elif a.side == 1024:
        scs = [scenarios.config_scale(seed=0)]
    else:
        scs = [scenarios.make_scenario(a.side, a.side, 256, 64, seed=0, placement="poisson", min_sep=8.0)]
    sts = [DeviceState.from_scenario(s) for s in scs]
    acts = [Actuation.from_scenario(s) for s in scs]
    plan = Plan.for_states(sts, [cfg] * len(scs), [0.01] * len(scs),
                           lbm_shape=tuple(a.lbm_shape) if a.lbm_shape else None, lbm_stages=a.lbm_stages)
    plan.begin(sts, actuations=acts)
    plan.advance(a.warmup, use_graph=a.graph)
    plan.advance(a.steps, use_graph=a.graph, last=True)
    plan.end()
    torch.cuda.synchronize()
    print(a.workload, "ok", len(scs), "rollouts", int(sum(s.H * s.W for s in scs)), "cells",
          "flags", int(np.count_nonzero(plan.read_flags())))


if __name__ == "__main__":
    main()
