"""The continuous-batching server: admission and ordering on CPU with a fake backend, and
on the GPU that every rollout's result is the same alone and in the mix."""
import numpy as np
import pytest

from microcosmos_b200 import serve


class FakeBackend:
    """Epochs complete a fixed number of polls after they are queued; memory = cells.
    Checks the scheduler's invariants as it goes: an epoch never runs a rollout past its
    step count, every rollout's actuation clock continues where its last epoch stopped,
    and epochs complete in the order they were queued."""

    def __init__(self, polls_per_epoch=2, grad_polls=3):
        self.polls = polls_per_epoch
        self.grad_polls = grad_polls
        self.live = set()
        self.log = []
        self.epochs = []
        self.queue = []

    def bytes_needed(self, r):
        return r.scenario.H * r.scenario.W

    def load(self, r):
        self.live.add(r.rid)
        self.log.append(("start", r.rid))
        return {"rid": r.rid, "target": r.steps, "steps": 0}

    def launch_epoch(self, handles, n, t0s):
        assert n >= 1
        for h, t in zip(handles, t0s):
            assert t == h["steps"]
            h["steps"] += n
            assert h["steps"] <= h["target"]
        e = {"polls": self.polls, "rids": [h["rid"] for h in handles], "n": n}
        self.epochs.append(e)
        self.queue.append(e)
        return e

    def epoch_done(self, e):
        assert e is self.queue[0]  # retired oldest first
        e["polls"] -= 1
        if e["polls"] <= 0:
            self.queue.pop(0)
            return True
        return False

    def collect(self, h, e=None):
        assert h["steps"] == h["target"]
        self.live.discard(h["rid"])
        self.log.append(("finish", h["rid"]))
        return {"steps": h["steps"]}, 0

    def release_epoch(self, e):
        pass

    def start_grad(self, r):
        self.live.add(r.rid)
        self.log.append(("start", r.rid))
        return {"rid": r.rid, "polls": self.grad_polls, "steps": r.steps}

    def grad_done(self, h):
        h["polls"] -= 1
        return h["polls"] <= 0

    def grad_result(self, h):
        self.live.discard(h["rid"])
        self.log.append(("finish", h["rid"]))
        return {"steps": h["steps"], "grad": True}, 0


class _Sc:
    def __init__(self, side):
        self.H = self.W = side


class ManualClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        self.t += 1e-4
        return self.t

    def sleep(self, s):
        self.t += max(s, 1e-4)


def _reqs(sides, steps, arrivals=None, grads=None):
    arrivals = arrivals or [0.0] * len(sides)
    grads = grads or [False] * len(sides)
    return [serve.Request(rid=i, arrival=a, scenario=_Sc(s), steps=n, want_grad=g)
            for i, (s, n, a, g) in enumerate(zip(sides, steps, arrivals, grads))]


def test_every_request_completes_with_its_step_count():
    be = FakeBackend()
    reqs = _reqs([8, 16, 32, 8, 64], [0, 5, 250, 99, 100])
    clock = ManualClock()
    res = serve.Server(be, hbm_budget_bytes=1e9, chunk=40, clock=clock, sleep=clock.sleep).run(reqs)
    assert [r.rid for r in res] == [0, 1, 2, 3, 4]
    assert [r.state["steps"] for r in res] == [0, 5, 250, 99, 100]
    assert not be.live


def test_budget_and_slots_are_never_exceeded():
    sides = [30, 20, 10, 30, 25, 5, 40, 12]
    budget = 2000

    class Checking(FakeBackend):
        def load(self, r):
            h = super().load(r)
            live_bytes = sum(s * s for i, s in enumerate(sides) if i in self.live)
            assert live_bytes <= budget
            assert len(self.live) <= 3
            return h

    be = Checking()
    clock = ManualClock()
    srv = serve.Server(be, hbm_budget_bytes=budget, max_active=3, chunk=7, clock=clock, sleep=clock.sleep)
    res = srv.run(_reqs(sides, [20] * len(sides)))
    assert len(res) == len(sides)
    assert srv.peak_bytes <= budget and srv.peak_active <= 3


def test_admission_follows_arrival_and_overlaps_running_work():
    be = FakeBackend(polls_per_epoch=50)
    clock = ManualClock()
    reqs = _reqs([8, 8, 8], [400, 400, 400], arrivals=[0.0, 0.001, 0.002])
    res = serve.Server(be, hbm_budget_bytes=1e6, chunk=100, clock=clock, sleep=clock.sleep).run(reqs)
    starts = [rid for kind, rid in be.log if kind == "start"]
    assert starts == [0, 1, 2]
    # the later requests were admitted while the first was still running
    assert be.log.index(("start", 2)) < be.log.index(("finish", 0))
    assert all(r.admitted >= r.arrival for r in res)


def test_request_larger_than_budget_is_rejected():
    with pytest.raises(ValueError, match="budget"):
        serve.Server(FakeBackend(), hbm_budget_bytes=100).run(_reqs([11], [10]))


def test_rollouts_advance_together_in_epochs():
    """All admitted forward rollouts share each epoch; an epoch ends at the nearest finish
    (or after `chunk` steps), the finished rollouts leave and the others go on."""
    be = FakeBackend()
    clock = ManualClock()
    reqs = _reqs([8, 8, 8, 8], [30, 100, 100, 250])
    srv = serve.Server(be, hbm_budget_bytes=1e6, chunk=80, clock=clock, sleep=clock.sleep)
    res = srv.run(reqs, realtime=False)
    assert [r.state["steps"] for r in res] == [30, 100, 100, 250]
    ep = [(e["rids"], e["n"]) for e in be.epochs]
    assert ep[0] == ([0, 1, 2, 3], 30)       # ends where rollout 0 finishes
    assert ep[1] == ([1, 2, 3], 70)          # rollouts 1 and 2 finish together
    assert ep[2] == ([3], 80) and ep[3] == ([3], 70)
    assert srv.epochs == 4


def test_least_remaining_work_epochs():
    """With a cell budget per epoch, each epoch takes the rollouts with the least remaining
    work (steps left x cells) up to the budget: the short requests finish first, every
    request still completes with its step count, and no epoch exceeds the budget unless it
    holds a single rollout."""
    be = FakeBackend()
    clock = ManualClock()
    # cells: 64, 64, 256, 1024; remaining work 64*300, 64*40, 256*40, 1024*20
    reqs = _reqs([8, 8, 16, 32], [300, 40, 40, 20])
    srv = serve.Server(be, hbm_budget_bytes=1e6, chunk=50, clock=clock, sleep=clock.sleep, epoch_cells=400)
    res = srv.run(reqs, realtime=False)
    assert [r.state["steps"] for r in res] == [300, 40, 40, 20]
    cells = {0: 64, 1: 64, 2: 256, 3: 1024}
    for e in be.epochs:
        assert len(e["rids"]) == 1 or sum(cells[r] for r in e["rids"]) <= 400
    assert be.epochs[0]["rids"] == [1, 2, 0]  # 2,560 < 10,240 < 19,200; rollout 3 (20,480) waits
    done = [rid for kind, rid in be.log if kind == "finish"]
    assert done.index(1) < done.index(3) and done.index(2) < done.index(3)
    with pytest.raises(ValueError):
        serve.Server(be, epoch_cells=0)


def test_gradient_requests_run_beside_the_epochs():
    be = FakeBackend(grad_polls=5)
    clock = ManualClock()
    reqs = _reqs([8, 16, 8], [40, 60, 10], grads=[False, True, False])
    res = serve.Server(be, hbm_budget_bytes=1e6, chunk=25, clock=clock, sleep=clock.sleep).run(reqs, realtime=False)
    assert [r.state["steps"] for r in res] == [40, 60, 10]
    assert res[1].state.get("grad") is True
    assert all(1 not in e["rids"] for e in be.epochs)
    assert not be.live


def test_summary_percentiles():
    res = [serve.Result(rid=i, arrival=0.0, admitted=0.0, done=float(i + 1), steps=10, cells=100) for i in range(100)]
    s = serve.summarize(res, wall_s=10.0)
    assert s["requests"] == 100 and s["rollouts_per_s"] == 10.0
    assert abs(s["p50_latency_s"] - 50.5) < 1e-9 and s["p99_latency_s"] > 99.0
    assert s["mlups"] == 100 * 100 * 10 / 10.0 / 1e6


def test_poisson_stream_is_seeded_and_in_range():
    a = serve.poisson_requests(12, 200.0, seed=3, filaments=(1, 4), nodes=(16, 24))
    b = serve.poisson_requests(12, 200.0, seed=3, filaments=(1, 4), nodes=(16, 24))
    assert [r.arrival for r in a] == [r.arrival for r in b]
    assert all(np.array_equal(x.scenario.position, y.scenario.position) for x, y in zip(a, b))
    assert all(64 <= r.scenario.H <= 1024 and r.scenario.H % 64 == 0 for r in a)
    assert all(500 <= r.steps <= 5000 for r in a)
    assert np.all(np.diff([r.arrival for r in a]) > 0)


@pytest.mark.gpu
def test_results_identical_alone_and_in_the_mix():
    torch = pytest.importorskip("torch")
    from microcosmos_b200 import baseline_config
    cfg = baseline_config()
    reqs = serve.poisson_requests(8, 2000.0, seed=11, sides=(64, 128, 192), filaments=(1, 6), nodes=(16, 40),
                                  steps=(30, 160), grad_fraction=0.0)
    be = serve.CudaBackend(cfg, dt=0.01)
    mixed = serve.Server(be, hbm_budget_bytes=4e9, max_active=8, chunk=16).run(reqs)
    alone = serve.run_plain(be, reqs)
    torch.cuda.synchronize()
    assert len(mixed) == len(reqs)
    for r, (rid, state, flags) in zip(mixed, alone):
        assert r.rid == rid and r.flags == 0 and flags == 0
        for k in ("position", "velocity", "f_grid", "steric", "fluid_velocity"):
            assert np.array_equal(r.state[k], state[k]), (rid, k)


@pytest.mark.gpu
def test_gradient_requests_in_the_mix_match_a_gradient_run_alone():
    torch = pytest.importorskip("torch")
    from microcosmos_b200 import baseline_config
    from microcosmos_b200.autodiff import GradPlan
    from microcosmos_b200.engine import Actuation, DeviceState
    cfg = baseline_config()
    reqs = serve.poisson_requests(6, 2000.0, seed=12, sides=(64, 128), filaments=(1, 4), nodes=(16, 30),
                                  steps=(20, 60), grad_fraction=0.5)
    assert any(r.want_grad for r in reqs) and not all(r.want_grad for r in reqs)
    be = serve.CudaBackend(cfg, dt=0.01)
    res = serve.Server(be, hbm_budget_bytes=4e9, max_active=4, chunk=16).run(reqs)
    for r, q in zip(res, reqs):
        if not q.want_grad:
            assert "grad" not in r.state
            continue
        sc = q.scenario
        st = DeviceState.from_scenario(sc)
        plan = GradPlan(sc.H, sc.W, st.N, sc.pairs, sc.bending_pairs, cfg, 0.01, q.steps)
        plan.forward(st, Actuation.from_scenario(sc))
        seed = torch.zeros((st.N, 2), dtype=torch.float32, device="cuda")
        seed[:, 0] = 1.0 / st.N
        g = plan.backward(seed)
        torch.cuda.synchronize()
        for k in ("act_c", "act_amp", "act_phase"):
            assert np.array_equal(r.state["grad"][k], g[k].cpu().numpy()), (q.rid, k)
        assert np.array_equal(r.state["position"], st.position.cpu().numpy())
