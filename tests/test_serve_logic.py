"""Host logic of the continuous-batching loop, on CPU with a fake engine:
FIFO admission under an HBM budget, jobs joining while others run, every
job advanced exactly its step count, memory returned on retirement."""
import numpy as np

from oidt_b200.engine import BudgetError
from oidt_b200.serve import Request, Server, latency_stats


class FakeSpec:
    def __init__(self, nt, bytes_, mode="tm2", shape=(40, 30)):
        self.nt, self.bytes, self.mode, self.shape = nt, bytes_, mode, shape
        self.ncells = int(np.prod(shape))
        self.nf = 2
        if mode == "yee3d":
            self.meta = {"power_window": ((2, shape[0] - 2), (2, shape[1] - 2))}
            self.win_lo, self.win_hi = (2, 2), (shape[0] - 2, shape[1] - 2)
        else:
            self.meta = {"power_window": (2, 28)}
            self.win_lo, self.win_hi = (0, 2), (1, 28)


class FakeJob:
    def __init__(self, eng, spec):
        self.eng, self.spec, self.steps, self.precision = eng, spec, 0, np.dtype(np.float32)
        self.released = False

    def advance(self, n):
        assert self.steps + n <= self.spec.nt
        self.steps += n
        self.eng.log.append(("advance", id(self), n))
        return self

    def sync(self, timeout_ms=-1):
        return self

    def dft(self, port, comp):
        return np.ones((self.spec.nf, self.spec.shape[1]), complex) * (1 + port)

    def port_power(self, port, minus=None, window=None):
        return np.full(self.spec.nf, 0.0 if minus is not None else 1.0 + port, complex)

    def release(self):
        self.released = True
        self.eng.in_use -= self.spec.bytes


class FakeEngine:
    def __init__(self, budget):
        self.budget, self.in_use, self.log, self.jobs = budget, 0, [], []

    def submit(self, spec, **kw):
        if self.in_use + spec.bytes > self.budget:
            raise BudgetError(-3, "budget")
        self.in_use += spec.bytes
        j = FakeJob(self, spec)
        self.jobs.append(j)
        return j

    def mark(self):  # the fake's work is done when it is enqueued
        class Done:
            def synchronize(self):
                pass
        return Done()

    def batch_advance(self, jobs, n):
        assert len({id(j) for j in jobs}) == len(jobs)
        for j in jobs:
            assert j.steps + n <= j.spec.nt
            j.steps += n
        self.log.append(("batch", len(jobs), n))


def test_admission_budget_and_completion():
    eng = FakeEngine(budget=250)
    reqs = [Request(k, arrival=0.0, spec=FakeSpec(nt=100 + 37 * k, bytes_=100)) for k in range(6)]
    srv = Server(eng, tick=32)
    res = srv.run(reqs, realtime=False)
    assert sorted(r.rid for r in res) == list(range(6))
    assert all(j.released and j.steps == j.spec.nt for j in eng.jobs)
    assert eng.in_use == 0
    assert srv.refused > 0            # budget forced some requests to wait
    assert max(n for kind, n, *_ in [e for e in eng.log if e[0] == "batch"]) <= 2  # at most 2 fit at once
    st = latency_stats(res)
    assert st["n"] == 6 and st["p99_s"] >= st["p50_s"]


def test_late_arrivals_join_running_batch():
    eng = FakeEngine(budget=10 ** 9)
    reqs = [Request(0, 0.0, FakeSpec(nt=640, bytes_=1)), Request(1, 0.0, FakeSpec(nt=640, bytes_=1))]
    srv = Server(eng, tick=64)
    # a request becomes visible after the first ticks: emulate by splitting the run
    srv.run(reqs[:1] + [Request(2, 0.0, FakeSpec(nt=128, bytes_=1))], realtime=False)
    sizes = [e[1] for e in eng.log if e[0] == "batch"]
    assert sizes[0] == 2 and 1 in sizes  # both ran together, then the long one alone


def test_fair_share_lets_small_jobs_leave_first():
    """Each job's steps per tick scale with (largest cells / its cells) in
    powers of two, capped at 64x: beside a large job, small jobs finish in
    the first tick while the large one needs many; every job still advances
    exactly its step count, in whole ring blocks plus one partial block."""
    class TickEngine(FakeEngine):
        ticks = 0

        def mark(self):
            TickEngine.ticks += 1
            return super().mark()

    def finish_ticks(fair):
        TickEngine.ticks = 0
        eng = TickEngine(budget=10 ** 9)
        reqs = [Request(0, 0.0, FakeSpec(nt=2000, bytes_=1, shape=(400, 400)))]
        reqs += [Request(k, 0.0, FakeSpec(nt=1990 + k, bytes_=1)) for k in range(1, 5)]
        srv = Server(eng, tick=64, fair_share=fair)
        order = []
        orig = srv._finish

        def record(entry, t0):
            order.append((entry[0].rid, TickEngine.ticks))
            orig(entry, t0)
        srv._finish = record
        srv.run(reqs, realtime=False, depth=1)
        assert all(j.steps == j.spec.nt for j in eng.jobs)
        return dict(order)

    fair, plain = finish_ticks(True), finish_ticks(False)
    assert all(fair[k] == 1 for k in range(1, 5)) and fair[0] >= 30
    assert all(plain[k] >= 30 for k in range(1, 5))
    srv = Server(FakeEngine(1), tick=64)
    assert srv.quota(160000, 160000) == 64 and srv.quota(1200, 160000) == 64 * 64
    assert srv.quota(40000, 160000) == 64 * 4 and srv.quota(30000, 160000) == 64 * 4


def test_fair_share_groups_share_launches():
    """Jobs of one size class advance together: with equal sizes every block
    is one multi-job launch of all of them."""
    eng = FakeEngine(budget=10 ** 9)
    reqs = [Request(k, 0.0, FakeSpec(nt=320, bytes_=1)) for k in range(3)]
    Server(eng, tick=64).run(reqs, realtime=False)
    batches = [e for e in eng.log if e[0] == "batch"]
    assert batches and all(n_jobs == 3 and n == 32 for _, n_jobs, n in batches)
    assert sum(n for _, _, n in batches) == 320


def test_small_first_large_fifo_with_cap():
    """Small requests (at most small_cells cells) are admitted as they arrive;
    large ones first-come, first-served, at most max_large active at once --
    later large requests wait even when memory allows, small ones never wait
    behind them."""
    eng = FakeEngine(budget=10 ** 9)
    big = lambda: FakeSpec(nt=640, bytes_=1, mode="yee3d", shape=(20, 20, 20))  # 8000 cells
    small = lambda: FakeSpec(nt=64, bytes_=1)                                   # 1200 cells
    reqs = [Request(k, 0.0, big(), meta={"kind": "3d"}) for k in range(4)]
    reqs += [Request(4 + k, 0.0, small(), meta={"kind": "2d"}) for k in range(3)]
    srv = Server(eng, tick=64, small_cells=5000, max_large=2)
    admitted = []
    orig = srv._admit

    def record(req, now):
        ok = orig(req, now)
        if ok:
            admitted.append((req.rid, len([e for e in srv.active if not srv.is_small(e[0])])))
        return ok
    srv._admit = record
    res = srv.run(reqs, realtime=False, depth=1)
    assert sorted(r.rid for r in res) == list(range(7))
    order = [rid for rid, _ in admitted]
    assert order[:5] == [0, 1, 4, 5, 6]            # two large, then every small one at once
    assert max(n for _, n in admitted) <= 2         # never more than max_large large jobs
    assert order.index(2) < order.index(3)          # large ones in arrival order
    assert srv.refused == 0                          # the cap, not the budget, held them back
    by = {r.rid: r for r in res}
    assert all(by[k].kind == ("3d" if k < 4 else "2d") and by[k].wait >= 0 for k in range(7))


def test_requests_built_on_arrival():
    """A request that carries a builder is built by the worker pool once it
    has arrived, admitted when built, and its host arrays are dropped once the
    job holds them; the served results equal those of prebuilt requests."""
    def mk(k):
        return FakeSpec(nt=96 + 32 * k, bytes_=1)

    class Spec(FakeSpec):
        def __init__(self, *a, **kw):
            super().__init__(*a, **kw)
            self.cb, self.kdx, self.twiddles = {"z": np.ones(3)}, {"xe": np.ones(3)}, (np.ones(2),)
            self.be = self.ce = self.bh = self.ch = self.j_src = np.ones(2)

    built = []

    def builder(k):
        def b():
            built.append(k)
            return Spec(nt=96 + 32 * k, bytes_=1), None
        return b
    eng = FakeEngine(budget=10 ** 9)
    reqs = [Request(k, 0.0, meta={"kind": "2d", "cells": 1200}, build=builder(k)) for k in range(4)]
    res = Server(eng, tick=32).run(reqs, realtime=False, workers=2)
    assert sorted(built) == [0, 1, 2, 3] and sorted(r.rid for r in res) == [0, 1, 2, 3]
    assert all(q.spec.cb == {} and q.spec.j_src is None for q in reqs)  # arrays dropped after admission
    assert all(j.steps == j.spec.nt for j in eng.jobs)
    ref = Server(FakeEngine(budget=10 ** 9), tick=32).run([Request(k, 0.0, mk(k)) for k in range(4)],
                                                          realtime=False)
    assert {r.rid: r.steps for r in res} == {r.rid: r.steps for r in ref}
