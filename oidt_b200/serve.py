"""Continuous-batching request loop for roughness-realization jobs.

Requests (a SimSpec each, or a builder for one) arrive over time.  The loop

1. admits waiting requests in arrival order while the context's HBM budget
   allows (``oidt_job_create`` refuses with OIDT_ERR_BUDGET otherwise; the
   request then waits for memory to be freed) -- admission copies the job's
   coefficients to the device while earlier jobs keep running;
2. advances every admitted job in one tick of multi-job launches
   (``oidt_batch_advance``), each by its share of the tick: ``tick`` steps
   times the power of two nearest below (largest active job's cells / its
   cells), at most 64x.  Every job then gets about the same cell-updates per
   tick, so a small job (a 2D run beside 3D ones) leaves after a tick or two
   instead of queuing behind the large jobs' steps; total work and every
   result are unchanged (``fair_share=False`` gives every job ``tick`` steps);
3. retires finished jobs: sums their port powers on the device, forms
   S11/S21, records latency = finish time - arrival time, frees their memory.

So requests that arrive while others are on the GPU join at the next tick
and share launches with them; nothing waits for a batch to drain.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import workloads as W
from .engine import BudgetError, Engine
from .sparams import forward_s_device


@dataclass
class Request:
    rid: int
    arrival: float                 # seconds from loop start
    spec: object                   # SimSpec (reflected / device-under-test run)
    incident: object = None        # optional SimSpec of the smooth incident run
    meta: dict = field(default_factory=dict)


@dataclass
class Result:
    rid: int
    arrival: float
    admitted: float
    finished: float
    cells: int
    steps: int
    S: dict = None
    dfts: dict = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


class Server:
    def __init__(self, engine: Engine, tick: int = 64, precision=np.float32, arith: str = "fast",
                 keep_dfts: bool = False, ring_steps: int = 32, fair_share: bool = True, max_boost_log2: int = 6):
        if tick % ring_steps:
            raise ValueError("tick must be a multiple of ring_steps")
        self.eng = engine
        self.tick = tick
        self.fair_share = fair_share
        self.max_boost_log2 = max_boost_log2
        self.precision = precision
        self.arith = arith
        self.keep_dfts = keep_dfts
        self.ring = ring_steps
        self.active = []   # (request, job, incident job or None, admit time)
        self.results = []
        self.refused = 0

    def _admit(self, req: Request, now: float) -> bool:
        try:
            j = self.eng.submit(req.spec, arith=self.arith, precision=self.precision, ring_steps=self.ring)
        except BudgetError:
            return False
        ji = None
        if req.incident is not None:
            try:
                ji = self.eng.submit(req.incident, arith=self.arith, precision=self.precision, ring_steps=self.ring)
            except BudgetError:
                j.release()
                return False
        self.active.append((req, j, ji, now))
        return True

    def _finish(self, entry, t0: float):
        """S of a completed request from its port powers, summed on the device
        (its DFT planes are read back only with ``keep_dfts``); free its jobs."""
        req, j, ji, adm = entry
        jobs = [x for x in (j, ji) if x is not None]
        for x in jobs:
            x.sync()
        nc = 4 if req.spec.mode == "yee3d" else 2
        S = forward_s_device(req.spec, ji if ji is not None else j, j)
        d_ref = {(p, c): j.dft(p, c) for p in (0, 1) for c in range(nc)} if self.keep_dfts else None
        fin = time.perf_counter() - t0
        self.results.append(Result(req.rid, req.arrival, adm, fin, req.spec.ncells, req.spec.nt,
                                   S={k: v for k, v in S.items() if k != "P_inc"},
                                   dfts=d_ref if self.keep_dfts else None))
        for x in jobs:
            x.release()

    def quota(self, cells: int, ref_cells: int) -> int:
        """Steps per tick of a job of ``cells`` cells beside a largest active
        job of ``ref_cells``: ``tick`` times 2^floor(log2(ref / cells)), at
        most 2^max_boost_log2."""
        if not self.fair_share:
            return self.tick
        r = max(1, int(ref_cells // max(1, cells)))
        return self.tick << min(self.max_boost_log2, r.bit_length() - 1)

    def _tick(self):
        """Enqueue one tick for every admitted request with steps left; returns
        the requests whose last steps are now enqueued.  Whole ring blocks go
        through multi-job launches: block b advances every job with more than
        b blocks in its share, so the groups shrink as the small shares end
        (each job replays its own captured block graph, so changing groups
        cost no capture); a share's last partial block, if any, runs alone."""
        jobs = []
        for (req, j, ji, adm) in self.active:
            jobs += [x for x in (j, ji) if x is not None and x.steps < x.spec.nt]
        if jobs:
            ref = max(x.spec.ncells for x in jobs)
            share = [min(x.spec.nt - x.steps, self.quota(x.spec.ncells, ref)) for x in jobs]
            K = self.ring
            blocks = [n // K for n in share]
            for b in range(max(blocks)):
                by_prec = {}
                for x, nb in zip(jobs, blocks):
                    if nb > b:
                        by_prec.setdefault(str(x.precision), []).append(x)
                for group in by_prec.values():
                    self.eng.batch_advance(group, K)
            for x, n in zip(jobs, share):
                if n % K:
                    x.advance(n % K)
        done, keep = [], []
        for e in self.active:
            (done if all(x.steps >= x.spec.nt for x in e[1:3] if x is not None) else keep).append(e)
        self.active = keep
        return done

    def run(self, requests, realtime: bool = True, max_wall: float = None, depth: int = 2):
        """Serve ``requests`` (sorted by arrival).  With ``realtime`` the
        arrival times are honoured against the wall clock; otherwise every
        request is available immediately (throughput mode).  Up to ``depth``
        ticks are in flight on the device while the host admits, reads out and
        retires, so the device does not wait for host work."""
        import collections
        pending = sorted(requests, key=lambda r: r.arrival)
        inflight = collections.deque()  # (event, requests completed by that tick)
        t0 = time.perf_counter()
        qi = 0
        while qi < len(pending) or self.active or inflight:
            now = time.perf_counter() - t0
            if max_wall is not None and now > max_wall:
                break
            # admission: arrived requests, FIFO, while memory allows
            while qi < len(pending) and (not realtime or pending[qi].arrival <= now):
                if not self._admit(pending[qi], now):
                    self.refused += 1
                    break
                qi += 1
            launched = False
            if self.active:
                done = self._tick()
                inflight.append((self.eng.mark(), done))
                launched = True
            # keep at most `depth` ticks queued; drain when there is nothing to launch
            while inflight and (len(inflight) >= depth or not launched):
                ev, done = inflight.popleft()
                ev.synchronize()
                for e in done:
                    self._finish(e, t0)
                if not launched:
                    break
            if not launched and not inflight and qi < len(pending) and realtime:
                time.sleep(max(0.0, min(0.01, pending[qi].arrival - (time.perf_counter() - t0))))
        return self.results


def latency_stats(results):
    lat = np.array([r.latency for r in results]) if results else np.zeros(1)
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "n": len(results)}


def requests_from_mix(mix, nf=21, precision=np.float32):
    """Requests for a served mix (``workloads.serving_mix``): each is a rough
    run with the smooth incident run of the same grid (S21 needs both)."""
    out = []
    for rid, (t, kw) in enumerate(mix):
        kw = dict(kw)
        kind = kw.pop("kind")
        if kind == "2d":
            nx = kw["nx"]
            common = dict(nx=nx, ny=kw["ny"], P=10, core_cells=10, src_x=40, ports=(60, nx - 60), steps=kw["steps"],
                          nf=nf, precision=precision, sigma_nm=kw["sigma_nm"], lc_nm=kw["lc_nm"], seed=kw["seed"])
            spec, inc = W.slab2d(rough=True, **common), W.slab2d(rough=False, **common)
        else:
            common = dict(nx=kw["nx"], ny=kw["ny"], nz=kw["nz"], P=10, steps=kw["steps"], nf=nf, precision=precision,
                          sigma_nm=kw["sigma_nm"], lc_nm=kw["lc_nm"], seed=kw["seed"])
            spec, inc = W.strip3d(rough=True, **common), W.strip3d(rough=False, **common)
        out.append(Request(rid, t, spec, incident=inc, meta={"kind": kind}))
    return out


def measure(eng: Engine, rate_hz=20.0, duration_s=3.0, seed=0, tick=64, max_wall=300.0, warmup=True,
            ring_steps=32):
    """Serve the first ``duration_s`` seconds of the served mix at ``rate_hz``
    with arrivals honoured on the wall clock; latency and throughput.  A
    server pays its start-up once (kernel module loads, the first graph
    instantiations, device memory pool growth); with ``warmup`` the same
    length of the mix with another seed is served first, untimed."""
    if warmup:
        Server(eng, tick=tick, ring_steps=ring_steps).run(requests_from_mix(W.serving_mix(rate_hz=rate_hz, duration_s=duration_s,
                                                                   seed=seed + 1)), realtime=True, max_wall=max_wall)
    reqs = requests_from_mix(W.serving_mix(rate_hz=rate_hz, duration_s=duration_s, seed=seed))
    srv = Server(eng, tick=tick, ring_steps=ring_steps)
    t0 = time.perf_counter()
    res = srv.run(reqs, realtime=True, max_wall=max_wall)
    wall = time.perf_counter() - t0
    cells = sum(r.cells * r.steps for r in res) + sum(q.incident.ncells * q.incident.nt for q in reqs
                                                        if q.rid in {r.rid for r in res})
    st = latency_stats(res)
    return {"rate_hz": rate_hz, "arrival_window_s": duration_s, "requests": len(reqs), "completed": len(res),
            "p50_s": round(st["p50_s"], 3), "p99_s": round(st["p99_s"], 3), "mean_s": round(st["mean_s"], 3),
            "wall_s": round(wall, 3), "jobs_per_s": round(len(res) / wall, 3),
            "gcell_updates_per_s": round(cells / wall / 1e9, 3), "admission_refusals": srv.refused,
            "policy": "work-fair shares, cap 64x" if srv.fair_share else "equal steps per tick",
            "warmed_up": bool(warmup)}

