"""Continuous-batching request loop for roughness-realization jobs.

Requests (a SimSpec each, or a builder for one) arrive over time.  The loop

1. admits waiting requests while the context's HBM budget allows
   (``oidt_job_create`` refuses with OIDT_ERR_BUDGET otherwise; the request
   then waits for memory to be freed) -- admission copies the job's
   coefficients to the device while earlier jobs keep running.  Small
   requests (at most ``small_cells`` cells: every 2D request of the served
   mix) are admitted as they arrive; large ones in arrival order, at most
   ``max_large`` at a time.  Under sustained overload this keeps a small
   request's latency at a tick or two and gives large requests first-come,
   first-served waits, where admitting everything would share the GPU among a
   growing set and slow every request alike;
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

A request may carry a builder instead of its specs: the server then builds
them on arrival in a pool of worker threads (NumPy releases the interpreter
lock in its array work), admits the request once they are ready -- the build
time is part of its latency, as in a server that receives a request's
geometry, not its arrays -- and drops their host arrays once the device holds
them.
"""
from __future__ import annotations

import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import workloads as W
from .engine import BudgetError, Engine
from .sparams import forward_s_device


@dataclass
class Request:
    rid: int
    arrival: float                 # seconds from loop start
    spec: object = None            # SimSpec (reflected / device-under-test run)
    incident: object = None        # optional SimSpec of the smooth incident run
    meta: dict = field(default_factory=dict)
    build: object = None           # () -> (spec, incident), when spec is None
    future: object = None


def drop_arrays(spec):
    """Free a spec's host arrays once a job holds them on the device; what
    the serving loop still reads (shape, steps, frequencies, windows, meta)
    stays."""
    spec.cb, spec.kdx, spec.twiddles = {}, {}, ()
    spec.be = spec.ce = spec.bh = spec.ch = spec.j_src = spec.mat_idx = spec.mat_tab = None
    spec.meta = {k: v for k, v in spec.meta.items() if k != "core_mask"}


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
    kind: str = ""

    @property
    def latency(self) -> float:
        return self.finished - self.arrival

    @property
    def wait(self) -> float:
        """Seconds between arrival and admission (queueing for a slot or memory)."""
        return self.admitted - self.arrival


class Server:
    def __init__(self, engine: Engine, tick: int = 64, precision=np.float32, arith: str = "fast",
                 keep_dfts: bool = False, ring_steps: int = 32, fair_share: bool = True, max_boost_log2: int = 6,
                 small_cells: int = 1_000_000, max_large: int = 4, variant_2d: str = "cell"):
        """``variant_2d``: the launch form of 2D jobs.  The loop advances many
        jobs at once, where the per-cell form (no halo recomputation, kernels
        of different jobs running side by side) has the higher throughput;
        the tile form, the engine's default for a job on its own, has the
        lower latency for one job."""
        if tick % ring_steps:
            raise ValueError("tick must be a multiple of ring_steps")
        self.eng = engine
        self.tick = tick
        self.small_cells = small_cells
        self.max_large = max_large
        self.fair_share = fair_share
        self.max_boost_log2 = max_boost_log2
        self.precision = precision
        self.arith = arith
        self.keep_dfts = keep_dfts
        self.ring = ring_steps
        self.variant_2d = variant_2d
        self.active = []   # (request, job, incident job or None, admit time)
        self.results = []
        self.refused = 0

    def _admit(self, req: Request, now: float) -> bool:
        v = self.variant_2d if req.spec.mode != "yee3d" else "auto"
        try:
            j = self.eng.submit(req.spec, arith=self.arith, precision=self.precision, ring_steps=self.ring, variant=v)
        except BudgetError:
            return False
        ji = None
        if req.incident is not None:
            try:
                ji = self.eng.submit(req.incident, arith=self.arith, precision=self.precision, ring_steps=self.ring,
                                     variant=v)
            except BudgetError:
                j.release()
                return False
        self.active.append((req, j, ji, now))
        if req.build is not None:  # rebuilt from its parameters if needed again
            for s in (req.spec, req.incident):
                if s is not None:
                    drop_arrays(s)
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
                                   dfts=d_ref if self.keep_dfts else None, kind=req.meta.get("kind", "")))
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

    def run(self, requests, realtime: bool = True, max_wall: float = None, depth: int = 2, workers: int = 8):
        """Serve ``requests`` (sorted by arrival).  With ``realtime`` the
        arrival times are honoured against the wall clock; otherwise every
        request is available immediately (throughput mode).  Up to ``depth``
        ticks are in flight on the device while the host admits, reads out and
        retires, so the device does not wait for host work.  Requests that
        carry a builder are built on arrival by ``workers`` threads."""
        import collections
        pending = sorted(requests, key=lambda r: r.arrival)
        waiting = []                    # arrived, not admitted, in arrival order
        inflight = collections.deque()  # (event, requests completed by that tick)
        pool = ThreadPoolExecutor(max_workers=workers) if any(r.spec is None for r in pending) else None
        t0 = time.perf_counter()
        qi = 0
        try:
            while qi < len(pending) or waiting or self.active or inflight:
                now = time.perf_counter() - t0
                if max_wall is not None and now > max_wall:
                    break
                while qi < len(pending) and (not realtime or pending[qi].arrival <= now):
                    r = pending[qi]
                    if r.spec is None:
                        r.future = pool.submit(r.build)
                    waiting.append(r)
                    qi += 1
                if waiting:
                    self._admit_waiting(waiting, now)
                self._step(inflight, depth, t0)
                if not self.active and not inflight and (waiting or qi < len(pending)):
                    nxt = pending[qi].arrival - (time.perf_counter() - t0) if qi < len(pending) and realtime else 0.01
                    time.sleep(max(0.0, min(0.002 if waiting else 0.01, nxt)))
        finally:
            if pool is not None:
                pool.shutdown(wait=False, cancel_futures=True)
        return self.results

    def _step(self, inflight, depth, t0):
        """Launch one tick if any request is active; retire the requests whose
        last tick has completed, keeping at most ``depth`` ticks queued."""
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

    def is_small(self, req: Request) -> bool:
        cells = req.spec.ncells if req.spec is not None else req.meta["cells"]
        return cells <= self.small_cells

    def _admit_waiting(self, waiting: list, now: float):
        """Admit from ``waiting`` (arrival order): every small request the
        budget allows; large requests first-come, first-served while fewer
        than ``max_large`` are active (a large request the budget refuses
        blocks the later large ones, not the small ones)."""
        large_active = sum(1 for e in self.active if not self.is_small(e[0]))
        large_blocked = False
        keep = []
        for req in waiting:
            if req.spec is None:
                if not req.future.done():
                    keep.append(req)
                    large_blocked |= not self.is_small(req)
                    continue
                req.spec, req.incident = req.future.result()
                req.future = None
            small = self.is_small(req)
            if not small and (large_blocked or large_active >= self.max_large):
                keep.append(req)
                continue
            if self._admit(req, now):
                large_active += 0 if small else 1
            else:
                self.refused += 1
                keep.append(req)
                large_blocked |= not small
        waiting[:] = keep


def latency_stats(results):
    lat = np.array([r.latency for r in results]) if results else np.zeros(1)
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "n": len(results)}


def accuracy_sample(eng: Engine, requests, results, per_kind: int = 4, seed: int = 0):
    """|S_served - S_FP64| of a seeded sample of served requests (``per_kind``
    of each kind): each sampled request runs again alone in float64 with the
    exact arithmetic (equal to the float64 oracle bit for bit on the parity
    grids), its S formed the same way, and the largest difference over
    frequency of S11 and S21 is recorded."""
    from .sparams import forward_s_device
    by_rid = {q.rid: q for q in requests}
    rng = np.random.default_rng(seed)
    out = []
    kinds = sorted({r.kind for r in results})
    for kind in kinds:
        pool = [r for r in results if r.kind == kind]
        for r in rng.choice(pool, size=min(per_kind, len(pool)), replace=False):
            q = by_rid[r.rid]
            spec, inc = q.build() if q.build is not None else (q.spec, q.incident)  # served specs dropped their arrays
            j = eng.submit(spec, arith="exact", precision=np.float64)
            ji = eng.submit(inc, arith="exact", precision=np.float64) if inc is not None else None
            j.run()
            if ji is not None:
                ji.run()
            j.sync()
            if ji is not None:
                ji.sync()
            S = forward_s_device(spec, ji if ji is not None else j, j)
            for x in (j, ji):
                if x is not None:
                    x.release()
            out.append({"rid": int(r.rid), "kind": kind, "cells": int(r.cells), "steps": int(r.steps),
                        "max_abs_dS11": float(np.max(np.abs(r.S["S11"] - S["S11"]))),
                        "max_abs_dS21": float(np.max(np.abs(r.S["S21"] - S["S21"])))})
    return out


def _mix_specs(kind, kw, nf, precision, short_incident):
    """(rough spec, incident spec) of one served request.  The incident run is
    the smooth guide of the same cross-section; with ``short_incident`` it is
    only as long as the source and port 1 need, as the reference shortens its
    incident runs to the port lengths (FDTD_3D fdtd_auto_setup.py:88-89) --
    only its port-1 power enters S."""
    from .batch import incident_length
    if kind == "2d":
        nx = kw["nx"]
        common = dict(ny=kw["ny"], P=10, core_cells=10, src_x=40, steps=kw["steps"], nf=nf, precision=precision,
                      sigma_nm=kw["sigma_nm"], lc_nm=kw["lc_nm"], seed=kw["seed"])
        spec = W.slab2d(rough=True, nx=nx, ports=(60, nx - 60), **common)
        nxi = 122 if short_incident else nx
        inc = W.slab2d(rough=False, nx=nxi, ports=(60, nxi - 60), **common)
    else:
        common = dict(nx=kw["nx"], ny=kw["ny"], P=10, steps=kw["steps"], nf=nf, precision=precision,
                      sigma_nm=kw["sigma_nm"], lc_nm=kw["lc_nm"], seed=kw["seed"])
        spec = W.strip3d(rough=True, nz=kw["nz"], **common)
        nzi = incident_length(common) if short_incident else kw["nz"]
        inc = W.strip3d(rough=False, nz=nzi, **common)
    return spec, inc


def requests_from_mix(mix, nf=21, precision=np.float32, lazy=False, short_incident=False):
    """Requests for a served mix (``workloads.serving_mix``): each is a rough
    run with a smooth incident run (S21 needs both).  ``lazy``: the requests
    carry builders and the server builds their specs on arrival."""
    out = []
    for rid, (t, kw) in enumerate(mix):
        kw = dict(kw)
        kind = kw.pop("kind")
        cells = kw["nx"] * kw["ny"] * (kw["nz"] if kind == "3d" else 1)
        if kind == "3d":
            from .batch import incident_length
            inc_cells = kw["nx"] * kw["ny"] * (incident_length({}) if short_incident else kw["nz"])
        else:
            inc_cells = (122 if short_incident else kw["nx"]) * kw["ny"]
        meta = {"kind": kind, "cells": cells, "work": (cells + inc_cells) * kw["steps"]}

        def build(kind=kind, kw=kw):
            return _mix_specs(kind, kw, nf, precision, short_incident)
        if lazy:
            out.append(Request(rid, t, meta=meta, build=build))
        else:
            spec, inc = build()
            out.append(Request(rid, t, spec, incident=inc, meta=meta, build=None))
    return out


def measure(eng: Engine, rate_hz=20.0, duration_s=60.0, seed=0, tick=64, max_wall=900.0, warmup_s=5.0,
            ring_steps=32, accuracy_per_kind=4, workers=8, small_cells=1_000_000, max_large=4):
    """Serve ``duration_s`` seconds of the served mix at ``rate_hz`` with
    arrivals honoured on the wall clock (specs built on arrival, incident runs
    shortened to the port span); latency of the whole window, throughput, and
    |S - S_FP64| of a seeded sample of served requests.  A server pays its
    start-up once (kernel module loads, the first graph instantiations, device
    memory pool growth); with ``warmup_s`` > 0 that many seconds of the mix with
    another seed are served first, untimed.  The HBM budget is ``eng``'s."""
    kw = dict(tick=tick, ring_steps=ring_steps, small_cells=small_cells, max_large=max_large)
    if warmup_s > 0:
        Server(eng, **kw).run(requests_from_mix(W.serving_mix(rate_hz=rate_hz, duration_s=warmup_s, seed=seed + 1),
                                                lazy=True, short_incident=True),
                              realtime=True, max_wall=max_wall, workers=workers)
    reqs = requests_from_mix(W.serving_mix(rate_hz=rate_hz, duration_s=duration_s, seed=seed), lazy=True,
                             short_incident=True)
    srv = Server(eng, **kw)
    t0 = time.perf_counter()
    res = srv.run(reqs, realtime=True, max_wall=max_wall, workers=workers)
    wall = time.perf_counter() - t0
    done = {r.rid for r in res}
    cells = sum(q.spec.ncells * q.spec.nt + q.incident.ncells * q.incident.nt for q in reqs if q.rid in done)
    st = latency_stats(res)
    by_kind = {}
    for kind in sorted({r.kind for r in res}):
        sub = [r for r in res if r.kind == kind]
        s = latency_stats(sub)
        by_kind[kind] = {"n": len(sub), "p50_s": round(s["p50_s"], 3), "p99_s": round(s["p99_s"], 3),
                         "mean_wait_s": round(float(np.mean([r.wait for r in sub])), 3)}
    acc = accuracy_sample(eng, reqs, res, per_kind=accuracy_per_kind, seed=seed) if accuracy_per_kind else []
    stats = eng.stats()
    return {"rate_hz": rate_hz, "arrival_window_s": duration_s, "requests": len(reqs), "completed": len(res),
            "p50_s": round(st["p50_s"], 3), "p99_s": round(st["p99_s"], 3), "mean_s": round(st["mean_s"], 3),
            "by_kind": by_kind, "wall_s": round(wall, 3), "jobs_per_s": round(len(res) / wall, 3),
            "gcell_updates_per_s": round(cells / wall / 1e9, 3),
            "offered_gcell_updates_per_s": round(sum(q.meta["work"] for q in reqs) / duration_s / 1e9, 3),
            "hbm_budget_gb": round(stats["hbm_budget"] / 1e9, 1), "admission_refusals": srv.refused,
            "policy": "small requests (<= %d cells) admitted on arrival; large ones first-come first-served, at most "
                      "%d active; work-fair step shares per tick (cap 64x)" % (small_cells, max_large),
            "spec_build": "on arrival, %d worker threads, inside the latency" % workers,
            "incident_runs": "smooth guide shortened to the source and port 1",
            "accuracy_vs_fp64": {"jobs": acc,
                                 "max_abs_dS21": max((a["max_abs_dS21"] for a in acc), default=None),
                                 "max_abs_dS11": max((a["max_abs_dS11"] for a in acc), default=None)},
            "warmup_s": warmup_s}
