"""Batched stochastic-roughness realizations.

Each realization is a rough 3D strip of its own (uneven) size plus the smooth
incident run of the same grid; S21 = sqrt(P_port2(rough) / P_port1(smooth)).

* :func:`run_batched` -- all realizations' runs advance together: one
  plane-sweep launch per time step over every job's work items (per-job tile
  tables), K-step blocks replayed from a CUDA graph.
* :func:`run_plain` -- the same kernels one run at a time, no graph (the
  baseline the batched rate is compared with).
"""
from __future__ import annotations

import time

import numpy as np

from . import workloads as W
from .engine import Engine
from .sparams import forward_s


def realization_specs(configs, nf=41, precision=np.float32, **common):
    out = []
    for c in configs:
        kw = dict(nx=c["nx"], ny=c["ny"], nz=c["nz"], steps=c["steps"], nf=nf, sigma_nm=c["sigma_nm"],
                  lc_nm=c["lc_nm"], seed=c["seed"], precision=precision)
        kw.update(common)
        out.append((W.strip3d(**kw), W.strip3d(rough=False, **kw)))
    return out


def _s21(spec_r, job_i, job_r):
    inc = {(p, c): job_i.dft(p, c) for p in (0, 1) for c in range(4)}
    ref = {(p, c): job_r.dft(p, c) for p in (0, 1) for c in range(4)}
    return forward_s(spec_r, inc, ref)


def run_batched(eng: Engine, specs, precision=np.float32, ring_steps=32, max_jobs=None):
    """Advance every run of every realization in multi-job launches (in groups
    of at most ``max_jobs`` jobs if given).  Returns (seconds, [S dict])."""
    t0 = time.perf_counter()
    flat = [s for pair in specs for s in pair]
    groups = [flat] if not max_jobs else [flat[i:i + max_jobs] for i in range(0, len(flat), max_jobs)]
    res = []
    for g in groups:
        jobs = [eng.submit(s, precision=precision, ring_steps=ring_steps) for s in g]
        steps = min(s.nt for s in g)
        eng.batch_advance(jobs, steps)
        for j in jobs:
            if j.spec.nt > steps:
                j.advance(j.spec.nt - steps)
        for j in jobs:
            j.sync()
        for k in range(0, len(jobs), 2):
            res.append(_s21(g[k], jobs[k + 1], jobs[k]))
        for j in jobs:
            j.release()
    return time.perf_counter() - t0, res


def run_plain(eng: Engine, specs, precision=np.float32):
    """One run at a time, no graph replay."""
    t0 = time.perf_counter()
    res = []
    for (sr, si) in specs:
        jr = eng.submit(sr, precision=precision, graphs=False)
        jr.run().sync()
        ji = eng.submit(si, precision=precision, graphs=False)
        ji.run().sync()
        res.append(_s21(sr, ji, jr))
        jr.release()
        ji.release()
    return time.perf_counter() - t0, res


def s21_loss_db(results, freqs=None):
    """Per-realization insertion loss -20 log10 |S21| averaged over the band."""
    return np.array([float(np.mean(-20 * np.log10(np.abs(r["S21"])))) for r in results])


def measure(eng: Engine, n=16, steps=3000, nf=41, master_seed=0):
    """Realizations/s of the batched path against the plain one-run-at-a-time
    path on ``n`` realizations drawn like the batched stochastic set (uneven
    grids), plus the largest |S21 difference| between the two (the same
    arithmetic, so 0 is expected).  Each realization is a rough run and the
    smooth incident run of its grid."""
    specs = realization_specs(W.batch_configs(n=n, master_seed=master_seed, steps=steps), nf=nf)
    cells = sum(r.ncells * r.nt + i.ncells * i.nt for r, i in specs)
    t_plain, s_plain = run_plain(eng, specs)
    t_batch, s_batch = run_batched(eng, specs)
    d = max(float(np.max(np.abs(a["S21"] - b["S21"]))) for a, b in zip(s_plain, s_batch))
    return {"realizations": n, "steps": steps, "nf": nf, "cell_updates": int(cells),
            "plain_s": round(t_plain, 3), "batched_s": round(t_batch, 3),
            "plain_realizations_per_s": round(n / t_plain, 3), "batched_realizations_per_s": round(n / t_batch, 3),
            "speedup": round(t_plain / t_batch, 3), "max_abs_dS21_batched_vs_plain": d,
            "s21_loss_db_mean": float(np.mean(s21_loss_db(s_batch))),
            "s21_loss_db_std": float(np.std(s21_loss_db(s_batch)))}

