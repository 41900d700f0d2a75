"""Batched stochastic-roughness realizations.

Each realization is a rough 3D strip of its own (uneven) size.  Its S21 is
sqrt(P_port2(rough) / P_port1(incident)), where the incident run is a smooth
guide just long enough for both ports -- the reference's incident runs shorten
the guide to the two port lengths (FDTD_3D fdtd_auto_setup.py:88-89).  The
incident run depends only on the cross-section, the time steps and the
source, not on the roughness or the guide length, so:

* :func:`run_plain` -- one run at a time, as the reference runs each line:
  every realization runs its rough guide and its own incident run, each
  launched step by step (no graph).
* :func:`run_batched` -- every rough run plus one shared incident run per
  cross-section advance together in multi-job launches (one branch per job,
  K-step blocks replayed from a CUDA graph).

Both take an optional :class:`oidt_b200.tune.Tuner`; each job is then launched
with the choices measured for its shape (results are unchanged by them).  Both
sum the S-parameter powers on the device (``forward_s_device``): the DFT planes
stay in HBM and only 3 x nf complex values per realization are read back.
"""
from __future__ import annotations

import time

import numpy as np

from . import workloads as W
from .engine import Engine
from .sparams import forward_s_device


def incident_length(kw: dict) -> int:
    """Cells along the guide of the incident run: the CPML, the source gap and
    the port gap on both sides, plus two cells between the ports."""
    P, src_gap, port_gap = kw.get("P", 10), kw.get("src_gap", 10), kw.get("port_gap", 20)
    return 2 * (P + src_gap + port_gap) + 2


def realization_set(configs, nf=41, precision=np.float32, **common):
    """Rough specs, the incident key of each, and the incident specs by key
    ((nx, ny, steps): realizations of one cross-section share one)."""
    roughs, keys, incidents = [], [], {}
    for c in configs:
        kw = dict(nx=c["nx"], ny=c["ny"], nz=c["nz"], steps=c["steps"], nf=nf, sigma_nm=c["sigma_nm"],
                  lc_nm=c["lc_nm"], seed=c["seed"], precision=precision)
        kw.update(common)
        roughs.append(W.strip3d(**kw))
        key = (c["nx"], c["ny"], c["steps"])
        if key not in incidents:
            incidents[key] = W.strip3d(**dict(kw, rough=False, nz=incident_length(kw)))
        keys.append(key)
    return roughs, keys, incidents


def _choice(tuner, spec, precision, ring_steps):
    return tuner.choose(spec, precision, ring_steps=ring_steps) if tuner is not None else {}


def tune_set(tuner, rset, precision=np.float32, ring_steps=32):
    """Measure the launch choices of every shape in the set (untimed work
    before a timed run)."""
    roughs, keys, incidents = rset
    for s in list(roughs) + list(incidents.values()):
        tuner.choose(s, precision, ring_steps=ring_steps)


def run_batched(eng: Engine, rset, precision=np.float32, ring_steps=32, tuner=None):
    """Advance every rough run and the shared incident runs together.
    Returns (seconds, [S dict per realization])."""
    roughs, keys, incidents = rset
    t0 = time.perf_counter()
    inc_keys = list(incidents)
    specs = roughs + [incidents[k] for k in inc_keys]
    jobs = [eng.submit(s, precision=precision, ring_steps=ring_steps, **_choice(tuner, s, precision, ring_steps))
            for s in specs]
    steps = min(s.nt for s in specs)
    eng.batch_advance(jobs, steps)
    for j in jobs:
        if j.spec.nt > steps:
            j.advance(j.spec.nt - steps)
    for j in jobs:
        j.sync()
    inc = {k: jobs[len(roughs) + n] for n, k in enumerate(inc_keys)}
    res = [forward_s_device(roughs[r], inc[keys[r]], jobs[r]) for r in range(len(roughs))]
    for j in jobs:
        j.release()
    return time.perf_counter() - t0, res


def run_plain(eng: Engine, rset, precision=np.float32, tuner=None, ring_steps=32):
    """One run at a time, launched step by step: each realization's rough
    run, then its own incident run."""
    roughs, keys, incidents = rset
    t0 = time.perf_counter()
    res = []
    for spec_r, key in zip(roughs, keys):
        jr = eng.submit(spec_r, precision=precision, graphs=False, ring_steps=ring_steps,
                        **_choice(tuner, spec_r, precision, ring_steps))
        jr.run().sync()
        ji = eng.submit(incidents[key], precision=precision, graphs=False, ring_steps=ring_steps,
                        **_choice(tuner, incidents[key], precision, ring_steps))
        ji.run().sync()
        res.append(forward_s_device(spec_r, ji, jr))
        jr.release()
        ji.release()
    return time.perf_counter() - t0, res


def s21_loss_db(results):
    """Per-realization insertion loss -20 log10 |S21| averaged over the band."""
    return np.array([float(np.mean(-20 * np.log10(np.abs(r["S21"])))) for r in results])


def measure(eng: Engine, n=16, steps=3000, nf=41, master_seed=0, tuned=True, ring_steps=32):
    """Realizations/s of the batched path against the plain one-run-at-a-time
    path on ``n`` realizations drawn like the batched stochastic set (uneven
    grids), and the largest |S21 difference| between the two (the same
    arithmetic on the same runs, so 0 is expected).  With ``tuned``, every
    shape's launch choice is measured first (untimed) and both paths use it,
    so the ratio is that of batching alone."""
    rset = realization_set(W.batch_configs(n=n, master_seed=master_seed, steps=steps), nf=nf)
    roughs, keys, incidents = rset
    plain_cells = sum(r.ncells * r.nt + incidents[k].ncells * incidents[k].nt for r, k in zip(roughs, keys))
    batched_cells = sum(r.ncells * r.nt for r in roughs) + sum(s.ncells * s.nt for s in incidents.values())
    tuner = None
    t_tune = 0.0
    if tuned:
        from .tune import Tuner
        tuner = Tuner(eng)
        t0 = time.perf_counter()
        tune_set(tuner, rset, ring_steps=ring_steps)
        t_tune = time.perf_counter() - t0
    t_plain, s_plain = run_plain(eng, rset, tuner=tuner, ring_steps=ring_steps)
    t_batch, s_batch = run_batched(eng, rset, ring_steps=ring_steps, tuner=tuner)
    d = max(float(np.max(np.abs(a["S21"] - b["S21"]))) for a, b in zip(s_plain, s_batch))
    loss = s21_loss_db(s_batch)
    return {"realizations": n, "steps": steps, "nf": nf, "ring_steps": ring_steps,
            "shared_incident_runs": len(incidents),
            "plain_cell_updates": int(plain_cells), "batched_cell_updates": int(batched_cells),
            "plain_s": round(t_plain, 3), "batched_s": round(t_batch, 3),
            "plain_realizations_per_s": round(n / t_plain, 3), "batched_realizations_per_s": round(n / t_batch, 3),
            "speedup": round(t_plain / t_batch, 3), "max_abs_dS21_batched_vs_plain": d,
            "s21_loss_db_mean": float(np.mean(loss)), "s21_loss_db_std": float(np.std(loss)),
            "s21_loss_db_percentiles": {str(q): float(np.percentile(loss, q)) for q in (0, 5, 25, 50, 75, 95, 100)},
            "launch_tuning": None if tuner is None else {
                "seconds": round(t_tune, 3), "shapes": len(tuner.table),
                "choices": _histogram(tuner, rset, ring_steps=ring_steps)}}


def _histogram(tuner, rset, precision=np.float32, ring_steps=32):
    from .tune import label
    roughs, keys, incidents = rset
    h = {}
    for s in list(roughs) + list(incidents.values()):
        c = label(tuner.choose(s, precision, ring_steps=ring_steps))
        h[c] = h.get(c, 0) + 1
    return h
