"""The large single 3D run: 384 x 384 cross-section x 1024 cells along the
guide (151 M cells), 15 nm cells, 16-cell CPML, a 220 x 1000 nm silicon guide
with rough sidewalls (sigma 10 nm, Lc 50 nm, seed 7), 2000 steps.

    python -m oidt_b200.large [--steps 2000] [--checkpoint 1000]

Runs the same kernels in FP32 (fast arithmetic) and in FP64 with the exact
arithmetic that equals the float64 oracle bit for bit, times both with CUDA
events on the engine's stream, and reports Gcell-updates/s and the FP32
fields' relative L2 error against the FP64 run at a checkpoint (pulse inside
the domain) and at the end.  Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import workloads as W
from .engine import Engine

FIELDS = ("EX", "EY", "EZ", "HX", "HY", "HZ")


def large_spec(steps=2000, nf=41):
    return W.strip3d(nx=384, ny=384, nz=1024, dx=15e-9, P=16, steps=steps, nf=nf, core_x_nm=220,
                     core_y_nm=1000, sigma_nm=10.0, lc_nm=50.0, seed=7)


def _timed_advance(eng, job, n):
    import torch
    st = torch.cuda.ExternalStream(eng.stream_handle(), device=eng.device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    job.advance(n)
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1) * 1e-3


def run(steps=2000, checkpoint=1000, device=0):
    import torch
    torch.cuda.set_device(device)
    t0 = time.perf_counter()
    spec = large_spec(steps)
    t_spec = time.perf_counter() - t0
    eng = Engine(device)
    out = {"workload": "strip3d 384x384x1024 (z = guide axis), 15 nm, CPML 16, %d steps" % steps,
           "cells": spec.ncells, "spec_build_s": round(t_spec, 1)}
    snaps = {}
    for prec, arith in ((np.float32, "fast"), (np.float64, "exact")):
        name = np.dtype(prec).name
        job = eng.submit(spec, arith=arith, precision=prec)
        job.sync()
        sec = _timed_advance(eng, job, checkpoint)
        at_ck = {f: job.field(f) for f in FIELDS}
        sec += _timed_advance(eng, job, steps - checkpoint)
        at_end = {f: job.field(f) for f in FIELDS}
        job.release()
        out[name] = {"arith": arith, "seconds": round(sec, 3),
                     "gcell_updates_per_s": round(spec.ncells * steps / sec / 1e9, 3)}
        if prec == np.float32:
            snaps = {"ck": at_ck, "end": at_end}
        else:
            err = {}
            for tag, ref in (("ck", at_ck), ("end", at_end)):
                e = {}
                for f in FIELDS:
                    a, b = snaps[tag][f].astype(np.float64), ref[f]
                    nb = float(np.linalg.norm(b))
                    e[f] = float(np.linalg.norm(a - b) / nb) if nb > 0 else 0.0
                err["step_%d" % (checkpoint if tag == "ck" else steps)] = e
            out["fp32_vs_fp64_rel_l2"] = err
    eng.close()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--checkpoint", type=int, default=1000)
    a = ap.parse_args(argv)
    print(json.dumps(run(a.steps, a.checkpoint)), flush=True)


if __name__ == "__main__":
    main()
