"""The large single 3D run: 384 x 384 cross-section x 1024 cells along the
guide (151 M cells), 15 nm cells, 16-cell CPML, 2000 steps, a 1 um-wide
silicon rib with rough sidewalls (sigma 10 nm, Lc 50 nm, seed 7).

The rib (``workloads.strip3d`` with ``slab_y_nm``): a 1000 nm wide, 220 nm
high ridge whose x-faces -- the sidewalls, the faces the reference roughens
(FDTD/GPU/FDTD_3D/s-parameter_extraction/fdtd_funcs.py:363-369, apply_mask) --
carry the roughness, on a 90 nm slab of the same index spanning the whole
cross-section, in n = 1.44 cladding.

    python -m oidt_b200.large [--steps 2000] [--checkpoint 1000]

Runs the same kernels in FP32 (fast arithmetic) and in FP64 with the exact
arithmetic that equals the float64 oracle bit for bit on the parity grids,
times both with CUDA events on the engine's stream, and reports
Gcell-updates/s, the time step against the HBM roofline (60 B per cell-update
plus 8 B per CPML psi element, the compulsory traffic) and the FP32 fields'
relative L2 error against the FP64 run at a checkpoint (pulse inside the
domain) and at the end.  Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import workloads as W
from .engine import Engine

FIELDS = ("EX", "EY", "EZ", "HX", "HY", "HZ")
SHAPE = (384, 384, 1024)


def large_spec(steps=2000, nf=41, shape=SHAPE, P=16):
    nx, ny, nz = shape
    return W.strip3d(nx=nx, ny=ny, nz=nz, dx=15e-9, P=P, steps=steps, nf=nf, core_x_nm=1000, core_y_nm=220,
                     slab_y_nm=90, sigma_nm=10.0, lc_nm=50.0, seed=7)


def roofline_bytes(spec, esz=4):
    """Compulsory HBM bytes of one 3D time step: every field read and written
    once and the three dt/eps grids read once (6 x 2 + 3 words per cell), plus
    one read and one write of every CPML psi element, 8 P (ny nz + nx nz +
    nx ny) of them."""
    nx, ny, nz = spec.shape
    P = spec.num_cpml
    return 15 * esz * nx * ny * nz + 2 * esz * 8 * P * (ny * nz + nx * nz + nx * ny)


def _timed_advance(eng, job, n):
    import torch
    st = torch.cuda.ExternalStream(eng.stream_handle(), device=eng.device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    job.advance(n)
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1) * 1e-3


def rel_l2(a, b):
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(a.astype(np.float64) - b) / nb) if nb > 0 else 0.0


def run(steps=2000, checkpoint=1000, device=0, eng=None, shape=SHAPE, peak_gbs=None):
    """FP32 then FP64-exact on the same spec; returns the measurement dict."""
    import torch
    torch.cuda.set_device(device)
    t0 = time.perf_counter()
    spec = large_spec(steps, shape=shape)
    t_spec = time.perf_counter() - t0
    own = eng is None
    eng = eng or Engine(device)
    out = {"workload": "rib3d %dx%dx%d (z = guide axis), 15 nm, CPML 16, 1 um rib (220 nm ridge on a 90 nm slab), "
                       "rough sidewalls sigma 10 nm / Lc 50 nm / seed 7, %d steps" % (shape + (steps,)),
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
        rate = spec.ncells * steps / sec / 1e9
        out[name] = {"arith": arith, "seconds": round(sec, 3), "gcell_updates_per_s": round(rate, 3),
                     "ms_per_time_step": round(sec / steps * 1e3, 4)}
        if prec == np.float32:
            alg = roofline_bytes(spec)
            achieved = alg / (sec / steps) / 1e9
            out[name]["roofline"] = {"bytes_per_step": int(alg), "achieved_gbs": round(achieved, 1)}
            if peak_gbs:
                out[name]["roofline"]["frac"] = round(achieved / peak_gbs, 4)
            snaps = {"ck": at_ck, "end": at_end}
        else:
            err = {}
            for tag, ref in (("ck", at_ck), ("end", at_end)):
                err["step_%d" % (checkpoint if tag == "ck" else steps)] = {
                    f: rel_l2(snaps[tag][f], ref[f]) for f in FIELDS}
            out["fp32_vs_fp64_rel_l2"] = err
            out["fp32_vs_fp64_rel_l2_max"] = max(v for e in err.values() for v in e.values())
        del at_ck, at_end
    if own:
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
