#!/usr/bin/env python
"""Benchmark: plain 3D FDTD S-parameter run on one B200 per rank.

Workload (one bench step = one whole simulation): silicon strip, 128 x 128
transverse cells x 256 cells along the guide (z), 20 nm cells, 10-cell CPML,
rough sidewalls (sigma 10 nm, Lc 50 nm, seed 0), Ey-sheet wave-packet source
at 1550 nm, 4000 time steps, FP32 fields / coefficients / CPML psi, FP64 port
DFT at 41 frequencies on two planes.  Metric: Gcell-updates/s = cells x time
steps / device time (the reference's MCells/s definition,
FDTD/GPU/FDTD_3D/s-parameter_extraction/fdtd_main.py:431, in G).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

Multi-GPU (torchrun, one rank per GPU): every rank runs its own independent
simulation (replicas; the path has no exchange step), the timed region is
bracketed by barriers and the slowest rank's time is used.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(nx=128, ny=128, nz=256, dx=20e-9, P=10, steps=4000, nf=41, sigma_nm=10.0, lc_nm=50.0, seed=0)
WORKLOAD_NAME = "strip3d 128x128x256 (z = guide axis), 20 nm, CPML 10, 4000 steps, 41-freq FP64 port DFT"
METRIC = "Gcell-updates/s (3D Yee + CPML, plain single run)"
UNIT = "Gcell/s"


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def dist_init(ws, local, backend="nccl"):
    """Process group of the replica ranks (NCCL on B200s; gloo serves
    the CPU tests of the same code).  A short timeout ends a rank that waits
    for a lost peer with an error instead of a hang."""
    if ws <= 1:
        return None
    import datetime
    import torch
    import torch.distributed as dist
    if backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return dist


def dist_max(dist, x, local):
    """Max over ranks (the slowest replica's time)."""
    if dist is None:
        return x
    import torch
    dev = "cuda:%d" % local if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(ws, cells_per_rank, steps, ms_max):
    """Gcell-updates/s of all replicas: every rank advances its own grid, the
    job takes as long as the slowest rank."""
    return ws * cells_per_rank * steps / (ms_max * 1e-3) / 1e9


def barrier(dist):
    if dist is not None:
        dist.barrier()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device, self.proc, self.path = device, None, None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9 and p[1].replace(".", "").isdigit():
                rows.append(p)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(rows[0][2]), "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit()) if rows else None,
                "reasons": reasons}


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------
def psi_elements(spec):
    from oidt_b200.spec import PSI
    return sum(2 * int(np.prod(spec.psi_shape(axis))) for _, axis in PSI[spec.mode])


def psi_elements_of(spec, half):
    """CPML psi elements updated by the E or H half-step (both sides)."""
    from oidt_b200.spec import PSI
    return sum(2 * int(np.prod(spec.psi_shape(axis))) for f, axis in PSI[spec.mode] if f.startswith(half))


def algorithmic_bytes(spec, esz=4):
    """Compulsory HBM bytes of the two per-cell launches of one 3D time step.
    E half-step: H (3 words), E (3) and dt/eps (3) read, E (3) written = 12
    words per cell; H half-step: E (3) and H (3) read, H (3) written = 9 words
    per cell; each CPML psi element read and written once.  DFT capture,
    source and twiddle traffic are not credited."""
    return {"E": 12 * esz * spec.ncells + 2 * esz * psi_elements_of(spec, "E"),
            "H": 9 * esz * spec.ncells + 2 * esz * psi_elements_of(spec, "H")}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs"), "measured"
    return 6650.0, "fallback"


PROFILE = os.path.join(ROOT, "profiles", "k_y3_e_strip3d_128x128x256.txt")


def ncu_traffic():
    """DRAM bytes of one E half-step launch (dram__bytes_read.sum +
    dram__bytes_write.sum) from the committed ncu summary (key=value line
    ``dram_bytes_per_launch=``)."""
    if not os.path.exists(PROFILE):
        return None
    for line in open(PROFILE):
        if line.startswith("dram_bytes_per_launch="):
            return float(line.split("=", 1)[1])
    return None


def pinned_spec(spec, prec):
    """Copy of the spec whose host arrays live in page-locked memory, already
    in the job's precision (the e2e host buffers)."""
    import copy
    import torch

    def pin(a, dt):
        a = np.asarray(a, dtype=dt)
        t = torch.empty(a.shape, dtype=torch.float32 if dt == np.float32 else torch.float64, pin_memory=True)
        out = t.numpy()
        out[...] = a
        keep.append(t)
        return out

    keep = []
    s = copy.copy(spec)
    s.cb = {k: pin(v, prec) for k, v in spec.cb.items()}
    s.kdx = {k: pin(v, prec) for k, v in spec.kdx.items()}
    s.be, s.ce, s.bh, s.ch = (pin(getattr(spec, n), prec) for n in ("be", "ce", "bh", "ch"))
    js = np.zeros(spec.nt)
    js[:len(spec.j_src)] = spec.j_src[:spec.nt]
    s.j_src = pin(js, prec)
    s.twiddles = tuple(pin(t, np.float64) for t in spec.twiddles)
    s.meta = dict(spec.meta, _pinned=keep)
    nbytes = sum(a.nbytes for a in list(s.cb.values()) + list(s.kdx.values()) +
                 [s.be, s.ce, s.bh, s.ch, s.j_src] + list(s.twiddles))
    return s, nbytes


# ---------------------------------------------------------------------------
# CPU baseline (the oracle, timed on the host cores)
# ---------------------------------------------------------------------------
def measure_slab2d(eng):
    """The 2D TMz slab case (400 x 200 cells, 2000 steps, float64, 21
    frequencies): device time of a whole run after a warm-up run, CUDA events
    on the engine stream, exact and fast arithmetic."""
    import torch
    from oidt_b200 import workloads as W
    spec = W.slab2d()
    st = torch.cuda.ExternalStream(eng.stream_handle(), device=eng.device)
    out = {"workload": "2D TMz slab %dx%d, %d steps, nf %d" % (spec.shape + (spec.nt, spec.nf)), "dtype": "f64"}
    for arith in ("exact", "fast"):
        job = eng.submit(spec, arith=arith, precision=np.float64)
        job.run().sync()
        job.reset()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        job.run()
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        job.release()
        out[arith] = {"ms_per_run": round(ms, 3), "gcell_updates_per_s": round(spec.ncells * spec.nt / ms / 1e6, 3)}
    return out


def cpu_baseline(spec, target_s=15.0):
    """Float64 oracle on the same workload, a bounded number of time steps."""
    from oracle import cpu as OC
    return OC.time_steps(spec, target_s=target_s)


# ---------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------
def run_reference(args, ws, rank, local):
    if rank != 0:
        return 0
    from oidt_b200 import workloads as W
    spec = W.strip3d(**WORKLOAD)
    vals = []
    info = None
    for _ in range(args.warmup):
        cpu_baseline(spec, target_s=min(5.0, args.cpu_seconds))
    for _ in range(args.steps):
        info = cpu_baseline(spec, target_s=args.cpu_seconds)
        vals.append(info["value"])
    v = float(np.median(vals))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": info["ms_per_time_step"] * spec.nt, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD_NAME, "grid": list(spec.shape), "steps_per_sim": spec.nt, "nf": spec.nf},
            "cpu_baseline": dict(info, value=v),
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_engine(args, ws, rank, local):
    import torch
    from oidt_b200.build import build
    from oidt_b200 import workloads as W
    from oidt_b200.engine import Engine
    build()
    dist = dist_init(ws, local)
    torch.cuda.set_device(local)
    spec = W.strip3d(**WORKLOAD)
    prec = np.float32
    eng = Engine(local)
    stream = torch.cuda.ExternalStream(eng.stream_handle(), device=local)

    # ---- device-resident throughput -------------------------------------
    job = eng.submit(spec, arith="fast", precision=prec)
    for _ in range(args.warmup):
        job.reset().run().sync()
    clocks = ClockSampler(local)
    barrier(dist)
    torch.cuda.synchronize()
    launches0 = eng.stats()["kernel_launches"]
    clocks.start()
    time.sleep(0.3)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        job.reset().run()
    ev1.record(stream)
    ev1.synchronize()
    clk = clocks.stop()
    launches = eng.stats()["kernel_launches"] - launches0
    torch.cuda.synchronize()
    barrier(dist)
    ms = ev0.elapsed_time(ev1) / args.steps
    ms = dist_max(dist, ms, local)
    value = whole_job_rate(ws, spec.ncells, spec.nt, ms)

    # ---- per-kernel roofline (live CUDA events on the engine stream) -----
    # A time step is two launches, the E half-step (k_y3_e, the larger one)
    # and the H half-step (k_y3_h); profile() times each launch with CUDA
    # events on the engine's stream, without graph replay.
    job.reset()
    job.advance(200)  # fields populated, source on
    prof = [job.profile(16) for _ in range(4)]
    ms_e = float(np.median([p[0] for p in prof]))
    ms_h = float(np.median([p[1] for p in prof]))
    ms_fold = float(np.median([p[2] for p in prof]))
    job.sync()
    alg = algorithmic_bytes(spec)
    achieved = alg["E"] / (ms_e * 1e-3) / 1e9
    achieved_h = alg["H"] / (ms_h * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = ncu_traffic()
    job.release()

    # ---- end to end through the C ABI, host buffers ---------------------
    # inputs and outputs live in page-locked host buffers allocated once,
    # outside the timed region (a serving host keeps such buffers)
    pspec, h2d = pinned_spec(spec, prec)
    ncomp = 4
    plane = spec.shape[0] * spec.shape[1]
    d2h = 2 * ncomp * spec.nf * plane * 16
    out_pinned = [torch.empty((spec.nf,) + tuple(spec.shape[:2]) + (2,), dtype=torch.float64, pin_memory=True)
                  for _ in range(2 * ncomp)]
    outs = [t.numpy().view(np.complex128)[..., 0] for t in out_pinned]
    e2e_ms = []
    for it in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        j = eng.submit(pspec, arith="fast", precision=prec)
        j.run()
        for q, (p, c) in enumerate((p, c) for p in (0, 1) for c in range(ncomp)):
            j.dft(p, c, out=outs[q])
        j.release()
        t1 = time.perf_counter()
        if it >= args.warmup:
            e2e_ms.append((t1 - t0) * 1e3)
    e2e = dist_max(dist, float(np.mean(e2e_ms)), local)
    e2e_value = whole_job_rate(ws, spec.ncells, spec.nt, e2e)

    # ---- batched realizations and the served mix (one GPU: at N > 1 they
    # would hold every GPU while rank 0 alone works) -------------------------
    batched = serving = slab2d = None
    if rank == 0 and ws == 1 and not args.no_extra:
        from oidt_b200 import batch as B, serve as SV
        # serving first: its latencies then see no host state left by the
        # batched leg's 64 realization specs
        serving = SV.measure(eng, rate_hz=20.0, duration_s=args.serve_window)
        batched = B.measure(eng, n=args.batch_n, steps=3000)
        slab2d = measure_slab2d(eng)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_baseline(spec, target_s=args.cpu_seconds)
    eng.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD_NAME, "grid": list(spec.shape), "steps_per_sim": spec.nt,
                       "nf": spec.nf, "parallelism": "replicas x%d" % ws,
                       "l2": "inputs larger than L2 (%.0f MB device state per run > 126 MB)" %
                             (spec.ncells * 4 * 9 / 1e6 + psi_elements(spec) * 4 / 1e6)},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "kernel": "k_y3_e (E half-step, one launch per time step)",
                         "ms_per_launch": round(ms_e, 5), "algorithmic_bytes": alg["E"], "peak_kind": peak_kind,
                         "h_half": {"kernel": "k_y3_h", "ms_per_launch": round(ms_h, 5),
                                    "algorithmic_bytes": alg["H"], "achieved": round(achieved_h, 1),
                                    "frac": round(achieved_h / peak, 4)},
                         "ms_dft_fold_per_16_steps": round(ms_fold, 5)},
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": round(e2e, 3)},
            "gpu_launches": int(launches),
            "batched": batched,
            "serving": serving,
            "slab2d": slab2d,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=("engine", "reference"))
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the batched-realization, served-mix and 2D slab measurements")
    ap.add_argument("--batch-n", type=int, default=64, help="realizations in the batched-vs-plain measurement")
    ap.add_argument("--serve-window", type=float, default=3.0, help="seconds of served-mix arrivals (20 jobs/s)")
    args = ap.parse_args()
    ws, rank, local = dist_env()
    if args.impl == "reference":
        return run_reference(args, ws, rank, local)
    return run_engine(args, ws, rank, local)


if __name__ == "__main__":
    sys.exit(main())
