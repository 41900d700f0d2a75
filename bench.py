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

``roofline`` is the time step against the HBM bound: the compulsory bytes of
one step (every field read and written once, the three dt/eps grids read once
-- 60 B per cell in FP32 -- plus 8 B per CPML psi element, 8 P (ny nz + nx nz
+ nx ny) of them) over the graph-replayed step time, against the measured copy
bandwidth.

At N = 1 the line also carries the other workloads, each with its own clock
record: ``serving`` (Poisson arrivals of mixed 2D/3D roughness jobs at 20/s
for 60 s under a 150 GB HBM budget, with |S - S_FP64| of a seeded sample),
``batched`` (64 uneven roughness realizations, batched against one at a time),
``slab2d`` (the 2D TMz slab) and ``large`` (a 151 M-cell rib guide, FP32
against FP64 on the GPU).

``--impl reference`` times the CPU restatement of the same loop (C/OpenMP, the
oracle) on the host cores: each bench step is a fixed sample of consecutive
time steps of the same simulation, in float32 (the engine's precision), with a
float64 sample beside it.

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
def psi_elements_of(spec, half):
    """CPML psi elements updated by the E or H half-step (both sides)."""
    from oidt_b200.spec import PSI
    return sum(2 * int(np.prod(spec.psi_shape(axis))) for f, axis in PSI[spec.mode] if f.startswith(half))


def half_step_bytes(spec, esz=4):
    """Bytes each half-step launch moves at least: E half-step H (3 words), E
    (3) and dt/eps (3) read, E (3) written = 12 words per cell; H half-step E
    (3) and H (3) read, H (3) written = 9 words per cell; each CPML psi
    element read and written once.  Per-launch diagnostics only: the two
    launches re-read each other's fields, which the step's compulsory bytes do
    not count."""
    return {"E": 12 * esz * spec.ncells + 2 * esz * psi_elements_of(spec, "E"),
            "H": 9 * esz * spec.ncells + 2 * esz * psi_elements_of(spec, "H")}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs"), "measured"
    return 6650.0, "fallback"


PROFILE = os.path.join(ROOT, "profiles", "v3_step_strip3d_128x128x256.txt")


def ncu_traffic():
    """DRAM bytes of one time step (dram__bytes_read.sum +
    dram__bytes_write.sum of the E and H half-step launches and the step's
    share of the DFT fold) from the committed ncu summary (key=value line
    ``dram_bytes_per_step=``)."""
    if not os.path.exists(PROFILE):
        return None
    for line in open(PROFILE):
        if line.startswith("dram_bytes_per_step="):
            return float(line.split("=", 1)[1])
    return None


SAMPLE_STEPS = 150  # time steps per CPU sample (reference-arm step, CPU baseline)


def bench_config(spec, ws):
    """The workload description both arms print."""
    from oidt_b200.spec import PSI
    state_mb = (spec.ncells * 9 + sum(2 * int(np.prod(spec.psi_shape(a))) for _, a in PSI[spec.mode])) * 4 / 1e6
    return {"workload": WORKLOAD_NAME, "grid": list(spec.shape), "steps_per_sim": spec.nt, "nf": spec.nf,
            "parallelism": "replicas x%d" % ws,
            "l2": "inputs larger than L2 (%.0f MB device state per run > 126 MB)" % state_mb}


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
    on the engine stream, exact and fast arithmetic, under the tile form
    (a ring block of steps per launch, the default) and the per-cell
    launches."""
    import torch
    from oidt_b200 import workloads as W
    spec = W.slab2d()
    st = torch.cuda.ExternalStream(eng.stream_handle(), device=eng.device)
    out = {"workload": "2D TMz slab %dx%d, %d steps, nf %d" % (spec.shape + (spec.nt, spec.nf)), "dtype": "f64"}
    for variant in ("tile", "cell"):
        for arith in ("exact", "fast"):
            job = eng.submit(spec, arith=arith, precision=np.float64, variant=variant)
            job.run().sync()
            job.reset()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            job.run()
            e1.record(st)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            job.release()
            r = {"ms_per_run": round(ms, 3), "us_per_step": round(1e3 * ms / spec.nt, 3),
                 "gcell_updates_per_s": round(spec.ncells * spec.nt / ms / 1e6, 3)}
            if variant == "tile":
                out[arith] = r
            else:
                out.setdefault("per_cell_launches", {})[arith] = r
    return out


def cpu_baseline(spec, samples=3):
    """The C/OpenMP oracle on the host cores, float32 (the engine's precision)
    and float64: ``samples`` timed samples of SAMPLE_STEPS consecutive time
    steps of the same workload each, after one untimed sample."""
    from oracle import cpu as OC
    f32, _ = OC.time_steps(spec, nsteps=SAMPLE_STEPS, samples=samples, precision="float32")
    f64, _ = OC.time_steps(spec, nsteps=SAMPLE_STEPS, samples=samples, precision="float64")
    return dict(f32, float64=f64)


# ---------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------
def run_reference(args, ws, rank, local):
    """The reference arm: the CPU restatement of the path on the host cores,
    rank 0 only.  One bench step is one sample of SAMPLE_STEPS consecutive
    time steps, continuing one simulation (a fresh one, untimed, when the
    workload's steps run out); value = cells x time steps / CPU time in
    float32, with a float64 sample of the same length beside it."""
    if rank != 0:
        return 0
    from oidt_b200 import workloads as W
    from oracle import cpu as OC
    from oracle import fdtd_ref as R
    spec = W.strip3d(**WORKLOAD)
    s = R.from_spec(spec)
    ms = []
    for it in range(args.warmup + args.steps):
        if s.n + SAMPLE_STEPS > spec.nt:
            s = R.from_spec(spec)
        t0 = time.perf_counter()
        OC.run_c(s, SAMPLE_STEPS, "float32")
        dt = (time.perf_counter() - t0) * 1e3
        if it >= args.warmup:
            ms.append(dt)
    ms_step = float(np.mean(ms))
    v = spec.ncells * SAMPLE_STEPS / (ms_step * 1e-3) / 1e9
    f64, _ = OC.time_steps(spec, nsteps=SAMPLE_STEPS, samples=3, precision="float64")
    sample = "%d consecutive time steps of the %d-step simulation per bench step, float32 fields (float64 DFT), " \
             "C/OpenMP restatement of the path" % (SAMPLE_STEPS, spec.nt)
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 5), "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 3),
            "step": "%d time steps" % SAMPLE_STEPS, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic", "config": bench_config(spec, ws),
            "cpu_baseline": {"value": round(v, 5), "unit": UNIT, "cores": OC.threads(), "kind": "port",
                             "precision": "float32", "sample": sample, "ms_per_time_step": round(ms_step / SAMPLE_STEPS, 4),
                             "float64": f64},
            "e2e": {"value": round(v, 5), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def with_clocks(device, fn, *a, **kw):
    """fn's result with the clock record sampled while it ran."""
    clk = ClockSampler(device)
    clk.start()
    try:
        out = fn(*a, **kw)
    finally:
        rec = clk.stop()
    if isinstance(out, dict):
        out["clocks"] = rec
    return out


def run_engine(args, ws, rank, local):
    import torch
    from oidt_b200.build import build
    from oidt_b200 import workloads as W
    from oidt_b200.engine import Engine
    from oidt_b200.large import roofline_bytes
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

    # ---- roofline of the time step ----------------------------------------
    # achieved = compulsory bytes of one step / graph-replayed step time; the
    # per-launch figures (CUDA events on the engine stream around each
    # launch, no graph replay) explain it.
    peak, peak_kind = measured_peaks()
    step_bytes = roofline_bytes(spec)
    ms_ts = ms / spec.nt
    achieved = step_bytes / (ms_ts * 1e-3) / 1e9
    job.reset()
    job.advance(200)  # fields populated, source on
    prof = [job.profile(16) for _ in range(4)]
    ms_e = float(np.median([p[0] for p in prof]))
    ms_h = float(np.median([p[1] for p in prof]))
    ms_fold = float(np.median([p[2] for p in prof]))
    job.sync()
    half = half_step_bytes(spec)
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

    # ---- the other workloads (one GPU: at N > 1 they would hold every GPU
    # while rank 0 alone works) -----------------------------------------------
    extra = {}
    if rank == 0 and ws == 1 and not args.no_extra:
        from oidt_b200 import batch as B, large as L, serve as SV
        # serving first: its latencies then see no host state left by the
        # batched leg's 64 realization specs; its context has the 150 GB budget
        eng_s = Engine(local, hbm_budget=int(args.serve_budget_gb * 1e9))
        extra["serving"] = with_clocks(local, SV.measure, eng_s, rate_hz=20.0, duration_s=args.serve_window,
                                       warmup_s=args.serve_warmup)
        eng_s.close()
        extra["batched"] = with_clocks(local, B.measure, eng, n=args.batch_n, steps=3000)
        extra["slab2d"] = with_clocks(local, measure_slab2d, eng)
        if not args.no_large:
            extra["large"] = with_clocks(local, L.run, eng=eng, peak_gbs=peak)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_baseline(spec)
    eng.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": bench_config(spec, ws),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": ncu_traffic(), "peak_kind": peak_kind,
                         "kernel": "one time step: k_v3_e + k_v3_h, and k_fold once per 32 steps",
                         "bytes_per_step": int(step_bytes), "ms_per_time_step": round(ms_ts, 5),
                         "per_launch": {"k_v3_e": {"ms": round(ms_e, 5), "bytes": half["E"],
                                                   "gbs": round(half["E"] / (ms_e * 1e-3) / 1e9, 1)},
                                        "k_v3_h": {"ms": round(ms_h, 5), "bytes": half["H"],
                                                   "gbs": round(half["H"] / (ms_h * 1e-3) / 1e9, 1)},
                                        "k_fold_per_16_steps_ms": round(ms_fold, 5)},
                         # the same graph-replayed step over the bytes its two launches move (each
                         # half-step re-reads the fields the other writes), not the fused 60 B/cell
                         "two_launch": {"bytes_per_step": int(half["E"] + half["H"]),
                                        "achieved_gbs": round((half["E"] + half["H"]) / (ms_ts * 1e-3) / 1e9, 1),
                                        "frac": round((half["E"] + half["H"]) / (ms_ts * 1e-3) / 1e9 / peak, 4)}},
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": round(e2e, 3)},
            "gpu_launches": int(launches),
            "clocks": clk,
        }
        line.update(extra)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


NCU_CASES = ("strip3d", "rib_section", "large", "slab2d", "scatter", "zwave")


def run_ncu_case(args):
    """A fixed workload for profiler captures: one job, ``--case-steps``
    steps, then exit.  strip3d is the benchmark grid (about 0.2 GB of device
    state in FP32); rib_section the large run's 384 x 384 cross-section on a
    256-cell guide (about 0.9 GB).  Captures that collect more than
    gpu__time_duration.sum use one of these two with a single -k kernel and a
    few launches; large (151 M cells, the large run itself), scatter and zwave
    (the scattering-loss and wave-impedance runs at their reference settings,
    75 M and 97 M cells) are for launch lists (gpu__time_duration.sum) only."""
    from oidt_b200 import workloads as W
    from oidt_b200.build import build
    from oidt_b200.engine import Engine
    build()
    n = max(args.case_steps, 64)
    if args.ncu_case == "strip3d":
        spec = W.strip3d(**dict(WORKLOAD, steps=n))
    elif args.ncu_case in ("rib_section", "large"):
        from oidt_b200 import large as L
        spec = L.large_spec(steps=n, shape=(384, 384, 256) if args.ncu_case == "rib_section" else L.SHAPE)
    elif args.ncu_case == "scatter":
        from oidt_b200 import scatter
        cfg = scatter.config()
        spec = scatter.build_spec(cfg, scatter.realization_profiles(cfg, 1)[0])
    elif args.ncu_case == "zwave":
        from oidt_b200 import zwave
        spec = zwave.build_spec(zwave.config())
    else:
        spec = W.slab2d(steps=n)
    eng = Engine(0)
    job = eng.submit(spec, precision=np.dtype(args.precision), variant=args.variant, graphs=not args.no_graphs)
    job.advance(args.case_steps).sync()
    print("ran", args.case_steps, "steps of", args.ncu_case, spec.shape)
    job.release()
    eng.close()
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
                    help="skip the served-mix, batched-realization, 2D slab and large-run measurements")
    ap.add_argument("--batch-n", type=int, default=64, help="realizations in the batched-vs-plain measurement")
    ap.add_argument("--serve-window", type=float, default=60.0, help="seconds of served-mix arrivals (20 jobs/s)")
    ap.add_argument("--serve-warmup", type=float, default=5.0, help="seconds of untimed served mix before it")
    ap.add_argument("--serve-budget-gb", type=float, default=150.0, help="HBM budget of the serving context")
    ap.add_argument("--no-large", action="store_true", help="skip the 151 M-cell rib run")
    ap.add_argument("--ncu-case", choices=NCU_CASES, help="run one fixed workload for a profiler capture and exit")
    ap.add_argument("--case-steps", type=int, default=32)
    ap.add_argument("--variant", default="auto", choices=("auto", "vec", "wave", "cell", "sweep", "tile"))
    ap.add_argument("--no-graphs", action="store_true")
    ap.add_argument("--precision", default="float32", choices=("float32", "float64"))
    args = ap.parse_args()
    if args.ncu_case:
        return run_ncu_case(args)
    ws, rank, local = dist_env()
    if args.impl == "reference":
        return run_reference(args, ws, rank, local)
    return run_engine(args, ws, rank, local)


if __name__ == "__main__":
    sys.exit(main())
