"""Launch tuner: per grid shape, time the launch choices that leave a job's
results unchanged and keep the fastest.

The choices are ``Engine.submit`` keywords:

* ``variant`` -- 'cell', the per-cell E-half / H-half launches; 'vec', the
  same half-steps with four cells per thread along z and 16-byte accesses;
  or 'sweep', one fused plane-sweep launch per step (TMA-staged tiles);
* ``rows`` -- per-cell form: a block is a tile of 32 cells along z (the guide
  axis, contiguous) by ``rows`` rows along y, rows 2, 4 or 8;
* ``march_depth`` -- plane sweep: x-planes per work item (0 = the engine's
  makespan estimate).

The DFT ring depth (``ring_steps``) is the caller's: jobs advanced together in
one multi-job block must share it, so it is an input of the tuning, not a
result.  Every candidate is bit-identical in what it computes (the parity
tests run each form against the oracle), so the tuner may pick freely.

Each candidate runs on a job of the caller's own grid and coefficients: one
K-step block captures its CUDA graph, then ``reps`` K-step blocks are timed
one by one with CUDA events on the engine's stream and the median counts.
Choices are cached per shape key -- mode, precision, arithmetic, the
cross-section (nx, ny), the CPML depth, the ring depth and the guide length
rounded up to a multiple of 64 cells -- in memory and, with ``cache_path``, in
a JSON file, so a batched or served mix tunes each shape class once.  Only 3D
jobs have choices; 2D jobs get the defaults without a measurement.
"""
from __future__ import annotations

import json
import os
import threading

import numpy as np

from .spec import SimSpec

DEFAULT = {"variant": "vec", "rows": 0, "march_depth": 0}
CANDIDATES = (
    {"variant": "wave", "rows": 0, "march_depth": 0},
    {"variant": "vec", "rows": 0, "march_depth": 0},
    {"variant": "cell", "rows": 4, "march_depth": 0},
    {"variant": "cell", "rows": 2, "march_depth": 0},
    {"variant": "cell", "rows": 8, "march_depth": 0},
    {"variant": "sweep", "rows": 0, "march_depth": 0},
    {"variant": "sweep", "rows": 0, "march_depth": 16},
)


def label(choice: dict) -> str:
    """'vec', 'wave', 'cell/rows4', 'sweep/depth16', 'sweep/depth-auto'."""
    if choice["variant"] in ("vec", "wave"):
        return choice["variant"]
    if choice["variant"] == "cell":
        return "cell/rows%d" % (choice["rows"] or 4)
    return "sweep/depth%s" % (choice["march_depth"] or "-auto")


def shape_key(spec: SimSpec, precision, arith: str, ring_steps: int) -> str:
    prec = np.dtype(precision if precision is not None else spec.precision).name
    nx, ny = spec.shape[0], spec.shape[1]
    nz64 = -(-int(spec.shape[2]) // 64) * 64 if spec.mode == "yee3d" else 0
    return "%s/%s/%s/%dx%d/z%d/P%d/K%d" % (spec.mode, prec, arith, nx, ny, nz64, spec.num_cpml,
                                           int(ring_steps) or 32)


class Tuner:
    """Measures and caches launch choices for the jobs of one engine."""

    def __init__(self, eng, cache_path: str | None = None, reps: int = 3, candidates=CANDIDATES):
        self.eng = eng
        self.cache_path = cache_path
        self.reps = int(reps)
        self.candidates = tuple(candidates)
        self.table: dict = {}  # key -> {"choice": ..., "ms_per_step": {label: ms}}
        self._lock = threading.Lock()
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                self.table.update(json.load(f))

    def choose(self, spec: SimSpec, precision=None, arith: str = "fast", ring_steps: int = 32) -> dict:
        """The ``submit`` keywords for ``spec``: the cached choice of its shape
        key, measured now if the key is new."""
        if spec.mode != "yee3d":  # 2D: the tile form
            return dict(DEFAULT, variant="auto")
        key = shape_key(spec, precision, arith, ring_steps)
        with self._lock:
            hit = self.table.get(key)
        if hit is None:
            hit = self._measure(spec, precision, arith, ring_steps)
            with self._lock:
                self.table[key] = hit
                self._save()
        return dict(hit["choice"])

    def _save(self):
        if not self.cache_path:
            return
        d = os.path.dirname(os.path.abspath(self.cache_path))
        os.makedirs(d, exist_ok=True)
        tmp = self.cache_path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(self.table, f, indent=1, sort_keys=True)
        os.replace(tmp, self.cache_path)

    def time_choice(self, spec: SimSpec, choice: dict, precision=None, arith: str = "fast",
                    ring_steps: int = 32) -> float:
        """Median ms per step of ``choice`` on ``spec``'s grid (K-step blocks
        replayed from the job's graph, CUDA events on the engine stream)."""
        import torch
        K = int(ring_steps) or 32
        if choice["variant"] == "sweep" and K % 2:
            K += 1
        if spec.nt < K * (self.reps + 1):
            raise ValueError("tuning needs %d steps, the job has %d" % (K * (self.reps + 1), spec.nt))
        eng = self.eng
        job = eng.submit(spec, arith=arith, precision=precision, ring_steps=K, **choice)
        try:
            st = torch.cuda.ExternalStream(eng.stream_handle(), device=eng.device)
            job.advance(K)  # captures the block's graph
            ts = []
            for _ in range(self.reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(st)
                job.advance(K)
                e1.record(st)
                e1.synchronize()
                ts.append(e0.elapsed_time(e1) / K)
            job.sync()
        finally:
            job.release()
        return float(np.median(ts))

    def _measure(self, spec, precision, arith, ring_steps):
        times = {}
        for c in self.candidates:
            times[label(c)] = round(self.time_choice(spec, c, precision, arith, ring_steps), 5)
        best = min(self.candidates, key=lambda c: times[label(c)])
        return {"choice": dict(best), "ms_per_step": times, "measured_on": [int(n) for n in spec.shape]}

    def summary(self) -> dict:
        """Per shape key: the choice and its gain over the default form."""
        out = {}
        for key, v in sorted(self.table.items()):
            t = v["ms_per_step"]
            out[key] = {"choice": label(v["choice"]), "ms_per_step": t[label(v["choice"])],
                        "default_ms_per_step": t.get(label(DEFAULT))}
        return out
