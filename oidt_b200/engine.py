"""Python binding of ``liboidt.so`` (ctypes) and the job wrapper.

The library is built in-tree (``oidt_b200/liboidt.so``, see ``build.py``).
Importing this module on a machine without the library raises: there is no
CPU fallback for the engine.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

from .spec import DFT_COMPS, FIELD_ID, FIELDS, PSI, SimSpec, to_desc

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboidt.so")

ABI_VERSION = 5  # OIDT_ABI_VERSION of include/oidt.h
OK, ERR_INVALID, ERR_CUDA, ERR_BUDGET, ERR_NOTFOUND, ERR_TIMEOUT, ERR_STATE = 0, -1, -2, -3, -4, -5, -6
EXPORTS = ("oidt_abi_version", "oidt_create", "oidt_destroy", "oidt_last_error", "oidt_stats_get",
           "oidt_job_bytes", "oidt_job_create", "oidt_job_advance", "oidt_batch_advance", "oidt_job_sync",
           "oidt_job_query", "oidt_job_read_dft", "oidt_job_read_field", "oidt_job_write_field",
           "oidt_job_read_psi", "oidt_job_release", "oidt_job_reset", "oidt_ctx_stream", "oidt_job_profile",
           "oidt_job_read_dft_window_static", "oidt_job_read_probe", "oidt_job_port_power",
           "oidt_job_set_wait_limit")


class OidtError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("oidt error %d: %s" % (code, msg))
        self.code = code


class BudgetError(OidtError):
    pass


class TimeoutError_(OidtError):
    pass


class Stats(C.Structure):
    _fields_ = [("hbm_budget", C.c_uint64), ("hbm_in_use", C.c_uint64), ("live_jobs", C.c_int32),
                ("device", C.c_int32), ("kernel_launches", C.c_int64)]


_lib = None
_lib_lock = threading.Lock()


def load_library(path: str = LIB_PATH):
    """Load (once) and type the C ABI.  Raises if the library is missing."""
    global _lib
    with _lib_lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise ImportError("liboidt.so not found at %s; run `python -m oidt_b200.build`" % path)
        L = C.CDLL(path)
        vp, u64, i32 = C.c_void_p, C.c_uint64, C.c_int32
        sig = {
            "oidt_abi_version": ([], i32),
            "oidt_create": ([i32, u64, C.POINTER(vp)], i32),
            "oidt_destroy": ([vp], i32),
            "oidt_last_error": ([vp], C.c_char_p),
            "oidt_stats_get": ([vp, C.POINTER(Stats)], i32),
            "oidt_job_bytes": ([vp, C.POINTER(u64)], i32),
            "oidt_job_create": ([vp, vp, C.POINTER(u64)], i32),
            "oidt_job_advance": ([vp, u64, i32], i32),
            "oidt_batch_advance": ([vp, C.POINTER(u64), i32, i32], i32),
            "oidt_job_sync": ([vp, u64, i32], i32),
            "oidt_job_query": ([vp, u64, C.POINTER(i32), C.POINTER(i32)], i32),
            "oidt_job_read_dft": ([vp, u64, i32, i32, vp, C.c_size_t], i32),
            "oidt_job_read_dft_window_static": ([vp, u64, i32, i32, vp, C.c_size_t], i32),
            "oidt_job_read_probe": ([vp, u64, i32, vp, C.c_size_t], i32),
            "oidt_job_port_power": ([vp, u64, u64, i32, C.POINTER(i32), vp, C.c_size_t], i32),
            "oidt_job_read_field": ([vp, u64, i32, vp, C.c_size_t], i32),
            "oidt_job_write_field": ([vp, u64, i32, vp, C.c_size_t], i32),
            "oidt_job_read_psi": ([vp, u64, i32, i32, i32, vp, C.c_size_t], i32),
            "oidt_job_release": ([vp, u64], i32),
            "oidt_job_reset": ([vp, u64], i32),
            "oidt_ctx_stream": ([vp, C.POINTER(vp)], i32),
            "oidt_job_profile": ([vp, u64, i32, C.POINTER(C.c_float)], i32),
            "oidt_job_set_wait_limit": ([vp, u64, C.c_int64], i32),
        }
        L.oidt_abi_version.argtypes, L.oidt_abi_version.restype = [], i32
        if L.oidt_abi_version() != ABI_VERSION:
            raise ImportError("%s has ABI %d, this package needs %d; rebuild it with `python -m oidt_b200.build`"
                              % (path, L.oidt_abi_version(), ABI_VERSION))
        for name, (args, res) in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
        return L


class Engine:
    """One context on one device (``oidt_create``)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        self.lib = load_library()
        self.ctx = C.c_void_p()
        rc = self.lib.oidt_create(device, hbm_budget, C.byref(self.ctx))
        if rc != OK:
            raise OidtError(rc, "oidt_create(device=%d) failed (no usable CUDA device?)" % device)
        self.device = device

    def _check(self, rc):
        if rc == OK:
            return
        msg = self.lib.oidt_last_error(self.ctx).decode()
        if rc == ERR_BUDGET:
            raise BudgetError(rc, msg)
        if rc == ERR_TIMEOUT:
            raise TimeoutError_(rc, msg)
        raise OidtError(rc, msg)

    def close(self):
        if self.ctx:
            self.lib.oidt_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def stats(self) -> dict:
        s = Stats()
        self._check(self.lib.oidt_stats_get(self.ctx, C.byref(s)))
        return {k: getattr(s, k) for k, _ in Stats._fields_}

    def job_bytes(self, spec: SimSpec, precision=None, ring_steps=0, variant: str = "auto", march_depth: int = 0,
                  material: bool = True, tile_steps: int = 0, tile_coop: bool = True) -> int:
        d, keep = to_desc(spec, precision=precision, ring_steps=ring_steps, variant=variant, march_depth=march_depth,
                          material=material, tile_steps=tile_steps, tile_coop=tile_coop)
        b = C.c_uint64()
        self._check(self.lib.oidt_job_bytes(C.byref(d), C.byref(b)))
        return b.value

    def submit(self, spec: SimSpec, arith: str = "fast", precision=None, ring_steps: int = 0,
               variant: str = "auto", graphs: bool = True, rows: int = 0, march_depth: int = 0,
               material: bool = True, tile_steps: int = 0, tile_coop: bool = True) -> "Job":
        """Create a job (the H2D boundary).  ``variant``, ``rows``,
        ``march_depth``, ``tile_steps``, ``tile_coop`` and ``ring_steps`` choose how it is
        launched, never what it computes (``oidt_b200.tune`` picks them by
        measurement); ``material`` passes a 3D spec's material index instead
        of its three dt/eps grids (the same values)."""
        d, keep = to_desc(spec, arith=arith, precision=precision, ring_steps=ring_steps, variant=variant,
                          graphs=graphs, rows=rows, march_depth=march_depth, material=material, tile_steps=tile_steps,
                          tile_coop=tile_coop)
        jid = C.c_uint64()
        self._check(self.lib.oidt_job_create(self.ctx, C.byref(d), C.byref(jid)))
        del keep
        return Job(self, jid.value, spec, np.dtype(precision if precision is not None else spec.precision))

    def mark(self):
        """A marker of the work enqueued so far on the context's stream (a CUDA
        event); ``.synchronize()`` waits for that work."""
        import torch
        ev = torch.cuda.Event()
        ev.record(torch.cuda.ExternalStream(self.stream_handle(), device=self.device))
        return ev

    def stream_handle(self) -> int:
        """The compute stream (cudaStream_t as an integer)."""
        h = C.c_void_p()
        self._check(self.lib.oidt_ctx_stream(self.ctx, C.byref(h)))
        return h.value or 0

    def batch_advance(self, jobs, nsteps: int):
        ids = (C.c_uint64 * len(jobs))(*[j.id for j in jobs])
        self._check(self.lib.oidt_batch_advance(self.ctx, ids, len(jobs), nsteps))
        for j in jobs:
            j.steps += nsteps


class Job:
    """One simulation's device state (``oidt_job_*``)."""

    def __init__(self, eng: Engine, jid: int, spec: SimSpec, precision):
        self.eng, self.id, self.spec, self.precision = eng, jid, spec, precision
        self.steps = 0
        self.released = False

    def advance(self, nsteps: int):
        self.eng._check(self.eng.lib.oidt_job_advance(self.eng.ctx, self.id, nsteps))
        self.steps += nsteps
        return self

    def run(self):
        """Advance through every remaining source step."""
        return self.advance(self.spec.nt - self.steps)

    def sync(self, timeout_ms: int = -1):
        self.eng._check(self.eng.lib.oidt_job_sync(self.eng.ctx, self.id, timeout_ms))
        return self

    def busy(self) -> bool:
        done, busy = C.c_int32(), C.c_int32()
        self.eng._check(self.eng.lib.oidt_job_query(self.eng.ctx, self.id, C.byref(done), C.byref(busy)))
        return bool(busy.value)

    def dft(self, port: int, comp, out: np.ndarray = None) -> np.ndarray:
        """complex128 DFT of one port component, reference layout
        ([nf][nx][ny] in 3D, [nf][ny] in 2D).  ``out``: a C-contiguous
        complex128 array of that shape to read into -- in page-locked memory
        the copy runs at full link speed and touches no fresh pages."""
        comps = DFT_COMPS[self.spec.mode]
        ci = comps.index(comp) if isinstance(comp, str) else comp
        plane = self.spec.shape[:2] if self.spec.mode == "yee3d" else (self.spec.shape[1],)
        shape = (self.spec.nf,) + tuple(plane)
        if out is None:
            out = np.empty(shape, dtype=np.complex128)
        elif out.shape != shape or out.dtype != np.complex128 or not out.flags["C_CONTIGUOUS"]:
            raise ValueError("out must be a C-contiguous complex128 array of shape %s" % (shape,))
        self.eng._check(self.eng.lib.oidt_job_read_dft(self.eng.ctx, self.id, port, ci,
                                                       out.ctypes.data, out.size * 2))
        return out

    def dft_window_static(self, port: int, comp) -> np.ndarray:
        """complex128 DFT of one port component over the DFT window only
        ([nf][wi][wj] in 3D, [nf][wj] in 2D), read through the entry point
        that allocates no device memory."""
        comps = DFT_COMPS[self.spec.mode]
        ci = comps.index(comp) if isinstance(comp, str) else comp
        (i0, j0), (i1, j1) = self.spec.win_lo, self.spec.win_hi
        win = (i1 - i0, j1 - j0) if self.spec.mode == "yee3d" else (j1 - j0,)
        out = np.empty((self.spec.nf,) + win, dtype=np.complex128)
        self.eng._check(self.eng.lib.oidt_job_read_dft_window_static(self.eng.ctx, self.id, port, ci,
                                                                     out.ctypes.data, out.size * 2))
        return out

    def port_power(self, port: int, minus: "Job" = None, window=None) -> np.ndarray:
        """complex128 [nf]: the port plane's Poynting flux summed over
        ``window`` on the device in float64 (``oidt_job_port_power``).
        ``minus``: a job whose DFT at the same port is subtracted first (the
        reflected wave).  ``window`` defaults to the spec's power window:
        3D ((i0, i1), (j0, j1)) over [nx][ny], 2D (j0, j1) over ny."""
        from .spec import power_window
        w = power_window(self.spec) if window is None else window
        if self.spec.mode == "yee3d":
            (i0, i1), (j0, j1) = w
        else:
            (i0, i1), (j0, j1) = (0, 1), w
        win = (C.c_int32 * 4)(int(i0), int(i1), int(j0), int(j1))
        out = np.empty(self.spec.nf, dtype=np.complex128)
        self.eng._check(self.eng.lib.oidt_job_port_power(self.eng.ctx, self.id, minus.id if minus is not None else 0,
                                                         port, win, out.ctypes.data, out.size * 2))
        return out

    PROBE_COMPS = ("ey", "ez", "hy", "hz")

    def probe(self, comp) -> np.ndarray:
        """Line-probe record [nt, nx] of one component ('ey', 'ez', 'hy',
        'hz'), in the job's precision; rows of steps not yet run are 0."""
        ci = self.PROBE_COMPS.index(comp) if isinstance(comp, str) else comp
        out = np.zeros((self.spec.nt, self.spec.shape[0]), dtype=self.precision)
        self.eng._check(self.eng.lib.oidt_job_read_probe(self.eng.ctx, self.id, ci, out.ctypes.data, out.nbytes))
        return out

    def field(self, name: str) -> np.ndarray:
        out = np.empty(self.spec.shape, dtype=self.precision)
        self.eng._check(self.eng.lib.oidt_job_read_field(self.eng.ctx, self.id, FIELD_ID[name],
                                                         out.ctypes.data, out.nbytes))
        return out

    def set_field(self, name: str, values: np.ndarray):
        a = np.ascontiguousarray(values, dtype=self.precision)
        if a.shape != tuple(self.spec.shape):
            raise ValueError("field shape must be %s" % (self.spec.shape,))
        self.eng._check(self.eng.lib.oidt_job_write_field(self.eng.ctx, self.id, FIELD_ID[name],
                                                          a.ctypes.data, a.nbytes))

    def psi(self, name: str, axis: int, side: int) -> np.ndarray:
        out = np.empty(self.spec.psi_shape(axis), dtype=self.precision)
        self.eng._check(self.eng.lib.oidt_job_read_psi(self.eng.ctx, self.id, FIELD_ID[name], axis, side,
                                                       out.ctypes.data, out.nbytes))
        return out

    def fields(self) -> dict:
        return {f: self.field(f) for f in FIELDS[self.spec.mode]}

    def reset(self):
        """Back to step 0 with coefficients kept on the device."""
        self.eng._check(self.eng.lib.oidt_job_reset(self.eng.ctx, self.id))
        self.steps = 0
        return self

    def profile(self, nsteps: int):
        """Average per-launch device ms of (E half, H half, DFT fold) over
        ``nsteps`` un-graphed steps."""
        ms = (C.c_float * 3)()
        self.eng._check(self.eng.lib.oidt_job_profile(self.eng.ctx, self.id, nsteps, ms))
        self.steps += nsteps
        return tuple(float(v) for v in ms)

    def set_wait_limit(self, cycles: int):
        """Bound (SM cycles) on the plane-sweep kernel's waits for its tile
        loads; 0 restores the default.  For tests of the failure path."""
        self.eng._check(self.eng.lib.oidt_job_set_wait_limit(self.eng.ctx, self.id, int(cycles)))
        return self

    def release(self):
        if not self.released:
            self.eng._check(self.eng.lib.oidt_job_release(self.eng.ctx, self.id))
            self.released = True


__all__ = ["Engine", "Job", "OidtError", "BudgetError", "load_library", "EXPORTS", "LIB_PATH", "PSI"]
