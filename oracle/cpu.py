"""ctypes driver for the C oracle (``oracle/c/oracle.c``) -- TEST
INFRASTRUCTURE ONLY (the timed CPU baseline and fast float64 reference results for the tests).

``run_c(s, nsteps)`` advances an oracle state made by
``oracle.fdtd_ref.build`` / ``from_arrays`` in place, exactly as
``fdtd_ref.run`` would (the tests require bit-equality); ``time_steps``
times a bounded sample of a workload on the host cores.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import time

import numpy as np

from . import fdtd_ref as R

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "c", "oracle.c")
LIB = os.path.join(HERE, "c", "liboracle.so")

P_ = C.POINTER(C.c_double)


class OracleState(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("P", C.c_int),
                ("ib", C.c_int), ("jb", C.c_int), ("kb", C.c_int), ("ie", C.c_int), ("je", C.c_int), ("ke", C.c_int),
                ("f", P_ * 6), ("cb", P_ * 3), ("kd", P_ * 6),
                ("be", P_), ("ce", P_), ("bh", P_), ("ch", P_), ("db", C.c_double), ("dx", C.c_double),
                ("psi", P_ * 2 * 3 * 6),
                ("src_field", C.c_int), ("slo", C.c_int * 3), ("shi", C.c_int * 3),
                ("jsrc", P_), ("port", C.c_int * 2), ("nf", C.c_int), ("nt", C.c_int),
                ("tw", P_ * 4), ("dft", P_ * 2 * 4 * 2)]


def build(force=False):
    """Compile the C oracle (gcc, OpenMP, no FMA contraction)."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    flags = ["-O3", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-std=c99"]
    r = subprocess.run(["gcc"] + flags + [SRC, "-o", LIB + ".tmp", "-lm"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("gcc failed: " + r.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = C.CDLL(LIB)
        _lib.oracle_run.argtypes = [C.POINTER(OracleState), C.c_int, C.c_int, C.c_int]
        _lib.oracle_run.restype = C.c_int
        _lib.oracle_state_size.restype = C.c_int
        assert _lib.oracle_state_size() == C.sizeof(OracleState), "OracleState layout mismatch"
    return _lib


FIDX = {"EX": 0, "EY": 1, "EZ": 2, "HX": 3, "HY": 4, "HZ": 5}


def _p(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(P_)


def state_of(s) -> OracleState:
    """Pointers into the oracle namespace ``s`` (float64 only)."""
    st = OracleState()
    shape = s.shape if len(s.shape) == 3 else (s.shape[0], s.shape[1], 1)
    st.nx, st.ny, st.nz = shape
    st.P = s.P
    st.ib, st.jb, st.ie, st.je = s.ib, s.jb, s.ie, s.je
    st.kb, st.ke = (s.kb, s.ke) if s.mode == "yee3d" else (0, 1)
    for name in R.field_names(s.mode):
        st.f[FIDX[name]] = _p(getattr(s, name))
    for k, ax in enumerate("XYZ"):
        if hasattr(s, "CB" + ax):
            st.cb[k] = _p(getattr(s, "CB" + ax))
    for k, nm in enumerate(("KXE", "KYE", "KZE", "KXH", "KYH", "KZH")):
        if hasattr(s, nm):
            st.kd[k] = _p(getattr(s, nm))
    st.be, st.ce, st.bh, st.ch = _p(s.BE), _p(s.CE), _p(s.BH), _p(s.CH)
    st.db = float(s.DB)
    st.dx = float(s.cfg.delta_x)
    for name in R.field_names(s.mode):
        for a, ax in enumerate("XYZ"):
            for side, sd in enumerate(("LO", "HI")):
                key = "PSI_%s_%s%s" % (name, ax, sd)
                if hasattr(s, key):
                    st.psi[FIDX[name]][a][side] = _p(getattr(s, key))
    box = s.src_box
    st.src_field = FIDX[box[0]]
    nd = len(s.shape)
    for a in range(3):
        st.slo[a] = box[1 + a] if a < nd else 0
        st.shi[a] = box[1 + nd + a] if a < nd else 1
    st.jsrc = _p(np.ascontiguousarray(s.cfg.J_SRC, dtype=np.float64))
    s._jsrc_keep = st.jsrc
    if s.mode == "yee3d":
        st.port[0], st.port[1] = s.cfg.p1z, s.cfg.p2z
        comps = ("EX", "EY", "HX", "HY")
    else:
        st.port[0], st.port[1] = s.cfg.p1x, s.cfg.p2x
        comps = ("E", "H")
    st.nf = s.nf
    st.nt = s.cosE.shape[1]
    for k, t in enumerate((s.cosE, s.sinE, s.cosH, s.sinH)):
        st.tw[k] = _p(t)
    for q in range(2):
        for c, cn in enumerate(comps):
            for ri, r in enumerate("ri"):
                st.dft[q][c][ri] = _p(s.dft["%s%d%s" % (cn, q + 1, r)])
    return st


def run_c(s, nsteps):
    """Advance the oracle state ``s`` (tm2 or yee3d, float64) by nsteps."""
    if s.mode not in ("tm2", "yee3d"):
        raise NotImplementedError("the C oracle covers the 2D TM and 3D solvers")
    jsrc = np.ascontiguousarray(s.cfg.J_SRC, dtype=np.float64)
    st = state_of(s)
    st.jsrc = jsrc.ctypes.data_as(P_)
    rc = lib().oracle_run(C.byref(st), 2 if s.mode == "yee3d" else 0, s.n, nsteps)
    if rc != 0:
        raise RuntimeError("oracle_run failed")
    s.n += nsteps
    return s


def threads():
    return int(os.environ.get("OMP_NUM_THREADS") or os.cpu_count() or 1)


def time_steps(spec, target_s=15.0, max_steps=None):
    """Gcell-updates/s of the float64 C oracle on the host cores over a
    bounded sample: the workload's first time steps, as many as fit in about
    ``target_s`` seconds (at least 2)."""
    s = R.from_spec(spec)
    t0 = time.perf_counter()
    run_c(s, 1)
    one = time.perf_counter() - t0
    n = max(2, int(target_s / max(one, 1e-6)))
    n = min(n, spec.nt - 1) if max_steps is None else min(n, max_steps, spec.nt - 1)
    t0 = time.perf_counter()
    run_c(s, n)
    el = time.perf_counter() - t0
    v = spec.ncells * n / el / 1e9
    return {"value": round(v, 5), "unit": "Gcell/s", "cores": threads(), "kind": "port",
            "sample": "first %d of %d time steps of the same workload, float64, C/OpenMP oracle" % (n, spec.nt),
            "ms_per_time_step": el / n * 1e3}
