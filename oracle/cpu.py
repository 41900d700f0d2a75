"""ctypes driver for the C oracle (``oracle/c/oracle.c``) -- TEST
INFRASTRUCTURE ONLY (the timed CPU baseline and fast float64 reference results for the tests).

``run_c(s, nsteps)`` advances an oracle state made by
``oracle.fdtd_ref.build`` / ``from_arrays`` in place, exactly as
``fdtd_ref.run`` would (the tests require bit-equality); ``time_steps``
times a bounded sample of a workload on the host cores, in float64 (the
oracle itself) or float32 (the same source built with ``-DORACLE_REAL=float``:
fields, coefficients and psi in float32, DFT accumulators in float64, the
precision of the engine's production path and the reference's default).
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
LIB32 = os.path.join(HERE, "c", "liboracle_f32.so")

P_ = C.POINTER(C.c_double)


def _state_type(real):
    """ctypes mirror of OracleState with fields, coefficients and psi of type
    ``real`` (c_double or c_float); twiddles and DFT accumulators are double."""
    R_ = C.POINTER(real)

    class S(C.Structure):
        _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("P", C.c_int),
                    ("ib", C.c_int), ("jb", C.c_int), ("kb", C.c_int), ("ie", C.c_int), ("je", C.c_int),
                    ("ke", C.c_int),
                    ("f", R_ * 6), ("cb", R_ * 3), ("kd", R_ * 6),
                    ("be", R_), ("ce", R_), ("bh", R_), ("ch", R_), ("db", real), ("dx", real),
                    ("psi", R_ * 2 * 3 * 6),
                    ("src_field", C.c_int), ("slo", C.c_int * 3), ("shi", C.c_int * 3),
                    ("jsrc", R_), ("port", C.c_int * 2), ("nf", C.c_int), ("nt", C.c_int),
                    ("tw", P_ * 4), ("dft", P_ * 2 * 4 * 2)]
    return S


OracleState = _state_type(C.c_double)
OracleState32 = _state_type(C.c_float)


def build(force=False):
    """Compile the C oracle (gcc, OpenMP, no FMA contraction): the float64
    library and its float32 build."""
    flags = ["-O3", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-std=c99"]
    for out, extra in ((LIB, []), (LIB32, ["-DORACLE_REAL=float"])):
        if not force and os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(SRC):
            continue
        r = subprocess.run(["gcc"] + flags + extra + [SRC, "-o", out + ".tmp", "-lm"], capture_output=True,
                           text=True)
        if r.returncode != 0:
            raise RuntimeError("gcc failed: " + r.stderr)
        os.replace(out + ".tmp", out)
    return LIB


_libs = {}


def lib(precision="float64"):
    """The float64 oracle library, or with precision 'float32' its float32 build."""
    key = np.dtype(precision).name
    if key not in _libs:
        path, st, size = (LIB, OracleState, 8) if key == "float64" else (LIB32, OracleState32, 4)
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(SRC):
            build()
        L = C.CDLL(path)
        L.oracle_run.argtypes = [C.POINTER(st), C.c_int, C.c_int, C.c_int]
        L.oracle_run.restype = C.c_int
        L.oracle_state_size.restype = C.c_int
        L.oracle_real_size.restype = C.c_int
        assert L.oracle_state_size() == C.sizeof(st), "OracleState layout mismatch"
        assert L.oracle_real_size() == size, "oracle element size mismatch"
        _libs[key] = L
    return _libs[key]


FIDX = {"EX": 0, "EY": 1, "EZ": 2, "HX": 3, "HY": 4, "HZ": 5}


def _p(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(P_)


def state_of(s, precision="float64"):
    """Pointers into the oracle namespace ``s``.  float64: the namespace's own
    arrays (results land there).  float32: float32 copies of the fields,
    coefficients, psi and source, made once and kept on ``s`` so successive
    calls continue one simulation; twiddles and DFT accumulators are the
    namespace's float64 arrays."""
    f32 = np.dtype(precision) == np.float32
    st = (OracleState32 if f32 else OracleState)()
    if f32:
        R_ = C.POINTER(C.c_float)
        if getattr(s, "_f32", None) is None:
            s._f32 = {}

        def _r(name, a):
            if name not in s._f32:
                s._f32[name] = np.ascontiguousarray(a, dtype=np.float32)
            return s._f32[name].ctypes.data_as(R_)
    else:
        def _r(name, a):
            return _p(a)
    shape = s.shape if len(s.shape) == 3 else (s.shape[0], s.shape[1], 1)
    st.nx, st.ny, st.nz = shape
    st.P = s.P
    st.ib, st.jb, st.ie, st.je = s.ib, s.jb, s.ie, s.je
    st.kb, st.ke = (s.kb, s.ke) if s.mode == "yee3d" else (0, 1)
    for name in R.field_names(s.mode):
        st.f[FIDX[name]] = _r(name, getattr(s, name))
    for k, ax in enumerate("XYZ"):
        if hasattr(s, "CB" + ax):
            st.cb[k] = _r("CB" + ax, getattr(s, "CB" + ax))
    for k, nm in enumerate(("KXE", "KYE", "KZE", "KXH", "KYH", "KZH")):
        if hasattr(s, nm):
            st.kd[k] = _r(nm, getattr(s, nm))
    st.be, st.ce, st.bh, st.ch = (_r(n, getattr(s, n)) for n in ("BE", "CE", "BH", "CH"))
    st.db = float(s.DB)
    st.dx = float(s.cfg.delta_x)
    for name in R.field_names(s.mode):
        for a, ax in enumerate("XYZ"):
            for side, sd in enumerate(("LO", "HI")):
                key = "PSI_%s_%s%s" % (name, ax, sd)
                if hasattr(s, key):
                    st.psi[FIDX[name]][a][side] = _r(key, getattr(s, key))
    box = s.src_box
    st.src_field = FIDX[box[0]]
    nd = len(s.shape)
    for a in range(3):
        st.slo[a] = box[1 + a] if a < nd else 0
        st.shi[a] = box[1 + nd + a] if a < nd else 1
    if f32:
        st.jsrc = _r("J_SRC", s.cfg.J_SRC)
    else:
        s._jsrc_keep = np.ascontiguousarray(s.cfg.J_SRC, dtype=np.float64)
        st.jsrc = _p(s._jsrc_keep)
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


def run_c(s, nsteps, precision="float64"):
    """Advance the oracle state ``s`` (tm2 or yee3d) by nsteps: in float64 on
    its own arrays, or in float32 on the float32 copies ``state_of`` keeps."""
    if s.mode not in ("tm2", "yee3d"):
        raise NotImplementedError("the C oracle covers the 2D TM and 3D solvers")
    st = state_of(s, precision)
    rc = lib(precision).oracle_run(C.byref(st), 2 if s.mode == "yee3d" else 0, s.n, nsteps)
    if rc != 0:
        raise RuntimeError("oracle_run failed")
    s.n += nsteps
    return s


def threads():
    return int(os.environ.get("OMP_NUM_THREADS") or os.cpu_count() or 1)


def time_steps(spec, nsteps=150, samples=3, precision="float32", state=None):
    """Gcell-updates/s of the C oracle on the host cores: ``samples`` timed
    runs of ``nsteps`` consecutive time steps of the workload, continuing one
    simulation from its first step (an untimed first sample warms the caches
    and threads up), median of the samples.  ``precision``: 'float32' (fields,
    coefficients, psi) or 'float64'.  Returns the figures and the state, which
    a later call can continue (``state=``)."""
    prec = np.dtype(precision).name
    s = state if state is not None else R.from_spec(spec)
    if state is None:
        if s.n + nsteps * (samples + 1) > spec.nt:
            raise ValueError("the workload has %d steps; %d samples of %d need more" % (spec.nt, samples + 1, nsteps))
        run_c(s, nsteps, prec)
    ms = []
    for _ in range(samples):
        t0 = time.perf_counter()
        run_c(s, nsteps, prec)
        ms.append((time.perf_counter() - t0) * 1e3)
    med = float(np.median(ms))
    v = spec.ncells * nsteps / (med * 1e-3) / 1e9
    return {"value": round(v, 5), "unit": "Gcell/s", "cores": threads(), "kind": "port",
            "precision": prec,
            "sample": "%d consecutive time steps of the %d-step workload per sample, median of %d samples, %s, "
                      "C/OpenMP oracle" % (nsteps, spec.nt, samples, prec),
            "ms_per_sample": round(med, 3), "ms_per_time_step": round(med / nsteps, 4)}, s
