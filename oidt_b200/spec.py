"""Engine job description (host side) and its C-ABI form.

A :class:`SimSpec` carries every array and scalar one simulation needs, in
the reference's layout and naming; :func:`to_desc` turns it into the
``oidt_job_desc`` struct of ``include/oidt.h`` (host pointers that the
library copies once at job creation).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

MODE_ID = {"tm2": 0, "te2": 1, "yee3d": 2}
FIELD_ID = {"EX": 0, "EY": 1, "EZ": 2, "HX": 3, "HY": 4, "HZ": 5}
FIELDS = {"tm2": ("EZ", "HX", "HY"), "te2": ("EX", "EY", "HZ"), "yee3d": ("EX", "EY", "EZ", "HX", "HY", "HZ")}
# DFT components per port, in ABI order (oidt_job_read_dft comp index)
DFT_COMPS = {"tm2": ("ez", "hy"), "te2": ("ey", "hz"), "yee3d": ("ex", "ey", "hx", "hy")}
# CPML psi arrays per solver: (field, slab axis)
PSI = {"tm2": (("EZ", 0), ("EZ", 1), ("HX", 1), ("HY", 0)),
       "te2": (("EX", 1), ("EY", 0), ("HZ", 0), ("HZ", 1)),
       "yee3d": (("EX", 1), ("EX", 2), ("EY", 0), ("EY", 2), ("EZ", 0), ("EZ", 1),
                 ("HX", 1), ("HX", 2), ("HY", 0), ("HY", 2), ("HZ", 0), ("HZ", 1))}


@dataclass
class SimSpec:
    mode: str
    precision: np.dtype
    shape: tuple
    num_cpml: int
    lim_lo: tuple
    lim_hi: tuple
    cb: dict          # 'x'/'y'/'z' -> dt/eps grid of that E component
    kdx: dict         # 'xe','xh','ye','yh'[,'ze','zh'] -> kappa*dx
    be: np.ndarray
    ce: np.ndarray
    bh: np.ndarray
    ch: np.ndarray
    db: float
    dx: float
    src_field: int
    src_lo: tuple
    src_hi: tuple
    j_src: np.ndarray
    port_pos: tuple
    win_lo: tuple
    win_hi: tuple
    freqs: np.ndarray
    twiddles: tuple   # cosE, sinE, cosH, sinH, float64 [nf][nt]
    nt: int
    meta: dict = field(default_factory=dict)
    # optional (3D): the dt/eps grids as a one-byte material index [nx][ny][nz]
    # and its float64 table [nmat][3]; tab[idx] equals (cb['x'], cb['y'], cb['z'])
    # (whoever changes cb drops these or rebuilds them)
    mat_idx: np.ndarray = None
    mat_tab: np.ndarray = None

    @property
    def ncells(self) -> int:
        return int(np.prod(self.shape))

    @property
    def nf(self) -> int:
        return len(self.freqs)

    def psi_shape(self, axis: int) -> tuple:
        s = list(self.shape)
        s[axis] = self.num_cpml
        return tuple(s)


class JobDesc(C.Structure):
    _fields_ = [
        ("mode", C.c_int32), ("precision", C.c_int32), ("arith", C.c_int32),
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("num_cpml", C.c_int32),
        ("ib", C.c_int32), ("jb", C.c_int32), ("kb", C.c_int32),
        ("ie", C.c_int32), ("je", C.c_int32), ("ke", C.c_int32),
        ("nt", C.c_int32), ("nf", C.c_int32),
        ("cb", C.c_void_p * 3), ("kdx", C.c_void_p * 6),
        ("be", C.c_void_p), ("ce", C.c_void_p), ("bh", C.c_void_p), ("ch", C.c_void_p),
        ("db", C.c_double), ("dx", C.c_double),
        ("src_field", C.c_int32), ("src_lo", C.c_int32 * 3), ("src_hi", C.c_int32 * 3),
        ("j_src", C.c_void_p),
        ("port_pos", C.c_int32 * 2), ("win_lo", C.c_int32 * 2), ("win_hi", C.c_int32 * 2),
        ("cos_e", C.c_void_p), ("sin_e", C.c_void_p), ("cos_h", C.c_void_p), ("sin_h", C.c_void_p),
        ("ring_steps", C.c_int32), ("reserved", C.c_int32 * 4), ("probe", C.c_int32 * 3),
        ("mat_idx", C.c_void_p), ("mat_tab", C.c_void_p), ("nmat", C.c_int32),
    ]


VARIANTS = {"cell": 0, "sweep": 1, "vec": 2, "wave": 3, "tile": 4}


def resolve_variant(spec: "SimSpec", variant: str) -> str:
    """'auto': the vector form in 3D, the tile form in 2D."""
    if variant != "auto":
        return variant
    return "vec" if spec.mode == "yee3d" else "tile"


def power_window(spec: SimSpec):
    """The window S-parameter powers are summed over: ``meta['power_window']``
    if set, else the DFT window.  3D ((i0, i1), (j0, j1)) over the [nx][ny]
    port plane; 2D (j0, j1) over its ny cells."""
    w = spec.meta.get("power_window")
    if spec.mode == "yee3d":
        return tuple(map(tuple, w)) if w else ((spec.win_lo[0], spec.win_hi[0]), (spec.win_lo[1], spec.win_hi[1]))
    return tuple(w) if w else (spec.win_lo[1], spec.win_hi[1])


def to_desc(spec: SimSpec, arith: str = "fast", precision=None, ring_steps: int = 0, variant: str = "auto",
            graphs: bool = True, rows: int = 0, march_depth: int = 0, material: bool = True, tile_steps: int = 0,
            tile_coop: bool = True):
    """Build the ABI descriptor; returns (desc, keepalive) -- the arrays in
    ``keepalive`` must outlive the ``oidt_job_create`` call.

    ``variant``: 'auto' (default) picks 'vec' in 3D and 'tile' in 2D.
    3D: 'vec' -- the E-half / H-half launches with four cells per thread
    along z and 16-byte accesses; 'wave' -- the same code in one launch per
    step, E and H half-steps ordered plane by plane; 'cell' -- the
    half-steps with one cell per thread; 'sweep' -- one plane-sweep launch
    per step (E and H fused, TMA-staged tiles).  2D: 'cell' -- the E-half /
    H-half launches with one cell per thread; 'tile' -- each block advances
    a tile of the grid (and a halo around it) in shared memory through
    sub-blocks of up to 8 steps.  ``tile_steps`` (2D tile form): steps per
    sub-block, 1 to 8 (0 = the engine's estimate); ``tile_coop``: a ring
    block in one cooperative launch where every tile fits on the device at
    once (default), else one launch per sub-block.  ``graphs=False``
    launches every step directly instead of replaying K-step CUDA graphs.
    ``rows`` (3D per-cell form): tile rows of a block, 2, 4 or 8 (0 = 4);
    ``march_depth`` (3D plane sweep): x-planes per work item (0 = the
    engine's makespan estimate).  ``oidt_b200.tune`` measures both.
    ``material``: pass the spec's material index (if it has one) instead of
    the three dt/eps grids -- the same values, one byte per cell."""
    prec = np.dtype(precision if precision is not None else spec.precision)
    if prec not in (np.dtype(np.float32), np.dtype(np.float64)):
        raise ValueError("precision must be float32 or float64")
    keep = []

    def arr(a, dt=prec):
        a = np.ascontiguousarray(np.asarray(a, dtype=dt))
        keep.append(a)
        return a.ctypes.data

    d = JobDesc()
    d.mode = MODE_ID[spec.mode]
    d.precision = 0 if prec == np.float32 else 1
    d.arith = {"fast": 0, "exact": 1}[arith]
    sh = tuple(spec.shape) + ((1,) if len(spec.shape) == 2 else ())
    d.nx, d.ny, d.nz = sh
    d.num_cpml = spec.num_cpml
    lo = tuple(spec.lim_lo) + ((0,) if len(spec.shape) == 2 else ())
    hi = tuple(spec.lim_hi) + ((1,) if len(spec.shape) == 2 else ())
    d.ib, d.jb, d.kb = lo
    d.ie, d.je, d.ke = hi
    d.nt = spec.nt
    d.nf = spec.nf
    if material and spec.mat_idx is not None and spec.mode == "yee3d":
        d.mat_idx = arr(spec.mat_idx, np.uint8)
        d.mat_tab = arr(spec.mat_tab)
        d.nmat = len(spec.mat_tab)
    else:
        for slot, ax in enumerate("xyz"):
            if ax in spec.cb:
                d.cb[slot] = arr(spec.cb[ax])
    for slot, key in enumerate(("xe", "ye", "ze", "xh", "yh", "zh")):
        if key in spec.kdx:
            d.kdx[slot] = arr(spec.kdx[key])
    d.be, d.ce, d.bh, d.ch = arr(spec.be), arr(spec.ce), arr(spec.bh), arr(spec.ch)
    d.db = float(spec.db)
    d.dx = float(spec.dx)
    d.src_field = spec.src_field
    for a in range(3):
        d.src_lo[a] = spec.src_lo[a] if a < len(spec.src_lo) else 0
        d.src_hi[a] = spec.src_hi[a] if a < len(spec.src_hi) else 1
    js = np.zeros(spec.nt, dtype=prec)
    js[:len(spec.j_src)] = spec.j_src[:spec.nt]
    d.j_src = arr(js)
    d.port_pos[0], d.port_pos[1] = spec.port_pos
    d.win_lo[0], d.win_lo[1] = spec.win_lo
    d.win_hi[0], d.win_hi[1] = spec.win_hi
    tw = [arr(t, np.float64) for t in spec.twiddles]
    d.cos_e, d.sin_e, d.cos_h, d.sin_h = tw
    d.ring_steps = ring_steps
    v = resolve_variant(spec, variant)
    d.reserved[0] = VARIANTS[v]
    d.reserved[1] = 0 if graphs else 1
    d.reserved[2] = int(rows)
    if v == "tile" and not tile_coop:
        d.reserved[2] = 1
    d.reserved[3] = int(march_depth) or int(tile_steps)
    probe = spec.meta.get("probe")  # (y, z) of a 3D line probe along x
    if probe is not None:
        d.probe[0], d.probe[1], d.probe[2] = 1, int(probe[0]), int(probe[1])
    return d, keep
