"""Launch choices and the tuner, without a device: the descriptor fields for
tile rows and march depth are validated by the host planner, and the tuner
picks the fastest measured choice, caches it per shape key and persists it."""
import ctypes
import json

import numpy as np
import pytest

from oidt_b200 import tune
from oidt_b200 import workloads as W


def _bytes(lib, d):
    b = ctypes.c_uint64()
    return lib.oidt_job_bytes(ctypes.byref(d), ctypes.byref(b)), b.value


def _strip(**kw):
    args = dict(nx=20, ny=19, nz=40, P=4, src_gap=2, port_gap=3, steps=200, nf=2, core_x_nm=120, core_y_nm=160)
    args.update(kw)
    return W.strip3d(**args)


def test_descriptor_launch_choices_validated_on_host():
    from oidt_b200.engine import load_library
    from oidt_b200.spec import to_desc
    lib = load_library()
    spec = _strip()
    rc, base = _bytes(lib, to_desc(spec, variant="cell")[0])
    assert rc == 0
    for rows in (2, 4, 8):  # tile rows change launches, not memory
        d, keep = to_desc(spec, variant="cell", rows=rows)
        assert _bytes(lib, d) == (0, base)
    for rows in (1, 3, 16, -2):
        d, keep = to_desc(spec, variant="cell", rows=rows)
        assert _bytes(lib, d)[0] == -1, rows
    d, keep = to_desc(spec, variant="sweep", rows=4)  # rows belong to the per-cell form
    assert _bytes(lib, d)[0] == -1
    d, keep = to_desc(spec, march_depth=8)  # march depth belongs to the plane sweep
    assert _bytes(lib, d)[0] == -1
    for depth in (1, 8, 10_000):
        d, keep = to_desc(spec, variant="sweep", march_depth=depth)
        assert _bytes(lib, d)[0] == 0, depth
    d, keep = to_desc(spec, variant="sweep", march_depth=-1)
    assert _bytes(lib, d)[0] == -1
    d, keep = to_desc(spec, variant="vec")  # the vector form: x/y-slab psi rows padded like the fields
    rc, vec = _bytes(lib, d)
    assert rc == 0 and vec >= base
    for bad in (dict(rows=2), dict(march_depth=4)):  # neither choice belongs to the vector form
        d, keep = to_desc(spec, variant="vec", **bad)
        assert _bytes(lib, d)[0] == -1, bad
    slab = W.slab2d(nx=60, ny=50, P=5, core_cells=6, src_x=10, ports=(15, 45), steps=10, nf=3)
    d, keep = to_desc(slab, rows=2)  # tile rows belong to the 3D per-cell form
    assert _bytes(lib, d)[0] == -1
    for v in ("cell", "tile"):  # the 2D forms
        d, keep = to_desc(slab, variant=v)
        assert _bytes(lib, d)[0] == 0, v
    for r0 in (1, 2, 3, 5):  # 3D forms, and no such form
        d, keep = to_desc(slab)
        d.reserved[0] = r0
        assert _bytes(lib, d)[0] == -1, r0
    d, keep = to_desc(spec, variant="tile")  # the tile form is 2D only
    assert _bytes(lib, d)[0] == -1
    for steps in (1, 4, 8, 100):  # steps per launch (clamped to 8 and the ring)
        d, keep = to_desc(slab, variant="tile", tile_steps=steps)
        assert _bytes(lib, d)[0] == 0, steps
    d, keep = to_desc(slab, variant="tile", tile_steps=-1)
    assert _bytes(lib, d)[0] == -1
    d, keep = to_desc(slab, variant="cell", tile_steps=4)  # steps per launch belong to the tile form
    assert _bytes(lib, d)[0] == -1
    d, keep = to_desc(slab, variant="tile", tile_coop=False)  # one launch per sub-block: reserved[2] = 1
    assert d.reserved[2] == 1 and _bytes(lib, d)[0] == 0
    d.reserved[2] = 2  # nothing else
    assert _bytes(lib, d)[0] == -1
    assert to_desc(slab)[0].reserved[0] == 4  # 'auto': tiles in 2D


class _FakeTuner(tune.Tuner):
    """Timings from a table instead of the device."""

    def __init__(self, table, **kw):
        super().__init__(eng=None, **kw)
        self.fake = table
        self.calls = []

    def time_choice(self, spec, choice, precision=None, arith="fast", ring_steps=32):
        self.calls.append((spec.shape, tune.label(choice)))
        return self.fake[tune.label(choice)]


TIMES = {"wave": 0.0895, "vec": 0.089, "cell/rows4": 0.090, "cell/rows2": 0.093, "cell/rows8": 0.088, "sweep/depth-auto": 0.140,
         "sweep/depth16": 0.150}


def test_tuner_picks_fastest_and_caches_per_shape(tmp_path):
    path = str(tmp_path / "tune.json")
    t = _FakeTuner(TIMES, cache_path=path)
    a = _strip(nz=150)
    c = t.choose(a, np.float32)
    assert c == {"variant": "cell", "rows": 8, "march_depth": 0}
    assert len(t.calls) == len(tune.CANDIDATES)
    t.choose(_strip(nz=170), np.float32)  # same cross-section, guide length in the same 64-cell class
    assert len(t.calls) == len(tune.CANDIDATES)
    t.choose(_strip(nz=200), np.float32)  # next class: measured again
    assert len(t.calls) == 2 * len(tune.CANDIDATES)
    t.choose(a, np.float64)  # precision is part of the key
    assert len(t.calls) == 3 * len(tune.CANDIDATES)
    slab = W.slab2d(nx=60, ny=50, P=5, core_cells=6, src_x=10, ports=(15, 45), steps=10, nf=3)
    assert t.choose(slab) == dict(tune.DEFAULT, variant="auto") and len(t.calls) == 3 * len(tune.CANDIDATES)
    saved = json.load(open(path))
    assert len(saved) == 3
    # a new tuner reads the file and measures nothing for known shapes
    t2 = _FakeTuner({k: 1.0 for k in TIMES}, cache_path=path)
    assert t2.choose(a, np.float32) == c and t2.calls == []
    s = t2.summary()
    key = tune.shape_key(a, np.float32, "fast", 32)
    assert s[key]["choice"] == "cell/rows8" and s[key]["default_ms_per_step"] == TIMES["vec"]


def test_tuning_needs_enough_steps():
    t = tune.Tuner(eng=None, reps=3)
    with pytest.raises(ValueError):
        t.time_choice(_strip(steps=100), dict(tune.DEFAULT), np.float32, ring_steps=32)


@pytest.mark.parametrize("nx,ny,nz,P", [(20, 19, 40, 4), (22, 18, 64, 3), (16, 15, 32, 1), (30, 44, 128, 10)])
@pytest.mark.parametrize("prec", [np.float32, np.float64])
def test_vector_form_pads_z_slab_rows_to_whole_groups(nx, ny, nz, P, prec):
    """The vector form's z-slab psi rows hold every four-cell group that meets
    the slab: slab cell d of the low side at k - floor4(kb), of the high side
    at k - floor4(ke - P), rows of the larger span rounded up to 4.  With nz a
    multiple of 4 (x- and y-slab rows then as long as the reference's), the
    form needs exactly those eight arrays' extra bytes over the per-cell form
    (256-byte aligned sub-buffers)."""
    from oidt_b200.engine import load_library
    from oidt_b200.spec import to_desc
    lib = load_library()
    spec = _strip(nx=nx, ny=ny, nz=nz, P=P, steps=50)
    kb, ke = spec.lim_lo[2], spec.lim_hi[2]
    zoff = (kb - kb // 4 * 4, (ke - P) - (ke - P) // 4 * 4)
    psz = (max(zoff) + P + 3) // 4 * 4
    esz = np.dtype(prec).itemsize
    al = lambda x: (x + 255) // 256 * 256  # noqa: E731
    sizes = {}
    for v in ("vec", "cell"):
        d, keep = to_desc(spec, variant=v, precision=prec)
        rc, sizes[v] = _bytes(lib, d)
        assert rc == 0
    # E: Ex, Ey; H: Hx, Hy; two sides each
    assert sizes["vec"] - sizes["cell"] == 8 * (al(nx * ny * psz * esz) - al(nx * ny * P * esz))
