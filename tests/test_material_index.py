"""The dt/eps grids as a one-byte material index (oidt_job_desc.mat_idx):
the workload builders' index and table reproduce the three grids bit for bit
(float64, and after the float32 cast a job makes), and the descriptor rules
refuse what the engine cannot use.  Host planning only; nothing allocated."""
import ctypes

import numpy as np
import pytest

from oidt_b200 import workloads as W
from oidt_b200.spec import to_desc

INVALID = -1


def _lib():
    from oidt_b200.engine import load_library
    return load_library()


def _bytes(lib, d):
    b = ctypes.c_uint64()
    return lib.oidt_job_bytes(ctypes.byref(d), ctypes.byref(b)), b.value


@pytest.mark.parametrize("kw", [dict(nx=22, ny=19, nz=37, P=4, src_gap=2, port_gap=3, steps=20, nf=2, core_x_nm=120,
                                     core_y_nm=160, sigma_nm=25, lc_nm=60, seed=5),
                                dict(nx=40, ny=40, nz=40, dx=15e-9, P=4, src_gap=2, port_gap=3, steps=10, nf=2,
                                     core_x_nm=300, core_y_nm=150, slab_y_nm=60, seed=7),
                                dict(nx=30, ny=28, nz=44, P=4, src_gap=2, port_gap=3, steps=10, nf=2, rough=False)])
def test_index_reproduces_the_grids(kw):
    spec = W.strip3d(**kw)
    assert spec.mat_idx.dtype == np.uint8 and spec.mat_idx.shape == spec.shape
    assert 1 <= len(spec.mat_tab) <= 18
    tab = spec.mat_tab[spec.mat_idx]
    for c, a in enumerate("xyz"):
        np.testing.assert_array_equal(tab[..., c], spec.cb[a])
        np.testing.assert_array_equal(tab[..., c].astype(np.float32), spec.cb[a].astype(np.float32))


def test_descriptor_rules():
    lib = _lib()
    spec = W.strip3d(nx=20, ny=19, nz=40, P=4, src_gap=2, port_gap=3, steps=30, nf=2, core_x_nm=120, core_y_nm=160)
    d, keep = to_desc(spec, material=False)
    rc, grids = _bytes(lib, d)
    assert rc == 0
    d, keep = to_desc(spec)
    assert d.nmat == len(spec.mat_tab) and not any(d.cb)  # the index replaces the grids
    rc, idx = _bytes(lib, d)
    assert rc == 0 and idx >= grids + 20 * 19 * 40  # plus one byte per cell and the table
    for field, value in (("nmat", 0), ("nmat", 257), ("mat_tab", None), ("mat_idx", None)):
        d, keep = to_desc(spec)
        setattr(d, field, value)
        assert _bytes(lib, d)[0] == INVALID, (field, value)
    slab = W.slab2d(nx=60, ny=50, P=5, core_cells=6, src_x=10, ports=(15, 45), steps=10, nf=3)
    d, keep = to_desc(slab)
    d.mat_idx, d.mat_tab, d.nmat = d.cb[2], d.cb[2], 1  # 2D has no index form
    assert _bytes(lib, d)[0] == INVALID
