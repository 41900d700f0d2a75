"""The C ABI library loads and exports every function include/oidt.h declares
(no device calls: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "oidt.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(oidt_[a-z_0-9]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared()
    assert "oidt_job_create" in names and "oidt_job_advance" in names and len(names) >= 16


def test_library_exports_all_declared_symbols():
    from oidt_b200.build import build
    from oidt_b200.engine import EXPORTS, LIB_PATH
    build()
    lib = ctypes.CDLL(LIB_PATH)
    for n in declared():
        assert hasattr(lib, n), n
    assert set(EXPORTS) <= set(declared())
    f = lib.oidt_abi_version
    f.restype = ctypes.c_int32
    assert f() == 2


def test_descriptor_validation_without_device():
    """oidt_job_bytes plans memory on the host: bad descriptors are
    rejected with OIDT_ERR_INVALID, good ones sized."""
    from oidt_b200 import workloads as W
    from oidt_b200.engine import load_library
    from oidt_b200.spec import to_desc
    lib = load_library()
    spec = W.slab2d(nx=60, ny=50, P=5, core_cells=6, src_x=10, ports=(15, 45), steps=10, nf=3)
    d, keep = to_desc(spec)
    b = ctypes.c_uint64()
    assert lib.oidt_job_bytes(ctypes.byref(d), ctypes.byref(b)) == 0 and b.value > 60 * 50 * 4
    d.num_cpml = 40  # slabs overlap
    assert lib.oidt_job_bytes(ctypes.byref(d), ctypes.byref(b)) == -1
    d.num_cpml = 5
    d.src_lo[0] = 0  # source on the PEC rim
    assert lib.oidt_job_bytes(ctypes.byref(d), ctypes.byref(b)) == -1
