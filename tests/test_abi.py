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
    from oidt_b200.engine import ABI_VERSION
    header = open(os.path.join(ROOT, "include", "oidt.h")).read()
    assert f() == ABI_VERSION == int(re.search(r"#define OIDT_ABI_VERSION (\d+)", header).group(1))


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


def test_line_probe_descriptor_without_device():
    """The line probe is 3D only, needs y + 1 < ny and z + 1 < nz, and adds
    its [4][nt][nx] record to the job's device bytes."""
    from oidt_b200 import workloads as W
    from oidt_b200.engine import load_library
    from oidt_b200.spec import to_desc
    lib = load_library()
    spec = W.strip3d(nx=20, ny=19, nz=40, P=4, src_gap=2, port_gap=3, steps=30, nf=2, core_x_nm=120,
                     core_y_nm=160)
    b0, b1 = ctypes.c_uint64(), ctypes.c_uint64()
    d, keep = to_desc(spec)
    assert lib.oidt_job_bytes(ctypes.byref(d), ctypes.byref(b0)) == 0
    spec.meta["probe"] = (9, 20)
    d, keep = to_desc(spec)
    assert list(d.probe) == [1, 9, 20] and list(d.reserved) == [2, 0, 0, 0]  # the vector launch form
    assert lib.oidt_job_bytes(ctypes.byref(d), ctypes.byref(b1)) == 0
    assert b1.value - b0.value >= 4 * 30 * 20 * 4  # float32 record [4][nt][nx]
    for bad in ((1, 18, 20), (1, 9, 39), (1, -1, 20), (2, 9, 20), (0, 9, 20)):
        d.probe[0], d.probe[1], d.probe[2] = bad
        assert lib.oidt_job_bytes(ctypes.byref(d), ctypes.byref(b1)) == -1, bad
    spec2 = W.slab2d(nx=60, ny=50, P=5, core_cells=6, src_x=10, ports=(15, 45), steps=10, nf=3)
    spec2.meta["probe"] = (5, 0)
    d2, keep2 = to_desc(spec2)
    assert lib.oidt_job_bytes(ctypes.byref(d2), ctypes.byref(b1)) == -1  # 2D: no line probe


def test_library_of_another_abi_is_refused(tmp_path, monkeypatch):
    """A stale liboidt.so (another OIDT_ABI_VERSION) is refused at load time
    instead of being called with a descriptor it reads differently."""
    import subprocess
    from oidt_b200 import engine
    src = tmp_path / "stub.c"
    src.write_text("int oidt_abi_version(void) { return %d; }\n" % (engine.ABI_VERSION - 1))
    so = tmp_path / "libstub.so"
    subprocess.run(["gcc", "-shared", "-fPIC", "-o", str(so), str(src)], check=True)
    monkeypatch.setattr(engine, "_lib", None)
    with pytest.raises(ImportError, match="ABI %d" % (engine.ABI_VERSION - 1)):
        engine.load_library(str(so))
    assert engine._lib is None
