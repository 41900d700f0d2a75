"""Every descriptor rule of the job planner, without a device: each mutation
of a valid 2D TM or 3D descriptor that breaks a rule is refused with
OIDT_ERR_INVALID by oidt_job_bytes (the admission check, which plans on the
host), the accepted edge cases are sized, and the sizes grow with what they
hold."""
import ctypes

import pytest

from oidt_b200 import workloads as W
from oidt_b200.spec import to_desc

INVALID = -1


@pytest.fixture(scope="module")
def lib():
    from oidt_b200.engine import load_library
    return load_library()


def _bytes(lib, d):
    b = ctypes.c_uint64()
    return lib.oidt_job_bytes(ctypes.byref(d), ctypes.byref(b)), b.value


def _d3():
    # the dt/eps grids themselves (the material-index rules: test_material_index.py)
    return to_desc(W.strip3d(nx=20, ny=19, nz=40, P=4, src_gap=2, port_gap=3, steps=30, nf=2, core_x_nm=120,
                             core_y_nm=160), material=False)


def _d2():
    return to_desc(W.slab2d(nx=60, ny=50, P=5, core_cells=6, src_x=10, ports=(15, 45), steps=10, nf=3))


def _set(d, path, v):
    obj, attr = d, path
    if "[" in path:
        attr, idx = path[:-1].split("[")
        getattr(d, attr)[int(idx)] = v
    else:
        setattr(obj, attr, v)


MUT3 = [
    ("mode", 3), ("precision", 2), ("arith", 2),
    ("nx", 4), ("nz", 4), ("num_cpml", 0), ("num_cpml", 9),          # 2 x 9 CPML cells > 16 updated
    ("ib", 0), ("kb", 0), ("ie", 20), ("ke", 40),                      # no ghost cell left
    ("nt", 0), ("nf", 0),
    ("j_src", None), ("cos_e", None), ("be", None), ("cb[1]", None), ("kdx[2]", None), ("kdx[5]", None),
    ("port_pos[0]", -1), ("port_pos[1]", 39),
    ("win_lo[1]", -1), ("win_hi[1]", 19), ("win_hi[0]", 20), ("win_lo[0]", 16),
    ("src_field", 6), ("src_lo[2]", 1), ("src_hi[1]", 19),
    ("probe[0]", 2), ("probe[1]", 3),
    ("reserved[0]", 4), ("reserved[1]", 2), ("reserved[2]", 3), ("reserved[3]", 4),
    ("ring_steps", 4097),
]

MUT2 = [
    ("nz", 2), ("src_field", 0), ("src_field", 5), ("kdx[0]", None), ("cb[2]", None),
    ("port_pos[1]", 59), ("win_hi[1]", 50), ("probe[0]", 1), ("reserved[2]", 4), ("reserved[3]", -1),
    ("reserved[0]", 1), ("reserved[0]", 2), ("reserved[0]", 5),
]


@pytest.mark.parametrize("path,value", MUT3)
def test_3d_rule_refused(lib, path, value):
    d, keep = _d3()
    assert _bytes(lib, d)[0] == 0
    _set(d, path, value)
    assert _bytes(lib, d)[0] == INVALID, (path, value)


@pytest.mark.parametrize("path,value", MUT2)
def test_2d_rule_refused(lib, path, value):
    d, keep = _d2()
    assert _bytes(lib, d)[0] == 0
    _set(d, path, value)
    assert _bytes(lib, d)[0] == INVALID, (path, value)


def test_accepted_edges_and_sizes(lib):
    d, keep = _d3()
    rc, base = _bytes(lib, d)
    assert rc == 0
    d.src_hi[0] = d.src_lo[0]  # an empty source box is allowed (no cell sourced)
    assert _bytes(lib, d)[0] == 0
    d, keep = _d3()
    d.src_field = -1  # no source at all
    assert _bytes(lib, d) == (0, base)
    d, keep = _d3()
    d.ring_steps = 4096  # the largest ring
    rc, big = _bytes(lib, d)
    assert rc == 0 and big > base
    d2, keep2 = _d2()  # 2D has no z kappa arrays
    assert d2.kdx[2] is None and _bytes(lib, d2)[0] == 0
    # more frequencies, more accumulator bytes (2 ports x 4 comps x nf x plane x 16 B, plus twiddles)
    small, k1 = to_desc(W.strip3d(nx=20, ny=19, nz=40, P=4, src_gap=2, port_gap=3, steps=30, nf=2, core_x_nm=120,
                                  core_y_nm=160))
    large, k2 = to_desc(W.strip3d(nx=20, ny=19, nz=40, P=4, src_gap=2, port_gap=3, steps=30, nf=5, core_x_nm=120,
                                  core_y_nm=160))
    assert _bytes(lib, large)[1] - _bytes(lib, small)[1] >= 3 * 2 * 4 * 20 * 19 * 16
    f64, k3 = to_desc(W.strip3d(nx=20, ny=19, nz=40, P=4, src_gap=2, port_gap=3, steps=30, nf=2, core_x_nm=120,
                                core_y_nm=160), precision="float64")
    assert _bytes(lib, f64)[1] > _bytes(lib, small)[1]


def test_plane_offsets_limit(lib):
    """The 3D kernels address an x-plane and each set of CPML slab layers
    with 32-bit offsets.  Grids whose plane, or whose P x ny x nz x-slab set,
    holds 2^31 or more elements are refused, and one just below is sized.
    Only host planning runs here; nothing is allocated."""
    d, keep = _d3()
    d.reserved[0] = 0  # the per-cell form: psi rows of nz cells
    P = d.num_cpml
    for ny, nz, ok in ((46341, 46344, False),   # the plane itself
                       (23171, 23171, False),   # P x ny x nz just above 2^31 - 1
                       (23170, 23170, True)):   # just below
        d.ny, d.nz = ny, nz
        d.je, d.ke = ny - 2, nz - 2
        d.win_hi[1] = ny - 5
        d.port_pos[0], d.port_pos[1] = 10, nz - 10
        rc, b = _bytes(lib, d)
        assert (P * ny * nz < 2 ** 31 - 1) == ok
        if ok:
            assert rc == 0 and b > ny * nz * 4 * 9 * d.nx
        else:
            assert rc == INVALID


def test_vector_form_pitched_slab_limit(lib):
    """The vector form keeps x- and y-slab psi rows padded to nzp cells, so
    its limit is P x ny x nzp < 2^31: a grid the per-cell form still takes
    (P ny nz just below the limit, nz not a multiple of 4) is refused."""
    d, keep = _d3()
    P = d.num_cpml
    ny, nz = 23170, 23170  # nzp = 23172
    d.ny, d.nz = ny, nz
    d.je, d.ke = ny - 2, nz - 2
    d.win_hi[1] = ny - 5
    d.port_pos[0], d.port_pos[1] = 10, nz - 10
    assert P * ny * nz < 2 ** 31 - 1 < P * ny * 23172
    d.reserved[0] = 0
    assert _bytes(lib, d)[0] == 0
    d.reserved[0] = 2
    assert _bytes(lib, d)[0] == INVALID
