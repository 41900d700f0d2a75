"""A 3D job created from the material index computes what the same job
created from the three dt/eps grids computes, bit for bit, in every launch
form and both precisions (the vector form reads the index, the others the
grids the engine expands from it); an index value beyond the table is
refused at job creation."""
import numpy as np
import pytest

from oidt_b200 import workloads as W
from oidt_b200.engine import Engine, OidtError

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = Engine(0)
    yield e
    e.close()


@pytest.mark.parametrize("variant", ["vec", "wave", "cell", "sweep"])
@pytest.mark.parametrize("prec,arith", [(np.float32, "fast"), (np.float64, "exact")])
def test_index_equals_grids(eng, variant, prec, arith):
    spec = W.strip3d(nx=30, ny=44, nz=130, P=4, src_gap=2, port_gap=26, steps=40, nf=3, core_x_nm=160,
                     core_y_nm=240, sigma_nm=20, lc_nm=60, seed=7)
    a = eng.submit(spec, arith=arith, precision=prec, variant=variant, ring_steps=8)
    b = eng.submit(spec, arith=arith, precision=prec, variant=variant, ring_steps=8, material=False)
    for j in (a, b):
        j.run().sync(60000)
    for f in ("EX", "EY", "EZ", "HX", "HY", "HZ"):
        np.testing.assert_array_equal(a.field(f), b.field(f), err_msg=f)
    for p in (0, 1):
        for c in range(4):
            np.testing.assert_array_equal(a.dft(p, c), b.dft(p, c))
    a.release()
    b.release()


def test_index_beyond_table_refused(eng):
    spec = W.strip3d(nx=20, ny=19, nz=40, P=4, src_gap=2, port_gap=3, steps=10, nf=2, core_x_nm=120,
                     core_y_nm=160)
    spec.mat_idx = spec.mat_idx.copy()
    spec.mat_idx[3, 4, 5] = len(spec.mat_tab)
    with pytest.raises(OidtError, match="material index"):
        eng.submit(spec)
    assert eng.stats()["live_jobs"] == 0
