"""EXACT arithmetic across the floating-point range, on a B200.

EXACT divisions (by kappa dx and by dx) are computed from the correctly
rounded reciprocal with two FMA corrections, and divided directly where the
numerator, quotient or reciprocal leave the range in which the corrections are
exact.  These runs start from random fields whose magnitudes spread over the
whole range of the precision -- float32 subnormals, float64 values near 1e-300
and near 1e250 -- so every path (corrected, direct, zero, overflow to inf and
NaN) is taken, and compare fields and CPML psi with the C oracle (IEEE
division, no FMA contraction) bit for bit, in float64 and float32.
"""
import numpy as np
import pytest

from oracle import cpu as OC
from oracle import fdtd_ref as R
from tests.helpers import oracle_from_spec, psi_key

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    from oidt_b200.engine import Engine
    e = Engine(0)
    yield e
    e.close()


def _spec(kind):
    from oidt_b200 import workloads as W
    if kind == "tm2":
        return W.slab2d(nx=70, ny=61, P=5, core_cells=9, src_x=12, ports=(20, 50), steps=40, nf=3,
                        rough=True, sigma_nm=30, lc_nm=60, seed=3)
    return W.strip3d(nx=22, ny=19, nz=37, P=4, src_gap=2, port_gap=3, steps=40, nf=3,
                     core_x_nm=120, core_y_nm=160, sigma_nm=25, lc_nm=60, seed=5)


def _spread(rng, shape, prec):
    """Random signs and magnitudes log-uniform over the precision's range
    (float32: 1e-44 .. 1e30, subnormals included; float64: 1e-300 .. 1e250),
    a tenth of the cells zero."""
    lo, hi = (-44.0, 30.0) if prec == np.float32 else (-300.0, 250.0)
    v = np.sign(rng.standard_normal(shape)) * 10.0 ** rng.uniform(lo, hi, shape)
    v[rng.random(shape) < 0.1] = 0.0
    return v.astype(prec).astype(np.float64)


@pytest.mark.parametrize("prec", [np.float64, np.float32])
@pytest.mark.parametrize("kind,variant", [("tm2", "tile"), ("tm2", "cell"), ("yee3d", "vec"), ("yee3d", "cell")])
def test_exact_matches_oracle_across_magnitudes(eng, kind, variant, prec):
    spec = _spec(kind)
    s = oracle_from_spec(spec)
    rng = np.random.default_rng(7 + (prec == np.float32))
    job = eng.submit(spec, arith="exact", precision=prec, ring_steps=6, variant=variant)
    for f in R.field_names(spec.mode):
        v = _spread(rng, spec.shape, prec)
        getattr(s, f)[...] = v
        job.set_field(f, v.astype(prec))
    job.advance(9).sync(60000)
    with np.errstate(all="ignore"):
        OC.run_c(s, 9, precision=np.dtype(prec).name)
    ref = s._f32 if prec == np.float32 else None
    for f in R.field_names(spec.mode):
        want = ref[f] if ref is not None else getattr(s, f)
        np.testing.assert_array_equal(job.field(f), want, err_msg=f)
    from oidt_b200.spec import PSI
    for name, axis in PSI[spec.mode]:
        for side in (0, 1):
            key = psi_key(name, axis, side)
            want = ref[key] if ref is not None else getattr(s, key)
            np.testing.assert_array_equal(job.psi(name, axis, side), want, err_msg=key)
    job.release()
