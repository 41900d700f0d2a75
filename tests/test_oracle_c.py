"""The C oracle (timed CPU baseline) equals the NumPy oracle bit for bit."""
import numpy as np
import pytest

from oidt_b200 import workloads as W
from oracle import cpu as OC
from oracle import fdtd_ref as R


def _cases():
    return {
        "yee3d_te": W.strip3d(nx=22, ny=19, nz=37, P=4, src_gap=2, port_gap=3, steps=40, nf=4, core_x_nm=120,
                              core_y_nm=160, sigma_nm=25, lc_nm=60, seed=5),
        "yee3d_tm": W.strip3d(nx=21, ny=24, nz=33, P=3, src_gap=2, port_gap=3, steps=40, nf=3, core_x_nm=140,
                              core_y_nm=180, source="TM", seed=6),
        "tm2": W.slab2d(nx=70, ny=61, P=5, core_cells=9, src_x=12, ports=(20, 50), steps=40, nf=5, rough=True,
                        sigma_nm=30, lc_nm=60, seed=3),
    }


@pytest.mark.parametrize("name", ["yee3d_te", "yee3d_tm", "tm2"])
def test_c_oracle_equals_numpy_oracle(name):
    OC.build()
    spec = _cases()[name]
    a, b = R.from_spec(spec), R.from_spec(spec)
    rng = np.random.default_rng(7)
    for f in R.field_names(spec.mode):
        v = rng.standard_normal(spec.shape) * 1e-2
        getattr(a, f)[...] = v
        getattr(b, f)[...] = v
    R.run(a, 23)
    OC.run_c(b, 11)
    OC.run_c(b, 12)
    for f in R.field_names(spec.mode):
        np.testing.assert_array_equal(getattr(a, f), getattr(b, f))
    for k in a.dft:
        np.testing.assert_array_equal(a.dft[k], b.dft[k])
    for k in dir(a):
        if k.startswith("PSI_"):
            np.testing.assert_array_equal(getattr(a, k), getattr(b, k))


@pytest.mark.parametrize("name", ["yee3d_te", "tm2"])
def test_c_oracle_float32_build_tracks_float64(name):
    """The float32 build of the C oracle (the CPU baseline timed at the
    engine's production precision) runs the same loop: after 23 steps from
    the same random fields its float32 fields agree with the float64 oracle
    to float32 rounding (relative L2 <= 1e-5), and its float64 DFT
    accumulators to 1e-4 of their largest magnitude."""
    OC.build()
    spec = _cases()[name]
    a, b = R.from_spec(spec), R.from_spec(spec)
    rng = np.random.default_rng(9)
    init = {}
    for f in R.field_names(spec.mode):
        v = rng.standard_normal(spec.shape) * 1e-2
        getattr(a, f)[...] = v
        getattr(b, f)[...] = v
        init[f] = v
    OC.run_c(a, 23)
    OC.run_c(b, 10, precision="float32")
    OC.run_c(b, 13, precision="float32")
    assert b.n == 23
    for f in R.field_names(spec.mode):
        got, ref = b._f32[f].astype(np.float64), getattr(a, f)
        assert b._f32[f].dtype == np.float32
        assert np.linalg.norm(got - ref) <= 1e-5 * np.linalg.norm(ref), f
        np.testing.assert_array_equal(getattr(b, f), init[f])  # the float64 arrays are not the float32 run's
    for k in a.dft:
        scale = np.max(np.abs(a.dft[k]))
        assert np.max(np.abs(a.dft[k] - b.dft[k])) <= 1e-4 * scale + 1e-300, k


def test_c_oracle_timing_continues_one_simulation():
    """time_steps times consecutive samples of one run and hands back its
    state, so a later call continues where the last sample ended."""
    spec = _cases()["tm2"]
    info, s = OC.time_steps(spec, nsteps=5, samples=2, precision="float32")
    assert s.n == 15 and info["precision"] == "float32" and info["value"] > 0
    info2, s2 = OC.time_steps(spec, nsteps=5, samples=1, precision="float32", state=s)
    assert s2 is s and s.n == 20
    with pytest.raises(ValueError):
        OC.time_steps(spec, nsteps=20, samples=2)
