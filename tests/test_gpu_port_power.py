"""Port powers summed on the device (oidt_job_port_power) against the same
sums formed on the host from the read-back DFT planes, for all three
solvers; the forward-protocol S-parameters from either; and the error
paths.  The device sums in a fixed tree order, the host in NumPy's
pairwise order, so they agree to float64 rounding (rtol 1e-12)."""
import numpy as np
import pytest

from oidt_b200 import workloads as W
from oidt_b200.sparams import forward_s, forward_s_device, power_density
from oidt_b200.spec import power_window

pytestmark = pytest.mark.gpu

RTOL = 1e-12


@pytest.fixture(scope="module")
def eng():
    from oidt_b200.engine import Engine
    e = Engine(0)
    yield e
    e.close()


def _te2():
    from tests.test_gpu_parity import _te2_spec
    return _te2_spec()


def _specs(mode):
    if mode == "yee3d":
        kw = dict(nx=22, ny=19, nz=37, P=4, src_gap=2, port_gap=3, steps=60, nf=5, core_x_nm=120, core_y_nm=160)
        return W.strip3d(rough=False, **kw), W.strip3d(sigma_nm=25, lc_nm=60, seed=5, **kw)
    if mode == "tm2":
        kw = dict(nx=70, ny=61, P=5, core_cells=9, src_x=12, ports=(20, 50), steps=60, nf=5)
        return W.slab2d(**kw), W.slab2d(rough=True, sigma_nm=30, lc_nm=60, seed=3, **kw)
    return _te2(), _te2()


def _run(eng, spec, seed, precision=np.float64):
    """A job advanced 40 steps from random fields (every DFT-window cell non-zero)."""
    from oracle import fdtd_ref as R
    job = eng.submit(spec, precision=precision)
    rng = np.random.default_rng(seed)
    for f in R.field_names(spec.mode):
        job.set_field(f, rng.standard_normal(spec.shape) * 1e-2)
    job.advance(40)
    return job


def _host_power(job, port, window, minus=None):
    nc = 4 if job.spec.mode == "yee3d" else 2
    comps = [job.dft(port, c) - (minus.dft(port, c) if minus is not None else 0) for c in range(nc)]
    sav = power_density(job.spec.mode, comps)
    if job.spec.mode == "yee3d":
        (i0, i1), (j0, j1) = window
        return sav[:, i0:i1, j0:j1].sum(axis=(1, 2))
    j0, j1 = window
    return sav[:, j0:j1].sum(axis=1)


@pytest.mark.parametrize("mode", ["yee3d", "tm2", "te2"])
@pytest.mark.parametrize("precision", [np.float64, np.float32])
def test_device_power_equals_host_sums(eng, mode, precision):
    inc_spec, ref_spec = _specs(mode)
    inc, ref = _run(eng, inc_spec, 1, precision), _run(eng, ref_spec, 2, precision)
    w = power_window(ref_spec)
    # windows meeting the DFT window, and a rim row outside it (DFT cells there stay 0)
    (wi0, wi1), (wj0, wj1) = (ref_spec.win_lo[0], ref_spec.win_hi[0]), (ref_spec.win_lo[1], ref_spec.win_hi[1])
    if mode == "yee3d":
        nx, ny = ref_spec.shape[:2]
        inside = [w, ((wi0, wi0 + 1), (wj0 + 3, wj0 + 4)), ((wi1 - 1, wi1), (wj0, wj1)), ((0, nx), (0, ny))]
        windows = inside + [((nx - 1, nx), (0, ny))]
    else:
        ny = ref_spec.shape[1]
        inside = [w, (wj0 + 3, wj0 + 4), (wj1 - 1, wj1), (0, ny)]
        windows = inside + [(ny - 1, ny)]
    for win in windows:
        for port in (0, 1):
            got = ref.port_power(port, window=win)
            want = _host_power(ref, port, win)
            assert np.abs(want).max() > 0 or win not in inside
            np.testing.assert_allclose(got, want, rtol=RTOL, atol=RTOL * np.abs(want).max(), err_msg=str(win))
            if win not in inside:
                assert not np.any(got)
            got = ref.port_power(port, minus=inc, window=win)
            want = _host_power(ref, port, win, minus=inc)
            np.testing.assert_allclose(got, want, rtol=RTOL, atol=RTOL * np.abs(want).max(), err_msg=str(win))
    d_inc = {(p, c): inc.dft(p, c) for p in (0, 1) for c in range(4 if mode == "yee3d" else 2)}
    d_ref = {(p, c): ref.dft(p, c) for p in (0, 1) for c in range(4 if mode == "yee3d" else 2)}
    s_host, s_dev = forward_s(ref_spec, d_inc, d_ref), forward_s_device(ref_spec, inc, ref)
    for k in ("S11", "S21", "P_inc"):
        np.testing.assert_allclose(s_dev[k], s_host[k], rtol=1e-11, err_msg=k)
    # deterministic: the same call gives the same bits
    np.testing.assert_array_equal(ref.port_power(1, window=w), ref.port_power(1, window=w))
    inc.release()
    ref.release()


def test_power_of_fresh_job_is_zero_and_errors(eng):
    inc_spec, ref_spec = _specs("yee3d")
    job = eng.submit(ref_spec, precision=np.float32)
    np.testing.assert_array_equal(job.port_power(0), np.zeros(ref_spec.nf, np.complex128))
    other = _run(eng, inc_spec, 3, np.float32)
    slab = eng.submit(_specs("tm2")[0], precision=np.float32)
    lib, ctx = eng.lib, eng.ctx
    import ctypes as C
    out = np.empty(ref_spec.nf, np.complex128)
    nx, ny = ref_spec.shape[:2]

    def call(jid, minus, port, win, n=out.size * 2):
        w = (C.c_int32 * 4)(*win)
        return lib.oidt_job_port_power(ctx, jid, minus, port, w, out.ctypes.data, n)

    assert call(job.id, 0, 0, (0, nx, 0, ny)) == 0
    assert call(job.id, 0, 2, (0, nx, 0, ny)) == -1            # bad port
    assert call(job.id, 0, 0, (0, nx + 1, 0, ny)) == -1        # outside the plane
    assert call(job.id, 0, 0, (3, 3, 0, ny)) == -1             # empty
    assert call(job.id, 0, 0, (-1, 2, 0, ny)) == -1
    assert call(job.id, 0, 0, (0, nx, 0, ny), n=2 * ref_spec.nf - 1) == -1  # short output
    assert call(job.id, job.id, 0, (0, nx, 0, ny)) == -1       # minus itself
    assert call(job.id, slab.id, 0, (0, nx, 0, ny)) == -1      # other solver / plane
    assert call(job.id, 10 ** 9, 0, (0, nx, 0, ny)) == -4      # unknown minus job
    assert call(10 ** 9, 0, 0, (0, nx, 0, ny)) == -4           # unknown job
    assert call(job.id, other.id, 0, (0, nx, 0, ny)) == 0      # same plane shape: allowed
    for j in (job, other, slab):
        j.release()
