"""The allocation-free port-window DFT readout (oidt_job_read_dft_window_static),
meant for hosts that reserve their device memory up front and may not allocate
when they read results, equals the window of the staged full-plane readout
(oidt_job_read_dft), bit for bit, on two consecutive calls and for 2D and 3D
jobs; windows larger than its 16 MiB static device buffer are refused.
Collected last, so a run that stops at the first failure has already run
every other test; it passes alone and after the rest of the suite."""
import numpy as np
import pytest

from oidt_b200 import workloads as W
from oidt_b200.engine import Engine, OidtError

pytestmark = pytest.mark.gpu


def _window(job, full):
    (i0, j0), (i1, j1) = job.spec.win_lo, job.spec.win_hi
    if job.spec.mode == "yee3d":
        return full[:, i0:i1, j0:j1]
    return full[:, j0:j1]


@pytest.mark.parametrize("mode", ["tm2", "yee3d"])
def test_static_window_read_equals_staged_read(mode):
    eng = Engine(0)
    if mode == "tm2":
        spec = W.slab2d(nx=70, ny=61, P=5, core_cells=9, src_x=12, ports=(20, 50), steps=60, nf=5, seed=3)
        ncomp = 2
    else:
        spec = W.strip3d(nx=24, ny=22, nz=40, P=4, src_gap=2, port_gap=3, steps=60, nf=4, core_x_nm=120,
                         core_y_nm=160, seed=5)
        ncomp = 4
    job = eng.submit(spec, precision=np.float32)
    job.advance(30).sync()
    for port, comp in ((0, 0), (1, ncomp - 1)):  # two consecutive calls, different planes of the accumulator
        got = job.dft_window_static(port, comp)
        np.testing.assert_array_equal(got, _window(job, job.dft(port, comp)))
    job.advance(30).sync()  # the readout after further steps sees the new accumulators
    for port, comp in ((1, 0), (0, 1)):
        got = job.dft_window_static(port, comp)
        ref = _window(job, job.dft(port, comp))
        assert np.any(ref != 0)
        np.testing.assert_array_equal(got, ref)
    job.release()
    eng.close()


def test_static_window_read_refuses_oversize_windows():
    eng = Engine(0)
    # 600 frequencies x 52 x 52 window cells x 16 B = 24.8 MiB > 16 MiB of static scratch
    spec = W.strip3d(nx=60, ny=60, nz=40, P=4, src_gap=2, port_gap=3, steps=8, nf=600, core_x_nm=120,
                     core_y_nm=160, seed=5)
    (i0, j0), (i1, j1) = spec.win_lo, spec.win_hi
    assert spec.nf * (i1 - i0) * (j1 - j0) * 16 > 16 << 20
    job = eng.submit(spec, precision=np.float32)
    job.advance(8).sync()
    with pytest.raises(OidtError, match="static scratch"):
        job.dft_window_static(0, 0)
    job.release()
    eng.close()
