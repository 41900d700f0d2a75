"""Failure handling at the host boundary, without any device fault: a wait
that runs out returns OIDT_ERR_TIMEOUT and leaves the job and the context
usable; misuse (unknown job, too many steps, short output buffers, a
budget refusal) returns an error code and changes nothing."""
import ctypes as C

import numpy as np
import pytest

from oidt_b200 import workloads as W
from oidt_b200.engine import BudgetError, Engine, OidtError, TimeoutError_

pytestmark = pytest.mark.gpu


def _spec(steps=400):
    return W.strip3d(nx=96, ny=96, nz=192, P=8, steps=steps, nf=5, seed=3)


def test_sync_timeout_leaves_the_job_usable():
    eng = Engine(0)
    spec = _spec()
    ref = eng.submit(spec)
    ref.run().sync()
    want = {f: ref.field(f) for f in ("EY", "HX")}
    ref.release()

    job = eng.submit(spec, graphs=False)  # one launch per step: the work outlasts a 1 ms wait
    job.run()
    with pytest.raises(TimeoutError_):
        job.sync(1)
    job.sync()  # unbounded wait completes
    assert not job.busy()
    for f, v in want.items():
        np.testing.assert_array_equal(job.field(f), v)
    job.release()
    eng.close()


def test_misuse_returns_errors_and_changes_nothing():
    eng = Engine(0)
    spec = _spec(steps=50)
    job = eng.submit(spec)
    job.advance(20).sync()
    before = job.field("EX")
    lib, ctx = eng.lib, eng.ctx
    assert lib.oidt_job_advance(ctx, job.id + 1000, 5) == -4          # unknown job
    assert lib.oidt_job_advance(ctx, job.id, 31) == -6                # past the source steps
    small = np.empty(4, np.float64)
    assert lib.oidt_job_read_dft(ctx, job.id, 0, 0, small.ctypes.data, small.size) == -1  # short output
    assert lib.oidt_job_read_dft(ctx, job.id, 2, 0, small.ctypes.data, small.size) == -1  # bad port
    assert b"bad port" in lib.oidt_last_error(ctx)
    np.testing.assert_array_equal(job.field("EX"), before)
    job.advance(30).sync()  # the job still runs to its end
    job.release()
    with pytest.raises(OidtError):
        job.eng._check(lib.oidt_job_sync(ctx, job.id, 0))  # released: unknown
    eng.close()


def test_budget_refusal_keeps_the_context_usable():
    spec = _spec(steps=20)
    probe = Engine(0)
    need = probe.job_bytes(spec)
    probe.close()
    eng = Engine(0, hbm_budget=need + need // 2)  # room for one job
    a = eng.submit(spec)
    with pytest.raises(BudgetError):
        eng.submit(spec)
    a.run().sync()
    a.release()
    b = eng.submit(spec)  # the freed memory admits the next job
    b.run().sync()
    b.release()
    eng.close()


def test_sweep_tile_wait_expiry_is_reported_and_recoverable():
    """The plane-sweep kernel's waits for its tile loads are bounded in the
    kernel.  With a bound of one cycle they run out on loads that are merely
    in flight; every CTA that gives up waits (with the default bound) for the
    copies it issued before it returns, so nothing lands in its shared memory
    afterwards.  oidt_job_sync reports the expiry as OIDT_ERR_TIMEOUT; the
    context and, after a reset with the default bound, the job itself run as
    before."""
    eng = Engine(0)
    spec = _spec(steps=64)
    ref = eng.submit(spec, variant="sweep")
    ref.advance(16).sync()
    want = {f: ref.field(f) for f in ("EY", "HX")}
    ref.release()

    job = eng.submit(spec, variant="sweep")
    job.set_wait_limit(1)
    job.advance(16)
    with pytest.raises(TimeoutError_, match="bounded wait"):
        job.sync(60000)
    other = eng.submit(spec, variant="sweep")  # the context still works
    other.advance(16).sync(60000)
    for f, v in want.items():
        np.testing.assert_array_equal(other.field(f), v)
    other.release()
    job.set_wait_limit(0).reset().advance(16).sync(60000)  # default bound: the job recovers
    for f, v in want.items():
        np.testing.assert_array_equal(job.field(f), v)
    job.release()
    eng.close()


def test_tile_neighbour_wait_expiry_is_reported_and_recoverable():
    """The 2D tile form's cooperative launches wait, between sub-blocks, for
    the neighbour tiles' counters; the waits are bounded in the kernel.  With
    a bound of one cycle they run out wherever a neighbour tile is still
    computing when a tile reaches its wait (144 tiles, hundreds of waits a
    launch); the tile records the expiry and goes on, later waits of the
    launch give up at once, and the launch ends.  oidt_job_sync reports
    OIDT_ERR_TIMEOUT; the context and, after a reset with the default bound,
    the job itself run as before."""
    eng = Engine(0)
    spec = W.slab2d(steps=256)
    ref = eng.submit(spec, variant="tile", precision=np.float64)
    ref.advance(128).sync()
    want = {f: ref.field(f) for f in ("EZ", "HY")}
    ref.release()

    job = eng.submit(spec, variant="tile", precision=np.float64)
    job.set_wait_limit(1)
    job.advance(128)
    with pytest.raises(TimeoutError_, match="bounded wait"):
        job.sync(60000)
    other = eng.submit(spec, variant="tile", precision=np.float64)  # the context still works
    other.advance(128).sync(60000)
    for f, v in want.items():
        np.testing.assert_array_equal(other.field(f), v)
    other.release()
    job.set_wait_limit(0).reset().advance(128).sync(60000)  # default bound: the job recovers
    for f, v in want.items():
        np.testing.assert_array_equal(job.field(f), v)
    job.release()
    eng.close()
