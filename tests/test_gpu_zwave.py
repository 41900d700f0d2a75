"""Line probe and wave-impedance workload on the GPU against the reference's
own run (``tests/golden/zwave_*.npz``) and the oracle.

* The engine's float32 EXACT run records Ey, Ez, Hy, Hz along the line bit
  for bit as the reference's float32 run does, in both 3D launch forms.
* A float32 fast-arithmetic run's records agree with the reference's to
  1e-4 of each record's maximum.
* A job without a probe refuses oidt_job_read_probe; reset clears the records.
"""
import json
import os

import numpy as np
import pytest

from oidt_b200 import zwave
from oidt_b200.engine import Engine, OidtError
from tests import golden_io as G

CASES = ["zwave_tm", "zwave_te"]
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not all(os.path.exists(os.path.join(G.GOLDEN, c + ".npz")) for c in CASES),
                                 reason="wave-impedance fixtures not generated (tests/golden/make_golden.py)")]
COMPS = (("ey", "EY_ZW"), ("ez", "EZ_ZW"), ("hy", "HY_ZW"), ("hz", "HZ_ZW"))


@pytest.fixture(scope="module")
def eng():
    e = Engine(0)
    yield e
    e.close()


def _load(case):
    z = np.load(os.path.join(G.GOLDEN, case + ".npz"))
    over = json.loads(str(z["over_json"]))
    return z, zwave.config(**{k: v for k, v in over.items() if k in zwave.REFERENCE_CONFIG})


@pytest.mark.parametrize("variant", ["cell", "sweep"])
@pytest.mark.parametrize("case", CASES)
def test_exact_f32_probe_equals_reference(eng, case, variant):
    z, cfg = _load(case)
    job = eng.submit(zwave.build_spec(cfg), arith="exact", precision=np.float32, ring_steps=5, variant=variant)
    job.advance(30).advance(job.spec.nt - 30).sync(60000)
    for comp, key in COMPS:
        np.testing.assert_array_equal(job.probe(comp), z["dev_" + key], err_msg=key)
    for f in ("EX", "EY", "EZ", "HX", "HY", "HZ"):
        np.testing.assert_array_equal(job.field(f), z["dev_" + f], err_msg=f)
    rec = zwave.records_from_job(job, cfg)
    for name, arr in rec.items():
        np.testing.assert_array_equal(arr, z["npy_" + name], err_msg=name)
    job.release()


@pytest.mark.parametrize("case", CASES)
def test_fast_f32_probe_within_tolerance(eng, case):
    z, cfg = _load(case)
    job = eng.submit(zwave.build_spec(cfg), arith="fast", precision=np.float32)
    job.run().sync(60000)
    for comp, key in COMPS:
        want = z["dev_" + key]
        got = job.probe(comp)
        assert np.max(np.abs(got - want)) <= 1e-4 * np.max(np.abs(want)), key
    job.release()


def test_probe_misuse_and_reset(eng):
    z, cfg = _load("zwave_tm")
    spec = zwave.build_spec(cfg)
    job = eng.submit(spec, arith="exact", precision=np.float32)
    job.advance(40).sync(60000)
    first = job.probe("ez")
    assert np.any(first[:40]) and not np.any(first[40:])  # rows of steps not yet run stay 0
    job.reset()
    assert not np.any(job.probe("ez"))
    job.run().sync(60000)
    np.testing.assert_array_equal(job.probe("ez"), z["dev_EZ_ZW"])
    job.release()
    spec.meta.pop("probe")
    plain = eng.submit(spec, arith="exact", precision=np.float32)
    with pytest.raises(OidtError):
        plain.probe("ez")
    plain.release()
