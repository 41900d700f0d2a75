"""Wave-impedance workload on the CPU: setup, the oracle's float32 line
records against the reference's own run (``tests/golden/zwave_*.npz``: the
reference's ``wave_impedance/fdtd_main.py`` on a tiny smooth guide, float32),
and the impedance and slab formulas."""
import json
import os

import numpy as np
import pytest

from oidt_b200 import zwave
from tests import golden_io as G

CASES = [c for c in ("zwave_tm", "zwave_te") if os.path.exists(os.path.join(G.GOLDEN, c + ".npz"))]


def _load(case):
    z = np.load(os.path.join(G.GOLDEN, case + ".npz"))
    return z, json.loads(str(z["over_json"]))


def _cfg(over):
    return zwave.config(**{k: v for k, v in over.items() if k in zwave.REFERENCE_CONFIG})


def test_fixtures_present():
    assert CASES == ["zwave_tm", "zwave_te"]


@pytest.mark.parametrize("case", CASES)
def test_setup_and_probe_line_equal_reference(case):
    z, over = _load(case)
    cfg = _cfg(over)
    dv = zwave.derive(cfg)
    assert (dv.nx, dv.ny, dv.nz, dv.nt) == tuple(int(z["cfg_" + k]) for k in ("nx", "ny", "nz", "nt"))
    assert (dv.extra["cy"], dv.extra["cz"]) == (int(z["cfg_cy"]), int(z["cfg_cz"]))
    spec = zwave.build_spec(cfg)
    assert spec.meta["probe"] == (int(z["cfg_cy"]), int(z["cfg_cz"]))
    for ax, name in (("x", "CBX"), ("y", "CBY"), ("z", "CBZ")):
        np.testing.assert_array_equal(spec.cb[ax], z["h2d_" + name], err_msg=name)
    np.testing.assert_array_equal(spec.j_src, z["h2d_J_SRC"])


@pytest.mark.parametrize("case", CASES)
def test_oracle_records_equal_reference(case):
    from oracle import zwave_ref as Z
    z, over = _load(case)
    s = Z.run(Z.build(Z.settings(**over)))
    for f in ("EX", "EY", "EZ", "HX", "HY", "HZ"):
        np.testing.assert_array_equal(getattr(s, f), z["dev_" + f], err_msg=f)
    for k in ("EY_ZW", "EZ_ZW", "HY_ZW", "HZ_ZW"):
        np.testing.assert_array_equal(s.rec[k], z["dev_" + k], err_msg=k)
        assert np.any(s.rec[k])
    saved = [k for k in z.files if k.startswith("npy_")]
    names = {n for _, n in zwave.RECORDS[over["source_condition"]]}
    assert {k[4:] for k in saved} == names  # the reference saves the two records of its mode


@pytest.mark.parametrize("case", CASES)
def test_impedance_of_reference_records(case):
    """The product's FFT ratio on the reference's saved records equals the
    oracle's restatement of zwave.py on its own (bit-equal) records."""
    from oracle import zwave_ref as Z
    z, over = _load(case)
    cfg = _cfg(over)
    rec = {k[4:]: z[k] for k in z.files if k.startswith("npy_")}
    ff, zz = zwave.impedance(rec, cfg)
    s = Z.run(Z.build(Z.settings(**over)))
    ff2, zz2 = Z.impedance(s)
    np.testing.assert_array_equal(ff, ff2)
    np.testing.assert_array_equal(zz, zz2)


def test_slab_impedance_formula():
    """TE: Im Z < 0 (inductive decay), TM: Im Z > 0, |Z| of the order of the
    cladding impedance (zwave.py:36-57)."""
    fa, te = zwave.analytic(zwave.config(source_condition="TE"), [150e12, 194.8e12, 250e12])
    _, tm = zwave.analytic(zwave.config(source_condition="TM"), [150e12, 194.8e12, 250e12])
    assert np.all(te.imag < 0) and np.all(tm.imag > 0)
    eta_clad = 120 * np.pi / 1.5
    assert np.all(np.abs(te) < 5 * eta_clad) and np.all(np.abs(tm) < 5 * eta_clad)
