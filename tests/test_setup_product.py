"""The product's setup (oidt_b200.refsetup) reproduces the reference's arrays
bit for bit: against the SHA-256 digests recorded from the reference itself
(float32 and float64) and against the oracle on the tiny run fixtures."""
import hashlib
import os

import numpy as np
import pytest

from oidt_b200.refsetup import build_spec
from oracle import fdtd_ref as R
from tests import golden_io as G

SETUP_CASES = ["setup_%s_%s" % (m, p) for m in ("tm2", "te2", "yee3d") for p in ("float32", "float64")]
RUN_CASES = ["tm2_smooth", "tm2_rough2", "tm2_lines2", "te2_smooth", "te2_rough2", "yee3d_smooth", "yee3d_rough2_tm"]


def spec_array(spec, name):
    """Reference device-array name -> the product spec's array."""
    m = {"CBX": ("cb", "x"), "CBY": ("cb", "y"), "CBZ": ("cb", "z"), "KXE": ("kdx", "xe"), "KYE": ("kdx", "ye"),
         "KZE": ("kdx", "ze"), "KXH": ("kdx", "xh"), "KYH": ("kdx", "yh"), "KZH": ("kdx", "zh")}
    if name in m:
        return getattr(spec, m[name][0])[m[name][1]]
    if name in ("BE", "CE", "BH", "CH"):
        return getattr(spec, name.lower())
    if name == "J_SRC":
        return spec.j_src
    if name in ("cosE", "sinE", "cosH", "sinH"):
        return spec.twiddles[("cosE", "sinE", "cosH", "sinH").index(name)]
    return None


def _have(c):
    return os.path.exists(os.path.join(G.GOLDEN, c + ".npz"))


@pytest.mark.parametrize("case", SETUP_CASES)
def test_product_setup_matches_reference_digests(case):
    if not _have(case):
        pytest.skip("fixture not generated")
    z = G.load(case)
    usr = G.usr_of(z)
    mode = case.split("_")[1]
    for (line, d, kind) in G.sims_of(z):
        tag = "%d%s%s" % (line, d, kind)
        spec = build_spec(usr, mode, line, d, kind)
        dv = spec.meta["derived"]
        checked = 0
        for key in z.files:
            if not key.startswith(tag + "/sha_h2d_"):
                continue
            name = key[len(tag + "/sha_h2d_"):]
            a = spec_array(spec, name)
            if a is None:
                continue
            if name in ("cosE", "sinE", "cosH", "sinH"):
                # the engine keeps float64 twiddles; the reference stores them in `precision`
                a = a.astype(str(z[tag + "/dtype_" + name]))
            a = np.ascontiguousarray(a)
            assert str(a.dtype) == str(z[tag + "/dtype_" + name]), name
            assert hashlib.sha256(a.tobytes()).hexdigest() == str(z[key]), (case, tag, name)
            checked += 1
        assert checked >= 12
        assert hashlib.sha256(np.ascontiguousarray(dv.j_src).tobytes()).hexdigest() == str(z[tag + "/sha_cfg_J_SRC"])
        assert dv.nt == int(z[tag + "/cfg_nt"])
        assert (dv.nx, dv.ny) == (int(z[tag + "/cfg_nx"]), int(z[tag + "/cfg_ny"]))
        db = z[tag + "/cfg_delta_t"] / (4.0e-7 * np.pi)
        assert spec.db == db


@pytest.mark.parametrize("case", RUN_CASES)
def test_product_setup_matches_oracle(case):
    if not _have(case):
        pytest.skip("fixture not generated")
    z = G.load(case)
    usr = G.usr_of(z)
    mode = case.split("_")[0]
    for (line, d, kind) in G.sims_of(z):
        spec = build_spec(usr, mode, line, d, kind, profiles=G.profiles_of(z))
        s = R.build(usr, mode, line, d, kind, profiles=G.profiles_of(z))
        for ax in spec.cb:
            np.testing.assert_array_equal(spec.cb[ax], getattr(s, "CB" + ax.upper()))
        for k, v in spec.kdx.items():
            np.testing.assert_array_equal(v, getattr(s, "K%s%s" % (k[0].upper(), k[1].upper())))
        for n in ("be", "ce", "bh", "ch"):
            np.testing.assert_array_equal(getattr(spec, n), getattr(s, n.upper()))
        np.testing.assert_array_equal(spec.j_src, s.cfg.J_SRC)
        for a, b in zip(spec.twiddles, (s.cosE, s.sinE, s.cosH, s.sinH)):
            np.testing.assert_array_equal(a, b)
        box = s.src_box
        nd = len(spec.shape)
        assert tuple(spec.src_lo[:nd]) == tuple(box[1:1 + nd]) and tuple(spec.src_hi[:nd]) == tuple(box[1 + nd:])
        assert spec.db == s.DB
        pp = (s.cfg.p1z, s.cfg.p2z) if mode == "yee3d" else (s.cfg.p1x, s.cfg.p2x)
        assert tuple(spec.port_pos) == pp


@pytest.mark.parametrize("case", [c for c in RUN_CASES if c.endswith("smooth") or c == "tm2_lines2"])
def test_product_extraction_matches_reference(case):
    """oidt_b200.sparams.extract_sparams on the reference's own saved .npy
    DFTs equals the S-matrix the reference's extract_sparams.py built."""
    if not _have(case):
        pytest.skip("fixture not generated")
    from oidt_b200.sparams import extract_sparams
    z = G.load(case)
    usr = G.usr_of(z)
    data = {}
    for k in z.files:
        if "/npy_" in k:
            data[k.split("/npy_")[1]] = z[k]
    S = extract_sparams(usr, case.split("_")[0], data)
    np.testing.assert_array_equal(S, z["S_mat"])
