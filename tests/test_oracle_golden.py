"""The oracle reproduces the reference itself, bit for bit, in float64.

Fixtures come from running the reference's own ``fdtd_main.py`` /
``extract_sparams.py`` under Numba's CUDA simulator
(``tests/golden/make_golden.py``).
"""
import hashlib
import os

import numpy as np
import pytest

from oracle import fdtd_ref as R
from tests import golden_io as G

RUN_CASES = ["tm2_smooth", "tm2_rough2", "tm2_lines2", "te2_smooth", "te2_rough2", "yee3d_smooth", "yee3d_rough2_tm"]
SETUP_CASES = ["setup_%s_%s" % (m, p) for m in ("tm2", "te2", "yee3d") for p in ("float32", "float64")]


def _mode(name):
    return name.split("_")[1] if name.startswith("setup_") else name.split("_")[0]


def _have(name):
    return os.path.exists(os.path.join(G.GOLDEN, name + ".npz"))


@pytest.mark.parametrize("case", SETUP_CASES)
def test_setup_matches_reference(case):
    if not _have(case):
        pytest.skip("fixture not generated")
    z = G.load(case)
    usr = G.usr_of(z)
    mode = _mode(case)
    for (line, d, kind) in G.sims_of(z):
        tag = "%d%s%s" % (line, d, kind)
        s = R.build(usr, mode, line, d, kind)
        for key in z.files:
            if not key.startswith(tag + "/sha_h2d_"):
                continue
            name = key[len(tag + "/sha_h2d_"):]
            a = np.ascontiguousarray(G.oracle_array(s, name))
            assert str(a.dtype) == str(z[tag + "/dtype_" + name]), name
            assert tuple(a.shape) == tuple(z[tag + "/shape_" + name]), name
            assert hashlib.sha256(a.tobytes()).hexdigest() == str(z[key]), (case, tag, name)
        for k in ("J_SRC", "sparam_freqs"):
            a = np.ascontiguousarray(s.cfg.J_SRC if k == "J_SRC" else s.cfg.sparam_freqs)
            assert hashlib.sha256(a.tobytes()).hexdigest() == str(z["%s/sha_cfg_%s" % (tag, k)]), (case, k)
        for k in ("nx", "ny", "nz", "nt", "p1x", "p2x", "p1z", "p2z", "pp", "ph", "bx", "by", "sx", "sz"):
            key = "%s/cfg_%s" % (tag, k)
            if key in z.files:
                assert getattr(s.cfg, k) == z[key], (case, k)


@pytest.mark.parametrize("case", RUN_CASES)
def test_run_matches_reference(case):
    if not _have(case):
        pytest.skip("fixture not generated")
    z = G.load(case)
    usr = G.usr_of(z)
    mode = _mode(case)
    outs = {}
    for (line, d, kind) in G.sims_of(z):
        tag = "%d%s%s" % (line, d, kind)
        s = R.build(usr, mode, line, d, kind, profiles=G.profiles_of(z))
        for key in z.files:
            if key.startswith(tag + "/h2d_"):
                name = key[len(tag + "/h2d_"):]
                np.testing.assert_array_equal(G.oracle_array(s, name), z[key], err_msg=name)
        R.run(s)
        n_checked = 0
        for key in z.files:
            if key.startswith(tag + "/dev_"):
                name = key[len(tag + "/dev_"):]
                np.testing.assert_array_equal(G.oracle_array(s, name), z[key], err_msg="%s %s" % (tag, name))
                n_checked += 1
        assert n_checked > 10
        o = R.outputs(s)
        for nm, arr in o.items():
            ref = z["%s/npy_%s" % (tag, nm)]
            assert arr.dtype == ref.dtype
            np.testing.assert_array_equal(arr, ref, err_msg=nm)
        outs.update(o)
    if "S_mat" in z.files:
        S = R.extract_sparams(usr, mode, outs)
        np.testing.assert_array_equal(S, z["S_mat"])
