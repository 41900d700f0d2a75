"""Scattering-loss workload on the CPU: the product's setup, plane
convention and loss formula, and the oracle's float32 run, each against the
reference's own run recorded in ``tests/golden/scatter_*.npz`` (made by
``tests/golden/make_golden.py``: the reference's ``scattering_loss/fdtd_main.py``
and ``automated_results_collection.py`` on a 16 x 20 x 30 grid, 82 steps)."""
import json
import os

import numpy as np
import pytest

from oidt_b200 import scatter
from tests import golden_io as G

CASES = [c for c in ("scatter_te", "scatter_tm") if os.path.exists(os.path.join(G.GOLDEN, c + ".npz"))]
# the fixtures' grid: 16 x 20 x 30 cells, 82 steps (make_golden.SCATTER_TINY)
TINY = dict(sgl_wg_length=1.5e-6, sgl_wg_width=0.6e-6, sgl_wg_height=0.3e-6, port1_length=0.3e-6,
            port2_length=0.0, points_per_wl=6, num_cpml=3, buffer_zhat=2, nx_clad_wl=0.25, ny_clad_wl=0.25,
            num_flights=1.0)


def _load(case):
    z = np.load(os.path.join(G.GOLDEN, case + ".npz"))
    over = json.loads(str(z["over_json"]))
    return z, over, (z["profile_upper"], z["profile_lower"])


def _tag(z):
    return [k[len("npy_ex1_fft"):] for k in z.files if k.startswith("npy_ex1_fft")][0]


def test_fixtures_present():
    assert CASES == ["scatter_te", "scatter_tm"]


@pytest.mark.parametrize("case", CASES)
def test_setup_equals_reference_arrays(case):
    """Grid, steps, cut planes, dt/eps grids, kappa*dx, CPML recursion
    coefficients and the source waveform equal the reference's, bit for bit."""
    z, over, prof = _load(case)
    cfg = scatter.config(**over)
    dv = scatter.derive(cfg)
    assert (dv.nx, dv.ny, dv.nz, dv.nt) == tuple(int(z["cfg_" + k]) for k in ("nx", "ny", "nz", "nt"))
    assert (dv.p1, dv.p2) == (int(z["cfg_p1z"]), int(z["cfg_p2z"]))
    assert dv.delta_x == z["cfg_delta_x"] and dv.delta_t == z["cfg_delta_t"]
    spec = scatter.build_spec(cfg, prof)
    for ax, name in (("x", "CBX"), ("y", "CBY"), ("z", "CBZ")):
        np.testing.assert_array_equal(spec.cb[ax], z["h2d_" + name], err_msg=name)
    for key, name in (("xe", "KXE"), ("xh", "KXH"), ("ye", "KYE"), ("yh", "KYH"), ("ze", "KZE"), ("zh", "KZH")):
        np.testing.assert_array_equal(spec.kdx[key], z["h2d_" + name], err_msg=name)
    for key, name in (("be", "BE"), ("ce", "CE"), ("bh", "BH"), ("ch", "CH")):
        np.testing.assert_array_equal(getattr(spec, key), z["h2d_" + name], err_msg=name)
    np.testing.assert_array_equal(spec.j_src, z["h2d_J_SRC"])
    assert spec.port_pos == (dv.p1, dv.p2) and spec.nf == 1 and spec.freqs[0] == cfg["f0"]


@pytest.mark.parametrize("case", CASES)
def test_oracle_float32_run_equals_reference(case):
    """The oracle's float32 run reproduces the reference's final fields and
    its twelve float32 DFT planes bit for bit."""
    from oracle import scatter_ref as S
    z, over, prof = _load(case)
    s = S.run(S.build(S.settings(**over), prof))
    for f in ("EX", "EY", "EZ", "HX", "HY", "HZ"):
        np.testing.assert_array_equal(getattr(s, f), z["dev_" + f], err_msg=f)
    tag = _tag(z)
    planes = S.complex_planes(s)
    for name, arr in planes.items():
        np.testing.assert_array_equal(arr, z["npy_%s%s_fft%s" % (name[:2], name[2], tag)], err_msg=name)


@pytest.mark.parametrize("case", CASES)
def test_loss_of_reference_planes_equals_reference_alpha(case):
    """alpha computed by the product from the reference's saved planes equals
    the value the reference's results collection wrote."""
    z, over, prof = _load(case)
    cfg = scatter.config(**over)
    dv = scatter.derive(cfg)
    tag = _tag(z)
    planes = {n + c: z["npy_%s%s_fft%s" % (n, c, tag)] for n in scatter.PLANE_COMPS for c in "12"}
    got = scatter.loss(planes, dv.delta_x, dv.extra["ell"])["alpha"]
    want = float(z["results"][2, 0])
    assert got == pytest.approx(want, rel=1e-6)
    assert z["results"][0, 0] == 15 and z["results"][1, 0] == 700


def test_plane_convention_is_conjugate_of_engine_accumulators():
    """The engine accumulates I = -sum x sin (the S-parameter kernels); the
    scattering-loss planes are R + i sum x sin, complex64."""
    spec = scatter.build_spec(scatter.config(**TINY))
    nx, ny = spec.shape[:2]
    rng = np.random.default_rng(3)
    dft = {(p, c): (rng.standard_normal((1, nx, ny)) + 1j * rng.standard_normal((1, nx, ny))) for p in (0, 1)
           for c in range(4)}
    pl = scatter.planes_from_dft(spec, dft)
    assert sorted(pl) == ["ex1", "ex2", "ey1", "ey2", "hx1", "hx2", "hy1", "hy2"]
    for p in (0, 1):
        for c, n in enumerate(scatter.PLANE_COMPS):
            a = pl["%s%d" % (n, p + 1)]
            assert a.dtype == np.complex64 and a.shape == (nx, ny)
            np.testing.assert_array_equal(a, np.conjugate(dft[(p, c)][0]).astype(np.complex64))


def test_loss_is_invariant_to_the_dft_sign_convention():
    """P = 1/2 Re(E H*) is unchanged by conjugating both planes, so alpha does
    not depend on which sign the accumulators use."""
    rng = np.random.default_rng(5)
    pl = {}
    for c, scale in (("1", 1.0), ("2", 0.8)):  # a forward wave: Hy ~ Ex, Hx ~ -Ey
        ex, ey = (scale * (rng.standard_normal((6, 7)) + 1j * rng.standard_normal((6, 7))) for _ in range(2))
        pl.update({"ex" + c: ex, "ey" + c: ey, "hx" + c: -0.9 * ey, "hy" + c: 1.1 * ex})
    pl = {k: v.astype(np.complex64) for k, v in pl.items()}
    a = scatter.loss(pl, np.float32(1e-8), np.float32(3e-6))
    b = scatter.loss({k: np.conjugate(v) for k, v in pl.items()}, np.float32(1e-8), np.float32(3e-6))
    assert a == b and np.isfinite(a["alpha"]) and a["alpha"] > 0


def test_save_planes_uses_reference_names(tmp_path):
    cfg = scatter.config()
    pl = {n + c: np.zeros((2, 2), np.complex64) for n in scatter.PLANE_COMPS for c in "12"}
    names = sorted(os.path.basename(p) for p in scatter.save_planes(str(tmp_path), scatter.profile_tag(cfg), pl))
    assert names[0] == "ex1_fft_s15nm_lc700nm_r0.npy" and len(names) == 8
    assert "hy2_fft_s15nm_lc700nm_r0.npy" in names


def test_payne_lacey_estimates():
    """The slab estimates the reference compares against (analysis.py:38-111)
    equal the values its own functions return on a 4 x 4 grid of sigma and Lc
    (``tests/golden/scatter_analytic.npz``); alpha grows with sigma^2 and the
    TE effective index lies between the cladding and core indices."""
    from oidt_b200.scatter import alpha_te, alpha_tm, find_neff
    f0 = scatter.REFERENCE_CONFIG["f0"]
    k0 = 2 * np.pi * f0 / 3e8
    ne = find_neff(3.5, 1.5, 100e-9, k0, "te")
    assert 1.5 < ne < 3.5
    a1, a2 = alpha_te(15e-9, 700e-9, f0), alpha_te(30e-9, 700e-9, f0)
    assert a2[0] == pytest.approx(4 * a1[0], rel=1e-9)
    tm = alpha_tm(15e-9, 700e-9, f0, 3.5, 1.5)
    assert len(tm) == 4 and all(t > 0 for t in tm)
    z = np.load(os.path.join(G.GOLDEN, "scatter_analytic.npz"))
    assert z["table"].shape == (16, 8)
    for s_nm, lc_nm, te0, te1, tm0, tm1, tm2, tm3 in z["table"]:
        got_te = alpha_te(s_nm * 1e-9, lc_nm * 1e-9, f0)
        got_tm = alpha_tm(s_nm * 1e-9, lc_nm * 1e-9, f0, 3.5, 1.5)
        np.testing.assert_allclose(got_te, (te0, te1), rtol=1e-9)
        np.testing.assert_allclose(got_tm, (tm0, tm1, tm2, tm3), rtol=1e-9)
