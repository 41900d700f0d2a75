"""Engine parity on a B200, through the C ABI (liboidt.so).

* float64 with OIDT_ARITH_EXACT must equal, bit for bit, (a) the reference's
  own device arrays recorded under Numba's CUDA simulator (golden fixtures)
  and (b) the float64 oracle, on random initial fields that exercise every
  CPML slab, the source and the port planes at once.
* float32 with OIDT_ARITH_FAST (the production path) against the float64
  oracle on identical inputs: field relative L2 <= 1e-5 and
  |S_fp32 - S_oracle| <= 1e-4 (the stated precision targets).
"""
import os

import numpy as np
import pytest

from oracle import fdtd_ref as R
from tests import golden_io as G
from tests.helpers import oracle_from_spec, psi_key, rel_l2

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-5
S_TOL = 1e-4


@pytest.fixture(scope="module")
def eng():
    from oidt_b200.engine import Engine
    e = Engine(0)
    yield e
    e.close()


def _fixture_cases():
    out = []
    for case in ["tm2_smooth", "tm2_rough2", "tm2_lines2", "te2_smooth", "te2_rough2", "yee3d_smooth",
                 "yee3d_rough2_tm"]:
        if os.path.exists(os.path.join(G.GOLDEN, case + ".npz")):
            out.append(case)
    return out


def _case_variants():
    """3D runs under every launch form (plane sweep, per-cell, vector, ordered); 2D under both of its
    forms (per-cell, tiles)."""
    return [(c, v) for c in _fixture_cases()
            for v in (("sweep", "cell", "vec", "wave") if c.startswith("yee3d") else ("cell", "tile"))]


@pytest.mark.parametrize("case,variant", _case_variants())
def test_exact_f64_equals_reference_device_arrays(eng, case, variant):
    """Engine float64 EXACT == the reference's recorded device arrays."""
    from oidt_b200.refsetup import build_spec
    z = G.load(case)
    usr = G.usr_of(z)
    mode = case.split("_")[0]
    for (line, d, kind) in G.sims_of(z):
        tag = "%d%s%s" % (line, d, kind)
        spec = build_spec(usr, mode, line, d, kind, profiles=G.profiles_of(z))
        job = eng.submit(spec, arith="exact", precision=np.float64, ring_steps=5, variant=variant)
        job.run().sync(60000)
        for f, arr in job.fields().items():
            np.testing.assert_array_equal(arr, z["%s/dev_%s" % (tag, f)], err_msg="%s %s" % (tag, f))
        from oidt_b200.spec import PSI
        for name, axis in PSI[mode]:
            for side in (0, 1):
                np.testing.assert_array_equal(job.psi(name, axis, side), z["%s/dev_%s" % (tag, psi_key(name, axis, side))])
        comps = {"tm2": ("EZ", "HY"), "te2": ("EY", "HZ"), "yee3d": ("EX", "EY", "HX", "HY")}[mode]
        for port in (0, 1):
            for ci, cn in enumerate(comps):
                ref = z["%s/dev_%s%dr" % (tag, cn, port + 1)] + 1j * z["%s/dev_%s%di" % (tag, cn, port + 1)]
                np.testing.assert_array_equal(job.dft(port, ci), ref, err_msg="%s port %d %s" % (tag, port, cn))
        job.release()


def _random_cases():
    from oidt_b200 import workloads as W
    return {
        "tm2": lambda: W.slab2d(nx=70, ny=61, P=5, core_cells=9, src_x=12, ports=(20, 50), steps=40, nf=5,
                                rough=True, sigma_nm=30, lc_nm=60, seed=3),
        "yee3d_te": lambda: W.strip3d(nx=22, ny=19, nz=37, P=4, src_gap=2, port_gap=3, steps=40, nf=4,
                                      core_x_nm=120, core_y_nm=160, sigma_nm=25, lc_nm=60, seed=5),
        "yee3d_tm": lambda: W.strip3d(nx=21, ny=24, nz=33, P=3, src_gap=2, port_gap=3, steps=40, nf=3,
                                      core_x_nm=140, core_y_nm=180, source="TM", seed=6),
        # large enough that both 3D launch forms have interior work units with
        # no CPML, edge or source cells (and a port plane inside one of them)
        "yee3d_wide": lambda: W.strip3d(nx=30, ny=44, nz=130, P=4, src_gap=2, port_gap=26, steps=40, nf=3,
                                        core_x_nm=160, core_y_nm=240, sigma_nm=20, lc_nm=60, seed=7),
        # the thinnest CPML: P = 1 (no H-slab cells) and P = 2; the DFT window then reaches the
        # rim cells no step updates
        "yee3d_p1": lambda: W.strip3d(nx=16, ny=15, nz=29, P=1, src_gap=2, port_gap=3, steps=40, nf=3,
                                      core_x_nm=100, core_y_nm=120, seed=8),
        "yee3d_p2": lambda: W.strip3d(nx=17, ny=18, nz=35, P=2, src_gap=2, port_gap=4, steps=40, nf=3,
                                      core_x_nm=100, core_y_nm=140, source="TM", seed=9),
        # z between the rims under 2P + 3 cells: four-cell groups holding cells of both z slabs
        # (the vector form's padded z-slab rows then take their per-cell path), the source
        # inside a slab
        "yee3d_zthin": lambda: W.strip3d(nx=18, ny=17, nz=14, P=4, src_gap=1, port_gap=1, steps=40, nf=3,
                                         core_x_nm=100, core_y_nm=120, sigma_nm=20, lc_nm=60, seed=12),
        "yee3d_zthin3": lambda: W.strip3d(nx=18, ny=17, nz=12, P=3, src_gap=1, port_gap=1, steps=40, nf=3,
                                          core_x_nm=100, core_y_nm=120, source="TM", seed=13),
        # the 2D tile form's shapes: a grid narrower than a halo, and rows longer than a
        # block's threads
        "tm2_narrow": lambda: W.slab2d(nx=14, ny=40, P=2, core_cells=7, src_x=4, ports=(6, 10), steps=40, nf=3),
        "tm2_tall": lambda: W.slab2d(nx=37, ny=1100, P=3, core_cells=9, src_x=6, ports=(10, 28), steps=40, nf=3),
        "tm2_p1": lambda: W.slab2d(nx=40, ny=31, P=1, core_cells=7, src_x=6, ports=(10, 30), steps=40, nf=4,
                                   rough=True, sigma_nm=30, lc_nm=60, seed=4),
        # dt/eps coefficient grids perturbed cell by cell (thousands of distinct (x, y, z) triples),
        # so no cell's update can lean on a neighbour's coefficients
        "yee3d_graded": lambda: _graded(W.strip3d(nx=22, ny=19, nz=37, P=4, src_gap=2, port_gap=3, steps=40,
                                                  nf=4, core_x_nm=120, core_y_nm=160, seed=10)),
    }


def _graded(spec):
    rng = np.random.default_rng(11)
    for k in spec.cb:
        spec.cb[k] = spec.cb[k] * (1.0 + 0.01 * rng.random(spec.cb[k].shape))
    spec.mat_idx = spec.mat_tab = None  # thousands of distinct triples: the grids themselves
    return spec


def _te2_spec():
    """A TE2 job: reuse the slab geometry with the TE solver arrays."""
    from oidt_b200 import workloads as W
    s = W.slab2d(nx=66, ny=57, P=4, core_cells=9, src_x=12, ports=(20, 46), steps=40, nf=4)
    s.mode = "te2"
    from oidt_b200.refsetup import staggered_eps
    eps_cell = s.meta["dt"] / s.cb["z"]
    ex, ey = staggered_eps(eps_cell, np.float64, (0, 1))
    s.cb = {"x": s.meta["dt"] / ex, "y": s.meta["dt"] / ey}
    by = s.src_lo[1] - 1
    s.src_field = 5  # HZ
    s.src_lo = (12, by + 2, 0)
    s.src_hi = (13, by + 9 - 2, 1)
    return s


@pytest.mark.parametrize("name", ["tm2", "te2", "yee3d_te", "yee3d_tm", "yee3d_wide", "yee3d_te_cell",
                                  "yee3d_tm_cell", "yee3d_wide_cell", "yee3d_p1", "yee3d_p1_cell",
                                  "yee3d_p2", "yee3d_p2_cell", "tm2_p1", "yee3d_graded", "yee3d_graded_cell",
                                  "yee3d_te_vec", "yee3d_tm_vec", "yee3d_wide_vec", "yee3d_p1_vec", "yee3d_p2_vec",
                                  "yee3d_graded_vec", "yee3d_te_wave", "yee3d_tm_wave", "yee3d_wide_wave",
                                  "yee3d_p1_wave", "yee3d_p2_wave", "yee3d_graded_wave", "tm2_tile",
                                  "te2_tile", "tm2_p1_tile", "tm2_narrow_tile", "tm2_tall_tile",
                                  "tm2_narrow", "tm2_tall", "tm2_tile2", "te2_tile2", "tm2_p1_tile2",
                                  "tm2_tile1", "te2_tile1", "yee3d_zthin", "yee3d_zthin_cell", "yee3d_zthin_vec",
                                  "yee3d_zthin_wave", "yee3d_zthin3_vec", "yee3d_zthin3_wave"])
@pytest.mark.parametrize("ring", [1, 7, 32])
def test_exact_f64_equals_oracle_random_fields(eng, name, ring):
    base, _, suffix = name.rpartition("_")
    variant = suffix if suffix in ("cell", "vec", "wave", "tile", "tile2", "tile1") else None
    base = base if variant else name
    variant = variant or ("sweep" if base.startswith("yee3d") else "cell")
    # tile2: two steps per sub-block, so a ring block is a cooperative launch of many sub-blocks;
    # tile1: one launch per sub-block
    choice = {"tile2": dict(variant="tile", tile_steps=2),
              "tile1": dict(variant="tile", tile_coop=False)}.get(variant, dict(variant=variant))
    spec = _te2_spec() if base == "te2" else _random_cases()[base]()
    rng = np.random.default_rng(sum(map(ord, name)) + ring)
    s = oracle_from_spec(spec)
    job = eng.submit(spec, arith="exact", precision=np.float64, ring_steps=ring, **choice)
    for f in R.field_names(spec.mode):
        v = rng.standard_normal(spec.shape) * 1e-2
        getattr(s, f)[...] = v
        job.set_field(f, v)
    nsteps = 23
    job.advance(10).advance(nsteps - 10).sync(60000)
    R.run(s, nsteps)
    for f, arr in job.fields().items():
        np.testing.assert_array_equal(arr, getattr(s, f), err_msg=f)
    from oidt_b200.spec import PSI
    for fname, axis in PSI[spec.mode]:
        for side in (0, 1):
            np.testing.assert_array_equal(job.psi(fname, axis, side), getattr(s, psi_key(fname, axis, side)))
    ncomp = 4 if spec.mode == "yee3d" else 2
    for port in (0, 1):
        for c in range(ncomp):
            np.testing.assert_array_equal(job.dft(port, c), R.dft_complex(s, port, c), err_msg="port %d comp %d" % (port, c))
    job.release()


@pytest.mark.parametrize("choice", [{"variant": "cell", "rows": 2}, {"variant": "cell", "rows": 8},
                                    {"variant": "sweep", "march_depth": 1}, {"variant": "sweep", "march_depth": 3},
                                    {"variant": "sweep", "march_depth": 500}, {"variant": "vec"},
                                    {"variant": "wave"}])
@pytest.mark.parametrize("name", ["yee3d_te", "yee3d_tm", "yee3d_wide", "yee3d_graded"])
def test_launch_choices_equal_oracle(eng, name, choice):
    """Every launch choice the tuner may pick (tile rows 2 and 8 with ragged
    last tiles; march depths 1, 3 and one longer than the guide) computes
    the oracle's fields, CPML state and DFTs bit for bit."""
    spec = _random_cases()[name]()
    rng = np.random.default_rng(sum(map(ord, name)) + 17)
    s = oracle_from_spec(spec)
    job = eng.submit(spec, arith="exact", precision=np.float64, ring_steps=6, **choice)
    for f in R.field_names(spec.mode):
        v = rng.standard_normal(spec.shape) * 1e-2
        getattr(s, f)[...] = v
        job.set_field(f, v)
    job.advance(7).advance(14).sync(60000)
    R.run(s, 21)
    for f, arr in job.fields().items():
        np.testing.assert_array_equal(arr, getattr(s, f), err_msg=f)
    from oidt_b200.spec import PSI
    for fname, axis in PSI[spec.mode]:
        for side in (0, 1):
            np.testing.assert_array_equal(job.psi(fname, axis, side), getattr(s, psi_key(fname, axis, side)))
    for port in (0, 1):
        for c in range(4):
            np.testing.assert_array_equal(job.dft(port, c), R.dft_complex(s, port, c), err_msg="port %d comp %d" % (port, c))
    job.release()


def _s_forward(spec, dfts_inc, dfts_ref):
    from oidt_b200.sparams import forward_s
    return forward_s(spec, dfts_inc, dfts_ref)


def _field_errors(job, s, names):
    return {f: (float(np.linalg.norm((job.field(f).astype(np.float64) - getattr(s, f)).ravel())),
                float(np.linalg.norm(getattr(s, f).ravel()))) for f in names}


@pytest.mark.parametrize("variant", ["tile", "cell"])
def test_fp32_slab2d_full_run_within_targets(eng, variant):
    """The 400 x 200, 2000-step 2D case: float32 engine vs float64 oracle.

    Field error is checked at checkpoints while the pulse is in the domain
    (relative L2 <= 1e-5) and, at the final step -- when the pulse has left
    through the CPML and the field has decayed ~4 orders of magnitude -- as
    the error norm relative to the largest field norm of the run (<= 1e-5);
    the final-step relative L2 itself is recorded, not asserted (it measures
    the float32 rounding floor against the decayed residual)."""
    from oidt_b200 import workloads as W
    from oidt_b200.sparams import forward_s
    from oracle import cpu as OC
    from tests.helpers import dft_dict_oracle
    spec = W.slab2d()
    job = eng.submit(spec, arith="fast", precision=np.float32, variant=variant)
    s = oracle_from_spec(spec)
    peak = {f: 0.0 for f in ("EZ", "HX", "HY")}
    prev = 0
    for cpt in (500, 1000, 1500, 2000):
        job.advance(cpt - prev).sync(120000)
        OC.run_c(s, cpt - prev)
        prev = cpt
        errs = _field_errors(job, s, peak)
        for f, (e, nrm) in errs.items():
            peak[f] = max(peak[f], nrm)
            if cpt < 2000:
                assert e <= FIELD_TOL * nrm, (cpt, f, e / nrm)
            else:
                assert e <= FIELD_TOL * peak[f], (cpt, f, e / peak[f])
    d_eng = {(p, c): job.dft(p, c) for p in (0, 1) for c in (0, 1)}
    d_ora = dft_dict_oracle(s)
    for k in d_eng:
        assert rel_l2(d_eng[k], d_ora[k]) <= S_TOL, k
    S_e = forward_s(spec, d_eng, d_eng)
    S_o = forward_s(spec, d_ora, d_ora)
    assert np.max(np.abs(S_e["S21"] - S_o["S21"])) <= S_TOL
    job.release()


@pytest.mark.parametrize("variant", ["cell", "sweep", "vec", "wave"])
def test_fp32_strip3d_within_targets(eng, variant):
    """A reduced 3D rough strip (64 x 56 x 120, 700 steps) in float32 vs the
    float64 oracle on identical inputs, both 3D launch forms."""
    from oidt_b200 import workloads as W
    from oidt_b200.sparams import forward_s
    from tests.helpers import dft_dict_oracle
    kw = dict(nx=64, ny=56, nz=120, P=8, steps=700, nf=9, src_gap=4, port_gap=10)
    spec_r = W.strip3d(**kw)
    spec_i = W.strip3d(rough=False, **kw)
    out = {}
    from oracle import cpu as OC
    for tag, spec in (("i", spec_i), ("r", spec_r)):
        job = eng.submit(spec, arith="fast", precision=np.float32, variant=variant)
        job.run().sync(120000)
        s = oracle_from_spec(spec)
        OC.run_c(s, spec.nt)
        for f in R.field_names("yee3d"):
            err = rel_l2(job.field(f), getattr(s, f))
            assert err <= FIELD_TOL, (tag, f, err)
        out[tag] = ({(p, c): job.dft(p, c) for p in (0, 1) for c in range(4)}, dft_dict_oracle(s))
        job.release()
    S_e = forward_s(spec_r, out["i"][0], out["r"][0])
    S_o = forward_s(spec_r, out["i"][1], out["r"][1])
    for k in ("S11", "S21"):
        assert np.max(np.abs(S_e[k] - S_o[k])) <= S_TOL, k


def test_batch_equals_single_jobs(eng):
    """One multi-job advance over jobs of different solvers and sizes (2D TM
    and TE in both 2D forms, 3D sweep, 3D per-cell, 3D vector and ordered
    forms) equals advancing each job alone, bit for bit (float64 EXACT),
    including an odd tail that flips sweep buffers."""
    specs = [_random_cases()["tm2"](), _te2_spec(), _random_cases()["yee3d_te"](), _random_cases()["yee3d_tm"](),
             _random_cases()["yee3d_wide"](), _random_cases()["yee3d_p2"](), _random_cases()["tm2"](), _te2_spec()]
    variants = ["cell", "cell", "sweep", "cell", "vec", "wave", "tile", "tile"]
    solo, mix = [], []
    for sp, v in zip(specs, variants):
        solo.append(eng.submit(sp, arith="exact", precision=np.float64, ring_steps=6, variant=v))
        mix.append(eng.submit(sp, arith="exact", precision=np.float64, ring_steps=6, variant=v))
    for j in solo:
        j.advance(15).advance(14).sync(60000)
    eng.batch_advance(mix, 15)
    eng.batch_advance(mix, 14)
    for a, b in zip(solo, mix):
        b.sync(60000)
        for f, arr in a.fields().items():
            np.testing.assert_array_equal(b.field(f), arr, err_msg=f)
        nc = 4 if a.spec.mode == "yee3d" else 2
        for p in (0, 1):
            for c in range(nc):
                np.testing.assert_array_equal(b.dft(p, c), a.dft(p, c))
    for j in solo + mix:
        j.release()


def test_tile_form_in_waves_equals_per_cell(eng):
    """A served-size 2D grid (800 x 300) has more tiles than the B200 has SMs,
    so its sub-blocks run as separate launches in waves: fields, CPML psi and
    DFTs equal the per-cell launches' bit for bit (float64 EXACT), at ring
    sizes that end blocks mid-sub-block."""
    from oidt_b200 import workloads as W
    from oidt_b200.spec import PSI
    spec = W.slab2d(nx=800, ny=300, P=10, core_cells=10, src_x=40, ports=(60, 740), steps=60, nf=5,
                    rough=True, sigma_nm=10, lc_nm=50, seed=2)
    rng = np.random.default_rng(5)
    init = {f: rng.standard_normal(spec.shape) * 1e-2 for f in R.field_names("tm2")}
    jobs = []
    for variant in ("tile", "cell"):
        j = eng.submit(spec, arith="exact", precision=np.float64, ring_steps=7, variant=variant)
        for f, v in init.items():
            j.set_field(f, v)
        j.advance(30).sync(60000)
        jobs.append(j)
    a, b = jobs
    for f in R.field_names("tm2"):
        np.testing.assert_array_equal(a.field(f), b.field(f), err_msg=f)
    for name, axis in PSI["tm2"]:
        for side in (0, 1):
            np.testing.assert_array_equal(a.psi(name, axis, side), b.psi(name, axis, side))
    for port in (0, 1):
        for c in range(2):
            np.testing.assert_array_equal(a.dft(port, c), b.dft(port, c))
    for j in jobs:
        j.release()


def test_reset_reruns_identically(eng):
    """oidt_job_reset returns a job to step 0: a second run equals the first."""
    spec = _random_cases()["yee3d_te"]()
    job = eng.submit(spec, arith="exact", precision=np.float64)
    job.run().sync(60000)
    first = job.fields()
    d1 = job.dft(1, 3)
    job.reset().run().sync(60000)
    for f, arr in job.fields().items():
        np.testing.assert_array_equal(arr, first[f])
    np.testing.assert_array_equal(job.dft(1, 3), d1)
    job.release()


@pytest.mark.parametrize("batch", [False, True])
def test_two_line_launcher_equals_reference_smatrix(tmp_path, batch):
    """The launcher's 8 runs of two coupled lines (one at a time, or all 8
    advanced together) give the reference's 4 x 4 S-matrix bit for bit
    (float64, exact arithmetic), and a touchstone file of 4 ports."""
    from oidt_b200.simulation_launcher import launch
    from oidt_b200.sparams import extract_sparams, read_touchstone
    z = G.load("tm2_lines2")
    usr = G.usr_of(z)
    path = launch(usr, "tm2", cwd=str(tmp_path), batch=batch, verbose=False)
    assert path.endswith(".s4p")
    out = os.path.join(str(tmp_path), usr["output_dir"])
    data = {f[:-4]: np.load(os.path.join(out, f)) for f in os.listdir(out) if f.endswith(".npy")}
    assert len(data) == 24  # per line: fi, bi, ft, br, fr, bt, each Ez and Hy, as the reference saves
    S = extract_sparams(usr, "tm2", data)
    np.testing.assert_array_equal(S, z["S_mat"])
    freqs, S_file, _ = read_touchstone(path)
    assert S_file.shape == S.shape



def test_dft_into_caller_buffer(eng):
    """Job.dft(out=...) reads into a caller's (here page-locked) buffer and
    equals the allocating read; a buffer of the wrong shape is refused."""
    import torch
    spec = _random_cases()["yee3d_te"]()
    job = eng.submit(spec, arith="exact", precision=np.float64)
    job.run().sync(60000)
    want = job.dft(1, "hy")
    t = torch.empty(want.shape + (2,), dtype=torch.float64, pin_memory=True)
    buf = t.numpy().view(np.complex128)[..., 0]
    got = job.dft(1, "hy", out=buf)
    assert got is buf
    np.testing.assert_array_equal(buf, want)
    with pytest.raises(ValueError):
        job.dft(1, "hy", out=np.empty(want.shape[1:], dtype=np.complex128))
    job.release()
