"""Scattering-loss workload on the GPU, against the reference's own run
(``tests/golden/scatter_*.npz``: ``scattering_loss/fdtd_main.py`` in float32
on a tiny grid, 82 steps, planted rough sidewalls) and the oracle.

* Fields: the engine's float32 EXACT instantiation equals the reference's
  final fields bit for bit (same IEEE operations in the same order).
* Planes: the reference accumulates its DFTs in float32, the engine in
  float64, so planes agree to float32 accumulation error:
  max |engine - reference| <= 2e-5 x max |reference| per plane.
* Loss: |alpha(engine) - alpha(reference)| <= 1e-4 |alpha(reference)|; the
  float32 fast-arithmetic engine against the float64 oracle likewise.
* Batched realizations equal one-at-a-time runs bit for bit."""
import json
import os

import numpy as np
import pytest

from oidt_b200 import scatter
from oidt_b200.engine import Engine
from tests import golden_io as G

CASES = ["scatter_te", "scatter_tm"]
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not all(os.path.exists(os.path.join(G.GOLDEN, c + ".npz")) for c in CASES),
                                 reason="scattering-loss fixtures not generated (tests/golden/make_golden.py)")]
PLANE_TOL = 2e-5
ALPHA_TOL = 1e-4


@pytest.fixture(scope="module")
def eng():
    e = Engine(0)
    yield e
    e.close()


def _load(case):
    z = np.load(os.path.join(G.GOLDEN, case + ".npz"))
    return z, json.loads(str(z["over_json"])), (z["profile_upper"], z["profile_lower"])


def _tag(z):
    return [k[len("npy_ex1_fft"):] for k in z.files if k.startswith("npy_ex1_fft")][0]


@pytest.mark.parametrize("variant", ["cell", "sweep"])
@pytest.mark.parametrize("case", CASES)
def test_exact_f32_run_equals_reference(eng, case, variant):
    z, over, prof = _load(case)
    cfg = scatter.config(**over)
    spec = scatter.build_spec(cfg, prof)
    job = eng.submit(spec, arith="exact", precision=np.float32, ring_steps=7, variant=variant)
    job.run().sync(60000)
    for f in ("EX", "EY", "EZ", "HX", "HY", "HZ"):
        np.testing.assert_array_equal(job.field(f), z["dev_" + f], err_msg=f)
    planes = scatter.planes_from_job(job)
    tag = _tag(z)
    for name, got in planes.items():
        want = z["npy_%s%s_fft%s" % (name[:2], name[2], tag)]
        scale = float(np.max(np.abs(want)))
        assert scale > 0, name
        assert float(np.max(np.abs(got.astype(np.complex128) - want))) <= PLANE_TOL * scale, name
    dv = scatter.derive(cfg)
    a = scatter.loss(planes, dv.delta_x, dv.extra["ell"])["alpha"]
    want = float(z["results"][2, 0])
    assert abs(a - want) <= ALPHA_TOL * abs(want), (a, want)
    job.release()


@pytest.mark.parametrize("case", CASES)
def test_fast_f32_alpha_against_float64_oracle(eng, case):
    from oracle import scatter_ref as S
    z, over, prof = _load(case)
    cfg = scatter.config(**over)
    job = eng.submit(scatter.build_spec(cfg, prof), arith="fast", precision=np.float32)
    job.run().sync(60000)
    dv = scatter.derive(cfg)
    a = scatter.loss(scatter.planes_from_job(job), dv.delta_x, dv.extra["ell"])["alpha"]
    job.release()
    s64 = _oracle64(over, prof)
    dx = np.float64(s64.cfg.delta_x)
    ref = float(S.alpha(_planes128(s64), dx, (s64.cfg.p2z - s64.cfg.p1z) * dx))
    assert abs(a - ref) <= ALPHA_TOL * abs(ref), (a, ref)


def _planes128(s):
    return {c.lower() + cut: s.planes[c + cut + "r"] + 1j * s.planes[c + cut + "i"]
            for cut in "12" for c in ("EX", "EY", "HX", "HY")}


def _oracle64(over, prof):
    """The oracle's run with every array in float64 (coefficients computed in
    float32 as the reference does, then widened)."""
    from oracle import scatter_ref as S
    s = S.build(S.settings(**over), prof)
    for name, v in list(vars(s).items()):
        if isinstance(v, np.ndarray) and v.dtype == np.float32:
            setattr(s, name, v.astype(np.float64))
    s.planes = {k: v.astype(np.float64) for k, v in s.planes.items()}
    s.dft = {k: v.astype(np.float64) for k, v in s.dft.items()}
    s.cfg.J_SRC = np.asarray(s.cfg.J_SRC, dtype=np.float64)
    S.run(s)
    return s


def _rough_cfg():
    """The fixture's tiny grid with roughness of about two cells (the
    default 15 nm is a fifth of a 73 nm cell: most draws leave the staircase
    mask unchanged)."""
    _, over, _ = _load("scatter_te")
    return scatter.config(**dict(over, rough_std=150e-9, rough_acl=300e-9))


def test_batched_realizations_equal_plain_runs(eng):
    cfg = _rough_cfg()
    profs = scatter.realization_profiles(cfg, 3, master_seed=4)
    _, plain = scatter.run(eng, cfg, profs, batched=False)
    _, batch = scatter.run(eng, cfg, profs, batched=True)
    for a, b in zip(plain, batch):
        assert a["alpha"] == b["alpha"]
        for k in a["planes"]:
            np.testing.assert_array_equal(a["planes"][k], b["planes"][k], err_msg=k)
    assert len({r["alpha"] for r in batch}) == 3  # distinct realizations


def test_batched_realizations_split_by_budget():
    """With a context budget that holds two of three jobs, the batched path
    runs them in two groups and still equals the one-at-a-time runs."""
    cfg = _rough_cfg()
    profs = scatter.realization_profiles(cfg, 3, master_seed=6)
    probe = Engine(0)
    need = probe.job_bytes(scatter.build_spec(cfg, profs[0]), precision=np.float32)
    _, plain = scatter.run(probe, cfg, profs, batched=False)
    probe.close()
    small = Engine(0, hbm_budget=int(2.5 * need))
    _, batch = scatter.run(small, cfg, profs, batched=True)
    small.close()
    assert [r["alpha"] for r in batch] == [r["alpha"] for r in plain]
