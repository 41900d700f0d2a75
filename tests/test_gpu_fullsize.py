"""Parity at the full benchmark size: the 3D strip of 128 x 128 x 256 cells
(20 nm, CPML 10, rough sidewalls sigma 10 nm / Lc 50 nm, 4000 steps, 41
frequencies) in FP32 against the FP64 exact-arithmetic instantiation of the
same kernels on the GPU, which equals the float64 oracle bit for bit on the
smaller grids of test_gpu_parity.py (the CPU oracle needs minutes here).

Tolerances: field relative L2 <= 1e-5 at step 1500 (the pulse inside the
domain) and |S21 difference| <= 1e-4 at the end of the run."""
import numpy as np
import pytest

from oidt_b200 import workloads as W
from oidt_b200.engine import Engine
from oidt_b200.sparams import forward_s
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-5
S_TOL = 1e-4
CHECKPOINT = 1500


@pytest.mark.parametrize("variant", ["cell", "sweep", "vec", "wave"])
def test_fp32_vs_fp64_exact_at_bench_size(variant):
    eng = Engine(0)
    kw = dict(nx=128, ny=128, nz=256, dx=20e-9, P=10, steps=4000, nf=41, sigma_nm=10.0, lc_nm=50.0, seed=0)
    spec_r, spec_i = W.strip3d(**kw), W.strip3d(rough=False, **kw)
    dft = {}
    for prec, arith in ((np.float32, "fast"), (np.float64, "exact")):
        for tag, spec in (("r", spec_r), ("i", spec_i)):
            job = eng.submit(spec, arith=arith, precision=prec, variant=variant)
            job.advance(CHECKPOINT).sync(120000)
            if tag == "r":
                fields = {f: job.field(f) for f in ("EX", "EY", "EZ", "HX", "HY", "HZ")}
                if prec == np.float32:
                    f32 = fields
                else:
                    for f, ref in fields.items():
                        err = rel_l2(f32[f].astype(np.float64), ref)
                        assert err <= FIELD_TOL, (f, err)
            job.run().sync(120000)
            dft[(np.dtype(prec).name, tag)] = {(p, c): job.dft(p, c) for p in (0, 1) for c in range(4)}
            job.release()
    s32 = forward_s(spec_r, dft[("float32", "i")], dft[("float32", "r")])
    s64 = forward_s(spec_r, dft[("float64", "i")], dft[("float64", "r")])
    for k in ("S11", "S21"):
        assert np.max(np.abs(s32[k] - s64[k])) <= S_TOL, (k, np.max(np.abs(s32[k] - s64[k])))
    eng.close()
