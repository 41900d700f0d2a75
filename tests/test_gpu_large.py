"""The large single 3D run at full size: 384 x 384 x 1024 cells (151 M), 15 nm,
16-cell CPML, a 1 um silicon rib with rough sidewalls, 2000 steps.  The FP32
production path against the FP64 exact-arithmetic instantiation of the same
kernels on the GPU -- equal to the float64 oracle bit for bit on the parity
grids of test_gpu_parity.py; the CPU oracle would need hours here.

Tolerance: field relative L2 <= 1e-5 for each of the six components at step
1000 (pulse inside the domain) and at step 2000."""
import pytest

from oidt_b200 import large

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-5


def test_fp32_vs_fp64_exact_at_large_size():
    out = large.run(steps=2000, checkpoint=1000)
    assert out["cells"] == 384 * 384 * 1024
    for step, errs in out["fp32_vs_fp64_rel_l2"].items():
        for f, e in errs.items():
            assert e <= FIELD_TOL, (step, f, e)
    assert out["float32"]["gcell_updates_per_s"] > 0 and out["float64"]["gcell_updates_per_s"] > 0
