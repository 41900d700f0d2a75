"""Output formats: touchstone files byte-identical to the reference's
examples after a read/write round trip; DFT .npy naming and dtype."""
import os

import numpy as np

from oidt_b200.sparams import read_touchstone, touchstone_text, write_touchstone
from tests import golden_io as G


def test_touchstone_roundtrip_is_byte_identical():
    for name in ("ref_example_3d.s2p", "ref_example_tm2.s4p"):
        path = os.path.join(G.GOLDEN, name)
        f, S, z0 = read_touchstone(path)
        assert touchstone_text(f, S, z0) == open(path).read()


def test_touchstone_write_read(tmp_path):
    rng = np.random.default_rng(0)
    for n in (2, 4, 6):
        S = rng.standard_normal((5, n, n)) + 1j * rng.standard_normal((5, n, n))
        f = np.linspace(1.8e14, 2.1e14, 5)
        p = write_touchstone(str(tmp_path / ("t%d" % n)), f, S)
        f2, S2, z0 = read_touchstone(p)
        np.testing.assert_array_equal(f, f2)
        np.testing.assert_array_equal(S, S2)
        assert z0 == 50.0
