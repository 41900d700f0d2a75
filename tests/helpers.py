"""Shared test helpers: run the oracle on exactly the inputs of an engine job."""
import numpy as np

from oracle import fdtd_ref as R

FIELD_NAMES = {0: "EX", 1: "EY", 2: "EZ", 3: "HX", 4: "HY", 5: "HZ"}


def oracle_from_spec(spec, dtype=np.float64):
    """Oracle state with the spec's arrays (cast to ``dtype``)."""
    return R.from_spec(spec, dtype)


def psi_key(name, axis, side):
    return "PSI_%s_%s%s" % (name, "XYZ"[axis], ("LO", "HI")[side])


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) or np.iscomplexobj(b) else np.float64)
    b = np.asarray(b, dtype=a.dtype)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))


def dft_dict_oracle(s):
    """{(port, comp): complex DFT} from an oracle state, engine comp order."""
    nc = 4 if s.mode == "yee3d" else 2
    return {(p, c): R.dft_complex(s, p, c) for p in (0, 1) for c in range(nc)}
