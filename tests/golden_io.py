"""Helpers that read the golden fixtures written by ``tests/golden/make_golden.py``."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    path = os.path.join(GOLDEN, name + ".npz")
    return np.load(path, allow_pickle=False)


def usr_of(z):
    usr = json.loads(str(z["usr_json"]))
    usr["precision"] = {"float32": np.float32, "float64": np.float64}[usr["precision"]]
    return usr


def sims_of(z):
    tags = sorted({k.split("/")[0] for k in z.files if "/" in k})
    return [(int(t[0]), t[1], t[2]) for t in tags]


def profiles_of(z):
    if "profile_upper" in z.files:
        return (z["profile_upper"], z["profile_lower"])
    return None


def oracle_array(s, name):
    """Map a reference device-array name (``fdtd_main.py`` ``d<NAME>``) to the
    oracle namespace ``s``."""
    if name == "J_SRC":
        return s.cfg.J_SRC
    if hasattr(s, name):
        return getattr(s, name)
    d = s.dft
    if s.mode == "yee3d":
        return d[name]
    # 2D: EZ1r / HY1r (TM) or EY1r / HZ1r (TE) -> E1r / H1r
    return d[name[0] + name[2:]]
