"""Drop-in for the reference's ``fdtd_main.py`` (one S-parameter simulation).

    python -m oidt_b200.fdtd_main <line> <f|b> <i|r> --mode tm2|te2|yee3d

or, in a reference working directory, a two-line ``fdtd_main.py``::

    from oidt_b200.fdtd_main import main
    main(mode="tm2")

Same inputs as the reference (``user_dict_<line>.pkl`` in the working
directory, else the ``user_config.py`` module there, ``fdtd_main.py:29-41``),
same run selector (``<line> <direction> <kind>``, ``:56-66``), same outputs
(``./<output_dir>/{ez,hy}_{fi,bi,ft,br,fr,bt}_l<k>.npy`` and the 3D
``{ex,ey,hx,hy}_...`` set, ``:349-386``), same roughness-profile files
(``rough_profiles/profile_{upper,lower}_s<..>nm_lc<..>nm_r<..>.npy``).
The time loop runs on the GPU through ``liboidt.so``; the DFT arrays are
saved with the reference's dtype (complex64 for float32 runs) unless
``--full-precision`` keeps the engine's complex128.
"""
from __future__ import annotations

import argparse
import os
import pickle
import sys
import time

import numpy as np

from .refsetup import derive, build_spec
from .spec import DFT_COMPS


def dict_from_module(module) -> dict:
    """Public scalar/str/type settings of a config module (aux_funcs.py:64-71)."""
    out = {}
    for k in dir(module):
        v = getattr(module, k)
        if k[0] != "_" and type(v) in (float, str, int, type, bool):
            out[k] = v
    return out


def load_user_dict(tag: str, cwd: str = ".") -> dict:
    """``user_dict_<tag>.pkl`` if present, else the working directory's
    ``user_config`` module (written to ``user_dict.pkl`` as the reference does)."""
    p = os.path.join(cwd, "user_dict_{}.pkl".format(tag))
    if os.path.exists(p):
        with open(p, "rb") as fh:
            return pickle.load(fh)
    print("loading default configuration")
    sys.path.insert(0, os.path.abspath(cwd))
    import user_config  # noqa: the reference's per-directory configuration module
    usr = dict_from_module(user_config)
    with open(os.path.join(cwd, "user_dict.pkl"), "wb") as fh:
        pickle.dump(usr, fh)
    return usr


def profiles_for(usr: dict, mode: str, line: int, direction: str, kind: str, cwd: str = "."):
    """Roughness profiles for this run: none for incident runs; generated and
    saved on the first reflected run of line 0 (forward), loaded otherwise
    (fdtd_main.py:67-79).  Generation is the seeded exponential-ACF sequence
    of ``workloads.sidewall_profile`` (seed = profile_number)."""
    from .workloads import sidewall_profile
    if kind == "i" or not usr.get("rough_toggle"):
        return None
    dv = derive(usr, mode, "r")
    up, lo = os.path.join(cwd, dv.profile_upper + ".npy"), os.path.join(cwd, dv.profile_lower + ".npy")
    if line == 0 and direction == "f" or not (os.path.exists(up) and os.path.exists(lo)):
        rng = np.random.default_rng(int(usr.get("profile_number", 0)))
        n = dv.p2 - dv.p1
        upper = sidewall_profile(n, float(dv.rstd), float(dv.racl), rng, round_cells=False)
        ctype = 3  # generate_fg_mask is called with its default correlation (fdtd_funcs.py:165)
        lower = sidewall_profile(n, float(dv.rstd), float(dv.racl), rng, round_cells=False) if ctype == 3 else upper
        os.makedirs(os.path.dirname(up), exist_ok=True)
        np.save(up, upper)
        np.save(lo, lower)
        return upper, lower
    return np.load(up), np.load(lo)


def output_names(mode: str, line: int, direction: str, kind: str):
    """{(port, comp index): file stem} saved by this run (fdtd_main.py:365-383)."""
    tags = {("i", "f"): ((0, "fi"),), ("i", "b"): ((1, "bi"),),
            ("r", "f"): ((0, "ft"), (1, "br")), ("r", "b"): ((0, "fr"), (1, "bt"))}[(kind, direction)]
    out = {}
    for port, tag in tags:
        for ci, c in enumerate(DFT_COMPS[mode]):
            out[(port, ci)] = "%s_%s_l%d" % (c, tag, line + 1)
    return out


def run(usr: dict, mode: str, line: int, direction: str, kind: str, cwd: str = ".", device: int = 0,
        arith: str = None, full_precision: bool = False, engine=None, verbose: bool = True) -> dict:
    """One simulation; returns {file stem: complex array} and writes the .npy files."""
    from .engine import Engine
    profiles = profiles_for(usr, mode, line, direction, kind, cwd)
    spec = build_spec(usr, mode, line, direction, kind, profiles=profiles)
    prec = np.dtype(spec.precision)
    arith = arith or ("exact" if prec == np.float64 else "fast")
    own = engine is None
    eng = engine or Engine(device)
    try:
        if verbose:
            shp = " x ".join(str(n) for n in spec.shape)
            print("The simulation size will be: {} cells over {} time steps".format(shp, spec.nt))
        t0 = time.time()
        job = eng.submit(spec, arith=arith, precision=prec)
        job.run().sync()
        loop = time.time() - t0
        if verbose:
            print("Speed in MCells/sec: {:}".format(spec.ncells * spec.nt / (1e6 * loop)))
        out_dir = os.path.join(cwd, spec.meta["derived"].usr["output_dir"])
        os.makedirs(out_dir, exist_ok=True)
        cdt = np.complex128 if (full_precision or prec == np.float64) else np.complex64
        res = {}
        for (port, ci), stem in output_names(mode, line, direction, kind).items():
            arr = job.dft(port, ci).astype(cdt)
            np.save(os.path.join(out_dir, stem), arr)
            res[stem] = arr
        job.release()
    finally:
        if own:
            eng.close()
    return res


def main(mode: str = None, argv=None):
    ap = argparse.ArgumentParser(description="OIDT S-parameter simulation on a B200 (drop-in for fdtd_main.py)")
    ap.add_argument("line", type=int)
    ap.add_argument("direction", choices=("f", "b"))
    ap.add_argument("kind", choices=("i", "r"))
    ap.add_argument("--mode", default=mode or os.environ.get("OIDT_MODE"), choices=("tm2", "te2", "yee3d"))
    ap.add_argument("--device", type=int, default=int(os.environ.get("OIDT_DEVICE", "0")))
    ap.add_argument("--arith", choices=("exact", "fast"))
    ap.add_argument("--full-precision", action="store_true")
    a = ap.parse_args(argv)
    if a.mode is None:
        ap.error("--mode is required (tm2, te2 or yee3d: the reference directory this replaces)")
    usr = load_user_dict(str(a.line))
    run(usr, a.mode, a.line, a.direction, a.kind, device=a.device, arith=a.arith, full_precision=a.full_precision)
    print("results saved!")


if __name__ == "__main__":
    main()
