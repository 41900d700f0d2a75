"""Drop-in for the reference's ``simulation_launcher.py``: the 4 runs per line
and the extraction (``FDTD_2D_TM/.../simulation_launcher.py:22-47``).

The reference spawns ``python fdtd_main.py <line> <f|b> <i|r>`` four times
per line with 5 s sleeps and ignores the exit codes.  Here the runs share one
engine context in one process; errors propagate.  The 4 L runs of L lines are
independent, so with ``--batch`` all of them advance together in multi-job
launches (``oidt_batch_advance``); when their device memory would exceed the
context's budget, the lines go in groups that fit.  The first reflected run
of line 0 generates the roughness profiles that the later rough runs load, as
in the reference (specs are built in the reference's run order).
"""
from __future__ import annotations

import argparse
import os

import numpy as np

from .engine import Engine
from .extract_sparams import extract
from .fdtd_main import load_user_dict, output_names, profiles_for, run
from .refsetup import build_spec

RUN_ORDER = ((0, "f", "i"), (0, "f", "r"), (0, "b", "i"), (0, "b", "r"))


def _advance_together(eng, specs, cwd, usr, mode):
    """Advance (line, direction, kind, spec) runs in one batch and save
    their .npy outputs."""
    prec = np.dtype(specs[0][3].precision)
    arith = "exact" if prec == np.float64 else "fast"
    jobs = [eng.submit(s, arith=arith, precision=prec) for (_, _, _, s) in specs]
    steps = min(s.nt for (_, _, _, s) in specs)
    eng.batch_advance(jobs, steps)
    for j, (l, d, k, s) in zip(jobs, specs):
        if s.nt > steps:
            j.advance(s.nt - steps)
    out_dir = os.path.join(cwd, usr["output_dir"])
    os.makedirs(out_dir, exist_ok=True)
    cdt = np.complex128 if prec == np.float64 else np.complex64
    for j, (l, d, k, s) in zip(jobs, specs):
        j.sync()
        for (port, ci), stem in output_names(mode, l, d, k).items():
            np.save(os.path.join(out_dir, stem), j.dft(port, ci).astype(cdt))
        j.release()


def batch_groups(sizes, free_bytes):
    """Consecutive groups of runs whose device bytes fit ``free_bytes``
    together (a run larger than that forms a group of its own)."""
    groups, cur, used = [], [], 0
    for i, b in enumerate(sizes):
        if cur and used + b > free_bytes:
            groups.append(cur)
            cur, used = [], 0
        cur.append(i)
        used += b
    if cur:
        groups.append(cur)
    return groups


def launch(usr: dict, mode: str, cwd: str = ".", device: int = 0, batch: bool = False, verbose=True) -> str:
    eng = Engine(device)
    try:
        runs = [(line, d, k) for line in range(usr["num_lines"]) for (_, d, k) in RUN_ORDER]
        if not batch:
            for (l, d, k) in runs:
                run(usr, mode, l, d, k, cwd=cwd, engine=eng, verbose=verbose)
        else:
            specs = []
            for (l, d, k) in runs:  # the reference's run order: profiles are made before they are loaded
                prof = profiles_for(usr, mode, l, d, k, cwd)
                specs.append((l, d, k, build_spec(usr, mode, l, d, k, profiles=prof)))
            st = eng.stats()
            free = st["hbm_budget"] - st["hbm_in_use"]
            sizes = [eng.job_bytes(s) for (_, _, _, s) in specs]
            for g in batch_groups(sizes, free):
                _advance_together(eng, [specs[i] for i in g], cwd, usr, mode)
    finally:
        eng.close()
    path = extract(usr, mode, cwd)
    if verbose:
        print("Done extracting S-parameters! The touchstone file is", path)
    return path


def main(mode: str = None, argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--mode", default=mode or os.environ.get("OIDT_MODE"), choices=("tm2", "te2", "yee3d"))
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--batch", action="store_true")
    a = ap.parse_args(argv)
    usr = load_user_dict("")
    launch(usr, a.mode, device=a.device, batch=a.batch)


if __name__ == "__main__":
    main()
