"""Drop-in for the reference's ``extract_sparams.py``.

    python -m oidt_b200.extract_sparams --mode tm2|te2|yee3d [<tag>]

Reads the DFT ``.npy`` files of the 4 runs per line from ``./<output_dir>``,
builds the S-matrix with the reference's conventions
(``extract_sparams.py:48-104``; 3D ``:48-131``) and writes
``./<output_dir>/<sparam_file>.s<2L>p`` (RI, z0 = 50, OIDT comment line
first), the file SROPEE's ``rf.Network('./Input/'+file)`` reads
(``SROPEE/1_Full synthesis/Run_full_synthesis.py:167-168``).  The
reference's dB/angle PDF plots are not produced.
"""
from __future__ import annotations

import argparse
import os

import numpy as np

from .fdtd_main import load_user_dict
from .refsetup import derive
from .sparams import extract_sparams, write_touchstone


def extract(usr: dict, mode: str, cwd: str = ".") -> str:
    dv = derive(usr, mode, "r")
    u = dv.usr
    out_dir = os.path.join(cwd, u["output_dir"])
    data = {f[:-4]: np.load(os.path.join(out_dir, f)) for f in os.listdir(out_dir) if f.endswith(".npy")}
    S = extract_sparams(usr, mode, data)
    return write_touchstone(os.path.join(out_dir, u["sparam_file"]), dv.sparam_freqs, S)


def main(mode: str = None, argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("tag", nargs="?", default="")
    ap.add_argument("--mode", default=mode or os.environ.get("OIDT_MODE"), choices=("tm2", "te2", "yee3d"))
    a = ap.parse_args(argv)
    usr = load_user_dict(a.tag) if a.tag else load_user_dict("")
    print("saved", extract(usr, a.mode))


if __name__ == "__main__":
    main()
