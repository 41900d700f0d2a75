"""Small fixed workloads for profiler captures (ncu launch lists and
single-kernel captures).

    python -m oidt_b200.prof --workload strip3d --steps 64 [--variant cell|sweep] [--no-graphs]

Workloads: strip3d (128 x 128 x 256), strip3d_large (384 x 384 x 1024),
slab2d (400 x 200), scatter and zwave (the scattering-loss and
wave-impedance runs at their reference settings, 75 M and 97 M cells).

Runs the named workload for a few hundred launches and exits; the device
state of the default 3D case (128 x 128 x 256 cells, FP32) is about 0.4 GB,
so a multi-pass capture of one launch stays small.
"""
from __future__ import annotations

import argparse

import numpy as np

from . import workloads as W
from .engine import Engine


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="strip3d",
                    choices=("strip3d", "slab2d", "strip3d_large", "scatter", "zwave"))
    ap.add_argument("--steps", type=int, default=64)
    ap.add_argument("--variant", default="cell", choices=("cell", "sweep"))
    ap.add_argument("--no-graphs", action="store_true")
    ap.add_argument("--precision", default="float32", choices=("float32", "float64"))
    a = ap.parse_args(argv)
    if a.workload == "strip3d":
        spec = W.strip3d(steps=max(a.steps, 64))
    elif a.workload == "strip3d_large":
        spec = W.strip3d(nx=384, ny=384, nz=1024, dx=15e-9, P=16, steps=max(a.steps, 64), core_x_nm=220,
                         core_y_nm=1000, seed=7)
    elif a.workload == "scatter":
        from . import scatter
        cfg = scatter.config()
        spec = scatter.build_spec(cfg, scatter.realization_profiles(cfg, 1)[0])
    elif a.workload == "zwave":
        from . import zwave
        spec = zwave.build_spec(zwave.config())
    else:
        spec = W.slab2d(steps=max(a.steps, 64))
    eng = Engine(0)
    job = eng.submit(spec, precision=np.dtype(a.precision), variant=a.variant, graphs=not a.no_graphs)
    job.advance(a.steps).sync()
    print("ran", a.steps, "steps of", a.workload, spec.shape)
    job.release()
    eng.close()


if __name__ == "__main__":
    main()
