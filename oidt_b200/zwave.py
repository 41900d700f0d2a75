"""Wave impedance of the guided mode just outside the core: a 3D run that
records colocated Ey, Ez, Hy, Hz along x through the guide's centre every
step, then Z(f) = E(f) / H(f) from their FFTs at a cell in the cladding,
against the slab-waveguide formula.

Reference: ``FDTD/GPU/FDTD_3D/wave_impedance``
  fdtd_config.py:17-60            settings (``REFERENCE_CONFIG`` below)
  fdtd_config.py:67-200           derived grid, steps, source; cy = ny // 2, cz = nz // 2
  fdtd_main.py:264-299            time loop (the S-parameter 3D launch order) and the
                                  per-step line recording (map_efield_zwave / map_hfield_zwave)
  fdtd_main.py:341-346            saved records: TE ey_te_zwave, hz_te_zwave; TM ez_tm_zwave, hy_tm_zwave
  zwave.py:17-64                  FFT ratio at x = bx - 3 and the slab formula

The solver is the S-parameter 3D solver (same kernels, launch order, source
boxes), so a run is an engine job built by :func:`oidt_b200.refsetup.build_spec`
from the equivalent settings, with the engine's line probe
(``oidt_job_desc.probe``) in place of the reference's recording kernels.
The engine also folds its port DFTs at the two cut planes (one frequency,
f0), which this workload does not read.
"""
from __future__ import annotations

import argparse
import json
import os

import numpy as np

from . import refsetup
from .scatter import find_neff, usr_of
from .spec import SimSpec

# fdtd_config.py:17-60 of wave_impedance
REFERENCE_CONFIG = dict(
    eps_rel_bg=1.5 ** 2, eps_rel_fg=3.5 ** 2, sgl_wg_length=14.0e-6, sgl_wg_width=2.0e-6, sgl_wg_height=0.2e-6,
    port1_length=4.0e-6, port2_length=0.0e-6, rough_std=15.0e-9, rough_acl=700.0e-9, tol_std=10.0, tol_acl=10.0,
    rough_toggle=False, ctype=3, output_dir="Results", profile_number=0, source_type=1, source_amp=5.0,
    wave_packet_bw=0.5, gauss_pulse_deg=-6, f0=194.8e12, source_condition="TM", harmonics=1.000, num_flights=2.0,
    points_per_wl=40, num_cpml=20, buffer_zhat=20, nx_clad_wl=0.75, ny_clad_wl=0.75)

# records the reference saves per source condition (fdtd_main.py:341-346)
RECORDS = {"TE": (("ey", "ey_te_zwave"), ("hz", "hz_te_zwave")),
           "TM": (("ez", "ez_tm_zwave"), ("hy", "hy_tm_zwave"))}


def config(**overrides) -> dict:
    unknown = set(overrides) - set(REFERENCE_CONFIG)
    if unknown:
        raise KeyError("unknown wave-impedance settings: %s" % sorted(unknown))
    return dict(REFERENCE_CONFIG, **overrides)


def derive(cfg: dict) -> refsetup.Derived:
    """Grid, steps and source (fdtd_config.py:67-200); ``extra`` adds the
    probe line (cy, cz) and the analysis cell x = bx - 3 (zwave.py:18-19)."""
    dv = refsetup.derive(usr_of(cfg), "yee3d", "r")
    dv.extra.update(cy=dv.ny // 2, cz=dv.nz // 2, xref=dv.bx - 3)
    return dv


def build_spec(cfg: dict, profiles=None) -> SimSpec:
    """Engine job with the line probe at (cy, cz); smooth unless
    ``rough_toggle`` and ``profiles`` = (upper, lower) are given."""
    u = usr_of(cfg)
    if profiles is None:
        u["rough_toggle"] = False
    spec = refsetup.build_spec(u, "yee3d", 0, "f", "r", profiles=profiles)
    dv = spec.meta["derived"]
    spec.meta.update(workload="wave_impedance", probe=(dv.ny // 2, dv.nz // 2))
    return spec


def records_from_job(job, cfg: dict) -> dict:
    """The reference-named [nt, nx] records of this source condition."""
    return {name: job.probe(comp) for comp, name in RECORDS[cfg["source_condition"]]}


def save_records(out_dir: str, records: dict) -> list:
    os.makedirs(out_dir, exist_ok=True)
    paths = []
    for name, arr in records.items():
        p = os.path.join(out_dir, name + ".npy")
        np.save(p, arr)
        paths.append(p)
    return paths


def impedance(records: dict, cfg: dict, dv=None, cell: int = 3):
    """(ff, Z) of the recorded line at x = bx - cell (zwave.py:19-34):
    TE Z = Ey(f) / Hz(f); TM Z = -Ez(f) / Hy(f), on the FFT's frequency grid
    ff = n / (dt nt)."""
    dv = dv or derive(cfg)
    x = dv.bx - cell
    if cfg["source_condition"] == "TE":
        z = np.fft.fft(records["ey_te_zwave"][:, x]) / np.fft.fft(records["hz_te_zwave"][:, x])
    else:
        z = -1 * np.fft.fft(records["ez_tm_zwave"][:, x]) / np.fft.fft(records["hy_tm_zwave"][:, x])
    ff = np.arange(0, dv.nt, 1) / (dv.delta_t * dv.nt)
    return ff, z


def analytic(cfg: dict, fa=None, n1=3.5, n2=1.5, d=100e-9):
    """Slab-mode wave impedance in the cladding (zwave.py:36-57): TE
    -j w mu / gamma, TM -gamma / (j w eps0 n2^2), gamma the decay constant."""
    fa = np.linspace(100e12, 300e12, num=100) if fa is None else np.asarray(fa, dtype=np.float64)
    mode = "te" if cfg["source_condition"] == "TE" else "tm"
    eps0 = 1e-9 / (36 * np.pi)
    mu = 4.0e-7 * np.pi
    k0 = 2 * np.pi * fa / 3e8
    neff = np.array([find_neff(n1, n2, d, k, mode=mode) for k in k0])
    beta = k0 * neff
    gamma = np.sqrt(beta ** 2 - n2 ** 2 * k0 ** 2)
    if mode == "te":
        return fa, -1j * 2 * np.pi * fa * mu / gamma
    return fa, -1 * gamma / (1j * 2 * np.pi * fa * eps0 * n2 ** 2)


def run(eng, cfg: dict, arith="fast", precision=np.float32, variant="cell"):
    """One run; returns (records, job steps)."""
    spec = build_spec(cfg)
    job = eng.submit(spec, arith=arith, precision=precision, variant=variant)
    job.run().sync()
    rec = records_from_job(job, cfg)
    job.release()
    return rec, spec.nt


def main(argv=None):
    ap = argparse.ArgumentParser(description="Wave impedance of the guided mode next to the core")
    ap.add_argument("--set", nargs="*", default=[], help="setting=value overrides of the reference config")
    ap.add_argument("--out", default=None, help="directory for the reference-named records")
    a = ap.parse_args(argv)
    over = {}
    for kv in a.set:
        k, v = kv.split("=", 1)
        over[k] = json.loads(v) if v[:1] in "0123456789-[{tf\"" else v
    cfg = config(**over)
    from .engine import Engine
    import time
    eng = Engine(0)
    dv = derive(cfg)
    t0 = time.perf_counter()
    rec, nt = run(eng, cfg)
    sec = time.perf_counter() - t0
    eng.close()
    if a.out:
        save_records(a.out, rec)
    ff, z = impedance(rec, cfg, dv)
    fa, za = analytic(cfg)
    # compare on the FFT bins inside the analytic band where the source has energy
    band = (ff >= fa[0]) & (ff <= fa[-1])
    za_bins = np.interp(ff[band], fa, za.imag)
    rel = np.abs(z[band].imag - za_bins) / np.abs(za_bins)
    near = np.argmin(np.abs(ff - cfg["f0"]))
    print(json.dumps({"grid": [dv.nx, dv.ny, dv.nz], "steps": nt, "seconds": round(sec, 3),
                      "gcell_updates_per_s": round(dv.nx * dv.ny * dv.nz * nt / sec / 1e9, 2),
                      "source_condition": cfg["source_condition"], "f0_bin_thz": float(ff[near] / 1e12),
                      "im_z_sim_at_f0_ohm": float(z[near].imag),
                      "im_z_slab_at_f0_ohm": float(np.interp(ff[near], fa, za.imag)),
                      "median_rel_dev_in_band": float(np.median(rel))}), flush=True)


if __name__ == "__main__":
    main()
