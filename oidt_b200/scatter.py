"""Sidewall scattering loss of a rough guide: one 3D run per realization,
a one-frequency DFT of the whole cross-section at two cuts along the guide,
and the loss alpha = ln(P1 / P2) / L from the Poynting power through them.

Reference: ``FDTD/GPU/FDTD_3D/scattering_loss``
  fdtd_config.py:17-60            settings (``REFERENCE_CONFIG`` below)
  fdtd_config.py:67-200           derived grid, steps, source, cut planes
  fdtd_main.py:33-46, 75-179      mask, materials, CPML grading, kappa*dx
  fdtd_main.py:339-366            time loop (the S-parameter 3D launch order)
  fdtd_funcs.py:217-241           plane DFTs (E 2-point, H 4-point colocation)
  automated_results_collection.py:59-64   S, P1, P2, alpha
  analysis.py:38-111, aux_funcs.py:17-36  Payne-Lacey slab estimate

The solver's update kernels, source boxes, cut planes, DFT window and
colocation are those of the S-parameter 3D solver
(``FDTD_3D/s-parameter_extraction``), so a scattering run is an engine job
built by :func:`oidt_b200.refsetup.build_spec` from the equivalent
settings with one frequency (f0).  Differences from the reference kept or
changed on purpose:

* the reference accumulates the plane DFTs in float32 with float32
  twiddles; the engine accumulates in float64 (float64 twiddles).  Planes
  are returned in the reference's convention (``I = +sum x sin``, the
  opposite of the S-parameter kernels), i.e. the complex conjugate of the
  engine's accumulators, as complex64 arrays [nx, ny] zero outside the DFT
  window;
* only Ex, Ey, Hx, Hy planes are produced: the reference also accumulates Ez
  and Hz, which its loss extraction never reads;
* sidewall profiles come from the caller (or the project's seeded
  exponential-ACF generator); the reference draws them with pyspeckle.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import refsetup
from .spec import SimSpec

# fdtd_config.py:17-60 (the settings a user edits)
REFERENCE_CONFIG = dict(
    eps_rel_bg=1.5 ** 2, eps_rel_fg=3.5 ** 2, sgl_wg_length=24.0e-6, sgl_wg_width=2.0e-6, sgl_wg_height=0.2e-6,
    port1_length=4.0e-6, port2_length=0.0e-6, rough_std=15.0e-9, rough_acl=700.0e-9, tol_std=10.0, tol_acl=10.0,
    rough_toggle=True, ctype=3, output_dir="Results", profile_number=0, source_type=1, source_amp=5.0,
    wave_packet_bw=0.5, gauss_pulse_deg=-6, f0=194.8e12, source_condition="TE", harmonics=1.000, num_flights=2.0,
    points_per_wl=30, num_cpml=20, buffer_zhat=20, nx_clad_wl=0.75, ny_clad_wl=0.75)

PLANE_COMPS = ("ex", "ey", "hx", "hy")  # engine DFT component order


def config(**overrides) -> dict:
    """The reference's settings with ``overrides`` applied."""
    unknown = set(overrides) - set(REFERENCE_CONFIG)
    if unknown:
        raise KeyError("unknown scattering-loss settings: %s" % sorted(unknown))
    return dict(REFERENCE_CONFIG, **overrides)


def usr_of(cfg: dict) -> dict:
    """The S-parameter setup keys that reproduce this configuration's grid,
    steps, source and cut planes (one guide, one frequency f0, float32)."""
    u = {k: cfg[k] for k in ("eps_rel_bg", "eps_rel_fg", "sgl_wg_length", "sgl_wg_width", "sgl_wg_height",
                             "port1_length", "port2_length", "rough_std", "rough_acl", "rough_toggle",
                             "profile_number", "source_type", "source_amp", "wave_packet_bw", "gauss_pulse_deg",
                             "f0", "source_condition", "harmonics", "num_flights", "points_per_wl", "num_cpml",
                             "buffer_zhat", "nx_clad_wl", "ny_clad_wl")}
    u.update(precision=np.float32, sim_type="s-param", auto_condition=False, num_lines=1, pitch=0.0,
             sparam_fmin=cfg["f0"], sparam_fmax=cfg["f0"], sparam_num_freqs=1, prof_dir="rough_profiles",
             output_dir=cfg["output_dir"])
    return u


def derive(cfg: dict) -> refsetup.Derived:
    """fdtd_config.py:67-200 (grid, steps, source, cut planes p1z / p2z);
    ``extra['n_eff']`` = sidewall profile length (cells between the cuts)."""
    dv = refsetup.derive(usr_of(cfg), "yee3d", "r")
    dv.extra["n_eff"] = dv.p2 - dv.p1
    dv.extra["ell"] = (dv.p2 - dv.p1) * dv.delta_x  # automated_results_collection.py:33
    return dv


def n_eff(cfg: dict) -> int:
    return derive(cfg).extra["n_eff"]


def build_spec(cfg: dict, profiles=None) -> SimSpec:
    """Engine job of one realization.  ``profiles`` = (upper, lower) sidewall
    offsets in cells over the ``n_eff`` cells between the cuts (None: the
    smooth guide)."""
    u = usr_of(cfg)
    if profiles is None:
        u["rough_toggle"] = False
    spec = refsetup.build_spec(u, "yee3d", 0, "f", "r", profiles=profiles)
    dv = spec.meta["derived"]
    spec.meta.update(workload="scattering_loss", ell=(dv.p2 - dv.p1) * dv.delta_x)
    return spec


def planes_from_dft(spec: SimSpec, dft: dict) -> dict:
    """Reference-convention planes {'ex1', 'ey1', 'hx1', 'hy1', 'ex2', ...}:
    complex64 [nx, ny], ``R + i I`` with ``I = +sum x sin``
    (fdtd_funcs.py:217-241, fdtd_main.py:427-447).  ``dft`` maps (port, comp
    index) to the engine's complex DFT [1, nx, ny]."""
    out = {}
    for port in (0, 1):
        for c, name in enumerate(PLANE_COMPS):
            out["%s%d" % (name, port + 1)] = np.conjugate(np.asarray(dft[(port, c)])[0]).astype(np.complex64)
    return out


def planes_from_job(job) -> dict:
    return planes_from_dft(job.spec, {(p, c): job.dft(p, c) for p in (0, 1) for c in range(4)})


def power(planes: dict, cut: int, dx) -> float:
    """P = sum over the plane of 1/2 Re(Ex Hy* - Ey Hx*) dx^2
    (automated_results_collection.py:59-62)."""
    ex, ey, hx, hy = (planes["%s%d" % (n, cut)] for n in PLANE_COMPS)
    s = 0.5 * (ex * np.conjugate(hy) - ey * np.conjugate(hx)).real
    return s.sum() * dx * dx


def loss(planes: dict, dx, ell) -> dict:
    """alpha = ln(P1 / P2) / L in Np/m (automated_results_collection.py:59-64)."""
    p1, p2 = power(planes, 1, dx), power(planes, 2, dx)
    return {"alpha": float(np.log(p1 / p2) / ell), "P1": float(p1), "P2": float(p2)}


def save_planes(out_dir: str, tag: str, planes: dict) -> list:
    """``<comp><cut>_fft<tag>.npy`` as the reference names them
    (fdtd_config.py:30-41, fdtd_main.py:448-459)."""
    os.makedirs(out_dir, exist_ok=True)
    paths = []
    for name, arr in planes.items():
        p = os.path.join(out_dir, "%s%s_fft%s.npy" % (name[:2], name[2], tag))
        np.save(p, arr)
        paths.append(p)
    return paths


def profile_tag(cfg: dict) -> str:
    """``_s<sigma nm>nm_lc<Lc nm>nm_r<profile>`` (fdtd_config.py:193-195)."""
    return "_s%snm_lc%snm_r%s" % (str(round(cfg["rough_std"] * 1e9)), str(round(cfg["rough_acl"] * 1e9)),
                                  cfg["profile_number"])


# ---------------------------------------------------------------------------
# Payne-Lacey estimate for a symmetric slab (analysis.py:38-111)
# ---------------------------------------------------------------------------
def find_neff(n1, n2, d, k0, mode="te"):
    """Effective index of the fundamental slab mode from the normalised
    dispersion relation, half-thickness d (aux_funcs.py:17-36)."""
    from scipy.optimize import fsolve

    V = k0 * 2 * d * np.sqrt(n1 ** 2 - n2 ** 2)
    if mode == "te":
        def f(neff):
            b = (neff ** 2 - n2 ** 2) / (n1 ** 2 - n2 ** 2)
            return 2 * np.arctan(np.sqrt(b / (1 - b))) - V * np.sqrt(1 - b)
    elif mode == "tm":
        def f(neff):
            qs = neff ** 2 / n1 ** 2 + neff ** 2 / n2 ** 2 - 1
            b = n1 ** 2 * (neff ** 2 - n2 ** 2) / (n2 ** 2 * qs * (n1 ** 2 - n2 ** 2))
            return 2 * np.arctan(np.sqrt(b / (1 - b))) - V * (n1 / n2) * np.sqrt(qs * (1 - b))
    else:
        raise ValueError("mode must be 'te' or 'tm'")
    return float(fsolve(f, x0=n2)[0])


def _radiation_integral(beta, n2, k0, sigma, lc):
    theta = np.linspace(0, np.pi, num=3142)
    k = beta - n2 * k0 * np.cos(theta)
    rxx = 2 * lc * sigma ** 2 / (1 + lc ** 2 * k ** 2)  # exponential-ACF spectral density
    return float(np.sum(rxx) * theta[1])


def alpha_te(sigma, lc, f0, n1=3.5, n2=1.5, d=100e-9):
    """TE slab estimate (analysis.py:38-57): (n2/n1, n2/neff) normalisations."""
    k0 = 2 * np.pi * f0 / 3e8
    neff = find_neff(n1, n2, d, k0, mode="te")
    beta = neff * k0
    kappa = np.sqrt((n1 * k0) ** 2 - beta ** 2)
    gamma = np.sqrt(beta ** 2 - (n2 * k0) ** 2)
    mw = (n1 ** 2 - n2 ** 2) ** 2 * k0 ** 3 / (4 * np.pi * n2)
    prad = np.cos(kappa * d) ** 2 * mw * _radiation_integral(beta, n2, k0, sigma, lc)
    base = prad / (d + 1 / gamma)
    return n2 / n1 * base, n2 / neff * base


def alpha_tm(sigma, lc, f0, n1, n2, d=100e-9):
    """TM slab estimate (analysis.py:60-111): four guided-power normalisations
    (Lacey-Payne, piecewise, access, effective impedance)."""
    eta0 = 120 * np.pi
    k0 = 2 * np.pi * f0 / 3e8
    neff = find_neff(n1, n2, d, k0, mode="tm")
    beta = neff * k0
    kappa = np.sqrt((n1 * k0) ** 2 - beta ** 2)
    gamma = np.sqrt(beta ** 2 - (n2 * k0) ** 2)
    mw = (n1 ** 2 - n2 ** 2) ** 2 * k0 ** 3 / (4 * np.pi * n2)
    prad = 0.5 * eta0 / n2 * np.cos(kappa * d) ** 2 * mw * _radiation_integral(beta, n2, k0, sigma, lc)
    F = n2 ** 2 / (n1 ** 4 * gamma ** 2 + n2 ** 4 * kappa ** 2)
    core, clad = d + n1 ** 2 * F * gamma, n2 ** 2 * kappa ** 2 * F / gamma

    def deff(scale, na, nb):
        return scale * (core / na + clad / nb)

    pg = (0.5 * eta0 / n1 * deff(n1, n1, n1), 0.5 * eta0 / n1 * deff(n1, n1, n2),
          0.5 * (neff * eta0 / n1 ** 2) * deff(n1 ** 2 / neff, n1 ** 2 / neff, n2 ** 2 / neff),
          0.5 * eta0 / neff * deff(neff, neff, neff))
    return tuple(prad / g for g in pg)


def analytic_alpha(cfg: dict):
    """The estimate the reference compares against for this configuration:
    TE from the hard-coded n = 3.5 / 1.5 slab, TM from the configured
    permittivities (analysis.py:38-45, 60-66)."""
    if cfg["source_condition"] == "TE":
        return alpha_te(cfg["rough_std"], cfg["rough_acl"], cfg["f0"])
    return alpha_tm(cfg["rough_std"], cfg["rough_acl"], cfg["f0"], np.sqrt(cfg["eps_rel_fg"]),
                    np.sqrt(cfg["eps_rel_bg"]))


# ---------------------------------------------------------------------------
# Runs
# ---------------------------------------------------------------------------
def realization_profiles(cfg: dict, n: int, master_seed=0):
    """``n`` (upper, lower) profile pairs of the configured sigma and Lc,
    drawn by the project's seeded exponential-ACF generator."""
    from .workloads import sidewall_profile
    dv = derive(cfg)
    ne = dv.extra["n_eff"]
    s_cells, lc_cells = cfg["rough_std"] / float(dv.delta_x), cfg["rough_acl"] / float(dv.delta_x)
    out = []
    for r in range(n):
        rng = np.random.default_rng([master_seed, r])
        out.append((sidewall_profile(ne, s_cells, lc_cells, rng), sidewall_profile(ne, s_cells, lc_cells, rng)))
    return out


def _finish(job) -> dict:
    pl = planes_from_job(job)
    r = loss(pl, job.spec.dx, job.spec.meta["ell"])
    r["planes"] = pl
    job.release()
    return r


def run(eng, cfg: dict, profile_sets, batched=True, precision=np.float32, arith="fast"):
    """Loss of every realization.  ``batched``: the jobs advance together in
    multi-job launches, in consecutive groups whose device memory fits the
    context's free budget; otherwise one job at a time.  Returns (seconds,
    [dict(alpha, P1, P2, planes)]) in the order of ``profile_sets``."""
    from .simulation_launcher import batch_groups
    specs = [build_spec(cfg, p) for p in profile_sets]
    t0 = time.perf_counter()
    res = []
    if batched:
        st = eng.stats()
        sizes = [eng.job_bytes(s, precision=precision) for s in specs]
        for g in batch_groups(sizes, st["hbm_budget"] - st["hbm_in_use"]):
            jobs = [eng.submit(specs[i], arith=arith, precision=precision) for i in g]
            steps = min(j.spec.nt for j in jobs)
            eng.batch_advance(jobs, steps)
            for j in jobs:
                if j.spec.nt > steps:
                    j.advance(j.spec.nt - steps)
            for j in jobs:
                j.sync()
            res.extend(_finish(j) for j in jobs)
    else:
        for s in specs:
            j = eng.submit(s, arith=arith, precision=precision, graphs=False)
            j.run().sync()
            res.append(_finish(j))
    return time.perf_counter() - t0, res


def main(argv=None):
    ap = argparse.ArgumentParser(description="Sidewall scattering loss, one or more rough realizations")
    ap.add_argument("--set", nargs="*", default=[], help="setting=value overrides of the reference config")
    ap.add_argument("--realizations", type=int, default=1)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--plain", action="store_true", help="one job at a time instead of batched launches")
    ap.add_argument("--out", default=None, help="directory for the reference-named plane files")
    a = ap.parse_args(argv)
    over = {}
    for kv in a.set:
        k, v = kv.split("=", 1)
        over[k] = json.loads(v) if v[:1] in "0123456789-[{tf\"" else v
    cfg = config(**over)
    from .engine import Engine
    eng = Engine(0)
    dv = derive(cfg)
    profs = realization_profiles(cfg, a.realizations, a.seed)
    sec, res = run(eng, cfg, profs, batched=not a.plain)
    eng.close()
    if a.out:
        for r in range(len(profs)):
            save_planes(a.out, profile_tag(dict(cfg, profile_number=r)), res[r]["planes"])
    alphas = np.array([r["alpha"] for r in res])
    cells = dv.nx * dv.ny * dv.nz
    print(json.dumps({"grid": [dv.nx, dv.ny, dv.nz], "steps": dv.nt, "realizations": a.realizations,
                      "seconds": round(sec, 3), "realizations_per_s": round(a.realizations / sec, 4),
                      "gcell_updates_per_s": round(cells * dv.nt * a.realizations / sec / 1e9, 2),
                      "alpha_mean_np_per_m": float(alphas.mean()), "alpha_std_np_per_m": float(alphas.std()),
                      "alpha_estimate_np_per_m": [float(x) for x in analytic_alpha(cfg)]}), flush=True)


if __name__ == "__main__":
    main()
