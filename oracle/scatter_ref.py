"""NumPy restatement of the reference's sidewall scattering-loss run (oracle).

TEST INFRASTRUCTURE ONLY -- see ``oracle/__init__.py``.

Follows ``FDTD/GPU/FDTD_3D/scattering_loss``:

* ``fdtd_config.py:17-60``    settings; ``:67-200`` derived values and the
  float32 twiddles ``cosE/sinE/cosH/sinH`` of f0 (``:204-211``)
* ``fdtd_main.py:33-179``     mask, materials, CPML grading, kappa*dx -- the
  same expressions as the S-parameter 3D solver, so ``fdtd_ref.build`` makes
  the state from the equivalent S-parameter settings
* ``fdtd_main.py:339-366``    the time loop: the S-parameter 3D update order
  (``fdtd_ref.step``) followed by four plane DFTs
* ``fdtd_funcs.py:217-241``   ``simul_fft_efield`` / ``simul_fft_hfield``:
  float32 accumulators over i in [P, nx - P), j in [P, ny - P) at the cut
  plane, E 2-point and H 4-point colocation, ``I += x sin``
* ``automated_results_collection.py:59-64``  S, P1, P2, alpha

Run in float32 this reproduces the reference's float32 run (its kernels
executed in order, without fused multiply-adds) bit for bit; the fixtures
``tests/golden/scatter_*.npz`` check that.
"""
from __future__ import annotations

import numpy as np

from . import fdtd_ref

SETTINGS = dict(
    eps_rel_bg=1.5 ** 2, eps_rel_fg=3.5 ** 2, sgl_wg_length=24.0e-6, sgl_wg_width=2.0e-6, sgl_wg_height=0.2e-6,
    port1_length=4.0e-6, port2_length=0.0e-6, rough_std=15.0e-9, rough_acl=700.0e-9, tol_std=10.0, tol_acl=10.0,
    rough_toggle=True, ctype=3, output_dir="Results", profile_number=0, source_type=1, source_amp=5.0,
    wave_packet_bw=0.5, gauss_pulse_deg=-6, f0=194.8e12, source_condition="TE", harmonics=1.000, num_flights=2.0,
    points_per_wl=30, num_cpml=20, buffer_zhat=20, nx_clad_wl=0.75, ny_clad_wl=0.75)


def settings(**over) -> dict:
    return dict(SETTINGS, **over)


def as_sparam_usr(st: dict) -> dict:
    """The S-parameter 3D settings with this run's grid, steps and source."""
    u = dict(st)
    u.update(precision=np.float32, sim_type="s-param", auto_condition=False, num_lines=1, pitch=0.0,
             sparam_fmin=st["f0"], sparam_fmax=st["f0"], sparam_num_freqs=1, prof_dir="rough_profiles")
    return u


def twiddles32(f0, delta_t, nt):
    """fdtd_config.py:204-211: float32 cos/sin of 2 pi f0 (n + 0 | 0.5) dt,
    the product taken with float32 ``delta_t`` last."""
    out = [np.zeros(nt, dtype=np.float32) for _ in range(4)]
    for n in range(nt):
        out[0][n] = np.cos(2 * np.pi * f0 * (n + 0.0) * delta_t, dtype=np.float32)
        out[1][n] = np.sin(2 * np.pi * f0 * (n + 0.0) * delta_t, dtype=np.float32)
        out[2][n] = np.cos(2 * np.pi * f0 * (n + 0.5) * delta_t, dtype=np.float32)
        out[3][n] = np.sin(2 * np.pi * f0 * (n + 0.5) * delta_t, dtype=np.float32)
    return out


def build(st: dict, profiles=None):
    """State of one run; ``profiles`` = (upper, lower) or None (smooth)."""
    u = as_sparam_usr(st)
    if profiles is None:
        u["rough_toggle"] = False
    s = fdtd_ref.build(u, "yee3d", 0, "f", "r", profiles=profiles)
    cfg = s.cfg
    s.cosE32, s.sinE32, s.cosH32, s.sinH32 = twiddles32(st["f0"], cfg.delta_t, cfg.nt)
    nx, ny = s.shape[:2]
    s.planes = {}
    for cut in "12":
        for c in ("EX", "EY", "EZ", "HX", "HY", "HZ"):
            s.planes[c + cut + "r"] = np.zeros((nx, ny), dtype=np.float32)
            s.planes[c + cut + "i"] = np.zeros((nx, ny), dtype=np.float32)
    return s


def dft_e(pl, cut, Ex, Ey, Ez, cos, sin, ib, jb, ie, je, kc):  # fdtd_funcs.py:217-227
    I, J, I1, J1 = slice(ib, ie), slice(jb, je), slice(ib + 1, ie + 1), slice(jb + 1, je + 1)
    x = 0.5 * (Ex[I, J, kc] + Ex[I1, J, kc])
    y = 0.5 * (Ey[I, J, kc] + Ey[I, J1, kc])
    z = 0.5 * (Ez[I, J, kc] + Ez[I, J, kc + 1])
    for c, v in (("EX", x), ("EY", y), ("EZ", z)):
        pl[c + cut + "r"][I, J] = pl[c + cut + "r"][I, J] + v * cos
        pl[c + cut + "i"][I, J] = pl[c + cut + "i"][I, J] + v * sin


def dft_h(pl, cut, Hx, Hy, Hz, cos, sin, ib, jb, ie, je, kc):  # fdtd_funcs.py:230-241
    I, J, I1, J1 = slice(ib, ie), slice(jb, je), slice(ib + 1, ie + 1), slice(jb + 1, je + 1)
    x = 0.25 * (Hx[I, J, kc] + Hx[I, J1, kc] + Hx[I, J, kc + 1] + Hx[I, J1, kc + 1])
    y = 0.25 * (Hy[I, J, kc] + Hy[I1, J, kc] + Hy[I, J, kc + 1] + Hy[I1, J, kc + 1])
    z = 0.25 * (Hz[I, J, kc] + Hz[I1, J, kc] + Hz[I, J1, kc] + Hz[I1, J1, kc])
    for c, v in (("HX", x), ("HY", y), ("HZ", z)):
        pl[c + cut + "r"][I, J] = pl[c + cut + "r"][I, J] + v * cos
        pl[c + cut + "i"][I, J] = pl[c + cut + "i"][I, J] + v * sin


def step(s):
    """One step: fields (S-parameter 3D order), then the four plane DFTs
    in the order of fdtd_main.py:362-365."""
    n = s.n
    fdtd_ref.step(s)
    P = s.P
    nx, ny = s.shape[:2]
    cfg = s.cfg
    for cut, kc in (("1", cfg.p1z), ("2", cfg.p2z)):
        dft_e(s.planes, cut, s.EX, s.EY, s.EZ, s.cosE32[n], s.sinE32[n], P, P, nx - P, ny - P, kc)
    for cut, kc in (("1", cfg.p1z), ("2", cfg.p2z)):
        dft_h(s.planes, cut, s.HX, s.HY, s.HZ, s.cosH32[n], s.sinH32[n], P, P, nx - P, ny - P, kc)


def run(s, nsteps=None):
    nsteps = s.cfg.nt - s.n if nsteps is None else nsteps
    for _ in range(nsteps):
        step(s)
    return s


def complex_planes(s) -> dict:
    """fdtd_main.py:427-447: complex64 R + 1j I, keyed ``ex1`` .. ``hz2``."""
    return {c.lower() + cut: (s.planes[c + cut + "r"] + 1j * s.planes[c + cut + "i"]).astype(np.complex64)
            for cut in "12" for c in ("EX", "EY", "EZ", "HX", "HY", "HZ")}


def alpha(planes: dict, delta_x, ell) -> float:
    """automated_results_collection.py:59-64."""
    s1 = 0.5 * (planes["ex1"] * np.conjugate(planes["hy1"]) - planes["ey1"] * np.conjugate(planes["hx1"])).real
    s2 = 0.5 * (planes["ex2"] * np.conjugate(planes["hy2"]) - planes["ey2"] * np.conjugate(planes["hx2"])).real
    p1 = s1.sum() * delta_x * delta_x
    p2 = s2.sum() * delta_x * delta_x
    return np.log(p1 / p2) / ell
