"""NumPy restatement of the reference's wave-impedance run (oracle).

TEST INFRASTRUCTURE ONLY -- see ``oracle/__init__.py``.

Follows ``FDTD/GPU/FDTD_3D/wave_impedance``:

* ``fdtd_config.py``          settings (the scattering-loss settings module
  with other defaults) and ``cy = ny // 2``, ``cz = nz // 2``
* ``fdtd_main.py:264-299``    the S-parameter 3D update order
  (``fdtd_ref.step``), then the line recording of step n
* ``fdtd_funcs.py``           ``map_efield_zwave`` / ``map_hfield_zwave``:
  for i < ie, Eyz[n, i] = 0.5 (Ey[i, cy, cz] + Ey[i, cy + 1, cz]),
  Ezz = 0.5 (Ez[i, cy, cz] + Ez[i, cy, cz + 1]), Hyz and Hzz the 4-point
  averages over (i, i + 1) x (cz, cz + 1) and (i, i + 1) x (cy, cy + 1)
* ``zwave.py:17-57``          the FFT ratio and the slab formula

In float32 this reproduces the reference's float32 records bit for bit
(``tests/golden/zwave_*.npz``).
"""
from __future__ import annotations

import numpy as np

from . import fdtd_ref
from .scatter_ref import as_sparam_usr

SETTINGS = dict(
    eps_rel_bg=1.5 ** 2, eps_rel_fg=3.5 ** 2, sgl_wg_length=14.0e-6, sgl_wg_width=2.0e-6, sgl_wg_height=0.2e-6,
    port1_length=4.0e-6, port2_length=0.0e-6, rough_std=15.0e-9, rough_acl=700.0e-9, tol_std=10.0, tol_acl=10.0,
    rough_toggle=False, ctype=3, output_dir="Results", profile_number=0, source_type=1, source_amp=5.0,
    wave_packet_bw=0.5, gauss_pulse_deg=-6, f0=194.8e12, source_condition="TM", harmonics=1.000, num_flights=2.0,
    points_per_wl=40, num_cpml=20, buffer_zhat=20, nx_clad_wl=0.75, ny_clad_wl=0.75)


def settings(**over) -> dict:
    return dict(SETTINGS, **over)


def build(st: dict):
    u = as_sparam_usr(st)
    u["rough_toggle"] = False
    s = fdtd_ref.build(u, "yee3d", 0, "f", "r")
    nt, nx = s.cfg.nt, s.shape[0]
    s.cy, s.cz = s.shape[1] // 2, s.shape[2] // 2
    s.rec = {k: np.zeros((nt, nx), dtype=s.prec) for k in ("EY_ZW", "EZ_ZW", "HY_ZW", "HZ_ZW")}
    return s


def record(s, n):
    I, I1 = slice(0, s.ie), slice(1, s.ie + 1)
    cy, cz = s.cy, s.cz
    s.rec["EY_ZW"][n, I] = 0.5 * (s.EY[I, cy, cz] + s.EY[I, cy + 1, cz])
    s.rec["EZ_ZW"][n, I] = 0.5 * (s.EZ[I, cy, cz] + s.EZ[I, cy, cz + 1])
    s.rec["HY_ZW"][n, I] = 0.25 * (s.HY[I, cy, cz] + s.HY[I1, cy, cz] + s.HY[I, cy, cz + 1] + s.HY[I1, cy, cz + 1])
    s.rec["HZ_ZW"][n, I] = 0.25 * (s.HZ[I, cy, cz] + s.HZ[I1, cy, cz] + s.HZ[I, cy + 1, cz] + s.HZ[I1, cy + 1, cz])


def run(s, nsteps=None):
    nsteps = s.cfg.nt - s.n if nsteps is None else nsteps
    for _ in range(nsteps):
        n = s.n
        fdtd_ref.step(s)
        record(s, n)
    return s


def impedance(s, cell=3):
    """zwave.py:19-34 at x = bx - cell."""
    x = s.cfg.bx - cell
    if s.usr["source_condition"] == "TE":
        z = np.fft.fft(s.rec["EY_ZW"][:, x]) / np.fft.fft(s.rec["HZ_ZW"][:, x])
    else:
        z = -1 * np.fft.fft(s.rec["EZ_ZW"][:, x]) / np.fft.fft(s.rec["HY_ZW"][:, x])
    return np.arange(0, s.cfg.nt, 1) / (s.cfg.delta_t * s.cfg.nt), z
