"""Simulation setup that accepts the reference's user dictionaries.

The reference derives everything from ``user_config.py`` (pickled to
``user_dict[_<line>].pkl``) in ``fdtd_auto_setup.py`` and the array section of
``fdtd_main.py``.  This module turns the same dictionary and the same
``<line> <f|b> <i|r>`` run selector into a :class:`~oidt_b200.spec.SimSpec`
(the engine's job description), reproducing the reference's numbers
exactly: scalars keep the reference's NumPy dtypes (``dx`` and ``dt`` are
cast to ``precision`` before any use), so integer grid sizes, coefficient
arrays and twiddle tables come out identical to the reference's.

Reference lines followed:
  setup        FDTD_2D_TM/s-parameter_extraction/fdtd_auto_setup.py:42-170
               FDTD_3D/s-parameter_extraction/fdtd_auto_setup.py:42-177
  geometry     FDTD_2D_TM/s-parameter_extraction/fdtd_funcs.py:165-210
               FDTD_3D/s-parameter_extraction/fdtd_funcs.py:295-369
  coefficients FDTD_2D_TM/s-parameter_extraction/fdtd_main.py:51-178
               FDTD_2D_TE/s-parameter_extraction/fdtd_main.py:51-180
               FDTD_3D/s-parameter_extraction/fdtd_main.py:51-221
  sources      FDTD_2D_TM/.../fdtd_main.py:280-286, FDTD_2D_TE/.../fdtd_main.py:291-297,
               FDTD_3D/.../fdtd_main.py:364-379
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .spec import FIELD_ID, SimSpec

PEC_RIM = 2  # update limits start 2 cells in (fdtd_main.py:113-117)


@dataclass
class Derived:
    """Quantities ``fdtd_auto_setup.py`` exposes as module globals."""
    usr: dict
    mode: str
    kind: str
    sparam_freqs: np.ndarray
    eps: float
    mu: float
    eta: float
    eps_rel_fg: float
    delta_x: np.floating
    delta_t: np.floating
    nt: int
    nx: int
    ny: int
    nz: int
    nx_swg: int
    ny_swg: int
    nz_swg: int
    pp: int
    bx: int
    by: int
    bz: int
    cx_swg: int
    cy_swg: int
    sx: int
    sz: int
    ph: int
    p1: int
    p2: int
    rstd: float
    racl: float
    j_src: np.ndarray
    profile_upper: str
    profile_lower: str
    extra: dict = field(default_factory=dict)


def conditioned(usr: dict) -> dict:
    """Apply ``auto_condition`` (fdtd_auto_setup.py:42-53)."""
    out = dict(usr)
    if out.get("auto_condition"):
        out.update(f0=0.5 * (out["sparam_fmin"] + out["sparam_fmax"]), harmonics=2.0,
                   points_per_wl=20, num_flights=2.0)
    return out


def waveform(usr: dict, dt, nt0: int):
    """Source time series and the final step count (fdtd_auto_setup.py:121-159).

    The step count grows only for the ramped time-harmonic source: the
    Gaussian and wave-packet branches add ``int(t_peak / nt)``, which is 0.
    """
    f0 = usr["f0"]
    tsp_g = np.sqrt(-2 * np.log(10 ** (usr["gauss_pulse_deg"] / 20))) / (2 * np.pi * f0)
    tpk_g = 9 * tsp_g
    tsp_w = 2 * np.sqrt(np.log(2)) / (usr["wave_packet_bw"] * 2 * np.pi * f0)
    tpk_w = 9 * tsp_w
    kind = usr["source_type"]
    nt = nt0
    if kind == 1:
        nt += int(tpk_g / nt)
    elif kind == 2:
        nt += int(tpk_w / nt)
    elif kind == 3:
        nt += int((tpk_g + tsp_g) / dt)
    else:
        raise ValueError("source_type must be 1 (Gaussian), 2 (wave packet) or 3 (time-harmonic)")
    prec = usr["precision"]
    gp, wp, th, ramp = (np.zeros(nt, dtype=prec) for _ in range(4))
    for n in range(nt):
        t = n * dt
        gp[n] = np.exp(-0.5 * ((t - tpk_g) / tsp_g) ** 2)
        wp[n] = np.exp(-0.5 * ((t - tpk_w) / tsp_w) ** 2) * np.exp(2j * np.pi * f0 * (t - tpk_w)).real
        ramp[n] = ramp[n - 1] + dt * gp[n]
        th[n] = np.exp(2j * np.pi * f0 * (t - tpk_g)).real
    ramp = ramp / np.max(ramp)
    amp = usr["source_amp"]
    if kind == 1:
        return amp * gp, nt
    if kind == 2:
        return amp * wp, nt
    return amp * ramp * th, nt


def derive(usr: dict, mode: str, kind: str = "r") -> Derived:
    """fdtd_auto_setup.py for one run (``kind`` 'i' shortens the guide to
    port1_length + port2_length; the step count does not change)."""
    if mode not in ("tm2", "te2", "yee3d"):
        raise ValueError("mode must be tm2, te2 or yee3d")
    u = conditioned(usr)
    prec = u["precision"]
    freqs = np.linspace(u["sparam_fmin"], u["sparam_fmax"], num=u["sparam_num_freqs"])
    eps = u["eps_rel_bg"] / (36.0e9 * np.pi)  # the reference's eps0 = 1/(36 pi 1e9)
    mu = 4.0e-7 * np.pi
    c_bg = 1 / np.sqrt(eps * mu)
    eta = np.sqrt(mu / eps)
    eps_rel_fg = u["eps_rel_fg"] / u["eps_rel_bg"]
    f_max = u["harmonics"] * u["f0"]
    vp = c_bg / np.sqrt(eps_rel_fg)
    wl = vp / f_max
    wl_clad = c_bg / f_max
    sim_time = u["num_flights"] * (u["sgl_wg_length"] / vp)
    dx_full = wl / u["points_per_wl"]
    dt_full = dx_full / (c_bg * np.sqrt(3 if mode == "yee3d" else 2))  # Courant limit
    dx = dx_full.astype(prec)
    dt = dt_full.astype(prec)
    P = u["num_cpml"]
    length = u["port1_length"] + u["port2_length"] if (u["sim_type"] == "s-param" and kind == "i") \
        else u["sgl_wg_length"]
    nt0 = int(sim_time / dt)
    g = {}
    if mode == "yee3d":
        buf_x = int(u["nx_clad_wl"] * wl_clad / dx)
        buf_y = int(u["ny_clad_wl"] * wl_clad / dx)
        g["nx_swg"] = int(u["sgl_wg_height"] / dx)
        g["ny_swg"] = int(u["sgl_wg_width"] / dx)
        g["nz_swg"] = int(length / dx)
        g["pp"] = int(u["pitch"] / dx)
        g["bx"], g["by"], g["bz"] = P + buf_x, P + buf_y, P + u["buffer_zhat"]
        g["nx"] = 2 * g["bx"] + (u["num_lines"] - 1) * g["pp"] + g["nx_swg"]
        g["ny"] = 2 * g["by"] + g["ny_swg"]
        g["nz"] = 2 * g["bz"] + g["nz_swg"]
        g["sx"] = g["bx"] + g["nx_swg"] // 2
        g["sz"] = g["bz"]
        if buf_x < g["pp"] // 2:
            raise ValueError("Boundary conditions too small for WG pitch setting. Reduce pitch or increase nx_clad_wl")
    else:
        buf_y = int(u["ny_clad_wl"] * wl_clad / dx)
        g["nx_swg"] = int(length / dx)
        g["ny_swg"] = int(u["sgl_wg_height"] / dx)
        g["nz_swg"] = 0
        g["pp"] = int(u["pitch"] / dx)
        g["bx"], g["by"], g["bz"] = P + u["buffer_xhat"], P + buf_y, 0
        g["nx"] = 2 * g["bx"] + g["nx_swg"]
        g["ny"] = 2 * g["by"] + (u["num_lines"] - 1) * g["pp"] + g["ny_swg"]
        g["nz"] = 1
        g["sx"] = g["bx"]
        g["sz"] = 0
        if buf_y < g["pp"] // 2:
            raise ValueError("Boundary conditions too small for WG pitch setting. Reduce pitch or increase ny_clad_wl")
    j_src, nt = waveform(u, dt, nt0)
    if mode == "yee3d":
        p1 = g["sz"] + int(u["port1_length"] / dx)
        p2 = g["sz"] + g["nz_swg"] - int(u["port2_length"] / dx)
        if p2 <= p1:
            raise ValueError("Port settling ranges overlap. Make the WG longer or decrease port settling range!")
    else:
        p1 = g["sx"] + int(u["port1_length"] / dx)
        p2 = g["sx"] + g["nx_swg"] - int(u["port2_length"] / dx)
        if p2 < p1:
            raise ValueError("Port settling ranges overlap. Make the WG longer or decrease port settling range!")
    tag = "_s{}nm_lc{}nm_r{}".format(str(round(u["rough_std"] * 1e9)), str(round(u["rough_acl"] * 1e9)),
                                      u["profile_number"])
    return Derived(usr=u, mode=mode, kind=kind, sparam_freqs=freqs, eps=eps, mu=mu, eta=eta,
                   eps_rel_fg=eps_rel_fg, delta_x=dx, delta_t=dt, nt=nt,
                   nx=g["nx"], ny=g["ny"], nz=g["nz"], nx_swg=g["nx_swg"], ny_swg=g["ny_swg"],
                   nz_swg=g["nz_swg"], pp=g["pp"], bx=g["bx"], by=g["by"], bz=g["bz"],
                   cx_swg=g["nx_swg"] // 2, cy_swg=g["ny_swg"] // 2, sx=g["sx"], sz=g["sz"],
                   ph=int(np.ceil(g["pp"] / 2)), p1=p1, p2=p2, rstd=u["rough_std"] / dx,
                   racl=u["rough_acl"] / dx, j_src=j_src,
                   profile_upper="./{}/profile_upper{}".format(u["prof_dir"], tag),
                   profile_lower="./{}/profile_lower{}".format(u["prof_dir"], tag))


# ---------------------------------------------------------------------------
# Geometry and coefficients
# ---------------------------------------------------------------------------
def _padded(profile, head, tail):
    return np.concatenate([np.zeros(head), np.asarray(profile, dtype=np.float64), np.zeros(tail)])


def core_mask(dv: Derived, upper=None, lower=None) -> np.ndarray:
    """Core (foreground) cells.  Sidewall offsets (cells, float) move the
    guide's faces between the two ports; zeros elsewhere
    (``generate_fg_mask``/``apply_mask``)."""
    u = dv.usr
    n_along = dv.nz if dv.mode == "yee3d" else dv.nx
    n_eff = dv.p2 - dv.p1
    upper = np.zeros(n_eff) if upper is None else upper
    lower = np.zeros(n_eff) if lower is None else lower
    if len(upper) != n_eff or len(lower) != n_eff:
        raise ValueError("roughness profiles must have %d samples (port1..port2)" % n_eff)
    up = _padded(upper, dv.p1, n_along - dv.p2)
    lo = _padded(lower, dv.p1, n_along - dv.p2)
    if dv.mode == "yee3d":
        m = np.zeros((dv.nx, dv.ny, dv.nz), dtype=bool)
        ii = np.arange(dv.nx)[:, None]
        jin = np.zeros(dv.ny, dtype=bool)
        jin[dv.by:dv.by + dv.ny_swg] = True
        for l in range(u["num_lines"]):
            o = l * dv.pp
            face = (ii >= (dv.bx + o + lo[None, :])) & (ii < (dv.bx + o + dv.nx_swg + up[None, :]))  # [nx, nz]
            m |= face[:, None, :] & jin[None, :, None]
        return m
    m = np.zeros((dv.nx, dv.ny), dtype=bool)
    jj = np.arange(dv.ny)[None, :]
    for l in range(u["num_lines"]):
        o = l * dv.pp
        m |= (jj >= (dv.by + o + lo[:, None])) & (jj < (dv.by + o + dv.ny_swg + up[:, None]))
    return m


def staggered_eps(eps_cell: np.ndarray, prec, axes):
    """Per-component permittivity: 2-point average along the component's
    axis on indices >= 1 of every axis, the cell value on the first layer
    (``average_materials``)."""
    out = []
    inner = tuple(slice(1, None) for _ in range(eps_cell.ndim))
    for a in axes:
        e = eps_cell.copy().astype(prec)
        lo = list(inner)
        lo[a] = slice(0, -1)
        e[inner] = 0.5 * (eps_cell[inner] + eps_cell[tuple(lo)])
        out.append(e)
    return out


def cpml_profiles(P, dx, dt, eps, eta, prec, m_grade=4, m_alpha=1, sigma_factor=1.2,
                  alpha_max=0.05, kappa_max=5):
    """Graded CPML sigma/kappa/alpha and the recursion coefficients b, c for
    the E (half-cell) and H (integer) positions (fdtd_main.py:119-168).  The
    defaults are the reference's constants."""
    s_max = sigma_factor * (0.8 * (m_grade + 1) / (eta * dx))
    tab = {k: np.zeros(P, dtype=prec) for k in ("se", "ke", "ae", "be", "ce", "sh", "kh", "ah", "bh", "ch")}
    for d in range(P):
        for pos, (s, k, a, b, c) in ((d + 0.5, ("se", "ke", "ae", "be", "ce")), (d, ("sh", "kh", "ah", "bh", "ch"))):
            tab[s][d] = s_max * (pos / P) ** m_grade
            tab[k][d] = 1 + (kappa_max - 1) * (pos / P) ** m_grade
            tab[a][d] = alpha_max * ((P - pos) / P) ** m_alpha
            tab[b][d] = np.exp(-1 * (tab[s][d] / tab[k][d] + tab[a][d]) * (dt / eps))
            tab[c][d] = tab[s][d] / (tab[s][d] * tab[k][d] + tab[k][d] ** 2 * tab[a][d]) * (tab[b][d] - 1)
    return tab


def kappa_axis(n, lo, hi, P, ke, kh, dx, prec):
    """kappa*dx along one axis: dx in the interior, kappa-graded in both
    slabs (fdtd_main.py:151-178)."""
    e = np.ones(n, dtype=prec) * dx
    h = np.ones(n, dtype=prec) * dx
    for d in range(P):
        e[lo + P - (d + 1)] = ke[d] * dx
        h[lo + P - d] = kh[d] * dx
        e[hi - (d + 1)] = ke[-(d + 1)] * dx
        h[hi - (d + 1)] = kh[-(d + 1)] * dx
    return e, h


def twiddles(freqs, dt, nt):
    """float64 DFT kernels cos/sin(2 pi f n dt) (E) and at (n + 1/2) dt (H),
    evaluated in the reference's operand order (``map_sfft_coeffs``)."""
    f = np.asarray(freqs, dtype=np.float64)[:, None]
    t = np.float64(dt)
    nE = np.arange(nt, dtype=np.float64)[None, :]
    aE = 2 * np.pi * f * (nE + 0.0) * t
    aH = 2 * np.pi * f * (nE + 0.5) * t
    return np.cos(aE), np.sin(aE), np.cos(aH), np.sin(aH)


def source_box(dv: Derived, line: int, direction: str):
    """(field, lo, hi) of the soft source for this run."""
    shift = line * dv.pp
    if dv.mode == "tm2":
        x = dv.sx if direction == "f" else dv.nx - dv.sx - 1
        return "EZ", (x, dv.by + shift + 1, 0), (x + 1, dv.by + shift + dv.ny_swg - 1, 1)
    if dv.mode == "te2":
        x = dv.sx if direction == "f" else dv.nx - dv.sx - 1
        return "HZ", (x, dv.by + shift + 2, 0), (x + 1, dv.by + shift + dv.ny_swg - 2, 1)
    z0, z1 = (dv.sz, dv.sz + 2) if direction == "f" else (dv.nz - dv.sz - 1, dv.nz - dv.sz)
    if dv.usr["source_condition"] == "TE":
        return "EY", (dv.bx + shift + 1, dv.by + 1, z0), (dv.bx + shift + dv.nx_swg - 1, dv.by + dv.ny_swg - 1, z1)
    return "HY", (dv.bx + shift + 2, dv.by + 2, z0), (dv.bx + shift + dv.nx_swg - 2, dv.by + dv.ny_swg - 2, z1)


def build_spec(usr: dict, mode: str, line: int = 0, direction: str = "f", kind: str = "r",
               profiles=None, cpml_overrides=None) -> SimSpec:
    """Job description for one reference run ``fdtd_main.py <line> <direction> <kind>``.

    ``profiles`` = (upper, lower) sidewall offsets in cells, used for rough
    reflected runs (the reference's ``rough_profiles/*.npy``); incident runs
    and ``rough_toggle=False`` use the smooth guide.
    """
    if usr.get("sim_type", "s-param") != "s-param":
        raise ValueError("only sim_type='s-param' is defined by the reference")
    dv = derive(usr, mode, kind)
    u = dv.usr
    prec = u["precision"]
    rough = u["rough_toggle"] and kind != "i" and profiles is not None
    mask = core_mask(dv, *(profiles if rough else (None, None)))
    eps_cell = dv.eps * (dv.eps_rel_fg * mask + 1 * ~mask)
    dt, dx = dv.delta_t, dv.delta_x
    if mode == "tm2":
        cb = {"z": dt / eps_cell.copy().astype(prec)}
    elif mode == "te2":
        ex, ey = staggered_eps(eps_cell, prec, (0, 1))
        cb = {"x": dt / ex, "y": dt / ey}
    else:
        ex, ey, ez = staggered_eps(eps_cell, prec, (0, 1, 2))
        cb = {"x": dt / ex, "y": dt / ey, "z": dt / ez}
    P = u["num_cpml"]
    tab = cpml_profiles(P, dx, dt, dv.eps, dv.eta, prec, **(cpml_overrides or {}))
    shape = (dv.nx, dv.ny, dv.nz) if mode == "yee3d" else (dv.nx, dv.ny)
    lim_lo = [PEC_RIM] * len(shape)
    lim_hi = [n - PEC_RIM for n in shape]
    kdx = {}
    for a, name in enumerate("xyz"[:len(shape)]):
        kdx[name + "e"], kdx[name + "h"] = kappa_axis(shape[a], lim_lo[a], lim_hi[a], P, tab["ke"], tab["kh"], dx, prec)
    fld, slo, shi = source_box(dv, line, direction)
    if mode == "yee3d":
        win_lo, win_hi = (P, P), (dv.nx - P, dv.ny - P)
    else:
        win_lo, win_hi = (0, P), (1, dv.ny - P)
    return SimSpec(
        mode=mode, precision=np.dtype(prec), shape=shape, num_cpml=P,
        lim_lo=tuple(lim_lo), lim_hi=tuple(lim_hi), cb=cb, kdx=kdx,
        be=tab["be"], ce=tab["ce"], bh=tab["bh"], ch=tab["ch"],
        db=dt / dv.mu, dx=dx, src_field=FIELD_ID[fld], src_lo=slo, src_hi=shi, j_src=dv.j_src,
        port_pos=(dv.p1, dv.p2), win_lo=win_lo, win_hi=win_hi,
        freqs=dv.sparam_freqs, twiddles=twiddles(dv.sparam_freqs, dt, dv.nt), nt=dv.nt,
        meta=dict(line=line, direction=direction, kind=kind, derived=dv, core_mask=mask))
