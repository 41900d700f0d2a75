"""Float64 NumPy restatement of the reference FDTD S-parameter path (oracle).

TEST INFRASTRUCTURE ONLY -- see ``oracle/__init__.py``.  Every function names
the reference lines it restates.  Expressions keep the reference's operand
order (``a + (b * c) / d`` stays exactly that) so that a float64 run
reproduces the reference's float64 run bit for bit; the golden fixtures made
by ``tests/golden/make_golden.py`` check this.

Three solvers share this module, named by the reference directory they
follow:

* ``tm2``   -- ``FDTD/GPU/FDTD_2D_TM/s-parameter_extraction`` (Ez, Hx, Hy)
* ``te2``   -- ``FDTD/GPU/FDTD_2D_TE/s-parameter_extraction`` (Ex, Ey, Hz)
* ``yee3d`` -- ``FDTD/GPU/FDTD_3D/s-parameter_extraction`` (all six)

Arrays use the reference layout: 2D ``[nx, ny]``, 3D ``[nx, ny, nz]``,
C order.
"""
from __future__ import annotations

import math
from types import SimpleNamespace

import numpy as np

MODES = ("tm2", "te2", "yee3d")
OFFSET = 2  # PEC rim width: ib = jb = kb = 2 (TM2/fdtd_main.py:113-117)


# ---------------------------------------------------------------------------
# Setup: fdtd_auto_setup.py
# ---------------------------------------------------------------------------
def condition(usr: dict) -> dict:
    """``auto_condition`` overrides (TM2/fdtd_auto_setup.py:42-53)."""
    usr = dict(usr)
    if usr["auto_condition"]:
        usr["f0"] = 0.5 * (usr["sparam_fmin"] + usr["sparam_fmax"])
        usr["harmonics"] = 2.0
        usr["points_per_wl"] = 20
        usr["num_flights"] = 2.0
    return usr


def autosetup(usr: dict, mode: str, kind: str = "r") -> SimpleNamespace:
    """Derived simulation constants.

    2D: ``FDTD_2D_TM/s-parameter_extraction/fdtd_auto_setup.py:59-170`` (TE
    identical); 3D: ``FDTD_3D/s-parameter_extraction/fdtd_auto_setup.py:59-177``.
    Scalar dtypes follow the reference expressions (``dx``/``dt`` are cast to
    ``precision`` before any use, ``fdtd_auto_setup.py:76-77``).
    """
    usr = condition(usr)
    prec = usr["precision"]
    c = SimpleNamespace()
    c.usr = usr
    c.sparam_freqs = np.linspace(usr["sparam_fmin"], usr["sparam_fmax"], num=usr["sparam_num_freqs"])
    c.eps = usr["eps_rel_bg"] / (36.0e9 * np.pi)
    c.mu = 4.0e-7 * np.pi
    c.c_bg = 1 / np.sqrt(c.eps * c.mu)
    c.eta = np.sqrt(c.mu / c.eps)
    c.eps_rel_fg = usr["eps_rel_fg"] / usr["eps_rel_bg"]
    f_max = usr["harmonics"] * usr["f0"]
    vp = c.c_bg / np.sqrt(c.eps_rel_fg)
    wl = vp / f_max
    wl_clad = c.c_bg / f_max
    flight_time = usr["sgl_wg_length"] / vp
    sim_time = usr["num_flights"] * flight_time
    delta_x = wl / usr["points_per_wl"]
    root = np.sqrt(3) if mode == "yee3d" else np.sqrt(2)
    delta_t = delta_x / (c.c_bg * root)
    c.delta_x = delta_x.astype(prec)
    c.delta_t = delta_t.astype(prec)
    dx = c.delta_x
    P = usr["num_cpml"]

    wg_length = usr["sgl_wg_length"]
    if usr["sim_type"] == "s-param" and kind == "i":
        wg_length = usr["port1_length"] + usr["port2_length"]

    c.nt = int(sim_time / c.delta_t)
    if mode == "yee3d":
        # FDTD_3D/.../fdtd_auto_setup.py:79-122
        buffer_xhat = int(usr["nx_clad_wl"] * wl_clad / dx)
        buffer_yhat = int(usr["ny_clad_wl"] * wl_clad / dx)
        c.nx_swg = int(usr["sgl_wg_height"] / dx)
        c.ny_swg = int(usr["sgl_wg_width"] / dx)
        c.nz_swg = int(wg_length / dx)
        c.pp = int(usr["pitch"] / dx)
        c.bx = P + buffer_xhat
        c.by = P + buffer_yhat
        c.bz = P + usr["buffer_zhat"]
        c.nx = 2 * c.bx + (usr["num_lines"] - 1) * c.pp + c.nx_swg
        c.ny = 2 * c.by + c.ny_swg
        c.nz = 2 * c.bz + c.nz_swg
        c.cx_swg = c.nx_swg // 2
        c.cy_swg = c.ny_swg // 2
        c.sx = c.bx + c.cx_swg
        c.sy = c.by + c.cy_swg
        c.sz = c.bz + 0
        c.ph = int(np.ceil(c.pp / 2))
        if buffer_xhat < c.pp // 2:
            raise Exception("Boundary conditions too small for WG pitch setting. Reduce pitch or increase nx_clad_wl")
    else:
        # FDTD_2D_TM/.../fdtd_auto_setup.py:79-115
        buffer_yhat = int(usr["ny_clad_wl"] * wl_clad / dx)
        c.nx_swg = int(wg_length / dx)
        c.ny_swg = int(usr["sgl_wg_height"] / dx)
        c.pp = int(usr["pitch"] / dx)
        c.bx = P + usr["buffer_xhat"]
        c.by = P + buffer_yhat
        c.nx = 2 * c.bx + c.nx_swg
        c.ny = 2 * c.by + (usr["num_lines"] - 1) * c.pp + c.ny_swg
        c.cx_swg = c.nx_swg // 2
        c.cy_swg = c.ny_swg // 2
        c.sx = c.bx + 0
        c.sy = c.by + c.cy_swg
        c.ph = int(np.ceil(c.pp / 2))
        if buffer_yhat < c.pp // 2:
            raise Exception("Boundary conditions too small for WG pitch setting. Reduce pitch or increase ny_clad_wl")
    c.rstd = usr["rough_std"] / dx
    c.racl = usr["rough_acl"] / dx
    c.tol_std = usr["tol_std"] / 100
    c.tol_acl = usr["tol_acl"] / 100

    # Source waveforms (fdtd_auto_setup.py:121-159).
    gp_tsp = np.sqrt(-2 * np.log(10 ** (usr["gauss_pulse_deg"] / 20))) / (2 * np.pi * usr["f0"])
    gp_tpk = 9 * gp_tsp
    wp_tsp = 2 * np.sqrt(np.log(2)) / (usr["wave_packet_bw"] * 2 * np.pi * usr["f0"])
    wp_tpk = 9 * wp_tsp
    nt = c.nt
    st = usr["source_type"]
    if st == 1:
        nt += int(gp_tpk / nt)  # adds 0: the reference divides by nt, not dt
    elif st == 2:
        nt += int(wp_tpk / nt)
    elif st == 3:
        nt += int((gp_tpk + gp_tsp) / c.delta_t)
    else:
        raise Exception("Pick a valid source type")
    c.nt = nt
    GP = np.zeros(nt, dtype=prec)
    WP = np.zeros(nt, dtype=prec)
    TH = np.zeros(nt, dtype=prec)
    RAMP = np.zeros(nt, dtype=prec)
    dt = c.delta_t
    for n in range(nt):
        GP[n] = np.exp(-0.5 * ((n * dt - gp_tpk) / gp_tsp) ** 2)
        WP[n] = np.exp(-0.5 * ((n * dt - wp_tpk) / wp_tsp) ** 2) * np.exp(2j * np.pi * usr["f0"] * (n * dt - wp_tpk)).real
        RAMP[n] = RAMP[n - 1] + dt * GP[n]
        TH[n] = np.exp(2j * np.pi * usr["f0"] * (n * dt - gp_tpk)).real
    RAMP = RAMP / np.max(RAMP)
    if st == 1:
        c.J_SRC = usr["source_amp"] * GP
    elif st == 2:
        c.J_SRC = usr["source_amp"] * WP
    else:
        c.J_SRC = usr["source_amp"] * RAMP * TH

    if mode == "yee3d":
        c.p1z = c.sz + int(usr["port1_length"] / dx)
        c.p2z = c.sz + c.nz_swg - int(usr["port2_length"] / dx)
        if c.p2z <= c.p1z:
            raise Exception("Port settling ranges overlap. Make the WG longer or decrease port settling range!")
    else:
        c.p1x = c.sx + int(usr["port1_length"] / dx)
        c.p2x = c.sx + c.nx_swg - int(usr["port2_length"] / dx)
        if c.p2x < c.p1x:
            raise Exception("Port settling ranges overlap. Make the WG longer or decrease port settling range!")
    profile_std = str(round(usr["rough_std"] * 1e9))
    profile_acl = str(round(usr["rough_acl"] * 1e9))
    rp = "_s{}nm_lc{}nm_r{}".format(profile_std, profile_acl, usr["profile_number"])
    c.up = "./{}/profile_upper{}".format(usr["prof_dir"], rp)
    c.lp = "./{}/profile_lower{}".format(usr["prof_dir"], rp)
    return c


# ---------------------------------------------------------------------------
# Geometry (fdtd_funcs.py generate_fg_mask / apply_mask / average_materials)
# ---------------------------------------------------------------------------
def fg_mask_2d(nx, ny, bord_y, wg_height, pitch, num_lines, settling, end, upper, lower):
    """``apply_mask`` (TM2/fdtd_funcs.py:165-210): profiles padded with zeros
    over the settling ranges, cell (i, j) is core when
    ``by + l*pitch + lower[i] <= j < by + l*pitch + h + upper[i]``."""
    up = np.append(np.append(np.zeros(settling), upper), np.zeros(end))
    lo = np.append(np.append(np.zeros(settling), lower), np.zeros(end))
    mask = np.zeros([nx, ny], dtype=bool)
    j = np.arange(ny)[None, :]
    for l in range(num_lines):
        off = l * pitch
        mask |= (j >= (bord_y + off + lo[:, None])) & (j < (bord_y + off + wg_height + up[:, None]))
    return mask


def fg_mask_3d(nx, ny, nz, bord_x, bord_y, wg_height, wg_width, pitch, num_lines, settling, end, upper, lower):
    """``apply_mask`` (FDTD_3D/.../fdtd_funcs.py:323-369): roughness moves the
    x-faces of the core along z."""
    up = np.append(np.append(np.zeros(settling), upper), np.zeros(end))
    lo = np.append(np.append(np.zeros(settling), lower), np.zeros(end))
    mask = np.zeros([nx, ny, nz], dtype=bool)
    i = np.arange(nx)[:, None, None]
    j = np.arange(ny)[None, :, None]
    jin = (j >= bord_y) & (j < bord_y + wg_width)
    for l in range(num_lines):
        off = l * pitch
        mask |= jin & (i >= (bord_x + off + lo[None, None, :])) & (i < (bord_x + off + wg_height + up[None, None, :]))
    return mask


def average_materials_2d(mask_eps, X, Y):
    """TE2/fdtd_funcs.py ``average_materials``: 2-point averages on i, j >= 1."""
    X[1:, 1:] = 0.5 * (mask_eps[1:, 1:] + mask_eps[:-1, 1:])
    Y[1:, 1:] = 0.5 * (mask_eps[1:, 1:] + mask_eps[1:, :-1])


def average_materials_3d(mask_eps, X, Y, Z):
    """FDTD_3D/.../fdtd_funcs.py:295-302."""
    X[1:, 1:, 1:] = 0.5 * (mask_eps[1:, 1:, 1:] + mask_eps[:-1, 1:, 1:])
    Y[1:, 1:, 1:] = 0.5 * (mask_eps[1:, 1:, 1:] + mask_eps[1:, :-1, 1:])
    Z[1:, 1:, 1:] = 0.5 * (mask_eps[1:, 1:, 1:] + mask_eps[1:, 1:, :-1])


def sfft_coeffs(freqs, dt, nt, prec):
    """``map_sfft_coeffs`` (TM2/fdtd_funcs.py:230-237): E twiddles at n*dt,
    H twiddles at (n+1/2)*dt, evaluated in float64 and stored in ``prec``."""
    f = np.asarray(freqs, dtype=np.float64)[:, None]
    dtf = np.float64(dt)
    n = np.arange(nt, dtype=np.float64)[None, :]
    argE = 2 * np.pi * f * (n + 0.0) * dtf
    argH = 2 * np.pi * f * (n + 0.5) * dtf
    return (np.cos(argE).astype(prec), np.sin(argE).astype(prec),
            np.cos(argH).astype(prec), np.sin(argH).astype(prec))


def cpml_grading(P, delta_x, delta_t, eps, eta, prec, m_grade=4, m_alpha=1,
                 sigma_factor=1.2, alpha_max=0.05, kappa_max=5):
    """CPML grading (TM2/fdtd_main.py:119-168)."""
    sigma_opt = 0.8 * (m_grade + 1) / (eta * delta_x)
    sigma_max = sigma_factor * sigma_opt
    g = {k: np.zeros(P, dtype=prec) for k in ("SE", "KE", "AE", "BE", "CE", "SH", "KH", "AH", "BH", "CH")}
    SE, KE, AE, BE, CE = g["SE"], g["KE"], g["AE"], g["BE"], g["CE"]
    SH, KH, AH, BH, CH = g["SH"], g["KH"], g["AH"], g["BH"], g["CH"]
    for d in range(P):
        SE[d] = sigma_max * ((d + 0.5) / P) ** m_grade
        KE[d] = 1 + (kappa_max - 1) * ((d + 0.5) / P) ** m_grade
        AE[d] = alpha_max * ((P - (d + 0.5)) / P) ** m_alpha
        BE[d] = np.exp(-1 * (SE[d] / KE[d] + AE[d]) * (delta_t / eps))
        CE[d] = SE[d] / (SE[d] * KE[d] + KE[d] ** 2 * AE[d]) * (BE[d] - 1)
        SH[d] = sigma_max * (d / P) ** m_grade
        KH[d] = 1 + (kappa_max - 1) * (d / P) ** m_grade
        AH[d] = alpha_max * ((P - d) / P) ** m_alpha
        BH[d] = np.exp(-1 * (SH[d] / KH[d] + AH[d]) * (delta_t / eps))
        CH[d] = SH[d] / (SH[d] * KH[d] + KH[d] ** 2 * AH[d]) * (BH[d] - 1)
    return g


def kappa_dx(n, b, e, P, KE, KH, delta_x, prec):
    """kappa*dx divisor arrays along one axis (TM2/fdtd_main.py:151-178)."""
    ke = np.ones(n, dtype=prec) * delta_x
    kh = np.ones(n, dtype=prec) * delta_x
    for d in range(P):
        ke[b + P - (d + 1)] = KE[d] * delta_x
        kh[b + P - d] = KH[d] * delta_x
        ke[e - (d + 1)] = KE[-(d + 1)] * delta_x
        kh[e - (d + 1)] = KH[-(d + 1)] * delta_x
    return ke, kh


# ---------------------------------------------------------------------------
# Simulation state (fdtd_main.py:51-178 / 3D :51-221)
# ---------------------------------------------------------------------------
def build(usr: dict, mode: str, line: int, direction: str, kind: str, profiles=None) -> SimpleNamespace:
    """Allocate and fill every array the reference copies to the device.

    ``profiles`` = ``(upper, lower)`` sidewall offsets in cells (the
    reference's ``rough_profiles/*.npy`` in ``mode='load'``); ``None`` or an
    incident run gives the smooth guide (TM2/fdtd_main.py:56-81).
    """
    cfg = autosetup(usr, mode, kind)
    usr = cfg.usr
    prec = usr["precision"]
    s = SimpleNamespace(mode=mode, cfg=cfg, usr=usr, line=line, direction=direction, kind=kind, prec=prec)
    P = usr["num_cpml"]
    s.P = P
    rough = usr["rough_toggle"] and kind != "i" and usr["sim_type"] == "s-param" and profiles is not None
    if mode == "yee3d":
        nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
        n_eff = nz - cfg.p1z - (nz - cfg.p2z)
        upper, lower = (profiles if rough else (np.zeros(n_eff), np.zeros(n_eff)))
        FG = fg_mask_3d(nx, ny, nz, cfg.bx, cfg.by, cfg.nx_swg, cfg.ny_swg, cfg.pp, usr["num_lines"],
                        cfg.p1z, nz - cfg.p2z, upper, lower)
        shape = (nx, ny, nz)
    else:
        nx, ny = cfg.nx, cfg.ny
        n_eff = nx - cfg.p1x - (nx - cfg.p2x)
        upper, lower = (profiles if rough else (np.zeros(n_eff), np.zeros(n_eff)))
        FG = fg_mask_2d(nx, ny, cfg.by, cfg.ny_swg, cfg.pp, usr["num_lines"], cfg.p1x, nx - cfg.p2x, upper, lower)
        shape = (nx, ny)
    s.FG = FG
    s.shape = shape
    EPS_MASK = cfg.eps * (cfg.eps_rel_fg * FG + 1 * ~FG)
    dt, dx = cfg.delta_t, cfg.delta_x
    if mode == "tm2":
        s.CBZ = dt / EPS_MASK.copy().astype(prec)
    elif mode == "te2":
        EX = EPS_MASK.copy().astype(prec)
        EY = EPS_MASK.copy().astype(prec)
        average_materials_2d(EPS_MASK, EX, EY)
        s.CBX = dt / EX
        s.CBY = dt / EY
    else:
        EX = EPS_MASK.copy().astype(prec)
        EY = EPS_MASK.copy().astype(prec)
        EZ = EPS_MASK.copy().astype(prec)
        average_materials_3d(EPS_MASK, EX, EY, EZ)
        s.CBX = dt / EX
        s.CBY = dt / EY
        s.CBZ = dt / EZ
    s.DB = dt / cfg.mu
    nf = usr["sparam_num_freqs"]
    s.cosE, s.sinE, s.cosH, s.sinH = sfft_coeffs(cfg.sparam_freqs, dt, cfg.nt, prec)

    s.ib = s.jb = s.kb = OFFSET
    s.ie = shape[0] - OFFSET
    s.je = shape[1] - OFFSET
    if mode == "yee3d":
        s.ke = shape[2] - OFFSET
    g = cpml_grading(P, dx, dt, cfg.eps, cfg.eta, prec)
    s.BE, s.CE, s.BH, s.CH = g["BE"], g["CE"], g["BH"], g["CH"]
    s.grading = g
    s.KXE, s.KXH = kappa_dx(shape[0], s.ib, s.ie, P, g["KE"], g["KH"], dx, prec)
    s.KYE, s.KYH = kappa_dx(shape[1], s.jb, s.je, P, g["KE"], g["KH"], dx, prec)
    if mode == "yee3d":
        s.KZE, s.KZH = kappa_dx(shape[2], s.kb, s.ke, P, g["KE"], g["KH"], dx, prec)

    z = lambda *sh: np.zeros(sh, dtype=prec)
    if mode == "tm2":
        s.EZ, s.HX, s.HY = z(*shape), z(*shape), z(*shape)
        s.PSI_EZ_XLO, s.PSI_EZ_XHI = z(P, ny), z(P, ny)
        s.PSI_EZ_YLO, s.PSI_EZ_YHI = z(nx, P), z(nx, P)
        s.PSI_HX_YLO, s.PSI_HX_YHI = z(nx, P), z(nx, P)
        s.PSI_HY_XLO, s.PSI_HY_XHI = z(P, ny), z(P, ny)
        s.dft = {k: z(nf, ny) for k in ("E1r", "E1i", "H1r", "H1i", "E2r", "E2i", "H2r", "H2i")}
    elif mode == "te2":
        s.EX, s.EY, s.HZ = z(*shape), z(*shape), z(*shape)
        s.PSI_EX_YLO, s.PSI_EX_YHI = z(nx, P), z(nx, P)
        s.PSI_EY_XLO, s.PSI_EY_XHI = z(P, ny), z(P, ny)
        s.PSI_HZ_XLO, s.PSI_HZ_XHI = z(P, ny), z(P, ny)
        s.PSI_HZ_YLO, s.PSI_HZ_YHI = z(nx, P), z(nx, P)
        s.dft = {k: z(nf, ny) for k in ("E1r", "E1i", "H1r", "H1i", "E2r", "E2i", "H2r", "H2i")}
    else:
        for f in ("EX", "EY", "EZ", "HX", "HY", "HZ"):
            setattr(s, f, z(*shape))
        for comp in ("EX", "EY", "EZ", "HX", "HY", "HZ"):
            for ax in "XYZ":
                if ax == comp[1]:
                    continue
                shp = {"X": (P, ny, nz), "Y": (nx, P, nz), "Z": (nx, ny, P)}[ax]
                setattr(s, "PSI_%s_%sLO" % (comp, ax), z(*shp))
                setattr(s, "PSI_%s_%sHI" % (comp, ax), z(*shp))
        s.dft = {}
        for port in "12":
            for c_ in ("EX", "EY", "HX", "HY"):
                s.dft[c_ + port + "r"] = z(nf, nx, ny)
                s.dft[c_ + port + "i"] = z(nf, nx, ny)
    s.nf = nf
    s.source_shift = line * cfg.pp
    s.src_box = source_box(s)
    s.n = 0
    return s


def source_box(s):
    """Soft-source box ``(field, xb, yb[, zb], xe, ye[, ze])`` for the run.

    TM2/fdtd_main.py:280-286 (Ez line), TE2/fdtd_main.py:291-297 (Hz line,
    inset by 2), FDTD_3D/.../fdtd_main.py:364-379 (Ey or Hy sheet)."""
    cfg, usr = s.cfg, s.usr
    sh = s.source_shift
    if usr["sim_type"] != "s-param":
        raise NotImplementedError("only sim_type='s-param' has a defined source")
    if s.mode == "tm2":
        ys, ye = cfg.by + sh + 1, cfg.by + sh + cfg.ny_swg - 1
        if s.direction == "f":
            return ("EZ", cfg.sx, ys, cfg.sx + 1, ye)
        return ("EZ", cfg.nx - cfg.sx - 1, ys, cfg.nx - cfg.sx, ye)
    if s.mode == "te2":
        ys, ye = cfg.by + sh + 2, cfg.by + sh + cfg.ny_swg - 2
        if s.direction == "f":
            return ("HZ", cfg.sx, ys, cfg.sx + 1, ye)
        return ("HZ", cfg.nx - cfg.sx - 1, ys, cfg.nx - cfg.sx, ye)
    sc = usr["source_condition"]
    if s.direction == "f":
        zb, ze = cfg.sz, cfg.sz + 2
    else:
        zb, ze = cfg.nz - cfg.sz - 1, cfg.nz - cfg.sz
    if sc == "TE":
        return ("EY", cfg.bx + sh + 1, cfg.by + 1, zb, cfg.bx + sh + cfg.nx_swg - 1, cfg.by + cfg.ny_swg - 1, ze)
    return ("HY", cfg.bx + sh + 2, cfg.by + 2, zb, cfg.bx + sh + cfg.nx_swg - 2, cfg.by + cfg.ny_swg - 2, ze)


def _box_slices(shape, lo, hi):
    return tuple(slice(max(0, a), max(0, min(n, b))) for n, a, b in zip(shape, lo, hi))


def update_source(F, src, lo, hi):
    """``update_source`` (TM2/fdtd_funcs.py:71-76; 3D :104-110): F -= J[n]."""
    sl = _box_slices(F.shape, lo, hi)
    F[sl] = F[sl] - src


# ---------------------------------------------------------------------------
# 2D TM kernels (FDTD_2D_TM/s-parameter_extraction/fdtd_funcs.py)
# ---------------------------------------------------------------------------
def tm_update_ez(Ez, Hx, Hy, kxe, kye, cb, ib, jb, ie, je):  # :44-49
    I, J = slice(ib, ie), slice(jb, je)
    Ez[I, J] = Ez[I, J] + cb[I, J] * ((Hy[ib + 1:ie + 1, J] - Hy[I, J]) / kxe[I, None]
                                      - (Hx[I, jb + 1:je + 1] - Hx[I, J]) / kye[None, J])


def tm_update_hx(Ez, Hx, kyh, db, ib, jb, ie, je):  # :53-58
    I, J = slice(ib, ie), slice(jb + 1, je)
    Hx[I, J] = Hx[I, J] + db * (Ez[I, jb:je - 1] - Ez[I, J]) / kyh[None, J]


def tm_update_hy(Ez, Hy, kxh, db, ib, jb, ie, je):  # :62-67
    I, J = slice(ib + 1, ie), slice(jb, je)
    Hy[I, J] = Hy[I, J] + db * (Ez[I, J] - Ez[ib:ie - 1, J]) / kxh[I, None]


def tm_pml_ez_xinc(plo, phi, Ez, Hy, be, ce, cb, dx, P, ib, jb, ie, je):  # :80-88
    J = slice(jb, je)
    plo[:, J] = be[::-1][:, None] * plo[:, J] + ce[::-1][:, None] * (Hy[ib + 1:ib + P + 1, J] - Hy[ib:ib + P, J]) / dx
    Ez[ib:ib + P, J] = Ez[ib:ib + P, J] + cb[ib:ib + P, J] * plo[:, J]
    phi[:, J] = be[:, None] * phi[:, J] + ce[:, None] * (Hy[ie - P + 1:ie + 1, J] - Hy[ie - P:ie, J]) / dx
    Ez[ie - P:ie, J] = Ez[ie - P:ie, J] + cb[ie - P:ie, J] * phi[:, J]


def tm_pml_ez_yinc(plo, phi, Ez, Hx, be, ce, cb, dy, P, ib, jb, ie, je):  # :92-100
    I = slice(ib, ie)
    plo[I, :] = be[::-1][None, :] * plo[I, :] + ce[::-1][None, :] * (Hx[I, jb + 1:jb + P + 1] - Hx[I, jb:jb + P]) / dy
    Ez[I, jb:jb + P] = Ez[I, jb:jb + P] - cb[I, jb:jb + P] * plo[I, :]
    phi[I, :] = be[None, :] * phi[I, :] + ce[None, :] * (Hx[I, je - P + 1:je + 1] - Hx[I, je - P:je]) / dy
    Ez[I, je - P:je] = Ez[I, je - P:je] - cb[I, je - P:je] * phi[I, :]


def tm_pml_hx_yinc(plo, phi, Ez, Hx, bh, ch, db, dy, P, ib, jb, ie, je):  # :104-112
    I = slice(ib, ie)
    bl, cl = bh[P - 1:0:-1][None, :], ch[P - 1:0:-1][None, :]
    plo[I, 1:P] = bl * plo[I, 1:P] + cl * (Ez[I, jb + 1:jb + P] - Ez[I, jb:jb + P - 1]) / dy
    Hx[I, jb + 1:jb + P] = Hx[I, jb + 1:jb + P] - db * plo[I, 1:P]
    phi[I, 1:P] = bh[None, 1:P] * phi[I, 1:P] + ch[None, 1:P] * (Ez[I, je - P + 1:je] - Ez[I, je - P:je - 1]) / dy
    Hx[I, je - P + 1:je] = Hx[I, je - P + 1:je] - db * phi[I, 1:P]


def tm_pml_hy_xinc(plo, phi, Ez, Hy, bh, ch, db, dx, P, ib, jb, ie, je):  # :116-124
    J = slice(jb, je)
    bl, cl = bh[P - 1:0:-1][:, None], ch[P - 1:0:-1][:, None]
    plo[1:P, J] = bl * plo[1:P, J] + cl * (Ez[ib + 1:ib + P, J] - Ez[ib:ib + P - 1, J]) / dx
    Hy[ib + 1:ib + P, J] = Hy[ib + 1:ib + P, J] + db * plo[1:P, J]
    phi[1:P, J] = bh[1:P, None] * phi[1:P, J] + ch[1:P, None] * (Ez[ie - P + 1:ie, J] - Ez[ie - P:ie - 1, J]) / dx
    Hy[ie - P + 1:ie, J] = Hy[ie - P + 1:ie, J] + db * phi[1:P, J]


# ---------------------------------------------------------------------------
# 2D TE kernels (FDTD_2D_TE/s-parameter_extraction/fdtd_funcs.py)
# ---------------------------------------------------------------------------
def te_update_ex(Ex, Hz, kye, cb, ib, jb, ie, je):  # :43-49
    I, J = slice(ib + 1, ie), slice(jb, je)
    Ex[I, J] = Ex[I, J] + cb[I, J] * (Hz[I, jb + 1:je + 1] - Hz[I, J]) / kye[None, J]


def te_update_ey(Ey, Hz, kxe, cb, ib, jb, ie, je):  # :52-58
    I, J = slice(ib, ie), slice(jb + 1, je)
    Ey[I, J] = Ey[I, J] + cb[I, J] * (Hz[I, J] - Hz[ib + 1:ie + 1, J]) / kxe[I, None]


def te_update_hz(Ex, Ey, Hz, kxh, kyh, db, ib, jb, ie, je):  # :61-67
    I, J = slice(ib + 1, ie), slice(jb + 1, je)
    Hz[I, J] = Hz[I, J] + db * ((Ex[I, J] - Ex[I, jb:je - 1]) / kyh[None, J]
                                - (Ey[I, J] - Ey[ib:ie - 1, J]) / kxh[I, None])


def te_pml_ex_yinc(plo, phi, Ex, Hz, be, ce, cb, dy, P, ib, jb, ie, je):  # :79-87
    I = slice(ib + 1, ie)
    plo[I, :] = be[::-1][None, :] * plo[I, :] + ce[::-1][None, :] * (Hz[I, jb + 1:jb + P + 1] - Hz[I, jb:jb + P]) / dy
    Ex[I, jb:jb + P] = Ex[I, jb:jb + P] + cb[I, jb:jb + P] * plo[I, :]
    phi[I, :] = be[None, :] * phi[I, :] + ce[None, :] * (Hz[I, je - P + 1:je + 1] - Hz[I, je - P:je]) / dy
    Ex[I, je - P:je] = Ex[I, je - P:je] + cb[I, je - P:je] * phi[I, :]


def te_pml_ey_xinc(plo, phi, Ey, Hz, be, ce, cb, dx, P, ib, jb, ie, je):  # :91-99
    J = slice(jb + 1, je)
    plo[:, J] = be[::-1][:, None] * plo[:, J] + ce[::-1][:, None] * (Hz[ib + 1:ib + P + 1, J] - Hz[ib:ib + P, J]) / dx
    Ey[ib:ib + P, J] = Ey[ib:ib + P, J] - cb[ib:ib + P, J] * plo[:, J]
    phi[:, J] = be[:, None] * phi[:, J] + ce[:, None] * (Hz[ie - P + 1:ie + 1, J] - Hz[ie - P:ie, J]) / dx
    Ey[ie - P:ie, J] = Ey[ie - P:ie, J] - cb[ie - P:ie, J] * phi[:, J]


def te_pml_hz_xinc(plo, phi, Ey, Hz, bh, ch, db, dx, P, ib, jb, ie, je):  # :103-111
    J = slice(jb + 1, je)
    bl, cl = bh[P - 1:0:-1][:, None], ch[P - 1:0:-1][:, None]
    plo[1:P, J] = bl * plo[1:P, J] + cl * (Ey[ib + 1:ib + P, J] - Ey[ib:ib + P - 1, J]) / dx
    Hz[ib + 1:ib + P, J] = Hz[ib + 1:ib + P, J] - db * plo[1:P, J]
    phi[1:P, J] = bh[1:P, None] * phi[1:P, J] + ch[1:P, None] * (Ey[ie - P + 1:ie, J] - Ey[ie - P:ie - 1, J]) / dx
    Hz[ie - P + 1:ie, J] = Hz[ie - P + 1:ie, J] - db * phi[1:P, J]


def te_pml_hz_yinc(plo, phi, Ex, Hz, bh, ch, db, dy, P, ib, jb, ie, je):  # :115-123
    I = slice(ib + 1, ie)
    bl, cl = bh[P - 1:0:-1][None, :], ch[P - 1:0:-1][None, :]
    plo[I, 1:P] = bl * plo[I, 1:P] + cl * (Ex[I, jb + 1:jb + P] - Ex[I, jb:jb + P - 1]) / dy
    Hz[I, jb + 1:jb + P] = Hz[I, jb + 1:jb + P] + db * plo[I, 1:P]
    phi[I, 1:P] = bh[None, 1:P] * phi[I, 1:P] + ch[None, 1:P] * (Ex[I, je - P + 1:je] - Ex[I, je - P:je - 1]) / dy
    Hz[I, je - P + 1:je] = Hz[I, je - P + 1:je] + db * phi[I, 1:P]


# ---------------------------------------------------------------------------
# 3D kernels (FDTD_3D/s-parameter_extraction/fdtd_funcs.py)
# ---------------------------------------------------------------------------
def y3_update_ex(Ex, Hy, Hz, kye, kze, cb, ib, jb, kb, ie, je, ke):  # :43-50
    I, J, K = slice(ib + 1, ie), slice(jb, je), slice(kb, ke)
    Ex[I, J, K] = Ex[I, J, K] + cb[I, J, K] * ((Hz[I, jb + 1:je + 1, K] - Hz[I, J, K]) / kye[None, J, None]
                                               - (Hy[I, J, kb + 1:ke + 1] - Hy[I, J, K]) / kze[None, None, K])


def y3_update_ey(Ey, Hx, Hz, kxe, kze, cb, ib, jb, kb, ie, je, ke):  # :53-60
    I, J, K = slice(ib, ie), slice(jb + 1, je), slice(kb, ke)
    Ey[I, J, K] = Ey[I, J, K] + cb[I, J, K] * ((Hx[I, J, kb + 1:ke + 1] - Hx[I, J, K]) / kze[None, None, K]
                                               - (Hz[ib + 1:ie + 1, J, K] - Hz[I, J, K]) / kxe[I, None, None])


def y3_update_ez(Ez, Hx, Hy, kxe, kye, cb, ib, jb, kb, ie, je, ke):  # :63-70
    I, J, K = slice(ib, ie), slice(jb, je), slice(kb + 1, ke)
    Ez[I, J, K] = Ez[I, J, K] + cb[I, J, K] * ((Hy[ib + 1:ie + 1, J, K] - Hy[I, J, K]) / kxe[I, None, None]
                                               - (Hx[I, jb + 1:je + 1, K] - Hx[I, J, K]) / kye[None, J, None])


def y3_update_hx(Ey, Ez, Hx, kyh, kzh, db, ib, jb, kb, ie, je, ke):  # :73-80
    I, J, K = slice(ib, ie), slice(jb + 1, je), slice(kb + 1, ke)
    Hx[I, J, K] = Hx[I, J, K] + db * ((Ey[I, J, K] - Ey[I, J, kb:ke - 1]) / kzh[None, None, K]
                                      - (Ez[I, J, K] - Ez[I, jb:je - 1, K]) / kyh[None, J, None])


def y3_update_hy(Ex, Ez, Hy, kxh, kzh, db, ib, jb, kb, ie, je, ke):  # :83-90
    I, J, K = slice(ib + 1, ie), slice(jb, je), slice(kb + 1, ke)
    Hy[I, J, K] = Hy[I, J, K] + db * ((Ez[I, J, K] - Ez[ib:ie - 1, J, K]) / kxh[I, None, None]
                                      - (Ex[I, J, K] - Ex[I, J, kb:ke - 1]) / kzh[None, None, K])


def y3_update_hz(Ex, Ey, Hz, kxh, kyh, db, ib, jb, kb, ie, je, ke):  # :93-100
    I, J, K = slice(ib + 1, ie), slice(jb + 1, je), slice(kb, ke)
    Hz[I, J, K] = Hz[I, J, K] + db * ((Ex[I, J, K] - Ex[I, jb:je - 1, K]) / kyh[None, J, None]
                                      - (Ey[I, J, K] - Ey[ib:ie - 1, J, K]) / kxh[I, None, None])


def _ax(v, axis, ndim=3):
    sh = [1] * ndim
    sh[axis] = -1
    return v.reshape(sh)


def y3_pml_e(plo, phi, E, H, be, ce, cb, dd, P, rng, axis, b, e, sign):
    """One E-field CPML kernel (FDTD_3D/.../fdtd_funcs.py:113-188).

    ``rng`` = slices for the two transverse axes (the slab axis entry is
    ignored); ``axis`` = the slab axis; ``b``/``e`` = its domain limits;
    ``sign`` = +1 (``E + cb*psi``) or -1 (``E - cb*psi``).
    ``psi = be[-(d+1)]*psi + ce[-(d+1)]*(H[b+d+1]-H[b+d])/dd`` on the low slab,
    ``be[d]`` and ``H[e-P+d+1]-H[e-P+d]`` on the high slab.
    """
    def sl(a0, a1):
        s = list(rng)
        s[axis] = slice(a0, a1)
        return tuple(s)
    ps = sl(0, P)
    blo, clo = _ax(be[::-1], axis), _ax(ce[::-1], axis)
    plo[ps] = blo * plo[ps] + clo * (H[sl(b + 1, b + P + 1)] - H[sl(b, b + P)]) / dd
    if sign > 0:
        E[sl(b, b + P)] = E[sl(b, b + P)] + cb[sl(b, b + P)] * plo[ps]
    else:
        E[sl(b, b + P)] = E[sl(b, b + P)] - cb[sl(b, b + P)] * plo[ps]
    phi[ps] = _ax(be, axis) * phi[ps] + _ax(ce, axis) * (H[sl(e - P + 1, e + 1)] - H[sl(e - P, e)]) / dd
    if sign > 0:
        E[sl(e - P, e)] = E[sl(e - P, e)] + cb[sl(e - P, e)] * phi[ps]
    else:
        E[sl(e - P, e)] = E[sl(e - P, e)] - cb[sl(e - P, e)] * phi[ps]


def y3_pml_h(plo, phi, E, H, bh, ch, db, dd, P, rng, axis, b, e, sign):
    """One H-field CPML kernel (FDTD_3D/.../fdtd_funcs.py:191-266); slab index
    d runs over 1..P-1 (``i > 0 and i < pmle``); low slab uses ``bh[-d]``."""
    def sl(a0, a1):
        s = list(rng)
        s[axis] = slice(a0, a1)
        return tuple(s)
    ps = sl(1, P)
    blo, clo = _ax(bh[P - 1:0:-1], axis), _ax(ch[P - 1:0:-1], axis)
    plo[ps] = blo * plo[ps] + clo * (E[sl(b + 1, b + P)] - E[sl(b, b + P - 1)]) / dd
    if sign > 0:
        H[sl(b + 1, b + P)] = H[sl(b + 1, b + P)] + db * plo[ps]
    else:
        H[sl(b + 1, b + P)] = H[sl(b + 1, b + P)] - db * plo[ps]
    phi[ps] = _ax(bh[1:P], axis) * phi[ps] + _ax(ch[1:P], axis) * (E[sl(e - P + 1, e)] - E[sl(e - P, e - 1)]) / dd
    if sign > 0:
        H[sl(e - P + 1, e)] = H[sl(e - P + 1, e)] + db * phi[ps]
    else:
        H[sl(e - P + 1, e)] = H[sl(e - P + 1, e)] - db * phi[ps]


# ---------------------------------------------------------------------------
# Running port DFTs
# ---------------------------------------------------------------------------
def dft_2d_e(R, I, F, cos, sin, n, ic, jb, je, avg_j=False):
    """``simul_fft_efield`` TM (TM2/fdtd_funcs.py:128-134) or TE (2-point
    average along j, TE2/fdtd_funcs.py:127-134)."""
    J = slice(jb, je)
    x = (0.5 * (F[ic, J] + F[ic, jb + 1:je + 1])) if avg_j else F[ic, J]
    R[:, J] = R[:, J] + x[None, :] * cos[:, n][:, None]
    I[:, J] = I[:, J] - x[None, :] * sin[:, n][:, None]


def dft_2d_h(R, I, F, cos, sin, n, ic, jb, je, four=False):
    """``simul_fft_hfield`` TM: 2-point along i (TM2/fdtd_funcs.py:138-144);
    TE: 4-point (TE2/fdtd_funcs.py:137-144)."""
    J = slice(jb, je)
    if four:
        x = 0.25 * (F[ic, J] + F[ic + 1, J] + F[ic, jb + 1:je + 1] + F[ic + 1, jb + 1:je + 1])
    else:
        x = 0.5 * (F[ic, J] + F[ic + 1, J])
    R[:, J] = R[:, J] + x[None, :] * cos[:, n][:, None]
    I[:, J] = I[:, J] - x[None, :] * sin[:, n][:, None]


def dft_3d_e(Rx, Ry, Ix, Iy, Ex, Ey, cos, sin, n, ib, jb, ie, je, kc):  # :269-279
    I, J = slice(ib, ie), slice(jb, je)
    c, s_ = cos[:, n][:, None, None], sin[:, n][:, None, None]
    x = (0.5 * (Ex[I, J, kc] + Ex[ib + 1:ie + 1, J, kc]))[None]
    y = (0.5 * (Ey[I, J, kc] + Ey[I, jb + 1:je + 1, kc]))[None]
    Rx[:, I, J] = Rx[:, I, J] + x * c
    Ix[:, I, J] = Ix[:, I, J] - x * s_
    Ry[:, I, J] = Ry[:, I, J] + y * c
    Iy[:, I, J] = Iy[:, I, J] - y * s_


def dft_3d_h(Rx, Ry, Ix, Iy, Hx, Hy, cos, sin, n, ib, jb, ie, je, kc):  # :282-292
    I, J = slice(ib, ie), slice(jb, je)
    J1, I1 = slice(jb + 1, je + 1), slice(ib + 1, ie + 1)
    c, s_ = cos[:, n][:, None, None], sin[:, n][:, None, None]
    x = (0.25 * (Hx[I, J, kc] + Hx[I, J1, kc] + Hx[I, J, kc + 1] + Hx[I, J1, kc + 1]))[None]
    y = (0.25 * (Hy[I, J, kc] + Hy[I1, J, kc] + Hy[I, J, kc + 1] + Hy[I1, J, kc + 1]))[None]
    Rx[:, I, J] = Rx[:, I, J] + x * c
    Ix[:, I, J] = Ix[:, I, J] - x * s_
    Ry[:, I, J] = Ry[:, I, J] + y * c
    Iy[:, I, J] = Iy[:, I, J] - y * s_


# ---------------------------------------------------------------------------
# Time step (fdtd_main.py hot loops)
# ---------------------------------------------------------------------------
def step(s):
    """Advance one time step n = ``s.n`` in the reference launch order."""
    n = s.n
    P, ib, jb, ie, je = s.P, s.ib, s.jb, s.ie, s.je
    dx = s.cfg.delta_x
    J = s.cfg.J_SRC[n]
    box = s.src_box
    d = s.dft
    nf = s.nf
    if s.mode == "tm2":  # TM2/fdtd_main.py:275-304
        tm_update_ez(s.EZ, s.HX, s.HY, s.KXE, s.KYE, s.CBZ, ib, jb, ie, je)
        update_source(s.EZ, J, box[1:3], box[3:5])
        tm_pml_ez_xinc(s.PSI_EZ_XLO, s.PSI_EZ_XHI, s.EZ, s.HY, s.BE, s.CE, s.CBZ, dx, P, ib, jb, ie, je)
        tm_pml_ez_yinc(s.PSI_EZ_YLO, s.PSI_EZ_YHI, s.EZ, s.HX, s.BE, s.CE, s.CBZ, dx, P, ib, jb, ie, je)
        tm_update_hx(s.EZ, s.HX, s.KYH, s.DB, ib, jb, ie, je)
        tm_update_hy(s.EZ, s.HY, s.KXH, s.DB, ib, jb, ie, je)
        tm_pml_hx_yinc(s.PSI_HX_YLO, s.PSI_HX_YHI, s.EZ, s.HX, s.BH, s.CH, s.DB, dx, P, ib, jb, ie, je)
        tm_pml_hy_xinc(s.PSI_HY_XLO, s.PSI_HY_XHI, s.EZ, s.HY, s.BH, s.CH, s.DB, dx, P, ib, jb, ie, je)
        ny = s.shape[1]
        for port, ic in (("1", s.cfg.p1x), ("2", s.cfg.p2x)):
            dft_2d_e(d["E%sr" % port], d["E%si" % port], s.EZ, s.cosE, s.sinE, n, ic, P, ny - P)
            dft_2d_h(d["H%sr" % port], d["H%si" % port], s.HY, s.cosH, s.sinH, n, ic, P, ny - P)
    elif s.mode == "te2":  # TE2/fdtd_main.py:279-308
        te_update_ex(s.EX, s.HZ, s.KYE, s.CBX, ib, jb, ie, je)
        te_update_ey(s.EY, s.HZ, s.KXE, s.CBY, ib, jb, ie, je)
        te_pml_ex_yinc(s.PSI_EX_YLO, s.PSI_EX_YHI, s.EX, s.HZ, s.BE, s.CE, s.CBX, dx, P, ib, jb, ie, je)
        te_pml_ey_xinc(s.PSI_EY_XLO, s.PSI_EY_XHI, s.EY, s.HZ, s.BE, s.CE, s.CBY, dx, P, ib, jb, ie, je)
        te_update_hz(s.EX, s.EY, s.HZ, s.KXH, s.KYH, s.DB, ib, jb, ie, je)
        update_source(s.HZ, J, box[1:3], box[3:5])
        te_pml_hz_xinc(s.PSI_HZ_XLO, s.PSI_HZ_XHI, s.EY, s.HZ, s.BH, s.CH, s.DB, dx, P, ib, jb, ie, je)
        te_pml_hz_yinc(s.PSI_HZ_YLO, s.PSI_HZ_YHI, s.EX, s.HZ, s.BH, s.CH, s.DB, dx, P, ib, jb, ie, je)
        ny = s.shape[1]
        for port, ic in (("1", s.cfg.p1x), ("2", s.cfg.p2x)):
            dft_2d_e(d["E%sr" % port], d["E%si" % port], s.EY, s.cosE, s.sinE, n, ic, P, ny - P, avg_j=True)
            dft_2d_h(d["H%sr" % port], d["H%si" % port], s.HZ, s.cosH, s.sinH, n, ic, P, ny - P, four=True)
    else:  # FDTD_3D/.../fdtd_main.py:357-406
        kb, ke = s.kb, s.ke
        nx, ny, nz = s.shape
        y3_update_ex(s.EX, s.HY, s.HZ, s.KYE, s.KZE, s.CBX, ib, jb, kb, ie, je, ke)
        y3_update_ey(s.EY, s.HX, s.HZ, s.KXE, s.KZE, s.CBY, ib, jb, kb, ie, je, ke)
        y3_update_ez(s.EZ, s.HX, s.HY, s.KXE, s.KYE, s.CBZ, ib, jb, kb, ie, je, ke)
        update_source(getattr(s, box[0]), J, box[1:4], box[4:7])
        A = slice(None)
        ex_t = (slice(ib + 1, ie), A, A)
        ey_t = (A, slice(jb + 1, je), A)
        ez_t = (A, A, slice(kb + 1, ke))
        # E-field CPML, launch order :382-387
        y3_pml_e(s.PSI_EX_YLO, s.PSI_EX_YHI, s.EX, s.HZ, s.BE, s.CE, s.CBX, dx, P, (ex_t[0], A, slice(kb, ke)), 1, jb, je, +1)
        y3_pml_e(s.PSI_EX_ZLO, s.PSI_EX_ZHI, s.EX, s.HY, s.BE, s.CE, s.CBX, dx, P, (ex_t[0], slice(jb, je), A), 2, kb, ke, -1)
        y3_pml_e(s.PSI_EY_XLO, s.PSI_EY_XHI, s.EY, s.HZ, s.BE, s.CE, s.CBY, dx, P, (A, ey_t[1], slice(kb, ke)), 0, ib, ie, -1)
        y3_pml_e(s.PSI_EY_ZLO, s.PSI_EY_ZHI, s.EY, s.HX, s.BE, s.CE, s.CBY, dx, P, (slice(ib, ie), ey_t[1], A), 2, kb, ke, +1)
        y3_pml_e(s.PSI_EZ_XLO, s.PSI_EZ_XHI, s.EZ, s.HY, s.BE, s.CE, s.CBZ, dx, P, (A, slice(jb, je), ez_t[2]), 0, ib, ie, +1)
        y3_pml_e(s.PSI_EZ_YLO, s.PSI_EZ_YHI, s.EZ, s.HX, s.BE, s.CE, s.CBZ, dx, P, (slice(ib, ie), A, ez_t[2]), 1, jb, je, -1)
        y3_update_hx(s.EY, s.EZ, s.HX, s.KYH, s.KZH, s.DB, ib, jb, kb, ie, je, ke)
        y3_update_hy(s.EX, s.EZ, s.HY, s.KXH, s.KZH, s.DB, ib, jb, kb, ie, je, ke)
        y3_update_hz(s.EX, s.EY, s.HZ, s.KXH, s.KYH, s.DB, ib, jb, kb, ie, je, ke)
        # H-field CPML, launch order :395-400
        y3_pml_h(s.PSI_HX_YLO, s.PSI_HX_YHI, s.EZ, s.HX, s.BH, s.CH, s.DB, dx, P, (slice(ib, ie), A, slice(kb + 1, ke)), 1, jb, je, -1)
        y3_pml_h(s.PSI_HX_ZLO, s.PSI_HX_ZHI, s.EY, s.HX, s.BH, s.CH, s.DB, dx, P, (slice(ib, ie), slice(jb + 1, je), A), 2, kb, ke, +1)
        y3_pml_h(s.PSI_HY_XLO, s.PSI_HY_XHI, s.EZ, s.HY, s.BH, s.CH, s.DB, dx, P, (A, slice(jb, je), slice(kb + 1, ke)), 0, ib, ie, +1)
        y3_pml_h(s.PSI_HY_ZLO, s.PSI_HY_ZHI, s.EX, s.HY, s.BH, s.CH, s.DB, dx, P, (slice(ib + 1, ie), slice(jb, je), A), 2, kb, ke, -1)
        y3_pml_h(s.PSI_HZ_XLO, s.PSI_HZ_XHI, s.EY, s.HZ, s.BH, s.CH, s.DB, dx, P, (A, slice(jb + 1, je), slice(kb, ke)), 0, ib, ie, -1)
        y3_pml_h(s.PSI_HZ_YLO, s.PSI_HZ_YHI, s.EX, s.HZ, s.BH, s.CH, s.DB, dx, P, (slice(ib + 1, ie), A, slice(kb, ke)), 1, jb, je, +1)
        for port, kc in (("1", s.cfg.p1z), ("2", s.cfg.p2z)):
            dft_3d_e(d["EX%sr" % port], d["EY%sr" % port], d["EX%si" % port], d["EY%si" % port],
                     s.EX, s.EY, s.cosE, s.sinE, n, P, P, nx - P, ny - P, kc)
            dft_3d_h(d["HX%sr" % port], d["HY%sr" % port], d["HX%si" % port], d["HY%si" % port],
                     s.HX, s.HY, s.cosH, s.sinH, n, P, P, nx - P, ny - P, kc)
    s.n += 1


def run(s, nsteps=None):
    """Run ``nsteps`` steps (default: the whole ``nt``)."""
    nsteps = s.cfg.nt - s.n if nsteps is None else nsteps
    for _ in range(nsteps):
        step(s)
    return s


# ---------------------------------------------------------------------------
# Outputs (fdtd_main.py:349-386, 3D :450-512)
# ---------------------------------------------------------------------------
def outputs(s) -> dict:
    """The ``.npy`` payloads the reference saves for this run, by file stem."""
    d, l = s.dft, s.line + 1
    res = {}
    comps = (("ez", "E"), ("hy", "H")) if s.mode == "tm2" else (("ey", "E"), ("hz", "H")) if s.mode == "te2" else \
        (("ex", "EX"), ("ey", "EY"), ("hx", "HX"), ("hy", "HY"))
    tags = {("i", "f"): (("fi", "1"),), ("i", "b"): (("bi", "2"),),
            ("r", "f"): (("ft", "1"), ("br", "2")), ("r", "b"): (("fr", "1"), ("bt", "2"))}[(s.kind, s.direction)]
    for tag, port in tags:
        for name, key in comps:
            res["%s_%s_l%d" % (name, tag, l)] = d[key + port + "r"] + 1j * d[key + port + "i"]
    return res


def extract_sparams(usr: dict, mode: str, data: dict) -> np.ndarray:
    """S-matrix from the saved DFTs.

    2D: TM2/extract_sparams.py:48-104 (``j >= i`` loop, ``sav = -1/2 Ez Hy*``;
    TE uses ``+1/2 Ey Hz*``, TE2/extract_sparams.py:88-89).
    3D: FDTD_3D/.../extract_sparams.py:48-131 (all (i, j) pairs, so the later
    pair wins the symmetric fill; power summed over y in [P, ny-P)).
    """
    cfg = autosetup(usr, mode, "r")
    usr = cfg.usr
    cprec = np.complex64 if usr["precision"] == np.float32 else np.complex128
    nports = 2 * usr["num_lines"]
    nf = usr["sparam_num_freqs"]
    S = np.zeros([nf, nports, nports], dtype=cprec)
    if mode == "yee3d":
        names = ("ex", "ey", "hx", "hy")
    elif mode == "tm2":
        names = ("ez", "hy")
    else:
        names = ("ey", "hz")
    P = usr["num_cpml"]
    for i in range(nports):
        for j in (range(nports) if mode == "yee3d" else range(i, nports)):
            iline, jline = i // 2 + 1, j // 2 + 1
            inc_tag = "fi" if j % 2 == 0 else "bi"
            if i % 2 == j % 2:
                ref_tag = "ft" if i % 2 == 0 else "bt"
            else:
                ref_tag = "fr" if i % 2 == 0 else "br"
            inc = [data["%s_%s_l%d" % (nm, inc_tag, jline)] for nm in names]
            ref = [data["%s_%s_l%d" % (nm, ref_tag, jline)].copy() for nm in names]
            if i == j:
                cor_tag = "fi" if i % 2 == 0 else "bi"
                cor = [data["%s_%s_l%d" % (nm, cor_tag, iline)] for nm in names]
                ref = [r - c_ for r, c_ in zip(ref, cor)]
            if mode == "yee3d":
                sav_inc = 0.5 * (inc[0] * np.conjugate(inc[3]) - inc[1] * np.conjugate(inc[2]))
                sav_ref = 0.5 * (ref[0] * np.conjugate(ref[3]) - ref[1] * np.conjugate(ref[2]))
                start_inc = cfg.bx + cfg.cx_swg - cfg.ph + cfg.pp * (jline - 1)
                start_ref = cfg.bx + cfg.cx_swg - cfg.ph + cfg.pp * (iline - 1)
            else:
                sgn = -0.5 if mode == "tm2" else 0.5
                sav_inc = sgn * (inc[0] * np.conjugate(inc[1]))
                sav_ref = sgn * (ref[0] * np.conjugate(ref[1]))
                start_inc = cfg.by + cfg.cy_swg - cfg.ph + cfg.pp * (jline - 1)
                start_ref = cfg.by + cfg.cy_swg - cfg.ph + cfg.pp * (iline - 1)
            Pinc = np.zeros(nf, dtype=cprec)
            Pref = np.zeros(nf, dtype=cprec)
            if mode == "yee3d":
                for y in range(P, cfg.ny - P):
                    for p in range(start_inc, start_inc + cfg.pp):
                        Pinc += sav_inc[:, p, y]
                    for p in range(start_ref, start_ref + cfg.pp):
                        Pref += sav_ref[:, p, y]
            else:
                for p in range(start_inc, start_inc + cfg.pp):
                    Pinc += sav_inc[:, p]
                for p in range(start_ref, start_ref + cfg.pp):
                    Pref += sav_ref[:, p]
            S[:, i, j] = np.sqrt(Pref / Pinc)
            S[:, j, i] = np.sqrt(Pref / Pinc)
    return S


def field_names(mode):
    return {"tm2": ("EZ", "HX", "HY"), "te2": ("EX", "EY", "HZ"),
            "yee3d": ("EX", "EY", "EZ", "HX", "HY", "HZ")}[mode]


# ---------------------------------------------------------------------------
# Explicit inputs (grids stated by cell counts rather than user_config)
# ---------------------------------------------------------------------------
def from_arrays(mode, shape, P, lim_lo, lim_hi, cb, kdx, be, ce, bh, ch, db, dx, src_field, src_lo,
                src_hi, j_src, port_pos, twiddles, nf, dtype=np.float64):
    """Oracle state from explicit arrays (the same inputs an engine job gets).

    ``cb`` maps 'x'/'y'/'z' to dt/eps grids, ``kdx`` maps 'xe','xh',... to
    kappa*dx, ``src_field`` is one of 'EX'..'HZ', ``twiddles`` =
    (cosE, sinE, cosH, sinH) [nf][nt].  The time loop is :func:`step`.
    """
    t = lambda a: np.asarray(a, dtype=dtype)
    s = SimpleNamespace(mode=mode, P=P, prec=dtype, shape=tuple(shape), n=0, nf=nf, line=0, direction="f", kind="r")
    cfg = SimpleNamespace(delta_x=dtype(dx), J_SRC=t(j_src))
    if mode == "yee3d":
        cfg.p1z, cfg.p2z = port_pos
    else:
        cfg.p1x, cfg.p2x = port_pos
    s.cfg = cfg
    s.ib, s.jb = lim_lo[0], lim_lo[1]
    s.ie, s.je = lim_hi[0], lim_hi[1]
    if mode == "yee3d":
        s.kb, s.ke = lim_lo[2], lim_hi[2]
    for ax in "xyz":
        if ax in cb:
            setattr(s, "CB" + ax.upper(), t(cb[ax]))
    for key, v in kdx.items():
        setattr(s, "K%s%s" % (key[0].upper(), key[1].upper()), t(v))
    s.BE, s.CE, s.BH, s.CH = t(be), t(ce), t(bh), t(ch)
    s.DB = dtype(db)
    s.cosE, s.sinE, s.cosH, s.sinH = (np.asarray(a, dtype=np.float64) for a in twiddles)
    z = lambda *sh: np.zeros(sh, dtype=dtype)
    nx, ny = shape[0], shape[1]
    for f in field_names(mode):
        setattr(s, f, z(*shape))
    if mode == "yee3d":
        nz = shape[2]
        for comp in field_names(mode):
            for ax in "XYZ":
                if ax == comp[1]:
                    continue
                shp = {"X": (P, ny, nz), "Y": (nx, P, nz), "Z": (nx, ny, P)}[ax]
                setattr(s, "PSI_%s_%sLO" % (comp, ax), z(*shp))
                setattr(s, "PSI_%s_%sHI" % (comp, ax), z(*shp))
        s.dft = {c_ + port + ri: z(nf, nx, ny) for port in "12" for c_ in ("EX", "EY", "HX", "HY") for ri in "ri"}
        s.src_box = (src_field,) + tuple(src_lo[:3]) + tuple(src_hi[:3])
    else:
        pairs = {"tm2": (("EZ", "X"), ("EZ", "Y"), ("HX", "Y"), ("HY", "X")),
                 "te2": (("EX", "Y"), ("EY", "X"), ("HZ", "X"), ("HZ", "Y"))}[mode]
        for comp, ax in pairs:
            shp = (P, ny) if ax == "X" else (nx, P)
            setattr(s, "PSI_%s_%sLO" % (comp, ax), z(*shp))
            setattr(s, "PSI_%s_%sHI" % (comp, ax), z(*shp))
        s.dft = {k: z(nf, ny) for k in ("E1r", "E1i", "H1r", "H1i", "E2r", "E2i", "H2r", "H2i")}
        s.src_box = (src_field, src_lo[0], src_lo[1], src_hi[0], src_hi[1])
    return s


def dft_complex(s, port, comp):
    """Complex DFT array of one port component in the engine's comp order
    (2D: 0 = E, 1 = H; 3D: 0 = Ex, 1 = Ey, 2 = Hx, 3 = Hy)."""
    p = str(port + 1)
    if s.mode == "yee3d":
        key = ("EX", "EY", "HX", "HY")[comp] + p
    else:
        key = ("E", "H")[comp] + p
    return s.dft[key + "r"] + 1j * s.dft[key + "i"]


FIELD_BY_ID = {0: "EX", 1: "EY", 2: "EZ", 3: "HX", 4: "HY", 5: "HZ"}


def from_spec(spec, dtype=np.float64):
    """Oracle state from an engine job description (read by attribute: mode,
    shape, num_cpml, lim_lo/hi, cb, kdx, be/ce/bh/ch, db, dx, src_field id,
    src_lo/hi, j_src, port_pos, twiddles, nf) -- the same inputs the engine
    receives, cast to ``dtype``."""
    return from_arrays(spec.mode, spec.shape, spec.num_cpml, spec.lim_lo, spec.lim_hi, spec.cb, spec.kdx,
                       spec.be, spec.ce, spec.bh, spec.ch, spec.db, spec.dx, FIELD_BY_ID[spec.src_field],
                       spec.src_lo, spec.src_hi, spec.j_src, spec.port_pos, spec.twiddles, spec.nf, dtype=dtype)
