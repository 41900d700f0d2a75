"""Synthetic waveguide workloads with explicit grid sizes.

The reference only builds grids from physical lengths (``fdtd_auto_setup``);
these builders place the same structures (slab / strip cores, CPML, soft
source, two port planes) on grids of a given cell count, which is how the
benchmark workloads are stated:

* ``slab2d``   2D TMz symmetric slab (400 x 200 cells, 20 nm, 2000 steps)
* ``strip3d``  3D silicon strip with rough sidewalls (256 x 128 x 128 cells
               along x, 20 nm, 4000 steps; uneven batched grids), or with
               ``slab_y_nm`` an etched rib (the 151 M cell run at 15 nm)

Axis convention is the reference's 3D one: z is the propagation axis and the
contiguous array axis, x carries the roughened core faces and y the other
transverse direction.  Coefficients are computed in float64 and rounded once
when a float32 job is created.

Roughness: each sidewall offset sequence is a stationary Gaussian process
with standard deviation sigma and exponential autocorrelation
exp(-|dz|/Lc), generated as the AR(1) recursion
``x[n] = rho x[n-1] + sqrt(1 - rho^2) sigma w[n]`` with rho = exp(-dz/Lc)
(the exact discretisation of an Ornstein-Uhlenbeck process), then rounded to
whole cells.  The reference draws its profiles with pyspeckle's
``create_exp_1D`` (same target statistics) and accepts them by rejection;
this generator replaces that step, so profiles are inputs here.
"""
from __future__ import annotations

import numpy as np

from .refsetup import cpml_profiles, kappa_axis, staggered_eps, twiddles
from .spec import FIELD_ID, SimSpec

C0 = 3.0e8            # the reference's eps0 = 1/(36 pi 1e9) gives exactly this
EPS0 = 1.0 / (36.0e9 * np.pi)
MU0 = 4.0e-7 * np.pi
PEC_RIM = 2


def sidewall_profile(n: int, sigma_cells: float, lc_cells: float, rng: np.random.Generator,
                     round_cells: bool = True) -> np.ndarray:
    """Gaussian offsets with exponential autocorrelation (AR(1)), in cells."""
    rho = np.exp(-1.0 / lc_cells)
    w = rng.standard_normal(n)
    x = np.empty(n)
    x[0] = sigma_cells * w[0]
    a = np.sqrt(1.0 - rho * rho) * sigma_cells
    for k in range(1, n):
        x[k] = rho * x[k - 1] + a * w[k]
    return np.rint(x) if round_cells else x


def wave_packet(nt: int, dt: float, f0: float, bw: float, amp: float = 5.0) -> np.ndarray:
    """The reference's wave-packet source (source_type 2,
    fdtd_auto_setup.py:126-157): Gaussian envelope of spread
    2 sqrt(ln 2) / (bw 2 pi f0), peak at 9 spreads, carrier cos(2 pi f0 t)."""
    tsp = 2 * np.sqrt(np.log(2)) / (bw * 2 * np.pi * f0)
    tpk = 9 * tsp
    t = np.arange(nt) * dt
    return amp * np.exp(-0.5 * ((t - tpk) / tsp) ** 2) * np.cos(2 * np.pi * f0 * (t - tpk))


def _freqs(lmin_nm, lmax_nm, nf):
    return np.linspace(C0 / (lmax_nm * 1e-9), C0 / (lmin_nm * 1e-9), nf)


def slab2d(nx=400, ny=200, dx=20e-9, P=10, n_core=3.48, n_clad=1.44, core_cells=10, src_x=40,
           ports=(60, 340), steps=2000, nf=21, lam=(1450.0, 1650.0), lam0=1550.0, bw=0.5,
           courant=0.99, m_grade=3, kappa_max=5, alpha_max=0.05, precision=np.float64,
           direction="f", rough=False, sigma_nm=10.0, lc_nm=50.0, seed=0) -> SimSpec:
    """2D TMz symmetric slab along x (Ez, Hx, Hy), the 400 x 200 benchmark case.

    ``rough=True`` moves both slab faces between the ports by seeded
    sidewall offsets (served 2D jobs)."""
    eps_bg = n_clad ** 2
    eps = eps_bg * EPS0
    eta = np.sqrt(MU0 / eps)
    c_bg = 1 / np.sqrt(eps * MU0)
    dt = courant * dx / (c_bg * np.sqrt(2))
    by = (ny - core_cells) // 2
    lo = np.zeros(nx)
    up = np.zeros(nx)
    if rough:
        rng = np.random.default_rng(seed)
        s_, l_ = sigma_nm * 1e-9 / dx, lc_nm * 1e-9 / dx
        up[ports[0]:ports[1]] = sidewall_profile(ports[1] - ports[0], s_, l_, rng)
        lo[ports[0]:ports[1]] = sidewall_profile(ports[1] - ports[0], s_, l_, rng)
    jj = np.arange(ny)[None, :]
    mask = (jj >= (by + lo[:, None])) & (jj < (by + core_cells + up[:, None]))
    eps_cell = eps * ((n_core ** 2 / eps_bg) * mask + 1 * ~mask)
    prec = np.float64
    cb = {"z": dt / eps_cell}
    tab = cpml_profiles(P, dx, dt, eps, eta, prec, m_grade=m_grade, kappa_max=kappa_max, alpha_max=alpha_max)
    kdx = {}
    for a, (n, name) in enumerate(((nx, "x"), (ny, "y"))):
        kdx[name + "e"], kdx[name + "h"] = kappa_axis(n, PEC_RIM, n - PEC_RIM, P, tab["ke"], tab["kh"], dx, prec)
    freqs = _freqs(*lam, nf)
    x = src_x if direction == "f" else nx - src_x - 1
    return SimSpec(
        mode="tm2", precision=np.dtype(precision), shape=(nx, ny), num_cpml=P,
        lim_lo=(PEC_RIM, PEC_RIM), lim_hi=(nx - PEC_RIM, ny - PEC_RIM), cb=cb, kdx=kdx,
        be=tab["be"], ce=tab["ce"], bh=tab["bh"], ch=tab["ch"], db=dt / MU0, dx=dx,
        src_field=FIELD_ID["EZ"], src_lo=(x, by + 1, 0), src_hi=(x + 1, by + core_cells - 1, 1),
        j_src=wave_packet(steps, dt, C0 / (lam0 * 1e-9), bw), port_pos=tuple(ports),
        win_lo=(0, P), win_hi=(1, ny - P), freqs=freqs, twiddles=twiddles(freqs, dt, steps), nt=steps,
        meta=dict(workload="slab2d", dt=dt, power_window=(P, ny - P), core_mask=mask))


def strip3d(nx=128, ny=128, nz=256, dx=20e-9, P=10, n_core=3.48, n_clad=1.44, core_x_nm=220.0,
            core_y_nm=500.0, src_gap=10, port_gap=20, steps=4000, nf=41, lam=(1450.0, 1650.0),
            lam0=1550.0, bw=0.5, courant=0.99, sigma_nm=10.0, lc_nm=50.0, seed=0, rough=True,
            source="TE", m_grade=3, kappa_max=5, alpha_max=0.05, precision=np.float32,
            slab_y_nm=0.0) -> SimSpec:
    """3D strip (or rib) along z with sidewall roughness on the x-faces.

    The core is centred; ``core_x_nm`` is its extent along x (the roughened
    faces, the reference's ``sgl_wg_height``) and ``core_y_nm`` along y (the
    reference's ``sgl_wg_width``).  The source sheet ('TE': Ey, 'TM': Hy)
    sits ``src_gap`` cells inside the z-CPML, ports ``port_gap`` cells past the
    source and mirrored at the far end; roughness spans the guide between the
    ports.

    ``slab_y_nm`` > 0 makes a rib: a core-index slab of that thickness along
    y, level with the bottom of the core and spanning the whole x extent (into
    the CPML, which absorbs its slab modes), under a ridge of ``core_x_nm``
    by ``core_y_nm`` total height whose x-faces carry the roughness -- an
    etched-rib silicon guide with rough rib sidewalls.
    """
    eps_bg = n_clad ** 2
    eps = eps_bg * EPS0
    eta = np.sqrt(MU0 / eps)
    c_bg = 1 / np.sqrt(eps * MU0)
    dt = courant * dx / (c_bg * np.sqrt(3))
    cx = max(1, int(round(core_x_nm * 1e-9 / dx)))
    cy = max(1, int(round(core_y_nm * 1e-9 / dx)))
    bx, by = (nx - cx) // 2, (ny - cy) // 2
    sz = P + src_gap
    p1, p2 = sz + port_gap, nz - sz - port_gap
    if p2 <= p1 + 1:
        raise ValueError("grid too short for source and port gaps")
    lo = np.zeros(nz)
    up = np.zeros(nz)
    if rough:
        rng = np.random.default_rng(seed)
        s, l = sigma_nm * 1e-9 / dx, lc_nm * 1e-9 / dx
        up[p1:p2] = sidewall_profile(p2 - p1, s, l, rng)
        lo[p1:p2] = sidewall_profile(p2 - p1, s, l, rng)
    ii = np.arange(nx)[:, None]
    face = (ii >= (bx + lo[None, :])) & (ii < (bx + cx + up[None, :]))  # [nx, nz]
    jin = np.zeros(ny, dtype=bool)
    jin[by:by + cy] = True
    mask = face[:, None, :] & jin[None, :, None]
    cs = 0
    if slab_y_nm > 0:
        cs = min(cy, max(1, int(round(slab_y_nm * 1e-9 / dx))))
        mask[:, by:by + cs, :] = True
    eps_cell = eps * ((n_core ** 2 / eps_bg) * mask + 1 * ~mask)
    prec = np.float64
    ex, ey, ez = staggered_eps(eps_cell, prec, (0, 1, 2))
    cb = {"x": dt / ex, "y": dt / ey, "z": dt / ez}
    two = np.array([False, True])
    mat_idx, mat_tab = material_index(mask, eps * ((n_core ** 2 / eps_bg) * two + 1 * ~two), dt)
    tab = cpml_profiles(P, dx, dt, eps, eta, prec, m_grade=m_grade, kappa_max=kappa_max, alpha_max=alpha_max)
    kdx = {}
    for n, name in ((nx, "x"), (ny, "y"), (nz, "z")):
        kdx[name + "e"], kdx[name + "h"] = kappa_axis(n, PEC_RIM, n - PEC_RIM, P, tab["ke"], tab["kh"], dx, prec)
    if source == "TE":
        fld, slo, shi = "EY", (bx + 1, by + 1, sz), (bx + cx - 1, by + cy - 1, sz + 2)
    else:
        fld, slo, shi = "HY", (bx + 2, by + 2, sz), (bx + cx - 2, by + cy - 2, sz + 2)
    freqs = _freqs(*lam, nf)
    return SimSpec(
        mode="yee3d", precision=np.dtype(precision), shape=(nx, ny, nz), num_cpml=P,
        lim_lo=(PEC_RIM,) * 3, lim_hi=(nx - PEC_RIM, ny - PEC_RIM, nz - PEC_RIM), cb=cb, kdx=kdx,
        be=tab["be"], ce=tab["ce"], bh=tab["bh"], ch=tab["ch"], db=dt / MU0, dx=dx,
        src_field=FIELD_ID[fld], src_lo=slo, src_hi=shi,
        j_src=wave_packet(steps, dt, C0 / (lam0 * 1e-9), bw), port_pos=(p1, p2),
        win_lo=(P, P), win_hi=(nx - P, ny - P), freqs=freqs, twiddles=twiddles(freqs, dt, steps), nt=steps,
        meta=dict(workload="rib3d" if cs else "strip3d", dt=dt, seed=seed, sigma_nm=sigma_nm, lc_nm=lc_nm,
                  rough=rough, power_window=((P, nx - P), (P, ny - P)), core=(bx, by, cx, cy), slab_cells=cs),
        mat_idx=mat_idx, mat_tab=mat_tab)


def material_index(mask: np.ndarray, eps_vals: np.ndarray, dt: float):
    """The dt/eps grids of a two-material 3D grid as a one-byte index and a
    table, equal to ``dt / staggered_eps(eps_cell)`` cell by cell.

    Every component's permittivity is a 2-point average of the cell and its
    lower neighbour along the component's axis on cells with all indices >= 1,
    the cell's own value on the first layer (``refsetup.staggered_eps``).  So
    a cell's (CBX, CBY, CBZ) depends only on the material of the cell and of
    its three lower neighbours, or on the cell alone on the first layer: at
    most 18 codes.  ``eps_vals`` = (cladding, core) permittivity as the
    permittivity grid holds them; the table entries repeat the grid's float64
    operations, so they equal the grids' values bit for bit.  Returns
    (idx uint8 [nx][ny][nz], tab float64 [nmat][3])."""
    m = mask.astype(np.uint8)
    code = (17 + m).astype(np.uint8)  # first layer: the cell's own material
    inner = (slice(1, None),) * 3
    code[inner] = 1 + m[1:, 1:, 1:] + 2 * m[:-1, 1:, 1:] + 4 * m[1:, :-1, 1:] + 8 * m[1:, 1:, :-1]
    present = np.nonzero(np.bincount(code.ravel(), minlength=19))[0]
    lut = np.zeros(19, dtype=np.uint8)
    lut[present] = np.arange(len(present), dtype=np.uint8)
    E = np.asarray(eps_vals, dtype=np.float64)
    tab = np.empty((len(present), 3))
    for q, c in enumerate(present):
        if c >= 17:
            e = np.full(3, E[c - 17])
        else:
            b = c - 1
            own = E[b & 1]
            e = np.array([0.5 * (own + E[(b >> s) & 1]) for s in (1, 2, 3)])
        tab[q] = dt / e
    return lut[code], tab


def with_smooth(spec_kwargs: dict) -> dict:
    """Keyword set for the incident run of a rough strip: same grid, smooth."""
    k = dict(spec_kwargs)
    k["rough"] = False
    return k


def batch_configs(n=64, master_seed=0, steps=3000):
    """The batched stochastic set: per realization sigma ~ U(5, 15) nm,
    Lc ~ U(30, 100) nm, nz ~ U{160..320}, nx, ny in {96, 112, 128}, drawn from
    one seeded PCG64 stream; realization r uses roughness seed r."""
    rng = np.random.default_rng(master_seed)
    out = []
    for r in range(n):
        out.append(dict(nx=int(rng.choice([96, 112, 128])), ny=int(rng.choice([96, 112, 128])),
                        nz=int(rng.integers(160, 321)), sigma_nm=float(rng.uniform(5, 15)),
                        lc_nm=float(rng.uniform(30, 100)), seed=r, steps=steps))
    return out


def serving_mix(rate_hz=20.0, duration_s=60.0, seed=0):
    """Poisson arrivals of mixed 2D/3D roughness jobs (70 % 2D TMz with
    x ~ U[300, 800], y ~ U[150, 300]; 30 % 3D with z ~ U[160, 384] along the
    guide and x, y ~ U[96, 160]); sigma 5-15 nm, Lc 30-100 nm, 2000-4000
    steps.  Returns a list of (arrival_time_s, kwargs-dict with 'kind')."""
    rng = np.random.default_rng(seed)
    t, jobs = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate_hz)
        if t >= duration_s:
            break
        steps = int(rng.integers(2000, 4001))
        sig, lc, s = float(rng.uniform(5, 15)), float(rng.uniform(30, 100)), int(rng.integers(0, 2 ** 31))
        if rng.random() < 0.7:
            jobs.append((t, dict(kind="2d", nx=int(rng.integers(300, 801)), ny=int(rng.integers(150, 301)),
                                 steps=steps, sigma_nm=sig, lc_nm=lc, seed=s)))
        else:
            jobs.append((t, dict(kind="3d", nz=int(rng.integers(160, 385)), nx=int(rng.integers(96, 161)),
                                 ny=int(rng.integers(96, 161)), steps=steps, sigma_nm=sig, lc_nm=lc, seed=s)))
    return jobs
