"""S-parameters from port DFTs, and the touchstone files SROPEE reads.

* :func:`extract_sparams` -- the reference's 4-simulations-per-line
  extraction (``FDTD_2D_TM/.../extract_sparams.py:48-104``,
  ``FDTD_3D/.../extract_sparams.py:48-131``) on the saved DFT arrays.
* :func:`forward_s` -- S11 / S21 from one incident and one reflected run
  (the two runs the forward protocol needs), summed over a power window;
  :func:`forward_s_device` -- the same with the sums reduced on the device.
* :func:`write_touchstone` / :func:`read_touchstone` -- RI-format ``.sNp`` in
  the layout the reference's scikit-rf 0.18 writer produces
  (``extract_sparams.py:106-117``), with the OIDT comment line first.

The S ratio is evaluated in complex128.
"""
from __future__ import annotations

import numpy as np

from .refsetup import derive
from .spec import power_window

OIDT_ACK = ("!This S-parameter file was generated as part of the OIDT. This project was completed as part of "
            "research conducted with my major professor and advisor, Prof. Ata Zadehgol, at the Applied and "
            "Computational Electromagnetics Signal and Power Integrity (ACEM-SPI) Lab while working toward the "
            "Ph.D. in Electrical Engineering at the University of Idaho, Moscow, Idaho, USA. This project was "
            "funded, in part, by the National Science Foundation (NSF); award #1816542 [1].\n")


def power_density(mode: str, comps):
    """Complex Poynting flux through the port plane.

    2D TM ``-1/2 Ez Hy*``, 2D TE ``+1/2 Ey Hz*`` (extract_sparams.py:88-89),
    3D ``1/2 (Ex Hy* - Ey Hx*)`` (FDTD_3D/.../extract_sparams.py:114-115)."""
    if mode == "tm2":
        return -0.5 * (comps[0] * np.conjugate(comps[1]))
    if mode == "te2":
        return 0.5 * (comps[0] * np.conjugate(comps[1]))
    return 0.5 * (comps[0] * np.conjugate(comps[3]) - comps[1] * np.conjugate(comps[2]))


def _window_power(spec, sav):
    w = power_window(spec)
    if spec.mode == "yee3d":
        (i0, i1), (j0, j1) = w
        return sav[:, i0:i1, j0:j1].sum(axis=(1, 2))
    j0, j1 = w
    return sav[:, j0:j1].sum(axis=1)


def forward_s(spec, inc: dict, ref: dict) -> dict:
    """S11 = sqrt(P[ref - inc at port 1] / P[inc at port 1]) and
    S21 = sqrt(P[ref at port 2] / P[inc at port 1]); ``inc``/``ref`` map
    (port, comp) to complex DFT arrays of the incident (smooth) and reflected
    (device under test) runs."""
    nc = 4 if spec.mode == "yee3d" else 2
    a1 = [np.asarray(inc[(0, c)], dtype=np.complex128) for c in range(nc)]
    r1 = [np.asarray(ref[(0, c)], dtype=np.complex128) - a1[c] for c in range(nc)]
    t2 = [np.asarray(ref[(1, c)], dtype=np.complex128) for c in range(nc)]
    p_inc = _window_power(spec, power_density(spec.mode, a1))
    p_ref = _window_power(spec, power_density(spec.mode, r1))
    p_tr = _window_power(spec, power_density(spec.mode, t2))
    return {"S11": np.sqrt(p_ref / p_inc), "S21": np.sqrt(p_tr / p_inc), "P_inc": p_inc}


def forward_s_device(spec, inc_job, ref_job) -> dict:
    """:func:`forward_s` with its three power sums reduced on the device
    (``Job.port_power``, float64): the DFT planes stay in HBM and 3 x nf
    complex values cross the link.  ``inc_job`` may be ``ref_job`` itself
    (no separate incident run), as ``forward_s(spec, d, d)`` allows: the
    reflected power is then 0."""
    w = power_window(spec)
    p_inc = inc_job.port_power(0, window=w)
    p_ref = np.zeros_like(p_inc) if inc_job is ref_job else ref_job.port_power(0, minus=inc_job, window=w)
    p_tr = ref_job.port_power(1, window=w)
    return {"S11": np.sqrt(p_ref / p_inc), "S21": np.sqrt(p_tr / p_inc), "P_inc": p_inc}


def extract_sparams(usr: dict, mode: str, data: dict) -> np.ndarray:
    """S-matrix [nf, 2L, 2L] from the reference-named DFT arrays in ``data``
    (``ez_fi_l1`` ...).  2D visits pairs j >= i; 3D visits all pairs so the
    later pair wins the symmetric fill, as the two reference scripts do.
    Power is summed over one pitch around each line's core (3D: also over
    y in [P, ny - P)); the result dtype follows the reference
    (complex64 for float32 runs)."""
    dv = derive(usr, mode, "r")
    u = dv.usr
    cdt = np.complex64 if u["precision"] == np.float32 else np.complex128
    nports, nf, P = 2 * u["num_lines"], u["sparam_num_freqs"], u["num_cpml"]
    names = {"tm2": ("ez", "hy"), "te2": ("ey", "hz"), "yee3d": ("ex", "ey", "hx", "hy")}[mode]
    S = np.zeros((nf, nports, nports), dtype=cdt)
    for i in range(nports):
        for j in (range(nports) if mode == "yee3d" else range(i, nports)):
            li, lj = i // 2 + 1, j // 2 + 1
            inc_tag = ("fi", "bi")[j % 2]
            ref_tag = (("ft", "bt") if i % 2 == j % 2 else ("fr", "br"))[i % 2]
            inc = [data["%s_%s_l%d" % (n, inc_tag, lj)] for n in names]
            ref = [data["%s_%s_l%d" % (n, ref_tag, lj)] for n in names]
            if i == j:
                cor = [data["%s_%s_l%d" % (n, ("fi", "bi")[i % 2], li)] for n in names]
                ref = [r - c for r, c in zip(ref, cor)]
            s_inc, s_ref = power_density(mode, inc), power_density(mode, ref)
            if mode == "yee3d":
                c0 = dv.bx + dv.cx_swg - dv.ph
                a, b = c0 + dv.pp * (lj - 1), c0 + dv.pp * (li - 1)
                p_inc = np.zeros(nf, dtype=cdt)
                p_ref = np.zeros(nf, dtype=cdt)
                for y in range(P, dv.ny - P):  # the reference's summation order
                    for p in range(a, a + dv.pp):
                        p_inc += s_inc[:, p, y]
                    for p in range(b, b + dv.pp):
                        p_ref += s_ref[:, p, y]
            else:
                c0 = dv.by + dv.cy_swg - dv.ph
                a, b = c0 + dv.pp * (lj - 1), c0 + dv.pp * (li - 1)
                p_inc = np.zeros(nf, dtype=cdt)
                p_ref = np.zeros(nf, dtype=cdt)
                for p in range(a, a + dv.pp):
                    p_inc += s_inc[:, p]
                for p in range(b, b + dv.pp):
                    p_ref += s_ref[:, p]
            S[:, i, j] = S[:, j, i] = np.sqrt(p_ref / p_inc)
    return S


# ---------------------------------------------------------------------------
# Touchstone (RI, z0 = 50)
# ---------------------------------------------------------------------------
def touchstone_text(freqs, S, z0=50.0) -> str:
    """Text of an RI-format ``.sNp``: header, per-port column comment, one
    record per frequency (2-port: S11 S21 S12 S22 on one line; N >= 3: one
    matrix row per line, at most 4 pairs per line), then a port-impedance
    comment line, with the OIDT acknowledgement first."""
    S = np.asarray(S)
    nf, n, _ = S.shape
    lines = [OIDT_ACK, "!Created with skrf (http://scikit-rf.org).\n", "# Hz S RI R %s \n" % repr(float(z0))]
    if n == 2:
        order = [(0, 0), (1, 0), (0, 1), (1, 1)]
        lines.append("!freq " + " ".join("ReS%d%d ImS%d%d" % (a + 1, b + 1, a + 1, b + 1) for a, b in order) + "\n")
    else:
        order = None
        first = True
        for a in range(n):
            pairs = ["ReS%d%d ImS%d%d" % (a + 1, b + 1, a + 1, b + 1) for b in range(n)]
            for c in range(0, n, 3):
                lines.append(("!freq " if first else "! ") + " ".join(pairs[c:c + 3]) + "\n")
                first = False
        lines.append("!\n")
    zline = "! Port Impedance" + "".join(" %.14f %.14f" % (z0, 0.0) for _ in range(n)) + "\n"
    for k in range(nf):
        f = repr(float(freqs[k]))
        if n == 2:
            vals = []
            for a, b in order:
                vals += [repr(float(S[k, a, b].real)), repr(float(S[k, a, b].imag))]
            lines.append(f + " " + " ".join(vals) + "\n")
        else:
            for a in range(n):
                vals = []
                for b in range(n):
                    vals += [repr(float(S[k, a, b].real)), repr(float(S[k, a, b].imag))]
                for c in range(0, len(vals), 8):
                    lines.append((f if (a == 0 and c == 0) else "") + " " + " ".join(vals[c:c + 8]) + "\n")
        lines.append(zline)
    return "".join(lines)


def write_touchstone(path_stem: str, freqs, S, z0=50.0) -> str:
    """Write ``<path_stem>.s<N>p`` and return its path."""
    n = np.asarray(S).shape[1]
    path = "%s.s%dp" % (path_stem, n)
    with open(path, "w") as fh:
        fh.write(touchstone_text(freqs, S, z0))
    return path


def read_touchstone(path: str):
    """(freqs, S, z0) from an RI touchstone file written as above (or by the
    reference)."""
    n = int(path.rsplit(".s", 1)[1][:-1])
    z0 = 50.0
    nums = []
    with open(path) as fh:
        for line in fh:
            s = line.strip()
            if not s or s.startswith("!"):
                continue
            if s.startswith("#"):
                parts = s.split()
                if "R" in parts:
                    z0 = float(parts[parts.index("R") + 1])
                continue
            nums += [float(v) for v in s.split()]
    rec = 1 + 2 * n * n
    nf = len(nums) // rec
    arr = np.asarray(nums[:nf * rec]).reshape(nf, rec)
    freqs = arr[:, 0]
    vals = arr[:, 1::2] + 1j * arr[:, 2::2]
    if n == 2:
        S = np.empty((nf, 2, 2), dtype=np.complex128)
        S[:, 0, 0], S[:, 1, 0], S[:, 0, 1], S[:, 1, 1] = vals.T
    else:
        S = vals.reshape(nf, n, n)
    return freqs, S, z0
