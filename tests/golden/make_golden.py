"""Generate the golden fixtures that pin the oracle to the reference itself.

Run in a container that has the reference checkout (read-only) and Numba:

    python tests/golden/make_golden.py --ref <reference checkout> [--only CASE]

For every case this script runs the reference's own, unmodified
``fdtd_main.py`` (and ``extract_sparams.py``) from
``FDTD/GPU/<solver>/s-parameter_extraction`` as a subprocess in a scratch
directory, with ``NUMBA_ENABLE_CUDASIM=1`` (Numba's CUDA simulator executes
the ``@cuda.jit`` kernels on the CPU) and a ``user_dict_<line>.pkl`` that
selects ``precision=np.float64`` and a tiny grid.  A small harness around
``runpy``:

* maps ``cuda.select_device(k)`` to device 0 (the simulator has one device;
  the TM solver hard-codes device 1, ``fdtd_main.py:45``),
* records every array passed to ``cuda.to_device`` (the reference's single
  host-to-device boundary, ``fdtd_main.py:216-261``) and, at exit, the final
  contents of the matching device arrays (fields, CPML psi, DFT
  accumulators), named by parsing the ``d<NAME> = cuda.to_device`` lines,
* stubs ``pyspeckle`` (absent here; only profile *generation* needs it, and
  the fixtures use ``mode='load'`` with profiles written by this script),
  ``skrf`` and ``matplotlib`` (absent; the ``skrf.Network`` stub records the
  S-matrix that ``extract_sparams.py`` builds).

``--setup-only`` cases stop at the reference's ``print('loop started')`` and
keep SHA-256 digests of the arrays (float32 and float64 setups at larger,
auto-conditioned sizes), pinning the setup and coefficient code.

The ``scatter_*`` cases run ``FDTD/GPU/FDTD_3D/scattering_loss/fdtd_main.py``
the same way.  That solver reads its settings from the module
``fdtd_config.py`` rather than a pickle, so the harness builds that module
from the reference's own source with a few top-level constants replaced
(grid size, tolerances), and the ``pyspeckle`` stub hands out planted
sidewall profiles (antisymmetric, so their integer parts average to exactly
zero and the reference's profile search accepts the first draw).  The
reference's ``automated_results_collection.py`` then computes the loss
alpha from the saved planes.

The outputs are ``tests/golden/<case>.npz``; nothing here runs at test time.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import pickle
import re
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SOLVER_DIR = {"tm2": "FDTD/GPU/FDTD_2D_TM/s-parameter_extraction",
              "te2": "FDTD/GPU/FDTD_2D_TE/s-parameter_extraction",
              "yee3d": "FDTD/GPU/FDTD_3D/s-parameter_extraction"}

HARNESS = r'''
import atexit, builtins, os, runpy, sys
import numpy as np
from numba import cuda
_sel = cuda.select_device
cuda.select_device = lambda dev: _sel(0)
REC = []
_to = cuda.to_device
def _rec(a, *args, **kw):
    d = _to(a, *args, **kw)
    REC.append((np.array(a, copy=True), d))
    return d
cuda.to_device = _rec
if os.environ.get("GOLDEN_CFG"):
    import json, re, types
    _over = json.loads(os.environ["GOLDEN_CFG"])
    _src = open(os.path.join(os.path.dirname(sys.argv[1]), "fdtd_config.py")).read()
    for _k, _v in _over.items():
        _src, _n = re.subn(r"^%s\s*=.*$" % _k, "%s = %r" % (_k, _v), _src, count=1, flags=re.M)
        assert _n == 1, _k
    _mod = types.ModuleType("fdtd_config")
    _mod.__file__ = "fdtd_config.py"
    sys.path.insert(0, os.path.dirname(sys.argv[1]))
    exec(compile(_src, "fdtd_config.py", "exec"), _mod.__dict__)
    sys.modules["fdtd_config"] = _mod
if os.environ.get("GOLDEN_STOP_AT_LOOP") == "1":
    _p = builtins.print
    def _print(*a, **k):
        if a and a[0] == "loop started":
            raise SystemExit(0)
        _p(*a, **k)
    builtins.print = _print
def _dump():
    out = {}
    for i, (h, d) in enumerate(REC):
        out["h2d_%03d" % i] = h
        if os.environ.get("GOLDEN_STOP_AT_LOOP") != "1":
            out["dev_%03d" % i] = np.asarray(d.copy_to_host())
    cfg = sys.modules.get("fdtd_auto_setup") or sys.modules.get("fdtd_config")
    if cfg is not None:
        for k in dir(cfg):
            v = getattr(cfg, k)
            if k.startswith("_"):
                continue
            if isinstance(v, (int, float, np.integer, np.floating)) and not isinstance(v, bool):
                out["cfg_" + k] = np.asarray(v)
        for k in ("J_SRC", "sparam_freqs", "cosE", "sinE", "cosH", "sinH"):
            if hasattr(cfg, k):
                out["cfg_" + k] = np.asarray(getattr(cfg, k))
    np.savez(os.environ["GOLDEN_OUT"], **out)
atexit.register(_dump)
script = sys.argv[1]
sys.path.insert(0, os.path.dirname(script))
sys.argv = [script] + sys.argv[2:]
runpy.run_path(script, run_name="__main__")
'''

STUB_PYSPECKLE = '''
def create_exp_1D(*a, **k):
    raise RuntimeError("pyspeckle stub: profile generation is not used by the fixtures")
def autocorrelation(*a, **k):
    raise RuntimeError("pyspeckle stub: profile generation is not used by the fixtures")
'''

STUB_PYSPECKLE_PLANTED = '''
import os
import numpy as np
_Z = np.load(os.environ["GOLDEN_PROFILES"])
_N = [0]
def create_exp_1D(n, mean, std, acl):
    v = _Z["upper" if _N[0] == 0 else "lower"]
    _N[0] += 1
    assert len(v) == n, (len(v), n)
    return v.copy()
def autocorrelation(x):
    x = np.asarray(x, dtype=np.float64) - np.mean(x)
    r = np.correlate(x, x, mode="full")[len(x) - 1:]
    return r / r[0] if r[0] != 0 else np.ones_like(r)
'''

STUB_SKRF = '''
import os
import numpy as np
class Frequency:
    def __init__(self, f):
        self.f = np.asarray(f)
    @classmethod
    def from_f(cls, f, unit="Hz"):
        return cls(f)
class Network:
    def __init__(self, frequency=None, s=None, z0=50, name=None):
        self.frequency, self.s = frequency, np.asarray(s)
        np.save(os.environ["GOLDEN_SMAT"], self.s)
    def write_touchstone(self, filename, dir, **kw):
        n = self.s.shape[1]
        open(os.path.join(dir, "%s.s%dp" % (filename, n)), "w").close()
    def plot_s_db(self, *a, **k):
        pass
    def plot_s_deg(self, *a, **k):
        pass
'''

STUB_MPL = '''
def figure(*a, **k):
    pass
def savefig(*a, **k):
    pass
def close(*a, **k):
    pass
'''


def device_names(ref, mode):
    src = open(os.path.join(ref, SOLVER_DIR[mode], "fdtd_main.py")).read()
    return re.findall(r"^(d[A-Za-z0-9_]+) = cuda\.to_device", src, flags=re.M)


def tiny_usr(ref, mode, **over):
    usr = pickle.load(open(os.path.join(ref, SOLVER_DIR[mode], "user_dict.pkl"), "rb"))
    usr = dict(usr)
    usr.update(precision=np.float64, auto_condition=False, harmonics=1.0, sparam_num_freqs=3,
               rough_toggle=False, num_lines=1, output_dir="Results", prof_dir="rough_profiles",
               feedback_at_n_percent=50)
    if mode == "yee3d":
        usr.update(num_cpml=3, buffer_zhat=2, nx_clad_wl=0.25, ny_clad_wl=0.25, points_per_wl=5,
                   sgl_wg_length=1.0e-6, port1_length=0.25e-6, port2_length=0.25e-6,
                   sgl_wg_height=0.45e-6, sgl_wg_width=0.45e-6, pitch=0.45e-6, num_flights=0.35,
                   source_condition="TE")
    else:
        usr.update(num_cpml=4, buffer_xhat=2, ny_clad_wl=0.5, points_per_wl=6, sgl_wg_length=1.2e-6,
                   port1_length=0.3e-6, port2_length=0.3e-6, sgl_wg_height=0.3e-6, pitch=0.4e-6,
                   num_flights=0.5)
    usr.update(over)
    return usr


def profile_len(usr, mode):
    sys.path.insert(0, os.path.dirname(HERE))
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from oracle import fdtd_ref
    c = fdtd_ref.autosetup(usr, mode, "r")
    if mode == "yee3d":
        return c.p2z - c.p1z, c.up, c.lp
    return c.p2x - c.p1x, c.up, c.lp


def run_case(ref, name, mode, usr, sims, extract=False, profiles_seed=None, setup_only=False):
    work = tempfile.mkdtemp(prefix="golden_%s_" % name)
    try:
        stub = os.path.join(work, "_stub")
        os.makedirs(os.path.join(stub, "matplotlib"))
        open(os.path.join(stub, "pyspeckle.py"), "w").write(STUB_PYSPECKLE)
        open(os.path.join(stub, "skrf.py"), "w").write(STUB_SKRF)
        open(os.path.join(stub, "matplotlib", "__init__.py"), "w").write("")
        open(os.path.join(stub, "matplotlib", "pyplot.py"), "w").write(STUB_MPL)
        harness = os.path.join(work, "_harness.py")
        open(harness, "w").write(HARNESS)
        out = {"usr_json": np.array(json.dumps({k: (v.__name__ if isinstance(v, type) else v)
                                                for k, v in usr.items()}))}
        if profiles_seed is not None:
            n, up, lp = profile_len(usr, mode)
            rng = np.random.default_rng(profiles_seed)
            upper = 1.4 * rng.standard_normal(n)
            lower = 1.4 * rng.standard_normal(n)
            os.makedirs(os.path.join(work, usr["prof_dir"]), exist_ok=True)
            np.save(os.path.join(work, up + ".npy"), upper)
            np.save(os.path.join(work, lp + ".npy"), lower)
            out["profile_upper"], out["profile_lower"] = upper, lower
        names = [n[1:] for n in device_names(ref, mode)]
        script = os.path.join(ref, SOLVER_DIR[mode], "fdtd_main.py")
        for (line, direction, kind) in sims:
            pickle.dump(usr, open(os.path.join(work, "user_dict_%d.pkl" % line), "wb"))
            rec = os.path.join(work, "_rec.npz")
            env = dict(os.environ, PYTHONPATH=stub, NUMBA_ENABLE_CUDASIM="1", GOLDEN_OUT=rec,
                       GOLDEN_STOP_AT_LOOP="1" if setup_only else "0")
            r = subprocess.run([sys.executable, harness, script, str(line), direction, kind],
                               cwd=work, env=env, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError("reference run failed:\n" + r.stdout[-2000:] + r.stderr[-4000:])
            z = np.load(rec)
            tag = "%d%s%s" % (line, direction, kind)
            for k in z.files:
                if k.startswith("cfg_"):
                    out["%s/%s" % (tag, k)] = z[k]
            for i, nm in enumerate(names):
                h = z["h2d_%03d" % i]
                d = None if setup_only else z["dev_%03d" % i]
                if setup_only:
                    out["%s/sha_h2d_%s" % (tag, nm)] = np.array(hashlib.sha256(np.ascontiguousarray(h).tobytes()).hexdigest())
                    out["%s/dtype_%s" % (tag, nm)] = np.array(str(h.dtype))
                    out["%s/shape_%s" % (tag, nm)] = np.array(h.shape)
                    if h.ndim == 1 and h.size <= 4096:
                        out["%s/h2d_%s" % (tag, nm)] = h
                else:
                    if np.any(h):
                        out["%s/h2d_%s" % (tag, nm)] = h
                    out["%s/dev_%s" % (tag, nm)] = d
            if setup_only:
                for k in ("cfg_J_SRC", "cfg_sparam_freqs"):
                    v = z[k]
                    out["%s/sha_%s" % (tag, k)] = np.array(hashlib.sha256(np.ascontiguousarray(v).tobytes()).hexdigest())
                    del out["%s/%s" % (tag, k)]
            res = os.path.join(work, usr["output_dir"])
            if not setup_only and os.path.isdir(res):
                for f in sorted(os.listdir(res)):
                    if f.endswith(".npy"):
                        out["%s/npy_%s" % (tag, f[:-4])] = np.load(os.path.join(res, f))
        if extract:
            smat = os.path.join(work, "_smat.npy")
            env = dict(os.environ, PYTHONPATH=stub, NUMBA_ENABLE_CUDASIM="1", GOLDEN_SMAT=smat,
                       GOLDEN_OUT=os.path.join(work, "_rec_x.npz"), GOLDEN_STOP_AT_LOOP="0")
            xs = os.path.join(ref, SOLVER_DIR[mode], "extract_sparams.py")
            r = subprocess.run([sys.executable, harness, xs, "0", "f", "r"], cwd=work, env=env,
                               capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError("extract_sparams failed:\n" + r.stdout[-2000:] + r.stderr[-4000:])
            out["S_mat"] = np.load(smat)
        dst = os.path.join(HERE, name + ".npz")
        np.savez_compressed(dst, **out)
        print("wrote", dst, os.path.getsize(dst), "bytes", flush=True)
    finally:
        shutil.rmtree(work, ignore_errors=True)


FOUR = [(0, "f", "i"), (0, "f", "r"), (0, "b", "i"), (0, "b", "r")]

SCATTER_DIR = "FDTD/GPU/FDTD_3D/scattering_loss"
# A grid of 16 x 20 x 30 cells and 82 steps: f0, materials, CPML grading and
# the source are the reference's defaults; the guide is 0.3 x 0.6 x 1.5 um
SCATTER_TINY = dict(sgl_wg_length=1.5e-6, sgl_wg_width=0.6e-6, sgl_wg_height=0.3e-6, port1_length=0.3e-6,
                    port2_length=0.0, tol_std=1.0e9, tol_acl=1.0e9, points_per_wl=6, num_cpml=3, buffer_zhat=2,
                    nx_clad_wl=0.25, ny_clad_wl=0.25, num_flights=1.0)


def planted_profile(rng, n):
    """Antisymmetric offsets (cells): the integer parts sum to zero."""
    h = 1.6 * rng.standard_normal((n + 1) // 2)
    v = np.concatenate([h, -h])[:n]
    if n % 2:
        v[-1] = 0.0
    return rng.permutation(v)


def run_scatter_case(ref, name, over, seed):
    """The reference's scattering-loss run and its loss extraction, tiny grid, float32."""
    work = tempfile.mkdtemp(prefix="golden_%s_" % name)
    try:
        stub = os.path.join(work, "_stub")
        os.makedirs(os.path.join(stub, "matplotlib"))
        open(os.path.join(stub, "pyspeckle.py"), "w").write(STUB_PYSPECKLE_PLANTED)
        open(os.path.join(stub, "matplotlib", "__init__.py"), "w").write("")
        open(os.path.join(stub, "matplotlib", "pyplot.py"), "w").write(STUB_MPL)
        harness = os.path.join(work, "_harness.py")
        open(harness, "w").write(HARNESS)
        over = dict(SCATTER_TINY, **over)
        sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
        from oidt_b200 import scatter
        n_eff = scatter.n_eff(scatter.config(**over))
        rng = np.random.default_rng(seed)
        upper, lower = planted_profile(rng, n_eff), planted_profile(rng, n_eff)
        prof = os.path.join(work, "_profiles.npz")
        np.savez(prof, upper=upper, lower=lower)
        out = {"over_json": np.array(json.dumps(over)), "profile_upper": upper, "profile_lower": lower}
        src = open(os.path.join(ref, SCATTER_DIR, "fdtd_main.py")).read()
        names = [n[1:] for n in re.findall(r"^(d[A-Za-z0-9_]+) = cuda\.to_device", src, flags=re.M)]
        env = dict(os.environ, PYTHONPATH=stub, NUMBA_ENABLE_CUDASIM="1", GOLDEN_OUT=os.path.join(work, "_rec.npz"),
                   GOLDEN_STOP_AT_LOOP="0", GOLDEN_CFG=json.dumps(over), GOLDEN_PROFILES=prof)
        r = subprocess.run([sys.executable, harness, os.path.join(ref, SCATTER_DIR, "fdtd_main.py")], cwd=work,
                           env=env, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("reference run failed:\n" + r.stdout[-2000:] + r.stderr[-4000:])
        z = np.load(os.path.join(work, "_rec.npz"))
        for k in z.files:
            if k.startswith("cfg_"):
                out[k] = z[k]
        for i, nm in enumerate(names):
            h = z["h2d_%03d" % i]
            if np.any(h):
                out["h2d_" + nm] = h
            out["dev_" + nm] = z["dev_%03d" % i]
        res = os.path.join(work, "Results")
        for f in sorted(os.listdir(res)):
            if f.endswith(".npy"):
                out["npy_" + f[:-4]] = np.load(os.path.join(res, f))
        env["GOLDEN_OUT"] = os.path.join(work, "_rec_c.npz")
        r = subprocess.run([sys.executable, harness, os.path.join(ref, SCATTER_DIR, "automated_results_collection.py")],
                           cwd=work, env=env, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("results collection failed:\n" + r.stdout[-2000:] + r.stderr[-4000:])
        out["results"] = np.load(os.path.join(res, "results_3D_%s.npy" % over.get("source_condition", "TE")))
        dst = os.path.join(HERE, name + ".npz")
        np.savez_compressed(dst, **out)
        print("wrote", dst, os.path.getsize(dst), "bytes", flush=True)
    finally:
        shutil.rmtree(work, ignore_errors=True)


def cases(ref):
    c = {}
    c["tm2_smooth"] = lambda: run_case(ref, "tm2_smooth", "tm2", tiny_usr(ref, "tm2"), FOUR, extract=True)
    c["tm2_rough2"] = lambda: run_case(ref, "tm2_rough2", "tm2",
                                       tiny_usr(ref, "tm2", num_lines=2, rough_toggle=True),
                                       [(1, "f", "r")], profiles_seed=11)
    c["tm2_lines2"] = lambda: run_case(ref, "tm2_lines2", "tm2", tiny_usr(ref, "tm2", num_lines=2),
                                       FOUR + [(1, d, k) for (_, d, k) in FOUR], extract=True)
    c["te2_smooth"] = lambda: run_case(ref, "te2_smooth", "te2", tiny_usr(ref, "te2"), FOUR, extract=True)
    c["te2_rough2"] = lambda: run_case(ref, "te2_rough2", "te2",
                                       tiny_usr(ref, "te2", num_lines=2, rough_toggle=True),
                                       [(1, "b", "r")], profiles_seed=12)
    c["yee3d_smooth"] = lambda: run_case(ref, "yee3d_smooth", "yee3d", tiny_usr(ref, "yee3d"), FOUR, extract=True)
    c["yee3d_rough2_tm"] = lambda: run_case(ref, "yee3d_rough2_tm", "yee3d",
                                            tiny_usr(ref, "yee3d", num_lines=2, rough_toggle=True,
                                                     source_condition="TM"),
                                            [(1, "f", "r")], profiles_seed=13)
    # Setup-only pins at auto-conditioned sizes, float32 and float64.
    for mode in ("tm2", "te2", "yee3d"):
        for prec in (np.float32, np.float64):
            nm = "setup_%s_%s" % (mode, np.dtype(prec).name)
            def mk(mode=mode, prec=prec, nm=nm):
                usr = pickle.load(open(os.path.join(ref, SOLVER_DIR[mode], "user_dict.pkl"), "rb"))
                usr = dict(usr, precision=prec, sparam_num_freqs=7, rough_toggle=False, feedback_at_n_percent=50)
                if mode == "yee3d":
                    # pitch 0.4 um: the reference's auto-setup requires a cladding buffer of at least
                    # half the waveguide pitch (fdtd_auto_setup.py:121-122); port lengths whose cell
                    # counts carry when summed: its incident runs set the guide length to
                    # port1 + port2 and require p2z > p1z (fdtd_auto_setup.py:88-89, 168-171)
                    usr.update(num_lines=1, sgl_wg_length=1.0e-6, port1_length=0.21e-6, port2_length=0.21e-6,
                               nx_clad_wl=0.5, ny_clad_wl=0.5, pitch=0.4e-6)
                run_case(ref, nm, mode, usr, [(0, "f", "r"), (0, "b", "i")], setup_only=True)
            c[nm] = mk
    c["scatter_analytic"] = lambda: scatter_analytic(ref)
    c["scatter_te"] = lambda: run_scatter_case(ref, "scatter_te", dict(source_condition="TE"), seed=21)
    # the 'TM' (Hy) source box is 4 cells narrower in x than the guide: a 6-cell-high guide
    c["scatter_tm"] = lambda: run_scatter_case(ref, "scatter_tm", dict(source_condition="TM", sgl_wg_height=0.45e-6),
                                               seed=22)
    c["zwave_tm"] = lambda: run_zwave_case(ref, "zwave_tm", dict(source_condition="TM", sgl_wg_height=0.45e-6))
    c["zwave_te"] = lambda: run_zwave_case(ref, "zwave_te", dict(source_condition="TE"))
    return c


ZWAVE_DIR = "FDTD/GPU/FDTD_3D/wave_impedance"


def run_zwave_case(ref, name, over):
    """The reference's wave-impedance run (smooth guide, float32, tiny grid):
    its device arrays, including the [nt, nx] line records, and saved records."""
    work = tempfile.mkdtemp(prefix="golden_%s_" % name)
    try:
        stub = os.path.join(work, "_stub")
        os.makedirs(os.path.join(stub, "matplotlib"))
        open(os.path.join(stub, "pyspeckle.py"), "w").write(STUB_PYSPECKLE)
        open(os.path.join(stub, "matplotlib", "__init__.py"), "w").write("")
        open(os.path.join(stub, "matplotlib", "pyplot.py"), "w").write(STUB_MPL)
        harness = os.path.join(work, "_harness.py")
        open(harness, "w").write(HARNESS)
        over = dict(SCATTER_TINY, rough_toggle=False, **over)
        out = {"over_json": np.array(json.dumps(over))}
        src = open(os.path.join(ref, ZWAVE_DIR, "fdtd_main.py")).read()
        names = [n[1:] for n in re.findall(r"^(d[A-Za-z0-9_]+) = cuda\.to_device", src, flags=re.M)]
        env = dict(os.environ, PYTHONPATH=stub, NUMBA_ENABLE_CUDASIM="1", GOLDEN_OUT=os.path.join(work, "_rec.npz"),
                   GOLDEN_STOP_AT_LOOP="0", GOLDEN_CFG=json.dumps(over))
        r = subprocess.run([sys.executable, harness, os.path.join(ref, ZWAVE_DIR, "fdtd_main.py")], cwd=work,
                           env=env, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("reference run failed:\n" + r.stdout[-2000:] + r.stderr[-4000:])
        z = np.load(os.path.join(work, "_rec.npz"))
        for k in z.files:
            if k.startswith("cfg_"):
                out[k] = z[k]
        for i, nm in enumerate(names):
            h = z["h2d_%03d" % i]
            if np.any(h):
                out["h2d_" + nm] = h
            out["dev_" + nm] = z["dev_%03d" % i]
        res = os.path.join(work, "Results")
        for f in sorted(os.listdir(res)):
            if f.endswith(".npy"):
                out["npy_" + f[:-4]] = np.load(os.path.join(res, f))
        dst = os.path.join(HERE, name + ".npz")
        np.savez_compressed(dst, **out)
        print("wrote", dst, os.path.getsize(dst), "bytes", flush=True)
    finally:
        shutil.rmtree(work, ignore_errors=True)


def scatter_analytic(ref):
    """The reference's Payne-Lacey slab estimates (``analysis.py``
    ``find_alpha_te`` / ``find_alpha_tm`` with ``aux_funcs.find_neff``) on a
    grid of sigma and Lc.  ``analysis.py`` runs its analysis at import, so
    only those function definitions are taken from its source (``ast``) and
    executed with the reference's settings module values they read."""
    import ast
    import types
    from scipy.optimize import fsolve

    d = os.path.join(ref, SCATTER_DIR)

    def defs(fname, names, ns):
        tree = ast.parse(open(os.path.join(d, fname)).read())
        body = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in names]
        assert len(body) == len(names), fname
        exec(compile(ast.Module(body=body, type_ignores=[]), fname, "exec"), ns)
        return ns

    aux = defs("aux_funcs.py", ("find_neff",), {"np": np, "fsolve": fsolve})
    cfg = types.SimpleNamespace(f0=194.8e12, eps_rel_bg=1.5 ** 2, eps_rel_fg=3.5 ** 2 / 1.5 ** 2)
    an = defs("analysis.py", ("find_alpha_te", "find_alpha_tm"),
              {"np": np, "aux": types.SimpleNamespace(find_neff=aux["find_neff"]), "cfg": cfg})
    rows = []
    for s_nm in (5, 10, 15, 30):
        for lc_nm in (50, 300, 700, 1500):
            rows.append([s_nm, lc_nm, *an["find_alpha_te"](s_nm * 1e-9, lc_nm * 1e-9),
                         *an["find_alpha_tm"](s_nm * 1e-9, lc_nm * 1e-9)])
    dst = os.path.join(HERE, "scatter_analytic.npz")
    np.savez_compressed(dst, table=np.array(rows, dtype=np.float64))
    print("wrote", dst, flush=True)


def copy_touchstone_examples(ref):
    """The reference's example touchstone outputs (format pins)."""
    for rel, dst in (("FDTD/GPU/FDTD_3D/s-parameter_extraction/Results/example.s2p", "ref_example_3d.s2p"),
                     ("FDTD/GPU/FDTD_2D_TM/s-parameter_extraction/Results/example.s4p", "ref_example_tm2.s4p")):
        shutil.copyfile(os.path.join(ref, rel), os.path.join(HERE, dst))
        print("copied", dst, flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="root of the reference checkout (read only)")
    ap.add_argument("--only", nargs="*")
    a = ap.parse_args()
    cs = cases(a.ref)
    cs["touchstone"] = lambda: copy_touchstone_examples(a.ref)
    for k, fn in cs.items():
        if a.only and k not in a.only:
            continue
        print("case", k, flush=True)
        fn()


if __name__ == "__main__":
    main()
