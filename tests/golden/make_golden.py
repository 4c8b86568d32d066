"""Generates the golden vectors under tests/golden/ by running the REFERENCE
itself (chenyk1990/pywave compiled from its own sources into oracle/_ref by
`make -C oracle ref`, with zero-initialised malloc).  Needs the reference
sources, found through the PYWAVE_REF variable (the root of a pywave checkout;
read in place), and is run by hand in the build container:

    export PYWAVE_REF=<pywave checkout>
    make -C oracle ref && python tests/golden/make_golden.py [fixture ...]

With no fixture names every fixture is regenerated.  The fixtures are small
.npz files; where a reference output is too large to keep (the 3-D and
config-geometry runs), the fixture holds its SHA-256 digest, which a
bit-exact result reproduces, plus a decimated copy for diagnostics.  The
tests compare both the oracle restatement (CPU) and the CUDA path (GPU)
against them.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import importlib.util
import os
import sys

import numpy as np

from models import (APS2, APS3, VISCO, aps2_velocity, aps3_velocity, visco_case)
from models import (BIG3D, BIG3D_BAND, BIG3D_TRI_JSNAP, BUTTER_CASES, LSTRI, MID, PAS, PAS_FHI,
                    PAS_FLO, WEIGHT_CASE, big3d_velocity, digest, lstri_case, mid_models,
                    mid_wavelet, pas_case, pfwi_scale_case)

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_PY = os.path.join(os.environ.get("PYWAVE_REF", ""), "pywave")
REF_BUILD = os.path.join(ROOT, "oracle", "_ref")
sys.path.insert(0, REF_BUILD)


def load(name):
    spec = importlib.util.spec_from_file_location("ref_" + name, os.path.join(REF_PY, name + ".py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def quiet(fn, *a, **k):
    """Run a reference call with its C-level stdout chatter discarded."""
    sys.stdout.flush()
    fd = os.dup(1)
    nul = os.open(os.devnull, os.O_WRONLY)
    os.dup2(nul, 1)
    try:
        return fn(*a, **k)
    finally:
        sys.stdout.flush()
        os.dup2(fd, 1)
        os.close(nul)
        os.close(fd)


def refdrv():
    L = C.CDLL(os.path.join(REF_BUILD, "libpwref.so"))
    f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
    L.refdrv_ricker.argtypes = [C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, f32p]
    L.refdrv_gradient.argtypes = [f32p, f32p, f32p, f32p, f32p, C.c_int, f32p, f32p]
    L.refdrv_gradient_pas.argtypes = [f32p, f32p, f32p, f32p, f32p, f32p, C.c_int, C.c_float,
                                      C.c_float, f32p, f32p]
    L.refdrv_butter.argtypes = [C.c_int, C.c_float, C.c_int, C.c_int, f32p]
    L.refdrv_forward_visco.argtypes = [f32p] * 5
    L.refdrv_gradient_visco.argtypes = [f32p] * 5 + [C.c_int, f32p, f32p]
    L.refdrv_residual_weights.argtypes = [C.c_int] * 7 + [f32p]
    return L


def layered(nz, nx, vals, ifaces):
    v = np.full((nz, nx), vals[0], np.float32)
    for val, z in zip(vals[1:], ifaces):
        v[z:] = val
    return v


def make_afd3d_big(a3, R):
    """afd3d forward and time reversal on an 80 x 72 x 64 interior with a
    10-cell taper: the expanded grid (100 x 92 x 84) has 32-cell z runs and
    4-column x runs free of taper and masks, so the untapered fast paths of
    a warp-tiled 3-D step run, over several y chunks.  The reference's
    outputs are kept as digests plus decimated copies."""
    vel = big3d_velocity()
    kw = dict(BIG3D, verb=0)
    d, w = quiet(a3.afd3d, vel, **kw)
    rick = []
    for fq, t0, A in zip(kw["f"], kw["t"], kw["A"]):
        r = np.zeros(kw["nt"], np.float32)
        R.refdrv_ricker(kw["nt"], kw["dt"], fq, t0, A, r)
        rick.append(r)
    # one receiver group's traces (x-band 18..36) reversed, snapshots every 4 steps
    dg = np.zeros_like(d)
    b0, b1 = BIG3D_BAND
    dg[:, b0:b1, :] = d[:, b0:b1, :]
    _, wt = quiet(a3.afd3d, vel, nt=kw["nt"], dt=0.001, ax=kw["ax"], ay=kw["ay"], az=kw["az"],
                  jsnap=BIG3D_TRI_JSNAP, dat=dg, tri=True, verb=0, nbt=10, ct=0.02)
    np.savez_compressed(os.path.join(HERE, "afd3d_big.npz"), vel_digest=digest(vel),
                        rick=np.stack(rick), traces_digest=digest(d), snaps_digest=digest(w),
                        tri_snaps_digest=digest(wt), traces_dec=d[::3, ::4, ::4],
                        snaps_last_dec=w[::4, ::4, ::4, -1], tri_last_dec=wt[::4, ::4, ::4, 0],
                        snaps_shape=np.array(w.shape), tri_shape=np.array(wt.shape))


def _fwi_parr(par):
    # the driver's parameter layout (oracle/ref_driver.c fill_acpar)
    return np.array([par[k] for k in ("nz", "nx", "dz", "dx", "oz", "ox", "nt", "dt", "ot", "ns",
                                      "ds", "os", "nb", "coef", "f0", "acqui_type", "interval")],
                    np.float32)


def _fwi_case(R, vt, vs, par, wav):
    """Reference forward data of vt and gradient_av at vs (rect 1 and 3)."""
    nz, nx, nt, ns = par["nz"], par["nx"], par["nt"], par["ns"]
    parr = _fwi_parr(par)
    q = np.full(nz * nx, 1e4, np.float32)
    data = np.zeros(ns * nx * nt, np.float32)
    quiet(R.refdrv_forward, parr, np.ascontiguousarray(vt.flatten(order="F")), q, wav.copy(), data)
    out = {}
    for rect in (1, 3):
        g = np.zeros(nz * nx, np.float32)
        fc = np.zeros(1, np.float32)
        quiet(R.refdrv_gradient, parr, np.ascontiguousarray(vs.flatten(order="F")), q.copy(),
              wav.copy(), data.copy(), rect, g, fc)
        out[rect] = (g.reshape(nz, nx, order="F"), float(fc[0]))
    # data [ns][nr][nt] -> (nt, nr, ns) as pfwi returns it
    return data.reshape(nt, nx, ns, order="F"), out


def make_pfwi_scale(R):
    """pfwi forward and gradient_av at the geometry of the 300 x 600 FWI
    benchmark (nb 60: a 420 x 720 padded grid) and on a 460 x 200 model
    (580 x 320 padded, deeper than one z tile of a step kernel), 2 shots and
    a reduced nt (models: models.pfwi_scale_case).  Outputs are kept as
    digests plus decimated copies."""
    for name in ("c4geo", "deep"):
        vt, vs, par, wav = pfwi_scale_case(name)
        data, g = _fwi_case(R, vt, vs, par, wav)
        np.savez_compressed(os.path.join(HERE, f"pfwi_{name}.npz"),
                            vtrue_digest=digest(vt), vstart_digest=digest(vs),
                            data_digest=digest(data), data_dec=data[::5, ::10, :],
                            grad1_digest=digest(g[1][0]), grad3_digest=digest(g[3][0]),
                            grad1_dec=g[1][0][::5, ::5], fcost=g[1][1],
                            **{"par_" + k: np.asarray(v) for k, v in par.items()})


def make_pfwi_mid(pf, R):
    """60 x 120, 4 shots, nt 800: the reference's raw gradient_av (rect 1,
    with its first-call scaling) at the start model, for the cosine of the
    exact adjoint against it, and 20 iterations of the reference's fwic
    (pfwi mode 2) from the start model."""
    vt, vs = mid_models()
    wav = mid_wavelet(MID["nt"])
    data, g = _fwi_case(R, vt, vs, MID, wav)
    q = np.full(vt.shape, 1e4, np.float32)
    vinv = quiet(pf.pfwi, vs, q, wav, None, data=data, mode=2, par=dict(MID))[1]
    np.savez_compressed(os.path.join(HERE, "pfwi_mid.npz"), vtrue=vt, vstart=vs, wav=wav,
                        data_digest=digest(data), grad_rect1=g[1][0], fcost=g[1][1], vinv=vinv,
                        **{"par_" + k: np.asarray(v) for k, v in MID.items()})


def _lstri_inv_child(out_path):
    """Runs in a fresh process: the reference's CG keeps its search
    directions in statics for the life of the process (wave_cgstep.c:28-33),
    so the inversion golden starts from a process that never ran it."""
    pf = load("pfwi")
    vel, src = lstri_case()
    nz, nx, nt, ns = src.shape
    q = np.full(vel.shape, 1e4, np.float32)
    wav = np.zeros(nt, np.float32)
    par = dict(LSTRI, inv=False)
    data = quiet(pf.pfwi, vel, q, wav, src, mode=4, par=dict(par))[0]
    par = dict(LSTRI, inv=True, onlysrc=True, onlyvel=False)
    srcinv = quiet(pf.pfwi, vel, q, wav, src, data=data, mode=4, par=dict(par))[3]
    np.savez(out_path, data=data, srcinv=srcinv)


def make_lstri():
    """pfwi mode 4 (lstric, pfwi.c:1031): modelling from a distributed source
    field (inv = 0) and least-squares time-reversal source inversion by
    conjugate gradients (inv = 1, niter 6), 20 x 24, 2 shots, nt 200."""
    import subprocess
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "lstri.npz")
        code = ("import sys; sys.path.insert(0, %r); import make_golden as M; "
                "M._lstri_inv_child(%r)" % (HERE, path))
        subprocess.run([sys.executable, "-c", code], check=True, env=dict(os.environ))
        with np.load(path) as z:
            data, srcinv = z["data"], z["srcinv"]
    vel, src = lstri_case()
    np.savez_compressed(os.path.join(HERE, "lstri.npz"), vel=vel, src_digest=digest(src),
                        data=data, srcinv=srcinv)


def _pas_child(out_path):
    """Runs in a fresh process: the passive data of the true model by the
    reference's lstric (pfwi mode 4, inv 0) and the reference's pfwic (mode
    4, inv 1, onlysrc False, onlyvel True) from the start model."""
    pf = load("pfwi")
    vt, vs, src = pas_case()
    q = np.full(vt.shape, 1e4, np.float32)
    wav = np.zeros(PAS["nt"], np.float32)
    data = quiet(pf.pfwi, vt, q, wav, src, mode=4, par=dict(PAS, inv=False))[0]
    out = quiet(pf.pfwi, vs, q, wav, src, data=data, mode=4,
                par=dict(PAS, inv=True, onlysrc=False, onlyvel=True))
    np.savez(out_path, data=data, vinv=out[1], ret0=out[0])


def make_pfwi_pas(R):
    """pfwi mode 4 with velocity update (pfwic, pfwi.c:1507): the reference's
    raw gradient_pas_av at the start model (rect 1 and 3, first-call
    scaling included) and 4 iterations of pfwic, 30 x 40, 2 shots, nt 400,
    data from the reference's lstric on the true model."""
    import subprocess
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "pas.npz")
        code = ("import sys; sys.path.insert(0, %r); import make_golden as M; "
                "M._pas_child(%r)" % (HERE, path))
        subprocess.run([sys.executable, "-c", code], check=True, env=dict(os.environ))
        with np.load(path) as z:
            data, vinv, ret0 = z["data"], z["vinv"], z["ret0"]
    vt, vs, src = pas_case()
    nz, nx, nt, ns = src.shape
    parr = _fwi_parr(PAS)
    q = np.full(nz * nx, 1e4, np.float32)
    wav = np.zeros(nt, np.float32)
    dflat = np.ascontiguousarray(data.flatten(order="F"))  # [ns][nr][nt]
    sflat = np.ascontiguousarray(src.flatten(order="F"))   # [ns][nt][nx][nz]
    g = {}
    fhi_off = float(np.float32(0.5) / np.float32(PAS["dt"]))  # pfwic's soupar->fhi
    for key, rect, flo, fhi in ((1, 1, 0.0, fhi_off), (3, 3, 0.0, fhi_off),
                                ("ms", 1, PAS_FLO, PAS_FHI)):
        gr = np.zeros(nz * nx, np.float32)
        fc = np.zeros(1, np.float32)
        quiet(R.refdrv_gradient_pas, parr, np.ascontiguousarray(vs.flatten(order="F")), q.copy(),
              wav.copy(), dflat.copy(), sflat.copy(), rect, flo, fhi, gr, fc)
        g[key] = (gr.reshape(nz, nx, order="F"), float(fc[0]))
    np.savez_compressed(os.path.join(HERE, "pfwi_pas.npz"), vtrue=vt, vstart=vs,
                        src_digest=digest(src), data=data, grad_rect1=g[1][0],
                        grad_rect3=g[3][0], fcost=g[1][1], vinv=vinv,
                        grad_ms_rect1=g["ms"][0], fcost_ms=g["ms"][1],
                        flo=np.float32(PAS_FLO), fhi=np.float32(PAS_FHI),
                        ret0_equals_data_flat=np.array_equal(ret0.reshape(-1),
                                                             data.flatten(order="F")))


def make_butter(R):
    """np_butter_apply (wave_butter.c) on seeded noise traces for low- and
    high-pass filters of 3 to 5 poles, and residual_weighting
    (wave_fwiutil.c:225-296) in both branches with an inner window."""
    rng = np.random.default_rng(23)
    x = rng.standard_normal((4, 300)).astype(np.float32)
    out = {"x": x}
    for i, (low, cut, nn) in enumerate(BUTTER_CASES):
        y = x.copy()
        for row in y:
            r = np.ascontiguousarray(row)
            R.refdrv_butter(low, cut, nn, r.size, r)
            row[:] = r
        out["y%d" % i] = y
    nt, nr, wtn1, wtn2, woffn1, woffn2 = WEIGHT_CASE
    for oreo in (0, 1):
        w = np.zeros(nr * nt, np.float32)
        R.refdrv_residual_weights(nt, nr, wtn1, wtn2, woffn1, woffn2, oreo, w)
        out["w_oreo%d" % oreo] = w.reshape(nr, nt)
    np.savez_compressed(os.path.join(HERE, "butter.npz"), **out)


def make_aps():
    """The reference's pseudo-spectral propagator (apscfun, aps.c ->
    psm2d / psm, wave_psp.c:25-635) through its unmodified aps2d.py /
    aps3d.py: 2-D forward modelling with snapshots, 2-D time reversal of
    one half of the traces, 3-D forward modelling."""
    a2 = load("aps2d")
    a3 = load("aps3d")
    v2 = aps2_velocity()
    d2, w2 = quiet(a2.aps2d, v2, ifsnaps=True, verb=False, **APS2)
    dt_ = np.zeros_like(d2)
    dt_[:, :30] = d2[:, :30]
    kw = {k: APS2[k] for k in ("nt", "dt", "ax", "az", "nbt", "ct", "jsnap")}
    _, wt = quiet(a2.aps2d, v2, tri=True, dat=dt_, ifsnaps=True, verb=False, **kw)
    v3 = aps3_velocity()
    d3, w3 = quiet(a3.aps3d, v3, ifsnaps=True, verb=False, **APS3)
    np.savez_compressed(os.path.join(HERE, "aps.npz"), v2=v2, d2=d2, w2=w2, dtri=dt_, wtri=wt,
                        v3=v3, d3=d3, w3=w3)


def make_visco(R):
    """Visco-acoustic pfwi, which the reference's Python glue cannot reach
    (pfwi.c:864 always takes the acoustic path): forward_modeling
    (wave_fwimodeling.c:116) of the true model and gradient_v
    (wave_fwigradient.c:264) at the start model, rect 1 and 3, both called
    through oracle/ref_driver.c."""
    vt, vs, q, wav = visco_case()
    nz, nx, nt, ns = VISCO["nz"], VISCO["nx"], VISCO["nt"], VISCO["ns"]
    parr = _fwi_parr(VISCO)
    qf = np.ascontiguousarray(q.flatten(order="F"))
    data = np.zeros(ns * nx * nt, np.float32)
    quiet(R.refdrv_forward_visco, parr, np.ascontiguousarray(vt.flatten(order="F")), qf.copy(),
          wav.copy(), data)
    g = {}
    for rect in (1, 3):
        gr = np.zeros(nz * nx, np.float32)
        fc = np.zeros(1, np.float32)
        quiet(R.refdrv_gradient_visco, parr, np.ascontiguousarray(vs.flatten(order="F")),
              qf.copy(), wav.copy(), data.copy(), rect, gr, fc)
        g[rect] = (gr.reshape(nz, nx, order="F"), float(fc[0]))
    np.savez_compressed(os.path.join(HERE, "visco.npz"), q=q,
                        data=data.reshape(nt, nx, ns, order="F"), grad_rect1=g[1][0],
                        grad_rect3=g[3][0], fcost=g[1][1])


class _Recorder:
    """Stands in for an extension module: records each call's arguments and
    returns the real module's result."""

    def __init__(self, real, names):
        self.calls = []
        self.real = real
        for n in names:
            setattr(self, n, self._wrap(n))
        self.__all__ = list(names)

    def _wrap(self, name):
        def f(*args):
            out = getattr(self.real, name)(*args)
            self.calls.append((name, args, out))
            return out
        return f


def make_dropin():
    """The exact positional arguments the reference's own, unmodified Python
    wrappers (pywave/afd2d.py:73, afd3d.py:77, pfwi.py:70,111) pass to their
    extension modules, with digests of what the reference's modules return:
    a replay through pywave_b200.afdcfun / pfwicfun tests the drop-in."""
    import types
    real_afd = importlib.import_module("afdcfun")
    real_pf = importlib.import_module("pfwicfun")
    rec_afd = _Recorder(real_afd, ["afd2dc", "afd3dc"])
    rec_pf = _Recorder(real_pf, ["forward_modeling_ac", "fwic"])
    saved = {k: sys.modules.get(k) for k in ("afdcfun", "pfwicfun")}
    for name, rec in (("afdcfun", rec_afd), ("pfwicfun", rec_pf)):
        m = types.ModuleType(name)
        for n in rec.__all__:
            setattr(m, n, getattr(rec, n))
        m.__all__ = rec.__all__
        sys.modules[name] = m
    try:
        a2, a3, pf = load("afd2d"), load("afd3d"), load("pfwi")
        vel = layered(41, 51, [2000, 2500, 3100], [15, 28])
        d, _ = quiet(a2.afd2d, vel, nt=300, dt=0.001, ax=[0, 20, 51], az=[0, 20, 41], ns=2,
                     sx=[20, 31], sz=[10, 17], f=[10, 12], t=[0.1, 0.12], A=[1, 2], nbt=30,
                     ct=0.01, jsnap=3, verb=0)
        dg = np.zeros_like(d)
        dg[:, 10:30] = d[:, 10:30]
        quiet(a2.afd2d, vel, nt=300, dt=0.001, ax=[0, 20, 51], az=[0, 20, 41], jsnap=4, dat=dg,
              tri=True, verb=0, nbt=30, ct=0.01)
        rng = np.random.default_rng(0)
        vel3 = (2000 + 300 * rng.random((24, 20, 22))).astype(np.float32)
        d3, _ = quiet(a3.afd3d, vel3, nt=120, dt=0.001, ax=[0, 20, 20], ay=[0, 20, 22],
                      az=[0, 20, 24], ns=2, sx=[8, 12], sy=[9, 11], sz=[10, 6], f=[12, 15],
                      t=[0.03, 0.05], A=[1, 1.5], nbt=8, ct=0.02, jsnap=5, verb=0)
        dg3 = np.zeros_like(d3)
        dg3[:, 5:15, :] = d3[:, 5:15, :]
        quiet(a3.afd3d, vel3, nt=120, dt=0.001, ax=[0, 20, 20], ay=[0, 20, 22], az=[0, 20, 24],
              jsnap=4, dat=dg3, tri=True, verb=0, nbt=8, ct=0.02)
        nz, nx, nt = 30, 50, 400
        vt = layered(nz, nx, [2.0, 2.5, 3.0], [12, 22])
        q = np.full((nz, nx), 1e4, np.float32)
        tt = np.arange(nt) * 0.001
        arg = (np.pi * 10 * (tt - 0.1)) ** 2
        wav = ((1 - 2 * arg) * np.exp(-arg)).astype(np.float32)
        par = dict(nz=nz, nx=nx, dz=0.01, dx=0.01, oz=0, ox=0, nt=nt, dt=0.001, ot=0, ns=3,
                   ds=0.15, os=0.05, nb=20, coef=0.005, f0=10, acqui_type=1, interval=1, niter=2)
        data = quiet(pf.pfwi, vt, q, wav, None, mode=1, par=dict(par))[0]
        vs = np.full((nz, nx), 2.4, np.float32)
        quiet(pf.pfwi, vs, q, wav, None, data=data, mode=2, par=dict(par))
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
    out = {}
    calls = rec_afd.calls + rec_pf.calls
    for i, (name, args, res) in enumerate(calls):
        out[f"c{i}_name"] = np.asarray(name)
        out[f"c{i}_nargs"] = np.asarray(len(args))
        for j, x in enumerate(args):
            out[f"c{i}_a{j}"] = np.asarray(x)
        out[f"c{i}_out_digest"] = np.asarray(digest(np.asarray(res)))
        out[f"c{i}_out_shape"] = np.asarray(np.asarray(res).shape)
        out[f"c{i}_out_dec"] = np.asarray(res).reshape(-1)[::97]
    out["ncalls"] = np.asarray(len(calls))
    np.savez_compressed(os.path.join(HERE, "dropin_calls.npz"), **out)


def main(names=()):
    a2, a3, pf = load("afd2d"), load("afd3d"), load("pfwi")
    R = refdrv()
    R.refdrv_forward.argtypes = [np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")] * 5
    extra = {"afd3d_big": lambda: make_afd3d_big(a3, R), "pfwi_scale": lambda: make_pfwi_scale(R),
             "pfwi_mid": lambda: make_pfwi_mid(pf, R), "dropin": make_dropin,
             "lstri": make_lstri, "pfwi_pas": lambda: make_pfwi_pas(R),
             "butter": lambda: make_butter(R), "aps": make_aps,
             "visco": lambda: make_visco(R)}
    if names:
        for n in names:
            extra[n]()
        return
    for fn in extra.values():
        fn()
    out = {}

    # ---- afd2d forward, 2 sources, snapshots ---------------------------
    vel = layered(41, 51, [2000, 2500, 3100], [15, 28])
    kw = dict(nt=300, dt=0.001, ax=[0, 20, 51], az=[0, 20, 41], ns=2, sx=[20, 31], sz=[10, 17],
              f=[10, 12], t=[0.1, 0.12], A=[1, 2], nbt=30, ct=0.01, jsnap=3, verb=0)
    d, w = quiet(a2.afd2d, vel, **kw)
    rick = []
    for fq, t0, A in zip(kw["f"], kw["t"], kw["A"]):
        r = np.zeros(kw["nt"], np.float32)
        R.refdrv_ricker(kw["nt"], kw["dt"], fq, t0, A, r)
        rick.append(r)
    np.savez_compressed(os.path.join(HERE, "afd2d_fwd.npz"), vel=vel, traces=d, snaps=w,
                        rick=np.stack(rick), **{k: np.asarray(v) for k, v in kw.items()})

    # ---- afd2d time reversal of one group's traces -----------------------
    dg = np.zeros_like(d)
    dg[:, 10:30] = d[:, 10:30]
    echo, wt = quiet(a2.afd2d, vel, nt=300, dt=0.001, ax=[0, 20, 51], az=[0, 20, 41], jsnap=4,
                     dat=dg, tri=True, verb=0, nbt=30, ct=0.01)
    np.savez_compressed(os.path.join(HERE, "afd2d_tri.npz"), vel=vel, dat=dg, echo=echo, snaps=wt)

    # ---- afd3d forward, small ------------------------------------------
    rng = np.random.default_rng(0)
    vel3 = (2000 + 300 * rng.random((24, 20, 22))).astype(np.float32)
    kw3 = dict(nt=120, dt=0.001, ax=[0, 20, 20], ay=[0, 20, 22], az=[0, 20, 24], ns=2, sx=[8, 12],
               sy=[9, 11], sz=[10, 6], f=[12, 15], t=[0.03, 0.05], A=[1, 1.5], nbt=8, ct=0.02,
               jsnap=5, verb=0)
    d3, w3 = quiet(a3.afd3d, vel3, **kw3)
    rick3 = []
    for fq, t0, A in zip(kw3["f"], kw3["t"], kw3["A"]):
        r = np.zeros(kw3["nt"], np.float32)
        R.refdrv_ricker(kw3["nt"], kw3["dt"], fq, t0, A, r)
        rick3.append(r)
    np.savez_compressed(os.path.join(HERE, "afd3d_fwd.npz"), vel=vel3, traces=d3, snaps=w3,
                        rick=np.stack(rick3), **{k: np.asarray(v) for k, v in kw3.items()})

    # ---- afd3d time reversal -------------------------------------------
    dg3 = np.zeros_like(d3)
    dg3[:, 5:15, :] = d3[:, 5:15, :]
    echo3, wt3 = quiet(a3.afd3d, vel3, nt=120, dt=0.001, ax=[0, 20, 20], ay=[0, 20, 22],
                       az=[0, 20, 24], jsnap=4, dat=dg3, tri=True, verb=0, nbt=8, ct=0.02)
    np.savez_compressed(os.path.join(HERE, "afd3d_tri.npz"), vel=vel3, dat=dg3, snaps=wt3)

    # ---- 201x201 three-layer gather, receivers at z=5 (wfd[5].T with jsnap=1) ------
    vc1 = layered(201, 201, [1500, 2200, 3000], [60, 130])
    _, wc1 = quiet(a2.afd2d, vc1, nt=1501, dt=0.001, ax=[0, 10, 201], az=[0, 10, 201], ns=1,
                   sx=[100], sz=[5], f=[20], t=[0.05], A=[1], nbt=30, ct=0.01, jsnap=1, verb=0)
    rc1 = np.zeros(1501, np.float32)
    R.refdrv_ricker(1501, 0.001, 20, 0.05, 1, rc1)
    np.savez_compressed(os.path.join(HERE, "c1_gather_z5.npz"),
                        gather=np.ascontiguousarray(wc1[5].T), rick=rc1[None, :])
    del wc1

    # ---- pfwi forward modelling + gradient_av ----------------------------
    nz, nx, nt = 30, 50, 400
    vt = layered(nz, nx, [2.0, 2.5, 3.0], [12, 22])
    q = np.full((nz, nx), 1e4, np.float32)
    tt = np.arange(nt) * 0.001
    arg = (np.pi * 10 * (tt - 0.1)) ** 2
    wav = ((1 - 2 * arg) * np.exp(-arg)).astype(np.float32)
    par = dict(nz=nz, nx=nx, dz=0.01, dx=0.01, oz=0, ox=0, nt=nt, dt=0.001, ot=0, ns=3, ds=0.15,
               os=0.05, nb=20, coef=0.005, f0=10, acqui_type=1, interval=1, niter=2)
    data = quiet(pf.pfwi, vt, q, wav, None, mode=1, par=dict(par))[0]
    vs = np.full((nz, nx), 2.4, np.float32)
    parr = np.array([nz, nx, 0.01, 0.01, 0, 0, nt, 0.001, 0, 3, 0.15, 0.05, 20, 0.005, 10, 1, 1],
                    np.float32)
    grads = {}
    for rect in (1, 3):
        g = np.zeros(nz * nx, np.float32)
        fc = np.zeros(1, np.float32)
        quiet(R.refdrv_gradient, parr, np.ascontiguousarray(vs.flatten(order="F")),
              np.ascontiguousarray(q.flatten(order="F")), wav.copy(),
              np.ascontiguousarray(data.flatten(order="F")), rect, g, fc)
        grads[rect] = (g.reshape(nz, nx, order="F"), float(fc[0]))
    vinv = quiet(pf.pfwi, vs, q, wav, None, data=data, mode=2, par=dict(par))[1]
    np.savez_compressed(os.path.join(HERE, "pfwi.npz"), vtrue=vt, vstart=vs, wav=wav, data=data,
                        grad_rect1=grads[1][0], fcost=grads[1][1], grad_rect3=grads[3][0],
                        vinv=vinv, **{"par_" + k: np.asarray(v) for k, v in par.items()})
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main(sys.argv[1:])
