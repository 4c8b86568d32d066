"""ctypes front-end of the CPU oracle (oracle/pw_oracle.c).

TEST INFRASTRUCTURE ONLY.  Only tests/, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import this
module, and only as the checker or the timed CPU baseline.  The product
(``pywave_b200``) never imports it and fails loudly when its CUDA library is
missing.

Array conventions follow the reference: column-major with z fastest
(``vel.flatten(order='F')`` in pywave/afd2d.py:48), traces ``[nx][nt]`` with
time fastest (pywave/src/afd.c:473-486).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle restatement (gcc, no FMA contraction)."""
    srcs = [os.path.join(HERE, f) for f in ("pw_oracle.c", "pw_oracle_body.h",
                                             "pw_oracle3d_body.h", "pw_oracle_lstri_body.h")]
    stale = (not os.path.exists(LIB_PATH)) or any(
        os.path.getmtime(s) > os.path.getmtime(LIB_PATH) for s in srcs)
    if force or stale:
        subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    return LIB_PATH


def build_ref() -> bool:
    """Compile the reference itself into oracle/_ref from the sources under
    $PYWAVE_REF (the pywave checkout); False when they are not there."""
    root = os.environ.get("PYWAVE_REF", "")
    if not root or not os.path.isdir(os.path.join(root, "pywave", "src")):
        return False
    subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)
    return True


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        L.or_next_fast.argtypes = [C.c_int]
        L.or_next_fast.restype = C.c_int
        L.or_pad_first.argtypes = [C.c_int]
        L.or_pad_first.restype = C.c_int
        L.or_ricker.argtypes = [C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, _f64p]
        L.or_ricker.restype = None
        L.or_smooth2d.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _f32p]
        L.or_smooth2d.restype = None
        L.or_residual_weights.argtypes = [C.c_int] * 6 + [_f32p]
        L.or_residual_weights.restype = None
        L.or_residual_weights_oreo.argtypes = [C.c_int] * 6 + [_f32p]
        L.or_residual_weights_oreo.restype = None
        L.or_butter_coefs.argtypes = [C.c_int, C.c_float, C.c_int, _f32p, _f32p]
        L.or_butter_coefs.restype = None
        for sfx, rp in (("f32", _f32p), ("f64", _f64p)):
            f = getattr(L, "or_afd_" + sfx)
            f.argtypes = ([C.c_int] * 5 + [C.c_float] * 5 + [C.c_int, C.c_int, _i32p, _i32p, _i32p,
                          rp, C.c_int, rp, C.c_int, C.c_int, rp, rp, C.c_void_p])
            f.restype = C.c_int
            geo = [C.c_int, _i32p, C.c_int, C.c_int, _i32p, _i32p, _i32p, C.c_int, C.c_int]
            f = getattr(L, "or_pfwi_forward_" + sfx)
            f.argtypes = [C.c_int] * 3 + [C.c_float] * 2 + [C.c_int] + [C.c_float] * 2 + geo + [rp, rp, rp]
            f.restype = None
            real = C.c_float if sfx == "f32" else C.c_double
            f = getattr(L, "or_pfwi_gradient_ref_" + sfx)
            f.argtypes = ([C.c_int] * 3 + [C.c_float] * 2 + [C.c_int] + [C.c_float] * 2 + [C.c_int]
                          + geo + [rp, rp, rp, rp, rp])
            f.restype = real
            f = getattr(L, "or_pfwi_gradient_pas_" + sfx)
            f.argtypes = ([C.c_int] * 3 + [C.c_float] * 2 + [C.c_int] + [C.c_float] * 2 + [C.c_int]
                          + [C.c_int, C.c_int, _i32p, _i32p, _i32p, C.c_int, C.c_int]
                          + [rp, rp, rp, rp, rp, C.c_float, C.c_float])
            f.restype = real
            f = getattr(L, "or_pfwi_forward_visco_" + sfx)
            f.argtypes = ([C.c_int] * 3 + [C.c_float] * 2 + [C.c_int] + [C.c_float] * 3 + geo
                          + [rp, rp, rp, rp])
            f.restype = None
            f = getattr(L, "or_pfwi_gradient_visco_" + sfx)
            f.argtypes = ([C.c_int] * 3 + [C.c_float] * 2 + [C.c_int] + [C.c_float] * 3 + [C.c_int]
                          + geo + [rp, rp, rp, rp, rp, rp])
            f.restype = real
            f = getattr(L, "or_butter_apply_" + sfx)
            f.argtypes = [C.c_int, C.c_float, C.c_int, C.c_int, rp]
            f.restype = None
            f = getattr(L, "or_pfwi_gradient_exact_" + sfx)
            f.argtypes = ([C.c_int] * 3 + [C.c_float] * 2 + [C.c_int] + [C.c_float] * 2 + geo
                          + [rp, rp, rp, C.c_void_p, rp])
            f.restype = real
            f = getattr(L, "or_pfwi_misfit_" + sfx)
            f.argtypes = ([C.c_int] * 3 + [C.c_float] * 2 + [C.c_int] + [C.c_float] * 2 + geo
                          + [rp, rp, rp, C.c_void_p])
            f.restype = real
            geo3 = [C.c_int] * 4 + [C.c_float] * 3 + [C.c_int, C.c_float, C.c_float, C.c_int,
                                                        _i32p, C.c_int, C.c_int, C.c_int, _i32p,
                                                        _i32p]
            f = getattr(L, "or_pf3_forward_" + sfx)
            f.argtypes = geo3 + [rp, rp, rp]
            f.restype = None
            f = getattr(L, "or_pf3_gradient_exact_" + sfx)
            f.argtypes = geo3 + [rp, rp, rp, C.c_void_p, rp]
            f.restype = real
            f = getattr(L, "or_pf3_misfit_" + sfx)
            f.argtypes = geo3 + [rp, rp, rp, C.c_void_p]
            f.restype = real
            f = getattr(L, "or_lstri_" + sfx)
            f.argtypes = [C.c_int] * 7 + [C.c_float] * 4 + [C.c_int, _f32p, rp, rp, C.c_void_p]
            f.restype = None
            f = getattr(L, "or_timerev_" + sfx)
            f.argtypes = [C.c_int] * 6 + [C.c_float] * 4 + [_f32p, rp, rp]
            f.restype = None
        _lib = L
    return _lib


# --------------------------------------------------------------------------
# afd (pywave/afd2d.py, afd3d.py -> afd.c -> wave_fdm.c)
# --------------------------------------------------------------------------

def next_fast(n: int) -> int:
    return lib().or_next_fast(int(n))


def ricker(nt: int, dt: float, f0: float, t0: float, A: float) -> np.ndarray:
    """Ricker table of fdm2d/fdm (wave_fdm.c:502-516), float64."""
    out = np.zeros(nt, np.float64)
    lib().or_ricker(int(nt), float(dt), float(f0), float(t0), float(A), out)
    return out


def _ntsnap(nt, jsnap):
    return sum(1 for it in range(nt) if jsnap and it % jsnap == 0)


def afd(vel, nt, dt, d, nbt=30, ct=0.01, src=None, tri=False, dat=None, jsnap=0, gz=0,
        precision="f32", rick=None):
    """Run the afd propagator (fdm2d when vel is 2-D, fdm when 3-D).

    vel: (nz,nx) or (nz,nx,ny).  d: (dz,dx) or (dz,dx,dy).
    src: dict with sx, sz, [sy], f, t, A (forward mode).
    dat: TRI traces, (nt,nx) or (nt,nx,ny) as afd2d/afd3d receive them.
    rick: optional [ns][nt] wavelet table replacing the Ricker table.
    Returns (traces (nt,nx[,ny]) or None, snapshots (nz,nx[,ny],ntsnap) or None).
    """
    vel = np.asarray(vel)
    dim = vel.ndim
    R = np.float32 if precision == "f32" else np.float64
    fn = getattr(lib(), "or_afd_" + precision)
    if dim == 2:
        nz1, nx1 = vel.shape
        ny1 = 1
        dz, dx = d
        dy = 1.0
    else:
        nz1, nx1, ny1 = vel.shape
        dz, dx, dy = d
    velf = np.ascontiguousarray(vel.astype(np.float32).flatten(order="F").astype(R))
    if tri:
        ns = 0
        spz = spx = spy = np.zeros(1, np.int32)
        rick = np.zeros(1, R)
        datin = np.ascontiguousarray(np.asarray(dat, np.float32).flatten(order="F").astype(R))
    else:
        sx = np.asarray(src["sx"]).astype(np.float32).astype(np.int32)
        sz = np.asarray(src["sz"]).astype(np.float32).astype(np.int32)
        sy = np.asarray(src.get("sy", np.zeros_like(sx))).astype(np.float32).astype(np.int32)
        ns = len(sx)
        spz, spx, spy = (np.ascontiguousarray(a, dtype=np.int32) for a in (sz, sx, sy))
        f = np.asarray(src["f"], np.float32)
        t = np.asarray(src["t"], np.float32)
        A = np.asarray(src["A"], np.float32)
        if rick is None:
            rick = np.stack([ricker(nt, dt, f[i], t[i], A[i]) for i in range(ns)])
        rick = np.ascontiguousarray(np.asarray(rick).astype(np.float32).astype(R))
        datin = np.zeros(1, R)
    dout = np.zeros(nt * nx1 * ny1, R)
    ntsnap = _ntsnap(nt, jsnap)
    wfd = np.zeros(max(1, ntsnap * nz1 * nx1 * ny1), R)
    rc = fn(dim, nz1, nx1, ny1, nbt, ct, dt, dz, dx, dy, nt, ns, spz, spx, spy, rick,
            1 if tri else 0, datin, int(jsnap), int(gz), velf, dout,
            wfd.ctypes.data if ntsnap > 0 else None)
    if rc != 0:
        raise MemoryError("oracle allocation failed")
    traces = None
    if not tri:
        traces = dout.reshape((nt, nx1) if dim == 2 else (nt, nx1, ny1), order="F")
    snaps = None
    if ntsnap > 0:
        shp = (nz1, nx1, ntsnap) if dim == 2 else (nz1, nx1, ny1, ntsnap)
        snaps = wfd.reshape(shp, order="F")
    return traces, snaps


def tri_groups_image(snaps_per_group):
    """The demos' TRI image (demos/test_third_tri.py:71-77,
    demos/test_mod2d_tri_psVSfd.py:184-190): sum over snapshots of the
    product over groups of the squared snapshot, divided by its maximum."""
    img = 1
    for s in snaps_per_group:
        img = img * s * s
    img = np.sum(img, axis=-1)
    return img / img.max()


def group_bands(nx: int, ng: int):
    """Receiver groups of the TRI demos: x-bands of width nx//ng; columns
    beyond ng*(nx//ng) belong to no group (demos/test_third_tri.py:63-66)."""
    dg = nx // ng
    return [np.arange(g * dg, g * dg + dg) for g in range(ng)]


# --------------------------------------------------------------------------
# pfwi (pywave/pfwi.py -> pfwi.c -> wave_fwi*.c)
# --------------------------------------------------------------------------

def pfwi_geometry(nz, nx, dz, dx, oz, ox, ns, ds, os_, nb, acqui_type=1, sz=5, rz=1):
    """Resolved acquisition geometry of preparation (wave_fwiutil.c:44-71)
    with the fixed settings of pfwi.c:796-801 (sz=5, rz=1, nr=nx, dr=dx,
    r0=ox).  Float arithmetic in the reference's order."""
    f32 = np.float32
    dx32 = f32(dx)
    ds_v = int(float(f32(ds) / dx32) + 0.5)
    s0_v = int(float(f32(os_) / dx32) + 0.5 + nb)
    nr = nx
    dr = dx32
    r0 = f32(ox)
    x0 = f32(ox)
    dr_v = int(float(dr / dx32) + 0.5)
    sx = np.array([s0_v + i * ds_v for i in range(ns)], np.int32)
    xend = f32(x0 + f32((nx - 1) * dx32))
    r0v = np.zeros(ns, np.int32)
    r02 = np.zeros(ns, np.int32)
    nr2 = np.zeros(ns, np.int32)
    for i in range(ns):
        if acqui_type == 1:
            r0v[i] = int(float((r0 - x0) / dx32) + 0.5 + nb)
            r02[i] = 0
            nr2[i] = nr
        else:
            sxf = f32(f32(os_) + f32(f32(ds) * i))
            rbegin = x0 if f32(sxf + r0) < x0 else f32(sxf + r0)
            rend = f32(f32(sxf + r0) + f32((nr - 1) * dr))
            rend = rend if rend < xend else xend
            r0v[i] = int(float(rbegin / dx32) + 0.5 + nb)
            r02[i] = int(float(f32(f32(rbegin - sxf) - r0) / dx32) + 0.5)
            nr2[i] = int(float(f32(rend - rbegin) / dx32) + 1.5)
    return dict(sx=sx, sz=sz + nb, nr=nr, r0v=r0v, r02=r02, nr2=nr2, drv=dr_v, rz=rz + nb)


def _geo_args(g, ns):
    return (ns, g["sx"], g["sz"], g["nr"], g["r0v"], g["r02"], g["nr2"], g["drv"], g["rz"])


def pfwi_forward(vel, wav, nb, coef, dz, dx, dt, geo, ns, precision="f32"):
    """forward_modeling_a; vel (nz,nx); returns data (nt,nr,ns) like pfwi.py:74."""
    R = np.float32 if precision == "f32" else np.float64
    nz, nx = vel.shape
    nt = len(wav)
    v = np.ascontiguousarray(np.asarray(vel, np.float32).flatten(order="F").astype(R))
    w = np.ascontiguousarray(np.asarray(wav, np.float32).astype(R))
    out = np.zeros(ns * geo["nr"] * nt, R)
    getattr(lib(), "or_pfwi_forward_" + precision)(nz, nx, nb, dz, dx, nt, dt, coef,
                                                   *_geo_args(geo, ns), v, w, out)
    return out.reshape(nt, geo["nr"], ns, order="F")


def residual_weights(nt, nr, wtn1=None, wtn2=None, woffn1=None, woffn2=None, oreo=False):
    """residual_weighting (oreo=false as fwic configures it, or the oreo
    branch); (nr,nt) C-order."""
    w = np.zeros(nr * nt, np.float32)
    fn = lib().or_residual_weights_oreo if oreo else lib().or_residual_weights
    fn(nt, nr, 0 if wtn1 is None else wtn1, nt - 1 if wtn2 is None else wtn2,
       0 if woffn1 is None else woffn1, nr - 1 if woffn2 is None else woffn2, w)
    return w.reshape(nr, nt)


def butter_apply(x, low, cutoff, npoles=3, precision="f32"):
    """np_butter_apply over each row of x (a copy), cutoff in cycles per
    sample (wave_butter.c)."""
    R = np.float32 if precision == "f32" else np.float64
    y = np.ascontiguousarray(np.array(x, dtype=R, ndmin=2))
    for row in y:
        r = np.ascontiguousarray(row)
        getattr(lib(), "or_butter_apply_" + precision)(int(low), float(cutoff), int(npoles),
                                                       r.size, r)
        row[:] = r
    return y.reshape(np.shape(x))


def butter_coefs(low, cutoff, npoles=3):
    """(den [nsections][2], mid) of np_butter_init."""
    den = np.zeros(2 * (npoles // 2 + npoles % 2), np.float32)
    mid = np.zeros(1, np.float32)
    lib().or_butter_coefs(int(low), float(cutoff), int(npoles), den, mid)
    return den.reshape(-1, 2), float(mid[0])


def _dobs_flat(dobs, R):
    # dobs (nt,nr,ns) F-order -> flat [ns][nr][nt]
    return np.ascontiguousarray(np.asarray(dobs, np.float32).flatten(order="F").astype(R))


def pfwi_gradient_ref(vel, wav, dobs, nb, coef, dz, dx, dt, geo, ns, interval=1, weight=None,
                      precision="f32"):
    """gradient_av before scaling/smoothing.  Returns (grad (nz,nx), fcost)."""
    R = np.float32 if precision == "f32" else np.float64
    nz, nx = vel.shape
    nt = len(wav)
    if weight is None:
        weight = residual_weights(nt, geo["nr"])
    v = np.ascontiguousarray(np.asarray(vel, np.float32).flatten(order="F").astype(R))
    w = np.ascontiguousarray(np.asarray(wav, np.float32).astype(R))
    g = np.zeros(nz * nx, R)
    f = getattr(lib(), "or_pfwi_gradient_ref_" + precision)(
        nz, nx, nb, dz, dx, nt, dt, coef, interval, *_geo_args(geo, ns), v, w,
        _dobs_flat(dobs, R), np.ascontiguousarray(np.asarray(weight, np.float32).astype(R)), g)
    return g.reshape(nz, nx, order="F"), float(f)


def pfwi_forward_visco(vel, q, wav, nb, coef, dz, dx, dt, f0, geo, ns, precision="f32"):
    """Visco-acoustic forward_modeling (wave_fwimodeling.c:116); vel, q
    (nz, nx); returns data (nt, nr, ns)."""
    R = np.float32 if precision == "f32" else np.float64
    nz, nx = vel.shape
    nt = len(wav)
    v = np.ascontiguousarray(np.asarray(vel, np.float32).flatten(order="F").astype(R))
    qq = np.ascontiguousarray(np.asarray(q, np.float32).flatten(order="F").astype(R))
    w = np.ascontiguousarray(np.asarray(wav, np.float32).astype(R))
    out = np.zeros(ns * geo["nr"] * nt, R)
    getattr(lib(), "or_pfwi_forward_visco_" + precision)(nz, nx, nb, dz, dx, nt, dt, coef, f0,
                                                         *_geo_args(geo, ns), v, qq, w, out)
    return out.reshape(nt, geo["nr"], ns, order="F")


def pfwi_gradient_visco(vel, q, wav, dobs, nb, coef, dz, dx, dt, f0, geo, ns, interval=1,
                        weight=None, precision="f32"):
    """gradient_v (wave_fwigradient.c:264) before scaling / smoothing.
    Returns (grad (nz, nx), fcost)."""
    R = np.float32 if precision == "f32" else np.float64
    nz, nx = vel.shape
    nt = len(wav)
    if weight is None:
        weight = residual_weights(nt, geo["nr"])
    v = np.ascontiguousarray(np.asarray(vel, np.float32).flatten(order="F").astype(R))
    qq = np.ascontiguousarray(np.asarray(q, np.float32).flatten(order="F").astype(R))
    w = np.ascontiguousarray(np.asarray(wav, np.float32).astype(R))
    g = np.zeros(nz * nx, R)
    f = getattr(lib(), "or_pfwi_gradient_visco_" + precision)(
        nz, nx, nb, dz, dx, nt, dt, coef, f0, interval, *_geo_args(geo, ns), v, qq, w,
        _dobs_flat(dobs, R), np.ascontiguousarray(np.asarray(weight, np.float32).astype(R)), g)
    return g.reshape(nz, nx, order="F"), float(f)


def pfwi_gradient_pas(vel, src, dobs, nb, coef, dz, dx, dt, geo, ns, nt, interval=1,
                      weight=None, precision="f32", flo=0.0, fhi=None):
    """gradient_pas_av (pfwic's passive gradient) before scaling/smoothing;
    src (nz, nx, nt, ns) source fields, dobs (nt, nr, ns).  Returns
    (grad (nz, nx), fcost)."""
    R = np.float32 if precision == "f32" else np.float64
    nz, nx = vel.shape
    if weight is None:
        weight = residual_weights(nt, geo["nr"])
    v = np.ascontiguousarray(np.asarray(vel, np.float32).flatten(order="F").astype(R))
    sv = np.ascontiguousarray(np.asarray(src, np.float32).flatten(order="F").astype(R))
    g = np.zeros(nz * nx, R)
    f = getattr(lib(), "or_pfwi_gradient_pas_" + precision)(
        nz, nx, nb, dz, dx, nt, dt, coef, interval, ns, geo["nr"], geo["r0v"], geo["r02"],
        geo["nr2"], geo["drv"], geo["rz"], v, sv, _dobs_flat(dobs, R),
        np.ascontiguousarray(np.asarray(weight, np.float32).astype(R)), g, float(flo),
        float(np.float32(0.5) / np.float32(dt)) if fhi is None else float(fhi))
    return g.reshape(nz, nx, order="F"), float(f)


def pfwi_postprocess(grad, rect=3, scaling=None):
    """gradient_av's tail (wave_fwigradient.c:244-255): first-call scaling
    0.1/max|g| (float), triangle smoothing rect x rect, times the scale."""
    g = np.ascontiguousarray(np.asarray(grad, np.float32).flatten(order="F"))
    if scaling is None:
        scaling = np.float32(0.1 / float(np.max(np.abs(g))))
    nz, nx = grad.shape
    lib().or_smooth2d(rect, rect, nz, nx, g)
    g = g * np.float32(scaling)
    return g.reshape(nz, nx, order="F"), scaling


def pfwi_gradient_exact(vel, wav, dobs, nb, coef, dz, dx, dt, geo, ns, weight=None,
                        precision="f64"):
    """Exact discrete adjoint gradient dJ/dv and J (FP64 by default)."""
    R = np.float32 if precision == "f32" else np.float64
    nz, nx = vel.shape
    nt = len(wav)
    v = np.ascontiguousarray(np.asarray(vel, np.float64).flatten(order="F").astype(R))
    w = np.ascontiguousarray(np.asarray(wav, np.float64).astype(R))
    wt = None if weight is None else np.ascontiguousarray(np.asarray(weight).astype(R))
    g = np.zeros(nz * nx, R)
    J = getattr(lib(), "or_pfwi_gradient_exact_" + precision)(
        nz, nx, nb, dz, dx, nt, dt, coef, *_geo_args(geo, ns), v, w,
        _dobs_flat(dobs, R), None if wt is None else wt.ctypes.data, g)
    return g.reshape(nz, nx, order="F"), float(J)


def pfwi_misfit(vel, wav, dobs, nb, coef, dz, dx, dt, geo, ns, weight=None, precision="f64"):
    R = np.float32 if precision == "f32" else np.float64
    nz, nx = vel.shape
    nt = len(wav)
    v = np.ascontiguousarray(np.asarray(vel, np.float64).flatten(order="F").astype(R))
    w = np.ascontiguousarray(np.asarray(wav, np.float64).astype(R))
    wt = None if weight is None else np.ascontiguousarray(np.asarray(weight).astype(R))
    return float(getattr(lib(), "or_pfwi_misfit_" + precision)(
        nz, nx, nb, dz, dx, nt, dt, coef, *_geo_args(geo, ns), v, w, _dobs_flat(dobs, R),
        None if wt is None else wt.ctypes.data))


# --------------------------------------------------------------------------
# 3-D extension of the pfwi scheme (pw_oracle3d_body.h; no reference 3-D FWI)
# --------------------------------------------------------------------------

def _geo3(vel, g):
    nz, nx, ny = vel.shape
    src = np.ascontiguousarray(np.asarray(g["src"], np.int32).reshape(-1))
    rx = np.ascontiguousarray(np.asarray(g["rx"], np.int32))
    ry = np.ascontiguousarray(np.asarray(g["ry"], np.int32))
    return (nz, nx, ny, int(g["nb"]), float(g["dz"]), float(g["dx"]), float(g["dy"]),
            int(g["nt"]), float(g["dt"]), float(g["coef"]), len(src) // 3, src, int(g["rz"]),
            len(rx), len(ry), rx, ry)


def _vel3(vel, R):
    # (nz, nx, ny) -> [ny][nx][nz]
    return np.ascontiguousarray(np.asarray(vel, np.float32).transpose(2, 1, 0).astype(R))


def pf3_forward(vel, wav, g, precision="f32"):
    """3-D forward modelling; vel (nz, nx, ny); g: dict nb, dz, dx, dy, nt, dt,
    coef, src [(z, x, y)], rz, rx, ry.  Returns data [ns][nry*nrx][nt]."""
    R = np.float32 if precision == "f32" else np.float64
    geo = _geo3(vel, g)
    ns, nr, nt = geo[10], geo[13] * geo[14], geo[7]
    out = np.zeros(ns * nr * nt, R)
    getattr(lib(), "or_pf3_forward_" + precision)(*geo, _vel3(vel, R),
                                                 np.ascontiguousarray(np.asarray(wav).astype(R)),
                                                 out)
    return out.reshape(ns, nr, nt)


def pf3_gradient_exact(vel, wav, dobs, g, weight=None, precision="f64"):
    """Exact adjoint gradient dJ/dv (nz, nx, ny) and J (whole history in host
    memory: small grids only)."""
    R = np.float32 if precision == "f32" else np.float64
    geo = _geo3(vel, g)
    nz, nx, ny = vel.shape
    grad = np.zeros(nz * nx * ny, R)
    wt = None if weight is None else np.ascontiguousarray(np.asarray(weight).astype(R))
    J = getattr(lib(), "or_pf3_gradient_exact_" + precision)(
        *geo, _vel3(vel, R), np.ascontiguousarray(np.asarray(wav).astype(R)),
        np.ascontiguousarray(np.asarray(dobs).astype(R).reshape(-1)),
        None if wt is None else wt.ctypes.data, grad)
    return grad.reshape(ny, nx, nz).transpose(2, 1, 0), float(J)


def pf3_misfit(vel, wav, dobs, g, weight=None, precision="f64"):
    R = np.float32 if precision == "f32" else np.float64
    geo = _geo3(vel, g)
    wt = None if weight is None else np.ascontiguousarray(np.asarray(weight).astype(R))
    return float(getattr(lib(), "or_pf3_misfit_" + precision)(
        *geo, _vel3(vel, R), np.ascontiguousarray(np.asarray(wav).astype(R)),
        np.ascontiguousarray(np.asarray(dobs).astype(R).reshape(-1)),
        None if wt is None else wt.ctypes.data))


# --------------------------------------------------------------------------
# pfwi passive mode 4: timerev_lop and the LS-TRI inversion
# (pw_oracle_lstri_body.h; wave_triutil.c:48-316, wave_fwi.c:121,
# wave_bigsolver.c:1170, wave_cgstep.c:16)
# --------------------------------------------------------------------------

def _vel2(vel):
    # (nz, nx) -> [nx][nz]
    return np.ascontiguousarray(np.asarray(vel, np.float32).T)


def timerev(adj, vel, nt, nb, coef, dz, dx, dt, rz=1, mod=None, dat=None, precision="f32"):
    """One application of timerev_lop: adj=False maps mod (nz, nx, nt) to
    data (nt, nx); adj=True maps dat (nt, nx) to mod (nz, nx, nt)."""
    R = np.float32 if precision == "f32" else np.float64
    nz, nx = np.shape(vel)
    if adj:
        d = np.ascontiguousarray(np.asarray(dat).astype(R).T)  # [nx][nt]
        m = np.zeros(nt * nx * nz, R)
    else:
        m = np.ascontiguousarray(np.asarray(mod).astype(R).transpose(2, 1, 0))  # [nt][nx][nz]
        d = np.zeros(nx * nt, R)
    getattr(lib(), "or_timerev_" + precision)(int(adj), nz, nx, nt, nb, rz, dt, dx, dz, coef,
                                              _vel2(vel), m.reshape(-1), d.reshape(-1))
    if adj:
        return m.reshape(nt, nx, nz).transpose(2, 1, 0)
    return d.reshape(nx, nt).T


def lstri(inv, vel, par, src=None, data=None, precision="f32"):
    """pfwicfun.lstric restated: inv=0 maps src (nz, nx, nt, ns) to data
    (nt, nx, ns); inv=1 inverts data for src with par['niter'] CG
    iterations per shot.  par: nz, nx, dz, dx, nt, dt, ns, nb, coef, niter.
    Returns (result, iterations per shot)."""
    R = np.float32 if precision == "f32" else np.float64
    nz, nx = np.shape(vel)
    nt, ns = int(par["nt"]), int(par["ns"])
    if inv:
        d = np.ascontiguousarray(np.asarray(data).astype(R).reshape(nt, nx, ns).transpose(2, 1, 0))
        s = np.zeros((ns, nt, nx, nz), R)
    else:
        s = np.ascontiguousarray(np.asarray(src).astype(R).reshape(nz, nx, nt, ns)
                                 .transpose(3, 2, 1, 0))
        d = np.zeros((ns, nx, nt), R)
    iters = np.zeros(ns, np.int32)
    getattr(lib(), "or_lstri_" + precision)(
        int(inv), nz, nx, nt, ns, int(par["nb"]), int(par.get("rz", 1)), float(par["dt"]),
        float(par["dx"]), float(par["dz"]), float(par["coef"]), int(par.get("niter", 0)),
        _vel2(vel), s.reshape(-1), d.reshape(-1), iters.ctypes.data)
    if inv:
        return s.transpose(3, 2, 1, 0), iters
    return d.transpose(2, 1, 0), iters


# --------------------------------------------------------------------------
# pseudo-spectral propagator psm2d / psm (wave_psp.c:25-635, aps.c glue),
# restated in FP64 with numpy's FFT (the reference runs KISS FFT in float)
# --------------------------------------------------------------------------

def psm(vel, nt, dt, d, nbt=30, ct=0.01, src=None, tri=False, dat=None, jsnap=0, rick=None):
    """aps2d / aps3d in FP64: vel (nz,nx) or (nz,nx,ny), d (dz,dx[,dy]).
    The expanded grid (nbt cells on every face, edge-replicated velocity) is
    padded for the FFT to nz2 = 2*next_fast((nz+1)/2), nx2 = next_fast(nx),
    ny2 = next_fast(ny).  Per step: wave = sign * IFFT(lapl * FFT(sign *
    curr)) with sign = (-1)^(ix [+ iy]) (the reference's FFT centering) and
    lapl = -(2 pi |k|)^2 on the centred grid kx = -0.5/dx + ix/(nx2 dx),
    kz = iz/(nz2 dz); then curr' = 2 curr - prev + wave vv on the expanded
    grid, the 3x3(x3) source spread (or, time-reversed, the traces on row
    nbt), the taper on curr and prev (abc_apply over the padded grid, bottom
    and right faces counted from the padded size), traces and snapshots.
    Returns (traces, snapshots) shaped as oracle.afd returns them."""
    vel = np.asarray(vel, np.float64)
    dim = vel.ndim
    if dim == 2:
        vel = vel[:, :, None]
        dz, dx = d
        dy = 1.0
    else:
        dz, dx, dy = d
    nz1, nx1, ny1 = vel.shape
    nb = nbt
    nby = nb if dim == 3 else 0
    nz, nx, ny = nz1 + 2 * nb, nx1 + 2 * nb, ny1 + 2 * nby
    ez = np.clip(np.arange(nz) - nb, 0, nz1 - 1)
    ex = np.clip(np.arange(nx) - nb, 0, nx1 - 1)
    ey = np.clip(np.arange(ny) - nby, 0, ny1 - 1)
    ve = vel[np.ix_(ez, ex, ey)]
    vv = ve * ve * dt * dt
    nz2 = 2 * next_fast((nz + 1) // 2)
    nx2 = next_fast(nx)
    ny2 = next_fast(ny) if dim == 3 else 1
    kz = np.arange(nz2 // 2 + 1) / (nz2 * dz)
    kx = -0.5 / dx + np.arange(nx2) / (nx2 * dx)
    ky = (-0.5 / dy + np.arange(ny2) / (ny2 * dy)) if dim == 3 else np.zeros(1)
    K = np.sqrt(kz[:, None, None] ** 2 + kx[None, :, None] ** 2 + ky[None, None, :] ** 2)
    lapl = -(2 * np.pi * K) ** 2
    sign = ((-1.0) ** (np.arange(nx2)[:, None] + np.arange(ny2)[None, :]))[None, :, :]
    w = np.exp(-(ct ** 2) * (nb - 1 - np.arange(nb)) ** 2) if nb else np.zeros(0)

    def taper(a):
        for ib in range(nb):
            a[ib, :, :] *= w[ib]
            a[nz2 - 1 - ib, :, :] *= w[ib]
        for ib in range(nb):
            a[:, ib, :] *= w[ib]
            a[:, nx2 - 1 - ib, :] *= w[ib]
        if dim == 3:
            for ib in range(nb):
                a[:, :, ib] *= w[ib]
                a[:, :, ny2 - 1 - ib] *= w[ib]

    axes = (1, 2) if dim == 3 else (1,)
    curr = np.zeros((nz2, nx2, ny2))
    prev = np.zeros((nz2, nx2, ny2))
    ntsnap = _ntsnap(nt, jsnap)
    snaps = np.zeros((nz1, nx1, ny1, max(ntsnap, 1)))
    traces = np.zeros((nt, nx1, ny1))
    if tri:
        dd = np.asarray(dat, np.float64).reshape(nt, nx1, ny1)
        steps = range(nt - 1, -1, -1)
    else:
        sx = np.asarray(src["sx"]).astype(np.float32).astype(int)
        sz = np.asarray(src["sz"]).astype(np.float32).astype(int)
        sy = np.asarray(src.get("sy", np.zeros_like(sx))).astype(np.float32).astype(int)
        if rick is None:
            rick = np.stack([ricker(nt, dt, src["f"][i], src["t"][i], src["A"][i])
                             for i in range(len(sx))])
        steps = range(nt)
    for it in steps:
        spec = np.fft.rfft(curr * sign, axis=0)
        for ax in axes:
            spec = np.fft.fft(spec, axis=ax)
        spec = spec * lapl
        for ax in axes:
            spec = np.fft.ifft(spec, axis=ax)
        wave = np.fft.irfft(spec, n=nz2, axis=0).real * sign
        c = curr[:nz, :nx, :ny]
        new = c + (c - prev[:nz, :nx, :ny]) + wave[:nz, :nx, :ny] * vv
        prev[:nz, :nx, :ny] = c
        curr[:nz, :nx, :ny] = new
        if tri:
            curr[nb, nb:nb + nx1, nby:nby + ny1] += vv[nb, nb:nb + nx1, nby:nby + ny1] * dd[it]
        else:
            for i in range(len(sx)):
                for jy in ((-1, 0, 1) if dim == 3 else (0,)):
                    for jx in (-1, 0, 1):
                        for jz in (-1, 0, 1):
                            z_, x_, y_ = sz[i] + nb + jz, sx[i] + nb + jx, sy[i] + nby + jy
                            den = abs(jx) + abs(jz) + abs(jy) + 1
                            curr[z_, x_, y_] += vv[z_, x_, y_] * rick[i][it] / den
        taper(curr)
        taper(prev)
        if not tri:
            traces[it] = curr[nb, nb:nb + nx1, nby:nby + ny1]
        if jsnap > 0 and it % jsnap == 0:
            snaps[..., it // jsnap] = curr[nb:nb + nz1, nb:nb + nx1, nby:nby + ny1]
    if dim == 2:
        traces, snaps = traces[:, :, 0], snaps[:, :, 0, :]
    return (None if tri else traces), (snaps if ntsnap > 0 else None)
