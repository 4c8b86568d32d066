"""Python API of the afd propagator: ``afd2d``, ``afd3d`` (the reference's
signatures, pywave/afd2d.py:4 and pywave/afd3d.py:4) and ``tri_image``.

The keyword lists and return conventions are the reference's: traces are
returned as ``(nt, nx[, ny])`` and, when ``jsnap > 0``, snapshots as
``(nz, nx[, ny], ntsnap)`` (afd2d.py:75-90, afd3d.py:77-88).  Two optional
keywords are added at the end: ``gz`` (receiver depth below the top interior
row; the reference records at 0 only, afd.c:449) and ``wavelet`` (explicit
``[ns][nt]`` source time functions instead of the Ricker table).
"""
from __future__ import annotations

import numpy as np

from . import _lib as L
from .afdcfun import afd2dc, afd3dc, _ntsnap


def afd2d(vel, nt=1501, dt=0.001, ax=[0, 20, 81], az=[0, 20, 81], ns=2, sx=[30, 40], sz=[30, 40],
          f=[10, 10], t=[0.2, 0.35], A=[1, 2], nbt=30, ct=0.01, jsnap=4, abc=True, ifsnaps=False,
          ps=True, tri=False, dat=None, verb=True, gz=0, wavelet=None):
    """2-D acoustic finite-difference modelling (tri=False) or time-reversal
    propagation of ``dat`` (tri=True), as pywave.afd2d.  vel: [nz, nx]."""
    return _model2d(afd2dc, vel, nt, dt, ax, az, ns, sx, sz, f, t, A, nbt, ct, jsnap, abc,
                    ifsnaps, tri, dat, verb, gz, wavelet)


def _model2d(cfun, vel, nt, dt, ax, az, ns, sx, sz, f, t, A, nbt, ct, jsnap, abc, ifsnaps, tri,
             dat, verb, gz, wavelet):
    # the body of pywave's afd2d.py / aps2d.py around their C call
    vel = np.asarray(vel).flatten(order="F").astype(np.float32)
    ox, dx, nx = ax
    oz, dz, nz = az
    if tri:
        if dat is None:
            raise ValueError("tri=True needs dat (nt, nx)")
        source = np.asarray(dat).flatten(order="F").astype(np.float32)
    else:
        source = np.concatenate([np.array(sx), np.array(sz), np.array(f), np.array(t),
                                 np.array(A)], axis=0, dtype="float32")
    dout = cfun(vel, source, 1 if tri else 0, nt, nx, nz, ns, verb, jsnap, ifsnaps, abc, nbt,
                ct, dt, ox, dx, oz, dz, gz=gz, wavelet=wavelet)
    if jsnap > 0:
        ntsnap = _ntsnap(nt, jsnap)
        wfd = dout[nt * nx:].reshape(nz, nx, ntsnap, order="F")
        dout = dout[0:nt * nx].reshape(nt, nx, order="F")
        return dout, wfd
    return dout


def afd3d(vel, nt=1501, dt=0.001, ax=[0, 20, 81], ay=[0, 20, 81], az=[0, 20, 81], ns=3,
          sx=[30, 40, 50], sy=[30, 40, 50], sz=[30, 40, 50], f=[10, 10, 10], t=[0.2, 0.35, 0.5],
          A=[1, 2, 2], nbt=30, ct=0.01, jsnap=4, abc=True, ifsnaps=False, ps=True, tri=False,
          dat=None, verb=True, gz=0, wavelet=None):
    """3-D acoustic finite-difference modelling / time reversal, as
    pywave.afd3d.  vel: [nz, nx, ny]."""
    return _model3d(afd3dc, vel, nt, dt, ax, ay, az, ns, sx, sy, sz, f, t, A, nbt, ct, jsnap,
                    abc, ifsnaps, tri, dat, verb, gz, wavelet)


def _model3d(cfun, vel, nt, dt, ax, ay, az, ns, sx, sy, sz, f, t, A, nbt, ct, jsnap, abc, ifsnaps,
             tri, dat, verb, gz, wavelet):
    # the body of pywave's afd3d.py / aps3d.py around their C call
    vel = np.asarray(vel).flatten(order="F").astype(np.float32)
    ox, dx, nx = ax
    oy, dy, ny = ay
    oz, dz, nz = az
    if tri:
        if dat is None:
            raise ValueError("tri=True needs dat (nt, nx, ny)")
        source = np.asarray(dat).flatten(order="F").astype(np.float32)
    else:
        source = np.concatenate([np.array(sx), np.array(sy), np.array(sz), np.array(f),
                                 np.array(t), np.array(A)], axis=0, dtype="float32")
    dout = cfun(vel, source, 1 if tri else 0, nt, nx, ny, nz, ns, verb, jsnap, ifsnaps, abc,
                nbt, ct, dt, ox, dx, oy, dy, oz, dz, gz=gz, wavelet=wavelet)
    if jsnap > 0:
        ntsnap = _ntsnap(nt, jsnap)
        wfd = dout[nt * nx * ny:].reshape(nz, nx, ny, ntsnap, order="F")
        dout = dout[0:nt * nx * ny].reshape(nt, nx, ny, order="F")
        return dout, wfd
    return dout


def group_bands(nx: int, ngroups: int, ny: int = 1):
    """The TRI demos' receiver groups: x-bands of width nx//ngroups; columns
    beyond ngroups*(nx//ngroups) belong to no group (-1).  Returns an int32
    [ny, nx] array (C order, x fastest)."""
    dg = nx // ngroups
    gx = np.full(nx, -1, np.int32)
    if dg > 0:
        for g in range(ngroups):
            gx[g * dg:(g + 1) * dg] = g
    return np.ascontiguousarray(np.tile(gx, (ny, 1)))


def tri_image(vel, dat, dt=0.001, d=None, ngroups=4, groups=None, nbt=30, ct=0.01, jsnap=4,
              normalize=True):
    """Time-reversal source image of ``ngroups`` receiver groups propagated in
    lockstep: sum over snapshot steps of the product over groups of the
    squared wavefield, divided by its maximum (the TRI demos' image,
    demos/test_third_tri.py:61-77, computed in one fused GPU pass).

    vel: [nz, nx] or [nz, nx, ny]; dat: traces (nt, nx) or (nt, nx, ny) as
    afd2d/afd3d record them; d: grid spacing (dz, dx[, dy]);
    groups: [ny, nx] group id per receiver (-1 = unused), default x-bands.
    Returns the image [nz, nx(, ny)] (float32)."""
    vel = np.asarray(vel, np.float32)
    dim = vel.ndim
    if dim == 2:
        nz, nx = vel.shape
        ny = 1
    else:
        nz, nx, ny = vel.shape
    dat = np.asarray(dat, np.float32)
    nt = dat.shape[0]
    if d is None:
        d = (10.0,) * dim
    if len(d) != dim:
        raise ValueError("d needs one spacing per axis")
    dz, dx = float(d[0]), float(d[1])
    dy = float(d[2]) if dim == 3 else 1.0
    a = L.AfdArgs(dim=dim, nz=nz, nx=nx, ny=ny, nt=nt, nbt=nbt, ct=ct, dt=dt, dz=dz, dx=dx,
                  dy=dy, ns=0, tri=1, jsnap=jsnap, gz=0, flags=L.PW_HOST_PTRS)
    src = np.ascontiguousarray(dat.flatten(order="F"))
    if groups is None:
        groups = group_bands(nx, ngroups, ny)
    groups = np.ascontiguousarray(np.asarray(groups, np.int32).reshape(ny, nx))
    img = np.empty(nz * nx * ny, np.float32)
    vflat = np.ascontiguousarray(vel.flatten(order="F"))  # keep alive across the call
    L.check(L.lib().pw_tri_image(a, int(ngroups), L.ptr(groups), L.ptr(vflat), L.ptr(src),
                                 L.ptr(img), 1 if normalize else 0, None))
    return img.reshape((nz, nx) if dim == 2 else (nz, nx, ny), order="F")


def afd2d_batch(shots, stream=None):
    """Forward modelling of many 2-D shots of uneven size and length in one
    lockstep time loop (pw_afd_batch).  ``shots`` is a list of dicts with
    afd2d's keywords: ``vel`` [nz, nx], ``nt``, ``dt``, ``ax``, ``az``, ``ns``,
    ``sx``, ``sz``, ``f``, ``t``, ``A``, ``nbt``, ``ct`` and optionally ``gz``
    and ``wavelet`` [ns][nt].  Returns the list of gathers (nt, nx), each
    identical to what afd2d(..., jsnap=0) returns for that shot."""
    import ctypes as C
    n = len(shots)
    args = (L.AfdArgs * n)()
    keep, vp, sp, wp, dp = [], [], [], [], []
    outs = []
    any_wav = any(sh.get("wavelet") is not None for sh in shots)
    for k, sh in enumerate(shots):
        vel = L.f32(np.asarray(sh["vel"]).flatten(order="F"))
        ox, dx, nx = sh["ax"]
        oz, dz, nz = sh["az"]
        nt, ns = sh["nt"], sh["ns"]
        src = L.f32(np.concatenate([np.asarray(sh[key], np.float32).reshape(-1)
                                    for key in ("sx", "sz", "f", "t", "A")]))
        a = args[k]
        a.dim, a.nz, a.nx, a.ny, a.nt = 2, nz, nx, 1, nt
        a.nbt, a.ct, a.dt, a.dz, a.dx, a.dy = sh.get("nbt", 30), sh.get("ct", 0.01), sh["dt"], dz, dx, dx
        a.ns, a.tri, a.jsnap, a.gz, a.flags = ns, 0, 0, sh.get("gz", 0), L.PW_HOST_PTRS
        wav = sh.get("wavelet")
        wav = None if wav is None else L.f32(wav)
        out = np.empty(nt * nx, np.float32)
        keep += [vel, src, wav, out]
        vp.append(vel.ctypes.data)
        sp.append(src.ctypes.data)
        wp.append(None if wav is None else wav.ctypes.data)
        dp.append(out.ctypes.data)
        outs.append((out, nt, nx))
    VP = (C.c_void_p * n)(*vp)
    SP = (C.c_void_p * n)(*sp)
    WP = (C.c_void_p * n)(*wp) if any_wav else None
    DP = (C.c_void_p * n)(*dp)
    L.check(L.lib().pw_afd_batch(n, C.cast(args, C.c_void_p), C.cast(VP, C.c_void_p),
                                 C.cast(SP, C.c_void_p),
                                 None if WP is None else C.cast(WP, C.c_void_p),
                                 C.cast(DP, C.c_void_p), stream))
    return [o.reshape(nt, nx, order="F") for o, nt, nx in outs]
