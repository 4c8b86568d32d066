"""Drop-in for the reference's ``afdcfun`` extension module (pywave/src/afd.c).

``afd2dc`` / ``afd3dc`` take the same positional arguments as the reference's
CPython functions (parse formats afd.c:366 and afd.c:73) and return the same
flat float32 array: ``nt*nx[*ny]`` traces (time fastest) followed by the
``nz*nx[*ny]*ntsnap`` snapshots when ``jsnap > 0`` (afd.c:551-576,
287-310).  Like the reference, time-reversal mode returns the input traces
unchanged in the trace slot (afd.c:470-479, 562-566): the TRI image is
available from :func:`pywave_b200.tri_image`.

Differences from the reference, all on error paths: sizes are validated and a
mismatch raises ``ValueError`` instead of printing and returning NULL
(afd.c:381-385); ``abc`` and ``ifsnaps`` are accepted and ignored exactly as
the reference ignores them (afd.c:98, 389).
"""
from __future__ import annotations

import numpy as np

from . import _lib as L


def _ntsnap(nt, jsnap):
    return (nt - 1) // jsnap + 1 if jsnap > 0 else 0


def _run(dim, vel, source, tri, nt, nx, ny, nz, ns, jsnap, nbt, ct, dt, dx, dy, dz,
         gz=0, wavelet=None, entry="pw_afd"):
    vel = L.f32(vel).reshape(-1)
    if vel.size != nz * nx * ny:
        raise L.ShapeError(L.PW_ERR_SHAPE,
                           f"Dimension mismatch, N_input = {vel.size}, N_data = {nz * nx * ny}")
    source = L.f32(source).reshape(-1)
    a = L.AfdArgs(dim=dim, nz=nz, nx=nx, ny=ny, nt=nt, nbt=nbt, ct=ct, dt=dt, dz=dz, dx=dx,
                  dy=dy, ns=0 if tri else ns, tri=1 if tri else 0, jsnap=max(jsnap, 0), gz=gz,
                  flags=L.PW_HOST_PTRS)
    ntsnap = _ntsnap(nt, jsnap)
    out = np.empty(nt * nx * ny + nz * nx * ny * ntsnap, np.float32)
    if tri:
        if source.size != nt * nx * ny:
            raise L.ShapeError(L.PW_ERR_SHAPE, f"TRI traces must hold nt*nx*ny = {nt * nx * ny} "
                                               f"values (got {source.size})")
        out[:nt * nx * ny] = source
        dat = None
    else:
        rows = 5 if dim == 2 else 6
        if source.size < rows * ns:
            raise L.ShapeError(L.PW_ERR_SHAPE, f"source array needs {rows}*ns values")
        dat = out[:nt * nx * ny]
    wfd = out[nt * nx * ny:] if ntsnap > 0 else None
    wav = None if wavelet is None else L.f32(wavelet).reshape(-1)
    fn = getattr(L.lib(), entry)
    L.check(fn(a, L.ptr(vel), L.ptr(source), L.ptr(wav), L.ptr(dat), L.ptr(wfd), None))
    return out


def afd2dc(vel, source, tri, nt, nx, nz, ns, verb, jsnap, ifsnaps, abc, nbt, ct, dt, ox, dx,
           oz, dz, gz=0, wavelet=None):
    """2-D afd modelling / time reversal (afd.c:316-578 -> fdm2d)."""
    return _run(2, vel, source, bool(tri), int(nt), int(nx), 1, int(nz), int(ns), int(jsnap),
                int(nbt), float(ct), float(dt), float(dx), 1.0, float(dz), int(gz), wavelet)


def afd3dc(vel, source, tri, nt, nx, ny, nz, ns, verb, jsnap, ifsnaps, abc, nbt, ct, dt, ox, dx,
           oy, dy, oz, dz, gz=0, wavelet=None):
    """3-D afd modelling / time reversal (afd.c:23-314 -> fdm)."""
    return _run(3, vel, source, bool(tri), int(nt), int(nx), int(ny), int(nz), int(ns),
                int(jsnap), int(nbt), float(ct), float(dt), float(dx), float(dy), float(dz),
                int(gz), wavelet)
