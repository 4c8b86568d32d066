"""Drop-in for the reference's ``pfwicfun`` extension module (pywave/src/pfwi.c).

``forward_modeling_ac`` and ``fwic`` take the reference's positional
arguments (``(vel, q, wav, pararray)`` and ``(vel, q, wav, data, pararray)``,
pfwi.c:85 and :555) and return the same flat float32 arrays
(``nt*nx*ns`` traces, time fastest, shot slowest; ``nz*nx*niter`` models).
The quality factor ``q`` is read and ignored, as the acoustic path ignores it
(pfwi.c:864 sends every call to the acoustic gradient).  ``lstric``
(passive mode 4 without velocity update, pfwi.c:1031) takes
``(vel, q, wav, datasrc, pararray)`` and returns the data (``inv`` = 0) or
the inverted source field (``inv`` = 1); ``pfwic`` (passive FWI with the
sources known, pfwi.c:1507) takes the same tuple with ``datasrc`` the data
followed by the source fields and returns the model after each iteration.
"""
from __future__ import annotations

import numpy as np

from . import _lib as L


def _args(pararray, flags=L.PW_HOST_PTRS):
    par = L.f32(pararray).reshape(-1)
    if par.size < 20:
        raise L.ShapeError(L.PW_ERR_SHAPE, "pararray needs 20 values (pfwi.py:40-61)")
    a = L.FwiArgs()
    L.check(L.lib().pw_fwi_args_from_pararray(L.ptr(par), int(par.size), a))
    a.flags = flags
    return a


def forward_modeling_ac(vel, q, wav, pararray):
    """Acoustic modelling of every shot (pfwi.c:27-495 -> forward_modeling_a)."""
    a = _args(pararray)
    vel = L.f32(vel).reshape(-1)
    wav = L.f32(wav).reshape(-1)
    if vel.size != a.nz * a.nx or wav.size < a.nt:
        raise L.ShapeError(L.PW_ERR_SHAPE, "vel must hold nz*nx and wav nt values")
    out = np.empty(a.nt * a.nx * a.ns, np.float32)
    L.check(L.lib().pw_pfwi_forward(a, L.ptr(vel), L.ptr(wav), L.ptr(out), None))
    return out


def fwic(vel, q, wav, data, pararray):
    """Acoustic FWI from starting model ``vel`` (pfwi.c:497-1029 -> fwi)."""
    a = _args(pararray)
    vel = L.f32(vel).reshape(-1)
    wav = L.f32(wav).reshape(-1)
    data = L.f32(data).reshape(-1)
    if vel.size != a.nz * a.nx or data.size != a.nt * a.nx * a.ns:
        raise L.ShapeError(L.PW_ERR_SHAPE, "vel must hold nz*nx and data nt*nx*ns values")
    vinv = np.zeros(a.nz * a.nx * max(a.niter, 0), np.float32)
    import ctypes
    done = ctypes.c_int(0)
    L.check(L.lib().pw_fwi(a, L.ptr(vel), L.ptr(wav), L.ptr(data), L.ptr(vinv), ctypes.byref(done),
                           None))
    return vinv


def lstric(vel, q, wav, datasrc, pararray):
    """Passive least-squares time-reversal imaging (pfwi.c:1031-1444 -> lstri).

    ``pararray[9]`` (inv) = 0: ``datasrc`` is the source field of every shot
    (nz*nx*nt*ns, z fastest) and the result the data (nt*nx*ns, time
    fastest).  inv = 1: ``datasrc`` is the data and the result the source
    field inverted by ``pararray[19]`` (niter) conjugate-gradient iterations
    per shot.  ``q`` and ``wav`` are read and ignored (lstri uses neither)."""
    par = L.f32(pararray).reshape(-1)
    a = _args(par)
    inv = int(par[9])
    vel = L.f32(vel).reshape(-1)
    ds = L.f32(datasrc).reshape(-1)
    nm, nd = a.nz * a.nx * a.nt, a.nx * a.nt
    if vel.size != a.nz * a.nx:
        raise L.ShapeError(L.PW_ERR_SHAPE, "vel must hold nz*nx values")
    if inv:
        if ds.size != nd * a.ns:
            raise L.ShapeError(L.PW_ERR_SHAPE, "data must hold nt*nx*ns values")
        out = np.empty(nm * a.ns, np.float32)
        L.check(L.lib().pw_lstri_invert(a, L.ptr(vel), L.ptr(ds), L.ptr(out), None))
    else:
        if ds.size != nm * a.ns:
            raise L.ShapeError(L.PW_ERR_SHAPE, "src must hold nz*nx*nt*ns values")
        out = np.empty(nd * a.ns, np.float32)
        L.check(L.lib().pw_lstri_forward(a, L.ptr(vel), L.ptr(ds), L.ptr(out), None))
    return out


def pfwic(vel, q, wav, datasrc, pararray):
    """Passive-source FWI with known sources (pfwi.c:1507-2036 -> pfwi,
    wave_fwi.c:212-322, gradient_pas_av): ``datasrc`` is the data
    (nt*nx*ns, time fastest) followed by the source fields (nz*nx*nt*ns, z
    fastest), the result the model after each of ``pararray[19]`` (niter)
    L-BFGS iterations (nz*nx*niter, zero after an early stop).  ``q`` and
    ``wav`` are read and ignored.  With ``pararray[9]`` (inv) = 0 the
    reference returns an unset array; here that raises ``ValueError``."""
    par = L.f32(pararray).reshape(-1)
    a = _args(par)
    if int(par[9]) == 0:
        raise L.ShapeError(L.PW_ERR_VALUE, "pfwic needs inv = 1 (pfwi.c:1997-2018)")
    vel = L.f32(vel).reshape(-1)
    ds = L.f32(datasrc).reshape(-1)
    nd, nm = a.nt * a.nx * a.ns, a.nz * a.nx * a.nt * a.ns
    if vel.size != a.nz * a.nx or ds.size != nd + nm:
        raise L.ShapeError(L.PW_ERR_SHAPE, "vel must hold nz*nx and datasrc nt*nx*ns + "
                                           "nz*nx*nt*ns values")
    data = np.ascontiguousarray(ds[:nd])
    src = np.ascontiguousarray(ds[nd:])
    vinv = np.zeros(a.nz * a.nx * max(a.niter, 0), np.float32)
    import ctypes
    done = ctypes.c_int(0)
    L.check(L.lib().pw_pfwi_passive(a, L.ptr(vel), L.ptr(src), L.ptr(data), L.ptr(vinv),
                                    ctypes.byref(done), None))
    return vinv
