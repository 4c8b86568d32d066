"""Drop-in for the reference's ``pfwicfun`` extension module (pywave/src/pfwi.c).

``forward_modeling_ac`` and ``fwic`` take the reference's positional
arguments (``(vel, q, wav, pararray)`` and ``(vel, q, wav, data, pararray)``,
pfwi.c:85 and :555) and return the same flat float32 arrays
(``nt*nx*ns`` traces, time fastest, shot slowest; ``nz*nx*niter`` models).
The quality factor ``q`` is read and ignored, as the acoustic path ignores it
(pfwi.c:864 sends every call to the acoustic gradient).  The passive-source
entry points ``lstric`` and ``pfwic`` (mode 4) are not built on this engine
and raise ``NotImplementedError``.
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


def lstric(*args, **kwargs):
    raise NotImplementedError("passive least-squares TRI (pfwi mode=4, pfwi.c:1031) is not built")


def pfwic(*args, **kwargs):
    raise NotImplementedError("passive-source FWI (pfwi mode=4, pfwi.c:1507) is not built")
