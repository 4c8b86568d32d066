"""pfwi's passive mode 4 on the GPU engine: the time-reversal operator
``timerev_lop`` (pywave/src/wave_triutil.c:86-180) and lstric's modelling and
least-squares source inversion (pfwi.c:1031, wave_fwi.c:121,
wave_fwigradient.c:454-520), through the C ABI (``pw_timerev``,
``pw_lstri_forward``, ``pw_lstri_invert``).

Arrays use the reference's Python shapes: velocity (nz, nx), source fields
(nz, nx, nt) per shot or (nz, nx, nt, ns), data (nt, nx) or (nt, nx, ns).
``par`` is a pfwi parameter dict (``fillpar`` fills the defaults; ``rz`` is 1
as in the reference).  Torch CUDA tensors in the C layout go straight to the
device entry points (``timerev_torch``, ``lstri_forward_torch``,
``lstri_invert_torch``).
"""
from __future__ import annotations

import numpy as np

from . import _lib as L
from .pfwi import fillpar, pararray

try:
    import torch
except ImportError:  # pragma: no cover
    torch = None


def lstri_args(par, flags=L.PW_HOST_PTRS):
    """pw_fwi_args for mode 4 from a pfwi parameter dict."""
    p = fillpar(dict(par))
    arr = pararray(p)
    a = L.FwiArgs()
    L.check(L.lib().pw_fwi_args_from_pararray(L.ptr(arr), int(arr.size), a))
    a.rz = int(p.get("rz", 1))
    a.flags = flags
    return a


def _vel(vel):
    return np.ascontiguousarray(np.asarray(vel, np.float32).T)  # (nz, nx) -> [nx][nz]


def timerev(adj, vel, par, mod=None, dat=None):
    """One application of timerev_lop (add = false) for one shot: adj=False
    maps mod (nz, nx, nt) to data (nt, nx); adj=True maps dat (nt, nx) to
    mod (nz, nx, nt)."""
    a = lstri_args(par)
    v = _vel(vel)
    nz, nx, nt = a.nz, a.nx, a.nt
    if adj:
        d = np.ascontiguousarray(np.asarray(dat, np.float32).T)  # [nx][nt]
        m = np.empty((nt, nx, nz), np.float32)
    else:
        m = np.ascontiguousarray(np.asarray(mod, np.float32).transpose(2, 1, 0))  # [nt][nx][nz]
        d = np.empty((nx, nt), np.float32)
    L.check(L.lib().pw_timerev(a, int(adj), L.ptr(v), L.ptr(m), L.ptr(d), None))
    return m.transpose(2, 1, 0) if adj else d.T


def lstri_forward(vel, src, par):
    """Data (nt, nx, ns) of the source fields src (nz, nx, nt, ns)."""
    a = lstri_args(par)
    s = np.asarray(src, np.float32).reshape(a.nz, a.nx, a.nt, a.ns)
    s = np.ascontiguousarray(s.transpose(3, 2, 1, 0))
    d = np.empty((a.ns, a.nx, a.nt), np.float32)
    v = _vel(vel)  # held here: ptr() keeps no reference
    L.check(L.lib().pw_lstri_forward(a, L.ptr(v), L.ptr(s), L.ptr(d), None))
    return d.transpose(2, 1, 0)


def lstri_invert(vel, data, par):
    """Source fields (nz, nx, nt, ns) inverted from data (nt, nx, ns) by
    par['niter'] conjugate-gradient iterations per shot."""
    a = lstri_args(par)
    d = np.asarray(data, np.float32).reshape(a.nt, a.nx, a.ns)
    d = np.ascontiguousarray(d.transpose(2, 1, 0))
    s = np.empty((a.ns, a.nt, a.nx, a.nz), np.float32)
    v = _vel(vel)
    L.check(L.lib().pw_lstri_invert(a, L.ptr(v), L.ptr(d), L.ptr(s), None))
    return s.transpose(3, 2, 1, 0)


if torch is not None:

    def _dev(t):
        assert t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()
        return t.data_ptr()

    def timerev_torch(adj, vel_xz, par, mod, dat):
        """Device form: vel [nx][nz], mod [nt][nx][nz], dat [nx][nt] CUDA
        float32 tensors; writes dat (adj=False) or mod (adj=True)."""
        a = lstri_args(par, 0)
        s = torch.cuda.current_stream(vel_xz.device).cuda_stream
        L.check(L.lib().pw_timerev(a, int(adj), _dev(vel_xz), _dev(mod), _dev(dat), s))

    def lstri_forward_torch(vel_xz, src, data, par):
        """Device form of lstri_forward: src [ns][nt][nx][nz] in, data
        [ns][nx][nt] out."""
        a = lstri_args(par, 0)
        s = torch.cuda.current_stream(vel_xz.device).cuda_stream
        L.check(L.lib().pw_lstri_forward(a, _dev(vel_xz), _dev(src), _dev(data), s))

    def lstri_invert_torch(vel_xz, data, src, par):
        """Device form of lstri_invert: data [ns][nx][nt] in, src
        [ns][nt][nx][nz] out."""
        a = lstri_args(par, 0)
        s = torch.cuda.current_stream(vel_xz.device).cuda_stream
        L.check(L.lib().pw_lstri_invert(a, _dev(vel_xz), _dev(data), _dev(src), s))
