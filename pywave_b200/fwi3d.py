"""3-D FWI on the GPU engine: forward modelling and the exact-adjoint gradient
of the 3-D extension of pfwi's acoustic scheme (the reference has no 3-D
FWI; pywave/src/wave_fwimodeling.c:21-114 and wave_fwiutil.c:19-223 restated
on three axes, see include/pywave_b200.h pw_fwi3d_args).

A geometry is a dict: ``nb`` (sponge width), ``coef``, ``dz``, ``dx``, ``dy``,
``nt``, ``dt``, ``src`` (list of (z, x, y) interior indices, one per shot),
``rz`` (receiver depth), ``rx`` and ``ry`` (receiver columns and planes; the
receivers are the grid of every (rx[i], ry[j]), trace j * len(rx) + i).
Velocity (nz, nx, ny); data (ns, nr, nt).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L

try:
    import torch
except ImportError:  # pragma: no cover
    torch = None


def fwi3d_args(shape, geom, flags=0, hbm_budget=0):
    """(pw_fwi3d_args, the int arrays it points to); keep both alive."""
    nz, nx, ny = shape
    src = np.ascontiguousarray(np.asarray(geom["src"], np.int32).reshape(-1))
    rx = np.ascontiguousarray(np.asarray(geom["rx"], np.int32))
    ry = np.ascontiguousarray(np.asarray(geom["ry"], np.int32))
    ip = ctypes.POINTER(ctypes.c_int)
    a = L.Fwi3dArgs(nz=nz, nx=nx, ny=ny, dz=geom["dz"], dx=geom["dx"], dy=geom["dy"],
                    nt=geom["nt"], dt=geom["dt"], nb=geom["nb"], coef=geom["coef"],
                    ns=len(src) // 3, src=src.ctypes.data_as(ip), nrx=len(rx), nry=len(ry),
                    rx=rx.ctypes.data_as(ip), ry=ry.ctypes.data_as(ip), rz=geom["rz"],
                    flags=flags, hbm_budget=int(hbm_budget))
    return a, (src, rx, ry)


def _vel(vel):
    # (nz, nx, ny) -> [ny][nx][nz]
    return np.ascontiguousarray(np.asarray(vel, np.float32).flatten(order="F"))


def forward3d(vel, wav, geom):
    """Traces (ns, nr, nt) of every shot, host arrays in and out."""
    vel = np.asarray(vel, np.float32)
    a, keep = fwi3d_args(vel.shape, geom, L.PW_HOST_PTRS)
    ns, nr, nt = a.ns, a.nrx * a.nry, a.nt
    v = _vel(vel)
    w = np.ascontiguousarray(np.asarray(wav, np.float32).reshape(-1))
    out = np.empty(ns * nr * nt, np.float32)
    L.check(L.lib().pw_pfwi3d_forward(a, L.ptr(v), L.ptr(w), L.ptr(out), None))
    return out.reshape(ns, nr, nt)


def gradient3d(vel, wav, dobs, geom, weight=None, ckpt_k=0, hbm_budget=0):
    """Exact-adjoint gradient dJ/dv (nz, nx, ny) and the FP64 misfit
    J = 0.5 * sum(w * (d - dobs)^2); checkpoint interval ckpt_k, or planned
    within hbm_budget bytes when 0 (pywave_b200._lib.last_fwi_plan)."""
    vel = np.asarray(vel, np.float32)
    nz, nx, ny = vel.shape
    a, keep = fwi3d_args(vel.shape, geom, L.PW_HOST_PTRS, hbm_budget)
    v = _vel(vel)
    w = np.ascontiguousarray(np.asarray(wav, np.float32).reshape(-1))
    d = np.ascontiguousarray(np.asarray(dobs, np.float32).reshape(-1))
    wt = None if weight is None else np.ascontiguousarray(np.asarray(weight, np.float32))
    g = np.empty(nz * nx * ny, np.float32)
    J = ctypes.c_double(0.0)
    L.check(L.lib().pw_pfwi3d_gradient(a, L.ptr(v), L.ptr(w), L.ptr(d), L.ptr(wt), L.ptr(g),
                                       ctypes.byref(J), int(ckpt_k), None))
    return g.reshape(nz, nx, ny, order="F"), J.value


if torch is not None:

    class Fwi3dMisfit(torch.autograd.Function):
        """J(v) = 0.5 * sum(w * (d(v) - dobs)^2) over all shots of a 3-D
        geometry, in FP64; forward runs the forward and the exact adjoint in
        one pass and keeps dJ/dv for backward.  vel (nz, nx, ny) CUDA float32,
        wav (nt,), dobs (ns, nr, nt) CUDA float32."""

        @staticmethod
        def forward(ctx, vel, wav, dobs, geom, ckpt_k=0, hbm_budget=0):
            a, keep = fwi3d_args(tuple(vel.shape), geom, 0, hbm_budget)
            v = vel.detach().permute(2, 1, 0).contiguous().float()  # [ny][nx][nz]
            w = wav.detach().contiguous().float()
            d = dobs.detach().contiguous().float()
            g = torch.empty_like(v)
            J = ctypes.c_double(0.0)
            s = torch.cuda.current_stream(v.device).cuda_stream
            L.check(L.lib().pw_pfwi3d_gradient(a, v.data_ptr(), w.data_ptr(), d.data_ptr(), None,
                                               g.data_ptr(), ctypes.byref(J), int(ckpt_k), s))
            ctx.save_for_backward(g.permute(2, 1, 0))
            return torch.tensor(J.value, dtype=torch.float64, device=vel.device)

        @staticmethod
        def backward(ctx, gJ):
            (g,) = ctx.saved_tensors
            return (g * gJ.to(g.dtype)), None, None, None, None, None

    def fwi3d_misfit(vel, wav, dobs, geom, ckpt_k=0, hbm_budget=0):
        """Differentiable 3-D misfit (see Fwi3dMisfit)."""
        return Fwi3dMisfit.apply(vel, wav, dobs, geom, ckpt_k, hbm_budget)
