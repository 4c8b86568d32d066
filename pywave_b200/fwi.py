"""FWI gradient on the GPU engine: the reference's gradient_av imaging and the
exact discrete adjoint, and a ``torch.autograd.Function`` mapping velocity to
the data misfit.

The exact adjoint back-propagates the weighted residual with the forward
scheme's own transpose (sponge and edge-replicated padding included) and
images with the zero-lag condition fused into the adjoint step kernel:
    dJ/dv = pad2d^T( 2/v * sum_n phi_n * (Lap8 a_n + r w_n) ).
Memory is capped by checkpoints of the forward state every k steps and a
per-segment recompute; with ``ckpt_k=0`` the planner picks k and the shots
per batch within an HBM budget (``hbm_budget`` bytes, default a quarter of
the device), minimising the recomputed forward steps.

Arrays follow pfwi: velocity (nz, nx), wavelet (nt,), data (nt, nr, ns).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L

try:
    import torch
except ImportError:  # pragma: no cover
    torch = None


def fwi_args(par, flags=0, hbm_budget=0):
    """pw_fwi_args from a pfwi ``par`` dictionary (after fillpar);
    ``hbm_budget`` bytes bound the exact gradient's working set (0: a quarter
    of the device)."""
    from .pfwi import pararray, fillpar
    arr = pararray(fillpar(dict(par)))
    a = L.FwiArgs()
    L.check(L.lib().pw_fwi_args_from_pararray(L.ptr(arr), int(arr.size), a))
    a.flags = flags
    a.hbm_budget = int(hbm_budget)
    return a


def _data_flat(dobs):
    # (nt, nr, ns) -> [ns][nr][nt]
    return np.ascontiguousarray(np.asarray(dobs, np.float32).flatten(order="F"))


def gradient(vel, wav, dobs, par, mode="exact", ckpt_k=0, per_shot=False, weight=None,
             hbm_budget=0):
    """FWI gradient dJ/dv (nz, nx) and the FP64 misfit, host arrays in/out.

    mode "reference": gradient_av's imaging (wave_fwigradient.c:93-242) before
    its smoothing / scaling; misfit 0.5*sum((dobs-d)^2).
    mode "exact": exact adjoint of the scheme; misfit 0.5*sum(w*(d-dobs)^2);
    checkpoint interval ckpt_k, or planned within hbm_budget bytes when 0
    (pywave_b200._lib.last_fwi_plan reports the plan).
    weight: (nr, nt) residual weights, default the reference's tapers."""
    flags = L.PW_HOST_PTRS | (L.PW_PER_SHOT if per_shot else 0)
    a = fwi_args(par, flags, hbm_budget)
    v = np.ascontiguousarray(np.asarray(vel, np.float32).flatten(order="F"))
    w = np.ascontiguousarray(np.asarray(wav, np.float32).reshape(-1))
    d = _data_flat(dobs)
    wt = None if weight is None else np.ascontiguousarray(np.asarray(weight, np.float32))
    g = np.empty(a.nz * a.nx, np.float32)
    J = ctypes.c_double(0.0)
    m = L.PW_GRAD_EXACT if mode == "exact" else L.PW_GRAD_REFERENCE
    L.check(L.lib().pw_pfwi_gradient(a, m, L.ptr(v), L.ptr(w), L.ptr(d), L.ptr(wt), L.ptr(g),
                                     ctypes.byref(J), int(ckpt_k), None))
    return g.reshape(a.nz, a.nx, order="F"), J.value


def gradient_passive(vel, src, dobs, par, mode="reference", ckpt_k=0, per_shot=False,
                     weight=None, hbm_budget=0, flo=0.0, fhi=0.0):
    """The same gradient with distributed sources (pfwi's passive mode 4,
    gradient_pas_av, wave_fwigradient.c:667-870): src (nz, nx, nt, ns)
    source fields in place of the point source and wavelet.  flo, fhi (Hz):
    the multiscale residual filter (3-pole zero-phase Butterworth high- /
    low-pass, wave_fwigradient.c:767-780), reference mode only; 0 = off."""
    flags = L.PW_HOST_PTRS | (L.PW_PER_SHOT if per_shot else 0)
    a = fwi_args(par, flags, hbm_budget)
    a.flo, a.fhi = float(flo), float(fhi)
    v = np.ascontiguousarray(np.asarray(vel, np.float32).flatten(order="F"))
    sv = np.ascontiguousarray(np.asarray(src, np.float32).flatten(order="F"))  # [ns][nt][nx][nz]
    if sv.size != a.nz * a.nx * a.nt * a.ns:
        raise L.ShapeError(L.PW_ERR_SHAPE, "src must hold nz*nx*nt*ns values")
    d = _data_flat(dobs)
    wt = None if weight is None else np.ascontiguousarray(np.asarray(weight, np.float32))
    g = np.empty(a.nz * a.nx, np.float32)
    J = ctypes.c_double(0.0)
    m = L.PW_GRAD_EXACT if mode == "exact" else L.PW_GRAD_REFERENCE
    L.check(L.lib().pw_pfwi_gradient_passive(a, m, L.ptr(v), L.ptr(sv), L.ptr(d), L.ptr(wt),
                                             L.ptr(g), ctypes.byref(J), int(ckpt_k), None))
    return g.reshape(a.nz, a.nx, order="F"), J.value


def forward_visco(vel, q, wav, par):
    """Visco-acoustic forward modelling (forward_modeling,
    wave_fwimodeling.c:116-220): vel, q (nz, nx), par a pfwi parameter dict
    (its f0 sets the relaxation times); returns data (nt, nr, ns)."""
    a = fwi_args(par, L.PW_HOST_PTRS)
    v = np.ascontiguousarray(np.asarray(vel, np.float32).flatten(order="F"))
    qq = np.ascontiguousarray(np.asarray(q, np.float32).flatten(order="F"))
    w = np.ascontiguousarray(np.asarray(wav, np.float32).reshape(-1))
    out = np.empty(a.ns * a.nx * a.nt, np.float32)
    L.check(L.lib().pw_pfwi_forward_visco(a, L.ptr(v), L.ptr(qq), L.ptr(w), L.ptr(out), None))
    return out.reshape(a.nt, a.nx, a.ns, order="F")


def gradient_visco(vel, q, wav, dobs, par, weight=None):
    """Visco-acoustic gradient_v (wave_fwigradient.c:264-452) before its
    smoothing / scaling, and the FP64 misfit 0.5*sum((dobs-d)^2)."""
    a = fwi_args(par, L.PW_HOST_PTRS)
    v = np.ascontiguousarray(np.asarray(vel, np.float32).flatten(order="F"))
    qq = np.ascontiguousarray(np.asarray(q, np.float32).flatten(order="F"))
    w = np.ascontiguousarray(np.asarray(wav, np.float32).reshape(-1))
    d = _data_flat(dobs)
    wt = None if weight is None else np.ascontiguousarray(np.asarray(weight, np.float32))
    g = np.empty(a.nz * a.nx, np.float32)
    J = ctypes.c_double(0.0)
    L.check(L.lib().pw_pfwi_gradient_visco(a, L.ptr(v), L.ptr(qq), L.ptr(w), L.ptr(d), L.ptr(wt),
                                           L.ptr(g), ctypes.byref(J), None))
    return g.reshape(a.nz, a.nx, order="F"), J.value


def postprocess(grad, rect=3, waterz=0, scaling=None):
    """gradient_av's tail: triangle smoothing and the (first-call) scale."""
    g = np.ascontiguousarray(np.asarray(grad, np.float32).flatten(order="F"))
    nz, nx = np.asarray(grad).shape
    sc = ctypes.c_float(0.0 if scaling is None else float(scaling))
    L.check(L.lib().pw_gradient_postprocess(nz, nx, rect, waterz, L.ptr(g), ctypes.byref(sc),
                                            L.PW_HOST_PTRS, None))
    return g.reshape(nz, nx, order="F"), sc.value


if torch is not None:

    class FwiMisfit(torch.autograd.Function):
        """J(v) = 0.5 * sum(w * (d(v) - dobs)^2) over all shots, J in FP64.

        forward(vel (nz, nx) CUDA float32, wav (nt,), dobs (ns, nr, nt) CUDA
        float32, par dict, ckpt_k) runs the forward and the exact adjoint in
        one pass and keeps dJ/dv for backward."""

        @staticmethod
        def forward(ctx, vel, wav, dobs, par, ckpt_k=0, weight=None, hbm_budget=0):
            a = fwi_args(par, 0, hbm_budget)
            v = vel.detach().t().contiguous().float()          # [nx][nz]
            w = wav.detach().contiguous().float()
            d = dobs.detach().contiguous().float()              # [ns][nr][nt]
            wt = None if weight is None else weight.detach().contiguous().float()
            g = torch.empty_like(v)
            J = ctypes.c_double(0.0)
            s = torch.cuda.current_stream(v.device).cuda_stream
            L.check(L.lib().pw_pfwi_gradient(a, L.PW_GRAD_EXACT, v.data_ptr(), w.data_ptr(),
                                             d.data_ptr(), None if wt is None else wt.data_ptr(),
                                             g.data_ptr(), ctypes.byref(J), int(ckpt_k), s))
            ctx.save_for_backward(g.t())
            return torch.tensor(J.value, dtype=torch.float64, device=vel.device)

        @staticmethod
        def backward(ctx, gJ):
            (g,) = ctx.saved_tensors
            return (g * gJ.to(g.dtype)), None, None, None, None, None, None

    def fwi_misfit(vel, wav, dobs, par, ckpt_k=0, weight=None, hbm_budget=0):
        """Differentiable misfit (see FwiMisfit); the checkpoints of the exact
        adjoint fit hbm_budget bytes (0: a quarter of the device)."""
        return FwiMisfit.apply(vel, wav, dobs, par, ckpt_k, weight, hbm_budget)


def residual_weights(nt, nr, wtn1=None, wtn2=None, woffn1=None, woffn2=None, oreo=False):
    """residual_weighting (wave_fwiutil.c:225-296) as an (nr, nt) array:
    the window defaults to the whole record (fwic's and pfwic's set-up)."""
    w = np.empty((nr, nt), np.float32)
    L.check(L.lib().pw_residual_weights(nt, nr, 0 if wtn1 is None else wtn1,
                                        nt - 1 if wtn2 is None else wtn2,
                                        0 if woffn1 is None else woffn1,
                                        nr - 1 if woffn2 is None else woffn2, int(oreo),
                                        L.ptr(w)))
    return w


def butter_apply(x, low, cutoff, npoles=3):
    """np_butter_apply (wave_butter.c) on the GPU: each row of x (traces
    [ntr][n]) filtered causally by a Butterworth low- or high-pass of npoles
    poles at cutoff cycles per sample; returns a new array."""
    y = np.ascontiguousarray(np.array(x, dtype=np.float32, ndmin=2))
    L.check(L.lib().pw_butter_apply(y.shape[-1], y.size // y.shape[-1], int(low), float(cutoff),
                                    int(npoles), L.ptr(y), L.PW_HOST_PTRS, None))
    return y.reshape(np.shape(x))
