"""ctypes binding of libpywave_b200.so (the C ABI declared in include/pywave_b200.h).

The shared library is the only compute path of the package.  If it is missing
or fails to load, every entry point raises ``RuntimeError``; there is no CPU
fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpywave_b200.so")

PW_OK = 0
PW_ERR_SHAPE = -1
PW_ERR_CFL = -2
PW_ERR_OOM = -3
PW_ERR_TIMEOUT = -4
PW_ERR_CUDA = -5
PW_ERR_VALUE = -6
PW_HOST_PTRS = 1
PW_NO_CFL_CHECK = 2
PW_PER_SHOT = 4
PW_GRAD_REFERENCE = 0
PW_GRAD_EXACT = 1


class PywaveError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class CFLError(PywaveError, ValueError):
    pass


class ShapeError(PywaveError, ValueError):
    pass


class DeviceTimeout(PywaveError):
    pass


class AfdArgs(C.Structure):
    _fields_ = [("dim", C.c_int), ("nz", C.c_int), ("nx", C.c_int), ("ny", C.c_int),
                ("nt", C.c_int), ("nbt", C.c_int), ("ct", C.c_float), ("dt", C.c_float),
                ("dz", C.c_float), ("dx", C.c_float), ("dy", C.c_float), ("ns", C.c_int),
                ("tri", C.c_int), ("jsnap", C.c_int), ("gz", C.c_int), ("flags", C.c_int)]


class FwiArgs(C.Structure):
    _fields_ = [("nz", C.c_int), ("nx", C.c_int), ("dz", C.c_float), ("dx", C.c_float),
                ("oz", C.c_float), ("ox", C.c_float), ("nt", C.c_int), ("dt", C.c_float),
                ("ot", C.c_float), ("ns", C.c_int), ("ds", C.c_float), ("os", C.c_float),
                ("nb", C.c_int), ("coef", C.c_float), ("f0", C.c_float),
                ("acqui_type", C.c_int), ("interval", C.c_int), ("niter", C.c_int),
                ("sz", C.c_int), ("rz", C.c_int), ("flags", C.c_int),
                ("hbm_budget", C.c_longlong), ("flo", C.c_float), ("fhi", C.c_float)]


class Fwi3dArgs(C.Structure):
    _fields_ = [("nz", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("dz", C.c_float),
                ("dx", C.c_float), ("dy", C.c_float), ("nt", C.c_int), ("dt", C.c_float),
                ("nb", C.c_int), ("coef", C.c_float), ("ns", C.c_int),
                ("src", C.POINTER(C.c_int)), ("nrx", C.c_int), ("nry", C.c_int),
                ("rx", C.POINTER(C.c_int)), ("ry", C.POINTER(C.c_int)), ("rz", C.c_int),
                ("flags", C.c_int), ("hbm_budget", C.c_longlong)]


_lib = None
_lock = threading.Lock()
_vp = C.c_void_p

# name -> (restype, argtypes); every array argument is a raw pointer (host or device)
_SIGS = {
    "pw_afd": (C.c_int, [C.POINTER(AfdArgs), _vp, _vp, _vp, _vp, _vp, _vp]),
    "pw_afd_noalloc": (C.c_int, [C.POINTER(AfdArgs), _vp, _vp, _vp, _vp, _vp, _vp]),
    "pw_afd_batch": (C.c_int, [C.c_int, _vp, _vp, _vp, _vp, _vp, _vp]),
    "pw_tri_image": (C.c_int, [C.POINTER(AfdArgs), C.c_int, _vp, _vp, _vp, _vp, C.c_int, _vp]),
    "pw_fwi_args_from_pararray": (C.c_int, [_vp, C.c_int, C.POINTER(FwiArgs)]),
    "pw_pfwi_forward": (C.c_int, [C.POINTER(FwiArgs), _vp, _vp, _vp, _vp]),
    "pw_pfwi_gradient": (C.c_int, [C.POINTER(FwiArgs), C.c_int, _vp, _vp, _vp, _vp, _vp, _vp,
                                   C.c_int, _vp]),
    "pw_gradient_postprocess": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, _vp, _vp, C.c_int,
                                          _vp]),
    "pw_fwi": (C.c_int, [C.POINTER(FwiArgs), _vp, _vp, _vp, _vp, C.POINTER(C.c_int), _vp]),
    "pw_pfwi3d_forward": (C.c_int, [C.POINTER(Fwi3dArgs), _vp, _vp, _vp, _vp]),
    "pw_pfwi3d_gradient": (C.c_int, [C.POINTER(Fwi3dArgs), _vp, _vp, _vp, _vp, _vp, _vp,
                                     C.c_int, _vp]),
    "pw_pfwi_gradient_passive": (C.c_int, [C.POINTER(FwiArgs), C.c_int, _vp, _vp, _vp, _vp, _vp,
                                           C.POINTER(C.c_double), C.c_int, _vp]),
    "pw_pfwi_passive": (C.c_int, [C.POINTER(FwiArgs), _vp, _vp, _vp, _vp, C.POINTER(C.c_int),
                                  _vp]),
    "pw_aps": (C.c_int, [C.POINTER(AfdArgs), _vp, _vp, _vp, _vp, _vp, _vp]),
    "pw_pfwi_forward_visco": (C.c_int, [C.POINTER(FwiArgs), _vp, _vp, _vp, _vp, _vp]),
    "pw_pfwi_gradient_visco": (C.c_int, [C.POINTER(FwiArgs), _vp, _vp, _vp, _vp, _vp, _vp,
                                         C.POINTER(C.c_double), _vp]),
    "pw_timerev": (C.c_int, [C.POINTER(FwiArgs), C.c_int, _vp, _vp, _vp, _vp]),
    "pw_butter_apply": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, _vp, C.c_int,
                                  _vp]),
    "pw_residual_weights": (C.c_int, [C.c_int] * 7 + [_vp]),
    "pw_lstri_forward": (C.c_int, [C.POINTER(FwiArgs), _vp, _vp, _vp, _vp]),
    "pw_lstri_invert": (C.c_int, [C.POINTER(FwiArgs), _vp, _vp, _vp, _vp]),
    "pw_last_fwi_plan": (C.c_int, [C.POINTER(C.c_int), C.POINTER(C.c_int),
                                   C.POINTER(C.c_longlong), C.POINTER(C.c_double)]),
    "pw_last_error": (C.c_char_p, []),
    "pw_version": (C.c_char_p, []),
    "pw_release_cache": (C.c_int, []),
    "pw_last_timing": (C.c_int, [C.POINTER(C.c_double), C.POINTER(C.c_longlong),
                                 C.POINTER(C.c_longlong)]),
}


def exported_symbols():
    """Names the C header declares (every one must be exported by the .so)."""
    return [k for k in _SIGS]


def lib():
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build it with `python -m pywave_b200.build` "
                    "(there is no CPU fallback)")
            L = C.CDLL(LIB_PATH)
            for name, (res, args) in _SIGS.items():
                if hasattr(L, name):
                    f = getattr(L, name)
                    f.restype = res
                    f.argtypes = args
            _lib = L
    return _lib


def check(rc: int):
    if rc == PW_OK:
        return
    msg = lib().pw_last_error().decode(errors="replace")
    cls = {PW_ERR_CFL: CFLError, PW_ERR_SHAPE: ShapeError, PW_ERR_TIMEOUT: DeviceTimeout,
           PW_ERR_VALUE: ShapeError}.get(rc, PywaveError)
    raise cls(rc, msg)


def ptr(a):
    """Raw address of a C-contiguous numpy array or a CUDA torch tensor.
    No reference is kept: the caller holds the array for the whole call."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
        return a.ctypes.data
    return a.data_ptr()


def last_timing():
    """(time-loop ms, step launches, all launches) of this thread's last call."""
    ms, n, t = C.c_double(), C.c_longlong(), C.c_longlong()
    lib().pw_last_timing(C.byref(ms), C.byref(n), C.byref(t))
    return ms.value, n.value, t.value


def last_fwi_plan():
    """(checkpoint interval, shots per batch, device bytes, recompute factor)
    of this thread's last exact gradient."""
    k, nsb, b, rc = C.c_int(), C.c_int(), C.c_longlong(), C.c_double()
    lib().pw_last_fwi_plan(C.byref(k), C.byref(nsb), C.byref(b), C.byref(rc))
    return k.value, nsb.value, b.value, rc.value


def f32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))
