"""pywave_b200: B200-native acoustic finite-difference propagator, time-reversal
imaging and FWI gradient with the call signatures of chenyk1990/pywave.

Drop-in entry points (pywave/__init__.py re-exports the same names):
  afd2d, afd3d   -- pywave/afd2d.py:4, pywave/afd3d.py:4
  aps2d, aps3d   -- pywave/aps2d.py:4, pywave/aps3d.py:4 (pseudo-spectral, cuFFT)
  pfwi, fillpar  -- pywave/pfwi.py:5, :262
Additions on the same engine:
  tri_image      -- fused lockstep multi-group TRI image
  fwi.gradient   -- FWI gradient: the reference's imaging or the exact adjoint
  fwi.fwi_misfit / fwi.FwiMisfit -- torch.autograd.Function velocity -> misfit
  pfwi(mode=2)   -- L-BFGS FWI with FP64 inner products on the GPU

All compute runs in libpywave_b200.so (hand-written sm_100a CUDA behind a C
ABI, include/pywave_b200.h); nothing falls back to the CPU.
"""
from .afd import afd2d, afd3d, tri_image, group_bands  # noqa: F401
from .aps import aps2d, aps3d  # noqa: F401
from . import _lib  # noqa: F401

try:  # pfwi needs nothing beyond numpy, but keep the afd API importable alone
    from .pfwi import pfwi, fillpar  # noqa: F401
    from . import fwi  # noqa: F401
except ImportError:  # pragma: no cover
    pass

__all__ = ["afd2d", "afd3d", "aps2d", "aps3d", "tri_image", "group_bands", "pfwi", "fillpar",
           "fwi"]
