"""``aps2d`` and ``aps3d`` with the reference's signatures (pywave/aps2d.py:4,
pywave/aps3d.py:4): pseudo-spectral acoustic modelling or time reversal on
the GPU (``pw_aps``, cuFFT).  Outputs as afd2d / afd3d: traces (nt, nx[, ny])
and, when jsnap > 0, snapshots (nz, nx[, ny], ntsnap)."""
from __future__ import annotations

from .afd import _model2d, _model3d
from .apscfun import aps2dc, aps3dc


def aps2d(vel, nt=1501, dt=0.001, ax=[0, 20, 81], az=[0, 20, 81], ns=2, sx=[30, 40], sz=[30, 40],
          f=[10, 10], t=[0.2, 0.35], A=[1, 2], nbt=30, ct=0.01, jsnap=4, abc=True, ifsnaps=False,
          ps=True, tri=False, dat=None, verb=True, gz=0, wavelet=None):
    """2-D pseudo-spectral modelling / time reversal, as pywave.aps2d.
    vel: [nz, nx]."""
    return _model2d(aps2dc, vel, nt, dt, ax, az, ns, sx, sz, f, t, A, nbt, ct, jsnap, abc,
                    ifsnaps, tri, dat, verb, gz, wavelet)


def aps3d(vel, nt=1501, dt=0.001, ax=[0, 20, 81], ay=[0, 20, 81], az=[0, 20, 81], ns=3,
          sx=[30, 40, 50], sy=[30, 40, 50], sz=[30, 40, 50], f=[10, 10, 10], t=[0.2, 0.35, 0.5],
          A=[1, 2, 2], nbt=30, ct=0.01, jsnap=4, abc=True, ifsnaps=False, ps=True, tri=False,
          dat=None, verb=True, gz=0, wavelet=None):
    """3-D pseudo-spectral modelling / time reversal, as pywave.aps3d.
    vel: [nz, nx, ny]."""
    return _model3d(aps3dc, vel, nt, dt, ax, ay, az, ns, sx, sy, sz, f, t, A, nbt, ct, jsnap,
                    abc, ifsnaps, tri, dat, verb, gz, wavelet)
