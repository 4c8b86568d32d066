"""Drop-in for the reference's ``apscfun`` extension module (pywave/src/aps.c).

``aps2dc`` / ``aps3dc`` take the reference's positional arguments (parse
formats aps.c:365 and aps.c:72, the same tuples as afdcfun's) and return the
same flat float32 array: ``nt*nx[*ny]`` traces (time fastest) followed by
the ``nz*nx[*ny]*ntsnap`` snapshots when ``jsnap > 0``; time reversal
returns the input traces in the trace slot, as the reference does.  The
propagator is the pseudo-spectral one of psm2d / psm (wave_psp.c) through
``pw_aps``; its FFTs are cuFFT's, so results match the reference's to float
rounding.  Size mismatches raise ``ValueError`` where the reference printed
and returned NULL.
"""
from __future__ import annotations

from .afdcfun import _run


def aps2dc(vel, source, tri, nt, nx, nz, ns, verb, jsnap, ifsnaps, abc, nbt, ct, dt, ox, dx,
           oz, dz, gz=0, wavelet=None):
    """2-D pseudo-spectral modelling / time reversal (aps.c:315-578 -> psm2d)."""
    return _run(2, vel, source, bool(tri), int(nt), int(nx), 1, int(nz), int(ns), int(jsnap),
                int(nbt), float(ct), float(dt), float(dx), 1.0, float(dz), int(gz), wavelet,
                entry="pw_aps")


def aps3dc(vel, source, tri, nt, nx, ny, nz, ns, verb, jsnap, ifsnaps, abc, nbt, ct, dt, ox, dx,
           oy, dy, oz, dz, gz=0, wavelet=None):
    """3-D pseudo-spectral modelling / time reversal (aps.c:22-313 -> psm)."""
    return _run(3, vel, source, bool(tri), int(nt), int(nx), int(ny), int(nz), int(ns),
                int(jsnap), int(nbt), float(ct), float(dt), float(dx), float(dy), float(dz),
                int(gz), wavelet, entry="pw_aps")
