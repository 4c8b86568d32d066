"""Seeded inputs shared by the golden-vector generator (make_golden.py, run
against the reference) and the tests that replay them on the GPU.  Only
numpy / scipy and the benchmark's own model generators: nothing here reads
the reference.  Where a fixture keeps only a digest of a large reference
output, the test rebuilds the inputs here and checks their digests first."""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def digest(a) -> str:
    """SHA-256 of an array's bytes in C order (dtype and shape as given)."""
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


# ---- afd3d on an 80 x 72 x 64 interior (untapered warp patches exist) ----
BIG3D = dict(nt=60, dt=0.001, ax=[0, 20, 72], ay=[0, 20, 64], az=[0, 20, 80], ns=2, sx=[30, 41],
             sy=[25, 38], sz=[40, 22], f=[25, 20], t=[0.012, 0.02], A=[1, 1.5], nbt=10, ct=0.02,
             jsnap=20)
BIG3D_BAND = (18, 36)   # x columns of the time-reversed receiver group
BIG3D_TRI_JSNAP = 4


def big3d_velocity():
    """80 x 72 x 64 (z, x, y) velocity: a 2000 -> 2600 m/s depth gradient plus
    seeded uniform noise of 200 m/s."""
    rng = np.random.default_rng(11)
    z = np.arange(80, dtype=np.float32)[:, None, None]
    return (2000 + 600 * z / 79 + 200 * rng.random((80, 72, 64))).astype(np.float32)


# ---- pfwi at the 300 x 600 FWI benchmark geometry and deeper ------------
def shallow_anomaly(v, cz, cx, r, amp):
    """v times (1 + amp * a Gaussian bump of radius r cells at (cz, cx)),
    clipped to [1.5, 4.5] km/s: a perturbation that short records see."""
    nz, nx = v.shape
    z = np.arange(nz)[:, None]
    x = np.arange(nx)[None, :]
    bump = np.exp(-((z - cz) ** 2 + (x - cx) ** 2) / (2.0 * r * r))
    return np.clip(v * (1.0 + amp * bump), 1.5, 4.5).astype(np.float32)


def pfwi_scale_case(name):
    """(vtrue, vstart, par, wavelet) of the pfwi scale fixtures.
    c4geo: the 300 x 600 benchmark models (bench.fwi2d_models(7)), nb 60
    (420 x 720 padded), 2 shots, nt 600.  deep: their left 200 columns
    extended by repeating the last 160 rows to 460 x 200 (580 x 320 padded,
    more than one z tile of the step kernel), 2 shots, nt 600.  The true
    model gets a +10% anomaly 30 cells deep under the first shot, which 0.6 s
    of data sees (the benchmark's own anomalies lie deeper than such a record
    reaches)."""
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    import bench
    vt, vs = bench.fwi2d_models(7)
    if name == "c4geo":
        nz, nx, nt = 300, 600, 600
    elif name == "deep":
        nz, nx, nt = 460, 200, 600
        vt = np.ascontiguousarray(np.concatenate([vt[:, :200], vt[-160:, :200]], axis=0))
        vs = np.ascontiguousarray(np.concatenate([vs[:, :200], vs[-160:, :200]], axis=0))
    else:
        raise KeyError(name)
    vt = shallow_anomaly(vt, 30, nx // 4, 12, 0.1)
    par = dict(nz=nz, nx=nx, dz=0.01, dx=0.01, oz=0.0, ox=0.0, nt=nt, dt=0.001, ot=0.0, ns=2,
               ds=nx * 0.01 / 2, os=nx * 0.01 / 4, nb=60, coef=0.005, f0=10.0, acqui_type=1,
               interval=1)
    return vt, vs, par, bench.fwi2d_wavelet(nt)


# ---- pfwi 60 x 120, 4 shots, nt 800: gradient cosine and 20 L-BFGS steps -
MID = dict(nz=60, nx=120, dz=0.01, dx=0.01, oz=0.0, ox=0.0, nt=800, dt=0.001, ot=0.0, ns=4,
           ds=0.3, os=0.15, nb=30, coef=0.005, f0=10.0, acqui_type=1, interval=1, niter=20)


def mid_models():
    """60 x 120 models at 10 m (km units): 4 seeded layers in [1.8, 3.2] km/s
    with a +8% Gaussian anomaly (true) and the true model smoothed with
    sigma 6 points (start)."""
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(5)
    nz, nx = 60, 120
    z = np.arange(nz)[:, None] + np.zeros((1, nx))
    x = np.zeros((nz, 1)) + np.arange(nx)[None, :]
    ifaces = np.sort(rng.choice(np.arange(10, nz - 5), 3, replace=False))
    vals = np.sort(rng.uniform(1.8, 3.2, 4))
    v = np.full((nz, nx), vals[0])
    for val, zi in zip(vals[1:], ifaces):
        v[z >= zi] = val
    v *= 1.0 + 0.08 * np.exp(-((z - 35) ** 2 + (x - 60) ** 2) / (2 * 8.0 ** 2))
    v = v.astype(np.float32)
    return v, gaussian_filter(v.astype(np.float64), 6.0).astype(np.float32)


def mid_wavelet(nt):
    """10 Hz Ricker peaking at 0.12 s, scaled by 1e6 as the reference's FWI
    demos scale theirs (demos/test_fwi_vel2d.py): fwic's line search compares
    the misfit with a gradient rescaled to 0.1 / max|g|, so it only makes
    progress when the data carry the demos' amplitude."""
    t = np.arange(nt) * 0.001 - 0.12
    a = (np.pi * 10.0 * t) ** 2
    return (1e6 * (1 - 2 * a) * np.exp(-a)).astype(np.float32)


# ---- passive mode 4 (lstric): distributed sources, 24 x 32, 2 shots -------
LSTRI = dict(nz=20, nx=24, dz=0.01, dx=0.01, oz=0.0, ox=0.0, nt=200, dt=0.001, ot=0.0, ns=2,
             ds=0.1, os=0.05, nb=20, coef=0.005, f0=15.0, acqui_type=1, interval=1, niter=6)


def lstri_case():
    """Velocity (nz, nx) and the source field src (nz, nx, nt, ns) of the
    pfwi mode-4 fixtures: per shot three point sources carrying seeded,
    delayed 15 Hz Ricker pulses of amplitude 1e3 (the demos scale theirs by
    1e6, demos/test_pfwi_vel2d.py)."""
    p = LSTRI
    rng = np.random.default_rng(9)
    nz, nx, nt, ns = p["nz"], p["nx"], p["nt"], p["ns"]
    z = np.arange(nz, dtype=np.float32)[:, None]
    vel = (1.8 + 0.6 * z / nz + 0.1 * rng.random((nz, nx))).astype(np.float32)
    t = np.arange(nt) * p["dt"]
    src = np.zeros((nz, nx, nt, ns), np.float32)
    for s in range(ns):
        for _ in range(3):
            iz, ix = int(rng.integers(5, nz - 3)), int(rng.integers(3, nx - 3))
            t0 = float(rng.uniform(0.03, 0.1))
            a = (np.pi * 15.0 * (t - t0)) ** 2
            src[iz, ix, :, s] += (1e3 * (1 - 2 * a) * np.exp(-a)).astype(np.float32)
    return vel, src


# ---- passive mode 4 with velocity update (pfwic): 30 x 40, 2 shots ---------
PAS = dict(nz=30, nx=40, dz=0.01, dx=0.01, oz=0.0, ox=0.0, nt=400, dt=0.001, ot=0.0, ns=2,
           ds=0.1, os=0.05, nb=20, coef=0.005, f0=10.0, acqui_type=1, interval=1, niter=4)
PAS_FLO, PAS_FHI = 4.0, 25.0  # multiscale cutoffs (Hz) of the filtered passive gradient

# Butterworth cases (low-pass?, cutoff in cycles per sample, poles) and a
# residual-weighting window (nt, nr, wtn1, wtn2, woffn1, woffn2)
BUTTER_CASES = [(1, 0.02, 3), (0, 0.004, 3), (1, 0.1, 4), (0, 0.05, 5)]
WEIGHT_CASE = (120, 50, 10, 100, 12, 40)


def pas_case():
    """True velocity (2.0 -> 2.6 km/s with depth and a +8% lens), the start
    model (the linear trend alone), and the source field (nz, nx, nt, ns):
    per shot three buried point sources carrying seeded, delayed 15 Hz
    Ricker pulses of amplitude 1e6 (the demos' scale,
    demos/test_pfwi_vel2d.py)."""
    p = PAS
    rng = np.random.default_rng(17)
    nz, nx, nt, ns = p["nz"], p["nx"], p["nt"], p["ns"]
    z = np.arange(nz, dtype=np.float32)[:, None]
    vs = (2.0 + 0.6 * z / nz + np.zeros((nz, nx))).astype(np.float32)
    iz, ix = np.ogrid[:nz, :nx]
    lens = ((iz - 14) / 5.0) ** 2 + ((ix - 20) / 8.0) ** 2 <= 1.0
    vt = np.where(lens, vs * 1.08, vs).astype(np.float32)
    t = np.arange(nt) * p["dt"]
    src = np.zeros((nz, nx, nt, ns), np.float32)
    for s in range(ns):
        for _ in range(3):
            jz, jx = int(rng.integers(18, nz - 3)), int(rng.integers(4, nx - 4))
            a = (np.pi * 15.0 * (t - float(rng.uniform(0.05, 0.12)))) ** 2
            src[jz, jx, :, s] += (1e6 * (1 - 2 * a) * np.exp(-a)).astype(np.float32)
    return vt, vs, src


# ---- pseudo-spectral aps2d / aps3d (apscfun) ------------------------------
APS2 = dict(nt=300, dt=0.001, ax=[0, 10, 60], az=[0, 10, 40], ns=2, sx=[20, 40], sz=[10, 15],
            f=[20, 20], t=[0.05, 0.08], A=[1, 2], nbt=20, ct=0.01, jsnap=10)
APS3 = dict(nt=120, dt=0.001, ax=[0, 10, 24], ay=[0, 10, 22], az=[0, 10, 20], ns=2, sx=[8, 15],
            sy=[9, 12], sz=[6, 10], f=[25, 25], t=[0.04, 0.06], A=[1, 2], nbt=8, ct=0.02,
            jsnap=10)


def aps2_velocity():
    """40 x 60: 2000 m/s over 2500 m/s at depth 20 with a seeded 3% texture."""
    rng = np.random.default_rng(31)
    v = np.full((40, 60), 2000.0, np.float32)
    v[20:] = 2500.0
    return (v * (1.0 + 0.03 * rng.random(v.shape))).astype(np.float32)


def aps3_velocity():
    """20 x 24 x 22: linear 1800 -> 2400 m/s with depth plus a seeded 3% texture."""
    rng = np.random.default_rng(32)
    z = np.arange(20, dtype=np.float32)[:, None, None]
    v = 1800.0 + 600.0 * z / 20 + np.zeros((20, 24, 22), np.float32)
    return (v * (1.0 + 0.03 * rng.random(v.shape))).astype(np.float32)


# ---- visco-acoustic pfwi (forward_modeling / gradient_v) --------------------
VISCO = dict(nz=30, nx=50, dz=0.01, dx=0.01, oz=0, ox=0, nt=400, dt=0.001, ot=0, ns=3, ds=0.15,
             os=0.05, nb=20, coef=0.005, f0=10, acqui_type=1, interval=1, niter=2)


def visco_case():
    """True velocity (2.0 / 2.5 / 3.0 km/s layers at 12 and 22), the start
    model (2.4 constant), a seeded quality factor between 20 and 80, and the
    10 Hz Ricker wavelet of the pfwi golden."""
    nz, nx, nt = VISCO["nz"], VISCO["nx"], VISCO["nt"]
    vt = np.full((nz, nx), 2.0, np.float32)
    vt[12:] = 2.5
    vt[22:] = 3.0
    vs = np.full((nz, nx), 2.4, np.float32)
    rng = np.random.default_rng(41)
    q = (20.0 + 60.0 * rng.random((nz, nx))).astype(np.float32)
    tt = np.arange(nt) * 0.001
    arg = (np.pi * 10 * (tt - 0.1)) ** 2
    wav = ((1 - 2 * arg) * np.exp(-arg)).astype(np.float32)
    return vt, vs, q, wav
