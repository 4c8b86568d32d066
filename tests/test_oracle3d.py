"""The 3-D oracle (oracle/pw_oracle3d_body.h): its FP64 exact adjoint against
central differences of its FP64 misfit, and its FP32 forward against its
FP64 forward.  CPU only.  (The reference has no 3-D FWI; these checks pin
the 3-D restatement the GPU tests compare with.)"""
import numpy as np


def _case():
    rng = np.random.default_rng(1)
    nz, nx, ny = 14, 16, 12
    vt = (2.0 + 0.3 * rng.random((nz, nx, ny))).astype(np.float32)
    vs = np.full((nz, nx, ny), 2.1, np.float32)
    nt = 150
    t = np.arange(nt) * 0.001 - 0.05
    a = (np.pi * 20 * t) ** 2
    wav = ((1 - 2 * a) * np.exp(-a)).astype(np.float32)
    g = dict(nb=6, dz=0.01, dx=0.01, dy=0.01, nt=nt, dt=0.001, coef=0.02,
             src=[(3, 5, 4), (3, 10, 7)], rz=1, rx=[2, 5, 8, 11, 13], ry=[1, 4, 7, 10])
    return vt, vs, wav, g


def test_exact_adjoint_3d_matches_finite_differences(oracle):
    vt, vs, wav, g = _case()
    d = oracle.pf3_forward(vt, wav, g, "f64")
    assert np.abs(d).max() > 0
    gr, J = oracle.pf3_gradient_exact(vs, wav, d, g)
    assert J > 0
    fd, an = [], []
    for c in [(5, 7, 5), (8, 3, 6), (2, 12, 3), (10, 9, 8), (6, 6, 2), (11, 14, 10)]:
        h = 1e-4 * float(vs[c])
        vp = vs.astype(np.float64)
        vm = vp.copy()
        vp[c] += h
        vm[c] -= h
        fd.append((oracle.pf3_misfit(vp, wav, d, g) - oracle.pf3_misfit(vm, wav, d, g)) / (2 * h))
        an.append(gr[c])
    fd, an = np.array(fd), np.array(an)
    cos = float(fd @ an / np.linalg.norm(fd) / np.linalg.norm(an))
    assert cos >= 0.99999
    assert np.max(np.abs(fd - an)) <= 1e-3 * np.max(np.abs(an))


def test_fp32_forward_3d_close_to_fp64(oracle):
    vt, _, wav, g = _case()
    d32 = oracle.pf3_forward(vt, wav, g, "f32").astype(np.float64)
    d64 = oracle.pf3_forward(vt, wav, g, "f64")
    assert np.linalg.norm(d32 - d64) <= 1e-5 * np.linalg.norm(d64)
