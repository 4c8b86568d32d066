"""Pins the oracle's restatement of pfwi's passive mode 4 (lstric:
timerev_lop and the np_solver / np_cgstep source inversion,
oracle/pw_oracle_lstri_body.h) to the reference's own outputs
(tests/golden/lstri.npz, generated by tests/golden/make_golden.py from the
reference compiled under oracle/_ref).  CPU only."""
import os
import sys

import numpy as np

from conftest import GOLDEN, rel_l2

sys.path.insert(0, GOLDEN)
import models as M  # noqa: E402


def _case(golden):
    g = golden("lstri")
    vel, src = M.lstri_case()
    assert np.array_equal(vel, g["vel"]) and M.digest(src) == str(g["src_digest"])
    return g, vel, src


def test_lstri_modelling_bit_exact(golden, oracle):
    g, vel, src = _case(golden)
    d, _ = oracle.lstri(0, vel, M.LSTRI, src=src)
    assert np.abs(d).max() > 0
    assert np.array_equal(d.view(np.uint32), g["data"].view(np.uint32))
    d64, _ = oracle.lstri(0, vel, M.LSTRI, src=src, precision="f64")
    print(f"lstri modelling: rel-L2 of the float result vs FP64 {rel_l2(d, d64):.2e}")
    assert rel_l2(d, d64) < 1e-4


def test_lstri_inversion_bit_exact(golden, oracle):
    """6 CG iterations per shot; the second shot starts from the first
    shot's step vectors, as the reference's statics do."""
    g, vel, _ = _case(golden)
    s, iters = oracle.lstri(1, vel, M.LSTRI, data=g["data"])
    assert list(iters) == [M.LSTRI["niter"]] * M.LSTRI["ns"]
    assert np.array_equal(s.view(np.uint32), g["srcinv"].view(np.uint32))
    # the carry-over is visible: shot 2 alone (fresh step vectors) differs
    alone, _ = oracle.lstri(1, vel, dict(M.LSTRI, ns=1), data=g["data"][:, :, 1:])
    assert np.array_equal(s[..., 0], oracle.lstri(1, vel, dict(M.LSTRI, ns=1),
                                                  data=g["data"][:, :, :1])[0][..., 0])
    assert not np.array_equal(alone[..., 0], s[..., 1])


def test_timerev_is_an_exact_adjoint_pair(oracle):
    """<A m, d> = <m, A' d> for the modelling / adjoint pair of timerev_lop
    (FP64 instance: to rounding; the float instance to 1e-5)."""
    rng = np.random.default_rng(0)
    nz, nx, nt, nb = 14, 18, 60, 6
    vel = (1.5 + rng.random((nz, nx))).astype(np.float32)
    m = rng.standard_normal((nz, nx, nt))
    d = rng.standard_normal((nt, nx))
    for prec, tol in (("f64", 1e-12), ("f32", 1e-4)):
        Am = oracle.timerev(False, vel, nt, nb, 0.05, 0.01, 0.01, 0.001, mod=m, precision=prec)
        Ad = oracle.timerev(True, vel, nt, nb, 0.05, 0.01, 0.01, 0.001, dat=d, precision=prec)
        a = float(np.sum(Am.astype(np.float64) * d))
        b = float(np.sum(m * Ad.astype(np.float64)))
        assert abs(a - b) <= tol * abs(a)


def _pas(golden, oracle):
    g = golden("pfwi_pas")
    vt, vs, src = M.pas_case()
    assert np.array_equal(vt, g["vtrue"]) and np.array_equal(vs, g["vstart"])
    assert M.digest(src) == str(g["src_digest"])
    p = M.PAS
    geo = oracle.pfwi_geometry(p["nz"], p["nx"], p["dz"], p["dx"], 0, 0, p["ns"], p["ds"],
                               p["os"], p["nb"])
    kw = dict(nb=p["nb"], coef=p["coef"], dz=p["dz"], dx=p["dx"], dt=p["dt"], geo=geo,
              ns=p["ns"], nt=p["nt"])
    return g, vs, src, kw


def test_gradient_pas_av_bit_exact(golden, oracle):
    """pfwic's passive gradient (gradient_pas_av with the source fields, the
    first-call scaling and the rect 1 / 3 smoothing) identical to the
    reference's, and its misfit."""
    g, vs, src, kw = _pas(golden, oracle)
    raw, fcost = oracle.pfwi_gradient_pas(vs, src, g["data"], **kw)
    assert np.float32(fcost) == np.float32(g["fcost"])
    for rect in (1, 3):
        pp, _ = oracle.pfwi_postprocess(raw, rect=rect)
        assert np.array_equal(pp, g["grad_rect%d" % rect])


def test_passive_multiscale_gradient_bit_exact(golden, oracle):
    """gradient_pas_av with the multiscale residual filter switched on
    (flo 4 Hz, fhi 25 Hz: 3-pole zero-phase high- and low-pass,
    wave_fwigradient.c:657-658,767-780) identical to the reference's."""
    g, vs, src, kw = _pas(golden, oracle)
    raw, fcost = oracle.pfwi_gradient_pas(vs, src, g["data"], flo=float(g["flo"]),
                                          fhi=float(g["fhi"]), **kw)
    assert np.float32(fcost) == np.float32(g["fcost_ms"])
    pp, _ = oracle.pfwi_postprocess(raw, rect=1)
    assert np.array_equal(pp, g["grad_ms_rect1"])
    assert not np.array_equal(pp, g["grad_rect1"])


def test_butterworth_and_weights_bit_exact(golden, oracle):
    """np_butter_init / np_butter_apply (wave_butter.c) for low- and high-pass
    filters of 3 to 5 poles, and residual_weighting in both branches
    (wave_fwiutil.c:225-296), identical to the reference's."""
    g = golden("butter")
    for i, (low, cut, nn) in enumerate(M.BUTTER_CASES):
        y = oracle.butter_apply(g["x"], low, cut, nn)
        assert np.array_equal(y, g["y%d" % i]), (low, cut, nn)
    nt, nr, wtn1, wtn2, woffn1, woffn2 = M.WEIGHT_CASE
    for oreo in (0, 1):
        w = oracle.residual_weights(nt, nr, wtn1, wtn2, woffn1, woffn2, oreo=bool(oreo))
        assert np.array_equal(w, g["w_oreo%d" % oreo]), oreo
