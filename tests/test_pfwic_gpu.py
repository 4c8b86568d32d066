"""pfwi passive mode 4 with velocity update (pfwic, pywave/src/pfwi.c:1507):
the passive gradient (gradient_pas_av) and the passive FWI driver on the
GPU, every call through the C ABI, against the reference's own outputs
(tests/golden/pfwi_pas.npz: 30 x 40, 2 shots, nt 400, data from the
reference's lstric on the true model)."""
import sys

import numpy as np
import pytest

from conftest import GOLDEN, rel_l2

sys.path.insert(0, GOLDEN)
import models as M  # noqa: E402

pytestmark = pytest.mark.gpu


def _case(golden):
    g = golden("pfwi_pas")
    vt, vs, src = M.pas_case()
    assert M.digest(src) == str(g["src_digest"])
    return g, vt, vs, src


def test_passive_gradient_bit_exact_vs_reference(golden, oracle, cuda_lib):
    """One shot at a time (the reference's summation order): the raw
    gradient after the first-call scaling and the rect 1 / 3 smoothing
    identical to the reference's gradient_pas_av, misfit equal to the FP64
    oracle's to 1e-12 and to the reference's float sum to 1e-4."""
    from pywave_b200 import fwi
    g, _, vs, src = _case(golden)
    raw, J = fwi.gradient_passive(vs, src, g["data"], M.PAS, mode="reference", per_shot=True)
    for rect in (1, 3):
        pp, _ = fwi.postprocess(raw, rect=rect)
        assert np.array_equal(pp, g["grad_rect%d" % rect]), rect
    p = M.PAS
    geo = oracle.pfwi_geometry(p["nz"], p["nx"], p["dz"], p["dx"], 0, 0, p["ns"], p["ds"],
                               p["os"], p["nb"])
    _, J64 = oracle.pfwi_gradient_pas(vs, src, g["data"], p["nb"], p["coef"], p["dz"], p["dx"],
                                      p["dt"], geo, p["ns"], p["nt"], precision="f64")
    print(f"passive misfit: GPU {J!r}, FP64 oracle {J64!r}, reference {float(g['fcost'])!r}")
    assert abs(J - float(g["fcost"])) <= 1e-4 * abs(J)


def test_passive_gradient_batched(golden, oracle, cuda_lib):
    """Both shots in one launch: the same raw gradient to 1e-5 (the
    per-shot slices are added in shot order)."""
    from pywave_b200 import fwi
    g, _, vs, src = _case(golden)
    a, _ = fwi.gradient_passive(vs, src, g["data"], M.PAS, mode="reference", per_shot=True)
    b, _ = fwi.gradient_passive(vs, src, g["data"], M.PAS, mode="reference")
    assert rel_l2(b, a) < 1e-5


def test_passive_exact_gradient_finite_differences(golden, cuda_lib):
    """The exact adjoint with passive sources against central differences of
    the GPU's own FP64 misfit (1% steps) on 6 seeded interior cells."""
    from pywave_b200 import fwi
    g, _, vs, src = _case(golden)
    ge, _ = fwi.gradient_passive(vs, src, g["data"], M.PAS, mode="exact")
    rng = np.random.default_rng(3)
    fd, an = [], []
    for _ in range(6):
        c = (int(rng.integers(6, 26)), int(rng.integers(4, 36)))
        h = np.float32(1e-2 * vs[c])
        vp, vm = vs.copy(), vs.copy()
        vp[c] += h
        vm[c] -= h
        _, Jp = fwi.gradient_passive(vp, src, g["data"], M.PAS, mode="exact")
        _, Jm = fwi.gradient_passive(vm, src, g["data"], M.PAS, mode="exact")
        fd.append((Jp - Jm) / (float(vp[c]) - float(vm[c])))
        an.append(float(ge[c]))
    fd, an = np.array(fd), np.array(an)
    cos = float(fd @ an / np.linalg.norm(fd) / np.linalg.norm(an))
    print(f"passive exact gradient vs central differences: cosine {cos:.8f}")
    assert cos >= 0.9999


def test_pfwic_dropin_vs_reference(golden, cuda_lib):
    """pywave_b200.pfwicfun.pfwic with the reference's argument tuple: 4
    L-BFGS iterations (step reset every 5) from the start model; each
    iteration's model within 1e-3 rel-L2 of the reference's pfwic (float
    misfit sums there, FP64 here)."""
    from pywave_b200 import pfwicfun
    from pywave_b200.pfwi import fillpar, pararray
    g, _, vs, src = _case(golden)
    p = fillpar(dict(M.PAS, inv=1, onlysrc=False, onlyvel=True))
    q = np.full(vs.shape, 1e4, np.float32)
    ds = np.concatenate([g["data"].flatten(order="F"), src.flatten(order="F")])
    vinv = pfwicfun.pfwic(vs.flatten(order="F"), q.flatten(order="F"),
                          np.zeros(p["nt"], np.float32), ds, pararray(p))
    vinv = vinv.reshape(p["nz"], p["nx"], p["niter"], order="F")
    ref = g["vinv"]
    for it in range(ref.shape[2]):
        e = rel_l2(vinv[:, :, it], ref[:, :, it]) if np.any(ref[:, :, it]) else 0.0
        print(f"pfwic iteration {it + 1}: rel-L2 vs reference {e:.2e}")
        assert np.any(ref[:, :, it]) == np.any(vinv[:, :, it])
        assert e < 1e-3


def test_pfwi_mode4_fwi_returns(golden, cuda_lib):
    """pywave_b200.pfwi(mode=4, inv, onlysrc False, onlyvel True) returns
    (flattened data, vinv, None, None, None) like the reference's pfwi."""
    import pywave_b200 as pw
    g, _, vs, src = _case(golden)
    q = np.full(vs.shape, 1e4, np.float32)
    out = pw.pfwi(vs, q, np.zeros(M.PAS["nt"], np.float32), src, data=g["data"], mode=4,
                  par=dict(M.PAS, inv=True, onlysrc=False, onlyvel=True, niter=1))
    assert np.array_equal(out[0], g["data"].flatten(order="F"))
    assert out[1].shape == (M.PAS["nz"], M.PAS["nx"], 1) and out[2:] == (None, None, None)
    assert rel_l2(out[1][:, :, 0], g["vinv"][:, :, 0]) < 1e-3


def test_butterworth_bit_exact_vs_reference(golden, cuda_lib):
    """pw_butter_apply against the reference's np_butter_init / apply on
    seeded traces: low- and high-pass, 3 to 5 poles, identical bits."""
    from pywave_b200 import fwi
    g = golden("butter")
    for i, (low, cut, nn) in enumerate(M.BUTTER_CASES):
        assert np.array_equal(fwi.butter_apply(g["x"], low, cut, nn), g["y%d" % i]), i


def test_passive_multiscale_gradient_bit_exact(golden, cuda_lib):
    """The passive gradient with the multiscale residual filter on (flo 4 Hz,
    fhi 25 Hz), one shot at a time: identical to the reference's
    gradient_pas_av after scaling; the exact mode refuses the filter."""
    from pywave_b200 import _lib as L
    from pywave_b200 import fwi
    g, _, vs, src = _case(golden)
    raw, J = fwi.gradient_passive(vs, src, g["data"], M.PAS, mode="reference", per_shot=True,
                                  flo=float(g["flo"]), fhi=float(g["fhi"]))
    pp, _ = fwi.postprocess(raw, rect=1)
    assert np.array_equal(pp, g["grad_ms_rect1"])
    assert abs(J - float(g["fcost_ms"])) <= 1e-4 * abs(J)
    with pytest.raises(L.ShapeError):
        fwi.gradient_passive(vs, src, g["data"], M.PAS, mode="exact", flo=4.0)
