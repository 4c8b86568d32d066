"""Pins the oracle's restatement of the visco-acoustic pfwi path
(forward_modeling, gradient_v: oracle/pw_oracle_body.h) to the reference's
own outputs (tests/golden/visco.npz, produced through oracle/ref_driver.c:
the reference's Python glue cannot reach this path, pfwi.c:864).  CPU only."""
import sys

import numpy as np

from conftest import GOLDEN, rel_l2

sys.path.insert(0, GOLDEN)
import models as M  # noqa: E402


def _geo(oracle):
    p = M.VISCO
    geo = oracle.pfwi_geometry(p["nz"], p["nx"], p["dz"], p["dx"], 0, 0, p["ns"], p["ds"],
                               p["os"], p["nb"])
    return p, geo


def test_visco_forward_bit_exact(golden, oracle):
    g = golden("visco")
    vt, vs, q, wav = M.visco_case()
    assert np.array_equal(q, g["q"])
    p, geo = _geo(oracle)
    d = oracle.pfwi_forward_visco(vt, q, wav, p["nb"], p["coef"], p["dz"], p["dx"], p["dt"],
                                  p["f0"], geo, p["ns"])
    assert np.abs(d).max() > 0
    assert np.array_equal(d, g["data"])
    d64 = oracle.pfwi_forward_visco(vt, q, wav, p["nb"], p["coef"], p["dz"], p["dx"], p["dt"],
                                    p["f0"], geo, p["ns"], precision="f64")
    print(f"visco forward: float vs FP64 {rel_l2(d, d64):.2e}")
    assert rel_l2(d, d64) < 1e-4


def test_visco_gradient_bit_exact(golden, oracle):
    g = golden("visco")
    vt, vs, q, wav = M.visco_case()
    p, geo = _geo(oracle)
    raw, fcost = oracle.pfwi_gradient_visco(vs, q, wav, g["data"], p["nb"], p["coef"], p["dz"],
                                            p["dx"], p["dt"], p["f0"], geo, p["ns"])
    assert np.float32(fcost) == np.float32(g["fcost"])
    for rect in (1, 3):
        pp, _ = oracle.pfwi_postprocess(raw, rect=rect)
        assert np.array_equal(pp, g["grad_rect%d" % rect]), rect
