"""Pins the FP64 restatement of the pseudo-spectral propagator
(oracle.psm: psm2d / psm, pywave/src/wave_psp.c) to the reference's own
apscfun outputs (tests/golden/aps.npz).  The reference transforms with a
float KISS FFT, so agreement is to float rounding.  CPU only."""
import sys

import numpy as np

from conftest import GOLDEN, rel_l2

sys.path.insert(0, GOLDEN)
import models as M  # noqa: E402


def test_psm2d_forward_and_tri_vs_reference(golden, oracle):
    g = golden("aps")
    p = M.APS2
    assert np.array_equal(g["v2"], M.aps2_velocity())
    src = dict(sx=p["sx"], sz=p["sz"], f=p["f"], t=p["t"], A=p["A"])
    tr, sn = oracle.psm(g["v2"], p["nt"], p["dt"], (p["az"][1], p["ax"][1]), p["nbt"], p["ct"],
                        src=src, jsnap=p["jsnap"])
    print(f"psm2d FP64 vs reference: traces {rel_l2(tr, g['d2']):.2e}, "
          f"snapshots {rel_l2(sn, g['w2']):.2e}")
    assert rel_l2(tr, g["d2"]) < 2e-5 and rel_l2(sn, g["w2"]) < 2e-5
    _, st = oracle.psm(g["v2"], p["nt"], p["dt"], (p["az"][1], p["ax"][1]), p["nbt"], p["ct"],
                       tri=True, dat=g["dtri"], jsnap=p["jsnap"])
    assert rel_l2(st, g["wtri"]) < 2e-5


def test_psm3d_forward_vs_reference(golden, oracle):
    g = golden("aps")
    p = M.APS3
    assert np.array_equal(g["v3"], M.aps3_velocity())
    src = dict(sx=p["sx"], sy=p["sy"], sz=p["sz"], f=p["f"], t=p["t"], A=p["A"])
    tr, sn = oracle.psm(g["v3"], p["nt"], p["dt"], (10.0, 10.0, 10.0), p["nbt"], p["ct"],
                        src=src, jsnap=p["jsnap"])
    assert rel_l2(tr, g["d3"]) < 2e-5 and rel_l2(sn, g["w3"]) < 2e-5
