"""Pseudo-spectral propagation (aps2d / aps3d, pw_aps on cuFFT) against the
reference's own apscfun outputs (tests/golden/aps.npz) and the FP64
restatement (oracle.psm).  cuFFT and the reference's KISS FFT round
differently, so agreement is to float rounding: rel-L2 <= 1e-4 is asserted
(both sit ~5e-6 from FP64)."""
import sys

import numpy as np
import pytest

from conftest import GOLDEN, rel_l2

sys.path.insert(0, GOLDEN)
import models as M  # noqa: E402

pytestmark = pytest.mark.gpu


def test_aps2d_forward_vs_reference(golden, oracle, cuda_lib):
    import pywave_b200 as pw
    g = golden("aps")
    p = M.APS2
    d, w = pw.aps2d(g["v2"], ifsnaps=True, verb=False, **p)
    src = dict(sx=p["sx"], sz=p["sz"], f=p["f"], t=p["t"], A=p["A"])
    to, so = oracle.psm(g["v2"], p["nt"], p["dt"], (p["az"][1], p["ax"][1]), p["nbt"], p["ct"],
                        src=src, jsnap=p["jsnap"])
    print(f"aps2d GPU: traces vs reference {rel_l2(d, g['d2']):.2e}, vs FP64 {rel_l2(d, to):.2e}; "
          f"snapshots vs reference {rel_l2(w, g['w2']):.2e}")
    assert d.shape == g["d2"].shape and w.shape == g["w2"].shape
    assert rel_l2(d, g["d2"]) < 1e-4 and rel_l2(w, g["w2"]) < 1e-4
    assert rel_l2(d, to) < 1e-4 and rel_l2(w, so) < 1e-4


def test_aps2d_tri_vs_reference(golden, cuda_lib):
    """Time reversal of half the traces: snapshots as the reference's, and
    the input traces echoed in the trace slot (aps.c keeps afd.c's output)."""
    import pywave_b200 as pw
    g = golden("aps")
    p = M.APS2
    kw = {k: p[k] for k in ("nt", "dt", "ax", "az", "nbt", "ct", "jsnap")}
    echo, w = pw.aps2d(g["v2"], tri=True, dat=g["dtri"], ifsnaps=True, verb=False, **kw)
    print(f"aps2d TRI: snapshots vs reference {rel_l2(w, g['wtri']):.2e}")
    assert np.array_equal(echo, g["dtri"])
    assert rel_l2(w, g["wtri"]) < 1e-4


def test_aps3d_forward_vs_reference(golden, cuda_lib):
    import pywave_b200 as pw
    g = golden("aps")
    p = M.APS3
    d, w = pw.aps3d(g["v3"], ifsnaps=True, verb=False, **p)
    print(f"aps3d GPU: traces vs reference {rel_l2(d, g['d3']):.2e}, "
          f"snapshots {rel_l2(w, g['w3']):.2e}")
    assert d.shape == g["d3"].shape and w.shape == g["w3"].shape
    assert rel_l2(d, g["d3"]) < 1e-4 and rel_l2(w, g["w3"]) < 1e-4


def test_apscfun_dropin_tuple(golden, cuda_lib):
    """apscfun.aps2dc with the reference's positional tuple (aps2d.py:72)
    returns traces then snapshots, as the reference's module does."""
    from pywave_b200 import apscfun
    g = golden("aps")
    p = M.APS2
    nx, nz = p["ax"][2], p["az"][2]
    source = np.concatenate([p["sx"], p["sz"], p["f"], p["t"], p["A"]]).astype(np.float32)
    out = apscfun.aps2dc(g["v2"].flatten(order="F"), source, 0, p["nt"], nx, nz, p["ns"], 0,
                         p["jsnap"], 1, 1, p["nbt"], p["ct"], p["dt"], 0.0, 10.0, 0.0, 10.0)
    nsn = (p["nt"] - 1) // p["jsnap"] + 1
    assert out.size == p["nt"] * nx + nz * nx * nsn
    d = out[:p["nt"] * nx].reshape(p["nt"], nx, order="F")
    assert rel_l2(d, g["d2"]) < 1e-4


def test_aps2d_reference_defaults_vs_fp64(oracle, cuda_lib):
    """aps2d's own defaults (81 x 81 at 20 m, nbt 30, nt 1501, 2 sources):
    traces and snapshots within 1e-4 of the FP64 restatement."""
    import pywave_b200 as pw
    rng = np.random.default_rng(5)
    vel = (2000.0 + 500.0 * rng.random((81, 81))).astype(np.float32)
    d, w = pw.aps2d(vel, verb=False)
    src = dict(sx=[30, 40], sz=[30, 40], f=[10, 10], t=[0.2, 0.35], A=[1, 2])
    to, so = oracle.psm(vel, 1501, 0.001, (20.0, 20.0), 30, 0.01, src=src, jsnap=4)
    print(f"aps2d defaults: traces vs FP64 {rel_l2(d, to):.2e}, snapshots {rel_l2(w, so):.2e}")
    assert rel_l2(d, to) < 1e-4 and rel_l2(w, so) < 1e-4
