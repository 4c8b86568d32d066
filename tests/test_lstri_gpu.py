"""pfwi passive mode 4 (lstric) on the GPU, every call through the C ABI:
the time-reversal operator against the oracle (bit for bit, both kernel
paths), lstric's modelling and CG source inversion against the reference's
own outputs (tests/golden/lstri.npz), the drop-in module and pfwi mode 4,
and the demo-scale geometry (pywave demos/test_pfwi_mod2d.py: 130 x 334,
nb 60, nt 3001) against the oracle and through the adjoint identity."""
import os
import re
import sys

import numpy as np
import pytest

from conftest import GOLDEN, rel_l2

sys.path.insert(0, GOLDEN)
import models as M  # noqa: E402

pytestmark = pytest.mark.gpu

GEOMS = [  # nz, nx, nt, nb, rz, coef
    (14, 18, 60, 4, 1, 0.05),
    (13, 21, 37, 5, 2, 0.03),
    (20, 24, 50, 20, 1, 0.005),
]


def _par(nz, nx, nt, nb, rz, coef, ns=1, niter=3):
    return dict(nz=nz, nx=nx, dz=0.01, dx=0.012, oz=0, ox=0, nt=nt, dt=0.001, ot=0, ns=ns,
                ds=0.1, os=0.0, nb=nb, coef=coef, f0=10, acqui_type=1, interval=1,
                niter=niter, rz=rz)


def _model(nz, nx, seed):
    rng = np.random.default_rng(seed)
    return (1.5 + 2.0 * rng.random((nz, nx))).astype(np.float32)


def _plan(err):
    m = re.findall(r"lstri (\w+) plan: (resident|step)", err)
    assert m, "no lstri plan printed"
    return m


@pytest.mark.parametrize("resident", ["1", "0"])
@pytest.mark.parametrize("geom", GEOMS)
def test_timerev_bit_exact_vs_oracle(oracle, cuda_lib, monkeypatch, capfd, geom, resident):
    """Modelling and adjoint of timerev_lop, cluster-resident and
    step-per-launch kernels, against the FP32 oracle (the reference's float
    order): identical bits."""
    from pywave_b200 import lstri
    nz, nx, nt, nb, rz, coef = geom
    par = _par(*geom)
    vel = _model(nz, nx, 1)
    rng = np.random.default_rng(2)
    m = rng.standard_normal((nz, nx, nt)).astype(np.float32)
    d = rng.standard_normal((nt, nx)).astype(np.float32)
    monkeypatch.setenv("PW_LSTRI_VERBOSE", "1")
    monkeypatch.setenv("PW_LSTRI_RESIDENT", resident)
    dg = lstri.timerev(False, vel, par, mod=m)
    mg = lstri.timerev(True, vel, par, dat=d)
    plans = _plan(capfd.readouterr().err)
    assert all(p[1] == ("resident" if resident == "1" else "step") for p in plans)
    do = oracle.timerev(False, vel, nt, nb, coef, 0.01, 0.012, 0.001, rz=rz, mod=m)
    mo = oracle.timerev(True, vel, nt, nb, coef, 0.01, 0.012, 0.001, rz=rz, dat=d)
    assert np.abs(do).max() > 0 and np.abs(mo).max() > 0
    assert np.array_equal(dg.view(np.uint32), do.view(np.uint32))
    assert np.array_equal(mg.view(np.uint32), mo.view(np.uint32))


def test_lstric_dropin_bit_exact_vs_reference(golden, cuda_lib):
    """pywave_b200.pfwicfun.lstric with the reference's argument tuple:
    modelling (inv 0) and 6 CG iterations per shot (inv 1, the second shot
    continuing from the first shot's step vectors) identical to the
    reference's lstric."""
    from pywave_b200 import pfwicfun
    from pywave_b200.pfwi import fillpar, pararray
    g = golden("lstri")
    vel, src = M.lstri_case()
    assert M.digest(src) == str(g["src_digest"])
    q = np.full(vel.shape, 1e4, np.float32)
    wav = np.zeros(M.LSTRI["nt"], np.float32)
    p0 = fillpar(dict(M.LSTRI, inv=0))
    d = pfwicfun.lstric(vel.flatten(order="F"), q.flatten(order="F"), wav,
                        src.flatten(order="F"), pararray(p0))
    d = d.reshape(p0["nt"], p0["nx"], p0["ns"], order="F")
    assert np.array_equal(d.view(np.uint32), g["data"].view(np.uint32))
    p1 = fillpar(dict(M.LSTRI, inv=1))
    s = pfwicfun.lstric(vel.flatten(order="F"), q.flatten(order="F"), wav,
                        g["data"].flatten(order="F"), pararray(p1))
    s = s.reshape(p1["nz"], p1["nx"], p1["nt"], p1["ns"], order="F")
    print(f"lstric inversion: rel-L2 vs reference {rel_l2(s, g['srcinv']):.2e}")
    assert np.array_equal(s.view(np.uint32), g["srcinv"].view(np.uint32))


def test_pfwi_mode4_matches_reference(golden, cuda_lib):
    """pywave_b200.pfwi(mode=4) returns what the reference's pfwi returns:
    (data, [], [], [], []) for modelling, ([], None, None, src, []) for
    source inversion."""
    import pywave_b200 as pw
    g = golden("lstri")
    vel, src = M.lstri_case()
    q = np.full(vel.shape, 1e4, np.float32)
    wav = np.zeros(M.LSTRI["nt"], np.float32)
    out = pw.pfwi(vel, q, wav, src, mode=4, par=dict(M.LSTRI, inv=False))
    assert np.array_equal(out[0], g["data"]) and out[1:] == ([], [], [], [])
    out = pw.pfwi(vel, q, wav, src, data=g["data"], mode=4,
                  par=dict(M.LSTRI, inv=True, onlysrc=True))
    assert out[0] == [] and out[1] is None and out[2] is None and out[4] == []
    assert np.array_equal(out[3], g["srcinv"])


def test_multishot_launch_equals_single_shots(oracle, cuda_lib):
    """All shots of lstri_forward run as clusters of one launch (device
    pointers); each equals its own single-shot call."""
    import torch
    from pywave_b200 import lstri
    nz, nx, nt, nb = 20, 30, 80, 8
    par = _par(nz, nx, nt, nb, 1, 0.02, ns=5)
    vel = _model(nz, nx, 3)
    rng = np.random.default_rng(4)
    src = rng.standard_normal((5, nt, nx, nz)).astype(np.float32)  # [ns][nt][nx][nz]
    v = torch.tensor(np.ascontiguousarray(vel.T), device="cuda")
    s = torch.tensor(src, device="cuda")
    d = torch.empty((5, nx, nt), device="cuda")
    lstri.lstri_forward_torch(v, s, d, par)
    d = d.cpu().numpy()
    for i in range(5):
        one = lstri.timerev(False, vel, dict(par, ns=1), mod=src[i].transpose(2, 1, 0))
        assert np.array_equal(d[i].T, one)


def test_lstri_errors(cuda_lib):
    from pywave_b200 import _lib as L
    from pywave_b200 import lstri
    vel = _model(10, 12, 5)
    with pytest.raises(L.ShapeError):  # the stencil's rim needs nb >= 4
        lstri.timerev(False, vel, _par(10, 12, 20, 3, 1, 0.05), mod=np.zeros((10, 12, 20)))
    with pytest.raises(L.ShapeError):  # data row outside the stencil's rows
        lstri.timerev(False, vel, _par(10, 12, 20, 4, 11, 0.05), mod=np.zeros((10, 12, 20)))


# ------------------------------------------------------ demo-scale grid ----

SCALE = dict(nz=130, nx=334, dz=0.008, dx=0.012, oz=0, ox=0, nt=3001, dt=0.001, ot=0, ns=2,
             ds=0.1, os=0.0, nb=60, coef=0.005, f0=10, acqui_type=1, interval=1, niter=2)


def _scale_case():
    rng = np.random.default_rng(11)
    nz, nx, nt = SCALE["nz"], SCALE["nx"], SCALE["nt"]
    z = np.arange(nz, dtype=np.float32)[:, None]
    vel = (1.8 + 1.2 * z / nz + 0.2 * rng.random((nz, nx))).astype(np.float32)
    src = np.zeros((nz, nx, nt, SCALE["ns"]), np.float32)
    t = np.arange(nt) * SCALE["dt"]
    for s in range(SCALE["ns"]):
        for _ in range(3):
            iz, ix = int(rng.integers(60, 125)), int(rng.integers(20, 314))
            a = (np.pi * 10.0 * (t - float(rng.uniform(0.1, 0.5)))) ** 2
            src[iz, ix, :, s] = (1e6 * (1 - 2 * a) * np.exp(-a)).astype(np.float32)
    return vel, src


def test_scale_modelling_bit_exact_and_adjoint_identity(oracle, cuda_lib, monkeypatch, capfd):
    """130 x 334, nb 60 (250 x 454 padded), nt 3001, 2 shots in one
    resident launch: data identical to the FP32 oracle; the adjoint through
    the GPU pair satisfies <A m, d> = <m, A' d> to 1e-4 (FP32 sums over
    3001 steps; the FP64 oracle meets it to 1e-14)."""
    from pywave_b200 import lstri
    vel, src = _scale_case()
    monkeypatch.setenv("PW_LSTRI_VERBOSE", "1")
    d = lstri.lstri_forward(vel, src, SCALE)
    assert all(p[1] == "resident" for p in _plan(capfd.readouterr().err))
    do, _ = oracle.lstri(0, vel, SCALE, src=src)
    assert np.abs(do).max() > 0
    assert np.array_equal(d.view(np.uint32), do.view(np.uint32))
    rng = np.random.default_rng(12)
    dd = rng.standard_normal((SCALE["nt"], SCALE["nx"])).astype(np.float32)
    m = lstri.timerev(True, vel, dict(SCALE, ns=1), dat=dd)
    a = float(np.sum(d[:, :, 0].astype(np.float64) * dd))
    b = float(np.sum(src[..., 0].astype(np.float64) * m))
    print(f"adjoint identity at scale: {a:.6e} vs {b:.6e}, rel {abs(a - b) / abs(a):.2e}")
    assert abs(a - b) <= 1e-4 * abs(a)


def test_scale_inversion_vs_oracle(oracle, cuda_lib):
    """Source inversion, 2 CG iterations, one shot of the demo-scale grid,
    against the FP32 oracle (sequential FP64 dots there, block-order FP64 dots
    here; the float work is identical): rel-L2 <= 1e-5."""
    from pywave_b200 import lstri
    vel, src = _scale_case()
    par = dict(SCALE, ns=1)
    d, _ = oracle.lstri(0, vel, par, src=src[..., :1])
    s = lstri.lstri_invert(vel, d, par)
    so, iters = oracle.lstri(1, vel, par, data=d)
    assert list(iters) == [2]
    exact = np.array_equal(s.view(np.uint32), so.view(np.uint32))
    print(f"scale inversion: rel-L2 vs oracle {rel_l2(s, so):.2e}, bit-exact {exact}")
    assert rel_l2(s, so) <= 1e-5
