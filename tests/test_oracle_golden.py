"""Pins the oracle restatement (oracle/pw_oracle.c) to golden vectors produced
by the reference itself (tests/golden/make_golden.py).  CPU only."""
import numpy as np
import pytest

from conftest import rel_l2


def _src(g, three=False):
    s = dict(sx=g["sx"], sz=g["sz"], f=g["f"], t=g["t"], A=g["A"])
    if three:
        s["sy"] = g["sy"]
    return s


def test_padding_rule(oracle):
    # kiss_fft_next_fast_size and fft2_init's first-axis rule
    assert [oracle.next_fast(n) for n in (1, 7, 131, 135, 751, 1021)] == [1, 8, 135, 135, 768, 1024]
    assert oracle.lib().or_pad_first(261) == 270
    assert oracle.lib().or_pad_first(101) == 108  # 101^3 expanded -> 108^3 padded


def test_ricker_matches_reference_table(golden, oracle):
    g = golden("afd2d_fwd")
    for i in range(2):
        mine = oracle.ricker(int(g["nt"]), float(g["dt"]), float(g["f"][i]), float(g["t"][i]),
                             float(g["A"][i]))
        ref = g["rick"][i]
        # the reference evaluates the same DFT with a float KISS FFT
        assert np.max(np.abs(mine - ref)) <= 2e-7 * np.max(np.abs(ref))


def test_afd2d_bit_exact_given_reference_wavelet(golden, oracle):
    g = golden("afd2d_fwd")
    tr, sn = oracle.afd(g["vel"], int(g["nt"]), float(g["dt"]), (20., 20.), nbt=30, ct=0.01,
                        src=_src(g), jsnap=3, rick=g["rick"])
    assert np.array_equal(tr, g["traces"])
    assert np.array_equal(sn, g["snaps"])


def test_afd2d_own_wavelet_within_tolerance(golden, oracle):
    g = golden("afd2d_fwd")
    tr, sn = oracle.afd(g["vel"], int(g["nt"]), float(g["dt"]), (20., 20.), nbt=30, ct=0.01,
                        src=_src(g), jsnap=3)
    assert rel_l2(tr, g["traces"]) < 1e-5
    assert rel_l2(sn, g["snaps"]) < 1e-5


def test_afd2d_tri_bit_exact(golden, oracle):
    g = golden("afd2d_tri")
    _, sn = oracle.afd(g["vel"], g["dat"].shape[0], 0.001, (20., 20.), nbt=30, ct=0.01, tri=True,
                       dat=g["dat"], jsnap=4)
    assert np.array_equal(sn, g["snaps"])
    # the reference's afd2d returns the input traces in TRI mode
    assert np.array_equal(g["echo"], g["dat"])


def test_afd3d_bit_exact_given_reference_wavelet(golden, oracle):
    g = golden("afd3d_fwd")
    tr, sn = oracle.afd(g["vel"], int(g["nt"]), float(g["dt"]), (20., 20., 20.), nbt=8, ct=0.02,
                        src=_src(g, True), jsnap=5, rick=g["rick"])
    assert np.array_equal(tr, g["traces"])
    assert np.array_equal(sn, g["snaps"])


def test_afd3d_tri_bit_exact(golden, oracle):
    g = golden("afd3d_tri")
    _, sn = oracle.afd(g["vel"], g["dat"].shape[0], 0.001, (20., 20., 20.), nbt=8, ct=0.02,
                       tri=True, dat=g["dat"], jsnap=4)
    assert np.array_equal(sn, g["snaps"])


def test_config1_gather_at_depth5(golden, oracle):
    g = golden("c1_gather_z5")
    vel = np.full((201, 201), 1500, np.float32)
    vel[60:] = 2200
    vel[130:] = 3000
    src = dict(sx=[100], sz=[5], f=[20], t=[0.05], A=[1])
    tr, _ = oracle.afd(vel, 1501, 0.001, (10., 10.), nbt=30, ct=0.01, src=src, gz=5,
                       rick=g["rick"])
    assert np.array_equal(tr, g["gather"])
    tr2, _ = oracle.afd(vel, 1501, 0.001, (10., 10.), nbt=30, ct=0.01, src=src, gz=5)
    assert rel_l2(tr2, g["gather"]) < 1e-5


def _pf(g, oracle):
    nz, nx = g["vtrue"].shape
    geo = oracle.pfwi_geometry(nz, nx, float(g["par_dz"]), float(g["par_dx"]), 0, 0,
                               int(g["par_ns"]), float(g["par_ds"]), float(g["par_os"]),
                               int(g["par_nb"]))
    return geo, dict(nb=int(g["par_nb"]), coef=float(g["par_coef"]), dz=float(g["par_dz"]),
                     dx=float(g["par_dx"]), dt=float(g["par_dt"]), geo=geo, ns=int(g["par_ns"]))


def test_pfwi_forward_bit_exact(golden, oracle):
    g = golden("pfwi")
    _, kw = _pf(g, oracle)
    d = oracle.pfwi_forward(g["vtrue"], g["wav"], **kw)
    assert np.array_equal(d, g["data"])


def test_pfwi_gradient_av_bit_exact(golden, oracle):
    g = golden("pfwi")
    _, kw = _pf(g, oracle)
    raw, fcost = oracle.pfwi_gradient_ref(g["vstart"], g["wav"], g["data"], **kw)
    assert np.float32(fcost) == np.float32(g["fcost"])
    for rect in (1, 3):
        pp, _ = oracle.pfwi_postprocess(raw, rect=rect)
        assert np.array_equal(pp, g["grad_rect%d" % rect])


def test_exact_adjoint_matches_finite_differences(golden, oracle):
    g = golden("pfwi")
    _, kw = _pf(g, oracle)
    vs = g["vstart"].astype(np.float64)
    W = oracle.residual_weights(len(g["wav"]), kw["geo"]["nr"])
    ge, J = oracle.pfwi_gradient_exact(vs, g["wav"], g["data"], weight=W, **kw)
    rng = np.random.default_rng(3)
    cells = [(0, 0), (29, 49)] + [tuple(c) for c in zip(rng.integers(0, 30, 6), rng.integers(0, 50, 6))]
    for iz, ix in cells:
        h = 1e-4
        vp = vs.copy(); vp[iz, ix] += h
        vm = vs.copy(); vm[iz, ix] -= h
        fd = (oracle.pfwi_misfit(vp, g["wav"], g["data"], weight=W, **kw) -
              oracle.pfwi_misfit(vm, g["wav"], g["data"], weight=W, **kw)) / (2 * h)
        assert abs(fd - ge[iz, ix]) <= 1e-5 * abs(ge).max() + 1e-4 * abs(fd)


# ---- fixtures kept as digests of the reference's outputs (larger runs) ----

def _models():
    import os
    import sys
    from conftest import ROOT
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import models
    return models


def test_afd3d_big_bit_exact_vs_reference_digests(golden, oracle):
    """80 x 72 x 64 interior with nbt 10 (the size whose untapered warp
    patches the GPU tests exercise): forward traces, snapshots and the
    time reversal of one x-band group reproduce the reference's digests."""
    M = _models()
    g = golden("afd3d_big")
    vel = M.big3d_velocity()
    assert M.digest(vel) == str(g["vel_digest"])
    B = M.BIG3D
    src = dict(sx=B["sx"], sy=B["sy"], sz=B["sz"], f=B["f"], t=B["t"], A=B["A"])
    d, w = oracle.afd(vel, B["nt"], B["dt"], (20., 20., 20.), nbt=B["nbt"], ct=B["ct"], src=src,
                      jsnap=B["jsnap"], rick=g["rick"])
    assert M.digest(d) == str(g["traces_digest"]) and M.digest(w) == str(g["snaps_digest"])
    dg = np.zeros_like(d)
    b0, b1 = M.BIG3D_BAND
    dg[:, b0:b1, :] = d[:, b0:b1, :]
    _, wt = oracle.afd(vel, B["nt"], B["dt"], (20., 20., 20.), nbt=B["nbt"], ct=B["ct"], tri=True,
                       dat=dg, jsnap=M.BIG3D_TRI_JSNAP)
    assert M.digest(wt) == str(g["tri_snaps_digest"])


@pytest.mark.parametrize("name", ["c4geo", "deep"])
def test_pfwi_scale_bit_exact_vs_reference_digests(golden, oracle, name):
    """pfwi forward data and gradient_av (rect 1 and 3, with the first-call
    scale) at the 300 x 600 benchmark geometry and on the 460 x 200 model
    reproduce the reference's digests; the misfit equals the reference's."""
    M = _models()
    g = golden("pfwi_" + name)
    vt, vs, par, wav = M.pfwi_scale_case(name)
    assert M.digest(vt) == str(g["vtrue_digest"]) and M.digest(vs) == str(g["vstart_digest"])
    geo = oracle.pfwi_geometry(par["nz"], par["nx"], par["dz"], par["dx"], 0, 0, par["ns"],
                               par["ds"], par["os"], par["nb"])
    kw = dict(nb=par["nb"], coef=par["coef"], dz=par["dz"], dx=par["dx"], dt=par["dt"], geo=geo,
              ns=par["ns"])
    d = oracle.pfwi_forward(vt, wav, **kw)
    assert M.digest(d) == str(g["data_digest"])
    gr, f = oracle.pfwi_gradient_ref(vs, wav, d, **kw)
    assert f == float(g["fcost"])
    p1, _ = oracle.pfwi_postprocess(gr, rect=1)
    p3, _ = oracle.pfwi_postprocess(gr, rect=3)
    assert M.digest(p1) == str(g["grad1_digest"]) and M.digest(p3) == str(g["grad3_digest"])
