"""Parity of the CUDA path at the sizes and branches the benchmarks run.

The small goldens of test_afd_gpu.py / test_pfwi_gpu.py never reach some of
the code paths that carry the benchmarked workloads: the untapered fast
paths of the 3-D warp-tile step (a warp's 32-cell z patch free of taper),
several y chunks per launch, the 201^3 four-group TRI launch, the pfwi step
kernel with 128-float4 z segments and with more than one z tile, and the
batched 2-D forward on a shot of 1024 x 2048 cells.  These tests run those
paths against the reference (digests of its outputs, generated by
tests/golden/make_golden.py from the compiled reference) or against the
oracle restatement (pinned bit-exactly to the reference by
test_oracle_golden.py), and read the library's branch counters
(PW_AFD_VERBOSE) to show which paths ran.  GPU only; every call goes
through the C ABI.
"""
import os
import re
import sys
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from conftest import ROOT, rel_l2

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import models as M  # noqa: E402

pytestmark = pytest.mark.gpu


def _counts(err: str):
    m = re.findall(r"afd tile paths \(warp-planes\): (.*)", err)
    assert m, "no branch counts printed (PW_AFD_VERBOSE)"
    return [{k: int(v) for k, v in (kv.split("=") for kv in line.split())} for line in m]


def _plan_grid(err: str):
    m = re.findall(r"afd tile plan: .* grid=(\d+)x(\d+)", err)
    assert m, "no tile plan printed"
    return [(int(a), int(b)) for a, b in m]


# ------------------------------------------------------------ afd 3-D ----

# (ring filling as the plan prints it, PW_AFD_TMA, columns per lane, PW_AFD_SPLIT)
RINGS = [("cp.async", "0", "1", "0"), ("cp.async+split", "0", "1", "1"),
         ("cp.async+split", "0", "2", "0"), ("tma", "1", "1", "0"), ("tma", "1", "2", "0")]


@pytest.mark.parametrize("ring,env,nc,split", RINGS)
def test_afd3d_untapered_paths_bit_exact_vs_reference(golden, cuda_lib, monkeypatch, capfd, ring,
                                                      env, nc, split):
    """80 x 72 x 64 interior, nbt 10, 2 sources, nt 60: traces and snapshots
    identical to the reference's afd3d with either ring filling (per-lane
    cp.async or TMA tile loads) and one or two columns per lane, every
    taper path of the 3-D step (0: none,
    1: y only, 2: z / x only, 3: face by face) taken, and the launch split
    into several y chunks."""
    import pywave_b200 as pw
    g = golden("afd3d_big")
    vel = M.big3d_velocity()
    assert M.digest(vel) == str(g["vel_digest"])
    kw = {k: v for k, v in M.BIG3D.items()}
    monkeypatch.setenv("PW_AFD_VERBOSE", "1")
    monkeypatch.setenv("PW_AFD_TMA", env)
    monkeypatch.setenv("PW_AFD_NC", nc)
    monkeypatch.setenv("PW_AFD_SPLIT", split)
    d, w = pw.afd3d(vel, wavelet=g["rick"], **kw)
    err = capfd.readouterr().err
    c = _counts(err)[-1]
    print(err)
    assert re.search(rf"ring={re.escape(ring)}\s", err) and f"NC={nc}" in err
    assert all(c[f"fwd_path{k}"] > 0 for k in range(4))
    assert any(gy > 1 for _, gy in _plan_grid(err))
    assert np.array_equal(d[::3, ::4, ::4], g["traces_dec"])
    assert M.digest(d) == str(g["traces_digest"])
    assert tuple(w.shape) == tuple(g["snaps_shape"])
    assert np.array_equal(w[::4, ::4, ::4, -1], g["snaps_last_dec"])
    assert M.digest(w) == str(g["snaps_digest"])


@pytest.mark.parametrize("ring,env,nc,split", RINGS)
def test_afd3d_tri_untapered_paths_bit_exact_vs_reference(golden, cuda_lib, monkeypatch, capfd,
                                                          ring, env, nc, split):
    """Time reversal of one x-band group's traces on the same grid: every
    snapshot identical to the reference's with either ring filling, every
    taper path taken."""
    import pywave_b200 as pw
    g = golden("afd3d_big")
    vel = M.big3d_velocity()
    kw = {k: v for k, v in M.BIG3D.items()}
    d, _ = pw.afd3d(vel, wavelet=g["rick"], **kw)
    dg = np.zeros_like(d)
    b0, b1 = M.BIG3D_BAND
    dg[:, b0:b1, :] = d[:, b0:b1, :]
    capfd.readouterr()
    monkeypatch.setenv("PW_AFD_VERBOSE", "1")
    monkeypatch.setenv("PW_AFD_TMA", env)
    monkeypatch.setenv("PW_AFD_NC", nc)
    monkeypatch.setenv("PW_AFD_SPLIT", split)
    _, wt = pw.afd3d(vel, nt=kw["nt"], dt=0.001, ax=kw["ax"], ay=kw["ay"], az=kw["az"],
                     jsnap=M.BIG3D_TRI_JSNAP, dat=dg, tri=True, nbt=10, ct=0.02)
    err = capfd.readouterr().err
    c = _counts(err)[-1]
    print(err)
    assert re.search(rf"ring={re.escape(ring)}\s", err) and f"NC={nc}" in err
    assert all(c[f"tri_path{k}"] > 0 for k in range(4))
    assert tuple(wt.shape) == tuple(g["tri_shape"])
    assert np.array_equal(wt[::4, ::4, ::4, 0], g["tri_last_dec"])
    assert M.digest(wt) == str(g["tri_snaps_digest"])


def _oracle_group_runs(oracle, vel, d, groups, ng, nt, precision):
    """The demos' image from ng separate time-reversal runs of the oracle
    (threads: the oracle's C code runs without the GIL), keeping only the
    running product over groups."""
    ny, nx = groups.shape

    def run(gi):
        mask = (groups == gi).T  # [nx, ny]
        dg = (d * mask[None, :, :]).astype(np.float32)
        return oracle.afd(vel, nt, 0.001, (10., 10., 10.), nbt=30, ct=0.01, tri=True, dat=dg,
                          jsnap=4, precision=precision)[1]

    prod = None
    with ThreadPoolExecutor(max_workers=min(ng, os.cpu_count() or 1)) as ex:
        for s in ex.map(run, range(ng)):
            prod = s * s if prod is None else prod * s * s
            del s
    img = np.sum(prod, axis=-1)
    return img / img.max()


def test_config2_grid_tri_image_vs_oracle(oracle, cuda_lib, monkeypatch, capfd):
    """The benchmark's TRI image launch at its own size: the 201^3 model of
    bench.c2_model (1500 -> 3000 m/s plus 5% perturbation), nbt 30, four
    groups in lockstep, jsnap 4, here over 32 steps.  Over so few steps the
    wavefields of the benchmark's x-band groups cannot overlap (their image
    is identically zero), so receivers are assigned to the four groups in an
    interleaved pattern: the same kernels, tile plan and group count, with
    every group injecting across the surface.  The fused image is within
    1e-5 (rel-L2) of the image built from four separate oracle runs (FP32),
    and its error against the FP64 oracle is stated."""
    import bench
    import pywave_b200 as pw
    from scipy.ndimage import gaussian_filter1d
    n, nt, ng = 201, 32, 4
    vel, _, _, _ = bench.c2_model(n, seed=0)
    rng = np.random.default_rng(3)
    d = gaussian_filter1d(rng.standard_normal((nt, n, n)), 2.0, axis=0).astype(np.float32)
    iy, ix = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    groups = ((ix % 2) + 2 * (iy % 2)).astype(np.int32)  # [ny, nx]
    monkeypatch.setenv("PW_AFD_VERBOSE", "1")
    img = pw.tri_image(vel, d, dt=0.001, d=(10., 10., 10.), ngroups=ng, groups=groups, nbt=30,
                       ct=0.01, jsnap=4)
    err = capfd.readouterr().err
    print(err)
    c = _counts(err)[-1]
    assert all(c[f"tri_path{k}"] > 0 for k in range(4))
    ref32 = _oracle_group_runs(oracle, vel, d, groups, ng, nt, "f32")
    e32 = rel_l2(img, ref32)
    # the upper ~10 rows are imaged by 32 steps: a non-trivial image
    assert np.count_nonzero(ref32) > 0.01 * ref32.size
    ref64 = _oracle_group_runs(oracle, vel, d, groups, ng, nt, "f64")
    e64, o64 = rel_l2(img, ref64), rel_l2(ref32, ref64)
    print(f"201^3 benchmark grid TRI image (nt {nt}): rel-L2 vs FP32 oracle {e32:.2e}; "
          f"vs FP64 oracle: GPU {e64:.2e}, FP32 oracle {o64:.2e}")
    assert e32 <= 1e-5
    assert e64 <= 1e-4


# ---------------------------------------------------------------- pfwi ----

def _pfwi_kw(par, oracle):
    geo = oracle.pfwi_geometry(par["nz"], par["nx"], par["dz"], par["dx"], 0, 0, par["ns"],
                               par["ds"], par["os"], par["nb"])
    return dict(nb=par["nb"], coef=par["coef"], dz=par["dz"], dx=par["dx"], dt=par["dt"],
                geo=geo, ns=par["ns"])


@pytest.mark.parametrize("name,zw,ztiles", [("c4geo", 128, 1), ("deep", 128, 2)])
def test_pfwi_forward_and_reference_gradient_at_scale(golden, oracle, cuda_lib, monkeypatch,
                                                      capfd, name, zw, ztiles):
    """Forward data and the per-shot gradient_av (then its post-processing,
    rect 1 and 3) identical to the reference's at the 300 x 600 benchmark
    geometry (420 x 720 padded) and on a 580 x 320 padded grid (two z tiles);
    the batched reference gradient within 1e-5 of the oracle's."""
    import pywave_b200 as pw
    from pywave_b200 import fwi
    g = golden("pfwi_" + name)
    vt, vs, par, wav = M.pfwi_scale_case(name)
    assert M.digest(vt) == str(g["vtrue_digest"]) and M.digest(vs) == str(g["vstart_digest"])
    monkeypatch.setenv("PW_PFWI_VERBOSE", "1")
    q = np.full(vt.shape, 1e4, np.float32)
    data = pw.pfwi(vt, q, wav, None, mode=1, par=dict(par, niter=1))[0]
    err = capfd.readouterr().err
    assert f"ZW={zw} ztiles={ztiles}" in err, err
    assert np.array_equal(data[::5, ::10, :], g["data_dec"])
    assert M.digest(data) == str(g["data_digest"])
    raw, _ = fwi.gradient(vs, wav, data, dict(par, niter=1), mode="reference", per_shot=True)
    p1, _ = fwi.postprocess(raw, rect=1)
    assert np.array_equal(p1[::5, ::5], g["grad1_dec"])
    assert M.digest(p1) == str(g["grad1_digest"])
    p3, _ = fwi.postprocess(raw, rect=3)
    assert M.digest(p3) == str(g["grad3_digest"])
    rb, _ = fwi.gradient(vs, wav, data, dict(par, niter=1), mode="reference")
    ro, _ = oracle.pfwi_gradient_ref(vs, wav, data, **_pfwi_kw(par, oracle))
    e = rel_l2(rb, ro)
    print(f"{name}: batched reference gradient rel-L2 vs oracle {e:.2e}")
    assert e < 1e-5


@pytest.mark.parametrize("name", ["c4geo", "deep"])
def test_pfwi_exact_gradient_at_scale_vs_fp64(oracle, cuda_lib, name):
    """The exact adjoint at the scale geometries against the FP64 oracle's
    exact adjoint: cosine >= 0.9999."""
    from pywave_b200 import fwi
    vt, vs, par, wav = M.pfwi_scale_case(name)
    kw = _pfwi_kw(par, oracle)
    data = oracle.pfwi_forward(vt, wav, **kw)
    W = oracle.residual_weights(par["nt"], kw["geo"]["nr"])
    ge, J = fwi.gradient(vs, wav, data, dict(par, niter=1), mode="exact")
    go, Jo = oracle.pfwi_gradient_exact(vs, wav, data, weight=W, **kw)
    cos = float(np.sum(ge * go) / np.linalg.norm(ge) / np.linalg.norm(go))
    print(f"{name}: exact gradient cosine vs FP64 {cos:.8f}, rel-L2 {rel_l2(ge, go):.2e}, "
          f"misfit rel diff {abs(J - Jo) / abs(Jo):.2e}")
    assert cos >= 0.9999
    # the residual is a small difference of two FP32 records here, so the
    # FP32 misfit sits further from the FP64 one than on the small golden
    assert abs(J - Jo) <= 1e-3 * abs(Jo)


def test_exact_gradient_finite_differences_gpu(cuda_lib):
    """The GPU's own exact gradient against central differences of the GPU's
    own FP64 misfit on 20 seeded cells of a 120 x 240 window of the 300 x 600
    benchmark models (true model with a +10% anomaly 30 cells deep; nb 30,
    4 shots, nt 700): cosine over the 20 cells >= 0.9999 and each cell within
    1% (relative to the largest of them)."""
    import bench
    from pywave_b200 import fwi
    vt, vs = bench.fwi2d_models(7)
    vt = M.shallow_anomaly(np.ascontiguousarray(vt[:120, 180:420]), 30, 120, 12, 0.1)
    vs = np.ascontiguousarray(vs[:120, 180:420])
    nz, nx = vt.shape
    par = dict(nz=nz, nx=nx, dz=0.01, dx=0.01, oz=0.0, ox=0.0, nt=700, dt=0.001, ot=0.0, ns=4,
               ds=nx * 0.01 / 4, os=nx * 0.01 / 8, nb=30, coef=0.005, f0=10.0, acqui_type=1,
               interval=1, niter=1)
    wav = bench.fwi2d_wavelet(700)
    from pywave_b200 import _lib as L  # noqa: F401
    import pywave_b200 as pw
    q = np.full(vt.shape, 1e4, np.float32)
    dobs = pw.pfwi(vt, q, wav, None, mode=1, par=par)[0]
    g, J0 = fwi.gradient(vs, wav, dobs, par, mode="exact")
    rng = np.random.default_rng(20)
    # cells in the upper half, which the 0.7 s record reaches
    cells = [(int(rng.integers(8, 60)), int(rng.integers(8, nx - 8))) for _ in range(20)]
    fd, an = [], []
    for iz, ix in cells:
        v0 = float(vs[iz, ix])
        # a 1% step: the FP32 wavefields put rounding noise of about 1e-6 of J
        # into each misfit, which a smaller step would amplify; the step's own
        # truncation error is 1e-3 of the largest cell (FP64 oracle)
        h = np.float32(1e-2 * v0)
        vp, vm = vs.copy(), vs.copy()
        vp[iz, ix] = np.float32(v0 + h)
        vm[iz, ix] = np.float32(v0 - h)
        _, Jp = fwi.gradient(vp, wav, dobs, par, mode="exact")
        _, Jm = fwi.gradient(vm, wav, dobs, par, mode="exact")
        fd.append((Jp - Jm) / (float(vp[iz, ix]) - float(vm[iz, ix])))
        an.append(float(g[iz, ix]))
    fd, an = np.array(fd), np.array(an)
    cos = float(fd @ an / np.linalg.norm(fd) / np.linalg.norm(an))
    rel = np.abs(fd - an) / np.abs(an).max()
    print(f"GPU exact gradient vs central differences on 20 cells: cosine {cos:.8f}, "
          f"max |fd - g| / max|g| {rel.max():.2e}")
    assert cos >= 0.9999
    assert rel.max() <= 0.01


def test_exact_gradient_vs_reference_gradient_av(golden, cuda_lib):
    """Cosine between the GPU's exact adjoint gradient and the reference's own
    gradient_av (raw, rect 1, from the compiled reference) on the 60 x 120,
    4-shot, nt 800 case.  The reference's imaging is a consistent but not
    exact adjoint (snapshot-difference u_tt, first and last snapshots
    skipped, sponge not adjointed), so the two agree in direction only
    approximately; the value is reported."""
    import pywave_b200 as pw
    from pywave_b200 import fwi
    g = golden("pfwi_mid")
    vt, vs = M.mid_models()
    assert np.array_equal(vt, g["vtrue"]) and np.array_equal(vs, g["vstart"])
    par = dict(M.MID, niter=1)
    q = np.full(vt.shape, 1e4, np.float32)
    data = pw.pfwi(vt, q, g["wav"], None, mode=1, par=par)[0]
    assert M.digest(data) == str(g["data_digest"])
    ge, _ = fwi.gradient(vs, g["wav"], data, par, mode="exact")
    gr = g["grad_rect1"]
    cos = float(np.sum(ge * gr) / np.linalg.norm(ge) / np.linalg.norm(gr))
    nb = 8  # away from the source / receiver rows
    gi, ri = ge[nb:, :], gr[nb:, :]
    cos_in = float(np.sum(gi * ri) / np.linalg.norm(gi) / np.linalg.norm(ri))
    print(f"exact adjoint vs reference gradient_av: cosine {cos:.5f} (whole model), "
          f"{cos_in:.5f} (below row {nb})")
    # they part mostly in the source / receiver rows, where the reference's
    # imaging is furthest from the exact adjoint
    assert cos >= 0.8
    assert cos_in >= 0.99


# ------------------------------------------------------------- batch ----

def test_batch_with_large_shot_vs_oracle(oracle, cuda_lib):
    """pw_afd_batch on four of the batch benchmark's seeded shots (its
    generator, seed 5), the largest of them (1023 x 1994 interior, 1083 x
    2054 expanded) included, at reduced nt (200..290, past every source
    onset): every gather identical to the oracle's restatement of afd2d
    (the reference's own afd2dc corrupts its heap on a shot that large)."""
    import bench
    from pywave_b200.afd import afd2d_batch
    shots = bench.batch2d_shots(5)
    big = max(range(len(shots)), key=lambda k: shots[k]["az"][2] * shots[k]["ax"][2])
    pick = [big] + [k for k in range(len(shots)) if k != big][:3]
    sub = []
    for j, k in enumerate(pick):
        sh = dict(shots[k])
        sh["nt"] = 200 + 30 * j
        sub.append(sh)
    assert sub[0]["az"][2] >= 1000 and sub[0]["ax"][2] >= 1900
    got = afd2d_batch(sub)

    def ref(sh):
        src = dict(sx=sh["sx"], sz=sh["sz"], f=sh["f"], t=sh["t"], A=sh["A"])
        return oracle.afd(sh["vel"], sh["nt"], sh["dt"], (sh["az"][1], sh["ax"][1]), nbt=sh["nbt"],
                          ct=sh["ct"], src=src, gz=sh["gz"])[0]

    with ThreadPoolExecutor(max_workers=4) as ex:
        refs = list(ex.map(ref, sub))
    for k, (gk, rk) in enumerate(zip(got, refs)):
        assert np.abs(rk).max() > 0, k
        assert np.array_equal(gk, rk), k


# ------------------------------------------------------------ L-BFGS ----

def test_fwic_20_iterations_vs_reference(golden, cuda_lib):
    """20 iterations of fwic (pfwi mode 2: gradient_av, smoothing rect 3,
    L-BFGS with the reference's Wolfe line search) from the 60 x 120 start
    model, 4 shots, nt 800, against the reference's own 20 models.  The GPU
    takes every inner product in FP64 (deterministically), the reference in
    float, so the trajectories may part slowly; the per-iteration model
    difference and both misfit sequences are reported."""
    import pywave_b200 as pw
    from pywave_b200 import fwi
    g = golden("pfwi_mid")
    vt, vs = M.mid_models()
    par = dict(M.MID)
    q = np.full(vt.shape, 1e4, np.float32)
    data = pw.pfwi(vt, q, g["wav"], None, mode=1, par=dict(par, niter=1))[0]
    assert M.digest(data) == str(g["data_digest"])
    vinv = pw.pfwi(vs, q, g["wav"], None, data=data, mode=2, par=par)[1]
    again = pw.pfwi(vs, q, g["wav"], None, data=data, mode=2, par=par)[1]
    assert np.array_equal(vinv, again)  # deterministic
    ref = g["vinv"]
    assert vinv.shape == ref.shape
    # iterations completed (an early stop leaves the later models zero)
    n_ref = sum(1 for it in range(ref.shape[2]) if np.any(ref[:, :, it]))
    n_gpu = sum(1 for it in range(vinv.shape[2]) if np.any(vinv[:, :, it]))
    errs, jg, jr, mg, mr = [], [], [], [], []
    for it in range(min(n_ref, n_gpu)):
        errs.append(rel_l2(vinv[:, :, it], ref[:, :, it]))
        jg.append(fwi.gradient(vinv[:, :, it], g["wav"], data, dict(par, niter=1),
                               mode="reference")[1])
        jr.append(fwi.gradient(ref[:, :, it], g["wav"], data, dict(par, niter=1),
                               mode="reference")[1])
        mg.append(rel_l2(vinv[:, :, it], vt))
        mr.append(rel_l2(ref[:, :, it], vt))
    print(f"iterations completed: GPU {n_gpu}, reference {n_ref}; start model error "
          f"{rel_l2(vs, vt):.4e}")
    print("iteration: model rel-L2 vs reference | misfit GPU / reference | "
          "model error GPU / reference")
    for it in range(len(errs)):
        print(f"  {it + 1:2d}: {errs[it]:.2e} | {jg[it]:.6e} / {jr[it]:.6e} | "
              f"{mg[it]:.4e} / {mr[it]:.4e}")
    assert n_ref >= 5 and abs(n_gpu - n_ref) <= 1
    assert all(b < a for a, b in zip(jr, jr[1:])) and all(b < a for a, b in zip(jg, jg[1:]))
    assert max(errs[:3]) < 1e-3
    assert max(errs) < 2e-2
    assert abs(jg[-1] - jr[-1]) <= 0.05 * jr[-1]
