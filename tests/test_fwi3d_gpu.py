"""The 3-D FWI gradient (the 3-D extension of pfwi's scheme; the reference has
no 3-D FWI, so parity is pinned by the oracle restatement in
oracle/pw_oracle3d_body.h: its FP32 instance follows the GPU's operation
order, its FP64 instance is the exact adjoint that tests/test_oracle3d.py
checks against finite differences).  GPU only; every call goes through the
C ABI."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _case(seed=1, ns=2, nt=160):
    rng = np.random.default_rng(seed)
    nz, nx, ny = 22, 26, 20
    z = np.arange(nz, dtype=np.float32)[:, None, None]
    vt = (2.0 + 0.5 * z / nz + 0.2 * rng.random((nz, nx, ny))).astype(np.float32)
    vs = (2.0 + 0.5 * z / nz + np.zeros((nz, nx, ny))).astype(np.float32)
    t = np.arange(nt) * 0.001 - 0.05
    a = (np.pi * 20 * t) ** 2
    wav = (1e3 * (1 - 2 * a) * np.exp(-a)).astype(np.float32)
    src = [(3, 5 + 5 * i, 4 + 4 * i) for i in range(ns)]
    geom = dict(nb=8, coef=0.02, dz=0.01, dx=0.01, dy=0.01, nt=nt, dt=0.001, src=src, rz=1,
                rx=list(range(1, nx - 1, 3)), ry=list(range(1, ny - 1, 3)))
    return vt, vs, wav, geom


def test_forward_bit_exact_vs_fp32_oracle(oracle, cuda_lib):
    """Traces identical to the FP32 oracle, which runs the same float
    operations in the same order; their error against FP64 is stated."""
    from pywave_b200 import fwi3d
    vt, _, wav, geom = _case()
    d = fwi3d.forward3d(vt, wav, geom)
    d32 = oracle.pf3_forward(vt, wav, geom, "f32")
    d64 = oracle.pf3_forward(vt, wav, geom, "f64")
    assert np.abs(d32).max() > 0
    print(f"3-D forward: rel-L2 vs FP64 oracle {rel_l2(d, d64):.2e}")
    assert np.array_equal(d.view(np.uint32), d32.view(np.uint32))


@pytest.mark.parametrize("ckpt_k", [0, 1, 13, 160])
def test_exact_gradient_vs_fp64_oracle(oracle, cuda_lib, ckpt_k):
    """Exact adjoint (checkpoint interval k; 0 = planned) against the FP64
    oracle: cosine >= 0.9999, and identical gradients for every k."""
    from pywave_b200 import fwi3d
    vt, vs, wav, geom = _case()
    dobs = oracle.pf3_forward(vt, wav, geom, "f32")
    g, J = fwi3d.gradient3d(vs, wav, dobs, geom, ckpt_k=ckpt_k)
    go, Jo = oracle.pf3_gradient_exact(vs, wav, dobs, geom)
    cos = float(np.sum(g * go) / np.linalg.norm(g) / np.linalg.norm(go))
    print(f"3-D exact gradient k={ckpt_k}: cosine vs FP64 {cos:.8f}, rel-L2 {rel_l2(g, go):.2e}, "
          f"misfit rel diff {abs(J - Jo) / Jo:.2e}")
    assert cos >= 0.9999
    assert abs(J - Jo) <= 1e-4 * abs(Jo)
    g1, _ = fwi3d.gradient3d(vs, wav, dobs, geom, ckpt_k=1)
    assert np.array_equal(g, g1)


def test_exact_gradient_independent_of_budget_and_batch(oracle, cuda_lib):
    """Four shots: budgets that force smaller intervals and two-shot batches
    give the same gradient bit for bit."""
    from pywave_b200 import _lib as L
    from pywave_b200 import fwi3d
    vt, vs, wav, geom = _case(seed=3, ns=4)
    dobs = oracle.pf3_forward(vt, wav, geom, "f32")
    ref, Jr = fwi3d.gradient3d(vs, wav, dobs, geom)
    k0, nsb0, b0, rc0 = L.last_fwi_plan()
    assert nsb0 == 4 and rc0 == 1.0
    for budget in (b0 // 2, b0 // 4):
        g, J = fwi3d.gradient3d(vs, wav, dobs, geom, hbm_budget=budget)
        k, nsb, nbytes, rc = L.last_fwi_plan()
        print(f"budget {budget}: k {k}, shots per batch {nsb}, held {nbytes}, recompute {rc:.3f}")
        assert (k, nsb) != (k0, nsb0)
        assert np.array_equal(g, ref) and abs(J - Jr) <= 1e-12 * abs(Jr)


def test_gradient_finite_differences_gpu(oracle, cuda_lib):
    """The GPU's exact gradient against central differences of the GPU's own
    FP64 misfit (a 1% step, see the 2-D check) on 8 seeded cells."""
    from pywave_b200 import fwi3d
    vt, vs, wav, geom = _case(seed=5)
    dobs = oracle.pf3_forward(vt, wav, geom, "f32")
    g, _ = fwi3d.gradient3d(vs, wav, dobs, geom)
    rng = np.random.default_rng(8)
    nz, nx, ny = vs.shape
    fd, an = [], []
    for _ in range(8):
        c = (int(rng.integers(2, 12)), int(rng.integers(3, nx - 3)), int(rng.integers(3, ny - 3)))
        h = np.float32(1e-2 * vs[c])
        vp, vm = vs.copy(), vs.copy()
        vp[c] = vs[c] + h
        vm[c] = vs[c] - h
        _, Jp = fwi3d.gradient3d(vp, wav, dobs, geom)
        _, Jm = fwi3d.gradient3d(vm, wav, dobs, geom)
        fd.append((Jp - Jm) / (float(vp[c]) - float(vm[c])))
        an.append(float(g[c]))
    fd, an = np.array(fd), np.array(an)
    cos = float(fd @ an / np.linalg.norm(fd) / np.linalg.norm(an))
    rel = np.abs(fd - an) / np.abs(an).max()
    print(f"3-D GPU gradient vs central differences: cosine {cos:.8f}, max rel {rel.max():.2e}")
    assert cos >= 0.9999 and rel.max() <= 0.01


def test_autograd_function_3d(oracle, cuda_lib):
    import torch
    from pywave_b200 import fwi3d
    vt, vs, wav, geom = _case(seed=7)
    dobs = oracle.pf3_forward(vt, wav, geom, "f32")
    v = torch.tensor(vs, device="cuda", requires_grad=True)
    J = fwi3d.fwi3d_misfit(v, torch.tensor(wav, device="cuda"), torch.tensor(dobs, device="cuda"),
                           geom)
    J.backward()
    g, Jh = fwi3d.gradient3d(vs, wav, dobs, geom)
    assert J.item() == Jh
    assert np.array_equal(v.grad.cpu().numpy(), g)
