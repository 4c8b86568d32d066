"""Parity of the CUDA pfwi path (K4/K5/K6/K7) against the reference's golden
vectors and the FP64 oracle.  GPU only; every call goes through the C ABI."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _par(g, **over):
    par = {k[4:]: (g[k].item() if g[k].ndim == 0 else g[k]) for k in g if k.startswith("par_")}
    for k in ("nz", "nx", "nt", "ns", "nb", "acqui_type", "interval", "niter"):
        par[k] = int(par[k])
    par.update(over)
    return par


def _kw(g, oracle):
    nz, nx = g["vtrue"].shape
    geo = oracle.pfwi_geometry(nz, nx, float(g["par_dz"]), float(g["par_dx"]), 0, 0,
                               int(g["par_ns"]), float(g["par_ds"]), float(g["par_os"]),
                               int(g["par_nb"]))
    return dict(nb=int(g["par_nb"]), coef=float(g["par_coef"]), dz=float(g["par_dz"]),
                dx=float(g["par_dx"]), dt=float(g["par_dt"]), geo=geo, ns=int(g["par_ns"]))


def _misfit_f64(g, oracle):
    """0.5*sum(r^2), r = dobs-d formed in float32 and squared and summed in
    FP64, over the float32 synthetics of the starting model (the oracle's
    forward, bit-identical to the reference's)."""
    d = oracle.pfwi_forward(g["vstart"], g["wav"], **_kw(g, oracle))
    r = (np.asarray(g["data"], np.float32) - d).astype(np.float64)
    return 0.5 * float(np.sum(r * r))


def test_forward_modeling_bit_exact(golden, cuda_lib):
    import pywave_b200 as pw
    g = golden("pfwi")
    q = np.full(g["vtrue"].shape, 1e4, np.float32)
    d = pw.pfwi(g["vtrue"], q, g["wav"], None, mode=1, par=_par(g))[0]
    assert d.shape == g["data"].shape
    assert np.array_equal(d, g["data"])


@pytest.mark.parametrize("dz,dx,vmax", [(10.0, 10.0, 2500.0), (0.008, 0.012, 2.5),
                                         (0.03, 0.03, 4.0), (0.005, 0.025, 2.0)])
def test_forward_bit_exact_across_spacings(oracle, cuda_lib, dz, dx, vmax):
    """The Laplacian's divisions by dx^2 and dz^2 are correctly rounded for
    every numerator, the tiny and subnormal ones at the edge of the wavefield
    included (dx = 10 gives many ties on the subnormal grid): the data equal
    the oracle's float32 forward bit for bit."""
    import pywave_b200 as pw
    nz, nx, nt, ns, nb, dt = 40, 64, 500, 2, 12, 0.001
    rng = np.random.default_rng(int(dx * 1000))
    vel = (vmax * (0.6 + 0.4 * rng.random((nz, nx)))).astype(np.float32)
    t = np.arange(nt) * dt - 0.05
    a = (np.pi * 25.0 * t) ** 2
    wav = ((1 - 2 * a) * np.exp(-a)).astype(np.float32)
    ds = nx * dx / ns
    par = dict(nz=nz, nx=nx, dz=dz, dx=dx, oz=0.0, ox=0.0, nt=nt, dt=dt, ot=0.0, ns=ns, ds=ds,
               os=ds / 2, nb=nb, coef=0.005, f0=25.0, acqui_type=1, interval=1, niter=1)
    q = np.full(vel.shape, 1e4, np.float32)
    d = pw.pfwi(vel, q, wav, None, mode=1, par=par)[0]
    geo = oracle.pfwi_geometry(nz, nx, dz, dx, 0, 0, ns, ds, ds / 2, nb)
    ref = oracle.pfwi_forward(vel, wav, nb=nb, coef=0.005, dz=dz, dx=dx, dt=dt, geo=geo, ns=ns)
    assert np.abs(ref).max() > 0
    assert np.array_equal(d.view(np.uint32), ref.view(np.uint32))


def test_reference_gradient_bit_exact_per_shot(golden, oracle, cuda_lib):
    """gradient_av one shot at a time (the reference's summation order),
    then its smoothing and first-call scaling: identical to the reference.
    The misfit is summed in FP64 here; the reference sums it in float
    (wave_fwigradient.c:182), which is 1e-5 off the FP64 value."""
    from pywave_b200 import fwi
    g = golden("pfwi")
    par = _par(g)
    raw, J = fwi.gradient(g["vstart"], g["wav"], g["data"], par, mode="reference", per_shot=True)
    for rect in (1, 3):
        pp, _ = fwi.postprocess(raw, rect=rect)
        assert np.array_equal(pp, g["grad_rect%d" % rect]), rect
    J64 = _misfit_f64(g, oracle)
    assert abs(J - J64) <= 1e-12 * abs(J64)
    assert abs(J - float(g["fcost"])) <= 1e-4 * abs(J)


def test_reference_gradient_batched(golden, oracle, cuda_lib):
    """All shots in one launch sum per time step: same gradient to rounding."""
    from pywave_b200 import fwi
    g = golden("pfwi")
    raw_b, Jb = fwi.gradient(g["vstart"], g["wav"], g["data"], _par(g), mode="reference")
    raw_o, _ = oracle.pfwi_gradient_ref(g["vstart"], g["wav"], g["data"], **_kw(g, oracle))
    J64 = _misfit_f64(g, oracle)
    assert rel_l2(raw_b, raw_o) < 1e-5
    assert abs(Jb - J64) <= 1e-12 * abs(J64)


@pytest.mark.parametrize("k", [0, 1, 7, 400])
def test_exact_gradient_vs_fp64_oracle(golden, oracle, cuda_lib, k):
    """Exact adjoint (checkpoint interval k; 0 = planner) against the FP64
    oracle's exact adjoint, which is itself checked against finite
    differences on the CPU."""
    from pywave_b200 import fwi
    g = golden("pfwi")
    kw = _kw(g, oracle)
    W = oracle.residual_weights(len(g["wav"]), kw["geo"]["nr"])
    ge, J = fwi.gradient(g["vstart"], g["wav"], g["data"], _par(g), mode="exact", ckpt_k=k)
    go, Jo = oracle.pfwi_gradient_exact(g["vstart"], g["wav"], g["data"], weight=W, **kw)
    cos = float(np.sum(ge * go) / np.linalg.norm(ge) / np.linalg.norm(go))
    print(f"exact gradient k={k}: cosine vs FP64 {cos:.8f}, rel-L2 {rel_l2(ge, go):.2e}")
    assert cos >= 0.9999
    assert rel_l2(ge, go) < 1e-3
    assert abs(J - Jo) <= 1e-5 * abs(Jo)


def test_exact_gradient_independent_of_checkpoint_interval(golden, cuda_lib):
    from pywave_b200 import fwi
    g = golden("pfwi")
    ref, _ = fwi.gradient(g["vstart"], g["wav"], g["data"], _par(g), mode="exact", ckpt_k=1)
    for k in (3, 50, 400):
        gk, _ = fwi.gradient(g["vstart"], g["wav"], g["data"], _par(g), mode="exact", ckpt_k=k)
        assert np.array_equal(gk, ref), k


def test_exact_gradient_independent_of_hbm_budget(golden, cuda_lib):
    """The planner fits the checkpoints into the budget (a tighter budget: a
    smaller interval and more recompute, or fewer shots per batch) and the
    gradient stays bit-identical."""
    from pywave_b200 import _lib as L
    from pywave_b200 import fwi
    g = golden("pfwi")
    ref, Jr = fwi.gradient(g["vstart"], g["wav"], g["data"], _par(g), mode="exact", ckpt_k=1)
    plans = []
    for budget in (0, 40 << 20, 12 << 20, 6 << 20, 3 << 20):
        gb, Jb = fwi.gradient(g["vstart"], g["wav"], g["data"], _par(g), mode="exact",
                              hbm_budget=budget)
        k, nsb, nbytes, rc = L.last_fwi_plan()
        plans.append((budget, k, nsb, nbytes, rc))
        print(f"budget {budget >> 20} MiB: k {k}, shots per batch {nsb}, held {nbytes / 2**20:.1f} "
              f"MiB, recompute factor {rc:.3f}")
        assert np.array_equal(gb, ref), budget
        # the FP64 misfit's partial sums follow the batching
        assert abs(Jb - Jr) <= 1e-12 * abs(Jr)
    assert plans[0][1] == 400 and plans[0][4] == 1.0  # the default budget keeps every term
    assert plans[-1][1] < plans[1][1] and plans[-1][4] > 1.0
    for budget, k, nsb, nbytes, rc in plans[1:]:
        # the checkpoints and segment buffer fit; the rest is data and traces
        assert rc >= 1.0 and (nbytes < budget + (4 << 20))


def test_autograd_function(golden, cuda_lib):
    import torch
    from pywave_b200 import fwi
    g = golden("pfwi")
    par = _par(g)
    v = torch.tensor(g["vstart"], device="cuda", requires_grad=True)
    wav = torch.tensor(g["wav"], device="cuda")
    dobs = torch.tensor(np.asarray(g["data"]).transpose(2, 1, 0).copy(), device="cuda")  # [ns][nr][nt]
    J = fwi.fwi_misfit(v, wav, dobs, par)
    J.backward()
    ge, Je = fwi.gradient(g["vstart"], g["wav"], g["data"], par, mode="exact")
    assert abs(J.item() - Je) <= 1e-12 * abs(Je) + 1e-30
    assert np.array_equal(v.grad.cpu().numpy(), ge)


def test_fwic_runs_reference_lbfgs(golden, cuda_lib):
    """Two L-BFGS iterations from the golden start model: the models follow
    the reference's within the FP32/FP64 inner-product difference."""
    import pywave_b200 as pw
    g = golden("pfwi")
    par = _par(g, niter=2)
    q = np.full(g["vstart"].shape, 1e4, np.float32)
    _, vinv, _, _, _ = pw.pfwi(g["vstart"], q, g["wav"], None, data=g["data"], mode=2, par=par)
    ref = g["vinv"]
    assert vinv.shape == ref.shape
    for it in range(ref.shape[2]):
        if np.any(ref[:, :, it]):
            assert rel_l2(vinv[:, :, it], ref[:, :, it]) < 1e-3


def test_pfwi_errors(cuda_lib):
    import pywave_b200 as pw
    vel = np.full((20, 30), 2.0, np.float32)
    q = np.ones_like(vel)
    par = dict(nz=20, nx=30, dz=0.01, dx=0.01, oz=0, ox=0, nt=50, dt=0.01, ot=0, ns=1, ds=0.1,
               os=0.1, nb=10, coef=0.005, f0=10, acqui_type=1, interval=1, niter=1)
    with pytest.raises(ValueError):  # 2.0 * 0.01 / 0.01 > 0.555
        pw.pfwi(vel, q, np.zeros(50, np.float32), None, mode=1, par=par)
    with pytest.raises(ValueError):  # passive FWI (pfwic): the same stability check
        pw.pfwi(vel, q, np.zeros(50, np.float32), np.zeros((20, 30, 50, 1), np.float32),
                data=np.zeros((50, 30, 1), np.float32), mode=4,
                par=dict(par, inv=True, onlysrc=False))
