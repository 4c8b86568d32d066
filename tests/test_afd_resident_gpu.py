"""The cluster-resident 2-D path (one launch for the whole time loop, fields in
distributed shared memory) against the step-per-launch path: traces,
snapshots and TRI images must be identical.  PW_AFD_RESIDENT=0 forces the
step-per-launch path.  GPU only."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _both(fn):
    """fn() on the resident path, then with it switched off; (out, launches) each."""
    from pywave_b200 import _lib as L
    old = os.environ.pop("PW_AFD_RESIDENT", None)
    try:
        res = fn()
        n_res = L.last_timing()[1]
        os.environ["PW_AFD_RESIDENT"] = "0"
        ref = fn()
        n_ref = L.last_timing()[1]
    finally:
        os.environ.pop("PW_AFD_RESIDENT", None)
        if old is not None:
            os.environ["PW_AFD_RESIDENT"] = old
    return res, n_res, ref, n_ref


@pytest.mark.parametrize("nz,nx,nbt,gz", [(201, 201, 30, 5), (41, 51, 30, 0), (3, 5, 5, 1),
                                         (1, 1, 5, 0), (130, 17, 12, 3), (64, 300, 20, 2)])
def test_forward_matches_step_path(cuda_lib, nz, nx, nbt, gz):
    import pywave_b200 as pw
    rng = np.random.default_rng(nz * 7 + nx)
    vel = (1600 + 1200 * rng.random((nz, nx))).astype(np.float32)
    ns = 2 if nz > 2 and nx > 2 else 1
    sx = [int(v) for v in rng.integers(0, nx, ns)]
    sz = [int(v) for v in rng.integers(0, nz, ns)]
    nt = 240
    kw = dict(nt=nt, dt=0.001, ax=[0, 10, nx], az=[0, 10, nz], ns=ns, sx=sx, sz=sz,
              f=[25.0] * ns, t=[0.02 + 0.01 * i for i in range(ns)], A=[1.0] * ns, nbt=nbt,
              ct=0.01, jsnap=7, gz=gz)
    (d1, w1), n1, (d0, w0), n0 = _both(lambda: pw.afd2d(vel, **kw))
    assert n1 == 1 and n0 == nt  # one resident launch vs one launch per step
    assert np.abs(d0).max() > 0
    assert np.array_equal(d1.view(np.uint32), d0.view(np.uint32))
    assert np.array_equal(w1.view(np.uint32), w0.view(np.uint32))


def test_tri_snapshots_match_step_path(golden, cuda_lib):
    import pywave_b200 as pw
    g = golden("afd2d_tri")
    kw = dict(nt=g["dat"].shape[0], dt=0.001, ax=[0, 20, 51], az=[0, 20, 41], jsnap=4,
              dat=g["dat"], tri=True, nbt=30, ct=0.01)
    (e1, w1), n1, (e0, w0), n0 = _both(lambda: pw.afd2d(g["vel"], **kw))
    assert n1 == 1 and n0 == kw["nt"]
    assert np.array_equal(w1, w0) and np.array_equal(w1, g["snaps"])


@pytest.mark.parametrize("ng", [1, 3, 4])
def test_tri_image_matches_step_path(oracle, cuda_lib, ng):
    import pywave_b200 as pw
    vel = np.full((60, 90), 2000, np.float32)
    vel[30:] = 2700
    src = dict(sx=[45], sz=[40], f=[15], t=[0.04], A=[1])
    d, _ = oracle.afd(vel, 300, 0.001, (15., 15.), nbt=20, ct=0.02, src=src)
    img1, n1, img0, n0 = _both(lambda: pw.tri_image(vel, d, dt=0.001, d=(15., 15.), ngroups=ng,
                                                    nbt=20, ct=0.02, jsnap=4))
    assert n1 == 1 and n0 == 300
    assert np.abs(img0).max() > 0
    assert np.array_equal(img1.view(np.uint32), img0.view(np.uint32))


def test_large_grid_takes_the_step_path(cuda_lib):
    """A grid beyond one cluster's shared memory runs one launch per step."""
    import pywave_b200 as pw
    from pywave_b200 import _lib as L
    vel = np.full((900, 900), 2000, np.float32)
    pw.afd2d(vel, nt=12, dt=0.001, ax=[0, 10, 900], az=[0, 10, 900], ns=1, sx=[450], sz=[450],
             f=[20.0], t=[0.0], A=[1.0], nbt=30, ct=0.01, jsnap=0)
    assert L.last_timing()[1] == 12
