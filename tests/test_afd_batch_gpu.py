"""pw_afd_batch (uneven 2-D shots in one lockstep time loop) against pw_afd
run shot by shot: the traces must be identical (same kernel arithmetic, any
tile shape).  GPU only."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _shots(seed=0):
    rng = np.random.default_rng(seed)
    shots = []
    for nz, nx, nt, dx in [(40, 50, 300, 10.0), (64, 33, 120, 12.0), (20, 90, 250, 8.0),
                           (31, 31, 80, 10.0), (70, 120, 200, 10.0)]:
        vel = (1500 + 1000 * rng.random((nz, nx))).astype(np.float32)
        ns = int(rng.integers(1, 3))
        shots.append(dict(vel=vel, nt=nt, dt=0.001, ax=[0, dx, nx], az=[0, dx, nz], ns=ns,
                          sx=list(rng.integers(3, nx - 3, ns)), sz=list(rng.integers(3, nz - 3, ns)),
                          f=[20.0] * ns, t=[0.02 + 0.01 * i for i in range(ns)], A=[1.0] * ns,
                          nbt=12, ct=0.02, gz=int(rng.integers(0, 3))))
    return shots


def _single(sh):
    import pywave_b200 as pw
    kw = {k: sh[k] for k in ("nt", "dt", "ax", "az", "ns", "sx", "sz", "f", "t", "A", "nbt", "ct",
                             "gz")}
    return pw.afd2d(sh["vel"], jsnap=0, **kw).reshape(sh["nt"], sh["ax"][2], order="F")


def test_batch_host_pointers_match_single_shots(cuda_lib):
    from pywave_b200.afd import afd2d_batch
    shots = _shots()
    got = afd2d_batch(shots)
    for k, sh in enumerate(shots):
        ref = _single(sh)
        assert np.abs(ref).max() > 0
        assert np.array_equal(got[k], ref), k


def test_batch_device_pointers_on_a_stream_match(cuda_lib):
    """Device pointers on a side stream: the tuned steps and the graph replay."""
    import torch
    from pywave_b200 import _lib as L
    shots = _shots(seed=3)
    n = len(shots)
    args = (L.AfdArgs * n)()
    keep, vp, sp, dp = [], [], [], []
    for k, sh in enumerate(shots):
        ox, dx, nx = sh["ax"]
        oz, dz, nz = sh["az"]
        a = args[k]
        a.dim, a.nz, a.nx, a.ny, a.nt, a.nbt, a.ct = 2, nz, nx, 1, sh["nt"], sh["nbt"], sh["ct"]
        a.dt, a.dz, a.dx, a.dy, a.ns, a.tri, a.jsnap, a.gz, a.flags = (
            sh["dt"], dz, dx, dx, sh["ns"], 0, 0, sh["gz"], 0)
        v = torch.tensor(np.asarray(sh["vel"]).flatten(order="F"), device="cuda")
        s = torch.tensor(np.concatenate([np.asarray(sh[key], np.float32)
                                         for key in ("sx", "sz", "f", "t", "A")]), device="cuda")
        d = torch.full((sh["nt"] * nx,), float("nan"), device="cuda")
        keep += [v, s, d]
        vp.append(v.data_ptr())
        sp.append(s.data_ptr())
        dp.append(d.data_ptr())
    side = torch.cuda.Stream()
    for call in range(2):
        with torch.cuda.stream(side):
            L.check(cuda_lib.pw_afd_batch(n, C.cast(args, C.c_void_p),
                                          C.cast((C.c_void_p * n)(*vp), C.c_void_p),
                                          C.cast((C.c_void_p * n)(*sp), C.c_void_p), None,
                                          C.cast((C.c_void_p * n)(*dp), C.c_void_p),
                                          side.cuda_stream))
        side.synchronize()
        for k, sh in enumerate(shots):
            got = keep[3 * k + 2].cpu().numpy().reshape(sh["nt"], sh["ax"][2], order="F")
            assert np.array_equal(got, _single(sh)), (call, k)


def test_batch_rejects_3d_and_snapshots(cuda_lib):
    from pywave_b200 import _lib as L
    from pywave_b200.afd import afd2d_batch
    sh = _shots()[0]
    with pytest.raises(L.PywaveError):
        afd2d_batch([dict(sh, nt=0)])
    args = (L.AfdArgs * 1)()
    args[0].dim, args[0].nz, args[0].nx, args[0].ny, args[0].nt = 3, 10, 10, 10, 10
    args[0].flags = L.PW_HOST_PTRS
    dummy = np.zeros(1000, np.float32)
    P = (C.c_void_p * 1)(dummy.ctypes.data)
    with pytest.raises(L.ShapeError, match="2-D"):
        L.check(cuda_lib.pw_afd_batch(1, C.cast(args, C.c_void_p), C.cast(P, C.c_void_p),
                                      C.cast(P, C.c_void_p), None, C.cast(P, C.c_void_p), None))
