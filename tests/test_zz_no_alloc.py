"""pw_afd_noalloc (scratch in a fixed device array) against pw_afd (cached
workspace) on the same device inputs: two consecutive calls must both give
pw_afd's traces and snapshots.  Both entry points run the same step kernel
in the same order, so the tolerance is zero (bit-exact).  A second test
checks, in a fresh process, that its calls take no device memory.  GPU
only."""
import ctypes
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ricker(nt, dt, f0, t0, A=1.0):
    t = np.arange(nt) * dt - t0
    x = (np.pi * f0 * t) ** 2
    return (A * (1 - 2 * x) * np.exp(-x)).astype(np.float32)


def _case(dim, n, nt, nb, ns, jsnap, seed):
    import torch
    from pywave_b200 import _lib as L
    rng = np.random.default_rng(seed)
    nz, nx = n[0], n[1]
    ny = n[2] if dim == 3 else 1
    a = L.AfdArgs()
    a.dim, a.nz, a.nx, a.ny, a.nt, a.nbt, a.ct = dim, nz, nx, ny, nt, nb, 0.01
    a.dt, a.dz, a.dx, a.dy = 0.001, 0.01, 0.01, 0.01
    a.ns, a.tri, a.jsnap, a.gz, a.flags = ns, 0, jsnap, 0, 0
    vel = (1.5 + rng.random((ny, nx, nz))).astype(np.float32)  # CFL <= 0.25
    if dim == 2:
        src = np.stack([rng.integers(5, nx - 5, ns), rng.integers(5, nz - 5, ns),
                        np.full(ns, 20.0), np.full(ns, 0.05), np.ones(ns)]).astype(np.float32)
    else:
        src = np.stack([rng.integers(5, nx - 5, ns), rng.integers(5, ny - 5, ns),
                        rng.integers(5, nz - 5, ns), np.full(ns, 20.0), np.full(ns, 0.05),
                        np.ones(ns)]).astype(np.float32)
    wav = np.stack([_ricker(nt, a.dt, 20.0, 0.05 + 0.01 * i, 1.0 + i) for i in range(ns)])
    d = "cuda"
    dev = dict(vel=torch.tensor(vel, device=d), src=torch.tensor(src, device=d),
               wav=torch.tensor(wav, device=d))
    ntsnap = len(range(0, nt, jsnap)) if jsnap else 0
    shapes = dict(dat=(ny, nx, nt), wfd=(max(ntsnap, 1), ny, nx, nz))
    return a, dev, shapes


def _run(fn, a, dev, shapes):
    import torch
    from pywave_b200 import _lib as L
    dat = torch.full(shapes["dat"], float("nan"), device="cuda")
    wfd = torch.full(shapes["wfd"], float("nan"), device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    L.check(fn(ctypes.byref(a), dev["vel"].data_ptr(), dev["src"].data_ptr(),
               dev["wav"].data_ptr(), dat.data_ptr(), wfd.data_ptr() if a.jsnap else None, s))
    torch.cuda.synchronize()
    return dat.cpu().numpy(), wfd.cpu().numpy()


@pytest.mark.parametrize("dim,n,nt,nb,ns,jsnap", [
    (2, (101, 121), 300, 20, 2, 50),
    (3, (40, 36, 44), 80, 10, 1, 20),
])
def test_noalloc_matches_pw_afd_twice(cuda_lib, dim, n, nt, nb, ns, jsnap):
    a, dev, shapes = _case(dim, n, nt, nb, ns, jsnap, seed=7 + dim)
    ref_dat, ref_wfd = _run(cuda_lib.pw_afd, a, dev, shapes)
    assert np.isfinite(ref_dat).all() and np.abs(ref_dat).max() > 0
    for call in range(2):
        dat, wfd = _run(cuda_lib.pw_afd_noalloc, a, dev, shapes)
        assert np.array_equal(dat, ref_dat), (dim, call)
        assert np.array_equal(wfd, ref_wfd), (dim, call)


def test_noalloc_rejects_oversize_and_host_pointers(cuda_lib):
    from pywave_b200 import _lib as L
    a, dev, shapes = _case(2, (64, 64), 20, 10, 1, 0, seed=1)
    big = L.AfdArgs.from_buffer_copy(a)
    big.nz, big.nx = 2000, 2000  # about 50 MB of wavefields
    with pytest.raises(L.ShapeError, match="scratch"):
        L.check(cuda_lib.pw_afd_noalloc(ctypes.byref(big), dev["vel"].data_ptr(),
                                        dev["src"].data_ptr(), dev["wav"].data_ptr(), None,
                                        None, None))
    host = L.AfdArgs.from_buffer_copy(a)
    host.flags = L.PW_HOST_PTRS
    with pytest.raises(L.ShapeError, match="device pointers"):
        L.check(cuda_lib.pw_afd_noalloc(ctypes.byref(host), dev["vel"].data_ptr(),
                                        dev["src"].data_ptr(), dev["wav"].data_ptr(), None,
                                        None, None))


def test_noalloc_takes_no_device_memory(cuda_lib):
    """In a fresh process: after one warm-up call per model size (the first
    loads the library's modules and the scratch array), further calls of
    both sizes leave the device's free memory unchanged; pw_afd's cached
    workspace is never created, so a caller whose memory pool or budget
    owns the device is not bypassed."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = textwrap.dedent("""
        import sys
        sys.path.insert(0, %r)
        sys.path.insert(0, %r)
        import torch
        from pywave_b200 import _lib as L
        import test_zz_no_alloc as T
        lib = L.lib()
        cases = [T._case(2, (101, 121), 200, 20, 2, 50, seed=3),
                 T._case(3, (40, 36, 44), 60, 10, 1, 20, seed=4)]
        outs = []
        for a, dev, shapes in cases:
            outs.append((torch.empty(shapes["dat"], device="cuda"),
                         torch.empty(shapes["wfd"], device="cuda")))
        s = torch.cuda.current_stream().cuda_stream

        def call(k):
            a, dev, _ = cases[k]
            dat, wfd = outs[k]
            L.check(lib.pw_afd_noalloc(T.ctypes.byref(a), dev["vel"].data_ptr(),
                                       dev["src"].data_ptr(), dev["wav"].data_ptr(),
                                       dat.data_ptr(), wfd.data_ptr(), s))

        call(0); call(1)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        for _ in range(2):
            call(0); call(1)
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info()[0]
        print("free bytes before/after:", free0, free1)
        assert free1 == free0, (free0, free1)
    """ % (root, os.path.join(root, "tests")))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    print(r.stdout, r.stderr)
    assert r.returncode == 0
