"""Generates the golden vectors under tests/golden/ by running the REFERENCE
itself (chenyk1990/pywave compiled from its own sources into oracle/_ref by
`make -C oracle ref`, with zero-initialised malloc).  Needs the reference
sources (read in place) and is run by hand in the build container:

    make -C oracle ref && python tests/golden/make_golden.py

The fixtures are small .npz files; the tests compare both the oracle
restatement (CPU) and the CUDA path (GPU) against them.
"""
from __future__ import annotations

import ctypes as C
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_PY = "/root/reference/pywave"
REF_BUILD = os.path.join(ROOT, "oracle", "_ref")
sys.path.insert(0, REF_BUILD)


def load(name):
    spec = importlib.util.spec_from_file_location("ref_" + name, os.path.join(REF_PY, name + ".py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def quiet(fn, *a, **k):
    """Run a reference call with its C-level stdout chatter discarded."""
    sys.stdout.flush()
    fd = os.dup(1)
    nul = os.open(os.devnull, os.O_WRONLY)
    os.dup2(nul, 1)
    try:
        return fn(*a, **k)
    finally:
        sys.stdout.flush()
        os.dup2(fd, 1)
        os.close(nul)
        os.close(fd)


def refdrv():
    L = C.CDLL(os.path.join(REF_BUILD, "libpwref.so"))
    f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
    L.refdrv_ricker.argtypes = [C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, f32p]
    L.refdrv_gradient.argtypes = [f32p, f32p, f32p, f32p, f32p, C.c_int, f32p, f32p]
    return L


def layered(nz, nx, vals, ifaces):
    v = np.full((nz, nx), vals[0], np.float32)
    for val, z in zip(vals[1:], ifaces):
        v[z:] = val
    return v


def main():
    a2, a3, pf = load("afd2d"), load("afd3d"), load("pfwi")
    R = refdrv()
    out = {}

    # ---- afd2d forward, 2 sources, snapshots ---------------------------
    vel = layered(41, 51, [2000, 2500, 3100], [15, 28])
    kw = dict(nt=300, dt=0.001, ax=[0, 20, 51], az=[0, 20, 41], ns=2, sx=[20, 31], sz=[10, 17],
              f=[10, 12], t=[0.1, 0.12], A=[1, 2], nbt=30, ct=0.01, jsnap=3, verb=0)
    d, w = quiet(a2.afd2d, vel, **kw)
    rick = []
    for fq, t0, A in zip(kw["f"], kw["t"], kw["A"]):
        r = np.zeros(kw["nt"], np.float32)
        R.refdrv_ricker(kw["nt"], kw["dt"], fq, t0, A, r)
        rick.append(r)
    np.savez_compressed(os.path.join(HERE, "afd2d_fwd.npz"), vel=vel, traces=d, snaps=w,
                        rick=np.stack(rick), **{k: np.asarray(v) for k, v in kw.items()})

    # ---- afd2d time reversal of one group's traces -----------------------
    dg = np.zeros_like(d)
    dg[:, 10:30] = d[:, 10:30]
    echo, wt = quiet(a2.afd2d, vel, nt=300, dt=0.001, ax=[0, 20, 51], az=[0, 20, 41], jsnap=4,
                     dat=dg, tri=True, verb=0, nbt=30, ct=0.01)
    np.savez_compressed(os.path.join(HERE, "afd2d_tri.npz"), vel=vel, dat=dg, echo=echo, snaps=wt)

    # ---- afd3d forward, small ------------------------------------------
    rng = np.random.default_rng(0)
    vel3 = (2000 + 300 * rng.random((24, 20, 22))).astype(np.float32)
    kw3 = dict(nt=120, dt=0.001, ax=[0, 20, 20], ay=[0, 20, 22], az=[0, 20, 24], ns=2, sx=[8, 12],
               sy=[9, 11], sz=[10, 6], f=[12, 15], t=[0.03, 0.05], A=[1, 1.5], nbt=8, ct=0.02,
               jsnap=5, verb=0)
    d3, w3 = quiet(a3.afd3d, vel3, **kw3)
    rick3 = []
    for fq, t0, A in zip(kw3["f"], kw3["t"], kw3["A"]):
        r = np.zeros(kw3["nt"], np.float32)
        R.refdrv_ricker(kw3["nt"], kw3["dt"], fq, t0, A, r)
        rick3.append(r)
    np.savez_compressed(os.path.join(HERE, "afd3d_fwd.npz"), vel=vel3, traces=d3, snaps=w3,
                        rick=np.stack(rick3), **{k: np.asarray(v) for k, v in kw3.items()})

    # ---- afd3d time reversal -------------------------------------------
    dg3 = np.zeros_like(d3)
    dg3[:, 5:15, :] = d3[:, 5:15, :]
    echo3, wt3 = quiet(a3.afd3d, vel3, nt=120, dt=0.001, ax=[0, 20, 20], ay=[0, 20, 22],
                       az=[0, 20, 24], jsnap=4, dat=dg3, tri=True, verb=0, nbt=8, ct=0.02)
    np.savez_compressed(os.path.join(HERE, "afd3d_tri.npz"), vel=vel3, dat=dg3, snaps=wt3)

    # ---- 201x201 three-layer gather, receivers at z=5 (wfd[5].T with jsnap=1) ------
    vc1 = layered(201, 201, [1500, 2200, 3000], [60, 130])
    _, wc1 = quiet(a2.afd2d, vc1, nt=1501, dt=0.001, ax=[0, 10, 201], az=[0, 10, 201], ns=1,
                   sx=[100], sz=[5], f=[20], t=[0.05], A=[1], nbt=30, ct=0.01, jsnap=1, verb=0)
    rc1 = np.zeros(1501, np.float32)
    R.refdrv_ricker(1501, 0.001, 20, 0.05, 1, rc1)
    np.savez_compressed(os.path.join(HERE, "c1_gather_z5.npz"),
                        gather=np.ascontiguousarray(wc1[5].T), rick=rc1[None, :])
    del wc1

    # ---- pfwi forward modelling + gradient_av ----------------------------
    nz, nx, nt = 30, 50, 400
    vt = layered(nz, nx, [2.0, 2.5, 3.0], [12, 22])
    q = np.full((nz, nx), 1e4, np.float32)
    tt = np.arange(nt) * 0.001
    arg = (np.pi * 10 * (tt - 0.1)) ** 2
    wav = ((1 - 2 * arg) * np.exp(-arg)).astype(np.float32)
    par = dict(nz=nz, nx=nx, dz=0.01, dx=0.01, oz=0, ox=0, nt=nt, dt=0.001, ot=0, ns=3, ds=0.15,
               os=0.05, nb=20, coef=0.005, f0=10, acqui_type=1, interval=1, niter=2)
    data = quiet(pf.pfwi, vt, q, wav, None, mode=1, par=dict(par))[0]
    vs = np.full((nz, nx), 2.4, np.float32)
    parr = np.array([nz, nx, 0.01, 0.01, 0, 0, nt, 0.001, 0, 3, 0.15, 0.05, 20, 0.005, 10, 1, 1],
                    np.float32)
    grads = {}
    for rect in (1, 3):
        g = np.zeros(nz * nx, np.float32)
        fc = np.zeros(1, np.float32)
        quiet(R.refdrv_gradient, parr, np.ascontiguousarray(vs.flatten(order="F")),
              np.ascontiguousarray(q.flatten(order="F")), wav.copy(),
              np.ascontiguousarray(data.flatten(order="F")), rect, g, fc)
        grads[rect] = (g.reshape(nz, nx, order="F"), float(fc[0]))
    vinv = quiet(pf.pfwi, vs, q, wav, None, data=data, mode=2, par=dict(par))[1]
    np.savez_compressed(os.path.join(HERE, "pfwi.npz"), vtrue=vt, vstart=vs, wav=wav, data=data,
                        grad_rect1=grads[1][0], fcost=grads[1][1], grad_rect3=grads[3][0],
                        vinv=vinv, **{"par_" + k: np.asarray(v) for k, v in par.items()})
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
