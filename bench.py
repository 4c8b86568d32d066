#!/usr/bin/env python
"""Benchmark of the B200 acoustic FD / TRI path.

Workload (default): 3-D time-reversal source imaging on a 201^3 grid at 10 m,
nt=1501, dt=1 ms, taper 30, velocity 1500->3000 m/s linear in depth plus a
seeded 5% Gaussian-smoothed perturbation, three seeded point sources (15-25 Hz
Ricker, onsets 0.1-0.5 s) recorded on the 201x201 surface; the traces are
split into 4 x-band receiver groups, back-propagated in lockstep and imaged
with the fused product-of-energies condition.  One step = one full TRI image
(4 groups x 1501 time steps on the 261^3 expanded grid).

Metric: Gpt-updates/s = 261^3 * 1501 * 4 / time.  `value` has inputs resident
in HBM; `e2e` runs the same C-ABI call with host buffers (traces and velocity
copied in, image copied out inside the timed region).

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]
Multi-GPU: one process per GPU (torchrun); each rank images its own seeded
event (weak scaling, no data-path collective).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n", type=int, default=201, help="interior grid size per axis")
    p.add_argument("--nt", type=int, default=1501)
    p.add_argument("--groups", type=int, default=4)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-fwi2d", action="store_true",
                   help="tri3d: skip the secondary 2-D FWI gradients/s field")
    p.add_argument("--workload", default="tri3d",
                   choices=["tri3d", "fwi2d", "batch2d", "c1", "fwi3d", "lstri", "pfwic", "aps3d",
                            "afd3d"],
                   help="tri3d: the 3-D TRI image (default); fwi2d: 2-D FWI gradients/s; "
                        "batch2d: uneven 2-D forward shots in one batch; c1: one 2-D shot; "
                        "fwi3d: 3-D FWI gradients/s; lstri: pfwi mode 4 source inversion; "
                        "pfwic: pfwi mode 4 passive FWI gradients/s; aps3d: pseudo-spectral 3-D; "
                        "afd3d: 3-D forward modelling of the tri3d model")
    p.add_argument("--lstri-niter", type=int, default=30, help="lstri: CG iterations per shot")
    p.add_argument("--lstri-nt", type=int, default=3001, help="lstri / pfwic: time samples")
    p.add_argument("--fwi3d-nt", type=int, default=2500, help="fwi3d: time samples")
    p.add_argument("--fwi3d-shots", type=int, default=16, help="fwi3d: shots per gradient")
    p.add_argument("--shots", type=int, default=32, help="fwi2d: shots per gradient")
    p.add_argument("--fwi-nt", type=int, default=2000, help="fwi2d: time samples")
    p.add_argument("--b2-nt", type=int, default=0,
                   help="batch2d: cut every shot's time samples to this many (0: as drawn)")
    return p.parse_args()


NBT, CT, H, DT = 30, 0.01, 10.0, 0.001


def c2_model(n, seed, nt=1501):
    """Velocity 1500 -> 3000 m/s linear in z plus a 5% seeded perturbation
    (N(0,1) field, Gaussian-smoothed sigma=5 points, scaled to +-5%)."""
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    z = np.arange(n, dtype=np.float64)[:, None, None]
    v0 = 1500.0 + 1500.0 * z / max(n - 1, 1) + np.zeros((n, n, n))
    p = gaussian_filter(rng.standard_normal((n, n, n)), sigma=5.0)
    p /= np.abs(p).max()
    vel = (v0 * (1.0 + 0.05 * p)).astype(np.float32)
    lo, hi = min(40, n // 4), max(n - 40, n - n // 4)
    pos = rng.integers(lo, hi, size=(3, 3))  # (sx, sy, sz) per source
    f = rng.uniform(15, 25, 3)
    t = rng.uniform(0.1, 0.5, 3)
    t = np.minimum(t, 0.5 * (nt - 1) * DT)  # short profiling runs keep the onsets inside nt
    return vel, pos, f, t


def gen_traces(vel, pos, f, t, nt, stream):
    """Surface traces [ny][nx][nt] of the three sources (afd3d forward) on the GPU."""
    import torch
    from pywave_b200 import _lib as L
    n = vel.shape[0]
    src = np.concatenate([pos[:, 0], pos[:, 1], pos[:, 2], f, t, np.ones(3)]).astype(np.float32)
    a = L.AfdArgs(dim=3, nz=n, nx=n, ny=n, nt=nt, nbt=NBT, ct=CT, dt=DT, dz=H, dx=H, dy=H, ns=3,
                  tri=0, jsnap=0, gz=0, flags=0)
    vel_d = torch.from_numpy(np.ascontiguousarray(vel.flatten(order="F"))).cuda()
    src_d = torch.from_numpy(src).cuda()
    dat = torch.empty(n * n * nt, device="cuda")
    L.check(L.lib().pw_afd(a, vel_d.data_ptr(), src_d.data_ptr(), None, dat.data_ptr(), None,
                           stream))
    return vel_d, dat


class Clocks:
    """nvidia-smi sampler (200 ms) around the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.dev = dev_index
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except (ValueError, IndexError):
                continue
            for i, nm in enumerate(names):
                if len(r) > 5 + i and r[5 + i].lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def pool_map(fn, arglist, timeout_s=600):
    """fn(*args) for each args in independent spawned processes, bounded in
    time: a worker that dies or stalls raises instead of hanging the run."""
    import multiprocessing as mp
    pool = mp.get_context("spawn").Pool(len(arglist))
    try:
        res = pool.starmap_async(fn, arglist).get(timeout=timeout_s)
        pool.close()
        return res
    finally:
        pool.terminate()
        pool.join()


REF_STEPS = (4, 12)  # two step counts per reference call: their difference excludes set-up


def ref_inputs(n, seed):
    """The benchmark's own velocity model (c2_model, the GPU arm's rank-0
    seed) and time-reversal traces of the first receiver group's x-band
    (seeded band-limited noise at the amplitude of the recorded traces) for
    the reference's time reversal; written to a temporary .npz that the
    spawned workers read."""
    from scipy.ndimage import gaussian_filter1d
    vel, _, _, _ = c2_model(n, seed)
    rng = np.random.default_rng(seed)
    nt_s = max(REF_STEPS)
    dat = np.zeros((nt_s, n, n), np.float32)
    band = n // 4
    dat[:, :band, :] = 1e-2 * gaussian_filter1d(rng.standard_normal((nt_s, band, n)), 2.0,
                                                axis=0)
    fd, path = tempfile.mkstemp(suffix=".npz")
    os.close(fd)
    np.savez(path, vel=vel, dat=dat)
    return path


def reference_sample(n, path, workers):
    """Per-step rate of the reference's own afd3dc (compiled from its sources
    into oracle/_ref; the oracle port when that is absent) time-reversing one
    receiver group on the full grid, in `workers` independent processes.
    Each process times a call of REF_STEPS[0] and one of REF_STEPS[1] steps;
    the difference of the two walls is the time of the extra steps alone
    (the reference's per-call set-up -- allocation, vel_expand and the
    unused pseudo-spectral Laplacian of wave_fdm.c:28-200 -- cancels).
    Returns (Gpt/s over all workers, kind, per-step seconds, set-up seconds)."""
    res = pool_map(_ref_worker, [(n, path)] * workers)
    d = max(r[1] - r[0] for r in res)  # slowest worker's extra-steps time
    if d <= 0:
        raise RuntimeError(f"reference timing: {REF_STEPS[1]} steps took no longer than "
                           f"{REF_STEPS[0]} ({res})")
    kind = res[0][2]
    extra = REF_STEPS[1] - REF_STEPS[0]
    pts = (n + 2 * NBT) ** 3 * extra * workers
    per_step = d / extra
    setup = max(r[0] for r in res) - REF_STEPS[0] * per_step
    return pts / d / 1e9, kind, per_step, setup


def _ref_worker(n, path):
    sys.path.insert(0, ROOT)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    with np.load(path) as z:
        vel, dat = z["vel"], z["dat"]
    vflat = vel.flatten(order="F")
    refdir = os.path.join(ROOT, "oracle", "_ref")
    walls = []
    try:
        sys.path.insert(0, refdir)
        import afdcfun  # the reference's own extension module
        kind = "reference"
        for nt_s in REF_STEPS:
            d = dat[-nt_s:].flatten(order="F")
            t0 = time.perf_counter()
            afdcfun.afd3dc(vflat, d, 1, nt_s, n, n, n, -1, 0, 4, 0, 1, NBT, CT, DT, 0.0, H, 0.0, H,
                           0.0, H)
            walls.append(time.perf_counter() - t0)
    except ImportError:
        from oracle import oracle as O
        kind = "port"
        O.lib()  # load (and if needed compile) the port before the timed calls
        for nt_s in REF_STEPS:
            t0 = time.perf_counter()
            O.afd(vel, nt_s, DT, (H, H, H), nbt=NBT, ct=CT, tri=True, dat=dat[-nt_s:], jsnap=4)
            walls.append(time.perf_counter() - t0)
    return walls[0], walls[1], kind


def max_over_ranks(x, world, device="cuda"):
    """Largest value of x over the ranks (identity on one rank)."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    tt = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def job_rate(units_per_rank_step, steps, world, ms_max):
    """Whole-job throughput: the units every rank processed over the
    slowest rank's time (weak scaling: each rank has the same work)."""
    return units_per_rank_step * steps * world / (ms_max / 1e3)


def run_reference(args, rank):
    if rank != 0:
        return
    n = args.n
    workers = max(1, min(os.cpu_count() or 1, 16))
    path = ref_inputs(n, 1234)
    vals, steps_s, setups = [], [], []
    try:
        for i in range(args.warmup + args.steps):
            v, kind, per_step, setup = reference_sample(n, path, workers)
            if i >= args.warmup:
                vals.append(v)
                steps_s.append(per_step)
                setups.append(setup)
    finally:
        os.unlink(path)
    value = statistics.median(vals)
    sample = (f"afd3dc time reversal of the first receiver group on the {n + 2 * NBT}^3 expanded "
              f"grid of the benchmark's velocity model, {workers} independent single-threaded "
              f"processes; per-step rate from calls of {REF_STEPS[0]} and {REF_STEPS[1]} steps "
              f"(difference of walls: {statistics.median(steps_s):.3f} s per step, the "
              f"{statistics.median(setups):.2f} s per-call set-up excluded)")
    line = {
        "impl": "reference", "metric": "Gpt-updates/s (3-D TRI, 4 lockstep groups)",
        "value": value, "unit": "Gpt/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (the benchmark's seeded velocity model; seeded traces)",
        "config": {"workload": f"3-D TRI image {n}^3 h=10m nt={args.nt} nbt={NBT} "
                               f"groups={args.groups} jsnap=4", "same_model": True,
                   "sample": f"{REF_STEPS[0]} and {REF_STEPS[1]} steps x {workers} procs"},
        "cpu_baseline": {"value": value, "unit": "Gpt/s", "cores": workers, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": "Gpt/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
# fwi2d: FWI gradients/s on a 300 x 600 model at 10 m (km units as pfwi uses)
# --------------------------------------------------------------------------
FWI_NZ, FWI_NX, FWI_H, FWI_DT, FWI_NB, FWI_COEF, FWI_F0 = 300, 600, 0.01, 0.001, 60, 0.005, 10.0
FWI_BUDGET = 40 << 30  # device bytes the exact gradient's checkpoints may hold


def fwi2d_models(seed):
    """True model: 8 seeded layers with velocities in [1.5, 4.5] km/s growing
    with depth, plus two Gaussian anomalies of +10% and -10%; start model:
    the true model Gaussian-smoothed with sigma = 15 points."""
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    z = np.arange(FWI_NZ)[:, None] + np.zeros((1, FWI_NX))
    x = np.zeros((FWI_NZ, 1)) + np.arange(FWI_NX)[None, :]
    ifaces = np.sort(rng.choice(np.arange(20, FWI_NZ - 10), 7, replace=False))
    vals = np.sort(rng.uniform(1.5, 4.5, 8))
    v = np.full((FWI_NZ, FWI_NX), vals[0])
    for val, zi in zip(vals[1:], ifaces):
        v[z >= zi] = val
    for sign in (1.0, -1.0):
        cz, cx = rng.uniform(0.3, 0.8) * FWI_NZ, rng.uniform(0.2, 0.8) * FWI_NX
        v *= 1.0 + 0.1 * sign * np.exp(-((z - cz) ** 2 + (x - cx) ** 2) / (2 * 20.0 ** 2))
    v = np.clip(v, 1.5, 4.5).astype(np.float32)
    return v, gaussian_filter(v.astype(np.float64), 15.0).astype(np.float32)


def fwi2d_par(ns, nt):
    ds = FWI_NX * FWI_H / ns
    return dict(nz=FWI_NZ, nx=FWI_NX, dz=FWI_H, dx=FWI_H, oz=0.0, ox=0.0, nt=nt, dt=FWI_DT,
                ot=0.0, ns=ns, ds=ds, os=ds / 2, nb=FWI_NB, coef=FWI_COEF, f0=FWI_F0,
                acqui_type=1, interval=1, niter=1)


def fwi2d_wavelet(nt):
    t = np.arange(nt) * FWI_DT - 1.2 / FWI_F0
    a = (np.pi * FWI_F0 * t) ** 2
    return ((1 - 2 * a) * np.exp(-a)).astype(np.float32)


def _fwi_ref_worker(nt_s, seed):
    """The reference's gradient_av (oracle/_ref/libpwref.so, built from its
    sources) for one shot over nt_s steps on the full grid; wall seconds."""
    sys.path.insert(0, ROOT)
    import ctypes
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    L = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libpwref.so"))
    f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
    L.refdrv_gradient.argtypes = [f32p, f32p, f32p, f32p, f32p, ctypes.c_int, f32p, f32p]
    vt, vs = fwi2d_models(seed)
    par = fwi2d_par(1, nt_s)
    # the driver's parameter layout (oracle/ref_driver.c fill_acpar)
    parr = np.array([par[k] for k in ("nz", "nx", "dz", "dx", "oz", "ox", "nt", "dt", "ot", "ns",
                                      "ds", "os", "nb", "coef", "f0", "acqui_type", "interval")],
                    np.float32)
    wav = fwi2d_wavelet(nt_s)
    dobs = np.zeros(nt_s * FWI_NX, np.float32)
    q = np.ones(FWI_NZ * FWI_NX, np.float32)
    g = np.zeros(FWI_NZ * FWI_NX, np.float32)
    fc = np.zeros(1, np.float32)
    t0 = time.perf_counter()
    L.refdrv_gradient(parr, np.ascontiguousarray(vs.flatten(order="F")), q, wav, dobs, 1, g, fc)
    return time.perf_counter() - t0


def _fwi_ref_worker_spawned(nt_s):
    return pool_map(_fwi_ref_worker, [(nt_s, 7)])[0]


class FwiBench:
    """Device state of the 2-D FWI gradient measurement: the seeded models,
    observed data modelled on the GPU from the true model, and a timer of
    pw_pfwi_gradient calls from the start model."""

    def __init__(self, ns, nt, seed, stream):
        import ctypes
        import torch
        from pywave_b200 import _lib as L
        from pywave_b200 import fwi
        self.L, self.lib, self.st = L, L.lib(), stream
        self.vt, self.vs = fwi2d_models(seed)
        self.par = fwi2d_par(ns, nt)
        self.wav = fwi2d_wavelet(nt)
        self.a = fwi.fwi_args(self.par, 0, FWI_BUDGET)
        dev = lambda arr: torch.from_numpy(np.ascontiguousarray(arr)).cuda()
        self.vt_d = dev(self.vt.flatten(order="F"))
        self.vs_d = dev(self.vs.flatten(order="F"))
        self.wav_d = dev(self.wav)
        self.dobs_d = torch.empty(ns * FWI_NX * nt, device="cuda")
        L.check(self.lib.pw_pfwi_forward(self.a, self.vt_d.data_ptr(), self.wav_d.data_ptr(),
                                         self.dobs_d.data_ptr(), stream))
        self.g_d = torch.empty(FWI_NZ * FWI_NX, device="cuda")
        self.J = ctypes.c_double(0.0)

    def grad(self, flags, mode):
        import ctypes
        self.a.flags = flags
        self.L.check(self.lib.pw_pfwi_gradient(self.a, mode, self.vs_d.data_ptr(),
                                               self.wav_d.data_ptr(), self.dobs_d.data_ptr(), None,
                                               self.g_d.data_ptr(), ctypes.byref(self.J), 0,
                                               self.st))
        return self.L.last_timing()

    def timed(self, flags, steps, warmup, world, mode):
        """(max-over-ranks ms of `steps` gradients, median loop ms, launches)."""
        import torch
        import torch.distributed as dist
        for _ in range(warmup):
            self.grad(flags, mode)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        loops, launches = [], 0
        e0.record()
        for _ in range(steps):
            ms, nst, tot = self.grad(flags, mode)
            loops.append(ms)
            launches += tot
        e1.record()
        torch.cuda.synchronize()
        return max_over_ranks(e0.elapsed_time(e1), world), statistics.median(loops), launches

    def plan(self):
        """The last exact gradient's checkpoint plan, as a JSON field."""
        k, nsb, nbytes, rc = self.L.last_fwi_plan()
        return {"budget_bytes": FWI_BUDGET, "interval_k": k, "shots_per_batch": nsb,
                "device_bytes": nbytes, "recompute_factor": rc}


def fwi2d_secondary(world, rank, stream, steps=2):
    """The 2-D FWI benchmark's headline pair, for the default line: exact
    gradients/s with the 32 shots batched, and with one shot at a time
    (PW_PER_SHOT, the plain per-shot path), same models and data."""
    from pywave_b200 import _lib as L
    ns, nt = 32, 2000
    fb = FwiBench(ns, nt, 11 + rank, stream)
    ms_b, _, lb = fb.timed(0, steps, 1, world, L.PW_GRAD_EXACT)
    plan = fb.plan()
    ms_p, _, lp = fb.timed(L.PW_PER_SHOT, 1, 1, world, L.PW_GRAD_EXACT)
    batched = job_rate(1, steps, world, ms_b)
    plain = job_rate(1, 1, world, ms_p)
    return {"workload": f"2-D FWI exact gradient {FWI_NZ}x{FWI_NX} h=10m nt={nt} shots={ns} "
                        f"nb={FWI_NB}", "batched": batched, "plain_per_shot": plain,
            "unit": "gradients/s", "batched_over_plain": batched / plain,
            "steps": {"batched": steps, "plain_per_shot": 1}, "gpu_launches": lb + lp,
            "checkpoint": plan}


def run_fwi2d(args, world, rank, local):
    ns, nt = args.shots, args.fwi_nt
    pad = (FWI_NZ + 2 * FWI_NB) * (FWI_NX + 2 * FWI_NB)
    if args.impl == "reference":
        if rank != 0:
            return
        nt_s, workers = 200, max(1, min(os.cpu_count() or 1, 16))
        rates = []
        for i in range(args.warmup + args.steps):
            walls = pool_map(_fwi_ref_worker, [(nt_s, 7)] * workers)
            if i >= args.warmup:
                rates.append(workers / max(walls) * nt_s / (ns * nt))
        value = statistics.median(rates)
        print(json.dumps({
            "impl": "reference", "metric": f"FWI gradients/s (2-D, {ns} shots)", "value": value,
            "unit": "gradients/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": f"2-D FWI gradient {FWI_NZ}x{FWI_NX} h=10m "
                                                         f"nt={nt} shots={ns} nb={FWI_NB}"},
            "cpu_baseline": {"value": value, "unit": "gradients/s", "cores": workers,
                             "kind": "reference",
                             "sample": f"gradient_av of 1 shot, {nt_s} of {nt} steps, {workers} "
                                       f"independent single-threaded processes, scaled to "
                                       f"{ns} shots x {nt} steps"},
            "e2e": {"value": value, "unit": "gradients/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}), flush=True)
        return
    import ctypes
    import torch
    import torch.distributed as dist
    from pywave_b200 import _lib as L
    from pywave_b200 import build as B
    from pywave_b200 import fwi
    B.build()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    st = torch.cuda.current_stream().cuda_stream
    lib = L.lib()
    fb = FwiBench(ns, nt, 11 + rank, st)
    vs, wav, par, dobs_d, J = fb.vs, fb.wav, fb.par, fb.dobs_d, fb.J

    def timed(flags, steps, mode=L.PW_GRAD_EXACT):
        return fb.timed(flags, steps, args.warmup, world, mode)

    clk = Clocks(local)
    clk.start()
    ms_b, loop_b, launches = timed(0, args.steps)
    clocks = clk.stop()
    plan = fb.plan()
    value = job_rate(1, args.steps, world, ms_b)
    nplain = max(1, args.steps // 2)
    ms_p, _, _ = timed(L.PW_PER_SHOT, nplain)
    plain = job_rate(1, nplain, world, ms_p)
    ms_r, _, _ = timed(0, args.steps, L.PW_GRAD_REFERENCE)
    ref_mode = job_rate(1, args.steps, world, ms_r)

    e2e = None
    if not args.no_e2e:
        vs_h = torch.from_numpy(np.ascontiguousarray(vs.flatten(order="F"))).pin_memory()
        dobs_h = dobs_d.cpu().pin_memory()
        g_h = torch.empty(FWI_NZ * FWI_NX).pin_memory()
        ah = fwi.fwi_args(par, L.PW_HOST_PTRS, FWI_BUDGET)
        wav_h = torch.from_numpy(wav).pin_memory()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            L.check(lib.pw_pfwi_gradient(ah, L.PW_GRAD_EXACT, vs_h.data_ptr(), wav_h.data_ptr(),
                                         dobs_h.data_ptr(), None, g_h.data_ptr(), ctypes.byref(J),
                                         0, st))
        torch.cuda.synchronize()
        ems = max_over_ranks((time.perf_counter() - t0) * 1e3, world)
        e2e = {"value": job_rate(1, args.steps, world, ems), "unit": "gradients/s",
               "h2d_bytes_per_step": int(vs.nbytes + wav.nbytes + dobs_h.numel() * 4),
               "d2h_bytes_per_step": int(g_h.numel() * 4 + 8)}

    peak, peak_kind = peaks()
    # algorithmic bytes per padded point-step-shot: forward 20 B (cur, prev,
    # V read; next, term write) + exact adjoint 28 B (cur, prev, V, term,
    # gradient read; next, gradient write) = 48 B; recomputed forward steps
    # (plan["recompute_factor"] - 1 of them per step) are not counted
    alg = 48.0 * pad * nt * ns
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as fh:
            per_step = json.load(fh).get(f"fwi2d_s{ns}_step")
        traffic = per_step * nt if per_step else None
    except (OSError, ValueError):
        pass
    achieved = alg / (loop_b / 1e3) / 1e9
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            wall = _fwi_ref_worker_spawned(200)
            cpu = {"value": 200 / (ns * nt) / wall, "unit": "gradients/s", "cores": 1,
                   "kind": "reference",
                   "sample": f"gradient_av of 1 shot, 200 of {nt} steps, 1 core ({wall:.1f} s), "
                             f"scaled to {ns} shots x {nt} steps"}
        except Exception as ex:  # noqa: BLE001
            cpu = {"value": None, "unit": "gradients/s", "cores": 1, "kind": "reference",
                   "sample": f"failed: {ex!r}"[:200]}
    if rank == 0:
        print(json.dumps({
            "metric": f"FWI gradients/s (2-D exact adjoint, {ns} shots batched)", "value": value,
            "unit": "gradients/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_b / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (FP64 misfit)",
            "data": "synthetic (seeded layered model, start = smoothed true model)",
            "config": {"workload": f"2-D FWI gradient {FWI_NZ}x{FWI_NX} h=10m nt={nt} dt=1ms "
                                   f"shots={ns} nb={FWI_NB} 10 Hz Ricker, exact adjoint with "
                                   f"checkpoints", "padded_cells": pad,
                       "l2": "inputs larger than L2 (observed data "
                             f"{dobs_d.numel() * 4 / 1e6:.0f} MB)"},
            "plain_per_shot": {"value": plain, "unit": "gradients/s"},
            "batched_over_plain": value / plain,
            "reference_mode_gradient": {"value": ref_mode, "unit": "gradients/s",
                                        "note": "gradient_av imaging, batched"},
            "checkpoint": plan,
            "e2e": e2e, "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "traffic_unit": "bytes per gradient (ncu, one FWD + one ADJ_EXACT "
                                         "launch per step)",
                         "traffic_source": "stored ncu figure (profiles/traffic.json), "
                                           "not measured in this run",
                         "kernel": "pf_step_kernel FWD + ADJ_EXACT (whole gradient loop)",
                         "alg_bytes_per_gradient": alg, "loop_ms": loop_b,
                         "peak_source": peak_kind},
            "cpu_baseline": cpu, "clocks": clocks}), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# --------------------------------------------------------------------------
# batch2d: uneven 2-D forward shots in one lockstep time loop
# --------------------------------------------------------------------------
B2_NSHOT, B2_H, B2_DT, B2_NBT = 64, 10.0, 0.001, 30


def batch2d_shots(seed, nshot=B2_NSHOT, scale=1.0):
    """Seeded shots: grids (nz, nx) in [256,1024] x [256,2048] (times
    `scale`), nt in [1000, 4000], layered velocity plus a smooth anomaly in
    [1500, 4500] m/s, one Ricker source of 10-30 Hz near the surface."""
    rng = np.random.default_rng(seed)
    shots = []
    for _ in range(nshot):
        nz = max(16, int(rng.integers(256, 1025) * scale))
        nx = max(16, int(rng.integers(256, 2049) * scale))
        nt = int(rng.integers(1000, 4001))
        z = np.arange(nz)[:, None]
        x = np.arange(nx)[None, :]
        nl = int(rng.integers(3, 8))
        ifaces = np.sort(rng.integers(1, nz, nl))
        vals = np.sort(rng.uniform(1500, 4000, nl + 1))
        v = np.full((nz, nx), vals[0])
        for val, zi in zip(vals[1:], ifaces):
            v = np.where(z >= zi, val, v)
        cz, cx, r = rng.uniform(0.3, 0.7) * nz, rng.uniform(0.2, 0.8) * nx, 0.1 * min(nz, nx)
        v = v * (1 + 0.1 * np.exp(-((z - cz) ** 2 + (x - cx) ** 2) / (2 * r * r)))
        v = np.clip(v, 1500, 4500).astype(np.float32)
        f0 = float(rng.uniform(10, 30))
        shots.append(dict(vel=v, nt=nt, dt=B2_DT, ax=[0, B2_H, nx], az=[0, B2_H, nz], ns=1,
                          sx=[int(rng.integers(nx // 4, 3 * nx // 4))], sz=[5], f=[f0],
                          t=[1.2 / f0], A=[1.0], nbt=B2_NBT, ct=0.01, gz=5))
    return shots


def _b2_cells(sh):
    return (sh["az"][2] + 2 * B2_NBT) * (sh["ax"][2] + 2 * B2_NBT) * sh["nt"]


B2_CROP = 400  # the reference's afd2dc corrupts its heap on the largest shots


def _b2_ref_worker(nt_s, seed, kind="reference"):
    """The reference's afd2dc (oracle/_ref; kind "port": the oracle's C
    restatement) on a B2_CROP^2 crop of the largest seeded shot for nt_s
    steps; returns (cell-updates, wall seconds)."""
    sys.path.insert(0, ROOT)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    sh = max(batch2d_shots(seed), key=lambda s: s["az"][2] * s["ax"][2])
    vel = np.ascontiguousarray(sh["vel"][:B2_CROP, :B2_CROP])
    nz, nx = vel.shape
    src = dict(sx=[nx // 2], sz=sh["sz"], f=sh["f"], t=sh["t"], A=sh["A"])
    t0 = time.perf_counter()
    if kind == "reference":
        sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
        import afdcfun  # the reference's own extension module
        s = np.array(src["sx"] + src["sz"] + src["f"] + src["t"] + src["A"], np.float32)
        afdcfun.afd2dc(vel.flatten(order="F"), s, 0, nt_s, nx, nz, 1, 0, nt_s, 0, 1, B2_NBT,
                       0.01, B2_DT, 0.0, B2_H, 0.0, B2_H)
    else:
        from oracle import oracle as O
        O.afd(vel, nt_s, B2_DT, (B2_H, B2_H), nbt=B2_NBT, ct=0.01, src=src)
    wall = time.perf_counter() - t0
    return (nz + 2 * B2_NBT) * (nx + 2 * B2_NBT) * nt_s, wall


def _b2_cpu_sample(workers, nt_s=100):
    """(Gpt/s, kind) of the CPU path on `workers` processes: the reference,
    or the oracle port when the reference's run fails."""
    for kind in ("reference", "port"):
        try:
            res = pool_map(_b2_ref_worker, [(nt_s, 5, kind)] * workers, timeout_s=300)
            return sum(r[0] for r in res) / max(r[1] for r in res) / 1e9, kind
        except Exception:  # noqa: BLE001
            continue
    raise RuntimeError("neither the reference nor the port ran")


def run_batch2d(args, world, rank, local):
    shots = batch2d_shots(5 + rank)
    if args.b2_nt > 0:
        for sh in shots:
            sh["nt"] = min(sh["nt"], args.b2_nt)
    cells = sum(_b2_cells(sh) for sh in shots)
    if args.impl == "reference":
        if rank != 0:
            return
        workers = max(1, min(os.cpu_count() or 1, 16))
        rates = []
        for i in range(args.warmup + args.steps):
            v, kind = _b2_cpu_sample(workers)
            if i >= args.warmup:
                rates.append(v)
        value = statistics.median(rates)
        print(json.dumps({
            "impl": "reference", "metric": "Gpt-updates/s (2-D uneven shot batch)",
            "value": value, "unit": "Gpt/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{len(shots)} 2-D shots, grids 256-1024 x 256-2048, "
                                   f"nt {'1000-4000' if args.b2_nt <= 0 else f'cut to {args.b2_nt}'}, "
                                   f"h=10m, nbt={B2_NBT}"},
            "cpu_baseline": {"value": value, "unit": "Gpt/s", "cores": workers, "kind": kind,
                             "sample": f"afd2dc on a {B2_CROP}^2 crop of the largest shot, 100 "
                                       f"steps, {workers} independent single-threaded processes"},
            "e2e": {"value": value, "unit": "Gpt/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}), flush=True)
        return
    import ctypes as C
    import torch
    import torch.distributed as dist
    from pywave_b200 import _lib as L
    from pywave_b200 import build as B
    from pywave_b200.afd import afd2d_batch
    B.build()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    lib = L.lib()
    n = len(shots)
    a = (L.AfdArgs * n)()
    keep, vp, sp, dp = [], [], [], []
    for k, sh in enumerate(shots):
        nz, nx = sh["az"][2], sh["ax"][2]
        x = a[k]
        x.dim, x.nz, x.nx, x.ny, x.nt, x.nbt, x.ct = 2, nz, nx, 1, sh["nt"], B2_NBT, 0.01
        x.dt, x.dz, x.dx, x.dy, x.ns, x.tri, x.jsnap, x.gz, x.flags = (
            B2_DT, B2_H, B2_H, B2_H, 1, 0, 0, sh["gz"], 0)
        v = torch.from_numpy(np.ascontiguousarray(sh["vel"].flatten(order="F"))).cuda()
        s = torch.tensor(sh["sx"] + sh["sz"] + sh["f"] + sh["t"] + sh["A"], dtype=torch.float32,
                         device="cuda")
        d = torch.empty(sh["nt"] * nx, device="cuda")
        keep += [v, s, d]
        vp.append(v.data_ptr())
        sp.append(s.data_ptr())
        dp.append(d.data_ptr())
    VP, SP, DP = ((C.c_void_p * n)(*q) for q in (vp, sp, dp))
    side = torch.cuda.Stream()

    def batch():
        L.check(lib.pw_afd_batch(n, C.cast(a, C.c_void_p), C.cast(VP, C.c_void_p),
                                 C.cast(SP, C.c_void_p), None, C.cast(DP, C.c_void_p),
                                 side.cuda_stream))
        return L.last_timing()

    def plain():
        for k in range(n):
            L.check(lib.pw_afd(C.byref(a[k]), vp[k], sp[k], None, dp[k], None, side.cuda_stream))

    with torch.cuda.stream(side):
        for _ in range(args.warmup):
            batch()
        clk = Clocks(local)
        clk.start()
        if world > 1:
            dist.barrier()
        side.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        loops, launches = [], 0
        e0.record(side)
        for _ in range(args.steps):
            ms, nst, tot = batch()
            loops.append(ms)
            launches += tot
        e1.record(side)
        side.synchronize()
        clocks = clk.stop()
        ms_b = max_over_ranks(e0.elapsed_time(e1), world)
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(side)
        plain()
        p1.record(side)
        side.synchronize()
        ms_p = max_over_ranks(p0.elapsed_time(p1), world)
    value = job_rate(cells, args.steps, world, ms_b) / 1e9
    plain_v = job_rate(cells, 1, world, ms_p) / 1e9
    e2e = None
    if not args.no_e2e:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            afd2d_batch(shots, stream=side.cuda_stream)
        side.synchronize()
        ems = max_over_ranks((time.perf_counter() - t0) * 1e3, world)
        e2e = {"value": job_rate(cells, args.steps, world, ems) / 1e9, "unit": "Gpt/s",
               "h2d_bytes_per_step": int(sum(sh["vel"].nbytes + 20 for sh in shots)),
               "d2h_bytes_per_step": int(sum(sh["nt"] * sh["ax"][2] * 4 for sh in shots))}
    peak, peak_kind = peaks()
    loop_ms = statistics.median(loops)
    achieved = cells * 16 / (loop_ms / 1e3) / 1e9
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            v, kind = _b2_cpu_sample(1)
            cpu = {"value": v, "unit": "Gpt/s", "cores": 1, "kind": kind,
                   "sample": f"afd2dc on a {B2_CROP}^2 crop of the largest shot, 100 steps, "
                             f"1 core"}
        except Exception as ex:  # noqa: BLE001
            cpu = {"value": None, "unit": "Gpt/s", "cores": 1, "kind": "reference",
                   "sample": f"failed: {ex!r}"[:200]}
    if rank == 0:
        print(json.dumps({
            "metric": "Gpt-updates/s (2-D uneven shot batch)", "value": value, "unit": "Gpt/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_b / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded layered models, Ricker sources)",
            "config": {"workload": f"{n} 2-D shots, grids 256-1024 x 256-2048, "
                                   f"nt {'1000-4000' if args.b2_nt <= 0 else f'cut to {args.b2_nt}'}, "
                                   f"h=10m dt=1ms nbt={B2_NBT}, one lockstep batch",
                       "cell_updates_per_step": cells,
                       "l2": "inputs larger than L2 (fields of all shots)"},
            "plain_per_shot": {"value": plain_v, "unit": "Gpt/s",
                               "note": "pw_afd one shot after another"},
            "batched_over_plain": value / plain_v,
            "e2e": e2e, "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "kernel": "batch_kernel (2-D march, all running shots)",
                         "loop_ms": loop_ms, "alg_bytes_per_step": cells * 16,
                         "peak_source": peak_kind},
            "cpu_baseline": cpu, "clocks": clocks}), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# --------------------------------------------------------------------------
# c1: one 2-D shot, three-layer 201x201 model, receivers at depth 5

C1_N, C1_NT = 201, 1501


def c1_model():
    vel = np.full((C1_N, C1_N), 1500, np.float32)
    vel[60:130] = 2200
    vel[130:] = 3000
    kw = dict(nt=C1_NT, dt=0.001, ax=[0, 10, C1_N], az=[0, 10, C1_N], ns=1, sx=[100], sz=[5],
              f=[20], t=[0.05], A=[1], nbt=NBT, ct=CT, jsnap=0, gz=5)
    return vel, kw


def _c1_ref_worker(kind="reference"):
    """One whole C1 propagation by the reference's afd2dc (oracle/_ref; kind
    "port": the oracle's C restatement), receivers at z=0 and no snapshots
    (afd2dc has no depth receivers; the propagation work is the same)."""
    sys.path.insert(0, ROOT)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    vel, kw = c1_model()
    t0 = time.perf_counter()
    if kind == "reference":
        sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
        import afdcfun  # the reference's own extension module
        s = np.array(kw["sx"] + kw["sz"] + kw["f"] + kw["t"] + kw["A"], np.float32)
        afdcfun.afd2dc(vel.flatten(order="F"), s, 0, C1_NT, C1_N, C1_N, 1, 0, C1_NT, 0, 1, NBT,
                       CT, 0.001, 0.0, 10.0, 0.0, 10.0)
    else:
        from oracle import oracle as O
        O.afd(vel, C1_NT, 0.001, (10.0, 10.0), nbt=NBT, ct=CT,
              src=dict(sx=kw["sx"], sz=kw["sz"], f=kw["f"], t=kw["t"], A=kw["A"]))
    return (C1_N + 2 * NBT) ** 2 * C1_NT, time.perf_counter() - t0


def _c1_cpu(workers):
    for kind in ("reference", "port"):
        try:
            res = pool_map(_c1_ref_worker, [(kind,)] * workers, timeout_s=300)
            return sum(r[0] for r in res) / max(r[1] for r in res) / 1e9, kind
        except Exception:  # noqa: BLE001
            continue
    raise RuntimeError("neither the reference nor the port ran")


def run_c1(args, world, rank, local):
    pts = (C1_N + 2 * NBT) ** 2 * C1_NT
    if args.impl == "reference":
        if rank != 0:
            return
        workers = max(1, min(os.cpu_count() or 1, 16))
        rates = []
        for i in range(args.warmup + args.steps):
            v, kind = _c1_cpu(workers)
            if i >= args.warmup:
                rates.append(v)
        value = statistics.median(rates)
        print(json.dumps({
            "impl": "reference", "metric": "Gpt-updates/s (2-D single shot)", "value": value,
            "unit": "Gpt/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": f"2-D shot {C1_N}^2 three layers h=10m "
                                                        f"nt={C1_NT} nbt={NBT}"},
            "cpu_baseline": {"value": value, "unit": "Gpt/s", "cores": workers, "kind": kind,
                             "sample": f"whole afd2dc propagation, {workers} independent "
                                       "single-threaded processes"},
            "e2e": {"value": value, "unit": "Gpt/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}), flush=True)
        return
    import ctypes as C
    import torch
    import torch.distributed as dist
    import pywave_b200 as pw
    from pywave_b200 import _lib as L
    from pywave_b200 import build as B
    B.build()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    lib = L.lib()
    vel, kw = c1_model()
    a = L.AfdArgs(dim=2, nz=C1_N, nx=C1_N, ny=1, nt=C1_NT, nbt=NBT, ct=CT, dt=0.001, dz=10.0,
                  dx=10.0, dy=10.0, ns=1, tri=0, jsnap=0, gz=5, flags=0)
    v_d = torch.from_numpy(np.ascontiguousarray(vel.flatten(order="F"))).cuda()
    s_d = torch.tensor(kw["sx"] + kw["sz"] + kw["f"] + kw["t"] + kw["A"], dtype=torch.float32,
                       device="cuda")
    d_d = torch.empty(C1_NT * C1_N, device="cuda")
    st = torch.cuda.current_stream().cuda_stream

    def shot():
        L.check(lib.pw_afd(C.byref(a), v_d.data_ptr(), s_d.data_ptr(), None, d_d.data_ptr(),
                           None, st))
        return L.last_timing()

    for _ in range(args.warmup):
        shot()
    clk = Clocks(local)
    clk.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    loops, launches = [], 0
    e0.record()
    step_launches = 0
    for _ in range(args.steps):
        ms, nst, tot = shot()
        loops.append(ms)
        launches += tot
        step_launches = nst
    e1.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms_b = max_over_ranks(e0.elapsed_time(e1), world)
    value = job_rate(pts, args.steps, world, ms_b) / 1e9
    kernel = ("resident_kernel (one cluster launch for all steps, fields in shared memory)"
              if step_launches == 1 else "march_kernel<TWO_D> (one launch per step)")
    e2e = None
    if not args.no_e2e:
        pw.afd2d(vel, **kw)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            pw.afd2d(vel, **kw)
        ems = max_over_ranks((time.perf_counter() - t0) * 1e3, world)
        e2e = {"value": job_rate(pts, args.steps, world, ems) / 1e9, "unit": "Gpt/s",
               "h2d_bytes_per_step": int(vel.nbytes + 20),
               "d2h_bytes_per_step": int(C1_NT * C1_N * 4)}
    peak, peak_kind = peaks()
    loop_ms = statistics.median(loops)
    achieved = pts * 16 / (loop_ms / 1e3) / 1e9
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            v, kind = _c1_cpu(1)
            cpu = {"value": v, "unit": "Gpt/s", "cores": 1, "kind": kind,
                   "sample": "the whole C1 propagation by afd2dc, 1 core"}
        except Exception as ex:  # noqa: BLE001
            cpu = {"value": None, "unit": "Gpt/s", "cores": 1, "kind": "reference",
                   "sample": f"failed: {ex!r}"[:200]}
    if rank == 0:
        print(json.dumps({
            "metric": "Gpt-updates/s (2-D single shot)", "value": value, "unit": "Gpt/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_b / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (three-layer model)",
            "config": {"workload": f"2-D shot {C1_N}^2 h=10m nt={C1_NT} dt=1ms nbt={NBT}, 20 Hz "
                                   "source at (5,100), receivers at z=5",
                       "points_per_step": pts,
                       "l2": "working set (3 fields, 0.8 MB) inside L2: no flush, "
                             "an L2-resident latency/launch-bound case"},
            "e2e": e2e, "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "kernel": kernel, "loop_ms": loop_ms,
                         "alg_bytes_per_step": pts * 16, "peak_source": peak_kind},
            "cpu_baseline": cpu, "clocks": clocks}), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# --------------------------------------------------------------------------
# afd3d: 3-D forward modelling of the headline's model (traces of 3 sources)
# --------------------------------------------------------------------------
def a3_sources(pos, f, t):
    """The afd3d source array (sx, sy, sz, f, t, A rows) of c2_model's shots."""
    return np.concatenate([pos[:, 0], pos[:, 1], pos[:, 2], f, t, np.ones(3)]).astype(np.float32)


def _a3_ref_worker(n, nt_s, kind):
    """Forward modelling of the 3 sources by the reference's afd3dc
    (oracle/_ref; kind "port": the oracle's C restatement) for nt_s steps;
    wall seconds."""
    sys.path.insert(0, ROOT)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    vel, pos, f, t = c2_model(n, 1234, nt_s)
    src = a3_sources(pos, f, t)
    if kind == "reference":
        sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
        import afdcfun  # the reference's own extension module
        t0 = time.perf_counter()
        afdcfun.afd3dc(vel.flatten(order="F"), src, 0, nt_s, n, n, n, 3, 0, 0, 0, 1, NBT, CT, DT,
                       0.0, H, 0.0, H, 0.0, H)
    else:
        from oracle import oracle as O
        O.lib()
        t0 = time.perf_counter()
        O.afd(vel, nt_s, DT, (H, H, H), nbt=NBT, ct=CT,
              src=dict(sx=pos[:, 0], sy=pos[:, 1], sz=pos[:, 2], f=f, t=t, A=np.ones(3)))
    return time.perf_counter() - t0


def _a3_cpu(n, workers):
    """Per-step rate of the reference's 3-D forward in `workers` processes:
    calls of REF_STEPS[0] and REF_STEPS[1] steps, their difference excluding
    the per-call set-up.  Returns (Gpt/s, kind, seconds per step)."""
    for kind in ("reference", "port"):
        try:
            a = pool_map(_a3_ref_worker, [(n, REF_STEPS[0], kind)] * workers, timeout_s=600)
            b = pool_map(_a3_ref_worker, [(n, REF_STEPS[1], kind)] * workers, timeout_s=600)
        except Exception:  # noqa: BLE001
            continue
        d = max(b) - max(a)
        if d <= 0:
            raise RuntimeError(f"reference timing: {REF_STEPS[1]} steps took no longer than "
                               f"{REF_STEPS[0]}")
        extra = REF_STEPS[1] - REF_STEPS[0]
        return (n + 2 * NBT) ** 3 * extra * workers / d / 1e9, kind, d / extra
    raise RuntimeError("neither the reference nor the port ran")


def run_afd3d(args, world, rank, local):
    n, nt = args.n, args.nt
    pts = (n + 2 * NBT) ** 3 * nt
    metric = "Gpt-updates/s (3-D forward modelling, 3 sources)"
    workload = (f"3-D forward modelling {n}^3 h=10m nt={nt} nbt={NBT}, the TRI benchmark's "
                "velocity model, 3 seeded Ricker sources, receivers on the surface")
    if args.impl == "reference":
        if rank != 0:
            return
        workers = max(1, min(os.cpu_count() or 1, 16))
        rates, per = [], []
        for i in range(args.warmup + args.steps):
            v, kind, ps = _a3_cpu(n, workers)
            if i >= args.warmup:
                rates.append(v)
                per.append(ps)
        value = statistics.median(rates)
        print(json.dumps({
            "impl": "reference", "metric": metric, "value": value, "unit": "Gpt/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": workload},
            "cpu_baseline": {"value": value, "unit": "Gpt/s", "cores": workers, "kind": kind,
                             "sample": f"afd3dc forward, {workers} independent single-threaded "
                                       f"processes, calls of {REF_STEPS[0]} and {REF_STEPS[1]} "
                                       f"steps ({statistics.median(per):.3f} s per step from "
                                       "their difference)"},
            "e2e": {"value": value, "unit": "Gpt/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}), flush=True)
        return
    import ctypes as C
    import torch
    import torch.distributed as dist
    from pywave_b200 import _lib as L
    from pywave_b200 import build as B
    B.build()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    lib = L.lib()
    vel, pos, f, t = c2_model(n, 1234 + rank, nt)
    src = a3_sources(pos, f, t)
    a = L.AfdArgs(dim=3, nz=n, nx=n, ny=n, nt=nt, nbt=NBT, ct=CT, dt=DT, dz=H, dx=H, dy=H, ns=3,
                  tri=0, jsnap=0, gz=0, flags=0)
    v_d = torch.from_numpy(np.ascontiguousarray(vel.flatten(order="F"))).cuda()
    s_d = torch.from_numpy(src).cuda()
    d_d = torch.empty(n * n * nt, device="cuda")
    st = torch.cuda.current_stream().cuda_stream

    def shot():
        L.check(lib.pw_afd(C.byref(a), v_d.data_ptr(), s_d.data_ptr(), None, d_d.data_ptr(),
                           None, st))
        return L.last_timing()

    for _ in range(args.warmup):
        shot()
    clk = Clocks(local)
    clk.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    loops, launches = [], 0
    e0.record()
    for _ in range(args.steps):
        ms, nst, tot = shot()
        loops.append(ms)
        launches += tot
    e1.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms_b = max_over_ranks(e0.elapsed_time(e1), world)
    value = job_rate(pts, args.steps, world, ms_b) / 1e9
    # e2e: the same C-ABI call with host buffers (copies inside the timed region)
    e2e = None
    if not args.no_e2e:
        vel_h = torch.from_numpy(np.ascontiguousarray(vel.flatten(order="F"))).pin_memory()
        dat_h = torch.empty(n * n * nt).pin_memory()
        ah = L.AfdArgs(dim=3, nz=n, nx=n, ny=n, nt=nt, nbt=NBT, ct=CT, dt=DT, dz=H, dx=H, dy=H,
                       ns=3, tri=0, jsnap=0, gz=0, flags=L.PW_HOST_PTRS)

        def shot_host():
            L.check(lib.pw_afd(C.byref(ah), vel_h.data_ptr(), src.ctypes.data, None,
                               dat_h.data_ptr(), None, st))

        shot_host()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            shot_host()
        torch.cuda.synchronize()
        ems = max_over_ranks((time.perf_counter() - t0) * 1e3, world)
        e2e = {"value": job_rate(pts, args.steps, world, ems) / 1e9, "unit": "Gpt/s",
               "h2d_bytes_per_step": int(vel.nbytes + src.nbytes),
               "d2h_bytes_per_step": int(dat_h.numel() * 4)}
    peak, peak_kind = peaks()
    loop_ms = statistics.median(loops)
    kern_ms = loop_ms / nt
    alg = (n + 2 * NBT) ** 3 * 16  # A, B, vv read and B written per expanded point per step
    achieved = alg / (kern_ms / 1e3) / 1e9
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            v, kind, ps = _a3_cpu(n, 1)
            cpu = {"value": v, "unit": "Gpt/s", "cores": 1, "kind": kind,
                   "sample": f"afd3dc forward on the {n + 2 * NBT}^3 expanded grid of the same "
                             f"model and sources, 1 core; calls of {REF_STEPS[0]} and "
                             f"{REF_STEPS[1]} steps, {ps:.3f} s per step from their difference"}
        except Exception as ex:  # noqa: BLE001
            cpu = {"value": None, "unit": "Gpt/s", "cores": 1, "kind": "reference",
                   "sample": f"failed: {ex!r}"[:200]}
    if rank == 0:
        print(json.dumps({
            "metric": metric, "value": value, "unit": "Gpt/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_b / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded velocity and sources)",
            "config": {"workload": workload, "points_per_step": pts,
                       "l2": "inputs larger than L2 (fields 0.21 GB, vv 0.07 GB)"},
            "e2e": e2e, "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "kernel": "tile_kernel<forward> (one launch per step)",
                         "kernel_ms": kern_ms, "alg_bytes_per_launch": alg,
                         "peak_source": peak_kind},
            "cpu_baseline": cpu, "clocks": clocks}), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# --------------------------------------------------------------------------
# fwi3d: 3-D FWI gradients/s, 400 x 400 x 200 at 12.5 m (km units)
# --------------------------------------------------------------------------
F3_NZ, F3_NX, F3_NY, F3_H, F3_DT, F3_NB, F3_COEF, F3_F0 = 200, 400, 400, 0.0125, 0.001, 20, 0.015, 12.0


def fwi3d_models(seed):
    """True model: a smooth gradient 1.8 -> 3.6 km/s over the depth with a
    seeded 3% smooth perturbation and a salt-like body of 4.5 km/s (an
    ellipsoid of seeded centre and radii); start model: the true model
    Gaussian-smoothed with sigma 10 points.  (nz, nx, ny) float32."""
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    z = np.arange(F3_NZ, dtype=np.float32)[:, None, None] / (F3_NZ - 1)
    v = 1.8 + 1.8 * z + np.zeros((F3_NZ, F3_NX, F3_NY), np.float32)
    p = gaussian_filter(rng.standard_normal((F3_NZ // 4, F3_NX // 4, F3_NY // 4)), 2.0)
    p = np.repeat(np.repeat(np.repeat(p / np.abs(p).max(), 4, 0), 4, 1), 4, 2)
    v = v * (1.0 + 0.03 * p.astype(np.float32))
    cz, cx, cy = rng.uniform(0.45, 0.65) * F3_NZ, rng.uniform(0.35, 0.65) * F3_NX, \
        rng.uniform(0.35, 0.65) * F3_NY
    rz, rx, ry = 0.12 * F3_NZ, rng.uniform(0.1, 0.2) * F3_NX, rng.uniform(0.1, 0.2) * F3_NY
    iz, ix, iy = np.ogrid[:F3_NZ, :F3_NX, :F3_NY]
    salt = ((iz - cz) / rz) ** 2 + ((ix - cx) / rx) ** 2 + ((iy - cy) / ry) ** 2 <= 1.0
    v = np.where(salt, 4.5, v).astype(np.float32)
    vs = gaussian_filter(v.astype(np.float64), 10.0).astype(np.float32)
    return v, vs


def fwi3d_geom(ns, nt):
    """ns shots on a square grid at depth 5, 160 x 160 receivers spread over
    the surface at depth 1, 12 Hz Ricker."""
    side = int(round(np.sqrt(ns)))
    sxs = [int((i + 0.5) * F3_NX / side) for i in range(side)]
    sys_ = [int((j + 0.5) * F3_NY / side) for j in range(side)]
    src = [(5, x, y) for y in sys_ for x in sxs][:ns]
    rx = [int((i + 0.5) * F3_NX / 160) for i in range(160)]
    ry = [int((j + 0.5) * F3_NY / 160) for j in range(160)]
    return dict(nb=F3_NB, coef=F3_COEF, dz=F3_H, dx=F3_H, dy=F3_H, nt=nt, dt=F3_DT, src=src,
                rz=1, rx=rx, ry=ry)


def fwi3d_wavelet(nt):
    t = np.arange(nt) * F3_DT - 1.2 / F3_F0
    a = (np.pi * F3_F0 * t) ** 2
    return (1e6 * (1 - 2 * a) * np.exp(-a)).astype(np.float32)


def run_fwi3d(args, world, rank, local):
    ns, nt = args.fwi3d_shots, args.fwi3d_nt
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable":
                              "the reference has no 3-D FWI (pywave's FWI is 2-D only)"}),
                  flush=True)
        return
    import ctypes
    import torch
    from pywave_b200 import _lib as L
    from pywave_b200 import build as B
    from pywave_b200 import fwi3d
    B.build()
    torch.cuda.set_device(local)
    st = torch.cuda.current_stream().cuda_stream
    lib = L.lib()
    vt, vs = fwi3d_models(21 + rank)
    geom = fwi3d_geom(ns, nt)
    wav = fwi3d_wavelet(nt)
    a, keep = fwi3d.fwi3d_args(vt.shape, geom, 0, FWI_BUDGET)
    dev = lambda arr: torch.from_numpy(np.ascontiguousarray(arr)).cuda()
    vt_d = dev(vt.flatten(order="F"))
    vs_d = dev(vs.flatten(order="F"))
    wav_d = dev(wav)
    nr = a.nrx * a.nry
    dobs_d = torch.empty(ns * nr * nt, device="cuda")
    L.check(lib.pw_pfwi3d_forward(a, vt_d.data_ptr(), wav_d.data_ptr(), dobs_d.data_ptr(), st))
    g_d = torch.empty(vt.size, device="cuda")
    J = ctypes.c_double(0.0)

    def grad():
        L.check(lib.pw_pfwi3d_gradient(a, vs_d.data_ptr(), wav_d.data_ptr(), dobs_d.data_ptr(),
                                       None, g_d.data_ptr(), ctypes.byref(J), 0, st))
        return L.last_timing()

    for _ in range(args.warmup):
        grad()
    torch.cuda.synchronize()
    clk = Clocks(local)
    clk.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches, loops = 0, []
    e0.record()
    for _ in range(args.steps):
        ms, nst, tot = grad()
        loops.append(ms)
        launches += tot
    e1.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1)
    k, nsb, nbytes, rc = L.last_fwi_plan()
    pad = (F3_NZ + 2 * F3_NB) * (F3_NX + 2 * F3_NB) * (F3_NY + 2 * F3_NB)
    # algorithmic bytes per padded point-step-shot as in fwi2d (forward 20 B +
    # exact adjoint 28 B), plus the recomputed forward steps (20 B each)
    alg = (48.0 + 20.0 * (rc - 1.0)) * pad * nt * ns
    peak, peak_kind = peaks()
    loop_ms = statistics.median(loops)
    achieved = alg / (loop_ms / 1e3) / 1e9
    if rank == 0:
        print(json.dumps({
            "metric": f"FWI gradients/s (3-D exact adjoint, {ns} shots)",
            "value": job_rate(1, args.steps, world, ms), "unit": "gradients/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (FP64 misfit)",
            "data": "synthetic (seeded gradient model with a 4.5 km/s salt body, start = smoothed)",
            "config": {"workload": f"3-D FWI gradient {F3_NZ}x{F3_NX}x{F3_NY} h=12.5m nt={nt} "
                                   f"dt=1ms shots={ns} receivers=160x160 nb={F3_NB} 12 Hz",
                       "padded_cells": pad},
            # forward (recomputed steps included) and adjoint point-updates
            "point_updates_per_s": pad * nt * ns * (rc + 1.0) / (ms / args.steps / 1e3),
            "checkpoint": {"budget_bytes": FWI_BUDGET, "interval_k": k, "shots_per_batch": nsb,
                           "device_bytes": nbytes, "recompute_factor": rc},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "kernel": "pf3_step_kernel FWD + ADJ_EXACT (whole gradient loop)",
                         "alg_bytes_per_gradient": alg, "loop_ms": loop_ms,
                         "peak_source": peak_kind},
            "cpu_baseline": {"value": None, "unit": "gradients/s", "cores": 0,
                             "kind": "unavailable",
                             "sample": "the reference has no 3-D FWI"},
            "clocks": clocks}), flush=True)


# pfwi passive mode 4 at the size of the reference's passive demos
# (demos/test_pfwi_mod2d.py): 130 x 334 at 8 x 12 m, nb 60, nt 3001, 3 shots,
# 30 CG iterations of the source inversion per shot
LS_NZ, LS_NX, LS_DZ, LS_DX, LS_NT, LS_DT, LS_NB, LS_COEF, LS_NS = \
    130, 334, 0.008, 0.012, 3001, 0.001, 60, 0.005, 3


def lstri_par(niter, ns=LS_NS, nt=LS_NT):
    return dict(nz=LS_NZ, nx=LS_NX, dz=LS_DZ, dx=LS_DX, oz=0, ox=0, nt=nt, dt=LS_DT, ot=0,
                ns=ns, ds=0.1, os=0.0, nb=LS_NB, coef=LS_COEF, f0=10, acqui_type=1, interval=1,
                niter=niter)


def lstri_case(seed, ns=LS_NS, nt=LS_NT):
    """Velocity 1.8 -> 3.0 km/s with depth plus 0.2 seeded noise; per shot
    three buried point sources carrying 10 Hz Ricker pulses of amplitude 1e6
    at seeded delays (the demos' source scale)."""
    rng = np.random.default_rng(seed)
    z = np.arange(LS_NZ, dtype=np.float32)[:, None]
    vel = (1.8 + 1.2 * z / LS_NZ + 0.2 * rng.random((LS_NZ, LS_NX))).astype(np.float32)
    src = np.zeros((ns, nt, LS_NX, LS_NZ), np.float32)  # [ns][nt][nx][nz]
    t = np.arange(nt) * LS_DT
    for s in range(ns):
        for _ in range(3):
            iz, ix = int(rng.integers(60, 125)), int(rng.integers(20, LS_NX - 20))
            a = (np.pi * 10.0 * (t - float(rng.uniform(0.1, 0.5)))) ** 2
            src[s, :, ix, iz] = (1e6 * (1 - 2 * a) * np.exp(-a)).astype(np.float32)
    return vel, src


def _ls_ref_worker(kind):
    """One lstric modelling call (inv 0) of one shot at the benchmark size by
    the reference itself (oracle/_ref pfwicfun; kind "port": the oracle's
    restatement); returns (point-updates, seconds)."""
    sys.path.insert(0, ROOT)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    vel, src = lstri_case(7, ns=1)
    par = lstri_par(1, ns=1)
    pts = (LS_NZ + 2 * LS_NB) * (LS_NX + 2 * LS_NB) * LS_NT
    if kind == "reference":
        sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
        import pfwicfun  # the reference's own extension module
        from pywave_b200.pfwi import fillpar, pararray
        arr = pararray(fillpar(dict(par, inv=0)))
        q = np.full(LS_NZ * LS_NX, 1e4, np.float32)
        flat = np.ascontiguousarray(src[0].reshape(-1))  # [nt][nx][nz] = F-order (nz,nx,nt)
        t0 = time.perf_counter()
        pfwicfun.lstric(vel.flatten(order="F"), q, np.zeros(LS_NT, np.float32), flat, arr)
    else:
        from oracle import oracle as O
        m = src[0].transpose(2, 1, 0)
        t0 = time.perf_counter()
        O.timerev(False, vel, LS_NT, LS_NB, LS_COEF, LS_DZ, LS_DX, LS_DT, mod=m)
    return pts, time.perf_counter() - t0


def _ls_cpu(workers):
    for kind in ("reference", "port"):
        try:
            res = pool_map(_ls_ref_worker, [(kind,)] * workers, timeout_s=600)
            return sum(r[0] for r in res) / max(r[1] for r in res) / 1e9, kind
        except Exception:  # noqa: BLE001
            continue
    raise RuntimeError("neither the reference nor the port ran")


def run_lstri(args, world, rank, local):
    niter, nt = args.lstri_niter, args.lstri_nt
    pad = (LS_NZ + 2 * LS_NB) * (LS_NX + 2 * LS_NB)
    cfg = {"workload": f"pfwi mode 4 LS-TRI source inversion {LS_NZ}x{LS_NX} dz=8m dx=12m "
                       f"nt={nt} nb={LS_NB} shots={LS_NS} CG iterations={niter}",
           "padded_cells": pad}
    metric = "Gpt-updates/s (2-D time-reversal operator, LS-TRI inversion)"
    if args.impl == "reference":
        if rank != 0:
            return
        workers = max(1, min(os.cpu_count() or 1, 16))
        rates = []
        for i in range(args.warmup + args.steps):
            v, kind = _ls_cpu(workers)
            if i >= args.warmup:
                rates.append(v)
        value = statistics.median(rates)
        print(json.dumps({
            "impl": "reference", "metric": metric, "value": value, "unit": "Gpt/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": value, "unit": "Gpt/s", "cores": workers, "kind": kind,
                             "sample": f"one lstric modelling call (inv 0, one shot, nt={LS_NT}) "
                                       f"per process, {workers} single-threaded processes"},
            "e2e": {"value": value, "unit": "Gpt/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}), flush=True)
        return
    import torch
    import torch.distributed as dist
    from pywave_b200 import _lib as L
    from pywave_b200 import build as B
    from pywave_b200 import lstri, pfwicfun
    from pywave_b200.pfwi import fillpar, pararray
    B.build()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    vel, src = lstri_case(7 + rank, nt=nt)
    par = lstri_par(niter, nt=nt)
    v_d = torch.from_numpy(np.ascontiguousarray(vel.T)).cuda()
    s_d = torch.from_numpy(src).cuda()
    d_d = torch.empty((LS_NS, LS_NX, nt), device="cuda")
    lstri.lstri_forward_torch(v_d, s_d, d_d, par)  # the observed data
    inv_d = torch.empty_like(s_d)
    del s_d

    def step():
        lstri.lstri_invert_torch(v_d, d_d, inv_d, par)
        return L.last_timing()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = Clocks(local)
    clk.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = 0
    e0.record()
    for _ in range(args.steps):
        launches += step()[2]
    e1.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    updates = pad * nt * 2 * niter * LS_NS  # adjoint + modelling per iteration
    # one modelling operator alone, timed on the device (resident launch)
    fwd_ms = []
    scratch = torch.empty_like(d_d[0])
    for _ in range(3):
        lstri.timerev_torch(False, v_d, dict(par, ns=1), inv_d[0], scratch)
        fwd_ms.append(L.last_timing()[0])
    op_ms = statistics.median(fwd_ms)
    # fp32 issue bound of one 16-SM cluster: 40 float operations per cell
    # (Laplacian 30, update 3, two sponge products, injection 2)
    sm_clk = (clocks or {}).get("sm_mhz") or 1965.0
    cluster_flops = 16 * 128 * sm_clk * 1e6
    op_flops = 40.0 * pad * nt
    # end to end through the drop-in module: host data in, host source field out
    e2e = None
    if not args.no_e2e:
        dh = np.ascontiguousarray(d_d.cpu().numpy().reshape(-1))  # [ns][nx][nt]
        arr = pararray(fillpar(dict(par, inv=1)))
        q = np.full(LS_NZ * LS_NX, 1e4, np.float32)
        t0 = time.perf_counter()
        out = pfwicfun.lstric(vel.flatten(order="F"), q, np.zeros(nt, np.float32), dh, arr)
        wall = time.perf_counter() - t0
        e2e = {"value": updates / wall / 1e9, "unit": "Gpt/s",
               "h2d_bytes_per_step": int(dh.nbytes + vel.nbytes),
               "d2h_bytes_per_step": int(out.nbytes)}
    cpu = None
    if not args.no_cpu_baseline and rank == 0:
        workers = max(1, min(os.cpu_count() or 1, 16))
        v, kind = _ls_cpu(workers)
        cpu = {"value": v, "unit": "Gpt/s", "cores": workers, "kind": kind,
               "sample": f"one lstric modelling call (inv 0, one shot, nt={LS_NT}) per process, "
                         f"{workers} single-threaded processes"}
    peak, peak_kind = peaks()
    src_bytes = 4.0 * LS_NZ * LS_NX * nt  # the modelling operator reads the source field
    if rank == 0:
        print(json.dumps({
            "metric": metric, "value": job_rate(updates, args.steps, world, ms) / 1e9,
            "unit": "Gpt/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (FP64 CG dots)",
            "data": "synthetic (seeded layered model, 3 buried Ricker sources per shot)",
            "config": cfg, "inversions_per_s": 1000.0 * args.steps / ms,
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": src_bytes / (op_ms / 1e3) / 1e9,
                         "peak": peak, "unit": "GB/s",
                         "frac": src_bytes / (op_ms / 1e3) / 1e9 / peak, "traffic": None,
                         "kernel": "tr::resident_kernel modelling (one shot, one launch)",
                         "op_ms": op_ms, "peak_source": peak_kind,
                         "cluster_fp32_frac": op_flops / (op_ms / 1e3) / cluster_flops,
                         "note": "one 16-SM cluster per shot: bound by that cluster's fp32 "
                                 "issue and its per-step barrier, not by HBM"},
            "e2e": e2e, "cpu_baseline": cpu, "clocks": clocks}), flush=True)


def _pas_ref_worker(kind, nt_s):
    """One passive gradient (gradient_pas_av) of one shot at the benchmark
    grid over nt_s steps by the reference itself (oracle/_ref libpwref;
    kind "port": the oracle's restatement); returns (point-updates, s)."""
    sys.path.insert(0, ROOT)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    vel, src = lstri_case(7, ns=1, nt=nt_s)
    par = lstri_par(1, ns=1, nt=nt_s)
    pts = 2.0 * (LS_NZ + 2 * LS_NB) * (LS_NX + 2 * LS_NB) * nt_s  # forward + backward
    dobs = np.zeros((1, LS_NX, nt_s), np.float32)
    sflat = np.ascontiguousarray(src.reshape(-1))
    if kind == "reference":
        import ctypes as C
        L = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libpwref.so"))
        f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
        L.refdrv_gradient_pas.argtypes = [f32p] * 6 + [C.c_int, C.c_float, C.c_float, f32p, f32p]
        parr = np.array([par[k] for k in ("nz", "nx", "dz", "dx", "oz", "ox", "nt", "dt", "ot",
                                          "ns", "ds", "os", "nb", "coef", "f0", "acqui_type",
                                          "interval")], np.float32)
        g = np.zeros(LS_NZ * LS_NX, np.float32)
        fc = np.zeros(1, np.float32)
        t0 = time.perf_counter()
        L.refdrv_gradient_pas(parr, np.ascontiguousarray(vel.flatten(order="F")),
                              np.full(LS_NZ * LS_NX, 1e4, np.float32), np.zeros(nt_s, np.float32),
                              np.ascontiguousarray(dobs.reshape(-1)), sflat, 1, 0.0,
                              float(np.float32(0.5) / np.float32(LS_DT)), g, fc)
    else:
        from oracle import oracle as O
        geo = O.pfwi_geometry(LS_NZ, LS_NX, LS_DZ, LS_DX, 0, 0, 1, 0.1, 0.0, LS_NB)
        t0 = time.perf_counter()
        O.pfwi_gradient_pas(vel, src.transpose(3, 2, 1, 0), dobs.transpose(2, 1, 0), LS_NB, LS_COEF,
                            LS_DZ, LS_DX, LS_DT, geo, 1, nt_s)
    return pts, time.perf_counter() - t0


def _pas_cpu(workers, nt_s):
    for kind in ("reference", "port"):
        try:
            res = pool_map(_pas_ref_worker, [(kind, nt_s)] * workers, timeout_s=600)
            return sum(r[0] for r in res) / max(r[1] for r in res) / 1e9, kind
        except Exception:  # noqa: BLE001
            continue
    raise RuntimeError("neither the reference nor the port ran")


def run_pfwic(args, world, rank, local):
    """Passive FWI (pfwic) at the passive demos' grid: a step is one passive
    gradient (gradient_pas_av: forward with the source fields, backward with
    the residual, imaging) of all shots, the unit pfwic's L-BFGS spends its
    time in."""
    nt = args.lstri_nt
    pad = (LS_NZ + 2 * LS_NB) * (LS_NX + 2 * LS_NB)
    cfg = {"workload": f"pfwi mode 4 passive FWI gradient {LS_NZ}x{LS_NX} dz=8m dx=12m nt={nt} "
                       f"nb={LS_NB} shots={LS_NS} (gradient_pas_av, reference mode)",
           "padded_cells": pad}
    metric = "passive FWI gradients/s (pfwic's gradient_pas_av)"
    nt_ref = min(nt, 600)
    if args.impl == "reference":
        if rank != 0:
            return
        workers = max(1, min(os.cpu_count() or 1, 16))
        rates = []
        for i in range(args.warmup + args.steps):
            v, kind = _pas_cpu(workers, nt_ref)
            if i >= args.warmup:
                rates.append(v)
        gps = statistics.median(rates) * 1e9 / (2.0 * pad * nt * LS_NS)
        print(json.dumps({
            "impl": "reference", "metric": metric, "value": gps, "unit": "gradients/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": gps, "unit": "gradients/s", "cores": workers, "kind": kind,
                             "sample": f"one gradient_pas_av of one shot over nt={nt_ref} per "
                                       f"process, {workers} single-threaded processes, scaled to "
                                       f"{LS_NS} shots x nt={nt}"},
            "e2e": {"value": gps, "unit": "gradients/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}), flush=True)
        return
    import ctypes
    import torch
    import torch.distributed as dist
    from pywave_b200 import _lib as L
    from pywave_b200 import build as B
    from pywave_b200 import fwi, lstri
    B.build()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from scipy.ndimage import gaussian_filter
    vel, src = lstri_case(7 + rank, nt=nt)
    vs = gaussian_filter(vel.astype(np.float64), 8.0).astype(np.float32)
    par = lstri_par(1, nt=nt)
    st = torch.cuda.current_stream().cuda_stream
    v_d = torch.from_numpy(np.ascontiguousarray(vel.T)).cuda()
    s_d = torch.from_numpy(src).cuda()  # [ns][nt][nx][nz]
    d_d = torch.empty((LS_NS, LS_NX, nt), device="cuda")
    lstri.lstri_forward_torch(v_d, s_d, d_d, par)  # observed data as the demos make it
    vs_d = torch.from_numpy(np.ascontiguousarray(vs.T)).cuda()
    g_d = torch.empty(LS_NZ * LS_NX, device="cuda")
    a = fwi.fwi_args(par, 0)
    J = ctypes.c_double(0.0)
    lib = L.lib()

    def grad():
        L.check(lib.pw_pfwi_gradient_passive(a, L.PW_GRAD_REFERENCE, vs_d.data_ptr(),
                                             s_d.data_ptr(), d_d.data_ptr(), None, g_d.data_ptr(),
                                             ctypes.byref(J), 0, st))
        return L.last_timing()

    for _ in range(args.warmup):
        grad()
    torch.cuda.synchronize()
    clk = Clocks(local)
    clk.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches, loops = 0, []
    e0.record()
    for _ in range(args.steps):
        ms_, nst, tot = grad()
        loops.append(ms_)
        launches += tot
    e1.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    # algorithmic bytes per padded point-step-shot: forward 20 B (+4 B of the
    # source field on the interior), reference backward 20 B + imaging reads
    loop_ms = statistics.median(loops)
    nzx = LS_NZ * LS_NX
    # algorithmic bytes per step and shot: forward 16 B per padded point (A,
    # B, V read; B write) + 8 B per interior cell (source sample, snapshot);
    # reference backward 16 B per padded point + 24 B per imaged interior
    # cell (three snapshots, -2/v^3, gradient read and write)
    alg = (32.0 * pad + 32.0 * nzx) * nt * LS_NS
    peak, peak_kind = peaks()
    e2e = None
    if not args.no_e2e:
        # the same gradient through the public API with host arrays (the
        # source fields, data and model copied in, the gradient copied out)
        dh = np.ascontiguousarray(d_d.cpu().numpy().transpose(2, 1, 0))  # (nt, nr, ns)
        sh = np.ascontiguousarray(src.transpose(3, 2, 1, 0))             # (nz, nx, nt, ns)
        fwi.gradient_passive(vs, sh, dh, par)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            fwi.gradient_passive(vs, sh, dh, par)
        wall = time.perf_counter() - t0
        e2e = {"value": args.steps / wall, "unit": "gradients/s",
               "h2d_bytes_per_step": int(dh.nbytes + sh.nbytes + vs.nbytes),
               "d2h_bytes_per_step": 4 * nzx}
    cpu = None
    if not args.no_cpu_baseline and rank == 0:
        workers = max(1, min(os.cpu_count() or 1, 16))
        v, kind = _pas_cpu(workers, nt_ref)
        cpu = {"value": v * 1e9 / (2.0 * pad * nt * LS_NS), "unit": "gradients/s",
               "cores": workers, "kind": kind,
               "sample": f"one gradient_pas_av of one shot over nt={nt_ref} per process, "
                         f"{workers} single-threaded processes, scaled to {LS_NS} shots x nt={nt}"}
    if rank == 0:
        print(json.dumps({
            "metric": metric, "value": job_rate(1, args.steps, world, ms), "unit": "gradients/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (FP64 misfit)",
            "data": "synthetic (seeded layered model, 3 buried Ricker sources per shot; data by "
                    "lstric on the true model, start = smoothed)",
            "config": cfg, "gpu_launches": launches,
            "point_updates_per_s": 2.0 * pad * nt * LS_NS / (ms / args.steps / 1e3),
            "roofline": {"bound": "hbm", "achieved": alg / (loop_ms / 1e3) / 1e9, "peak": peak,
                         "unit": "GB/s", "frac": alg / (loop_ms / 1e3) / 1e9 / peak,
                         "traffic": None, "kernel": "pf_step_kernel FWD(passive) + ADJ_REF",
                         "loop_ms": loop_ms, "peak_source": peak_kind},
            "e2e": e2e, "cpu_baseline": cpu, "clocks": clocks}), flush=True)


APS_STEPS = (2, 4)  # reference arm: two step counts per call, their difference excludes set-up


def _aps_ref_worker(n, kind):
    """The reference's aps3dc (oracle/_ref apscfun; kind "port": the FP64
    restatement) forward-modelling the benchmark model for APS_STEPS[0] and
    APS_STEPS[1] steps; returns the two walls."""
    sys.path.insert(0, ROOT)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    vel, pos, f, t = c2_model(n, 1234)
    t = np.zeros(3) + 0.001  # onsets inside the short runs
    walls = []
    for nt_s in APS_STEPS:
        if kind == "reference":
            sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
            import apscfun  # the reference's own extension module
            src = np.concatenate([pos[:, 0], pos[:, 1], pos[:, 2], f, t, np.ones(3)]).astype(
                np.float32)
            t0 = time.perf_counter()
            apscfun.aps3dc(vel.flatten(order="F"), src, 0, nt_s, n, n, n, 3, 0, 0, 0, 1, NBT, CT,
                           DT, 0.0, H, 0.0, H, 0.0, H)
        else:
            from oracle import oracle as O
            t0 = time.perf_counter()
            O.psm(vel, nt_s, DT, (H, H, H), NBT, CT,
                  src=dict(sx=pos[:, 0], sy=pos[:, 1], sz=pos[:, 2], f=f, t=t, A=np.ones(3)))
        walls.append(time.perf_counter() - t0)
    return walls[0], walls[1]


def _aps_cpu(n, workers):
    pts = (n + 2 * NBT) ** 3
    for kind in ("reference", "port"):
        try:
            res = pool_map(_aps_ref_worker, [(n, kind)] * workers, timeout_s=900)
            d = max(r[1] - r[0] for r in res)
            return pts * (APS_STEPS[1] - APS_STEPS[0]) * workers / d / 1e9, kind, d
        except Exception:  # noqa: BLE001
            continue
    raise RuntimeError("neither the reference nor the port ran")


def run_aps3d(args, world, rank, local):
    """3-D pseudo-spectral forward modelling (aps3d) of the headline's model
    (201^3 interior at 10 m, nbt 30: 261^3 expanded, 270^3 FFT grid, three
    seeded Ricker sources, surface traces), nt from --nt."""
    n, nt = args.n, args.nt
    pts = (n + 2 * NBT) ** 3
    nz2 = 2 * int(next_fast_size((n + 2 * NBT + 1) // 2))
    nx2 = int(next_fast_size(n + 2 * NBT))
    cfg = {"workload": f"aps3d pseudo-spectral forward {n}^3 h={H:g}m nt={nt} nbt={NBT} "
                       f"(FFT grid {nz2}x{nx2}x{nx2})", "expanded_points": pts}
    metric = "Gpt-updates/s (3-D pseudo-spectral, aps3d)"
    if args.impl == "reference":
        if rank != 0:
            return
        workers = max(1, min(os.cpu_count() or 1, 8))
        rates = []
        for i in range(args.warmup + args.steps):
            v, kind, _ = _aps_cpu(n, workers)
            if i >= args.warmup:
                rates.append(v)
        value = statistics.median(rates)
        print(json.dumps({
            "impl": "reference", "metric": metric, "value": value, "unit": "Gpt/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": cfg,
            "cpu_baseline": {"value": value, "unit": "Gpt/s", "cores": workers, "kind": kind,
                             "sample": f"aps3dc for {APS_STEPS[0]} and {APS_STEPS[1]} steps per "
                                       f"process (difference = steps alone), {workers} processes"},
            "e2e": {"value": value, "unit": "Gpt/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}), flush=True)
        return
    import torch
    import torch.distributed as dist
    from pywave_b200 import _lib as L
    from pywave_b200 import build as B
    import pywave_b200 as pw
    B.build()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    vel, pos, f, t = c2_model(n, 1234 + rank, nt)
    src = np.concatenate([pos[:, 0], pos[:, 1], pos[:, 2], f, t, np.ones(3)]).astype(np.float32)
    a = L.AfdArgs(dim=3, nz=n, nx=n, ny=n, nt=nt, nbt=NBT, ct=CT, dt=DT, dz=H, dx=H, dy=H, ns=3,
                  tri=0, jsnap=0, gz=0, flags=0)
    st = torch.cuda.current_stream().cuda_stream
    vel_d = torch.from_numpy(np.ascontiguousarray(vel.flatten(order="F"))).cuda()
    src_d = torch.from_numpy(src).cuda()
    dat = torch.empty(n * n * nt, device="cuda")
    lib = L.lib()

    def step():
        L.check(lib.pw_aps(a, vel_d.data_ptr(), src_d.data_ptr(), None, dat.data_ptr(), None, st))
        return L.last_timing()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clk = Clocks(local)
    clk.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches, loops = 0, []
    e0.record()
    for _ in range(args.steps):
        ms_, nst, tot = step()
        loops.append(ms_)
        launches += tot
    e1.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    loop_ms = statistics.median(loops)
    # algorithmic bytes per step: R2C reads the real grid and writes the
    # half spectrum, the multiply reads and writes it, C2R the reverse, the
    # update reads S, P, F, vv and writes S, P (each transform's own passes
    # not counted)
    nre = nz2 * nx2 * nx2
    ncx = (nz2 // 2 + 1) * nx2 * nx2
    alg_step = 4.0 * nre + 8.0 * ncx + 16.0 * ncx + 8.0 * ncx + 4.0 * nre + 24.0 * pts
    peak, peak_kind = peaks()
    e2e = None
    if not args.no_e2e:
        t0 = time.perf_counter()
        d, _ = pw.aps3d(vel, nt=nt, dt=DT, ax=[0, H, n], ay=[0, H, n], az=[0, H, n], ns=3,
                        sx=list(pos[:, 0]), sy=list(pos[:, 1]), sz=list(pos[:, 2]), f=list(f),
                        t=list(t), A=[1, 1, 1], nbt=NBT, ct=CT, jsnap=0, verb=False), None
        wall = time.perf_counter() - t0
        e2e = {"value": pts * nt / wall / 1e9, "unit": "Gpt/s",
               "h2d_bytes_per_step": int(vel.nbytes + src.nbytes),
               "d2h_bytes_per_step": int(4 * n * n * nt)}
    cpu = None
    if not args.no_cpu_baseline and rank == 0:
        v, kind, d = _aps_cpu(n, 1)
        cpu = {"value": v, "unit": "Gpt/s", "cores": 1, "kind": kind,
               "sample": f"aps3dc for {APS_STEPS[0]} and {APS_STEPS[1]} steps, one process "
                         f"(difference = {APS_STEPS[1] - APS_STEPS[0]} steps, {d:.1f} s)"}
    if rank == 0:
        print(json.dumps({
            "metric": metric, "value": job_rate(pts * nt, args.steps, world, ms) / 1e9,
            "unit": "Gpt/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (cuFFT)",
            "data": "synthetic (the headline's seeded velocity model and sources)",
            "config": cfg, "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": alg_step * nt / (loop_ms / 1e3) / 1e9,
                         "peak": peak, "unit": "GB/s",
                         "frac": alg_step * nt / (loop_ms / 1e3) / 1e9 / peak, "traffic": None,
                         "kernel": "cuFFT R2C + lapl multiply + cuFFT C2R + update per step",
                         "loop_ms": loop_ms, "peak_source": peak_kind},
            "e2e": e2e, "cpu_baseline": cpu, "clocks": clocks}), flush=True)


def next_fast_size(n):
    while True:
        m = n
        for p_ in (2, 3, 5):
            while m % p_ == 0:
                m //= p_
        if m <= 1:
            return n
        n += 1


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload == "fwi2d":
        return run_fwi2d(args, world, rank, local)
    if args.workload == "batch2d":
        return run_batch2d(args, world, rank, local)
    if args.workload == "c1":
        return run_c1(args, world, rank, local)
    if args.workload == "fwi3d":
        return run_fwi3d(args, world, rank, local)
    if args.workload == "lstri":
        return run_lstri(args, world, rank, local)
    if args.workload == "pfwic":
        return run_pfwic(args, world, rank, local)
    if args.workload == "aps3d":
        return run_aps3d(args, world, rank, local)
    if args.workload == "afd3d":
        return run_afd3d(args, world, rank, local)
    if args.impl == "reference":
        return run_reference(args, rank)

    import torch
    import torch.distributed as dist
    from pywave_b200 import _lib as L
    from pywave_b200 import build as B
    B.build()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    stream = torch.cuda.current_stream().cuda_stream
    n, nt, G = args.n, args.nt, args.groups
    vel, pos, f, t = c2_model(n, 1234 + rank, nt)
    vel_d, dat_d = gen_traces(vel, pos, f, t, nt, stream)
    groups = np.ascontiguousarray(np.tile(np.where(np.arange(n) // (n // G) < G,
                                                   np.arange(n) // (n // G), -1), (n, 1)).astype(np.int32))
    grp_d = torch.from_numpy(groups).cuda()
    img_d = torch.empty(n * n * n, device="cuda")
    a = L.AfdArgs(dim=3, nz=n, nx=n, ny=n, nt=nt, nbt=NBT, ct=CT, dt=DT, dz=H, dx=H, dy=H, ns=0,
                  tri=1, jsnap=4, gz=0, flags=0)
    lib = L.lib()

    def step_dev():
        L.check(lib.pw_tri_image(a, G, grp_d.data_ptr(), vel_d.data_ptr(), dat_d.data_ptr(),
                                 img_d.data_ptr(), 1, stream))

    for _ in range(args.warmup):
        step_dev()
    torch.cuda.synchronize()
    clk = Clocks(local)
    clk.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    loop_ms = []
    launches = 0
    e0.record()
    for _ in range(args.steps):
        step_dev()
        ms, nsteps, tot = L.last_timing()
        loop_ms.append(ms)
        launches += tot
    e1.record()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = clk.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    ms_step = ms / args.steps
    pts = (n + 2 * NBT) ** 3 * nt * G
    value = job_rate(pts, args.steps, world, ms) / 1e9

    # e2e: the same C-ABI call with pinned host buffers (copies inside the timed region)
    e2e = None
    if not args.no_e2e:
        vel_h = torch.from_numpy(np.ascontiguousarray(vel.flatten(order="F"))).pin_memory()
        dat_h = dat_d.cpu().pin_memory()
        img_h = torch.empty(n * n * n).pin_memory()
        ah = L.AfdArgs(dim=3, nz=n, nx=n, ny=n, nt=nt, nbt=NBT, ct=CT, dt=DT, dz=H, dx=H, dy=H,
                       ns=0, tri=1, jsnap=4, gz=0, flags=L.PW_HOST_PTRS)

        def step_host():
            L.check(lib.pw_tri_image(ah, G, groups.ctypes.data, vel_h.data_ptr(), dat_h.data_ptr(),
                                     img_h.data_ptr(), 1, stream))

        step_host()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        h0.record()
        for _ in range(args.steps):
            step_host()
        h1.record()
        torch.cuda.synchronize()
        ems = max_over_ranks(max(h0.elapsed_time(h1), (time.perf_counter() - t0) * 1e3), world)
        e2e = {"value": job_rate(pts, args.steps, world, ems) / 1e9, "unit": "Gpt/s",
               "h2d_bytes_per_step": int(vel.nbytes + dat_h.numel() * 4 + groups.nbytes),
               "d2h_bytes_per_step": int(img_h.numel() * 4)}

    # roofline of the dominant kernel (the fused lockstep step kernel)
    cells = (n + 2 * NBT) ** 3
    kern_ms = statistics.median(loop_ms) / nt
    alg_bytes = cells * (12 * G + 4) + cells * 8 / 4  # fields + vv per step, image RMW every 4th
    peak, peak_kind = peaks()
    achieved = alg_bytes / (kern_ms / 1e3) / 1e9
    # DRAM bytes of one step launch from an ncu capture of this workload
    # (profiles/traffic.json, a stored figure: not measured in this run)
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as fh:
            traffic = json.load(fh).get(f"tri3d_G{G}_n{n}")
    except (OSError, ValueError):
        pass

    # secondary field: the 2-D FWI gradient benchmark's batched / per-shot pair
    fwi2d = None
    if not args.no_fwi2d and n == 201 and nt == 1501:
        fwi2d = fwi2d_secondary(world, rank, stream)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        path = ref_inputs(n, 1234)
        try:
            v, kind, per_step, setup = reference_sample(n, path, 1)
            cpu = {"value": v, "unit": "Gpt/s", "cores": 1, "kind": kind,
                   "sample": f"afd3dc time reversal of the first receiver group on the "
                             f"{n + 2 * NBT}^3 expanded grid of the same velocity model, 1 core; "
                             f"calls of {REF_STEPS[0]} and {REF_STEPS[1]} steps, per-step time "
                             f"{per_step:.3f} s from their difference ({setup:.2f} s per-call "
                             f"set-up excluded)"}
        except Exception as ex:  # noqa: BLE001
            cpu = {"value": None, "unit": "Gpt/s", "cores": 1, "kind": "reference",
                   "sample": f"failed: {ex!r}"[:200]}
        finally:
            os.unlink(path)

    if rank == 0:
        line = {
            "metric": "Gpt-updates/s (3-D TRI, 4 lockstep groups)",
            "value": value, "unit": "Gpt/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded velocity, sources and traces)",
            "config": {"workload": f"3-D TRI image {n}^3 h=10m nt={nt} nbt={NBT} groups={G} "
                                   "jsnap=4",
                       "points_per_step": pts, "l2": "inputs larger than L2 (fields+traces "
                       f"{(cells * 4 * (2 * G + 2) + n * n * nt * 4) / 1e9:.2f} GB)",
                       "parallelism": f"replicas x{world} (one event per GPU)"},
            "e2e": e2e,
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "traffic_source": "stored ncu figure (profiles/traffic.json), "
                                           "not measured in this run",
                         "kernel": f"tile_kernel<TRI> x{G} groups + image_kernel every 4th step",
                         "kernel_ms": kern_ms, "alg_bytes_per_launch": alg_bytes,
                         "peak_source": peak_kind},
            "cpu_baseline": cpu,
            "clocks": clocks,
            "fwi2d": fwi2d,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
