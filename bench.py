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


def reference_sample(n, nt_s, seed, workers):
    """The reference's own afd3dc (compiled from its sources into oracle/_ref;
    the oracle port when that is absent), time-reversing one receiver group
    for nt_s steps on the full grid, in `workers` independent processes."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool:
        res = pool.starmap(_ref_worker, [(n, nt_s, seed + w) for w in range(workers)])
    wall = max(r[0] for r in res)
    kind = res[0][1]
    pts = (n + 2 * NBT) ** 3 * nt_s * workers
    return pts / wall / 1e9, kind, wall


def _ref_worker(n, nt_s, seed):
    sys.path.insert(0, ROOT)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    rng = np.random.default_rng(seed)
    vel = (2000 + 500 * rng.random((n, n, n))).astype(np.float32)
    dat = np.zeros((nt_s, n, n), np.float32)
    dat[:, : n // 4, :] = rng.standard_normal((nt_s, n // 4, n)).astype(np.float32) * 1e-3
    refdir = os.path.join(ROOT, "oracle", "_ref")
    try:
        sys.path.insert(0, refdir)
        import afdcfun  # the reference's own extension module
        kind = "reference"
        t0 = time.perf_counter()
        afdcfun.afd3dc(vel.flatten(order="F"), dat.flatten(order="F"), 1, nt_s, n, n, n, -1, 0, 4,
                       0, 1, NBT, CT, DT, 0.0, H, 0.0, H, 0.0, H)
        wall = time.perf_counter() - t0
    except ImportError:
        from oracle import oracle as O
        kind = "port"
        t0 = time.perf_counter()
        O.afd(vel, nt_s, DT, (H, H, H), nbt=NBT, ct=CT, tri=True, dat=dat, jsnap=4)
        wall = time.perf_counter() - t0
    return wall, kind


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
    nt_s = 4
    workers = max(1, min(os.cpu_count() or 1, 16))
    vals = []
    for i in range(args.warmup + args.steps):
        v, kind, wall = reference_sample(n, nt_s, 100 + i, workers)
        if i >= args.warmup:
            vals.append(v)
    value = statistics.median(vals)
    line = {
        "impl": "reference", "metric": "Gpt-updates/s (3-D TRI, 4 lockstep groups)",
        "value": value, "unit": "Gpt/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"3-D TRI image {n}^3 h=10m nt={args.nt} nbt={NBT} "
                               f"groups={args.groups}", "sample": f"{nt_s} steps x {workers} procs"},
        "cpu_baseline": {"value": value, "unit": "Gpt/s", "cores": workers, "kind": kind,
                         "sample": f"afd3dc time reversal of one group, {nt_s} of {args.nt} steps "
                                   f"on the {n + 2 * NBT}^3 expanded grid, {workers} independent "
                                   f"single-threaded processes"},
        "e2e": {"value": value, "unit": "Gpt/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
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
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as fh:
            traffic = json.load(fh).get(f"tri3d_G{G}_n{n}")
    except (OSError, ValueError):
        pass

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            workers = 1
            v, kind, wall = reference_sample(n, 16, 7, workers)
            cpu = {"value": v, "unit": "Gpt/s", "cores": workers, "kind": kind,
                   "sample": f"afd3dc time reversal of one group, 16 of {nt} steps on the "
                             f"{n + 2 * NBT}^3 expanded grid, 1 core ({wall:.1f} s)"}
        except Exception as ex:  # noqa: BLE001
            cpu = {"value": None, "unit": "Gpt/s", "cores": 1, "kind": "reference",
                   "sample": f"failed: {ex!r}"[:200]}

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
                         "kernel": f"tile_kernel<TRI> x{G} groups + image_kernel every 4th step", "kernel_ms": kern_ms,
                         "alg_bytes_per_launch": alg_bytes, "peak_source": peak_kind},
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
