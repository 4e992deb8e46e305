#!/usr/bin/env python
"""Benchmark: plane integrals/s of the grid-sampled 3D Radon transform at 128^3.

Workload (one "step"): the forward Radon transform of a 128^3 volume (sum of
16 seeded ellipsoids, seed 1001) on the Gauss-uniform sphere grid of 64
latitudes x 128 longitudes x 256 shifts = 2,097,152 plane integrals, each the
reference's lattice (step 1/n) restricted to [-n, n)^2 = 256 x 256 points with
the trilinear sampler (radon_grid/src/integral.c:26-58 with
cube_trilinear_interp).  Synthetic data, generated here.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  ``value`` is device-timed throughput with the
volume resident in HBM (CUDA events on the library's stream, L2 flushed before
every timed step); ``e2e`` is the same metric through the public API with the
FP64 host volume copied in from pinned memory and the FP64 results copied
back every step.  ``--impl reference`` times the reference's own C code
(oracle/_ref, compiled from the reference sources) on the host cores.
With N > 1 every rank runs the whole workload on its own GPU (independent
replicas, weak scaling); time is the maximum over ranks.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG_DIR = ROOT / "wrt-project_b200"

N, ELLIPSOIDS, SEED = 128, 16, 1001
NPHI, NTHETA, NSHIFT = 128, 64, 256
HALF_EXTENT = N  # lattice [-n, n)^2 -> 256 x 256 samples per plane
BYTES_PER_SAMPLE = 32  # eight FP32 voxel reads per trilinear sample
METRIC = "plane integrals/s @128^3 (64x128 sphere grid x 256 shifts, trilinear, 256^2 lattice)"
UNIT = "plane integrals/s"


def load_package():
    spec = importlib.util.spec_from_file_location(
        "wrt_b200", PKG_DIR / "__init__.py", submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["wrt_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


# ------------------------------------------------------------ distributed
class Dist:
    def __init__(self, gpus: int):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist

            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch

        t = torch.tensor([x], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples every 200 ms while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device, self.proc, self.lines = device, None, []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(self.device), "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------ CPU baselines
def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def plane_sample(count: int, seed: int):
    """A seeded random subset of the workload's planes (phi, theta, shift)."""
    sys.path.insert(0, str(ROOT))
    import oracle as O

    phi, theta, _, shift = O.radon_grid(NPHI, NTHETA, NSHIFT)
    rng = np.random.default_rng(seed)
    idx = rng.integers(0, NPHI * NTHETA * NSHIFT, size=count)
    it, ip, i_s = idx % NTHETA, (idx // NTHETA) % NPHI, idx // (NTHETA * NPHI)
    return phi[ip], theta[it], shift[i_s]


def time_reference_planes(vol, count, seed, threads):
    """The reference's plane_integral (nearest sampler, lattice [-2n,2n)^2, as
    shipped in radon_grid) over `count` sampled planes; returns planes/s."""
    sys.path.insert(0, str(ROOT))
    import oracle as O

    ref = O.Reference()
    p, t, s = plane_sample(count, seed)
    t0 = time.perf_counter()
    ref.plane_integrals(vol, p, t, s, nthreads=threads)
    return count / (time.perf_counter() - t0)


def cpu_baseline(vol, budget_s=12.0):
    threads = cpu_threads()
    sys.path.insert(0, str(ROOT))
    import oracle as O

    if not O.Reference.available():
        return {"value": None, "unit": UNIT, "cores": threads, "kind": "reference",
                "sample": "oracle/_ref not built"}
    # calibrate on a small sample, then size the measured sample to ~budget_s
    rate = time_reference_planes(vol, 256, 1, threads)
    count = int(max(512, min(200000, rate * budget_s)))
    rate = time_reference_planes(vol, count, 2, threads)
    # the FP64 restatement with the benchmark's own sampler and lattice
    p, t, s = plane_sample(max(256, count // 8), 3)
    t0 = time.perf_counter()
    O.radon_planes(vol, p, t, s, sampler=O.TRILINEAR, half_extent=HALF_EXTENT, nthreads=threads)
    port_rate = len(p) / (time.perf_counter() - t0)
    return {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"{count} seeded random planes of the 128^3 workload; the reference's "
                      f"radon_grid plane_integral as shipped (nearest sampler, 512^2 lattice, "
                      f"FP64), gcc -O2, OpenMP over planes",
            "port_trilinear": {"value": port_rate, "unit": UNIT, "kind": "port",
                               "sample": f"{len(p)} planes, the benchmark's own definition "
                                         f"(trilinear, 256^2 lattice), FP64 oracle restatement"}}


def run_reference(args, dist):
    if dist.rank != 0:
        return 0
    sys.path.insert(0, str(PKG_DIR))
    from phantom import ellipsoid_phantom
    sys.path.insert(0, str(ROOT))
    import oracle as O

    threads = cpu_threads()
    if not O.Reference.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built "
                          "(reference sources were not present at build time)"}))
        return 0
    vol = ellipsoid_phantom(N, ELLIPSOIDS, SEED)
    per_step = int(os.environ.get("WRT_REF_PLANES_PER_STEP", "2048"))
    for w in range(args.warmup):
        time_reference_planes(vol, per_step, 100 + w, threads)
    t_total = 0.0
    for k in range(args.steps):
        t0 = time.perf_counter()
        time_reference_planes(vol, per_step, 1000 + k, threads)
        t_total += time.perf_counter() - t0
    value = per_step * args.steps / t_total
    ms_per_step = 1e3 * t_total / args.steps
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "radon_grid 128^3, 64x128x256 planes", "n": N,
                   "sphere_grid": [NTHETA, NPHI], "shifts": NSHIFT,
                   "per_step": f"{per_step} seeded random planes of the workload"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"{per_step} planes per step; radon_grid plane_integral as "
                                   f"shipped (nearest sampler, 512^2 lattice), FP64"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------ our arm
def traffic_from_profiles():
    """DRAM bytes per launch of the plane kernel from the committed ncu summary."""
    f = ROOT / "profiles" / "plane_staged_kernel_128cubed.md"
    if not f.exists():
        return None
    for ln in f.read_text().splitlines():
        if ln.strip().startswith("dram_bytes_per_launch:"):
            try:
                return float(ln.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def served_stream(wrt, srv, pin_vol, pin_outs, steps):
    """K requests of the workload through the serving loop, each with its FP32
    volume in pinned host memory and its FP64 result copied back to pinned
    host memory.  Returns (wall seconds, infos)."""
    t0 = time.perf_counter()
    ids = [srv.submit_forward(pin_vol, NPHI, NTHETA, NSHIFT, pin_outs[k % len(pin_outs)],
                              half_extent=HALF_EXTENT, tag=k) for k in range(steps)]
    infos = [srv.wait(i) for i in ids]
    return time.perf_counter() - t0, infos


def serving_mix(wrt, dev, count, seed, budget):
    """A Poisson stream of mixed requests (the serving configuration, scaled to
    `count` requests): edge 64/96/128/192/256 w.p. .30/.25/.20/.15/.10,
    forward (80 %) or adjoint (20 %), sphere grids 32x64 .. 96x192 (latitudes
    x longitudes), 128-384 shifts, FP32 volumes of seeded ellipsoids, seeded
    Gaussian Radon data for the adjoints.  Arrival rate: ~90 % of the measured
    service rate of a first batch."""
    from wrt_b200.phantom import ellipsoid_phantom

    rng = np.random.default_rng(seed)
    edges = rng.choice([64, 96, 128, 192, 256], size=count, p=[0.30, 0.25, 0.20, 0.15, 0.10])
    vol_cache = {}
    reqs = []
    for k in range(count):
        n = int(edges[k])
        nth = int(rng.integers(32, 97))
        ns = int(rng.integers(128, 385))
        if rng.random() < 0.8:
            if n not in vol_cache:
                vol_cache[n] = ellipsoid_phantom(n, 12, seed + n).astype(np.float32)
            reqs.append(("fwd", n, nth, ns))
        else:
            reqs.append(("adj", n, nth, ns))
    adj_data = {}
    with wrt.Server(dev, budget_bytes=budget, max_batch=16, max_inflight=2) as srv:
        def submit(r):
            op, n, nth, ns = r
            if op == "fwd":
                out = np.empty((ns, 2 * nth, nth))
                return srv.submit_forward(vol_cache[n], 2 * nth, nth, ns, out, half_extent=n), out
            key = (nth, ns)
            if key not in adj_data:
                adj_data[key] = rng.standard_normal((ns, 2 * nth, nth))
            out = np.empty((n, n, n))
            return srv.submit_adjoint(adj_data[key], n, out), out
        # service-rate estimate from the first few requests run back to back
        t0 = time.perf_counter()
        warm = [submit(r) for r in reqs[:8]]
        for rid, _ in warm:
            srv.wait(rid)
        rate = 8 / (time.perf_counter() - t0) * 0.9
        gaps = rng.exponential(1.0 / rate, size=count)
        t_start = time.perf_counter()
        pending, t_next = [], t_start
        for k, r in enumerate(reqs):
            t_next += gaps[k]
            delay = t_next - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            pending.append((r, submit(r)))
        infos = [(r, srv.wait(rid)) for r, (rid, _) in pending]
        wall = time.perf_counter() - t_start
        st = srv.stats()
    lat = np.array([i.done_ms - i.submit_ms for _, i in infos])
    planes = sum(r[3] * 2 * r[2] * r[2] for r, _ in infos if r[0] == "fwd")
    return {"requests": count, "forward": sum(r[0] == "fwd" for r in reqs),
            "arrival_rate_per_s": rate, "wall_s": wall,
            "requests_per_s": count / wall, "plane_integrals_per_s": planes / wall,
            "latency_ms": {"p50": float(np.percentile(lat, 50)),
                           "p99": float(np.percentile(lat, 99))},
            "launches": int(st.launches), "hbm_peak_bytes": int(st.bytes_peak),
            "budget_bytes": int(st.budget),
            "mean_batch": float(np.mean([i.batch_size for _, i in infos]))}


def run_ours(args, dist):
    wrt = load_package()
    from wrt_b200.phantom import ellipsoid_phantom

    dev = dist.local_rank
    ctx = wrt.Context(dev)
    phantom = ellipsoid_phantom(N, ELLIPSOIDS, SEED)
    vol = wrt.Volume(ctx, N)
    vol.upload(phantom.astype(np.float32))
    grid = wrt.Grid(ctx, NPHI, NTHETA, NSHIFT)
    nplanes = grid.nplanes
    out = wrt.DeviceBuffer(ctx, nplanes * 8)
    kernel = {"plain": wrt.KERNEL_PLAIN, "staged": wrt.KERNEL_STAGED, "auto": wrt.KERNEL_AUTO}[args.kernel]

    def step(k=kernel):
        if k == wrt.KERNEL_PLAIN:
            wrt.radon_forward_device(ctx, vol, grid, out.ptr, sampler=wrt.TRILINEAR,
                                     half_extent=HALF_EXTENT, kernel=k)
        else:  # the batched persistent kernel through its captured graph
            wrt.radon_forward_batch(ctx, [(vol, grid, out.ptr, HALF_EXTENT)])

    # the autotuner picks the staged kernel's tile shape on this request
    tile = None
    if kernel != wrt.KERNEL_PLAIN:
        if args.tile is not None:
            best, best_ms = args.tile, None
            wrt.set_plane_kernel_config(ctx, best)
        else:
            best, best_ms = wrt.tune_plane_kernel(ctx, vol, grid, out.ptr, sampler=wrt.TRILINEAR,
                                                  half_extent=HALF_EXTENT)
        t, g, s = wrt.plane_kernel_configs()[best]
        tile = {"threads": t, "rows_per_warp_group": g, "shifts_per_lane": s,
                "tuner_ms": best_ms}

    # samples evaluated per launch (one counted launch, outside the timed region)
    ctx.count_samples(True)
    step()
    samples = ctx.sample_count()
    ctx.count_samples(False)

    for _ in range(max(args.warmup, 3)):
        step()
    ctx.synchronize()

    clocks = ClockSampler(dev)
    clocks.start()
    dist.barrier()
    ctx.synchronize()
    launches0 = ctx.launches
    times = []
    for _ in range(args.steps):
        ctx.flush_l2()
        ctx.timer_start()
        step()
        times.append(ctx.timer_stop())
    launches = ctx.launches - launches0
    ctx.synchronize()
    dist.barrier()
    clk = clocks.stop()
    total_ms = dist.max(sum(times))
    ms_per_step = total_ms / args.steps
    value = nplanes * args.steps * dist.world / (total_ms * 1e-3)
    result_dev = out.download(np.empty((NSHIFT, NPHI, NTHETA)))

    if args.only_kernel:  # profiling captures: the timed kernel launches and nothing else
        if dist.rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT,
                              "ms_per_step": ms_per_step, "samples_per_step": samples,
                              "tile": tile, "note": "kernel only (profiling run)"}))
        out.close(); vol.close(); grid.close(); ctx.close()
        return 0

    # plain kernel alongside (the one-request-per-launch baseline)
    plain = None
    if kernel != wrt.KERNEL_PLAIN:
        step(wrt.KERNEL_PLAIN)
        pt = []
        for _ in range(max(2, min(args.steps, 5))):
            ctx.flush_l2()
            ctx.timer_start()
            step(wrt.KERNEL_PLAIN)
            pt.append(ctx.timer_stop())
        plain_res = out.download(np.empty((NSHIFT, NPHI, NTHETA)))
        plain = {"value": nplanes / (statistics.mean(pt) * 1e-3), "unit": UNIT,
                 "ms_per_step": statistics.mean(pt),
                 "rel_l2_vs_staged": float(np.linalg.norm(plain_res - result_dev) /
                                           np.linalg.norm(result_dev))}

    # end to end through the serving loop (the public API a caller uses): each
    # step is one request of the workload, its FP32 volume copied in from pinned
    # host memory and its FP64 plane integrals copied back to pinned host memory
    pin_vol = wrt.PinnedArray(ctx, (N, N, N), np.float32)
    pin_vol.array[...] = phantom
    pin_outs = [wrt.PinnedArray(ctx, (NSHIFT, NPHI, NTHETA), np.float64) for _ in range(4)]
    srv = wrt.Server(dev, budget_bytes=4 << 30, max_batch=8, max_inflight=2)
    served_stream(wrt, srv, pin_vol.array, [p.array for p in pin_outs], 3)  # warm-up
    dist.barrier()
    wall, infos = served_stream(wrt, srv, pin_vol.array, [p.array for p in pin_outs], args.steps)
    served_res = np.array(pin_outs[(args.steps - 1) % len(pin_outs)].array)
    srv.close()
    wall = dist.max(wall)
    e2e_value = nplanes * args.steps * dist.world / wall
    lat = np.array([i.done_ms - i.submit_ms for i in infos])
    served_equal = bool(np.array_equal(served_res, result_dev))

    # roofline of the plane kernel: 32 B of staged voxel reads per sample
    # against the measured shared-memory bandwidth of this device
    smem_bw = ctx.smem_bandwidth()
    per_launch_s = ms_per_step * 1e-3
    achieved = samples * BYTES_PER_SAMPLE / per_launch_s / 1e9
    peak = smem_bw / 1e9
    hbm_bytes = N ** 3 * 4 + nplanes * 8  # compulsory: FP32 volume in, FP64 results out
    peaks_file = ROOT / "MEASURED_PEAKS.json"
    hbm_peak = json.loads(peaks_file.read_text()).get("hbm_gbs") if peaks_file.exists() else 6650.0

    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world,
        "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "radon_grid forward, 128^3 volume of 16 seeded ellipsoids, "
                               "64x128 Gauss-uniform sphere grid x 256 shifts, trilinear, "
                               "lattice step 1/n on [-n,n)^2",
                   "n": N, "sphere_grid": [NTHETA, NPHI], "shifts": NSHIFT,
                   "planes_per_step": nplanes, "kernel": args.kernel, "tile": tile,
                   "path": "batched persistent kernel, graph launch (wrt_radon_forward_batch)",
                   "l2": "flushed before every timed step (2x L2 memset)",
                   "parallelism": f"replicas x{dist.world}"},
        "samples_per_step": samples,
        "samples_per_s": samples * args.steps * dist.world / (total_ms * 1e-3),
        "gpu_launches": launches,
        "roofline": {"bound": "l1tex", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak if peak else None, "traffic": traffic_from_profiles(),
                     "peak_source": "shared-memory read bandwidth measured in this run "
                                    "(wrt_measure_smem_bandwidth); 32 B per trilinear sample",
                     "hbm": {"achieved": hbm_bytes / per_launch_s / 1e9, "peak": hbm_peak,
                             "unit": "GB/s", "frac": hbm_bytes / per_launch_s / 1e9 / hbm_peak,
                             "note": "compulsory bytes only; the volume is re-read from L2"}},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": N ** 3 * 4,
                "d2h_bytes_per_step": nplanes * 8,
                "path": "wrt_server: one request per step, pinned FP32 volume in, pinned FP64 "
                        "results out, 2 launches in flight",
                "latency_ms": {"p50": float(np.percentile(lat, 50)),
                               "p99": float(np.percentile(lat, 99))},
                "result_bitwise_equal_to_kernel_path": served_equal},
        "clocks": clk,
    }
    if plain:
        result["plain"] = plain
        result["served_over_plain"] = e2e_value / plain["value"]
    if dist.rank == 0 and dist.world == 1 and not args.no_serving_mix:
        result["serving"] = serving_mix(wrt, dev, args.mix_requests, 4000, 60 << 30)
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_baseline(phantom)
    if dist.rank == 0:
        print(json.dumps(result))
    pin_vol.close()
    for p in pin_outs:
        p.close()
    out.close()
    vol.close()
    grid.close()
    ctx.close()
    return 0


# ------------------------------------------------------------ other paths
PATHS = {
    # path: (metric, unit, workload)
    "ray": ("rays/s @128^3 (128 layers x 128 shifts x 128 angles, reference frame)", "rays/s",
            "ray_grid, 128^3 volume of 16 seeded ellipsoids, 128 z-layers x 128 shifts x 128 "
            "angles, trilinear, 513 samples per ray (255 inside the unit ball)"),
    "ray_rotated": ("rays/s @128^3 (128 layers x 128 shifts x 128 angles, rotated frame)",
                    "rays/s",
                    "ray_grid in one seeded random rotation of the layer frame (one of the "
                    "configuration's orientations), 128^3 volume, 128 layers x 128 shifts x 128 "
                    "angles, trilinear"),
    "reduction": ("plane integrals/s from 128^3 ray data (64x128 sphere grid x 256 shifts)",
                  "plane integrals/s",
                  "radon_reduction, rays 128 layers x 128 shifts x 128 angles -> 64x128 sphere "
                  "grid x 256 shifts (ray shift grid decoupled: spline over 128 offsets)"),
    "adjoint": ("voxels/s of the backprojection to 128^3 (64x128 sphere grid x 256 shifts)",
                "voxels/s",
                "radon3d_adjoint, seeded N(0,1) Radon data 64x128 sphere grid x 256 shifts -> "
                "128^3 voxels, 8192 spline evaluations per voxel"),
}


def run_path(args, dist):
    """One of the other hot paths through its drop-in entry point (host arrays
    in and out, as the reference's programs take them): K timed calls after W
    warm-up calls, CUDA events on the library's stream around each call (the
    calls are synchronous, so this is end to end), the reference's own code on
    a bounded sample of the same workload on the host cores beside it."""
    wrt = load_package()
    from wrt_b200.phantom import ellipsoid_phantom

    sys.path.insert(0, str(ROOT))
    import oracle as O

    metric, unit, workload = PATHS[args.path]
    ctx = wrt.Context(dist.local_rank)
    n = N
    rng = np.random.default_rng(SEED)
    vol = ellipsoid_phantom(n, ELLIPSOIDS, SEED)
    frame = None
    if args.path == "ray_rotated":
        q, r = np.linalg.qr(rng.standard_normal((3, 3)))
        frame = q * np.sign(np.diag(r))
        if np.linalg.det(frame) < 0:
            frame[:, 0] = -frame[:, 0]
    if args.path in ("ray", "ray_rotated"):
        call = lambda: ctx.ray_grid(vol, n, 128, 128, frame=frame)
        units, h2d, d2h = n * 128 * 128, vol.nbytes, n * 128 * 128 * 8
    elif args.path == "reduction":
        rays = ctx.ray_grid(vol, n, 128, 128)
        call = lambda: ctx.radon_reduction(rays, NSHIFT, NTHETA)
        units, h2d, d2h = NSHIFT * NPHI * NTHETA, rays.nbytes, NSHIFT * NPHI * NTHETA * 8
    else:
        radon = rng.standard_normal((NSHIFT, NPHI, NTHETA))
        call = lambda: ctx.radon3d_adjoint(radon, n)
        units, h2d, d2h = n ** 3, radon.nbytes, n ** 3 * 8
    for _ in range(max(args.warmup, 3)):
        result = call()
    ctx.synchronize()
    clocks = ClockSampler(dist.local_rank)
    clocks.start()
    dist.barrier()
    times = []
    for _ in range(args.steps):
        ctx.timer_start()
        result = call()
        times.append(ctx.timer_stop())
    dist.barrier()
    clk = clocks.stop()
    total_ms = dist.max(sum(times))
    value = units * args.steps * dist.world / (total_ms * 1e-3)

    # the reference on the host cores: a bounded seeded sample of the same units
    cpu = None
    if dist.rank == 0 and not args.no_cpu_baseline and O.Reference.available():
        ref, cores = O.Reference(), cpu_threads()
        t0 = time.perf_counter()
        if args.path == "ray":
            m = 65536
            idx = rng.integers(0, units, size=m)
            s_grid, phi_grid = O.ray_grid(128, 128)
            z = -1.0 + (idx // (128 * 128)) * (2.0 / (n - 1))
            got = ref.rays(vol, z, s_grid[(idx // 128) % 128], phi_grid[idx % 128], cores)
            ours = result.reshape(-1)[idx]
        elif args.path == "ray_rotated":
            # the reference has no layer frames: the FP64 restatement, all rays
            m = units
            got = O.ray_forward(vol, n, 128, 128, frame=frame, nthreads=cores).reshape(-1)
            ours = result.reshape(-1)
        elif args.path == "reduction":
            m = 4096
            idx = rng.integers(0, units, size=m)
            # the reference couples the ray and Radon shift grids: rays on 256 shifts
            rays_c = ctx.ray_grid(vol, n, NSHIFT, 128)
            t0 = time.perf_counter()
            got = ref.reduction_planes(rays_c, NTHETA, idx // (NPHI * NTHETA),
                                       (idx // NTHETA) % NPHI, idx % NTHETA, cores)
            ours = None
        else:
            m = 64
            idx = rng.integers(0, units, size=m)
            iz, ix, iy = idx // (n * n), (idx // n) % n, idx % n
            c = lambda i: -1.0 + (2.0 * i + 1.0) / n
            got = ref.adjoint_points(radon, c(ix), c(iy), c(iz), cores)
            ours = result.reshape(-1)[idx]
        wall = time.perf_counter() - t0
        cpu = {"value": m / wall, "unit": unit, "cores": cores, "kind": "reference",
               "sample": f"{m} seeded random units of this workload, the reference's own code "
                         "(oracle/_ref) with OpenMP over units"}
        if args.path == "ray_rotated":
            cpu.update(kind="port", sample=f"all {m} rays, the FP64 oracle restatement with the "
                                           "frame (the reference has no layer frames)")
        if ours is not None:
            cpu["rel_l2_gpu_vs_reference_on_sample"] = float(
                np.linalg.norm(ours - got) / max(np.linalg.norm(got), 1e-300))
    if dist.rank == 0:
        print(json.dumps({
            "metric": metric, "value": value, "unit": unit, "n_gpus": dist.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "ms_per_step_median": statistics.median(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "path": args.path,
            "config": {"workload": workload, "api": "drop-in entry point, host arrays"},
            "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "clocks": clk, "cpu_baseline": cpu}))
    ctx.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--kernel", choices=["auto", "plain", "staged"], default="auto")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving-mix", action="store_true")
    ap.add_argument("--only-kernel", action="store_true",
                    help="time the kernel steps only (for profiling captures)")
    ap.add_argument("--mix-requests", type=int, default=96,
                    help="requests in the mixed serving stream")
    ap.add_argument("--tile", type=int, default=None,
                    help="use this tile configuration of the staged kernel instead of tuning")
    ap.add_argument("--path", choices=["forward", *PATHS], default="forward",
                    help="forward: the headline (plane integrals at 128^3); ray, reduction, "
                         "adjoint: the other hot paths through their drop-in entry points")
    ap.add_argument("--grid", default=None,
                    help="NPHI,NTHETA,NSHIFT: a smaller sphere grid (profiling captures only)")
    args = ap.parse_args()
    if args.grid:
        global NPHI, NTHETA, NSHIFT
        NPHI, NTHETA, NSHIFT = (int(x) for x in args.grid.split(","))
    dist = Dist(args.gpus)
    try:
        if args.path != "forward":
            rc = run_path(args, dist) if args.impl == "ours" else 0
        else:
            rc = run_reference(args, dist) if args.impl == "reference" else run_ours(args, dist)
    finally:
        dist.close()
    return rc


if __name__ == "__main__":
    sys.exit(main())
