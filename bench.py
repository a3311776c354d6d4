#!/usr/bin/env python
"""Benchmark of the mesh signed-distance query path (one JSON line on rank 0).

Workload (default): the level-8 displaced icosphere (1,310,720 triangles, Morton-built 4-wide BVH)
queried on the 512^3 cell-centre grid over [-1.25,1.25]^3 (134,217,728 points) plus 16,777,216
points within +-1e-3 of the surface: 150,994,944 queries per step, FP32 traversal with the FP64
near-surface band.  A step is one pass of the query path over all of them.  Inputs are seeded
synthetic data of that shape (no dataset).

  python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

--impl ours (default): device-resident timing (``value``, CUDA events around K steps, max over
ranks), end-to-end timing through the host entry point with pinned buffers (``e2e``), the roofline
of the traversal kernel from per-phase CUDA events recorded on the launching stream during the timed
steps, nvidia-smi clock samples during the timed region, and (rank 0, N=1) the reference CPU
implementation timed on a bounded sample of the same points (``cpu_baseline``).
--impl reference: the reference's own CPU implementation (compiled from its headers into
oracle/_ref) on all host threads, each step a bounded sample of the same workload.
Multi-GPU (torchrun): each rank runs the full workload on its own GPU (weak scaling, replicas with
no data-path collective).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from ebgeometry_b200.ranks import max_over_ranks  # noqa: E402  (pure Python, no library load)

METRIC = "SDF queries/s on 1 B200: learned-seeded vs plain GPU BVH at equal accuracy"
UNIT = "queries/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["mesh", "knn", "grid", "csg"], default="mesh",
                    help="mesh: the headline mesh-SDF configuration; knn: 16M-point cloud, 4M queries, k=1 and 8; "
                         "grid: the uniform-grid cloud against the BVH cloud on a uniform and a clustered 16M-point "
                         "cloud; csg: 4,096 spheres + 256 posed meshes, 2,048 query batches in one launch")
    ap.add_argument("--knn-points", type=int, default=16 * 1024 * 1024)
    ap.add_argument("--knn-queries", type=int, default=4 * 1024 * 1024)
    ap.add_argument("--csg-batches", type=int, default=2048)
    ap.add_argument("--csg-meshes", type=int, default=256)
    ap.add_argument("--csg-spheres", type=int, default=4096)
    ap.add_argument("--level", type=int, default=8)
    ap.add_argument("--grid", type=int, default=512)
    ap.add_argument("--band-points", type=int, default=16 * 1024 * 1024)
    ap.add_argument("--build", default="Morton")
    ap.add_argument("--leaf", type=int, default=8)
    ap.add_argument("--host-build", action="store_true",
                    help="build the tree on the host (default: on the GPU, for Morton and SAH builds alike)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU work of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--no-seed", action="store_true", help="time the plain traversal only")
    ap.add_argument("--perfect-seed", action="store_true",
                    help="also time the traversal seeded with the exact distances (the bound any seed can reach)")
    ap.add_argument("--hint-slack", default="0.02:4e-4,0.005:1e-4",
                    help="with --perfect-seed: also time radius hints |d|(1+a)+b for these a:b pairs")
    ap.add_argument("--seed-samples", type=int, default=1 << 25)
    ap.add_argument("--seed-steps", type=int, default=2000)
    ap.add_argument("--seed-batch", type=int, default=1 << 18)
    ap.add_argument("--seed-save", default=None, help="write the trained model to this path")
    ap.add_argument("--seed-load", default=None, help="load a trained model instead of training one")
    return ap.parse_args()


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def workload(args):
    from ebgeometry_b200 import workloads as W
    v, f = W.displaced_icosphere(args.level, 1)
    grid = W.grid_points(args.grid, -1.25, 1.25)
    band = W.band_points(v, f, args.band_points, 2, 1e-3)
    pts = np.concatenate([grid, band])
    return v, f, pts


def sample_indices(n_grid, n_band, n, seed=17):
    """Seeded stratified sample of the workload: grid and band points in their workload proportion."""
    rng = np.random.default_rng(seed)
    ng = int(round(n * n_grid / (n_grid + n_band)))
    gi = rng.choice(n_grid, size=min(ng, n_grid), replace=False)
    bi = n_grid + rng.choice(n_band, size=min(n - ng, n_band), replace=False)
    return np.sort(np.concatenate([gi, bi]))


# --- reference CPU implementation -----------------------------------------------------------------
def reference_mesh(v, f):
    import oracle
    R = oracle.ref()
    t0 = time.time()
    m = R.mesh(v, f, kind=0, build=1, max_leaf_groups=4)  # TriMeshSDF<double,short,4,4>, Morton
    return R, m, time.time() - t0


def time_reference(m, pts, threads=0):
    p = pts.astype(np.float64)
    t0 = time.perf_counter()
    m.sdf(p, threads=threads)
    return time.perf_counter() - t0


def calibrated_sample(m, pts, n_grid, n_band, target_s):
    """Sizes a stratified sample so the reference spends about target_s seconds on it."""
    n0 = 16384
    idx = sample_indices(n_grid, n_band, n0, seed=5)
    dt = time_reference(m, pts[idx])
    qps = n0 / max(dt, 1e-6)
    n = int(min(max(qps * target_s, 16384), 8_000_000))
    return sample_indices(n_grid, n_band, n), qps


def cpu_info():
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return model


# --- clocks sampler -------------------------------------------------------------------------------
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def l2_read_bandwidth():
    """Read bandwidth of a 48 MB L2-resident buffer streamed by the library's own kernel."""
    import ctypes as C

    from ebgeometry_b200 import _capi
    out = C.c_double()
    _capi.check(_capi.lib.ebg_measure_read_bandwidth(48 << 20, 20, C.byref(out)))
    return out.value


# --- arms -------------------------------------------------------------------------------------------
def run_reference(args, rank, world):
    if rank != 0:
        return 0
    import oracle
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference oracle library not built (oracle/_ref)"}))
        return 0
    v, f, pts = workload(args)
    n_grid, n_band = args.grid ** 3, args.band_points
    R, m, tbuild = reference_mesh(v, f)
    # each step: a fresh stratified sample sized for ~4 s of CPU work
    _, qps0 = calibrated_sample(m, pts, n_grid, n_band, 1.0)
    n = int(min(max(qps0 * 4.0, 16384), 4_000_000))
    for s in range(args.warmup):
        time_reference(m, pts[sample_indices(n_grid, n_band, n, seed=100 + s)])
    times = []
    for s in range(args.steps):
        times.append(time_reference(m, pts[sample_indices(n_grid, n_band, n, seed=200 + s)]))
    tot = sum(times)
    qps = n * args.steps / tot
    cores = R.max_threads()
    sample = (f"{n} points per step: a seeded stratified sample of the {n_grid + n_band} workload points "
              f"({n_grid} grid + {n_band} band in proportion)")
    line = {"impl": "reference", "metric": METRIC, "value": qps, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"mesh SDF, displaced icosphere level {args.level} ({f.shape[0]} triangles), "
                                   f"{args.grid}^3 grid + {n_band} band points",
                       "implementation": "reference TriMeshSDF<double,short,4,4> (Morton build), value() per "
                                         "point in an OpenMP parallel-for", "build_s": tbuild,
                       "cpu": cpu_info()},
            "cpu_baseline": {"value": qps, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
            "e2e": {"value": qps, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def timed_steps(mesh, pd, out, steps, seed, dev, world, stream, _capi, torch, dist, local_rank, hint=None):
    """K steps bracketed by barrier + synchronize, CUDA events on the launching stream, clocks
    sampled meanwhile; per-phase events recorded inside each call.  Returns (ms/step max over
    ranks, phase array, clocks)."""
    clocks = Clocks(local_rank)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    tms = []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        tm = _capi.PhaseTimings()
        mesh.signed_distance(pd, out=out, timings=tm, seed=seed, radius_hint=hint)
        tms.append((tm.order_ms, tm.traverse_ms, tm.band_ms, tm.total_ms))
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ck = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), dev)
    mesh.check_status()
    return ms / steps, np.array(tms), ck


def run_ours(args, rank, world, local_rank):
    import ctypes as C

    import torch
    import torch.distributed as dist

    from ebgeometry_b200 import SeedModel, TriMeshSDF, _capi

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    v, f, pts = workload(args)
    n = pts.shape[0]
    n_grid, n_band = args.grid ** 3, args.band_points
    t0 = time.time()
    on_device = not args.host_build
    mesh = TriMeshSDF(v, f, build=args.build, leaf_size=args.leaf, device=local_rank, on_device=on_device)
    t_build = time.time() - t0
    log(f"[rank {rank}] mesh {f.shape[0]} tris built in {t_build:.2f}s: {mesh.info}")

    pd = torch.from_numpy(pts).to(dev)
    out = torch.empty(n, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    tsteps = (mesh, pd, out, args.steps)
    tctx = (dev, world, stream, _capi, torch, dist, local_rank)

    # plain traversal: counters (untimed; the roofline's per-query work unit), warm-up, timed steps
    _, st = mesh.stats(pd)
    log(f"[rank {rank}] plain stats {st}")
    for _ in range(args.warmup):
        mesh.signed_distance(pd, out=out)
    torch.cuda.synchronize(dev)
    ms_plain, tms_plain, ck_plain = timed_steps(*tsteps, None, *tctx)
    plain_ref = out.clone() if not args.no_seed else None
    log(f"[rank {rank}] plain {ms_plain:.1f} ms/step")

    # what ANY pruning-radius seed could save at best: the exact |d| (from the plain run) as radius
    perfect = None
    if args.perfect_seed:
        hint = out.abs() * (1 + 1e-5) + 1e-6
        _, st_hint = mesh.stats(pd, radius_hint=hint)
        hout = torch.empty_like(out)
        for _ in range(2):
            mesh.signed_distance(pd, out=hout, radius_hint=hint)
        ms_hint, _, _ = timed_steps(mesh, pd, hout, max(2, args.steps // 2), None, *tctx, hint=hint)
        perfect = {"ms_per_step": ms_hint, "value": n * world / (ms_hint * 1e-3),
                   "speedup_vs_plain": ms_plain / ms_hint, "stats": st_hint,
                   "equal_to_plain_fraction": float((hout == out).float().mean().item())}
        log(f"[rank {rank}] perfect radius {ms_hint:.1f} ms/step {st_hint}")
        # radius slack a seed would carry: |d| (1 + a) + b
        slack = []
        for pair in filter(None, args.hint_slack.split(",")):
            sa, sb = (float(x) for x in pair.split(":"))
            hint = out.abs() * (1 + sa) + sb
            _, st_s = mesh.stats(pd, radius_hint=hint)
            mesh.signed_distance(pd, out=hout, radius_hint=hint)
            ms_s, _, _ = timed_steps(mesh, pd, hout, max(2, args.steps // 2), None, *tctx, hint=hint)
            slack.append({"a": sa, "b": sb, "ms_per_step": ms_s, "speedup_vs_plain": ms_plain / ms_s,
                          "nodes_per_query": st_s["nodes_visited"] / n, "leaves_per_query": st_s["leaves_visited"] / n,
                          "triangles_per_query": st_s["triangles_tested"] / n})
            log(f"[rank {rank}] radius |d|(1+{sa})+{sb}: {ms_s:.1f} ms/step")
        perfect["slack"] = slack
        del hout, hint

    seed, rep, st_seed = None, None, None
    if not args.no_seed:
        t0 = time.time()
        if args.seed_load:
            seed = SeedModel.load(args.seed_load, device=local_rank)
        else:
            seed = SeedModel.train(mesh, num_samples=args.seed_samples, steps=args.seed_steps,
                                   batch=args.seed_batch, rng_seed=7, lo=[-1.25] * 3, hi=[1.25] * 3)
        rep = seed.report()
        rep["wall_s"] = time.time() - t0
        rep["loaded_from"] = args.seed_load
        if args.seed_save:
            seed.save(args.seed_save)
        log(f"[rank {rank}] seed trained: {rep}")
        _, st_seed = mesh.stats(pd, seed=seed)
        log(f"[rank {rank}] seeded stats {st_seed}")
        for _ in range(args.warmup):
            mesh.signed_distance(pd, out=out, seed=seed)
        torch.cuda.synchronize(dev)
        ms_seed, tms_seed, ck_seed = timed_steps(*tsteps, seed, *tctx)
        log(f"[rank {rank}] seeded {ms_seed:.1f} ms/step")
        diff = (out - plain_ref).abs()
        same_frac = float((out == plain_ref).float().mean().item())
        max_diff = float(diff.max().item())
    ms_step, tms, ck = (ms_seed, tms_seed, ck_seed) if seed is not None else (ms_plain, tms_plain, ck_plain)
    value = n * world / (ms_step * 1e-3)
    plain_value = n * world / (ms_plain * 1e-3)

    # end to end through the host entry point: pinned input, H2D + query + D2H every step
    e2e_steps = args.e2e_steps or max(2, min(args.steps, 3))
    ph = torch.from_numpy(pts).pin_memory()
    oh = torch.empty(n, dtype=torch.float32).pin_memory()
    opts = _capi.QueryOpts()
    if seed is not None:
        opts.seed = seed.handle

    def host_call():
        _capi.check(_capi.lib.ebg_mesh_signed_distance_host(
            mesh.handle, C.c_void_p(ph.data_ptr()), n, C.c_void_p(oh.data_ptr()), None, C.byref(opts),
            C.c_void_p(stream.cuda_stream)))

    host_call()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h0.record(stream)
    for _ in range(e2e_steps):
        host_call()
    h1.record(stream)
    torch.cuda.synchronize(dev)
    e2e_ms = max_over_ranks(h0.elapsed_time(h1) / e2e_steps, dev)
    same = bool(torch.equal(oh, out.cpu()))

    if rank != 0:
        return 0

    # roofline of the traversal kernel: per-query algorithmic bytes of the PLAIN traversal (the
    # equal work unit for both runs) over the traversal phase's event-timed duration
    hbm_peak, peak_kind = measured_peaks()
    l2_gbs = l2_read_bandwidth()
    node_b, box_b, tri_b = 128, 64, 48
    nq = float(n)
    bq = (12 + 4 + st["nodes_visited"] / nq * node_b + st["boxes_tested"] / nq * box_b +
          st["triangles_tested"] / nq * tri_b)
    trav_ms = float(tms[:, 1].mean())
    achieved = nq * bq / (trav_ms * 1e-3) / 1e9
    # DRAM bytes of one traversal launch on this workload, from a single-pass ncu capture recorded
    # in the profile summaries as "traffic <workload key> <bytes>" lines
    traffic = None
    key = f"L{args.level}_g{args.grid}_b{args.band_points}_{args.build}_leaf{args.leaf}"
    for fn in sorted(os.listdir(os.path.join(ROOT, "profiles"))):
        if fn.endswith(".md"):
            with open(os.path.join(ROOT, "profiles", fn)) as fh:
                for ln in fh:
                    parts = ln.split()
                    if len(parts) >= 3 and parts[0] == "traffic" and parts[1] == key:
                        traffic = int(parts[2])

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        import oracle
        if oracle.ref_available():
            R, m, tb = reference_mesh(v, f)
            # bounded sample: probe the reference's rate, then size the sample to ~cpu_seconds
            sidx, qps_probe = calibrated_sample(m, pts, n_grid, n_band, args.cpu_seconds)
            ns = len(sidx)
            dt = time_reference(m, pts[sidx])
            # parity on that sample while it is at hand (reported, not asserted)
            d_ref = m.sdf(pts[sidx].astype(np.float64))
            d_gpu = out.index_select(0, torch.from_numpy(sidx).to(dev)).cpu().numpy().astype(np.float64)
            err = np.abs(d_gpu - d_ref)
            bandm = np.abs(d_ref) > 1e-4 * mesh.diagonal
            cpu = {"value": ns / dt, "unit": UNIT, "cores": R.max_threads(), "kind": "reference",
                   "sample": f"{ns} seeded stratified points of the workload ({n_grid} grid : {n_band} band), "
                             f"reference TriMeshSDF<double,short,4,4> Morton build ({tb:.1f}s), OpenMP over "
                             f"value(); host CPU: {cpu_info()}",
                   "parity_on_sample": {"max_abs_err": float(err.max()), "tol": 1e-6 * mesh.diagonal,
                                        "sign_mismatch_outside_band": int(np.sum(np.sign(d_gpu[bandm]) !=
                                                                                 np.sign(d_ref[bandm])))}}

    def per_query(s):
        return None if s is None else {"nodes": s["nodes_visited"] / nq, "leaves": s["leaves_visited"] / nq,
                                       "triangles": s["triangles_tested"] / nq,
                                       "oriented_boxes": s["boxes_tested"] / nq,
                                       "band_fraction": s["band_queries"] / nq,
                                       "seed_fallback_fraction": s["seed_fallbacks"] / nq}

    phases = lambda t: {"order": float(t[:, 0].mean()), "traverse": float(t[:, 1].mean()),
                        "band64": float(t[:, 2].mean()), "total": float(t[:, 3].mean())}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"mesh SDF: displaced icosphere level {args.level} ({f.shape[0]} triangles, "
                               f"{args.build} 4-wide BVH, leaf {args.leaf}), {args.grid}^3 grid over [-1.25,1.25]^3 "
                               f"+ {n_band} points within 1e-3 of the surface = {n} queries/step; FP32 traversal, "
                               f"FP64 band |d| <= 1e-4 diag",
                   "seed": ("learned pruning radius (16-level hash grid + 3x64 BF16 MLP, trained on the GPU)"
                            if seed is not None else "none (plain traversal)"),
                   "build_on_device": bool(on_device),
                   "queries_per_step": n, "l2": "inputs larger than L2 "
                   f"({pts.nbytes / 1e9:.2f} GB of points per step)", "build_s": t_build,
                   "plain": {"value": plain_value, "ms_per_step": ms_plain, "phase_ms_mean": phases(tms_plain),
                             "per_query": per_query(st), "clocks": ck_plain},
                   "perfect_radius_bound": perfect,
                   "seeded": None if seed is None else {
                       "value": value, "ms_per_step": ms_seed, "speedup_vs_plain": value / plain_value,
                       "phase_ms_mean": phases(tms_seed), "per_query": per_query(st_seed),
                       "equal_to_plain_fraction": same_frac, "max_abs_diff_vs_plain": max_diff,
                       "training": rep}},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": achieved / hbm_peak, "traffic": traffic, "peak_kind": peak_kind,
                     "kernel": "kMeshSdf32 (FP32 packet traversal" + (", seeded)" if seed is not None else ")"),
                     "bytes_per_query": bq, "bytes_basis": "plain traversal visit counts (equal work unit): 16 B query in/out + 128 B per node + "
                                    "64 B per oriented box + 48 B per triangle",
                     "l2_read_gbs_measured": l2_gbs, "frac_of_l2": achieved / l2_gbs,
                     # the floor: every byte the step must touch once (the mesh's device arrays, the
                     # points in, the distances out) at the measured HBM rate
                     "unique_bytes_per_step": int(mesh.info["device_bytes"]) + 16 * n,
                     "unique_floor_ms": (int(mesh.info["device_bytes"]) + 16 * n) / (hbm_peak * 1e6)},
        "e2e": {"value": n * world / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": int(pts.nbytes),
                "d2h_bytes_per_step": int(n * 4), "ms_per_step": e2e_ms, "matches_device_path": same},
        "gpu_launches": (4 if seed is not None else 3) * args.steps,
        "gpu_launches_note": "per step: Morton-key kernel, " + ("seed inference, " if seed is not None else "") +
                             "FP32 traversal, FP64 band pass (plus the CUB radix-sort passes of the point ordering)",
        "clocks": ck,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    return 0


def device_timed(fn, steps, warmup, torch, dev, stream):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    return e0.elapsed_time(e1) / steps


def run_knn(args, rank, world, local_rank):
    """Point-cloud k-NN (16M points: half uniform, half in 64 anisotropic clusters; 4M uniform
    queries; k = 1 and 8)."""
    import torch

    from ebgeometry_b200 import PointCloudBVH
    from ebgeometry_b200 import workloads as W
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    pts = W.point_cloud(args.knn_points, 1)
    q = W.uniform_points(args.knn_queries, 2, 0.0, 1.0)
    pd = torch.from_numpy(pts).to(dev)
    qd = torch.from_numpy(q).to(dev)
    t0 = time.time()
    cloud = PointCloudBVH(pd)
    torch.cuda.synchronize(dev)
    build_ms = (time.time() - t0) * 1e3
    build_dev = device_timed(lambda: PointCloudBVH(pd), 2, 1, torch, dev, stream)
    res = {}
    for k in (1, 8):
        ms = device_timed(lambda: cloud.knn(qd, k), args.steps, args.warmup, torch, dev, stream)
        res[f"k{k}"] = {"ms_per_step": ms, "value": q.shape[0] * world / (ms * 1e-3)}
    # the same queries on the balanced tree (fixed runs of 8 points grouped four at a time)
    bal_cloud = PointCloudBVH(pd, balanced=True)
    balanced = {"tree": bal_cloud.tree_info()}
    for k in (1, 8):
        ms = device_timed(lambda: bal_cloud.knn(qd, k), args.steps, args.warmup, torch, dev, stream)
        balanced[f"k{k}"] = {"ms_per_step": ms, "value": q.shape[0] * world / (ms * 1e-3)}
    del bal_cloud
    if rank != 0:
        return 0
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        import oracle
        if oracle.ref_available():
            R = oracle.ref()
            t0 = time.time()
            rc = R.cloud(pts)
            tb = time.time() - t0
            ns = 200000
            sq = q[:ns]
            cpu = {}
            for k in (1, 8):
                t0 = time.perf_counter()
                ri, rd = rc.knn(sq, k, lex=False)
                dt = time.perf_counter() - t0
                gi, gd = cloud.knn(torch.from_numpy(sq).to(dev), k)
                cpu[f"k{k}"] = {"value": ns / dt, "unit": UNIT, "cores": R.max_threads(), "kind": "reference",
                                "sample": f"first {ns} queries, reference PointCloudBVH<float> closestPoints "
                                          f"(build {tb:.1f}s)",
                                "d2_equal_fraction": float(np.mean(gd.cpu().numpy() == rd))}
    print(json.dumps({"metric": "k-NN queries/s on 1 B200", "workload": "knn", "n_gpus": world,
                      "config": {"points": int(pts.shape[0]), "queries": int(q.shape[0]), "leaf": 8,
                                 "tree": cloud.tree_info()},
                      "build_ms_device": build_dev, "results": res, "balanced_tree": balanced,
                      "cpu_baseline": cpu}), flush=True)
    return 0


def run_grid(args, rank, world, local_rank):
    """PointCloudHashGrid k-NN against PointCloudBVH on the same clouds: --knn-points uniform points
    (the grid's case) and the knn workload's clustered cloud; --knn-queries uniform queries; k = 1
    and 8; allNearestNeighbors (k = 1, 8) of each cloud."""
    import torch

    from ebgeometry_b200 import PointCloudBVH, PointCloudHashGrid
    from ebgeometry_b200 import workloads as W
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    q = W.uniform_points(args.knn_queries, 2, 0.0, 1.0)
    qd = torch.from_numpy(q).to(dev)
    out = {}
    clouds = {"uniform": np.random.default_rng(5).random((args.knn_points, 3), dtype=np.float32),
              "clustered": W.point_cloud(args.knn_points, 1)}
    for name, pts in clouds.items():
        t0 = time.time()
        grid = PointCloudHashGrid(pts)
        torch.cuda.synchronize(dev)
        build_s = time.time() - t0
        bvh = PointCloudBVH(torch.from_numpy(pts).to(dev))
        row = {"grid_build_s": build_s, "cells": list(grid.grid_info()[0])}
        for k in (1, 8):
            gms = device_timed(lambda: grid.knn(qd, k), args.steps, args.warmup, torch, dev, stream)
            bms = device_timed(lambda: bvh.knn(qd, k), args.steps, args.warmup, torch, dev, stream)
            gi, gd = grid.knn(qd, k)
            bi, bd = bvh.knn(qd, k)
            same = bool(torch.equal(gi, bi) and torch.equal(gd, bd))
            row[f"k{k}"] = {"grid_qps": q.shape[0] / (gms * 1e-3), "bvh_qps": q.shape[0] / (bms * 1e-3),
                            "identical": same}
            gms = device_timed(lambda: grid.all_nearest_neighbors(k, device=True), args.steps, args.warmup, torch,
                               dev, stream)
            bms = device_timed(lambda: bvh.all_nearest_neighbors(k, device=True), args.steps, args.warmup, torch,
                               dev, stream)
            gi, gd = grid.all_nearest_neighbors(k, device=True)
            bi, bd = bvh.all_nearest_neighbors(k, device=True)
            same = bool(torch.equal(gi, bi) and torch.equal(gd, bd))
            row[f"self_k{k}"] = {"grid_qps": pts.shape[0] / (gms * 1e-3), "bvh_qps": pts.shape[0] / (bms * 1e-3),
                                 "identical": same}
        grid.check_status()
        bvh.check_status()
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            import oracle
            if oracle.ref_available():
                R = oracle.ref()
                t0 = time.time()
                rg = R.grid(pts)
                tb = time.time() - t0
                ns = 200000
                sq = q[:ns]
                for k in (1, 8):
                    t0 = time.perf_counter()
                    _, rd = rg.knn(sq, k)
                    dt = time.perf_counter() - t0
                    _, gd = grid.knn(sq, k)
                    row[f"k{k}"]["cpu_baseline"] = {
                        "value": ns / dt, "unit": UNIT, "cores": R.max_threads(), "kind": "reference",
                        "sample": f"first {ns} queries, reference PointCloudHashGrid<float> closestPoints "
                                  f"(build {tb:.1f}s)", "d2_equal_fraction": float(np.mean(gd == rd))}
        out[name] = row
        del grid, bvh
    if rank == 0:
        print(json.dumps({"metric": "k-NN queries/s on 1 B200", "workload": "grid", "n_gpus": world,
                          "config": {"points": args.knn_points, "queries": int(q.shape[0])}, "results": out}),
              flush=True)
    return 0


def run_csg(args, rank, world, local_rank):
    """Batched CSG union: spheres + posed displaced icospheres (levels 3-7), batches of log-uniform
    length 1k-1M concatenated into one call (one persistent launch)."""
    import torch

    from ebgeometry_b200 import BVHUnion, TriMeshSDF
    from ebgeometry_b200 import workloads as W
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    t0 = time.time()
    sc = W.csg_scene(11, n_spheres=args.csg_spheres, n_meshes=args.csg_meshes)
    tms = [TriMeshSDF(v, f, device=local_rank, on_device=True) for v, f in sc["meshes"]]
    scene = BVHUnion(sc["spheres"], tms, sc["poses"], device=local_rank)
    t_build = time.time() - t0
    rng = np.random.default_rng(12)
    lens = np.exp(rng.uniform(np.log(1e3), np.log(1e6), args.csg_batches)).astype(np.int64)
    n = int(lens.sum())
    lo = np.minimum(sc["spheres"][:, :3].min(0), sc["poses"][:, 2:5].min(0)) - 0.2
    hi = np.maximum(sc["spheres"][:, :3].max(0), sc["poses"][:, 2:5].max(0)) + 0.2
    pts = (rng.random((n, 3), dtype=np.float32) * (hi - lo).astype(np.float32) + lo.astype(np.float32))
    pd = torch.from_numpy(pts).to(dev)
    out = torch.empty(n, dtype=torch.float32, device=dev)
    ms = device_timed(lambda: scene.values(pd, out=out), args.steps, args.warmup, torch, dev, stream)
    scene.check_status()
    if rank != 0:
        return 0
    ntris = int(sum(f.shape[0] for _, f in sc["meshes"]))
    print(json.dumps({"metric": "CSG union queries/s on 1 B200", "workload": "csg", "n_gpus": world,
                      "value": n * world / (ms * 1e-3), "ms_per_step": ms,
                      "config": {"spheres": args.csg_spheres, "meshes": args.csg_meshes, "mesh_triangles": ntris,
                                 "batches": args.csg_batches, "points": n, "build_s": t_build}}), flush=True)
    return 0


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and args.impl == "ours":
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        if args.impl == "reference":
            return run_reference(args, rank, world)
        if args.workload == "knn":
            return run_knn(args, rank, world, local_rank)
        if args.workload == "grid":
            return run_grid(args, rank, world, local_rank)
        if args.workload == "csg":
            return run_csg(args, rank, world, local_rank)
        return run_ours(args, rank, world, local_rank)
    finally:
        if world > 1 and args.impl == "ours":
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
