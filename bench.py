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


def _module(name):
    """A pure-Python module of the package, loaded from its file without running the package's
    __init__ (which loads the CUDA library): the reference arm maps only the oracle's libraries."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(f"_bench_{name}", os.path.join(ROOT, "ebgeometry_b200", f"{name}.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


max_over_ranks = _module("ranks").max_over_ranks

METRIC = "SDF queries/s on 1 B200: learned-seeded vs plain GPU BVH at equal accuracy"
UNIT = "queries/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["mesh", "fp64", "knn", "grid", "csg"], default="mesh",
                    help="mesh: the headline mesh-SDF configuration; fp64: the level-5 mesh, 1M FP64 queries; "
                         "knn: 16M-point cloud, 4M queries, k=1 and 8; "
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
    ap.add_argument("--cells", type=int, default=0, help="seed attach: cells per axis (0 = the library default)")
    ap.add_argument("--cut-entries", type=int, default=0, help="seed attach: subtrees per cell (0 = default)")
    ap.add_argument("--cell-margin", type=float, default=0.0, help="seed attach: cell growth in cells (0 = default)")
    ap.add_argument("--seed-ablation", action="store_true",
                    help="also time the seeded traversal with no radius, with the exact cell radius and without "
                         "anchors (what each part of the seed buys)")
    ap.add_argument("--traffic-csv", default=None,
                    help="ncu CSV (dram__bytes_read.sum, dram__bytes_write.sum of the traversal kernel) captured "
                         "from this same command; fills roofline.traffic")
    ap.add_argument("--no-wide", action="store_true",
                    help="skip the plain traversal through the tree's 8-wide copy (the node-width comparison)")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the FP64 level-5 and k-NN configurations measured beside the headline line")
    ap.add_argument("--seed-samples", type=int, default=1 << 25)
    ap.add_argument("--seed-steps", type=int, default=2000)
    ap.add_argument("--seed-batch", type=int, default=1 << 18)
    ap.add_argument("--seed-save", default=None, help="write the trained model to this path")
    ap.add_argument("--seed-load", default=None, help="load a trained model instead of training one")
    return ap.parse_args()


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def workload(args):
    W = _module("workloads")
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
def reference_mesh(v, f, kind=0, timing=True):
    """The reference's TriMeshSDF (Morton build): kind 0 <double,short,4,4>, kind 1 the ISA-default
    K/W; from the timing build (or the parity build with timing=False)."""
    import oracle
    R = oracle.ref(timing=timing)
    t0 = time.time()
    m = R.mesh(v, f, kind=kind, build=1, max_leaf_groups=4)
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
    """Read bandwidth of a 48 MB L2-resident buffer streamed by the bench's probe kernel
    (ebgeometry_b200/libebgprobe.so, built beside the library, outside its C ABI)."""
    import ctypes as C
    lib = C.CDLL(os.path.join(ROOT, "ebgeometry_b200", "libebgprobe.so"))
    lib.ebgprobe_read_bandwidth.restype = C.c_int
    lib.ebgprobe_read_bandwidth.argtypes = [C.c_int64, C.c_int32, C.POINTER(C.c_double)]
    out = C.c_double()
    rc = lib.ebgprobe_read_bandwidth(48 << 20, 20, C.byref(out))
    return out.value if rc == 0 else None


def traffic_from_csv(path, kernel="kMeshSdf32"):
    """DRAM bytes (read + write) per launch of `kernel`, averaged over the launches an ncu CSV
    (--metrics dram__bytes_read.sum,dram__bytes_write.sum --csv) recorded."""
    import csv
    if not path or not os.path.exists(path):
        return None
    per = {}
    with open(path) as fh:
        rows = [ln for ln in fh if ln.startswith('"')]
    for r in csv.DictReader(rows):
        if kernel not in r.get("Kernel Name", ""):
            continue
        name, unit, val = r.get("Metric Name"), r.get("Metric Unit", ""), r.get("Metric Value", "0")
        if name not in ("dram__bytes_read.sum", "dram__bytes_write.sum"):
            continue
        scale = {"byte": 1, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9, "KB": 1e3, "MB": 1e6, "GB": 1e9}.get(unit, 1)
        per.setdefault(r.get("ID"), 0.0)
        per[r.get("ID")] += float(val.replace(",", "")) * scale
    return (sum(per.values()) / len(per)) if per else None


def packet_bytes(st, n):
    """Bytes the traversal's warps load per call, counted per packet (each distinct line once per
    packet: the packet is what a warp executes): 128 B per interior node opened, 64 B per oriented
    box tested, 48 B per triangle record of an opened leaf, 32 B per entry of a cell's cut plus the
    cell's count and radius and one anchor index and record (the lanes read those of their own
    cells, one to eight per packet: counting one keeps this a lower bound); and per query its 12-B
    point, 4-B order index, 4-B result and the winner's 96-B sign record."""
    return (128 * st["packet_nodes"] + 64 * st["packet_boxes"] + 48 * st["packet_triangle_records"] +
            32 * st["cut_entries"] + 60 * st["cut_packets"] + n * (12 + 4 + 4 + 96))


def reference_rates(v, f, pts, n_grid, n_band, build=1, cpu_seconds=12.0):
    """The reference's TriMeshSDF<double,short,4,4> and its ISA-default K/W, from the timing build
    (oracle/_ref, -O3 -march=sapphirerapids with fused multiply-adds) on all host threads, on one
    seeded stratified sample of the workload sized for about cpu_seconds of work in total.  Returns
    (queries/s by kind, sample indices, build seconds by kind, library, threads)."""
    import oracle
    R = oracle.ref(timing=True)
    rates, builds, sidx = {}, {}, None
    for kind in (0, 1):
        t0 = time.time()
        m = R.mesh(v, f, kind=kind, build=build, max_leaf_groups=4)
        builds[kind] = time.time() - t0
        if sidx is None:
            probe = sample_indices(n_grid, n_band, 16384, seed=5)
            qps0 = probe.shape[0] / max(time_reference(m, pts[probe]), 1e-6)
            sidx = sample_indices(n_grid, n_band, int(min(max(qps0 * cpu_seconds / 2, 16384), 8_000_000)))
        rates[kind] = sidx.shape[0] / time_reference(m, pts[sidx])
        del m
    return rates, sidx, builds, os.path.basename(R.path), R.max_threads()


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
    # the faster of the reference's 4-wide and ISA-default trees on a short probe
    best = None
    for kind in (0, 1):
        R, m, tbuild = reference_mesh(v, f, kind)
        _, qps0 = calibrated_sample(m, pts, n_grid, n_band, 1.0)
        if best is None or qps0 > best[3]:
            best = (R, m, tbuild, qps0, kind)
        else:
            del m
    R, m, tbuild, qps0, kind = best
    # each step: a fresh stratified sample sized for ~4 s of CPU work
    n = int(min(max(qps0 * 4.0, 16384), 4_000_000))
    for s in range(args.warmup):
        time_reference(m, pts[sample_indices(n_grid, n_band, n, seed=100 + s)])
    times = []
    for s in range(args.steps):
        times.append(time_reference(m, pts[sample_indices(n_grid, n_band, n, seed=200 + s)]))
    tot = sum(times)
    qps = n * args.steps / tot
    cores = R.max_threads()
    impl = ("reference TriMeshSDF<double,short,4,4>" if kind == 0 else
            "reference TriMeshSDF<double,short> with the ISA-default branching and SoA width")
    sample = (f"{n} points per step: a seeded stratified sample of the {n_grid + n_band} workload points "
              f"({n_grid} grid + {n_band} band in proportion); {impl}, Morton build, "
              f"{os.path.basename(R.path)} (-O3 -march=sapphirerapids with fused multiply-adds)")
    line = {"impl": "reference", "metric": METRIC, "value": qps, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"mesh SDF, displaced icosphere level {args.level} ({f.shape[0]} triangles), "
                                   f"{args.grid}^3 grid + {n_band} band points",
                       "implementation": impl + " (Morton build), value() per point in an OpenMP parallel-for, "
                                                "the faster of the 4-wide and ISA-default configurations",
                       "build_s": tbuild,
                       "cpu": cpu_info()},
            "cpu_baseline": {"value": qps, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
            "e2e": {"value": qps, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def timed_steps(mesh, pd, out, steps, seed, dev, world, stream, _capi, torch, dist, local_rank, hint=None,
                node_width=None):
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
        mesh.signed_distance(pd, out=out, timings=tm, seed=seed, radius_hint=hint, node_width=node_width)
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

    # node width: the same plain traversal through the tree's 8-wide copy (same results)
    wide = None
    if not args.no_wide:
        from ebgeometry_b200 import EbgError
        try:
            t0 = time.time()
            winfo = mesh.widen()
            winfo["widen_s"] = time.time() - t0
            _, st_w = mesh.stats(pd, node_width=8)
            wout = torch.empty_like(out)
            for _ in range(args.warmup):
                mesh.signed_distance(pd, out=wout, node_width=8)
            torch.cuda.synchronize(dev)
            ms_w, tms_w, _ = timed_steps(mesh, pd, wout, args.steps, None, *tctx, node_width=8)
            wide = {"ms_per_step": ms_w, "value": n * world / (ms_w * 1e-3), "vs_width4": ms_plain / ms_w,
                    "phase_ms_mean": tms_w, "per_packet": st_w, "tree": winfo,
                    "equal_to_width4": bool(torch.equal(wout, out))}
            del wout
            log(f"[rank {rank}] plain, 8-wide copy {ms_w:.1f} ms/step {winfo}")
        except EbgError as e:
            wide = {"error": str(e)}

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

    seed, rep, att, st_seed, ablation = None, None, None, None, None
    if not args.no_seed:
        t0 = time.time()
        if args.seed_load:
            seed = SeedModel.load(args.seed_load, device=local_rank)
        else:
            seed = SeedModel.train(mesh, num_samples=args.seed_samples, steps=args.seed_steps,
                                   batch=args.seed_batch, rng_seed=7, lo=[-1.25] * 3, hi=[1.25] * 3, attach=False)
        rep = seed.report()
        rep["wall_s"] = time.time() - t0
        rep["loaded_from"] = args.seed_load
        if args.seed_save:
            seed.save(args.seed_save)
        log(f"[rank {rank}] seed trained: {rep}")
        attach_kw = dict(cells_per_axis=args.cells, max_entries=args.cut_entries, margin_cells=args.cell_margin)
        t0 = time.time()
        att = mesh.attach_seed(seed, **attach_kw)
        att["wall_s"] = time.time() - t0
        log(f"[rank {rank}] seed attached: {att}")
        _, st_seed = mesh.stats(pd, seed=seed)
        log(f"[rank {rank}] seeded stats {st_seed}")
        for _ in range(args.warmup):
            mesh.signed_distance(pd, out=out, seed=seed)
        torch.cuda.synchronize(dev)
        ms_seed, tms_seed, ck_seed = timed_steps(*tsteps, seed, *tctx)
        log(f"[rank {rank}] seeded {ms_seed:.1f} ms/step")
        same_frac = float((out == plain_ref).float().mean().item())
        max_diff = float((out - plain_ref).abs().max().item())
        if args.seed_ablation:
            # what each part of the seed buys: no radius (cuts by distance order only), the exact
            # distance at the cell centres instead of the model's radius, no anchor triangles
            ablation = []
            aout = torch.empty_like(out)
            for mode, anchors, what in ((1, True, "no radius (cuts by distance order only)"),
                                        (2, True, "exact cell-centre distance instead of the model"),
                                        (0, False, "model radius, no anchor triangles")):
                mesh.attach_seed(seed, radius_mode=mode, anchors=anchors, **attach_kw)
                mesh.signed_distance(pd, out=aout, seed=seed)
                ms_a, _, _ = timed_steps(mesh, pd, aout, max(2, args.steps // 2), seed, *tctx)
                ablation.append({"variant": what, "ms_per_step": ms_a, "speedup_vs_plain": ms_plain / ms_a,
                                 "equal_to_plain": bool(torch.equal(aout, plain_ref))})
                log(f"[rank {rank}] ablation {what}: {ms_a:.1f} ms/step")
            del aout
            mesh.attach_seed(seed, **attach_kw)
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

    # roofline of the traversal kernel (the launch timed as the "traverse" phase): the bytes its warps
    # load per call, counted per packet from the measured run's own counters, over the phase's
    # event-timed duration, against the measured HBM copy roof and the measured L2 read roof
    hbm_peak, peak_kind = measured_peaks()
    l2_gbs = l2_read_bandwidth()
    st_run = st_seed if seed is not None else st
    nq = float(n)
    bytes_call = float(packet_bytes(st_run, n))
    trav_ms = float(tms[:, 1].mean())
    achieved = bytes_call / (trav_ms * 1e-3) / 1e9
    traffic = traffic_from_csv(args.traffic_csv)

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        import oracle
        if oracle.ref_available():
            rates, sidx, builds, lib_name, threads = reference_rates(v, f, pts, n_grid, n_band, build=1,
                                                                     cpu_seconds=args.cpu_seconds)
            kind = max(rates, key=rates.get)
            # parity on that sample against the parity build of the reference (reported here; the
            # gpu tests assert it)
            _, mref, _ = reference_mesh(v, f, 0, timing=False)
            d_ref = mref.sdf(pts[sidx].astype(np.float64))
            del mref
            d_gpu = out.index_select(0, torch.from_numpy(sidx).to(dev)).cpu().numpy().astype(np.float64)
            err = np.abs(d_gpu - d_ref)
            bandm = np.abs(d_ref) > 1e-4 * mesh.diagonal
            cpu = {"value": rates[kind], "unit": UNIT, "cores": threads, "kind": "reference",
                   "sample": f"{sidx.shape[0]} seeded stratified points of the workload ({n_grid} grid : {n_band} "
                             f"band), reference TriMeshSDF Morton build, OpenMP over value(), {lib_name} "
                             f"(-O3 -march=sapphirerapids, fused multiply-adds); host CPU: {cpu_info()}",
                   "by_configuration": {"TriMeshSDF<double,short,4,4>": {"value": rates[0], "build_s": builds[0]},
                                        "TriMeshSDF<double,short> (ISA-default K, W)": {"value": rates[1],
                                                                                         "build_s": builds[1]}},
                   "parity_on_sample": {"max_abs_err": float(err.max()), "tol": 1e-6 * mesh.diagonal,
                                        "sign_mismatch_outside_band": int(np.sum(np.sign(d_gpu[bandm]) !=
                                                                                 np.sign(d_ref[bandm])))}}

    def per_query(s):
        return None if s is None else {"nodes": s["nodes_visited"] / nq, "leaves": s["leaves_visited"] / nq,
                                       "triangles": s["triangles_tested"] / nq,
                                       "oriented_boxes": s["boxes_tested"] / nq,
                                       "band_fraction": s["band_queries"] / nq,
                                       "seed_fallback_fraction": s["seed_fallbacks"] / nq}

    def per_packet(s):
        pk = max(s["packets"], 1)
        return {"pops": s["packet_pops"] / pk, "nodes": s["packet_nodes"] / pk, "leaves": s["packet_leaves"] / pk,
                "triangle_passes": s["packet_triangles"] / pk, "oriented_boxes": s["packet_boxes"] / pk,
                "triangle_records": s["packet_triangle_records"] / pk,
                "cut_packet_fraction": s["cut_packets"] / pk,
                "cut_entries_per_cut_packet": s["cut_entries"] / max(s["cut_packets"], 1)}

    phases = lambda t: {"order": float(t[:, 0].mean()), "traverse": float(t[:, 1].mean()),
                        "band64": float(t[:, 2].mean()), "total": float(t[:, 3].mean())}
    if wide is not None and "error" not in wide:
        wide["phase_ms_mean"] = phases(wide["phase_ms_mean"])
        wide["per_packet"] = per_packet(wide["per_packet"])
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"mesh SDF: displaced icosphere level {args.level} ({f.shape[0]} triangles, "
                               f"{args.build} 4-wide BVH, leaf {args.leaf}), {args.grid}^3 grid over [-1.25,1.25]^3 "
                               f"+ {n_band} points within 1e-3 of the surface = {n} queries/step; FP32 traversal, "
                               f"FP64 band |d| <= 1e-4 diag",
                   "seed": ("learned pruning radius (16-level hash grid + 3x64 BF16 MLP, trained on the GPU) "
                            "attached as per-cell entry cuts of the tree with anchor triangles"
                            if seed is not None else "none (plain traversal)"),
                   "build_on_device": bool(on_device),
                   "queries_per_step": n, "l2": "inputs larger than L2 "
                   f"({pts.nbytes / 1e9:.2f} GB of points per step)", "build_s": t_build,
                   "plain": {"value": plain_value, "ms_per_step": ms_plain, "phase_ms_mean": phases(tms_plain),
                             "per_query": per_query(st), "per_packet": per_packet(st), "clocks": ck_plain,
                             "node_width8": wide},
                   "perfect_radius_bound": perfect,
                   "seeded": None if seed is None else {
                       "value": value, "ms_per_step": ms_seed, "speedup_vs_plain": value / plain_value,
                       "phase_ms_mean": phases(tms_seed), "per_query": per_query(st_seed),
                       "per_packet": per_packet(st_seed), "equal_to_plain_fraction": same_frac,
                       "max_abs_diff_vs_plain": max_diff, "training": rep, "attach": att,
                       "ablation": ablation}},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": achieved / hbm_peak, "traffic": traffic, "peak_kind": peak_kind,
                     "traffic_source": (f"ncu capture {os.path.basename(args.traffic_csv)}" if traffic is not None
                                        else "none in this run (pass --traffic-csv from an ncu capture of it)"),
                     "kernel": "kMeshSdf32 (FP32 packet traversal" + (", seeded)" if seed is not None else ")"),
                     "bytes_per_query": bytes_call / nq,
                     "bytes_basis": "per packet: 128 B per interior node opened + 64 B per oriented box + 48 B per "
                                    "triangle record of an opened leaf + 32 B per cut entry (+60 B per cut); per "
                                    "query: 12 B point + 4 B order + 4 B result + 96 B sign record",
                     "l2_read_gbs_measured": l2_gbs, "frac_of_l2": (achieved / l2_gbs) if l2_gbs else None,
                     "limiter": "instruction issue and L1/L2 latency on the SMs (ncu: issue-active ~75 %, about "
                                "2 eligible warps per cycle, L2 throughput a few %), not DRAM or L2 bandwidth",
                     # the floor: every byte the step must touch once (the mesh's device arrays, the
                     # points in, the distances out) at the measured HBM rate
                     "unique_bytes_per_step": int(mesh.info["device_bytes"]) + 16 * n,
                     "unique_floor_ms": (int(mesh.info["device_bytes"]) + 16 * n) / (hbm_peak * 1e6)},
        "e2e": {"value": n * world / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": int(pts.nbytes),
                "d2h_bytes_per_step": int(n * 4), "ms_per_step": e2e_ms, "matches_device_path": same},
        "gpu_launches": 3 * args.steps,
        "gpu_launches_note": "per step: Morton-key kernel, FP32 traversal, FP64 band pass (plus the CUB radix-sort "
                             "and band-list compaction passes)",
        "clocks": ck,
        "cpu_baseline": cpu,
    }
    if world == 1 and not args.no_extra:
        # the other configurations' device throughput, end-to-end throughput and CPU baseline
        del pd, out, plain_ref
        torch.cuda.empty_cache()
        line["other_configurations"] = {"fp64_level5": measure_fp64(args, torch, dev, stream,
                                                                    cpu=not args.no_cpu_baseline),
                                        "knn": measure_knn(args, torch, dev, stream, cpu=not args.no_cpu_baseline)}
    print(json.dumps(line), flush=True)
    return 0


def measure_fp64(args, torch, dev, stream, cpu=True):
    """The CPU-runnable configuration: level-5 displaced icosphere (20,480 triangles, 4-wide SAH
    tree), 1,048,576 FP64 points uniform in [-1.5,1.5]^3, FP64 signed distance end to end."""
    from ebgeometry_b200 import TriMeshSDF
    W = _module("workloads")
    v, f = W.displaced_icosphere(5, 1)
    p = np.random.default_rng(3).uniform(-1.5, 1.5, size=(1 << 20, 3))
    mesh = TriMeshSDF(v, f, build="SAH", leaf_size=8)
    pd = torch.from_numpy(p).to(dev)
    out = torch.empty(p.shape[0], dtype=torch.float64, device=dev)
    ms = device_timed(lambda: mesh.signed_distance(pd, out=out), max(3, args.steps), 3, torch, dev, stream)
    ph = torch.from_numpy(p).pin_memory()
    oh = torch.empty(p.shape[0], dtype=torch.float64).pin_memory()
    hn = ph.numpy()
    ohn = oh.numpy()
    mesh.signed_distance(hn, out=ohn)
    t0 = time.perf_counter()
    reps = 3
    for _ in range(reps):
        mesh.signed_distance(hn, out=ohn)  # the host entry point: H2D, query, D2H (synchronous)
    e2e_ms = (time.perf_counter() - t0) * 1e3 / reps
    res = {"workload": "level-5 displaced icosphere (20,480 triangles, SAH), 1,048,576 FP64 points uniform in "
                       "[-1.5,1.5]^3, FP64 signed distance", "unit": UNIT,
           "value": p.shape[0] / (ms * 1e-3), "ms_per_step": ms,
           "e2e": {"value": p.shape[0] / (e2e_ms * 1e-3), "ms_per_step": e2e_ms, "h2d_bytes_per_step": int(p.nbytes),
                   "d2h_bytes_per_step": int(p.shape[0] * 8), "timer": "host wall clock around the synchronous "
                                                                       "host entry point"}}
    if cpu:
        import oracle
        if oracle.ref_available():
            d = out.cpu().numpy()
            rates = {}
            for kind, name in ((0, "TriMeshSDF<double,short,4,4>"), (1, "TriMeshSDF<double,short> (ISA-default K, W)")):
                R = oracle.ref(timing=True)
                m = R.mesh(v, f, kind=kind, build=0, max_leaf_groups=4)
                m.sdf(p[:20000])
                t0 = time.perf_counter()
                m.sdf(p)
                rates[name] = p.shape[0] / (time.perf_counter() - t0)
                del m
            best = max(rates, key=rates.get)
            ref = oracle.ref().mesh(v, f, kind=0, build=0, max_leaf_groups=4).sdf(p)
            res["cpu_baseline"] = {"value": rates[best], "unit": UNIT, "cores": oracle.ref(timing=True).max_threads(),
                                   "kind": "reference", "sample": f"all {p.shape[0]} points, reference {best} SAH "
                                   "(the faster configuration), -O3 -march=sapphirerapids",
                                   "by_configuration": rates}
            res["parity"] = {"bit_identical_fraction": float(np.mean(d == ref)),
                             "max_abs_err": float(np.abs(d - ref).max()), "tol": 1e-6 * mesh.diagonal}
    return res


def measure_knn(args, torch, dev, stream, cpu=True):
    """Point-cloud nearest neighbours: 16M FP32 points (half uniform, half in 64 anisotropic
    clusters), 4M uniform queries, k = 1 and 8; int32 indices, ties to the lowest index."""
    from ebgeometry_b200 import PointCloudBVH
    W = _module("workloads")
    pts = W.point_cloud(args.knn_points, 1)
    q = W.uniform_points(args.knn_queries, 2, 0.0, 1.0)
    cloud = PointCloudBVH(torch.from_numpy(pts).to(dev))
    qd = torch.from_numpy(q).to(dev)
    res = {"workload": f"{pts.shape[0]} points (half uniform, half in 64 anisotropic clusters), {q.shape[0]} uniform "
                       "queries; int32 indices", "unit": UNIT}
    qh = torch.from_numpy(q).pin_memory().numpy()  # the caller's queries in pinned host memory
    for k in (1, 8):
        ms = device_timed(lambda: cloud.knn(qd, k), max(3, args.steps), 3, torch, dev, stream)
        cloud.knn(qh[:1000], k)
        reps = 3
        t0 = time.perf_counter()
        for _ in range(reps):
            cloud.knn(qh, k)  # the host entry point: H2D, query, D2H (synchronous)
        e2e_ms = (time.perf_counter() - t0) * 1e3 / reps
        res[f"k{k}"] = {"value": q.shape[0] / (ms * 1e-3), "ms_per_step": ms,
                        "e2e": {"value": q.shape[0] / (e2e_ms * 1e-3), "ms_per_step": e2e_ms,
                                "h2d_bytes_per_step": int(q.nbytes), "d2h_bytes_per_step": int(q.shape[0] * k * 8)}}
    if cpu:
        import oracle
        if oracle.ref_available():
            R = oracle.ref(timing=True)
            t0 = time.time()
            rc = R.cloud(pts)
            tb = time.time() - t0
            ns = 200000
            for k in (1, 8):
                t0 = time.perf_counter()
                rc.knn(q[:ns], k, lex=False)
                dt = time.perf_counter() - t0
                res[f"k{k}"]["cpu_baseline"] = {
                    "value": ns / dt, "unit": UNIT, "cores": R.max_threads(), "kind": "reference",
                    "sample": f"first {ns} queries, reference PointCloudBVH<float> closestPoints (build {tb:.1f}s), "
                              "-O3 -march=sapphirerapids"}
            del rc
            # parity against the reference's parity build (its float arithmetic without fused
            # multiply-adds, which the timing build contracts)
            rp = oracle.ref().cloud(pts)
            for k in (1, 8):
                ri, rd = rp.knn(q[:ns], k, lex=True)
                gi, gd = cloud.knn(q[:ns], k)
                res[f"k{k}"]["parity"] = {"queries": ns, "d2_equal_fraction": float(np.mean(gd == rd)),
                                          "index_equal_fraction": float(np.mean(gi == ri))}
    return res


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
    """Batched CSG union: 4,096 spheres + 256 posed displaced icospheres (levels 3-7), 2,048 query
    batches of log-uniform length 1k-1M points, all in one call (ebg_scene_eval_batches: one
    persistent launch over all batches, then the FP64 near-surface pass)."""
    import torch

    from ebgeometry_b200 import BVHUnion, TriMeshSDF
    W = _module("workloads")
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
    starts = np.concatenate([[0], np.cumsum(lens)])
    pd = torch.from_numpy(pts).to(dev)
    out = torch.empty(n, dtype=torch.float32, device=dev)
    batches = [pd[starts[i]:starts[i + 1]] for i in range(len(lens))]
    outs = [out[starts[i]:starts[i + 1]] for i in range(len(lens))]
    ms = device_timed(lambda: scene.values_batches(batches, outs=outs), args.steps, args.warmup, torch, dev, stream)
    scene.check_status()
    # end to end: every step copies each batch in from pinned host memory, evaluates all of them in
    # one call and copies the results out
    ph = torch.from_numpy(pts).pin_memory()
    oh = torch.empty(n, dtype=torch.float32).pin_memory()

    def e2e_step():
        for i in range(len(lens)):
            batches[i].copy_(ph[starts[i]:starts[i + 1]], non_blocking=True)
        scene.values_batches(batches, outs=outs)
        oh.copy_(out, non_blocking=True)

    e2e_ms = device_timed(e2e_step, max(2, min(args.steps, 3)), 1, torch, dev, stream)
    same = bool(torch.equal(oh, out.cpu()))
    if rank != 0:
        return 0
    ntris = int(sum(f.shape[0] for _, f in sc["meshes"]))
    mesh_bytes = int(sum(t.info["device_bytes"] for t in tms))
    hbm_peak, peak_kind = measured_peaks()
    unique = mesh_bytes + 16 * n
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        import oracle
        if oracle.ref_available():
            bb = []
            for (v, f), ps in zip(sc["meshes"], sc["poses"]):
                w = W.rotate_points(v, -ps[0], int(ps[1])) + ps[2:5]
                bb.append(np.concatenate([w.min(0) - 1e-9, w.max(0) + 1e-9]))
            R = oracle.ref(timing=True)
            t0 = time.time()
            rs = R.scene(sc["spheres"], sc["meshes"], sc["poses"], np.array(bb))
            tb = time.time() - t0
            sidx = np.sort(rng.choice(n, size=min(n, 200000), replace=False))
            sp = pts[sidx].astype(np.float64)
            rs.value(sp[:5000])
            t0 = time.perf_counter()
            ref = rs.value(sp)
            dt = time.perf_counter() - t0
            d = out.index_select(0, torch.from_numpy(sidx).to(dev)).cpu().numpy().astype(np.float64)
            diag = float(np.linalg.norm(hi - lo))
            outside = np.abs(ref) > 1e-4 * diag
            cpu = {"value": sidx.shape[0] / dt, "unit": UNIT, "cores": R.max_threads(), "kind": "reference",
                   "sample": f"{sidx.shape[0]} seeded points of the batches, reference BVHUnion<double, "
                             f"ImplicitFunction<double>, AABB, 4> over SphereSDF and Translate(Rotate(TriMeshSDF"
                             f"<double,short,4,4>)) (build {tb:.1f}s on all threads), -O3 -march=sapphirerapids",
                   "parity_on_sample": {"max_abs_err": float(np.abs(d - ref).max()), "tol": 1e-6 * diag,
                                        "sign_mismatch_outside_band": int(np.sum(np.sign(d[outside]) !=
                                                                                 np.sign(ref[outside])))}}
    print(json.dumps({"metric": "CSG union queries/s on 1 B200", "workload": "csg", "n_gpus": world,
                      "value": n * world / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms, "steps": args.steps,
                      "warmup": args.warmup, "dtype": "f32", "data": "synthetic",
                      "config": {"workload": f"{args.csg_spheres} spheres + {args.csg_meshes} displaced icospheres "
                                             f"(levels 3-7, {ntris} triangles) at random poses; {args.csg_batches} "
                                             f"batches of log-uniform length 1k-1M = {n} points in one "
                                             "ebg_scene_eval_batches call; FP32 with the FP64 near-surface pass",
                                 "points": n, "build_s": t_build, "l2": "inputs larger than L2"},
                      "roofline": {"bound": "hbm", "achieved": unique / (ms * 1e-3) / 1e9, "peak": hbm_peak,
                                   "unit": "GB/s", "frac": unique / (ms * 1e-3) / 1e9 / hbm_peak, "traffic": None,
                                   "peak_kind": peak_kind,
                                   "bytes_basis": "unique bytes (the meshes' device arrays once, 16 B per query); "
                                                  "the union kernel keeps no per-packet counters"},
                      "e2e": {"value": n * world / (e2e_ms * 1e-3), "unit": UNIT, "ms_per_step": e2e_ms,
                              "h2d_bytes_per_step": int(pts.nbytes), "d2h_bytes_per_step": int(4 * n),
                              "matches_device_path": same},
                      "gpu_launches": 6 * args.steps,
                      "cpu_baseline": cpu}), flush=True)
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
        if args.workload == "fp64":
            import torch
            dev = torch.device("cuda", local_rank)
            torch.cuda.set_device(dev)
            r = measure_fp64(args, torch, dev, torch.cuda.current_stream(dev), cpu=not args.no_cpu_baseline)
            if rank == 0:
                print(json.dumps({"metric": "FP64 mesh SDF queries/s on 1 B200", "n_gpus": world, **r}), flush=True)
            return 0
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
