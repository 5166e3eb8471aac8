"""Benchmark of the generate_grid_sdf / generate_sdf hot path on B200.

Workload (one "step"): generate_grid_sdf with SignMethod::Raycast on a 256^3
grid over the bounding box (padded 10 %) of the displaced star icosphere,
subdivision 6 (40,962 vertices, 81,920 triangles) — the medium plain-method
configuration.  `value` is cells/s with the mesh resident in HBM; `e2e` is the
same metric through the host-pointer C ABI (mesh H2D and result D2H inside the
timed region).  The 1M-point queries of the same configuration (Bvh+Raycast,
Rtree) and the brute force on 65,536 points are reported beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun every rank runs an independent replica (the path has no
exchange step), timed on the device, max over ranks.
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

GRID_N = 256
N_POINTS = 1_000_000
N_BRUTE = 65_536
SEED = 0


# DRAM bytes (read + write) of one propagation launch of the bench grid, from
# an ncu capture of dram__bytes_read.sum and dram__bytes_write.sum (one launch).
PROPAGATE_DRAM_BYTES = 145_844_224 + 243_579_392
PROPAGATE_DRAM_SOURCE = "profiles/k_propagate_star_s6_grid256.md (ncu, one 256^3 launch)"


# FP32 operations of one propagation evaluation, counting every add, sub, mul,
# div and sqrt as one: the closest point on the interior path (67), the
# squared distance (8) and its square root (1); Normal adds the sign's dot
# product (5).  The strict build issues no fused multiply-add.
EVAL_OPS = {"raycast": 76, "normal": 81}


def grid_roofline(cells, n_vertices, n_tris, phases, stats, hbm_peak, peak_source, sm_mhz, sign):
    """Roofline of the dominant kernel of a grid (propagation).  Algorithmic
    bytes: 4 B per output cell plus the mesh once (12 B per vertex, 12 B of
    u32 indices per triangle) — the HBM bytes the result itself needs.
    `implementation_bytes` counts what the kernel's own data structures move
    (per relaxed state its 8 B entry and 48 B triangle record, per proposal
    the neighbour's 8 B key read and its 8 B atomic), mostly L2 hits.
    `traffic` is the ncu DRAM count of one launch of the bench grid and
    `traffic_ratio` its multiple of the algorithmic bytes.  `fp32` sets the
    evaluated proposals' FP32 operations against the FP32 peak (148 SMs x
    128 lanes x the SM clock, one operation per lane and cycle: no FMA)."""
    prop_s = phases["propagation"] / 1e3
    algo = 4 * cells + 12 * n_vertices + 12 * n_tris
    achieved = algo / prop_s / 1e9 if prop_s > 0 else 0.0
    impl = stats["states_relaxed"] * 56 + stats["neighbour_evals"] * 16
    evaluated = stats["neighbour_evals"] - stats.get("dropped_same", 0) - stats.get("dropped_bound", 0)
    peak_tops = 148 * 128 * sm_mhz * 1e6 / 1e12
    tops = evaluated * EVAL_OPS[sign] / prop_s / 1e12 if prop_s > 0 else 0.0
    return {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
            "traffic": PROPAGATE_DRAM_BYTES, "traffic_ratio": PROPAGATE_DRAM_BYTES / algo,
            "traffic_source": PROPAGATE_DRAM_SOURCE, "algorithmic_bytes": algo,
            "implementation_bytes": impl, "implementation_gbs": impl / prop_s / 1e9 if prop_s > 0 else 0.0,
            "kernel": "k_propagate (propagation rounds)", "peak_source": peak_source,
            "fp32": {"proposals": stats["neighbour_evals"], "evaluated": evaluated,
                     "ops_per_evaluation": EVAL_OPS[sign], "achieved_tops": tops, "peak_tops": peak_tops,
                     "frac": tops / peak_tops, "proposals_per_s": stats["neighbour_evals"] / prop_s},
            "phase_ms": phases, "stats": stats}


def workload():
    from mesh_to_sdf_b200 import synth

    v, idx = synth.star(6, seed=SEED)
    lo, hi = synth.padded_bbox(v, 0.1)
    return v, idx, lo, hi


def grid_for(lo, hi, n=(GRID_N, GRID_N, GRID_N)):
    import mesh_to_sdf_b200 as m2s

    return m2s.Grid.from_bounding_box(lo, hi, list(n))


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons every 20 ms.  Started
    before the timed region (nvidia-smi needs a moment to print its first
    row); summary() keeps the rows that arrived inside [t0, t1]."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None
        self.t0, self.t1 = 0.0, float("inf")

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            deadline = time.perf_counter() + 5.0
            while not self.rows and time.perf_counter() < deadline:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append((time.perf_counter(), [x.strip() for x in line.split(",")]))

    def mark_start(self):
        self.t0 = time.perf_counter()

    def mark_end(self):
        self.t1 = time.perf_counter() + 0.025  # a row printed at the end arrives a moment later

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = [r for t, r in self.rows if self.t0 <= t <= self.t1]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    """One process per GPU (replicas): NCCL on GPUs; gloo where there is no
    GPU, so the launch and the max-over-ranks plumbing run on CPU too."""
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        timeout = datetime.timedelta(seconds=120)
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            torch.distributed.init_process_group("nccl", timeout=timeout, device_id=torch.device("cuda", local))
        else:
            torch.distributed.init_process_group("gloo", timeout=timeout)
    return world, rank, local


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch

    dev = "cuda" if torch.distributed.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    import torch

    if world > 1:
        torch.distributed.barrier()
    if torch.cuda.is_available():
        torch.cuda.synchronize()


# --------------------------------------------------------------------------- CPU baseline
def cpu_slab(grid):
    """A bounded sample of the same grid: the 32 middle z-layers (1/8 of the cells), same cells."""
    import mesh_to_sdf_b200 as m2s

    nz = 32
    z0 = GRID_N // 2 - nz // 2
    first = grid.first_cell.copy()
    first[2] = np.float32(grid.first_cell[2] + np.float32(z0) * grid.cell_size[2])
    return m2s.Grid.new(first, grid.cell_size, [GRID_N, GRID_N, nz])


def run_cpu_grid(v, idx, g, threads):
    import oracle

    t = time.perf_counter()
    oracle.generate_grid_sdf(v, idx, g.first_cell, g.cell_size, g.cell_count, "raycast", n_threads=threads)
    return time.perf_counter() - t


def fp64_report(v, idx, points, values, threads, strip=False, raycast_sign=True, diag=None, ref64=None):
    """Error of f32 results against an FP64 brute force at the same points
    (reported, not timed): max / RMS of | |value| - d64 |, the max relative to
    the bounding-box diagonal, and — for Raycast-signed results — sign
    mismatches against the FP64 3-ray vote, those within 1e-5 of the diagonal
    of the surface counted apart as ambiguous."""
    import oracle

    d64, inside64 = ref64 if ref64 is not None else oracle.generate_sdf_f64(v, idx, points, strip=strip,
                                                                             n_threads=threads)
    if diag is None:
        lo, hi = synth_bbox(v)
        diag = float(np.linalg.norm(hi - lo))
    vals = np.asarray(values, np.float32)
    err = np.abs(np.abs(vals.astype(np.float64)) - d64)
    out = {"sample": int(len(points)), "max_err": float(err.max()) if len(err) else 0.0,
           "rms_err": float(np.sqrt(np.mean(err ** 2))) if len(err) else 0.0,
           "max_err_rel_bbox_diag": float(err.max() / diag) if len(err) else 0.0}
    if raycast_sign:
        flip = np.signbit(vals) != inside64
        near = d64 <= 1e-5 * diag
        out["sign_mismatch"] = int((flip & ~near).sum())
        out["sign_mismatch_ambiguous"] = int((flip & near).sum())
    return out


def sample_cells(grid, n, seed):
    """n seeded distinct cells of the grid and their centres (grid.rs:135-141 arithmetic)."""
    nx, ny, nz = (int(c) for c in grid.cell_count)
    rng = np.random.default_rng(seed)
    cells = rng.choice(nx * ny * nz, min(n, nx * ny * nz), replace=False)
    ijk = np.stack([cells // (ny * nz), (cells // nz) % ny, cells % nz], axis=1)
    centres = (grid.first_cell.astype(np.float32) + ijk.astype(np.float32) * grid.cell_size.astype(np.float32))
    return cells, centres.astype(np.float32)


def approx_eq_band(a, b):
    """float-cmp's approx_eq!(f32, a, b, ulps = 2, epsilon = 1e-6) on
    non-negative magnitudes (lib.rs:321): within 1e-6, or at most 2 ulps apart."""
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    ulps = np.abs(a.view(np.uint32).astype(np.int64) - b.view(np.uint32).astype(np.int64))
    return (np.abs(a.astype(np.float64) - b.astype(np.float64)) <= np.float32(1e-6)) | (ulps <= 2)


def grid_vs_restatement(gpu, ref, cell_diag, threads):
    """Cells whose value or sign differ between the GPU grid and the
    restatement's.  The reference's propagation is order-dependent, so values
    may differ where triangles compete; a sign difference means the two sides
    hold different triangles there (the same triangle gives the same signed
    value), split by how their distances compare: the same bits, inside
    compare_distances' tie band (lib.rs:315-332), or apart (a different
    triangle won through the propagation order)."""
    ga, ra = np.abs(gpu), np.abs(ref)
    differ = ga.view(np.uint32) != ra.view(np.uint32)
    flip = np.signbit(gpu) != np.signbit(ref)
    fa_, fr = ga[flip], ra[flip]
    same = fa_.view(np.uint32) == fr.view(np.uint32)
    band = ~same & approx_eq_band(fa_, fr)
    order = ~same & ~band
    gap = np.abs(fa_[order].astype(np.float64) - fr[order]) / cell_diag
    return {"cells": int(len(gpu)), "value_differs": int(differ.sum()), "value_differs_frac": float(differ.mean()),
            "max_value_diff_cell_diagonals": float(np.abs(ga.astype(np.float64) - ra).max() / cell_diag),
            "sign_differs": int(flip.sum()), "sign_differs_same_distance": int(same.sum()),
            "sign_differs_tie_band": int(band.sum()), "sign_differs_order": int(order.sum()),
            "sign_differs_order_max_gap_cell_diagonals": float(gap.max()) if len(gap) else 0.0,
            "threads": threads}


def grid_accuracy(v, idx, grid, gpu, threads, sign="raycast", strip=False, n_sample=10_000, ref=None):
    """Accuracy of a GPU grid (reported, not timed): against the restatement's
    own grid on all host threads, and against an FP64 brute force on seeded
    sample cells — beside the restatement's own FP64 error on the same cells,
    which shows what the reference's propagation itself gives up there."""
    import oracle

    t0 = time.perf_counter()
    if ref is None:
        ref = oracle.generate_grid_sdf(v, idx, grid.first_cell, grid.cell_size, grid.cell_count, sign, strip=strip,
                                       n_threads=threads)
    ref_s = time.perf_counter() - t0
    cell_diag = float(np.linalg.norm(grid.cell_size.astype(np.float64)))
    cells, centres = sample_cells(grid, n_sample, SEED + 3)
    raycast = sign == "raycast"
    gpu_err = fp64_report(v, idx, centres, gpu[cells], threads, strip=strip, raycast_sign=raycast)
    ref_err = fp64_report(v, idx, centres, ref[cells], threads, strip=strip, raycast_sign=raycast)
    return {"restatement": grid_vs_restatement(gpu, ref, cell_diag, threads),
            "fp64": {"gpu": gpu_err, "restatement": ref_err}}, ref_s


ORACLE_ACCEL = {0: "none", 1: "bvh", 2: "rtree", 3: "rtree_bvh"}


def point_accuracy(v, idx, q, outs, points, threads, n_parity=50_000, n_fp64=20_000, strip=False):
    """Point results against the oracle and FP64 (reported, not timed): every
    LBVH method on a seeded sample of `n_parity` of its points, the brute
    force (None) on all of its points — bit for bit; and each method's FP64
    max / RMS error on a seeded sample of `n_fp64` points (the FP64 distances
    are computed once per sample and shared)."""
    import oracle

    rng = np.random.default_rng(SEED + 5)
    cache = {}
    for name, (am, gpu) in outs.items():
        n = len(gpu)
        if am.kind == 0:
            pick = np.arange(n)
        else:
            pick = np.sort(rng.choice(n, min(n_parity, n), replace=False))
        ref = oracle.generate_sdf(v, idx, q[pick], ORACLE_ACCEL[am.kind], int(am.sign), strip=strip,
                                  n_threads=threads)
        points[name]["parity"] = {"points": int(len(pick)),
                                  "bits_differ": int(np.sum(gpu[pick].view(np.uint32) != ref.view(np.uint32))),
                                  "against": "oracle (C++ restatement), bit for bit"}
        key = min(n, N_BRUTE) if am.kind == 0 else n
        if key not in cache:
            sel = np.sort(np.random.default_rng(SEED + 6).choice(key, min(n_fp64, key), replace=False))
            cache[key] = (sel, oracle.generate_sdf_f64(v, idx, q[sel], strip=strip, n_threads=threads))
        sel, ref64 = cache[key]
        raycast = int(am.sign) == 0 and am.kind != 2  # Rtree signs by the normal
        points[name]["fp64"] = fp64_report(v, idx, q[sel], gpu[sel], threads, strip=strip, raycast_sign=raycast,
                                           ref64=ref64)


def synth_bbox(v):
    v = np.asarray(v, np.float64)
    return v.min(axis=0), v.max(axis=0)


def reference_workloads(args):
    """The CPU baseline of the other configurations: the oracle port (the
    reference's decomposition: parallel seeding, per-thread heaps and rays for
    grids; queries in parallel, RtreeBvh serially as the reference does) on the
    host cores, on bounded samples of each configuration.  One JSON line."""
    import oracle

    import mesh_to_sdf_b200 as m2s
    from mesh_to_sdf_b200 import synth

    cores = os.cpu_count() or 1

    def grid_rate(v, idx, g, sign, strip=False):
        t = time.perf_counter()
        oracle.generate_grid_sdf(v, idx, g.first_cell, g.cell_size, g.cell_count, sign, strip=strip, n_threads=cores)
        return g.get_total_cell_count() / (time.perf_counter() - t)

    def point_rate(v, idx, q, accel, sign="raycast", strip=False, threads=cores):
        t = time.perf_counter()
        oracle.generate_sdf(v, idx, q, accel, sign, strip=strip, n_threads=threads)
        return len(q) / (time.perf_counter() - t)

    out = {"impl": "reference", "workload": args.workload, "cores": cores, "kind": "port"}
    if args.workload == "c1":
        v, idx = synth.icosphere(3)
        g = m2s.Grid.from_bounding_box([-1.2] * 3, [1.2] * 3, [32, 32, 32])
        q = synth.uniform_points(10_000, [-1.2] * 3, [1.2] * 3, seed=SEED)
        out["grid_cells_per_s"] = grid_rate(v, idx, g, "raycast")
        out["rtree_bvh_points_per_s"] = point_rate(v, idx, q, "rtree_bvh", threads=1)  # serial in the reference
        out["sample"] = "the whole configuration"
    elif args.workload == "c3":
        v, idx = synth.terrain(512, seed=SEED)
        lo, hi = synth.padded_bbox(v, 0.1)
        g = m2s.Grid.from_bounding_box(lo, hi, [384, 384, 128])
        q = synth.uniform_points(200_000, lo, hi, seed=SEED)
        out["grid_cells_per_s"] = grid_rate(v, idx, g, "normal", strip=True)
        out["rtree_points_per_s"] = point_rate(v, idx, q, "rtree", "normal", strip=True)
        out["sample"] = "the whole grid; 200,000 of the 4M points"
    else:
        items = synth.batch_meshes(args.batch, seed=SEED)[::16]
        cells, t = 0, time.perf_counter()
        for v, i, lo, hi, e in items:
            g = m2s.Grid.from_bounding_box(lo, hi, [e, e, e])
            oracle.generate_grid_sdf(v, i, g.first_cell, g.cell_size, g.cell_count, "raycast", n_threads=cores)
            cells += g.get_total_cell_count()
        out["grid_cells_per_s"] = cells / (time.perf_counter() - t)
        out["sample"] = f"every 16th of the {args.batch} meshes ({len(items)} grids, {cells} cells), one call each"
    print(json.dumps(out), flush=True)


def c2_point_baseline(cores):
    """The C2 point methods on the host cores (oracle port; samples)."""
    import oracle

    from mesh_to_sdf_b200 import synth

    v, idx, lo, hi = workload()
    q = synth.mixed_points(v, idx, 100_000, seed=SEED)
    res = {}
    for name, accel, sign, n in (("bvh_raycast", "bvh", "raycast", 100_000), ("rtree", "rtree", "normal", 100_000),
                                 ("none_raycast", "none", "raycast", 1_000), ("none_normal", "none", "normal", 1_000)):
        t = time.perf_counter()
        oracle.generate_sdf(v, idx, q[:n], accel, sign, n_threads=cores)
        res[name] = {"points": n, "points_per_s": n / (time.perf_counter() - t)}
    return res


def reference_arm(args, world, rank):
    """The reference's CPU path (its C++ restatement; cargo is not on this image), all host cores.
    Every timed step is the whole 256^3 grid of the GPU arm's configuration;
    the warm-up steps run its 256x256x32 middle slab (they only warm the host),
    which keeps the run within a few minutes."""
    if rank != 0:
        return
    v, idx, lo, hi = workload()
    grid = grid_for(lo, hi)
    slab = cpu_slab(grid)
    cores = os.cpu_count() or 1
    points = c2_point_baseline(cores)
    for _ in range(args.warmup):
        run_cpu_grid(v, idx, slab, cores)
    ts = [run_cpu_grid(v, idx, grid, cores) for _ in range(args.steps)]
    sec = float(np.mean(ts))
    N = grid.get_total_cell_count()
    value = N / sec
    line = {"impl": "reference", "metric": "SDF cells/s (generate_grid_sdf, Raycast)", "value": value,
            "unit": "cells/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded star icosphere s6, 81,920 triangles)",
            "config": reference_config(len(idx) // 3),
            "cpu_baseline": {"value": value, "unit": "cells/s", "cores": cores, "kind": "port",
                             "sample": "the whole 256^3 grid per timed step (warm-up steps: its 256x256x32 "
                                       "middle slab)"},
            "e2e": {"value": value, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "points": points}
    print(json.dumps(line), flush=True)


def reference_config(n_tris):
    """The configuration both arms report: the workload and its sizes."""
    return {"workload": "star_s6_grid256_raycast", "grid": [GRID_N] * 3, "triangles": n_tris, "sign": "Raycast"}


# --------------------------------------------------------------------------- GPU arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-points", action="store_true")
    ap.add_argument("--no-workloads", action="store_true",
                    help="leave the bounded c1 / c3 / c4 / c5 entries out of the default line")
    ap.add_argument("--small", action="store_true",
                    help="one short pass for profilers: one grid, 100k Rtree / RtreeBvh points, 8k brute-force points")
    ap.add_argument("--grid", type=int, default=128, help="grid edge of the --small pass")
    ap.add_argument("--points", type=int, default=100_000, help="query points of the --small pass")
    ap.add_argument("--bound-filter", action="store_true",
                    help="--small: run the grid with the filtered propagation variant (same results)")
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c4", "c5"],
                    help="c2 (default): the headline line; c1 / c3: the small and the terrain configurations; "
                         "c4: 256 grids batched in one plan against 256 single-grid calls; "
                         "c5: the serving loop under Poisson arrivals at swept rates")
    ap.add_argument("--rates", default="50,100,200,400", help="c5 arrival rates, requests/s")
    ap.add_argument("--requests", type=int, default=200, help="c5 requests per rate")
    ap.add_argument("--batch", type=int, default=256, help="meshes of the c4 batch")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--wave-cells", type=int, default=0, help="c4: cells per batched job (0 = the library default)")
    args = ap.parse_args()
    if args.small:
        return small_case(args.grid, args.points, args.bound_filter)
    if args.impl == "reference" and args.workload in ("c1", "c3", "c4"):
        return reference_workloads(args)
    if args.workload == "c4":
        return batch_workload(args)
    if args.workload == "c5":
        return serving_workload(args)
    if args.workload != "c2":
        return other_workload(args)
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup

    world, rank, local = dist_setup()
    if args.impl == "reference":
        reference_arm(args, world, rank)
        if world > 1:
            torch_destroy()
        return

    import torch

    import mesh_to_sdf_b200 as m2s
    from mesh_to_sdf_b200 import synth

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    v, idx, lo, hi = workload()
    grid = grid_for(lo, hi)
    N = grid.get_total_cell_count()
    T = len(idx) // 3
    A, S = m2s.AccelerationMethod, m2s.SignMethod
    mesh = m2s.build_sdf_acceleration(v, m2s.Topology.TriangleList(idx), A.none(S.Raycast))
    out = torch.empty(N, dtype=torch.float32, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2
    stream = torch.cuda.current_stream().cuda_stream

    def step():
        mesh.grid_device(grid, S.Raycast, out, status, stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    assert int(status.item()) == 0, f"device status {int(status.item())}"

    # ---- timed region: K steps, L2 flushed between steps (untimed), device events per step
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier(world)
    with ClockSampler(local) as clk:
        clk.mark_start()
        t_wall = time.perf_counter()
        for i in range(args.steps):
            flush.fill_(i & 0xFF)
            ev[i][0].record()
            step()
            ev[i][1].record()
        torch.cuda.synchronize()
        t_wall = time.perf_counter() - t_wall
        clk.mark_end()
    barrier(world)
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = max_over_ranks(float(np.sum(step_ms)), world)
    launches = m2s.last_grid_stats()["kernel_launches"] * args.steps
    ms_per_step = total_ms / args.steps
    value = world * N * args.steps / (total_ms / 1e3)
    assert int(status.item()) == 0

    # ---- roofline of the dominant phase: propagation (k_propagate), profiled on the same stream
    m2s.set_profiling(True)
    flush.fill_(1)
    step()
    torch.cuda.synchronize()
    m2s.set_profiling(False)
    phases = m2s.last_grid_phase_ms()
    stats = m2s.last_grid_stats()
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    roofline = grid_roofline(N, len(v), T, phases, stats, hbm_peak, "measured" if peaks else "fallback",
                             float(peaks.get("sm_max_mhz", 1965.0)), "raycast")
    # the filtered propagation variant on the same grid (untimed beside the
    # step; results are identical), and the FP64 audit of the grid's f32
    # decisions (counts only)
    m2s.set_grid_bound_filter(True)
    m2s.set_profiling(True)
    flush.fill_(1)
    step()
    torch.cuda.synchronize()
    m2s.set_profiling(False)
    m2s.set_grid_bound_filter(False)
    fst = m2s.last_grid_stats()
    roofline["filter_variant"] = {"propagation_ms": m2s.last_grid_phase_ms()["propagation"],
                                  "proposals": fst["neighbour_evals"], "dropped_same": fst["dropped_same"],
                                  "dropped_bound": fst["dropped_bound"]}
    m2s.set_fp64_audit(True)
    step()
    torch.cuda.synchronize()
    m2s.set_fp64_audit(False)
    grid_audit = m2s.last_grid_audit()
    assert int(status.item()) == 0

    # ---- e2e: the host-pointer C ABI with pinned buffers, H2D + D2H inside the timed region
    vh = torch.from_numpy(np.ascontiguousarray(v)).pin_memory().numpy()
    ih = torch.from_numpy(np.ascontiguousarray(idx.view(np.int32))).pin_memory().numpy().view(np.uint32)
    oh = torch.empty(N, dtype=torch.float32).pin_memory().numpy()
    import ctypes

    L = m2s._lib.lib()
    first = np.ascontiguousarray(grid.first_cell)
    size = np.ascontiguousarray(grid.cell_size)
    count = np.array(grid.cell_count, np.uint64)
    nout = ctypes.c_uint64(0)

    def e2e_step():
        st = L.m2s_generate_grid_sdf(vh.ctypes.data, len(vh), ih.ctypes.data, len(ih), 32, 0, first.ctypes.data,
                                     size.ctypes.data, count.ctypes.data, 0, oh.ctypes.data, ctypes.byref(nout), None)
        assert st == 0, st

    for _ in range(2):
        e2e_step()
    barrier(world)
    e2e_times = []
    for i in range(args.steps):
        flush.fill_(i & 0xFF)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_step()
        e2e_times.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(float(np.sum(e2e_times)), world)
    e2e = {"value": world * N * args.steps / e2e_s, "unit": "cells/s", "h2d_bytes_per_step": int(vh.nbytes + ih.nbytes),
           "d2h_bytes_per_step": int(oh.nbytes)}
    assert np.array_equal(oh.view(np.uint32), out.cpu().numpy().view(np.uint32)), "e2e result differs from device path"

    # ---- point queries of the same configuration
    points, point_outs = {}, {}
    q_host = synth.mixed_points(v, idx, N_POINTS, seed=SEED)
    if not args.no_points:
        q = torch.from_numpy(q_host).to(dev)
        qo = torch.empty(N_POINTS, dtype=torch.float32, device=dev)
        # the library's query autotuner picks the node budget (one thread per
        # query, then one warp) on the Bvh+Raycast batch; the process-wide
        # budget it sets is put back after these lines, so later entries
        # start from the library default
        saved_budget = m2s._lib.lib().m2s_query_budget()
        acc = m2s.build_sdf_acceleration(v, m2s.Topology.TriangleList(idx), A.bvh(S.Raycast))
        best_budget, tune = acc.autotune_queries(q, stream)
        acc.close()
        points["budget_sweep_ms"] = {str(k): round(v_, 3) for k, v_ in tune.items()}
        points["node_budget"] = best_budget
        for name, am, n in (("bvh_raycast", A.bvh(S.Raycast), N_POINTS), ("rtree", A.rtree(), N_POINTS),
                            ("rtree_bvh", A.rtree_bvh(), N_POINTS), ("none_raycast", A.none(S.Raycast), N_BRUTE),
                            ("none_normal", A.none(S.Normal), N_BRUTE)):
            acc = m2s.build_sdf_acceleration(v, m2s.Topology.TriangleList(idx), am)
            qq = q[:n].contiguous()
            for _ in range(2):
                acc.query_device(qq, qo, status, stream)
            torch.cuda.synchronize()
            reps = 3
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            flush.fill_(2)
            e0.record()
            for _ in range(reps):
                acc.query_device(qq, qo, status, stream)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps
            point_outs[name] = (am, qo[:n].cpu().numpy().copy())
            points[name] = {"points": n, "ms": ms, "pts_per_s": n / (ms / 1e3)}
            if name.startswith("none"):
                points[name]["pairs_per_s"] = n * T / (ms / 1e3)
            else:  # traversal counts per query and the FP64 audit, from one untimed run
                m2s.set_profiling(True)
                m2s.set_fp64_audit(True)
                acc.query_device(qq, qo, status, stream)
                torch.cuda.synchronize()
                qs = m2s.last_query_stats()
                points[name]["fp64_audit"] = m2s.last_query_audit()
                m2s.set_fp64_audit(False)
                m2s.set_profiling(False)
                points[name]["per_query"] = {k[:-len("_per_query")]: round(v_, 2) for k, v_ in qs.items()
                                             if k.endswith("_per_query")}
            acc.close()
        m2s._lib.lib().m2s_set_query_budget(saved_budget)
        assert int(status.item()) == 0

    # ---- result-side rows on this grid and mesh: the viewer's distance-ordered
    # cell list (device arrays) and the watertightness check (host arrays)
    results = {}
    if not args.no_points:
        order = torch.empty(N, dtype=torch.int32, device=dev)
        mm = torch.empty(2, dtype=torch.float32, device=dev)
        m2s.sort_cells_by_distance_device(out, order, mm, stream)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        flush.fill_(3)
        e0.record()
        for _ in range(3):
            m2s.sort_cells_by_distance_device(out, order, mm, stream)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 3
        results["cell_order"] = {"cells": N, "ms": ms, "cells_per_s": N / (ms / 1e3)}
        m2s.check_mesh_triangle_list(v, idx)
        t0 = time.perf_counter()
        verdict = m2s.check_mesh_triangle_list(v, idx)
        results["mesh_check"] = {"faces": T, "ms_host_to_verdict": (time.perf_counter() - t0) * 1e3,
                                 "watertight": verdict is None}

    # ---- CPU baseline (rank 0, N = 1 only): the oracle port on a bounded sample
    cpu = accuracy = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores = os.cpu_count() or 1
        # the restatement's whole 256^3 grid on all host threads: timed as the
        # CPU baseline, and compared with the GPU grid
        accuracy, ref_s = grid_accuracy(v, idx, grid, out.cpu().numpy(), cores)
        cpu = {"value": N / ref_s, "unit": "cells/s", "cores": cores, "kind": "port",
               "sample": "the whole 256^3 grid once, C++ restatement, all host threads"}
        point_accuracy(v, idx, q_host, point_outs, points, cores)

    # ---- the other configurations, bounded (rank 0, one GPU): each with its
    # own CPU baseline and accuracy figures
    workloads = {}
    if rank == 0 and world == 1 and not args.no_workloads:
        mesh.close()
        acc_on = not args.no_cpu_baseline
        jobs = (("c1", lambda: small_or_terrain_entry("c1", 5, 3, acc_on, peaks)),
                ("c3", lambda: small_or_terrain_entry("c3", 3, 2, acc_on, peaks)),
                ("c4", lambda: batch_entry(256, 2, True, 0, acc_on, cpu_every=32)),
                ("c5", lambda: serving_entry((100.0, 400.0), 200, True)))
        for name, fn in jobs:
            t0 = time.perf_counter()
            try:
                workloads[name] = fn()
            except Exception as e:  # reported in the line; the headline stands
                workloads[name] = {"error": f"{type(e).__name__}: {e}"}
            workloads[name]["wall_s"] = round(time.perf_counter() - t0, 1)

    if rank == 0:
        line = {"metric": "SDF cells/s (generate_grid_sdf, Raycast)", "value": value, "unit": "cells/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded star icosphere s6, 81,920 triangles)",
                "config": {**reference_config(T), "parallelism": f"replicas x{world}",
                           "l2": "flushed between steps (256 MiB write, untimed)"},
                "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "gpu_launches": int(launches),
                "clocks": clk.summary(), "points": points, "results": results, "accuracy": accuracy,
                "fp64_audit": grid_audit,
                "workloads": workloads, "wall_s_timed": t_wall}
        print(json.dumps(line), flush=True)
    if not workloads:
        mesh.close()
    if world > 1:
        torch_destroy()


def small_or_terrain_entry(which, steps=5, warmup=3, accuracy=True, peaks=None):
    """c1: icosphere s3, 32^3 Raycast grid over [-1.2, 1.2]^3, 10,000 RtreeBvh
    points.  c3: 512 x 512 fBm terrain as one TriangleStrip, 384 x 384 x 128
    Normal grid over the 10 %-padded bbox, 4M uniform Rtree points.  Returns
    one dict: GPU rates, the propagation roofline, and (accuracy=True) the
    restatement's grid and the oracle's points on the host cores — both the
    accuracy checks and the CPU baseline of this configuration."""
    import torch

    import mesh_to_sdf_b200 as m2s
    from mesh_to_sdf_b200 import synth

    A, S = m2s.AccelerationMethod, m2s.SignMethod
    strip = which == "c3"
    if which == "c1":
        v, idx = synth.icosphere(3)
        topo = m2s.Topology.TriangleList(idx)
        grid = m2s.Grid.from_bounding_box([-1.2] * 3, [1.2] * 3, [32, 32, 32])
        sign, am, npts = S.Raycast, A.rtree_bvh(), 10_000
        q = synth.uniform_points(npts, [-1.2] * 3, [1.2] * 3, seed=SEED)
    else:
        v, idx = synth.terrain(512, seed=SEED)
        topo = m2s.Topology.TriangleStrip(idx)
        lo, hi = synth.padded_bbox(v, 0.1)
        grid = m2s.Grid.from_bounding_box(lo, hi, [384, 384, 128])
        sign, am, npts = S.Normal, A.rtree(), 4_000_000
        q = synth.uniform_points(npts, lo, hi, seed=SEED)
    N = grid.get_total_cell_count()
    mesh = m2s.build_sdf_acceleration(v, topo, am)
    out = torch.empty(N, dtype=torch.float32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for _ in range(max(warmup, 1)):
        mesh.grid_device(grid, sign, out, status)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for i in range(steps):
        flush.fill_(i & 0xFF)
        ev[i][0].record()
        mesh.grid_device(grid, sign, out, status)
        ev[i][1].record()
    torch.cuda.synchronize()
    gms = float(np.mean([a.elapsed_time(b_) for a, b_ in ev]))
    m2s.set_profiling(True)
    flush.fill_(1)
    mesh.grid_device(grid, sign, out, status)
    torch.cuda.synchronize()
    m2s.set_profiling(False)
    phases, stats = m2s.last_grid_phase_ms(), m2s.last_grid_stats()
    m2s.set_fp64_audit(True)
    mesh.grid_device(grid, sign, out, status)
    torch.cuda.synchronize()
    m2s.set_fp64_audit(False)
    grid_audit = m2s.last_grid_audit()
    peaks = peaks or {}
    sname = "raycast" if int(sign) == 0 else "normal"
    roof = grid_roofline(N, len(v), mesh.triangle_count, phases, stats, float(peaks.get("hbm_gbs", 6650.0)),
                         "measured" if peaks else "fallback", float(peaks.get("sm_max_mhz", 1965.0)), sname)
    for k in ("traffic", "traffic_ratio", "traffic_source", "stats", "phase_ms"):
        roof.pop(k)  # the ncu traffic figure belongs to the bench grid
    qd = torch.from_numpy(q).cuda()
    qo = torch.empty(npts, dtype=torch.float32, device="cuda")
    # the library's query autotuner, on these points; the process-wide budget
    # it sets is put back below, so it does not carry over to other entries
    saved_budget = m2s._lib.lib().m2s_query_budget()
    budget, _ = mesh.autotune_queries(qd)
    for _ in range(2):
        mesh.query_device(qd, qo, status)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    mesh.query_device(qd, qo, status)
    e1.record()
    torch.cuda.synchronize()
    qms = e0.elapsed_time(e1)
    m2s.set_fp64_audit(True)
    mesh.query_device(qd, qo, status)
    torch.cuda.synchronize()
    m2s.set_fp64_audit(False)
    points_audit = m2s.last_query_audit()
    m2s._lib.lib().m2s_set_query_budget(saved_budget)
    assert int(status.item()) == 0, int(status.item())
    line = {"workload": which, "triangles": mesh.triangle_count, "grid": [int(c) for c in grid.cell_count],
            "sign": sign.name, "grid_ms": gms, "cells_per_s": N / (gms / 1e3), "grid_phase_ms": phases,
            "grid_stats": stats, "roofline": roof, "points": npts, "method": repr(am), "points_ms": qms,
            "pts_per_s": npts / (qms / 1e3), "node_budget": budget,
            "fp64_audit": {"grid": grid_audit, "points": points_audit}}
    mesh.close()
    if accuracy:
        import oracle

        threads = os.cpu_count() or 1
        gpu_grid, gpu_pts = out.cpu().numpy(), qo.cpu().numpy()
        acc, ref_s = grid_accuracy(v, idx, grid, gpu_grid, threads, sname, strip,
                                   n_sample=10_000 if which == "c1" else 2_000)
        pts = {which: {"points": npts}}
        point_accuracy(v, idx, q, {which: (am, gpu_pts)}, pts, threads,
                       n_parity=10_000 if which == "c1" else 50_000, n_fp64=10_000 if which == "c1" else 2_000,
                       strip=strip)
        acc["points"] = pts[which]
        line["accuracy"] = acc
        # the CPU baseline of this configuration: the restatement's grid above,
        # and its points (RtreeBvh: a serial loop, as in the reference)
        ncpu = npts if which == "c1" else 200_000
        t0 = time.perf_counter()
        oracle.generate_sdf(v, idx, q[:ncpu], ORACLE_ACCEL[am.kind], int(am.sign), strip=strip,
                            n_threads=1 if am.kind == 3 else threads)
        pt_s = time.perf_counter() - t0
        line["cpu_baseline"] = {"cells_per_s": N / ref_s, "points_per_s": ncpu / pt_s, "cores": threads,
                                "kind": "port",
                                "sample": f"the whole grid; {ncpu} of the {npts} points"
                                          + (" (RtreeBvh: one thread, as the reference's serial loop)"
                                             if am.kind == 3 else "")}
    return line


def other_workload(args):
    print(json.dumps(small_or_terrain_entry(args.workload, args.steps, args.warmup, not args.no_cpu_baseline,
                                            load_peaks())), flush=True)


def load_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def batch_entry(n_meshes=256, steps=3, autotune=True, wave_cells=0, accuracy=True, cpu_every=16):
    """c4: `n_meshes` displaced spheres (subdivision 2..6, scale U[0.5, 2],
    random rotation) with cubic Raycast grids of edge 32..192 over their
    padded boxes, all resident.  Times one pass of single-grid calls (one per
    mesh: the plain path) against the same grids as one batched plan replayed
    from its CUDA graph, after checking that both give the same bits.  With
    accuracy: FP64 errors on sample cells of every 16th grid, and the CPU
    baseline (the restatement, one generate_grid_sdf call per mesh, on every
    `cpu_every`-th mesh).  Returns one dict."""
    import torch

    import mesh_to_sdf_b200 as m2s
    from mesh_to_sdf_b200 import synth

    A, S = m2s.AccelerationMethod, m2s.SignMethod
    items = synth.batch_meshes(n_meshes, seed=SEED)
    meshes = [m2s.build_sdf_acceleration(v, m2s.Topology.TriangleList(i), A.none(S.Raycast)) for v, i, *_ in items]
    grids = [m2s.Grid.from_bounding_box(lo, hi, [e, e, e]) for _, _, lo, hi, e in items]
    off = m2s.grid_offsets(grids)
    N = int(off[-1])
    tris = sum(m.triangle_count for m in meshes)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    plain = torch.empty(N, dtype=torch.float32, device="cuda")
    views = [plain[int(off[k]):int(off[k + 1])] for k in range(len(grids))]

    def plain_pass():
        for m, g, o in zip(meshes, grids, views):
            m.grid_device(g, S.Raycast, o, status)

    def plain_by_edge():
        """Device time of the single-grid calls, summed per grid edge."""
        per = {}
        for m, g, o, it in zip(meshes, grids, views, items):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            m.grid_device(g, S.Raycast, o, status)
            b.record()
            b.synchronize()
            e = it[4]
            n_, t_ = per.get(e, (0, 0.0))
            per[e] = (n_ + 1, t_ + a.elapsed_time(b))
        return {str(e): {"grids": n_, "ms": round(t_, 2)} for e, (n_, t_) in sorted(per.items())}

    def timed(fn, k):
        ms = []
        for _ in range(k):
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        return float(np.median(ms))

    plain_pass()
    plain_ms = timed(plain_pass, max(1, min(steps, 3)))
    per_edge = plain_by_edge()
    batched = torch.empty(N, dtype=torch.float32, device="cuda")
    if wave_cells:
        m2s.set_grid_tuning(wave_cells=wave_cells)
    plan = m2s.GridPlan(meshes, grids, S.Raycast, batched, status)
    blocks0 = plan.blocks
    plan.run()
    t0 = time.time()
    chosen = plan.autotune() if autotune else blocks0
    tune_s = time.time() - t0
    plan.run()
    stats = m2s.last_grid_stats()
    batch_ms = timed(plan.run, max(3, steps))
    diff = plain.view(torch.int32) != batched.view(torch.int32)
    ndiff = int(diff.sum().item())
    same = ndiff == 0
    bad_grids = [k for k in range(len(grids)) if bool(diff[int(off[k]):int(off[k + 1])].any().item())] if ndiff else []
    assert int(status.item()) == 0, int(status.item())
    line = {"workload": "c4_batch", "grids": len(grids), "cells": N, "triangles": tris,
            "plain_ms": plain_ms, "plain_cells_per_s": N / (plain_ms / 1e3),
            "batched_ms": batch_ms, "batched_cells_per_s": N / (batch_ms / 1e3),
            "speedup": plain_ms / batch_ms, "bit_identical": same, "cells_differing": ndiff,
            "grids_differing": bad_grids[:16], "waves": plan.waves, "plain_ms_by_edge": per_edge,
            "blocks_default": blocks0, "blocks_autotuned": chosen, "autotune_s": tune_s,
            "plan_device_gb": plan.device_bytes / 1e9, "grid_stats": stats}
    plan.close()
    if wave_cells:
        m2s.set_grid_tuning()
    if accuracy:
        import oracle

        threads = os.cpu_count() or 1
        host = batched.cpu().numpy()
        errs = []
        for k in range(0, len(grids), 16):
            v, i = items[k][:2]
            cells, centres = sample_cells(grids[k], 500, SEED + 100 + k)
            vals = host[int(off[k]):int(off[k + 1])][cells]
            errs.append(fp64_report(v, i, centres, vals, threads))
        worst = max(errs, key=lambda e: e["max_err_rel_bbox_diag"])
        line["accuracy"] = {"fp64": {"grids": len(errs), "sample_cells_per_grid": 500,
                                     "max_err_rel_bbox_diag": worst["max_err_rel_bbox_diag"],
                                     "max_err": max(e["max_err"] for e in errs),
                                     "rms_err": float(np.sqrt(np.mean([e["rms_err"] ** 2 for e in errs]))),
                                     "sign_mismatch": sum(e["sign_mismatch"] for e in errs),
                                     "sign_mismatch_ambiguous": sum(e["sign_mismatch_ambiguous"] for e in errs)}}
        sub = items[::cpu_every]
        cells, t0 = 0, time.perf_counter()
        for v, i, lo, hi, e in sub:
            g = m2s.Grid.from_bounding_box(lo, hi, [e, e, e])
            oracle.generate_grid_sdf(v, i, g.first_cell, g.cell_size, g.cell_count, "raycast", n_threads=threads)
            cells += g.get_total_cell_count()
        line["cpu_baseline"] = {"cells_per_s": cells / (time.perf_counter() - t0), "cores": threads, "kind": "port",
                                "sample": f"every {cpu_every}th of the {n_meshes} meshes ({len(sub)} grids, "
                                          f"{cells} cells), one generate_grid_sdf call each"}
    for m in meshes:
        m.close()
    return line


def batch_workload(args):
    line = batch_entry(args.batch, args.steps, not args.no_autotune, args.wave_cells, not args.no_cpu_baseline)
    print(json.dumps(line), flush=True)
    if not line["bit_identical"]:
        raise SystemExit("batched grids differ from single-grid calls")


def serving_entry(rates=(50.0, 100.0, 200.0, 400.0), n_req=200, plain=True):
    """c5: a server with a 120 GB device-memory budget and 64 resident meshes
    of the batched-grid kind (RtreeBvh), fed Poisson arrivals at each rate:
    5 % uploads of new meshes (built on the GPU), 60 % point requests (Q
    log-uniform in [1e3, 1e6], uniform in the mesh's padded box), 40 % Raycast
    grid requests (edge log-uniform in [64, 256] over the padded box).  Host
    buffers are pinned.  Latency is arrival to completion.  With `plain`, the
    same arrivals also go through the plain path — one library call per
    request (query_sdf, a resident-mesh grid call with its copies, or
    build_sdf_acceleration), served in arrival order by one host thread — and
    both arms report p50 / p99 and aggregate cells/s and points/s.  Point
    requests use the process-wide node budget as found (the library default
    unless a caller set one; the entries above restore theirs).  Returns one
    dict."""
    import torch

    import mesh_to_sdf_b200 as m2s
    from mesh_to_sdf_b200 import synth

    A, S = m2s.AccelerationMethod, m2s.SignMethod
    srv = m2s.Server(120 * 10**9, point_streams=4)
    resident = synth.batch_meshes(64, seed=SEED + 5)
    fresh = synth.batch_meshes(32, seed=SEED + 6)
    ids = []
    for v, i, *_ in resident:
        mid, t = srv.submit_upload(v, m2s.Topology.TriangleList(i), A.rtree_bvh())
        ids.append((mid, t))
    for mid, t in ids:
        assert srv.wait(t)[0] == 0
    boxes = [(lo, hi) for _, _, lo, hi, _ in resident]
    ids = [mid for mid, _ in ids]
    rng = np.random.default_rng(SEED + 7)
    unit = torch.from_numpy(rng.random((1_000_000, 3), dtype=np.float32)).pin_memory()
    # Warm-up, untimed: every kernel loaded once and the memory pool grown to
    # its working size (a pool growth may synchronise the device), as a
    # server does before it takes traffic.
    wq = unit.numpy()
    wg = torch.empty(256 ** 3, dtype=torch.float32).pin_memory().numpy()
    wp = torch.empty(len(wq), dtype=torch.float32).pin_memory().numpy()
    for j, e in enumerate((64, 96, 128, 192, 256, 256)):
        lo, hi = boxes[j]
        warm = [srv.submit_grid(ids[j], m2s.Grid.from_bounding_box(lo, hi, [e, e, e]), S.Raycast, wg[:e ** 3]),
                srv.submit_points(ids[j], wq, wp)]
        for t in warm:
            assert srv.wait(t)[0] == 0
    plain_meshes = []
    if plain:
        plain_meshes = [m2s.build_sdf_acceleration(v, m2s.Topology.TriangleList(i), A.rtree_bvh())
                        for v, i, *_ in resident]
        dev_grid = torch.empty(256 ** 3, dtype=torch.float32, device="cuda")
        for j, e in enumerate((64, 256)):
            g = m2s.Grid.from_bounding_box(*boxes[j], [e, e, e])
            plain_meshes[j].grid_device(g, S.Raycast, dev_grid[:e ** 3])
            m2s.query_sdf(plain_meshes[j], wq[:1000])
        torch.cuda.synchronize()

    def pct(a, p):
        return round(float(np.percentile(a, p)) * 1e3, 3) if len(a) else None

    def summary(lat, work, span):
        allv = np.array(sum(lat.values(), []))
        return {"span_s": round(span, 3), "achieved_rps": round(n_req / span, 1),
                "p50_ms": pct(allv, 50), "p99_ms": pct(allv, 99),
                "cells_per_s": work["grid"] / span, "points_per_s": work["points"] / span,
                "points": {"n": len(lat["points"]), "p50_ms": pct(lat["points"], 50), "p99_ms": pct(lat["points"], 99)},
                "grid": {"n": len(lat["grid"]), "p50_ms": pct(lat["grid"], 50), "p99_ms": pct(lat["grid"], 99)},
                "upload": {"n": len(lat["upload"]), "p50_ms": pct(lat["upload"], 50),
                           "p99_ms": pct(lat["upload"], 99)}}

    lines = []
    fresh_next = 0
    for rate in rates:
        # the stream: kinds, sizes, arrival times
        kinds = rng.choice(3, size=n_req, p=[0.05, 0.95 * 0.60, 0.95 * 0.40])
        arrivals = np.cumsum(rng.exponential(1.0 / rate, n_req))
        reqs, out_elems = [], 0
        for k in kinds:
            j = int(rng.integers(len(ids)))
            if k == 1:
                q = int(10 ** rng.uniform(3, 6))
                reqs.append(("points", j, q, out_elems))
                out_elems += q
            elif k == 2:
                e = int(round(2 ** rng.uniform(6, 8)))
                reqs.append(("grid", j, e, out_elems))
                out_elems += e ** 3
            else:
                reqs.append(("upload", fresh_next % len(fresh), 0, out_elems))
                fresh_next += 1
        out = torch.empty(out_elems, dtype=torch.float32).pin_memory()
        outn = out.numpy()
        # per-request query arrays: the pinned unit cube scaled into the mesh's box
        qbufs = {}
        for r_, (kind, j, n, o) in enumerate(reqs):
            if kind == "points":
                lo, hi = boxes[j]
                qbufs[r_] = (unit[:n] * torch.from_numpy(hi - lo) + torch.from_numpy(lo)).pin_memory().numpy()
        # ---- served: submissions at the arrival times, completions as the server records them
        tickets = []
        t0 = time.perf_counter()
        for r_, (kind, j, n, o) in enumerate(reqs):
            wait = t0 + arrivals[r_] - time.perf_counter()
            if wait > 0:
                time.sleep(wait)
            if kind == "points":
                tickets.append((kind, n, srv.submit_points(ids[j], qbufs[r_], outn[o:o + n])))
            elif kind == "grid":
                g = m2s.Grid.from_bounding_box(*boxes[j], [n, n, n])
                tickets.append((kind, n ** 3, srv.submit_grid(ids[j], g, S.Raycast, outn[o:o + n ** 3])))
            else:
                v, i = fresh[j][:2]
                mid, t = srv.submit_upload(v, m2s.Topology.TriangleList(i), A.rtree_bvh())
                tickets.append((kind, len(i) // 3, t))
        lat = {"points": [], "grid": [], "upload": []}
        work = {"points": 0, "grid": 0, "upload": 0}
        for kind, n, t in tickets:
            st, l = srv.wait(t)
            assert st == 0, (kind, st)
            lat[kind].append(l)
            work[kind] += n
        entry = {"rate_rps": rate, "requests": n_req, "served": summary(lat, work, time.perf_counter() - t0)}
        # ---- plain: the same arrivals, one call per request, in arrival order on one thread
        if plain:
            lat = {"points": [], "grid": [], "upload": []}
            work = {"points": 0, "grid": 0, "upload": 0}
            t0 = time.perf_counter()
            for r_, (kind, j, n, o) in enumerate(reqs):
                arrive = t0 + arrivals[r_]
                wait = arrive - time.perf_counter()
                if wait > 0:
                    time.sleep(wait)
                if kind == "points":
                    outn[o:o + n] = m2s.query_sdf(plain_meshes[j], qbufs[r_])
                    work["points"] += n
                elif kind == "grid":
                    g = m2s.Grid.from_bounding_box(*boxes[j], [n, n, n])
                    plain_meshes[j].grid_device(g, S.Raycast, dev_grid[:n ** 3])
                    out[o:o + n ** 3].copy_(dev_grid[:n ** 3])
                    work["grid"] += n ** 3
                else:
                    v, i = fresh[j][:2]
                    m2s.build_sdf_acceleration(v, m2s.Topology.TriangleList(i), A.rtree_bvh()).close()
                lat[kind].append(time.perf_counter() - arrive)
            entry["plain"] = summary(lat, work, time.perf_counter() - t0)
            entry["served_over_plain_cells_per_s"] = (entry["served"]["cells_per_s"] /
                                                      max(entry["plain"]["cells_per_s"], 1e-9))
        lines.append(entry)
    stats = srv.stats()
    srv.close()
    for m in plain_meshes:
        m.close()
    return {"workload": "c5_serving", "budget_bytes": 120 * 10**9, "resident_meshes": 64,
            "mix": {"upload": 0.05, "points": 0.57, "grid": 0.38}, "sweep": lines, "server_stats": stats}


def serving_workload(args):
    rates = [float(r) for r in args.rates.split(",") if r]
    print(json.dumps(serving_entry(rates, args.requests, not args.no_cpu_baseline)), flush=True)


def small_case(edge=128, points=100_000, bound_filter=False):
    """A short, fixed workload for ncu captures (at most ~1.5 GB on the device);
    from 2^19 points the queries take the warp-packet search.  The grid comes
    first, so `-k regex:k_propagate -c 1` captures it."""
    import torch

    import mesh_to_sdf_b200 as m2s
    from mesh_to_sdf_b200 import synth

    A, S = m2s.AccelerationMethod, m2s.SignMethod
    v, idx, lo, hi = workload()
    grid = grid_for(lo, hi, (edge, edge, edge))
    mesh = m2s.build_sdf_acceleration(v, m2s.Topology.TriangleList(idx), A.rtree_bvh())
    out = torch.empty(grid.get_total_cell_count(), dtype=torch.float32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    m2s.set_grid_bound_filter(bound_filter)
    mesh.grid_device(grid, S.Raycast, out, status)
    m2s.set_grid_bound_filter(False)
    q = torch.from_numpy(synth.mixed_points(v, idx, points, seed=SEED)).cuda()
    qo = torch.empty(points, dtype=torch.float32, device="cuda")
    mesh.query_device(q, qo, status)
    rt = m2s.build_sdf_acceleration(v, m2s.Topology.TriangleList(idx), A.rtree())
    rt.query_device(q, qo, status)
    bf = m2s.build_sdf_acceleration(v, m2s.Topology.TriangleList(idx), A.none(S.Raycast))
    bf.query_device(q[:8192].contiguous(), qo[:8192], status)
    bn = m2s.build_sdf_acceleration(v, m2s.Topology.TriangleList(idx), A.none(S.Normal))
    bn.query_device(q[:8192].contiguous(), qo[:8192], status)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    print("small ok", m2s.last_grid_stats())


def torch_destroy():
    import torch

    if torch.distributed.is_initialized():
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
