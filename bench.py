#!/usr/bin/env python
"""Map-integration benchmark on the README-scale workload.

Workload (one "step" = one scan of the trajectory, update then recenter):
  grid 701 x 701 x 151 voxels (74.2M) at 0.1 m, FP32 log-odds from the
  yaml probabilities; 64 beams (elevation -22.5..22.5 deg) x 1024 azimuths =
  65,536 points per scan, 50 m max range, sigma 0.02 m; seeded scene of a
  ground plane and 400 boxes over +-60 m; circle trajectory of radius 25 m at
  1.5 m/s and 10 Hz, recentering with the 4 m threshold.

Metric: voxel-steps/s, the reference's own work unit (DDA iterations that
did not break + 1 endpoint per ray), counted for every scan by
cublox_grid_reference_steps; p50/p99 per-scan latency beside it.

  value  device time, scans already resident in HBM, CUDA events on the
         grid's stream, L2 flushed (512 MiB write) between steps
  e2e    wall time through the public API from pinned host memory, each step
         = host->device copy of the scan + update + recenter + a 4-byte
         device->host read of the map
  --impl reference  the reference's own kernels (oracle/_ref, built from its
         src/kernels.cu for sm_100a) in its OccupancyGrid call sequence
         (pageable copies, two syncs per update, device recenter plan)

Under torchrun every rank integrates its own replica of the workload (maps
shard across GPUs with no exchange); value = all ranks' steps / max time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "voxel-steps/s & p50/p99 scan latency, batched/served vs plain on 1 B200"
UNIT = "voxel-steps/s"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if "Active" in r[5 + i]
                          and "Not" not in r[5 + i]})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(mx)) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def build_workload(n_scans: int):
    from cublox_b200 import synth
    w = synth.readme_scale(n_scans)
    scans = [w.scan(k) for k in range(n_scans)]
    origins = [w.sensor_origin(k) for k in range(n_scans)]
    return w, scans, origins


def count_steps(w, scans, origins):
    import cublox_b200 as C
    g = C.OccupancyGrid(w.half, w.resolution, False, None)
    g.setMaxRaycastRange(w.sensor.max_range)
    steps = [g.reference_steps(s, o) for s, o in zip(scans, origins)]
    g.close()
    return np.asarray(steps, dtype=np.int64)


def cpu_baseline(w, scans, origins, steps, budget_s=12.0):
    """The oracle (CPU restatement of the reference's path) on the host cores."""
    import oracle as O
    import cublox_b200 as C
    threads = os.cpu_count() or 1
    g = O.OracleGrid(w.half, w.resolution, False, w.threshold)
    g.set_log_odds(*C.yaml_log_odds())
    g.set_max_range(w.sensor.max_range)
    t0 = time.perf_counter()
    done = 0
    vs = 0
    while done < len(scans) and (done < 2 or time.perf_counter() - t0 < budget_s):
        g.update(scans[done], origins[done], threads=threads)
        g.recenter(origins[done])
        vs += int(steps[done])
        done += 1
    dt = time.perf_counter() - t0
    return {"value": vs / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"first {done} scans of the trajectory (update + recenter), "
                      f"{threads} threads, {dt:.1f} s"}


def run_cublox(args, rank, world, dist):
    import torch
    import cublox_b200 as C

    n_scans = args.warmup + args.steps
    w, scans, origins = build_workload(n_scans)
    steps = count_steps(w, scans, origins)
    N = scans[0].shape[0]
    # A dedicated stream shared by torch (events, L2 flush) and the grid.
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    lo = C.yaml_log_odds()

    def new_grid():
        g = C.OccupancyGrid(w.half, w.resolution, False, w.threshold, stream=stream.cuda_stream)
        g.setLogOddsParams(*lo)
        g.setMaxRaycastRange(w.sensor.max_range)
        return g

    # ---- value: device-resident scans ------------------------------------
    dev = [torch.from_numpy(np.ascontiguousarray(s.T)).cuda() for s in scans]  # (3, N) SoA
    g = new_grid()
    g.enable_stats(True)
    g.enable_timing(True)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(n_scans)]
    ray_ms, fold_ms, clear_ms, touched, actions = [], [], [], [], []
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    with Clocks(torch.cuda.current_device()) as clk:
        for k in range(n_scans):
            flush.zero_()
            ev[k][0].record(stream)
            g.update(dev[k], origins[k])
            a = g.recenter(origins[k])
            ev[k][1].record(stream)
            t = g.last_timing()
            st = g.last_stats()
            if k >= args.warmup:
                ray_ms.append(t[0])
                fold_ms.append(t[1])
                if t[2] >= 0:
                    clear_ms.append(t[2])
                touched.append(st["touched"])
                actions.append(a)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    step_ms = np.asarray([ev[k][0].elapsed_time(ev[k][1]) for k in range(args.warmup, n_scans)])
    timed_steps = int(steps[args.warmup:].sum())
    tot_ms = float(step_ms.sum())
    if dist:
        t = torch.tensor([tot_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tot_ms = float(t.item())
    value = world * timed_steps / (tot_ms / 1e3)
    assert g.check() == 0, "device error word set"
    g.close()

    # ---- e2e: public API from pinned host memory ---------------------------
    pinned = [torch.from_numpy(s).pin_memory() for s in scans]  # (N, 3) AoS
    g = new_grid()
    wall = []
    for k in range(n_scans):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g.update_ptr(pinned[k].data_ptr(), N, origins[k], C.LAYOUT_AOS)
        g.recenter(origins[k])
        _ = g.storedAt(0)
        t1 = time.perf_counter()
        if k >= args.warmup:
            wall.append(t1 - t0)
    e2e_s = float(np.sum(wall))
    if dist:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = world * timed_steps / e2e_s
    g.close()

    # ---- roofline of the update (raycast + fold), HBM-bound by definition --
    peak, peak_kind = _peaks()
    upd_ms = np.asarray(ray_ms) + np.asarray(fold_ms)
    alg_bytes = 12.0 * N + 8.0 * np.asarray(touched, dtype=np.float64)
    achieved = float(np.mean(alg_bytes) / (np.mean(upd_ms) / 1e3) / 1e9)
    dom = "raycast" if np.mean(ray_ms) >= np.mean(fold_ms) else "fold"
    launches = 2 * args.steps + int(sum(1 for a in actions if a == 1))
    out = None
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": tot_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded ray-cast LiDAR scans)",
            "config": {"workload": w.name, "grid": [701, 701, 151], "resolution_m": 0.1,
                       "points_per_scan": N, "max_range_m": 50.0, "recenter_threshold_m": 4.0,
                       "form": "plain drop-in (one map, one scan per step)",
                       "l2": "flushed between steps (512 MiB write)",
                       "parallelism": f"replicas x{world} (map-sharded, no collective)"},
            "p50_ms": float(np.percentile(step_ms, 50)), "p99_ms": float(np.percentile(step_ms, 99)),
            "kernel_ms": {"raycast": float(np.mean(ray_ms)), "fold": float(np.mean(fold_ms)),
                          "recenter_clear": float(np.mean(clear_ms)) if clear_ms else None},
            "recenters": int(sum(1 for a in actions if a)),
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 12 * N, "d2h_bytes_per_step": 4,
                    "p50_ms": float(np.percentile(wall, 50) * 1e3),
                    "p99_ms": float(np.percentile(wall, 99) * 1e3)},
            "roofline": {"bound": "hbm", "kernel": f"update (raycast+fold; {dom} dominant)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": peak_kind, "traffic": None,
                         "algorithmic_bytes": "12 B per point + 8 B per touched voxel (occ read+write)"},
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        if world == 1 and not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(w, scans, origins, steps)
    return out


def run_reference(args):
    import oracle as O
    import cublox_b200 as C

    if not O.ref_available():
        return {"impl": "reference", "unavailable": "reference harness oracle/_ref/libcublox_ref.so "
                                                     "was not built (needs the reference tree)"}
    n_scans = args.warmup + args.steps
    w, scans, origins = build_workload(n_scans)
    steps = count_steps(w, scans, origins)
    N = scans[0].shape[0]
    import torch
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    r = O.RefGrid(w.half, w.resolution, False, w.threshold)
    r.set_log_odds(*C.yaml_log_odds())
    r.set_max_range(w.sensor.max_range)
    soa = [tuple(np.ascontiguousarray(s[:, a]) for a in range(3)) for s in scans]
    wall = []
    with Clocks(torch.cuda.current_device()) as clk:
        for k in range(n_scans):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r.update(None, origins[k], xyz=soa[k])
            r.recenter(origins[k])
            t1 = time.perf_counter()
            if k >= args.warmup:
                wall.append(t1 - t0)
    r.close()
    tot = float(np.sum(wall))
    value = int(steps[args.warmup:].sum()) / tot
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": tot * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded ray-cast LiDAR scans)", "impl": "reference",
        "config": {"workload": w.name, "grid": [701, 701, 151], "resolution_m": 0.1,
                   "points_per_scan": N, "max_range_m": 50.0, "recenter_threshold_m": 4.0,
                   "form": "reference OccupancyGrid call sequence",
                   "l2": "flushed between steps (512 MiB write)", "parallelism": "single map"},
        "p50_ms": float(np.percentile(wall, 50) * 1e3), "p99_ms": float(np.percentile(wall, 99) * 1e3),
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 12 * N, "d2h_bytes_per_step": 0},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": "the reference's src/kernels.cu (sm_100a build) driven by one host "
                                   f"thread in its OccupancyGrid sequence, {args.steps} scans on the B200"},
        "clocks": clk.summary(),
    }


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=120)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["cublox", "reference"], default="cublox")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    torch.cuda.set_device(local)
    if args.impl == "reference":
        if rank != 0:
            return 0
        print(json.dumps(run_reference(args)), flush=True)
        return 0
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    out = run_cublox(args, rank, world, dist)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
