"""QuickSampling throughput on B200 — QS nodes/s.

Workload (the benchmark configuration that fits one GPU): binary sinuous-
channel training image 250x250 (20 channels, ~25-30 % facies 1, seed 1),
unconditional categorical simulation of a 500x500 grid, n=80 neighbours,
k=1.5, seed 100 (+ rank): 250,000 path nodes per step.  One step is one
complete simulation on the GPU (neighbour search, dependency levels, every
node's mismatch map, k-best and draw).  Synthetic seeded data only.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU: replicas only — each rank simulates its own realisation (seed +
rank); no data-path collective exists in this algorithm.  ``value`` is the
total nodes of all ranks divided by the slowest rank's device time.

The reference arm (``--impl reference``) runs the G2S reference CPU
QuickSampling (built from the G2S sources, FFTW replaced by the project's
FFT shim) on the host cores with all threads, on a bounded sample of the same
workload (a smaller grid with the same TI, n and k; per-node cost of the
reference is dominated by its FFTs over the TI and does not depend on the
grid size).
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

METRIC = "QS nodes/s on 1 B200: tensor-core/learned vs plain FP32 at ≤1% k-best regret"
UNIT = "nodes/s"
TI_SHAPE = (250, 250)
DI_SHAPE = (500, 500)
N_NB, K_CAND, SEED = 80, 1.5, 100
WORKLOAD = "config1-categorical-channels-250x250-to-500x500-n80-k1.5"
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
# DRAM bytes (read + write) per launch, averaged over every launch of one
# step of the default workload, from one ncu capture of this script
# (dram__bytes_read.sum + dram__bytes_write.sum; cold-cache, launches serialised)
TRAFFIC_PER_LAUNCH = {("config1", "k_replay"): 14.54e6, ("config1", "k_map_bits"): 12.07e6}


def peaks():
    try:
        with open(MEASURED_PEAKS) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, index: int = 0):
        self.index = index
        self.proc = None
        self.path = os.path.join(os.environ.get("QSK_CLOCKS_DIR", tempfile.gettempdir()), f"clocks_{os.getpid()}.csv")

    def __enter__(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [l.split(",") for l in open(self.path).read().strip().splitlines() if l.strip()]
        except Exception:
            return None
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
            except Exception:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def replica_seed(base: int, rank: int) -> int:
    """Replicas only: rank r simulates its own realisation with seed base + r."""
    return base + rank


def slowest(value: float, dist=None, device=None) -> float:
    """Max over ranks (device time of the slowest rank)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(nodes_per_rank: int, steps: int, world: int, slowest_ms: float) -> float:
    """Nodes of all ranks divided by the slowest rank's time."""
    return nodes_per_rank * steps * world / (slowest_ms / 1000.0)


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def reference_arm(args):
    """G2S reference CPU QS on the host cores: bounded sample of the workload."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    from oracle import ref
    from g2s_b200 import synthetic as syn
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libg2sref.so not built (needs the G2S sources)"}))
        return 0
    cores = os.cpu_count() or 1
    ti = syn.channels2d(TI_SHAPE, n_channels=20, seed=1)
    side = int(args.ref_side)
    di = np.full((side, side), np.nan, np.float32)
    qsargs = ["-k", str(K_CAND), "-n", str(N_NB), "-s", str(SEED), "-j", str(cores)]
    for _ in range(args.warmup if args.warmup < 1 else 1):
        ref.run_qs(ti, np.full((32, 32), np.nan, np.float32), [1], qsargs, job_id=9000)
    vals = []
    for s in range(args.steps):
        sim, idx, ms, _ = ref.run_qs(ti, di, [1], qsargs, job_id=9100 + s)
        vals.append(side * side / (ms / 1000.0))
    v = float(np.mean(vals))
    out = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": float(side * side / v * 1000.0), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample": f"{side}x{side} grid ({side * side} of the 250000 nodes), same TI/n/k",
                   "threads": cores},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"G2S qs (FFTW-API shim), {side}x{side} grid, -j {cores}, reported compute time"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))
    return 0


def cpu_baseline_leg(side: int):
    """Reference CPU QS timed on the host cores (rank 0, N=1 only)."""
    from oracle import ref
    from g2s_b200 import synthetic as syn
    if not ref.available():
        return None
    cores = os.cpu_count() or 1
    ti = syn.channels2d(TI_SHAPE, n_channels=20, seed=1)
    di = np.full((side, side), np.nan, np.float32)
    sim, idx, ms, _ = ref.run_qs(ti, di, [1], ["-k", str(K_CAND), "-n", str(N_NB), "-s", str(SEED), "-j", str(cores)],
                                 job_id=9500)
    v = side * side / (ms / 1000.0)
    return {"value": v, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"G2S qs (FFTW-API shim) on {side}x{side} grid ({side * side} nodes), same TI/n/k, -j {cores}"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200")
    ap.add_argument("--ref-side", type=int, default=120)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--workload", default="config1", choices=["config1", "config0"],
                    help="config1 (default, the benchmark line) or config0 (continuous GRF 200x200, n=50, k=1.2)")
    ap.add_argument("--di-side", type=int, default=0,
                    help="simulate an SxS grid instead of the workload's (small cases for profiling)")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)

    import torch
    import g2s_b200 as g2s
    from g2s_b200 import synthetic as syn

    global TI_SHAPE, DI_SHAPE, N_NB, K_CAND, WORKLOAD
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    dev = local

    types = [1]
    if args.workload == "config0":
        TI_SHAPE, DI_SHAPE, N_NB, K_CAND = (200, 200), (200, 200), 50, 1.2
        WORKLOAD = "config0-continuous-grf-200x200-to-200x200-n50-k1.2"
        ti = syn.grf(TI_SHAPE, (12, 12), seed=1)
        types = [0]
    else:
        ti = syn.channels2d(TI_SHAPE, n_channels=20, seed=1)
    if args.di_side > 0:
        DI_SHAPE = (args.di_side, args.di_side)
        WORKLOAD += f"-grid{args.di_side}x{args.di_side}"
    di = np.full(DI_SHAPE, np.nan, np.float32)
    seed = replica_seed(SEED, rank)
    sim = g2s.Simulation(ti, di, types, n=N_NB, k=K_CAND, seed=seed, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{dev}")  # > 126 MB L2

    for _ in range(max(args.warmup, 0)):
        sim.run()
    torch.cuda.synchronize()

    # timed region: device time of each full simulation (CUDA events inside
    # the engine, first to last kernel on its stream); L2 flushed between steps
    step_ms = []
    launches = 0
    with ClockSampler(dev) as clk:
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            sim.run()
            inf = sim.info()
            step_ms.append(inf["ms_total"])
            launches += int(inf["launches"])
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
    clocks = clk.summary()
    total_ms = float(sum(step_ms))
    nodes = int(sim.info()["nodes"])
    total_ms = slowest(total_ms, dist, f"cuda:{dev}")
    value = whole_job_rate(nodes, args.steps, ws, total_ms)

    # roofline of the dominant kernel: one extra profiled step records events
    # around every launch.  Algorithmic bytes per node of the reference
    # path: the fused map reads 4*N*L bytes of correlation layers, the k-best
    # scan 4*N bytes of scores.
    sim.set_profiling(True)
    sim.run()
    pinf = sim.info()
    sim.set_profiling(False)
    map_kernel = "k_map_bits" if types == [1] else "k_map_records"
    N = TI_SHAPE[0] * TI_SHAPE[1]
    L = 2  # continuous: TI^2 and TI; binary categorical: 2 class indicators
    launches_l = max(pinf["map_launches"], 1)
    nodes_per_launch = pinf["map_positions"] / launches_l / N
    peak, peak_kind = peaks()
    kernels = {}
    for name, ms, bpn in ((map_kernel, pinf["ms_map"], 4 * N * L), ("k_replay", pinf["ms_replay"], 4 * N)):
        avg_ms = ms / launches_l
        ach = bpn * nodes_per_launch / (avg_ms / 1000.0) / 1e9
        kernels[name] = {"ms_per_step": ms, "launches": launches_l, "avg_launch_ms": avg_ms,
                         "algorithmic_bytes_per_node": bpn, "achieved": ach, "frac": ach / peak,
                         "share_of_step": ms / max(pinf["ms_total"], 1e-9),
                         "traffic": TRAFFIC_PER_LAUNCH.get((args.workload, name)) if args.di_side == 0 else None}
    dom = max(kernels, key=lambda k: kernels[k]["ms_per_step"])
    roofline = {"bound": "hbm", "achieved": kernels[dom]["achieved"], "peak": peak, "unit": "GB/s",
                "frac": kernels[dom]["frac"], "traffic": kernels[dom]["traffic"], "kernel": dom,
                "peak_kind": f"{peak_kind} hbm_gbs", "nodes_per_launch": nodes_per_launch,
                "algorithmic_bytes": f"{map_kernel}: 4*N*L per node, k_replay: 4*N per node (N={N}, L={L})",
                "kernels": kernels}
    out_info = sim.info()
    sim.close()

    # e2e: the public one-call API with host buffers (H2D of TI+grid, D2H of
    # grid+index image inside the timed region), wall clock around the call
    e2e_vals = []
    for _ in range(0 if args.no_e2e else max(1, min(args.steps, 3))):
        d = np.full(DI_SHAPE, np.nan, np.float32)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g2s.qs(ti, d, types, k=K_CAND, n=N_NB, s=seed, device=dev)
        torch.cuda.synchronize()
        e2e_vals.append(time.perf_counter() - t0)
    e2e_s = float(np.mean(e2e_vals)) if e2e_vals else float("nan")
    e2e_s = slowest(e2e_s, dist, f"cuda:{dev}")
    e2e = {"value": nodes * ws / e2e_s if e2e_vals else None, "unit": UNIT,
           "h2d_bytes_per_step": int(ti.nbytes + di.nbytes),
           "d2h_bytes_per_step": int(di.nbytes + di.size * 4)}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline and args.workload == "config1":
        cpu = cpu_baseline_leg(args.ref_side)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u8" if types == [1] else "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD,
                       "path": ("bit-sliced categorical match counts (equal to the FP32 map)" if types == [1] else
                                "FP32 direct-sum map") + " + exact reservoir k-best replay (CUDA cores)",
                       "nodes_per_step": nodes, "levels": out_info["levels"], "max_batch": out_info["max_batch"],
                       "l2": "flushed between steps (256 MB write)", "parallelism": f"replicas x{ws}"},
            "roofline": roofline,
            "breakdown_ms": {"neighbours": pinf["ms_setup_neighbours"], "levels": pinf["ms_levels"],
                             "prep": pinf["ms_prep"], "map": pinf["ms_map"], "replay": pinf["ms_replay"],
                             "total": pinf["ms_total"]},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clocks,
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
