"""QuickSampling throughput on B200 — QS nodes/s, tensor-core form against the
plain FP32 path, at the k-best regret the audit measures.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload config1|config0|config2|config3|config4]
                    [--path bf16|fp8|learned|plain|fp32]

Workloads (seeded synthetic inputs; no public dataset is involved):
  config1 (default)  binary sinuous-channel TI 250x250 (20 channels, seed 1),
                     unconditional categorical simulation 500x500, n=80,
                     k=1.5, seed 100 (+ rank): 250,000 path nodes per step,
                     one step = one whole simulation (levels of independent
                     nodes, every node's map, k best and draw).  Default
                     path: BF16 tensor-core form.
  config0            continuous GRF TI 200x200 (exponential covariance, range
                     12 px), simulation 200x200, n=50, k=1.2.  BF16.
  config3            continuous 3-D GRF TI 180x150x120 (ranges 20,20,5
                     voxels), simulation 200x200x100 (4 M nodes), n=60,
                     k=1.2.  A step is the teacher-forced draw of a fixed
                     sample of 16,000 path nodes (every 250th) against a
                     completed 200x200x100 GRF grid (seed 2): the whole
                     simulation is too long to repeat K times on the plain
                     path.  Default path: FP8 E4M3.
  config2            64 jobs in one call (qsk_jobs_run: each job on its own
                     streams, 16 host threads feeding them) over 3 TIs
                     (continuous GRF 512^2, range 20 px; binary channels
                     500^2; GRF 512^2 plus its indicator at the 0.7
                     quantile), grids log-uniform from 128^2 to 1024^2
                     (16.2 M nodes), n from {20, 40, 60, 100}, k=1.2; the
                     tensor-core form autotuned per (TI, n) shape (untimed,
                     reported) against the plain path.  A step is all 64
                     whole simulations.
  config4            bivariate 3-D TI 256^3 (continuous GRF, ranges 24,24,8
                     voxels, plus a sinusoid-tube indicator, ~20 % facies 1),
                     simulation 256^3, n=64, k=1.5; a step is the
                     teacher-forced draw of every 4096th path node (4,096
                     nodes) against a completed grid of other seeds.
                     Default path: the learned proposal, its encoder trained
                     first (untimed) on 2 M pairs drawn by the exact path on
                     96^3 TIs of other seeds.  The line also reports the
                     proposal with every node accepted (no confidence check,
                     no fallback): its rate and its regret.
Paths: bf16 / fp8 (tensor-core form, 1 % of the nodes audited on the plain
path), learned (top-256 inner-product shortlist of the encoder's
embeddings, exact re-scoring, confidence check with the plain path as
fallback, 1 % audited), plain (the exact reference path: bit-sliced counts for categorical
unit-weight patterns, FP32 gather otherwise), fp32 (the exact path with the
FP32 gather map forced).  The headline path is timed over K steps; the
plain and fp32 paths of the same workload over two steps each, for the
ratio.

Multi-GPU: replicas only — each rank simulates its own realisation (seed +
rank); no data-path collective exists in this algorithm.  ``value`` is the
total nodes of all ranks divided by the slowest rank's device time.

The reference arm (``--impl reference``) runs the G2S reference CPU
QuickSampling (built from the G2S sources; FFTW replaced by the project's
FFT shim unless the host has a libfftw3f) on the host cores with all
threads, on the same TI, n and k: the full grid for configs 0 and 1, a
small grid for config 3 (the reference's cost per node is its FFTs over the
TI, independent of the grid).
"""
from __future__ import annotations

import argparse
import ctypes.util
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
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
# DRAM bytes (read + write) per launch of the dominant kernel, from the ncu
# captures summarised under profiles/ (per workload and kernel)
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "dram_traffic.json")

WORKLOADS = {
    "config1": dict(ti=("channels", (250, 250)), di=(500, 500), types=[1], n=80, k=1.5, path="bf16",
                    name="config1-categorical-channels-250x250-to-500x500-n80-k1.5"),
    "config0": dict(ti=("grf", (200, 200), (12, 12)), di=(200, 200), types=[0], n=50, k=1.2, path="bf16",
                    name="config0-continuous-grf-200x200-to-200x200-n50-k1.2"),
    "config3": dict(ti=("grf", (120, 150, 180), (5, 20, 20)), di=(100, 200, 200), types=[0], n=60, k=1.2, path="fp8",
                    sample=250, name="config3-continuous-grf3d-180x150x120-to-200x200x100-n60-k1.2-sample16000"),
    "config2": dict(jobs=64, path="bf16", k=1.2, ns=(20, 40, 60, 100), sides=(128, 1024), ref_grid=(24, 24),
                    name="config2-batched-64-jobs-3-TIs-grids-128^2-1024^2-n20-100-k1.2"),
    "config4": dict(ti=("bivariate3d", (256, 256, 256), (8, 24, 24)), di=(256, 256, 256), types=[0, 1], n=64, k=1.5,
                    path="learned", sample=4096, ref_grid=(2, 4, 4),
                    train=dict(pairs=2_000_000, size=96, per_ti=300_000, epochs=20, batch=1024),
                    name="config4-learned-bivariate3d-256^3-to-256^3-n64-k1.5-sample4096"),
}
SEED = 100


def peaks():
    try:
        with open(MEASURED_PEAKS) as f:
            p = json.load(f)
        return p, "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


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


_T0 = time.perf_counter()


def log(msg: str):
    """Progress on stderr (the result line alone goes to stdout)."""
    print(f"[bench {time.perf_counter() - _T0:7.1f} s] {msg}", file=sys.stderr, flush=True)


def bivariate3d(shape, ranges, seed):
    """Continuous GRF and the 3-D sinusoid-tube indicator (about 20 % facies
    1), variables interleaved."""
    from g2s_b200 import synthetic as syn
    return np.stack([syn.grf(shape, ranges, seed=seed), syn.tubes3d(shape, seed=seed)], axis=-1)


def make_inputs(w):
    from g2s_b200 import synthetic as syn
    kind = w["ti"][0]
    nv = len(w["types"])
    if kind == "channels":
        ti = syn.channels2d(w["ti"][1], n_channels=20, seed=1)
    elif kind == "bivariate3d":
        ti = bivariate3d(w["ti"][1], w["ti"][2], 1)
    else:
        ti = syn.grf(w["ti"][1], w["ti"][2], seed=1)
    di = np.full(tuple(w["di"]) + ((nv,) if nv > 1 else ()), np.nan, np.float32)
    done = None
    if w.get("sample"):
        done = bivariate3d(w["di"], w["ti"][2], 2) if kind == "bivariate3d" else syn.grf(w["di"], w["ti"][2], seed=2)
    return ti, di, done


def train_encoder(g2s, w, dev):
    """The learned proposal's encoder, trained on (neighbourhood, drawn TI
    cell) pairs that the exact path draws, teacher-forced, on TIs and
    completed grids of other seeds (1000 + i, 2000 + i) of the workload's
    generator; returns the encoder and a description."""
    t = w["train"]
    m = t["size"]
    enc = g2s.Encoder(nvar=len(w["types"]), seed=11, device=dev)
    t0 = time.perf_counter()
    # a fixed number of training TIs, each giving up to per_ti pairs (path
    # nodes without neighbours give none)
    per = min(t["per_ti"], m ** 3)
    n_ti = -(-t["pairs"] // per)
    for i in range(n_ti):
        tis = bivariate3d((m, m, m), w["ti"][2], 1000 + i)
        done = bivariate3d((m, m, m), w["ti"][2], 2000 + i)
        sim = g2s.Simulation(tis, np.full(done.shape, np.nan, np.float32), w["types"], n=w["n"], k=w["k"],
                             seed=5 + i, device=dev)
        take = min(per, t["pairs"] - per * i)
        nodes = np.arange(0, m ** 3, max(1, m ** 3 // take), dtype=np.int32)[:take]
        enc.add_pairs(sim, done, nodes)
        sim.close()
        log(f"training pairs: {enc.pairs()}")
    i = n_ti
    t1 = time.perf_counter()
    loss = enc.train(epochs=t["epochs"] // 2, batch=t["batch"], lr=1e-3, tau=1.0, seed=1)
    loss = enc.train(epochs=t["epochs"] - t["epochs"] // 2, batch=t["batch"], lr=3e-4, tau=1.0, seed=2)
    t2 = time.perf_counter()
    return enc, {"pairs": enc.pairs(), "training_tis": i, "training_ti": f"{m}^3 bivariate, seeds 1000..{999 + i}",
                 "epochs": t["epochs"], "batch": t["batch"], "loss": loss, "pair_s": t1 - t0, "train_s": t2 - t1}


def set_path(sim, path, enc=None, audit=0.01, tuned=None):
    if path in ("bf16", "fp8") and tuned:
        from g2s_b200 import autotune as at
        at.apply(sim, tuned, mode=path, audit=audit)
    elif path in ("bf16", "fp8"):
        sim.set_tensor(path, audit=audit)
    elif path == "learned":
        sim.set_learned(enc, shortlist=256, audit=audit)


def fft_kind() -> str:
    """The FFT under the reference build: always the project FFT behind the
    FFTW3f API ("shim"); a host libfftw3f, if any, is not linked."""
    return "shim"


def fft_in_use() -> str:
    lib = ctypes.util.find_library("fftw3f")
    return f"FFTW3f API shim (project FFT; no libfftw3f on this host)" if not lib else \
        f"FFTW3f API shim (project FFT; this host also has {lib}, not linked)"


def reference_measure(args, w, steps: int):
    """G2S reference CPU QS on the host cores: (nodes/s per step, description)."""
    from oracle import ref
    cores = os.cpu_count() or 1
    ti, di, _ = make_inputs(w)
    nv = len(w["types"])
    if w.get("sample"):
        # per-node cost: FFTs over the TI, not the grid
        g = w.get("ref_grid", (5, 10, 10))
        di = np.full(tuple(g) + ((nv,) if nv > 1 else ()), np.nan, np.float32)
        what = f"{'x'.join(str(d) for d in g)} grid ({int(np.prod(g))} nodes) on the same TI, n and k"
    else:
        what = f"the full {'x'.join(str(d) for d in w['di'])} grid ({int(np.prod(w['di']))} nodes)"
    nodes = int(di.size // nv)
    qsargs = ["-k", str(w["k"]), "-n", str(w["n"]), "-s", str(SEED), "-j", str(cores)]
    vals = []
    for s in range(max(1, steps)):
        _, _, ms, _ = ref.run_qs(ti, di, w["types"], qsargs, job_id=9100 + s)
        vals.append(nodes / (ms / 1000.0))
    return vals, cores, f"G2S qs, {what}, -j {cores}, its reported compute time; {fft_in_use()}"


def reference_arm(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libg2sref.so not built (needs the G2S sources)"}))
        return 0
    w = WORKLOADS[args.workload]
    if w.get("jobs"):
        v, cores, sample = jobs_reference(w, config2_jobs(w))
    else:
        vals, cores, sample = reference_measure(args, w, args.steps)
        v = float(np.mean(vals))
    out = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": float(1000.0 * np.prod(w["di"]) / v) if not (w.get("sample") or w.get("jobs")) else None,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": w["name"], "threads": cores},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "reference", "fft": fft_kind(),
                         "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))
    return 0


def run_step(sim, w, done, sample):
    """One step on the device; returns the engine's info (device time in ms_total)."""
    if w.get("sample"):
        sim.run_teacher_nodes(done, sample)
    else:
        sim.run()
    return sim.info()


def time_path(g2s, w, ti, di, done, sample, seed, dev, path, steps, warmup, flush, enc=None, tuned=None):
    """Timed steps of one path; returns (total device ms, per-step infos, profiled info)."""
    sim = g2s.Simulation(ti, di, w["types"], n=w["n"], k=w["k"], seed=seed, device=dev)
    set_path(sim, path, enc, tuned=tuned)
    g2s.set_map_mode(1 if path == "fp32" else 0)
    import torch
    for _ in range(max(warmup, 0)):
        run_step(sim, w, done, sample)
    torch.cuda.synchronize()
    infos = []
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        infos.append(run_step(sim, w, done, sample))
    torch.cuda.synchronize()
    total = float(sum(i["ms_total"] for i in infos))
    sim.set_profiling(True)
    pinf = run_step(sim, w, done, sample)
    sim.set_profiling(False)
    g2s.set_map_mode(0)
    sim.close()
    return total, infos, pinf


def config2_jobs(w):
    """The 64 jobs: TI j mod 3 (continuous GRF 512^2, range 20 px; binary
    channels 500^2, 40 channels, ~25-30 % facies 1; the GRF 512^2 of another
    seed with its indicator at the 0.7 quantile), n = ns[j mod 4], grid side
    128 * 8^r with r = ((37 j) mod 64) / 63 (log-uniform from 128 to 1024),
    seed 100 + j."""
    from g2s_b200 import synthetic as syn
    tis = [("grf512", syn.grf((512, 512), (20, 20), seed=21), [0]),
           ("channels500", syn.channels2d((500, 500), n_channels=40, seed=22), [1]),
           ("bivariate512", syn.bivariate(syn.grf((512, 512), (20, 20), seed=23)), [0, 1])]
    jobs = []
    J = w["jobs"]
    lo, hi = w["sides"]
    for j in range(J):
        r = ((37 * j) % J) / max(1, J - 1)
        side = int(round(lo * (hi / lo) ** r))
        name, ti, types = tis[j % 3]
        jobs.append(dict(ti_name=name, ti=ti, types=types, n=w["ns"][j % 4], k=w["k"], seed=SEED + j,
                         shape=(side, side) + ((2,) if len(types) > 1 else ())))
    return jobs


def jobs_reference(w, jobs):
    """G2S reference CPU QS on the first job of each TI type, on a small grid
    (its TI, n, k): (harmonic mean of the rates, cores, description)."""
    from oracle import ref
    cores = os.cpu_count() or 1
    rates, done = [], set()
    g = w["ref_grid"]
    for j in jobs:
        if j["ti_name"] in done:
            continue
        done.add(j["ti_name"])
        di = np.full(tuple(g) + j["shape"][2:], np.nan, np.float32)
        qsargs = ["-k", str(j["k"]), "-n", str(j["n"]), "-s", str(j["seed"]), "-j", str(cores)]
        _, _, rms, _ = ref.run_qs(j["ti"], di, j["types"], qsargs, job_id=9200 + len(done))
        rates.append(int(np.prod(g)) / (rms / 1000.0))
    v = float(len(rates) / sum(1.0 / r for r in rates))
    return v, cores, (f"G2S qs, the first job of each TI type on a {g[0]}x{g[1]} grid (its TI, n, k), -j {cores}, "
                      f"harmonic mean of the rates; {fft_in_use()}")


def jobs_main(args, w, g2s, dev):
    """Config 2: all jobs in one qsk_jobs_run call per step (each job on its
    own streams, host threads feeding them), the tensor-core form with
    settings autotuned per (TI, n) shape, against the plain path."""
    import torch
    from g2s_b200 import autotune as at
    path = args.path or w["path"]
    jobs = config2_jobs(w)
    nodes = int(sum(int(np.prod(j["shape"][:2])) for j in jobs))
    log(f"{len(jobs)} jobs, {nodes} nodes")
    tuned, t0 = {}, time.perf_counter()
    if path in ("bf16", "fp8"):
        cache = os.path.join(tempfile.gettempdir(), f"g2s_b200_tune_{os.getpid()}.json")
        for j in jobs:
            key = (j["ti_name"], j["n"])
            if key not in tuned:
                tuned[key] = at.tune(j["ti"], j["types"], j["n"], j["k"], mode=path, device=dev, cache=cache)
                log(f"tuned {key}: {tuned[key]}")
    tune_s = time.perf_counter() - t0

    def make(p, audit=0.01):
        sims = []
        for j in jobs:
            sim = g2s.Simulation(j["ti"], np.full(j["shape"], np.nan, np.float32), j["types"], n=j["n"], k=j["k"],
                                 seed=j["seed"], device=dev)
            if p in ("bf16", "fp8"):
                at.apply(sim, tuned[(j["ti_name"], j["n"])], mode=p, audit=audit)
            sims.append(sim)
        return sims

    def timed(sims):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record()
        g2s.run_jobs(sims, threads=16)
        b.record()
        b.synchronize()
        return a.elapsed_time(b)

    with ClockSampler(dev) as clk:
        sims = make(path)
        for _ in range(max(args.warmup, 0)):
            timed(sims)
        ms = [timed(sims) for _ in range(args.steps)]
        infos = [s.info() for s in sims]
        for s in sims:
            s.close()
    clocks = clk.summary()
    total_ms = float(sum(ms))
    value = nodes * args.steps / (total_ms / 1000.0)
    log(f"{path}: {ms} ms per step")
    compare = {}
    if not args.no_compare and path != "plain":
        sims = make("plain")
        pm = timed(sims)
        compare["plain"] = {"value": nodes / (pm / 1000.0), "ms_per_step": pm,
                            "kernel": "k_map_bits / k_map_records + k_replay (exact reservoir k-best)"}
        for s in sims:
            s.close()
        log(f"plain: {pm:.0f} ms")
    e2e_vals = []
    for _ in range(0 if args.no_e2e else 1):
        t1 = time.perf_counter()
        sims = make(path)
        g2s.run_jobs(sims, threads=16)
        for s in sims:
            s.read()
            s.close()
        e2e_vals.append(time.perf_counter() - t1)
        log(f"e2e: {e2e_vals[-1]:.2f} s")
    h2d = int(sum(j["ti"].nbytes + int(np.prod(j["shape"])) * 4 for j in jobs))
    d2h = int(sum(int(np.prod(j["shape"])) * 4 + int(np.prod(j["shape"][:2])) * 8 for j in jobs))
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import ref
        if ref.available():
            v, cores, samp = jobs_reference(w, jobs)
            cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "reference", "fft": fft_kind(), "sample": samp}
            log(f"cpu baseline: {cpu}")
    plain_v = compare.get("plain", {}).get("value")
    tensor = path in ("bf16", "fp8")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": {"bf16": "bf16", "fp8": "fp8-e4m3", "plain": "mixed (u8 bit-sliced / f32)"}[path],
        "data": "synthetic",
        "config": {"workload": w["name"], "path": path, "jobs": len(jobs), "nodes_per_step": nodes,
                   "one_call": "qsk_jobs_run over all jobs (16 host threads, each job on its own streams)",
                   "tuned": {f"{a}|n={b}": {k2: v[k2] for k2 in ("width", "prefix", "batch", "ms", "runs", "ok")}
                             for (a, b), v in tuned.items()},
                   "tuning_s": tune_s, "l2": "inputs and working set larger than L2 (16 M nodes per step)",
                   "parallelism": "jobs x64 on one GPU"},
        "vs_plain": {"plain": compare.get("plain"), "speedup_vs_plain": value / plain_v if plain_v else None},
        "regret": {"audited": int(sum(i["audited"] for i in infos)), "regret": int(sum(i["regret"] for i in infos)),
                   "near_tie": int(sum(i["regret_near"] for i in infos)),
                   "rate": sum(i["regret"] for i in infos) / max(1, sum(i["audited"] for i in infos)),
                   "definition": "audited nodes (1 % per job) whose drawn candidate scores below the exact k-th best"}
        if tensor else {"regret": 0, "definition": "exact reference path: regret 0 by construction"},
        "map_error_vs_fp64": {"max": max(i["map_err_max"] for i in infos),
                              "mean": float(np.mean([i["map_err_mean"] for i in infos]))} if tensor else None,
        "roofline": None,
        "roofline_note": "jobs of different shapes overlap on separate streams; the kernel rooflines are the "
                         "single-job workloads' (config1, config3)",
        "breakdown_ms_summed_over_jobs": {"total": float(sum(i["ms_total"] for i in infos)),
                                          "tensor_pattern_build_once": float(sum(i["ms_tensor_pattern"] for i in infos))},
        "cpu_baseline": cpu,
        "e2e": {"value": nodes / float(np.mean(e2e_vals)) if e2e_vals else None, "unit": UNIT,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": int(sum(i["launches"] for i in infos)) * args.steps,
        "clocks": clocks,
    }
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200")
    ap.add_argument("--workload", default="config1", choices=sorted(WORKLOADS))
    ap.add_argument("--path", default="", choices=["", "bf16", "fp8", "learned", "plain", "fp32"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--no-compare", action="store_true", help="skip the plain / fp32 comparison arms")
    ap.add_argument("--no-tune", action="store_true",
                    help="whole-simulation tensor workloads: the automatic settings instead of the autotuner's")
    ap.add_argument("--tune-cache", default="",
                    help="autotuner cache file (default: a new one per run); a run given the file of an earlier run "
                         "reuses its choice (profiling)")
    ap.add_argument("--grid", type=int, default=0,
                    help="profiling only: simulation grid side (2-D whole-simulation workloads); not a bench line")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)

    import torch
    import g2s_b200 as g2s

    w = WORKLOADS[args.workload]
    if args.grid:
        if w.get("sample") or w.get("jobs") or len(w["di"]) != 2:
            raise SystemExit("--grid applies to the 2-D whole-simulation workloads")
        w = dict(w, di=(args.grid, args.grid), name=w["name"] + f"-profiling-grid{args.grid}")
    path = args.path or w["path"]
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if w.get("jobs"):
        if ws > 1:
            print(json.dumps({"unavailable": "the batched-jobs workload runs on one GPU"}))
            return 0
        return jobs_main(args, w, g2s, local)
    dist = None
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    dev = local
    log(f"inputs of {w['name']}")
    ti, di, done = make_inputs(w)
    sample = None
    if w.get("sample"):
        sample = np.arange(0, int(np.prod(w["di"])), w["sample"], dtype=np.int32)
    seed = replica_seed(SEED, rank)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{dev}")  # > 126 MB L2
    own_peaks = g2s.measure_peaks(dev)
    log("peaks measured")
    enc, enc_info = (train_encoder(g2s, w, dev) if path == "learned" else (None, None))
    if enc_info:
        log(f"encoder trained: {enc_info}")
    # whole simulations on the tensor-core form: width, prefix tile and batch
    # from the autotuner (tuned on a smaller grid of the same shape, untimed)
    tuned, tune_s = None, 0.0
    if path in ("bf16", "fp8") and not w.get("sample") and not args.no_tune:
        from g2s_b200 import autotune as at
        t0 = time.perf_counter()
        tuned = at.tune(ti, w["types"], w["n"], w["k"], mode=path, device=dev,
                        cache=args.tune_cache or os.path.join(tempfile.gettempdir(), f"g2s_b200_tune_{os.getpid()}.json"))
        tune_s = time.perf_counter() - t0
        log(f"tuned: {tuned}")

    # headline path: K timed steps (CUDA events inside the engine, first to
    # last kernel of each step on its stream), L2 flushed between steps
    with ClockSampler(dev) as clk:
        if dist:
            dist.barrier()
        total_ms, infos, pinf = time_path(g2s, w, ti, di, done, sample, seed, dev, path, args.steps, args.warmup,
                                          flush, enc, tuned)
        if dist:
            dist.barrier()
    clocks = clk.summary()
    log(f"headline path {path}: {total_ms:.1f} ms over {args.steps} steps")
    nodes = int(infos[-1]["nodes"])
    total_ms = slowest(total_ms, dist, f"cuda:{dev}")
    value = whole_job_rate(nodes, args.steps, ws, total_ms)
    launches = int(sum(i["launches"] for i in infos))

    # the plain paths on the same workload (two steps each): the ratio's denominator
    compare = {}
    if not args.no_compare:
        for p in ("plain", "fp32"):
            if p == path or (p == "fp32" and w["types"] != [1]):
                continue   # continuous patterns: the plain path is the FP32 gather map already
            t, inf2, _ = time_path(g2s, w, ti, di, done, sample, seed, dev, p, 2, 1, flush)
            log(f"comparison path {p}: {t:.1f} ms over 2 steps")
            t = slowest(t, dist, f"cuda:{dev}")
            compare[p] = {"value": whole_job_rate(nodes, 2, ws, t), "ms_per_step": t / 2,
                          "kernel": ("k_map_bits" if (p == "plain" and w["types"] == [1]) else "k_map_records") +
                                    " + k_replay (exact reservoir k-best)"}

    # learned proposal, diagnostic: every proposal accepted (no confidence
    # check, no fallback): its rate and its regret over all nodes
    accept_all = None
    if path == "learned":
        sim = g2s.Simulation(ti, di, w["types"], n=w["n"], k=w["k"], seed=seed, device=dev)
        sim.set_learned(enc, shortlist=256, conf_z=0.0, conf_rank=256, audit=1.0)
        run_step(sim, w, done, sample)
        a = sim.info()
        sim.set_learned(enc, shortlist=256, conf_z=0.0, conf_rank=256, audit=0.0)
        run_step(sim, w, done, sample)
        sim.set_profiling(True)
        b = run_step(sim, w, done, sample)
        sim.set_profiling(False)
        sim.close()
        accept_all = {"value": a["nodes"] / (b["ms_total"] / 1000.0), "unit": UNIT, "ms_per_step": b["ms_total"],
                      "ms_gemm": b["ms_tensor_gemm"], "ms_select": b["ms_tensor_select"],
                      "regret": a["regret"], "audited": a["audited"],
                      "rate": a["regret"] / max(1, a["audited"])}

    if accept_all:
        log(f"accept-all diagnostic: {accept_all}")
    # roofline of the dominant kernel of the profiled step
    pk, pk_kind = peaks()
    tensor = path in ("bf16", "fp8", "learned")
    kernels = {}
    if tensor:
        gemm_ms = max(pinf["ms_tensor_gemm"], 1e-9)
        tc_peak = pk.get("bf16_tflops", 1590.0) if path != "fp8" else own_peaks["fp8_tflops"]
        tc_peak_kind = (f"{pk_kind} bf16_tflops (cuBLAS, burst)" if path != "fp8" else
                        "fp8 E4M3 dense, this library's tcgen05 microbenchmark (qsk_measure_peaks)")
        ach = pinf["tensor_flops"] / (gemm_ms / 1000.0) / 1e12
        kernels["k_tc_shortlist"] = {"ms_per_step": pinf["ms_tensor_gemm"], "bound": "tensor",
                                     "achieved_tflops": ach, "peak_tflops": tc_peak, "frac": ach / tc_peak,
                                     "issued_flops_per_step": pinf["tensor_flops"]}
        kernels["k_prep_sim+k_tc_nodes+k_tc_select"] = {"ms_per_step": pinf["ms_tensor_select"]}
        kernels["pattern_matrix_build_once"] = {"ms": pinf["ms_tensor_pattern"]}
    kernels["exact_map (" + ("k_map_bits" if w["types"] == [1] else "k_map_records") + ")"] = {
        "ms_per_step": pinf["ms_map"], "map_launches": pinf["map_launches"]}
    kernels["k_replay / k_hash_select"] = {"ms_per_step": pinf["ms_replay"]}
    # the dominant kernel of the step by device time: the shortlist GEMM, or
    # the exact map (plain path; a tensor path's exact-map and fallback nodes)
    gemm_dominant = tensor and pinf["ms_tensor_gemm"] >= pinf["ms_map"]
    map_nodes = nodes if not tensor else int(pinf["plain_nodes"] + pinf["learned_fallback"])
    traffic = None
    try:
        traffic = json.load(open(TRAFFIC_FILE)).get(args.workload, {}).get("k_tc_shortlist" if gemm_dominant else "map")
    except Exception:
        pass
    if gemm_dominant:
        k = kernels["k_tc_shortlist"]
        # per tensor step: terms + node rows (one launch; two when learned), shortlist, select
        launches_gemm = max(1, int(pinf["tensor_launches"]) // (4 if path == "learned" else 3))
        roofline = {"bound": "tensor", "achieved": k["achieved_tflops"], "peak": k["peak_tflops"], "unit": "TFLOP/s",
                    "frac": k["frac"], "traffic": traffic, "kernel": "k_tc_shortlist", "peak_kind": tc_peak_kind,
                    "launches_per_step": launches_gemm,
                    "algorithmic_work": "issued MMA flops 2 x 128 x 256 x K per (node tile, position tile); "
                                        "K = template offsets up to the tile's widest node x pattern layers",
                    "kernels": kernels}
    else:
        fp32 = own_peaks["fp32_tflops"]
        N = int(np.prod(w["ti"][1]))
        L = 2 * len(w["types"])
        useful = 2.0 * w["n"] * N * L * map_nodes / (max(pinf["ms_map"], 1e-9) / 1000.0) / 1e12
        roofline = {"bound": "fp32" if w["types"] != [1] else "alu", "achieved": useful, "peak": fp32,
                    "unit": "TFLOP/s (FP32-equivalent 2*n*N*L per node, L = 2 per variable)", "frac": useful / fp32,
                    "traffic": traffic, "kernel": "exact map", "map_nodes_per_step": map_nodes,
                    "peak_kind": "FP32 FMA, this library's microbenchmark (qsk_measure_peaks)", "kernels": kernels}

    # e2e: the public one-call API with host buffers (H2D of the inputs, D2H
    # of the results inside the timed region), wall clock around the call
    e2e_vals = []
    h2d = d2h = 0
    for _ in range(0 if args.no_e2e else max(1, min(args.steps, 3))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if w.get("sample"):
            sim = g2s.Simulation(ti, di, w["types"], n=w["n"], k=w["k"], seed=seed, device=dev)
            set_path(sim, path, enc, tuned=tuned)
            sim.run_teacher_nodes(done, sample)
            _, _, cells = sim.read()
            sim.close()
            h2d, d2h = ti.nbytes + done.nbytes + di.nbytes + sample.nbytes, int(done.nbytes + di.size * 4 + cells.nbytes)
        else:
            d = np.full(di.shape, np.nan, np.float32)
            tensor = None
            if path in ("bf16", "fp8"):
                tensor = dict(mode=path, prefix=tuned["prefix"], width=tuned["width"],
                              batch=tuned["batch"]) if tuned else path
            g2s.qs(ti, d, w["types"], k=w["k"], n=w["n"], s=seed, device=dev, tensor=tensor)
            h2d, d2h = ti.nbytes + di.nbytes, int(di.nbytes + di.size * 4)
        torch.cuda.synchronize()
        e2e_vals.append(time.perf_counter() - t0)
        log(f"e2e call: {e2e_vals[-1]:.2f} s")
    e2e_s = float(np.mean(e2e_vals)) if e2e_vals else float("nan")
    e2e_s = slowest(e2e_s, dist, f"cuda:{dev}")
    e2e = {"value": nodes * ws / e2e_s if e2e_vals else None, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": int(d2h)}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        from oracle import ref
        if ref.available():
            log("cpu baseline (reference) ...")
            vals, cores, samp = reference_measure(args, w, 1)
            log(f"cpu baseline: {vals}")
            cpu = {"value": float(np.mean(vals)), "unit": UNIT, "cores": cores, "kind": "reference", "fft": fft_kind(),
                   "sample": samp}

    if rank == 0:
        last = infos[-1]
        plain_v = compare.get("plain", {}).get("value")
        fp32_v = compare.get("fp32", {}).get("value")
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"bf16": "bf16", "fp8": "fp8-e4m3", "learned": "bf16", "plain": "u8" if w["types"] == [1] else "f32",
                      "fp32": "f32"}[path],
            "data": "synthetic",
            "config": {"workload": w["name"], "path": path,
                       "tensor": {"prefix": last["tensor_prefix"], "width": last["tensor_width"],
                                  "shortlist": last["tensor_shortlist"], "tensor_nodes": last["tensor_nodes"],
                                  "exact_map_nodes": last["plain_nodes"], "audit_fraction": 0.01,
                                  "autotuned": {k2: tuned[k2] for k2 in ("width", "prefix", "batch", "ms", "runs",
                                                                         "grid", "ok")} if tuned else None,
                                  "tuning_s": tune_s} if tensor else None,
                       "learned": {"encoder": enc_info, "shortlist": 256, "confidence": "fit R^2 >= 0.2, z = 2",
                                   "confident_nodes": int(last["tensor_nodes"] - last["learned_fallback"]),
                                   "fallback_nodes": int(last["learned_fallback"]),
                                   "accept_all_diagnostic": accept_all} if path == "learned" else None,
                       "nodes_per_step": nodes, "levels": last["levels"], "max_batch": last["max_batch"],
                       "l2": "flushed between steps (256 MB write)", "parallelism": f"replicas x{ws}"},
            "vs_plain": {"plain": compare.get("plain"), "fp32_gather": compare.get("fp32"),
                         "speedup_vs_plain": value / plain_v if plain_v else None,
                         "speedup_vs_fp32_gather": value / fp32_v if fp32_v else None},
            "regret": {"audited": int(sum(i["audited"] for i in infos)), "regret": int(sum(i["regret"] for i in infos)),
                       "near_tie": int(sum(i["regret_near"] for i in infos)),
                       "rate": (sum(i["regret"] for i in infos) / max(1, sum(i["audited"] for i in infos))),
                       "definition": "audited nodes whose drawn candidate scores below the exact k-th best "
                                     "(plain FP32 path, teacher-forced on the final grid); near_tie: below it by at "
                                     "most 1e-5 of the term scale"} if tensor else
                      {"regret": 0, "definition": "exact reference path: regret 0 by construction"},
            "map_error_vs_fp64": {"max": max(i["map_err_max"] for i in infos),
                                  "mean": float(np.mean([i["map_err_mean"] for i in infos])),
                                  "unit": "|score - FP64 score| / term scale over the re-scored shortlists"}
            if path in ("bf16", "fp8") else None,
            "roofline": roofline,
            "own_peaks": own_peaks,
            "breakdown_ms": {"neighbours": pinf["ms_setup_neighbours"], "levels": pinf["ms_levels"],
                             "prep": pinf["ms_prep"], "exact_map": pinf["ms_map"], "replay": pinf["ms_replay"],
                             "tensor_gemm": pinf["ms_tensor_gemm"], "tensor_select": pinf["ms_tensor_select"],
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
