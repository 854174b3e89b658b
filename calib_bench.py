"""Throughput of the auto_qs calibration: GPU (qsk_calibrate) against the
reference's own auto_qs program on the host cores, on the categorical
channels TI 250x250 (20 channels, seed 1) with auto_qs' default setups
(neighbour configurations 1..79, the 7 default densities, one 21x21 Gaussian
kernel, max_k 1, power 2) and pruning off (min iterations = max
iterations), so both arms search every setup every iteration.  Prints one
JSON line: searches per second of each arm.

    python calib_bench.py [--iterations 200] [--ref-iterations 100]

The reference needs at least 100 iterations (its progress report divides the
iteration counter by max_iterations/100).
"""
import argparse
import json
import os
import subprocess
import time

import sys

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--iterations", type=int, default=200)
    ap.add_argument("--ref-iterations", type=int, default=100)
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args()
    import g2s_b200 as g
    from g2s_b200 import synthetic as syn
    ti = syn.channels2d((250, 250), n_channels=20, seed=1)
    r = np.arange(21) - 10
    kernel = np.exp(-(r[:, None] ** 2 + r[None, :] ** 2) / 50.0).astype(np.float32)
    counts = g.default_neighbour_counts(80)
    # warm-up (context, module load), then the timed run
    g.calibrate(ti, [1], [kernel], counts, None, max_iterations=1, min_iterations=1, seed=1, device=args.device)
    t0 = time.perf_counter()
    _, _, n, searches = g.calibrate(ti, [1], [kernel], counts, None, max_iterations=args.iterations,
                                    min_iterations=args.iterations, seed=1, device=args.device)
    gpu_s = time.perf_counter() - t0
    out = {"metric": "auto_qs calibration searches/s", "unit": "searches/s", "gpu": searches / gpu_s,
           "gpu_searches": searches, "gpu_seconds": gpu_s, "setups": int(n[..., 0].size),
           "config": "channels 250x250 (20 channels), maxn 80, 7 densities, 21x21 Gaussian kernel, max_k 1"}
    exe = os.path.join(ROOT, "oracle", "_ref", "auto_qs")
    if os.path.exists(exe):
        from oracle import ref as R
        R.write_image("calbench_ti", ti, [1])
        R.write_image("calbench_k", kernel, [0])
        cores = os.cpu_count() or 1
        cmd = [exe, "-ti", "calbench_ti", "-ki", "calbench_k", "-maxk", "1", "-maxn", "80", "-maxIter",
               str(args.ref_iterations), "-minIter", str(args.ref_iterations), "-j", str(cores), "-r",
               "/tmp/G2S/logs/calbench.log"]
        t0 = time.perf_counter()
        subprocess.run(cmd, cwd="/tmp/G2S/data", check=True, capture_output=True)
        ref_s = time.perf_counter() - t0
        ref_n = R.read_image("im_3_4294967295")
        ref_n = ref_n.view(np.uint32) if ref_n.dtype == np.float32 else ref_n
        ref_searches = int(np.asarray(ref_n).sum())   # max_k 1: one count per search
        out.update({"reference": ref_searches / ref_s, "reference_searches": ref_searches,
                    "reference_seconds": ref_s, "reference_cores": cores})
    print(json.dumps(out))


if __name__ == "__main__":
    main()
