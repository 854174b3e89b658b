"""auto_qs calibration (f3): the oracle's calibration loop against the
reference's own auto_qs program (built from the G2S sources into
oracle/_ref/auto_qs).  The reference seeds its generators from the clock and
hands setups to OpenMP threads dynamically, so its estimates are compared
statistically: without pruning (min iterations = max iterations) every setup
collects the same number of samples in both, and the mean error of every
(configuration, density, candidate rank) must agree within a few standard
errors."""
import os
import subprocess

import numpy as np
import pytest

from g2s_b200 import synthetic as syn

HERE = os.path.dirname(os.path.abspath(__file__))
AUTO_QS = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "auto_qs")


@pytest.fixture(scope="module")
def ref():
    from oracle import ref as R
    if not (R.available() and os.path.exists(AUTO_QS)):
        pytest.fail("oracle/_ref/auto_qs is missing: run `make -C oracle`")
    return R


def test_calibration_means_agree_with_reference(oracle, ref):
    ti = syn.grf((48, 48), (5, 5), seed=21)      # ny*(nx/2+1) = 1200, a multiple of 8
    r = np.arange(11) - 5
    kernel = np.exp(-(r[:, None] ** 2 + r[None, :] ** 2) / 20.0).astype(np.float32)
    max_n, dens, max_k, iters = 6, [0.1, 0.5], 2, 1500
    tag = f"calref{os.getpid()}"
    ref.write_image(tag + "_ti", ti, [0])
    ref.write_image(tag + "_k", kernel, [0])
    data = "/tmp/G2S/data"
    outs = [os.path.join(data, f"im_{i}_4294967295.bgrid{z}") for i in (1, 2, 3) for z in ("", ".gz")]
    for f in outs:
        if os.path.exists(f):
            os.remove(f)
    # the program reads its grids from, and writes im_1/2/3_<id> (id -1) to, its
    # working directory, the G2S data directory
    cmd = [AUTO_QS, "-ti", tag + "_ti", "-ki", tag + "_k", "-maxk", str(max_k), "-maxn", str(max_n), "-densities"] + \
        [str(d) for d in dens] + ["-maxIter", str(iters), "-minIter", str(iters), "-j", "4", "-r",
                                  f"/tmp/G2S/logs/{tag}.log"]
    p = subprocess.run(cmd, cwd=data, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    rm = ref.read_image("im_1_4294967295").astype(np.float64)
    rd = ref.read_image("im_2_4294967295").astype(np.float64)
    rn = ref.read_image("im_3_4294967295")
    rn = (rn.view(np.uint32) if rn.dtype == np.float32 else rn).astype(np.float64)   # unsigned counts
    for f in outs:
        if os.path.exists(f):
            os.remove(f)
    counts = np.arange(1, max_n, dtype=np.uint32)[:, None]
    om, od, on, _ = oracle.calibrate(ti, [0], [kernel], counts, dens, max_k=max_k, power=2.0, max_iter=iters,
                                     min_iter=iters, seed=5)
    # reference images: dims (configs, kernels, densities), max_k variables -> numpy (d, k, c, rank)
    rm, rd, rn = (a.reshape(om.shape) for a in (rm, rd, rn))
    assert np.array_equal(rn, on) or np.abs(rn - on).max() <= 0.02 * iters, (rn, on)
    ok = (rn > 30) & (on > 30)
    # squared error means (power 2) and their standard errors
    m1, m2 = om[ok].astype(np.float64) ** 2, rm[ok] ** 2
    se1 = od[ok].astype(np.float64) ** 4 / on[ok]
    se2 = rd[ok] ** 4 / rn[ok]
    z = np.abs(m1 - m2) / np.sqrt(se1 + se2)
    assert ok.sum() >= 10
    assert np.all(z < 5.0), (z.max(), m1, m2)
