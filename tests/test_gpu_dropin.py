"""Drop-in boundary: the unmodified G2S `qs` program (compiled from the G2S
sources, oracle/_ref/qs) loads this project's g2s_cuda.so through its own
`-W_CUDA` dlopen path and simulates with it."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden

pytestmark = pytest.mark.gpu

QS = os.path.join(ROOT, "oracle", "_ref", "qs")
DROPIN_DIR = os.path.join(ROOT, "g2s_b200", "dropin")


def _cleanup(names):
    for name in names:
        for ext in (".bgrid", ".bgrid.gz"):
            try:
                os.remove(f"/tmp/G2S/data/{name}{ext}")
            except OSError:
                pass


def run_qs_dropin(g, job):
    from oracle import ref
    if not (os.path.exists(QS) and os.path.exists(os.path.join(DROPIN_DIR, "g2s_cuda.so"))):
        pytest.fail("oracle/_ref/qs or g2s_b200/dropin/g2s_cuda.so missing (build them with __graft_entry__.build)")
    types = [int(t) for t in g["types"]]
    outputs = [str(job), f"id_{job}", f"im_1_{job}", f"im_2_{job}"]
    _cleanup(outputs)
    ref.write_image(f"dropin_ti_{job}", g["ti"], types)
    ref.write_image(f"dropin_di_{job}", g["di"], types)
    log = f"/tmp/G2S/logs/dropin_{job}.log"
    cmd = [QS, "-ti", f"dropin_ti_{job}", "-di", f"dropin_di_{job}", "-k", str(float(g["k"])), "-n", str(int(g["n"])),
           "-s", str(int(g["seed"])), "-j", "1", "-W_CUDA", "0", "-id", str(job), "-r", log]
    r = subprocess.run(cmd, cwd=DROPIN_DIR, capture_output=True, text=True, timeout=600)
    text = open(log).read() if os.path.exists(log) else ""
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:], text[-2000:])
    sim = ref.read_image(str(job))
    idx = ref.read_image("id_" + str(job))
    _cleanup(outputs + [f"dropin_ti_{job}", f"dropin_di_{job}"])
    if idx.dtype != np.uint32:
        idx = idx.view(np.uint32)
    assert sim.shape == g["di"].shape
    return sim, idx, text


def test_qs_w_cuda_equals_reference_cpu():
    g = golden("grf2d_small")
    sim, idx, log = run_qs_dropin(g, 31001)
    assert "Could not load g2s_cuda.so" not in log
    assert np.array_equal(sim, g["sim"])
    assert np.array_equal(idx.ravel(), g["idx"].ravel())


@pytest.mark.parametrize("name", ["cat2d_small", "bivar2d_small", "grf3d_small"])
def test_qs_w_cuda_equals_oracle(oracle, name):
    g = golden(name)
    types = [int(t) for t in g["types"]]
    job = {"cat2d_small": 31011, "bivar2d_small": 31012, "grf3d_small": 31013}[name]
    sim, idx, log = run_qs_dropin(g, job)
    o = oracle.simulate(g["ti"], g["di"], types, int(g["n"]), float(g["k"]), int(g["seed"]), mode=0)
    assert np.array_equal(sim, o["sim"])
    assert np.array_equal(idx.ravel(), o["id"])


def test_qs_w_cuda_no_verbatim_equals_reference():
    g = golden("grf2d_nv")
    from oracle import ref
    types = [0]
    job = 31020
    outputs = [str(job), f"id_{job}", f"im_1_{job}", f"im_2_{job}"]
    _cleanup(outputs)
    ref.write_image(f"dropin_ti_{job}", g["ti"], types)
    ref.write_image(f"dropin_di_{job}", g["di"], types)
    log = f"/tmp/G2S/logs/dropin_{job}.log"
    cmd = [QS, "-ti", f"dropin_ti_{job}", "-di", f"dropin_di_{job}", "-k", str(float(g["k"])), "-n", str(int(g["n"])),
           "-s", str(int(g["seed"])), "-j", "1", "-nV", "-W_CUDA", "0", "-id", str(job), "-r", log]
    r = subprocess.run(cmd, cwd=DROPIN_DIR, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:])
    sim = ref.read_image(str(job))
    _cleanup(outputs + [f"dropin_ti_{job}", f"dropin_di_{job}"])
    assert np.array_equal(sim, g["sim"])


def test_qs_w_cuda_missing_data_equals_oracle(oracle):
    g = golden("grf2d_holes")
    sim, idx, log = run_qs_dropin(g, 31021)
    o = oracle.simulate(g["ti"], g["di"], [0], int(g["n"]), float(g["k"]), int(g["seed"]), mode=0)
    assert np.array_equal(sim, o["sim"]) and np.array_equal(idx.ravel(), o["id"])


def test_auto_qs_w_cuda_calibration_agrees_with_oracle(oracle):
    """The unmodified G2S auto_qs (oracle/_ref/auto_qs_cuda: src/auto_qs.cpp
    with its -W_CUDA dlopen path) calibrating on the drop-in device: every
    distribution() query, with the verbatim exclusion of the sample's
    neighbourhood (radius (cells*0.005)^(1/2) here), runs on the GPU.  The
    program seeds its generators from the clock, so its estimates are
    compared statistically with the oracle's calibration: without pruning
    every setup collects the same number of samples, and every mean error
    agrees within a few standard errors."""
    from oracle import ref
    from g2s_b200 import synthetic as syn
    exe = os.path.join(ROOT, "oracle", "_ref", "auto_qs_cuda")
    if not (os.path.exists(exe) and os.path.exists(os.path.join(DROPIN_DIR, "g2s_cuda.so"))):
        pytest.fail("oracle/_ref/auto_qs_cuda or g2s_b200/dropin/g2s_cuda.so missing (__graft_entry__.build)")
    ti = syn.grf((48, 48), (5, 5), seed=21)
    r = np.arange(11) - 5
    kernel = np.exp(-(r[:, None] ** 2 + r[None, :] ** 2) / 20.0).astype(np.float32)
    max_n, dens, max_k, iters = 6, [0.1, 0.5], 2, 1500
    job = 31030
    # auto_qs ignores -id: its outputs are im_1/2/3_4294967295 (src/auto_qs.cpp:758-760)
    outputs = [f"im_{i}_4294967295" for i in (1, 2, 3)]
    _cleanup(outputs)
    ref.write_image(f"dropin_ti_{job}", ti, [0])
    ref.write_image(f"dropin_k_{job}", kernel, [0])
    log = f"/tmp/G2S/logs/dropin_{job}.log"
    cmd = [exe, "-ti", f"dropin_ti_{job}", "-ki", f"dropin_k_{job}", "-maxk", str(max_k), "-maxn", str(max_n),
           "-densities"] + [str(d) for d in dens] + ["-maxIter", str(iters), "-minIter", str(iters), "-j", "1",
                                                   "-W_CUDA", "0", "-r", log]
    # auto_qs falls back to CPU devices without a word when the dlopen fails:
    # the loader's own trace shows that the drop-in and this library were loaded
    env = dict(os.environ, LD_DEBUG="files")
    p = subprocess.run(cmd, cwd=DROPIN_DIR, capture_output=True, text=True, timeout=600, env=env)
    text = open(log).read() if os.path.exists(log) else ""
    assert p.returncode == 0, (p.stdout[-2000:], p.stderr[-2000:], text[-2000:])
    assert "could not load" not in text
    inits = [ln for ln in p.stderr.splitlines() if "calling init:" in ln]
    assert any("g2s_cuda.so" in ln for ln in inits) and any("libg2s_b200.so" in ln for ln in inits), inits[-20:]
    rm, rd, rn = (ref.read_image(name) for name in outputs)
    rm, rd = rm.astype(np.float64), rd.astype(np.float64)
    rn = (rn.view(np.uint32) if rn.dtype == np.float32 else rn).astype(np.float64)
    _cleanup(outputs + [f"dropin_ti_{job}", f"dropin_k_{job}"])
    counts = np.arange(1, max_n, dtype=np.uint32)[:, None]
    om, od, on, _ = oracle.calibrate(ti, [0], [kernel], counts, dens, max_k=max_k, power=2.0, max_iter=iters,
                                     min_iter=iters, seed=5)
    rm, rd, rn = (a.reshape(om.shape) for a in (rm, rd, rn))
    assert np.abs(rn - on).max() <= 0.02 * iters, (rn, on)
    ok = (rn > 30) & (on > 30)
    m1, m2 = om[ok].astype(np.float64) ** 2, rm[ok] ** 2
    z = np.abs(m1 - m2) / np.sqrt(od[ok].astype(np.float64) ** 4 / on[ok] + rd[ok] ** 4 / rn[ok])
    assert ok.sum() >= 10
    assert np.all(z < 5.0), (z.max(), m1, m2)


@pytest.mark.parametrize("name,job", [("multi_ti", 31040), ("multi_ti_ii", 31041), ("multi_ti3", 31042),
                                      ("multi_ti_eq", 31043)])
def test_qs_w_cuda_several_training_images_equal_oracle(oracle, name, job):
    """Several training images (`-ti a b [c]`, and `-ii`, the TI each cell
    samples from): the unmodified G2S `qs -W_CUDA` gives every TI its own
    device of this library (src/qs.cpp:1560-1598), asks each for its k best
    with the same seed and merges them itself (quantileSamplingModule.hpp:
    90-126; the index image is index * nTI + TI, simulation.hpp:658).  The
    simulation and index image equal the oracle's several-TI simulation bit
    for bit (the oracle is pinned to the reference in
    test_oracle_multi_ti.py)."""
    from oracle import ref
    g = golden(name)
    types = [int(t) for t in g["types"]]
    nti = int(g["nti"])
    tis = [f"dropin_ti{i}_{job}" for i in range(nti)]
    for i, nm in enumerate(tis):
        ref.write_image(nm, g[f"ti{i}"], types)
    ref.write_image(f"dropin_di_{job}", g["di"], types)
    outputs = [str(job), f"id_{job}", f"im_1_{job}", f"im_2_{job}"]
    _cleanup(outputs)
    log = f"/tmp/G2S/logs/dropin_{job}.log"
    cmd = [QS, "-ti", tis[0], "-di", f"dropin_di_{job}", "-k", str(float(g["k"])), "-n", str(int(g["n"])),
           "-s", str(int(g["seed"])), "-j", "1", "-W_CUDA", "0", "-id", str(job), "-r", log]
    for nm in tis[1:]:
        cmd += ["-ti", nm]
    extra = []
    if "ii" in g:
        ref.write_image(f"dropin_ii_{job}", g["ii"], [0])
        cmd += ["-ii", f"dropin_ii_{job}"]
        extra.append(f"dropin_ii_{job}")
    r = subprocess.run(cmd, cwd=DROPIN_DIR, capture_output=True, text=True, timeout=600)
    text = open(log).read() if os.path.exists(log) else ""
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:], text[-2000:])
    assert "Could not load g2s_cuda.so" not in text
    sim = ref.read_image(str(job))
    idx = ref.read_image("id_" + str(job))
    _cleanup(outputs + tis + [f"dropin_di_{job}"] + extra)
    if idx.dtype != np.uint32:
        idx = idx.view(np.uint32)
    o = oracle.simulate_multi([g[f"ti{i}"] for i in range(nti)], g["di"], types, int(g["n"]), float(g["k"]),
                              int(g["seed"]), ii=g.get("ii"))
    assert np.array_equal(sim, o["sim"])
    assert np.array_equal(idx.ravel(), o["id"])
    assert len(np.unique(idx.ravel() % nti)) > 1   # candidates come from more than one TI
