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
