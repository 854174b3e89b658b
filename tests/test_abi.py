"""C ABI boundary: the library loads without a GPU, exports every entry point
declared in include/g2s_b200.h, and its host-only planning helpers agree with
the oracle."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "g2s_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(qsk_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(g2s):
    L = g2s.lib()
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) == set(g2s.SIGNATURES), "Python bindings and header disagree"
    out = subprocess.run(["nm", "-D", "--defined-only", g2s.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (qsk_[a-z0-9_]+)", out))
    assert set(names) <= exported


def test_library_is_sm100a():
    out = subprocess.run(["/usr/local/cuda/bin/cuobjdump", "--list-elf", os.path.join(ROOT, "g2s_b200", "libg2s_b200.so")],
                         capture_output=True, text=True).stdout
    assert "sm_100a" in out


def test_device_count_without_gpu_is_safe(g2s):
    assert g2s.device_count() >= 0


@pytest.mark.parametrize("kd", [[101, 101], [126, 126], [31, 26, 21], [1501]])
def test_template_matches_oracle(g2s, oracle, kd):
    a, w = g2s.search_template(kd)
    b = oracle.template(kd)
    assert np.array_equal(a, b)
    assert np.all(w == 1.0)


def test_template_with_kernel_weights(g2s, oracle):
    rng = np.random.default_rng(0)
    kern = rng.random((9, 11)).astype(np.float32)
    kern[0, 0] = np.nan
    a, w = g2s.search_template([11, 9], kernel=kern)
    b = oracle.template([11, 9], kernel=kern)
    assert np.array_equal(a, b)
    # weights are looked up with the kernel centred at dims/2
    for (ox, oy), wt in zip(a[:20], w[:20, 0]):
        assert wt == kern[9 // 2 + oy, 11 // 2 + ox]


@pytest.mark.parametrize("shape,seed", [((200, 200), 100), ((30, 40, 2), 7), ((8, 9, 10), 5)])
def test_path_matches_oracle(g2s, oracle, shape, seed):
    nvar = 2 if len(shape) == 3 and shape[-1] == 2 else 1
    di = np.full(shape, np.nan, np.float32)
    di.reshape(-1)[::37] = 1.0
    o1, s1, b1 = g2s.random_path(di, nvar, seed)
    o2, s2, p2, b2 = oracle.path(di, nvar, seed)
    assert b1 == b2 and np.array_equal(o1, o2) and np.array_equal(s1, s2)


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    import g2s_b200
    monkeypatch.setattr(g2s_b200, "_lib", None)
    monkeypatch.setattr(g2s_b200, "LIB_PATH", str(tmp_path / "nope.so"))
    with pytest.raises(RuntimeError):
        g2s_b200.lib()


def test_jobs_run_checks_arguments_without_a_gpu(g2s):
    L = g2s.lib()
    assert L.qsk_jobs_run(None, 0, 0, None) == 0
    assert L.qsk_jobs_run(None, 1, 0, None) != 0
    assert L.qsk_jobs_run(None, -1, 0, None) != 0
    arr = (__import__("ctypes").c_void_p * 2)(None, None)
    assert L.qsk_jobs_run(arr, 2, 2, None) != 0
    assert b"null simulation" in L.qsk_last_error()


def test_kept_blocks_without_a_gpu(g2s):
    """Nothing kept before any simulation ends; limit and release need no GPU."""
    g2s.blocks_set_limit(1 << 30)
    g2s.blocks_release()
    info = g2s.blocks_info(0)
    assert info["bytes"] == 0 and info["blocks"] == 0
    g2s.blocks_set_limit(8 << 30)


def test_qs_needs_a_training_image(g2s):
    """qs() takes one training image or a list (-ti a b ...); an empty list is
    refused before any device work."""
    with pytest.raises(ValueError):
        g2s.qs([], np.full((8, 8), np.nan, np.float32), [0], k=1.2, n=4, s=1)
