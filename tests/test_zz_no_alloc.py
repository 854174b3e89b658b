"""qsk_pattern_kbest_noalloc (device scratch in a fixed array, no allocation)
against qsk_pattern_kbest through the C ABI: same scores and scan indices,
on two calls in a row per pattern (the second call reuses the scratch the
first one left behind), on both map kernels (FP32 gather and bit-sliced).
Collected last so that it also runs after every other GPU test."""
import ctypes
import zlib

import numpy as np
import pytest

from g2s_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

_f32p = ctypes.POINTER(ctypes.c_float)
_u32p = ctypes.POINTER(ctypes.c_uint)
_i32p = ctypes.POINTER(ctypes.c_int)
QSK_ERR_UNSUPPORTED = 4   # include/g2s_b200.h


def _terms(g2s, offsets, values, types):
    out = []
    for j in range(len(offsets)):
        for v, t in enumerate(types):
            x = values[j][v]
            if np.isnan(x):
                continue
            if t == 0:
                out.append((j, v, g2s.QSK_OP_SQLIN, -1.0, float(np.float32(2.0) * np.float32(x))))
            else:
                out.append((j, v, g2s.QSK_OP_EQ, 1.0, float(x)))
    return out


def _pattern(rng, ti, types, n, radius, nd):
    n = min(n, (2 * radius + 1) ** nd)
    offs = [np.zeros(nd, np.int32)]
    seen = {tuple(offs[0])}
    while len(offs) < n:
        o = rng.integers(-radius, radius + 1, nd).astype(np.int32)
        if tuple(o) not in seen:
            seen.add(tuple(o))
            offs.append(o)
    flat = ti.reshape(-1, len(types))
    vals = flat[rng.integers(0, flat.shape[0], n)].astype(np.float32)
    vals[0] = np.nan
    return np.array(offs, np.int32), vals


def _noalloc(g2s, T, offs, terms, k, seed, stream=None):
    offs = np.ascontiguousarray(offs, np.int32)
    tarr = (g2s.QskTerm * max(len(terms), 1))(*[g2s.QskTerm(int(t[0]), int(t[1]), int(t[2]), float(t[3]),
                                                            float(t[4])) for t in terms])
    sc = np.zeros(k, np.float32)
    ix = np.zeros(k, np.uint32)
    mn = np.zeros(T.ndim, np.int32)
    rc = g2s.lib().qsk_pattern_kbest_noalloc(T.handle, stream, offs.shape[0], offs.ctypes.data_as(_i32p), len(terms),
                                             tarr, k, seed, sc.ctypes.data_as(_f32p), ix.ctypes.data_as(_u32p),
                                             mn.ctypes.data_as(_i32p))
    return rc, sc, ix, mn


CASES = [
    ("grf2d", lambda: syn.grf((120, 100), (10, 10), seed=3), [0], 2),
    ("cat2d", lambda: syn.channels2d((90, 110), n_channels=8, seed=2), [1], 2),
    ("bivar2d", lambda: syn.bivariate(syn.grf((70, 80), (8, 8), seed=5)), [0, 1], 2),
    ("grf3d", lambda: syn.grf((20, 24, 28), (5, 6, 6), seed=9), [0], 3),
]


@pytest.mark.parametrize("name,mk,types,nd", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("k", [1, 3, 16])
def test_noalloc_equals_pattern_kbest(g2s, gpu, name, mk, types, nd, k):
    ti = mk()
    rng = np.random.default_rng(zlib.crc32(f"noalloc-{name}-{k}".encode()))
    T = g2s.TrainingImage(ti, types)
    W = g2s.Worker(T)
    for trial in range(4):
        offs, vals = _pattern(rng, ti, types, int(rng.integers(1, 40)), int(rng.integers(1, 9)), nd)
        terms = _terms(g2s, offs, vals, types)
        seed = float(np.float32(rng.random()))
        sc, ix, mn = W.pattern_kbest(offs, terms, k, seed)
        for call in range(2):   # two calls in a row on the same scratch
            rc, sc2, ix2, mn2 = _noalloc(g2s, T, offs, terms, k, seed)
            assert rc == 0, g2s.lib().qsk_last_error()
            # same kernels on the same inputs: equal scores (tolerance 0) and indices
            assert np.array_equal(sc2, sc), (name, k, trial, call, sc2, sc)
            assert np.array_equal(ix2, ix), (name, k, trial, call)
            assert np.array_equal(mn2, mn)
    W.close()
    T.close()


def test_noalloc_on_a_stream(g2s, gpu):
    """A caller's stream (here one made by torch) instead of the default stream."""
    torch = pytest.importorskip("torch")
    ti = syn.grf((64, 64), (6, 6), seed=11)
    T = g2s.TrainingImage(ti, [0])
    W = g2s.Worker(T)
    rng = np.random.default_rng(5)
    s = torch.cuda.Stream(device=0)
    for _ in range(2):
        offs, vals = _pattern(rng, ti, [0], 20, 4, 2)
        terms = _terms(g2s, offs, vals, [0])
        sc, ix, _ = W.pattern_kbest(offs, terms, 4, 0.375)
        rc, sc2, ix2, _ = _noalloc(g2s, T, offs, terms, 4, 0.375, stream=ctypes.c_void_p(s.cuda_stream))
        assert rc == 0, g2s.lib().qsk_last_error()
        assert np.array_equal(sc2, sc) and np.array_equal(ix2, ix)
    W.close()
    T.close()


def test_noalloc_rejects_a_training_image_beyond_the_scratch(g2s, gpu):
    """8 bytes per position: 1500 x 1500 positions need more than 16 MiB."""
    ti = np.random.default_rng(1).standard_normal((1500, 1500)).astype(np.float32)
    T = g2s.TrainingImage(ti, [0])
    offs = np.array([[0, 0], [1, 0]], np.int32)
    terms = [(1, 0, g2s.QSK_OP_SQLIN, -1.0, 0.5)]
    rc, *_ = _noalloc(g2s, T, offs, terms, 1, 0.5)
    assert rc == QSK_ERR_UNSUPPORTED
    assert b"scratch" in g2s.lib().qsk_last_error()
    T.close()


def test_noalloc_rejects_too_many_terms(g2s, gpu):
    ti = syn.grf((40, 40), (5, 5), seed=2)
    T = g2s.TrainingImage(ti, [0])
    offs = np.array([[0, 0], [1, 0]], np.int32)
    terms = [(1, 0, g2s.QSK_OP_LIN, 1.0, 0.0)] * 2049
    rc, *_ = _noalloc(g2s, T, offs, terms, 1, 0.5)
    assert rc == QSK_ERR_UNSUPPORTED
    T.close()
