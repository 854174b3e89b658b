"""Per-pattern parity: map + k-best of the CUDA path against the oracle (bit
for bit: same FP32 term order, same reservoir tie-breaking), against FP64
(tolerance 1e-5 of the term scale) and the reference's self-match KAT."""
import zlib

import numpy as np
import pytest

from g2s_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

TOL = 1e-5


def make_terms(offsets, values, types):
    """Terms exactly as the simulation builds them (uniform kernel weight 1):
    continuous (SQLIN, -w, 2*(w*v)); categorical (EQ, w, v); NaN skipped."""
    from g2s_b200 import QSK_OP_SQLIN, QSK_OP_EQ
    terms = []
    for j in range(len(offsets)):
        for v, t in enumerate(types):
            x = values[j][v]
            if np.isnan(x):
                continue
            if t == 0:
                terms.append((j, v, QSK_OP_SQLIN, -1.0, float(np.float32(2.0) * np.float32(x))))
            else:
                terms.append((j, v, QSK_OP_EQ, 1.0, float(x)))
    return terms


def random_pattern(rng, ti, types, n, radius, nd):
    nvar = len(types)
    n = min(n, (2 * radius + 1) ** nd)   # distinct offsets available in the box
    offs = [np.zeros(nd, np.int32)]
    seen = {tuple(offs[0])}
    while len(offs) < n:
        o = rng.integers(-radius, radius + 1, nd).astype(np.int32)
        if tuple(o) not in seen:
            seen.add(tuple(o))
            offs.append(o)
    offs = np.array(offs)
    vals = np.empty((n, nvar), np.float32)
    flat = ti.reshape(-1, nvar)
    for j in range(n):
        vals[j] = flat[rng.integers(0, flat.shape[0])]
    vals[0] = np.nan  # the node itself: uninformed
    return offs, vals


def oracle_kbest(oracle, ti, types, offs, vals, k, seed):
    m32, m64, sc, mn, mx = oracle.pattern_map(ti, types, offs, vals)
    v, p = oracle.kbiggest(m32, k, seed)
    return v, p, mn, m32, m64, sc


CASES = [
    ("grf2d", lambda: syn.grf((120, 100), (10, 10), seed=3), [0], 2),
    ("cat2d", lambda: syn.channels2d((90, 110), n_channels=8, seed=2), [1], 2),
    ("bivar2d", lambda: syn.bivariate(syn.grf((70, 80), (8, 8), seed=5)), [0, 1], 2),
    ("grf3d", lambda: syn.grf((20, 24, 28), (5, 6, 6), seed=9), [0], 3),
    ("grf1d", lambda: syn.grf((900,), (15,), seed=4), [0], 1),
]


@pytest.mark.parametrize("name,mk,types,nd", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("k", [1, 2, 3, 5, 16])
def test_pattern_kbest_bit_exact(g2s, gpu, oracle, name, mk, types, nd, k):
    ti = mk()
    rng = np.random.default_rng(zlib.crc32(f"{name}-{k}".encode()))
    T = g2s.TrainingImage(ti, types)
    W = g2s.Worker(T)
    for trial in range(6):
        n = int(rng.integers(1, 40))
        offs, vals = random_pattern(rng, ti, types, n, radius=int(rng.integers(1, 9)), nd=nd)
        seed = float(np.float32(rng.random()))
        sc, ix, mn = W.pattern_kbest(offs, make_terms(offs, vals, types), k, seed)
        v, p, omn, m32, m64, scale = oracle_kbest(oracle, ti, types, offs, vals, k, seed)
        assert np.array_equal(mn, omn)
        assert np.array_equal(sc, v), (trial, sc, v)
        assert np.array_equal(ix, p), (trial, ix, p)
        finite = np.isfinite(m64)
        err = np.abs(m32[finite].astype(np.float64) - m64[finite])
        assert np.all(err <= TOL * np.maximum(scale[finite], 1e-30) + 1e-30)


def test_layers_form_equals_grid_form(g2s, gpu, oracle):
    """Reference-format layers (TI^2 and TI, flipped) with LIN terms — what the
    drop-in device receives from G2S — give the same bits as the fused form."""
    ti = syn.grf((64, 72), (8, 8), seed=11)
    T = g2s.TrainingImage(ti, [0])
    W = g2s.Worker(T)
    flat = ti.reshape(-1)
    lay1 = flat[::-1].copy()             # flipped TI (fft == src)
    lay0 = (lay1 * lay1).astype(np.float32)
    L = g2s.TrainingImage.from_layers([lay0, lay1], src_size=[72, 64], fft_size=[72, 64])
    WL = g2s.Worker(L)
    rng = np.random.default_rng(0)
    for _ in range(5):
        offs, vals = random_pattern(rng, ti, [0], 25, 6, 2)
        terms = make_terms(offs, vals, [0])
        lin = []
        for (j, v, op, a, b) in terms:
            lin.append((j, 0, g2s.QSK_OP_LIN, a, 0.0))
            lin.append((j, 1, g2s.QSK_OP_LIN, b, 0.0))
        s1, i1, m1 = W.pattern_kbest(offs, terms, 2, 0.3)
        s2, i2, m2 = WL.pattern_kbest(offs, lin, 2, 0.3)
        assert np.array_equal(s1, s2) and np.array_equal(i1, i2)


@pytest.mark.parametrize("nd,shape", [(1, (1500,)), (2, (128, 256)), (3, (24, 32, 40))])
def test_self_match_kat(g2s, gpu, nd, shape):
    """Idea of the reference KAT (G2S src/test.cpp:191-457): a TI cell's own
    neighbourhood (the cell itself left out) finds that cell as best match."""
    rng = np.random.default_rng(1)
    ti = rng.random(shape).astype(np.float32)
    T = g2s.TrainingImage(ti, [0])
    W = g2s.Worker(T)
    tpl, _ = g2s.search_template([9] * nd)
    dims = list(reversed(shape))
    for _ in range(30):
        c = [int(rng.integers(5, d - 5)) for d in dims]
        offs = tpl[:20]
        vals = np.empty((20, 1), np.float32)
        for j, o in enumerate(offs):
            idx = tuple(reversed([c[d] + o[d] for d in range(nd)]))
            vals[j, 0] = ti[idx]
        vals[0, 0] = np.nan
        sc, ix, mn = W.pattern_kbest(offs, make_terms(offs, vals, [0]), 2, 0.0)
        pos = T.index_to_position(mn, int(ix[0]))
        flat_c = 0
        for d in reversed(range(nd)):
            flat_c = flat_c * dims[d] + c[d]
        assert pos == flat_c


def test_degenerate_pattern_wider_than_ti(g2s, gpu, oracle):
    """Fewer valid positions than k: masked entries become candidates
    (the reference's -inf handling); compare with the oracle."""
    ti = syn.grf((6, 7), (2, 2), seed=1)
    T = g2s.TrainingImage(ti, [0])
    W = g2s.Worker(T)
    offs = np.array([[0, 0], [5, 4], [-1, 0]], np.int32)   # extent 6x4 -> 1 valid position in 7x6
    vals = np.array([[np.nan], [0.3], [-0.2]], np.float32)
    for k in (1, 2, 4):
        sc, ix, mn = W.pattern_kbest(offs, make_terms(offs, vals, [0]), k, 0.77)
        v, p, omn, *_ = oracle_kbest(oracle, ti, [0], offs, vals, k, 0.77)
        assert np.array_equal(sc, v) and np.array_equal(ix, p)


def test_empty_pattern_gives_minus_inf(g2s, gpu):
    ti = syn.grf((16, 16), (3, 3), seed=1)
    W = g2s.Worker(g2s.TrainingImage(ti, [0]))
    sc, ix, mn = W.pattern_kbest(np.zeros((0, 2), np.int32), [], 2, 0.5)
    assert np.all(np.isneginf(sc))


def test_batch_equals_single(g2s, gpu):
    import ctypes
    ti = syn.channels2d((60, 70), n_channels=5, seed=4)
    T = g2s.TrainingImage(ti, [1])
    W = g2s.Worker(T)
    rng = np.random.default_rng(5)
    pats = [random_pattern(rng, ti, [1], int(rng.integers(2, 30)), 5, 2) for _ in range(7)]
    seeds = rng.random(7).astype(np.float32)
    single = [W.pattern_kbest(o, make_terms(o, v, [1]), 2, float(s)) for (o, v), s in zip(pats, seeds)]
    nb_ptr = np.cumsum([0] + [len(o) for o, _ in pats]).astype(np.int32)
    allterms = [make_terms(o, v, [1]) for o, v in pats]
    term_ptr = np.cumsum([0] + [len(t) for t in allterms]).astype(np.int32)
    offs = np.concatenate([o for o, _ in pats]).astype(np.int32)
    flat = [t for ts in allterms for t in ts]
    tarr = (g2s.QskTerm * len(flat))(*[g2s.QskTerm(*t) for t in flat])
    out_s = np.zeros(14, np.float32)
    out_i = np.zeros(14, np.uint32)
    out_m = np.zeros(14, np.int32)
    rc = g2s.lib().qsk_pattern_kbest_batch(W.handle, 7, g2s._p(nb_ptr, g2s._i32p), g2s._p(offs, g2s._i32p),
                                           g2s._p(term_ptr, g2s._i32p), tarr, 2, g2s._p(seeds, g2s._f32p),
                                           g2s._p(out_s, g2s._f32p), g2s._p(out_i, g2s._u32p), g2s._p(out_m, g2s._i32p))
    assert rc == 0
    for b, (sc, ix, mn) in enumerate(single):
        assert np.array_equal(out_s[2 * b:2 * b + 2], sc) and np.array_equal(out_i[2 * b:2 * b + 2], ix)
        assert np.array_equal(out_m[2 * b:2 * b + 2], mn)


@pytest.mark.parametrize("mode", [0, 1])
def test_categorical_bit_and_float_kernels_agree(g2s, gpu, oracle, mode):
    """Unit-weight categorical patterns run on the bit-sliced kernel (mode 0)
    or the FP32 gather kernel (mode 1); both equal the oracle bit for bit."""
    ti = syn.channels2d((100, 130), n_channels=9, seed=7)
    T = g2s.TrainingImage(ti, [1])
    W = g2s.Worker(T)
    rng = np.random.default_rng(42)
    g2s.set_map_mode(mode)
    try:
        for trial in range(8):
            n = int(rng.integers(2, 90))
            offs, vals = random_pattern(rng, ti, [1], n, radius=7, nd=2)
            seed = float(np.float32(rng.random()))
            for k in (1, 2, 4):
                sc, ix, mn = W.pattern_kbest(offs, make_terms(offs, vals, [1]), k, seed)
                v, p, *_ = oracle_kbest(oracle, ti, [1], offs, vals, k, seed)
                assert np.array_equal(sc, v) and np.array_equal(ix, p), (trial, k)
    finally:
        g2s.set_map_mode(0)


def test_missing_data_pattern_scores(g2s, gpu):
    """Training image with missing values: every valid position's score
    -|S / c^4| (S the masked squared mismatch, c the informed overlap times
    the centre mask; -inf where c == 0) against a direct numpy evaluation."""
    rng = np.random.default_rng(3)
    ti = rng.standard_normal((7, 9)).astype(np.float32)
    ti[2, 3] = np.nan
    ti[5, 6] = np.nan
    T = g2s.TrainingImage(ti, [0])
    W = g2s.Worker(T)
    offs = np.array([[0, 0], [1, 0], [-1, 2]], np.int32)
    vals = np.array([np.nan, 0.4, -1.1], np.float32)
    # reference-format layers: TI^2 (NaN->0), TI (NaN->0), mask; flipped (fft == src)
    flat = ti.reshape(-1)
    m = (~np.isnan(flat)).astype(np.float32)
    t0 = np.where(np.isnan(flat), 0, flat).astype(np.float32)
    L = g2s.TrainingImage.from_layers([(t0 * t0)[::-1].copy(), t0[::-1].copy(), m[::-1].copy()],
                                      src_size=[9, 7], fft_size=[9, 7])
    WL = g2s.Worker(L)
    terms = []
    for j in (1, 2):
        w, v = np.float32(1), vals[j]
        terms += [(j, 0, g2s.QSK_OP_LIN, float(-w), 0.0), (j, 1, g2s.QSK_OP_LIN, float(2 * w * v), 0.0),
                  (j, 2, g2s.QSK_OP_LIN, float(-(w * v) * v), 0.0), (j, 2, g2s.QSK_OP_LIN_CROSS, float(w), 0.0)]
    K = 16
    sc, ix, mn = WL.pattern_kbest(offs, terms, K, 0.5, missing_data=True, centre_mask_layer=2)
    expect = []
    for py in range(7):
        for px in range(9):
            ok = all(0 <= px + ox < 9 and 0 <= py + oy < 7 for ox, oy in offs)
            if not ok:
                continue
            reg, c = 0.0, 0.0
            for (ox, oy), v in zip(offs[1:], vals[1:]):
                t = ti[py + oy, px + ox]
                if np.isnan(t):
                    continue
                reg += -(t - v) ** 2
                c += 1
            if np.isnan(ti[py, px]):
                c = 0
            expect.append(-np.inf if c == 0 else -abs(reg / c ** 4))
    expect = np.sort(np.array(expect, np.float64))[::-1][:K]
    got = sc.astype(np.float64)
    assert np.allclose(got[np.isfinite(expect)], expect[np.isfinite(expect)], rtol=1e-5, atol=1e-7), (got, expect)


def test_missing_data_exclusion_over_masked_positions(g2s, gpu, oracle):
    """-nV with a training image with missing values: the excluded scan index
    is -inf after the -|S/c^4| compensation, also where it falls on the NaN
    border (quantileSamplingModule.hpp:559-571 writes it into the error
    array).  A -inf there takes part in the reservoir's ties while fewer than
    K finite values have been seen, a NaN never does.  Integer TI values and
    pattern values make every score exact in FP32, so the expected map is
    built here and run through the oracle's k-biggest; every scan index is
    tried as the excluded one."""
    rng = np.random.default_rng(11)
    ti = rng.integers(0, 3, (7, 9)).astype(np.float32)
    ti[2, 3] = np.nan
    ti[5, 6] = np.nan
    ti[0, 1] = np.nan
    ny, nx = ti.shape
    offs = np.array([[0, 0], [1, 0], [-1, 2]], np.int32)
    vals = np.array([np.nan, 1.0, 2.0], np.float32)
    flat = ti.reshape(-1)
    m = (~np.isnan(flat)).astype(np.float32)
    t0 = np.where(np.isnan(flat), 0, flat).astype(np.float32)
    L = g2s.TrainingImage.from_layers([(t0 * t0)[::-1].copy(), t0[::-1].copy(), m[::-1].copy()],
                                      src_size=[nx, ny], fft_size=[nx, ny])
    W = g2s.Worker(L)
    terms = []
    for j in (1, 2):
        v = float(vals[j])
        terms += [(j, 0, g2s.QSK_OP_LIN, -1.0, 0.0), (j, 1, g2s.QSK_OP_LIN, 2.0 * v, 0.0),
                  (j, 2, g2s.QSK_OP_LIN, -v * v, 0.0), (j, 2, g2s.QSK_OP_LIN_CROSS, 1.0, 0.0)]
    mn = offs.min(axis=0)
    mx = offs.max(axis=0)
    N = nx * ny
    base = np.full(N, np.nan, np.float32)
    valid = np.zeros(N, bool)
    for i in range(N):
        ix, iy = i % nx, i // nx
        # scan index -> TI cell (cvtIndexToPosition with fft == src)
        px = (nx - ix - mn[0] - 1 + nx) % nx
        py = (ny - iy - mn[1] - 1 + ny) % ny
        if ix < mx[0] - mn[0] or iy < mx[1] - mn[1]:
            continue
        valid[i] = True
        S, c = 0.0, 0.0
        for (ox, oy), v in zip(offs[1:], vals[1:]):
            t = ti[py + oy, px + ox]
            if np.isnan(t):
                continue
            S -= (float(t) - float(v)) ** 2
            c += 1.0
        if np.isnan(ti[py, px]):
            c = 0.0
        base[i] = -np.inf if c == 0 else -abs(np.float32(S) / np.float32(c ** 4))
    sensitive = 0
    for K in (1, 3, 8):
        for seed in (0.25, 0.8125):
            for x in range(N):
                ref = base.copy()
                ref[x] = -np.inf
                ev, ep = oracle.kbiggest(ref, K, seed)
                sc, ix, _ = W.pattern_kbest(offs, terms, K, seed, exclude_index=x, missing_data=True,
                                            centre_mask_layer=2)
                assert np.array_equal(sc, ev) and np.array_equal(ix, ep), (K, seed, x, sc, ev, ix, ep)
                if not valid[x]:
                    nv, npos = oracle.kbiggest(base, K, seed)
                    sensitive += int(not (np.array_equal(nv, ev) and np.array_equal(npos, ep)))
    # the case where -inf and NaN differ is met
    assert sensitive > 0
    W.close()
    L.close()
