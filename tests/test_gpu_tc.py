"""Tensor-core shortlist kernel (tcgen05, BF16 and FP8 E4M3) against a numpy
reference.  Inputs are small integers, exact in both formats, so every FP32
accumulation is exact and the kernel's keys (ordered score, tie hash) must
equal the reference's bit for bit: per range, and for the union of ranges
the overall top W.  Ties are frequent by construction (few distinct values),
so the tie-hash ordering is exercised too."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def tie_hash(seed, pos):
    """numpy restatement of the library's 32-bit tie hash (qsk_internal.h)."""
    m = np.uint64(0xFFFFFFFF)
    x = (np.uint64(seed) ^ ((pos.astype(np.uint64) * np.uint64(0x9E3779B9)) & m)) & m
    x ^= x >> np.uint64(16)
    x = (x * np.uint64(0x7FEB352D)) & m
    x ^= x >> np.uint64(15)
    x = (x * np.uint64(0x846CA68B)) & m
    x ^= x >> np.uint64(16)
    return x


def ordered(f32):
    u = f32.astype(np.float32).view(np.uint32).astype(np.uint64)
    neg = (u & np.uint64(0x80000000)) != 0
    return np.where(neg, (~u) & np.uint64(0xFFFFFFFF), u | np.uint64(0x80000000))


def e4m3_code_table():
    vals = {}
    for c in range(256):
        s, e, m = c >> 7, (c >> 3) & 15, c & 7
        if e == 15 and m == 7:
            continue
        v = (m / 8.0) * 2.0 ** -6 if e == 0 else (1 + m / 8.0) * 2.0 ** (e - 7)
        vals.setdefault(-v if s else v, c)
    return vals


def to_bits(x, fmt):
    if fmt == 0:
        return (x.astype(np.float32).view(np.uint32) >> 16).astype(np.uint16)
    tab = e4m3_code_table()
    return np.vectorize(lambda v: tab[float(v)], otypes=[np.uint8])(x)


def reference(q, r, box, X, Y, W, ranges, qs, qb, ps, seed, n_tiles):
    B, N = q.shape[0], r.shape[0]
    s = (q.astype(np.float64) @ r.astype(np.float64).T) * qs[:, None] * ps[np.arange(N) // 256][None, :] + qb[:, None]
    s32 = s.astype(np.float32)
    p = np.arange(N)
    x, y, z = p % X, (p // X) % Y, p // (X * Y)
    tpr = -(-n_tiles // ranges)
    out = []
    for b in range(B):
        valid = ((x >= box[b, 0]) & (x < box[b, 1]) & (y >= box[b, 2]) & (y < box[b, 3]) & (z >= box[b, 4])
                 & (z < box[b, 5]))
        key = (ordered(s32[b]) << np.uint64(32)) | tie_hash(seed[b], p.astype(np.uint64))
        per = []
        for g in range(ranges):
            lo, hi = g * tpr * 256, min((g + 1) * tpr * 256, N)
            sel = np.nonzero(valid[lo:hi])[0] + lo
            k = key[sel]
            o = sorted(range(len(sel)), key=lambda i: -int(k[i]))[:W]
            per.append({(int(k[i]), int(sel[i])) for i in o})
        out.append(per)
    return out


@pytest.mark.parametrize("fmt,K,W,ranges", [(0, 100, 8, 4), (1, 200, 8, 3), (0, 700, 16, 2), (1, 300, 32, 5),
                                           (0, 64, 32, 1)])
def test_tc_topk_exact_integer_data(g2s, gpu, fmt, K, W, ranges):
    rng = np.random.default_rng(fmt * 100 + K)
    X, Y, Z = 40, 30, 3
    N = X * Y * Z
    B = 200
    q = rng.integers(-3, 4, (B, K)).astype(np.float32)
    r = rng.integers(-2, 3, (N, K)).astype(np.float32)
    r[::7] = r[3]                                  # repeated rows: exact score ties
    qs = (2.0 ** rng.integers(-2, 3, B)).astype(np.float32)
    qb = rng.integers(-50, 50, B).astype(np.float32)
    ps = (2.0 ** rng.integers(-1, 2, -(-N // 256))).astype(np.float32) if fmt == 1 else np.ones(-(-N // 256), np.float32)
    seed = rng.integers(0, 2 ** 32, B, dtype=np.uint64).astype(np.uint32)
    box = np.zeros((B, 6), np.int32)
    box[:, 0] = rng.integers(0, 10, B)
    box[:, 1] = rng.integers(25, X + 1, B)
    box[:, 2] = rng.integers(0, 8, B)
    box[:, 3] = rng.integers(20, Y + 1, B)
    box[:, 4] = rng.integers(0, 2, B)
    box[:, 5] = Z
    keys, pos = g2s.tc_topk(to_bits(q, fmt), to_bits(r, fmt), fmt, X, Y, box, W=W, ranges=ranges, q_scale=qs,
                            q_bias=qb, p_scale=ps if fmt == 1 else None, q_seed=seed)
    n_tiles = -(-N // 256)
    ref = reference(q, r, box, X, Y, W, ranges, qs, qb, ps, seed, n_tiles)
    for b in range(B):
        for g in range(ranges):
            got = {(int(k), int(p)) for k, p in zip(keys[b, g], pos[b, g]) if k != 0}
            assert got == ref[b][g], (b, g)
        allg = sorted({kp for g in range(ranges) for kp in ref[b][g]}, key=lambda t: -t[0])[:W]
        got_all = sorted({(int(k), int(p)) for k, p in zip(keys[b].ravel(), pos[b].ravel()) if k != 0},
                         key=lambda t: -t[0])[:W]
        assert got_all == allg


def bf16_round(x):
    """Round float32 to the nearest-even BF16 value (as float64)."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


@pytest.mark.parametrize("M,N,K", [(1, 1, 1), (5, 7, 3), (130, 70, 100), (300, 257, 384), (1024, 64, 2048),
                                   (17, 384, 256), (256, 256, 64), (129, 128, 65)])
def test_gemm_bf16_matches_float64_of_rounded_operands(g2s, gpu, M, N, K):
    """The encoder's tcgen05 product: every output of bf16(A) bf16(B)^T +
    bias within the FP32-accumulation bound of the float64 product (edges of
    the 128-row, 64/128/256-column tiles and of the 64-element K blocks)."""
    rng = np.random.default_rng(M * 7919 + N * 31 + K)
    a = rng.standard_normal((M, K)).astype(np.float32)
    b = rng.standard_normal((N, K)).astype(np.float32)
    bias = rng.standard_normal(N).astype(np.float32)
    c = g2s.gemm_bf16(a, b, bias)
    ar, br = bf16_round(a), bf16_round(b)
    ref = ar @ br.T + bias.astype(np.float64)
    scale = np.abs(ar) @ np.abs(br).T + np.abs(bias)
    assert np.all(np.abs(c - ref) <= 2e-4 * scale + 1e-6)
    c0 = g2s.gemm_bf16(a, b)
    assert np.all(np.abs(c0 - (ar @ br.T)) <= 2e-4 * (np.abs(ar) @ np.abs(br).T) + 1e-6)
