"""Unit checks of the oracle's restated pieces (RNG conversion, k-biggest
reservoir semantics, draw index, template, path)."""
import numpy as np
import pytest


def mt19937_py(seed, n):
    """Independent pure-Python MT19937 (Matsumoto & Nishimura) + the float
    conversion of std::uniform_real_distribution<float> in libstdc++."""
    mt = [0] * 624
    mt[0] = seed & 0xffffffff
    for i in range(1, 624):
        mt[i] = (1812433253 * (mt[i - 1] ^ (mt[i - 1] >> 30)) + i) & 0xffffffff
    idx = 624
    out = []
    for _ in range(n):
        if idx >= 624:
            for k in range(624):
                y = (mt[k] & 0x80000000) | (mt[(k + 1) % 624] & 0x7fffffff)
                mt[k] = mt[(k + 397) % 624] ^ (y >> 1) ^ (0x9908B0DF if y & 1 else 0)
            idx = 0
        y = mt[idx]
        idx += 1
        y ^= y >> 11
        y ^= (y << 7) & 0x9D2C5680
        y ^= (y << 15) & 0xEFC60000
        y ^= y >> 18
        u = np.float32(y) * np.float32(2.0 ** -32)
        if u >= 1:
            u = np.nextafter(np.float32(1), np.float32(0))
        out.append(np.float32(u))
    return np.array(out, dtype=np.float32)


@pytest.mark.parametrize("seed", [0, 1, 5489, 123456789, 0xffffffff])
def test_rng_stream_matches_restated_mt19937(oracle, seed):
    got = oracle.rng_stream(seed, 1500)
    assert np.array_equal(got, mt19937_py(seed, 1500))


def kbiggest_py(data, k, seed):
    """Pure-Python restatement of fKb findKBiggest with generator (fKb.hpp:58-92)."""
    s = oracle_seed(seed)
    stream = iter(mt19937_py(s, 4 * len(data) + 16))
    out = [-np.inf] * k
    pos = [0xffffffff] * k
    cpt = 0
    for i, v in enumerate(np.asarray(data, np.float32)):
        if not v >= out[k - 1]:
            continue
        position = k - 2
        ll = k - 2
        while ll > -1 and out[k - 1] == out[ll]:
            ll -= 1
        xes = k - ll - 1
        x = k - xes + int(np.floor(np.float32(next(stream)) * np.float32(xes)))
        pos[x], pos[k - 1] = pos[k - 1], pos[x]
        if v > out[k - 1]:
            cpt = 0 if xes == 1 else cpt + 1
            while position > -1 and v > out[position]:
                out[position + 1] = out[position]
                pos[position + 1] = pos[position]
                position -= 1
            out[position + 1] = v
            pos[position + 1] = i
        else:
            cpt += 1
            if np.float32(xes + cpt) * np.float32(next(stream)) < np.float32(xes):
                pos[position + 1] = i
    res_v, res_p = [], []
    o = list(out)
    for _ in range(k):
        b = 0
        for l in range(1, k):
            if o[l] > o[b]:
                b = l
        res_v.append(o[b])
        res_p.append(pos[b])
        o[b] = -np.inf
    return np.array(res_v, np.float32), np.array(res_p, np.uint32)


def oracle_seed(seed):
    seed = np.float32(seed)
    if not np.isfinite(seed) or seed <= 0:
        return 0
    if seed >= 1:
        return 0xffffffff
    return int(np.floor(np.float64(seed) * 4294967295.0))


@pytest.mark.parametrize("case", range(12))
def test_kbiggest_reservoir_semantics(oracle, case):
    rng = np.random.default_rng(case)
    n = 300
    if case % 3 == 0:
        data = rng.integers(0, 6, n).astype(np.float32)          # heavy ties
    elif case % 3 == 1:
        data = rng.standard_normal(n).astype(np.float32)
        data[:40] = -np.inf                                       # masked prefix
    else:
        data = np.round(rng.standard_normal(n), 1).astype(np.float32)
    k = [1, 2, 3, 5][case % 4]
    seed = float(rng.random())
    v, p = oracle.kbiggest(data, k, seed)
    v2, p2 = kbiggest_py(data, k, seed)
    assert np.array_equal(v, v2) and np.array_equal(p, p2)


def test_selected_index_formula(oracle):
    # quantileSamplingModule.hpp:113 compiled with the double overloads
    for k in (1.0, 1.2, 1.5, 2.0, 3.7):
        for s in np.linspace(0, 0.9999999, 97, dtype=np.float32):
            expect = int(np.floor(np.float64(np.float32(s) * np.float32(k)) * (np.ceil(np.float64(np.float32(1) / np.float32(k))) / 1)))
            assert oracle.lib().orc_selected_index(float(s), k, 1) == expect


def test_template_nearest_first(oracle):
    t = oracle.template([11, 11])
    d2 = (t ** 2).sum(1)
    assert t.shape == (121, 2) and np.all(np.diff(d2) >= 0) and np.array_equal(t[0], [0, 0])


def test_path_informed_first(oracle):
    di = np.full((10, 12), np.nan, np.float32)
    di[3, 4] = 1.0
    di[7, 1] = 2.0
    order, seeds, post, begin = oracle.path(di, 1, 42)
    assert begin == 2
    assert set(order[:2]) == {3 * 12 + 4, 7 * 12 + 1}
    assert sorted(order) == list(range(120))
    assert np.all((seeds >= 0) & (seeds < 1))
