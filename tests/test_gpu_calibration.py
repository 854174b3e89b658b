"""auto_qs calibration (f3) on the GPU against the oracle, bit for bit: the
batched queries with the verbatim exclusion of distribution() (one index, or
the reference's radius marks), and the whole calibration loop (same setups,
same per-setup generators, same batched order)."""
import zlib

import numpy as np
import pytest

from g2s_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def gauss_kernel(side, scale, nvar=1):
    r = np.arange(side) - side // 2
    k = np.exp(-(r[:, None] ** 2 + r[None, :] ** 2) / scale).astype(np.float32)
    return np.repeat(k[..., None], nvar, axis=-1) if nvar > 1 else k


def kweight(kernel, nvar, off, v):
    """kernel weight of offset off for variable v, centred at dims/2 (0 outside)"""
    k = kernel if kernel.ndim == 3 else kernel[..., None]
    ky, kx = k.shape[:2]
    cx, cy = kx // 2 + off[0], ky // 2 + off[1]
    if not (0 <= cx < kx and 0 <= cy < ky):
        return np.float32(0.0)
    return np.float32(k[cy, cx, v % k.shape[2]])


def terms_of(offs, vals, types, kernel, g2s):
    """The simulation's conversion with kernel weights: continuous
    (SQLIN, -w, 2*(w*v)); categorical (EQ, w, v); NaN values and zero weights
    left out."""
    out = []
    for j in range(len(offs)):
        for v, t in enumerate(types):
            x = np.float32(vals[j][v])
            if np.isnan(x):
                continue
            w = kweight(kernel, len(types), offs[j], v)
            if w == 0:
                continue
            if t == 0:
                out.append((j, v, g2s.QSK_OP_SQLIN, float(-w), float(np.float32(2.0) * np.float32(w * x))))
            else:
                out.append((j, v, g2s.QSK_OP_EQ, float(w), float(x)))
    return out


def sample_pattern(rng, ti, nvar, n, half):
    ny, nx = ti.shape[:2]
    flat = ti.reshape(ny * nx, nvar)
    origin = int(rng.integers(0, ny * nx))
    oy, ox = divmod(origin, nx)
    offs, vals, seen = [], [], set()
    while len(offs) < n:
        o = (int(rng.integers(-half, half + 1)), int(rng.integers(-half, half + 1)))
        y, x = oy + o[1], ox + o[0]
        if o in seen or not (0 <= y < ny and 0 <= x < nx):
            continue
        seen.add(o)
        offs.append(o)
        vals.append(flat[y * nx + x])
    return origin, np.array(offs, np.int32), np.array(vals, np.float32)


CASES = [
    ("grf64", lambda: syn.grf((64, 64), (6, 6), seed=2), [0]),
    ("grf90x70", lambda: syn.grf((70, 90), (6, 6), seed=5), [0]),
    ("cat64x48", lambda: syn.channels2d((48, 64), n_channels=6, seed=3), [1]),
    ("bivar48", lambda: syn.bivariate(syn.grf((48, 48), (5, 5), seed=7)), [0, 1]),
]


@pytest.mark.parametrize("name,mk,types", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("k", [1, 3, 8])
def test_verbatim_batch_equals_oracle(g2s, gpu, oracle, name, mk, types, k):
    ti = mk()
    nvar = len(types)
    rng = np.random.default_rng(zlib.crc32(f"{name}-{k}".encode()))
    kernel = gauss_kernel(21, 60.0, nvar)
    ny, nx = ti.shape[:2]
    T = g2s.TrainingImage(ti, types)
    W = g2s.Worker(T)
    pats, seeds, origins, radii, raw = [], [], [], [], []
    for b in range(24):
        origin, offs, vals = sample_pattern(rng, ti, nvar, int(rng.integers(2, 40)), 10)
        pats.append((offs, terms_of(offs, vals, types, kernel, g2s)))
        seeds.append(np.float32(rng.random()))
        origins.append(origin if b % 6 else 0xFFFFFFFF)
        radii.append([0.0, 0.9, 2.5, float(np.float32((ny * nx * 0.005) ** 0.5)), 6.0, 11.0][b % 6])
        raw.append((offs, vals))
    sc, ix, mn = W.pattern_kbest_verbatim(pats, k, seeds, origins, radii)
    for b, (offs, vals) in enumerate(raw):
        osc, oix, opos, omn = oracle.distribution(ti, types, kernel, offs, vals, k, float(seeds[b]), origins[b],
                                                  radii[b])
        assert np.array_equal(mn[b], omn), (name, k, b)
        assert np.array_equal(sc[b], osc), (name, k, b, sc[b], osc)
        assert np.array_equal(ix[b], oix), (name, k, b, ix[b], oix)
        pos = [g2s.lib().qsk_index_to_position(T.handle, g2s._p(mn[b], g2s._i32p), int(i)) for i in ix[b]]
        assert list(pos) == [int(p) for p in opos], (name, k, b)
    W.close()
    T.close()


@pytest.mark.parametrize("k", [1, 4])
def test_single_query_radius_option_equals_oracle(g2s, gpu, oracle, k):
    """qsk_pattern_kbest_ex with exclude_radius (what the drop-in device does
    for setValueInErrorArrayWithRadius under auto_qs -W_CUDA): the scan index
    of the origin and every index the reference's radius recursion marks
    around it are -inf; equal to the oracle's distribution()."""
    ti = syn.grf((64, 64), (6, 6), seed=2)
    rng = np.random.default_rng(100 + k)
    kernel = gauss_kernel(21, 60.0)
    T = g2s.TrainingImage(ti, [0])
    W = g2s.Worker(T)
    for trial in range(12):
        origin, offs, vals = sample_pattern(rng, ti, 1, int(rng.integers(2, 40)), 10)
        radius = [1.0, 2.5, 4.5, 11.0][trial % 4]
        seed = float(np.float32(rng.random()))
        mn = np.minimum(offs.min(axis=0), 0).astype(np.int32)
        idx = g2s.lib().qsk_position_to_index(T.handle, g2s._p(mn, g2s._i32p), origin)
        sc, ix, gmn = W.pattern_kbest(offs, terms_of(offs, vals, [0], kernel, g2s), k, seed, exclude_index=idx,
                                      exclude_radius=radius)
        osc, oix, opos, omn = oracle.distribution(ti, [0], kernel, offs, vals, k, seed, origin, radius)
        assert np.array_equal(gmn, omn)
        assert np.array_equal(sc, osc), (trial, sc, osc)
        assert np.array_equal(ix, oix), (trial, ix, oix)
    W.close()
    T.close()


@pytest.mark.parametrize("noise", [0.0, 0.4])
def test_calibrate_equals_oracle(g2s, gpu, oracle, noise):
    ti = syn.grf((64, 64), (6, 6), seed=12)
    kernels = [gauss_kernel(15, 30.0), np.ones((9, 9), np.float32)]
    counts = g2s.default_neighbour_counts(10)
    dens = [0.05, 0.3, 1.0]
    kw = dict(max_k=3, power=2.0, noise=noise, seed=7)
    m, d, n, s = g2s.calibrate(ti, [0], kernels, counts, dens, max_iterations=25, min_iterations=8, **kw)
    om, od, on, os_ = oracle.calibrate(ti, [0], kernels, counts, dens, max_iter=25, min_iter=8, **kw)
    assert s == os_ and s > 0
    assert np.array_equal(n, on)
    assert np.array_equal(m, om, equal_nan=True)
    assert np.array_equal(d, od, equal_nan=True)
    # pruning took effect: some setups stopped before the last iteration
    assert n[..., 0].min() < n[..., 0].max()


def test_calibrate_categorical_bivariate_equals_oracle(g2s, gpu, oracle):
    ti = syn.bivariate(syn.grf((48, 48), (5, 5), seed=3))
    kernels = [gauss_kernel(11, 20.0, 2)]
    counts = g2s.default_neighbour_counts([8, 4])
    kw = dict(max_k=2, power=1.0, noise=0.0, seed=3)
    m, d, n, s = g2s.calibrate(ti, [0, 1], kernels, counts, [0.2, 0.6], max_iterations=15, min_iterations=5, **kw)
    om, od, on, os_ = oracle.calibrate(ti, [0, 1], kernels, counts, [0.2, 0.6], max_iter=15, min_iter=5, **kw)
    assert s == os_
    assert np.array_equal(n, on)
    assert np.array_equal(m, om, equal_nan=True)
    assert np.array_equal(d, od, equal_nan=True)
