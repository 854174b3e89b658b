"""auto_qs calibration (f3) on the CPU: the oracle's restatement of
QuantileSamplingModule::distribution (the calibration's per-sample search:
weighted map, verbatim exclusion of the sample's own neighbourhood with the
reference's radius, reservoir k-best) against the reference itself, run
in-process from oracle/_ref/libg2sref.so; and the calibration loop's host
logic in the oracle.

The reference's AVX complex multiply-add (include/complexMulti.hpp:163-194)
adds the last four frequency bins twice when ny*(nx/2+1) is 4..7 modulo 8, so
its maps are wrong for such TI shapes (60x60, 50x50, 250x250, ...); the
comparisons use shapes where that product is a multiple of 8."""
import zlib

import numpy as np
import pytest

from g2s_b200 import synthetic as syn

TOL = 1e-5


@pytest.fixture(scope="module")
def ref():
    from oracle import ref as R
    if not R.available():
        pytest.fail("oracle/_ref/libg2sref.so is missing: run `make -C oracle`")
    return R


def gauss_kernel(side, scale, nvar=1):
    r = np.arange(side) - side // 2
    k = np.exp(-(r[:, None] ** 2 + r[None, :] ** 2) / scale).astype(np.float32)
    return np.repeat(k[..., None], nvar, axis=-1) if nvar > 1 else k


def sample_pattern(rng, ti, nvar, n, half):
    """n distinct offsets in the (2 half+1)^2 box around a random cell, with the
    TI's values there (as the calibration samples them)."""
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
    ("cat64x48", lambda: syn.channels2d((48, 64), n_channels=6, seed=3), [1]),
    ("bivar48", lambda: syn.bivariate(syn.grf((48, 48), (5, 5), seed=7)), [0, 1]),
]


@pytest.mark.parametrize("name,mk,types", CASES, ids=[c[0] for c in CASES])
def test_distribution_equals_reference(oracle, ref, name, mk, types):
    ti = mk()
    nvar = len(types)
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    kernel = gauss_kernel(21, 60.0, nvar)
    ny, nx = ti.shape[:2]
    radius_ref = float(np.float32((ny * nx * 0.005) ** 0.5))
    exact = 0
    for trial in range(16):
        n = int(rng.integers(2, 30))
        origin, offs, vals = sample_pattern(rng, ti, nvar, n, 10)
        k = int(rng.integers(1, 6))
        seed = float(np.float32(rng.random()))
        radius = [0.0, 2.5, radius_ref, 7.0][trial % 4]
        sc, ix, pos, mn, m32, m64, scale = oracle.distribution(ti, types, kernel, offs, vals, k, seed, origin, radius,
                                                               maps=True)
        rp = ref.distribution(ti, types, kernel, offs, vals, k, seed, origin, radius)
        if np.array_equal(pos, rp):
            exact += 1
            continue
        # the reference's FFT scores may order near-equal candidates differently
        ours = np.sort(m64[ix])[::-1]
        ref_idx = [int(i) for i in ix]   # FP64 scores of the reference's picks, via their scan indices
        for q, p in enumerate(rp):
            hit = np.nonzero(pos == p)[0]
            if hit.size:
                ref_idx[q] = int(ix[hit[0]])
            else:
                cand = np.nonzero((m32 > -np.inf))[0]
                flat = [c for c in cand if oracle_position(oracle, ti, types, kernel, offs, vals, c, mn) == p]
                ref_idx[q] = flat[0] if flat else -1
        assert -1 not in ref_idx, (name, trial, pos, rp)
        theirs = np.sort(m64[ref_idx])[::-1]
        gap = np.abs(ours - theirs) / np.maximum(scale[ix], 1e-30)
        assert np.all(gap <= TOL), (name, trial, pos, rp, ours, theirs)
    # categorical scores tie exactly (homogeneous neighbourhoods); the
    # reference's FFT rounding then decides where the reservoir decides here
    if 1 not in types:
        assert exact >= 12, (name, exact)


def oracle_position(oracle, ti, types, kernel, offs, vals, index, mn):
    """TI position of scan index `index` for a pattern with minimum mn
    (CPUThreadDevice::cvtIndexToPosition on an unpadded scan)."""
    nvar = len(types)
    spatial = ti.shape if nvar == 1 else ti.shape[:-1]
    dims = list(reversed(spatial))
    N = int(np.prod(dims))
    pos, div = 0, N
    for i in reversed(range(len(dims))):
        div //= dims[i]
        f = dims[i]
        pos = pos * dims[i] + ((f - (index // div) % f - int(mn[i]) - 1) + dims[i]) % dims[i]
    return pos


def test_distribution_radius_marks(oracle):
    """Every scan index of the radius marks is -inf in the map, the others keep
    their scores; radius < 1 excludes the origin's index only."""
    ti = syn.grf((40, 40), (5, 5), seed=4)
    kernel = np.ones((11, 11), np.float32)
    rng = np.random.default_rng(3)
    origin, offs, vals = sample_pattern(rng, ti, 1, 8, 5)
    base = oracle.distribution(ti, [0], kernel, offs, vals, 1, 0.5, 0xFFFFFFFF, 0.0, maps=True)[4]
    one = oracle.distribution(ti, [0], kernel, offs, vals, 1, 0.5, origin, 0.5, maps=True)[4]
    wide = oracle.distribution(ti, [0], kernel, offs, vals, 1, 0.5, origin, 3.0, maps=True)[4]
    valid = base > -np.inf
    assert np.sum(valid & (one == -np.inf)) == 1
    changed = valid & (wide == -np.inf)
    assert 1 < changed.sum() <= 49
    assert np.array_equal(wide[valid & ~changed], base[valid & ~changed])


def test_calibrate_oracle_is_deterministic(oracle):
    ti = syn.grf((40, 40), (5, 5), seed=8)
    kernels = [gauss_kernel(11, 20.0), np.ones((7, 7), np.float32)]
    counts = np.arange(1, 7, dtype=np.uint32)[:, None]
    kw = dict(max_k=2, power=2.0, noise=0.0, max_iter=12, min_iter=4, seed=11)
    a = oracle.calibrate(ti, [0], kernels, counts, [0.1, 0.5], **kw)
    b = oracle.calibrate(ti, [0], kernels, counts, [0.1, 0.5], **kw)
    for x, y in zip(a[:3], b[:3]):
        assert np.array_equal(x, y, equal_nan=True)
    mean, dev, ns, searches = a
    assert searches > 0 and ns.max() <= 12
    assert np.all(mean[ns > 0] >= 0)


def test_default_neighbour_counts(g2s):
    c = g2s.default_neighbour_counts([80, 40])
    assert c.shape == (79, 2)
    assert list(c[0]) == [1, 0] and list(c[-1]) == [79, 39] and list(c[2]) == [3, 1]
