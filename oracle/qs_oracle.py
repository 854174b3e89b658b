"""Test infrastructure only: Python access to the CPU oracle (qs_oracle.cpp).

The oracle restates the G2S reference QuickSampling path (see the header of
``qs_oracle.cpp`` for the file:line of every step).  Tests, the smoke check
and the CPU-baseline leg of bench.py use it as the checker; the product never
imports it.
"""
from __future__ import annotations

import ctypes
import os
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libqsoracle.so")
_lib = None

_f32p = ctypes.POINTER(ctypes.c_float)
_u32p = ctypes.POINTER(ctypes.c_uint)
_i32p = ctypes.POINTER(ctypes.c_int)
_f64p = ctypes.POINTER(ctypes.c_double)


def available() -> bool:
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB)
        L.orc_template.argtypes = [ctypes.c_int, _u32p, _f32p, ctypes.c_int, _i32p, ctypes.c_int]
        L.orc_template.restype = ctypes.c_int
        L.orc_path.argtypes = [ctypes.c_int, _u32p, ctypes.c_int, _f32p, ctypes.c_uint, _u32p, _f32p, _u32p]
        L.orc_path.restype = ctypes.c_int
        L.orc_path_full.argtypes = L.orc_path.argtypes
        L.orc_path_full.restype = ctypes.c_int
        L.orc_kbiggest.argtypes = [_f32p, ctypes.c_uint, ctypes.c_uint, ctypes.c_float, _f32p, _u32p]
        L.orc_rng.argtypes = [ctypes.c_uint, ctypes.c_int, _f32p]
        L.orc_seed_from_unit_float.argtypes = [ctypes.c_float]
        L.orc_seed_from_unit_float.restype = ctypes.c_uint
        L.orc_selected_index.argtypes = [ctypes.c_float, ctypes.c_float, ctypes.c_uint]
        L.orc_selected_index.restype = ctypes.c_uint
        L.orc_simulate.argtypes = [ctypes.c_int, ctypes.c_int, _u32p, ctypes.c_int, _i32p, _f32p, _u32p, _f32p, _f32p,
                                   _u32p,
                                   _f32p, ctypes.c_int, ctypes.c_float, ctypes.c_uint, ctypes.c_int, ctypes.c_double,
                                   ctypes.c_long, ctypes.c_long, _u32p, _i32p, _i32p, _f64p, _u32p, ctypes.c_int,
                                   _u32p, _u32p, _f64p]
        L.orc_simulate.restype = ctypes.c_long
        L.orc_simulate_ex.argtypes = L.orc_simulate.argtypes + [ctypes.c_void_p]
        L.orc_simulate_ex.restype = ctypes.c_long
        L.orc_simulate_multi.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _u32p, ctypes.c_int, _i32p,
                                         ctypes.POINTER(ctypes.c_void_p), _u32p, _f32p, _f32p, _u32p, _f32p,
                                         ctypes.c_int, ctypes.c_float, ctypes.c_uint, _f32p, ctypes.c_double, _u32p,
                                         _u32p, _u32p, _i32p, _i32p]
        L.orc_simulate_multi.restype = ctypes.c_long
        L.orc_pattern_map.argtypes = [ctypes.c_int, _u32p, ctypes.c_int, _i32p, _f32p, ctypes.c_int, _i32p, _f32p,
                                      _f32p, _f64p, _f64p, _i32p, _i32p]
        L.orc_pattern_map.restype = ctypes.c_long
        _lib = L
    return _lib


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


def grid_dims(arr: np.ndarray, nvar: int):
    spatial = arr.shape if nvar == 1 else arr.shape[:-1]
    return np.array(list(reversed(spatial)), dtype=np.uint32)


def template(kdims, kernel=None, nvar=1):
    kd = np.asarray(kdims, dtype=np.uint32)
    cap = int(np.prod(kd))
    out = np.zeros(cap * len(kd), dtype=np.int32)
    kern = None if kernel is None else np.ascontiguousarray(kernel, dtype=np.float32)
    n = lib().orc_template(len(kd), _p(kd, _u32p), _p(kern, _f32p), nvar, _p(out, _i32p), cap)
    return out[: n * len(kd)].reshape(n, len(kd))


def path(di: np.ndarray, nvar: int, seed: int, full: bool = False):
    """(order, seeds, posterior, begin); with ``full`` (-fs) over the
    cells*nvar values instead of the cells."""
    dims = grid_dims(di, nvar)
    cells = int(np.prod(dims)) * (nvar if full else 1)
    d = np.ascontiguousarray(di, dtype=np.float32)
    order = np.zeros(cells, np.uint32)
    seeds = np.zeros(cells, np.float32)
    post = np.zeros(cells, np.uint32)
    fn = lib().orc_path_full if full else lib().orc_path
    begin = fn(len(dims), _p(dims, _u32p), nvar, _p(d, _f32p), seed, _p(order, _u32p), _p(seeds, _f32p),
               _p(post, _u32p))
    return order, seeds, post, begin


def kbiggest(data: np.ndarray, k: int, seed: float):
    d = np.ascontiguousarray(data, dtype=np.float32)
    out = np.zeros(k, np.float32)
    pos = np.zeros(k, np.uint32)
    lib().orc_kbiggest(_p(d, _f32p), d.size, k, seed, _p(out, _f32p), _p(pos, _u32p))
    return out, pos


def rng_stream(seed: int, n: int):
    out = np.zeros(n, np.float32)
    lib().orc_rng(seed, n, _p(out, _f32p))
    return out


class _Controls(ctypes.Structure):
    _fields_ = [("n_counts", ctypes.c_int), ("n_per_var", ctypes.c_void_p), ("ni_vars", ctypes.c_int),
                ("ni", ctypes.c_void_p), ("kvi", ctypes.c_void_p), ("n_kernels", ctypes.c_int),
                ("kernels_dims", ctypes.c_void_p), ("kernels", ctypes.c_void_p), ("kii", ctypes.c_void_p),
                ("full", ctypes.c_int)]


def _controls(cells, n_per_var=None, ni=None, kvi=None, kernels=None, kii=None, full=False):
    """Local controls (-n per variable, -ni, -kvi, -kii with its kernels, -fs);
    returns (struct, keep-alive list) or (None, []) when none is given."""
    if n_per_var is None and ni is None and kvi is None and kernels is None and kii is None and not full:
        return None, []
    c = _Controls()
    c.full = int(full)
    keep = []

    def arr(a, dt):
        x = np.ascontiguousarray(a, dtype=dt)
        keep.append(x)
        return x.ctypes.data

    if n_per_var is not None:
        c.n_counts = len(n_per_var)
        c.n_per_var = arr(n_per_var, np.int32)
    if ni is not None:
        ni = np.asarray(ni, np.float32)
        c.ni_vars = max(1, ni.size // cells)
        c.ni = arr(ni, np.float32)
    if kvi is not None:
        c.kvi = arr(kvi, np.float32)
    if kernels is not None:
        # list of (weights array with numpy shape (..., ky, kx[, nvar]), dims x-first)
        dims = []
        ptrs = (ctypes.c_void_p * len(kernels))()
        for q, (w, kd) in enumerate(kernels):
            ptrs[q] = arr(w, np.float32)
            dims += list(kd)
        keep.append(ptrs)
        c.n_kernels = len(kernels)
        c.kernels_dims = arr(dims, np.uint32)
        c.kernels = ctypes.cast(ptrs, ctypes.c_void_p).value
    if kii is not None:
        c.kii = arr(kii, np.float32)
    keep.append(c)
    return c, keep


def simulate_multi(tis, di, types, n, k, seed, ii=None, kernel=None, kdims=None, mode=0, di_init=None, tol=1e-5):
    """Vector simulation with several training images, as G2S runs it with
    one accelerator device per TI: per node every TI's k best (or only the
    -ii image's TI), scored as the CUDA device reports them, merged with
    std::sort and drawn with the TI count.  mode 0: sequential simulation of
    ``di``; mode 1: every path node teacher-forced against the completed grid
    ``di`` (path from ``di_init``) with its FP64 near-tie flag.  Returns
    dict(sim, id, ti, cell, near_tie, marginal, begin); id = TI cell *
    len(tis) + TI; the per-node arrays are in path order."""
    nvar = len(types)
    dims = [grid_dims(t, nvar) for t in tis]
    nd = len(dims[0])
    assert all(len(d) == nd for d in dims)
    tdims = np.concatenate(dims).astype(np.uint32)
    arrs = [np.ascontiguousarray(t, dtype=np.float32) for t in tis]
    ptrs = (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
    ddims = grid_dims(di, nvar)
    d = np.ascontiguousarray(di, dtype=np.float32).copy()
    init = d if di_init is None else np.ascontiguousarray(di_init, dtype=np.float32)
    cells = int(np.prod(ddims))
    nodes = cells - int(np.sum(~np.isnan(init.reshape(cells, nvar)).any(axis=1)))
    ty = np.asarray(types, dtype=np.int32)
    oid = np.zeros(cells, np.uint32)
    oti = np.zeros(max(nodes, 1), np.uint32)
    ocell = np.zeros(max(nodes, 1), np.uint32)
    ont = np.zeros(max(nodes, 1), np.int32)
    omg = np.zeros(max(nodes, 1), np.int32)
    iiw = None if ii is None else np.ascontiguousarray(ii, dtype=np.float32).ravel()
    kd = None if kdims is None else np.asarray(kdims, dtype=np.uint32)
    kern = None if kernel is None else np.ascontiguousarray(kernel, dtype=np.float32)
    rc = lib().orc_simulate_multi(int(mode), nd, len(arrs), _p(tdims, _u32p), nvar, _p(ty, _i32p), ptrs,
                                  _p(ddims, _u32p), _p(d, _f32p), None if di_init is None else _p(init, _f32p),
                                  _p(kd, _u32p), _p(kern, _f32p), int(n), float(k), int(seed), _p(iiw, _f32p),
                                  float(tol), _p(oid, _u32p), _p(oti, _u32p), _p(ocell, _u32p), _p(ont, _i32p),
                                  _p(omg, _i32p))
    if rc < 0:
        raise ValueError("orc_simulate_multi: training images with missing values are not supported")
    return {"sim": d, "id": oid, "ti": oti[:nodes], "cell": ocell[:nodes], "near_tie": ont[:nodes].astype(bool),
            "marginal": omg[:nodes].astype(bool), "begin": cells - nodes}


def simulate(ti, di, types, n, k, seed, mode=0, kernel=None, kdims=None, want_fp64=False, tol=1e-5,
             node_begin=0, node_end=-1, di_init=None, no_verbatim=False, id_init=None, probe=None,
             n_per_var=None, ni=None, kvi=None, kernels=None, kii=None, full=False):
    """mode 0: sequential vector simulation of ``di`` (NaN = unknown);
    mode 1: teacher-forced evaluation of every path node against the completed
    grid ``di``, the path being built from ``di_init`` (the grid before
    simulation).  ``no_verbatim`` is -nV; in mode 1 it needs ``id_init``, the
    index image of the completed grid.  Local controls: ``n_per_var`` (-n
    with one count per variable), ``ni`` (-ni image, numpy shape of the grid
    [, counts]), ``kvi`` (-kvi image), ``kernels`` (list of (weights, dims
    x-first), the -ki files) with ``kii`` (-kii image of kernel indices).

    Returns dict(sim, id, cell, near_tie, marginal, gap, begin)."""
    nvar = len(types)
    tdims = grid_dims(ti, nvar)
    ddims = grid_dims(di, nvar)
    t = np.ascontiguousarray(ti, dtype=np.float32)
    d = np.ascontiguousarray(di, dtype=np.float32).copy()
    ty = np.asarray(types, dtype=np.int32)
    cells = int(np.prod(ddims))
    init = d if di_init is None else np.ascontiguousarray(di_init, dtype=np.float32)
    informed = int(np.sum(~np.isnan(init.reshape(cells, nvar)).any(axis=1)))
    nodes = cells - informed
    ne = nodes if node_end < 0 else min(node_end, nodes)
    cnt = max(ne - node_begin, 0)
    cell = np.zeros(cnt, np.uint32)
    nt = np.zeros(cnt, np.int32)
    mg = np.zeros(cnt, np.int32)
    gap = np.zeros(cnt, np.float64)
    oid = np.zeros(cells, np.uint32)
    kd = None if kdims is None else np.asarray(kdims, dtype=np.uint32)
    kern = None if kernel is None else np.ascontiguousarray(kernel, dtype=np.float32)
    idi = None if id_init is None else np.ascontiguousarray(id_init, dtype=np.uint32).ravel()
    prb = None if probe is None else np.ascontiguousarray(probe, dtype=np.uint32).ravel()
    pcross = np.full(cnt, np.nan, np.float64)
    ctl, keep = _controls(cells, n_per_var, ni, kvi, kernels, kii, full)
    if full:
        oid = np.zeros(cells * nvar, np.uint32)
        nodes = int(np.sum(np.isnan(init)))
        ne = nodes if node_end < 0 else min(node_end, nodes)
        cnt = max(ne - node_begin, 0)
        cell = np.zeros(cnt, np.uint32)
        nt = np.zeros(cnt, np.int32)
        mg = np.zeros(cnt, np.int32)
        gap = np.zeros(cnt, np.float64)
    rc = lib().orc_simulate_ex(mode, len(tdims), _p(tdims, _u32p), nvar, _p(ty, _i32p), _p(t, _f32p), _p(ddims, _u32p),
                       _p(d, _f32p), None if di_init is None else _p(init, _f32p), _p(kd, _u32p), _p(kern, _f32p), n, k, seed, int(want_fp64), tol, node_begin,
                       ne, _p(cell, _u32p), _p(nt, _i32p), _p(mg, _i32p), _p(gap, _f64p), _p(oid, _u32p),
                       int(no_verbatim), _p(idi, _u32p), _p(prb, _u32p), _p(pcross, _f64p),
                       None if ctl is None else ctypes.addressof(ctl))
    if rc == -2:
        raise ValueError("oracle: categorical variables with missing training-image values are undefined")
    if rc == -3:
        raise ValueError("oracle: kernel index image out of range")
    if rc == -4:
        raise ValueError("oracle: -fs is restated for complete training images and mode 0 only")
    return dict(sim=d, id=oid, cell=cell, near_tie=nt.astype(bool), marginal=mg.astype(bool), gap=gap,
                probe_cross=pcross)


def pattern_map(ti, types, offsets, values):
    """FP32 and FP64 maps (scan order) of one explicit pattern; returns (m32, m64, scale, mn, mx)."""
    nvar = len(types)
    tdims = grid_dims(ti, nvar)
    t = np.ascontiguousarray(ti, dtype=np.float32)
    ty = np.asarray(types, dtype=np.int32)
    offs = np.ascontiguousarray(offsets, dtype=np.int32)
    vals = np.ascontiguousarray(values, dtype=np.float32)
    N = int(np.prod(tdims))
    m32 = np.zeros(N, np.float32)
    m64 = np.zeros(N, np.float64)
    sc = np.zeros(N, np.float64)
    mn = np.zeros(len(tdims), np.int32)
    mx = np.zeros(len(tdims), np.int32)
    lib().orc_pattern_map(len(tdims), _p(tdims, _u32p), nvar, _p(ty, _i32p), _p(t, _f32p), offs.shape[0],
                          _p(offs, _i32p), _p(vals, _f32p), _p(m32, _f32p), _p(m64, _f64p), _p(sc, _f64p),
                          _p(mn, _i32p), _p(mx, _i32p))
    return m32, m64, sc, mn, mx


def _kernel_arrays(kernel, nd, nvar):
    """(kdims x-first uint32, knvar, float32 data) of a weight kernel given as
    a numpy array of spatial shape (.., ny, nx) [+ (nvar,) when it has one
    weight per variable]."""
    k = np.ascontiguousarray(kernel, dtype=np.float32)
    if k.ndim == nd + 1:
        knvar = k.shape[-1]
        spatial = k.shape[:-1]
    else:
        knvar = 1
        spatial = k.shape
    return np.array(list(reversed(spatial)), np.uint32), knvar, k


def distribution(ti, types, kernel, offsets, values, k, seed, origin=0xFFFFFFFF, radius=0.0, maps=False):
    """QuantileSamplingModule::distribution on one TI (auto_qs' per-sample search):
    returns (scores, scan indices, TI positions, pattern min) and, with maps=True,
    (map32 after the exclusion, map64, scale)."""
    nvar = len(types)
    tdims = grid_dims(ti, nvar)
    nd = len(tdims)
    t = np.ascontiguousarray(ti, dtype=np.float32)
    ty = np.asarray(types, dtype=np.int32)
    kd, knvar, kk = _kernel_arrays(kernel, nd, nvar)
    offs = np.ascontiguousarray(offsets, dtype=np.int32)
    vals = np.ascontiguousarray(values, dtype=np.float32)
    sc = np.zeros(k, np.float32)
    ix = np.zeros(k, np.uint32)
    pos = np.zeros(k, np.uint32)
    mn = np.zeros(nd, np.int32)
    N = int(np.prod(tdims))
    m32 = np.zeros(N, np.float32) if maps else None
    m64 = np.zeros(N, np.float64) if maps else None
    scl = np.zeros(N, np.float64) if maps else None
    L = lib()
    L.orc_distribution.argtypes = [ctypes.c_int, _u32p, ctypes.c_int, _i32p, _f32p, _u32p, ctypes.c_int, _f32p,
                                   ctypes.c_int, _i32p, _f32p, ctypes.c_uint, ctypes.c_float, ctypes.c_uint,
                                   ctypes.c_float, _f32p, _u32p, _u32p, _i32p, _f32p, _f64p, _f64p]
    L.orc_distribution.restype = ctypes.c_long
    L.orc_distribution(nd, _p(tdims, _u32p), nvar, _p(ty, _i32p), _p(t, _f32p), _p(kd, _u32p), knvar, _p(kk, _f32p),
                       offs.shape[0], _p(offs, _i32p), _p(vals, _f32p), k, seed, int(origin), float(radius),
                       _p(sc, _f32p), _p(ix, _u32p), _p(pos, _u32p), _p(mn, _i32p),
                       _p(m32, _f32p) if maps else None, _p(m64, _f64p) if maps else None,
                       _p(scl, _f64p) if maps else None)
    if maps:
        return sc, ix, pos, mn, m32, m64, scl
    return sc, ix, pos, mn


def calibrate(ti, types, kernels, counts, densities, max_k=1, power=2.0, noise=0.0, max_iter=10, min_iter=1000,
              seed=0):
    """The auto_qs calibration loop (batched setup order, per-setup generators);
    returns (mean, dev, nsamp) shaped (n_densities, n_kernels, n_configs, max_k)
    and the number of searches."""
    nvar = len(types)
    tdims = grid_dims(ti, nvar)
    nd = len(tdims)
    t = np.ascontiguousarray(ti, dtype=np.float32)
    ty = np.asarray(types, dtype=np.int32)
    kds, knv, kdata = [], [], []
    for kern in kernels:
        kd, knvar, kk = _kernel_arrays(kern, nd, nvar)
        kds.append(kd)
        knv.append(knvar)
        kdata.append(kk.ravel())
    kds = np.ascontiguousarray(np.concatenate(kds), np.uint32)
    knv = np.asarray(knv, np.int32)
    kdata = np.ascontiguousarray(np.concatenate(kdata), np.float32)
    cnt = np.ascontiguousarray(np.atleast_2d(np.asarray(counts, np.uint32)))
    den = np.ascontiguousarray(densities, np.float32)
    S = cnt.shape[0] * len(kernels) * den.size
    mean = np.zeros(S * max_k, np.float32)
    dev = np.zeros(S * max_k, np.float32)
    ns = np.zeros(S * max_k, np.uint32)
    L = lib()
    L.orc_calibrate.argtypes = [ctypes.c_int, _u32p, ctypes.c_int, _i32p, _f32p, ctypes.c_int, _u32p, _i32p, _f32p,
                                ctypes.c_int, ctypes.c_int, _u32p, ctypes.c_int, _f32p, ctypes.c_uint, ctypes.c_float,
                                ctypes.c_float, ctypes.c_uint, ctypes.c_uint, ctypes.c_uint, _f32p, _f32p, _u32p]
    L.orc_calibrate.restype = ctypes.c_long
    n = L.orc_calibrate(nd, _p(tdims, _u32p), nvar, _p(ty, _i32p), _p(t, _f32p), len(kernels), _p(kds, _u32p),
                        _p(knv, _i32p), _p(kdata, _f32p), cnt.shape[0], cnt.shape[1], _p(cnt, _u32p), den.size,
                        _p(den, _f32p), max_k, power, noise, max_iter, min_iter, seed, _p(mean, _f32p),
                        _p(dev, _f32p), _p(ns, _u32p))
    shape = (den.size, len(kernels), cnt.shape[0], max_k)
    return mean.reshape(shape), dev.reshape(shape), ns.reshape(shape), n
