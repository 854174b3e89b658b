"""Test infrastructure only: runs the G2S reference CPU QuickSampling.

The reference is compiled from the G2S sources by ``oracle/Makefile`` into
``oracle/_ref/libg2sref.so`` (see ``oracle/ref_harness.cpp``).  This module
feeds it numpy grids through the reference's own ``.bgrid`` serialisation
(``/tmp/G2S/data``) and calls its ``g2sQsProgramMain`` (G2S src/qs.cpp:364)
in-process.  Only tests, ``__graft_entry__.smoke`` and the CPU-baseline leg of
``bench.py`` use it, as the checker / baseline — never as the product path.
"""
from __future__ import annotations

import ctypes
import os
import re
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libg2sref.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(LIB, mode=ctypes.RTLD_GLOBAL)
        _lib.g2sref_write_image.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_uint), ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_int), ctypes.c_void_p, ctypes.c_int]
        _lib.g2sref_read_image.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_uint),
                                           ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), ctypes.c_void_p,
                                           ctypes.c_long]
        _lib.g2sref_read_image.restype = ctypes.c_long
        _lib.g2sref_qs_main.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p)]
    return _lib


def write_image(name: str, arr: np.ndarray, types, compressed: bool = False) -> None:
    """``arr`` has numpy shape (..., ny, nx[, nvar]) when len(types)>1, else (..., ny, nx)."""
    nvar = len(types)
    a = np.ascontiguousarray(arr, dtype=np.float32)
    spatial = a.shape if nvar == 1 else a.shape[:-1]
    dims = list(reversed(spatial))
    cd = (ctypes.c_uint * len(dims))(*dims)
    ct = (ctypes.c_int * nvar)(*[int(t) for t in types])
    lib().g2sref_write_image(name.encode(), len(dims), cd, nvar, ct, a.ctypes.data, int(compressed))


def read_image(name: str):
    L = lib()
    nd, nv, enc = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    dims = (ctypes.c_uint * 16)()
    n = L.g2sref_read_image(name.encode(), ctypes.byref(nd), dims, ctypes.byref(nv), ctypes.byref(enc), None, 0)
    if n < 0:
        raise FileNotFoundError(name)
    out = np.empty(n, dtype=np.float32)
    L.g2sref_read_image(name.encode(), ctypes.byref(nd), dims, ctypes.byref(nv), ctypes.byref(enc), out.ctypes.data, n)
    shape = tuple(reversed([dims[i] for i in range(nd.value)]))
    if nv.value > 1:
        shape = shape + (nv.value,)
    out = out.reshape(shape)
    if enc.value == 2:
        out = out.view(np.uint32)
    return out


def run_qs(ti: np.ndarray, di: np.ndarray, types, args, job_id: int = 4242, tag: str = "g2sb200", images=None):
    """Run reference ``qs`` with ``-ti``/``-di`` set; returns (sim, index, compute_ms, log_text).

    ``args`` is a list of extra qs flags, e.g. ``['-dt','0','-k','1.2','-n','50','-s','100','-j','8']``.
    ``images`` maps further image flags to lists of (array, types), e.g.
    ``{'-ni': [(ni, [0])], '-ki': [(k1, [0]), (k2, [0])]}``; each array is
    written as a ``.bgrid`` and its name passed after the flag.
    ``compute_ms`` is the reference's own "compuattion time" (G2S src/qs.cpp:2229-2235).
    """
    ti_name = f"{tag}_ti_{job_id}"
    di_name = f"{tag}_di_{job_id}"
    write_image(ti_name, ti, types)
    write_image(di_name, di, types)
    extra_names = []
    extra_args = []
    for flag, items in (images or {}).items():
        extra_args.append(flag)
        for q, (arr, ty) in enumerate(items):
            name = f"{tag}_{flag.strip('-')}{q}_{job_id}"
            write_image(name, arr, ty)
            extra_names.append(name)
            extra_args.append(name)
    log = f"/tmp/G2S/logs/{tag}_{job_id}.log"
    argv = (["qs", "-ti", ti_name, "-di", di_name, "-id", str(job_id), "-r", log] + [str(a) for a in args] +
            extra_args)
    arr = (ctypes.c_char_p * len(argv))(*[a.encode() for a in argv])
    rc = lib().g2sref_qs_main(len(argv), arr)
    if rc != 0:
        raise RuntimeError(f"reference qs returned {rc}")
    sim = read_image(str(job_id))
    idx = read_image("id_" + str(job_id))
    if idx.dtype != np.uint32:
        idx = idx.view(np.uint32)  # importDataIndex is a uint32 buffer (G2S src/qs.cpp:1426)
    text = open(log).read() if os.path.exists(log) else ""
    m = re.findall(r"compuattion time: (\d+) ms", text)
    ms = float(m[-1]) if m else float("nan")
    for name in [ti_name, di_name, str(job_id), "id_" + str(job_id), "im_1_" + str(job_id),
                 "im_2_" + str(job_id)] + extra_names:
        for ext in (".bgrid", ".bgrid.gz"):
            try:
                os.remove(f"/tmp/G2S/data/{name}{ext}")
            except OSError:
                pass
    return sim, idx, ms, text


def distribution(ti, types, kernel, offsets, values, k, seed, origin, radius):
    """The reference's QuantileSamplingModule::distribution (auto_qs' per-sample
    search) on a CPU device: the k TI positions it returns."""
    nvar = len(types)
    a = np.ascontiguousarray(ti, dtype=np.float32)
    spatial = a.shape if nvar == 1 else a.shape[:-1]
    nd = len(spatial)
    dims = np.array(list(reversed(spatial)), np.uint32)
    kk = np.ascontiguousarray(kernel, dtype=np.float32)
    if kk.ndim == nd + 1:
        knvar, kspatial = kk.shape[-1], kk.shape[:-1]
    else:
        knvar, kspatial = 1, kk.shape
    kdims = np.array(list(reversed(kspatial)), np.uint32)
    ty = np.asarray(types, np.int32)
    offs = np.ascontiguousarray(offsets, np.int32)
    vals = np.ascontiguousarray(values, np.float32)
    out = np.zeros(k, np.uint32)
    L = lib()
    u32 = ctypes.POINTER(ctypes.c_uint)
    i32 = ctypes.POINTER(ctypes.c_int)
    f32 = ctypes.POINTER(ctypes.c_float)
    L.g2sref_distribution.argtypes = [ctypes.c_int, u32, ctypes.c_int, i32, f32, u32, ctypes.c_int, f32, ctypes.c_int,
                                      i32, f32, ctypes.c_uint, ctypes.c_float, ctypes.c_uint, ctypes.c_float, u32]
    L.g2sref_distribution(nd, dims.ctypes.data_as(u32), nvar, ty.ctypes.data_as(i32), a.ctypes.data_as(f32),
                          kdims.ctypes.data_as(u32), knvar, kk.ctypes.data_as(f32), offs.shape[0],
                          offs.ctypes.data_as(i32), vals.ctypes.data_as(f32), k, seed, int(origin), float(radius),
                          out.ctypes.data_as(u32))
    return out
