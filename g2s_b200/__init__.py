"""g2s_b200: B200-native QuickSampling (QS) hot path.

Python access to ``libg2s_b200.so`` (C ABI declared in ``include/g2s_b200.h``).
The CUDA library is the only compute path: importing works without a GPU,
but every call that computes needs the built library and a CUDA device and
raises ``RuntimeError`` otherwise — there is no CPU fallback.

The high-level call mirrors G2S' QuickSampling interface
(``g2s('-a','qs','-ti',ti,'-di',di,'-dt',types,'-k',k,'-n',n,'-s',seed)``,
G2S docs/algorithms/QuickSampling.md:21-37) and returns the simulation and
the index image like the reference does.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libg2s_b200.so")

QSK_OP_LIN, QSK_OP_SQLIN, QSK_OP_EQ, QSK_OP_LIN_CROSS = 0, 1, 2, 3

_lib = None
_f32p = ctypes.POINTER(ctypes.c_float)
_u32p = ctypes.POINTER(ctypes.c_uint)
_i32p = ctypes.POINTER(ctypes.c_int)


class QskTerm(ctypes.Structure):
    _fields_ = [("neighbour", ctypes.c_int), ("layer", ctypes.c_int), ("op", ctypes.c_int),
                ("a", ctypes.c_float), ("b", ctypes.c_float)]


class QskParams(ctypes.Structure):
    _fields_ = [("ndim", ctypes.c_int), ("ti_dims", _u32p), ("nvar", ctypes.c_int), ("types", _i32p),
                ("ti", _f32p), ("di_dims", _u32p), ("kernel_dims", _u32p), ("kernel", _f32p),
                ("n", ctypes.c_int), ("k", ctypes.c_float), ("seed", ctypes.c_uint), ("no_verbatim", ctypes.c_int),
                ("n_counts", ctypes.c_int), ("n_per_variable", _i32p), ("n_image_vars", ctypes.c_int),
                ("n_image", _f32p), ("k_image", _f32p), ("n_kernels", ctypes.c_int), ("kernels_dims", _u32p),
                ("kernels", ctypes.POINTER(_f32p)), ("kernel_index_image", _f32p), ("full_simulation", ctypes.c_int),
                ("n_extra_tis", ctypes.c_int), ("extra_ti_dims", _u32p), ("extra_tis", ctypes.POINTER(_f32p)),
                ("ti_index_image", _f32p)]


class QskPatternOpts(ctypes.Structure):
    _fields_ = [("exclude_index", ctypes.c_int), ("missing_data", ctypes.c_int), ("centre_mask_layer", ctypes.c_int),
                ("exclude_radius", ctypes.c_float)]


class QskCalibParams(ctypes.Structure):
    _fields_ = [("ndim", ctypes.c_int), ("ti_dims", _u32p), ("nvar", ctypes.c_int), ("types", _i32p),
                ("ti", _f32p), ("n_kernels", ctypes.c_int), ("kernel_dims", _u32p), ("kernel_nvar", _i32p),
                ("kernels", ctypes.POINTER(_f32p)), ("n_configs", ctypes.c_int), ("n_counts", ctypes.c_int),
                ("counts", _u32p), ("n_densities", ctypes.c_int), ("densities", _f32p), ("max_k", ctypes.c_uint),
                ("power", ctypes.c_float), ("noise", ctypes.c_float), ("max_iterations", ctypes.c_uint),
                ("min_iterations", ctypes.c_uint), ("max_seconds", ctypes.c_float), ("seed", ctypes.c_uint)]


class QskSimInfo(ctypes.Structure):
    _fields_ = [("nodes", ctypes.c_longlong), ("levels", ctypes.c_int), ("max_batch", ctypes.c_int),
                ("template_size", ctypes.c_int), ("ms_setup_neighbours", ctypes.c_float),
                ("ms_levels", ctypes.c_float), ("ms_batches", ctypes.c_float), ("ms_total", ctypes.c_float),
                ("launches", ctypes.c_longlong), ("map_launches", ctypes.c_longlong), ("ms_map", ctypes.c_float),
                ("ms_prep", ctypes.c_float), ("ms_replay", ctypes.c_float), ("map_positions", ctypes.c_longlong),
                ("tensor_mode", ctypes.c_int), ("tensor_prefix", ctypes.c_int), ("tensor_width", ctypes.c_int),
                ("tensor_shortlist", ctypes.c_int), ("tensor_nodes", ctypes.c_longlong),
                ("plain_nodes", ctypes.c_longlong), ("audited", ctypes.c_longlong), ("regret", ctypes.c_longlong),
                ("regret_near", ctypes.c_longlong), ("map_err_max", ctypes.c_float), ("map_err_mean", ctypes.c_float),
                ("tensor_flops", ctypes.c_double), ("ms_tensor_gemm", ctypes.c_float),
                ("ms_tensor_select", ctypes.c_float), ("ms_tensor_pattern", ctypes.c_float),
                ("tensor_launches", ctypes.c_longlong), ("path_nodes", ctypes.c_longlong),
                ("learned_fallback", ctypes.c_longlong), ("graph_nodes", ctypes.c_longlong),
                ("ms_graph_build", ctypes.c_float)]


class QskLearnedOpts(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int), ("shortlist", ctypes.c_int), ("conf_rank", ctypes.c_int),
                ("audit", ctypes.c_float), ("conf_z", ctypes.c_float), ("conf_r2", ctypes.c_float)]


class QskTensorOpts(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int), ("prefix", ctypes.c_int), ("width", ctypes.c_int),
                ("shortlist", ctypes.c_int), ("audit", ctypes.c_float), ("batch", ctypes.c_int)]


# name -> (restype, argtypes): every entry point of include/g2s_b200.h
SIGNATURES = {
    "qsk_last_error": (ctypes.c_char_p, []),
    "qsk_device_count": (ctypes.c_int, [_i32p]),
    "qsk_ti_create_layers": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _u32p, _u32p, ctypes.c_int,
                                            ctypes.POINTER(_f32p), ctypes.POINTER(ctypes.c_void_p)]),
    "qsk_ti_create_grid": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _u32p, ctypes.c_int, _i32p, _f32p,
                                          ctypes.POINTER(ctypes.c_void_p)]),
    "qsk_ti_fft_size": (ctypes.c_int, [ctypes.c_void_p, _u32p]),
    "qsk_ti_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "qsk_worker_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    "qsk_worker_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "qsk_pattern_kbest": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _i32p, ctypes.c_int,
                                         ctypes.POINTER(QskTerm), ctypes.c_uint, ctypes.c_float, _f32p, _u32p, _i32p]),
    "qsk_pattern_kbest_ex": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _i32p, ctypes.c_int,
                                            ctypes.POINTER(QskTerm), ctypes.c_uint, ctypes.c_float,
                                            ctypes.POINTER(QskPatternOpts), _f32p, _u32p, _i32p]),
    "qsk_pattern_kbest_batch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _i32p, _i32p, _i32p,
                                               ctypes.POINTER(QskTerm), ctypes.c_uint, _f32p, _f32p, _u32p, _i32p]),
    "qsk_pattern_kbest_batch_verbatim": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _i32p, _i32p, _i32p,
                                                        ctypes.POINTER(QskTerm), ctypes.c_uint, _f32p, _u32p, _f32p,
                                                        _f32p, _u32p, _i32p]),
    "qsk_calibrate": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(QskCalibParams), _f32p, _f32p, _u32p,
                                     ctypes.POINTER(ctypes.c_longlong)]),
    "qsk_pattern_kbest_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, _i32p, ctypes.c_int,
                                                 ctypes.POINTER(QskTerm), ctypes.c_uint, ctypes.c_float, _f32p, _u32p,
                                                 _i32p]),
    "qsk_tc_topk": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_longlong, ctypes.c_int,
                                   ctypes.c_void_p, ctypes.c_void_p, _f32p, _f32p, _f32p, _u32p, _i32p, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_ulonglong), _u32p]),
    "qsk_measure_peaks": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    "qsk_encoder_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_uint, ctypes.POINTER(ctypes.c_void_p)]),
    "qsk_encoder_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "qsk_encoder_param_count": (ctypes.c_longlong, [ctypes.c_void_p]),
    "qsk_encoder_input_dim": (ctypes.c_int, [ctypes.c_void_p]),
    "qsk_encoder_set_scales": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_float]),
    "qsk_encoder_set_tensor_cores": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "qsk_gemm_bf16": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f32p, _f32p, _f32p,
                                     _f32p]),
    "qsk_encoder_get_pairs": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_longlong, _f32p, _f32p]),
    "qsk_encoder_get_weights": (ctypes.c_int, [ctypes.c_void_p, _f32p]),
    "qsk_encoder_set_weights": (ctypes.c_int, [ctypes.c_void_p, _f32p]),
    "qsk_encoder_loss_grad": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _f32p, _f32p, ctypes.c_float, _f32p, _f32p]),
    "qsk_encoder_embed": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, _f32p, _f32p]),
    "qsk_encoder_add_pairs": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, _f32p, _i32p, ctypes.c_int,
                                             ctypes.POINTER(ctypes.c_longlong)]),
    "qsk_encoder_add_pairs_host": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, _f32p, _f32p]),
    "qsk_encoder_pairs": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)]),
    "qsk_encoder_clear_pairs": (ctypes.c_int, [ctypes.c_void_p]),
    "qsk_encoder_train": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                         ctypes.c_uint, _f32p]),
    "qsk_sim_set_learned": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(QskLearnedOpts)]),
    "qsk_index_to_position": (ctypes.c_uint, [ctypes.c_void_p, _i32p, ctypes.c_uint]),
    "qsk_position_to_index": (ctypes.c_uint, [ctypes.c_void_p, _i32p, ctypes.c_uint]),
    "qsk_sim_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(QskParams), _f32p,
                                      ctypes.POINTER(ctypes.c_void_p)]),
    "qsk_sim_run": (ctypes.c_int, [ctypes.c_void_p]),
    "qsk_sim_run_teacher": (ctypes.c_int, [ctypes.c_void_p, _f32p, _u32p]),
    "qsk_sim_run_teacher_nodes": (ctypes.c_int, [ctypes.c_void_p, _f32p, _i32p, ctypes.c_int]),
    "qsk_sim_read": (ctypes.c_int, [ctypes.c_void_p, _f32p, _u32p, _u32p]),
    "qsk_sim_get_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(QskSimInfo)]),
    "qsk_sim_get_path": (ctypes.c_int, [ctypes.c_void_p, _u32p, _f32p, _u32p]),
    "qsk_sim_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "qsk_sim_set_profiling": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "qsk_sim_set_level_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint, ctypes.c_longlong]),
    "qsk_sim_set_graph": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "qsk_jobs_run": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_int, _i32p]),
    "qsk_blocks_set_limit": (ctypes.c_int, [ctypes.c_ulonglong]),
    "qsk_blocks_release": (ctypes.c_int, []),
    "qsk_blocks_info": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_ulonglong),
                                       ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong),
                                       ctypes.POINTER(ctypes.c_longlong)]),
    "qsk_sim_set_tensor": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(QskTensorOpts)]),
    "qsk_simulate": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(QskParams), _f32p, _u32p]),
    "qsk_qs_template": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _u32p, _f32p, _i32p, _f32p, ctypes.c_int]),
    "qsk_set_map_mode": (ctypes.c_int, [ctypes.c_int]),
    "qsk_qs_path": (ctypes.c_longlong, [ctypes.c_longlong, ctypes.c_int, _f32p, ctypes.c_uint, _u32p, _f32p]),
    "qsk_bgrid_read": (ctypes.c_int, [ctypes.c_char_p, _i32p, _u32p, _i32p, _i32p, ctypes.c_int, _i32p,
                                      ctypes.c_void_p, ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong)]),
    "qsk_bgrid_write": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, _u32p, ctypes.c_int, _i32p, ctypes.c_int,
                                       ctypes.c_void_p, ctypes.c_int]),
}


def lib():
    """Load libg2s_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m g2s_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(rc: int, what: str):
    if rc != 0:
        msg = lib().qsk_last_error()
        raise RuntimeError(f"{what} failed (status {rc}): {msg.decode() if msg else ''}")


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


def device_count() -> int:
    c = ctypes.c_int(0)
    rc = lib().qsk_device_count(ctypes.byref(c))
    return c.value if rc == 0 else 0


def set_map_mode(mode: int) -> None:
    """0: automatic (bit-sliced kernel for unit-weight categorical patterns),
    1: always the FP32 gather kernel.  Identical results either way."""
    _check(lib().qsk_set_map_mode(int(mode)), "qsk_set_map_mode")


def search_template(kernel_dims, nvar: int = 1, kernel: Optional[np.ndarray] = None):
    """Host-only: sorted neighbour search template and kernel weights."""
    kd = np.asarray(kernel_dims, dtype=np.uint32)
    cap = int(np.prod(kd))
    offs = np.zeros(cap * len(kd), np.int32)
    w = np.zeros(cap * nvar, np.float32)
    kern = None if kernel is None else np.ascontiguousarray(kernel, dtype=np.float32)
    n = lib().qsk_qs_template(len(kd), nvar, _p(kd, _u32p), _p(kern, _f32p), _p(offs, _i32p), _p(w, _f32p), cap)
    if n < 0:
        raise RuntimeError("qsk_qs_template failed")
    return offs[: n * len(kd)].reshape(n, len(kd)), w[: n * nvar].reshape(n, nvar)


def random_path(di: np.ndarray, nvar: int, seed: int):
    """Host-only: (order, seeds, begin) of the simulation path for grid di."""
    d = np.ascontiguousarray(di, dtype=np.float32)
    cells = d.size // nvar
    order = np.zeros(cells, np.uint32)
    seeds = np.zeros(cells, np.float32)
    b = lib().qsk_qs_path(cells, nvar, _p(d, _f32p), int(seed) & 0xffffffff, _p(order, _u32p), _p(seeds, _f32p))
    if b < 0:
        raise RuntimeError("qsk_qs_path failed")
    return order, seeds, int(b)


def _grid_dims(arr: np.ndarray, nvar: int) -> np.ndarray:
    spatial = arr.shape if nvar == 1 else arr.shape[:-1]
    return np.array(list(reversed(spatial)), dtype=np.uint32)


class TrainingImage:
    """A training image resident on one GPU (layers built on the device)."""

    def __init__(self, ti: np.ndarray, types: Sequence[int], device: int = 0):
        self.nvar = len(types)
        self.dims = _grid_dims(ti, self.nvar)
        self.data = np.ascontiguousarray(ti, dtype=np.float32)
        self.types = np.asarray(types, dtype=np.int32)
        h = ctypes.c_void_p()
        _check(lib().qsk_ti_create_grid(device, len(self.dims), _p(self.dims, _u32p), self.nvar,
                                        _p(self.types, _i32p), _p(self.data, _f32p), ctypes.byref(h)),
               "qsk_ti_create_grid")
        self.handle = h
        self.ndim = len(self.dims)

    @classmethod
    def from_layers(cls, layers: Sequence[np.ndarray], src_size, fft_size, device: int = 0):
        """Reference-format layers (flipped, prod(fft_size) floats each)."""
        self = cls.__new__(cls)
        self.nvar = 0
        self.dims = np.asarray(src_size, dtype=np.uint32)
        fft = np.asarray(fft_size, dtype=np.uint32)
        arrs = [np.ascontiguousarray(l, dtype=np.float32).ravel() for l in layers]
        ptrs = (_f32p * len(arrs))(*[a.ctypes.data_as(_f32p) for a in arrs])
        h = ctypes.c_void_p()
        _check(lib().qsk_ti_create_layers(device, len(self.dims), _p(self.dims, _u32p), _p(fft, _u32p), len(arrs),
                                          ptrs, ctypes.byref(h)), "qsk_ti_create_layers")
        self._keep = arrs
        self.handle = h
        self.ndim = len(self.dims)
        return self

    def fft_size(self) -> np.ndarray:
        out = np.zeros(self.ndim, np.uint32)
        _check(lib().qsk_ti_fft_size(self.handle, _p(out, _u32p)), "qsk_ti_fft_size")
        return out

    def index_to_position(self, mn, index: int) -> int:
        m = np.asarray(mn, dtype=np.int32)
        return int(lib().qsk_index_to_position(self.handle, _p(m, _i32p), int(index)))

    def position_to_index(self, mn, position: int) -> int:
        m = np.asarray(mn, dtype=np.int32)
        return int(lib().qsk_position_to_index(self.handle, _p(m, _i32p), int(position)))

    def close(self):
        if getattr(self, "handle", None):
            lib().qsk_ti_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Worker:
    """Per-thread pattern queries against one TrainingImage."""

    def __init__(self, ti: TrainingImage):
        self.ti = ti
        h = ctypes.c_void_p()
        _check(lib().qsk_worker_create(ti.handle, ctypes.byref(h)), "qsk_worker_create")
        self.handle = h

    def pattern_kbest(self, offsets: np.ndarray, terms, k: int, seed: float, exclude_index: int = -1,
                      missing_data: bool = False, centre_mask_layer: int = -1, exclude_radius: float = 0.0):
        """offsets: (n, ndim) int; terms: list of (neighbour, layer, op, a, b).
        ``exclude_index`` (scan index) is forced to -inf, with
        ``exclude_radius`` >= 1 every index the reference's radius exclusion
        marks around it.  Returns (scores[k], scan_indices[k], min_offset[ndim])."""
        offs = np.ascontiguousarray(offsets, dtype=np.int32).reshape(-1, self.ti.ndim)
        tarr = (QskTerm * max(len(terms), 1))(*[QskTerm(int(t[0]), int(t[1]), int(t[2]), float(t[3]), float(t[4]))
                                               for t in terms])
        sc = np.zeros(k, np.float32)
        ix = np.zeros(k, np.uint32)
        mn = np.zeros(self.ti.ndim, np.int32)
        if exclude_index < 0 and not missing_data:
            _check(lib().qsk_pattern_kbest(self.handle, offs.shape[0], _p(offs, _i32p), len(terms), tarr, k, seed,
                                           _p(sc, _f32p), _p(ix, _u32p), _p(mn, _i32p)), "qsk_pattern_kbest")
        else:
            opts = QskPatternOpts(int(exclude_index), int(missing_data), int(centre_mask_layer), float(exclude_radius))
            _check(lib().qsk_pattern_kbest_ex(self.handle, offs.shape[0], _p(offs, _i32p), len(terms), tarr, k, seed,
                                              ctypes.byref(opts), _p(sc, _f32p), _p(ix, _u32p), _p(mn, _i32p)),
                   "qsk_pattern_kbest_ex")
        return sc, ix, mn

    def pattern_kbest_verbatim(self, patterns, k: int, seeds, origins, radii=None):
        """Batched queries with the verbatim exclusion of distribution():
        patterns is a list of (offsets (n, ndim), terms); origins the TI cell
        each pattern came from (0xffffffff: none); radii the exclusion radius
        (< 1: the cell's index only).  Returns (scores[B,k], scan_indices[B,k],
        min_offsets[B,ndim])."""
        nd = self.ti.ndim
        B = len(patterns)
        nb_ptr = np.zeros(B + 1, np.int32)
        term_ptr = np.zeros(B + 1, np.int32)
        offs, tl = [], []
        for b, (o, terms) in enumerate(patterns):
            o = np.asarray(o, np.int32).reshape(-1, nd)
            offs.append(o)
            nb_ptr[b + 1] = nb_ptr[b] + o.shape[0]
            tl.extend(terms)
            term_ptr[b + 1] = term_ptr[b] + len(terms)
        offs = np.ascontiguousarray(np.concatenate(offs) if offs else np.zeros((0, nd), np.int32), np.int32)
        tarr = (QskTerm * max(len(tl), 1))(*[QskTerm(int(t[0]), int(t[1]), int(t[2]), float(t[3]), float(t[4]))
                                            for t in tl])
        sd = np.ascontiguousarray(seeds, np.float32)
        org = np.ascontiguousarray(origins, np.uint32)
        rad = None if radii is None else np.ascontiguousarray(radii, np.float32)
        sc = np.zeros((B, k), np.float32)
        ix = np.zeros((B, k), np.uint32)
        mn = np.zeros((B, nd), np.int32)
        _check(lib().qsk_pattern_kbest_batch_verbatim(self.handle, B, _p(nb_ptr, _i32p), _p(offs, _i32p),
                                                      _p(term_ptr, _i32p), tarr, k, _p(sd, _f32p), _p(org, _u32p),
                                                      _p(rad, _f32p), _p(sc, _f32p), _p(ix, _u32p), _p(mn, _i32p)),
               "qsk_pattern_kbest_batch_verbatim")
        return sc, ix, mn

    def close(self):
        if getattr(self, "handle", None):
            lib().qsk_worker_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Simulation:
    """A QS vector simulation resident on one GPU."""

    def __init__(self, ti: np.ndarray, di: np.ndarray, types: Sequence[int], n: int, k: float, seed: int,
                 kernel: Optional[np.ndarray] = None, device: int = 0, no_verbatim: bool = False,
                 n_per_var: Optional[Sequence[int]] = None, ni: Optional[np.ndarray] = None,
                 kvi: Optional[np.ndarray] = None, kernels: Optional[Sequence[np.ndarray]] = None,
                 kii: Optional[np.ndarray] = None, full: bool = False,
                 extra_tis: Optional[Sequence[np.ndarray]] = None, ii: Optional[np.ndarray] = None):
        """Local controls as in G2S: ``n_per_var`` (-n n1 n2 ...), ``ni``
        (-ni image, grid shape [+ counts]), ``kvi`` (-kvi image), ``kernels``
        (the -ki list) with ``kii`` (-kii image of kernel indices); ``full``
        is -fs (one path node per cell value; the index image then has one
        entry per value).  ``extra_tis``: further training images (-ti a b
        ...; the index image holds TI cell * nTI + TI) with ``ii`` (-ii, the
        TI each grid cell samples from)."""
        self.nvar = len(types)
        self._ti = np.ascontiguousarray(ti, dtype=np.float32)
        self._di = np.ascontiguousarray(di, dtype=np.float32)
        self._types = np.asarray(types, dtype=np.int32)
        self._tdims = _grid_dims(self._ti, self.nvar)
        self._ddims = _grid_dims(self._di, self.nvar)
        self._kdims = None if kernel is None else _grid_dims(np.asarray(kernel), self.nvar)
        self._kern = None if kernel is None else np.ascontiguousarray(kernel, dtype=np.float32)
        self.params = QskParams(len(self._tdims), _p(self._tdims, _u32p), self.nvar, _p(self._types, _i32p),
                                _p(self._ti, _f32p), _p(self._ddims, _u32p), _p(self._kdims, _u32p),
                                _p(self._kern, _f32p), int(n), float(k), int(seed) & 0xffffffff, int(no_verbatim))
        cells = int(np.prod(self._ddims))
        self._keep = []
        self.full = bool(full)
        self.params.full_simulation = int(full)

        def keep(a, dt):
            x = np.ascontiguousarray(a, dtype=dt).ravel()
            self._keep.append(x)
            return x

        if n_per_var is not None:
            a = keep(n_per_var, np.int32)
            self.params.n_counts = a.size
            self.params.n_per_variable = _p(a, _i32p)
        if ni is not None:
            a = keep(ni, np.float32)
            self.params.n_image_vars = max(1, a.size // cells)
            self.params.n_image = _p(a, _f32p)
        if kvi is not None:
            self.params.k_image = _p(keep(kvi, np.float32), _f32p)
        if kernels is not None:
            arrs = [keep(kq, np.float32) for kq in kernels]
            dims = keep(np.concatenate([_grid_dims(np.asarray(kq), self.nvar) for kq in kernels]), np.uint32)
            ptrs = (_f32p * len(arrs))(*[_p(a, _f32p) for a in arrs])
            self._keep.append(ptrs)
            self.params.n_kernels = len(arrs)
            self.params.kernels_dims = _p(dims, _u32p)
            self.params.kernels = ptrs
        if kii is not None:
            self.params.kernel_index_image = _p(keep(kii, np.float32), _f32p)
        self.nti = 1
        if extra_tis:
            arrs = [keep(t, np.float32) for t in extra_tis]
            dims = keep(np.concatenate([_grid_dims(np.asarray(t), self.nvar) for t in extra_tis]), np.uint32)
            ptrs = (_f32p * len(arrs))(*[_p(a, _f32p) for a in arrs])
            self._keep.append(ptrs)
            self.params.n_extra_tis = len(arrs)
            self.params.extra_ti_dims = _p(dims, _u32p)
            self.params.extra_tis = ptrs
            self.nti = 1 + len(arrs)
        if ii is not None:
            self.params.ti_index_image = _p(keep(ii, np.float32), _f32p)
        h = ctypes.c_void_p()
        _check(lib().qsk_sim_create(device, ctypes.byref(self.params), _p(self._di, _f32p), ctypes.byref(h)),
               "qsk_sim_create")
        self.handle = h
        self.shape = self._di.shape

    def run(self):
        _check(lib().qsk_sim_run(self.handle), "qsk_sim_run")
        return self

    def set_profiling(self, on: bool = True):
        _check(lib().qsk_sim_set_profiling(self.handle, int(on)), "qsk_sim_set_profiling")
        return self

    def set_tensor(self, mode: str = "bf16", prefix: int = 0, width: int = 0, shortlist: int = 0,
                   audit: float = 0.0, batch: int = 0):
        """Tensor-core form of the map: mode "plain" (the exact reference path),
        "bf16" or "fp8"; zero fields take the automatic choice."""
        m = {"plain": 0, "bf16": 1, "fp8": 2}[mode]
        o = QskTensorOpts(m, int(prefix), int(width), int(shortlist), float(audit), int(batch))
        _check(lib().qsk_sim_set_tensor(self.handle, ctypes.byref(o)), "qsk_sim_set_tensor")
        return self

    def set_learned(self, encoder: Optional["Encoder"], width: int = 0, shortlist: int = 0, conf_rank: int = 0,
                    audit: float = 0.0, conf_z: float = 2.0, conf_r2: float = 0.2):
        """The learned proposal as the map (qsk_sim_set_learned); None: off.
        conf_z > 0: the statistical confidence check, else the rank check."""
        o = QskLearnedOpts(int(width), int(shortlist), int(conf_rank), float(audit), float(conf_z), float(conf_r2))
        _check(lib().qsk_sim_set_learned(self.handle, encoder.handle if encoder else None, ctypes.byref(o)),
               "qsk_sim_set_learned")
        self._encoder = encoder
        return self

    def set_level_wait(self, spin_limit: int = 0, hold_node: int = -1):
        """Bound of the dependency-level waits (polls; 0 = default) and, for
        failure-path tests, a path node whose level is never published."""
        _check(lib().qsk_sim_set_level_wait(self.handle, int(spin_limit), int(hold_node)), "qsk_sim_set_level_wait")
        return self

    def set_graph(self, on: bool = True):
        """Graph mode of the plain path (qsk_sim_set_graph)."""
        _check(lib().qsk_sim_set_graph(self.handle, int(bool(on))), "qsk_sim_set_graph")
        return self

    def run_teacher(self, completed: np.ndarray, index: Optional[np.ndarray] = None):
        c = np.ascontiguousarray(completed, dtype=np.float32)
        ix = None if index is None else np.ascontiguousarray(index, dtype=np.uint32).ravel()
        _check(lib().qsk_sim_run_teacher(self.handle, _p(c, _f32p), _p(ix, _u32p)), "qsk_sim_run_teacher")
        return self

    def run_teacher_nodes(self, completed: np.ndarray, path_nodes):
        """Teacher-forced draw of a sample of path nodes (no write-back)."""
        c = np.ascontiguousarray(completed, dtype=np.float32)
        nodes = np.ascontiguousarray(path_nodes, dtype=np.int32)
        _check(lib().qsk_sim_run_teacher_nodes(self.handle, _p(c, _f32p), _p(nodes, _i32p), int(nodes.size)),
               "qsk_sim_run_teacher_nodes")
        return self

    def info(self) -> dict:
        inf = QskSimInfo()
        _check(lib().qsk_sim_get_info(self.handle, ctypes.byref(inf)), "qsk_sim_get_info")
        return {f: getattr(inf, f) for f, _ in QskSimInfo._fields_}

    def path(self):
        cells = int(np.prod(self._ddims))
        order = np.zeros(cells, np.uint32)
        seeds = np.zeros(cells, np.float32)
        begin = ctypes.c_uint(0)
        _check(lib().qsk_sim_get_path(self.handle, _p(order, _u32p), _p(seeds, _f32p), ctypes.byref(begin)),
               "qsk_sim_get_path")
        return order, seeds, begin.value

    def read(self):
        """Returns (grid, index_image, node_cells)."""
        cells = int(np.prod(self._ddims))
        out = np.empty_like(self._di)
        idx = np.zeros(cells * (self.nvar if self.full else 1), np.uint32)
        nodes = self.info()["path_nodes"]
        nc = np.zeros(max(nodes, 1), np.uint32)
        _check(lib().qsk_sim_read(self.handle, _p(out, _f32p), _p(idx, _u32p), _p(nc, _u32p)), "qsk_sim_read")
        shape = self._di.shape if self.full else self._di.shape[:len(self._ddims)]
        return out, idx.reshape(shape), nc[:nodes]

    def close(self):
        if getattr(self, "handle", None):
            lib().qsk_sim_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Encoder:
    """The learned proposal's neighbourhood encoder (qsk_encoder_*)."""

    def __init__(self, nvar: int, seed: int = 0, device: int = 0):
        h = ctypes.c_void_p()
        _check(lib().qsk_encoder_create(device, int(nvar), int(seed) & 0xffffffff, ctypes.byref(h)),
               "qsk_encoder_create")
        self.handle = h
        self.nvar = nvar
        self.input_dim = lib().qsk_encoder_input_dim(h)
        self.param_count = lib().qsk_encoder_param_count(h)

    def set_tensor_cores(self, on: bool = True):
        """Encoder products on the tensor cores (BF16, default) or in FP32
        on the CUDA cores (qsk_encoder_set_tensor_cores)."""
        _check(lib().qsk_encoder_set_tensor_cores(self.handle, int(bool(on))), "qsk_encoder_set_tensor_cores")
        return self

    def set_scales(self, nscales: int = 4, cov_min: float = 0.9):
        """Stencil scales of the inputs (qsk_encoder_set_scales)."""
        _check(lib().qsk_encoder_set_scales(self.handle, int(nscales), float(cov_min)), "qsk_encoder_set_scales")
        return self

    def weights(self) -> np.ndarray:
        w = np.zeros(self.param_count, np.float32)
        _check(lib().qsk_encoder_get_weights(self.handle, _p(w, _f32p)), "qsk_encoder_get_weights")
        return w

    def set_weights(self, w: np.ndarray):
        a = np.ascontiguousarray(w, dtype=np.float32)
        assert a.size == self.param_count
        _check(lib().qsk_encoder_set_weights(self.handle, _p(a, _f32p)), "qsk_encoder_set_weights")

    def loss_grad(self, xq: np.ndarray, xp: np.ndarray, tau: float = 0.05, grad: bool = True):
        q = np.ascontiguousarray(xq, dtype=np.float32)
        p = np.ascontiguousarray(xp, dtype=np.float32)
        B = q.shape[0]
        loss = np.zeros(1, np.float32)
        g = np.zeros(self.param_count, np.float32) if grad else None
        _check(lib().qsk_encoder_loss_grad(self.handle, B, _p(q, _f32p), _p(p, _f32p), float(tau), _p(loss, _f32p),
                                           _p(g, _f32p)), "qsk_encoder_loss_grad")
        return float(loss[0]), g

    def embed(self, x: np.ndarray, head: str = "query") -> np.ndarray:
        """Embeddings by the query head ("query") or the TI-pattern head ("pattern")."""
        a = np.ascontiguousarray(x, dtype=np.float32)
        out = np.zeros((a.shape[0], 64), np.float32)
        _check(lib().qsk_encoder_embed(self.handle, {"query": 0, "pattern": 1}[head], a.shape[0], _p(a, _f32p),
                                       _p(out, _f32p)), "qsk_encoder_embed")
        return out

    def add_pairs(self, sim: "Simulation", completed: np.ndarray, path_nodes) -> int:
        c = np.ascontiguousarray(completed, dtype=np.float32)
        nodes = np.ascontiguousarray(path_nodes, dtype=np.int32)
        added = ctypes.c_longlong(0)
        _check(lib().qsk_encoder_add_pairs(self.handle, sim.handle, _p(c, _f32p), _p(nodes, _i32p), int(nodes.size),
                                           ctypes.byref(added)), "qsk_encoder_add_pairs")
        return added.value

    def add_pairs_host(self, xq: np.ndarray, xp: np.ndarray) -> int:
        q = np.ascontiguousarray(xq, dtype=np.float32)
        p = np.ascontiguousarray(xp, dtype=np.float32)
        assert q.shape == p.shape and q.shape[1] == self.input_dim
        _check(lib().qsk_encoder_add_pairs_host(self.handle, q.shape[0], _p(q, _f32p), _p(p, _f32p)),
               "qsk_encoder_add_pairs_host")
        return q.shape[0]

    def pairs(self) -> int:
        n = ctypes.c_longlong(0)
        _check(lib().qsk_encoder_pairs(self.handle, ctypes.byref(n)), "qsk_encoder_pairs")
        return n.value

    def get_pairs(self, first: int = 0, n: Optional[int] = None):
        """Stored (query, positive) input rows [first, first + n) as two arrays."""
        n = self.pairs() - first if n is None else n
        q = np.zeros((n, self.input_dim), np.float32)
        p = np.zeros((n, self.input_dim), np.float32)
        _check(lib().qsk_encoder_get_pairs(self.handle, int(first), int(n), _p(q, _f32p), _p(p, _f32p)),
               "qsk_encoder_get_pairs")
        return q, p

    def clear_pairs(self):
        _check(lib().qsk_encoder_clear_pairs(self.handle), "qsk_encoder_clear_pairs")

    def train(self, epochs: int = 1, batch: int = 1024, lr: float = 1e-3, tau: float = 0.05, seed: int = 0) -> float:
        loss = np.zeros(1, np.float32)
        _check(lib().qsk_encoder_train(self.handle, int(epochs), int(batch), float(lr), float(tau),
                                       int(seed) & 0xffffffff, _p(loss, _f32p)), "qsk_encoder_train")
        return float(loss[0])

    def close(self):
        if getattr(self, "handle", None):
            lib().qsk_encoder_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gemm_bf16(a: np.ndarray, b: np.ndarray, bias: Optional[np.ndarray] = None, device: int = 0) -> np.ndarray:
    """C = bf16(a) @ bf16(b).T (+ bias) on the tensor cores (qsk_gemm_bf16)."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(b, dtype=np.float32)
    M, K = a.shape
    N, K2 = b.shape
    assert K == K2
    bi = None if bias is None else np.ascontiguousarray(bias, dtype=np.float32)
    c = np.zeros((M, N), np.float32)
    _check(lib().qsk_gemm_bf16(device, M, N, K, _p(a, _f32p), _p(b, _f32p), _p(bi, _f32p), _p(c, _f32p)),
           "qsk_gemm_bf16")
    return c


def run_jobs(sims: Sequence["Simulation"], threads: int = 0) -> np.ndarray:
    """Run several distinct simulations in one call (qsk_jobs_run); returns
    each job's status (all 0 on success; the first error raises)."""
    n = len(sims)
    if len({id(s) for s in sims}) != n:
        raise ValueError("run_jobs: every simulation must be distinct")
    arr = (ctypes.c_void_p * max(n, 1))(*[s.handle for s in sims])
    status = np.zeros(max(n, 1), np.int32)
    _check(lib().qsk_jobs_run(arr, n, int(threads), _p(status, _i32p)), "qsk_jobs_run")
    return status[:n]


def blocks_info(device: int = 0) -> dict:
    """Device blocks kept from ended simulations (qsk_blocks_info): bytes and
    blocks kept on ``device``, allocations served from them (hits) or not."""
    by, nb, h, m = ctypes.c_ulonglong(), ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
    _check(lib().qsk_blocks_info(int(device), ctypes.byref(by), ctypes.byref(nb), ctypes.byref(h), ctypes.byref(m)),
           "qsk_blocks_info")
    return {"bytes": by.value, "blocks": nb.value, "hits": h.value, "misses": m.value}


def blocks_release() -> None:
    """Free every kept device block (qsk_blocks_release)."""
    _check(lib().qsk_blocks_release(), "qsk_blocks_release")


def blocks_set_limit(nbytes: int) -> None:
    """Bytes kept per device from ended simulations (0: keep none)."""
    _check(lib().qsk_blocks_set_limit(int(nbytes)), "qsk_blocks_set_limit")


def measure_peaks(device: int = 0) -> dict:
    """The library's own peak microbenchmarks (qsk_measure_peaks)."""
    out = (ctypes.c_double * 4)()
    _check(lib().qsk_measure_peaks(device, out), "qsk_measure_peaks")
    return {"fp32_tflops": out[0], "int32_lop3_tops": out[1], "bf16_tflops": out[2], "fp8_tflops": out[3]}


def tc_topk(queries: np.ndarray, rows: np.ndarray, fmt: int, X: int, Y: int, box: np.ndarray, W: int = 8,
            ranges: int = 1, q_scale=None, q_bias=None, p_scale=None, q_seed=None, device: int = 0):
    """Top-W inner products on the tensor cores (qsk_tc_topk).  ``queries``
    (B x K) and ``rows`` (N x K) hold bit patterns: uint16 BF16 (fmt 0) or
    uint8 FP8 E4M3 (fmt 1).  Returns (keys, positions), each [B, ranges, W]."""
    q = np.ascontiguousarray(queries)
    r = np.ascontiguousarray(rows)
    want = np.uint16 if fmt == 0 else np.uint8
    if q.dtype != want or r.dtype != want or q.ndim != 2 or r.ndim != 2 or q.shape[1] != r.shape[1]:
        raise ValueError("queries/rows: 2-D bit-pattern arrays of one K (uint16 BF16 or uint8 FP8)")
    B, K = q.shape
    N = r.shape[0]
    bx = np.ascontiguousarray(box, dtype=np.int32).reshape(B, 6)
    f = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float32)
    qs_, qb_, ps_ = f(q_scale), f(q_bias), f(p_scale)
    sd = None if q_seed is None else np.ascontiguousarray(q_seed, dtype=np.uint32)
    keys = np.zeros((B, ranges, W), np.uint64)
    pos = np.zeros((B, ranges, W), np.uint32)
    _check(lib().qsk_tc_topk(device, fmt, B, N, K, q.ctypes.data, r.ctypes.data, _p(qs_, _f32p), _p(qb_, _f32p),
                             _p(ps_, _f32p), _p(sd, _u32p), _p(bx, _i32p), X, Y, W, ranges,
                             keys.ctypes.data_as(ctypes.POINTER(ctypes.c_ulonglong)), _p(pos, _u32p)), "qsk_tc_topk")
    return keys, pos


def qs(ti, di: np.ndarray, dt: Sequence[int], k: float, n, s: int,
       ki=None, nV: bool = False, ni: Optional[np.ndarray] = None, kvi: Optional[np.ndarray] = None,
       kii: Optional[np.ndarray] = None, fs: bool = False, device: int = 0, tensor=None,
       audit: float = 0.01, ii: Optional[np.ndarray] = None):
    """QuickSampling on one GPU; arguments named after the G2S flags
    (-ti -di -dt -k -n -s -ki -nV -ni -kvi -kii -fs -ii).  ``ti`` is one
    training image or a list of them (-ti a b ...; the index image then holds
    TI cell * number of TIs + TI, and ``ii`` may name each cell's TI).  ``n``
    is one count or one per variable; ``ki`` one kernel or a list of kernels
    (selected per cell by ``kii``).  ``tensor`` selects the tensor-core form of
    the map ("bf16" or "fp8", or a dict {"mode", "prefix", "width",
    "shortlist", "batch"} such as the autotuner's choice), with the regret
    audit fraction ``audit``; None is the exact reference path.  Returns
    (simulation, index) as G2S does."""
    extra = None
    if isinstance(ti, (list, tuple)):
        if not ti:
            raise ValueError("qs: no training image")
        ti, extra = ti[0], list(ti[1:]) or None
    n_list = None
    if np.ndim(n) > 0:
        n_list = [int(x) for x in np.ravel(n)]
        n = max(n_list)
    kernel, kernels = ki, None
    if isinstance(ki, (list, tuple)):
        kernel, kernels = None, list(ki)
    sim = Simulation(ti, di, dt, n=n if n is not None else 0, k=k, seed=s, kernel=kernel, device=device,
                     no_verbatim=nV, n_per_var=n_list, ni=ni, kvi=kvi, kernels=kernels, kii=kii, full=fs,
                     extra_tis=extra, ii=ii)
    try:
        if isinstance(tensor, dict):
            sim.set_tensor(tensor["mode"], prefix=int(tensor.get("prefix", 0)), width=int(tensor.get("width", 0)),
                           shortlist=int(tensor.get("shortlist", 0)), batch=int(tensor.get("batch", 0)), audit=audit)
        elif tensor:
            sim.set_tensor(tensor, audit=audit)
        sim.run()
        out, idx, _ = sim.read()
    finally:
        sim.close()
    return out, idx


def default_neighbour_counts(max_n) -> np.ndarray:
    """auto_qs' configurations without -nl: for i in 1..max_n[0]-1 the counts
    i * max_n[j] / max_n[0] in unsigned integer arithmetic (the round() there
    applies to an integer quotient; G2S src/auto_qs.cpp:650-661)."""
    mx = [int(m) for m in np.atleast_1d(max_n)]
    rows = [[(i * mx[j]) // mx[0] for j in range(len(mx))] for i in range(1, mx[0])]
    return np.array(rows, np.uint32).reshape(-1, len(mx))


def calibrate(ti: np.ndarray, types: Sequence[int], kernels, counts=None, densities=None, max_k: int = 1,
              power: float = 2.0, noise: float = 0.0, max_iterations: int = 25000, min_iterations: int = 1000,
              max_seconds: float = float("inf"), seed: int = 0, device: int = 0, max_n=80):
    """auto_qs calibration (G2S src/auto_qs.cpp) on the GPU.  kernels: list of
    weight kernels (numpy spatial shape [+ (nvar,)]); counts: (n_configs,
    n_counts) neighbours per variable (default: auto_qs' list for max_n);
    densities: default auto_qs' 7 values.  Returns (mean_error, deviation,
    sample_count, searches) with the arrays shaped (n_densities, n_kernels,
    n_configs, max_k)."""
    nvar = len(types)
    t = np.ascontiguousarray(ti, dtype=np.float32)
    tdims = _grid_dims(t, nvar)
    nd = len(tdims)
    if counts is None:
        counts = default_neighbour_counts(max_n)
    cnt = np.ascontiguousarray(np.atleast_2d(np.asarray(counts, np.uint32)))
    if densities is None:
        densities = [0.0078, 0.0156, 0.0312, 0.0625, 0.1250, 0.2500, 0.5000]
    den = np.ascontiguousarray(densities, np.float32)
    karr, kd, knv = [], [], []
    for k in kernels:
        kk = np.ascontiguousarray(k, dtype=np.float32)
        if kk.ndim == nd + 1:
            knv.append(kk.shape[-1])
            kd.extend(reversed(kk.shape[:-1]))
        else:
            knv.append(1)
            kd.extend(reversed(kk.shape))
        karr.append(kk)
    kd = np.ascontiguousarray(kd, np.uint32)
    knv = np.ascontiguousarray(knv, np.int32)
    kptrs = (_f32p * len(karr))(*[_p(k, _f32p) for k in karr])
    ty = np.ascontiguousarray(types, np.int32)
    p = QskCalibParams(nd, _p(tdims, _u32p), nvar, _p(ty, _i32p), _p(t, _f32p), len(karr), _p(kd, _u32p),
                       _p(knv, _i32p), kptrs, cnt.shape[0], cnt.shape[1], _p(cnt, _u32p), den.size, _p(den, _f32p),
                       int(max_k), float(power), float(noise), int(max_iterations), int(min_iterations),
                       float(max_seconds), int(seed))
    S = cnt.shape[0] * len(karr) * den.size
    mean = np.zeros(S * max_k, np.float32)
    dev = np.zeros(S * max_k, np.float32)
    ns = np.zeros(S * max_k, np.uint32)
    nsearch = ctypes.c_longlong(0)
    _check(lib().qsk_calibrate(device, ctypes.byref(p), _p(mean, _f32p), _p(dev, _f32p), _p(ns, _u32p),
                               ctypes.byref(nsearch)), "qsk_calibrate")
    shape = (den.size, len(karr), cnt.shape[0], max_k)
    return mean.reshape(shape), dev.reshape(shape), ns.reshape(shape), int(nsearch.value)


def read_bgrid(path: str):
    """Read a G2S .bgrid(.gz) grid: returns (array with numpy shape
    (..., ny, nx[, nvar]), types).  Unsigned-integer grids (index images)
    come back as uint32."""
    nd, nv, enc = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    dims = (ctypes.c_uint * 16)()
    types = (ctypes.c_int * 4096)()
    count = ctypes.c_longlong()
    _check(lib().qsk_bgrid_read(path.encode(), ctypes.byref(nd), dims, ctypes.byref(nv), types, 4096,
                                ctypes.byref(enc), None, 0, ctypes.byref(count)), "qsk_bgrid_read")
    dt = {0: np.float32, 1: np.int32, 2: np.uint32}[enc.value]
    out = np.empty(count.value, dt)
    _check(lib().qsk_bgrid_read(path.encode(), ctypes.byref(nd), dims, ctypes.byref(nv), types, 4096,
                                ctypes.byref(enc), out.ctypes.data, count.value, ctypes.byref(count)),
           "qsk_bgrid_read")
    shape = tuple(reversed([dims[i] for i in range(nd.value)])) + ((nv.value,) if nv.value > 1 else ())
    return out.reshape(shape), [types[i] for i in range(nv.value)]


def write_bgrid(path: str, arr: np.ndarray, types: Sequence[int], compress: bool = False) -> None:
    """Write a G2S .bgrid grid; ``arr`` has numpy shape (..., ny, nx[, nvar])
    with nvar = len(types) > 1; float32 (encoding 0) or uint32 (encoding 2)."""
    a = np.ascontiguousarray(arr)
    enc = 2 if a.dtype == np.uint32 else (1 if a.dtype == np.int32 else 0)
    if enc == 0:
        a = np.ascontiguousarray(a, dtype=np.float32)
    nvar = len(types)
    dims = _grid_dims(a, nvar)
    ty = np.asarray(types, np.int32)
    _check(lib().qsk_bgrid_write(path.encode(), len(dims), _p(dims, _u32p), nvar, _p(ty, _i32p), enc, a.ctypes.data,
                                 int(compress)), "qsk_bgrid_write")
