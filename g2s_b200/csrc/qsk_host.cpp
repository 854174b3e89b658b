// Host engine of the B200 QuickSampling path: the C ABI of include/g2s_b200.h.
//
// Host work mirrors what G2S does on the CPU before its simulation loop
// (search template, random path, per-node seeds: src/qs.cpp:975-1258,
// 1604-1641) with the same libstdc++ algorithms, so paths and seeds are
// identical for a given -s.  Everything per node runs on the GPU.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <numeric>
#include <chrono>
#include <random>
#include <thread>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/g2s_b200.h"
#include "qsk_internal.h"
#include "qsk_host_util.h"
#include "qsk_encoder.h"

using namespace qsk;

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

}  // namespace

namespace qsk {
int set_error(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

// Kept device blocks (DBuf::alloc / DBuf::release): per device, by size.
namespace {
struct KeptBlocks {
    std::mutex mu;
    std::map<int, std::multimap<size_t, void *>> free;   // device -> cap -> block
    std::map<int, size_t> bytes;
    unsigned long long limit = 8ull << 30;               // per device
    long long hits = 0, misses = 0;
};
KeptBlocks &kept() {
    static KeptBlocks *k = new KeptBlocks();   // never destroyed: no CUDA call at process exit
    return *k;
}
}  // namespace

thread_local bool g_keep_blocks = false;

void *block_take(size_t bytes, size_t *cap) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    KeptBlocks &k = kept();
    std::lock_guard<std::mutex> lock(k.mu);
    auto f = k.free.find(dev);
    if (f == k.free.end() || f->second.empty()) {
        ++k.misses;
        return nullptr;
    }
    auto it = f->second.lower_bound(bytes);
    if (it == f->second.end() || it->first > 2 * bytes + (2u << 20)) {
        ++k.misses;
        return nullptr;
    }
    void *p = it->second;
    *cap = it->first;
    k.bytes[dev] -= it->first;
    f->second.erase(it);
    ++k.hits;
    return p;
}

bool block_keep(void *p, size_t cap) {
    int dev = -1;
    if (!p || cap == 0 || cudaGetDevice(&dev) != cudaSuccess) return false;
    KeptBlocks &k = kept();
    std::lock_guard<std::mutex> lock(k.mu);
    if (k.bytes[dev] + cap > k.limit) return false;
    k.free[dev].emplace(cap, p);
    k.bytes[dev] += cap;
    return true;
}
}  // namespace qsk

int qsk_blocks_set_limit(unsigned long long bytes) {
    KeptBlocks &k = kept();
    std::lock_guard<std::mutex> lock(k.mu);
    k.limit = bytes;
    return QSK_OK;
}

int qsk_blocks_release(void) {
    KeptBlocks &k = kept();
    std::lock_guard<std::mutex> lock(k.mu);
    int rc = QSK_OK;
    for (auto &f : k.free) {
        DeviceGuard dg(f.first);
        for (auto &b : f.second)
            if (cudaFree(b.second) != cudaSuccess && rc == QSK_OK)
                rc = fail(QSK_ERR_CUDA, "cudaFree of a kept block on device %d", f.first);
        f.second.clear();
        k.bytes[f.first] = 0;
    }
    return rc;
}

int qsk_blocks_info(int device, unsigned long long *bytes, long long *blocks, long long *hits, long long *misses) {
    KeptBlocks &k = kept();
    std::lock_guard<std::mutex> lock(k.mu);
    auto f = k.free.find(device);
    if (bytes) *bytes = k.bytes.count(device) ? k.bytes[device] : 0;
    if (blocks) *blocks = f == k.free.end() ? 0 : (long long)f->second.size();
    if (hits) *hits = k.hits;
    if (misses) *misses = k.misses;
    return QSK_OK;
}

namespace {

#define CK(expr)                                                                                          \
    do {                                                                                                  \
        cudaError_t e_ = (expr);                                                                          \
        if (e_ != cudaSuccess) {                                                                          \
            int code_ = (e_ == cudaErrorMemoryAllocation) ? QSK_ERR_NOMEM : QSK_ERR_CUDA;                  \
            return fail(code_, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, __LINE__);         \
        }                                                                                                 \
    } while (0)


// smallest size >= s of the form 7-smooth times optionally one 11 or 13
// (G2S src/sharedMemoryManager.cpp:26-58)
unsigned fft_size_for(unsigned s) {
    if (s == 1) return 1;
    unsigned upper = 1u << (32 - __builtin_clz(s - 1));
    for (unsigned i = s; i <= upper; ++i) {
        unsigned v = i;
        for (unsigned p = 2; p < 8; ++p)
            while (v % p == 0) v /= p;
        if (v % 11 == 0) v /= 11;
        else if (v % 13 == 0) v /= 13;
        if (v == 1) return i;
    }
    return s;
}

Geom make_geom(int nd, const unsigned *src, const unsigned *fft) {
    Geom g;
    std::memset(&g, 0, sizeof(g));
    g.nd = nd;
    long long s = 1;
    for (int d = 0; d < QSK_MAXD; ++d) {
        if (d < nd) {
            g.fft[d] = int(fft[d]);
            g.src[d] = int(src[d]);
            g.sstride[d] = s;
            s *= fft[d];
        } else {
            g.fft[d] = 1;
            g.src[d] = 1;
            g.sstride[d] = s;
        }
    }
    g.N = s;
    g.nseg = int((s + QSK_SEG - 1) / QSK_SEG);
    return g;
}

}  // namespace

// ---------------------------------------------------------------------------
// TI context
// ---------------------------------------------------------------------------
struct qsk_ti {
    int device = 0;
    Geom g;
    int nlayers = 0;
    int nvar = 0;                 // grid-built contexts only
    std::vector<int> types;       // grid-built contexts only
    DBuf<float> layers;           // nlayers * N
    DBuf<float> grid;             // raw TI (grid-built): cells * nvar
    DBuf<int> dtypes;
    long long cells = 0;
    // missing values (grid-built): cells with any NaN variable are all-NaN, an
    // extra mask layer (index nvar) and complete-cell prefix counts
    bool missing = false;
    DBuf<int> complete_prefix;
    // bit planes of categorical variables (grid-built, every variable categorical
    // with at most QSK_CMAX categories)
    bool planes_ok = false;
    int pw = 0;
    DBuf<unsigned> planes;
    DBuf<int> ncat;
    DBuf<float> catv;
    // category codes of every categorical variable (grid-built; at most
    // QSK_CMAX each, cat_ok false beyond): the indicator layers of the
    // tensor-core pattern matrix
    bool cat_ok = true;
    std::vector<int> cat_n;           // nvar
    std::vector<float> cat_v;         // nvar x QSK_CMAX
};

namespace {
int g_map_mode = 0;   // 0: automatic, 1: always the FP32 gather kernel
}

struct qsk_worker {
    qsk_ti *ti = nullptr;
    cudaStream_t st = nullptr;
    DBuf<Slot> slots;
    DBuf<Term> terms;
    DBuf<float> rec_val;
    DBuf<int> rec_idx;
    DBuf<int> rec_cnt;
    DBuf<float> rec_max;
    DBuf<float> out_val;
    DBuf<unsigned> out_pos;
    DBuf<int> xcenter;        // verbatim exclusion with a radius: scan index per pattern
    DBuf<float> xradius;
    DBuf<unsigned> xmask;     // [pattern][ceil(N/32)] excluded positions
    std::vector<Slot> h_slots;
    std::vector<Term> h_terms;
};

namespace {

int smem_configured_device = -1;

cudaError_t ensure_records(const Geom &g, int nslots, DBuf<float> &rv, DBuf<int> &ri, DBuf<int> &rc,
                           DBuf<float> &rm) {
    size_t per = size_t(g.nseg) * QSK_SEG;
    cudaError_t e = rv.ensure(per * nslots);
    if (e != cudaSuccess) return e;
    e = ri.ensure(per * nslots);
    if (e != cudaSuccess) return e;
    e = rm.ensure(size_t(g.nseg) * nslots);
    if (e != cudaSuccess) return e;
    return rc.ensure(size_t(g.nseg) * nslots);
}

// host-side slot/terms for one explicit pattern
int build_pattern_slot(const qsk_ti *ti, int nnb, const int *offsets, int nterms, const qsk_term *terms, unsigned K,
                       float seed, int node, Slot &s, std::vector<Term> &out, int *out_min,
                       const qsk_pattern_opts *opts = nullptr) {
    const Geom &g = ti->g;
    const int nd = g.nd;
    std::memset(&s, 0, sizeof(s));
    s.node = node;
    s.seed = seed;
    s.sel = 0;
    s.excl = -1;
    s.K = int(K);
    int mn[QSK_MAXD] = {0}, mx[QSK_MAXD] = {0};
    for (int j = 0; j < nnb; ++j)
        for (int d = 0; d < nd; ++d) {
            mn[d] = std::min(mn[d], offsets[j * nd + d]);
            mx[d] = std::max(mx[d], offsets[j * nd + d]);
        }
    long long nvalid = 1;
    for (int d = 0; d < QSK_MAXD; ++d) {
        s.mn[d] = mn[d];
        int lo = 0;
        if (d < nd) {
            lo = g.fft[d] - (g.src[d] - (mx[d] - mn[d]));
            lo = std::max(0, std::min(lo, g.fft[d]));
            nvalid *= (g.fft[d] - lo);
        }
        s.lo[d] = lo;
        if (out_min && d < nd) out_min[d] = mn[d];
    }
    if (nnb == 0) {
        s.flags = SLOT_SKIP;  // candidateForPattern returns false on an empty pattern
        s.nterms = 0;
        return QSK_OK;
    }
    if (nvalid < (long long)K) s.flags |= SLOT_EMIT_MASKED;
    if (opts) {
        // a radius exclusion is a mask made by the caller (k_radius_mask)
        if (opts->exclude_index >= 0 && (long long)opts->exclude_index < g.N && !(opts->exclude_radius >= 1.f))
            s.excl = opts->exclude_index;
        if (opts->missing_data) {
            if (opts->centre_mask_layer < 0 || opts->centre_mask_layer >= ti->nlayers)
                return fail(QSK_ERR_ARG, "centre_mask_layer %d out of range", opts->centre_mask_layer);
            s.flags |= SLOT_MISSING;
            long long fmn = 0;
            for (int d = 0; d < nd; ++d) fmn += (long long)mn[d] * g.sstride[d];
            s.cmask_base = int((long long)opts->centre_mask_layer * g.N + fmn);
        }
    }
    out.clear();
    for (int t = 0; t < nterms; ++t) {
        const qsk_term &q = terms[t];
        if (q.neighbour < 0 || q.neighbour >= nnb || q.layer < 0 || q.layer >= ti->nlayers || q.op < 0 || q.op > 3)
            return fail(QSK_ERR_ARG, "pattern term %d out of range", t);
        long long dflat = 0;
        for (int d = 0; d < nd; ++d) dflat += (long long)(offsets[q.neighbour * nd + d] - mn[d]) * g.sstride[d];
        Term tm;
        tm.base = int((long long)q.layer * g.N - dflat);
        tm.a = q.a;
        tm.b = q.b;
        tm.op = q.op == QSK_OP_LIN_CROSS ? OP_LINX : q.op;
        out.push_back(tm);
    }
    s.nterms = int(out.size());
    return QSK_OK;
}

}  // namespace

extern "C" {

const char *qsk_last_error(void) { return g_err.c_str(); }

int qsk_device_count(int *count) {
    if (!count) return fail(QSK_ERR_ARG, "null count");
    int c = 0;
    cudaError_t e = cudaGetDeviceCount(&c);
    if (e != cudaSuccess) {
        *count = 0;
        return fail(QSK_ERR_CUDA, "cudaGetDeviceCount: %s", cudaGetErrorString(e));
    }
    *count = c;
    return QSK_OK;
}

static int check_sizes(int ndim, const unsigned *src, const unsigned *fft, int nlayers) {
    if (ndim < 1 || ndim > QSK_MAXD) return fail(QSK_ERR_UNSUPPORTED, "ndim %d not in [1,%d]", ndim, QSK_MAXD);
    long long N = 1;
    for (int d = 0; d < ndim; ++d) {
        if (src[d] == 0 || fft[d] < src[d]) return fail(QSK_ERR_ARG, "bad size in dimension %d", d);
        N *= fft[d];
    }
    if (N * (long long)std::max(nlayers, 1) >= (1LL << 31))
        return fail(QSK_ERR_UNSUPPORTED, "layers too large for 32-bit scan offsets (%lld x %d)", N, nlayers);
    return QSK_OK;
}

int qsk_ti_create_layers(int device, int ndim, const unsigned *src_size, const unsigned *fft_size, int nlayers,
                         const float *const *layers, qsk_ti **out) {
    if (!out || !src_size || !fft_size || !layers || nlayers < 1) return fail(QSK_ERR_ARG, "null argument");
    int rc = check_sizes(ndim, src_size, fft_size, nlayers);
    if (rc) return rc;
    DeviceGuard dgd(device);
    qsk_ti *t = new qsk_ti();
    t->device = device;
    t->g = make_geom(ndim, src_size, fft_size);
    t->nlayers = nlayers;
    cudaError_t e = t->layers.alloc(size_t(nlayers) * t->g.N);
    if (e != cudaSuccess) {
        delete t;
        return fail(QSK_ERR_NOMEM, "layers: %s", cudaGetErrorString(e));
    }
    for (int l = 0; l < nlayers; ++l) {
        e = cudaMemcpy(t->layers.p + size_t(l) * t->g.N, layers[l], sizeof(float) * t->g.N, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            delete t;
            return fail(QSK_ERR_CUDA, "layer upload: %s", cudaGetErrorString(e));
        }
    }
    *out = t;
    return QSK_OK;
}

static int ti_create_grid_impl(int device, int ndim, const unsigned *dims, int nvar, const int *types,
                               const float *data_in, bool data_on_device, qsk_ti **out) {
    if (!out || !dims || !types || !data_in || nvar < 1) return fail(QSK_ERR_ARG, "null argument");
    if (nvar > 4) return fail(QSK_ERR_UNSUPPORTED, "at most 4 variables (got %d)", nvar);
    if (data_on_device) return fail(QSK_ERR_UNSUPPORTED, "device-resident TI");
    std::vector<unsigned> fft(ndim);
    for (int d = 0; d < ndim && d < QSK_MAXD; ++d) fft[d] = fft_size_for(dims[d]);
    int rc = check_sizes(ndim, dims, fft.data(), nvar + 1);
    if (rc) return rc;
    long long cells = 1;
    for (int d = 0; d < ndim; ++d) cells *= dims[d];
    // missing values: for vector simulation a cell with any NaN variable is
    // treated as missing in every variable (src/qs.cpp:1436-1467)
    std::vector<float> data(data_in, data_in + size_t(cells) * nvar);
    bool missing = false;
    for (long long c = 0; c < cells; ++c) {
        bool hasNan = false;
        for (int v = 0; v < nvar; ++v) hasNan |= std::isnan(data[size_t(c) * nvar + v]);
        if (hasNan) {
            missing = true;
            for (int v = 0; v < nvar; ++v) data[size_t(c) * nvar + v] = NAN;
        }
    }
    if (missing)
        for (int v = 0; v < nvar; ++v)
            if (types[v] != 0)
                return fail(QSK_ERR_UNSUPPORTED,
                            "categorical variables with missing training-image values are undefined in G2S "
                            "(its converted neighbour values misalign, quantileSamplingModule.hpp:368-410)");
    DeviceGuard dgd(device);
    qsk_ti *t = new qsk_ti();
    t->device = device;
    t->g = make_geom(ndim, dims, fft.data());
    t->missing = missing;
    t->nlayers = nvar + (missing ? 1 : 0);
    t->nvar = nvar;
    t->types.assign(types, types + nvar);
    t->cells = cells;
    auto bail = [&](cudaError_t e) {
        delete t;
        return fail(e == cudaErrorMemoryAllocation ? QSK_ERR_NOMEM : QSK_ERR_CUDA, "ti upload: %s",
                    cudaGetErrorString(e));
    };
    cudaError_t e;
    if ((e = t->grid.alloc(size_t(t->cells) * nvar)) != cudaSuccess) return bail(e);
    if ((e = cudaMemcpy(t->grid.p, data.data(), sizeof(float) * t->cells * nvar, cudaMemcpyHostToDevice)) != cudaSuccess)
        return bail(e);
    if ((e = t->dtypes.alloc(nvar)) != cudaSuccess) return bail(e);
    if ((e = cudaMemcpy(t->dtypes.p, types, sizeof(int) * nvar, cudaMemcpyHostToDevice)) != cudaSuccess) return bail(e);
    if ((e = t->layers.alloc(size_t(t->nlayers) * t->g.N)) != cudaSuccess) return bail(e);
    if ((e = launch_build_layers(t->grid.p, nvar, t->dtypes.p, t->g, t->layers.p, missing ? 1 : 0, 0)) != cudaSuccess)
        return bail(e);
    if (missing) {
        std::vector<int> prefix(static_cast<size_t>(cells));
        int run = 0;
        for (long long c = 0; c < cells; ++c) {
            run += std::isnan(data[size_t(c) * nvar]) ? 0 : 1;
            prefix[size_t(c)] = run;
        }
        if ((e = t->complete_prefix.alloc(size_t(cells))) != cudaSuccess) return bail(e);
        if ((e = cudaMemcpy(t->complete_prefix.p, prefix.data(), sizeof(int) * cells, cudaMemcpyHostToDevice)) !=
            cudaSuccess)
            return bail(e);
    }
    // categories of every categorical variable (tensor-core indicator layers)
    t->cat_n.assign(nvar, 0);
    t->cat_v.assign(size_t(nvar) * QSK_CMAX, 0.f);
    for (int v = 0; v < nvar; ++v) {
        if (types[v] != 1) continue;
        for (long long i = 0; i < t->cells && t->cat_ok; ++i) {
            float x = data[size_t(i) * nvar + v];
            if (std::isnan(x)) continue;
            bool seen = false;
            for (int q = 0; q < t->cat_n[v]; ++q) seen |= (t->cat_v[size_t(v) * QSK_CMAX + q] == x);
            if (!seen) {
                if (t->cat_n[v] == QSK_CMAX) t->cat_ok = false;
                else t->cat_v[size_t(v) * QSK_CMAX + t->cat_n[v]++] = x;
            }
        }
    }
    // categories (distinct non-NaN codes) of categorical variables, for the bit planes
    bool all_cat = !missing;
    std::vector<int> ncat(nvar, 0);
    std::vector<float> catv(size_t(nvar) * QSK_CMAX, 0.f);
    for (int v = 0; v < nvar && all_cat; ++v) {
        if (types[v] != 1) { all_cat = false; break; }
        for (long long i = 0; i < t->cells && all_cat; ++i) {
            float x = data[size_t(i) * nvar + v];
            if (std::isnan(x)) continue;
            bool seen = false;
            for (int q = 0; q < ncat[v]; ++q) seen |= (catv[size_t(v) * QSK_CMAX + q] == x);
            if (!seen) {
                if (ncat[v] == QSK_CMAX) all_cat = false;
                else catv[size_t(v) * QSK_CMAX + ncat[v]++] = x;
            }
        }
    }
    if (all_cat) {
        t->pw = plane_words(t->g.N);
        if ((e = t->ncat.alloc(nvar)) != cudaSuccess) return bail(e);
        if ((e = t->catv.alloc(catv.size())) != cudaSuccess) return bail(e);
        if ((e = t->planes.alloc(size_t(nvar) * (QSK_CMAX + 1) * t->pw)) != cudaSuccess) return bail(e);
        if ((e = cudaMemcpy(t->ncat.p, ncat.data(), sizeof(int) * nvar, cudaMemcpyHostToDevice)) != cudaSuccess) return bail(e);
        if ((e = cudaMemcpy(t->catv.p, catv.data(), sizeof(float) * catv.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
            return bail(e);
        if ((e = launch_build_planes(t->layers.p, t->g, nvar, t->ncat.p, t->catv.p, t->pw, t->planes.p, 0)) != cudaSuccess)
            return bail(e);
        t->planes_ok = true;
    }
    if ((e = cudaStreamSynchronize(0)) != cudaSuccess) return bail(e);
    *out = t;
    return QSK_OK;
}

int qsk_ti_create_grid(int device, int ndim, const unsigned *dims, int nvar, const int *types, const float *data,
                       qsk_ti **out) {
    return ti_create_grid_impl(device, ndim, dims, nvar, types, data, false, out);
}

int qsk_ti_fft_size(const qsk_ti *ti, unsigned *fft_size) {
    if (!ti || !fft_size) return fail(QSK_ERR_ARG, "null argument");
    for (int d = 0; d < ti->g.nd; ++d) fft_size[d] = unsigned(ti->g.fft[d]);
    return QSK_OK;
}

int qsk_ti_destroy(qsk_ti *ti) {
    if (!ti) return QSK_OK;
    DeviceGuard dgd(ti->device);
    delete ti;
    return QSK_OK;
}

int qsk_worker_create(qsk_ti *ti, qsk_worker **out) {
    if (!ti || !out) return fail(QSK_ERR_ARG, "null argument");
    DeviceGuard dgd(ti->device);
    qsk_worker *w = new qsk_worker();
    w->ti = ti;
    cudaError_t e = cudaStreamCreateWithFlags(&w->st, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete w;
        return fail(QSK_ERR_CUDA, "stream: %s", cudaGetErrorString(e));
    }
    *out = w;
    return QSK_OK;
}

int qsk_worker_destroy(qsk_worker *w) {
    if (!w) return QSK_OK;
    DeviceGuard dgd(w->ti->device);
    if (w->st) cudaStreamDestroy(w->st);
    delete w;
    return QSK_OK;
}

static int pattern_batch_impl(qsk_worker *w, int B, const int *nb_ptr, const int *offsets, const int *term_ptr,
                              const qsk_term *terms, unsigned k, const float *seeds, float *out_score,
                              unsigned *out_index, int *out_min, const qsk_pattern_opts *opts,
                              const unsigned *origin = nullptr, const float *radius = nullptr) {
    if (!w || B < 0 || !nb_ptr || !term_ptr || !seeds || !out_score || !out_index) return fail(QSK_ERR_ARG, "null argument");
    if (k < 1 || k > QSK_KMAX) return fail(QSK_ERR_UNSUPPORTED, "k=%u outside [1,%d]", k, QSK_KMAX);
    if (B == 0) return QSK_OK;
    if (B > 65535) return fail(QSK_ERR_UNSUPPORTED, "at most 65535 patterns per batch (got %d)", B);
    qsk_ti *ti = w->ti;
    DeviceGuard dgd(ti->device);
    const Geom &g = ti->g;
    const int nd = g.nd;
    w->h_slots.resize(B);
    int maxterms = 1;
    for (int b = 0; b < B; ++b) maxterms = std::max(maxterms, term_ptr[b + 1] - term_ptr[b]);
    w->h_terms.assign(size_t(B) * maxterms, Term{0, 0.f, 0.f, 0});
    std::vector<Term> tmp;
    for (int b = 0; b < B; ++b) {
        int nnb = nb_ptr[b + 1] - nb_ptr[b];
        int nt = term_ptr[b + 1] - term_ptr[b];
        int rc = build_pattern_slot(ti, nnb, offsets + size_t(nb_ptr[b]) * nd, nt, terms + term_ptr[b], k, seeds[b], b,
                                    w->h_slots[b], tmp, out_min ? out_min + size_t(b) * nd : nullptr, opts);
        if (rc) return rc;
        std::copy(tmp.begin(), tmp.end(), w->h_terms.begin() + size_t(b) * maxterms);
    }
    // verbatim exclusion of each pattern's origin (the TI cell the pattern was
    // taken from): one scan index, or every index within the radius
    std::vector<int> xc;
    std::vector<float> xr;
    bool any_radius = false;
    if (opts && opts->exclude_radius >= 1.f && opts->exclude_index >= 0 && (long long)opts->exclude_index < g.N) {
        xc.assign(B, -1);
        xr.assign(B, 0.f);
        for (int b = 0; b < B; ++b) {
            if (w->h_slots[b].flags & SLOT_SKIP) continue;
            xc[b] = opts->exclude_index;
            xr[b] = opts->exclude_radius;
            any_radius = true;
        }
    } else if (origin) {
        xc.assign(B, -1);
        xr.assign(B, 0.f);
        for (int b = 0; b < B; ++b) {
            Slot &sl = w->h_slots[b];
            if (origin[b] == 0xffffffffu || (sl.flags & SLOT_SKIP)) continue;
            if ((long long)origin[b] >= ti->cells) return fail(QSK_ERR_ARG, "origin %u of pattern %d outside the TI", origin[b], b);
            const unsigned idx = qsk_position_to_index(ti, sl.mn, origin[b]);
            const float rad = radius ? radius[b] : 0.f;
            if (rad >= 1.f) {
                xc[b] = int(idx);
                xr[b] = rad;
                any_radius = true;
            } else if ((long long)idx < g.N) {
                sl.excl = int(idx);
            }
        }
    }
    if (smem_configured_device != ti->device) {
        CK(set_map_smem_limit(200 * 1024));
        smem_configured_device = ti->device;
    }
    if ((size_t)maxterms * sizeof(Term) > 200 * 1024) return fail(QSK_ERR_UNSUPPORTED, "too many terms (%d)", maxterms);
    CK(w->slots.upload(w->h_slots.data(), B, w->st));
    CK(w->terms.upload(w->h_terms.data(), w->h_terms.size(), w->st));
    CK(ensure_records(g, B, w->rec_val, w->rec_idx, w->rec_cnt, w->rec_max));
    CK(w->out_val.ensure(size_t(B) * k));
    CK(w->out_pos.ensure(size_t(B) * k));
    // the radius masks are applied by the FP32 kernel (the bit-sliced one gives
    // the same scores, so the choice changes no result)
    bool bits = ti->planes_ok && g_map_mode == 0 && maxterms <= 255 && !opts && !any_radius;
    for (size_t i = 0; i < w->h_terms.size() && bits; ++i) {
        int b = int(i / maxterms), t = int(i % maxterms);
        if (t >= w->h_slots[b].nterms) continue;
        bits &= (w->h_terms[i].op == OP_EQ && w->h_terms[i].a == 1.f);
    }
    if (bits) {
        BitArgs ba;
        ba.g = g;
        ba.planes = ti->planes.p;
        ba.pw = ti->pw;
        ba.ncat = ti->ncat.p;
        ba.catv = ti->catv.p;
        ba.slots = w->slots.p;
        ba.terms = w->terms.p;
        ba.maxterms = maxterms;
        ba.segs_per_cta = map_bits_segs_per_cta(g, B);
        ba.rec_val = w->rec_val.p;
        ba.rec_idx = w->rec_idx.p;
        ba.rec_cnt = w->rec_cnt.p;
        ba.rec_max = w->rec_max.p;
        CK(launch_map_bits(ba, B, int(k), maxterms, w->st));
    } else {
        MapArgs ma;
        ma.g = g;
        ma.layers = ti->layers.p;
        ma.slots = w->slots.p;
        ma.terms = w->terms.p;
        ma.maxterms = maxterms;
        ma.segs_per_cta = map_segs_per_cta(g, B);
        ma.rec_val = w->rec_val.p;
        ma.rec_idx = w->rec_idx.p;
        ma.rec_cnt = w->rec_cnt.p;
        ma.rec_max = w->rec_max.p;
        if (any_radius) {
            const long long xwords = (g.N + 31) / 32;
            CK(w->xcenter.upload(xc.data(), size_t(B), w->st));
            CK(w->xradius.upload(xr.data(), size_t(B), w->st));
            CK(w->xmask.ensure(size_t(B) * size_t(xwords)));
            CK(launch_radius_mask(w->xcenter.p, w->xradius.p, B, g, w->xmask.p, xwords, w->st));
            ma.xmask = w->xmask.p;
            ma.xwords = xwords;
        }
        CK(launch_map_records(ma, B, int(k), maxterms, w->st));
    }
    ReplayArgs ra;
    std::memset(&ra, 0, sizeof(ra));
    ra.g = g;
    ra.slots = w->slots.p;
    ra.nslots = B;
    ra.K = int(k);
    ra.rec_val = w->rec_val.p;
    ra.rec_idx = w->rec_idx.p;
    ra.rec_cnt = w->rec_cnt.p;
    ra.rec_max = w->rec_max.p;
    ra.out_val = w->out_val.p;
    ra.out_pos = w->out_pos.p;
    CK(launch_replay(ra, w->st));
    CK(cudaMemcpyAsync(out_score, w->out_val.p, sizeof(float) * B * k, cudaMemcpyDeviceToHost, w->st));
    CK(cudaMemcpyAsync(out_index, w->out_pos.p, sizeof(unsigned) * B * k, cudaMemcpyDeviceToHost, w->st));
    CK(cudaStreamSynchronize(w->st));
    // empty patterns keep -inf scores (candidateForPattern returned false)
    for (int b = 0; b < B; ++b)
        if (w->h_slots[b].flags & SLOT_SKIP)
            for (unsigned j = 0; j < k; ++j) {
                out_score[size_t(b) * k + j] = -INFINITY;
                out_index[size_t(b) * k + j] = 0xffffffffu;
            }
    return QSK_OK;
}

int qsk_pattern_kbest_batch(qsk_worker *w, int B, const int *nb_ptr, const int *offsets, const int *term_ptr,
                            const qsk_term *terms, unsigned k, const float *seeds, float *out_score,
                            unsigned *out_index, int *out_min) {
    return pattern_batch_impl(w, B, nb_ptr, offsets, term_ptr, terms, k, seeds, out_score, out_index, out_min, nullptr);
}

int qsk_pattern_kbest_batch_verbatim(qsk_worker *w, int B, const int *nb_ptr, const int *offsets, const int *term_ptr,
                                     const qsk_term *terms, unsigned k, const float *seeds, const unsigned *origin,
                                     const float *radius, float *out_score, unsigned *out_index, int *out_min) {
    if (!origin) return fail(QSK_ERR_ARG, "null origin");
    return pattern_batch_impl(w, B, nb_ptr, offsets, term_ptr, terms, k, seeds, out_score, out_index, out_min, nullptr,
                              origin, radius);
}

int qsk_pattern_kbest(qsk_worker *w, int n_neighbours, const int *offsets, int n_terms, const qsk_term *terms,
                      unsigned k, float seed, float *out_score, unsigned *out_index, int *out_min) {
    int nb_ptr[2] = {0, n_neighbours};
    int term_ptr[2] = {0, n_terms};
    return pattern_batch_impl(w, 1, nb_ptr, offsets, term_ptr, terms, k, &seed, out_score, out_index, out_min,
                              nullptr);
}

int qsk_pattern_kbest_ex(qsk_worker *w, int n_neighbours, const int *offsets, int n_terms, const qsk_term *terms,
                         unsigned k, float seed, const qsk_pattern_opts *opts, float *out_score, unsigned *out_index,
                         int *out_min) {
    int nb_ptr[2] = {0, n_neighbours};
    int term_ptr[2] = {0, n_terms};
    return pattern_batch_impl(w, 1, nb_ptr, offsets, term_ptr, terms, k, &seed, out_score, out_index, out_min, opts);
}

unsigned qsk_index_to_position(const qsk_ti *ti, const int *min_offset, unsigned index) {
    const Geom &g = ti->g;
    unsigned position = 0;
    unsigned div = unsigned(g.N);
    for (int i = g.nd - 1; i >= 0; --i) {
        unsigned f = unsigned(g.fft[i]), s = unsigned(g.src[i]);
        div /= f;
        position = position * s + ((f - (index / div) % f - unsigned(min_offset[i]) - 1u) + s) % s;
    }
    return position;
}

unsigned qsk_position_to_index(const qsk_ti *ti, const int *min_offset, unsigned position) {
    const Geom &g = ti->g;
    unsigned index = 0;
    unsigned div = 1;
    for (int i = g.nd - 1; i >= 0; --i) div *= unsigned(g.src[i]);
    for (int i = g.nd - 1; i >= 0; --i) {
        unsigned f = unsigned(g.fft[i]), s = unsigned(g.src[i]);
        div /= s;
        index = index * f + (f - (position / div + unsigned(min_offset[i])) % s - 1u);
    }
    return index;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// full simulation
// ---------------------------------------------------------------------------
struct qsk_sim {
    int device = 0;
    cudaStream_t st = nullptr;
    // generator states are prepared on st_rng while st runs the map
    cudaStream_t st_rng = nullptr;
    cudaEvent_t ev_ready[2] = {nullptr, nullptr}, ev_used[2] = {nullptr, nullptr};
    // tensor-core form: a level's exact-map steps run on st2 beside its
    // tensor steps on st (ev_level: the level's start on st; ev_side: the
    // end of st2's work, which the next level waits for)
    cudaStream_t st2 = nullptr;
    cudaEvent_t ev_level = nullptr, ev_side = nullptr;
    qsk_ti *ti = nullptr;
    int nd = 0, nvar = 0, n = 0, K = 1;
    float k = 1.f;
    unsigned seed = 0;
    int no_verbatim = 0;
    GridDesc dg;
    long long cells = 0, nodes = 0;
    unsigned begin = 0;
    // host plan
    std::vector<int> tpl;            // ntpl * nd
    std::vector<float> wtab;         // ntpl * nvar
    std::vector<unsigned> order;     // path (all cells)
    std::vector<float> seeds;        // per path index
    std::vector<unsigned> posterior; // per cell
    std::vector<int> node_of_cell;   // per cell
    std::vector<float> init;         // grid before simulation
    int ntpl = 0;
    // local controls: per kernel template range (begin, count); per path
    // node kernel, neighbour limit, neighbour count per variable, k
    std::vector<int> tpl_range;
    std::vector<int> node_kernel, node_lim, node_nv;
    std::vector<float> node_k;
    bool local = false;
    bool full = false;               // -fs: nodes are (cell, variable) values
    // device
    DBuf<int> d_tpl, d_types;
    DBuf<float> d_wtab, d_seeds, d_init, d_state;
    DBuf<unsigned> d_path, d_post, d_id, d_node_cell, d_nb_cell;
    DBuf<int> d_node_of_cell, d_nb_count, d_nb_tpl, d_level_nodes, d_status;
    // dependency levels (Kahn frontiers over the reverse edges)
    DBuf<int> d_level, d_cursor, d_tile_sum, d_lcnt, d_start, d_nl;
    DBuf<Slot> d_slots;
    DBuf<Term> d_terms;
    DBuf<float> d_rec_val;
    DBuf<int> d_rec_idx, d_rec_cnt;
    DBuf<float> d_rec_max;
    DBuf<unsigned> d_mt_state;       // [2][slot][624]: two batches
    DBuf<Slot> d_sslots;             // bit-sliced path: [2][slot] slots written one batch ahead
    DBuf<StaticTerm> d_sterms;       // and their terms without values [2][slot][maxterms]
    DBuf<int> d_mt_pre;
    DBuf<int> d_tpl_range, d_node_kernel, d_node_lim, d_node_nv;
    DBuf<unsigned char> d_nb_mask;
    DBuf<float> d_node_k;
    int maxterms = 0;
    int max_slots = 0;
    bool use_bits = false;
    qsk_sim_info info;
    bool neighbours_ready = false;
    bool profiling = false;
    bool use_graph = false;             // plain path: the batch chain as one CUDA graph
    // tensor-core form (qsk_sim_set_tensor)
    qsk_tensor_opts topt{};             // mode 0: off
    int tc_T = 0, tc_L = 0, tc_W = 0, tc_S = 0, tc_fmt = 0;
    int tc_T_auto = 0;                  // automatic prefix, chosen at the first tensor run
    long long tc_Kp = 0, tc_rows = 0;
    bool tc_ready = false;              // pattern matrix built for (tc_T, tc_fmt)
    std::vector<int> var_layer0;
    DBuf<unsigned char> d_tc_P;         // tc_rows x tc_Kp
    DBuf<float> d_tc_pscale;
    DBuf<unsigned char> d_tc_A;         // slots x tc_Kp
    DBuf<float> d_tc_nscale, d_tc_bias;
    DBuf<int> d_tc_box, d_tc_tmax, d_tc_kb, d_var_layer0, d_var_ncat;
    DBuf<unsigned> d_tc_seed, d_tc_pos, d_tc_thr;
    DBuf<float> d_var_catv, d_drawn_score, d_drawn_scale;
    DBuf<unsigned long long> d_tc_key, d_tc_counts;
    DBuf<Slot> d_tc_slots;
    DBuf<Term> d_tc_terms;
    DBuf<int> d_audit_nodes;
    DBuf<float> d_audit_val;
    DBuf<unsigned> d_audit_pos, d_err_max;
    DBuf<double> d_err_sum;
    DBuf<unsigned long long> d_err_n;
    int max_tc_slots = 0;
    int sm_count = 0;
    // several training images: the TIs after ti, the -ii image, and every
    // TI's K best per slot of a batch ([ti][slot][K], TI cells)
    std::vector<qsk_ti *> xti;
    DBuf<float> d_ii, d_mval;
    DBuf<unsigned> d_mcell;
    std::vector<qsk_ti *> all_tis() const {
        std::vector<qsk_ti *> v{ti};
        v.insert(v.end(), xti.begin(), xti.end());
        return v;
    }                   // SMs of the device (grid sizing of the shortlist kernel)
    // learned proposal (qsk_sim_set_learned): tensor mode 3
    qsk_encoder *enc = nullptr;
    qsk_learned_opts lopt{};
    int enc_built = -1;                 // encoder Adam step count the TI embeddings were built at
    int enc_ns = 0;                     // ... and its number of stencil scales (P holds one matrix per scale)
    DBuf<int> d_ent_cube;               // stencil entry of every offset of the stencil's box (-1: none)
    int cube_lo[3] = {0, 0, 0}, cube_dim[3] = {1, 1, 1};
    DBuf<int> d_lscale;                 // stencil scale per position of the level order
    DBuf<float> d_feat;                 // encoder input rows of a step / a chunk of TI cells
    DBuf<int> d_fb;                     // per slot: confidence check failed
    DBuf<int> d_fb_nodes;
    std::vector<cudaEvent_t> tc_ev;     // profiling: 3 events per tensor step
    size_t tc_ev_used = 0;
    unsigned level_spin_limit = 0;      // 0: the kernel's default
    long long level_hold = -1;          // failure-path test: a node whose level is never published
    std::vector<cudaEvent_t> prof_ev;   // 4 events per batch in profiling mode
    size_t prof_used = 0;
};

namespace {

// a1: sorted search template (src/qs.cpp:1055-1135); fills tpl (ntpl*nd) and
// the kernel weight of every offset and variable (wtab, ntpl*nvar)
int make_template(int nd, int nvar, const unsigned *kdims, const float *kernel, std::vector<int> &tpl_out,
                  std::vector<float> &wtab_out) {
    std::vector<std::vector<int>> pos;
    pos.push_back(std::vector<int>());
    for (int i = 0; i < nd; ++i) {
        size_t orig = pos.size();
        int half = (int(kdims[i]) + 1) / 2;
        pos.resize(orig * (2 * half - 1));
        for (size_t q = 0; q < orig; ++q) pos[q].push_back(0);
        for (int j = 1; j < half; ++j) {
            std::copy(pos.begin(), pos.begin() + orig, pos.begin() + orig * (2 * j - 1));
            std::copy(pos.begin(), pos.begin() + orig, pos.begin() + orig * (2 * j));
            for (size_t q = orig * (2 * j - 1); q < orig * (2 * j); ++q) pos[q][i] = j;
            for (size_t q = orig * (2 * j); q < orig * (2 * j + 1); ++q) pos[q][i] = -j;
        }
    }
    long long kstride[QSK_MAXD];
    long long ks = 1;
    for (int d = 0; d < nd; ++d) {
        kstride[d] = ks;
        ks *= kdims[d];
    }
    if (kernel) {  // remove offsets whose kernel weight (variable 0) is NaN (src/qs.cpp:1107-1128)
        std::vector<std::vector<int>> kept;
        for (auto &v : pos) {
            long long f = 0;
            for (int d = 0; d < nd; ++d) f += (long long)(int((kdims[d] - 1) / 2) + v[d]) * kstride[d];
            if (!std::isnan(kernel[size_t(f) * nvar])) kept.push_back(v);
        }
        pos.swap(kept);
    }
    std::sort(pos.begin(), pos.end(), [](const std::vector<int> &a, const std::vector<int> &b) {
        float da = 0.f, db = 0.f;
        for (size_t i = 0; i < a.size(); ++i) da += float(a[i] * a[i]);
        for (size_t i = 0; i < b.size(); ++i) db += float(b[i] * b[i]);
        return -da > -db;
    });
    const int ntpl = int(pos.size());
    tpl_out.resize(size_t(ntpl) * nd);
    wtab_out.resize(size_t(ntpl) * nvar);
    for (int t = 0; t < ntpl; ++t) {
        for (int d = 0; d < nd; ++d) tpl_out[size_t(t) * nd + d] = pos[t][d];
        // weight lookup centred at dims/2 (quantileSamplingModule.hpp:362-366)
        for (int v = 0; v < nvar; ++v) {
            float w = 1.f;
            if (kernel) {
                long long f = 0;
                bool ok = true;
                for (int d = 0; d < nd; ++d) {
                    int c = int(kdims[d] / 2) + pos[t][d];
                    ok &= c >= 0 && c < int(kdims[d]);
                    f += (long long)c * kstride[d];
                }
                w = ok ? kernel[size_t(f) * nvar + v] : 0.f;
            }
            wtab_out[size_t(t) * nvar + v] = w;
        }
    }
    return ntpl;
}

// append one kernel's template and weights to the concatenated tables
void add_template(qsk_sim *s, const unsigned *kdims, const float *kernel) {
    std::vector<int> t;
    std::vector<float> w;
    int nt = make_template(s->nd, s->nvar, kdims, kernel, t, w);
    s->tpl_range.push_back(s->ntpl);
    s->tpl_range.push_back(nt);
    s->tpl.insert(s->tpl.end(), t.begin(), t.end());
    s->wtab.insert(s->wtab.end(), w.begin(), w.end());
    s->ntpl += nt;
}

// a2: path and per-node seeds (src/qs.cpp:975,1159-1201,1250-1258): informed
// cells first, the rest shuffled by mt19937(seed); then one U[0,1) float per
// path position from the same generator.  Returns the number of informed cells.
unsigned make_path(size_t n, int nvar, const float *init, unsigned seed, std::vector<unsigned> &order,
                   std::vector<float> &seeds) {
    std::mt19937 gen(seed);
    order.resize(n);
    std::iota(order.begin(), order.end(), 0u);
    unsigned begin = 0;
    for (size_t i = 0; i < n; ++i) {
        bool set = true;
        for (int v = 0; v < nvar; ++v)
            if (std::isnan(init[i * nvar + v])) set = false;
        if (set) {
            std::swap(order[begin], order[i]);
            begin++;
        }
    }
    std::shuffle(order.begin() + begin, order.end(), gen);
    std::uniform_real_distribution<float> u(0.f, 1.f);
    seeds.resize(n);
    for (size_t i = 0; i < n; ++i) {
        seeds[i] = u(gen);
        if (seeds[i] == 1.f) seeds[i] = u(gen);
    }
    return begin;
}

// -fs: path over the cells*nvar values, informed values first
// (src/qs.cpp:1159-1183,1250-1258,1614-1638)
void build_path_full(qsk_sim *s) {
    const size_t n = size_t(s->cells) * s->nvar;
    std::mt19937 gen(s->seed);
    s->order.resize(n);
    std::iota(s->order.begin(), s->order.end(), 0u);
    unsigned begin = 0;
    for (size_t i = 0; i < n; ++i)
        if (!std::isnan(s->init[i])) {
            std::swap(s->order[begin], s->order[i]);
            begin++;
        }
    std::shuffle(s->order.begin() + begin, s->order.end(), gen);
    std::uniform_real_distribution<float> u(0.f, 1.f);
    s->seeds.resize(n);
    for (size_t i = 0; i < n; ++i) {
        s->seeds[i] = u(gen);
        if (s->seeds[i] == 1.f) s->seeds[i] = u(gen);
    }
    s->begin = begin;
    s->nodes = (long long)n - begin;
    s->posterior.assign(n, std::numeric_limits<unsigned>::max());
    s->node_of_cell.assign(n, -1);   // per value
    for (size_t i = 0; i < n; ++i)
        if (!std::isnan(s->init[i])) s->posterior[i] = 0;
    for (long long i = 0; i < s->nodes; ++i) {
        s->posterior[s->order[begin + i]] = unsigned(i);
        s->node_of_cell[s->order[begin + i]] = int(i);
    }
}

// posterior order (src/qs.cpp:1604-1641)
void build_path(qsk_sim *s) {
    const size_t n = size_t(s->cells);
    unsigned begin = make_path(n, s->nvar, s->init.data(), s->seed, s->order, s->seeds);
    s->begin = begin;
    s->nodes = (long long)n - begin;
    s->posterior.assign(n, std::numeric_limits<unsigned>::max());
    s->node_of_cell.assign(n, -1);
    for (size_t i = 0; i < n; ++i) {
        bool withNan = false;
        for (int v = 0; v < s->nvar; ++v) withNan |= std::isnan(s->init[i * s->nvar + v]);
        if (!withNan) s->posterior[i] = 0;
    }
    for (long long i = 0; i < s->nodes; ++i) {
        s->posterior[s->order[begin + i]] = unsigned(i);
        s->node_of_cell[s->order[begin + i]] = int(i);
    }
}

int sim_neighbours(qsk_sim *s) {
    if (s->neighbours_ready) return QSK_OK;
    if (s->full) {
        CK(launch_neighbours_full(s->dg, s->d_tpl.p, s->ntpl, s->d_path.p, s->begin, s->nodes, s->d_post.p, s->nvar,
                                  s->n, s->local ? s->d_node_nv.p : nullptr, s->d_nb_count.p, s->d_nb_tpl.p,
                                  s->d_nb_cell.p, s->d_nb_mask.p, s->local ? s->d_node_kernel.p : nullptr,
                                  s->local ? s->d_tpl_range.p : nullptr, s->st));
        s->neighbours_ready = true;
        return QSK_OK;
    }
    CK(launch_neighbours(s->dg, s->d_tpl.p, s->ntpl, s->d_path.p, s->begin, s->nodes,
                         s->d_post.p, s->n, s->d_nb_count.p, s->d_nb_tpl.p, s->d_nb_cell.p,
                         s->local ? s->d_node_kernel.p : nullptr, s->local ? s->d_tpl_range.p : nullptr,
                         s->local ? s->d_node_lim.p : nullptr, s->st));
    s->neighbours_ready = true;
    return QSK_OK;
}

// run the batches of nodes listed in d_level_nodes[start[l]..start[l+1]) for each level
cudaEvent_t prof_event(qsk_sim *s) {
    if (s->prof_used == s->prof_ev.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        s->prof_ev.push_back(e);
    }
    return s->prof_ev[s->prof_used++];
}

// One launch group of the batched engine: `B` nodes from `nodes + off`.
//   PLAIN   the exact path (prep, map, k-best replay, write-back)
//   TENSOR  the tensor-core form (node rows, GEMM shortlist, re-score, draw)
//   AUDIT   the exact path without write-back, k best to the audit buffers
//   HASH    the exact map, then the k best by (score, tie hash) over its
//           records (the tensor-core form's draw rule, for the nodes it
//           leaves to the map); marginal draws still replay
enum StepKind { STEP_PLAIN = 0, STEP_TENSOR = 1, STEP_AUDIT = 2, STEP_HASH = 3 };
struct Step {
    int kind;
    const int *nodes;   // device node list
    int off, B;
    int kb_off;         // TENSOR: this step's tile K-blocks in d_tc_kb
    int scale = 1;      // TENSOR, learned proposal: the nodes' stencil scale
    int level = -1;     // tensor-core form: the dependency level (-1: one stream for all steps)
};

int tc_step(qsk_sim *s, const Step &st, bool teacher);

// plain steps, one per slot budget of every level (levels in order)
std::vector<Step> plain_steps(qsk_sim *s, const std::vector<int> &start) {
    std::vector<Step> steps;
    for (size_t l = 0; l + 1 < start.size(); ++l)
        for (int off = start[l]; off < start[l + 1]; off += s->max_slots)
            steps.push_back({STEP_PLAIN, s->d_level_nodes.p, off, std::min(s->max_slots, start[l + 1] - off), 0});
    return steps;
}

int sim_batches(qsk_sim *s, const std::vector<Step> &steps, bool teacher) {
    const Geom &g = s->ti->g;
    s->prof_used = 0;
    s->tc_ev_used = 0;
    // plain / audit steps (the generator-state pipeline runs over these only)
    std::vector<size_t> pl;
    for (size_t j = 0; j < steps.size(); ++j)
        if (steps[j].kind != STEP_TENSOR) pl.push_back(j);
    auto prep_args = [&](const int *nodes, int off, int B) {
        SimPrepArgs pa;
        pa.g = g;
        pa.dg = s->dg;
        pa.nvar = s->nvar;
        pa.types = s->d_types.p;
        pa.tpl = s->d_tpl.p;
        pa.wtab = s->d_wtab.p;
        pa.path = s->d_path.p;
        pa.begin = s->begin;
        pa.seeds = s->d_seeds.p;
        pa.nb_count = s->d_nb_count.p;
        pa.nb_tpl = s->d_nb_tpl.p;
        pa.nb_cell = s->d_nb_cell.p;
        pa.n = s->n;
        pa.state = s->d_state.p;
        pa.init = s->d_init.p;
        pa.nodes = nodes + off;
        pa.nslots = B;
        pa.k = s->k;
        pa.K = s->K;
        pa.nti = 1;
        pa.slots = s->d_slots.p;
        pa.terms = s->d_terms.p;
        pa.maxterms = s->maxterms;
        pa.status = s->d_status.p;
        pa.missing = s->ti->missing ? 1 : 0;
        pa.mask_layer = s->nvar;
        pa.no_verbatim = s->no_verbatim;
        pa.id_image = s->d_id.p;
        pa.node_nv = s->local ? s->d_node_nv.p : nullptr;
        pa.node_k = s->local ? s->d_node_k.p : nullptr;
        pa.full = s->full ? 1 : 0;
        pa.nb_mask = s->full ? s->d_nb_mask.p : nullptr;
        return pa;
    };
    // Generator states of batch j go to buffer j % 2 on st_rng, one batch
    // ahead of the simulation on st; buffer p is rewritten only after the
    // replay that read it (ev_used[p]).
    const size_t mt_words = size_t(s->max_slots) * 624;
    // bit-sliced map: slots and value-free terms also come one batch ahead
    // (k_mt_prep); the map reads the neighbour values itself, so nothing
    // runs before it on st
    const bool bits = s->use_bits && g_map_mode == 0;
    const size_t st_words = size_t(s->max_slots) * s->maxterms;
    auto launch_rng = [&](size_t j) -> int {
        const int p = int(j & 1);
        CK(cudaStreamWaitEvent(s->st_rng, s->ev_used[p], 0));
        const Step &sj = steps[pl[j]];
        SimPrepArgs pa = prep_args(sj.nodes, sj.off, sj.B);
        if (bits) {
            pa.slots = s->d_sslots.p + size_t(p) * s->max_slots;
            pa.sterms = s->d_sterms.p + p * st_words;
        }
        CK(launch_mt_prep(pa, s->d_mt_state.p + p * mt_words, s->d_mt_pre.p + size_t(p) * s->max_slots, s->st_rng));
        CK(cudaEventRecord(s->ev_ready[p], s->st_rng));
        return QSK_OK;
    };
    CK(cudaEventRecord(s->ev_used[0], s->st));   // after everything queued so far on st
    CK(cudaEventRecord(s->ev_used[1], s->st));
    int rc = pl.empty() ? QSK_OK : launch_rng(0);
    if (rc) return rc;
    size_t j = 0;   // plain / audit step counter
    // tensor-core form: the exact-map steps of a level (its nodes beyond the
    // prefix) run on st2 while its tensor steps run on st; the nodes of a
    // level are independent (they read earlier levels only and write their
    // own cells) and the two kinds of step share no scratch.  A level
    // starts when both streams have finished the one before.
    int cur_level = -1, side_level = -1;
    bool side_pending = false;
    for (const Step &step : steps) {
        if (step.level >= 0 && step.level != cur_level) {
            if (side_pending) CK(cudaStreamWaitEvent(s->st, s->ev_side, 0));
            side_pending = false;
            CK(cudaEventRecord(s->ev_level, s->st));
            cur_level = step.level;
        }
        if (step.kind == STEP_TENSOR) {
            if ((rc = tc_step(s, step, teacher)) != QSK_OK) return rc;
            continue;
        }
        const bool side = step.kind == STEP_HASH && step.level >= 0;
        cudaStream_t ws = side ? s->st2 : s->st;
        if (side && side_level != step.level) {
            CK(cudaStreamWaitEvent(s->st2, s->ev_level, 0));
            side_level = step.level;
        }
        const int B = step.B, p = int(j & 1);
        const bool audit = step.kind == STEP_AUDIT;
        if (j + 1 < pl.size() && (rc = launch_rng(j + 1)) != QSK_OK) return rc;
        ++j;
        {
            Slot *slots = bits ? s->d_sslots.p + size_t(p) * s->max_slots : s->d_slots.p;
            if (s->profiling) CK(cudaEventRecord(prof_event(s), ws));
            if (!bits) CK(launch_prep_sim(prep_args(step.nodes, step.off, B), ws));
            if (s->profiling) CK(cudaEventRecord(prof_event(s), ws));
            if (bits) {
                // the slots and static terms of this batch come from k_mt_prep
                CK(cudaStreamWaitEvent(ws, s->ev_ready[p], 0));
                BitArgs ba;
                ba.g = g;
                ba.planes = s->ti->planes.p;
                ba.pw = s->ti->pw;
                ba.ncat = s->ti->ncat.p;
                ba.catv = s->ti->catv.p;
                ba.slots = slots;
                ba.terms = nullptr;
                ba.sterms = s->d_sterms.p + p * st_words;
                ba.state = s->d_state.p;
                ba.init = s->d_init.p;
                ba.id_image = s->d_id.p;
                ba.tpl = s->d_tpl.p;
                ba.no_verbatim = s->no_verbatim;
                ba.maxterms = s->maxterms;
                ba.segs_per_cta = map_bits_segs_per_cta(g, B);
                ba.rec_val = s->d_rec_val.p;
                ba.rec_idx = s->d_rec_idx.p;
                ba.rec_cnt = s->d_rec_cnt.p;
                ba.rec_max = s->d_rec_max.p;
                CK(launch_map_bits(ba, B, s->K, s->maxterms, ws));
            } else {
                MapArgs ma;
                ma.g = g;
                ma.layers = s->ti->layers.p;
                ma.slots = s->d_slots.p;
                ma.terms = s->d_terms.p;
                ma.maxterms = s->maxterms;
                ma.segs_per_cta = map_segs_per_cta(g, B);
                ma.rec_val = s->d_rec_val.p;
                ma.rec_idx = s->d_rec_idx.p;
                ma.rec_cnt = s->d_rec_cnt.p;
                ma.rec_max = s->d_rec_max.p;
                CK(launch_map_records(ma, B, s->K, s->maxterms, ws));
            }
            if (s->profiling) CK(cudaEventRecord(prof_event(s), ws));
            s->info.launches += bits ? 3 : 4;
            s->info.map_launches += 1;
            s->info.map_positions += (long long)B * g.N;
            ReplayArgs ra;
            std::memset(&ra, 0, sizeof(ra));
            ra.g = g;
            ra.slots = slots;
            ra.nslots = B;
            ra.K = s->K;
            ra.rec_val = s->d_rec_val.p;
            ra.rec_idx = s->d_rec_idx.p;
            ra.rec_cnt = s->d_rec_cnt.p;
            ra.rec_max = s->d_rec_max.p;
            ra.nvar = s->nvar;
            ra.ti = s->ti->grid.p;
            ra.ti_cells = s->ti->cells;
            ra.complete_prefix = s->ti->missing ? s->ti->complete_prefix.p : nullptr;
            ra.nti = 1;
            ra.ti_id = 0;
            ra.state = (teacher || audit) ? nullptr : s->d_state.p;
            ra.id_image = (teacher || audit) ? nullptr : s->d_id.p;
            ra.node_cell = audit ? nullptr : s->d_node_cell.p;
            if (audit) {
                ra.out_val = s->d_audit_val.p + (size_t)step.off * s->K;
                ra.out_pos = s->d_audit_pos.p + (size_t)step.off * s->K;
            }
            ra.full = s->full ? 1 : 0;
            ra.mt_state = s->d_mt_state.p + p * mt_words;
            ra.mt_pre = s->d_mt_pre.p + size_t(p) * s->max_slots;
            CK(cudaStreamWaitEvent(ws, s->ev_ready[p], 0));
            if (step.kind == STEP_HASH) {
                ra.drawn_score = s->d_drawn_score.p;
                ra.drawn_scale = s->d_drawn_scale.p;
                CK(launch_hash_select(ra, ws));
                ra.only_flagged = 1;
                s->info.launches += 1;
            }
            CK(launch_replay(ra, ws));
            CK(cudaEventRecord(s->ev_used[p], ws));
            if (s->profiling) CK(cudaEventRecord(prof_event(s), ws));
            if (side) {
                CK(cudaEventRecord(s->ev_side, s->st2));
                side_pending = true;
            }
        }
    }
    if (side_pending) CK(cudaStreamWaitEvent(s->st, s->ev_side, 0));
    return QSK_OK;
}

// ---------------------------------------------------------------------------
// tensor-core form
// ---------------------------------------------------------------------------
cudaEvent_t tc_event(qsk_sim *s) {
    if (s->tc_ev_used == s->tc_ev.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        s->tc_ev.push_back(e);
    }
    return s->tc_ev[s->tc_ev_used++];
}

long long rup(long long x, long long m) { return (x + m - 1) / m * m; }

// the encoder stencil's lookup: entry e (template offset e + 1, e < 64) at
// its offset in the bounding box of those offsets, -1 elsewhere
int stencil_cube(qsk_sim *s) {
    const int nd = s->ti->g.nd;
    const int E = std::min(QSK_ENC_ENTRIES, s->ntpl - 1);
    int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (int t = 1; t <= E; ++t)
        for (int d = 0; d < nd; ++d) {
            lo[d] = std::min(lo[d], s->tpl[size_t(t * nd + d)]);
            hi[d] = std::max(hi[d], s->tpl[size_t(t * nd + d)]);
        }
    size_t n = 1;
    for (int d = 0; d < 3; ++d) {
        s->cube_lo[d] = d < nd ? lo[d] : 0;
        s->cube_dim[d] = d < nd ? hi[d] - lo[d] + 1 : 1;
        n *= size_t(s->cube_dim[d]);
    }
    std::vector<int> cube(n, -1);
    for (int t = 1; t <= E; ++t) {
        size_t idx = 0, st = 1;
        for (int d = 0; d < nd; ++d) {
            idx += size_t(s->tpl[size_t(t * nd + d)] - s->cube_lo[d]) * st;
            st *= size_t(s->cube_dim[d]);
        }
        cube[idx] = t - 1;
    }
    CK(s->d_ent_cube.upload(cube.data(), cube.size(), s->st));
    CK(cudaStreamSynchronize(s->st));   // the host vector goes out of scope
    return QSK_OK;
}

void feat_stencil(const qsk_sim *s, const qsk_encoder *e, FeatArgs &fa) {
    fa.cube = s->d_ent_cube.p;
    for (int d = 0; d < 3; ++d) {
        fa.cube_lo[d] = s->cube_lo[d];
        fa.cube_dim[d] = s->cube_dim[d];
    }
    fa.nscales = e->nscales;
    fa.cov_min = e->cov_min;
}

// the stencil scale (encoder e's) of each of `rows` nodes (device list) into scale_out
int node_scales(qsk_sim *s, const qsk_encoder *e, const int *nodes, long long rows, int *scale_out) {
    if (!s->d_ent_cube.p) {
        int rc = stencil_cube(s);
        if (rc) return rc;
    }
    FeatArgs fa;
    fa.rows = rows;
    fa.nodes = nodes;
    fa.path = s->d_path.p;
    fa.begin = s->begin;
    fa.nb_count = s->d_nb_count.p;
    fa.nb_tpl = s->d_nb_tpl.p;
    fa.nb_cell = s->d_nb_cell.p;
    fa.n = s->n;
    fa.tpl = s->d_tpl.p;
    fa.nd = s->ti->g.nd;
    fa.nvar = s->nvar;
    fa.ntpl = s->ntpl;
    fa.entries = QSK_ENC_ENTRIES;
    feat_stencil(s, e, fa);
    fa.scale_out = scale_out;
    CK(launch_node_scale(fa, s->st));
    return QSK_OK;
}

// pattern matrix of the template prefix (built once per simulation and mode)
// learned proposal: the pattern matrices are the TI cells' embeddings (BF16,
// 64 columns), one per stencil scale, built once per encoder state
int tc_configure_learned(qsk_sim *s) {
    const Geom &g = s->ti->g;
    qsk_encoder *e = s->enc;
    const long long rows = rup(g.N, 256);
    s->tc_T = 0;
    s->tc_L = 1;
    s->tc_W = s->lopt.width > 0 ? s->lopt.width : 32;
    s->tc_S = s->lopt.shortlist > 0 ? s->lopt.shortlist : 256;
    if (s->tc_S < s->K) s->tc_S = s->K;
    s->tc_fmt = 0;
    s->tc_Kp = ENC_E;
    s->tc_rows = rows;
    if (s->tc_ready && s->enc_built == e->t && s->enc_ns == e->nscales) return QSK_OK;
    s->tc_ready = false;
    int rc = stencil_cube(s);
    if (rc) return rc;
    const size_t per_scale = size_t(rows) * ENC_E * 2;
    CK(s->d_tc_P.ensure(per_scale * size_t(e->nscales)));
    CK(cudaMemsetAsync(s->d_tc_P.p, 0, per_scale * size_t(e->nscales), s->st));
    const long long chunk = 131072;
    CK(s->d_feat.ensure(size_t(chunk) * size_t(e->D0)));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, s->st));
    for (int sc = 1; sc <= e->nscales; ++sc) {
        uint16_t *P = reinterpret_cast<uint16_t *>(s->d_tc_P.p + per_scale * size_t(sc - 1));
        for (long long c0 = 0; c0 < s->ti->cells; c0 += chunk) {
            const long long n = std::min(chunk, s->ti->cells - c0);
            FeatArgs fa;
            fa.rows = n;
            fa.cell0 = c0;
            fa.cells = s->ti->cells;
            fa.ti = s->ti->grid.p;
            for (int d = 0; d < 3; ++d) fa.src[d] = d < g.nd ? g.src[d] : 1;
            fa.ntpl = s->ntpl;
            fa.tpl = s->d_tpl.p;
            fa.nd = g.nd;
            fa.nvar = s->nvar;
            fa.inv_radius = 0.125f;
            fa.entries = QSK_ENC_ENTRIES;
            fa.scale = sc;
            fa.out = s->d_feat.p;
            CK(launch_feat_cells(fa, s->st));
            rc = enc_forward(e, n, 0, s->d_feat.p, s->st);   // TI-pattern head
            if (rc) return rc;
            CK(launch_to_bf16(n * ENC_E, e->y.p, P + size_t(c0) * ENC_E, s->st));
        }
    }
    CK(cudaEventRecord(e1, s->st));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    s->info.ms_tensor_pattern = ms;
    if ((rc = enc_check(e, s->st)) != QSK_OK) return rc;
    s->enc_built = e->t;
    s->enc_ns = e->nscales;
    s->tc_ready = true;
    return QSK_OK;
}

int tc_configure(qsk_sim *s, int T_auto) {
    if (s->topt.mode == 3) return tc_configure_learned(s);
    const Geom &g = s->ti->g;
    const int fmt = s->topt.mode == 2 ? 1 : 0;
    const int elem = fmt == 0 ? 2 : 1;
    // layers: t^2, t per continuous variable; one indicator per category
    std::vector<TcLayer> layers;
    s->var_layer0.assign(s->nvar, 0);
    for (int v = 0; v < s->nvar; ++v) {
        s->var_layer0[v] = int(layers.size());
        if (s->ti->types[v] == 0) {
            layers.push_back({v, 0, 0.f});
            layers.push_back({v, 1, 0.f});
        } else {
            for (int c = 0; c + 1 < s->ti->cat_n[v]; ++c)
                layers.push_back({v, 2, s->ti->cat_v[size_t(v) * QSK_CMAX + c]});
        }
    }
    if (layers.empty() || layers.size() > QSK_TC_MAXL)
        return fail(QSK_ERR_UNSUPPORTED, "tensor-core form: %zu pattern layers (1..%d)", layers.size(), QSK_TC_MAXL);
    const int L = int(layers.size());
    const long long rows = rup(g.N, 256);
    int T = s->topt.prefix > 0 ? s->topt.prefix : T_auto;
    T = std::max(1, std::min(T, s->ntpl));
    // cap the pattern matrix at 48 GiB (a quarter of the B200's HBM)
    while (T > 64 && (double)rows * rup((long long)T * L, 128 / elem) * elem > 48.0 * (1ull << 30)) T = T / 2 / 64 * 64;
    const long long Kp = rup((long long)T * L, 128 / elem);
    const int W = s->topt.width > 0 ? s->topt.width : (fmt == 1 ? 32 : 8);
    int S = s->topt.shortlist > 0 ? s->topt.shortlist : (fmt == 1 ? 128 : 4 * s->K);
    if (!tc_supported_width(W)) return fail(QSK_ERR_ARG, "tensor-core width %d (8, 16 or 32)", W);
    if (S > 128) return fail(QSK_ERR_ARG, "tensor-core shortlist %d (at most 128)", S);
    if (S < s->K) S = s->K;
    const bool same = s->tc_ready && s->tc_T == T && s->tc_fmt == fmt && s->tc_L == L;
    s->tc_T = T;
    s->tc_L = L;
    s->tc_W = W;
    s->tc_S = S;
    s->tc_fmt = fmt;
    s->tc_Kp = Kp;
    s->tc_rows = rows;
    if (same) return QSK_OK;
    s->tc_ready = false;
    // every element is written by the pattern kernel: a large enough buffer
    // (a job runner's scratch included) is reused as it is
    CK(s->d_tc_P.ensure(size_t(rows * Kp * elem)));
    CK(s->d_tc_pscale.ensure(size_t(rows / 256)));
    DBuf<float> rowmax;
    if (fmt == 1) CK(rowmax.alloc(size_t(rows)));
    TcPatternArgs pa{};
    pa.ti = s->ti->grid.p;
    pa.nvar = s->nvar;
    pa.nd = g.nd;
    for (int d = 0; d < QSK_MAXD; ++d) pa.src[d] = d < g.nd ? g.src[d] : 1;
    pa.N = s->ti->cells;
    pa.rows = rows;
    pa.tpl = s->d_tpl.p;
    pa.T = T;
    pa.L = L;
    for (int l = 0; l < L; ++l) pa.layer[l] = layers[size_t(l)];
    pa.Kp = Kp;
    pa.fmt = fmt;
    pa.P = s->d_tc_P.p;
    pa.pos_scale = s->d_tc_pscale.p;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, s->st));
    CK(launch_tc_pattern(pa, rowmax.p, s->st));
    CK(cudaEventRecord(e1, s->st));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    s->info.ms_tensor_pattern = ms;
    std::vector<int> ncat(s->nvar, 0);
    for (int v = 0; v < s->nvar; ++v) ncat[v] = s->ti->types[v] == 1 ? s->ti->cat_n[v] : 0;
    CK(s->d_var_layer0.upload(s->var_layer0.data(), s->var_layer0.size(), s->st));
    CK(s->d_var_ncat.upload(ncat.data(), ncat.size(), s->st));
    CK(s->d_var_catv.upload(s->ti->cat_v.data(), s->ti->cat_v.size(), s->st));
    s->tc_ready = true;
    return QSK_OK;
}

// Tensor steps of a run: every level's nodes whose neighbours all lie in the
// template prefix (sorted by their largest template index, so that a tile of
// 128 nodes needs few K blocks) take the tensor-core form, the rest the plain
// path.  Rewrites the level node list in that order.
// largest template index of every path node (-1: no neighbour but the centre)
int tc_tmax(qsk_sim *s, std::vector<int> &tmax) {
    const long long nodes = s->nodes;
    CK(s->d_tc_tmax.ensure(size_t(std::max<long long>(nodes, 1))));
    CK(launch_tc_tmax(nodes, s->n, s->d_nb_count.p, s->d_nb_tpl.p, s->d_tc_tmax.p, s->st));
    tmax.resize((size_t)nodes);
    CK(cudaMemcpyAsync(tmax.data(), s->d_tc_tmax.p, sizeof(int) * nodes, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return QSK_OK;
}

// Automatic template prefix: the smallest multiple of 256 offsets that
// covers 97 % of the nodes with neighbours (the rest take the exact map with
// the same hash tie rule).
// The prefix sets the K of the GEMM for the nodes near it; the sorted nodes
// of a level keep most 128-node tiles far below it.
int tc_auto_prefix(const std::vector<int> &tmax) {
    std::vector<int> v;
    v.reserve(tmax.size());
    for (int t : tmax)
        if (t >= 0) v.push_back(t);
    if (v.empty()) return 256;
    const size_t q = std::min(v.size() - 1, size_t(double(v.size()) * 0.97));
    std::nth_element(v.begin(), v.begin() + long(q), v.end());
    return int((v[q] + 1 + 255) / 256 * 256);
}

int tc_plan(qsk_sim *s, const std::vector<int> &start, const std::vector<int> &tmax, std::vector<Step> &steps,
            std::vector<int> &audit_nodes) {
    const long long nodes = s->nodes;
    std::vector<int> order((size_t)nodes);
    CK(cudaMemcpyAsync(order.data(), s->d_level_nodes.p, sizeof(int) * nodes, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    const int kbe = s->tc_fmt == 0 ? 64 : 128;
    const int T = s->tc_T, L = s->tc_L;
    std::vector<int> kb;   // K blocks of every 128-node tile of every tensor step
    steps.clear();
    audit_nodes.clear();
    long long ntc = 0, npl = 0;
    double flops = 0.0;
    const long long ntiles_pos = s->tc_rows / 256;
    const unsigned athr = s->topt.audit >= 1.f ? 0xFFFFFFFFu : unsigned(double(s->topt.audit) * 4294967296.0);
    const bool learned = s->topt.mode == 3;
    // learned proposal: every node's stencil scale (per position of the level order)
    std::vector<int> lscale;
    if (learned && !start.empty() && start.back() > 0) {
        const long long tot = start.back();
        CK(s->d_lscale.ensure(size_t(tot)));
        int rc = node_scales(s, s->enc, s->d_level_nodes.p, tot, s->d_lscale.p);
        if (rc) return rc;
        lscale.resize(size_t(tot));
        CK(cudaMemcpyAsync(lscale.data(), s->d_lscale.p, sizeof(int) * size_t(tot), cudaMemcpyDeviceToHost, s->st));
        CK(cudaStreamSynchronize(s->st));
    }
    std::vector<int> el, pl, esc, idx;
    for (size_t l = 0; l + 1 < start.size(); ++l) {
        el.clear();
        pl.clear();
        esc.clear();
        for (int q = start[l]; q < start[l + 1]; ++q) {
            const int i = order[size_t(q)];
            const bool tc = tmax[size_t(i)] >= 0 && (learned || tmax[size_t(i)] < T);
            (tc ? el : pl).push_back(i);
            if (tc && learned) esc.push_back(lscale[size_t(q)]);
        }
        if (learned) {
            // one stencil scale per step: the level's nodes grouped by scale
            idx.resize(el.size());
            for (size_t j = 0; j < idx.size(); ++j) idx[j] = int(j);
            std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return esc[size_t(a)] < esc[size_t(b)]; });
            std::vector<int> e2(el.size()), s2(el.size());
            for (size_t j = 0; j < idx.size(); ++j) {
                e2[j] = el[size_t(idx[j])];
                s2[j] = esc[size_t(idx[j])];
            }
            el.swap(e2);
            esc.swap(s2);
        } else {
            std::stable_sort(el.begin(), el.end(), [&](int a, int b) { return tmax[size_t(a)] < tmax[size_t(b)]; });
        }
        int q = start[l];
        for (int i : el) order[size_t(q++)] = i;
        for (int i : pl) order[size_t(q++)] = i;
        for (int g0 = 0; g0 < int(el.size());) {
            int g1 = int(el.size());
            if (learned) {
                g1 = g0 + 1;
                while (g1 < int(el.size()) && esc[size_t(g1)] == esc[size_t(g0)]) ++g1;
            }
            for (int off = g0; off < g1; off += s->max_tc_slots) {
                const int B = std::min(s->max_tc_slots, g1 - off);
                Step st{STEP_TENSOR, s->d_level_nodes.p, start[l] + off, B, int(kb.size())};
                st.scale = learned ? esc[size_t(off)] : 1;
                st.level = int(l);
                for (int t0 = 0; t0 < B; t0 += 128) {
                    const int last = el[size_t(off + std::min(B, t0 + 128) - 1)];
                    const int k = learned ? 1 : int((((long long)tmax[size_t(last)] + 1) * L + kbe - 1) / kbe);
                    kb.push_back(k);
                    flops += 2.0 * 128 * 256 * double(ntiles_pos) * double(k) * kbe;
                }
                steps.push_back(st);
            }
            g0 = g1;
        }
        for (int off = 0; off < int(pl.size()); off += s->max_slots) {
            Step st{STEP_HASH, s->d_level_nodes.p, start[l] + int(el.size()) + off,
                    std::min(s->max_slots, int(pl.size()) - off), 0};
            // the learned proposal's fallback uses the exact map's buffers
            // inside its tensor steps: its levels stay on one stream
            st.level = learned ? -1 : int(l);
            steps.push_back(st);
        }
        ntc += (long long)el.size();
        npl += (long long)pl.size();
        if (athr) {
            for (int i : el)
                if (tie_hash(0xA5D17u, unsigned(i)) < athr || s->topt.audit >= 1.f) audit_nodes.push_back(i);
            // the exact map's nodes with neighbours (marginal draws have no k best)
            for (int i : pl)
                if (tmax[size_t(i)] >= 0 && (tie_hash(0xA5D17u, unsigned(i)) < athr || s->topt.audit >= 1.f))
                    audit_nodes.push_back(i);
        }
    }
    CK(cudaMemcpyAsync(s->d_level_nodes.p, order.data(), sizeof(int) * nodes, cudaMemcpyHostToDevice, s->st));
    if (kb.empty()) kb.push_back(0);   // no tensor step: a valid (unused) upload
    CK(s->d_tc_kb.upload(kb.data(), kb.size(), s->st));
    CK(cudaStreamSynchronize(s->st));   // host vectors go out of scope
    s->info.tensor_nodes = ntc;
    s->info.plain_nodes = npl;
    s->info.tensor_flops = flops;
    return QSK_OK;
}

// the exact map over the whole TI (FP32 gather) with the tensor-core form's
// draw rule, for a device list of path nodes (the learned proposal's
// fallback); records must hold max_slots slots
int exact_nodes(qsk_sim *s, const int *nodes, int count, bool teacher) {
    const Geom &g = s->ti->g;
    for (int off = 0; off < count; off += s->max_slots) {
        const int B = std::min(s->max_slots, count - off);
        SimPrepArgs pa;
        pa.g = g;
        pa.dg = s->dg;
        pa.nvar = s->nvar;
        pa.types = s->d_types.p;
        pa.tpl = s->d_tpl.p;
        pa.wtab = s->d_wtab.p;
        pa.path = s->d_path.p;
        pa.begin = s->begin;
        pa.seeds = s->d_seeds.p;
        pa.nb_count = s->d_nb_count.p;
        pa.nb_tpl = s->d_nb_tpl.p;
        pa.nb_cell = s->d_nb_cell.p;
        pa.n = s->n;
        pa.state = s->d_state.p;
        pa.init = s->d_init.p;
        pa.nodes = nodes + off;
        pa.nslots = B;
        pa.k = s->k;
        pa.K = s->K;
        pa.nti = 1;
        pa.slots = s->d_slots.p;
        pa.terms = s->d_terms.p;
        pa.maxterms = s->maxterms;
        pa.status = s->d_status.p;
        pa.missing = 0;
        pa.mask_layer = s->nvar;
        pa.no_verbatim = 0;
        pa.id_image = s->d_id.p;
        pa.node_nv = nullptr;
        pa.node_k = nullptr;
        pa.full = 0;
        pa.nb_mask = nullptr;
        if (s->profiling) CK(cudaEventRecord(prof_event(s), s->st));
        CK(launch_prep_sim(pa, s->st));
        if (s->profiling) CK(cudaEventRecord(prof_event(s), s->st));
        MapArgs ma;
        ma.g = g;
        ma.layers = s->ti->layers.p;
        ma.slots = s->d_slots.p;
        ma.terms = s->d_terms.p;
        ma.maxterms = s->maxterms;
        ma.segs_per_cta = map_segs_per_cta(g, B);
        ma.rec_val = s->d_rec_val.p;
        ma.rec_idx = s->d_rec_idx.p;
        ma.rec_cnt = s->d_rec_cnt.p;
        ma.rec_max = s->d_rec_max.p;
        CK(launch_map_records(ma, B, s->K, s->maxterms, s->st));
        if (s->profiling) CK(cudaEventRecord(prof_event(s), s->st));
        ReplayArgs ra;
        std::memset(&ra, 0, sizeof(ra));
        ra.g = g;
        ra.slots = s->d_slots.p;
        ra.nslots = B;
        ra.K = s->K;
        ra.rec_val = s->d_rec_val.p;
        ra.rec_idx = s->d_rec_idx.p;
        ra.rec_cnt = s->d_rec_cnt.p;
        ra.rec_max = s->d_rec_max.p;
        ra.nvar = s->nvar;
        ra.ti = s->ti->grid.p;
        ra.ti_cells = s->ti->cells;
        ra.nti = 1;
        ra.state = teacher ? nullptr : s->d_state.p;
        ra.id_image = teacher ? nullptr : s->d_id.p;
        ra.node_cell = s->d_node_cell.p;
        ra.drawn_score = s->d_drawn_score.p;
        ra.drawn_scale = s->d_drawn_scale.p;
        CK(launch_hash_select(ra, s->st));
        ra.only_flagged = 1;
        CK(launch_replay(ra, s->st));
        if (s->profiling) CK(cudaEventRecord(prof_event(s), s->st));
        s->info.launches += 4;
        s->info.map_launches += 1;
        s->info.map_positions += (long long)B * g.N;
    }
    return QSK_OK;
}

int tc_step(qsk_sim *s, const Step &step, bool teacher) {
    const Geom &g = s->ti->g;
    const int B = step.B;
    const int elem = s->tc_fmt == 0 ? 2 : 1;
    const long long Bp = rup(B, 128);
    if (s->profiling) CK(cudaEventRecord(tc_event(s), s->st));
    // exact terms and slot geometry (the plain path's prep)
    SimPrepArgs pa;
    pa.g = g;
    pa.dg = s->dg;
    pa.nvar = s->nvar;
    pa.types = s->d_types.p;
    pa.tpl = s->d_tpl.p;
    pa.wtab = s->d_wtab.p;
    pa.path = s->d_path.p;
    pa.begin = s->begin;
    pa.seeds = s->d_seeds.p;
    pa.nb_count = s->d_nb_count.p;
    pa.nb_tpl = s->d_nb_tpl.p;
    pa.nb_cell = s->d_nb_cell.p;
    pa.n = s->n;
    pa.state = s->d_state.p;
    pa.init = s->d_init.p;
    pa.nodes = step.nodes + step.off;
    pa.nslots = B;
    pa.k = s->k;
    pa.K = s->K;
    pa.nti = 1;
    pa.slots = s->d_tc_slots.p;
    pa.terms = s->d_tc_terms.p;
    pa.maxterms = s->maxterms;
    pa.status = s->d_status.p;
    pa.missing = 0;
    pa.mask_layer = s->nvar;
    pa.no_verbatim = 0;
    pa.id_image = s->d_id.p;
    pa.node_nv = nullptr;
    pa.node_k = nullptr;
    pa.full = 0;
    pa.nb_mask = nullptr;
    const bool learned = s->topt.mode == 3;
    if (learned) {
        CK(launch_prep_sim(pa, s->st));
        // node rows of A: the encoder's embeddings of the nodes' neighbourhoods
        qsk_encoder *e = s->enc;
        FeatArgs fa;
        fa.rows = B;
        fa.nodes = step.nodes + step.off;
        fa.path = s->d_path.p;
        fa.begin = s->begin;
        fa.nb_count = s->d_nb_count.p;
        fa.nb_tpl = s->d_nb_tpl.p;
        fa.nb_cell = s->d_nb_cell.p;
        fa.n = s->n;
        fa.state = s->d_state.p;
        fa.tpl = s->d_tpl.p;
        fa.nd = g.nd;
        fa.nvar = s->nvar;
        fa.inv_radius = 0.125f;
        fa.ntpl = s->ntpl;
        fa.entries = QSK_ENC_ENTRIES;
        feat_stencil(s, e, fa);
        fa.scale = step.scale;
        fa.out = s->d_feat.p;
        CK(launch_feat_nodes(fa, s->st));
        int rc = enc_forward(e, B, B, s->d_feat.p, s->st);   // query head
        if (rc) return rc;
        CK(launch_to_bf16((long long)B * ENC_E, e->y.p, reinterpret_cast<uint16_t *>(s->d_tc_A.p), s->st));
    }
    TcNodeArgs na{};
    na.nd = g.nd;
    na.nvar = s->nvar;
    for (int d = 0; d < QSK_MAXD; ++d) na.src[d] = d < g.nd ? g.src[d] : 1;
    na.nodes = step.nodes + step.off;
    na.nslots = B;
    na.path = s->d_path.p;
    na.begin = s->begin;
    na.nb_count = s->d_nb_count.p;
    na.nb_tpl = s->d_nb_tpl.p;
    na.nb_cell = s->d_nb_cell.p;
    na.n = s->n;
    na.tpl = s->d_tpl.p;
    na.wtab = s->d_wtab.p;
    na.state = s->d_state.p;
    na.init = s->d_init.p;
    na.seeds = s->d_seeds.p;
    na.types = s->d_types.p;
    na.var_layer0 = s->d_var_layer0.p;
    na.var_ncat = s->d_var_ncat.p;
    na.var_catv = s->d_var_catv.p;
    na.L = s->tc_L;
    na.Kp = s->tc_Kp;
    na.fmt = s->tc_fmt;
    na.A = learned ? nullptr : s->d_tc_A.p;   // rows zeroed by the kernel
    na.rows = Bp;
    na.node_thr = s->d_tc_thr.p;
    na.node_scale = s->d_tc_nscale.p;
    na.node_bias = s->d_tc_bias.p;
    na.node_box = s->d_tc_box.p;
    na.node_seed = s->d_tc_seed.p;
    // the exact terms and the node rows in one launch (learned: the rows of
    // A come from the encoder, after the terms)
    if (learned) CK(launch_tc_nodes(na, s->st));
    else CK(launch_prep_tc_nodes(pa, na, s->st));
    if (s->profiling) CK(cudaEventRecord(tc_event(s), s->st));
    // GEMM shortlist: enough position ranges to fill the GPU, at most
    // SEL_CAND / W candidates per node.  With a shortlist of at most W the
    // shared bound makes the ranges' union hold the exact overall top W for
    // any number of ranges: one wave of CTAs (one per SM), each scanning
    // more position tiles, saves a second wave's set-up (TMEM allocation,
    // pipeline fill) on the short levels.  A longer shortlist keeps two
    // waves' worth of ranges, whose heaps it is drawn from.
    if (s->sm_count <= 0) {
        int sms = 0;
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device));
        s->sm_count = std::max(1, sms);
    }
    const int node_tiles = int(Bp / 128);
    const long long ntiles = s->tc_rows / 256;
    const long long sms = s->sm_count;
    int ranges = int(s->tc_S <= s->tc_W ? std::max<long long>(1, sms / node_tiles)
                                        : std::max<long long>(1, (2 * sms + node_tiles - 1) / node_tiles));
    ranges = int(std::min<long long>({(long long)ranges, ntiles, 768LL / s->tc_W}));
    TcArgs a{};
    a.n_nodes = B;
    a.n_pos = s->ti->cells;
    a.n_tiles = ntiles;
    a.ranges = ranges;
    a.tiles_per_range = int((ntiles + ranges - 1) / ranges);
    a.ranges = int((ntiles + a.tiles_per_range - 1) / a.tiles_per_range);
    a.kblocks = int(s->tc_Kp * elem / 128);
    a.tile_kblocks = s->d_tc_kb.p + step.kb_off;
    a.node_scale = s->tc_fmt == 1 ? s->d_tc_nscale.p : nullptr;
    a.node_bias = s->d_tc_bias.p;
    a.pos_scale = s->tc_fmt == 1 ? s->d_tc_pscale.p : nullptr;
    a.node_seed = s->d_tc_seed.p;
    a.node_box = s->d_tc_box.p;
    a.X = g.src[0];
    a.Y = g.nd > 1 ? g.src[1] : 1;
    // a shared bound across ranges keeps the overall top W in the union of the
    // ranges' heaps: enough when the shortlist takes at most W of them
    a.node_thr = s->tc_S <= s->tc_W ? s->d_tc_thr.p : nullptr;
    a.out_key = s->d_tc_key.p;
    a.out_pos = s->d_tc_pos.p;
    a.status = s->d_status.p;
    // learned proposal: the pattern matrix of the step's stencil scale
    const unsigned char *P = s->d_tc_P.p + (learned ? size_t(step.scale - 1) * size_t(s->tc_rows) * ENC_E * 2 : 0);
    CK(launch_tc_shortlist(s->tc_fmt, s->tc_W, s->d_tc_A.p, Bp, P, s->tc_rows, s->tc_Kp, a, s->st));
    if (s->profiling) CK(cudaEventRecord(tc_event(s), s->st));
    TcSelectArgs sa{};
    sa.g = g;
    sa.slots = s->d_tc_slots.p;
    sa.terms = s->d_tc_terms.p;
    sa.maxterms = s->maxterms;
    sa.nslots = B;
    sa.layers = s->ti->layers.p;
    sa.cand_key = s->d_tc_key.p;
    sa.cand_pos = s->d_tc_pos.p;
    sa.ncand = a.ranges * s->tc_W;
    sa.S = s->tc_S;
    sa.fp64 = s->tc_fmt == 1 ? 1 : 0;
    sa.ti = s->ti->grid.p;
    sa.nvar = s->nvar;
    sa.nti = 1;
    sa.ti_id = 0;
    sa.state = teacher ? nullptr : s->d_state.p;
    sa.id_image = teacher ? nullptr : s->d_id.p;
    sa.node_cell = s->d_node_cell.p;
    sa.drawn_score = s->d_drawn_score.p;
    sa.drawn_scale = s->d_drawn_scale.p;
    sa.err_max = s->d_err_max.p;
    sa.err_sum = s->d_err_sum.p;
    sa.err_n = s->d_err_n.p;
    sa.status = s->d_status.p;
    if (learned) {
        sa.fallback = s->d_fb.p;
        sa.conf_rank = s->lopt.conf_rank > 0 ? s->lopt.conf_rank : 1;
        sa.conf_z = s->lopt.conf_z;
        sa.conf_r2 = s->lopt.conf_r2 > 0.f ? s->lopt.conf_r2 : 0.2f;
        sa.range_w = s->tc_W;
    }
    CK(launch_tc_select(sa, s->st));
    if (s->profiling) CK(cudaEventRecord(tc_event(s), s->st));
    s->info.launches += learned ? 4 : 3;
    s->info.tensor_launches += learned ? 4 : 3;
    if (learned) {
        // nodes whose confidence check failed: the exact map, in the same level
        std::vector<int> fb((size_t)B), nd((size_t)B);
        CK(cudaMemcpyAsync(fb.data(), s->d_fb.p, sizeof(int) * B, cudaMemcpyDeviceToHost, s->st));
        CK(cudaMemcpyAsync(nd.data(), step.nodes + step.off, sizeof(int) * B, cudaMemcpyDeviceToHost, s->st));
        if (int rc = enc_check(s->enc, s->st)) return rc;
        std::vector<int> list;
        for (int q = 0; q < B; ++q)
            if (fb[size_t(q)]) list.push_back(nd[size_t(q)]);
        s->info.learned_fallback += (long long)list.size();
        if (!list.empty()) {
            CK(s->d_fb_nodes.ensure(list.size()));
            CK(cudaMemcpyAsync(s->d_fb_nodes.p, list.data(), sizeof(int) * list.size(), cudaMemcpyHostToDevice, s->st));
            int rc = exact_nodes(s, s->d_fb_nodes.p, int(list.size()), teacher);
            if (rc) return rc;
            CK(cudaStreamSynchronize(s->st));   // the host list goes out of scope
        }
    }
    return QSK_OK;
}

// buffers of the tensor steps (sized for max_tc_slots) and the statistics
int tc_buffers(qsk_sim *s, size_t n_audit) {
    const int elem = s->tc_fmt == 0 ? 2 : 1;
    const size_t slots = size_t(s->max_tc_slots), bp = size_t(rup(s->max_tc_slots, 128));
    CK(s->d_tc_A.ensure(bp * size_t(s->tc_Kp) * elem));
    CK(s->d_tc_nscale.ensure(bp));
    CK(s->d_tc_bias.ensure(bp));
    CK(s->d_tc_box.ensure(bp * 6));
    CK(s->d_tc_seed.ensure(bp));
    CK(s->d_tc_thr.ensure(bp));
    CK(s->d_tc_key.ensure(slots * 768));
    CK(s->d_tc_pos.ensure(slots * 768));
    CK(s->d_tc_slots.ensure(slots));
    CK(s->d_tc_terms.ensure(slots * size_t(s->maxterms)));
    CK(s->d_drawn_score.ensure(size_t(std::max<long long>(s->nodes, 1))));
    CK(s->d_drawn_scale.ensure(size_t(std::max<long long>(s->nodes, 1))));
    CK(s->d_err_max.ensure(1));
    CK(s->d_err_sum.ensure(1));
    CK(s->d_err_n.ensure(1));
    CK(s->d_tc_counts.ensure(3));
    if (s->topt.mode == 3) {
        CK(s->d_feat.ensure(bp * size_t(s->enc->D0)));
        CK(s->d_fb.ensure(bp));
    }
    CK(cudaMemsetAsync(s->d_err_max.p, 0, sizeof(unsigned), s->st));
    CK(cudaMemsetAsync(s->d_err_sum.p, 0, sizeof(double), s->st));
    CK(cudaMemsetAsync(s->d_err_n.p, 0, sizeof(unsigned long long), s->st));
    CK(cudaMemsetAsync(s->d_tc_counts.p, 0, 3 * sizeof(unsigned long long), s->st));
    if (n_audit) {
        CK(s->d_audit_nodes.ensure(n_audit));
        CK(s->d_audit_val.ensure(n_audit * size_t(s->K)));
        CK(s->d_audit_pos.ensure(n_audit * size_t(s->K)));
    }
    return QSK_OK;
}

int sim_records(qsk_sim *s, long long slots);

// tensor-core run: plan, steps, audit, statistics.  `start`: level bounds of
// the level node list (one level under teacher forcing)
int tc_run(qsk_sim *s, const std::vector<int> &start, bool teacher) {
    std::vector<int> tmax;
    int rc = tc_tmax(s, tmax);
    if (rc) return rc;
    if (s->tc_T_auto == 0) s->tc_T_auto = tc_auto_prefix(tmax);
    if ((rc = tc_configure(s, s->tc_T_auto)) != QSK_OK) return rc;
    std::vector<Step> steps;
    std::vector<int> audit;
    if ((rc = tc_plan(s, start, tmax, steps, audit)) != QSK_OK) return rc;
    if ((rc = tc_buffers(s, audit.size())) != QSK_OK) return rc;
    int mb = 1;
    for (const Step &st : steps)
        if (st.kind == STEP_PLAIN || st.kind == STEP_HASH) mb = std::max(mb, st.B);
    if (!audit.empty()) mb = std::max(mb, std::min<int>(int(audit.size()), s->max_slots));
    if (s->topt.mode == 3) mb = s->max_slots;   // fallback batches of up to max_slots
    s->info.learned_fallback = 0;
    if ((rc = sim_records(s, mb)) != QSK_OK) return rc;
    if ((rc = sim_batches(s, steps, teacher)) != QSK_OK) return rc;
    // audit: the plain path, teacher-forced on the final grid (every node's
    // neighbours hold the values they had at its turn), k best per node
    if (!audit.empty()) {
        CK(cudaMemcpyAsync(s->d_audit_nodes.p, audit.data(), sizeof(int) * audit.size(), cudaMemcpyHostToDevice, s->st));
        std::vector<Step> as;
        for (int off = 0; off < int(audit.size()); off += s->max_slots)
            as.push_back({STEP_AUDIT, s->d_audit_nodes.p, off, std::min(s->max_slots, int(audit.size()) - off), 0});
        const bool prof = s->profiling;
        s->profiling = false;
        const size_t used = s->prof_used, tused = s->tc_ev_used;
        rc = sim_batches(s, as, true);
        s->prof_used = used;
        s->tc_ev_used = tused;
        s->profiling = prof;
        if (rc) return rc;
        CK(launch_tc_audit(int(audit.size()), s->d_audit_nodes.p, s->K, s->d_audit_val.p, s->d_drawn_score.p,
                           s->d_drawn_scale.p, 1e-5f, s->d_tc_counts.p, s->st));
    }
    unsigned long long counts[3] = {0, 0, 0}, en = 0;
    unsigned emax = 0;
    double esum = 0.0;
    CK(cudaMemcpyAsync(counts, s->d_tc_counts.p, sizeof(counts), cudaMemcpyDeviceToHost, s->st));
    CK(cudaMemcpyAsync(&emax, s->d_err_max.p, sizeof(unsigned), cudaMemcpyDeviceToHost, s->st));
    CK(cudaMemcpyAsync(&esum, s->d_err_sum.p, sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(cudaMemcpyAsync(&en, s->d_err_n.p, sizeof(en), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    s->info.tensor_mode = s->topt.mode;
    s->info.tensor_prefix = s->tc_T;
    s->info.tensor_width = s->tc_W;
    s->info.tensor_shortlist = s->tc_S;
    s->info.audited = (long long)counts[0];
    s->info.regret = (long long)counts[1];
    s->info.regret_near = (long long)counts[2];
    float fm;
    std::memcpy(&fm, &emax, sizeof(float));
    s->info.map_err_max = fm;
    s->info.map_err_mean = en ? float(esum / double(en)) : 0.f;
    return QSK_OK;
}

// several training images (the plain path): per batch and TI the exact map
// and the reservoir k best with the same seed (quantileSamplingModule.hpp:
// 455-575), each TI's K best kept as TI cells, then one merge and draw over
// the TIs (k_multi_draw); levels in order on s->st
int sim_batches_multi(qsk_sim *s, const std::vector<Step> &steps) {
    const std::vector<qsk_ti *> tis = s->all_tis();
    const int nti = int(tis.size());
    const size_t stride = size_t(s->max_slots) * size_t(s->K);
    CK(s->d_mval.ensure(stride * nti));
    CK(s->d_mcell.ensure(stride * nti));
    for (const Step &step : steps) {
        const int B = step.B;
        for (int t = 0; t < nti; ++t) {
            const qsk_ti *T = tis[size_t(t)];
            SimPrepArgs pa;
            std::memset(&pa, 0, sizeof(pa));
            pa.g = T->g;
            pa.dg = s->dg;
            pa.nvar = s->nvar;
            pa.types = s->d_types.p;
            pa.tpl = s->d_tpl.p;
            pa.wtab = s->d_wtab.p;
            pa.path = s->d_path.p;
            pa.begin = s->begin;
            pa.seeds = s->d_seeds.p;
            pa.nb_count = s->d_nb_count.p;
            pa.nb_tpl = s->d_nb_tpl.p;
            pa.nb_cell = s->d_nb_cell.p;
            pa.n = s->n;
            pa.state = s->d_state.p;
            pa.init = s->d_init.p;
            pa.nodes = step.nodes + step.off;
            pa.nslots = B;
            pa.k = s->k;
            pa.K = s->K;
            pa.nti = unsigned(nti);
            pa.slots = s->d_slots.p;
            pa.terms = s->d_terms.p;
            pa.maxterms = s->maxterms;
            pa.status = s->d_status.p;
            pa.mask_layer = s->nvar;
            pa.id_image = s->d_id.p;
            pa.sterms = nullptr;
            CK(launch_prep_sim(pa, s->st));
            MapArgs ma;
            std::memset(&ma, 0, sizeof(ma));
            ma.g = T->g;
            ma.layers = T->layers.p;
            ma.slots = s->d_slots.p;
            ma.terms = s->d_terms.p;
            ma.maxterms = s->maxterms;
            ma.segs_per_cta = map_segs_per_cta(T->g, B);
            ma.rec_val = s->d_rec_val.p;
            ma.rec_idx = s->d_rec_idx.p;
            ma.rec_cnt = s->d_rec_cnt.p;
            ma.rec_max = s->d_rec_max.p;
            CK(launch_map_records(ma, B, s->K, s->maxterms, s->st));
            ReplayArgs ra;
            std::memset(&ra, 0, sizeof(ra));
            ra.g = T->g;
            ra.slots = s->d_slots.p;
            ra.nslots = B;
            ra.K = s->K;
            ra.rec_val = s->d_rec_val.p;
            ra.rec_idx = s->d_rec_idx.p;
            ra.rec_cnt = s->d_rec_cnt.p;
            ra.rec_max = s->d_rec_max.p;
            ra.out_val = s->d_mval.p + stride * size_t(t);
            ra.out_pos = s->d_mcell.p + stride * size_t(t);
            ra.out_cells = 1;
            ra.nvar = s->nvar;
            ra.ti = T->grid.p;
            ra.ti_cells = T->cells;
            ra.nti = unsigned(nti);
            ra.ti_id = unsigned(t);
            CK(launch_replay(ra, s->st));
            s->info.launches += 3;
            s->info.map_launches += 1;
            s->info.map_positions += (long long)B * T->g.N;
        }
        MultiDrawArgs md;
        md.slots = s->d_slots.p;
        md.nslots = B;
        md.K = s->K;
        md.nti = nti;
        md.nvar = s->nvar;
        md.vals = s->d_mval.p;
        md.cells = s->d_mcell.p;
        md.ti_stride = (long long)stride;
        for (int t = 0; t < nti; ++t) {
            md.ti[t] = tis[size_t(t)]->grid.p;
            md.ti_cells[t] = tis[size_t(t)]->cells;
        }
        md.types = s->d_types.p;
        md.nb_count = s->d_nb_count.p;
        md.nb_tpl = s->d_nb_tpl.p;
        md.nb_cell = s->d_nb_cell.p;
        md.n = s->n;
        md.wtab = s->d_wtab.p;
        md.ii = s->d_ii.p;
        md.state = s->d_state.p;
        md.id_image = s->d_id.p;
        md.node_cell = s->d_node_cell.p;
        CK(launch_multi_draw(md, s->st));
        s->info.launches += 1;
    }
    return QSK_OK;
}

// the batch chain of a plain run captured into one CUDA graph (both
// streams: the generator pipeline joins through its events), instantiated
// and launched on s->st; the graph is released once the run has finished
int sim_batches_graph(qsk_sim *s, const std::vector<Step> &steps, cudaGraphExec_t *exec_out) {
    const auto t0 = std::chrono::steady_clock::now();
    CK(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
    int rc = sim_batches(s, steps, false);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s->st, &graph);
    if (rc != QSK_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) return fail(QSK_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    size_t nn = 0;
    cudaError_t e2 = cudaGraphGetNodes(graph, nullptr, &nn);
    if (e2 == cudaSuccess) e2 = cudaGraphInstantiate(exec_out, graph, 0);
    cudaGraphDestroy(graph);
    if (e2 != cudaSuccess) return fail(QSK_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e2));
    s->info.graph_nodes = (long long)nn;
    s->info.ms_graph_build =
        float(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
    CK(cudaGraphLaunch(*exec_out, s->st));
    return QSK_OK;
}

void collect_profile(qsk_sim *s) {
    if (!s->profiling || (s->prof_used == 0 && s->tc_ev_used == 0)) return;
    if (s->prof_used) cudaEventSynchronize(s->prof_ev[s->prof_used - 1]);
    if (s->tc_ev_used) cudaEventSynchronize(s->tc_ev[s->tc_ev_used - 1]);
    float prep = 0, map = 0, rep = 0;
    for (size_t i = 0; i + 3 < s->prof_used; i += 4) {
        float a = 0, b = 0, c = 0;
        cudaEventElapsedTime(&a, s->prof_ev[i], s->prof_ev[i + 1]);
        cudaEventElapsedTime(&b, s->prof_ev[i + 1], s->prof_ev[i + 2]);
        cudaEventElapsedTime(&c, s->prof_ev[i + 2], s->prof_ev[i + 3]);
        prep += a;
        map += b;
        rep += c;
    }
    s->info.ms_prep = prep;
    s->info.ms_map = map;
    s->info.ms_replay = rep;
    float gemm = 0, sel = 0;
    for (size_t i = 0; i + 3 < s->tc_ev_used; i += 4) {
        float a = 0, b = 0, c = 0;
        cudaEventElapsedTime(&a, s->tc_ev[i], s->tc_ev[i + 1]);
        cudaEventElapsedTime(&b, s->tc_ev[i + 1], s->tc_ev[i + 2]);
        cudaEventElapsedTime(&c, s->tc_ev[i + 2], s->tc_ev[i + 3]);
        sel += a + c;
        gemm += b;
    }
    s->info.ms_tensor_gemm = gemm;
    s->info.ms_tensor_select = sel;
}

// records for the largest batch a run launches (its largest level, cut at
// the slot budget), allocated when the levels are known: a run that needs
// fewer slots than the budget allows never maps the whole budget
int sim_records(qsk_sim *s, long long slots) {
    const int n = int(std::max<long long>(1, std::min<long long>(slots, s->max_slots)));
    cudaError_t e = cudaSuccess;
    for (qsk_ti *x : s->all_tis())
        if (e == cudaSuccess) e = ensure_records(x->g, n, s->d_rec_val, s->d_rec_idx, s->d_rec_cnt, s->d_rec_max);
    if (e != cudaSuccess)
        return fail(e == cudaErrorMemoryAllocation ? QSK_ERR_NOMEM : QSK_ERR_CUDA, "records: %s", cudaGetErrorString(e));
    return QSK_OK;
}

int sim_check_status(qsk_sim *s) {
    int st = 0;
    CK(cudaMemcpyAsync(&st, s->d_status.p, sizeof(int), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    if (st != DEV_OK)
        return fail(QSK_ERR_DEVICE, "device status %d (%s)", st,
                    st == DEV_TOO_MANY_TERMS ? "too many terms for a node"
                    : st == DEV_LEVEL_WAIT   ? "a dependency level did not appear within the wait limit"
                    : st == DEV_BAD_INDEX    ? "index out of range"
                                             : "unknown");
    return QSK_OK;
}

}  // namespace

extern "C" {

int qsk_sim_create(int device, const qsk_qs_params *p, const float *di_init, qsk_sim **out) {
    if (!p || !out || !di_init || !p->ti_dims || !p->di_dims || !p->types || !p->ti) return fail(QSK_ERR_ARG, "null argument");
    if (p->ndim < 1 || p->ndim > QSK_MAXD) return fail(QSK_ERR_UNSUPPORTED, "ndim %d", p->ndim);
    const bool counts_given = (p->n_counts > 0 && p->n_per_variable) || (p->n_image_vars > 0 && p->n_image);
    if (p->n < 1 && !counts_given) return fail(QSK_ERR_ARG, "n must be >= 1");
    if (p->n_counts > 0 && p->n_per_variable)
        for (int q = 0; q < p->n_counts; ++q)
            if (p->n_per_variable[q] < 0) return fail(QSK_ERR_ARG, "negative neighbour count");
    if (p->n_kernels > 1 && !p->kernel_index_image)
        return fail(QSK_ERR_ARG, "several kernels need a kernel index image (-kii)");
    if (p->n_kernels > 0 && (!p->kernels_dims || !p->kernels)) return fail(QSK_ERR_ARG, "null kernel list");
    if (p->full_simulation && p->nvar > 4) return fail(QSK_ERR_UNSUPPORTED, "-fs with more than 4 variables");
    if (p->full_simulation && p->k_image && p->nvar > 1)
        return fail(QSK_ERR_UNSUPPORTED, "-fs with -kvi needs one value per cell and variable (G2S indexes it so)");
    // -kvi: the module's k becomes max(k, max k_image) (src/qs.cpp:1281-1292)
    float kbase = p->k;
    if (p->k_image) {
        if (!(kbase > 0.f)) kbase = 1.f;
        long long cells = 1;
        for (int d = 0; d < p->ndim; ++d) cells *= p->di_dims[d];
        for (long long c = 0; c < cells; ++c) kbase = std::max(kbase, p->k_image[c]);
    }
    if (!(kbase > 0.f)) return fail(QSK_ERR_UNSUPPORTED, "k must be > 0 (got %g)", double(p->k));
    int K = int(std::ceil(double(kbase)));
    if (K > QSK_KMAX) return fail(QSK_ERR_UNSUPPORTED, "ceil(k)=%d > %d", K, QSK_KMAX);
    DeviceGuard dgd(device);
    qsk_sim *s = new qsk_sim();
    std::memset(&s->info, 0, sizeof(s->info));
    s->device = device;
    s->nd = p->ndim;
    s->nvar = p->nvar;
    s->n = p->n;
    s->k = kbase;
    s->K = K;
    s->seed = p->seed;
    s->full = p->full_simulation != 0;
    s->no_verbatim = s->full ? 0 : p->no_verbatim;   // -fs has no verbatim record
    auto bail = [&](int rc) {
        qsk_sim_destroy(s);
        return rc;
    };
    int rc = qsk_ti_create_grid(device, p->ndim, p->ti_dims, p->nvar, p->types, p->ti, &s->ti);
    if (rc) {
        delete s;
        return rc;
    }
    if (p->n_extra_tis > 0) {
        if (!p->extra_ti_dims || !p->extra_tis) return bail(fail(QSK_ERR_ARG, "null extra training images"));
        if (p->n_extra_tis + 1 > QSK_MAX_TIS)
            return bail(fail(QSK_ERR_UNSUPPORTED, "%d training images (at most %d)", p->n_extra_tis + 1, QSK_MAX_TIS));
        if ((p->n_extra_tis + 1) * K > 16)
            return bail(fail(QSK_ERR_UNSUPPORTED, "%d candidates to merge (TIs x ceil(k), at most 16)",
                             (p->n_extra_tis + 1) * K));
        if (counts_given || p->k_image || p->kernel_index_image || p->n_kernels > 1 || s->full || s->no_verbatim)
            return bail(fail(QSK_ERR_UNSUPPORTED, "several training images: no local controls, -fs or -nV"));
        for (int t = 0; t < p->n_extra_tis; ++t) {
            qsk_ti *x = nullptr;
            rc = qsk_ti_create_grid(device, p->ndim, p->extra_ti_dims + size_t(t) * p->ndim, p->nvar, p->types,
                                    p->extra_tis[t], &x);
            if (rc) return bail(rc);
            s->xti.push_back(x);
        }
        for (qsk_ti *x : s->all_tis())
            if (x->missing) return bail(fail(QSK_ERR_UNSUPPORTED, "several training images: missing values"));
    }
    if (s->full && s->ti->missing)
        return bail(fail(QSK_ERR_UNSUPPORTED, "-fs with missing training-image values is not implemented"));
    cudaError_t e = cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->st_rng, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->st2, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_level, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_side, cudaEventDisableTiming);
    for (int p = 0; p < 2 && e == cudaSuccess; ++p) {
        e = cudaEventCreateWithFlags(&s->ev_ready[p], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_used[p], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) return bail(fail(QSK_ERR_CUDA, "stream: %s", cudaGetErrorString(e)));
    s->cells = 1;
    std::memset(&s->dg, 0, sizeof(s->dg));
    s->dg.nd = p->ndim;
    for (int d = 0; d < p->ndim; ++d) {
        s->dg.dims[d] = int(p->di_dims[d]);
        s->dg.stride[d] = s->cells;
        s->cells *= p->di_dims[d];
    }
    if (s->cells >= (1LL << 32) - 1) return bail(fail(QSK_ERR_UNSUPPORTED, "grid too large"));
    s->init.assign(di_init, di_init + size_t(s->cells) * s->nvar);
    if (p->ti_index_image) {
        // -ii: the TI of each cell, int(value) (samplingModule.hpp:70-73); a
        // negative value leaves the cell to every TI
        const int nti = int(s->xti.size()) + 1;
        for (long long c = 0; c < s->cells; ++c)
            if (int(p->ti_index_image[c]) >= nti)
                return bail(fail(QSK_ERR_ARG, "-ii: cell %lld names TI %d of %d", c, int(p->ti_index_image[c]), nti));
        if ((e = s->d_ii.upload(p->ti_index_image, size_t(s->cells), s->st)) != cudaSuccess)
            return bail(fail(QSK_ERR_CUDA, "-ii upload: %s", cudaGetErrorString(e)));
    }
    // kernels: the -ki list, the given one, or uniform of size min(TI/2+1)
    // (src/qs.cpp:1000-1042); one sorted template per kernel
    std::vector<unsigned> kd(p->ndim);
    if (p->n_kernels > 0) {
        for (int q = 0; q < p->n_kernels; ++q) add_template(s, p->kernels_dims + size_t(q) * p->ndim, p->kernels[q]);
    } else if (p->kernel && p->kernel_dims) {
        for (int d = 0; d < p->ndim; ++d) kd[d] = p->kernel_dims[d];
        add_template(s, kd.data(), p->kernel);
    } else {
        for (int d = 0; d < p->ndim; ++d) {
            kd[d] = std::min(p->ti_dims[d] / 2 + 1, p->ti_dims[d]);
            for (int t = 0; t < p->n_extra_tis; ++t) kd[d] = std::min(kd[d], p->extra_ti_dims[t * p->ndim + d] / 2 + 1);
        }
        add_template(s, kd.data(), nullptr);
    }
    if (s->full) build_path_full(s);
    else build_path(s);
    // local controls per path node (simulation.hpp:337-358,447-507; -fs 793-815)
    s->local = counts_given || p->k_image || p->kernel_index_image || p->n_kernels > 1 || s->full;
    if (s->local) {
        const long long nn = std::max<long long>(s->nodes, 1);
        s->node_kernel.assign(size_t(nn), 0);
        s->node_lim.assign(size_t(nn), 0);
        s->node_nv.assign(size_t(nn) * s->nvar, 0);
        s->node_k.assign(size_t(nn), kbase);
        const int nk = int(s->tpl_range.size() / 2);
        int nmax_all = 0;
        float kmax = kbase;
        std::vector<int> counts;
        for (long long i = 0; i < s->nodes; ++i) {
            const unsigned pv = s->order[s->begin + i];
            const unsigned cell = s->full ? pv / unsigned(s->nvar) : pv;
            if (p->n_image_vars > 0 && p->n_image) {
                counts.assign(size_t(p->n_image_vars), 0);
                for (int q = 0; q < p->n_image_vars; ++q)
                    counts[q] = int(p->n_image[size_t(cell) * p->n_image_vars + q]);
            } else if (p->n_counts > 0 && p->n_per_variable) {
                counts.assign(p->n_per_variable, p->n_per_variable + p->n_counts);
            } else {
                counts.assign(1, p->n);
            }
            int nmax = 0, nsum = 0;
            for (int v = 0; v < s->nvar; ++v) {
                int c = std::max(0, counts[size_t(v) % counts.size()]);
                s->node_nv[size_t(i) * s->nvar + v] = c;
                nmax = std::max(nmax, c);
                nsum += c;
            }
            // with one count per variable the vector walk also keeps the next
            // informed cell; under -fs a cell may serve a single variable, so up
            // to the sum of the counts are taken
            s->node_lim[size_t(i)] = s->full ? nsum : nmax + (counts.size() > 1 ? 1 : 0);
            nmax_all = std::max(nmax_all, s->node_lim[size_t(i)]);
            if (p->kernel_index_image) {
                int q = int(p->kernel_index_image[cell]);
                if (q < 0 || q >= nk) return bail(fail(QSK_ERR_ARG, "kernel index %d at cell %u outside [0,%d)", q, cell, nk));
                s->node_kernel[size_t(i)] = q;
            }
            if (p->k_image && p->k_image[cell] > 0.f) s->node_k[size_t(i)] = p->k_image[cell];   // nvar 1 under -fs
            kmax = std::max(kmax, s->node_k[size_t(i)]);
        }
        s->n = std::max(1, nmax_all);
        s->K = int(std::ceil(double(kmax)));
        if (s->K > QSK_KMAX) return bail(fail(QSK_ERR_UNSUPPORTED, "ceil(k)=%d > %d", s->K, QSK_KMAX));
    }
    s->maxterms = std::max(1, s->n * s->nvar * (s->ti->missing ? 2 : 1));
    // bit-sliced map: every variable categorical with bit planes, unit weights
    s->use_bits = s->ti->planes_ok && s->maxterms <= 255 && s->xti.empty();
    for (float wv : s->wtab) s->use_bits &= (wv == 1.f);
    // uploads
    if ((e = s->d_tpl.upload(s->tpl.data(), s->tpl.size(), s->st)) != cudaSuccess ||
        (e = s->d_wtab.upload(s->wtab.data(), s->wtab.size(), s->st)) != cudaSuccess ||
        (e = s->d_types.upload(p->types, size_t(p->nvar), s->st)) != cudaSuccess ||
        (e = s->d_path.upload(s->order.data(), s->order.size(), s->st)) != cudaSuccess ||
        (e = s->d_seeds.upload(s->seeds.data(), s->seeds.size(), s->st)) != cudaSuccess ||
        (e = s->d_post.upload(s->posterior.data(), s->posterior.size(), s->st)) != cudaSuccess ||
        (e = s->d_node_of_cell.upload(s->node_of_cell.data(), s->node_of_cell.size(), s->st)) != cudaSuccess ||
        (e = s->d_init.upload(s->init.data(), s->init.size(), s->st)) != cudaSuccess ||
        (e = s->d_state.alloc(s->init.size())) != cudaSuccess ||
        (e = s->d_id.alloc(size_t(s->cells) * (s->full ? s->nvar : 1))) != cudaSuccess ||
        (s->full && (e = s->d_nb_mask.alloc(size_t(std::max<long long>(s->nodes, 1)) * s->n)) != cudaSuccess) ||
        (e = s->d_node_cell.alloc(size_t(std::max<long long>(s->nodes, 1)))) != cudaSuccess ||
        (e = s->d_nb_count.alloc(size_t(std::max<long long>(s->nodes, 1)))) != cudaSuccess ||
        (e = s->d_nb_tpl.alloc(size_t(std::max<long long>(s->nodes, 1)) * s->n)) != cudaSuccess ||
        (e = s->d_nb_cell.alloc(size_t(std::max<long long>(s->nodes, 1)) * s->n)) != cudaSuccess ||
        (e = s->d_level.alloc(size_t(std::max<long long>(s->nodes, 1)))) != cudaSuccess ||
        (e = s->d_cursor.alloc(size_t(std::max<long long>(s->nodes, 1)))) != cudaSuccess ||
        (e = s->d_tile_sum.alloc(size_t((s->nodes + 1023) / 1024) + 2)) != cudaSuccess ||
        (e = s->d_lcnt.alloc(size_t(s->nodes) + 2)) != cudaSuccess ||
        (e = s->d_start.alloc(size_t(s->nodes) + 1)) != cudaSuccess ||
        (e = s->d_level_nodes.alloc(size_t(std::max<long long>(s->nodes, 1)))) != cudaSuccess ||
        (e = s->d_nl.alloc(1)) != cudaSuccess || (e = s->d_status.alloc(1)) != cudaSuccess ||
        (s->local && ((e = s->d_tpl_range.upload(s->tpl_range.data(), s->tpl_range.size(), s->st)) != cudaSuccess ||
                      (e = s->d_node_kernel.upload(s->node_kernel.data(), s->node_kernel.size(), s->st)) != cudaSuccess ||
                      (e = s->d_node_lim.upload(s->node_lim.data(), s->node_lim.size(), s->st)) != cudaSuccess ||
                      (e = s->d_node_nv.upload(s->node_nv.data(), s->node_nv.size(), s->st)) != cudaSuccess ||
                      (e = s->d_node_k.upload(s->node_k.data(), s->node_k.size(), s->st)) != cudaSuccess)))
        return bail(fail(e == cudaErrorMemoryAllocation ? QSK_ERR_NOMEM : QSK_ERR_CUDA, "upload: %s",
                         cudaGetErrorString(e)));
    // batch scratch: slots up to a record budget of ~2 GiB (records sized
    // for the largest training image)
    int nseg_max = 0;
    for (qsk_ti *x : s->all_tis()) nseg_max = std::max(nseg_max, x->g.nseg);
    size_t per_slot = size_t(nseg_max) * QSK_SEG * 8 + size_t(nseg_max) * 8 + sizeof(Term) * s->maxterms +
                      (s->use_bits ? 2 * (sizeof(StaticTerm) * s->maxterms + sizeof(Slot)) : 0);
    size_t budget = size_t(2) << 30;
    long long ms = (long long)(budget / per_slot);
    ms = std::max<long long>(1, std::min<long long>(ms, std::max<long long>(s->nodes, 1)));
    ms = std::min<long long>(ms, 65535);
    s->max_slots = int(ms);
    if ((e = s->d_slots.alloc(size_t(s->max_slots))) != cudaSuccess ||
        (e = s->d_mt_state.alloc(size_t(2) * s->max_slots * 624)) != cudaSuccess ||
        (e = s->d_mt_pre.alloc(size_t(2) * s->max_slots)) != cudaSuccess ||
        (s->use_bits && ((e = s->d_sslots.alloc(size_t(2) * s->max_slots)) != cudaSuccess ||
                         (e = s->d_sterms.alloc(size_t(2) * s->max_slots * s->maxterms)) != cudaSuccess)) ||
        (e = s->d_terms.alloc(size_t(s->max_slots) * s->maxterms)) != cudaSuccess)
        return bail(fail(e == cudaErrorMemoryAllocation ? QSK_ERR_NOMEM : QSK_ERR_CUDA, "scratch: %s",
                         cudaGetErrorString(e)));
    if ((size_t)s->maxterms * sizeof(Term) > 200 * 1024) return bail(fail(QSK_ERR_UNSUPPORTED, "n*nvar too large"));
    if (smem_configured_device != device) {
        if ((e = set_map_smem_limit(200 * 1024)) != cudaSuccess) return bail(fail(QSK_ERR_CUDA, "smem attr"));
        smem_configured_device = device;
    }
    if ((e = cudaStreamSynchronize(s->st)) != cudaSuccess) return bail(fail(QSK_ERR_CUDA, "%s", cudaGetErrorString(e)));
    s->info.nodes = s->nodes;
    s->info.template_size = s->ntpl;
    *out = s;
    return QSK_OK;
}

int qsk_sim_run(qsk_sim *s) {
    if (!s) return fail(QSK_ERR_ARG, "null sim");
    DeviceGuard dgd(s->device);
    cudaEvent_t ev[4];
    for (auto &x : ev) CK(cudaEventCreate(&x));
    CK(cudaMemcpyAsync(s->d_state.p, s->d_init.p, sizeof(float) * s->init.size(), cudaMemcpyDeviceToDevice, s->st));
    CK(cudaMemsetAsync(s->d_id.p, 0, sizeof(unsigned) * s->cells * (s->full ? s->nvar : 1), s->st));
    CK(cudaMemsetAsync(s->d_status.p, 0, sizeof(int), s->st));
    s->info.launches = 0;
    s->info.map_launches = 0;
    s->info.map_positions = 0;
    s->info.tensor_launches = 0;
    s->info.graph_nodes = 0;
    s->info.ms_graph_build = 0.f;
    CK(cudaEventRecord(ev[0], s->st));
    s->neighbours_ready = false;
    int rc = sim_neighbours(s);
    if (rc) return rc;
    CK(cudaEventRecord(ev[1], s->st));
    LevelArgs la;
    la.nodes = s->nodes;
    la.n = s->n;
    la.nb_count = s->d_nb_count.p;
    la.nb_cell = s->d_nb_cell.p;
    la.nb_mask = s->full ? s->d_nb_mask.p : nullptr;
    la.nvar = s->nvar;
    la.node_of_cell = s->d_node_of_cell.p;
    la.level = s->d_level.p;
    la.cursor = s->d_cursor.p;
    la.tile_sum = s->d_tile_sum.p;
    la.cnt = s->d_lcnt.p;
    la.status = s->d_status.p;
    la.level_nodes = s->d_level_nodes.p;
    la.start = s->d_start.p;
    la.nl_out = s->d_nl.p;
    la.spin_limit = s->level_spin_limit;
    la.hold = s->level_hold;
    CK(cudaMemsetAsync(s->d_nl.p, 0, sizeof(int), s->st));
    CK(launch_levels(la, s->st));
    s->info.launches += 7;  // neighbours, level pass, count, 3 scan passes, scatter
    int nl = 0;
    CK(cudaMemcpyAsync(&nl, s->d_nl.p, sizeof(int), cudaMemcpyDeviceToHost, s->st));
    rc = sim_check_status(s);
    if (rc) return rc;
    std::vector<int> start(size_t(nl) + 1, 0);
    if (nl > 0) {
        CK(cudaMemcpyAsync(start.data(), s->d_start.p, sizeof(int) * (nl + 1), cudaMemcpyDeviceToHost, s->st));
        CK(cudaStreamSynchronize(s->st));
    }
    if (s->nodes > 0 && (nl < 1 || start[size_t(nl)] != s->nodes))
        return fail(QSK_ERR_DEVICE, "dependency levels cover %d of %lld nodes", nl > 0 ? start[size_t(nl)] : 0,
                    s->nodes);
    int mb = 0;
    for (int l = 0; l < nl; ++l) mb = std::max(mb, start[l + 1] - start[l]);
    CK(cudaEventRecord(ev[2], s->st));
    cudaGraphExec_t gexec = nullptr;
    if (s->topt.mode != 0) {
        rc = tc_run(s, start, false);
    } else {
        rc = sim_records(s, mb);
        if (rc) return rc;
        if (!s->xti.empty())
            rc = sim_batches_multi(s, plain_steps(s, start));
        else if (s->use_graph && !s->profiling)
            rc = sim_batches_graph(s, plain_steps(s, start), &gexec);
        else
            rc = sim_batches(s, plain_steps(s, start), false);
    }
    if (rc) return rc;
    CK(cudaEventRecord(ev[3], s->st));
    CK(cudaEventSynchronize(ev[3]));
    if (gexec) cudaGraphExecDestroy(gexec);
    s->info.levels = nl;
    s->info.max_batch = mb;
    cudaEventElapsedTime(&s->info.ms_setup_neighbours, ev[0], ev[1]);
    cudaEventElapsedTime(&s->info.ms_levels, ev[1], ev[2]);
    cudaEventElapsedTime(&s->info.ms_batches, ev[2], ev[3]);
    cudaEventElapsedTime(&s->info.ms_total, ev[0], ev[3]);
    for (auto &x : ev) cudaEventDestroy(x);
    collect_profile(s);
    return sim_check_status(s);
}

int qsk_sim_run_teacher(qsk_sim *s, const float *di_completed, const unsigned *id_completed) {
    if (!s || !di_completed) return fail(QSK_ERR_ARG, "null argument");
    if (!s->xti.empty()) return fail(QSK_ERR_UNSUPPORTED, "teacher forcing with several training images");
    if (s->no_verbatim && !id_completed) return fail(QSK_ERR_ARG, "-nV teacher forcing needs the index image");
    DeviceGuard dgd(s->device);
    CK(cudaMemcpyAsync(s->d_state.p, di_completed, sizeof(float) * s->init.size(), cudaMemcpyHostToDevice, s->st));
    if (id_completed)
        CK(cudaMemcpyAsync(s->d_id.p, id_completed, sizeof(unsigned) * s->cells, cudaMemcpyHostToDevice, s->st));
    else
        CK(cudaMemsetAsync(s->d_id.p, 0, sizeof(unsigned) * s->cells * (s->full ? s->nvar : 1), s->st));
    CK(cudaMemsetAsync(s->d_status.p, 0, sizeof(int), s->st));
    int rc = sim_neighbours(s);
    if (rc) return rc;
    // every node is independent under teacher forcing: one level of all nodes in path order
    std::vector<int> ident(size_t(std::max<long long>(s->nodes, 1)));
    std::iota(ident.begin(), ident.end(), 0);
    CK(cudaMemcpyAsync(s->d_level_nodes.p, ident.data(), sizeof(int) * s->nodes, cudaMemcpyHostToDevice, s->st));
    std::vector<int> start = {0, int(s->nodes)};
    if (s->topt.mode != 0) {
        rc = tc_run(s, start, true);
    } else {
        rc = sim_records(s, s->nodes);
        if (rc) return rc;
        rc = sim_batches(s, plain_steps(s, start), true);
    }
    if (rc) return rc;
    s->info.nodes = s->nodes;
    s->info.levels = 1;
    s->info.max_batch = int(s->nodes);
    CK(cudaStreamSynchronize(s->st));
    return sim_check_status(s);
}

int qsk_sim_run_teacher_nodes(qsk_sim *s, const float *di_completed, const int *path_nodes, int count) {
    if (s && !s->xti.empty()) return fail(QSK_ERR_UNSUPPORTED, "teacher forcing with several training images");
    if (!s || !di_completed || (!path_nodes && count > 0) || count < 0) return fail(QSK_ERR_ARG, "null argument");
    if (s->no_verbatim) return fail(QSK_ERR_UNSUPPORTED, "-nV teacher forcing on a node sample");
    for (int q = 0; q < count; ++q)
        if (path_nodes[q] < 0 || path_nodes[q] >= s->nodes)
            return fail(QSK_ERR_ARG, "path node %d of %lld", path_nodes[q], s->nodes);
    DeviceGuard dgd(s->device);
    cudaEvent_t ev[2];
    for (auto &x : ev) CK(cudaEventCreate(&x));
    CK(cudaMemcpyAsync(s->d_state.p, di_completed, sizeof(float) * s->init.size(), cudaMemcpyHostToDevice, s->st));
    CK(cudaMemsetAsync(s->d_id.p, 0, sizeof(unsigned) * s->cells * (s->full ? s->nvar : 1), s->st));
    CK(cudaMemsetAsync(s->d_status.p, 0, sizeof(int), s->st));
    int rc = QSK_OK;
    if (!s->neighbours_ready) {
        rc = sim_neighbours(s);
        if (rc) return rc;
    }
    s->info.launches = 0;
    s->info.map_launches = 0;
    s->info.map_positions = 0;
    s->info.tensor_launches = 0;
    CK(cudaEventRecord(ev[0], s->st));
    if (count > 0)
        CK(cudaMemcpyAsync(s->d_level_nodes.p, path_nodes, sizeof(int) * count, cudaMemcpyHostToDevice, s->st));
    std::vector<int> start = {0, count};
    if (s->topt.mode != 0) {
        rc = tc_run(s, start, true);
    } else {
        rc = sim_records(s, count);
        if (rc) return rc;
        rc = sim_batches(s, plain_steps(s, start), true);
    }
    if (rc) return rc;
    CK(cudaEventRecord(ev[1], s->st));
    CK(cudaEventSynchronize(ev[1]));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev[0], ev[1]);
    for (auto &x : ev) cudaEventDestroy(x);
    s->info.nodes = count;
    s->info.levels = 1;
    s->info.max_batch = count;
    s->info.ms_batches = ms;
    s->info.ms_total = ms;
    collect_profile(s);
    return sim_check_status(s);
}

int qsk_sim_read(qsk_sim *s, float *di_out, unsigned *id_out, unsigned *node_cell_out) {
    if (!s) return fail(QSK_ERR_ARG, "null sim");
    DeviceGuard dgd(s->device);
    if (di_out)
        CK(cudaMemcpyAsync(di_out, s->d_state.p, sizeof(float) * s->init.size(), cudaMemcpyDeviceToHost, s->st));
    if (id_out)
        CK(cudaMemcpyAsync(id_out, s->d_id.p, sizeof(unsigned) * s->cells * (s->full ? s->nvar : 1),
                           cudaMemcpyDeviceToHost, s->st));
    if (node_cell_out && s->nodes > 0)
        CK(cudaMemcpyAsync(node_cell_out, s->d_node_cell.p, sizeof(unsigned) * s->nodes, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return QSK_OK;
}

int qsk_sim_get_info(const qsk_sim *s, qsk_sim_info *info) {
    if (!s || !info) return fail(QSK_ERR_ARG, "null argument");
    *info = s->info;
    info->path_nodes = s->nodes;
    return QSK_OK;
}

int qsk_sim_get_path(const qsk_sim *s, unsigned *order, float *seeds, unsigned *begin) {
    if (!s) return fail(QSK_ERR_ARG, "null sim");
    if (order) std::copy(s->order.begin(), s->order.end(), order);
    if (seeds) std::copy(s->seeds.begin(), s->seeds.end(), seeds);
    if (begin) *begin = s->begin;
    return QSK_OK;
}

int qsk_sim_set_profiling(qsk_sim *s, int on) {
    if (!s) return fail(QSK_ERR_ARG, "null sim");
    s->profiling = on != 0;
    return QSK_OK;
}

int qsk_sim_set_tensor(qsk_sim *s, const qsk_tensor_opts *o) {
    if (!s || !o) return fail(QSK_ERR_ARG, "null argument");
    if (o->mode != 0 && !s->xti.empty())
        return fail(QSK_ERR_UNSUPPORTED, "tensor-core form: one training image (several run on the plain path)");
    if (o->mode < 0 || o->mode > 2) return fail(QSK_ERR_ARG, "tensor mode %d (0 plain, 1 BF16, 2 FP8)", o->mode);
    if (!(o->audit >= 0.f && o->audit <= 1.f)) return fail(QSK_ERR_ARG, "audit fraction %g", double(o->audit));
    if (o->width != 0 && !tc_supported_width(o->width)) return fail(QSK_ERR_ARG, "width %d (8, 16 or 32)", o->width);
    if (o->shortlist < 0 || o->shortlist > 128) return fail(QSK_ERR_ARG, "shortlist %d (at most 128)", o->shortlist);
    if (o->prefix < 0) return fail(QSK_ERR_ARG, "prefix %d", o->prefix);
    if (o->batch < 0 || o->batch > 16384 || o->batch % 128)
        return fail(QSK_ERR_ARG, "batch %d (a multiple of 128 up to 16384)", o->batch);
    if (o->mode != 0) {
        if (s->ti->missing) return fail(QSK_ERR_UNSUPPORTED, "tensor-core form: training image with missing values");
        if (s->no_verbatim || s->full || s->local)
            return fail(QSK_ERR_UNSUPPORTED, "tensor-core form: -nV, -fs and local controls run on the plain path");
        if (!s->ti->cat_ok) return fail(QSK_ERR_UNSUPPORTED, "tensor-core form: more than %d categories", QSK_CMAX);
        if (s->ti->g.nd > 3) return fail(QSK_ERR_UNSUPPORTED, "tensor-core form: %d dimensions (at most 3)", s->ti->g.nd);
        if (s->ti->cells > (1LL << 31)) return fail(QSK_ERR_UNSUPPORTED, "tensor-core form: TI of %lld cells", s->ti->cells);
    }
    s->topt = *o;
    s->max_tc_slots = o->batch > 0 ? o->batch : 4096;
    if (o->mode == 0) {
        s->info.tensor_mode = 0;
        s->info.tensor_nodes = s->info.plain_nodes = s->info.audited = s->info.regret = s->info.regret_near = 0;
    }
    return QSK_OK;
}

int qsk_sim_set_learned(qsk_sim *s, qsk_encoder *e, const qsk_learned_opts *o) {
    if (!s) return fail(QSK_ERR_ARG, "null sim");
    if (e && !s->xti.empty()) return fail(QSK_ERR_UNSUPPORTED, "learned proposal: one training image");
    if (!e) {
        s->enc = nullptr;
        s->topt = qsk_tensor_opts{};
        s->tc_ready = false;
        return QSK_OK;
    }
    qsk_learned_opts d{};
    if (!o) o = &d;
    if (o->width != 0 && !tc_supported_width(o->width)) return fail(QSK_ERR_ARG, "width %d (8, 16 or 32)", o->width);
    if (o->shortlist < 0 || o->shortlist > 256) return fail(QSK_ERR_ARG, "shortlist %d (at most 256)", o->shortlist);
    if (!(o->audit >= 0.f && o->audit <= 1.f) || o->conf_rank < 0) return fail(QSK_ERR_ARG, "audit / confidence rank");
    if (e->nvar != s->nvar) return fail(QSK_ERR_ARG, "encoder for %d variables, simulation of %d", e->nvar, s->nvar);
    if (e->device != s->device) return fail(QSK_ERR_ARG, "encoder on device %d, simulation on %d", e->device, s->device);
    if (s->ti->missing || s->no_verbatim || s->full || s->local)
        return fail(QSK_ERR_UNSUPPORTED, "learned proposal: complete TIs without -nV, -fs or local controls");
    if (s->ti->g.nd > 3 || s->ti->cells > (1LL << 31))
        return fail(QSK_ERR_UNSUPPORTED, "learned proposal: at most 3 dimensions and 2^31 cells");
    // the pre-embedded TI stays while the same encoder is set again (it is
    // rebuilt when the encoder has trained or changed its scales since)
    const bool same = s->enc == e && s->topt.mode == 3;
    s->enc = e;
    s->lopt = *o;
    s->topt = qsk_tensor_opts{};
    s->topt.mode = 3;
    s->topt.audit = o->audit;
    s->max_tc_slots = 4096;
    if (!same) {
        s->tc_ready = false;
        s->enc_built = -1;
    }
    return QSK_OK;
}

int qsk_encoder_add_pairs(qsk_encoder *e, qsk_sim *s, const float *di_completed, const int *path_nodes, int count,
                          long long *added) {
    if (!e || !s || !di_completed || (!path_nodes && count > 0) || count < 0) return fail(QSK_ERR_ARG, "null argument");
    if (e->nvar != s->nvar || e->device != s->device) return fail(QSK_ERR_ARG, "encoder and simulation differ");
    DeviceGuard dgd(s->device);
    // the exact path draws the nodes (teacher-forced), nodes without
    // neighbours left out (their draw is the marginal one)
    const qsk_tensor_opts keep = s->topt;
    s->topt = qsk_tensor_opts{};
    int rc = QSK_OK;
    if (!s->neighbours_ready && (rc = sim_neighbours(s)) != QSK_OK) return rc;
    std::vector<int> tmax;
    if ((rc = tc_tmax(s, tmax)) != QSK_OK) return rc;
    std::vector<int> nodes;
    for (int q = 0; q < count; ++q) {
        const int i = path_nodes[q];
        if (i < 0 || i >= s->nodes) {
            s->topt = keep;
            return fail(QSK_ERR_ARG, "path node %d of %lld", i, s->nodes);
        }
        if (tmax[size_t(i)] >= 0) nodes.push_back(i);
    }
    rc = qsk_sim_run_teacher_nodes(s, di_completed, nodes.data(), int(nodes.size()));
    s->topt = keep;
    if (rc) return rc;
    std::vector<unsigned> cell_all(size_t(s->nodes));
    CK(cudaMemcpyAsync(cell_all.data(), s->d_node_cell.p, sizeof(unsigned) * size_t(s->nodes), cudaMemcpyDeviceToHost,
                       s->st));
    CK(cudaStreamSynchronize(s->st));
    std::vector<unsigned> cells(nodes.size());
    for (size_t q = 0; q < nodes.size(); ++q) cells[q] = cell_all[size_t(nodes[q])];
    const long long n = (long long)nodes.size();
    const size_t rowf = size_t(e->D0);
    if (e->npairs + n > e->pair_cap) {
        const long long cap = std::max<long long>(e->npairs + n, 2 * e->pair_cap);
        DBuf<float> q2, p2;
        CK(q2.alloc(size_t(cap) * rowf));
        CK(p2.alloc(size_t(cap) * rowf));
        if (e->npairs) {
            CK(cudaMemcpyAsync(q2.p, e->xq.p, sizeof(float) * size_t(e->npairs) * rowf, cudaMemcpyDeviceToDevice, s->st));
            CK(cudaMemcpyAsync(p2.p, e->xp.p, sizeof(float) * size_t(e->npairs) * rowf, cudaMemcpyDeviceToDevice, s->st));
            CK(cudaStreamSynchronize(s->st));
        }
        e->xq.swap(q2);
        e->xp.swap(p2);
        e->pair_cap = cap;
    }
    DBuf<unsigned> dcells;
    CK(dcells.upload(cells.data(), cells.size(), s->st));
    // both sides of a pair at the node's stencil scale
    DBuf<int> dscale;
    CK(dscale.ensure(size_t(std::max<long long>(n, 1))));
    if ((rc = node_scales(s, e, s->d_level_nodes.p, n, dscale.p)) != QSK_OK) return rc;
    const Geom &g = s->ti->g;
    FeatArgs fa;
    fa.rows = n;
    fa.nodes = s->d_level_nodes.p;   // the sample, in order (run_teacher_nodes)
    fa.path = s->d_path.p;
    fa.begin = s->begin;
    fa.nb_count = s->d_nb_count.p;
    fa.nb_tpl = s->d_nb_tpl.p;
    fa.nb_cell = s->d_nb_cell.p;
    fa.n = s->n;
    fa.state = s->d_state.p;
    fa.tpl = s->d_tpl.p;
    fa.nd = g.nd;
    fa.nvar = s->nvar;
    fa.inv_radius = 0.125f;
    fa.ntpl = s->ntpl;
    fa.entries = QSK_ENC_ENTRIES;
    feat_stencil(s, e, fa);
    fa.row_scale = dscale.p;
    fa.out = e->xq.p + size_t(e->npairs) * rowf;
    CK(launch_feat_nodes(fa, s->st));
    FeatArgs fc = fa;
    fc.cell_list = dcells.p;
    fc.cells = s->ti->cells;
    fc.ti = s->ti->grid.p;
    for (int d = 0; d < 3; ++d) fc.src[d] = d < g.nd ? g.src[d] : 1;
    fc.ntpl = s->ntpl;
    fc.entries = QSK_ENC_ENTRIES;
    fc.out = e->xp.p + size_t(e->npairs) * rowf;
    CK(launch_feat_cells(fc, s->st));
    CK(cudaStreamSynchronize(s->st));
    e->npairs += n;
    if (added) *added = n;
    return QSK_OK;
}

int qsk_sim_set_graph(qsk_sim *s, int on) {
    if (!s) return fail(QSK_ERR_ARG, "null sim");
    s->use_graph = on != 0;
    return QSK_OK;
}

int qsk_jobs_run(qsk_sim *const *sims, int count, int threads, int *status) {
    if (count < 0 || (count > 0 && !sims)) return fail(QSK_ERR_ARG, "jobs: %d simulations", count);
    for (int i = 0; i < count; ++i) {
        if (!sims[i]) return fail(QSK_ERR_ARG, "job %d: null simulation", i);
        for (int j = 0; j < i; ++j)
            if (sims[j] == sims[i]) return fail(QSK_ERR_ARG, "jobs %d and %d are the same simulation", j, i);
    }
    if (count == 0) return QSK_OK;
    const int T = std::max(1, std::min(threads > 0 ? threads : 16, count));
    // largest jobs first (a long job started last would end the call late)
    std::vector<int> order((size_t)count);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return sims[a]->nodes > sims[b]->nodes; });
    std::atomic<int> next{0};
    std::vector<int> rc((size_t)count, QSK_OK);
    std::vector<std::string> msg((size_t)count);
    // each thread lends its own batch scratch (map records, pattern matrix)
    // to the job it runs, so that the memory held is that of the jobs in
    // flight and buffers are not freed and reallocated between jobs; a
    // simulation's own buffers are left as they were
    struct Scratch {
        DBuf<float> rv, rm;
        DBuf<int> ri, rc;
        DBuf<unsigned char> P;
        DBuf<float> pscale;
    };
    auto swap_scratch = [](qsk_sim *s, Scratch &x) {
        auto sw = [](auto &a, auto &b) { a.swap(b); };
        sw(s->d_rec_val, x.rv);
        sw(s->d_rec_idx, x.ri);
        sw(s->d_rec_cnt, x.rc);
        sw(s->d_rec_max, x.rm);
        sw(s->d_tc_P, x.P);
        sw(s->d_tc_pscale, x.pscale);
        s->tc_ready = false;   // the pattern matrix now in s (if any) is not its own
    };
    auto worker = [&]() {
        std::vector<std::pair<int, Scratch *>> mine;   // per device
        for (int q = next.fetch_add(1); q < count; q = next.fetch_add(1)) {
            const int i = order[size_t(q)];
            qsk_sim *s = sims[i];
            Scratch *x = nullptr;
            for (auto &m : mine)
                if (m.first == s->device) x = m.second;
            if (!x) {
                x = new Scratch();
                mine.emplace_back(s->device, x);
            }
            {
                DeviceGuard dg(s->device);
                swap_scratch(s, *x);
                rc[size_t(i)] = qsk_sim_run(s);
                cudaStreamSynchronize(s->st);   // nothing of the run still reads the scratch
                swap_scratch(s, *x);
            }
            if (rc[size_t(i)] != QSK_OK) msg[size_t(i)] = g_err;
        }
        for (auto &m : mine) {
            DeviceGuard dg(m.first);
            delete m.second;
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < T; ++t) pool.emplace_back(worker);
    worker();
    for (auto &th : pool) th.join();
    int first = QSK_OK;
    for (int i = 0; i < count; ++i) {
        if (status) status[i] = rc[size_t(i)];
        if (first == QSK_OK && rc[size_t(i)] != QSK_OK) {
            first = rc[size_t(i)];
            g_err = "job " + std::to_string(i) + ": " + msg[size_t(i)];
        }
    }
    return first;
}

int qsk_sim_set_level_wait(qsk_sim *s, unsigned spin_limit, long long hold_node) {
    if (!s) return fail(QSK_ERR_ARG, "null sim");
    if (hold_node < -1 || hold_node >= s->nodes) return fail(QSK_ERR_ARG, "hold node %lld of %lld", hold_node, s->nodes);
    s->level_spin_limit = spin_limit;
    s->level_hold = hold_node;
    return QSK_OK;
}

int qsk_sim_destroy(qsk_sim *s) {
    if (!s) return QSK_OK;
    {
        DeviceGuard dgd(s->device);
        // the simulation's device buffers go to the kept blocks (reused by
        // the next simulations of this device) once nothing on the device
        // reads them any more: cudaFree would wait for the device as well
        g_keep_blocks = cudaDeviceSynchronize() == cudaSuccess;
        for (auto e : s->prof_ev) cudaEventDestroy(e);
        for (auto e : s->tc_ev) cudaEventDestroy(e);
        for (int p = 0; p < 2; ++p) {
            if (s->ev_ready[p]) cudaEventDestroy(s->ev_ready[p]);
            if (s->ev_used[p]) cudaEventDestroy(s->ev_used[p]);
        }
        if (s->ev_level) cudaEventDestroy(s->ev_level);
        if (s->ev_side) cudaEventDestroy(s->ev_side);
        if (s->st2) cudaStreamDestroy(s->st2);
        if (s->st_rng) cudaStreamDestroy(s->st_rng);
        if (s->st) cudaStreamDestroy(s->st);
        s->st = nullptr;
        if (s->ti) qsk_ti_destroy(s->ti);
        for (qsk_ti *x : s->xti) qsk_ti_destroy(x);
        s->xti.clear();
        s->ti = nullptr;
        delete s;
        g_keep_blocks = false;
    }
    return QSK_OK;
}

int qsk_set_map_mode(int mode) {
    if (mode < 0 || mode > 1) return fail(QSK_ERR_ARG, "map mode %d", mode);
    g_map_mode = mode;
    return QSK_OK;
}

int qsk_qs_template(int ndim, int nvar, const unsigned *kernel_dims, const float *kernel, int *offsets, float *weights,
                    int capacity) {
    if (!kernel_dims || ndim < 1 || ndim > QSK_MAXD || nvar < 1) return -QSK_ERR_ARG;
    std::vector<int> tpl;
    std::vector<float> w;
    int n = make_template(ndim, nvar, kernel_dims, kernel, tpl, w);
    for (int t = 0; t < n && t < capacity; ++t) {
        if (offsets)
            for (int d = 0; d < ndim; ++d) offsets[t * ndim + d] = tpl[size_t(t) * ndim + d];
        if (weights)
            for (int v = 0; v < nvar; ++v) weights[t * nvar + v] = w[size_t(t) * nvar + v];
    }
    return n;
}

long long qsk_qs_path(long long cells, int nvar, const float *di_init, unsigned seed, unsigned *order, float *seeds) {
    if (!di_init || cells < 1 || nvar < 1) return -QSK_ERR_ARG;
    std::vector<unsigned> o;
    std::vector<float> sd;
    unsigned begin = make_path(size_t(cells), nvar, di_init, seed, o, sd);
    if (order) std::copy(o.begin(), o.end(), order);
    if (seeds) std::copy(sd.begin(), sd.end(), seeds);
    return (long long)begin;
}

int qsk_simulate(int device, const qsk_qs_params *p, float *di_inout, unsigned *id_out) {
    qsk_sim *s = nullptr;
    int rc = qsk_sim_create(device, p, di_inout, &s);
    if (rc) return rc;
    rc = qsk_sim_run(s);
    if (!rc) rc = qsk_sim_read(s, di_inout, id_out, nullptr);
    qsk_sim_destroy(s);
    return rc;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// qsk_pattern_kbest_noalloc: the map + k-best of qsk_pattern_kbest for callers
// that cannot allocate (their device memory is held by another allocator, or
// they must not stall the device's other streams with cudaFree's implicit
// synchronisation).  Its device scratch is the fixed array below; the host
// side stages the slot and the terms on the stack.  Nothing in it calls
// cudaMalloc, cudaFree or an allocating library routine.
// ---------------------------------------------------------------------------
namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[QSK_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned char *g_noalloc_addr[kMaxDevices] = {};

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// scratch layout of one call; every region 256-byte aligned
struct NoallocLayout {
    size_t slot, terms, rec_val, rec_idx, rec_cnt, rec_max, out_val, out_pos, total;
};

NoallocLayout noalloc_layout(const Geom &g, int nterms, unsigned k) {
    NoallocLayout L;
    const size_t recs = size_t(g.nseg) * QSK_SEG;
    size_t o = 0;
    L.slot = o;
    o = align256(o + sizeof(Slot));
    L.terms = o;
    o = align256(o + sizeof(Term) * size_t(std::max(nterms, 1)));
    L.rec_val = o;
    o = align256(o + sizeof(float) * recs);
    L.rec_idx = o;
    o = align256(o + sizeof(int) * recs);
    L.rec_cnt = o;
    o = align256(o + sizeof(int) * size_t(g.nseg));
    L.rec_max = o;
    o = align256(o + sizeof(float) * size_t(g.nseg));
    L.out_val = o;
    o = align256(o + sizeof(float) * k);
    L.out_pos = o;
    o = align256(o + sizeof(unsigned) * k);
    L.total = o;
    return L;
}

// address of the scratch array on `device` (current), looked up once per device
int noalloc_scratch(int device, unsigned char **out) {
    if (device < 0 || device >= kMaxDevices) return fail(QSK_ERR_UNSUPPORTED, "device %d out of range", device);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return fail(QSK_ERR_CUDA, "cudaGetSymbolAddress(scratch) on device %d: %s", device, cudaGetErrorString(e));
        g_noalloc_addr[device] = static_cast<unsigned char *>(p);
    }
    *out = g_noalloc_addr[device];
    return QSK_OK;
}

}  // namespace

extern "C" {

int qsk_pattern_kbest_noalloc(const qsk_ti *ti, void *stream, int n_neighbours, const int *offsets, int n_terms,
                              const qsk_term *terms, unsigned k, float seed, float *out_score, unsigned *out_index,
                              int *out_min) {
    if (!ti || n_neighbours < 0 || n_terms < 0 || !out_score || !out_index || (n_neighbours > 0 && !offsets) ||
        (n_terms > 0 && !terms))
        return fail(QSK_ERR_ARG, "null argument");
    if (k < 1 || k > QSK_KMAX) return fail(QSK_ERR_UNSUPPORTED, "k=%u outside [1,%d]", k, QSK_KMAX);
    if (n_terms > QSK_NOALLOC_MAX_TERMS)
        return fail(QSK_ERR_UNSUPPORTED, "qsk_pattern_kbest_noalloc: %d terms, at most %d", n_terms,
                    QSK_NOALLOC_MAX_TERMS);
    const Geom &g = ti->g;
    const int nd = g.nd;
    const NoallocLayout L = noalloc_layout(g, n_terms, k);
    if (L.total > size_t(QSK_NOALLOC_SCRATCH_BYTES))
        return fail(QSK_ERR_UNSUPPORTED,
                    "qsk_pattern_kbest_noalloc: a training image of %lld positions with %d terms needs %zu bytes of "
                    "scratch; the fixed scratch holds %zu (use qsk_pattern_kbest)",
                    g.N, n_terms, L.total, size_t(QSK_NOALLOC_SCRATCH_BYTES));
    DeviceGuard dgd(ti->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned char *base = nullptr;
    int rc = noalloc_scratch(ti->device, &base);
    if (rc) return rc;

    // slot and terms on the stack (same rules as build_pattern_slot)
    Slot s;
    std::memset(&s, 0, sizeof(s));
    s.node = 0;
    s.seed = seed;
    s.excl = -1;
    s.K = int(k);
    int mn[QSK_MAXD] = {0}, mx[QSK_MAXD] = {0};
    for (int j = 0; j < n_neighbours; ++j)
        for (int d = 0; d < nd; ++d) {
            mn[d] = std::min(mn[d], offsets[j * nd + d]);
            mx[d] = std::max(mx[d], offsets[j * nd + d]);
        }
    long long nvalid = 1;
    for (int d = 0; d < QSK_MAXD; ++d) {
        s.mn[d] = mn[d];
        int lo = 0;
        if (d < nd) {
            lo = g.fft[d] - (g.src[d] - (mx[d] - mn[d]));
            lo = std::max(0, std::min(lo, g.fft[d]));
            nvalid *= (g.fft[d] - lo);
        }
        s.lo[d] = lo;
        if (out_min && d < nd) out_min[d] = mn[d];
    }
    if (n_neighbours == 0) {
        // candidateForPattern returns false on an empty pattern
        for (unsigned j = 0; j < k; ++j) {
            out_score[j] = -INFINITY;
            out_index[j] = 0xffffffffu;
        }
        return QSK_OK;
    }
    if (nvalid < (long long)k) s.flags |= SLOT_EMIT_MASKED;
    Term h_terms[QSK_NOALLOC_MAX_TERMS];
    bool bits = ti->planes_ok && g_map_mode == 0 && n_terms <= 255;
    for (int t = 0; t < n_terms; ++t) {
        const qsk_term &q = terms[t];
        if (q.neighbour < 0 || q.neighbour >= n_neighbours || q.layer < 0 || q.layer >= ti->nlayers || q.op < 0 ||
            q.op > 3)
            return fail(QSK_ERR_ARG, "pattern term %d out of range", t);
        long long dflat = 0;
        for (int d = 0; d < nd; ++d) dflat += (long long)(offsets[q.neighbour * nd + d] - mn[d]) * g.sstride[d];
        Term &tm = h_terms[t];
        tm.base = int((long long)q.layer * g.N - dflat);
        tm.a = q.a;
        tm.b = q.b;
        tm.op = q.op == QSK_OP_LIN_CROSS ? OP_LINX : q.op;
        bits &= (tm.op == OP_EQ && tm.a == 1.f);
    }
    s.nterms = n_terms;
    const int maxterms = std::max(n_terms, 1);

    Slot *d_slot = reinterpret_cast<Slot *>(base + L.slot);
    Term *d_terms = reinterpret_cast<Term *>(base + L.terms);
    float *rec_val = reinterpret_cast<float *>(base + L.rec_val);
    int *rec_idx = reinterpret_cast<int *>(base + L.rec_idx);
    int *rec_cnt = reinterpret_cast<int *>(base + L.rec_cnt);
    float *rec_max = reinterpret_cast<float *>(base + L.rec_max);
    float *out_val = reinterpret_cast<float *>(base + L.out_val);
    unsigned *out_pos = reinterpret_cast<unsigned *>(base + L.out_pos);

    CK(set_map_smem_limit(200 * 1024));
    CK(cudaMemcpyAsync(d_slot, &s, sizeof(Slot), cudaMemcpyHostToDevice, st));
    if (n_terms > 0) CK(cudaMemcpyAsync(d_terms, h_terms, sizeof(Term) * n_terms, cudaMemcpyHostToDevice, st));
    if (bits) {
        BitArgs ba;
        ba.g = g;
        ba.planes = ti->planes.p;
        ba.pw = ti->pw;
        ba.ncat = ti->ncat.p;
        ba.catv = ti->catv.p;
        ba.slots = d_slot;
        ba.terms = d_terms;
        ba.maxterms = maxterms;
        ba.segs_per_cta = map_bits_segs_per_cta(g, 1);
        ba.rec_val = rec_val;
        ba.rec_idx = rec_idx;
        ba.rec_cnt = rec_cnt;
        ba.rec_max = rec_max;
        CK(launch_map_bits(ba, 1, int(k), maxterms, st));
    } else {
        MapArgs ma;
        ma.g = g;
        ma.layers = ti->layers.p;
        ma.slots = d_slot;
        ma.terms = d_terms;
        ma.maxterms = maxterms;
        ma.segs_per_cta = map_segs_per_cta(g, 1);
        ma.rec_val = rec_val;
        ma.rec_idx = rec_idx;
        ma.rec_cnt = rec_cnt;
        ma.rec_max = rec_max;
        CK(launch_map_records(ma, 1, int(k), maxterms, st));
    }
    ReplayArgs ra;
    std::memset(&ra, 0, sizeof(ra));
    ra.g = g;
    ra.slots = d_slot;
    ra.nslots = 1;
    ra.K = int(k);
    ra.rec_val = rec_val;
    ra.rec_idx = rec_idx;
    ra.rec_cnt = rec_cnt;
    ra.rec_max = rec_max;
    ra.out_val = out_val;
    ra.out_pos = out_pos;
    CK(launch_replay(ra, st));
    CK(cudaMemcpyAsync(out_score, out_val, sizeof(float) * k, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(out_index, out_pos, sizeof(unsigned) * k, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return QSK_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// f3: auto_qs calibration (G2S include/calibration.hpp:30-284, src/auto_qs.cpp:
// 640-700) on the batched engine.  Setup s = (neighbour configuration, kernel,
// density), configurations fastest, draws its samples from its own
// std::mt19937(seed + s).  Every iteration tests all setups against the
// statistics as they stood when it began, searches the samples of the unpruned
// ones in one batched query (verbatim exclusion of the sample's own cell with
// the reference's radius), then accumulates their errors and updates the best
// mean error per density in setup order.  The reference draws from one
// generator per OpenMP thread (seeded from the clock) and tests each setup
// after the updates of the setups before it in the same iteration; its
// results depend on the thread schedule and the clock, so the order here is
// this engine's (the oracle restates the same order).
// ---------------------------------------------------------------------------
namespace {

struct CalibSample {
    unsigned cell = 0;
    std::vector<int> offs;
    std::vector<float> vals;
    float seed = 0.f;
    bool search = false;
};

// the sample of one setup (include/calibration.hpp:113-224 up to the search)
CalibSample calib_draw(const qsk_calib_params *p, const std::vector<int> &tpl, int ntpl, const unsigned *nn, int ncounts,
                       float density, std::mt19937 &gen) {
    std::uniform_real_distribution<float> U(0.f, 1.f);
    const int nd = p->ndim, nvar = p->nvar;
    CalibSample S;
    unsigned cells = 1;
    for (int d = 0; d < nd; ++d) cells *= p->ti_dims[d];
    (void)int(std::floor(U(gen) * 1.f));   // TI index (one TI)
    S.cell = unsigned(std::floor(U(gen) * float(cells * unsigned(nvar)) / float(unsigned(nvar))));
    int c0[QSK_MAXD];
    unsigned rest = S.cell;
    for (int d = 0; d < nd; ++d) {
        c0[d] = int(rest % p->ti_dims[d]);
        rest /= p->ti_dims[d];
    }
    std::vector<unsigned> per(size_t(nvar), 0u);
    int ps = 0;
    while ((ncounts > 1 || S.offs.size() / size_t(nd) < nn[0]) && ps < ntpl) {
        bool take = U(gen) < density;
        long long dataIndex = 0;
        if (take) {
            long long stride = 1;
            for (int d = 0; d < nd; ++d) {
                const int c = c0[d] + tpl[size_t(ps) * nd + d];
                if (c < 0 || c >= int(p->ti_dims[d])) take = false;
                dataIndex += (long long)c * stride;
                stride *= p->ti_dims[d];
            }
        }
        if (take) {
            unsigned cpt = 0;
            for (int v = 0; v < nvar; ++v) {
                if (per[v] < nn[v % ncounts]) {
                    S.vals.push_back(p->ti[size_t(dataIndex) * nvar + v]);
                    cpt++;
                    per[v]++;
                } else {
                    S.vals.push_back(NAN);
                }
            }
            for (int d = 0; d < nd; ++d) S.offs.push_back(tpl[size_t(ps) * nd + d]);
            if (cpt == 0) break;
        }
        ps++;
    }
    if (ps >= ntpl) return S;
    const size_t n = S.offs.size() / size_t(nd);
    if (n > 1 && p->noise > 0.f) {
        float fraction = p->noise / float(n) / 2.f;
        if (p->noise < 1.0f) fraction = p->noise / 2.f;
        for (size_t j = 0; j < n; ++j)
            if (U(gen) < fraction) {
                const size_t a = size_t(std::floor(U(gen) * float(n)));
                const size_t b = size_t(std::floor(U(gen) * float(n)));
                for (int d = 0; d < nd; ++d) std::swap(S.offs[a * nd + d], S.offs[b * nd + d]);
            }
    }
    if (n > 1) {
        S.seed = U(gen);
        S.search = true;
    }
    return S;
}

// kernel weight of offset o for variable v, centred at dims/2 (0 outside)
float calib_weight(int nd, const unsigned *kd, int knvar, const float *k, const int *o, int v) {
    long long f = 0, stride = 1;
    for (int d = 0; d < nd; ++d) {
        const int c = int(kd[d] / 2) + o[d];
        if (c < 0 || c >= int(kd[d])) return 0.f;
        f += (long long)c * stride;
        stride *= kd[d];
    }
    return k[size_t(f) * knvar + (v % knvar)];
}

}  // namespace

extern "C" {

int qsk_calibrate(int device, const qsk_calib_params *p, float *mean_error, float *dev_error, unsigned *n_samples,
                  long long *n_searches) {
    if (!p || !p->ti_dims || !p->types || !p->ti || !p->kernel_dims || !p->kernels || !p->counts || !p->densities ||
        !mean_error || !dev_error || !n_samples)
        return fail(QSK_ERR_ARG, "null argument");
    if (p->ndim < 1 || p->ndim > QSK_MAXD || p->nvar < 1 || p->n_kernels < 1 || p->n_configs < 1 || p->n_counts < 1 ||
        p->n_densities < 1 || !(p->power > 0.f))
        return fail(QSK_ERR_ARG, "invalid calibration parameters");
    if (p->max_k < 1 || p->max_k > QSK_KMAX) return fail(QSK_ERR_UNSUPPORTED, "max_k=%u outside [1,%d]", p->max_k, QSK_KMAX);
    for (int i = 0; i < p->n_kernels; ++i)
        if (!p->kernels[i] || !p->kernel_nvar || p->kernel_nvar[i] < 1)
            return fail(QSK_ERR_ARG, "kernel %d missing", i);
    const int nd = p->ndim, nvar = p->nvar;
    size_t cells = 1;
    for (int d = 0; d < nd; ++d) cells *= p->ti_dims[d];
    for (size_t i = 0; i < cells * size_t(nvar); ++i)
        if (std::isnan(p->ti[i]))
            return fail(QSK_ERR_UNSUPPORTED, "calibration with missing training-image values is not implemented");
    // pathPosition: the box of kernel 0, nearest first (src/auto_qs.cpp:452-492)
    std::vector<int> tpl;
    std::vector<float> wtab_unused;
    int ntpl = make_template(nd, 1, p->kernel_dims, nullptr, tpl, wtab_unused);
    if (ntpl <= 0) return fail(QSK_ERR_ARG, "empty template");
    // exclusion radius of the sample's own cell (include/calibration.hpp:33)
    const float radius = float(std::pow(double(unsigned(cells) * unsigned(nvar) / unsigned(nvar)) * 0.005,
                                        1.f / float(nd)));
    qsk_ti *ti = nullptr;
    int rc = qsk_ti_create_grid(device, nd, p->ti_dims, nvar, p->types, p->ti, &ti);
    if (rc) return rc;
    qsk_worker *w = nullptr;
    if ((rc = qsk_worker_create(ti, &w)) != QSK_OK) {
        qsk_ti_destroy(ti);
        return rc;
    }
    const size_t setups = size_t(p->n_configs) * p->n_kernels * p->n_densities;
    const size_t K = p->max_k;
    std::vector<double> cum(setups * K, 0.0), cum2(setups * K, 0.0);
    std::vector<uint16_t> ns(setups * K, 0);
    std::vector<float> best(p->n_densities, INFINITY), devBest(p->n_densities, 0.f);
    std::vector<std::mt19937> gens;
    gens.reserve(setups);
    for (size_t s = 0; s < setups; ++s) gens.emplace_back(p->seed + unsigned(s));
    std::vector<size_t> koff(p->n_kernels);
    const float nbSigmas = 1.f / p->power;
    std::vector<CalibSample> samples(setups);
    std::vector<float> before(setups);
    std::vector<int> nb_ptr, offs, term_ptr, mins;
    std::vector<qsk_term> terms;
    std::vector<float> seeds, radii, scores;
    std::vector<unsigned> origins, index, which;
    long long searches = 0;
    const auto t0 = std::chrono::steady_clock::now();
    // samples are drawn on host threads (each setup owns its generator, so the
    // draws do not depend on the thread count), then gathered in setup order
    std::vector<std::vector<qsk_term>> sterms(setups);
    const unsigned nthreads = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    auto draw_range = [&](size_t s0, size_t s1) {
        for (size_t s = s0; s < s1; ++s) {
            samples[s].search = false;
            sterms[s].clear();
            const size_t ni = s % p->n_configs, ki = (s / p->n_configs) % p->n_kernels,
                         di = s / (size_t(p->n_configs) * p->n_kernels);
            const float eb = float(cum[s * K] / ns[s * K]);
            const float db = float(std::sqrt(cum2[s * K] / ns[s * K] - eb * eb));
            before[s] = eb;
            if (ns[s * K] > p->min_iterations && (eb - nbSigmas * db) > (best[di] + nbSigmas * devBest[di])) continue;
            samples[s] = calib_draw(p, tpl, ntpl, p->counts + ni * p->n_counts, p->n_counts, p->densities[di], gens[s]);
            const CalibSample &S = samples[s];
            if (!S.search) continue;
            // the sample's pattern as terms (the simulation's conversion)
            const unsigned *kd = p->kernel_dims + ki * nd;
            const int n = int(S.offs.size() / size_t(nd));
            for (int j = 0; j < n; ++j) {
                for (int v = 0; v < nvar; ++v) {
                    const float val = S.vals[size_t(j) * nvar + v];
                    if (std::isnan(val)) continue;
                    const float wgt = calib_weight(nd, kd, p->kernel_nvar[ki], p->kernels[ki], &S.offs[size_t(j) * nd], v);
                    if (wgt == 0.f) continue;
                    qsk_term t;
                    t.neighbour = j;
                    t.layer = v;
                    if (p->types[v] == 0) {
                        t.op = QSK_OP_SQLIN;
                        t.a = -wgt;
                        t.b = 2.f * (wgt * val);
                    } else {
                        t.op = QSK_OP_EQ;
                        t.a = wgt;
                        t.b = val;
                    }
                    sterms[s].push_back(t);
                }
            }
        }
    };
    for (unsigned it = 0; it < p->max_iterations && rc == QSK_OK; ++it) {
        nb_ptr.assign(1, 0);
        term_ptr.assign(1, 0);
        offs.clear();
        terms.clear();
        seeds.clear();
        radii.clear();
        origins.clear();
        which.clear();
        if (nthreads > 1 && setups >= 64) {
            std::vector<std::thread> pool;
            const size_t chunk = (setups + nthreads - 1) / nthreads;
            for (unsigned t = 0; t < nthreads; ++t) {
                const size_t s0 = size_t(t) * chunk, s1 = std::min(setups, s0 + chunk);
                if (s0 < s1) pool.emplace_back(draw_range, s0, s1);
            }
            for (auto &th : pool) th.join();
        } else {
            draw_range(0, setups);
        }
        for (size_t s = 0; s < setups; ++s) {
            const CalibSample &S = samples[s];
            if (!S.search) continue;
            terms.insert(terms.end(), sterms[s].begin(), sterms[s].end());
            offs.insert(offs.end(), S.offs.begin(), S.offs.end());
            nb_ptr.push_back(int(offs.size() / size_t(nd)));
            term_ptr.push_back(int(terms.size()));
            seeds.push_back(S.seed);
            origins.push_back(S.cell);
            radii.push_back(radius);
            which.push_back(unsigned(s));
        }
        const int B = int(which.size());
        if (B > 0) {
            scores.resize(size_t(B) * K);
            index.resize(size_t(B) * K);
            mins.resize(size_t(B) * nd);
            rc = pattern_batch_impl(w, B, nb_ptr.data(), offs.data(), term_ptr.data(), terms.data(), unsigned(K),
                                    seeds.data(), scores.data(), index.data(), mins.data(), nullptr, origins.data(),
                                    radii.data());
            if (rc != QSK_OK) break;
            searches += B;
        }
        for (int b = 0; b < B; ++b) {
            const size_t s = which[b];
            const size_t di = s / (size_t(p->n_configs) * p->n_kernels);
            const CalibSample &S = samples[s];
            for (size_t i = 0; i < K; ++i) {
                const unsigned pos = qsk_index_to_position(ti, &mins[size_t(b) * nd], index[size_t(b) * K + i]);
                // the reference reads _data[index] of the raw array (one value per
                // cell for single-variable TIs)
                const double e = double(std::pow(std::fabs(p->ti[pos] - p->ti[S.cell]), p->power));
                cum[s * K + i] += e;
                cum2[s * K + i] += e * e;
                ns[s * K + i]++;
            }
            const float ea = float(cum[s * K] / ns[s * K]);
            if (before[s] > ea && best[di] > ea) {
                best[di] = ea;
                devBest[di] = float(std::sqrt(cum2[s * K] / ns[s * K] - ea * ea));
            }
        }
        if (p->max_seconds > 0.f && std::isfinite(p->max_seconds) &&
            std::chrono::duration_cast<std::chrono::seconds>(std::chrono::steady_clock::now() - t0).count() > p->max_seconds)
            break;
    }
    if (rc == QSK_OK) {
        for (size_t i = 0; i < setups * K; ++i) {
            const float m = float(cum[i] / ns[i]);
            mean_error[i] = std::pow(m, 1.f / p->power);
            dev_error[i] = float(std::pow(cum2[i] / ns[i] - m * m, 0.5 / double(p->power)));
            n_samples[i] = ns[i];
        }
        if (n_searches) *n_searches = searches;
    }
    qsk_worker_destroy(w);
    qsk_ti_destroy(ti);
    return rc;
}

}  // extern "C"
