/*
 * Test infrastructure only — the CPU oracle for the QuickSampling (QS)
 * per-node hot path.  It restates, in this project's own code, the G2S
 * reference algorithm for a vector (all variables at once) QS simulation:
 *
 *   search template          G2S src/qs.cpp:1010-1137, include/DataImage.hpp:433-490
 *   path, per-node seeds     G2S src/qs.cpp:975,1159-1201,1250-1258,1604-1641
 *   neighbour gathering      G2S include/simulation.hpp:447-537
 *   weights / constant       G2S include/quantileSamplingModule.hpp:368-457
 *   layers and coefficients  G2S include/DataImage.hpp:538-599,626-710
 *   mismatch map + border    G2S src/CPUThreadDevice.cpp:349-490 (direct sum here,
 *                            not FFT: in FP32 with a fixed term order, and in FP64)
 *   k-best with reservoir    G2S include/fKb.hpp:58-92,121-132,907-954,
 *                            include/quantileSamplingModule.hpp:45-49,525-557
 *   draw                     G2S include/quantileSamplingModule.hpp:90-126,
 *                            src/CPUThreadDevice.cpp:257-268, include/simulation.hpp:556-666
 *   local controls           G2S include/simulation.hpp:337-358,447-507 (-n per variable,
 *                            -ni, -kii with one template and weight kernel per -ki file,
 *                            -kvi), include/quantileSamplingModule.hpp:90-113,
 *                            src/qs.cpp:1010-1137,1281-1292
 *
 * The FP32 map uses exactly the term order and the fused multiply-adds that
 * the CUDA kernels use, so the GPU path can be checked bit for bit; the FP64
 * map gives the exact reference scores used to classify near-ties.  Only the
 * tests, the smoke check and the CPU-baseline leg of bench.py load this
 * library; the product never does.
 */
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <numeric>
#include <random>
#include <vector>

namespace {

/* ------------------------------------------------------------------ */
/* problem description                                                 */
/* ------------------------------------------------------------------ */
struct Grid {
    int nd = 0;
    unsigned dims[8] = {0};
    int nvar = 0;
    size_t cells() const {
        size_t c = 1;
        for (int i = 0; i < nd; ++i) c *= dims[i];
        return c;
    }
};

/* x-fastest flat index of a coordinate vector */
static inline long flat(const Grid &g, const int *c) {
    long f = 0;
    for (int d = g.nd - 1; d >= 0; --d) f = f * long(g.dims[d]) + c[d];
    return f;
}

static inline void coords(const Grid &g, long f, int *c) {
    for (int d = 0; d < g.nd; ++d) {
        c[d] = int(f % long(g.dims[d]));
        f /= long(g.dims[d]);
    }
}

/* ------------------------------------------------------------------ */
/* a1: search template                                                 */
/* ------------------------------------------------------------------ */
/* Offsets of the kernel box, in the generation order of G2S
 * src/qs.cpp:1055-1080, kernel-NaN offsets removed (:1107-1128), then sorted
 * nearest first with the reference's (unstable) std::sort on -|o|^2
 * (:1085-1089,1130-1135). */
std::vector<std::vector<int>> make_template(int nd, const unsigned *kdims, const float *kernel, int knvar) {
    std::vector<std::vector<int>> pos;
    pos.push_back(std::vector<int>());
    for (int i = 0; i < nd; ++i) {
        size_t orig = pos.size();
        int half = (int(kdims[i]) + 1) / 2;
        pos.resize(orig * (2 * half - 1));
        for (size_t k = 0; k < orig; ++k) pos[k].push_back(0);
        for (int j = 1; j < half; ++j) {
            std::copy(pos.begin(), pos.begin() + orig, pos.begin() + orig * (2 * j - 1));
            std::copy(pos.begin(), pos.begin() + orig, pos.begin() + orig * (2 * j));
            for (size_t k = orig * (2 * j - 1); k < orig * (2 * j); ++k) pos[k][i] = j;
            for (size_t k = orig * (2 * j); k < orig * (2 * j + 1); ++k) pos[k][i] = -j;
        }
    }
    if (kernel) {
        Grid kg;
        kg.nd = nd;
        for (int d = 0; d < nd; ++d) kg.dims[d] = kdims[d];
        std::vector<std::vector<int>> kept;
        for (auto &v : pos) {
            int c[8];
            for (int d = 0; d < nd; ++d) c[d] = int((kdims[d] - 1) / 2) + v[d];
            if (!std::isnan(kernel[size_t(flat(kg, c)) * knvar + 0])) kept.push_back(v);
        }
        pos.swap(kept);
    }
    std::sort(pos.begin(), pos.end(), [](const std::vector<int> &a, const std::vector<int> &b) {
        float da = 0.f, db = 0.f;
        for (size_t i = 0; i < a.size(); ++i) da += float(a[i] * a[i]);
        for (size_t i = 0; i < b.size(); ++i) db += float(b[i] * b[i]);
        return -da > -db;
    });
    return pos;
}

/* ------------------------------------------------------------------ */
/* a2: path and seeds                                                  */
/* ------------------------------------------------------------------ */
struct Path {
    std::vector<unsigned> order;   /* cell index per path position, informed cells first */
    std::vector<float> seeds;      /* U[0,1) per path position (not offset by begin) */
    unsigned begin = 0;            /* number of fully informed cells */
    std::vector<unsigned> posterior; /* per cell: path order, 0 for informed, UINT_MAX never */
};

Path make_path(const Grid &di, const float *dival, unsigned seed) {
    Path p;
    std::mt19937 gen(seed);
    const size_t n = di.cells();
    p.order.resize(n);
    std::iota(p.order.begin(), p.order.end(), 0u);
    unsigned begin = 0;
    for (size_t i = 0; i < n; ++i) {
        bool set = true;
        for (int v = 0; v < di.nvar; ++v)
            if (std::isnan(dival[i * di.nvar + v])) set = false;
        if (set) {
            std::swap(p.order[begin], p.order[i]);
            begin++;
        }
    }
    std::shuffle(p.order.begin() + begin, p.order.end(), gen);
    std::uniform_real_distribution<float> u(0.f, 1.f);
    p.seeds.resize(n);
    for (size_t i = 0; i < n; ++i) {
        p.seeds[i] = u(gen);
        if (p.seeds[i] == 1.f) p.seeds[i] = u(gen);
    }
    p.begin = begin;
    p.posterior.assign(n, UINT_MAX);
    for (size_t i = 0; i < n; ++i) {
        bool withNan = false;
        for (int v = 0; v < di.nvar; ++v) withNan |= std::isnan(dival[i * di.nvar + v]);
        if (!withNan) p.posterior[i] = 0;
    }
    for (size_t i = 0; i < n - begin; ++i) p.posterior[p.order[begin + i]] = unsigned(i);
    return p;
}

/* -fs: the path runs over (cell, variable) values: informed values first,
 * the rest shuffled by the same generator, one seed per value
 * (src/qs.cpp:1159-1183,1250-1258,1614-1638) */
Path make_path_full(const Grid &di, const float *dival, unsigned seed) {
    Path p;
    std::mt19937 gen(seed);
    const size_t n = di.cells() * size_t(di.nvar);
    p.order.resize(n);
    std::iota(p.order.begin(), p.order.end(), 0u);
    unsigned begin = 0;
    for (size_t i = 0; i < n; ++i)
        if (!std::isnan(dival[i])) {
            std::swap(p.order[begin], p.order[i]);
            begin++;
        }
    std::shuffle(p.order.begin() + begin, p.order.end(), gen);
    std::uniform_real_distribution<float> u(0.f, 1.f);
    p.seeds.resize(n);
    for (size_t i = 0; i < n; ++i) {
        p.seeds[i] = u(gen);
        if (p.seeds[i] == 1.f) p.seeds[i] = u(gen);
    }
    p.begin = begin;
    p.posterior.assign(n, UINT_MAX);
    for (size_t i = 0; i < n; ++i)
        if (!std::isnan(dival[i])) p.posterior[i] = 0;
    for (size_t i = begin; i < n; ++i) p.posterior[p.order[i]] = unsigned(i - begin);
    return p;
}

/* ------------------------------------------------------------------ */
/* a6: neighbours of one path node                                     */
/* ------------------------------------------------------------------ */
/* Walk the sorted template; accept an offset when the cell is inside the
 * grid and its path order is <= the node's (the node itself included),
 * until n cells are accepted (single neighbour count for all variables). */
int neighbours(const Grid &di, const std::vector<std::vector<int>> &tpl, const unsigned *posterior, unsigned cell,
               unsigned order, int n, int *out_tpl_index, unsigned *out_cell) {
    int c0[8], c[8];
    coords(di, long(cell), c0);
    int cnt = 0;
    for (size_t t = 0; t < tpl.size() && cnt < n; ++t) {
        bool ok = true;
        for (int d = 0; d < di.nd; ++d) {
            c[d] = c0[d] + tpl[t][d];
            ok &= (c[d] >= 0) && (c[d] < int(di.dims[d]));
        }
        if (!ok) continue;
        unsigned nc = unsigned(flat(di, c));
        if (posterior[nc] <= order) {
            out_tpl_index[cnt] = int(t);
            out_cell[cnt] = nc;
            cnt++;
        }
    }
    return cnt;
}

/* ------------------------------------------------------------------ */
/* a8/a9: per-node terms and the map                                   */
/* ------------------------------------------------------------------ */
struct Term {
    long off;      /* flat TI offset of the neighbour (src strides) */
    int var;       /* variable */
    int cat;       /* 1 categorical */
    float a;       /* continuous: -w (TI^2 term); categorical: w */
    float b;       /* continuous: 2*(w*v) (TI term); categorical: category code v */
    float cm;      /* missing-data mode: coefficient of the mask layer, -((w*v)*v) */
    float cw;      /* missing-data mode: weight added to the overlap ("cross") sum */
    double w, v;   /* exact weight and value for the FP64 map */
};

struct Node {
    std::vector<Term> terms;
    int mn[8], mx[8];
    bool incomplete = false;   /* the TI has missing values: cross-measurement scoring */
};

/* kernel weight for offset o and variable v (uniform 1 when kernel==nullptr);
 * the weight lookup centres the kernel at dims/2
 * (quantileSamplingModule.hpp:362-366), unlike the template (dims-1)/2. */
static inline float kweight(const Grid &kg, const float *kernel, const int *o, int v) {
    if (!kernel) return 1.f;
    int c[8];
    for (int d = 0; d < kg.nd; ++d) {
        c[d] = int(kg.dims[d] / 2) + o[d];
        if (c[d] < 0 || c[d] >= int(kg.dims[d])) return 0.f;
    }
    return kernel[size_t(flat(kg, c)) * kg.nvar + (v % kg.nvar)];
}

Node build_node(const Grid &ti, const int *types, const Grid &kg, const float *kernel, int nnb, const int *offs /* nnb*nd */,
                const float *vals /* nnb*nvar, NaN allowed */) {
    Node nd;
    for (int d = 0; d < ti.nd; ++d) nd.mn[d] = nd.mx[d] = 0;
    for (int j = 0; j < nnb; ++j)
        for (int d = 0; d < ti.nd; ++d) {
            nd.mn[d] = std::min(nd.mn[d], offs[j * ti.nd + d]);
            nd.mx[d] = std::max(nd.mx[d], offs[j * ti.nd + d]);
        }
    long strides[8];
    long s = 1;
    for (int d = 0; d < ti.nd; ++d) { strides[d] = s; s *= ti.dims[d]; }
    for (int j = 0; j < nnb; ++j) {
        long off = 0;
        for (int d = 0; d < ti.nd; ++d) off += long(offs[j * ti.nd + d]) * strides[d];
        for (int v = 0; v < ti.nvar; ++v) {
            float val = vals[j * ti.nvar + v];
            if (std::isnan(val)) continue;            /* weight 0 (quantileSamplingModule.hpp:378-392) */
            float w = kweight(kg, kernel, offs + j * ti.nd, v);
            if (w == 0.f) continue;
            Term t;
            t.off = off; t.var = v; t.cat = types[v];
            t.w = w; t.v = val;
            if (types[v] == 0) { t.a = -w; t.b = 2.f * (w * val); }
            else { t.a = w; t.b = val; }
            /* P2 = (w*v)*v on the mask layer with coefficient -1, and the
             * XMeasurement matrix adds P0 = w on the mask layer
             * (DataImage.hpp:640-660, quantileSamplingModule.hpp:398-402) */
            t.cm = -((w * val) * val);
            t.cw = w;
            nd.terms.push_back(t);
        }
    }
    return nd;
}

/* scan geometry of the (flipped) correlation space: fft == src here */
struct Scan {
    int nd;
    long fft[8], lo[8], stride[8];
    long N;
};

Scan make_scan(const Grid &ti, const Node &nd) {
    Scan sc;
    sc.nd = ti.nd;
    long s = 1;
    for (int d = 0; d < ti.nd; ++d) {
        sc.fft[d] = ti.dims[d];
        sc.stride[d] = s;
        s *= ti.dims[d];
        /* first fft-(src-(max-min)) entries along d are invalid (CPUThreadDevice.cpp:454-477) */
        sc.lo[d] = sc.fft[d] - (long(ti.dims[d]) - (nd.mx[d] - nd.mn[d]));
    }
    sc.N = s;
    return sc;
}

/* TI flat index of the pattern centre for scan index m (inverse of the
 * flipped layout, CPUThreadDevice.cpp:257-268 without the wrap). Returns
 * false when m is masked. */
static inline bool centre_of(const Scan &sc, const Grid &ti, const Node &nd, long m, long *p) {
    long pf = 0;
    bool ok = true;
    for (int d = sc.nd - 1; d >= 0; --d) {
        long md = (m / sc.stride[d]) % sc.fft[d];
        ok &= md >= sc.lo[d];
        long pd = sc.fft[d] - 1 - nd.mn[d] - md;
        pf = pf * long(ti.dims[d]) + pd;
    }
    *p = pf;
    return ok;
}

/* FP32 map in the kernels' fixed term order (terms in neighbour order, each
 * neighbour's variables in order; continuous: acc=fma(-w,t*t,acc);
 * acc=fma(2wv,t,acc); categorical: acc+=w when t==v). */
void map_fp32(const Grid &ti, const float *tival, const Node &nd, const Scan &sc, float *out) {
    for (long m = 0; m < sc.N; ++m) {
        long p;
        if (!centre_of(sc, ti, nd, m, &p)) { out[m] = nd.incomplete ? NAN : -INFINITY; continue; }
        if (nd.incomplete) {
            /* regular and cross outputs (CPUThreadDevice.cpp:426-444), the cross
             * output masked by the centre (CPUThreadDevice.cpp:501-524), then
             * -|S / c^4|, -inf where c == 0 (quantileSamplingModule.hpp:507-516) */
            float reg = 0.f, cross = 0.f;
            for (const Term &t : nd.terms) {
                float xr = tival[size_t(p + t.off) * ti.nvar + t.var];
                float mask = std::isnan(xr) ? 0.f : 1.f;
                float x = std::isnan(xr) ? 0.f : xr;
                reg = std::fmaf(t.a, x * x, reg);
                reg = std::fmaf(t.b, x, reg);
                reg = std::fmaf(t.cm, mask, reg);
                cross = std::fmaf(t.cw, mask, cross);
            }
            float cmask = std::isnan(tival[size_t(p) * ti.nvar + 0]) ? 0.f : 1.f;
            float c = cross * cmask;
            float e = -std::fabs(reg / (((c * c) * c) * c));
            if (c == 0.0f) e = -INFINITY;
            out[m] = e;
            continue;
        }
        float acc = 0.f;
        for (const Term &t : nd.terms) {
            float x = tival[size_t(p + t.off) * ti.nvar + t.var];
            if (t.cat) {
                if (x == t.b) acc = acc + t.a;
            } else {
                if (std::isnan(x)) x = 0.f;   /* layers store NaN as 0 (DataImage.hpp:554-559) */
                float x2 = x * x;
                acc = std::fmaf(t.a, x2, acc);
                acc = std::fmaf(t.b, x, acc);
            }
        }
        out[m] = acc;
    }
}

/* FP64 map: S = sum_j w_j * (2 v_j t - t^2) (continuous, i.e. -w(v-t)^2 without
 * the constant) and sum_j w_j [t==v_j] (categorical); scale = sum w (v^2+t^2)
 * or sum w. */
void map_fp64(const Grid &ti, const float *tival, const Node &nd, const Scan &sc, double *out, double *scale) {
    for (long m = 0; m < sc.N; ++m) {
        long p;
        if (!centre_of(sc, ti, nd, m, &p)) { out[m] = -INFINITY; if (scale) scale[m] = 0; continue; }
        if (nd.incomplete) {
            double reg = 0.0, cross = 0.0;
            for (const Term &t : nd.terms) {
                double xr = tival[size_t(p + t.off) * ti.nvar + t.var];
                if (std::isnan(xr)) continue;
                reg += t.w * (2.0 * t.v * xr - xr * xr - t.v * t.v);
                cross += t.w;
            }
            if (std::isnan(tival[size_t(p) * ti.nvar + 0])) cross = 0.0;
            double e = cross == 0.0 ? -INFINITY : -std::fabs(reg / (cross * cross * cross * cross));
            out[m] = e;
            if (scale) scale[m] = std::fabs(e);
            continue;
        }
        double acc = 0.0, sc2 = 0.0;
        for (const Term &t : nd.terms) {
            double x = tival[size_t(p + t.off) * ti.nvar + t.var];
            if (t.cat) {
                if (float(x) == float(t.v)) acc += t.w;
                sc2 += t.w;
            } else {
                if (std::isnan(x)) x = 0.0;
                acc += t.w * (2.0 * t.v * x - x * x);
                sc2 += t.w * (t.v * t.v + x * x);
            }
        }
        out[m] = acc;
        if (scale) scale[m] = sc2;
    }
}

/* ------------------------------------------------------------------ */
/* a10: k-biggest with the reference's reservoir tie-breaking          */
/* ------------------------------------------------------------------ */
static inline unsigned seed_from_unit_float(float seed) {
    if (!std::isfinite(seed) || seed <= 0.f) return 0;
    if (seed >= 1.f) return std::numeric_limits<unsigned>::max();
    return static_cast<unsigned>(std::floor(static_cast<double>(seed) * static_cast<double>(std::numeric_limits<unsigned>::max())));
}

template <typename R>
static inline void add_value(const float *data, unsigned short k, float *out, unsigned *pos, R &gen, unsigned &cpt,
                             unsigned i) {
    short position = short(k - 2);
    short likeLast = short(k - 2);
    while (likeLast > -1 && out[k - 1] == out[likeLast]) likeLast--;
    int xes = k - likeLast - 1;
    int x = k - xes + int(std::floor(double(gen() * float(xes))));
    std::swap(pos[x], pos[k - 1]);
    if (data[i] > out[k - 1]) {
        if (xes == 1) cpt = 0;
        else cpt++;
        while (position > -1 && data[i] > out[position]) {
            out[position + 1] = out[position];
            pos[position + 1] = pos[position];
            position--;
        }
        out[position + 1] = data[i];
        pos[position + 1] = i;
    } else {
        cpt++;
        if (float(unsigned(xes) + cpt) * gen() < float(xes)) pos[position + 1] = i;
    }
}

/* fKst::findKBiggest(data, N, k, out, pos, rng) followed by the merge loop
 * of quantileSamplingModule.hpp:546-557 for one chunk (threadRatio 1). */
void kbiggest(const float *data, unsigned N, unsigned short k, float seed, float *out, unsigned *pos) {
    std::mt19937 generator;
    generator.seed(seed_from_unit_float(seed) + 0);
    std::uniform_real_distribution<float> distribution(0.0, 1.0);
    auto rng = std::bind(distribution, std::ref(generator));
    std::vector<float> o(k, -INFINITY);
    std::vector<unsigned> p(k, UINT_MAX);
    unsigned cpt = 0;
    for (unsigned i = 0; i < N; ++i)
        if (data[i] >= o[k - 1]) add_value(data, k, o.data(), p.data(), rng, cpt, i);
    for (int j = 0; j < k; ++j) {
        unsigned best = 0;
        for (unsigned l = 1; l < k; ++l)
            if (o[l] > o[best]) best = l;
        out[j] = o[best];
        pos[j] = p[best];
        o[best] = -INFINITY;
    }
}

/* ------------------------------------------------------------------ */
/* a11-a13: draw                                                       */
/* ------------------------------------------------------------------ */
/* quantileSamplingModule.hpp:113 as compiled in the reference (ceil and
 * floor resolve to the double overloads there). */
static inline unsigned selected_index(float seed, float localk, unsigned vectorSize) {
    return unsigned(int(std::floor(double(seed * localk) * (std::ceil(double(float(vectorSize) / localk)) / vectorSize))));
}

/* CPUThreadDevice.cpp:257-268 */
static inline unsigned index_to_position(const Scan &sc, const Grid &ti, const Node &nd, unsigned index) {
    unsigned position = 0;
    unsigned div = unsigned(sc.N);
    for (int i = sc.nd - 1; i >= 0; --i) {
        div /= unsigned(sc.fft[i]);
        position = position * ti.dims[i] +
                   ((unsigned(sc.fft[i]) - (index / div) % unsigned(sc.fft[i]) - nd.mn[i] - 1) + ti.dims[i]) % ti.dims[i];
    }
    return position;
}

struct NodeResult {
    double probe_cross; /* missing-data mode: overlap weight sum at a probed TI cell */
    unsigned ti_cell;   /* chosen TI cell */
    int near_tie;       /* FP64 top-(K+1) adjacent gap within tol*scale */
    int marginal;       /* drawn from the marginal (no informed neighbour) */
    double gap_min;     /* smallest relative adjacent gap among the FP64 top-(K+1) */
    float top_score[8];
    unsigned top_index[8];
};

/* one weight kernel and its sorted search template */
struct KernelTpl {
    Grid kg;
    const float *kernel = nullptr;   /* nullptr: uniform 1 */
    std::vector<std::vector<int>> tpl;
};

struct Problem {
    Grid ti, di, kg;
    const float *tival = nullptr;
    const int *types = nullptr;
    const float *kernel = nullptr;
    std::vector<KernelTpl> kernels;      /* index 0: the main kernel; -kii selects one */
    std::vector<int> n_per_var;          /* -n n1 n2 ... (size 1: one count for all variables) */
    int ni_vars = 0;                     /* -ni: counts per cell */
    const float *ni = nullptr;
    const float *kvi = nullptr;          /* -kvi: candidate count per cell (<= 0: k) */
    const float *kii = nullptr;          /* -kii: kernel index per cell */
    int n = 0;
    float k = 1.f;
    double tol = 1e-5;
    bool incomplete = false;   /* some TI value is NaN */
    bool no_verbatim = false;  /* -nV */
    std::vector<long> complete_prefix;  /* complete TI cells in [0..c] (missing-data marginal draw) */
};

/* CPUThreadDevice::cvtPositionToIndex (CPUThreadDevice.cpp:270-284), unsigned arithmetic */
static inline unsigned position_to_index(const Scan &sc, const Grid &ti, const Node &nd, unsigned position) {
    unsigned index = 0;
    unsigned div = 1;
    for (int i = sc.nd - 1; i >= 0; --i) div *= ti.dims[i];
    for (int i = sc.nd - 1; i >= 0; --i) {
        div /= ti.dims[i];
        index = index * unsigned(sc.fft[i]) +
                (unsigned(sc.fft[i]) - (position / div + unsigned(nd.mn[i])) % ti.dims[i] - 1u);
    }
    return index;
}

void fp64_gap(const Problem &P, const Node &nd, const Scan &sc, int K, NodeResult &r);

/* one node, given the current state of the grid */
NodeResult run_node(const Problem &P, const Path &path, const float *state, const unsigned *id_state,
                    unsigned idx_path, bool want_fp64, bool own_cell_unknown, long probe_cell = -1) {
    NodeResult r;
    std::memset(&r, 0, sizeof(r));
    const Grid &di = P.di;
    unsigned cell = path.order[path.begin + idx_path];
    unsigned order = path.posterior[cell];
    float seed = path.seeds[idx_path];
    /* local controls (simulation.hpp:337-358): neighbour count per variable,
     * kernel (template + weights), candidate count */
    std::vector<int> nnb = P.n_per_var;
    if (P.ni) {
        nnb.assign(size_t(P.ni_vars), 0);
        for (int q = 0; q < P.ni_vars; ++q) nnb[q] = int(P.ni[size_t(cell) * P.ni_vars + q]);
    }
    int ki = P.kii ? int(P.kii[cell]) : 0;
    const KernelTpl &KT = P.kernels[size_t(ki)];
    float localk = P.kvi ? P.kvi[cell] : 0.f;
    if (localk <= 0.f) localk = P.k;
    /* every accepted cell counts for each variable still below its count;
     * with more than one count the walk also keeps the next informed cell
     * (values all dropped) before it stops (simulation.hpp:447-507) */
    int nmax = 0;
    for (int v = 0; v < di.nvar; ++v) nmax = std::max(nmax, nnb[size_t(v) % nnb.size()]);
    const int nlim = nmax + (nnb.size() > 1 ? 1 : 0);
    const std::vector<std::vector<int>> &tpl = KT.tpl;
    std::vector<int> tix(size_t(std::max(nlim, 1)));
    std::vector<unsigned> ncell(size_t(std::max(nlim, 1)));
    int cnt = neighbours(di, tpl, path.posterior.data(), cell, order, nlim, tix.data(), ncell.data());
    auto value = [&](unsigned c, int v) -> float {
        if (own_cell_unknown && c == cell) return NAN;
        return state[size_t(c) * di.nvar + v];
    };
    bool withDataInCenter = false;
    for (int v = 0; v < di.nvar; ++v) withDataInCenter |= !std::isnan(value(cell, v));
    if (cnt <= 1 && !withDataInCenter) {
        /* marginal draw (simulation.hpp:586-655), single TI */
        unsigned cells = unsigned(P.ti.cells());
        unsigned position = unsigned(int(std::floor(double(seed * float(cells)))));
        bool hasNaN = false;
        for (int v = 0; v < P.ti.nvar; ++v) hasNaN |= std::isnan(P.tival[size_t(position) * P.ti.nvar + v]);
        if (hasNaN) {
            /* NaN-safe draw: position = floor(seed*(complete/nvar))*nvar, first cell
             * whose running count of complete cells reaches it */
            unsigned complete = unsigned(P.complete_prefix.back());
            unsigned pos2 = unsigned(int(std::floor(double(seed * float(complete / unsigned(P.ti.nvar)))))) *
                            unsigned(P.ti.nvar);
            long k = std::lower_bound(P.complete_prefix.begin(), P.complete_prefix.end(), long(pos2)) -
                     P.complete_prefix.begin();
            position = unsigned(k);
        }
        r.ti_cell = position;
        r.marginal = 1;
        return r;
    }
    std::vector<int> offs(size_t(cnt) * di.nd);
    std::vector<float> vals(size_t(cnt) * di.nvar);
    for (int j = 0; j < cnt; ++j) {
        for (int d = 0; d < di.nd; ++d) offs[j * di.nd + d] = tpl[tix[j]][d];
        for (int v = 0; v < di.nvar; ++v)
            vals[j * di.nvar + v] = j < nnb[size_t(v) % nnb.size()] ? value(ncell[j], v) : NAN;
    }
    Node nd = build_node(P.ti, P.types, KT.kg, KT.kernel, cnt, offs.data(), vals.data());
    nd.incomplete = P.incomplete;
    Scan sc = make_scan(P.ti, nd);
    if (probe_cell >= 0 && P.incomplete) {
        /* exact overlap weight (cross output times the centre mask) at the
         * probed candidate centre */
        double cross = 0.0;
        long pc = probe_cell;
        bool inside = true;
        long rem = pc;
        int cc[8];
        for (int d = 0; d < P.ti.nd; ++d) { cc[d] = int(rem % P.ti.dims[d]); rem /= P.ti.dims[d]; }
        for (int j = 0; j < cnt && inside; ++j) {
            bool in = true;
            long f = 0, st = 1;
            for (int d = 0; d < P.ti.nd; ++d) {
                int c = cc[d] + offs[j * di.nd + d];
                in &= c >= 0 && c < int(P.ti.dims[d]);
                f += long(c) * st;
                st *= P.ti.dims[d];
            }
            if (!in) { inside = false; break; }
            for (int v = 0; v < P.ti.nvar; ++v) {
                float val = vals[j * di.nvar + v];
                if (std::isnan(val)) continue;
                if (!std::isnan(P.tival[size_t(f) * P.ti.nvar + v])) cross += kweight(KT.kg, KT.kernel, offs.data() + j * di.nd, v);
            }
        }
        if (std::isnan(P.tival[size_t(pc) * P.ti.nvar])) cross = 0.0;
        r.probe_cross = inside ? cross : -1.0;
    }
    std::vector<float> map(sc.N);
    map_fp32(P.ti, P.tival, nd, sc, map.data());
    if (P.no_verbatim && cnt > 1) {
        /* the TI position continuing neighbour 1's own source is excluded
         * (simulation.hpp:556-583, quantileSamplingModule.hpp:518-523) */
        unsigned src = id_state[ncell[1]];
        long rem = long(src);
        long pf = 0, stride = 1;
        for (int d = 0; d < P.ti.nd; ++d) {
            int dim = int(P.ti.dims[d]);
            int c = int(rem % dim) - offs[1 * di.nd + d];
            rem /= dim;
            c = ((c % dim) + dim) % dim;
            pf += long(c) * stride;
            stride *= dim;
        }
        unsigned ex = position_to_index(sc, P.ti, nd, unsigned(pf));
        if (ex < unsigned(sc.N)) map[ex] = -INFINITY;
    }
    unsigned short K = (unsigned short)int(std::ceil(localk));
    std::vector<float> ev(K);
    std::vector<unsigned> ep(K);
    kbiggest(map.data(), unsigned(sc.N), K, seed, ev.data(), ep.data());
    /* sample(): sort the K candidates by score (std::sort), draw */
    std::vector<unsigned> lp(K);
    std::iota(lp.begin(), lp.end(), 0u);
    const float *errors = ev.data();
    std::sort(lp.begin(), lp.end(), [errors](unsigned a, unsigned b) { return errors[a] > errors[b]; });
    unsigned sel = selected_index(seed, localk, 1);
    unsigned enc = ep[lp[sel]];
    r.ti_cell = index_to_position(sc, P.ti, nd, enc);
    for (int j = 0; j < K && j < 8; ++j) { r.top_score[j] = ev[lp[j]]; r.top_index[j] = ep[lp[j]]; }
    if (want_fp64) fp64_gap(P, nd, sc, K, r);
    return r;
}

/* FP64 map of the node: smallest adjacent gap among its top-(K+1) scores,
 * relative to the term scale (continuous) or the scores (missing data) */
void fp64_gap(const Problem &P, const Node &nd, const Scan &sc, int K, NodeResult &r) {
    {
        std::vector<double> m64(sc.N), s64(sc.N);
        map_fp64(P.ti, P.tival, nd, sc, m64.data(), s64.data());
        std::vector<long> ord(sc.N);
        std::iota(ord.begin(), ord.end(), 0L);
        size_t top = std::min<size_t>(size_t(K) + 1, ord.size());
        std::partial_sort(ord.begin(), ord.begin() + top, ord.end(),
                          [&](long a, long b) { return m64[a] > m64[b]; });
        double scale = 0.0;
        for (size_t j = 0; j < top; ++j) scale = std::max(scale, s64[ord[j]]);
        double gmin = INFINITY;
        for (size_t j = 0; j + 1 < top; ++j) {
            double g = m64[ord[j]] - m64[ord[j + 1]];
            gmin = std::min(gmin, scale > 0 ? g / scale : g);
        }
        if (nd.incomplete) {
            /* scores are -|S/c^4|: relative gaps */
            gmin = INFINITY;
            for (size_t j = 0; j + 1 < top; ++j) {
                double a = m64[ord[j]], b2 = m64[ord[j + 1]];
                double g = a - b2;
                double sc2 = std::max(std::fabs(a), std::fabs(b2));
                gmin = std::min(gmin, std::isfinite(g) && sc2 > 0 ? g / sc2 : (a == b2 ? 0.0 : INFINITY));
            }
        }
        r.gap_min = gmin;
        r.near_tie = gmin <= P.tol;
    }
}

/* -fs: one value (cell, variable) per path node (simulation.hpp:712-1024).
 * A cell is taken when some variable still needs neighbours and its value
 * there was simulated strictly before this node (posterior < order); only
 * those variables carry values.  The draw writes the node's variable only;
 * without two neighbours it draws from the marginal. */
NodeResult run_node_full(const Problem &P, const Path &path, const float *state, unsigned idx_path, bool want_fp64) {
    NodeResult r;
    std::memset(&r, 0, sizeof(r));
    const Grid &di = P.di;
    const int nvar = di.nvar;
    unsigned value = path.order[path.begin + idx_path];
    unsigned cell = value / unsigned(nvar), var = value % unsigned(nvar);
    unsigned order = path.posterior[value];
    float seed = path.seeds[idx_path];
    std::vector<int> nnb = P.n_per_var;
    if (P.ni) {
        nnb.assign(size_t(P.ni_vars), 0);
        for (int q = 0; q < P.ni_vars; ++q) nnb[q] = int(P.ni[size_t(cell) * P.ni_vars + q]);
    }
    int ki = P.kii ? int(P.kii[cell]) : 0;
    const KernelTpl &KT = P.kernels[size_t(ki)];
    float localk = P.kvi ? P.kvi[size_t(cell) * nvar + var] : 0.f;
    if (localk <= 0.f) localk = P.k;
    std::vector<int> count(size_t(nvar), 0);
    std::vector<int> offs;
    std::vector<float> vals;
    int c0[8], c[8];
    coords(di, long(cell), c0);
    int cnt = 0;
    for (size_t t = 0; t < KT.tpl.size(); ++t) {
        bool need = false;
        for (int v = 0; v < nvar; ++v) need |= count[v] < nnb[size_t(v) % nnb.size()];
        if (!need && nnb.size() == 1) break;
        bool ok = true;
        for (int d = 0; d < di.nd; ++d) {
            c[d] = c0[d] + KT.tpl[t][d];
            ok &= (c[d] >= 0) && (c[d] < int(di.dims[d]));
        }
        if (!ok) continue;
        unsigned nc = unsigned(flat(di, c));
        bool add = false;
        for (int v = 0; v < nvar; ++v)
            add |= count[v] < nnb[size_t(v) % nnb.size()] && path.posterior[size_t(nc) * nvar + v] < order;
        if (!add) continue;
        for (int d = 0; d < di.nd; ++d) offs.push_back(KT.tpl[t][d]);
        for (int v = 0; v < nvar; ++v) {
            if (count[v] < nnb[size_t(v) % nnb.size()] && path.posterior[size_t(nc) * nvar + v] < order) {
                vals.push_back(state[size_t(nc) * nvar + v]);
                count[v]++;
            } else {
                vals.push_back(NAN);
            }
        }
        cnt++;
    }
    if (cnt <= 1) {
        /* marginal draw of the node's variable (simulation.hpp:965-1014), complete TI */
        r.ti_cell = unsigned(int(std::floor(double(seed * float(unsigned(P.ti.cells()))))));
        r.marginal = 1;
        return r;
    }
    Node nd = build_node(P.ti, P.types, KT.kg, KT.kernel, cnt, offs.data(), vals.data());
    Scan sc = make_scan(P.ti, nd);
    std::vector<float> map(sc.N);
    map_fp32(P.ti, P.tival, nd, sc, map.data());
    unsigned short K = (unsigned short)int(std::ceil(localk));
    std::vector<float> ev(K);
    std::vector<unsigned> ep(K);
    kbiggest(map.data(), unsigned(sc.N), K, seed, ev.data(), ep.data());
    std::vector<unsigned> lp(K);
    std::iota(lp.begin(), lp.end(), 0u);
    const float *errors = ev.data();
    std::sort(lp.begin(), lp.end(), [errors](unsigned a, unsigned b) { return errors[a] > errors[b]; });
    unsigned sel = selected_index(seed, localk, 1);
    r.ti_cell = index_to_position(sc, P.ti, nd, ep[lp[sel]]);
    if (want_fp64) fp64_gap(P, nd, sc, K, r);
    return r;
}

/* Several training images (-ti with more than one grid), one node, as G2S
 * runs it with one accelerator device per TI (src/qs.cpp:1560-1598):
 *  - no informed neighbour and no centre value: the marginal draw over the
 *    TIs' cells laid end to end (simulation.hpp:586-610);
 *  - otherwise every TI (or only the cell's TI of the -ii image,
 *    simulation.hpp:560, samplingModule.hpp:70-73; QS leaves nodes without
 *    neighbours to the marginal draw) reports its K best with the same seed
 *    (quantileSamplingModule.hpp:455-575), scored as the CUDA device reports
 *    them: the map plus the constant delta = sum over continuous variables
 *    and informed neighbours of -1 * (w * v * v) in the reference's float
 *    order (quantileSamplingModule.hpp:412-457, DataImage.hpp:660-676);
 *  - the TIs x K candidates are sorted by score with std::sort (the same
 *    call and comparator as quantileSamplingModule.hpp:101-104), the rank
 *    drawn with the TI count (:113) names the TI (rank / K) and the
 *    candidate.
 * Complete TIs only. */
struct MultiResult {
    unsigned ti;
    unsigned cell;
    int marginal;
    int near_tie;   /* FP64: an adjacent gap among the merged top-(K+1) within tol of the term scale */
};

MultiResult run_node_multi(const std::vector<Grid> &tis, const std::vector<const float *> &tivals, const Grid &di,
                           const int *types, const KernelTpl &KT, int n, float k, const Path &path, const float *state,
                           unsigned idx_path, const float *ii, bool own_cell_unknown, bool want_fp64, double tol) {
    MultiResult r{0u, 0u, 0, 0};
    const unsigned cell = path.order[path.begin + idx_path];
    const unsigned order = path.posterior[cell];
    const float seed = path.seeds[idx_path];
    const int nvar = di.nvar;
    auto value = [&](unsigned c, int v) -> float {
        if (own_cell_unknown && c == cell) return NAN;
        return state[size_t(c) * nvar + v];
    };
    std::vector<int> tix(size_t(std::max(n, 1)));
    std::vector<unsigned> ncell(size_t(std::max(n, 1)));
    const int cnt = neighbours(di, KT.tpl, path.posterior.data(), cell, order, n, tix.data(), ncell.data());
    bool withDataInCenter = false;
    for (int v = 0; v < nvar; ++v) withDataInCenter |= !std::isnan(value(cell, v));
    if (cnt <= 1 && !withDataInCenter) {
        r.marginal = 1;
        unsigned cumulated = 0;
        for (const Grid &t : tis) cumulated += unsigned(t.cells()) * unsigned(nvar);
        const unsigned position = unsigned(int(std::floor(double(seed * float(cumulated / unsigned(nvar))))));
        cumulated = 0;
        for (size_t t = 0; t < tis.size(); ++t) {
            const unsigned size = unsigned(tis[t].cells()) * unsigned(nvar);
            if (position * unsigned(nvar) < cumulated + size) {
                r.ti = unsigned(t);
                r.cell = position - cumulated / unsigned(nvar);
                break;
            }
            cumulated += size;
        }
        return r;
    }
    std::vector<int> offs(size_t(cnt) * di.nd);
    std::vector<float> vals(size_t(cnt) * nvar);
    for (int j = 0; j < cnt; ++j) {
        for (int d = 0; d < di.nd; ++d) offs[j * di.nd + d] = KT.tpl[tix[j]][d];
        for (int v = 0; v < nvar; ++v) vals[j * nvar + v] = value(ncell[j], v);
    }
    float delta = 0.f;
    for (int i = 0; i < nvar; ++i) {
        if (types[i] != 0) continue;
        for (int j = 0; j < cnt; ++j) {
            const float v = vals[j * nvar + i];
            if (std::isnan(v)) continue;
            const float w = kweight(KT.kg, KT.kernel, offs.data() + j * di.nd, i);
            delta += -1.f * (w * v * v);
        }
    }
    const int req = ii ? int(ii[cell]) : -1;
    const unsigned nti = unsigned(tis.size());
    const unsigned short K = (unsigned short)int(std::ceil(k));
    std::vector<float> errors(size_t(nti) * K, -INFINITY);
    std::vector<unsigned> enc(size_t(nti) * K, 0u);
    std::vector<Node> nodes(nti);
    std::vector<Scan> scans(nti);
    for (unsigned t = 0; t < nti; ++t) {
        if (req >= 0 && int(t) != req) continue;
        nodes[t] = build_node(tis[t], types, KT.kg, KT.kernel, cnt, offs.data(), vals.data());
        scans[t] = make_scan(tis[t], nodes[t]);
        std::vector<float> map(scans[t].N);
        map_fp32(tis[t], tivals[t], nodes[t], scans[t], map.data());
        std::vector<float> ev(K);
        std::vector<unsigned> ep(K);
        kbiggest(map.data(), unsigned(scans[t].N), K, seed, ev.data(), ep.data());
        for (int j = 0; j < K; ++j) {
            errors[size_t(t) * K + j] = ev[j] + delta;
            enc[size_t(t) * K + j] = ep[j];
        }
    }
    std::vector<unsigned> lp(errors.size());
    std::iota(lp.begin(), lp.end(), 0u);
    const float *e = errors.data();
    std::sort(lp.begin(), lp.end(), [e](unsigned a, unsigned b) { return e[a] > e[b]; });
    const unsigned sel = selected_index(seed, k, nti);
    const unsigned t = lp[sel] / K;
    r.ti = t;
    r.cell = index_to_position(scans[t], tis[t], nodes[t], enc[lp[sel]]);
    if (want_fp64) {
        /* the FP64 scores of every updated TI's top K+1, merged */
        std::vector<std::pair<double, double>> top;   /* (score, term scale) */
        for (unsigned u = 0; u < nti; ++u) {
            if (req >= 0 && int(u) != req) continue;
            std::vector<double> m64(scans[u].N), s64(scans[u].N);
            map_fp64(tis[u], tivals[u], nodes[u], scans[u], m64.data(), s64.data());
            std::vector<long> ord(scans[u].N);
            std::iota(ord.begin(), ord.end(), 0L);
            const size_t m = std::min<size_t>(size_t(K) + 1, ord.size());
            std::partial_sort(ord.begin(), ord.begin() + m, ord.end(), [&](long a, long b) { return m64[a] > m64[b]; });
            for (size_t j = 0; j < m; ++j) top.push_back({m64[ord[j]], s64[ord[j]]});
        }
        std::sort(top.begin(), top.end(), [](const std::pair<double, double> &a, const std::pair<double, double> &b) {
            return a.first > b.first;
        });
        const size_t m = std::min<size_t>(size_t(K) + 1, top.size());
        double scale = 0.0;
        for (size_t j = 0; j < m; ++j) scale = std::max(scale, top[j].second);
        double gmin = INFINITY;
        for (size_t j = 0; j + 1 < m; ++j) {
            const double g = top[j].first - top[j + 1].first;
            gmin = std::min(gmin, scale > 0 ? g / scale : g);
        }
        r.near_tie = gmin <= tol;
    }
    return r;
}

}  // namespace

extern "C" {

/* Sorted search template: writes up to cap offsets (nd ints each); returns count. */
int orc_template(int nd, const unsigned *kdims, const float *kernel, int knvar, int *out, int cap) {
    auto tpl = make_template(nd, kdims, kernel, knvar);
    int n = int(tpl.size());
    for (int i = 0; i < n && i < cap; ++i)
        for (int d = 0; d < nd; ++d) out[i * nd + d] = tpl[i][d];
    return n;
}

/* Path, seeds and posterior order.  Returns begin (number of informed cells). */
int orc_path(int nd, const unsigned *dims, int nvar, const float *dival, unsigned seed, unsigned *order, float *seeds,
             unsigned *posterior) {
    Grid g;
    g.nd = nd;
    g.nvar = nvar;
    for (int d = 0; d < nd; ++d) g.dims[d] = dims[d];
    Path p = make_path(g, dival, seed);
    std::copy(p.order.begin(), p.order.end(), order);
    std::copy(p.seeds.begin(), p.seeds.end(), seeds);
    std::copy(p.posterior.begin(), p.posterior.end(), posterior);
    return int(p.begin);
}

/* -fs path over (cell, variable) values; arrays of cells*nvar entries. */
int orc_path_full(int nd, const unsigned *dims, int nvar, const float *dival, unsigned seed, unsigned *order,
                  float *seeds, unsigned *posterior) {
    Grid g;
    g.nd = nd;
    g.nvar = nvar;
    for (int d = 0; d < nd; ++d) g.dims[d] = dims[d];
    Path p = make_path_full(g, dival, seed);
    std::copy(p.order.begin(), p.order.end(), order);
    std::copy(p.seeds.begin(), p.seeds.end(), seeds);
    std::copy(p.posterior.begin(), p.posterior.end(), posterior);
    return int(p.begin);
}

/* k-biggest with reservoir ties on an arbitrary array (fKb.hpp semantics). */
void orc_kbiggest(const float *data, unsigned N, unsigned k, float seed, float *out, unsigned *pos) {
    kbiggest(data, N, (unsigned short)k, seed, out, pos);
}

/* MT19937 + uniform_real_distribution<float> stream, for RNG unit tests */
void orc_rng(unsigned s, int n, float *out) {
    std::mt19937 g;
    g.seed(s);
    std::uniform_real_distribution<float> d(0.0, 1.0);
    for (int i = 0; i < n; ++i) out[i] = d(g);
}

unsigned orc_seed_from_unit_float(float seed) { return seed_from_unit_float(seed); }
unsigned orc_selected_index(float seed, float k, unsigned nti) { return selected_index(seed, k, nti); }

/*
 * Vector QS simulation (mode 0) or teacher-forced per-node evaluation (mode 1).
 *   ti: nd dims (x first) ti_dims, nvar interleaved variables, types[v] 0/1
 *   di: di_dims, nvar, NaN = to simulate (mode 0: simulated in place;
 *       mode 1: the completed grid whose values are used as neighbour values,
 *       with each node's own cell treated as not yet simulated)
 *   di_init: mode 1 only, the grid before simulation (defines the path)
 *   kernel: optional weights (kdims, nvar interleaved); nullptr = uniform 1
 *           of size min(TI/2+1)
 * Outputs per path node (size = cells - begin): chosen TI cell, near-tie
 * flag (if want_fp64), marginal flag.  out_id (mode 0): per DI cell the
 * reference's index image (TI cell * nTI + TI, nTI = 1).
 * Returns the number of path nodes.
 */
/* local controls of orc_simulate_ex (all optional, per DI cell where noted) */
struct OrcControls {
    int n_counts;                  /* entries of n_per_var (-n n1 n2 ...); 0: n for every variable */
    const int *n_per_var;
    int ni_vars;                   /* -ni: counts per cell (0: none) */
    const float *ni;
    const float *kvi;              /* -kvi */
    int n_kernels;                 /* kernels for -kii (0: the main kernel only) */
    const unsigned *kernels_dims;  /* n_kernels * nd */
    const float *const *kernels;
    const float *kii;              /* -kii */
    int full;                      /* -fs: one path node per (cell, variable) value */
};

long orc_simulate_ex(int mode, int nd, const unsigned *ti_dims, int nvar, const int *types, const float *ti,
                     const unsigned *di_dims, float *di, const float *di_init, const unsigned *kdims, const float *kernel,
                     int n, float k, unsigned seed, int want_fp64, double tol, long node_begin, long node_end,
                     unsigned *out_cell, int *out_near_tie, int *out_marginal, double *out_gap, unsigned *out_id,
                     int no_verbatim, const unsigned *id_init, const unsigned *probe, double *probe_cross,
                     const OrcControls *ctl) {
    Problem P;
    P.ti.nd = P.di.nd = P.kg.nd = nd;
    P.ti.nvar = P.di.nvar = nvar;
    for (int d = 0; d < nd; ++d) { P.ti.dims[d] = ti_dims[d]; P.di.dims[d] = di_dims[d]; }
    /* missing values: cells with any NaN variable become all-NaN for vector
     * simulation (src/qs.cpp:1436-1467) */
    std::vector<float> tiw(ti, ti + P.ti.cells() * nvar);
    for (size_t c = 0; c < P.ti.cells(); ++c) {
        bool hasNan = false;
        for (int v = 0; v < nvar; ++v) hasNan |= std::isnan(tiw[c * nvar + v]);
        if (hasNan) {
            P.incomplete = true;
            for (int v = 0; v < nvar; ++v) tiw[c * nvar + v] = NAN;
        }
    }
    if (P.incomplete)
        for (int v = 0; v < nvar; ++v)
            if (types[v] != 0) return -2;  /* categorical + missing values: undefined in the reference */
    P.complete_prefix.resize(P.ti.cells());
    long run = 0;
    for (size_t c = 0; c < P.ti.cells(); ++c) {
        run += std::isnan(tiw[c * nvar]) ? 0 : 1;
        P.complete_prefix[c] = run;
    }
    P.tival = tiw.data();
    P.types = types;
    P.n = n;
    P.k = k;
    P.tol = tol;
    P.no_verbatim = no_verbatim != 0;
    if (kernel) {
        P.kernel = kernel;
        P.kg.nvar = nvar;
        for (int d = 0; d < nd; ++d) P.kg.dims[d] = kdims[d];
    } else {
        P.kg.nvar = nvar;
        for (int d = 0; d < nd; ++d) P.kg.dims[d] = std::min(ti_dims[d] / 2 + 1, ti_dims[d]);
    }
    /* kernels: the main one, or the -kii list (src/qs.cpp:1000-1042) */
    if (ctl && ctl->n_kernels > 0) {
        for (int q = 0; q < ctl->n_kernels; ++q) {
            KernelTpl kt;
            kt.kg.nd = nd;
            kt.kg.nvar = nvar;
            for (int d = 0; d < nd; ++d) kt.kg.dims[d] = ctl->kernels_dims[q * nd + d];
            kt.kernel = ctl->kernels[q];
            P.kernels.push_back(kt);
        }
    } else {
        KernelTpl kt;
        kt.kg = P.kg;
        kt.kernel = P.kernel;
        P.kernels.push_back(kt);
    }
    for (auto &kt : P.kernels) kt.tpl = make_template(nd, kt.kg.dims, kt.kernel, nvar);
    P.n_per_var.assign(1, n);
    if (ctl && ctl->n_counts > 0) P.n_per_var.assign(ctl->n_per_var, ctl->n_per_var + ctl->n_counts);
    if (ctl && ctl->ni_vars > 0 && ctl->ni) {
        P.ni_vars = ctl->ni_vars;
        P.ni = ctl->ni;
    }
    if (ctl && ctl->kii) {
        P.kii = ctl->kii;
        for (size_t c = 0; c < P.di.cells(); ++c) {
            int q = int(P.kii[c]);
            if (q < 0 || q >= int(P.kernels.size())) return -3;
        }
    }
    if (ctl && ctl->kvi) {
        /* -kvi: the module's k becomes max(k, max kvi) (src/qs.cpp:1281-1292) */
        P.kvi = ctl->kvi;
        float kb = std::isnan(k) || k <= 0.f ? 1.f : k;
        for (size_t c = 0; c < P.di.cells(); ++c) kb = std::max(kb, P.kvi[c]);
        P.k = kb;
    }
    std::vector<float> state(di, di + P.di.cells() * nvar);
    if (ctl && ctl->full) {
        /* -fs (complete TIs only here); out_id holds one index per value.
         * mode 1: every node against the completed grid (values visible by
         * posterior order only, so no masking is needed) */
        if (P.incomplete) return -4;
        Path fp = make_path_full(P.di, di_init ? di_init : state.data(), seed);
        long fnodes = long(P.di.cells()) * nvar - long(fp.begin);
        if (node_end < 0 || node_end > fnodes) node_end = fnodes;
        if (mode == 1) {
#pragma omp parallel for schedule(dynamic, 16)
            for (long i = node_begin; i < node_end; ++i) {
                NodeResult r = run_node_full(P, fp, state.data(), unsigned(i), want_fp64 != 0);
                long o = i - node_begin;
                if (out_cell) out_cell[o] = r.ti_cell;
                if (out_near_tie) out_near_tie[o] = r.near_tie;
                if (out_marginal) out_marginal[o] = r.marginal;
                if (out_gap) out_gap[o] = r.gap_min;
            }
            return fnodes;
        }
        for (long i = 0; i < node_end; ++i) {
            unsigned value = fp.order[fp.begin + i];
            NodeResult r = run_node_full(P, fp, state.data(), unsigned(i), i >= node_begin && want_fp64 != 0);
            unsigned var = value % unsigned(nvar);
            if (std::isnan(state[value])) state[value] = P.tival[size_t(r.ti_cell) * nvar + var];
            if (out_id) out_id[value] = r.ti_cell;
            if (i >= node_begin) {
                long o = i - node_begin;
                if (out_cell) out_cell[o] = r.ti_cell;
                if (out_near_tie) out_near_tie[o] = r.near_tie;
                if (out_marginal) out_marginal[o] = r.marginal;
                if (out_gap) out_gap[o] = r.gap_min;
            }
        }
        std::copy(state.begin(), state.end(), di);
        return fnodes;
    }
    /* the path is always built from the grid before simulation (NaN = unknown) */
    Path path = make_path(P.di, di_init ? di_init : state.data(), seed);
    long nodes = long(P.di.cells()) - long(path.begin);
    if (node_end < 0 || node_end > nodes) node_end = nodes;
    std::vector<unsigned> idw(P.di.cells(), 0u);
    if (id_init) std::copy(id_init, id_init + P.di.cells(), idw.begin());
    if (mode == 1) {
        /* teacher forcing: every path cell is "not yet simulated" at its own turn */
#pragma omp parallel for schedule(dynamic, 16)
        for (long i = node_begin; i < node_end; ++i) {
            long o = i - node_begin;
            NodeResult r = run_node(P, path, state.data(), idw.data(), unsigned(i), want_fp64 != 0, true,
                                    probe ? long(probe[o]) : -1L);
            if (probe_cross) probe_cross[o] = r.probe_cross;
            if (out_cell) out_cell[o] = r.ti_cell;
            if (out_near_tie) out_near_tie[o] = r.near_tie;
            if (out_marginal) out_marginal[o] = r.marginal;
            if (out_gap) out_gap[o] = r.gap_min;
        }
        return nodes;
    }
    for (long i = 0; i < node_end; ++i) {
        unsigned cell = path.order[path.begin + i];
        bool active = i >= node_begin;
        NodeResult r = run_node(P, path, state.data(), idw.data(), unsigned(i), active && want_fp64 != 0, false);
        for (int v = 0; v < nvar; ++v)
            if (std::isnan(state[size_t(cell) * nvar + v])) state[size_t(cell) * nvar + v] = P.tival[size_t(r.ti_cell) * nvar + v];
        idw[cell] = r.ti_cell;
        if (out_id) out_id[cell] = r.ti_cell;
        if (active) {
            long o = i - node_begin;
            if (out_cell) out_cell[o] = r.ti_cell;
            if (out_near_tie) out_near_tie[o] = r.near_tie;
            if (out_marginal) out_marginal[o] = r.marginal;
            if (out_gap) out_gap[o] = r.gap_min;
        }
    }
    std::copy(state.begin(), state.end(), di);
    return nodes;
}

long orc_simulate(int mode, int nd, const unsigned *ti_dims, int nvar, const int *types, const float *ti,
                  const unsigned *di_dims, float *di, const float *di_init, const unsigned *kdims, const float *kernel, int n, float k,
                  unsigned seed, int want_fp64, double tol, long node_begin, long node_end, unsigned *out_cell,
                  int *out_near_tie, int *out_marginal, double *out_gap, unsigned *out_id, int no_verbatim,
                  const unsigned *id_init, const unsigned *probe, double *probe_cross) {
    return orc_simulate_ex(mode, nd, ti_dims, nvar, types, ti, di_dims, di, di_init, kdims, kernel, n, k, seed, want_fp64,
                           tol, node_begin, node_end, out_cell, out_near_tie, out_marginal, out_gap, out_id, no_verbatim,
                           id_init, probe, probe_cross, nullptr);
}

/* FP32 and FP64 maps of one explicit pattern (offsets/values) against the TI
 * in scan (flipped) order, plus the node's min/max; for map-level tests. */
long orc_pattern_map(int nd, const unsigned *ti_dims, int nvar, const int *types, const float *ti, int nnb,
                     const int *offs, const float *vals, float *out32, double *out64, double *scale, int *mn, int *mx) {
    Grid g, kg;
    g.nd = kg.nd = nd;
    g.nvar = kg.nvar = nvar;
    for (int d = 0; d < nd; ++d) g.dims[d] = ti_dims[d];
    Node node = build_node(g, types, kg, nullptr, nnb, offs, vals);
    Scan sc = make_scan(g, node);
    if (out32) map_fp32(g, ti, node, sc, out32);
    if (out64) map_fp64(g, ti, node, sc, out64, scale);
    for (int d = 0; d < nd; ++d) { mn[d] = node.mn[d]; mx[d] = node.mx[d]; }
    return sc.N;
}


/* Vector QS simulation with several training images: nti TIs of the same
 * nvar (dims per TI, x first, in ti_dims[t*nd..]), the default uniform
 * kernel of size min over TIs of (dims/2 + 1) per dimension
 * (src/qs.cpp:1010-1042) or the given kernel, one neighbour count; ii
 * (optional, per DI cell) the -ii image.  mode 0: di simulated in place,
 * out_id the index image, TI cell * nti + TI (simulation.hpp:658); mode 1:
 * every path node teacher-forced against the completed grid di, the path
 * built from di_init, with the FP64 near-tie flag (tol of the term scale).
 * Per path node: chosen TI and TI cell, near-tie and marginal flags.
 * Returns the path nodes, -1 for a TI with missing values. */
long orc_simulate_multi(int mode, int nd, int nti, const unsigned *ti_dims, int nvar, const int *types,
                        const float *const *ti, const unsigned *di_dims, float *di, const float *di_init,
                        const unsigned *kdims, const float *kernel, int n, float k, unsigned seed, const float *ii,
                        double tol, unsigned *out_id, unsigned *out_ti, unsigned *out_cell, int *out_near_tie,
                        int *out_marginal) {
    std::vector<Grid> tis((size_t)nti);
    std::vector<const float *> tivals((size_t)nti);
    for (int t = 0; t < nti; ++t) {
        tis[t].nd = nd;
        tis[t].nvar = nvar;
        for (int d = 0; d < nd; ++d) tis[t].dims[d] = ti_dims[t * nd + d];
        tivals[t] = ti[t];
        for (size_t c = 0; c < tis[t].cells() * size_t(nvar); ++c)
            if (std::isnan(ti[t][c])) return -1;
    }
    Grid dg;
    dg.nd = nd;
    dg.nvar = nvar;
    for (int d = 0; d < nd; ++d) dg.dims[d] = di_dims[d];
    KernelTpl KT;
    KT.kg.nd = nd;
    KT.kg.nvar = nvar;
    if (kernel) {
        KT.kernel = kernel;
        for (int d = 0; d < nd; ++d) KT.kg.dims[d] = kdims[d];
    } else {
        for (int d = 0; d < nd; ++d) {
            unsigned m = ti_dims[d];
            for (int t = 0; t < nti; ++t) m = std::min(m, ti_dims[t * nd + d] / 2 + 1);
            KT.kg.dims[d] = m;
        }
    }
    KT.tpl = make_template(nd, KT.kg.dims, KT.kernel, nvar);
    std::vector<float> state(di, di + dg.cells() * nvar);
    Path path = make_path(dg, di_init ? di_init : state.data(), seed);
    const long nodes = long(dg.cells()) - long(path.begin);
    auto record = [&](long i, const MultiResult &r) {
        if (out_ti) out_ti[i] = r.ti;
        if (out_cell) out_cell[i] = r.cell;
        if (out_near_tie) out_near_tie[i] = r.near_tie;
        if (out_marginal) out_marginal[i] = r.marginal;
    };
    if (mode == 1) {
        /* teacher forcing: every node against the completed grid di, its own
         * cell not yet simulated */
#pragma omp parallel for schedule(dynamic, 16)
        for (long i = 0; i < nodes; ++i)
            record(i, run_node_multi(tis, tivals, dg, types, KT, n, k, path, state.data(), unsigned(i), ii, true,
                                     true, tol));
        return nodes;
    }
    for (long i = 0; i < nodes; ++i) {
        const unsigned cell = path.order[path.begin + i];
        MultiResult r = run_node_multi(tis, tivals, dg, types, KT, n, k, path, state.data(), unsigned(i), ii, false,
                                       false, tol);
        for (int v = 0; v < nvar; ++v)
            if (std::isnan(state[size_t(cell) * nvar + v]))
                state[size_t(cell) * nvar + v] = tivals[r.ti][size_t(r.cell) * nvar + v];
        if (out_id) out_id[cell] = r.cell * unsigned(nti) + r.ti;
        record(i, r);
    }
    std::copy(state.begin(), state.end(), di);
    return nodes;
}
}  /* extern "C" */

/* ------------------------------------------------------------------ */
/* f3: auto_qs calibration                                             */
/* ------------------------------------------------------------------ */
namespace {

/* scan indices marked by CPUThreadDevice::setValueInErrorArrayWithRadius
 * (src/CPUThreadDevice.cpp:310-342): level L > 1 steps i in [-r, r],
 * r = ceil(sqrt(R2 - d2)), by fft[L-1]; level 1 steps by fft[0] and marks
 * (pos + i*fft[0] + N) % N; unsigned 32-bit arithmetic throughout. */
void radius_marks(const Scan &sc, unsigned pos, float R2, int level, unsigned d2, std::vector<unsigned> &out) {
    if (!(float(d2) <= R2)) return;
    const int r = int(std::ceil(std::sqrt(double(R2 - float(d2)))));
    const unsigned s = unsigned(sc.N);
    for (int i = -r; i <= r; ++i) {
        if (level == 1) out.push_back((pos + unsigned(i * int(sc.fft[0])) + s) % s);
        else radius_marks(sc, pos + unsigned(i * int(sc.fft[level - 1])), R2, level - 1, d2 + unsigned(i * i), out);
    }
}

/* QuantileSamplingModule::distribution for one TI on the CPU device
 * (include/quantileSamplingModule.hpp:128-175,342-600): the weighted map, the
 * verbatim exclusion of the origin (one index, or the radius marks), the
 * k-biggest with reservoir ties, the stable order by score, TI positions. */
struct Dist {
    std::vector<float> score;
    std::vector<unsigned> index, position;
    int mn[8];
};

Dist distribution(const Grid &g, const int *types, const float *ti, const Grid &kg, const float *kernel, int nnb,
                  const int *offs, const float *vals, unsigned k, float seed, unsigned origin, float radius,
                  std::vector<float> *map_out = nullptr, std::vector<double> *m64 = nullptr,
                  std::vector<double> *scale = nullptr) {
    Node node = build_node(g, types, kg, kernel, nnb, offs, vals);
    Scan sc = make_scan(g, node);
    std::vector<float> m(size_t(sc.N));
    map_fp32(g, ti, node, sc, m.data());
    if (origin != UINT_MAX) {
        const unsigned idx = position_to_index(sc, g, node, origin);
        if (radius < 1.f) {
            if (idx < unsigned(sc.N)) m[idx] = -INFINITY;
        } else {
            std::vector<unsigned> marks;
            radius_marks(sc, idx, radius * radius, sc.nd, 0, marks);
            for (unsigned q : marks) m[q] = -INFINITY;
        }
    }
    Dist d;
    d.score.resize(k);
    d.index.resize(k);
    kbiggest(m.data(), unsigned(sc.N), (unsigned short)k, seed, d.score.data(), d.index.data());
    d.position.resize(k);
    for (unsigned i = 0; i < k; ++i) d.position[i] = index_to_position(sc, g, node, d.index[i]);
    for (int i = 0; i < g.nd; ++i) d.mn[i] = node.mn[i];
    if (map_out) *map_out = m;
    if (m64) {
        m64->resize(size_t(sc.N));
        scale->resize(size_t(sc.N));
        map_fp64(g, ti, node, sc, m64->data(), scale->data());
    }
    return d;
}

}  /* namespace */

extern "C" {

/* One distribution() query: TI (x fastest, variables interleaved), weight
 * kernel (kdims, knvar variables), nnb neighbour offsets and values (NaN:
 * left out), k candidates, seed, origin TI cell (0xffffffff: none) and
 * exclusion radius.  Outputs k scores, scan indices, TI positions and the
 * pattern minimum; map32 (N floats, after the exclusion) and map64/scale
 * (N doubles) when not null.  Returns N. */
long orc_distribution(int nd, const unsigned *ti_dims, int nvar, const int *types, const float *ti,
                      const unsigned *kdims, int knvar, const float *kernel, int nnb, const int *offs,
                      const float *vals, unsigned k, float seed, unsigned origin, float radius, float *out_score,
                      unsigned *out_index, unsigned *out_position, int *out_min, float *map32, double *map64,
                      double *scale) {
    Grid g, kg;
    g.nd = kg.nd = nd;
    g.nvar = nvar;
    kg.nvar = knvar;
    for (int d = 0; d < nd; ++d) {
        g.dims[d] = ti_dims[d];
        kg.dims[d] = kdims[d];
    }
    std::vector<float> m32;
    std::vector<double> m64, sc;
    Dist r = distribution(g, types, ti, kg, kernel, nnb, offs, vals, k, seed, origin, radius, map32 ? &m32 : nullptr,
                          map64 ? &m64 : nullptr, map64 ? &sc : nullptr);
    for (unsigned i = 0; i < k; ++i) {
        out_score[i] = r.score[i];
        out_index[i] = r.index[i];
        out_position[i] = r.position[i];
    }
    for (int d = 0; d < nd; ++d) out_min[d] = r.mn[d];
    if (map32) std::copy(m32.begin(), m32.end(), map32);
    if (map64) {
        std::copy(m64.begin(), m64.end(), map64);
        if (scale) std::copy(sc.begin(), sc.end(), scale);
    }
    long N = 1;
    for (int d = 0; d < nd; ++d) N *= long(ti_dims[d]);
    return N;
}

}  /* extern "C" */

namespace {

/* One calibration sample of setup (neighbour counts nn, density), drawn from
 * the setup's generator: the body of the reference's loop in
 * include/calibration.hpp:113-224 up to the distribution() call. */
struct Sample {
    unsigned cell = 0;
    std::vector<int> offs;
    std::vector<float> vals;
    float seed = 0.f;
    bool search = false;
};

Sample draw_sample(const Grid &g, const float *ti, const std::vector<std::vector<int>> &tpl,
                   const std::vector<unsigned> &nn, float density, float noise, std::mt19937 &gen) {
    std::uniform_real_distribution<float> U(0.f, 1.f);
    Sample S;
    (void)int(std::floor(U(gen) * 1.f));   /* TI index: one TI */
    const unsigned dataSize = unsigned(g.cells()) * unsigned(g.nvar);
    S.cell = unsigned(std::floor(U(gen) * float(dataSize) / float(unsigned(g.nvar))));
    std::vector<unsigned> per(g.nvar, 0);
    size_t P = tpl.size(), ps = 0;
    int c0[8];
    coords(g, long(S.cell), c0);
    while ((nn.size() > 1 || S.offs.size() / size_t(g.nd) < nn[0]) && ps < P) {
        bool take = U(gen) < density;
        long dataIndex = 0;
        if (take) {
            int c[8];
            for (int d = 0; d < g.nd; ++d) {
                c[d] = c0[d] + tpl[ps][d];
                if (c[d] < 0 || c[d] >= int(g.dims[d])) take = false;
            }
            if (take) dataIndex = flat(g, c);
        }
        if (take) {
            unsigned cpt = 0;
            for (int v = 0; v < g.nvar; ++v) {
                if (per[v] < nn[v % nn.size()]) {
                    S.vals.push_back(ti[size_t(dataIndex) * g.nvar + v]);
                    cpt++;
                    per[v]++;
                } else {
                    S.vals.push_back(NAN);
                }
            }
            for (int d = 0; d < g.nd; ++d) S.offs.push_back(tpl[ps][d]);
            if (cpt == 0) break;
        }
        ps++;
    }
    if (ps >= P) return S;   /* not enough neighbours: no search */
    const size_t n = S.offs.size() / size_t(g.nd);
    if (n > 1 && noise > 0.f) {
        float fraction = noise / float(n) / 2.f;
        if (noise < 1.0f) fraction = noise / 2.f;
        for (size_t j = 0; j < n; ++j)
            if (U(gen) < fraction) {
                /* the two indices of iter_swap; a swap is symmetric, so their
                 * order of evaluation does not matter */
                const size_t a = size_t(std::floor(U(gen) * float(n)));
                const size_t b = size_t(std::floor(U(gen) * float(n)));
                for (int d = 0; d < g.nd; ++d) std::swap(S.offs[a * g.nd + d], S.offs[b * g.nd + d]);
            }
    }
    if (n > 1) {
        S.seed = U(gen);
        S.search = true;
    }
    return S;
}

}  /* namespace */

extern "C" {

/* auto_qs calibration (include/calibration.hpp:30-284, src/auto_qs.cpp:640-
 * 700), restated with the batched order of this project's GPU driver:
 * setup s = (neighbour configuration, kernel, density), x fastest, draws
 * from its own std::mt19937(seed + s); in every iteration the pruning test of
 * all setups uses the statistics as they stood when the iteration began, the
 * samples of all unpruned setups are searched, and their errors are then
 * accumulated (and the best mean error per density updated) in setup order.
 * Outputs per setup and candidate rank (max_k of them): mean error^(1/p),
 * deviation^(0.5/p) and the 16-bit sample count.  Returns the number of
 * searches. */
long orc_calibrate(int nd, const unsigned *ti_dims, int nvar, const int *types, const float *ti, int n_kernels,
                   const unsigned *kdims, const int *knvar, const float *kernels, int n_configs, int n_counts,
                   const unsigned *counts, int n_densities, const float *densities, unsigned max_k, float power,
                   float noise, unsigned max_iter, unsigned min_iter, unsigned seed, float *mean, float *dev,
                   unsigned *nsamp) {
    Grid g;
    g.nd = nd;
    g.nvar = nvar;
    for (int d = 0; d < nd; ++d) g.dims[d] = ti_dims[d];
    std::vector<Grid> kg(n_kernels);
    std::vector<const float *> kp(n_kernels);
    size_t koff = 0;
    for (int i = 0; i < n_kernels; ++i) {
        kg[i].nd = nd;
        kg[i].nvar = knvar[i];
        for (int d = 0; d < nd; ++d) kg[i].dims[d] = kdims[i * nd + d];
        kp[i] = kernels + koff;
        koff += kg[i].cells() * size_t(knvar[i]);
    }
    /* pathPosition: the box of kernel 0 nearest first (src/auto_qs.cpp:452-492) */
    const auto tpl = make_template(nd, kdims, nullptr, 1);
    const float radius = float(std::pow(double(unsigned(g.cells()) * unsigned(nvar) / unsigned(nvar)) * 0.005,
                                        1.f / float(nd)));
    const size_t setups = size_t(n_configs) * n_kernels * n_densities;
    const size_t K = max_k;
    std::vector<double> cum(setups * K, 0.0), cum2(setups * K, 0.0);
    std::vector<uint16_t> ns(setups * K, 0);
    std::vector<float> best(n_densities, INFINITY), devBest(n_densities, 0.f);
    std::vector<std::mt19937> gens;
    gens.reserve(setups);
    for (size_t s = 0; s < setups; ++s) gens.emplace_back(seed + unsigned(s));
    const float nbSigmas = 1.f / power;
    long searches = 0;
    std::vector<Sample> samples(setups);
    std::vector<float> before(setups);
    for (unsigned it = 0; it < max_iter; ++it) {
        for (size_t s = 0; s < setups; ++s) {
            samples[s].search = false;
            const size_t ni = s % n_configs, ki = (s / n_configs) % n_kernels, di = s / (size_t(n_configs) * n_kernels);
            (void)ki;
            const float eb = float(cum[s * K] / ns[s * K]);
            const float db = float(std::sqrt(cum2[s * K] / ns[s * K] - eb * eb));
            before[s] = eb;
            if (ns[s * K] > min_iter && (eb - nbSigmas * db) > (best[di] + nbSigmas * devBest[di])) continue;
            std::vector<unsigned> nn(counts + ni * n_counts, counts + (ni + 1) * n_counts);
            samples[s] = draw_sample(g, ti, tpl, nn, densities[di], noise, gens[s]);
        }
        for (size_t s = 0; s < setups; ++s) {
            const Sample &S = samples[s];
            if (!S.search) continue;
            const size_t ki = (s / n_configs) % n_kernels, di = s / (size_t(n_configs) * n_kernels);
            const int n = int(S.offs.size() / size_t(nd));
            Dist r = distribution(g, types, ti, kg[ki], kp[ki], n, S.offs.data(), S.vals.data(), max_k, S.seed, S.cell,
                                  radius);
            searches++;
            for (size_t i = 0; i < K; ++i) {
                const double e = double(std::pow(std::fabs(ti[r.position[i]] - ti[S.cell]), power));
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
    }
    for (size_t i = 0; i < setups * K; ++i) {
        const float m = float(cum[i] / ns[i]);
        mean[i] = std::pow(m, 1.f / power);
        dev[i] = float(std::pow(cum2[i] / ns[i] - m * m, 0.5 / double(power)));
        nsamp[i] = ns[i];
    }
    return searches;
}

}  /* extern "C" */
