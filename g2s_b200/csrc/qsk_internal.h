// Internal declarations shared by the host engine (qsk_host.cpp) and the
// CUDA kernels (qsk_kernels.cu) of the B200 QuickSampling path.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime_api.h>

#define QSK_MAXD 4          // grid dimensions supported
#define QSK_SEG 128         // scan positions per warp segment (32 lanes x 4)
#define QSK_KMAX 16         // largest extendK handled on device
#define QSK_CMAX 32         // categories per variable with bit planes

namespace qsk {

// Operation applied to one gathered layer value x for one term.
enum TermOp : int {
    OP_LIN = 0,    // acc = fma(a, x, acc)
    OP_SQLIN = 1,  // acc = fma(a, x*x, acc); acc = fma(b, x, acc)   (continuous variable)
    OP_EQ = 2,     // acc = (x == b) ? acc + a : acc                  (categorical variable)
    OP_LINX = 3,   // cross = fma(a, x, cross)                       (overlap output, missing data)
    OP_SQLINM = 4, // missing data: mask = !isnan(x), x0 = mask ? x : 0:
                   //   acc = fma(a, x0*x0, acc); acc = fma(b, x0, acc);
                   //   acc = fma(next.a, mask, acc); cross = fma(next.b, mask, cross)
                   // (the next term carries the two mask coefficients and is skipped)
    OP_NOP = 5,    // payload of the previous term
};

struct Term {
    int base;   // layer offset minus the neighbour's flat scan offset: address = base + m
    float a;
    float b;
    int op;
};

// Scan geometry of one training image (the reference's flipped correlation
// space, G2S src/CPUThreadDevice.cpp:257-284,454-477).
struct Geom {
    int nd;
    int fft[QSK_MAXD];       // fft size per dimension (x first)
    int src[QSK_MAXD];       // TI size per dimension
    long long sstride[QSK_MAXD];  // scan (fft) strides
    long long N;             // prod(fft)
    int nseg;                // ceil(N / QSK_SEG)
};

// Per node (batch slot) description written by the prep step.
struct Slot {
    int node;                // path index (simulation) or pattern id
    int nterms;
    int mn[QSK_MAXD];        // min neighbour offset per dim (init 0)
    int lo[QSK_MAXD];        // first valid scan coordinate per dim
    float seed;
    int sel;                 // drawn candidate rank
    int flags;               // SLOT_* bits
    unsigned cell;           // DI cell (simulation)
    int excl;                // scan index forced to -inf (-nV), -1 for none
    int cmask_base;          // missing data: centre-mask layer address minus m
    int K;                   // candidates kept (extendK = ceil(k) of this node)
    int var;                 // -fs: the node's variable (the only one written)
    // -nV with static terms: neighbour 1's cell and template index, from
    // which the map derives excl (vtpl < 0: no exclusion)
    unsigned vcell;
    int vtpl;
};

// A simulation term whose value is read when the map runs: the layer offset
// (as Term::base) and where the neighbour's value lives (src >= 0: the grid
// state at src, src < 0: the initial grid at -src - 1).  A NaN value there
// contributes nothing (the reference leaves it out of the pattern).
struct StaticTerm {
    int base;
    int src;
};

enum SlotFlags : int {
    SLOT_SKIP = 1,           // no map: marginal draw or empty pattern
    SLOT_EMIT_MASKED = 2,    // fewer than K valid positions: masked entries are candidates too
    SLOT_MISSING = 4,        // TI with missing values: score -|S/c^4| with the overlap c, border NaN
};

// Status words written by kernels (bounded waits / argument checks).
enum DevStatus : int {
    DEV_OK = 0,
    DEV_BAD_INDEX = 1,
    DEV_TOO_MANY_TERMS = 2,
    DEV_LEVEL_WAIT = 3,       // a dependency level did not appear within the wait limit
    DEV_TC_WAIT = 4,          // a tensor-core kernel's pipeline wait ran out (kernel returned early)
};

// Grid (destination image) description for the neighbour search.
struct GridDesc {
    int nd;
    int dims[QSK_MAXD];
    long long stride[QSK_MAXD];
};

struct SimPrepArgs {
    Geom g;
    GridDesc dg;
    int nvar;
    const int *types;
    const int *tpl;        // ntpl x nd offsets
    const float *wtab;     // ntpl x nvar kernel weights
    const unsigned *path;
    unsigned begin;
    const float *seeds;    // per path index
    const int *nb_count;
    const int *nb_tpl;
    const unsigned *nb_cell;
    int n;
    const float *state;    // current grid values (cells x nvar)
    const float *init;     // grid before simulation (centre values)
    const int *nodes;      // slot -> path index
    int nslots;
    float k;
    int K;
    unsigned nti;
    Slot *slots;
    Term *terms;
    int maxterms;
    int *status;
    int missing;           // TI with missing values (terms OP_SQLINM + payload)
    int mask_layer;        // layer index of the TI mask (missing data)
    int no_verbatim;       // -nV
    const unsigned *id_image;  // index image of the grid (-nV)
    // local controls (nullable): neighbour count per path node and variable,
    // candidate count per path node
    const int *node_nv;
    const float *node_k;
    int full;                       // -fs: path entries are cell values, neighbours carry nb_mask
    const unsigned char *nb_mask;
    StaticTerm *sterms = nullptr;   // k_mt_prep: slots + static terms of the batch (null: none)
};

struct MapArgs {
    Geom g;
    const float *layers;
    const Slot *slots;
    const Term *terms;
    int maxterms;
    int segs_per_cta;
    float *rec_val;   // [slot][nseg*SEG]
    int *rec_idx;
    int *rec_cnt;     // [slot][nseg]
    float *rec_max;   // [slot][nseg] largest valid score of the segment
    // verbatim exclusion with a radius: bit m of slot b's mask
    // (xmask[b * xwords + m / 32]) forces valid position m to -inf; null: none
    const unsigned *xmask = nullptr;
    long long xwords = 0;
};

// Bit-plane layout: every plane is `plane_words(N)` words, of which the
// first `plane_guard(N)` are zero and word plane_guard(N) + w holds positions
// 32w..32w+31; the guard and the zero tail make every funnel-shifted read of
// the map kernel, for any term offset, an in-bounds read without a test.
__host__ __device__ inline int plane_guard(long long N) { return int((N + 31) / 32) + 1; }
__host__ __device__ inline int plane_words(long long N) { return plane_guard(N) + int((N + 31) / 32) + 34; }

struct BitArgs {
    Geom g;
    const unsigned *planes;   // [var][QSK_CMAX+1][pw] words (slot QSK_CMAX all zero)
    int pw;                   // words per plane: plane_words(N)
    const int *ncat;          // categories per variable
    const float *catv;        // [var][QSK_CMAX] category codes
    const Slot *slots;
    const Term *terms;
    int maxterms;
    int segs_per_cta;         // 1024-position segments per CTA
    float *rec_val;
    int *rec_idx;
    int *rec_cnt;
    float *rec_max;
    // simulation with static terms (null sterms: the terms above are used):
    // values from state / init, -nV exclusion from the index image
    const StaticTerm *sterms = nullptr;
    const float *state = nullptr;
    const float *init = nullptr;
    const unsigned *id_image = nullptr;
    const int *tpl = nullptr;           // template offsets (ntpl x nd)
    int no_verbatim = 0;
    int stage_words = 0;                // shared-memory words for staged planes (set by the launcher)
};

struct ReplayArgs {
    Geom g;
    const Slot *slots;
    int nslots;
    int K;
    const float *rec_val;
    const int *rec_idx;
    const int *rec_cnt;
    const float *rec_max;
    // pattern outputs (may be null)
    float *out_val;       // [slot][K]
    unsigned *out_pos;    // [slot][K]
    // simulation outputs (may be null)
    int nvar;
    const float *ti;      // TI grid (cells x nvar)
    long long ti_cells;
    unsigned nti, ti_id;
    const int *complete_prefix;  // missing data: complete TI cells in [0..c]; null for a complete TI
    float *state;         // grid written in simulation mode (null in teacher-forced mode)
    unsigned *id_image;   // per grid cell (-fs: per cell value)
    unsigned *node_cell;  // per path index: chosen TI cell
    int full;             // -fs: write the slot's variable only
    // generator states from k_mt_prep ([slot][624]) and the draws their
    // skipped blocks stand for; null: each slot is seeded in the replay
    const unsigned *mt_state;
    const int *mt_pre;
    // replay only the slots flagged SLOT_SKIP / SLOT_EMIT_MASKED (the hash
    // select takes the others)
    int only_flagged = 0;
    // hash select: per path node, the drawn candidate's score (regret audit)
    float *drawn_score = nullptr;
    float *drawn_scale = nullptr;
    // pattern outputs: out_pos holds TI cells (cvtIndexToPosition of the
    // slot's geometry) instead of scan indices
    int out_cells = 0;
};

// several training images (batched engine): per slot, every TI's K best
// (vals / cells, [ti][slot][K], TI cells) merged and drawn as G2S does with
// one CUDA device per TI (quantileSamplingModule.hpp:90-126): scores plus the
// constant delta, stable sort of the TIs x K candidates, the slot's rank
// (drawn with the TI count) naming TI and cell; slots flagged SLOT_SKIP draw
// from the TIs' cells laid end to end (simulation.hpp:586-610); write-back of
// the value and the index image (cell * nti + TI)
#define QSK_MAX_TIS 8
struct MultiDrawArgs {
    const Slot *slots = nullptr;
    int nslots = 0;
    int K = 0;
    int nti = 0;
    int nvar = 0;
    const float *vals = nullptr;
    const unsigned *cells = nullptr;
    long long ti_stride = 0;              // entries between two TIs' blocks of vals / cells
    const float *ti[QSK_MAX_TIS] = {};    // TI grids (cells x nvar)
    long long ti_cells[QSK_MAX_TIS] = {};
    const int *types = nullptr;
    // delta: the node's neighbours and weights
    const int *nb_count = nullptr;
    const int *nb_tpl = nullptr;
    const unsigned *nb_cell = nullptr;
    int n = 0;
    const float *wtab = nullptr;          // ntpl x nvar
    const float *ii = nullptr;            // -ii: the TI each grid cell samples from (null: all)
    float *state = nullptr;
    unsigned *id_image = nullptr;
    unsigned *node_cell = nullptr;
};
cudaError_t launch_multi_draw(const MultiDrawArgs &a, cudaStream_t st);


// record the calling thread's error message (qsk_last_error) and return code
int set_error(int code, const char *fmt, ...);

// launch wrappers (qsk_kernels.cu)
cudaError_t launch_build_layers(const float *ti, int nvar, const int *types, const Geom &g, float *layers, int missing,
                                cudaStream_t st);
// node_kernel / tpl_range / node_lim: optional per-node kernel (template
// range [begin, begin+count) of the concatenated templates) and neighbour limit
cudaError_t launch_neighbours(const GridDesc &dg, const int *tpl, int ntpl, const unsigned *path, unsigned begin,
                              long long nodes, const unsigned *posterior, int n, int *nb_count, int *nb_tpl,
                              unsigned *nb_cell, const int *node_kernel, const int *tpl_range, const int *node_lim,
                              cudaStream_t st);
cudaError_t launch_neighbours_full(const GridDesc &dg, const int *tpl, int ntpl, const unsigned *path, unsigned begin,
                                   long long nodes, const unsigned *posterior, int nvar, int n, const int *node_nv,
                                   int *nb_count, int *nb_tpl, unsigned *nb_cell, unsigned char *nb_mask,
                                   const int *node_kernel, const int *tpl_range, cudaStream_t st);

// dependency levels of the path DAG (Kahn frontiers)
struct LevelArgs {
    long long nodes;
    int n;
    const int *nb_count;
    const unsigned *nb_cell;
    const unsigned char *nb_mask;  // -fs: variables each neighbour contributes (null otherwise)
    int nvar;
    const int *node_of_cell;       // per cell, or (-fs) per cell value
    int *level;         // nodes: level of each path node
    int *cursor;        // nodes
    int *tile_sum;      // ceil(nodes / 1024) + 1
    int *cnt;           // nodes + 2: nodes per level, then the node ticket
    int *level_nodes;   // nodes: grouped by level
    int *start;         // nodes + 1: level L is level_nodes[start[L] .. start[L+1])
    int *nl_out;        // 1: number of levels
    int *status;        // DevStatus
    unsigned spin_limit = 0;   // polls of one dependency before DEV_LEVEL_WAIT (0: 2^22)
    long long hold = -1;       // node whose level is never published (failure-path test), -1 none
};
cudaError_t launch_levels(const LevelArgs &a, cudaStream_t st);
cudaError_t launch_prep_sim(const SimPrepArgs &a, cudaStream_t st);
int map_segs_per_cta(const Geom &g, int nslots);
cudaError_t launch_map_records(const MapArgs &a, int nslots, int K, int maxterms_in_batch, cudaStream_t st);
cudaError_t set_map_smem_limit(int bytes);
cudaError_t launch_build_planes(const float *layers, const Geom &g, int nvar, const int *ncat, const float *catv,
                                int pw, unsigned *planes, cudaStream_t st);
int map_bits_segs_per_cta(const Geom &g, int nslots);
cudaError_t launch_map_bits(const BitArgs &a, int nslots, int K, int maxterms_in_batch, cudaStream_t st);
cudaError_t launch_replay(const ReplayArgs &a, cudaStream_t st);
// k best by (score, tie hash) over the records; slots with SLOT_SKIP or
// SLOT_EMIT_MASKED are left to launch_replay with only_flagged
cudaError_t launch_hash_select(const ReplayArgs &a, cudaStream_t st);
// exclusion masks: slot b's positions around scan index center[b] (radius[b] >= 1)
cudaError_t launch_radius_mask(const int *center, const float *radius, int nslots, const Geom &g, unsigned *mask,
                               long long xwords, cudaStream_t st);
cudaError_t launch_mt_prep(const SimPrepArgs &a, unsigned *state, int *pre, cudaStream_t st);

// ---------------------------------------------------------------------------
// tensor-core shortlist (qsk_tc.cu): D = A * P^T on tcgen05 for 128-row tiles
// of A (nodes / queries) against 256-row tiles of P (TI positions), K in
// 128-byte blocks (64 BF16 or 128 FP8 E4M3 values); per A row and position
// range the W largest scores (acc * node_scale * tile_scale + node_bias)
// whose position lies in the row's validity box are kept.
// ---------------------------------------------------------------------------
struct TcArgs {
    int n_nodes;               // live rows of A
    long long n_pos;           // live rows of P
    long long n_tiles;         // position tiles of 256 rows
    int ranges;                // position ranges (grid.y)
    int tiles_per_range;
    int kblocks;               // K blocks of A and P
    const int *tile_kblocks;   // per 128-row tile of A: K blocks used (null: kblocks)
    int k_per_block;           // elements per K block (set by the launcher)
    const float *node_scale;   // per A row (null: 1)
    const float *node_bias;    // per A row (null: 0)
    const float *pos_scale;    // per tile of 256 P rows (null: 1)
    const unsigned *node_seed; // per A row tie-break seed (null: 0)
    const int *node_box;       // per A row: x0, x1, y0, y1, z0, z1 (p valid iff x0 <= x < x1, ...)
    int X, Y;                  // P row p is TI cell (x, y, z), x fastest
    unsigned *node_thr;        // per A row, zeroed before the launch: the best heap minimum of any range
                               // (ordered score), a lower bound of the row's W-th best (null: none)
    unsigned long long *out_key;   // [row][range][W]: (ordered score << 32) | tie hash; 0 = empty
    unsigned *out_pos;             // [row][range][W]
    int *status;
};
int tc_supported_width(int w);
// kind 0: BF16 (kind::f16), 1: FP8 E4M3 (kind::f8f6f4); a_rows % 128 == 0,
// p_rows % 256 == 0, k_elems * element size % 128 == 0
// C[M x N] = A * B^T (+ bias) on the tensor cores: A (a_rows x kpad) and B
// (b_rows x kpad) BF16 K-major, a_rows a multiple of 128, b_rows of the N
// tile (tc_gemm_bn(N)), kpad of 64, padding zero; C FP32 row-major (ldc)
struct TcGemmArgs {
    int M = 0, N = 0, kpad = 0;
    float *C = nullptr;
    long long ldc = 0;
    const float *bias = nullptr;
    int *status = nullptr;   // DEV_TC_WAIT when a wait ran out
};
int tc_gemm_bn(int N);
cudaError_t launch_tc_gemm(const void *a_bf16, long long a_rows, const void *b_bf16, long long b_rows,
                           const TcGemmArgs &g, cudaStream_t st);
cudaError_t launch_tc_shortlist(int kind, int W, const void *a_mat, long long a_rows, const void *p_mat,
                                long long p_rows, long long k_elems, const TcArgs &args, cudaStream_t st);
// Tensor-core form inside the simulation.  Pattern matrix P: one row per TI
// cell p (natural order, x fastest; rows padded to 256), row length Kp with
// column j * L + l = layer l at cell p + o_j for the first T template
// offsets (0 outside the TI), in BF16 or FP8 E4M3 (rows scaled to their
// largest magnitude).  Layers: a continuous variable gives t^2 and t, a
// categorical one with C categories an indicator of each of its first C-1
// codes (a match of the last code is 1 minus the others: a node constant).
#define QSK_TC_MAXL 64
struct TcLayer {
    int var;
    int kind;     // 0: t^2, 1: t, 2: [t == code]
    float code;
};
struct TcPatternArgs {
    const float *ti;           // raw TI, cells x nvar
    int nvar, nd;
    int src[QSK_MAXD];
    long long N;               // TI cells
    long long rows;            // padded rows
    const int *tpl;            // template offsets (ntpl x nd)
    int T, L;
    TcLayer layer[QSK_TC_MAXL];
    long long Kp;
    int fmt;                   // 0 BF16, 1 FP8 E4M3
    void *P;
    float *pos_scale;          // FP8: per tile of 256 rows
};
struct TcNodeArgs {
    int nd, nvar;
    int src[QSK_MAXD];
    const int *nodes;          // slot -> path index
    int nslots;
    const unsigned *path;
    unsigned begin;
    const int *nb_count;
    const int *nb_tpl;
    const unsigned *nb_cell;
    int n;
    const int *tpl;
    const float *wtab;
    const float *state, *init, *seeds;
    const int *types;
    const int *var_layer0;     // first pattern layer of each variable
    const int *var_ncat;       // categorical: codes per variable
    const float *var_catv;     // [var][QSK_CMAX]
    int L;
    long long Kp;
    int fmt;
    void *A;                   // rows x Kp, zeroed here (rows >= nslots: the padding rows too)
    long long rows;
    unsigned *node_thr;        // the shortlist's per-node bound, zeroed here (may be null)
    float *node_scale;
    float *node_bias;          // sum of the weights of neighbours in a variable's last category
    int *node_box;
    unsigned *node_seed;
};
struct TcSelectArgs {
    Geom g;
    const Slot *slots;
    const Term *terms;
    int maxterms;
    int nslots;
    const float *layers;                 // FP32 flipped layers (exact scores)
    const unsigned long long *cand_key;  // [slot][ncand]
    const unsigned *cand_pos;
    int ncand;                           // ranges x W
    int S;                               // candidates scored exactly (<= 256)
    int fp64;                            // rank by the FP64 exact score
    const float *ti;
    int nvar;
    unsigned nti, ti_id;
    float *state;
    unsigned *id_image;
    unsigned *node_cell;
    float *drawn_score;                  // per path node: FP32 exact score of the draw
    float *drawn_scale;                  // per path node: its term scale
    unsigned *err_max;                   // float bits: largest |approx - FP64| / scale
    double *err_sum;
    unsigned long long *err_n;
    int *status;
    // learned proposal: per slot 1 when the confidence check fails (the exact
    // best of the shortlist ranks at conf_rank or later by the proposal's
    // score); null: no check
    int *fallback = nullptr;
    int conf_rank = 0;
    // > 0: the statistical check (the k-th best exact score must clear the
    // regression bound a L_out + b + conf_z sd of the positions left out;
    // range_w: heap entries per position range)
    float conf_z = 0.f;
    float conf_r2 = 0.2f;      // smallest R^2 of the fit
    int range_w = 0;
};
// FP8: rowmax is scratch of `rows` floats
cudaError_t launch_tc_pattern(const TcPatternArgs &a, float *rowmax, cudaStream_t st);
cudaError_t launch_tc_tmax(long long nodes, int n, const int *nb_count, const int *nb_tpl, int *tmax, cudaStream_t st);
cudaError_t launch_tc_nodes(const TcNodeArgs &a, cudaStream_t st);
// k_prep_sim and k_tc_nodes of one tensor-core step in one launch (rows of A
// written, not learned)
cudaError_t launch_prep_tc_nodes(const SimPrepArgs &p, const TcNodeArgs &a, cudaStream_t st);
cudaError_t launch_tc_select(const TcSelectArgs &a, cudaStream_t st);
cudaError_t launch_tc_audit(int n, const int *nodes, int K, const float *plain_val, const float *drawn_score,
                            const float *drawn_scale, float tol, unsigned long long *counts, cudaStream_t st);

// ---------------------------------------------------------------------------
// learned proposal (qsk_learn.cu): encoder inputs, FP32 GEMM and training ops
// ---------------------------------------------------------------------------
#define QSK_ENC_ENTRIES 64   // neighbourhood entries of an encoder input
struct FeatArgs {
    long long rows;
    // nodes (k_feat_nodes): path indices and their neighbour lists
    const int *nodes = nullptr;
    const unsigned *path = nullptr;
    unsigned begin = 0;
    const int *nb_count = nullptr;
    const int *nb_tpl = nullptr;
    const unsigned *nb_cell = nullptr;
    int n = 0;
    const float *state = nullptr;     // grid values (cells x nvar)
    // TI cells (k_feat_cells): cell0 + r, or cell_list[r] when given
    long long cell0 = 0;
    const unsigned *cell_list = nullptr;
    long long cells = 0;
    const float *ti = nullptr;
    int src[3] = {1, 1, 1};
    int ntpl = 0;
    // both
    const int *tpl = nullptr;         // template offsets (ntpl x nd)
    int nd = 0, nvar = 0;
    float inv_radius = 1.f;           // offsets are scaled by this
    int entries = QSK_ENC_ENTRIES;    // template offsets 1..entries represented (at most 64)
    float *out = nullptr;             // rows x (64 x (nvar + 4))
    // multi-scale stencil: at scale s, entry e sits at s x (template offset
    // e + 1); a neighbour at offset o falls in the entry whose offset is
    // round(o / s) (half away from zero), the values falling in one entry
    // averaged
    int scale = 1;                    // the rows' scale when row_scale is null
    const int *row_scale = nullptr;   // per row scale (1..nscales)
    const int *cube = nullptr;        // entry of every offset of the stencil's box (-1: none)
    int cube_lo[3] = {0, 0, 0};
    int cube_dim[3] = {1, 1, 1};
    int nscales = 1;
    float cov_min = 0.9f;             // k_node_scale: smallest scale covering this fraction of the neighbours
    int *scale_out = nullptr;         // k_node_scale: the chosen scale per row
};
cudaError_t launch_node_scale(const FeatArgs &a, cudaStream_t st);
cudaError_t launch_sgemm(int M, int N, int K, const float *A, int lda, int ta, const float *B, int ldb, int tb, float *C,
                         int ldc, float alpha, float beta, const float *bias, cudaStream_t st);
cudaError_t launch_gelu(long long n, const float *pre, float *out, cudaStream_t st);
cudaError_t launch_gelu_back(long long n, const float *pre, float *d, cudaStream_t st);
cudaError_t launch_colsum(int rows, int cols, const float *d, float *out, int accumulate, cudaStream_t st);
cudaError_t launch_infonce(int B, float tau, const float *S, float *dS, float *loss, cudaStream_t st);
cudaError_t launch_adam(long long n, float *w, const float *g, float *m, float *v, float lr, int t, cudaStream_t st);
cudaError_t launch_feat_nodes(const FeatArgs &a, cudaStream_t st);
// rows_pad x kpad BF16 copy of a rows x cols FP32 matrix (tr: of its
// transpose, src then cols x rows), zero-padded; both pads multiples of 32
cudaError_t launch_pack_bf16(int rows, int cols, const float *src, long long ld, int tr, long long rows_pad, int kpad,
                             void *dst, cudaStream_t st);
cudaError_t launch_feat_cells(const FeatArgs &a, cudaStream_t st);
cudaError_t launch_to_bf16(long long n, const float *x, uint16_t *y, cudaStream_t st);
cudaError_t launch_gather_rows(int n, int cols, const int *idx, const float *src, float *dst, cudaStream_t st);

// 32-bit mix of a node seed and a position: the tie-break part of a
// shortlist key (equal scores are ordered by it, uniformly at random over
// positions for a given seed)
__host__ __device__ inline unsigned tie_hash(unsigned seed, unsigned pos) {
    unsigned x = seed ^ (pos * 0x9E3779B9u);
    x ^= x >> 16;
    x *= 0x7FEB352Du;
    x ^= x >> 15;
    x *= 0x846CA68Bu;
    x ^= x >> 16;
    return x;
}

}  // namespace qsk
