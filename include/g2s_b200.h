/*
 * g2s_b200 — B200-native QuickSampling (QS) hot path behind a C ABI.
 *
 * Plain C: POD arguments, host pointers, int status codes; no C++ or torch
 * types cross this boundary.  Shared library: libg2s_b200.so (sm_100a).
 *
 * Every entry point names the G2S interface it replaces.  G2S binds its
 * accelerator device by dlopen("./g2s_cuda.so") and two symbols
 * (src/qs.cpp:861-911); the drop-in g2s_cuda.so of this project
 * (g2s_b200/dropin/) implements that AcceleratorDevice on top of the
 * functions below.
 *
 * Threading: a qsk_ti is immutable after creation and may be shared; a
 * qsk_worker or qsk_sim must be used by one host thread at a time.
 */
#ifndef G2S_B200_H
#define G2S_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* status codes (G2S has none: CUDA errors call exit(), .cu:45-54) */
#define QSK_OK 0
#define QSK_ERR_ARG 1          /* invalid argument / unsupported size */
#define QSK_ERR_CUDA 2         /* CUDA runtime error (message in qsk_last_error) */
#define QSK_ERR_NOMEM 3        /* device allocation failed */
#define QSK_ERR_UNSUPPORTED 4  /* feature outside the implemented path */
#define QSK_ERR_DEVICE 5       /* a kernel reported an inconsistent input */

/* term operations of a pattern: x = layer value at the neighbour's position */
#define QSK_OP_LIN 0           /* acc = fma(a, x, acc) */
#define QSK_OP_SQLIN 1         /* acc = fma(a, x*x, acc); acc = fma(b, x, acc) */
#define QSK_OP_EQ 2            /* acc = (x == b) ? acc + a : acc */
#define QSK_OP_LIN_CROSS 3     /* cross = fma(a, x, cross): the overlap output of a TI with missing values */

/* Last error message of the calling thread ("" when none). */
const char *qsk_last_error(void);

/* Number of usable CUDA devices.
 * Replaces g2s_cudaGetDeviceCount (G2S src/NvidiaGPUAcceleratorDevice.cu:26-30,
 * resolved by src/qs.cpp:876). */
int qsk_device_count(int *count);

/* ------------------------------------------------------------------------
 * Training image on one GPU (the per-device shared memory of G2S'
 * SharedMemoryManager + AcceleratorDevice::allocAndInitSharedMemory).
 * ---------------------------------------------------------------------- */
typedef struct qsk_ti qsk_ti;

/* Upload nlayers correlation layers, each prod(fft_size) floats in the
 * reference's flipped layout (DataImage::convertInput4Xcorr).
 * Replaces NvidiaGPUAcceleratorDevice::allocAndInitSharedMemory
 * (G2S src/NvidiaGPUAcceleratorDevice.cu:350-390, interface
 * include/AcceleratorDevice.hpp:46). */
int qsk_ti_create_layers(int device, int ndim, const unsigned *src_size, const unsigned *fft_size, int nlayers,
                         const float *const *layers, qsk_ti **out);

/* Upload a raw training image (x fastest, nvar interleaved variables,
 * types[v] 0 continuous / 1 categorical) and build its layers on the GPU:
 * one layer per variable (value, NaN->0, for continuous; category code for
 * categorical).  Replaces DataImage::convertInput4Xcorr + SharedMemoryManager
 * (G2S include/DataImage.hpp:538-599, src/sharedMemoryManager.cpp:26-58). */
int qsk_ti_create_grid(int device, int ndim, const unsigned *dims, int nvar, const int *types, const float *data,
                       qsk_ti **out);

/* Scan (fft) size of a TI context: writes ndim values. */
int qsk_ti_fft_size(const qsk_ti *ti, unsigned *fft_size);

/* Releases the device copy. Replaces freeSharedMemory (.cu:392-404). */
int qsk_ti_destroy(qsk_ti *ti);

/* ------------------------------------------------------------------------
 * Per-thread worker: stream + scratch for pattern queries (one per G2S path
 * thread, like one NvidiaGPUAcceleratorDevice per thread, src/qs.cpp:1577-1588).
 * ---------------------------------------------------------------------- */
typedef struct qsk_worker qsk_worker;
int qsk_worker_create(qsk_ti *ti, qsk_worker **out);
int qsk_worker_destroy(qsk_worker *w);

/* One term of a pattern: op applied to layer[layer] at the position of
 * neighbour `neighbour`, coefficients a, b (see QSK_OP_*). */
typedef struct {
    int neighbour;
    int layer;
    int op;
    float a;
    float b;
} qsk_term;

/* Mismatch map of one pattern against every TI position (terms summed in
 * the given order in FP32 with fused multiply-adds), positions whose template
 * leaves the TI set to -inf, then the k best positions with the reference's
 * reservoir tie-breaking seeded from `seed`.  Outputs: out_score[k] (map
 * values S, descending), out_index[k] (scan index in the reference's flipped
 * space, i.e. its "encodedPosition"), out_min[ndim] (pattern min offset,
 * needed by cvtIndexToPosition).
 * Replaces AcceleratorDevice::candidateForPattern + searchKBiggest
 * (G2S src/AcceleratorDevice.cpp:92-136, include/AcceleratorDevice.hpp:45,68,
 * src/NvidiaGPUAcceleratorDevice.cu:462-614,688-727), with the k-biggest
 * semantics of the CPU path (include/fKb.hpp:58-132,907-954,
 * include/quantileSamplingModule.hpp:525-557). */
int qsk_pattern_kbest(qsk_worker *w, int n_neighbours, const int *offsets, int n_terms, const qsk_term *terms,
                      unsigned k, float seed, float *out_score, unsigned *out_index, int *out_min);

/* Options of a pattern query beyond the plain map (zero-initialise):
 *   exclude_index      scan index forced to -inf before the k-best (-nV:
 *                      AcceleratorDevice::setValueInErrorArray, G2S
 *                      include/quantileSamplingModule.hpp:566-571); -1 none
 *   missing_data       1 when the TI has missing values: the score becomes
 *                      -|S / c^4| with c the QSK_OP_LIN_CROSS sum times the
 *                      centre mask, -inf where c == 0, NaN outside the border
 *                      (maskCroossErrorWithVariable + compensateMissingData,
 *                      quantileSamplingModule.hpp:559-564, .cu:617-686)
 *   centre_mask_layer  layer holding the TI mask (1 informed, 0 missing)
 *   exclude_radius     >= 1: instead of exclude_index alone, every scan index
 *                      that CPUThreadDevice::setValueInErrorArrayWithRadius
 *                      (G2S src/CPUThreadDevice.cpp:310-342) marks around it
 *                      is forced to -inf (distribution() with a verbatim
 *                      radius, quantileSamplingModule.hpp:518-523); < 1: the
 *                      single index
 * The exclusion is written after the missing-data score, over the NaN border
 * too, as the reference writes it into its error array. */
typedef struct {
    int exclude_index;
    int missing_data;
    int centre_mask_layer;
    float exclude_radius;
} qsk_pattern_opts;

int qsk_pattern_kbest_ex(qsk_worker *w, int n_neighbours, const int *offsets, int n_terms, const qsk_term *terms,
                         unsigned k, float seed, const qsk_pattern_opts *opts, float *out_score, unsigned *out_index,
                         int *out_min);

/* Batched form: B patterns in CSR form (nb_ptr[B+1] into offsets rows,
 * term_ptr[B+1] into terms; term.neighbour is relative to its pattern).
 * Outputs are B*k scores/indices and B*ndim minima. */
int qsk_pattern_kbest_batch(qsk_worker *w, int B, const int *nb_ptr, const int *offsets, const int *term_ptr,
                            const qsk_term *terms, unsigned k, const float *seeds, float *out_score,
                            unsigned *out_index, int *out_min);

/* Batched form with the verbatim exclusion of QuantileSamplingModule::
 * distribution (G2S include/quantileSamplingModule.hpp:128-175,518-523,
 * 566-571): pattern b was taken from TI cell origin[b] (0xffffffff: none);
 * with radius[b] < 1 the scan index of that cell is excluded
 * (setValueInErrorArray), otherwise every index that
 * CPUThreadDevice::setValueInErrorArrayWithRadius marks around it
 * (src/CPUThreadDevice.cpp:310-342).  radius may be null (all < 1).  The
 * auto_qs calibration queries its samples this way (include/calibration.hpp:
 * 221-224). */
int qsk_pattern_kbest_batch_verbatim(qsk_worker *w, int B, const int *nb_ptr, const int *offsets, const int *term_ptr,
                                     const qsk_term *terms, unsigned k, const float *seeds, const unsigned *origin,
                                     const float *radius, float *out_score, unsigned *out_index, int *out_min);

/* auto_qs calibration (G2S src/auto_qs.cpp:640-700, include/calibration.hpp:
 * 30-284) on the batched engine: for every setup (neighbour configuration,
 * kernel, density) samples are drawn from the TI itself (a random cell, its
 * template neighbours kept with probability `density`, optional position
 * noise), searched with the verbatim exclusion of the cell's own
 * neighbourhood (radius (cells*0.005)^(1/ndim)), and the error
 * |TI[match] - TI[cell]|^power of each of the max_k candidates is
 * accumulated; setups whose mean error is worse than the density's best by
 * more than 1/power deviations (after min_iterations samples) stop drawing.
 *   counts        [n_configs][n_counts] neighbours per variable (v % n_counts)
 *   kernels       n_kernels weight kernels (kernel_dims: n_kernels*ndim, x
 *                 first; kernel_nvar[i] weights per cell)
 * Outputs (n_densities*n_kernels*n_configs*max_k, configurations fastest and
 * candidate rank innermost, the reference's im_1/im_2/im_3 images): mean
 * error^(1/power), deviation^(0.5/power), 16-bit sample counts.  Each setup
 * draws from std::mt19937(seed + setup); one iteration tests all setups on
 * the statistics it began with, searches the unpruned samples in one batch,
 * then accumulates in setup order (the reference's OpenMP order depends on
 * the thread schedule; its seed on the clock).  Complete TIs only. */
typedef struct {
    int ndim;
    const unsigned *ti_dims;
    int nvar;
    const int *types;
    const float *ti;
    int n_kernels;
    const unsigned *kernel_dims;
    const int *kernel_nvar;
    const float *const *kernels;
    int n_configs;
    int n_counts;
    const unsigned *counts;
    int n_densities;
    const float *densities;
    unsigned max_k;
    float power;
    float noise;
    unsigned max_iterations;
    unsigned min_iterations;
    float max_seconds;
    unsigned seed;
} qsk_calib_params;

int qsk_calibrate(int device, const qsk_calib_params *p, float *mean_error, float *dev_error, unsigned *n_samples,
                  long long *n_searches);

/* qsk_pattern_kbest without any allocation.  No counterpart in the reference
 * (G2S' devices allocate their buffers when they are created).
 *
 * Same arguments (a qsk_ti instead of a worker), same results as
 * qsk_pattern_kbest, for callers that cannot allocate device memory:
 *  - a process whose device memory is already held by another allocator
 *    (a caching allocator that reserved the HBM, or a host program that
 *    sized its training images to fill the GPU), where cudaMalloc fails;
 *  - a caller that must not stall the other streams of the device:
 *    qsk_pattern_kbest grows its worker's buffers with cudaFree + cudaMalloc,
 *    and cudaFree waits for the whole device.
 * The call makes no cudaMalloc, cudaFree or other allocating call.  Its
 * device scratch (the pattern's slot and terms, the map's records, the k
 * results) lives in one fixed array of QSK_NOALLOC_SCRATCH_BYTES bytes in the
 * library's device code, one per device; the host side stages on the stack.
 *
 * Limit: the scratch needs, each region rounded up to 256 bytes, 8 bytes per
 * TI scan position (positions rounded up to a multiple of 128), 8 bytes per
 * 128 positions, 16 bytes per term and 8*k bytes: training images of up to
 * about 2 million scan positions fit.  A larger request, or more than
 * QSK_NOALLOC_MAX_TERMS terms, returns QSK_ERR_UNSUPPORTED before any GPU
 * work, with the sizes in qsk_last_error().
 * Nothing in the scratch needs to start at zero: every byte a call reads was
 * written earlier in the same call.
 * One scratch per device: calls on the same device that overlap in time
 * (from several threads, or on several streams) race on it and give wrong
 * results; serialise them.
 * The first call on a device looks the scratch address up with
 * cudaGetSymbolAddress (with that device current, the return code checked)
 * and keeps it for the life of the process: do not call it again after a
 * cudaDeviceReset of that device (the module, and the scratch, reload at
 * another address).
 * `stream` is a cudaStream_t of ti's device (NULL: the legacy default
 * stream); the call returns after its work on that stream has finished. */
#define QSK_NOALLOC_SCRATCH_BYTES (16u << 20)
#define QSK_NOALLOC_MAX_TERMS 2048
int qsk_pattern_kbest_noalloc(const qsk_ti *ti, void *stream, int n_neighbours, const int *offsets, int n_terms,
                              const qsk_term *terms, unsigned k, float seed, float *out_score, unsigned *out_index,
                              int *out_min);

/* Top-W inner products on the tensor cores (tcgen05).  No G2S counterpart:
 * it is the building block of this library's tensor-core map (the cross term
 * of a batch of nodes over a template prefix, which replaces the per-node
 * FFT correlation of CPUThreadDevice::candidateForPattern, G2S
 * src/CPUThreadDevice.cpp:349-490) and of its learned proposal (node
 * embeddings against pre-embedded TI patterns).
 *   fmt       0: BF16 (queries/rows hold uint16 bit patterns), 1: FP8 E4M3
 *             (uint8 bit patterns)
 *   queries   B x K row-major, rows N x K row-major (N: positions of a TI
 *             of X x Y x (N / (X*Y)) cells, x fastest)
 *   score(q, p) = (queries[q] . rows[p]) * q_scale[q] * p_scale[p / 256] + q_bias[q]
 *             accumulated in FP32; p_scale holds one scale per tile of 256
 *             rows (scales and bias may be NULL: 1 and 0)
 *   q_box     6 ints per query: p = (x, y, z) is a candidate iff
 *             q_box[0] <= x < q_box[1], q_box[2] <= y < q_box[3],
 *             q_box[4] <= z < q_box[5]
 * The positions are cut into `ranges` contiguous ranges; for every query and
 * range the W (8, 16 or 32) largest keys are written, in no particular order,
 * to out_key / out_pos [B][ranges][W]: key = (ordered score << 32) | tie hash
 * of (q_seed[q], p), where the ordered score is the float's bits made
 * monotone (negative: all bits inverted; otherwise the sign bit set); key 0
 * marks an unused entry.  The union over the ranges holds the overall top W.
 */
int qsk_tc_topk(int device, int fmt, int B, long long N, int K, const void *queries, const void *rows,
                const float *q_scale, const float *q_bias, const float *p_scale, const unsigned *q_seed,
                const int *q_box, int X, int Y, int W, int ranges, unsigned long long *out_key, unsigned *out_pos);

/* Peak rates of this GPU measured by the library's own microbenchmarks (no
 * G2S counterpart): out[0] FP32 FMA TFLOP/s, out[1] 32-bit LOP3 Tops/s,
 * out[2] tcgen05 BF16 dense TFLOP/s, out[3] tcgen05 FP8 E4M3 dense TFLOP/s.
 * The roofline denominators of kernels with no driver-measured peak. */
int qsk_measure_peaks(int device, double *out);

/* Reference scan index -> TI cell (CPUThreadDevice::cvtIndexToPosition,
 * G2S src/CPUThreadDevice.cpp:257-268). */
unsigned qsk_index_to_position(const qsk_ti *ti, const int *min_offset, unsigned index);
/* TI cell -> reference scan index (cvtPositionToIndex, :270-284). */
unsigned qsk_position_to_index(const qsk_ti *ti, const int *min_offset, unsigned position);

/* ------------------------------------------------------------------------
 * Whole vector QS simulation on the GPU: the per-node loop of G2S
 * simulation() (include/simulation.hpp:43-710) with QuantileSamplingModule
 * (include/quantileSamplingModule.hpp:90-126,342-577), driven by the path,
 * seeds and search template of g2sQsProgramMain (src/qs.cpp:975-1258,
 * 1604-1641).  Nodes whose neighbourhoods do not depend on each other run
 * together; results equal the sequential order.
 * ---------------------------------------------------------------------- */
typedef struct {
    int ndim;
    const unsigned *ti_dims;      /* x first */
    int nvar;
    const int *types;             /* nvar entries: 0 continuous, 1 categorical */
    const float *ti;              /* prod(ti_dims) * nvar */
    const unsigned *di_dims;      /* simulation grid, x first */
    const unsigned *kernel_dims;  /* NULL: uniform kernel of size min(TI/2+1) (src/qs.cpp:1010-1042) */
    const float *kernel;          /* prod(kernel_dims) * nvar weights, or NULL */
    int n;                        /* -n */
    float k;                      /* -k */
    unsigned seed;                /* -s */
    int no_verbatim;              /* -nV */
    /* Local controls (G2S include/simulation.hpp:337-358,447-507,
     * src/qs.cpp:1264-1292); zero / NULL when unused.  Images hold values per
     * grid cell, x fastest. */
    int n_counts;                 /* -n n1 n2 ...: entries of n_per_variable (0: n for every variable) */
    const int *n_per_variable;
    int n_image_vars;             /* -ni: counts per cell (0: no image) */
    const float *n_image;
    const float *k_image;         /* -kvi: candidate count per cell (<= 0: k); k becomes max(k, max k_image) */
    int n_kernels;                /* -ki list (0: kernel_dims / kernel above) */
    const unsigned *kernels_dims; /* n_kernels * ndim */
    const float *const *kernels;  /* n_kernels weight arrays, prod(dims) * nvar each */
    const float *kernel_index_image; /* -kii: kernel index per cell (required when n_kernels > 1) */
    int full_simulation;          /* -fs: one path node per (cell, variable) value (simulationFull,
                                     include/simulation.hpp:712-1066); index image per value */
    /* Several training images (-ti with more than one grid, src/qs.cpp;
     * merged as quantileSamplingModule.hpp:90-126 does with one CUDA device
     * per TI): the grids after `ti`, each of ndim dims and nvar variables;
     * complete TIs, one neighbour count, no -nV, -fs or local controls, the
     * plain map, at most 8 TIs and 16 candidates (TIs x ceil(k)).  The index
     * image holds TI cell * nTI + TI (simulation.hpp:658). */
    int n_extra_tis;
    const unsigned *extra_ti_dims; /* n_extra_tis * ndim, x first */
    const float *const *extra_tis;
    const float *ti_index_image;   /* -ii: the TI each grid cell samples from (its value, as an int); NULL: all */
} qsk_qs_params;

typedef struct {
    long long nodes;              /* path nodes simulated */
    int levels;                   /* dependency levels (1 under teacher forcing) */
    int max_batch;                /* largest level (batches are cut at the slot budget) */
    int template_size;
    float ms_setup_neighbours;    /* device time of the neighbour search */
    float ms_levels;              /* device time of the level computation */
    float ms_batches;             /* device time of all batches */
    float ms_total;               /* device time of the whole run (first to last kernel) */
    long long launches;           /* kernels launched by the run */
    long long map_launches;       /* launches of the fused map kernel */
    float ms_map;                 /* device time inside the map kernel (profiling mode only) */
    float ms_prep;                /* ... inside the per-batch prep kernel (profiling mode only) */
    float ms_replay;              /* ... inside the k-best replay kernel (profiling mode only) */
    long long map_positions;      /* scan positions evaluated by the map kernel (nodes x N) */
    /* tensor-core form (qsk_sim_set_tensor); zero when it is off */
    int tensor_mode;              /* 0 plain, 1 BF16, 2 FP8 E4M3 */
    int tensor_prefix;            /* template offsets in the pattern matrix */
    int tensor_width;             /* heap entries per node and position range */
    int tensor_shortlist;         /* candidates re-scored exactly per node */
    long long tensor_nodes;       /* nodes drawn by the tensor-core form */
    long long plain_nodes;        /* nodes left to the exact map (neighbours beyond the prefix, marginal draws) */
    long long audited;            /* nodes re-run on the plain path for the regret audit */
    long long regret;             /* audited nodes whose draw lies outside the exact k best */
    long long regret_near;        /* audited nodes below the exact k-th score by at most 1e-5 of the term scale */
    float map_err_max;            /* largest |tensor-core score - FP64 score| / term scale, re-scored candidates */
    float map_err_mean;
    double tensor_flops;          /* MMA flops issued (2 x 128 x 256 x K per tile) */
    float ms_tensor_gemm;         /* device time of the tensor-core kernel (profiling mode only) */
    float ms_tensor_select;       /* ... of node rows, re-score and draw (profiling mode only) */
    float ms_tensor_pattern;      /* device time of building the pattern matrix (once per simulation) */
    long long tensor_launches;
    long long path_nodes;         /* path nodes of the simulation (nodes: those of the last run) */
    long long learned_fallback;   /* learned proposal: nodes whose confidence check sent them to the exact map */
    long long graph_nodes;        /* graph mode: nodes of the captured batch chain of the last run (0: direct launches) */
    float ms_graph_build;         /* graph mode: host time of capture and instantiation of the last run */
} qsk_sim_info;

typedef struct qsk_sim qsk_sim;

/* Host setup (template, path, seeds as src/qs.cpp does) and uploads.
 * di_init: prod(di_dims)*nvar values, NaN = to simulate. */
int qsk_sim_create(int device, const qsk_qs_params *p, const float *di_init, qsk_sim **out);
/* Simulate on the GPU (device-resident data only; resets the grid first). */
int qsk_sim_run(qsk_sim *s);
/* Teacher-forced evaluation: draw every path node against the completed
 * grid (host array), as the sequential run would at that node's turn.
 * id_completed (the run's index image) is needed with -nV, else may be NULL. */
int qsk_sim_run_teacher(qsk_sim *s, const float *di_completed, const unsigned *id_completed);
/* Teacher-forced evaluation of a sample of path nodes (indices into the
 * path, 0 .. nodes-1, any order): each is drawn against the completed grid as
 * the sequential run would at its turn, nothing is written back; the
 * neighbour search over the whole path runs once per simulation object and
 * is not part of the run's device time (qsk_sim_info.ms_total).  For
 * simulations too large to time in full (G2S times its own runs whole,
 * src/qs.cpp:2229-2235).  node_cell of qsk_sim_read holds the sample's
 * choices at their path indices. */
int qsk_sim_run_teacher_nodes(qsk_sim *s, const float *di_completed, const int *path_nodes, int count);
/* Copy results to the host: the grid, the index image (TI cell * nTI + TI,
 * src/qs.cpp:2277), and the chosen TI cell per path node (any may be NULL;
 * node_cell_out holds qsk_sim_info.path_nodes entries). */
int qsk_sim_read(qsk_sim *s, float *di_out, unsigned *id_out, unsigned *node_cell_out);
int qsk_sim_get_info(const qsk_sim *s, qsk_sim_info *info);
/* Profiling mode: record CUDA events around every kernel of the next runs so
 * that qsk_sim_info reports per-kernel device time (adds event overhead). */
int qsk_sim_set_profiling(qsk_sim *s, int on);
/* Bounded wait of the dependency-level pass (no G2S counterpart: G2S' path
 * threads wait for their neighbours with unbounded 250 us sleeps,
 * include/simulation.hpp:459-474).  A node waits for each dependency's level
 * for at most spin_limit polls (0: 2^22, about a second); past it the run
 * returns QSK_ERR_DEVICE ("a dependency level did not appear within the wait
 * limit") instead of hanging.  hold_node >= 0 is a failure-path test: that
 * path node's level is never published, so its dependants' waits run out
 * (-1: normal operation). */
int qsk_sim_set_level_wait(qsk_sim *s, unsigned spin_limit, long long hold_node);
/* Graph mode (plain path): qsk_sim_run captures its whole chain of batches
 * (prep, map, draw of every level, and the generator pipeline on the second
 * stream) into one CUDA graph, instantiates it and launches it, instead of
 * launching each kernel on the streams.  Results are identical.  Ignored by
 * the tensor-core and learned forms and in profiling mode. */
int qsk_sim_set_graph(qsk_sim *s, int on);
/* Several simulations in one call (the reference's concurrency over
 * realisations: one qs run per realisation, src/qs.cpp): each simulation's
 * qsk_sim_run on its own streams, `threads` host threads (0: up to 16)
 * taking the jobs in order, so that the levels of different jobs (TIs,
 * grids, n) share the GPU.  Every simulation must be distinct.  status
 * (optional, count entries) receives each job's return code; the call
 * returns the first job error (its message prefixed with the job index). */
int qsk_jobs_run(qsk_sim *const *sims, int count, int threads, int *status);
/* Path (cell order), per-path-index seeds and number of informed cells. */
int qsk_sim_get_path(const qsk_sim *s, unsigned *order, float *seeds, unsigned *begin);
/* Ends a simulation: waits for the device (as cudaFree does) and keeps the
 * simulation's device buffers as blocks for the next simulations created on
 * that device, up to a limit per device (default 8 GiB); buffers beyond it
 * are freed.  No G2S counterpart: each G2S run allocates and frees its own. */
int qsk_sim_destroy(qsk_sim *s);
/* Kept blocks: the limit per device (0: keep none), freeing every kept block
 * of every device (nothing reads them), and the kept bytes and blocks of one
 * device with the process-wide count of allocations served from them (hits)
 * or not (misses).  Kept blocks belong to the device's primary context: call
 * qsk_blocks_release before a cudaDeviceReset (or any reset of that context),
 * after which they would no longer be valid device memory. */
int qsk_blocks_set_limit(unsigned long long bytes);
int qsk_blocks_release(void);
int qsk_blocks_info(int device, unsigned long long *bytes, long long *blocks, long long *hits, long long *misses);

/* Tensor-core form of the map (no G2S counterpart; it replaces, for the nodes
 * it can take, the per-node FFT correlation and k-best of
 * CPUThreadDevice::candidateForPattern + fKst::findKBiggest, G2S
 * src/CPUThreadDevice.cpp:349-490, include/fKb.hpp:907-954, and of the CUDA
 * device's cuFFT + cublasIsamin, src/NvidiaGPUAcceleratorDevice.cu:462-727).
 * Nodes of one dependency level share the TI, so their cross terms over the
 * first `prefix` template offsets are one GEMM: (nodes x K) . (K x TI cells)
 * on tcgen05 in BF16 or FP8 E4M3 (per-row scales), FP32 accumulation in TMEM.
 * Per node the `width` best approximate scores of every position range are
 * kept, the best `shortlist` of them re-scored exactly (the plain map's FP32
 * term order; FP64 for FP8), the node's k best taken by exact score (equal
 * scores in the order of a per-node hash, not the reference's reservoir) and
 * the quantile rank drawn.  Nodes with a neighbour beyond the prefix take the
 * exact map in the same level with the same draw rule (k best by score, ties
 * by the hash, over the map's records); nodes without neighbours the
 * reference's marginal draw.  A fraction `audit` of the nodes with
 * neighbours is re-run on the plain path after the simulation,
 * teacher-forced on the final grid: `regret` counts those whose drawn
 * candidate scores below the exact k-th (qsk_sim_info).
 * Complete TIs only, without -nV, -fs or local controls.  Zero fields take
 * the automatic choice: prefix = the smallest multiple of 256 offsets that
 * covers 97 % of the path's nodes (chosen at the first tensor run from the
 * nodes' neighbour lists), capped by a 48 GiB pattern matrix; width 8 (FP8:
 * 32), shortlist 4 x extendK (FP8: 128). */
typedef struct {
    int mode;          /* 0 plain (the exact reference path), 1 BF16, 2 FP8 E4M3 */
    int prefix;        /* template offsets in the pattern matrix */
    int width;         /* 8, 16 or 32 */
    int shortlist;     /* <= 128 */
    float audit;       /* fraction of tensor-path nodes audited, 0..1 */
    int batch;         /* nodes per tensor step (GEMM launch): a multiple of 128 up to 16384; 0: 4096 */
} qsk_tensor_opts;
int qsk_sim_set_tensor(qsk_sim *s, const qsk_tensor_opts *opts);

/* ------------------------------------------------------------------------
 * Learned proposal (no G2S counterpart).  A small MLP encoder embeds a
 * node's informed neighbourhood and the neighbourhood of every TI cell as 64
 * entries of [variable values, mask, dx, dy, dz] (offsets divided by 8).
 * The entries form a stencil: the template's first 64 offsets dilated by a
 * scale s in 1..nscales (qsk_encoder_set_scales); a node takes the smallest
 * scale whose stencil holds most of its neighbours, each entry holding the
 * mean of the neighbour values falling in it (mask 1) or nothing (mask 0); a
 * TI cell's entry holds the TI value at s x the offset (mask 0 outside the
 * TI), and the TI is embedded once per scale.  Shared trunk
 * 64 x (nvar + 4) -> 256 -> 256 -> 256 (GELU), then a query head (nodes) or
 * a TI-pattern head (TI cells) -> 64, unnormalised, so that the inner
 * product can take the form of the QS score (2 v . t - |t|^2 for a
 * continuous variable is the inner product of [2v, -1] and [t, |t|^2]).
 * The tensor-core top-W
 * kernel proposes, per node, the TI cells of largest inner product; the
 * exact map (the plain path's FP32 terms) scores that shortlist; a node
 * that fails the confidence check (qsk_learned_opts) goes to the exact map
 * over the whole TI (the reference method,
 * CPUThreadDevice::candidateForPattern + fKst::findKBiggest,
 * src/CPUThreadDevice.cpp:349-490, include/fKb.hpp:907-954).
 * ---------------------------------------------------------------------- */
typedef struct qsk_encoder qsk_encoder;
/* Encoder for TIs of nvar variables, weights uniform in +-1/sqrt(fan-in)
 * from mt19937(seed), biases 0. */
int qsk_encoder_create(int device, int nvar, unsigned seed, qsk_encoder **out);
int qsk_encoder_destroy(qsk_encoder *e);
long long qsk_encoder_param_count(const qsk_encoder *e);
int qsk_encoder_input_dim(const qsk_encoder *e);
/* Stencil scales of the inputs (default 4 and 0.9): an input's 64 entries
 * are the template's first 64 offsets dilated by a scale in 1..nscales; a
 * node takes the smallest scale whose stencil holds cov_min of its informed
 * neighbours (values falling in one entry averaged), and the TI is embedded
 * once per scale.  Applies to pairs added and pattern matrices built
 * afterwards. */
int qsk_encoder_set_scales(qsk_encoder *e, int nscales, float cov_min);
/* Matrix products of the encoder's layers (forward and backward): on = 1
 * (default) on the tensor cores (tcgen05, operands rounded to BF16, FP32
 * accumulation), on = 0 on the CUDA cores in FP32.  The InfoNCE logits and
 * their gradient (B x B x 64 products), parameters, Adam state and
 * activations are FP32 either way. */
int qsk_encoder_set_tensor_cores(qsk_encoder *e, int on);
/* The encoder's tensor-core product on its own (host arrays, row-major):
 * C[M x N] = bf16(A)[M x K] * bf16(B)[N x K]^T (+ bias[N] when not NULL),
 * FP32 accumulation; operands rounded to nearest-even BF16. */
int qsk_gemm_bf16(int device, int M, int N, int K, const float *A, const float *B, const float *bias, float *C);
/* All parameters, flattened: W1 (256 x D0), b1, W2 (256 x 256), b2, W3, b3,
 * W4q (64 x 256), b4q (query head), W4p, b4p (TI-pattern head); weights
 * row-major (out x in).  set resets Adam. */
int qsk_encoder_get_weights(const qsk_encoder *e, float *out);
int qsk_encoder_set_weights(qsk_encoder *e, const float *w);
/* Symmetric InfoNCE loss of B (query, positive) input pairs (host, B x D0
 * each; logits q . p / tau, in-batch negatives) and, if grad is not NULL,
 * its gradient with respect to every parameter; no update. */
int qsk_encoder_loss_grad(qsk_encoder *e, int B, const float *xq, const float *xp, float tau, float *loss,
                          float *grad);
/* Embeddings (rows x 64) of input rows (rows x D0), host arrays; head 0 the
 * query head, 1 the TI-pattern head. */
int qsk_encoder_embed(qsk_encoder *e, int head, long long rows, const float *x, float *out);
/* Training pairs: the listed path nodes of simulation s are drawn by the
 * exact path, teacher-forced on the completed grid; each (node
 * neighbourhood, drawn TI cell's neighbourhood) pair is kept on the device.
 * Nodes without neighbours are skipped.  *added: pairs appended. */
int qsk_encoder_add_pairs(qsk_encoder *e, qsk_sim *s, const float *di_completed, const int *path_nodes, int count,
                          long long *added);
/* Training pairs from host arrays (n x D0 each): queries and their positives. */
int qsk_encoder_add_pairs_host(qsk_encoder *e, long long n, const float *xq, const float *xp);
int qsk_encoder_pairs(const qsk_encoder *e, long long *count);
/* Stored pairs [first, first + n) to host arrays (n x D0 each). */
int qsk_encoder_get_pairs(const qsk_encoder *e, long long first, long long n, float *xq, float *xp);
int qsk_encoder_clear_pairs(qsk_encoder *e);
/* Adam (lr, betas 0.9 / 0.999) on the stored pairs, shuffled every epoch by
 * mt19937(seed), minibatches of `batch`; *last_loss: the last batch's loss. */
int qsk_encoder_train(qsk_encoder *e, int epochs, int batch, float lr, float tau, unsigned seed, float *last_loss);

/* The learned proposal as the simulation's map: every node with neighbours
 * is embedded, its `width` best TI cells per position range proposed on the
 * tensor cores (BF16 inner products with the pre-embedded TI, built once per
 * simulation and encoder state), the best `shortlist` (<= 256) scored
 * exactly and drawn as in the tensor-core form; nodes failing the confidence
 * check (exact best ranked at conf_rank or later by the proposal) and nodes
 * without neighbours take the exact map.  The encoder must outlive its use
 * by s.  `audit` as in qsk_tensor_opts.  e = NULL turns it off. */
typedef struct {
    int width;         /* 8, 16 or 32 (0: 32) */
    int shortlist;     /* <= 256 (0: 256) */
    int conf_rank;     /* rank check (used when conf_z <= 0): the exact best of the shortlist must be among
                          the proposal's first conf_rank candidates (0: 1) */
    float audit;
    float conf_z;      /* statistical check (> 0): exact score against proposal score is fitted over the
                          shortlist (s = a L + b, residual sd); the node's k-th best exact score must clear
                          a L_out + b + conf_z sd, L_out the largest proposal score of a position left out */
    float conf_r2;     /* ... and the fit must explain this fraction of the exact scores' variance (0: 0.2) */
} qsk_learned_opts;
int qsk_sim_set_learned(qsk_sim *s, qsk_encoder *e, const qsk_learned_opts *opts);

/* Host-only planning helpers (no GPU needed), identical to what
 * qsk_sim_create computes.
 * Sorted search template of a kernel: offsets (nd ints each, nearest first,
 * G2S src/qs.cpp:1055-1135) and the kernel weight of every offset/variable
 * (quantileSamplingModule.hpp:362-392); kernel NULL = uniform.  Writes at
 * most `capacity` offsets and returns the template size (<0: error). */
int qsk_qs_template(int ndim, int nvar, const unsigned *kernel_dims, const float *kernel, int *offsets, float *weights,
                    int capacity);
/* Random path (cell order, informed cells first) and per-path-index seeds
 * for grid di_init (NaN = unknown), G2S src/qs.cpp:975,1159-1201,1250-1258.
 * Returns the number of informed cells (<0: error). */
long long qsk_qs_path(long long cells, int nvar, const float *di_init, unsigned seed, unsigned *order, float *seeds);

/* Map kernel selection, process-wide: 0 (default) picks the bit-sliced
 * kernel for categorical patterns with unit weights and the FP32 gather
 * kernel otherwise; 1 always uses the FP32 gather kernel.  Both give the same
 * scores bit for bit; the switch exists to test exactly that. */
int qsk_set_map_mode(int mode);

/* One call: setup, simulate, read back into di_inout / id_out (host). */
int qsk_simulate(int device, const qsk_qs_params *p, float *di_inout, unsigned *id_out);

/* ------------------------------------------------------------------------
 * G2S grid files (.bgrid, optionally gzip-compressed .bgrid.gz): the
 * serialised DataImage of the G2S data directory.  Replace
 * DataImage::createFromFile / write (G2S include/DataImage.hpp:96-104,143-223,
 * 281-323; src/DataImage.cpp:35-165) so that grids move between G2S and this
 * library unchanged.
 * ---------------------------------------------------------------------- */
/* Read `path`.  Writes ndim, dims[ndim] (x first, up to 16), nvar, up to
 * types_capacity variable types, the encoding (0 float, 1 int, 2 uint) and
 * *count = prod(dims) * nvar; copies the 32-bit values (variables
 * interleaved) to data when data is not NULL (capacity in values). */
int qsk_bgrid_read(const char *path, int *ndim, unsigned *dims, int *nvar, int *types, int types_capacity,
                   int *encoding, void *data, long long capacity, long long *count);
/* Write a grid to `path` (gzip when compress != 0). */
int qsk_bgrid_write(const char *path, int ndim, const unsigned *dims, int nvar, const int *types, int encoding,
                    const void *data, int compress);

#ifdef __cplusplus
}
#endif

#endif /* G2S_B200_H */
