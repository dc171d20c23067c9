/*
 * rfx_b200 — C ABI of the B200 (sm_100a) post-growth random-forest analysis
 * path: OOB / in-bag / test-set leaf routing, OOB votes, exact INT32 proximity
 * pair counts, finishprox normalisation, permutation importance (overall and
 * local), and the low-rank proximity + MDS forms.
 *
 * Every entry point returns an rfx_status (0 = success) and never throws.
 * Pointers are plain host or device pointers (the library inspects each one
 * with cudaPointerGetAttributes): outputs written to DEVICE memory are
 * enqueued on the context's stream and the call returns without waiting;
 * outputs written to HOST memory are complete when the call returns.
 * All output buffers are caller-allocated.
 *
 * Reference interfaces replaced (chriskuchar/RFX):
 *   the post-growth section of gpu_growtree_batch (cuda/rf_growtree.cu:2706-4130,
 *   declared in src/rf_random_forest.cpp:35-51) and the per-tree CPU sequence of
 *   RandomForest::grow_tree_single (src/rf_random_forest.cpp:1043-1309), plus the
 *   low-rank handle API get_lowrank_factors_host / compute_mds_from_factors_host
 *   (cuda/rf_lowrank_helpers.cu:13,55).
 */
#ifndef RFX_B200_H
#define RFX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int rfx_status;

enum {
    RFX_OK = 0,
    RFX_ERR_INVALID = 1,      /* bad argument or size */
    RFX_ERR_CUDA = 2,         /* CUDA runtime error (message in rfx_last_error) */
    RFX_ERR_OOM = 3,          /* device allocation failed */
    RFX_ERR_STATE = 4,        /* call order (e.g. no forest loaded) */
    RFX_ERR_UNSUPPORTED = 5,  /* feature outside the supported set (e.g. casewise) */
    RFX_ERR_TIMEOUT = 6,      /* a bounded device wait gave up */
    RFX_ERR_FOREST = 7,       /* forest failed validation */
    RFX_ERR_NO_DEVICE = 8     /* no CUDA device / extension unusable */
};

typedef struct rfx_ctx rfx_ctx;

/* Per-context settings, passed by value (the reference's mutable global
 * rf::g_config, include/rf_config.hpp:17-114, has no counterpart here). */
typedef struct rfx_config {
    int32_t device;          /* CUDA device ordinal */
    int32_t use_casewise;    /* 1: the reference's use_casewise=True weighting
                                (votes, importance and pair sums weighted by
                                bootstrap multiplicities; see rfx_casewise_votes,
                                rfx_proximity_upper_f64) */
    int32_t n_threads_cpu;   /* host threads for rfx_grow_forest (0 = all) */
    int32_t reserved[5];
} rfx_config;

/* A forest and the training data it was grown on, in the compact layout:
 * tree t owns nodes [offs[t], offs[t+1]) of nodestatus/bestvar/xbestsplit/
 * nodeclass, 2 entries per node of treemap (left, right), and maxcat entries
 * per node of catgoleft (NULL = all zero, as the reference's CPU grower leaves
 * it).  nin is ntree x n bootstrap multiplicities; X is n x p float32
 * row-major; y holds labels 0..nclass-1; cat[p] is 1 for numeric features and
 * the number of levels for categorical ones.  Replaces the padded
 * ntree x maxnode arrays of rf::RandomForest (src/rf_random_forest.cpp:326-335). */
typedef struct rfx_forest_view {
    int32_t n, p, nclass, maxcat, ntree;
    const int64_t* offs;        /* ntree + 1 */
    const int32_t* nodestatus;  /* -1 terminal, 1 split, 2 unsplit */
    const int32_t* bestvar;
    const float* xbestsplit;
    const int32_t* treemap;     /* 2 per node */
    const int32_t* nodeclass;
    const int32_t* catgoleft;   /* maxcat per node, or NULL */
    const int32_t* nin;         /* ntree * n */
    const float* X;             /* n * p */
    const int32_t* y;           /* n */
    const int32_t* cat;         /* p */
} rfx_forest_view;

/* Last error message of the calling thread ("" if none). */
const char* rfx_last_error(void);

rfx_status rfx_ctx_create(const rfx_config* cfg, rfx_ctx** out);
rfx_status rfx_ctx_destroy(rfx_ctx* ctx);
/* The context's CUDA stream (a cudaStream_t) for event timing by callers. */
rfx_status rfx_ctx_stream(rfx_ctx* ctx, void** stream);
rfx_status rfx_synchronize(rfx_ctx* ctx);

/* Validate and upload a forest (replaces the per-tree H2D copies of
 * cuda/rf_growtree.cu:2618-2657).  Labels and node counts are checked on the
 * host; node status, bestvar, children and bootstrap counts by the packing
 * kernels, before any analysis runs.  A forest that fails validation returns
 * RFX_ERR_FOREST and leaves no forest loaded.  The library keeps its own
 * device copies (pinned host arrays upload fastest); reloading a forest of the
 * same shape reuses the context's device buffers. */
rfx_status rfx_forest_load(rfx_ctx* ctx, const rfx_forest_view* view);

/* A forest left in device memory by a GPU grower, in the reference's padded
 * layout: tree t owns slots [t*maxnode, t*maxnode + nnode[t]) of nodestatus,
 * bestvar, xbestsplit and nodeclass, 2*maxnode slots per tree of treemap and
 * maxnode*maxcat of catgoleft (NULL = all zero); nin is ntree x n, X n x p
 * row-major, y n labels, cat p feature kinds.  nnode is a HOST array of
 * ntree node counts (the reference keeps nnode_all on the host); every other
 * array is device memory of the context's device. */
typedef struct rfx_forest_device_view {
    int32_t n, p, nclass, maxcat, ntree, maxnode;
    const int32_t* nnode;       /* host, ntree */
    const int32_t* nodestatus;  /* device, ntree * maxnode */
    const int32_t* bestvar;     /* device, ntree * maxnode */
    const float* xbestsplit;    /* device, ntree * maxnode */
    const int32_t* treemap;     /* device, ntree * 2 * maxnode */
    const int32_t* nodeclass;   /* device, ntree * maxnode */
    const int32_t* catgoleft;   /* device, ntree * maxnode * maxcat, or NULL */
    const int32_t* nin;         /* device, ntree * n */
    const float* X;             /* device, n * p */
    const int32_t* y;           /* device, n */
    const int32_t* cat;         /* device, p */
} rfx_forest_device_view;

/* Load a device-resident forest without a round trip through the host: the
 * hand-off from the reference's GPU grower (gpu_growtree_batch,
 * cuda/rf_growtree.cu:888 and :2706-2771, whose node arrays stay on the device
 * with tree_offset = tree_id * maxnode) to the analysis path.  The trees are
 * gathered into the compact layout on the device (device-to-device copies and
 * one gather kernel), then validated and packed exactly as rfx_forest_load
 * does; the labels and feature kinds are read back (n + p ints) for the
 * host-side checks.  Results are identical to loading the same forest from
 * host arrays. */
rfx_status rfx_forest_load_device(rfx_ctx* ctx, const rfx_forest_device_view* view);

/* OOB routing + votes: cpu_testreebag (src/rf_testreebag.cpp:13-125) and the
 * vote loop of grow_tree_single (src/rf_random_forest.cpp:1107-1153) over all
 * trees.  q[n*nclass] receives integer vote counts; nout[n] the reference's
 * doubled OOB count (src/rf_bootstrap.cpp:61 and src/rf_random_forest.cpp:1110).
 * leaf (optional, ntree*n) receives per-tree node ids: OOB samples from the
 * testreebag walk, in-bag samples from find_terminal_node
 * (src/rf_random_forest.cpp:2194-2244). */
rfx_status rfx_route_oob(rfx_ctx* ctx, int32_t* q, int32_t* nout, int32_t* leaf);

/* OOB error, predictions and probabilities from the votes of rfx_route_oob
 * (compute_classification_error src/rf_random_forest.cpp:2413-2462,
 * compute_oob_predictions :2246-2301).  Any output may be NULL. */
rfx_status rfx_oob_summary(rfx_ctx* ctx, float* oob_error, int32_t* pred, float* proba);

/* Exact pair counts: S[i,j] = C[i,j] + C[j,i] for i <= j, packed row-major
 * upper triangle with the diagonal (len = n(n+1)/2, diagonal 0), where C[i,j]
 * counts trees with i out-of-bag, j in-bag and both in the same terminal node:
 * the dense branch of cpu_proximity (src/rf_proximity.cpp:99-231) accumulated
 * over all trees.  Replaces cuda_proximity_upper_triangle_fp16_kernel
 * (cuda/rf_proximity_upper_triangle.cu:149). */
rfx_status rfx_proximity_upper_i32(rfx_ctx* ctx, int32_t* S, size_t len);

/* Total pair updates sum_t sum_leaf noob_leaf * nin_leaf of the last
 * rfx_proximity_upper_i32 (the unit of the pair-update throughput). */
rfx_status rfx_pair_updates(rfx_ctx* ctx, int64_t* count);

/* cpu_finishprox (src/rf_finishprox.cpp:12-74) applied to S (device or host,
 * packed as above) with the doubled nout:
 *   P[i,j] = 0.5 * ((S/2)/nout_i + (S/2)/nout_j), P[i,i] = 1, rows with
 * nout_i = 0 unscaled, in FP64, stored as float32 — full n x n (full = 1, the
 * layout get_proximity_matrix returns, python/randomforest_py.cpp:1114-1177)
 * or packed upper triangle (full = 0). */
rfx_status rfx_finishprox(rfx_ctx* ctx, const int32_t* S, float* P, int full);

/* Permutation importance over all trees and all features
 * (cpu_varimp src/rf_varimp.cpp:106-302 with cpu_testreeimp :32-104 and
 * cpu_permobmr :16-30, accumulated as src/rf_random_forest.cpp:1217-1230).
 * avimp[p] = feature_importances_, sqsd[p], qimp[n], qimpm[n*p] (sample-major,
 * before localimp); impn = 1 computes qimp/qimpm (local importance), which may
 * then be NULL when impn = 0.  A tree with no OOB sample gives the reference's
 * 0/0 (NaN) for the features it splits on.  When a categorical value rounds
 * outside 0..maxcat-1 in a permuted walk, cpu_testreeimp stops without a vote
 * and the reference keeps a vote that depends on its OpenMP thread count; this
 * call then returns RFX_ERR_UNSUPPORTED with a message naming the cause.
 * A walk decides up to 256 features at once (one bit each); with more
 * features the walks run once per block of 256. */
rfx_status rfx_varimp(rfx_ctx* ctx, int impn, float* avimp, float* sqsd, float* qimp, float* qimpm);

/* localimp (src/rf_utilities.cpp:28-43) as get_local_importance returns it:
 * out[idx] = 100 * (qimp[idx % n] - qimpm[idx]) / ntree for idx < n*p. */
rfx_status rfx_localimp(rfx_ctx* ctx, const float* qimp, const float* qimpm, float* out);

/* Test-set votes (predict_classification / predict_proba,
 * src/rf_random_forest.cpp:1925-2036, :2303-2411): votes[m*nclass]. */
rfx_status rfx_predict(rfx_ctx* ctx, const float* X, int32_t m, int32_t* votes);

/* Classical 3-D MDS of the full proximity matrix, as compute_mds_3d_cpu
 * (src/rf_mds_cpu.cpp:88-341) computes it when called by the binding
 * (python/randomforest_py.cpp:1221-1243): P is the n x n float32 matrix of
 * rfx_finishprox(full = 1) (host or device); rows are divided by nout again,
 * D = max - P, double centring of D^2, the 3 largest eigenpairs (eigenvalues
 * > 1e-10, descending) in FP64; coords = n x 3 row-major float64, each column
 * defined up to sign.  evals (optional, host) receives the 3 eigenvalues. */
rfx_status rfx_mds3d_full(rfx_ctx* ctx, const float* P, double* coords, double* evals);

/* Low-rank proximity (replaces the rank-1-per-tree QLORA accumulation of
 * LowRankProximityMatrix, cuda/rf_proximity_lowrank.cu:863-1071, and the
 * handle API get_lowrank_factors_host, cuda/rf_lowrank_helpers.cu:13):
 * P ~= I + A A^T with A (n x rank, float32 row-major) from a randomised range
 * finder over the leaf indicators of the loaded forest (rank + oversample
 * columns rounded up to a multiple of 8, at most 120 and at most n;
 * power_iters power iterations, CholeskyQR2 in FP64, FP64
 * Rayleigh-Ritz).  precision 0 = FP32 throughout; 1 = BF16 storage of the
 * sketch inputs and leaf sums with FP32 accumulation; 2 = as 1 with the last
 * product (the Rayleigh-Ritz projection) in FP32; 3 = FP8 e4m3 storage of the
 * sketch rows and leaf sums, one FP32 scale per row, FP32 accumulation.
 * The context keeps the factors for the calls below; A and evals (host, the
 * rank eigenvalues) may be NULL. */
typedef struct rfx_lowrank_opts {
    int32_t rank;
    int32_t oversample;
    int32_t power_iters;
    int32_t precision;
    uint64_t seed;
    /* trees per pass of the leaf sums: 0 = as many as 4 GB of leaf sums hold
     * (the batched form); 1 = one tree per pass, the per-tree structure of the
     * reference's GPU accumulation (slower: every pass re-reads the n x 2w
     * accumulator) */
    int32_t trees_per_pass;
    int32_t reserved;
} rfx_lowrank_opts;
rfx_status rfx_lowrank(rfx_ctx* ctx, const rfx_lowrank_opts* opts, float* A, float* evals);

/* One product MV = M V of the low-rank path's operator M = P - I (P the
 * finishprox proximity of the loaded forest, never formed) with a block V
 * (n x w, w a multiple of 8 up to 120, row-major), computed as rfx_lowrank's
 * range finder computes it (precision 0: FP32 storage, 1: BF16 storage of the
 * sketch rows and leaf sums, 3: FP8 e4m3 rows with a scale each; FP32
 * accumulation).  No reference counterpart:
 * it exposes the range finder's product so that callers (and tests) can apply
 * M without the n x n matrix.  V and MV may be host or device pointers. */
rfx_status rfx_lowrank_operator(rfx_ctx* ctx, int w, int precision, const float* V, float* MV);

/* Quantised factors with one scale per column (format 1: INT8, q = round(A/s),
 * s = max|A[:,c]|/127; format 2: FP8 e4m3, s = max|A[:,c]|/448; format 3:
 * NF4, the reference's 16-level code of A/s with s = max|A[:,c]|, two codes
 * per byte over the row-major entries, the lower nibble first; format 4: FP16
 * with scales 1).  q is n x rank bytes (NF4: ceil(n x rank / 2), FP16:
 * 2 x n x rank), scales
 * rank floats (either may be NULL).  The reference quantises INT8 with one
 * per-tensor scale (cuda/rf_quantization_kernels.cu:107-120), NF4 without a
 * scale (cuda/rf_proximity_lowrank.cu:353-411) and FP16 without a scale; the
 * factors of P ~= I + A A^T are what is quantised. */
rfx_status rfx_lowrank_quantize(rfx_ctx* ctx, int format, void* q, float* scales);

/* k-dimensional classical MDS from the factors (compute_mds_from_factors,
 * cuda/rf_proximity_lowrank.cu:1935-2531): D = 1 - P off the diagonal with
 * P = I + A A^T, double centring applied in factor space, the k largest
 * eigenpairs; coords n x k row-major float64.  use_quantized = 1 uses the
 * dequantised factors of rfx_lowrank_quantize.  precision 0 applies the
 * operator in FP32; precision 1 (rank 32 or 64) runs tcgen05 BF16 GEMMs with
 * FP32 accumulation until the iteration stalls at the BF16 rounding level, then
 * takes one FP32 step (an FP32 operator product and Rayleigh-Ritz) from that
 * basis; precision 3 does the same with FP8 E4M3 operands (tcgen05
 * kind::f8f6f4, a scale per factor column, per stack row and per block
 * column, FP32 accumulation).  Other non-zero values mean 1. */
rfx_status rfx_mds_from_factors(rfx_ctx* ctx, int k, int use_quantized, int precision, double* coords,
                                double* evals);

/* One application W = B V of the double-centred factor-space MDS operator of
 * rfx_mds_from_factors to an n x 16 FP64 block V (row-major; host or device);
 * precision 0 = FP32 products, 1 = tcgen05 BF16 products, 3 = tcgen05 FP8
 * E4M3 products (rank 32 or 64 for either). */
rfx_status rfx_factor_mds_operator(rfx_ctx* ctx, int use_quantized, int precision, const double* V, double* W);

/* Outlier scores from the factors (compute_outlier_scores,
 * src/rf_random_forest.cpp:2489-2520): 1 / sum_j P_ij^2, divided by the
 * median element sorted[n/2]. */
rfx_status rfx_outlier_scores(rfx_ctx* ctx, int use_quantized, float* scores);

/* Batched analysis of many independent forests in one CUDA graph (the
 * reference analyses one forest per fit, so a batch of forests is a loop of
 * separate fits, src/rf_random_forest.cpp:485-830).  Each item is a context
 * with a loaded forest (its own stream) and DEVICE output buffers; NULL
 * outputs skip that part: votes (n*nclass) and nout (n) as rfx_route_oob,
 * oob_error / oob_pred as rfx_oob_summary, S (n(n+1)/2) as
 * rfx_proximity_upper_i32, avimp/sqsd (and with impn, qimp/qimpm) as
 * rfx_varimp.  Capture runs every item once eagerly (allocating what the
 * chains need and checking the device flags), then records all items into
 * one graph whose per-forest chains run concurrently; kernel_nodes (may be
 * NULL) receives the graph's kernel count.  rfx_graph_launch replays the
 * whole batch with one launch on `stream` (a cudaStream_t) and returns after
 * enqueueing; it refuses a graph whose contexts were reloaded or released
 * since capture.  Contexts must outlive the graph. */
typedef struct rfx_batch_item {
    rfx_ctx* ctx;
    int32_t* votes;
    int32_t* nout;
    float* oob_error;
    int32_t* oob_pred;
    int32_t* S;
    float* avimp;
    float* sqsd;
    float* qimp;
    float* qimpm;
    int32_t impn;
    int32_t reserved;
} rfx_batch_item;
typedef struct rfx_graph rfx_graph;
rfx_status rfx_graph_capture_batch(const rfx_batch_item* items, int32_t count, rfx_graph** out,
                                   int64_t* kernel_nodes);
rfx_status rfx_graph_launch(rfx_graph* g, void* stream);
rfx_status rfx_graph_destroy(rfx_graph* g);

/* Launch-shape autotuner (no counterpart in the reference).  The routing,
 * pair-count, varimp-walk, per-sample importance and low-rank leaf-sum stages
 * each offer a few launch shapes with identical results; the first run for a
 * problem shape (device and power-of-two buckets of n, ntree, p) runs each
 * once untimed, then times each once on the context stream and keeps the
 * fastest for the process.  Setting RFX_AUTOTUNE=0 keeps the default shapes,
 * and RFX_TUNE_ROUTE / RFX_TUNE_PAIRS / RFX_TUNE_VWALK / RFX_TUNE_ROUTE_LEAF /
 * RFX_TUNE_PAIRS_HUB / RFX_TUNE_SEGSUM / RFX_TUNE_VSAMPLE = <shape> force one
 * shape; nothing is tuned while a stream is being captured.
 * rfx_tuned_shapes copies up to `cap` records of 6 int32 {stage (0 routing,
 * 1 pair counts, 2 varimp walk, 3 routing in leaf order, 4 pair counts with
 * hub tiles, 5-7 low-rank leaf sums in FP32 / BF16 / FP8, 8 per-sample
 * importance sums), device, log2 n, log2 ntree, log2 p, shape}
 * and sets *count to the number of records. */
rfx_status rfx_tuned_shapes(int32_t* out, int32_t cap, int32_t* count);

/* Allocation-free pair counts.  No counterpart in the reference.
 *
 * For callers that cannot allocate device memory while they run (a process
 * that reserves the GPU's memory for its own arena up front and bans
 * cudaMalloc/cudaFree afterwards, or a framework that lends the library only
 * buffers it owns).  Computes the packed upper-triangle pair counts of
 * rfx_proximity_upper_i32 from leaf indices the caller already holds:
 *   leaf[t*n + i]  dense terminal-node index of sample i in tree t (terminal
 *                  nodes numbered 0.. in node order), or -1 to leave it out;
 *   inbag[t*n + i] nonzero when sample i is in-bag in tree t;
 *   S[len]         output, len = n(n+1)/2.
 * All three must be device memory of the current device; the work runs on
 * `stream` (a cudaStream_t, NULL = default stream) and the call waits for that
 * stream before it returns.  It calls no cudaMalloc, cudaFree or allocating
 * library routine: its temporaries live in one fixed array of about 26 MB
 * inside the library.  CUDA creates that array, and loads the kernels' code,
 * on a device when the library is first used there (lazy module loading, the
 * default since CUDA 12.2), so the FIRST call on each device is where that
 * device memory is taken: a caller that reserves the GPU's memory for its own
 * arena should make one call per device before it reserves the rest (or set
 * CUDA_MODULE_LOADING=EAGER); the device then holds the array until its
 * context is destroyed.  The first call on a device (and the first after the
 * device's context was reset) also looks up the array's device address with
 * cudaGetSymbolAddress.  Every call is synchronous (it reads its error flag
 * back to the host and waits for `stream`), so it cannot be recorded into a
 * CUDA graph by stream capture.  Limits:
 * n <= 32768, ntree <= 65535, ntree * n <= 1048576, 1 <= max_leaves <= n; larger
 * inputs are rejected with RFX_ERR_INVALID, as is a leaf index >= max_leaves
 * (those samples are left out of S).  Every call uses the same array and it
 * keeps the last call's contents, so calls whose work overlaps on a GPU race
 * with each other: serialise them. */
rfx_status rfx_pair_counts_noalloc(const int32_t* leaf, const uint8_t* inbag, int32_t n, int32_t ntree,
                                   int32_t max_leaves, int32_t* S, size_t len, void* stream);

/* Case-wise weighting (use_casewise = 1 in rfx_config; the reference's
 * bootstrap-frequency weighting, src/rf_random_forest.cpp:1049-1153,
 * src/rf_varimp.cpp:138-236, src/rf_proximity.cpp:195-222).  tnodewt of a
 * terminal node = the mean bootstrap multiplicity of the in-bag samples that
 * reach it; an OOB vote counts tnodewt of the node it ends on.
 * rfx_casewise_votes writes the weighted OOB votes q (n x nclass float, the
 * reference's q_) and optionally the doubled nout; rfx_oob_summary and
 * rfx_varimp of a case-wise context use these weights (importance: right,
 * rightimp, qimp, qimpm weighted by tnodewt of the node each (permuted) walk
 * reaches).  In a case-wise context rfx_route_oob refuses an int32 q and
 * rfx_proximity_upper_i32 refuses (the pair weights are FP64).  Every sum runs
 * in the reference's order: results are bit-identical to it. */
rfx_status rfx_casewise_votes(rfx_ctx* ctx, float* q, int32_t* nout);

/* FP64 pair sums S = C + C^T (packed upper triangle with the diagonal, 0 on
 * it): C[i][j] += nin[j] / nodesize for every tree where i is OOB and j is
 * in-bag in i's leaf (nodesize = the leaf's in-bag multiplicities summed) in a
 * case-wise context, += 1 otherwise (then S equals the INT32 counts);
 * cpu_proximity's dense branch, src/rf_proximity.cpp:99-231, summed tree by
 * tree as the reference does.  S: host or device, n(n+1)/2 doubles. */
rfx_status rfx_proximity_upper_f64(rfx_ctx* ctx, double* S, size_t len);

/* cpu_finishprox (src/rf_finishprox.cpp:12-74) of FP64 sums from
 * rfx_proximity_upper_f64; S and P host or device memory, P as in
 * rfx_finishprox (full n x n or the packed upper triangle, float32). */
rfx_status rfx_finishprox_f64(rfx_ctx* ctx, const double* S, float* P, int full);

/* RF-GAP proximity (cpu_proximity_rfgap, src/rf_proximity.cpp:238-391, the
 * reference's use_rfgap=True): pGAP(i,j) = (1/|S_i|) sum over the trees where
 * i is OOB of c_j / |M_i| for the in-bag samples j of i's node (c_j = j's
 * bootstrap multiplicity, |M_i| = the multiplicities of those samples summed,
 * nodes = the node ids of testreebag for OOB samples and of
 * find_terminal_node for in-bag ones), P = (pGAP + pGAP^T) / 2 off the
 * diagonal, 1 on the diagonal of a sample never OOB (else 0).  P: host or
 * device, the packed upper triangle with the diagonal, FP64 — the final
 * matrix (no finishprox).  Bit-identical to the reference. */
rfx_status rfx_proximity_rfgap(rfx_ctx* ctx, double* P, size_t len);

/* Per-stage device timing.  With profiling enabled, every stage launch is
 * bracketed by CUDA events on the context stream; rfx_profile_read waits for
 * the stream and returns, per stage, the mean duration of its launches since
 * profiling was (re)enabled (the last 64 at most; ms, -1 if never run), and
 * the number of kernels the library has launched since the context was
 * created.  Stage order: route, leaf lists, pair counts,
 * finishprox, varimp per-tree, varimp per-sample, varimp per-feature, predict,
 * oob summary, localimp, pair-range table, low-rank operator product,
 * low-rank orthonormalisation, MDS from factors, full-matrix MDS, hub-leaf
 * pair counts on the tensor cores (the pair counts of one call are the hub
 * stage plus the pair-count stage). */
enum { RFX_NUM_STAGES = 16 };
rfx_status rfx_profile_enable(rfx_ctx* ctx, int enable);
rfx_status rfx_profile_read(rfx_ctx* ctx, float* stage_ms, int64_t* kernel_launches);

/* Forest producer (not on the analysis path): cpu_bootstrap + cpu_growtree
 * (src/rf_bootstrap.cpp:14-82, src/rf_growtree.cpp:382-945) restated with a
 * partition per node; trees grown in parallel host threads.  Arrays are
 * allocated by the library and released with rfx_free_forest. */
typedef struct rfx_grown_forest {
    int32_t ntree;
    int64_t* offs;
    int32_t* nodestatus;
    int32_t* bestvar;
    float* xbestsplit;
    int32_t* treemap;
    int32_t* nodeclass;
    int32_t* nin;
} rfx_grown_forest;

rfx_status rfx_grow_forest(const float* X, const int32_t* y, int32_t n, int32_t p, int32_t nclass,
                           int32_t ntree, int32_t mtry, int32_t minndsize, int32_t maxnode, int32_t iseed,
                           int32_t n_threads, rfx_grown_forest* out);
rfx_status rfx_free_forest(rfx_grown_forest* f);

#ifdef __cplusplus
}
#endif

#endif /* RFX_B200_H */
