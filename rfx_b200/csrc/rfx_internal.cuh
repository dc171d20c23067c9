// Internal declarations shared by the CUDA translation units of librfx_b200.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <functional>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "rfx_b200.h"

namespace rfx {

// Device node record (16 bytes, one int4 load per traversal step):
//   x = split threshold (float bits), y = left child, z = right child,
//   w = var (bits 0..15) | status as int8 (bits 16..23) | categorical (bit 24).
// Node ids are local to their tree.
struct __align__(16) DNode {
    float split;
    int32_t left;
    int32_t right;
    int32_t meta;
};

__host__ __device__ inline int node_var(int32_t meta) { return meta & 0xffff; }
__host__ __device__ inline int node_status(int32_t meta) { return (int)(int8_t)((meta >> 16) & 0xff); }
__host__ __device__ inline bool node_cat(int32_t meta) { return (meta >> 24) & 1; }

// Error bits raised by kernels into ctx->d_err (checked by the host after sync).
enum : uint32_t {
    ERR_STALE_JVR = 1u,       // testreeimp broke without assigning (stale jvr in the reference)
    ERR_TRAVERSAL_LIMIT = 2u, // a bounded walk hit its step limit
    ERR_SMEM_KEYS = 4u,       // per-tree key table exceeded its shared-memory budget
    ERR_WAIT_LIMIT = 8u,      // a bounded mbarrier wait of a tensor-core pipeline gave up
};

enum Stage : int {
    ST_ROUTE = 0, ST_CSR, ST_PAIRS, ST_FINISHPROX, ST_VARIMP_TREE, ST_VARIMP_SAMPLE, ST_VARIMP_FEATURE,
    ST_PREDICT, ST_OOB, ST_LOCALIMP, ST_OPP, ST_LR_PRODUCT, ST_LR_ORTH, ST_MDS_FACTORS, ST_MDS_FULL, ST_HUBS,
    ST_COUNT
};

struct Ctx {
    int device = 0;
    bool profile = false;
    static constexpr int EV_RING = 64;  // launches remembered per stage
    std::vector<cudaEvent_t> ev_start[ST_COUNT];
    std::vector<cudaEvent_t> ev_end[ST_COUNT];
    long long ev_count[ST_COUNT] = {};
    long long launches = 0;
    cudaStream_t stream = nullptr;
    rfx_config cfg{};

    // forest
    bool loaded = false;
    int n = 0, p = 0, nclass = 0, maxcat = 0, T = 0;
    int64_t N = 0;                      // total nodes
    std::vector<int64_t> h_offs;        // T+1
    std::vector<int32_t> h_nnode;       // T
    std::vector<int32_t> h_nleaf;       // T: terminal nodes per tree
    std::vector<int64_t> h_segbase;     // T+1: start of each tree's key-offset table
    std::vector<int32_t> h_noob;        // T
    int max_keys = 0;                   // max_t 2*nleaf_t
    int max_nnode = 0;
    int iv_words = 0;                   // ceil(p / 64)

    float* d_X = nullptr;               // n*p
    int32_t* d_y = nullptr;             // n
    int32_t* d_cat = nullptr;           // p
    DNode* d_nodes = nullptr;           // N
    int32_t* d_nodeclass = nullptr;     // N
    int32_t* d_leafidx = nullptr;       // N: dense terminal index (node order) or -1
    int32_t* d_catgoleft = nullptr;     // N*maxcat or null
    int64_t* d_offs = nullptr;          // T+1
    int32_t* d_nnode = nullptr;         // T
    uint8_t* d_inbag = nullptr;         // T*n
    int32_t* d_nin = nullptr;           // T*n bootstrap multiplicities (case-wise weights, RF-GAP)
    float* d_tnodewt = nullptr;         // N: case-wise terminal-node weights
    int64_t* d_segbase = nullptr;       // T+1
    uint64_t* d_iv = nullptr;           // T*iv_words: features used by non-terminal nodes
    int32_t* d_noob = nullptr;          // T
    int32_t* d_permoff = nullptr;       // T: offset of the tree's permutation in d_perm
    int32_t* d_perm = nullptr;          // concatenated permutations per distinct noob
    float* d_invnoob = nullptr;         // T: 1.0f / noob

    // analysis scratch (allocated lazily)
    int32_t* d_key = nullptr;           // T*n: 2*leafidx + inbag, or -1
    int32_t* d_segoff = nullptr;        // segbase[T]: per-tree key offsets (+1 sentinel each)
    int32_t* d_memb = nullptr;          // T*n: members grouped by key, ascending within a key;
                                        // samples without a terminal node follow the keyed members
    int2* d_opp = nullptr;              // n*T: opposite-status member range cut to members > i
    uint8_t* d_hubflag = nullptr;       // segbase[T]: 1 for the keys of hub leaves (hubs.cu)
    uint8_t* d_hubtiles = nullptr;      // S_hub upper-triangle tiles, one byte per entry
    int32_t* d_hubstate = nullptr;      // [0] threshold bin, [1] hub count, [4..5] hub pair updates (u64)
    int32_t* d_order = nullptr;         // n: row processing order
    int32_t* d_votes = nullptr;         // n*nclass
    int32_t* d_nout = nullptr;          // n
    uint32_t* d_err = nullptr;          // error bits
    unsigned long long* d_pairs = nullptr;  // pair-update counter
    bool routed = false;
    bool csr_built = false;
    uint64_t generation = 0;            // bumped whenever the forest buffers are released
    int64_t last_pairs = 0;

    // varimp scratch
    int32_t* d_joob = nullptr;          // T*n
    int32_t* d_partner = nullptr;       // T*n: permutation partner of each OOB sample
    int32_t* d_oobord = nullptr;        // T*n: each tree's OOB samples in member-list (leaf) order
    uint8_t* d_vflags = nullptr;        // T*n: bit1 testreebag correct, bit2 testreeimp correct
    uint64_t* d_flips = nullptr;        // T*n*varimp_flip_words(iv_words)
    int32_t* d_right = nullptr;         // 2T: per tree #correct (testreebag), #correct (testreeimp)
    int32_t* d_rightimp = nullptr;      // T*p: signed flip counts per tree and feature
    float* d_qimp = nullptr;            // n (internal accumulators)
    float* d_qimpm = nullptr;           // n*p
    float* d_avimp = nullptr;           // p
    float* d_sqsd = nullptr;            // p

    // low-rank factors (P ~= I + A A^T)
    float* d_lrA = nullptr;             // n*lr_rank FP32
    float* d_lrAq = nullptr;            // n*lr_rank dequantised copy
    void* d_lrQ = nullptr;              // n*lr_rank quantised (int8 or fp8)
    float* d_lrScale = nullptr;         // lr_rank per-column scales
    int lr_rank = 0;
    int lr_qformat = 0;                 // 0 none, 1 INT8, 2 FP8 e4m3
    int last_mds_tc_iters = 0;          // iterations of the last factor MDS (tensor-core phase)
    int last_mds_f32_iters = 0;         // and its FP32 phase

    size_t bytes = 0;                   // device bytes held

    // Scratch blocks of finished calls, kept by size for the next call with
    // the same shapes.  All work of a context runs on its one stream, so a
    // block handed back while its kernels are still queued is only reused by
    // later work on that stream.
    std::multimap<size_t, void*> scratch_free;
    std::map<void*, size_t> dsize;  // sizes of the buffers dalloc handed out
    void scratch_release() {
        for (auto& kv : scratch_free) cudaFree(kv.second);
        scratch_free.clear();
    }
    void pool_put(void* p) {
        auto it = dsize.find(p);
        if (it == dsize.end()) {
            cudaFree(p);
            return;
        }
        scratch_free.emplace(it->second, p);
        bytes -= it->second;
        dsize.erase(it);
    }
    std::vector<int> perm_noobs;  // distinct noob values whose tables d_perm holds
};

// First failure found by the forest-packing kernels (code 0 = none).
struct LoadError {
    int code;  // 1 nodestatus, 2 bestvar, 3 child, 4 negative nin
    int tree;
    int node;  // node within the tree, or sample for code 4
    int pad;
};

// Per-call scratch drawn from the context's pool: get() reuses a kept block of
// the same size or allocates one (after releasing the pool if memory is
// short); the destructor returns every block to the pool.
struct Scratch {
    Ctx* c;
    std::vector<std::pair<size_t, void*>> held;
    explicit Scratch(Ctx* c_) : c(c_) {}
    Scratch(const Scratch&) = delete;
    Scratch& operator=(const Scratch&) = delete;
    ~Scratch() {
        for (auto& b : held) c->scratch_free.emplace(b.first, b.second);
    }
    template <typename T>
    T* get(size_t count) {
        const size_t bytes = ((sizeof(T) * (count ? count : 1)) + 255) & ~(size_t)255;
        auto it = c->scratch_free.find(bytes);
        void* x = nullptr;
        if (it != c->scratch_free.end()) {
            x = it->second;
            c->scratch_free.erase(it);
        } else if (cudaMalloc(&x, bytes) != cudaSuccess) {
            cudaGetLastError();
            c->scratch_release();
            if (cudaMalloc(&x, bytes) != cudaSuccess) {
                cudaGetLastError();
                return nullptr;
            }
        }
        held.emplace_back(bytes, x);
        return static_cast<T*>(x);
    }
};

// RAII stage bracket: records events around a stage when profiling is on and
// counts the kernels the stage launches.
struct StageTimer {
    Ctx* c;
    int s;
    int slot = -1;
    StageTimer(Ctx* c_, int s_, int kernels) : c(c_), s(s_) {
        c->launches += kernels;
        if (c->profile && !c->ev_start[s].empty()) {
            slot = (int)(c->ev_count[s] % Ctx::EV_RING);
            cudaEventRecord(c->ev_start[s][slot], c->stream);
        }
    }
    ~StageTimer() {
        if (slot >= 0) {
            cudaEventRecord(c->ev_end[s][slot], c->stream);
            c->ev_count[s]++;
        }
    }
};

// error helpers (thread-local message)
void set_error(const std::string& msg);
rfx_status cuda_fail(cudaError_t e, const char* what);

#define RFX_CUDA(call)                                         \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return ::rfx::cuda_fail(e_, #call); \
    } while (0)

// device allocation tracked in ctx->bytes
template <typename T>
rfx_status dalloc(Ctx* c, T** p, size_t count) {
    if (*p) return RFX_OK;
    if (count == 0) count = 1;
    const size_t bytes = (count * sizeof(T) + 255) & ~(size_t)255;
    auto it = c->scratch_free.find(bytes);
    if (it != c->scratch_free.end()) {
        *p = static_cast<T*>(it->second);
        c->scratch_free.erase(it);
        c->dsize[(void*)*p] = bytes;
        c->bytes += bytes;
        return RFX_OK;
    }
    cudaError_t e = cudaMalloc((void**)p, bytes);
    if (e == cudaErrorMemoryAllocation && !c->scratch_free.empty()) {
        cudaGetLastError();
        cudaStreamSynchronize(c->stream);
        c->scratch_release();
        e = cudaMalloc((void**)p, bytes);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        set_error(std::string("device allocation of ") + std::to_string(bytes) + " bytes failed: " +
                  cudaGetErrorString(e));
        return RFX_ERR_OOM;
    }
    c->dsize[(void*)*p] = bytes;
    c->bytes += bytes;
    return RFX_OK;
}

bool is_device_ptr(const void* p);

// Raise a kernel's dynamic shared-memory limit to everything the device allows
// beside its static shared memory.  Setting the limit (not the launch's own
// size) keeps launches of other sizes, e.g. ones captured in a graph for other
// forests, valid.
template <typename K>
rfx_status allow_dyn_smem(K* kernel, int dev_smem) {
    cudaFuncAttributes a;
    RFX_CUDA(cudaFuncGetAttributes(&a, kernel));
    RFX_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  dev_smem - (int)a.sharedSizeBytes));
    return RFX_OK;
}

// kernel launchers (each returns after enqueueing on ctx->stream)
rfx_status launch_route(Ctx* c);
rfx_status launch_build_csr(Ctx* c);

// Autotuned stages: kernel ids and the launch shapes each offers.
enum TuneKernel : int { TK_ROUTE = 0, TK_PAIRS16 = 1, TK_VWALK = 2, TK_ROUTE_LEAF = 3, TK_PAIRS_HUB = 4,
                        TK_SEGSUM_F32 = 5, TK_SEGSUM_BF16 = 6, TK_SEGSUM_FP8 = 7, TK_VSAMPLE = 8 };
rfx_status autotune(Ctx* c, int kernel, int nvar, int def, const std::function<rfx_status(int)>& run);
rfx_status launch_pack_forest(cudaStream_t s, int T, int n, int p, const int64_t* d_offs, const int32_t* status,
                              const int32_t* bestvar, const float* split, const int32_t* treemap,
                              const int32_t* d_cat, const int32_t* nin, DNode* nodes, int32_t* leafidx,
                              uint64_t* iv, int32_t* nleaf, uint8_t* inbag, int32_t* noob, LoadError* err);
cudaError_t launch_gather_padded(cudaStream_t s, int T, int maxnode, int maxcat, const int64_t* d_offs,
                                 const int32_t* status_p, const int32_t* bestvar_p, const float* split_p,
                                 const int32_t* treemap_p, const int32_t* nodeclass_p, const int32_t* catgoleft_p,
                                 int32_t* status, int32_t* bestvar, float* split, int32_t* treemap,
                                 int32_t* nodeclass, int32_t* catgoleft);
rfx_status launch_pairs_upper(Ctx* c, int32_t* dS);
rfx_status launch_build_csr_raw(cudaStream_t s, int device, const int32_t* key, int n, int T, const int64_t* segbase,
                                int32_t* segoff, int32_t* memb, int max_keys, uint32_t* err);
rfx_status launch_joob_partner(Ctx* c);
// case-wise weighting and RF-GAP (weighted.cu)
rfx_status launch_tnodewt(Ctx* c);
rfx_status launch_casewise_votes(Ctx* c, const int32_t* d_leafnode, float* d_q);
rfx_status launch_weighted_rows(Ctx* c, int mode, const int32_t* key, const int64_t* segbase, const int32_t* segoff,
                                const int32_t* memb, int64_t nkeys, double* out);
rfx_status launch_gap_keys(Ctx* c, const int32_t* d_leafnode, int32_t* d_key);
rfx_status launch_casewise_varimp(Ctx* c, const int32_t* d_leafnode, int impn, float* d_avimp, float* d_sqsd,
                                  float* d_qimp, float* d_qimpm);
rfx_status launch_route_leaf(Ctx* c, int32_t* d_leaf);
rfx_status launch_oob_summary_f32(Ctx* c, const float* d_q, float* d_errout, int32_t* d_pred, float* d_proba);
rfx_status launch_finishprox_f64(Ctx* c, const double* dS, float* dP, int full);
// S_hub tiles of the hub leaves (hubs.cu)
int hub_tiles_nj(int n);
size_t hub_tile_bytes(int n);
// first tile of row block I (128 rows) in the S_hub tile list: the tiles
// (I, J), J = I/2 .. NJ-1 (256 columns each), row block after row block
__host__ __device__ inline long long hub_row_start(int I, int NJ) {
    if (I <= 0) return 0;
    const long long a = (long long)(I - 1);
    return (long long)I * NJ - (a * a) / 4;
}
rfx_status launch_hub_tiles(Ctx* c, uint8_t* keyflag, uint8_t* tiles, int32_t* hub_state,
                            unsigned long long* hub_pairs);
rfx_status launch_finishprox(Ctx* c, const int32_t* dS, float* dP, int full);
rfx_status launch_oob_summary(Ctx* c, float* d_err_out, int32_t* d_pred, float* d_proba);
rfx_status launch_varimp(Ctx* c, int impn);
// Flip words per (tree, sample) of the varimp walk: one per 64 features, at
// most four (features beyond 256 are decided in blocks of 256).
constexpr int VARIMP_BLOCK_WORDS = 4;
inline int varimp_flip_words(int iv_words) { return iv_words < VARIMP_BLOCK_WORDS ? iv_words : VARIMP_BLOCK_WORDS; }
rfx_status launch_localimp(Ctx* c, const float* d_qimp, const float* d_qimpm, float* d_out);
rfx_status launch_predict(Ctx* c, const float* dX, int m, int32_t* d_votes);
rfx_status check_device_errors(Ctx* c);
rfx_status launch_mds3d_full(Ctx* c, const float* dP, double* d_coords, double* evals);
rfx_status launch_mds_factors(Ctx* c, const float* dA, int k, int ndim, int max_iter, double tol, double* d_coords,
                              double* evals, int* iters, int precision);
rfx_status launch_outlier_scores(Ctx* c, const float* dA, int k, float* d_out);
rfx_status launch_factor_operator(Ctx* c, const float* dA, int k, const double* V, double* W, int precision);
rfx_status lowrank_compute(Ctx* c, int k, int oversample, int power_iters, int precision, uint64_t seed,
                           float* d_A_out, float* h_evals, const float* d_apply_in = nullptr,
                           int trees_per_pass = 0);
rfx_status lowrank_quantize(Ctx* c, const float* dA, int k, int format, void* dq, float* dscale);
rfx_status lowrank_dequantize(Ctx* c, const void* dq, const float* dscale, int k, int format, float* dA);

inline int64_t upper_len(int64_t n) { return n * (n + 1) / 2; }

// Device buffers of the pair-count pipeline when they are not owned by a
// context (see noalloc.cu).
struct PairsRawArgs {
    int n, T, max_leaves;
    const int32_t* key;      // T*n
    const int64_t* segbase;  // T+1
    int32_t* segoff;         // segbase[T]
    int32_t* memb;           // T*n
    int2* opp;               // n*T
    int32_t* order;          // n
    uint32_t* err;
    int32_t* S;              // n(n+1)/2
};
rfx_status launch_pairs_pipeline_raw(const PairsRawArgs& a, cudaStream_t stream);

}  // namespace rfx
