// Allocation-free pair counts.
//
// Some callers cannot allocate device memory when they call in: for example a
// serving process that reserves all of the GPU's memory for its own arena at
// start-up and forbids cudaMalloc/cudaFree afterwards (an allocation there can
// synchronise the whole device, stall other streams and fragment the arena),
// or a host framework that hands this library only the buffers it owns.  For
// them rfx_pair_counts_noalloc computes the same packed upper-triangle pair
// counts as rfx_proximity_upper_i32, from per-(tree, sample) leaf indices the
// caller already holds on the device, and keeps all of its temporary data in
// one fixed-size array defined in this file (a __device__ variable).
//
// CUDA loads a module's code and its __device__ variables into a device's
// context when the module is first used there (lazy module loading, the
// default since CUDA 12.2), not when the library is opened.  The first call
// on each device is that first use: it looks up the array's device address
// and launches the kernels for the first time, and that is when the array and
// the kernels' code take their device memory.  A caller that reserves the
// GPU's memory up front should therefore make one call per device before it
// reserves the rest (or run with CUDA_MODULE_LOADING=EAGER, which loads
// everything when the context is created); from then on the device holds the
// array until the context is destroyed and calls allocate nothing.
#include <mutex>

#include "rfx_internal.cuh"

namespace rfx {
namespace {

// Limits of the allocation-free form.
constexpr int64_t NA_MAX_CELLS = 1 << 20;  // ntree * n
constexpr int NA_MAX_N = 32768;
constexpr int NA_MAX_TREES = 65535;        // u16 row counters

constexpr int64_t align64(int64_t w) { return (w + 63) & ~int64_t(63); }  // 256-byte units of int32 words

// Word offsets of the regions at the largest sizes.
constexpr int64_t NA_KEY = 0;
constexpr int64_t NA_MEMB = align64(NA_KEY + NA_MAX_CELLS);
constexpr int64_t NA_OPP = align64(NA_MEMB + NA_MAX_CELLS);                      // int2 per cell
constexpr int64_t NA_SEGOFF = align64(NA_OPP + 2 * NA_MAX_CELLS);                // <= ntree*(2n+1)
constexpr int64_t NA_ORDER = align64(NA_SEGOFF + 2 * NA_MAX_CELLS + NA_MAX_TREES);
constexpr int64_t NA_SEGBASE = align64(NA_ORDER + NA_MAX_N);                     // int64 per tree + 1
constexpr int64_t NA_ERR = align64(NA_SEGBASE + 2 * (NA_MAX_TREES + 1));
constexpr int64_t NA_WORDS = align64(NA_ERR + 64);

static __device__ __align__(256) int32_t g_noalloc_scratch[NA_WORDS];

constexpr int NA_MAX_DEVICES = 64;
std::mutex g_na_mutex;
// Per device: the scratch array's device address and the id of the context it
// was looked up in.  A context destroyed and created again (cudaDeviceReset)
// gets a new id, so the address is looked up again instead of reusing a stale
// one.
int32_t* g_na_addr[NA_MAX_DEVICES] = {};
unsigned long long g_na_ctx[NA_MAX_DEVICES] = {};

// Current context id through the driver entry points (cuCtxGetCurrent and
// cuCtxGetId, CUDA 12.0+), fetched once; 0 when they are unavailable, in which
// case the address is looked up on every call.
typedef int (*na_ctx_get_current_t)(void**);
typedef int (*na_ctx_get_id_t)(void*, unsigned long long*);

unsigned long long current_ctx_id() {
    static na_ctx_get_current_t get_cur = nullptr;
    static na_ctx_get_id_t get_id = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* f0 = nullptr;
        void* f1 = nullptr;
        cudaDriverEntryPointQueryResult q0 = cudaDriverEntryPointSymbolNotFound, q1 = q0;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f0, cudaEnableDefault, &q0) == cudaSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &f1, cudaEnableDefault, &q1) == cudaSuccess &&
            q0 == cudaDriverEntryPointSuccess && q1 == cudaDriverEntryPointSuccess) {
            get_cur = reinterpret_cast<na_ctx_get_current_t>(f0);
            get_id = reinterpret_cast<na_ctx_get_id_t>(f1);
        }
        cudaGetLastError();
    }
    if (!get_cur || !get_id) return 0;
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (get_cur(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
    return id;
}

// True when p is device memory of device `dev` (managed memory counts).
bool on_device(const void* p, int dev) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (a.type == cudaMemoryTypeDevice && a.device == dev) || a.type == cudaMemoryTypeManaged;
}

__global__ void na_keys_kernel(const int32_t* __restrict__ leaf, const uint8_t* __restrict__ inbag, int64_t cells,
                               int max_leaves, int32_t* __restrict__ key, uint32_t* __restrict__ err) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= cells) return;
    const int l = leaf[idx];
    int k = -1;
    if (l >= 0) {
        if (l < max_leaves) k = 2 * l + (inbag[idx] ? 1 : 0);
        else atomicOr(err, 1u);
    }
    key[idx] = k;
}

__global__ void na_segbase_kernel(int T, int max_leaves, int64_t* __restrict__ segbase) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t <= T) segbase[t] = (int64_t)t * (2 * (int64_t)max_leaves + 1);
}

}  // namespace
}  // namespace rfx

using namespace rfx;

extern "C" rfx_status rfx_pair_counts_noalloc(const int32_t* leaf, const uint8_t* inbag, int32_t n, int32_t ntree,
                                              int32_t max_leaves, int32_t* S, size_t len, void* stream) {
    if (!leaf || !inbag || !S) {
        set_error("rfx_pair_counts_noalloc: null buffer");
        return RFX_ERR_INVALID;
    }
    if (n < 1 || ntree < 1 || max_leaves < 1) {
        set_error("rfx_pair_counts_noalloc: n, ntree and max_leaves must be >= 1");
        return RFX_ERR_INVALID;
    }
    if (n > NA_MAX_N || ntree > NA_MAX_TREES || (int64_t)n * ntree > NA_MAX_CELLS || max_leaves > n) {
        set_error("rfx_pair_counts_noalloc: size beyond the allocation-free limits (n <= 32768, ntree <= 65535, "
                  "ntree * n <= 1048576, max_leaves <= n); use rfx_proximity_upper_i32");
        return RFX_ERR_INVALID;
    }
    if (len != (size_t)upper_len(n)) {
        set_error("rfx_pair_counts_noalloc: S must hold n(n+1)/2 entries");
        return RFX_ERR_INVALID;
    }
    int dev = 0;
    RFX_CUDA(cudaGetDevice(&dev));
    if (!on_device(leaf, dev) || !on_device(inbag, dev) || !on_device(S, dev)) {
        set_error("rfx_pair_counts_noalloc: leaf, inbag and S must be device memory of the current device");
        return RFX_ERR_INVALID;
    }
    if (dev < 0 || dev >= NA_MAX_DEVICES) {
        set_error("rfx_pair_counts_noalloc: device ordinal beyond the address table");
        return RFX_ERR_UNSUPPORTED;
    }
    int32_t* base = nullptr;
    {
        // set-up, once per device and context: look up the device address of
        // the scratch array with this device current (host code cannot use
        // the symbol itself; it names a host-side stand-in)
        std::lock_guard<std::mutex> lk(g_na_mutex);
        const unsigned long long cid = current_ctx_id();
        if (!g_na_addr[dev] || cid == 0 || cid != g_na_ctx[dev]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess) return cuda_fail(e, "rfx_pair_counts_noalloc: cudaGetSymbolAddress");
            g_na_addr[dev] = static_cast<int32_t*>(p);
            g_na_ctx[dev] = cid;
        }
        base = g_na_addr[dev];
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t cells = (int64_t)n * ntree;
    PairsRawArgs a;
    a.n = n;
    a.T = ntree;
    a.max_leaves = max_leaves;
    int32_t* key = base + NA_KEY;
    a.key = key;
    a.memb = base + NA_MEMB;
    a.opp = reinterpret_cast<int2*>(base + NA_OPP);
    a.segoff = base + NA_SEGOFF;
    a.order = base + NA_ORDER;
    int64_t* segbase = reinterpret_cast<int64_t*>(base + NA_SEGBASE);
    a.segbase = segbase;
    a.err = reinterpret_cast<uint32_t*>(base + NA_ERR);
    a.S = S;
    // the array keeps the previous call's contents: clear the error word; every
    // other region is fully rewritten before it is read
    RFX_CUDA(cudaMemsetAsync(a.err, 0, sizeof(uint32_t), s));
    na_keys_kernel<<<(unsigned)((cells + 255) / 256), 256, 0, s>>>(leaf, inbag, cells, max_leaves, key, a.err);
    RFX_CUDA(cudaGetLastError());
    na_segbase_kernel<<<(ntree + 1 + 255) / 256, 256, 0, s>>>(ntree, max_leaves, segbase);
    RFX_CUDA(cudaGetLastError());
    rfx_status st = launch_pairs_pipeline_raw(a, s);
    if (st != RFX_OK) return st;
    uint32_t bits = 0;
    RFX_CUDA(cudaMemcpyAsync(&bits, a.err, sizeof(bits), cudaMemcpyDeviceToHost, s));
    RFX_CUDA(cudaStreamSynchronize(s));
    if (bits & 1u) {
        set_error("rfx_pair_counts_noalloc: a leaf index is >= max_leaves (those samples were left out)");
        return RFX_ERR_INVALID;
    }
    return RFX_OK;
}
