// Tensor-core (tcgen05, BF16 inputs, FP32 accumulation in TMEM) kernels of the
// factor-space MDS operator (mds.cu), for rank k = 32 or 64 and a block of
// S = 16 vectors:
//
//   mstack_tc_kernel:   M_j = A^T diag(u_j) A for all j, as one GEMM
//                       D[(j,a), b] = sum_i (u_ij A_ia) A_ib with M = S*k rows
//                       (4 or 8 tiles of 128, all resident in TMEM), N = k and
//                       the n samples as the reduction, in chunks of 32.  A
//                       persistent CTA per SM owns one contiguous range of
//                       chunks and writes its FP32 partial; mstack_reduce_kernel
//                       adds the partials in CTA order (reproducible) and lays
//                       M out as the next kernel's BF16 operand.
//   quadform_tc_kernel: T2_ij = a_i^T M_j a_i: D[i, (j,b)] = sum_a A_ia M_j[b][a]
//                       for a 128-sample tile, N = S*k in passes of 256 TMEM
//                       columns (two buffers, so the epilogue of one pass
//                       overlaps the MMAs of the next); the epilogue dots every
//                       k-column block of a row with a_i, so the n x (S*k)
//                       product never leaves the SM.  Persistent CTAs load the
//                       whole M stack once.
//
// Operands sit in shared memory in the canonical K-major, no-swizzle UMMA
// layout: 8-row x 16-byte core matrices, the two 8-element K halves of a
// 16-wide K step 128 bytes apart (leading byte offset) and consecutive 8-row
// groups 256 bytes apart (stride byte offset).  The factor A, which is fixed
// for a whole MDS call, is packed once into that layout in two forms (128-
// sample tiles with K = rank for the quadratic forms, and 32-sample chunks
// with K = samples for the M stack), so every operand tile arrives by one
// cp.async.bulk copy.  Roles: one thread issues the bulk copies, one the
// MMAs (tcgen05.commit to mbarriers), four warps build the scaled operand or
// run the epilogue.  Every mbarrier wait is bounded; a wait that gives up
// raises ERR_WAIT_LIMIT, and the CTA drains its copies and MMAs (again with
// bounded waits) before it frees TMEM and returns.
#include <cuda_bf16.h>
#include <cuda_fp8.h>

#include "rfx_internal.cuh"

namespace rfx {
namespace {

constexpr int S_ = 16;    // vectors per block
constexpr int CH = 32;    // samples per M-stack chunk
constexpr int NP = 256;   // TMEM columns per quadratic-form pass
constexpr int WAIT_LIMIT = 1 << 24;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)(256u >> 4) << 32) |
           (1ull << 46);
}

__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__host__ __device__ constexpr uint32_t idesc_e4m3_f32(int M, int N) {
    // kind::f8f6f4 with A and B both E4M3 (type code 0), FP32 accumulation
    return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// byte offset of (row r, K byte kb) in a canonical tile of R rows: K steps of
// 32 bytes (16 BF16 or 32 FP8 elements, one MMA's K), R * 32 bytes each
__host__ __device__ __forceinline__ uint32_t canon_off_b(int r, int kb, int R) {
    return (uint32_t)((kb >> 5) * (R * 32) + (r >> 3) * 256 + ((kb >> 4) & 1) * 128 + (r & 7) * 16 + (kb & 15));
}

// the same for the BF16 element k
__host__ __device__ __forceinline__ uint32_t canon_off(int r, int k, int R) { return canon_off_b(r, 2 * k, R); }

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_e4m3(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

template <bool F8>
__device__ __forceinline__ void mma_op(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    if constexpr (F8) mma_e4m3(tmem_d, a, b, idesc, acc);
    else mma_bf16(tmem_d, a, b, idesc, acc);
}

// FP8 E4M3 conversions (round to nearest, saturating to +-448)
__device__ __forceinline__ uint32_t pack_e4m3x4(float a, float b, float c, float d) {
    const uint32_t lo = __nv_cvt_float2_to_fp8x2(make_float2(a, b), __NV_SATFINITE, __NV_E4M3);
    const uint32_t hi = __nv_cvt_float2_to_fp8x2(make_float2(c, d), __NV_SATFINITE, __NV_E4M3);
    return lo | (hi << 16);
}

__device__ __forceinline__ float2 e4m3x2_to_float2(uint32_t two) {
    const __half2_raw h = __nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)two, __NV_E4M3);
    return __half22float2(*reinterpret_cast<const __half2*>(&h));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(mbar),
                 "r"(bytes)
                 : "memory");
}

// bounded wait for the phase with parity `parity` to complete
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    for (int it = 0; it < WAIT_LIMIT; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

// 16 consecutive columns of this thread's TMEM lane (no wait)
__device__ __forceinline__ void tmem_ld16_nw(uint32_t taddr, uint32_t* r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// ---------------------------------------------------------------------------
// Packing (once per MDS call for A, once per product for u)

// Aq: 128-sample tiles of A (K = rank), canonical, rows >= n zero.
template <int K_>
__global__ void pack_aq_kernel(const float* __restrict__ A, int n, int ntiles, uint8_t* __restrict__ Aq) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;  // one (tile row, 8-wide K group)
    const size_t total = (size_t)ntiles * 128 * (K_ / 8);
    if (idx >= total) return;
    const int kg = (int)(idx % (K_ / 8));
    const size_t row = idx / (K_ / 8);
    const int tile = (int)(row / 128), r = (int)(row % 128);
    const size_t i = row;
    float v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = i < (size_t)n ? A[i * K_ + kg * 8 + q] : 0.0f;
    uint4 o;
    o.x = pack_bf16x2(v[0], v[1]);
    o.y = pack_bf16x2(v[2], v[3]);
    o.z = pack_bf16x2(v[4], v[5]);
    o.w = pack_bf16x2(v[6], v[7]);
    *reinterpret_cast<uint4*>(Aq + (size_t)tile * (128 * K_ * 2) + canon_off(r, kg * 8, 128)) = o;
}

// At: 32-sample chunks of A^T (rows = rank index, K = samples), canonical,
// samples >= n zero.
template <int K_>
__global__ void pack_at_kernel(const float* __restrict__ A, int n, int nch, uint8_t* __restrict__ At) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;  // one (chunk, a, 8-sample group)
    const size_t total = (size_t)nch * K_ * (CH / 8);
    if (idx >= total) return;
    const int g = (int)(idx % (CH / 8));
    const int a = (int)((idx / (CH / 8)) % K_);
    const size_t ch = idx / ((size_t)(CH / 8) * K_);
    float v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const size_t i = ch * CH + g * 8 + q;
        v[q] = i < (size_t)n ? A[i * K_ + a] : 0.0f;
    }
    uint4 o;
    o.x = pack_bf16x2(v[0], v[1]);
    o.y = pack_bf16x2(v[2], v[3]);
    o.z = pack_bf16x2(v[4], v[5]);
    o.w = pack_bf16x2(v[6], v[7]);
    *reinterpret_cast<uint4*>(At + ch * (size_t)(K_ * CH * 2) + canon_off(a, g * 8, K_)) = o;
}

// uT: 32-sample chunks of u^T in FP32, [chunk][j][32], samples >= n zero;
// with umax (the FP8 form) every column j divided by its largest magnitude.
__global__ void pack_ut_kernel(const float* __restrict__ u, int n, int nch, const unsigned* __restrict__ umax,
                               float* __restrict__ uT) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t)nch * CH * S_) return;
    const size_t i = idx / S_;
    const int j = (int)(idx % S_);
    const size_t ch = i / CH;
    const int w = (int)(i % CH);
    float v = i < (size_t)n ? u[idx] : 0.0f;
    if (umax) {
        const float m = __uint_as_float(umax[j]);
        v = m > 0.0f ? v / m : 0.0f;
    }
    uT[(ch * S_ + j) * CH + w] = v;
}

// largest |x| of every column of a rows x cols FP32 matrix (cols divides
// 256; bit patterns of non-negative floats order like the values), into
// zeroed mx: thread t keeps column t % cols over a stride of rows, the CTA
// combines in shared memory, one global atomic per CTA and column
constexpr int CAM_THREADS = 256;
constexpr int CAM_CTAS = 592;
__global__ void __launch_bounds__(CAM_THREADS) col_absmax_kernel(const float* __restrict__ X, int64_t rows, int cols,
                                                                 unsigned* __restrict__ mx) {
    __shared__ unsigned s_mx[CAM_THREADS];
    const int c = threadIdx.x % cols;
    const int rpb = CAM_THREADS / cols;  // rows per CTA step
    unsigned m = 0u;
    for (int64_t r = (int64_t)blockIdx.x * rpb + threadIdx.x / cols; r < rows; r += (int64_t)gridDim.x * rpb)
        m = max(m, __float_as_uint(fabsf(X[r * cols + c])));
    if (threadIdx.x < cols) s_mx[threadIdx.x] = 0u;
    __syncthreads();
    atomicMax(s_mx + c, m);
    __syncthreads();
    if (threadIdx.x < cols && s_mx[threadIdx.x]) atomicMax(mx + threadIdx.x, s_mx[threadIdx.x]);
}

inline unsigned col_absmax_grid(int64_t rows, int cols) {
    const int64_t need = (rows + CAM_THREADS / cols - 1) / (CAM_THREADS / cols);
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(CAM_CTAS, need));
}

// FP8 operands of the factor (the FP8 form): column scales sA[a] = max |A[:, a]| / 448,
// Aq8 as Aq with E4M3(A / sA) bytes (K = rank bytes), At8 as At (K = 32
// samples = one 32-byte K step).
__global__ void col_scale_kernel(const unsigned* __restrict__ mx, int k, float* __restrict__ sA) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= k) return;
    const float m = __uint_as_float(mx[a]);
    sA[a] = m > 0.0f ? m / 448.0f : 1.0f;
}

template <int K_>
__global__ void pack_aq8_kernel(const float* __restrict__ A, const float* __restrict__ sA, int n, int ntiles,
                                uint8_t* __restrict__ Aq) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;  // one (tile row, 16-wide K group)
    const size_t total = (size_t)ntiles * 128 * (K_ / 16);
    if (idx >= total) return;
    const int kg = (int)(idx % (K_ / 16));
    const size_t row = idx / (K_ / 16);
    const int tile = (int)(row / 128), r = (int)(row % 128);
    float v[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = row < (size_t)n ? A[row * K_ + kg * 16 + q] / sA[kg * 16 + q] : 0.0f;
    uint4 o;
    o.x = pack_e4m3x4(v[0], v[1], v[2], v[3]);
    o.y = pack_e4m3x4(v[4], v[5], v[6], v[7]);
    o.z = pack_e4m3x4(v[8], v[9], v[10], v[11]);
    o.w = pack_e4m3x4(v[12], v[13], v[14], v[15]);
    *reinterpret_cast<uint4*>(Aq + (size_t)tile * (128 * K_) + canon_off_b(r, kg * 16, 128)) = o;
}

template <int K_>
__global__ void pack_at8_kernel(const float* __restrict__ A, const float* __restrict__ sA, int n, int nch,
                                uint8_t* __restrict__ At) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;  // one (chunk, a, 16-sample group)
    const size_t total = (size_t)nch * K_ * (CH / 16);
    if (idx >= total) return;
    const int g = (int)(idx % (CH / 16));
    const int a = (int)((idx / (CH / 16)) % K_);
    const size_t ch = idx / ((size_t)(CH / 16) * K_);
    const float inv = 1.0f / sA[a];
    float v[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        const size_t i = ch * CH + g * 16 + q;
        v[q] = i < (size_t)n ? A[i * K_ + a] * inv : 0.0f;
    }
    uint4 o;
    o.x = pack_e4m3x4(v[0], v[1], v[2], v[3]);
    o.y = pack_e4m3x4(v[4], v[5], v[6], v[7]);
    o.z = pack_e4m3x4(v[8], v[9], v[10], v[11]);
    o.w = pack_e4m3x4(v[12], v[13], v[14], v[15]);
    *reinterpret_cast<uint4*>(At + ch * (size_t)(K_ * CH) + canon_off_b(a, g * 16, K_)) = o;
}

// ---------------------------------------------------------------------------
// M stack

template <int K_, bool F8>
struct MsCfg {
    static constexpr int EB = F8 ? 1 : 2;                  // bytes per operand element
    static constexpr int MT = S_ * K_ / 128;               // M tiles
    static constexpr uint32_t AOP = MT * 128 * CH * EB;    // scaled operand per stage
    static constexpr uint32_t ATB = K_ * CH * EB;          // A^T chunk
    static constexpr uint32_t UTB = S_ * CH * 4;           // u^T chunk
    static constexpr uint32_t STB = AOP + ATB + UTB;
    static constexpr int ST = K_ == 64 ? 3 : 4;            // stages
    static constexpr uint32_t SMEM = ST * STB;
    static constexpr uint32_t TMC = MT * K_ < 32 ? 32 : MT * K_;  // TMEM columns
};

// 192 threads: warps 0-3 build the scaled operand and run the epilogue, warp 4
// lane 0 loads, warp 5 lane 0 issues the MMAs.  CTA b owns chunks
// [b * per, min(nch, (b + 1) * per)) and writes partial b.
template <int K_, bool F8>
__global__ void __launch_bounds__(192, 1) mstack_tc_kernel(const uint8_t* __restrict__ At, const float* __restrict__ uT,
                                                          int nch, int per, float* __restrict__ Mpart,
                                                          uint32_t* __restrict__ err) {
    using C = MsCfg<K_, F8>;
    extern __shared__ __align__(1024) uint8_t sm[];
    __shared__ __align__(8) uint64_t full[C::ST], aready[C::ST], empty[C::ST], done;
    __shared__ uint32_t tmem_base;
    __shared__ int s_fail;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int c0 = blockIdx.x * per, c1 = min(nch, c0 + per);
    const int cnt = max(0, c1 - c0);
    if (warp == 0) tmem_alloc(smem_u32(&tmem_base), C::TMC);
    if (tid == 0) {
        for (int s = 0; s < C::ST; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&aready[s]), 128);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        mbar_init(smem_u32(&done), 1);
        s_fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;
    const uint32_t base = smem_u32(sm);
    bool ok = true;
    if (warp == 4) {
        if (lane == 0) {
            int it = 0;
            for (; it < cnt; ++it) {
                const int s = it % C::ST;
                if (it >= C::ST && !mbar_wait(smem_u32(&empty[s]), (uint32_t)((it / C::ST - 1) & 1))) {
                    ok = false;
                    break;
                }
                const uint32_t st = base + s * C::STB;
                mbar_expect_tx(smem_u32(&full[s]), C::ATB + C::UTB);
                bulk_g2s(st + C::AOP, At + (size_t)(c0 + it) * C::ATB, C::ATB, smem_u32(&full[s]));
                bulk_g2s(st + C::AOP + C::ATB, uT + (size_t)(c0 + it) * S_ * CH, C::UTB, smem_u32(&full[s]));
            }
            // the last copies land before the CTA can leave
            for (int q = max(0, it - C::ST); q < it; ++q)
                mbar_wait(smem_u32(&full[q % C::ST]), (uint32_t)((q / C::ST) & 1));
        }
    } else if (warp == 5) {
        if (lane == 0) {
            constexpr uint32_t idesc = F8 ? idesc_e4m3_f32(128, K_) : idesc_bf16_f32(128, K_);
            for (int it = 0; it < cnt && ok; ++it) {
                const int s = it % C::ST;
                if (!mbar_wait(smem_u32(&aready[s]), (uint32_t)((it / C::ST) & 1))) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;");
                const uint32_t st = base + s * C::STB;
#pragma unroll
                for (int m = 0; m < C::MT; ++m)
#pragma unroll
                    for (int ks = 0; ks < CH * C::EB / 32; ++ks)
                        mma_op<F8>(tmem + m * K_, umma_desc(st + m * (128 * CH * C::EB) + ks * (128 * 32)),
                                   umma_desc(st + C::AOP + ks * (K_ * 32)), idesc, (it > 0 || ks > 0) ? 1u : 0u);
                mma_commit(smem_u32(&empty[s]));
            }
            mma_commit(smem_u32(&done));  // arrives once every MMA issued above has finished
        }
    } else {
        // scaled operand: thread r builds row r of every M tile, (j, a) =
        // (m * 128 / K_ + r / K_, r % K_), 8 samples per 16-byte store
        const int r = tid;
        const int a = r % K_, jr = r / K_;
        for (int it = 0; it < cnt; ++it) {
            const int s = it % C::ST;
            if (!mbar_wait(smem_u32(&full[s]), (uint32_t)((it / C::ST) & 1))) {
                ok = false;
                break;
            }
            uint8_t* st = sm + s * C::STB;
            const uint8_t* at = st + C::AOP;
            const float* ut = reinterpret_cast<const float*>(st + C::AOP + C::ATB);
            if constexpr (F8) {
                // 16 samples per 16-byte store; u^T arrives divided by its
                // column's largest magnitude, so every product fits E4M3
#pragma unroll
                for (int g = 0; g < CH / 16; ++g) {
                    const uint4 av = *reinterpret_cast<const uint4*>(at + canon_off_b(a, g * 16, K_));
                    const uint32_t aw[4] = {av.x, av.y, av.z, av.w};
                    float x[16];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const float2 lo = e4m3x2_to_float2(aw[q] & 0xffffu), hi = e4m3x2_to_float2(aw[q] >> 16);
                        x[4 * q] = lo.x;
                        x[4 * q + 1] = lo.y;
                        x[4 * q + 2] = hi.x;
                        x[4 * q + 3] = hi.y;
                    }
#pragma unroll
                    for (int m = 0; m < C::MT; ++m) {
                        const int j = m * (128 / K_) + jr;
                        const float4* up = reinterpret_cast<const float4*>(ut + j * CH + g * 16);
                        const float4 u0 = up[0], u1 = up[1], u2 = up[2], u3 = up[3];
                        uint4 o;
                        o.x = pack_e4m3x4(u0.x * x[0], u0.y * x[1], u0.z * x[2], u0.w * x[3]);
                        o.y = pack_e4m3x4(u1.x * x[4], u1.y * x[5], u1.z * x[6], u1.w * x[7]);
                        o.z = pack_e4m3x4(u2.x * x[8], u2.y * x[9], u2.z * x[10], u2.w * x[11]);
                        o.w = pack_e4m3x4(u3.x * x[12], u3.y * x[13], u3.z * x[14], u3.w * x[15]);
                        *reinterpret_cast<uint4*>(st + m * (128 * CH) + canon_off_b(r, g * 16, 128)) = o;
                    }
                }
            } else {
#pragma unroll
                for (int g = 0; g < CH / 8; ++g) {
                    const uint4 av = *reinterpret_cast<const uint4*>(at + canon_off(a, g * 8, K_));
                    const __nv_bfloat162* ab = reinterpret_cast<const __nv_bfloat162*>(&av);
                    float x[8];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const float2 f = __bfloat1622float2(ab[q]);
                        x[2 * q] = f.x;
                        x[2 * q + 1] = f.y;
                    }
#pragma unroll
                    for (int m = 0; m < C::MT; ++m) {
                        const int j = m * (128 / K_) + jr;
                        const float4 u0 = *reinterpret_cast<const float4*>(ut + j * CH + g * 8);
                        const float4 u1 = *reinterpret_cast<const float4*>(ut + j * CH + g * 8 + 4);
                        uint4 o;
                        o.x = pack_bf16x2(u0.x * x[0], u0.y * x[1]);
                        o.y = pack_bf16x2(u0.z * x[2], u0.w * x[3]);
                        o.z = pack_bf16x2(u1.x * x[4], u1.y * x[5]);
                        o.w = pack_bf16x2(u1.z * x[6], u1.w * x[7]);
                        *reinterpret_cast<uint4*>(st + m * (128 * CH * 2) + canon_off(r, g * 8, 128)) = o;
                    }
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_arrive(smem_u32(&aready[s]));
        }
        if (!ok) s_fail = 1;
    }
    if (!ok) {
        s_fail = 1;
        atomicOr(err, ERR_WAIT_LIMIT);
    }
    __syncthreads();
    // epilogue (warps 0-3: TMEM lanes 32w..32w+31), or the drain after a failure
    if (warp < 4) {
        const bool fin = mbar_wait(smem_u32(&done), 0u);
        asm volatile("tcgen05.fence::after_thread_sync;");
        if (!fin) {
            if (lane == 0) atomicOr(err, ERR_WAIT_LIMIT);
        } else if (!s_fail) {
            float* M = Mpart + (size_t)blockIdx.x * (S_ * K_ * K_);
#pragma unroll 1
            for (int m = 0; m < C::MT; ++m) {
                const int row = m * 128 + warp * 32 + lane;
#pragma unroll
                for (int c = 0; c < K_; c += 16) {
                    uint32_t v[16];
                    if (cnt > 0) {
                        tmem_ld16_nw(tmem + ((uint32_t)(warp * 32) << 16) + m * K_ + c, v);
                        tmem_wait_ld();
                    } else {
#pragma unroll
                        for (int q = 0; q < 16; ++q) v[q] = 0u;  // an empty range adds nothing
                    }
                    float4* dst = reinterpret_cast<float4*>(M + (size_t)row * K_ + c);
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        dst[q] = make_float4(__uint_as_float(v[4 * q]), __uint_as_float(v[4 * q + 1]),
                                             __uint_as_float(v[4 * q + 2]), __uint_as_float(v[4 * q + 3]));
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, C::TMC);
}

// M = sum of the partials in CTA order (FP32, rows (j, a), columns b), and Mq
// = the same values as the quadratic-form operand: rows (j, b) in passes of
// 256, K = a, canonical BF16 (M_j is symmetric, so row (j, b) column a is
// D[(j, b), a]).
template <int K_>
__global__ void mstack_reduce_kernel(const float* __restrict__ Mpart, int parts, float* __restrict__ M,
                                     uint8_t* __restrict__ Mq) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    constexpr int count = S_ * K_ * K_;
    if (e >= count) return;
    float acc = 0.0f;
    for (int p = 0; p < parts; ++p) acc += Mpart[(size_t)p * count + e];
    M[e] = acc;
    const int row = e / K_, col = e % K_;
    const int pass = row / NP, rl = row % NP;
    *reinterpret_cast<__nv_bfloat16*>(Mq + (size_t)pass * (NP * K_ * 2) + canon_off(rl, col, NP)) =
        __float2bfloat16_rn(acc);
}

// FP8 form: one warp per row R = (j, x) of the stack.  M[R][y] = U_j s_x s_y
// D[R][y] (the partials summed in CTA order; U_j = the largest |u| of column
// j, s = the factor's column scales), and the quadratic-form operand row
// (j, x), K = y: E4M3(M[R][y] s_y / t_R) with t_R = max_y |M[R][y] s_y| / 448
// kept in tq.
template <int K_>
__global__ void mstack_reduce8_kernel(const float* __restrict__ Mpart, int parts, const unsigned* __restrict__ umax,
                                      const float* __restrict__ sA, float* __restrict__ M, uint8_t* __restrict__ Mq,
                                      float* __restrict__ tq) {
    const int R = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    constexpr int count = S_ * K_ * K_;
    constexpr int PL = K_ / 32;  // columns per lane
    if (R >= S_ * K_) return;
    const int j = R / K_, x = R % K_;
    const float sc = __uint_as_float(umax[j]) * sA[x];
    float v[PL];
    float amax = 0.0f;
#pragma unroll
    for (int q = 0; q < PL; ++q) {
        const int y = q * 32 + lane;
        float acc = 0.0f;
        for (int p = 0; p < parts; ++p) acc += Mpart[(size_t)p * count + (size_t)R * K_ + y];
        const float m = acc * sc * sA[y];
        M[(size_t)R * K_ + y] = m;
        v[q] = m * sA[y];
        amax = fmaxf(amax, fabsf(v[q]));
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, d));
    const float t = amax > 0.0f ? amax / 448.0f : 1.0f;
    const int pass = R / NP, rl = R % NP;
#pragma unroll
    for (int q = 0; q < PL; ++q) {
        const int y = q * 32 + lane;
        Mq[(size_t)pass * (NP * K_) + canon_off_b(rl, y, NP)] =
            (uint8_t)(__nv_cvt_float2_to_fp8x2(make_float2(v[q] / t, 0.0f), __NV_SATFINITE, __NV_E4M3) & 0xffu);
    }
    if (lane == 0) tq[R] = t;
}

// ---------------------------------------------------------------------------
// Quadratic forms

template <int K_, bool F8>
struct QfCfg {
    static constexpr int EB = F8 ? 1 : 2;        // bytes per operand element
    static constexpr int PASSES = S_ * K_ / NP;  // 4 or 2
    static constexpr int JP = NP / K_;           // j per pass
    static constexpr uint32_t MQB = S_ * K_ * K_ * EB;
    static constexpr uint32_t AQB = 128 * K_ * EB;
    static constexpr int ST = 2;
    static constexpr uint32_t SMEM = MQB + ST * AQB;
};

// 192 threads: warps 0-3 epilogue (tile rows 32w..32w+31), warp 4 lane 0
// loads, warp 5 lane 0 issues the MMAs.  CTA b takes tiles b, b + grid, ...
template <int K_, bool F8>
__global__ void __launch_bounds__(192, 1) quadform_tc_kernel(const uint8_t* __restrict__ Aq,
                                                            const uint8_t* __restrict__ Mq,
                                                            const float* __restrict__ A, int n, int ntiles,
                                                            const float* __restrict__ tq, float* __restrict__ T2,
                                                            uint32_t* __restrict__ err) {
    using C = QfCfg<K_, F8>;
    __shared__ float s_tq[F8 ? S_ * K_ : 1];  // FP8 form: the stack rows' scales
    if constexpr (F8)
        for (int e = threadIdx.x; e < S_ * K_; e += blockDim.x) s_tq[e] = tq[e];
    extern __shared__ __align__(1024) uint8_t sm[];
    __shared__ __align__(8) uint64_t mq_full, afull[C::ST], aempty[C::ST], tfull[2], tempty[2], done;
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int my_tiles = blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    if (warp == 0) tmem_alloc(smem_u32(&tmem_base), 2 * NP);
    if (tid == 0) {
        mbar_init(smem_u32(&mq_full), 1);
        for (int s = 0; s < C::ST; ++s) {
            mbar_init(smem_u32(&afull[s]), 1);
            mbar_init(smem_u32(&aempty[s]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(&tfull[b]), 1);
            mbar_init(smem_u32(&tempty[b]), 4);
        }
        mbar_init(smem_u32(&done), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;
    const uint32_t base = smem_u32(sm);
    const uint32_t abase = base + C::MQB;
    bool ok = true;
    if (warp == 4) {
        if (lane == 0 && my_tiles > 0) {
            mbar_expect_tx(smem_u32(&mq_full), C::MQB);
            bulk_g2s(base, Mq, C::MQB, smem_u32(&mq_full));
            int it = 0;
            for (; it < my_tiles; ++it) {
                const int s = it % C::ST;
                if (it >= C::ST && !mbar_wait(smem_u32(&aempty[s]), (uint32_t)((it / C::ST - 1) & 1))) {
                    ok = false;
                    break;
                }
                const int q = blockIdx.x + it * gridDim.x;
                mbar_expect_tx(smem_u32(&afull[s]), C::AQB);
                bulk_g2s(abase + s * C::AQB, Aq + (size_t)q * C::AQB, C::AQB, smem_u32(&afull[s]));
            }
            mbar_wait(smem_u32(&mq_full), 0u);
            for (int q = max(0, it - C::ST); q < it; ++q)
                mbar_wait(smem_u32(&afull[q % C::ST]), (uint32_t)((q / C::ST) & 1));
        }
    } else if (warp == 5) {
        if (lane == 0 && my_tiles > 0) {
            constexpr uint32_t idesc = F8 ? idesc_e4m3_f32(128, NP) : idesc_bf16_f32(128, NP);
            ok = mbar_wait(smem_u32(&mq_full), 0u);
            int pc = 0;  // passes issued
            for (int it = 0; it < my_tiles && ok; ++it) {
                const int s = it % C::ST;
                if (!mbar_wait(smem_u32(&afull[s]), (uint32_t)((it / C::ST) & 1))) {
                    ok = false;
                    break;
                }
                for (int p = 0; p < C::PASSES && ok; ++p, ++pc) {
                    const int b = pc & 1;
                    if (pc >= 2 && !mbar_wait(smem_u32(&tempty[b]), (uint32_t)((pc / 2 - 1) & 1))) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
                    for (int ks = 0; ks < K_ * C::EB / 32; ++ks)
                        mma_op<F8>(tmem + b * NP, umma_desc(abase + s * C::AQB + ks * (128 * 32)),
                                   umma_desc(base + p * (NP * K_ * C::EB) + ks * (NP * 32)), idesc, ks > 0 ? 1u : 0u);
                    mma_commit(smem_u32(&tfull[b]));
                }
                if (ok) mma_commit(smem_u32(&aempty[s]));  // the A tile is free once these MMAs finish
            }
        }
        if (lane == 0) mma_commit(smem_u32(&done));  // arrives once every MMA issued above has finished
    } else {
        int pc = 0;
        for (int it = 0; it < my_tiles && ok; ++it) {
            const int q = blockIdx.x + it * gridDim.x;
            const int i = q * 128 + warp * 32 + lane;
            float arow[K_];
            const float4* ar = reinterpret_cast<const float4*>(A + (size_t)i * K_);
#pragma unroll
            for (int c = 0; c < K_ / 4; ++c) {
                const float4 v = i < n ? __ldg(ar + c) : make_float4(0.f, 0.f, 0.f, 0.f);
                arow[4 * c] = v.x;
                arow[4 * c + 1] = v.y;
                arow[4 * c + 2] = v.z;
                arow[4 * c + 3] = v.w;
            }
#pragma unroll 1
            for (int p = 0; p < C::PASSES; ++p, ++pc) {
                const int b = pc & 1;
                if (!mbar_wait(smem_u32(&tfull[b]), (uint32_t)((pc / 2) & 1))) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll 1
                for (int jj = 0; jj < C::JP; ++jj) {
                    float acc = 0.0f;
                    const float* tr = s_tq + (F8 ? (p * C::JP + jj) * K_ : 0);
#pragma unroll
                    for (int c = 0; c < K_; c += 32) {
                        uint32_t v0[16], v1[16];
                        const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16) + b * NP + jj * K_ + c;
                        tmem_ld16_nw(ta, v0);
                        tmem_ld16_nw(ta + 16, v1);
                        tmem_wait_ld();
                        if constexpr (F8) {
                            // the FP8 stack rows carry a scale each (D = t D')
#pragma unroll
                            for (int e = 0; e < 16; ++e)
                                acc = fmaf(__uint_as_float(v0[e]), arow[c + e] * tr[c + e], acc);
#pragma unroll
                            for (int e = 0; e < 16; ++e)
                                acc = fmaf(__uint_as_float(v1[e]), arow[c + 16 + e] * tr[c + 16 + e], acc);
                        } else {
#pragma unroll
                            for (int e = 0; e < 16; ++e) acc = fmaf(__uint_as_float(v0[e]), arow[c + e], acc);
#pragma unroll
                            for (int e = 0; e < 16; ++e) acc = fmaf(__uint_as_float(v1[e]), arow[c + 16 + e], acc);
                        }
                    }
                    if (i < n) T2[(size_t)i * S_ + p * C::JP + jj] = acc;
                }
                asm volatile("tcgen05.fence::before_thread_sync;");
                __syncwarp();
                if (lane == 0) mbar_arrive(smem_u32(&tempty[b]));
            }
        }
    }
    if (!ok && (lane == 0)) atomicOr(err, ERR_WAIT_LIMIT);
    __syncthreads();
    // every MMA has finished before TMEM is freed (bounded wait)
    if (warp == 5 && lane == 0) mbar_wait(smem_u32(&done), 0u);
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, 2 * NP);
}

}  // namespace

// Packed forms of the factor A for one MDS call (pack_factor_tc) and the
// products with them.  With sA (the FP8 form) the operands are E4M3 bytes of
// A / sA with sA = the column scales, written there; otherwise BF16.
rfx_status pack_factor_tc(Ctx* c, const float* dA, int k, uint8_t* Aq, uint8_t* At, float* sA) {
    const int n = c->n;
    const int ntiles = (n + 127) / 128, nch = (n + CH - 1) / CH;
    cudaStream_t s = c->stream;
    if (k != 64 && k != 32) {
        set_error("tensor-core factor MDS supports rank 32 or 64");
        return RFX_ERR_UNSUPPORTED;
    }
    if (sA) {
        Scratch sc(c);
        unsigned* mx = sc.get<unsigned>((size_t)k);
        if (!mx) {
            set_error("tensor-core factor MDS: scratch allocation failed");
            return RFX_ERR_OOM;
        }
        RFX_CUDA(cudaMemsetAsync(mx, 0, sizeof(unsigned) * k, s));
        col_absmax_kernel<<<col_absmax_grid(n, k), CAM_THREADS, 0, s>>>(dA, n, k, mx);
        col_scale_kernel<<<1, 64, 0, s>>>(mx, k, sA);
        const size_t tq = (size_t)ntiles * 128 * (k / 16), ta = (size_t)nch * k * (CH / 16);
        if (k == 64) {
            pack_aq8_kernel<64><<<(unsigned)((tq + 255) / 256), 256, 0, s>>>(dA, sA, n, ntiles, Aq);
            pack_at8_kernel<64><<<(unsigned)((ta + 255) / 256), 256, 0, s>>>(dA, sA, n, nch, At);
        } else {
            pack_aq8_kernel<32><<<(unsigned)((tq + 255) / 256), 256, 0, s>>>(dA, sA, n, ntiles, Aq);
            pack_at8_kernel<32><<<(unsigned)((ta + 255) / 256), 256, 0, s>>>(dA, sA, n, nch, At);
        }
        c->launches += 4;
        RFX_CUDA(cudaGetLastError());
        return RFX_OK;
    }
    const size_t tq = (size_t)ntiles * 128 * (k / 8), ta = (size_t)nch * k * (CH / 8);
    if (k == 64) {
        pack_aq_kernel<64><<<(unsigned)((tq + 255) / 256), 256, 0, s>>>(dA, n, ntiles, Aq);
        pack_at_kernel<64><<<(unsigned)((ta + 255) / 256), 256, 0, s>>>(dA, n, nch, At);
    } else {
        pack_aq_kernel<32><<<(unsigned)((tq + 255) / 256), 256, 0, s>>>(dA, n, ntiles, Aq);
        pack_at_kernel<32><<<(unsigned)((ta + 255) / 256), 256, 0, s>>>(dA, n, nch, At);
    }
    c->launches += 2;
    RFX_CUDA(cudaGetLastError());
    return RFX_OK;
}

size_t factor_tc_aq_bytes(int n, int k) { return (size_t)((n + 127) / 128) * 128 * k * 2; }
size_t factor_tc_at_bytes(int n, int k) { return (size_t)((n + CH - 1) / CH) * CH * k * 2; }

// M (S x k x k) and T2 (n x S) for the factor A (n x k, with its packed forms
// Aq / At from pack_factor_tc; sA its FP8 column scales, null for BF16) and
// the centred block u (n x S), on the tensor cores.
rfx_status launch_factor_ops_tc(Ctx* c, const float* dA, int k, const uint8_t* Aq, const uint8_t* At,
                                const float* sA, const float* u32, float* M, float* T2) {
    cudaStream_t s = c->stream;
    const int n = c->n;
    const int ntiles = (n + 127) / 128, nch = (n + CH - 1) / CH;
    int sms = 148;
    RFX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
    const int per = (nch + sms - 1) / sms;
    const int parts = (nch + per - 1) / per;
    const int qgrid = std::min(ntiles, sms);
    const bool f8 = sA != nullptr;
    Scratch sc(c);
    const size_t count = (size_t)S_ * k * k;
    float* Mpart = sc.get<float>(count * parts);
    float* uT = sc.get<float>((size_t)nch * CH * S_);
    uint8_t* Mq = sc.get<uint8_t>(count * 2);
    unsigned* umax = f8 ? sc.get<unsigned>(S_) : nullptr;
    float* tq = f8 ? sc.get<float>((size_t)S_ * k) : nullptr;
    if (!Mpart || !uT || !Mq || (f8 && (!umax || !tq))) {
        set_error("tensor-core factor MDS: scratch allocation failed");
        return RFX_ERR_OOM;
    }
    if (f8) {
        RFX_CUDA(cudaMemsetAsync(umax, 0, sizeof(unsigned) * S_, s));
        col_absmax_kernel<<<col_absmax_grid(n, S_), CAM_THREADS, 0, s>>>(u32, n, S_, umax);
        c->launches += 1;
    }
    pack_ut_kernel<<<(unsigned)(((size_t)nch * CH * S_ + 255) / 256), 256, 0, s>>>(u32, n, nch, umax, uT);
    auto run = [&](auto mk, auto qk, uint32_t sm_m, uint32_t sm_q, auto reduce) -> rfx_status {
        RFX_CUDA(cudaFuncSetAttribute(mk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_m));
        RFX_CUDA(cudaFuncSetAttribute(qk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_q));
        mk<<<parts, 192, sm_m, s>>>(At, uT, nch, per, Mpart, c->d_err);
        reduce();
        qk<<<qgrid, 192, sm_q, s>>>(Aq, Mq, dA, n, ntiles, tq, T2, c->d_err);
        RFX_CUDA(cudaGetLastError());
        return RFX_OK;
    };
    // BF16: M and Mq element by element; FP8: a warp per stack row (scales)
    auto red16 = [&](auto rk) {
        return [&, rk]() { rk<<<(unsigned)((count + 255) / 256), 256, 0, s>>>(Mpart, parts, M, Mq); };
    };
    auto red8 = [&](auto rk) {
        return [&, rk]() { rk<<<(unsigned)(((size_t)S_ * k * 32 + 255) / 256), 256, 0, s>>>(Mpart, parts, umax, sA, M, Mq, tq); };
    };
    rfx_status st;
    if (k == 64 && f8)
        st = run(mstack_tc_kernel<64, true>, quadform_tc_kernel<64, true>, MsCfg<64, true>::SMEM,
                 QfCfg<64, true>::SMEM, red8(mstack_reduce8_kernel<64>));
    else if (k == 32 && f8)
        st = run(mstack_tc_kernel<32, true>, quadform_tc_kernel<32, true>, MsCfg<32, true>::SMEM,
                 QfCfg<32, true>::SMEM, red8(mstack_reduce8_kernel<32>));
    else if (k == 64)
        st = run(mstack_tc_kernel<64, false>, quadform_tc_kernel<64, false>, MsCfg<64, false>::SMEM,
                 QfCfg<64, false>::SMEM, red16(mstack_reduce_kernel<64>));
    else if (k == 32)
        st = run(mstack_tc_kernel<32, false>, quadform_tc_kernel<32, false>, MsCfg<32, false>::SMEM,
                 QfCfg<32, false>::SMEM, red16(mstack_reduce_kernel<32>));
    else {
        set_error("tensor-core factor MDS supports rank 32 or 64");
        return RFX_ERR_UNSUPPORTED;
    }
    if (st != RFX_OK) return st;
    c->launches += 4;
    return RFX_OK;
}

}  // namespace rfx
