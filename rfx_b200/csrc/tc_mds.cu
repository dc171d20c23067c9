// Tensor-core (tcgen05, BF16 inputs, FP32 accumulation in TMEM) kernels of the
// factor-space MDS operator (mds.cu):
//
//   mstack_tc_kernel:   M_j = A^T diag(u_j) A for all j, as one GEMM
//                       D[(j,a), b] = sum_i (u_ij A_ia) A_ib, M = s*k rows,
//                       N = k, reduction over the n samples split across CTAs
//                       (each CTA owns one 128-row M tile and one K range and
//                       writes its FP32 tile to its own slot of a partial
//                       stack; mstack_reduce_kernel adds the slots in K-range
//                       order, so the result does not depend on CTA timing).
//   quadform_tc_kernel: T2_ij = a_i^T M_j a_i: D[i, (j,b)] = sum_a A_ia M_j[b][a]
//                       for a 128-sample tile in TMEM, then the epilogue reads
//                       each row from TMEM and dots every 64-column block with
//                       a_i; the n x (s*k) product never leaves the SM.
//
// Operands are staged in shared memory by the CTA's threads in the canonical
// K-major, no-swizzle UMMA layout: 8-row x 16-byte core matrices, the two
// 8-element K halves of a 16-wide K step 128 bytes apart (leading byte offset)
// and consecutive 8-row groups 256 bytes apart (stride byte offset).  One
// elected thread issues tcgen05.mma and commits to an mbarrier; two operand
// stages let the next tile be built while the tensor core works.  Every
// mbarrier wait is bounded and records a timeout in the error word.
#include <cuda_bf16.h>

#include "rfx_internal.cuh"

namespace rfx {
namespace {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)(256u >> 4) << 32) |
           (1ull << 46);
}

__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// byte offset of (row r, k) inside an R-row tile of 64 K: four 16-wide K steps
// of R*32 bytes each
__device__ __forceinline__ uint32_t tile_off(int r, int k, int R) {
    return (uint32_t)((k >> 4) * (R * 32) + (r >> 3) * 256 + ((k >> 3) & 1) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar));
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count));
}

// bounded wait for phase `parity` of the mbarrier
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    for (int it = 0; it < (1 << 22); ++it) {
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

__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;");
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

constexpr int TC_THREADS = 128;
constexpr int KCH = 64;  // samples per K chunk

// grid: (s*k/128 M tiles, K splits); k in {16, 32, 64}; u is n x S (S = 16)
template <int K_, int S_>
__global__ void __launch_bounds__(TC_THREADS) mstack_tc_kernel(const float* __restrict__ A, const float* __restrict__ u,
                                                              int n, float* __restrict__ Mpart,
                                                              uint32_t* __restrict__ err) {
    constexpr int JT = 128 / K_;  // j values per M tile
    constexpr uint32_t A_BYTES = 128 * KCH * 2, B_BYTES = K_ * KCH * 2;
    constexpr uint32_t TM_COLS = K_ < 32 ? 32 : K_;
    extern __shared__ __align__(1024) uint8_t sm[];  // 2 * (A_BYTES + B_BYTES)
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int j0 = blockIdx.x * JT;
    const int chunks = (n + KCH - 1) / KCH;
    const int per = (chunks + gridDim.y - 1) / gridDim.y;
    const int c0 = blockIdx.y * per, c1 = min(chunks, c0 + per);
    if (warp == 0) tmem_alloc(smem_u32(&tmem_base), TM_COLS);
    if (tid == 0) {
        mbar_init(smem_u32(&mbar[0]), 1);
        mbar_init(smem_u32(&mbar[1]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;
    constexpr uint32_t idesc = idesc_bf16_f32(128, K_);
    uint32_t phase[2] = {0u, 0u};
    bool ok = true;
    int it = 0;
    for (int ch = c0; ch < c1; ++ch, ++it) {
        const int st = it & 1;
        uint8_t* As = sm + st * (A_BYTES + B_BYTES);
        uint8_t* Bs = As + A_BYTES;
        if (it >= 2) {  // the MMAs that read this stage must have finished
            ok = ok && mbar_wait(smem_u32(&mbar[st]), phase[st]);
            phase[st] ^= 1u;
        }
        // build the tiles: thread -> (sample kk, half of the a range)
        const int kk = tid & 63, half = tid >> 6;
        const int i = ch * KCH + kk;
        const bool valid = i < n;
        float uj[JT];
#pragma unroll
        for (int jj = 0; jj < JT; ++jj) uj[jj] = valid ? u[(size_t)i * S_ + j0 + jj] : 0.0f;
#pragma unroll 4
        for (int a = half * (K_ / 2); a < (half + 1) * (K_ / 2); ++a) {
            const float x = valid ? A[(size_t)i * K_ + a] : 0.0f;
            *reinterpret_cast<__nv_bfloat16*>(Bs + tile_off(a, kk, K_)) = __float2bfloat16_rn(x);
#pragma unroll
            for (int jj = 0; jj < JT; ++jj)
                *reinterpret_cast<__nv_bfloat16*>(As + tile_off(jj * K_ + a, kk, 128)) =
                    __float2bfloat16_rn(uj[jj] * x);
        }
        asm volatile("fence.proxy.async.shared::cta;");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
            for (int ks = 0; ks < KCH / 16; ++ks) {
                const uint64_t ad = umma_desc(smem_u32(As) + ks * 128 * 32);
                const uint64_t bd = umma_desc(smem_u32(Bs) + ks * K_ * 32);
                mma_bf16(tmem, ad, bd, idesc, (it > 0 || ks > 0) ? 1u : 0u);
            }
            mma_commit(smem_u32(&mbar[st]));
        }
        __syncwarp();
    }
    // drain: each used stage has exactly one commit not yet waited for
    const int issued = it;
    for (int st = 0; st < 2; ++st)
        if (issued > st) {
            ok = ok && mbar_wait(smem_u32(&mbar[st]), phase[st]);
            phase[st] ^= 1u;
        }
    asm volatile("tcgen05.fence::after_thread_sync;");
    // this K range's slot of the partial stack
    float* M = Mpart + (size_t)blockIdx.y * S_ * K_ * K_;
    const int r = warp * 32 + lane;
    const int j = j0 + r / K_, a = r % K_;
    if (!ok) {
        if (lane == 0) atomicOr(err, ERR_WAIT_LIMIT);
    } else if (issued > 0) {
        // warp w reads TMEM lanes 32w..32w+31 = tile rows; K_ columns
#pragma unroll
        for (int c = 0; c < K_; c += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + c, v);
            float4* dst = reinterpret_cast<float4*>(M + ((size_t)j * K_ + a) * K_ + c);
#pragma unroll
            for (int q = 0; q < 4; ++q) dst[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        }
    } else {
        for (int c = 0; c < K_; ++c) M[((size_t)j * K_ + a) * K_ + c] = 0.0f;  // an empty K range adds nothing
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, TM_COLS);
}

// M = sum over the K ranges of their partial stacks, in K-range order
__global__ void mstack_reduce_kernel(const float* __restrict__ Mpart, int parts, size_t count, float* __restrict__ M) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count) return;
    float acc = 0.0f;
    for (int p = 0; p < parts; ++p) acc += Mpart[(size_t)p * count + e];
    M[e] = acc;
}

// grid: n/128 sample tiles; the s*k rows of the M stack in passes of NP rows
template <int K_, int S_>
__global__ void __launch_bounds__(TC_THREADS) quadform_tc_kernel(const float* __restrict__ A,
                                                                const float* __restrict__ M, int n,
                                                                float* __restrict__ T2, uint32_t* __restrict__ err) {
    constexpr int NP = 256;                 // N per pass
    constexpr int JP = NP / K_;             // j per pass
    constexpr int PASSES = (S_ * K_) / NP;  // >= 1
    constexpr uint32_t A_BYTES = 128 * K_ * 2, B_BYTES = NP * K_ * 2;
    extern __shared__ __align__(1024) uint8_t sm[];  // A_BYTES + B_BYTES
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    static_assert(K_ % 16 == 0 && (S_ * K_) % NP == 0, "tile shape");
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int i0 = blockIdx.x * 128;
    uint8_t* As = sm;
    uint8_t* Bs = sm + A_BYTES;
    if (warp == 0) tmem_alloc(smem_u32(&tmem_base), NP);
    if (tid == 0) {
        mbar_init(smem_u32(&mbar), 1);
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    // A tile: 128 samples x K_ (the a index is the reduction)
    const int i = i0 + tid;
    float arow[K_];
#pragma unroll
    for (int a = 0; a < K_; ++a) arow[a] = i < n ? A[(size_t)i * K_ + a] : 0.0f;
    // tile_off assumes 64-wide K; with K_ < 64 only the first K_/16 steps exist
#pragma unroll
    for (int a = 0; a < K_; ++a)
        *reinterpret_cast<__nv_bfloat16*>(As + tile_off(tid, a, 128)) = __float2bfloat16_rn(arow[a]);
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;
    constexpr uint32_t idesc = idesc_bf16_f32(128, NP);
    uint32_t phase = 0;
    bool ok = true;
    for (int ps = 0; ps < PASSES; ++ps) {
        // B tile: rows (j, b) of this pass, K = a: M[j][b][a]
        for (int e = tid; e < NP * K_; e += TC_THREADS) {
            const int row = e / K_, a = e % K_;
            const int j = ps * JP + row / K_, b = row % K_;
            *reinterpret_cast<__nv_bfloat16*>(Bs + tile_off(row, a, NP)) =
                __float2bfloat16_rn(M[((size_t)j * K_ + b) * K_ + a]);
        }
        asm volatile("fence.proxy.async.shared::cta;");
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
            for (int ks = 0; ks < K_ / 16; ++ks)
                mma_bf16(tmem, umma_desc(smem_u32(As) + ks * 128 * 32), umma_desc(smem_u32(Bs) + ks * NP * 32), idesc,
                         ks > 0 ? 1u : 0u);
            mma_commit(smem_u32(&mbar));
        }
        __syncwarp();
        ok = ok && mbar_wait(smem_u32(&mbar), phase);
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;");
        if (ok) {
            float t[JP];
#pragma unroll
            for (int jj = 0; jj < JP; ++jj) t[jj] = 0.0f;
#pragma unroll
            for (int c = 0; c < NP; c += 16) {
                float v[16];
                tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + c, v);
                const int jj = c / K_, b0 = c % K_;
#pragma unroll
                for (int q = 0; q < 16; ++q) t[jj] = fmaf(v[q], arow[b0 + q], t[jj]);
            }
            if (i < n)
#pragma unroll
                for (int jj = 0; jj < JP; ++jj) T2[(size_t)i * S_ + ps * JP + jj] = t[jj];
        }
        // all TMEM reads and B-tile reads of this pass are done before the next
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
    }
    if (!ok && lane == 0) atomicOr(err, ERR_WAIT_LIMIT);
    if (warp == 0) tmem_dealloc(tmem, NP);
}

}  // namespace

// M (S x k x k, zeroed here) and T2 (n x S) for the factor A (n x k) and the
// centred block u (n x S), on the tensor cores.
rfx_status launch_factor_ops_tc(Ctx* c, const float* dA, int k, const float* u32, float* M, float* T2) {
    cudaStream_t s = c->stream;
    const int n = c->n;
    constexpr int S = 16;
    const int ksplit = 37;  // 296 CTAs for rank 64: two per SM
    Scratch sc(c);
    const size_t count = (size_t)S * k * k;
    float* Mpart = sc.get<float>(count * ksplit);
    if (!Mpart) {
        set_error("tensor-core factor MDS: scratch allocation failed");
        return RFX_ERR_OOM;
    }
    auto run = [&](auto mk, auto qk, int K) -> rfx_status {
        const int sm_m = 2 * (128 * KCH * 2 + K * KCH * 2);
        const int sm_q = 128 * K * 2 + 256 * K * 2;
        RFX_CUDA(cudaFuncSetAttribute(mk, cudaFuncAttributeMaxDynamicSharedMemorySize, sm_m));
        RFX_CUDA(cudaFuncSetAttribute(qk, cudaFuncAttributeMaxDynamicSharedMemorySize, sm_q));
        mk<<<dim3(S * K / 128, ksplit), TC_THREADS, sm_m, s>>>(dA, u32, n, Mpart, c->d_err);
        mstack_reduce_kernel<<<(unsigned)((count + 255) / 256), 256, 0, s>>>(Mpart, ksplit, count, M);
        qk<<<(n + 127) / 128, TC_THREADS, sm_q, s>>>(dA, M, n, T2, c->d_err);
        RFX_CUDA(cudaGetLastError());
        return RFX_OK;
    };
    rfx_status st = RFX_OK;
    switch (k) {
        case 64:
            st = run(mstack_tc_kernel<64, S>, quadform_tc_kernel<64, S>, 64);
            break;
        case 32:
            st = run(mstack_tc_kernel<32, S>, quadform_tc_kernel<32, S>, 32);
            break;
        default:
            set_error("tensor-core factor MDS supports rank 32 or 64");
            return RFX_ERR_UNSUPPORTED;
    }
    if (st != RFX_OK) return st;
    c->launches += 3;
    return RFX_OK;
}

}  // namespace rfx
