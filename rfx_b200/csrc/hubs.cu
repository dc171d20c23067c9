// Hub leaves of the exact pair counts on the tensor cores.
//
// cpu_proximity's dense branch (src/rf_proximity.cpp:173-230) adds 1 to
// C[i][j] for every OOB i and in-bag j of the same leaf; S = C + C^T.  At the
// benchmarked sizes a few hundred leaves of the whole forest carry most of the
// pair updates (n = 50,000, 1,000 trees: the 255 leaves with the largest
// OOB x in-bag products carry 77 % of 2.42e9), because OOB rows that the
// reference's routing sends right at every categorical split pile up in a few
// leaves per tree.  For those "hub" leaves h (OOB member set A_h, in-bag member
// set B_h) the counts are
//     S_hub = ZA ZB^T + ZB ZA^T = X Y^T,  X = [ZA | ZB],  Y = [ZB | ZA]
// with 0/1 indicator matrices ZA, ZB (n x H).  That is an integer GEMM, which
// tcgen05.mma kind::i8 (u8 x u8, s32 accumulators in TMEM) computes exactly.
// A pair gains at most 1 per hub (a sample is OOB or in-bag in a tree, not
// both), so S_hub <= H <= 255 and is stored as one byte per entry.  The row
// kernel (prox.cu) starts each row's counters from S_hub and counts the other
// leaves only; the hub leaves' two keys are flagged so that their ranges are
// left out there.  The split changes which kernel counts a pair, never the
// count: results are bit-identical with or without the tensor-core part.
//
// Kernels:
//   hub_hist_kernel  per tree: each leaf's product a*b of OOB and in-bag member
//                    counts (from the leaf lists' key offsets), binned on a
//                    log scale (8 bins per power of two) into a histogram,
//                    for leaves with a*b >= the break-even product.
//   hub_pick_kernel  one CTA: the lowest bin such that the leaves in it and
//                    above number at most HUB_MAX.
//   hub_mark_kernel  per tree: those leaves get a hub number, their two keys
//                    are flagged, their a*b is added to the pair counter.
//   hub_z_kernel     per hub: 1s into X (layout below) for its members.
//   hub_gemm_kernel  persistent, one CTA per SM: the upper-triangle tiles of
//                    S_hub, 128 rows x 256 columns each.
//
// X in global memory: 256-row blocks, each made of 128-byte K chunks of
// 32 KB in the canonical K-major no-swizzle UMMA layout (core matrices of
// 8 rows x 16 bytes; byte (r, kb) of a chunk at (kb / 16) * 4096 + r * 16 +
// kb % 16).  Row width Kx = 2 * Hpad bytes, Hpad = 128 or 256 (hub columns
// past the hub count stay 0).  Y's K chunk c is X's chunk (c + Kc/2) mod Kc,
// so one matrix serves both operands.
//   A operand (rows of the tile): 128 rows x Kx, brought in once per row block
//     by Kx/16 bulk copies of 2 KB (one 16-byte K slice of 128 rows each).
//   B operand (columns of the tile): one 32 KB bulk copy per K chunk, three
//     stages.
// S_hub tiles: the upper-triangle tiles (I, J), row block I = 128 rows, column
// tile J = 256 columns, J >= I / 2, stored one after another in row-block
// order, 32 KB each: row r at r * 256, its 16-byte chunk q (columns 16q..16q+15
// of the tile) at slot q ^ (r % 16) (so that the epilogue's shared-memory
// stores are free of bank conflicts); written by one bulk store per tile.
//
// Every mbarrier wait is bounded; a wait that gives up raises ERR_WAIT_LIMIT,
// makes the CTA stop issuing work, and the CTA still waits (bounded) for the
// copies and tensor-core work it started before it frees TMEM and exits.
#include <algorithm>
#include <cstdlib>

#include "rfx_internal.cuh"

namespace rfx {
namespace {

constexpr int HUB_MAX = 255;  // S_hub entries stay <= 255 (one byte)
constexpr int HUB_BINS = 8 * 64;
constexpr int HG_THREADS = 192;      // warp 0 loads, warp 1 issues MMAs, warps 2-5 epilogue
constexpr int HG_STAGES = 3;
constexpr uint32_t HG_CHUNK = 32768; // 256 rows x 128 bytes
constexpr uint32_t HG_A_MAX = 65536; // 128 rows x 512 bytes
constexpr uint32_t HG_OUT = 32768;   // 128 x 256 bytes
constexpr uint32_t HG_SMEM = HG_A_MAX + HG_STAGES * HG_CHUNK + 2 * HG_OUT + 1024;  // + alignment slack

__device__ __forceinline__ int hub_bin(unsigned long long prod) {
    const int lz = 63 - __clzll((long long)prod);
    const int frac = lz >= 3 ? (int)((prod >> (lz - 3)) & 7ull) : (int)((prod << (3 - lz)) & 7ull);
    return 8 * lz + frac;
}

__global__ void hub_hist_kernel(const int64_t* __restrict__ segbase, const int32_t* __restrict__ segoff,
                                unsigned long long min_prod, uint32_t* __restrict__ hist) {
    __shared__ uint32_t h[HUB_BINS];
    for (int k = threadIdx.x; k < HUB_BINS; k += blockDim.x) h[k] = 0;
    __syncthreads();
    const int t = blockIdx.x;
    const int64_t sb = segbase[t];
    const int L = (int)((segbase[t + 1] - sb - 1) >> 1);
    const int32_t* so = segoff + sb;
    for (int l = threadIdx.x; l < L; l += blockDim.x) {
        const unsigned long long a = (unsigned long long)(so[2 * l + 1] - so[2 * l]);
        const unsigned long long b = (unsigned long long)(so[2 * l + 2] - so[2 * l + 1]);
        const unsigned long long pr = a * b;
        if (pr >= min_prod && pr > 0) atomicAdd(&h[hub_bin(pr)], 1u);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < HUB_BINS; k += blockDim.x)
        if (h[k]) atomicAdd(hist + k, h[k]);
}

// state[0] = threshold bin, state[1] = hub count (filled by hub_mark_kernel)
__global__ void hub_pick_kernel(const uint32_t* __restrict__ hist, int hub_max, int32_t* __restrict__ state) {
    if (threadIdx.x != 0) return;
    uint32_t cum = 0;
    int thr = HUB_BINS;
    for (int k = HUB_BINS - 1; k >= 0; --k) {
        if (cum + hist[k] > (uint32_t)hub_max) break;
        cum += hist[k];
        thr = k;
    }
    state[0] = thr;
    state[1] = 0;
}

__global__ void hub_mark_kernel(const int64_t* __restrict__ segbase, const int32_t* __restrict__ segoff,
                                unsigned long long min_prod, int hub_max, int32_t* __restrict__ state,
                                int2* __restrict__ hubs, uint8_t* __restrict__ keyflag,
                                unsigned long long* __restrict__ pairs) {
    const int t = blockIdx.x;
    const int thr = state[0];
    const int64_t sb = segbase[t];
    const int L = (int)((segbase[t + 1] - sb - 1) >> 1);
    const int32_t* so = segoff + sb;
    unsigned long long mine = 0;
    for (int l = threadIdx.x; l < L; l += blockDim.x) {
        const unsigned long long a = (unsigned long long)(so[2 * l + 1] - so[2 * l]);
        const unsigned long long b = (unsigned long long)(so[2 * l + 2] - so[2 * l + 1]);
        const unsigned long long pr = a * b;
        if (pr >= min_prod && pr > 0 && hub_bin(pr) >= thr) {
            const int h = atomicAdd(state + 1, 1);
            if (h < hub_max) {  // always true: the picked bins hold at most hub_max leaves
                hubs[h] = make_int2(t, l);
                keyflag[sb + 2 * l] = 1;
                keyflag[sb + 2 * l + 1] = 1;
                mine += pr;
            }
        }
    }
    if (pairs && mine) atomicAdd(pairs, mine);
}

__device__ __forceinline__ int hub_pad(int count) { return count <= 128 ? 128 : 256; }

// byte offset of X[row j][column kb] (Kx = 2 * Hpad bytes per row)
__device__ __forceinline__ size_t xoff(int j, int kb, int Kx) {
    return (size_t)(j >> 8) * (256u * (size_t)Kx) + (size_t)(kb >> 7) * HG_CHUNK + ((kb & 127) >> 4) * 4096 +
           (j & 255) * 16 + (kb & 15);
}

__global__ void hub_z_kernel(const int2* __restrict__ hubs, const int32_t* __restrict__ state,
                             const int64_t* __restrict__ segbase, const int32_t* __restrict__ segoff,
                             const int32_t* __restrict__ memb, int n, uint8_t* __restrict__ X) {
    const int count = min(state[1], 255);
    const int h = blockIdx.x;
    if (h >= count) return;
    const int Hp = hub_pad(count), Kx = 2 * Hp;
    const int2 hl = hubs[h];
    const int t = hl.x, l = hl.y;
    const int32_t* so = segoff + segbase[t];
    const int32_t* mt = memb + (size_t)t * n;
    // OOB members: column h (ZA); in-bag members: column Hp + h (ZB)
    for (int q = so[2 * l] + threadIdx.x; q < so[2 * l + 1]; q += blockDim.x) X[xoff(mt[q], h, Kx)] = 1;
    for (int q = so[2 * l + 1] + threadIdx.x; q < so[2 * l + 2]; q += blockDim.x) X[xoff(mt[q], Hp + h, Kx)] = 1;
}

// ---------------------------------------------------------------------------
// tcgen05 helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// K-major, no swizzle: LBO = byte distance of K-adjacent core matrices, SBO =
// byte distance of adjacent 8-row groups (sm100 descriptor, version bit 46).
__device__ __forceinline__ uint64_t kdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// kind::i8 instruction descriptor: D s32, A and B unsigned 8-bit, K-major both
__host__ __device__ constexpr uint32_t idesc_u8_s32(int M, int N) {
    return (2u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void commit_to(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
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

constexpr int HG_WAIT_LIMIT = 1 << 24;

// bounded wait for completion number `k` (parity k & 1) of the mbarrier
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    for (int it = 0; it < HG_WAIT_LIMIT; ++it) {
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

__device__ __forceinline__ void bulk_s2g(void* dst, uint32_t src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(src), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

__device__ __forceinline__ void epi_bar() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t* r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}


__global__ void __launch_bounds__(HG_THREADS, 1)
hub_gemm_kernel(const uint8_t* __restrict__ X, const int32_t* __restrict__ state, int n, uint8_t* __restrict__ out,
                uint32_t* __restrict__ err) {
    extern __shared__ uint8_t smraw[];
    __shared__ __align__(8) uint64_t bar_afull, bar_aempty, bar_bfull[HG_STAGES], bar_bempty[HG_STAGES],
        bar_accfull[2], bar_accempty[2], bar_done;
    __shared__ uint32_t tmem_base;
    __shared__ int abort_flag, epi_stop;
    const int count = min(state[1], 255);
    if (count <= 0) return;  // no hub leaves: nothing to compute (the row kernel then starts from zero)
    const int Hp = hub_pad(count), Kx = 2 * Hp, Kc = Kx / 128;
    const int NI = (n + 127) >> 7, NJ = (n + 255) >> 8;
    const long long ntiles = hub_row_start(NI, NJ);
    const long long per = (ntiles + gridDim.x - 1) / gridDim.x;
    const long long tile0 = (long long)blockIdx.x * per;
    const long long tile1 = min(ntiles, tile0 + per);
    if (tile0 >= tile1) return;
    // 1024-aligned dynamic shared memory: A | B stages | two output buffers
    uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smraw) + 1023) & ~(uintptr_t)1023);
    uint8_t* As = sm;
    uint8_t* Bs = sm + HG_A_MAX;
    uint8_t* Os = Bs + HG_STAGES * HG_CHUNK;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(su32(&tmem_base)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        mbar_init(su32(&bar_afull), 1);
        mbar_init(su32(&bar_aempty), 1);
        for (int s = 0; s < HG_STAGES; ++s) {
            mbar_init(su32(&bar_bfull[s]), 1);
            mbar_init(su32(&bar_bempty[s]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(su32(&bar_accfull[b]), 1);
            mbar_init(su32(&bar_accempty[b]), 128);
        }
        mbar_init(su32(&bar_done), 1);
        abort_flag = 0;
        epi_stop = 0;
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;
    // row block of the first tile
    int I0 = 0;
    {
        int lo = 0, hi = NI;  // largest I with row_start(I) <= tile0
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (hub_row_start(mid, NJ) <= tile0) lo = mid;
            else hi = mid;
        }
        I0 = lo;
    }
    const int J0 = (I0 >> 1) + (int)(tile0 - hub_row_start(I0, NJ));

    if (warp == 0) {
        // ---------------- loads ----------------
        if (lane == 0) {
            int I = I0, J = J0, curI = -1;
            uint32_t afills = 0, bfills = 0;
            bool ok = true;
            for (long long tt = tile0; tt < tile1 && ok; ++tt) {
                if (I != curI) {
                    if (afills > 0) ok = mbar_wait(su32(&bar_aempty), (afills - 1) & 1);
                    if (!ok) break;
                    mbar_expect_tx(su32(&bar_afull), 128u * (uint32_t)Kx);
                    const uint8_t* xb = X + (size_t)(I >> 1) * (256u * (size_t)Kx) + (I & 1) * 2048;
                    for (int s = 0; s < Kx / 16; ++s)
                        bulk_g2s(su32(As + s * 2048), xb + (size_t)(s >> 3) * HG_CHUNK + (s & 7) * 4096, 2048,
                                 su32(&bar_afull));
                    ++afills;
                    curI = I;
                }
                const uint8_t* yb = X + (size_t)J * (256u * (size_t)Kx);
                for (int kc = 0; kc < Kc; ++kc) {
                    const int s = (int)(bfills % HG_STAGES);
                    const uint32_t use = bfills / HG_STAGES;
                    if (use > 0 && !(ok = mbar_wait(su32(&bar_bempty[s]), (use - 1) & 1))) break;
                    if (*(volatile int*)&abort_flag) {
                        ok = false;
                        break;
                    }
                    mbar_expect_tx(su32(&bar_bfull[s]), HG_CHUNK);
                    bulk_g2s(su32(Bs + s * HG_CHUNK), yb + (size_t)((kc + Kc / 2) % Kc) * HG_CHUNK, HG_CHUNK,
                             su32(&bar_bfull[s]));
                    ++bfills;
                }
                if (++J == NJ) {
                    ++I;
                    J = I >> 1;
                }
            }
            if (!ok) {
                atomicOr(err, ERR_WAIT_LIMIT);
                abort_flag = 1;
            }
            // every fill issued has landed before the CTA may exit (bounded)
            if (afills > 0) mbar_wait(su32(&bar_afull), (afills - 1) & 1);
            for (uint32_t f = bfills > HG_STAGES ? bfills - HG_STAGES : 0; f < bfills; ++f)
                mbar_wait(su32(&bar_bfull[f % HG_STAGES]), (f / HG_STAGES) & 1);
        }
    } else if (warp == 1) {
        // ---------------- MMA issue ----------------
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_u8_s32(128, 256);
            int I = I0, J = J0, curI = -1;
            uint32_t afills = 0, bfills = 0, nt = 0;
            bool ok = true;
            for (long long tt = tile0; tt < tile1 && ok; ++tt, ++nt) {
                if (I != curI) {
                    ok = mbar_wait(su32(&bar_afull), afills & 1);
                    ++afills;
                    curI = I;
                    if (!ok) break;
                }
                const int b = (int)(nt & 1);
                const uint32_t use = nt >> 1;
                if (use > 0 && !(ok = mbar_wait(su32(&bar_accempty[b]), (use - 1) & 1))) break;
                asm volatile("tcgen05.fence::after_thread_sync;");
                const uint32_t dacc = tmem + (uint32_t)(b * 256);
                for (int kc = 0; kc < Kc; ++kc) {
                    const int s = (int)(bfills % HG_STAGES);
                    if (!(ok = mbar_wait(su32(&bar_bfull[s]), (bfills / HG_STAGES) & 1))) break;
                    asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
                    for (int ks = 0; ks < 4; ++ks) {
                        const uint64_t ad = kdesc(su32(As) + (uint32_t)(kc * 8 + ks * 2) * 2048u, 2048u, 128u);
                        const uint64_t bd = kdesc(su32(Bs + s * HG_CHUNK) + (uint32_t)ks * 8192u, 4096u, 128u);
                        mma_i8(dacc, ad, bd, idesc, (kc > 0 || ks > 0) ? 1u : 0u);
                    }
                    commit_to(su32(&bar_bempty[s]));  // the stage is free once these MMAs finish
                    ++bfills;
                }
                if (!ok) break;
                commit_to(su32(&bar_accfull[b]));
                int nI = I, nJ = J + 1;
                if (nJ == NJ) {
                    ++nI;
                    nJ = nI >> 1;
                }
                if (nI != I || tt + 1 == tile1) commit_to(su32(&bar_aempty));  // A of this row block is free
                I = nI;
                J = nJ;
            }
            if (!ok) {
                atomicOr(err, ERR_WAIT_LIMIT);
                abort_flag = 1;
                // let the epilogue of a tile that will never be computed go
                commit_to(su32(&bar_accfull[nt & 1]));
            }
            // every MMA this thread issued has finished before TMEM is freed
            commit_to(su32(&bar_done));
            mbar_wait(su32(&bar_done), 0);
        }
        __syncwarp();
    } else {
        // ---------------- epilogue: TMEM -> u8 tile -> bulk store ----------------
        // The leader thread waits for the accumulator and decides for all 128
        // threads whether to go on (a shared flag read after the named
        // barrier), so that every thread takes the same number of barriers.
        const int q4 = warp & 3;          // TMEM lane quarter this warp may access
        const int r = q4 * 32 + lane;     // tile row
        const bool leader = (warp == 2 && lane == 0);
        uint32_t nt = 0;
        for (long long tt = tile0; tt < tile1; ++tt, ++nt) {
            const int b = (int)(nt & 1);
            uint8_t* ob = Os + b * HG_OUT;
            if (leader) {
                // the bulk store that last read this output buffer (two tiles ago) is done
                asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
                const bool okw = mbar_wait(su32(&bar_accfull[b]), (nt >> 1) & 1);
                if (!okw) atomicOr(err, ERR_WAIT_LIMIT);
                epi_stop = (!okw || *(volatile int*)&abort_flag) ? 1 : 0;
                if (!okw) abort_flag = 1;
            }
            epi_bar();
            if (*(volatile int*)&epi_stop) break;
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t tbase = tmem + ((uint32_t)(q4 * 32) << 16) + (uint32_t)(b * 256);
#pragma unroll 1
            for (int c = 0; c < 256; c += 32) {
                uint32_t v[32];
                tmem_ld16(tbase + c, v);
                tmem_ld16(tbase + c + 16, v + 16);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const uint32_t* w = v + 16 * h;
                    uint4 pk;
                    pk.x = (w[0] & 255u) | ((w[1] & 255u) << 8) | ((w[2] & 255u) << 16) | ((w[3] & 255u) << 24);
                    pk.y = (w[4] & 255u) | ((w[5] & 255u) << 8) | ((w[6] & 255u) << 16) | ((w[7] & 255u) << 24);
                    pk.z = (w[8] & 255u) | ((w[9] & 255u) << 8) | ((w[10] & 255u) << 16) | ((w[11] & 255u) << 24);
                    pk.w = (w[12] & 255u) | ((w[13] & 255u) << 8) | ((w[14] & 255u) << 16) | ((w[15] & 255u) << 24);
                    const int q = (c >> 4) + h;  // logical 16-column chunk
                    *reinterpret_cast<uint4*>(ob + r * 256 + ((q ^ (r & 15)) << 4)) = pk;
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;");
            mbar_arrive(su32(&bar_accempty[b]));  // TMEM buffer b may be overwritten
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            epi_bar();
            if (leader) bulk_s2g(out + (size_t)tt * HG_OUT, su32(ob), HG_OUT);
        }
        if (leader) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem));
    }
}

}  // namespace

int hub_tiles_nj(int n) { return (n + 255) >> 8; }

size_t hub_tile_bytes(int n) {
    const int NI = (n + 127) >> 7, NJ = hub_tiles_nj(n);
    return (size_t)hub_row_start(NI, NJ) * HG_OUT;
}

// Hub selection, X, and the S_hub tiles for the context's current leaf lists.
// hub_state[1] receives the hub count (0: no tiles were written) and
// *hub_pairs (zeroed by the caller) the hub leaves' pair updates.
rfx_status launch_hub_tiles(Ctx* c, uint8_t* keyflag, uint8_t* tiles, int32_t* hub_state,
                            unsigned long long* hub_pairs) {
    Scratch sc(c);
    const int n = c->n;
    uint32_t* hist = sc.get<uint32_t>(HUB_BINS);
    int2* hubs = sc.get<int2>(HUB_MAX);
    const size_t xbytes = (size_t)((n + 255) >> 8) * 256u * 512u;
    uint8_t* X = sc.get<uint8_t>(xbytes);
    if (!hist || !hubs || !X) {
        set_error("hub tiles: scratch allocation failed");
        return RFX_ERR_OOM;
    }
    // a hub leaf adds n*n/2 * 2 MACs (two K columns over the upper triangle);
    // at ~2e15 MAC/s against ~1e12 counter increments/s that pays from about
    // a*b >= n*n / 2000
    unsigned long long min_prod = std::max<unsigned long long>(1ull, (unsigned long long)n * n / 2000ull);
    // RFX_PAIRS_HUB_MIN=<product> sets the smallest a*b of a hub leaf (the
    // tests use it to fill both operand widths at small n)
    if (const char* e = std::getenv("RFX_PAIRS_HUB_MIN")) {
        const long long v = std::atoll(e);
        if (v >= 1) min_prod = (unsigned long long)v;
    }
    RFX_CUDA(cudaMemsetAsync(hist, 0, sizeof(uint32_t) * HUB_BINS, c->stream));
    RFX_CUDA(cudaMemsetAsync(keyflag, 0, (size_t)c->h_segbase[c->T], c->stream));
    RFX_CUDA(cudaMemsetAsync(X, 0, xbytes, c->stream));
    hub_hist_kernel<<<c->T, 256, 0, c->stream>>>(c->d_segbase, c->d_segoff, min_prod, hist);
    hub_pick_kernel<<<1, 32, 0, c->stream>>>(hist, HUB_MAX, hub_state);
    hub_mark_kernel<<<c->T, 256, 0, c->stream>>>(c->d_segbase, c->d_segoff, min_prod, HUB_MAX, hub_state, hubs,
                                                 keyflag, hub_pairs);
    hub_z_kernel<<<HUB_MAX, 256, 0, c->stream>>>(hubs, hub_state, c->d_segbase, c->d_segoff, c->d_memb, n, X);
    RFX_CUDA(cudaGetLastError());
    int nsm = 0;
    RFX_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
    RFX_CUDA(cudaFuncSetAttribute(hub_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)HG_SMEM));
    hub_gemm_kernel<<<nsm, HG_THREADS, HG_SMEM, c->stream>>>(X, hub_state, n, tiles, c->d_err);
    RFX_CUDA(cudaGetLastError());
    return RFX_OK;
}

}  // namespace rfx
