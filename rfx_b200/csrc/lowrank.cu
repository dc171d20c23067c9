// Low-rank proximity: a randomised range finder over the leaf indicators.
//
// The normalised proximity of cpu_finishprox (src/rf_finishprox.cpp:12-74) is
//   P = I + M,  M = 1/4 (D S + S D),  D = diag(1/nout_i) (1 where nout_i = 0),
// with S = C + C^T the pair counts of cpu_proximity's dense branch.  S is never
// formed: S X = sum_t (Z_oob,t Z_in,t^T + Z_in,t Z_oob,t^T) X is applied tree by
// tree through the leaf member lists (per leaf key, the sum of the members'
// rows of X, then every sample adds the sum of the opposite bag status of its
// own leaf).  The factors replace the reference's rank-1-per-tree QLORA
// accumulation (cuda/rf_proximity_lowrank.cu:863-1071) and satisfy
// P ~= I + A A^T with A = Q U_k Lambda_k^(1/2) from the top-k eigenpairs of
// M restricted to the range Q of the sketch M^(q+1) Omega.
//
// Forms:
//   FP32  - X, leaf sums and products in FP32;
//   mixed - X and leaf sums stored in BF16, FP32 accumulation (precision 1);
//           precision 2 also recomputes the last product M Q, which builds the
//           Rayleigh-Ritz projection, in FP32; precision 3 stores X and the
//           leaf sums as FP8 e4m3 rows, each with its own FP32 scale (the
//           row's largest magnitude maps to 448), FP32 accumulation.
// FP64 is used for the k' x k' Gram (CholeskyQR2) and the eigensolve only.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <type_traits>
#include <cstdlib>
#include <vector>

#include "dense.cuh"
#include "rfx_internal.cuh"

namespace rfx {
namespace {

__device__ __forceinline__ void st_val(float* p, float v) { *p = v; }
__device__ __forceinline__ void st_val(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }

// Gaussian from a counter hash (splitmix64) and Box-Muller.
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

template <typename T>
__global__ void gauss_kernel(T* __restrict__ out, int64_t count, uint64_t seed) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= count) return;
    const uint64_t h = mix64(seed ^ mix64((uint64_t)idx));
    const double u1 = ((h >> 11) + 1.0) * (1.0 / 9007199254740993.0);
    const double u2 = (double)(mix64(h) >> 11) * (1.0 / 9007199254740992.0);
    const double g = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
    st_val(out + idx, (float)g);
}

// X = [V | D V] in the storage type (n x 2w), from V (n x w, FP32).
template <typename TX>
__global__ void pack_x_kernel(const float* __restrict__ V, const float* __restrict__ dinv, int n, int w,
                              TX* __restrict__ X) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)n * w) return;
    const int i = (int)(idx / w), c = (int)(idx % w);
    const float v = V[idx];
    st_val(X + (size_t)i * 2 * w + c, v);
    st_val(X + (size_t)i * 2 * w + w + c, __fmul_rn(v, dinv[i]));
}

// Row chunks owned by one lane: E values of type T (16 bytes, or 8 bytes for
// BF16 rows too narrow to give every lane a 16-byte chunk).
template <typename T, int E>
struct Chunk;
template <>
struct Chunk<float, 4> {
    __device__ static void load(const float* p, float* v) {
        const float4 x = __ldg(reinterpret_cast<const float4*>(p));
        v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
    }
    __device__ static void store(float* p, const float* v) {
        *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    }
};
template <>
struct Chunk<__nv_bfloat16, 8> {
    __device__ static void load(const __nv_bfloat16* p, float* v) {
        const uint4 x = __ldg(reinterpret_cast<const uint4*>(p));
        const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&x);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float2 f = __bfloat1622float2(h[q]);
            v[2 * q] = f.x;
            v[2 * q + 1] = f.y;
        }
    }
    __device__ static void store(__nv_bfloat16* p, const float* v) {
        uint4 x;
        __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&x);
#pragma unroll
        for (int q = 0; q < 4; ++q) h[q] = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
        *reinterpret_cast<uint4*>(p) = x;
    }
};
template <>
struct Chunk<__nv_bfloat16, 4> {
    __device__ static void load(const __nv_bfloat16* p, float* v) {
        const uint2 x = __ldg(reinterpret_cast<const uint2*>(p));
        const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&x);
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const float2 f = __bfloat1622float2(h[q]);
            v[2 * q] = f.x;
            v[2 * q + 1] = f.y;
        }
    }
    __device__ static void store(__nv_bfloat16* p, const float* v) {
        uint2 x;
        __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&x);
#pragma unroll
        for (int q = 0; q < 2; ++q) h[q] = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
        *reinterpret_cast<uint2*>(p) = x;
    }
};

// FP8 e4m3 rows (precision 3): 8 codes per lane chunk; the row's FP32 scale
// lives beside it (values = code x scale).
template <>
struct Chunk<uint8_t, 8> {
    __device__ static void load(const uint8_t* p, float* v) {
        const uint2 x = __ldg(reinterpret_cast<const uint2*>(p));
        const uint32_t w[2] = {x.x, x.y};
#pragma unroll
        for (int h = 0; h < 2; ++h) {
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const __half2_raw hr = __nv_cvt_fp8x2_to_halfraw2(
                    (__nv_fp8x2_storage_t)((w[h] >> (16 * q)) & 0xffffu), __NV_E4M3);
                const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&hr));
                v[4 * h + 2 * q] = f.x;
                v[4 * h + 2 * q + 1] = f.y;
            }
        }
    }
    __device__ static void store(uint8_t* p, const float* v) {
        uint32_t w[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const uint32_t lo = __nv_cvt_float2_to_fp8x2(make_float2(v[4 * h], v[4 * h + 1]), __NV_SATFINITE, __NV_E4M3);
            const uint32_t hi =
                __nv_cvt_float2_to_fp8x2(make_float2(v[4 * h + 2], v[4 * h + 3]), __NV_SATFINITE, __NV_E4M3);
            w[h] = lo | (hi << 16);
        }
        *reinterpret_cast<uint2*>(p) = make_uint2(w[0], w[1]);
    }
};

template <typename T>
constexpr bool is_fp8() { return std::is_same<T, uint8_t>::value; }

// X = [V | D V] as FP8 rows with one scale per row (448 = the largest e4m3
// value maps to the row's largest magnitude); one warp per row.
__global__ void pack_x_fp8_kernel(const float* __restrict__ V, const float* __restrict__ dinv, int n, int w,
                                  uint8_t* __restrict__ X, float* __restrict__ xs) {
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= n) return;
    const int i = (int)warp;
    const float di = dinv[i];
    float amax = 0.0f;
    for (int c = lane; c < w; c += 32) amax = fmaxf(amax, fmaxf(fabsf(V[(size_t)i * w + c]), fabsf(V[(size_t)i * w + c] * di)));
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, d));
    const float sc = amax > 0.0f ? 448.0f / amax : 1.0f;
    for (int c = lane; c < w; c += 32) {
        const float v = V[(size_t)i * w + c];
        X[(size_t)i * 2 * w + c] = (uint8_t)(__nv_cvt_float2_to_fp8x2(make_float2(v * sc, 0.0f), __NV_SATFINITE,
                                                                      __NV_E4M3) & 0xffu);
        X[(size_t)i * 2 * w + w + c] = (uint8_t)(__nv_cvt_float2_to_fp8x2(
                                                     make_float2(__fmul_rn(v, di) * sc, 0.0f), __NV_SATFINITE,
                                                     __NV_E4M3) & 0xffu);
    }
    if (lane == 0) xs[i] = 1.0f / sc;
}

// Leaf-key sums of X rows for trees [t0, t1): G[gofs[t-t0] + key][:] = sum
// over members j of key of X[j][:].  The member list of each tree (keys in
// order, members of a key contiguous) is cut into chunks of SEG_CH positions,
// one warp per chunk, so a leaf with thousands of members is spread over many
// warps.  A key that lies inside one chunk is written to G directly; a key that
// crosses a chunk boundary leaves FP32 partial sums (Pf: the chunk's first key,
// Pl: its last key) that segsum_fix_kernel adds up in chunk order.  Rows move
// as 16-byte chunks (lane l owns chunks l and l + 32).  G rows of empty keys
// must be zero beforehand.
constexpr int SEG_CH = 64;

// adds the row (times its scale sc, for FP8 rows) to the lane's sums
template <typename T, int E>
__device__ __forceinline__ void add_row(const T* xr, float sc, int lane, bool c0ok, bool c1ok, float* a0, float* a1) {
    float v[E];
    if (c0ok) {
        Chunk<T, E>::load(xr + lane * E, v);
#pragma unroll
        for (int e = 0; e < E; ++e) a0[e] = is_fp8<T>() ? fmaf(v[e], sc, a0[e]) : a0[e] + v[e];
    }
    if (c1ok) {
        Chunk<T, E>::load(xr + (lane + 32) * E, v);
#pragma unroll
        for (int e = 0; e < E; ++e) a1[e] = is_fp8<T>() ? fmaf(v[e], sc, a1[e]) : a1[e] + v[e];
    }
}

template <typename TO, int E>
__device__ __forceinline__ void store_row(TO* out, int lane, bool c0ok, bool c1ok, const float* a0, const float* a1) {
    if (c0ok) Chunk<TO, E>::store(out + lane * E, a0);
    if (c1ok) Chunk<TO, E>::store(out + (lane + 32) * E, a1);
}

// A finished G row: FP8 rows get their own scale (the warp's largest
// magnitude maps to 448), written beside the row; other types store as is.
// Called by the whole warp.
template <typename TO, int E>
__device__ __forceinline__ void store_grow(TO* out, float* scale_out, int lane, bool c0ok, bool c1ok, const float* a0,
                                           const float* a1) {
    if constexpr (is_fp8<TO>()) {
        float amax = 0.0f;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            if (c0ok) amax = fmaxf(amax, fabsf(a0[e]));
            if (c1ok) amax = fmaxf(amax, fabsf(a1[e]));
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, d));
        const float sc = amax > 0.0f ? 448.0f / amax : 1.0f;
        float b0[E], b1[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            b0[e] = a0[e] * sc;
            b1[e] = a1[e] * sc;
        }
        store_row<TO, E>(out, lane, c0ok, c1ok, b0, b1);
        if (lane == 0) *scale_out = 1.0f / sc;
    } else {
        (void)scale_out;
        store_row<TO, E>(out, lane, c0ok, c1ok, a0, a1);
    }
}

// FP32 partial rows use 4-float chunks; a lane chunk of E values is stored as
// E / 4 float chunks.
template <typename T, int E>
__device__ __forceinline__ void store_partial(float* out, int lane, bool c0ok, bool c1ok, const float* a0,
                                              const float* a1) {
#pragma unroll
    for (int h = 0; h < E / 4; ++h) {
        if (c0ok) Chunk<float, 4>::store(out + lane * E + 4 * h, a0 + 4 * h);
        if (c1ok) Chunk<float, 4>::store(out + (lane + 32) * E + 4 * h, a1 + 4 * h);
    }
}

template <typename T, int E>
__device__ __forceinline__ void add_partial(const float* in, int lane, bool c0ok, bool c1ok, float* a0, float* a1) {
    float v[4];
#pragma unroll
    for (int h = 0; h < E / 4; ++h) {
        if (c0ok) {
            Chunk<float, 4>::load(in + lane * E + 4 * h, v);
#pragma unroll
            for (int e = 0; e < 4; ++e) a0[4 * h + e] += v[e];
        }
        if (c1ok) {
            Chunk<float, 4>::load(in + (lane + 32) * E + 4 * h, v);
#pragma unroll
            for (int e = 0; e < 4; ++e) a1[4 * h + e] += v[e];
        }
    }
}

template <typename T, int E>
__global__ void segsum_kernel(const T* __restrict__ X, int n, int W, const int32_t* __restrict__ memb,
                              const int32_t* __restrict__ segoff, const int64_t* __restrict__ segbase, int t0,
                              int t1, int cpt, const int64_t* __restrict__ gofs, T* __restrict__ G,
                              float* __restrict__ Pf, float* __restrict__ Pl, int32_t* __restrict__ fk,
                              const float* __restrict__ xs, float* __restrict__ gs) {
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= (int64_t)(t1 - t0) * cpt) return;
    const int tb = (int)(warp / cpt), ch = (int)(warp % cpt);
    const int t = t0 + tb;
    const int32_t* so = segoff + segbase[t];
    const int K = (int)(segbase[t + 1] - segbase[t]) - 1;
    const int ntot = __ldg(so + K);
    const int cs = ch * SEG_CH;
    if (cs >= ntot) {
        if (lane == 0) fk[warp] = -1;
        return;
    }
    const int ce = min(cs + SEG_CH, ntot);
    // key holding position cs: the largest k with so[k] <= cs (so[0] = 0)
    int lo = 0, hi = K;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(so + mid) <= cs) lo = mid;
        else hi = mid;
    }
    int key = lo;
    if (lane == 0) fk[warp] = key;
    const int32_t* mt = memb + (size_t)t * n;
    const int m0 = cs + lane < ce ? __ldg(mt + cs + lane) : 0;
    const int m1 = cs + 32 + lane < ce ? __ldg(mt + cs + 32 + lane) : 0;
    const int CH = W / E;
    const bool c0ok = lane < CH, c1ok = lane + 32 < CH;
    int pos = cs;
    while (pos < ce) {
        const int kbeg = __ldg(so + key), kend = __ldg(so + key + 1);
        const int e = min(kend, ce);
        float a0[E], a1[E];
#pragma unroll
        for (int q = 0; q < E; ++q) a0[q] = a1[q] = 0.0f;
#pragma unroll 4
        for (int q = pos; q < e; ++q) {
            const int r = q - cs;  // warp-uniform
            const int j = __shfl_sync(0xffffffffu, r < 32 ? m0 : m1, r & 31);
            add_row<T, E>(X + (size_t)j * W, is_fp8<T>() ? __ldg(xs + j) : 1.0f, lane, c0ok, c1ok, a0, a1);
        }
        if (kbeg >= cs && kend <= ce) {
            store_grow<T, E>(G + (size_t)(gofs[tb] + key) * W, gs + gofs[tb] + key, lane, c0ok, c1ok, a0, a1);
        } else if (pos == cs) {
            store_partial<T, E>(Pf + (size_t)warp * W, lane, c0ok, c1ok, a0, a1);
        } else {
            store_partial<T, E>(Pl + (size_t)warp * W, lane, c0ok, c1ok, a0, a1);
        }
        pos = e;
        if (pos < ce) {
            ++key;
            while (__ldg(so + key + 1) <= pos) ++key;  // skip empty keys; pos < ntot = so[K] bounds key < K
        }
    }
}

// The same sums with the warp split into slots: a row is
// held by LPR = ceil(CPR / CPL) lanes of CPL chunks each, and the warp's
// 32 / LPR slots take that many of the chunk's keys at once, each slot adding
// its key's member rows in order.  Keys are short (a few members), so the
// slots replace the per-key turns of the whole warp.
template <typename T, int E, int CPL>
__global__ void segsum_slot_kernel(const T* __restrict__ X, int n, int W, const int32_t* __restrict__ memb,
                                   const int32_t* __restrict__ segoff, const int64_t* __restrict__ segbase, int t0,
                                   int t1, int cpt, const int64_t* __restrict__ gofs, T* __restrict__ G,
                                   float* __restrict__ Pf, float* __restrict__ Pl, int32_t* __restrict__ fk,
                                   const float* __restrict__ xs, float* __restrict__ gs) {
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= (int64_t)(t1 - t0) * cpt) return;
    const int tb = (int)(warp / cpt), ch = (int)(warp % cpt);
    const int t = t0 + tb;
    const int32_t* so = segoff + segbase[t];
    const int K = (int)(segbase[t + 1] - segbase[t]) - 1;
    const int ntot = __ldg(so + K);
    const int cs = ch * SEG_CH;
    if (cs >= ntot) {
        if (lane == 0) fk[warp] = -1;
        return;
    }
    const int ce = min(cs + SEG_CH, ntot);
    // first key: the largest k with so[k] <= cs; last key: the largest k with
    // so[k] <= ce - 1 (so[0] = 0, so[K] = ntot > ce - 1)
    int lo = 0, hi = K;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(so + mid) <= cs) lo = mid;
        else hi = mid;
    }
    const int key0 = lo;
    hi = K;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(so + mid) <= ce - 1) lo = mid;
        else hi = mid;
    }
    const int nkeys = lo - key0 + 1;
    if (lane == 0) fk[warp] = key0;
    const int32_t* mt = memb + (size_t)t * n;
    const int m0 = cs + lane < ce ? __ldg(mt + cs + lane) : 0;
    const int m1 = cs + 32 + lane < ce ? __ldg(mt + cs + 32 + lane) : 0;
    const int CPR = W / E;
    const int LPR = (CPR + CPL - 1) / CPL;
    const int SL = 32 / LPR;
    const int slot = lane / LPR, lr = lane % LPR;
    const bool live = slot < SL;
    for (int kb = 0; kb < nkeys; kb += SL) {
        const int k = key0 + kb + slot;
        const bool act = live && kb + slot < nkeys;
        const int kbeg = act ? __ldg(so + k) : 0, kend = act ? __ldg(so + k + 1) : 0;
        const int p0 = max(kbeg, cs), p1 = min(kend, ce);
        const int cntm = act ? max(0, p1 - p0) : 0;
        const int maxc = __reduce_max_sync(0xffffffffu, cntm);
        float acc[CPL][E];
#pragma unroll
        for (int c = 0; c < CPL; ++c)
#pragma unroll
            for (int e = 0; e < E; ++e) acc[c][e] = 0.0f;
        for (int m = 0; m < maxc; ++m) {
            const int q = p0 - cs + m;  // this slot's member position in the chunk
            const int j0 = __shfl_sync(0xffffffffu, m0, q & 31);
            const int j1 = __shfl_sync(0xffffffffu, m1, q & 31);
            if (m >= cntm) continue;
            const int j = q < 32 ? j0 : j1;
            const T* xr = X + (size_t)j * W;
            const float sc = is_fp8<T>() ? __ldg(xs + j) : 1.0f;
#pragma unroll
            for (int c = 0; c < CPL; ++c) {
                const int ci = c * LPR + lr;
                if (ci < CPR) {
                    float v[E];
                    Chunk<T, E>::load(xr + ci * E, v);
#pragma unroll
                    for (int e = 0; e < E; ++e) acc[c][e] = is_fp8<T>() ? fmaf(v[e], sc, acc[c][e]) : acc[c][e] + v[e];
                }
            }
        }
        // a key cut by the chunk edges leaves a partial: the chunk's first
        // key in Pf, its last in Pl (segsum_fix_kernel reads them so)
        const bool whole = kbeg >= cs && kend <= ce;
        float scale = 1.0f;
        if constexpr (is_fp8<T>()) {
            // the row's largest magnitude over the slot's lanes maps to 448
            float amax = 0.0f;
#pragma unroll
            for (int c = 0; c < CPL; ++c)
#pragma unroll
                for (int e = 0; e < E; ++e) amax = fmaxf(amax, fabsf(acc[c][e]));
            for (int d = 1; d < LPR; ++d)
                amax = fmaxf(amax, __shfl_sync(0xffffffffu, amax, min(31, slot * LPR + (lr + d) % LPR)));
            scale = amax > 0.0f ? 448.0f / amax : 1.0f;
        }
        if (cntm == 0) continue;  // empty key: its zero row was cleared beforehand
        if (whole) {
            T* gr = G + (size_t)(gofs[tb] + k) * W;
#pragma unroll
            for (int c = 0; c < CPL; ++c) {
                const int ci = c * LPR + lr;
                if (ci < CPR) {
                    float v[E];
#pragma unroll
                    for (int e = 0; e < E; ++e) v[e] = acc[c][e] * scale;
                    Chunk<T, E>::store(gr + ci * E, v);
                }
            }
            if (is_fp8<T>() && lr == 0) gs[gofs[tb] + k] = 1.0f / scale;
        } else {
            float* pr = (p0 == cs ? Pf : Pl) + (size_t)warp * W;
#pragma unroll
            for (int c = 0; c < CPL; ++c) {
                const int ci = c * LPR + lr;
                if (ci < CPR)
#pragma unroll
                    for (int h = 0; h < E / 4; ++h) Chunk<float, 4>::store(pr + ci * E + 4 * h, &acc[c][4 * h]);
            }
        }
    }
}

// Keys that cross chunk boundaries: the chunk after the one a key starts in
// sums the key's partial rows in chunk order and writes its G row.
template <typename T, int E>
__global__ void segsum_fix_kernel(int n, int W, const int32_t* __restrict__ segoff, const int64_t* __restrict__ segbase,
                                  int t0, int t1, int cpt, const int64_t* __restrict__ gofs, T* __restrict__ G,
                                  const float* __restrict__ Pf, const float* __restrict__ Pl,
                                  const int32_t* __restrict__ fk, float* __restrict__ gs) {
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= (int64_t)(t1 - t0) * cpt) return;
    const int tb = (int)(warp / cpt), ch = (int)(warp % cpt);
    if (ch == 0) return;
    const int key = fk[warp];
    if (key < 0) return;
    const int32_t* so = segoff + segbase[t0 + tb];
    const int kbeg = __ldg(so + key), kend = __ldg(so + key + 1);
    const int cs = ch * SEG_CH;
    if (!(kbeg < cs && kbeg >= cs - SEG_CH)) return;  // owned by this chunk iff the key starts in the previous one
    const int CH = W / E;
    const bool c0ok = lane < CH, c1ok = lane + 32 < CH;
    float a0[E], a1[E];
#pragma unroll
    for (int q = 0; q < E; ++q) a0[q] = a1[q] = 0.0f;
    add_partial<T, E>((kbeg == cs - SEG_CH ? Pf : Pl) + (size_t)(warp - 1) * W, lane, c0ok, c1ok, a0, a1);
    for (int c2 = ch; c2 * SEG_CH < kend; ++c2)
        add_partial<T, E>(Pf + (size_t)(warp - ch + c2) * W, lane, c0ok, c1ok, a0, a1);
    store_grow<T, E>(G + (size_t)(gofs[tb] + key) * W, gs + gofs[tb] + key, lane, c0ok, c1ok, a0, a1);
}

// Y[i] (+)= sum over trees [t0, t1) of G_t[key_t(i) ^ 1]; one warp per sample,
// 16-byte chunks per lane, 32 trees' keys fetched at once.
template <typename T, int E>
__global__ void pull_kernel(const T* __restrict__ G, const int32_t* __restrict__ key, int n, int W, int t0, int t1,
                            const int64_t* __restrict__ gofs, float* __restrict__ Y, int accumulate,
                            const float* __restrict__ gs) {
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= n) return;
    const int i = (int)warp;
    const int CH = W / E;
    const bool c0ok = lane < CH, c1ok = lane + 32 < CH;
    float a0[E], a1[E];
#pragma unroll
    for (int e = 0; e < E; ++e) a0[e] = a1[e] = 0.0f;
    for (int tb = t0; tb < t1; tb += 32) {
        const int t = tb + lane;
        long long gi = -1;
        if (t < t1) {
            const int k = __ldg(key + (size_t)t * n + i);
            if (k >= 0) gi = gofs[t - t0] + (k ^ 1);
        }
        const int cnt = min(32, t1 - tb);
#pragma unroll 4
        for (int q = 0; q < cnt; ++q) {
            const long long r = __shfl_sync(0xffffffffu, gi, q);
            if (r < 0) continue;
            const T* gr = G + (size_t)r * W;
            float v[E];
            if constexpr (is_fp8<T>()) {
                const float sc = __ldg(gs + r);
                if (c0ok) {
                    Chunk<T, E>::load(gr + lane * E, v);
#pragma unroll
                    for (int e = 0; e < E; ++e) a0[e] = fmaf(v[e], sc, a0[e]);
                }
            } else {
                if (c0ok) {
                    Chunk<T, E>::load(gr + lane * E, v);
#pragma unroll
                    for (int e = 0; e < E; ++e) a0[e] += v[e];
                }
                if (c1ok) {
                    Chunk<T, E>::load(gr + (lane + 32) * E, v);
#pragma unroll
                    for (int e = 0; e < E; ++e) a1[e] += v[e];
                }
            }
        }
    }
    float* y = Y + (size_t)i * W;
    if (c0ok)
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int c = lane * E + e;
            y[c] = accumulate ? y[c] + a0[e] : a0[e];
        }
    if (c1ok)
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int c = (lane + 32) * E + e;
            y[c] = accumulate ? y[c] + a1[e] : a1[e];
        }
}

// MV = 1/4 (D Y[:, :w] + Y[:, w:])
__global__ void combine_kernel(const float* __restrict__ Y, const float* __restrict__ dinv, int n, int w,
                               float* __restrict__ out) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)n * w) return;
    const int i = (int)(idx / w), c = (int)(idx % w);
    const float a = Y[(size_t)i * 2 * w + c], b = Y[(size_t)i * 2 * w + w + c];
    out[idx] = 0.25f * (dinv[i] * a + b);
}

__global__ void dinv_kernel(const int32_t* __restrict__ nout, int n, float* __restrict__ dinv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dinv[i] = nout[i] > 0 ? (float)(1.0 / (double)nout[i]) : 1.0f;
}

// G[w x w] (FP64) += X^T Y over rows; X, Y n x w FP32.  Block: 256 threads,
// 64-row chunks, each thread accumulates (w*w)/256 entries.
constexpr int GW = 128;  // maximum width

// Per-CTA partial Gram matrices part[cta] = X^T Y over the CTA's rows (FP32
// inputs, FP64 products and sums), w x w with w a multiple of 4: thread
// (ta, tb) owns the 4 x 4 block of rows 4ta.. and columns 4tb.. of the
// result; rows arrive in shared-memory tiles of 32.  gram_sum_w_kernel adds
// the partials in CTA order (reproducible).
constexpr int GRAM_CTAS = 296;
__global__ void __launch_bounds__(1024) gram_f32_kernel(const float* __restrict__ X, const float* __restrict__ Y,
                                                        int n, int w, double* __restrict__ part) {
    __shared__ float Xs[32][GW], Ys[32][GW];
    const int tid = threadIdx.x, nth = blockDim.x;
    const int qw = w / 4;
    const int ta = tid / qw, tb = tid % qw;
    const bool own = tid < qw * qw;
    double acc[4][4];
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[p][q] = 0.0;
    for (int r0 = blockIdx.x * 32; r0 < n; r0 += gridDim.x * 32) {
        for (int e = tid; e < 32 * w; e += nth) {
            const int r = e / w, c = e % w;
            Xs[r][c] = (r0 + r < n) ? X[(size_t)(r0 + r) * w + c] : 0.0f;
            Ys[r][c] = (r0 + r < n) ? Y[(size_t)(r0 + r) * w + c] : 0.0f;
        }
        __syncthreads();
        if (own) {
#pragma unroll 4
            for (int r = 0; r < 32; ++r) {
                const float4 xa = *reinterpret_cast<const float4*>(&Xs[r][4 * ta]);
                const float4 yb = *reinterpret_cast<const float4*>(&Ys[r][4 * tb]);
                const double x[4] = {xa.x, xa.y, xa.z, xa.w}, y[4] = {yb.x, yb.y, yb.z, yb.w};
#pragma unroll
                for (int p = 0; p < 4; ++p)
#pragma unroll
                    for (int q = 0; q < 4; ++q) acc[p][q] = fma(x[p], y[q], acc[p][q]);
            }
        }
        __syncthreads();
    }
    if (own) {
        double* pp = part + (size_t)blockIdx.x * w * w;
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
            for (int q = 0; q < 4; ++q) pp[(size_t)(4 * ta + p) * w + 4 * tb + q] = acc[p][q];
    }
}

// G[e] = sum over the partials, one warp per entry (lane l the partials l,
// l + 32, ..., then a fixed shuffle tree)
__global__ void gram_sum_w_kernel(const double* __restrict__ part, int nparts, int cnt, double* __restrict__ G) {
    const int e = (int)(((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (e >= cnt) return;
    double v = 0.0;
    for (int q = lane; q < nparts; q += 32) v += part[(size_t)q * cnt + e];
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    if (lane == 0) G[e] = v;
}

// One CTA: T = L^{-T} for G = L L^T (w x w), in shared memory (dynamic).
__global__ void chol_inv_w_kernel(const double* __restrict__ G, int w, double* __restrict__ Tm, int* __restrict__ bad) {
    extern __shared__ double sm[];
    double* L = sm;
    double* Li = sm + w * w;
    __shared__ double flag;
    for (int e = threadIdx.x; e < w * w; e += blockDim.x) L[e] = G[e];
    __syncthreads();
    if (!cta_cholesky(L, w, w, &flag) && threadIdx.x == 0) *bad = 1;
    cta_tri_inverse(L, Li, w, w);
    for (int e = threadIdx.x; e < w * w; e += blockDim.x) {
        const int i = e / w, j = e % w;
        Tm[i * w + j] = Li[j * w + i];
    }
}

// out[n x m] = X[n x w] T[w x m] (FP32 X, FP64 T and sums), m a multiple of
// 4: a CTA takes 64 rows (staged in shared memory with T); thread (ra, cb)
// owns the 4 x 4 block of rows 4ra.. and columns 4cb.. .
constexpr int RM_ROWS = 64;
__global__ void __launch_bounds__(1024) right_mul_kernel(const float* __restrict__ X, const double* __restrict__ Tm,
                                                         int n, int w, int m, float* __restrict__ out) {
    const int mp = (m + 3) & ~3;                                            // columns padded to 4
    extern __shared__ double Ts[];                                          // w x mp
    float* Xs = reinterpret_cast<float*>(Ts + (size_t)w * mp);             // RM_ROWS x (w + 1)
    const int tid = threadIdx.x, nth = blockDim.x;
    const int r0 = blockIdx.x * RM_ROWS;
    for (int e = tid; e < w * mp; e += nth) {
        const int kk = e / mp, c = e % mp;
        Ts[e] = c < m ? Tm[(size_t)kk * m + c] : 0.0;
    }
    for (int e = tid; e < RM_ROWS * w; e += nth) {
        const int r = e / w, c = e % w;
        Xs[r * (w + 1) + c] = r0 + r < n ? X[(size_t)(r0 + r) * w + c] : 0.0f;
    }
    __syncthreads();
    const int qm = mp / 4;
    const int ra = tid / qm, cb = tid % qm;
    if (ra >= RM_ROWS / 4) return;
    double acc[4][4];
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[p][q] = 0.0;
#pragma unroll 4
    for (int kk = 0; kk < w; ++kk) {
        double x[4], t[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) x[p] = Xs[(4 * ra + p) * (w + 1) + kk];
#pragma unroll
        for (int q = 0; q < 4; ++q) t[q] = Ts[(size_t)kk * mp + 4 * cb + q];
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[p][q] = fma(x[p], t[q], acc[p][q]);
    }
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        const int r = r0 + 4 * ra + p;
        if (r >= n) continue;
        if (mp == m) {
            *reinterpret_cast<float4*>(out + (size_t)r * m + 4 * cb) =
                make_float4((float)acc[p][0], (float)acc[p][1], (float)acc[p][2], (float)acc[p][3]);
        } else {
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (4 * cb + q < m) out[(size_t)r * m + 4 * cb + q] = (float)acc[p][q];
        }
    }
}

inline size_t right_mul_smem(int w, int m) {
    return sizeof(double) * (size_t)w * ((m + 3) & ~3) + sizeof(float) * RM_ROWS * (size_t)(w + 1);
}
inline int right_mul_threads(int m) { return std::max(32, (RM_ROWS / 4) * (((m + 3) & ~3) / 4)); }

// One CTA: eigen-decomposition of the symmetrised w x w H.
__global__ void __launch_bounds__(1024, 1) eig_w_kernel(const double* __restrict__ H, int w, double* __restrict__ evals,
                             double* __restrict__ evecs) {
    extern __shared__ double sm[];  // two w x (w + 1) arrays
    const int ld = w + 1;
    double* A = sm;
    double* U = sm + w * ld;
    __shared__ int pairs[2 * 64];
    for (int e = threadIdx.x; e < w * w; e += blockDim.x) {
        const int i = e / w, j = e % w;
        A[i * ld + j] = 0.5 * (H[i * w + j] + H[j * w + i]);
    }
    __syncthreads();
    // the top k of w eigenpairs are kept (and stored in FP32): an absolute
    // stop at 1e-12 of the largest eigenvalue
    cta_jacobi(A, U, w, ld, 30, pairs, 1e-12);
    for (int e = threadIdx.x; e < w * w; e += blockDim.x) evecs[e] = U[(e / w) * ld + (e % w)];
    for (int i = threadIdx.x; i < w; i += blockDim.x) evals[i] = A[i * ld + i];
}

__global__ void colmax_kernel(const float* __restrict__ A, int n, int k, unsigned int* __restrict__ mx) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)n * k) return;
    atomicMax(mx + (idx % k), __float_as_uint(fabsf(A[idx])));
}

__global__ void quant_i8_kernel(const float* __restrict__ A, int n, int k, const unsigned int* __restrict__ mx,
                                int8_t* __restrict__ q, float* __restrict__ scale) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < k) scale[idx] = __uint_as_float(mx[idx]) / 127.0f;
    if (idx >= (int64_t)n * k) return;
    const float s = __uint_as_float(mx[idx % k]) / 127.0f;
    const float v = s > 0.0f ? rintf(A[idx] / s) : 0.0f;
    q[idx] = (int8_t)fmaxf(-127.0f, fminf(127.0f, v));
}

__global__ void quant_fp8_kernel(const float* __restrict__ A, int n, int k, const unsigned int* __restrict__ mx,
                                 __nv_fp8_e4m3* __restrict__ q, float* __restrict__ scale) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < k) scale[idx] = __uint_as_float(mx[idx]) / 448.0f;
    if (idx >= (int64_t)n * k) return;
    const float s = __uint_as_float(mx[idx % k]) / 448.0f;
    q[idx] = __nv_fp8_e4m3(s > 0.0f ? A[idx] / s : 0.0f);
}

// NF4 storage: the reference's 16-level code (fp32_to_nf4 / nf4_to_fp32,
// include/rf_quantization_kernels.hpp:37-65: codes 0..7 hold v/7 for v in
// [0, 1], codes 8..15 hold -(code - 8)/7 for v in [-1, 0)), applied to A / s
// with one scale s = max |A[:, c]| per column so that every column uses the
// whole code range (the reference applies the code to unscaled factors);
// two codes per byte, the lower nibble first, over the row-major n x k entries
// (cuda/rf_proximity_lowrank.cu:353-383 packs its flat factor array the same
// way); an odd count leaves the last upper nibble 0.
__device__ __forceinline__ uint32_t nf4_code(float v) {
    if (v >= 0.0f) return (uint32_t)fminf(7.0f, roundf(v * 7.0f));
    return (uint32_t)fmaxf(8.0f, roundf(8.0f - v * 7.0f));
}

__device__ __forceinline__ float nf4_value(uint32_t code) {
    return code <= 7 ? (float)code / 7.0f : -(float)(code - 8) / 7.0f;
}

__global__ void quant_nf4_kernel(const float* __restrict__ A, int n, int k, const unsigned int* __restrict__ mx,
                                 uint8_t* __restrict__ q, float* __restrict__ scale) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;  // one byte = two entries
    if (idx < k) scale[idx] = __uint_as_float(mx[idx]);
    const int64_t count = (int64_t)n * k;
    if (idx >= (count + 1) / 2) return;
    const int64_t e = 2 * idx;
    const float s0 = __uint_as_float(mx[e % k]);
    const uint32_t lo = nf4_code(s0 > 0.0f ? A[e] / s0 : 0.0f);
    uint32_t hi = 0;
    if (e + 1 < count) {
        const float s1 = __uint_as_float(mx[(e + 1) % k]);
        hi = nf4_code(s1 > 0.0f ? A[e + 1] / s1 : 0.0f);
    }
    q[idx] = (uint8_t)(lo | (hi << 4));
}

__global__ void dequant_nf4_kernel(const uint8_t* __restrict__ q, const float* __restrict__ scale, int n, int k,
                                   float* __restrict__ A) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)n * k) return;
    const uint32_t b = q[idx >> 1];
    A[idx] = nf4_value((idx & 1) ? (b >> 4) : (b & 15u)) * scale[idx % k];
}

// FP16 storage (the reference's FP16 level stores the factors as __half with
// no scale, cuda/rf_proximity_lowrank.cu:300-331); the scales are 1.
__global__ void quant_f16_kernel(const float* __restrict__ A, int n, int k, __half* __restrict__ q,
                                 float* __restrict__ scale) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < k) scale[idx] = 1.0f;
    if (idx >= (int64_t)n * k) return;
    q[idx] = __float2half_rn(A[idx]);
}

template <typename TQ>
__global__ void dequant_kernel(const TQ* __restrict__ q, const float* __restrict__ scale, int n, int k,
                               float* __restrict__ A) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)n * k) return;
    A[idx] = (float)q[idx] * scale[idx % k];
}


inline unsigned nblk(int64_t count, int b = 256) { return (unsigned)((count + b - 1) / b); }

}  // namespace

// Apply M to V (n x w FP32) into MV (n x w FP32).  TX/TG: storage types of the
// packed inputs and the leaf sums.
template <typename TX, typename TG>
rfx_status apply_m(Ctx* c, const float* V, int w, float* MV, const float* dinv, TX* X, TG* G, float* Y,
                   const std::vector<int64_t>& batch_start, int64_t* d_gofs, const std::vector<int64_t>& h_gofs_all,
                   float* Pf, float* Pl, int32_t* fk, float* xs = nullptr, float* gs = nullptr) {
    cudaStream_t s = c->stream;
    const int n = c->n, W = 2 * w;
    StageTimer stt(c, ST_LR_PRODUCT, 0);
    if constexpr (is_fp8<TX>())
        pack_x_fp8_kernel<<<nblk((int64_t)n * 32), 256, 0, s>>>(V, dinv, n, w, X, xs);
    else
        pack_x_kernel<TX><<<nblk((int64_t)n * w), 256, 0, s>>>(V, dinv, n, w, X);
    RFX_CUDA(cudaGetLastError());
    c->launches += 1;
    for (size_t b = 0; b + 1 < batch_start.size(); ++b) {
        const int t0 = (int)batch_start[b], t1 = (int)batch_start[b + 1];
        // key prefix of this batch (device copy prepared by the caller)
        const int64_t* gofs = d_gofs + (h_gofs_all[b]);
        const int64_t keys = h_gofs_all[b + 1] - h_gofs_all[b] - 1;  // stored with one sentinel per batch
        (void)keys;
        const int64_t total_keys = c->h_segbase[t1] - c->h_segbase[t0] - (t1 - t0);
        static_assert(std::is_same<TX, TG>::value, "X and the leaf sums share one storage type");
        const int cpt = (n + SEG_CH - 1) / SEG_CH;
        const int64_t chunks = (int64_t)(t1 - t0) * cpt;
        RFX_CUDA(cudaMemsetAsync(G, 0, sizeof(TG) * (size_t)total_keys * W, s));
        if constexpr (is_fp8<TG>()) RFX_CUDA(cudaMemsetAsync(gs, 0, sizeof(float) * (size_t)total_keys, s));
        auto run = [&](auto e_tag) -> rfx_status {
            constexpr int E = decltype(e_tag)::value;
            // shape 0: the warp takes the chunk's keys in turn; 1: slots of
            // the warp take several keys at once
            const int tk = is_fp8<TX>() ? TK_SEGSUM_FP8 : std::is_same<TX, float>::value ? TK_SEGSUM_F32 : TK_SEGSUM_BF16;
            rfx_status st0 = autotune(c, tk, 2, 0, [&](int shape) -> rfx_status {
                if (shape == 1)
                    segsum_slot_kernel<TX, E, 4><<<nblk(chunks * 32), 256, 0, s>>>(
                        X, n, W, c->d_memb, c->d_segoff, c->d_segbase, t0, t1, cpt, gofs, G, Pf, Pl, fk, xs, gs);
                else
                    segsum_kernel<TX, E><<<nblk(chunks * 32), 256, 0, s>>>(X, n, W, c->d_memb, c->d_segoff,
                                                                           c->d_segbase, t0, t1, cpt, gofs, G, Pf,
                                                                           Pl, fk, xs, gs);
                RFX_CUDA(cudaGetLastError());
                return RFX_OK;
            });
            if (st0 != RFX_OK) return st0;
            segsum_fix_kernel<TG, E><<<nblk(chunks * 32), 256, 0, s>>>(n, W, c->d_segoff, c->d_segbase, t0, t1, cpt,
                                                                       gofs, G, Pf, Pl, fk, gs);
            pull_kernel<TG, E><<<nblk((int64_t)n * 32), 256, 0, s>>>(G, c->d_key, n, W, t0, t1, gofs, Y, b > 0, gs);
            return RFX_OK;
        };
        // BF16 rows narrower than 32 16-byte chunks use 8-byte chunks, so more lanes carry data
        rfx_status rs;
        if constexpr (std::is_same<TX, float>::value) {
            rs = run(std::integral_constant<int, 4>{});
        } else if constexpr (is_fp8<TX>()) {
            rs = run(std::integral_constant<int, 8>{});
        } else {
            if (W / 8 > 16) rs = run(std::integral_constant<int, 8>{});
            else rs = run(std::integral_constant<int, 4>{});
        }
        if (rs != RFX_OK) return rs;
        c->launches += 3;
        RFX_CUDA(cudaGetLastError());
    }
    combine_kernel<<<nblk((int64_t)n * w), 256, 0, s>>>(Y, dinv, n, w, MV);
    c->launches += 1;
    RFX_CUDA(cudaGetLastError());
    return RFX_OK;
}

rfx_status lowrank_compute(Ctx* c, int k, int oversample, int power_iters, int precision, uint64_t seed,
                           float* d_A_out, float* h_evals, const float* d_apply_in, int trees_per_pass) {
    cudaStream_t s = c->stream;
    const int n = c->n, T = c->T;
    const int w = (k + oversample + 7) / 8 * 8;  // rows of whole 16-byte chunks
    if (k < 1 || w > 120 || w > n) {  // 120: two w x (w + 1) FP64 arrays in one CTA's shared memory
        set_error("rfx_lowrank: need 1 <= rank and rank + oversample (rounded up to a multiple of 8) <= min(120, n)");
        return RFX_ERR_INVALID;
    }
    // leaf keys and member lists: reused when this forest's are already built
    rfx_status st = RFX_OK;
    if (!c->csr_built) {
        st = launch_route(c);
        if (st == RFX_OK) st = launch_build_csr(c);
        if (st != RFX_OK) return st;
        c->routed = true;
        c->csr_built = true;
    }
    const int W = 2 * w;
    // tree batches: leaf sums of up to 4 GB per batch (fewer passes over the
    // n x 2w accumulator beat L2-sized batches; RFX_LR_BATCH_MB overrides)
    const bool f8 = precision == 3;  // FP8 e4m3 rows with one scale each
    const size_t gbytes_row = f8 ? (size_t)W + 4 : (size_t)W * (precision ? 2 : 4);
    size_t batch_budget = (size_t)4 << 30;
    if (const char* e = std::getenv("RFX_LR_BATCH_MB")) {
        const long v = std::atol(e);
        if (v > 0) batch_budget = (size_t)v << 20;
    }
    std::vector<int64_t> batch_start{0};
    std::vector<int64_t> h_gofs;  // per batch: key prefix (batch-local), with a sentinel
    std::vector<int64_t> gofs_index;  // offset of each batch's prefix inside h_gofs
    int64_t max_batch_keys = 0;
    int max_batch_trees = 0;
    {
        int t = 0;
        while (t < T) {
            int64_t keys = 0;
            int t1 = t;
            while (t1 < T) {
                const int64_t kt = c->h_segbase[t1 + 1] - c->h_segbase[t1] - 1;
                if (t1 > t && ((size_t)(keys + kt) * gbytes_row > batch_budget ||
                               (trees_per_pass > 0 && t1 - t >= trees_per_pass)))
                    break;
                keys += kt;
                ++t1;
            }
            gofs_index.push_back((int64_t)h_gofs.size());
            int64_t acc = 0;
            for (int q = t; q < t1; ++q) {
                h_gofs.push_back(acc);
                acc += c->h_segbase[q + 1] - c->h_segbase[q] - 1;
            }
            h_gofs.push_back(acc);
            max_batch_keys = std::max(max_batch_keys, acc);
            max_batch_trees = std::max(max_batch_trees, t1 - t);
            batch_start.push_back(t1);
            t = t1;
        }
        gofs_index.push_back((int64_t)h_gofs.size());
    }
    Scratch d(c);
    float* dinv = d.get<float>(n);
    float* Om = d.get<float>((size_t)n * w);
    float* Yw = d.get<float>((size_t)n * w);
    float* Q = d.get<float>((size_t)n * w);
    float* Z = d.get<float>((size_t)n * w);
    float* Ybig = d.get<float>((size_t)n * W);
    int64_t* d_gofs = d.get<int64_t>(h_gofs.size());
    double* Gm = d.get<double>((size_t)w * w);
    double* Tm = d.get<double>((size_t)w * w);
    double* ev = d.get<double>(w);
    double* U = d.get<double>((size_t)w * w);
    int* bad = d.get<int>(1);
    void* X = f8 ? (void*)d.get<uint8_t>((size_t)n * W)
              : precision ? (void*)d.get<__nv_bfloat16>((size_t)n * W) : (void*)d.get<float>((size_t)n * W);
    void* G = f8 ? (void*)d.get<uint8_t>((size_t)max_batch_keys * W)
              : precision ? (void*)d.get<__nv_bfloat16>((size_t)max_batch_keys * W)
                          : (void*)d.get<float>((size_t)max_batch_keys * W);
    float* xs = f8 ? d.get<float>(n) : nullptr;
    float* gs = f8 ? d.get<float>((size_t)max_batch_keys) : nullptr;
    void* X32 = precision == 2 ? (void*)d.get<float>((size_t)n * W) : X;
    void* G32 = precision == 2 ? (void*)d.get<float>((size_t)max_batch_keys * W) : G;
    const size_t nchunks = (size_t)max_batch_trees * ((n + SEG_CH - 1) / SEG_CH);
    float* Pf = d.get<float>(nchunks * W);
    float* Pl = d.get<float>(nchunks * W);
    int32_t* fk = d.get<int32_t>(nchunks);
    if (!dinv || !Om || !Yw || !Q || !Z || !Ybig || !d_gofs || !Gm || !Tm || !ev || !U || !bad || !X || !G || !X32 ||
        !G32 || !Pf || !Pl || !fk || (f8 && (!xs || !gs))) {
        set_error("rfx_lowrank: device allocation failed");
        return RFX_ERR_OOM;
    }
    RFX_CUDA(cudaMemcpyAsync(d_gofs, h_gofs.data(), sizeof(int64_t) * h_gofs.size(), cudaMemcpyHostToDevice, s));
    RFX_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), s));
    dinv_kernel<<<nblk(n), 256, 0, s>>>(c->d_nout, n, dinv);
    gauss_kernel<float><<<nblk((int64_t)n * w), 256, 0, s>>>(Om, (int64_t)n * w, seed);
    c->launches += 2;
    // per-batch prefix pointers: apply_m takes the whole table and indexes it
    std::vector<int64_t> pref_at(gofs_index.begin(), gofs_index.end());
    auto apply = [&](const float* V, float* MV, bool fp32) -> rfx_status {
        if (fp32)
            return apply_m<float, float>(c, V, w, MV, dinv, (float*)X32, (float*)G32, Ybig, batch_start, d_gofs,
                                         pref_at, Pf, Pl, fk);
        if (f8)
            return apply_m<uint8_t, uint8_t>(c, V, w, MV, dinv, (uint8_t*)X, (uint8_t*)G, Ybig, batch_start, d_gofs,
                                             pref_at, Pf, Pl, fk, xs, gs);
        return apply_m<__nv_bfloat16, __nv_bfloat16>(c, V, w, MV, dinv, (__nv_bfloat16*)X, (__nv_bfloat16*)G, Ybig,
                                                     batch_start, d_gofs, pref_at, Pf, Pl, fk);
    };
    if (d_apply_in) {
        // one product MV = M V of the block V (n x w) in the chosen storage
        // form, into d_A_out (n x w)
        if ((st = apply(d_apply_in, d_A_out, precision == 0 || precision == 2)) != RFX_OK) return st;
        RFX_CUDA(cudaStreamSynchronize(s));
        return RFX_OK;
    }
    const size_t sm2 = 2 * (size_t)w * w * sizeof(double);
    RFX_CUDA(cudaFuncSetAttribute(chol_inv_w_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2));
    const size_t sm_eig = 2 * (size_t)w * (w + 1) * sizeof(double);
    RFX_CUDA(cudaFuncSetAttribute(eig_w_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_eig));
    RFX_CUDA(cudaFuncSetAttribute(right_mul_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)right_mul_smem(GW, GW)));
    const int gram_ctas = std::min(GRAM_CTAS, (n + 31) / 32);
    const int gram_threads = std::max(32, (w / 4) * (w / 4));
    double* gpart = d.get<double>((size_t)gram_ctas * w * w);
    if (!gpart) {
        set_error("rfx_lowrank: device allocation failed");
        return RFX_ERR_OOM;
    }
    auto gram = [&](const float* Xa, const float* Ya) {
        gram_f32_kernel<<<gram_ctas, gram_threads, 0, s>>>(Xa, Ya, n, w, gpart);
        gram_sum_w_kernel<<<(unsigned)(((size_t)w * w * 32 + 255) / 256), 256, 0, s>>>(gpart, gram_ctas, w * w, Gm);
    };
    auto orth = [&](const float* src, float* out) -> rfx_status {
        // CholeskyQR2 with FP64 Gram and FP64 triangular factors
        StageTimer stt(c, ST_LR_ORTH, 0);
        const float* cur = src;
        float* tmp = Z;
        for (int pass = 0; pass < 2; ++pass) {
            gram(cur, cur);
            chol_inv_w_kernel<<<1, 256, sm2, s>>>(Gm, w, Tm, bad);
            float* dst = pass == 0 ? tmp : out;
            right_mul_kernel<<<(n + RM_ROWS - 1) / RM_ROWS, right_mul_threads(w), right_mul_smem(w, w), s>>>(
                cur, Tm, n, w, w, dst);
            c->launches += 4;
            RFX_CUDA(cudaGetLastError());
            cur = dst;
        }
        return RFX_OK;
    };
    const bool mixed = precision != 0;
    // sketch: Yw = M Om, then power iterations
    if ((st = apply(Om, Yw, !mixed)) != RFX_OK) return st;
    for (int q = 0; q < power_iters; ++q) {
        if ((st = orth(Yw, Q)) != RFX_OK) return st;
        if ((st = apply(Q, Yw, !mixed)) != RFX_OK) return st;
    }
    if ((st = orth(Yw, Q)) != RFX_OK) return st;
    // Rayleigh-Ritz projection; precision 2 recomputes this last product in FP32
    if ((st = apply(Q, Yw, !mixed || precision == 2)) != RFX_OK) return st;
    gram(Q, Yw);
    eig_w_kernel<<<1, 1024, sm_eig, s>>>(Gm, w, ev, U);
    c->launches += 3;
    RFX_CUDA(cudaGetLastError());
    std::vector<double> hev(w), hU((size_t)w * w);
    RFX_CUDA(cudaMemcpyAsync(hev.data(), ev, sizeof(double) * w, cudaMemcpyDeviceToHost, s));
    RFX_CUDA(cudaMemcpyAsync(hU.data(), U, sizeof(double) * w * w, cudaMemcpyDeviceToHost, s));
    RFX_CUDA(cudaStreamSynchronize(s));
    int hbad = 0;
    RFX_CUDA(cudaMemcpy(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost));
    if (hbad) {
        set_error("rfx_lowrank: the sketch lost rank (Cholesky pivot <= 0)");
        return RFX_ERR_UNSUPPORTED;
    }
    // top-k eigenpairs (largest first); A = Q U_k sqrt(max(lambda, 0))
    std::vector<int> idx(w);
    for (int q = 0; q < w; ++q) idx[q] = q;
    std::sort(idx.begin(), idx.end(), [&](int a, int b) { return hev[a] > hev[b]; });
    std::vector<double> Tk((size_t)w * k);
    for (int col = 0; col < k; ++col) {
        const double lam = hev[idx[col]];
        const double sc = lam > 0 ? std::sqrt(lam) : 0.0;
        if (h_evals) h_evals[col] = (float)lam;
        for (int r = 0; r < w; ++r) Tk[(size_t)r * k + col] = hU[(size_t)r * w + idx[col]] * sc;
    }
    RFX_CUDA(cudaMemcpyAsync(Tm, Tk.data(), sizeof(double) * w * k, cudaMemcpyHostToDevice, s));
    right_mul_kernel<<<(n + RM_ROWS - 1) / RM_ROWS, right_mul_threads(k), right_mul_smem(w, k), s>>>(Q, Tm, n, w, k,
                                                                                                   d_A_out);
    c->launches += 1;
    RFX_CUDA(cudaGetLastError());
    RFX_CUDA(cudaStreamSynchronize(s));
    return RFX_OK;
}

rfx_status lowrank_quantize(Ctx* c, const float* dA, int k, int format, void* dq, float* dscale) {
    cudaStream_t s = c->stream;
    const int n = c->n;
    Scratch d(c);
    unsigned int* mx = d.get<unsigned int>(k);
    if (!mx) return RFX_ERR_OOM;
    RFX_CUDA(cudaMemsetAsync(mx, 0, sizeof(unsigned int) * k, s));
    colmax_kernel<<<nblk((int64_t)n * k), 256, 0, s>>>(dA, n, k, mx);
    if (format == 1)
        quant_i8_kernel<<<nblk((int64_t)n * k), 256, 0, s>>>(dA, n, k, mx, (int8_t*)dq, dscale);
    else if (format == 2)
        quant_fp8_kernel<<<nblk((int64_t)n * k), 256, 0, s>>>(dA, n, k, mx, (__nv_fp8_e4m3*)dq, dscale);
    else if (format == 3)
        quant_nf4_kernel<<<nblk(std::max<int64_t>(((int64_t)n * k + 1) / 2, k)), 256, 0, s>>>(dA, n, k, mx,
                                                                                             (uint8_t*)dq, dscale);
    else
        quant_f16_kernel<<<nblk((int64_t)n * k), 256, 0, s>>>(dA, n, k, (__half*)dq, dscale);
    c->launches += 2;
    RFX_CUDA(cudaGetLastError());
    RFX_CUDA(cudaStreamSynchronize(s));
    return RFX_OK;
}

rfx_status lowrank_dequantize(Ctx* c, const void* dq, const float* dscale, int k, int format, float* dA) {
    cudaStream_t s = c->stream;
    const int n = c->n;
    if (format == 1)
        dequant_kernel<int8_t><<<nblk((int64_t)n * k), 256, 0, s>>>((const int8_t*)dq, dscale, n, k, dA);
    else if (format == 2)
        dequant_kernel<__nv_fp8_e4m3><<<nblk((int64_t)n * k), 256, 0, s>>>((const __nv_fp8_e4m3*)dq, dscale, n, k,
                                                                           dA);
    else if (format == 3)
        dequant_nf4_kernel<<<nblk((int64_t)n * k), 256, 0, s>>>((const uint8_t*)dq, dscale, n, k, dA);
    else
        dequant_kernel<__half><<<nblk((int64_t)n * k), 256, 0, s>>>((const __half*)dq, dscale, n, k, dA);
    c->launches += 1;
    RFX_CUDA(cudaGetLastError());
    return RFX_OK;
}

}  // namespace rfx
