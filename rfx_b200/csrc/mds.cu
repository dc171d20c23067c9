// Classical 3-D MDS of the full proximity matrix, as compute_mds_3d_cpu
// (src/rf_mds_cpu.cpp:88-341) computes it from the float32 matrix
// get_proximity_matrix returns (python/randomforest_py.cpp:1221-1243):
//   Q = rows divided again by nout (rows with nout = 0 kept), symmetrised by
//       averaging, diagonal 1;
//   D = max(Q) - Q, diagonal 0;  B = -1/2 (D^2 - row means - column means +
//       grand mean);
//   the 3 largest eigenvalues above 1e-10, coordinates = eigenvector *
//       sqrt(eigenvalue), row-major n x 3.
// All arithmetic in FP64.  The eigenpairs come from subspace iteration on B
// with a block of S_BLK vectors, CholeskyQR2 re-orthonormalisation and a
// Rayleigh-Ritz step (Jacobi on the S_BLK x S_BLK projection) instead of a full
// dsyevd; eigenvectors are defined up to sign.  The full-matrix form filters
// the block with Chebyshev polynomials of B (degree 8) between Rayleigh-Ritz
// steps, so that a third eigenvalue close to a cluster below it (the plain
// method at n = 2,000 / 500 trees has lambda3 / lambda17 = 1.02) still
// converges in a few hundred products.
#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

#include "dense.cuh"
#include "rfx_internal.cuh"

namespace rfx {
namespace {

constexpr int S_BLK = 16;  // subspace width

__device__ __forceinline__ double q_value(const float* __restrict__ P, const int32_t* __restrict__ nout, int n,
                                          int i, int j) {
    if (i == j) return 1.0;
    // P is read through the reference's column-major view of the C-order array
    const double pij = (double)P[(size_t)j * n + i];
    const double pji = (double)P[(size_t)i * n + j];
    const int ni = nout[i], nj = nout[j];
    const double a = ni > 0 ? __ddiv_rn(pij, (double)ni) : pij;
    const double b = nj > 0 ? __ddiv_rn(pji, (double)nj) : pji;
    return __dmul_rn(0.5, __dadd_rn(a, b));
}

__global__ void mds_max_kernel(const float* __restrict__ P, const int32_t* __restrict__ nout, int n,
                               unsigned long long* __restrict__ maxbits) {
    double m = 0.0;
    const size_t total = (size_t)n * n;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(e / n), j = (int)(e % n);
        m = fmax(m, q_value(P, nout, n, i, j));
    }
    for (int d = 16; d > 0; d >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, d));
    // non-negative doubles order like their bit patterns
    if ((threadIdx.x & 31) == 0) atomicMax(maxbits, (unsigned long long)__double_as_longlong(m));
}

// B and row sums of D^2 in two passes: (1) row sums, (2) B.
__global__ void mds_rowsum_kernel(const float* __restrict__ P, const int32_t* __restrict__ nout, int n,
                                  const unsigned long long* __restrict__ maxbits, double* __restrict__ rowmean) {
    const int i = blockIdx.x;
    const double mx = __longlong_as_double((long long)*maxbits);
    double s = 0.0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const double d = (i == j) ? 0.0 : __dsub_rn(mx, q_value(P, nout, n, i, j));
        s = __dadd_rn(s, __dmul_rn(d, d));
    }
    __shared__ double red[32];
    for (int d = 16; d > 0; d >>= 1) s += __shfl_down_sync(0xffffffffu, s, d);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
        if (threadIdx.x == 0) rowmean[i] = v / (double)n;
    }
}

__global__ void mds_grand_kernel(const double* __restrict__ rowmean, int n, double* __restrict__ grand) {
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += rowmean[i];
    __shared__ double red[32];
    for (int d = 16; d > 0; d >>= 1) s += __shfl_down_sync(0xffffffffu, s, d);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
        if (threadIdx.x == 0) *grand = v / (double)n;
    }
}

// B in 64 x 64 tiles, tile (I, K) at (I * nt + K) * TILE_D doubles, rows of
// TILE_LD doubles (64 values and 4 of padding, so that one bulk copy brings a
// tile straight into the product kernel's bank-conflict-free layout); values
// outside the n x n matrix and the padding are zero.
constexpr int TILE_LD = 68;
constexpr int TILE_D = 64 * TILE_LD;

__global__ void mds_b_kernel(const float* __restrict__ P, const int32_t* __restrict__ nout, int n, int nt,
                             const unsigned long long* __restrict__ maxbits, const double* __restrict__ rowmean,
                             const double* __restrict__ grand, double* __restrict__ B) {
    const double mx = __longlong_as_double((long long)*maxbits);
    const double g = *grand;
    const size_t total = (size_t)nt * nt * TILE_D;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const size_t tile = e / TILE_D;
        const int within = (int)(e % TILE_D);
        const int r = within / TILE_LD, cc = within % TILE_LD;
        const int i = (int)(tile / nt) * 64 + r, j = (int)(tile % nt) * 64 + cc;
        if (cc >= 64 || i >= n || j >= n) {
            B[e] = 0.0;
            continue;
        }
        const double d = (i == j) ? 0.0 : __dsub_rn(mx, q_value(P, nout, n, i, j));
        const double v = __dadd_rn(__dsub_rn(__dsub_rn(__dmul_rn(d, d), rowmean[i]), rowmean[j]), g);
        B[e] = __dmul_rn(-0.5, v);
    }
}

// W[n x S] = B[n x n] V[n x S] in FP64 on the tensor cores (mma.sync
// m16n8k4 .f64; Blackwell's tcgen05 has no FP64 kind).  B is stored in
// 64 x 64 tiles with rows 544 bytes apart (mds_b_kernel), so a tile is one
// contiguous bulk copy that lands in a layout whose fragment reads are free
// of bank conflicts.  A CTA of four warps owns 64 rows and one range of
// kchunk columns; each 64-column step brings the B tile and the matching
// 64 x 16 block of V (pre-arranged in fragment order by bv_pack_kernel)
// through a DB_STAGES-deep mbarrier pipeline, two bulk copies per step.  Warp w multiplies rows 16w..16w+15 by both 8-column halves of V.
// The partial products go to Wpart[range] and are added in range order.
constexpr int GT = 64;
constexpr int BV_KSPLIT = 8;  // column ranges per row tile (enough CTAs to fill the GPU in several waves)
constexpr int DB_STAGES = 4;
constexpr int DB_RS = GT * 8 + 32;                          // bytes between tile rows in shared memory
constexpr int DB_VBYTES = GT * S_BLK * 8;                   // one 64 x 16 block of V
constexpr int DB_STAGE = GT * DB_RS + DB_VBYTES;            // 43,008 bytes
static_assert(DB_RS == TILE_LD * 8, "a bulk-copied B tile keeps its row stride in shared memory");
constexpr size_t DB_SMEM = (size_t)DB_STAGES * DB_STAGE;    // 172,032 bytes
constexpr int DB_WAIT_LIMIT = 1 << 24;

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void db_mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count));
}

__device__ __forceinline__ void db_expect_tx(uint32_t mbar, uint32_t bytes) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(mbar),
                 "r"(bytes)
                 : "memory");
}

// bounded wait for the completion with parity `parity`
__device__ __forceinline__ bool db_wait(uint32_t mbar, uint32_t parity) {
    for (int it = 0; it < DB_WAIT_LIMIT; ++it) {
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

__device__ __forceinline__ void db_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(mbar)
                 : "memory");
}

// D += A B for one m16n8k4 FP64 tile: a0/a1 = A[g][t], A[g+8][t]; b = B[t][g];
// c0..c3 = D[g][2t], D[g][2t+1], D[g+8][2t], D[g+8][2t+1] (g = lane / 4,
// t = lane % 4)
__device__ __forceinline__ void dmma(double* c, double a0, double a1, double b) {
    asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
                 : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
                 : "d"(a0), "d"(a1), "d"(b));
}

// Vf = V in fragment order, npad rows (rows >= n zero): within each 4-row
// step, element (k, c) sits at (c / 8) * 32 + (c % 8) * 4 + k % 4, so the
// lanes of a warp read 32 consecutive doubles per fragment.
__global__ void bv_pack_kernel(const double* __restrict__ V, int n, int npad, double* __restrict__ Vf) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t)npad * S_BLK) return;
    const int k = (int)(idx / S_BLK), c = (int)(idx % S_BLK);
    const size_t dst = (size_t)(k >> 2) * 64 + (c >> 3) * 32 + (c & 7) * 4 + (k & 3);
    Vf[dst] = k < n ? V[idx] : 0.0;
}

__global__ void __launch_bounds__(128, 1) dgemm_bv_kernel(const double* __restrict__ B, int nt,
                                                         const double* __restrict__ Vf, int n, int kchunk,
                                                         double* __restrict__ Wpart, uint32_t* __restrict__ err) {
    extern __shared__ __align__(128) uint8_t dsm[];
    __shared__ __align__(8) uint64_t full[DB_STAGES];
    __shared__ int s_fail;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t = lane & 3;
    const int r0 = blockIdx.x * GT;
    const int kbeg = blockIdx.y * kchunk, kend = min(n, kbeg + kchunk);
    const int ntile = (kend - kbeg + GT - 1) / GT;  // >= 1: every range starts below n
    const uint32_t base = su32(dsm);
    if (tid == 0) {
        for (int s = 0; s < DB_STAGES; ++s) db_mbar_init(su32(&full[s]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_fail = 0;
    }
    __syncthreads();
    // warp 0 brings tile `it` into its stage: 64 row copies and the V block
    auto issue = [&](int it) {
        const int s = it % DB_STAGES;
        const int k0 = kbeg + it * GT;
        const uint32_t dst = base + (uint32_t)(s * DB_STAGE);
        const uint32_t bar = su32(&full[s]);
        if (lane == 0) {
            db_expect_tx(bar, GT * DB_RS + DB_VBYTES);
            db_g2s(dst, B + ((size_t)blockIdx.x * nt + k0 / GT) * TILE_D, GT * DB_RS, bar);
            db_g2s(dst + (uint32_t)(GT * DB_RS), Vf + (size_t)k0 * S_BLK, DB_VBYTES, bar);
        }
    };
    int issued = 0;
    if (warp == 0)
        for (; issued < min(DB_STAGES - 1, ntile); ++issued) issue(issued);
    double acc[2][4] = {{0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0}};
    const int arow = (warp * 16 + g) * (DB_RS / 8) + t;  // A[g][t] of this warp's rows, in doubles
    int it = 0;
    for (; it < ntile; ++it) {
        // every warp is done with tile it - 1, so its stage can be refilled
        __syncthreads();
        if (s_fail) break;
        if (warp == 0 && it + DB_STAGES - 1 < ntile) {
            issue(it + DB_STAGES - 1);
            issued = it + DB_STAGES;
        }
        const int s = it % DB_STAGES;
        if (!db_wait(su32(&full[s]), (uint32_t)((it / DB_STAGES) & 1))) {
            if (lane == 0) {
                s_fail = 1;
                atomicOr(err, ERR_WAIT_LIMIT);
            }
            continue;  // the next barrier ends the loop for every warp
        }
        const double* Bs = reinterpret_cast<const double*>(dsm + s * DB_STAGE);
        const double* Vs = reinterpret_cast<const double*>(dsm + s * DB_STAGE + GT * DB_RS);
#pragma unroll
        for (int ks = 0; ks < GT / 4; ++ks) {
            const double a0 = Bs[arow + ks * 4];
            const double a1 = Bs[arow + 8 * (DB_RS / 8) + ks * 4];
            const double b0 = Vs[ks * 64 + g * 4 + t];
            const double b1 = Vs[ks * 64 + 32 + g * 4 + t];
            dmma(acc[0], a0, a1, b0);
            dmma(acc[1], a0, a1, b1);
        }
    }
    __syncthreads();
    if (s_fail) {
        // a wait gave up at tile it - 1 (or at the last tile): the copies
        // issued from there on land before the CTA leaves (bounded waits;
        // a completed tile's wait returns at once)
        if (warp == 0 && lane == 0)
            for (int q = max(0, it - 1); q < issued; ++q)
                db_wait(su32(&full[q % DB_STAGES]), (uint32_t)((q / DB_STAGES) & 1));
        return;
    }
    double* out = Wpart + ((size_t)blockIdx.y * n) * S_BLK;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int col = h * 8 + 2 * t;
        const int ra = r0 + warp * 16 + g, rb = ra + 8;
        if (ra < n) *reinterpret_cast<double2*>(out + (size_t)ra * S_BLK + col) = make_double2(acc[h][0], acc[h][1]);
        if (rb < n) *reinterpret_cast<double2*>(out + (size_t)rb * S_BLK + col) = make_double2(acc[h][2], acc[h][3]);
    }
}

// W = sum of the ksn partial products, added in range order (reproducible).
__global__ void bv_reduce_kernel(const double* __restrict__ Wpart, int n, int ksn, double* __restrict__ W) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t cnt = (size_t)n * S_BLK;
    if (idx >= cnt) return;
    double a = Wpart[idx];
    for (int s = 1; s < ksn; ++s) a += Wpart[(size_t)s * cnt + idx];
    W[idx] = a;
}

// G[S x S] += X^T Y over rows (atomics into a zeroed G).
// Per-CTA partial Gram matrices X^T Y (16 x 16) into part[blockIdx.x], added
// by gram_sum_kernel in a fixed order (reproducible run to run).
__global__ void __launch_bounds__(256) dgram_kernel(const double* __restrict__ X, const double* __restrict__ Y, int n,
                                                    double* __restrict__ part) {
    __shared__ double Xs[64][S_BLK], Ys[64][S_BLK];
    const int tid = threadIdx.x;
    const int a = tid / S_BLK, b = tid % S_BLK;  // 16 x 16 outputs
    double acc = 0.0;
    for (int r0 = blockIdx.x * 64; r0 < n; r0 += gridDim.x * 64) {
        for (int e = tid; e < 64 * S_BLK; e += 256) {
            const int r = e / S_BLK, c = e % S_BLK;
            Xs[r][c] = (r0 + r < n) ? X[(size_t)(r0 + r) * S_BLK + c] : 0.0;
            Ys[r][c] = (r0 + r < n) ? Y[(size_t)(r0 + r) * S_BLK + c] : 0.0;
        }
        __syncthreads();
        for (int r = 0; r < 64; ++r) acc = fma(Xs[r][a], Ys[r][b], acc);
        __syncthreads();
    }
    part[(size_t)blockIdx.x * (S_BLK * S_BLK) + a * S_BLK + b] = acc;
}

// G[e] = sum over the partials, one warp per entry (lane l the partials l,
// l + 32, ..., then a fixed shuffle tree)
__global__ void gram_sum_kernel(const double* __restrict__ part, int nparts, double* __restrict__ G) {
    const int e = (int)(((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (e >= S_BLK * S_BLK) return;
    double v = 0.0;
    for (int q = lane; q < nparts; q += 32) v += part[(size_t)q * (S_BLK * S_BLK) + e];
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    if (lane == 0) G[e] = v;
}

// One CTA: Cholesky of G and the inverse of its factor, T = L^{-T} (S x S).
__global__ void chol_inv_kernel(const double* __restrict__ G, double* __restrict__ Tm, int* __restrict__ bad) {
    __shared__ double L[S_BLK * S_BLK], Li[S_BLK * S_BLK];
    __shared__ double flag;
    for (int e = threadIdx.x; e < S_BLK * S_BLK; e += blockDim.x) L[e] = G[e];
    __syncthreads();
    if (!cta_cholesky(L, S_BLK, S_BLK, &flag) && threadIdx.x == 0) *bad = 1;
    cta_tri_inverse(L, Li, S_BLK, S_BLK);
    for (int e = threadIdx.x; e < S_BLK * S_BLK; e += blockDim.x) {
        const int i = e / S_BLK, j = e % S_BLK;
        Tm[i * S_BLK + j] = Li[j * S_BLK + i];  // (L^{-1})^T
    }
}

// V = W T (rows of W times an S x S matrix).
__global__ void dright_kernel(const double* __restrict__ W, const double* __restrict__ Tm, int n,
                              double* __restrict__ V) {
    __shared__ double Ts[S_BLK * S_BLK];
    for (int e = threadIdx.x; e < S_BLK * S_BLK; e += blockDim.x) Ts[e] = Tm[e];
    __syncthreads();
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t)n * S_BLK) return;
    const int r = (int)(idx / S_BLK), c = (int)(idx % S_BLK);
    double v = 0.0;
    for (int k = 0; k < S_BLK; ++k) v = fma(W[(size_t)r * S_BLK + k], Ts[k * S_BLK + c], v);
    V[idx] = v;
}

// One CTA: eigen-decomposition of the S x S projection H (symmetrised).
__global__ void rr_kernel(const double* __restrict__ H, double* __restrict__ evals, double* __restrict__ evecs) {
    constexpr int LD = S_BLK + 1;
    __shared__ double A[S_BLK * LD], U[S_BLK * LD];
    __shared__ int pairs[2 * 64];
    for (int e = threadIdx.x; e < S_BLK * S_BLK; e += blockDim.x) {
        const int i = e / S_BLK, j = e % S_BLK;
        A[i * LD + j] = 0.5 * (H[i * S_BLK + j] + H[j * S_BLK + i]);
    }
    __syncthreads();
    cta_jacobi(A, U, S_BLK, LD, 30, pairs);
    for (int e = threadIdx.x; e < S_BLK * S_BLK; e += blockDim.x) evecs[e] = U[(e / S_BLK) * LD + (e % S_BLK)];
    for (int i = threadIdx.x; i < S_BLK; i += blockDim.x) evals[i] = A[i * LD + i];
}

// coords[i][c] = (V U)[i][sel[c]] * scale[c]
__global__ void coords_kernel(const double* __restrict__ V, const double* __restrict__ U, const int* __restrict__ sel,
                              const double* __restrict__ scale, int n, int k, double* __restrict__ out) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t)n * k) return;
    const int i = (int)(idx / k), c = (int)(idx % k);
    double v = 0.0;
    for (int q = 0; q < S_BLK; ++q) v = fma(V[(size_t)i * S_BLK + q], U[q * S_BLK + sel[c]], v);
    out[idx] = v * scale[c];
}


}  // namespace

// Seeded Gaussian start block on the device (counter hash splitmix64 and
// Box-Muller); any full-rank start converges to the same subspace.
__device__ __forceinline__ uint64_t start_mix(uint64_t z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// out = a X + b Y + c Z over an n x S_BLK block (Z may be null); the
// three-term recurrence of the Chebyshev filter.
__global__ void block_axpby_kernel(double a, const double* __restrict__ X, double b, const double* __restrict__ Y,
                                   double c, const double* __restrict__ Z, int64_t count, double* __restrict__ out) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count) return;
    double v = __dadd_rn(__dmul_rn(a, X[e]), __dmul_rn(b, Y[e]));
    if (Z) v = __dadd_rn(v, __dmul_rn(c, Z[e]));
    out[e] = v;
}

__global__ void start_block_kernel(double* __restrict__ V, int64_t count, uint64_t seed) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= count) return;
    const uint64_t h = start_mix(seed ^ start_mix((uint64_t)idx));
    const double u1 = ((h >> 11) + 1.0) * (1.0 / 9007199254740993.0);
    const double u2 = (double)(start_mix(h) >> 11) * (1.0 / 9007199254740992.0);
    V[idx] = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
}

// Subspace iteration on the symmetric operator applied by `apply` (W = B V),
// returning the k largest eigenpairs above 1e-10: coordinates n x k in `out`
// (device) and eigenvalues in `evals_out` (host).  Shared by the full-matrix
// and the factor MDS.
template <typename Apply>
rfx_status subspace_topk(Ctx* c, int n, int k, Apply apply, int max_iter, double* d_out, double* evals_out,
                         uint64_t seed, double tol = 1e-14, const double* warm_in = nullptr, double* keep_out = nullptr,
                         int* iters_out = nullptr, bool floor_stop = false, int cheb = 0) {
    cudaStream_t s = c->stream;
    Scratch d(c);
    double* V = d.get<double>((size_t)n * S_BLK);
    double* W = d.get<double>((size_t)n * S_BLK);
    double* G = d.get<double>(S_BLK * S_BLK);
    double* Tm = d.get<double>(S_BLK * S_BLK);
    double* ev = d.get<double>(S_BLK);
    double* U = d.get<double>(S_BLK * S_BLK);
    int* bad = d.get<int>(1);
    int* sel = d.get<int>(8);
    double* scale = d.get<double>(8);
    if (!V || !W || !G || !Tm || !ev || !U || !bad || !sel || !scale) {
        set_error("MDS: device allocation failed");
        return RFX_ERR_OOM;
    }
    // start block: a warm start (a previous basis) or a seeded Gaussian
    // (srand(12345 + 1000*eig) seeds the reference's factor MDS; any start
    // converges to the same subspace)
    if (warm_in) {
        RFX_CUDA(cudaMemcpyAsync(V, warm_in, sizeof(double) * (size_t)n * S_BLK, cudaMemcpyDeviceToDevice, s));
    } else {
        const int64_t cnt = (int64_t)n * S_BLK;
        start_block_kernel<<<(unsigned)((cnt + 255) / 256), 256, 0, s>>>(V, cnt, seed);
        c->launches += 1;
        RFX_CUDA(cudaGetLastError());
    }
    RFX_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), s));
    double* Xt = d.get<double>((size_t)n * S_BLK);
    if (!Xt) {
        set_error("MDS: device allocation failed");
        return RFX_ERR_OOM;
    }
    const int gb = std::min(1024, (n + 63) / 64);
    double* gpart = d.get<double>((size_t)gb * S_BLK * S_BLK);
    if (!gpart) {
        set_error("MDS: device allocation failed");
        return RFX_ERR_OOM;
    }
    auto gram = [&](const double* X, const double* Y) {
        dgram_kernel<<<gb, 256, 0, s>>>(X, Y, n, gpart);
        gram_sum_kernel<<<S_BLK * S_BLK * 32 / 256, 256, 0, s>>>(gpart, gb, G);
    };
    // CholeskyQR2: Out = (src L1^{-T}) L2^{-T}, through the temporary Xt
    auto orth = [&](const double* src, double* Out) -> rfx_status {
        const unsigned gr = (unsigned)(((size_t)n * S_BLK + 255) / 256);
        gram(src, src);
        chol_inv_kernel<<<1, 128, 0, s>>>(G, Tm, bad);
        dright_kernel<<<gr, 256, 0, s>>>(src, Tm, n, Xt);
        gram(Xt, Xt);
        chol_inv_kernel<<<1, 128, 0, s>>>(G, Tm, bad);
        dright_kernel<<<gr, 256, 0, s>>>(Xt, Tm, n, Out);
        c->launches += 8;
        RFX_CUDA(cudaGetLastError());
        return RFX_OK;
    };
    rfx_status st;
    if ((st = orth(V, V)) != RFX_OK) return st;  // src and Out may alias: Xt sits between
    std::vector<double> prev(S_BLK, 0.0), cur(S_BLK, 0.0), hist;
    std::vector<double> hU(S_BLK * S_BLK);
    // Rayleigh-Ritz on span(V) with W = B V: eigenvalues into cur, change of
    // the k largest against the previous check into *delta
    auto ritz = [&](double* delta) -> rfx_status {
        gram(V, W);
        rr_kernel<<<1, 128, 0, s>>>(G, ev, U);
        c->launches += 3;
        RFX_CUDA(cudaMemcpyAsync(cur.data(), ev, sizeof(double) * S_BLK, cudaMemcpyDeviceToHost, s));
        RFX_CUDA(cudaStreamSynchronize(s));
        std::vector<double> a = cur, b = prev;
        std::sort(a.rbegin(), a.rend());
        std::sort(b.rbegin(), b.rend());
        double dl = 0.0;
        for (int q = 0; q < k; ++q) dl = std::max(dl, std::fabs(a[q] - b[q]) / std::max(std::fabs(a[q]), 1e-300));
        prev = cur;
        *delta = dl;
        return RFX_OK;
    };
    if (cheb > 0) {
        // Chebyshev-filtered subspace iteration: after a few plain steps, each
        // outer step applies T_cheb of B mapped so that [-|theta|max,
        // theta_min] (theta = the block's Ritz values; |lambda_min| <= the
        // largest |Ritz value| for the operators used here) goes to [-1, 1]:
        // the components below the block's smallest Ritz value are damped,
        // the top ones grow like cosh(cheb * acosh(x)), so a cluster of close
        // eigenvalues below the wanted ones costs far fewer products than
        // plain powers.  The stop rule is the eigenvalue change < tol.
        Scratch dc(c);
        double* Y0 = dc.get<double>((size_t)n * S_BLK);
        double* Y1 = dc.get<double>((size_t)n * S_BLK);
        double* Y2 = dc.get<double>((size_t)n * S_BLK);
        if (!Y0 || !Y1 || !Y2) {
            set_error("MDS: device allocation failed");
            return RFX_ERR_OOM;
        }
        const int64_t cnt = (int64_t)n * S_BLK;
        const unsigned gb = (unsigned)((cnt + 255) / 256);
        for (int q = 0; q < 10; ++q) {
            if ((st = apply(V, W)) != RFX_OK) return st;
            if ((st = orth(W, V)) != RFX_OK) return st;
        }
        int matvecs = 10;
        for (int outer = 0; matvecs < max_iter; ++outer) {
            if ((st = apply(V, W)) != RFX_OK) return st;
            ++matvecs;
            double delta = 0.0;
            if ((st = ritz(&delta)) != RFX_OK) return st;
            if (iters_out) *iters_out = matvecs;
            // also stop at the rounding floor: below 1e-9 a change that is no
            // smaller than the last three means the products' rounding, not
            // the iteration, sets it
            hist.push_back(delta);
            const size_t hn = hist.size();
            const bool floor = hn >= 4 && delta < 1e-9 &&
                               delta >= std::min(hist[hn - 2], std::min(hist[hn - 3], hist[hn - 4]));
            if (delta < tol || floor || matvecs + cheb > max_iter) break;
            double thmax = 0.0, thmin = cur[0];
            for (double v : cur) {
                thmax = std::max(thmax, std::fabs(v));
                thmin = std::min(thmin, v);
            }
            const double lo = -thmax, hi = thmin;
            const double cc = 0.5 * (lo + hi), ee = 0.5 * (hi - lo);
            if (!(ee > 0.0)) break;
            // Y0 = V, Y1 = (B V - cc V) / ee, Y_{j+1} = 2 (B Y_j - cc Y_j) / ee - Y_{j-1}
            RFX_CUDA(cudaMemcpyAsync(Y0, V, sizeof(double) * cnt, cudaMemcpyDeviceToDevice, s));
            block_axpby_kernel<<<gb, 256, 0, s>>>(1.0 / ee, W, -cc / ee, V, 0.0, nullptr, cnt, Y1);
            c->launches += 1;
            for (int j = 2; j <= cheb; ++j) {
                if ((st = apply(Y1, W)) != RFX_OK) return st;
                ++matvecs;
                block_axpby_kernel<<<gb, 256, 0, s>>>(2.0 / ee, W, -2.0 * cc / ee, Y1, -1.0, Y0, cnt, Y2);
                c->launches += 1;
                std::swap(Y0, Y1);
                std::swap(Y1, Y2);
            }
            RFX_CUDA(cudaGetLastError());
            if ((st = orth(Y1, V)) != RFX_OK) return st;
        }
    } else
    for (int it = 1; it <= max_iter; ++it) {
        if ((st = apply(V, W)) != RFX_OK) return st;
        const bool check = (it % 10 == 0) || it == max_iter;
        if (check) {
            // Rayleigh-Ritz on span(V): H = V^T (B V)
            gram(V, W);
            rr_kernel<<<1, 128, 0, s>>>(G, ev, U);
            c->launches += 3;
            RFX_CUDA(cudaMemcpyAsync(cur.data(), ev, sizeof(double) * S_BLK, cudaMemcpyDeviceToHost, s));
            RFX_CUDA(cudaStreamSynchronize(s));
            std::vector<double> a = cur, b = prev;
            std::sort(a.rbegin(), a.rend());
            std::sort(b.rbegin(), b.rend());
            double delta = 0.0;
            for (int q = 0; q < k; ++q) delta = std::max(delta, std::fabs(a[q] - b[q]) / std::max(std::fabs(a[q]), 1e-300));
            prev = cur;
            if (iters_out) *iters_out = it;
            // stop at the tolerance, or when the change no longer shrinks (the
            // operator's rounding floor has been reached)
            hist.push_back(delta);
            const size_t hn = hist.size();
            // (no new minimum over the last three checks: the change only
            // fluctuates; with floor_stop, for operators applied in FP32 or
            // BF16, already when it has not halved over the last three checks)
            const bool stalled =
                it >= 40 && hn >= 4 &&
                (floor_stop ? hist[hn - 1] > 0.5 * hist[hn - 4]
                            : std::min(hist[hn - 1], std::min(hist[hn - 2], hist[hn - 3])) >= hist[hn - 4]);
            if (delta < tol || stalled || it == max_iter) break;
        }
        if ((st = orth(W, V)) != RFX_OK) return st;
    }
    int hbad = 0;
    RFX_CUDA(cudaMemcpy(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost));
    if (hbad) {
        set_error("MDS: the subspace lost rank (Cholesky pivot <= 0)");
        return RFX_ERR_UNSUPPORTED;
    }
    // select the k largest eigenvalues above 1e-10 (descending)
    std::vector<int> idx(S_BLK);
    for (int q = 0; q < S_BLK; ++q) idx[q] = q;
    std::sort(idx.begin(), idx.end(), [&](int x, int y) { return cur[x] > cur[y]; });
    std::vector<int> hs(k);
    std::vector<double> hsc(k);
    for (int q = 0; q < k; ++q) {
        if (!(cur[idx[q]] > 1e-10)) {
            set_error("Not enough positive eigenvalues for MDS. Proximity matrix may not be Euclidean.");
            return RFX_ERR_UNSUPPORTED;
        }
        hs[q] = idx[q];
        hsc[q] = std::sqrt(std::fabs(cur[idx[q]]));
        if (evals_out) evals_out[q] = cur[idx[q]];
    }
    RFX_CUDA(cudaMemcpyAsync(sel, hs.data(), sizeof(int) * k, cudaMemcpyHostToDevice, s));
    RFX_CUDA(cudaMemcpyAsync(scale, hsc.data(), sizeof(double) * k, cudaMemcpyHostToDevice, s));
    coords_kernel<<<(unsigned)(((size_t)n * k + 255) / 256), 256, 0, s>>>(V, U, sel, scale, n, k, d_out);
    if (keep_out) RFX_CUDA(cudaMemcpyAsync(keep_out, V, sizeof(double) * (size_t)n * S_BLK, cudaMemcpyDeviceToDevice, s));
    c->launches += 1;
    RFX_CUDA(cudaGetLastError());
    RFX_CUDA(cudaStreamSynchronize(s));
    return RFX_OK;
}

// ---------------------------------------------------------------------------
// MDS from low-rank factors.
//
// With P ~= I + A A^T (A: n x k) and D_ij = 1 - P_ij off the diagonal, 0 on it
// (the reference's compute_mds_from_factors distance D = 1 - P / max(diag P),
// cuda/rf_proximity_lowrank.cu:1966-2003, with the unit diagonal of P),
//   D^2 = 11^T - 2 A A^T + (A.A)(A.A)^T - diag(c),  c_i = (1 - |a_i|^2)^2,
// where (A.A) is the row-wise Kronecker square, and the double-centred
//   B = J A A^T J - 1/2 J (A.A)(A.A)^T J + 1/2 J diag(c) J.
// B V is applied without forming n x n objects:
//   u = J V;  T1 = A (A^T u);  M_j = A^T diag(u_j) A (k x k);
//   T2_ij = a_i^T M_j a_i;  B V = J (T1 - T2/2 + c.u/2).
// The two k^2-wide reductions (M_j and the quadratic forms) carry the work.
// ---------------------------------------------------------------------------
namespace {

// Column means of an n x 16 FP64 block in a fixed summation order: per-CTA
// partial sums over a strided row set, then one warp per output adds the
// partials (lane l the partials l, l + 32, ..., then a fixed shuffle tree), so
// the result is reproducible run to run.
constexpr int RED_CTAS = 1184;  // eight CTAs per SM

// out[e] = scale * sum over p of part[p * cnt + e], one warp per e
template <typename TV>
__global__ void part_sum_kernel(const TV* __restrict__ part, int nparts, int cnt, TV scale, TV* __restrict__ out) {
    const int e = (int)(((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (e >= cnt) return;
    TV s = 0;
    for (int q = lane; q < nparts; q += 32) s += part[(size_t)q * cnt + e];
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) s += __shfl_xor_sync(0xffffffffu, s, d);
    if (lane == 0) out[e] = s * scale;
}

__global__ void __launch_bounds__(256) colsum_part_kernel(const double* __restrict__ V, int n,
                                                          double* __restrict__ part) {
    const int r = threadIdx.x / S_BLK, j = threadIdx.x % S_BLK;  // 16 rows x 16 columns per pass
    double s = 0.0;
    for (int i = blockIdx.x * 16 + r; i < n; i += gridDim.x * 16) s += V[(size_t)i * S_BLK + j];
    __shared__ double red[16][S_BLK];
    red[r][j] = s;
    __syncthreads();
    if (threadIdx.x < S_BLK) {
        double t = 0.0;
        for (int q = 0; q < 16; ++q) t += red[q][threadIdx.x];
        part[(size_t)blockIdx.x * S_BLK + threadIdx.x] = t;
    }
}

// u = V - mean (FP64), also as FP32
__global__ void center_kernel(const double* __restrict__ V, const double* __restrict__ mean, int n,
                              double* __restrict__ u, float* __restrict__ u32) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)n * S_BLK) return;
    const double v = V[idx] - mean[idx % S_BLK];
    u[idx] = v;
    u32[idx] = (float)v;
}

// AtU[a][j] = sum_i A[i][a] u[i][j] in FP64: per-CTA partials (64 columns x
// 4 row groups per CTA, all 16 j per thread), then a fixed-order sum over CTAs.
__global__ void __launch_bounds__(256) atu_part_kernel(const float* __restrict__ A, const double* __restrict__ u, int n,
                                                       int k, double* __restrict__ part) {
    const int a = threadIdx.x % 64, rg = threadIdx.x / 64;
    double acc[S_BLK];
#pragma unroll
    for (int j = 0; j < S_BLK; ++j) acc[j] = 0.0;
    if (a < k) {
#pragma unroll 4
        for (int i = blockIdx.x * 4 + rg; i < n; i += gridDim.x * 4) {
            const double x = (double)__ldg(A + (size_t)i * k + a);
            // the FP64 row of u (shared by the CTA's 64 columns): no conversions per product
            const double2* ur = reinterpret_cast<const double2*>(u + (size_t)i * S_BLK);
#pragma unroll
            for (int q = 0; q < S_BLK / 2; ++q) {
                const double2 v = __ldg(ur + q);
                acc[2 * q] = fma(x, v.x, acc[2 * q]);
                acc[2 * q + 1] = fma(x, v.y, acc[2 * q + 1]);
            }
        }
    }
    __shared__ double red[4][64][S_BLK + 1];
#pragma unroll
    for (int j = 0; j < S_BLK; ++j) red[rg][a][j] = acc[j];
    __syncthreads();
    for (int e = threadIdx.x; e < k * S_BLK; e += blockDim.x) {
        const int aa = e / S_BLK, j = e % S_BLK;
        part[(size_t)blockIdx.x * k * S_BLK + e] = ((red[0][aa][j] + red[1][aa][j]) + red[2][aa][j]) + red[3][aa][j];
    }
}

// Partial M[j][a][b] = sum over the CTA's row chunks of u[i][j] A[i][a]
// A[i][b]; one CTA per (row-chunk set, j); each thread a 4 x 4 block of
// (a, b).  k <= 64.
constexpr int MS_ROWS = 128;
__global__ void __launch_bounds__(256) mstack_f32_kernel(const float* __restrict__ A, const float* __restrict__ u,
                                                         int n, int k, float* __restrict__ M) {
    __shared__ float As[MS_ROWS][65];
    __shared__ float us[MS_ROWS];
    const int j = blockIdx.y;
    const int tid = threadIdx.x;
    const int ab = tid;  // 16 x 16 blocks of 4 x 4
    const int a0 = (ab / 16) * 4, b0 = (ab % 16) * 4;
    float acc[4][4] = {};
    for (int r0 = blockIdx.x * MS_ROWS; r0 < n; r0 += gridDim.x * MS_ROWS) {
        for (int e = tid; e < MS_ROWS * 64; e += 256) {
            const int r = e / 64, c = e % 64;
            As[r][c] = (r0 + r < n && c < k) ? A[(size_t)(r0 + r) * k + c] : 0.0f;
        }
        for (int r = tid; r < MS_ROWS; r += 256) us[r] = (r0 + r < n) ? u[(size_t)(r0 + r) * S_BLK + j] : 0.0f;
        __syncthreads();
        for (int r = 0; r < MS_ROWS; ++r) {
            const float w = us[r];
            float x[4], y[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                x[q] = As[r][a0 + q] * w;
                y[q] = As[r][b0 + q];
            }
#pragma unroll
            for (int p = 0; p < 4; ++p)
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[p][q] = fmaf(x[p], y[q], acc[p][q]);
        }
        __syncthreads();
    }
    // this CTA's partial of M_j (added over the CTAs by part_sum_kernel)
    float* Mp = M + (size_t)blockIdx.x * S_BLK * k * k;
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (a0 + p < k && b0 + q < k) Mp[((size_t)j * k + a0 + p) * k + b0 + q] = acc[p][q];
}

// M = the stack of the FP32 form: per-CTA partials, then a fixed-order sum
constexpr int MSF_CTAS = 148;
void mstack_f32(const float* dA, const float* u32, int n, int k, float* Mpart, float* M, cudaStream_t s) {
    const int gx = std::min(MSF_CTAS, (n + MS_ROWS - 1) / MS_ROWS);
    mstack_f32_kernel<<<dim3(gx, S_BLK), 256, 0, s>>>(dA, u32, n, k, Mpart);
    const int cnt = S_BLK * k * k;
    part_sum_kernel<float><<<(unsigned)(((size_t)cnt * 32 + 255) / 256), 256, 0, s>>>(Mpart, gx, cnt, 1.0f, M);
}

// T2[i][j] = a_i^T M_j a_i for 4 consecutive j per CTA (M slices in shared memory)
__global__ void __launch_bounds__(256) quadform_f32_kernel(const float* __restrict__ A, const float* __restrict__ M,
                                                           int n, int k, float* __restrict__ T2) {
    extern __shared__ float Ms[];  // 4 * k * k
    const int j0 = blockIdx.y * 4;
    for (int e = threadIdx.x; e < 4 * k * k; e += blockDim.x) Ms[e] = M[(size_t)j0 * k * k + e];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float a[64];
#pragma unroll
    for (int q = 0; q < 64; ++q) a[q] = q < k ? A[(size_t)i * k + q] : 0.0f;
    for (int jj = 0; jj < 4; ++jj) {
        const float* Mj = Ms + jj * k * k;
        float t = 0.0f;
#pragma unroll 4
        for (int r = 0; r < k; ++r) {
            float v = 0.0f;
#pragma unroll
            for (int q = 0; q < 64; ++q)
                if (q < k) v = fmaf(Mj[r * k + q], a[q], v);
            t = fmaf(a[r], v, t);
        }
        T2[(size_t)i * S_BLK + j0 + jj] = t;
    }
}

// The same quadratic forms for k = 32 or 64 known at compile time: a_i stays in
// registers (fully unrolled loops, no dynamic indexing) and every M row is
// read from shared memory as float4 broadcasts.
template <int K>
__global__ void __launch_bounds__(256) quadform_f32k_kernel(const float* __restrict__ A, const float* __restrict__ M,
                                                            int n, float* __restrict__ T2) {
    extern __shared__ float Ms[];  // 4 * K * K
    const int j0 = blockIdx.y * 4;
    for (int e = threadIdx.x; e < 4 * K * K; e += blockDim.x) Ms[e] = M[(size_t)j0 * K * K + e];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float a[K];
    const float4* ar = reinterpret_cast<const float4*>(A + (size_t)i * K);
#pragma unroll
    for (int q = 0; q < K / 4; ++q) {
        const float4 v = __ldg(ar + q);
        a[4 * q] = v.x;
        a[4 * q + 1] = v.y;
        a[4 * q + 2] = v.z;
        a[4 * q + 3] = v.w;
    }
#pragma unroll 1
    for (int jj = 0; jj < 4; ++jj) {
        const float4* Mj = reinterpret_cast<const float4*>(Ms + jj * K * K);
        float t = 0.0f;
#pragma unroll
        for (int r = 0; r < K; ++r) {
            float v = 0.0f;
#pragma unroll
            for (int q = 0; q < K / 4; ++q) {
                const float4 m = Mj[r * (K / 4) + q];
                v = fmaf(m.x, a[4 * q], v);
                v = fmaf(m.y, a[4 * q + 1], v);
                v = fmaf(m.z, a[4 * q + 2], v);
                v = fmaf(m.w, a[4 * q + 3], v);
            }
            t = fmaf(a[r], v, t);
        }
        T2[(size_t)i * S_BLK + j0 + jj] = t;
    }
}

// T2 for any k <= 64 (the compile-time forms for 32 and 64)
void quadform_f32(const float* dA, const float* M, int n, int k, float* T2, cudaStream_t s) {
    const size_t qsm = 4 * (size_t)k * k * sizeof(float);
    const dim3 grid((n + 255) / 256, S_BLK / 4);
    if (k == 64) {
        cudaFuncSetAttribute(quadform_f32k_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)qsm);
        quadform_f32k_kernel<64><<<grid, 256, qsm, s>>>(dA, M, n, T2);
    } else if (k == 32) {
        quadform_f32k_kernel<32><<<grid, 256, qsm, s>>>(dA, M, n, T2);
    } else {
        cudaFuncSetAttribute(quadform_f32_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)qsm);
        quadform_f32_kernel<<<grid, 256, qsm, s>>>(dA, M, n, k, T2);
    }
}

// W = T1 - T2/2 + c.u/2 with T1 = A (A^T u) (FP64 accumulation), before centring
__global__ void __launch_bounds__(256) factor_combine_kernel(const float* __restrict__ A,
                                                             const double* __restrict__ AtU,
                                                             const float* __restrict__ T2,
                                                             const double* __restrict__ u, int n, int k,
                                                             double* __restrict__ W) {
    // one thread per row: the row of A is read once for all 16 columns and
    // for |a_i|^2; A^T u sits in shared memory
    __shared__ __align__(16) double s_atu[64 * S_BLK];
    for (int e = threadIdx.x; e < k * S_BLK; e += blockDim.x) s_atu[e] = AtU[e];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double t1[S_BLK];
#pragma unroll
    for (int j = 0; j < S_BLK; ++j) t1[j] = 0.0;
    double nrm = 0.0;
    const float* arow = A + (size_t)i * k;
    auto step = [&](double x, int a) {
        nrm += x * x;
        const double2* ar = reinterpret_cast<const double2*>(s_atu + a * S_BLK);
#pragma unroll
        for (int j = 0; j < S_BLK / 2; ++j) {
            const double2 v = ar[j];
            t1[2 * j] += x * v.x;
            t1[2 * j + 1] += x * v.y;
        }
    };
    if ((k & 3) == 0) {
        // the row as 16-byte loads, four in flight
        for (int a = 0; a < k; a += 16) {
            float4 q[4];
#pragma unroll
            for (int h = 0; h < 4; ++h)
                q[h] = a + 4 * h < k ? __ldg(reinterpret_cast<const float4*>(arow + a) + h) : make_float4(0, 0, 0, 0);
#pragma unroll
            for (int h = 0; h < 4; ++h)
                if (a + 4 * h < k) {
                    step(q[h].x, a + 4 * h);
                    step(q[h].y, a + 4 * h + 1);
                    step(q[h].z, a + 4 * h + 2);
                    step(q[h].w, a + 4 * h + 3);
                }
        }
    } else {
        for (int a = 0; a < k; ++a) step(A[(size_t)i * k + a], a);
    }
    const double cc = (1.0 - nrm) * (1.0 - nrm);
    const size_t o = (size_t)i * S_BLK;
#pragma unroll
    for (int j = 0; j < S_BLK; ++j) W[o + j] = t1[j] - 0.5 * (double)T2[o + j] + 0.5 * cc * u[o + j];
}

__global__ void subtract_mean_kernel(double* __restrict__ W, const double* __restrict__ mean, int n) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)n * S_BLK) return;
    W[idx] -= mean[idx % S_BLK];
}

// o_i = 1 / sum_j P_ij^2 with P = I + A A^T off the diagonal plus the unit
// diagonal: sum_j P_ij^2 = 1 + (a_i^T (A^T A) a_i - |a_i|^4)  (exact algebra of
// the factor form; compute_outlier_scores, src/rf_random_forest.cpp:2489-2520,
// on the full matrix).
__global__ void outlier_raw_kernel(const float* __restrict__ A, const double* __restrict__ AtA, int n, int k,
                                   float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double q = 0.0, nrm = 0.0;
    for (int a = 0; a < k; ++a) {
        const double x = A[(size_t)i * k + a];
        nrm += x * x;
        double v = 0.0;
        for (int b = 0; b < k; ++b) v += AtA[a * k + b] * (double)A[(size_t)i * k + b];
        q += x * v;
    }
    const double ss = 1.0 + (q - nrm * nrm);
    out[i] = (float)(1.0 / ss);
}

// Partial A^T A over the rows blockIdx.x, blockIdx.x + gridDim.x, ... into
// part[blockIdx.x] (k x k), added by part_sum_kernel in a fixed order.
__global__ void ata_kernel(const float* __restrict__ A, int n, int k, double* __restrict__ part) {
    const int e = blockIdx.y * blockDim.x + threadIdx.x;  // output index
    if (e >= k * k) return;
    const int a = e / k, b = e % k;
    double s = 0.0;
    for (int i = blockIdx.x; i < n; i += gridDim.x) s += (double)A[(size_t)i * k + a] * (double)A[(size_t)i * k + b];
    part[(size_t)blockIdx.x * k * k + e] = s;
}

}  // namespace

rfx_status launch_factor_ops_tc(Ctx* c, const float* dA, int k, const uint8_t* Aq, const uint8_t* At,
                                const float* sA, const float* u32, float* M, float* T2);
rfx_status pack_factor_tc(Ctx* c, const float* dA, int k, uint8_t* Aq, uint8_t* At, float* sA);
size_t factor_tc_aq_bytes(int n, int k);
size_t factor_tc_at_bytes(int n, int k);

namespace {
void col_mean(const double* V, int n, double* part, double* mean, cudaStream_t s) {
    colsum_part_kernel<<<RED_CTAS, 256, 0, s>>>(V, n, part);
    part_sum_kernel<double><<<(S_BLK * 32 + 255) / 256, 256, 0, s>>>(part, RED_CTAS, S_BLK, 1.0 / (double)n, mean);
}
void at_u(const float* A, const double* u, int n, int k, double* part, double* AtU, cudaStream_t s) {
    atu_part_kernel<<<RED_CTAS, 256, 0, s>>>(A, u, n, k, part);
    part_sum_kernel<double><<<(k * S_BLK * 32 + 255) / 256, 256, 0, s>>>(part, RED_CTAS, k * S_BLK, 1.0, AtU);
}
}  // namespace

rfx_status launch_mds_factors(Ctx* c, const float* dA, int k, int ndim, int max_iter, double tol, double* d_coords,
                              double* evals, int* iters, int precision) {
    const int n = c->n;
    cudaStream_t s = c->stream;
    if (k < 1 || k > 64 || ndim < 1 || ndim > 8 || n < S_BLK) {
        set_error("compute_mds_from_factors: need rank <= 64, 1 <= k <= 8 and n >= 16");
        return RFX_ERR_UNSUPPORTED;
    }
    Scratch d(c);
    double* mean = d.get<double>(S_BLK);
    double* u = d.get<double>((size_t)n * S_BLK);
    float* u32 = d.get<float>((size_t)n * S_BLK);
    double* AtU = d.get<double>((size_t)k * S_BLK);
    float* M = d.get<float>((size_t)S_BLK * k * k);
    float* Mpart = d.get<float>((size_t)MSF_CTAS * S_BLK * k * k);
    float* T2 = d.get<float>((size_t)n * S_BLK);
    double* part = d.get<double>((size_t)RED_CTAS * k * S_BLK);
    if (!mean || !u || !u32 || !AtU || !M || !Mpart || !T2 || !part) {
        set_error("compute_mds_from_factors: device allocation failed");
        return RFX_ERR_OOM;
    }
    StageTimer stt(c, ST_MDS_FACTORS, 0);
    const size_t qsm = 4 * (size_t)k * k * sizeof(float);
    RFX_CUDA(cudaFuncSetAttribute(quadform_f32_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)qsm));
    bool tensor = false;
    uint8_t* Aq = nullptr;
    uint8_t* At = nullptr;
    float* sA = nullptr;  // FP8 column scales (precision 3)
    auto apply = [&](const double* V, double* W) -> rfx_status {
        const unsigned gr = (unsigned)(((size_t)n * S_BLK + 255) / 256);
        col_mean(V, n, part, mean, s);
        center_kernel<<<gr, 256, 0, s>>>(V, mean, n, u, u32);
        at_u(dA, u, n, k, part, AtU, s);
        if (tensor) {
            rfx_status st = launch_factor_ops_tc(c, dA, k, Aq, At, sA, u32, M, T2);
            if (st != RFX_OK) return st;
        } else {
            mstack_f32(dA, u32, n, k, Mpart, M, s);
            quadform_f32(dA, M, n, k, T2, s);
            c->launches += 2;
        }
        factor_combine_kernel<<<(n + 255) / 256, 256, 0, s>>>(dA, AtU, T2, u, n, k, W);
        col_mean(W, n, part, mean, s);
        subtract_mean_kernel<<<gr, 256, 0, s>>>(W, mean, n);
        c->launches += 9;
        RFX_CUDA(cudaGetLastError());
        return RFX_OK;
    };
    if (precision == 0 || (k != 32 && k != 64))
        return subspace_topk(c, n, ndim, apply, max_iter, d_coords, evals, 12345, tol, nullptr, nullptr, iters, true);
    // mixed: tensor-core iterations (BF16, or FP8 E4M3 for precision 3) to
    // their rounding floor, then one FP32 refinement step from that basis
    double* basis = d.get<double>((size_t)n * S_BLK);
    Aq = d.get<uint8_t>(factor_tc_aq_bytes(n, k));
    At = d.get<uint8_t>(factor_tc_at_bytes(n, k));
    if (precision == 3) sA = d.get<float>((size_t)k);
    if (!basis || !Aq || !At || (precision == 3 && !sA)) {
        set_error("compute_mds_from_factors: device allocation failed");
        return RFX_ERR_OOM;
    }
    // the factor's tensor-core operands, packed once for every product
    if (rfx_status pst = pack_factor_tc(c, dA, k, Aq, At, sA)) return pst;
    tensor = true;
    int it1 = 0, it2 = 0;
    rfx_status st =
        subspace_topk(c, n, ndim, apply, max_iter, d_coords, evals, 12345, 1e-7, nullptr, basis, &it1, true);
    if (st != RFX_OK) return st;
    // one FP32 step from that basis: an FP32 product and its Rayleigh-Ritz
    tensor = false;
    st = subspace_topk(c, n, ndim, apply, 1, d_coords, evals, 12345, tol, basis, nullptr, &it2, true);
    if (iters) *iters = it1 + it2;
    c->last_mds_tc_iters = it1;
    c->last_mds_f32_iters = it2;
    return st;
}

// One application W = B V of the factor-space MDS operator (n x 16 blocks, FP64).
rfx_status launch_factor_operator(Ctx* c, const float* dA, int k, const double* V, double* W, int precision) {
    const int n = c->n;
    cudaStream_t s = c->stream;
    if (k < 1 || k > 64) {
        set_error("factor operator: rank must be 1..64");
        return RFX_ERR_UNSUPPORTED;
    }
    if (precision && k != 32 && k != 64) {
        set_error("factor operator: the tensor-core form needs rank 32 or 64");
        return RFX_ERR_UNSUPPORTED;
    }
    Scratch d(c);
    double* mean = d.get<double>(S_BLK);
    double* u = d.get<double>((size_t)n * S_BLK);
    float* u32 = d.get<float>((size_t)n * S_BLK);
    double* AtU = d.get<double>((size_t)k * S_BLK);
    float* M = d.get<float>((size_t)S_BLK * k * k);
    float* Mpart = d.get<float>((size_t)MSF_CTAS * S_BLK * k * k);
    float* T2 = d.get<float>((size_t)n * S_BLK);
    double* part = d.get<double>((size_t)RED_CTAS * k * S_BLK);
    if (!mean || !u || !u32 || !AtU || !M || !Mpart || !T2 || !part) return RFX_ERR_OOM;
    const unsigned gr = (unsigned)(((size_t)n * S_BLK + 255) / 256);
    col_mean(V, n, part, mean, s);
    center_kernel<<<gr, 256, 0, s>>>(V, mean, n, u, u32);
    at_u(dA, u, n, k, part, AtU, s);
    rfx_status st = RFX_OK;
    if (precision) {
        uint8_t* Aq = d.get<uint8_t>(factor_tc_aq_bytes(n, k));
        uint8_t* At = d.get<uint8_t>(factor_tc_at_bytes(n, k));
        float* sA = precision == 3 ? d.get<float>((size_t)k) : nullptr;
        if (!Aq || !At || (precision == 3 && !sA)) return RFX_ERR_OOM;
        st = pack_factor_tc(c, dA, k, Aq, At, sA);
        if (st == RFX_OK) st = launch_factor_ops_tc(c, dA, k, Aq, At, sA, u32, M, T2);
    } else {
        const size_t qsm = 4 * (size_t)k * k * sizeof(float);
        RFX_CUDA(cudaFuncSetAttribute(quadform_f32_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)qsm));
        mstack_f32(dA, u32, n, k, Mpart, M, s);
        quadform_f32(dA, M, n, k, T2, s);
    }
    if (st != RFX_OK) return st;
    factor_combine_kernel<<<(n + 255) / 256, 256, 0, s>>>(dA, AtU, T2, u, n, k, W);
    col_mean(W, n, part, mean, s);
    subtract_mean_kernel<<<gr, 256, 0, s>>>(W, mean, n);
    RFX_CUDA(cudaGetLastError());
    RFX_CUDA(cudaStreamSynchronize(s));
    return RFX_OK;
}

rfx_status launch_outlier_scores(Ctx* c, const float* dA, int k, float* d_out) {
    const int n = c->n;
    cudaStream_t s = c->stream;
    Scratch d(c);
    double* AtA = d.get<double>((size_t)k * k);
    double* apart = d.get<double>((size_t)256 * k * k);
    if (!AtA || !apart) return RFX_ERR_OOM;
    ata_kernel<<<dim3(256, (k * k + 255) / 256), 256, 0, s>>>(dA, n, k, apart);
    part_sum_kernel<double><<<(k * k * 32 + 255) / 256, 256, 0, s>>>(apart, 256, k * k, 1.0, AtA);
    outlier_raw_kernel<<<(n + 255) / 256, 256, 0, s>>>(dA, AtA, n, k, d_out);
    c->launches += 3;
    RFX_CUDA(cudaGetLastError());
    RFX_CUDA(cudaStreamSynchronize(s));
    return RFX_OK;
}

rfx_status launch_mds3d_full(Ctx* c, const float* dP, double* d_coords, double* evals) {
    const int n = c->n;
    cudaStream_t s = c->stream;
    StageTimer stt(c, ST_MDS_FULL, 0);
    if (n < 2) {
        set_error("MDS requires at least 2 samples");
        return RFX_ERR_INVALID;
    }
    if (n < S_BLK) {
        set_error("rfx_mds3d_full: n must be at least 16");
        return RFX_ERR_UNSUPPORTED;
    }
    Scratch d(c);
    const int nt = (n + GT - 1) / GT;
    const int npad = nt * GT;
    double* B = d.get<double>((size_t)nt * nt * TILE_D);
    double* rowmean = d.get<double>(n);
    double* grand = d.get<double>(1);
    unsigned long long* mx = d.get<unsigned long long>(1);
    if (!B || !rowmean || !grand || !mx) {
        set_error("rfx_mds3d_full: device allocation of the n x n FP64 matrix failed");
        return RFX_ERR_OOM;
    }
    RFX_CUDA(cudaMemsetAsync(mx, 0, sizeof(unsigned long long), s));
    mds_max_kernel<<<1024, 256, 0, s>>>(dP, c->d_nout, n, mx);
    mds_rowsum_kernel<<<n, 256, 0, s>>>(dP, c->d_nout, n, mx, rowmean);
    mds_grand_kernel<<<1, 1024, 0, s>>>(rowmean, n, grand);
    mds_b_kernel<<<2048, 256, 0, s>>>(dP, c->d_nout, n, nt, mx, rowmean, grand, B);
    c->launches += 4;
    RFX_CUDA(cudaGetLastError());
    const int kchunk = ((n + BV_KSPLIT - 1) / BV_KSPLIT + GT - 1) / GT * GT;
    const int ksn = (n + kchunk - 1) / kchunk;
    double* Wpart = d.get<double>((size_t)ksn * n * S_BLK);
    double* Vf = d.get<double>((size_t)npad * S_BLK);
    if (!Wpart || !Vf) {
        set_error("rfx_mds3d_full: device allocation failed");
        return RFX_ERR_OOM;
    }
    RFX_CUDA(cudaFuncSetAttribute(dgemm_bv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)DB_SMEM));
    auto apply = [&](const double* V, double* W) -> rfx_status {
        bv_pack_kernel<<<(unsigned)(((size_t)npad * S_BLK + 255) / 256), 256, 0, s>>>(V, n, npad, Vf);
        dgemm_bv_kernel<<<dim3(nt, ksn), 128, DB_SMEM, s>>>(B, nt, Vf, n, kchunk, Wpart, c->d_err);
        bv_reduce_kernel<<<(unsigned)(((size_t)n * S_BLK + 255) / 256), 256, 0, s>>>(Wpart, n, ksn, W);
        c->launches += 3;
        RFX_CUDA(cudaGetLastError());
        return RFX_OK;
    };
    // Chebyshev degree 8; up to 4000 products (the eigenvalue-change
    // criterion of 1e-14 ends it far earlier unless the third eigenvalue sits
    // in a tight cluster)
    return subspace_topk(c, n, 3, apply, 4000, d_coords, evals, 12345, 1e-14, nullptr, nullptr, nullptr, false, 8);
}

}  // namespace rfx
