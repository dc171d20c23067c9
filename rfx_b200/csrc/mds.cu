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
// dsyevd; eigenvectors are defined up to sign.
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

__global__ void mds_b_kernel(const float* __restrict__ P, const int32_t* __restrict__ nout, int n,
                             const unsigned long long* __restrict__ maxbits, const double* __restrict__ rowmean,
                             const double* __restrict__ grand, double* __restrict__ B) {
    const double mx = __longlong_as_double((long long)*maxbits);
    const double g = *grand;
    const size_t total = (size_t)n * n;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(e / n), j = (int)(e % n);
        const double d = (i == j) ? 0.0 : __dsub_rn(mx, q_value(P, nout, n, i, j));
        const double v = __dadd_rn(__dsub_rn(__dsub_rn(__dmul_rn(d, d), rowmean[i]), rowmean[j]), g);
        B[e] = __dmul_rn(-0.5, v);
    }
}

// W[n x S] = B[n x n] V[n x S], FP64, 64-row tiles.
constexpr int GT = 64;
__global__ void __launch_bounds__(256) dgemm_bv_kernel(const double* __restrict__ B, const double* __restrict__ V,
                                                       int n, double* __restrict__ W) {
    __shared__ double Bs[GT][GT + 1];
    __shared__ double Vs[GT][S_BLK];
    const int r0 = blockIdx.x * GT;
    const int tid = threadIdx.x;
    // thread owns rows (tid / 4) and columns (tid % 4) * 4 .. +3
    const int rr = tid >> 2, cc = (tid & 3) * 4;
    double acc[4] = {0, 0, 0, 0};
    for (int k0 = 0; k0 < n; k0 += GT) {
        for (int e = tid; e < GT * GT; e += 256) {
            const int r = e / GT, k = e % GT;
            Bs[r][k] = (r0 + r < n && k0 + k < n) ? B[(size_t)(r0 + r) * n + k0 + k] : 0.0;
        }
        for (int e = tid; e < GT * S_BLK; e += 256) {
            const int k = e / S_BLK, c = e % S_BLK;
            Vs[k][c] = (k0 + k < n) ? V[(size_t)(k0 + k) * S_BLK + c] : 0.0;
        }
        __syncthreads();
#pragma unroll 8
        for (int k = 0; k < GT; ++k) {
            const double b = Bs[rr][k];
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[q] = fma(b, Vs[k][cc + q], acc[q]);
        }
        __syncthreads();
    }
    if (r0 + rr < n)
#pragma unroll
        for (int q = 0; q < 4; ++q) W[(size_t)(r0 + rr) * S_BLK + cc + q] = acc[q];
}

// G[S x S] += X^T Y over rows (atomics into a zeroed G).
__global__ void __launch_bounds__(256) dgram_kernel(const double* __restrict__ X, const double* __restrict__ Y, int n,
                                                    double* __restrict__ G) {
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
    atomicAdd(G + a * S_BLK + b, acc);
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
    __shared__ double A[S_BLK * S_BLK], U[S_BLK * S_BLK];
    __shared__ int pairs[2 * 64];
    for (int e = threadIdx.x; e < S_BLK * S_BLK; e += blockDim.x) {
        const int i = e / S_BLK, j = e % S_BLK;
        A[e] = 0.5 * (H[i * S_BLK + j] + H[j * S_BLK + i]);
    }
    __syncthreads();
    cta_jacobi(A, U, S_BLK, S_BLK, 12, pairs);
    for (int e = threadIdx.x; e < S_BLK * S_BLK; e += blockDim.x) evecs[e] = U[e];
    for (int i = threadIdx.x; i < S_BLK; i += blockDim.x) evals[i] = A[i * S_BLK + i];
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

struct Dev {
    std::vector<void*> ptrs;
    ~Dev() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <typename T>
    T* get(size_t count) {
        void* p = nullptr;
        if (cudaMalloc(&p, sizeof(T) * std::max<size_t>(count, 1)) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
};

}  // namespace

// Subspace iteration on the symmetric operator applied by `apply` (W = B V),
// returning the k largest eigenpairs above 1e-10: coordinates n x k in `out`
// (device) and eigenvalues in `evals_out` (host).  Shared by the full-matrix
// and the factor MDS.
template <typename Apply>
rfx_status subspace_topk(Ctx* c, int n, int k, Apply apply, int max_iter, double* d_out, double* evals_out,
                         uint64_t seed) {
    cudaStream_t s = c->stream;
    Dev d;
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
    // start block: seeded Gaussian (srand(12345 + 1000*eig) seeds the reference's
    // factor MDS; any start converges to the same subspace)
    {
        std::vector<double> h((size_t)n * S_BLK);
        std::mt19937_64 rng(seed);
        std::normal_distribution<double> nd(0.0, 1.0);
        for (auto& x : h) x = nd(rng);
        RFX_CUDA(cudaMemcpyAsync(V, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, s));
        RFX_CUDA(cudaStreamSynchronize(s));
    }
    RFX_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), s));
    double* Xt = d.get<double>((size_t)n * S_BLK);
    if (!Xt) {
        set_error("MDS: device allocation failed");
        return RFX_ERR_OOM;
    }
    // CholeskyQR2: Out = (src L1^{-T}) L2^{-T}, through the temporary Xt
    auto orth = [&](const double* src, double* Out) -> rfx_status {
        const unsigned gb = (unsigned)std::min(1024, (n + 63) / 64);
        const unsigned gr = (unsigned)(((size_t)n * S_BLK + 255) / 256);
        RFX_CUDA(cudaMemsetAsync(G, 0, sizeof(double) * S_BLK * S_BLK, s));
        dgram_kernel<<<gb, 256, 0, s>>>(src, src, n, G);
        chol_inv_kernel<<<1, 128, 0, s>>>(G, Tm, bad);
        dright_kernel<<<gr, 256, 0, s>>>(src, Tm, n, Xt);
        RFX_CUDA(cudaMemsetAsync(G, 0, sizeof(double) * S_BLK * S_BLK, s));
        dgram_kernel<<<gb, 256, 0, s>>>(Xt, Xt, n, G);
        chol_inv_kernel<<<1, 128, 0, s>>>(G, Tm, bad);
        dright_kernel<<<gr, 256, 0, s>>>(Xt, Tm, n, Out);
        c->launches += 6;
        RFX_CUDA(cudaGetLastError());
        return RFX_OK;
    };
    rfx_status st;
    if ((st = orth(V, V)) != RFX_OK) return st;  // src and Out may alias: Xt sits between
    std::vector<double> prev(S_BLK, 0.0), cur(S_BLK, 0.0);
    std::vector<double> hU(S_BLK * S_BLK);
    for (int it = 1; it <= max_iter; ++it) {
        if ((st = apply(V, W)) != RFX_OK) return st;
        const bool check = (it % 10 == 0) || it == max_iter;
        if (check) {
            // Rayleigh-Ritz on span(V): H = V^T (B V)
            RFX_CUDA(cudaMemsetAsync(G, 0, sizeof(double) * S_BLK * S_BLK, s));
            dgram_kernel<<<std::min(1024, (n + 63) / 64), 256, 0, s>>>(V, W, n, G);
            rr_kernel<<<1, 128, 0, s>>>(G, ev, U);
            c->launches += 2;
            RFX_CUDA(cudaMemcpyAsync(cur.data(), ev, sizeof(double) * S_BLK, cudaMemcpyDeviceToHost, s));
            RFX_CUDA(cudaStreamSynchronize(s));
            std::vector<double> a = cur, b = prev;
            std::sort(a.rbegin(), a.rend());
            std::sort(b.rbegin(), b.rend());
            double delta = 0.0;
            for (int q = 0; q < k; ++q) delta = std::max(delta, std::fabs(a[q] - b[q]) / std::max(std::fabs(a[q]), 1e-300));
            prev = cur;
            if (delta < 1e-14 || it == max_iter) break;
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
    c->launches += 1;
    RFX_CUDA(cudaGetLastError());
    RFX_CUDA(cudaStreamSynchronize(s));
    return RFX_OK;
}

rfx_status launch_mds3d_full(Ctx* c, const float* dP, double* d_coords, double* evals) {
    const int n = c->n;
    cudaStream_t s = c->stream;
    if (n < 2) {
        set_error("MDS requires at least 2 samples");
        return RFX_ERR_INVALID;
    }
    if (n < S_BLK) {
        set_error("rfx_mds3d_full: n must be at least 16");
        return RFX_ERR_UNSUPPORTED;
    }
    Dev d;
    double* B = d.get<double>((size_t)n * n);
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
    mds_b_kernel<<<2048, 256, 0, s>>>(dP, c->d_nout, n, mx, rowmean, grand, B);
    c->launches += 4;
    RFX_CUDA(cudaGetLastError());
    auto apply = [&](const double* V, double* W) -> rfx_status {
        dgemm_bv_kernel<<<(n + GT - 1) / GT, 256, 0, s>>>(B, V, n, W);
        c->launches += 1;
        RFX_CUDA(cudaGetLastError());
        return RFX_OK;
    };
    return subspace_topk(c, n, 3, apply, 600, d_coords, evals, 12345);
}

}  // namespace rfx
