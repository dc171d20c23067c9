// Small dense FP64 linear algebra run inside one CTA (matrices of at most
// 128 x 128 held in shared memory): Cholesky, inverse of a lower triangle and
// a cyclic Jacobi eigensolver.  Used for the s x s Gram / Rayleigh-Ritz
// problems of the MDS and low-rank paths.
#pragma once
#include <cuda_runtime.h>

namespace rfx {

// In-place Cholesky of the s x s SPD matrix G (row-major, leading dim ld):
// G = L L^T, L written to the lower triangle, upper triangle zeroed.
// Returns false (in every thread) if a pivot is not positive.
__device__ inline bool cta_cholesky(double* G, int s, int ld, double* flag) {
    const int tid = threadIdx.x, nt = blockDim.x;
    if (tid == 0) *flag = 1.0;
    __syncthreads();
    for (int j = 0; j < s; ++j) {
        if (tid == 0) {
            double d = G[j * ld + j];
            for (int k = 0; k < j; ++k) d -= G[j * ld + k] * G[j * ld + k];
            if (!(d > 0.0)) {
                *flag = 0.0;
                d = 1.0;
            }
            G[j * ld + j] = sqrt(d);
        }
        __syncthreads();
        const double djj = G[j * ld + j];
        for (int i = j + 1 + tid; i < s; i += nt) {
            double v = G[i * ld + j];
            for (int k = 0; k < j; ++k) v -= G[i * ld + k] * G[j * ld + k];
            G[i * ld + j] = v / djj;
        }
        __syncthreads();
    }
    for (int e = tid; e < s * s; e += nt) {
        const int i = e / s, j = e % s;
        if (j > i) G[i * ld + j] = 0.0;
    }
    __syncthreads();
    return *flag > 0.5;
}

// Inverse of the lower-triangular L (s x s) into Linv (lower), one column per thread.
__device__ inline void cta_tri_inverse(const double* L, double* Linv, int s, int ld) {
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int c = tid; c < s; c += nt) {
        for (int r = 0; r < s; ++r) {
            double v = (r == c) ? 1.0 : 0.0;
            for (int k = c; k < r; ++k) v -= L[r * ld + k] * Linv[k * ld + c];
            Linv[r * ld + c] = (r >= c) ? v / L[r * ld + r] : 0.0;
        }
    }
    __syncthreads();
}

// Cyclic Jacobi eigendecomposition of the symmetric s x s matrix A (destroyed):
// eigenvalues on the diagonal of A, eigenvectors in the columns of V.
// Rotations of disjoint index pairs are applied in parallel (round-robin
// ordering); at most `sweeps` full sweeps, fewer once every off-diagonal entry
// is at FP64 rounding relative to its diagonal pair, or (abs_tol > 0) below
// abs_tol times the largest diagonal magnitude: the absolute stop ends a
// spectrum with eigenvalues near zero, whose relative test rounding keeps
// open, and leaves the large eigenpairs accurate to abs_tol.  A leading
// dimension ld = s + 1 keeps the column passes free of shared-memory bank
// conflicts.
__device__ inline void cta_jacobi(double* A, double* V, int s, int ld, int sweeps, int* pairs, double abs_tol = 0.0) {
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int e = tid; e < s * s; e += nt) V[(e / s) * ld + (e % s)] = ((e / s) == (e % s)) ? 1.0 : 0.0;
    __syncthreads();
    const int m = (s % 2) ? s + 1 : s;  // round-robin needs an even count (index s = dummy)
    __shared__ double cs[64][2];
    for (int sw = 0; sw < sweeps; ++sw) {
        // converged when every off-diagonal entry is negligible against its
        // diagonal pair, |a_pq| <= 1e-16 sqrt(|a_pp a_qq|) (the relative
        // criterion, which keeps small eigenvalues accurate)
        double floor2 = 0.0;
        if (abs_tol > 0.0) {
            double dmax = 0.0;
            for (int r = 0; r < s; ++r) dmax = fmax(dmax, fabs(A[r * ld + r]));
            floor2 = (abs_tol * dmax) * (abs_tol * dmax);
        }
        int active = 0;
        for (int e = tid; e < s * s; e += nt) {
            const int r = e / s, q = e % s;
            if (r < q) {
                const double v = A[r * ld + q];
                if (v * v > 1e-32 * fabs(A[r * ld + r] * A[q * ld + q]) && v * v > floor2) active = 1;
            }
        }
        if (!__syncthreads_or(active)) break;
        for (int round = 0; round < m - 1; ++round) {
            // round-robin tournament: index 0 stays, indices 1..m-1 rotate;
            // pair k joins positions k and m-1-k
            // (the thread that numbers pair k also computes its rotation; the
            // barrier below publishes both)
            int rot = 0;
            for (int k = tid; k < m / 2; k += nt) {
                const int pa = k, pb = m - 1 - k;
                const int a = (pa == 0) ? 0 : ((pa - 1 + round) % (m - 1)) + 1;
                const int b = ((pb - 1 + round) % (m - 1)) + 1;
                const int p = min(a, b), q = max(a, b);
                pairs[2 * k] = p;
                pairs[2 * k + 1] = q;
                double c = 1.0, sn = 0.0;
                if (q < s && p != q) {
                    const double apq = A[p * ld + q];
                    // entries already below the stop test are not rotated
                    if (fabs(apq) > 1e-300 && apq * apq > 1e-32 * fabs(A[p * ld + p] * A[q * ld + q]) &&
                        apq * apq > floor2) {
                        rot = 1;
                        const double app = A[p * ld + p], aqq = A[q * ld + q];
                        const double tau = (aqq - app) / (2.0 * apq);
                        const double t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                        c = 1.0 / sqrt(1.0 + t * t);
                        sn = t * c;
                    }
                }
                cs[k][0] = c;
                cs[k][1] = sn;
            }
            // a round without a rotation leaves A and V as they are
            if (!__syncthreads_or(rot)) continue;
            // A <- J^T A J applied as rows then columns; V <- V J goes with the
            // row pass, so both passes move two pairs of entries per element
            for (int e = tid; e < (m / 2) * s; e += nt) {
                const int k = e / s, r = e % s;
                const int p = pairs[2 * k], q = pairs[2 * k + 1];
                if (q >= s) continue;
                const double c = cs[k][0], sn = cs[k][1];
                const double ap = A[p * ld + r], aq = A[q * ld + r];
                A[p * ld + r] = c * ap - sn * aq;
                A[q * ld + r] = sn * ap + c * aq;
                const double vp = V[r * ld + p], vq = V[r * ld + q];
                V[r * ld + p] = c * vp - sn * vq;
                V[r * ld + q] = sn * vp + c * vq;
            }
            __syncthreads();
            for (int e = tid; e < (m / 2) * s; e += nt) {
                const int k = e / s, r = e % s;
                const int p = pairs[2 * k], q = pairs[2 * k + 1];
                if (q >= s) continue;
                const double c = cs[k][0], sn = cs[k][1];
                const double ap = A[r * ld + p], aq = A[r * ld + q];
                A[r * ld + p] = c * ap - sn * aq;
                A[r * ld + q] = sn * ap + c * aq;
            }
            __syncthreads();
        }
    }
}

}  // namespace rfx
