// Case-wise weighting and RF-GAP proximity.
//
// Case-wise (use_casewise, the reference's bootstrap-frequency weighting):
//   tnodewt   per terminal node, the mean bootstrap multiplicity of the
//             in-bag samples that reach it, walked with the rule of
//             grow_tree_single's tnodewt block (src/rf_random_forest.cpp:
//             1049-1102); float(sum) / float(count), 0 for other nodes.
//   votes     q[i][jtr] += tnodewt[nodextr] per OOB tree, in tree order
//             (:1107-1153) — one thread per sample, trees in order.
//   pair sums C[i][j] += nin[j] / nodesize for OOB i and in-bag j of a leaf,
//             nodesize = the leaf's in-bag multiplicities summed, FP64
//             (src/rf_proximity.cpp:195-222); S = C + C^T is written as the
//             packed upper triangle.
//   importance (src/rf_varimp.cpp:138-148, 203-236): right, rightimp, qimp
//             and qimpm weighted by tnodewt of the node the (permuted) walk
//             reaches.
// RF-GAP (src/rf_proximity.cpp:238-391): pGAP(i,j) = (1/|S_i|) sum over the
//   trees where i is OOB of c_j / |M_i| for the in-bag samples j of i's node,
//   then P = (pGAP + pGAP^T) / 2; nodes are the per-tree node ids the
//   reference keeps (OOB: testreebag, in-bag: find_terminal_node), so any node
//   id matches, the root included.
//
// Every float and double sum runs in the reference's order, so the results
// are bit-identical to it: the pair-sum rows add tree after tree (a CTA
// barrier between trees orders the adds into a column slot; within one tree a
// row meets each column at most once), votes and qimp/qimpm loop over trees
// in order per sample, rightimp loops over a tree's OOB samples in order.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "walks.cuh"

namespace rfx {
namespace {

constexpr int WR_THREADS = 128;
constexpr int WR_WINDOW = 4096;  // columns per CTA: two FP64 accumulators each (64 KB)

__device__ __forceinline__ int lower_bound_memb(const int32_t* __restrict__ a, int lo, int hi, int v) {
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(a + mid) < v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// tnodewt: one thread per (sample, tree) of the in-bag samples; integer sums
// (exact, so the order of the float sums of the reference does not matter).
__global__ void tnodewt_walk_kernel(const float* __restrict__ X, int n, int p, const DNode* __restrict__ nodes,
                                    const int64_t* __restrict__ offs, const int32_t* __restrict__ nnode,
                                    const int32_t* __restrict__ catgoleft, int maxcat, const int32_t* __restrict__ nin,
                                    int32_t* __restrict__ wsum, int32_t* __restrict__ wcnt) {
    const int t = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = nin[(size_t)t * n + i];
    if (c <= 0) return;
    const int64_t o = offs[t];
    const int nn = nnode[t];
    const DNode* tn = nodes + o;
    const int32_t* cgl = catgoleft ? catgoleft + o * maxcat : nullptr;
    const float* xr = X + (size_t)i * p;
    int cur = 0;
    for (int guard = 0; guard < nn + 1; ++guard) {  // a grown tree reaches a leaf within nnode steps
        const DNode nd = load_node(tn, cur);
        if (node_status(nd.meta) != 1) break;
        const int m = node_var(nd.meta);
        const float x = __ldg(xr + m);
        bool left;
        if (node_cat(nd.meta)) {
            const int idx = __float2int_rz(__fadd_rn(x, 0.5f));
            left = idx >= 0 && idx < maxcat && cgl_at(cgl, maxcat, cur, idx) == 1;
        } else {
            left = x <= nd.split;
        }
        cur = left ? nd.left : nd.right;
        if (cur < 0 || cur >= nn) break;
    }
    if (cur >= 0 && cur < nn && node_status(load_node(tn, cur).meta) == -1) {
        atomicAdd(wsum + o + cur, c);
        atomicAdd(wcnt + o + cur, 1);
    }
}

__global__ void tnodewt_final_kernel(int64_t N, const int32_t* __restrict__ wsum, const int32_t* __restrict__ wcnt,
                                     float* __restrict__ tnodewt) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= N) return;
    const int k = wcnt[g];
    tnodewt[g] = k > 0 ? __fdiv_rn((float)wsum[g], (float)k) : 0.0f;
}

// weight of an OOB vote that ends on node nd of a tree with nn nodes
__device__ __forceinline__ float vote_w(const float* __restrict__ tw, int nd, int nn) {
    return (nd >= 0 && nd < nn) ? __ldg(tw + nd) : 1.0f;
}

// Case-wise OOB votes: one thread per sample, trees in order; the class of an
// OOB walk is the class of the node testreebag ends on (the root on its
// fallback path, whose node id is 0).
__global__ void casewise_votes_kernel(const int32_t* __restrict__ leafnode, const uint8_t* __restrict__ inbag,
                                      const int64_t* __restrict__ offs, const int32_t* __restrict__ nnode,
                                      const int32_t* __restrict__ nodeclass, const float* __restrict__ tnodewt,
                                      int n, int T, int nclass, float* __restrict__ q) {
    extern __shared__ float qs[];  // blockDim.x * nclass
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float* my = qs + (size_t)threadIdx.x * nclass;
    for (int c = 0; c < nclass; ++c) my[c] = 0.0f;
    if (i >= n) return;
    for (int t = 0; t < T; ++t) {
        const size_t ti = (size_t)t * n + i;
        if (inbag[ti]) continue;
        const int nd = leafnode[ti];
        const int64_t o = offs[t];
        const int nn = nnode[t];
        const int cls = __ldg(nodeclass + o + nd);
        if (cls >= 0 && cls < nclass) my[cls] = __fadd_rn(my[cls], vote_w(tnodewt + o, nd, nn));
    }
    for (int c = 0; c < nclass; ++c) q[(size_t)i * nclass + c] = my[c];
}

// Sum of the bootstrap multiplicities of every key's members (per tree, per
// key of the leaf lists).
__global__ void key_mass_kernel(const int64_t* __restrict__ segbase, const int32_t* __restrict__ segoff,
                                const int32_t* __restrict__ memb, const int32_t* __restrict__ nin, int n,
                                long long* __restrict__ mass) {
    const int t = blockIdx.x;
    const int64_t sb = segbase[t];
    const int K = (int)(segbase[t + 1] - sb) - 1;
    const int32_t* so = segoff + sb;
    const int32_t* mt = memb + (size_t)t * n;
    const int32_t* nt = nin + (size_t)t * n;
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
        long long s = 0;
        for (int q = so[k]; q < so[k + 1]; ++q) s += nt[mt[q]];
        mass[sb + k] = s;
    }
}

enum { WR_CASEWISE = 0, WR_RFGAP = 1, WR_PLAIN = 2 };

// One CTA per (row i, window of WR_WINDOW columns); trees in order.  For every
// tree, the row's key k (2 * node + in-bag) gives the opposite key's members,
// cut to the window's columns > i.
//   i OOB (k even):   accA[j] += w(j) for the in-bag members j
//   i in-bag (k odd): accB[j] += w(i) for the OOB members j
// casewise: w(s) = nin[s] / nodesize (nodesize = mass of the in-bag key);
//           S[i][j] = accA[j] + accB[j].
// plain:    w = 1 (the reference's weights without use_casewise), as FP64.
// rfgap:    w(s) = nin[s] * (1 / M), M = mass of the in-bag key;
//           P[i][j] = (accA[j] / |S_i| + accB[j] / |S_j|) / 2, with the
//           reference's multiplication by 1 / |S|.
template <int MODE>
__global__ void __launch_bounds__(WR_THREADS)
weighted_row_kernel(const int32_t* __restrict__ key, const int64_t* __restrict__ segbase,
                    const int32_t* __restrict__ segoff, const int32_t* __restrict__ memb,
                    const long long* __restrict__ mass, const int32_t* __restrict__ nin,
                    const int32_t* __restrict__ nout, int n, int T, double* __restrict__ out) {
    extern __shared__ double wr_acc[];  // accA | accB, WR_WINDOW each
    double* accA = wr_acc;
    double* accB = wr_acc + WR_WINDOW;
    const int i = blockIdx.x;
    const int c0 = blockIdx.y * WR_WINDOW;
    const int c1 = min(n, c0 + WR_WINDOW);
    if (c1 <= i) return;  // every column of the window lies left of the diagonal
    const int lo = max(c0, i + 1);
    const int tid = threadIdx.x;
    for (int k = tid; k < WR_WINDOW; k += WR_THREADS) {
        accA[k] = 0.0;
        accB[k] = 0.0;
    }
    __syncthreads();
    for (int t = 0; t < T; ++t) {
        const int k = __ldg(key + (size_t)t * n + i);
        if (k >= 0 && lo < c1) {
            const int64_t sb = segbase[t];
            const int32_t* so = segoff + sb;
            const int32_t* mt = memb + (size_t)t * n;
            const int ok = k ^ 1;
            int b = __ldg(so + ok), e = __ldg(so + ok + 1);
            if (b < e) {
                b = lower_bound_memb(mt, b, e, lo);
                e = lower_bound_memb(mt, b, e, c1);
            }
            const int32_t* nt = nin + (size_t)t * n;
            if ((k & 1) == 0) {
                const long long m = mass[sb + ok];
                if (m > 0 || MODE == WR_PLAIN) {
                    const double inv = MODE == WR_RFGAP ? __ddiv_rn(1.0, (double)m) : 0.0;
                    for (int q = b + tid; q < e; q += WR_THREADS) {
                        const int j = __ldg(mt + q);
                        const double c = (double)__ldg(nt + j);
                        const double w = MODE == WR_PLAIN   ? 1.0
                                         : MODE == WR_RFGAP ? __dmul_rn(c, inv)
                                                            : __ddiv_rn(c, (double)m);
                        accA[j - c0] = __dadd_rn(accA[j - c0], w);
                    }
                }
            } else {
                const long long m = mass[sb + k];
                if (m > 0 || MODE == WR_PLAIN) {
                    const double c = (double)__ldg(nt + i);
                    const double w = MODE == WR_PLAIN   ? 1.0
                                     : MODE == WR_RFGAP ? __dmul_rn(c, __ddiv_rn(1.0, (double)m))
                                                        : __ddiv_rn(c, (double)m);
                    for (int q = b + tid; q < e; q += WR_THREADS) {
                        const int j = __ldg(mt + q);
                        accB[j - c0] = __dadd_rn(accB[j - c0], w);
                    }
                }
            }
        }
        __syncthreads();  // this tree's adds land before the next tree's
    }
    const int64_t rowoff = (int64_t)i * n - ((int64_t)i * (i - 1)) / 2 - i;  // + j gives [i][j]
    const int sI = nout[i] / 2;  // trees where i is OOB
    const double invI = sI > 0 ? __ddiv_rn(1.0, (double)sI) : 0.0;
    for (int j = max(c0, i) + tid; j < c1; j += WR_THREADS) {
        double v;
        if (j == i) {
            v = MODE == WR_RFGAP ? (sI == 0 ? 1.0 : 0.0) : 0.0;
        } else if (MODE == WR_RFGAP) {
            const int sJ = nout[j] / 2;
            const double a = sI > 0 ? __dmul_rn(accA[j - c0], invI) : accA[j - c0];
            const double bj = sJ > 0 ? __dmul_rn(accB[j - c0], __ddiv_rn(1.0, (double)sJ)) : accB[j - c0];
            v = __ddiv_rn(__dadd_rn(a, bj), 2.0);
        } else {
            v = __dadd_rn(accA[j - c0], accB[j - c0]);
        }
        out[rowoff + j] = v;
    }
}

// RF-GAP keys: 2 * node + in-bag from the per-tree node ids.
__global__ void gap_key_kernel(const int32_t* __restrict__ leafnode, const uint8_t* __restrict__ inbag, int64_t cells,
                               int32_t* __restrict__ key) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= cells) return;
    const int nd = leafnode[e];
    key[e] = nd >= 0 ? 2 * nd + (inbag[e] ? 1 : 0) : -1;
}

// ---------------------------------------------------------------------------
// Case-wise importance
// ---------------------------------------------------------------------------

// cpu_testreeimp's walk (src/rf_varimp.cpp:45-103) with feature mr taken
// from xperm: returns the node reached and sets *cls, or -1 when the
// reference breaks without assigning.
__device__ __forceinline__ int imp_walk(const float* __restrict__ xr, const float* __restrict__ xp, int mr, int p,
                                        const DNode* __restrict__ tn, const int32_t* __restrict__ tc, int nnv,
                                        const int32_t* __restrict__ cgl, int maxcat, int* cls) {
    int kt = 0;
    for (int s = 0; s < nnv; ++s) {
        const DNode nd = load_node(tn, kt);
        if (node_status(nd.meta) == -1) {
            *cls = __ldg(tc + kt);
            return kt;
        }
        const int m = node_var(nd.meta);
        if (m >= p) return -1;
        const float x = __ldg((m == mr ? xp : xr) + m);
        if (!node_cat(nd.meta)) {
            kt = (x <= nd.split) ? nd.left : nd.right;
        } else {
            const int jcat = __float2int_rz(__fadd_rn(x, 0.5f));
            if (jcat < 0 || jcat >= maxcat) return -1;
            kt = (cgl_at(cgl, maxcat, kt, jcat) == 1) ? nd.left : nd.right;
        }
    }
    return -1;
}

// One thread per (tree, feature): the tree's weighted right count (from the
// testreebag nodes), and for a feature split on in the tree the weighted
// permuted right count, both summed over the OOB samples in order; writes
// rr = (right - rightimp) / noob (0 for a feature the tree does not use).
__global__ void cw_tree_kernel(const float* __restrict__ X, const int32_t* __restrict__ y, int n, int p, int T,
                               const DNode* __restrict__ nodes, const int32_t* __restrict__ nodeclass,
                               const int64_t* __restrict__ offs, const int32_t* __restrict__ nnode,
                               const int32_t* __restrict__ catgoleft, int maxcat, const uint64_t* __restrict__ iv,
                               int ivw, const int32_t* __restrict__ joob, const int32_t* __restrict__ noob_arr,
                               const int32_t* __restrict__ partner, const int32_t* __restrict__ leafnode,
                               const float* __restrict__ tnodewt, float* __restrict__ rr, uint32_t* __restrict__ err) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)T * p) return;
    const int t = (int)(idx / p), k = (int)(idx % p);
    const int64_t o = offs[t];
    const int nn = nnode[t];
    const int nnv = nn > 0 ? nn : 1;
    const DNode* tn = nodes + o;
    const int32_t* tc = nodeclass + o;
    const float* tw = tnodewt + o;
    const int32_t* cgl = catgoleft ? catgoleft + o * maxcat : nullptr;
    const int noob = noob_arr[t];
    const int32_t* jo = joob + (size_t)t * n;
    const bool used = (__ldg(iv + (size_t)t * ivw + (k >> 6)) >> (k & 63)) & 1ull;
    if (!used) {
        rr[idx] = 0.0f;
        return;
    }
    float right = 0.0f, rightimp = 0.0f;
    for (int r = 0; r < noob; ++r) {
        const int i = __ldg(jo + r);
        const int nd = __ldg(leafnode + (size_t)t * n + i);
        if (__ldg(tc + nd) == __ldg(y + i)) right = __fadd_rn(right, vote_w(tw, nd, nn));
        int cls = -1;
        const int ip = __ldg(partner + (size_t)t * n + i);
        const int pn = imp_walk(X + (size_t)i * p, X + (size_t)ip * p, k, p, tn, tc, nnv, cgl, maxcat, &cls);
        if (pn < 0) {
            atomicOr(err, ERR_STALE_JVR);
            continue;
        }
        if (cls == __ldg(y + i)) rightimp = __fadd_rn(rightimp, vote_w(tw, pn, nn));
    }
    rr[idx] = __fdiv_rn(__fsub_rn(right, rightimp), (float)noob);
}

// One thread per (sample, feature): qimpm[i][k] = sum over the trees where i
// is OOB, in tree order, of w / noob for a correct vote (the permuted walk's
// node for a feature the tree splits on, the testreebag node otherwise);
// feature 0's thread also sums qimp[i] (the unpermuted votes).
__global__ void cw_sample_kernel(const float* __restrict__ X, const int32_t* __restrict__ y, int n, int p, int T,
                                 const DNode* __restrict__ nodes, const int32_t* __restrict__ nodeclass,
                                 const int64_t* __restrict__ offs, const int32_t* __restrict__ nnode,
                                 const int32_t* __restrict__ catgoleft, int maxcat, const uint64_t* __restrict__ iv,
                                 int ivw, const uint8_t* __restrict__ inbag, const int32_t* __restrict__ partner,
                                 const int32_t* __restrict__ leafnode, const float* __restrict__ tnodewt,
                                 const int32_t* __restrict__ noob_arr, int impn, float* __restrict__ qimp,
                                 float* __restrict__ qimpm, uint32_t* __restrict__ err) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)n * p) return;
    const int i = (int)(idx / p), k = (int)(idx % p);
    const int yi = __ldg(y + i);
    float acc = 0.0f, accq = 0.0f;
    for (int t = 0; t < T; ++t) {
        const size_t ti = (size_t)t * n + i;
        if (inbag[ti]) continue;
        const int64_t o = offs[t];
        const int nn = nnode[t];
        const float* tw = tnodewt + o;
        const int32_t* tc = nodeclass + o;
        const int nd = __ldg(leafnode + ti);
        const float fnoob = (float)__ldg(noob_arr + t);
        const bool base_ok = __ldg(tc + nd) == yi;
        if (k == 0 && base_ok) accq = __fadd_rn(accq, __fdiv_rn(vote_w(tw, nd, nn), fnoob));
        if (!impn) continue;
        const bool used = (__ldg(iv + (size_t)t * ivw + (k >> 6)) >> (k & 63)) & 1ull;
        if (used) {
            int cls = -1;
            const int ip = __ldg(partner + ti);
            const int pn = imp_walk(X + (size_t)i * p, X + (size_t)ip * p, k, p, nodes + o, tc, nn > 0 ? nn : 1,
                                    catgoleft ? catgoleft + o * maxcat : nullptr, maxcat, &cls);
            if (pn < 0) {
                atomicOr(err, ERR_STALE_JVR);
                continue;
            }
            if (cls == yi) acc = __fadd_rn(acc, __fdiv_rn(vote_w(tw, pn, nn), fnoob));
        } else if (base_ok) {
            acc = __fadd_rn(acc, __fdiv_rn(vote_w(tw, nd, nn), fnoob));
        }
    }
    if (impn) qimpm[idx] = acc;
    if (k == 0) qimp[i] = accq;
}

// avimp[k] and sqsd[k]: sums over the trees in order of rr and rr * rr.
__global__ void cw_feature_kernel(const float* __restrict__ rr, int p, int T, float* __restrict__ avimp,
                                  float* __restrict__ sqsd) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= p) return;
    float a = 0.0f, s = 0.0f;
    for (int t = 0; t < T; ++t) {
        const float r = rr[(size_t)t * p + k];
        a = __fadd_rn(a, r);
        s = __fadd_rn(s, __fmul_rn(r, r));
    }
    avimp[k] = a;
    sqsd[k] = s;
}

inline unsigned nblk(int64_t count, int b = 256) { return (unsigned)((count + b - 1) / b); }

}  // namespace

// Per-node tnodewt of the loaded forest into c->d_tnodewt (allocated here).
rfx_status launch_tnodewt(Ctx* c) {
    rfx_status st = dalloc(c, &c->d_tnodewt, (size_t)c->N);
    if (st) return st;
    Scratch sc(c);
    int32_t* wsum = sc.get<int32_t>((size_t)c->N);
    int32_t* wcnt = sc.get<int32_t>((size_t)c->N);
    if (!wsum || !wcnt) {
        set_error("case-wise weights: scratch allocation failed");
        return RFX_ERR_OOM;
    }
    RFX_CUDA(cudaMemsetAsync(wsum, 0, sizeof(int32_t) * (size_t)c->N, c->stream));
    RFX_CUDA(cudaMemsetAsync(wcnt, 0, sizeof(int32_t) * (size_t)c->N, c->stream));
    dim3 g(nblk(c->n), c->T);
    tnodewt_walk_kernel<<<g, 256, 0, c->stream>>>(c->d_X, c->n, c->p, c->d_nodes, c->d_offs, c->d_nnode,
                                                  c->d_catgoleft, c->maxcat, c->d_nin, wsum, wcnt);
    tnodewt_final_kernel<<<nblk(c->N), 256, 0, c->stream>>>(c->N, wsum, wcnt, c->d_tnodewt);
    RFX_CUDA(cudaGetLastError());
    c->launches += 2;
    return RFX_OK;
}

rfx_status launch_casewise_votes(Ctx* c, const int32_t* d_leafnode, float* d_q) {
    if (c->nclass > 64) {
        set_error("case-wise votes: at most 64 classes");
        return RFX_ERR_UNSUPPORTED;
    }
    const int th = 128;
    const size_t smem = (size_t)th * c->nclass * sizeof(float);
    casewise_votes_kernel<<<nblk(c->n, th), th, smem, c->stream>>>(d_leafnode, c->d_inbag, c->d_offs, c->d_nnode,
                                                                   c->d_nodeclass, c->d_tnodewt, c->n, c->T,
                                                                   c->nclass, d_q);
    RFX_CUDA(cudaGetLastError());
    c->launches += 1;
    return RFX_OK;
}

// Weighted FP64 pair sums (mode 0 case-wise, 2 unweighted) or the RF-GAP
// matrix (mode 1), packed upper triangle, from leaf lists of keys `key`
// (segbase/segoff/memb of those keys).
rfx_status launch_weighted_rows(Ctx* c, int mode, const int32_t* key, const int64_t* segbase, const int32_t* segoff,
                                const int32_t* memb, int64_t nkeys, double* out) {
    Scratch sc(c);
    long long* mass = sc.get<long long>((size_t)nkeys);
    if (!mass) {
        set_error("weighted pair sums: scratch allocation failed");
        return RFX_ERR_OOM;
    }
    key_mass_kernel<<<c->T, 128, 0, c->stream>>>(segbase, segoff, memb, c->d_nin, c->n, mass);
    dim3 g(c->n, (c->n + WR_WINDOW - 1) / WR_WINDOW);
    const size_t smem = 2 * (size_t)WR_WINDOW * sizeof(double);
    RFX_CUDA(cudaFuncSetAttribute(weighted_row_kernel<WR_RFGAP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem));
    RFX_CUDA(cudaFuncSetAttribute(weighted_row_kernel<WR_CASEWISE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem));
    RFX_CUDA(cudaFuncSetAttribute(weighted_row_kernel<WR_PLAIN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem));
    if (mode == WR_PLAIN)
        weighted_row_kernel<WR_PLAIN><<<g, WR_THREADS, smem, c->stream>>>(key, segbase, segoff, memb, mass, c->d_nin,
                                                                          c->d_nout, c->n, c->T, out);
    else if (mode == WR_RFGAP)
        weighted_row_kernel<WR_RFGAP><<<g, WR_THREADS, smem, c->stream>>>(key, segbase, segoff, memb, mass, c->d_nin,
                                                                          c->d_nout, c->n, c->T, out);
    else
        weighted_row_kernel<WR_CASEWISE><<<g, WR_THREADS, smem, c->stream>>>(key, segbase, segoff, memb, mass,
                                                                             c->d_nin, c->d_nout, c->n, c->T, out);
    RFX_CUDA(cudaGetLastError());
    c->launches += 2;
    return RFX_OK;
}

rfx_status launch_gap_keys(Ctx* c, const int32_t* d_leafnode, int32_t* d_key) {
    const int64_t cells = (int64_t)c->T * c->n;
    gap_key_kernel<<<nblk(cells), 256, 0, c->stream>>>(d_leafnode, c->d_inbag, cells, d_key);
    RFX_CUDA(cudaGetLastError());
    c->launches += 1;
    return RFX_OK;
}

// Case-wise importance: rr per (tree, feature), then the per-sample and
// per-feature sums; needs d_joob / d_partner (OOB lists and permutation
// partners) and the testreebag node ids.
rfx_status launch_casewise_varimp(Ctx* c, const int32_t* d_leafnode, int impn, float* d_avimp, float* d_sqsd,
                                  float* d_qimp, float* d_qimpm) {
    Scratch sc(c);
    float* rr = sc.get<float>((size_t)c->T * c->p);
    if (!rr) {
        set_error("case-wise importance: scratch allocation failed");
        return RFX_ERR_OOM;
    }
    const int ivw = c->iv_words;
    cw_tree_kernel<<<nblk((int64_t)c->T * c->p, 128), 128, 0, c->stream>>>(
        c->d_X, c->d_y, c->n, c->p, c->T, c->d_nodes, c->d_nodeclass, c->d_offs, c->d_nnode, c->d_catgoleft,
        c->maxcat, c->d_iv, ivw, c->d_joob, c->d_noob, c->d_partner, d_leafnode, c->d_tnodewt, rr, c->d_err);
    cw_feature_kernel<<<nblk(c->p, 128), 128, 0, c->stream>>>(rr, c->p, c->T, d_avimp, d_sqsd);
    cw_sample_kernel<<<nblk((int64_t)c->n * c->p, 128), 128, 0, c->stream>>>(
        c->d_X, c->d_y, c->n, c->p, c->T, c->d_nodes, c->d_nodeclass, c->d_offs, c->d_nnode, c->d_catgoleft,
        c->maxcat, c->d_iv, ivw, c->d_inbag, c->d_partner, d_leafnode, c->d_tnodewt, c->d_noob, impn, d_qimp,
        d_qimpm, c->d_err);
    RFX_CUDA(cudaGetLastError());
    c->launches += 3;
    return RFX_OK;
}

}  // namespace rfx
