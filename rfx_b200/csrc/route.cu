// Leaf routing of every (tree, sample): OOB samples with the testreebag walk
// (their votes go to q), in-bag samples with find_terminal_node.  The output
// key feeds the pair-count kernels:
//   key = 2 * leafidx + (in-bag ? 1 : 0)   when the node is terminal,
//   key = -1                               otherwise (excluded from proximity,
//                                          as nod[] = -1 excludes it in
//                                          cpu_proximity, src/rf_proximity.cpp:114-136).
// Grid: x = sample chunk, y = tree, so CTAs resident at the same time work on
// the same few trees and their node arrays stay in L2.
#include "walks.cuh"

namespace rfx {

namespace {

// Launch shapes the autotuner chooses from: threads per CTA x trees per
// thread (a thread walks TPC consecutive trees for its sample, reusing the
// sample's feature row from L1).
template <int RT, int TPC>
__global__ void __launch_bounds__(RT)
route_kernel(const float* __restrict__ X, int n, int p, int T, int nclass, const DNode* __restrict__ nodes,
             const int32_t* __restrict__ nodeclass, const int32_t* __restrict__ leafidx,
             const int64_t* __restrict__ offs, const int32_t* __restrict__ nnode_arr,
             const uint8_t* __restrict__ inbag, const int32_t* __restrict__ cat,
             const int32_t* __restrict__ catgoleft, int maxcat, int32_t* __restrict__ key_out,
             int32_t* __restrict__ leaf_out, int32_t* __restrict__ votes) {
    const int i = blockIdx.x * RT + threadIdx.x;
    if (i >= n) return;
    const float* xrow = X + (size_t)i * p;
#pragma unroll 1
    for (int q = 0; q < TPC; ++q) {
        const int t = blockIdx.y * TPC + q;
        if (t >= T) return;
        const int64_t o = offs[t];
        const DNode* tn = nodes + o;
        const int32_t* tc = nodeclass + o;
        const int32_t* cgl = catgoleft ? catgoleft + o * maxcat : nullptr;
        const int nn = nnode_arr[t];
        const size_t ti = (size_t)t * n + i;
        const bool ib = inbag[ti] != 0;
        int node;
        if (!ib) {
            int cls;
            node = walk_testreebag(xrow, p, tn, tc, nn, cat, cgl, maxcat, &cls);
            if (cls >= 0 && cls < nclass) atomicAdd(votes + (size_t)i * nclass + cls, 1);
        } else {
            node = walk_terminal(xrow, p, tn, cat, cgl, maxcat, 2 * n + 1);
        }
        const int li = (node >= 0 && node < nn) ? __ldg(leafidx + o + node) : -1;
        key_out[ti] = li >= 0 ? 2 * li + (ib ? 1 : 0) : -1;
        if (leaf_out) leaf_out[ti] = node;
    }
}

// One (tree, sample) walk advanced one node at a time, so that a thread can
// keep two walks in flight: cpu_testreebag for an OOB sample, find_terminal_node
// for an in-bag one, each restated exactly as in walks.cuh.
struct Walk {
    const DNode* tn;
    const int32_t* tc;
    const int32_t* cgl;
    int nn, kt, steps, node, cls;
    bool oob, done;
    DNode nd;
};

__device__ __forceinline__ void walk_begin(Walk& w, const DNode* tn, const int32_t* tc, const int32_t* cgl, int nn,
                                           bool oob) {
    w.tn = tn;
    w.tc = tc;
    w.cgl = cgl;
    w.nn = nn;
    w.kt = 0;
    w.steps = 0;
    w.node = 0;
    w.cls = -1;
    w.oob = oob;
    w.done = false;
}

// Decide at the current node w.nd (already loaded); on return either w.done
// with node/cls set, or w.kt is the next node to load.
__device__ __forceinline__ void walk_advance(Walk& w, const float* __restrict__ xrow, int p,
                                             const int32_t* __restrict__ cat, int maxcat, int maxnode) {
    const int st = node_status(w.nd.meta);
    if (w.oob) {  // cpu_testreebag
        if (st != 1) {
            if (st == -1 || st == 2) {
                w.cls = __ldg(w.tc + w.kt);
                w.node = w.kt;
            } else {
                w.cls = __ldg(w.tc);
                w.node = 0;
            }
            w.done = true;
            return;
        }
        const int m = node_var(w.nd.meta);
        if (++w.steps >= 1000 || m >= p) {
            w.cls = __ldg(w.tc);
            w.node = 0;
            w.done = true;
            return;
        }
        const float v = __ldg(xrow + m);
        int nx;
        if (!node_cat(w.nd.meta)) {
            nx = (v <= w.nd.split) ? w.nd.left : w.nd.right;
        } else {
            const int iv = __float2int_rz(v);
            nx = (iv >= 0 && iv < __ldg(cat + m)) ? ((cgl_at(w.cgl, maxcat, w.kt, iv) == 1) ? w.nd.left : w.nd.right)
                                                 : w.nd.right;
        }
        if (nx < 0 || nx >= w.nn) {  // the root and its class
            w.cls = __ldg(w.tc);
            w.node = 0;
            w.done = true;
            return;
        }
        w.kt = nx;
        return;
    }
    // find_terminal_node: at most maxnode nodes are examined
    if (w.steps >= maxnode) {
        w.node = 0;
        w.done = true;
        return;
    }
    ++w.steps;
    if (st == -1) {
        w.node = w.kt;
        w.done = true;
        return;
    }
    const int m = node_var(w.nd.meta);
    if (m >= p) {
        w.node = 0;
        w.done = true;
        return;
    }
    const float v = __ldg(xrow + m);
    if (!node_cat(w.nd.meta)) {
        w.kt = (v <= w.nd.split) ? w.nd.left : w.nd.right;
    } else {
        const int j = __double2int_rz(__dadd_rn((double)v, 0.5));
        if (j >= 1 && j <= __ldg(cat + m)) {
            w.kt = (cgl_at(w.cgl, maxcat, w.kt, j - 1) == 1) ? w.nd.left : w.nd.right;
        } else {
            w.node = 0;
            w.done = true;
        }
    }
}

// Two trees per step of the loop: both walks' node loads are in flight at once.
template <int RT, int TPC>
__global__ void __launch_bounds__(RT)
route2_kernel(const float* __restrict__ X, int n, int p, int T, int nclass, const DNode* __restrict__ nodes,
              const int32_t* __restrict__ nodeclass, const int32_t* __restrict__ leafidx,
              const int64_t* __restrict__ offs, const int32_t* __restrict__ nnode_arr,
              const uint8_t* __restrict__ inbag, const int32_t* __restrict__ cat,
              const int32_t* __restrict__ catgoleft, int maxcat, int32_t* __restrict__ key_out,
              int32_t* __restrict__ leaf_out, int32_t* __restrict__ votes) {
    static_assert(TPC % 2 == 0, "trees in pairs");
    const int i = blockIdx.x * RT + threadIdx.x;
    if (i >= n) return;
    const float* xrow = X + (size_t)i * p;
    const int maxnode = 2 * n + 1;
#pragma unroll 1
    for (int q = 0; q < TPC; q += 2) {
        const int ta = blockIdx.y * TPC + q;
        if (ta >= T) return;
        const int tb = ta + 1 < T ? ta + 1 : -1;
        Walk w[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int t = h == 0 ? ta : tb;
            if (t < 0) {
                w[h].done = true;
                continue;
            }
            const int64_t o = offs[t];
            walk_begin(w[h], nodes + o, nodeclass + o, catgoleft ? catgoleft + o * maxcat : nullptr, nnode_arr[t],
                       inbag[(size_t)t * n + i] == 0);
        }
#pragma unroll
        for (int h = 0; h < 2; ++h)
            if (!w[h].done) w[h].nd = load_node(w[h].tn, 0);
        while (!w[0].done || !w[1].done) {
#pragma unroll
            for (int h = 0; h < 2; ++h)
                if (!w[h].done) walk_advance(w[h], xrow, p, cat, maxcat, maxnode);
#pragma unroll
            for (int h = 0; h < 2; ++h)
                if (!w[h].done) w[h].nd = load_node(w[h].tn, w[h].kt);
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int t = h == 0 ? ta : tb;
            if (t < 0) continue;
            const int64_t o = offs[t];
            if (w[h].oob && w[h].cls >= 0 && w[h].cls < nclass) atomicAdd(votes + (size_t)i * nclass + w[h].cls, 1);
            const int node = w[h].node;
            const int li = (node >= 0 && node < w[h].nn) ? __ldg(leafidx + o + node) : -1;
            const size_t ti = (size_t)t * n + i;
            key_out[ti] = li >= 0 ? 2 * li + (w[h].oob ? 0 : 1) : -1;
            if (leaf_out) leaf_out[ti] = node;
        }
    }
}

// Routing in leaf order: when the member lists of this forest exist from an
// earlier pass, tree t's samples are taken in that order (members of one leaf
// and bag status together, then the samples without a terminal node), so the
// threads of a warp follow the same path with the same walk rule.  Every
// result is indexed by sample, so only the order of work changes.  With PF
// the walks load both children of each split node with the feature value
// (walk_testreebag_pf / walk_terminal_pf).
template <int RT, bool PF = false>
__global__ void __launch_bounds__(RT)
route_leaf_order_kernel(const float* __restrict__ X, int n, int p, int nclass, const DNode* __restrict__ nodes,
                        const int32_t* __restrict__ nodeclass, const int32_t* __restrict__ leafidx,
                        const int64_t* __restrict__ offs, const int32_t* __restrict__ nnode_arr,
                        const uint8_t* __restrict__ inbag, const int32_t* __restrict__ cat,
                        const int32_t* __restrict__ catgoleft, int maxcat, const int32_t* __restrict__ memb,
                        int32_t* __restrict__ key_out, int32_t* __restrict__ votes) {
    const int t = blockIdx.y;
    const int q = blockIdx.x * RT + threadIdx.x;
    if (q >= n) return;
    const size_t tq = (size_t)t * n + q;
    const int i = __ldg(memb + tq);
    const float* xrow = X + (size_t)i * p;
    const int64_t o = offs[t];
    const DNode* tn = nodes + o;
    const int32_t* tc = nodeclass + o;
    const int32_t* cgl = catgoleft ? catgoleft + o * maxcat : nullptr;
    const int nn = nnode_arr[t];
    const size_t ti = (size_t)t * n + i;
    const bool ib = inbag[ti] != 0;
    int node;
    if (!ib) {
        int cls;
        if constexpr (PF) node = walk_testreebag_pf(GlobalRow{xrow}, p, tn, tc, nn, cat, cgl, maxcat, &cls);
        else node = walk_testreebag(xrow, p, tn, tc, nn, cat, cgl, maxcat, &cls);
        if (cls >= 0 && cls < nclass) atomicAdd(votes + (size_t)i * nclass + cls, 1);
    } else {
        if constexpr (PF) node = walk_terminal_pf(GlobalRow{xrow}, p, tn, cat, cgl, maxcat, 2 * n + 1);
        else node = walk_terminal(xrow, p, tn, cat, cgl, maxcat, 2 * n + 1);
    }
    const int li = (node >= 0 && node < nn) ? __ldg(leafidx + o + node) : -1;
    key_out[ti] = li >= 0 ? 2 * li + (ib ? 1 : 0) : -1;
}

// The same with the CTA's feature rows staged in shared memory first (row
// stride p | 1 floats, so that the lanes of a warp reading one feature hit
// different banks): each walk step then waits for one node load (L1, the
// CTA's samples share a tree) instead of a node load and an L2 feature load.
template <int RT>
__global__ void __launch_bounds__(RT)
route_leaf_staged_kernel(const float* __restrict__ X, int n, int p, int nclass, const DNode* __restrict__ nodes,
                         const int32_t* __restrict__ nodeclass, const int32_t* __restrict__ leafidx,
                         const int64_t* __restrict__ offs, const int32_t* __restrict__ nnode_arr,
                         const uint8_t* __restrict__ inbag, const int32_t* __restrict__ cat,
                         const int32_t* __restrict__ catgoleft, int maxcat, const int32_t* __restrict__ memb,
                         int32_t* __restrict__ key_out, int32_t* __restrict__ votes) {
    extern __shared__ float xs[];  // RT rows of ps floats
    const int ps = p | 1;
    const int t = blockIdx.y;
    const int q = blockIdx.x * RT + threadIdx.x;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int i = q < n ? __ldg(memb + (size_t)t * n + q) : -1;
    // each warp stages its 32 rows
    stage_warp_rows(xs + (size_t)(w * 32) * ps, ps, X, p, i, lane);
    __syncwarp();
    if (q >= n) return;
    const SharedRow xrow{xs + (size_t)threadIdx.x * ps};
    const int64_t o = offs[t];
    const DNode* tn = nodes + o;
    const int32_t* tc = nodeclass + o;
    const int32_t* cgl = catgoleft ? catgoleft + o * maxcat : nullptr;
    const int nn = nnode_arr[t];
    const size_t ti = (size_t)t * n + i;
    const bool ib = inbag[ti] != 0;
    int node;
    if (!ib) {
        int cls;
        node = walk_testreebag_x(xrow, p, GlobalNodes{tn}, tc, nn, cat, cgl, maxcat, &cls);
        if (cls >= 0 && cls < nclass) atomicAdd(votes + (size_t)i * nclass + cls, 1);
    } else {
        node = walk_terminal_x(xrow, p, GlobalNodes{tn}, cat, cgl, maxcat, 2 * n + 1);
    }
    const int li = (node >= 0 && node < nn) ? __ldg(leafidx + o + node) : -1;
    key_out[ti] = li >= 0 ? 2 * li + (ib ? 1 : 0) : -1;
}

// The first KN nodes of tree t (the top levels: the grower numbers nodes in
// the order it creates them, level by level) staged in shared memory; a CTA
// then walks SUB x RT samples of that tree, so the staging is paid once per
// RT * SUB samples.  Deeper nodes are read from global memory.
struct StagedNodes {
    const DNode* g;
    const int4* s;
    int k;
    __device__ __forceinline__ DNode operator()(int j) const { return j < k ? as_node(s[j]) : load_node(g, j); }
};

template <int RT, int SUB, int KN>
__global__ void __launch_bounds__(RT)
route_nodes_kernel(const float* __restrict__ X, int n, int p, int T, int nclass, const DNode* __restrict__ nodes,
                   const int32_t* __restrict__ nodeclass, const int32_t* __restrict__ leafidx,
                   const int64_t* __restrict__ offs, const int32_t* __restrict__ nnode_arr,
                   const uint8_t* __restrict__ inbag, const int32_t* __restrict__ cat,
                   const int32_t* __restrict__ catgoleft, int maxcat, int32_t* __restrict__ key_out,
                   int32_t* __restrict__ leaf_out, int32_t* __restrict__ votes) {
    __shared__ int4 sn[KN];
    const int t = blockIdx.y;
    const int64_t o = offs[t];
    const int nn = nnode_arr[t];
    const int kn = min(KN, nn);
    const DNode* tn = nodes + o;
    for (int j = threadIdx.x; j < kn; j += RT) sn[j] = __ldg(reinterpret_cast<const int4*>(tn) + j);
    __syncthreads();
    const StagedNodes src{tn, sn, kn};
    const int32_t* tc = nodeclass + o;
    const int32_t* cgl = catgoleft ? catgoleft + o * maxcat : nullptr;
#pragma unroll 1
    for (int s = 0; s < SUB; ++s) {
        const int i = (blockIdx.x * SUB + s) * RT + threadIdx.x;
        if (i >= n) return;
        const float* xrow = X + (size_t)i * p;
        const size_t ti = (size_t)t * n + i;
        const bool ib = inbag[ti] != 0;
        int node;
        if (!ib) {
            int cls;
            node = walk_testreebag_src(xrow, p, src, tc, nn, cat, cgl, maxcat, &cls);
            if (cls >= 0 && cls < nclass) atomicAdd(votes + (size_t)i * nclass + cls, 1);
        } else {
            node = walk_terminal_src(xrow, p, src, cat, cgl, maxcat, 2 * n + 1);
        }
        const int li = (node >= 0 && node < nn) ? __ldg(leafidx + o + node) : -1;
        key_out[ti] = li >= 0 ? 2 * li + (ib ? 1 : 0) : -1;
        if (leaf_out) leaf_out[ti] = node;
    }
}

constexpr int ROUTE_SHAPES = 10;

// votes must be zero beforehand (the kernel adds to them)
void route_launch(Ctx* c, int shape, int32_t* d_leaf) {
    auto go = [&](auto kernel, int rt, int tpc) {
        dim3 grid((c->n + rt - 1) / rt, (c->T + tpc - 1) / tpc);
        kernel<<<grid, rt, 0, c->stream>>>(c->d_X, c->n, c->p, c->T, c->nclass, c->d_nodes, c->d_nodeclass,
                                           c->d_leafidx, c->d_offs, c->d_nnode, c->d_inbag, c->d_cat,
                                           c->d_catgoleft, c->maxcat, c->d_key, d_leaf, c->d_votes);
    };
    auto go_nodes = [&](auto kernel, int rt, int sub) {
        dim3 grid((c->n + rt * sub - 1) / (rt * sub), c->T);
        kernel<<<grid, rt, 0, c->stream>>>(c->d_X, c->n, c->p, c->T, c->nclass, c->d_nodes, c->d_nodeclass,
                                           c->d_leafidx, c->d_offs, c->d_nnode, c->d_inbag, c->d_cat,
                                           c->d_catgoleft, c->maxcat, c->d_key, d_leaf, c->d_votes);
    };
    switch (shape) {
        case 1: go(route_kernel<128, 1>, 128, 1); break;
        case 2: go(route_kernel<512, 1>, 512, 1); break;
        case 3: go(route_kernel<256, 2>, 256, 2); break;
        case 4: go(route_kernel<256, 4>, 256, 4); break;
        case 5: go(route2_kernel<256, 2>, 256, 2); break;
        case 6: go(route2_kernel<256, 4>, 256, 4); break;
        case 7: go(route2_kernel<128, 4>, 128, 4); break;
        case 8: go_nodes(route_nodes_kernel<256, 8, 2048>, 256, 8); break;
        case 9: go_nodes(route_nodes_kernel<256, 4, 1024>, 256, 4); break;
        default: go(route_kernel<256, 1>, 256, 1); break;
    }
}

// nout[i] = 2 * (number of trees with i out of bag): the reference increments
// it in cpu_bootstrap and again in the vote loop.
__global__ void nout_kernel(const uint8_t* __restrict__ inbag, int n, int T, int32_t* __restrict__ nout) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = 0;
    for (int t = 0; t < T; ++t) c += inbag[(size_t)t * n + i] == 0;
    nout[i] = 2 * c;
}

// OOB error / prediction / probability from integer votes, with the
// reference's float arithmetic: argmax with >= (ties to the higher class),
// total votes summed in float, probability = q / total (or 1/nclass).
template <typename TV>
__global__ void oob_summary_kernel(const TV* __restrict__ votes, const int32_t* __restrict__ nout,
                                   const int32_t* __restrict__ y, int n, int nclass, int32_t* __restrict__ pred,
                                   float* __restrict__ proba, unsigned int* __restrict__ counts) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const TV* q = votes + (size_t)i * nclass;
    const float uni = __double2float_rn(1.0 / (double)nclass);
    if (nout[i] > 0) {
        int best = 0;
        float mx = (float)q[0];
        float tot = 0.0f;
        for (int c = 0; c < nclass; ++c) {
            const float v = (float)q[c];
            tot = __fadd_rn(tot, v);
            if (v >= mx) {
                mx = v;
                best = c;
            }
        }
        if (pred) pred[i] = best;
        if (proba)
            for (int c = 0; c < nclass; ++c)
                proba[(size_t)i * nclass + c] = tot > 0.0f ? __fdiv_rn((float)q[c], tot) : uni;
        atomicAdd(counts + 0, 1u);
        if (best == y[i]) atomicAdd(counts + 1, 1u);
    } else {
        if (pred) pred[i] = 0;
        if (proba)
            for (int c = 0; c < nclass; ++c) proba[(size_t)i * nclass + c] = uni;
    }
}

__global__ void oob_error_kernel(const unsigned int* __restrict__ counts, float* __restrict__ err) {
    const unsigned total = counts[0], correct = counts[1];
    *err = total > 0 ? __fsub_rn(1.0f, __fdiv_rn((float)correct, (float)total)) : 0.0f;
}

constexpr int PRED_THREADS = 256;

__global__ void __launch_bounds__(PRED_THREADS)
predict_kernel(const float* __restrict__ X, int m, int p, int nclass, int maxnode, const DNode* __restrict__ nodes,
               const int32_t* __restrict__ nodeclass, const int64_t* __restrict__ offs,
               const int32_t* __restrict__ cat, const int32_t* __restrict__ catgoleft, int maxcat,
               int32_t* __restrict__ votes) {
    const int t = blockIdx.y;
    const int s = blockIdx.x * PRED_THREADS + threadIdx.x;
    if (s >= m) return;
    const int64_t o = offs[t];
    const int c = walk_predict(X + (size_t)s * p, p, nclass, nodes + o, nodeclass + o, cat,
                               catgoleft ? catgoleft + o * maxcat : nullptr, maxcat, maxnode);
    if (c >= 0) atomicAdd(votes + (size_t)s * nclass + c, 1);
}

}  // namespace

rfx_status launch_route(Ctx* c) {
    StageTimer st(c, ST_ROUTE, 2);
    rfx_status r;
    if (c->csr_built) {
        // the member lists of an earlier pass over this forest give the order
        // shapes 0-2: 128 / 256 / 512 threads; 3-5: 64 / 128 / 256 threads
        // with the feature rows staged in shared memory (when they fit in
        // 96 KB; otherwise the unstaged kernel of that width runs); 6-8:
        // 128 / 256 / 512 threads with child-prefetching walks
        const size_t row_bytes = sizeof(float) * (size_t)(c->p | 1);
        int dev_smem = 0;
        RFX_CUDA(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
        if (rfx_status s0 = allow_dyn_smem(route_leaf_staged_kernel<64>, dev_smem)) return s0;
        if (rfx_status s0 = allow_dyn_smem(route_leaf_staged_kernel<128>, dev_smem)) return s0;
        if (rfx_status s0 = allow_dyn_smem(route_leaf_staged_kernel<256>, dev_smem)) return s0;
        r = autotune(c, TK_ROUTE_LEAF, 9, 1, [&](int shape) -> rfx_status {
            RFX_CUDA(cudaMemsetAsync(c->d_votes, 0, sizeof(int32_t) * (size_t)c->n * c->nclass, c->stream));
            auto go = [&](auto kernel, int rt, size_t smem) {
                dim3 grid((c->n + rt - 1) / rt, c->T);
                kernel<<<grid, rt, smem, c->stream>>>(c->d_X, c->n, c->p, c->nclass, c->d_nodes, c->d_nodeclass,
                                                      c->d_leafidx, c->d_offs, c->d_nnode, c->d_inbag, c->d_cat,
                                                      c->d_catgoleft, c->maxcat, c->d_memb, c->d_key, c->d_votes);
            };
            const int srt = shape == 3 ? 64 : shape == 4 ? 128 : 256;
            const bool staged = shape >= 3 && shape <= 5 && (size_t)srt * row_bytes <= 96 * 1024;
            if (shape == 6) {
                go(route_leaf_order_kernel<128, true>, 128, 0);
            } else if (shape == 7) {
                go(route_leaf_order_kernel<256, true>, 256, 0);
            } else if (shape == 8) {
                go(route_leaf_order_kernel<512, true>, 512, 0);
            } else if (staged) {
                const size_t sm = (size_t)srt * row_bytes;
                if (srt == 64) go(route_leaf_staged_kernel<64>, 64, sm);
                else if (srt == 128) go(route_leaf_staged_kernel<128>, 128, sm);
                else go(route_leaf_staged_kernel<256>, 256, sm);
            } else if (shape == 0 || shape == 4) {
                go(route_leaf_order_kernel<128>, 128, 0);
            } else if (shape == 2) {
                go(route_leaf_order_kernel<512>, 512, 0);
            } else {
                go(route_leaf_order_kernel<256>, 256, 0);
            }
            RFX_CUDA(cudaGetLastError());
            return RFX_OK;
        });
    } else {
        r = autotune(c, TK_ROUTE, ROUTE_SHAPES, 0, [&](int shape) -> rfx_status {
            RFX_CUDA(cudaMemsetAsync(c->d_votes, 0, sizeof(int32_t) * (size_t)c->n * c->nclass, c->stream));
            route_launch(c, shape, nullptr);
            RFX_CUDA(cudaGetLastError());
            return RFX_OK;
        });
    }
    if (r != RFX_OK) return r;
    nout_kernel<<<(c->n + 255) / 256, 256, 0, c->stream>>>(c->d_inbag, c->n, c->T, c->d_nout);
    RFX_CUDA(cudaGetLastError());
    return RFX_OK;
}

rfx_status launch_route_leaf(Ctx* c, int32_t* d_leaf) {
    StageTimer st(c, ST_ROUTE, 1);
    // votes are recomputed identically; clear first so they stay exact
    RFX_CUDA(cudaMemsetAsync(c->d_votes, 0, sizeof(int32_t) * (size_t)c->n * c->nclass, c->stream));
    route_launch(c, 0, d_leaf);
    RFX_CUDA(cudaGetLastError());
    return RFX_OK;
}

rfx_status launch_oob_summary(Ctx* c, float* d_errout, int32_t* d_pred, float* d_proba) {
    StageTimer st(c, ST_OOB, d_errout ? 2 : 1);
    unsigned int* counts = reinterpret_cast<unsigned int*>(c->d_pairs) + 2;  // scratch words after the pair counter
    RFX_CUDA(cudaMemsetAsync(counts, 0, 2 * sizeof(unsigned int), c->stream));
    oob_summary_kernel<int32_t><<<(c->n + 255) / 256, 256, 0, c->stream>>>(c->d_votes, c->d_nout, c->d_y, c->n,
                                                                            c->nclass, d_pred, d_proba, counts);
    RFX_CUDA(cudaGetLastError());
    if (d_errout) {
        oob_error_kernel<<<1, 1, 0, c->stream>>>(counts, d_errout);
        RFX_CUDA(cudaGetLastError());
    }
    return RFX_OK;
}

// the same from float votes (case-wise weights)
rfx_status launch_oob_summary_f32(Ctx* c, const float* d_q, float* d_errout, int32_t* d_pred, float* d_proba) {
    StageTimer st(c, ST_OOB, d_errout ? 2 : 1);
    unsigned int* counts = reinterpret_cast<unsigned int*>(c->d_pairs) + 2;  // scratch words after the pair counter
    RFX_CUDA(cudaMemsetAsync(counts, 0, 2 * sizeof(unsigned int), c->stream));
    oob_summary_kernel<float><<<(c->n + 255) / 256, 256, 0, c->stream>>>(d_q, c->d_nout, c->d_y, c->n,
                                                                            c->nclass, d_pred, d_proba, counts);
    RFX_CUDA(cudaGetLastError());
    if (d_errout) {
        oob_error_kernel<<<1, 1, 0, c->stream>>>(counts, d_errout);
        RFX_CUDA(cudaGetLastError());
    }
    return RFX_OK;
}

rfx_status launch_predict(Ctx* c, const float* dX, int m, int32_t* d_votes) {
    StageTimer st(c, ST_PREDICT, m > 0 ? 1 : 0);
    RFX_CUDA(cudaMemsetAsync(d_votes, 0, sizeof(int32_t) * (size_t)m * c->nclass, c->stream));
    if (m == 0) return RFX_OK;
    dim3 grid((m + PRED_THREADS - 1) / PRED_THREADS, c->T);
    predict_kernel<<<grid, PRED_THREADS, 0, c->stream>>>(dX, m, c->p, c->nclass, 2 * c->n + 1, c->d_nodes,
                                                         c->d_nodeclass, c->d_offs, c->d_cat, c->d_catgoleft,
                                                         c->maxcat, d_votes);
    RFX_CUDA(cudaGetLastError());
    return RFX_OK;
}

}  // namespace rfx
