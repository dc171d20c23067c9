// Forest upload on the device: validation and packing of the node arrays and
// the bootstrap multiplicities, one CTA per tree.  Replaces a host pass over
// every node and every (tree, sample) with two kernels behind the raw H2D
// copies of the caller's arrays.
#include <cuda_runtime.h>

#include <cstdint>

#include "rfx_internal.cuh"

namespace rfx {
namespace {

constexpr int LD_THREADS = 256;

// First failure wins: code, tree, node.  code 0 = none.
__device__ __forceinline__ void load_fail(LoadError* e, int code, int t, int k) {
    if (atomicCAS(&e->code, 0, code) == 0) {
        e->tree = t;
        e->node = k;
    }
}

// Per tree: validate every node, pack {split, left, right, var|status|cat}
// records, number the terminal nodes in node order (leafidx), collect the
// features split on by non-terminal nodes (iv bit set) and count the leaves.
__global__ void __launch_bounds__(LD_THREADS)
pack_nodes_kernel(const int64_t* __restrict__ offs, const int32_t* __restrict__ status,
                  const int32_t* __restrict__ bestvar, const float* __restrict__ split,
                  const int32_t* __restrict__ treemap, const int32_t* __restrict__ cat, int p, int W,
                  DNode* __restrict__ nodes, int32_t* __restrict__ leafidx, uint64_t* __restrict__ iv,
                  int32_t* __restrict__ nleaf, LoadError* __restrict__ err) {
    __shared__ unsigned long long ivs[1024];  // ceil(65535 / 64) words
    __shared__ int wsum[LD_THREADS / 32];
    __shared__ int base;
    const int t = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int64_t o = offs[t];
    const int nn = (int)(offs[t + 1] - o);
    for (int q = tid; q < W; q += LD_THREADS) ivs[q] = 0ull;
    if (tid == 0) base = 0;
    __syncthreads();
    for (int k0 = 0; k0 < nn; k0 += LD_THREADS) {
        const int k = k0 + tid;
        int leaf = 0;
        if (k < nn) {
            const int64_t g = o + k;
            const int st = status[g];
            const int bv = bestvar[g];
            const int l = treemap[2 * g], r = treemap[2 * g + 1];
            if (st < -128 || st > 127) load_fail(err, 1, t, k);
            int var = 0, catf = 0;
            if (st != -1) {
                if (bv < 0 || bv >= p) {
                    load_fail(err, 2, t, k);
                } else {
                    var = bv;
                    catf = cat[bv] != 1 ? 1 : 0;
                    atomicOr(&ivs[bv >> 6], 1ull << (bv & 63));
                }
                if (l < 0 || l >= nn || r < 0 || r >= nn) load_fail(err, 3, t, k);
            }
            DNode d;
            d.split = split[g];
            d.left = l;
            d.right = r;
            d.meta = (var & 0xffff) | ((st & 0xff) << 16) | (catf << 24);
            nodes[g] = d;
            leaf = st == -1 ? 1 : 0;
        }
        // exclusive scan of the terminal flags over this chunk, in node order
        const unsigned bal = __ballot_sync(0xffffffffu, leaf);
        if (lane == 0) wsum[wid] = __popc(bal);
        __syncthreads();
        int woff = 0, tot = 0;
#pragma unroll
        for (int q = 0; q < LD_THREADS / 32; ++q) {
            if (q < wid) woff += wsum[q];
            tot += wsum[q];
        }
        if (k < nn) leafidx[o + k] = leaf ? base + woff + __popc(bal & ((1u << lane) - 1u)) : -1;
        __syncthreads();
        if (tid == 0) base += tot;
        __syncthreads();
    }
    for (int q = tid; q < W; q += LD_THREADS) iv[(size_t)t * W + q] = ivs[q];
    if (tid == 0) nleaf[t] = base;
}

// Per tree: bag flags (nin > 0) and the OOB count; negative multiplicities fail.
__global__ void __launch_bounds__(LD_THREADS)
bag_kernel(const int32_t* __restrict__ nin, int n, uint8_t* __restrict__ inbag, int32_t* __restrict__ noob,
           LoadError* __restrict__ err) {
    __shared__ int wsum[LD_THREADS / 32];
    const int t = blockIdx.x;
    const int32_t* row = nin + (size_t)t * n;
    uint8_t* out = inbag + (size_t)t * n;
    int cnt = 0;
    for (int i = threadIdx.x; i < n; i += LD_THREADS) {
        const int m = row[i];
        if (m < 0) load_fail(err, 4, t, i);
        out[i] = m > 0 ? 1 : 0;
        cnt += m == 0;
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, d);
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int q = 0; q < LD_THREADS / 32; ++q) s += wsum[q];
        noob[t] = s;
    }
}

// Padded device trees (tree t at slots t*maxnode.., as the reference's GPU
// grower leaves them, cuda/rf_growtree.cu:888-) gathered into the compact
// layout (tree t at offs[t]..offs[t+1]); one CTA per tree.
__global__ void __launch_bounds__(LD_THREADS)
gather_padded_kernel(const int64_t* __restrict__ offs, int maxnode, int maxcat, const int32_t* __restrict__ ps,
                     const int32_t* __restrict__ pbv, const float* __restrict__ pxs, const int32_t* __restrict__ ptm,
                     const int32_t* __restrict__ pnc, const int32_t* __restrict__ pcg, int32_t* __restrict__ status,
                     int32_t* __restrict__ bestvar, float* __restrict__ split, int32_t* __restrict__ treemap,
                     int32_t* __restrict__ nodeclass, int32_t* __restrict__ catgoleft) {
    const int t = blockIdx.x;
    const int64_t o = offs[t];
    const int nn = (int)(offs[t + 1] - o);
    const size_t src = (size_t)t * maxnode;
    for (int k = threadIdx.x; k < nn; k += LD_THREADS) {
        status[o + k] = ps[src + k];
        bestvar[o + k] = pbv[src + k];
        split[o + k] = pxs[src + k];
        nodeclass[o + k] = pnc[src + k];
    }
    for (int k = threadIdx.x; k < 2 * nn; k += LD_THREADS) treemap[2 * o + k] = ptm[2 * src + k];
    if (pcg)
        for (long long k = threadIdx.x; k < (long long)nn * maxcat; k += LD_THREADS)
            catgoleft[o * maxcat + k] = pcg[src * maxcat + k];
}

}  // namespace

cudaError_t launch_gather_padded(cudaStream_t s, int T, int maxnode, int maxcat, const int64_t* d_offs,
                                 const int32_t* status_p, const int32_t* bestvar_p, const float* split_p,
                                 const int32_t* treemap_p, const int32_t* nodeclass_p, const int32_t* catgoleft_p,
                                 int32_t* status, int32_t* bestvar, float* split, int32_t* treemap,
                                 int32_t* nodeclass, int32_t* catgoleft) {
    gather_padded_kernel<<<T, LD_THREADS, 0, s>>>(d_offs, maxnode, maxcat, status_p, bestvar_p, split_p, treemap_p,
                                                  nodeclass_p, catgoleft_p, status, bestvar, split, treemap, nodeclass,
                                                  catgoleft);
    return cudaGetLastError();
}

rfx_status launch_pack_forest(cudaStream_t s, int T, int n, int p, const int64_t* d_offs, const int32_t* status,
                              const int32_t* bestvar, const float* split, const int32_t* treemap,
                              const int32_t* d_cat, const int32_t* nin, DNode* nodes, int32_t* leafidx,
                              uint64_t* iv, int32_t* nleaf, uint8_t* inbag, int32_t* noob, LoadError* err) {
    const int W = (p + 63) / 64;
    pack_nodes_kernel<<<T, LD_THREADS, 0, s>>>(d_offs, status, bestvar, split, treemap, d_cat, p, W, nodes, leafidx,
                                               iv, nleaf, err);
    bag_kernel<<<T, LD_THREADS, 0, s>>>(nin, n, inbag, noob, err);
    RFX_CUDA(cudaGetLastError());
    return RFX_OK;
}

}  // namespace rfx
