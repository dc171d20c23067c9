// Device tree walks, one per routing rule of the reference.  They differ in
// their stopping rule and categorical handling, and each is restated exactly:
//   walk_testreebag  - cpu_testreebag        (src/rf_testreebag.cpp:39-123)
//   walk_terminal    - find_terminal_node    (src/rf_random_forest.cpp:2194-2244)
//   walk_predict     - predict_classification (src/rf_random_forest.cpp:1959-2013)
//   (the testreeimp walk lives in varimp.cu: it also tracks permutations)
// Float conversions and roundings are spelled with explicit intrinsics so that
// no compiler contraction changes a result.
#pragma once
#include "rfx_internal.cuh"

namespace rfx {

__device__ __forceinline__ DNode as_node(int4 v) {
    DNode d;
    d.split = __int_as_float(v.x);
    d.left = v.y;
    d.right = v.z;
    d.meta = v.w;
    return d;
}

__device__ __forceinline__ DNode load_node(const DNode* __restrict__ nodes, int k) {
    return as_node(__ldg(reinterpret_cast<const int4*>(nodes) + k));
}

struct GlobalNodes {
    const DNode* g;
    __device__ __forceinline__ DNode operator()(int k) const { return load_node(g, k); }
};

// A node record loaded by an explicit instruction.  The child-prefetching
// walks below load both children of a split node before the decision picks
// one; written as plain loads followed by a select, the compiler may turn the
// pair into one load from the selected address, which waits for the decision
// again.
__device__ __forceinline__ DNode load_node_now(const DNode* __restrict__ nodes, int k) {
    int4 v;
    asm volatile("ld.global.nc.v4.s32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(reinterpret_cast<const int4*>(nodes) + k));
    return as_node(v);
}

__device__ __forceinline__ int cgl_at(const int32_t* __restrict__ cgl, int maxcat, int node, int idx) {
    return cgl ? __ldg(cgl + (size_t)node * maxcat + idx) : 0;
}

// A sample's feature row: in global memory (read through the read-only
// cache) or staged in shared memory by the calling kernel.
struct GlobalRow {
    const float* r;
    __device__ __forceinline__ float operator()(int m) const { return __ldg(r + m); }
};
struct SharedRow {
    const float* r;
    __device__ __forceinline__ float operator()(int m) const { return r[m]; }
};

// Stage the feature rows of the 32 samples of a warp (lane l's sample id in
// `id`, -1 for none) into dst + r * ps (row r = lane r's sample), 16 rows per
// batch with every load of a batch in flight at once.  All 32 lanes call it.
__device__ __forceinline__ void stage_warp_rows(float* dst, int ps, const float* __restrict__ X, int p, int id,
                                                int lane) {
    for (int mb = 0; mb < p; mb += 64) {
        const int m0 = mb + lane, m1 = mb + 32 + lane;
#pragma unroll
        for (int r0 = 0; r0 < 32; r0 += 16) {
            int ids[16];
            float v0[16], v1[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) ids[q] = __shfl_sync(0xffffffffu, id, r0 + q);
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const float* src = X + (size_t)(ids[q] < 0 ? 0 : ids[q]) * p;
                v0[q] = (ids[q] >= 0 && m0 < p) ? __ldg(src + m0) : 0.0f;
                v1[q] = (ids[q] >= 0 && m1 < p) ? __ldg(src + m1) : 0.0f;
            }
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                if (ids[q] < 0) continue;
                float* d = dst + (size_t)(r0 + q) * ps;
                if (m0 < p) d[m0] = v0[q];
                if (m1 < p) d[m1] = v1[q];
            }
        }
    }
}

// Returns the node id; *cls receives the class (nodeclass of the final node,
// or of the root on the fallback path).
template <typename Src, typename XR>
__device__ __forceinline__ int walk_testreebag_x(const XR& xrow, int p, const Src& nodes,
                                                 const int32_t* __restrict__ nclass_of, int nnode,
                                                 const int32_t* __restrict__ cat, const int32_t* __restrict__ cgl,
                                                 int maxcat, int* cls) {
    int kt = 0;
    int steps = 0;
    DNode nd = nodes(0);
    while (node_status(nd.meta) == 1 && steps < 1000) {
        steps++;
        if (steps >= 1000) break;
        const int m = node_var(nd.meta);
        if (m >= p) break;
        const float v = xrow(m);
        if (!node_cat(nd.meta)) {
            kt = (v <= nd.split) ? nd.left : nd.right;
        } else {
            const int iv = __float2int_rz(v);
            if (iv >= 0 && iv < __ldg(cat + m)) {
                kt = (cgl_at(cgl, maxcat, kt, iv) == 1) ? nd.left : nd.right;
            } else {
                kt = nd.right;
            }
        }
        if (kt < 0 || kt >= nnode) {
            kt = 0;
            nd = nodes(0);
            break;
        }
        nd = nodes(kt);
        if (node_status(nd.meta) != 1) break;
    }
    const int st = node_status(nd.meta);
    if (st == -1 || st == 2) {
        *cls = __ldg(nclass_of + kt);
        return kt;
    }
    *cls = __ldg(nclass_of + 0);
    return 0;
}

// Child-prefetching forms of the two routing walks.  At a split node both
// children are loaded together with the feature value the decision needs, so
// a step waits for one round trip to memory instead of two (node, then
// feature).  The loads stay in bounds: pack_nodes_kernel (load.cu) checks
// that every node with status != -1 has both children in [0, nnode).  The
// decisions, stopping rules and results are those of walk_testreebag_x and
// walk_terminal_x.
template <typename XR>
__device__ __forceinline__ int walk_testreebag_pf(const XR& xrow, int p, const DNode* __restrict__ nodes,
                                                  const int32_t* __restrict__ nclass_of, int nnode,
                                                  const int32_t* __restrict__ cat, const int32_t* __restrict__ cgl,
                                                  int maxcat, int* cls) {
    int kt = 0;
    int steps = 0;
    DNode nd = load_node_now(nodes, 0);
    while (node_status(nd.meta) == 1 && steps < 1000) {
        steps++;
        if (steps >= 1000) break;
        const int m = node_var(nd.meta);
        if (m >= p) break;
        const DNode cl = load_node_now(nodes, nd.left);
        const DNode cr = load_node_now(nodes, nd.right);
        const float v = xrow(m);
        bool go_left;
        if (!node_cat(nd.meta)) {
            go_left = v <= nd.split;
        } else {
            const int iv = __float2int_rz(v);
            go_left = iv >= 0 && iv < __ldg(cat + m) && cgl_at(cgl, maxcat, kt, iv) == 1;
        }
        kt = go_left ? nd.left : nd.right;
        nd = go_left ? cl : cr;
        if (node_status(nd.meta) != 1) break;
    }
    const int st = node_status(nd.meta);
    if (st == -1 || st == 2) {
        *cls = __ldg(nclass_of + kt);
        return kt;
    }
    *cls = __ldg(nclass_of + 0);
    return 0;
}

template <typename XR>
__device__ __forceinline__ int walk_terminal_pf(const XR& xrow, int p, const DNode* __restrict__ nodes,
                                                const int32_t* __restrict__ cat, const int32_t* __restrict__ cgl,
                                                int maxcat, int maxnode) {
    int cur = 0;
    DNode nd = load_node_now(nodes, 0);
    for (int k = 0; k < maxnode; ++k) {
        if (node_status(nd.meta) == -1) return cur;
        const int m = node_var(nd.meta);
        if (m >= p) return 0;
        const DNode cl = load_node_now(nodes, nd.left);
        const DNode cr = load_node_now(nodes, nd.right);
        const float v = xrow(m);
        bool go_left;
        if (!node_cat(nd.meta)) {
            go_left = v <= nd.split;
        } else {
            const int j = __double2int_rz(__dadd_rn((double)v, 0.5));
            if (j >= 1 && j <= __ldg(cat + m)) {
                go_left = cgl_at(cgl, maxcat, cur, j - 1) == 1;
            } else {
                return 0;
            }
        }
        cur = go_left ? nd.left : nd.right;
        nd = go_left ? cl : cr;
    }
    return 0;
}

template <typename Src>
__device__ __forceinline__ int walk_testreebag_src(const float* __restrict__ xrow, int p, const Src& nodes,
                                                   const int32_t* __restrict__ nclass_of, int nnode,
                                                   const int32_t* __restrict__ cat, const int32_t* __restrict__ cgl,
                                                   int maxcat, int* cls) {
    return walk_testreebag_x(GlobalRow{xrow}, p, nodes, nclass_of, nnode, cat, cgl, maxcat, cls);
}

__device__ __forceinline__ int walk_testreebag(const float* __restrict__ xrow, int p, const DNode* __restrict__ nodes,
                                               const int32_t* __restrict__ nclass_of, int nnode,
                                               const int32_t* __restrict__ cat, const int32_t* __restrict__ cgl,
                                               int maxcat, int* cls) {
    return walk_testreebag_src(xrow, p, GlobalNodes{nodes}, nclass_of, nnode, cat, cgl, maxcat, cls);
}

// find_terminal_node: stops only at status -1; invalid category or variable
// returns the root.  maxnode is the reference's loop bound (2n+1).
template <typename Src, typename XR>
__device__ __forceinline__ int walk_terminal_x(const XR& xrow, int p, const Src& nodes,
                                               const int32_t* __restrict__ cat, const int32_t* __restrict__ cgl,
                                               int maxcat, int maxnode) {
    int cur = 0;
    for (int k = 0; k < maxnode; ++k) {
        const DNode nd = nodes(cur);
        if (node_status(nd.meta) == -1) return cur;
        const int m = node_var(nd.meta);
        if (m >= p) return 0;
        const float v = xrow(m);
        if (!node_cat(nd.meta)) {
            cur = (v <= nd.split) ? nd.left : nd.right;
        } else {
            const int j = __double2int_rz(__dadd_rn((double)v, 0.5));
            if (j >= 1 && j <= __ldg(cat + m)) {
                cur = (cgl_at(cgl, maxcat, cur, j - 1) == 1) ? nd.left : nd.right;
            } else {
                return 0;
            }
        }
    }
    return 0;
}

template <typename Src>
__device__ __forceinline__ int walk_terminal_src(const float* __restrict__ xrow, int p, const Src& nodes,
                                                 const int32_t* __restrict__ cat, const int32_t* __restrict__ cgl,
                                                 int maxcat, int maxnode) {
    return walk_terminal_x(GlobalRow{xrow}, p, nodes, cat, cgl, maxcat, maxnode);
}

__device__ __forceinline__ int walk_terminal(const float* __restrict__ xrow, int p, const DNode* __restrict__ nodes,
                                             const int32_t* __restrict__ cat, const int32_t* __restrict__ cgl,
                                             int maxcat, int maxnode) {
    return walk_terminal_src(xrow, p, GlobalNodes{nodes}, cat, cgl, maxcat, maxnode);
}

// predict_classification's walk: returns the voted class, or -1 for no vote
// (loop bound reached).  Invalid paths vote for class 0.
__device__ __forceinline__ int walk_predict(const float* __restrict__ xrow, int p, int nclass,
                                            const DNode* __restrict__ nodes, const int32_t* __restrict__ nclass_of,
                                            const int32_t* __restrict__ cat, const int32_t* __restrict__ cgl,
                                            int maxcat, int maxnode) {
    int kt = 0;
    for (int k = 0; k < maxnode; ++k) {
        if (kt >= maxnode) return 0;
        const DNode nd = load_node(nodes, kt);
        if (node_status(nd.meta) == -1) {
            const int c = __ldg(nclass_of + kt);
            return (c >= 0 && c < nclass) ? c : 0;
        }
        const int m = node_var(nd.meta);
        if (m >= p) return 0;
        const float v = __ldg(xrow + m);
        if (!node_cat(nd.meta)) {
            kt = (v <= nd.split) ? nd.left : nd.right;
        } else {
            const int j = __double2int_rz(__dadd_rn((double)v, 0.5));
            if (j >= 1 && j <= __ldg(cat + m)) {
                kt = (cgl_at(cgl, maxcat, kt, j - 1) == 1) ? nd.left : nd.right;
            } else {
                return 0;
            }
        }
    }
    return -1;
}

}  // namespace rfx
