// Permutation importance for all trees and all features in four or five
// launches (with more than 256 features the walk and the per-sample sums run
// once per block of 256 features).
//
// cpu_varimp (src/rf_varimp.cpp:106-302) re-routes every OOB sample once per
// used feature k, with x[pjoob[r]][k] in place of x[joob[r]][k], where pjoob is
// cpu_permobmr's permutation (:16-30; it depends on noob only).  A permuted walk
// can only leave the unpermuted path at a node that splits on k, so one walk
// along the unpermuted cpu_testreeimp path (:45-103) decides every feature at
// once: at each node on the path whose feature k has not yet diverged, the
// permuted value is tried; where it goes the other way, a side walk from the
// other child (with k permuted) gives that feature's class.  Features that
// never diverge keep the unpermuted class.  Per (tree, sample) this yields
//   bit "testreebag correct", bit "testreeimp correct", and a flip mask over
//   features, from which
//   rightimp[t][k] = #testreeimp-correct + sum of signed flips (exact integers).
//
// joob_kernel        - one CTA per tree: OOB list (joob, ascending), the
//                       permutation partners and, once member lists exist,
//                       the OOB samples in leaf order (oobord).
// varimp_walk_kernel - one thread per (tree, OOB sample) over the whole grid
//                       (in leaf order when oobord exists, so a warp's main
//                       paths coincide): walks, flip masks, per-tree integer
//                       counts.
// varimp_sample_kernel - one thread per (sample, 16 features): qimp / qimpm
//                       float sums in tree order, 1/noob per correct OOB
//                       tree (the reference adds each tree's temporaries in
//                       tree order, src/rf_random_forest.cpp:1217-1230).
//                       Its other launch shape, oob_trees_kernel +
//                       varimp_sample_oob_kernel, visits only each sample's
//                       OOB trees, from per-sample lists, in the same order.
// varimp_feature_kernel - one thread per feature: avimp / sqsd sums of
//                       rr = (right - rightimp) / noob in tree order.
#include "walks.cuh"

#include <algorithm>

namespace rfx {

namespace {

constexpr int VT = 256;  // threads of the per-tree OOB-list kernel

enum { DIR_BREAK = -2 };

// A sample's feature row for the walks: staged in shared memory (SX) or read
// from global memory through the read-only cache.
template <bool SX>
struct RowSel {
    const float* g;
    const float* s;
    __device__ __forceinline__ float operator()(int m) const { return SX ? s[m] : __ldg(g + m); }
};

// One decision of the cpu_testreeimp walk at node nd (local id kt) for value x.
__device__ __forceinline__ int imp_decide(const DNode& nd, int kt, float x, const int32_t* __restrict__ cgl,
                                          int maxcat) {
    if (!node_cat(nd.meta)) return (x <= nd.split) ? nd.left : nd.right;
    const int jcat = __float2int_rz(__fadd_rn(x, 0.5f));
    if (jcat >= 0 && jcat < maxcat) return (cgl_at(cgl, maxcat, kt, jcat) == 1) ? nd.left : nd.right;
    return DIR_BREAK;
}

// Side walk of the permuted traversal from node kt with feature mr taken from
// xperm; budget = remaining loop iterations of the reference's k < nnode loop.
// Returns the class, or -1 when the reference would break without assigning.
template <typename Src, typename XR>
__device__ __forceinline__ int imp_side_walk(const XR& xrow, const XR& xperm, int mr, int p, int kt, int budget,
                                             const Src& nodes, const int32_t* __restrict__ nclass_of,
                                             const int32_t* __restrict__ cgl, int maxcat) {
    for (int s = 0; s < budget; ++s) {
        const DNode nd = nodes(kt);
        if (node_status(nd.meta) == -1) return __ldg(nclass_of + kt);
        const int m = node_var(nd.meta);
        if (m >= p) return -1;
        const float x = m == mr ? xperm(m) : xrow(m);
        const int nx = imp_decide(nd, kt, x, cgl, maxcat);
        if (nx == DIR_BREAK) return -1;
        kt = nx;
    }
    return -1;
}

// The same side walk with both children of each split node loaded together
// with the feature value (walks.cuh, load_node_now): one round trip to memory
// per step.  Children of nodes with status != -1 are in [0, nnode) (checked
// at load), so the loads stay in bounds.
template <typename XR>
__device__ __forceinline__ int imp_side_walk_pf(const XR& xrow, const XR& xperm, int mr, int p, int kt, int budget,
                                                const DNode* __restrict__ tn, const int32_t* __restrict__ nclass_of,
                                                const int32_t* __restrict__ cgl, int maxcat) {
    if (budget <= 0) return -1;
    DNode nd = load_node_now(tn, kt);
    for (int s = 0; s < budget; ++s) {
        if (node_status(nd.meta) == -1) return __ldg(nclass_of + kt);
        const int m = node_var(nd.meta);
        if (m >= p) return -1;
        const DNode cl = load_node_now(tn, nd.left);
        const DNode cr = load_node_now(tn, nd.right);
        const float x = m == mr ? xperm(m) : xrow(m);
        const int nx = imp_decide(nd, kt, x, cgl, maxcat);
        if (nx == DIR_BREAK) return -1;
        nd = nx == nd.left ? cl : cr;
        kt = nx;
    }
    return -1;
}

// OOB samples of every tree in ascending order (joob of cpu_varimp).
__global__ void __launch_bounds__(VT)
joob_kernel(const uint8_t* __restrict__ inbag, int n, int32_t* __restrict__ joob_all,
            const int32_t* __restrict__ permoff, const int32_t* __restrict__ perm_all,
            int32_t* __restrict__ partner_all, const int32_t* __restrict__ memb = nullptr,
            int32_t* __restrict__ oobord = nullptr) {
    __shared__ int wsum[VT / 32];
    __shared__ int s_base;
    const int t = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const uint8_t* ib = inbag + (size_t)t * n;
    int32_t* joob = joob_all + (size_t)t * n;
    if (tid == 0) s_base = 0;
    __syncthreads();
    // JB consecutive samples per thread (their flag loads in flight
    // together), JB * VT samples per round
    constexpr int JB = 4;
    for (int base = 0; base < n; base += JB * VT) {
        const int i0 = base + JB * tid;
        unsigned fl = 0;
#pragma unroll
        for (int u = 0; u < JB; ++u)
            if (i0 + u < n && ib[i0 + u] == 0) fl |= 1u << u;
        const int cnt = __popc(fl);
        int incl = cnt;  // inclusive warp scan of the per-thread counts
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += v;
        }
        if (lane == 31) wsum[wid] = incl;
        __syncthreads();
        int woff = 0, tot = 0;
        for (int q = 0; q < VT / 32; ++q) {
            if (q < wid) woff += wsum[q];
            tot += wsum[q];
        }
        int pos = s_base + woff + incl - cnt;
#pragma unroll
        for (int u = 0; u < JB; ++u)
            if ((fl >> u) & 1u) joob[pos++] = i0 + u;
        __syncthreads();
        if (tid == 0) s_base += tot;
        __syncthreads();
    }
    if (!partner_all) return;
    // the permutation partner of every OOB sample, indexed by sample:
    // partner[joob[r]] = joob[perm[r]] (cpu_permobmr's swap order)
    const int noob = s_base;
    const int32_t* perm = perm_all + permoff[t];
    int32_t* partner = partner_all + (size_t)t * n;
    for (int r = tid; r < noob; r += VT) partner[joob[r]] = joob[__ldg(perm + r)];
    if (!memb) return;
    // the OOB samples in member-list order (by leaf): the walk's thread order
    const int32_t* mt = memb + (size_t)t * n;
    int32_t* ord = oobord + (size_t)t * n;
    __syncthreads();
    if (tid == 0) s_base = 0;
    __syncthreads();
    for (int base = 0; base < n; base += JB * VT) {
        const int q0 = base + JB * tid;
        int mv[JB];
        unsigned fl = 0;
#pragma unroll
        for (int u = 0; u < JB; ++u) {
            mv[u] = q0 + u < n ? __ldg(mt + q0 + u) : 0;
            if (q0 + u < n && ib[mv[u]] == 0) fl |= 1u << u;
        }
        const int cnt = __popc(fl);
        int incl = cnt;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += v;
        }
        if (lane == 31) wsum[wid] = incl;
        __syncthreads();
        int woff = 0, tot = 0;
        for (int q = 0; q < VT / 32; ++q) {
            if (q < wid) woff += wsum[q];
            tot += wsum[q];
        }
        int pos = s_base + woff + incl - cnt;
#pragma unroll
        for (int u = 0; u < JB; ++u)
            if ((fl >> u) & 1u) ord[pos++] = mv[u];
        __syncthreads();
        if (tid == 0) s_base += tot;
        __syncthreads();
    }
}

// One thread per (tree, OOB position r): grid = (ceil(max noob / VW), T),
// VW threads per CTA (a launch shape the autotuner picks: 64, 128 or 256).
// With FB (more than 64 W features) one launch decides the features of one
// block [fb, fb + 64 W): flip bits and delta counters are block-local, other
// features' splits are followed without a permuted decision, and the per-tree
// correct counts are added by the fb == 0 launch only.  With PF the main
// path and the side walks load both children of each split node with the
// feature values (one round trip to memory per step).
template <int W, int VW, bool FB = false, bool SX = false, bool PF = false>
__global__ void __launch_bounds__(VW, (PF ? 1024 : 1536) / VW)  // PF: room for the children's registers
varimp_walk_kernel(const float* __restrict__ X, const int32_t* __restrict__ y, int n, int p,
                   const DNode* __restrict__ nodes, const int32_t* __restrict__ nodeclass,
                   const int64_t* __restrict__ offs, const int32_t* __restrict__ nnode_arr,
                   const int32_t* __restrict__ noob_arr, const int32_t* __restrict__ cat,
                   const int32_t* __restrict__ catgoleft, int maxcat, const int32_t* __restrict__ permoff,
                   const int32_t* __restrict__ perm_all, const int32_t* __restrict__ joob_all,
                   const int32_t* __restrict__ oobord, const int32_t* __restrict__ partner_all,
                   const uint8_t* __restrict__ inbag, uint8_t* __restrict__ vflags, uint64_t* __restrict__ flips,
                   int32_t* __restrict__ counts, int32_t* __restrict__ delta_out, uint32_t* __restrict__ err,
                   int fb) {
    extern __shared__ int32_t delta[];  // pw counters (the features of this launch), then with SX the
                                        // staged feature rows: VW own rows and VW partner rows of p | 1 floats
    __shared__ int s_red[2];
    // Side walks found along the main paths are queued and then shared out
    // over the whole CTA, so a thread with many of them does not hold its
    // warp: {thread, feature, start node, step budget}.
    constexpr int QCAP = VW * 6;
    __shared__ int4 q_ent[QCAP];
    __shared__ int q_n;
    __shared__ unsigned long long s_pcorr[VW][W];
    __shared__ int s_i[VW], s_ip[VW], s_y[VW];
    const int t = blockIdx.y;
    const int noob = noob_arr[t];
    const int r0 = blockIdx.x * VW;
    const int tid = threadIdx.x, lane = tid & 31;
    // This thread's OOB sample i and its permutation partner ip.  With the
    // OOB samples in leaf order (oobord != null: the member lists' order, in
    // the bag dropped) neighbouring threads share their main path.  Otherwise
    // thread r takes joob position r.
    int i = 0, ip = 0;
    bool active;
    if (oobord) {
        if (r0 >= noob) return;
        active = r0 + tid < noob;
        if (active) {
            i = __ldg(oobord + (size_t)t * n + r0 + tid);
            ip = __ldg(partner_all + (size_t)t * n + i);
        }
    } else {
        if (r0 >= noob) return;
        active = r0 + tid < noob;
        if (active) {
            const int32_t* joob = joob_all + (size_t)t * n;
            i = joob[r0 + tid];
            ip = joob[__ldg(perm_all + permoff[t] + r0 + tid)];
        }
    }
    const int pw = FB ? min(64 * W, p - fb) : p;
    for (int k = tid; k < pw; k += VW) delta[k] = 0;
    // with SX: every warp stages its lanes' own and partner rows (one row at
    // a time across the lanes), so each walk step reads features from shared
    // memory; without it the rows are read through the read-only cache
    const int ps = p | 1;
    float* xs_own = reinterpret_cast<float*>(delta + ((pw + 3) & ~3));
    float* xs_par = xs_own + (size_t)VW * ps;
    if (SX) {
        const int w = tid >> 5;
        stage_warp_rows(xs_own + (size_t)(w * 32) * ps, ps, X, p, active ? i : -1, lane);
        stage_warp_rows(xs_par + (size_t)(w * 32) * ps, ps, X, p, active ? ip : -1, lane);
    }
    if (tid == 0) {
        s_red[0] = 0;
        s_red[1] = 0;
        q_n = 0;
    }
#pragma unroll
    for (int q = 0; q < W; ++q) s_pcorr[tid][q] = 0ull;
    __syncthreads();
    const int64_t o = offs[t];
    const DNode* tn = nodes + o;
    const int32_t* tc = nodeclass + o;
    const int32_t* cgl = catgoleft ? catgoleft + o * maxcat : nullptr;
    const int nn = nnode_arr[t];
    const int nnv = nn > 0 ? nn : 1;
    const GlobalNodes src{tn};
    int my_right = 0, my_imp = 0;
    uint32_t my_err = 0;
    uint64_t done[W], pcorr[W];
#pragma unroll
    for (int q = 0; q < W; ++q) done[q] = pcorr[q] = 0ull;
    int yi = -1, base_tb = 0, base_imp = 0;
    if (active) {
        s_i[tid] = i;
        s_ip[tid] = ip;
        const RowSel<SX> xi{X + (size_t)i * p, xs_own + (size_t)tid * ps};
        const RowSel<SX> xp{X + (size_t)ip * p, xs_par + (size_t)tid * ps};
        yi = y[i];
        s_y[tid] = yi;
        // The cpu_testreebag walk of the same sample follows the main path
        // below node by node until the two rules disagree (categorical
        // conventions, unsplit nodes, the step guard); it is decided along
        // the way and walked on its own only when the paths part.
        int cls_tb = -1;
        bool tb_done = false, tb_sync = true;
        int tb_steps = 0;
        int kt = 0, jvr0 = -1;
        bool ok = false;
        DNode nd_next;
        if constexpr (PF) nd_next = load_node_now(tn, 0);
        for (int step = 0; step < nnv; ++step) {
            const DNode nd = PF ? nd_next : src(kt);
            const int st = node_status(nd.meta);
            const int m = node_var(nd.meta);
            if (tb_sync && !tb_done) {
                if (st != 1) {
                    cls_tb = (st == -1 || st == 2) ? __ldg(tc + kt) : __ldg(tc);
                    tb_done = true;
                } else if (++tb_steps >= 1000 || m >= p) {
                    cls_tb = __ldg(tc);
                    tb_done = true;
                }
            }
            if (st == -1) {
                jvr0 = __ldg(tc + kt);
                ok = true;
                break;
            }
            if (m >= p) break;
            DNode cl, cr;
            if constexpr (PF) {
                cl = load_node_now(tn, nd.left);
                cr = load_node_now(tn, nd.right);
            }
            const float xv = xi(m);
            const int dir_o = imp_decide(nd, kt, xv, cgl, maxcat);
            if (tb_sync && !tb_done) {
                int tb_next;
                if (!node_cat(nd.meta)) {
                    tb_next = dir_o;  // numeric splits: the same comparison
                } else {
                    const int iv = __float2int_rz(xv);
                    tb_next = (iv >= 0 && iv < __ldg(cat + m))
                                  ? ((cgl_at(cgl, maxcat, kt, iv) == 1) ? nd.left : nd.right)
                                  : nd.right;
                }
                if (tb_next < 0 || tb_next >= nn) {
                    cls_tb = __ldg(tc);  // out-of-range child: the root's class
                    tb_done = true;
                } else if (tb_next != dir_o) {
                    tb_sync = false;  // the walks part: cpu_testreebag is walked on its own below
                }
            }
            if (dir_o == DIR_BREAK) break;
            const int mm = FB ? m - fb : m;  // the feature's bit within this launch's block
            const int wq = mm >> 6;
            const uint64_t bit = 1ull << (mm & 63);
            uint64_t dword = 0;
#pragma unroll
            for (int q = 0; q < W; ++q)
                if (q == wq) dword = done[q];
            if ((!FB || (unsigned)mm < (unsigned)(64 * W)) && !(dword & bit)) {
                const int dir_p = imp_decide(nd, kt, xp(m), cgl, maxcat);
                if (dir_p != dir_o) {
                    int cls_m = -2;  // -2: queued, decided in the shared phase
                    if (dir_p == DIR_BREAK) {
                        cls_m = -1;
                    } else {
                        const int slot = atomicAdd(&q_n, 1);
                        if (slot < QCAP)
                            q_ent[slot] = make_int4(tid, m, dir_p, nnv - step - 1);
                        else if constexpr (PF)
                            cls_m = imp_side_walk_pf(xi, xp, m, p, dir_p, nnv - step - 1, tn, tc, cgl, maxcat);
                        else
                            cls_m = imp_side_walk(xi, xp, m, p, dir_p, nnv - step - 1, src, tc, cgl, maxcat);
                    }
                    if (cls_m == -1) my_err |= ERR_STALE_JVR;
#pragma unroll
                    for (int q = 0; q < W; ++q)
                        if (q == wq) {
                            done[q] |= bit;
                            if (cls_m == yi) pcorr[q] |= bit;
                        }
                }
            }
            if constexpr (PF) nd_next = dir_o == nd.left ? cl : cr;
            kt = dir_o;
        }
        if (!ok) my_err |= ERR_STALE_JVR;
        if (!tb_done) walk_testreebag_x(xi, p, src, tc, nn, cat, cgl, maxcat, &cls_tb);
        base_tb = (cls_tb == yi);
        base_imp = (ok && jvr0 == yi);
    }
    __syncthreads();
    // shared phase: every queued side walk, spread over the CTA's threads
    const int qn = min(q_n, QCAP);
    for (int e = tid; e < qn; e += VW) {
        const int4 en = q_ent[e];
        const int lt = en.x, m = en.y;
        const RowSel<SX> xo{X + (size_t)s_i[lt] * p, xs_own + (size_t)lt * ps};
        const RowSel<SX> xq{X + (size_t)s_ip[lt] * p, xs_par + (size_t)lt * ps};
        int cls_m;
        if constexpr (PF) cls_m = imp_side_walk_pf(xo, xq, m, p, en.z, en.w, tn, tc, cgl, maxcat);
        else cls_m = imp_side_walk(xo, xq, m, p, en.z, en.w, src, tc, cgl, maxcat);
        if (cls_m < 0) my_err |= ERR_STALE_JVR;
        const int mb = FB ? m - fb : m;
        if (cls_m >= 0 && cls_m == s_y[lt]) atomicOr(&s_pcorr[lt][mb >> 6], 1ull << (mb & 63));
    }
    __syncthreads();
    if (active) {
#pragma unroll
        for (int q = 0; q < W; ++q) pcorr[q] |= s_pcorr[tid][q];
        const uint64_t bmask = base_imp ? ~0ull : 0ull;
        const size_t ti = (size_t)t * n + i;
        vflags[ti] = (uint8_t)(1 | (base_tb << 1) | (base_imp << 2));
#pragma unroll
        for (int q = 0; q < W; ++q) {
            const uint64_t fl = done[q] & (pcorr[q] ^ bmask);
            flips[ti * W + q] = fl;
            uint64_t f = fl;
            while (f) {
                const int b = __ffsll((long long)f) - 1;
                f &= f - 1;
                atomicAdd(delta + q * 64 + b, base_imp ? -1 : 1);
            }
        }
        my_right = base_tb;
        my_imp = base_imp;
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        my_right += __shfl_down_sync(0xffffffffu, my_right, d);
        my_imp += __shfl_down_sync(0xffffffffu, my_imp, d);
    }
    if (lane == 0) {
        atomicAdd(&s_red[0], my_right);
        atomicAdd(&s_red[1], my_imp);
    }
    if (my_err) atomicOr(err, my_err);
    __syncthreads();
    if (tid == 0 && (!FB || fb == 0)) {
        if (s_red[0]) atomicAdd(counts + 2 * t, s_red[0]);
        if (s_red[1]) atomicAdd(counts + 2 * t + 1, s_red[1]);
    }
    for (int k = tid; k < pw; k += VW)
        if (delta[k]) atomicAdd(delta_out + (size_t)t * p + fb + k, delta[k]);
}

// qimp / qimpm: one thread per (sample, group of VS_FEAT features); each thread
// keeps its running sums in registers and walks the trees in order, adding
// 1/noob for every OOB tree where the feature's permuted vote is correct
// (group 0 also sums qimp from the testreebag votes).  The float sums follow
// the reference's tree order exactly.  One launch covers the pw features
// [fb, fb + pw) whose flip bits the walk wrote (fb = 0 and pw = p unless the
// features come in blocks); iv rows are ivw words long.
constexpr int VS_FEAT = 16;  // features per thread (a group never straddles a 64-bit word)

template <int W>
__global__ void __launch_bounds__(256, 3)
varimp_sample_kernel(const uint8_t* __restrict__ inbag, const uint8_t* __restrict__ vflags,
                     const uint64_t* __restrict__ flips, const uint64_t* __restrict__ iv,
                     const float* __restrict__ invnoob, int n, int p, int T, float* __restrict__ qimp,
                     float* __restrict__ qimpm, int fb, int pw, int ivw) {
    const int G = (pw + VS_FEAT - 1) / VS_FEAT;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)n * G) return;
    const int i = (int)(idx / G);
    const int g = (int)(idx % G);
    const int kl = g * VS_FEAT;  // first feature of the group within the block
    const int k0 = fb + kl;
    const int wq = kl >> 6, sh = kl & 63;  // groups never straddle a 64-bit word
    const int iq = k0 >> 6;                // the group's word of the iv row
    float acc[VS_FEAT];
#pragma unroll
    for (int u = 0; u < VS_FEAT; ++u) acc[u] = 0.0f;
    float q = 0.0f;
    // trees in blocks of TB: all loads of a block are issued before its sums
    // (the flip words of in-bag units are read but not used), then the sums
    // are added in tree order
    constexpr int TB = 8;
    int t0 = 0;
    for (; t0 + TB <= T; t0 += TB) {
        uint8_t ib[TB], fl[TB];
        float inv[TB];
        uint64_t fw[TB], ivv[TB];
#pragma unroll
        for (int u = 0; u < TB; ++u) {
            const size_t ti = (size_t)(t0 + u) * n + i;
            ib[u] = __ldg(inbag + ti);
            fl[u] = __ldg(vflags + ti);
            inv[u] = __ldg(invnoob + t0 + u);
            fw[u] = __ldg(flips + ti * W + wq);
            ivv[u] = __ldg(iv + (size_t)(t0 + u) * ivw + iq);
        }
#pragma unroll
        for (int u = 0; u < TB; ++u) {
            if (ib[u] != 0) continue;
            const bool btb = (fl[u] >> 1) & 1, bimp = (fl[u] >> 2) & 1;
            if (btb) q = __fadd_rn(q, inv[u]);
            const uint64_t corr = (ivv[u] & ((bimp ? ~0ull : 0ull) ^ fw[u])) | (~ivv[u] & (btb ? ~0ull : 0ull));
            const uint32_t cb = (uint32_t)(corr >> sh) & ((1u << VS_FEAT) - 1u);
#pragma unroll
            for (int v = 0; v < VS_FEAT; ++v)
                if ((cb >> v) & 1u) acc[v] = __fadd_rn(acc[v], inv[u]);
        }
    }
    for (int t = t0; t < T; ++t) {
        const size_t ti = (size_t)t * n + i;
        if (__ldg(inbag + ti) != 0) continue;
        const uint8_t fl = __ldg(vflags + ti);
        const float inv = __ldg(invnoob + t);
        const bool btb = (fl >> 1) & 1, bimp = (fl >> 2) & 1;
        if (btb) q = __fadd_rn(q, inv);
        const uint64_t fw = __ldg(flips + ti * W + wq);
        const uint64_t ivt = __ldg(iv + (size_t)t * ivw + iq);
        const uint64_t corr = (ivt & ((bimp ? ~0ull : 0ull) ^ fw)) | (~ivt & (btb ? ~0ull : 0ull));
        const uint32_t cb = (uint32_t)(corr >> sh) & ((1u << VS_FEAT) - 1u);
#pragma unroll
        for (int u = 0; u < VS_FEAT; ++u)
            if ((cb >> u) & 1u) acc[u] = __fadd_rn(acc[u], inv);
    }
    if (g == 0 && fb == 0) qimp[i] = q;
#pragma unroll
    for (int u = 0; u < VS_FEAT; ++u)
        if (kl + u < pw) qimpm[(size_t)i * p + k0 + u] = acc[u];
}

// The same sums from per-sample lists of OOB trees (the second launch shape
// of the stage).  oob_trees_kernel lists, for every sample, the trees where it
// is out of bag in ascending order (oobt[k * n + i] = k-th such tree, at most
// 65,535 trees); varimp_sample_oob_kernel then visits only those trees, so a
// thread does no work for its in-bag trees and the lanes of a warp do not wait
// on each other's OOB trees.  The sums still run in tree order.  The flip word
// and the used-feature mask are read as the 16-bit piece that holds the
// thread's sixteen features.
__global__ void __launch_bounds__(256)
oob_trees_kernel(const uint8_t* __restrict__ inbag, int n, int T, uint16_t* __restrict__ oobt,
                 int32_t* __restrict__ cnt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int k = 0;
    constexpr int TB = 16;
    int t0 = 0;
    for (; t0 + TB <= T; t0 += TB) {
        uint8_t b[TB];
#pragma unroll
        for (int u = 0; u < TB; ++u) b[u] = __ldg(inbag + (size_t)(t0 + u) * n + i);
#pragma unroll
        for (int u = 0; u < TB; ++u)
            if (b[u] == 0) oobt[(size_t)(k++) * n + i] = (uint16_t)(t0 + u);
    }
    for (int t = t0; t < T; ++t)
        if (__ldg(inbag + (size_t)t * n + i) == 0) oobt[(size_t)(k++) * n + i] = (uint16_t)t;
    cnt[i] = k;
}

template <int W>
__global__ void __launch_bounds__(256, 4)
varimp_sample_oob_kernel(const uint16_t* __restrict__ oobt, const int32_t* __restrict__ cnt,
                         const uint8_t* __restrict__ vflags, const uint64_t* __restrict__ flips,
                         const uint64_t* __restrict__ iv, const float* __restrict__ invnoob, int n, int p,
                         float* __restrict__ qimp, float* __restrict__ qimpm, int fb, int pw, int ivw) {
    const int G = (pw + VS_FEAT - 1) / VS_FEAT;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)n * G) return;
    const int i = (int)(idx / G);
    const int g = (int)(idx % G);
    const int kl = g * VS_FEAT;  // first feature of the group within the block
    const int k0 = fb + kl;
    const int wq = kl >> 6, sh = kl & 63;  // groups never straddle a 64-bit word
    const int iq = k0 >> 6;                // the group's word of the iv row
    const int pc = sh >> 4;                // the 16-bit piece of those words
    const uint16_t* fl16 = reinterpret_cast<const uint16_t*>(flips);
    const uint16_t* iv16 = reinterpret_cast<const uint16_t*>(iv);
    const int K = __ldg(cnt + i);
    float acc[VS_FEAT];
#pragma unroll
    for (int u = 0; u < VS_FEAT; ++u) acc[u] = 0.0f;
    float q = 0.0f;
    constexpr int TB = 4;
    // the next block's tree ids are loaded with the current block's data
    int tn[TB];
#pragma unroll
    for (int u = 0; u < TB; ++u) tn[u] = u < K ? (int)__ldg(oobt + (size_t)u * n + i) : -1;
    for (int kb = 0; kb < K; kb += TB) {
        int tt[TB];
#pragma unroll
        for (int u = 0; u < TB; ++u) {
            tt[u] = tn[u];
            const int kn = kb + TB + u;
            tn[u] = kn < K ? (int)__ldg(oobt + (size_t)kn * n + i) : -1;
        }
        uint8_t fl[TB];
        float inv[TB];
        uint32_t fw[TB], ivv[TB];
#pragma unroll
        for (int u = 0; u < TB; ++u) {
            const int t = tt[u] < 0 ? 0 : tt[u];
            const size_t ti = (size_t)t * n + i;
            fl[u] = tt[u] < 0 ? 0 : __ldg(vflags + ti);
            inv[u] = __ldg(invnoob + t);
            fw[u] = tt[u] < 0 ? 0u : __ldg(fl16 + ((ti * W + wq) << 2) + pc);
            ivv[u] = __ldg(iv16 + (((size_t)t * ivw + iq) << 2) + pc);
        }
#pragma unroll
        for (int u = 0; u < TB; ++u) {
            if (tt[u] < 0) break;
            const bool btb = (fl[u] >> 1) & 1, bimp = (fl[u] >> 2) & 1;
            if (btb) q = __fadd_rn(q, inv[u]);
            const uint32_t corr = (ivv[u] & ((bimp ? 0xffffu : 0u) ^ fw[u])) | (~ivv[u] & (btb ? 0xffffu : 0u));
#pragma unroll
            for (int v = 0; v < VS_FEAT; ++v)
                if ((corr >> v) & 1u) acc[v] = __fadd_rn(acc[v], inv[u]);
        }
    }
    if (g == 0 && fb == 0) qimp[i] = q;
#pragma unroll
    for (int u = 0; u < VS_FEAT; ++u)
        if (kl + u < pw) qimpm[(size_t)i * p + k0 + u] = acc[u];
}

// counts[2t] = #OOB correct by testreebag (right), counts[2t+1] = #OOB correct
// by the unpermuted testreeimp walk; rightimp[t][k] = counts[2t+1] + delta[t][k].
// One warp per feature: the lanes compute rr for 32 trees at once, then the
// sums are added in tree order through shuffles (the float order of the
// reference's per-tree accumulation).
__global__ void varimp_feature_kernel(const int32_t* __restrict__ counts, const int32_t* __restrict__ delta,
                                      const int32_t* __restrict__ noob, const uint64_t* __restrict__ iv, int W,
                                      int p, int T, float* __restrict__ avimp, float* __restrict__ sqsd) {
    const int k = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (k >= p) return;
    float a = 0.0f, s = 0.0f;
    for (int t0 = 0; t0 < T; t0 += 32) {
        const int t = t0 + lane;
        bool used = false;
        float rr = 0.0f, r2 = 0.0f;
        if (t < T) {
            used = (iv[(size_t)t * W + (k >> 6)] >> (k & 63)) & 1ull;
            if (used) {
                const int rightimp = counts[2 * t + 1] + delta[(size_t)t * p + k];
                rr = __fdiv_rn(__fsub_rn((float)counts[2 * t], (float)rightimp), (float)noob[t]);
                r2 = __fmul_rn(rr, rr);
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, used);
#pragma unroll 8
        for (int l = 0; l < 32; ++l) {
            const float x = __shfl_sync(0xffffffffu, rr, l);
            const float x2 = __shfl_sync(0xffffffffu, r2, l);
            if ((m >> l) & 1u) {
                a = __fadd_rn(a, x);
                s = __fadd_rn(s, x2);
            }
        }
    }
    if (lane == 0) {
        avimp[k] = a;
        sqsd[k] = s;
    }
}

__global__ void localimp_kernel(const float* __restrict__ qimp, const float* __restrict__ qimpm, int n, int p, int T,
                                float* __restrict__ out) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t)n * p) return;
    const int nn = (int)(idx % (size_t)n);
    out[idx] = __fdiv_rn(__fmul_rn(100.0f, __fsub_rn(qimp[nn], qimpm[idx])), (float)T);
}

template <int W>
rfx_status launch_varimp_w(Ctx* c, int impn) {
    const size_t smem = (size_t)c->p * sizeof(int32_t);
    {
        StageTimer st(c, ST_VARIMP_TREE, 2);
        const bool ordered = c->csr_built && c->d_partner;
        joob_kernel<<<c->T, VT, 0, c->stream>>>(c->d_inbag, c->n, c->d_joob, c->d_permoff, c->d_perm,
                                                ordered ? c->d_partner : nullptr, ordered ? c->d_memb : nullptr,
                                                c->d_oobord);
        RFX_CUDA(cudaGetLastError());
        int max_noob = 1;
        for (int t = 0; t < c->T; ++t) max_noob = std::max(max_noob, c->h_noob[t]);
        // staged shapes hold VW own rows and VW partner rows of p | 1 floats
        // after the counters (offset rounded to 16 bytes)
        const size_t cnt_bytes = sizeof(int32_t) * (((size_t)c->p + 3) & ~(size_t)3);
        auto staged_smem = [&](int vw) { return cnt_bytes + 2 * sizeof(float) * (size_t)vw * (size_t)(c->p | 1); };
        // the staged kernels may take up to the device maximum (set once, so a
        // captured launch of another forest's size stays valid)
        int dev_smem = 0;
        RFX_CUDA(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
        if (rfx_status s0 = allow_dyn_smem(varimp_walk_kernel<W, 64, false, true>, dev_smem)) return s0;
        if (rfx_status s0 = allow_dyn_smem(varimp_walk_kernel<W, 128, false, true>, dev_smem)) return s0;
        if (rfx_status s0 = allow_dyn_smem(varimp_walk_kernel<W, 256, false, true>, dev_smem)) return s0;
        auto go = [&](auto kernel, int vw, size_t sm) -> rfx_status {
            dim3 grid((max_noob + vw - 1) / vw, c->T);
            kernel<<<grid, vw, sm, c->stream>>>(c->d_X, c->d_y, c->n, c->p, c->d_nodes, c->d_nodeclass, c->d_offs,
                                                 c->d_nnode, c->d_noob, c->d_cat, c->d_catgoleft, c->maxcat,
                                                 c->d_permoff, c->d_perm, c->d_joob,
                                                 ordered ? c->d_oobord : nullptr, c->d_partner, c->d_inbag,
                                                 c->d_vflags, c->d_flips,
                                                 c->d_right, c->d_rightimp, c->d_err, 0);
            return RFX_OK;
        };
        // shapes 0-2: rows through the read-only cache at 64/128/256 threads;
        // 3-5: the same with staged rows, where they fit in 96 KB; 6-8: rows
        // through the read-only cache with child-prefetching walks
        rfx_status r = autotune(c, TK_VWALK, 9, 1, [&](int shape) -> rfx_status {
            // the walk adds to the per-tree counts: clear them for every run
            RFX_CUDA(cudaMemsetAsync(c->d_right, 0, sizeof(int32_t) * 2 * (size_t)c->T, c->stream));
            RFX_CUDA(cudaMemsetAsync(c->d_rightimp, 0, sizeof(int32_t) * (size_t)c->T * c->p, c->stream));
            const int vw = (shape % 3) == 0 ? 64 : (shape % 3) == 2 ? 256 : 128;
            const bool staged = shape >= 3 && shape <= 5 && staged_smem(vw) <= 96 * 1024;
            rfx_status g;
            if (shape >= 6) {
                g = vw == 64 ? go(varimp_walk_kernel<W, 64, false, false, true>, 64, smem)
                    : vw == 256 ? go(varimp_walk_kernel<W, 256, false, false, true>, 256, smem)
                                : go(varimp_walk_kernel<W, 128, false, false, true>, 128, smem);
            } else if (staged) {
                const size_t sm = staged_smem(vw);
                g = vw == 64 ? go(varimp_walk_kernel<W, 64, false, true>, 64, sm)
                    : vw == 256 ? go(varimp_walk_kernel<W, 256, false, true>, 256, sm)
                                : go(varimp_walk_kernel<W, 128, false, true>, 128, sm);
            } else {
                g = vw == 64 ? go(varimp_walk_kernel<W, 64>, 64, smem)
                    : vw == 256 ? go(varimp_walk_kernel<W, 256>, 256, smem)
                                : go(varimp_walk_kernel<W, 128>, 128, smem);
            }
            if (g != RFX_OK) return g;
            RFX_CUDA(cudaGetLastError());
            return RFX_OK;
        });
        if (r != RFX_OK) return r;
    }
    if (impn) {
        StageTimer st(c, ST_VARIMP_SAMPLE, 1);
        const long long G = (c->p + VS_FEAT - 1) / VS_FEAT;
        const long long threads = (long long)c->n * G;
        const unsigned blocks = (unsigned)((threads + 255) / 256);
        // shape 0: every thread loops over all trees; 1: over its sample's
        // OOB trees from per-sample lists (tree ids in 16 bits; the lists
        // live in per-call scratch, so a stream capture takes shape 0)
        const int nshape = c->T < 65536 ? 2 : 1;
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        RFX_CUDA(cudaStreamIsCapturing(c->stream, &cap));
        const bool capturing = cap != cudaStreamCaptureStatusNone;
        rfx_status r = autotune(c, TK_VSAMPLE, nshape, 0, [&](int shape) -> rfx_status {
            bool listed = false;
            if (shape == 1 && !capturing) {
                // (where the lists do not fit in device memory the tree loop runs)
                Scratch sc(c);
                uint16_t* oobt = sc.get<uint16_t>((size_t)c->T * c->n);
                int32_t* cnt = oobt ? sc.get<int32_t>((size_t)c->n) : nullptr;
                if (oobt && cnt) {
                    oob_trees_kernel<<<(c->n + 255) / 256, 256, 0, c->stream>>>(c->d_inbag, c->n, c->T, oobt, cnt);
                    RFX_CUDA(cudaGetLastError());
                    varimp_sample_oob_kernel<W><<<blocks, 256, 0, c->stream>>>(
                        oobt, cnt, c->d_vflags, c->d_flips, c->d_iv, c->d_invnoob, c->n, c->p, c->d_qimp,
                        c->d_qimpm, 0, c->p, W);
                    c->launches += 1;  // the list kernel (the stage counts one kernel)
                    listed = true;
                }
            }
            if (!listed) {
                varimp_sample_kernel<W><<<blocks, 256, 0, c->stream>>>(c->d_inbag, c->d_vflags, c->d_flips, c->d_iv,
                                                                       c->d_invnoob, c->n, c->p, c->T, c->d_qimp,
                                                                       c->d_qimpm, 0, c->p, W);
            }
            RFX_CUDA(cudaGetLastError());
            return RFX_OK;
        });
        if (r != RFX_OK) return r;
    }
    StageTimer st(c, ST_VARIMP_FEATURE, 1);
    varimp_feature_kernel<<<(c->p + 3) / 4, 128, 0, c->stream>>>(c->d_right, c->d_rightimp, c->d_noob, c->d_iv,
                                                                      W, c->p, c->T, c->d_avimp, c->d_sqsd);
    RFX_CUDA(cudaGetLastError());
    return RFX_OK;
}

// More than 256 features: the walk and the per-sample sums run once per block
// of 256 features (flip words and delta counters are per block; the flips
// buffer holds one block), then the per-feature sums once for all features.
// Launch shapes are the defaults (no tuning trials).
rfx_status launch_varimp_blocked(Ctx* c, int impn) {
    constexpr int W = VARIMP_BLOCK_WORDS, VW = 128, FW = 64 * W;
    {
        StageTimer st(c, ST_VARIMP_TREE, 1 + (impn ? 2 : 1) * ((c->p + FW - 1) / FW));
        const bool ordered = c->csr_built && c->d_partner;
        joob_kernel<<<c->T, VT, 0, c->stream>>>(c->d_inbag, c->n, c->d_joob, c->d_permoff, c->d_perm,
                                                ordered ? c->d_partner : nullptr, ordered ? c->d_memb : nullptr,
                                                c->d_oobord);
        RFX_CUDA(cudaGetLastError());
        int max_noob = 1;
        for (int t = 0; t < c->T; ++t) max_noob = std::max(max_noob, c->h_noob[t]);
        RFX_CUDA(cudaMemsetAsync(c->d_right, 0, sizeof(int32_t) * 2 * (size_t)c->T, c->stream));
        RFX_CUDA(cudaMemsetAsync(c->d_rightimp, 0, sizeof(int32_t) * (size_t)c->T * c->p, c->stream));
        const dim3 grid((max_noob + VW - 1) / VW, c->T);
        for (int fb = 0; fb < c->p; fb += FW) {
            const int pw = std::min(FW, c->p - fb);
            varimp_walk_kernel<W, VW, true><<<grid, VW, sizeof(int32_t) * pw, c->stream>>>(
                c->d_X, c->d_y, c->n, c->p, c->d_nodes, c->d_nodeclass, c->d_offs, c->d_nnode, c->d_noob, c->d_cat,
                c->d_catgoleft, c->maxcat, c->d_permoff, c->d_perm, c->d_joob, ordered ? c->d_oobord : nullptr,
                c->d_partner, c->d_inbag, c->d_vflags, c->d_flips, c->d_right, c->d_rightimp, c->d_err, fb);
            RFX_CUDA(cudaGetLastError());
            if (impn) {
                const long long threads = (long long)c->n * ((pw + VS_FEAT - 1) / VS_FEAT);
                varimp_sample_kernel<W><<<(unsigned)((threads + 255) / 256), 256, 0, c->stream>>>(
                    c->d_inbag, c->d_vflags, c->d_flips, c->d_iv, c->d_invnoob, c->n, c->p, c->T, c->d_qimp,
                    c->d_qimpm, fb, pw, c->iv_words);
                RFX_CUDA(cudaGetLastError());
            }
        }
    }
    StageTimer st(c, ST_VARIMP_FEATURE, 1);
    varimp_feature_kernel<<<(c->p + 3) / 4, 128, 0, c->stream>>>(c->d_right, c->d_rightimp, c->d_noob, c->d_iv,
                                                                      c->iv_words, c->p, c->T, c->d_avimp, c->d_sqsd);
    RFX_CUDA(cudaGetLastError());
    return RFX_OK;
}

}  // namespace

// OOB lists and permutation partners of every tree (case-wise importance).
rfx_status launch_joob_partner(Ctx* c) {
    joob_kernel<<<c->T, VT, 0, c->stream>>>(c->d_inbag, c->n, c->d_joob, c->d_permoff, c->d_perm, c->d_partner);
    RFX_CUDA(cudaGetLastError());
    c->launches += 1;
    return RFX_OK;
}

rfx_status launch_varimp(Ctx* c, int impn) {
    switch (c->iv_words) {
        case 1: return launch_varimp_w<1>(c, impn);
        case 2: return launch_varimp_w<2>(c, impn);
        case 3: return launch_varimp_w<3>(c, impn);
        case 4: return launch_varimp_w<4>(c, impn);
        default: return launch_varimp_blocked(c, impn);
    }
}

rfx_status launch_localimp(Ctx* c, const float* d_qimp, const float* d_qimpm, float* d_out) {
    StageTimer st(c, ST_LOCALIMP, 1);
    const size_t total = (size_t)c->n * c->p;
    localimp_kernel<<<(unsigned)((total + 255) / 256), 256, 0, c->stream>>>(d_qimp, d_qimpm, c->n, c->p, c->T, d_out);
    RFX_CUDA(cudaGetLastError());
    return RFX_OK;
}

}  // namespace rfx
