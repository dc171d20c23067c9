// Exact proximity pair counts.
//
// Per tree t, the samples of every terminal node ("leaf") are split into an
// out-of-bag list and an in-bag list.  cpu_proximity's dense branch
// (src/rf_proximity.cpp:173-230) adds 1 to C[i][j] for every OOB i and in-bag j
// of the same leaf.  Here S = C + C^T is produced directly in its packed
// upper-triangle form.
//
// Stage 1 (build_csr_kernel, one CTA per tree): a stable counting sort of the
//   tree's samples by key = 2*leaf + inbag.  seg[t][k] .. seg[t][k+1] is the
//   member range of key k in memb[t*n ...], members ascending by sample id.
//   The CTA counts and scans the keys; a single warp then places the samples
//   in index order, so equal keys keep index order.
// Stage 2, row-owner: one CTA owns row i of S; for every tree it takes, in the
//   member list of the opposite bag status of i's leaf, the members j > i and
//   adds 1 to a shared-memory counter per member; the accumulated row is then
//   written once, coalesced.  Work is proportional to the pair updates, and S
//   is written exactly once.  The full-row form (opp_kernel, row_order_kernel,
//   pairs_row16_kernel: u16 counters for the whole row) is used when a row of
//   counters fits in shared memory and ntree < 65536; otherwise the windowed
//   form (pairs_row_kernel: u32 counters over a column window, binary searches
//   per window) runs.
#include "rfx_internal.cuh"

#include <algorithm>
#include <cstdlib>
#include <string>

namespace rfx {

namespace {

// ---------------------------------------------------------------------------
// Stage 1
// ---------------------------------------------------------------------------
constexpr int CSR_THREADS = 128;
constexpr int CSR_PREFETCH = 16;  // 32-sample groups loaded ahead by the scattering warp

// Key counters of the CSR build: in shared memory as CT (16-bit when every
// count and offset stays below 65536, so twice as many trees fit per SM), or
// the tree's own 32-bit segment-offset table in global memory.
template <typename CT>
struct CsrCounters {
    CT* s;
    int32_t* g;
    bool sm;
    __device__ __forceinline__ int get(int k) const { return sm ? (int)s[k] : g[k]; }
    __device__ __forceinline__ void set(int k, int v) {
        if (sm) s[k] = (CT)v;
        else g[k] = v;
    }
    __device__ __forceinline__ void inc(int k) {
        if (!sm) atomicAdd(g + k, 1);
        else if (sizeof(CT) == 2) atomicAdd(reinterpret_cast<unsigned int*>(s) + (k >> 1), 1u << ((k & 1) << 4));
        else atomicAdd(reinterpret_cast<int*>(s) + k, 1);
    }
};

// One CTA per tree.  All warps build the key histogram; the exclusive scan
// runs over four quarters in parallel; warp 0 alone then scatters the samples
// in index order (equal keys inside a 32-sample group are ranked by lane), so
// every key's member list is ascending by sample id.
template <typename CT>
__global__ void __launch_bounds__(CSR_THREADS)
build_csr_kernel(const int32_t* __restrict__ key, int n, const int64_t* __restrict__ segbase,
                 int32_t* __restrict__ segoff, int32_t* __restrict__ memb, int smem_keys,
                 uint32_t* __restrict__ err) {
    extern __shared__ int32_t cnt[];
    __shared__ int qtot[CSR_THREADS / 32];
    const int t = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int64_t sb = segbase[t];
    const int K = (int)(segbase[t + 1] - sb) - 1;  // number of keys of this tree
    const int32_t* kt = key + (size_t)t * n;
    int32_t* mt = memb + (size_t)t * n;
    int32_t* so = segoff + sb;
    // counters: shared memory when the key table fits, else the tree's own
    // segment-offset table in global memory (slower, still exact)
    const bool use_smem = K + 1 <= smem_keys;
    CsrCounters<CT> ctr{reinterpret_cast<CT*>(cnt), so, use_smem};
    for (int k = tid; k <= K; k += CSR_THREADS) ctr.set(k, 0);
    if (use_smem && sizeof(CT) == 2 && tid == 0) ctr.s[K + 1] = 0;  // the other half of the last counter word
    __syncthreads();
    // samples without a terminal node (key -1) go to the slot after the
    // last key, so they follow every key's members (segoff[K] still marks
    // the end of the keyed members)
    for (int i = tid; i < n; i += CSR_THREADS) {
        const int k = __ldg(kt + i);
        ctr.inc(k >= 0 ? k : K);
    }
    __syncthreads();
    // exclusive scan of K+1 counters: quarter q = [q*Q, min((q+1)*Q, K+1))
    const int Q = (K + 1 + 3) / 4;
    const int q0 = w * Q, q1 = min(K + 1, q0 + Q);
    int carry = 0;
    for (int k0 = q0; k0 < q1; k0 += 32) {
        const int k = k0 + lane;
        const int v = k < q1 ? ctr.get(k) : 0;
        int incl = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += u;
        }
        if (k < q1) ctr.set(k, carry + incl - v);
        carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) qtot[w] = carry;
    __syncthreads();
    int qoff = 0;
    for (int q = 0; q < w; ++q) qoff += qtot[q];
    for (int k = q0 + lane; k < q1; k += 32) {
        const int v = ctr.get(k) + qoff;
        ctr.set(k, v);
        if (use_smem) so[k] = v;
    }
    __syncthreads();
    if (w != 0) return;
    // stable scatter by one warp, samples in index order; the next batch of
    // keys is loaded while the current one is placed
    int kv[CSR_PREFETCH], kn[CSR_PREFETCH];
    // slot per sample: its key, K for key -1, -1 past the end
#pragma unroll
    for (int u = 0; u < CSR_PREFETCH; ++u) {
        const int i = u * 32 + lane;
        const int k = i < n ? __ldg(kt + i) : 0;
        kv[u] = i < n ? (k >= 0 ? k : K) : -1;
    }
    for (int base = 0; base < n; base += 32 * CSR_PREFETCH) {
        const int nb = base + 32 * CSR_PREFETCH;
#pragma unroll
        for (int u = 0; u < CSR_PREFETCH; ++u) {
            const int i = nb + u * 32 + lane;
            const int k = i < n ? __ldg(kt + i) : 0;
            kn[u] = i < n ? (k >= 0 ? k : K) : -1;
        }
#pragma unroll
        for (int u = 0; u < CSR_PREFETCH; ++u) {
            const int i = base + u * 32 + lane;
            const int k = kv[u];
            const unsigned grp = __match_any_sync(0xffffffffu, k);
            const int leader = __ffs(grp) - 1;
            const int rank = __popc(grp & ((1u << lane) - 1u));
            int start = 0;
            if (k >= 0 && lane == leader) {
                start = ctr.get(k);
                ctr.set(k, start + __popc(grp));
            }
            start = __shfl_sync(0xffffffffu, start, leader);
            if (k >= 0) mt[start + rank] = i;
            __syncwarp();
        }
#pragma unroll
        for (int u = 0; u < CSR_PREFETCH; ++u) kv[u] = kn[u];
    }
    // global-counter path: the counters now hold segment ends; a follow-up
    // kernel (fix_global_segoff_kernel) turns them back into starts
}

// Fallback pass for trees whose key table did not fit in shared memory:
// rebuild segment starts from the ends left by the scatter (start[k] = end[k-1]).
__global__ void fix_global_segoff_kernel(const int64_t* __restrict__ segbase, int32_t* __restrict__ segoff,
                                         int smem_keys) {
    const int t = blockIdx.x;
    const int64_t sb = segbase[t];
    const int K = (int)(segbase[t + 1] - sb) - 1;
    if (K + 1 <= smem_keys) return;
    if (threadIdx.x != 0) return;
    int32_t* so = segoff + sb;
    for (int k = K; k >= 1; --k) so[k] = so[k - 1];
    so[0] = 0;
}

// ---------------------------------------------------------------------------
// Stage 2
// ---------------------------------------------------------------------------
constexpr int ROW_THREADS = 512;
constexpr int ROW_WARPS = ROW_THREADS / 32;

__device__ __forceinline__ int lower_bound_i32(const int32_t* __restrict__ a, int lo, int hi, int v) {
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(a + mid) < v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(ROW_THREADS)
pairs_row_kernel(const int32_t* __restrict__ key, const int32_t* __restrict__ segoff,
                 const int64_t* __restrict__ segbase, const int32_t* __restrict__ memb, int n, int T,
                 int win, int32_t* __restrict__ S, unsigned long long* __restrict__ pairs) {
    extern __shared__ uint32_t acc[];
    __shared__ int pref[ROW_WARPS][33];
    __shared__ long long segb[ROW_WARPS][32];
    const int i = blockIdx.x;
    const int c0 = blockIdx.y * win;
    if (c0 >= n) return;
    const int c1 = min(n, c0 + win);
    if (c1 <= i) return;  // window entirely left of the diagonal
    const int lo_col = max(i + 1, c0);
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int width = c1 - c0;
    for (int k = tid; k < width; k += ROW_THREADS) acc[k] = 0u;
    __syncthreads();
    unsigned long long my_pairs = 0;
    for (int t0 = w * 32; t0 < T; t0 += ROW_WARPS * 32) {
        const int t = t0 + lane;
        long long b = 0;
        int len = 0;
        if (t < T && lo_col < c1) {
            const int k = __ldg(key + (size_t)t * n + i);
            if (k >= 0) {
                const int ok = k ^ 1;  // the opposite bag status in the same leaf
                const int32_t* so = segoff + segbase[t];
                const int s0 = __ldg(so + ok), s1 = __ldg(so + ok + 1);
                const int32_t* mt = memb + (size_t)t * n;
                int bb = s0, ee = s1;
                if (s1 > s0) {
                    bb = lower_bound_i32(mt, s0, s1, lo_col);
                    ee = (c1 >= n) ? s1 : lower_bound_i32(mt, bb, s1, c1);
                }
                b = (long long)t * n + bb;  // absolute index into memb
                len = ee - bb;
            }
        }
        // warp-level load-balanced expansion of the 32 member ranges
        int incl = len;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            int u = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += u;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        pref[w][lane + 1] = incl;
        if (lane == 0) pref[w][0] = 0;
        segb[w][lane] = b;
        __syncwarp();
        for (int pos = lane; pos < total; pos += 32) {
            // find the range s with pref[s] <= pos < pref[s+1]
            int lo = 0, hi = 32;
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (pref[w][mid] <= pos) lo = mid;
                else hi = mid;
            }
            const int j = __ldg(memb + (size_t)segb[w][lo] + (pos - pref[w][lo]));
            atomicAdd(acc + (j - c0), 1u);
        }
        my_pairs += (unsigned long long)len;
        __syncwarp();
    }
    __syncthreads();
    // write row i, columns [max(i, c0), c1) of the packed upper triangle
    const int64_t rowoff = (int64_t)i * n - ((int64_t)i * (i - 1)) / 2 - i;  // + j gives S[i][j]
    for (int j = max(i, c0) + tid; j < c1; j += ROW_THREADS) S[rowoff + j] = (int32_t)acc[j - c0];
    if (pairs) {
        // block reduction of the pair-update count
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) my_pairs += __shfl_down_sync(0xffffffffu, my_pairs, d);
        if (lane == 0 && my_pairs) atomicAdd(pairs, my_pairs);
    }
}

// ---------------------------------------------------------------------------
// Stage 2, full-row form (used when a whole row of u16 counters fits in shared
// memory and ntree < 65536).
//   opp_kernel: per (tree, sample), the member range of the opposite bag status
//     in the sample's leaf, already cut to members > sample (binary search
//     done once here, with full memory-level parallelism), stored sample-major
//     opp[i][t] = {start within the tree's member list, length}.
//   row_order_kernel: rows are processed in tree 0's leaf order (then the
//     samples tree 0 excludes), so CTAs running at the same time own rows that
//     share leaves and read the same member lists from L2.
//   pairs_row16_kernel: one CTA per row; u16 counters packed two per 32-bit
//     word; every (row, tree) range expanded across a warp with several member
//     loads in flight per lane.
// ---------------------------------------------------------------------------
constexpr int OPP_TILE = 32;

__global__ void __launch_bounds__(OPP_TILE * 8)
opp_kernel(const int32_t* __restrict__ key, const int32_t* __restrict__ segoff, const int64_t* __restrict__ segbase,
           const int32_t* __restrict__ memb, int n, int T, const uint8_t* __restrict__ keyflag,
           int2* __restrict__ opp) {
    __shared__ int2 tile[OPP_TILE][OPP_TILE + 1];
    const int i0 = blockIdx.x * OPP_TILE, t0 = blockIdx.y * OPP_TILE;
    const int tx = threadIdx.x % OPP_TILE, ty = threadIdx.x / OPP_TILE;
    for (int r = ty; r < OPP_TILE; r += 8) {
        const int t = t0 + r, i = i0 + tx;
        int2 v = make_int2(0, 0);
        if (t < T && i < n) {
            const int k = __ldg(key + (size_t)t * n + i);
            // keys of hub leaves (counted on the tensor cores, hubs.cu) are left out
            if (k >= 0 && !(keyflag && keyflag[segbase[t] + k])) {
                const int32_t* so = segoff + segbase[t];
                int lo = __ldg(so + (k ^ 1)), hi = __ldg(so + (k ^ 1) + 1);
                const int s1 = hi;
                const int32_t* mt = memb + (size_t)t * n;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (__ldg(mt + mid) <= i) lo = mid + 1;
                    else hi = mid;
                }
                v = make_int2(lo, s1 - lo);
            }
        }
        tile[r][tx] = v;
    }
    __syncthreads();
    for (int r = ty; r < OPP_TILE; r += 8) {
        const int i = i0 + r, t = t0 + tx;
        if (i < n && t < T) opp[(size_t)i * T + t] = tile[tx][r];
    }
}

__global__ void __launch_bounds__(1024)
row_order_kernel(const int32_t* __restrict__ key, const int32_t* __restrict__ segoff,
                 const int64_t* __restrict__ segbase, const int32_t* __restrict__ memb, int n,
                 int32_t* __restrict__ order) {
    // thread t owns the samples [t * R, (t + 1) * R): it counts those
    // without a tree-0 leaf, one block-wide scan places its run, and it
    // writes them in ascending order after tree 0's keyed members
    __shared__ int wsum[32];
    const int K0 = (int)(segbase[1] - segbase[0]) - 1;
    const int cnt0 = segoff[segbase[0] + K0];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    for (int q = tid; q < cnt0; q += 1024) order[q] = memb[q];
    const int R = (n + 1023) / 1024;
    const int b = min(n, tid * R), e = min(n, b + R);
    int f = 0;
    for (int i = b; i < e; ++i) f += __ldg(key + i) < 0 ? 1 : 0;
    int incl = f;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += u;
    }
    if (lane == 31) wsum[wid] = incl;
    __syncthreads();
    int woff = 0;
    for (int q = 0; q < wid; ++q) woff += wsum[q];
    int pos = cnt0 + woff + incl - f;
    for (int i = b; i < e && f > 0; ++i)
        if (__ldg(key + i) < 0) {
            order[pos++] = i;
            --f;
        }
}

// Launch shapes of the row kernels the autotuner chooses from: 0..2
// pairs_row16_kernel with 256/512/1024 threads, 3..5 pairs_row2_kernel with
// 256/512/1024 threads.
constexpr int R16_THREADS = 512;
constexpr int PAIRS_SHAPES = 8;
constexpr int PAIRS_DEFAULT_SHAPE = 4;

template <int NW>
__device__ __forceinline__ int block_exclusive_scan(int v, int* wtot, int lane, int w, int* total) {
    int incl = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += u;
    }
    if (lane == 31) wtot[w] = incl;
    __syncthreads();
    if (w == 0) {
        static_assert(NW <= 32, "one warp scans the per-warp totals");
        const int x0 = lane < NW ? wtot[lane] : 0;
        int x = x0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, x, d);
            if (lane >= d) x += u;
        }
        if (lane < NW) wtot[lane] = x - x0;
        if (lane == NW - 1) wtot[NW] = x;
    }
    __syncthreads();
    *total = wtot[NW];
    const int r = wtot[w] + incl - v;
    __syncthreads();  // wtot is reused by the next scan
    return r;
}

// Counter words of the row kernel: ceil(n/2) rounded up to whole 4-counter
// groups plus one zero group, so the write-out can read every group it
// touches (and the one after) with aligned 8-byte loads.
__host__ __device__ inline int r16_words(int n) { return (((n + 1) / 2 + 1) & ~1) + 2; }

// Ranges shorter than this are counted by the thread that loaded them.
constexpr int PAIRS_SHORT = 32;

// One CTA of NT threads per row.  Each round takes NT trees' member ranges of this row,
// drops the empty ones, and cuts the rest into 32-member pieces; every warp
// owns a contiguous run of pieces (so warps finish together whatever the range
// lengths) and processes a piece with its 32 lanes on 32 consecutive members:
// coalesced loads and one shared-memory atomic per member.
template <int NT>
__global__ void __launch_bounds__(NT)
pairs_row16_kernel(const int2* __restrict__ opp, const int32_t* __restrict__ memb, const int32_t* __restrict__ order,
                   int n, int T, int32_t* __restrict__ S, unsigned long long* __restrict__ pairs) {
    constexpr int NW = NT / 32;
    extern __shared__ uint32_t acc[];  // r16_words(n) words, two u16 counters each
    __shared__ long long cb[NT];      // absolute start of each non-empty range
    __shared__ int clen[NT];          // its length
    __shared__ int cp0[NT + 1];       // its first piece index (+ sentinel)
    __shared__ int wtot[NW + 1];
    const int i = order[blockIdx.x];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int words = r16_words(n);
    {
        uint4* a4 = reinterpret_cast<uint4*>(acc);
        const int w4 = words >> 2;
        for (int k = tid; k < w4; k += NT) a4[k] = make_uint4(0u, 0u, 0u, 0u);
        for (int k = (w4 << 2) + tid; k < words; k += NT) acc[k] = 0u;
    }
    unsigned long long my_pairs = 0;
    const int2* orow = opp + (size_t)i * T;
    for (int t0 = 0; t0 < T; t0 += NT) {
        const int t = t0 + tid;
        long long b = 0;
        int len = 0;
        if (t < T) {
            const int2 v = __ldg(orow + t);
            b = (long long)t * n + v.x;
            len = v.y;
        }
        my_pairs += (unsigned long long)len;
        // short ranges (most ranges, few members) are walked by their own
        // thread below; only the long ones are cut into 32-member pieces
        const bool shortr = len < PAIRS_SHORT;
        const int np = shortr ? 0 : (len + 31) >> 5;
        int nseg, P;
        const int cidx = block_exclusive_scan<NW>(np > 0 ? 1 : 0, wtot, lane, w, &nseg);
        const int pfx = block_exclusive_scan<NW>(np, wtot, lane, w, &P);
        if (np > 0) {
            cb[cidx] = b;
            clen[cidx] = len;
            cp0[cidx] = pfx;
        }
        if (tid == 0) cp0[nseg] = P;
        __syncthreads();  // also orders the accumulator zeroing before any update
        if (shortr && len > 0) {
            const int32_t* mp = memb + b;
            for (int q = 0; q < len; ++q) {
                const int j = __ldg(mp + q);
                atomicAdd(acc + (j >> 1), 1u << ((j & 1) << 4));
            }
        }
        // warp w owns pieces [q0, q1); walk the ranges they cover, 32 lanes on
        // consecutive members, four loads in flight per lane
        const int per = (P + NW - 1) / NW;
        const int q0 = w * per;
        const int q1 = min(P, q0 + per);
        if (q0 < q1) {
            int lo = 0, hi = nseg;  // cp0[lo] <= q0 < cp0[hi]
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (cp0[mid] <= q0) lo = mid;
                else hi = mid;
            }
            uint32_t* accw = acc;
            for (int c = lo; c < nseg; ++c) {
                const int pc = cp0[c];
                if (pc >= q1) break;
                const int a = (max(pc, q0) - pc) << 5;
                const int e = min((q1 - pc) << 5, clen[c]);
                const int32_t* mp = memb + cb[c];
                int off = a + lane;
                for (; off + 96 < e; off += 128) {
                    const int j0 = __ldg(mp + off), j1 = __ldg(mp + off + 32);
                    const int j2 = __ldg(mp + off + 64), j3 = __ldg(mp + off + 96);
                    atomicAdd(accw + (j0 >> 1), 1u << ((j0 & 1) << 4));
                    atomicAdd(accw + (j1 >> 1), 1u << ((j1 & 1) << 4));
                    atomicAdd(accw + (j2 >> 1), 1u << ((j2 & 1) << 4));
                    atomicAdd(accw + (j3 >> 1), 1u << ((j3 & 1) << 4));
                }
                for (; off < e; off += 32) {
                    const int j = __ldg(mp + off);
                    atomicAdd(accw + (j >> 1), 1u << ((j & 1) << 4));
                }
            }
        }
        __syncthreads();  // the range tables are rewritten by the next round
    }
    const int64_t rowoff = (int64_t)i * n - ((int64_t)i * (i - 1)) / 2 - i;  // + j gives S[i][j]
    const uint16_t* a16 = reinterpret_cast<const uint16_t*>(acc);
    // the row S[i][i..n) as 16-byte stores between a scalar head and tail
    int32_t* srow = S + rowoff + i;
    const int len = n - i;
    int head = len, nv = 0;
    if ((reinterpret_cast<uintptr_t>(S) & 15) == 0) {
        head = min(len, (int)((4 - ((rowoff + i) & 3)) & 3));
        nv = (len - head) >> 2;
    }
    for (int h = tid; h < head; h += NT) srow[h] = (int32_t)a16[i + h];
    // body: lane L of a warp stores group v = v0 + L (entries jg + 4v ..+3);
    // it reads the aligned 4-counter group containing its first entry, takes
    // the next group from lane L + 1, and shifts by jg's offset in its group
    // (one 8-byte shared load per 4 entries)
    int4* s4 = reinterpret_cast<int4*>(srow + head);
    const int jg = i + head;
    const int sh = (jg & 3) * 16;
    const int gb = jg >> 2;
    const int ngroups = words >> 1;  // 4-counter groups in the array (the last one is padding)
    const uint2* a64 = reinterpret_cast<const uint2*>(acc);
    for (int v0 = w * 32; v0 < nv; v0 += NT) {
        const int v = v0 + lane;
        const int g = gb + v;
        const uint2 cg = g < ngroups ? a64[g] : make_uint2(0u, 0u);
        uint2 nx;
        nx.x = __shfl_down_sync(0xffffffffu, cg.x, 1);
        nx.y = __shfl_down_sync(0xffffffffu, cg.y, 1);
        if (lane == 31) nx = g + 1 < ngroups ? a64[g + 1] : make_uint2(0u, 0u);
        const unsigned long long lo = ((unsigned long long)cg.y << 32) | cg.x;
        const unsigned long long hi = ((unsigned long long)nx.y << 32) | nx.x;
        const unsigned long long e = sh ? (lo >> sh) | (hi << (64 - sh)) : lo;
        if (v < nv)
            s4[v] = make_int4((int)(e & 0xffffu), (int)((e >> 16) & 0xffffu), (int)((e >> 32) & 0xffffu),
                              (int)(e >> 48));
    }
    for (int j = i + head + 4 * nv + tid; j < n; j += NT) srow[j - i] = (int32_t)a16[j];
    if (pairs) {
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) my_pairs += __shfl_down_sync(0xffffffffu, my_pairs, d);
        if (lane == 0 && my_pairs) atomicAdd(pairs, my_pairs);
    }
}

// L2 prefetch of the inputs of row `ip`, which a CTA of a later wave takes
// (the CTA ahead = resident CTAs after this one): its range row (T x 8 bytes)
// and its hub tile row (256 bytes per column tile), one 128-byte line per
// thread, so that row's first loads find them in L2 rather than DRAM.
__device__ __forceinline__ void prefetch_row_l2(const int2* __restrict__ opp, int T, int n, int ip,
                                                const uint8_t* __restrict__ hubt, int tid, int nt) {
    const char* orow = reinterpret_cast<const char*>(opp + (size_t)ip * T);
    const int olines = (T * 8 + 127) >> 7;
    int k = tid;
    for (; k < olines; k += nt)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(orow + ((size_t)k << 7)));
    if (!hubt) return;
    const int NJ = (n + 255) >> 8, I = ip >> 7, r = ip & 127, J0 = ip >> 8;
    const uint8_t* rowt = hubt + (size_t)(hub_row_start(I, NJ) - (I >> 1)) * 32768u + (size_t)r * 256u;
    for (k -= olines; k < (NJ - J0) * 2; k += nt)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(rowt + (size_t)(J0 + (k >> 1)) * 32768u + (k & 1) * 128));
}

// Row i's counters start from the hub leaves' counts when the hub tiles exist
// and hold a hub: row i of the S_hub tiles (row block I = i / 128, column
// tiles J = i / 256 .. NJ - 1; 16-byte chunk q of a tile row stored at slot
// q ^ (row % 16)), u8 -> u16; otherwise from zero.
template <int NT>
__device__ __forceinline__ void row_counters_init(uint32_t* acc, int words, int n, int i,
                                                  const uint8_t* __restrict__ hubt,
                                                  const int32_t* __restrict__ hub_state, int tid) {
    if (hubt) {
        // the tile loads go out with the load of the hub count (the tiles are
        // allocated whether or not any hub was found), two per thread at a time
        const int nh = __ldg(hub_state + 1);
        const int NJ = (n + 255) >> 8, I = i >> 7, r = i & 127, J0 = i >> 8;
        const uint8_t* rowt = hubt + (size_t)(hub_row_start(I, NJ) - (I >> 1)) * 32768u + (size_t)r * 256u;
        const int nch = (NJ - J0) * 16;
        for (int k0 = tid; k0 < nch; k0 += 2 * NT) {
            uint4 v[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int k = k0 + u * NT;
                const int J = J0 + (k >> 4), slot = k & 15;
                v[u] = k < nch ? __ldg(reinterpret_cast<const uint4*>(rowt + (size_t)J * 32768u + slot * 16))
                               : make_uint4(0u, 0u, 0u, 0u);
            }
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int k = k0 + u * NT;
                if (k >= nch) break;
                const int J = J0 + (k >> 4), q = (k & 15) ^ (r & 15);
                const uint32_t b[4] = {v[u].x, v[u].y, v[u].z, v[u].w};
                uint32_t o[8];
                // bytes (b0 b1 b2 b3) -> u16 pairs (b0, b1) and (b2, b3): one byte permute each
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    o[2 * h] = nh > 0 ? __byte_perm(b[h], 0u, 0x4140u) : 0u;
                    o[2 * h + 1] = nh > 0 ? __byte_perm(b[h], 0u, 0x4342u) : 0u;
                }
                uint4* dst = reinterpret_cast<uint4*>(acc + (size_t)J * 128 + q * 8);
                dst[0] = make_uint4(o[0], o[1], o[2], o[3]);
                dst[1] = make_uint4(o[4], o[5], o[6], o[7]);
            }
        }
        // (words below J0 * 128 hold columns before i: never counted or written)
        for (int k = NJ * 128 + tid; k < words; k += NT) acc[k] = 0u;
    } else {
        uint4* a4 = reinterpret_cast<uint4*>(acc);
        const int w4 = words >> 2;
        for (int k = tid; k < w4; k += NT) a4[k] = make_uint4(0u, 0u, 0u, 0u);
        for (int k = (w4 << 2) + tid; k < words; k += NT) acc[k] = 0u;
    }
}

// Row i of S (entries j >= i of the packed upper triangle) from the u16
// counters.
template <int NT>
__device__ __forceinline__ void row_write_out(const uint32_t* acc, int words, int n, int i, int32_t* __restrict__ S,
                                              int tid) {
    const int lane = tid & 31, w = tid >> 5;
    const int64_t rowoff = (int64_t)i * n - ((int64_t)i * (i - 1)) / 2 - i;  // + j gives S[i][j]
    const uint16_t* a16 = reinterpret_cast<const uint16_t*>(acc);
    int32_t* srow = S + rowoff + i;
    const int len = n - i;
    int head = len, nv = 0;
    if ((reinterpret_cast<uintptr_t>(S) & 15) == 0) {
        head = min(len, (int)((4 - ((rowoff + i) & 3)) & 3));
        nv = (len - head) >> 2;
    }
    for (int h = tid; h < head; h += NT) srow[h] = (int32_t)a16[i + h];
    // body: lane L of a warp stores group v = v0 + L (entries jg + 4v ..+3);
    // it reads the aligned 4-counter group holding its first entry (one
    // 8-byte shared load), takes the next group from lane L + 1, and picks its
    // four 16-bit counters with byte permutes (the offset o of jg in its group
    // is the same for the whole row)
    int4* s4 = reinterpret_cast<int4*>(srow + head);
    const int jg = i + head;
    const int o = jg & 3;
    const int gb = jg >> 2;
    const int ngroups = words >> 1;  // 4-counter groups in the array (the last one is padding)
    const uint2* a64 = reinterpret_cast<const uint2*>(acc);
    for (int v0 = w * 32; v0 < nv; v0 += NT) {
        const int v = v0 + lane;
        const int g = gb + v;
        const uint2 cg = g < ngroups ? a64[g] : make_uint2(0u, 0u);
        uint2 nx;
        nx.x = __shfl_down_sync(0xffffffffu, cg.x, 1);
        nx.y = __shfl_down_sync(0xffffffffu, cg.y, 1);
        if (lane == 31) nx = g + 1 < ngroups ? a64[g + 1] : make_uint2(0u, 0u);
        uint32_t q0, q1, q2, q3;
        if (o == 0) {
            q0 = __byte_perm(cg.x, 0u, 0x4410u); q1 = __byte_perm(cg.x, 0u, 0x4432u);
            q2 = __byte_perm(cg.y, 0u, 0x4410u); q3 = __byte_perm(cg.y, 0u, 0x4432u);
        } else if (o == 1) {
            q0 = __byte_perm(cg.x, 0u, 0x4432u); q1 = __byte_perm(cg.y, 0u, 0x4410u);
            q2 = __byte_perm(cg.y, 0u, 0x4432u); q3 = __byte_perm(nx.x, 0u, 0x4410u);
        } else if (o == 2) {
            q0 = __byte_perm(cg.y, 0u, 0x4410u); q1 = __byte_perm(cg.y, 0u, 0x4432u);
            q2 = __byte_perm(nx.x, 0u, 0x4410u); q3 = __byte_perm(nx.x, 0u, 0x4432u);
        } else {
            q0 = __byte_perm(cg.y, 0u, 0x4432u); q1 = __byte_perm(nx.x, 0u, 0x4410u);
            q2 = __byte_perm(nx.x, 0u, 0x4432u); q3 = __byte_perm(nx.y, 0u, 0x4410u);
        }
        if (v < nv) s4[v] = make_int4((int)q0, (int)q1, (int)q2, (int)q3);
    }
    for (int j = i + head + 4 * nv + tid; j < n; j += NT) srow[j - i] = (int32_t)a16[j];
}

// ---------------------------------------------------------------------------
// Stage 2, full-row form without per-round block barriers (pairs_row2_kernel).
//   One CTA per row, u16 counters for the whole row as in pairs_row16_kernel.
//   Phase A: warps claim chunks of 32 trees from a CTA counter (lane = tree)
//     and count the chunk's short ranges themselves: ranges shorter than 32
//     members are expanded element by element over the warp (a lane finds
//     its range by a binary search over the warp's inclusive length scan, so
//     no lane idles on a short range).  Ranges of 32 members or more are put
//     on a per-CTA list (those beyond its capacity are walked by the whole
//     warp, four loads in flight per lane).
//   Phase B (after one barrier): the listed ranges are cut into pieces of 32
//     members dealt round-robin over the warps, so every warp gets the same
//     share of them whatever the chunks held; four loads in flight per lane.
//   Three barriers per row: after zeroing, between the phases, before the
//   write-out.
// ---------------------------------------------------------------------------
constexpr int V2_LONG = 32;   // ranges of this many members or more go on the CTA list
constexpr int V2_LIST = 256;  // listed ranges per row (more are walked in phase A)

__device__ __forceinline__ void count16(uint32_t* acc, int j) { atomicAdd(acc + (j >> 1), 1u << ((j & 1) << 4)); }

template <int NT, int SV>
__global__ void __launch_bounds__(NT, 2048 / NT)
pairs_row2_kernel(const int2* __restrict__ opp, const int32_t* __restrict__ memb, const int32_t* __restrict__ order,
                  int n, int T, int words, const uint8_t* __restrict__ hubt, const int32_t* __restrict__ hub_state,
                  int32_t* __restrict__ S, unsigned long long* __restrict__ pairs, int ahead) {
    constexpr int NW = NT / 32;
    extern __shared__ uint32_t acc[];  // `words` words, two u16 counters each
    __shared__ long long lbase[V2_LIST];
    __shared__ int llen[V2_LIST];
    __shared__ int s_nlong, s_chunk, s_np;
    __shared__ int lpre[V2_LIST];       // first piece number of each listed long range
    __shared__ uint8_t s_lid[NW][32];  // per warp: lanes with a non-empty short range
    const int i = order[blockIdx.x];
    const int ipf = blockIdx.x + ahead < n ? order[blockIdx.x + ahead] : -1;  // the row prefetched below
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    row_counters_init<NT>(acc, words, n, i, hubt, hub_state, tid);
    if (ipf >= 0) prefetch_row_l2(opp, T, n, ipf, hubt, tid, NT);
    if (tid == 0) {
        s_nlong = 0;
        s_chunk = 0;
    }
    __syncthreads();
    unsigned long long my_pairs = 0;
    const int2* orow = opp + (size_t)i * T;
    const int nchunks = (T + 31) >> 5;
    for (;;) {
        int ch = 0;
        if (lane == 0) ch = atomicAdd(&s_chunk, 1);
        ch = __shfl_sync(0xffffffffu, ch, 0);
        if (ch >= nchunks) break;
        const int t = (ch << 5) + lane;
        const int2 v = t < T ? __ldg(orow + t) : make_int2(0, 0);
        int len = v.y;
        my_pairs += (unsigned long long)len;
        if (len >= V2_LONG) {
            const int slot = atomicAdd(&s_nlong, 1);
            if (slot < V2_LIST) {
                lbase[slot] = (long long)t * n + v.x;
                llen[slot] = len;
                len = 0;
            }
        }
        // ranges of 32 members or more that stayed here: the whole warp walks each
        unsigned med = __ballot_sync(0xffffffffu, len >= 32);
        while (med) {
            const int src = __ffs(med) - 1;
            med &= med - 1;
            const int ml = __shfl_sync(0xffffffffu, len, src);
            const int ts = (ch << 5) + src;
            const int xs = __shfl_sync(0xffffffffu, v.x, src);
            const int32_t* mp = memb + (size_t)ts * n + xs;
            int off = lane;
            for (; off + 96 < ml; off += 128) {
                const int j0 = __ldg(mp + off), j1 = __ldg(mp + off + 32);
                const int j2 = __ldg(mp + off + 64), j3 = __ldg(mp + off + 96);
                count16(acc, j0);
                count16(acc, j1);
                count16(acc, j2);
                count16(acc, j3);
            }
            for (; off < ml; off += 32) count16(acc, __ldg(mp + off));
        }
        if (len >= 32) len = 0;
        // the short ranges, element by element over the warp
        int incl = len;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += u;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        const int xoff = v.x - (incl - len);  // member index = tree base + xoff + element
        if constexpr (SV == 0) {
            // a lane finds the range of its element by a binary search over
            // the warp's inclusive length scan
            for (int base = 0; base < total; base += 64) {
                int j[2];
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int e = base + (u << 5) + lane;
                    const int ec = min(e, total - 1);
                    int c = 0;  // number of lanes whose inclusive end is <= ec
#pragma unroll
                    for (int d = 16; d > 0; d >>= 1) {
                        const int x = __shfl_sync(0xffffffffu, incl, c + d - 1);
                        if (x <= ec) c += d;
                    }
                    const int xo = __shfl_sync(0xffffffffu, xoff, c);
                    j[u] = e < total ? __ldg(memb + (size_t)((ch << 5) + c) * n + (xo + e)) : -1;
                }
#pragma unroll
                for (int u = 0; u < 2; ++u)
                    if (j[u] >= 0) count16(acc, j[u]);
            }
        } else if (total > 0) {
            // element e belongs to the last non-empty range starting at or
            // before e: the warp lists its non-empty ranges (lane ids, in lane
            // order) and, per window of 64 elements, ORs the range starts into
            // a 64-bit mask, so an element finds its range with population
            // counts
            const int ex = incl - len;  // this range's first element
            const unsigned ne = __ballot_sync(0xffffffffu, len > 0);
            if (len > 0) s_lid[w][__popc(ne & ((1u << lane) - 1u))] = (uint8_t)lane;
            __syncwarp();
            for (int base = 0; base < total; base += 64) {
                const int sb = ex - base;
                const bool st = len > 0 && sb >= 0 && sb < 64;
                const unsigned lo = __reduce_or_sync(0xffffffffu, st && sb < 32 ? 1u << (sb & 31) : 0u);
                const unsigned hi = __reduce_or_sync(0xffffffffu, st && sb >= 32 ? 1u << (sb & 31) : 0u);
                const int before = __popc(__ballot_sync(0xffffffffu, len > 0 && sb < 0));
                const unsigned upto = 0xffffffffu >> (31 - lane);  // bits 0..lane
                int j[2];
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int e = base + (u << 5) + lane;
                    const int cnt = u == 0 ? __popc(lo & upto) : __popc(lo) + __popc(hi & upto);
                    const int c = s_lid[w][max(0, before + cnt - 1)];
                    const int xo = __shfl_sync(0xffffffffu, xoff, c);
                    j[u] = e < total ? __ldg(memb + (size_t)((ch << 5) + c) * n + (xo + e)) : -1;
                }
#pragma unroll
                for (int u = 0; u < 2; ++u)
                    if (j[u] >= 0) count16(acc, j[u]);
            }
            __syncwarp();  // the list is rewritten by this warp's next chunk
        }
    }
    __syncthreads();
    // phase B: the listed ranges cut into pieces of 32 members; piece g (ranges
    // in list order) goes to warp g % NW.  Lane l of warp w looks up piece
    // w + NW * (32 r + l) of round r (a binary search over the ranges' first
    // piece numbers, lpre) and the warp then takes its pieces four at a time,
    // the piece's start and length broadcast from the lane that found it.
    const int L = min(s_nlong, V2_LIST);
    if (w == 0) {
        constexpr int PL = V2_LIST / 32;  // ranges per lane
        int loc[PL];
        int sum = 0;
#pragma unroll
        for (int u = 0; u < PL; ++u) {
            const int c = lane * PL + u;
            loc[u] = sum;
            sum += c < L ? (llen[c] + 31) >> 5 : 0;
        }
        int incl = sum;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += u;
        }
#pragma unroll
        for (int u = 0; u < PL; ++u) lpre[lane * PL + u] = incl - sum + loc[u];
        if (lane == 31) s_np = incl;
    }
    __syncthreads();
    const int P = s_np;
    for (int r0 = w; r0 < P; r0 += NW * 32) {
        const int g = r0 + NW * lane;
        long long ps = 0;
        int lim = 0;
        if (g < P) {
            int lo = 0, hi = L;  // the last range whose first piece is <= g
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (lpre[mid] <= g) lo = mid;
                else hi = mid;
            }
            const int k = g - lpre[lo];
            ps = lbase[lo] + ((long long)k << 5);
            lim = min(32, llen[lo] - (k << 5));
        }
        const int cnt = min(32, (P - r0 + NW - 1) / NW);  // pieces of this warp in this round
        for (int u0 = 0; u0 < cnt; u0 += 4) {
            int j[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const long long pv = __shfl_sync(0xffffffffu, ps, (u0 + v) & 31);
                const int lv = __shfl_sync(0xffffffffu, lim, (u0 + v) & 31);
                j[v] = (u0 + v < cnt && lane < lv) ? __ldg(memb + pv + lane) : -1;
            }
#pragma unroll
            for (int v = 0; v < 4; ++v)
                if (j[v] >= 0) count16(acc, j[v]);
        }
    }
    __syncthreads();
    row_write_out<NT>(acc, words, n, i, S, tid);
    if (pairs) {
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) my_pairs += __shfl_down_sync(0xffffffffu, my_pairs, d);
        if (lane == 0 && my_pairs) atomicAdd(pairs, my_pairs);
    }
}

// ---------------------------------------------------------------------------
// Stage 2, balanced full-row form (pairs_row3_kernel).
//   One CTA per row with the u16 counters, start values and write-out of
//   pairs_row2_kernel.  The row's ranges are taken in rounds of NT trees:
//   thread t loads the range of tree t of the round, a CTA-wide scan of the
//   lengths lists the non-empty ranges (s_pre: the first element of each in
//   the round's element sequence; s_off: its member-list position minus that
//   element number), and the E elements of the round are cut into NW
//   contiguous slices, one per warp, so every warp gets the same count
//   whatever the lengths.  A warp walks its slice in windows of 32 elements
//   (lane x takes element W + x): the ranges that start inside a window are
//   the next listed ones after the range r holding element W - 1, so one
//   shared-memory load of the next 32 starts and an OR of the bits
//   (start - W) give each lane its range by a population count.  The member
//   loads of R3_BATCH windows are issued before their counts.  Member-list
//   positions are 32-bit here (ntree x n < 2^31, checked by the launcher).
// ---------------------------------------------------------------------------
constexpr int R3_BATCH = 8;

// (two CTAs per SM: a row's counters take up to half the shared memory at the
// sizes this form serves, so 512 threads get 64 registers and 1024 get 32)
template <int NT>
__global__ void __launch_bounds__(NT, 2)
pairs_row3_kernel(const int2* __restrict__ opp, const int32_t* __restrict__ memb, const int32_t* __restrict__ order,
                  int n, int T, int words, const uint8_t* __restrict__ hubt, const int32_t* __restrict__ hub_state,
                  int32_t* __restrict__ S, unsigned long long* __restrict__ pairs, int ahead) {
    constexpr int NW = NT / 32;
    extern __shared__ uint32_t acc[];  // `words` words, two u16 counters each
    __shared__ int s_off[NT];
    __shared__ int s_pre[NT + 32];     // INT_MAX after the last listed range
    __shared__ int s_wf[NW], s_wl[NW];  // per-warp totals: non-empty ranges, elements
    const int i = order[blockIdx.x];
    const int ipf = blockIdx.x + ahead < n ? order[blockIdx.x + ahead] : -1;  // the row prefetched below
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    // the first round's ranges are loaded before the counters are set up, so
    // the two loads are in flight together
    const int2* orow = opp + (size_t)i * T;
    const int2 v0 = tid < T ? __ldg(orow + tid) : make_int2(0, 0);
    row_counters_init<NT>(acc, words, n, i, hubt, hub_state, tid);
    if (ipf >= 0) prefetch_row_l2(opp, T, n, ipf, hubt, tid, NT);
    unsigned long long my_pairs = 0;
    for (int tb = 0; tb < T; tb += NT) {
        const int t = tb + tid;
        const int2 v = tb == 0 ? v0 : t < T ? __ldg(orow + t) : make_int2(0, 0);
        const int len = v.y;
        const int f = len > 0 ? 1 : 0;
        my_pairs += (unsigned long long)len;
        int fi = f, li = len;  // inclusive warp scans
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int a = __shfl_up_sync(0xffffffffu, fi, d);
            const int b = __shfl_up_sync(0xffffffffu, li, d);
            if (lane >= d) {
                fi += a;
                li += b;
            }
        }
        if (lane == 31) {
            s_wf[w] = fi;
            s_wl[w] = li;
        }
        // (also: every warp has finished the previous round's element phase
        // before its list is overwritten below)
        __syncthreads();
        int wf = lane < NW ? s_wf[lane] : 0, wl = lane < NW ? s_wl[lane] : 0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int a = __shfl_up_sync(0xffffffffu, wf, d);
            const int b = __shfl_up_sync(0xffffffffu, wl, d);
            if (lane >= d) {
                wf += a;
                wl += b;
            }
        }
        const int R = __shfl_sync(0xffffffffu, wf, 31);
        const int E = __shfl_sync(0xffffffffu, wl, 31);
        const int fb = __shfl_sync(0xffffffffu, wf, (w + 31) & 31);
        const int lb = __shfl_sync(0xffffffffu, wl, (w + 31) & 31);
        if (f) {
            const int c = (w > 0 ? fb : 0) + fi - 1;
            const int e0 = (w > 0 ? lb : 0) + li - len;
            s_pre[c] = e0;
            s_off[c] = t * n + v.x - e0;
        }
        if (tid < 32) s_pre[R + tid] = 0x7fffffff;
        __syncthreads();
        const int per = (E + NW - 1) / NW;
        const int e_beg = w * per, e_end = min(E, e_beg + per);
        if (e_beg < e_end) {
            // r: the listed range holding element e_beg (the last c with
            // s_pre[c] <= e_beg), by a 32-way search: lane l probes
            // lo + l * step, the probes at or below e_beg are a prefix of the
            // lanes (s_pre rises), two rounds for up to 1024 ranges
            int lo = 0, hi = R;
            while (hi - lo > 1) {
                const int step = (hi - lo + 31) >> 5;
                const int c = lo + lane * step;
                const unsigned le = __ballot_sync(0xffffffffu, c < hi && s_pre[c] <= e_beg);
                lo += (__popc(le) - 1) * step;
                hi = min(hi, lo + step);
            }
            int r = lo;
            for (int W = e_beg; W < e_end; W += 32 * R3_BATCH) {
                int j[R3_BATCH];
#pragma unroll
                for (int u = 0; u < R3_BATCH; ++u) {
                    const int Wu = W + 32 * u;
                    j[u] = -1;
                    if (Wu < e_end) {  // the same for the whole warp: windows past the slice are skipped
                        // ranges r + 1 ... start at or after Wu; those before Wu + 32 set bit (start - Wu)
                        const int nl = s_pre[r + 1 + lane];
                        const unsigned P = __reduce_or_sync(0xffffffffu, nl < Wu + 32 ? 1u << (nl - Wu) : 0u);
                        const int x = Wu + lane;
                        const int rc = r + __popc(P & (0xffffffffu >> (31 - lane)));
                        if (x < e_end) j[u] = __ldg(memb + (unsigned)(s_off[rc] + x));
                        r += __popc(P);
                    }
                }
#pragma unroll
                for (int u = 0; u < R3_BATCH; ++u)
                    if (j[u] >= 0) count16(acc, j[u]);
            }
        }
    }
    __syncthreads();
    row_write_out<NT>(acc, words, n, i, S, tid);
    if (pairs) {
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) my_pairs += __shfl_down_sync(0xffffffffu, my_pairs, d);
        if (lane == 0 && my_pairs) atomicAdd(pairs, my_pairs);
    }
}

// ---------------------------------------------------------------------------
// finishprox
// ---------------------------------------------------------------------------
constexpr int FP_TILE = 32;
constexpr int FP_JT = 8;  // column tiles per CTA

// S/2 is exact for an integer S, so it is formed as S * 0.5 (the same double
// as the reference's division by 2).  inv_i is 1/nout[i], or 1.0 where
// nout[i] == 0: the reference then uses S/2 unscaled, and S/2 * 1.0 is
// that same double, so one product covers both cases.
__device__ __forceinline__ double fp_value(double s, double inv_i, double inv_j) {
    const double h = __dmul_rn(s, 0.5);
    return __dmul_rn(0.5, __dadd_rn(__dmul_rn(h, inv_i), __dmul_rn(h, inv_j)));
}

// 1/nout per sample, formed once per call (1.0 where nout == 0).
__global__ void finish_inv_kernel(const int32_t* __restrict__ nout, int n, double* __restrict__ inv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const int ni = nout[i];
        inv[i] = ni > 0 ? __ddiv_rn(1.0, (double)ni) : 1.0;
    }
}

// Runs of FP_JT column tiles J >= I of row tile I.
__host__ __device__ __forceinline__ int fp_runs(int nt, int I) { return (nt - I + FP_JT - 1) / FP_JT; }

// One CTA per run of FP_JT column tiles J >= I of one row tile I; computes
// the 32x32 values of each tile (I, J) from the packed S rows of tile I and
// writes tile (I, J) and its mirror (J, I) of the full matrix, or tile (I, J)
// of the packed triangle.  Grid: y = row-tile pair (I, nt - 1 - I), whose run
// counts add up to about nt / FP_JT, x = run within the pair, so no CTA lies
// left of the diagonal.  The next tile's S values and column factors are
// loaded before the current tile's values are formed.
template <typename TS>
__global__ void __launch_bounds__(FP_TILE * 8)
finishprox_kernel(const TS* __restrict__ S, const double* __restrict__ inv, int n, int full,
                  float* __restrict__ P) {
    __shared__ float tile[FP_TILE][FP_TILE + 1];
    __shared__ double s_inv[FP_TILE];
    const int nt = (n + FP_TILE - 1) / FP_TILE;
    int I = blockIdx.y, run = blockIdx.x;
    const int ra = fp_runs(nt, I);
    if (run >= ra) {
        I = nt - 1 - I;
        run -= ra;
        if (I <= (int)blockIdx.y || run >= fp_runs(nt, I)) return;
    }
    const int J0 = I + run * FP_JT;
    const int J1 = min(J0 + FP_JT, nt);
    const int tx = threadIdx.x % FP_TILE, ty = threadIdx.x / FP_TILE;  // 32 x 8
    if (threadIdx.x < FP_TILE) {
        const int i = I * FP_TILE + threadIdx.x;
        s_inv[threadIdx.x] = i < n ? __ldg(inv + i) : 1.0;
    }
    constexpr int RU = FP_TILE / 8;  // rows per thread
    // row offsets of the packed triangle: S[i][j] = S[base_i + j]
    int64_t base[RU];
#pragma unroll
    for (int u = 0; u < RU; ++u) {
        const int64_t i = I * FP_TILE + ty + 8 * u;
        base[u] = i * n - (i * (i - 1)) / 2 - i;
    }
    auto load = [&](int J, TS* sv, double& invj) {
        const int j = J * FP_TILE + tx;
        const bool jv = j < n;
        invj = jv ? __ldg(inv + j) : 1.0;
#pragma unroll
        for (int u = 0; u < RU; ++u) {
            const int i = I * FP_TILE + ty + 8 * u;
            sv[u] = (i < n && jv && j > i) ? __ldg(S + base[u] + j) : (TS)0;
        }
    };
    TS cur[RU], nxt[RU];
    double inv_c = 1.0, inv_n = 1.0;
    load(J0, cur, inv_c);
    __syncthreads();
    for (int J = J0; J < J1; ++J) {
        if (J + 1 < J1) load(J + 1, nxt, inv_n);
        const int j = J * FP_TILE + tx;
        const bool jv = j < n;
#pragma unroll
        for (int u = 0; u < RU; ++u) {
            const int r = ty + 8 * u;
            const int i = I * FP_TILE + r;
            float v = 0.0f;
            if (i < n && jv && j >= i) {
                const double d = (j == i) ? 1.0 : fp_value((double)cur[u], s_inv[r], inv_c);
                v = __double2float_rn(d);
                if (full) P[(size_t)i * n + j] = v;
                else P[base[u] + j] = v;
            }
            if (full) tile[r][tx] = v;
        }
        if (full) {
            __syncthreads();
            // mirror: P[j][i] for j in tile J rows, i in tile I columns (strictly lower part)
            for (int r = ty; r < FP_TILE; r += 8) {
                const int jj = J * FP_TILE + r;
                const int ii = I * FP_TILE + tx;
                if (jj < n && ii < n && jj > ii) P[(size_t)jj * n + ii] = tile[tx][r];
            }
            __syncthreads();  // the tile is rewritten for the next J
        }
#pragma unroll
        for (int u = 0; u < RU; ++u) cur[u] = nxt[u];
        inv_c = inv_n;
    }
}

}  // namespace

// Leaf lists of arbitrary keys (key per (tree, sample) in [0, K_t), or -1),
// for callers with their own key tables (RF-GAP's node-id keys).
rfx_status launch_build_csr_raw(cudaStream_t s, int device, const int32_t* key, int n, int T, const int64_t* segbase,
                                int32_t* segoff, int32_t* memb, int max_keys, uint32_t* err) {
    int dev_smem = 0;
    RFX_CUDA(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    int smem_keys = std::min(max_keys + 1, (dev_smem - 1024) / 4);
    smem_keys = std::max(smem_keys, 32);
    const size_t smem = (size_t)smem_keys * sizeof(int32_t);
    if (rfx_status s0 = allow_dyn_smem(build_csr_kernel<int32_t>, dev_smem)) return s0;
    build_csr_kernel<int32_t><<<T, CSR_THREADS, smem, s>>>(key, n, segbase, segoff, memb, smem_keys, err);
    RFX_CUDA(cudaGetLastError());
    if (max_keys + 1 > smem_keys) {
        fix_global_segoff_kernel<<<T, 32, 0, s>>>(segbase, segoff, smem_keys);
        RFX_CUDA(cudaGetLastError());
    }
    return RFX_OK;
}

rfx_status launch_build_csr(Ctx* c) {
    int dev_smem = 0;
    RFX_CUDA(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
    // budget per tree-warp; several warps (trees) share an SM
    const bool narrow = c->n < 65536;  // counts and offsets fit 16 bits
    const int csz = narrow ? 2 : 4;
    int smem_keys = std::min(c->max_keys + 1, (dev_smem - 1024) / csz - 2);
    smem_keys = std::max(smem_keys, 32);
    const size_t smem = ((size_t)(smem_keys + 2) * csz + 3) & ~(size_t)3;
    StageTimer st(c, ST_CSR, c->max_keys + 1 > smem_keys ? 2 : 1);
    if (rfx_status s0 = allow_dyn_smem(build_csr_kernel<uint16_t>, dev_smem)) return s0;
    if (rfx_status s0 = allow_dyn_smem(build_csr_kernel<int32_t>, dev_smem)) return s0;
    (narrow ? build_csr_kernel<uint16_t> : build_csr_kernel<int32_t>)<<<c->T, CSR_THREADS, smem, c->stream>>>(
        c->d_key, c->n, c->d_segbase, c->d_segoff, c->d_memb, smem_keys,
                                                    c->d_err);
    RFX_CUDA(cudaGetLastError());
    if (c->max_keys + 1 > smem_keys) {
        fix_global_segoff_kernel<<<c->T, 32, 0, c->stream>>>(c->d_segbase, c->d_segoff, smem_keys);
        RFX_CUDA(cudaGetLastError());
    }
    return RFX_OK;
}

int pairs_window(const Ctx* c) {
    // columns per CTA: 96 KB of u32 accumulators (two CTAs per SM)
    const int win_max = 24 * 1024;
    return std::min(c->n, win_max);
}

bool use_row16(const Ctx* c, int dev_smem) {
    // RFX_PAIRS_KERNEL=windowed selects the windowed u32 kernel (used for
    // large n or ntree >= 65536) so that it can be tested at small sizes.
    const char* force = getenv("RFX_PAIRS_KERNEL");
    if (force && std::string(force) == "windowed") return false;
    const size_t words = ((size_t)c->n + 1) / 2;
    return c->T < 65536 && words * 4 + 20 * 1024 <= (size_t)dev_smem;
}

// Hub leaves on the tensor cores (hubs.cu): by default from n = 16,384 and
// 512 trees.  The tiles cost a fixed n x n pass (the GEMM and the row
// kernel's read of the tiles) while the updates they take over grow with the
// number of trees: 64 forests of 300 trees at n <= 50,000 ran 1.3x slower
// with them.  RFX_PAIRS_HUBS=0 turns the part off, =1 forces it on at any
// size.  The counts are the same either way.
bool use_hubs(const Ctx* c) {
    const char* e = getenv("RFX_PAIRS_HUBS");
    if (e && std::string(e) == "0") return false;
    if (e && std::string(e) == "1") return true;
    return c->n >= 16384 && c->T >= 512;
}

rfx_status launch_pairs_upper(Ctx* c, int32_t* dS) {
    int dev_smem = 0;
    RFX_CUDA(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
    if (use_row16(c, dev_smem)) {
        const int NJ = hub_tiles_nj(c->n);
        const int hub_words = NJ * 128 + 2;
        const bool hubs = use_hubs(c) && (size_t)hub_words * 4 + 20 * 1024 <= (size_t)dev_smem;
        rfx_status st0 = dalloc(c, &c->d_opp, (size_t)c->T * c->n);
        if (st0 == RFX_OK) st0 = dalloc(c, &c->d_order, (size_t)c->n);
        if (st0 == RFX_OK && hubs) st0 = dalloc(c, &c->d_hubflag, (size_t)c->h_segbase[c->T]);
        if (st0 == RFX_OK && hubs) st0 = dalloc(c, &c->d_hubtiles, hub_tile_bytes(c->n));
        if (st0 == RFX_OK && hubs) st0 = dalloc(c, &c->d_hubstate, (size_t)8);
        if (st0 != RFX_OK) return st0;
        unsigned long long* hub_pairs = reinterpret_cast<unsigned long long*>(c->d_hubstate + 4);
        if (hubs) {
            RFX_CUDA(cudaMemsetAsync(c->d_hubstate, 0, 8 * sizeof(int32_t), c->stream));
            StageTimer st(c, ST_HUBS, 5);
            if (rfx_status s1 = launch_hub_tiles(c, c->d_hubflag, c->d_hubtiles, c->d_hubstate, hub_pairs)) return s1;
        }
        {
            StageTimer st(c, ST_OPP, 2);
            dim3 g((c->n + OPP_TILE - 1) / OPP_TILE, (c->T + OPP_TILE - 1) / OPP_TILE);
            opp_kernel<<<g, OPP_TILE * 8, 0, c->stream>>>(c->d_key, c->d_segoff, c->d_segbase, c->d_memb, c->n,
                                                           c->T, hubs ? c->d_hubflag : nullptr, c->d_opp);
            RFX_CUDA(cudaGetLastError());
            row_order_kernel<<<1, 1024, 0, c->stream>>>(c->d_key, c->d_segoff, c->d_segbase, c->d_memb, c->n,
                                                        c->d_order);
            RFX_CUDA(cudaGetLastError());
        }
        const int words = hubs ? std::max(r16_words(c->n), hub_words) : r16_words(c->n);
        const size_t smem = (size_t)words * sizeof(uint32_t);
        if (rfx_status s0 = allow_dyn_smem(pairs_row16_kernel<256>, dev_smem)) return s0;
        if (rfx_status s0 = allow_dyn_smem(pairs_row16_kernel<512>, dev_smem)) return s0;
        if (rfx_status s0 = allow_dyn_smem(pairs_row16_kernel<1024>, dev_smem)) return s0;
        if (rfx_status s0 = allow_dyn_smem(pairs_row2_kernel<256, 0>, dev_smem)) return s0;
        if (rfx_status s0 = allow_dyn_smem(pairs_row2_kernel<512, 0>, dev_smem)) return s0;
        if (rfx_status s0 = allow_dyn_smem(pairs_row2_kernel<1024, 0>, dev_smem)) return s0;
        if (rfx_status s0 = allow_dyn_smem(pairs_row2_kernel<256, 1>, dev_smem)) return s0;
        if (rfx_status s0 = allow_dyn_smem(pairs_row2_kernel<512, 1>, dev_smem)) return s0;
        if (rfx_status s0 = allow_dyn_smem(pairs_row2_kernel<1024, 1>, dev_smem)) return s0;
        if (rfx_status s0 = allow_dyn_smem(pairs_row3_kernel<512>, dev_smem)) return s0;
        if (rfx_status s0 = allow_dyn_smem(pairs_row3_kernel<1024>, dev_smem)) return s0;
        // the balanced row kernel keeps member-list positions in 32 bits
        const bool row3_ok = (long long)c->T * c->n < (1ll << 31);
        StageTimer st(c, ST_PAIRS, 1);
        // with hub tiles only the second row kernel (which starts from them) runs
        const int tk = hubs ? TK_PAIRS_HUB : TK_PAIRS16;
        const int nshape = PAIRS_SHAPES;
        const int defshape = hubs ? 1 : PAIRS_DEFAULT_SHAPE;
        return autotune(c, tk, nshape, defshape, [&](int shape) -> rfx_status {
            // the pair counter restarts from the hub leaves' pair updates
            if (hubs)
                RFX_CUDA(cudaMemcpyAsync(c->d_pairs, hub_pairs, sizeof(unsigned long long), cudaMemcpyDeviceToDevice,
                                         c->stream));
            else
                RFX_CUDA(cudaMemsetAsync(c->d_pairs, 0, sizeof(unsigned long long), c->stream));
            // shapes 6-7 (with or without hub tiles): row3 with 512 / 1024
            // threads (row2 1024 where row3 does not apply); hub shapes 0-2:
            // row2 with 256/512/1024 threads, binary-search short ranges, 3-5:
            // the same with the start-mask lookup; otherwise 0-2 row16 and
            // 3-5 row2 with 256/512/1024 threads
            // a CTA prefetches into L2 the inputs of the row that the CTA one
            // wave of resident CTAs later takes
            // (resident CTAs per SM from the thread count and the shared memory
            // of a row, with 10 KB for the kernels' static arrays; device
            // attributes only, so this also holds inside a graph capture)
            auto ahead_of = [&](auto, int nt) -> int {
                int sms = 148, smem_sm = 233472;
                cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
                cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, c->device);
                const int by_smem = smem_sm / (int)(smem + 10 * 1024);
                return sms * std::max(1, std::min(2048 / nt, by_smem));
            };
            if (shape >= 6 && row3_ok) {
                auto kern = shape == 6 ? pairs_row3_kernel<512> : pairs_row3_kernel<1024>;
                const int nt = shape == 6 ? 512 : 1024;
                kern<<<c->n, nt, smem, c->stream>>>(c->d_opp, c->d_memb, c->d_order, c->n, c->T, words,
                                                    hubs ? c->d_hubtiles : nullptr, c->d_hubstate, dS, c->d_pairs,
                                                    ahead_of(kern, nt));
                RFX_CUDA(cudaGetLastError());
                return RFX_OK;
            }
            if (shape >= 6) shape = 5;
            int sv = 0;
            if (hubs) {
                sv = shape >= 3;
                shape = 3 + shape % 3;
            }
            if (shape >= 3) {
                const int nt = 256 << (shape - 3);
                auto kern = sv ? (shape == 3 ? pairs_row2_kernel<256, 1> : shape == 4 ? pairs_row2_kernel<512, 1>
                                                                                        : pairs_row2_kernel<1024, 1>)
                               : (shape == 3 ? pairs_row2_kernel<256, 0> : shape == 4 ? pairs_row2_kernel<512, 0>
                                                                                        : pairs_row2_kernel<1024, 0>);
                kern<<<c->n, nt, smem, c->stream>>>(c->d_opp, c->d_memb, c->d_order, c->n, c->T, words,
                                                    hubs ? c->d_hubtiles : nullptr, c->d_hubstate, dS, c->d_pairs,
                                                    ahead_of(kern, nt));
            } else if (shape == 0)
                pairs_row16_kernel<256><<<c->n, 256, smem, c->stream>>>(c->d_opp, c->d_memb, c->d_order, c->n, c->T,
                                                                       dS, c->d_pairs);
            else if (shape == 2)
                pairs_row16_kernel<1024><<<c->n, 1024, smem, c->stream>>>(c->d_opp, c->d_memb, c->d_order, c->n,
                                                                         c->T, dS, c->d_pairs);
            else
                pairs_row16_kernel<512><<<c->n, 512, smem, c->stream>>>(c->d_opp, c->d_memb, c->d_order, c->n, c->T,
                                                                       dS, c->d_pairs);
            RFX_CUDA(cudaGetLastError());
            return RFX_OK;
        });
    }
    const int win = pairs_window(c);
    const size_t smem = (size_t)win * sizeof(uint32_t);
    if (rfx_status s0 = allow_dyn_smem(pairs_row_kernel, dev_smem)) return s0;
    RFX_CUDA(cudaMemsetAsync(c->d_pairs, 0, sizeof(unsigned long long), c->stream));
    StageTimer st(c, ST_PAIRS, 1);
    dim3 grid(c->n, (c->n + win - 1) / win);
    pairs_row_kernel<<<grid, ROW_THREADS, smem, c->stream>>>(c->d_key, c->d_segoff, c->d_segbase, c->d_memb, c->n,
                                                             c->T, win, dS, c->d_pairs);
    RFX_CUDA(cudaGetLastError());
    return RFX_OK;
}

// Pair-count pipeline on caller-provided device buffers (no context, no
// allocation): leaf lists, opposite ranges, row order, then the full-row
// kernel.  Used by the allocation-free entry point in noalloc.cu.
rfx_status launch_pairs_pipeline_raw(const PairsRawArgs& a, cudaStream_t stream) {
    int dev = 0, dev_smem = 0;
    RFX_CUDA(cudaGetDevice(&dev));
    RFX_CUDA(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const int max_keys = 2 * a.max_leaves;
    int smem_keys = std::min(max_keys + 1, (dev_smem - 1024) / 4);
    smem_keys = std::max(smem_keys, 32);
    const size_t smem = (size_t)smem_keys * sizeof(int32_t);
    if (rfx_status s0 = allow_dyn_smem(build_csr_kernel<int32_t>, dev_smem)) return s0;
    build_csr_kernel<int32_t><<<a.T, CSR_THREADS, smem, stream>>>(a.key, a.n, a.segbase, a.segoff, a.memb, smem_keys,
                                                         a.err);
    RFX_CUDA(cudaGetLastError());
    if (max_keys + 1 > smem_keys) {
        fix_global_segoff_kernel<<<a.T, 32, 0, stream>>>(a.segbase, a.segoff, smem_keys);
        RFX_CUDA(cudaGetLastError());
    }
    dim3 g((a.n + OPP_TILE - 1) / OPP_TILE, (a.T + OPP_TILE - 1) / OPP_TILE);
    opp_kernel<<<g, OPP_TILE * 8, 0, stream>>>(a.key, a.segoff, a.segbase, a.memb, a.n, a.T, nullptr, a.opp);
    RFX_CUDA(cudaGetLastError());
    row_order_kernel<<<1, 1024, 0, stream>>>(a.key, a.segoff, a.segbase, a.memb, a.n, a.order);
    RFX_CUDA(cudaGetLastError());
    const size_t smem2 = (size_t)r16_words(a.n) * sizeof(uint32_t);
    if (rfx_status s0 = allow_dyn_smem(pairs_row16_kernel<R16_THREADS>, dev_smem)) return s0;
    pairs_row16_kernel<R16_THREADS><<<a.n, R16_THREADS, smem2, stream>>>(a.opp, a.memb, a.order, a.n, a.T, a.S,
                                                                         nullptr);
    RFX_CUDA(cudaGetLastError());
    return RFX_OK;
}

namespace {
// Grid of the finishprox kernel: x = run within a row-tile pair, y = pair.
dim3 finishprox_grid(int n) {
    const int nt = (n + FP_TILE - 1) / FP_TILE;
    int bx = 1;
    for (int I = 0; I < (nt + 1) / 2; ++I) {
        const int I2 = nt - 1 - I;
        bx = std::max(bx, fp_runs(nt, I) + (I2 > I ? fp_runs(nt, I2) : 0));
    }
    return dim3(bx, (nt + 1) / 2);
}

template <typename TS>
rfx_status finishprox_run(Ctx* c, const TS* dS, float* dP, int full) {
    StageTimer st(c, ST_FINISHPROX, 2);
    Scratch sc(c);
    double* inv = sc.get<double>((size_t)c->n);
    if (!inv) {
        set_error("finishprox: scratch allocation failed");
        return RFX_ERR_OOM;
    }
    finish_inv_kernel<<<(c->n + 255) / 256, 256, 0, c->stream>>>(c->d_nout, c->n, inv);
    RFX_CUDA(cudaGetLastError());
    finishprox_kernel<TS><<<finishprox_grid(c->n), FP_TILE * 8, 0, c->stream>>>(dS, inv, c->n, full, dP);
    RFX_CUDA(cudaGetLastError());
    return RFX_OK;
}
}  // namespace

rfx_status launch_finishprox(Ctx* c, const int32_t* dS, float* dP, int full) {
    return finishprox_run<int32_t>(c, dS, dP, full);
}

// finishprox of FP64 sums (case-wise weights): the same arithmetic on
// S = C + C^T in double
rfx_status launch_finishprox_f64(Ctx* c, const double* dS, float* dP, int full) {
    return finishprox_run<double>(c, dS, dP, full);
}

}  // namespace rfx
