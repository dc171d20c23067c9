// Forest producer: a partition-based restatement of the reference's CPU
// grower, so that forests of the analysis workloads can be made where the
// reference is not available.  It is NOT on the GPU analysis path; it only
// produces that path's input.
//
// Semantics followed (chriskuchar/RFX):
//   * bootstrap: cpu_bootstrap (src/rf_bootstrap.cpp:14-82) — MT19937 seeded
//     12345 + tree, i = (int)(randomu() * n) clamped to n-1, nin[i]++;
//     jinbag = in-bag samples in ascending order.
//   * growth: cpu_growtree (src/rf_growtree.cpp:382-945) — MT19937 seeded
//     iseed + tree; nodes processed in creation order; a node's samples are the
//     distinct in-bag samples reaching it (ascending); terminal when smaller
//     than minndsize or pure; otherwise mtry features drawn as
//     (int)(randomu() * p); each candidate sorts (value, sample) pairs and
//     scans split points, skipping ties BEFORE updating the running class
//     weights (:626-629), with the Gini criterion rln/rld + rrn/rrd in float;
//     strict '>' keeps the first best; the split value is the left sample's
//     value; children are (nnode, nnode+1); terminal class = majority with
//     strict '>' (lowest class on ties).
//   The reference finds a node's samples by re-routing every in-bag sample from
//   the root (O(nodes * n * depth)); a stable partition of the parent's
//   ascending sample list gives the same sets in the same order.
//
// Determinism: every tree depends only on (data, tree id, seeds), so trees are
// grown in parallel threads with identical results.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

namespace rfxhost {

namespace {

struct MT {
    uint32_t mt[624];
    int mti = 625;
    void seed(uint32_t s) {
        mt[0] = s;
        for (mti = 1; mti < 624; ++mti) mt[mti] = 1812433253UL * (mt[mti - 1] ^ (mt[mti - 1] >> 30)) + (uint32_t)mti;
    }
    double grnd() {
        static const uint32_t mag01[2] = {0x0UL, 0x9908b0dfUL};
        uint32_t y;
        if (mti >= 624) {
            if (mti == 625) seed(5489UL);
            int kk;
            for (kk = 0; kk < 624 - 397; ++kk) {
                y = (mt[kk] & 0x80000000UL) | (mt[kk + 1] & 0x7fffffffUL);
                mt[kk] = mt[kk + 397] ^ (y >> 1) ^ mag01[y & 1];
            }
            for (; kk < 623; ++kk) {
                y = (mt[kk] & 0x80000000UL) | (mt[kk + 1] & 0x7fffffffUL);
                mt[kk] = mt[kk + (397 - 624)] ^ (y >> 1) ^ mag01[y & 1];
            }
            y = (mt[623] & 0x80000000UL) | (mt[0] & 0x7fffffffUL);
            mt[623] = mt[396] ^ (y >> 1) ^ mag01[y & 1];
            mti = 0;
        }
        y = mt[mti++];
        y ^= (y >> 11);
        y ^= (y << 7) & 0x9d2c5680UL;
        y ^= (y << 15) & 0xefc60000UL;
        y ^= (y >> 18);
        return (double)y / (double)0xffffffffUL;
    }
    float randomu() { return (float)grnd(); }
};

// Order-preserving map of a float to uint32 (ascending), with -0.0 folded onto
// +0.0 because std::pair<float,int> compares them equal (then by index).
inline uint32_t fkey(float v) {
    if (v == 0.0f) v = 0.0f;
    uint32_t u;
    std::memcpy(&u, &v, 4);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

struct TreeOut {
    std::vector<int32_t> ns, bv, tm, nc;
    std::vector<float> xs;
};

// Sorted (value key, sample) lists kept for one large node and handed down to
// its larger child: when a split peels only a few samples off a big node (long
// chains of such splits occur where a forest isolates scattered points one at
// a time), the child's sorted order per feature is the parent's minus the
// peeled samples, which are marked dead instead of re-sorting.  Lists are built
// per feature on first use and compacted once half their entries are dead.
struct FeatSlot {
    int owner = -1;                            // node the lists describe
    int live = 0;                              // its sample count
    long long used = 0;                        // last use (for eviction)
    std::vector<std::vector<uint64_t>> lists;  // per feature; empty = not built
    std::vector<std::vector<uint16_t>> cls;    // class of each list entry (sequential reads)
    std::vector<uint64_t> dead;                // bit per sample: peeled off since the lists were built
    bool is_dead(uint32_t i) const { return (dead[i >> 6] >> (i & 63)) & 1u; }
    void set_dead(uint32_t i, bool d) {
        if (d) dead[i >> 6] |= 1ull << (i & 63);
        else dead[i >> 6] &= ~(1ull << (i & 63));
    }
};
// Several chains (one per dense cluster) grow side by side in the node order,
// so a few slots are kept, each with its own dead flags.
constexpr int FEAT_SLOTS = 8;
struct FeatCache {
    FeatSlot slot[FEAT_SLOTS];
    long long clock = 0;
};

struct Work {
    std::vector<int32_t> idx, tmp;       // node sample lists (ascending within a node)
    std::vector<int32_t> start, stop;    // node ranges into idx
    std::vector<uint64_t> keys, keys2;
    std::vector<float> cc, wl, wr;
    std::vector<float> ca, cb, cc2, cd, crit;  // candidate splits of one feature scan
    std::vector<int32_t> cn;
    FeatCache fc;
};

// Gini criterion (rln / rld) + (rrn / rrd) of every candidate; the same IEEE
// divisions and addition as one at a time, vectorised where the CPU allows.
__attribute__((target_clones("avx2", "default")))
void gini_crit(const float* a, const float* b, const float* c, const float* d, float* out, int m) {
    for (int i = 0; i < m; ++i) out[i] = (a[i] / b[i]) + (c[i] / d[i]);
}

int cache_min_samples() {
    static const int v = [] {
        const char* e = std::getenv("RFX_GROW_CACHE_MIN");
        const int x = e ? std::atoi(e) : 0;
        return x > 0 ? x : 16384;
    }();
    return v;
}

// Majority class with strict '>' and initial max 0 (class 0 when empty).
inline int majority(const float* cc, int c) {
    int maj = 0;
    float mx = 0.0f;
    for (int j = 0; j < c; ++j)
        if (cc[j] > mx) { mx = cc[j]; maj = j; }
    return maj;
}

// Sorts (value key << 32 | sample) pairs.  The samples of a node arrive in
// ascending order, so a stable LSD radix sort on the value half gives the same
// order as sorting the whole 64-bit keys; large nodes use it (3 passes of 11
// bits, a pass skipped when all keys share its digit), small ones std::sort.
void sort_keys(uint64_t* keys, int m, Work& w) {
    if (m < 4096) {
        std::sort(keys, keys + m);
        return;
    }
    if ((int)w.keys2.size() < m) w.keys2.resize(m);
    uint64_t* a = keys;
    uint64_t* b = w.keys2.data();
    static const int SH[3] = {32, 43, 54};
    static const int BITS[3] = {11, 11, 10};
    std::vector<int> cnt(2048);
    for (int pass = 0; pass < 3; ++pass) {
        const int sh = SH[pass], nb = 1 << BITS[pass];
        const uint64_t mask = (uint64_t)nb - 1;
        std::fill(cnt.begin(), cnt.begin() + nb, 0);
        for (int q = 0; q < m; ++q) cnt[(a[q] >> sh) & mask]++;
        if (cnt[(a[0] >> sh) & mask] == m) continue;  // one digit: order unchanged
        int run = 0;
        for (int d = 0; d < nb; ++d) {
            const int c = cnt[d];
            cnt[d] = run;
            run += c;
        }
        for (int q = 0; q < m; ++q) b[cnt[(a[q] >> sh) & mask]++] = a[q];
        std::swap(a, b);
    }
    if (a != keys) std::memcpy(keys, a, sizeof(uint64_t) * (size_t)m);
}

void grow_one(const float* Xc /* p x n column-major */, const int32_t* y, int n, int p, int nclass, int mtry,
              int minndsize, int maxnode, uint32_t grow_seed, const int32_t* nin, TreeOut& out, Work& w) {
    // root sample list: in-bag samples ascending (jinbag)
    w.idx.clear();
    for (int i = 0; i < n; ++i)
        if (nin[i] > 0) w.idx.push_back(i);
    const int ninbag = (int)w.idx.size();
    w.tmp.resize(ninbag > 0 ? ninbag : 1);
    w.keys.resize(ninbag > 0 ? ninbag : 1);
    for (auto* v : {&w.ca, &w.cb, &w.cc2, &w.cd, &w.crit}) v->resize(ninbag > 0 ? ninbag : 1);
    w.cn.resize(ninbag > 0 ? ninbag : 1);
    out.ns.assign(1, 2);
    out.bv.assign(1, 0);
    out.xs.assign(1, 0.0f);
    out.tm.assign(2, 0);
    out.nc.assign(1, 0);
    w.start.assign(1, 0);
    w.stop.assign(1, ninbag);
    w.cc.assign(nclass, 0.0f);
    w.wl.assign(nclass, 0.0f);
    w.wr.assign(nclass, 0.0f);
    MT rng;
    rng.seed(grow_seed);
    const int min_size = (nclass == 1) ? 2 * minndsize : minndsize;
    const int cmin = cache_min_samples();
    FeatCache& fc = w.fc;
    for (FeatSlot& sl : fc.slot) {
        sl.owner = -1;
        sl.lists.resize(p);
        sl.cls.resize(p);
        if (sl.dead.size() < (size_t)(n + 63) / 64) sl.dead.assign((n + 63) / 64, 0ull);
    }
    int nnode = 1;
    for (int k = 0; k < nnode; ++k) {
        if (out.ns[k] != 2) continue;
        const int s = w.start[k], e = w.stop[k], m = e - s;
        if (m < min_size) {
            out.ns[k] = -1;
            continue;
        }
        float* cc = w.cc.data();
        std::fill(cc, cc + nclass, 0.0f);
        for (int q = s; q < e; ++q) {
            int cl = y[w.idx[q]];
            if (cl >= 0 && cl < nclass) cc[cl] += 1.0f;
        }
        int nonzero = 0, maj = 0;
        float mx = 0.0f;
        for (int j = 0; j < nclass; ++j)
            if (cc[j] > 0.0f) {
                nonzero++;
                if (cc[j] > mx) { mx = cc[j]; maj = j; }
            }
        if (nonzero <= 1) {
            out.ns[k] = -1;
            out.nc[k] = maj;
            continue;
        }
        float best = -2.0f, best_split = 0.0f;
        int best_var = 0;
        bool found = false;
        // large nodes keep (or take over from their parent) sorted lists
        const bool cached = m >= cmin && nclass <= 65535;
        FeatSlot* sl = nullptr;
        if (cached) {
            for (FeatSlot& x : fc.slot)
                if (x.owner == k) sl = &x;
            if (!sl) {  // a free slot, else the least recently used one
                sl = &fc.slot[0];
                for (FeatSlot& x : fc.slot) {
                    if (x.owner < 0) {
                        sl = &x;
                        break;
                    }
                    if (x.used < sl->used) sl = &x;
                }
                sl->owner = k;
                sl->live = m;
                for (auto& l : sl->lists) l.clear();
                for (int q = s; q < e; ++q) sl->set_dead(w.idx[q], false);
            }
            sl->used = ++fc.clock;
        }
        for (int mv = 0; mv < mtry; ++mv) {
            float r = rng.randomu();
            int mvar = (int)(r * (float)p);
            if (mvar >= p) mvar = p - 1;
            float rrn = 0.0f, rrd = 0.0f;
            for (int j = 0; j < nclass; ++j) {
                rrn += cc[j] * cc[j];
                rrd += cc[j];
            }
            float rln = 0.0f, rld = 0.0f;
            float* wl = w.wl.data();
            float* wr = w.wr.data();
            for (int j = 0; j < nclass; ++j) {
                wl[j] = 0.0f;
                wr[j] = cc[j];
            }
            const float* col = Xc + (size_t)mvar * n;
            const uint64_t* sorted;
            const uint16_t* scls = nullptr;  // classes of the cached list entries
            int len;
            if (cached) {
                std::vector<uint64_t>& l = sl->lists[mvar];
                std::vector<uint16_t>& lc = sl->cls[mvar];
                if (l.empty()) {
                    l.resize(m);
                    for (int q = 0; q < m; ++q) {
                        const int i = w.idx[s + q];
                        l[q] = ((uint64_t)fkey(col[i]) << 32) | (uint32_t)i;
                    }
                    sort_keys(l.data(), m, w);
                    lc.resize(m);
                    for (int q = 0; q < m; ++q) lc[q] = (uint16_t)y[(uint32_t)l[q]];
                } else if ((int)l.size() > 2 * sl->live) {
                    size_t o = 0;
                    for (size_t q = 0; q < l.size(); ++q)
                        if (!sl->is_dead((uint32_t)l[q])) {
                            l[o] = l[q];
                            lc[o] = lc[q];
                            ++o;
                        }
                    l.resize(o);
                    lc.resize(o);
                }
                sorted = l.data();
                scls = lc.data();
                len = (int)l.size();
            } else {
                uint64_t* keys = w.keys.data();
                for (int q = 0; q < m; ++q) {
                    int i = w.idx[s + q];
                    keys[q] = ((uint64_t)fkey(col[i]) << 32) | (uint32_t)i;
                }
                sort_keys(keys, m, w);
                sorted = keys;
                len = m;
            }
            // element `cur` moves to the left side when its value differs from
            // the next sample's (ties are skipped, as the reference does); fkey
            // is monotonic and maps -0 to +0, so equal value keys are exactly
            // the pairs with v1 >= v2
            // pass 1 (sequential running sums) records every candidate split;
            // pass 2 evaluates the Gini criteria with vector divisions; the
            // first position of the largest criterion is the one the
            // sequential "crit > best" rule keeps
            float* ca = w.ca.data();
            float* cb = w.cb.data();
            float* cc2 = w.cc2.data();
            float* cd = w.cd.data();
            int32_t* cn = w.cn.data();
            int nc_cand = 0;
            int prev = -1;
            for (int q = 0; q < len; ++q) {
                const uint64_t kq = sorted[q];
                if (cached && sl->is_dead((uint32_t)kq)) continue;
                if (prev >= 0) {
                    const uint64_t kp = sorted[prev];
                    if ((kp >> 32) != (kq >> 32)) {
                        const int nc = (int)(uint32_t)kp;
                        const int kc = scls ? (int)scls[prev] : y[nc];
                        const float u = 1.0f;
                        rln += u * (u + 2.0f * wl[kc]);
                        rrn += u * (u - 2.0f * wr[kc]);
                        rld += u;
                        rrd -= u;
                        wl[kc] += u;
                        wr[kc] -= u;
                        if (std::min(rrd, rld) > 1.0e-5f) {
                            ca[nc_cand] = rln;
                            cb[nc_cand] = rld;
                            cc2[nc_cand] = rrn;
                            cd[nc_cand] = rrd;
                            cn[nc_cand] = nc;
                            ++nc_cand;
                        }
                    }
                }
                prev = q;
            }
            if (nc_cand > 0) {
                float* crit = w.crit.data();
                gini_crit(ca, cb, cc2, cd, crit, nc_cand);
                int bi = 0;
                for (int q = 1; q < nc_cand; ++q)
                    if (crit[q] > crit[bi]) bi = q;
                if (crit[bi] > best) {
                    best = crit[bi];
                    best_var = mvar;
                    best_split = col[cn[bi]];
                    found = true;
                }
            }
        }
        if (!found || best < -1.0f || nnode + 2 > maxnode) {
            out.ns[k] = -1;
            out.nc[k] = maj;
            if (sl) sl->owner = -1;
            continue;
        }
        out.ns[k] = 1;
        out.bv[k] = best_var;
        out.xs[k] = best_split;
        out.tm[2 * k] = nnode;
        out.tm[2 * k + 1] = nnode + 1;
        // stable partition of [s, e) into left (x <= split) then right
        const float* col = Xc + (size_t)best_var * n;
        int nl = 0, nr = 0;
        for (int q = s; q < e; ++q) {
            int i = w.idx[q];
            if (col[i] <= best_split) w.idx[s + nl++] = i;
            else w.tmp[nr++] = i;
        }
        std::memcpy(&w.idx[s + nl], w.tmp.data(), sizeof(int32_t) * nr);
        if (sl) {
            // the larger child inherits the lists; the other child's samples die
            const bool left_big = nl >= nr;
            const int big = left_big ? nl : nr;
            if (big >= cmin) {
                const int q0 = left_big ? s + nl : s, q1 = left_big ? e : s + nl;
                for (int q = q0; q < q1; ++q) sl->set_dead(w.idx[q], true);
                sl->owner = left_big ? nnode : nnode + 1;
                sl->live = big;
            } else {
                sl->owner = -1;
            }
        }
        for (int c2 = 0; c2 < 2; ++c2) {
            out.ns.push_back(2);
            out.bv.push_back(0);
            out.xs.push_back(0.0f);
            out.tm.push_back(0);
            out.tm.push_back(0);
            out.nc.push_back(0);
        }
        w.start.push_back(s);
        w.stop.push_back(s + nl);
        w.start.push_back(s + nl);
        w.stop.push_back(e);
        nnode += 2;
    }
    // finalize terminal classes over each terminal node's samples
    for (int k = 0; k < nnode; ++k) {
        if (out.ns[k] != -1) continue;
        float* cc = w.cc.data();
        std::fill(cc, cc + nclass, 0.0f);
        for (int q = w.start[k]; q < w.stop[k]; ++q) {
            int cl = y[w.idx[q]];
            if (cl >= 0 && cl < nclass) cc[cl] += 1.0f;
        }
        out.nc[k] = majority(cc, nclass);
    }
}

}  // namespace

void bootstrap(int n, int tree, int32_t* nin) {
    MT rng;
    rng.seed((uint32_t)(12345 + tree));
    std::memset(nin, 0, sizeof(int32_t) * (size_t)n);
    for (int k = 0; k < n; ++k) {
        float u = rng.randomu();
        int i = (int)(u * (float)n);
        if (i >= n) i = n - 1;
        if (i < 0) i = 0;
        nin[i]++;
    }
}

// Grows trees [0, ntree) and returns them compactly.  offs has ntree+1
// entries; node arrays are appended in tree order.
int grow_forest(const float* X, const int32_t* y, int n, int p, int nclass, int ntree, int mtry, int minndsize,
                int maxnode, int iseed, int nthreads, std::vector<int64_t>& offs, std::vector<int32_t>& nodestatus,
                std::vector<int32_t>& bestvar, std::vector<float>& xbestsplit, std::vector<int32_t>& treemap,
                std::vector<int32_t>& nodeclass, int32_t* nin_all) {
    std::vector<float> Xc((size_t)n * p);
    for (int i = 0; i < n; ++i)
        for (int f = 0; f < p; ++f) Xc[(size_t)f * n + i] = X[(size_t)i * p + f];
    std::vector<TreeOut> trees(ntree);
    std::atomic<int> next{0};
    if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
    nthreads = std::min(nthreads, std::max(ntree, 1));
    auto worker = [&]() {
        Work w;
        for (;;) {
            int t = next.fetch_add(1);
            if (t >= ntree) break;
            int32_t* nin = nin_all + (size_t)t * n;
            bootstrap(n, t, nin);
            grow_one(Xc.data(), y, n, p, nclass, mtry, minndsize, maxnode, (uint32_t)(iseed + t), nin, trees[t], w);
        }
    };
    std::vector<std::thread> pool;
    for (int k = 1; k < nthreads; ++k) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    offs.assign(ntree + 1, 0);
    for (int t = 0; t < ntree; ++t) offs[t + 1] = offs[t] + (int64_t)trees[t].ns.size();
    const size_t N = (size_t)offs[ntree];
    nodestatus.resize(N);
    bestvar.resize(N);
    xbestsplit.resize(N);
    treemap.resize(2 * N);
    nodeclass.resize(N);
    for (int t = 0; t < ntree; ++t) {
        const size_t o = (size_t)offs[t];
        const TreeOut& tr = trees[t];
        std::copy(tr.ns.begin(), tr.ns.end(), nodestatus.begin() + o);
        std::copy(tr.bv.begin(), tr.bv.end(), bestvar.begin() + o);
        std::copy(tr.xs.begin(), tr.xs.end(), xbestsplit.begin() + o);
        std::copy(tr.tm.begin(), tr.tm.end(), treemap.begin() + 2 * o);
        std::copy(tr.nc.begin(), tr.nc.end(), nodeclass.begin() + o);
    }
    return 0;
}

}  // namespace rfxhost
