/*
 * ORACLE — test infrastructure, not product code.
 *
 * A plain-C restatement of the reference's post-growth CPU path
 * (chriskuchar/RFX), used only by tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py as the checker.  Every function cites the
 * reference file:line whose behaviour it restates.  The oracle is pinned
 * against the reference itself (oracle/_ref/librfxref.so built from the
 * reference's own sources) by tests/test_oracle_vs_reference.py and against
 * committed golden fixtures in tests/golden/.
 *
 * Forest layout shared with the product library (compact, 0-based):
 *   tree t owns nodes [offs[t], offs[t] + nnode[t]) of nodestatus, bestvar,
 *   xbestsplit, nodeclass; treemap holds 2 ints per node (left, right);
 *   catgoleft (optional, may be NULL = all zero) holds maxcat ints per node.
 *   nin is T x n (bootstrap multiplicity), X is n x p float32 row-major.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

/* ------------------------------------------------------------------------ */
/* MT19937 as the reference implements it (include/rf_utils.hpp:74-141).      */
/* grnd() = y / 0xffffffff in double; randomu() = (float)grnd().              */
/* ------------------------------------------------------------------------ */
typedef struct {
    uint32_t mt[624];
    int mti;
} orc_mt;

static void mt_seed(orc_mt* s, uint32_t seed) {
    s->mt[0] = seed;
    for (s->mti = 1; s->mti < 624; s->mti++)
        s->mt[s->mti] = (1812433253UL * (s->mt[s->mti - 1] ^ (s->mt[s->mti - 1] >> 30)) + (uint32_t)s->mti);
}

static double mt_grnd(orc_mt* s) {
    static const uint32_t mag01[2] = {0x0UL, 0x9908b0dfUL};
    uint32_t y;
    int kk;
    if (s->mti >= 624) {
        for (kk = 0; kk < 624 - 397; kk++) {
            y = (s->mt[kk] & 0x80000000UL) | (s->mt[kk + 1] & 0x7fffffffUL);
            s->mt[kk] = s->mt[kk + 397] ^ (y >> 1) ^ mag01[y & 1];
        }
        for (; kk < 623; kk++) {
            y = (s->mt[kk] & 0x80000000UL) | (s->mt[kk + 1] & 0x7fffffffUL);
            s->mt[kk] = s->mt[kk + (397 - 624)] ^ (y >> 1) ^ mag01[y & 1];
        }
        y = (s->mt[623] & 0x80000000UL) | (s->mt[0] & 0x7fffffffUL);
        s->mt[623] = s->mt[396] ^ (y >> 1) ^ mag01[y & 1];
        s->mti = 0;
    }
    y = s->mt[s->mti++];
    y ^= (y >> 11);
    y ^= (y << 7) & 0x9d2c5680UL;
    y ^= (y << 15) & 0xefc60000UL;
    y ^= (y >> 18);
    return (double)y / (double)0xffffffffUL;
}

static float mt_randomu(orc_mt* s) { return (float)mt_grnd(s); }

/*
 * Permutation of OOB positions used by cpu_permobmr (src/rf_varimp.cpp:16-30):
 * pjoob starts as joob, then for i < noob: j = (int)(randomu() * noob);
 * swap(pjoob[i], pjoob[j]).  The stream is MT19937 seeded 42 afresh on every
 * call, so the permutation depends on noob only.  perm[r] is the OOB position
 * whose sample is used in place of position r.
 *
 * When randomu() rounds to 1.0f, j == noob and the reference swaps with the
 * element one past the end of its vector (undefined behaviour).  The oracle
 * returns the number of such draws (the caller must treat that noob as
 * unpinned) and uses j = noob - 1 in their place.
 */
int orc_perm(int noob, int32_t* perm) {
    orc_mt s;
    int bad = 0;
    mt_seed(&s, 42u);
    for (int i = 0; i < noob; ++i) perm[i] = i;
    for (int i = 0; i < noob; ++i) {
        float u = mt_randomu(&s);
        int j = (int)(u * (float)noob);
        if (j >= noob) { j = noob - 1; ++bad; }
        int32_t tmp = perm[i];
        perm[i] = perm[j];
        perm[j] = tmp;
    }
    return bad;
}

/* Bootstrap multiplicities of cpu_bootstrap (src/rf_bootstrap.cpp:14-82):
 * MT19937 seeded 12345 + tree (g_config.iseed is never assigned, so the
 * user's iseed does not reach it), i = (int)(randomu() * n), clamped.        */
void orc_bootstrap(int n, int tree, int32_t* nin) {
    orc_mt s;
    mt_seed(&s, (uint32_t)(12345 + tree));
    memset(nin, 0, sizeof(int32_t) * (size_t)n);
    for (int k = 0; k < n; ++k) {
        float u = mt_randomu(&s);
        int i = (int)(u * (float)n);
        if (i >= n) i = n - 1;
        if (i < 0) i = 0;
        nin[i]++;
    }
}

/* ------------------------------------------------------------------------ */
/* Routing variants.                                                         */
/* ------------------------------------------------------------------------ */

/* cpu_testreebag (src/rf_testreebag.cpp:13-125) for one OOB sample.
 * Returns the node id (nodextr) and writes the class (jtr).                 */
static int route_testreebag(const float* xrow, int p, const int32_t* ns, const int32_t* bv,
                            const float* xs, const int32_t* tm, const int32_t* nc, int nnode,
                            const int32_t* cat, const int32_t* cgl, int maxcat, int32_t* cls) {
    int kt = 0, steps = 0;
    while (ns[kt] == 1 && steps < 1000) {
        steps++;
        if (steps >= 1000) break;
        int m = bv[kt];
        if (m < 0 || m >= p) break;
        if (cat == NULL || cat[m] == 1) {
            kt = (xrow[m] <= xs[kt]) ? tm[2 * kt] : tm[2 * kt + 1];
        } else {
            int v = (int)xrow[m];
            if (v >= 0 && v < cat[m]) {
                int gl = cgl ? cgl[(size_t)kt * maxcat + v] : 0;
                kt = (gl == 1) ? tm[2 * kt] : tm[2 * kt + 1];
            } else {
                kt = tm[2 * kt + 1];
            }
        }
        if (kt < 0 || kt >= nnode) { kt = 0; break; }
        if (ns[kt] != 1) break;
    }
    if (ns[kt] == -1 || ns[kt] == 2) {
        *cls = nc[kt];
        return kt;
    }
    *cls = nc[0];
    return 0;
}

/* RandomForest::find_terminal_node (src/rf_random_forest.cpp:2194-2244) used
 * for in-bag samples before cpu_proximity (:1295-1303).  maxnode is the loop
 * bound of the reference (2n+1).                                            */
static int route_terminal(const float* xrow, int p, const int32_t* ns, const int32_t* bv,
                          const float* xs, const int32_t* tm, const int32_t* cat,
                          const int32_t* cgl, int maxcat, int maxnode) {
    int cur = 0;
    for (int k = 0; k < maxnode; ++k) {
        if (ns[cur] == -1) return cur;
        int m = bv[cur];
        if (m >= 0 && m < p) {
            float v = xrow[m];
            if (cat[m] == 1) {
                cur = (v <= xs[cur]) ? tm[2 * cur] : tm[2 * cur + 1];
            } else {
                int j = (int)((double)v + 0.5);
                if (j >= 1 && j <= cat[m]) {
                    int gl = cgl ? cgl[(size_t)cur * maxcat + (j - 1)] : 0;
                    cur = (gl == 1) ? tm[2 * cur] : tm[2 * cur + 1];
                } else {
                    return 0;
                }
            }
        } else {
            return 0;
        }
    }
    return 0;
}

/* cpu_testreeimp traversal (src/rf_varimp.cpp:45-103) for one OOB sample with
 * feature mr taken from row xperm instead of xrow.  Returns 1 and sets
 * *cls/*node when a terminal node is reached, 0 when the reference would
 * break without assigning (its jvr slot then keeps a stale value).           */
static int route_testreeimp(const float* xrow, const float* xperm, int mr, int p, const int32_t* ns,
                            const int32_t* bv, const float* xs, const int32_t* tm, const int32_t* nc,
                            int nnode, const int32_t* cat, const int32_t* cgl, int maxcat,
                            int32_t* cls, int32_t* node) {
    int kt = 0;
    for (int k = 0; k < nnode; ++k) {
        if (ns[kt] == -1) {
            *cls = nc[kt];
            *node = kt;
            return 1;
        }
        int m = bv[kt];
        if (m < 0 || m >= p) return 0;
        float xmn = (m == mr) ? xperm[m] : xrow[m];
        if (cat == NULL || cat[m] == 1) {
            kt = (xmn <= xs[kt]) ? tm[2 * kt] : tm[2 * kt + 1];
        } else {
            int jcat = (int)(xmn + 0.5f);
            if (jcat >= 0 && jcat < maxcat) {
                int gl = cgl ? cgl[(size_t)kt * maxcat + jcat] : 0;
                kt = (gl == 1) ? tm[2 * kt] : tm[2 * kt + 1];
            } else {
                return 0;
            }
        }
    }
    return 0;
}

/* The in-bag walk of grow_tree_single's casewise tnodewt block
 * (src/rf_random_forest.cpp:1052-1095): categorical splits take
 * idx = (int)(x + 0.5f) and go left iff 0 <= idx < maxcat and the go-left
 * table says 1 (otherwise right); numeric splits go left iff x <= split; the
 * walk runs while the node status is 1 and stops at a child outside
 * [0, nnode).  Returns the node reached (checked by the caller).            */
static int route_tnodewt(const float* xrow, int p, const int32_t* ns, const int32_t* bv, const float* xs,
                         const int32_t* tm, const int32_t* cat, const int32_t* cgl, int maxcat, int nnode) {
    int cur = 0;
    while (ns[cur] == 1) {
        int m = bv[cur];
        int numcat = (cat == NULL || m >= p) ? 1 : cat[m];
        int left;
        if (numcat > 1) {
            int idx = (int)(xrow[m] + 0.5f);
            left = (idx >= 0 && idx < maxcat && cgl != NULL && cgl[(size_t)cur * maxcat + idx] == 1);
        } else {
            left = xrow[m] <= xs[cur];
        }
        cur = tm[2 * cur + (left ? 0 : 1)];
        if (cur < 0 || cur >= nnode) break;
    }
    return cur;
}

/* Predict traversal (src/rf_random_forest.cpp:1959-2013): returns the voted
 * class (0 on every invalid path), as predict_classification counts it.     */
static int route_predict(const float* xrow, int p, int nclass, const int32_t* ns, const int32_t* bv,
                         const float* xs, const int32_t* tm, const int32_t* nc, const int32_t* cat,
                         const int32_t* cgl, int maxcat, int maxnode) {
    int kt = 0;
    for (int k = 0; k < maxnode; ++k) {
        if (kt >= maxnode) return 0;
        if (ns[kt] == -1) {
            int c = nc[kt];
            return (c >= 0 && c < nclass) ? c : 0;
        }
        int m = bv[kt];
        if (m >= 0 && m < p) {
            float v = xrow[m];
            if (cat[m] == 1) {
                kt = (v <= xs[kt]) ? tm[2 * kt] : tm[2 * kt + 1];
            } else {
                int j = (int)((double)v + 0.5);
                if (j >= 1 && j <= cat[m]) {
                    int gl = cgl ? cgl[(size_t)kt * maxcat + (j - 1)] : 0;
                    kt = (gl == 1) ? tm[2 * kt] : tm[2 * kt + 1];
                } else {
                    return 0;
                }
            }
        } else {
            return 0;
        }
    }
    /* loop bound reached without a terminal node: no vote in the reference */
    return -1;
}

/* ------------------------------------------------------------------------ */
/* Packed upper-triangle index (row-major, diagonal included).               */
/* ------------------------------------------------------------------------ */
static inline size_t upidx(int64_t n, int64_t i, int64_t j) {
    return (size_t)(i * n - (i * (i - 1)) / 2 + (j - i));
}

/* ------------------------------------------------------------------------ */
/* Whole-forest analysis in the reference's per-tree order                   */
/* (src/rf_random_forest.cpp:1043-1309 per tree, then :2413-2462, :2246-2301, */
/* :1637-1852).                                                               */
/*                                                                            */
/* Outputs (any may be NULL to skip):                                         */
/*   q_raw[n*c]  float OOB votes before normalisation (:1107-1153)            */
/*   nout[n]     doubled OOB counts (src/rf_bootstrap.cpp:61 and :1110)       */
/*   qimp[n], qimpm[n*p] (sample-major, before localimp), avimp[p], sqsd[p]   */
/*   S[n(n+1)/2] int32: S_ij = C_ij + C_ji for i<j, where C is the raw pair   */
/*               count cpu_proximity's dense branch accumulates (:99-231);    */
/*               diagonal 0                                                   */
/*   leaf[T*n]   per-tree node id each sample ends in (OOB: testreebag,       */
/*               in-bag: find_terminal_node)                                  */
/*   jtr[T*n]    testreebag class for OOB samples, 0 for in-bag               */
/*   perm_bad    number of trees whose permutation hit j == noob              */
/* impn selects local importance (qimp/qimpm).                                */
/* ------------------------------------------------------------------------ */
int orc_analyse(const float* X, const int32_t* y, const int32_t* cat, int n, int p, int nclass, int maxcat,
                int T, const int64_t* offs, const int32_t* nnode, const int32_t* nodestatus,
                const int32_t* bestvar, const float* xbestsplit, const int32_t* treemap,
                const int32_t* nodeclass, const int32_t* catgoleft, const int32_t* nin_all,
                int do_imp, int impn, int do_prox, int casewise,
                float* q_raw, int32_t* nout, float* qimp, float* qimpm, float* avimp, float* sqsd,
                int32_t* S, double* Cw, int32_t* leaf, int32_t* jtr_out, int32_t* perm_bad) {
    const int maxnode = 2 * n + 1;
    int32_t* jtr = (int32_t*)calloc((size_t)n, sizeof(int32_t));
    int32_t* nodextr = (int32_t*)calloc((size_t)n, sizeof(int32_t));
    int32_t* joob = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int32_t* perm = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int32_t* jvr = (int32_t*)calloc((size_t)n, sizeof(int32_t));
    int32_t* nod = (int32_t*)malloc(sizeof(int32_t) * (size_t)maxnode);
    int32_t* ncount = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int32_t* ncn = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int32_t* nodexb = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int32_t* ndbegin = (int32_t*)malloc(sizeof(int32_t) * (size_t)(maxnode + 1));
    int32_t* npcase = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    float* qimpm_t = (float*)malloc(sizeof(float) * (size_t)n * p);
    int32_t* iv = (int32_t*)malloc(sizeof(int32_t) * (size_t)p);
    int32_t* nodexvr = (int32_t*)calloc((size_t)n, sizeof(int32_t));
    float* tnodewt = (float*)calloc((size_t)maxnode, sizeof(float));
    float* wsum = (float*)malloc(sizeof(float) * (size_t)maxnode);
    int32_t* wcnt = (int32_t*)malloc(sizeof(int32_t) * (size_t)maxnode);
    if (perm_bad) *perm_bad = 0;

    for (int t = 0; t < T; ++t) {
        const int64_t o = offs[t];
        const int nn = nnode[t];
        const int32_t* ns = nodestatus + o;
        const int32_t* bv = bestvar + o;
        const float* xs = xbestsplit + o;
        const int32_t* tm = treemap + 2 * o;
        const int32_t* nc = nodeclass + o;
        const int32_t* cgl = catgoleft ? catgoleft + o * maxcat : NULL;
        const int32_t* nin = nin_all + (size_t)t * n;

        /* cpu_testreebag: in-bag entries zeroed (src/rf_testreebag.cpp:22-23) */
        for (int i = 0; i < n; ++i) {
            jtr[i] = 0;
            nodextr[i] = 0;
        }
        for (int i = 0; i < n; ++i) {
            if (nin[i] != 0) continue;
            int32_t c;
            nodextr[i] = route_testreebag(X + (size_t)i * p, p, ns, bv, xs, tm, nc, nn, cat, cgl, maxcat, &c);
            jtr[i] = c;
        }
        /* casewise: tnodewt = mean bootstrap multiplicity of the in-bag
         * samples that reach each terminal node (src/rf_random_forest.cpp:
         * 1049-1102); 0 for every other node */
        if (casewise) {
            for (int k = 0; k < maxnode; ++k) {
                tnodewt[k] = 0.0f;
                wsum[k] = 0.0f;
                wcnt[k] = 0;
            }
            for (int i = 0; i < n; ++i) {
                if (nin[i] <= 0) continue;
                int nd = route_tnodewt(X + (size_t)i * p, p, ns, bv, xs, tm, cat, cgl, maxcat, nn);
                if (nd >= 0 && nd < nn && ns[nd] == -1) {
                    wsum[nd] += (float)nin[i];
                    wcnt[nd]++;
                }
            }
            for (int k = 0; k < nn; ++k)
                if (wcnt[k] > 0) tnodewt[k] = wsum[k] / (float)wcnt[k];
        }
        /* OOB votes (weight tnodewt[nodextr] when casewise, :1107-1153) and
         * the two nout increments */
        for (int i = 0; i < n; ++i) {
            if (nin[i] != 0) continue;
            if (nout) nout[i] += 2;
            if (q_raw && jtr[i] >= 0 && jtr[i] < nclass) {
                float w = 1.0f;
                if (casewise && nodextr[i] >= 0 && nodextr[i] < nn) w = tnodewt[nodextr[i]];
                q_raw[(size_t)i * nclass + jtr[i]] += w;
            }
        }
        if (jtr_out) memcpy(jtr_out + (size_t)t * n, jtr, sizeof(int32_t) * (size_t)n);

        /* cpu_varimp (src/rf_varimp.cpp:106-302), non-casewise */
        if (do_imp) {
            /* weight of an OOB vote that lands on node nd (src/rf_varimp.cpp:
             * 138-148, 203-217): tnodewt[nd] when casewise and nd is a node
             * of the tree, else 1 */
#define ORC_W(nd) ((casewise && (nd) >= 0 && (nd) < nn) ? tnodewt[(nd)] : 1.0f)
            int noob = 0;
            float right = 0.0f;
            for (int i = 0; i < n; ++i) {
                if (nin[i] == 0) {
                    if (jtr[i] == y[i]) right += ORC_W(nodextr[i]);
                    joob[noob++] = i;
                }
            }
            const float fnoob = (float)noob;
            /* jvr and nodexvr are fresh zero vectors per cpu_varimp call */
            memset(jvr, 0, sizeof(int32_t) * (size_t)n);
            memset(nodexvr, 0, sizeof(int32_t) * (size_t)n);
            if (impn == 1) {
                for (int r = 0; r < noob; ++r) {
                    int i = joob[r];
                    /* qimp_temp[i] = 0 + w/noob, then qimp_[i] += qimp_temp[i] */
                    if (jtr[i] == y[i]) qimp[i] += 0.0f + ORC_W(nodextr[i]) / fnoob;
                }
            }
            for (int k = 0; k < p; ++k) iv[k] = 0;
            for (int j = 0; j < (nn > 0 ? nn : 1); ++j)
                if (ns[j] != -1) iv[bv[j]] = 1;
            if (orc_perm(noob, perm) && perm_bad) (*perm_bad)++;
            if (impn == 1) memset(qimpm_t, 0, sizeof(float) * (size_t)n * p);
            const int nnv = nn > 0 ? nn : 1;
            for (int k = 0; k < p; ++k) {
                float rr;
                if (iv[k] == 1) {
                    float rightimp = 0.0f;
                    for (int r = 0; r < noob; ++r) {
                        int i = joob[r];
                        int ip = joob[perm[r]];
                        int32_t c, node;
                        if (route_testreeimp(X + (size_t)i * p, X + (size_t)ip * p, k, p, ns, bv, xs, tm, nc,
                                             nnv, cat, cgl, maxcat, &c, &node)) {
                            jvr[r] = c;
                            nodexvr[r] = node;
                        }
                        /* else: jvr[r] and nodexvr[r] keep their previous (stale)
                         * values, as in the reference */
                        if (jvr[r] == y[i]) {
                            const float w = ORC_W(nodexvr[r]);
                            if (impn == 1) qimpm_t[(size_t)i * p + k] += w / fnoob;
                            rightimp += w;
                        }
                    }
                    rr = (right - rightimp) / fnoob;
                    volatile float sq = rr * rr;
                    avimp[k] += 0.0f + rr;
                    sqsd[k] += 0.0f + sq;
                } else if (impn == 1) {
                    for (int r = 0; r < noob; ++r) {
                        int i = joob[r];
                        if (jtr[i] == y[i]) qimpm_t[(size_t)i * p + k] += ORC_W(nodextr[i]) / fnoob;
                    }
                }
            }
            if (impn == 1)
                for (size_t e = 0; e < (size_t)n * p; ++e) qimpm[e] += qimpm_t[e];
#undef ORC_W
        }

        /* in-bag routing, then cpu_proximity's dense branch */
        if (do_prox || leaf || Cw) {
            for (int i = 0; i < n; ++i)
                if (nin[i] > 0)
                    nodextr[i] = route_terminal(X + (size_t)i * p, p, ns, bv, xs, tm, cat, cgl, maxcat, maxnode);
            if (leaf) memcpy(leaf + (size_t)t * n, nodextr, sizeof(int32_t) * (size_t)n);
        }
        if (do_prox || Cw) {
            int nterm = 0;
            for (int k = 0; k < nn; ++k) nod[k] = (ns[k] == -1) ? nterm++ : -1;
            for (int i = 0; i < n; ++i) {
                ncount[i] = 0;
                ncn[i] = 0;
                nodexb[i] = -1;
            }
            for (int i = 0; i < n; ++i) {
                int nd = nodextr[i];
                if (nd >= 0 && nd < nn) {
                    int k = nod[nd];
                    if (k >= 0 && k < nterm) {
                        ncount[k]++;
                        ncn[i] = ncount[k];
                        nodexb[i] = k;
                    }
                }
            }
            ndbegin[0] = 0;
            for (int k = 1; k <= nterm; ++k) ndbegin[k] = ndbegin[k - 1] + ncount[k - 1];
            for (int j = 0; j < n; ++j) npcase[j] = -1;
            for (int i = 0; i < n; ++i) {
                int k = nodexb[i];
                if (k >= 0 && k < nterm) npcase[ndbegin[k] + ncn[i] - 1] = i;
            }
            for (int i = 0; i < n; ++i) {
                if (nin[i] != 0) continue;
                int k = nodexb[i];
                if (k < 0 || k >= nterm) continue;
                /* nodesize = sum of the in-bag multiplicities of the leaf (:195-204) */
                int nodesize = 0;
                for (int jj = ndbegin[k]; jj < ndbegin[k + 1]; ++jj)
                    if (npcase[jj] >= 0 && nin[npcase[jj]] > 0) nodesize += nin[npcase[jj]];
                for (int jj = ndbegin[k]; jj < ndbegin[k + 1]; ++jj) {
                    int kk = npcase[jj];
                    if (kk >= 0 && nin[kk] > 0) {
                        if (S) {
                            /* C[i][kk] += 1  ->  S[min][max] += 1 */
                            int a = i < kk ? i : kk, b = i < kk ? kk : i;
                            S[upidx(n, a, b)] += 1;
                        }
                        if (Cw && (nodesize > 0 || !casewise)) {
                            /* C[i][kk] += nin[kk] / nodesize (casewise) or 1, FP64 (:205-222) */
                            double w = (casewise && nodesize > 0) ? (double)nin[kk] / (double)nodesize : 1.0;
                            Cw[(size_t)i * n + kk] += w;
                        }
                    }
                }
            }
        }
    }
    free(jtr); free(nodextr); free(joob); free(perm); free(jvr); free(nod); free(ncount);
    free(ncn); free(nodexb); free(ndbegin); free(npcase); free(qimpm_t); free(iv);
    free(nodexvr); free(tnodewt); free(wsum); free(wcnt);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* cpu_proximity's dense branch (src/rf_proximity.cpp:108-231) from leaf      */
/* indices the caller supplies instead of routing a forest: per tree t,        */
/* leaf[t*n+i] is sample i's terminal index (0..max_leaves-1, the nod[] map    */
/* of :108-115 already applied) or -1 to leave it out, and inbag[t*n+i] its    */
/* bag flag.  Members of a leaf are bucketed stable by sample index (:116-140)*/
/* and every OOB i adds 1 for every in-bag kk of its leaf (:173-230), into    */
/* S[min][max] of the packed upper triangle.  Indices >= max_leaves are left  */
/* out and counted in the return value.                                        */
/* ------------------------------------------------------------------------ */
int64_t orc_pairs_from_leaves(int n, int T, int max_leaves, const int32_t* leaf, const uint8_t* inbag,
                              int32_t* S) {
    int32_t* ncount = (int32_t*)malloc(sizeof(int32_t) * (size_t)(max_leaves + 1));
    int32_t* ndbegin = (int32_t*)malloc(sizeof(int32_t) * (size_t)(max_leaves + 1));
    int32_t* npcase = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int64_t bad = 0;
    for (int t = 0; t < T; ++t) {
        const int32_t* lf = leaf + (size_t)t * n;
        const uint8_t* ib = inbag + (size_t)t * n;
        for (int k = 0; k <= max_leaves; ++k) ncount[k] = 0;
        for (int i = 0; i < n; ++i) {
            if (lf[i] >= max_leaves) bad++;
            else if (lf[i] >= 0) ncount[lf[i]]++;
        }
        ndbegin[0] = 0;
        for (int k = 1; k <= max_leaves; ++k) ndbegin[k] = ndbegin[k - 1] + ncount[k - 1];
        for (int k = 0; k < max_leaves; ++k) ncount[k] = 0;
        for (int i = 0; i < n; ++i) {
            const int k = lf[i];
            if (k >= 0 && k < max_leaves) npcase[ndbegin[k] + ncount[k]++] = i;
        }
        for (int i = 0; i < n; ++i) {
            const int k = lf[i];
            if (ib[i] || k < 0 || k >= max_leaves) continue;
            for (int jj = ndbegin[k]; jj < ndbegin[k + 1]; ++jj) {
                const int kk = npcase[jj];
                if (ib[kk]) {
                    const int a = i < kk ? i : kk, b = i < kk ? kk : i;
                    S[upidx(n, a, b)] += 1;
                }
            }
        }
    }
    free(ncount);
    free(ndbegin);
    free(npcase);
    return bad;
}

/* ------------------------------------------------------------------------ */
/* cpu_finishprox (src/rf_finishprox.cpp:12-74) from FP64 sums: Sd is the     */
/* packed upper triangle of C + C^T (C the raw FP64 matrix cpu_proximity     */
/* accumulates, e.g. casewise weights), the same arithmetic as               */
/* orc_finishprox.                                                            */
/* ------------------------------------------------------------------------ */
void orc_finishprox_f64(int n, const double* Sd, const int32_t* nout, int full, float* P, double* Pd) {
    double* inv = (double*)malloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < n; ++i) inv[i] = nout[i] > 0 ? 1.0 / (double)nout[i] : 1.0;
    for (int64_t i = 0; i < n; ++i) {
        for (int64_t j = i; j < n; ++j) {
            double v;
            if (i == j) {
                v = 1.0;
            } else {
                double h = Sd[upidx(n, i, j)] / 2.0;
                double a = nout[i] > 0 ? h * inv[i] : h;
                double b = nout[j] > 0 ? h * inv[j] : h;
                v = 0.5 * (a + b);
            }
            if (full) {
                if (P) { P[i * n + j] = (float)v; P[j * n + i] = (float)v; }
                if (Pd) { Pd[i * n + j] = v; Pd[j * n + i] = v; }
            } else {
                if (P) P[upidx(n, i, j)] = (float)v;
                if (Pd) Pd[upidx(n, i, j)] = v;
            }
        }
    }
    free(inv);
}

/* ------------------------------------------------------------------------ */
/* RF-GAP proximity, cpu_proximity_rfgap (src/rf_proximity.cpp:238-391):      */
/*   pGAP(i,j) = (1/|S_i|) sum_{t in S_i} c_j(t) [j in-bag in i's node] /     */
/*               |M_i(t)|                                                     */
/* S_i = trees where i is OOB, c_j(t) = j's bootstrap multiplicity, |M_i(t)| */
/* = the multiplicities of the in-bag samples in i's node summed.  Nodes are */
/* the per-tree node ids the reference stores (OOB: testreebag, in-bag:      */
/* find_terminal_node; any node id matches, the root included).  A sample    */
/* never OOB gets 1 on the diagonal.  Then P = (pGAP + pGAP^T) / 2 off the   */
/* diagonal.  node and nin are T x n; P is n x n row-major (FP64).           */
/* ------------------------------------------------------------------------ */
void orc_rfgap(int n, int T, const int32_t* nin, const int32_t* node, double* P) {
    memset(P, 0, sizeof(double) * (size_t)n * n);
    for (int i = 0; i < n; ++i) {
        int noob_i = 0;
        for (int t = 0; t < T; ++t)
            if (nin[(size_t)t * n + i] == 0) noob_i++;
        if (noob_i == 0) {
            P[(size_t)i * n + i] = 1.0;
            continue;
        }
        double* row = P + (size_t)i * n;
        for (int t = 0; t < T; ++t) {
            const int32_t* nt = nin + (size_t)t * n;
            const int32_t* dt = node + (size_t)t * n;
            if (nt[i] != 0) continue;
            const int v = dt[i];
            if (v < 0) continue;
            int64_t m = 0;
            for (int j = 0; j < n; ++j)
                if (nt[j] > 0 && dt[j] == v) m += nt[j];
            if (m == 0) continue;
            const double inv = 1.0 / (double)m;
            for (int j = 0; j < n; ++j)
                if (nt[j] > 0 && dt[j] == v) row[j] += (double)nt[j] * inv;
        }
        const double norm = 1.0 / (double)noob_i;
        for (int j = 0; j < n; ++j) row[j] *= norm;
    }
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j) {
            const double avg = (P[(size_t)i * n + j] + P[(size_t)j * n + i]) / 2.0;
            P[(size_t)i * n + j] = avg;
            P[(size_t)j * n + i] = avg;
        }
}

/* OOB error / predictions / probabilities from raw votes                    */
/* (compute_classification_error :2413-2462, compute_oob_predictions          */
/* :2246-2301; argmax with >=, so ties go to the higher class).               */
void orc_oob_summary(int n, int nclass, const float* q_raw, const int32_t* nout, const int32_t* y,
                     float* oob_error, int32_t* pred, float* proba) {
    int correct = 0, total = 0;
    for (int i = 0; i < n; ++i) {
        const float* q = q_raw + (size_t)i * nclass;
        if (nout[i] > 0) {
            int best = 0;
            float mx = q[0];
            float tot = 0.0f;
            for (int c = 0; c < nclass; ++c) {
                tot += q[c];
                if (q[c] >= mx) { mx = q[c]; best = c; }
            }
            pred[i] = best;
            total++;
            if (best == y[i]) correct++;
            for (int c = 0; c < nclass; ++c)
                proba[(size_t)i * nclass + c] = (tot > 0.0f) ? q[c] / tot : (float)(1.0 / nclass);
        } else {
            pred[i] = 0;
            for (int c = 0; c < nclass; ++c) proba[(size_t)i * nclass + c] = (float)(1.0 / nclass);
        }
    }
    *oob_error = total > 0 ? 1.0f - (float)correct / (float)total : 0.0f;
}

/* cpu_finishprox (src/rf_finishprox.cpp:12-74) written from S and nout:      */
/*   P_ij = 0.5 * ((S_ij/2) * (1/nout_i) + (S_ij/2) * (1/nout_j)), diag 1,     */
/* with a row left unscaled when nout_i == 0.  full != 0 writes the n x n     */
/* float32 matrix get_proximity_matrix returns (python/randomforest_py.cpp    */
/* :1114-1177); full == 0 writes the packed upper triangle.                   */
void orc_finishprox(int n, const int32_t* S, const int32_t* nout, int full, float* P, double* Pd) {
    double* inv = (double*)malloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < n; ++i) inv[i] = nout[i] > 0 ? 1.0 / (double)nout[i] : 1.0;
    for (int64_t i = 0; i < n; ++i) {
        for (int64_t j = i; j < n; ++j) {
            double v;
            if (i == j) {
                v = 1.0;
            } else {
                double h = (double)S[upidx(n, i, j)] / 2.0;
                double a = nout[i] > 0 ? h * inv[i] : h;
                double b = nout[j] > 0 ? h * inv[j] : h;
                v = 0.5 * (a + b);
            }
            if (full) {
                if (P) { P[i * n + j] = (float)v; P[j * n + i] = (float)v; }
                if (Pd) { Pd[i * n + j] = v; Pd[j * n + i] = v; }
            } else {
                if (P) P[upidx(n, i, j)] = (float)v;
                if (Pd) Pd[upidx(n, i, j)] = v;
            }
        }
    }
    free(inv);
}

/* localimp (src/rf_utilities.cpp:28-43): the sample-major qimpm buffer is    */
/* indexed as feature-major, so out[idx] = 100*(qimp[idx % n] - qimpm[idx])/T */
void orc_localimp(int n, int p, int T, const float* qimp, const float* qimpm, float* out) {
    for (int nn = 0; nn < n; ++nn)
        for (int m = 0; m < p; ++m) {
            size_t idx = (size_t)m * n + nn;
            out[idx] = 100.0f * (qimp[nn] - qimpm[idx]) / (float)T;
        }
}

/* predict_classification / predict_proba on held-out rows                   */
/* (src/rf_random_forest.cpp:1925-2036, :2303-2411).                           */
void orc_predict(const float* X, int m, int p, int nclass, int maxcat, int n_train, int T, const int64_t* offs,
                 const int32_t* nnode, const int32_t* nodestatus, const int32_t* bestvar,
                 const float* xbestsplit, const int32_t* treemap, const int32_t* nodeclass,
                 const int32_t* catgoleft, const int32_t* cat, int32_t* votes, int32_t* pred, float* proba) {
    const int maxnode = 2 * n_train + 1;
    for (int s = 0; s < m; ++s) {
        int32_t* v = votes + (size_t)s * nclass;
        for (int c = 0; c < nclass; ++c) v[c] = 0;
        for (int t = 0; t < T; ++t) {
            const int64_t o = offs[t];
            int c = route_predict(X + (size_t)s * p, p, nclass, nodestatus + o, bestvar + o, xbestsplit + o,
                                  treemap + 2 * o, nodeclass + o, cat, catgoleft ? catgoleft + o * maxcat : NULL,
                                  maxcat, maxnode);
            if (c >= 0) v[c]++;
        }
        int best = 0, mx = v[0];
        for (int c = 1; c < nclass; ++c)
            if (v[c] > mx) { mx = v[c]; best = c; }
        pred[s] = best;
        for (int c = 0; c < nclass; ++c) proba[(size_t)s * nclass + c] = (float)v[c] / (float)T;
    }
}
