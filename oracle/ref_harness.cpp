// Test/bench harness around the REFERENCE's own CPU functions.
//
// This file is test infrastructure, not product code.  It is compiled together
// with the reference's unmodified sources (src/*.cpp of chriskuchar/RFX, read
// where they lie) into oracle/_ref/librfxref.so by oracle/Makefile.  Only the
// tests, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm
// load it.  It exposes plain extern "C" entry points so Python can drive the
// reference through ctypes:
//
//   * rh_fit_capture   - runs rf::RandomForest::fit (src/rf_random_forest.cpp:440)
//                        on the CPU path and captures per-tree state through the
//                        reference's own progress callback (called after every
//                        grow_tree_single, src/rf_random_forest.cpp:518-521).
//   * rh_grow_forest   - cpu_bootstrap + cpu_growtree_wrapper per tree, exactly
//                        as grow_tree_single calls them (:952, :1020).
//   * rh_* stage calls - cpu_testreebag, find_terminal_node, cpu_varimp,
//                        cpu_proximity, cpu_finishprox, localimp,
//                        compute_mds_3d_cpu on a caller-supplied forest.
//
// RandomForest keeps its tree arrays and find_terminal_node private; the
// harness reads them by compiling the class declaration with private members
// made public (layout is unchanged).
#include <cstdint>
#include <cstring>
#include <vector>
#include <stdexcept>
#include <string>
#include <atomic>

#define private public
#include "rf_random_forest.hpp"
#undef private
#include "rf_config.hpp"
#include "rf_bootstrap.hpp"
#include "rf_growtree.hpp"
#include "rf_testreebag.hpp"
#include "rf_varimp.hpp"
#include "rf_proximity.hpp"
#include "rf_finishprox.hpp"
#include "rf_utilities.hpp"
#include "rf_mds_cpu.hpp"
#ifdef _OPENMP
#include <omp.h>
#endif

using rf::integer_t;
using rf::real_t;
using rf::dp_t;

static thread_local std::string g_err;

extern "C" const char* rh_last_error() { return g_err.c_str(); }

extern "C" int rh_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

// ---------------------------------------------------------------------------
// Full reference fit with per-tree capture.
//
// Outputs (caller-allocated, sizes in brackets; maxnode = 2n+1):
//   nnode[T], nodestatus/bestvar/nodeclass[T*maxnode], xbestsplit[T*maxnode],
//   treemap[T*2*maxnode], nin[T*n], jtr[T*n] (OOB class, 0 for in-bag),
//   nodextr[T*n] (leaf per sample after the tree: OOB from testreebag,
//   in-bag from find_terminal_node when proximity is on),
//   q_raw[n*c] (raw OOB votes, before finalize), nout[n],
//   scalars[0] = oob_error, oob_pred[n], oob_proba[n*c],
//   importances[p], qimp[n], qimpm[n*p] (after localimp), avimp[p], sqsd[p],
//   prox[n*n] (finalised, column-major FP64; with use_rfgap the RF-GAP
//   matrix of cpu_proximity_rfgap) or null.
// use_casewise / use_rfgap set the reference's config flags of the same names.
// ---------------------------------------------------------------------------
struct CaptureState {
    rf::RandomForest* rfp;
    int n, T;
    int maxnode;
    int* nin;
    int* jtr;
    int* nodextr;
    float* q_raw;
    int nclass;
};

extern "C" int rh_fit_capture(const float* X, const int* y, const int* cat,
                              int n, int p, int ntree, int mtry, int minndsize,
                              int maxcat, int iseed,
                              int compute_prox, int compute_imp, int compute_local_imp,
                              int use_casewise, int use_rfgap,
                              int* nclass_out,
                              int* nnode, int* nodestatus, int* bestvar, float* xbestsplit,
                              int* treemap, int* nodeclass,
                              int* nin, int* jtr, int* nodextr,
                              float* q_raw, int* nout, float* scalars,
                              int* oob_pred, float* oob_proba,
                              float* importances, float* qimp, float* qimpm,
                              float* avimp, float* sqsd, double* prox) {
    try {
        rf::RandomForestConfig cfg;
        cfg.task_type = rf::TaskType::CLASSIFICATION;
        cfg.nsample = n;
        cfg.ntree = ntree;
        cfg.mdim = p;
        // nclass as the Python binding computes it: number of distinct labels.
        {
            std::vector<char> seen(1 << 16, 0);
            int c = 0;
            for (int i = 0; i < n; ++i) {
                if (y[i] < 0 || y[i] >= (1 << 16)) throw std::runtime_error("label range");
                if (!seen[y[i]]) { seen[y[i]] = 1; ++c; }
            }
            cfg.nclass = c;
        }
        cfg.maxcat = maxcat;
        cfg.mtry = mtry > 0 ? mtry : (int)std::sqrt((float)p);
        cfg.maxnode = 2 * n + 1;
        cfg.minndsize = minndsize;
        cfg.iseed = iseed;
        cfg.compute_proximity = compute_prox != 0;
        cfg.compute_importance = compute_imp != 0;
        cfg.compute_local_importance = compute_local_imp != 0;
        cfg.use_gpu = false;
        cfg.use_qlora = false;
        cfg.use_casewise = use_casewise != 0;
        cfg.use_rfgap = use_rfgap != 0;
        *nclass_out = cfg.nclass;

        rf::RandomForest model(cfg);
        model.set_categorical_features(cat, p);

        CaptureState st{&model, n, ntree, cfg.maxnode, nin, jtr, nodextr, q_raw, cfg.nclass};
        model.set_progress_callback([&st](integer_t cur, integer_t total) {
            const int t = cur - 1;
            rf::RandomForest& m = *st.rfp;
            std::memcpy(st.nin + (size_t)t * st.n, m.nin_workspace_.data(), sizeof(int) * st.n);
            std::memcpy(st.jtr + (size_t)t * st.n, m.jtr_workspace_.data(), sizeof(int) * st.n);
            std::memcpy(st.nodextr + (size_t)t * st.n, m.nodextr_workspace_.data(), sizeof(int) * st.n);
            if (cur == total) {
                std::memcpy(st.q_raw, m.q_.data(), sizeof(float) * (size_t)st.n * st.nclass);
            }
        });
        model.fit(X, y, nullptr);

        const int mx = cfg.maxnode;
        for (int t = 0; t < ntree; ++t) nnode[t] = model.nnode_[t];
        std::memcpy(nodestatus, model.nodestatus_.data(), sizeof(int) * (size_t)ntree * mx);
        std::memcpy(bestvar, model.bestvar_.data(), sizeof(int) * (size_t)ntree * mx);
        std::memcpy(xbestsplit, model.xbestsplit_.data(), sizeof(float) * (size_t)ntree * mx);
        std::memcpy(treemap, model.treemap_.data(), sizeof(int) * (size_t)ntree * 2 * mx);
        std::memcpy(nodeclass, model.nodeclass_.data(), sizeof(int) * (size_t)ntree * mx);
        std::memcpy(nout, model.nout_.data(), sizeof(int) * n);
        scalars[0] = model.get_oob_error();
        std::memcpy(oob_pred, model.oob_class_predictions_.data(), sizeof(int) * n);
        std::memcpy(oob_proba, model.oob_probabilities_.data(), sizeof(float) * (size_t)n * cfg.nclass);
        if (compute_imp) {
            std::memcpy(importances, model.feature_importances_.data(), sizeof(float) * p);
            std::memcpy(qimp, model.qimp_.data(), sizeof(float) * n);
            if (compute_local_imp)
                std::memcpy(qimpm, model.qimpm_.data(), sizeof(float) * (size_t)n * p);
            std::memcpy(avimp, model.avimp_.data(), sizeof(float) * p);
            std::memcpy(sqsd, model.sqsd_.data(), sizeof(float) * p);
        }
        if (compute_prox && prox) {
            std::memcpy(prox, model.proximity_matrix_.data(), sizeof(double) * (size_t)n * n);
        }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// Reference predict / predict_proba on held-out rows, using a fitted forest
// rebuilt from caller arrays (padded to maxnode = 2n+1 per tree).
static void load_forest(rf::RandomForest& m, int T, int maxnode, int maxcat, const int* nnode,
                        const int* nodestatus, const int* bestvar, const float* xbestsplit,
                        const int* treemap, const int* nodeclass, const int* catgoleft) {
    for (int t = 0; t < T; ++t) m.nnode_[t] = nnode[t];
    std::memcpy(m.nodestatus_.data(), nodestatus, sizeof(int) * (size_t)T * maxnode);
    std::memcpy(m.bestvar_.data(), bestvar, sizeof(int) * (size_t)T * maxnode);
    std::memcpy(m.xbestsplit_.data(), xbestsplit, sizeof(float) * (size_t)T * maxnode);
    std::memcpy(m.treemap_.data(), treemap, sizeof(int) * (size_t)T * 2 * maxnode);
    std::memcpy(m.nodeclass_.data(), nodeclass, sizeof(int) * (size_t)T * maxnode);
    if (catgoleft) std::memcpy(m.catgoleft_.data(), catgoleft, sizeof(int) * (size_t)T * maxnode * maxcat);
}

static rf::RandomForestConfig make_cfg(int n, int p, int nclass, int T, int maxcat) {
    rf::RandomForestConfig cfg;
    cfg.task_type = rf::TaskType::CLASSIFICATION;
    cfg.nsample = n;
    cfg.ntree = T;
    cfg.mdim = p;
    cfg.nclass = nclass;
    cfg.maxcat = maxcat;
    cfg.maxnode = 2 * n + 1;
    cfg.compute_proximity = false;
    cfg.compute_importance = false;
    cfg.use_gpu = false;
    return cfg;
}

extern "C" int rh_predict(int n_train, int p, int nclass, int T, int maxcat, const int* cat,
                          const int* nnode, const int* nodestatus, const int* bestvar,
                          const float* xbestsplit, const int* treemap, const int* nodeclass,
                          const int* catgoleft, const float* Xtest, int m, int* pred, float* proba) {
    try {
        rf::RandomForestConfig cfg = make_cfg(n_train, p, nclass, T, maxcat);
        rf::RandomForest model(cfg);
        model.set_categorical_features(cat, p);
        load_forest(model, T, cfg.maxnode, maxcat, nnode, nodestatus, bestvar, xbestsplit, treemap, nodeclass,
                    catgoleft);
        model.predict_classification(Xtest, m, pred);
        model.predict_proba(Xtest, m, proba);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// ---------------------------------------------------------------------------
// Growth only: the same bootstrap + growtree calls grow_tree_single makes.
// Trees are independent given (tree id, seed), so they run in parallel.
// Arrays are padded per tree to maxnode = 2n+1.
// ---------------------------------------------------------------------------
extern "C" int rh_grow_forest(const float* X, const int* y, int n, int p, int nclass,
                              int ntree, int mtry, int minndsize, int maxcat, int iseed,
                              int* nnode, int* nodestatus, int* bestvar, float* xbestsplit,
                              int* treemap, int* nodeclass, int* nin) {
    const int maxnode = 2 * n + 1;
    std::atomic<int> failed{0};
#pragma omp parallel
    {
        std::vector<real_t> weight(n, 1.0f), win(n), tnodewt(maxnode), tcat(maxcat), classpop((size_t)nclass * maxnode);
        std::vector<real_t> wr(nclass), wl(nclass), tclasscat((size_t)nclass * maxcat), tclasspop(nclass), tmpclass(nclass);
        std::vector<integer_t> nout(n, 0), jinbag(n), joobag(n), amat((size_t)p * n), idmove(n), igoleft(maxcat),
            igl(maxcat), nodestart(maxnode), nodestop(maxnode), itemp(n), itmp(maxcat), icat(maxcat),
            jtr(n), nodextr(n), ties((size_t)p * n, 0), catv(p, 1), catgoleft((size_t)maxcat * maxnode);
#pragma omp for schedule(dynamic, 1)
        for (int t = 0; t < ntree; ++t) {
            integer_t ninbag = 0, noobag = 0;
            int* nin_t = nin + (size_t)t * n;
            rf::cpu_bootstrap(weight.data(), n, win.data(), nin_t, nout.data(), jinbag.data(), joobag.data(),
                              ninbag, noobag, t);
            int* ns = nodestatus + (size_t)t * maxnode;
            int* bv = bestvar + (size_t)t * maxnode;
            float* xs = xbestsplit + (size_t)t * maxnode;
            int* tm = treemap + (size_t)t * 2 * maxnode;
            int* nc = nodeclass + (size_t)t * maxnode;
            std::fill(ns, ns + maxnode, 0);
            std::fill(bv, bv + maxnode, 0);
            std::fill(xs, xs + maxnode, 0.0f);
            std::fill(tm, tm + 2 * maxnode, 0);
            std::fill(nc, nc + maxnode, 0);
            integer_t nn = 0;
            rf::cpu_growtree_wrapper(X, win.data(), y, catv.data(), ties.data(), nin_t, p, n, nclass, maxnode,
                                     minndsize, mtry, ninbag, maxcat, iseed + t, 25, 25, amat.data(),
                                     jinbag.data(), tnodewt.data(), xs, ns, bv, tm, catgoleft.data(), nc,
                                     jtr.data(), nodextr.data(), nn, idmove.data(), igoleft.data(), igl.data(),
                                     nodestart.data(), nodestop.data(), itemp.data(), itmp.data(), icat.data(),
                                     tcat.data(), classpop.data(), wr.data(), wl.data(), tclasscat.data(),
                                     tclasspop.data(), tmpclass.data());
            nnode[t] = nn;
        }
    }
    return failed.load();
}

// ---------------------------------------------------------------------------
// Per-stage reference calls on a compact forest (tree t's arrays start at
// offs[t], length nnode[t]; treemap is 2*nnode[t] at 2*offs[t]).
// catgoleft is all zero for forests from the reference's CPU grower (it is
// never written, src/rf_growtree.cpp:408); the stage calls pass a zero table.
// ---------------------------------------------------------------------------
struct TreeView {
    std::vector<int> ns, bv, tm, nc, cgl;
    std::vector<float> xs;
};

static void expand_tree(TreeView& v, int maxnode, int maxcat, int nn, const int* ns, const int* bv,
                        const float* xs, const int* tm, const int* nc, const int* cgl = nullptr) {
    v.ns.assign(maxnode, 0);
    v.bv.assign(maxnode, 0);
    v.xs.assign(maxnode, 0.0f);
    v.tm.assign(2 * (size_t)maxnode, 0);
    v.nc.assign(maxnode, 0);
    v.cgl.assign((size_t)maxcat * maxnode, 0);
    std::memcpy(v.ns.data(), ns, sizeof(int) * nn);
    std::memcpy(v.bv.data(), bv, sizeof(int) * nn);
    std::memcpy(v.xs.data(), xs, sizeof(float) * nn);
    std::memcpy(v.tm.data(), tm, sizeof(int) * 2 * nn);
    std::memcpy(v.nc.data(), nc, sizeof(int) * nn);
    if (cgl) std::memcpy(v.cgl.data(), cgl, sizeof(int) * (size_t)maxcat * nn);
}

// The per-tree analysis sequence of grow_tree_single (src/rf_random_forest.cpp:1043-1309)
// for trees [t0, t1): testreebag, OOB votes, varimp, in-bag routing, proximity.
// Accumulators follow the reference types: q float, nout int (incremented twice
// per OOB tree as the reference does), qimp/qimpm/avimp/sqsd float.
// prox: n*n FP64 column-major, or null to skip proximity.  catgoleft: maxcat
// entries per node in the compact layout (tree t from offs[t] * maxcat), or
// null for the all-zero table the reference's CPU grower leaves.
extern "C" int rh_analyse_trees(const float* X, const int* y, const int* cat, int n, int p, int nclass,
                                int maxcat, int t0, int t1, const long long* offs, const int* nnode,
                                const int* nodestatus, const int* bestvar, const float* xbestsplit,
                                const int* treemap, const int* nodeclass, const int* catgoleft, const int* nin_all,
                                int do_imp, int impn,
                                float* q, int* nout, float* qimp, float* qimpm, float* avimp, float* sqsd,
                                double* prox, int* leaf_out) {
    try {
        rf::RandomForestConfig cfg = make_cfg(n, p, nclass, 1, maxcat);
        rf::RandomForest model(cfg);
        model.set_categorical_features(cat, p);
        rf::g_config.use_casewise = false;
        const int maxnode = cfg.maxnode;
        TreeView v;
        std::vector<int> jtr(n), nodextr(n);
        std::vector<real_t> qimp_t(n), qimpm_t((size_t)n * p), avimp_t(p), sqsd_t(p), tnodewt(maxnode, 0.0f);
        std::vector<int> jvr(n), nodexvr(n);
        std::vector<int> nod(maxnode), ncount(n), ncn(n), nodexb(n), ndbegin(maxnode + 1), npcase(n);
        for (int t = t0; t < t1; ++t) {
            const long long o = offs[t];
            const int nn = nnode[t];
            expand_tree(v, maxnode, maxcat, nn, nodestatus + o, bestvar + o, xbestsplit + o, treemap + 2 * o,
                        nodeclass + o, catgoleft ? catgoleft + o * maxcat : nullptr);
            const int* nin = nin_all + (size_t)t * n;
            // cpu_bootstrap's own nout increment (src/rf_bootstrap.cpp:60-61)
            for (int i = 0; i < n; ++i) if (nin[i] == 0) nout[i]++;
            rf::cpu_testreebag(X, v.xs.data(), nin, v.tm.data(), v.bv.data(), v.nc.data(), cat, v.ns.data(),
                               v.cgl.data(), n, p, nn, maxcat, jtr.data(), nodextr.data());
            for (int i = 0; i < n; ++i) {
                if (nin[i] == 0) {
                    nout[i]++;
                    if (jtr[i] >= 0 && jtr[i] < nclass) q[(size_t)i * nclass + jtr[i]] += 1.0f;
                }
            }
            if (do_imp) {
                std::fill(qimp_t.begin(), qimp_t.end(), 0.0f);
                std::fill(qimpm_t.begin(), qimpm_t.end(), 0.0f);
                std::fill(avimp_t.begin(), avimp_t.end(), 0.0f);
                std::fill(sqsd_t.begin(), sqsd_t.end(), 0.0f);
                std::fill(jvr.begin(), jvr.end(), 0);
                std::fill(nodexvr.begin(), nodexvr.end(), 0);
                rf::cpu_varimp(X, n, p, y, nin, jtr.data(), impn, qimp_t.data(), qimpm_t.data(), avimp_t.data(),
                               sqsd_t.data(), v.tm.data(), v.ns.data(), v.xs.data(), v.bv.data(), v.nc.data(),
                               nn > 0 ? nn : 1, cat, jvr.data(), nodexvr.data(), maxcat, v.cgl.data(),
                               tnodewt.data(), nodextr.data());
                for (int i = 0; i < n; ++i) qimp[i] += qimp_t[i];
                if (impn)
                    for (size_t i = 0; i < (size_t)n * p; ++i) qimpm[i] += qimpm_t[i];
                for (int k = 0; k < p; ++k) {
                    avimp[k] += avimp_t[k];
                    sqsd[k] += sqsd_t[k];
                }
            }
            if (prox || leaf_out) {
                for (int i = 0; i < n; ++i)
                    if (nin[i] > 0)
                        nodextr[i] = model.find_terminal_node(X + (size_t)i * p, v.ns.data(), v.bv.data(),
                                                              v.xs.data(), v.tm.data(), v.cgl.data());
                if (leaf_out) std::memcpy(leaf_out + (size_t)(t - t0) * n, nodextr.data(), sizeof(int) * n);
                if (prox)
                    rf::cpu_proximity(v.ns.data(), nodextr.data(), nin, n, nn, prox, nod.data(), ncount.data(),
                                      ncn.data(), nodexb.data(), ndbegin.data(), npcase.data());
            }
        }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// cpu_permobmr (src/rf_varimp.cpp:16-30) on joob = 0..noob-1: the permuted
// OOB positions.  Only call it for noob values whose MT19937(42) stream has no
// draw that rounds to 1.0f (the reference then indexes past its vector).
extern "C" int rh_permobmr(int noob, int* out) {
    std::vector<integer_t> joob(noob);
    for (int i = 0; i < noob; ++i) joob[i] = i;
    rf::cpu_permobmr(joob.data(), out, noob);
    return 0;
}

extern "C" int rh_finishprox(int n, const int* nout, double* prox, double* proxsym) {
    rf::cpu_finishprox(n, nout, prox, proxsym);
    return 0;
}

extern "C" int rh_localimp(int n, int p, int T, const float* qimp, float* qimpm) {
    rf::localimp(n, p, T, qimp, qimpm);
    return 0;
}

// compute_mds_3d_cpu exactly as the binding calls it (python/randomforest_py.cpp:1221-1243):
// prox is the float32 matrix get_proximity_matrix returns, promoted to FP64.
extern "C" int rh_mds3d(const double* prox, int n, const int* nout, double* coords) {
    try {
        std::vector<double> c = rf::compute_mds_3d_cpu(prox, n, false, nout, false);
        std::memcpy(coords, c.data(), sizeof(double) * (size_t)n * 3);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}
