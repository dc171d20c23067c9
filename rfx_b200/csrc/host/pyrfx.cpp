// pybind11 module `rfx_b200._rfx`: the reference's Python surface for
// classification (python/randomforest_py.cpp:606-1420, module functions
// :4138-4146 and :4262-4290) on top of the C ABI in rfx_b200.h.
//
// Same class and method names, argument names and defaults, array shapes,
// dtypes and layouts, and the same errors (RuntimeError) and warnings.  The
// reference's quirks that change results are kept on purpose:
//   * mtry and maxnode are fixed in the constructor from its nsample/mdim
//     arguments (sqrt(mdim), 2 * nsample + 1) and fit() does not revisit them;
//   * predict / predict_proba on as many rows as the training set return the
//     stored OOB predictions / probabilities;
//   * get_local_importance returns localimp's feature-major reading of the
//     sample-major buffer as an (n, p) array;
//   * get_lowrank_factors returns (A, B, r) with B == A and a column-major
//     buffer behind the C-order (n, r) arrays; the factors are those of
//     P ~= I + A A^T (the identity is not part of them: a caller rebuilding P
//     adds it).
// Every call into the library releases the GIL; the library never calls back
// into Python.  All analysis runs on CUDA device 0; fit() raises when no
// usable device or library is present (there is no CPU fallback).
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstring>
#include <cstdint>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

#include "rfx_b200.h"

namespace py = pybind11;

namespace {

enum class TaskType { CLASSIFICATION, REGRESSION, UNSUPERVISED };

using FArray = py::array_t<float, py::array::c_style | py::array::forcecast>;
using IArray = py::array_t<int32_t, py::array::c_style | py::array::forcecast>;

void check(rfx_status st, const std::string& what) {
    if (st != RFX_OK) throw std::runtime_error(what + ": " + rfx_last_error());
}

std::string lower(std::string s) {
    std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return (char)std::tolower(c); });
    return s;
}

// IEEE binary16 bits -> float (FP16 factor storage read back on the host).
float half_to_float(uint16_t h) {
    const uint32_t sign = (uint32_t)(h >> 15) << 31;
    const int e = (h >> 10) & 31;
    uint32_t m = h & 1023u;
    uint32_t bits;
    if (e == 0) {
        if (m == 0) {
            bits = sign;
        } else {  // subnormal: normalise
            int k = -1;
            do {
                ++k;
                m <<= 1;
            } while (!(m & 1024u));
            bits = sign | ((uint32_t)(127 - 15 - k) << 23) | ((m & 1023u) << 13);
        }
    } else if (e == 31) {
        bits = sign | 0x7f800000u | (m << 13);
    } else {
        bits = sign | ((uint32_t)(e - 15 + 127) << 23) | (m << 13);
    }
    float f;
    std::memcpy(&f, &bits, sizeof(f));
    return f;
}

// quantization_string_to_int (python/randomforest_py.cpp:271-287)
int quant_mode_code(const std::string& q) {
    const std::string l = lower(q);
    if (l == "fp32") return 0;
    if (l == "fp16") return 1;
    if (l == "int8") return 2;
    if (l == "nf4") return 3;
    throw std::runtime_error("Unknown quantization level: '" + q + "'. Valid Options: 'fp32', 'fp16', 'int8', 'nf4'");
}

// loss_function_string_to_int for classification (python/randomforest_py.cpp:246-269)
void check_loss(const std::string& loss) {
    const std::string l = lower(loss);
    if (l == "gini" || l == "gini_impurity") return;
    if (l == "mse" || l == "mean_squared_error" || l == "l2")
        throw std::runtime_error("MSE/L2 can only be used for regression tasks, not classification");
    throw std::runtime_error("Unknown loss function: '" + loss +
                             "'. Valid options: Classification: 'gini'; Regression: 'mse'; "
                             "Ranking/Survival: 'ranking', 'survival'");
}

struct NoGil {
    py::gil_scoped_release r;
};

class RandomForestClassifier {
  public:
    RandomForestClassifier(int nsample, int ntree, int mdim, int nclass, int maxcat, int mtry, int maxnode,
                           int minndsize, int ncsplit, int ncmax, int iseed, bool compute_proximity,
                           bool compute_importance, bool compute_local_importance, bool use_gpu, bool use_qlora,
                           std::string quant_mode, bool use_sparse, float sparsity_threshold, int batch_size,
                           int nodesize, float cutoff, bool show_progress, std::string progress_desc,
                           std::string gpu_loss_function, int rank, int n_threads_cpu, bool use_rfgap,
                           std::string importance_method, int clique_M, bool use_casewise)
        : nsample_(nsample),
          ntree_(ntree),
          mdim_(mdim),
          nclass_(nclass),
          maxcat_(maxcat),
          minndsize_(minndsize),
          ncsplit_(ncsplit),
          ncmax_(ncmax),
          iseed_(iseed),
          compute_proximity_(compute_proximity),
          compute_importance_(compute_importance),
          compute_local_importance_(compute_local_importance),
          use_gpu_(use_gpu),
          use_qlora_(use_qlora),
          quant_mode_(quant_mode),
          use_sparse_(use_sparse),
          sparsity_threshold_(sparsity_threshold),
          batch_size_(batch_size),
          nodesize_(nodesize),
          cutoff_(cutoff),
          show_progress_(show_progress),
          progress_desc_(progress_desc),
          gpu_loss_function_(gpu_loss_function),
          rank_(rank),
          n_threads_cpu_(n_threads_cpu),
          use_rfgap_(use_rfgap),
          importance_method_(importance_method),
          clique_M_(clique_M),
          use_casewise_(use_casewise) {
        // the constructor fixes mtry and maxnode (python/randomforest_py.cpp:649-650)
        mtry_ = mtry > 0 ? mtry : (int)std::sqrt((float)mdim);
        maxnode_ = maxnode > 0 ? maxnode : 2 * nsample + 1;
        quant_code_ = quant_mode_code(quant_mode);
        check_loss(gpu_loss_function);
    }

    ~RandomForestClassifier() { release_ctx(); }

    void fit(py::array X, py::array y, py::object sample_weight) {
        (void)sample_weight;  // classification ignores sample weights, as the reference does
        if (X.ndim() != 2) throw std::runtime_error("X must be 2-dimensional (samples, features)");
        FArray Xf = FArray::ensure(X);
        if (!Xf) throw std::runtime_error("X must be convertible to float32");
        const int n = (int)Xf.shape(0), p = (int)Xf.shape(1);
        if ((py::ssize_t)y.size() != n) throw std::runtime_error("y must hold one label per row of X");
        const bool y_float = y.dtype().kind() == 'f';
        IArray yi = IArray::ensure(y);
        if (!yi) throw std::runtime_error("y must be convertible to int32");
        int c = nclass_;
        if (!y_float) {
            std::set<int32_t> u(yi.data(), yi.data() + n);
            c = (int)u.size();
        }
        check_loss(gpu_loss_function_);
        if (compute_proximity_ && use_rfgap_ && use_qlora_)
            throw std::runtime_error(
                "use_rfgap=True with use_qlora=True is not supported by rfx_b200: RF-GAP proximity is computed as "
                "the full matrix (use_qlora=False)");
        if (compute_importance_ && compute_local_importance_ && importance_method_ == "clique")
            throw std::runtime_error(
                "CLIQUE importance is not available in v1.0. Use importance_method='local_imp' instead.");

        release_ctx();
        fitted_ = false;
        nsample_ = n;
        mdim_ = p;
        nclass_ = c;
        X_.assign(Xf.data(), Xf.data() + (size_t)n * p);
        y_.assign(yi.data(), yi.data() + n);
        detect_categorical();
        py::module_::import("builtins")
            .attr("print")(py::str("Training Random Forest Classifier with {} trees...").format(ntree_));

        rfx_grown_forest g{};
        {
            NoGil ng;
            check(rfx_grow_forest(X_.data(), y_.data(), n, p, c, ntree_, mtry_, minndsize_, maxnode_, iseed_,
                                  n_threads_cpu_, &g),
                  "fit (forest growth)");
        }
        const int64_t N = g.offs[ntree_];
        offs_.assign(g.offs, g.offs + ntree_ + 1);
        nodestatus_.assign(g.nodestatus, g.nodestatus + N);
        bestvar_.assign(g.bestvar, g.bestvar + N);
        xbestsplit_.assign(g.xbestsplit, g.xbestsplit + N);
        treemap_.assign(g.treemap, g.treemap + 2 * N);
        nodeclass_.assign(g.nodeclass, g.nodeclass + N);
        nin_.assign(g.nin, g.nin + (size_t)ntree_ * n);
        rfx_free_forest(&g);

        ensure_ctx();
        nout_.assign(n, 0);
        oob_pred_.assign(n, 0);
        oob_proba_.assign((size_t)n * c, 0.0f);
        importances_.assign(p, 0.0f);
        local_imp_.clear();
        S_.clear();
        Sd_.clear();
        lowrank_ready_ = false;
        {
            NoGil ng;
            if (use_casewise_) {  // votes weighted by tnodewt
                std::vector<float> q((size_t)n * c);
                check(rfx_casewise_votes(ctx_, q.data(), nout_.data()), "fit (OOB routing)");
            } else {
                std::vector<int32_t> q((size_t)n * c);
                check(rfx_route_oob(ctx_, q.data(), nout_.data(), nullptr), "fit (OOB routing)");
            }
            check(rfx_oob_summary(ctx_, &oob_error_, oob_pred_.data(), oob_proba_.data()), "fit (OOB summary)");
            if (compute_importance_) {
                std::vector<float> sqsd(p), qimp(n), qimpm;
                if (compute_local_importance_) qimpm.resize((size_t)n * p);
                check(rfx_varimp(ctx_, compute_local_importance_ ? 1 : 0, importances_.data(), sqsd.data(),
                                 qimp.data(), compute_local_importance_ ? qimpm.data() : nullptr),
                      "fit (permutation importance)");
                if (compute_local_importance_) {
                    local_imp_.resize((size_t)n * p);
                    check(rfx_localimp(ctx_, qimp.data(), qimpm.data(), local_imp_.data()), "fit (local importance)");
                }
            }
        }
        if (compute_proximity_) {
            if (use_qlora_) {
                compute_lowrank();
            } else {
                NoGil ng;
                const size_t len = (size_t)n * (n + 1) / 2;
                if (use_rfgap_) {  // the final RF-GAP matrix
                    Sd_.resize(len);
                    check(rfx_proximity_rfgap(ctx_, Sd_.data(), len), "fit (RF-GAP proximity)");
                } else if (use_casewise_) {  // FP64 weighted sums, finished on request
                    Sd_.resize(len);
                    check(rfx_proximity_upper_f64(ctx_, Sd_.data(), len), "fit (proximity)");
                } else {
                    S_.resize(len);
                    check(rfx_proximity_upper_i32(ctx_, S_.data(), len), "fit (proximity)");
                }
            }
        }
        fitted_ = true;
    }

    py::array_t<int32_t> predict(py::array X) {
        need_fit("predict");
        FArray Xf = as_features(X);
        const int m = (int)Xf.shape(0);
        py::array_t<int32_t> out(m);
        int32_t* o = out.mutable_data();
        if (m == nsample_) {  // training-set size: the stored OOB predictions
            std::copy(oob_pred_.begin(), oob_pred_.end(), o);
            return out;
        }
        const std::vector<int32_t> v = votes(Xf);
        for (int i = 0; i < m; ++i) {
            int best = 0, bv = v[(size_t)i * nclass_];
            for (int k = 1; k < nclass_; ++k)
                if (v[(size_t)i * nclass_ + k] > bv) {
                    bv = v[(size_t)i * nclass_ + k];
                    best = k;
                }
            o[i] = best;
        }
        return out;
    }

    py::array_t<float> predict_proba(py::array X) {
        need_fit("predict_proba");
        FArray Xf = as_features(X);
        const int m = (int)Xf.shape(0);
        py::array_t<float> out({(py::ssize_t)m, (py::ssize_t)nclass_});
        float* o = out.mutable_data();
        if (m == nsample_) {
            std::copy(oob_proba_.begin(), oob_proba_.end(), o);
            return out;
        }
        const std::vector<int32_t> v = votes(Xf);
        const float total = (float)ntree_;
        for (size_t e = 0; e < v.size(); ++e) o[e] = (float)v[e] / total;
        return out;
    }

    float get_oob_error() const {
        need_fit("get_oob_error");
        return oob_error_;
    }

    py::array_t<float> feature_importances_() const {
        need_fit("feature_importances_");
        py::array_t<float> out(mdim_);
        std::copy(importances_.begin(), importances_.end(), out.mutable_data());
        return out;
    }

    TaskType get_task_type() const { return TaskType::CLASSIFICATION; }
    int get_n_samples() const { return nsample_; }
    int get_n_features() const { return mdim_; }
    int get_n_classes() const { return nclass_; }

    py::array_t<float> get_local_importance() const {
        need_fit("get_local_importance");
        py::array_t<float> out({(py::ssize_t)nsample_, (py::ssize_t)mdim_});
        float* o = out.mutable_data();
        if (local_imp_.empty()) std::fill(o, o + (size_t)nsample_ * mdim_, 0.0f);
        else std::copy(local_imp_.begin(), local_imp_.end(), o);
        return out;
    }

    // get_proximity_matrix (python/randomforest_py.cpp:1114-1177)
    py::array_t<float> get_proximity_matrix() {
        need_fit("get_proximity_matrix");
        const int n = nsample_;
        if (compute_proximity_ && use_qlora_) {
            std::string msg =
                "Proximity matrix not available in full form. Low-rank mode is active (use_qlora=True). "
                "Full matrix reconstruction would require O(n\xc2\xb2) memory and can CRASH your system! "
                "Example: 100k samples = ~80 GB (likely to crash!). "
                "Proximity is stored in low-rank factors (A and B). "
                "Use get_lowrank_factors() or compute_mds_3d_from_factors() instead. "
                "Or disable use_qlora=True for smaller datasets that can fit full matrix.";
            if (n > 50000)
                msg += " ERROR: Dataset too large (" + std::to_string(n) +
                       " samples) - reconstruction aborted to prevent system crash.";
            throw std::runtime_error(msg);
        }
        py::array_t<float> out({(py::ssize_t)n, (py::ssize_t)n});
        float* o = out.mutable_data();
        if (!compute_proximity_) {
            std::fill(o, o + (size_t)n * n, 0.0f);
            for (int i = 0; i < n; ++i) o[(size_t)i * n + i] = 1.0f;
            return out;
        }
        if (PyErr_WarnEx(PyExc_RuntimeWarning,
                         "WARNING: get_proximity_matrix() may have reconstructed full matrix from low-rank "
                         "factors. This requires O(n\xc2\xb2) memory and may crash your system for large datasets! "
                         "For low-rank mode (use_qlora=True), use get_lowrank_factors() or "
                         "compute_mds_3d_from_factors() instead.",
                         1) != 0)
            throw py::error_already_set();
        ensure_ctx();
        NoGil ng;
        if (use_rfgap_) {
            // the RF-GAP matrix is final: float32 copy of the packed triangle
            const int64_t nn = n;
            for (int64_t i = 0; i < nn; ++i)
                for (int64_t j = i; j < nn; ++j) {
                    const float v = (float)Sd_[(size_t)(i * nn - i * (i - 1) / 2 + (j - i))];
                    o[i * nn + j] = v;
                    o[j * nn + i] = v;
                }
        } else if (use_casewise_) {
            check(rfx_finishprox_f64(ctx_, Sd_.data(), o, 1), "get_proximity_matrix");
        } else {
            check(rfx_finishprox(ctx_, S_.data(), o, 1), "get_proximity_matrix");
        }
        return out;
    }

    py::array_t<float> get_oob_predictions() const {
        need_fit("get_oob_predictions");
        py::array_t<float> out(nsample_);
        float* o = out.mutable_data();
        for (int i = 0; i < nsample_; ++i) o[i] = (float)oob_pred_[i];
        return out;
    }

    // get_lowrank_factors (python/randomforest_py.cpp:1179-1219)
    py::tuple get_lowrank_factors() {
        need_fit("get_lowrank_factors");
        if (!(compute_proximity_ && use_qlora_))
            throw std::runtime_error(
                "Low-rank factors not available. Either low-rank mode is not active (use_qlora=True required), "
                "or factors have not been computed yet.");
        const int n = nsample_, r = lr_rank_;
        py::array_t<double> A(std::vector<py::ssize_t>{n, r}), B(std::vector<py::ssize_t>{n, r});
        double* a = A.mutable_data();
        double* b = B.mutable_data();
        // column-major n x r buffer behind the C-order (n, r) arrays
        for (int col = 0; col < r; ++col)
            for (int i = 0; i < n; ++i) a[(size_t)col * n + i] = (double)factors_[(size_t)i * r + col];
        std::copy(a, a + (size_t)n * r, b);
        return py::make_tuple(A, B, r);
    }

    // compute_mds_3d_cpu (python/randomforest_py.cpp:1221-1243): the MDS of
    // the float32 proximity matrix get_proximity_matrix returns
    py::array_t<double> compute_mds_3d_cpu() {
        need_fit("compute_mds_3d_cpu");
        py::array_t<float> P = get_proximity_matrix();
        ensure_ctx();
        const int n = nsample_;
        py::array_t<double> out(std::vector<py::ssize_t>{n, 3});
        double ev[3];
        NoGil ng;
        check(rfx_mds3d_full(ctx_, P.data(), out.mutable_data(), ev), "compute_mds_3d_cpu");
        return out;
    }

    // compute_mds_from_factors (python/randomforest_py.cpp:1245-1306)
    py::array_t<double> compute_mds_from_factors(int k) {
        need_fit("compute_mds_from_factors");
        if (k < 1) throw std::runtime_error("MDS dimension k must be >= 1");
        if (!(compute_proximity_ && use_qlora_))
            throw std::runtime_error(
                "MDS computation failed. Low-rank factors may not be available (use_qlora=True required), "
                "or computation failed.");
        if (!lowrank_ready_) compute_lowrank();
        const int n = nsample_;
        py::array_t<double> out(std::vector<py::ssize_t>{n, (py::ssize_t)k});
        {
            std::vector<double> ev(k);
            NoGil ng;
            check(rfx_mds_from_factors(ctx_, k, lr_quantized_ ? 1 : 0, lr_precision_, out.mutable_data(), ev.data()),
                  "compute_mds_from_factors");
        }
        duplicate_warning(out);
        return out;
    }

    py::array_t<double> compute_mds_3d_from_factors() { return compute_mds_from_factors(3); }

    // cleanup: release the device state; results already returned or cached
    // on the host stay valid, and a later call that needs the device loads
    // the forest again
    void cleanup() { release_ctx(); }

  private:
    void need_fit(const char* what) const {
        if (!fitted_) throw std::runtime_error(std::string("Model must be fitted before calling ") + what + "()");
    }

    FArray as_features(py::array X) const {
        if (X.ndim() != 2) throw std::runtime_error("X must be 2-dimensional (samples, features)");
        FArray Xf = FArray::ensure(X);
        if (!Xf) throw std::runtime_error("X must be convertible to float32");
        if ((int)Xf.shape(1) != mdim_)
            throw std::runtime_error("X has " + std::to_string(Xf.shape(1)) + " features; the forest was fitted on " +
                                     std::to_string(mdim_));
        return Xf;
    }

    std::vector<int32_t> votes(const FArray& Xf) {
        ensure_ctx();
        const int m = (int)Xf.shape(0);
        std::vector<int32_t> v((size_t)m * nclass_);
        NoGil ng;
        check(rfx_predict(ctx_, Xf.data(), m, v.data()), "predict");
        return v;
    }

    // categorical auto-detection of fit (python/randomforest_py.cpp:771-805)
    void detect_categorical() {
        const int n = nsample_, p = mdim_;
        cat_.assign(p, 1);
        for (int m = 0; m < p; ++m) {
            std::set<float> u;
            bool all_int = true;
            float mn = 1e10f, mx = -1e10f;
            for (int i = 0; i < n; ++i) {
                const float v = X_[(size_t)i * p + m];
                u.insert(v);
                mn = std::min(mn, v);
                mx = std::max(mx, v);
                if (std::abs(v - std::round(v)) > 1e-5f) all_int = false;
            }
            const int nu = (int)u.size();
            if (all_int && nu > 1 && nu <= maxcat_ && mn >= 0.0f && mx < (float)maxcat_) cat_[m] = nu;
        }
    }

    void ensure_ctx() {
        if (ctx_) return;
        rfx_config cfg{};
        cfg.device = 0;
        cfg.use_casewise = use_casewise_ ? 1 : 0;
        cfg.n_threads_cpu = n_threads_cpu_;
        rfx_forest_view v{};
        v.n = nsample_;
        v.p = mdim_;
        v.nclass = nclass_;
        v.maxcat = maxcat_;
        v.ntree = ntree_;
        v.offs = offs_.data();
        v.nodestatus = nodestatus_.data();
        v.bestvar = bestvar_.data();
        v.xbestsplit = xbestsplit_.data();
        v.treemap = treemap_.data();
        v.nodeclass = nodeclass_.data();
        v.catgoleft = nullptr;  // the CPU grower leaves catgoleft all zero
        v.nin = nin_.data();
        v.X = X_.data();
        v.y = y_.data();
        v.cat = cat_.data();
        NoGil ng;
        rfx_ctx* c = nullptr;
        check(rfx_ctx_create(&cfg, &c), "CUDA context");
        rfx_status st = rfx_forest_load(c, &v);
        if (st != RFX_OK) {
            const std::string msg = rfx_last_error();
            rfx_ctx_destroy(c);
            throw std::runtime_error("forest load: " + msg);
        }
        ctx_ = c;
        lowrank_ready_ = false;
    }

    void release_ctx() {
        if (ctx_) {
            rfx_ctx_destroy(ctx_);
            ctx_ = nullptr;
        }
        lowrank_ready_ = false;
    }

    // Low-rank proximity factors of P ~= I + A A^T: rank `rank`, 16 extra
    // sketch columns, one power iteration; BF16 sketch storage with FP32
    // accumulation unless quant_mode is 'fp32'.  The factors are then stored
    // in the quant_mode's format ('fp16': FP16; 'int8': INT8 with one scale
    // per column; 'nf4': the reference's 4-bit code, two per byte, with one
    // scale per column) and every later use (get_lowrank_factors, MDS) reads
    // the stored values back; 'fp32' keeps the FP32 factors.
    void compute_lowrank() {
        ensure_ctx();
        const int n = nsample_;
        const int r = std::max(1, std::min(rank_, 64));
        lr_rank_ = r;
        lr_precision_ = quant_code_ == 0 ? 0 : 1;
        lr_quantized_ = quant_code_ >= 1;
        factors_.assign((size_t)n * r, 0.0f);
        NoGil ng;
        rfx_lowrank_opts o{};
        o.rank = r;
        o.oversample = 16;
        o.power_iters = 1;
        o.precision = lr_precision_;
        o.seed = (uint64_t)iseed_;
        std::vector<float> ev(r);
        check(rfx_lowrank(ctx_, &o, factors_.data(), ev.data()), "low-rank proximity");
        if (lr_quantized_) {
            const size_t nk = (size_t)n * r;
            std::vector<float> sc(r);
            if (quant_code_ == 1) {  // FP16
                std::vector<uint16_t> q(nk);
                check(rfx_lowrank_quantize(ctx_, 4, q.data(), sc.data()), "low-rank quantisation");
                for (size_t e = 0; e < nk; ++e) factors_[e] = half_to_float(q[e]);
            } else if (quant_code_ == 2) {  // INT8
                std::vector<int8_t> q(nk);
                check(rfx_lowrank_quantize(ctx_, 1, q.data(), sc.data()), "low-rank quantisation");
                for (int i = 0; i < n; ++i)
                    for (int col = 0; col < r; ++col)
                        factors_[(size_t)i * r + col] = (float)q[(size_t)i * r + col] * sc[col];
            } else {  // NF4
                std::vector<uint8_t> q((nk + 1) / 2);
                check(rfx_lowrank_quantize(ctx_, 3, q.data(), sc.data()), "low-rank quantisation");
                for (int i = 0; i < n; ++i)
                    for (int col = 0; col < r; ++col) {
                        const size_t e = (size_t)i * r + col;
                        const unsigned b = q[e >> 1];
                        const unsigned code = (e & 1) ? (b >> 4) : (b & 15u);
                        const float v = code <= 7 ? (float)code / 7.0f : -(float)(code - 8) / 7.0f;
                        factors_[e] = v * sc[col];
                    }
            }
        }
        lowrank_ready_ = true;
    }

    void duplicate_warning(const py::array_t<double>& coords) const {
        py::module_ np = py::module_::import("numpy");
        py::object rounded = np.attr("round")(coords, 6);
        py::object uniq = np.attr("unique")(rounded, py::arg("axis") = 0);
        const py::ssize_t n_unique = uniq.attr("shape").cast<py::tuple>()[0].cast<py::ssize_t>();
        const py::ssize_t n = nsample_;
        const py::ssize_t dup = n - n_unique;
        if (dup <= 0) return;
        const double pct = (double)dup / (double)n * 100.0;
        int rec;
        std::string cat;
        if (n < 500) {
            rec = (int)n * 8;
            cat = "8-10\xc3\x97 samples";
        } else if (n < 2000) {
            rec = (int)n * 6;
            cat = "6-8\xc3\x97 samples";
        } else if (n < 10000) {
            rec = (int)n * 5;
            cat = "5-7\xc3\x97 samples";
        } else {
            rec = (int)n * 4;
            cat = "3-5\xc3\x97 samples";
        }
        const std::string msg = "MDS coordinates have " + std::to_string(dup) + " duplicate points (" +
                                std::to_string((int)pct) + "% of " + std::to_string(n) + " samples). Only " +
                                std::to_string(n_unique) +
                                " unique positions will be visible. This typically indicates insufficient tree "
                                "coverage for proximity computation. Recommend ntree \xe2\x89\xa5 " +
                                std::to_string(rec) + " (" + cat + ") for complete MDS coverage.";
        py::module_::import("warnings").attr("warn")(msg, py::module_::import("builtins").attr("UserWarning"));
    }

    // configuration (constructor arguments)
    int nsample_, ntree_, mdim_, nclass_, maxcat_, mtry_ = 0, maxnode_ = 0, minndsize_, ncsplit_, ncmax_, iseed_;
    bool compute_proximity_, compute_importance_, compute_local_importance_, use_gpu_, use_qlora_;
    std::string quant_mode_;
    bool use_sparse_;
    float sparsity_threshold_;
    int batch_size_, nodesize_;
    float cutoff_;
    bool show_progress_;
    std::string progress_desc_, gpu_loss_function_;
    int rank_, n_threads_cpu_;
    bool use_rfgap_;
    std::string importance_method_;
    int clique_M_;
    bool use_casewise_;
    int quant_code_ = 3;

    // fitted state (host copies; the device holds its own)
    bool fitted_ = false;
    rfx_ctx* ctx_ = nullptr;
    std::vector<float> X_;
    std::vector<int32_t> y_, cat_;
    std::vector<int64_t> offs_;
    std::vector<int32_t> nodestatus_, bestvar_, treemap_, nodeclass_, nin_;
    std::vector<float> xbestsplit_;
    float oob_error_ = 0.0f;
    std::vector<int32_t> nout_, oob_pred_;
    std::vector<float> oob_proba_, importances_, local_imp_;
    std::vector<int32_t> S_;  // packed upper-triangle pair counts (full proximity mode)
    std::vector<double> Sd_;  // case-wise FP64 pair sums, or the RF-GAP matrix (packed upper triangle)
    bool lowrank_ready_ = false, lr_quantized_ = false;
    int lr_rank_ = 0, lr_precision_ = 0;
    std::vector<float> factors_;  // n x r row-major, as stored (dequantised when quantised)
};

}  // namespace

PYBIND11_MODULE(_rfx, m) {
    m.doc() = "rfx_b200: B200 post-growth random-forest analysis behind the rfx classification API";

    py::enum_<TaskType>(m, "TaskType")
        .value("CLASSIFICATION", TaskType::CLASSIFICATION)
        .value("REGRESSION", TaskType::REGRESSION)
        .value("UNSUPERVISED", TaskType::UNSUPERVISED);

    py::class_<RandomForestClassifier>(m, "RandomForestClassifier")
        .def(py::init<int, int, int, int, int, int, int, int, int, int, int, bool, bool, bool, bool, bool,
                      std::string, bool, float, int, int, float, bool, std::string, std::string, int, int, bool,
                      std::string, int, bool>(),
             py::arg("nsample") = 1000, py::arg("ntree") = 100, py::arg("mdim") = 10, py::arg("nclass") = 2,
             py::arg("maxcat") = 10, py::arg("mtry") = 0, py::arg("maxnode") = 0, py::arg("minndsize") = 1,
             py::arg("ncsplit") = 25, py::arg("ncmax") = 25, py::arg("iseed") = 12345,
             py::arg("compute_proximity") = false, py::arg("compute_importance") = true,
             py::arg("compute_local_importance") = false, py::arg("use_gpu") = false, py::arg("use_qlora") = false,
             py::arg("quant_mode") = "nf4", py::arg("use_sparse") = false, py::arg("sparsity_threshold") = 1e-6f,
             py::arg("batch_size") = 0, py::arg("nodesize") = 5, py::arg("cutoff") = 0.01f,
             py::arg("show_progress") = true, py::arg("progress_desc") = "Training Random Forest",
             py::arg("gpu_loss_function") = "gini", py::arg("rank") = 32, py::arg("n_threads_cpu") = 0,
             py::arg("use_rfgap") = false, py::arg("importance_method") = "local_imp", py::arg("clique_M") = -1,
             py::arg("use_casewise") = false)
        .def("fit", &RandomForestClassifier::fit, py::arg("X"), py::arg("y"), py::arg("sample_weight") = py::none())
        .def("predict", &RandomForestClassifier::predict)
        .def("predict_proba", &RandomForestClassifier::predict_proba)
        .def("get_oob_error", &RandomForestClassifier::get_oob_error)
        .def("feature_importances_", &RandomForestClassifier::feature_importances_)
        .def("get_task_type", &RandomForestClassifier::get_task_type)
        .def("get_n_samples", &RandomForestClassifier::get_n_samples)
        .def("get_n_features", &RandomForestClassifier::get_n_features)
        .def("get_n_classes", &RandomForestClassifier::get_n_classes)
        .def("get_local_importance", &RandomForestClassifier::get_local_importance)
        .def("get_proximity_matrix", &RandomForestClassifier::get_proximity_matrix)
        .def("compute_proximity_matrix", &RandomForestClassifier::get_proximity_matrix,
             "Alias for get_proximity_matrix()")
        .def("get_oob_predictions", &RandomForestClassifier::get_oob_predictions)
        .def("get_lowrank_factors", &RandomForestClassifier::get_lowrank_factors,
             "(A, B, r): factors of the low-rank proximity P ~= I + A A^T, float64 (n, r) arrays over a column-major "
             "buffer, B == A; quantised modes return the stored (dequantised) values.")
        .def("compute_mds_3d_cpu", &RandomForestClassifier::compute_mds_3d_cpu,
             "3-D MDS coordinates (n, 3) of the full proximity matrix; needs compute_proximity=True.")
        .def("compute_mds_from_factors", &RandomForestClassifier::compute_mds_from_factors, py::arg("k") = 3,
             "k-dimensional MDS coordinates (n, k) from the low-rank factors; needs use_qlora=True.")
        .def("compute_mds_3d_from_factors", &RandomForestClassifier::compute_mds_3d_from_factors)
        .def("cleanup", &RandomForestClassifier::cleanup,
             "Release the device memory; later calls that need the device load the forest again.");

    // confusion_matrix (python/randomforest_py.cpp:4262-4290)
    m.def(
        "confusion_matrix",
        [](IArray y_true, IArray y_pred) {
            const py::ssize_t n = y_true.shape(0);
            if (y_pred.shape(0) != n) throw std::runtime_error("y_true and y_pred must have the same length");
            const int32_t* t = y_true.data();
            const int32_t* p = y_pred.data();
            int32_t c = 0;
            for (py::ssize_t i = 0; i < n; ++i) {
                if (t[i] >= c) c = t[i] + 1;
                if (p[i] >= c) c = p[i] + 1;
            }
            py::array_t<int32_t> cm({(py::ssize_t)c, (py::ssize_t)c});
            int32_t* o = cm.mutable_data();
            std::fill(o, o + (size_t)c * c, 0);
            for (py::ssize_t i = 0; i < n; ++i)
                if (t[i] >= 0 && p[i] >= 0) o[(size_t)t[i] * c + p[i]]++;
            return cm;
        },
        "Compute confusion matrix", py::arg("y_true"), py::arg("y_pred"));

    // cuda_is_available (python/randomforest_py.cpp:4138-4146)
    m.def(
        "cuda_is_available",
        []() {
            rfx_config cfg{};
            rfx_ctx* c = nullptr;
            const bool ok = rfx_ctx_create(&cfg, &c) == RFX_OK;
            if (c) rfx_ctx_destroy(c);
            return ok;
        },
        "True if a CUDA device the library can use is present.");

    m.attr("__version__") = "1.0.2";
}
