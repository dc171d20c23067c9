// C ABI of librfx_b200: context, forest validation/upload, and the analysis
// entry points declared in include/rfx_b200.h.  No exception crosses the ABI.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "rfx_internal.cuh"

namespace rfxhost {
void bootstrap(int n, int tree, int32_t* nin);
int grow_forest(const float* X, const int32_t* y, int n, int p, int nclass, int ntree, int mtry, int minndsize,
                int maxnode, int iseed, int nthreads, std::vector<int64_t>& offs, std::vector<int32_t>& nodestatus,
                std::vector<int32_t>& bestvar, std::vector<float>& xbestsplit, std::vector<int32_t>& treemap,
                std::vector<int32_t>& nodeclass, int32_t* nin_all);
}

namespace rfx {

rfx_status launch_route_leaf(Ctx* c, int32_t* d_leaf);

namespace {
thread_local std::string g_last_error;

// MT19937 of include/rf_utils.hpp:74-141, for cpu_permobmr's permutations.
struct MT {
    uint32_t mt[624];
    int mti;
    void seed(uint32_t s) {
        mt[0] = s;
        for (mti = 1; mti < 624; ++mti) mt[mti] = 1812433253UL * (mt[mti - 1] ^ (mt[mti - 1] >> 30)) + (uint32_t)mti;
    }
    float randomu() {
        static const uint32_t mag01[2] = {0x0UL, 0x9908b0dfUL};
        uint32_t y;
        if (mti >= 624) {
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
        return (float)((double)y / (double)0xffffffffUL);
    }
};

// cpu_permobmr (src/rf_varimp.cpp:16-30): positions permuted by swaps with
// j = (int)(randomu() * noob), the generator reseeded with 42 for every call,
// so every noob uses the same draws u_0, u_1, ... (computed once, `u`).  A
// draw that rounds to 1.0f gives j == noob, which the reference uses to index
// one past its vector; it is counted and clamped here.
int make_perm(int noob, const float* u, int32_t* perm) {
    int bad = 0;
    for (int i = 0; i < noob; ++i) perm[i] = i;
    const float fn = (float)noob;
    for (int i = 0; i < noob; ++i) {
        int j = (int)(u[i] * fn);
        if (j >= noob) {
            j = noob - 1;
            ++bad;
        }
        std::swap(perm[i], perm[j]);
    }
    return bad;
}

std::vector<float> mt_draws(int count) {
    MT rng;
    rng.seed(42u);
    std::vector<float> u((size_t)std::max(count, 1));
    for (int i = 0; i < count; ++i) u[i] = rng.randomu();
    return u;
}

// Forest buffers go back to the context's pool, so reloading a forest of the
// same shape allocates nothing.
template <typename T>
void dfree(Ctx* c, T*& p) {
    if (p) c->pool_put(p);
    p = nullptr;
}

// cudaMalloc that, when device memory is short, first hands the context's
// kept scratch blocks back to the driver and tries once more.
cudaError_t ctx_malloc(Ctx* c, void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e == cudaErrorMemoryAllocation && !c->scratch_free.empty()) {
        cudaGetLastError();
        cudaStreamSynchronize(c->stream);
        c->scratch_release();
        e = cudaMalloc(p, bytes);
    }
    return e;
}

void free_forest(Ctx* c) {
    dfree(c, c->d_X); dfree(c, c->d_y); dfree(c, c->d_cat); dfree(c, c->d_nodes); dfree(c, c->d_nodeclass);
    dfree(c, c->d_leafidx); dfree(c, c->d_catgoleft); dfree(c, c->d_offs); dfree(c, c->d_nnode);
    dfree(c, c->d_inbag); dfree(c, c->d_segbase); dfree(c, c->d_iv); dfree(c, c->d_noob); dfree(c, c->d_permoff);
    dfree(c, c->d_invnoob); dfree(c, c->d_key); dfree(c, c->d_segoff); dfree(c, c->d_memb);
    dfree(c, c->d_votes); dfree(c, c->d_nout); dfree(c, c->d_joob); dfree(c, c->d_partner); dfree(c, c->d_oobord); dfree(c, c->d_vflags); dfree(c, c->d_flips);
    dfree(c, c->d_right); dfree(c, c->d_rightimp); dfree(c, c->d_qimp); dfree(c, c->d_qimpm); dfree(c, c->d_avimp);
    dfree(c, c->d_sqsd); dfree(c, c->d_opp); dfree(c, c->d_order);
    dfree(c, c->d_hubflag); dfree(c, c->d_hubtiles); dfree(c, c->d_hubstate);
    dfree(c, c->d_nin); dfree(c, c->d_tnodewt);
    dfree(c, c->d_lrA); dfree(c, c->d_lrAq); dfree(c, c->d_lrScale);
    if (c->d_lrQ) cudaFree(c->d_lrQ);
    c->d_lrQ = nullptr;
    c->lr_rank = 0;
    c->lr_qformat = 0;
    c->loaded = c->routed = c->csr_built = false;
    c->bytes = 0;
    c->generation++;
}

// Copy helper: device->(device|host) of `bytes` bytes on the context stream.
rfx_status copy_out(Ctx* c, void* dst, const void* src, size_t bytes) {
    if (!dst || bytes == 0) return RFX_OK;
    RFX_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, c->stream));
    return RFX_OK;
}

rfx_status finish_host(Ctx* c, bool any_host) {
    if (!any_host) return RFX_OK;
    RFX_CUDA(cudaStreamSynchronize(c->stream));
    return check_device_errors(c);
}

}  // namespace

void set_error(const std::string& msg) { g_last_error = msg; }

rfx_status cuda_fail(cudaError_t e, const char* what) {
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return RFX_ERR_OOM;
    }
    return RFX_ERR_CUDA;
}

bool is_device_ptr(const void* p) {
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

rfx_status check_device_errors(Ctx* c) {
    uint32_t bits = 0;
    RFX_CUDA(cudaMemcpy(&bits, c->d_err, sizeof(bits), cudaMemcpyDeviceToHost));
    if (!bits) return RFX_OK;
    RFX_CUDA(cudaMemset(c->d_err, 0, sizeof(uint32_t)));
    std::string m = "device checks raised:";
    if (bits & ERR_STALE_JVR)
        m += " a cpu_testreeimp walk ended without a terminal node (the reference would keep a stale vote);";
    if (bits & ERR_TRAVERSAL_LIMIT) m += " a walk hit its step limit;";
    if (bits & ERR_WAIT_LIMIT) m += " a tensor-core pipeline wait gave up;";
    set_error(m);
    return (bits & ERR_WAIT_LIMIT) ? RFX_ERR_TIMEOUT : RFX_ERR_UNSUPPORTED;
}

}  // namespace rfx

using namespace rfx;

// Device or host FP64 output of n(n+1)/2 entries through pooled staging.
template <typename F>
static rfx_status with_f64_out(Ctx* c, double* out, size_t len, const char* who, F&& fill) {
    const bool dev = is_device_ptr(out);
    Scratch staging(c);
    double* d = out;
    if (!dev) {
        d = staging.get<double>(len);
        if (!d) {
            set_error(std::string(who) + ": device staging allocation failed");
            return RFX_ERR_OOM;
        }
    }
    rfx_status st = fill(d);
    if (st == RFX_OK && !dev) {
        st = copy_out(c, out, d, sizeof(double) * len);
        if (st == RFX_OK) st = finish_host(c, true);
    }
    cudaStreamSynchronize(c->stream);
    return st;
}

extern "C" {

const char* rfx_last_error(void) { return g_last_error.c_str(); }

rfx_status rfx_ctx_create(const rfx_config* cfg, rfx_ctx** out) {
    if (!out) {
        set_error("rfx_ctx_create: out is null");
        return RFX_ERR_INVALID;
    }
    *out = nullptr;
    rfx_config conf{};
    if (cfg) conf = *cfg;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_error(std::string("no CUDA device: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "count is 0"));
        return RFX_ERR_NO_DEVICE;
    }
    if (conf.device < 0 || conf.device >= ndev) {
        set_error("device ordinal out of range");
        return RFX_ERR_INVALID;
    }
    Ctx* c = new (std::nothrow) Ctx();
    if (!c) return RFX_ERR_OOM;
    c->cfg = conf;
    c->device = conf.device;
    e = cudaSetDevice(c->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return cuda_fail(e, "rfx_ctx_create");
    }
    rfx_status st = dalloc(c, &c->d_err, 1);
    if (st == RFX_OK) st = dalloc(c, &c->d_pairs, 4);
    if (st != RFX_OK) {
        cudaStreamDestroy(c->stream);
        delete c;
        return st;
    }
    cudaMemset(c->d_err, 0, sizeof(uint32_t));
    *out = reinterpret_cast<rfx_ctx*>(c);
    return RFX_OK;
}

rfx_status rfx_ctx_destroy(rfx_ctx* ctx) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c) return RFX_OK;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    free_forest(c);
    for (int s = 0; s < ST_COUNT; ++s) {
        for (cudaEvent_t e : c->ev_start[s]) cudaEventDestroy(e);
        for (cudaEvent_t e : c->ev_end[s]) cudaEventDestroy(e);
    }
    dfree(c, c->d_perm);
    c->scratch_release();
    if (c->d_err) cudaFree(c->d_err);
    if (c->d_pairs) cudaFree(c->d_pairs);
    cudaStreamDestroy(c->stream);
    delete c;
    return RFX_OK;
}

rfx_status rfx_ctx_stream(rfx_ctx* ctx, void** stream) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c || !stream) return RFX_ERR_INVALID;
    *stream = (void*)c->stream;
    return RFX_OK;
}

rfx_status rfx_synchronize(rfx_ctx* ctx) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c) return RFX_ERR_INVALID;
    cudaSetDevice(c->device);
    RFX_CUDA(cudaStreamSynchronize(c->stream));
    return check_device_errors(c);
}

// What a forest load needs besides the context: sizes, the compact node
// offsets on the host, host copies of the labels and feature kinds (checked
// here), and a function that fills the device buffers from the caller's
// arrays (host arrays: H2D copies; device arrays: D2D copies and a gather of
// padded trees).
struct LoadInput {
    int n = 0, p = 0, nclass = 0, maxcat = 0, T = 0;
    const int64_t* offs = nullptr;  // host, T + 1
    const int32_t* y = nullptr;     // host, n
    const int32_t* cat = nullptr;   // host, p
    bool has_catgoleft = false;
    const char* who = "rfx_forest_load";
    // fills c->d_X, d_y, d_cat, d_nodeclass, d_catgoleft (if any) and the
    // compact raw node arrays and nin; c->d_offs is already on the device
    std::function<cudaError_t(cudaStream_t, Ctx*, int32_t*, int32_t*, float*, int32_t*, int32_t*)> upload;
};

static rfx_status load_forest(Ctx* c, const LoadInput& in) {
    const std::string who = in.who;
    try {
        cudaSetDevice(c->device);
        const int n = in.n, p = in.p, nclass = in.nclass, T = in.T;
        const int maxcat = in.maxcat;
        if (n < 1 || p < 1 || nclass < 1 || T < 1 || maxcat < 1) {
            set_error(who + ": n, p, nclass, ntree and maxcat must be >= 1");
            return RFX_ERR_INVALID;
        }
        if (p > 65535) {
            set_error(who + ": at most 65535 features");
            return RFX_ERR_UNSUPPORTED;
        }
        if (in.offs[0] != 0) {
            set_error(who + ": offs[0] must be 0");
            return RFX_ERR_FOREST;
        }
        for (int i = 0; i < n; ++i)
            if (in.y[i] < 0 || in.y[i] >= nclass) {
                set_error(who + ": label out of [0, nclass) at sample " + std::to_string(i));
                return RFX_ERR_INVALID;
            }
        if (in.has_catgoleft)
            for (int m = 0; m < p; ++m)
                if (in.cat[m] != 1 && in.cat[m] > maxcat) {
                    set_error(who + ": cat[m] exceeds maxcat with a catgoleft table");
                    return RFX_ERR_FOREST;
                }
        std::vector<int32_t> nnode(T), nleaf(T), noob(T);
        for (int t = 0; t < T; ++t) {
            const int64_t a = in.offs[t], b = in.offs[t + 1];
            // trees may come from a larger training set than the rows loaded
            // here (a row subsample), so only positivity and int32 range are checked
            if (b <= a || b - a > (int64_t)INT32_MAX / 2) {
                set_error(who + ": tree " + std::to_string(t) + " has an invalid node count");
                return RFX_ERR_FOREST;
            }
            nnode[t] = (int)(b - a);
        }
        const int64_t N = in.offs[T];
        const int W = (p + 63) / 64;

        // device buffers (from the pool when a forest of this shape was loaded
        // before); a load that fails leaves no forest loaded
        free_forest(c);
        c->n = n; c->p = p; c->nclass = nclass; c->maxcat = maxcat; c->T = T; c->N = N;
        rfx_status st = RFX_OK;
#define ALLOC(ptr, cnt) \
    if (st == RFX_OK) st = dalloc(c, &c->ptr, (size_t)(cnt));
        ALLOC(d_X, (size_t)n * p);
        ALLOC(d_y, n);
        ALLOC(d_cat, p);
        ALLOC(d_nodes, N);
        ALLOC(d_nodeclass, N);
        ALLOC(d_leafidx, N);
        if (in.has_catgoleft) ALLOC(d_catgoleft, (size_t)N * maxcat);
        ALLOC(d_offs, T + 1);
        ALLOC(d_nnode, T);
        ALLOC(d_inbag, (size_t)T * n);
        ALLOC(d_segbase, T + 1);
        ALLOC(d_iv, (size_t)T * W);
        ALLOC(d_noob, T);
        ALLOC(d_permoff, T);
        ALLOC(d_invnoob, T);
        ALLOC(d_key, (size_t)T * n);
        ALLOC(d_memb, (size_t)T * n);
        ALLOC(d_votes, (size_t)n * nclass);
        ALLOC(d_nout, n);
        if (st != RFX_OK) {
            free_forest(c);
            return st;
        }
        Scratch raw(c);
        int32_t* r_status = raw.get<int32_t>(N);
        int32_t* r_bestvar = raw.get<int32_t>(N);
        float* r_split = raw.get<float>(N);
        int32_t* r_treemap = raw.get<int32_t>(2 * (size_t)N);
        ALLOC(d_nin, (size_t)T * n);  // kept: case-wise weights and RF-GAP read the multiplicities
        int32_t* r_nin = c->d_nin;
        int32_t* r_nleaf = raw.get<int32_t>(T);
        LoadError* r_err = raw.get<LoadError>(1);
        if (!r_status || !r_bestvar || !r_split || !r_treemap || !r_nin || !r_nleaf || !r_err) {
            free_forest(c);
            set_error("rfx_forest_load: device allocation failed");
            return RFX_ERR_OOM;
        }
        cudaStream_t s = c->stream;
        auto up = [&](void* d, const void* h, size_t bytes) {
            return cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, s);
        };
        cudaError_t e = cudaMemsetAsync(r_err, 0, sizeof(LoadError), s);
        if (e == cudaSuccess) e = up(c->d_offs, in.offs, sizeof(int64_t) * (T + 1));
        if (e == cudaSuccess) e = up(c->d_nnode, nnode.data(), sizeof(int32_t) * T);
        if (e == cudaSuccess) e = in.upload(s, c, r_status, r_bestvar, r_split, r_treemap, r_nin);
        if (e != cudaSuccess) {
            free_forest(c);
            return cuda_fail(e, (who + " upload").c_str());
        }
        st = launch_pack_forest(s, T, n, p, c->d_offs, r_status, r_bestvar, r_split, r_treemap, c->d_cat, r_nin,
                                c->d_nodes, c->d_leafidx, c->d_iv, r_nleaf, c->d_inbag, c->d_noob, r_err);
        c->launches += 2;
        LoadError herr{};
        if (st == RFX_OK) {
            e = cudaMemcpyAsync(nleaf.data(), r_nleaf, sizeof(int32_t) * T, cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(noob.data(), c->d_noob, sizeof(int32_t) * T, cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, r_err, sizeof(LoadError), cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) st = cuda_fail(e, (who + " pack").c_str());
        }
        if (st == RFX_OK && herr.code) {
            const std::string where = " at tree " + std::to_string(herr.tree) + " node " + std::to_string(herr.node);
            switch (herr.code) {
                case 1: set_error(who + ": nodestatus out of range" + where); break;
                case 2: set_error(who + ": bestvar out of range" + where); break;
                case 3: set_error(who + ": child out of range" + where); break;
                default:
                    set_error(who + ": negative nin at tree " + std::to_string(herr.tree) + " sample " +
                              std::to_string(herr.node));
            }
            st = RFX_ERR_FOREST;
        }
        if (st != RFX_OK) {
            free_forest(c);
            return st;
        }
        std::vector<int64_t> segbase(T + 1, 0);
        for (int t = 0; t < T; ++t) segbase[t + 1] = segbase[t] + 2 * (int64_t)nleaf[t] + 1;

        // permutation tables per distinct noob (kept while the set of noob values repeats)
        std::vector<int> distinct(noob.begin(), noob.end());
        std::sort(distinct.begin(), distinct.end());
        distinct.erase(std::unique(distinct.begin(), distinct.end()), distinct.end());
        std::vector<int64_t> at(distinct.size());
        int64_t total = 0;
        for (size_t d = 0; d < distinct.size(); ++d) {
            at[d] = total;
            total += std::max(distinct[d], 1);
        }
        if (total > INT32_MAX) {
            free_forest(c);
            set_error(who + ": permutation tables too large");
            return RFX_ERR_UNSUPPORTED;
        }
        if (!c->d_perm || distinct != c->perm_noobs) {
            dfree(c, c->d_perm);
            c->perm_noobs.clear();
            std::vector<int32_t> perm((size_t)total);
            const std::vector<float> u = mt_draws(distinct.empty() ? 1 : distinct.back());
            std::vector<std::thread> th;
            const int nth = std::max(1, std::min<int>((int)std::thread::hardware_concurrency(), (int)distinct.size()));
            std::atomic<int> next{0};
            for (int q = 0; q < nth; ++q)
                th.emplace_back([&]() {
                    for (;;) {
                        const int d = next.fetch_add(1);
                        if (d >= (int)distinct.size()) break;
                        make_perm(distinct[d], u.data(), perm.data() + at[d]);
                    }
                });
            for (auto& x : th) x.join();
            if ((st = dalloc(c, &c->d_perm, (size_t)total)) != RFX_OK) {
                free_forest(c);
                return st;
            }
            e = up(c->d_perm, perm.data(), sizeof(int32_t) * (size_t)total);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) {
                free_forest(c);
                return cuda_fail(e, (who + " permutation upload").c_str());
            }
            c->perm_noobs = distinct;
        }
        std::vector<int32_t> permoff(T);
        std::vector<float> invnoob(T);
        for (int t = 0; t < T; ++t) {
            permoff[t] = (int32_t)at[std::lower_bound(distinct.begin(), distinct.end(), noob[t]) - distinct.begin()];
            volatile float f = (float)noob[t];
            invnoob[t] = 1.0f / f;
        }
        c->h_offs.assign(in.offs, in.offs + T + 1);
        c->h_nnode = nnode;
        c->h_nleaf = nleaf;
        c->h_segbase = segbase;
        c->h_noob = noob;
        c->iv_words = W;
        c->max_keys = 0;
        c->max_nnode = 0;
        for (int t = 0; t < T; ++t) {
            c->max_keys = std::max(c->max_keys, 2 * nleaf[t]);
            c->max_nnode = std::max(c->max_nnode, nnode[t]);
        }
        ALLOC(d_segoff, segbase[T]);
#undef ALLOC
        if (st != RFX_OK) {
            free_forest(c);
            return st;
        }
        e = up(c->d_segbase, segbase.data(), sizeof(int64_t) * (T + 1));
        if (e == cudaSuccess) e = up(c->d_permoff, permoff.data(), sizeof(int32_t) * T);
        if (e == cudaSuccess) e = up(c->d_invnoob, invnoob.data(), sizeof(float) * T);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            free_forest(c);
            return cuda_fail(e, (who + " upload").c_str());
        }
        c->loaded = true;
        return RFX_OK;
    } catch (const std::bad_alloc&) {
        set_error(who + ": host allocation failed");
        return RFX_ERR_OOM;
    } catch (const std::exception& ex) {
        set_error(who + ": " + ex.what());
        return RFX_ERR_INVALID;
    }
}

rfx_status rfx_forest_load(rfx_ctx* ctx, const rfx_forest_view* v) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c || !v) {
        set_error("rfx_forest_load: null argument");
        return RFX_ERR_INVALID;
    }
    if (!v->offs || !v->nodestatus || !v->bestvar || !v->xbestsplit || !v->treemap || !v->nodeclass || !v->nin ||
        !v->X || !v->y || !v->cat) {
        set_error("rfx_forest_load: a required array is null");
        return RFX_ERR_INVALID;
    }
    LoadInput in;
    in.n = v->n; in.p = v->p; in.nclass = v->nclass; in.maxcat = v->maxcat; in.T = v->ntree;
    in.offs = v->offs; in.y = v->y; in.cat = v->cat; in.has_catgoleft = v->catgoleft != nullptr;
    in.upload = [v](cudaStream_t s, Ctx* c, int32_t* r_status, int32_t* r_bestvar, float* r_split, int32_t* r_treemap,
                    int32_t* r_nin) -> cudaError_t {
        const int n = v->n, p = v->p, T = v->ntree;
        const size_t N = (size_t)v->offs[T];
        auto up = [&](void* d, const void* h, size_t bytes) {
            return cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, s);
        };
        cudaError_t e = up(c->d_X, v->X, sizeof(float) * (size_t)n * p);
        if (e == cudaSuccess) e = up(c->d_y, v->y, sizeof(int32_t) * n);
        if (e == cudaSuccess) e = up(c->d_cat, v->cat, sizeof(int32_t) * p);
        if (e == cudaSuccess) e = up(r_status, v->nodestatus, sizeof(int32_t) * N);
        if (e == cudaSuccess) e = up(r_bestvar, v->bestvar, sizeof(int32_t) * N);
        if (e == cudaSuccess) e = up(r_split, v->xbestsplit, sizeof(float) * N);
        if (e == cudaSuccess) e = up(r_treemap, v->treemap, sizeof(int32_t) * 2 * N);
        if (e == cudaSuccess) e = up(c->d_nodeclass, v->nodeclass, sizeof(int32_t) * N);
        if (e == cudaSuccess && v->catgoleft) e = up(c->d_catgoleft, v->catgoleft, sizeof(int32_t) * N * v->maxcat);
        if (e == cudaSuccess) e = up(r_nin, v->nin, sizeof(int32_t) * (size_t)T * n);
        return e;
    };
    return load_forest(c, in);
}

rfx_status rfx_forest_load_device(rfx_ctx* ctx, const rfx_forest_device_view* v) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c || !v) {
        set_error("rfx_forest_load_device: null argument");
        return RFX_ERR_INVALID;
    }
    if (!v->nnode || !v->nodestatus || !v->bestvar || !v->xbestsplit || !v->treemap || !v->nodeclass || !v->nin ||
        !v->X || !v->y || !v->cat) {
        set_error("rfx_forest_load_device: a required array is null");
        return RFX_ERR_INVALID;
    }
    const int n = v->n, p = v->p, T = v->ntree, maxnode = v->maxnode, maxcat = v->maxcat;
    if (n < 1 || p < 1 || T < 1 || maxnode < 1 || maxcat < 1) {
        set_error("rfx_forest_load_device: n, p, ntree, maxnode and maxcat must be >= 1");
        return RFX_ERR_INVALID;
    }
    cudaSetDevice(c->device);
    const void* dev_arrays[] = {v->nodestatus, v->bestvar, v->xbestsplit, v->treemap, v->nodeclass, v->nin,
                                v->X, v->y, v->cat};
    for (const void* a : dev_arrays)
        if (!is_device_ptr(a)) {
            set_error("rfx_forest_load_device: the forest and data arrays must be device memory (nnode stays on the host)");
            return RFX_ERR_INVALID;
        }
    if (v->catgoleft && !is_device_ptr(v->catgoleft)) {
        set_error("rfx_forest_load_device: catgoleft must be device memory");
        return RFX_ERR_INVALID;
    }
    try {
        std::vector<int64_t> offs(T + 1, 0);
        for (int t = 0; t < T; ++t) {
            if (v->nnode[t] < 1 || v->nnode[t] > maxnode) {
                set_error("rfx_forest_load_device: nnode[" + std::to_string(t) + "] outside [1, maxnode]");
                return RFX_ERR_FOREST;
            }
            offs[t + 1] = offs[t] + v->nnode[t];
        }
        std::vector<int32_t> y(n), cat(p);
        RFX_CUDA(cudaMemcpy(y.data(), v->y, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
        RFX_CUDA(cudaMemcpy(cat.data(), v->cat, sizeof(int32_t) * p, cudaMemcpyDeviceToHost));
        LoadInput in;
        in.n = n; in.p = p; in.nclass = v->nclass; in.maxcat = maxcat; in.T = T;
        in.offs = offs.data(); in.y = y.data(); in.cat = cat.data(); in.has_catgoleft = v->catgoleft != nullptr;
        in.who = "rfx_forest_load_device";
        in.upload = [v](cudaStream_t s, Ctx* c, int32_t* r_status, int32_t* r_bestvar, float* r_split,
                        int32_t* r_treemap, int32_t* r_nin) -> cudaError_t {
            const int n = v->n, p = v->p, T = v->ntree;
            auto cp = [&](void* d, const void* src, size_t bytes) {
                return cudaMemcpyAsync(d, src, bytes, cudaMemcpyDeviceToDevice, s);
            };
            cudaError_t e = cp(c->d_X, v->X, sizeof(float) * (size_t)n * p);
            if (e == cudaSuccess) e = cp(c->d_y, v->y, sizeof(int32_t) * n);
            if (e == cudaSuccess) e = cp(c->d_cat, v->cat, sizeof(int32_t) * p);
            if (e == cudaSuccess) e = cp(r_nin, v->nin, sizeof(int32_t) * (size_t)T * n);
            if (e == cudaSuccess)
                e = launch_gather_padded(s, T, v->maxnode, v->maxcat, c->d_offs, v->nodestatus, v->bestvar,
                                         v->xbestsplit, v->treemap, v->nodeclass, v->catgoleft, r_status, r_bestvar,
                                         r_split, r_treemap, c->d_nodeclass, c->d_catgoleft);
            return e;
        };
        return load_forest(c, in);
    } catch (const std::bad_alloc&) {
        set_error("rfx_forest_load_device: host allocation failed");
        return RFX_ERR_OOM;
    }
}

static rfx_status casewise_votes_into(Ctx* c, float* dq);

static rfx_status need_forest(Ctx* c) {
    if (!c) {
        set_error("null context");
        return RFX_ERR_INVALID;
    }
    if (!c->loaded) {
        set_error("no forest loaded");
        return RFX_ERR_STATE;
    }
    cudaSetDevice(c->device);
    return RFX_OK;
}

rfx_status rfx_route_oob(rfx_ctx* ctx, int32_t* q, int32_t* nout, int32_t* leaf) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    rfx_status st = need_forest(c);
    if (st) return st;
    if (q && c->cfg.use_casewise) {
        set_error("rfx_route_oob: a case-wise context weighs the votes (float): use rfx_casewise_votes");
        return RFX_ERR_STATE;
    }
    bool any_host = false;
    if (leaf) {
        int32_t* dleaf = leaf;
        const bool dev = is_device_ptr(leaf);
        if (!dev) {
            if ((st = dalloc(c, &c->d_joob, (size_t)c->T * c->n))) return st;  // reuse as staging
            dleaf = c->d_joob;
        }
        if ((st = launch_route_leaf(c, dleaf))) return st;
        RFX_CUDA(cudaGetLastError());
        if (!dev) {
            if ((st = copy_out(c, leaf, dleaf, sizeof(int32_t) * (size_t)c->T * c->n))) return st;
            any_host = true;
        }
        // nout is produced by launch_route; run it as well (cheap)
    }
    if ((st = launch_route(c))) return st;
    c->routed = true;
    c->csr_built = false;
    if (q) {
        any_host |= !is_device_ptr(q);
        if ((st = copy_out(c, q, c->d_votes, sizeof(int32_t) * (size_t)c->n * c->nclass))) return st;
    }
    if (nout) {
        any_host |= !is_device_ptr(nout);
        if ((st = copy_out(c, nout, c->d_nout, sizeof(int32_t) * (size_t)c->n))) return st;
    }
    return finish_host(c, any_host);
}

rfx_status rfx_oob_summary(rfx_ctx* ctx, float* oob_error, int32_t* pred, float* proba) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    rfx_status st = need_forest(c);
    if (st) return st;
    if (!c->routed) {
        if ((st = launch_route(c))) return st;
        c->routed = true;
    }
    float* d_e = nullptr;
    int32_t* d_p = nullptr;
    float* d_pr = nullptr;
    const bool he = oob_error && !is_device_ptr(oob_error);
    const bool hp = pred && !is_device_ptr(pred);
    const bool hpr = proba && !is_device_ptr(proba);
    std::vector<void*> tmp;
    auto tmpalloc = [&](size_t bytes) -> void* {
        void* d = nullptr;
        if (ctx_malloc(c, (void**)&d, bytes) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        tmp.push_back(d);
        return d;
    };
    d_e = he ? (float*)tmpalloc(sizeof(float)) : oob_error;
    d_p = hp ? (int32_t*)tmpalloc(sizeof(int32_t) * c->n) : pred;
    d_pr = hpr ? (float*)tmpalloc(sizeof(float) * (size_t)c->n * c->nclass) : proba;
    if ((he && !d_e) || (hp && !d_p) || (hpr && !d_pr)) {
        for (void* d : tmp) cudaFree(d);
        set_error("rfx_oob_summary: staging allocation failed");
        return RFX_ERR_OOM;
    }
    if (c->cfg.use_casewise) {
        // the weighted votes of rfx_casewise_votes (computed here)
        Scratch sq(c);
        float* dq = sq.get<float>((size_t)c->n * c->nclass);
        if (!dq) st = RFX_ERR_OOM;
        if (st == RFX_OK) st = casewise_votes_into(c, dq);
        if (st == RFX_OK) st = launch_oob_summary_f32(c, dq, d_e, d_p, d_pr);
        if (st == RFX_OK) cudaStreamSynchronize(c->stream);
    } else {
        st = launch_oob_summary(c, d_e, d_p, d_pr);
    }
    if (st == RFX_OK && he) st = copy_out(c, oob_error, d_e, sizeof(float));
    if (st == RFX_OK && hp) st = copy_out(c, pred, d_p, sizeof(int32_t) * c->n);
    if (st == RFX_OK && hpr) st = copy_out(c, proba, d_pr, sizeof(float) * (size_t)c->n * c->nclass);
    if (st == RFX_OK) st = finish_host(c, he || hp || hpr);
    cudaStreamSynchronize(c->stream);
    for (void* d : tmp) cudaFree(d);
    return st;
}

rfx_status rfx_proximity_upper_i32(rfx_ctx* ctx, int32_t* S, size_t len) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    rfx_status st = need_forest(c);
    if (st) return st;
    if (c->cfg.use_casewise) {
        set_error("rfx_proximity_upper_i32: a case-wise context weighs the pairs (FP64): use rfx_proximity_upper_f64");
        return RFX_ERR_STATE;
    }
    if (!S || len != (size_t)upper_len(c->n)) {
        set_error("rfx_proximity_upper_i32: S must hold n(n+1)/2 entries");
        return RFX_ERR_INVALID;
    }
    const bool dev = is_device_ptr(S);
    int32_t* dS = S;
    Scratch staging(c);  // device staging for a host S, kept in the context's pool between calls
    if (!dev) {
        dS = staging.get<int32_t>(len);
        if (!dS) {
            set_error("rfx_proximity_upper_i32: device staging allocation failed");
            return RFX_ERR_OOM;
        }
    }
    // every call does the full pass: routing, per-tree leaf lists, pair counts
    st = launch_route(c);
    if (st == RFX_OK) st = launch_build_csr(c);
    if (st == RFX_OK) st = launch_pairs_upper(c, dS);
    if (st == RFX_OK) {
        c->routed = true;
        c->csr_built = true;
    }
    if (st == RFX_OK && !dev) {
        st = copy_out(c, S, dS, sizeof(int32_t) * len);
        if (st == RFX_OK) st = finish_host(c, true);
    }
    if (!dev) cudaStreamSynchronize(c->stream);
    return st;
}

// Case-wise weighted OOB votes (n x nclass float) into device memory.
static rfx_status casewise_votes_into(Ctx* c, float* dq) {
    Scratch sl(c);
    int32_t* dleaf = sl.get<int32_t>((size_t)c->T * c->n);
    if (!dleaf) {
        set_error("case-wise votes: scratch allocation failed");
        return RFX_ERR_OOM;
    }
    rfx_status st = launch_route_leaf(c, dleaf);  // node ids, and nout
    if (st == RFX_OK) st = launch_route(c);
    if (st == RFX_OK) {
        c->routed = true;
        c->csr_built = false;
        st = launch_tnodewt(c);
    }
    if (st == RFX_OK) st = launch_casewise_votes(c, dleaf, dq);
    if (st == RFX_OK) RFX_CUDA(cudaStreamSynchronize(c->stream));  // the scratch goes back to the pool
    return st;
}

rfx_status rfx_casewise_votes(rfx_ctx* ctx, float* q, int32_t* nout) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    rfx_status st = need_forest(c);
    if (st) return st;
    if (!c->cfg.use_casewise) {
        set_error("rfx_casewise_votes: the context was created without use_casewise");
        return RFX_ERR_STATE;
    }
    if (!q) {
        set_error("rfx_casewise_votes: q is null");
        return RFX_ERR_INVALID;
    }
    const size_t nq = (size_t)c->n * c->nclass;
    Scratch sq(c);
    const bool dev = is_device_ptr(q);
    float* dq = dev ? q : sq.get<float>(nq);
    if (!dq) return RFX_ERR_OOM;
    if ((st = casewise_votes_into(c, dq))) return st;
    bool any_host = false;
    if (!dev) {
        if ((st = copy_out(c, q, dq, sizeof(float) * nq))) return st;
        any_host = true;
    }
    if (nout) {
        any_host |= !is_device_ptr(nout);
        if ((st = copy_out(c, nout, c->d_nout, sizeof(int32_t) * (size_t)c->n))) return st;
    }
    st = finish_host(c, any_host);
    cudaStreamSynchronize(c->stream);
    return st;
}

rfx_status rfx_proximity_upper_f64(rfx_ctx* ctx, double* S, size_t len) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    rfx_status st = need_forest(c);
    if (st) return st;
    if (!S || len != (size_t)upper_len(c->n)) {
        set_error("rfx_proximity_upper_f64: S must hold n(n+1)/2 entries");
        return RFX_ERR_INVALID;
    }
    return with_f64_out(c, S, len, "rfx_proximity_upper_f64", [&](double* dS) -> rfx_status {
        rfx_status s = launch_route(c);
        if (s == RFX_OK) s = launch_build_csr(c);
        if (s != RFX_OK) return s;
        c->routed = true;
        c->csr_built = true;
        StageTimer stt(c, ST_PAIRS, 0);
        return launch_weighted_rows(c, c->cfg.use_casewise ? 0 : 2, c->d_key, c->d_segbase, c->d_segoff, c->d_memb,
                                    c->h_segbase[c->T], dS);
    });
}

rfx_status rfx_finishprox_f64(rfx_ctx* ctx, const double* S, float* P, int full) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    rfx_status st = need_forest(c);
    if (st) return st;
    if (!S || !P) {
        set_error("rfx_finishprox_f64: null argument");
        return RFX_ERR_INVALID;
    }
    if (!c->routed) {
        if ((st = launch_route(c))) return st;
        c->routed = true;
    }
    const size_t slen = (size_t)upper_len(c->n);
    const size_t plen = full ? (size_t)c->n * c->n : slen;
    const bool sdev = is_device_ptr(S), pdev = is_device_ptr(P);
    Scratch sc(c);
    const double* dS = S;
    float* dP = P;
    if (!sdev) {
        double* t = sc.get<double>(slen);
        if (!t) return RFX_ERR_OOM;
        RFX_CUDA(cudaMemcpyAsync(t, S, sizeof(double) * slen, cudaMemcpyHostToDevice, c->stream));
        dS = t;
    }
    if (!pdev) {
        dP = sc.get<float>(plen);
        if (!dP) return RFX_ERR_OOM;
    }
    st = launch_finishprox_f64(c, dS, dP, full);
    if (st == RFX_OK && !pdev) st = copy_out(c, P, dP, sizeof(float) * plen);
    if (st == RFX_OK) st = finish_host(c, !sdev || !pdev);
    cudaStreamSynchronize(c->stream);
    return st;
}

rfx_status rfx_proximity_rfgap(rfx_ctx* ctx, double* P, size_t len) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    rfx_status st = need_forest(c);
    if (st) return st;
    if (!P || len != (size_t)upper_len(c->n)) {
        set_error("rfx_proximity_rfgap: P must hold n(n+1)/2 entries");
        return RFX_ERR_INVALID;
    }
    return with_f64_out(c, P, len, "rfx_proximity_rfgap", [&](double* dP) -> rfx_status {
        const int T = c->T, n = c->n;
        Scratch sc(c);
        int32_t* leaf = sc.get<int32_t>((size_t)T * n);
        int32_t* key = sc.get<int32_t>((size_t)T * n);
        int32_t* memb = sc.get<int32_t>((size_t)T * n);
        // node-id keys: 2 * nnode + 1 slots per tree
        std::vector<int64_t> sb(T + 1, 0);
        for (int t = 0; t < T; ++t) sb[t + 1] = sb[t] + 2 * (int64_t)c->h_nnode[t] + 1;
        int64_t* dsb = sc.get<int64_t>((size_t)T + 1);
        int32_t* segoff = sc.get<int32_t>((size_t)sb[T]);
        if (!leaf || !key || !memb || !dsb || !segoff) {
            set_error("rfx_proximity_rfgap: scratch allocation failed");
            return RFX_ERR_OOM;
        }
        RFX_CUDA(cudaMemcpyAsync(dsb, sb.data(), sizeof(int64_t) * (T + 1), cudaMemcpyHostToDevice, c->stream));
        rfx_status s = launch_route_leaf(c, leaf);  // node ids (and nout)
        if (s == RFX_OK) s = launch_route(c);
        if (s != RFX_OK) return s;
        c->routed = true;
        c->csr_built = false;
        if ((s = launch_gap_keys(c, leaf, key))) return s;
        if ((s = launch_build_csr_raw(c->stream, c->device, key, n, T, dsb, segoff, memb, 2 * c->max_nnode,
                                      c->d_err)))
            return s;
        StageTimer stt(c, ST_PAIRS, 0);
        s = launch_weighted_rows(c, 1, key, dsb, segoff, memb, sb[T], dP);
        if (s == RFX_OK) RFX_CUDA(cudaStreamSynchronize(c->stream));  // the scratch goes back to the pool
        return s;
    });
}

rfx_status rfx_pair_updates(rfx_ctx* ctx, int64_t* count) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    rfx_status st = need_forest(c);
    if (st) return st;
    if (!count) return RFX_ERR_INVALID;
    unsigned long long v = 0;
    RFX_CUDA(cudaStreamSynchronize(c->stream));
    RFX_CUDA(cudaMemcpy(&v, c->d_pairs, sizeof(v), cudaMemcpyDeviceToHost));
    *count = (int64_t)v;
    return RFX_OK;
}

rfx_status rfx_finishprox(rfx_ctx* ctx, const int32_t* S, float* P, int full) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    rfx_status st = need_forest(c);
    if (st) return st;
    if (!S || !P) {
        set_error("rfx_finishprox: null argument");
        return RFX_ERR_INVALID;
    }
    if (!c->routed) {
        if ((st = launch_route(c))) return st;
        c->routed = true;
    }
    const size_t slen = (size_t)upper_len(c->n);
    const size_t plen = full ? (size_t)c->n * c->n : slen;
    const bool sdev = is_device_ptr(S), pdev = is_device_ptr(P);
    const int32_t* dS = S;
    float* dP = P;
    int32_t* sS = nullptr;
    if (!sdev) {
        cudaError_t e = ctx_malloc(c, (void**)&sS, sizeof(int32_t) * slen);
        if (e != cudaSuccess) return cuda_fail(e, "rfx_finishprox staging");
        e = cudaMemcpyAsync(sS, S, sizeof(int32_t) * slen, cudaMemcpyHostToDevice, c->stream);
        if (e != cudaSuccess) {
            cudaFree(sS);
            return cuda_fail(e, "rfx_finishprox H2D");
        }
        dS = sS;
    }
    if (!pdev) {
        cudaError_t e = ctx_malloc(c, (void**)&dP, sizeof(float) * plen);
        if (e != cudaSuccess) {
            if (sS) cudaFree(sS);
            return cuda_fail(e, "rfx_finishprox staging");
        }
    }
    st = launch_finishprox(c, dS, dP, full);
    if (st == RFX_OK && !pdev) st = copy_out(c, P, dP, sizeof(float) * plen);
    if (st == RFX_OK) st = finish_host(c, !sdev || !pdev);
    if (!sdev || !pdev) cudaStreamSynchronize(c->stream);
    if (sS) cudaFree(sS);
    if (!pdev) cudaFree(dP);
    return st;
}

rfx_status rfx_varimp(rfx_ctx* ctx, int impn, float* avimp, float* sqsd, float* qimp, float* qimpm) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    rfx_status st = need_forest(c);
    if (st) return st;
    const int T = c->T, n = c->n, p = c->p, W = varimp_flip_words(c->iv_words);
#define ALLOC(ptr, cnt) \
    if (st == RFX_OK) st = dalloc(c, &c->ptr, (size_t)(cnt));
    ALLOC(d_joob, (size_t)T * n);
    ALLOC(d_partner, (size_t)T * n);
    ALLOC(d_oobord, (size_t)T * n);
    ALLOC(d_vflags, (size_t)T * n);
    ALLOC(d_flips, (size_t)T * n * W);
    ALLOC(d_right, 2 * (size_t)T);
    ALLOC(d_rightimp, (size_t)T * p);
    ALLOC(d_qimp, n);
    ALLOC(d_qimpm, (size_t)n * p);
    ALLOC(d_avimp, p);
    ALLOC(d_sqsd, p);
#undef ALLOC
    if (st) return st;
    if (c->cfg.use_casewise) {
        // weights of the testreebag nodes; OOB lists and permutation partners
        Scratch sl(c);
        int32_t* dleaf = sl.get<int32_t>((size_t)T * n);
        if (!dleaf) return RFX_ERR_OOM;
        if ((st = launch_route_leaf(c, dleaf))) return st;
        if ((st = launch_tnodewt(c))) return st;
        if ((st = launch_joob_partner(c))) return st;
        RFX_CUDA(cudaMemsetAsync(c->d_err, 0, sizeof(uint32_t), c->stream));
        {
            StageTimer stt(c, ST_VARIMP_TREE, 0);
            if ((st = launch_casewise_varimp(c, dleaf, impn ? 1 : 0, c->d_avimp, c->d_sqsd, c->d_qimp, c->d_qimpm)))
                return st;
        }
        RFX_CUDA(cudaStreamSynchronize(c->stream));
        if ((st = check_device_errors(c))) return st;
    } else if ((st = launch_varimp(c, impn ? 1 : 0))) {
        return st;
    }
    bool any_host = false;
    auto out = [&](float* dst, const float* src, size_t cnt) -> rfx_status {
        if (!dst) return RFX_OK;
        any_host |= !is_device_ptr(dst);
        return copy_out(c, dst, src, sizeof(float) * cnt);
    };
    if ((st = out(avimp, c->d_avimp, p))) return st;
    if ((st = out(sqsd, c->d_sqsd, p))) return st;
    if (impn) {
        if ((st = out(qimp, c->d_qimp, n))) return st;
        if ((st = out(qimpm, c->d_qimpm, (size_t)n * p))) return st;
    }
    return finish_host(c, any_host);
}

rfx_status rfx_localimp(rfx_ctx* ctx, const float* qimp, const float* qimpm, float* outp) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    rfx_status st = need_forest(c);
    if (st) return st;
    if (!qimp || !qimpm || !outp) return RFX_ERR_INVALID;
    const size_t np = (size_t)c->n * c->p;
    std::vector<void*> tmp;
    auto stage_in = [&](const float* h, size_t cnt) -> const float* {
        if (is_device_ptr(h)) return h;
        float* d = nullptr;
        if (ctx_malloc(c, (void**)&d, sizeof(float) * cnt) != cudaSuccess) return nullptr;
        tmp.push_back(d);
        cudaMemcpyAsync(d, h, sizeof(float) * cnt, cudaMemcpyHostToDevice, c->stream);
        return d;
    };
    const float* dq = stage_in(qimp, c->n);
    const float* dqm = stage_in(qimpm, np);
    const bool odev = is_device_ptr(outp);
    float* dout = outp;
    if (!odev) {
        if (ctx_malloc(c, (void**)&dout, sizeof(float) * np) != cudaSuccess) dout = nullptr;
        else tmp.push_back(dout);
    }
    if (!dq || !dqm || !dout) {
        cudaGetLastError();
        cudaStreamSynchronize(c->stream);
        for (void* d : tmp) cudaFree(d);
        set_error("rfx_localimp: staging allocation failed");
        return RFX_ERR_OOM;
    }
    st = launch_localimp(c, dq, dqm, dout);
    if (st == RFX_OK && !odev) st = copy_out(c, outp, dout, sizeof(float) * np);
    if (st == RFX_OK) st = finish_host(c, !tmp.empty());
    cudaStreamSynchronize(c->stream);
    for (void* d : tmp) cudaFree(d);
    return st;
}

rfx_status rfx_predict(rfx_ctx* ctx, const float* X, int32_t m, int32_t* votes) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    rfx_status st = need_forest(c);
    if (st) return st;
    if (m < 0 || (!X && m > 0) || !votes) return RFX_ERR_INVALID;
    const bool xdev = is_device_ptr(X), vdev = is_device_ptr(votes);
    const float* dX = X;
    int32_t* dv = votes;
    std::vector<void*> tmp;
    if (!xdev && m > 0) {
        float* d = nullptr;
        cudaError_t e = ctx_malloc(c, (void**)&d, sizeof(float) * (size_t)m * c->p);
        if (e != cudaSuccess) return cuda_fail(e, "rfx_predict staging");
        tmp.push_back(d);
        cudaMemcpyAsync(d, X, sizeof(float) * (size_t)m * c->p, cudaMemcpyHostToDevice, c->stream);
        dX = d;
    }
    if (!vdev) {
        int32_t* d = nullptr;
        cudaError_t e = ctx_malloc(c, (void**)&d, sizeof(int32_t) * std::max<size_t>(1, (size_t)m * c->nclass));
        if (e != cudaSuccess) {
            for (void* q : tmp) cudaFree(q);
            return cuda_fail(e, "rfx_predict staging");
        }
        tmp.push_back(d);
        dv = d;
    }
    st = launch_predict(c, dX, m, dv);
    if (st == RFX_OK && !vdev) st = copy_out(c, votes, dv, sizeof(int32_t) * (size_t)m * c->nclass);
    if (st == RFX_OK) st = finish_host(c, !tmp.empty());
    cudaStreamSynchronize(c->stream);
    for (void* q : tmp) cudaFree(q);
    return st;
}

rfx_status rfx_mds3d_full(rfx_ctx* ctx, const float* P, double* coords, double* evals) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    rfx_status st = need_forest(c);
    if (st) return st;
    if (!P || !coords) {
        set_error("rfx_mds3d_full: null argument");
        return RFX_ERR_INVALID;
    }
    if (!c->routed) {
        if ((st = launch_route(c))) return st;
        c->routed = true;
    }
    const size_t nn = (size_t)c->n * c->n;
    const float* dP = P;
    float* sP = nullptr;
    if (!is_device_ptr(P)) {
        cudaError_t e = ctx_malloc(c, (void**)&sP, sizeof(float) * nn);
        if (e != cudaSuccess) return cuda_fail(e, "rfx_mds3d_full staging");
        e = cudaMemcpyAsync(sP, P, sizeof(float) * nn, cudaMemcpyHostToDevice, c->stream);
        if (e != cudaSuccess) {
            cudaFree(sP);
            return cuda_fail(e, "rfx_mds3d_full H2D");
        }
        dP = sP;
    }
    const bool cdev = is_device_ptr(coords);
    double* dC = coords;
    if (!cdev) {
        cudaError_t e = ctx_malloc(c, (void**)&dC, sizeof(double) * (size_t)c->n * 3);
        if (e != cudaSuccess) {
            if (sP) cudaFree(sP);
            return cuda_fail(e, "rfx_mds3d_full staging");
        }
    }
    double ev[3] = {0, 0, 0};
    st = launch_mds3d_full(c, dP, dC, ev);
    if (st == RFX_OK && !cdev) st = copy_out(c, coords, dC, sizeof(double) * (size_t)c->n * 3);
    if (st == RFX_OK) st = finish_host(c, true);
    cudaStreamSynchronize(c->stream);
    if (sP) cudaFree(sP);
    if (!cdev) cudaFree(dC);
    if (st == RFX_OK && evals) std::copy(ev, ev + 3, evals);
    return st;
}

rfx_status rfx_lowrank(rfx_ctx* ctx, const rfx_lowrank_opts* o, float* A, float* evals) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    rfx_status st = need_forest(c);
    if (st) return st;
    if (!o) return RFX_ERR_INVALID;
    const int k = o->rank;
    if (k < 1 || o->oversample < 0 || o->power_iters < 0 || o->power_iters > 8 || o->precision < 0 ||
        o->precision > 3) {
        set_error("rfx_lowrank: invalid options");
        return RFX_ERR_INVALID;
    }
    dfree(c, c->d_lrA);
    dfree(c, c->d_lrAq);
    dfree(c, c->d_lrScale);
    if (c->d_lrQ) cudaFree(c->d_lrQ);
    c->d_lrQ = nullptr;
    c->lr_rank = 0;
    c->lr_qformat = 0;
    if ((st = dalloc(c, &c->d_lrA, (size_t)c->n * k))) return st;
    std::vector<float> ev(k);
    st = lowrank_compute(c, k, o->oversample, o->power_iters, o->precision, o->seed ? o->seed : 12345ull, c->d_lrA,
                         ev.data(), nullptr, std::max(0, o->trees_per_pass));
    if (st) return st;
    c->lr_rank = k;
    if (evals) std::copy(ev.begin(), ev.end(), evals);
    if (A) {
        if ((st = copy_out(c, A, c->d_lrA, sizeof(float) * (size_t)c->n * k))) return st;
        RFX_CUDA(cudaStreamSynchronize(c->stream));
    }
    return check_device_errors(c);
}

rfx_status rfx_lowrank_operator(rfx_ctx* ctx, int w, int precision, const float* V, float* MV) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    rfx_status st = need_forest(c);
    if (st) return st;
    if (!V || !MV) {
        set_error("rfx_lowrank_operator: null argument");
        return RFX_ERR_INVALID;
    }
    if (w < 8 || w > 120 || w % 8 != 0 || w > c->n || (precision != 0 && precision != 1 && precision != 3)) {
        set_error("rfx_lowrank_operator: w must be a multiple of 8 in 8..min(120, n) and precision 0, 1 or 3");
        return RFX_ERR_INVALID;
    }
    const size_t bytes = sizeof(float) * (size_t)c->n * w;
    const float* dV = V;
    float* sV = nullptr;
    float* dMV = MV;
    float* sMV = nullptr;
    if (!is_device_ptr(V)) {
        cudaError_t e = ctx_malloc(c, (void**)&sV, bytes);
        if (e != cudaSuccess) return cuda_fail(e, "rfx_lowrank_operator staging");
        e = cudaMemcpyAsync(sV, V, bytes, cudaMemcpyHostToDevice, c->stream);
        if (e != cudaSuccess) {
            cudaFree(sV);
            return cuda_fail(e, "rfx_lowrank_operator H2D");
        }
        dV = sV;
    }
    const bool mdev = is_device_ptr(MV);
    if (!mdev) {
        cudaError_t e = ctx_malloc(c, (void**)&sMV, bytes);
        if (e != cudaSuccess) {
            if (sV) cudaFree(sV);
            return cuda_fail(e, "rfx_lowrank_operator staging");
        }
        dMV = sMV;
    }
    st = lowrank_compute(c, w, 0, 0, precision, 1ull, dMV, nullptr, dV);
    if (st == RFX_OK && !mdev) st = copy_out(c, MV, dMV, bytes);
    cudaStreamSynchronize(c->stream);
    if (sV) cudaFree(sV);
    if (sMV) cudaFree(sMV);
    if (st) return st;
    return check_device_errors(c);
}

rfx_status rfx_lowrank_quantize(rfx_ctx* ctx, int format, void* q, float* scales) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    rfx_status st = need_forest(c);
    if (st) return st;
    if (!c->lr_rank) {
        set_error("rfx_lowrank_quantize: no factors (call rfx_lowrank first)");
        return RFX_ERR_STATE;
    }
    if (format < 1 || format > 4) {
        set_error("rfx_lowrank_quantize: format must be 1 (INT8), 2 (FP8 e4m3), 3 (NF4) or 4 (FP16)");
        return RFX_ERR_INVALID;
    }
    const int k = c->lr_rank;
    const size_t nk = (size_t)c->n * k;
    // stored bytes: INT8 / FP8 one per entry, NF4 half, FP16 two
    const size_t qbytes = format == 3 ? (nk + 1) / 2 : format == 4 ? 2 * nk : nk;
    if (c->d_lrQ) cudaFree(c->d_lrQ);
    c->d_lrQ = nullptr;
    if (ctx_malloc(c, (void**)&c->d_lrQ, qbytes) != cudaSuccess) {
        cudaGetLastError();
        set_error("rfx_lowrank_quantize: allocation failed");
        return RFX_ERR_OOM;
    }
    if ((st = dalloc(c, &c->d_lrScale, k))) return st;
    if ((st = dalloc(c, &c->d_lrAq, nk))) return st;
    if ((st = lowrank_quantize(c, c->d_lrA, k, format, c->d_lrQ, c->d_lrScale))) return st;
    if ((st = lowrank_dequantize(c, c->d_lrQ, c->d_lrScale, k, format, c->d_lrAq))) return st;
    c->lr_qformat = format;
    if (q && (st = copy_out(c, q, c->d_lrQ, qbytes))) return st;
    if (scales && (st = copy_out(c, scales, c->d_lrScale, sizeof(float) * k))) return st;
    RFX_CUDA(cudaStreamSynchronize(c->stream));
    return RFX_OK;
}

static const float* factors_for(Ctx* c, int use_quantized) {
    if (use_quantized) return c->lr_qformat ? c->d_lrAq : nullptr;
    return c->d_lrA;
}

rfx_status rfx_mds_from_factors(rfx_ctx* ctx, int k, int use_quantized, int precision, double* coords,
                                double* evals) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    rfx_status st = need_forest(c);
    if (st) return st;
    const float* dA = c->lr_rank ? factors_for(c, use_quantized) : nullptr;
    if (!dA) {
        set_error("Low-rank factors not available (call rfx_lowrank, and rfx_lowrank_quantize for quantized factors)");
        return RFX_ERR_STATE;
    }
    if (!coords || k < 1) return RFX_ERR_INVALID;
    const bool cdev = is_device_ptr(coords);
    double* dC = coords;
    Scratch staging(c);
    if (!cdev) {
        dC = staging.get<double>((size_t)c->n * k);
        if (!dC) {
            set_error("rfx_mds_from_factors: staging allocation failed");
            return RFX_ERR_OOM;
        }
    }
    std::vector<double> ev(8, 0.0);
    int iters = 0;
    c->last_mds_tc_iters = c->last_mds_f32_iters = 0;
    st = launch_mds_factors(c, dA, c->lr_rank, k, 600, 1e-10, dC, ev.data(), &iters, precision);
    if (precision == 0) c->last_mds_f32_iters = iters;
    if (st == RFX_OK && !cdev) st = copy_out(c, coords, dC, sizeof(double) * (size_t)c->n * k);
    if (st == RFX_OK) st = finish_host(c, true);
    cudaStreamSynchronize(c->stream);
    if (st == RFX_OK && evals) std::copy(ev.begin(), ev.begin() + k, evals);
    return st;
}

rfx_status rfx_factor_mds_operator(rfx_ctx* ctx, int use_quantized, int precision, const double* V, double* W) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    rfx_status st = need_forest(c);
    if (st) return st;
    const float* dA = c->lr_rank ? factors_for(c, use_quantized) : nullptr;
    if (!dA || !V || !W) {
        set_error("rfx_factor_mds_operator: factors not available or null block");
        return RFX_ERR_STATE;
    }
    const size_t cnt = (size_t)c->n * 16;
    double *dV = nullptr, *dW = nullptr;
    RFX_CUDA(ctx_malloc(c, (void**)&dV, sizeof(double) * cnt));
    cudaError_t e = ctx_malloc(c, (void**)&dW, sizeof(double) * cnt);
    if (e != cudaSuccess) {
        cudaFree(dV);
        return cuda_fail(e, "rfx_factor_mds_operator");
    }
    e = cudaMemcpy(dV, V, sizeof(double) * cnt, cudaMemcpyDefault);
    st = e == cudaSuccess ? launch_factor_operator(c, dA, c->lr_rank, dV, dW, precision) : cuda_fail(e, "copy");
    if (st == RFX_OK) {
        e = cudaMemcpy(W, dW, sizeof(double) * cnt, cudaMemcpyDefault);
        if (e != cudaSuccess) st = cuda_fail(e, "copy");
    }
    cudaFree(dV);
    cudaFree(dW);
    if (st == RFX_OK) st = check_device_errors(c);
    return st;
}

rfx_status rfx_outlier_scores(rfx_ctx* ctx, int use_quantized, float* scores) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    rfx_status st = need_forest(c);
    if (st) return st;
    const float* dA = c->lr_rank ? factors_for(c, use_quantized) : nullptr;
    if (!dA || !scores) {
        set_error("rfx_outlier_scores: factors not available");
        return RFX_ERR_STATE;
    }
    float* d = nullptr;
    cudaError_t e = ctx_malloc(c, (void**)&d, sizeof(float) * c->n);
    if (e != cudaSuccess) return cuda_fail(e, "rfx_outlier_scores");
    st = launch_outlier_scores(c, dA, c->lr_rank, d);
    std::vector<float> h(c->n);
    if (st == RFX_OK) {
        e = cudaMemcpy(h.data(), d, sizeof(float) * c->n, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) st = cuda_fail(e, "rfx_outlier_scores D2H");
    }
    cudaFree(d);
    if (st) return st;
    // normalise by the median element sorted[n/2], as compute_outlier_scores does
    std::vector<float> srt = h;
    std::nth_element(srt.begin(), srt.begin() + c->n / 2, srt.end());
    const float med = srt[c->n / 2];
    if (med > 0)
        for (auto& x : h) x /= med;
    if (is_device_ptr(scores)) {
        RFX_CUDA(cudaMemcpy(scores, h.data(), sizeof(float) * c->n, cudaMemcpyHostToDevice));
    } else {
        std::copy(h.begin(), h.end(), scores);
    }
    return RFX_OK;
}

rfx_status rfx_profile_enable(rfx_ctx* ctx, int enable) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c) return RFX_ERR_INVALID;
    cudaSetDevice(c->device);
    RFX_CUDA(cudaStreamSynchronize(c->stream));
    if (enable && c->ev_start[0].empty()) {
        for (int s = 0; s < ST_COUNT; ++s) {
            c->ev_start[s].resize(Ctx::EV_RING);
            c->ev_end[s].resize(Ctx::EV_RING);
            for (int k = 0; k < Ctx::EV_RING; ++k) {
                RFX_CUDA(cudaEventCreate(&c->ev_start[s][k]));
                RFX_CUDA(cudaEventCreate(&c->ev_end[s][k]));
            }
        }
    }
    for (int s = 0; s < ST_COUNT; ++s) c->ev_count[s] = 0;
    c->profile = enable != 0;
    return RFX_OK;
}

rfx_status rfx_profile_read(rfx_ctx* ctx, float* stage_ms, int64_t* kernel_launches) {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c) return RFX_ERR_INVALID;
    cudaSetDevice(c->device);
    RFX_CUDA(cudaStreamSynchronize(c->stream));
    if (stage_ms) {
        for (int s = 0; s < ST_COUNT; ++s) {
            stage_ms[s] = -1.0f;
            const long long cnt = std::min<long long>(c->ev_count[s], Ctx::EV_RING);
            if (cnt <= 0 || c->ev_start[s].empty()) continue;
            double sum = 0.0;
            int good = 0;
            for (int k = 0; k < cnt; ++k) {
                float ms = 0.0f;
                if (cudaEventElapsedTime(&ms, c->ev_start[s][k], c->ev_end[s][k]) == cudaSuccess) {
                    sum += ms;
                    ++good;
                } else {
                    cudaGetLastError();
                }
            }
            if (good) stage_ms[s] = (float)(sum / good);
        }
    }
    if (kernel_launches) *kernel_launches = c->launches;
    return RFX_OK;
}

rfx_status rfx_grow_forest(const float* X, const int32_t* y, int32_t n, int32_t p, int32_t nclass, int32_t ntree,
                           int32_t mtry, int32_t minndsize, int32_t maxnode, int32_t iseed, int32_t n_threads,
                           rfx_grown_forest* out) {
    if (!X || !y || !out || n < 1 || p < 1 || nclass < 1 || ntree < 1 || mtry < 1 || minndsize < 1) {
        set_error("rfx_grow_forest: invalid argument");
        return RFX_ERR_INVALID;
    }
    try {
        std::memset(out, 0, sizeof(*out));
        std::vector<int64_t> offs;
        std::vector<int32_t> ns, bv, tm, nc;
        std::vector<float> xs;
        int32_t* nin = (int32_t*)std::malloc(sizeof(int32_t) * (size_t)ntree * n);
        if (!nin) return RFX_ERR_OOM;
        const int mx = maxnode > 0 ? maxnode : 2 * n + 1;
        rfxhost::grow_forest(X, y, n, p, nclass, ntree, mtry, minndsize, mx, iseed, n_threads, offs, ns, bv, xs, tm,
                             nc, nin);
        auto dup = [](const auto& vec) {
            using T = typename std::decay_t<decltype(vec)>::value_type;
            T* d = (T*)std::malloc(sizeof(T) * std::max<size_t>(1, vec.size()));
            if (d) std::copy(vec.begin(), vec.end(), d);
            return d;
        };
        out->ntree = ntree;
        out->offs = dup(offs);
        out->nodestatus = dup(ns);
        out->bestvar = dup(bv);
        out->xbestsplit = dup(xs);
        out->treemap = dup(tm);
        out->nodeclass = dup(nc);
        out->nin = nin;
        if (!out->offs || !out->nodestatus || !out->bestvar || !out->xbestsplit || !out->treemap || !out->nodeclass) {
            rfx_free_forest(out);
            return RFX_ERR_OOM;
        }
        return RFX_OK;
    } catch (const std::bad_alloc&) {
        set_error("rfx_grow_forest: host allocation failed");
        return RFX_ERR_OOM;
    }
}

rfx_status rfx_free_forest(rfx_grown_forest* f) {
    if (!f) return RFX_OK;
    std::free(f->offs);
    std::free(f->nodestatus);
    std::free(f->bestvar);
    std::free(f->xbestsplit);
    std::free(f->treemap);
    std::free(f->nodeclass);
    std::free(f->nin);
    std::memset(f, 0, sizeof(*f));
    return RFX_OK;
}

}  // extern "C"
