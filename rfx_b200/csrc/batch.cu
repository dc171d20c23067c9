// Many independent forests in one CUDA graph.
//
// Each forest is a loaded context with its own stream.  Capture runs every
// context's analysis once eagerly (so every lazily allocated buffer exists and
// is validated), then records all of them again into one graph: a capture
// stream forks into the contexts' streams and joins them back, so the graph's
// per-forest chains run side by side on the GPU.  A replay is one
// cudaGraphLaunch for the whole batch.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "rfx_internal.cuh"

namespace rfx {
namespace {

bool dev_or_null(const void* p) { return !p || is_device_ptr(p); }

// One forest's analysis, enqueued on its context's stream with device outputs.
rfx_status enqueue_item(Ctx* c, const rfx_batch_item& it) {
    rfx_status st = launch_route(c);
    if (st != RFX_OK) return st;
    c->routed = true;
    cudaStream_t s = c->stream;
    if (it.votes)
        RFX_CUDA(cudaMemcpyAsync(it.votes, c->d_votes, sizeof(int32_t) * (size_t)c->n * c->nclass,
                                 cudaMemcpyDeviceToDevice, s));
    if (it.nout) RFX_CUDA(cudaMemcpyAsync(it.nout, c->d_nout, sizeof(int32_t) * c->n, cudaMemcpyDeviceToDevice, s));
    if (it.oob_error || it.oob_pred) {
        if ((st = launch_oob_summary(c, it.oob_error, it.oob_pred, nullptr)) != RFX_OK) return st;
    }
    if (it.S) {
        if ((st = launch_build_csr(c)) != RFX_OK) return st;
        if ((st = launch_pairs_upper(c, it.S)) != RFX_OK) return st;
        c->csr_built = true;
    }
    if (it.avimp) {
        if ((st = launch_varimp(c, it.impn ? 1 : 0)) != RFX_OK) return st;
        auto cp = [&](float* dst, const float* src, size_t cnt) -> rfx_status {
            if (dst) RFX_CUDA(cudaMemcpyAsync(dst, src, sizeof(float) * cnt, cudaMemcpyDeviceToDevice, s));
            return RFX_OK;
        };
        if ((st = cp(it.avimp, c->d_avimp, c->p)) != RFX_OK) return st;
        if ((st = cp(it.sqsd, c->d_sqsd, c->p)) != RFX_OK) return st;
        if (it.impn) {
            if ((st = cp(it.qimp, c->d_qimp, c->n)) != RFX_OK) return st;
            if ((st = cp(it.qimpm, c->d_qimpm, (size_t)c->n * c->p)) != RFX_OK) return st;
        }
    }
    return RFX_OK;
}

// varimp's scratch buffers, allocated as rfx_varimp does
rfx_status varimp_buffers(Ctx* c) {
    const int T = c->T, n = c->n, p = c->p, W = varimp_flip_words(c->iv_words);
    rfx_status st = RFX_OK;
    if (st == RFX_OK) st = dalloc(c, &c->d_joob, (size_t)T * n);
    if (st == RFX_OK) st = dalloc(c, &c->d_partner, (size_t)T * n);
    if (st == RFX_OK) st = dalloc(c, &c->d_oobord, (size_t)T * n);
    if (st == RFX_OK) st = dalloc(c, &c->d_vflags, (size_t)T * n);
    if (st == RFX_OK) st = dalloc(c, &c->d_flips, (size_t)T * n * W);
    if (st == RFX_OK) st = dalloc(c, &c->d_right, 2 * (size_t)T);
    if (st == RFX_OK) st = dalloc(c, &c->d_rightimp, (size_t)T * p);
    if (st == RFX_OK) st = dalloc(c, &c->d_qimp, n);
    if (st == RFX_OK) st = dalloc(c, &c->d_qimpm, (size_t)n * p);
    if (st == RFX_OK) st = dalloc(c, &c->d_avimp, p);
    if (st == RFX_OK) st = dalloc(c, &c->d_sqsd, p);
    return st;
}

}  // namespace
}  // namespace rfx

struct rfx_graph {
    std::vector<rfx::Ctx*> ctx;
    std::vector<uint64_t> gen;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int device = 0;
    int64_t kernels = 0;
};

extern "C" {

rfx_status rfx_graph_capture_batch(const rfx_batch_item* items, int32_t count, rfx_graph** out,
                                   int64_t* kernel_nodes) {
    using namespace rfx;
    if (!items || count < 1 || !out) {
        set_error("rfx_graph_capture_batch: need items, count >= 1 and an output handle");
        return RFX_ERR_INVALID;
    }
    *out = nullptr;
    Ctx* c0 = reinterpret_cast<Ctx*>(items[0].ctx);
    if (!c0) {
        set_error("rfx_graph_capture_batch: item 0 has no context");
        return RFX_ERR_INVALID;
    }
    cudaSetDevice(c0->device);
    for (int i = 0; i < count; ++i) {
        Ctx* c = reinterpret_cast<Ctx*>(items[i].ctx);
        const rfx_batch_item& it = items[i];
        if (!c || !c->loaded) {
            set_error("rfx_graph_capture_batch: item " + std::to_string(i) + " has no loaded forest");
            return RFX_ERR_STATE;
        }
        if (c->device != c0->device) {
            set_error("rfx_graph_capture_batch: all contexts must use one device");
            return RFX_ERR_INVALID;
        }
        for (int j = 0; j < i; ++j)
            if (items[j].ctx == it.ctx) {
                set_error("rfx_graph_capture_batch: a context appears twice");
                return RFX_ERR_INVALID;
            }
        if (!dev_or_null(it.S) || !dev_or_null(it.votes) || !dev_or_null(it.nout) || !dev_or_null(it.oob_error) ||
            !dev_or_null(it.oob_pred) || !dev_or_null(it.avimp) || !dev_or_null(it.sqsd) || !dev_or_null(it.qimp) ||
            !dev_or_null(it.qimpm)) {
            set_error("rfx_graph_capture_batch: outputs of item " + std::to_string(i) + " must be device memory");
            return RFX_ERR_INVALID;
        }
        if (it.avimp && it.impn && (!it.qimp || !it.qimpm)) {
            set_error("rfx_graph_capture_batch: impn needs qimp and qimpm");
            return RFX_ERR_INVALID;
        }
    }
    // eager pass: allocates every buffer the chains use and checks the device flags
    for (int i = 0; i < count; ++i) {
        Ctx* c = reinterpret_cast<Ctx*>(items[i].ctx);
        rfx_status st = RFX_OK;
        if (items[i].avimp && (st = varimp_buffers(c)) != RFX_OK) return st;
        if ((st = enqueue_item(c, items[i])) != RFX_OK) return st;
    }
    for (int i = 0; i < count; ++i) {
        Ctx* c = reinterpret_cast<Ctx*>(items[i].ctx);
        RFX_CUDA(cudaStreamSynchronize(c->stream));
        rfx_status st = check_device_errors(c);
        if (st != RFX_OK) return st;
    }

    rfx_graph* g = new rfx_graph();
    g->device = c0->device;
    cudaStream_t cs = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> joins(count, nullptr);
    std::vector<bool> prof(count);
    rfx_status st = RFX_OK;
    cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
    for (int i = 0; i < count && e == cudaSuccess; ++i) e = cudaEventCreateWithFlags(&joins[i], cudaEventDisableTiming);
    bool capturing = false;
    if (e == cudaSuccess) {
        e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed);
        capturing = e == cudaSuccess;
    }
    if (e == cudaSuccess) e = cudaEventRecord(fork, cs);
    for (int i = 0; i < count && e == cudaSuccess && st == RFX_OK; ++i) {
        Ctx* c = reinterpret_cast<Ctx*>(items[i].ctx);
        prof[i] = c->profile;
        c->profile = false;  // no timing events inside the graph
        e = cudaStreamWaitEvent(c->stream, fork, 0);
        if (e == cudaSuccess) st = enqueue_item(c, items[i]);
        if (e == cudaSuccess && st == RFX_OK) e = cudaEventRecord(joins[i], c->stream);
        if (e == cudaSuccess && st == RFX_OK) e = cudaStreamWaitEvent(cs, joins[i], 0);
        c->profile = prof[i];
    }
    if (capturing) {
        cudaGraph_t graph = nullptr;
        const cudaError_t e2 = cudaStreamEndCapture(cs, &graph);
        if (e == cudaSuccess) e = e2;
        g->graph = graph;
    }
    if (e == cudaSuccess && st == RFX_OK) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
    if (e == cudaSuccess && st == RFX_OK) {
        size_t nn = 0;
        e = cudaGraphGetNodes(g->graph, nullptr, &nn);
        std::vector<cudaGraphNode_t> nodes(nn);
        if (e == cudaSuccess && nn) e = cudaGraphGetNodes(g->graph, nodes.data(), &nn);
        for (size_t q = 0; q < nn && e == cudaSuccess; ++q) {
            cudaGraphNodeType ty;
            e = cudaGraphNodeGetType(nodes[q], &ty);
            if (e == cudaSuccess && ty == cudaGraphNodeTypeKernel) g->kernels++;
        }
    }
    for (cudaEvent_t j : joins)
        if (j) cudaEventDestroy(j);
    if (fork) cudaEventDestroy(fork);
    if (cs) cudaStreamDestroy(cs);
    if (e != cudaSuccess || st != RFX_OK) {
        rfx_graph_destroy(g);
        if (st != RFX_OK) return st;
        return cuda_fail(e, "rfx_graph_capture_batch");
    }
    for (int i = 0; i < count; ++i) {
        Ctx* c = reinterpret_cast<Ctx*>(items[i].ctx);
        g->ctx.push_back(c);
        g->gen.push_back(c->generation);
    }
    if (kernel_nodes) *kernel_nodes = g->kernels;
    *out = g;
    return RFX_OK;
}

rfx_status rfx_graph_launch(rfx_graph* g, void* stream) {
    using namespace rfx;
    if (!g || !g->exec) {
        set_error("rfx_graph_launch: no graph");
        return RFX_ERR_INVALID;
    }
    for (size_t i = 0; i < g->ctx.size(); ++i)
        if (g->ctx[i]->generation != g->gen[i] || !g->ctx[i]->loaded) {
            set_error("rfx_graph_launch: context " + std::to_string(i) +
                      " was reloaded or released after capture; capture the batch again");
            return RFX_ERR_STATE;
        }
    cudaSetDevice(g->device);
    RFX_CUDA(cudaGraphLaunch(g->exec, (cudaStream_t)stream));
    return RFX_OK;
}

rfx_status rfx_graph_destroy(rfx_graph* g) {
    if (!g) return RFX_OK;
    cudaSetDevice(g->device);
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return RFX_OK;
}

}  // extern "C"
