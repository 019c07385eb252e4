// batch.cpp -- several scans through one pipeline: every scan's filter stage,
// then one persistent backprojection launch over the tiles of all scans
// (bp_batch_kernel), optionally recorded once as a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "jfdk_internal.h"

using namespace jfdk;

struct jfdk_batch {
    std::vector<jfdk_ctx*> ctx;
    int flags = 0;
    int mixed = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    BatchScan* d_scans = nullptr;
    unsigned* d_counter = nullptr;
    int ctas = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<const uint16_t*> raw;   // the buffers the graph was recorded with
    std::vector<float*> out;
    long long launches = 0;
    long long graph_kernels = 0;        // kernels one replay of the graph runs
    std::string err;
};

namespace {

jfdk_status berr(jfdk_batch* b, jfdk_status st, const std::string& m) {
    b->err = m;
    return st;
}

#define BATCH_CUDA(b, call, what)                                                                 \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return berr(b, e_ == cudaErrorMemoryAllocation ? JFDK_ERR_OOM : JFDK_ERR_CUDA,         \
                        std::string(what) + ": " + cudaGetErrorString(e_));                        \
    } while (0)

void drop_graph(jfdk_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

// Scan descriptors for the given outputs: each scan's finalizing BP params,
// its grid of 32 x 8 x ZPT tiles and its first tile in the work list.
jfdk_status upload_scans(jfdk_batch* b, float* const* d_hu, unsigned* total) {
    std::vector<BatchScan> h(b->ctx.size());
    unsigned first = 0;
    for (size_t i = 0; i < b->ctx.size(); ++i) {
        jfdk_ctx* c = b->ctx[i];
        BatchScan& s = h[i];
        std::memset(&s, 0, sizeof s);
        s.p = reconstruct_bp_params(c, d_hu[i], nullptr);
        s.zpt = bp_slices_per_thread(c) == 4 ? 4 : 8;
        s.wz = c->w_depends_on_z ? 1 : 0;
        s.gx = (c->X + 31) / 32;
        s.gy = (c->Y + kBPTileY - 1) / kBPTileY;
        s.gz = (c->Z + s.zpt - 1) / s.zpt;
        s.first_tile = first;
        first += (unsigned)s.gx * s.gy * s.gz;
    }
    BATCH_CUDA(b, cudaMemcpy(b->d_scans, h.data(), sizeof(BatchScan) * h.size(), cudaMemcpyHostToDevice),
               "uploading the scan table");
    *total = first;
    return JFDK_OK;
}

// Every scan's filter stage on the batch stream, then the persistent BP.
jfdk_status enqueue(jfdk_batch* b, const uint16_t* const* d_raw, unsigned total) {
    for (size_t i = 0; i < b->ctx.size(); ++i) {
        jfdk_ctx* c = b->ctx[i];
        cudaStream_t saved = c->stream;
        c->stream = b->stream;
        jfdk_status st = reconstruct_filter_stage(c, d_raw[i], c->nviews);
        c->stream = saved;
        if (st) return berr(b, st, std::string("scan ") + std::to_string(i) + ": " + c->err);
    }
    BATCH_CUDA(b, launch_bp_batch(b->d_scans, (int)b->ctx.size(), total, b->mixed != 0, b->d_counter, b->ctas,
                                  b->stream),
               "batched backprojection");
    ++b->launches;
    return JFDK_OK;
}

}  // namespace

extern "C" {

jfdk_status jfdk_batch_create(jfdk_batch** out, jfdk_ctx* const* ctxs, int n, int flags, void* cuda_stream) {
    if (!out || !ctxs || n < 1) return JFDK_ERR_INVALID;
    *out = nullptr;
    jfdk_batch* b = new (std::nothrow) jfdk_batch();
    if (!b) return JFDK_ERR_OOM;
    *out = b;   // the caller reads the message, then destroys
    b->flags = flags;
    for (int i = 0; i < n; ++i) {
        if (!ctxs[i]) return berr(b, JFDK_ERR_INVALID, "null context");
        b->ctx.push_back(ctxs[i]);
    }
    b->mixed = mixed_form(ctxs[0]) ? 1 : 0;
    for (jfdk_ctx* c : b->ctx)
        if ((mixed_form(c) ? 1 : 0) != b->mixed) return berr(b, JFDK_ERR_INVALID, "all scans of a batch use one form");
    if (cuda_stream) {
        b->stream = static_cast<cudaStream_t>(cuda_stream);
    } else {
        BATCH_CUDA(b, cudaStreamCreate(&b->stream), "creating the batch stream");   // ordered after the legacy stream
        b->own_stream = true;
    }
    BATCH_CUDA(b, cudaMalloc(&b->d_scans, sizeof(BatchScan) * n), "CUDA failed to malloc the scan table");
    BATCH_CUDA(b, cudaMalloc(&b->d_counter, sizeof(unsigned)), "CUDA failed to malloc the work counter");
    BATCH_CUDA(b, bp_batch_ctas(b->mixed != 0, &b->ctas), "occupancy query");
    if (flags & JFDK_BATCH_AUTOTUNE)
        for (jfdk_ctx* c : b->ctx) {
            cudaStream_t saved = c->stream;
            c->stream = b->stream;
            jfdk_status st = jfdk_autotune(c, 0);
            c->stream = saved;
            if (st) return berr(b, st, std::string("autotune: ") + c->err);
        }
    return JFDK_OK;
}

void jfdk_batch_destroy(jfdk_batch* b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graph(b);
    if (b->d_scans) cudaFree(b->d_scans);
    if (b->d_counter) cudaFree(b->d_counter);
    if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

const char* jfdk_batch_last_error(const jfdk_batch* b) { return b ? b->err.c_str() : "null batch"; }

long long jfdk_batch_launches(const jfdk_batch* b) { return b ? b->launches : 0; }

jfdk_status jfdk_batch_run(jfdk_batch* b, const uint16_t* const* d_raw, float* const* d_hu) {
    if (!b || !d_raw || !d_hu) return JFDK_ERR_INVALID;
    const size_t n = b->ctx.size();
    for (size_t i = 0; i < n; ++i)
        if (!d_raw[i] || !d_hu[i]) return berr(b, JFDK_ERR_INVALID, "batch_run: null buffer");
    const bool same = b->exec && std::equal(d_raw, d_raw + n, b->raw.begin()) &&
                      std::equal(d_hu, d_hu + n, b->out.begin());
    if (same) {
        BATCH_CUDA(b, cudaGraphLaunch(b->exec, b->stream), "graph launch");
        b->launches += b->graph_kernels;
        return JFDK_OK;
    }
    drop_graph(b);
    unsigned total = 0;
    jfdk_status st = upload_scans(b, d_hu, &total);
    if (st) return st;
    // run directly (allocates whatever the contexts still need)
    if ((st = enqueue(b, d_raw, total))) return st;
    if (!(b->flags & JFDK_BATCH_GRAPH)) return JFDK_OK;
    // record the same work as a graph for the next runs with these buffers
    BATCH_CUDA(b, cudaStreamSynchronize(b->stream), "batch run");
    std::vector<long long> counted(n);
    for (size_t i = 0; i < n; ++i) counted[i] = b->ctx[i]->launches;
    const long long own = b->launches;
    BATCH_CUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "graph capture");
    st = enqueue(b, d_raw, total);
    cudaGraph_t g = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(b->stream, &g);
    for (size_t i = 0; i < n; ++i) b->ctx[i]->launches = counted[i];   // recorded, not run
    b->launches = own;
    if (st) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (ec != cudaSuccess) return berr(b, JFDK_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ec));
    b->graph = g;
    BATCH_CUDA(b, cudaGraphInstantiate(&b->exec, b->graph, 0), "graph instantiate");
    size_t nodes = 0;
    BATCH_CUDA(b, cudaGraphGetNodes(b->graph, nullptr, &nodes), "graph nodes");
    std::vector<cudaGraphNode_t> list(nodes);
    BATCH_CUDA(b, cudaGraphGetNodes(b->graph, list.data(), &nodes), "graph nodes");
    b->graph_kernels = 0;
    for (cudaGraphNode_t nd : list) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++b->graph_kernels;
    }
    b->raw.assign(d_raw, d_raw + n);
    b->out.assign(d_hu, d_hu + n);
    return JFDK_OK;
}

}  // extern "C"
