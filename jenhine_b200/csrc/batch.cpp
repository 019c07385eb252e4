// batch.cpp -- several scans through one pipeline, on one of two schedules:
// persistent (every scan's filter stage, then persistent backprojection
// launches over the tiles of all scans -- bp_batch_kernel, one launch per run
// of up to 16 consecutive scans that share W's z-dependence, each scan with
// its own tile depth) or pipelined (each scan's own backprojection, the next
// scan's filter stage beside it on a second stream); optionally recorded
// once as a CUDA graph and replayed.
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
    struct Group {                      // one persistent launch
        BatchSlots slots;
        int n, wz, wv, deep, ctas;      // wv: every scan divides by its weight volume; deep: 16-slice tiles
        unsigned total;
    };
    std::vector<Group> groups;
    unsigned* d_counter = nullptr;      // one work cursor per group
    int schedule = 0;                   // JFDK_BATCH_PERSISTENT / _PIPELINED, 0 not chosen
    cudaStream_t aux = nullptr;         // the pipelined schedule's filter stream
    // the persistent schedule's filter stages run on the batch stream and
    // these, scans dealt round-robin, joined before the persistent launch
    std::vector<cudaStream_t> filt;
    std::vector<cudaEvent_t> filt_ev;   // [fork, join] per stream of filt
    std::vector<cudaEvent_t> ev;        // [scans] filtered, fork, join, two timing events
    std::vector<float*> hu;             // the outputs of the run being enqueued
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
// its grid of kBPTileX x kBPTileY x ZPT tiles and its first tile in its group's
// work list.  Scans with the same W(z), weight-volume use and tile-depth
// class (16 slices, the mixed form's default on large volumes, or 4 / 8)
// share a group of up to kBatchSlots, in scan order, whatever lies between
// them: a batch whose scans were tuned to 16 and to 8 slices is two launches,
// not one per change of depth (8 launches for the 16-scan workload, whose
// mixed-form persistent schedule then ran 2.7 % behind the pipelined one).
jfdk_status plan_groups(jfdk_batch* b, float* const* d_hu) {
    b->groups.clear();
    for (size_t i = 0; i < b->ctx.size(); ++i) {
        jfdk_ctx* c = b->ctx[i];
        BatchScan s;
        std::memset(&s, 0, sizeof s);
        s.p = reconstruct_bp_params(c, d_hu[i], nullptr);
        const int zpt = bp_slices_per_thread(c);
        s.zpt = zpt == 4 ? 4 : (zpt == 16 && b->mixed) ? 16 : 8;
        s.wz = c->w_depends_on_z ? 1 : 0;
        s.gx = (c->X + kBPTileX - 1) / kBPTileX;
        s.gy = (c->Y + kBPTileY - 1) / kBPTileY;
        s.gz = (c->Z + s.zpt - 1) / s.zpt;
        // the weights of the tile depth the launch runs (the mixed form's
        // coordinates, and with them its weights, follow the depth)
        const float* wvol = bp_slices_per_thread(c) == s.zpt ? bp_weight_volume(c) : nullptr;
        s.p.wvol = wvol;
        const int wv = wvol ? 1 : 0, deep = s.zpt == 16 ? 1 : 0;
        size_t gi = b->groups.size();
        for (size_t k = 0; k < b->groups.size(); ++k) {
            const jfdk_batch::Group& o = b->groups[k];
            if (o.n < kBatchSlots && o.wz == s.wz && o.wv == wv && o.deep == deep) gi = k;
        }
        if (gi == b->groups.size()) {
            jfdk_batch::Group g;
            std::memset(&g, 0, sizeof g);
            g.wz = s.wz;
            g.wv = wv;
            g.deep = deep;
            BATCH_CUDA(b, bp_batch_ctas(b->mixed != 0, g.wz != 0, g.wv != 0, g.deep != 0, &g.ctas),
                       "occupancy query");
            b->groups.push_back(g);
        }
        jfdk_batch::Group& g = b->groups[gi];
        s.first_tile = g.total;
        g.total += (unsigned)s.gx * s.gy * s.gz;
        g.slots.s[g.n++] = s;
    }
    return JFDK_OK;
}

// Persistent: every scan's filter stage -- dealt round-robin over the batch
// stream and kFilterStreams - 1 more, so the stages of small scans, which
// leave most of the GPU idle, run side by side -- then the persistent BP
// launches once all have joined.
constexpr int kFilterStreams = 4;

jfdk_status enqueue_persistent(jfdk_batch* b, const uint16_t* const* d_raw) {
    const size_t ns = b->filt.size() + 1;
    for (size_t j = 0; j + 1 < ns; ++j) {
        BATCH_CUDA(b, cudaEventRecord(b->filt_ev[2 * j], b->stream), "event");
        BATCH_CUDA(b, cudaStreamWaitEvent(b->filt[j], b->filt_ev[2 * j], 0), "event");
    }
    for (size_t i = 0; i < b->ctx.size(); ++i) {
        jfdk_ctx* c = b->ctx[i];
        cudaStream_t saved = c->stream;
        c->stream = i % ns == 0 ? b->stream : b->filt[i % ns - 1];
        jfdk_status st = reconstruct_filter_stage(c, d_raw[i], c->nviews);
        c->stream = saved;
        if (st) return berr(b, st, std::string("scan ") + std::to_string(i) + ": " + c->err);
    }
    for (size_t j = 0; j + 1 < ns; ++j) {
        BATCH_CUDA(b, cudaEventRecord(b->filt_ev[2 * j + 1], b->filt[j]), "event");
        BATCH_CUDA(b, cudaStreamWaitEvent(b->stream, b->filt_ev[2 * j + 1], 0), "event");
    }
    for (size_t k = 0; k < b->groups.size(); ++k) {
        const jfdk_batch::Group& g = b->groups[k];
        BATCH_CUDA(b, launch_bp_batch(g.slots, g.n, g.total, b->mixed != 0, g.wz != 0, g.wv != 0, b->d_counter + k, g.ctas,
                                      b->stream),
                   "batched backprojection");
        ++b->launches;
    }
    return JFDK_OK;
}

// Pipelined: the filter stages in order on the second stream, each scan's
// backprojection on the batch stream once its own filter stage is done.
jfdk_status enqueue_pipelined(jfdk_batch* b, const uint16_t* const* d_raw) {
    const size_t n = b->ctx.size();
    cudaEvent_t fork = b->ev[n], join = b->ev[n + 1];
    BATCH_CUDA(b, cudaEventRecord(fork, b->stream), "event");
    BATCH_CUDA(b, cudaStreamWaitEvent(b->aux, fork, 0), "event");
    for (size_t i = 0; i < n; ++i) {
        jfdk_ctx* c = b->ctx[i];
        cudaStream_t saved = c->stream;
        c->stream = b->aux;
        jfdk_status st = reconstruct_filter_stage(c, d_raw[i], c->nviews);
        c->stream = saved;
        if (st) return berr(b, st, std::string("scan ") + std::to_string(i) + ": " + c->err);
        BATCH_CUDA(b, cudaEventRecord(b->ev[i], b->aux), "event");
        BATCH_CUDA(b, cudaStreamWaitEvent(b->stream, b->ev[i], 0), "event");
        if ((st = reconstruct_bp(c, b->hu[i], b->stream)))
            return berr(b, st, std::string("scan ") + std::to_string(i) + ": " + c->err);
    }
    BATCH_CUDA(b, cudaEventRecord(join, b->aux), "event");
    BATCH_CUDA(b, cudaStreamWaitEvent(b->stream, join, 0), "event");
    return JFDK_OK;
}

jfdk_status enqueue(jfdk_batch* b, const uint16_t* const* d_raw) {
    return b->schedule == JFDK_BATCH_PIPELINED ? enqueue_pipelined(b, d_raw) : enqueue_persistent(b, d_raw);
}

// The first run: with JFDK_BATCH_AUTOTUNE and no schedule fixed, both
// schedules run (the outputs are the same) and the faster is kept.
jfdk_status first_run(jfdk_batch* b, const uint16_t* const* d_raw) {
    if (b->schedule) return enqueue(b, d_raw);
    if (!(b->flags & JFDK_BATCH_AUTOTUNE)) {
        b->schedule = JFDK_BATCH_PERSISTENT;
        return enqueue(b, d_raw);
    }
    const size_t n = b->ctx.size();
    cudaEvent_t t0 = b->ev[n + 2], t1 = b->ev[n + 3];
    float ms[2] = {0.0f, 0.0f};
    const int order[2] = {JFDK_BATCH_PERSISTENT, JFDK_BATCH_PIPELINED};
    for (int k = 0; k < 2; ++k) {
        b->schedule = order[k];
        jfdk_status st = enqueue(b, d_raw);   // the first pass also allocates what the contexts still need
        if (st) return st;
        BATCH_CUDA(b, cudaEventRecord(t0, b->stream), "event");
        if ((st = enqueue(b, d_raw))) return st;
        BATCH_CUDA(b, cudaEventRecord(t1, b->stream), "event");
        BATCH_CUDA(b, cudaEventSynchronize(t1), "timing the schedules");
        BATCH_CUDA(b, cudaEventElapsedTime(&ms[k], t0, t1), "timing the schedules");
    }
    b->schedule = ms[0] <= ms[1] ? JFDK_BATCH_PERSISTENT : JFDK_BATCH_PIPELINED;
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
    BATCH_CUDA(b, cudaMalloc(&b->d_counter, sizeof(unsigned) * n), "CUDA failed to malloc the work counters");
    if ((flags & JFDK_BATCH_PERSISTENT) && (flags & JFDK_BATCH_PIPELINED))
        return berr(b, JFDK_ERR_INVALID, "one schedule at most");
    b->schedule = (flags & JFDK_BATCH_PIPELINED) ? JFDK_BATCH_PIPELINED
                  : (flags & JFDK_BATCH_PERSISTENT) ? JFDK_BATCH_PERSISTENT : 0;
    BATCH_CUDA(b, cudaStreamCreateWithFlags(&b->aux, cudaStreamNonBlocking), "creating the filter stream");
    const int extra = std::min(kFilterStreams, n) - 1;
    for (int j = 0; j < extra; ++j) {
        cudaStream_t st = nullptr;
        BATCH_CUDA(b, cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "creating a filter stream");
        b->filt.push_back(st);
        for (int k = 0; k < 2; ++k) {
            cudaEvent_t e = nullptr;
            BATCH_CUDA(b, cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "creating an event");
            b->filt_ev.push_back(e);
        }
    }
    b->ev.assign((size_t)n + 4, nullptr);
    for (auto& e : b->ev) BATCH_CUDA(b, cudaEventCreate(&e), "creating an event");
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
    if (b->aux) cudaStreamSynchronize(b->aux);
    for (cudaStream_t st : b->filt) cudaStreamSynchronize(st);
    if (b->d_counter) cudaFree(b->d_counter);
    for (cudaEvent_t e : b->ev)
        if (e) cudaEventDestroy(e);
    if (b->aux) cudaStreamDestroy(b->aux);
    for (cudaStream_t st : b->filt) cudaStreamDestroy(st);
    for (cudaEvent_t e : b->filt_ev) cudaEventDestroy(e);
    if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

const char* jfdk_batch_last_error(const jfdk_batch* b) { return b ? b->err.c_str() : "null batch"; }

long long jfdk_batch_launches(const jfdk_batch* b) { return b ? b->launches : 0; }

int jfdk_batch_schedule(const jfdk_batch* b) { return b ? b->schedule : 0; }

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
    // the stores first: the persistent launches' parameters name them, and a
    // context that has not reconstructed yet (or whose shape the autotuner
    // answered from its cache) would otherwise get its store from the filter
    // stage after those parameters were taken
    jfdk_status st = JFDK_OK;
    for (size_t i = 0; i < n; ++i)
        if ((st = ensure_store(b->ctx[i])))
            return berr(b, st, std::string("scan ") + std::to_string(i) + ": " + b->ctx[i]->err);
    if ((st = plan_groups(b, d_hu))) return st;
    b->hu.assign(d_hu, d_hu + n);
    // run directly (allocates whatever the contexts still need; picks the
    // schedule on the first run)
    if ((st = first_run(b, d_raw))) return st;
    if (!(b->flags & JFDK_BATCH_GRAPH)) return JFDK_OK;
    // record the same work as a graph for the next runs with these buffers
    BATCH_CUDA(b, cudaStreamSynchronize(b->stream), "batch run");
    std::vector<long long> counted(n);
    for (size_t i = 0; i < n; ++i) counted[i] = b->ctx[i]->launches;
    const long long own = b->launches;
    BATCH_CUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "graph capture");
    st = enqueue(b, d_raw);
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
