// noalloc.cu -- the ramp-filter stage without any device allocation.
//
// Who needs this: callers that must not allocate device memory while they
// run -- hosts whose framework owns every allocation through its own pool or
// budget, and real-time or interrupt-driven acquisition threads where a
// cudaMalloc (which can synchronise the device and take milliseconds) is not
// acceptable.  jfdk_filter_frames allocates its working rows on first use;
// jfdk_filter_frames_noalloc runs the pre-weight + edge-mean kernel and the
// FP32 CUDA-core ramp product (the JFDK_RAMP_FP32_SIMT path of
// jfdk_filter_frames, whatever the context's form) with that working storage
// taken from one fixed array compiled into the library.
//
// The array is a file-scope __device__ variable, so every GPU that loads
// libjfdk.so holds its 4 MiB until the process exits, and every call shares
// it: calls whose kernels overlap on the GPU (two streams, or two threads)
// race on it and must be serialised by the caller.  Each call overwrites all
// of the part it reads (the pre-weight kernel writes every row element,
// including the zero padding up to the row pitch, and every edge mean), so
// nothing needs clearing between calls.  Its device address is looked up
// once per device and kept for the life of the process; a cudaDeviceReset
// makes it stale.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <string>

#include "jfdk_internal.h"

namespace {

// Working rows (nv * rows * pitch floats) followed by the edge means
// (nv * rows floats, starting on a 256-byte boundary).
constexpr size_t kScratchFloats = size_t(1) << 20;  // 4 MiB
__device__ __align__(256) float g_filter_scratch[kScratchFloats];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
float* g_scratch_addr[kMaxDevices] = {};

// Device address of g_filter_scratch on `device`.  In host code the name of a
// __device__ array is only a host-side stand-in, not a device address: it is
// resolved once per device, with that device current, and cached.
cudaError_t scratch_address(int device, float** out) {
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[device]) {
        int prev = -1;
        cudaError_t e = cudaGetDevice(&prev);
        if (e != cudaSuccess) return e;
        if (prev != device && (e = cudaSetDevice(device)) != cudaSuccess) return e;
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_filter_scratch);
        if (prev != device) cudaSetDevice(prev);
        if (e != cudaSuccess) return e;
        g_scratch_addr[device] = static_cast<float*>(p);
    }
    *out = g_scratch_addr[device];
    return cudaSuccess;
}

}  // namespace

extern "C" jfdk_status jfdk_filter_frames_noalloc(jfdk_ctx* c, const float* d_in, int v0, int nv, float* d_out) {
    if (!c) return JFDK_ERR_INVALID;
    if (!d_in || !d_out || nv < 0 || v0 < 0) {
        c->err = "filter_frames_noalloc: bad argument";
        return JFDK_ERR_INVALID;
    }
    if (nv == 0) return JFDK_OK;
    const size_t pitch = (size_t)(c->in_w + 63) / 64 * 64;       // the row pitch of the context's ramp operator
    const size_t rows = (size_t)nv * c->rows;
    const size_t edge_off = (rows * pitch + 63) / 64 * 64;          // 256-byte aligned
    if (edge_off + rows > kScratchFloats) {
        char msg[256];
        std::snprintf(msg, sizeof msg,
                      "filter_frames_noalloc: %d views of %d rows x %zu need %zu floats, more than the static "
                      "scratch of %zu floats (4 MiB); pass fewer views per call",
                      nv, c->rows, pitch, edge_off + rows, kScratchFloats);
        c->err = msg;
        return JFDK_ERR_INVALID;
    }
    float* scratch = nullptr;
    cudaError_t e = scratch_address(c->device, &scratch);
    if (e != cudaSuccess) {
        c->err = std::string("filter_frames_noalloc: scratch address: ") + cudaGetErrorString(e);
        return JFDK_ERR_CUDA;
    }
    float* A = scratch;
    float* edge = scratch + edge_off;

    jfdk::WeightParams w{};
    w.tinv = c->d_tinv;
    w.dmin = c->d_dmin;
    w.num_views = c->nviews;
    w.L = c->L;
    w.det_right = c->mirror;
    w.mirror = c->mirror;
    w.pw = c->d_pw;
    jfdk::AOperand a{};
    a.kind = jfdk::AOUT_F32;
    a.hi = A;
    a.pitch = (int)pitch;
    e = jfdk::launch_weight(d_in, nv, v0, c->in_w, c->rows, w, a, edge, c->stream);
    if (e != cudaSuccess) {
        c->err = std::string("filter_frames_noalloc: pre-weight: ") + cudaGetErrorString(e);
        return JFDK_ERR_CUDA;
    }
    ++c->launches;

    jfdk::RampParams r{};
    r.A = A; r.e = edge; r.B = c->d_T; r.c = c->d_c;
    r.M = nv * c->rows; r.N = c->out_w; r.K = c->in_w; r.a_pitch = (int)pitch;
    r.rows = c->rows;
    r.q = d_out; r.q_frame_stride = (long long)c->rows * c->out_w; r.q_pitch = c->out_w;
    r.b_scale = 1.0f;
    e = jfdk::launch_ramp_gemm(r, c->stream);
    if (e != cudaSuccess) {
        c->err = std::string("filter_frames_noalloc: ramp filter: ") + cudaGetErrorString(e);
        return JFDK_ERR_CUDA;
    }
    ++c->launches;
    return JFDK_OK;
}
