// gather_rate.cu -- the measured ceiling of the backprojector's sample
// fetches (sm_100a).
//
// Every backprojection sample is one gather: each lane of a warp loads the
// record that holds its sample's bilinear footprint (16 bytes in the FP32
// store, 8 bytes in the FP16 store), plus, where the form keeps the taper
// apart, the 8-byte taper pair of its column.  The lanes of a warp (4 x 8
// voxels) fall on a handful of neighbouring records, so a warp-wide load
// touches few distinct records.  This kernel issues exactly those loads --
// the same widths, `distinct` consecutive records per warp request,
// read-only path through L1 -- from a table small enough to stay resident in
// every SM's L1, with almost no other instructions, so its rate is what the
// load path can deliver when nothing else limits it: the ceiling a
// backprojector's samples per second are compared with.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "jfdk_internal.h"

namespace jfdk {
namespace {

constexpr int kGatherLoads = 16;        // loads per iteration, at immediate offsets
constexpr int kGatherStride = 1024;     // bytes between them
constexpr unsigned kGatherSpan = 32768; // bytes the per-iteration base ranges over
constexpr int kGatherThreads = 128;

__device__ __forceinline__ unsigned ld16(const char* p) {
    unsigned a, b, c, d;
    asm("ld.global.nc.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(a), "=r"(b), "=r"(c), "=r"(d) : "l"(p));
    return a ^ d;
}

__device__ __forceinline__ unsigned ld8(const char* p) {
    unsigned a, b;
    asm("ld.global.nc.v2.u32 {%0, %1}, [%2];" : "=r"(a), "=r"(b) : "l"(p));
    return a ^ b;
}

// RB: record bytes (16 or 8); TAPER: also an 8-byte taper load per sample.
// Each warp's base moves pseudo-randomly over the table from iteration to
// iteration (one multiply-add), the loads of an iteration sit at fixed
// offsets from it, and lane l reads record (l mod distinct).
template <int RB, bool TAPER>
__global__ void __launch_bounds__(kGatherThreads) gather_rate_kernel(const char* __restrict__ rec,
                                                                      const char* __restrict__ taper, int iters,
                                                                      int distinct, unsigned* sink) {
    const unsigned lane = threadIdx.x & 31u;
    const unsigned slot = lane % (unsigned)distinct;
    unsigned h = (blockIdx.x * (unsigned)kGatherThreads + threadIdx.x) >> 5;
    unsigned acc = 0;
    for (int i = 0; i < iters; ++i) {
        h = h * 1664525u + 1013904223u;
        const unsigned base = (h >> 8) & (kGatherSpan - 1u) & ~63u;
        const char* p = rec + base + slot * RB;
        const char* q = taper + (base >> 1) + slot * 8u;
        unsigned r[kGatherLoads], t[kGatherLoads];
#pragma unroll
        for (int k = 0; k < kGatherLoads; ++k) {   // all loads of the iteration before any use
            r[k] = RB == 16 ? ld16(p + k * kGatherStride) : ld8(p + k * kGatherStride);
            t[k] = TAPER ? ld8(q + k * (kGatherStride / 2)) : 0u;
        }
#pragma unroll
        for (int k = 0; k < kGatherLoads; ++k) acc = (acc ^ r[k]) + t[k];
    }
    if (acc == 0x9e3779b9u) sink[0] = acc;   // keeps the loads' results live
}

template <int RB, bool TAPER>
cudaError_t launch_gather(const char* rec, const char* taper, int ctas, int iters, int distinct, unsigned* sink,
                          cudaStream_t s) {
    gather_rate_kernel<RB, TAPER><<<ctas, kGatherThreads, 0, s>>>(rec, taper, iters, distinct, sink);
    return cudaGetLastError();
}

cudaError_t launch_gather_any(int rb, bool taper, const char* rec, const char* tw, int ctas, int iters, int distinct,
                              unsigned* sink, cudaStream_t s) {
    if (rb == 16) return taper ? launch_gather<16, true>(rec, tw, ctas, iters, distinct, sink, s)
                               : launch_gather<16, false>(rec, tw, ctas, iters, distinct, sink, s);
    return taper ? launch_gather<8, true>(rec, tw, ctas, iters, distinct, sink, s)
                 : launch_gather<8, false>(rec, tw, ctas, iters, distinct, sink, s);
}

}  // namespace
}  // namespace jfdk

extern "C" jfdk_status jfdk_measure_gather_rate(int record_bytes, int with_taper, int distinct, int warps_per_sm,
                                                double* samples_per_s) {
    using namespace jfdk;
    if (!samples_per_s || (record_bytes != 16 && record_bytes != 8) || distinct < 1 || distinct > 32 ||
        warps_per_sm < 4 || warps_per_sm > 64 || warps_per_sm % 4 != 0)
        return JFDK_ERR_INVALID;
    *samples_per_s = 0.0;
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return JFDK_ERR_CUDA;
    }
    // table: the span, the loads' reach beyond it and a warp's records
    // (largest offset read: 32704 + 31 * 16 + 15 * 1024 + 16 < bytes)
    const size_t bytes = kGatherSpan + (size_t)kGatherLoads * kGatherStride + 32 * 16 + 256;
    char* rec = nullptr;
    char* tw = nullptr;
    unsigned* sink = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    jfdk_status st = JFDK_OK;
    const int ctas = sms * (warps_per_sm / (kGatherThreads / 32));
    const int iters = 2048;
    float best = 0.0f;
    if (cudaMalloc(&rec, bytes) != cudaSuccess || cudaMalloc(&tw, bytes) != cudaSuccess ||
        cudaMalloc(&sink, sizeof(unsigned)) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess || cudaEventCreate(&a) != cudaSuccess ||
        cudaEventCreate(&b) != cudaSuccess || cudaMemsetAsync(rec, 0x3c, bytes, s) != cudaSuccess ||
        cudaMemsetAsync(tw, 0x3c, bytes, s) != cudaSuccess) {
        st = JFDK_ERR_CUDA;
    }
    for (int rep = 0; st == JFDK_OK && rep < 6; ++rep) {   // the first run warms the caches and is dropped
        if (cudaEventRecord(a, s) != cudaSuccess ||
            launch_gather_any(record_bytes, with_taper != 0, rec, tw, ctas, iters, distinct, sink, s) != cudaSuccess ||
            cudaEventRecord(b, s) != cudaSuccess || cudaEventSynchronize(b) != cudaSuccess) {
            st = JFDK_ERR_CUDA;
            break;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, a, b);
        if (rep > 0 && ms > 0.0f && (best == 0.0f || ms < best)) best = ms;
    }
    // samples: one per lane and load (with the taper, a record and a taper
    // pair make one sample)
    if (st == JFDK_OK && best > 0.0f)
        *samples_per_s = (double)ctas * kGatherThreads * iters * kGatherLoads / (best * 1e-3);
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (s) cudaStreamDestroy(s);
    cudaFree(rec);
    cudaFree(tw);
    cudaFree(sink);
    cudaGetLastError();
    return st;
}
