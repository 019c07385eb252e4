// prep.cu -- fused preprocessing and cosine pre-weight (sm_100a).
//
// One pass over the raw uint16 frames produces the A operand of the ramp
// product: A[row][i] = preprocess(raw)[row][i] * preweight[row][i], plus the
// unweighted edge mean of every row (the truncation-ramp level).  Each CTA
// handles one detector row of one view; a thread owns 4 consecutive columns
// (8-byte raw loads, 16-byte stores when the crop is 4-aligned).
//
// Reference semantics:
//   PreProcessingCore::Process   PreProcessingAgent/PreProcessingCore.cpp:67-86
//     (Convert_16u_to_32f, LowerBound(1), crop, GainCorr /BrightField,
//      NLog -ln, BeamHardeningCorr p*(a0 + p*(a1 + a2*p)) in the order of
//      PreProcessingAgent/BeamHardeningCorr.cpp:17-27)
//   PreFilterWeightGenerator::Generate  FilterAgent/PreFilterWeightGenerator.cpp:52-124
//     (distance between the back-projected points at w = 0 and w = 1 through
//      the inverse transform matrix; weight = frame minimum / distance)
//   FilterCore::ProcessRow edge mean    FilterAgent/FilterCore.cpp:201-214
// The float expressions are written with explicit _rn intrinsics so no FMA
// contraction changes their rounding relative to the reference.
#include <cuda_runtime.h>

#include <cstdint>

#include "jfdk_internal.h"

namespace jfdk {
namespace {

__device__ __forceinline__ float prep_pixel(float p, const PrepParams& P) {
    p = fmaxf(p, 1.0f);                 // LowerBound(1.0f); p is never NaN here
    p = __fdiv_rn(p, P.bright_field);   // GainCorr
    p = -logf(p);                       // NLog: ln, then * -1
    if (P.do_bhc) {                     // BeamHardeningCorr
        float buf = __fmul_rn(p, P.bhc2);
        buf = __fadd_rn(buf, P.bhc1);
        buf = __fmul_rn(buf, p);
        buf = __fadd_rn(buf, P.bhc0);
        p = __fmul_rn(p, buf);
    }
    return p;
}

// Per-row constants of the pre-weight distance (Generate's scalars).
struct PWRow {
    float t30, t31v, n0c, n1c;
    float tr0[3], trv[3], c0[3], c1[3];
};

__device__ __forceinline__ PWRow pw_row(const float* T, float v) {
    PWRow r;
    r.t30 = T[12];
    r.t31v = __fmul_rn(v, T[13]);
    r.n0c = __fadd_rn(__fmul_rn(0.0f, T[14]), T[15]);   // w0 * T32 + T33
    r.n1c = __fadd_rn(__fmul_rn(1.0f, T[14]), T[15]);   // w1 * T32 + T33
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        r.tr0[k] = T[k * 4 + 0];
        r.trv[k] = __fmul_rn(v, T[k * 4 + 1]);
        r.c0[k] = __fadd_rn(__fmul_rn(0.0f, T[k * 4 + 2]), T[k * 4 + 3]);
        r.c1[k] = __fadd_rn(__fmul_rn(1.0f, T[k * 4 + 2]), T[k * 4 + 3]);
    }
    return r;
}

__device__ __forceinline__ float pw_dist(const PWRow& r, float u) {
    const float t = __fadd_rn(__fmul_rn(u, r.t30), r.t31v);
    const float norm0 = __fadd_rn(t, r.n0c);
    const float norm1 = __fadd_rn(t, r.n1c);
    float acc = 0.0f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float s = __fadd_rn(__fmul_rn(u, r.tr0[k]), r.trv[k]);
        const float a0 = __fdiv_rn(__fadd_rn(s, r.c0[k]), norm0);
        const float a1 = __fdiv_rn(__fadd_rn(s, r.c1[k]), norm1);
        const float d = __fsub_rn(a0, a1);
        acc = (k == 0) ? __fmul_rn(d, d) : __fadd_rn(acc, __fmul_rn(d, d));
    }
    return __fsqrt_rn(acc);
}

__device__ __forceinline__ float u_axis(int i, int in_w, int det_right) {
    // PreFilterWeightGenerator.cpp:35-40
    return det_right ? __fsub_rn((float)i, (float)in_w / 2) : (float)i;
}

// ---- frame minimum of the distance, per 9-view group -----------------------
__global__ void __launch_bounds__(256) preweight_dmin_kernel(const float* __restrict__ tinv,
                                                             int rows, int L, int in_w,
                                                             int det_right, float* dmin) {
    const int g = blockIdx.y, row = blockIdx.x;
    __shared__ float T[16];
    if (threadIdx.x < 16) T[threadIdx.x] = tinv[g * 16 + threadIdx.x];
    __syncthreads();
    const PWRow r = pw_row(T, (float)row);
    float m = __int_as_float(0x7f800000);
    for (int i = threadIdx.x; i < L; i += blockDim.x) m = fminf(m, pw_dist(r, u_axis(i, in_w, det_right)));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fminf(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ float wm[8];
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fminf(m, wm[w]);
        atomicMin((int*)&dmin[g], __float_as_int(m));  // distances are >= 0
    }
}

// ---- raw -> preprocessed frame (agent path) ---------------------------------
__global__ void __launch_bounds__(256) preprocess_kernel(PrepParams P, float* __restrict__ out) {
    const int row = blockIdx.x, v = blockIdx.y;
    const uint16_t* src = P.raw + ((size_t)v * P.in_h + row + P.crop_y) * P.in_w + P.crop_x;
    float* dst = out + ((size_t)v * P.rows + row) * P.width;
    for (int i = threadIdx.x; i < P.width; i += blockDim.x) dst[i] = prep_pixel((float)src[i], P);
}

// ---- pre-weight + edge mean of a preprocessed row --------------------------
template <bool FROM_RAW>
__global__ void __launch_bounds__(256) weight_kernel(PrepParams P, const float* __restrict__ in,
                                                     int width, int rows, int v0, WeightParams W,
                                                     float* __restrict__ A, int a_pitch,
                                                     float* __restrict__ e) {
    const int row = blockIdx.x, vl = blockIdx.y;
    const int view = (v0 + vl) % W.num_views;
    const int g = view / 9;
    __shared__ float T[16];
    if (threadIdx.x < 16) T[threadIdx.x] = W.tinv[g * 16 + threadIdx.x];
    __syncthreads();
    const float dmin = W.dmin[g];
    const PWRow r = pw_row(T, (float)row);
    const size_t m = (size_t)vl * rows + row;
    float* a = A + m * a_pitch;
    const uint16_t* src = FROM_RAW ? P.raw + ((size_t)vl * P.in_h + row + P.crop_y) * P.in_w + P.crop_x
                                   : nullptr;
    const float* fin = FROM_RAW ? nullptr : in + m * width;
    auto pix = [&](int i) -> float { return FROM_RAW ? prep_pixel((float)src[i], P) : fin[i]; };
    const bool vec = FROM_RAW && ((reinterpret_cast<uintptr_t>(P.raw) & 7) == 0) &&
                     ((reinterpret_cast<uintptr_t>(A) & 15) == 0) && ((P.crop_x & 3) == 0) &&
                     ((P.in_w & 3) == 0) && ((width & 3) == 0) && ((a_pitch & 3) == 0);
    if (vec) {
        for (int i4 = threadIdx.x * 4; i4 < width; i4 += blockDim.x * 4) {
            const uint2 raw4 = *reinterpret_cast<const uint2*>(src + i4);
            float p[4] = {(float)(raw4.x & 0xffffu), (float)(raw4.x >> 16), (float)(raw4.y & 0xffffu),
                          (float)(raw4.y >> 16)};
            float4 o;
            float* op = &o.x;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const float pw = __fdiv_rn(dmin, pw_dist(r, u_axis(i4 + k, width, W.det_right)));
                op[k] = __fmul_rn(prep_pixel(p[k], P), pw);
            }
            *reinterpret_cast<float4*>(a + i4) = o;
        }
    } else {
        for (int i = threadIdx.x; i < width; i += blockDim.x) {
            const float pw = __fdiv_rn(dmin, pw_dist(r, u_axis(i, width, W.det_right)));
            a[i] = __fmul_rn(pix(i), pw);
        }
    }
    for (int i = width + threadIdx.x; i < a_pitch; i += blockDim.x) a[i] = 0.0f;
    if (threadIdx.x == 0) {
        // FilterCore.cpp:203-214 -- mean of the three outermost unweighted samples
        const float edge = W.mirror ? __fdiv_rn(__fadd_rn(__fadd_rn(pix(width - 1), pix(width - 2)), pix(width - 3)), 3.0f)
                                    : __fdiv_rn(__fadd_rn(__fadd_rn(pix(0), pix(1)), pix(2)), 3.0f);
        e[m] = edge;
    }
}

}  // namespace

cudaError_t launch_preweight_dmin(const float* tinv, int groups, int rows, int L, int in_w,
                                  int det_right, float* dmin, cudaStream_t s) {
    cudaError_t err = cudaMemsetAsync(dmin, 0x7f, sizeof(float) * groups, s);
    if (err != cudaSuccess) return err;
    preweight_dmin_kernel<<<dim3(rows, groups), 256, 0, s>>>(tinv, rows, L, in_w, det_right, dmin);
    return cudaGetLastError();
}

cudaError_t launch_preprocess(const PrepParams& p, int nv, float* out, cudaStream_t s) {
    preprocess_kernel<<<dim3(p.rows, nv), 256, 0, s>>>(p, out);
    return cudaGetLastError();
}

cudaError_t launch_weight(const float* in, int nv, int v0, int width, int rows, const WeightParams& w,
                          float* A, int a_pitch, float* e, cudaStream_t s) {
    PrepParams p{};
    weight_kernel<false><<<dim3(rows, nv), 256, 0, s>>>(p, in, width, rows, v0, w, A, a_pitch, e);
    return cudaGetLastError();
}

cudaError_t launch_prep_weight(const PrepParams& p, int nv, int v0, const WeightParams& w, float* A,
                               int a_pitch, float* e, cudaStream_t s) {
    weight_kernel<true><<<dim3(p.rows, nv), 192, 0, s>>>(p, nullptr, p.width, p.rows, v0, w, A, a_pitch, e);
    return cudaGetLastError();
}

}  // namespace jfdk
