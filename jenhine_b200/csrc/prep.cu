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
#include <cuda_bf16.h>
#include <cuda_fp16.h>
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

// ---- the pre-weight of every group, row and column --------------------------
// weight = frame minimum / distance, the same expression the row kernels
// would evaluate, computed once per context (per 9-view group the reference
// regenerates it, FilterAgent.cpp:161-192).
__global__ void __launch_bounds__(256) preweight_table_kernel(const float* __restrict__ tinv,
                                                              const float* __restrict__ dmin, int rows,
                                                              int in_w, int det_right, float* __restrict__ pw) {
    const int g = blockIdx.y, row = blockIdx.x;
    __shared__ float T[16];
    if (threadIdx.x < 16) T[threadIdx.x] = tinv[g * 16 + threadIdx.x];
    __syncthreads();
    const PWRow r = pw_row(T, (float)row);
    const float dm = dmin[g];
    float* out = pw + ((size_t)g * rows + row) * in_w;
    for (int i = threadIdx.x; i < in_w; i += blockDim.x)
        out[i] = __fdiv_rn(dm, pw_dist(r, u_axis(i, in_w, det_right)));
}

// ---- raw -> preprocessed frame (agent path) ---------------------------------
__global__ void __launch_bounds__(256) preprocess_kernel(PrepParams P, float* __restrict__ out) {
    const int row = blockIdx.x, v = blockIdx.y;
    const uint16_t* src = P.raw + ((size_t)v * P.in_h + row + P.crop_y) * P.in_w + P.crop_x;
    float* dst = out + ((size_t)v * P.rows + row) * P.width;
    for (int i = threadIdx.x; i < P.width; i += blockDim.x) dst[i] = prep_pixel((float)src[i], P);
}

// ---- conjugate-view compositing (CompositeAgent/CompositeCore.cpp:59-149) ----
// Value of column c in [0, 2W) of row r of view k's composite row, the float
// operations in CompositeCore's order: the conjugate half resampled at the
// points the direct view's extended detector would see (MatrixMultiplier
// products of the view's inverse TM and the conjugate PTM, quotients, v
// clamped, ippiRemap's inside-only rule and lerps), the 40 columns next to
// the direct half blended with the direct row's 5-sample edge mean, the
// direct half copied.  dirc(i) and conj(iy, ix) return preprocessed pixels.
template <class D, class C>
__device__ __forceinline__ float composite_value(const CompositeParams& cp, int k, int r, int c, float edge, D dirc,
                                                 C conj) {
    const int W = cp.W, tw = 40;
    const int dircOff = cp.det_right ? W : 0, conjOff = cp.det_right ? 0 : W;
    if (c >= dircOff && c < dircOff + W) return dirc(c - dircOff);
    const int cc = c - conjOff;
    const float* T = cp.tinv + (size_t)k * 16;
    const float* P = cp.ptm + (size_t)((k + cp.num_views / 2) % cp.num_views) * 12;
    const float uvw[4] = {cp.det_right ? __fsub_rn((float)cc, (float)W) : (float)(cc + W), (float)r, 0.0f, 1.0f};
    float xyz[4], q[3];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        float a = 0.0f;
#pragma unroll
        for (int j = 0; j < 4; ++j) a = __fadd_rn(a, __fmul_rn(T[i * 4 + j], uvw[j]));
        xyz[i] = a;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float a = 0.0f;
#pragma unroll
        for (int j = 0; j < 4; ++j) a = __fadd_rn(a, __fmul_rn(P[i * 4 + j], xyz[j]));
        q[i] = a;
    }
    const float u = __fdiv_rn(q[0], q[2]);
    float v = __fdiv_rn(q[1], q[2]);
    if (v < 0.0f) v = 0.0f;
    if (v > (float)cp.H - 1.0f) v = (float)cp.H - 1.0f;
    float o = 0.0f;
    if (u >= 0.0f && u <= (float)(W - 1) && v >= 0.0f && v <= (float)(cp.H - 1)) {
        const int ix = (int)floorf(u), iy = (int)floorf(v);
        const int ix1 = ix + 1 < W ? ix + 1 : W - 1, iy1 = iy + 1 < cp.H ? iy + 1 : cp.H - 1;
        const float fx = __fsub_rn(u, (float)ix), fy = __fsub_rn(v, (float)iy);
        const float p00 = conj(iy, ix), p01 = conj(iy, ix1), p10 = conj(iy1, ix), p11 = conj(iy1, ix1);
        const float t0 = __fadd_rn(p00, __fmul_rn(fx, __fsub_rn(p01, p00)));
        const float t1 = __fadd_rn(p10, __fmul_rn(fx, __fsub_rn(p11, p10)));
        o = __fadd_rn(t0, __fmul_rn(fy, __fsub_rn(t1, t0)));
    }
    const int transOff = cp.det_right ? W - tw : W;
    if (c >= transOff && c < transOff + tw) {
        const int i = c - transOff;
        o = __fadd_rn(__fmul_rn(o, cp.mask[tw + i]), __fmul_rn(edge, cp.mask[i]));
    }
    return o;
}

// The direct row's edge mean: its first (detector right) or last 5 samples,
// summed in double and divided in float (as the library's ippsMean stand-in).
template <class D>
__device__ __forceinline__ float composite_edge(const CompositeParams& cp, D dirc) {
    double sum = 0.0;
    const int b = cp.det_right ? 0 : cp.W - 5;
    for (int i = 0; i < 5; ++i) sum += (double)dirc(b + i);
    return __fdiv_rn((float)sum, 5.0f);
}

__global__ void __launch_bounds__(256) composite_frames_kernel(const float* __restrict__ dirc,
                                                               const float* __restrict__ conj, int v0,
                                                               CompositeParams cp, float* __restrict__ out) {
    const int r = blockIdx.x, f = blockIdx.y, k = (v0 + f) % cp.num_views;
    const float* drow = dirc + ((size_t)f * cp.H + r) * cp.W;
    const float* cfr = conj + (size_t)f * cp.H * cp.W;
    auto D = [&](int i) { return drow[i]; };
    auto Cj = [&](int iy, int ix) { return cfr[(size_t)iy * cp.W + ix]; };
    __shared__ float edge;
    if (threadIdx.x == 0) edge = composite_edge(cp, D);
    __syncthreads();
    float* o = out + ((size_t)f * cp.H + r) * 2 * cp.W;
    for (int c = threadIdx.x; c < 2 * cp.W; c += blockDim.x) o[c] = composite_value(cp, k, r, c, edge, D, Cj);
}

// ---- pre-weight + edge mean of a preprocessed row --------------------------
// The weighted row goes out as the ramp product's A operand in the form the
// product reads (AOut): fp32, or split into a high and a low part -- tf32
// (fp32 storage), bf16, or fp16 of the row scaled by a power of two so its
// largest value lies in [2^14, 2^15) (row_scale[m] = 1 / that factor).

// Round to the nearest TF32 value (10 explicit mantissa bits, ties to even).
__device__ __forceinline__ float tf32_rn(float x) {
    uint32_t b = __float_as_uint(x);
    if ((b & 0x7f800000u) != 0x7f800000u) b = (b + 0xfffu + ((b >> 13) & 1u)) & 0xffffe000u;
    return __uint_as_float(b);
}

template <int OUT>
__device__ __forceinline__ void store4(void* hi, void* lo, size_t at, const float v[4]) {
    if constexpr (OUT == AOUT_F32) {
        *reinterpret_cast<float4*>(static_cast<float*>(hi) + at) = make_float4(v[0], v[1], v[2], v[3]);
    } else if constexpr (OUT == AOUT_TF32X2) {
        float h[4], l[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) { h[k] = tf32_rn(v[k]); l[k] = tf32_rn(v[k] - h[k]); }
        *reinterpret_cast<float4*>(static_cast<float*>(hi) + at) = make_float4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<float4*>(static_cast<float*>(lo) + at) = make_float4(l[0], l[1], l[2], l[3]);
    } else if constexpr (OUT == AOUT_BF16X2) {
        __nv_bfloat162 h[2], l[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            h[k] = __floats2bfloat162_rn(v[2 * k], v[2 * k + 1]);
            const float2 hf = __bfloat1622float2(h[k]);
            l[k] = __floats2bfloat162_rn(v[2 * k] - hf.x, v[2 * k + 1] - hf.y);
        }
        *reinterpret_cast<uint2*>(static_cast<__nv_bfloat16*>(hi) + at) = *reinterpret_cast<uint2*>(h);
        *reinterpret_cast<uint2*>(static_cast<__nv_bfloat16*>(lo) + at) = *reinterpret_cast<uint2*>(l);
    } else {
        __half2 h[2], l[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            h[k] = __floats2half2_rn(v[2 * k], v[2 * k + 1]);
            const float2 hf = __half22float2(h[k]);
            l[k] = __floats2half2_rn(v[2 * k] - hf.x, v[2 * k + 1] - hf.y);
        }
        *reinterpret_cast<uint2*>(static_cast<__half*>(hi) + at) = *reinterpret_cast<uint2*>(h);
        *reinterpret_cast<uint2*>(static_cast<__half*>(lo) + at) = *reinterpret_cast<uint2*>(l);
    }
}

template <int OUT>
__device__ __forceinline__ void store1(void* hi, void* lo, size_t at, float v) {
    if constexpr (OUT == AOUT_F32) {
        static_cast<float*>(hi)[at] = v;
    } else if constexpr (OUT == AOUT_TF32X2) {
        const float h = tf32_rn(v);
        static_cast<float*>(hi)[at] = h;
        static_cast<float*>(lo)[at] = tf32_rn(v - h);
    } else if constexpr (OUT == AOUT_BF16X2) {
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        static_cast<__nv_bfloat16*>(hi)[at] = h;
        static_cast<__nv_bfloat16*>(lo)[at] = __float2bfloat16_rn(v - __bfloat162float(h));
    } else {
        const __half h = __float2half_rn(v);
        static_cast<__half*>(hi)[at] = h;
        static_cast<__half*>(lo)[at] = __float2half_rn(v - __half2float(h));
    }
}

template <bool FROM_RAW, int OUT>
__global__ void __launch_bounds__(256) weight_kernel(PrepParams P, const float* __restrict__ in,
                                                     int width, int rows, int v0, WeightParams W,
                                                     AOperand A, float* __restrict__ e) {
    const int row = blockIdx.x, vl = blockIdx.y;
    const int view = (v0 + vl) % W.num_views;
    const int g = view / 9;
    __shared__ float T[16];
    __shared__ float red[8];
    if (threadIdx.x < 16) T[threadIdx.x] = W.tinv[g * 16 + threadIdx.x];
    __syncthreads();
    const float dmin = W.dmin[g];
    const PWRow r = pw_row(T, (float)row);
    const size_t m = (size_t)vl * rows + row;
    const size_t a0 = m * A.pitch;
    const uint16_t* src = FROM_RAW ? P.raw + ((size_t)vl * P.in_h + row + P.crop_y) * P.in_w + P.crop_x
                                   : nullptr;
    const float* fin = FROM_RAW ? nullptr : in + m * width;
    // compositing from raw frames: direct frame = this view's, conjugate =
    // view (view + N/2) % N of the rotation, both preprocessed on the fly
    const CompositeParams& cp = W.comp;
    const bool comp = FROM_RAW && cp.W > 0;
    const uint16_t* craw = comp ? P.raw_rotation + (size_t)((view + cp.num_views / 2) % cp.num_views) * P.raw_frame +
                                      (size_t)P.crop_y * P.in_w + P.crop_x
                                : nullptr;
    auto dpix = [&](int i) -> float { return prep_pixel((float)src[i], P); };
    auto cpix = [&](int iy, int ix) -> float { return prep_pixel((float)craw[(size_t)iy * P.in_w + ix], P); };
    __shared__ float s_edge;
    if (comp) {
        if (threadIdx.x == 0) s_edge = composite_edge(cp, dpix);
        __syncthreads();
    }
    auto pix = [&](int i) -> float {
        if (!FROM_RAW) return fin[i];
        if (comp) return composite_value(cp, view, row, i, s_edge, dpix, cpix);
        return prep_pixel((float)src[i], P);
    };
    const float* pwrow = W.pw ? W.pw + ((size_t)g * rows + row) * width : nullptr;
    auto value = [&](int i, float p) -> float {
        return __fmul_rn(p, pwrow ? __ldg(pwrow + i) : __fdiv_rn(dmin, pw_dist(r, u_axis(i, width, W.det_right))));
    };
    const int elem = OUT == AOUT_F32 || OUT == AOUT_TF32X2 ? 4 : OUT == AOUT_I8X4 ? 1 : 2;
    const bool vec = FROM_RAW && !comp && ((reinterpret_cast<uintptr_t>(P.raw) & 7) == 0) &&
                     ((reinterpret_cast<uintptr_t>(A.hi) & 15) == 0) &&
                     (OUT == AOUT_F32 || (reinterpret_cast<uintptr_t>(A.lo) & 15) == 0) &&
                     ((P.crop_x & 3) == 0) && ((P.in_w & 3) == 0) && ((width & 3) == 0) &&
                     (((size_t)A.pitch * elem) % 16 == 0);
    // fp16: the row's largest magnitude sets its power-of-two scale first
    float scale = 1.0f;
    if (OUT == AOUT_FP16X2) {
        float mx = 0.0f;
        for (int i = threadIdx.x; i < width; i += blockDim.x) mx = fmaxf(mx, fabsf(value(i, pix(i))));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
        __syncthreads();
        mx = red[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) mx = fmaxf(mx, red[w]);
        scale = (mx > 0.0f && mx <= 3.0e38f) ? ldexpf(1.0f, 14 - ilogbf(mx)) : 1.0f;
        if (threadIdx.x == 0) A.row_scale[m] = __fdiv_rn(1.0f, scale);
    }
    if constexpr (OUT == AOUT_I8X4) {
        // The row's values (staged in shared memory), its power-of-two scale
        // 2^E (the least E with max |a| <= 127 * 2^E), then per element the
        // 32-bit fixed point Q = round(a * 2^(24 - E)) (|Q| < 2^31; exact for
        // every a down to 2^-31 of the row's largest) as four balanced signed
        // bytes, Q = d0 2^24 + d1 2^16 + d2 2^8 + d3, each in [-128, 127].
        extern __shared__ float s_row[];
        float mx = 0.0f;
        if (vec) {
            for (int i4 = threadIdx.x * 4; i4 < width; i4 += blockDim.x * 4) {
                const uint2 raw4 = *reinterpret_cast<const uint2*>(src + i4);
                const float p[4] = {(float)(raw4.x & 0xffffu), (float)(raw4.x >> 16), (float)(raw4.y & 0xffffu),
                                    (float)(raw4.y >> 16)};
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const float v = value(i4 + k, prep_pixel(p[k], P));
                    s_row[i4 + k] = v;
                    mx = fmaxf(mx, fabsf(v));
                }
            }
        } else {
            for (int i = threadIdx.x; i < width; i += blockDim.x) {
                const float v = value(i, pix(i));
                s_row[i] = v;
                mx = fmaxf(mx, fabsf(v));
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
        __syncthreads();
        mx = red[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) mx = fmaxf(mx, red[w]);
        int E = 0;
        if (mx > 0.0f && mx <= 3.0e38f) {
            E = ilogbf(mx) - 6;
            if (mx > ldexpf(127.0f, E)) ++E;
        }
        const float up = ldexpf(1.0f, 24 - E);
        if (threadIdx.x == 0) A.row_scale[m] = ldexpf(1.0f, E);
        int8_t* plane = static_cast<int8_t*>(A.hi);
        const size_t pstride = (size_t)(static_cast<int8_t*>(A.lo) - static_cast<int8_t*>(A.hi));
        for (int i4 = threadIdx.x * 4; i4 < A.pitch; i4 += blockDim.x * 4) {
            int q[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                // |x| <= 127 * 2^24 < 2^31; non-finite rows (E = 0) are clamped
                const float x = i4 + k < width ? s_row[i4 + k] * up : 0.0f;
                q[k] = __float2int_rn(fmaxf(-2130706432.0f, fminf(2130706432.0f, x)));
            }
            signed char d[kI8RowDigits][4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
#pragma unroll
                for (int s = kI8RowDigits - 1; s > 0; --s) {
                    const int lo = ((q[k] + 128) & 255) - 128;
                    d[s][k] = (signed char)lo;
                    q[k] = (q[k] - lo) >> 8;
                }
                d[0][k] = (signed char)q[k];
            }
#pragma unroll
            for (int s = 0; s < kI8RowDigits; ++s)
                *reinterpret_cast<char4*>(plane + s * pstride + a0 + i4) = make_char4(d[s][0], d[s][1], d[s][2], d[s][3]);
        }
    } else if (vec) {
        for (int i4 = threadIdx.x * 4; i4 < width; i4 += blockDim.x * 4) {
            const uint2 raw4 = *reinterpret_cast<const uint2*>(src + i4);
            const float p[4] = {(float)(raw4.x & 0xffffu), (float)(raw4.x >> 16), (float)(raw4.y & 0xffffu),
                                (float)(raw4.y >> 16)};
            float o[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) o[k] = value(i4 + k, prep_pixel(p[k], P)) * scale;
            store4<OUT>(A.hi, A.lo, a0 + i4, o);
        }
    } else {
        for (int i = threadIdx.x; i < width; i += blockDim.x) store1<OUT>(A.hi, A.lo, a0 + i, value(i, pix(i)) * scale);
    }
    if constexpr (OUT != AOUT_I8X4)
        for (int i = width + threadIdx.x; i < A.pitch; i += blockDim.x) store1<OUT>(A.hi, A.lo, a0 + i, 0.0f);
    if (threadIdx.x == 0) {
        // FilterCore.cpp:203-214 -- mean of the three outermost unweighted samples
        const float edge = W.mirror ? __fdiv_rn(__fadd_rn(__fadd_rn(pix(width - 1), pix(width - 2)), pix(width - 3)), 3.0f)
                                    : __fdiv_rn(__fadd_rn(__fadd_rn(pix(0), pix(1)), pix(2)), 3.0f);
        e[m] = edge;
    }
}

// One warp per row, for the int8 digit form and the BF16 pairs: the row's
// values stay in registers (pitch <= 128 * G); for the digits the scale's
// maximum is a warp reduction.  The same values, scale and digits as
// weight_kernel's AOUT_I8X4 / AOUT_BF16X2 paths.  No compositing
// (weight_kernel handles it).
constexpr int kI8WarpGroups = 16;
template <bool FROM_RAW, int G, int OUT>
__global__ void __launch_bounds__(256) weight_warp_kernel(PrepParams P, const float* __restrict__ in, int width,
                                                        int rows, int v0, WeightParams W, AOperand A,
                                                        float* __restrict__ e) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row = blockIdx.x * 8 + warp, vl = blockIdx.y;
    const int view = (v0 + vl) % W.num_views;
    const int g = view / 9;
    __shared__ float T[16];
    if (threadIdx.x < 16) T[threadIdx.x] = W.tinv[g * 16 + threadIdx.x];
    __syncthreads();
    if (row >= rows) return;
    const float dmin = W.dmin[g];
    const PWRow r = pw_row(T, (float)row);
    const size_t m = (size_t)vl * rows + row;
    const size_t a0 = m * A.pitch;
    const uint16_t* src = FROM_RAW ? P.raw + ((size_t)vl * P.in_h + row + P.crop_y) * P.in_w + P.crop_x : nullptr;
    const float* fin = FROM_RAW ? nullptr : in + m * width;
    const float* pwrow = W.pw ? W.pw + ((size_t)g * rows + row) * width : nullptr;
    auto weight = [&](int i) -> float {
        return pwrow ? __ldg(pwrow + i) : __fdiv_rn(dmin, pw_dist(r, u_axis(i, width, W.det_right)));
    };
    auto pix = [&](int i) -> float { return FROM_RAW ? prep_pixel((float)src[i], P) : fin[i]; };
    const bool vec4 = (width & 3) == 0 &&
                      (FROM_RAW ? ((reinterpret_cast<uintptr_t>(src) & 7) == 0)
                                : ((reinterpret_cast<uintptr_t>(fin) & 15) == 0)) &&
                      (!pwrow || (reinterpret_cast<uintptr_t>(pwrow) & 15) == 0);
    float v[G][4];
    float mx = 0.0f;
#pragma unroll
    for (int gi = 0; gi < G; ++gi) {
        const int i4 = gi * 128 + lane * 4;
        if (gi * 128 >= width) break;
        if (vec4 && i4 < width) {
            float p[4], w[4];
            if constexpr (FROM_RAW) {
                const uint2 raw4 = *reinterpret_cast<const uint2*>(src + i4);
                p[0] = prep_pixel((float)(raw4.x & 0xffffu), P); p[1] = prep_pixel((float)(raw4.x >> 16), P);
                p[2] = prep_pixel((float)(raw4.y & 0xffffu), P); p[3] = prep_pixel((float)(raw4.y >> 16), P);
            } else {
                const float4 f = *reinterpret_cast<const float4*>(fin + i4);
                p[0] = f.x; p[1] = f.y; p[2] = f.z; p[3] = f.w;
            }
            if (pwrow) {
                const float4 q = __ldg(reinterpret_cast<const float4*>(pwrow + i4));
                w[0] = q.x; w[1] = q.y; w[2] = q.z; w[3] = q.w;
            } else {
#pragma unroll
                for (int k = 0; k < 4; ++k) w[k] = weight(i4 + k);
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) v[gi][k] = __fmul_rn(p[k], w[k]);
        } else {
#pragma unroll
            for (int k = 0; k < 4; ++k) v[gi][k] = i4 + k < width ? __fmul_rn(pix(i4 + k), weight(i4 + k)) : 0.0f;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) mx = fmaxf(mx, fabsf(v[gi][k]));
    }
    if constexpr (OUT == AOUT_BF16X2) {
#pragma unroll
        for (int gi = 0; gi < G; ++gi) {
            const int i4 = gi * 128 + lane * 4;
            if (gi * 128 >= A.pitch) break;
            if (i4 >= A.pitch) continue;
            float o[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) o[k] = gi * 128 < width ? v[gi][k] : 0.0f;
            store4<AOUT_BF16X2>(A.hi, A.lo, a0 + i4, o);
        }
    } else {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    int E = 0;
    if (mx > 0.0f && mx <= 3.0e38f) {
        E = ilogbf(mx) - 6;
        if (mx > ldexpf(127.0f, E)) ++E;
    }
    const float up = ldexpf(1.0f, 24 - E);
    if (lane == 0) A.row_scale[m] = ldexpf(1.0f, E);
    int8_t* plane = static_cast<int8_t*>(A.hi);
    const size_t pstride = (size_t)(static_cast<int8_t*>(A.lo) - static_cast<int8_t*>(A.hi));
#pragma unroll
    for (int gi = 0; gi < G; ++gi) {
        const int i4 = gi * 128 + lane * 4;
        if (gi * 128 >= A.pitch) break;
        if (i4 >= A.pitch) continue;
        signed char d[kI8RowDigits][4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float x = (gi * 128 < width ? v[gi][k] : 0.0f) * up;
            int q = __float2int_rn(fmaxf(-2130706432.0f, fminf(2130706432.0f, x)));
#pragma unroll
            for (int s2 = kI8RowDigits - 1; s2 > 0; --s2) {
                const int lo = ((q + 128) & 255) - 128;
                d[s2][k] = (signed char)lo;
                q = (q - lo) >> 8;
            }
            d[0][k] = (signed char)q;
        }
#pragma unroll
        for (int s2 = 0; s2 < kI8RowDigits; ++s2)
            *reinterpret_cast<char4*>(plane + s2 * pstride + a0 + i4) = make_char4(d[s2][0], d[s2][1], d[s2][2], d[s2][3]);
    }
    }
    if (lane == 0) {
        // FilterCore.cpp:203-214 -- mean of the three outermost unweighted samples
        const float edge = W.mirror ? __fdiv_rn(__fadd_rn(__fadd_rn(pix(width - 1), pix(width - 2)), pix(width - 3)), 3.0f)
                                    : __fdiv_rn(__fadd_rn(__fadd_rn(pix(0), pix(1)), pix(2)), 3.0f);
        e[m] = edge;
    }
}

template <bool FROM_RAW, int OUT>
cudaError_t launch_weight_warp(const PrepParams& p, const float* in, int nv, int v0, int width, int rows,
                               const WeightParams& w, const AOperand& A, float* e, cudaStream_t s) {
    const dim3 g8((rows + 7) / 8, nv);
    if (A.pitch <= 128 * 6)
        weight_warp_kernel<FROM_RAW, 6, OUT><<<g8, 256, 0, s>>>(p, in, width, rows, v0, w, A, e);
    else if (A.pitch <= 128 * 8)
        weight_warp_kernel<FROM_RAW, 8, OUT><<<g8, 256, 0, s>>>(p, in, width, rows, v0, w, A, e);
    else
        weight_warp_kernel<FROM_RAW, kI8WarpGroups, OUT><<<g8, 256, 0, s>>>(p, in, width, rows, v0, w, A, e);
    return cudaGetLastError();
}

template <bool FROM_RAW>
cudaError_t launch_weight_t(const PrepParams& p, const float* in, int nv, int v0, int width, int rows,
                            const WeightParams& w, const AOperand& A, float* e, int threads, cudaStream_t s) {
    const dim3 grid(rows, nv);
    switch (A.kind) {
        case AOUT_F32: weight_kernel<FROM_RAW, AOUT_F32><<<grid, threads, 0, s>>>(p, in, width, rows, v0, w, A, e); break;
        case AOUT_TF32X2: weight_kernel<FROM_RAW, AOUT_TF32X2><<<grid, threads, 0, s>>>(p, in, width, rows, v0, w, A, e); break;
        case AOUT_BF16X2:
            if (!(FROM_RAW && w.comp.W > 0) && A.pitch <= 128 * kI8WarpGroups && (A.pitch & 3) == 0)
                return launch_weight_warp<FROM_RAW, AOUT_BF16X2>(p, in, nv, v0, width, rows, w, A, e, s);
            weight_kernel<FROM_RAW, AOUT_BF16X2><<<grid, threads, 0, s>>>(p, in, width, rows, v0, w, A, e);
            break;
        case AOUT_FP16X2: weight_kernel<FROM_RAW, AOUT_FP16X2><<<grid, threads, 0, s>>>(p, in, width, rows, v0, w, A, e); break;
        case AOUT_I8X4:
            if (A.pitch % 4 != 0) return cudaErrorInvalidValue;
            if (!(FROM_RAW && w.comp.W > 0) && A.pitch <= 128 * kI8WarpGroups)
                return launch_weight_warp<FROM_RAW, AOUT_I8X4>(p, in, nv, v0, width, rows, w, A, e, s);
            if (width > 12288) return cudaErrorInvalidValue;   // the row in 48 KB of shared memory
            weight_kernel<FROM_RAW, AOUT_I8X4><<<grid, threads, sizeof(float) * width, s>>>(p, in, width, rows, v0, w, A, e);
            break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_preweight_dmin(const float* tinv, int groups, int rows, int L, int in_w,
                                  int det_right, float* dmin, cudaStream_t s) {
    cudaError_t err = cudaMemsetAsync(dmin, 0x7f, sizeof(float) * groups, s);
    if (err != cudaSuccess) return err;
    preweight_dmin_kernel<<<dim3(rows, groups), 256, 0, s>>>(tinv, rows, L, in_w, det_right, dmin);
    return cudaGetLastError();
}

cudaError_t launch_preweight_table(const float* tinv, const float* dmin, int groups, int rows, int in_w,
                                   int det_right, float* pw, cudaStream_t s) {
    preweight_table_kernel<<<dim3(rows, groups), 256, 0, s>>>(tinv, dmin, rows, in_w, det_right, pw);
    return cudaGetLastError();
}

cudaError_t launch_preprocess(const PrepParams& p, int nv, float* out, cudaStream_t s) {
    preprocess_kernel<<<dim3(p.rows, nv), 256, 0, s>>>(p, out);
    return cudaGetLastError();
}

cudaError_t launch_composite_frames(const float* dirc, const float* conj, int v0, int nv, const CompositeParams& c,
                                    float* out, cudaStream_t s) {
    composite_frames_kernel<<<dim3(c.H, nv), 256, 0, s>>>(dirc, conj, v0, c, out);
    return cudaGetLastError();
}

cudaError_t launch_weight(const float* in, int nv, int v0, int width, int rows, const WeightParams& w,
                          const AOperand& A, float* e, cudaStream_t s) {
    PrepParams p{};
    return launch_weight_t<false>(p, in, nv, v0, width, rows, w, A, e, 256, s);
}

cudaError_t launch_prep_weight(const PrepParams& p, int nv, int v0, const WeightParams& w, const AOperand& A,
                               float* e, cudaStream_t s) {
    return launch_weight_t<true>(p, nullptr, nv, v0, p.width, p.rows, w, A, e, 192, s);
}

}  // namespace jfdk
