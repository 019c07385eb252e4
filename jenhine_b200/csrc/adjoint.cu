// adjoint.cu -- derivatives of the FP32 FDK form (sm_100a):
//
//   * the adjoint of the backprojector, vol = S q / C: with the weights C
//     (the backprojected taper) fixed, q_bar = S^T (vol_bar / C) -- for every
//     voxel and view the transposed bilinear weights of its sample point,
//     scattered into "quad space" (the forward's tapered footprint records,
//     one 16-byte vector atomic per sample) and folded back to detector
//     pixels and multiplied by the taper;
//   * the adjoint of the ramp filter, y = T (w o x) + c e(x) with
//     e(x) = (x0 + x1 + x2) / 3 (or the last three for a mirrored filter):
//     x_bar = w o (T^T y_bar) + (c . y_bar) / 3 on the edge samples;
//   * the gradient with respect to per-view projection-matrix parameters:
//     for a loss L(vol), dL/dtheta_j = sum over voxels of
//     vol_bar / C * [(dS/du - vol dC/du) du/dtheta_j + dS/dv dv/dtheta_j],
//     with u = U/W, du/dtheta_j = (dU_j - u dW_j) / W for (dU_j, dV_j, dW_j)
//     = (dP/dtheta_j) X; per-CTA partial sums in FP32, the reduction over
//     CTAs in FP64.
// Every kernel uses the forward's sample points and in-range decisions
// (bp_common.cuh), so the adjoint is the transpose of the forward as computed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "bp_common.cuh"
#include "jfdk_internal.h"

namespace jfdk {
namespace {

__device__ __forceinline__ void red_add_v4(float4* p, float4 v) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w)
                 : "memory");
}

// rt = vol_bar / C (0 where no view saw the voxel).
__global__ void residual_over_weight_kernel(const float* __restrict__ vol_bar, const float* __restrict__ cnt,
                                            size_t n, float* __restrict__ rt) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float c = cnt[i];
        rt[i] = c != 0.0f ? vol_bar[i] / c : 0.0f;
    }
}

// Quad-space adjoint: Qbar[view - v0][iv][iu] += rt * (bilinear weights).
template <int ZPT, bool WZ>
__global__ void __launch_bounds__(256) bp_adjoint_kernel(AdjParams p) {
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    const int zb = blockIdx.z * ZPT;
    if (x >= p.X || y >= p.Y) return;
    const float ax = bp_axis(x, p.X, p.pxy), ay = bp_axis(y, p.Y, p.pxy);
    const size_t plane = (size_t)p.X * p.Y, base = (size_t)y * p.X + x;
    float az[ZPT], rt[ZPT];
    bool any = false;
#pragma unroll
    for (int k = 0; k < ZPT; ++k) {
        az[k] = bp_axis(zb + k, p.Z, p.pz);
        rt[k] = zb + k < p.Z ? p.rt[(size_t)(zb + k) * plane + base] : 0.0f;
        any |= rt[k] != 0.0f;
    }
    if (!any) return;
    const float umax = (float)(p.U - 1), vmax = (float)(p.V - 1);
    const float4* P4 = reinterpret_cast<const float4*>(p.ptm + (size_t)p.v0 * 12);
    float4* __restrict__ qb = p.qbar;
#pragma unroll 1
    for (int n = 0; n < p.nv; ++n, P4 += 3, qb += p.q_frame) {
        const float4 r0 = __ldg(P4), r1 = __ldg(P4 + 1), r2 = __ldg(P4 + 2);
        const XYTerms xy = bp_xy_terms(ax, ay, r0, r1, r2);
        const float rxy = WZ ? 0.0f : rcp_rn_nr(xy.W);
#pragma unroll
        for (int k = 0; k < ZPT; ++k) {
            const float2 uv = bp_uv(xy, bp_w_r<WZ>(xy, rxy, az[k], r2.z), az[k], r0.z, r1.z);
            const bool in = (uv.x >= 0.0f) & (uv.x <= umax) & (uv.y >= 0.0f) & (uv.y <= vmax);
            if (in && rt[k] != 0.0f) {
                // floor by the 2^23 add rounded toward -inf (exact for 0 <= u, v < 2^23)
                const float2 t = padd_rm(uv, f2(kMagic, kMagic));
                const float2 f = psub(uv, psub(t, f2(kMagic, kMagic)));
                const unsigned iu = __float_as_uint(t.x) - (unsigned)kMagicBits;
                const unsigned iv = __float_as_uint(t.y) - (unsigned)kMagicBits;
                const float a = rt[k] * (1.0f - f.x), b = rt[k] * f.x;
                red_add_v4(qb + (size_t)iv * p.U + iu, make_float4(a * (1.0f - f.y), a * f.y, b * (1.0f - f.y), b * f.y));
            }
        }
    }
}

// Quad space -> detector pixels: p[r][c] appears in quads (r, c).x,
// (r-1, c).y, (r, c-1).z, (r-1, c-1).w, each times the taper w[c].
__global__ void __launch_bounds__(256) unpack_adjoint_kernel(const float4* __restrict__ qbar, long long q_frame,
                                                             int rows, int U, const float2* __restrict__ tw,
                                                             int view0, int num_views, float* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y, f = blockIdx.z;
    if (c >= U) return;
    const float4* q = qbar + (size_t)f * q_frame;
    float s = q[(size_t)r * U + c].x;
    if (r > 0) s += q[(size_t)(r - 1) * U + c].y;
    if (c > 0) s += q[(size_t)r * U + c - 1].z;
    if (r > 0 && c > 0) s += q[(size_t)(r - 1) * U + c - 1].w;
    const float w = tw[(size_t)((view0 + f) % num_views) * U + c].x;
    out[(size_t)f * rows * U + (size_t)r * U + c] = w * s;
}

// Geometry gradient: per (CTA, view) partial sums of the 6 components.
//
// For a sample with a_u = rt (dS/du - vol dC/du) / W, a_v = rt dS/dv / W and
// s = a_u u + a_v v, the contribution to component j is
// a_u dU_j + a_v dV_j - s dW_j with (dU_j, dV_j, dW_j) = dP_j (x, y, z, 1).
// That is linear in dP_j, so a thread only sums, over its slices, the six
// moments a_u, a_u z, a_v, a_v z, s, s z; per view they become the twelve
// coefficients m of the 3x4 matrix dP_j (m = (x A, y A, A_z, A) for the U
// row, likewise B for V and -C for W); the CTA sums m over its threads
// (a transposing butterfly in each warp, then shared memory), and six
// threads form sum_i dP_j[i] m[i].  dP is read once per CTA and view.
template <int ZPT, bool WZ>
__global__ void __launch_bounds__(256) geometry_gradient_kernel(AdjParams p) {
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    const int zb = blockIdx.z * ZPT;
    const bool valid = x < p.X && y < p.Y;
    const float ax = bp_axis(x, p.X, p.pxy), ay = bp_axis(y, p.Y, p.pxy);
    const size_t plane = (size_t)p.X * p.Y, base = (size_t)y * p.X + x;
    float az[ZPT], rt[ZPT], vo[ZPT];
#pragma unroll
    for (int k = 0; k < ZPT; ++k) {
        az[k] = bp_axis(zb + k, p.Z, p.pz);
        const bool in = valid && zb + k < p.Z;
        rt[k] = in ? p.rt[(size_t)(zb + k) * plane + base] : 0.0f;
        vo[k] = in ? p.vol[(size_t)(zb + k) * plane + base] : 0.0f;
        if (!(vo[k] == vo[k])) rt[k] = 0.0f;   // unseen voxel: no contribution
    }
    const float umax = (float)(p.U - 1), vmax = (float)(p.V - 1);
    const int tid = threadIdx.y * 32 + threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const size_t cta = ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    const size_t ncta = (size_t)gridDim.x * gridDim.y * gridDim.z;
    __shared__ float red[2][8][16];
    const float4* P4 = reinterpret_cast<const float4*>(p.ptm + (size_t)p.v0 * 12);
#pragma unroll 1
    for (int n = 0; n < p.nv; ++n, P4 += 3) {
        float A0 = 0.f, A1 = 0.f, B0 = 0.f, B1 = 0.f, C0 = 0.f, C1 = 0.f;
        if (valid) {
            const float4 r0 = __ldg(P4), r1 = __ldg(P4 + 1), r2 = __ldg(P4 + 2);
            const XYTerms xy = bp_xy_terms(ax, ay, r0, r1, r2);
            const float rxy = WZ ? 0.0f : rcp_rn_nr(xy.W);
            const float4* __restrict__ q = p.q4 + (size_t)n * p.q_frame;
            const float2* __restrict__ tw = p.tw + (size_t)((p.v0 + n) % p.num_views) * p.U;
#pragma unroll
            for (int k = 0; k < ZPT; ++k) {
                const float2 wr = bp_w_r<WZ>(xy, rxy, az[k], r2.z);
                const float2 uv = bp_uv(xy, wr, az[k], r0.z, r1.z);
                const bool in = (uv.x >= 0.0f) & (uv.x <= umax) & (uv.y >= 0.0f) & (uv.y <= vmax);
                if (in && rt[k] != 0.0f) {
                    const float2 t = padd_rm(uv, f2(kMagic, kMagic));          // 2^23 + floor
                    const float2 f = psub(uv, psub(t, f2(kMagic, kMagic)));
                    const float fx = f.x, fy = f.y;
                    const unsigned iu = __float_as_uint(t.x) - (unsigned)kMagicBits;
                    const unsigned iv = __float_as_uint(t.y) - (unsigned)kMagicBits;
                    const float4 Q = q[(size_t)iv * p.U + iu];
                    const float2 w = tw[iu];
                    // quads: (t00, t10, t01 - t00, t11 - t10); taper pairs (w0, w1 - w0)
                    const float dSu = (1.0f - fy) * Q.z + fy * Q.w;
                    const float dSv = (Q.y - Q.x) + fx * (Q.w - Q.z);
                    const float iw = wr.y;                                 // RN(1 / W)
                    const float au = rt[k] * (dSu - vo[k] * w.y) * iw;
                    const float av = rt[k] * dSv * iw;
                    const float sk = au * (uv.x - 0.5f) + av * (uv.y - 0.5f);   // u = U / W, v = V / W
                    A0 += au; A1 = fmaf(au, az[k], A1);
                    B0 += av; B1 = fmaf(av, az[k], B1);
                    C0 += sk; C1 = fmaf(sk, az[k], C1);
                }
            }
        }
        // the coefficients of dP_j's twelve entries (padded to 16)
        float m[16] = {ax * A0, ay * A0, A1, A0, ax * B0, ay * B0, B1, B0,
                       -ax * C0, -ay * C0, -C1, -C0, 0.f, 0.f, 0.f, 0.f};
        // transposing butterfly: after the steps at 16, 8, 4, 2 lanes apart
        // lane l holds one coefficient, index (l >> 1) & 15, summed over 16
        // lanes; the step at 1 completes the warp's sum
#pragma unroll
        for (int o = 16, h = 8; o >= 2; o >>= 1, h >>= 1) {
            const bool upper = (lane & o) != 0;
#pragma unroll
            for (int i = 0; i < h; ++i) {
                const float send = upper ? m[i] : m[i + h];
                const float keep = upper ? m[i + h] : m[i];
                m[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
            }
        }
        m[0] += __shfl_xor_sync(0xffffffffu, m[0], 1);
        const int buf = n & 1;
        if ((lane & 1) == 0) red[buf][warp][lane >> 1] = m[0];
        __syncthreads();
        if (tid < 6) {
            float mc[12];
#pragma unroll
            for (int i = 0; i < 12; ++i) {
                float t = 0.0f;
#pragma unroll
                for (int w = 0; w < 8; ++w) t += red[buf][w][i];
                mc[i] = t;
            }
            const float* d = p.dptm + (size_t)n * 72 + tid * 12;
            float g = 0.0f;
#pragma unroll
            for (int i = 0; i < 12; ++i) g = fmaf(__ldg(d + i), mc[i], g);
            p.partial[((size_t)n * ncta + cta) * 6 + tid] = g;
        }
    }
}

// grad[view][j] = sum over CTAs of the partials, in FP64.
__global__ void reduce_partials_kernel(const float* __restrict__ partial, size_t ncta, int nv, double* grad) {
    const int n = blockIdx.x, j = threadIdx.y;
    double s = 0.0;
    for (size_t c = threadIdx.x; c < ncta; c += blockDim.x) s += (double)partial[((size_t)n * ncta + c) * 6 + j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) grad[(size_t)n * 6 + j] = s;
}

// Filter adjoint, after out = T^T y_bar (rows of in_w): out *= w (the
// pre-weight of the row), then (c . y_bar) / 3 added to the edge samples.
__global__ void __launch_bounds__(256) filter_adjoint_finish_kernel(const float* __restrict__ ybar, int out_w,
                                                                    float* __restrict__ xbar, int in_w, int rows,
                                                                    int v0, int num_views,
                                                                    const float* __restrict__ pw,
                                                                    const float* __restrict__ c, int mirror) {
    const size_t m = (size_t)blockIdx.y * rows + blockIdx.x;
    const int row = blockIdx.x, view = (v0 + blockIdx.y) % num_views, g = view / 9;
    const float* yb = ybar + m * out_w;
    float* xb = xbar + m * in_w;
    const float* w = pw + ((size_t)g * rows + row) * in_w;
    float dot = 0.0f;
    for (int j = threadIdx.x; j < out_w; j += blockDim.x) dot = fmaf(c[j], yb[j], dot);
    __shared__ float part[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = dot;
    __syncthreads();
    float e = 0.0f;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) e += part[i];
    e /= 3.0f;
    for (int i = threadIdx.x; i < in_w; i += blockDim.x) {
        float v = xb[i] * w[i];
        if (mirror ? (i >= in_w - 3) : (i < 3)) v += e;
        xb[i] = v;
    }
}

// y_bar [M][out_w] -> A operand rows [M][pitch], zero padded.
__global__ void pad_rows_kernel(const float* __restrict__ src, int w, float* __restrict__ dst, int pitch) {
    const size_t m = blockIdx.x;
    for (int i = threadIdx.x; i < pitch; i += blockDim.x) dst[m * pitch + i] = i < w ? src[m * w + i] : 0.0f;
}

template <int ZPT>
dim3 bp_grid(const AdjParams& p) {
    return dim3((p.X + 31) / 32, (p.Y + 7) / 8, (p.Z + ZPT - 1) / ZPT);
}

constexpr int kAdjZpt = 8;

}  // namespace

cudaError_t launch_residual_over_weight(const float* vol_bar, const float* cnt, size_t n, float* rt, cudaStream_t s) {
    const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
    residual_over_weight_kernel<<<blocks, 256, 0, s>>>(vol_bar, cnt, n, rt);
    return cudaGetLastError();
}

cudaError_t launch_bp_adjoint(const AdjParams& p, bool wz, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(p.qbar, 0, sizeof(float4) * (size_t)p.nv * p.q_frame, s);
    if (e != cudaSuccess) return e;
    if (wz)
        bp_adjoint_kernel<kAdjZpt, true><<<bp_grid<kAdjZpt>(p), dim3(32, 8), 0, s>>>(p);
    else
        bp_adjoint_kernel<kAdjZpt, false><<<bp_grid<kAdjZpt>(p), dim3(32, 8), 0, s>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_unpack_adjoint(const float4* qbar, long long q_frame, int nv, int rows, int U, const float2* tw,
                                  int view0, int num_views, float* out, cudaStream_t s) {
    dim3 grid((U + 255) / 256, rows, nv);
    unpack_adjoint_kernel<<<grid, 256, 0, s>>>(qbar, q_frame, rows, U, tw, view0, num_views, out);
    return cudaGetLastError();
}

size_t geometry_gradient_ctas(const AdjParams& p) {
    const dim3 g = bp_grid<kAdjZpt>(p);
    return (size_t)g.x * g.y * g.z;
}

cudaError_t launch_geometry_gradient(const AdjParams& p, bool wz, double* grad, cudaStream_t s) {
    if (wz)
        geometry_gradient_kernel<kAdjZpt, true><<<bp_grid<kAdjZpt>(p), dim3(32, 8), 0, s>>>(p);
    else
        geometry_gradient_kernel<kAdjZpt, false><<<bp_grid<kAdjZpt>(p), dim3(32, 8), 0, s>>>(p);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    reduce_partials_kernel<<<p.nv, dim3(32, 6), 0, s>>>(p.partial, geometry_gradient_ctas(p), p.nv, grad);
    return cudaGetLastError();
}

cudaError_t launch_pad_rows(const float* src, size_t rows, int w, float* dst, int pitch, cudaStream_t s) {
    pad_rows_kernel<<<(unsigned)rows, 256, 0, s>>>(src, w, dst, pitch);
    return cudaGetLastError();
}

cudaError_t launch_filter_adjoint_finish(const float* ybar, int out_w, float* xbar, int in_w, int rows, int nv, int v0,
                                         int num_views, const float* pw, const float* c, int mirror, cudaStream_t s) {
    filter_adjoint_finish_kernel<<<dim3(rows, nv), 256, 0, s>>>(ybar, out_w, xbar, in_w, rows, v0, num_views, pw, c,
                                                                mirror);
    return cudaGetLastError();
}

}  // namespace jfdk
