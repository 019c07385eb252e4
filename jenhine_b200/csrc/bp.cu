// bp.cu -- voxel-driven cone-beam backprojection with fused normalisation and
// CT numbers (sm_100a).
//
// Semantics follow the reference's CPU backprojector, BPCore
// (BPAgent/BPCore.cpp:115-220):
//   * per view the projection is multiplied by the view's u-taper and an
//     image of the taper is backprojected alongside it (the weight);
//   * for voxel (x, y, z): U = (x*P0 + (y*P1 + P3)) + z*P2, likewise V, W;
//     u = U / W + 0.5, v = V / W + 0.5;
//   * bilinear sample with pixel centres at integers, taken only when
//     0 <= u <= cols-1 and 0 <= v <= rows-1 (ippiRemap leaves the destination
//     untouched otherwise, so the view then adds nothing to sum or weight);
//   * voxel = sum / weight, then CTNumCore (CTNumAgent/CTNumCore.cpp:22-36).
// The reference GPU kernel (BPCUDAAgent/BPCUDACore.cu:25-66) differs: it
// samples the taper without interpolation, checks only u and clamps v.
//
// Layout and work split: the volume is [z][y][x] with x fastest.  A CTA is
// 32 x 8 threads over (x, y); each thread owns ZPT consecutive slices of its
// (x, y) column and keeps their sums and weights in registers across all
// views of the launch, so a launch that covers every view touches the volume
// in HBM exactly once (the final store).  Filtered projections are read
// through L1 from a padded store ([rows + 1][pitch] per view, zero padded) so
// the bilinear +1 neighbours never need clamping.
//
// EXACT = true reproduces BPCore's rounding step for step (IEEE division,
// every product and sum rounded separately); EXACT = false uses one
// reciprocal per sample point and fused multiply-adds.
#include <cuda_runtime.h>

#include <cstdint>

#include "jfdk_internal.h"

namespace jfdk {
namespace {

__device__ __forceinline__ float ct_number(float mu, float s, float n1) {
    // CTNumCore::Process: h = mu * s - 1000; above 300 HU the slope is norm1,
    // capped at 8191.  Separately rounded, no contraction.
    float h = __fsub_rn(__fmul_rn(mu, s), 1000.f);
    if (h > 300.0f) {
        const float t = __fadd_rn(__fmul_rn(__fsub_rn(h, 300.0f), n1), 300.0f);
        h = (t < 8191.f) ? t : 8191.f;
    }
    return h;
}

__device__ __forceinline__ int16_t to_i16(float f) {
    if (f != f) return 0;
    const float t = truncf(f);
    return t >= 32767.0f ? (int16_t)32767 : (t <= -32768.0f ? (int16_t)-32768 : (int16_t)t);
}

template <int ZPT, bool FINALIZE, bool TAPERED, bool EXACT>
__global__ void __launch_bounds__(256) bp_kernel(BPParams p) {
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    const int zb = p.z_begin + blockIdx.z * ZPT;
    if (x >= p.X || y >= p.Y) return;

    // Axes as BPCore builds them (BPCore.cpp:47-66): (i - (n-1)/2) * pitch.
    const float ax = __fmul_rn(__fadd_rn(-((float)p.X - 1.0f) / 2.0f, (float)x), p.pxy);
    const float ay = __fmul_rn(__fadd_rn(-((float)p.Y - 1.0f) / 2.0f, (float)y), p.pxy);
    float az[ZPT], sum[ZPT], cnt[ZPT];
    const size_t plane = (size_t)p.X * p.Y;
    const size_t base = (size_t)y * p.X + x;
#pragma unroll
    for (int k = 0; k < ZPT; ++k) {
        az[k] = __fmul_rn(__fadd_rn(-((float)p.Z - 1.0f) / 2.0f, (float)(zb + k)), p.pz);
        const bool in = zb + k < p.z_end;
        sum[k] = (p.load_acc && in) ? p.sum[(size_t)(zb + k) * plane + base] : 0.0f;
        cnt[k] = (p.load_acc && in) ? p.cnt[(size_t)(zb + k) * plane + base] : 0.0f;
    }
    const float umax = (float)(p.U - 1), vmax = (float)(p.V - 1);

    for (int view = p.v0; view < p.v0 + p.nv; ++view) {
        const float4* P4 = reinterpret_cast<const float4*>(p.ptm + (size_t)view * 12);
        const float4 r0 = __ldg(P4), r1 = __ldg(P4 + 1), r2 = __ldg(P4 + 2);
        // XxPM0 + (YxPM1 + PM3), etc. (BPCore.cpp:120-145)
        const float Uxy = __fadd_rn(__fmul_rn(ax, r0.x), __fadd_rn(__fmul_rn(ay, r0.y), r0.w));
        const float Vxy = __fadd_rn(__fmul_rn(ax, r1.x), __fadd_rn(__fmul_rn(ay, r1.y), r1.w));
        const float Wxy = __fadd_rn(__fmul_rn(ax, r2.x), __fadd_rn(__fmul_rn(ay, r2.y), r2.w));
        const float* __restrict__ q = p.q + (size_t)(view - p.view_base) * p.frame_stride;
        const float* __restrict__ w = p.uw + (size_t)view * p.pitch;
#pragma unroll
        for (int k = 0; k < ZPT; ++k) {
            float u, v;
            if (EXACT) {
                const float Uz = __fadd_rn(Uxy, __fmul_rn(az[k], r0.z));
                const float Vz = __fadd_rn(Vxy, __fmul_rn(az[k], r1.z));
                const float Wz = __fadd_rn(Wxy, __fmul_rn(az[k], r2.z));
                u = __fadd_rn(__fdiv_rn(Uz, Wz), 0.5f);
                v = __fadd_rn(__fdiv_rn(Vz, Wz), 0.5f);
            } else {
                const float Uz = fmaf(az[k], r0.z, Uxy);
                const float Vz = fmaf(az[k], r1.z, Vxy);
                const float Wz = fmaf(az[k], r2.z, Wxy);
                const float rw = __frcp_rn(Wz);
                u = fmaf(Uz, rw, 0.5f);
                v = fmaf(Vz, rw, 0.5f);
            }
            if (u >= 0.0f && u <= umax && v >= 0.0f && v <= vmax) {
                const float fu = floorf(u), fv = floorf(v);
                const int ix = (int)fu, iy = (int)fv;
                const float fx = u - fu, fy = v - fv;   // exact (Sterbenz)
                const float* r = q + (size_t)iy * p.pitch + ix;
                float p00 = __ldg(r), p01 = __ldg(r + 1);
                float p10 = __ldg(r + p.pitch), p11 = __ldg(r + p.pitch + 1);
                const float w0 = __ldg(w + ix), w1 = __ldg(w + ix + 1);
                if (!TAPERED) {  // InitView's in-place projection *= uWeight
                    p00 = __fmul_rn(p00, w0); p01 = __fmul_rn(p01, w1);
                    p10 = __fmul_rn(p10, w0); p11 = __fmul_rn(p11, w1);
                }
                float val, c;
                if (EXACT) {
                    const float t0 = __fadd_rn(p00, __fmul_rn(fx, __fsub_rn(p01, p00)));
                    const float t1 = __fadd_rn(p10, __fmul_rn(fx, __fsub_rn(p11, p10)));
                    val = __fadd_rn(t0, __fmul_rn(fy, __fsub_rn(t1, t0)));
                    c = __fadd_rn(w0, __fmul_rn(fx, __fsub_rn(w1, w0)));
                    sum[k] = __fadd_rn(sum[k], val);
                    cnt[k] = __fadd_rn(cnt[k], c);
                } else {
                    const float t0 = fmaf(fx, p01 - p00, p00);
                    const float t1 = fmaf(fx, p11 - p10, p10);
                    val = fmaf(fy, t1 - t0, t0);
                    c = fmaf(fx, w1 - w0, w0);
                    sum[k] += val;
                    cnt[k] += c;
                }
            }
        }
    }

#pragma unroll
    for (int k = 0; k < ZPT; ++k) {
        if (zb + k >= p.z_end) break;
        const size_t idx = (size_t)(zb + k) * plane + base;
        if (FINALIZE) {
            float o = __fdiv_rn(sum[k], cnt[k]);   // BPCore::DoneSlice
            if (p.apply_ct) o = ct_number(o, p.ct_scale, p.ct_norm1);
            if (p.out) p.out[idx] = o;
            if (p.out16) p.out16[idx] = to_i16(o);
        } else {
            p.sum[idx] = sum[k];
            p.cnt[idx] = cnt[k];
        }
    }
}

__global__ void finalize_kernel(const float* __restrict__ sum, const float* __restrict__ cnt, size_t n,
                                int apply_ct, float s, float n1, float* out, int16_t* out16) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float o = __fdiv_rn(sum[i], cnt[i]);
        if (apply_ct) o = ct_number(o, s, n1);
        if (out) out[i] = o;
        if (out16) out16[i] = to_i16(o);
    }
}

__global__ void ctnum_kernel(float* d, size_t n, float s, float n1) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        d[i] = ct_number(d[i], s, n1);
}

// ZFilterAgent::ProcessTask (FilterAgent/ZFilterAgent.cpp:49-71): out[v] =
// 0.5 in[v] + 0.25 in[max(v-1,0)] + 0.25 in[min(v+1,rows-1)], each product
// and sum rounded in the reference's order.  One thread walks one column of
// one frame top to bottom, keeping the previous input row in a register, so
// the update is in place.
__global__ void zfilter_kernel(float* frames, int nv, int rows, int width, long long stride, int pitch) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x, f = blockIdx.y;
    if (col >= width || f >= nv) return;
    float* c = frames + (size_t)f * stride + col;
    float prev = c[0], cur = c[0];
    for (int r = 0; r < rows; ++r) {
        const float next = c[(size_t)(r + 1 < rows ? r + 1 : rows - 1) * pitch];
        float o = __fmul_rn(cur, 0.5f);
        o = __fadd_rn(o, __fmul_rn(prev, 0.25f));
        o = __fadd_rn(o, __fmul_rn(next, 0.25f));
        c[(size_t)r * pitch] = o;
        prev = cur;
        cur = next;
    }
}

template <int ZPT, bool F, bool T, bool E>
cudaError_t go(const BPParams& p, cudaStream_t s) {
    const int nz = p.z_end - p.z_begin;
    dim3 grid((p.X + 31) / 32, (p.Y + 7) / 8, (nz + ZPT - 1) / ZPT);
    bp_kernel<ZPT, F, T, E><<<grid, dim3(32, 8), 0, s>>>(p);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_bp(const BPParams& p, bool finalize, bool tapered, bool exact, cudaStream_t s) {
    constexpr int Z = 8;
    if (finalize) {
        if (tapered) return exact ? go<Z, true, true, true>(p, s) : go<Z, true, true, false>(p, s);
        return exact ? go<Z, true, false, true>(p, s) : go<Z, true, false, false>(p, s);
    }
    if (tapered) return exact ? go<Z, false, true, true>(p, s) : go<Z, false, true, false>(p, s);
    return exact ? go<Z, false, false, true>(p, s) : go<Z, false, false, false>(p, s);
}

cudaError_t launch_finalize(const float* sum, const float* cnt, size_t n, int apply_ct, float ct_scale,
                            float norm1, float* out, int16_t* out16, cudaStream_t s) {
    const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
    finalize_kernel<<<blocks, 256, 0, s>>>(sum, cnt, n, apply_ct, ct_scale, norm1, out, out16);
    return cudaGetLastError();
}

cudaError_t launch_ctnum(float* d, size_t n, float ct_scale, float norm1, cudaStream_t s) {
    const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
    ctnum_kernel<<<blocks, 256, 0, s>>>(d, n, ct_scale, norm1);
    return cudaGetLastError();
}

cudaError_t launch_zfilter(float* frames, int nv, int rows, int width, long long frame_stride, int pitch,
                           cudaStream_t s) {
    dim3 grid((width + 127) / 128, nv);
    zfilter_kernel<<<grid, 128, 0, s>>>(frames, nv, rows, width, frame_stride, pitch);
    return cudaGetLastError();
}

}  // namespace jfdk
