// bp.cu -- voxel-driven cone-beam backprojection with fused normalisation and
// CT numbers (sm_100a).
//
// Semantics follow the reference's CPU backprojector, BPCore
// (BPAgent/BPCore.cpp:115-220):
//   * per view the projection is multiplied by the view's u-taper and an
//     image of the taper is backprojected alongside it (the weight);
//   * for voxel (x, y, z): U = (x*P0 + (y*P1 + P3)) + z*P2, likewise V, W,
//     every product and sum rounded separately; u = U / W + 0.5,
//     v = V / W + 0.5 with the quotient correctly rounded;
//   * bilinear sample with pixel centres at integers, taken only when
//     0 <= u <= cols-1 and 0 <= v <= rows-1 (ippiRemap leaves the destination
//     untouched otherwise, so the view then adds nothing to sum or weight);
//   * voxel = sum / weight, then CTNumCore (CTNumAgent/CTNumCore.cpp:22-36).
// The reference GPU kernel (BPCUDAAgent/BPCUDACore.cu:25-66) differs: it
// samples the taper without interpolation, checks only u and clamps v.
//
// Data layout.  The filtered, tapered projections are stored as "quads": for
// every view, row r and column c one float4 (p[r][c], p[r+1][c], p[r][c+1],
// p[r+1][c+1]) -- the whole bilinear footprint of a sample point in one
// 16-byte load -- with zeros past the last row and column (pack_quads_kernel
// writes it).  The taper is stored as pairs (w[c], w[c+1]).  The volume is
// [z][y][x], x fastest.
//
// Work split.  A CTA is 32 x 8 threads over (x, y); each thread owns ZPT
// consecutive slices of its (x, y) column and keeps (sum, weight) pairs in
// registers across all views of the launch, so a launch covering every view
// stores the volume once and never reads it.
//
// Arithmetic.  U, V are formed exactly as BPCore rounds them.  The quotients
// are computed as a pair (packed f32x2) from one correctly
// rounded reciprocal r = RN(1/W) and Markstein's correction q = RN(q0 + RN(U -
// W q0) r), q0 = RN(U r), which yields RN(U / W); when P[10] == 0 for every
// view W does not depend on z (BPCore adds z*0) and r is computed once per
// (x, y, view).  EXACT additionally rounds the lerps step by step like
// BPCore (every product and sum separately) instead of fusing them.
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

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

// Packed f32x2 arithmetic.  Each lane of a single mul / add / fma rounds like
// the scalar operation, but a packed multiply whose result feeds a packed add
// can be fused into one fma by the compiler (measured on sm_100a with this
// toolchain, for both the intrinsics and inline PTX with .rn), so every
// product that BPCore rounds before adding is computed with scalar
// __fmul_rn / __fadd_rn, which are never contracted.
#define JFDK_PACKED_OP(name, op)                                                              \
    __device__ __forceinline__ float2 name(float2 a, float2 b) {                              \
        float2 d;                                                                             \
        asm("{\n .reg .b64 ra, rb, rd;\n mov.b64 ra, {%2, %3};\n mov.b64 rb, {%4, %5};\n " op \
            " rd, ra, rb;\n mov.b64 {%0, %1}, rd;\n}"                                          \
            : "=f"(d.x), "=f"(d.y)                                                            \
            : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));                                        \
        return d;                                                                             \
    }
JFDK_PACKED_OP(pmul, "mul.rn.f32x2")
JFDK_PACKED_OP(padd, "add.rn.f32x2")
#undef JFDK_PACKED_OP

// a * b + c per lane, one rounding (fma.rn.f32x2).
__device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) {
    float2 d;
    asm("{\n .reg .b64 ra, rb, rc, rd;\n mov.b64 ra, {%2, %3};\n mov.b64 rb, {%4, %5};\n"
        " mov.b64 rc, {%6, %7};\n fma.rn.f32x2 rd, ra, rb, rc;\n mov.b64 {%0, %1}, rd;\n}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return d;
}

template <int ZPT, bool FINALIZE, bool EXACT, bool WZ>
__global__ void __launch_bounds__(256) bp_kernel(BPParams p) {
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    const int zb = p.z_begin + blockIdx.z * ZPT;
    if (x >= p.X || y >= p.Y) return;

    // Axes as BPCore builds them (BPCore.cpp:47-66): (i - (n-1)/2) * pitch.
    const float ax = __fmul_rn(__fadd_rn(-((float)p.X - 1.0f) / 2.0f, (float)x), p.pxy);
    const float ay = __fmul_rn(__fadd_rn(-((float)p.Y - 1.0f) / 2.0f, (float)y), p.pxy);
    float az[ZPT];
    float2 acc[ZPT];  // (sum, weight)
    const size_t plane = (size_t)p.X * p.Y;
    const size_t base = (size_t)y * p.X + x;
#pragma unroll
    for (int k = 0; k < ZPT; ++k) {
        const float a = __fmul_rn(__fadd_rn(-((float)p.Z - 1.0f) / 2.0f, (float)(zb + k)), p.pz);
        az[k] = a;
        const bool in = zb + k < p.z_end;
        acc[k] = (p.load_acc && in) ? f2(p.sum[(size_t)(zb + k) * plane + base], p.cnt[(size_t)(zb + k) * plane + base])
                                    : f2(0.0f, 0.0f);
    }
    const float umax = (float)(p.U - 1), vmax = (float)(p.V - 1), fU = (float)p.U;
    const float2 neg1 = f2(-1.0f, -1.0f);

    for (int view = p.v0; view < p.v0 + p.nv; ++view) {
        const float4* P4 = reinterpret_cast<const float4*>(p.ptm + (size_t)view * 12);
        const float4 r0 = __ldg(P4), r1 = __ldg(P4 + 1), r2 = __ldg(P4 + 2);
        // (XxPM0 + (YxPM1 + PM3), XxPM4 + (YxPM5 + PM7)) and W (BPCore.cpp:120-145)
        const float Uxy = __fadd_rn(__fmul_rn(ax, r0.x), __fadd_rn(__fmul_rn(ay, r0.y), r0.w));
        const float Vxy = __fadd_rn(__fmul_rn(ax, r1.x), __fadd_rn(__fmul_rn(ay, r1.y), r1.w));
        const float Wxy = __fadd_rn(__fmul_rn(ax, r2.x), __fadd_rn(__fmul_rn(ay, r2.y), r2.w));
        const float rxy = WZ ? 0.0f : __frcp_rn(Wxy);
        const float4* __restrict__ q = p.q4 + (size_t)(view - p.view_base) * p.q4_frame;
        const float2* __restrict__ tw = p.tw + (size_t)view * p.U;
#pragma unroll
        for (int k = 0; k < ZPT; ++k) {
            const float2 UV = f2(__fadd_rn(Uxy, __fmul_rn(az[k], r0.z)), __fadd_rn(Vxy, __fmul_rn(az[k], r1.z)));
            float W = Wxy, r = rxy;
            if (WZ) {
                W = __fadd_rn(Wxy, __fmul_rn(az[k], r2.z));
                r = __frcp_rn(W);
            }
            const float2 rr = f2(r, r);
            const float2 q0 = pmul(UV, rr);
            const float2 rem = pfma(f2(-W, -W), q0, UV);           // exact remainder
            float2 uv = padd(pfma(rem, rr, q0), f2(0.5f, 0.5f));
            // Branch-free so the loads of all ZPT slices can be in flight at
            // once: a point off the detector reads quad (0, 0) and adds nothing.
            const bool in = (uv.x >= 0.0f) & (uv.x <= umax) & (uv.y >= 0.0f) & (uv.y <= vmax);
            uv = in ? uv : f2(0.0f, 0.0f);
            const float fu = floorf(uv.x), fv = floorf(uv.y);
            const float2 fxy = pfma(f2(fu, fv), neg1, uv);            // (u - fu, v - fv), exact
            const int idx = __float2int_rz(fmaf(fv, fU, fu));         // exact: < 2^24
            const int ix = __float2int_rz(fu);
            const float4 Q = __ldg(q + idx);
            const float2 w = __ldg(tw + ix);
            const float2 lo = f2(Q.x, Q.y), hi = f2(Q.z, Q.w);       // columns ix, ix + 1
            const float2 d = pfma(lo, neg1, hi);                      // RN(hi - lo)
            float val, c;
            if (EXACT) {
                const float t0 = __fadd_rn(lo.x, __fmul_rn(fxy.x, d.x));
                const float t1 = __fadd_rn(lo.y, __fmul_rn(fxy.x, d.y));
                val = __fadd_rn(t0, __fmul_rn(fxy.y, __fsub_rn(t1, t0)));
                c = __fadd_rn(w.x, __fmul_rn(fxy.x, __fsub_rn(w.y, w.x)));
            } else {
                const float2 t = pfma(f2(fxy.x, fxy.x), d, lo);
                val = fmaf(fxy.y, t.y - t.x, t.x);
                c = fmaf(fxy.x, w.y - w.x, w.x);
            }
            if (in) acc[k] = padd(acc[k], f2(val, c));
        }
    }

#pragma unroll
    for (int k = 0; k < ZPT; ++k) {
        if (zb + k >= p.z_end) break;
        const size_t idx = (size_t)(zb + k) * plane + base;
        if (FINALIZE) {
            float o = __fdiv_rn(acc[k].x, acc[k].y);   // BPCore::DoneSlice
            if (p.apply_ct) o = ct_number(o, p.ct_scale, p.ct_norm1);
            if (p.out) p.out[idx] = o;
            if (p.out16) p.out16[idx] = to_i16(o);
        } else {
            p.sum[idx] = acc[k].x;
            p.cnt[idx] = acc[k].y;
        }
    }
}

// Filtered frames -> tapered quads.  One thread per (row, column) of a frame:
// (w[c] p[r][c], w[c] p[r+1][c], w[c+1] p[r][c+1], w[c+1] p[r+1][c+1]), the
// products rounded as InitView's in-place multiply (BPCore.cpp:147-151).
__global__ void __launch_bounds__(256) pack_quads_kernel(const float* __restrict__ plain, long long plain_frame,
                                                         int rows, int U, const float2* __restrict__ tw,
                                                         int view0, int num_views, int apply_taper,
                                                         float4* __restrict__ q4, long long q4_frame, int slot0) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y, f = blockIdx.z;
    if (c >= U) return;
    const float* s = plain + (size_t)f * plain_frame + (size_t)r * U + c;
    const bool right = c + 1 < U, down = r + 1 < rows;
    float p00 = s[0], p01 = right ? s[1] : 0.0f;
    float p10 = down ? s[U] : 0.0f, p11 = (right && down) ? s[U + 1] : 0.0f;
    if (apply_taper) {
        const float2 w = tw[(size_t)((view0 + f) % num_views) * U + c];
        p00 = __fmul_rn(p00, w.x); p10 = __fmul_rn(p10, w.x);
        p01 = __fmul_rn(p01, w.y); p11 = __fmul_rn(p11, w.y);
    }
    q4[(size_t)(slot0 + f) * q4_frame + (size_t)r * U + c] = make_float4(p00, p10, p01, p11);
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

template <int ZPT, bool F, bool E, bool WZ>
cudaError_t go(const BPParams& p, cudaStream_t s) {
    const int nz = p.z_end - p.z_begin;
    dim3 grid((p.X + 31) / 32, (p.Y + 7) / 8, (nz + ZPT - 1) / ZPT);
    bp_kernel<ZPT, F, E, WZ><<<grid, dim3(32, 8), 0, s>>>(p);
    return cudaGetLastError();
}

template <int ZPT, bool F, bool E>
cudaError_t go2(const BPParams& p, bool wz, cudaStream_t s) {
    return wz ? go<ZPT, F, E, true>(p, s) : go<ZPT, F, E, false>(p, s);
}

template <bool F, bool E>
cudaError_t go3(const BPParams& p, bool wz, int zpt, cudaStream_t s) {
    switch (zpt) {
        case 16: return go2<16, F, E>(p, wz, s);
        case 8: return go2<8, F, E>(p, wz, s);
        default: return go2<4, F, E>(p, wz, s);
    }
}

}  // namespace

cudaError_t launch_bp(const BPParams& p, bool finalize, bool exact, bool w_depends_on_z, int zpt, cudaStream_t s) {
    if (finalize) return exact ? go3<true, true>(p, w_depends_on_z, zpt, s) : go3<true, false>(p, w_depends_on_z, zpt, s);
    return exact ? go3<false, true>(p, w_depends_on_z, zpt, s) : go3<false, false>(p, w_depends_on_z, zpt, s);
}

cudaError_t launch_pack_quads(const float* plain, long long plain_frame, int nv, int rows, int U, const float2* tw,
                              int view0, int num_views, int apply_taper, float4* q4, long long q4_frame, int slot0,
                              cudaStream_t s) {
    dim3 grid((U + 255) / 256, rows, nv);
    pack_quads_kernel<<<grid, 256, 0, s>>>(plain, plain_frame, rows, U, tw, view0, num_views, apply_taper, q4,
                                           q4_frame, slot0);
    return cudaGetLastError();
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
