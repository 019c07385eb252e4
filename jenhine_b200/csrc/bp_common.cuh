// bp_common.cuh -- device helpers shared by the backprojector (bp.cu) and its
// adjoint / geometry gradient (adjoint.cu): packed f32x2 arithmetic, the
// floor trick, CT numbers, and the sample coordinates of the FP32 form, so the
// adjoint sees exactly the forward's sample points and in-range decisions.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

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
JFDK_PACKED_OP(psub, "sub.rn.f32x2")
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

// add.rm.f32x2: the lanewise sum rounded toward -infinity.
__device__ __forceinline__ float2 padd_rm(float2 a, float2 b) {
    float2 d;
    asm("{\n .reg .b64 ra, rb, rd;\n mov.b64 ra, {%2, %3};\n mov.b64 rb, {%4, %5};\n"
        " add.rm.f32x2 rd, ra, rb;\n mov.b64 {%0, %1}, rd;\n}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}

// Floor without the conversion unit: for 0 <= x < 2^23 the sum 2^23 + x has
// a unit in the last place of 1, so rounding it toward -infinity gives
// 2^23 + floor(x) exactly; its bit pattern minus that of 2^23 is floor(x) as
// an integer, and subtracting 2^23 back gives floor(x) as a float.
constexpr float kMagic = 8388608.0f;   // 2^23
constexpr int kMagicBits = 0x4B000000;  // bit pattern of 2^23

// Sample point of the FP32 form, as BPCore rounds it (BPCore.cpp:120-145,
// 207-220): Uxy = x*P0 + (y*P1 + P3), likewise V, W; U = Uxy + z*P2 etc.,
// every product and sum rounded separately; u = RN(U / W) + 0.5 from one
// correctly rounded reciprocal r = RN(1/W) and Markstein's correction
// q = RN(q0 + RN(U - W q0) r), q0 = RN(U r).
struct XYTerms { float U, V, W; };

__device__ __forceinline__ XYTerms bp_xy_terms(float ax, float ay, const float4& r0, const float4& r1,
                                               const float4& r2) {
    XYTerms t;
    t.U = __fadd_rn(__fmul_rn(ax, r0.x), __fadd_rn(__fmul_rn(ay, r0.y), r0.w));
    t.V = __fadd_rn(__fmul_rn(ax, r1.x), __fadd_rn(__fmul_rn(ay, r1.y), r1.w));
    t.W = __fadd_rn(__fmul_rn(ax, r2.x), __fadd_rn(__fmul_rn(ay, r2.y), r2.w));
    return t;
}

// RN(1/w) from the approximate reciprocal (rcp.approx, at most 1 ulp off)
// and one Newton-Raphson step with a fused residual, y' = RN(y + y RN(1 - w y))
// (Markstein, IBM J. Res. Dev. 34(1), 1990).  Equal to __frcp_rn for every
// float w whose reciprocal is a normal float, both signs (all 4.2e9 of them,
// tests/cuda/reciprocal_check.cu); W of a voxel lies far inside that range.
__device__ __forceinline__ float rcp_rn_nr(float w) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(w));
    return fmaf(fmaf(-w, y, 1.0f), y, y);
}

// W and r = RN(1/W) at slice coordinate az (W independent of z unless WZ).
template <bool WZ>
__device__ __forceinline__ float2 bp_w_r(const XYTerms& t, float rxy, float az, float P10) {
    if (WZ) {
        const float W = __fadd_rn(t.W, __fmul_rn(az, P10));
        return f2(W, rcp_rn_nr(W));
    }
    return f2(t.W, rxy);
}

__device__ __forceinline__ float2 bp_uv(const XYTerms& t, float2 wr, float az, float P2, float P6) {
    const float2 UV = f2(__fadd_rn(t.U, __fmul_rn(az, P2)), __fadd_rn(t.V, __fmul_rn(az, P6)));
    const float2 rr = f2(wr.y, wr.y);
    const float2 q0 = pmul(UV, rr);
    const float2 rem = pfma(f2(-wr.x, -wr.x), q0, UV);           // exact remainder
    return padd(pfma(rem, rr, q0), f2(0.5f, 0.5f));
}

// The BPCore axis value (i - (n-1)/2) * pitch (BPCore.cpp:47-66).
__device__ __forceinline__ float bp_axis(int i, int n, float pitch) {
    return __fmul_rn(__fadd_rn(-((float)n - 1.0f) / 2.0f, (float)i), pitch);
}

}  // namespace
}  // namespace jfdk
