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
// every view, row r and column c one float4 (p[r][c], p[r+1][c],
// RN(p[r][c+1] - p[r][c]), RN(p[r+1][c+1] - p[r+1][c])) -- the whole bilinear
// footprint of a sample point in one 16-byte load, with the column
// differences BPCore's lerp rounds already formed -- with zeros past the last
// row and column (pack_quads_kernel writes it).  The taper is stored as pairs
// (w[c], RN(w[c+1] - w[c])), w[U] = 0.  The volume is [z][y][x], x fastest.
//
// Work split.  A CTA is 128 threads over (x, y), TX x (128 / TX) (4 x 32 by
// default, 8 x 16 or 32 x 4 by option or autotuner); each thread owns ZPT
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

#include <algorithm>
#include <cstdint>

#include "bp_common.cuh"
#include "jfdk_internal.h"

namespace jfdk {
namespace {

constexpr int kBPThreads = kBPTileX * kBPTileY;

// Resident CTAs per SM the compiler must allow for, with 8 slices per
// thread: the mixed form fits 64 registers at 32 warps per SM (8 CTAs), which
// measured faster than 80 registers at 24 warps (102 vs 120 ms on c2); the
// FP32 form measured the other way round (160.6 ms at 80 registers and 24
// warps against 164.0 ms at 64 and 32).  Small CTAs (4 warps) measured 4 %
// faster than 8-warp ones: a finishing CTA leaves fewer warps idle while the
// SM waits for the next.  Each warp covers 4 x 8 voxels in (x, y) rather than
// a row of 32: its sample points spread less on the detector (1.5-1.7 %
// faster than 32 x 1 in both forms).  The mixed form with 16 slices per
// thread (its default tile on large volumes when W does not depend on z)
// halves the per-view
// work per sample and fits 96 registers at 20 warps per SM: 88.0 ms on c2
// against 88.9 at 80 registers and 24 warps and 93.6 with 8 slices.
constexpr int bp_min_blocks(int zpt) { return zpt == 8 ? 1024 / kBPThreads : zpt == 16 ? 5 : 1; }
constexpr int bp_fp32_min_blocks(int zpt) { return zpt == 8 ? 6 : 1; }

// Where a CTA's tile lies: the launch grid's block index for the per-scan
// kernels, the current work item of the batch kernel.  The tile bodies ask
// for it at the start and again after the view loop: the batch kernel's
// tile is re-read from shared memory then rather than held in registers
// through the loop (at the 64-register bound that made the FP32 body spill).
// GridTile reads the block index with volatile moves, so the compiler reads
// it again after the loop instead of keeping x, y and z live through it:
// with the W(z) mixed body's U, V, W stepped per slice, that removed its
// spills (12 bytes stored, 360 bytes of reloads) and made it 6.5 % faster
// on a tilted c2 orbit; the FP32 kernels ran 0.8 % faster on c2.  The mixed
// body with z-independent W measured 1 % slower with it and keeps the plain
// read (GridTileHeld).  TX is the tile's width in x (threads along x); the
// CTA is TX x (128 / TX) threads, each warp 32 consecutive threads of it.
template <int TX>
struct GridTile {
    static constexpr int kX = TX, kY = kBPThreads / TX;
    __device__ static int ctaid(int d) {
        unsigned r;
        if (d == 0) asm volatile("mov.u32 %0, %%ctaid.x;" : "=r"(r));
        else if (d == 1) asm volatile("mov.u32 %0, %%ctaid.y;" : "=r"(r));
        else asm volatile("mov.u32 %0, %%ctaid.z;" : "=r"(r));
        return (int)r;
    }
    __device__ int bx() const { return ctaid(0); }
    __device__ int by() const { return ctaid(1); }
    __device__ int bz() const { return ctaid(2); }
};

template <int TX>
struct GridTileHeld {
    static constexpr int kX = TX, kY = kBPThreads / TX;
    __device__ int bx() const { return blockIdx.x; }
    __device__ int by() const { return blockIdx.y; }
    __device__ int bz() const { return blockIdx.z; }
};

__shared__ unsigned g_batch_tile;   // the batch kernel's current work item

struct BatchTile {
    static constexpr int kX = kBPTileX, kY = kBPTileY;
    const BatchScan& b;
    __device__ unsigned local() const { return *static_cast<volatile unsigned*>(&g_batch_tile) - b.first_tile; }
    __device__ int bx() const { return (int)(local() % (unsigned)b.gx); }
    __device__ int by() const { return (int)((local() / (unsigned)b.gx) % (unsigned)b.gy); }
    __device__ int bz() const { return (int)(local() / ((unsigned)b.gx * (unsigned)b.gy)); }
};

// The tile's (sum, weight) pairs: normalised, CT numbers, stored (FINALIZE),
// or stored as accumulators.  The coordinates are asked for again here.
// WV: the weights come from p.wvol (the whole volume, absolute slices).
template <int ZPT, bool FINALIZE, class Tile, bool WV = false>
__device__ __forceinline__ void epilogue(const BPParams& p, const Tile& tile, const float2 (&acc)[ZPT]) {
    const int x = tile.bx() * Tile::kX + threadIdx.x;
    const int y = tile.by() * Tile::kY + threadIdx.y;
    const int zb = p.z_begin + tile.bz() * ZPT;
#pragma unroll
    for (int k = 0; k < ZPT; ++k) {
        if (zb + k >= p.z_end) break;
        if (FINALIZE) {
            const size_t idx = ((size_t)(zb + k - p.out_z0) * p.Y + y) * p.X + x;
            const float wsum = WV ? __ldg(p.wvol + ((size_t)(zb + k) * p.Y + y) * p.X + x) : acc[k].y;
            float o = __fdiv_rn(acc[k].x, wsum);   // BPCore::DoneSlice
            if (p.apply_ct) o = ct_number(o, p.ct_scale, p.ct_norm1);
            if (p.out) p.out[idx] = o;
            if (p.out16) p.out16[idx] = to_i16(o);
        } else {
            const size_t idx = ((size_t)(zb + k - p.acc_z0) * p.Y + y) * p.X + x;
            p.sum[idx] = acc[k].x;
            p.cnt[idx] = acc[k].y;
        }
    }
}

// WV: the normalisation weights come from p.wvol (finalize over every view):
// the view loop loads and accumulates only the projection samples.
// WEIGHTS: the loop accumulates only the weights and stores them to out at
// absolute slices (launch_bp_weights).
template <int ZPT, bool FINALIZE, bool EXACT, bool WZ, class Tile, bool WV = false, bool WEIGHTS = false>
__device__ __forceinline__ void bp_block(const BPParams& p, const Tile& tile, float* wout = nullptr) {
    const int x = tile.bx() * Tile::kX + threadIdx.x;
    const int y = tile.by() * Tile::kY + threadIdx.y;
    const int zb = p.z_begin + tile.bz() * ZPT;
    if (x >= p.X || y >= p.Y) return;

    const float ax = bp_axis(x, p.X, p.pxy), ay = bp_axis(y, p.Y, p.pxy);
    float az[ZPT];
    float2 acc[ZPT];  // (sum, weight)
#pragma unroll
    for (int k = 0; k < ZPT; ++k) {
        az[k] = bp_axis(zb + k, p.Z, p.pz);
        acc[k] = f2(0.0f, 0.0f);
        if (!FINALIZE && p.load_acc && zb + k < p.z_end) {
            const size_t i = ((size_t)(zb + k - p.acc_z0) * p.Y + y) * p.X + x;
            acc[k] = f2(p.sum[i], p.cnt[i]);
        }
    }
    const unsigned umax_bits = __float_as_uint((float)(p.U - 1)), vmax_bits = __float_as_uint((float)(p.V - 1));

    // Pointers step from view to view (index arithmetic on v0 and view_base
    // inside the loop measured over 10% slower at the 64-register bound).
    const float4* P4 = reinterpret_cast<const float4*>(p.ptm + (size_t)p.v0 * 12);
    const float4* __restrict__ q = p.q4 + (size_t)(p.v0 - p.view_base) * p.q4_frame;
    const float2* __restrict__ tw = p.tw + (size_t)p.v0 * p.U;
#pragma unroll 1
    for (int n = 0; n < p.nv; ++n, P4 += 3, q += p.q4_frame, tw += p.U) {
        const float4 r0 = __ldg(P4), r1 = __ldg(P4 + 1), r2 = __ldg(P4 + 2);
        const XYTerms xy = bp_xy_terms(ax, ay, r0, r1, r2);
        const float rxy = WZ ? 0.0f : rcp_rn_nr(xy.W);
#pragma unroll
        for (int k = 0; k < ZPT; ++k) {
            float2 uv = bp_uv(xy, bp_w_r<WZ>(xy, rxy, az[k], r2.z), az[k], r0.z, r1.z);
            // Branch-free so the loads of all ZPT slices can be in flight at
            // once: a point off the detector reads quad (0, 0) and adds nothing.
            // 0 <= u <= umax on the bit patterns: non-negative floats order like
            // their bits, negatives and NaN have larger unsigned patterns (u is
            // never -0: RN(U / W) + 0.5 rounds an exact zero to +0)
            const bool in = (__float_as_uint(uv.x) <= umax_bits) & (__float_as_uint(uv.y) <= vmax_bits);
            uv = in ? uv : f2(0.0f, 0.0f);
            const float2 t = padd_rm(uv, f2(kMagic, kMagic));         // 2^23 + floor(uv)
            const float2 fxy = psub(uv, psub(t, f2(kMagic, kMagic)));  // (u - fu, v - fv), exact
            const int ix = __float_as_int(t.x) - kMagicBits;
            const int idx = (__float_as_int(t.y) - kMagicBits) * p.U + ix;
            float val = 0.0f, c = 0.0f;
            if constexpr (!WEIGHTS) {
                const float4 Q = __ldg(q + idx);
                const float2 lo = f2(Q.x, Q.y), d = f2(Q.z, Q.w);    // column ix, RN(column ix+1 - ix)
                if (EXACT) {
                    const float t0 = __fadd_rn(lo.x, __fmul_rn(fxy.x, d.x));
                    const float t1 = __fadd_rn(lo.y, __fmul_rn(fxy.x, d.y));
                    val = __fadd_rn(t0, __fmul_rn(fxy.y, __fsub_rn(t1, t0)));
                } else {
                    const float2 t = pfma(f2(fxy.x, fxy.x), d, lo);
                    val = fmaf(fxy.y, t.y - t.x, t.x);
                }
            }
            if constexpr (!WV) {
                const float2 w = __ldg(tw + ix);
                c = EXACT ? __fadd_rn(w.x, __fmul_rn(fxy.x, w.y)) : fmaf(fxy.x, w.y, w.x);
            }
            if (in) {   // the same roundings as the packed add of (val, c)
                if constexpr (WV) acc[k].x = __fadd_rn(acc[k].x, val);
                else if constexpr (WEIGHTS) acc[k].y = __fadd_rn(acc[k].y, c);
                else acc[k] = padd(acc[k], f2(val, c));
            }
        }
    }

    if constexpr (WEIGHTS) {
#pragma unroll
        for (int k = 0; k < ZPT; ++k)
            if (zb + k < p.z_end) wout[((size_t)(zb + k) * p.Y + y) * p.X + x] = acc[k].y;
        return;
    }
    // The output index is formed here, not before the view loop, so that it
    // holds no registers across the loop.
    epilogue<ZPT, FINALIZE, Tile, WV>(p, tile, acc);
}

// ---- mixed precision ---------------------------------------------------------
// Record per (slot, row r, column c), 8 bytes, the tapered footprint
// p00 = p[r][c], p01 = p[r][c+1], p10 = p[r+1][c], p11 = p[r+1][c+1] divided
// by the view's power-of-two scale s, in FP16, as the coefficients of the
// bilinear form  val = p00 + fx dx + fy (dy + fx dxy):
//   .x  half2 (p00, dx = p01 - p00)
//   .y  half2 (dy = p10 - p00, dxy = p11 - p10 - p01 + p00)
// each difference rounded against the already rounded coefficients, so every
// corner the form reproduces carries the rounding of one coefficient only.
// The records of the last row and the last column are zero: their samples
// are not taken (below), and an index clamped onto them reads nothing.
// The interpolation is two FP16 x FP16 + FP32 fused multiply-adds
// (fma.rn.f32.f16, products exact in FP32) and one FP32 one.
// The coordinates use an approximate reciprocal of W and fused
// multiply-adds; when W does not depend on z the slices of a thread are
// equally spaced on the detector and u, v advance by a constant per slice.
// A sample is taken when floor(u) <= cols-2 and floor(v) <= rows-2 (the
// same set as 0 <= u <= cols-1, 0 <= v <= rows-1 up to the measure-zero
// points u = cols-1, v = rows-1) and W > 0.  The lerps, the rescale by s and
// the (sum, weight) accumulation are FP32; the weight is the FP32 taper
// pair's lerp at the sample's FP32 fraction.
// WV: the weights come from p.wvol (finalize over every view), so the loop
// clamps the index onto the zero records instead of testing the range and
// loads one record per sample.  WEIGHTS: the loop accumulates only the
// weights and stores them to out at absolute slices.
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// p00 + fx dx + fy (dy + fx dxy) of an 8-byte record (fx rounded to FP16).
__device__ __forceinline__ float mixed_lerp(uint2 rec, float2 f) {
    float v1, inner;
    asm("{\n .reg .f16 p0, dx, dy, dxy, fh;\n .reg .f32 p0f, dyf;\n"
        " mov.b32 {p0, dx}, %2;\n mov.b32 {dy, dxy}, %3;\n"
        " cvt.rn.f16.f32 fh, %4;\n cvt.f32.f16 p0f, p0;\n cvt.f32.f16 dyf, dy;\n"
        " fma.rn.f32.f16 %0, fh, dx, p0f;\n fma.rn.f32.f16 %1, fh, dxy, dyf;\n}"
        : "=f"(v1), "=f"(inner)
        : "r"(rec.x), "r"(rec.y), "f"(f.x));
    return fmaf(f.y, inner, v1);
}

template <int ZPT, bool FINALIZE, bool WZ, class Tile, bool WV = false, bool WEIGHTS = false>
__device__ __forceinline__ void bp_mixed_block(const BPParams& p, const Tile& tile, float* wout = nullptr) {
    const int x = tile.bx() * Tile::kX + threadIdx.x;
    const int y = tile.by() * Tile::kY + threadIdx.y;
    const int zb = p.z_begin + tile.bz() * ZPT;
    if (x >= p.X || y >= p.Y) return;
    // every rounding explicit, so that each kernel built from this body
    // (per-scan, batch, weights) forms the same coordinates
    const float ax = __fmul_rn(__fadd_rn((float)x, -0.5f * (float)(p.X - 1)), p.pxy);
    const float ay = __fmul_rn(__fadd_rn((float)y, -0.5f * (float)(p.Y - 1)), p.pxy);
    const float az0 = __fmul_rn(__fadd_rn((float)zb, -0.5f * (float)(p.Z - 1)), p.pz);
    float2 acc[ZPT];  // (sum, weight)
#pragma unroll
    for (int k = 0; k < ZPT; ++k) {
        acc[k] = f2(0.0f, 0.0f);
        if (!FINALIZE && p.load_acc && zb + k < p.z_end) {
            const size_t i = ((size_t)(zb + k - p.acc_z0) * p.Y + y) * p.X + x;
            acc[k] = f2(p.sum[i], p.cnt[i]);
        }
    }
    const unsigned um1 = (unsigned)(p.U - 1), vm1 = (unsigned)(p.V - 1), uu = (unsigned)p.U;
    const float2 magic = f2(kMagic, kMagic);

    const float4* P4 = reinterpret_cast<const float4*>(p.ptm + (size_t)p.v0 * 12);
    const float* sc = p.qscale + p.v0;
    const uint2* __restrict__ q = p.qh + (size_t)(p.v0 - p.view_base) * p.q4_frame;
    const float2* __restrict__ tw = p.tw + (size_t)p.v0 * p.U;
#pragma unroll 2   // two views in flight: 93.6 against 97.7 ms on c2 (unrolling the FP32 loop spills)
    for (int n = 0; n < p.nv; ++n, P4 += 3, ++sc, q += p.q4_frame, tw += p.U) {
        const float4 r0 = __ldg(P4), r1 = __ldg(P4 + 1), r2 = __ldg(P4 + 2);
        const float2 P26 = f2(r0.z, r1.z);
        // U, V, W at slice zb
        const float2 UV0 = pfma(f2(az0, az0), P26,
                                pfma(f2(ax, ax), f2(r0.x, r1.x), pfma(f2(ay, ay), f2(r0.y, r1.y), f2(r0.w, r1.w))));
        const float W0 = fmaf(az0, r2.z, fmaf(ax, r2.x, fmaf(ay, r2.y, r2.w)));
        if (!WZ && !(W0 > 0.0f)) continue;   // a point at or behind the source plane samples nothing
        // !WZ: (u, v) itself steps from slice to slice.  WZ: U, V and W step
        // (one add each per slice, no per-slice offsets held through the loop)
        float2 uv = f2(0.f, 0.f), duv = f2(0.f, 0.f), UVk = UV0;
        float Wk = W0, dW = 0.f;
        if (!WZ) {
            const float r = rcp_approx(W0);
            uv = pfma(UV0, f2(r, r), f2(0.5f, 0.5f));
            const float rz = __fmul_rn(r, p.pz);
            duv = f2(__fmul_rn(P26.x, rz), __fmul_rn(P26.y, rz));
        } else {
            duv = f2(__fmul_rn(P26.x, p.pz), __fmul_rn(P26.y, p.pz));
            dW = __fmul_rn(p.pz, r2.z);
        }
        // (scalar products: a packed product feeding the packed adds below
        // may be fused into them, differently in each kernel built from here)
        const float s = __ldg(sc);
#pragma unroll
        for (int k = 0; k < ZPT; ++k) {
            float2 cuv;
            bool front = true;
            if (WZ) {
                const float r = rcp_approx(Wk);
                front = Wk > 0.0f;
                cuv = pfma(UVk, f2(r, r), f2(0.5f, 0.5f));
                UVk = padd(UVk, duv);
                Wk = __fadd_rn(Wk, dW);
            } else {
                cuv = uv;              // slice k: uv0 + k duv, stepped
                uv = padd(uv, duv);
            }
            const float2 t = padd_rm(cuv, magic);                     // 2^23 + floor(uv)
            const float2 f = psub(cuv, psub(t, magic));               // fractions
            const unsigned iu = __float_as_uint(t.x) - (unsigned)kMagicBits;
            const unsigned iv = __float_as_uint(t.y) - (unsigned)kMagicBits;
            if constexpr (WV) {
                // out of range (negative / NaN wrap to large): a zero record
                const float val = mixed_lerp(__ldg(q + (min(iv, vm1) * uu + min(iu, um1))), f);
                if (front) acc[k].x = fmaf(s, val, acc[k].x);
            } else {
                const bool in = (iu < um1) & (iv < vm1) & front;
                const float2 w = __ldg(tw + (in ? iu : 0u));
                const float c = fmaf(f.x, w.y, w.x);
                if constexpr (WEIGHTS) {
                    if (in) acc[k].y = __fadd_rn(acc[k].y, c);
                } else {
                    const float val = mixed_lerp(__ldg(q + (in ? iv * uu + iu : 0u)), f);
                    if (in) acc[k] = pfma(f2(s, 1.0f), f2(val, c), acc[k]);   // (s val + sum, c + weight)
                }
            }
        }
    }
    if constexpr (WEIGHTS) {
#pragma unroll
        for (int k = 0; k < ZPT; ++k)
            if (zb + k < p.z_end) wout[((size_t)(zb + k) * p.Y + y) * p.X + x] = acc[k].y;
        return;
    }
    epilogue<ZPT, FINALIZE, Tile, WV>(p, tile, acc);
}

// One CTA = one TX x (128 / TX) x ZPT voxel tile of one launch's grid.
template <int ZPT, bool FINALIZE, bool EXACT, bool WZ, int TX, bool WV = false>
__global__ void __launch_bounds__(kBPThreads, bp_fp32_min_blocks(ZPT)) bp_kernel(BPParams p) {
    bp_block<ZPT, FINALIZE, EXACT, WZ, GridTile<TX>, WV>(p, GridTile<TX>{});
}

template <int ZPT, bool EXACT, bool WZ, int TX>
__global__ void __launch_bounds__(kBPThreads, bp_fp32_min_blocks(ZPT)) bp_weights_kernel(BPParams p, float* out) {
    bp_block<ZPT, true, EXACT, WZ, GridTile<TX>, false, true>(p, GridTile<TX>{}, out);
}

template <int ZPT, bool FINALIZE, bool WZ, int TX, bool WV = false>
__global__ void __launch_bounds__(kBPThreads, bp_min_blocks(ZPT)) bp_mixed_kernel(BPParams p) {
    if constexpr (WZ)
        bp_mixed_block<ZPT, FINALIZE, WZ, GridTile<TX>, WV>(p, GridTile<TX>{});
    else
        bp_mixed_block<ZPT, FINALIZE, WZ, GridTileHeld<TX>, WV>(p, GridTileHeld<TX>{});
}

// (once per geometry; with 16 slices at 128 registers, which the weights'
// taper lerps fill without spilling)
template <int ZPT, bool WZ, int TX>
__global__ void __launch_bounds__(kBPThreads, ZPT == 16 ? 4 : bp_min_blocks(ZPT))
    bp_mixed_weights_kernel(BPParams p, float* out) {
    bp_mixed_block<ZPT, true, WZ, GridTile<TX>, false, true>(p, GridTile<TX>{}, out);
}

// Persistent backprojection over the tiles of up to kBatchSlots scans: each
// CTA takes the next tile of the launch's work list (scans in order, tiles
// of a scan in the grid order x, y, z) until the list is exhausted, so the
// tail of one scan runs beside the start of the next.  Each scan's
// parameters sit at a fixed offset of the kernel's parameter space (slot S,
// a compile-time index), so the tile body reads them as constant operands
// exactly as the single-scan kernels do; a shared-memory or indexed copy of
// them measured 16-27 % slower at the 64-register bound.  Each slot holds its
// scan's own tile depth (4 or 8 slices, a uniform branch per tile), so scans
// tuned to either depth share the launch.  DEEP: a launch of the mixed
// form's 16-slice tiles only, at that body's register bound (96 registers;
// the 4- and 8-slice bodies run at 64).  The next tile's index is fetched
// while the current one runs.
// WV: every scan of the launch divides by its weight volume (p.wvol).
template <int S, bool MIXED, bool WZ, bool WV, bool DEEP>
__device__ __forceinline__ void batch_slot_tile(const BatchSlots& t) {
    const BatchTile tile{t.s[S]};
    if constexpr (DEEP) {
        static_assert(MIXED, "16-slice batch tiles are the mixed form's");
        bp_mixed_block<16, true, WZ, BatchTile, WV>(t.s[S].p, tile);
    } else if (t.s[S].zpt == 8) {
        if (MIXED)
            bp_mixed_block<8, true, WZ, BatchTile, WV>(t.s[S].p, tile);
        else
            bp_block<8, true, false, WZ, BatchTile, WV>(t.s[S].p, tile);
    } else {
        if (MIXED)
            bp_mixed_block<4, true, WZ, BatchTile, WV>(t.s[S].p, tile);
        else
            bp_block<4, true, false, WZ, BatchTile, WV>(t.s[S].p, tile);
    }
}

// The tile of slot si (si < kBatchSlots): a compile-time slot per case.
template <int S, bool MIXED, bool WZ, bool WV, bool DEEP>
__device__ __forceinline__ void batch_dispatch(const BatchSlots& t, int si) {
    if constexpr (S < kBatchSlots) {
        if (si == S)
            batch_slot_tile<S, MIXED, WZ, WV, DEEP>(t);
        else
            batch_dispatch<S + 1, MIXED, WZ, WV, DEEP>(t, si);
    }
}

template <bool MIXED, bool WZ, bool WV, bool DEEP>
__global__ void __launch_bounds__(kBPThreads, DEEP    ? bp_min_blocks(16)
                                              : MIXED ? bp_min_blocks(8)
                                                      : bp_fp32_min_blocks(8))
    bp_batch_kernel(const __grid_constant__ BatchSlots t, int nscans, unsigned* __restrict__ counter,
                    unsigned total) {
    __shared__ unsigned s_next;
    const int tid = threadIdx.y * kBPTileX + threadIdx.x;
    if (tid == 0) g_batch_tile = atomicAdd(counter, 1u);
    __syncthreads();
    for (;;) {
        const unsigned it = *static_cast<volatile unsigned*>(&g_batch_tile);
        if (it >= total) break;
        if (tid == 0) s_next = atomicAdd(counter, 1u);   // the next tile, while this one runs
        int si = 0;
        while (si + 1 < nscans && it >= t.s[si + 1].first_tile) ++si;
        batch_dispatch<0, MIXED, WZ, WV, DEEP>(t, si);
        __syncthreads();   // every thread is done with the current tile
        if (tid == 0) g_batch_tile = s_next;
        __syncthreads();
    }
}

// Largest |value| of each frame as float bits; for non-negative floats the
// bit patterns order like the values, so an integer atomicMax reduces them.
// out[] must be zero before the launch.
__global__ void __launch_bounds__(256) frame_absmax_kernel(const float* __restrict__ plain, long long frame,
                                                           unsigned* __restrict__ out) {
    const float* fr = plain + (size_t)blockIdx.y * frame;
    float m = 0.0f;
    for (long long i = blockIdx.x * 256LL + threadIdx.x; i < frame; i += (long long)gridDim.x * 256)
        m = fmaxf(m, fabsf(__ldg(fr + i)));   // fmaxf drops NaN operands
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out + blockIdx.y, __float_as_uint(m));
}

// Power-of-two scale of a view: max |q| / s lies in [2^12, 2^13), so every
// coefficient of the bilinear form (|dxy| < 4 max) stays inside the FP16
// range (65504), and dividing by s is exact.  An all-zero (or non-finite)
// view gets 1.
__device__ __forceinline__ float view_scale(unsigned maxbits) {
    const float m = __uint_as_float(maxbits);
    if (!(m > 0.0f) || !(m <= 3.0e38f)) return 1.0f;
    return ldexpf(1.0f, ilogbf(m) - 12);
}

// Filtered frames -> mixed-precision records in slots [slot0, slot0 + nv),
// tapered with the taper of rotation view (view0 + f) mod num_views; writes
// that view's scale to scale[view].
__global__ void __launch_bounds__(256) pack_mixed_kernel(const float* __restrict__ plain, long long plain_frame,
                                                         int rows, int U, const float2* __restrict__ tw, int view0,
                                                         int num_views, const unsigned* __restrict__ absmax,
                                                         float* __restrict__ scale, uint2* __restrict__ qh,
                                                         long long q_frame, int slot0) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y, f = blockIdx.z;
    if (c >= U) return;
    const int view = (view0 + f) % num_views;
    const float s = view_scale(absmax[f]);
    const float inv = __fdiv_rn(1.0f, s);
    if (r == 0 && c == 0) scale[view] = s;
    uint2 rec = make_uint2(0u, 0u);   // the last row and column: samples not taken
    if (c + 1 < U && r + 1 < rows) {
        const float* src = plain + (size_t)f * plain_frame + (size_t)r * U + c;
        const float w0 = tw[(size_t)view * U + c].x, w1 = tw[(size_t)view * U + c + 1].x;
        // the tapered footprint over the view's scale (exact: inv a power of two)
        const float a = (src[0] * w0) * inv, b = (src[1] * w1) * inv;
        const float cc = (src[U] * w0) * inv, d = (src[U + 1] * w1) * inv;
        const __half hp = __float2half_rn(a);
        const float ap = __half2float(hp);
        const __half hdx = __float2half_rn(b - ap), hdy = __float2half_rn(cc - ap);
        const __half hdxy = __float2half_rn(d - (ap + __half2float(hdx) + __half2float(hdy)));
        const __half2 h1 = __halves2half2(hp, hdx), h2 = __halves2half2(hdy, hdxy);
        rec.x = *reinterpret_cast<const unsigned*>(&h1);
        rec.y = *reinterpret_cast<const unsigned*>(&h2);
    }
    qh[(size_t)(slot0 + f) * q_frame + (size_t)r * U + c] = rec;
}

// Filtered frames -> tapered quads.  One thread per (row, column) of a frame:
// the tapered values w[c] p[r][c], w[c] p[r+1][c], w[c+1] p[r][c+1],
// w[c+1] p[r+1][c+1], each product rounded as InitView's in-place multiply
// (BPCore.cpp:147-151), stored as (t00, t10, RN(t01 - t00), RN(t11 - t10)).
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
        const float2* wv = tw + (size_t)((view0 + f) % num_views) * U;
        const float w0 = wv[c].x, w1 = right ? wv[c + 1].x : 0.0f;
        p00 = __fmul_rn(p00, w0); p10 = __fmul_rn(p10, w0);
        p01 = __fmul_rn(p01, w1); p11 = __fmul_rn(p11, w1);
    }
    q4[(size_t)(slot0 + f) * q4_frame + (size_t)r * U + c] =
        make_float4(p00, p10, __fsub_rn(p01, p00), __fsub_rn(p11, p10));
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
// one frame top to bottom, in place: the previous and current input rows in
// registers, and the next kZRows input rows loaded together before any of
// them is overwritten, so kZRows loads are in flight instead of one (a
// column walked row by row waited out one load latency per row: 349 us per
// 32-view chunk of 768 x 768).
constexpr int kZRows = 16;

__global__ void __launch_bounds__(128) zfilter_kernel(float* frames, int nv, int rows, int width, long long stride,
                                                      int pitch) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x, f = blockIdx.y;
    if (col >= width || f >= nv) return;
    float* c = frames + (size_t)f * stride + col;
    float prev = c[0], cur = c[0];
    for (int r0 = 0; r0 < rows; r0 += kZRows) {
        float nxt[kZRows];
#pragma unroll
        for (int i = 0; i < kZRows; ++i) nxt[i] = c[(size_t)min(r0 + 1 + i, rows - 1) * pitch];
#pragma unroll
        for (int i = 0; i < kZRows; ++i) {
            if (r0 + i >= rows) break;
            float o = __fmul_rn(cur, 0.5f);
            o = __fadd_rn(o, __fmul_rn(prev, 0.25f));
            o = __fadd_rn(o, __fmul_rn(nxt[i], 0.25f));
            c[(size_t)(r0 + i) * pitch] = o;
            prev = cur;
            cur = nxt[i];
        }
    }
}

// The launch grid covers the volume's columns with TX x (128 / TX) tiles and
// the launch's slices with ZPT-deep ones; threads outside the volume return
// at once, slices past z_end are skipped.
template <int TX>
dim3 bp_grid(const BPParams& p, int zpt) {
    constexpr int TY = kBPThreads / TX;
    const int nz = p.z_end - p.z_begin;
    return dim3((p.X + TX - 1) / TX, (p.Y + TY - 1) / TY, (nz + zpt - 1) / zpt);
}

template <int ZPT, bool F, bool E, bool WZ, int TX>
cudaError_t go(const BPParams& p, cudaStream_t s) {
    if constexpr (F) {
        if (p.wvol) {
            bp_kernel<ZPT, F, E, WZ, TX, true><<<bp_grid<TX>(p, ZPT), dim3(TX, kBPThreads / TX), 0, s>>>(p);
            return cudaGetLastError();
        }
    }
    bp_kernel<ZPT, F, E, WZ, TX><<<bp_grid<TX>(p, ZPT), dim3(TX, kBPThreads / TX), 0, s>>>(p);
    return cudaGetLastError();
}

template <int ZPT, bool E, bool WZ>
cudaError_t go_weights(const BPParams& p, int tx, float* out, cudaStream_t s) {
    if constexpr (ZPT != 16) {
        if (tx == 8) {
            bp_weights_kernel<ZPT, E, WZ, 8><<<bp_grid<8>(p, ZPT), dim3(8, kBPThreads / 8), 0, s>>>(p, out);
            return cudaGetLastError();
        }
        if (tx == 32) {
            bp_weights_kernel<ZPT, E, WZ, 32><<<bp_grid<32>(p, ZPT), dim3(32, kBPThreads / 32), 0, s>>>(p, out);
            return cudaGetLastError();
        }
    }
    bp_weights_kernel<ZPT, E, WZ, 4><<<bp_grid<4>(p, ZPT), dim3(4, kBPThreads / 4), 0, s>>>(p, out);
    return cudaGetLastError();
}

template <bool E, bool WZ>
cudaError_t go_weights2(const BPParams& p, int zpt, int tx, float* out, cudaStream_t s) {
    switch (zpt) {
        case 16: return go_weights<16, E, WZ>(p, tx, out, s);
        case 8: return go_weights<8, E, WZ>(p, tx, out, s);
        default: return go_weights<4, E, WZ>(p, tx, out, s);
    }
}

// Tile widths 4, 8 and 32 for the tile depths the autotuner chooses between
// (4 and 8 slices); 16-slice tiles are 4 wide.
template <int ZPT, bool F, bool E, bool WZ>
cudaError_t go_tx(const BPParams& p, int tx, cudaStream_t s) {
    if constexpr (ZPT != 16) {
        if (tx == 8) return go<ZPT, F, E, WZ, 8>(p, s);
        if (tx == 32) return go<ZPT, F, E, WZ, 32>(p, s);
    }
    return go<ZPT, F, E, WZ, 4>(p, s);
}

template <int ZPT, bool F, bool E>
cudaError_t go2(const BPParams& p, bool wz, int tx, cudaStream_t s) {
    return wz ? go_tx<ZPT, F, E, true>(p, tx, s) : go_tx<ZPT, F, E, false>(p, tx, s);
}

template <int ZPT, bool F, bool WZ, int TX>
cudaError_t go_mixed(const BPParams& p, cudaStream_t s) {
    if constexpr (F) {
        if (p.wvol) {
            bp_mixed_kernel<ZPT, F, WZ, TX, true><<<bp_grid<TX>(p, ZPT), dim3(TX, kBPThreads / TX), 0, s>>>(p);
            return cudaGetLastError();
        }
    }
    bp_mixed_kernel<ZPT, F, WZ, TX><<<bp_grid<TX>(p, ZPT), dim3(TX, kBPThreads / TX), 0, s>>>(p);
    return cudaGetLastError();
}

template <int ZPT, bool WZ>
cudaError_t go_mixed_weights(const BPParams& p, int tx, float* out, cudaStream_t s) {
    if constexpr (ZPT != 16) {
        if (tx == 8) {
            bp_mixed_weights_kernel<ZPT, WZ, 8><<<bp_grid<8>(p, ZPT), dim3(8, kBPThreads / 8), 0, s>>>(p, out);
            return cudaGetLastError();
        }
        if (tx == 32) {
            bp_mixed_weights_kernel<ZPT, WZ, 32><<<bp_grid<32>(p, ZPT), dim3(32, kBPThreads / 32), 0, s>>>(p, out);
            return cudaGetLastError();
        }
    }
    bp_mixed_weights_kernel<ZPT, WZ, 4><<<bp_grid<4>(p, ZPT), dim3(4, kBPThreads / 4), 0, s>>>(p, out);
    return cudaGetLastError();
}

template <bool WZ>
cudaError_t go_mixed_weights2(const BPParams& p, int zpt, int tx, float* out, cudaStream_t s) {
    switch (zpt) {
        case 16: return go_mixed_weights<16, WZ>(p, tx, out, s);
        case 8: return go_mixed_weights<8, WZ>(p, tx, out, s);
        default: return go_mixed_weights<4, WZ>(p, tx, out, s);
    }
}

template <int ZPT, bool F, bool WZ>
cudaError_t go_mixed_tx(const BPParams& p, int tx, cudaStream_t s) {
    if constexpr (ZPT != 16) {
        if (tx == 8) return go_mixed<ZPT, F, WZ, 8>(p, s);
        if (tx == 32) return go_mixed<ZPT, F, WZ, 32>(p, s);
    }
    return go_mixed<ZPT, F, WZ, 4>(p, s);
}

template <bool F, bool WZ>
cudaError_t go_mixed2(const BPParams& p, int zpt, int tx, cudaStream_t s) {
    switch (zpt) {
        case 16: return go_mixed_tx<16, F, WZ>(p, tx, s);
        case 8: return go_mixed_tx<8, F, WZ>(p, tx, s);
        default: return go_mixed_tx<4, F, WZ>(p, tx, s);
    }
}

template <bool F, bool E>
cudaError_t go3(const BPParams& p, bool wz, int zpt, int tx, cudaStream_t s) {
    switch (zpt) {
        case 16: return go2<16, F, E>(p, wz, tx, s);
        case 8: return go2<8, F, E>(p, wz, tx, s);
        default: return go2<4, F, E>(p, wz, tx, s);
    }
}

}  // namespace

cudaError_t launch_bp(const BPParams& p, bool finalize, bool exact, bool w_depends_on_z, int zpt, int tile_x,
                      cudaStream_t s) {
    if (finalize)
        return exact ? go3<true, true>(p, w_depends_on_z, zpt, tile_x, s)
                     : go3<true, false>(p, w_depends_on_z, zpt, tile_x, s);
    return exact ? go3<false, true>(p, w_depends_on_z, zpt, tile_x, s)
                 : go3<false, false>(p, w_depends_on_z, zpt, tile_x, s);
}

cudaError_t launch_bp_weights(const BPParams& p, bool exact, bool w_depends_on_z, int zpt, int tile_x, float* out,
                              cudaStream_t s) {
    if (!out || p.v0 != 0) return cudaErrorInvalidValue;
    if (exact)
        return w_depends_on_z ? go_weights2<true, true>(p, zpt, tile_x, out, s)
                              : go_weights2<true, false>(p, zpt, tile_x, out, s);
    return w_depends_on_z ? go_weights2<false, true>(p, zpt, tile_x, out, s)
                          : go_weights2<false, false>(p, zpt, tile_x, out, s);
}

cudaError_t launch_bp_mixed_weights(const BPParams& p, bool w_depends_on_z, int zpt, int tile_x, float* out,
                                    cudaStream_t s) {
    if (!out || p.v0 != 0) return cudaErrorInvalidValue;
    return w_depends_on_z ? go_mixed_weights2<true>(p, zpt, tile_x, out, s)
                          : go_mixed_weights2<false>(p, zpt, tile_x, out, s);
}

cudaError_t launch_bp_mixed(const BPParams& p, bool finalize, bool w_depends_on_z, int zpt, int tile_x,
                            cudaStream_t s) {
    if (finalize)
        return w_depends_on_z ? go_mixed2<true, true>(p, zpt, tile_x, s) : go_mixed2<true, false>(p, zpt, tile_x, s);
    return w_depends_on_z ? go_mixed2<false, true>(p, zpt, tile_x, s) : go_mixed2<false, false>(p, zpt, tile_x, s);
}

namespace {

template <bool M, bool W, bool V, bool D>
cudaError_t batch_go(const BatchSlots& t, int nscans, unsigned total, unsigned* counter, int ctas, cudaStream_t s) {
    bp_batch_kernel<M, W, V, D><<<ctas, dim3(kBPTileX, kBPTileY), 0, s>>>(t, nscans, counter, total);
    return cudaGetLastError();
}

template <bool M, bool W, bool V, bool D>
cudaError_t batch_occ(int* per) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per, bp_batch_kernel<M, W, V, D>, kBPThreads, 0);
}

// deep: 16-slice tiles (the mixed form only)
template <bool M, bool W>
cudaError_t batch_go2(const BatchSlots& t, int nscans, unsigned total, unsigned* counter, int ctas, bool wv,
                      bool deep, cudaStream_t s) {
    if constexpr (M) {
        if (deep)
            return wv ? batch_go<M, W, true, true>(t, nscans, total, counter, ctas, s)
                      : batch_go<M, W, false, true>(t, nscans, total, counter, ctas, s);
    }
    return wv ? batch_go<M, W, true, false>(t, nscans, total, counter, ctas, s)
              : batch_go<M, W, false, false>(t, nscans, total, counter, ctas, s);
}

template <bool M, bool W>
cudaError_t batch_occ2(bool wv, bool deep, int* per) {
    if constexpr (M) {
        if (deep) return wv ? batch_occ<M, W, true, true>(per) : batch_occ<M, W, false, true>(per);
    }
    return wv ? batch_occ<M, W, true, false>(per) : batch_occ<M, W, false, false>(per);
}

}  // namespace

cudaError_t launch_bp_batch(const BatchSlots& t, int nscans, unsigned total_tiles, bool mixed_form, bool wz,
                            bool wv, unsigned* counter, int ctas, cudaStream_t s) {
    if (nscans < 1 || nscans > kBatchSlots) return cudaErrorInvalidValue;
    const bool deep = t.s[0].zpt == 16;   // a launch of 16-slice tiles holds those only
    if (deep && !mixed_form) return cudaErrorInvalidValue;
    for (int i = 0; i < nscans; ++i) {
        const int z = t.s[i].zpt;
        if ((deep ? z != 16 : (z != 4 && z != 8)) || (wv && !t.s[i].p.wvol)) return cudaErrorInvalidValue;
    }
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    if (mixed_form)
        return wz ? batch_go2<true, true>(t, nscans, total_tiles, counter, ctas, wv, deep, s)
                  : batch_go2<true, false>(t, nscans, total_tiles, counter, ctas, wv, deep, s);
    return wz ? batch_go2<false, true>(t, nscans, total_tiles, counter, ctas, wv, false, s)
              : batch_go2<false, false>(t, nscans, total_tiles, counter, ctas, wv, false, s);
}

cudaError_t bp_batch_ctas(bool mixed_form, bool wz, bool wv, bool deep, int* ctas) {
    int dev = 0, sms = 0, per = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
        e = mixed_form ? (wz ? batch_occ2<true, true>(wv, deep, &per) : batch_occ2<true, false>(wv, deep, &per))
                       : (wz ? batch_occ2<false, true>(wv, false, &per) : batch_occ2<false, false>(wv, false, &per));
    *ctas = sms * (per > 0 ? per : 1);
    return e;
}

cudaError_t launch_frame_absmax(const float* plain, long long frame, int nv, unsigned* absmax, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(absmax, 0, sizeof(unsigned) * nv, s);
    if (e != cudaSuccess) return e;
    const int bx = (int)std::min<long long>((frame + 255) / 256, 64);
    frame_absmax_kernel<<<dim3(bx, nv), 256, 0, s>>>(plain, frame, absmax);
    return cudaGetLastError();
}

cudaError_t launch_pack_mixed(const float* plain, long long plain_frame, int nv, int rows, int U, const float2* tw,
                              int view0, int num_views, const unsigned* absmax, float* scale, uint2* qh,
                              long long q_frame, int slot0, cudaStream_t s) {
    dim3 grid((U + 255) / 256, rows, nv);
    pack_mixed_kernel<<<grid, 256, 0, s>>>(plain, plain_frame, rows, U, tw, view0, num_views, absmax, scale, qh,
                                           q_frame, slot0);
    return cudaGetLastError();
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
