// ramp_gemm.cu -- the ramp filter of every detector row as one dense product.
//
// FilterCore::ProcessRow (FilterAgent/FilterCore.cpp:189-222) zero-pads a row
// to L = CalFFTLength(W), multiplies by the cosine pre-weight, writes a linear
// truncation ramp of the row's edge mean into the padding, convolves
// circularly with the real even kernel h = IDFT_L(H) (FFT -> x H -> IFFT / L)
// and crops W_out samples at offset off.  That is exactly linear:
//
//     out[r][j] = sum_i T[j][i] * (pw o x)[r][i] + c[j] * e[r],
//     T[j][i]   = h[(off + j - i) mod L],
//     c[j]      = sum_k ramp_k * h[(off + j - pos_k) mod L],
//
// so the whole projection set is Q = A * T^T + e c^T with M = views * rows,
// N = W_out, K = W.  The epilogue adds the rank-1 edge term and stores the
// filtered rows (the backprojector's packer applies the u-taper).
//
// This file holds the FP32 CUDA-core (SIMT) form: 128 x 128 output tile per
// CTA, K staged through shared memory in steps of 16, 8 x 8 outputs per
// thread.
#include <cuda_runtime.h>

#include "jfdk_internal.h"

namespace jfdk {
namespace {

constexpr int BM = 128, BN = 128, BK = 16, PADS = 4;

__global__ void __launch_bounds__(256) ramp_gemm_simt_kernel(RampParams p) {
    __shared__ __align__(16) float As[BK][BM + PADS];
    __shared__ __align__(16) float Bs[BK][BN + PADS];
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    // loader coordinates: 128 rows x 16 k per tile, 8 floats per thread
    const int lr = tid >> 1, lk = (tid & 1) * 8;
    const int am = m0 + lr, bn = n0 + lr;
    const float* ap = p.A + (size_t)am * p.a_pitch + lk;
    const float* bp = p.B + (size_t)bn * p.a_pitch + lk;
    const bool aok = am < p.M, bok = bn < p.N;

    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.0f;

    for (int k0 = 0; k0 < p.a_pitch; k0 += BK) {
        float4 a0 = make_float4(0.f, 0.f, 0.f, 0.f), a1 = a0, b0 = a0, b1 = a0;
        if (aok) { a0 = *reinterpret_cast<const float4*>(ap + k0); a1 = *reinterpret_cast<const float4*>(ap + k0 + 4); }
        if (bok) { b0 = *reinterpret_cast<const float4*>(bp + k0); b1 = *reinterpret_cast<const float4*>(bp + k0 + 4); }
        __syncthreads();
        As[lk + 0][lr] = a0.x; As[lk + 1][lr] = a0.y; As[lk + 2][lr] = a0.z; As[lk + 3][lr] = a0.w;
        As[lk + 4][lr] = a1.x; As[lk + 5][lr] = a1.y; As[lk + 6][lr] = a1.z; As[lk + 7][lr] = a1.w;
        Bs[lk + 0][lr] = b0.x; Bs[lk + 1][lr] = b0.y; Bs[lk + 2][lr] = b0.z; Bs[lk + 3][lr] = b0.w;
        Bs[lk + 4][lr] = b1.x; Bs[lk + 5][lr] = b1.y; Bs[lk + 6][lr] = b1.z; Bs[lk + 7][lr] = b1.w;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < BK; ++k) {
            const float4 x0 = *reinterpret_cast<const float4*>(&As[k][ty * 4]);
            const float4 x1 = *reinterpret_cast<const float4*>(&As[k][64 + ty * 4]);
            const float4 y0 = *reinterpret_cast<const float4*>(&Bs[k][tx * 4]);
            const float4 y1 = *reinterpret_cast<const float4*>(&Bs[k][64 + tx * 4]);
            const float xa[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
            const float yb[8] = {y0.x, y0.y, y0.z, y0.w, y1.x, y1.y, y1.z, y1.w};
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(xa[i], yb[j], acc[i][j]);
        }
    }
    // epilogue: + c[n] e[m] (the truncation ramp), store the filtered rows
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int m = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + i - 4);
        if (m >= p.M) continue;
        const int vl = m / p.rows, row = m - vl * p.rows;
        const float em = p.c ? p.e[m] : 0.0f;   // no c: the plain product (filter adjoint)
        float* q = p.q + (size_t)vl * p.q_frame_stride + (size_t)row * p.q_pitch;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int n = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + j - 4);
            if (n >= p.N) continue;
            q[n] = p.c ? fmaf(p.c[n], em, acc[i][j]) : acc[i][j];
        }
    }
}

}  // namespace

cudaError_t launch_ramp_gemm(const RampParams& p, cudaStream_t s) {
    dim3 grid((p.N + BN - 1) / BN, (p.M + BM - 1) / BM);
    ramp_gemm_simt_kernel<<<grid, 256, 0, s>>>(p);
    return cudaGetLastError();
}

}  // namespace jfdk
