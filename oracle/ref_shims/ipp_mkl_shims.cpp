// ipp_mkl_shims.cpp -- scalar stand-ins for the Intel IPP / MKL wrappers the
// reference Core classes call, so that those classes compile from their own
// sources with g++ (TEST INFRASTRUCTURE: links only into oracle/_ref).
//
// The declarations come from the reference headers (Performance/BasicMathIPP.h,
// Performance/ImgEditor.h, Performance/RealFFT.h, Performance/LinearAlgebraMath.h,
// Performance/ImgResizer.h, Common/Exception.h); every body here is a restatement
// of the semantics of the IPP / MKL call the reference wrapper makes:
//   BasicMathIPP  -> Performance/BasicMathIPP.cpp:21-276 (operand order of the
//                    wrapper, e.g. Div(dst, c) is dst / c, Div(c, dst) is c / dst)
//   ImgEditor     -> Performance/ImgEditor.cpp:92-113 (ippiRemap_32f_C1R linear)
//   RealFFT       -> Performance/RealFFT.cpp:13-61 (MKL DFTI real, CCS, 1/n back)
//   LinearAlgebra -> Performance/LinearAlgebraMath.cpp:26-78 (sgemm, sgesv)
//   ImgResizer    -> Performance/ImgResizer.cpp:10-59 (ippiResizeLinear)
// Third-party versions the reference names: Intel IPP 2020.0.166 and MKL
// 2020.0.166 (.vscode/c_cpp_properties.json:7-9); neither is vendored.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../fdk_oracle.h"

// Reference headers (resolved through the include forwarders that
// oracle/build.py writes into oracle/_ref/inc).
#include "Common/Exception.h"
#include "Performance/BasicMathIPP.h"
#include "Performance/ImgEditor.h"
#include "Performance/ImgResizer.h"
#include "Performance/LinearAlgebraMath.h"
#include "Performance/RealFFT.h"

namespace JEngine {

// Common/Exception.cpp:9-23 uses the MSVC-only std::exception(const char*).
Exception::Exception(const std::string&, const size_t, const std::string&, const bool)
    : std::exception() {}

namespace BasicMathIPP {
void Add(float* d, const float* s, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = d[i] + s[i]; }
void Add(float* d, const float* a, const float* b, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = a[i] + b[i]; }
void Add(float* d, const float c, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = d[i] + c; }
void Add(float* d, const float* s, const float c, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = s[i] + c; }
void Sub(float* d, const float* s, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = d[i] - s[i]; }
void Sub(float* d, const float* a, const float* b, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = a[i] - b[i]; }
void Sub(float* d, const float c, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = d[i] - c; }
void Sub(const float c, float* d, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = c - d[i]; }
void Sub(float* d, const float* s, const float c, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = s[i] - c; }
void Sub(float* d, const float c, const float* s, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = c - s[i]; }
void Mul(float* d, const float* s, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = d[i] * s[i]; }
void Mul(float* d, const float* a, const float* b, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = a[i] * b[i]; }
void Mul(float* d, const float c, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = d[i] * c; }
void Mul(float* d, const float* s, const float c, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = s[i] * c; }
void Div(float* d, const float* s, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = d[i] / s[i]; }
void Div(float* d, const float* a, const float* b, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = a[i] / b[i]; }
void Div(float* d, const float c, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = d[i] / c; }
void Div(const float c, float* d, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = c / d[i]; }
void Div(float* d, const float* s, const float c, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = s[i] / c; }
void Div(float* d, const float c, const float* s, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = c / s[i]; }
float Sum(const float* p, const size_t n) { double s = 0; for (size_t i = 0; i < n; ++i) s += p[i]; return (float)s; }
float Mean(const float* p, const size_t n) { return Sum(p, n) / (float)n; }
void Abs(float* d, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = std::fabs(d[i]); }
void Abs(float* d, const float* s, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = std::fabs(s[i]); }
void Ln(float* d, size_t n) { for (size_t i = 0; i < n; ++i) d[i] = std::log(d[i]); }
void Ln(float* d, const float* s, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = std::log(s[i]); }
void Exp(float* d, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = std::exp(d[i]); }
void Exp(float* d, const float* s, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = std::exp(s[i]); }
void Sqrt(float* d, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = std::sqrt(d[i]); }
void Sqrt(float* d, const float* s, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = std::sqrt(s[i]); }
void Convert_16u_to_32f(float* d, const unsigned short* s, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = (float)s[i]; }
void Convert_32f_to_16s(signed short* d, const float* s, const size_t n) { jo_to_int16((int16_t*)d, s, n); }
void Convert_16f_to_32f(float* d, const signed short* s, const size_t n) {
    for (size_t i = 0; i < n; ++i) {
        const uint16_t h = (uint16_t)s[i];
        const uint32_t sign = (uint32_t)(h >> 15) << 31;
        int e = (h >> 10) & 31; uint32_t m = h & 1023u, bits;
        if (e == 0) {
            if (m == 0) bits = sign;
            else { e = 127 - 15 + 1; while (!(m & 1024u)) { m <<= 1; --e; } m &= 1023u; bits = sign | ((uint32_t)e << 23) | (m << 13); }
        } else if (e == 31) bits = sign | 0x7f800000u | (m << 13);
        else bits = sign | ((uint32_t)(e - 15 + 127) << 23) | (m << 13);
        std::memcpy(&d[i], &bits, 4);
    }
}
void Convert_32f_to_16f(signed short* d, const float* s, const size_t n) {
    for (size_t i = 0; i < n; ++i) {  // round to nearest even
        uint32_t x; std::memcpy(&x, &s[i], 4);
        const uint32_t sign = (x >> 16) & 0x8000u;
        int e = (int)((x >> 23) & 255) - 127 + 15; uint32_t m = x & 0x7fffffu; uint16_t h;
        if (((x >> 23) & 255) == 255) h = (uint16_t)(sign | 0x7c00u | (m ? 0x200u : 0));
        else if (e >= 31) h = (uint16_t)(sign | 0x7c00u);
        else if (e <= 0) {
            if (e < -10) h = (uint16_t)sign;
            else { m |= 0x800000u; const int sh = 14 - e; uint32_t hm = m >> sh; const uint32_t rem = m & ((1u << sh) - 1), half = 1u << (sh - 1);
                   if (rem > half || (rem == half && (hm & 1))) ++hm; h = (uint16_t)(sign | hm); }
        } else {
            uint32_t hm = m >> 13; const uint32_t rem = m & 0x1fffu; uint32_t he = (uint32_t)e;
            if (rem > 0x1000u || (rem == 0x1000u && (hm & 1))) { if (++hm == 1024u) { hm = 0; ++he; } }
            h = (uint16_t)(sign | (he >= 31 ? 0x7c00u : ((he << 10) | hm)));
        }
        d[i] = (signed short)h;
    }
}
void Cpy(float* d, const float* s, const size_t n) { std::memcpy(d, s, n * sizeof(float)); }
void Set(float* d, const float c, const size_t n) { for (size_t i = 0; i < n; ++i) d[i] = c; }
void ReplaceNAN(float* p, const float c, const size_t n) { for (size_t i = 0; i < n; ++i) if (p[i] != p[i]) p[i] = c; }
void UpperBound(float* p, const float l, const size_t n) { for (size_t i = 0; i < n; ++i) if (p[i] > l) p[i] = l; }
void LowerBound(float* p, const float l, const size_t n) { for (size_t i = 0; i < n; ++i) if (p[i] < l) p[i] = l; }
float Min(float* p, const size_t n) { float m = p[0]; for (size_t i = 1; i < n; ++i) if (p[i] < m) m = p[i]; return m; }
}  // namespace BasicMathIPP

namespace ImgEditor {
static inline const float* roi_ptr(const float* p, const ROI& r) { return p + r.OffsetPixels; }
void Cpy(float* d, const ROI& dr, const float* s, const ROI& sr) {
    for (int y = 0; y < dr.RoiHeight; ++y)
        std::memcpy(d + dr.OffsetPixels + (size_t)y * dr.FullWidth, roi_ptr(s, sr) + (size_t)y * sr.FullWidth, sizeof(float) * dr.RoiWidth);
}
void Add(float* d, const ROI& dr, const float* s, const ROI& sr) {
    for (int y = 0; y < dr.RoiHeight; ++y) for (int x = 0; x < dr.RoiWidth; ++x)
        d[dr.OffsetPixels + (size_t)y * dr.FullWidth + x] += roi_ptr(s, sr)[(size_t)y * sr.FullWidth + x];
}
void Sub(float* d, const ROI& dr, const float* s, const ROI& sr) {
    for (int y = 0; y < dr.RoiHeight; ++y) for (int x = 0; x < dr.RoiWidth; ++x)
        d[dr.OffsetPixels + (size_t)y * dr.FullWidth + x] -= roi_ptr(s, sr)[(size_t)y * sr.FullWidth + x];
}
void Mul(float* d, const ROI& dr, const float* a, const ROI& ar, const float* b, const ROI& br) {
    for (int y = 0; y < dr.RoiHeight; ++y) for (int x = 0; x < dr.RoiWidth; ++x)
        d[dr.OffsetPixels + (size_t)y * dr.FullWidth + x] =
            roi_ptr(a, ar)[(size_t)y * ar.FullWidth + x] * roi_ptr(b, br)[(size_t)y * br.FullWidth + x];
}
void Mul(float* d, const ROI& dr, const float* s, const ROI& sr) {
    for (int y = 0; y < dr.RoiHeight; ++y) for (int x = 0; x < dr.RoiWidth; ++x)
        d[dr.OffsetPixels + (size_t)y * dr.FullWidth + x] *= roi_ptr(s, sr)[(size_t)y * sr.FullWidth + x];
}
void Mul(float* d, const ROI& dr, const float c) {
    for (int y = 0; y < dr.RoiHeight; ++y) for (int x = 0; x < dr.RoiWidth; ++x)
        d[dr.OffsetPixels + (size_t)y * dr.FullWidth + x] *= c;
}
// ippiRemap_32f_C1R with IPPI_INTER_LINEAR: the destination pixel is written
// only when the mapped point lies in [0, W-1] x [0, H-1] (pixel centres at
// integers); the +1 neighbour is clamped to the last column / row, where its
// weight is exactly zero.  The same rule is restated in fdk_oracle.c.
void Remap(float* pDst, const ROI& dstROI, const float* pSrc, const ROI& srcROI,
           const float* pX, const float* pY, const ROI& mapROI) {
    const float* src = pSrc + srcROI.OffsetPixels;
    const int W = srcROI.RoiWidth, H = srcROI.RoiHeight, sp = srcROI.FullWidth;
    for (int y = 0; y < dstROI.RoiHeight; ++y) {
        for (int x = 0; x < dstROI.RoiWidth; ++x) {
            const float u = pX[mapROI.OffsetPixels + (size_t)y * mapROI.FullWidth + x];
            const float v = pY[mapROI.OffsetPixels + (size_t)y * mapROI.FullWidth + x];
            if (!(u >= 0.0f && u <= (float)(W - 1) && v >= 0.0f && v <= (float)(H - 1))) continue;
            const int ix = (int)std::floor(u), iy = (int)std::floor(v);
            const int ix1 = ix + 1 < W ? ix + 1 : W - 1, iy1 = iy + 1 < H ? iy + 1 : H - 1;
            const float fx = u - (float)ix, fy = v - (float)iy;
            const float p00 = src[(size_t)iy * sp + ix], p01 = src[(size_t)iy * sp + ix1];
            const float p10 = src[(size_t)iy1 * sp + ix], p11 = src[(size_t)iy1 * sp + ix1];
            const float t0 = p00 + fx * (p01 - p00);
            const float t1 = p10 + fx * (p11 - p10);
            pDst[dstROI.OffsetPixels + (size_t)y * dstROI.FullWidth + x] = t0 + fy * (t1 - t0);
        }
    }
}
}  // namespace ImgEditor

// ---- RealFFT (MKL DFTI real transform; CCS packing; backward scale 1/n) ----
RealFFT::RealFFT(const size_t n) : length((int)n), pDescHandle(nullptr) {}
RealFFT::RealFFT(const RealFFT& o) : length(o.length), pDescHandle(nullptr) {}
RealFFT::~RealFFT() {}
void RealFFT::Foward(float* pCCS, float* pSpace) const { jo_rfft_forward(pCCS, pSpace, length); }
void RealFFT::Backward(float* pSpace, float* pCCS) const { jo_rfft_backward(pSpace, pCCS, length); }
void RealFFT::ExtracPositiveRealFromCCS(float* r, const float* c) const { for (int i = 0; i <= length / 2; ++i) r[i] = c[i * 2]; }
void RealFFT::ExtracPositiveImagFromCCS(float* r, const float* c) const { for (int i = 0; i <= length / 2; ++i) r[i] = c[i * 2 + 1]; }

namespace LinearAlgebraMath {
MatrixMultiplier::MatrixMultiplier(const size_t m_, const size_t n_, const size_t p_) : m((int)m_), n((int)n_), p((int)p_) {}
void MatrixMultiplier::Execute(float* C, const float* A, const float* B) const { Execute(C, 1.0f, A, B, 0.0f); }
void MatrixMultiplier::Execute(float* C, const float alpha, const float* A, const float* B, const float beta) const {
    for (int i = 0; i < m; ++i) for (int j = 0; j < p; ++j) {
        float s = 0.0f;
        for (int k = 0; k < n; ++k) s += A[i * n + k] * B[k * p + j];
        C[i * p + j] = (beta == 0.0f) ? alpha * s : alpha * s + beta * C[i * p + j];
    }
}
LinearEquationSolver::LinearEquationSolver(const size_t m_, const size_t p_)
    : m((int)m_), p((int)p_), bufferA(m_ * m_), bufferB(m_ * p_), bufferPivotIdx(m_) {}
void LinearEquationSolver::Execute(float* X, const float* A, const float* B) {
    std::memcpy(bufferA.data(), A, bufferA.size() * sizeof(float));
    std::memcpy(bufferB.data(), B, bufferB.size() * sizeof(float));
    jo_solve_f32(m, p, bufferA.data(), bufferB.data());
    std::memcpy(X, bufferB.data(), bufferB.size() * sizeof(float));
}
void LinearEquationSolver::Execute(float* XB, float* A) { jo_solve_f32(m, p, A, XB); }
}  // namespace LinearAlgebraMath

// ---- ImgResizer (ippiResizeLinear_32f, border replicate) ----
ImgResizer::ImgResizer(const ROI& d, const ROI& s) : srcROI(s), dstROI(d), pSpec(nullptr), pBuffer(nullptr) {}
ImgResizer::~ImgResizer() {}
void ImgResizer::Execute(float* pDst, const float* pSrc) const {
    const int sw = srcROI.RoiWidth, sh = srcROI.RoiHeight, dw = dstROI.RoiWidth, dh = dstROI.RoiHeight;
    const float* s = pSrc + srcROI.OffsetPixels;
    float* d = pDst + dstROI.OffsetPixels;
    if (sw == dw && sh == dh) {  // identity: a crop
        for (int y = 0; y < dh; ++y) std::memcpy(d + (size_t)y * dstROI.FullWidth, s + (size_t)y * srcROI.FullWidth, sizeof(float) * dw);
        return;
    }
    for (int y = 0; y < dh; ++y) for (int x = 0; x < dw; ++x) {
        float sx = ((float)x + 0.5f) * sw / dw - 0.5f, sy = ((float)y + 0.5f) * sh / dh - 0.5f;
        sx = sx < 0 ? 0 : (sx > sw - 1 ? (float)(sw - 1) : sx);
        sy = sy < 0 ? 0 : (sy > sh - 1 ? (float)(sh - 1) : sy);
        const int ix = (int)sx, iy = (int)sy;
        const int ix1 = ix + 1 < sw ? ix + 1 : sw - 1, iy1 = iy + 1 < sh ? iy + 1 : sh - 1;
        const float fx = sx - ix, fy = sy - iy;
        const float* r0 = s + (size_t)iy * srcROI.FullWidth; const float* r1 = s + (size_t)iy1 * srcROI.FullWidth;
        const float t0 = r0[ix] + fx * (r0[ix1] - r0[ix]), t1 = r1[ix] + fx * (r1[ix1] - r1[ix]);
        d[(size_t)y * dstROI.FullWidth + x] = t0 + fy * (t1 - t0);
    }
}

}  // namespace JEngine
