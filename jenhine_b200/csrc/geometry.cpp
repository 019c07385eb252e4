// geometry.cpp -- per-context host operators: BP u-taper, pre-weight inverse
// transforms, filter spectrum and the dense ramp operator the tensor-core
// filter multiplies by.  Composition and inversion of the matrices run in FP64;
// values the reference computes in float (tapers, spectrum samples) follow the
// reference's float expressions so they match it bit for bit.
#include <cmath>
#include <complex>
#include <cstring>

#include "jfdk_internal.h"

namespace jfdk {

namespace {
constexpr float kPiF = (float)3.141592653589793L;  // Common/Constants.h:6
constexpr double kPiD = 3.141592653589793238462643383279502884;

// In-place radix-2 complex FFT in double, sign -1 forward / +1 inverse.
void fft_pow2(std::vector<std::complex<double>>& a, int sign) {
    const int n = (int)a.size();
    for (int i = 1, j = 0; i < n; ++i) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    for (int len = 2; len <= n; len <<= 1) {
        const int half = len >> 1;
        for (int k = 0; k < half; ++k) {
            const double ang = sign * 2.0 * kPiD * k / len;
            const std::complex<double> w(std::cos(ang), std::sin(ang));
            for (int i = 0; i < n; i += len) {
                const std::complex<double> t = a[i + k + half] * w;
                a[i + k + half] = a[i + k] - t;
                a[i + k] += t;
            }
        }
    }
}

// Small dense solve in float in the order of LAPACK's sgetf2 + sgetrs (the
// routines LAPACKE_sgesv runs for the 4x4 systems of FilterCore::SmoothInterp,
// FilterAgent/FilterCore.cpp:280-303).
void solve4_f32(float* A, float* B) {
    const int m = 4;
    int ipiv[4];
    for (int j = 0; j < m; ++j) {
        int piv = j;
        float best = std::fabs(A[j * m + j]);
        for (int i = j + 1; i < m; ++i)
            if (std::fabs(A[i * m + j]) > best) { best = std::fabs(A[i * m + j]); piv = i; }
        ipiv[j] = piv;
        if (A[piv * m + j] != 0.0f) {
            if (piv != j)
                for (int c = 0; c < m; ++c) std::swap(A[j * m + c], A[piv * m + c]);
            const float r = 1.0f / A[j * m + j];
            for (int i = j + 1; i < m; ++i) A[i * m + j] *= r;
        }
        for (int c = j + 1; c < m; ++c) {
            const float t = A[j * m + c];
            if (t != 0.0f)
                for (int i = j + 1; i < m; ++i) A[i * m + c] -= A[i * m + j] * t;
        }
    }
    for (int j = 0; j < m; ++j)
        if (ipiv[j] != j) std::swap(B[j], B[ipiv[j]]);
    for (int k = 0; k < m; ++k)
        if (B[k] != 0.0f)
            for (int i = k + 1; i < m; ++i) B[i] -= B[k] * A[i * m + k];
    for (int k = m - 1; k >= 0; --k)
        if (B[k] != 0.0f) {
            B[k] = B[k] / A[k * m + k];
            for (int i = 0; i < k; ++i) B[i] -= B[k] * A[i * m + k];
        }
}

// FilterCore::SmoothInterp (FilterAgent/FilterCore.cpp:262-318).
std::vector<float> smooth_interp(const std::vector<float>& x0, const std::vector<float>& y0,
                                 const std::vector<float>& xq) {
    const size_t n = x0.size();
    std::vector<float> yPi(n, 0.0f);
    for (size_t i = 1; i + 1 < n; ++i) {
        if ((y0[i] - y0[i - 1]) * (y0[i + 1] - y0[i]) < 0) {
            const float l = x0[i] - x0[i - 1], r = x0[i + 1] - x0[i];
            const float dl = (y0[i] - y0[i - 1]) / l, dr = (y0[i + 1] - y0[i]) / r;
            yPi[i] = (dl * r + dr * l) / (l + r);
        }
    }
    std::vector<float> a(n - 1), b(n - 1), c(n - 1), d(n - 1);
    for (size_t i = 0; i + 1 < n; ++i) {
        const float xl = x0[i], xr = x0[i + 1];
        float X[16] = {xl * xl * xl, xl * xl, xl, 1.f, xr * xr * xr, xr * xr, xr, 1.f,
                       3 * xl * xl, 2 * xl, 1, 0, 3 * xr * xr, 2 * xr, 1, 0};
        float Y[4] = {y0[i], y0[i + 1], yPi[i], yPi[i + 1]};
        solve4_f32(X, Y);
        a[i] = Y[0]; b[i] = Y[1]; c[i] = Y[2]; d[i] = Y[3];
    }
    std::vector<float> yq(xq.size(), 1.0f);
    for (size_t i = 0; i < xq.size(); ++i)
        for (size_t j = 0; j + 1 < n; ++j)
            if (xq[i] >= x0[j] && xq[i] <= x0[j + 1]) {
                yq[i] = xq[i] * (xq[i] * (xq[i] * a[j] + b[j]) + c[j]) + d[j];
                break;
            }
    return yq;
}

// FilterCore constructor spectrum (FilterCore.cpp:30-43, 69-138, 224-242).
std::vector<float> filter_spectrum(int L, float hsr, float cutStart, float cutEnd,
                                   const std::vector<float>& adjPts,
                                   const std::vector<float>& adjDB) {
    const int nf = L / 2 + 1;
    // Ram-Lak in space, then the real part of its spectrum (computed in
    // double, rounded once to float as the single-precision FFT returns it).
    std::vector<float> ramLak(L, 0.0f);
    const float pipi = kPiF * kPiF;
    ramLak[0] = 0.25f;
    for (int i = 1; i <= L / 2; i += 2) ramLak[i] = ramLak[L - i] = -1.0f / (pipi * (float)i * (float)i);
    std::vector<std::complex<double>> z(L);
    for (int i = 0; i < L; ++i) z[i] = ramLak[i];
    fft_pow2(z, -1);
    std::vector<float> freq(nf);
    for (int i = 0; i < nf; ++i) freq[i] = (float)i * hsr * 2.0f / (float)L;
    std::vector<float> ax{0.0f}, ay{0.0f};
    ax.insert(ax.end(), adjPts.begin(), adjPts.end());
    ay.insert(ay.end(), adjDB.begin(), adjDB.end());
    ax.push_back(hsr); ay.push_back(0.0f);
    for (float& v : ay) v = powf(10, v / 20.0f);
    std::vector<float> H = smooth_interp(ax, ay, freq);
    const float halfPi = kPiF * (float)0.5;
    if (cutStart == 0 && cutEnd == 0) {
        for (int i = 0; i < nf; ++i) {
            if (freq[i] < hsr) H[i] *= cosf(freq[i] / hsr * halfPi);
            else H[i] = 0.0f;
        }
    } else {
        for (int i = 0; i < nf; ++i) {
            const float f = freq[i];
            if (f <= cutStart) continue;
            if (f < cutEnd) H[i] *= cosf((f - cutStart) / (cutEnd - cutStart) * kPiF) * 0.5f + 0.5f;
            else H[i] = 0.0f;
        }
    }
    const float scale = kPiF * hsr * 2.0f;
    for (int i = 0; i < nf; ++i) {
        H[i] = H[i] * (float)z[i].real();
        H[i] = H[i] * scale;
    }
    return H;
}

}  // namespace

int fft_length(int width) {  // FilterAgent/FilterCore.cpp:254-260
    long length = 1;
    while (length < (long)width * 2 - 1) length *= 2;
    return (int)length;
}

std::string build_host_operators(const jfdk_scan_params& scan, const jfdk_recon_params& recon,
                                 const std::vector<float>& adj_pts,
                                 const std::vector<float>& adj_db, const float* ptms, int in_w,
                                 int out_w, int rows, int mirror, float hsr, HostOperators& ops) {
    const int N = scan.num_views;
    // -- BP u-taper per view (BPAgent/BPCore.cpp:68-100; the PTM sanity checks
    //    of BPCUDAAgent/BPCUDACore.cpp:86-92) --
    ops.uw.assign((size_t)N * out_w, 1.0f);
    for (int v = 0; v < N; ++v) {
        const float* P = ptms + (size_t)v * 12;
        const float uf = P[3] / P[11];
        if (uf != uf || uf < 0.0f || uf > (float)out_w)
            return "Something wrong with PTM: isocentre column of view " + std::to_string(v) +
                   " is outside the detector";
        const long u = (long)uf;
        float* w = ops.uw.data() + (size_t)v * out_w;
        if (u > out_w / 2) {
            const long nTrans = (out_w - u) * 2;
            for (long i = 0; i < nTrans; ++i)
                w[out_w - nTrans + i] = cosf((float)i * kPiF / (float)nTrans) * 0.5f + 0.5f;
        } else {
            const long nTrans = u * 2;
            for (long i = 0; i < nTrans; ++i) w[i] = cosf((float)i * kPiF / (float)nTrans) * -0.5f + 0.5f;
        }
    }
    // -- inverse transform matrix per 9-view pre-weight group: PTM2TM in
    //    float (TransformMatrix/MatrixConvertor.cpp:8-27), then TM^-1 solved
    //    in float against the identity as PreFilterWeightGenerator.cpp:20-31
    //    does (LinearEquationSolver, LAPACK's sgesv order), one column at a
    //    time: the weights' distance is a difference of two back-projected
    //    points, so the inverse must round as the reference's does --
    const int G = (N + 8) / 9;
    ops.tinv.assign((size_t)G * 16, 0.0f);
    const float dso = scan.dso;
    const float far_ = (1.0f + 1.0f / dso) * dso, near_ = (1.0f - 1.0f / dso) * dso;
    const float s20 = (far_ + near_) / (far_ - near_);
    const float s23 = ((far_ + near_) - 2.0f * far_ * near_ / dso) / (far_ - near_) / dso;
    for (int g = 0; g < G; ++g) {
        const int src = std::min(9 * g + 9 / 2, N - 1);  // FilterAgent.cpp:120-122
        const float* P = ptms + (size_t)src * 12;
        float tm[16];
        std::memcpy(tm, P, 8 * sizeof(float));
        tm[8] = s20 * P[8]; tm[9] = s20 * P[9]; tm[10] = 0.0f; tm[11] = s23 * P[11];
        std::memcpy(tm + 12, P + 8, 4 * sizeof(float));
        for (int j = 0; j < 4; ++j) {
            float A[16], e[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            std::memcpy(A, tm, sizeof A);
            e[j] = 1.0f;
            solve4_f32(A, e);
            for (int i = 0; i < 4; ++i) {
                if (!std::isfinite(e[i])) return "singular transform matrix for view " + std::to_string(src);
                ops.tinv[(size_t)g * 16 + i * 4 + j] = e[i];
            }
        }
    }
    // -- inverse transform matrix of every view, solved in float in LAPACK's
    //    order like CompositeCore::Inverse (CompositeAgent/CompositeCore.cpp:186-191),
    //    one right-hand side (a column of I) at a time --
    ops.tinv_view.assign((size_t)N * 16, 0.0f);
    for (int v = 0; v < N; ++v) {
        const float* P = ptms + (size_t)v * 12;
        float tm[16];
        std::memcpy(tm, P, 8 * sizeof(float));
        tm[8] = s20 * P[8]; tm[9] = s20 * P[9]; tm[10] = 0.0f; tm[11] = s23 * P[11];
        std::memcpy(tm + 12, P + 8, 4 * sizeof(float));
        for (int j = 0; j < 4; ++j) {
            float A[16], e[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            std::memcpy(A, tm, sizeof A);
            e[j] = 1.0f;
            solve4_f32(A, e);
            for (int i = 0; i < 4; ++i) ops.tinv_view[(size_t)v * 16 + i * 4 + j] = e[i];
        }
    }
    // -- filter spectrum and the equivalent dense operator --
    const int L = fft_length(in_w);
    ops.H = filter_spectrum(L, hsr, recon.filter_cutoff_start, recon.filter_cutoff_end, adj_pts, adj_db);
    // h_eff = IDFT_L(H) with H_{L-k} = H_k: real and even (the circular
    // convolution kernel FilterCore applies through FFT -> xH -> IFFT(1/L)).
    std::vector<std::complex<double>> z(L);
    for (int k = 0; k <= L / 2; ++k) z[k] = ops.H[k];
    for (int k = L / 2 + 1; k < L; ++k) z[k] = ops.H[L - k];
    fft_pow2(z, +1);
    std::vector<double> h(L);
    for (int i = 0; i < L; ++i) h[i] = z[i].real() / L;
    const int off = mirror ? out_w : 0;                  // FilterCore.cpp:28
    ops.h = h;
    ops.off = off;
    ops.T.assign((size_t)out_w * in_w, 0.0f);
    for (int j = 0; j < out_w; ++j)
        for (int i = 0; i < in_w; ++i) {
            int d = (off + j - i) % L;
            if (d < 0) d += L;
            ops.T[(size_t)j * in_w + i] = (float)h[d];
        }
    // Truncation ramp (FilterCore.cpp:45-60, 201-214): b[pos_k] = ramp_k * e.
    const int R = (L - in_w) / 2;
    ops.c.assign(out_w, 0.0f);
    for (int j = 0; j < out_w; ++j) {
        double acc = 0.0;
        for (int k = 0; k < R; ++k) {
            const float rk = mirror ? (float)(R - 1 - k) / (float)R : (float)k / (float)R;
            const int pos = mirror ? in_w + k : L - R + k;
            int d = (off + j - pos) % L;
            if (d < 0) d += L;
            acc += (double)rk * h[d];
        }
        ops.c[j] = (float)acc;
    }
    (void)rows;
    return "";
}

}  // namespace jfdk
