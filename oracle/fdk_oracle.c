/*
 * fdk_oracle.c -- CPU restatement of the JEngine FDK hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA engine.  Nothing
 * on the product path links or calls this file.  Build with
 * -ffp-contract=off so float expressions round exactly as written.
 *
 * Reference citations are file:line within the JEngine source tree.
 */
#include "fdk_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define JO_PI_F ((float)3.141592653589793L) /* Common/Constants.h:6 */
#define JO_PI_D 3.141592653589793238462643383279502884

/* ======================================================================
 * Geometry
 * ==================================================================== */

/* TransformMatrix/ProjectionMatrixModifier.cpp:5-11 */
void jo_ptm_move_u(float p[12], float u) {
    for (int j = 0; j < 4; ++j) p[0 * 4 + j] -= p[2 * 4 + j] * u;
}
/* TransformMatrix/ProjectionMatrixModifier.cpp:13-19 */
void jo_ptm_move_v(float p[12], float v) {
    for (int j = 0; j < 4; ++j) p[1 * 4 + j] -= p[2 * 4 + j] * v;
}
/* TransformMatrix/ProjectionMatrixModifier.cpp:21-27 */
void jo_ptm_reverse_x(float p[12]) {
    for (int j = 0; j < 3; ++j) p[j * 4 + 0] *= -1.0f;
}
/* TransformMatrix/ProjectionMatrixModifier.cpp:29-35 */
void jo_ptm_reverse_y(float p[12]) {
    for (int j = 0; j < 3; ++j) p[j * 4 + 1] *= -1.0f;
}
/* TransformMatrix/ProjectionMatrixModifier.cpp:37-43 */
void jo_ptm_move_z(float p[12], float z) {
    for (int i = 0; i < 3; ++i) p[i * 4 + 3] += p[i * 4 + 2] * z;
}

/* TransformMatrix/MatrixConvertor.cpp:8-27: rows 0,1 of the PTM, a depth row
 * built from PTM row 2 scaled by near/far planes at DSO -/+ 1, then PTM row 2
 * as the homogeneous row. */
void jo_ptm2tm(float tm[16], const float ptm[12], float dso) {
    const float far_ = (1.0f + 1.0f / dso) * dso;
    const float near_ = (1.0f - 1.0f / dso) * dso;
    const float s20 = (far_ + near_) / (far_ - near_);
    const float s21 = (far_ + near_) / (far_ - near_);
    const float s23 = ((far_ + near_) - 2.0f * far_ * near_ / dso) / (far_ - near_) / dso;
    memcpy(tm, ptm, 8 * sizeof(float));
    tm[8] = s20 * ptm[8];
    tm[9] = s21 * ptm[9];
    tm[10] = 0.0f;
    tm[11] = s23 * ptm[11];
    memcpy(tm + 12, ptm + 8, 4 * sizeof(float));
}

/* LAPACKE_sgesv semantics (Performance/LinearAlgebraMath.cpp:50-61), restated
 * from the published LAPACK reference algorithms the call resolves to:
 * sgetf2 (LU with partial pivoting, column below the pivot scaled by the
 * pivot's reciprocal, rank-1 trailing update) and sgetrs (row interchanges,
 * then column-oriented unit-lower and upper triangular solves as in the
 * reference strsm).  Row-major storage; the arithmetic is that of the
 * column-major routine on the same matrix. */
int jo_solve_f32(int m, int p, float* A, float* B) {
    int info = 0;
    int* ipiv = (int*)malloc(sizeof(int) * m);
#define Af(i, j) A[(i) * m + (j)]
#define Bf(i, j) B[(i) * p + (j)]
    for (int j = 0; j < m; ++j) {
        int piv = j;
        float best = fabsf(Af(j, j));
        for (int i = j + 1; i < m; ++i)
            if (fabsf(Af(i, j)) > best) { best = fabsf(Af(i, j)); piv = i; }
        ipiv[j] = piv;
        if (Af(piv, j) != 0.0f) {
            if (piv != j)
                for (int c = 0; c < m; ++c) { float t = Af(j, c); Af(j, c) = Af(piv, c); Af(piv, c) = t; }
            const float r = 1.0f / Af(j, j);
            for (int i = j + 1; i < m; ++i) Af(i, j) *= r;
        } else if (!info) {
            info = j + 1;
        }
        for (int c = j + 1; c < m; ++c) {
            const float t = Af(j, c);
            if (t != 0.0f)
                for (int i = j + 1; i < m; ++i) Af(i, c) -= Af(i, j) * t;
        }
    }
    if (!info) {
        for (int j = 0; j < m; ++j)
            if (ipiv[j] != j)
                for (int c = 0; c < p; ++c) { float t = Bf(j, c); Bf(j, c) = Bf(ipiv[j], c); Bf(ipiv[j], c) = t; }
        for (int c = 0; c < p; ++c) {
            for (int k = 0; k < m; ++k)
                if (Bf(k, c) != 0.0f)
                    for (int i = k + 1; i < m; ++i) Bf(i, c) -= Bf(k, c) * Af(i, k);
            for (int k = m - 1; k >= 0; --k)
                if (Bf(k, c) != 0.0f) {
                    Bf(k, c) = Bf(k, c) / Af(k, k);
                    for (int i = 0; i < k; ++i) Bf(i, c) -= Bf(k, c) * Af(i, k);
                }
        }
    }
#undef Af
#undef Bf
    free(ipiv);
    return info;
}

int jo_solve_f64(int m, int p, double* A, double* B) {
    int info = 0;
    for (int k = 0; k < m; ++k) {
        int piv = k;
        double best = fabs(A[k * m + k]);
        for (int i = k + 1; i < m; ++i) {
            double a = fabs(A[i * m + k]);
            if (a > best) { best = a; piv = i; }
        }
        if (piv != k) {
            for (int j = 0; j < m; ++j) { double t = A[k * m + j]; A[k * m + j] = A[piv * m + j]; A[piv * m + j] = t; }
            for (int j = 0; j < p; ++j) { double t = B[k * p + j]; B[k * p + j] = B[piv * p + j]; B[piv * p + j] = t; }
        }
        const double d = A[k * m + k];
        if (d == 0.0) { if (!info) info = k + 1; continue; }
        for (int i = k + 1; i < m; ++i) {
            const double l = A[i * m + k] / d;
            A[i * m + k] = l;
            for (int j = k + 1; j < m; ++j) A[i * m + j] -= l * A[k * m + j];
            for (int j = 0; j < p; ++j) B[i * p + j] -= l * B[k * p + j];
        }
    }
    if (info) return info;
    for (int j = 0; j < p; ++j) {
        for (int i = m - 1; i >= 0; --i) {
            double s = B[i * p + j];
            for (int k = i + 1; k < m; ++k) s -= A[i * m + k] * B[k * p + j];
            B[i * p + j] = s / A[i * m + i];
        }
    }
    return 0;
}

/* ======================================================================
 * Preprocessing -- PreProcessingAgent/PreProcessingCore.cpp:67-86
 * ==================================================================== */
int jo_preprocess(float* out, const uint16_t* in, int inW, int inH,
                  int bUp, int bDown, int bLeft, int bRight, int outW, int outH,
                  float brightField, const float bhc[3]) {
    const int roiW = inW - bLeft - bRight, roiH = inH - bUp - bDown;
    if (roiW != outW || roiH != outH) return -1; /* only the identity resize */
    const int doBhc = !(bhc[0] == 1.0f && bhc[1] == 0.0f && bhc[2] == 0.0f); /* :56 */
    for (int r = 0; r < outH; ++r) {
        for (int c = 0; c < outW; ++c) {
            float p = (float)in[(size_t)(r + bUp) * inW + (c + bLeft)]; /* Convert_16u_to_32f */
            if (p < 1.0f) p = 1.0f;          /* LowerBound(1): ippsThreshold_LT */
            p = p / brightField;             /* GainCorr.cpp:10-13 */
            p = logf(p);                     /* NLog.cpp:9-13 */
            p = p * -1.0f;
            if (doBhc) {                     /* BeamHardeningCorr.cpp:17-27 */
                float buf = p * bhc[2];
                buf = buf + bhc[1];
                buf = buf * p;
                buf = buf + bhc[0];
                p = p * buf;
            }
            out[(size_t)r * outW + c] = p;
        }
    }
    return 0;
}

/* ======================================================================
 * Pre-filter cosine weight -- FilterAgent/PreFilterWeightGenerator.cpp
 * ==================================================================== */
int jo_fft_length(int width) { /* FilterAgent/FilterCore.cpp:254-260 */
    long length = 1;
    while (length < (long)width * 2 - 1) length *= 2;
    return (int)length;
}

/* PreFilterWeightGenerator.cpp:52-124, float op order preserved. */
void jo_preweight_generate(float* weights, const float* T, int inputWidth,
                           int height, int detOnRight) {
    const int width = jo_fft_length(inputWidth);
    float* uAxis = (float*)malloc(sizeof(float) * width);
    for (int i = 0; i < width; ++i) uAxis[i] = (float)i; /* :35-37 */
    if (detOnRight)
        for (int i = 0; i < width; ++i) uAxis[i] = uAxis[i] - (float)inputWidth / 2; /* :39-40 */
    const float w0 = 0.0f, w1 = 1.f;
#define TM(r, c) T[(r) * 4 + (c)]
    for (int iV = 0; iV < height; ++iV) {
        const float v = (float)iV;
        float* pw = weights + (size_t)iV * width;
        const float c30 = v * TM(3, 1);
        const float n0c = w0 * TM(3, 2) + TM(3, 3);
        const float n1c = w1 * TM(3, 2) + TM(3, 3);
        float cr[3][3];
        for (int r = 0; r < 3; ++r) {
            cr[r][0] = v * TM(r, 1);
            cr[r][1] = w0 * TM(r, 2) + TM(r, 3);
            cr[r][2] = w1 * TM(r, 2) + TM(r, 3);
        }
        for (int i = 0; i < width; ++i) {
            float t = uAxis[i] * TM(3, 0);
            t = t + c30;
            const float norm0 = t + n0c;
            const float norm1 = t + n1c;
            float acc = 0.0f;
            for (int r = 0; r < 3; ++r) {
                float s = uAxis[i] * TM(r, 0);
                s = s + cr[r][0];
                const float a0 = (s + cr[r][1]) / norm0;
                const float a1 = (s + cr[r][2]) / norm1;
                float d = a0 - a1;
                d = d * d;
                if (r == 0) acc = d; else acc = acc + d;
            }
            pw[i] = sqrtf(acc); /* :119 */
        }
    }
#undef TM
    const size_t n = (size_t)height * width;
    float mn = weights[0];
    for (size_t i = 1; i < n; ++i) if (weights[i] < mn) mn = weights[i]; /* :122 */
    for (size_t i = 0; i < n; ++i) weights[i] = mn / weights[i];         /* :123 */
    free(uAxis);
}

/* PreFilterWeightGenerator.cpp:20-31 (PTM2TM then TM^-1 via sgesv against I),
 * followed by Generate. */
void jo_preweight_for_view(float* weights, const float ptm[12], float dso,
                           int inputWidth, int height, int detOnRight) {
    float tm[16], eye[16];
    jo_ptm2tm(tm, ptm, dso);
    memset(eye, 0, sizeof(eye));
    for (int i = 0; i < 4; ++i) eye[i * 4 + i] = 1.0f;
    jo_solve_f32(4, 4, tm, eye);
    jo_preweight_generate(weights, eye, inputWidth, height, detOnRight);
}

/* FilterAgent/FilterAgent.cpp:101-126: regenerated when view % 9 == 0 from
 * view min(v + 4, N - 1), reused for the next 8 views. */
int jo_preweight_source_view(int v, int numViews) {
    const int g = (v / 9) * 9;
    const int s = g + 9 / 2;
    return s < numViews - 1 ? s : numViews - 1;
}

/* ======================================================================
 * Real FFT with MKL CCS packing (Performance/RealFFT.cpp, Performance/RealFFT.h:11-17)
 * computed in double.
 * ==================================================================== */
static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

/* In-place iterative radix-2 complex FFT, sign = -1 forward, +1 inverse. */
static void fft_c2c_pow2(double* re, double* im, int n, int sign) {
    for (int i = 1, j = 0; i < n; ++i) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double t = re[i]; re[i] = re[j]; re[j] = t;
            t = im[i]; im[i] = im[j]; im[j] = t;
        }
    }
    for (int len = 2; len <= n; len <<= 1) {
        const int half = len >> 1;
        for (int k = 0; k < half; ++k) {
            const double ang = sign * 2.0 * JO_PI_D * k / len;
            const double wr = cos(ang), wi = sin(ang);
            for (int i = 0; i < n; i += len) {
                double* ar = re + i + k; double* ai = im + i + k;
                double* br = re + i + k + half; double* bi = im + i + k + half;
                const double tr = *br * wr - *bi * wi;
                const double ti = *br * wi + *bi * wr;
                *br = *ar - tr; *bi = *ai - ti;
                *ar += tr; *ai += ti;
            }
        }
    }
}

static void dft_forward_d(double* re, double* im, const double* x, int n) {
    if (is_pow2(n)) {
        for (int i = 0; i < n; ++i) { re[i] = x[i]; im[i] = 0.0; }
        fft_c2c_pow2(re, im, n, -1);
        return;
    }
    for (int k = 0; k < n; ++k) {
        double sr = 0.0, si = 0.0;
        for (int t = 0; t < n; ++t) {
            const double ang = -2.0 * JO_PI_D * (double)(((long)k * t) % n) / n;
            sr += x[t] * cos(ang);
            si += x[t] * sin(ang);
        }
        re[k] = sr; im[k] = si;
    }
}

void jo_rfft_forward(float* ccs, const float* x, int n) {
    double* xd = (double*)malloc(sizeof(double) * n);
    double* re = (double*)malloc(sizeof(double) * n);
    double* im = (double*)malloc(sizeof(double) * n);
    for (int i = 0; i < n; ++i) xd[i] = x[i];
    dft_forward_d(re, im, xd, n);
    for (int k = 0; k <= n / 2; ++k) {
        ccs[2 * k] = (float)re[k];
        ccs[2 * k + 1] = (k == 0 || (n % 2 == 0 && k == n / 2)) ? 0.0f : (float)im[k];
    }
    free(xd); free(re); free(im);
}

/* Backward with DFTI_BACKWARD_SCALE = 1/n (RealFFT.cpp:19). */
void jo_rfft_backward(float* x, const float* ccs, int n) {
    double* re = (double*)malloc(sizeof(double) * n);
    double* im = (double*)malloc(sizeof(double) * n);
    for (int k = 0; k <= n / 2; ++k) {
        re[k] = ccs[2 * k];
        im[k] = (k == 0 || (n % 2 == 0 && k == n / 2)) ? 0.0 : ccs[2 * k + 1];
    }
    for (int k = n / 2 + 1; k < n; ++k) { re[k] = re[n - k]; im[k] = -im[n - k]; }
    if (is_pow2(n)) {
        fft_c2c_pow2(re, im, n, +1);
        for (int i = 0; i < n; ++i) x[i] = (float)(re[i] / n);
    } else {
        for (int t = 0; t < n; ++t) {
            double s = 0.0;
            for (int k = 0; k < n; ++k) {
                const double ang = 2.0 * JO_PI_D * (double)(((long)k * t) % n) / n;
                s += re[k] * cos(ang) - im[k] * sin(ang);
            }
            x[t] = (float)(s / n);
        }
    }
    free(re); free(im);
}

/* ======================================================================
 * Filter spectrum -- FilterAgent/FilterCore.cpp:13-61, 69-138, 224-318
 * ==================================================================== */

/* FilterCore::SmoothInterp (FilterCore.cpp:262-318): piecewise cubic Hermite
 * through (x0, y0) with slopes that are zero except at interior extrema-free
 * points, each segment solved as a 4x4 system in float. */
static void smooth_interp(float* yq, const float* x0, const float* y0, int n,
                          const float* xq, int nq) {
    float* yPi = (float*)calloc(n, sizeof(float));
    for (int i = 1; i < n - 1; ++i) {
        if ((y0[i] - y0[i - 1]) * (y0[i + 1] - y0[i]) < 0) {
            float l = x0[i] - x0[i - 1];
            float r = x0[i + 1] - x0[i];
            float dl = (y0[i] - y0[i - 1]) / l;
            float dr = (y0[i + 1] - y0[i]) / r;
            yPi[i] = (dl * r + dr * l) / (l + r);
        }
    }
    float* a = (float*)malloc(sizeof(float) * (n - 1));
    float* b = (float*)malloc(sizeof(float) * (n - 1));
    float* c = (float*)malloc(sizeof(float) * (n - 1));
    float* d = (float*)malloc(sizeof(float) * (n - 1));
    for (int i = 0; i < n - 1; ++i) {
        const float xl = x0[i], xr = x0[i + 1], yl = y0[i], yr = y0[i + 1];
        float X[16];
        X[0] = xl * xl * xl; X[1] = xl * xl; X[2] = xl; X[3] = 1.f;
        X[4] = xr * xr * xr; X[5] = xr * xr; X[6] = xr; X[7] = 1.f;
        X[8] = 3 * xl * xl;  X[9] = 2 * xl;  X[10] = 1; X[11] = 0;
        X[12] = 3 * xr * xr; X[13] = 2 * xr; X[14] = 1; X[15] = 0;
        float Y[4] = {yl, yr, yPi[i], yPi[i + 1]};
        jo_solve_f32(4, 1, X, Y);
        a[i] = Y[0]; b[i] = Y[1]; c[i] = Y[2]; d[i] = Y[3];
    }
    for (int i = 0; i < nq; ++i) {
        yq[i] = 1.0f;
        for (int j = 0; j < n - 1; ++j) {
            if (xq[i] >= x0[j] && xq[i] <= x0[j + 1]) {
                yq[i] = xq[i] * (xq[i] * (xq[i] * a[j] + b[j]) + c[j]) + d[j];
                break;
            }
        }
    }
    free(yPi); free(a); free(b); free(c); free(d);
}

void jo_filter_spectrum(float* H, int L, float halfSampleRate, float cutStart,
                        float cutEnd, const float* adjPts, const float* adjDB, int nAdj) {
    const int nf = L / 2 + 1;
    /* GenerateRamLak (FilterCore.cpp:224-242) */
    float* ramLak = (float*)calloc(L, sizeof(float));
    const float pipi = JO_PI_F * JO_PI_F; /* Constants.h:15 */
    ramLak[0] = 0.25f;
    for (int i = 1; i <= L / 2; i += 2) {
        const float v = -1.0f / (pipi * (float)i * (float)i);
        ramLak[i] = v;
        ramLak[L - i] = v;
    }
    float* ccs = (float*)malloc(sizeof(float) * (L + 2));
    jo_rfft_forward(ccs, ramLak, L);
    /* GenerateFilter (FilterCore.cpp:69-138) */
    float* freq = (float*)malloc(sizeof(float) * nf);
    for (int i = 0; i < nf; ++i) freq[i] = (float)i * halfSampleRate * 2.0f / (float)L;
    const int n = nAdj + 2;
    float* ax = (float*)malloc(sizeof(float) * n);
    float* ay = (float*)malloc(sizeof(float) * n);
    ax[0] = 0.0f; ay[0] = 0.0f;
    for (int i = 0; i < nAdj; ++i) { ax[i + 1] = adjPts[i]; ay[i + 1] = adjDB[i]; }
    ax[n - 1] = halfSampleRate; ay[n - 1] = 0.0f;
    for (int i = 0; i < n; ++i) ay[i] = powf(10, ay[i] / 20.0f);
    smooth_interp(H, ax, ay, n, freq, nf);
    const float halfPi = JO_PI_F * (float)0.5;
    if (cutStart == 0 && cutEnd == 0) {
        for (int i = 0; i < nf; ++i) {
            const float f = freq[i];
            if (f < halfSampleRate) H[i] *= cosf(f / halfSampleRate * halfPi);
            else H[i] = 0.0f;
        }
    } else {
        for (int i = 0; i < nf; ++i) {
            const float f = freq[i];
            if (f <= cutStart) continue;
            else if (f < cutEnd)
                H[i] *= cosf((f - cutStart) / (cutEnd - cutStart) * JO_PI_F) * 0.5f + 0.5f;
            else H[i] = 0.0f;
        }
    }
    /* FilterCore.cpp:40-43: x RamLak real part, CCS magnitude, x pi*fN*2 */
    const float scale = JO_PI_F * halfSampleRate * 2.0f;
    for (int i = 0; i < nf; ++i) {
        H[i] = H[i] * ccs[2 * i];
        H[i] = H[i] * scale;
    }
    free(ramLak); free(ccs); free(freq); free(ax); free(ay);
}

/* h_eff[n] = (1/L) sum_k H_k cos(2 pi k n / L), H_{L-k} = H_k. */
void jo_filter_kernel_f64(double* h, const float* H, int L) {
    double* re = (double*)malloc(sizeof(double) * L);
    double* im = (double*)malloc(sizeof(double) * L);
    for (int k = 0; k <= L / 2; ++k) { re[k] = H[k]; im[k] = 0.0; }
    for (int k = L / 2 + 1; k < L; ++k) { re[k] = H[L - k]; im[k] = 0.0; }
    fft_c2c_pow2(re, im, L, +1);
    for (int i = 0; i < L; ++i) h[i] = re[i] / L;
    free(re); free(im);
}

/* FilterCore::ProcessRow with pre-weight (FilterCore.cpp:189-222). */
void jo_filter_rows(float* out, const float* in, const float* preweight,
                    int rows, int W, int Wout, int mirror, const float* H, int L) {
    const int R = (L - W) / 2;                       /* ramp length :46 */
    const int off = mirror ? Wout : 0;               /* outputOffset :28 */
    float* ramp = (float*)malloc(sizeof(float) * (R > 0 ? R : 1));
    for (int i = 0; i < R; ++i)
        ramp[i] = mirror ? (float)(R - 1 - i) / (float)R : (float)i / (float)R; /* :47-60 */
    float* buf = (float*)malloc(sizeof(float) * L);
    double* re = (double*)malloc(sizeof(double) * L);
    double* im = (double*)malloc(sizeof(double) * L);
    for (int r = 0; r < rows; ++r) {
        const float* x = in + (size_t)r * W;
        memcpy(buf, x, sizeof(float) * W);
        for (int i = W; i < L; ++i) buf[i] = 0.0f;
        if (preweight) {
            const float* pw = preweight + (size_t)r * L;
            for (int i = 0; i < L; ++i) buf[i] = buf[i] * pw[i];
        }
        if (mirror) {
            const float edge = (x[W - 1] + x[W - 2] + x[W - 3]) / 3.0f;
            for (int k = 0; k < R; ++k) buf[W + k] = ramp[k] * edge;
        } else {
            const float edge = (x[0] + x[1] + x[2]) / 3.0f;
            for (int k = 0; k < R; ++k) buf[L - R + k] = ramp[k] * edge;
        }
        for (int i = 0; i < L; ++i) { re[i] = buf[i]; im[i] = 0.0; }
        fft_c2c_pow2(re, im, L, -1);
        for (int k = 0; k < L; ++k) {
            const double h = (k <= L / 2) ? H[k] : H[L - k];
            re[k] *= h; im[k] *= h;
        }
        fft_c2c_pow2(re, im, L, +1);
        float* y = out + (size_t)r * Wout;
        for (int j = 0; j < Wout; ++j) y[j] = (float)(re[off + j] / L);
    }
    free(ramp); free(buf); free(re); free(im);
}

/* FP64 oracle of FilterCore::ProcessRow: the same steps as jo_filter_rows
 * (pre-weight product, truncation ramp of the edge mean, filtering by H over
 * L points, crop) with every buffer and operation in double. */
void jo_filter_rows_f64(double* out, const float* in, const float* preweight,
                        int rows, int W, int Wout, int mirror, const float* H, int L) {
    const int R = (L - W) / 2;
    const int off = mirror ? Wout : 0;
    double* re = (double*)malloc(sizeof(double) * L);
    double* im = (double*)malloc(sizeof(double) * L);
    for (int r = 0; r < rows; ++r) {
        const float* x = in + (size_t)r * W;
        for (int i = 0; i < L; ++i) {
            double v = i < W ? (double)x[i] : 0.0;
            if (preweight) v *= (double)preweight[(size_t)r * L + i];
            re[i] = v;
            im[i] = 0.0;
        }
        if (mirror) {
            const double edge = ((double)x[W - 1] + x[W - 2] + x[W - 3]) / 3.0;
            for (int k = 0; k < R; ++k) re[W + k] = (double)(R - 1 - k) / R * edge;
        } else {
            const double edge = ((double)x[0] + x[1] + x[2]) / 3.0;
            for (int k = 0; k < R; ++k) re[L - R + k] = (double)k / R * edge;
        }
        fft_c2c_pow2(re, im, L, -1);
        for (int k = 0; k < L; ++k) {
            const double h = (k <= L / 2) ? H[k] : H[L - k];
            re[k] *= h; im[k] *= h;
        }
        fft_c2c_pow2(re, im, L, +1);
        double* y = out + (size_t)r * Wout;
        for (int j = 0; j < Wout; ++j) y[j] = re[off + j] / L;
    }
    free(re); free(im);
}

/* ======================================================================
 * Conjugate-view compositing -- CompositeAgent/CompositeCore.cpp
 * ==================================================================== */

/* CompositeCore::Process (CompositeCore.cpp:59-149) for one view: out is
 * [H][2W], the direct frame in one half and, in the other, the conjugate
 * frame resampled at the points the direct view's extended detector would
 * see, blended with the direct frame's edge over 40 columns. */
void jo_composite(float* out, const float* dirc, const float* conj, const float ptm_dirc[12],
                  const float ptm_conj[12], float dso, int W, int H, int detRight) {
    const int tw = 40, ew = 5;                       /* transWidth, edgeWidth :36-37 */
    const int W2 = 2 * W;
    for (size_t i = 0; i < (size_t)W2 * H; ++i) out[i] = 0.0f;
    /* TM of the direct view and its inverse (LinearEquationSolver, A X = I) */
    float tm[16], A[16], tinv[16];
    jo_ptm2tm(tm, ptm_dirc, dso);
    for (int i = 0; i < 16; ++i) { A[i] = tm[i]; tinv[i] = (i % 5 == 0) ? 1.0f : 0.0f; }
    jo_solve_f32(4, 4, A, tinv);
    const int conjOff = detRight ? 0 : W, dircOff = detRight ? W : 0;
    for (int r = 0; r < H; ++r) {
        for (int c = 0; c < W; ++c) {
            /* GenerateUVW1Grid :153-183: (u, v, 0, 1) beyond the direct edge */
            const float uvw[4] = {detRight ? (float)c - (float)W : (float)(c + W), (float)r, 0.0f, 1.0f};
            float xyz[4], q[3];
            for (int i = 0; i < 4; ++i) {               /* MatrixMultiplier 4x4 . 4x1 */
                float acc = 0.0f;
                for (int k = 0; k < 4; ++k) acc += tinv[i * 4 + k] * uvw[k];
                xyz[i] = acc;
            }
            for (int i = 0; i < 3; ++i) {               /* 3x4 . 4x1, the conjugate PTM */
                float acc = 0.0f;
                for (int k = 0; k < 4; ++k) acc += ptm_conj[i * 4 + k] * xyz[k];
                q[i] = acc;
            }
            const float u = q[0] / q[2];
            float v = q[1] / q[2];
            if (v < 0.0f) v = 0.0f;                     /* LowerBound, UpperBound :84-85 */
            if (v > (float)H - 1.0f) v = (float)H - 1.0f;
            /* ImgEditor::Remap, restated: written only inside the frame */
            if (!(u >= 0.0f && u <= (float)(W - 1) && v >= 0.0f && v <= (float)(H - 1))) continue;
            const int ix = (int)floorf(u), iy = (int)floorf(v);
            const int ix1 = ix + 1 < W ? ix + 1 : W - 1, iy1 = iy + 1 < H ? iy + 1 : H - 1;
            const float fx = u - (float)ix, fy = v - (float)iy;
            const float p00 = conj[(size_t)iy * W + ix], p01 = conj[(size_t)iy * W + ix1];
            const float p10 = conj[(size_t)iy1 * W + ix], p11 = conj[(size_t)iy1 * W + ix1];
            const float t0 = p00 + fx * (p01 - p00), t1 = p10 + fx * (p11 - p10);
            out[(size_t)r * W2 + conjOff + c] = t0 + fy * (t1 - t0);
        }
    }
    /* transition masks :195-223: direct 1 -> 0 (or 0 -> 1), conjugate 1 - that */
    float md[40], mc[40];
    for (int i = 0; i < tw; ++i) {
        md[i] = detRight ? cosf((float)i / (float)tw * JO_PI_F) * -0.5f + 0.5f
                         : cosf((float)i / (float)tw * JO_PI_F) * 0.5f + 0.5f;
        mc[i] = 1.0f - md[i];
    }
    const int transOff = detRight ? W - tw : W, tempOff = detRight ? W : 0;
    for (int r = 0; r < H; ++r) {
        float* o = out + (size_t)r * W2;
        for (int i = 0; i < tw; ++i) o[transOff + i] = o[transOff + i] * mc[i];
        /* the direct row's edge mean (ippsMean over 5 samples: summed in
         * double, divided in float) into the temporary region :103-124 */
        const float* d = dirc + (size_t)r * W + (detRight ? 0 : W - ew);
        double sum = 0.0;
        for (int i = 0; i < ew; ++i) sum += d[i];
        const float edge = (float)sum / (float)ew;
        for (int i = 0; i < tw; ++i) o[tempOff + i] = edge * md[i];
        for (int i = 0; i < tw; ++i) o[transOff + i] = o[transOff + i] + o[tempOff + i];
        for (int i = 0; i < W; ++i) o[dircOff + i] = dirc[(size_t)r * W + i];
    }
}

/* ======================================================================
 * Backprojection -- BPAgent/BPCore.cpp
 * ==================================================================== */

/* BPCore.cpp:68-100: the u-taper of each view, from the isocentre's column. */
void jo_bp_uweights(float* w, const float* ptms, int nViews, int U) {
    for (int v = 0; v < nViews; ++v) {
        const float* P = ptms + (size_t)v * 12;
        float* wv = w + (size_t)v * U;
        const float uf = P[3] / P[11];        /* uvw = P (0,0,0,1)^T */
        long u = (uf >= 0.0f) ? (long)uf : 0; /* size_t(u) truncation */
        for (int i = 0; i < U; ++i) wv[i] = 1.0f;
        if (u > U / 2) {
            const long nTrans = (U - u) * 2;
            for (long i = 0; i < nTrans; ++i)
                wv[U - nTrans + i] = cosf((float)i * JO_PI_F / (float)nTrans) * 0.5f + 0.5f;
        } else {
            const long nTrans = u * 2;
            for (long i = 0; i < nTrans; ++i)
                wv[i] = cosf((float)i * JO_PI_F / (float)nTrans) * -0.5f + 0.5f;
        }
    }
}

/* Volume axes: BPCore.cpp:47-66 (start at -(n-1)/2, step 1, times pitch). */
static void make_axis(float* a, int n, float pitch) {
    float x = -((float)n - 1.0f) / 2.0f;
    for (int i = 0; i < n; ++i) { a[i] = x; x = x + 1.0f; }
    for (int i = 0; i < n; ++i) a[i] = a[i] * pitch;
}

typedef struct {
    float* sumf; float* cntf; double* sumd; double* cntd;
    const float* proj; const float* ptms; const float* uw;
    int v0, nv, U, V, X, Y, Z; float pitchXY, pitchZ; int zb, ze, z0;
} bp_job;

/* ippiRemap_32f_C1R, IPPI_INTER_LINEAR, as restated here: a destination
 * pixel is written only when 0 <= x <= W-1 and 0 <= y <= H-1, with pixel
 * centres at integer coordinates; the +1 neighbour is clamped to the last
 * column/row (its weight is then exactly 0). */
static void* bp_worker(void* arg) {
    bp_job* j = (bp_job*)arg;
    const int U = j->U, V = j->V, X = j->X, Y = j->Y;
    float* ax = (float*)malloc(sizeof(float) * X);
    float* ay = (float*)malloc(sizeof(float) * Y);
    float* az = (float*)malloc(sizeof(float) * j->Z);
    make_axis(ax, X, j->pitchXY);
    make_axis(ay, Y, j->pitchXY);
    make_axis(az, j->Z, j->pitchZ);
    float* pt = (float*)malloc(sizeof(float) * (size_t)U * V);
    for (int iv = 0; iv < j->nv; ++iv) {
        const int view = j->v0 + iv;
        const float* P = j->ptms + (size_t)view * 12;
        const float* w = j->uw + (size_t)view * U;
        const float* src = j->proj + (size_t)iv * U * V;
        for (int r = 0; r < V; ++r)            /* InitView :147-151 */
            for (int c = 0; c < U; ++c) pt[(size_t)r * U + c] = src[(size_t)r * U + c] * w[c];
        for (int z = j->zb; z < j->ze; ++z) {
            const float zu = az[z] * P[2], zv = az[z] * P[6], zw = az[z] * P[10];
            const size_t zoff = (size_t)(z - j->z0) * X * Y;
            for (int y = 0; y < Y; ++y) {
                const float yu = ay[y] * P[1] + P[3];   /* YxPM1 + PM3 :142-144 */
                const float yv = ay[y] * P[5] + P[7];
                const float yw = ay[y] * P[9] + P[11];
                for (int x = 0; x < X; ++x) {
                    const float Uxy = ax[x] * P[0] + yu;
                    const float Vxy = ax[x] * P[4] + yv;
                    const float Wxy = ax[x] * P[8] + yw;
                    float u = Uxy + zu, vv = Vxy + zv;  /* CalculateUV :207-220 */
                    const float W = Wxy + zw;
                    u = u / W; vv = vv / W;
                    u = u + 0.5f; vv = vv + 0.5f;
                    if (!(u >= 0.0f && u <= (float)(U - 1) && vv >= 0.0f && vv <= (float)(V - 1)))
                        continue;
                    const int ix = (int)floorf(u), iy = (int)floorf(vv);
                    const int ix1 = ix + 1 < U ? ix + 1 : U - 1;
                    const int iy1 = iy + 1 < V ? iy + 1 : V - 1;
                    const size_t idx = zoff + (size_t)y * X + x;
                    if (j->sumf) {
                        const float fx = u - (float)ix, fy = vv - (float)iy;
                        const float p00 = pt[(size_t)iy * U + ix], p01 = pt[(size_t)iy * U + ix1];
                        const float p10 = pt[(size_t)iy1 * U + ix], p11 = pt[(size_t)iy1 * U + ix1];
                        const float t0 = p00 + fx * (p01 - p00);
                        const float t1 = p10 + fx * (p11 - p10);
                        const float val = t0 + fy * (t1 - t0);
                        const float c = w[ix] + fx * (w[ix1] - w[ix]);
                        j->sumf[idx] = j->sumf[idx] + val;   /* BPCore.cpp:192-193 */
                        j->cntf[idx] = j->cntf[idx] + c;
                    } else {
                        const double fx = (double)u - ix, fy = (double)vv - iy;
                        const double p00 = pt[(size_t)iy * U + ix], p01 = pt[(size_t)iy * U + ix1];
                        const double p10 = pt[(size_t)iy1 * U + ix], p11 = pt[(size_t)iy1 * U + ix1];
                        const double t0 = p00 + fx * (p01 - p00);
                        const double t1 = p10 + fx * (p11 - p10);
                        j->sumd[idx] += t0 + fy * (t1 - t0);
                        j->cntd[idx] += (double)w[ix] + fx * ((double)w[ix1] - w[ix]);
                    }
                }
            }
        }
    }
    free(ax); free(ay); free(az); free(pt);
    return NULL;
}

static void bp_run(float* sumf, float* cntf, double* sumd, double* cntd,
                   const float* proj, const float* ptms, const float* uw, int v0, int nv,
                   int U, int V, int X, int Y, int Z, float pitchXY, float pitchZ,
                   int z0, int nz, int nthreads) {
    if (nthreads < 1) nthreads = 1;
    if (nthreads > nz) nthreads = nz > 0 ? nz : 1;
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * nthreads);
    bp_job* jobs = (bp_job*)malloc(sizeof(bp_job) * nthreads);
    for (int t = 0; t < nthreads; ++t) {
        bp_job j = {sumf, cntf, sumd, cntd, proj, ptms, uw, v0, nv, U, V, X, Y, Z,
                    pitchXY, pitchZ, z0 + (int)((long)nz * t / nthreads),
                    z0 + (int)((long)nz * (t + 1) / nthreads), z0};
        jobs[t] = j;
        pthread_create(&th[t], NULL, bp_worker, &jobs[t]);
    }
    for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
    free(th); free(jobs);
}

void jo_bp_accumulate(float* sum, float* cnt, const float* proj, const float* ptms,
                      const float* uw, int v0, int nv, int U, int V, int X, int Y, int Z,
                      float pitchXY, float pitchZ, int z0, int nz, int nthreads) {
    bp_run(sum, cnt, NULL, NULL, proj, ptms, uw, v0, nv, U, V, X, Y, Z, pitchXY, pitchZ,
           z0, nz, nthreads);
}

void jo_bp_accumulate_f64(double* sum, double* cnt, const float* proj, const float* ptms,
                          const float* uw, int v0, int nv, int U, int V, int X, int Y, int Z,
                          float pitchXY, float pitchZ, int z0, int nz, int nthreads) {
    bp_run(NULL, NULL, sum, cnt, proj, ptms, uw, v0, nv, U, V, X, Y, Z, pitchXY, pitchZ,
           z0, nz, nthreads);
}

/* FP64 oracle of BPCore for a list of voxels: the same rule as bp_worker
 * (taper product, u = U/W + 0.5, v = V/W + 0.5, sample only when
 * 0 <= u <= U-1 and 0 <= v <= V-1, bilinear lerps, sum and weight) with the
 * axes, coordinates, projections and arithmetic in double. */
typedef struct {
    double* sum; double* cnt; const double* proj; const double* ptms; const float* uw;
    int v0, nv, U, V, X, Y, Z; double pitchXY, pitchZ; const int* pts; int p0, p1;
} bpp_job;

static void* bpp_worker(void* arg) {
    /* Points in blocks of BPP_BLOCK, views inside a block: a view's rows stay
     * in cache while the block's points sample them (a view per point misses
     * the cache on every sample).  The sums per point run over the views in
     * order. */
    enum { BPP_BLOCK = 1024 };
    bpp_job* j = (bpp_job*)arg;
    const int U = j->U, V = j->V;
    double xs[BPP_BLOCK], ys[BPP_BLOCK], zs[BPP_BLOCK], ss[BPP_BLOCK], cs[BPP_BLOCK];
    for (int b = j->p0; b < j->p1; b += BPP_BLOCK) {
        const int n = j->p1 - b < BPP_BLOCK ? j->p1 - b : BPP_BLOCK;
        for (int k = 0; k < n; ++k) {
            const int i = b + k;
            xs[k] = ((double)j->pts[3 * i] - (j->X - 1) / 2.0) * j->pitchXY;
            ys[k] = ((double)j->pts[3 * i + 1] - (j->Y - 1) / 2.0) * j->pitchXY;
            zs[k] = ((double)j->pts[3 * i + 2] - (j->Z - 1) / 2.0) * j->pitchZ;
            ss[k] = 0.0;
            cs[k] = 0.0;
        }
        for (int iv = 0; iv < j->nv; ++iv) {
            const int view = j->v0 + iv;
            const double* P = j->ptms + (size_t)view * 12;
            const double* p = j->proj + (size_t)iv * U * V;
            const float* w = j->uw + (size_t)view * U;
            for (int k = 0; k < n; ++k) {
                const double x = xs[k], y = ys[k], z = zs[k];
                const double Uc = x * P[0] + y * P[1] + z * P[2] + P[3];
                const double Vc = x * P[4] + y * P[5] + z * P[6] + P[7];
                const double Wc = x * P[8] + y * P[9] + z * P[10] + P[11];
                const double u = Uc / Wc + 0.5, v = Vc / Wc + 0.5;
                if (!(u >= 0.0 && u <= U - 1 && v >= 0.0 && v <= V - 1)) continue;
                const int ix = (int)floor(u), iy = (int)floor(v);
                const int ix1 = ix + 1 < U ? ix + 1 : U - 1;
                const int iy1 = iy + 1 < V ? iy + 1 : V - 1;
                const double fx = u - ix, fy = v - iy;
                const double p00 = p[(size_t)iy * U + ix] * w[ix], p01 = p[(size_t)iy * U + ix1] * w[ix1];
                const double p10 = p[(size_t)iy1 * U + ix] * w[ix], p11 = p[(size_t)iy1 * U + ix1] * w[ix1];
                const double t0 = p00 + fx * (p01 - p00), t1 = p10 + fx * (p11 - p10);
                ss[k] += t0 + fy * (t1 - t0);
                cs[k] += (double)w[ix] + fx * ((double)w[ix1] - w[ix]);
            }
        }
        for (int k = 0; k < n; ++k) {
            j->sum[b + k] += ss[k];
            j->cnt[b + k] += cs[k];
        }
    }
    return NULL;
}

void jo_bp_points_f64d(double* sum, double* cnt, const double* proj, const double* ptms,
                       const float* uw, int v0, int nv, int U, int V, const int* pts, int npts,
                       int X, int Y, int Z, float pitchXY, float pitchZ, int nthreads) {
    if (nthreads < 1) nthreads = 1;
    if (nthreads > npts) nthreads = npts > 0 ? npts : 1;
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * nthreads);
    bpp_job* jobs = (bpp_job*)malloc(sizeof(bpp_job) * nthreads);
    for (int t = 0; t < nthreads; ++t) {
        bpp_job jb = {sum, cnt, proj, ptms, uw, v0, nv, U, V, X, Y, Z, pitchXY, pitchZ, pts,
                      (int)((long)npts * t / nthreads), (int)((long)npts * (t + 1) / nthreads)};
        jobs[t] = jb;
        pthread_create(&th[t], NULL, bpp_worker, &jobs[t]);
    }
    for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
    free(th); free(jobs);
}

void jo_bp_points_f64(double* sum, double* cnt, const double* proj, const float* ptms,
                      const float* uw, int v0, int nv, int U, int V, const int* pts, int npts,
                      int X, int Y, int Z, float pitchXY, float pitchZ, int nthreads) {
    const int nviews = v0 + nv;
    double* pd = (double*)malloc(sizeof(double) * 12 * (size_t)nviews);
    for (size_t i = 0; i < 12 * (size_t)nviews; ++i) pd[i] = ptms[i];
    jo_bp_points_f64d(sum, cnt, proj, pd, uw, v0, nv, U, V, pts, npts, X, Y, Z, pitchXY, pitchZ, nthreads);
    free(pd);
}

/* Where voxels project, in double (test bookkeeping for the FP64 checks):
 * interior[i] = 1 when every view samples point i at least `margin` pixels
 * inside the detector; vrange = the smallest and largest v of the samples
 * that fall inside the detector (0 <= u <= U-1, 0 <= v <= V-1), over all
 * points and views (vrange[0] > vrange[1] when there are none). */
typedef struct {
    const int* pts; int p0, p1; const double* ptms; int nv, X, Y, Z; double pxy, pz; int U, V; double margin;
    unsigned char* interior; double vmin, vmax;
} survey_job;

static void* survey_worker(void* arg) {
    survey_job* j = (survey_job*)arg;
    j->vmin = 1e300;
    j->vmax = -1e300;
    for (int i = j->p0; i < j->p1; ++i) {
        const double x = ((double)j->pts[3 * i] - (j->X - 1) / 2.0) * j->pxy;
        const double y = ((double)j->pts[3 * i + 1] - (j->Y - 1) / 2.0) * j->pxy;
        const double z = ((double)j->pts[3 * i + 2] - (j->Z - 1) / 2.0) * j->pz;
        int inside = 1;
        for (int k = 0; k < j->nv; ++k) {
            const double* P = j->ptms + (size_t)k * 12;
            const double Wc = x * P[8] + y * P[9] + z * P[10] + P[11];
            const double u = (x * P[0] + y * P[1] + z * P[2] + P[3]) / Wc + 0.5;
            const double v = (x * P[4] + y * P[5] + z * P[6] + P[7]) / Wc + 0.5;
            if (!(u >= j->margin && u <= j->U - 1 - j->margin && v >= j->margin && v <= j->V - 1 - j->margin))
                inside = 0;
            if (u >= 0.0 && u <= j->U - 1 && v >= 0.0 && v <= j->V - 1) {
                if (v < j->vmin) j->vmin = v;
                if (v > j->vmax) j->vmax = v;
            }
        }
        j->interior[i] = (unsigned char)inside;
    }
    return NULL;
}

void jo_points_survey(unsigned char* interior, double* vrange, const int* pts, int npts, const double* ptms,
                      int nv, int X, int Y, int Z, double pitchXY, double pitchZ, int U, int V, double margin,
                      int nthreads) {
    if (nthreads < 1) nthreads = 1;
    if (nthreads > npts) nthreads = npts > 0 ? npts : 1;
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * nthreads);
    survey_job* jobs = (survey_job*)malloc(sizeof(survey_job) * nthreads);
    for (int t = 0; t < nthreads; ++t) {
        survey_job jb = {pts, (int)((long)npts * t / nthreads), (int)((long)npts * (t + 1) / nthreads), ptms, nv,
                         X, Y, Z, pitchXY, pitchZ, U, V, margin, interior, 0.0, 0.0};
        jobs[t] = jb;
        pthread_create(&th[t], NULL, survey_worker, &jobs[t]);
    }
    vrange[0] = 1e300;
    vrange[1] = -1e300;
    for (int t = 0; t < nthreads; ++t) {
        pthread_join(th[t], NULL);
        if (jobs[t].vmin < vrange[0]) vrange[0] = jobs[t].vmin;
        if (jobs[t].vmax > vrange[1]) vrange[1] = jobs[t].vmax;
    }
    free(th);
    free(jobs);
}

/* BPCore::DoneSlice (BPCore.cpp:198-205): out = sum / cnt. */
void jo_bp_finalize(float* out, const float* sum, const float* cnt, size_t n) {
    for (size_t i = 0; i < n; ++i) out[i] = sum[i] / cnt[i];
}

/* ======================================================================
 * CT numbers -- CTNumAgent/CTNumCore.cpp:22-36
 * ==================================================================== */
void jo_ctnum(float* p, size_t n, float norm0, float norm1, float muWater) {
    const float s = norm0 * 1000.f / muWater;
    for (size_t i = 0; i < n; ++i) {
        float h = p[i] * s;
        h = h - 1000.f;
        if (h > 300.0f) {
            const float t = (h - 300.0f) * norm1 + 300.0f;
            h = (t < 8191.f) ? t : 8191.f; /* std::min(8191.f, t) */
        }
        p[i] = h;
    }
}

void jo_to_int16(int16_t* out, const float* in, size_t n) {
    for (size_t i = 0; i < n; ++i) {
        const float f = in[i];
        if (f != f) { out[i] = 0; continue; }
        const float t = truncf(f);
        out[i] = t >= 32767.0f ? 32767 : (t <= -32768.0f ? -32768 : (int16_t)t);
    }
}
