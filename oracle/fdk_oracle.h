/*
 * fdk_oracle.h -- CPU restatement of the JEngine FDK hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the
 * CUDA engine in jenhine_b200/csrc.  Only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline / --impl reference legs may load it.  The
 * product path never calls into it (and has no CPU fallback).
 *
 * Every function restates one piece of the reference and cites the file:line
 * it follows (paths are relative to the JEngine source tree).  Single
 * precision functions reproduce the reference's float operation order
 * (compiled with -ffp-contract=off so that no FMA contraction changes the
 * rounding).  The *_f64 functions are the FP64 oracle used to state the error
 * of the reduced-precision forms.
 *
 * Parity pinning: the restatement is checked against the golden values of the
 * reference's own unit tests (UTPreFilterWeightGenerator, UTTransformMatrix,
 * UTRealFFT, UTProjectionMatrixModifier) and against the reference Core
 * classes compiled from source with project shims for IPP/MKL (oracle/_ref).
 */
#ifndef JFDK_ORACLE_H
#define JFDK_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- geometry (TransformMatrix/) ------------------------------------- */
void jo_ptm_move_u(float ptm[12], float u);
void jo_ptm_move_v(float ptm[12], float v);
void jo_ptm_reverse_x(float ptm[12]);
void jo_ptm_reverse_y(float ptm[12]);
void jo_ptm_move_z(float ptm[12], float z);
void jo_ptm2tm(float tm[16], const float ptm[12], float dso);
/* Solve A X = B in float (Gaussian elimination, partial pivoting); A is m*m,
 * B is m*p, both row-major, overwritten (A by its LU factors, B by X).
 * Returns 0, or i+1 when pivot i is exactly zero. */
int jo_solve_f32(int m, int p, float* A, float* B);
int jo_solve_f64(int m, int p, double* A, double* B);

/* ---- preprocessing (PreProcessingAgent/) ----------------------------- */
/* in: uint16 [inH][inW]; out: float [outH][outW].  Only the identity resize
 * (ROI size == output size) is restated; returns -1 otherwise. */
int jo_preprocess(float* out, const uint16_t* in, int inW, int inH,
                  int bUp, int bDown, int bLeft, int bRight, int outW, int outH,
                  float brightField, const float bhc[3]);

/* ---- pre-filter cosine weight (FilterAgent/PreFilterWeightGenerator) - */
/* weights: [height][L] with L = jo_fft_length(inputWidth).  tm_inv is the
 * inverse of the 4x4 transform matrix of the chosen view. */
void jo_preweight_generate(float* weights, const float tm_inv[16],
                           int inputWidth, int height, int detOnRight);
/* Full reference procedure for one view: PTM2TM, float inverse, Generate. */
void jo_preweight_for_view(float* weights, const float ptm[12], float dso,
                           int inputWidth, int height, int detOnRight);
/* View whose PTM generates the weight used for view v (9-view grouping). */
int jo_preweight_source_view(int v, int numViews);

/* ---- ramp filter (FilterAgent/FilterCore, Performance/RealFFT) ------- */
int jo_fft_length(int width);
/* Real FFT in CCS layout (length n+2 for even n, n+1 rounded up to even for
 * odd n), computed in double, stored in float.  Backward includes 1/n. */
void jo_rfft_forward(float* ccs, const float* x, int n);
void jo_rfft_backward(float* x, const float* ccs, int n);
/* Filter spectrum H[0..L/2] (RamLak x window x dB spline x 2*pi*fN). */
void jo_filter_spectrum(float* H, int L, float halfSampleRate,
                        float cutStart, float cutEnd,
                        const float* adjPts, const float* adjDB, int nAdj);
/* FilterCore::ProcessRow over `rows` rows.  in: [rows][W]; out: [rows][Wout];
 * preweight: [rows][L] or NULL.  FFT math in double, buffers in float. */
void jo_filter_rows(float* out, const float* in, const float* preweight,
                    int rows, int W, int Wout, int mirror,
                    const float* H, int L);
/* The same in double throughout (FP64 oracle); out is double. */
void jo_filter_rows_f64(double* out, const float* in, const float* preweight,
                        int rows, int W, int Wout, int mirror, const float* H, int L);
/* Equivalent real, even space kernel h_eff[L] = IDFT_L(H) (double). */
void jo_filter_kernel_f64(double* h, const float* H, int L);

/* ---- conjugate-view compositing (CompositeAgent/CompositeCore) -------- */
/* One view: dirc, conj [H][W] preprocessed frames of views k and
 * (k + N/2) % N, out [H][2W]. */
void jo_composite(float* out, const float* dirc, const float* conj, const float ptm_dirc[12],
                  const float ptm_conj[12], float dso, int W, int H, int detRight);

/* ---- backprojection (BPAgent/BPCore) ---------------------------------- */
/* u-taper per view: w[nViews][U]. */
void jo_bp_uweights(float* w, const float* ptms, int nViews, int U);
/* Accumulate views [v0, v0+nv) of `proj` ([nv][V][U], already filtered and
 * NOT yet tapered) into sum/cnt for slices [z0, z0+nz) ([nz][Y][X]).  The
 * projections are multiplied by the view's u-taper exactly as InitView does
 * (into a private copy). */
void jo_bp_accumulate(float* sum, float* cnt, const float* proj,
                      const float* ptms, const float* uw, int v0, int nv,
                      int U, int V, int X, int Y, int Z, float pitchXY,
                      float pitchZ, int z0, int nz, int nthreads);
void jo_bp_accumulate_f64(double* sum, double* cnt, const float* proj,
                          const float* ptms, const float* uw, int v0, int nv,
                          int U, int V, int X, int Y, int Z, float pitchXY,
                          float pitchZ, int z0, int nz, int nthreads);
/* FP64 oracle for a list of voxels pts[npts][3] = (x, y, z) indices:
 * coordinates, taper product, lerps and sums in double; projections proj
 * [nv][V][U] in double, NOT yet tapered.  Adds into sum[npts], cnt[npts]. */
void jo_bp_points_f64(double* sum, double* cnt, const double* proj, const float* ptms,
                      const float* uw, int v0, int nv, int U, int V, const int* pts, int npts,
                      int X, int Y, int Z, float pitchXY, float pitchZ, int nthreads);
/* The same with FP64 projection matrices (finite-difference checks of the
 * geometry gradient); the u-taper uw stays as given. */
void jo_bp_points_f64d(double* sum, double* cnt, const double* proj, const double* ptms,
                       const float* uw, int v0, int nv, int U, int V, const int* pts, int npts,
                       int X, int Y, int Z, float pitchXY, float pitchZ, int nthreads);
/* interior[i]: every view samples point i at least `margin` pixels inside
 * the detector; vrange[2]: least and largest v of the in-detector samples.
 * Double precision; ptms [nv][12] in double. */
void jo_points_survey(unsigned char* interior, double* vrange, const int* pts, int npts, const double* ptms,
                      int nv, int X, int Y, int Z, double pitchXY, double pitchZ, int U, int V, double margin,
                      int nthreads);
/* out = sum / cnt (BPCore::DoneSlice). */
void jo_bp_finalize(float* out, const float* sum, const float* cnt, size_t n);

/* ---- CT numbers (CTNumAgent/CTNumCore) -------------------------------- */
void jo_ctnum(float* inout, size_t n, float norm0, float norm1, float muWater);
/* float -> int16 with round toward zero and saturation
 * (Performance/BasicMathIPP.cpp:224-227). */
void jo_to_int16(int16_t* out, const float* in, size_t n);

#ifdef __cplusplus
}
#endif
#endif
