// jfdk_internal.h -- context layout and helpers shared by the engine's
// translation units.  Not part of the public ABI (include/jfdk.h is).
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/jfdk.h"

namespace jfdk {

// Host-side operators derived from the geometry and filter parameters
// (geometry.cpp).  All are per-context constants.
struct HostOperators {
    std::vector<float> uw;      // [views][out_w]   BP u-taper (BPCore.cpp:68-100)
    std::vector<float> tinv;    // [groups][16]     inverse TM per 9-view group
    std::vector<float> tinv_view;  // [views][16]   inverse TM per view, float solve (compositing)
    std::vector<float> T;       // [out_w][in_w]    ramp operator (Toeplitz)
    std::vector<double> h;      // [L]              its kernel in double: T[j][i] = h[(off + j - i) mod L]
    int off = 0;                // output offset of the kernel (FilterCore.cpp:28)
    std::vector<float> c;       // [out_w]          edge-ramp response
    std::vector<float> H;       // [L/2+1]          filter spectrum
};

int fft_length(int width);  // FilterCore::CalFFTLength
// Fills ops from the context's parameters; returns "" or an error message.
std::string build_host_operators(const jfdk_scan_params& scan, const jfdk_recon_params& recon,
                                 const std::vector<float>& adj_pts,
                                 const std::vector<float>& adj_db, const float* ptms,
                                 int in_w, int out_w, int rows, int mirror, float hsr,
                                 HostOperators& ops);

// Backprojection CTA: kBPTileX x kBPTileY threads over (x, y) by default and
// in the batch kernel, each thread a run of slices in z (4 or 8 per thread).
constexpr int kBPTileX = 4;
constexpr int kBPTileY = 32;

// Parameters of the backprojection kernel (bp.cu).
struct BPParams {
    const float4* q4;        // quads, [slots][rows][U]: (p[r][c], p[r+1][c], p[r][c+1] - p[r][c], p[r+1][c+1] - p[r+1][c])
    const float2* tw;        // [views][U] taper pairs (w[c], RN(w[c+1] - w[c])), w[U] = 0
    const uint2* qh;         // mixed precision: 8-byte records [slots][rows][U] (bp.cu)
    const float* qscale;     // mixed precision: [views] power-of-two scale of each view
    const float* ptm;        // [views][12]
    long long q4_frame;      // quads per slot (rows * U)
    int view_base;           // rotation index held by slot 0
    int v0, nv;              // views to accumulate (rotation indices)
    int U, V;                // columns, rows
    int X, Y, Z;
    float pxy, pz;
    int z_begin, z_end;      // slices handled by this launch
    float* sum;              // accumulators (chunked mode): [slices][Y][X] from slice acc_z0
    float* cnt;
    int acc_z0;
    int load_acc;            // add to sum/cnt already in memory
    float* out;              // finalize: [slices][Y][X] float from slice out_z0, or null
    int16_t* out16;          // finalize: int16 HU, the same layout, or null
    int out_z0;
    int apply_ct;
    float ct_scale, ct_norm1;
    // finalize over every view of the rotation: the normalisation weights of
    // the whole volume [Z][Y][X] (launch_bp_weights / launch_bp_mixed_weights),
    // so the view loop accumulates the projections only; null: accumulated
    // per sample
    const float* wvol;
};

// One scan of a batched backprojection (bp_batch_kernel): its parameters
// (finalizing launch over all its views), its grid and its first tile in the
// batch's work list.
struct BatchScan {
    BPParams p;
    unsigned first_tile;
    int gx, gy, gz;
    int zpt;                 // 4 or 8; 16 (mixed form) in a launch of 16-slice tiles only
    int wz;                  // W depends on z
    int pad[2];
};

// Launchers (return cudaError_t of the launch).
// zpt: slices per thread (4, 8 or 16); tile_x: CTA width in x, 4, 8 or 32
// (CTAs of 128 threads; other values and 16-slice tiles take 4).
cudaError_t launch_bp(const BPParams& p, bool finalize, bool exact, bool w_depends_on_z, int zpt, int tile_x,
                      cudaStream_t s);
// The FP32 form's normalisation weights of every voxel of the volume over
// every view of the rotation (p.v0 = 0, p.nv = all views, slices
// [p.z_begin, p.z_end)), into out [Z][Y][X] at absolute slices: the weight
// sums bp_kernel accumulates beside the projections, bit for bit (the same
// coordinates, taper lerp and view order).
cudaError_t launch_bp_weights(const BPParams& p, bool exact, bool w_depends_on_z, int zpt, int tile_x, float* out,
                              cudaStream_t s);
// The same for the mixed form (its coordinates, range test and FP32 taper lerp).
cudaError_t launch_bp_mixed_weights(const BPParams& p, bool w_depends_on_z, int zpt, int tile_x, float* out,
                                    cudaStream_t s);
// A batched backprojection launch covers up to kBatchSlots scans that share
// whether W depends on z (each with its own tile depth, 4 or 8 slices, or
// all of them the mixed form's 16); their
// parameters travel in the kernel's parameter space (16 slots: ~4.4 KB of the
// 32 KB a launch may carry).
constexpr int kBatchSlots = 16;
struct BatchSlots {
    BatchScan s[kBatchSlots];
};
// All tiles of nscans scans in one persistent launch of `ctas` CTAs (the
// SMs' resident CTAs); *counter is the work-list cursor (cleared here).
cudaError_t launch_bp_batch(const BatchSlots& t, int nscans, unsigned total_tiles, bool mixed_form, bool wz,
                            bool wv, unsigned* counter, int ctas, cudaStream_t s);
// CTAs of a full persistent wave: SMs x resident CTAs per SM.
cudaError_t bp_batch_ctas(bool mixed_form, bool wz, bool wv, bool deep, int* ctas);
// The context's backprojection store for every view (allocated if missing).
jfdk_status ensure_store(jfdk_ctx* c);
// Mixed-precision form: FP16 footprints with a per-view scale (qh, qscale).
cudaError_t launch_bp_mixed(const BPParams& p, bool finalize, bool w_depends_on_z, int zpt, int tile_x,
                            cudaStream_t s);
// absmax[f] = bit pattern of max |plain[f][...]| over each of nv frames.
cudaError_t launch_frame_absmax(const float* plain, long long frame, int nv, unsigned* absmax, cudaStream_t s);
// Filtered frames -> mixed-precision records in slots [slot0, slot0 + nv);
// writes the scale of rotation view (view0 + f) mod num_views to scale[].
cudaError_t launch_pack_mixed(const float* plain, long long plain_frame, int nv, int rows, int U, const float2* tw,
                              int view0, int num_views, const unsigned* absmax, float* scale, uint2* qh,
                              long long q_frame, int slot0, cudaStream_t s);
// Filtered frames [nv][rows][U] -> quads in slots [slot0, slot0 + nv), tapered
// with the taper of rotation view (view0 + f) when apply_taper.
cudaError_t launch_pack_quads(const float* plain, long long plain_frame, int nv, int rows, int U, const float2* tw,
                              int view0, int num_views, int apply_taper, float4* q4, long long q4_frame, int slot0,
                              cudaStream_t s);
cudaError_t launch_finalize(const float* sum, const float* cnt, size_t n, int apply_ct,
                            float ct_scale, float norm1, float* out, int16_t* out16,
                            cudaStream_t s);
cudaError_t launch_ctnum(float* d, size_t n, float ct_scale, float norm1, cudaStream_t s);

// Conjugate-view compositing (CompositeCore): the direct frame of view k in
// one half of a 2W-wide row, the frame of view (k + N/2) % N resampled into the
// other half, blended over 40 columns with the direct edge.
struct CompositeParams {
    const float* tinv;       // [views][16] inverse TM of each view
    const float* ptm;        // [views][12]
    const float* mask;       // [80]: the direct frame's transition mask, then the conjugate's
    int num_views;           // views per rotation
    int W, H;                // frame (half the composite row)
    int det_right;           // the detector sits right of the principal point: direct half on the right
};

struct PrepParams {
    const uint16_t* raw;     // [nv][in_h][in_w]
    int in_w, in_h, crop_x, crop_y;
    int width, rows;         // used (cropped) frame size
    float bright_field;
    float bhc0, bhc1, bhc2;
    int do_bhc;
    const uint16_t* raw_rotation;   // compositing: frame 0 of the rotation (conjugate frames), else null
    long long raw_frame;            // compositing: elements per raw frame
};
struct WeightParams {
    const float* tinv;       // [groups][16]
    const float* dmin;       // [groups]
    int num_views;           // views per rotation
    int L;                   // FFT length (pre-weight row length)
    int det_right;
    int mirror;
    const float* pw;         // [groups][rows][width] weights, or null: computed per row
    CompositeParams comp;    // comp.W > 0: rows are composited from raw frames first (width = 2 comp.W)
};
cudaError_t launch_preprocess(const PrepParams& p, int nv, float* out, cudaStream_t s);

// The ramp product's A operand as the weight kernels write it.
enum AOutKind { AOUT_F32 = 0, AOUT_TF32X2 = 1, AOUT_BF16X2 = 2, AOUT_FP16X2 = 3, AOUT_I8X4 = 4 };
struct AOperand {
    int kind;             // AOutKind
    void* hi;             // [M][pitch]: fp32 (F32, TF32X2), 16-bit values, or int8 digit plane 0 (I8X4)
    void* lo;             // low parts (split kinds); I8X4: digit plane 1 (planes lo - hi bytes apart)
    float* row_scale;     // FP16X2: [M] 1 / the row's power-of-two scale; I8X4: [M] 2^E of the row
    int pitch;            // elements per row (K padded)
};
// Digits of the int8 product: rows and operator as 32-bit fixed point below
// power-of-two scales (|x| <= 127 * 2^E, Q = round(x * 2^(24 - E))), each
// split into four balanced signed bytes, most significant first.
constexpr int kI8RowDigits = 4;
constexpr int kI8OpDigits = 4;
// Composite nv preprocessed direct / conjugate frame pairs of views
// v0.. into out [nv][H][2W] (CompositeAgent path).
cudaError_t launch_composite_frames(const float* dirc, const float* conj, int v0, int nv, const CompositeParams& c,
                                    float* out, cudaStream_t s);
// Pre-weight + edge mean of frames already preprocessed (agent path).
cudaError_t launch_weight(const float* in, int nv, int v0, int width, int rows, const WeightParams& w,
                          const AOperand& A, float* e, cudaStream_t s);
// Raw -> weighted A operand + edge means in one pass (whole-volume path).
cudaError_t launch_prep_weight(const PrepParams& p, int nv, int v0, const WeightParams& w, const AOperand& A,
                               float* e, cudaStream_t s);
// The table of pre-weights (needs dmin).
cudaError_t launch_preweight_table(const float* tinv, const float* dmin, int groups, int rows, int in_w,
                                   int det_right, float* pw, cudaStream_t s);
// Frame minimum of the pre-weight distance per group.
cudaError_t launch_preweight_dmin(const float* tinv, int groups, int rows, int L,
                                  int in_w, int det_right, float* dmin, cudaStream_t s);

struct RampParams {
    const float* A;          // [M][a_pitch]
    const float* e;          // [M]
    const float* B;          // [N][K] Toeplitz operator
    const float* c;          // [N]
    int M, N, K, a_pitch;
    int rows;                // rows per view (M = nv * rows)
    float* q;                // output frames, row r of view f at q + f * q_frame_stride + r * q_pitch
    long long q_frame_stride;
    int q_pitch;
    const float* row_scale;  // tensor-core FP16X3: [M] row factors, else null
    float b_scale;           // tensor-core FP16X3: 1 / the operator's scale, else 1
    int vec_store;           // q rows 16-byte aligned: store float4s
    unsigned* absmax;        // tensor-core kinds: [views] max |q| as float bits (atomicMax; zeroed by the caller), or null
};
cudaError_t launch_ramp_gemm(const RampParams& p, cudaStream_t s);
// Tensor-core split products (ramp_gemm_tc.cu).
enum RampKind { RAMP_TF32X3 = 0, RAMP_BF16X3 = 1, RAMP_FP16X3 = 2, RAMP_I8X14 = 3 };
// Ah, Al [M][a_pitch] and Bh, Bl [N][a_pitch] in the kind's element type;
// a_pitch a multiple of 32 (TF32X3) or 64.  A timed-out pipeline wait sets
// *status (device word) and the CTA skips the rest of its work.
cudaError_t launch_ramp_gemm_tc(const RampParams& p, int kind, const void* Ah, const void* Al, const void* Bh,
                                const void* Bl, int* status, cudaStream_t s);
float tf32_round_host(float x);
// The exact int8 product (ramp_gemm_tc.cu): A digit planes [kI8RowDigits]
// [M][a_pitch] (a_plane bytes apart, p.row_scale the rows' 2^E), operator
// digit planes [kI8OpDigits][N][a_pitch] (b_plane bytes apart, p.b_scale
// its 2^F), and per output tile x K block the mask of operator digit planes
// that are not all zero ([ceil(N / kI8TileN)][ceil(a_pitch / kI8BlockK)]).
constexpr int kI8TileN = 64;
constexpr int kI8BlockK = 128;
cudaError_t launch_ramp_i8(const RampParams& p, const int8_t* A, long long a_plane, const int8_t* B,
                           long long b_plane, const uint8_t* masks, int* status, cudaStream_t s);

// Derivatives (adjoint.cu).
struct AdjParams {
    const float* ptm;        // [views][12] backprojection geometry
    int v0, nv, num_views;   // views [v0, v0 + nv) of the rotation
    int U, V, X, Y, Z;
    float pxy, pz;
    const float* rt;         // [Z][Y][X] vol_bar / weight
    float4* qbar;            // adjoint out: quad space [nv][V][U]
    long long q_frame;       // V * U
    const float4* q4;        // gradient: the forward's tapered quads [nv][V][U]
    const float2* tw;        // [views][U] taper pairs (w[c], RN(w[c+1] - w[c]))
    const float* vol;        // gradient: the forward volume
    const float* dptm;       // gradient: [nv][6][12] dP / dtheta_j
    float* partial;          // gradient: [nv][ctas][6] scratch
};
cudaError_t launch_residual_over_weight(const float* vol_bar, const float* cnt, size_t n, float* rt, cudaStream_t s);
cudaError_t launch_bp_adjoint(const AdjParams& p, bool w_depends_on_z, cudaStream_t s);
cudaError_t launch_unpack_adjoint(const float4* qbar, long long q_frame, int nv, int rows, int U, const float2* tw,
                                  int view0, int num_views, float* out, cudaStream_t s);
size_t geometry_gradient_ctas(const AdjParams& p);
cudaError_t launch_geometry_gradient(const AdjParams& p, bool w_depends_on_z, double* grad, cudaStream_t s);
cudaError_t launch_pad_rows(const float* src, size_t rows, int w, float* dst, int pitch, cudaStream_t s);
cudaError_t launch_filter_adjoint_finish(const float* ybar, int out_w, float* xbar, int in_w, int rows, int nv, int v0,
                                         int num_views, const float* pw, const float* c, int mirror, cudaStream_t s);

cudaError_t launch_zfilter(float* frames, int nv, int rows, int width, long long frame_stride,
                           int pitch, cudaStream_t s);

}  // namespace jfdk

struct jfdk_ctx {
    jfdk_scan_params scan{};
    jfdk_recon_params recon{};
    std::vector<float> adj_pts, adj_db;
    int precision = 0;
    int device = 0;
    int sms = 148;                // the device's SMs
    cudaStream_t stream = nullptr;
    bool own_stream = false;

    // sizes
    int nviews = 0;
    int used_u = 0, used_v = 0;   // cropped frame
    int in_w = 0, out_w = 0;      // filter input / output widths
    int rows = 0, L = 0, mirror = 0;
    float hsr = 0.f;
    int X = 0, Y = 0, Z = 0;
    float pxy = 0.f, pz = 0.f;
    int groups = 0;
    float ct_scale = 0.f;

    std::vector<float> ptms;
    jfdk::HostOperators ops;
    bool w_depends_on_z = false;  // some view has P[10] != 0

    // device constants
    float* d_ptm = nullptr;
    float2* d_tw = nullptr;      // [views][out_w] taper pairs (w[c], RN(w[c+1] - w[c]))
    float* d_tinv = nullptr;
    float* d_dmin = nullptr;
    float* d_pw = nullptr;       // [groups][rows][in_w] pre-weights
    float* d_tinv_view = nullptr;  // [views][16] (compositing)
    float* d_cmask = nullptr;      // [80] compositing transition masks
    float* d_T = nullptr;
    float* d_Th = nullptr;       // TF32-exact split of the ramp operator
    float* d_Tl = nullptr;
    uint16_t* d_Tb = nullptr;    // BF16 split: [2][out_w][a_pitch] (high, low)
    uint16_t* d_Tf = nullptr;    // FP16 split of the scaled operator (high, low)
    float tf_inv_scale = 1.0f;   // 1 / the FP16 operator's scale
    float* d_Tt = nullptr;       // transposed operator [in_w][round64(out_w)] (filter adjoint)
    int8_t* d_Ti8 = nullptr;     // int8 digits of the operator [kI8OpDigits][out_w][a_pitch]
    uint8_t* d_i8mask = nullptr; // [ceil(out_w / kI8TileN)][a_pitch / kI8BlockK] non-zero digit planes
    float i8_scale = 1.0f;       // 2^F of the operator's digits
    float* d_czero = nullptr;    // [in_w] zeros
    float* d_c = nullptr;
    int* d_status = nullptr;     // nonzero: a kernel's bounded wait gave up

    // device working storage (allocated on demand)
    void* d_A = nullptr;  size_t a_rows = 0;    // weighted rows: high then low part, pitch a_pitch
    float* d_arow = nullptr;                     // FP16X3: per-row factors
    float* d_e = nullptr;
    float* d_plain = nullptr; int plain_views = 0;  // filtered frames of one chunk
    float4* d_q4 = nullptr; int q4_views = 0;       // quad store (mixed: 8-byte records)
    float* d_qscale = nullptr;                      // mixed: [views] scales
    unsigned* d_absmax = nullptr; int absmax_n = 0; // mixed: per-frame maxima
    float* d_sum = nullptr;                          // accumulators of the slab:
    float* d_cnt = nullptr;                          // [acc_slices][Y][X]
    int acc_slices = 0;                              // planes allocated
    int slab_z0 = 0, slab_nz = 0;                    // jfdk_bp_set_slab (nz 0: every slice)
    uint16_t* d_raw_stage = nullptr; size_t raw_stage_bytes = 0;
    float* d_hu_stage = nullptr; size_t hu_stage_bytes = 0;
    bool bp_has_views = false;
    // derivatives (allocated on demand)
    float* d_rt = nullptr;                           // vol_bar / weight
    float4* d_qadj = nullptr; int qadj_views = 0;    // quad-space adjoint
    float* d_partial = nullptr; size_t partial_n = 0;
    float* d_dptm = nullptr; int dptm_views = 0;

    // JFDK_OPT_* settings
    int opt_bp_exact = 0;
    int opt_view_chunk = 32;
    int opt_stage_timing = 0;
    int opt_bp_zpt = 0;          // 0: default (bp_zpt() in jfdk_api.cpp)
    int opt_bp_tile = 0;         // tile width in x: 4, 8 or 32; 0: default (4)
    int opt_ramp = 0;            // JFDK_OPT_RAMP_PRODUCT (0: the form's default)
    int opt_bp_weights = 1;      // JFDK_OPT_BP_WEIGHTS
    float* d_wvol = nullptr;     // normalisation weights [Z][Y][X] (FP32 form)
    int wvol_state = 0;          // 0: none; valid for 1: the fast rounding, 2: EXACT, 100 + tile depth: the mixed form
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    // jfdk_reconstruct_host: a copy stream and a second compute stream, and
    // their events (created on first use)
    cudaStream_t copy_stream = nullptr, aux_stream = nullptr;
    std::vector<cudaEvent_t> xfer_ev;

    long long launches = 0;
    // device memory held (dev_alloc / dev_free) and the JFDK_OPT_DEVICE_MEMORY_LIMIT
    long long dev_bytes = 0, mem_limit = 0;
    std::unordered_map<const void*, size_t> alloc_bytes;
    std::string err;
};

namespace jfdk {
// Stages of jfdk_reconstruct, shared with the batch (batch.cpp).
// nviews: the first views only (the autotuner), or all when out of range.
// chunk_ready (optional): one event per chunk of views; the stage waits for
// chunk k's event before its first kernel (frames still in transfer).
jfdk_status reconstruct_filter_stage(jfdk_ctx* c, const uint16_t* d_raw, int nviews,
                                     const cudaEvent_t* chunk_ready = nullptr);
// The same for views [vbeg, vend) only (d_raw: the rotation's frames).
jfdk_status filter_stage_range(jfdk_ctx* c, const uint16_t* d_raw, int vbeg, int vend,
                               const cudaEvent_t* chunk_ready = nullptr);
BPParams reconstruct_bp_params(const jfdk_ctx* c, float* d_hu, int16_t* d_hu16);
// The finalizing backprojection of every view into d_hu, on stream s.
jfdk_status reconstruct_bp(jfdk_ctx* c, float* d_hu, cudaStream_t s);
int bp_slices_per_thread(const jfdk_ctx* c);
bool mixed_form(const jfdk_ctx* c);
// The context's normalisation-weight volume for a backprojection over every
// view with its current options (computed now if needed, the context's
// stream synchronised), or null when it has none (JFDK_OPT_BP_WEIGHTS off,
// no room, or a capture under way).
const float* bp_weight_volume(jfdk_ctx* c);
}  // namespace jfdk
