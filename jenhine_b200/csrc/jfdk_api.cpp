// jfdk_api.cpp -- the C ABI (include/jfdk.h): context setup, device memory,
// and the stage / whole-volume entry points.  No exception leaves this file.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <map>
#include <mutex>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>

#include <cuda_bf16.h>

#include "jfdk_internal.h"

using namespace jfdk;

namespace {

inline size_t round_up(size_t a, size_t b) { return (a + b - 1) / b * b; }

// A failed CUDA call sets the context's message and returns a status.
jfdk_status fail(jfdk_ctx* c, jfdk_status st, const std::string& msg) {
    if (c) c->err = msg;
    return st;
}

jfdk_status cuda_fail(jfdk_ctx* c, cudaError_t e, const char* what) {
    if (e == cudaErrorMemoryAllocation)
        return fail(c, JFDK_ERR_OOM, std::string("CUDA failed to malloc ") + what);
    return fail(c, JFDK_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define JFDK_CUDA(ctx, call, what)                          \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, what); \
    } while (0)

#define JFDK_LAUNCH(ctx, call, what)                        \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, what); \
        ++(ctx)->launches;                                  \
    } while (0)

// Every device allocation of a context goes through dev_alloc / dev_free,
// which keep the context's total; a request that would take the total past
// JFDK_OPT_DEVICE_MEMORY_LIMIT fails exactly like a failed cudaMalloc.
template <class T>
jfdk_status dev_alloc(jfdk_ctx* c, T** p, size_t count, const char* what) {
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    void* q = nullptr;
    cudaError_t e = cudaErrorMemoryAllocation;
    if (c->mem_limit <= 0 || c->dev_bytes + (long long)bytes <= c->mem_limit) e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(c, e == cudaErrorMemoryAllocation ? JFDK_ERR_OOM : JFDK_ERR_CUDA,
                    std::string("CUDA failed to malloc ") + std::to_string(count * sizeof(T)) +
                        " bytes for " + what);
    }
    c->alloc_bytes[q] = bytes;
    c->dev_bytes += (long long)bytes;
    *p = static_cast<T*>(q);
    return JFDK_OK;
}

template <class T>
void dev_free(jfdk_ctx* c, T*& p) {
    if (p) {
        auto it = c->alloc_bytes.find(p);
        if (it != c->alloc_bytes.end()) {
            c->dev_bytes -= (long long)it->second;
            c->alloc_bytes.erase(it);
        }
        cudaFree(p);
    }
    p = nullptr;
}

// K padded to 64 elements: whole 128-byte rows for every operand kind.
int a_pitch(const jfdk_ctx* c) { return (int)round_up(c->in_w, 64); }
long long frame_px(const jfdk_ctx* c) { return (long long)c->rows * c->out_w; }

jfdk_status ensure_A(jfdk_ctx* c, size_t rows) {
    if (c->a_rows >= rows) return JFDK_OK;
    dev_free(c, c->d_A);
    dev_free(c, c->d_e);
    dev_free(c, c->d_arow);
    c->a_rows = 0;
    // room for a high and a low part of up to 4 bytes each
    jfdk_status st = dev_alloc(c, reinterpret_cast<float**>(&c->d_A), rows * a_pitch(c) * 2, "the weighted rows");
    if (st) return st;
    if ((st = dev_alloc(c, &c->d_e, rows, "the edge means"))) return st;
    if ((st = dev_alloc(c, &c->d_arow, rows, "the row scales"))) return st;
    c->a_rows = rows;
    return JFDK_OK;
}

bool mixed(const jfdk_ctx* c) { return c->precision == JFDK_PRECISION_MIXED; }

int ramp_kind(const jfdk_ctx* c) {
    if (c->opt_ramp != JFDK_RAMP_DEFAULT) return c->opt_ramp;
    return mixed(c) ? JFDK_RAMP_BF16X3 : JFDK_RAMP_I8X14;
}

// The A operand in the layout the chosen ramp product reads: the high part
// at d_A, the low part after a_rows rows of it.
AOperand a_operand(const jfdk_ctx* c) {
    AOperand a{};
    const int k = ramp_kind(c);
    a.kind = k == JFDK_RAMP_TF32X3 ? AOUT_TF32X2
             : k == JFDK_RAMP_BF16X3 ? AOUT_BF16X2
             : k == JFDK_RAMP_FP16X3 ? AOUT_FP16X2
             : k == JFDK_RAMP_I8X14 ? AOUT_I8X4 : AOUT_F32;
    const size_t elem = a.kind == AOUT_I8X4 ? 1 : (a.kind == AOUT_BF16X2 || a.kind == AOUT_FP16X2) ? 2 : 4;
    a.hi = c->d_A;
    a.lo = static_cast<char*>(c->d_A) + c->a_rows * a_pitch(c) * elem;
    a.row_scale = c->d_arow;
    a.pitch = a_pitch(c);
    return a;
}

jfdk_status ensure_plain(jfdk_ctx* c, int views) {
    if (c->plain_views >= views) return JFDK_OK;
    dev_free(c, c->d_plain);
    c->plain_views = 0;
    jfdk_status st = dev_alloc(c, &c->d_plain, (size_t)views * frame_px(c), "the filtered frames");
    if (st) return st;
    c->plain_views = views;
    return JFDK_OK;
}

// Bytes of one record of the backprojection store: a 16-byte quad (FP32
// form) or an 8-byte FP16 record (mixed form).
size_t record_size(const jfdk_ctx* c) { return mixed(c) ? 8 : 16; }

jfdk_status ensure_Q4(jfdk_ctx* c, int views) {
    if (c->q4_views >= views) return JFDK_OK;
    dev_free(c, c->d_q4);
    c->q4_views = 0;
    const size_t bytes = (size_t)views * frame_px(c) * record_size(c);
    jfdk_status st = dev_alloc(c, &c->d_q4, (bytes + 15) / 16, "the backprojection store");
    if (st) return st;
    c->q4_views = views;
    return JFDK_OK;
}

jfdk_status ensure_absmax(jfdk_ctx* c, int n) {
    if (c->absmax_n >= n) return JFDK_OK;
    dev_free(c, c->d_absmax);
    c->absmax_n = 0;
    jfdk_status st = dev_alloc(c, &c->d_absmax, (size_t)n, "the per-view maxima");
    if (st) return st;
    c->absmax_n = n;
    return JFDK_OK;
}

// The accumulating backprojection's slab: slices [slab_z0, slab_z0 + n).
int slab_slices(const jfdk_ctx* c) { return c->slab_nz > 0 ? c->slab_nz : c->Z; }
bool whole_volume(const jfdk_ctx* c) { return c->slab_z0 == 0 && slab_slices(c) == c->Z; }

// Accumulators for the slab's slices (BPCUDACore's accumulatedVol of
// numSlicesEachPart planes, BPCUDAAgent/BPCUDACore.cpp:38).
jfdk_status ensure_acc(jfdk_ctx* c) {
    const int need = slab_slices(c);
    if (c->d_sum && c->acc_slices >= need) return JFDK_OK;
    dev_free(c, c->d_sum);
    dev_free(c, c->d_cnt);
    c->acc_slices = 0;
    const size_t n = (size_t)c->X * c->Y * need;
    jfdk_status st = dev_alloc(c, &c->d_sum, n, "the backprojection sum volume");
    if (!st) st = dev_alloc(c, &c->d_cnt, n, "the backprojection weight volume");
    if (st) {
        dev_free(c, c->d_sum);
        return st;
    }
    c->acc_slices = need;
    return JFDK_OK;
}

// Conjugate-view compositing is on when the filter reads rows twice the
// frame width (the reference's CompositeAgent -> FilterAgent(2U) chain).
bool compositing(const jfdk_ctx* c) { return c->in_w == 2 * c->used_u; }

CompositeParams composite_params(const jfdk_ctx* c) {
    CompositeParams p{};
    if (!compositing(c)) return p;
    p.tinv = c->d_tinv_view;
    p.ptm = c->d_ptm;
    p.mask = c->d_cmask;
    p.num_views = c->nviews;
    p.W = c->used_u;
    p.H = c->used_v;
    p.det_right = c->mirror;
    return p;
}

WeightParams weight_params(const jfdk_ctx* c) {
    WeightParams w{};
    w.tinv = c->d_tinv;
    w.dmin = c->d_dmin;
    w.num_views = c->nviews;
    w.L = c->L;
    w.det_right = c->mirror;
    w.mirror = c->mirror;
    w.pw = c->d_pw;
    return w;
}

// Weight pass over raw frames: with compositing, rows are composited first
// (the conjugate frames come from the same rotation).
WeightParams weight_params_raw(const jfdk_ctx* c) {
    WeightParams w = weight_params(c);
    w.comp = composite_params(c);
    return w;
}

PrepParams prep_params(const jfdk_ctx* c, const uint16_t* raw) {
    PrepParams p{};
    p.raw = raw;
    p.in_w = c->scan.num_dets_u;
    p.in_h = c->scan.num_dets_v;
    p.crop_x = c->scan.border_left;
    p.crop_y = c->scan.border_up;
    p.width = c->used_u;
    p.rows = c->used_v;
    p.bright_field = c->scan.bright_field;
    p.bhc0 = c->scan.beam_hardening[0];
    p.bhc1 = c->scan.beam_hardening[1];
    p.bhc2 = c->scan.beam_hardening[2];
    // PreProcessingCore.cpp:56 -- skipped when the parameters are (1, 0, 0)
    p.do_bhc = !(p.bhc0 == 1.0f && p.bhc1 == 0.0f && p.bhc2 == 0.0f);
    return p;
}

BPParams bp_params(const jfdk_ctx* c) {
    BPParams b{};
    b.q4 = c->d_q4;
    b.tw = c->d_tw;
    b.ptm = c->d_ptm;
    b.q4_frame = frame_px(c);
    b.U = c->out_w;
    b.V = c->rows;
    b.X = c->X; b.Y = c->Y; b.Z = c->Z;
    b.pxy = c->pxy; b.pz = c->pz;
    b.z_begin = 0; b.z_end = c->Z;
    b.ct_scale = c->ct_scale;
    b.ct_norm1 = c->recon.ct_norm1;
    return b;
}

// Slices per thread: the option, else 16 in the mixed form when W does not
// depend on z and the volume holds at least 8 waves of 16-slice tiles (5
// CTAs per SM), 8 otherwise.  16 slices halve the mixed loop's per-view work
// (87.8 against 93.6 ms on c2, 130 waves), but a small volume then fills the
// GPU in few waves (c1, 128^3: 1.4 waves, 1.39 against 1.22 ms with 8); the
// FP32 form measured 139 ms with 16 against 128 with 8 (its per-slice
// coordinates leave no per-view work to amortise).
int bp_zpt(const jfdk_ctx* c) {
    if (c->opt_bp_zpt) return c->opt_bp_zpt;
    if (!mixed(c) || c->w_depends_on_z) return 8;
    const long long tiles = (long long)((c->X + kBPTileX - 1) / kBPTileX) * ((c->Y + kBPTileY - 1) / kBPTileY) *
                            ((c->Z + 15) / 16);
    return tiles >= 8LL * 5 * c->sms ? 16 : 8;
}

// CTA width in x: the option, else 4 (4 x 32 threads).
int bp_tile(const jfdk_ctx* c) { return c->opt_bp_tile ? c->opt_bp_tile : kBPTileX; }

// Filtered frames [nv][rows][out_w] of rotation views view0.. -> the BP store,
// slots slot0..: tapered FP32 quads, or in the mixed form FP16 records with
// the views' scales.
// have_absmax: the ramp product already left the frames' maxima in d_absmax.
jfdk_status pack_frames(jfdk_ctx* c, const float* plain, int nv, int view0, int slot0, bool have_absmax = false) {
    if (mixed(c)) {
        jfdk_status st = ensure_absmax(c, nv);
        if (st) return st;
        if (!have_absmax)
            JFDK_LAUNCH(c, launch_frame_absmax(plain, frame_px(c), nv, c->d_absmax, c->stream), "per-view maxima");
        JFDK_LAUNCH(c, launch_pack_mixed(plain, frame_px(c), nv, c->rows, c->out_w, c->d_tw, view0, c->nviews,
                                         c->d_absmax, c->d_qscale, reinterpret_cast<uint2*>(c->d_q4), frame_px(c),
                                         slot0, c->stream),
                    "packing projections");
        return JFDK_OK;
    }
    JFDK_LAUNCH(c, launch_pack_quads(plain, frame_px(c), nv, c->rows, c->out_w, c->d_tw, view0, c->nviews, 1, c->d_q4,
                                     frame_px(c), slot0, c->stream),
                "packing projections");
    return JFDK_OK;
}

bool capturing(cudaStream_t s) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &st) != cudaSuccess) {
        cudaGetLastError();
        return true;   // the legacy stream while another stream captures
    }
    return st != cudaStreamCaptureStatusNone;
}

// The FP32 form's normalisation weights over every view (JFDK_OPT_BP_WEIGHTS),
// computed once per geometry and rounding mode on the context's stream,
// which is then synchronised, so later launches on any stream (and graph
// captures) read finished weights with no event between them.  False
// (nothing set) when the option is off, when a capture is under way and the
// weights are not ready, or when the volume does not fit -- within
// JFDK_OPT_DEVICE_MEMORY_LIMIT and the device -- and the weights are then
// accumulated per sample.
bool ensure_weights(jfdk_ctx* c, cudaStream_t s) {
    if (!c->opt_bp_weights) return false;
    // the mixed form's coordinates step from each thread's first slice, so
    // its weights follow the tile depth too
    const int want = mixed(c) ? 100 + bp_zpt(c) : c->opt_bp_exact ? 2 : 1;
    if (c->d_wvol && c->wvol_state == want) return true;
    if (capturing(c->stream) || capturing(s)) return false;
    if (!c->d_wvol) {
        const size_t bytes = (size_t)c->X * c->Y * c->Z * sizeof(float);
        if (c->mem_limit > 0 && c->dev_bytes + (long long)bytes > c->mem_limit) return false;
        void* q = nullptr;
        if (cudaMalloc(&q, bytes) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        c->alloc_bytes[q] = bytes;
        c->dev_bytes += (long long)bytes;
        c->d_wvol = static_cast<float*>(q);
    }
    BPParams b = bp_params(c);
    b.view_base = 0; b.v0 = 0; b.nv = c->nviews;
    c->wvol_state = 0;
    const cudaError_t e =
        mixed(c) ? launch_bp_mixed_weights(b, c->w_depends_on_z, bp_zpt(c), bp_tile(c), c->d_wvol, c->stream)
                 : launch_bp_weights(b, c->opt_bp_exact != 0, c->w_depends_on_z, bp_zpt(c), bp_tile(c), c->d_wvol,
                                     c->stream);
    if (e != cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    c->wvol_state = want;
    return true;
}

jfdk_status run_bp_on(jfdk_ctx* c, BPParams b, bool finalize, cudaStream_t s) {
    if (finalize && b.v0 == 0 && b.nv == c->nviews && ensure_weights(c, s)) b.wvol = c->d_wvol;
    if (mixed(c)) {
        b.qh = reinterpret_cast<const uint2*>(c->d_q4);
        b.qscale = c->d_qscale;
        JFDK_LAUNCH(c, launch_bp_mixed(b, finalize, c->w_depends_on_z, bp_zpt(c), bp_tile(c), s), "backprojection");
        return JFDK_OK;
    }
    JFDK_LAUNCH(c, launch_bp(b, finalize, c->opt_bp_exact != 0, c->w_depends_on_z, bp_zpt(c), bp_tile(c), s),
                "backprojection");
    return JFDK_OK;
}

jfdk_status run_bp(jfdk_ctx* c, BPParams b, bool finalize) { return run_bp_on(c, b, finalize, c->stream); }

cudaError_t launch_ramp(jfdk_ctx* c, RampParams r) {
    const AOperand a = a_operand(c);
    switch (ramp_kind(c)) {
        case JFDK_RAMP_FP32_SIMT:
            r.A = static_cast<const float*>(a.hi);
            return launch_ramp_gemm(r, c->stream);
        case JFDK_RAMP_TF32X3:
            return launch_ramp_gemm_tc(r, RAMP_TF32X3, a.hi, a.lo, c->d_Th, c->d_Tl, c->d_status, c->stream);
        case JFDK_RAMP_BF16X3:
            return launch_ramp_gemm_tc(r, RAMP_BF16X3, a.hi, a.lo, c->d_Tb, c->d_Tb + (size_t)c->out_w * a_pitch(c),
                                       c->d_status, c->stream);
        case JFDK_RAMP_I8X14:
            r.row_scale = c->d_arow;
            r.b_scale = c->i8_scale;
            return launch_ramp_i8(r, static_cast<const int8_t*>(a.hi),
                                  (long long)(static_cast<const int8_t*>(a.lo) - static_cast<const int8_t*>(a.hi)),
                                  c->d_Ti8, (long long)c->out_w * a_pitch(c), c->d_i8mask, c->d_status, c->stream);
        default:
            r.row_scale = c->d_arow;
            r.b_scale = c->tf_inv_scale;
            return launch_ramp_gemm_tc(r, RAMP_FP16X3, a.hi, a.lo, c->d_Tf, c->d_Tf + (size_t)c->out_w * a_pitch(c),
                                       c->d_status, c->stream);
    }
}

RampParams ramp_params(const jfdk_ctx* c, int nv, float* out) {
    RampParams r{};
    r.A = nullptr; r.e = c->d_e; r.B = c->d_T; r.c = c->d_c;
    r.M = nv * c->rows; r.N = c->out_w; r.K = c->in_w; r.a_pitch = a_pitch(c);
    r.rows = c->rows;
    r.q = out; r.q_frame_stride = frame_px(c); r.q_pitch = c->out_w;
    r.row_scale = nullptr;
    r.b_scale = 1.0f;
    r.vec_store = (reinterpret_cast<uintptr_t>(out) % 16 == 0) && (c->out_w % 4 == 0);
    r.absmax = nullptr;
    return r;
}

}  // namespace

namespace jfdk {

// Everything jfdk_reconstruct does before the backprojection, for the first
// nviews views: per chunk of views raw -> weighted rows -> filtered frames
// (L2-sized buffers) -> [z-filter] -> the BP store of the rotation.
jfdk_status reconstruct_filter_stage(jfdk_ctx* c, const uint16_t* d_raw, int nviews, const cudaEvent_t* chunk_ready) {
    if (nviews < 0 || nviews > c->nviews) nviews = c->nviews;
    return filter_stage_range(c, d_raw, 0, nviews, chunk_ready);
}

jfdk_status filter_stage_range(jfdk_ctx* c, const uint16_t* d_raw, int vbeg, int vend, const cudaEvent_t* chunk_ready) {
    if (c->in_w != c->used_u && !compositing(c))
        return fail(c, JFDK_ERR_UNSUPPORTED,
                    "reconstruct: filter input width must be the frame width or twice it (compositing)");
    jfdk_status st = ensure_Q4(c, c->nviews);
    if (st) return st;
    const int chunk = std::min(c->opt_view_chunk, c->nviews);
    if ((st = ensure_A(c, (size_t)chunk * c->rows))) return st;
    if ((st = ensure_plain(c, chunk))) return st;
    const size_t frame = (size_t)c->scan.num_dets_u * c->scan.num_dets_v;
    for (int v0 = vbeg; v0 < vend; v0 += chunk) {
        const int nv = std::min(chunk, vend - v0);
        if (chunk_ready)
            JFDK_CUDA(c, cudaStreamWaitEvent(c->stream, chunk_ready[(v0 - vbeg) / chunk], 0), "frame transfer");
        PrepParams pp = prep_params(c, d_raw + (size_t)v0 * frame);
        if (compositing(c)) {
            pp.width = c->in_w;
            pp.raw_rotation = d_raw;
            pp.raw_frame = (long long)frame;
        }
        JFDK_LAUNCH(c, launch_prep_weight(pp, nv, v0, weight_params_raw(c), a_operand(c), c->d_e, c->stream),
                    compositing(c) ? "preprocess + compositing + pre-weight" : "preprocess + pre-weight");
        // mixed form with a tensor-core product: the product's epilogue
        // leaves each frame's max |q| for the packer (no z-filter between)
        RampParams rp = ramp_params(c, nv, c->d_plain);
        const bool fused_max = mixed(c) && ramp_kind(c) != JFDK_RAMP_FP32_SIMT && !c->recon.z_filter;
        if (fused_max) {
            if ((st = ensure_absmax(c, nv))) return st;
            JFDK_CUDA(c, cudaMemsetAsync(c->d_absmax, 0, sizeof(unsigned) * nv, c->stream), "clearing the maxima");
            rp.absmax = c->d_absmax;
        }
        JFDK_LAUNCH(c, launch_ramp(c, rp), "ramp filter");
        if (c->recon.z_filter)
            JFDK_LAUNCH(c, launch_zfilter(c->d_plain, nv, c->rows, c->out_w, frame_px(c), c->out_w, c->stream),
                        "z-filter");
        if ((st = pack_frames(c, c->d_plain, nv, v0, v0, fused_max))) return st;
    }
    return JFDK_OK;
}

// The finalizing backprojection of every view into d_hu / d_hu16 with CT
// numbers (the store filled by reconstruct_filter_stage).
// The backprojection store of every view, allocated now, so that parameters
// taken before a filter stage (the batch's persistent launches) name the
// buffer that filter stage fills.
jfdk_status ensure_store(jfdk_ctx* c) { return ensure_Q4(c, c->nviews); }

BPParams reconstruct_bp_params(const jfdk_ctx* c, float* d_hu, int16_t* d_hu16) {
    BPParams b = bp_params(c);
    b.view_base = 0; b.v0 = 0; b.nv = c->nviews;
    b.out = d_hu; b.out16 = d_hu16; b.apply_ct = 1;
    if (mixed(c)) {
        b.qh = reinterpret_cast<const uint2*>(c->d_q4);
        b.qscale = c->d_qscale;
    }
    return b;
}

jfdk_status reconstruct_bp(jfdk_ctx* c, float* d_hu, cudaStream_t s) {
    return run_bp_on(c, reconstruct_bp_params(c, d_hu, nullptr), true, s);
}

int bp_slices_per_thread(const jfdk_ctx* c) { return bp_zpt(c); }
bool mixed_form(const jfdk_ctx* c) { return mixed(c); }
const float* bp_weight_volume(jfdk_ctx* c) { return ensure_weights(c, c->stream) ? c->d_wvol : nullptr; }

}  // namespace jfdk

extern "C" {

jfdk_status jfdk_device_check(char* msg, int msg_len) {
    int dev = 0, n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    std::string m;
    jfdk_status st = JFDK_OK;
    if (e != cudaSuccess || n == 0) {
        m = std::string("no CUDA device: ") + cudaGetErrorString(e);
        st = JFDK_ERR_NO_DEVICE;
        cudaGetLastError();
    } else {
        cudaGetDevice(&dev);
        cudaDeviceProp prop{};
        cudaGetDeviceProperties(&prop, dev);
        m = std::string(prop.name) + " sm_" + std::to_string(prop.major) + std::to_string(prop.minor);
        if (prop.major != 10) st = JFDK_ERR_NO_DEVICE;
    }
    if (msg && msg_len > 0) {
        std::strncpy(msg, m.c_str(), msg_len - 1);
        msg[msg_len - 1] = 0;
    }
    return st;
}

const char* jfdk_last_error(const jfdk_ctx* c) { return c ? c->err.c_str() : "null context"; }

long long jfdk_kernel_launches(const jfdk_ctx* c) { return c ? c->launches : 0; }
long long jfdk_device_bytes(const jfdk_ctx* c) { return c ? c->dev_bytes : 0; }

void jfdk_destroy(jfdk_ctx* c) {
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    dev_free(c, c->d_ptm); dev_free(c, c->d_tw); dev_free(c, c->d_tinv); dev_free(c, c->d_dmin); dev_free(c, c->d_pw);
    dev_free(c, c->d_tinv_view); dev_free(c, c->d_cmask);
    dev_free(c, c->d_T); dev_free(c, c->d_Th); dev_free(c, c->d_Tl); dev_free(c, c->d_Tb); dev_free(c, c->d_Tf);
    dev_free(c, c->d_Ti8); dev_free(c, c->d_i8mask);
    dev_free(c, c->d_status); dev_free(c, c->d_c); dev_free(c, c->d_A); dev_free(c, c->d_e); dev_free(c, c->d_arow);
    dev_free(c, c->d_plain);
    dev_free(c, c->d_q4); dev_free(c, c->d_qscale); dev_free(c, c->d_absmax);
    dev_free(c, c->d_sum); dev_free(c, c->d_cnt); dev_free(c, c->d_raw_stage); dev_free(c, c->d_hu_stage);
    dev_free(c, c->d_Tt); dev_free(c, c->d_rt); dev_free(c, c->d_qadj); dev_free(c, c->d_partial);
    dev_free(c, c->d_dptm);
    dev_free(c, c->d_wvol);
    for (auto& e : c->ev)
        if (e) cudaEventDestroy(e);
    for (cudaStream_t s : {c->copy_stream, c->aux_stream}) {
        if (!s) continue;
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
    for (auto& e : c->xfer_ev) cudaEventDestroy(e);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

jfdk_status jfdk_create(jfdk_ctx** out, const jfdk_scan_params* scan, const jfdk_recon_params* recon,
                        const float* h_ptms, int precision, void* cuda_stream) {
    if (!out || !scan || !recon || !h_ptms) return JFDK_ERR_INVALID;
    *out = nullptr;
    jfdk_ctx* c = new (std::nothrow) jfdk_ctx();
    if (!c) return JFDK_ERR_OOM;
    auto bail = [&](jfdk_status st) { *out = c; return st; };  // caller reads the message, then destroys
    c->scan = *scan;
    c->recon = *recon;
    if (recon->num_adjust > 0) {
        if (!recon->adjust_points || !recon->adjust_level_db)
            return bail(fail(c, JFDK_ERR_INVALID, "adjust points without values"));
        c->adj_pts.assign(recon->adjust_points, recon->adjust_points + recon->num_adjust);
        c->adj_db.assign(recon->adjust_level_db, recon->adjust_level_db + recon->num_adjust);
    }
    c->recon.adjust_points = nullptr;
    c->recon.adjust_level_db = nullptr;
    c->precision = precision;
    if (precision != JFDK_PRECISION_FP32 && precision != JFDK_PRECISION_MIXED)
        return bail(fail(c, JFDK_ERR_INVALID, "unknown precision mode"));
    c->nviews = scan->num_views;
    c->used_u = scan->num_dets_u - scan->border_left - scan->border_right;
    c->used_v = scan->num_dets_v - scan->border_up - scan->border_down;
    c->in_w = scan->filter_input_width > 0 ? scan->filter_input_width : c->used_u;
    c->out_w = c->used_u;
    c->rows = c->used_v;
    c->mirror = scan->detector_on_right ? 1 : 0;
    c->X = recon->num_pixels_x; c->Y = recon->num_pixels_y; c->Z = recon->num_pixels_z;
    c->pxy = recon->pitch_xy; c->pz = recon->pitch_z;
    if (c->nviews < 1 || c->used_u < 3 || c->used_v < 1 || c->in_w < 3 || c->X < 1 || c->Y < 1 || c->Z < 1 ||
        scan->border_left < 0 || scan->border_right < 0 || scan->border_up < 0 || scan->border_down < 0 ||
        !(scan->dso > 1.0f) || !(scan->bright_field > 0.0f) || !(recon->mu_water != 0.0f) ||
        (long long)c->rows * c->in_w > (1LL << 31) || (long long)c->X * c->Y > (1LL << 31))
        return bail(fail(c, JFDK_ERR_INVALID, "invalid scan or reconstruction size"));
    if (c->mirror && c->in_w < c->out_w)
        return bail(fail(c, JFDK_ERR_INVALID, "mirrored filter needs input width >= output width"));
    c->L = fft_length(c->in_w);
    if (scan->half_sample_rate > 0.0f) {
        c->hsr = scan->half_sample_rate;
    } else {  // Config/ConfigHelper.cpp:52-53
        const float det_at_iso = scan->detector_pixel_size / scan->dsd * scan->dso;
        c->hsr = 0.5f * (1.0f / det_at_iso);
    }
    c->groups = (c->nviews + 8) / 9;
    c->ct_scale = recon->ct_norm0 * 1000.f / recon->mu_water;  // CTNumCore.cpp:24
    c->ptms.assign(h_ptms, h_ptms + (size_t)c->nviews * 12);
    for (int v = 0; v < c->nviews; ++v)
        if (c->ptms[(size_t)v * 12 + 10] != 0.0f) c->w_depends_on_z = true;

    int dev = 0;
    JFDK_CUDA(c, cudaGetDevice(&dev), "cudaGetDevice");
    cudaDeviceProp prop{};
    JFDK_CUDA(c, cudaGetDeviceProperties(&prop, dev), "cudaGetDeviceProperties");
    if (prop.major != 10) return bail(fail(c, JFDK_ERR_NO_DEVICE, "libjfdk needs an sm_100 (B200) device"));
    c->device = dev;
    c->sms = prop.multiProcessorCount;
    // NULL selects the legacy default stream, so the context's work is
    // ordered with every other default-stream operation of the process.
    c->stream = static_cast<cudaStream_t>(cuda_stream);
    c->own_stream = false;

    const std::string msg = build_host_operators(*scan, c->recon, c->adj_pts, c->adj_db, h_ptms, c->in_w,
                                                 c->out_w, c->rows, c->mirror, c->hsr, c->ops);
    if (!msg.empty()) return bail(fail(c, JFDK_ERR_INVALID, msg));

    // device constants
    jfdk_status st;
    if ((st = dev_alloc(c, &c->d_ptm, (size_t)c->nviews * 12, "the projection matrices"))) return bail(st);
    if ((st = dev_alloc(c, &c->d_tw, (size_t)c->nviews * c->out_w, "the u-taper pairs"))) return bail(st);
    if ((st = dev_alloc(c, &c->d_tinv, (size_t)c->groups * 16, "the inverse transforms"))) return bail(st);
    if ((st = dev_alloc(c, &c->d_dmin, (size_t)c->groups, "the pre-weight minima"))) return bail(st);
    if ((st = dev_alloc(c, &c->d_T, (size_t)c->out_w * a_pitch(c), "the ramp operator"))) return bail(st);
    if ((st = dev_alloc(c, &c->d_Th, (size_t)c->out_w * a_pitch(c), "the ramp operator"))) return bail(st);
    if ((st = dev_alloc(c, &c->d_Tl, (size_t)c->out_w * a_pitch(c), "the ramp operator"))) return bail(st);
    if ((st = dev_alloc(c, &c->d_Tb, (size_t)2 * c->out_w * a_pitch(c), "the ramp operator"))) return bail(st);
    if ((st = dev_alloc(c, &c->d_Tf, (size_t)2 * c->out_w * a_pitch(c), "the ramp operator"))) return bail(st);
    const int tt_pitch = (int)round_up(c->out_w, 64);
    if ((st = dev_alloc(c, &c->d_Tt, (size_t)c->in_w * tt_pitch, "the transposed ramp operator"))) return bail(st);
    if ((st = dev_alloc(c, &c->d_c, (size_t)c->out_w, "the edge response"))) return bail(st);
    if ((st = dev_alloc(c, &c->d_status, 1, "the status word"))) return bail(st);
    if ((st = dev_alloc(c, &c->d_qscale, (size_t)c->nviews, "the view scales"))) return bail(st);
    JFDK_CUDA(c, cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream), "clearing the status word");
    std::vector<float2> twp((size_t)c->nviews * c->out_w);
    for (int v = 0; v < c->nviews; ++v)
        for (int i = 0; i < c->out_w; ++i) {
            const float* w = &c->ops.uw[(size_t)v * c->out_w];
            twp[(size_t)v * c->out_w + i] = make_float2(w[i], (i + 1 < c->out_w ? w[i + 1] : 0.0f) - w[i]);
        }
    std::vector<float> Tp((size_t)c->out_w * a_pitch(c), 0.0f);
    for (int j = 0; j < c->out_w; ++j)
        std::memcpy(&Tp[(size_t)j * a_pitch(c)], &c->ops.T[(size_t)j * c->in_w], sizeof(float) * c->in_w);
    JFDK_CUDA(c, cudaMemcpyAsync(c->d_ptm, h_ptms, sizeof(float) * c->nviews * 12, cudaMemcpyHostToDevice, c->stream), "upload");
    JFDK_CUDA(c, cudaMemcpyAsync(c->d_tw, twp.data(), sizeof(float2) * twp.size(), cudaMemcpyHostToDevice, c->stream), "upload");
    JFDK_CUDA(c, cudaMemcpyAsync(c->d_tinv, c->ops.tinv.data(), sizeof(float) * c->ops.tinv.size(), cudaMemcpyHostToDevice, c->stream), "upload");
    JFDK_CUDA(c, cudaMemcpyAsync(c->d_T, Tp.data(), sizeof(float) * Tp.size(), cudaMemcpyHostToDevice, c->stream), "upload");
    {   // TF32-exact split for the tensor-core product: T = Th + Tl + O(2^-22 T)
        std::vector<float> th(Tp.size()), tl(Tp.size());
        for (size_t i = 0; i < Tp.size(); ++i) {
            th[i] = tf32_round_host(Tp[i]);
            tl[i] = tf32_round_host(Tp[i] - th[i]);
        }
        JFDK_CUDA(c, cudaMemcpyAsync(c->d_Th, th.data(), sizeof(float) * th.size(), cudaMemcpyHostToDevice, c->stream), "upload");
        JFDK_CUDA(c, cudaMemcpyAsync(c->d_Tl, tl.data(), sizeof(float) * tl.size(), cudaMemcpyHostToDevice, c->stream), "upload");
        // BF16 split, and FP16 split of the operator scaled by a power of
        // two that puts its largest entry in [2^14, 2^15)
        const size_t n = Tp.size();
        std::vector<uint16_t> tb(2 * n), tf(2 * n);
        float tmax = 0.0f;
        for (float v : Tp) tmax = std::max(tmax, std::fabs(v));
        const float fs = tmax > 0.0f ? std::ldexp(1.0f, 14 - std::ilogb(tmax)) : 1.0f;
        c->tf_inv_scale = 1.0f / fs;
        for (size_t i = 0; i < n; ++i) {
            const __nv_bfloat16 bh = __float2bfloat16_rn(Tp[i]);
            const __nv_bfloat16 bl = __float2bfloat16_rn(Tp[i] - __bfloat162float(bh));
            std::memcpy(&tb[i], &bh, 2);
            std::memcpy(&tb[n + i], &bl, 2);
            const float v = Tp[i] * fs;
            const __half fh = __float2half_rn(v);
            const __half fl = __float2half_rn(v - __half2float(fh));
            std::memcpy(&tf[i], &fh, 2);
            std::memcpy(&tf[n + i], &fl, 2);
        }
        JFDK_CUDA(c, cudaMemcpyAsync(c->d_Tb, tb.data(), 2 * tb.size(), cudaMemcpyHostToDevice, c->stream), "upload");
        JFDK_CUDA(c, cudaMemcpyAsync(c->d_Tf, tf.data(), 2 * tf.size(), cudaMemcpyHostToDevice, c->stream), "upload");
        JFDK_CUDA(c, cudaStreamSynchronize(c->stream), "upload");
    }
    JFDK_CUDA(c, cudaMemcpyAsync(c->d_c, c->ops.c.data(), sizeof(float) * c->out_w, cudaMemcpyHostToDevice, c->stream), "upload");
    {   // int8 digits of the operator from its FP64 kernel (32-bit fixed
        // point below 2^F in four balanced bytes, as the weight kernel cuts
        // the rows), and which digit planes each (output tile, K block) of
        // the int8 product needs
        const int P = a_pitch(c), N = c->out_w, K = c->in_w, L = (int)c->ops.h.size();
        double tmax = 0.0;
        for (double v : c->ops.h) tmax = std::max(tmax, std::fabs(v));
        int F = 0;
        if (tmax > 0.0) {
            F = std::ilogb(tmax) - 6;
            if (tmax > std::ldexp(127.0, F)) ++F;
        }
        c->i8_scale = (float)std::ldexp(1.0, F);
        const size_t plane = (size_t)N * P;
        std::vector<int8_t> td((size_t)kI8OpDigits * plane, 0);
        for (int j = 0; j < N; ++j)
            for (int i = 0; i < K; ++i) {
                int d = (c->ops.off + j - i) % L;
                if (d < 0) d += L;
                long long q = std::llrint(std::ldexp(c->ops.h[d], 24 - F));   // |q| <= 127 * 2^24
                for (int t = kI8OpDigits - 1; t > 0; --t) {
                    const long long lo = ((q + 128) & 255) - 128;
                    td[t * plane + (size_t)j * P + i] = (int8_t)lo;
                    q = (q - lo) / 256;
                }
                td[(size_t)j * P + i] = (int8_t)q;
            }
        const int tn = (N + kI8TileN - 1) / kI8TileN, nk = (P + kI8BlockK - 1) / kI8BlockK;
        std::vector<uint8_t> mask((size_t)tn * nk, 0);
        for (int t = 0; t < kI8OpDigits; ++t)
            for (int j = 0; j < N; ++j)
                for (int i = 0; i < P; ++i)
                    if (td[t * plane + (size_t)j * P + i]) mask[(size_t)(j / kI8TileN) * nk + i / kI8BlockK] |= (uint8_t)(1u << t);
        if ((st = dev_alloc(c, &c->d_Ti8, td.size(), "the operator's digits"))) return bail(st);
        if ((st = dev_alloc(c, &c->d_i8mask, mask.size(), "the digit masks"))) return bail(st);
        JFDK_CUDA(c, cudaMemcpyAsync(c->d_Ti8, td.data(), td.size(), cudaMemcpyHostToDevice, c->stream), "upload");
        JFDK_CUDA(c, cudaMemcpyAsync(c->d_i8mask, mask.data(), mask.size(), cudaMemcpyHostToDevice, c->stream), "upload");
        JFDK_CUDA(c, cudaStreamSynchronize(c->stream), "upload");
    }
    {   // T^T [in_w][round64(out_w)] for the filter adjoint
        std::vector<float> tt((size_t)c->in_w * tt_pitch, 0.0f);
        for (int j = 0; j < c->out_w; ++j)
            for (int i = 0; i < c->in_w; ++i) tt[(size_t)i * tt_pitch + j] = c->ops.T[(size_t)j * c->in_w + i];
        JFDK_CUDA(c, cudaMemcpyAsync(c->d_Tt, tt.data(), sizeof(float) * tt.size(), cudaMemcpyHostToDevice, c->stream),
                  "upload");
        JFDK_CUDA(c, cudaStreamSynchronize(c->stream), "upload");
    }
    JFDK_LAUNCH(c, launch_preweight_dmin(c->d_tinv, c->groups, c->rows, c->L, c->in_w, c->mirror, c->d_dmin, c->stream),
                "pre-weight minimum");
    if ((st = dev_alloc(c, &c->d_pw, (size_t)c->groups * c->rows * c->in_w, "the pre-weight table"))) return bail(st);
    JFDK_LAUNCH(c, launch_preweight_table(c->d_tinv, c->d_dmin, c->groups, c->rows, c->in_w, c->mirror, c->d_pw,
                                          c->stream),
                "pre-weight table");
    if (compositing(c)) {   // per-view inverse TMs and CompositeCore's 40-column masks
        if ((st = dev_alloc(c, &c->d_tinv_view, (size_t)c->nviews * 16, "the inverse transforms"))) return bail(st);
        if ((st = dev_alloc(c, &c->d_cmask, 80, "the compositing masks"))) return bail(st);
        float mask[80];
        const float pi = 3.14159265358979323846f;
        for (int i = 0; i < 40; ++i) {   // CompositeCore.cpp:195-223
            mask[i] = c->mirror ? std::cos((float)i / 40.0f * pi) * -0.5f + 0.5f
                                : std::cos((float)i / 40.0f * pi) * 0.5f + 0.5f;
            mask[40 + i] = 1.0f - mask[i];
        }
        JFDK_CUDA(c, cudaMemcpyAsync(c->d_tinv_view, c->ops.tinv_view.data(), sizeof(float) * c->nviews * 16,
                                     cudaMemcpyHostToDevice, c->stream),
                  "upload");
        JFDK_CUDA(c, cudaMemcpyAsync(c->d_cmask, mask, sizeof mask, cudaMemcpyHostToDevice, c->stream), "upload");
    }
    JFDK_CUDA(c, cudaStreamSynchronize(c->stream), "context setup");
    *out = c;
    return JFDK_OK;
}

jfdk_status jfdk_set_option(jfdk_ctx* c, int key, long long value) {
    if (!c) return JFDK_ERR_INVALID;
    switch (key) {
        case JFDK_OPT_BP_EXACT: c->opt_bp_exact = value ? 1 : 0; return JFDK_OK;
        case JFDK_OPT_VIEW_CHUNK:
            if (value < 1 || value > 4096) return fail(c, JFDK_ERR_INVALID, "view chunk out of range");
            c->opt_view_chunk = (int)value;
            return JFDK_OK;
        case JFDK_OPT_BP_ZPT:
            if (value != 0 && value != 4 && value != 8 && value != 16)
                return fail(c, JFDK_ERR_INVALID, "slices per thread must be 0 (default), 4, 8 or 16");
            c->opt_bp_zpt = (int)value;
            return JFDK_OK;
        case JFDK_OPT_BP_TILE:
            if (value != 0 && value != 4 && value != 8 && value != 32)
                return fail(c, JFDK_ERR_INVALID, "backprojection tile width must be 0 (default), 4, 8 or 32");
            c->opt_bp_tile = (int)value;
            return JFDK_OK;
        case JFDK_OPT_FILTER_SIMT: c->opt_ramp = value ? JFDK_RAMP_FP32_SIMT : JFDK_RAMP_DEFAULT; return JFDK_OK;
        case JFDK_OPT_BP_WEIGHTS: c->opt_bp_weights = value ? 1 : 0; return JFDK_OK;
        case JFDK_OPT_RAMP_PRODUCT:
            if (value < JFDK_RAMP_DEFAULT || value > JFDK_RAMP_I8X14)
                return fail(c, JFDK_ERR_INVALID, "unknown ramp product");
            c->opt_ramp = (int)value;
            return JFDK_OK;
        case JFDK_OPT_STAGE_TIMING:
            if (value && !c->ev[0])
                for (auto& e : c->ev) JFDK_CUDA(c, cudaEventCreate(&e), "cudaEventCreate");
            c->opt_stage_timing = value ? 1 : 0;
            return JFDK_OK;
        case JFDK_OPT_DEVICE_MEMORY_LIMIT:
            if (value < 0) return fail(c, JFDK_ERR_INVALID, "negative memory limit");
            c->mem_limit = value;
            return JFDK_OK;
        default: return fail(c, JFDK_ERR_INVALID, "unknown option");
    }
}

jfdk_status jfdk_get_option(jfdk_ctx* c, int key, long long* value) {
    if (!c || !value) return JFDK_ERR_INVALID;
    switch (key) {
        case JFDK_OPT_BP_EXACT: *value = c->opt_bp_exact; return JFDK_OK;
        case JFDK_OPT_VIEW_CHUNK: *value = c->opt_view_chunk; return JFDK_OK;
        case JFDK_OPT_STAGE_TIMING: *value = c->opt_stage_timing; return JFDK_OK;
        case JFDK_OPT_BP_ZPT: *value = bp_zpt(c); return JFDK_OK;
        case JFDK_OPT_BP_TILE: *value = bp_zpt(c) == 16 ? kBPTileX : bp_tile(c); return JFDK_OK;
        case JFDK_OPT_FILTER_SIMT: *value = ramp_kind(c) == JFDK_RAMP_FP32_SIMT ? 1 : 0; return JFDK_OK;
        case JFDK_OPT_RAMP_PRODUCT: *value = ramp_kind(c); return JFDK_OK;
        case JFDK_OPT_DEVICE_MEMORY_LIMIT: *value = c->mem_limit; return JFDK_OK;
        case JFDK_OPT_BP_WEIGHTS: *value = c->opt_bp_weights; return JFDK_OK;
        default: return fail(c, JFDK_ERR_INVALID, "unknown option");
    }
}

jfdk_status jfdk_stage_times(jfdk_ctx* c, float* ms) {
    if (!c || !ms) return JFDK_ERR_INVALID;
    if (!c->opt_stage_timing || !c->ev[0]) return fail(c, JFDK_ERR_STATE, "stage timing is off");
    JFDK_CUDA(c, cudaEventSynchronize(c->ev[3]), "stage timing");
    for (int i = 0; i < 3; ++i) JFDK_CUDA(c, cudaEventElapsedTime(&ms[i], c->ev[i], c->ev[i + 1]), "stage timing");
    return JFDK_OK;
}

jfdk_status jfdk_sync(jfdk_ctx* c) {
    if (!c) return JFDK_ERR_INVALID;
    JFDK_CUDA(c, cudaStreamSynchronize(c->stream), "stream synchronize");
    int status = 0;
    JFDK_CUDA(c, cudaMemcpy(&status, c->d_status, sizeof(int), cudaMemcpyDeviceToHost), "reading the status word");
    if (status) {
        cudaMemset(c->d_status, 0, sizeof(int));
        return fail(c, JFDK_ERR_CUDA, "a tensor-core pipeline wait timed out; results of the last calls are invalid");
    }
    return JFDK_OK;
}

jfdk_status jfdk_get_dims(const jfdk_ctx* c, int* in_w, int* out_w, int* L, int* rows) {
    if (!c) return JFDK_ERR_INVALID;
    if (in_w) *in_w = c->in_w;
    if (out_w) *out_w = c->out_w;
    if (L) *L = c->L;
    if (rows) *rows = c->rows;
    return JFDK_OK;
}

jfdk_status jfdk_get_uweights(const jfdk_ctx* c, float* h) {
    if (!c || !h) return JFDK_ERR_INVALID;
    std::memcpy(h, c->ops.uw.data(), sizeof(float) * c->ops.uw.size());
    return JFDK_OK;
}

jfdk_status jfdk_get_ramp_operator(const jfdk_ctx* c, float* T, float* cc) {
    if (!c) return JFDK_ERR_INVALID;
    if (T) std::memcpy(T, c->ops.T.data(), sizeof(float) * c->ops.T.size());
    if (cc) std::memcpy(cc, c->ops.c.data(), sizeof(float) * c->ops.c.size());
    return JFDK_OK;
}

jfdk_status jfdk_preprocess_frames(jfdk_ctx* c, const uint16_t* d_raw, int nv, float* d_out) {
    if (!c || !d_raw || !d_out || nv < 0) return fail(c, JFDK_ERR_INVALID, "preprocess: bad argument");
    if (nv == 0) return JFDK_OK;
    JFDK_LAUNCH(c, launch_preprocess(prep_params(c, d_raw), nv, d_out, c->stream), "preprocess");
    return JFDK_OK;
}

jfdk_status jfdk_filter_frames(jfdk_ctx* c, const float* d_in, int v0, int nv, float* d_out) {
    if (!c || !d_in || !d_out || nv < 0 || v0 < 0) return fail(c, JFDK_ERR_INVALID, "filter: bad argument");
    if (nv == 0) return JFDK_OK;
    jfdk_status st = ensure_A(c, (size_t)nv * c->rows);
    if (st) return st;
    JFDK_LAUNCH(c, launch_weight(d_in, nv, v0, c->in_w, c->rows, weight_params(c), a_operand(c), c->d_e, c->stream),
                "pre-weight");
    JFDK_LAUNCH(c, launch_ramp(c, ramp_params(c, nv, d_out)), "ramp filter");
    return JFDK_OK;
}

jfdk_status jfdk_composite_frames(jfdk_ctx* c, const float* d_dirc, const float* d_conj, int v0, int nv,
                                  float* d_out) {
    if (!c || !d_dirc || !d_conj || !d_out || nv < 0 || v0 < 0)
        return fail(c, JFDK_ERR_INVALID, "composite: bad argument");
    if (!compositing(c))
        return fail(c, JFDK_ERR_STATE, "composite: the context's filter input width is not twice the frame width");
    if (nv == 0) return JFDK_OK;
    JFDK_LAUNCH(c, launch_composite_frames(d_dirc, d_conj, v0, nv, composite_params(c), d_out, c->stream),
                "compositing");
    return JFDK_OK;
}

jfdk_status jfdk_zfilter_frames(jfdk_ctx* c, float* d, int nv) {
    if (!c || !d || nv < 0) return fail(c, JFDK_ERR_INVALID, "zfilter: bad argument");
    if (nv == 0) return JFDK_OK;
    JFDK_LAUNCH(c, launch_zfilter(d, nv, c->rows, c->out_w, (long long)c->rows * c->out_w, c->out_w, c->stream),
                "z-filter");
    return JFDK_OK;
}

jfdk_status jfdk_bp_set_slab(jfdk_ctx* c, int z_begin, int z_count) {
    if (!c || z_begin < 0 || z_count < 1 || z_begin > c->Z - z_count)
        return fail(c, JFDK_ERR_INVALID, "bp_set_slab: slices outside the volume");
    c->slab_z0 = z_begin;
    c->slab_nz = z_count;
    c->bp_has_views = false;
    return ensure_acc(c);
}

jfdk_status jfdk_bp_reserve(jfdk_ctx* c, int views) {
    if (!c || views < 1 || views > c->nviews) return fail(c, JFDK_ERR_INVALID, "bp_reserve: bad view count");
    jfdk_status st = ensure_Q4(c, views);
    if (!st && mixed(c)) st = ensure_absmax(c, views);
    return st;
}

jfdk_status jfdk_bp_reset(jfdk_ctx* c) {
    if (!c) return JFDK_ERR_INVALID;
    jfdk_status st = ensure_acc(c);
    if (st) return st;
    const size_t n = (size_t)c->X * c->Y * slab_slices(c) * sizeof(float);
    JFDK_CUDA(c, cudaMemsetAsync(c->d_sum, 0, n, c->stream), "clearing the sum volume");
    JFDK_CUDA(c, cudaMemsetAsync(c->d_cnt, 0, n, c->stream), "clearing the weight volume");
    c->bp_has_views = true;
    return JFDK_OK;
}

jfdk_status jfdk_bp_accumulate(jfdk_ctx* c, const float* d_proj, int v0, int nv) {
    if (!c || !d_proj || nv < 0 || v0 < 0 || v0 + nv > c->nviews)
        return fail(c, JFDK_ERR_INVALID, "bp_accumulate: bad argument");
    if (!c->d_sum) return fail(c, JFDK_ERR_STATE, "bp_accumulate before bp_reset");
    if (nv == 0) return JFDK_OK;
    jfdk_status st = ensure_Q4(c, nv);
    if (st) return st;
    // InitView: taper the caller's frames while packing them
    if ((st = pack_frames(c, d_proj, nv, v0, 0))) return st;
    BPParams b = bp_params(c);
    b.view_base = v0; b.v0 = v0; b.nv = nv;
    b.z_begin = c->slab_z0; b.z_end = c->slab_z0 + slab_slices(c);
    b.sum = c->d_sum; b.cnt = c->d_cnt; b.acc_z0 = c->slab_z0; b.load_acc = 1;
    return run_bp(c, b, false);
}

jfdk_status jfdk_finalize(jfdk_ctx* c, int z0, int nz, int apply_ct, float* d_out, int16_t* d_out16) {
    if (!c || z0 < 0 || nz < 0 || z0 + nz > c->Z || (!d_out && !d_out16))
        return fail(c, JFDK_ERR_INVALID, "finalize: bad argument");
    if (!c->d_sum) return fail(c, JFDK_ERR_STATE, "finalize before any backprojection");
    if (z0 < c->slab_z0 || z0 + nz > c->slab_z0 + slab_slices(c))
        return fail(c, JFDK_ERR_INVALID, "finalize: slices outside the slab set by bp_set_slab");
    const size_t plane = (size_t)c->X * c->Y;
    const size_t off = (size_t)(z0 - c->slab_z0) * plane;
    JFDK_LAUNCH(c, launch_finalize(c->d_sum + off, c->d_cnt + off, nz * plane, apply_ct, c->ct_scale,
                                   c->recon.ct_norm1, d_out, d_out16, c->stream),
                "finalize");
    return JFDK_OK;
}

jfdk_status jfdk_ctnum(jfdk_ctx* c, float* d, size_t n) {
    if (!c || !d) return fail(c, JFDK_ERR_INVALID, "ctnum: bad argument");
    if (n == 0) return JFDK_OK;
    JFDK_LAUNCH(c, launch_ctnum(d, n, c->ct_scale, c->recon.ct_norm1, c->stream), "ct numbers");
    return JFDK_OK;
}

jfdk_status jfdk_reconstruct(jfdk_ctx* c, const uint16_t* d_raw, float* d_hu, int16_t* d_hu16) {
    if (!c || !d_raw || (!d_hu && !d_hu16)) return fail(c, JFDK_ERR_INVALID, "reconstruct: bad argument");
    const bool timing = c->opt_stage_timing != 0;
    if (timing) JFDK_CUDA(c, cudaEventRecord(c->ev[0], c->stream), "event");
    jfdk_status st = jfdk::reconstruct_filter_stage(c, d_raw, c->nviews);
    if (st) return st;
    if (timing) JFDK_CUDA(c, cudaEventRecord(c->ev[1], c->stream), "event");
    ensure_weights(c, c->stream);   // once per geometry, outside the timed stages
    if (timing) JFDK_CUDA(c, cudaEventRecord(c->ev[2], c->stream), "event");
    if ((st = run_bp(c, jfdk::reconstruct_bp_params(c, d_hu, d_hu16), true))) return st;
    if (timing) JFDK_CUDA(c, cudaEventRecord(c->ev[3], c->stream), "event");
    return JFDK_OK;
}

jfdk_status jfdk_filter_raw(jfdk_ctx* c, const uint16_t* d_raw, int v0, int nv, float* d_frames) {
    if (!c || !d_raw || !d_frames || v0 < 0 || nv < 0 || v0 > c->nviews - nv)
        return fail(c, JFDK_ERR_INVALID, "filter_raw: bad argument");
    if (nv == 0) return JFDK_OK;
    if (c->in_w != c->used_u && !compositing(c))
        return fail(c, JFDK_ERR_UNSUPPORTED,
                    "filter_raw: filter input width must be the frame width or twice it (compositing)");
    const int chunk = std::min(c->opt_view_chunk, c->nviews);
    jfdk_status st = ensure_A(c, (size_t)chunk * c->rows);
    if (st) return st;
    const size_t frame = (size_t)c->scan.num_dets_u * c->scan.num_dets_v;
    for (int a = v0; a < v0 + nv; a += chunk) {
        const int n = std::min(chunk, v0 + nv - a);
        PrepParams pp = prep_params(c, d_raw + (size_t)a * frame);
        if (compositing(c)) {
            pp.width = c->in_w;
            pp.raw_rotation = d_raw;
            pp.raw_frame = (long long)frame;
        }
        JFDK_LAUNCH(c, launch_prep_weight(pp, n, a, weight_params_raw(c), a_operand(c), c->d_e, c->stream),
                    compositing(c) ? "preprocess + compositing + pre-weight" : "preprocess + pre-weight");
        float* out = d_frames + (size_t)(a - v0) * frame_px(c);
        JFDK_LAUNCH(c, launch_ramp(c, ramp_params(c, n, out)), "ramp filter");
        if (c->recon.z_filter)
            JFDK_LAUNCH(c, launch_zfilter(out, n, c->rows, c->out_w, frame_px(c), c->out_w, c->stream), "z-filter");
    }
    return JFDK_OK;
}

jfdk_status jfdk_filter_to_store(jfdk_ctx* c, const uint16_t* d_raw, int v0, int nv) {
    if (!c || !d_raw || v0 < 0 || nv < 0 || v0 > c->nviews - nv)
        return fail(c, JFDK_ERR_INVALID, "filter_to_store: bad argument");
    if (nv == 0) return JFDK_OK;
    return jfdk::filter_stage_range(c, d_raw, v0, v0 + nv);
}

jfdk_status jfdk_store_range(jfdk_ctx* c, int v0, int nv, void** d_records, size_t* record_bytes, float** d_scales) {
    if (!c || !d_records || !record_bytes || !d_scales || v0 < 0 || nv < 0 || v0 > c->nviews - nv)
        return fail(c, JFDK_ERR_INVALID, "store_range: bad argument");
    jfdk_status st = ensure_Q4(c, c->nviews);
    if (st) return st;
    *d_records = reinterpret_cast<char*>(c->d_q4) + (size_t)v0 * frame_px(c) * record_size(c);
    *record_bytes = (size_t)nv * frame_px(c) * record_size(c);
    *d_scales = mixed(c) ? c->d_qscale + v0 : nullptr;
    return JFDK_OK;
}

jfdk_status jfdk_backproject_store(jfdk_ctx* c, int z0, int nz, float* d_hu, int16_t* d_hu16) {
    if (!c || z0 < 0 || nz < 1 || z0 > c->Z - nz || (!d_hu && !d_hu16))
        return fail(c, JFDK_ERR_INVALID, "backproject_store: bad argument");
    if (!c->d_q4 || c->q4_views < c->nviews) return fail(c, JFDK_ERR_STATE, "backproject_store: the store is empty");
    BPParams b = jfdk::reconstruct_bp_params(c, d_hu, d_hu16);
    b.z_begin = z0;
    b.z_end = z0 + nz;
    b.out_z0 = z0;
    return run_bp(c, b, true);
}

}  // extern "C"

namespace {

// Slabs the host path backprojects and downloads one after another.
constexpr int kHostSlabs = 8;

jfdk_status ensure_overlap(jfdk_ctx* c, size_t events) {
    if (!c->copy_stream)
        JFDK_CUDA(c, cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking), "creating the copy stream");
    if (!c->aux_stream)
        JFDK_CUDA(c, cudaStreamCreateWithFlags(&c->aux_stream, cudaStreamNonBlocking), "creating a compute stream");
    while (c->xfer_ev.size() < events) {
        cudaEvent_t e = nullptr;
        JFDK_CUDA(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "creating an event");
        c->xfer_ev.push_back(e);
    }
    return JFDK_OK;
}

// Uploads the frames chunk k of the filter stage reads that are not on the
// device yet (its views and, when compositing, their conjugates), as
// contiguous runs, on the copy stream.
jfdk_status upload_chunk(jfdk_ctx* c, const uint16_t* h_raw, int v0, int nv, std::vector<char>& up) {
    const int N = c->nviews;
    const size_t frame = (size_t)c->scan.num_dets_u * c->scan.num_dets_v;
    std::vector<int> need;
    for (int v = v0; v < v0 + nv; ++v) {
        need.push_back(v);
        if (compositing(c)) need.push_back((v + N / 2) % N);
    }
    std::sort(need.begin(), need.end());
    for (size_t i = 0; i < need.size();) {
        if (up[need[i]]) { ++i; continue; }
        size_t j = i;
        while (j + 1 < need.size() && need[j + 1] == need[j] + 1 && !up[need[j + 1]]) ++j;
        const int a = need[i], n = need[j] - need[i] + 1;
        JFDK_CUDA(c, cudaMemcpyAsync(c->d_raw_stage + (size_t)a * frame, h_raw + (size_t)a * frame,
                                     (size_t)n * frame * sizeof(uint16_t), cudaMemcpyHostToDevice, c->copy_stream),
                  "raw upload");
        for (int v = a; v < a + n; ++v) up[v] = 1;
        i = j + 1;
    }
    return JFDK_OK;
}

}  // namespace

extern "C" {

// Host buffers in and out, with the transfers overlapped: the frames go up
// chunk by chunk on a copy stream, each chunk of the filter stage waiting
// only for its own frames; the backprojection runs as slabs of slices on
// two compute streams (no launch tail between slabs), and each slab goes
// down as soon as it is done.  The results equal jfdk_reconstruct's bit for
// bit: the slabs start at multiples of the tile depth, so every thread
// covers the slices it covers in one launch.
jfdk_status jfdk_reconstruct_host(jfdk_ctx* c, const uint16_t* h_raw, float* h_hu) {
    if (!c || !h_raw || !h_hu) return fail(c, JFDK_ERR_INVALID, "reconstruct_host: bad argument");
    const size_t raw_bytes = (size_t)c->nviews * c->scan.num_dets_u * c->scan.num_dets_v * sizeof(uint16_t);
    const size_t hu_bytes = (size_t)c->X * c->Y * c->Z * sizeof(float);
    jfdk_status st;
    if (c->raw_stage_bytes < raw_bytes) {
        dev_free(c, c->d_raw_stage);
        c->raw_stage_bytes = 0;
        if ((st = dev_alloc(c, &c->d_raw_stage, raw_bytes / sizeof(uint16_t), "the raw frames"))) return st;
        c->raw_stage_bytes = raw_bytes;
    }
    if (c->hu_stage_bytes < hu_bytes) {
        dev_free(c, c->d_hu_stage);
        c->hu_stage_bytes = 0;
        if ((st = dev_alloc(c, &c->d_hu_stage, hu_bytes / sizeof(float), "the output volume"))) return st;
        c->hu_stage_bytes = hu_bytes;
    }
    const int chunk = std::min(c->opt_view_chunk, c->nviews);
    const int nchunks = (c->nviews + chunk - 1) / chunk;
    const int zpt = bp_zpt(c);
    const int slab = (int)round_up((c->Z + kHostSlabs - 1) / kHostSlabs, zpt);
    const int nslabs = (c->Z + slab - 1) / slab;
    if ((st = ensure_overlap(c, (size_t)nchunks + nslabs + 3))) return st;
    cudaEvent_t* ev = c->xfer_ev.data();   // [chunks][slabs] start, filtered, copies done
    cudaEvent_t ev_start = ev[nchunks + nslabs], ev_filtered = ev[nchunks + nslabs + 1],
                ev_done = ev[nchunks + nslabs + 2];
    // on any failure below, wait for what is queued before returning: the
    // copies still reference the caller's host buffers
    auto drain = [c](jfdk_status s) {
        cudaStreamSynchronize(c->copy_stream);
        cudaStreamSynchronize(c->aux_stream);
        cudaStreamSynchronize(c->stream);
        return s;
    };
    const bool timing = c->opt_stage_timing != 0;
    if (timing) JFDK_CUDA(c, cudaEventRecord(c->ev[0], c->stream), "event");
    // the transfers start after the work already queued on the context's stream
    JFDK_CUDA(c, cudaEventRecord(ev_start, c->stream), "event");
    JFDK_CUDA(c, cudaStreamWaitEvent(c->copy_stream, ev_start, 0), "event");
    std::vector<char> up((size_t)c->nviews, 0);
    for (int k = 0; k < nchunks; ++k) {
        const int v0 = k * chunk;
        if ((st = upload_chunk(c, h_raw, v0, std::min(chunk, c->nviews - v0), up))) return drain(st);
        JFDK_CUDA(c, cudaEventRecord(ev[k], c->copy_stream), "event");
    }
    if ((st = jfdk::reconstruct_filter_stage(c, c->d_raw_stage, c->nviews, ev))) return drain(st);
    if (timing) {
        JFDK_CUDA(c, cudaEventRecord(c->ev[1], c->stream), "event");
        JFDK_CUDA(c, cudaEventRecord(c->ev[2], c->stream), "event");
    }
    JFDK_CUDA(c, cudaEventRecord(ev_filtered, c->stream), "event");
    JFDK_CUDA(c, cudaStreamWaitEvent(c->aux_stream, ev_filtered, 0), "event");
    const size_t plane = (size_t)c->X * c->Y;
    for (int sl = 0; sl < nslabs; ++sl) {
        const int z0 = sl * slab, z1 = std::min(c->Z, z0 + slab);
        cudaStream_t s = (sl & 1) ? c->aux_stream : c->stream;
        BPParams b = jfdk::reconstruct_bp_params(c, c->d_hu_stage, nullptr);
        b.z_begin = z0;
        b.z_end = z1;
        if ((st = run_bp_on(c, b, true, s))) return drain(st);
        JFDK_CUDA(c, cudaEventRecord(ev[nchunks + sl], s), "event");
        JFDK_CUDA(c, cudaStreamWaitEvent(c->copy_stream, ev[nchunks + sl], 0), "event");
        JFDK_CUDA(c, cudaMemcpyAsync(h_hu + z0 * plane, c->d_hu_stage + z0 * plane, (size_t)(z1 - z0) * plane * 4,
                                     cudaMemcpyDeviceToHost, c->copy_stream),
                  "volume download");
    }
    JFDK_CUDA(c, cudaEventRecord(ev_done, c->copy_stream), "event");
    JFDK_CUDA(c, cudaStreamWaitEvent(c->stream, ev_done, 0), "event");
    if (timing) JFDK_CUDA(c, cudaEventRecord(c->ev[3], c->stream), "event");
    JFDK_CUDA(c, cudaStreamSynchronize(c->stream), "reconstruct_host");
    return JFDK_OK;
}

}  // extern "C"

// ---- derivatives ---------------------------------------------------------

namespace {

jfdk_status deriv_check(jfdk_ctx* c, const char* what) {
    if (mixed(c)) return fail(c, JFDK_ERR_UNSUPPORTED, std::string(what) + ": derivatives are of the FP32 form");
    if (!c->d_cnt || !c->bp_has_views)
        return fail(c, JFDK_ERR_STATE, std::string(what) + ": needs the weights of a backprojection (bp_accumulate)");
    if (!whole_volume(c))
        return fail(c, JFDK_ERR_STATE, std::string(what) + ": needs the weights of the whole volume, not a slab");
    return JFDK_OK;
}

jfdk_status ensure_rt(jfdk_ctx* c, const float* d_vol_bar) {
    const size_t n = (size_t)c->X * c->Y * c->Z;
    if (!c->d_rt) {
        jfdk_status st = dev_alloc(c, &c->d_rt, n, "the adjoint residual");
        if (st) return st;
    }
    JFDK_LAUNCH(c, launch_residual_over_weight(d_vol_bar, c->d_cnt, n, c->d_rt, c->stream), "residual / weight");
    return JFDK_OK;
}

AdjParams adj_params(const jfdk_ctx* c, int v0, int nv) {
    AdjParams a{};
    a.ptm = c->d_ptm;
    a.v0 = v0; a.nv = nv; a.num_views = c->nviews;
    a.U = c->out_w; a.V = c->rows; a.X = c->X; a.Y = c->Y; a.Z = c->Z;
    a.pxy = c->pxy; a.pz = c->pz;
    a.rt = c->d_rt;
    a.q_frame = frame_px(c);
    a.tw = c->d_tw;
    return a;
}

}  // namespace

extern "C" {

jfdk_status jfdk_set_bp_geometry(jfdk_ctx* c, const float* h_ptms) {
    if (!c || !h_ptms) return fail(c, JFDK_ERR_INVALID, "set_bp_geometry: bad argument");
    c->ptms.assign(h_ptms, h_ptms + (size_t)c->nviews * 12);
    c->wvol_state = 0;   // the normalisation weights follow the geometry
    c->w_depends_on_z = false;
    for (int v = 0; v < c->nviews; ++v)
        if (c->ptms[(size_t)v * 12 + 10] != 0.0f) c->w_depends_on_z = true;
    JFDK_CUDA(c, cudaMemcpyAsync(c->d_ptm, c->ptms.data(), sizeof(float) * c->ptms.size(), cudaMemcpyHostToDevice,
                                 c->stream),
              "projection matrices upload");
    JFDK_CUDA(c, cudaStreamSynchronize(c->stream), "projection matrices upload");
    return JFDK_OK;
}

jfdk_status jfdk_bp_adjoint(jfdk_ctx* c, const float* d_vol_bar, int v0, int nv, float* d_q_bar) {
    if (!c || !d_vol_bar || !d_q_bar || nv < 0 || v0 < 0 || v0 + nv > c->nviews)
        return fail(c, JFDK_ERR_INVALID, "bp_adjoint: bad argument");
    jfdk_status st = deriv_check(c, "bp_adjoint");
    if (st || nv == 0) return st;
    if (c->qadj_views < nv) {
        dev_free(c, c->d_qadj);
        c->qadj_views = 0;
        if ((st = dev_alloc(c, &c->d_qadj, (size_t)nv * frame_px(c), "the quad-space adjoint"))) return st;
        c->qadj_views = nv;
    }
    if ((st = ensure_rt(c, d_vol_bar))) return st;
    AdjParams a = adj_params(c, v0, nv);
    a.qbar = c->d_qadj;
    JFDK_LAUNCH(c, launch_bp_adjoint(a, c->w_depends_on_z, c->stream), "backprojection adjoint");
    JFDK_LAUNCH(c, launch_unpack_adjoint(c->d_qadj, frame_px(c), nv, c->rows, c->out_w, c->d_tw, v0, c->nviews,
                                         d_q_bar, c->stream),
                "backprojection adjoint (unpack)");
    return JFDK_OK;
}

jfdk_status jfdk_filter_adjoint(jfdk_ctx* c, const float* d_q_bar, int v0, int nv, float* d_p_bar) {
    if (!c || !d_q_bar || !d_p_bar || nv < 0 || v0 < 0) return fail(c, JFDK_ERR_INVALID, "filter_adjoint: bad argument");
    if (nv == 0) return JFDK_OK;
    const int kp = (int)round_up(c->out_w, 64);
    const size_t m = (size_t)nv * c->rows;
    // the padded rows of q_bar go where the forward keeps its A operand
    jfdk_status st = ensure_A(c, (m * kp + 2 * a_pitch(c) - 1) / (2 * a_pitch(c)));
    if (st) return st;
    float* ypad = static_cast<float*>(c->d_A);
    JFDK_LAUNCH(c, launch_pad_rows(d_q_bar, m, c->out_w, ypad, kp, c->stream), "filter adjoint (pad)");
    RampParams r{};
    r.A = ypad; r.e = nullptr; r.B = c->d_Tt; r.c = nullptr;
    r.M = (int)m; r.N = c->in_w; r.K = c->out_w; r.a_pitch = kp;
    r.rows = c->rows;
    r.q = d_p_bar; r.q_frame_stride = (long long)c->rows * c->in_w; r.q_pitch = c->in_w;
    r.b_scale = 1.0f;
    JFDK_LAUNCH(c, launch_ramp_gemm(r, c->stream), "filter adjoint (transposed product)");
    JFDK_LAUNCH(c, launch_filter_adjoint_finish(d_q_bar, c->out_w, d_p_bar, c->in_w, c->rows, nv, v0, c->nviews, c->d_pw,
                                                c->d_c, c->mirror, c->stream),
                "filter adjoint (weights)");
    return JFDK_OK;
}

jfdk_status jfdk_geometry_gradient(jfdk_ctx* c, const float* d_q, int v0, int nv, const float* d_vol,
                                   const float* d_vol_bar, const float* d_dptm, double* d_grad) {
    if (!c || !d_q || !d_vol || !d_vol_bar || !d_dptm || !d_grad || nv < 0 || v0 < 0 || v0 + nv > c->nviews)
        return fail(c, JFDK_ERR_INVALID, "geometry_gradient: bad argument");
    jfdk_status st = deriv_check(c, "geometry_gradient");
    if (st || nv == 0) return st;
    if ((st = ensure_Q4(c, nv))) return st;
    JFDK_LAUNCH(c, launch_pack_quads(d_q, frame_px(c), nv, c->rows, c->out_w, c->d_tw, v0, c->nviews, 1, c->d_q4,
                                     frame_px(c), 0, c->stream),
                "packing projections");
    if ((st = ensure_rt(c, d_vol_bar))) return st;
    AdjParams a = adj_params(c, v0, nv);
    a.q4 = c->d_q4;
    a.vol = d_vol;
    a.dptm = d_dptm;
    const size_t need = geometry_gradient_ctas(a) * 6 * (size_t)nv;
    if (c->partial_n < need) {
        dev_free(c, c->d_partial);
        c->partial_n = 0;
        if ((st = dev_alloc(c, &c->d_partial, need, "the gradient partial sums"))) return st;
        c->partial_n = need;
    }
    a.partial = c->d_partial;
    JFDK_LAUNCH(c, launch_geometry_gradient(a, c->w_depends_on_z, d_grad, c->stream), "geometry gradient");
    ++c->launches;  // the FP64 reduction
    return JFDK_OK;
}

}  // extern "C"

// ---- autotuner -------------------------------------------------------------

namespace {

std::mutex g_tune_mutex;
struct TuneChoice {
    int zpt, chunk, tile;   // slices per thread, views per chunk, tile width in x
};
std::map<std::string, TuneChoice> g_tune_cache;   // shape -> choice
bool g_tune_file_read = false;

std::string tune_key(const jfdk_ctx* c) {
    char k[256];
    std::snprintf(k, sizeof k, "p%d_r%d_v%d_u%d_h%d_w%d_x%d_y%d_z%d_wz%d", c->precision, ramp_kind(c), c->nviews,
                  c->used_u, c->used_v, c->in_w, c->X, c->Y, c->Z, c->w_depends_on_z ? 1 : 0);
    return k;
}

// Optional persistent cache: $JFDK_AUTOTUNE_CACHE, lines "key zpt chunk tile"
// (lines without the tile width, from earlier builds, read as width 4).
void tune_file_load() {
    if (g_tune_file_read) return;
    g_tune_file_read = true;
    const char* path = std::getenv("JFDK_AUTOTUNE_CACHE");
    if (!path) return;
    std::FILE* f = std::fopen(path, "r");
    if (!f) return;
    char line[512], key[256];
    while (std::fgets(line, sizeof line, f)) {
        int z = 0, ch = 0, tx = kBPTileX;
        if (std::sscanf(line, "%255s %d %d %d", key, &z, &ch, &tx) < 3) continue;
        if ((z == 4 || z == 8 || z == 16) && (ch == 16 || ch == 32 || ch == 64) && (tx == 4 || tx == 8 || tx == 32))
            g_tune_cache[key] = {z, ch, tx};
    }
    std::fclose(f);
}

void tune_file_append(const std::string& key, const TuneChoice& t) {
    const char* path = std::getenv("JFDK_AUTOTUNE_CACHE");
    if (!path) return;
    std::FILE* f = std::fopen(path, "a");
    if (!f) return;
    std::fprintf(f, "%s %d %d %d\n", key.c_str(), t.zpt, t.chunk, t.tile);
    std::fclose(f);
}

// The smaller of two timed runs after one warm-up run.
template <class F>
jfdk_status time_ms(jfdk_ctx* c, F&& run, float* ms) {
    cudaEvent_t a, b;
    JFDK_CUDA(c, cudaEventCreate(&a), "event");
    JFDK_CUDA(c, cudaEventCreate(&b), "event");
    jfdk_status st = run();
    float best = 1e30f;
    for (int i = 0; i < 2 && !st; ++i) {
        cudaEventRecord(a, c->stream);
        st = run();
        cudaEventRecord(b, c->stream);
        cudaEventSynchronize(b);
        float t = 0.0f;
        cudaEventElapsedTime(&t, a, b);
        best = std::min(best, t);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *ms = best;
    return st;
}

}  // namespace

extern "C" jfdk_status jfdk_autotune(jfdk_ctx* c, int flags) {
    if (!c) return JFDK_ERR_INVALID;
    const std::string key = tune_key(c);
    {
        std::lock_guard<std::mutex> lk(g_tune_mutex);
        tune_file_load();
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end() && !(flags & JFDK_AUTOTUNE_FORCE)) {
            c->opt_bp_zpt = it->second.zpt;
            c->opt_view_chunk = it->second.chunk;
            c->opt_bp_tile = it->second.tile;
            return JFDK_OK;
        }
    }
    jfdk_status st = ensure_Q4(c, c->nviews);
    if (st) return st;
    // voxel tile (depth x width): a finalizing backprojection of a central
    // slab into a slab-sized buffer (the kernel indexes the output by
    // absolute slice, so it is given the buffer's address minus the slab's
    // offset)
    const int nz = std::min(c->Z, 32);
    const int z0 = (c->Z - nz) / 2;
    const size_t plane = (size_t)c->X * c->Y;
    float* slab = nullptr;
    if ((st = dev_alloc(c, &slab, plane * nz, "the autotuner's slab"))) return st;
    int best_z = 8, best_x = kBPTileX;
    float best_t = 1e30f;
    ensure_weights(c, c->stream);   // not inside the first candidate's time
    for (int zpt : {4, 8, 16}) {
        if (zpt == 16 && !mixed(c)) continue;   // the FP32 form: 139 against 128 ms on c2
        for (int tx : {4, 8, 32}) {
            if (zpt == 16 && tx != kBPTileX) continue;   // 16-slice tiles are 4 wide
            c->opt_bp_zpt = zpt;
            c->opt_bp_tile = tx;
            BPParams b = jfdk::reconstruct_bp_params(c, slab - (ptrdiff_t)(z0 * plane), nullptr);
            b.z_begin = z0;
            b.z_end = z0 + nz;
            b.apply_ct = 0;
            float t = 0.0f;
            st = time_ms(c, [&] { return run_bp(c, b, true); }, &t);
            if (st) break;
            if (t < best_t) { best_t = t; best_z = zpt; best_x = tx; }
        }
        if (st) break;
    }
    dev_free(c, slab);
    if (st) return st;
    c->opt_bp_zpt = best_z;
    c->opt_bp_tile = best_x;
    // views per chunk: the filter stage over the first views of zero frames
    int best_c = c->opt_view_chunk;
    if (c->in_w == c->used_u) {   // (compositing reads conjugate frames of the whole rotation)
        const int nsub = std::min(c->nviews, 128);
        uint16_t* raw = nullptr;
        const size_t frame = (size_t)c->scan.num_dets_u * c->scan.num_dets_v;
        if ((st = dev_alloc(c, &raw, frame * nsub, "the autotuner's frames"))) return st;
        JFDK_CUDA(c, cudaMemsetAsync(raw, 0, frame * nsub * sizeof(uint16_t), c->stream), "autotune");
        best_t = 1e30f;
        for (int ch : {16, 32, 64}) {
            c->opt_view_chunk = ch;
            float t = 0.0f;
            st = time_ms(c, [&] { return jfdk::reconstruct_filter_stage(c, raw, nsub); }, &t);
            if (st) break;
            if (t < best_t) { best_t = t; best_c = ch; }
        }
        cudaStreamSynchronize(c->stream);
        dev_free(c, raw);
        if (st) return st;
    }
    c->opt_view_chunk = best_c;
    std::lock_guard<std::mutex> lk(g_tune_mutex);
    g_tune_cache[key] = {best_z, best_c, best_x};
    tune_file_append(key, g_tune_cache[key]);
    return JFDK_OK;
}
