/*
 * jfdk.h -- C ABI of the B200-native FDK reconstruction engine (libjfdk.so).
 *
 * This is the drop-in boundary under JEngine's Agent/Pipe surface: the C++
 * agents in jenhine_b200/host (PreProcessingAgent, FilterAgent, BPCUDAAgent,
 * CTNumAgent) call these entry points; nothing else in the engine is exposed.
 *
 * Conventions
 *  - Plain C types only: pointers, sizes, floats.  Device pointers ("d_") are
 *    CUDA device addresses owned by the caller; host pointers ("h_") are host
 *    memory (pinned is faster, pageable works).
 *  - Every call returns jfdk_status; no C++ exception crosses the ABI.  The
 *    message of the last failure is jfdk_last_error(ctx).
 *  - One context per CUDA stream.  A context is not thread-safe: callers
 *    serialise on it (the reference issues all CUDA work of BPCUDAAgent from
 *    its single WorkFlow0 thread, BPCUDAAgent/BPCUDAAgent.cpp:84-111).
 *  - All work is enqueued on the context's stream; calls return without
 *    synchronising unless stated.  jfdk_sync waits for the stream.
 *  - An out-of-memory failure returns JFDK_ERR_OOM and a message starting with
 *    "CUDA failed to malloc " -- the prefix JEngine's retry loop matches
 *    (CUDA/DeviceMemory.cpp:60-66, JEngine/JEngine.cpp:413-421).
 *  - Sizes beyond what the kernels index with 32-bit offsets per frame are
 *    rejected with JFDK_ERR_INVALID; nothing is silently truncated.
 */
#ifndef JFDK_H
#define JFDK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int jfdk_status;
enum {
    JFDK_OK = 0,
    JFDK_ERR_INVALID = -1,      /* bad argument or size                         */
    JFDK_ERR_CUDA = -2,         /* CUDA runtime or launch failure               */
    JFDK_ERR_OOM = -3,          /* device allocation failed                     */
    JFDK_ERR_UNSUPPORTED = -4,  /* valid in the reference, not implemented here */
    JFDK_ERR_STATE = -5,        /* call out of order (e.g. finalize, no views)  */
    JFDK_ERR_NO_DEVICE = -6     /* no usable sm_100 device                      */
};

/* Arithmetic of the filtered projections and the ramp product. */
enum {
    JFDK_PRECISION_FP32 = 0,  /* plain form: FP32 end to end                    */
    JFDK_PRECISION_MIXED = 1  /* FP16 filtered projections with a per-view scale;
                                 BF16x3 split-precision ramp product            */
};

/* Scan parameters: Config/ScanParams.h:13-40. */
typedef struct jfdk_scan_params {
    int num_views;             /* NumViews: views per rotation                  */
    float dso;                 /* DSO, mm                                       */
    float dsd;                 /* DSD, mm                                       */
    int num_dets_u;            /* NumDetsU: raw frame columns                   */
    int num_dets_v;            /* NumDetsV: raw frame rows                      */
    float detector_pixel_size; /* DetectorPixelSize, mm                         */
    int border_up, border_down, border_left, border_right; /* BorderSize*     */
    float bright_field;        /* BrightField (scalar GainCorr divisor)         */
    float beam_hardening[3];   /* BeamHardeningParams (a0, a1, a2)              */
    float half_sample_rate;    /* HalfSampleRate; <= 0 derives it from the
                                  detector as Config/ConfigHelper.cpp:52-53      */
    int detector_on_right;     /* FilterAgent detectorAtTheRight / FilterCore
                                  yMirroring (JEngine/JEngine.cpp:153-162)       */
    int filter_input_width;    /* FilterAgent nInputWidth; 0 = used columns      */
} jfdk_scan_params;

/* Reconstruction parameters: Config/ReconParams.h:14-68. */
typedef struct jfdk_recon_params {
    int num_pixels_x, num_pixels_y, num_pixels_z; /* NumPixelsX/Y/Z              */
    float pitch_xy, pitch_z;                      /* PitchXY, PitchZ, mm          */
    float ct_norm0, ct_norm1;                     /* CTNumNorm0, CTNumNorm1       */
    float mu_water;                               /* MuWater (0.02 in the
                                                     reference, ConfigHelper.cpp:70) */
    float filter_cutoff_start, filter_cutoff_end; /* FilterCutOffStart/End        */
    int num_adjust;                               /* |FilterAdjustPoints|         */
    const float* adjust_points;                   /* FilterAdjustPoints           */
    const float* adjust_level_db;                 /* FilterAdjustLevelInDB        */
    int z_filter;                                 /* apply ZFilterAgent's [1/4,1/2,1/4]
                                                     row smoothing (FilterAgent/
                                                     ZFilterAgent.cpp:49-71)       */
} jfdk_recon_params;

typedef struct jfdk_ctx jfdk_ctx;

/* Create a context on the current device and the given CUDA stream (NULL =
 * the legacy default stream; the caller keeps ownership of a stream it
 * passes and must keep it alive until jfdk_destroy; all buffers the caller
 * hands in must be ready on that stream).  ptms: num_views x 12 floats, row-major 3x4 projection
 * matrices (TransformMatrix/ProjectionMatrix.h:11-19) already adjusted the
 * way JEngine/JEngine.cpp:139-150 does.  Replaces the constructors of
 * PreProcessingCore, FilterCore + PreFilterWeightGenerator, BPCUDACore and
 * CTNumCore (PreProcessingAgent/PreProcessingCore.cpp:15-65,
 * FilterAgent/FilterCore.cpp:13-61, FilterAgent/PreFilterWeightGenerator.cpp:
 * 10-50, BPCUDAAgent/BPCUDACore.cpp:17-127, CTNumAgent/CTNumCore.cpp:8-20). */
jfdk_status jfdk_create(jfdk_ctx** out, const jfdk_scan_params* scan,
                        const jfdk_recon_params* recon, const float* h_ptms,
                        int precision, void* cuda_stream);
void jfdk_destroy(jfdk_ctx* ctx);
const char* jfdk_last_error(const jfdk_ctx* ctx);
jfdk_status jfdk_sync(jfdk_ctx* ctx);
/* Geometry-derived sizes: filter input/output width, FFT length, rows. */
jfdk_status jfdk_get_dims(const jfdk_ctx* ctx, int* filter_in_w, int* filter_out_w,
                          int* fft_length, int* rows);

/* ---- stage entry points (the agents' Cores) ------------------------------ */

/* PreProcessingCore::Process for nv frames
 * (PreProcessingAgent/PreProcessingCore.cpp:67-86): uint16 -> float, clamp at
 * 1, border crop, / BrightField, -ln, beam hardening.  d_raw: nv x NumDetsV x
 * NumDetsU uint16; d_out: nv x NumUsedDetsV x NumUsedDetsU float. */
jfdk_status jfdk_preprocess_frames(jfdk_ctx* ctx, const uint16_t* d_raw, int nv, float* d_out);

/* FilterAgent::ProcessTask + FilterCore::ProcessRow for views [v0, v0+nv) of
 * the rotation (FilterAgent/FilterAgent.cpp:99-192, FilterCore.cpp:189-222):
 * cosine pre-weight of the view's 9-view group, truncation ramp, ramp filter.
 * d_in: nv x rows x filter_in_w float; d_out: nv x rows x filter_out_w float. */
jfdk_status jfdk_filter_frames(jfdk_ctx* ctx, const float* d_in, int v0, int nv, float* d_out);

/* jfdk_filter_frames for callers that must not allocate device memory while
 * they run: hosts whose framework owns all device memory through its own
 * pool or budget, and acquisition threads that cannot afford a cudaMalloc
 * (it can synchronise the device and take milliseconds).  No counterpart in
 * the reference: it is an addition of this library.  Same inputs and outputs
 * as jfdk_filter_frames; its working rows live in one 4 MiB array compiled
 * into libjfdk.so (held by every GPU that loads the library until the process
 * exits) instead of memory allocated on first use; nothing is allocated or
 * freed.  The ramp product always runs on FP32 CUDA cores, whatever the
 * context's precision or JFDK_OPT_RAMP_PRODUCT: the result equals
 * jfdk_filter_frames' under JFDK_RAMP_FP32_SIMT bit for bit and the other
 * products' within their rounding (rel-L2 <= 1e-5 against I8x14, TF32x3
 * and FP16x3, <= 5e-5 against BF16x3).  Limit: nv * rows * pitch + nv * rows
 * floats must fit in 1,048,576 floats, where pitch is filter_in_w rounded up
 * to a multiple of 64 (for a 768 x 768 frame: one view per call); larger
 * requests return JFDK_ERR_INVALID.  The first call on each device looks up
 * the array's device address (with that device current) and caches it for
 * the life of the process; the cache is not valid across cudaDeviceReset.
 * All calls share the array: calls whose kernels can overlap on the GPU race
 * and must be serialised. */
jfdk_status jfdk_filter_frames_noalloc(jfdk_ctx* ctx, const float* d_in, int v0, int nv, float* d_out);

/* CompositeAgent::ProcessTask + CompositeCore::Process
 * (CompositeAgent/CompositeAgent.cpp:72-83, CompositeCore.cpp:59-149):
 * nv pairs of preprocessed frames -- d_dirc[f] of view v0 + f and d_conj[f] of
 * view (v0 + f + N/2) % N, each rows x width -- into d_out, nv x rows x
 * (2 width): the direct frame in one half (the right half when
 * detector_on_right), in the other the conjugate frame resampled at the points
 * the direct view's extended detector sees, blended with the direct edge over
 * 40 columns.  The context must have filter_input_width = 2 x the frame width
 * (JFDK_ERR_STATE otherwise); jfdk_reconstruct then composites on the fly. */
jfdk_status jfdk_composite_frames(jfdk_ctx* ctx, const float* d_dirc, const float* d_conj, int v0, int nv,
                                  float* d_out);

/* ZFilterAgent::ProcessTask (FilterAgent/ZFilterAgent.cpp:49-71) in place on
 * nv frames of rows x width. */
jfdk_status jfdk_zfilter_frames(jfdk_ctx* ctx, float* d_frames, int nv);

/* BPCUDACore::DeployBackProj for views [v0, v0+nv) of filtered frames
 * (BPCUDAAgent/BPCUDACore.cu:25-66, with BPCore's edge semantics,
 * BPAgent/BPCore.cpp:115-196): u-taper, voxel-driven bilinear backprojection,
 * accumulated into the context's sum and weight volumes.  d_proj: nv x rows
 * x filter_out_w float.  A view with IsShotStart first calls jfdk_bp_reset. */
jfdk_status jfdk_bp_reset(jfdk_ctx* ctx);
/* Restrict jfdk_bp_reset, jfdk_bp_accumulate and jfdk_finalize to slices
 * [z_begin, z_begin + z_count) of the volume: one part of a volume
 * reconstructed in numReconParts parts of numSlicesPerRecon slices, all
 * views backprojected once per part (BPCUDAAgent/BPCUDAAgent.cpp:231-287,
 * BPCUDACore.cpp:17-38, JEngine/JEngine.cpp:167-175).  The accumulators are
 * sized to z_count slices here, so an out-of-memory failure surfaces at this
 * call (JFDK_ERR_OOM, "CUDA failed to malloc ..."), where JEngine's retry
 * loop expects it.  jfdk_finalize then takes slices of the slab only.  The
 * default slab is the whole volume; the derivatives need the whole volume. */
jfdk_status jfdk_bp_set_slab(jfdk_ctx* ctx, int z_begin, int z_count);
/* Allocate now the packed store jfdk_bp_accumulate needs for calls of up to
 * `views` views (otherwise the first such call allocates it), so that every
 * allocation of the accumulating backprojection happens before the first
 * frame arrives: with jfdk_bp_set_slab, at the agent's GetReady, where
 * JEngine's retry loop catches an out-of-memory failure. */
jfdk_status jfdk_bp_reserve(jfdk_ctx* ctx, int views);
jfdk_status jfdk_bp_accumulate(jfdk_ctx* ctx, const float* d_proj, int v0, int nv);

/* BPCore::DoneSlice + CTNumCore::Process for slices [z0, z0+nz)
 * (BPAgent/BPCore.cpp:198-205, CTNumAgent/CTNumCore.cpp:22-36): voxel =
 * sum / weight, then HU.  Either output may be NULL.  apply_ctnum = 0 gives
 * the raw normalised backprojection (the reference's "Slice" pipe before
 * CTNumAgent). d_out: nz x Y x X float; d_out16: int16 HU rounded toward zero
 * with saturation (Performance/BasicMathIPP.cpp:224-227). */
jfdk_status jfdk_finalize(jfdk_ctx* ctx, int z0, int nz, int apply_ctnum, float* d_out,
                          int16_t* d_out16);

/* CTNumCore::Process on n floats in place. */
jfdk_status jfdk_ctnum(jfdk_ctx* ctx, float* d_inout, size_t n);

/* ---- whole-volume path -------------------------------------------------- */

/* All stages for one rotation: raw frames (device) -> HU volume (device).
 * Views are preprocessed, weighted and filtered in chunks into the filtered
 * projection store, then backprojected in one pass with CT numbers fused into
 * the final store.  d_hu and/or d_hu16 may be NULL (not both). */
jfdk_status jfdk_reconstruct(jfdk_ctx* ctx, const uint16_t* d_raw, float* d_hu, int16_t* d_hu16);

/* Same with host buffers: h_raw (num_views x NumDetsV x NumDetsU uint16) is
 * copied in, h_hu (Z x Y x X float) copied out; synchronous. */
jfdk_status jfdk_reconstruct_host(jfdk_ctx* ctx, const uint16_t* h_raw, float* h_hu);

/* ---- one volume over several GPUs: z-slabs ------------------------------- */
/* The stages of jfdk_reconstruct, split so that GPUs can share a volume: each
 * filters a part of the views into its context's projection store
 * (jfdk_filter_to_store), the stores are completed by an all-gather of the
 * ranges jfdk_store_range names (one NCCL all-gather over NVLink; no
 * counterpart in the reference), and each GPU backprojects its own slab of
 * slices from every view (jfdk_backproject_store).  Results equal
 * jfdk_reconstruct's bit for bit when the slabs start at multiples of the
 * tile depth (jfdk_get_option(JFDK_OPT_BP_ZPT)). */
/* The filter stage of jfdk_reconstruct for views [v0, v0+nv) of the
 * rotation -- preprocessing (and compositing), pre-weight, ramp filter,
 * z-filter -- into caller-owned filtered frames: d_raw the rotation's frames
 * (num_views x NumDetsV x NumDetsU uint16; only these views, and their
 * conjugates when compositing, are read), d_frames nv x rows x filter_out_w
 * float.  A z-slab rank filters its share of the views with it; the frames
 * of all views (4 bytes a pixel) are then exchanged and each rank
 * backprojects them into its slab with jfdk_bp_set_slab / jfdk_bp_reset /
 * jfdk_bp_accumulate (views in order) / jfdk_finalize, which equals
 * jfdk_reconstruct on those slices bit for bit. */
jfdk_status jfdk_filter_raw(jfdk_ctx* ctx, const uint16_t* d_raw, int v0, int nv, float* d_frames);
/* Filter views [v0, v0+nv) into the store.  d_raw: the rotation's frames
 * (num_views x NumDetsV x NumDetsU uint16); only the frames of these views
 * (and, when compositing, of their conjugates) are read. */
jfdk_status jfdk_filter_to_store(jfdk_ctx* ctx, const uint16_t* d_raw, int v0, int nv);
/* Device address and size of the store's records of views [v0, v0+nv)
 * (contiguous, views in order; 16 bytes a pixel in the FP32 form, 8 in the
 * mixed form) and, in the mixed form, of their per-view scales (4 bytes a
 * view; *d_scales = NULL in the FP32 form). */
jfdk_status jfdk_store_range(jfdk_ctx* ctx, int v0, int nv, void** d_records, size_t* record_bytes,
                             float** d_scales);
/* The finalizing backprojection of every view in the store, with CT numbers,
 * into slices [z0, z0+nz): d_hu / d_hu16 hold those slices only
 * (nz x Y x X); either may be NULL. */
jfdk_status jfdk_backproject_store(jfdk_ctx* ctx, int z0, int nz, float* d_hu, int16_t* d_hu16);

/* ---- options --------------------------------------------------------------- */
enum {
    JFDK_OPT_BP_EXACT = 1,    /* FP32 form.  1: backprojection rounds every
                                 step like BPCore (bit-identical sums);
                                 0 (default): the same sample coordinates
                                 (correctly rounded quotients), lerps fused
                                 into FMAs                                      */
    JFDK_OPT_VIEW_CHUNK = 2,  /* views preprocessed + filtered per launch in
                                 jfdk_reconstruct (default 32)                   */
    JFDK_OPT_STAGE_TIMING = 3,/* 1: jfdk_reconstruct records CUDA events on its
                                 stream around each stage                        */
    JFDK_OPT_BP_ZPT = 4,      /* slices each backprojection thread keeps in
                                 registers: 4, 8 or 16; 0 (default): 16 in the
                                 mixed form when W does not depend on z and the
                                 volume holds at least 8 waves of 16-slice
                                 tiles (c2 does, c1 does not), else 8.
                                 The FP32 form's volume does not depend on it;
                                 the mixed form's coordinates step from each
                                 tile's first slice, so its volume does      */
    JFDK_OPT_FILTER_SIMT = 5, /* 1: ramp product on FP32 CUDA cores (same as
                                 JFDK_OPT_RAMP_PRODUCT = JFDK_RAMP_FP32_SIMT);
                                 0: the form's default                          */
    JFDK_OPT_RAMP_PRODUCT = 6,/* how the ramp product runs, a jfdk_ramp_product */
    JFDK_OPT_DEVICE_MEMORY_LIMIT = 7, /* bytes of device memory the context may hold
                                 in all (0, default: no limit).  An allocation
                                 that would exceed it fails like cudaMalloc:
                                 JFDK_ERR_OOM, "CUDA failed to malloc ...".  Lets
                                 a caller sharing the GPU bound the engine, and
                                 choose the z-parts of jfdk_bp_set_slab ahead  */
    JFDK_OPT_BP_TILE = 8,     /* backprojection CTA width in x: 4 (4 x 32
                                 threads), 8 (8 x 16) or 32 (32 x 4); 0
                                 (default): 4.  16-slice tiles are 4 wide.  The
                                 volume does not depend on it                  */
    JFDK_OPT_BP_WEIGHTS = 9   /* 1 (default): a backprojection over
                                 every view of the rotation (jfdk_reconstruct,
                                 jfdk_reconstruct_host, jfdk_backproject_store)
                                 divides by a volume of normalisation weights
                                 computed once per geometry and backprojection
                                 rounding (X*Y*Z floats, on first use) instead of
                                 accumulating the taper per sample; the volume is
                                 the same bit for bit.  Without room for it the
                                 weights are accumulated per sample.  0: always
                                 per sample                                     */
};
/* Ramp products (JFDK_OPT_RAMP_PRODUCT).  The split products run on the
 * tcgen05 tensor cores as hi*hi + hi*lo + lo*hi with FP32 accumulation; the
 * int8 product runs on them with exact int32 accumulation. */
typedef enum {
    JFDK_RAMP_DEFAULT = 0,    /* I8x14 in the FP32 form, BF16x3 in the mixed form  */
    JFDK_RAMP_TF32X3 = 1,     /* ~2^-22 relative                                    */
    JFDK_RAMP_BF16X3 = 2,     /* ~2^-17 relative, twice the tensor rate of TF32    */
    JFDK_RAMP_FP16X3 = 3,     /* rows and operator scaled by powers of two into the
                                 FP16 range; ~2^-22 relative at the BF16 rate     */
    JFDK_RAMP_FP32_SIMT = 4,  /* FP32 CUDA cores                                    */
    JFDK_RAMP_I8X14 = 5       /* rows and the operator (from its FP64 kernel) as
                                 32-bit fixed point below power-of-two scales, each
                                 cut into four signed bytes; the ten leading byte
                                 products summed exactly in int32, combined exactly
                                 in int64, rounded once: the product of the float
                                 rows to ~2^-30 of the leading term, independent of
                                 the tiling (the FP32 form's default)            */
} jfdk_ramp_product;
jfdk_status jfdk_set_option(jfdk_ctx* ctx, int key, long long value);
/* The value an option has in effect: the set value, or the default the
 * context resolves it to (JFDK_OPT_BP_ZPT: the tile depth its
 * backprojection runs with; JFDK_OPT_BP_TILE: its tile width;
 * JFDK_OPT_RAMP_PRODUCT: the product its filter runs). */
jfdk_status jfdk_get_option(jfdk_ctx* ctx, int key, long long* value);
/* Stage times (ms) of the last jfdk_reconstruct with JFDK_OPT_STAGE_TIMING:
 * [0] preprocess + pre-weight + ramp filter (+ z-filter) + packing for the
 * backprojector, [1] reserved (0), [2] backprojection with normalisation and
 * CT numbers.  Synchronises the stream. */
jfdk_status jfdk_stage_times(jfdk_ctx* ctx, float* ms3);

/* ---- derivatives of the FP32 form ------------------------------------------
 * vol = S q / C is the backprojection of filtered projections q with the
 * weights C (the backprojected u-taper) fixed; the filter is
 * y = T (w o x) + c e(x), e(x) the edge mean of x.  Both are linear; these
 * entry points are their adjoints and the gradient with respect to the
 * backprojection's projection matrices.  FP32 contexts only
 * (JFDK_ERR_UNSUPPORTED in the mixed form).  No counterpart in the
 * reference, which has no derivatives. */

/* Replace the projection matrices the backprojector uses (num_views x 12,
 * host); the filter's pre-weight and the u-taper keep the matrices given to
 * jfdk_create.  Used to backproject under per-view motion. */
jfdk_status jfdk_set_bp_geometry(jfdk_ctx* ctx, const float* h_ptms);
/* q_bar = S^T (vol_bar / C) for views [v0, v0 + nv): d_vol_bar is
 * num_pixels_z x y x x, d_q_bar nv x rows x filter_out_w.  C is the weight
 * volume of the last jfdk_bp_accumulate sequence (JFDK_ERR_STATE without). */
jfdk_status jfdk_bp_adjoint(jfdk_ctx* ctx, const float* d_vol_bar, int v0, int nv, float* d_q_bar);
/* x_bar = w o (T^T y_bar) + (c . y_bar) / 3 on the three edge samples:
 * d_q_bar nv x rows x filter_out_w in, d_p_bar nv x rows x filter_in_w out. */
jfdk_status jfdk_filter_adjoint(jfdk_ctx* ctx, const float* d_q_bar, int v0, int nv, float* d_p_bar);
/* Gradient of a loss L(vol) with respect to parameters theta_j of the
 * projection matrices of views [v0, v0 + nv): d_q the filtered projections
 * (nv x rows x filter_out_w) the volume d_vol was backprojected from,
 * d_vol_bar = dL/dvol, d_dptm = dP/dtheta_j (nv x 6 x 12, device),
 * d_grad (nv x 6 doubles, device) receives dL/dtheta.  Per-CTA partial sums
 * in FP32, the reduction over the volume in FP64. */
jfdk_status jfdk_geometry_gradient(jfdk_ctx* ctx, const float* d_q, int v0, int nv, const float* d_vol,
                                   const float* d_vol_bar, const float* d_dptm, double* d_grad);

/* ---- autotuner and batches (no counterpart in the reference) -------------- */

/* Pick the backprojection's voxel tile (JFDK_OPT_BP_ZPT: 4 or 8 slices per
 * thread, and 16 in the mixed form; JFDK_OPT_BP_TILE: 4, 8 or 32 threads wide
 * in x, 128 per CTA, 16-slice tiles 4 wide) and
 * the filter stage's views per chunk (JFDK_OPT_VIEW_CHUNK: 16, 32 or 64) for
 * this context's shape by timing the candidates on the device (a 32-slice
 * slab, the first 128 views of zero frames).  Results are cached per shape in the process and, when
 * $JFDK_AUTOTUNE_CACHE names a file, appended to it and read back by later
 * processes.  Synchronises the context's stream. */
enum { JFDK_AUTOTUNE_FORCE = 1 };  /* re-time even when the shape is cached */
jfdk_status jfdk_autotune(jfdk_ctx* ctx, int flags);

/* A batch of scans (one context each, all of the same form) reconstructed
 * together, on one of two schedules:
 *  - persistent: every scan's filter stage (the scans dealt over four
 *    streams, so small scans' stages run side by side), then ONE persistent
 *    backprojection launch over the tiles of up to 16 scans (scans in order;
 *    a CTA takes the next tile when it finishes one, so scans of uneven size
 *    leave no tail; each scan keeps its own tile depth; scans whose W depends
 *    on z differently, and the mixed form's 16-slice scans, share launches of
 *    their own kind);
 *  - pipelined: each scan's own backprojection launch, the filter stage of
 *    the next scan running beside it on a second stream.
 * JFDK_BATCH_AUTOTUNE tunes each context (jfdk_autotune) and, on the first
 * run, times both schedules and keeps the faster; JFDK_BATCH_PERSISTENT or
 * JFDK_BATCH_PIPELINED fixes one (default: persistent).  With
 * JFDK_BATCH_GRAPH the first jfdk_batch_run with a set of buffers runs the
 * pipeline directly and records it as a CUDA graph; later runs with the same
 * buffers replay the graph (one launch from the host).  The batch runs on
 * `cuda_stream` (NULL: a stream of its own, ordered after the legacy default
 * stream); the contexts' own streams are restored after each run.  Each
 * volume equals the scan's own jfdk_reconstruct bit for bit. */
typedef struct jfdk_batch jfdk_batch;
enum {
    JFDK_BATCH_AUTOTUNE = 1,
    JFDK_BATCH_GRAPH = 2,
    JFDK_BATCH_PERSISTENT = 4,
    JFDK_BATCH_PIPELINED = 8
};
jfdk_status jfdk_batch_create(jfdk_batch** out, jfdk_ctx* const* ctxs, int n, int flags, void* cuda_stream);
void jfdk_batch_destroy(jfdk_batch* batch);
const char* jfdk_batch_last_error(const jfdk_batch* batch);
/* d_raw[i]: scan i's raw frames (device), d_hu[i]: its HU volume (device). */
jfdk_status jfdk_batch_run(jfdk_batch* batch, const uint16_t* const* d_raw, float* const* d_hu);
/* Kernels the batch has run: its persistent launches, plus every kernel of
 * each graph replay (a direct run's filter-stage kernels are counted by the
 * contexts, jfdk_kernel_launches). */
long long jfdk_batch_launches(const jfdk_batch* batch);
/* The schedule in use: 0 not chosen yet (before the first run),
 * JFDK_BATCH_PERSISTENT or JFDK_BATCH_PIPELINED. */
int jfdk_batch_schedule(const jfdk_batch* batch);

/* ---- introspection (tests, autotuner) ------------------------------------ */

/* The per-view BP u-taper (num_views x filter_out_w floats, host), computed as
 * BPCore.cpp:68-100. */
jfdk_status jfdk_get_uweights(const jfdk_ctx* ctx, float* h_out);
/* The ramp operator: h_T is filter_out_w x filter_in_w (row j = output
 * column j), h_c the edge-ramp response (filter_out_w). */
jfdk_status jfdk_get_ramp_operator(const jfdk_ctx* ctx, float* h_T, float* h_c);
/* Number of kernels this context has launched (a counter, for benchmarks). */
long long jfdk_kernel_launches(const jfdk_ctx* ctx);
/* Bytes of device memory the context holds now (what
 * JFDK_OPT_DEVICE_MEMORY_LIMIT bounds). */
long long jfdk_device_bytes(const jfdk_ctx* ctx);

/* The backprojector's fetch ceiling on the current device (no counterpart in
 * the reference): samples per second that the load path delivers when warps
 * do nothing but a backprojection sample's loads -- one record_bytes (16 or
 * 8) record per lane, plus an 8-byte taper pair when with_taper, `distinct`
 * consecutive records per warp request (1-32), from an L1-resident table,
 * at warps_per_sm resident warps (a multiple of 4, 4-64).  The ceiling that
 * a backprojection's samples per second are measured against.  Allocates
 * and frees 100 KB of device memory; synchronises. */
jfdk_status jfdk_measure_gather_rate(int record_bytes, int with_taper, int distinct, int warps_per_sm,
                                     double* samples_per_s);

/* jfdk_sync also reports JFDK_ERR_CUDA when a kernel's bounded wait gave up
 * (the device status word is then cleared). */

/* Library build / device check: 0 when an sm_100 device is current. */
jfdk_status jfdk_device_check(char* msg, int msg_len);

#ifdef __cplusplus
}
#endif
#endif /* JFDK_H */
