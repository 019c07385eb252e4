// ramp_gemm_tc.cu -- the ramp filter product Q = A T^T + e c^T on the 5th
// generation tensor cores (tcgen05, sm_100a), as a split-precision product.
//
// Operands (all K-major, K = filter input columns padded to a multiple of 64):
//   Ah, Al [M][Kp]  the weighted detector rows split into a high and a low
//                   part by the producing kernel (prep.cu);
//   Bh, Bl [N][Kp]  the Toeplitz operator split the same way on the host.
// The CTA accumulates Ah*Bh + Ah*Bl + Al*Bh in FP32 in tensor memory (the
// dropped Al*Bl term is below the split's precision).  Element kinds:
//   TF32x3  tf32 parts in fp32 storage, kind::tf32 -- ~2^-22 relative, the
//           FP32 form's product;
//   BF16x3  bf16 parts, kind::f16 -- ~2^-17 relative, twice the MMA rate;
//   FP16x3  fp16 parts of rows scaled by a power of two per row (row_scale)
//           and of the operator scaled by b_scale, kind::f16 -- ~2^-22
//           relative at the bf16 rate; the epilogue undoes both scales.
//
// Persistent, warp-specialised CTA of 6 warps, one CTA per SM:
//   warp 0       TMA producer: 4 tiles per K block into a 3-stage ring;
//   warp 1       owns the tensor memory; one thread issues the MMAs of a tile
//                into one of two 128-column accumulators;
//   warps 2..5   epilogue: read their 32 accumulator lanes (tile rows) with
//                tcgen05.ld, add c[n] e[m], store rows of Q -- overlapping the
//                next tile's MMAs in the other accumulator.
// Every mbarrier wait is bounded: on timeout the CTA raises a shared abort
// flag and records a code in the context's device status word; every role
// then stops waiting, the MMA thread drains its MMAs, the producer waits
// (bounded) for its copies in flight, and the tensor memory is freed.
// TMA loads never use cluster multicast and read only this GPU's memory.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>

#include "jfdk_internal.h"

namespace jfdk {
namespace {

constexpr int BM = 128, BN = 128, STAGES = 3;
constexpr int TILE = 128 * 128;                       // bytes: 128 rows x 128 bytes of K
constexpr int STAGE_BYTES = 4 * TILE;                 // Ah, Al, Bh, Bl
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
constexpr uint32_t kWaitLimit = 1u << 22;            // polls before a wait gives up
constexpr int kThreads = 192;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Bounded parity wait: true when the phase with parity `parity` completed;
// false when it gave up or another role already aborted.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
    for (uint32_t i = 0; i < kWaitLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if ((i & 255u) == 255u && *abort_flag) return false;
    }
    *abort_flag = 1;
    return false;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// K-major operand tile of 128 rows x 128 bytes, 128-byte swizzle, 8-row atoms
// 1024 bytes apart (Blackwell shared-memory matrix descriptor, version 1).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Instruction descriptor: D = F32, A/B type, both K-major, M = 128, N = 128.
constexpr uint32_t idesc(uint32_t ab_type) {
    return (1u << 4) | (ab_type << 7) | (ab_type << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

template <int KIND>
__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
    if constexpr (KIND == RAMP_TF32X3) {
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}"
            ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc(2)), "r"(accumulate));
    } else {
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}"
            ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc(KIND == RAMP_BF16X3 ? 1u : 0u)), "r"(accumulate));
    }
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

struct TcArgs {
    RampParams p;
    int* status;
};

template <int KIND>
__global__ void __launch_bounds__(kThreads, 1) ramp_tc_kernel(const __grid_constant__ CUtensorMap mapAh,
                                                              const __grid_constant__ CUtensorMap mapAl,
                                                              const __grid_constant__ CUtensorMap mapBh,
                                                              const __grid_constant__ CUtensorMap mapBl,
                                                              TcArgs args) {
    constexpr int ELEM = KIND == RAMP_TF32X3 ? 4 : 2;
    constexpr int BK = 128 / ELEM;          // K elements per 128-byte row
    constexpr int KSTEPS = 128 / 32;        // MMAs per K block: 32 bytes of K each
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    const RampParams& p = args.p;
    const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;     // 1024-aligned for SW128
    uint8_t* gbase = smem_raw + (base - smem_u32(smem_raw));
    const uint32_t bars = base + STAGES * STAGE_BYTES;
    auto full = [&](int s) { return bars + 8u * s; };
    auto empty = [&](int s) { return bars + 8u * (STAGES + s); };
    auto tfull = [&](int b) { return bars + 8u * (2 * STAGES + b); };
    auto tempty = [&](int b) { return bars + 8u * (2 * STAGES + 2 + b); };
    const uint32_t drain_bar = bars + 8u * (2 * STAGES + 4);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(gbase + STAGES * STAGE_BYTES + 8 * (2 * STAGES + 5));
    __shared__ int abort_flag;
    volatile int* abort_v = &abort_flag;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nk = p.a_pitch / BK;
    const int tiles_n = (p.N + BN - 1) / BN, tiles = ((p.M + BM - 1) / BM) * tiles_n;

    if (tid == 0) {
        abort_flag = 0;
        for (int s = 0; s < STAGES; ++s) { mbar_init(full(s), 1); mbar_init(empty(s), 1); }
        for (int b = 0; b < 2; ++b) { mbar_init(tfull(b), 1); mbar_init(tempty(b), 4); }
        mbar_init(drain_bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {  // two 128-column FP32 accumulators
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(tmem_slot)), "r"(2 * BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    auto stage = [&](int s, int t) { return base + (uint32_t)(s * STAGE_BYTES + t * TILE); };

    if (warp == 0) {
        // ---- TMA producer ----
        if (lane == 0) {
            uint32_t it = 0;
            for (int t = blockIdx.x; t < tiles && !*abort_v; t += gridDim.x) {
                const int m0 = (t / tiles_n) * BM, n0 = (t % tiles_n) * BN;
                for (int kb = 0; kb < nk; ++kb, ++it) {
                    const int s = (int)(it % STAGES);
                    if (it >= STAGES && !mbar_wait(empty(s), ((it / STAGES) - 1) & 1u, abort_v)) break;
                    mbar_expect_tx(full(s), STAGE_BYTES);
                    tma_load_2d(stage(s, 0), &mapAh, kb * BK, m0, full(s));
                    tma_load_2d(stage(s, 1), &mapAl, kb * BK, m0, full(s));
                    tma_load_2d(stage(s, 2), &mapBh, kb * BK, n0, full(s));
                    tma_load_2d(stage(s, 3), &mapBl, kb * BK, n0, full(s));
                }
            }
            // copies still in flight land before the CTA exits (bounded)
            if (*abort_v) {
                const uint32_t first = it > STAGES ? it - STAGES : 0;
                for (uint32_t j = first; j < it; ++j) {
                    int dummy = 0;
                    mbar_wait(full((int)(j % STAGES)), (j / STAGES) & 1u, &dummy);
                }
            }
        }
    } else if (warp == 1) {
        // ---- MMA issuer ----
        if (lane == 0) {
            uint32_t it = 0, i = 0;
            for (int t = blockIdx.x; t < tiles && !*abort_v; t += gridDim.x, ++i) {
                const int b = (int)(i & 1u);
                if (i >= 2 && !mbar_wait(tempty(b), ((i >> 1) - 1) & 1u, abort_v)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t acc = tmem + (uint32_t)(b * BN);
                bool ok = true;
                for (int kb = 0; kb < nk; ++kb, ++it) {
                    const int s = (int)(it % STAGES);
                    if (!mbar_wait(full(s), (it / STAGES) & 1u, abort_v)) { ok = false; break; }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
                    for (int k = 0; k < KSTEPS; ++k) {
                        const uint32_t off = (uint32_t)k * 32u;
                        const uint64_t dah = smem_desc(stage(s, 0) + off), dal = smem_desc(stage(s, 1) + off);
                        const uint64_t dbh = smem_desc(stage(s, 2) + off), dbl = smem_desc(stage(s, 3) + off);
                        mma<KIND>(acc, dah, dbh, (kb > 0 || k > 0) ? 1u : 0u);
                        mma<KIND>(acc, dah, dbl, 1u);
                        mma<KIND>(acc, dal, dbh, 1u);
                    }
                    mma_commit(empty(s));
                }
                if (!ok) break;
                mma_commit(tfull(b));
            }
            // all issued MMAs complete before the tensor memory is freed
            mma_commit(drain_bar);
            int dummy = 0;
            mbar_wait(drain_bar, 0, &dummy);
        }
    } else {
        // ---- epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 ----
        const int quarter = warp & 3;
        uint32_t i = 0;
        for (int t = blockIdx.x; t < tiles && !*abort_v; t += gridDim.x, ++i) {
            const int b = (int)(i & 1u);
            if (!mbar_wait(tfull(b), (i >> 1) & 1u, abort_v)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int m0 = (t / tiles_n) * BM, n0 = (t % tiles_n) * BN;
            const int m = m0 + quarter * 32 + lane;
            const bool row_ok = m < p.M;
            float em = 0.0f, rs = 1.0f, amax = 0.0f;
            float* qrow = nullptr;
            int vl = -1;
            if (row_ok) {
                em = p.e[m];
                if (p.row_scale) rs = p.row_scale[m] * p.b_scale;
                vl = m / p.rows;
                const int row = m - vl * p.rows;
                qrow = p.q + (size_t)vl * p.q_frame_stride + (size_t)row * p.q_pitch;
            }
#pragma unroll 1
            for (int c0 = 0; c0 < BN; c0 += 16) {
                uint32_t r[16];
                const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(b * BN + c0);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                      "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                      "=r"(r[15])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                const int n = n0 + c0;
                if (row_ok && n < p.N) {
                    float o[16];
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        o[j] = fmaf(__ldg(p.c + (n + j < p.N ? n + j : p.N - 1)), em, __uint_as_float(r[j]) * rs);
                        if (n + j < p.N) amax = fmaxf(amax, fabsf(o[j]));
                    }
                    if (p.vec_store && n + 16 <= p.N) {
                        float4* d = reinterpret_cast<float4*>(qrow + n);
#pragma unroll
                        for (int j = 0; j < 4; ++j) d[j] = make_float4(o[4 * j], o[4 * j + 1], o[4 * j + 2], o[4 * j + 3]);
                    } else {
#pragma unroll
                        for (int j = 0; j < 16; ++j)
                            if (n + j < p.N) qrow[n + j] = o[j];
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(tempty(b));
            if (p.absmax) {  // per-view max |q|; non-negative floats order like their bits
                unsigned bits = __float_as_uint(amax);
                const int v_first = __shfl_sync(0xffffffffu, vl, 0);
                if (__all_sync(0xffffffffu, vl == v_first)) {
                    bits = __reduce_max_sync(0xffffffffu, bits);
                    if (lane == 0 && v_first >= 0) atomicMax(p.absmax + v_first, bits);
                } else if (vl >= 0) {
                    atomicMax(p.absmax + vl, bits);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * BN));
    if (tid == 0 && abort_flag) atomicOr(args.status, 1);
}

// ---- the int8 product -------------------------------------------------------
// Rows a = 2^(E-24) Q_a and the operator T = 2^(F-24) Q_b, Q 32-bit fixed
// point (|Q| <= 127 * 2^24) cut into balanced signed bytes d0..d3, Q =
// d0 2^24 + d1 2^16 + d2 2^8 + d3.  The CTA forms the ten byte products
// with s + t <= 3 on the tensor cores (kind::i8), each level l = s + t
// summed exactly in its own int32 accumulator (|sum| <= 4 K 2^14 < 2^31 for
// K < 32768), and the epilogue combines the levels exactly in int64, V =
// sum_l acc_l 2^(8 (3 - l)), and rounds once: q = RN(2^(E+F-24) V + c e),
// V and the edge term in FP64.  Integer accumulation is exact and order
// free, so q does not depend on the tiling; the digits hold the operands
// to 2^-31 of their largest values and the dropped products (s + t >= 4)
// are below 2^-30 of the leading one.
//
// Tile 128 rows x kI8TileN columns, K blocks of kI8BlockK bytes (128-byte
// swizzle, whole 128-byte rows as the TMA reads best): per stage the four
// row digit planes (one 3-D TMA load, 64 KB) and the operator digit planes
// that are not all zero in this block (the host's mask; far from the
// diagonal the leading bytes of the ramp are zero), up to 32 KB.  Two sets of four level accumulators of kI8TileN
// columns fill the tensor memory, so one tile's epilogue overlaps the next
// tile's MMAs.
constexpr int I8_BN = kI8TileN, I8_BK = kI8BlockK, I8_STAGES = 2, I8_LEVELS = 4, I8_PRODUCTS = 10;
constexpr int I8_ATILE = BM * I8_BK;                         // one row digit plane: 16 KB
constexpr int I8_BTILE = I8_BN * I8_BK;                      // one operator digit plane: 8 KB
constexpr int I8_STAGE_BYTES = kI8RowDigits * I8_ATILE + kI8OpDigits * I8_BTILE;
constexpr int I8_SMEM_BYTES = I8_STAGES * I8_STAGE_BYTES + 1024 + 256;
constexpr int I8_ACC_COLS = I8_LEVELS * I8_BN;               // one accumulator set
static_assert(2 * I8_ACC_COLS == 512, "two accumulator sets fill the tensor memory");
static_assert(I8_BK == 128 && I8_ATILE % 1024 == 0 && I8_BTILE % 1024 == 0 && I8_STAGE_BYTES % 1024 == 0,
              "128-byte swizzle atoms");
static_assert(I8_SMEM_BYTES <= 227 * 1024, "shared memory");
// (row byte, operator byte) of each product, by level; first[p]: the first
// product of its level (starts the accumulator in the first K step)
__constant__ const unsigned char kI8S[I8_PRODUCTS] = {0, 0, 1, 0, 1, 2, 0, 1, 2, 3};
__constant__ const unsigned char kI8T[I8_PRODUCTS] = {0, 1, 0, 2, 1, 0, 3, 2, 1, 0};
__constant__ const unsigned char kI8First[I8_PRODUCTS] = {1, 1, 0, 1, 0, 0, 1, 0, 0, 0};

// D = S32, A = B = signed 8-bit, both K-major, M = 128, N = I8_BN.
constexpr uint32_t kI8Idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(I8_BN >> 3) << 17) |
                              ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}"
        ::"r"(tmem_d), "l"(da), "l"(db), "r"(kI8Idesc), "r"(accumulate));
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int x, int y, int z, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}

struct I8Args {
    RampParams p;
    const uint8_t* masks;    // [tiles_n][nk]
    int* status;
};

__global__ void __launch_bounds__(kThreads, 1) ramp_i8_kernel(const __grid_constant__ CUtensorMap mapA,
                                                               const __grid_constant__ CUtensorMap mapB,
                                                               I8Args args) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    const RampParams& p = args.p;
    const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;
    uint8_t* gbase = smem_raw + (base - smem_u32(smem_raw));
    const uint32_t bars = base + I8_STAGES * I8_STAGE_BYTES;
    auto full = [&](int s) { return bars + 8u * s; };
    auto empty = [&](int s) { return bars + 8u * (I8_STAGES + s); };
    auto tfull = [&](int b) { return bars + 8u * (2 * I8_STAGES + b); };
    auto tempty = [&](int b) { return bars + 8u * (2 * I8_STAGES + 2 + b); };
    const uint32_t drain_bar = bars + 8u * (2 * I8_STAGES + 4);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(gbase + I8_STAGES * I8_STAGE_BYTES + 8 * (2 * I8_STAGES + 5));
    __shared__ int abort_flag;
    volatile int* abort_v = &abort_flag;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nk = (p.a_pitch + I8_BK - 1) / I8_BK;   // the last block reads zeros past K
    const int tiles_n = (p.N + I8_BN - 1) / I8_BN, tiles = ((p.M + BM - 1) / BM) * tiles_n;

    if (tid == 0) {
        abort_flag = 0;
        for (int s = 0; s < I8_STAGES; ++s) { mbar_init(full(s), 1); mbar_init(empty(s), 1); }
        for (int b = 0; b < 2; ++b) { mbar_init(tfull(b), 1); mbar_init(tempty(b), 4); }
        mbar_init(drain_bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {  // two sets of four level accumulators, I8_BN int32 columns each
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(tmem_slot)), "r"(2 * I8_ACC_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    auto a_tile = [&](int s) { return base + (uint32_t)(s * I8_STAGE_BYTES); };
    auto b_tile = [&](int s, int t) {
        return base + (uint32_t)(s * I8_STAGE_BYTES + kI8RowDigits * I8_ATILE + t * I8_BTILE);
    };
    // operator digit planes used in K block kb of output tile nt: all of
    // them in the first block (it starts every level's accumulator)
    auto block_mask = [&](int nt, int kb) -> uint32_t {
        return kb == 0 ? (1u << kI8OpDigits) - 1u : (uint32_t)__ldg(args.masks + (size_t)nt * nk + kb);
    };

    if (warp == 0) {
        // ---- TMA producer ----
        if (lane == 0) {
            uint32_t it = 0;
            for (int t = blockIdx.x; t < tiles && !*abort_v; t += gridDim.x) {
                const int nt = t % tiles_n;
                const int m0 = (t / tiles_n) * BM, n0 = nt * I8_BN;
                for (int kb = 0; kb < nk; ++kb, ++it) {
                    const int s = (int)(it % I8_STAGES);
                    if (it >= I8_STAGES && !mbar_wait(empty(s), ((it / I8_STAGES) - 1) & 1u, abort_v)) break;
                    const uint32_t mask = block_mask(nt, kb);
                    mbar_expect_tx(full(s), (uint32_t)(kI8RowDigits * I8_ATILE) + (uint32_t)__popc(mask) * I8_BTILE);
                    tma_load_3d(a_tile(s), &mapA, kb * I8_BK, m0, 0, full(s));
                    for (int d = 0; d < kI8OpDigits; ++d)
                        if ((mask >> d) & 1u) tma_load_3d(b_tile(s, d), &mapB, kb * I8_BK, n0, d, full(s));
                }
            }
            if (*abort_v) {   // copies still in flight land before the CTA exits (bounded)
                const uint32_t first = it > I8_STAGES ? it - I8_STAGES : 0;
                for (uint32_t j = first; j < it; ++j) {
                    int dummy = 0;
                    mbar_wait(full((int)(j % I8_STAGES)), (j / I8_STAGES) & 1u, &dummy);
                }
            }
        }
    } else if (warp == 1) {
        // ---- MMA issuer ----
        if (lane == 0) {
            uint32_t it = 0, i = 0;
            for (int t = blockIdx.x; t < tiles && !*abort_v; t += gridDim.x, ++i) {
                const int nt = t % tiles_n;
                const int b = (int)(i & 1u);
                if (i >= 2 && !mbar_wait(tempty(b), ((i >> 1) - 1) & 1u, abort_v)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t acc = tmem + (uint32_t)(b * I8_ACC_COLS);
                bool ok = true;
                for (int kb = 0; kb < nk; ++kb, ++it) {
                    const int s = (int)(it % I8_STAGES);
                    const uint32_t mask = block_mask(nt, kb);
                    if (!mbar_wait(full(s), (it / I8_STAGES) & 1u, abort_v)) { ok = false; break; }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
                    for (int ks = 0; ks < I8_BK / 32; ++ks) {
                        const uint32_t off = (uint32_t)ks * 32u;
#pragma unroll
                        for (int q = 0; q < I8_PRODUCTS; ++q) {
                            if (!((mask >> kI8T[q]) & 1u)) continue;
                            const uint32_t level = (uint32_t)(kI8S[q] + kI8T[q]);
                            const uint64_t da = smem_desc(a_tile(s) + (uint32_t)kI8S[q] * I8_ATILE + off);
                            const uint64_t db = smem_desc(b_tile(s, kI8T[q]) + off);
                            mma_i8(acc + level * (uint32_t)I8_BN, da, db, (kb == 0 && ks == 0 && kI8First[q]) ? 0u : 1u);
                        }
                    }
                    mma_commit(empty(s));
                }
                if (!ok) break;
                mma_commit(tfull(b));
            }
            mma_commit(drain_bar);   // all issued MMAs complete before the tensor memory is freed
            int dummy = 0;
            mbar_wait(drain_bar, 0, &dummy);
        }
    } else {
        // ---- epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 ----
        const int quarter = warp & 3;
        uint32_t i = 0;
        for (int t = blockIdx.x; t < tiles && !*abort_v; t += gridDim.x, ++i) {
            const int b = (int)(i & 1u);
            if (!mbar_wait(tfull(b), (i >> 1) & 1u, abort_v)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int m0 = (t / tiles_n) * BM, n0 = (t % tiles_n) * I8_BN;
            const int m = m0 + quarter * 32 + lane;
            const bool row_ok = m < p.M;
            double em = 0.0, scale = 0.0;
            float amax = 0.0f;
            float* qrow = nullptr;
            int vl = -1;
            if (row_ok) {
                em = (double)p.e[m];
                scale = (double)p.row_scale[m] * (double)p.b_scale * 0x1p-24;
                vl = m / p.rows;
                const int row = m - vl * p.rows;
                qrow = p.q + (size_t)vl * p.q_frame_stride + (size_t)row * p.q_pitch;
            }
#pragma unroll 1
            for (int c0 = 0; c0 < I8_BN; c0 += 16) {
                uint32_t r[I8_LEVELS][16];
#pragma unroll
                for (int l = 0; l < I8_LEVELS; ++l) {
                    const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) +
                                           (uint32_t)(b * I8_ACC_COLS + l * I8_BN + c0);
                    asm volatile(
                        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                        : "=r"(r[l][0]), "=r"(r[l][1]), "=r"(r[l][2]), "=r"(r[l][3]), "=r"(r[l][4]), "=r"(r[l][5]),
                          "=r"(r[l][6]), "=r"(r[l][7]), "=r"(r[l][8]), "=r"(r[l][9]), "=r"(r[l][10]), "=r"(r[l][11]),
                          "=r"(r[l][12]), "=r"(r[l][13]), "=r"(r[l][14]), "=r"(r[l][15])
                        : "r"(taddr));
                }
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                const int n = n0 + c0;
                if (row_ok && n < p.N) {
                    float o[16];
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        // exact: |acc_l| < 2^31, so |V| < 2^56
                        long long v = (int)r[0][j];
#pragma unroll
                        for (int l = 1; l < I8_LEVELS; ++l) v = v * 256 + (int)r[l][j];
                        const double cn = (double)__ldg(p.c + (n + j < p.N ? n + j : p.N - 1));
                        o[j] = (float)fma((double)v, scale, cn * em);
                        if (n + j < p.N) amax = fmaxf(amax, fabsf(o[j]));
                    }
                    if (p.vec_store && n + 16 <= p.N) {
                        float4* d = reinterpret_cast<float4*>(qrow + n);
#pragma unroll
                        for (int j = 0; j < 4; ++j) d[j] = make_float4(o[4 * j], o[4 * j + 1], o[4 * j + 2], o[4 * j + 3]);
                    } else {
#pragma unroll
                        for (int j = 0; j < 16; ++j)
                            if (n + j < p.N) qrow[n + j] = o[j];
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(tempty(b));
            if (p.absmax) {  // per-view max |q|; non-negative floats order like their bits
                unsigned bits = __float_as_uint(amax);
                const int v_first = __shfl_sync(0xffffffffu, vl, 0);
                if (__all_sync(0xffffffffu, vl == v_first)) {
                    bits = __reduce_max_sync(0xffffffffu, bits);
                    if (lane == 0 && v_first >= 0) atomicMax(p.absmax + v_first, bits);
                } else if (vl >= 0) {
                    atomicMax(p.absmax + vl, bits);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * I8_ACC_COLS));
    if (tid == 0 && abort_flag) atomicOr(args.status, 1);
}

// ---- host: tensor maps through the driver entry point --------------------

using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn encoder() {
    static EncodeFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeFn>(p);
    });
    return fn;
}

// rows x cols (elements) K-major matrix; box = 128 bytes of K x 128 rows.
bool make_map(CUtensorMap* map, const void* ptr, int kind, int rows, int cols) {
    EncodeFn enc = encoder();
    if (!enc) return false;
    const int elem = kind == RAMP_TF32X3 ? 4 : 2;
    const CUtensorMapDataType dt = kind == RAMP_TF32X3   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                   : kind == RAMP_BF16X3 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                                         : CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)cols * elem};
    const cuuint32_t box[2] = {(cuuint32_t)(128 / elem), 128u};
    const cuuint32_t estr[2] = {1, 1};
    return enc(map, dt, 2, const_cast<void*>(ptr), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// planes x rows x cols int8 (K-major planes, plane_bytes apart); box =
// 128 bytes of K x box_rows rows x box_planes planes, 128-byte swizzle.
bool make_map_i8(CUtensorMap* map, const void* ptr, int planes, int rows, int cols, long long plane_bytes,
                 int box_rows, int box_planes) {
    EncodeFn enc = encoder();
    if (!enc) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)cols, (cuuint64_t)rows, (cuuint64_t)planes};
    const cuuint64_t strides[2] = {(cuuint64_t)cols, (cuuint64_t)plane_bytes};
    const cuuint32_t box[3] = {(cuuint32_t)I8_BK, (cuuint32_t)box_rows, (cuuint32_t)box_planes};
    const cuuint32_t estr[3] = {1, 1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(ptr), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int sm_count() {
    static int n = 0;
    static std::once_flag once;
    std::call_once(once, [] {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1) n = 148;
    });
    return n;
}

template <int KIND>
cudaError_t launch_kind(const RampParams& p, const void* Ah, const void* Al, const void* Bh, const void* Bl,
                        int* status, cudaStream_t s) {
    CUtensorMap mah, mal, mbh, mbl;
    if (!make_map(&mah, Ah, KIND, p.M, p.a_pitch) || !make_map(&mal, Al, KIND, p.M, p.a_pitch) ||
        !make_map(&mbh, Bh, KIND, p.N, p.a_pitch) || !make_map(&mbl, Bl, KIND, p.N, p.a_pitch))
        return cudaErrorInvalidValue;
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [] {
        attr = cudaFuncSetAttribute(ramp_tc_kernel<KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    });
    if (attr != cudaSuccess) return attr;
    const int tiles = ((p.M + BM - 1) / BM) * ((p.N + BN - 1) / BN);
    const int grid = tiles < sm_count() ? tiles : sm_count();
    TcArgs a{p, status};
    ramp_tc_kernel<KIND><<<grid, kThreads, SMEM_BYTES, s>>>(mah, mal, mbh, mbl, a);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_ramp_i8(const RampParams& p, const int8_t* A, long long a_plane, const int8_t* B,
                           long long b_plane, const uint8_t* masks, int* status, cudaStream_t s) {
    if (p.a_pitch % 16 != 0 || p.M < 1 || p.N < 1 || !p.row_scale || !masks) return cudaErrorInvalidValue;
    if ((reinterpret_cast<uintptr_t>(A) & 15) || (reinterpret_cast<uintptr_t>(B) & 15) || a_plane % 16 ||
        b_plane % 16)
        return cudaErrorInvalidValue;
    CUtensorMap ma, mb;
    if (!make_map_i8(&ma, A, kI8RowDigits, p.M, p.a_pitch, a_plane, BM, kI8RowDigits) ||
        !make_map_i8(&mb, B, kI8OpDigits, p.N, p.a_pitch, b_plane, I8_BN, 1))
        return cudaErrorInvalidValue;
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [] {
        attr = cudaFuncSetAttribute(ramp_i8_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, I8_SMEM_BYTES);
    });
    if (attr != cudaSuccess) return attr;
    const int tiles = ((p.M + BM - 1) / BM) * ((p.N + I8_BN - 1) / I8_BN);
    const int grid = tiles < sm_count() ? tiles : sm_count();
    I8Args a{p, masks, status};
    ramp_i8_kernel<<<grid, kThreads, I8_SMEM_BYTES, s>>>(ma, mb, a);
    return cudaGetLastError();
}

float tf32_round_host(float x) {
    uint32_t b;
    std::memcpy(&b, &x, 4);
    if ((b & 0x7f800000u) != 0x7f800000u) b = (b + 0xfffu + ((b >> 13) & 1u)) & 0xffffe000u;
    float r;
    std::memcpy(&r, &b, 4);
    return r;
}

cudaError_t launch_ramp_gemm_tc(const RampParams& p, int kind, const void* Ah, const void* Al, const void* Bh,
                                const void* Bl, int* status, cudaStream_t s) {
    const int bk = kind == RAMP_TF32X3 ? 32 : 64;
    if (p.a_pitch % bk != 0 || p.M < 1 || p.N < 1) return cudaErrorInvalidValue;
    switch (kind) {
        case RAMP_TF32X3: return launch_kind<RAMP_TF32X3>(p, Ah, Al, Bh, Bl, status, s);
        case RAMP_BF16X3: return launch_kind<RAMP_BF16X3>(p, Ah, Al, Bh, Bl, status, s);
        case RAMP_FP16X3: return launch_kind<RAMP_FP16X3>(p, Ah, Al, Bh, Bl, status, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace jfdk
