// ramp_gemm_tc.cu -- the ramp filter product Q = A T^T + e c^T on the 5th
// generation tensor cores (tcgen05, sm_100a).
//
// Operands (all K-major, K = filter input columns padded to 32):
//   A  [M][Kp] fp32  weighted detector rows (prep.cu), loaded by TMA;
//   Bh [N][Kp], Bl [N][Kp]  the Toeplitz operator split on the host into two
//      TF32-exact parts (Bh = RN_tf32(T), Bl = RN_tf32(T - Bh)).
// FP32-class accuracy from TF32 tensor cores: each A tile is split in shared
// memory into Ah = RN_tf32(A) and Al = RN_tf32(A - Ah) and the CTA issues
// Ah*Bh + Ah*Bl + Al*Bh (the dropped Al*Bl term is ~2^-22 relative), all
// accumulated in FP32 in tensor memory.
//
// Tile 128 x 128 per CTA, K in blocks of 32 (one 128-byte swizzle atom per
// row), 3-stage TMA / mbarrier pipeline.  Thread 0 issues TMA and MMA; all four
// warps split A and, after the last MMA, read the accumulator out of tensor
// memory (warp w owns TMEM lanes 32w..32w+31 = tile rows) and store rows of Q
// with the rank-1 truncation-ramp term c[n] e[m] added.
//
// Every mbarrier wait is bounded: on timeout the CTA records a code in the
// context's device status word and skips the rest of its work (no trap).
// TMA loads never use cluster multicast and read only this GPU's memory.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>

#include "jfdk_internal.h"

namespace jfdk {
namespace {

constexpr int BM = 128, BN = 128, BK = 32, STAGES = 3;
constexpr int TILE_A = BM * BK * 4;          // 16 KB
constexpr int TILE_B = BN * BK * 4;          // 16 KB
constexpr int STAGE_BYTES = 2 * TILE_A + 2 * TILE_B;  // A, Al, Bh, Bl
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
constexpr uint32_t TX_BYTES = TILE_A + 2 * TILE_B;   // bytes TMA delivers per stage
constexpr uint32_t kWaitLimit = 1u << 22;           // polls before a wait gives up

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// Bounded parity wait: true when the phase with parity `parity` completed.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (uint32_t i = 0; i < kWaitLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// K-major operand tile of `rows` x 128 bytes, 128-byte swizzle, 8-row atoms
// 1024 bytes apart (Blackwell shared-memory matrix descriptor, version 1).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Instruction descriptor: kind::tf32, D = F32, A = B = TF32, both K-major,
// M = 128, N = 128.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(BN >> 3) << 17) |
                            ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}"
        ::"r"(tmem_d), "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// Round to the nearest TF32 value (10 explicit mantissa bits, ties to even).
__device__ __forceinline__ float tf32_rn(float x) {
    uint32_t b = __float_as_uint(x);
    if ((b & 0x7f800000u) != 0x7f800000u) b = (b + 0xfffu + ((b >> 13) & 1u)) & 0xffffe000u;
    return __uint_as_float(b);
}

struct TcArgs {
    RampParams p;
    int* status;
};

__global__ void __launch_bounds__(128, 1) ramp_gemm_tc_kernel(const __grid_constant__ CUtensorMap mapA,
                                                             const __grid_constant__ CUtensorMap mapBh,
                                                             const __grid_constant__ CUtensorMap mapBl,
                                                             TcArgs args) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    const RampParams& p = args.p;
    const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;     // 1024-aligned for SW128
    uint8_t* gbase = smem_raw + (base - smem_u32(smem_raw));
    // barrier block after the stages
    const uint32_t bars = base + STAGES * STAGE_BYTES;
    auto full = [&](int s) { return bars + 8u * s; };
    auto empty = [&](int s) { return bars + 8u * (STAGES + s); };
    const uint32_t done_bar = bars + 8u * (2 * STAGES);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(gbase + STAGES * STAGE_BYTES + 8 * (2 * STAGES + 1));
    __shared__ int abort_flag;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int n0 = blockIdx.x * BN, m0 = blockIdx.y * BM;
    const int nk = p.a_pitch / BK;

    if (tid == 0) {
        abort_flag = 0;
        for (int s = 0; s < STAGES; ++s) { mbar_init(full(s), 1); mbar_init(empty(s), 1); }
        mbar_init(done_bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mapA)) : "memory");
    }
    if (warp == 0) {  // 128 TMEM columns hold the 128 x 128 FP32 accumulator
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(tmem_slot)), "r"(128));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    auto stageA = [&](int s) { return base + (uint32_t)(s * STAGE_BYTES); };
    auto stageAl = [&](int s) { return stageA(s) + TILE_A; };
    auto stageBh = [&](int s) { return stageA(s) + 2 * TILE_A; };
    auto stageBl = [&](int s) { return stageA(s) + 2 * TILE_A + TILE_B; };
    auto load_stage = [&](int kb, int s) {
        mbar_expect_tx(full(s), TX_BYTES);
        tma_load_2d(stageA(s), &mapA, kb * BK, m0, full(s));
        tma_load_2d(stageBh(s), &mapBh, kb * BK, n0, full(s));
        tma_load_2d(stageBl(s), &mapBl, kb * BK, n0, full(s));
    };

    if (tid == 0)
        for (int kb = 0; kb < nk && kb < STAGES; ++kb) load_stage(kb, kb);

    for (int kb = 0; kb < nk; ++kb) {
        const int s = kb % STAGES;
        const uint32_t ph = (uint32_t)(kb / STAGES) & 1u;
        if (!abort_flag && !mbar_wait(full(s), ph)) abort_flag = 1;
        // Split A into RN_tf32(A) (in place) and RN_tf32(A - that).  The
        // swizzle permutes 16-byte chunks within the tile, so an elementwise
        // pass keeps both tiles in the layout the descriptors describe.
        if (!abort_flag) {
            float4* a = reinterpret_cast<float4*>(gbase + s * STAGE_BYTES);
            float4* al = reinterpret_cast<float4*>(gbase + s * STAGE_BYTES + TILE_A);
#pragma unroll 4
            for (int i = tid; i < TILE_A / 16; i += 128) {
                float4 v = a[i], h, l;
                h.x = tf32_rn(v.x); h.y = tf32_rn(v.y); h.z = tf32_rn(v.z); h.w = tf32_rn(v.w);
                l.x = tf32_rn(v.x - h.x); l.y = tf32_rn(v.y - h.y); l.z = tf32_rn(v.z - h.z); l.w = tf32_rn(v.w - h.w);
                a[i] = h;
                al[i] = l;
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0 && !abort_flag) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int k = 0; k < BK / 8; ++k) {  // kind::tf32: K = 8 per MMA (32 bytes)
                const uint32_t off = (uint32_t)k * 32u;
                const uint64_t da = smem_desc(stageA(s) + off), dal = smem_desc(stageAl(s) + off);
                const uint64_t dbh = smem_desc(stageBh(s) + off), dbl = smem_desc(stageBl(s) + off);
                mma_tf32(tmem, da, dbh, (kb > 0 || k > 0) ? 1u : 0u);
                mma_tf32(tmem, da, dbl, 1u);
                mma_tf32(tmem, dal, dbh, 1u);
            }
            mma_commit(empty(s));
            // refill the stage used one iteration ago (its MMAs overlap ours)
            if (kb >= 1 && kb - 1 + STAGES < nk) {
                const int sp = (kb - 1) % STAGES;
                if (!mbar_wait(empty(sp), (uint32_t)((kb - 1) / STAGES) & 1u)) abort_flag = 1;
                else load_stage(kb - 1 + STAGES, sp);
            }
        }
    }
    if (tid == 0) mma_commit(done_bar);
    __syncthreads();
    if (!abort_flag && !mbar_wait(done_bar, 0)) abort_flag = 1;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    // Epilogue: warp w holds tile rows 32w + lane.
    const int m = m0 + warp * 32 + lane;
    const bool row_ok = m < p.M && !abort_flag;
    const float em = row_ok ? p.e[m] : 0.0f;
    float* qrow = nullptr;
    if (row_ok) {
        const int vl = m / p.rows, row = m - vl * p.rows;
        qrow = p.q + (size_t)vl * p.q_frame_stride + (size_t)row * p.q_pitch;
    }
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 16) {
        uint32_t r[16];
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (row_ok) {
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int n = n0 + c0 + j;
                if (n < p.N) qrow[n] = fmaf(__ldg(p.c + n), em, __uint_as_float(r[j]));
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128));
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

bool make_map(CUtensorMap* map, const float* ptr, int rows, int cols_padded, int box_rows) {
    EncodeFn enc = encoder();
    if (!enc) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)cols_padded, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)cols_padded * 4};
    const cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(ptr), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

float tf32_round_host(float x) {
    uint32_t b;
    std::memcpy(&b, &x, 4);
    if ((b & 0x7f800000u) != 0x7f800000u) b = (b + 0xfffu + ((b >> 13) & 1u)) & 0xffffe000u;
    float r;
    std::memcpy(&r, &b, 4);
    return r;
}

cudaError_t launch_ramp_gemm_tc(const RampParams& p, const float* Bh, const float* Bl, int* status,
                                cudaStream_t s) {
    if (p.a_pitch % BK != 0) return cudaErrorInvalidValue;
    CUtensorMap ma, mbh, mbl;
    if (!make_map(&ma, p.A, p.M, p.a_pitch, BM) || !make_map(&mbh, Bh, p.N, p.a_pitch, BN) ||
        !make_map(&mbl, Bl, p.N, p.a_pitch, BN))
        return cudaErrorInvalidValue;
    static bool attr_set = false;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(ramp_gemm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             SMEM_BYTES);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    dim3 grid((p.N + BN - 1) / BN, (p.M + BM - 1) / BM);
    TcArgs a{p, status};
    ramp_gemm_tc_kernel<<<grid, 128, SMEM_BYTES, s>>>(ma, mbh, mbl, a);
    return cudaGetLastError();
}

}  // namespace jfdk
