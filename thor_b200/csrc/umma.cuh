// BF16 tensor-core GEMM on the 5th-generation tensor cores (tcgen05) of sm_100a.
//
//   D[M x N] = A[M x K] . B[N x K]^T      A, B bf16, row-major (K contiguous, "K-major"),
//                                         FP32 accumulation in tensor memory (TMEM)
//
// One CTA computes a 128 x BN tile of D; the operands move by TMA (gemm_tma_kernel below), the
// accumulator is read back with tcgen05.ld and a fused element-wise epilogue writes the outputs.
// Descriptor formats (shared-memory matrix descriptor, instruction descriptor for kind::f16)
// follow the PTX ISA for tcgen05; field positions as in CUTLASS's cute/arch/mma_sm100_desc.hpp.
// Requirements on the caller: M a multiple of 128, N a multiple of BN, K a multiple of 64, all
// row starts 16-byte aligned (K a multiple of 8).
#pragma once

#include <cstdint>
#include <mutex>

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace thorx {
namespace umma {

constexpr int kM       = 128; // rows of a CTA tile (tensor-core M)
constexpr int kKChunk  = 64;  // K elements staged per round
constexpr int kThreads = 128;

// Epilogues. z is the pre-activation of a layer (acc + bias), bias per output column.
enum Epi : int {
    kEpiF32         = 0, // out_f32[m][n] = acc
    kEpiBiasF32     = 1, // out_f32[m][n] = acc + bias[n]
    kEpiBiasGelu    = 2, // out_bf16[m][n] = gelu(z); out_dg[m][n] = bf16(gelu'(z)) if out_dg
    kEpiGeluBwdBf16 = 3, // out_bf16[m][n] = acc * dg_in[m][n]  (dg_in: the stored gelu'(z))
    kEpiBf16        = 4, // out_bf16[m][n] = acc
    kEpiBiasF32T    = 5, // out_f32[n][m] = acc + bias[n] (transposed: ldo = rows of the plane)
};

struct EpiArgs {
    float*               out_f32;
    __nv_bfloat16*       out_bf16;
    __nv_bfloat16*       out_dg; // gelu'(z), kept for the backward pass when training
    const __nv_bfloat16* dg_in;
    const float*         bias;
    int            ldo;     // leading dimension of the outputs (elements)
    size_t         zstride; // split-K: elements between the partial outputs of consecutive splits
};

// GELU in its tanh form, 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))) (Hendrycks & Gimpel,
// "Gaussian Error Linear Units", 2016), with the hardware tanh (tanh.approx.f32, relative error
// about 2^-11, below the bf16 rounding of the activations): value and derivative share one tanh.
__device__ __forceinline__ float tanh_fast(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ void gelu_and_grad(float z, float& g, float& dg) {
    const float c = 0.7978845608028654f, a = 0.044715f, z2 = z * z;
    const float t = tanh_fast(c * z * (1.0f + a * z2));
    g             = 0.5f * z * (1.0f + t);
    dg            = 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * c * (1.0f + 3.0f * a * z2);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Instruction descriptor, kind::f16: D f32, A and B bf16, both K-major, M x N.
__host__ __device__ constexpr uint32_t instr_desc_bf16(int M, int N) {
    return (1u << 4)                      // D format F32
           | (1u << 7)                    // A format BF16
           | (1u << 10)                   // B format BF16
           | ((uint32_t)(N >> 3) << 17)   // N / 8
           | ((uint32_t)(M >> 4) << 24);  // M / 16
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
    asm volatile("{\n\t"
                 ".reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
                 "}\n" ::"r"(tmem_d),
                 "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0),
                 "r"(0));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Waits for phase `parity` of the mbarrier; gives up after `limit` polls and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
    const uint32_t a = smem_u32(bar);
    for (uint32_t i = 0; i < limit; i++) {
        uint32_t done;
        asm volatile("{\n\t"
                     ".reg .pred P1;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                     "selp.b32 %0, 1, 0, P1;\n\t"
                     "}"
                     : "=r"(done)
                     : "r"(a), "r"(parity)
                     : "memory");
        if (done)
            return true;
    }
    return false;
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(dst_smem)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

// 32 lanes x 16 columns of 32-bit TMEM values: this thread's row, columns col..col+15.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                   "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++)
        v[i] = __uint_as_float(r[i]);
}

// ---------------------------------------------------------------------------------------------
// TMA form. The operand tiles move by the tensor memory accelerator: one thread issues, per
// 64-wide K chunk, a cp.async.bulk.tensor copy of the 128 x 64 A box and of the BN x 64 B box
// into a ring slot, with the 128-byte swizzle, and the copies complete on the slot's "full"
// mbarrier (expect_tx). Roles by warp: warp 0 copies, warp 1 owns the TMEM accumulator and issues
// the MMAs (each chunk's tcgen05.commit arrives on the slot's "empty" mbarrier, which frees it
// for the next copy, and after the last chunk on "acc"), warps 2-9 run the epilogue (warp w reads
// TMEM lanes 32 (w % 4) .. +31, the rule of tcgen05.ld; the two warps of a lane quarter take one
// half of the columns each). Shared-memory layout of a slot: the A
// box then the B box, each rows x 128 B with 16-byte chunk j of row r at chunk j ^ (r % 8) (the
// TMA 128-byte swizzle), which is the canonical K-major SWIZZLE_128B layout of the tensor core:
// 8-row groups 1024 B apart (stride-byte offset), the K steps of 16 elements 32 B apart inside the
// swizzle atom (start address + 32 kk). Slots start on 1024-byte boundaries. Every wait is bounded;
// a timeout sets *err, stops the copy and MMA loops, and the copy thread waits (bounded) for its
// copies still in flight before the CTA ends.
// ---------------------------------------------------------------------------------------------
constexpr int kTmaEpiWarps = 8;                      // two per TMEM lane quarter
constexpr int kTmaThreads  = 64 + 32 * kTmaEpiWarps; // copy warp, MMA warp, epilogue warps

// Ring slots per tile width: 192 KB of shared memory, one CTA per SM. After the main loop the
// ring holds the fp32 output tile (128 x (BN + 4) floats, at most 130 KB).
template<int BN> struct TmaStages {
    static constexpr int value = BN >= 256 ? 4 : (BN >= 128 ? 6 : 8);
};
__host__ __device__ constexpr uint32_t tma_stage_bytes(int BN) { return (kM + BN) * kKChunk * 2; }
inline size_t gemm_tma_smem_bytes(int BN) {
    const int S = BN >= 256 ? 4 : (BN >= 128 ? 6 : 8);
    return (size_t)S * tma_stage_bytes(BN) + 1024; // + alignment of the ring to 1024 B
}

// Shared-memory matrix descriptor, K-major with the 128-byte swizzle: leading-byte offset unused
// (1), stride-byte offset 1024 (8 rows x 128 B), version 1, layout type SWIZZLE_128B (2).
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(1024 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// 2-D tensor copy of one box (x = K element index, y = row index) into shared memory, completing
// on bar. No multicast: the box goes to this CTA only.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar) {
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes "
                 "[%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
                 "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
                 : "memory");
}

// The fused epilogue of one epilogue warp: its 32 rows of the tile (TMEM lanes 32 q .. 32 q + 31).
// Phase 1: row per thread, 16 columns per tcgen05.ld, into a shared-memory tile of fp32 rows
// (pitch BN + 4 floats: the 8 threads of a 16-byte store phase hit distinct banks). Phase 2: the
// warp walks the same rows with its lanes across the columns, so every global access is a
// contiguous 16-byte vector per lane (bias, GELU and its derivative, the stores). Only the warp's
// own rows are touched, so __syncwarp orders the two phases.
template<int BN, int EPI>
__device__ __forceinline__ void epilogue_warp(uint32_t tmem_q, float* tile, int q, int half, int lane,
                                              int m0, int n0, const EpiArgs& e) {
    constexpr int kHalf = BN / 2;      // columns of this warp: [c0, c0 + kHalf)
    const int     c0    = half * kHalf;
    if constexpr (EPI == kEpiBiasF32T) { // lanes are consecutive rows: each column coalesced
        const int row = m0 + q * 32 + lane;
        for (int c = c0; c < c0 + kHalf; c += 16) {
            float v[16];
            tmem_ld16(tmem_q + c, v);
#pragma unroll
            for (int i = 0; i < 16; i++)
                e.out_f32[(size_t)(n0 + c + i) * e.ldo + row] = v[i] + e.bias[n0 + c + i];
        }
        return;
    }
    constexpr int kPitch = BN + 4;
    float*        rows   = tile + (size_t)q * 32 * kPitch;
    for (int c = c0; c < c0 + kHalf; c += 16) {
        float v[16];
        tmem_ld16(tmem_q + c, v);
        float4* d = reinterpret_cast<float4*>(rows + (size_t)lane * kPitch + c);
#pragma unroll
        for (int i = 0; i < 4; i++)
            d[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
    }
    __syncwarp();
    constexpr int kVec   = kHalf / 4;                  // float4 per row (this warp's half)
    constexpr int kRowsP = kVec >= 32 ? 1 : 32 / kVec; // rows per pass of the warp
    constexpr int kPerL  = kVec >= 32 ? kVec / 32 : 1; // float4 per lane per row
    const int     sub = kVec >= 32 ? 0 : lane / kVec, cl = kVec >= 32 ? lane : lane % kVec;
#pragma unroll 4
    for (int r0 = 0; r0 < 32; r0 += kRowsP) {
        const int    r   = r0 + sub;
        const size_t row = (size_t)(m0 + q * 32 + r);
#pragma unroll
        for (int j = 0; j < kPerL; j++) {
            const int col = c0 + (j * (kVec >= 32 ? 32 : kVec) + cl) * 4;
            float4    v   = *reinterpret_cast<const float4*>(rows + (size_t)r * kPitch + col);
            const size_t o = row * e.ldo + n0 + col;
            if constexpr (EPI == kEpiBiasF32 || EPI == kEpiBiasGelu) {
                const float4 bb = *reinterpret_cast<const float4*>(e.bias + n0 + col);
                v.x += bb.x, v.y += bb.y, v.z += bb.z, v.w += bb.w;
            }
            if constexpr (EPI == kEpiF32 || EPI == kEpiBiasF32) {
                *reinterpret_cast<float4*>(e.out_f32 + blockIdx.z * e.zstride + o) = v;
            }
            else {
                if constexpr (EPI == kEpiBiasGelu) {
                    float4 g, dg;
                    gelu_and_grad(v.x, g.x, dg.x);
                    gelu_and_grad(v.y, g.y, dg.y);
                    gelu_and_grad(v.z, g.z, dg.z);
                    gelu_and_grad(v.w, g.w, dg.w);
                    if (e.out_dg) { // gelu'(z) for the backward pass, when training
                        __nv_bfloat162 l2 = __floats2bfloat162_rn(dg.x, dg.y),
                                       h2 = __floats2bfloat162_rn(dg.z, dg.w);
                        *reinterpret_cast<uint2*>(e.out_dg + o) = make_uint2(
                            *reinterpret_cast<uint32_t*>(&l2), *reinterpret_cast<uint32_t*>(&h2));
                    }
                    v = g;
                }
                else if constexpr (EPI == kEpiGeluBwdBf16) {
                    const uint2          u   = *reinterpret_cast<const uint2*>(e.dg_in + o);
                    const __nv_bfloat162 l2 = *reinterpret_cast<const __nv_bfloat162*>(&u.x),
                                         h2 = *reinterpret_cast<const __nv_bfloat162*>(&u.y);
                    const float2 a = __bfloat1622float2(l2), b = __bfloat1622float2(h2);
                    v = make_float4(v.x * a.x, v.y * a.y, v.z * b.x, v.w * b.y);
                }
                __nv_bfloat162 lo = __floats2bfloat162_rn(v.x, v.y), hi = __floats2bfloat162_rn(v.z, v.w);
                *reinterpret_cast<uint2*>(e.out_bf16 + o) =
                    make_uint2(*reinterpret_cast<uint32_t*>(&lo), *reinterpret_cast<uint32_t*>(&hi));
            }
        }
    }
}

template<int BN, int EPI>
__global__ void __launch_bounds__(kTmaThreads)
    gemm_tma_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                    int K, EpiArgs e, unsigned int* err) {
    static_assert(BN % 32 == 0 && BN >= 32 && BN <= 256, "N in 32..256, halves of 16-column chunks");
    static_assert(kTmaEpiWarps == 8, "two epilogue warps per TMEM lane quarter");
    constexpr int      S         = TmaStages<BN>::value;
    constexpr uint32_t kABytes   = kM * kKChunk * 2;
    constexpr uint32_t kStage    = tma_stage_bytes(BN);
    constexpr uint32_t kTmemCols = BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));
    constexpr uint32_t kLimit    = 1u << 22;
    extern __shared__ uint8_t smem_raw[];
    __shared__ uint64_t       full[S], empty[S], acc;
    __shared__ uint32_t       tmem_base;
    __shared__ volatile int   abort_flag;
    const uint32_t            ring = (smem_u32(smem_raw) + 1023u) & ~1023u;
    const int                 warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int                 m0 = blockIdx.x * kM, n0 = blockIdx.y * BN;
    const int                 kz = K / gridDim.z, k0 = blockIdx.z * kz, nk = kz / kKChunk;

    if (warp == 1)
        tmem_alloc(&tmem_base, kTmemCols);
    if (threadIdx.x == 0) {
        for (int b = 0; b < S; b++) {
            mbar_init(&full[b], 1);
            mbar_init(&empty[b], 1);
        }
        mbar_init(&acc, 1);
        abort_flag = 0;
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = tmem_base;

    if (warp == 0) {
        if (lane == 0) { // copies: chunk kc into slot kc % S once the MMAs of chunk kc - S are done
            int issued = 0;
            for (int kc = 0; kc < nk && !abort_flag; kc++) {
                const int b = kc % S;
                if (kc >= S && !mbar_wait(&empty[b], (uint32_t)(((kc / S) & 1) ^ 1), kLimit)) {
                    atomicOr(err, 1u);
                    abort_flag = 1;
                    break;
                }
                const uint32_t a = ring + b * kStage;
                mbar_expect_tx(&full[b], kStage);
                tma_load_2d(a, &tmA, k0 + kc * kKChunk, m0, &full[b]);
                tma_load_2d(a + kABytes, &tmB, k0 + kc * kKChunk, n0, &full[b]);
                issued = kc + 1;
            }
            // every copy this thread started has landed before the CTA ends
            for (int c = issued > S ? issued - S : 0; c < issued; c++)
                mbar_wait(&full[c % S], (uint32_t)((c / S) & 1), kLimit);
        }
    }
    else if (warp == 1) {
        if (lane == 0) { // MMAs: four K = 16 steps per chunk into the TMEM accumulator
            constexpr uint32_t idesc = instr_desc_bf16(kM, BN);
            for (int kc = 0; kc < nk && !abort_flag; kc++) {
                const int b = kc % S;
                if (!mbar_wait(&full[b], (uint32_t)((kc / S) & 1), kLimit)) {
                    atomicOr(err, 1u);
                    abort_flag = 1;
                    break;
                }
                fence_after_sync();
                const uint32_t a = ring + b * kStage, bb = a + kABytes;
#pragma unroll
                for (int kk = 0; kk < kKChunk / 16; kk++)
                    mma_bf16(tmem, smem_desc_sw128(a + kk * 32), smem_desc_sw128(bb + kk * 32), idesc,
                             (kc | kk) != 0);
                mma_commit(&empty[b]);
            }
            mma_commit(&acc); // arrives once every MMA issued above has completed
        }
    }
    else { // epilogue warps 2 .. 2 + kTmaEpiWarps - 1
        const bool done = mbar_wait(&acc, 0u, kLimit);
        if (!done) {
            if (lane == 0)
                atomicOr(err, 1u);
        }
        else if (!abort_flag) {
            // every MMA is complete, so the ring (read by the MMAs, filled by copies they waited
            // for) is free to hold the output tile
            fence_after_sync();
            const int q = warp & 3, half = (warp - 2) >> 2;
            epilogue_warp<BN, EPI>(tmem + ((uint32_t)(q * 32) << 16),
                                   reinterpret_cast<float*>(smem_raw + (ring - smem_u32(smem_raw))),
                                   q, half, lane, m0, n0, e);
        }
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 1)
        tmem_dealloc(tmem, kTmemCols);
}

// Tensor map of a row-major [rows x K] bf16 matrix, boxes of 64 x box_rows, 128-byte swizzle.
// Returns false if the driver rejects it (alignment, sizes).
inline bool make_kmajor_map(CUtensorMap* map, const void* ptr, int rows, int K, int box_rows) {
    static PFN_cuTensorMapEncodeTiled encode = nullptr;
    if (!encode) {
        void*                           fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q)
                != cudaSuccess
            || q != cudaDriverEntryPointSuccess || !fn)
            return false;
        encode = (PFN_cuTensorMapEncodeTiled)fn;
    }
    const cuuint64_t dims[2]    = {(cuuint64_t)K, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)K * 2};
    const cuuint32_t box[2]     = {(cuuint32_t)kKChunk, (cuuint32_t)box_rows};
    const cuuint32_t estr[2]    = {1, 1};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides,
                  box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE)
           == CUDA_SUCCESS;
}

// D = A . B^T through the TMA kernel; same contract as gemm(). A tensor map the driver rejects
// sets *err (the caller's error check reports it) and launches nothing.
template<int BN, int EPI>
inline void gemm_tma(const __nv_bfloat16* A, const __nv_bfloat16* B, int M, int N, int K,
                     const EpiArgs& e, unsigned int* err, cudaStream_t st, int splits = 1) {
    // the attribute is per device; recorded only once the driver accepted it, under a lock (host
    // threads may launch concurrently); a refusal sets *err and launches nothing
    static std::mutex mu;
    static bool       configured[64] = {};
    {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess)
            dev = -1;
        std::lock_guard<std::mutex> lock(mu);
        if (dev < 0 || dev >= 64 || !configured[dev]) {
            if (cudaFuncSetAttribute(gemm_tma_kernel<BN, EPI>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)gemm_tma_smem_bytes(BN))
                != cudaSuccess) {
                cudaMemsetAsync(err, 0xFF, sizeof(unsigned int), st);
                return;
            }
            if (dev >= 0 && dev < 64)
                configured[dev] = true;
        }
    }
    CUtensorMap ma, mb;
    if (!make_kmajor_map(&ma, A, M, K, kM) || !make_kmajor_map(&mb, B, N, K, BN)) {
        cudaMemsetAsync(err, 0xFF, sizeof(unsigned int), st);
        return;
    }
    dim3 grid(M / kM, N / BN, splits);
    gemm_tma_kernel<BN, EPI><<<grid, kTmaThreads, gemm_tma_smem_bytes(BN), st>>>(ma, mb, K, e, err);
}

} // namespace umma
} // namespace thorx
