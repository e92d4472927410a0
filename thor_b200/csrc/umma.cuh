// BF16 tensor-core GEMM on the 5th-generation tensor cores (tcgen05) of sm_100a.
//
//   D[M x N] = A[M x K] . B[N x K]^T      A, B bf16, row-major (K contiguous, "K-major"),
//                                         FP32 accumulation in tensor memory (TMEM)
//
// One CTA of 128 threads computes a 128 x BN tile of D. K is consumed in 64-wide chunks through
// a ring of 3-4 shared-memory slots: the four warps copy the A and B tiles of a chunk from global
// memory with 16-byte cp.async into the canonical no-swizzle K-major layout of the tensor core
// (8-row x 16-byte core matrices: element (r, k) at byte (r/8)*1024 + (k/8)*128 + (r%8)*16 +
// (k%8)*2, i.e. leading-byte offset 128 between the core matrices along K and stride-byte offset
// 1024 between 8-row groups), one thread issues four tcgen05.mma (K = 16 each) into the TMEM
// accumulator and commits them to the slot's mbarrier; a slot is refilled (S-1 chunks ahead)
// once the bounded wait on that mbarrier shows its MMAs done, so copies overlap the MMAs. The
// epilogue reads the accumulator back with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 = rows
// 32w.. of the tile) and applies a fused element-wise operation before storing.
//
// Descriptor formats (shared-memory matrix descriptor, instruction descriptor for kind::f16)
// follow the PTX ISA for tcgen05; field positions as in CUTLASS's cute/arch/mma_sm100_desc.hpp.
// Requirements on the caller: M a multiple of 128, N a multiple of BN, K a multiple of 64, all
// row starts 16-byte aligned (K a multiple of 8).
#pragma once

#include <cstdint>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace thorx {
namespace umma {

constexpr int kM       = 128; // rows of a CTA tile (tensor-core M)
constexpr int kKChunk  = 64;  // K elements staged per round
constexpr int kThreads = 128;

// Epilogues. Z is the FP32 pre-activation of a layer, bias per output column.
enum Epi : int {
    kEpiF32         = 0, // out_f32[m][n] = acc
    kEpiBiasF32     = 1, // out_f32[m][n] = acc + bias[n]
    kEpiBiasGelu    = 2, // z = acc + bias[n]; out_z[m][n] = z; out_bf16[m][n] = gelu(z)
    kEpiGeluBwdBf16 = 3, // out_bf16[m][n] = acc * gelu'(z_in[m][n])
    kEpiBf16        = 4, // out_bf16[m][n] = acc
};

struct EpiArgs {
    float*         out_f32;
    __nv_bfloat16* out_bf16;
    float*         out_z;
    const float*   z_in;
    const float*   bias;
    int            ldo;     // leading dimension of the outputs (elements)
    size_t         zstride; // split-K: elements between the partial outputs of consecutive splits
};

__device__ __forceinline__ float gelu(float z) {
    return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f));
}
__device__ __forceinline__ float gelu_grad(float z) {
    const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * __expf(-0.5f * z * z);
    return cdf + z * pdf;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor, no swizzle, version 1 (tcgen05).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46; // descriptor version for tcgen05
    return d;               // base offset 0, legacy LBO mode, layout SWIZZLE_NONE (0)
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

// Starts the copy of a rows x 64 bf16 block (row stride ld elements) into the canonical K-major
// layout with 16-byte cp.async (no register staging); completion via cp.async.wait_group.
__device__ __forceinline__ void stage_kmajor_async(uint8_t* dst, const __nv_bfloat16* __restrict__ src,
                                                   int rows, int ld) {
    for (int v = threadIdx.x; v < rows * 8; v += kThreads) {
        const int r = v >> 3, kv = v & 7;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                         smem_u32(dst + (r >> 3) * 1024 + kv * 128 + (r & 7) * 16)),
                     "l"(src + (size_t)r * ld + kv * 8)
                     : "memory");
    }
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template<int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Stages of the shared-memory ring: the largest tile keeps 3 (144 KB, one CTA per SM), the
// others 4 (two CTAs per SM).
template<int BN> struct Stages {
    static constexpr int value = BN >= 256 ? 3 : 4;
};

template<int BN, int EPI>
__global__ void __launch_bounds__(kThreads)
    gemm_kernel(const __nv_bfloat16* __restrict__ A, const __nv_bfloat16* __restrict__ B, int K,
                EpiArgs e, unsigned int* err) {
    static_assert(BN % 16 == 0 && BN >= 32 && BN <= 256, "tcgen05 M=128 needs N in 16..256");
    constexpr int      S         = Stages<BN>::value;
    constexpr int      kStage    = (kM + BN) * kKChunk * 2; // bytes per ring slot
    constexpr uint32_t kTmemCols = BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t bar[S];
    __shared__ uint32_t tmem_base;
    const int           warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int           m0 = blockIdx.x * kM, n0 = blockIdx.y * BN;
    const int           kz = K / gridDim.z;          // split-K: this CTA's share of K
    const int           k0 = blockIdx.z * kz;
    const int           nk = kz / kKChunk;
    auto                sA = [&](int b) { return smem + b * kStage; };
    auto                sB = [&](int b) { return smem + b * kStage + kM * kKChunk * 2; };
    auto                load = [&](int kc) {
        stage_kmajor_async(sA(kc % S), A + (size_t)m0 * K + k0 + kc * kKChunk, kM, K);
        stage_kmajor_async(sB(kc % S), B + (size_t)n0 * K + k0 + kc * kKChunk, BN, K);
    };

    if (warp == 0)
        tmem_alloc(&tmem_base, kTmemCols);
    if (threadIdx.x == 32)
        for (int b = 0; b < S; b++)
            mbar_init(&bar[b], 1);
    for (int st = 0; st < S - 1; st++) { // prologue: the first S-1 chunks in flight
        if (st < nk)
            load(st);
        cp_async_commit();
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t     tmem  = tmem_base;
    constexpr uint32_t idesc = instr_desc_bf16(kM, BN);
    bool               ok    = true;
    // chunk c's MMAs complete phase (c / S) of bar[c % S]; every completion is waited in order
    auto mma_done = [&](int c) { return mbar_wait(&bar[c % S], (uint32_t)((c / S) & 1), 1u << 22); };
    for (int kc = 0; kc < nk && ok; kc++) {
        cp_async_wait<S - 2>(); // this thread's part of chunk kc has landed
        fence_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) {
            fence_after_sync();
            const uint32_t a0 = smem_u32(sA(kc % S)), b0 = smem_u32(sB(kc % S));
#pragma unroll
            for (int kk = 0; kk < kKChunk / 16; kk++)
                mma_bf16(tmem, smem_desc(a0 + kk * 256, 128, 1024), smem_desc(b0 + kk * 256, 128, 1024),
                         idesc, (kc | kk) != 0);
            mma_commit(&bar[kc % S]);
        }
        const int next = kc + S - 1; // refills the slot of chunk kc - 1 once its MMAs are done
        if (next < nk) {
            if (kc >= 1)
                ok = __syncthreads_and(mma_done(kc - 1)) != 0;
            if (ok)
                load(next);
        }
        cp_async_commit();
    }
    if (ok) // MMAs complete in order: the last chunk's completion covers them all
        ok = __syncthreads_and(mma_done(nk - 1)) != 0;
    cp_async_wait<0>();
    if (!ok) {
        if (threadIdx.x == 0)
            atomicOr(err, 1u);
    }
    else {
        fence_after_sync();
        const int row = m0 + warp * 32 + lane;
        for (int c = 0; c < BN; c += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + c, v);
            // this thread's 16 consecutive outputs of its row, written as 16-byte vectors
            const size_t o = (size_t)row * e.ldo + n0 + c;
            if constexpr (EPI == kEpiBiasF32 || EPI == kEpiBiasGelu) {
#pragma unroll
                for (int i = 0; i < 16; i++)
                    v[i] += e.bias[n0 + c + i];
            }
            if constexpr (EPI == kEpiF32 || EPI == kEpiBiasF32) {
                float4* d = reinterpret_cast<float4*>(e.out_f32 + blockIdx.z * e.zstride + o);
#pragma unroll
                for (int q = 0; q < 4; q++)
                    d[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            }
            else {
                if constexpr (EPI == kEpiBiasGelu) {
                    float4* dz = reinterpret_cast<float4*>(e.out_z + o);
#pragma unroll
                    for (int q = 0; q < 4; q++)
                        dz[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
#pragma unroll
                    for (int i = 0; i < 16; i++)
                        v[i] = gelu(v[i]);
                }
                else if constexpr (EPI == kEpiGeluBwdBf16) {
                    const float4* zi = reinterpret_cast<const float4*>(e.z_in + o);
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const float4 z = zi[q];
                        v[4 * q] *= gelu_grad(z.x);
                        v[4 * q + 1] *= gelu_grad(z.y);
                        v[4 * q + 2] *= gelu_grad(z.z);
                        v[4 * q + 3] *= gelu_grad(z.w);
                    }
                }
                uint32_t pk[8];
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    __nv_bfloat162 h2 = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
                    pk[q]             = *reinterpret_cast<uint32_t*>(&h2);
                }
                uint4* d = reinterpret_cast<uint4*>(e.out_bf16 + o);
                d[0]     = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                d[1]     = make_uint4(pk[4], pk[5], pk[6], pk[7]);
            }
        }
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0)
        tmem_dealloc(tmem, kTmemCols);
}

inline size_t gemm_smem_bytes(int BN) {
    return (size_t)(BN >= 256 ? 3 : 4) * (kM + BN) * kKChunk * 2;
}

// D = A . B^T for A [M x K], B [N x K] (bf16, K contiguous) with the given epilogue.
// splits > 1 (kEpiF32 only): K is cut into `splits` equal parts, each written as a partial
// product at out_f32 + z * zstride for the caller to reduce.
template<int BN, int EPI>
inline void gemm(const __nv_bfloat16* A, const __nv_bfloat16* B, int M, int N, int K,
                 const EpiArgs& e, unsigned int* err, cudaStream_t st, int splits = 1) {
    static bool configured = false; // dynamic shared memory above the 48 KB default
    if (!configured) {
        cudaFuncSetAttribute(gemm_kernel<BN, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)gemm_smem_bytes(BN));
        configured = true;
    }
    dim3 grid(M / kM, N / BN, splits);
    gemm_kernel<BN, EPI><<<grid, kThreads, gemm_smem_bytes(BN), st>>>(A, B, K, e, err);
}

} // namespace umma
} // namespace thorx
