// mlp.cu -- dense layers of the brick-mode selector on the 5th-generation tensor cores.
//
// One GEMM form serves the forward and the backward pass:
//     C[M][N] = epilogue(A[M][K] . B[N][K]^T)
// with A and B bf16, row-major with K contiguous ("K-major"), fp32 accumulation
// in tensor memory, and an epilogue that adds a bias, applies ReLU or the ReLU
// gradient mask, and writes fp32 and/or bf16, plain or transposed.
//
// Per CTA: one 128 x N tile (N <= 256, a multiple of 16), 128 threads.  K runs
// in chunks of 64: the four warps copy the A and B chunks into shared memory in
// the canonical no-swizzle K-major layout (8-row x 16-byte core matrices; core
// matrix (row group g, column group c) at (g * 8 + c) * 128 bytes, so the
// K-adjacent core matrices are 128 bytes apart and the row-adjacent ones 1024),
// one thread issues four tcgen05.mma (M=128, N, K=16) with the accumulator in
// tensor memory and commits them to an mbarrier, and all threads wait for it
// (bounded) before the next chunk.  The epilogue reads the accumulator with
// tcgen05.ld (warp w owns lanes 32w..32w+31 = rows) and applies the fused ops.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "csv_internal.h"

namespace csv {
namespace {

constexpr uint32_t kGemmThreads = 128;
constexpr uint32_t kKChunk = 64;               // bf16 elements per row per chunk (128 bytes)
constexpr uint32_t kTileA = 128 * kKChunk * 2; // 16 KB
constexpr uint32_t kTileBMax = 256 * kKChunk * 2;  // 32 KB
constexpr uint32_t kWaitLimit = 1u << 24;

struct GemmArgs {
    const __nv_bfloat16* A;
    const __nv_bfloat16* B;
    uint32_t M, N, K;
    const float* bias;            // [N] or null
    const __nv_bfloat16* mask;    // [M][N] or null: multiply by (mask > 0), the ReLU gradient
    uint32_t relu;                // max(0, .) after the bias
    float* C;                     // [M][N] or null
    __nv_bfloat16* Cb;            // [M][N] or null
    __nv_bfloat16* CbT;           // [N][M] or null
    float* CT;                    // [N][M] or null
    uint32_t* err;                // set to 1 when a wait gives up
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    // start address, leading byte offset (K-adjacent core matrices), stride byte
    // offset (row-adjacent core matrices), descriptor version 1, no swizzle
    const uint64_t lbo = 128, sbo = 1024;
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((lbo >> 4) << 16) | ((sbo >> 4) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (uint32_t it = 0; it < kWaitLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__global__ void __launch_bounds__(kGemmThreads) gemm_bf16_kernel(GemmArgs G) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* sA = smem;                  // 16 KB
    uint8_t* sB = smem + kTileA;         // up to 32 KB
    __shared__ uint64_t bar;
    __shared__ uint32_t tmem_base;
    __shared__ uint32_t failed;
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    const uint32_t m0 = blockIdx.x * 128u, n0 = blockIdx.y * 256u;
    const uint32_t N = min(256u, G.N - n0);
    uint32_t ncols = 32;
    while (ncols < N) ncols <<= 1;
    if (tid == 0) {
        mbar_init(smem_u32(&bar), 1);
        failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;
    // M = 128, N, bf16 x bf16 -> f32, both operands K-major
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((128u >> 4) << 24);
    const uint32_t nchunks = G.K / kKChunk;
    uint32_t parity = 0;
    for (uint32_t c = 0; c < nchunks; ++c) {
        const uint32_t k0 = c * kKChunk;
        // A: 128 rows x 8 units of 16 bytes
        for (uint32_t u = tid; u < 128u * 8u; u += kGemmThreads) {
            const uint32_t r = u >> 3, kb = u & 7u;
            const uint4 v = *reinterpret_cast<const uint4*>(G.A + (size_t)(m0 + r) * G.K + k0 + kb * 8);
            *reinterpret_cast<uint4*>(sA + ((r >> 3) * 8 + kb) * 128 + (r & 7u) * 16) = v;
        }
        for (uint32_t u = tid; u < N * 8u; u += kGemmThreads) {
            const uint32_t r = u >> 3, kb = u & 7u;
            const uint4 v = *reinterpret_cast<const uint4*>(G.B + (size_t)(n0 + r) * G.K + k0 + kb * 8);
            *reinterpret_cast<uint4*>(sB + ((r >> 3) * 8 + kb) * 128 + (r & 7u) * 16) = v;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0 && !failed) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (uint32_t s = 0; s < kKChunk / 16; ++s) {
                const uint64_t ad = smem_desc(smem_u32(sA) + s * 256u);
                const uint64_t bd = smem_desc(smem_u32(sB) + s * 256u);
                const uint32_t acc = (c > 0 || s > 0) ? 1u : 0u;
                asm volatile(
                    "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                    " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                    "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&bar))
                         : "memory");
        }
        if (!failed) {
            if (!mbar_wait(smem_u32(&bar), parity)) {
                failed = 1;
                if (G.err) atomicExch(G.err, 1u);
            }
        }
        parity ^= 1u;
        __syncthreads();  // the chunk's shared memory is free again
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!failed) {
        const uint32_t row = m0 + warp * 32u + lane;
        for (uint32_t j0 = 0; j0 < N; j0 += 16) {
            uint32_t v[16];
            const uint32_t taddr = tmem + ((warp * 32u) << 16) + j0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                "[%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                  "=r"(v[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < G.M) {
#pragma unroll
                for (uint32_t j = 0; j < 16; ++j) {
                    const uint32_t n = n0 + j0 + j;
                    float x = __uint_as_float(v[j]);
                    if (G.bias) x += G.bias[n];
                    if (G.relu) x = fmaxf(x, 0.0f);
                    if (G.mask && !(__bfloat162float(G.mask[(size_t)row * G.N + n]) > 0.0f)) x = 0.0f;
                    if (G.C) G.C[(size_t)row * G.N + n] = x;
                    if (G.Cb) G.Cb[(size_t)row * G.N + n] = __float2bfloat16_rn(x);
                    if (G.CbT) G.CbT[(size_t)n * G.M + row] = __float2bfloat16_rn(x);
                    if (G.CT) G.CT[(size_t)n * G.M + row] = x;
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
}

}  // namespace

size_t gemm_smem_bytes() { return kTileA + kTileBMax; }

cudaError_t launch_gemm_bf16(const __nv_bfloat16* A, const __nv_bfloat16* B, uint32_t M, uint32_t N, uint32_t K,
                             const float* bias, const __nv_bfloat16* mask, uint32_t relu, float* C,
                             __nv_bfloat16* Cb, __nv_bfloat16* CbT, float* CT, uint32_t* err, cudaStream_t st) {
    if (M == 0 || N == 0 || K == 0) return cudaSuccess;
    if (M % 128 || N % 16 || K % kKChunk) return cudaErrorInvalidValue;
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(gemm_bf16_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)gemm_smem_bytes());
        if (e != cudaSuccess) return e;
        attr = true;
    }
    GemmArgs G;
    G.A = A;
    G.B = B;
    G.M = M;
    G.N = N;
    G.K = K;
    G.bias = bias;
    G.mask = mask;
    G.relu = relu;
    G.C = C;
    G.Cb = Cb;
    G.CbT = CbT;
    G.CT = CT;
    G.err = err;
    dim3 grid(M / 128, (N + 255) / 256);
    gemm_bf16_kernel<<<grid, kGemmThreads, gemm_smem_bytes(), st>>>(G);
    return cudaGetLastError();
}

}  // namespace csv

// ---------------------------------------------------------------- C ABI
#include "abi_internal.h"

extern "C" int csv_gemm_bf16(csv_ctx* ctx, const void* d_A, const void* d_B, uint32_t M, uint32_t N, uint32_t K,
                             const float* d_bias, const void* d_mask, uint32_t relu, float* d_C, void* d_Cb,
                             void* d_CbT, float* d_CT, uint32_t* d_err, void* stream) {
    using namespace csv;
    if (!ctx || !d_A || !d_B) return CSV_EINVAL;
    if (M % 128 || N % 16 || K % 64) return abi_fail(ctx, CSV_EINVAL, "gemm: M % 128, N % 16 and K % 64 must be 0");
    DeviceGuard g(ctx->device);
    cudaError_t e = launch_gemm_bf16((const __nv_bfloat16*)d_A, (const __nv_bfloat16*)d_B, M, N, K, d_bias,
                                     (const __nv_bfloat16*)d_mask, relu, d_C, (__nv_bfloat16*)d_Cb,
                                     (__nv_bfloat16*)d_CbT, d_CT, d_err, (cudaStream_t)stream);
    if (e != cudaSuccess) return abi_cuda_fail(ctx, e, "gemm");
    return CSV_OK;
}
