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

#include <algorithm>

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

// ------------------------------------------------------------ fused inference
// The selector's whole forward pass for 128 rows at a time, persistent (one CTA
// per SM, all 512 tensor-memory columns), activations never leaving the SM:
//   X (bf16, features padded to 64) -> acc1 = X W1^T (TMEM cols 0..255)
//   H1 = bf16(relu(acc1 + b1))      -> shared memory, the next A operand
//   acc2 = H1 W2^T (TMEM cols 256..511), W2 streamed from L2 in four 32 KB
//   K-chunks through a two-slot ring of bulk copies (it does not fit beside
//   the rest), H2 = bf16(relu(acc2 + b2)) -> shared memory
//   acc3 = H2 W3^T (TMEM cols 0..31), logits = acc3 + b3, argmax per head.
// The MMAs are the ones the layer-by-layer GEMMs issue (same shapes, same K
// order), so the logits are those of gemm_bf16_kernel's three launches.
// Weights come pre-tiled in the no-swizzle K-major core-matrix layout, so that
// each K-chunk is one contiguous bulk copy (tile_b_kernel).
constexpr uint32_t kInferThreads = 128;
constexpr uint32_t kHidN = 256, kInN = 64, kOutN = 32;
constexpr uint32_t kSelModes = 12, kSelTables = 16;  // the two heads: logits 0..11 and 12..27
constexpr uint32_t kChunkW2 = kHidN * kKChunk * 2;   // 32 KB
constexpr uint32_t kChunkW3 = kOutN * kKChunk * 2;   // 4 KB
constexpr uint32_t kChunkH = 128 * kKChunk * 2;      // 16 KB
constexpr uint32_t kOffW1 = 0;                       // 32 KB
constexpr uint32_t kOffW3 = kOffW1 + kHidN * kInN * 2;  // 16 KB (4 chunks)
constexpr uint32_t kOffH = kOffW3 + 4 * kChunkW3;       // 64 KB (4 chunks); chunk 0 holds X first
constexpr uint32_t kOffRing = kOffH + 4 * kChunkH;      // 2 x 32 KB
constexpr uint32_t kOffBias = kOffRing + 2 * kChunkW2;  // b1, b2, b3 (fp32)
constexpr uint32_t kInferSmem = kOffBias + (2 * kHidN + kOutN) * 4;

struct InferArgs {
    const float* feat;          // [count][32]
    uint32_t count;
    const __nv_bfloat16* W1t;   // tiled [256][64]
    const __nv_bfloat16* W2t;   // tiled [256][256]: four 32 KB chunks
    const __nv_bfloat16* W3t;   // tiled [32][256]: four 4 KB chunks
    const float *b1, *b2, *b3;
    float* logits;              // [count][32] or null
    uint8_t* sel;               // [count] or null: argmax(0..11) | argmax(12..27) << 4
    uint32_t* err;
};

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
        "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t v[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
          "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// (row r, K element k) of a 128-row A operand held as 64-wide K-chunks of core matrices
__device__ __forceinline__ uint32_t a_off(uint32_t r, uint32_t k) {
    return (k >> 6) * kChunkH + (((r >> 3) * 8 + ((k & 63) >> 3)) * 128) + (r & 7) * 16 + (k & 7) * 2;
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    const uint32_t lo = __bfloat16_as_ushort(__float2bfloat16_rn(a));
    const uint32_t hi = __bfloat16_as_ushort(__float2bfloat16_rn(b));
    return lo | (hi << 16);
}

// acc (TMEM, this warp's 32 rows, 256 columns from col0) + bias, ReLU, bf16 -> the A operand in shared memory
__device__ __forceinline__ void epilogue_hidden(uint32_t tmem_row, const float* bias, uint8_t* sH, uint32_t r) {
    for (uint32_t j0 = 0; j0 < kHidN; j0 += 16) {
        uint32_t v[16];
        tmem_ld16(tmem_row + j0, v);
        uint32_t w[8];
#pragma unroll
        for (uint32_t j = 0; j < 8; ++j) {
            const float a = fmaxf(__uint_as_float(v[2 * j]) + bias[j0 + 2 * j], 0.0f);
            const float b = fmaxf(__uint_as_float(v[2 * j + 1]) + bias[j0 + 2 * j + 1], 0.0f);
            w[j] = pack_bf16(a, b);
        }
        *reinterpret_cast<uint4*>(sH + a_off(r, j0)) = make_uint4(w[0], w[1], w[2], w[3]);
        *reinterpret_cast<uint4*>(sH + a_off(r, j0 + 8)) = make_uint4(w[4], w[5], w[6], w[7]);
    }
}

__global__ void __launch_bounds__(kInferThreads, 1) mlp_infer_kernel(InferArgs G) {
    extern __shared__ __align__(1024) uint8_t smem[];
    // barriers: 0 weights (W1, W3), 1..2 ring slot full, 3..4 ring slot free, 5 MMA done
    __shared__ __align__(8) uint64_t bars[6];
    __shared__ uint32_t tmem_base;
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    const uint32_t sbase = smem_u32(smem);
    const uint32_t b_w = smem_u32(&bars[0]), b_mma = smem_u32(&bars[5]);
    auto b_full = [&](uint32_t s) { return smem_u32(&bars[1 + s]); };
    auto b_free = [&](uint32_t s) { return smem_u32(&bars[3 + s]); };
    float* sb1 = reinterpret_cast<float*>(smem + kOffBias);
    float* sb2 = sb1 + kHidN;
    float* sb3 = sb2 + kHidN;
    for (uint32_t i = tid; i < kHidN; i += kInferThreads) {
        sb1[i] = G.b1[i];
        sb2[i] = G.b2[i];
    }
    if (tid < kOutN) sb3[tid] = G.b3[tid];
    if (tid == 0) {
        for (uint32_t i = 0; i < 6; ++i) mbar_init(smem_u32(&bars[i]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(512u)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;
    if (tid == 0) {
        // resident weights, and W2 chunks 0 and 1 into the ring
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b_w),
                     "r"(kHidN * kInN * 2 + 4 * kChunkW3)
                     : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                         sbase + kOffW1),
                     "l"(G.W1t), "r"(kHidN * kInN * 2), "r"(b_w)
                     : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                         sbase + kOffW3),
                     "l"(G.W3t), "r"(4 * kChunkW3), "r"(b_w)
                     : "memory");
        bulk_g2s(sbase + kOffRing, G.W2t, kChunkW2, b_full(0));
        bulk_g2s(sbase + kOffRing + kChunkW2, reinterpret_cast<const uint8_t*>(G.W2t) + kChunkW2, kChunkW2, b_full(1));
    }
    const uint32_t idesc256 = (1u << 4) | (1u << 7) | (1u << 10) | ((kHidN >> 3) << 17) | ((128u >> 4) << 24);
    const uint32_t idesc32 = (1u << 4) | (1u << 7) | (1u << 10) | ((kOutN >> 3) << 17) | ((128u >> 4) << 24);
    uint32_t ph_mma = 0, ph_full[2] = {0, 0}, ph_free[2] = {0, 0};
    bool pending[2] = {true, true};  // (thread 0) a bulk copy into the ring slot has not been waited for
    // every exit decision is taken by the whole block (__syncthreads_and), so that
    // no thread leaves a loop that the others stay in
    bool ok = __syncthreads_and(mbar_wait(b_w, 0));
    const uint32_t n_tiles = (G.count + 127) / 128;
    uint8_t* sH = smem + kOffH;
    const uint32_t tmem_row = tmem + ((warp * 32u) << 16);
    for (uint32_t t = blockIdx.x; t < n_tiles && ok; t += gridDim.x) {
        const uint32_t r = warp * 32u + lane, row = t * 128u + r;
        // ---- X: the row's 32 features as bf16, K padded to 64 with zeros (chunk 0 of sH)
        {
            float f[32];
            if (row < G.count) {
                const float4* src = reinterpret_cast<const float4*>(G.feat + (size_t)row * 32);
#pragma unroll
                for (uint32_t q = 0; q < 8; ++q) {
                    const float4 x = src[q];
                    f[4 * q] = x.x; f[4 * q + 1] = x.y; f[4 * q + 2] = x.z; f[4 * q + 3] = x.w;
                }
            } else {
#pragma unroll
                for (uint32_t q = 0; q < 32; ++q) f[q] = 0.0f;
            }
#pragma unroll
            for (uint32_t c = 0; c < 4; ++c)
                *reinterpret_cast<uint4*>(sH + a_off(r, 8 * c)) =
                    make_uint4(pack_bf16(f[8 * c], f[8 * c + 1]), pack_bf16(f[8 * c + 2], f[8 * c + 3]),
                               pack_bf16(f[8 * c + 4], f[8 * c + 5]), pack_bf16(f[8 * c + 6], f[8 * c + 7]));
#pragma unroll
            for (uint32_t c = 4; c < 8; ++c) *reinterpret_cast<uint4*>(sH + a_off(r, 8 * c)) = make_uint4(0, 0, 0, 0);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        // ---- layer 1
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (uint32_t s = 0; s < 4; ++s)
                mma_bf16(tmem, smem_desc(sbase + kOffH + s * 256u), smem_desc(sbase + kOffW1 + s * 256u), idesc256,
                         s > 0);
            mma_commit(b_mma);
        }
        bool w = mbar_wait(b_mma, ph_mma);
        ph_mma ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (w) epilogue_hidden(tmem_row, sb1, sH, r);
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        if (!(ok = __syncthreads_and(w))) break;
        // ---- layer 2: K-chunk q of H1 against W2 chunk q from ring slot q % 2; each
        // slot refills (chunk q + 2, or chunk q - 2 for the next tile) once its MMAs end
        w = true;
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            for (uint32_t q = 0; q < 4 && w; ++q) {
                const uint32_t sl = q & 1u;
                w = mbar_wait(b_full(sl), ph_full[sl]);
                ph_full[sl] ^= 1u;
                pending[sl] = false;
                if (!w) break;
                const uint32_t slot = sbase + kOffRing + sl * kChunkW2;
#pragma unroll
                for (uint32_t s = 0; s < 4; ++s)
                    mma_bf16(tmem + kHidN, smem_desc(sbase + kOffH + q * kChunkH + s * 256u), smem_desc(slot + s * 256u),
                             idesc256, (q > 0 || s > 0) ? 1u : 0u);
                mma_commit(b_free(sl));
                if (q == 3) mma_commit(b_mma);
                if (q >= 1) {
                    const uint32_t ps = (q - 1) & 1u, nq = (q + 1) & 3u;
                    w = mbar_wait(b_free(ps), ph_free[ps]);
                    ph_free[ps] ^= 1u;
                    if (w) {
                        bulk_g2s(sbase + kOffRing + ps * kChunkW2, reinterpret_cast<const uint8_t*>(G.W2t) + nq * kChunkW2,
                                 kChunkW2, b_full(ps));
                        pending[ps] = true;
                    }
                }
            }
            if (w) {  // the slot of chunk 3 refills with chunk 1 of the next tile
                w = mbar_wait(b_free(1), ph_free[1]);
                ph_free[1] ^= 1u;
                if (w) {
                    bulk_g2s(sbase + kOffRing + kChunkW2, reinterpret_cast<const uint8_t*>(G.W2t) + kChunkW2, kChunkW2,
                             b_full(1));
                    pending[1] = true;
                }
            }
        }
        if (!(ok = __syncthreads_and(w))) break;
        w = mbar_wait(b_mma, ph_mma);
        ph_mma ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (w) epilogue_hidden(tmem_row + kHidN, sb2, sH, r);
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        if (!(ok = __syncthreads_and(w))) break;
        // ---- layer 3
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            for (uint32_t q = 0; q < 4; ++q)
#pragma unroll
                for (uint32_t s = 0; s < 4; ++s)
                    mma_bf16(tmem, smem_desc(sbase + kOffH + q * kChunkH + s * 256u),
                             smem_desc(sbase + kOffW3 + q * kChunkW3 + s * 256u), idesc32, (q > 0 || s > 0) ? 1u : 0u);
            mma_commit(b_mma);
        }
        w = mbar_wait(b_mma, ph_mma);
        ph_mma ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (w) {
            uint32_t v[32];
            tmem_ld16(tmem_row, v);
            tmem_ld16(tmem_row + 16, v + 16);
            float z[32];
#pragma unroll
            for (uint32_t j = 0; j < 32; ++j) z[j] = __uint_as_float(v[j]) + sb3[j];
            if (row < G.count) {
                if (G.logits) {
                    float4* dst = reinterpret_cast<float4*>(G.logits + (size_t)row * 32);
#pragma unroll
                    for (uint32_t q = 0; q < 8; ++q) dst[q] = make_float4(z[4 * q], z[4 * q + 1], z[4 * q + 2], z[4 * q + 3]);
                }
                if (G.sel) {  // ties: the lower index
                    uint32_t bm = 0, bt = 0;
                    float zm = z[0], zt = z[kSelModes];
#pragma unroll
                    for (uint32_t k = 1; k < kSelModes; ++k)
                        if (z[k] > zm) { zm = z[k]; bm = k; }
#pragma unroll
                    for (uint32_t k = 1; k < kSelTables; ++k)
                        if (z[kSelModes + k] > zt) { zt = z[kSelModes + k]; bt = k; }
                    G.sel[row] = (uint8_t)(bm | (bt << 4));
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        ok = __syncthreads_and(w);  // sH is rewritten by the next tile
    }
    if (!ok && tid == 0 && G.err) atomicExch(G.err, 1u);
    // ring copies still in flight land before the CTA exits (bounded waits)
    if (tid == 0)
        for (uint32_t sl = 0; sl < 2; ++sl)
            if (pending[sl]) mbar_wait(b_full(sl), ph_full[sl]);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u) : "memory");
}

// B [N][K] row-major bf16 -> the tiled layout: K-chunks of 64, each N/8 x 8 core
// matrices of 8 rows x 16 bytes, core (g, c) at (g * 8 + c) * 128 bytes.
__global__ void tile_b_kernel(const __nv_bfloat16* __restrict__ B, uint32_t N, uint32_t K, __nv_bfloat16* __restrict__ T) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N * K) return;
    const uint32_t n = i / K, k = i % K;
    T[(size_t)(k >> 6) * N * 64 + ((n >> 3) * 8 + ((k & 63) >> 3)) * 64 + (n & 7) * 8 + (k & 7)] = B[i];
}

}  // namespace

size_t gemm_smem_bytes() { return kTileA + kTileBMax; }

cudaError_t launch_tile_b(const __nv_bfloat16* B, uint32_t N, uint32_t K, __nv_bfloat16* T, cudaStream_t st) {
    if (N % 8 || K % 64) return cudaErrorInvalidValue;
    tile_b_kernel<<<(N * K + 255) / 256, 256, 0, st>>>(B, N, K, T);
    return cudaGetLastError();
}

cudaError_t launch_mlp_infer(const float* feat, uint32_t count, const __nv_bfloat16* W1t, const __nv_bfloat16* W2t,
                             const __nv_bfloat16* W3t, const float* b1, const float* b2, const float* b3, float* logits,
                             uint8_t* sel, uint32_t* err, int device, cudaStream_t st) {
    if (count == 0) return cudaSuccess;
    static bool attr = false;
    if (!attr) {
        cudaError_t e =
            cudaFuncSetAttribute(mlp_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInferSmem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    InferArgs G;
    G.feat = feat;
    G.count = count;
    G.W1t = W1t;
    G.W2t = W2t;
    G.W3t = W3t;
    G.b1 = b1;
    G.b2 = b2;
    G.b3 = b3;
    G.logits = logits;
    G.sel = sel;
    G.err = err;
    const uint32_t tiles = (count + 127) / 128;
    const uint32_t grid = std::min<uint32_t>(tiles, (uint32_t)std::max(sms, 1));
    mlp_infer_kernel<<<grid, kInferThreads, kInferSmem, st>>>(G);
    return cudaGetLastError();
}

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
