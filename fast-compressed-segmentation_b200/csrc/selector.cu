// selector.cu -- per-brick encoding mode and shared rANS table: the exhaustive
// search, the cheap brick statistics, and the learned selector (a 3-layer MLP
// trained and run with the tensor-core dense layer of mlp.cu).
//
// No reference counterpart: the reference encodes every brick with one op
// preference order (brickEncoding.hpp:198-282) and one rANS model per dataset
// (brickEncoding.hpp:481-482).  A version-2 image (encode.cu) names a mode and
// one of up to 16 shared tables per brick; the decoder replays any mode
// unchanged and picks the brick's table, so decode stays exact.
//
//   features_kernel    32 statistics per brick from the volume (one CTA per brick)
//   select_kernel      exhaustive choice: per brick, the (mode, table) with the
//                      fewest estimated bits from the per-mode nibble histograms
//   MLP                features -> 256 -> 256 -> 12 mode logits + 16 table logits;
//                      bf16 weights, fp32 accumulation (tcgen05), Adam in fp32
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <string>
#include <vector>

#include "abi_internal.h"
#include "csv_internal.h"

namespace csv {
namespace {

constexpr uint32_t kFeat = 32, kFeatPad = 64, kHid = 256, kOut = 32, kOutPad = 64;
constexpr uint32_t kModesN = 12, kTablesN = 16;
constexpr uint32_t kFThreads = 256;

__device__ __forceinline__ uint32_t spread3(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

// majorityVote8 (brick.hpp:24-37) with the libstdc++ tie rule, as the encoder.
__device__ uint64_t maj8(const uint64_t v[8]) {
    bool all = true;
    for (int i = 1; i < 8; ++i) all &= (v[i] == v[0]);
    if (all) return v[0];
    int best = 0, bcnt = -1, bgrp = -1;
    for (int i = 0; i < 8; ++i) {
        bool first = true;
        int cnt = 0, grp = i;
        for (int j = 0; j < 8; ++j) {
            if (j < i && v[j] == v[i]) first = false;
            cnt += v[j] == v[i] ? 1 : 0;
        }
        for (int j = 7; j >= 0; --j) {
            if (j < i) {
                bool key_j = true;
                for (int k = 0; k < j; ++k)
                    if (v[k] == v[j]) key_j = false;
                if (key_j && (v[j] % 13ull) == (v[i] % 13ull)) grp = j;
            }
        }
        if (first && (cnt > bcnt || (cnt == bcnt && (grp > bgrp || (grp == bgrp && i > best))))) {
            best = i;
            bcnt = cnt;
            bgrp = grp;
        }
    }
    return v[best];
}

struct FeatShared {
    uint64_t samp[512];      // the 8^3 sample, Morton order
    uint64_t sorted[512];
    uint64_t lab[73];        // mini pyramid levels 0..2 (1 + 8 + 64); level 3 is samp
    uint8_t cst[585];        // constant flags of levels 0..3
    uint32_t cnt[16];        // eq1 x y z, eq4 x y z, zeros, runs per bucket [7], runs
    uint32_t nib[16];
};

__device__ __forceinline__ uint64_t vox(const uint64_t* vol, uint64_t W, uint64_t H, uint64_t D, uint64_t x, uint64_t y,
                                        uint64_t z) {
    return (x < W && y < H && z < D) ? __ldg(vol + x + W * (y + H * z)) : 0ull;  // padding, brick.hpp:181-183
}

__device__ __forceinline__ uint32_t bitlen(uint32_t v) { return v ? 32u - __clz(v) : 0u; }

// Mini-brick op histogram: encodeBrick's op choice (mode 0, brickEncoding.hpp:188-447)
// on the 8^3 sample, serial.  Nibbles counted: root, every op, Pd offsets.
__device__ void mini_ops(FeatShared& S) {
    auto lab = [&](uint32_t l, uint32_t m) -> uint64_t {
        return l == 3 ? S.samp[m] : S.lab[((1u << (3 * l)) - 1) / 7 + m];
    };
    auto cst = [&](uint32_t l, uint32_t m) -> bool { return S.cst[((1u << (3 * l)) - 1) / 7 + m] != 0; };
    uint64_t win[17];
    uint32_t P = 1;
    win[0] = lab(0, 0);
    S.nib[(4u << 1) | (cst(0, 0) ? 1u : 0u)]++;
    if (cst(0, 0)) return;
    for (uint32_t l = 0; l < 3; ++l) {
        const uint32_t np = 1u << (3 * l), lc = l + 1, lvlmask = (1u << (3 * lc)) - 1u;
        for (uint32_t p = 0; p < np; ++p) {
            if (cst(l, p)) continue;
            const uint64_t plab = lab(l, p);
            for (uint32_t c = 0; c < 8; ++c) {
                const uint32_t n = 8 * p + c;
                const uint64_t Lc = lab(lc, n);
                const uint32_t stop = cst(lc, n) ? 1u : 0u;
                uint32_t code = 7;
                if (plab == Lc) code = 0;
                for (uint32_t a = 0; a < 3 && code == 7; ++a) {
                    const uint32_t m = (0x09249249u << a) & lvlmask, bit = 1u << a;
                    if (n & bit) {
                        if ((n & m) == m) continue;
                        const uint32_t N = (((n | ~m) + bit) & m) | (n & ~m);
                        if (lab(lc - 1, N >> 3) == Lc) code = 1 + a;
                    } else {
                        if ((n & m) == 0) continue;
                        const uint32_t N = (((n & m) - bit) & m) | (n & ~m);
                        if (lab(lc, N) == Lc) code = 1 + a;
                    }
                }
                if (code == 7) {  // palette: reverse find within 17 (P0 / Pd), else Pa
                    int hit = -1;
                    for (uint32_t k = 0; k < min(P, 17u); ++k)
                        if (win[k] == Lc) {
                            hit = (int)k;
                            break;
                        }
                    if (hit == 0) code = 5;
                    else if (hit > 0) {
                        code = 6;
                        S.nib[hit - 1]++;
                    } else {
                        code = 4;
                        for (int k = 16; k > 0; --k) win[k] = win[k - 1];
                        win[0] = Lc;
                        ++P;
                    }
                }
                S.nib[(code << 1) | stop]++;
            }
        }
    }
}

__global__ void __launch_bounds__(kFThreads) features_kernel(const uint64_t* __restrict__ vol, uint64_t W, uint64_t H,
                                                             uint64_t D, uint32_t b, uint32_t nbx, uint32_t nby,
                                                             uint32_t nbz, float* __restrict__ feat) {
    __shared__ FeatShared S;
    const uint32_t i = blockIdx.x, tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const uint32_t bz = i % nbz, by = (i / nbz) % nby, bx = i / (nbz * nby);  // split order (brick.hpp:152-154)
    const uint64_t x0 = (uint64_t)bx * b, y0 = (uint64_t)by * b, z0 = (uint64_t)bz * b;
    if (tid < 16) {
        S.cnt[tid] = 0;
        S.nib[tid] = 0;
    }
    // the 8^3 sample at the centres of the 8^3 cells
    const uint32_t step = b / 8, off = step / 2;
    for (uint32_t k = tid; k < 512; k += kFThreads) {
        const uint32_t x = k & 7u, y = (k >> 3) & 7u, z = k >> 6;
        const uint64_t v = vox(vol, W, H, D, x0 + x * step + off, y0 + y * step + off, z0 + z * step + off);
        const uint32_t m = spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
        S.samp[m] = v;
        S.sorted[k] = v;
    }
    __syncthreads();
    // Counts over the rows of even y and even z (all x: a quarter of the voxels,
    // every pair within such a row, and each such voxel's +1 / +4 neighbours in y
    // and z).  Warp w takes the rows y = 2w, 2w + 16, ... and walks z in steps of
    // two with planes z .. z+4 of its row in registers (the z-neighbours), loads
    // rows (y+1, z) and (y+4, z) for the y-neighbours, and takes the x-neighbours
    // and the run starts from other lanes (lane l holds x = l and x = l + 32).
    uint32_t c[15] = {};
    {
        const uint32_t nch = (b + 31) / 32;  // values per lane: 1 or 2
        const bool interior = x0 + b <= W && y0 + b <= H && z0 + b <= D;
        auto row = [&](uint32_t y, uint32_t z, uint64_t out[2]) {
            if (interior) {
                const uint64_t* base = vol + x0 + W * (y0 + y + H * (z0 + z));
#pragma unroll
                for (uint32_t h = 0; h < 2; ++h) {
                    const uint32_t x = lane + 32 * h;
                    out[h] = (h < nch && x < b) ? __ldg(base + x) : 0ull;
                }
            } else {
#pragma unroll
                for (uint32_t h = 0; h < 2; ++h) {
                    const uint32_t x = lane + 32 * h;
                    out[h] = (h < nch && x < b) ? vox(vol, W, H, D, x0 + x, y0 + y, z0 + z) : 0ull;
                }
            }
        };
        for (uint32_t y = 2 * warp; y < b; y += 2 * (kFThreads / 32)) {
            uint64_t r[5][2];
#pragma unroll
            for (uint32_t k = 0; k < 5; ++k) {
                r[k][0] = r[k][1] = 0ull;
                if (k < b) row(y, k, r[k]);
            }
            for (uint32_t z = 0; z < b; z += 2) {
                uint64_t ya[2] = {0ull, 0ull}, yd[2] = {0ull, 0ull};
                if (y + 1 < b) row(y + 1, z, ya);
                if (y + 4 < b) row(y + 4, z, yd);
                uint32_t start_mask[2];
#pragma unroll
                for (uint32_t h = 0; h < 2; ++h) {
                    const uint32_t x = lane + 32 * h;
                    const bool in = h < nch && x < b;
                    const uint64_t v = r[0][h];
                    // x + 1, x + 4 and x - 1 from the lanes that hold them (all lanes shuffle)
                    const uint64_t nx = h == 0 ? r[0][1] : 0ull;
                    const uint64_t d1a = __shfl_down_sync(0xffffffffu, v, 1), d1b = __shfl_sync(0xffffffffu, nx, (lane + 1) & 31);
                    const uint64_t d4a = __shfl_down_sync(0xffffffffu, v, 4), d4b = __shfl_sync(0xffffffffu, nx, (lane + 4) & 31);
                    const uint64_t px = h == 1 ? r[0][0] : 0ull;
                    const uint64_t lfa = __shfl_up_sync(0xffffffffu, v, 1), lfb = __shfl_sync(0xffffffffu, px, 31);
                    const uint64_t x1 = lane + 1 < 32 ? d1a : d1b, x4 = lane + 4 < 32 ? d4a : d4b;
                    const uint64_t left = lane > 0 ? lfa : lfb;
                    if (in) {
                        if (x + 1 < b) c[0] += v == x1;
                        if (y + 1 < b) c[1] += v == ya[h];
                        if (z + 1 < b) c[2] += v == r[1][h];
                        if (x + 4 < b) c[3] += v == x4;
                        if (y + 4 < b) c[4] += v == yd[h];
                        if (z + 4 < b) c[5] += v == r[4][h];
                        c[6] += v == 0;
                    }
                    // a run starts where the label differs from its left neighbour
                    start_mask[h] = __ballot_sync(0xffffffffu, in && (x == 0 || left != v));
                }
                const uint64_t starts = (uint64_t)start_mask[0] | ((uint64_t)start_mask[1] << 32);
#pragma unroll
                for (uint32_t h = 0; h < 2; ++h) {
                    const uint32_t x = lane + 32 * h;
                    if ((starts >> x) & 1ull) {
                        // the run ends at the next start in the row, or at its end
                        const uint64_t after = x + 1 < 64 ? starts >> (x + 1) : 0ull;
                        const uint32_t len = after ? (uint32_t)__ffsll((long long)after) : b - x;
                        const uint32_t bucket = len <= 1    ? 0
                                                : len == 2  ? 1
                                                : len <= 4  ? 2
                                                : len <= 8  ? 3
                                                : len <= 16 ? 4
                                                : len <= 32 ? 5
                                                            : 6;
#pragma unroll
                        for (uint32_t k = 0; k < 7; ++k) c[7 + k] += bucket == k;  // (registers, not a local array)
                        c[14]++;
                    }
                }
#pragma unroll
                for (uint32_t k = 0; k < 3; ++k) {  // planes z+2 .. z+6 for the next step
                    r[k][0] = r[k + 2][0];
                    r[k][1] = r[k + 2][1];
                }
                r[3][0] = r[3][1] = r[4][0] = r[4][1] = 0ull;
                if (z + 5 < b) row(y, z + 5, r[3]);
                if (z + 6 < b) row(y, z + 6, r[4]);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 15; ++k) {
        uint32_t v = c[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0 && v) atomicAdd(&S.cnt[k], v);
    }
    // distinct labels of the sample: bitonic sort of 512 values
    for (uint32_t k2 = 2; k2 <= 512; k2 <<= 1)
        for (uint32_t j = k2 >> 1; j > 0; j >>= 1) {
            __syncthreads();
            for (uint32_t t = tid; t < 512; t += kFThreads) {
                const uint32_t p = t ^ j;
                if (p > t) {
                    const bool up = (t & k2) == 0;
                    const uint64_t a = S.sorted[t], bb = S.sorted[p];
                    if ((a > bb) == up) {
                        S.sorted[t] = bb;
                        S.sorted[p] = a;
                    }
                }
            }
        }
    __syncthreads();
    // mini pyramid of the sample (Brick::build on 8^3): levels 2, 1, 0
    for (int l = 2; l >= 0; --l) {
        const uint32_t cntl = 1u << (3 * l);
        for (uint32_t m = tid; m < cntl; m += kFThreads) {
            uint64_t v[8];
            bool cc = true;
            for (int k = 0; k < 8; ++k) {
                const uint32_t n = 8 * m + k;
                v[k] = l == 2 ? S.samp[n] : S.lab[((1u << (3 * (l + 1))) - 1) / 7 + n];
                cc &= l == 2 ? true : (S.cst[((1u << (3 * (l + 1))) - 1) / 7 + n] != 0);
            }
            const uint64_t mj = maj8(v);
            bool same = cc;
            for (int k = 0; k < 8; ++k) same &= v[k] == mj;
            S.lab[((1u << (3 * l)) - 1) / 7 + m] = mj;
            S.cst[((1u << (3 * l)) - 1) / 7 + m] = same ? 1 : 0;
        }
        __syncthreads();
    }
    for (uint32_t m = tid; m < 512; m += kFThreads) S.cst[73 + m] = 1;  // leaves are constant
    __syncthreads();
    if (tid == 0) mini_ops(S);
    __syncthreads();
    if (tid == 0) {
        uint32_t distinct = 1;
        for (uint32_t k = 1; k < 512; ++k) distinct += S.sorted[k] != S.sorted[k - 1];
        float* f = feat + (size_t)i * kFeat;
        // pairs tested: x within the sampled rows; y and z from the sampled rows outward
        const float hb = (float)(b / 2), fb = (float)b;
        const float px1 = hb * hb * (fb - 1.0f), px4 = hb * hb * (fb - 4.0f);
        const float pyz1 = hb * hb * fb, pyz4 = (float)((b - 4) / 2) * hb * fb;
        f[0] = (float)bitlen(distinct) / 10.0f;
        f[1] = (float)S.cnt[0] / px1;
        f[2] = (float)S.cnt[1] / pyz1;
        f[3] = (float)S.cnt[2] / pyz1;
        f[4] = (float)S.cnt[3] / px4;
        f[5] = (float)S.cnt[4] / pyz4;
        f[6] = (float)S.cnt[5] / pyz4;
        f[7] = (float)S.cnt[6] / (hb * hb * fb);
        const float runs = (float)max(S.cnt[14], 1u);
        for (int k = 0; k < 7; ++k) f[8 + k] = (float)S.cnt[7 + k] / runs;
        f[15] = (float)bitlen(S.cnt[14]) / 20.0f;
        uint32_t tot = 0;
        for (int k = 0; k < 16; ++k) tot += S.nib[k];
        for (int k = 0; k < 16; ++k) f[16 + k] = (float)S.nib[k] / (float)max(tot, 1u);
    }
}

// Exhaustive choice: the (mode, table) with the fewest estimated bits,
// sum_s hist[mode][s] * len[table][s] (len: bits per symbol, 16.16 fixed point);
// ties go to the lower mode, then the lower table.
__global__ void select_kernel(const uint32_t* __restrict__ hist, uint32_t nb, const uint32_t* __restrict__ len,
                              uint32_t n_tables, uint8_t* __restrict__ sel, uint64_t* __restrict__ cost_out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    uint64_t best = ~0ull;
    uint32_t bm = 0, bt = 0;
    for (uint32_t m = 0; m < kModesN; ++m) {
        const uint32_t* h = hist + ((size_t)i * kModesN + m) * 16;
        uint32_t hv[16];
        for (int s = 0; s < 16; ++s) hv[s] = h[s];
        for (uint32_t t = 0; t < n_tables; ++t) {
            uint64_t c = 0;
            for (int s = 0; s < 16; ++s) c += (uint64_t)hv[s] * len[t * 16 + s];
            if (cost_out) cost_out[((size_t)i * kModesN + m) * n_tables + t] = c;
            if (c < best) {
                best = c;
                bm = m;
                bt = t;
            }
        }
    }
    sel[i] = (uint8_t)(bm | (bt << 4));
}

// ---------------------------------------------------------------- MLP kernels
// Parameters, fp32, one array: W1 [256][64] (input columns 32..63 stay 0), b1 [256],
// W2 [256][256], b2 [256], W3 [32][256] (rows 28..31 stay 0), b3 [32].
constexpr uint32_t OFF_W1 = 0, OFF_B1 = OFF_W1 + kHid * kFeatPad, OFF_W2 = OFF_B1 + kHid,
                   OFF_B2 = OFF_W2 + kHid * kHid, OFF_W3 = OFF_B2 + kHid, OFF_B3 = OFF_W3 + kOut * kHid,
                   N_PARAMS = OFF_B3 + kOut;
static_assert(N_PARAMS == CSV_MLP_PARAMS, "parameter layout");

// features (n x 32, fp32) -> X (rows x 64, bf16, zero padded) and X^T (64 x rows)
__global__ void pack_input_kernel(const float* __restrict__ feat, uint32_t n, uint32_t rows,
                                  __nv_bfloat16* __restrict__ X, __nv_bfloat16* __restrict__ XT) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= rows * kFeatPad) return;
    const uint32_t r = k / kFeatPad, c = k % kFeatPad;
    const float v = (r < n && c < kFeat) ? feat[(size_t)r * kFeat + c] : 0.0f;
    const __nv_bfloat16 b = __float2bfloat16_rn(v);
    X[k] = b;
    XT[(size_t)c * rows + r] = b;
}

// Softmax cross-entropy of the mode head (logits 0..11) and the table head
// (12..27) against the labels; dZ = (softmax - onehot) / n as bf16 (rows x 64,
// zero beyond column 27 and row n) and its transpose (32 x rows).
__global__ void loss_grad_kernel(const float* __restrict__ Z, const uint8_t* __restrict__ label, uint32_t n,
                                 uint32_t rows, __nv_bfloat16* __restrict__ dZ, __nv_bfloat16* __restrict__ dZT,
                                 float* __restrict__ loss) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    float g[kOut];
    for (uint32_t k = 0; k < kOut; ++k) g[k] = 0.0f;
    if (r < n) {
        const float* z = Z + (size_t)r * kOut;
        const uint32_t lm = label[r] & 15u, lt = label[r] >> 4;
        float l = 0.0f;
        for (int head = 0; head < 2; ++head) {
            const uint32_t b0 = head ? kModesN : 0, cnt = head ? kTablesN : kModesN, y = head ? lt : lm;
            float mx = -INFINITY;
            for (uint32_t k = 0; k < cnt; ++k) mx = fmaxf(mx, z[b0 + k]);
            float se = 0.0f;
            for (uint32_t k = 0; k < cnt; ++k) se += expf(z[b0 + k] - mx);
            for (uint32_t k = 0; k < cnt; ++k)
                g[b0 + k] = (expf(z[b0 + k] - mx) / se - (k == y ? 1.0f : 0.0f)) / (float)n;
            l += logf(se) + mx - z[b0 + y];
        }
        atomicAdd(loss, l / (float)n);
    }
    for (uint32_t k = 0; k < kOutPad; ++k) {
        const __nv_bfloat16 v = __float2bfloat16_rn(k < kOut ? g[k] : 0.0f);
        dZ[(size_t)r * kOutPad + k] = v;
        if (k < kOut) dZT[(size_t)k * rows + r] = v;
    }
}

// Column sums of a bf16 [rows][N] matrix (row stride ld) into out[N] (fp32): the bias gradients.
__global__ void colsum_kernel(const __nv_bfloat16* __restrict__ M, uint32_t rows, uint32_t N, uint32_t ld,
                              float* __restrict__ out) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    float s = 0.0f;
    for (uint32_t r = 0; r < rows; ++r) s += __bfloat162float(M[(size_t)r * ld + c]);
    out[c] = s;
}

// Adam (Kingma & Ba 2015) on the fp32 parameters.
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, uint32_t n, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float gk = g[k];
    const float mk = b1 * m[k] + (1.0f - b1) * gk, vk = b2 * v[k] + (1.0f - b2) * gk * gk;
    m[k] = mk;
    v[k] = vk;
    p[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + eps);
}

// bf16 weight copies: W1b [256][64], W2b [256][256], W2bT, W3b [32][256], W3bT [256][64] (columns >= 32 zero)
__global__ void refresh_kernel(const float* __restrict__ P, __nv_bfloat16* W1b, __nv_bfloat16* W2b,
                               __nv_bfloat16* W2bT, __nv_bfloat16* W3b, __nv_bfloat16* W3bT) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < kHid * kFeatPad) W1b[k] = __float2bfloat16_rn(P[OFF_W1 + k]);
    if (k < kHid * kHid) {
        const uint32_t o = k / kHid, in = k % kHid;
        const __nv_bfloat16 w = __float2bfloat16_rn(P[OFF_W2 + k]);
        W2b[k] = w;
        W2bT[(size_t)in * kHid + o] = w;
    }
    if (k < kOut * kHid) {
        const uint32_t o = k / kHid, in = k % kHid;
        const __nv_bfloat16 w = __float2bfloat16_rn(P[OFF_W3 + k]);
        W3b[k] = w;
        W3bT[(size_t)in * kOutPad + o] = w;
    }
    if (k < kHid * (kOutPad - kOut)) {
        const uint32_t in = k / (kOutPad - kOut), o = kOut + k % (kOutPad - kOut);
        W3bT[(size_t)in * kOutPad + o] = __float2bfloat16_rn(0.0f);
    }
}

}  // namespace
}  // namespace csv

// ---------------------------------------------------------------- network and C ABI
using namespace csv;

struct csv_mlp {
    csv_ctx* ctx = nullptr;
    uint32_t cap = 0;  // batch rows the activations hold (multiple of 128)
    uint32_t t = 0;    // Adam steps taken
    float* P = nullptr;  // parameters, gradients, Adam moments (N_PARAMS each)
    float* G = nullptr;
    float* Mm = nullptr;
    float* Vm = nullptr;
    __nv_bfloat16 *W1b = nullptr, *W2b = nullptr, *W2bT = nullptr, *W3b = nullptr, *W3bT = nullptr;
    __nv_bfloat16 *W1t = nullptr, *W2t = nullptr, *W3t = nullptr;  // tiled for the fused forward
    __nv_bfloat16 *X = nullptr, *XT = nullptr, *H1 = nullptr, *H1T = nullptr, *H2 = nullptr, *H2T = nullptr;
    __nv_bfloat16 *dZ = nullptr, *dZT = nullptr, *dH2 = nullptr, *dH2T = nullptr, *dH1 = nullptr, *dH1T = nullptr;
    float* Z = nullptr;
    float* loss = nullptr;
    uint32_t* err = nullptr;
};

namespace {

void mlp_free_acts(csv_mlp* n) {
    for (void* p : {(void*)n->X, (void*)n->XT, (void*)n->H1, (void*)n->H1T, (void*)n->H2, (void*)n->H2T,
                    (void*)n->dZ, (void*)n->dZT, (void*)n->dH2, (void*)n->dH2T, (void*)n->dH1, (void*)n->dH1T,
                    (void*)n->Z})
        cudaFree(p);
    n->X = n->XT = n->H1 = n->H1T = n->H2 = n->H2T = n->dZ = n->dZT = n->dH2 = n->dH2T = n->dH1 = n->dH1T = nullptr;
    n->Z = nullptr;
    n->cap = 0;
}

cudaError_t mlp_reserve(csv_mlp* n, uint32_t rows) {
    if (rows <= n->cap) return cudaSuccess;
    mlp_free_acts(n);
    const size_t r = rows;
    cudaError_t e = cudaSuccess;
    auto al = [&](void** p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, bytes);
    };
    al((void**)&n->X, r * kFeatPad * 2);
    al((void**)&n->XT, r * kFeatPad * 2);
    al((void**)&n->H1, r * kHid * 2);
    al((void**)&n->H1T, r * kHid * 2);
    al((void**)&n->H2, r * kHid * 2);
    al((void**)&n->H2T, r * kHid * 2);
    al((void**)&n->dZ, r * kOutPad * 2);
    al((void**)&n->dZT, r * kOut * 2);
    al((void**)&n->dH2, r * kHid * 2);
    al((void**)&n->dH2T, r * kHid * 2);
    al((void**)&n->dH1, r * kHid * 2);
    al((void**)&n->dH1T, r * kHid * 2);
    al((void**)&n->Z, r * kOut * 4);
    if (e == cudaSuccess) n->cap = rows;
    return e;
}

cudaError_t mlp_refresh(csv_mlp* n, cudaStream_t st) {
    refresh_kernel<<<(kHid * kHid + 255) / 256, 256, 0, st>>>(n->P, n->W1b, n->W2b, n->W2bT, n->W3b, n->W3bT);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = launch_tile_b(n->W1b, kHid, kFeatPad, n->W1t, st);
    if (e == cudaSuccess) e = launch_tile_b(n->W2b, kHid, kHid, n->W2t, st);
    if (e == cudaSuccess) e = launch_tile_b(n->W3b, kOut, kHid, n->W3t, st);
    return e;
}

// Forward pass on `rows` (padded) rows of which `cnt` hold features; Z holds the logits.
cudaError_t mlp_forward(csv_mlp* n, const float* feat, uint32_t cnt, uint32_t rows, cudaStream_t st) {
    cudaError_t e;
    pack_input_kernel<<<(rows * kFeatPad + 255) / 256, 256, 0, st>>>(feat, cnt, rows, n->X, n->XT);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = launch_gemm_bf16(n->X, n->W1b, rows, kHid, kFeatPad, n->P + OFF_B1, nullptr, 1, nullptr, n->H1, n->H1T,
                              nullptr, n->err, st)) != cudaSuccess)
        return e;
    if ((e = launch_gemm_bf16(n->H1, n->W2b, rows, kHid, kHid, n->P + OFF_B2, nullptr, 1, nullptr, n->H2, n->H2T,
                              nullptr, n->err, st)) != cudaSuccess)
        return e;
    return launch_gemm_bf16(n->H2, n->W3b, rows, kOut, kHid, n->P + OFF_B3, nullptr, 0, n->Z, nullptr, nullptr,
                            nullptr, n->err, st);
}

}  // namespace

extern "C" {

void csv_mlp_destroy(csv_mlp* n) {
    if (!n) return;
    DeviceGuard g(n->ctx->device);
    mlp_free_acts(n);
    for (void* p : {(void*)n->P, (void*)n->G, (void*)n->Mm, (void*)n->Vm, (void*)n->W1b, (void*)n->W2b,
                    (void*)n->W2bT, (void*)n->W3b, (void*)n->W3bT, (void*)n->W1t, (void*)n->W2t, (void*)n->W3t,
                    (void*)n->loss, (void*)n->err})
        cudaFree(p);
    delete n;
}

int csv_mlp_create(csv_ctx* ctx, const float* params, csv_mlp** out) {
    if (!ctx || !params || !out) return CSV_EINVAL;
    *out = nullptr;
    DeviceGuard g(ctx->device);
    csv_mlp* n = new (std::nothrow) csv_mlp();
    if (!n) return abi_fail(ctx, CSV_ENOMEM, "mlp: host allocation");
    n->ctx = ctx;
    cudaError_t e = cudaSuccess;
    auto al = [&](void** p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, bytes);
    };
    al((void**)&n->P, N_PARAMS * 4);
    al((void**)&n->G, N_PARAMS * 4);
    al((void**)&n->Mm, N_PARAMS * 4);
    al((void**)&n->Vm, N_PARAMS * 4);
    al((void**)&n->W1b, kHid * kFeatPad * 2);
    al((void**)&n->W2b, kHid * kHid * 2);
    al((void**)&n->W2bT, kHid * kHid * 2);
    al((void**)&n->W3b, kOut * kHid * 2);
    al((void**)&n->W3bT, kHid * kOutPad * 2);
    al((void**)&n->W1t, kHid * kFeatPad * 2);
    al((void**)&n->W2t, kHid * kHid * 2);
    al((void**)&n->W3t, kOut * kHid * 2);
    al((void**)&n->loss, 4);
    al((void**)&n->err, 4);
    if (e == cudaSuccess) e = cudaMemcpy(n->P, params, N_PARAMS * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(n->Mm, 0, N_PARAMS * 4);
    if (e == cudaSuccess) e = cudaMemset(n->Vm, 0, N_PARAMS * 4);
    if (e == cudaSuccess) e = cudaMemset(n->G, 0, N_PARAMS * 4);
    if (e == cudaSuccess) e = cudaMemset(n->err, 0, 4);
    if (e == cudaSuccess) e = mlp_refresh(n, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        csv_mlp_destroy(n);
        return abi_cuda_fail(ctx, e, "mlp create");
    }
    *out = n;
    return CSV_OK;
}

int csv_mlp_params(const csv_mlp* n, float* params, float* grads) {
    if (!n) return CSV_EINVAL;
    DeviceGuard g(n->ctx->device);
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess && params) e = cudaMemcpy(params, n->P, N_PARAMS * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && grads) e = cudaMemcpy(grads, n->G, N_PARAMS * 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return abi_cuda_fail(n->ctx, e, "mlp params");
    return CSV_OK;
}

int csv_mlp_forward(csv_mlp* n, const float* d_feat, uint32_t count, float* d_logits, uint8_t* d_sel, void* stream) {
    if (!n || (count && !d_feat)) return CSV_EINVAL;
    if (count == 0) return CSV_OK;
    DeviceGuard g(n->ctx->device);
    if ((reinterpret_cast<uintptr_t>(d_feat) | reinterpret_cast<uintptr_t>(d_logits)) & 15u)
        return abi_fail(n->ctx, CSV_EINVAL, "mlp forward: features and logits must be 16-byte aligned");
    cudaStream_t st = (cudaStream_t)stream;
    // the fused forward: features in, logits / choices out, activations on chip
    cudaError_t e = launch_mlp_infer(d_feat, count, n->W1t, n->W2t, n->W3t, n->P + OFF_B1, n->P + OFF_B2, n->P + OFF_B3,
                                     d_logits, d_sel, n->err, n->ctx->device, st);
    if (e != cudaSuccess) return abi_cuda_fail(n->ctx, e, "mlp forward");
    return CSV_OK;
}

int csv_mlp_grad(csv_mlp* n, const float* d_feat, const uint8_t* d_label, uint32_t count, float* loss, void* stream) {
    if (!n || !d_feat || !d_label || count == 0) return CSV_EINVAL;
    DeviceGuard g(n->ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    const uint32_t rows = (count + 127) / 128 * 128;
    cudaError_t e = mlp_reserve(n, rows);
    if (e == cudaSuccess) e = mlp_forward(n, d_feat, count, rows, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(n->loss, 0, 4, st);
    if (e == cudaSuccess) {
        loss_grad_kernel<<<(rows + 127) / 128, 128, 0, st>>>(n->Z, d_label, count, rows, n->dZ, n->dZT, n->loss);
        e = cudaGetLastError();
    }
    float* G = n->G;
    // dW3^T = H2^T dZ (M 256, N 32, K rows), written transposed into W3's slot
    if (e == cudaSuccess)
        e = launch_gemm_bf16(n->H2T, n->dZT, kHid, kOut, rows, nullptr, nullptr, 0, nullptr, nullptr, nullptr,
                             G + OFF_W3, n->err, st);
    // dH2 = (dZ W3) * (H2 > 0)
    if (e == cudaSuccess)
        e = launch_gemm_bf16(n->dZ, n->W3bT, rows, kHid, kOutPad, nullptr, n->H2, 0, nullptr, n->dH2, n->dH2T,
                             nullptr, n->err, st);
    // dW2 = dH2^T H1
    if (e == cudaSuccess)
        e = launch_gemm_bf16(n->dH2T, n->H1T, kHid, kHid, rows, nullptr, nullptr, 0, G + OFF_W2, nullptr, nullptr,
                             nullptr, n->err, st);
    // dH1 = (dH2 W2) * (H1 > 0)
    if (e == cudaSuccess)
        e = launch_gemm_bf16(n->dH2, n->W2bT, rows, kHid, kHid, nullptr, n->H1, 0, nullptr, n->dH1, n->dH1T,
                             nullptr, n->err, st);
    // dW1 = dH1^T X
    if (e == cudaSuccess)
        e = launch_gemm_bf16(n->dH1T, n->XT, kHid, kFeatPad, rows, nullptr, nullptr, 0, G + OFF_W1, nullptr,
                             nullptr, nullptr, n->err, st);
    if (e == cudaSuccess) {
        colsum_kernel<<<1, 256, 0, st>>>(n->dZ, rows, kOut, kOutPad, G + OFF_B3);
        colsum_kernel<<<1, 256, 0, st>>>(n->dH2, rows, kHid, kHid, G + OFF_B2);
        colsum_kernel<<<1, 256, 0, st>>>(n->dH1, rows, kHid, kHid, G + OFF_B1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && loss) {
        e = cudaMemcpyAsync(loss, n->loss, 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (e != cudaSuccess) return abi_cuda_fail(n->ctx, e, "mlp grad");
    return CSV_OK;
}

int csv_mlp_adam(csv_mlp* n, float lr, float beta1, float beta2, float eps, void* stream) {
    if (!n) return CSV_EINVAL;
    DeviceGuard g(n->ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    n->t += 1;
    const float c1 = 1.0f - powf(beta1, (float)n->t), c2 = 1.0f - powf(beta2, (float)n->t);
    adam_kernel<<<(N_PARAMS + 255) / 256, 256, 0, st>>>(n->P, n->G, n->Mm, n->Vm, N_PARAMS, lr, beta1, beta2, eps, c1,
                                                         c2);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = mlp_refresh(n, st);
    if (e != cudaSuccess) return abi_cuda_fail(n->ctx, e, "mlp adam");
    return CSV_OK;
}

int csv_mlp_status(const csv_mlp* n) {
    if (!n) return CSV_EINVAL;
    DeviceGuard g(n->ctx->device);
    uint32_t err = 0;
    if (cudaMemcpy(&err, n->err, 4, cudaMemcpyDeviceToHost) != cudaSuccess) return CSV_ECUDA;
    return err ? CSV_ECUDA : CSV_OK;
}

int csv_brick_features(csv_ctx* ctx, const uint64_t* d_volume, uint32_t W, uint32_t H, uint32_t D,
                       uint32_t brick_size, float* d_features, void* stream) {
    if (!ctx || !d_volume || !d_features) return CSV_EINVAL;
    if (brick_size < 8 || brick_size > 64 || (brick_size & (brick_size - 1)))
        return abi_fail(ctx, CSV_EINVAL, "features: brick size must be a power of two in [8, 64]");
    DeviceGuard g(ctx->device);
    const uint32_t nbx = (W + brick_size - 1) / brick_size, nby = (H + brick_size - 1) / brick_size,
                   nbz = (D + brick_size - 1) / brick_size;
    const uint64_t nb = (uint64_t)nbx * nby * nbz;
    if (nb == 0) return CSV_OK;
    features_kernel<<<(uint32_t)nb, kFThreads, 0, (cudaStream_t)stream>>>(d_volume, W, H, D, brick_size, nbx, nby,
                                                                         nbz, d_features);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return abi_cuda_fail(ctx, e, "features");
    return CSV_OK;
}

int csv_encode_stats(csv_ctx* ctx, const uint64_t* d_volume, uint32_t W, uint32_t H, uint32_t D, uint32_t brick_size,
                     uint32_t* d_hist, void* stream) {
    if (!ctx || !d_volume || !d_hist) return CSV_EINVAL;
    if (brick_size < 8 || brick_size > 64 || (brick_size & (brick_size - 1)))
        return abi_fail(ctx, CSV_EINVAL, "brick size must be a power of two in [8, 64]");
    DeviceGuard g(ctx->device);
    if (!ctx->enc) ctx->enc = encoder_state_new();
    std::string err;
    int rc = encode_stats(ctx->enc, ctx->device, d_volume, W, H, D, brick_size, d_hist, (cudaStream_t)stream, err);
    if (rc) return abi_fail(ctx, rc, err);
    return CSV_OK;
}

int csv_select_exhaustive(csv_ctx* ctx, const uint32_t* d_hist, uint32_t n_bricks, const uint32_t* tables,
                          uint32_t n_tables, uint8_t* d_sel, uint64_t* d_cost, void* stream) {
    if (!ctx || !d_hist || !tables || !d_sel || n_tables == 0 || n_tables > kTablesN) return CSV_EINVAL;
    DeviceGuard g(ctx->device);
    // bits per symbol, 16.16 fixed point: -log2(f / 4096)
    uint32_t len[kTablesN * 16];
    for (uint32_t t = 0; t < n_tables; ++t)
        for (int s = 0; s < 16; ++s) {
            const uint32_t f = tables[t * 16 + s];
            if (f == 0 || f > kTot) return abi_fail(ctx, CSV_EINVAL, "select: table frequency out of range");
            len[t * 16 + s] = (uint32_t)llround(-log2((double)f / (double)kTot) * 65536.0);
        }
    uint32_t* d_len = nullptr;
    cudaError_t e = cudaMalloc(&d_len, sizeof len);
    if (e == cudaSuccess) e = cudaMemcpy(d_len, len, sizeof len, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && n_bricks) {
        select_kernel<<<(n_bricks + 127) / 128, 128, 0, (cudaStream_t)stream>>>(d_hist, n_bricks, d_len, n_tables,
                                                                                 d_sel, d_cost);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
    cudaFree(d_len);
    if (e != cudaSuccess) return abi_cuda_fail(ctx, e, "select");
    return CSV_OK;
}

int csv_encode_device_sel(csv_ctx* ctx, const uint64_t* d_volume, uint32_t W, uint32_t H, uint32_t D,
                          uint32_t brick_size, const uint32_t* tables, uint32_t n_tables, const uint8_t* d_sel,
                          void* stream, size_t* image_len) {
    if (!ctx || !d_volume || (n_tables && !tables) || n_tables > kTablesN) return CSV_EINVAL;
    if (brick_size < 8 || brick_size > 64 || (brick_size & (brick_size - 1)))
        return abi_fail(ctx, CSV_EINVAL, "brick size must be a power of two in [8, 64]");
    DeviceGuard g(ctx->device);
    if (!ctx->enc) ctx->enc = encoder_state_new();
    EncodeSelection sel;
    sel.n_tables = n_tables;
    for (uint32_t t = 0; t < n_tables; ++t)
        for (int s = 0; s < 16; ++s) sel.freq[t][s] = tables[t * 16 + s];
    sel.d_sel = d_sel;
    std::string err;
    int rc = encode_device(ctx->enc, ctx->device, d_volume, W, H, D, brick_size, (cudaStream_t)stream, err, &sel);
    if (rc) return abi_fail(ctx, rc, err);
    size_t len = 0;
    encoder_image(ctx->enc, &len);
    if (image_len) *image_len = len;
    return CSV_OK;
}

// ---- selector files: the fitted tables and the trained network, so that a
// learned encode needs no training run.  Little-endian: u32 magic "CSVS"
// (0x53565343), u32 version 1, u32 CSV_MLP_PARAMS, u32 n_tables (1..16), u32
// tables[n_tables][16], f32 params[CSV_MLP_PARAMS], u32 FNV-1a of every byte
// before it.
static uint32_t fnv1a(const uint8_t* p, size_t n, uint32_t h = 2166136261u) {
    for (size_t i = 0; i < n; ++i) h = (h ^ p[i]) * 16777619u;
    return h;
}
static bool tables_ok(const uint32_t* t, uint32_t n) {
    if (n == 0 || n > kTablesN) return false;
    for (uint32_t k = 0; k < n; ++k) {
        uint32_t sum = 0;
        for (int s = 0; s < 16; ++s) {
            if (t[k * 16 + s] == 0) return false;
            sum += t[k * 16 + s];
        }
        if (sum != kTot) return false;
    }
    return true;
}
constexpr uint32_t kSelMagic = 0x53565343u;

int csv_selector_write(const char* path, const float* params, const uint32_t* tables, uint32_t n_tables) {
    if (!path || !params || !tables) return CSV_EINVAL;
    if (!tables_ok(tables, n_tables)) return CSV_EINVAL;
    std::vector<uint8_t> buf;
    auto put = [&](const void* p, size_t n) {
        const uint8_t* b = (const uint8_t*)p;
        buf.insert(buf.end(), b, b + n);
    };
    const uint32_t head[4] = {kSelMagic, 1u, (uint32_t)N_PARAMS, n_tables};
    put(head, sizeof head);
    put(tables, 64ull * n_tables);
    put(params, 4ull * N_PARAMS);
    const uint32_t h = fnv1a(buf.data(), buf.size());
    put(&h, 4);
    FILE* f = fopen(path, "wb");
    if (!f) return CSV_EIO;
    const size_t w = fwrite(buf.data(), 1, buf.size(), f);
    const int c = fclose(f);
    return (w == buf.size() && c == 0) ? CSV_OK : CSV_EIO;
}

int csv_selector_read(const char* path, float* params, uint32_t* tables, uint32_t* n_tables) {
    if (!path || !params || !tables || !n_tables) return CSV_EINVAL;
    FILE* f = fopen(path, "rb");
    if (!f) return CSV_EIO;
    std::vector<uint8_t> buf;
    uint8_t tmp[65536];
    size_t r;
    while ((r = fread(tmp, 1, sizeof tmp, f)) > 0) buf.insert(buf.end(), tmp, tmp + r);
    fclose(f);
    if (buf.size() < 20) return CSV_EFORMAT;
    uint32_t head[4];
    memcpy(head, buf.data(), sizeof head);
    if (head[0] != kSelMagic || head[1] != 1u || head[2] != (uint32_t)N_PARAMS || head[3] == 0 || head[3] > kTablesN)
        return CSV_EFORMAT;
    const size_t need = 16 + 64ull * head[3] + 4ull * N_PARAMS + 4;
    if (buf.size() != need) return CSV_EFORMAT;
    uint32_t h;
    memcpy(&h, buf.data() + need - 4, 4);
    if (h != fnv1a(buf.data(), need - 4)) return CSV_EFORMAT;
    if (!tables_ok(reinterpret_cast<const uint32_t*>(buf.data() + 16), head[3])) return CSV_EFORMAT;
    memcpy(tables, buf.data() + 16, 64ull * head[3]);
    memcpy(params, buf.data() + 16 + 64ull * head[3], 4ull * N_PARAMS);
    *n_tables = head[3];
    return CSV_OK;
}

// The learned encode in one call: features of every brick, the network's
// choice, the encode with those choices into a version-2 image.
int csv_encode_learned(csv_ctx* ctx, const uint64_t* d_volume, uint32_t W, uint32_t H, uint32_t D,
                       uint32_t brick_size, csv_mlp* net, const uint32_t* tables, uint32_t n_tables, void* stream,
                       size_t* image_len) {
    if (!ctx || !d_volume || !net || !tables) return CSV_EINVAL;
    if (!tables_ok(tables, n_tables)) return abi_fail(ctx, CSV_EINVAL, "learned encode: tables must sum to 4096");
    if (brick_size < 8 || brick_size > 64 || (brick_size & (brick_size - 1)))
        return abi_fail(ctx, CSV_EINVAL, "brick size must be a power of two in [8, 64]");
    DeviceGuard g(ctx->device);
    const uint64_t nb = (uint64_t)((W + brick_size - 1) / brick_size) * ((H + brick_size - 1) / brick_size) *
                        ((D + brick_size - 1) / brick_size);
    if (nb == 0 || nb > 0xFFFFFFFFull) return abi_fail(ctx, CSV_ERANGE, "learned encode: brick count");
    float* d_feat = nullptr;
    uint8_t* d_sel = nullptr;
    cudaError_t e = cudaMalloc(&d_feat, nb * CSV_FEATURES * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&d_sel, nb);
    if (e != cudaSuccess) {
        cudaFree(d_feat);
        return abi_cuda_fail(ctx, e, "learned encode");
    }
    int rc = csv_brick_features(ctx, d_volume, W, H, D, brick_size, d_feat, stream);
    if (rc == CSV_OK) rc = csv_mlp_forward(net, d_feat, (uint32_t)nb, nullptr, d_sel, stream);
    if (rc == CSV_OK)
        rc = csv_encode_device_sel(ctx, d_volume, W, H, D, brick_size, tables, n_tables, d_sel, stream, image_len);
    cudaStreamSynchronize((cudaStream_t)stream);
    cudaFree(d_feat);
    cudaFree(d_sel);
    return rc;
}

}  // extern "C"
