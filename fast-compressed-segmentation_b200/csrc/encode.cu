// encode.cu -- sm_100a brick encoder, byte-identical to the reference encoder.
//
// Reference behaviour restated here (paths relative to the reference root):
//   splitGridIntoBricks   brick.hpp:133-195     Brick::build       brick.hpp:78-123
//   majorityVote8         brick.hpp:24-37       bestOperation      brickEncoding.hpp:188-318
//   encodeBrick           brickEncoding.hpp:348-447
//   packOperationsToNibbles brickEncoding.cpp:11-91
//   updateFrequencyTables brickEncoding.cpp:94-144 (bricks i % 512 == 0, brickEncoding.hpp:481-482)
//   buildRansModel        brickEncoding.cpp:146-200
//   ransEncodeSymbol/ransFlush brickEncoding.cpp:202-219, brickEncoding.hpp:452-526
//   saveDatasetToFile     fileIO.cpp:15-99
//
// Pipeline (one launch each):
//   K1 enc_bricks: one CTA per brick (persistent).  Builds the majority pyramid
//      straight from the volume (no Morton-ordered copy of the leaves), chooses
//      Rp/Rx/Ry/Rz for every child of every non-constant parent in parallel,
//      leaves the palette ops to one warp that walks the ops in stream order
//      with a 17-entry window of the most recent palette entries (reverse find
//      only matters up to distance 16: farther or absent means Pa), then lays
//      out nibbles with a block scan and packs them.  Also records, for the
//      seek index, the nibble and palette index of every S-th op.
//   K2 model: buildRansModel on the shared 16-bin histogram.
//   K3 rans: one thread per brick, symbols in reverse; while encoding it also
//      records the decoder state at the seek checkpoints (the decoder's state
//      before symbol i is the encoder's state after symbol i).
//   K4 serialize: header + records, file order.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "block_scan.cuh"
#include "csv_internal.h"

namespace csv {

constexpr int kEncThreads = 512;
constexpr uint32_t kEncSmemLevels = 5;  // levels 0..4 in shared memory
constexpr uint32_t kEncSmemNodes = 4681;
constexpr uint32_t OP_PALNEED = 7;  // placeholder code until the palette walk decides P0 / Pd / Pa
constexpr uint32_t EF_UNIFORM = 1u, EF_OVERFLOW = 2u;
// Encoder counters (u64 words): 0 nibble pool head, 1 palette pool head,
// 2..17 the sampled bricks' nibble histogram, 18 the brick work queue (low
// 32 bits), 19 checkpoint pool head.
constexpr uint32_t kMiscQueue = 18, kMiscCk = 19, kMiscWords = 32;
constexpr uint32_t kModes = 12;
constexpr uint32_t kMaxTables = 16;
constexpr uint32_t kModelWords = 65;  // freq[16] cum[16] total M[16] shift[16]

struct EncMeta {
    uint64_t nib_off, pal_off, enc_off;
    uint32_t P, nsym, nbytes, n_ops;
    uint32_t id, flags, n_ck, E;
    uint32_t level_start[8];
    uint32_t sel;     // mode | table << 4
    uint32_t ck_off;  // first of the brick's n_ck seek checkpoints in the checkpoint pool
};

struct EncoderState {
    int device = 0;
    uint32_t b = 0, L = 0, nb = 0, S = kOpsPerCheckpoint;
    uint64_t ck_used = 0;  // checkpoints of the last encode (pool entries in use)
    bool bricks_done = false;  // a shard's K1 ran; finish_encode_shard completes the image
    uint64_t W = 0, H = 0, D = 0;
    // buffers (grow-only)
    EncMeta* d_meta = nullptr;
    size_t meta_cap = 0;
    Checkpoint* d_ck = nullptr;
    size_t ck_cap_total = 0;
    uint8_t* d_nib = nullptr;
    size_t nib_cap = 0;
    uint64_t* d_pal = nullptr;
    size_t pal_cap = 0;
    uint8_t* d_enc = nullptr;
    size_t enc_cap = 0;
    uint64_t* d_enc_off = nullptr;
    uint64_t* d_rec_off = nullptr;
    size_t off_cap = 0, rec_cap = 0;
    uint8_t* d_scratch = nullptr;
    size_t scratch_cap = 0;
    unsigned long long* d_misc = nullptr;  // [0] nib head, [1] pal head, [2..17] histogram, [18] queue
    uint32_t* d_model = nullptr;           // freq[16] cum[17] M[16] sh[16]
    uint8_t* d_image = nullptr;
    size_t image_cap = 0, image_len = 0;
    uint32_t freq[16] = {}, cum[17] = {};
    uint32_t n_tables = 1;                       // rANS models of the last image
    uint32_t tab_freq[16][16] = {}, tab_cum[16][16] = {};
    bool v2 = false;
    std::vector<EncMeta> h_meta;
    bool valid = false;
};

EncoderState* encoder_state_new() { return new EncoderState(); }

void encoder_state_free(EncoderState* s) {
    if (!s) return;
    cudaFree(s->d_meta);
    cudaFree(s->d_ck);
    cudaFree(s->d_nib);
    cudaFree(s->d_pal);
    cudaFree(s->d_enc);
    cudaFree(s->d_enc_off);
    cudaFree(s->d_rec_off);
    cudaFree(s->d_scratch);
    cudaFree(s->d_misc);
    cudaFree(s->d_model);
    cudaFree(s->d_image);
    delete s;
}

// ------------------------------------------------------------ majority
// majorityVote8 (brick.hpp:24-37) under GNU libstdc++: the unordered_map has
// 13 buckets for <= 8 keys and the identity hash.  Its iteration list holds
// bucket groups newest-group-first and keys newest-first inside a group, and
// max_element keeps the first maximal count.  So among the labels with the
// largest count the winner is the one whose bucket group appeared last and,
// within the group, the label that appeared last.  Positions of first
// appearance stand in for insertion order.
__device__ __forceinline__ uint64_t majority8(const uint64_t v[8]) {
    bool all = true;
#pragma unroll
    for (int i = 1; i < 8; ++i) all &= (v[i] == v[0]);
    if (all) return v[0];
    uint32_t bkt[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) bkt[i] = (uint32_t)(v[i] % 13ull);
    int best = 0, bcnt = -1, bgrp = -1;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        bool first = true;
        int cnt = 0, grp = i;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            bool eq = v[j] == v[i];
            if (j < i && eq) first = false;
            cnt += eq ? 1 : 0;
        }
        // first key (by appearance) sharing this bucket
#pragma unroll
        for (int j = 7; j >= 0; --j) {
            if (j < i) {
                bool key_j = true;
#pragma unroll
                for (int k = 0; k < 8; ++k)
                    if (k < j && v[k] == v[j]) key_j = false;
                if (key_j && bkt[j] == bkt[i]) grp = j;
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

__device__ __forceinline__ uint32_t demorton_axis(uint32_t m) {
    m &= 0x09249249u;
    m = (m ^ (m >> 2)) & 0x030c30c3u;
    m = (m ^ (m >> 4)) & 0x0300f00fu;
    m = (m ^ (m >> 8)) & 0x030000ffu;
    m = (m ^ (m >> 16)) & 0x000003ffu;
    return m;
}
__device__ __forceinline__ uint32_t spread_axis(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}
__device__ __forceinline__ uint32_t morton3(uint32_t x, uint32_t y, uint32_t z) {
    return spread_axis(x) | (spread_axis(y) << 1) | (spread_axis(z) << 2);
}

// ------------------------------------------------------------ K1 bricks
struct EncArgs {
    const uint64_t* vol;
    uint64_t W, H, D;
    uint32_t b, L, nbx, nby, nbz, nb, S;
    uint8_t* scratch;
    uint64_t scratch_per_cta;
    EncMeta* meta;
    uint8_t* nib_pool;
    uint64_t nib_cap;
    uint64_t* pal_pool;
    uint64_t pal_cap;
    Checkpoint* ck;     // checkpoint pool, reserved per brick at misc[kMiscCk]
    uint64_t ck_cap;    // pool entries
    uint32_t bx0;         // brick-x offset of this volume in a larger one (brick IDs)
    uint32_t index_base;  // file index of brick 0 in the larger volume (the model's sample rule)
    unsigned long long* misc;
    const uint8_t* sel;  // per brick: mode | table << 4 (null: mode 0, table 0)
};

struct EncShared {
    uint64_t lab[kEncSmemNodes];
    uint8_t cst[kEncSmemNodes];
    uint32_t sh32[kEncThreads / 32 + 1];
    uint32_t hist[16];
    uint32_t work, P;
    uint64_t nib_off, pal_off, ck_off;
};

struct BrickCtx {
    const EncArgs* A;
    EncShared* S;
    uint64_t x0, y0, z0;
    uint64_t* lab_g;
    uint8_t* cst_g;
};

__device__ __forceinline__ uint64_t voxel(const BrickCtx& B, uint32_t x, uint32_t y, uint32_t z) {
    uint64_t gx = B.x0 + x, gy = B.y0 + y, gz = B.z0 + z;
    const EncArgs& A = *B.A;
    if (gx < A.W && gy < A.H && gz < A.D) return __ldg(A.vol + gx + A.W * (gy + A.H * gz));
    return 0;  // padding, brick.hpp:181-183
}
__device__ __forceinline__ uint64_t node_label(const BrickCtx& B, uint32_t l, uint32_t m) {
    if (l == B.A->L - 1) return voxel(B, demorton_axis(m), demorton_axis(m >> 1), demorton_axis(m >> 2));
    if (l < kEncSmemLevels) return B.S->lab[((1u << (3 * l)) - 1) / 7 + m];
    return B.lab_g[m];
}
__device__ __forceinline__ bool node_const(const BrickCtx& B, uint32_t l, uint32_t m) {
    if (l == B.A->L - 1) return true;  // leaves are constant (brick.hpp:188)
    if (l < kEncSmemLevels) return B.S->cst[((1u << (3 * l)) - 1) / 7 + m] != 0;
    return B.cst_g[m] != 0;
}

// Decoder-transparent encoding modes.  Where several ops reproduce a child's
// label, bestOperation (brickEncoding.hpp:198-282) takes Rp, then Rx, Ry, Rz,
// then a palette op.  A mode keeps the grammar and changes that preference:
// mode % 6 picks the order of the three neighbour axes, and modes >= 6 try the
// neighbours before the parent.  The decoder replays any of them unchanged;
// mode 0 is the reference's order.
__constant__ uint8_t kAxisOrder[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};

// Rp / Rx / Ry / Rz for child n on level lc (bestOperation, brickEncoding.hpp:198-282),
// or OP_PALNEED when only a palette op can express it.
__device__ __forceinline__ uint32_t choose_reuse(const BrickCtx& B, uint32_t lc, uint32_t n, uint64_t Lc,
                                                 uint64_t parent, uint32_t mode) {
    const bool nfirst = mode >= 6;
    if (!nfirst && parent == Lc) return OP_RP;
    const uint32_t ord = nfirst ? mode - 6 : mode;
    const uint32_t lvlmask = (1u << (3 * lc)) - 1u;
#pragma unroll
    for (uint32_t k = 0; k < 3; ++k) {
        const uint32_t a = kAxisOrder[ord][k];
        const uint32_t m = (0x09249249u << a) & lvlmask, bit = 1u << a;
        if (n & bit) {  // +1 side: later in Morton order -> the neighbour's parent (:265-272)
            if ((n & m) == m) continue;
            uint32_t N = (((n | ~m) + bit) & m) | (n & ~m);
            if (node_label(B, lc - 1, N >> 3) == Lc) return OP_RX + a;
        } else {  // -1 side: earlier in Morton order -> the neighbour itself (:256-261)
            if ((n & m) == 0) continue;
            uint32_t N = (((n & m) - bit) & m) | (n & ~m);
            if (node_label(B, lc, N) == Lc) return OP_RX + a;
        }
    }
    if (nfirst && parent == Lc) return OP_RP;
    return OP_PALNEED;
}

// Per-CTA scratch carved from the context's encoder scratch.
struct EncScratch {
    uint64_t* lab_g;  // level L-2 labels when that level does not fit in shared memory
    uint8_t* cst_g;
    uint8_t* ops;     // code | stop << 3 | delta << 4
    uint64_t* pal_lab;
    uint8_t* nib;
    uint64_t* pal_out;
};

__device__ __forceinline__ EncScratch enc_scratch(const EncArgs& A) {
    const uint64_t max_ops = ((1ull << (3 * A.L)) - 8) / 7;
    uint8_t* scr = A.scratch + (uint64_t)blockIdx.x * A.scratch_per_cta;
    auto align = [](uint64_t v) { return (v + 255) & ~255ull; };
    const uint32_t n_g = A.L >= kEncSmemLevels + 2 ? (1u << (3 * (A.L - 2))) : 0;  // level L-2 when it is big
    EncScratch X;
    uint64_t o = 0;
    X.lab_g = reinterpret_cast<uint64_t*>(scr + o);
    o = align(o + 8ull * n_g);
    X.cst_g = scr + o;
    o = align(o + n_g);
    X.ops = scr + o;
    o = align(o + max_ops);
    X.pal_lab = reinterpret_cast<uint64_t*>(scr + o);
    o = align(o + 8 * max_ops);
    X.nib = scr + o;
    o = align(o + 2 * max_ops + 2);
    X.pal_out = reinterpret_cast<uint64_t*>(scr + o);
    return X;
}

// The majority pyramid of one brick (Brick::build, brick.hpp:78-123): level L-2
// straight from the voxels (x fastest for coalescing), then the coarser levels.
__device__ void build_pyramid(const BrickCtx& B) {
    const EncArgs& A = *B.A;
    EncShared& S = *B.S;
    const uint32_t tid = threadIdx.x, T = blockDim.x, L = A.L;
    {
        const uint32_t s = A.b >> 1, cnt = s * s * s;
        const uint32_t lvl = L - 2;
        for (uint32_t k = tid; k < cnt; k += T) {
            uint32_t x = k % s, y = (k / s) % s, z = k / (s * s);
            uint64_t v[8];
#pragma unroll
            for (int c = 0; c < 8; ++c) v[c] = voxel(B, 2 * x + (c & 1), 2 * y + ((c >> 1) & 1), 2 * z + (c >> 2));
            uint64_t maj = majority8(v);
            bool same = true;
#pragma unroll
            for (int c = 0; c < 8; ++c) same &= (v[c] == maj);
            uint32_t m = morton3(x, y, z);
            if (lvl < kEncSmemLevels) {
                S.lab[((1u << (3 * lvl)) - 1) / 7 + m] = maj;
                S.cst[((1u << (3 * lvl)) - 1) / 7 + m] = same;
            } else {
                B.lab_g[m] = maj;
                B.cst_g[m] = same;
            }
        }
        __syncthreads();
    }
    for (int l = (int)L - 3; l >= 0; --l) {  // buildLevel (brick.hpp:92-123)
        const uint32_t cnt = 1u << (3 * l);
        for (uint32_t m = tid; m < cnt; m += T) {
            uint64_t v[8];
            bool cc = true;
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                v[c] = node_label(B, l + 1, 8 * m + c);
                cc &= node_const(B, l + 1, 8 * m + c);
            }
            uint64_t maj = majority8(v);
            bool same = cc;
#pragma unroll
            for (int c = 0; c < 8; ++c) same &= (v[c] == maj);
            S.lab[((1u << (3 * l)) - 1) / 7 + m] = maj;
            S.cst[((1u << (3 * l)) - 1) / 7 + m] = same;
        }
        __syncthreads();
    }
}

// Reuse ops, level by level in stream order (encodeBrick, :372-433); returns the
// op count and the first op of every level in ls.
__device__ uint32_t gen_reuse_ops(const BrickCtx& B, uint32_t mode, bool root_const, uint8_t* ops, uint64_t* pal_lab,
                                  uint32_t ls[8]) {
    const uint32_t tid = threadIdx.x, T = blockDim.x, L = B.A->L;
    uint32_t base = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) ls[k] = 0;
    if (!root_const) {
        for (uint32_t l = 0; l + 1 < L; ++l) {
            const uint32_t np = 1u << (3 * l), per = (np + T - 1) / T;
            const uint32_t p0 = min(np, tid * per), p1 = min(np, p0 + per);
            uint32_t cnt = 0;
            for (uint32_t p = p0; p < p1; ++p) cnt += node_const(B, l, p) ? 0u : 1u;
            uint32_t A_l;
            uint32_t r = block_exclusive<uint32_t>(cnt, B.S->sh32, &A_l);
            ls[l] = base;
            for (uint32_t p = p0; p < p1; ++p) {
                if (node_const(B, l, p)) continue;
                const uint64_t plab = node_label(B, l, p);
#pragma unroll 1
                for (uint32_t c = 0; c < 8; ++c) {
                    const uint32_t n = 8 * p + c, j = base + 8 * r + c;
                    const uint64_t Lc = node_label(B, l + 1, n);
                    const uint32_t code = choose_reuse(B, l + 1, n, Lc, plab, mode);
                    ops[j] = (uint8_t)(code | (node_const(B, l + 1, n) ? 8u : 0u));
                    if (code == OP_PALNEED) pal_lab[j] = Lc;
                }
                ++r;
            }
            base += 8 * A_l;
            __syncthreads();
        }
    }
#pragma unroll
    for (int k = 0; k < 8; ++k)
        if ((uint32_t)k >= L - 1) ls[k] = base;
    return base;
}

// Palette ops: one warp walks the ops in stream order with a 17-entry window of
// the most recent palette entries (reverse find only matters up to distance 16:
// farther or absent means Pa).  Leaves the palette size in S.P.
__device__ void palette_walk(const BrickCtx& B, uint64_t root, uint8_t* ops, const uint64_t* pal_lab, uint64_t* pal_out,
                             uint32_t n_ops) {
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (warp == 0) {
        uint64_t w = lane == 0 ? root : 0;
        uint32_t P = 1;
        if (lane == 0 && pal_out) pal_out[0] = root;
        for (uint32_t j0 = 0; j0 < n_ops; j0 += 32) {
            const uint32_t j = j0 + lane;
            const uint32_t op = j < n_ops ? ops[j] : 0u;
            const bool need = j < n_ops && (op & 7u) == OP_PALNEED;
            uint32_t mask = __ballot_sync(0xffffffffu, need);
            const uint64_t mine = need ? pal_lab[j] : 0ull;
            while (mask) {
                const int src = __ffs(mask) - 1;
                mask &= mask - 1;
                const uint64_t Lv = __shfl_sync(0xffffffffu, mine, src);
                const uint32_t hit = __ballot_sync(0xffffffffu, lane < min(P, 17u) && w == Lv);
                uint32_t code, delta = 0;
                if (hit) {
                    const int k = __ffs(hit) - 1;  // distance from the last entry
                    code = k == 0 ? OP_P0 : OP_PD;
                    delta = k == 0 ? 0u : (uint32_t)(k - 1);
                } else {
                    code = OP_PA;
                    const uint64_t up = __shfl_up_sync(0xffffffffu, w, 1);
                    w = lane == 0 ? Lv : up;
                    if (lane == 0 && pal_out) pal_out[P] = Lv;
                    ++P;
                }
                if (lane == src) ops[j] = (uint8_t)(code | (op & 8u) | (delta << 4));
            }
        }
        if (lane == 0) B.S->P = P;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kEncThreads, 2) enc_bricks_kernel(EncArgs A) {
    __shared__ EncShared S;
    const uint32_t tid = threadIdx.x, T = blockDim.x;
    const EncScratch X = enc_scratch(A);
    uint8_t* ops = X.ops;
    uint8_t* nib = X.nib;
    uint64_t* pal_out = X.pal_out;

    for (;;) {
        if (tid == 0) S.work = atomicAdd(reinterpret_cast<unsigned int*>(A.misc + kMiscQueue), 1u);
        if (tid < 16) S.hist[tid] = 0;
        __syncthreads();
        const uint32_t i = S.work;
        if (i >= A.nb) break;
        // split order: bx outer, bz inner (brick.hpp:152-154)
        const uint32_t bz = i % A.nbz, by = (i / A.nbz) % A.nby, bx = i / (A.nbz * A.nby);
        BrickCtx B{&A, &S, (uint64_t)bx * A.b, (uint64_t)by * A.b, (uint64_t)bz * A.b, X.lab_g, X.cst_g};
        const uint32_t sel = A.sel ? A.sel[i] : 0u;
        build_pyramid(B);
        const uint64_t root = node_label(B, 0, 0);
        const bool root_const = node_const(B, 0, 0);
        uint32_t ls[8];
        const uint32_t n_ops = gen_reuse_ops(B, sel & 15u, root_const, ops, X.pal_lab, ls);
        palette_walk(B, root, ops, X.pal_lab, pal_out, n_ops);
        const uint32_t P = S.P;

        // ---- nibble layout (packOperationsToNibbles) and seek checkpoints
        {
            const uint32_t per = (n_ops + T - 1) / T;
            const uint32_t j0 = min(n_ops, tid * per), j1 = min(n_ops, j0 + per);
            uint32_t nc = 0, pa = 0;
            for (uint32_t j = j0; j < j1; ++j) {
                uint32_t c = ops[j] & 7u;
                nc += c == OP_PD ? 2u : 1u;
                pa += c == OP_PA ? 1u : 0u;
            }
            // the brick's seek checkpoints (one per S ops) are reserved in the pool
            const uint32_t n_ck = (n_ops + A.S - 1) / A.S;
            if (tid == 0) S.ck_off = atomicAdd(A.misc + kMiscCk, (unsigned long long)n_ck);
            uint32_t NC, PA;
            uint32_t pos = 1 + block_exclusive<uint32_t>(nc, S.sh32, &NC);
            uint32_t ip = block_exclusive<uint32_t>(pa, S.sh32, &PA);
            __syncthreads();
            const uint64_t ck_off = S.ck_off;
            const bool ck_ok = ck_off + n_ck <= A.ck_cap;
            Checkpoint* ck = A.ck + ck_off;
            for (uint32_t j = j0; j < j1; ++j) {
                const uint32_t op = ops[j], c = op & 7u;
                if (j % A.S == 0 && ck_ok) ck[j / A.S] = Checkpoint{0, 0, pos, ip};
                nib[pos++] = (uint8_t)((c << 1) | ((op >> 3) & 1u));
                if (c == OP_PD) nib[pos++] = (uint8_t)(op >> 4);
                if (c == OP_PA) ++ip;
            }
            if (tid == 0) nib[0] = (uint8_t)((OP_PA << 1) | (root_const ? 1u : 0u));
            const uint32_t nsym = 1 + NC;
            const uint32_t nbytes = (nsym + 1) / 2;
            if (tid == 0) {
                S.nib_off = atomicAdd(A.misc + 0, (unsigned long long)((nbytes + 15) & ~15u));
                S.pal_off = atomicAdd(A.misc + 1, (unsigned long long)P);
            }
            __syncthreads();
            const uint64_t nib_off = S.nib_off, pal_off = S.pal_off;
            // the rANS kernel reads whole 16-byte chunks of the reservation
            const bool ok = nib_off + ((nbytes + 15) & ~15u) <= A.nib_cap && pal_off + P <= A.pal_cap && ck_ok;
            const bool sample = ((A.index_base + i) % 512) == 0;  // brickEncoding.hpp:482
            for (uint32_t q = tid; q < nbytes; q += T) {
                const uint32_t hi = nib[2 * q], lo = (2 * q + 1 < nsym) ? nib[2 * q + 1] : 0u;
                if (ok) A.nib_pool[nib_off + q] = (uint8_t)((hi << 4) | lo);
                if (sample) {  // every nibble of the packed bytes, pad included (brickEncoding.cpp:131-143)
                    atomicAdd(&S.hist[hi], 1u);
                    atomicAdd(&S.hist[lo], 1u);
                }
            }
            if (ok)
                for (uint32_t k = tid; k < P; k += T) A.pal_pool[pal_off + k] = pal_out[k];
            __syncthreads();
            if (sample && tid < 16 && S.hist[tid]) atomicAdd(A.misc + 2 + tid, (unsigned long long)S.hist[tid]);
            if (tid == 0) {
                EncMeta m;
                m.nib_off = nib_off;
                m.pal_off = pal_off;
                m.enc_off = 0;
                m.P = P;
                m.nsym = nsym;
                m.nbytes = nbytes;
                m.n_ops = n_ops;
                m.id = morton3(bx + A.bx0, by, bz);
                m.flags = (root_const ? EF_UNIFORM : 0u) | (ok ? 0u : EF_OVERFLOW);
                m.n_ck = n_ck;
                m.E = 0;
                m.sel = sel;
                m.ck_off = ck_ok ? (uint32_t)ck_off : 0u;
#pragma unroll
                for (int k = 0; k < 8; ++k) m.level_start[k] = ls[k];
                A.meta[i] = m;
            }
        }
        __syncthreads();
    }
}

// Exhaustive statistics for the mode / table choice: per brick and mode, the
// histogram of the 16 nibble values the rANS coder would see (root nibble, op
// nibbles, Pd offsets and the pad nibble of an odd count).
__global__ void __launch_bounds__(kEncThreads, 2) enc_stats_kernel(EncArgs A, uint32_t* __restrict__ hist_out) {
    __shared__ EncShared S;
    const uint32_t tid = threadIdx.x, T = blockDim.x;
    const EncScratch X = enc_scratch(A);
    for (;;) {
        if (tid == 0) S.work = atomicAdd(reinterpret_cast<unsigned int*>(A.misc + kMiscQueue), 1u);
        __syncthreads();
        const uint32_t i = S.work;
        if (i >= A.nb) break;
        const uint32_t bz = i % A.nbz, by = (i / A.nbz) % A.nby, bx = i / (A.nbz * A.nby);
        BrickCtx B{&A, &S, (uint64_t)bx * A.b, (uint64_t)by * A.b, (uint64_t)bz * A.b, X.lab_g, X.cst_g};
        build_pyramid(B);
        const uint64_t root = node_label(B, 0, 0);
        const bool root_const = node_const(B, 0, 0);
        for (uint32_t mode = 0; mode < kModes; ++mode) {
            if (tid < 16) S.hist[tid] = 0;
            uint32_t ls[8];
            const uint32_t n_ops = gen_reuse_ops(B, mode, root_const, X.ops, X.pal_lab, ls);
            palette_walk(B, root, X.ops, X.pal_lab, nullptr, n_ops);
            uint32_t nc = 0;
            for (uint32_t j = tid; j < n_ops; j += T) {
                const uint32_t op = X.ops[j], c = op & 7u;
                atomicAdd(&S.hist[(c << 1) | ((op >> 3) & 1u)], 1u);
                if (c == OP_PD) atomicAdd(&S.hist[op >> 4], 1u);
                nc += c == OP_PD ? 2u : 1u;
            }
            uint32_t NC;
            block_exclusive<uint32_t>(nc, S.sh32, &NC);
            if (tid == 0) {
                atomicAdd(&S.hist[(OP_PA << 1) | (root_const ? 1u : 0u)], 1u);  // root nibble
                if (((1 + NC) & 1u) != 0) atomicAdd(&S.hist[0], 1u);             // pad nibble
            }
            __syncthreads();
            if (tid < 16) hist_out[((size_t)i * kModes + mode) * 16 + tid] = S.hist[tid];
            __syncthreads();
        }
    }
}

// ------------------------------------------------------------ K2 model
// buildRansModel (brickEncoding.cpp:146-200) plus per-symbol constants for the
// encoder: M = ceil(2^(31+s) / f) with s = ceil(log2 f) gives floor(x / f) =
// (x * M) >> (31 + s) exactly for every x < 2^31 (the encoder's state bound):
// M = 2^(31+s)/f + e with 0 <= e < 1 adds less than x / 2^(31+s) < 2^-s <= 1/f
// to x/f, whose fractional part is at most 1 - 1/f (Granlund & Montgomery 1994).
__global__ void model_kernel(const unsigned long long* hist, uint32_t* model) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    uint32_t freq[16];
    uint64_t raw = 0, norm = 0;
    for (int i = 0; i < 16; ++i) {
        uint32_t f = (uint32_t)hist[i];  // size_t -> uint32_t as :157
        if (f == 0) f = 1;
        freq[i] = f;
        raw += f;
    }
    for (int i = 0; i < 16; ++i) {
        uint64_t s = ((uint64_t)freq[i] * kTot) / raw;
        if (s == 0) s = 1;
        freq[i] = (uint32_t)s;
        norm += s;
    }
    while (norm < kTot) { freq[0]++; norm++; }
    while (norm > kTot) {
        int largest = 0;
        for (int i = 1; i < 16; ++i)
            if (freq[i] > freq[largest]) largest = i;
        if (freq[largest] > 1) { freq[largest]--; norm--; } else break;
    }
    uint32_t acc = 0;
    for (int i = 0; i < 16; ++i) {
        model[i] = freq[i];
        model[16 + i] = acc;
        acc += freq[i];
        uint32_t s = 0;
        while ((1u << s) < freq[i]) ++s;
        uint64_t M = ((1ull << (31 + s)) + freq[i] - 1) / freq[i];
        model[33 + i] = (uint32_t)M;
        model[49 + i] = 31 + s;
    }
    model[32] = acc;
}

// ------------------------------------------------------------ K3 rANS
// One encode step (ransEncodeSymbol, brickEncoding.cpp:202-219).  tab: f |
// start << 13 | shift << 25 | M << 32.  The state is below 2^31 before the step
// (brickEncoding: 2^19 f after renormalisation, times 4096 / f), so at most two
// bytes leave per symbol and the reciprocal division is exact.
__device__ __forceinline__ void rans_enc_step(uint32_t& x, uint32_t& emitted, uint8_t* __restrict__ out,
                                              uint64_t e) {
    const uint32_t f = (uint32_t)e & 0x1FFFu;
    const uint32_t bound = ((kRansL >> kTotBits) << 8) * f;
    if (x >= bound) {
        out[emitted++] = (uint8_t)(x & 0xFF);
        x >>= 8;
        if (x >= bound) {
            out[emitted++] = (uint8_t)(x & 0xFF);
            x >>= 8;
        }
    }
    const uint32_t qd = (uint32_t)(((uint64_t)x * (uint32_t)(e >> 32)) >> ((uint32_t)(e >> 25) & 63u));
    x = (qd << kTotBits) + (x - qd * f) + (((uint32_t)e >> 13) & 0xFFFu);
}

__global__ void __launch_bounds__(128) enc_rans_kernel(EncMeta* __restrict__ meta, uint32_t nb,
                                                       const uint8_t* __restrict__ nib_pool,
                                                       const uint64_t* __restrict__ enc_off,
                                                       uint8_t* __restrict__ enc_pool, const uint32_t* __restrict__ model,
                                                       uint32_t n_tables, Checkpoint* __restrict__ ck_all,
                                                       uint32_t lanes) {
    __shared__ uint64_t tabs[kMaxTables * 16];
    for (uint32_t k = threadIdx.x; k < 16 * n_tables; k += blockDim.x) {
        const uint32_t* md = model + (k >> 4) * kModelWords;
        const uint32_t s = k & 15u;
        tabs[k] = (uint64_t)md[s] | ((uint64_t)md[16 + s] << 13) | ((uint64_t)md[49 + s] << 25) |
                  ((uint64_t)md[33 + s] << 32);
    }
    __syncthreads();
    // One serial chain per brick; a warp takes only `lanes` bricks (lanes
    // 0 .. lanes-1) when there are few bricks, so that lanes do not run the
    // union of other bricks' branch paths and the SM interleaves many warps.
    const uint32_t lane = threadIdx.x & 31;
    if (lane >= lanes) return;
    const uint32_t i = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * lanes + lane;
    if (i >= nb) return;
    const EncMeta m = meta[i];
    if (m.flags & EF_OVERFLOW) return;
    const uint64_t* tab = tabs + 16 * min((m.sel >> 4) & 15u, n_tables - 1);
    // the packed nibbles of a brick start 16-byte aligned and are padded to 16
    const uint4* src4 = reinterpret_cast<const uint4*>(nib_pool + m.nib_off);
    uint8_t* out = enc_pool + enc_off[i];
    Checkpoint* ck = ck_all + m.ck_off;
    int k = (int)m.n_ck - 1;
    // the next checkpoint's symbol index, and the one after it loaded a
    // checkpoint ahead so that the load is off the serial chain
    uint32_t next = k >= 0 ? ck[k].sym : 0xFFFFFFFFu;
    uint32_t after = k >= 1 ? ck[k - 1].sym : 0xFFFFFFFFu;
    uint32_t x = kRansL, emitted = 0;
    const int nchunk = (int)((m.nbytes + 15) / 16);
    uint4 cur = nchunk > 0 ? src4[nchunk - 1] : make_uint4(0, 0, 0, 0);
    for (int c16 = nchunk - 1; c16 >= 0; --c16) {
        const uint4 nxt = c16 > 0 ? src4[c16 - 1] : make_uint4(0, 0, 0, 0);  // prefetch
        const uint32_t words[4] = {cur.x, cur.y, cur.z, cur.w};
#pragma unroll
        for (int b = 15; b >= 0; --b) {
            const uint32_t q = 16u * (uint32_t)c16 + (uint32_t)b;
            if (q >= m.nbytes) continue;
            const uint32_t byte = (words[b >> 2] >> (8 * (b & 3))) & 0xFFu;
            // low nibble (symbol 2q+1) first: the symbols go in reverse order
            rans_enc_step(x, emitted, out, tab[byte & 15u]);
            if (2 * q + 1 == next) {
                ck[k].state = x;
                ck[k].pos = emitted;
                --k;
                next = after;
                after = k >= 1 ? ck[k - 1].sym : 0xFFFFFFFFu;
            }
            rans_enc_step(x, emitted, out, tab[byte >> 4]);
            if (2 * q == next) {
                ck[k].state = x;
                ck[k].pos = emitted;
                --k;
                next = after;
                after = k >= 1 ? ck[k - 1].sym : 0xFFFFFFFFu;
            }
        }
        cur = nxt;
    }
    for (int b = 0; b < 4; ++b) {  // ransFlush, little-endian
        out[emitted++] = (uint8_t)(x & 0xFF);
        x >>= 8;
    }
    meta[i].E = emitted;
}

// ------------------------------------------------------------ K4 serialize
// One block per brick record: ID, P, palette, E, stream, nSymbols (fileIO.cpp:57-96).
// Version 2 adds a u32 after the ID: the brick's table (bits 4..7) and mode (bits 0..3).
__global__ void serialize_kernel(const EncMeta* __restrict__ meta, const uint64_t* __restrict__ rec_off,
                                 const uint64_t* __restrict__ pal_pool, const uint8_t* __restrict__ enc_pool,
                                 const uint64_t* __restrict__ enc_off, uint8_t* __restrict__ image, uint32_t v2) {
    const uint32_t i = blockIdx.x;
    const EncMeta m = meta[i];
    uint8_t* dst = image + rec_off[i];
    const uint8_t* pal = reinterpret_cast<const uint8_t*>(pal_pool + m.pal_off);
    const uint8_t* enc = enc_pool + enc_off[i];
    const uint64_t pb = 8ull * m.P;
    const uint64_t h = v2 ? 12 : 8;  // ID [, sel], P
    const uint64_t total = h + 8 + pb + m.E;
    for (uint64_t k = threadIdx.x; k < total; k += blockDim.x) {
        uint8_t v;
        if (k < 4) v = (uint8_t)(m.id >> (8 * k));
        else if (k < h - 4) v = (uint8_t)((m.sel & 0xFFu) >> (8 * (k - 4)));
        else if (k < h) v = (uint8_t)(m.P >> (8 * (k - (h - 4))));
        else if (k < h + pb) v = pal[k - h];
        else if (k < h + 4 + pb) v = (uint8_t)(m.E >> (8 * (k - h - pb)));
        else if (k < h + 4 + pb + m.E) v = enc[k - h - 4 - pb];
        else v = (uint8_t)(m.nsym >> (8 * (k - h - 4 - pb - m.E)));
        dst[k] = v;
    }
}

// ------------------------------------------------------------ host driver
namespace {

template <class T>
cudaError_t grow(T** p, size_t* cap, size_t need) {
    if (*p && *cap >= need) return cudaSuccess;
    cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    size_t n = std::max<size_t>(need, 1);
    cudaError_t e = cudaMalloc(p, n * sizeof(T));
    if (e == cudaSuccess) *cap = n;
    return e;
}

size_t enc_scratch_per_cta(uint32_t b) {
    uint32_t L = levels_of(b);
    uint64_t mo = max_ops_of(b);
    auto al = [](uint64_t v) { return (v + 255) & ~255ull; };
    uint64_t n_g = L >= kEncSmemLevels + 2 ? (1ull << (3 * (L - 2))) : 0;
    return al(8 * n_g) + al(n_g) + al(mo) + al(8 * mo) + al(2 * mo + 2) + al(8 * (mo + 1));
}

int g_enc_occ[64] = {0};
uint32_t enc_grid(int device) {
    int& occ = g_enc_occ[device & 63];
    if (occ == 0) {
        int per_sm = 0, sms = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, enc_bricks_kernel, kEncThreads, 0);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        occ = std::max(1, per_sm) * std::max(1, sms);
    }
    return (uint32_t)occ;
}

}  // namespace

// Runs K1..K4 on a device volume; leaves the image in s->d_image.
// buildRansModel's per-symbol encoder constants for a given normalised table
// (the host side of model_kernel).
void table_model(const uint32_t* freq, uint32_t* model) {
    uint32_t acc = 0;
    for (int i = 0; i < 16; ++i) {
        model[i] = freq[i];
        model[16 + i] = acc;
        acc += freq[i];
        uint32_t s = 0;
        while ((1u << s) < freq[i]) ++s;
        const uint64_t M = ((1ull << (31 + s)) + freq[i] - 1) / freq[i];
        model[33 + i] = (uint32_t)M;
        model[49 + i] = 31 + s;
    }
    model[32] = acc;
}

int check_tables(const EncodeSelection* sel, std::string& err) {
    if (!sel || sel->n_tables == 0) return CSV_OK;
    if (sel->n_tables > kMaxTables) {
        err = "at most 16 shared rANS tables";
        return CSV_ERANGE;
    }
    for (uint32_t t = 0; t < sel->n_tables; ++t) {
        uint32_t sum = 0;
        for (int k = 0; k < 16; ++k) {
            if (sel->freq[t][k] == 0) {
                err = "a table frequency is 0";
                return CSV_EINVAL;
            }
            sum += sel->freq[t][k];
        }
        if (sum != kTot) {
            err = "a table's frequencies do not sum to 4096";
            return CSV_EINVAL;
        }
    }
    return CSV_OK;
}

// Per brick and mode, the 16-bin nibble histogram (the exhaustive search's statistics).
int encode_stats(EncoderState* s, int device, const uint64_t* d_vol, uint64_t W, uint64_t H, uint64_t D, uint32_t b,
                 uint32_t* d_hist, cudaStream_t st, std::string& err) {
    const uint64_t nbx = (W + b - 1) / b, nby = (H + b - 1) / b, nbz = (D + b - 1) / b;
    if (nbx > 1024 || nby > 1024 || nbz > 1024) {
        err = "volume needs more than 1024 bricks along an axis";
        return CSV_ERANGE;
    }
    const uint32_t nb = (uint32_t)(nbx * nby * nbz);
    cudaError_t e;
    if (!s->d_misc && (e = cudaMalloc(&s->d_misc, kMiscWords * sizeof(unsigned long long))) != cudaSuccess) {
        err = cudaGetErrorString(e);
        return CSV_ECUDA;
    }
    const uint32_t grid = std::min<uint32_t>(enc_grid(device), std::max<uint32_t>(nb, 1));
    const size_t per_cta = enc_scratch_per_cta(b);
    if ((e = grow(&s->d_scratch, &s->scratch_cap, per_cta * grid)) != cudaSuccess ||
        (e = cudaMemsetAsync(s->d_misc, 0, kMiscWords * sizeof(unsigned long long), st)) != cudaSuccess) {
        err = cudaGetErrorString(e);
        return CSV_ECUDA;
    }
    EncArgs A;
    memset(&A, 0, sizeof A);
    A.vol = d_vol;
    A.W = W; A.H = H; A.D = D;
    A.b = b; A.L = levels_of(b);
    A.nbx = (uint32_t)nbx; A.nby = (uint32_t)nby; A.nbz = (uint32_t)nbz;
    A.nb = nb;
    A.S = s->S;
    A.scratch = s->d_scratch;
    A.scratch_per_cta = per_cta;
    A.misc = s->d_misc;
    if (nb) enc_stats_kernel<<<grid, kEncThreads, 0, st>>>(A, d_hist);
    if ((e = cudaGetLastError()) != cudaSuccess) {
        err = cudaGetErrorString(e);
        return CSV_ECUDA;
    }
    return CSV_OK;
}

#define CK(x)                                                              \
    do {                                                                   \
        if ((e = (x)) != cudaSuccess) {                                    \
            err = std::string(#x) + ": " + cudaGetErrorString(e);          \
            return CSV_ECUDA;                                              \
        }                                                                  \
    } while (0)

// K3 + K4 (and the model) after K1: the model from the sample histogram in
// misc[2..17] (or the selection's tables), then the rANS pass and the image.
static int finish_encode(EncoderState* s, const EncodeSelection* sel, cudaStream_t st, std::string& err);

int encode_device(EncoderState* s, int device, const uint64_t* d_vol, uint64_t W, uint64_t H, uint64_t D, uint32_t b,
                  cudaStream_t st, std::string& err, const EncodeSelection* sel, const EncodeShard* shard,
                  uint64_t* hist_out) {
    s->valid = false;
    s->device = device;
    s->b = b;
    s->L = levels_of(b);
    s->W = W; s->H = H; s->D = D;
    const uint64_t nbx = (W + b - 1) / b, nby = (H + b - 1) / b, nbz = (D + b - 1) / b;
    const uint64_t nb64 = nbx * nby * nbz;
    if (nbx > 1024 || nby > 1024 || nbz > 1024 || nb64 > 0xFFFFFFFFull) {
        err = "volume needs more than 1024 bricks along an axis (10-bit Morton brick IDs, utils.cpp:10-14)";
        return CSV_ERANGE;
    }
    const uint32_t nb = (uint32_t)nb64;
    s->nb = nb;
    const uint64_t nvox = W * H * D;
    cudaError_t e;
    {
        int rc = check_tables(sel, err);
        if (rc) return rc;
    }
    if (hist_out && sel && sel->n_tables) {
        err = "a shard encodes version-1 images only";
        return CSV_EINVAL;
    }
    s->bricks_done = false;
    CK(grow(&s->d_meta, &s->meta_cap, nb));
    if (!s->d_model) CK(cudaMalloc(&s->d_model, kMaxTables * kModelWords * sizeof(uint32_t)));
    {
        static_assert(sizeof(unsigned long long) == 8, "");
        if (!s->d_misc) CK(cudaMalloc(&s->d_misc, kMiscWords * sizeof(unsigned long long)));
    }
    const uint32_t grid = std::min<uint32_t>(enc_grid(device), std::max<uint32_t>(nb, 1));
    const size_t per_cta = enc_scratch_per_cta(b);
    CK(grow(&s->d_scratch, &s->scratch_cap, per_cta * grid));
    size_t nib_need = std::max<size_t>(1 << 20, nvox / 4 + 16ull * nb);
    size_t pal_need = std::max<size_t>(1 << 16, nvox / 256 + 64ull * nb);
    // as many ops as the nibble estimate allows (a nibble or two each)
    size_t ck_need = std::max<size_t>(1 << 12, nib_need * 2 / s->S + nb);
    for (int attempt = 0; attempt < 2; ++attempt) {
        if (ck_need > 0xFFFFFFFFull) {  // checkpoint offsets are 32-bit
            err = "volume needs more than 2^32 seek checkpoints";
            return CSV_ERANGE;
        }
        CK(grow(&s->d_nib, &s->nib_cap, nib_need));
        CK(grow(&s->d_pal, &s->pal_cap, pal_need));
        CK(grow(&s->d_ck, &s->ck_cap_total, ck_need));
        CK(cudaMemsetAsync(s->d_misc, 0, kMiscWords * sizeof(unsigned long long), st));
        EncArgs A;
        A.vol = d_vol;
        A.W = W; A.H = H; A.D = D;
        A.b = b; A.L = s->L;
        A.nbx = (uint32_t)nbx; A.nby = (uint32_t)nby; A.nbz = (uint32_t)nbz;
        A.nb = nb;
        A.S = s->S;
        A.scratch = s->d_scratch;
        A.scratch_per_cta = per_cta;
        A.meta = s->d_meta;
        A.nib_pool = s->d_nib;
        A.nib_cap = s->nib_cap;
        A.pal_pool = s->d_pal;
        A.pal_cap = s->pal_cap;
        A.ck = s->d_ck;
        A.ck_cap = s->ck_cap_total;
        A.misc = s->d_misc;
        A.sel = sel ? sel->d_sel : nullptr;
        A.bx0 = shard ? shard->bx0 : 0u;
        A.index_base = shard ? shard->index_base : 0u;
        if (nb > 0) {
            enc_bricks_kernel<<<grid, kEncThreads, 0, st>>>(A);
            CK(cudaGetLastError());
        }
        unsigned long long misc[kMiscWords];
        CK(cudaMemcpyAsync(misc, s->d_misc, sizeof misc, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        s->ck_used = misc[kMiscCk];
        if (misc[0] <= s->nib_cap && misc[1] <= s->pal_cap && misc[kMiscCk] <= s->ck_cap_total) break;
        if (attempt == 1) {
            err = "encoder pools overflowed twice";
            return CSV_ENOMEM;
        }
        nib_need = std::max<size_t>(nib_need, misc[0]);
        pal_need = std::max<size_t>(pal_need, misc[1]);
        ck_need = std::max<size_t>(ck_need, misc[kMiscCk]);
    }
    if (hist_out) {  // a shard: stop here with the sample histogram; finish_encode_shard completes it
        unsigned long long h[16];
        CK(cudaMemcpyAsync(h, s->d_misc + 2, sizeof h, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        for (int k = 0; k < 16; ++k) hist_out[k] = h[k];
        s->bricks_done = true;
        return CSV_OK;
    }
    return finish_encode(s, sel, st, err);
}

int finish_encode_shard(EncoderState* s, const uint64_t hist[16], cudaStream_t st, std::string& err) {
    if (!s || !s->bricks_done) {
        err = "no encoder shard waiting for its model on this context";
        return CSV_EINVAL;
    }
    cudaError_t e;
    unsigned long long h[16];
    for (int k = 0; k < 16; ++k) h[k] = hist[k];
    CK(cudaMemcpyAsync(s->d_misc + 2, h, sizeof h, cudaMemcpyHostToDevice, st));
    s->bricks_done = false;
    return finish_encode(s, nullptr, st, err);
}

static int finish_encode(EncoderState* s, const EncodeSelection* sel, cudaStream_t st, std::string& err) {
    cudaError_t e;
    const uint32_t nb = s->nb, b = s->b;
    const uint32_t n_tables = sel ? sel->n_tables : 0;
    const bool v2 = n_tables > 0;
    const int device = s->device;
    std::vector<uint32_t> models(kMaxTables * kModelWords, 0);
    if (v2) {  // the caller's shared tables
        for (uint32_t t = 0; t < n_tables; ++t) table_model(sel->freq[t], &models[t * kModelWords]);
        CK(cudaMemcpyAsync(s->d_model, models.data(), n_tables * kModelWords * sizeof(uint32_t),
                           cudaMemcpyHostToDevice, st));
    } else {  // one model from the sampled bricks' histogram (brickEncoding.hpp:481-482)
        model_kernel<<<1, 1, 0, st>>>(s->d_misc + 2, s->d_model);
        CK(cudaGetLastError());
    }
    s->h_meta.resize(nb);
    if (nb) CK(cudaMemcpyAsync(s->h_meta.data(), s->d_meta, sizeof(EncMeta) * nb, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(models.data(), s->d_model, kModelWords * sizeof(uint32_t) * std::max<uint32_t>(1, n_tables),
                       cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const uint32_t* model = models.data();
    s->n_tables = std::max<uint32_t>(1, n_tables);
    for (uint32_t t = 0; t < s->n_tables; ++t)
        for (int k = 0; k < 16; ++k) {
            s->tab_freq[t][k] = models[t * kModelWords + k];
            s->tab_cum[t][k] = models[t * kModelWords + 16 + k];
        }
    s->v2 = v2;
    std::vector<uint64_t> enc_off(std::max<uint32_t>(nb, 1)), rec_off(std::max<uint32_t>(nb, 1));
    uint64_t eo = 0;
    for (uint32_t i = 0; i < nb; ++i) {
        enc_off[i] = eo;
        eo += (4ull * s->h_meta[i].nbytes + 4 + 15) & ~15ull;  // <= 2 bytes per symbol + flush
    }
    CK(grow(&s->d_enc, &s->enc_cap, std::max<uint64_t>(eo, 16)));
    CK(grow(&s->d_enc_off, &s->off_cap, std::max<uint32_t>(nb, 1)));
    CK(grow(&s->d_rec_off, &s->rec_cap, std::max<uint32_t>(nb, 1)));
    CK(cudaMemcpyAsync(s->d_enc_off, enc_off.data(), 8ull * nb, cudaMemcpyHostToDevice, st));
    if (nb) {
        // bricks per warp: the fewest (a power of two) that keeps about 32 warps per SM or fewer
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        uint32_t lanes = 1;
        while (lanes < 32 && (nb + lanes - 1) / lanes > 32ull * (uint64_t)std::max(sms, 1)) lanes <<= 1;
        const uint32_t per_block = 4 * lanes;  // four warps per block share the tables
        enc_rans_kernel<<<(nb + per_block - 1) / per_block, 128, 0, st>>>(
            s->d_meta, nb, s->d_nib, s->d_enc_off, s->d_enc, s->d_model, s->n_tables, s->d_ck, lanes);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(s->h_meta.data(), s->d_meta, sizeof(EncMeta) * nb, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    // version 1: 152-byte header (fileIO.cpp:25-49); version 2: 28 bytes + 128 per table
    const uint64_t hdr_bytes = v2 ? 28 + 128ull * n_tables : kHeaderBytes;
    uint64_t ro = hdr_bytes;
    for (uint32_t i = 0; i < nb; ++i) {
        s->h_meta[i].enc_off = enc_off[i];
        rec_off[i] = ro;
        ro += (v2 ? 20 : 16) + 8ull * s->h_meta[i].P + s->h_meta[i].E;
    }
    CK(grow(&s->d_image, &s->image_cap, ro));
    CK(cudaMemcpyAsync(s->d_rec_off, rec_off.data(), 8ull * nb, cudaMemcpyHostToDevice, st));
    std::vector<uint32_t> hdr(hdr_bytes / 4);
    hdr[0] = kMagic;
    hdr[1] = v2 ? 2 : 1;
    hdr[2] = nb;
    hdr[3] = b;  // the reference always writes BRICK_SIZE here (fileIO.cpp:28)
    hdr[4] = 16;
    hdr[5] = model[32];
    if (!v2) {
        for (int k = 0; k < 16; ++k) {
            hdr[6 + k] = model[k];
            hdr[22 + k] = model[16 + k];
        }
    } else {
        hdr[6] = n_tables;
        for (uint32_t t = 0; t < n_tables; ++t)
            for (int k = 0; k < 16; ++k) {
                hdr[7 + 32 * t + k] = models[t * kModelWords + k];
                hdr[7 + 32 * t + 16 + k] = models[t * kModelWords + 16 + k];
            }
    }
    for (int k = 0; k < 16; ++k) {
        s->freq[k] = model[k];
        s->cum[k] = model[16 + k];
    }
    s->cum[16] = model[32];
    CK(cudaMemcpyAsync(s->d_image, hdr.data(), hdr_bytes, cudaMemcpyHostToDevice, st));
    if (nb) {
        serialize_kernel<<<nb, 256, 0, st>>>(s->d_meta, s->d_rec_off, s->d_pal, s->d_enc, s->d_enc_off, s->d_image,
                                             v2 ? 1u : 0u);
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(st));
#undef CK
    s->image_len = ro;
    s->valid = true;
    return CSV_OK;
}

// Builds a decoder dataset from the last encode (no seek-index pass needed).
int encoder_to_dataset(EncoderState* s, DeviceDataset& d, std::string& err) {
    if (!s || !s->valid) {
        err = "no encoded image on this context";
        return CSV_EINVAL;
    }
    const uint32_t nb = s->nb;
    d.device = s->device;
    d.nb = nb;
    d.b = s->b;
    d.L = s->L;
    d.S = s->S;
    d.total = kTot;
    memcpy(d.freq, s->freq, sizeof d.freq);
    memcpy(d.cum, s->cum, sizeof d.cum);
    std::vector<BrickDesc> desc(std::max<uint32_t>(nb, 1));
    uint64_t pal_n = 0, enc_n = 0;
    d.h_ids = (uint32_t*)malloc(sizeof(uint32_t) * std::max<uint32_t>(1, nb));
    d.h_cost = (uint32_t*)malloc(sizeof(uint32_t) * std::max<uint32_t>(1, nb));
    for (uint32_t i = 0; i < nb; ++i) {
        const EncMeta& m = s->h_meta[i];
        BrickDesc& bd = desc[i];
        memset(&bd, 0, sizeof bd);
        bd.pal_off = m.pal_off;
        bd.enc_off = m.enc_off;
        bd.P = m.P;
        bd.E = m.E;
        bd.nsym = m.nsym;
        bd.id = m.id;
        bd.ck_off = m.ck_off;
        bd.ck_cap = m.n_ck;
        bd.n_ops = m.n_ops;
        bd.flags = ((m.flags & EF_UNIFORM) ? BF_UNIFORM : 0u) | (s->L << BF_LEVELS_SHIFT) |
                   ((s->v2 ? std::min((m.sel >> 4) & 15u, s->n_tables - 1) : 0u) << BF_MODEL_SHIFT);
        for (int k = 0; k < 8; ++k) bd.level_start[k] = m.level_start[k];
        d.h_ids[i] = m.id;
        d.h_cost[i] = m.nsym;
        pal_n = std::max<uint64_t>(pal_n, m.pal_off + m.P);
        enc_n = std::max<uint64_t>(enc_n, m.enc_off + ((m.E + 15) & ~15u));
        d.stream_bytes += m.E;
        d.palette_entries += m.P;
        d.max_nsym = std::max(d.max_nsym, m.nsym);
        d.max_P = std::max(d.max_P, m.P);
    }
    d.ck_entries = s->ck_used;
    d.enc_pool_bytes = std::max<uint64_t>(16, enc_n);
    d.pal_pool_entries = std::max<uint64_t>(1, pal_n);
    d.n_models = s->n_tables;
    std::vector<uint32_t> lut((size_t)kTot * s->n_tables);
    for (uint32_t t = 0; t < s->n_tables; ++t) build_lut(s->tab_freq[t], s->tab_cum[t], &lut[(size_t)t * kTot]);
    d.fast_models = lut_fast_mask(lut.data(), s->n_tables);
    cudaError_t e;
    if ((e = cudaMalloc(&d.d_bricks, sizeof(BrickDesc) * std::max<uint32_t>(1, nb))) != cudaSuccess ||
        (e = cudaMalloc(&d.d_pal, 8 * std::max<uint64_t>(1, pal_n))) != cudaSuccess ||
        (e = cudaMalloc(&d.d_enc, std::max<uint64_t>(16, enc_n))) != cudaSuccess ||
        (e = cudaMalloc(&d.d_ck, sizeof(Checkpoint) * std::max<uint64_t>(1, d.ck_entries))) != cudaSuccess ||
        (e = cudaMalloc(&d.d_lut, sizeof(uint32_t) * lut.size())) != cudaSuccess) {
        err = std::string("device allocation: ") + cudaGetErrorString(e);
        return CSV_ENOMEM;
    }
    if ((e = cudaMemcpy(d.d_bricks, desc.data(), sizeof(BrickDesc) * nb, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(d.d_pal, s->d_pal, 8 * pal_n, cudaMemcpyDeviceToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(d.d_enc, s->d_enc, enc_n, cudaMemcpyDeviceToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(d.d_ck, s->d_ck, sizeof(Checkpoint) * d.ck_entries, cudaMemcpyDeviceToDevice)) !=
            cudaSuccess ||
        (e = cudaMemcpy(d.d_lut, lut.data(), sizeof(uint32_t) * lut.size(), cudaMemcpyHostToDevice)) !=
            cudaSuccess) {
        err = std::string("dataset copy: ") + cudaGetErrorString(e);
        return CSV_ECUDA;
    }
    return CSV_OK;
}

const uint8_t* encoder_image(EncoderState* s, size_t* len) {
    if (!s || !s->valid) return nullptr;
    *len = s->image_len;
    return s->d_image;
}

}  // namespace csv
