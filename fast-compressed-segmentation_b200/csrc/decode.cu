// decode.cu -- sm_100a brick decoder: seek-index build and the batched decode kernel.
//
// Reference behaviour restated here (paths relative to the reference root):
//   rANS          brickDecoding.cpp:126-188 (== web/scripts/decode.js:36-104)
//   op parsing    brickDecoding.cpp:20-59, decode.wgsl:87-127
//   replay        brickDecoding.hpp:174-242 (full resolution), decode.wgsl:344-509 (any LOD)
//   neighbors     brickDecoding.cpp:77-124, decode.wgsl:247-306
//
// The reference replays every op of a brick in one serial chain (one leader
// thread per workgroup in decode.wgsl).  Here a brick is decoded by a whole
// CTA:
//   1. rANS: the brick's op stream is cut at seek checkpoints (decoder state
//      every S ops, built once per dataset or emitted by the encoder); each
//      thread decodes one segment and writes one 4-byte record per op (code,
//      stop, resolved palette index).
//   2. levels, coarse to fine, held in shared memory: the value of every node
//      as a palette index (16-bit when the palette allows), a bitmask of the
//      nodes with stop bit 0 ("active": their children have ops), and per
//      32-node word the count of active nodes before it, so the rank of an
//      active node -- which locates its children's ops -- is one popcount.
//      Children of inactive parents inherit the parent's value in one uniform
//      pass; the 8 children of each active parent (walked through a compacted
//      list) take their ops: Rp -> parent, Pa/P0/Pd -> palette index,
//      Rx/Ry/Rz -> the neighbour outside the sibling block.  A neighbour on the
//      +1 side is later in Morton order, so the reference reads its parent
//      (known, previous level).  A neighbour on the -1 side is earlier, on the
//      same level; its local index has one more 1-bit than the node's, so such
//      chains are at most three hops long and are resolved on the fly without
//      any ordering between threads.
//   3. the last level is written straight to HBM, 8 children (64 bytes) per
//      parent, with streaming 16-byte stores.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <vector>

#include "block_scan.cuh"
#include "csv_internal.h"

namespace csv {

// Threads per CTA (measured on mixed1024: 768 / 384 against 512 / 512 took the
// replay from 3.04 to 2.95 ms, and 320 threads at six CTAs per SM -- with the
// 32^3 variant's palette cache halved to fit -- from 2.68 to 2.61 ms: fewer warps
// of a brick wait at each phase barrier, more bricks are in flight per SM)
constexpr int kDecThreads = 320;      // the 32^3 variant: up to six CTAs per SM
constexpr int kDecThreadsBig = 768;   // the 64^3 variant: two CTAs per SM
constexpr int kDecThreadsNarrow = 512;  // the 64^3 variant with 8-bit node values: four CTAs per SM
// (8-bit node values halve the level arrays, so more 64^3 bricks fit per SM: mixed1024 replay 2.385 ->
// 2.29 ms at three CTAs of 512 threads, 2.27 at three of 640; with the compact rANS table below, four
// of 512 and the 32^3 variant at nine of 224: 2.196 -> 2.144 ms.  Four CTAs of 384 threads with the
// full table read through L1 instead measured no faster than two of 768)
// the 32^3 variant with 8-bit node values: nine CTAs per SM (seven of 288 threads with the full rANS
// table: mixed1024 replay 2.27 -> 2.19 ms)
constexpr int kDecThreadsSmallNarrow = 224;
template <class V, uint32_t KL>
__host__ __device__ constexpr int dec_threads() {
    return KL == 6 ? (sizeof(V) == 1 ? kDecThreadsNarrow : kDecThreadsBig)
                   : (sizeof(V) == 1 ? kDecThreadsSmallNarrow : kDecThreads);
}
template <class V, uint32_t KL>
__host__ __device__ constexpr int dec_ctas_per_sm() {
    return KL == 6 ? (sizeof(V) == 1 ? 4 : 2) : (sizeof(V) == 1 ? 9 : 6);
}
constexpr uint32_t kDecLevels = 6;       // parent levels 0..5 (a 64^3 brick has 7 levels)
constexpr uint32_t kPalCache = 1024;     // palettes up to this size are copied to shared memory
template <class V, uint32_t KL>
__host__ __device__ constexpr uint32_t pal_cache() { return sizeof(V) == 1 ? 256u : (KL == 6 ? kPalCache : 512u); }
constexpr uint32_t REC_MISSING = OP_RP | 8u;

// Node values of level l at val + voff(l): lvl_off rounded up to 8 entries (16 bytes for u16).
__host__ __device__ constexpr uint32_t lvl_off(uint32_t l) { return ((1u << (3 * l)) - 1) / 7; }
__host__ __device__ constexpr uint32_t voff(uint32_t l) { return (lvl_off(l) + 7) & ~7u; }
// Activity bitmask words of level l at mask + moff(l).
__host__ __device__ constexpr uint32_t mwords(uint32_t l) { return l < 2 ? 1u : (1u << (3 * l)) / 32; }
__host__ __device__ constexpr uint32_t moff(uint32_t l) { return l == 0 ? 0u : moff(l - 1) + mwords(l - 1); }
// Shared memory holds the node values of parent levels 0..KL-1 and the
// activity masks of all parent levels.  KL = 6: every level of a 64^3 brick
// (two CTAs per SM).  KL = 5: an eighth of the value space (six CTAs per SM);
// a 64^3 brick's level-5 values (its last parent level) then live in the CTA's
// global scratch, where they stay in L2.
constexpr uint32_t kSmallLevels = kSmallLod;
template <uint32_t KL>
struct LevelDims {
    static constexpr uint32_t val = voff(KL);            // 37456 for KL 6, 4688 for KL 5
    static constexpr uint32_t mask = moff(kDecLevels);   // 1172
};

// The 8-bit variants keep the rANS table compact in shared memory: a symbol byte per x (4 KB) and
// the 16 symbols' entries after it (an entry, symbol | freq << 4 | start << 17, depends only on the
// symbol, so this is exact for every table), one more dependent load per step for 12 KB less per CTA.
template <class V>
__host__ __device__ constexpr bool compact_lut() { return sizeof(V) == 1; }
constexpr uint32_t kLutCompactWords = kTot / 4 + 16;

template <class V, uint32_t KL>
struct DecShared {
    uint32_t lut[compact_lut<V>() ? kLutCompactWords : kTot];
    // During the rANS phase the level arrays (val, mask, pre: contiguous) are
    // idle: the brick's compressed stream is staged over them by one bulk
    // (TMA) copy when it fits (stage_cap bytes).
    alignas(16) V val[LevelDims<KL>::val];
    uint32_t mask[LevelDims<KL>::mask];
    uint16_t pre[LevelDims<KL>::mask];
    uint64_t pal[pal_cache<V, KL>()];
    uint32_t warp_sums[1024 / 32 + 1];
    BrickDesc br;
    csv_request req;
    uint32_t work, status;
    // the stream copy's bounded waits: rewait is set when the first wait gave up (one more wait before the
    // staging region is reused); drained when the second gave up too (the CTA decodes nothing more)
    uint32_t rewait, drained;
    alignas(8) uint64_t bar;  // mbarrier of the stream copy
};
template <class V, uint32_t KL>
__host__ __device__ constexpr uint32_t stage_cap() {
    return (uint32_t)(sizeof(V) * LevelDims<KL>::val + 6 * LevelDims<KL>::mask) & ~15u;
}
static_assert((sizeof(uint8_t) * LevelDims<kDecLevels>::val) % 16 == 0, "mask follows val without padding");
static_assert((sizeof(uint16_t) * LevelDims<kDecLevels>::val) % 16 == 0, "mask follows val without padding");
static_assert((sizeof(uint16_t) * LevelDims<kSmallLevels>::val) % 16 == 0, "mask follows val without padding");

// ---- bulk copy global -> shared with an mbarrier (cp.async.bulk, sm_90+)
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Issue one bulk copy of `bytes` (multiple of 16, 16-byte aligned ends) into shared memory.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
// Wait for the barrier phase `parity` to complete; gives up after a bounded number of polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t a = smem_addr(bar);
#pragma unroll 1
    for (uint32_t it = 0; it < (1u << 22); ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// ------------------------------------------------------------------ LUT
// findSymbol (brickDecoding.cpp:126-135) over the loaded 16-entry cumulative
// table, tabulated for all x in [0, 4096): symbol | freq << 4 | start << 17.
cudaError_t build_lut(const uint32_t* freq, const uint32_t* cum, uint32_t* h_lut) {
    for (uint32_t x = 0; x < kTot; ++x) {
        uint32_t s = 0;
        while (s + 1 < 16 && x >= cum[s + 1]) ++s;
        h_lut[x] = s | (freq[s] << 4) | (cum[s] << 17);
    }
    return cudaSuccess;
}

uint32_t lut_fast_mask(const uint32_t* h_lut, uint32_t n) {
    uint32_t m = 0;
    for (uint32_t t = 0; t < n && t < 32; ++t) {
        bool ok = true;
        for (uint32_t x = 0; x < kTot && ok; ++x) {
            const uint32_t e = h_lut[(size_t)t * kTot + x], f = (e >> 4) & 0x1FFFu, start = e >> 17;
            ok = start <= x && x - start < f;
        }
        if (ok) m |= 1u << t;
    }
    return m;
}

// One rANS decode step (ransDecodeSymbol, brickDecoding.cpp:137-151), totalFreq
// 4096 so % and / are a mask and a shift.  GLOBAL: enc is global memory (read
// through the non-coherent path); otherwise a generic pointer (shared staging).
template <bool GLOBAL = true, bool CLUT = false>
__device__ __forceinline__ uint32_t rans_step(uint32_t& x, uint32_t& pos, const uint8_t* __restrict__ enc,
                                              const uint32_t* __restrict__ lut) {
    uint32_t v = x & (kTot - 1);
    // CLUT: the compact table (symbol bytes, then the 16 entries)
    uint32_t e = CLUT ? lut[kTot / 4 + reinterpret_cast<const uint8_t*>(lut)[v]] : lut[v];
    uint32_t f = (e >> 4) & 0x1FFFu, st = e >> 17;
    x = f * (x >> kTotBits) + v - st;
    // renormalisation (the reference's while loop): in a well-formed stream it
    // reads at most two bytes, since after a step x >= f * 2^11 >= 2^11 and two
    // bytes lift that past 2^23; the loop only continues on malformed data
    if (x < kRansL && pos > 0) {
        x = (x << 8) | (GLOBAL ? __ldg(enc + (--pos)) : enc[--pos]);
        if (x < kRansL && pos > 0) {
            x = (x << 8) | (GLOBAL ? __ldg(enc + (--pos)) : enc[--pos]);
            while (x < kRansL && pos > 0) x = (x << 8) | (GLOBAL ? __ldg(enc + (--pos)) : enc[--pos]);
        }
    }
    return e & 15u;
}

// -------------------------------------------------------------- seek index
// The rANS step of the states pass (a checkpoint's state decoded again from the
// snapshot before it).  Same arithmetic as rans_step; both bytes
// a well-formed renormalisation can take are read before the state is known
// (their addresses depend only on pos), so the loads overlap the table lookup
// instead of following it on the chain.
__device__ __forceinline__ uint32_t index_step(uint32_t& x, uint32_t& pos, const uint8_t* __restrict__ enc,
                                               const uint32_t* lut) {
    const uint32_t b1 = __ldg(enc + (pos > 0 ? pos - 1 : 0));
    const uint32_t b2 = __ldg(enc + (pos > 1 ? pos - 2 : 0));
    const uint32_t v = x & (kTot - 1);
    const uint32_t e = __ldg(lut + v);
    x = ((e >> 4) & 0x1FFFu) * (x >> kTotBits) + v - (e >> 17);
    if (x < kRansL && pos > 0) {
        x = (x << 8) | b1;
        --pos;
        if (x < kRansL && pos > 0) {
            x = (x << 8) | b2;
            --pos;
            while (x < kRansL && pos > 0) x = (x << 8) | __ldg(enc + (--pos));  // malformed streams only
        }
    }
    return e & 15u;
}

// The seek index in three passes.  A brick's symbols form one dependent rANS
// chain, and the longest brick sets the time, so the per-symbol bookkeeping
// (Pd pairs, palette count, active children, ops per level, checkpoints) is
// taken off that chain:
//   1. index_symbols_kernel: one lane per brick runs the chain alone, writing
//      every symbol (packed nibbles) and the state before every kSnap-th one;
//   2. index_book_kernel: one warp per brick walks the nibbles 256 at a time:
//      which nibbles start ops (a Pd op's delta does not) is a two-state
//      automaton whose per-lane transfer functions compose in a warp scan; op,
//      palette and active counts are warp prefix sums; level boundaries
//      (level l+1 has 8 ops per active op of level l) are found by ballot; the
//      checkpoints before every S-th op get their symbol and palette index;
//   3. index_states_kernel: each checkpoint's (state, pos) is decoded again
//      from the snapshot before it (fewer than kSnap steps), all in parallel.
// The result equals the serial walk of the reference decoder
// (brickDecoding.hpp:174-242): the same checkpoints, op count, level starts and
// flags.
constexpr uint32_t kSnap = 32;  // symbols between state snapshots
static_assert(kSeedSymbols % kSnap == 0, "a sidecar's states fall on snapshots");

// Pass 1's chain step in two forms.
//
// ChainRef: ransDecodeSymbol and the renormalisation loop as the reference
// writes them (brickDecoding.cpp:137-151), for any table and start state.  The
// two bytes a well-formed renormalisation can take are loads at fixed offsets
// from a pointer to byte pos, issued (predicated on pos) before the state is
// known.
//
// ChainFast: for a well-formed table (every x lies in its symbol's range, so a
// step leaves x >= freq * 2^11 >= 2^11 when it began at x >= 2^23) and a chain
// that began at x >= 2^23.  Then a renormalisation takes one byte below 2^23
// and a second below 2^15 (x >= 2^27 after it), or stops at the stream's
// start: the reference's loop never needs a third byte, and the bits to take
// are min(want, 8 pos), shifted into x from a 64-bit buffer of the next stream
// bytes (next byte on top) by one funnel shift.  The buffer is fed from
// aligned 32-bit words walking down the stream (a stream starts 16-byte
// aligned), one word ahead of need, so no step waits on a byte load; it holds
// at least 32 bits at every second step.  Table form: (x - start) | symbol <<
// 12 | freq << 19, one shift or mask per field.
struct ChainRef {
    const uint8_t* q;
    uint32_t x, pos;
    const uint32_t* lut;  // symbol | freq << 4 | start << 17
    __device__ __forceinline__ void init(const uint8_t* enc, uint32_t x0, uint32_t pos0, const uint32_t* t) {
        q = enc + pos0;
        x = x0;
        pos = pos0;
        lut = t;
    }
    __device__ __forceinline__ uint32_t step() {
        const uint32_t b1 = pos > 0 ? (uint32_t)__ldg(q - 1) : 0u;
        const uint32_t b2 = pos > 1 ? (uint32_t)__ldg(q - 2) : 0u;
        const uint32_t v = x & (kTot - 1);
        const uint32_t e = lut[v];
        x = ((e >> 4) & 0x1FFFu) * (x >> kTotBits) + v - (e >> 17);
        // a second byte is taken exactly when x < 2^15, since (x << 8 | b1) < 2^23 then
        const bool n1 = x < kRansL && pos > 0, n2 = n1 && x < (kRansL >> 8) && pos > 1;
        const uint32_t c1 = (x << 8) | b1, c2 = (x << 16) | (b1 << 8) | b2;
        x = n2 ? c2 : (n1 ? c1 : x);
        const uint32_t nb = (n1 ? 1u : 0u) + (n2 ? 1u : 0u);
        pos -= nb;
        q -= nb;
        while (x < kRansL && pos > 0) {  // malformed streams only
            x = (x << 8) | __ldg(--q);
            --pos;
        }
        return e & 15u;
    }
    __device__ __forceinline__ void refill() {}
    __device__ __forceinline__ uint32_t where() const { return pos; }
};

struct ChainFast {
    const uint32_t* encw;  // the stream as aligned words
    uint32_t x, pos8;      // state and 8 x bytes left below the read position
    int32_t lo;            // lowest stream byte in bb (below 0: zero padding)
    uint64_t bb;           // the next bytes, next one in bits 63..56
    uint32_t nw;           // the word just below lo (0 below the stream)
    const uint32_t* lut;   // (x - start) | symbol << 12 | freq << 19
    __device__ __forceinline__ void init(const uint8_t* enc, uint32_t x0, uint32_t pos0, const uint32_t* t) {
        encw = reinterpret_cast<const uint32_t*>(enc);
        x = x0;
        pos8 = 8 * pos0;
        lut = t;
        bb = 0;
        lo = 0;
        nw = 0;
        if (pos0 == 0) return;
        // the word holding byte pos0 - 1 keeps its bytes below pos0 (c0 of them, on top), the word below follows
        const uint32_t a0 = (pos0 - 1) & ~3u, c0 = pos0 - a0;
        const uint32_t w0 = __ldg(encw + (a0 >> 2)) << (8 * (4 - c0));
        const uint32_t w1 = a0 >= 4 ? __ldg(encw + (a0 >> 2) - 1) : 0u;
        bb = ((uint64_t)w0 << 32) | ((uint64_t)w1 << (32 - 8 * c0));
        lo = (int32_t)a0 - 4;
        nw = lo >= 4 ? __ldg(encw + ((lo - 4) >> 2)) : 0u;
    }
    __device__ __forceinline__ uint32_t step() {
        const uint32_t e = lut[x & (kTot - 1)];
        x = (e >> 19) * (x >> kTotBits) + (e & (kTot - 1));
        const uint32_t want = x < (kRansL >> 8) ? 16u : (x < kRansL ? 8u : 0u);
        const uint32_t sh = min(want, pos8);
        x = __funnelshift_lc((uint32_t)(bb >> 32), x, sh);
        bb <<= sh;
        pos8 -= sh;
        return (e >> 12) & 15u;
    }
    // below 32 bits in the buffer: the prefetched word joins it, the next one is fetched
    __device__ __forceinline__ void refill() {
        const int32_t nbits = (int32_t)pos8 - 8 * lo;
        if (nbits < 32) {
            bb |= (uint64_t)nw << (32 - nbits);
            lo -= 4;
            nw = lo >= 4 ? __ldg(encw + ((lo - 4) >> 2)) : 0u;
        }
    }
    __device__ __forceinline__ uint32_t where() const { return pos8 >> 3; }
};

// Symbols [s0, s1) of one brick's chain (s0 a multiple of kSnap): packed
// nibbles to w (word s0 / 8 on), the state before every kSnap-th symbol to sn.
// The brick's first piece (s0 == 0) also takes the root nibble; returns false
// when the root's stop bit ends the brick there (its only nibble, the root, is
// in w[0]).
template <class Chain>
__device__ __forceinline__ bool index_walk(Chain& c, uint32_t s0, uint32_t s1, uint32_t* __restrict__ w,
                                           uint2* __restrict__ sn) {
    uint32_t k = s0 / 8;
    if (s0 == 0) {
        sn[0] = make_uint2(c.x, c.where());
        const uint32_t root = c.step();
        c.refill();
        if (root & 1u) {
            w[0] = root;
            return false;
        }
        // word 0: the root and symbols 1..7
        uint32_t word = root;
        for (uint32_t i = 1; i < 8 && i < s1; ++i) {
            word |= c.step() << (4 * i);
            c.refill();
        }
        w[0] = word;
        k = 1;
    }
    // whole words of 8 symbols (a snapshot before every 4th: symbol 32m)
    for (; 8 * k + 8 <= s1; ++k) {
        if ((k & 3u) == 0) sn[k >> 2] = make_uint2(c.x, c.where());
        uint32_t wd = 0;
#pragma unroll
        for (uint32_t j = 0; j < 8; ++j) {
            wd |= c.step() << (4 * j);
            if (j & 1u) c.refill();
        }
        w[k] = wd;
    }
    if (8 * k < s1) {  // the last, partial word
        if ((k & 3u) == 0) sn[k >> 2] = make_uint2(c.x, c.where());
        uint32_t wd = 0;
        for (uint32_t j = 0; 8 * k + j < s1; ++j) {
            wd |= c.step() << (4 * j);
            c.refill();
        }
        w[k] = wd;
    }
    return true;
}

// A table in ChainFast's form from the usual one (symbol | freq << 4 | start << 17).
__device__ __forceinline__ uint32_t fast_entry(uint32_t e, uint32_t i) {
    return ((i - (e >> 17)) & (kTot - 1)) | ((e & 15u) << 12) | (((e >> 4) & 0x1FFFu) << 19);
}

__global__ void __launch_bounds__(256) index_fast_lut_kernel(const uint32_t* __restrict__ g_lut, uint32_t n,
                                                            uint32_t* __restrict__ g_lutf) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) g_lutf[i] = fast_entry(g_lut[i], i & (kTot - 1));
}

// One brick's chain, or the piece [s0, s1) of it, from the state (x, pos);
// ChainFast when `fast` (model 0's table from shared memory, the others' from
// g_lutf), else ChainRef on the usual tables.  x and pos come back as the
// state after the last symbol.
__device__ __forceinline__ bool index_run(const uint8_t* enc, uint32_t& x, uint32_t& pos, const uint32_t* lut0f,
                                          const uint32_t* __restrict__ g_lutf, const uint32_t* __restrict__ g_lut,
                                          uint32_t model, bool fast, uint32_t s0, uint32_t s1, uint32_t* w,
                                          uint2* sn) {
    bool more;
    if (fast && model == 0) {
        ChainFast c;
        c.init(enc, x, pos, lut0f);
        more = index_walk(c, s0, s1, w, sn);
        x = c.x;
        pos = c.where();
    } else if (fast) {
        ChainFast c;
        c.init(enc, x, pos, g_lutf + (size_t)model * kTot);
        more = index_walk(c, s0, s1, w, sn);
        x = c.x;
        pos = c.where();
    } else {
        ChainRef c;
        c.init(enc, x, pos, g_lut + (size_t)model * kTot);
        more = index_walk(c, s0, s1, w, sn);
        x = c.x;
        pos = c.where();
    }
    return more;
}

// Model 0's table in ChainFast's form, in shared memory.
__device__ __forceinline__ void load_fast_lut(uint32_t* lut0f, const uint32_t* __restrict__ g_lut) {
    for (uint32_t i = threadIdx.x; i < kTot; i += blockDim.x) lut0f[i] = fast_entry(g_lut[i], i);
}

// The bricks' outcome of pass 1 that needs no bookkeeping: a brick with no
// chain to index (header too short, no symbols, the root's stop bit, or one
// level) gets no ops and its flags now; write_desc false leaves the
// descriptors as they are (the chain alone is wanted).
__device__ __forceinline__ void index_finish(BrickDesc* bricks, uint32_t bi, const BrickDesc& br, bool go,
                                             uint32_t flags, uint8_t* chain, bool write_desc) {
    chain[bi] = go ? 1 : 0;
    if (!go && write_desc) {
        BrickDesc& o = bricks[bi];
        o.n_ops = 0;
        o.flags = (br.flags & ~BF_STATUS_MASK) | flags;
#pragma unroll
        for (int k = 0; k < 8; ++k) o.level_start[k] = 0;
    }
}

__global__ void __launch_bounds__(128) index_symbols_kernel(BrickDesc* __restrict__ bricks, uint32_t nb,
                                                           const uint8_t* __restrict__ enc_pool,
                                                           const uint32_t* __restrict__ g_lut,
                                                           const uint32_t* __restrict__ g_lutf, uint32_t n_models,
                                                           uint32_t fast_models, uint32_t lanes,
                                                           const uint32_t* __restrict__ order,
                                                           const uint64_t* __restrict__ nib_off,
                                                           const uint64_t* __restrict__ snap_off,
                                                           uint32_t* __restrict__ nib, uint2* __restrict__ snap,
                                                           uint8_t* __restrict__ chain, uint32_t L, bool write_desc) {
    __shared__ uint32_t lut0[kTot];
    load_fast_lut(lut0, g_lut);
    __syncthreads();
    // The lanes of a warp take `lanes` bricks of similar length (order: longest
    // first), so that a warp's chains end together, and one warp instruction
    // steps them all: the longest chain then runs at its own latency instead of
    // sharing a scheduler's issue slots with the other long chains.
    const uint32_t lane = threadIdx.x & 31;
    if (lane >= lanes) return;
    const uint32_t slot = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * lanes + lane;
    if (slot >= nb) return;
    const uint32_t bi = order[slot];
    const BrickDesc br = bricks[bi];
    const uint32_t model = min((br.flags >> BF_MODEL_SHIFT) & 255u, n_models - 1);
    uint32_t flags = 0;
    bool go = false;
    if (br.E < 4 || br.nsym == 0) {
        flags = BF_TRUNCATED;
    } else {
        const uint8_t* enc = enc_pool + br.enc_off;
        uint32_t pos = br.E - 4;
        uint32_t x = ((uint32_t)enc[br.E - 1] << 24) | ((uint32_t)enc[br.E - 2] << 16) |
                     ((uint32_t)enc[br.E - 3] << 8) | enc[br.E - 4];
        const bool fast = x >= kRansL && model < 32 && ((fast_models >> model) & 1u);
        if (index_run(enc, x, pos, lut0, g_lutf, g_lut, model, fast, 0, br.nsym, nib + nib_off[bi],
                      snap + snap_off[bi]))
            go = L >= 2;
        else
            flags = BF_UNIFORM;  // the whole brick is palette[0]: nothing more to index
    }
    index_finish(bricks, bi, br, go, flags, chain, write_desc);
}

// Composition of the per-lane automaton transfers (bit 0: the state after, from
// state 0; bit 1: from state 1): apply `first`, then `then`.
__device__ __forceinline__ uint32_t compose2(uint32_t first, uint32_t then) {
    const uint32_t a0 = (then >> (first & 1u)) & 1u, a1 = (then >> ((first >> 1) & 1u)) & 1u;
    return a0 | (a1 << 1);
}

__global__ void __launch_bounds__(128) index_book_kernel(BrickDesc* __restrict__ bricks, uint32_t nb,
                                                        const uint32_t* __restrict__ nib,
                                                        const uint64_t* __restrict__ nib_off,
                                                        const uint8_t* __restrict__ chain, Checkpoint* __restrict__ ck,
                                                        uint32_t* __restrict__ n_ck_out, uint32_t L, uint32_t S) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t bi = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (bi >= nb) return;
    if (!chain[bi]) {
        if (lane == 0) n_ck_out[bi] = 0;
        return;
    }
    const uint32_t FULL = 0xFFFFFFFFu;
    const BrickDesc br = bricks[bi];
    const uint32_t* w = nib + nib_off[bi];
    const uint32_t nsym = br.nsym;
    // automaton state before the next chunk: 0 = the next nibble starts an op, 1 = it is a Pd op's delta
    uint32_t st_in = 0;
    uint32_t op_base = 0, ip_base = 0, act_base = 0;  // ops, Pa ops and active ops before the chunk
    uint32_t lvl = 0, b_next = 8, act_cur = 0;        // level lvl+1 ends before op b_next; actives before its start
    uint32_t ls[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    uint32_t end_ops = 0xFFFFFFFFu;
    bool done = false;
    // each chunk's nibble word is loaded one chunk ahead
    uint32_t word_next = 8 * lane < nsym ? w[lane] : 0u;
    for (uint32_t c0 = 0; c0 < nsym && !done; c0 += 256) {
        const uint32_t base = c0 + 8 * lane;
        const uint32_t word = word_next;
        word_next = base + 256 < nsym ? w[(base + 256) >> 3] : 0u;
        // The lane's eight nibbles as nibble-spaced masks (bit 4k: symbol base + k): V its symbols,
        // [max(base, 1), min(base + 8, nsym)) -- symbol 0 is the root; PD the Pd codes, PA the Pa
        // codes, ACT the nibbles whose stop bit is clear (an op there leaves its node active).
        const uint32_t hi = nsym > base ? min(nsym - base, 8u) : 0u;
        const uint32_t V = (hi == 8 ? 0x11111111u : (0x11111111u & ((1u << (4 * hi)) - 1u))) & (base == 0 ? ~1u : ~0u);
        const uint32_t codes = (word >> 1) & 0x77777777u;
        auto eq = [&](uint32_t K) {  // nibbles whose 3-bit code is K
            const uint32_t x = codes ^ (K * 0x11111111u);
            return ~(x | (x >> 1) | (x >> 2)) & 0x11111111u;
        };
        const uint32_t PD = eq(OP_PD) & V, PA = eq(OP_PA) & V, ACT = ~word & 0x11111111u & V;
        // which nibbles start ops, from entry state 0 and from entry state 1 (1: the first nibble is
        // a Pd op's delta), and the state after the lane's nibbles: the automaton unrolled
        uint32_t s0 = 0, s1 = 1, S0 = 0, S1 = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint32_t valid = (V >> (4 * k)) & 1u, pd = (PD >> (4 * k)) & 1u;
            S0 |= (valid & (s0 ^ 1u)) << (4 * k);
            S1 |= (valid & (s1 ^ 1u)) << (4 * k);
            s0 = valid ? ((s0 ^ 1u) & pd) : s0;
            s1 = valid ? ((s1 ^ 1u) & pd) : s1;
        }
        uint32_t inc = s0 | (s1 << 1);
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(FULL, inc, d);
            if (lane >= (uint32_t)d) inc = compose2(y, inc);
        }
        uint32_t excl = __shfl_up_sync(FULL, inc, 1);
        if (lane == 0) excl = 2u;  // identity
        const uint32_t entry = (excl >> st_in) & 1u;
        const uint32_t exit_all = (__shfl_sync(FULL, inc, 31) >> st_in) & 1u;
        // this lane's op starts, Pa ops and active ops
        const uint32_t starts = entry ? S1 : S0;
        const uint32_t np = __popc(starts), npa = __popc(starts & PA), nact = __popc(starts & ACT);
        const uint32_t packed = np | (npa << 10) | (nact << 20);
        uint32_t pin = packed;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(FULL, pin, d);
            if (lane >= (uint32_t)d) pin += y;
        }
        const uint32_t pex = pin - packed, ptot = __shfl_sync(FULL, pin, 31);
        const uint32_t my_op = op_base + (pex & 1023u), my_ip = ip_base + ((pex >> 10) & 1023u),
                       my_act = act_base + (pex >> 20);
        const uint32_t tot_np = ptot & 1023u;
        // level boundaries among this chunk's op starts
        while (!done && b_next < op_base + tot_np) {
            const bool has = my_op <= b_next && b_next < my_op + np;
            const uint32_t src = __ffs(__ballot_sync(FULL, has)) - 1;
            uint32_t ap = 0;
            if (has) {  // actives among the ops before b_next: the lane's first b_next - my_op starts
                uint32_t rest = starts;
                for (uint32_t t = my_op; t < b_next; ++t) rest &= rest - 1u;
                ap = my_act + __popc((starts ^ rest) & ACT);
            }
            ap = __shfl_sync(FULL, ap, src);
            ++lvl;
            ls[lvl] = b_next;
            const uint32_t need = 8 * (ap - act_cur);
            if (lvl + 1 >= L || need == 0) {
                done = true;
                end_ops = b_next;
                break;
            }
            act_cur = ap;
            b_next += need;
        }
        // checkpoints before every S-th op of the tree (at most one per lane when S > 8)
        for (uint32_t j = (my_op + S - 1) / S * S; j < my_op + np && j < end_ops; j += S) {
            uint32_t rest = starts;  // the (j - my_op)-th start of the lane is rest's lowest bit
            for (uint32_t t = my_op; t < j; ++t) rest &= rest - 1u;
            const uint32_t p = __ffs(rest) - 1;
            const uint32_t ipr = my_ip + __popc(starts & PA & ((1u << p) - 1u));
            const uint32_t c = j / S;
            if (c < br.ck_cap) ck[br.ck_off + c] = Checkpoint{0u, 0u, base + (p >> 2), ipr};
        }
        op_base += tot_np;
        ip_base += (ptot >> 10) & 1023u;
        act_base += ptot >> 20;
        st_in = exit_all;
    }
    uint32_t flags = 0, ops;
    if (done) {
        ops = end_ops;
    } else {
        // every symbol read: the level ending at the last op may still close the tree, unless that op is
        // a Pd op without its delta nibble (the walk counts it, and stops there truncated)
        ops = op_base;
        if (b_next == op_base && st_in == 0) {
            ++lvl;
            ls[lvl] = b_next;
            const uint32_t need = 8 * (act_base - act_cur);
            if (!(lvl + 1 >= L || need == 0)) flags = BF_TRUNCATED;
        } else {
            flags = BF_TRUNCATED;  // the stream ends inside the level structure
        }
    }
    // a checkpoint before every S-th op below ops (those past ck_cap are not stored)
    const uint32_t n_ck = (ops + S - 1) / S;
    if (lane == 0) {
        BrickDesc& o = bricks[bi];
        o.n_ops = ops;
        if (n_ck > br.ck_cap) flags |= BF_TRUNCATED;
        o.flags = (br.flags & ~BF_STATUS_MASK) | flags;
        for (uint32_t k = 0; k < 8; ++k) o.level_start[k] = k <= lvl ? ls[k] : ops;
        n_ck_out[bi] = min(n_ck, br.ck_cap);
    }
}

// One block of 512 threads per brick: its threads share the brick's checkpoints,
// so a long brick's re-decodes spread over the block instead of one warp (the
// table is read through L1: the decodes are short).
__global__ void __launch_bounds__(512) index_states_kernel(const BrickDesc* __restrict__ bricks, uint32_t nb,
                                                          const uint8_t* __restrict__ enc_pool,
                                                          const uint32_t* __restrict__ g_lut, uint32_t n_models,
                                                          const uint64_t* __restrict__ snap_off,
                                                          const uint2* __restrict__ snap,
                                                          const uint32_t* __restrict__ n_ck, Checkpoint* __restrict__ ck) {
    const uint32_t bi = blockIdx.x;
    if (bi >= nb) return;
    const uint32_t n = n_ck[bi];
    if (n == 0) return;
    const BrickDesc br = bricks[bi];
    const uint32_t model = min((br.flags >> BF_MODEL_SHIFT) & 255u, n_models - 1);
    const uint8_t* enc = enc_pool + br.enc_off;
    const uint2* sn = snap + snap_off[bi];
    const uint32_t* lut = g_lut + (size_t)model * kTot;
    for (uint32_t c = threadIdx.x; c < n; c += blockDim.x) {
        Checkpoint& k = ck[br.ck_off + c];
        const uint32_t s = k.sym, j = s / kSnap;
        const uint2 z = sn[j];
        uint32_t x = z.x, pos = z.y;
        for (uint32_t t = j * kSnap; t < s; ++t) index_step(x, pos, enc, lut);
        k.state = x;
        k.pos = pos;
    }
}

// Pass 1 from a seek-index sidecar: the state before every kSeedSymbols-th
// symbol of each brick is given, so the chain runs as independent pieces, one
// lane per piece.  A piece checks that it ends in the state given for the next
// one, and the first piece that its state is the stream header's: by induction
// every piece then ran from the true state, and the nibbles and snapshots are
// the serial pass's.  Any difference (a sidecar of another image, or damaged)
// counts in *bad and the host discards the result.  A brick the sidecar gives
// no states for (seed.y == kFromHeader) is one piece, run from its header.
constexpr uint32_t kFromHeader = 0xFFFFFFFFu;
__global__ void __launch_bounds__(128) index_seeded_kernel(BrickDesc* __restrict__ bricks, uint32_t nb,
                                                          const uint8_t* __restrict__ enc_pool,
                                                          const uint32_t* __restrict__ g_lut,
                                                          const uint32_t* __restrict__ g_lutf, uint32_t n_models,
                                                          uint32_t fast_models, const uint32_t* __restrict__ piece_base,
                                                          const uint2* __restrict__ seed, uint32_t n_pieces,
                                                          const uint64_t* __restrict__ nib_off,
                                                          const uint64_t* __restrict__ snap_off,
                                                          uint32_t* __restrict__ nib, uint2* __restrict__ snap,
                                                          uint8_t* __restrict__ chain, uint32_t L,
                                                          uint32_t* __restrict__ bad) {
    __shared__ uint32_t lut0[kTot];
    load_fast_lut(lut0, g_lut);
    __syncthreads();
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n_pieces) return;
    // the piece's brick: the last bi with piece_base[bi] <= p (piece_base[0] = 0, piece_base[nb] = n_pieces)
    uint32_t lo = 0, hi = nb;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (piece_base[mid] <= p) lo = mid;
        else hi = mid;
    }
    const uint32_t bi = lo, k = p - piece_base[bi], n_here = piece_base[bi + 1] - piece_base[bi];
    const BrickDesc br = bricks[bi];
    if (br.E < 4 || br.nsym == 0) {
        if (k == 0) index_finish(bricks, bi, br, false, BF_TRUNCATED, chain, true);
        return;
    }
    const uint32_t model = min((br.flags >> BF_MODEL_SHIFT) & 255u, n_models - 1);
    const uint8_t* enc = enc_pool + br.enc_off;
    const uint32_t x0 = ((uint32_t)enc[br.E - 1] << 24) | ((uint32_t)enc[br.E - 2] << 16) |
                        ((uint32_t)enc[br.E - 3] << 8) | enc[br.E - 4];
    // FAST depends on the chain's true start (the header), as in the serial pass
    const bool fast = x0 >= kRansL && model < 32 && ((fast_models >> model) & 1u);
    const uint2 sd = seed[p];
    uint32_t x = x0, pos = br.E - 4, s0 = 0, s1 = br.nsym;
    if (sd.y == kFromHeader) {
        if (k != 0 || n_here != 1) {
            atomicAdd(bad, 1u);
            return;
        }
    } else {
        s0 = k * kSeedSymbols;
        s1 = min(s0 + kSeedSymbols, br.nsym);
        // a state past the stream's end would read outside it: refused before any step
        if (s0 >= br.nsym || sd.y > br.E - 4 || (k == 0 && (sd.x != x0 || sd.y != br.E - 4))) {
            atomicAdd(bad, 1u);
            return;
        }
        x = sd.x;
        pos = sd.y;
    }
    const bool more =
        index_run(enc, x, pos, lut0, g_lutf, g_lut, model, fast, s0, s1, nib + nib_off[bi], snap + snap_off[bi]);
    if (k == 0) index_finish(bricks, bi, br, more && L >= 2, more ? 0u : BF_UNIFORM, chain, true);
    if (more && k + 1 < n_here) {
        const uint2 nx = seed[p + 1];
        if (nx.x != x || nx.y != pos) atomicAdd(bad, 1u);
    }
}

// The states a sidecar keeps, from pass 1's snapshots: for a brick with a chain,
// the state before symbols 0, kSeedSymbols, 2 kSeedSymbols, ... (one warp per brick).
__global__ void __launch_bounds__(128) index_seeds_gather_kernel(const BrickDesc* __restrict__ bricks, uint32_t nb,
                                                                const uint8_t* __restrict__ chain,
                                                                const uint32_t* __restrict__ seed_base,
                                                                const uint64_t* __restrict__ snap_off,
                                                                const uint2* __restrict__ snap,
                                                                uint2* __restrict__ seeds) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t bi = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (bi >= nb || !chain[bi]) return;
    const uint32_t n = seed_base[bi + 1] - seed_base[bi];
    for (uint32_t k = lane; k < n; k += 32)
        seeds[seed_base[bi] + k] = snap[snap_off[bi] + (uint64_t)k * (kSeedSymbols / kSnap)];
}

namespace {
// Device temporaries of the index passes: per brick its nibble words and its snapshots.
struct IndexTemps {
    uint32_t* nib = nullptr;
    uint2* snap = nullptr;
    uint64_t* off = nullptr;  // nib_off[nb] | snap_off[nb]
    uint32_t* order = nullptr;  // bricks by nSymbols, longest first
    uint8_t* chain = nullptr;
    uint32_t* nck = nullptr;
    uint32_t* bad = nullptr;
    uint32_t* lutf = nullptr;  // every model's table in ChainFast's form
};

cudaError_t index_alloc(const DeviceDataset& ds, cudaStream_t st, IndexTemps& t) {
    const uint32_t nb = ds.nb;
    std::vector<uint64_t> off(2 * (size_t)nb);
    uint64_t words = 0, snaps = 0;
    for (uint32_t i = 0; i < nb; ++i) {
        const uint64_t ns = ds.h_cost ? ds.h_cost[i] : ds.max_nsym;
        off[i] = words;
        off[nb + i] = snaps;
        words += ns / 8 + 1;
        snaps += ns / kSnap + 1;
    }
    std::vector<uint32_t> order(nb);
    for (uint32_t i = 0; i < nb; ++i) order[i] = i;
    if (ds.h_cost)
        std::stable_sort(order.begin(), order.end(),
                         [&](uint32_t a, uint32_t b) { return ds.h_cost[a] > ds.h_cost[b]; });
    cudaError_t e = tmp_alloc((void**)&t.nib, words * 4, ds.pool, st);
    if (e == cudaSuccess) e = tmp_alloc((void**)&t.snap, snaps * 8, ds.pool, st);
    if (e == cudaSuccess) e = tmp_alloc((void**)&t.off, off.size() * 8, ds.pool, st);
    if (e == cudaSuccess) e = tmp_alloc((void**)&t.order, (size_t)nb * 4, ds.pool, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(t.order, order.data(), (size_t)nb * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = tmp_alloc((void**)&t.chain, nb, ds.pool, st);
    if (e == cudaSuccess) e = tmp_alloc((void**)&t.nck, (size_t)nb * 4, ds.pool, st);
    if (e == cudaSuccess) e = tmp_alloc((void**)&t.bad, 4, ds.pool, st);
    const uint32_t nm = ds.n_models ? ds.n_models : 1u;
    if (e == cudaSuccess) e = tmp_alloc((void**)&t.lutf, (size_t)nm * kTot * 4, ds.pool, st);
    if (e == cudaSuccess) {
        index_fast_lut_kernel<<<(nm * kTot + 255) / 256, 256, 0, st>>>(ds.d_lut, nm * kTot, t.lutf);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(t.bad, 0, 4, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(t.off, off.data(), off.size() * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // the host offsets are released on return
    return e;
}

void index_free(IndexTemps& t, cudaStream_t st) {
    cudaFreeAsync(t.nib, st);
    cudaFreeAsync(t.snap, st);
    cudaFreeAsync(t.off, st);
    cudaFreeAsync(t.order, st);
    cudaFreeAsync(t.chain, st);
    cudaFreeAsync(t.nck, st);
    cudaFreeAsync(t.bad, st);
    cudaFreeAsync(t.lutf, st);
    t = IndexTemps();
}

// pass 1 from the stream headers: four bricks per warp, four warps per block.
// (Measured on the 2048 bricks of a 1024 x 1024 x 512 volume of 64^3 bricks,
// longest 126k symbols: one brick per warp 10.4 ms, its warps sharing the
// schedulers' issue slots; 32 per warp 15.8 ms, each step slowed by 32 lanes'
// scattered byte loads and table bank conflicts.)
void index_pass1_serial(const DeviceDataset& ds, const IndexTemps& t, cudaStream_t st, bool write_desc) {
    const uint32_t nb = ds.nb;
    constexpr uint32_t lanes = 4;
    const uint32_t per_block = 4 * lanes;
    const uint32_t nm = ds.n_models ? ds.n_models : 1u;
    index_symbols_kernel<<<(nb + per_block - 1) / per_block, 128, 0, st>>>(
        ds.d_bricks, nb, ds.d_enc, ds.d_lut, t.lutf, nm, ds.fast_models, lanes, t.order, t.off, t.off + nb, t.nib,
        t.snap, t.chain, ds.L, write_desc);
}
}  // namespace

cudaError_t launch_build_index(DeviceDataset& ds, cudaStream_t st, const IndexSeeds* seeds, bool* rejected) {
    if (rejected) *rejected = false;
    if (ds.nb == 0) return cudaSuccess;
    const uint32_t nb = ds.nb;
    const uint32_t nm = ds.n_models ? ds.n_models : 1u;
    IndexTemps t;
    uint32_t* d_base = nullptr;
    uint2* d_seed = nullptr;
    cudaError_t e = index_alloc(ds, st, t);
    if (e == cudaSuccess && seeds) {
        const uint32_t n_pieces = seeds->piece_base.back();
        e = tmp_alloc((void**)&d_base, 4 * seeds->piece_base.size(), ds.pool, st);
        if (e == cudaSuccess) e = tmp_alloc((void**)&d_seed, 8 * std::max<size_t>(1, seeds->seed.size()), ds.pool, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_base, seeds->piece_base.data(), 4 * seeds->piece_base.size(),
                                cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess && !seeds->seed.empty())
            e = cudaMemcpyAsync(d_seed, seeds->seed.data(), 8 * seeds->seed.size(), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) {
            index_seeded_kernel<<<(n_pieces + 127) / 128, 128, 0, st>>>(
                ds.d_bricks, nb, ds.d_enc, ds.d_lut, t.lutf, nm, ds.fast_models, d_base, d_seed, n_pieces, t.off,
                t.off + nb, t.nib, t.snap, t.chain, ds.L, t.bad);
            e = cudaGetLastError();
        }
        // the bookkeeping passes run only on a chain every piece confirmed (an unconfirmed
        // piece may have left snapshots that the states pass would follow outside a stream)
        uint32_t h_bad = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&h_bad, t.bad, 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e == cudaSuccess && h_bad) {
            if (rejected) *rejected = true;
            cudaFreeAsync(d_base, st);
            cudaFreeAsync(d_seed, st);
            index_free(t, st);
            return cudaSuccess;
        }
    } else if (e == cudaSuccess) {
        index_pass1_serial(ds, t, st, true);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        index_book_kernel<<<(nb + 3) / 4, 128, 0, st>>>(ds.d_bricks, nb, t.nib, t.off, t.chain, ds.d_ck, t.nck, ds.L,
                                                       ds.S);
        index_states_kernel<<<nb, 512, 0, st>>>(ds.d_bricks, nb, ds.d_enc, ds.d_lut, nm, t.off + nb,
                                                         t.snap, t.nck, ds.d_ck);
        e = cudaGetLastError();
    }
    cudaFreeAsync(d_base, st);
    cudaFreeAsync(d_seed, st);
    index_free(t, st);
    return e;
}

cudaError_t index_seeds_of(const DeviceDataset& ds, cudaStream_t st, std::vector<uint32_t>& n_seeds,
                           std::vector<uint2>& seeds) {
    n_seeds.assign(ds.nb, 0);
    seeds.clear();
    if (ds.nb == 0) return cudaSuccess;
    const uint32_t nb = ds.nb;
    IndexTemps t;
    uint32_t* d_base = nullptr;
    uint2* d_seeds = nullptr;
    std::vector<uint8_t> chain(nb);
    std::vector<BrickDesc> desc(nb);
    cudaError_t e = index_alloc(ds, st, t);
    if (e == cudaSuccess) {
        index_pass1_serial(ds, t, st, false);  // the dataset's descriptors stay as they are
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(chain.data(), t.chain, nb, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(desc.data(), ds.d_bricks, sizeof(BrickDesc) * nb, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    std::vector<uint32_t> base(nb + 1, 0);
    if (e == cudaSuccess) {
        for (uint32_t i = 0; i < nb; ++i) {
            n_seeds[i] = chain[i] ? (desc[i].nsym + kSeedSymbols - 1) / kSeedSymbols : 0u;
            base[i + 1] = base[i] + n_seeds[i];
        }
        seeds.resize(base[nb]);
        e = tmp_alloc((void**)&d_base, 4ull * (nb + 1), ds.pool, st);
        if (e == cudaSuccess) e = tmp_alloc((void**)&d_seeds, 8ull * std::max<uint32_t>(1, base[nb]), ds.pool, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_base, base.data(), 4ull * (nb + 1), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) {
            index_seeds_gather_kernel<<<(nb + 3) / 4, 128, 0, st>>>(ds.d_bricks, nb, t.chain, d_base, t.off + nb,
                                                                   t.snap, d_seeds);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess && base[nb])
            e = cudaMemcpyAsync(seeds.data(), d_seeds, 8ull * base[nb], cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    cudaFreeAsync(d_base, st);
    cudaFreeAsync(d_seeds, st);
    index_free(t, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e;
}

// ------------------------------------------------------------ decode kernel
struct DecodeArgs {
    const BrickDesc* bricks;
    const uint64_t* pal;
    const uint8_t* enc;
    const Checkpoint* ck;
    const uint32_t* lut;
    const csv_request* reqs;
    uint64_t* out;
    uint32_t* status;
    uint8_t* scratch;
    uint64_t scratch_per_cta;
    uint32_t* queue;
    uint32_t nb, L, S, n;   // n: queue length (requests, or entries of order)
    uint32_t n_reqs;        // requests at reqs (and statuses at status)
    const uint32_t* order;  // optional processing order: queue slot -> request
    const uint32_t* n_dev;  // optional device-resident queue length (at most n)
    uint32_t stage_cap;     // largest stream staged in shared memory (0: never)
    uint32_t n_models;      // LUTs at lut, kTot entries each
};

__device__ __forceinline__ void st_cs_v2(uint64_t* p, uint64_t a, uint64_t b) {
    asm volatile("st.global.cs.v2.u64 [%0], {%1, %2};" ::"l"(p), "l"(a), "l"(b) : "memory");
}
// One 32-byte store (sm_100's 256-bit global store; p 32-byte aligned), streaming.
__device__ __forceinline__ void st_cs_v4(uint64_t* p, uint64_t a, uint64_t b, uint64_t c, uint64_t d) {
    asm volatile("st.global.cs.v4.u64 [%0], {%1, %2, %3, %4};" ::"l"(p), "l"(a), "l"(b), "l"(c), "l"(d) : "memory");
}

// Writes `cnt` copies of `v` at out[0..cnt) (out 8-byte aligned).
__device__ void fill_labels(uint64_t* out, uint64_t cnt, uint64_t v) {
    uint64_t start = 0;
    if (((uintptr_t)out & 15) && cnt) {
        if (threadIdx.x == 0) out[0] = v;
        start = 1;
    }
    uint64_t pairs = (cnt - start) / 2;
    for (uint64_t i = threadIdx.x; i < pairs; i += blockDim.x) st_cs_v2(out + start + 2 * i, v, v);
    if (((cnt - start) & 1) && threadIdx.x == 0) out[cnt - 1] = v;
}

// Eight labels of one parent (64 bytes) at o8.
__device__ __forceinline__ void store8(uint64_t* o8, const uint64_t* lab, bool vec) {
    if (vec) {
#pragma unroll
        for (int c = 0; c < 8; c += 2) st_cs_v2(o8 + c, lab[c], lab[c + 1]);
    } else {
#pragma unroll
        for (int c = 0; c < 8; ++c) o8[c] = lab[c];
    }
}

// The parent level as the resolver sees it.
template <class V>
struct LevelView {
    const V* val;           // node values of the parent level
    const uint32_t* mask;   // activity bits of the parent level
    const uint16_t* pre;    // active nodes before each mask word
    const uint32_t* rec;    // op records of the brick
    uint32_t o;             // first op of the child level
    uint32_t n_rec;         // records available
};

template <class V>
__device__ __forceinline__ uint32_t get_rec(const LevelView<V>& v, uint32_t idx) {
    return idx < v.n_rec ? v.rec[idx] : REC_MISSING;
}
// The 8 records of the r-th active parent.  In a complete brick o is a sum of
// multiples of 8, so the group is 32-byte aligned and read as two vectors; a
// truncated brick (o arbitrary, records missing) takes the guarded scalar path.
template <class V>
__device__ __forceinline__ void get_rec8(const LevelView<V>& v, uint32_t r, uint32_t rec[8]) {
    const uint32_t i0 = v.o + 8 * r;
    if ((i0 & 7u) == 0 && i0 + 8 <= v.n_rec) {
        const uint4* p = reinterpret_cast<const uint4*>(v.rec + i0);
        const uint4 a = p[0], b = p[1];
        rec[0] = a.x; rec[1] = a.y; rec[2] = a.z; rec[3] = a.w;
        rec[4] = b.x; rec[5] = b.y; rec[6] = b.z; rec[7] = b.w;
    } else {
#pragma unroll
        for (uint32_t c = 0; c < 8; ++c) rec[c] = get_rec(v, i0 + c);
    }
}
// rank of an active parent-level node q (its children's ops start at o + 8 * rank)
template <class V>
__device__ __forceinline__ uint32_t rank_of(const LevelView<V>& v, uint32_t q) {
    return v.pre[q >> 5] + __popc(v.mask[q >> 5] & ((1u << (q & 31)) - 1u));
}
template <class V>
__device__ __forceinline__ bool is_active(const LevelView<V>& v, uint32_t q) {
    return (v.mask[q >> 5] >> (q & 31)) & 1u;
}

// Value (palette index) of node n on level lc whose op record is `rec`; the
// parent of n is active.  Follows getNeighborValue (brickDecoding.cpp:77-124,
// decode.wgsl:247-306) with the output array replaced by node values: the -1
// neighbour is read as a node of the same level, the +1 neighbour through its
// parent.  A neighbour outside the brick reads the reference's "parent slot",
// which for child c > 0 already holds child 0's value (slot aliasing of
// coarseNodeToOutputIndex); malformed streams only.  Morton indices strictly
// decrease along a chain, so it terminates; the iteration cap only guards
// against a corrupt seek index.  Sets *bad on a capped chain.
template <class V>
__device__ __forceinline__ uint32_t resolve(const LevelView<V>& v, uint32_t rec, uint32_t n, uint32_t lc, bool* bad) {
    const uint32_t lvlmask = (1u << (3 * lc)) - 1u;
#pragma unroll 1
    for (int hop = 0; hop < 4096; ++hop) {
        const uint32_t code = rec & 7u;
        if (code >= OP_PA) return rec >> REC_PIDX_SHIFT;
        if (code == OP_RP) return v.val[n >> 3];
        const uint32_t a = code - 1;
        const uint32_t m = (0x09249249u << a) & lvlmask;
        const uint32_t bit = 1u << a;
        if (n & bit) {
            if ((n & m) != m) return v.val[((((n | ~m) + bit) & m) | (n & ~m)) >> 3];
        } else if ((n & m) != 0) {
            const uint32_t N = (((n & m) - bit) & m) | (n & ~m);
            const uint32_t q = N >> 3;
            if (!is_active(v, q)) return v.val[q];
            rec = get_rec(v, v.o + 8 * rank_of(v, q) + (N & 7u));
            n = N;
            continue;
        }
        // outside the brick: the parent slot
        if ((n & 7u) == 0) return v.val[n >> 3];
        rec = get_rec(v, v.o + 8 * rank_of(v, n >> 3));
        n &= ~7u;
    }
    *bad = true;
    return 0;
}

__device__ __forceinline__ uint64_t label_of(const uint64_t* pal, uint32_t pidx, uint32_t label0) {
    return pidx == label0 ? 0ull : pal[pidx];
}

// Step 1: every thread decodes seek segments of the brick (S ops each) into op
// records.  One rANS step per iteration; a Pd op's delta nibble is its own
// iteration, so the lanes of a warp never differ in steps per iteration.
// One op of a segment whose symbols are all in the stream: a Pd op reads its
// delta nibble in the same call.  Returns the op's record.
template <bool GLOBAL, bool CLUT>
__device__ __forceinline__ uint32_t decode_op(uint32_t& x, uint32_t& pos, uint32_t& ip, const uint8_t* enc,
                                              const uint32_t* lut, uint32_t P, uint32_t& st, uint32_t LABEL0) {
    const uint32_t v = rans_step<GLOBAL, CLUT>(x, pos, enc, lut);
    const uint32_t code = v >> 1, stop = (v & 1u) << 3;
    uint32_t pidx;
    if (code == OP_PD) {
        pidx = ip - rans_step<GLOBAL, CLUT>(x, pos, enc, lut) - 1;
    } else {
        ip += (code == OP_PA);
        pidx = (code == OP_PA || code == OP_P0) ? ip : 0u;
        if (code == 7) {
            pidx = LABEL0;
            st |= CSV_BRICK_BADOP;
        }
    }
    if (code >= OP_PA && code <= OP_PD && pidx >= P) {  // past the palette: clamped as decode.wgsl:472-485
        pidx = P - 1;
        st |= CSV_BRICK_PALETTE;
    }
    return code | stop | (pidx << REC_PIDX_SHIFT);
}

template <bool GLOBAL, bool CLUT>
__device__ __forceinline__ void decode_segments(const DecodeArgs& A, const BrickDesc& br, const uint8_t* enc,
                                                const uint32_t* lut, uint32_t n_need, uint32_t nseg,
                                                uint32_t* __restrict__ recs, uint32_t& st, uint32_t LABEL0) {
    for (uint32_t k = threadIdx.x; k < nseg; k += blockDim.x) {
        const Checkpoint c = A.ck[br.ck_off + k];
        uint32_t x = c.state, pos = c.pos, sym = c.sym, ip = c.ip;
        uint32_t j = k * A.S;  // a multiple of 4 (S is)
        const uint32_t jend = min(j + A.S, n_need);
        // Fast path: an op takes at most two symbols, so a segment whose ops cannot
        // run past nSymbols needs no truncation test; four ops per iteration go to
        // one 16-byte record group.  The general loop below takes what is left
        // (a segment's last ops when fewer than four, or any segment near the end
        // of a stream).
        if (sym + 2 * (jend - j) <= br.nsym) {
            const uint32_t sym0 = sym;
            uint32_t n4 = (jend - j) & ~3u;
            for (uint32_t e = j + n4; j < e; j += 4) {
                const uint32_t r0 = decode_op<GLOBAL, CLUT>(x, pos, ip, enc, lut, br.P, st, LABEL0);
                const uint32_t r1 = decode_op<GLOBAL, CLUT>(x, pos, ip, enc, lut, br.P, st, LABEL0);
                const uint32_t r2 = decode_op<GLOBAL, CLUT>(x, pos, ip, enc, lut, br.P, st, LABEL0);
                const uint32_t r3 = decode_op<GLOBAL, CLUT>(x, pos, ip, enc, lut, br.P, st, LABEL0);
                reinterpret_cast<uint4*>(recs + j)[0] = make_uint4(r0, r1, r2, r3);
                n4 += (r0 & 7u) == OP_PD;  // symbols: one per op plus one per Pd
                n4 += (r1 & 7u) == OP_PD;
                n4 += (r2 & 7u) == OP_PD;
                n4 += (r3 & 7u) == OP_PD;
            }
            sym = sym0 + n4;
        }
        uint32_t pd_stop = 0xFFFFFFFFu;  // != ~0: the primary nibble of a Pd op was read
        // records leave in 16-byte groups: lanes write different segments, so a
        // 4-byte store per op would cost one memory transaction per lane per op
        uint32_t q0 = 0, q1 = 0, q2 = 0, q3 = 0;
        while (j < jend) {
            if (sym >= br.nsym) {
                st |= CSV_BRICK_TRUNCATED;
                if (pd_stop != 0xFFFFFFFFu) {  // Pd without its delta: delta 0
                    uint32_t pidx = ip - 1;
                    if (pidx >= br.P) { pidx = br.P - 1; st |= CSV_BRICK_PALETTE; }
                    q0 = q1; q1 = q2; q2 = q3;
                    q3 = OP_PD | pd_stop | (pidx << REC_PIDX_SHIFT);
                    ++j;
                }
                break;
            }
            const uint32_t v = rans_step<GLOBAL, CLUT>(x, pos, enc, lut);
            ++sym;
            uint32_t rec;
            if (pd_stop != 0xFFFFFFFFu) {
                uint32_t pidx = ip - v - 1;
                if (pidx >= br.P) { pidx = br.P - 1; st |= CSV_BRICK_PALETTE; }
                rec = OP_PD | pd_stop | (pidx << REC_PIDX_SHIFT);
                pd_stop = 0xFFFFFFFFu;
            } else {
                const uint32_t code = v >> 1;
                if (code == OP_PD) {
                    pd_stop = (v & 1u) << 3;
                    continue;
                }
                uint32_t pidx = 0;
                if (code == OP_PA || code == OP_P0) {
                    ip += (code == OP_PA);
                    pidx = ip;
                    if (pidx >= br.P) { pidx = br.P - 1; st |= CSV_BRICK_PALETTE; }
                } else if (code == 7) {
                    pidx = LABEL0;
                    st |= CSV_BRICK_BADOP;
                }
                rec = code | ((v & 1u) << 3) | (pidx << REC_PIDX_SHIFT);
            }
            q0 = q1; q1 = q2; q2 = q3; q3 = rec;
            ++j;
            if ((j & 3u) == 0) reinterpret_cast<uint4*>(recs + j - 4)[0] = make_uint4(q0, q1, q2, q3);
        }
        // the last partial group (segment end or truncation): q3 is record j-1, q2 is j-2, ...
        const uint32_t rem = j & 3u;
        if (rem >= 1) recs[j - 1] = q3;
        if (rem >= 2) recs[j - 2] = q2;
        if (rem >= 3) recs[j - 3] = q1;
    }
}

// One model's rANS table into shared memory, full or compact (compact_lut).
template <class V>
__device__ __forceinline__ void load_lut(uint32_t* lut, const uint32_t* __restrict__ g, uint32_t tid, uint32_t T) {
    if (compact_lut<V>()) {
        for (uint32_t i = tid; i < kTot; i += T) {
            const uint32_t e = g[i];
            reinterpret_cast<uint8_t*>(lut)[i] = (uint8_t)(e & 15u);
            lut[kTot / 4 + (e & 15u)] = e;  // every x of a symbol stores the same entry
        }
    } else {
        for (uint32_t i = tid; i < kTot; i += T) lut[i] = g[i];
    }
}

// V = uint8_t when every requested brick's palette has fewer than 255 entries
// (value 0xFF stands for "label 0"), uint16_t when every
// palette of the dataset has fewer than 65535 entries (0xFFFF), else uint32_t.
template <class V, uint32_t KL>
__global__ void __launch_bounds__(dec_threads<V, KL>(), dec_ctas_per_sm<V, KL>()) decode_kernel(DecodeArgs A) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    DecShared<V, KL>& S = *reinterpret_cast<DecShared<V, KL>*>(smem_raw);
    const uint32_t tid = threadIdx.x, T = blockDim.x;
    // A kernel launched as this one's programmatic dependent (the second part of a
    // split schedule: other requests, other scratch) may start on the SMs this
    // grid's CTAs leave; without one this is a no-op.
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    constexpr uint32_t LABEL0 = sizeof(V) == 1 ? 0xFFu : (sizeof(V) == 2 ? 0xFFFFu : PIDX_LABEL0);

    load_lut<V>(S.lut, A.lut, tid, T);
    if (tid == 0) {
        mbar_init(&S.bar);
        S.rewait = 0;
        // Set when a copy into the staging region was still unconfirmed after two
        // bounded waits.  The region is then never touched again: every request the
        // CTA takes from then on is reported CSV_BRICK_TIMEOUT without output.
        S.drained = 0;
    }
    uint32_t phase = 0;     // parity of the stream-copy barrier
    bool stage_ok = true;   // cleared if a copy ever fails to land in time

    // per-CTA scratch: op records | active-node lists of every parent level
    uint8_t* scr = A.scratch + (uint64_t)blockIdx.x * A.scratch_per_cta;
    uint32_t* recs = reinterpret_cast<uint32_t*>(scr);
    const uint64_t max_ops = ((1ull << (3 * A.L)) - 8) / 7;
    uint32_t* act = reinterpret_cast<uint32_t*>(scr + ((max_ops * 4 + 255) & ~255ull));
    // parent level KL (if the launch's bricks have one) in scratch, after the active lists
    V* spill = reinterpret_cast<V*>(reinterpret_cast<uint8_t*>(act) + ((4ull * lvl_off(A.L - 1) + 255) & ~255ull));

    // the request count: fixed at launch, or produced on the device by an
    // earlier kernel in the same stream (the serving loop's admission)
    const uint32_t n_req = A.n_dev ? min(*A.n_dev, A.n) : A.n;
    uint32_t cur_model = 0;  // the LUT in shared memory is model 0's
    for (;;) {
        if (tid == 0) {
            const uint32_t k = atomicAdd(A.queue, 1u);
            // an optional schedule (longest brick first, or one part of a
            // split by output size) maps queue slots to requests
            uint32_t wk = 0xFFFFFFFFu;  // past the end of the queue
            if (k < n_req) wk = A.order ? min(A.order[k], 0xFFFFFFFEu) : k;
            S.work = wk;
            S.status = 0;
            if (wk < A.n_reqs) {
                S.req = A.reqs[wk];
                if (S.req.brick < A.nb) S.br = A.bricks[S.req.brick];
            }
        }
        __syncthreads();
        const uint32_t w = S.work;
        if (w == 0xFFFFFFFFu) break;
        if (w >= A.n_reqs) {  // an order entry naming no request: nothing to decode or report
            __syncthreads();
            continue;
        }
        const csv_request req = S.req;
        const uint32_t t = req.lod;
        // bricks of a concatenated dataset carry their own level count and model;
        // a request at LOD t needs parent levels 0..t-1 in shared memory and the
        // op records of levels 1..t in scratch, both sized for A.L levels
        const uint32_t Lb = (S.br.flags >> BF_LEVELS_SHIFT) & 15u, model = (S.br.flags >> BF_MODEL_SHIFT) & 255u;
        if (req.brick >= A.nb || t >= Lb || t >= A.L || model >= A.n_models) {
            if (tid == 0) A.status[w] = CSV_BRICK_BADREQ;
            __syncthreads();
            continue;
        }
        if (S.drained) {  // the staging region may still receive a lost copy: decode nothing
            if (tid == 0) A.status[w] = CSV_BRICK_TIMEOUT;
            __syncthreads();
            continue;
        }
        if (model != cur_model) {  // made visible by the barrier after the palette copy
            load_lut<V>(S.lut, A.lut + (size_t)model * kTot, tid, T);
            cur_model = model;
        }
        const BrickDesc br = S.br;
        // stage the compressed stream in shared memory (one bulk copy) while the palette loads
        const uint32_t E16 = (br.E + 15u) & ~15u;
        const bool stage = stage_ok && t > 0 && !(br.flags & BF_UNIFORM) && E16 >= 16 && E16 <= A.stage_cap;
        if (stage && tid == 0) bulk_copy_g2s(S.val, A.enc + br.enc_off, E16, &S.bar);
        uint64_t* out = A.out + req.dst;
        const uint64_t* gpal = A.pal + br.pal_off;
        const uint64_t* pal = gpal;
        if (br.P <= pal_cache<V, KL>()) {
            for (uint32_t i = tid; i < br.P; i += T) S.pal[i] = gpal[i];
            pal = S.pal;
        }
        uint32_t st = (br.flags & BF_TRUNCATED) ? CSV_BRICK_TRUNCATED : 0;
        bool bad = false;
        __syncthreads();

        if (t == 0 || (br.flags & BF_UNIFORM)) {
            fill_labels(out, 1ull << (3 * t), pal[0]);
        } else {
            // ---- 1. rANS segments -> op records
            // (level_start is read from shared memory: a runtime index into a
            // register copy of the descriptor would put it on the stack)
            const uint32_t n_need = min(min(S.br.level_start[t], br.n_ops), br.ck_cap * A.S);
            const uint32_t nseg = (n_need + A.S - 1) / A.S;
            bool staged = false;
            if (stage) {
                // one decision for the whole CTA: staged only if every thread saw the copy land
                staged = __syncthreads_and(mbar_wait(&S.bar, phase)) != 0;
                if (staged) {
                    phase ^= 1u;
                } else {  // the copy did not land in time: read this brick from global memory
                    st |= CSV_BRICK_TIMEOUT;
                    stage_ok = false;  // and stage nothing more
                    if (tid == 0) S.rewait = 1;  // read after the barrier that ends the rANS phase
                }
            }
            if (staged)
                decode_segments<false, compact_lut<V>()>(A, br, reinterpret_cast<const uint8_t*>(S.val), S.lut, n_need, nseg, recs,
                                       st, LABEL0);
            else
                decode_segments<true, compact_lut<V>()>(A, br, A.enc + br.enc_off, S.lut, n_need, nseg, recs, st, LABEL0);
            __syncthreads();  // the staged stream is dead: its space becomes the level arrays
            if (S.rewait) {
                // The late copy must land before the staging region is written: a second
                // bounded wait on the same phase.  If it gives up too, this brick is
                // reported without output and the CTA decodes nothing more (drained).
                const bool landed = __syncthreads_and(mbar_wait(&S.bar, phase)) != 0;
                if (landed) phase ^= 1u;
                if (tid == 0) {
                    S.rewait = 0;
                    if (!landed) {
                        S.drained = 1;
                        A.status[w] = st | CSV_BRICK_TIMEOUT;
                    }
                }
                __syncthreads();
                if (!landed) continue;
            }
            // level 0: the root, value palette[0], active; clear the other masks
            for (uint32_t i = tid; i < moff(t); i += T) S.mask[i] = i == 0 ? 1u : 0u;
            if (tid == 0) {
                S.val[0] = 0;
                S.pre[0] = 0;
                act[0] = 0;
            }
            __syncthreads();

            // ---- 2./3. levels coarse to fine
            const bool vec = (((uintptr_t)out) & 15) == 0;
            const bool vec32 = (((uintptr_t)out) & 31) == 0;
            uint32_t n_act = 1;
            for (uint32_t l = 0; l < t; ++l) {
                const uint32_t lc = l + 1;
                LevelView<V> Vw;
                Vw.val = l < KL ? S.val + voff(l) : spill;
                Vw.mask = S.mask + moff(l);
                Vw.pre = S.pre + moff(l);
                Vw.rec = recs;
                Vw.o = S.br.level_start[l];
                Vw.n_rec = n_need;
                const uint32_t* act_l = act + lvl_off(l);
                const uint32_t n_par = 1u << (3 * l);
                if (lc < t) {
                    V* val_c = lc < KL ? S.val + voff(lc) : spill;
                    uint32_t* mask_c = S.mask + moff(lc);
                    // children of stop-filled parents inherit (8 bytes of u8, 16 of u16 or 2 x 16 of u32)
                    for (uint32_t p = tid; p < n_par; p += T) {
                        if (!is_active(Vw, p)) {
                            const uint32_t v = Vw.val[p];
                            if (sizeof(V) == 1) {
                                const uint32_t vv = v * 0x01010101u;
                                reinterpret_cast<uint2*>(val_c + 8 * p)[0] = make_uint2(vv, vv);
                            } else if (sizeof(V) == 2) {
                                const uint32_t vv = v | (v << 16);
                                reinterpret_cast<uint4*>(val_c + 8 * p)[0] = make_uint4(vv, vv, vv, vv);
                            } else {
                                reinterpret_cast<uint4*>(val_c + 8 * p)[0] = make_uint4(v, v, v, v);
                                reinterpret_cast<uint4*>(val_c + 8 * p)[1] = make_uint4(v, v, v, v);
                            }
                        }
                    }
                    // children of active parents take their ops (the r-th active
                    // parent's are records o + 8r .. o + 8r + 7).  With fewer
                    // children than threads, one thread per child, so that the
                    // record reads of neighbour chains overlap across lanes; lanes
                    // 8k..8k+7 then hold one parent (T is a multiple of 32) and
                    // merge their activity bits by ballot.  Otherwise one thread
                    // per parent.  (Measured: per child pays on every level of the
                    // 32^3 variant, on the 64^3 one only up to T children.)
                    const uint32_t n_kids = 8 * n_act;
                    if (n_kids <= (KL == kDecLevels ? T : 8 * T)) {
                        for (uint32_t base = 0; base < n_kids; base += T) {
                            const uint32_t i = base + tid;
                            uint32_t p = 0, child_active = 0;
                            if (i < n_kids) {
                                p = act_l[i >> 3];
                                const uint32_t rec = get_rec(Vw, Vw.o + i);
                                const uint32_t node = 8 * p + (i & 7u);
                                val_c[node] = (V)resolve(Vw, rec, node, lc, &bad);
                                child_active = (rec & 8u) ? 0u : 1u;
                            }
                            const uint32_t bits = (__ballot_sync(0xFFFFFFFFu, child_active) >> (tid & 24u)) & 0xFFu;
                            if (bits && (tid & 7u) == 0) atomicOr(mask_c + ((8 * p) >> 5), bits << ((8 * p) & 31));
                        }
                    } else {
                        for (uint32_t r = tid; r < n_act; r += T) {
                            const uint32_t p = act_l[r];
                            uint32_t rec[8];
                            get_rec8(Vw, r, rec);
                            uint32_t bits = 0;
#pragma unroll
                            for (uint32_t c = 0; c < 8; ++c) {
                                val_c[8 * p + c] = (V)resolve(Vw, rec[c], 8 * p + c, lc, &bad);
                                bits |= ((rec[c] & 8u) ? 0u : 1u) << c;
                            }
                            if (bits) atomicOr(mask_c + ((8 * p) >> 5), bits << ((8 * p) & 31));
                        }
                    }
                    __syncthreads();
                    // ranks: active nodes before each mask word, then the compacted list
                    const uint32_t nw = mwords(lc);
                    const uint32_t per = (nw + T - 1) / T;
                    const uint32_t w0 = min(nw, tid * per), w1 = min(nw, w0 + per);
                    uint32_t cnt = 0;
                    for (uint32_t i = w0; i < w1; ++i) cnt += __popc(mask_c[i]);
                    uint32_t n_act_c;
                    uint32_t run = block_exclusive<uint32_t>(cnt, S.warp_sums, &n_act_c);
                    uint32_t* act_c = act + lvl_off(lc);
                    for (uint32_t i = w0; i < w1; ++i) {
                        S.pre[moff(lc) + i] = (uint16_t)run;
                        uint32_t m = mask_c[i];
                        while (m) {
                            act_c[run++] = 32 * i + (__ffs(m) - 1);
                            m &= m - 1;
                        }
                    }
                    n_act = n_act_c;
                    __syncthreads();
                } else if (vec32) {
                    // last level: labels to HBM with 32-byte stores, two lanes per
                    // parent (four children each), so that a warp's store covers 1 KB
                    // of contiguous output.  Stop-filled parents first: chunk q is
                    // children 4(q&1) .. 4(q&1)+3 of parent q / 2.
                    const uint32_t n_chunk = 2 * n_par;
                    for (uint32_t q = tid; q < n_chunk; q += T) {
                        const uint32_t p = q >> 1;
                        if (!is_active(Vw, p)) {
                            const uint64_t x = label_of(pal, Vw.val[p], LABEL0);
                            st_cs_v4(out + 4ull * q, x, x, x, x);
                        }
                    }
                    // active parents: two lanes per parent, four children each from
                    // one 16-byte record load; the next parent's index and records
                    // are fetched before this one is resolved.
                    const uint32_t half = tid & 1u;
                    auto fetch = [&](uint32_t g, uint32_t& p, uint4& r) {
                        p = act_l[g];
                        const uint32_t i0 = Vw.o + 8 * g + 4 * half;
                        if ((i0 & 3u) == 0 && i0 + 4 <= Vw.n_rec) {
                            r = *reinterpret_cast<const uint4*>(Vw.rec + i0);
                        } else {
                            r = make_uint4(get_rec(Vw, i0), get_rec(Vw, i0 + 1), get_rec(Vw, i0 + 2),
                                           get_rec(Vw, i0 + 3));
                        }
                    };
                    uint32_t g = tid >> 1, p_next = 0;
                    uint4 r_next = make_uint4(0, 0, 0, 0);
                    if (g < n_act) fetch(g, p_next, r_next);
                    for (; g < n_act; g += T >> 1) {
                        const uint32_t p = p_next;
                        const uint4 r = r_next;
                        if (g + (T >> 1) < n_act) fetch(g + (T >> 1), p_next, r_next);
                        const uint32_t n0 = 8 * p + 4 * half;
                        const uint64_t a = label_of(pal, resolve(Vw, r.x, n0, lc, &bad), LABEL0);
                        const uint64_t b = label_of(pal, resolve(Vw, r.y, n0 + 1, lc, &bad), LABEL0);
                        const uint64_t c = label_of(pal, resolve(Vw, r.z, n0 + 2, lc, &bad), LABEL0);
                        const uint64_t d = label_of(pal, resolve(Vw, r.w, n0 + 3, lc, &bad), LABEL0);
                        st_cs_v4(out + n0, a, b, c, d);
                    }
                } else {
                    // last level, output not 32-byte aligned.  Each thread writes 16 bytes (two
                    // children) per step so that a warp's store covers 512
                    // contiguous bytes.  Stop-filled parents: chunk q is children
                    // 2q, 2q+1 of parent q / 4.
                    const uint32_t n_chunk = 4 * n_par;
                    for (uint32_t q = tid; q < n_chunk; q += T) {
                        const uint32_t p = q >> 2;
                        if (!is_active(Vw, p)) {
                            const uint64_t x = label_of(pal, Vw.val[p], LABEL0);
                            uint64_t* o2 = out + 2ull * q;
                            if (vec) {
                                st_cs_v2(o2, x, x);
                            } else {
                                o2[0] = x;
                                o2[1] = x;
                            }
                        }
                    }
                    // active parents: four lanes per parent, two children each.
                    // The next parent's index and records are fetched before
                    // this one is resolved, so that two global reads per lane
                    // are in flight.
                    const uint32_t sub = tid & 3u;
                    auto fetch = [&](uint32_t g, uint32_t& p, uint32_t& r0, uint32_t& r1) {
                        p = act_l[g];
                        const uint32_t i0 = Vw.o + 8 * g + 2 * sub;
                        if ((i0 & 1u) == 0 && i0 + 2 <= Vw.n_rec) {
                            const uint2 rr = *reinterpret_cast<const uint2*>(Vw.rec + i0);
                            r0 = rr.x;
                            r1 = rr.y;
                        } else {
                            r0 = get_rec(Vw, i0);
                            r1 = get_rec(Vw, i0 + 1);
                        }
                    };
                    uint32_t g = tid >> 2, p_next = 0, r0_next = 0, r1_next = 0;
                    if (g < n_act) fetch(g, p_next, r0_next, r1_next);
                    for (; g < n_act; g += T >> 2) {
                        const uint32_t p = p_next, r0 = r0_next, r1 = r1_next;
                        if (g + (T >> 2) < n_act) fetch(g + (T >> 2), p_next, r0_next, r1_next);
                        const uint32_t n0 = 8 * p + 2 * sub;
                        const uint64_t a = label_of(pal, resolve(Vw, r0, n0, lc, &bad), LABEL0);
                        const uint64_t b = label_of(pal, resolve(Vw, r1, n0 + 1, lc, &bad), LABEL0);
                        uint64_t* o2 = out + n0;
                        if (vec) {
                            st_cs_v2(o2, a, b);
                        } else {
                            o2[0] = a;
                            o2[1] = b;
                        }
                    }
                }
            }
        }
        if (bad) st |= CSV_BRICK_BADOP;
        if (st) atomicOr(&S.status, st);
        __syncthreads();
        if (tid == 0) A.status[w] = S.status;
        __syncthreads();
    }
    // Launched as a programmatic dependent: finish only after the kernel before
    // this one has, so that work after this grid in the stream sees both grids'
    // results.  Otherwise a no-op.
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

size_t decode_scratch_per_cta(uint32_t b, uint32_t kl) {
    uint32_t L = levels_of(b);
    uint64_t rec_bytes = (max_ops_of(b) * 4 + 255) & ~255ull;
    uint64_t act_bytes = (4ull * lvl_off(L - 1) + 255) & ~255ull;  // active lists of levels 0 .. L-2
    // node values of parent level kl when the brick has one (up to 32-bit entries)
    uint64_t spill_bytes = L - 1 > kl ? 4ull << (3 * kl) : 0;
    return (size_t)(rec_bytes + act_bytes + spill_bytes);
}

static int g_dec_occ[6][64] = {{0}};

template <class V, uint32_t KL>
static int occupancy(int device) {
    int& occ = g_dec_occ[2 * (sizeof(V) == 1 ? 2 : sizeof(V) == 2 ? 0 : 1) + (KL == kDecLevels ? 0 : 1)][device & 63];
    if (occ == 0) {
        cudaFuncSetAttribute(decode_kernel<V, KL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(DecShared<V, KL>));
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, decode_kernel<V, KL>, dec_threads<V, KL>(),
                                                      sizeof(DecShared<V, KL>));
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        occ = (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
    }
    return occ;
}

uint32_t decode_grid(int device, uint32_t n) {
    uint32_t occ = (uint32_t)std::max({occupancy<uint8_t, kDecLevels>(device), occupancy<uint16_t, kDecLevels>(device),
                                       occupancy<uint32_t, kDecLevels>(device)});
    return n < occ ? n : occ;
}

// Scratch for every variant a dataset of bricks up to b^3 can use: the 64^3
// variant's CTAs at b's size, or the 32^3 variant's CTAs at min(b, 32)'s size.
size_t decode_scratch_bytes(int device, uint32_t b) {
    const size_t big = decode_scratch_per_cta(b, kDecLevels) * (size_t)decode_grid(device, 0xFFFFFFFFu);
    const size_t small = decode_scratch_per_cta(b, kSmallLevels) *
                         (size_t)std::max({occupancy<uint8_t, kSmallLevels>(device),
                                           occupancy<uint16_t, kSmallLevels>(device),
                                           occupancy<uint32_t, kSmallLevels>(device)});
    return std::max(big, small);
}

size_t decode_scratch_wide_bytes(int device, uint32_t b) {
    return decode_scratch_per_cta(b, kDecLevels) *
           (size_t)std::max(occupancy<uint16_t, kDecLevels>(device), occupancy<uint32_t, kDecLevels>(device));
}

size_t decode_scratch_small_bytes(int device) {
    return decode_scratch_per_cta(1u << kSmallLevels, kSmallLevels) *
           (size_t)std::max({occupancy<uint8_t, kSmallLevels>(device), occupancy<uint16_t, kSmallLevels>(device),
                             occupancy<uint32_t, kSmallLevels>(device)});
}

template <class V, uint32_t KL>
static cudaError_t launch_variant(const DecodeArgs& A0, const DecodeScratch& scr, cudaStream_t st,
                                  const DecodeConfig* cfg, int device) {
    DecodeArgs A = A0;
    uint32_t grid = (uint32_t)occupancy<V, KL>(device);
    if (cfg && cfg->ctas_per_sm) {
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        const uint32_t per_sm = KL == kDecLevels ? cfg->ctas_per_sm : 2 * cfg->ctas_per_sm;
        grid = std::min<uint32_t>(grid, per_sm * (uint32_t)std::max(sms, 1));
    }
    A.scratch_per_cta = decode_scratch_per_cta(1u << (A.L - 1), KL);
    const uint64_t cap = scr.bytes / A.scratch_per_cta;
    if (grid > A.n) grid = A.n;
    if (grid > cap) grid = (uint32_t)cap;
    if (grid == 0) return cudaErrorInvalidValue;
    A.stage_cap = (cfg && !cfg->stage) ? 0u : stage_cap<V, KL>();
    if (cfg && cfg->pdl) {
        cudaLaunchConfig_t lc = {};
        lc.gridDim = dim3(grid);
        lc.blockDim = dim3(dec_threads<V, KL>());
        lc.dynamicSmemBytes = sizeof(DecShared<V, KL>);
        lc.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[0].val.programmaticStreamSerializationAllowed = 1;
        lc.attrs = at;
        lc.numAttrs = 1;
        return cudaLaunchKernelEx(&lc, decode_kernel<V, KL>, A);
    }
    decode_kernel<V, KL><<<grid, dec_threads<V, KL>(), sizeof(DecShared<V, KL>), st>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_decode(const DeviceDataset& ds, const csv_request* d_reqs, uint32_t n, uint64_t* d_out,
                          uint32_t* d_status, const DecodeScratch& scr, cudaStream_t st, const DecodeConfig* cfg) {
    if (n == 0) return cudaSuccess;
    if (ds.L > kDecLevels + 1) return cudaErrorInvalidValue;  // bricks up to 64^3
    const bool narrow = ds.max_P < 0xFFFFu;
    // 8-bit node values: every palette of the dataset, or of the requested bricks (the caller's word,
    // from a schedule that split the requests by palette size), below 255 entries
    const bool narrow8 = (ds.max_P < 0xFFu || (cfg && cfg->narrow8)) && !(cfg && cfg->layout == 2);
    // the small variant when the dataset's bricks are 32^3 or smaller, when the caller
    // says every request is at LOD 5 or coarser, or when asked to take every request
    const bool small = ds.L <= kSmallLevels + 1 || (cfg && (cfg->small_only || cfg->layout == 1));
    if (!(cfg && cfg->pdl)) {  // a programmatic dependent follows a kernel, not this reset
        cudaError_t e = cudaMemsetAsync(scr.d_queue, 0, sizeof(uint32_t), st);
        if (e != cudaSuccess) return e;
    }
    DecodeArgs A;
    A.bricks = ds.d_bricks;
    A.pal = ds.d_pal;
    A.enc = ds.d_enc;
    A.ck = ds.d_ck;
    A.lut = ds.d_lut;
    A.reqs = d_reqs;
    A.out = d_out;
    A.status = d_status;
    A.scratch = scr.base;
    A.scratch_per_cta = scr.per_cta;
    A.queue = scr.d_queue;
    A.nb = ds.nb;
    // levels of the largest output this launch decodes (a request above it is refused with
    // CSV_BRICK_BADREQ), so the per-CTA scratch can be laid out for that size
    A.L = (cfg && cfg->small_only) ? std::min<uint32_t>(ds.L, kSmallLevels + 1) : ds.L;
    A.S = ds.S;
    A.n_reqs = n;
    A.n = (cfg && cfg->order && cfg->n_order) ? cfg->n_order : n;
    A.order = cfg ? cfg->order : nullptr;
    A.n_dev = cfg ? cfg->n_dev : nullptr;
    A.stage_cap = 0;
    A.n_models = ds.n_models ? ds.n_models : 1u;
    if (small) {
        if (narrow8) return launch_variant<uint8_t, kSmallLevels>(A, scr, st, cfg, ds.device);
        if (narrow) return launch_variant<uint16_t, kSmallLevels>(A, scr, st, cfg, ds.device);
        return launch_variant<uint32_t, kSmallLevels>(A, scr, st, cfg, ds.device);
    }
    if (narrow8) return launch_variant<uint8_t, kDecLevels>(A, scr, st, cfg, ds.device);
    if (narrow) return launch_variant<uint16_t, kDecLevels>(A, scr, st, cfg, ds.device);
    return launch_variant<uint32_t, kDecLevels>(A, scr, st, cfg, ds.device);
}

}  // namespace csv
