// serve.cu -- the viewer's frame loop on the device: plan, cache, decode, render.
//
// The reference runs this loop in JavaScript on the host (renderLoop.js:208-340,
// cacheProcessing.js:99-232, cacheManager.js:10-246, camera.js:103-137,
// culling.js:22-171) and hands the GPU one work queue per frame.  Here every
// per-brick decision runs on the device, in one stream, with no host round
// trip between the steps of a frame:
//
//   plan_kernel    per brick: the LOD each open session asks for
//                  (camera.js:103-137) and the cone test (culling.js:87-153);
//                  the (brick, LOD) blocks to keep, free and admit; per-CTA counts
//   scan_kernel    one CTA: per-CTA bases of those counts, then the cache policy
//                  (free stacks per LOD, bump pointer, rebuild) for the step
//   push_kernel    per brick: freed blocks onto their LOD's stack
//   pop_kernel     per brick: admitted blocks pop a stack entry or take fresh
//                  space; their decode requests; every open session's slot table
//   decode_kernel  (decode.cu) the admitted requests, count read on the device
//   render_kernel  (ray.cu) one launch per session with a new frame
//   census_kernel  per brick: bricks each session's rays entered, and how many
//                  had no data
//
// Admission by rays (CSV_ADMIT_RAYS, the reference's switched-off useGPUCulling
// path): the plan keeps only the bricks a session's last render entered (its
// request words, which the census then leaves for the plan to consume).
// Compaction (csv_serve_compact, CacheState.compact()) is a step whose plan is
// the resident set itself, placed again as a rebuild places blocks.
//
// Sessions share the cache but not their LODs: a block is keyed by (brick,
// LOD), each session's slot table points at the blocks of its own LODs, and a
// session's plan uses the camera of its own last re-plan (it re-plans when it
// moved more than 0.5 units or turned more than 0.05 rad, culling.js:6-56).
// So a session's image is the same whichever other sessions are open, as long
// as the cache has room for all of them.
//
// Orders the reference leaves open are fixed so that the result is
// deterministic and equal to the CPU restatement (oracle/csv_oracle_serve.c):
// frees are pushed in brick order; admissions are served LOD by LOD (coarse
// first), in brick order within a LOD, popping the LOD's stack from the top and
// then taking fresh space; a step whose fresh space does not fit rebuilds the
// cache (every needed block placed again, coarse LODs first, while space
// remains).  LOD-0 bricks and uniform bricks take no block: their slot reads
// palette[0] from a table at the start of the cache.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <deque>
#include <new>
#include <string>
#include <vector>

#include "abi_internal.h"
#include "csv_internal.h"

using namespace csv;

namespace csv {
namespace {

constexpr uint32_t kMaxViews = 8;
constexpr uint32_t kBlk = 256;  // bricks per CTA in the per-brick kernels
constexpr uint32_t kWarps = kBlk / 32;
constexpr uint32_t kLods = 8;   // LOD slots; bricks up to 64^3 use 0..6
constexpr uint8_t kNone = 0xFF;
constexpr uint32_t kRing = 64;  // steps in flight before the host harvests one
enum : uint32_t { CNT_FREE = 0, CNT_ALLOC = kLods, CNT_NEED = 2 * kLods, kCnt = 3 * kLods };
enum : uint8_t { BK_HAS = 1, BK_UNIFORM = 2 };

struct ViewD {
    double p[3], d[3];
};

// Device-resident cache state and the plan of the current step.
struct ServeState {
    uint32_t top[kLods];       // free-stack sizes
    uint32_t T[kLods];         // stack sizes after this step's pushes
    uint32_t top_old[kLods];   // stack sizes before them
    uint32_t fit[kLods];       // rebuild: blocks placed per LOD
    uint32_t req_base[kLods];  // first request index of each LOD
    uint64_t base[kLods];      // first fresh offset per LOD (overflow / rebuild placement)
    uint64_t bump, cap;
    uint32_t mode;             // 0: keep the cache, 1: rebuild
    uint32_t n_req;            // admitted requests (read by the decode kernel)
    uint32_t resident;         // resident blocks
    uint32_t pad;
};

// One step's counters; entered/missing per rendered session.
struct StepStats {
    uint32_t planned, visible, decoded, freed, resident, rebuilt, vox_lo, vox_hi;
    uint32_t entered[kMaxViews], missing[kMaxViews];
};

struct PlanArgs {
    ViewD v[kMaxViews];
    uint32_t sid[kMaxViews];
    uint32_t n_views, b, max_lod, nb, n_cta;
    double focal, cos_half, radius, half;
    const uint32_t* ids;
    const uint8_t* bflag;
    const uint8_t* res;   // bit l: block at LOD l resident
    uint32_t* req_words;  // [session][n_slots]: the last render's request words (admission by rays)
    uint64_t n_slots;
    uint32_t ready;       // bit s: view s has request words to apply (and consume)
    uint8_t* want;        // [session][brick]
    uint8_t* need;        // bit l: some open session needs LOD l of the brick
    uint32_t* cnt;        // [kCnt][n_cta]
    StepStats* stats;
};

__device__ __forceinline__ uint32_t compact3(uint32_t v) {
    v &= 0x09249249u;
    v = (v | (v >> 2)) & 0x030c30c3u;
    v = (v | (v >> 4)) & 0x0300f00fu;
    v = (v | (v >> 8)) & 0x030000ffu;
    v = (v | (v >> 16)) & 0x000003ffu;
    return v;
}

// culling.js:87-153 (margin sin(atan2(r, d)) as r / sqrt(r^2 + d^2)); bricks
// closer than twice their radius are always in.
__device__ __forceinline__ bool in_cone(const PlanArgs& A, const double* c, const ViewD& v) {
    const double tx = c[0] - v.p[0], ty = c[1] - v.p[1], tz = c[2] - v.p[2];
    const double dist = sqrt(tx * tx + ty * ty + tz * tz);
    if (dist < 2.0 * A.radius) return true;
    const double dot = (tx / dist) * v.d[0] + (ty / dist) * v.d[1] + (tz / dist) * v.d[2];
    const double margin = A.radius / sqrt(A.radius * A.radius + dist * dist);
    return !(dot < A.cos_half - margin);
}

// camera.js:103-137: the finest LOD whose voxels still cover a pixel.
__device__ __forceinline__ uint32_t brick_lod(const PlanArgs& A, const double* c, const ViewD& v) {
    const double dx = c[0] - v.p[0], dy = c[1] - v.p[1], dz = c[2] - v.p[2];
    const double dist = sqrt(dx * dx + dy * dy + dz * dz);
    const double d = dist > 0.1 ? dist : 0.1;
    uint32_t best = 0;
    for (uint32_t lod = 0; lod <= A.max_lod; ++lod) {
        const double voxel = (double)A.b / (double)(1u << lod);
        if ((A.focal * voxel) / d >= 1.0) best = lod;
        else break;
    }
    return best;
}

// Per LOD l: counts of the CTA's threads whose `mask` has bit l (s_tot[l]) and,
// in rank[l], this thread's rank among them in thread order.  Every thread of
// the CTA calls it; s_wc is [kWarps][kLods] shared scratch.
__device__ __forceinline__ void cta_ranks(uint32_t mask, uint32_t (&rank)[kLods], uint32_t (*s_wc)[kLods],
                                          uint32_t* s_tot) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
    for (uint32_t l = 0; l < kLods; ++l) {
        const uint32_t b = __ballot_sync(0xffffffffu, (mask >> l) & 1u);
        rank[l] = __popc(b & lt);
        if (lane == 0) s_wc[warp][l] = __popc(b);
    }
    __syncthreads();
    if (threadIdx.x < kLods) {
        uint32_t acc = 0;
        for (uint32_t w = 0; w < kWarps; ++w) {
            const uint32_t t = s_wc[w][threadIdx.x];
            s_wc[w][threadIdx.x] = acc;
            acc += t;
        }
        s_tot[threadIdx.x] = acc;
    }
    __syncthreads();
#pragma unroll
    for (uint32_t l = 0; l < kLods; ++l) rank[l] += s_wc[warp][l];
}

__global__ void __launch_bounds__(kBlk) plan_kernel(PlanArgs A) {
    __shared__ uint32_t s_wc[kWarps][kLods];
    __shared__ uint32_t s_tot[kLods];
    __shared__ uint32_t s_vis;
    const uint32_t tid = threadIdx.x, i = blockIdx.x * kBlk + tid;
    if (tid == 0) s_vis = 0;
    uint32_t need = 0, res = 0;
    bool vis = false;
    if (i < A.nb) {
        const uint8_t bf = A.bflag[i];
        const bool uni = (bf & BK_UNIFORM) != 0;
        res = A.res[i];
        const uint32_t id = A.ids[i];
        const double c[3] = {(double)compact3(id) * (double)A.b + A.half,
                             (double)compact3(id >> 1) * (double)A.b + A.half,
                             (double)compact3(id >> 2) * (double)A.b + A.half};
        for (uint32_t s = 0; s < A.n_views; ++s) {
            uint32_t w = kNone;
            if ((bf & BK_HAS) && in_cone(A, c, A.v[s])) w = brick_lod(A, c, A.v[s]);
            if ((A.ready >> s) & 1u) {  // admission by rays: only what the last render entered
                uint32_t* rw = A.req_words + (size_t)A.sid[s] * A.n_slots + id;
                if (*rw == 0u) w = kNone;
                else *rw = 0u;  // consumed
            }
            A.want[(size_t)A.sid[s] * A.nb + i] = (uint8_t)w;
            if (w != kNone) {
                vis = true;
                if (w > 0 && !uni) need |= 1u << w;
            }
        }
        A.need[i] = (uint8_t)need;
    }
    const uint32_t nv = __popc(__ballot_sync(0xffffffffu, vis));
    __syncthreads();
    if ((tid & 31u) == 0 && nv) atomicAdd(&s_vis, nv);
    uint32_t rank[kLods];
    const uint32_t masks[3] = {res & ~need, need & ~res, need};
#pragma unroll
    for (uint32_t kind = 0; kind < 3; ++kind) {
        cta_ranks(masks[kind], rank, s_wc, s_tot);
        if (tid < kLods) A.cnt[(kind * kLods + tid) * A.n_cta + blockIdx.x] = s_tot[tid];
        __syncthreads();
    }
    if (tid == 0 && s_vis) atomicAdd(&A.stats->visible, s_vis);
}

// Compaction's plan: every brick needs exactly its resident blocks (no frees,
// no admissions); the scan then places them all again as a rebuild does.
__global__ void __launch_bounds__(kBlk) compact_plan_kernel(const uint8_t* __restrict__ res, uint8_t* __restrict__ need,
                                                            uint32_t nb, uint32_t* __restrict__ cnt, uint32_t n_cta) {
    __shared__ uint32_t s_wc[kWarps][kLods];
    __shared__ uint32_t s_tot[kLods];
    const uint32_t i = blockIdx.x * kBlk + threadIdx.x;
    uint32_t r = 0;
    if (i < nb) {
        r = res[i];
        need[i] = (uint8_t)r;
    }
    uint32_t rank[kLods];
    cta_ranks(r, rank, s_wc, s_tot);
    if (threadIdx.x < kLods) {
        cnt[(CNT_FREE + threadIdx.x) * n_cta + blockIdx.x] = 0;
        cnt[(CNT_ALLOC + threadIdx.x) * n_cta + blockIdx.x] = 0;
        cnt[(CNT_NEED + threadIdx.x) * n_cta + blockIdx.x] = s_tot[threadIdx.x];
    }
}

// One CTA: exclusive scans of the per-CTA counts (one warp per counter), then
// the step's cache policy by thread 0.
__global__ void __launch_bounds__(1024) scan_kernel(const uint32_t* __restrict__ cnt, uint32_t* __restrict__ base,
                                                    uint32_t n_cta, uint32_t max_lod, uint32_t nb,
                                                    ServeState* __restrict__ S, StepStats* __restrict__ st,
                                                    uint32_t force_rebuild) {
    __shared__ uint32_t tot[kCnt];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (warp < kCnt) {
        uint32_t carry = 0;
        for (uint32_t c0 = 0; c0 < n_cta; c0 += 32) {
            const uint32_t j = c0 + lane;
            const uint32_t v = j < n_cta ? cnt[warp * n_cta + j] : 0u;
            uint32_t x = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
                if ((int)lane >= o) x += y;
            }
            if (j < n_cta) base[warp * n_cta + j] = carry + x - v;
            carry += __shfl_sync(0xffffffffu, x, 31);
        }
        if (lane == 0) tot[warp] = carry;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    uint64_t need = 0;
    uint32_t over[kLods] = {}, nfree = 0, nalloc = 0;
    bool rebuild = false;
    for (uint32_t l = 1; l <= max_lod; ++l) {
        const uint32_t F = tot[CNT_FREE + l], A = tot[CNT_ALLOC + l];
        S->top_old[l] = S->top[l];
        S->T[l] = S->top[l] + F;
        if (S->T[l] > nb) rebuild = true;  // cannot happen: a LOD never holds more blocks than bricks
        over[l] = A > S->T[l] ? A - S->T[l] : 0u;
        need += (uint64_t)over[l] << (3 * l);
        nfree += F;
        nalloc += A;
    }
    if (S->bump + need > S->cap || force_rebuild) rebuild = true;
    uint64_t vox = 0;
    if (!rebuild) {
        uint64_t b = S->bump;
        for (uint32_t l = 1; l <= max_lod; ++l) {
            S->base[l] = b;
            b += (uint64_t)over[l] << (3 * l);
            const uint32_t A = tot[CNT_ALLOC + l];
            S->top[l] = S->T[l] - (A < S->T[l] ? A : S->T[l]);
            vox += (uint64_t)A << (3 * l);
        }
        S->bump = b;
        uint32_t acc = 0;
        for (uint32_t l = max_lod; l >= 1; --l) {  // finest LOD first: the longest decodes start first
            S->req_base[l] = acc;
            acc += tot[CNT_ALLOC + l];
        }
        S->n_req = acc;
        S->mode = 0;
        S->resident = S->resident - nfree + nalloc;
    } else {
        uint64_t b = 0;
        for (uint32_t l = 1; l <= max_lod; ++l) {
            const uint32_t W = tot[CNT_NEED + l];
            const uint64_t room = S->cap > b ? (S->cap - b) >> (3 * l) : 0ull;
            S->fit[l] = (uint32_t)(room < W ? room : W);
            S->base[l] = b;
            b += (uint64_t)S->fit[l] << (3 * l);
            S->top[l] = 0;
            S->top_old[l] = 0;
            S->T[l] = 0;
            vox += (uint64_t)S->fit[l] << (3 * l);
        }
        S->bump = b;
        uint32_t acc = 0;
        for (uint32_t l = max_lod; l >= 1; --l) {
            S->req_base[l] = acc;
            acc += S->fit[l];
        }
        S->n_req = acc;
        S->mode = 1;
        S->resident = acc;
    }
    st->planned = 1;
    st->decoded = S->n_req;
    st->freed = nfree;
    st->rebuilt = rebuild ? 1u : 0u;
    st->vox_lo = (uint32_t)vox;
    st->vox_hi = (uint32_t)(vox >> 32);
}

struct CacheArgs {
    uint32_t sid[kMaxViews];
    uint32_t n_views, nb, n_cta, max_lod;
    uint64_t n_slots;
    const uint8_t* bflag;
    const uint8_t* want;   // [session][brick]
    const uint8_t* need;
    const uint32_t* base;  // [kCnt][n_cta]
    const uint32_t* ids;
    uint8_t* res;
    uint64_t* off;         // [brick][kLods]
    uint64_t* stack;       // [kLods][nb]
    const ServeState* S;
    csv_request* reqs;
    csv_brick_slot* slots; // [session][n_slots]
    uint64_t pal_region;
};

__global__ void __launch_bounds__(kBlk) push_kernel(CacheArgs A) {
    __shared__ uint32_t s_wc[kWarps][kLods];
    __shared__ uint32_t s_tot[kLods];
    const uint32_t i = blockIdx.x * kBlk + threadIdx.x;
    const uint32_t mode = A.S->mode;
    uint32_t res = 0, need = 0;
    if (i < A.nb) {
        res = A.res[i];
        need = A.need[i];
    }
    if (mode == 1) {  // rebuild: every block is dropped
        if (i < A.nb && res) A.res[i] = 0;
        return;
    }
    const uint32_t fr = res & ~need;
    uint32_t rank[kLods];
    cta_ranks(fr, rank, s_wc, s_tot);
    if (i >= A.nb || !fr) return;
#pragma unroll
    for (uint32_t l = 1; l < kLods; ++l) {
        if (!((fr >> l) & 1u)) continue;
        const uint32_t pos = A.S->top_old[l] + A.base[(CNT_FREE + l) * A.n_cta + blockIdx.x] + rank[l];
        A.stack[(size_t)l * A.nb + pos] = A.off[(size_t)i * kLods + l];
    }
    A.res[i] = (uint8_t)(res & need);
}

__global__ void __launch_bounds__(kBlk) pop_kernel(CacheArgs A) {
    __shared__ uint32_t s_wc[kWarps][kLods];
    __shared__ uint32_t s_tot[kLods];
    const uint32_t i = blockIdx.x * kBlk + threadIdx.x;
    const uint32_t mode = A.S->mode;
    uint32_t res = 0, need = 0;
    if (i < A.nb) {
        res = A.res[i];
        need = A.need[i];
    }
    const uint32_t adm = mode == 0 ? (need & ~res) : need;
    uint32_t rank[kLods];
    cta_ranks(adm, rank, s_wc, s_tot);
    if (i >= A.nb) return;
    if (adm) {
#pragma unroll
        for (uint32_t l = 1; l < kLods; ++l) {
            if (!((adm >> l) & 1u)) continue;
            uint32_t k;
            uint64_t o;
            if (mode == 0) {
                k = A.base[(CNT_ALLOC + l) * A.n_cta + blockIdx.x] + rank[l];
                const uint32_t T = A.S->T[l];
                o = k < T ? A.stack[(size_t)l * A.nb + (T - 1 - k)] : A.S->base[l] + ((uint64_t)(k - T) << (3 * l));
            } else {
                k = A.base[(CNT_NEED + l) * A.n_cta + blockIdx.x] + rank[l];
                if (k >= A.S->fit[l]) continue;
                o = A.S->base[l] + ((uint64_t)k << (3 * l));
            }
            res |= 1u << l;
            A.off[(size_t)i * kLods + l] = o;
            csv_request q;
            q.brick = i;
            q.lod = l;
            q.dst = A.pal_region + o;
            A.reqs[A.S->req_base[l] + k] = q;
        }
        A.res[i] = (uint8_t)res;
    }
    const uint8_t bf = A.bflag[i];
    const uint32_t m = A.ids[i];
    for (uint32_t s = 0; s < A.n_views; ++s) {
        const uint32_t w = A.want[(size_t)A.sid[s] * A.nb + i];
        csv_brick_slot sl;
        sl.offset = 0;
        sl.lod = 0;
        sl.flags = 0;
        if (!(bf & BK_HAS)) sl.flags = CSV_SLOT_EMPTY;
        else if ((bf & BK_UNIFORM) || w == 0) sl.offset = i;
        else if (w != kNone && ((res >> w) & 1u)) {
            sl.offset = A.pal_region + A.off[(size_t)i * kLods + w];
            sl.lod = w;
        } else sl.flags = CSV_SLOT_MISSING;
        A.slots[(size_t)A.sid[s] * A.n_slots + m] = sl;
    }
}

struct CensusArgs {
    uint32_t sid[kMaxViews];
    uint32_t n_views, nb;
    uint64_t n_slots;
    const uint32_t* ids;
    uint32_t* req_words;  // [session][n_slots]
    uint32_t keep;        // admission by rays: leave the words for the next plan
    const ServeState* S;
    StepStats* st;
};

__global__ void __launch_bounds__(kBlk) census_kernel(CensusArgs A) {
    __shared__ uint32_t s_e[kMaxViews], s_m[kMaxViews];
    const uint32_t i = blockIdx.x * kBlk + threadIdx.x;
    if (threadIdx.x < kMaxViews) s_e[threadIdx.x] = s_m[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t m = i < A.nb ? A.ids[i] : 0u;
    for (uint32_t s = 0; s < A.n_views; ++s) {
        uint32_t v = 0;
        if (i < A.nb) {
            uint32_t* w = A.req_words + (size_t)A.sid[s] * A.n_slots + m;
            v = *w;
            if (v && !A.keep) *w = 0;
        }
        const uint32_t e = __popc(__ballot_sync(0xffffffffu, v != 0));
        const uint32_t ms = __popc(__ballot_sync(0xffffffffu, v == 3));
        if ((threadIdx.x & 31u) == 0) {
            if (e) atomicAdd(&s_e[s], e);
            if (ms) atomicAdd(&s_m[s], ms);
        }
    }
    __syncthreads();
    if (threadIdx.x < A.n_views) {
        if (s_e[threadIdx.x]) atomicAdd(&A.st->entered[threadIdx.x], s_e[threadIdx.x]);
        if (s_m[threadIdx.x]) atomicAdd(&A.st->missing[threadIdx.x], s_m[threadIdx.x]);
    }
    if (threadIdx.x == 0 && blockIdx.x == 0) A.st->resident = A.S->resident;
}

// Per brick: the palette-0 table, the transfer-function flag (culling.js:162-171)
// and the uniform flag.
__global__ void __launch_bounds__(kBlk) setup_kernel(const BrickDesc* __restrict__ bricks, const uint64_t* __restrict__ pal,
                                                     uint32_t nb, const uint64_t* __restrict__ hidden, uint32_t n_hidden,
                                                     uint64_t* __restrict__ cache, uint8_t* __restrict__ bflag,
                                                     uint32_t* __restrict__ ids) {
    const uint32_t i = blockIdx.x * kBlk + threadIdx.x;
    if (i >= nb) return;
    const BrickDesc br = bricks[i];
    const uint64_t* p = pal + br.pal_off;
    uint8_t f = (br.flags & BF_UNIFORM) ? BK_UNIFORM : 0;
    for (uint32_t k = 0; k < br.P; ++k) {
        const uint64_t v = p[k];
        if (v == 0) continue;
        uint32_t lo = 0, hi = n_hidden;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (hidden[mid] < v) lo = mid + 1;
            else hi = mid;
        }
        if (!(lo < n_hidden && hidden[lo] == v)) {
            f |= BK_HAS;
            break;
        }
    }
    bflag[i] = f;
    cache[i] = br.P ? p[0] : 0ull;
    ids[i] = br.id;
}

__global__ void slots_clear_kernel(csv_brick_slot* slots, uint64_t n) {
    for (uint64_t m = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; m < n; m += (uint64_t)gridDim.x * blockDim.x) {
        csv_brick_slot s;
        s.offset = 0;
        s.lod = 0;
        s.flags = CSV_SLOT_EMPTY;
        slots[m] = s;
    }
}

}  // namespace
}  // namespace csv

struct csv_server {
    csv_ctx* ctx = nullptr;
    const csv_dataset* ds = nullptr;
    uint32_t W = 0, H = 0, cone = 0, b = 0, max_lod = 0, nb = 0, bpa = 0, n_cta = 0, max_sessions = 1;
    uint32_t admit = CSV_ADMIT_CONE;
    double fov = 0, focal = 0, cos_half = 0, radius = 0;
    uint64_t total = 0, pal_region = 0, n_slots = 0;
    uint64_t* d_cache = nullptr;
    csv_brick_slot* d_slots = nullptr;  // [session][n_slots]
    uint32_t* d_req_words = nullptr;    // [session][n_slots]
    uint32_t* d_ids = nullptr;
    uint8_t* d_bflag = nullptr;
    uint8_t* d_res = nullptr;
    uint64_t* d_off = nullptr;
    uint8_t* d_want = nullptr;
    uint8_t* d_need = nullptr;
    uint64_t* d_stack = nullptr;
    uint32_t* d_cnt = nullptr;
    uint32_t* d_base = nullptr;
    ServeState* d_state = nullptr;
    csv_request* d_reqs = nullptr;
    uint32_t* d_status = nullptr;
    uint64_t* d_hidden = nullptr;
    uint32_t n_hidden = 0;
    // the colour path: the dataset's transfer function (hidden labels transparent) and the light
    uint64_t* d_tf_keys = nullptr;
    uint32_t* d_tf_rgba = nullptr;
    uint32_t n_tf = 0;
    csv_lighting light;
    StepStats* d_stats = nullptr;  // kRing slots
    StepStats* h_stats = nullptr;  // pinned mirror
    struct Session {
        bool open = false, pending = false, planned = false;
        bool ready = false;  // admission by rays: rendered since the last plan (request words on the device)
        double v[6];      // latest submitted camera (raw direction)
        double pv[6];     // camera of the session's last re-plan (unit direction)
        uint64_t* lab = nullptr;
        float* dep = nullptr;
        uint32_t* rgba = nullptr;  // set: the frame is an RGBA8 image (csv_serve_submit_rgba)
    };
    std::vector<Session> ses;
    std::vector<uint32_t> last_open;  // open sessions at the last plan
    struct StepRec {
        uint64_t seq = 0;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        std::vector<uint32_t> rendered;
    };
    StepRec ring[kRing];
    uint64_t next_seq = 0, harvest_seq = 0;
    std::deque<csv_frame_stats> done;
};

namespace {

int fail(csv_ctx* ctx, int code, const std::string& m) { return abi_fail(ctx, code, m); }
int cfail(csv_ctx* ctx, cudaError_t e, const char* w) { return abi_cuda_fail(ctx, e, w); }

void server_free(csv_server* s) {
    cudaFree(s->d_tf_keys);
    cudaFree(s->d_tf_rgba);
    cudaFree(s->d_cache);
    cudaFree(s->d_slots);
    cudaFree(s->d_req_words);
    cudaFree(s->d_ids);
    cudaFree(s->d_bflag);
    cudaFree(s->d_res);
    cudaFree(s->d_off);
    cudaFree(s->d_want);
    cudaFree(s->d_need);
    cudaFree(s->d_stack);
    cudaFree(s->d_cnt);
    cudaFree(s->d_base);
    cudaFree(s->d_state);
    cudaFree(s->d_reqs);
    cudaFree(s->d_status);
    cudaFree(s->d_hidden);
    cudaFree(s->d_stats);
    if (s->h_stats) cudaFreeHost(s->h_stats);
    for (auto& r : s->ring) {
        if (r.e0) cudaEventDestroy(r.e0);
        if (r.e1) cudaEventDestroy(r.e1);
    }
    delete s;
}

// culling.js:22-56: moved more than 0.5 units or turned more than 0.05 rad.
bool view_moved(const double* v, const double* p) {
    const double dx = v[0] - p[0], dy = v[1] - p[1], dz = v[2] - p[2];
    const double moved = dx * dx + dy * dy + dz * dz;
    const double dot = v[3] * p[3] + v[4] * p[4] + v[5] * p[5];
    return moved > 0.5 * 0.5 || dot < cos(0.05);
}

// camera.js:61-77 (getUniformData) in double, then float.
void camera_of(const double* v, double fov, csv_camera* c) {
    double f[3], r[3], u[3], wu[3];
    double n = sqrt(v[3] * v[3] + v[4] * v[4] + v[5] * v[5]);
    if (n == 0.0) n = 1.0;
    for (int a = 0; a < 3; ++a) f[a] = v[3 + a] / n;
    if (fabs(f[1]) > 0.999) {
        wu[0] = 1.0;
        wu[1] = 0.0;
        wu[2] = 0.0;
    } else {
        wu[0] = 0.0;
        wu[1] = 1.0;
        wu[2] = 0.0;
    }
    r[0] = f[1] * wu[2] - f[2] * wu[1];
    r[1] = f[2] * wu[0] - f[0] * wu[2];
    r[2] = f[0] * wu[1] - f[1] * wu[0];
    n = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    if (n == 0.0) n = 1.0;
    for (int a = 0; a < 3; ++a) r[a] /= n;
    u[0] = r[1] * f[2] - r[2] * f[1];
    u[1] = r[2] * f[0] - r[0] * f[2];
    u[2] = r[0] * f[1] - r[1] * f[0];
    n = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    if (n == 0.0) n = 1.0;
    for (int a = 0; a < 3; ++a) u[a] /= n;
    for (int a = 0; a < 3; ++a) {
        c->position[a] = (float)v[a];
        c->forward[a] = (float)f[a];
        c->right[a] = (float)r[a];
        c->up[a] = (float)u[a];
    }
    c->tan_half_fov = (float)tan(fov * 0.5);
    c->pad0 = c->pad1 = c->pad2 = 0.f;
}

// Move finished steps from the ring to the host queue (wait_all: block until
// every step finished; wait_one: block on the oldest only).
int harvest(csv_server* s, bool wait_all, bool wait_one) {
    while (s->harvest_seq < s->next_seq) {
        auto& r = s->ring[s->harvest_seq % kRing];
        cudaError_t e = (wait_all || wait_one) ? cudaEventSynchronize(r.e1) : cudaEventQuery(r.e1);
        if (e == cudaErrorNotReady) return CSV_OK;
        if (e != cudaSuccess) return cfail(s->ctx, e, "serve step");
        float ms = 0.f;
        cudaEventElapsedTime(&ms, r.e0, r.e1);
        const StepStats& t = s->h_stats[s->harvest_seq % kRing];
        for (size_t j = 0; j < r.rendered.size(); ++j) {
            csv_frame_stats f;
            memset(&f, 0, sizeof f);
            f.step = r.seq;
            f.session = r.rendered[j];
            f.planned = t.planned;
            f.visible = t.visible;
            f.decoded = t.decoded;
            f.freed = t.freed;
            f.resident = t.resident;
            f.rebuilt = t.rebuilt;
            f.entered = t.entered[j];
            f.missing = t.missing[j];
            f.decoded_voxels = (uint64_t)t.vox_lo | ((uint64_t)t.vox_hi << 32);
            f.ms = ms;
            s->done.push_back(f);
        }
        ++s->harvest_seq;
        wait_one = false;
    }
    return CSV_OK;
}

}  // namespace

extern "C" {

int csv_serve_create(csv_ctx* ctx, const csv_dataset* ds, const csv_serve_config* cfg, const uint64_t* hidden,
                     uint32_t n_hidden, csv_server** out) {
    if (!ctx || !ds || !cfg || !out) return CSV_EINVAL;
    *out = nullptr;
    if (cfg->width == 0 || cfg->height == 0 || !(cfg->fov > 0.0 && cfg->fov < 3.14159))
        return fail(ctx, CSV_EINVAL, "serve: viewport and field of view must be positive");
    const uint32_t ms = cfg->max_sessions ? cfg->max_sessions : 1u;
    if (ms > kMaxViews) return fail(ctx, CSV_ERANGE, "serve: at most 8 sessions per server");
    if (ds->d.mixed_b) return fail(ctx, CSV_EINVAL, "serve: one brick size per server");
    if (n_hidden && !hidden) return fail(ctx, CSV_EINVAL, "serve: hidden labels pointer is null");
    DeviceGuard g(ctx->device);
    const DeviceDataset& d = ds->d;
    csv_server* s = new (std::nothrow) csv_server();
    if (!s) return fail(ctx, CSV_ENOMEM, "serve: host allocation");
    s->ctx = ctx;
    s->ds = ds;
    s->W = cfg->width;
    s->H = cfg->height;
    s->cone = cfg->cone;
    if (cfg->admit > CSV_ADMIT_RAYS) {
        delete s;
        return fail(ctx, CSV_EINVAL, "serve: unknown admission policy");
    }
    s->admit = cfg->admit;
    s->fov = cfg->fov;
    s->b = d.b;
    s->nb = d.nb;
    s->max_sessions = ms;
    while ((1u << s->max_lod) < s->b) ++s->max_lod;
    const double screen = (double)std::min(s->W, s->H);
    s->focal = (screen / 2.0) / tan(s->fov / 2.0);
    if (s->cone == 0) {
        s->cos_half = cos(s->fov / 2.0);
    } else {
        const double a = (double)s->W / (double)s->H;
        s->cos_half = cos(atan(tan(s->fov / 2.0) * sqrt(a * a + 1.0)));
    }
    s->radius = sqrt(3.0) * ((double)s->b / 2.0);
    uint32_t maxc = 0;
    for (uint32_t i = 0; i < s->nb; ++i) {
        uint32_t id = d.h_ids[i], c[3] = {0, 0, 0};
        for (int bit = 0; bit < 10; ++bit)
            for (int a = 0; a < 3; ++a) c[a] |= ((id >> (3 * bit + a)) & 1u) << bit;
        maxc = std::max({maxc, c[0], c[1], c[2]});
    }
    s->bpa = maxc + 1;
    uint64_t p2 = 1;
    while (p2 < s->bpa) p2 <<= 1;
    s->n_slots = p2 * p2 * p2;
    s->n_cta = (s->nb + kBlk - 1) / kBlk;
    s->total = (cfg->cache_bytes ? cfg->cache_bytes : (24ull << 30)) / 8;
    s->pal_region = ((uint64_t)s->nb + 31) & ~31ull;
    if (s->total <= s->pal_region) {
        server_free(s);
        return fail(ctx, CSV_ERANGE, "serve: cache smaller than its palette table");
    }
    const size_t nbx = std::max<uint32_t>(s->nb, 1);
    const size_t ncx = std::max<uint32_t>(s->n_cta, 1);
    cudaError_t e = cudaSuccess;
    auto alloc = [&](void** p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, std::max<size_t>(bytes, 16));
    };
    alloc((void**)&s->d_cache, s->total * 8);
    alloc((void**)&s->d_slots, (size_t)ms * s->n_slots * sizeof(csv_brick_slot));
    alloc((void**)&s->d_req_words, (size_t)ms * s->n_slots * 4);
    alloc((void**)&s->d_ids, nbx * 4);
    alloc((void**)&s->d_bflag, nbx);
    alloc((void**)&s->d_res, nbx);
    alloc((void**)&s->d_off, nbx * kLods * 8);
    alloc((void**)&s->d_want, (size_t)kMaxViews * nbx);
    alloc((void**)&s->d_need, nbx);
    alloc((void**)&s->d_stack, (size_t)kLods * nbx * 8);
    alloc((void**)&s->d_cnt, (size_t)kCnt * ncx * 4);
    alloc((void**)&s->d_base, (size_t)kCnt * ncx * 4);
    alloc((void**)&s->d_state, sizeof(ServeState));
    alloc((void**)&s->d_reqs, nbx * kLods * sizeof(csv_request));
    alloc((void**)&s->d_status, nbx * kLods * 4);
    alloc((void**)&s->d_hidden, std::max<uint32_t>(n_hidden, 1) * 8);
    alloc((void**)&s->d_stats, kRing * sizeof(StepStats));
    if (e == cudaSuccess) e = cudaMallocHost((void**)&s->h_stats, kRing * sizeof(StepStats));
    if (e != cudaSuccess) {
        server_free(s);
        return fail(ctx, CSV_ENOMEM, std::string("serve: device allocation: ") + cudaGetErrorString(e));
    }
    for (auto& r : s->ring) {
        if (e == cudaSuccess) e = cudaEventCreate(&r.e0);
        if (e == cudaSuccess) e = cudaEventCreate(&r.e1);
    }
    if (e == cudaSuccess && n_hidden) {
        std::vector<uint64_t> h(hidden, hidden + n_hidden);
        std::sort(h.begin(), h.end());
        e = cudaMemcpy(s->d_hidden, h.data(), 8ull * n_hidden, cudaMemcpyHostToDevice);
    }
    s->n_hidden = n_hidden;
    if (e == cudaSuccess) {  // the transfer function of RGBA frames
        std::vector<uint64_t> k;
        std::vector<uint32_t> c;
        e = transfer_function(d, hidden, n_hidden, k, c);
        s->n_tf = (uint32_t)k.size();
        if (e == cudaSuccess) e = cudaMalloc(&s->d_tf_keys, 8 * std::max<size_t>(1, k.size()));
        if (e == cudaSuccess) e = cudaMalloc(&s->d_tf_rgba, 4 * std::max<size_t>(1, c.size()));
        if (e == cudaSuccess && !k.empty()) e = cudaMemcpy(s->d_tf_keys, k.data(), 8 * k.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess && !c.empty()) e = cudaMemcpy(s->d_tf_rgba, c.data(), 4 * c.size(), cudaMemcpyHostToDevice);
    }
    csv_lighting_default(25.0, &s->light);
    ServeState st0;
    memset(&st0, 0, sizeof st0);
    st0.cap = s->total - s->pal_region;
    if (e == cudaSuccess) e = cudaMemcpy(s->d_state, &st0, sizeof st0, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(s->d_res, 0, nbx);
    if (e == cudaSuccess) e = cudaMemset(s->d_req_words, 0, (size_t)ms * s->n_slots * 4);
    if (e == cudaSuccess && s->nb) {
        setup_kernel<<<s->n_cta, kBlk>>>(d.d_bricks, d.d_pal, s->nb, s->d_hidden, s->n_hidden, s->d_cache, s->d_bflag,
                                         s->d_ids);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        slots_clear_kernel<<<1024, 256>>>(s->d_slots, (uint64_t)ms * s->n_slots);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        server_free(s);
        return cfail(ctx, e, "serve: setup");
    }
    int rc = abi_ensure_scratch(ctx, s->b);
    if (rc) {
        server_free(s);
        return rc;
    }
    s->ses.resize(ms);
    *out = s;
    return CSV_OK;
}

int csv_serve_submit(csv_server* s, uint32_t session, const csv_view* view, uint64_t* d_label, float* d_depth) {
    if (!s || !view || !d_label || !d_depth) return CSV_EINVAL;
    if (session >= s->max_sessions) return fail(s->ctx, CSV_ERANGE, "serve: session id beyond max_sessions");
    auto& p = s->ses[session];
    p.open = true;     // a submit opens the session
    p.pending = true;  // a newer frame of the same session replaces one not yet stepped
    for (int a = 0; a < 3; ++a) {
        p.v[a] = view->position[a];
        p.v[3 + a] = view->direction[a];
    }
    p.lab = d_label;
    p.dep = d_depth;
    p.rgba = nullptr;
    return CSV_OK;
}

int csv_serve_submit_rgba(csv_server* s, uint32_t session, const csv_view* view, uint32_t* d_rgba) {
    if (!s || !view || !d_rgba) return CSV_EINVAL;
    if (session >= s->max_sessions) return fail(s->ctx, CSV_ERANGE, "serve: session id beyond max_sessions");
    auto& p = s->ses[session];
    p.open = true;
    p.pending = true;
    for (int a = 0; a < 3; ++a) {
        p.v[a] = view->position[a];
        p.v[3 + a] = view->direction[a];
    }
    p.lab = nullptr;
    p.dep = nullptr;
    p.rgba = d_rgba;
    return CSV_OK;
}

int csv_serve_set_lighting(csv_server* s, const csv_lighting* light) {
    if (!s || !light) return CSV_EINVAL;
    s->light = *light;  // used by the RGBA frames of the next steps
    return CSV_OK;
}

int csv_serve_close(csv_server* s, uint32_t session) {
    if (!s) return CSV_EINVAL;
    if (session >= s->max_sessions) return fail(s->ctx, CSV_ERANGE, "serve: session id beyond max_sessions");
    auto& p = s->ses[session];
    p.open = p.pending = p.planned = false;  // its blocks are released at the next step
    return CSV_OK;
}

int csv_serve_step(csv_server* s, void* stream, uint64_t* step_id) {
    if (!s) return CSV_EINVAL;
    cudaStream_t st = (cudaStream_t)stream;
    std::vector<uint32_t> open, rendered;
    bool changed = false;
    for (uint32_t k = 0; k < s->max_sessions; ++k) {
        auto& p = s->ses[k];
        if (!p.open) continue;
        open.push_back(k);
        if (p.pending) rendered.push_back(k);
        double n = sqrt(p.v[3] * p.v[3] + p.v[4] * p.v[4] + p.v[5] * p.v[5]);
        if (n == 0.0) n = 1.0;
        const double u[6] = {p.v[0], p.v[1], p.v[2], p.v[3] / n, p.v[4] / n, p.v[5] / n};
        if (!p.planned || view_moved(u, p.pv)) {
            memcpy(p.pv, u, sizeof u);
            p.planned = true;
            changed = true;
        }
    }
    if (open != s->last_open) changed = true;
    uint32_t ready = 0;  // admission by rays: views (plan order) with request words to apply
    if (s->admit == CSV_ADMIT_RAYS)
        for (size_t k = 0; k < open.size(); ++k)
            if (s->ses[open[k]].ready) {
                ready |= 1u << k;
                changed = true;
            }
    if (rendered.empty() && !changed) return fail(s->ctx, CSV_EINVAL, "serve: no frame submitted since the last step");
    DeviceGuard g(s->ctx->device);
    // a full ring: wait for the oldest step and keep its counters for csv_serve_poll
    if (s->next_seq - s->harvest_seq >= kRing) {
        int rc = harvest(s, false, true);
        if (rc) return rc;
    }
    const uint32_t slot = (uint32_t)(s->next_seq % kRing);
    auto& rec = s->ring[slot];
    StepStats* stats = s->d_stats + slot;
    cudaError_t e = cudaEventRecord(rec.e0, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(stats, 0, sizeof(StepStats), st);
    // a session that left with request words not yet applied: drop them
    for (uint32_t k = 0; k < s->max_sessions && e == cudaSuccess; ++k) {
        auto& p = s->ses[k];
        if (!p.open && p.ready) {
            e = cudaMemsetAsync(s->d_req_words + (size_t)k * s->n_slots, 0, s->n_slots * 4, st);
            p.ready = false;
        }
    }
    if (e == cudaSuccess && changed && s->nb) {
        PlanArgs P;
        memset(&P, 0, sizeof P);
        for (size_t k = 0; k < open.size(); ++k) {
            const auto& p = s->ses[open[k]];
            for (int a = 0; a < 3; ++a) {
                P.v[k].p[a] = p.pv[a];
                P.v[k].d[a] = p.pv[3 + a];
            }
            P.sid[k] = open[k];
        }
        P.n_views = (uint32_t)open.size();
        P.b = s->b;
        P.max_lod = s->max_lod;
        P.nb = s->nb;
        P.n_cta = s->n_cta;
        P.focal = s->focal;
        P.cos_half = s->cos_half;
        P.radius = s->radius;
        P.half = (double)s->b / 2.0;
        P.ids = s->d_ids;
        P.bflag = s->d_bflag;
        P.res = s->d_res;
        P.req_words = s->d_req_words;
        P.n_slots = s->n_slots;
        P.ready = (e == cudaSuccess) ? ready : 0u;
        P.want = s->d_want;
        P.need = s->d_need;
        P.cnt = s->d_cnt;
        P.stats = stats;
        plan_kernel<<<s->n_cta, kBlk, 0, st>>>(P);
        scan_kernel<<<1, 1024, 0, st>>>(s->d_cnt, s->d_base, s->n_cta, s->max_lod, s->nb, s->d_state, stats, 0u);
        for (size_t k = 0; k < open.size(); ++k)
            if ((ready >> k) & 1u) s->ses[open[k]].ready = false;  // consumed by this plan
        CacheArgs C;
        memset(&C, 0, sizeof C);
        for (size_t k = 0; k < open.size(); ++k) C.sid[k] = open[k];
        C.n_views = (uint32_t)open.size();
        C.nb = s->nb;
        C.n_cta = s->n_cta;
        C.max_lod = s->max_lod;
        C.n_slots = s->n_slots;
        C.bflag = s->d_bflag;
        C.want = s->d_want;
        C.need = s->d_need;
        C.base = s->d_base;
        C.ids = s->d_ids;
        C.res = s->d_res;
        C.off = s->d_off;
        C.stack = s->d_stack;
        C.S = s->d_state;
        C.reqs = s->d_reqs;
        C.slots = s->d_slots;
        C.pal_region = s->pal_region;
        push_kernel<<<s->n_cta, kBlk, 0, st>>>(C);
        pop_kernel<<<s->n_cta, kBlk, 0, st>>>(C);
        e = cudaGetLastError();
        if (e == cudaSuccess) {
            DecodeConfig dc;
            dc.n_dev = &s->d_state->n_req;
            e = launch_decode(s->ds->d, s->d_reqs, s->nb * kLods, s->d_cache, s->d_status, s->ctx->scr, st, &dc);
        }
        if (e == cudaSuccess) s->last_open = open;
    }
    for (size_t k = 0; k < rendered.size() && e == cudaSuccess; ++k) {
        const auto& p = s->ses[rendered[k]];
        csv_camera cam;
        camera_of(p.v, s->fov, &cam);
        if (p.rgba)
            e = launch_render_rgba(cam, s->W, s->H, (float)(s->bpa * s->b), s->b, s->bpa,
                                   s->d_slots + (size_t)rendered[k] * s->n_slots, s->n_slots, s->d_cache,
                                   s->n_tf ? s->d_tf_keys : nullptr, s->d_tf_rgba, s->n_tf, s->light.light_dir,
                                   s->light.ambient, s->light.diffuse, p.rgba,
                                   s->d_req_words + (size_t)rendered[k] * s->n_slots, st);
        else
            e = launch_render(cam, s->W, s->H, (float)(s->bpa * s->b), s->b, s->bpa,
                              s->d_slots + (size_t)rendered[k] * s->n_slots, s->n_slots, s->d_cache,
                              s->n_hidden ? s->d_hidden : nullptr, s->n_hidden, p.lab, p.dep,
                              s->d_req_words + (size_t)rendered[k] * s->n_slots, st);
    }
    if (e == cudaSuccess && s->nb && !rendered.empty()) {
        CensusArgs A;
        memset(&A, 0, sizeof A);
        for (size_t k = 0; k < rendered.size(); ++k) A.sid[k] = rendered[k];
        A.n_views = (uint32_t)rendered.size();
        A.nb = s->nb;
        A.n_slots = s->n_slots;
        A.ids = s->d_ids;
        A.req_words = s->d_req_words;
        A.keep = s->admit == CSV_ADMIT_RAYS ? 1u : 0u;
        A.S = s->d_state;
        A.st = stats;
        census_kernel<<<s->n_cta, kBlk, 0, st>>>(A);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->h_stats + slot, stats, sizeof(StepStats), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaEventRecord(rec.e1, st);
    if (e != cudaSuccess) return cfail(s->ctx, e, "serve step");
    rec.seq = s->next_seq;
    rec.rendered = rendered;
    if (step_id) *step_id = s->next_seq;
    ++s->next_seq;
    for (uint32_t k : rendered) {
        s->ses[k].pending = false;
        if (s->admit == CSV_ADMIT_RAYS) s->ses[k].ready = true;
    }
    return CSV_OK;
}

int csv_serve_compact(csv_server* s, void* stream) {
    if (!s) return CSV_EINVAL;
    if (!s->nb) return CSV_OK;
    cudaStream_t st = (cudaStream_t)stream;
    DeviceGuard g(s->ctx->device);
    if (s->next_seq - s->harvest_seq >= kRing) {
        int rc = harvest(s, false, true);
        if (rc) return rc;
    }
    const uint32_t slot = (uint32_t)(s->next_seq % kRing);
    auto& rec = s->ring[slot];
    StepStats* stats = s->d_stats + slot;
    cudaError_t e = cudaEventRecord(rec.e0, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(stats, 0, sizeof(StepStats), st);
    if (e == cudaSuccess) {
        compact_plan_kernel<<<s->n_cta, kBlk, 0, st>>>(s->d_res, s->d_need, s->nb, s->d_cnt, s->n_cta);
        scan_kernel<<<1, 1024, 0, st>>>(s->d_cnt, s->d_base, s->n_cta, s->max_lod, s->nb, s->d_state, stats, 1u);
        CacheArgs C;
        memset(&C, 0, sizeof C);
        // the slot tables of the sessions open at the last plan, whose wants stand
        for (size_t k = 0; k < s->last_open.size(); ++k) C.sid[k] = s->last_open[k];
        C.n_views = (uint32_t)s->last_open.size();
        C.nb = s->nb;
        C.n_cta = s->n_cta;
        C.max_lod = s->max_lod;
        C.n_slots = s->n_slots;
        C.bflag = s->d_bflag;
        C.want = s->d_want;
        C.need = s->d_need;
        C.base = s->d_base;
        C.ids = s->d_ids;
        C.res = s->d_res;
        C.off = s->d_off;
        C.stack = s->d_stack;
        C.S = s->d_state;
        C.reqs = s->d_reqs;
        C.slots = s->d_slots;
        C.pal_region = s->pal_region;
        push_kernel<<<s->n_cta, kBlk, 0, st>>>(C);
        pop_kernel<<<s->n_cta, kBlk, 0, st>>>(C);
        e = cudaGetLastError();
        if (e == cudaSuccess) {
            DecodeConfig dc;
            dc.n_dev = &s->d_state->n_req;
            e = launch_decode(s->ds->d, s->d_reqs, s->nb * kLods, s->d_cache, s->d_status, s->ctx->scr, st, &dc);
        }
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->h_stats + slot, stats, sizeof(StepStats), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaEventRecord(rec.e1, st);
    if (e != cudaSuccess) return cfail(s->ctx, e, "serve compact");
    rec.seq = s->next_seq;
    rec.rendered.clear();  // no frame
    ++s->next_seq;
    return CSV_OK;
}

int csv_serve_poll(csv_server* s, csv_frame_stats* out, uint32_t max, uint32_t* n_out, int wait) {
    if (!s || !n_out || (max && !out)) return CSV_EINVAL;
    *n_out = 0;
    DeviceGuard g(s->ctx->device);
    int rc = harvest(s, wait != 0, false);
    if (rc) return rc;
    uint32_t n = 0;
    while (n < max && !s->done.empty()) {
        out[n++] = s->done.front();
        s->done.pop_front();
    }
    *n_out = n;
    return CSV_OK;
}

int csv_serve_camera(const csv_server* s, const csv_view* view, csv_camera* out) {
    if (!s || !view || !out) return CSV_EINVAL;
    double v[6] = {view->position[0], view->position[1], view->position[2],
                   view->direction[0], view->direction[1], view->direction[2]};
    camera_of(v, s->fov, out);
    return CSV_OK;
}

int csv_serve_state(const csv_server* s, uint32_t session, csv_serve_info* info) {
    if (!s || !info) return CSV_EINVAL;
    if (session >= s->max_sessions) return fail(s->ctx, CSV_ERANGE, "serve: session id beyond max_sessions");
    info->slots = s->d_slots + (size_t)session * s->n_slots;
    info->n_slots = s->n_slots;
    info->cache = s->d_cache;
    info->cache_labels = s->total;
    info->palette_table = s->pal_region;
    info->bricks_per_axis = s->bpa;
    info->brick_size = s->b;
    info->grid_size = (float)(s->bpa * s->b);
    info->focal = s->focal;
    info->cos_half = s->cos_half;
    info->decode_status = s->d_status;
    return CSV_OK;
}

int csv_serve_destroy(csv_server* s) {
    if (!s) return CSV_OK;
    DeviceGuard g(s->ctx->device);
    for (uint64_t q = s->harvest_seq; q < s->next_seq; ++q) cudaEventSynchronize(s->ring[q % kRing].e1);
    server_free(s);
    return CSV_OK;
}

}  // extern "C"
