// abi.cu -- the C ABI (include/csv.h): contexts, .csbd staging, and launches.
//
// Host-side work here is parsing and bookkeeping only; every codec step runs
// in the sm_100a kernels of decode.cu / encode.cu.  There is no CPU decode or
// encode path: without a usable CUDA device every call fails with CSV_ECUDA.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <new>
#include <string>
#include <vector>

#include "abi_internal.h"
#include "csv_internal.h"

using namespace csv;

namespace csv {

int abi_fail(csv_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return code;
}
int abi_cuda_fail(csv_ctx* ctx, cudaError_t e, const char* where) {
    return abi_fail(ctx, CSV_ECUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

cudaError_t transfer_function(const DeviceDataset& d, const uint64_t* hidden, uint32_t n_hidden,
                              std::vector<uint64_t>& keys, std::vector<uint32_t>& rgba) {
    // buildTransferFunctionBuffers (webgpuSetup.js:389-465): every distinct non-zero
    // palette label of the dataset, ascending; entry i gets hue 137.5 i (golden
    // angle), saturation, lightness and opacity cycling with i, HSL -> RGB
    // (hslToRgb, :490-515), RGB scaled by 0.92 for lighting headroom
    std::vector<uint64_t> pal(d.pal_pool_entries);
    if (!pal.empty()) {
        cudaError_t e = cudaMemcpy(pal.data(), d.d_pal, 8 * pal.size(), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return e;
    }
    std::sort(pal.begin(), pal.end());
    pal.erase(std::unique(pal.begin(), pal.end()), pal.end());
    if (!pal.empty() && pal[0] == 0) pal.erase(pal.begin());
    keys.resize(pal.size());
    rgba.resize(pal.size());
    std::vector<uint64_t> hid(hidden, hidden + n_hidden);
    std::sort(hid.begin(), hid.end());
    auto js_round = [](double x) { return floor(x + 0.5); };  // Math.round
    for (size_t i = 0; i < pal.size(); ++i) {
        const double h = fmod((double)i * 137.5, 360.0);
        const double sat = 0.55 + (double)(i % 3) * 0.08, lig = 0.35 + (double)(i % 4) * 0.05;
        const double op = 0.25 + (double)(i % 5) * 0.08;
        const double c = (1 - fabs(2 * lig - 1)) * sat;
        const double x = c * (1 - fabs(fmod(h / 60, 2) - 1));
        const double m = lig - c / 2;
        double r, gg, b;
        if (h < 60) { r = c; gg = x; b = 0; }
        else if (h < 120) { r = x; gg = c; b = 0; }
        else if (h < 180) { r = 0; gg = c; b = x; }
        else if (h < 240) { r = 0; gg = x; b = c; }
        else if (h < 300) { r = x; gg = 0; b = c; }
        else { r = c; gg = 0; b = x; }
        const double rr = js_round((r + m) * 255), rg = js_round((gg + m) * 255), rb = js_round((b + m) * 255);
        const uint32_t R = (uint32_t)std::min(floor(rr * 0.92), 255.0), G = (uint32_t)std::min(floor(rg * 0.92), 255.0),
                       B = (uint32_t)std::min(floor(rb * 0.92), 255.0), A = (uint32_t)floor(op * 255);
        keys[i] = pal[i];
        // a hidden label is transparent (rebuildLabelColors, webgpuSetup.js:826-834)
        rgba[i] = std::binary_search(hid.begin(), hid.end(), pal[i]) ? 0u : (R | (G << 8) | (B << 16) | (A << 24));
    }
    return cudaSuccess;
}

int abi_ensure_scratch(csv_ctx* ctx, uint32_t b) {
    if (ctx->scr.base && ctx->scr_b >= b) return CSV_OK;
    size_t per = decode_scratch_per_cta(b);
    uint32_t ctas = decode_grid(ctx->device, 0xFFFFFFFFu);
    const size_t bytes = decode_scratch_bytes(ctx->device, b);
    cudaFree(ctx->scr.base);
    ctx->scr.base = nullptr;
    cudaError_t e = cudaMalloc(&ctx->scr.base, bytes);
    if (e != cudaSuccess) return abi_fail(ctx, CSV_ENOMEM, std::string("decode scratch: ") + cudaGetErrorString(e));
    if (!ctx->scr.d_queue) {
        e = cudaMalloc(&ctx->scr.d_queue, 64);
        if (e != cudaSuccess) return abi_fail(ctx, CSV_ENOMEM, "decode queue");
    }
    ctx->scr.per_cta = per;
    ctx->scr.ctas = ctas;
    ctx->scr.bytes = bytes;
    ctx->scr_b = b;
    return CSV_OK;
}

int abi_ensure_scratch_small(csv_ctx* ctx) {
    if (ctx->scr_small.base) return CSV_OK;
    const size_t bytes = decode_scratch_small_bytes(ctx->device);
    cudaError_t e = cudaMalloc(&ctx->scr_small.base, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->scr_small.d_queue, 64);
    if (e != cudaSuccess) {
        cudaFree(ctx->scr_small.base);
        ctx->scr_small.base = nullptr;
        return abi_fail(ctx, CSV_ENOMEM, std::string("decode scratch: ") + cudaGetErrorString(e));
    }
    ctx->scr_small.per_cta = decode_scratch_per_cta(1u << kSmallLod, kSmallLod);
    ctx->scr_small.ctas = (uint32_t)(bytes / ctx->scr_small.per_cta);
    ctx->scr_small.bytes = bytes;
    return CSV_OK;
}

int abi_ensure_scratch_wide(csv_ctx* ctx, uint32_t b) {
    if (ctx->scr_wide.base && ctx->scr_wide_b >= b) return CSV_OK;
    cudaFree(ctx->scr_wide.base);
    cudaFree(ctx->scr_wide.d_queue);
    ctx->scr_wide = DecodeScratch();
    ctx->scr_wide_b = 0;
    const size_t bytes = decode_scratch_wide_bytes(ctx->device, b);
    cudaError_t e = cudaMalloc(&ctx->scr_wide.base, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->scr_wide.d_queue, 64);
    if (e != cudaSuccess) {
        cudaFree(ctx->scr_wide.base);
        ctx->scr_wide = DecodeScratch();
        return abi_fail(ctx, CSV_ENOMEM, std::string("decode scratch: ") + cudaGetErrorString(e));
    }
    ctx->scr_wide.per_cta = decode_scratch_per_cta(b);  // the 64^3 variant's layout
    ctx->scr_wide.ctas = (uint32_t)(bytes / ctx->scr_wide.per_cta);
    ctx->scr_wide.bytes = bytes;
    ctx->scr_wide_b = b;
    return CSV_OK;
}

}  // namespace csv

namespace {

int fail(csv_ctx* ctx, int code, const std::string& msg) { return abi_fail(ctx, code, msg); }
int cuda_fail(csv_ctx* ctx, cudaError_t e, const char* where) { return abi_cuda_fail(ctx, e, where); }
int ensure_scratch(csv_ctx* ctx, uint32_t b) { return abi_ensure_scratch(ctx, b); }

uint32_t rd32(const uint8_t* p) {
    uint32_t v;
    memcpy(&v, p, 4);
    return v;
}

// Host view of a .csbd image: version 1 (fileIO.cpp:25-96, datasetLoader.js:39-146),
// or version 2, which carries up to 16 shared rANS tables (28-byte header, then
// freq[16] and cum[16] per table) and, after each brick's ID, a u32 naming the
// brick's table (bits 4..7) and encoding mode (bits 0..3).
struct ImageView {
    uint32_t version = 1, nb = 0, b = 0, total = 0, n_tables = 1;
    size_t image_len = 0;  // bytes up to the end of the last brick record
    uint32_t freq[16][16], cum[16][16];
    struct Rec {
        size_t pal_at, enc_at;
        uint32_t id, P, E, nsym, sel;
    };
    std::vector<Rec> recs;
};

int parse_image(csv_ctx* ctx, const uint8_t* img, size_t len, ImageView& v) {
    if (!img || len < 28) return fail(ctx, CSV_EFORMAT, "image shorter than its header");
    if (rd32(img) != kMagic) return fail(ctx, CSV_EFORMAT, "Invalid file format (bad magic)");
    v.version = rd32(img + 4);
    if (v.version != 1 && v.version != 2) return fail(ctx, CSV_EFORMAT, "unsupported .csbd version");
    v.nb = rd32(img + 8);
    v.b = rd32(img + 12);
    if (v.b < 2 || v.b > 64 || (v.b & (v.b - 1)))
        return fail(ctx, CSV_EFORMAT, "brick size must be a power of two in [2, 64]");
    if (rd32(img + 16) != 16) return fail(ctx, CSV_EFORMAT, "symbol count must be 16");
    v.total = rd32(img + 20);
    if (v.total != kTot) return fail(ctx, CSV_EFORMAT, "total frequency must be 4096");
    size_t o;
    if (v.version == 1) {
        if (len < kHeaderBytes) return fail(ctx, CSV_EFORMAT, "image shorter than the 152-byte header");
        v.n_tables = 1;
        for (int i = 0; i < 16; ++i) {
            v.freq[0][i] = rd32(img + 24 + 4 * i);
            v.cum[0][i] = rd32(img + 88 + 4 * i);
        }
        o = kHeaderBytes;
    } else {
        v.n_tables = rd32(img + 24);
        if (v.n_tables == 0 || v.n_tables > 16) return fail(ctx, CSV_EFORMAT, "version 2: 1..16 tables");
        o = 28 + 128ull * v.n_tables;
        if (len < o) return fail(ctx, CSV_EFORMAT, "truncated table header");
        for (uint32_t t = 0; t < v.n_tables; ++t)
            for (int i = 0; i < 16; ++i) {
                v.freq[t][i] = rd32(img + 28 + 128 * t + 4 * i);
                v.cum[t][i] = rd32(img + 28 + 128 * t + 64 + 4 * i);
            }
    }
    for (uint32_t t = 0; t < v.n_tables; ++t)
        for (int i = 0; i < 16; ++i)
            if (v.freq[t][i] > kTot || v.cum[t][i] >= kTot)
                return fail(ctx, CSV_EFORMAT, "rANS model entry out of range");
    v.recs.resize(v.nb);
    for (uint32_t i = 0; i < v.nb; ++i) {
        ImageView::Rec& r = v.recs[i];
        r.sel = 0;
        if (o + 8 > len) return fail(ctx, CSV_EFORMAT, "truncated brick header");
        r.id = rd32(img + o);
        if (v.version == 2) {
            r.sel = rd32(img + o + 4);
            if (((r.sel >> 4) & 15u) >= v.n_tables) return fail(ctx, CSV_EFORMAT, "brick names a missing table");
            o += 4;
            if (o + 8 > len) return fail(ctx, CSV_EFORMAT, "truncated brick header");
        }
        r.P = rd32(img + o + 4);
        if (r.P == 0 || r.P > kMaxPalette) return fail(ctx, CSV_EFORMAT, "palette size out of range");
        r.pal_at = o + 8;
        o += 8 + 8ull * r.P;
        if (o + 4 > len) return fail(ctx, CSV_EFORMAT, "truncated palette");
        r.E = rd32(img + o);
        r.enc_at = o + 4;
        o += 4 + (size_t)r.E;
        if (o + 4 > len) return fail(ctx, CSV_EFORMAT, "truncated stream");
        r.nsym = rd32(img + o);
        o += 4;
    }
    v.image_len = o;
    return CSV_OK;
}

void free_dataset(DeviceDataset& d) {
    cudaFree(d.d_bricks);
    cudaFree(d.d_pal);
    cudaFree(d.d_enc);
    cudaFree(d.d_ck);
    cudaFree(d.d_lut);
    free(d.h_ids);
    free(d.h_cost);
    d = DeviceDataset();
}


// The image's palettes and streams into their device pools: one block per brick, from a device copy of
// the image (records are byte-aligned there: a palette entry is read a byte at a time).
__global__ void __launch_bounds__(128) stage_gather_kernel(const uint8_t* __restrict__ img,
                                                          const uint64_t* __restrict__ src,
                                                          const BrickDesc* __restrict__ bricks, uint32_t nb,
                                                          uint64_t* __restrict__ pal, uint8_t* __restrict__ enc) {
    const uint32_t i = blockIdx.x;
    if (i >= nb) return;
    const BrickDesc& b = bricks[i];
    const uint8_t* ps = img + src[2 * i];
    for (uint32_t k = threadIdx.x; k < b.P; k += blockDim.x) {
        uint64_t x = 0;
#pragma unroll
        for (int j = 7; j >= 0; --j) x = (x << 8) | ps[8ull * k + j];
        pal[b.pal_off + k] = x;
    }
    const uint8_t* es = img + src[2 * i + 1];
    for (uint32_t j = threadIdx.x; j < b.E; j += blockDim.x) enc[b.enc_off + j] = es[j];
}

int stage_dataset(csv_ctx* ctx, const uint8_t* img, const ImageView& v, DeviceDataset& d, cudaStream_t st) {
    d.device = ctx->device;
    d.pool = ctx->pool;
    d.nb = v.nb;
    d.b = v.b;
    d.L = levels_of(v.b);
    d.S = kOpsPerCheckpoint;
    d.total = v.total;
    memcpy(d.freq, v.freq[0], sizeof d.freq);
    memcpy(d.cum, v.cum[0], sizeof d.cum);
    d.n_models = v.n_tables;
    std::vector<BrickDesc> desc(v.nb);
    uint64_t pal_n = 0, enc_n = 0, ck_n = 0;
    d.h_ids = (uint32_t*)malloc(sizeof(uint32_t) * std::max<uint32_t>(1, v.nb));
    d.h_cost = (uint32_t*)malloc(sizeof(uint32_t) * std::max<uint32_t>(1, v.nb));
    for (uint32_t i = 0; i < v.nb; ++i) {
        const auto& r = v.recs[i];
        BrickDesc& b = desc[i];
        memset(&b, 0, sizeof b);
        b.pal_off = pal_n;
        b.enc_off = enc_n;
        b.P = r.P;
        b.E = r.E;
        b.nsym = r.nsym;
        b.id = r.id;
        b.ck_off = (uint32_t)ck_n;
        b.ck_cap = (r.nsym + d.S - 1) / d.S + 1;
        b.flags = BF_NOINDEX | (d.L << BF_LEVELS_SHIFT) | (((r.sel >> 4) & 15u) << BF_MODEL_SHIFT);
        d.h_ids[i] = r.id;
        d.h_cost[i] = r.nsym;
        pal_n += r.P;
        enc_n += (r.E + 15) & ~15ull;
        ck_n += b.ck_cap;
        d.max_nsym = std::max(d.max_nsym, r.nsym);
        d.max_P = std::max(d.max_P, r.P);
    }
    if (ck_n > 0xFFFFFFFFull) return fail(ctx, CSV_ERANGE, "dataset too large for the seek index");
    d.stream_bytes = 0;
    for (auto& r : v.recs) d.stream_bytes += r.E;
    d.palette_entries = pal_n;
    d.ck_entries = ck_n;
    d.enc_pool_bytes = std::max<uint64_t>(16, enc_n);
    d.pal_pool_entries = std::max<uint64_t>(1, pal_n);
    // where each brick's palette and stream start in the image (the pools are gathered on the device
    // from one copy of the image, instead of repacked on the host)
    std::vector<uint64_t> src(2 * (size_t)std::max<uint32_t>(1, v.nb));
    for (uint32_t i = 0; i < v.nb; ++i) {
        src[2 * i] = v.recs[i].pal_at;
        src[2 * i + 1] = v.recs[i].enc_at;
    }
    std::vector<uint32_t> lut((size_t)kTot * v.n_tables);
    for (uint32_t t = 0; t < v.n_tables; ++t) build_lut(v.freq[t], v.cum[t], &lut[(size_t)t * kTot]);
    d.fast_models = lut_fast_mask(lut.data(), v.n_tables);
    cudaError_t e;
    if ((e = cudaMalloc(&d.d_bricks, sizeof(BrickDesc) * std::max<uint32_t>(1, v.nb))) != cudaSuccess ||
        (e = cudaMalloc(&d.d_pal, 8 * d.pal_pool_entries)) != cudaSuccess ||
        (e = cudaMalloc(&d.d_enc, d.enc_pool_bytes)) != cudaSuccess ||
        (e = cudaMalloc(&d.d_ck, sizeof(Checkpoint) * std::max<uint64_t>(1, ck_n))) != cudaSuccess ||
        (e = cudaMalloc(&d.d_lut, sizeof(uint32_t) * lut.size())) != cudaSuccess)
        return fail(ctx, CSV_ENOMEM, std::string("device allocation: ") + cudaGetErrorString(e));
    uint8_t* d_img = nullptr;
    uint64_t* d_src = nullptr;
    if ((e = tmp_alloc((void**)&d_img, std::max<size_t>(1, v.image_len), d.pool, st)) != cudaSuccess ||
        (e = tmp_alloc((void**)&d_src, 8 * src.size(), d.pool, st)) != cudaSuccess) {
        cudaFreeAsync(d_img, st);
        cudaStreamSynchronize(st);
        return fail(ctx, CSV_ENOMEM, std::string("device allocation: ") + cudaGetErrorString(e));
    }
    if ((e = cudaMemcpyAsync(d.d_bricks, desc.data(), sizeof(BrickDesc) * v.nb, cudaMemcpyHostToDevice, st)) ==
            cudaSuccess &&
        (e = cudaMemcpyAsync(d_img, img, v.image_len, cudaMemcpyHostToDevice, st)) == cudaSuccess &&
        (e = cudaMemcpyAsync(d_src, src.data(), 8 * src.size(), cudaMemcpyHostToDevice, st)) == cudaSuccess &&
        (e = cudaMemcpyAsync(d.d_lut, lut.data(), sizeof(uint32_t) * lut.size(), cudaMemcpyHostToDevice, st)) ==
            cudaSuccess &&
        (e = cudaMemsetAsync(d.d_enc, 0, d.enc_pool_bytes, st)) == cudaSuccess && v.nb) {
        stage_gather_kernel<<<v.nb, 128, 0, st>>>(d_img, d_src, d.d_bricks, v.nb, d.d_pal, d.d_enc);
        e = cudaGetLastError();
    }
    cudaFreeAsync(d_img, st);
    cudaFreeAsync(d_src, st);
    // the host vectors go out of scope: finish the copies first
    const cudaError_t e2 = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) return cuda_fail(ctx, e, "staging copy");
    return CSV_OK;
}

// Seek-index sidecar (little endian): u32 magic "CSVX", u32 version 1, u32 bricks,
// u32 symbols between states (kSeedSymbols), u64 states in all; per brick u32 E,
// u32 nSymbols, u32 states (0, or one per kSeedSymbols symbols begun); then the
// states {u32 x, u32 pos}, brick after brick.
constexpr uint32_t kSidecarMagic = 0x58565343u;  // "CSVX"
constexpr size_t kSidecarHead = 24;

// The pieces of pass 1 a sidecar gives for image v, or an error naming the mismatch.
int sidecar_pieces(csv_ctx* ctx, const ImageView& v, const uint8_t* sc, size_t len, IndexSeeds& out) {
    if (!sc || len < kSidecarHead) return fail(ctx, CSV_EFORMAT, "index sidecar shorter than its header");
    uint64_t total;
    memcpy(&total, sc + 16, 8);
    if (rd32(sc) != kSidecarMagic || rd32(sc + 4) != 1)
        return fail(ctx, CSV_EFORMAT, "not a version-1 index sidecar");
    if (rd32(sc + 8) != v.nb || rd32(sc + 12) != kSeedSymbols)
        return fail(ctx, CSV_EFORMAT, "index sidecar does not match the image: brick count or state spacing");
    if (total > 0xFFFFFFFFull || len != kSidecarHead + 12ull * v.nb + 8 * total)
        return fail(ctx, CSV_EFORMAT, "index sidecar length does not match its header");
    out.piece_base.assign((size_t)v.nb + 1, 0);
    out.seed.clear();
    out.seed.reserve((size_t)total + v.nb);
    const uint8_t* states = sc + kSidecarHead + 12ull * v.nb;
    uint64_t used = 0;
    for (uint32_t i = 0; i < v.nb; ++i) {
        const uint8_t* r = sc + kSidecarHead + 12ull * i;
        const uint32_t E = rd32(r), ns = rd32(r + 4), n = rd32(r + 8);
        const uint32_t full = (ns + kSeedSymbols - 1) / kSeedSymbols;
        if (E != v.recs[i].E || ns != v.recs[i].nsym || (n != 0 && n != full) || used + n > total)
            return fail(ctx, CSV_EFORMAT, "index sidecar does not match the image at brick " + std::to_string(i));
        if (n == 0) {
            out.seed.push_back(make_uint2(0, 0xFFFFFFFFu));  // one piece, from the stream header
        } else {
            for (uint32_t k = 0; k < n; ++k)
                out.seed.push_back(make_uint2(rd32(states + 8 * (used + k)), rd32(states + 8 * (used + k) + 4)));
        }
        used += n;
        out.piece_base[i + 1] = (uint32_t)out.seed.size();
    }
    if (used != total) return fail(ctx, CSV_EFORMAT, "index sidecar holds states for no brick");
    return CSV_OK;
}

// csv_open and csv_open_indexed: stage the image, then the seek index from the
// stream headers or from a sidecar's states.
int open_dataset(csv_ctx* ctx, const uint8_t* image, size_t len, const uint8_t* sidecar, size_t sidecar_len,
                 csv_dataset** out) {
    if (!ctx || !out) return CSV_EINVAL;
    *out = nullptr;
    DeviceGuard g(ctx->device);
    ImageView v;
    int rc = parse_image(ctx, image, len, v);
    if (rc) return rc;
    IndexSeeds seeds;
    if (sidecar && (rc = sidecar_pieces(ctx, v, sidecar, sidecar_len, seeds))) return rc;
    csv_dataset* ds = new (std::nothrow) csv_dataset();
    if (!ds) return fail(ctx, CSV_ENOMEM, "host allocation");
    ds->ctx = ctx;
    cudaStream_t st = 0;
    rc = stage_dataset(ctx, image, v, ds->d, st);
    if (rc == CSV_OK) {
        // the passes' device time, from events on the stream around them
        cudaEvent_t ev[2] = {nullptr, nullptr};
        const bool timed = cudaEventCreate(&ev[0]) == cudaSuccess && cudaEventCreate(&ev[1]) == cudaSuccess;
        if (timed) cudaEventRecord(ev[0], st);
        bool rejected = false;
        cudaError_t e = launch_build_index(ds->d, st, sidecar ? &seeds : nullptr, &rejected);
        if (timed) cudaEventRecord(ev[1], st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "seek index");
        else if (rejected)
            rc = fail(ctx, CSV_EFORMAT, "index sidecar does not match the image: a stored rANS state differs");
        float ms = 0;
        if (rc == CSV_OK && timed && cudaEventElapsedTime(&ms, ev[0], ev[1]) == cudaSuccess) ds->d.index_ms = ms;
        for (cudaEvent_t x : ev)
            if (x) cudaEventDestroy(x);
    }
    if (rc) {
        free_dataset(ds->d);
        delete ds;
        return rc;
    }
    *out = ds;
    return CSV_OK;
}

}  // namespace

extern "C" {

int csv_abi_version(void) { return CSV_ABI_VERSION; }

void csv_free(void* p) { free(p); }

int csv_create(int device, csv_ctx** out) {
    if (!out) return CSV_EINVAL;
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || device < 0 || device >= n) return CSV_ECUDA;
    csv_ctx* c = new (std::nothrow) csv_ctx();
    if (!c) return CSV_ENOMEM;
    c->device = device;
    DeviceGuard g(device);
    if ((e = cudaFree(nullptr)) != cudaSuccess) {
        delete c;
        return CSV_ECUDA;
    }
    // The temporaries of each open (the image copy, the seek index's nibbles and snapshots: ~130 MB for
    // a 27.9 MB image) come from a pool of the context that keeps up to 1 GiB of freed memory, so that
    // the next open does not map it again; without a pool, the device's default one.
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if (cudaMemPoolCreate(&c->pool, &props) == cudaSuccess) {
        uint64_t keep = 1ull << 30;
        cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    } else {
        c->pool = nullptr;
        cudaGetLastError();
    }
    *out = c;
    return CSV_OK;
}

void csv_destroy(csv_ctx* ctx) {
    if (!ctx) return;
    DeviceGuard g(ctx->device);
    cudaFree(ctx->scr.base);
    cudaFree(ctx->scr.d_queue);
    cudaFree(ctx->scr_small.base);
    cudaFree(ctx->scr_small.d_queue);
    cudaFree(ctx->scr_wide.base);
    cudaFree(ctx->scr_wide.d_queue);
    for (int i = 0; i < 2; ++i) {
        cudaFree(ctx->chunk_buf[i]);
        if (ctx->pipe_stream[i]) cudaStreamDestroy(ctx->pipe_stream[i]);
    }
    for (cudaEvent_t ev : ctx->pipe_event)
        if (ev) cudaEventDestroy(ev);
    encoder_state_free(ctx->enc);
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    delete ctx;
}

const char* csv_last_error(const csv_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int csv_open(csv_ctx* ctx, const uint8_t* image, size_t len, csv_dataset** out) {
    return open_dataset(ctx, image, len, nullptr, 0, out);
}

int csv_open_indexed(csv_ctx* ctx, const uint8_t* image, size_t len, const uint8_t* sidecar, size_t sidecar_len,
                     csv_dataset** out) {
    if (!sidecar) return ctx ? fail(ctx, CSV_EINVAL, "null index sidecar") : CSV_EINVAL;
    return open_dataset(ctx, image, len, sidecar, sidecar_len, out);
}

int csv_index_save(csv_ctx* ctx, const csv_dataset* ds, uint8_t** out, size_t* out_len) {
    if (!ctx || !ds || !out || !out_len) return CSV_EINVAL;
    *out = nullptr;
    *out_len = 0;
    DeviceGuard g(ctx->device);
    std::vector<uint32_t> n_seeds;
    std::vector<uint2> seeds;
    cudaError_t e = index_seeds_of(ds->d, 0, n_seeds, seeds);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "index sidecar");
    const uint32_t nb = ds->d.nb;
    std::vector<BrickDesc> desc(nb);
    if (nb && (e = cudaMemcpy(desc.data(), ds->d.d_bricks, sizeof(BrickDesc) * nb, cudaMemcpyDeviceToHost)) !=
                  cudaSuccess)
        return cuda_fail(ctx, e, "index sidecar");
    const size_t len = kSidecarHead + 12ull * nb + 8ull * seeds.size();
    uint8_t* buf = (uint8_t*)malloc(len);
    if (!buf) return fail(ctx, CSV_ENOMEM, "host allocation");
    auto wr32 = [&](size_t at, uint32_t x) { memcpy(buf + at, &x, 4); };
    wr32(0, kSidecarMagic);
    wr32(4, 1);
    wr32(8, nb);
    wr32(12, kSeedSymbols);
    const uint64_t total = seeds.size();
    memcpy(buf + 16, &total, 8);
    for (uint32_t i = 0; i < nb; ++i) {
        wr32(kSidecarHead + 12ull * i, desc[i].E);
        wr32(kSidecarHead + 12ull * i + 4, desc[i].nsym);
        wr32(kSidecarHead + 12ull * i + 8, n_seeds[i]);
    }
    for (size_t k = 0; k < seeds.size(); ++k) {
        wr32(kSidecarHead + 12ull * nb + 8 * k, seeds[k].x);
        wr32(kSidecarHead + 12ull * nb + 8 * k + 4, seeds[k].y);
    }
    *out = buf;
    *out_len = len;
    return CSV_OK;
}

int csv_dataset_info_get(const csv_dataset* ds, csv_dataset_info* info) {
    if (!ds || !info) return CSV_EINVAL;
    info->num_bricks = ds->d.nb;
    info->brick_size = ds->d.b;
    info->levels = ds->d.L;
    info->ops_per_checkpoint = ds->d.S;
    info->stream_bytes = ds->d.stream_bytes;
    info->palette_entries = ds->d.palette_entries;
    memcpy(info->freq, ds->d.freq, sizeof info->freq);
    memcpy(info->cum, ds->d.cum, sizeof info->cum);
    return CSV_OK;
}

int csv_dataset_index_ms(const csv_dataset* ds, float* ms) {
    if (!ds || !ms) return CSV_EINVAL;
    *ms = ds->d.index_ms;
    return CSV_OK;
}

int csv_dataset_ids(const csv_dataset* ds, uint32_t* ids, uint32_t n) {
    if (!ds || !ids || n < ds->d.nb) return CSV_EINVAL;
    memcpy(ids, ds->d.h_ids, sizeof(uint32_t) * ds->d.nb);
    return CSV_OK;
}

void csv_close(csv_dataset* ds) {
    if (!ds) return;
    DeviceGuard g(ds->d.device);
    free_dataset(ds->d);
    delete ds;
}

int csv_decode_batch(csv_ctx* ctx, const csv_dataset* ds, const csv_request* d_reqs, uint32_t n, uint64_t* d_out,
                     uint32_t* d_status, void* stream) {
    if (!ctx || !ds) return CSV_EINVAL;
    if (n == 0) return CSV_OK;
    if (!d_reqs || !d_out || !d_status) return fail(ctx, CSV_EINVAL, "null request, output or status pointer");
    DeviceGuard g(ctx->device);
    int rc = ensure_scratch(ctx, ds->d.b);
    if (rc) return rc;
    cudaError_t e = launch_decode(ds->d, d_reqs, n, d_out, d_status, ctx->scr, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "decode launch");
    return CSV_OK;
}

int csv_decode_batch_static(csv_ctx* ctx, const csv_dataset* ds, const csv_request* d_reqs, uint32_t n,
                            uint64_t* d_out, uint32_t* d_status, void* stream) {
    if (!ctx || !ds) return CSV_EINVAL;
    if (n == 0) return CSV_OK;
    if (!d_reqs || !d_out || !d_status) return fail(ctx, CSV_EINVAL, "null request, output or status pointer");
    DeviceGuard g(ctx->device);
    std::string err;
    int rc = decode_batch_static(ctx->device, ds->d, d_reqs, n, d_out, d_status, (cudaStream_t)stream, err);
    return rc ? fail(ctx, rc, err) : CSV_OK;
}

// Labels per csv_decode_image chunk: two such device buffers per context.
constexpr uint64_t kImageChunkBytes = 256ull << 20;

int csv_decode_image(csv_ctx* ctx, const uint8_t* image, size_t len, uint32_t lod, uint64_t* out, uint32_t* status) {
    if (!ctx || !out) return CSV_EINVAL;
    DeviceGuard g(ctx->device);
    csv_dataset* ds = nullptr;
    int rc = csv_open(ctx, image, len, &ds);
    if (rc) return rc;
    if (lod >= ds->d.L) {
        csv_close(ds);
        return fail(ctx, CSV_EINVAL, "lod beyond log2(brick size)");
    }
    const uint32_t nb = ds->d.nb;
    const uint64_t per = 1ull << (3 * lod);
    // chunks of whole bricks, at most kImageChunkBytes of labels each (at least one brick):
    // chunk k decodes into buffer k % 2 while chunk k - 1 drains to the host
    const uint64_t brick_bytes = 8 * per;
    const uint32_t per_chunk = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(nb, kImageChunkBytes / brick_bytes));
    std::vector<csv_request> reqs(nb);
    for (uint32_t i = 0; i < nb; ++i) reqs[i] = csv_request{i, lod, per * (i % per_chunk)};
    csv_request* d_reqs = nullptr;
    uint32_t* d_st = nullptr;
    cudaError_t e = cudaSuccess;
    const size_t need = (size_t)per_chunk * brick_bytes;
    if (!ctx->pipe_stream[0]) {
        for (int i = 0; i < 2 && e == cudaSuccess; ++i) e = cudaStreamCreateWithFlags(&ctx->pipe_stream[i], cudaStreamNonBlocking);
        for (int i = 0; i < 4 && e == cudaSuccess; ++i) e = cudaEventCreateWithFlags(&ctx->pipe_event[i], cudaEventDisableTiming);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "pipeline streams");
    }
    if (rc == CSV_OK && need > ctx->chunk_bytes) {
        for (int i = 0; i < 2; ++i) {
            cudaFree(ctx->chunk_buf[i]);
            ctx->chunk_buf[i] = nullptr;
        }
        ctx->chunk_bytes = 0;
        for (int i = 0; i < 2 && e == cudaSuccess; ++i) e = cudaMalloc(&ctx->chunk_buf[i], need);
        if (e == cudaSuccess) ctx->chunk_bytes = need;
        else rc = fail(ctx, CSV_ENOMEM, std::string("chunk buffers: ") + cudaGetErrorString(e));
    }
    cudaStream_t s_dec = ctx->pipe_stream[0], s_copy = ctx->pipe_stream[1];
    if (rc == CSV_OK &&
        ((e = cudaMalloc(&d_reqs, sizeof(csv_request) * std::max<uint32_t>(1, nb))) != cudaSuccess ||
         (e = cudaMalloc(&d_st, 4 * std::max<uint32_t>(1, nb))) != cudaSuccess)) {
        rc = fail(ctx, CSV_ENOMEM, std::string("device allocation: ") + cudaGetErrorString(e));
    } else if (rc == CSV_OK &&
               (e = cudaMemcpyAsync(d_reqs, reqs.data(), sizeof(csv_request) * nb, cudaMemcpyHostToDevice, s_dec)) !=
                   cudaSuccess) {
        rc = cuda_fail(ctx, e, "request copy");
    }
    for (uint32_t k0 = 0, c = 0; rc == CSV_OK && k0 < nb; k0 += per_chunk, ++c) {
        const uint32_t cnt = std::min(per_chunk, nb - k0), b = c & 1u;
        if (c >= 2 && (e = cudaStreamWaitEvent(s_dec, ctx->pipe_event[2 + b], 0)) != cudaSuccess) {
            rc = cuda_fail(ctx, e, "pipeline wait");
            break;
        }
        rc = csv_decode_batch(ctx, ds, d_reqs + k0, cnt, ctx->chunk_buf[b], d_st + k0, s_dec);
        if (rc) break;
        if ((e = cudaEventRecord(ctx->pipe_event[b], s_dec)) != cudaSuccess ||
            (e = cudaStreamWaitEvent(s_copy, ctx->pipe_event[b], 0)) != cudaSuccess ||
            (e = cudaMemcpyAsync(out + (uint64_t)k0 * per, ctx->chunk_buf[b], cnt * brick_bytes, cudaMemcpyDeviceToHost,
                                 s_copy)) != cudaSuccess ||
            (e = cudaEventRecord(ctx->pipe_event[2 + b], s_copy)) != cudaSuccess)
            rc = cuda_fail(ctx, e, "pipeline copy");
    }
    if (rc == CSV_OK) {
        std::vector<uint32_t> hst(nb);
        if ((e = cudaEventRecord(ctx->pipe_event[0], s_dec)) != cudaSuccess ||
            (e = cudaStreamWaitEvent(s_copy, ctx->pipe_event[0], 0)) != cudaSuccess ||
            (e = cudaMemcpyAsync(hst.data(), d_st, 4 * nb, cudaMemcpyDeviceToHost, s_copy)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s_copy)) != cudaSuccess) {
            rc = cuda_fail(ctx, e, "decode");
        } else {
            if (status) memcpy(status, hst.data(), 4 * nb);
            for (uint32_t i = 0; i < nb && rc == CSV_OK; ++i)
                if (hst[i]) rc = fail(ctx, CSV_EBRICK, "brick " + std::to_string(i) + " status " +
                                                           std::to_string(hst[i]));
        }
    }
    // both streams idle before the request and status buffers go
    cudaStreamSynchronize(s_dec);
    cudaStreamSynchronize(s_copy);
    cudaFree(d_reqs);
    cudaFree(d_st);
    csv_close(ds);
    return rc;
}

int csv_encode_device(csv_ctx* ctx, const uint64_t* d_volume, uint32_t W, uint32_t H, uint32_t D, uint32_t brick_size,
                      void* stream, size_t* image_len) {
    if (!ctx || !image_len) return CSV_EINVAL;
    if (brick_size < 2 || brick_size > 64 || (brick_size & (brick_size - 1)))
        return fail(ctx, CSV_EINVAL, "brick size must be a power of two in [2, 64]");
    if ((uint64_t)W * H * D > 0 && !d_volume) return fail(ctx, CSV_EINVAL, "null volume");
    DeviceGuard g(ctx->device);
    if (!ctx->enc) ctx->enc = encoder_state_new();
    std::string err;
    int rc = encode_device(ctx->enc, ctx->device, d_volume, W, H, D, brick_size, (cudaStream_t)stream, err);
    if (rc) return fail(ctx, rc, err);
    const uint8_t* img = encoder_image(ctx->enc, image_len);
    return img ? CSV_OK : fail(ctx, CSV_EINVAL, "encode produced no image");
}

int csv_encode_shard_bricks(csv_ctx* ctx, const uint64_t* d_slab, uint32_t W, uint32_t H, uint32_t D,
                            uint32_t brick_size, uint32_t bx0, uint32_t index_base, uint64_t* hist, void* stream) {
    if (!ctx || !hist) return CSV_EINVAL;
    if (brick_size < 2 || brick_size > 64 || (brick_size & (brick_size - 1)))
        return fail(ctx, CSV_EINVAL, "brick size must be a power of two in [2, 64]");
    if ((uint64_t)W * H * D > 0 && !d_slab) return fail(ctx, CSV_EINVAL, "null volume");
    if ((uint64_t)bx0 + (W + brick_size - 1) / brick_size > 1024)
        return fail(ctx, CSV_ERANGE, "brick x beyond 1023 (10-bit Morton brick IDs, utils.cpp:10-14)");
    DeviceGuard g(ctx->device);
    if (!ctx->enc) ctx->enc = encoder_state_new();
    std::string err;
    EncodeShard sh;
    sh.bx0 = bx0;
    sh.index_base = index_base;
    int rc = encode_device(ctx->enc, ctx->device, d_slab, W, H, D, brick_size, (cudaStream_t)stream, err, nullptr, &sh,
                           hist);
    return rc ? fail(ctx, rc, err) : CSV_OK;
}

int csv_encode_shard_finish(csv_ctx* ctx, const uint64_t* hist, void* stream, size_t* image_len) {
    if (!ctx || !hist || !image_len) return CSV_EINVAL;
    DeviceGuard g(ctx->device);
    std::string err;
    int rc = finish_encode_shard(ctx->enc, hist, (cudaStream_t)stream, err);
    if (rc) return fail(ctx, rc, err);
    const uint8_t* img = encoder_image(ctx->enc, image_len);
    return img ? CSV_OK : fail(ctx, CSV_EINVAL, "encode produced no image");
}

int csv_encoded_image(csv_ctx* ctx, const uint8_t** d_image, size_t* len) {
    if (!ctx || !d_image || !len) return CSV_EINVAL;
    const uint8_t* p = encoder_image(ctx->enc, len);
    if (!p) return fail(ctx, CSV_EINVAL, "no encoded image on this context");
    *d_image = p;
    return CSV_OK;
}

int csv_encode(csv_ctx* ctx, const uint64_t* volume, uint32_t W, uint32_t H, uint32_t D, uint32_t brick_size,
               uint8_t** out, size_t* out_len) {
    if (!ctx || !out || !out_len) return CSV_EINVAL;
    *out = nullptr;
    *out_len = 0;
    uint64_t n = (uint64_t)W * H * D;
    if (n && !volume) return fail(ctx, CSV_EINVAL, "null volume");
    DeviceGuard g(ctx->device);
    uint64_t* d_vol = nullptr;
    cudaStream_t st = 0;
    cudaError_t e = cudaMalloc(&d_vol, 8 * std::max<uint64_t>(n, 1));
    if (e != cudaSuccess) return fail(ctx, CSV_ENOMEM, std::string("volume: ") + cudaGetErrorString(e));
    if (n && (e = cudaMemcpyAsync(d_vol, volume, 8 * n, cudaMemcpyHostToDevice, st)) != cudaSuccess) {
        cudaFree(d_vol);
        return cuda_fail(ctx, e, "volume copy");
    }
    size_t len = 0;
    int rc = csv_encode_device(ctx, d_vol, W, H, D, brick_size, st, &len);
    cudaFree(d_vol);
    if (rc) return rc;
    const uint8_t* d_img = encoder_image(ctx->enc, &len);
    uint8_t* h = (uint8_t*)malloc(std::max<size_t>(len, 1));
    if (!h) return fail(ctx, CSV_ENOMEM, "host allocation");
    if ((e = cudaMemcpy(h, d_img, len, cudaMemcpyDeviceToHost)) != cudaSuccess) {
        free(h);
        return cuda_fail(ctx, e, "image copy");
    }
    *out = h;
    *out_len = len;
    return CSV_OK;
}

int csv_open_encoded(csv_ctx* ctx, csv_dataset** out) {
    if (!ctx || !out) return CSV_EINVAL;
    *out = nullptr;
    DeviceGuard g(ctx->device);
    csv_dataset* ds = new (std::nothrow) csv_dataset();
    if (!ds) return fail(ctx, CSV_ENOMEM, "host allocation");
    ds->ctx = ctx;
    std::string err;
    int rc = encoder_to_dataset(ctx->enc, ds->d, err);
    if (rc) {
        free_dataset(ds->d);
        delete ds;
        return fail(ctx, rc, err);
    }
    *out = ds;
    return CSV_OK;
}

int csv_dataset_concat(csv_ctx* ctx, const csv_dataset* const* parts, uint32_t n, csv_dataset** out) {
    if (!ctx || !parts || !out || n == 0) return CSV_EINVAL;
    *out = nullptr;
    DeviceGuard g(ctx->device);
    uint64_t nb = 0, pal_n = 0, enc_n = 0, ck_n = 0;
    uint32_t n_models = 0;
    for (uint32_t k = 0; k < n; ++k) {
        if (!parts[k]) return fail(ctx, CSV_EINVAL, "null part");
        const DeviceDataset& p = parts[k]->d;
        if (p.S != kOpsPerCheckpoint) return fail(ctx, CSV_EINVAL, "parts with different seek-index spacing");
        nb += p.nb;
        pal_n += p.pal_pool_entries;
        enc_n += (p.enc_pool_bytes + 15) & ~15ull;
        ck_n += p.ck_entries;
        n_models += p.n_models;
    }
    if (nb > 0xFFFFFFFFull || ck_n > 0xFFFFFFFFull || n_models > 255)
        return fail(ctx, CSV_ERANGE, "concatenation too large");
    csv_dataset* ds = new (std::nothrow) csv_dataset();
    if (!ds) return fail(ctx, CSV_ENOMEM, "host allocation");
    ds->ctx = ctx;
    DeviceDataset& d = ds->d;
    d.device = ctx->device;
    d.nb = (uint32_t)nb;
    d.S = kOpsPerCheckpoint;
    d.total = kTot;
    d.n_models = n_models;
    d.h_ids = (uint32_t*)malloc(sizeof(uint32_t) * std::max<uint64_t>(1, nb));
    d.h_cost = (uint32_t*)malloc(sizeof(uint32_t) * std::max<uint64_t>(1, nb));
    d.enc_pool_bytes = std::max<uint64_t>(16, enc_n);
    d.pal_pool_entries = std::max<uint64_t>(1, pal_n);
    d.ck_entries = ck_n;
    std::vector<BrickDesc> all;
    all.reserve(nb);
    cudaError_t e;
    int rc = CSV_OK;
    if ((e = cudaMalloc(&d.d_bricks, sizeof(BrickDesc) * std::max<uint64_t>(1, nb))) != cudaSuccess ||
        (e = cudaMalloc(&d.d_pal, 8 * d.pal_pool_entries)) != cudaSuccess ||
        (e = cudaMalloc(&d.d_enc, d.enc_pool_bytes)) != cudaSuccess ||
        (e = cudaMalloc(&d.d_ck, sizeof(Checkpoint) * std::max<uint64_t>(1, ck_n))) != cudaSuccess ||
        (e = cudaMalloc(&d.d_lut, sizeof(uint32_t) * kTot * n_models)) != cudaSuccess) {
        rc = fail(ctx, CSV_ENOMEM, std::string("device allocation: ") + cudaGetErrorString(e));
    }
    uint64_t pal_base = 0, enc_base = 0, ck_base = 0;
    uint32_t model_base = 0, id_base = 0;
    for (uint32_t k = 0; k < n && rc == CSV_OK; ++k) {
        const DeviceDataset& p = parts[k]->d;
        std::vector<BrickDesc> pb(p.nb);
        if ((p.nb && (e = cudaMemcpy(pb.data(), p.d_bricks, sizeof(BrickDesc) * p.nb, cudaMemcpyDeviceToHost)) !=
                         cudaSuccess) ||
            (e = cudaMemcpy(d.d_pal + pal_base, p.d_pal, 8 * p.pal_pool_entries, cudaMemcpyDeviceToDevice)) !=
                cudaSuccess ||
            (e = cudaMemcpy(d.d_enc + enc_base, p.d_enc, p.enc_pool_bytes, cudaMemcpyDeviceToDevice)) != cudaSuccess ||
            (p.ck_entries && (e = cudaMemcpy(d.d_ck + ck_base, p.d_ck, sizeof(Checkpoint) * p.ck_entries,
                                             cudaMemcpyDeviceToDevice)) != cudaSuccess) ||
            (e = cudaMemcpy(d.d_lut + (size_t)kTot * model_base, p.d_lut, sizeof(uint32_t) * kTot * p.n_models,
                            cudaMemcpyDeviceToDevice)) != cudaSuccess) {
            rc = cuda_fail(ctx, e, "concat copy");
            break;
        }
        for (BrickDesc& b : pb) {
            const uint32_t model = ((b.flags >> BF_MODEL_SHIFT) & 255u) + model_base;
            b.pal_off += pal_base;
            b.enc_off += enc_base;
            b.ck_off += (uint32_t)ck_base;
            b.flags = (b.flags & ~(255u << BF_MODEL_SHIFT)) | (model << BF_MODEL_SHIFT);
            all.push_back(b);
        }
        memcpy(d.h_ids + id_base, p.h_ids, sizeof(uint32_t) * p.nb);
        memcpy(d.h_cost + id_base, p.h_cost, sizeof(uint32_t) * p.nb);
        if (k > 0 && p.b != d.b) d.mixed_b = 1;
        d.b = std::max(d.b, p.b);
        d.L = std::max(d.L, p.L);
        d.max_P = std::max(d.max_P, p.max_P);
        d.max_nsym = std::max(d.max_nsym, p.max_nsym);
        d.stream_bytes += p.stream_bytes;
        d.palette_entries += p.palette_entries;
        if (k == 0) {
            memcpy(d.freq, p.freq, sizeof d.freq);
            memcpy(d.cum, p.cum, sizeof d.cum);
        }
        pal_base += p.pal_pool_entries;
        enc_base += (p.enc_pool_bytes + 15) & ~15ull;
        ck_base += p.ck_entries;
        if (model_base < 32) d.fast_models |= p.fast_models << model_base;
        model_base += p.n_models;
        id_base += p.nb;
    }
    if (rc == CSV_OK && nb &&
        (e = cudaMemcpy(d.d_bricks, all.data(), sizeof(BrickDesc) * nb, cudaMemcpyHostToDevice)) != cudaSuccess)
        rc = cuda_fail(ctx, e, "concat copy");
    if (rc) {
        free_dataset(d);
        delete ds;
        return rc;
    }
    *out = ds;
    return CSV_OK;
}

}  // extern "C"

struct csv_graph {
    csv_ctx* ctx = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t* d_order = nullptr;
    uint32_t kernels = 0;  // decode kernels one replay launches
};

namespace {

// The graph's schedule.  Requests above LOD 5 (64^3 outputs) go to the decode
// kernel's large variant, the rest to its small-footprint variant with three
// times the CTAs per SM; each part keeps the request order, or with `lpt` runs
// largest first (estimated work = nSymbols of the brick, rANS + replay, plus a
// quarter of the labels written).  ord = [large part | small part].
// The requests in launch order: outputs above 32^3 whose brick has fewer than 255 palette entries (when
// narrow8: the 8-bit variant's part, n8 of them), the other outputs above 32^3 (n_large in all, with the
// first part), then the rest (small8: every one of them with fewer than 255 palette entries, when
// narrow8); each part longest first when lpt.
int graph_schedule(csv_ctx* ctx, const csv_dataset* ds, const csv_request* d_reqs, uint32_t n, bool lpt,
                   bool narrow8, std::vector<uint32_t>& ord, uint32_t& n8, uint32_t& n_large, bool& small8) {
    std::vector<csv_request> h(n);
    cudaError_t e = cudaMemcpy(h.data(), d_reqs, sizeof(csv_request) * n, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "request copy");
    std::vector<uint8_t> small_pal(ds->d.nb, 0);
    if (narrow8 && ds->d.nb) {
        std::vector<BrickDesc> desc(ds->d.nb);
        e = cudaMemcpy(desc.data(), ds->d.d_bricks, sizeof(BrickDesc) * ds->d.nb, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "brick table copy");
        for (uint32_t i = 0; i < ds->d.nb; ++i) small_pal[i] = desc[i].P < 0xFFu;
    }
    std::vector<uint64_t> cost(n);
    for (uint32_t i = 0; i < n; ++i) {
        uint64_t c = 0;
        if (h[i].brick < ds->d.nb && h[i].lod < 8) c = ds->d.h_cost[h[i].brick] + ((1ull << (3 * h[i].lod)) >> 2);
        cost[i] = c;
    }
    ord.clear();
    auto narrow_req = [&](uint32_t i) { return h[i].brick < ds->d.nb && small_pal[h[i].brick]; };
    for (uint32_t i = 0; i < n; ++i)
        if (h[i].lod > kSmallLod && narrow_req(i)) ord.push_back(i);
    n8 = (uint32_t)ord.size();
    for (uint32_t i = 0; i < n; ++i)
        if (h[i].lod > kSmallLod && !narrow_req(i)) ord.push_back(i);
    n_large = (uint32_t)ord.size();
    small8 = narrow8;
    for (uint32_t i = 0; i < n; ++i)
        if (h[i].lod <= kSmallLod) {
            ord.push_back(i);
            small8 = small8 && narrow_req(i);
        }
    if (lpt) {
        auto by_cost = [&](uint32_t a, uint32_t b) { return cost[a] > cost[b]; };
        std::stable_sort(ord.begin(), ord.begin() + n8, by_cost);
        std::stable_sort(ord.begin() + n8, ord.begin() + n_large, by_cost);
        std::stable_sort(ord.begin() + n_large, ord.end(), by_cost);
    }
    return CSV_OK;
}

}  // namespace

extern "C" {

int csv_decode_graph_create(csv_ctx* ctx, const csv_dataset* ds, const csv_request* d_reqs, uint32_t n,
                            uint64_t* d_out, uint32_t* d_status, const csv_decode_config* cfg, csv_graph** out) {
    if (!ctx || !ds || !out) return CSV_EINVAL;
    *out = nullptr;
    if (n && (!d_reqs || !d_out || !d_status)) return fail(ctx, CSV_EINVAL, "null request, output or status pointer");
    DeviceGuard g(ctx->device);
    int rc = ensure_scratch(ctx, ds->d.b);
    if (rc) return rc;
    decode_grid(ctx->device, 1);  // occupancy queries happen outside the capture
    const uint32_t layout = cfg ? cfg->layout : 0;
    if (layout > 2) return fail(ctx, CSV_EINVAL, "layout is 0, 1 or 2");
    const bool split = ds->d.L > kSmallLod + 1 && n && layout != 1;
    if (split && (rc = abi_ensure_scratch_small(ctx))) return rc;
    csv_graph* gr = new (std::nothrow) csv_graph();
    if (!gr) return fail(ctx, CSV_ENOMEM, "host allocation");
    gr->ctx = ctx;
    DecodeConfig dc;
    if (cfg) {
        dc.ctas_per_sm = cfg->ctas_per_sm;
        dc.stage = cfg->stage;
        dc.layout = cfg->layout;
    }
    // a dataset with 64^3 bricks: split the requests by output size and, for the outputs above 32^3, by
    // palette size (up to three launches), else one launch
    uint32_t n_large = n, n8 = 0;
    bool small8 = false;
    if (split || (cfg && cfg->lpt && n)) {
        std::vector<uint32_t> ord;
        rc = graph_schedule(ctx, ds, d_reqs, n, cfg && cfg->lpt, split && layout == 0, ord, n8, n_large, small8);
        if (!rc && !split) n_large = n, n8 = 0, small8 = false;  // one part: all of them, in the scheduled order
        // the wide 64^3 part beside the 8-bit one needs scratch of its own
        if (!rc && n8 && n_large > n8) rc = abi_ensure_scratch_wide(ctx, ds->d.b);
        cudaError_t e = rc ? cudaSuccess : cudaMalloc(&gr->d_order, sizeof(uint32_t) * n);
        if (!rc && e != cudaSuccess) rc = fail(ctx, CSV_ENOMEM, "order allocation");
        if (!rc && (e = cudaMemcpy(gr->d_order, ord.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice)) != cudaSuccess)
            rc = cuda_fail(ctx, e, "order copy");
        if (rc) {
            csv_graph_destroy(gr);
            return rc;
        }
        dc.order = gr->d_order;
    }
    cudaStream_t s;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        csv_graph_destroy(gr);
        return cuda_fail(ctx, e, "capture stream");
    }
    e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        cudaError_t le = cudaSuccess;
        if (!split) {
            le = launch_decode(ds->d, d_reqs, n, d_out, d_status, ctx->scr, s, &dc);
            gr->kernels = n ? 1u : 0u;
        } else {
            // the large outputs first (longest bricks; those with palettes below 255 entries in
            // the 8-bit variant, three CTAs per SM, then the others), then the small ones at three
            // times the occupancy.  Each launch after the first is a programmatic dependent of the
            // one before, with its own scratch and queue (all reset before the first launch): its
            // CTAs fill the SMs that the earlier launches' CTAs leave once their queues run dry.
            struct Part {
                uint32_t first, count;
                bool narrow8, small;
            };
            const Part parts[3] = {{0, n8, true, false}, {n8, n_large - n8, false, false},
                                   {n_large, n - n_large, small8, true}};
            const csv::DecodeScratch* scrs[3] = {&ctx->scr, n8 ? &ctx->scr_wide : &ctx->scr, &ctx->scr_small};
            uint32_t n_parts = 0;
            for (const Part& p : parts) n_parts += p.count > 0;
            // each launch's queue: the first one's is reset by launch_decode, the others here
            bool first = true;
            for (int k = 0; k < 3 && le == cudaSuccess; ++k)
                if (parts[k].count && !first) le = cudaMemsetAsync(scrs[k]->d_queue, 0, sizeof(uint32_t), s);
                else if (parts[k].count) first = false;
            first = true;
            for (int k = 0; k < 3 && le == cudaSuccess; ++k) {
                if (!parts[k].count) continue;
                DecodeConfig part = dc;
                part.order = gr->d_order + parts[k].first;
                part.n_order = parts[k].count;
                part.narrow8 = parts[k].narrow8;
                part.small_only = parts[k].small;
                part.pdl = !first;
                // a part alone uses the context's main scratch
                le = launch_decode(ds->d, d_reqs, n, d_out, d_status, n_parts == 1 ? ctx->scr : *scrs[k], s, &part);
                ++gr->kernels;
                first = false;
            }
        }
        e = cudaStreamEndCapture(s, &gr->graph);
        if (le != cudaSuccess) e = le;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&gr->exec, gr->graph, 0);
    cudaStreamDestroy(s);
    if (e != cudaSuccess) {
        csv_graph_destroy(gr);
        return cuda_fail(ctx, e, "graph capture");
    }
    *out = gr;
    return CSV_OK;
}

int csv_graph_launch(csv_graph* gr, void* stream) {
    if (!gr || !gr->exec) return CSV_EINVAL;
    DeviceGuard g(gr->ctx->device);
    cudaError_t e = cudaGraphLaunch(gr->exec, (cudaStream_t)stream);
    return e == cudaSuccess ? CSV_OK : cuda_fail(gr->ctx, e, "graph launch");
}

int csv_graph_kernels(const csv_graph* gr, uint32_t* n) {
    if (!gr || !n) return CSV_EINVAL;
    *n = gr->kernels;
    return CSV_OK;
}

void csv_graph_destroy(csv_graph* gr) {
    if (!gr) return;
    DeviceGuard g(gr->ctx->device);
    if (gr->exec) cudaGraphExecDestroy(gr->exec);
    if (gr->graph) cudaGraphDestroy(gr->graph);
    cudaFree(gr->d_order);
    delete gr;
}

int csv_decode_autotune(csv_ctx* ctx, const csv_dataset* ds, const csv_request* d_reqs, uint32_t n, uint64_t* d_out,
                        uint32_t* d_status, uint32_t reps, csv_decode_config* best, float* best_ms) {
    if (!ctx || !ds || !best) return CSV_EINVAL;
    DeviceGuard g(ctx->device);
    if (reps == 0) reps = 5;
    cudaStream_t s;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "tune stream");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best_t = 1e30f;
    csv_decode_config bestc{0, 1, 0, 0};
    int rc = CSV_OK;
    const uint32_t per_sm_options[] = {0, 2, 1};  // 0: as many CTAs as fit
    const uint32_t n_layouts = ds->d.L > kSmallLod + 1 ? 3 : 1;  // layout matters with 64^3 bricks only
    for (uint32_t layout = 0; layout < n_layouts && rc == CSV_OK; ++layout)
    for (uint32_t ps : per_sm_options) {
        for (uint32_t stage = 0; stage <= 1 && rc == CSV_OK; ++stage) {
            for (uint32_t lpt = 0; lpt <= 1 && rc == CSV_OK; ++lpt) {
                csv_decode_config c{ps, stage, lpt, layout};
                csv_graph* gr = nullptr;
                rc = csv_decode_graph_create(ctx, ds, d_reqs, n, d_out, d_status, &c, &gr);
                if (rc) break;
                std::vector<float> ts;
                csv_graph_launch(gr, s);  // warm-up
                for (uint32_t r = 0; r < reps; ++r) {
                    cudaEventRecord(e0, s);
                    csv_graph_launch(gr, s);
                    cudaEventRecord(e1, s);
                    cudaEventSynchronize(e1);
                    float ms = 0;
                    cudaEventElapsedTime(&ms, e0, e1);
                    ts.push_back(ms);
                }
                csv_graph_destroy(gr);
                std::sort(ts.begin(), ts.end());
                const float med = ts[ts.size() / 2];
                if (med < best_t) {
                    best_t = med;
                    bestc = c;
                }
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    e = cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(ctx, e, "tune");
    *best = bestc;
    if (best_ms) *best_ms = best_t;
    return CSV_OK;
}

int csv_render(csv_ctx* ctx, const csv_camera* camera, uint32_t width, uint32_t height, float grid_size,
               uint32_t brick_size, uint32_t bricks_per_axis, const csv_brick_slot* d_slots, uint64_t n_slots,
               const uint64_t* d_labels, const uint64_t* d_hidden, uint32_t n_hidden, uint64_t* d_label_out,
               float* d_depth_out, uint32_t* d_requests, void* stream) {
    if (!ctx || !camera) return CSV_EINVAL;
    if (width == 0 || height == 0) return CSV_OK;
    if (!d_label_out || !d_depth_out || (n_slots && (!d_slots || !d_labels)))
        return fail(ctx, CSV_EINVAL, "null render buffer");
    if (brick_size < 1 || brick_size > 1024 || (brick_size & (brick_size - 1)))
        return fail(ctx, CSV_EINVAL, "brick size must be a power of two");
    if (bricks_per_axis > 1024) return fail(ctx, CSV_ERANGE, "more than 1024 bricks per axis");
    DeviceGuard g(ctx->device);
    cudaError_t e = launch_render(*camera, width, height, grid_size, brick_size, bricks_per_axis, d_slots, n_slots,
                                  d_labels, d_hidden, n_hidden, d_label_out, d_depth_out, d_requests,
                                  (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "render launch");
    return CSV_OK;
}

int csv_lighting_default(double light_angle_deg, csv_lighting* out) {
    if (!out) return CSV_EINVAL;
    // webgpuSetup.js:24-31 (defaults) and :205-219 (the uniform): the light on a
    // west-east arc at a fixed elevation, ambient 0.5, diffuse 0.8
    const double a = light_angle_deg * 3.14159265358979323846 / 180.0;
    memset(out, 0, sizeof *out);
    out->light_dir[0] = (float)sin(a);
    out->light_dir[1] = 0.6f;
    out->light_dir[2] = (float)-cos(a);
    out->ambient = 0.5f;
    out->diffuse = 0.8f;
    return CSV_OK;
}

int csv_transfer_function(const csv_dataset* ds, const uint64_t* hidden, uint32_t n_hidden, uint64_t* keys,
                          uint32_t* rgba, uint32_t cap, uint32_t* n_out) {
    if (!ds || !n_out || (n_hidden && !hidden)) return CSV_EINVAL;
    DeviceGuard g(ds->ctx->device);
    std::vector<uint64_t> k;
    std::vector<uint32_t> c;
    cudaError_t e = transfer_function(ds->d, hidden, n_hidden, k, c);
    if (e != cudaSuccess) return cuda_fail(ds->ctx, e, "palette copy");
    *n_out = (uint32_t)k.size();
    if (k.size() > cap || (!k.empty() && (!keys || !rgba)))
        return fail(ds->ctx, CSV_ERANGE, "transfer function: " + std::to_string(k.size()) + " labels, room for " +
                                             std::to_string(cap));
    if (!k.empty()) {
        memcpy(keys, k.data(), 8 * k.size());
        memcpy(rgba, c.data(), 4 * c.size());
    }
    return CSV_OK;
}

int csv_render_rgba(csv_ctx* ctx, const csv_camera* camera, uint32_t width, uint32_t height, float grid_size,
                    uint32_t brick_size, uint32_t bricks_per_axis, const csv_brick_slot* d_slots, uint64_t n_slots,
                    const uint64_t* d_labels, const uint64_t* d_tf_keys, const uint32_t* d_tf_rgba, uint32_t n_tf,
                    const csv_lighting* lighting, uint32_t* d_rgba_out, uint32_t* d_requests, void* stream) {
    if (!ctx || !camera || !lighting) return CSV_EINVAL;
    if (width == 0 || height == 0) return CSV_OK;
    if (!d_rgba_out || (n_slots && (!d_slots || !d_labels)) || (n_tf && (!d_tf_keys || !d_tf_rgba)))
        return fail(ctx, CSV_EINVAL, "null render buffer");
    if (brick_size < 1 || brick_size > 1024 || (brick_size & (brick_size - 1)))
        return fail(ctx, CSV_EINVAL, "brick size must be a power of two");
    if (bricks_per_axis > 1024) return fail(ctx, CSV_ERANGE, "more than 1024 bricks per axis");
    DeviceGuard g(ctx->device);
    cudaError_t e = launch_render_rgba(*camera, width, height, grid_size, brick_size, bricks_per_axis, d_slots, n_slots,
                                       d_labels, d_tf_keys, d_tf_rgba, n_tf, lighting->light_dir, lighting->ambient,
                                       lighting->diffuse, d_rgba_out, d_requests, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "render launch");
    return CSV_OK;
}

int csv_synth_volume(csv_ctx* ctx, uint64_t* d_volume, uint32_t W, uint32_t H, uint32_t D, int kind, uint32_t n_cells,
                     uint32_t n_tubes, float r_min, float r_max, float zero_frac, uint64_t seed, void* stream) {
    if (!ctx || !d_volume || kind < 0 || kind > 2) return CSV_EINVAL;
    DeviceGuard g(ctx->device);
    cudaError_t e = synth_volume(d_volume, W, H, D, kind, n_cells, n_tubes, r_min, r_max, zero_frac, seed,
                                 (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "synth");
    return CSV_OK;
}

}  // extern "C"
