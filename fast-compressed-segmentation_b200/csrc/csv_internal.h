// csv_internal.h -- shared device/host definitions of the B200 CSV codec.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/csv.h"

namespace csv {

// Codec constants (types.hpp:18-28).
constexpr uint32_t kRansL = 1u << 23;     // RANS_LIMIT / RANS_INIT
constexpr uint32_t kTotBits = 12;         // LOG_TOTAL_FREQ
constexpr uint32_t kTot = 1u << kTotBits; // RANS_TOTAL
constexpr uint32_t kMagic = 0x43534244u;  // fileIO.cpp:25
constexpr uint32_t kHeaderBytes = 152;    // 16 B header + 136 B model (fileIO.cpp:25-49)
// Seek-index spacing: one decoder checkpoint (16 bytes) every this many ops.
// Each checkpoint starts one independent rANS segment in the decoder, so the
// spacing trades the serial segment length (latency) against index size.
constexpr uint32_t kOpsPerCheckpoint = 16;

// Op codes (types.hpp:162-171) and nibble layout (op << 1 | stop, brickEncoding.cpp:66-67).
enum : uint32_t { OP_RP = 0, OP_RX = 1, OP_RY = 2, OP_RZ = 3, OP_PA = 4, OP_P0 = 5, OP_PD = 6 };

// Brick descriptor flags.
constexpr uint32_t BF_UNIFORM = 1u;   // root stop bit set: the whole brick is palette[0]
constexpr uint32_t BF_TRUNCATED = 2u; // the stream ends inside the level structure
constexpr uint32_t BF_NOINDEX = 4u;   // no seek index (not built)
constexpr uint32_t BF_STATUS_MASK = 0xFFu;
constexpr uint32_t BF_LEVELS_SHIFT = 8;   // bits 8..11: levels of this brick, log2(b) + 1
constexpr uint32_t BF_MODEL_SHIFT = 16;   // bits 16..23: rANS model (LUT) of this brick

// Per-brick device descriptor, file order.
struct BrickDesc {
    uint64_t pal_off;        // first palette entry in the palette pool
    uint64_t enc_off;        // first byte of the rANS stream in the stream pool (16-byte aligned)
    uint32_t P, E, nsym, id; // palette size, stream bytes, nibble count, Morton brick ID
    uint32_t ck_off, ck_cap; // seek checkpoints: first entry and capacity
    uint32_t n_ops, flags;   // ops after the root nibble; BF_* flags
    uint32_t level_start[8]; // level_start[l] = first op whose node is on level l+1
};
static_assert(sizeof(BrickDesc) == 80, "BrickDesc layout");

// One seek checkpoint: decoder state before an op (see csv_oracle.c:or_seek_index).
struct Checkpoint {
    uint32_t state, pos, sym, ip;
};

// Decoded-op record (4 bytes): code | stop << 3 | palette index << 8.
constexpr uint32_t REC_PIDX_SHIFT = 8;
constexpr uint32_t PIDX_LABEL0 = 0xFFFFFFu; // "label 0" (op code 7, decode.wgsl:487-489)
constexpr uint32_t kMaxPalette = 0xFFFFFEu;

// Node info word: inactive -> palette index; active -> ACT | rank among active nodes of its level.
constexpr uint32_t NI_ACT = 0x80000000u;

inline uint32_t levels_of(uint32_t b) {
    uint32_t L = 0;
    while ((1u << L) < b) ++L;
    return L + 1;
}
// Ops after the root nibble in the fullest brick: sum_{l=1}^{L-1} 8^l.
inline uint64_t max_ops_of(uint32_t b) {
    uint32_t L = levels_of(b);
    return ((1ull << (3 * L)) - 8) / 7;
}

// Device-resident dataset.
struct DeviceDataset {
    int device = 0;
    uint32_t nb = 0, b = 0, L = 0, S = 0;
    uint32_t freq[16] = {}, cum[16] = {}, total = 0;
    uint64_t stream_bytes = 0, palette_entries = 0, ck_entries = 0;
    uint32_t max_nsym = 0, max_P = 0;
    uint32_t n_models = 1;  // LUTs at d_lut (a version-2 image's tables; a concatenation keeps each part's)
    uint32_t fast_models = 0;  // bit m: model m's table is well formed (the seek index's fast step)
    float index_ms = 0;        // device time of the seek-index passes csv_open ran (0: none ran)
    // pool for the stream-ordered temporaries of staging and the seek index (the opening context's;
    // null: the device's default pool)
    cudaMemPool_t pool = nullptr;
    uint32_t mixed_b = 0;   // a concatenation of different brick sizes
    uint64_t enc_pool_bytes = 0, pal_pool_entries = 0;  // sizes of d_enc and d_pal
    uint32_t* h_cost = nullptr;  // per brick: decode work estimate (nSymbols), for scheduling
    BrickDesc* d_bricks = nullptr;
    uint64_t* d_pal = nullptr;
    uint8_t* d_enc = nullptr;
    Checkpoint* d_ck = nullptr;
    uint32_t* d_lut = nullptr; // 4096 packed entries: sym | freq << 4 | start << 17
    uint32_t* h_ids = nullptr;
};

// A stream-ordered temporary from `pool`, or from the device's default pool when it is null.
inline cudaError_t tmp_alloc(void** p, size_t bytes, cudaMemPool_t pool, cudaStream_t st) {
    return pool ? cudaMallocFromPoolAsync(p, bytes, pool, st) : cudaMallocAsync(p, bytes, st);
}

// Launch helpers implemented in decode.cu.
cudaError_t build_lut(const uint32_t* freq, const uint32_t* cum, uint32_t* h_lut);
// Bit t set when table t (of n, the first 32) is well formed: every x in
// [0, 4096) lies in its symbol's range [start, start + freq).
uint32_t lut_fast_mask(const uint32_t* h_lut, uint32_t n);
// A seek-index sidecar keeps the rANS state before every kSeedSymbols-th symbol.
constexpr uint32_t kSeedSymbols = 512;
// Pass 1 as pieces from given states: piece_base[i] .. piece_base[i + 1] are
// brick i's pieces (piece_base has nb + 1 entries), seed[p] the state {x, pos}
// before piece p's first symbol, or {0, 0xFFFFFFFF}: brick i's only piece,
// run from its header.
struct IndexSeeds {
    std::vector<uint32_t> piece_base;
    std::vector<uint2> seed;
};
// The seek index (checkpoints, op counts, level starts, flags) of every brick,
// from the stream headers (seeds null) or from a sidecar's states; with seeds,
// *rejected is set, and nothing is written past the chain pass, when a piece
// did not end in the state given for the next (the dataset then needs a
// rebuild from its headers).
cudaError_t launch_build_index(DeviceDataset& ds, cudaStream_t st, const IndexSeeds* seeds = nullptr,
                               bool* rejected = nullptr);
// The states a sidecar keeps for ds (bricks whose chain the index walks; 0 for
// the others), computed again from the stream headers.
cudaError_t index_seeds_of(const DeviceDataset& ds, cudaStream_t st, std::vector<uint32_t>& n_seeds,
                           std::vector<uint2>& seeds);

struct DecodeScratch {
    uint8_t* base = nullptr;
    size_t per_cta = 0;   // per-CTA scratch of the largest brick size it was sized for
    uint32_t ctas = 0;
    size_t bytes = 0;     // total; a launch runs at most bytes / (its per-CTA scratch) CTAs
    uint32_t* d_queue = nullptr;
};
size_t decode_scratch_per_cta(uint32_t b, uint32_t kl = 6);
size_t decode_scratch_bytes(int device, uint32_t b);
// Scratch for the small variant's CTAs at 32^3 outputs (the second part of a split schedule).
size_t decode_scratch_small_bytes(int device);
// Scratch for the 64^3 variant with 16- or 32-bit node values at its occupancy (the part of a split
// schedule with the 64^3 bricks of 255 or more palette entries).
size_t decode_scratch_wide_bytes(int device, uint32_t b);
uint32_t decode_grid(int device, uint32_t n);
// Requests at this LOD (32^3 labels) or coarser can run in the decode kernel's
// small-footprint variant (six CTAs per SM instead of two).
constexpr uint32_t kSmallLod = 5;
// Launch knobs the autotuner chooses (defaults: occupancy-limited grid, staging on, request order).
struct DecodeConfig {
    uint32_t ctas_per_sm = 0;         // 0: as many as fit
    uint32_t stage = 1;               // stage brick streams in shared memory
    const uint32_t* order = nullptr;  // device list of request indices to decode, in this order, or null
    uint32_t n_order = 0;             // entries of order (0: n)
    const uint32_t* n_dev = nullptr;  // device-resident queue length (<= n or n_order), or null
    bool small_only = false;          // every queued request is at LOD 5 (32^3) or coarser
    uint32_t layout = 0;              // 1: every request in the small (six-CTA-per-SM) kernel; 2: no 8-bit values
    bool narrow8 = false;             // every queued request's brick has fewer than 255 palette entries
    // launched as a programmatic dependent of the previous kernel in the stream: its CTAs
    // start on the SMs that kernel's CTAs leave; the caller has reset scr.d_queue
    bool pdl = false;
};
cudaError_t launch_decode(const DeviceDataset& ds, const csv_request* d_reqs, uint32_t n, uint64_t* d_out,
                          uint32_t* d_status, const DecodeScratch& scr, cudaStream_t st,
                          const DecodeConfig* cfg = nullptr);

// Encoder state owned by a context (encode.cu).
struct EncoderState;
EncoderState* encoder_state_new();
void encoder_state_free(EncoderState* s);
// Per-brick mode / shared-table choice for an encode (version-2 image).
struct EncodeSelection {
    uint32_t n_tables = 0;           // 0: version 1, one model from the sampled bricks' histogram
    uint32_t freq[16][16] = {};      // each table's frequencies (each >= 1, sum 4096)
    const uint8_t* d_sel = nullptr;  // per brick, device: mode | table << 4 (null: mode 0, table 0)
};
// One x-slab of a larger volume, encoded by one rank: brick x-offset (IDs) and
// the file index of its first brick (the model's every-512th sample rule).
struct EncodeShard {
    uint32_t bx0 = 0;
    uint32_t index_base = 0;
};
// With hist_out, stops after the brick pass and returns the 16-bin histogram of
// the sampled bricks; finish_encode_shard then builds the image from the
// histogram summed over every shard (version 1 only).
int encode_device(EncoderState* s, int device, const uint64_t* d_vol, uint64_t W, uint64_t H, uint64_t D, uint32_t b,
                  cudaStream_t st, std::string& err, const EncodeSelection* sel = nullptr,
                  const EncodeShard* shard = nullptr, uint64_t* hist_out = nullptr);
int finish_encode_shard(EncoderState* s, const uint64_t hist[16], cudaStream_t st, std::string& err);
int encode_stats(EncoderState* s, int device, const uint64_t* d_vol, uint64_t W, uint64_t H, uint64_t D, uint32_t b,
                 uint32_t* d_hist, cudaStream_t st, std::string& err);
int encoder_to_dataset(EncoderState* s, DeviceDataset& d, std::string& err);
const uint8_t* encoder_image(EncoderState* s, size_t* len);

int decode_batch_static(int device, const DeviceDataset& ds, const csv_request* d_reqs, uint32_t n, uint64_t* d_out,
                        uint32_t* d_status, cudaStream_t st, std::string& err);

cudaError_t launch_render(const csv_camera& cam, uint32_t W, uint32_t H, float grid, uint32_t bs, uint32_t bpa,
                          const csv_brick_slot* slots, uint64_t n_slots, const uint64_t* labels, const uint64_t* hidden,
                          uint32_t n_hidden, uint64_t* out_label, float* out_depth, uint32_t* requests,
                          cudaStream_t st);
cudaError_t launch_render_rgba(const csv_camera& cam, uint32_t W, uint32_t H, float grid, uint32_t bs, uint32_t bpa,
                               const csv_brick_slot* slots, uint64_t n_slots, const uint64_t* labels,
                               const uint64_t* tf_keys, const uint32_t* tf_rgba, uint32_t n_tf, const float* light,
                               float ambient, float diffuse, uint32_t* out_rgba, uint32_t* requests, cudaStream_t st);

size_t gemm_smem_bytes();
// B [N][K] bf16 -> the tensor cores' no-swizzle K-major core-matrix tiling (K-chunks of 64).
cudaError_t launch_tile_b(const __nv_bfloat16* B, uint32_t N, uint32_t K, __nv_bfloat16* T, cudaStream_t st);
// The selector network's forward pass fused in one persistent kernel (mlp.cu): features [count][32]
// -> logits [count][32] and/or sel (argmax of logits 0..11 | argmax of logits 12..27 << 4).
cudaError_t launch_mlp_infer(const float* feat, uint32_t count, const __nv_bfloat16* W1t, const __nv_bfloat16* W2t,
                             const __nv_bfloat16* W3t, const float* b1, const float* b2, const float* b3, float* logits,
                             uint8_t* sel, uint32_t* err, int device, cudaStream_t st);
cudaError_t launch_gemm_bf16(const __nv_bfloat16* A, const __nv_bfloat16* B, uint32_t M, uint32_t N, uint32_t K,
                             const float* bias, const __nv_bfloat16* mask, uint32_t relu, float* C,
                             __nv_bfloat16* Cb, __nv_bfloat16* CbT, float* CT, uint32_t* err, cudaStream_t st);

cudaError_t synth_volume(uint64_t* d_vol, uint32_t W, uint32_t H, uint32_t D, int kind, uint32_t n_cells,
                         uint32_t n_tubes, float r_min, float r_max, float zero_frac, uint64_t seed,
                         cudaStream_t st);

}  // namespace csv
