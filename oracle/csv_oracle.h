/* csv_oracle.h -- CPU restatement of the reference codec, TEST INFRASTRUCTURE ONLY.
 *
 * This is the oracle: a plain-C restatement of the reference algorithm for the
 * compressed-segmentation brick codec (encoder/CSVEncoder/src, web/shaders/
 * decode.wgsl, web/shaders/rayTrace.wgsl, web/scripts/camera.js).  It is
 * pinned against the reference sources compiled as oracle/_ref/libcsvref.so
 * and against the reference's shipped compressed_dataset.csbd (decode-only
 * golden).  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it, and only as the checker; the product never links it.
 */
#ifndef CSV_ORACLE_H
#define CSV_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

uint32_t or_morton3(uint32_t x, uint32_t y, uint32_t z);
void or_demorton3(uint32_t m, uint32_t* x, uint32_t* y, uint32_t* z);
uint64_t or_majority8(const uint64_t* labels);
void or_build_model(const uint64_t* raw16, uint32_t* freq16, uint32_t* cum17);

/* Whole-volume encode to a .csbd v1 image (malloc'd; free with or_free). */
int or_encode(const uint64_t* vol, size_t W, size_t H, size_t D, uint32_t b,
              uint8_t** out, size_t* out_len);
/* Coarse-first pyramid of brick `brick_index` (split order): level l holds 8^l
 * nodes in Morton order at offset (8^l - 1)/7. */
int or_pyramid(const uint64_t* vol, size_t W, size_t H, size_t D, uint32_t b, uint32_t brick_index,
               uint64_t* labels, uint8_t* constant);

/* rANS stage of one brick: repacked nibble bytes, ceil(nsym/2) of them. */
int or_rans_decode(const uint32_t* freq16, const uint32_t* cum16, uint32_t total_freq,
                   const uint8_t* enc, uint32_t enc_len, uint32_t nsym, uint8_t* nib_out);
/* Label-space decode of one brick at target LOD t (2^t voxels per axis). */
int or_decode_brick(const uint64_t* palette, uint32_t P, const uint8_t* nib, uint32_t nib_bytes,
                    uint32_t b, uint32_t t, uint64_t* out);
/* Whole image: every brick at LOD t, brick i (file order) at out + i*8^t. */
int or_decode_image(const uint8_t* img, size_t len, uint32_t t, uint64_t* out, uint32_t* status);

/* Seek index of one brick (the project's sidecar format; see csv.h). */
/* The rANS state {x, pos} before every `every`-th symbol of a brick's chain. */
int or_rans_states(const uint32_t* freq16, const uint32_t* cum16, const uint8_t* enc, uint32_t enc_len, uint32_t nsym,
                   uint32_t every, uint32_t* states);
int or_seek_index(const uint32_t* freq16, const uint32_t* cum16, const uint8_t* enc, uint32_t enc_len,
                  uint32_t nsym, uint32_t P, uint32_t b, uint32_t ops_per_ckpt,
                  uint32_t* n_ops, uint32_t* level_start /* [8] */, uint32_t* ckpt /* 4 per */,
                  uint32_t max_ckpt, uint32_t* n_ckpt);

/* Per-brick LOD (camera.js:103-137) in double precision, as JS computes it;
 * focal = (screen_px / 2) / tan(fov / 2) computed once by the caller. */
uint32_t or_brick_lod(const double* center3, double brick_size, const double* cam3, double focal, uint32_t max_lod);

/* Brick slot of the decoded cache, indexed by the brick's Morton code. */
typedef struct {
    uint64_t offset;  /* first label of the brick's 8^lod decoded labels */
    uint32_t lod;     /* targetLOD */
    uint32_t flags;   /* bit 0: empty (all palette entries 0), bit 1: not resident */
} or_slot;

/* Scalar DDA (rayTrace.wgsl:565-906) in label/depth space.  cam: position[3],
 * tanHalfFov, forward[3], pad, right[3], pad, up[3], pad (camera.js:61-77).
 * First visible voxel (label != 0 and not in the sorted `hidden` list) gives
 * the pixel's label and the ray parameter t at which its cell was entered;
 * no hit gives label 0 and depth +inf.  miss[i] counts non-resident bricks
 * ray i crossed before its hit. */
void or_render(const float* cam, uint32_t W, uint32_t H, float grid_size, uint32_t brick_size,
               uint32_t bricks_per_axis, const or_slot* slots, uint64_t n_slots, const uint64_t* labels,
               const uint64_t* hidden, uint32_t n_hidden, uint64_t* out_label, float* out_depth, uint32_t* miss);
/* The same for rows y0, y0 + ystep, ... only (the other rows of the outputs
 * are left as they are); requests (n_slots words or NULL) receives 1 for every
 * non-empty resident brick a ray entered and 3 for every missing one. */
void or_render_rows(const float* cam, uint32_t W, uint32_t H, uint32_t y0, uint32_t ystep, float grid_size,
                    uint32_t brick_size, uint32_t bricks_per_axis, const or_slot* slots, uint64_t n_slots,
                    const uint64_t* labels, const uint64_t* hidden, uint32_t n_hidden, uint64_t* out_label,
                    float* out_depth, uint32_t* miss, uint32_t* requests);

/* The colour path (csv_oracle_rgba.c).  Transfer function of n distinct
 * labels ascending (buildTransferFunctionBuffers + hslToRgb,
 * webgpuSetup.js:389-515), hidden ones transparent; hashLabel
 * (decode.wgsl:135-172); the RGBA ray march for rows y0, y0 + ystep, ...
 * (lighting: light_dir[3], ambient, diffuse). */
void or_transfer_function(const uint64_t* labels, uint32_t n, const uint64_t* hidden, uint32_t n_hidden,
                          uint32_t* rgba);
uint32_t or_label_rgba(uint64_t v, const uint64_t* keys, const uint32_t* cols, uint32_t n_tf);
void or_render_rgba_rows(const float* cam, uint32_t W, uint32_t H, uint32_t y0, uint32_t ystep, float grid,
                         uint32_t bsz, uint32_t bpa, const or_slot* slots, uint64_t n_slots, const uint64_t* labels,
                         const uint64_t* keys, const uint32_t* cols, uint32_t n_tf, const float* lighting,
                         uint32_t* out_rgba);

/* camera.js:61-77 (getUniformData): float32[16] from a double position,
 * direction and vertical field of view. */
void or_camera_uniform(const double* pos, const double* dir, double fov, float* out16);
/* Planning constants of a W x H viewer: focal length (camera.js:114 with
 * min(W, H), renderLoop.js:374), the cosine of the cone's half-angle (cone 0:
 * fov/2 as culling.js:132; cone 1: the screen's half-diagonal) and the brick's
 * bounding radius (culling.js:128). */
void or_serve_constants(uint32_t W, uint32_t H, double fov, uint32_t cone, uint32_t b, double* focal,
                        double* cos_half, double* radius);

/* The viewer's frame loop (csv_oracle_serve.c): plan, cache, decode, render. */
typedef struct or_server or_server;
enum {
    OR_ST_PLANNED = 0,  /* 1 when the step re-planned */
    OR_ST_VISIBLE = 1,  /* bricks some open session needs */
    OR_ST_DECODED = 2,  /* (brick, LOD) blocks admitted and decoded */
    OR_ST_FREED = 3,    /* blocks returned to the free stacks */
    OR_ST_RESIDENT = 4, /* blocks resident after the step */
    OR_ST_REBUILT = 5,  /* 1 when the cache was rebuilt */
    OR_ST_VOX_LO = 6,   /* decoded labels, low and high words */
    OR_ST_VOX_HI = 7,
    OR_ST_SESSION = 8,  /* then per rendered session k: entered (8 + 2k), missing (9 + 2k) */
    OR_SERVE_STATS = 8 + 2 * 8
};
#define OR_MAX_SESSIONS 8
or_server* or_serve_new(const uint8_t* img, size_t len, uint32_t W, uint32_t H, double fov, uint32_t cone,
                        uint64_t cache_bytes, const uint64_t* hidden, uint32_t n_hidden);
/* One step.  The n open sessions sess[k] (ascending ids) with their latest
 * views (position[3], direction[3]); render[k] != 0 for the sessions that
 * submitted a frame this step, whose images are written in order at
 * out_label + j*W*H, out_depth + j*W*H (j counts rendered sessions).
 * A session absent from sess is closed: its blocks are released at the next
 * plan.  stats: OR_SERVE_STATS words. */
int or_serve_step(or_server* s, const uint32_t* sess, const double* views, const uint8_t* render, uint32_t n,
                  uint64_t* out_label, float* out_depth, uint32_t* stats);
/* Admission policy: 0 the cone plan (the reference as it runs), 1 by the rays' requests (the reference's
 * disabled useGPUCulling path). */
void or_serve_set_admit(or_server* s, uint32_t admit);
/* CacheState.compact(): resident blocks packed from offset 0, coarse LODs first, brick order. */
int or_serve_compact(or_server* s);
uint64_t or_serve_n_slots(const or_server* s);
uint32_t or_serve_bricks_per_axis(const or_server* s);
/* The slot table session `session` renders with. */
const or_slot* or_serve_slots(const or_server* s, uint32_t session);
const uint64_t* or_serve_cache(const or_server* s);
void or_serve_free(or_server* s);

/* Encode with a per-brick mode and table (sel: mode | table << 4, or NULL);
 * n_tables > 0 writes a version-2 image with those tables (n_tables x 16
 * frequencies); n_tables == 0 writes version 1 with the dataset's model. */
int or_encode_sel(const uint64_t* vol, size_t W, size_t H, size_t D, uint32_t b, const uint8_t* sel,
                  const uint32_t* tables, uint32_t n_tables, uint8_t** out, size_t* out_len);
/* One x-slab of a larger volume (first brick at x-brick bx0, file index
 * index_base): hist_out receives the sample histogram of its bricks (the
 * every-512th rule in whole-volume numbering); hist_in, when given, is the
 * histogram the model is built from (summed over every slab).  The image holds
 * the slab's bricks only. */
int or_encode_shard(const uint64_t* slab, size_t W, size_t H, size_t D, uint32_t b, uint32_t bx0, uint32_t index_base,
                    const uint64_t* hist_in, uint64_t* hist_out, uint8_t** out, size_t* out_len);

/* The mode / table selector (csv_oracle_select.c). */
int or_encode_stats(const uint64_t* vol, size_t W, size_t H, size_t D, uint32_t b, uint32_t* hist);
void or_table_lengths(const uint32_t* tables, uint32_t n_tables, uint32_t* len);
void or_select_exhaustive(const uint32_t* hist, uint32_t nb, const uint32_t* tables, uint32_t n_tables, uint8_t* sel,
                          uint64_t* cost);
int or_brick_features(const uint64_t* vol, size_t W, size_t H, size_t D, uint32_t b, float* feat);
void or_mlp_forward(const float* params, const float* feat, uint32_t n, float* logits);
float or_mlp_grad(const float* params, const float* feat, const uint8_t* label, uint32_t n, float* grads);

/* or_encode with the bricks spread over `threads` threads (the same bytes). */
int or_encode_threads(const uint64_t* vol, size_t W, size_t H, size_t D, uint32_t b, uint32_t threads,
                      uint8_t** out, size_t* out_len);
/* The native library's seeded synthetic volume (csv_synth_volume, kinds 0-2),
 * restated on the CPU with the same draws and float operations; vol is W*H*D
 * u64, x fastest (csv_oracle_synth.c). */
int or_synth_volume(uint64_t* vol, uint32_t W, uint32_t H, uint32_t D, int kind, uint32_t n_cells, uint32_t n_tubes,
                    float r_min, float r_max, float zero_frac, uint64_t seed, uint32_t threads);

void or_free(void* p);

#ifdef __cplusplus
}
#endif
#endif
