/* csv.h -- C ABI of the B200 compressed-segmentation-volume (CSV) brick codec.
 *
 * One thin C boundary (C linkage, plain pointers and sizes, no C++ or torch
 * types) over the sm_100a CUDA kernels.  It replaces, for this path, the
 * reference's in-process C++ encoder/decoder calls and its WebGPU decode
 * dispatch; each entry point names the reference interface it stands in for
 * (paths relative to the reference project root).
 *
 * Conventions
 *  - Every call returns CSV_OK (0) or a negative CSV_E* code; the message of
 *    the last failure on a context is csv_last_error(ctx).  The reference
 *    throws std::runtime_error in the same places (fileIO.cpp:20,105,119;
 *    brickDecoding.cpp:23; brick.hpp:137).
 *  - A context owns its device buffers and is used by one host thread at a
 *    time.  Pointers named d_* are device pointers on the context's device;
 *    all others are host pointers.  `stream` is a cudaStream_t (0 = legacy
 *    default stream).
 *  - Volumes are uint64 labels, x fastest: vol[x + W*(y + H*z)]
 *    (brick.hpp:183).  Decoded bricks are 8^lod labels in Morton order
 *    (brickDecoding.hpp:174-242, decode.wgsl:239-245).
 *  - lod is the reference's targetLOD: the output has 2^lod voxels per axis,
 *    log2(brick size) is full resolution and 0 is one voxel
 *    (decode.wgsl:22-27, camera.js:118).
 */
#ifndef CSV_B200_H
#define CSV_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CSV_ABI_VERSION 1

enum {
    CSV_OK = 0,
    CSV_EINVAL = -1,   /* bad argument */
    CSV_EFORMAT = -2,  /* malformed .csbd image (fileIO.cpp:118-119) */
    CSV_ECUDA = -3,    /* a CUDA call failed */
    CSV_ENOMEM = -4,   /* device or host allocation failed */
    CSV_ERANGE = -5,   /* size beyond a documented limit */
    CSV_EBRICK = -6,   /* at least one brick reported a nonzero status */
    CSV_EIO = -7       /* a file could not be opened, read or written (fileIO.cpp:20-22, 105-107) */
};

/* Per-brick status bits written by the batched decoder (d_status).  The
 * reference clamps or skips silently in these places; here they are reported. */
#define CSV_BRICK_TRUNCATED 0x1u /* stream ended inside the level structure (decode.wgsl:449) */
#define CSV_BRICK_PALETTE 0x2u   /* palette index past the palette, clamped (decode.wgsl:472-485) */
#define CSV_BRICK_BADOP 0x4u     /* op code 7, label 0 written (decode.wgsl:487-489) */
#define CSV_BRICK_BADREQ 0x8u    /* brick index or lod out of range (decode.wgsl:365-373) */
#define CSV_BRICK_TIMEOUT 0x10u  /* a bounded wait gave up */

typedef struct csv_ctx csv_ctx;
typedef struct csv_dataset csv_dataset;

/* One decode request: brick index in file order (the order of the .csbd and of
 * splitGridIntoBricks, brick.hpp:152-154), target lod, and the element offset
 * of its 8^lod output labels in d_out.  Mirrors DynamicBrickInfo
 * (decode.wgsl:22-27) plus the work-queue entry (decode.wgsl:358). */
typedef struct csv_request {
    uint32_t brick;
    uint32_t lod;
    uint64_t dst;
} csv_request;

typedef struct csv_dataset_info {
    uint32_t num_bricks;
    uint32_t brick_size;
    uint32_t levels;             /* log2(brick_size) + 1 (brick.hpp:50) */
    uint32_t ops_per_checkpoint; /* seek-index spacing */
    uint64_t stream_bytes;       /* sum of rANS stream lengths */
    uint64_t palette_entries;    /* sum of palette sizes */
    uint32_t freq[16];           /* the shared rANS model (fileIO.cpp:38-49) */
    uint32_t cum[16];
} csv_dataset_info;

/* ---- context --------------------------------------------------------
 * A context keeps its decode scratch (grown to the largest brick size seen)
 * and a stream-ordered memory pool for the temporaries of csv_open that holds
 * up to 1 GiB of freed memory between opens; csv_destroy releases both. */
int csv_create(int device, csv_ctx** out);
void csv_destroy(csv_ctx* ctx);
const char* csv_last_error(const csv_ctx* ctx);
int csv_abi_version(void);
void csv_free(void* p); /* frees buffers this library returned (csv_encode) */

/* ---- encoder ----------------------------------------------------------
 * splitGridIntoBricks<b> (brick.hpp:134) + Encoding::compressDataset<b>
 * (brickEncoding.hpp:467) + saveDatasetToFile (fileIO.cpp:15), as main.cpp:76-84
 * runs them: the whole volume becomes one .csbd v1 image, byte-identical to
 * the reference encoder's file (with brick_size stored in the header; the
 * reference always writes 64 there, fileIO.cpp:28).  brick_size is a power of
 * two in [8, 64]. */
int csv_encode(csv_ctx* ctx, const uint64_t* volume, uint32_t W, uint32_t H, uint32_t D,
               uint32_t brick_size, uint8_t** out, size_t* out_len);
/* Same, volume already in device memory; the image stays in a context-owned
 * device buffer (valid until the next encode on ctx) and its length is
 * returned; csv_encoded_image() gives the device pointer.  The per-brick
 * seek index the encoder produced as a by-product is kept with it. */
int csv_encode_device(csv_ctx* ctx, const uint64_t* d_volume, uint32_t W, uint32_t H, uint32_t D,
                      uint32_t brick_size, void* stream, size_t* image_len);
int csv_encoded_image(csv_ctx* ctx, const uint8_t** d_image, size_t* len);

/* No counterpart in the reference: one rank's part of a volume split into
 * x-slabs of whole bricks (the split order puts bx outermost, brick.hpp:152-154,
 * so a slab is a contiguous range of file indices).  The only exchange step of
 * the encoder is the rANS model: it comes from the bricks whose file index is a
 * multiple of 512 (brickEncoding.hpp:481-482), wherever they live.
 *   1. csv_encode_shard_bricks: the slab (d_slab: W x H x D, x fastest, W the
 *      slab's width) with its first brick at x-brick bx0 of the whole volume and
 *      file index index_base; returns hist[16], the nibble histogram of its
 *      sampled bricks.
 *   2. the caller sums hist over the ranks (an all-reduce);
 *   3. csv_encode_shard_finish: the model from the summed histogram, then the
 *      slab's image (header + its brick records, as csv_encode_device leaves it).
 * The whole file is the header with numBricks set to the total, then every
 * rank's records in rank order: byte-identical to csv_encode of the whole
 * volume (csvb200/dist.py runs the protocol over torch.distributed). */
int csv_encode_shard_bricks(csv_ctx* ctx, const uint64_t* d_slab, uint32_t W, uint32_t H, uint32_t D,
                            uint32_t brick_size, uint32_t bx0, uint32_t index_base, uint64_t* hist, void* stream);
int csv_encode_shard_finish(csv_ctx* ctx, const uint64_t* hist, void* stream, size_t* image_len);

/* ---- dataset -----------------------------------------------------------
 * loadDatasetFromFile (fileIO.cpp:101-182) / loadDatasetFromArrayBuffer
 * (web/scripts/datasetLoader.js:39-146): parse a .csbd v1 image, stage
 * palettes and rANS streams in HBM, and build the seek index on the GPU (one
 * serial rANS pass per brick; the "cold" step).  Bricks keep file order. */
int csv_open(csv_ctx* ctx, const uint8_t* image, size_t len, csv_dataset** out);
/* Open the image the last csv_encode_device produced on ctx, taking its seek
 * index from the encoder instead of rebuilding it. */
int csv_open_encoded(csv_ctx* ctx, csv_dataset** out);
int csv_dataset_info_get(const csv_dataset* ds, csv_dataset_info* info);
/* Device time in ms of the seek-index passes csv_open ran for this dataset
 * (CUDA events on its stream around them); 0 when none ran (csv_open_encoded,
 * csv_dataset_concat).  No reference counterpart: the reference's index is the
 * serial walk inside decodeRansStream (brickDecoding.cpp:153-188). */
int csv_dataset_index_ms(const csv_dataset* ds, float* ms);
/* Seek-index sidecar.  csv_index_save writes, for the dataset's image, the
 * rANS state before every 512th symbol of each brick (8 bytes per 512
 * symbols; the buffer is this library's, free it with csv_free).
 * csv_open_indexed opens the image as csv_open does, with pass 1 of the index
 * run as independent 512-symbol pieces from those states: each piece checks
 * that it ends in the next stored state, so the index equals csv_open's, and a
 * sidecar of another image, or a damaged one, fails with CSV_EFORMAT (open
 * without it then).  No reference counterpart: the reference rebuilds the walk
 * on every load (brickDecoding.cpp:153-188). */
int csv_index_save(csv_ctx* ctx, const csv_dataset* ds, uint8_t** out, size_t* out_len);
int csv_open_indexed(csv_ctx* ctx, const uint8_t* image, size_t len, const uint8_t* sidecar, size_t sidecar_len,
                     csv_dataset** out);
/* Morton brick IDs (datasetLoader.js:113-123) in file order, host array. */
int csv_dataset_ids(const csv_dataset* ds, uint32_t* ids, uint32_t n);
void csv_close(csv_dataset* ds);

/* ---- decoder -----------------------------------------------------------
 * decodeRansStream (brickDecoding.cpp:153-188) + decodeBrick<b>
 * (brickDecoding.hpp:174-242) at full resolution, and decode.wgsl:decodeBrick
 * (decode.wgsl:344-509) at any lod, in label space, for a batch of requests
 * in one launch.  d_reqs: n requests in device memory.  d_out: labels;
 * request k writes 8^lod labels at d_out + d_reqs[k].dst.  d_status: n
 * per-request CSV_BRICK_* words (0 = clean).  A brick whose root stop bit is
 * set (the whole brick is one label) decodes to palette[0] everywhere.
 * Asynchronous on `stream`. */
int csv_decode_batch(csv_ctx* ctx, const csv_dataset* ds, const csv_request* d_reqs, uint32_t n,
                     uint64_t* d_out, uint32_t* d_status, void* stream);

/* No counterpart in the reference.  csv_decode_batch without any allocation,
 * for callers that cannot call cudaMalloc when they decode: render or serving
 * loops that must not stall the device (cudaMalloc can synchronize it), and
 * hosts that route all device memory through their own arena.  The decode
 * scratch (op records, active-node lists, the work-queue counter) lives in one
 * file-scope device array of CSV_STATIC_SCRATCH_BYTES that every GPU loading
 * this library reserves until the process exits; the caller still passes the
 * dataset, requests, outputs and status words.  The array holds as many
 * concurrent bricks as fit (47 for 64^3 bricks), so large batches run slower
 * than with csv_decode_batch; a brick size whose per-CTA scratch exceeds the
 * array is rejected with CSV_ERANGE.  The first call on a device looks up the
 * array's device address with that device current (make that first call
 * before any stream capture).  Every call shares the one array and leaves its
 * contents behind: calls that overlap on the GPU (other streams, other host
 * threads) race and must be serialized by the caller. */
#define CSV_STATIC_SCRATCH_BYTES (64u << 20)
int csv_decode_batch_static(csv_ctx* ctx, const csv_dataset* ds, const csv_request* d_reqs, uint32_t n,
                            uint64_t* d_out, uint32_t* d_status, void* stream);

/* ---- mixed brick sizes ---------------------------------------------------
 * One dataset made of several: the bricks of parts[0], then of parts[1], ...
 * (file order inside each part), every brick keeping its own brick size and
 * rANS model, so that one decode launch can mix, e.g., 32^3 and 64^3 bricks.
 * (A .csbd file holds one brick size, fileIO.cpp:28.)  Brick indices of
 * requests are global: brick i of part k is sum_{j<k} num_bricks(parts[j]) + i.
 * The parts stay valid and independent of the result. */
int csv_dataset_concat(csv_ctx* ctx, const csv_dataset* const* parts, uint32_t n, csv_dataset** out);

/* ---- captured decode and its autotuner (no reference counterpart) ---------
 * The decode of a fixed request array into a fixed output, captured once into
 * a CUDA graph (work-queue reset + the persistent decode kernel) and replayed
 * by csv_graph_launch.  Knobs: ctas_per_sm (0 = as many as fit), stage (1 =
 * stage each brick's compressed stream in shared memory by a bulk copy), lpt
 * (1 = hand out the largest bricks first: a request permutation computed at
 * creation), layout (for datasets with 64^3 bricks: 0 = requests above LOD 5
 * in the decode kernel that holds every level in shared memory -- those whose
 * brick has fewer than 255 palette entries with 8-bit node values, three CTAs
 * per SM, the others with 16- or 32-bit values, two CTAs per SM -- then the
 * rest in the six-CTA-per-SM kernel, up to three launches; 1 = every request
 * in the six-CTA kernel, which keeps a 64^3 brick's last parent level in its
 * global scratch; 2 = as 0 without the 8-bit part). */
typedef struct csv_decode_config {
    uint32_t ctas_per_sm;
    uint32_t stage;
    uint32_t lpt;
    uint32_t layout;
} csv_decode_config;

typedef struct csv_graph csv_graph;

int csv_decode_graph_create(csv_ctx* ctx, const csv_dataset* ds, const csv_request* d_reqs, uint32_t n,
                            uint64_t* d_out, uint32_t* d_status, const csv_decode_config* cfg, csv_graph** out);
int csv_graph_launch(csv_graph* g, void* stream);
/* Decode kernels one replay of the graph launches (1; 2 or 3 when it splits the
 * requests by output size and palette size; 0 for an empty batch).  In a split
 * replay each kernel may start while the one before still has bricks decoding;
 * the replay as a whole still completes in stream order like any other graph
 * launch.  A split graph uses further decode scratch of the context (allocated
 * on the first split graph's creation that needs it), so graphs of one context
 * replay one at a time. */
int csv_graph_kernels(const csv_graph* g, uint32_t* n);
void csv_graph_destroy(csv_graph* g);
/* Times every candidate configuration on this batch (a captured graph each,
 * `reps` timed replays after one warm-up, median) and returns the fastest and
 * its time in milliseconds.  Writes d_out / d_status like a decode. */
int csv_decode_autotune(csv_ctx* ctx, const csv_dataset* ds, const csv_request* d_reqs, uint32_t n, uint64_t* d_out,
                        uint32_t* d_status, uint32_t reps, csv_decode_config* best, float* best_ms);

/* Host convenience over the above, as main.cpp:86-118 uses the reference
 * decoder: parse `image`, decode every brick at `lod` and copy the labels to
 * the host (brick i at out + i*8^lod).  status: numBricks words or NULL. */
int csv_decode_image(csv_ctx* ctx, const uint8_t* image, size_t len, uint32_t lod, uint64_t* out,
                     uint32_t* status);

/* ---- ray marcher ---------------------------------------------------------
 * rayTrace.wgsl:rayTrace (rayTrace.wgsl:565-906) in label/depth space: per
 * pixel of a width x height image, the first visible voxel along the camera
 * ray through the decoded brick cache.  A voxel is visible when its label is
 * not 0 and not in `d_hidden` (sorted ascending, n_hidden entries; labels the
 * transfer function hides).  d_label_out receives the label (0 = no hit),
 * d_depth_out the ray parameter t at which the hit cell was entered (+inf =
 * no hit).  The camera is camera.js:getUniformData (camera.js:61-77); the
 * volume is the cube [0, grid_size)^3 of bricks_per_axis^3 bricks
 * (SceneInfo, rayTrace.wgsl:87-96).  Slots are indexed by brick Morton code
 * (rayTrace.wgsl:654-657).  d_requests (optional, n_slots words, zeroed by
 * the caller) gets 1 for every non-empty resident brick a ray entered and 3
 * for every missing one it crossed (brickRequests, rayTrace.wgsl:684-686).
 * Bit-identical to the scalar restatement on the CPU (same float operations,
 * no fused multiply-add). */
typedef struct csv_camera {
    float position[3];
    float tan_half_fov;
    float forward[3];
    float pad0;
    float right[3];
    float pad1;
    float up[3];
    float pad2;
} csv_camera;

#define CSV_SLOT_EMPTY 0x1u   /* every palette entry is 0 (webgpuSetup.js:315-322) */
#define CSV_SLOT_MISSING 0x2u /* not resident in the decoded cache */

typedef struct csv_brick_slot {
    uint64_t offset; /* first of the brick's 8^lod labels in d_labels */
    uint32_t lod;    /* targetLOD of the resident copy */
    uint32_t flags;  /* CSV_SLOT_* */
} csv_brick_slot;

int csv_render(csv_ctx* ctx, const csv_camera* camera, uint32_t width, uint32_t height, float grid_size,
               uint32_t brick_size, uint32_t bricks_per_axis, const csv_brick_slot* d_slots, uint64_t n_slots,
               const uint64_t* d_labels, const uint64_t* d_hidden, uint32_t n_hidden, uint64_t* d_label_out,
               float* d_depth_out, uint32_t* d_requests, void* stream);

/* The shader's colour path on the same traversal (rayTrace.wgsl:565-906 with
 * getVoxelColor's colours): every sample's label is coloured by the transfer
 * function (d_tf_keys sorted ascending with their RGBA8 d_tf_rgba, as
 * csv_transfer_function builds them; a label not in it takes hashLabel's
 * colour, decode.wgsl:135-172; label 0 is transparent), composited front to
 * back with the LOD opacity correction, shaded above alpha 0.35 by the
 * LOD-strided alpha gradient, the diffuse light and, above 0.4, a 64-step
 * shadow ray; the ray stops at alpha 0.95.  d_rgba_out: width x height RGBA8
 * (r | g << 8 | b << 16 | a << 24).  Differences from the shader: a brick at
 * LOD 0 is coloured by the transfer function of its label (the shader reads
 * the label's low bytes as a colour, rayTrace.wgsl:165-177), and samples in
 * bricks that are not resident have alpha 0.  Floating point follows the
 * CPU restatement's order without fused multiply-add; powf and expf are
 * CUDA's, so images agree with it to rounding. */
typedef struct csv_lighting {
    float light_dir[3]; /* towards the light (unnormalised) */
    float ambient;
    float diffuse;
    float pad[3];
} csv_lighting;
/* The viewer's default lighting (webgpuSetup.js:24-31, 205-219) for a light
 * at angle `light_angle_deg` on its west-east arc (25 by default). */
int csv_lighting_default(double light_angle_deg, csv_lighting* out);
/* buildTransferFunctionBuffers (webgpuSetup.js:389-465) on a dataset: its
 * distinct non-zero palette labels ascending (host keys) and their RGBA8
 * (host rgba); labels in `hidden` (host, any order) get 0.  *n receives the
 * count; CSV_ERANGE when it exceeds cap. */
int csv_transfer_function(const csv_dataset* ds, const uint64_t* hidden, uint32_t n_hidden, uint64_t* keys,
                          uint32_t* rgba, uint32_t cap, uint32_t* n);
int csv_render_rgba(csv_ctx* ctx, const csv_camera* camera, uint32_t width, uint32_t height, float grid_size,
                    uint32_t brick_size, uint32_t bricks_per_axis, const csv_brick_slot* d_slots, uint64_t n_slots,
                    const uint64_t* d_labels, const uint64_t* d_tf_keys, const uint32_t* d_tf_rgba, uint32_t n_tf,
                    const csv_lighting* lighting, uint32_t* d_rgba_out, uint32_t* d_requests, void* stream);

/* ---- serving loop --------------------------------------------------------
 * The viewer's frame loop with its cache on the device.  Replaces the host
 * side of renderLoop.js:208-340 (frame), cacheProcessing.js:99-232
 * (processCache), cacheManager.js:10-246 (CacheState), camera.js:103-137
 * (calculateBrickLOD), culling.js:22-171 (camera-moved, cone and
 * transfer-function tests), and drives the decoder and ray marcher above.
 *
 * A server holds one dataset (one brick size), a label cache in HBM and the
 * brick slot table.  Up to max_sessions viewers share it: each submits frames
 * (a camera and two device images); csv_serve_step serves every session with
 * a pending frame in one step -- one plan over every open session, one
 * decode launch for all admitted blocks, one render per new frame -- all
 * enqueued on `stream` with no host synchronisation.  Sessions join (first
 * submit) and leave (csv_serve_close) between steps; their decode work shares
 * the launches of the sessions already open.  Cache blocks are keyed by
 * (brick, LOD) and every session has its own slot table and LODs, so a
 * session's image does not depend on which other sessions are open while the
 * cache has room for all of them.  A session that submits again before the
 * step replaces its pending frame (the newest camera wins).  A session's LODs
 * are re-planned when its camera moved more than 0.5 units or turned more
 * than 0.05 rad since its last re-plan (culling.js:6-56); a step with no such
 * change and no session joining or leaving only renders.  csv_serve_poll
 * returns per-frame counters and the device time of each finished step.  One
 * host thread per server. */
typedef struct csv_server csv_server;

#define CSV_CONE_REFERENCE 0u /* cone half-angle fov/2 (culling.js:132) */
#define CSV_CONE_SCREEN 1u    /* cone half-angle to the screen corner: every brick a ray can reach */

/* Admission policy (csv_serve_config.admit).  CONE: a session needs every
 * brick its cone and LOD tests pass (the reference's loop as it runs,
 * cacheProcessing.js:99-232).  RAYS: of those, only the bricks its rays entered
 * in its last render (the request words of rayTrace.wgsl:682-686 driving
 * admission and eviction: the reference's useGPUCulling path,
 * cacheProcessing.js:134-164, which it ships switched off).  A session with no
 * render since the last plan (its first frame) keeps the cone plan; a step
 * re-plans when an open session rendered since the last plan, so bricks that
 * rays stop reaching (hidden behind bricks that arrived) are released while
 * the camera stands still. */
#define CSV_ADMIT_CONE 0u
#define CSV_ADMIT_RAYS 1u

typedef struct csv_serve_config {
    uint32_t width, height;   /* viewport of every session (pixels) */
    uint32_t max_sessions;    /* sessions served together, 1..8 (0 = 1) */
    uint32_t cone;            /* CSV_CONE_* */
    double fov;               /* vertical field of view, radians (camera.js:19: pi/3) */
    uint64_t cache_bytes;     /* label cache incl. a palette-0 table of 8 B per brick; 0 = 24 GiB */
    uint32_t admit;           /* CSV_ADMIT_* */
    uint32_t reserved;        /* 0 */
} csv_serve_config;

typedef struct csv_view {
    double position[3];  /* camera position, voxel units */
    double direction[3]; /* view direction (normalised by the server) */
} csv_view;

typedef struct csv_frame_stats {
    uint64_t step;           /* step sequence number */
    uint32_t session;
    uint32_t planned;        /* 1 when the step re-planned */
    uint32_t visible;        /* bricks some open session needs */
    uint32_t decoded;        /* (brick, LOD) blocks admitted and decoded */
    uint32_t freed;          /* cache blocks released */
    uint32_t resident;       /* cache blocks resident after the step */
    uint32_t rebuilt;        /* 1 when the cache was rebuilt (allocation failure) */
    uint32_t entered;        /* non-empty bricks this session's rays entered */
    uint32_t missing;        /* of those, bricks with no data in its slot table */
    uint32_t reserved;
    uint64_t decoded_voxels;
    float ms;                /* device time of the whole step (CUDA events) */
    uint32_t reserved2;
} csv_frame_stats;

/* Device views of a server's state, for checks and custom passes. */
typedef struct csv_serve_info {
    const csv_brick_slot* slots; /* n_slots entries, by brick Morton code */
    uint64_t n_slots;
    const uint64_t* cache;       /* cache_labels u64: palette-0 table, then blocks */
    uint64_t cache_labels;
    uint64_t palette_table;      /* labels before the first block */
    uint32_t bricks_per_axis, brick_size;
    float grid_size;
    uint32_t pad;
    double focal;                /* LOD focal length, (min(W, H)/2) / tan(fov/2) */
    double cos_half;             /* cosine of the cone's half-angle */
    const uint32_t* decode_status; /* per admitted request of the last planned step */
} csv_serve_info;

/* `hidden`: labels the transfer function hides (host array, any order); a
 * brick whose palette has no other non-zero label is empty.  Creation also
 * builds the dataset's transfer function for RGBA frames (csv_transfer_function:
 * a host copy and sort of every palette label, once). */
int csv_serve_create(csv_ctx* ctx, const csv_dataset* ds, const csv_serve_config* cfg, const uint64_t* hidden,
                     uint32_t n_hidden, csv_server** out);
/* d_label (W*H u64) and d_depth (W*H f32) are device images the step writes. */
int csv_serve_submit(csv_server* srv, uint32_t session, const csv_view* view, uint64_t* d_label, float* d_depth);
/* The same frame as the viewer shows it: an RGBA8 image (W*H words, device)
 * from csv_render_rgba's colour path through the dataset's transfer function
 * (built at create; the hidden labels transparent) and the server's lighting
 * (csv_lighting_default(25) until csv_serve_set_lighting). */
int csv_serve_submit_rgba(csv_server* srv, uint32_t session, const csv_view* view, uint32_t* d_rgba);
int csv_serve_set_lighting(csv_server* srv, const csv_lighting* light);
int csv_serve_step(csv_server* srv, void* stream, uint64_t* step_id);
/* Up to `max` finished frames (one per session of each finished step), oldest
 * first; wait != 0 blocks until every step enqueued so far has finished. */
int csv_serve_poll(csv_server* srv, csv_frame_stats* out, uint32_t max, uint32_t* n_out, int wait);
/* Compaction (CacheState.compact(), cacheManager.js:170-211; the reference
 * defines it and never calls it): every resident block is kept and placed
 * again from the start of the block space, coarse LODs first and brick order
 * within a LOD, the free stacks are emptied and fresh space starts after the
 * last block, so that fragmented free blocks of one LOD become space for any.
 * Enqueued on `stream` like a step (the blocks are decoded again into their new
 * places, which costs what moving them would at the HBM rate, and needs no
 * second buffer); every open session's slot table points at the new places
 * when it completes.  Renders nothing and reports no frame. */
int csv_serve_compact(csv_server* srv, void* stream);
/* A session leaves: its cache blocks are released by the next step. */
int csv_serve_close(csv_server* srv, uint32_t session);
/* The float camera the server renders a view with (camera.js:61-77). */
int csv_serve_camera(const csv_server* srv, const csv_view* view, csv_camera* out);
/* Device views of the cache and of `session`'s slot table. */
int csv_serve_state(const csv_server* srv, uint32_t session, csv_serve_info* info);
int csv_serve_destroy(csv_server* srv);

/* ---- learned mode / table selector (no reference counterpart) ---------
 * Dense layer on the tensor cores (tcgen05, accumulator in tensor memory):
 * C[M][N] = epilogue(A[M][K] . B[N][K]^T), A and B bf16 row-major (K
 * contiguous), fp32 accumulation.  Epilogue, in order: + d_bias[n] (if not
 * NULL), max(0, .) (if relu), * (d_mask[m][n] > 0) (if d_mask, bf16 [M][N]: the
 * ReLU gradient); outputs (each optional): d_C fp32 [M][N], d_Cb bf16 [M][N],
 * d_CbT bf16 [N][M], d_CT fp32 [N][M].  M % 128 == 0, N % 16 == 0, K % 64 == 0.
 * d_err (optional) is set to 1 if a bounded wait gave up. */
int csv_gemm_bf16(csv_ctx* ctx, const void* d_A, const void* d_B, uint32_t M, uint32_t N, uint32_t K,
                  const float* d_bias, const void* d_mask, uint32_t relu, float* d_C, void* d_Cb, void* d_CbT,
                  float* d_CT, uint32_t* d_err, void* stream);

/* Encoding modes: where several ops reproduce a child's label, the reference
 * takes Rp, then Rx, Ry, Rz, then a palette op (brickEncoding.hpp:198-282).
 * Mode m keeps that grammar and changes the preference: m % 6 picks the order
 * of the neighbour axes (xyz, xzy, yxz, yzx, zxy, zyx), m >= 6 tries the
 * neighbours before the parent.  Mode 0 is the reference's order.  Decoding
 * does not depend on the mode.
 *
 * Version-2 images (`.csbd` version 2): a 28-byte header (magic, version 2,
 * numBricks, brickSize, 16, 4096, n_tables), n_tables x (freq[16], cum[16])
 * shared rANS tables, and brick records with a u32 after the ID naming the
 * brick's table (bits 4..7) and mode (bits 0..3).  csv_open reads both
 * versions. */
#define CSV_MODES 12
#define CSV_MAX_TABLES 16
#define CSV_FEATURES 32
/* Per brick (split order) and mode: the 16-bin histogram of the nibbles the
 * rANS coder would code (d_hist: numBricks x 12 x 16 u32). */
int csv_encode_stats(csv_ctx* ctx, const uint64_t* d_volume, uint32_t W, uint32_t H, uint32_t D, uint32_t brick_size,
                     uint32_t* d_hist, void* stream);
/* Exhaustive choice: per brick the (mode, table) with the fewest estimated
 * bits, sum_s hist[mode][s] * -log2(freq[table][s] / 4096), ties to the lower
 * mode then table.  tables: host, n_tables x 16 frequencies.  d_sel: per brick
 * mode | table << 4.  d_cost (optional): numBricks x 12 x n_tables estimated
 * bits in 16.16 fixed point. */
int csv_select_exhaustive(csv_ctx* ctx, const uint32_t* d_hist, uint32_t n_bricks, const uint32_t* tables,
                          uint32_t n_tables, uint8_t* d_sel, uint64_t* d_cost, void* stream);
/* csv_encode_device with a per-brick mode and shared table (d_sel, device, one
 * byte per brick: mode | table << 4; NULL = mode 0, table 0).  n_tables > 0
 * writes a version-2 image with these tables (host, n_tables x 16
 * frequencies, each >= 1, summing to 4096); n_tables == 0 writes version 1. */
int csv_encode_device_sel(csv_ctx* ctx, const uint64_t* d_volume, uint32_t W, uint32_t H, uint32_t D,
                          uint32_t brick_size, const uint32_t* tables, uint32_t n_tables, const uint8_t* d_sel,
                          void* stream, size_t* image_len);
/* 32 cheap statistics per brick (d_features: numBricks x 32 fp32): distinct
 * labels of an 8^3 sample; over the rows of even y and even z (all x), label
 * equality of neighbours at distance 1 and 4 per axis, the fraction of label
 * 0, the histogram of run lengths along x and the run count; and the
 * op-nibble histogram of the 8^3 sample encoded as a brick. */
int csv_brick_features(csv_ctx* ctx, const uint64_t* d_volume, uint32_t W, uint32_t H, uint32_t D,
                       uint32_t brick_size, float* d_features, void* stream);

/* The selector network: 32 features -> 256 -> 256 (ReLU) -> 12 mode logits
 * and 16 table logits, bf16 weights with fp32 masters, fp32 accumulation on
 * the tensor cores (csv_gemm_bf16).  params (host, CSV_MLP_PARAMS floats):
 * W1 [256][64] (columns 32..63 unused), b1 [256], W2 [256][256], b2 [256],
 * W3 [32][256] (rows 28..31 unused), b3 [32]. */
#define CSV_MLP_PARAMS (256 * 64 + 256 + 256 * 256 + 256 + 32 * 256 + 32)
typedef struct csv_mlp csv_mlp;
int csv_mlp_create(csv_ctx* ctx, const float* params, csv_mlp** out);
void csv_mlp_destroy(csv_mlp* net);
/* Host copies of the parameters and of the last gradients (either may be NULL). */
int csv_mlp_params(const csv_mlp* net, float* params, float* grads);
/* Logits (d_logits: count x 32 fp32, optional) and the argmax choice per brick
 * (d_sel: mode | table << 4, optional) for count feature rows, in one fused
 * kernel (activations stay on the SM).  d_features and d_logits 16-byte aligned. */
int csv_mlp_forward(csv_mlp* net, const float* d_features, uint32_t count, float* d_logits, uint8_t* d_sel,
                    void* stream);
/* Forward and backward of the mean cross-entropy of both heads against
 * d_label (mode | table << 4 per row); gradients stay in the network; *loss
 * (host, optional) receives the loss. */
int csv_mlp_grad(csv_mlp* net, const float* d_features, const uint8_t* d_label, uint32_t count, float* loss,
                 void* stream);
/* One Adam step (Kingma & Ba) with the last gradients. */
int csv_mlp_adam(csv_mlp* net, float lr, float beta1, float beta2, float eps, void* stream);
/* CSV_OK, or CSV_ECUDA when a tensor-core wait gave up since creation. */
int csv_mlp_status(const csv_mlp* net);

/* Selector files (no reference counterpart): the shared tables and the
 * network's parameters, so that a learned encode runs without a training run.
 * Little-endian: u32 magic "CSVS" (0x53565343), u32 version 1, u32
 * CSV_MLP_PARAMS, u32 n_tables (1..16), u32 tables[n_tables][16], f32
 * params[CSV_MLP_PARAMS], u32 FNV-1a hash of every byte before it.  Host only:
 * write takes params as csv_mlp_params returns them; read fills params
 * (CSV_MLP_PARAMS floats), tables (room for 16 x 16) and *n_tables, and
 * refuses a file whose size, header, hash or tables (each >= 1, summing to
 * 4096) are wrong with CSV_EFORMAT, a missing file with CSV_EIO. */
int csv_selector_write(const char* path, const float* params, const uint32_t* tables, uint32_t n_tables);
int csv_selector_read(const char* path, float* params, uint32_t* tables, uint32_t* n_tables);
/* The learned encode in one call: csv_brick_features, csv_mlp_forward's choice
 * per brick, csv_encode_device_sel with those choices and tables (a version-2
 * image, as csv_encode_device leaves it for csv_encoded_image).  Allocates the
 * per-brick features and choices for the call. */
int csv_encode_learned(csv_ctx* ctx, const uint64_t* d_volume, uint32_t W, uint32_t H, uint32_t D,
                       uint32_t brick_size, csv_mlp* net, const uint32_t* tables, uint32_t n_tables, void* stream,
                       size_t* image_len);

/* ---- workload generator (no reference counterpart) --------------------
 * Seeded synthetic label volume on the device, x fastest: kind 0 = Voronoi
 * (n_cells cells, then a random half-space slab of label 0 covering about
 * zero_frac of the volume); kind 1 = n_tubes cubic tubes with radius in
 * [r_min, r_max] over a Voronoi background with about zero_frac of its cells
 * set to 0.  IDs are uniform in [1, 2^64-2]. */
int csv_synth_volume(csv_ctx* ctx, uint64_t* d_volume, uint32_t W, uint32_t H, uint32_t D, int kind,
                     uint32_t n_cells, uint32_t n_tubes, float r_min, float r_max, float zero_frac,
                     uint64_t seed, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CSV_B200_H */
