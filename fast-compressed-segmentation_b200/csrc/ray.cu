// ray.cu -- label/depth brick ray marcher (sm_100a).
//
// Restates rayTrace.wgsl:565-906 (paths relative to the reference root) in
// label space: per pixel, the slab test against the volume, the brick DDA,
// the LOD-strided voxel DDA inside each non-empty brick, and the first visible
// voxel.  The output is the voxel's label and the ray parameter t at which its
// cell was entered (label 0, depth +inf when nothing is hit), not RGBA: the
// shading, shadow rays and compositing of the shader do not change which voxel
// is hit first.  Every float operation follows the shader's order with one
// rounding each; this file is compiled with --fmad=false so that no multiply-
// add is contracted, which makes the image bit-identical to the scalar CPU
// restatement in the oracle.
//
// Brick slots are indexed by the brick's Morton code (rayTrace.wgsl:654-657,
// bricks sorted by ID in datasetLoader.js:143).  A slot flagged empty is
// skipped (rayTrace.wgsl:673-682).  Every other brick a ray enters gets its
// request word set, as brickRequests (rayTrace.wgsl:684-686): 1 when the brick
// is resident, 3 when its slot is flagged missing (not in the decoded cache),
// in which case the ray skips it.
//
// The RGBA mode (render_kernel<true>) restates the shader's colour path on the
// same traversal: each sample's label goes through the transfer function
// (decode.wgsl:135-172: a table of (label, RGBA8) sorted by label, else the
// label hash; label 0 transparent), samples with alpha above 0.05 are
// composited front to back with the per-LOD opacity correction
// (rayTrace.wgsl:794-837), those above 0.35 shaded with the LOD-strided alpha
// gradient (computeGradientLOD, :428-455), the diffuse light and, above 0.4,
// the shadow ray (traceShadowRay, :329-397); the ray stops at alpha 0.95.  The
// pixel is RGBA8 (:897-905).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "csv_internal.h"

namespace csv {

struct RayArgs {
    float o[3], thf, fwd[3], right[3], up[3];
    uint32_t W, H;
    float grid;
    int bs, lb, num_bricks;
    const csv_brick_slot* slots;
    uint64_t n_slots;
    const uint64_t* labels;
    const uint64_t* hidden;
    uint32_t n_hidden;
    uint64_t* out_label;
    float* out_depth;
    uint32_t* requests;
    // RGBA mode
    const uint64_t* tf_keys;  // sorted labels of the transfer function
    const uint32_t* tf_rgba;  // their RGBA8 (r | g << 8 | b << 16 | a << 24)
    uint32_t n_tf;
    float light[3], ambient, diffuse;
    uint32_t* out_rgba;
};

__device__ __forceinline__ float fsgn(float x) { return x > 0.f ? 1.f : (x < 0.f ? -1.f : 0.f); }
__device__ __forceinline__ int isgn(float x) { return (x > 0.f ? 1 : 0) + (x < 0.f ? -1 : 0); }
__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ uint32_t spread10(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}
__device__ __forceinline__ uint32_t mort(uint32_t x, uint32_t y, uint32_t z) {
    return spread10(x) | (spread10(y) << 1) | (spread10(z) << 2);
}

__device__ __forceinline__ bool is_hidden(const RayArgs& A, uint64_t v) {
    uint32_t lo = 0, hi = A.n_hidden;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (A.hidden[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    return lo < A.n_hidden && A.hidden[lo] == v;
}

// hashLabel (decode.wgsl:135-172): the transfer function's colour, else a
// colour mixed from the label's two 32-bit halves with alpha 0x40; label 0 is
// transparent.  The table's keys are unique, so a binary search finds the entry
// the shader's linear search finds.
__device__ __forceinline__ uint32_t label_rgba(const RayArgs& A, uint64_t v) {
    if (v == 0) return 0u;
    uint32_t lo = 0, hi = A.n_tf;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (A.tf_keys[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    if (lo < A.n_tf && A.tf_keys[lo] == v) return A.tf_rgba[lo];
    uint32_t sl = (uint32_t)v, sh = (uint32_t)(v >> 32);
    sl = sl ^ sh;
    sl = sl ^ (sl >> 16);
    sl = sl * 0x7feb352du;
    sl = sl ^ (sl >> 15);
    sh = sh ^ sl;
    sh = sh ^ (sh >> 16);
    sh = sh * 0x85ebca6bu;
    sh = sh ^ (sh >> 13);
    return (sl & 0xFFu) | (((sl >> 8) & 0xFFu) << 8) | (((sh >> 8) & 0xFFu) << 16) | (0x40u << 24);
}

__device__ __forceinline__ float chan(uint32_t rgba, int k) { return (float)((rgba >> (8 * k)) & 0xFFu) / 255.0f; }

// getVoxelColor (:159-198) of a resident slot at brick-local voxel (x, y, z), as RGBA8
__device__ __forceinline__ uint32_t slot_rgba(const RayArgs& A, const csv_brick_slot& sl, int x, int y, int z) {
    const int sh = A.lb - (int)sl.lod;
    const uint64_t lab = sl.lod == 0 ? __ldg(A.labels + sl.offset)
                                     : __ldg(A.labels + sl.offset + mort((uint32_t)x >> sh, (uint32_t)y >> sh,
                                                                          (uint32_t)z >> sh));
    return label_rgba(A, lab);
}

// sampleAlpha (:272-299): alpha at a world voxel through its brick's slot (0 outside
// the volume, for empty bricks, and for bricks not resident in the cache)
__device__ float sample_alpha(const RayArgs& A, int wx, int wy, int wz) {
    const int g = (int)A.grid;
    if (wx < 0 || wy < 0 || wz < 0 || wx >= g || wy >= g || wz >= g) return 0.0f;
    const int bx = wx / A.bs, by = wy / A.bs, bz = wz / A.bs;
    if (bx >= A.num_bricks || by >= A.num_bricks || bz >= A.num_bricks) return 0.0f;
    const uint32_t m = mort((uint32_t)bx, (uint32_t)by, (uint32_t)bz);
    if (m >= A.n_slots) return 0.0f;
    const csv_brick_slot sl = A.slots[m];
    if (sl.flags & (CSV_SLOT_EMPTY | CSV_SLOT_MISSING)) return 0.0f;
    return chan(slot_rgba(A, sl, wx - bx * A.bs, wy - by * A.bs, wz - bz * A.bs), 3);
}

// sampleAlphaInBrick (:301-318)
__device__ __forceinline__ float sample_alpha_in(const RayArgs& A, const csv_brick_slot& sl, const int* bmin, int wx,
                                                 int wy, int wz) {
    const int g = (int)A.grid;
    if (wx < 0 || wy < 0 || wz < 0 || wx >= g || wy >= g || wz >= g) return 0.0f;
    const int lx = wx - bmin[0], ly = wy - bmin[1], lz = wz - bmin[2];
    if (lx < 0 || ly < 0 || lz < 0 || lx >= A.bs || ly >= A.bs || lz >= A.bs) return sample_alpha(A, wx, wy, wz);
    return chan(slot_rgba(A, sl, lx, ly, lz), 3);
}

// traceShadowRay (:329-397): 1 = lit, 0 = occluded
__device__ float shadow_ray(const RayArgs& A, const float* start, const float* nrm, float acc_alpha, float trans) {
    if (trans < 0.1f || acc_alpha < 0.2f) return 1.0f;
    const uint32_t steps = max(24u, (uint32_t)(64.0f * trans));
    const float ll = sqrtf((A.light[0] * A.light[0] + A.light[1] * A.light[1]) + A.light[2] * A.light[2]);
    float dir[3], rs[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        dir[a] = A.light[a] / ll;
        rs[a] = start[a] + nrm[a] * 0.6f;
    }
    float t = 0.5f, occ = 0.0f;
    for (uint32_t i = 0; i < steps; ++i) {
        float p[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) p[a] = rs[a] + dir[a] * t;
        if (p[0] < 0.0f || p[1] < 0.0f || p[2] < 0.0f || p[0] >= A.grid || p[1] >= A.grid || p[2] >= A.grid) break;
        occ = occ + sample_alpha(A, (int)floorf(p[0]), (int)floorf(p[1]), (int)floorf(p[2])) * 1.0f;
        if (occ > 0.8f) return 0.0f;
        t = t + 1.0f;
    }
    const float vis = expf(-occ * 1.5f);
    return 1.0f * (1.0f - trans) + vis * trans;  // mix(1, vis, trans)
}

template <bool RGBA>
__global__ void __launch_bounds__(128) render_kernel(RayArgs A) {
    const uint32_t px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y * blockDim.y + threadIdx.y;
    if (px >= A.W || py >= A.H) return;
    const size_t pix = (size_t)py * A.W + px;
    uint64_t out_lab = 0;
    float out_t = INFINITY;
    float hc[4] = {0.0f, 0.0f, 0.0f, 0.0f};  // RGBA mode: front-to-back accumulated colour
    const float fw = (float)A.W, fh = (float)A.H, aspect = fw / fh;
    const float ndc_x = (((float)px + 0.5f) / fw) * 2.0f - 1.0f;
    const float ndc_y = 1.0f - (((float)py + 0.5f) / fh) * 2.0f;
    float d[3], inv[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float r = ((A.right[a] * ndc_x) * aspect) * A.thf;
        float u = (A.up[a] * ndc_y) * A.thf;
        d[a] = (A.fwd[a] + r) + u;
    }
    const float len = sqrtf((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]);
#pragma unroll
    for (int a = 0; a < 3; ++a) d[a] = d[a] / len;
#pragma unroll
    for (int a = 0; a < 3; ++a) inv[a] = fsgn(d[a]) / fmaxf(fabsf(d[a]), 1e-6f);
    // intersectVolume (:457-471)
    float t0[3], t1[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        t0[a] = (0.0f - A.o[a]) * inv[a];
        t1[a] = (A.grid - A.o[a]) * inv[a];
    }
    const float tmin = fmaxf(fmaxf(fminf(t0[0], t1[0]), fminf(t0[1], t1[1])), fminf(t0[2], t1[2]));
    const float tmax = fminf(fminf(fmaxf(t0[0], t1[0]), fmaxf(t0[1], t1[1])), fmaxf(t0[2], t1[2]));
    if (!(tmax < 0.0f || tmin > tmax)) {
        const float tEnter = fmaxf(tmin, 0.0f), tExit = tmax;
        const int bs = A.bs;
        // initBrickDDA (:519-545)
        int brick[3], step[3];
        float btMax[3], btDelta[3];
        {
            const float ts = tEnter + fmaxf(tEnter * 1e-6f, 1e-5f);
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                float pos = A.o[a] + d[a] * ts;
                brick[a] = (int)floorf(pos) / bs;
                step[a] = isgn(d[a]);
                float bf = (float)brick[a] * (float)bs;
                float nb = d[a] > 0.0f ? bf + (float)bs : bf;
                btMax[a] = (nb - A.o[a]) * inv[a];
                btDelta[a] = fabsf((float)bs * inv[a]);
            }
        }
        int be[3], bx[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            be[a] = (int)(A.o[a] + d[a] * tEnter) / bs;
            bx[a] = (int)(A.o[a] + d[a] * tExit) / bs;
        }
        const uint32_t maxCross = (uint32_t)(abs(bx[0] - be[0]) + abs(bx[1] - be[1]) + abs(bx[2] - be[2])) + 6u;
        float brickEntryT = tEnter;
        bool done = false;
        for (uint32_t it = 0; it < maxCross && !done; ++it) {
            if (brick[0] < 0 || brick[1] < 0 || brick[2] < 0 || brick[0] >= A.num_bricks || brick[1] >= A.num_bricks ||
                brick[2] >= A.num_bricks)
                break;
            const uint32_t m = mort((uint32_t)brick[0], (uint32_t)brick[1], (uint32_t)brick[2]);
            bool skip = m >= A.n_slots;
            csv_brick_slot sl{0, 0, 0};
            if (!skip) {
                sl = A.slots[m];
                if (sl.flags & CSV_SLOT_EMPTY) {
                    skip = true;
                } else {
                    // a non-empty brick entered by the ray (rayTrace.wgsl:684-686); the value is a
                    // property of the slot, so concurrent writers store the same word
                    const uint32_t rq = (sl.flags & CSV_SLOT_MISSING) ? 3u : 1u;
                    if (A.requests && A.requests[m] != rq) A.requests[m] = rq;
                    skip = (sl.flags & CSV_SLOT_MISSING) != 0;
                }
            }
            if (!skip) {
                int bmin[3];
#pragma unroll
                for (int a = 0; a < 3; ++a) bmin[a] = brick[a] * bs;
                const float tEnterBrick = fmaxf(brickEntryT, tEnter);
                float tExitBrick = fminf(fminf(btMax[0], btMax[1]), btMax[2]);
                const float exitBias = fmaxf(tExitBrick * 1e-6f, 1e-5f);
                tExitBrick = fmaxf(tEnterBrick, tExitBrick - exitBias);
                // initDDA (:473-499)
                int vox[3];
                float vtMax[3], vtDelta[3];
                const float ts = tEnterBrick + fmaxf(tEnterBrick * 1e-6f, 1e-5f);
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    float pos = A.o[a] + d[a] * ts;
                    vox[a] = (int)floorf(pos);
                    float nb = d[a] > 0.0f ? (float)(vox[a] + 1) : (float)vox[a];
                    vtMax[a] = (nb - A.o[a]) * inv[a];
                    vtDelta[a] = fabsf(inv[a]);
                }
                const int lodSize = 1 << sl.lod;
                const int stride = bs / lodSize;
#pragma unroll
                for (int a = 0; a < 3; ++a) vox[a] -= bmin[a];
                if (stride > 1) {  // LOD quantisation (:706-731)
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        int lv = (vox[a] / stride) * stride;
                        vox[a] = clampi(lv, 0, bs - 1);
                        vtDelta[a] = fabsf(inv[a]) * (float)stride;
                        float lw = (float)bmin[a] + (float)vox[a];
                        float nb = d[a] > 0.0f ? lw + (float)stride : lw;
                        vtMax[a] = (nb - A.o[a]) * inv[a];
                    }
                } else {
#pragma unroll
                    for (int a = 0; a < 3; ++a) vox[a] = clampi(vox[a], 0, bs - 1);
                }
                int le[3], lx[3];
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    float ve = A.o[a] + d[a] * tEnterBrick, vx = A.o[a] + d[a] * tExitBrick;
                    le[a] = (int)floorf((ve - (float)bmin[a]) / (float)stride);
                    lx[a] = (int)ceilf((vx - (float)bmin[a]) / (float)stride);
                }
                const uint32_t maxSteps =
                    (uint32_t)(abs(lx[0] - le[0]) + abs(lx[1] - le[1]) + abs(lx[2] - le[2])) + 128u;
                const int sh = A.lb - (int)sl.lod;
                float tcell = tEnterBrick;
                for (uint32_t vi = 0; vi < maxSteps; ++vi) {
                    if (RGBA && vox[0] >= 0 && vox[1] >= 0 && vox[2] >= 0 && vox[0] < bs && vox[1] < bs &&
                        vox[2] < bs) {
                        const uint32_t rgba = slot_rgba(A, sl, vox[0], vox[1], vox[2]);
                        float c[4];
#pragma unroll
                        for (int k = 0; k < 4; ++k) c[k] = chan(rgba, k);
                        if (c[3] > 0.05f) {
                            float sc[3] = {c[0], c[1], c[2]};
                            if (c[3] > 0.35f) {  // shading (:803-826)
                                float wp[3];
                                int vp[3];
#pragma unroll
                                for (int a = 0; a < 3; ++a) {
                                    wp[a] = (float)(bmin[a] + vox[a]) + 0.5f;
                                    vp[a] = (int)wp[a];
                                }
                                float gr[3];  // computeGradientLOD (:428-455)
#pragma unroll
                                for (int a = 0; a < 3; ++a) {
                                    int qp[3] = {vp[0], vp[1], vp[2]}, qn[3] = {vp[0], vp[1], vp[2]};
                                    qp[a] += stride;
                                    qn[a] -= stride;
                                    float ap = sample_alpha_in(A, sl, bmin, qp[0], qp[1], qp[2]);
                                    float an = sample_alpha_in(A, sl, bmin, qn[0], qn[1], qn[2]);
                                    ap = ap > 0.05f ? ap : c[3];
                                    an = an > 0.05f ? an : c[3];
                                    gr[a] = (ap - an) * 0.5f;
                                }
                                const float gl = sqrtf((gr[0] * gr[0] + gr[1] * gr[1]) + gr[2] * gr[2]);
                                float nrm[3];
#pragma unroll
                                for (int a = 0; a < 3; ++a) nrm[a] = -gr[a] / fmaxf(gl, 0.001f);
                                float shadow = 1.0f;
                                if (c[3] > 0.4f) shadow = shadow_ray(A, wp, nrm, hc[3], 1.0f - hc[3]);
                                const float ll = sqrtf((A.light[0] * A.light[0] + A.light[1] * A.light[1]) +
                                                       A.light[2] * A.light[2]);
                                const float ld = fmaxf(0.0f, (nrm[0] * (A.light[0] / ll) + nrm[1] * (A.light[1] / ll)) +
                                                                 nrm[2] * (A.light[2] / ll));
                                const float ds = A.diffuse * shadow;
                                const float min_amb = ld > 0.01f ? 0.3f : 0.1f;
                                const float sf = fminf(fmaxf(A.ambient + ld * ds, min_amb), 1.0f);
                                const float lum = (c[0] * 0.299f + c[1] * 0.587f) + c[2] * 0.114f;
                                const float smix = fminf(fmaxf(1.0f - shadow, 0.0f), 1.0f) * 0.5f;
#pragma unroll
                                for (int k = 0; k < 3; ++k) {
                                    const float gray = lum * 0.8f + c[k] * 0.2f;
                                    sc[k] = (c[k] * (1.0f - smix) + gray * smix) * sf;  // mix(c, gray, smix)
                                }
                            }
                            // compositing (:828-836): opacity corrected for the LOD stride
                            const float ca = fminf(fmaxf(1.0f - powf(1.0f - c[3], (float)stride), 0.0f), 1.0f);
                            const float sa = ca * (1.0f - hc[3]);
#pragma unroll
                            for (int k = 0; k < 3; ++k) hc[k] = hc[k] + sc[k] * sa;
                            hc[3] = hc[3] + sa;
                            if (hc[3] > 0.95f) {
                                done = true;
                                break;
                            }
                        }
                    } else if (!RGBA && vox[0] >= 0 && vox[1] >= 0 && vox[2] >= 0 && vox[0] < bs && vox[1] < bs &&
                               vox[2] < bs) {
                        uint64_t lab;
                        if (sl.lod == 0) lab = __ldg(A.labels + sl.offset);
                        else
                            lab = __ldg(A.labels + sl.offset +
                                        mort((uint32_t)vox[0] >> sh, (uint32_t)vox[1] >> sh, (uint32_t)vox[2] >> sh));
                        if (lab != 0 && !(A.n_hidden && is_hidden(A, lab))) {
                            out_lab = lab;
                            out_t = tcell;
                            done = true;
                            break;
                        }
                    }
                    float t;  // advanceDDA (:501-517)
                    if (vtMax[0] < vtMax[1] && vtMax[0] < vtMax[2]) {
                        t = vtMax[0]; vtMax[0] += vtDelta[0]; vox[0] += step[0];
                    } else if (vtMax[1] < vtMax[2]) {
                        t = vtMax[1]; vtMax[1] += vtDelta[1]; vox[1] += step[1];
                    } else {
                        t = vtMax[2]; vtMax[2] += vtDelta[2]; vox[2] += step[2];
                    }
                    tcell = t;
                    if (t > tExitBrick) break;
                }
                if (done) break;
            }
            float t;  // advanceBrickDDA (:547-563)
            if (btMax[0] < btMax[1] && btMax[0] < btMax[2]) {
                t = btMax[0]; btMax[0] += btDelta[0]; brick[0] += step[0];
            } else if (btMax[1] < btMax[2]) {
                t = btMax[1]; btMax[1] += btDelta[1]; brick[1] += step[1];
            } else {
                t = btMax[2]; btMax[2] += btDelta[2]; brick[2] += step[2];
            }
            brickEntryT = t + fmaxf(t * 1e-6f, 1e-5f);
            if (t > tExit) break;
        }
    }
    if (RGBA) {
        A.out_rgba[pix] = (uint32_t)(hc[0] * 255.0f) | ((uint32_t)(hc[1] * 255.0f) << 8) |
                          ((uint32_t)(hc[2] * 255.0f) << 16) | ((uint32_t)(hc[3] * 255.0f) << 24);
    } else {
        A.out_label[pix] = out_lab;
        A.out_depth[pix] = out_t;
    }
}

cudaError_t launch_render(const csv_camera& cam, uint32_t W, uint32_t H, float grid, uint32_t bs, uint32_t bpa,
                          const csv_brick_slot* slots, uint64_t n_slots, const uint64_t* labels, const uint64_t* hidden,
                          uint32_t n_hidden, uint64_t* out_label, float* out_depth, uint32_t* requests,
                          cudaStream_t st) {
    RayArgs A;
    for (int a = 0; a < 3; ++a) {
        A.o[a] = cam.position[a];
        A.fwd[a] = cam.forward[a];
        A.right[a] = cam.right[a];
        A.up[a] = cam.up[a];
    }
    A.thf = cam.tan_half_fov;
    A.W = W;
    A.H = H;
    A.grid = grid;
    A.bs = (int)bs;
    int lb = 0;
    while ((1u << lb) < bs) ++lb;
    A.lb = lb;
    A.num_bricks = bpa > 1 ? (int)bpa : 1;
    A.slots = slots;
    A.n_slots = n_slots;
    A.labels = labels;
    A.hidden = hidden;
    A.n_hidden = hidden ? n_hidden : 0;
    A.out_label = out_label;
    A.out_depth = out_depth;
    A.requests = requests;
    A.tf_keys = nullptr;
    A.tf_rgba = nullptr;
    A.n_tf = 0;
    A.out_rgba = nullptr;
    dim3 block(16, 8), grid2((W + 15) / 16, (H + 7) / 8);
    render_kernel<false><<<grid2, block, 0, st>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_render_rgba(const csv_camera& cam, uint32_t W, uint32_t H, float grid, uint32_t bs, uint32_t bpa,
                               const csv_brick_slot* slots, uint64_t n_slots, const uint64_t* labels,
                               const uint64_t* tf_keys, const uint32_t* tf_rgba, uint32_t n_tf, const float* light,
                               float ambient, float diffuse, uint32_t* out_rgba, uint32_t* requests, cudaStream_t st) {
    RayArgs A;
    for (int a = 0; a < 3; ++a) {
        A.o[a] = cam.position[a];
        A.fwd[a] = cam.forward[a];
        A.right[a] = cam.right[a];
        A.up[a] = cam.up[a];
        A.light[a] = light[a];
    }
    A.thf = cam.tan_half_fov;
    A.W = W;
    A.H = H;
    A.grid = grid;
    A.bs = (int)bs;
    int lb = 0;
    while ((1u << lb) < bs) ++lb;
    A.lb = lb;
    A.num_bricks = bpa > 1 ? (int)bpa : 1;
    A.slots = slots;
    A.n_slots = n_slots;
    A.labels = labels;
    A.hidden = nullptr;
    A.n_hidden = 0;
    A.out_label = nullptr;
    A.out_depth = nullptr;
    A.requests = requests;
    A.tf_keys = tf_keys;
    A.tf_rgba = tf_rgba;
    A.n_tf = tf_keys ? n_tf : 0;
    A.ambient = ambient;
    A.diffuse = diffuse;
    A.out_rgba = out_rgba;
    dim3 block(16, 8), grid2((W + 15) / 16, (H + 7) / 8);
    render_kernel<true><<<grid2, block, 0, st>>>(A);
    return cudaGetLastError();
}

}  // namespace csv
