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

__global__ void __launch_bounds__(128) render_kernel(RayArgs A) {
    const uint32_t px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y * blockDim.y + threadIdx.y;
    if (px >= A.W || py >= A.H) return;
    const size_t pix = (size_t)py * A.W + px;
    uint64_t out_lab = 0;
    float out_t = INFINITY;
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
                    if (vox[0] >= 0 && vox[1] >= 0 && vox[2] >= 0 && vox[0] < bs && vox[1] < bs && vox[2] < bs) {
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
    A.out_label[pix] = out_lab;
    A.out_depth[pix] = out_t;
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
    dim3 block(16, 8), grid2((W + 15) / 16, (H + 7) / 8);
    render_kernel<<<grid2, block, 0, st>>>(A);
    return cudaGetLastError();
}

}  // namespace csv
