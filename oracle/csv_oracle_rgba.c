/* csv_oracle_rgba.c -- CPU restatement of the viewer's colour path.  Test
 * infrastructure only: the checker for csv_transfer_function and
 * csv_render_rgba, never the thing measured or shipped.
 *
 *   or_transfer_function  buildTransferFunctionBuffers + hslToRgb
 *                         (web/scripts/webgpuSetup.js:389-465, 490-515),
 *                         hidden labels transparent (:826-834)
 *   or_label_rgba         hashLabel (web/shaders/decode.wgsl:135-172)
 *   or_render_rgba_rows   rayTrace (web/shaders/rayTrace.wgsl:565-906) with its
 *                         colours: getVoxelColor (:159-198), sampleAlpha
 *                         (:272-299), sampleAlphaInBrick (:301-318),
 *                         traceShadowRay (:329-397), computeGradientLOD
 *                         (:428-455), shading and compositing (:794-837),
 *                         RGBA8 output (:897-905)
 *
 * The traversal is or_render_rows' (csv_oracle.c).  Float operations are
 * written one rounding each in the order the device code uses (compiled with
 * -ffp-contract=off); powf and expf are the C library's.  Where the shader has
 * no defined outcome: a LOD-0 brick is coloured by the transfer function of
 * its label (the shader reads the label's low bytes as a colour, :165-177),
 * and bricks that are not resident sample as alpha 0. */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "csv_oracle.h"

static double js_round(double x) { return floor(x + 0.5); } /* Math.round */

void or_transfer_function(const uint64_t* labels, uint32_t n, const uint64_t* hidden, uint32_t n_hidden,
                          uint32_t* rgba) {
    for (uint32_t i = 0; i < n; ++i) {
        const double h = fmod((double)i * 137.5, 360.0);
        const double sat = 0.55 + (double)(i % 3) * 0.08, lig = 0.35 + (double)(i % 4) * 0.05;
        const double op = 0.25 + (double)(i % 5) * 0.08;
        const double c = (1 - fabs(2 * lig - 1)) * sat;
        const double x = c * (1 - fabs(fmod(h / 60, 2) - 1));
        const double m = lig - c / 2;
        double r, g, b;
        if (h < 60) { r = c; g = x; b = 0; }
        else if (h < 120) { r = x; g = c; b = 0; }
        else if (h < 180) { r = 0; g = c; b = x; }
        else if (h < 240) { r = 0; g = x; b = c; }
        else if (h < 300) { r = x; g = 0; b = c; }
        else { r = c; g = 0; b = x; }
        double R = floor(js_round((r + m) * 255) * 0.92), G = floor(js_round((g + m) * 255) * 0.92),
               B = floor(js_round((b + m) * 255) * 0.92);
        if (R > 255) R = 255;
        if (G > 255) G = 255;
        if (B > 255) B = 255;
        const uint32_t A = (uint32_t)floor(op * 255);
        int hid = 0;
        for (uint32_t k = 0; k < n_hidden && !hid; ++k) hid = hidden[k] == labels[i];
        rgba[i] = hid ? 0u : ((uint32_t)R | ((uint32_t)G << 8) | ((uint32_t)B << 16) | (A << 24));
    }
}

typedef struct {
    float grid;
    int bs, lb, nbpa;
    const or_slot* slots;
    uint64_t n_slots;
    const uint64_t* labels;
    const uint64_t* keys;
    const uint32_t* cols;
    uint32_t n_tf;
    float light[3], ambient, diffuse;
} rgba_ctx;

uint32_t or_label_rgba(uint64_t v, const uint64_t* keys, const uint32_t* cols, uint32_t n_tf) {
    if (v == 0) return 0u;
    for (uint32_t i = 0; i < n_tf; ++i) /* the shader's linear search */
        if (keys[i] == v) return cols[i];
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

static float chan(uint32_t rgba, int k) { return (float)((rgba >> (8 * k)) & 0xFFu) / 255.0f; }

static uint32_t slot_rgba(const rgba_ctx* C, const or_slot* sl, int x, int y, int z) {
    uint64_t lab;
    if (sl->lod == 0) lab = C->labels[sl->offset];
    else {
        int sh = C->lb - (int)sl->lod;
        lab = C->labels[sl->offset + or_morton3((uint32_t)x >> sh, (uint32_t)y >> sh, (uint32_t)z >> sh)];
    }
    return or_label_rgba(lab, C->keys, C->cols, C->n_tf);
}

static float sample_alpha(const rgba_ctx* C, int wx, int wy, int wz) {
    const int g = (int)C->grid;
    if (wx < 0 || wy < 0 || wz < 0 || wx >= g || wy >= g || wz >= g) return 0.0f;
    const int bx = wx / C->bs, by = wy / C->bs, bz = wz / C->bs;
    if (bx >= C->nbpa || by >= C->nbpa || bz >= C->nbpa) return 0.0f;
    uint32_t m = or_morton3((uint32_t)bx, (uint32_t)by, (uint32_t)bz);
    if (m >= C->n_slots) return 0.0f;
    const or_slot* sl = &C->slots[m];
    if (sl->flags & 3u) return 0.0f; /* empty, or not resident */
    return chan(slot_rgba(C, sl, wx - bx * C->bs, wy - by * C->bs, wz - bz * C->bs), 3);
}

static float sample_alpha_in(const rgba_ctx* C, const or_slot* sl, const int* bmin, int wx, int wy, int wz) {
    const int g = (int)C->grid;
    if (wx < 0 || wy < 0 || wz < 0 || wx >= g || wy >= g || wz >= g) return 0.0f;
    int lx = wx - bmin[0], ly = wy - bmin[1], lz = wz - bmin[2];
    if (lx < 0 || ly < 0 || lz < 0 || lx >= C->bs || ly >= C->bs || lz >= C->bs) return sample_alpha(C, wx, wy, wz);
    return chan(slot_rgba(C, sl, lx, ly, lz), 3);
}

static float shadow_ray(const rgba_ctx* C, const float* start, const float* nrm, float acc_alpha, float trans) {
    if (trans < 0.1f || acc_alpha < 0.2f) return 1.0f;
    uint32_t steps = (uint32_t)(64.0f * trans);
    if (steps < 24u) steps = 24u;
    const float ll = sqrtf((C->light[0] * C->light[0] + C->light[1] * C->light[1]) + C->light[2] * C->light[2]);
    float dir[3], rs[3];
    for (int a = 0; a < 3; ++a) {
        dir[a] = C->light[a] / ll;
        rs[a] = start[a] + nrm[a] * 0.6f;
    }
    float t = 0.5f, occ = 0.0f;
    for (uint32_t i = 0; i < steps; ++i) {
        float p[3];
        for (int a = 0; a < 3; ++a) p[a] = rs[a] + dir[a] * t;
        if (p[0] < 0.0f || p[1] < 0.0f || p[2] < 0.0f || p[0] >= C->grid || p[1] >= C->grid || p[2] >= C->grid) break;
        occ = occ + sample_alpha(C, (int)floorf(p[0]), (int)floorf(p[1]), (int)floorf(p[2])) * 1.0f;
        if (occ > 0.8f) return 0.0f;
        t = t + 1.0f;
    }
    const float vis = expf(-occ * 1.5f);
    return 1.0f * (1.0f - trans) + vis * trans;
}

static float fsgn2(float x) { return x > 0.f ? 1.f : (x < 0.f ? -1.f : 0.f); }
static int isgn2(float x) { return (x > 0.f ? 1 : 0) + (x < 0.f ? -1 : 0); }
static int clampi2(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

void or_render_rgba_rows(const float* cam, uint32_t W, uint32_t H, uint32_t y0, uint32_t ystep, float grid, uint32_t bsz,
                         uint32_t bpa, const or_slot* slots, uint64_t n_slots, const uint64_t* labels,
                         const uint64_t* keys, const uint32_t* cols, uint32_t n_tf, const float* lighting,
                         uint32_t* out_rgba) {
    rgba_ctx C;
    C.grid = grid;
    C.bs = (int)bsz;
    C.lb = 0;
    while ((1 << C.lb) < C.bs) ++C.lb;
    C.nbpa = (int)bpa > 1 ? (int)bpa : 1;
    C.slots = slots;
    C.n_slots = n_slots;
    C.labels = labels;
    C.keys = keys;
    C.cols = cols;
    C.n_tf = n_tf;
    for (int a = 0; a < 3; ++a) C.light[a] = lighting[a];
    C.ambient = lighting[3];
    C.diffuse = lighting[4];
    const float o[3] = {cam[0], cam[1], cam[2]};
    const float thf = cam[3];
    const float fw = (float)W, fh = (float)H, aspect = fw / fh;
    const int bs = C.bs;
    if (ystep == 0) ystep = 1;
    for (uint32_t py = y0; py < H; py += ystep)
        for (uint32_t px = 0; px < W; ++px) {
            const size_t pix = (size_t)py * W + px;
            float hc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            float ndc_x = (((float)px + 0.5f) / fw) * 2.0f - 1.0f;
            float ndc_y = 1.0f - (((float)py + 0.5f) / fh) * 2.0f;
            float d[3], inv[3];
            for (int a = 0; a < 3; ++a) {
                float r = ((cam[8 + a] * ndc_x) * aspect) * thf;
                float u = (cam[12 + a] * ndc_y) * thf;
                d[a] = (cam[4 + a] + r) + u;
            }
            float len = sqrtf((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]);
            for (int a = 0; a < 3; ++a) d[a] = d[a] / len;
            for (int a = 0; a < 3; ++a) inv[a] = fsgn2(d[a]) / fmaxf(fabsf(d[a]), 1e-6f);
            float t0[3], t1[3];
            for (int a = 0; a < 3; ++a) {
                t0[a] = (0.0f - o[a]) * inv[a];
                t1[a] = (grid - o[a]) * inv[a];
            }
            float tmin = fmaxf(fmaxf(fminf(t0[0], t1[0]), fminf(t0[1], t1[1])), fminf(t0[2], t1[2]));
            float tmax = fminf(fminf(fmaxf(t0[0], t1[0]), fmaxf(t0[1], t1[1])), fmaxf(t0[2], t1[2]));
            if (!(tmax < 0.0f || tmin > tmax)) {
                const float tEnter = fmaxf(tmin, 0.0f), tExit = tmax;
                int brick[3], step[3];
                float btMax[3], btDelta[3];
                {
                    float ts = tEnter + fmaxf(tEnter * 1e-6f, 1e-5f);
                    for (int a = 0; a < 3; ++a) {
                        float pos = o[a] + d[a] * ts;
                        brick[a] = (int)floorf(pos) / bs;
                        step[a] = isgn2(d[a]);
                        float bf = (float)brick[a] * (float)bs;
                        float nb = d[a] > 0.0f ? bf + (float)bs : bf;
                        btMax[a] = (nb - o[a]) * inv[a];
                        btDelta[a] = fabsf((float)bs * inv[a]);
                    }
                }
                int be[3], bx[3];
                for (int a = 0; a < 3; ++a) {
                    be[a] = (int)(o[a] + d[a] * tEnter) / bs;
                    bx[a] = (int)(o[a] + d[a] * tExit) / bs;
                }
                uint32_t maxCross = (uint32_t)(abs(bx[0] - be[0]) + abs(bx[1] - be[1]) + abs(bx[2] - be[2])) + 6u;
                float brickEntryT = tEnter;
                int done = 0;
                for (uint32_t it = 0; it < maxCross && !done; ++it) {
                    if (brick[0] < 0 || brick[1] < 0 || brick[2] < 0 || brick[0] >= C.nbpa || brick[1] >= C.nbpa ||
                        brick[2] >= C.nbpa)
                        break;
                    uint32_t m = or_morton3((uint32_t)brick[0], (uint32_t)brick[1], (uint32_t)brick[2]);
                    int skip = m >= n_slots;
                    or_slot sl = {0, 0, 0};
                    if (!skip) {
                        sl = slots[m];
                        skip = (sl.flags & 3u) != 0;
                    }
                    if (!skip) {
                        int bmin[3];
                        for (int a = 0; a < 3; ++a) bmin[a] = brick[a] * bs;
                        float tEnterBrick = fmaxf(brickEntryT, tEnter);
                        float tExitBrick = fminf(fminf(btMax[0], btMax[1]), btMax[2]);
                        float exitBias = fmaxf(tExitBrick * 1e-6f, 1e-5f);
                        tExitBrick = fmaxf(tEnterBrick, tExitBrick - exitBias);
                        int vox[3];
                        float vtMax[3], vtDelta[3];
                        float ts = tEnterBrick + fmaxf(tEnterBrick * 1e-6f, 1e-5f);
                        for (int a = 0; a < 3; ++a) {
                            float pos = o[a] + d[a] * ts;
                            vox[a] = (int)floorf(pos);
                            float nb = d[a] > 0.0f ? (float)(vox[a] + 1) : (float)vox[a];
                            vtMax[a] = (nb - o[a]) * inv[a];
                            vtDelta[a] = fabsf(inv[a]);
                        }
                        const int lodSize = 1 << sl.lod;
                        const int stride = bs / lodSize;
                        for (int a = 0; a < 3; ++a) vox[a] -= bmin[a];
                        if (stride > 1) {
                            for (int a = 0; a < 3; ++a) {
                                int lv = (vox[a] / stride) * stride;
                                vox[a] = clampi2(lv, 0, bs - 1);
                                vtDelta[a] = fabsf(inv[a]) * (float)stride;
                                float lw = (float)bmin[a] + (float)vox[a];
                                float nb = d[a] > 0.0f ? lw + (float)stride : lw;
                                vtMax[a] = (nb - o[a]) * inv[a];
                            }
                        } else {
                            for (int a = 0; a < 3; ++a) vox[a] = clampi2(vox[a], 0, bs - 1);
                        }
                        int le[3], lx[3];
                        for (int a = 0; a < 3; ++a) {
                            float ve = o[a] + d[a] * tEnterBrick, vx = o[a] + d[a] * tExitBrick;
                            le[a] = (int)floorf((ve - (float)bmin[a]) / (float)stride);
                            lx[a] = (int)ceilf((vx - (float)bmin[a]) / (float)stride);
                        }
                        uint32_t maxSteps =
                            (uint32_t)(abs(lx[0] - le[0]) + abs(lx[1] - le[1]) + abs(lx[2] - le[2])) + 128u;
                        for (uint32_t vi = 0; vi < maxSteps; ++vi) {
                            if (vox[0] >= 0 && vox[1] >= 0 && vox[2] >= 0 && vox[0] < bs && vox[1] < bs && vox[2] < bs) {
                                const uint32_t rgba = slot_rgba(&C, &sl, vox[0], vox[1], vox[2]);
                                float c[4];
                                for (int k = 0; k < 4; ++k) c[k] = chan(rgba, k);
                                if (c[3] > 0.05f) {
                                    float sc[3] = {c[0], c[1], c[2]};
                                    if (c[3] > 0.35f) {
                                        float wp[3];
                                        int vp[3];
                                        for (int a = 0; a < 3; ++a) {
                                            wp[a] = (float)(bmin[a] + vox[a]) + 0.5f;
                                            vp[a] = (int)wp[a];
                                        }
                                        float gr[3];
                                        for (int a = 0; a < 3; ++a) {
                                            int qp[3] = {vp[0], vp[1], vp[2]}, qn[3] = {vp[0], vp[1], vp[2]};
                                            qp[a] += stride;
                                            qn[a] -= stride;
                                            float ap = sample_alpha_in(&C, &sl, bmin, qp[0], qp[1], qp[2]);
                                            float an = sample_alpha_in(&C, &sl, bmin, qn[0], qn[1], qn[2]);
                                            ap = ap > 0.05f ? ap : c[3];
                                            an = an > 0.05f ? an : c[3];
                                            gr[a] = (ap - an) * 0.5f;
                                        }
                                        const float gl = sqrtf((gr[0] * gr[0] + gr[1] * gr[1]) + gr[2] * gr[2]);
                                        float nrm[3];
                                        for (int a = 0; a < 3; ++a) nrm[a] = -gr[a] / fmaxf(gl, 0.001f);
                                        float shadow = 1.0f;
                                        if (c[3] > 0.4f) shadow = shadow_ray(&C, wp, nrm, hc[3], 1.0f - hc[3]);
                                        const float ll = sqrtf((C.light[0] * C.light[0] + C.light[1] * C.light[1]) +
                                                               C.light[2] * C.light[2]);
                                        const float ld = fmaxf(0.0f, (nrm[0] * (C.light[0] / ll) +
                                                                      nrm[1] * (C.light[1] / ll)) +
                                                                         nrm[2] * (C.light[2] / ll));
                                        const float ds = C.diffuse * shadow;
                                        const float min_amb = ld > 0.01f ? 0.3f : 0.1f;
                                        const float sf = fminf(fmaxf(C.ambient + ld * ds, min_amb), 1.0f);
                                        const float lum = (c[0] * 0.299f + c[1] * 0.587f) + c[2] * 0.114f;
                                        const float smix = fminf(fmaxf(1.0f - shadow, 0.0f), 1.0f) * 0.5f;
                                        for (int k = 0; k < 3; ++k) {
                                            const float gray = lum * 0.8f + c[k] * 0.2f;
                                            sc[k] = (c[k] * (1.0f - smix) + gray * smix) * sf;
                                        }
                                    }
                                    const float ca =
                                        fminf(fmaxf(1.0f - powf(1.0f - c[3], (float)stride), 0.0f), 1.0f);
                                    const float sa = ca * (1.0f - hc[3]);
                                    for (int k = 0; k < 3; ++k) hc[k] = hc[k] + sc[k] * sa;
                                    hc[3] = hc[3] + sa;
                                    if (hc[3] > 0.95f) {
                                        done = 1;
                                        break;
                                    }
                                }
                            }
                            float t;
                            if (vtMax[0] < vtMax[1] && vtMax[0] < vtMax[2]) {
                                t = vtMax[0]; vtMax[0] += vtDelta[0]; vox[0] += step[0];
                            } else if (vtMax[1] < vtMax[2]) {
                                t = vtMax[1]; vtMax[1] += vtDelta[1]; vox[1] += step[1];
                            } else {
                                t = vtMax[2]; vtMax[2] += vtDelta[2]; vox[2] += step[2];
                            }
                            if (t > tExitBrick) break;
                        }
                        if (done) break;
                    }
                    float t;
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
            out_rgba[pix] = (uint32_t)(hc[0] * 255.0f) | ((uint32_t)(hc[1] * 255.0f) << 8) |
                            ((uint32_t)(hc[2] * 255.0f) << 16) | ((uint32_t)(hc[3] * 255.0f) << 24);
        }
}
