/* csv_oracle_serve.c -- CPU restatement of the viewer's frame loop: plan,
 * cache policy, decode of the admitted bricks, render.  Test infrastructure
 * only: it is the checker the device server is compared with, slot table for
 * slot table and pixel for pixel.
 *
 * Follows, per frame (renderLoop.js:208-340 with LOD_UPDATE_INTERVAL 1):
 *   - the camera-moved test (culling.js:22-56): re-plan only when a camera
 *     moved more than 0.5 units or turned more than 0.05 rad since the last plan;
 *   - the LOD of every brick (camera.js:103-137, screen size min(W, H),
 *     renderLoop.js:374) and the cone test (culling.js:87-153), with the
 *     transfer-function test (culling.js:162-171) as a per-brick flag;
 *   - the cache (cacheManager.js:10-246, cacheProcessing.js:99-232): per-LOD
 *     free stacks of blocks of 8^lod labels, a bump pointer, eviction of the
 *     bricks the frame does not need, a rebuild when an allocation fails;
 *   - the decode of the newly admitted (brick, LOD) pairs and the label/depth
 *     render of every view (or_render_rows).
 *
 * Where the reference leaves an order or a corner case open, this file fixes
 * it, and the device server follows the same rules:
 *   - frees are pushed in brick (file) order; allocations are served LOD by
 *     LOD (coarse first), in brick order within a LOD, each popping its LOD's
 *     stack (last pushed first) and taking fresh space from the bump pointer
 *     once the stack is empty;
 *   - when the frame's fresh space does not fit, the cache is rebuilt: every
 *     block is dropped and every needed brick is placed again, LOD by LOD
 *     (coarse first) in brick order, until the space runs out (the bricks
 *     that do not fit stay missing for this frame);
 *   - LOD-0 bricks and uniform bricks (root stop bit: the whole brick is
 *     palette[0]) take no block: their slot reads palette[0] from a table at
 *     the start of the cache (rayTrace.wgsl:167-178 reads palette[0] for LOD 0;
 *     a uniform brick decodes to palette[0] at every LOD, so the image is the
 *     one a decoded copy would give);
 *   - several views in one step (sessions served together) need a brick when
 *     any of them does, at the finest LOD any of them asks for;
 *   - the cone's margin sin(atan2(r, d)) is evaluated as r / sqrt(r^2 + d^2),
 *     the same number for d > 0 up to rounding; the half-angle is fov/2
 *     (cone 0, the reference) or the half-diagonal of the screen (cone 1), and
 *     bricks whose centre is closer than twice their radius are always kept.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "csv_oracle.h"

#define OR_NONE 0xFFu
#define OR_MAXV 8

struct or_server {
    uint32_t nb, b, max_lod, bpa, W, H, cone, n_hidden;
    double fov, focal, cos_half, radius, half;
    uint32_t freq[16], cum[16];
    /* per brick */
    uint32_t* id;
    uint8_t* has;      /* a palette entry is neither 0 nor hidden */
    uint8_t* uni;      /* uniform brick */
    uint64_t* pal0;    /* palette[0] */
    const uint8_t** enc;
    uint32_t* E;
    uint32_t* nsym;
    const uint64_t** pal;
    uint32_t* P;
    uint8_t* res_lod;
    uint64_t* res_off;
    /* cache */
    uint64_t pal_region, cap, bump;
    uint64_t* cache;
    uint64_t* stack[OR_MAXV]; /* per LOD, nb entries */
    uint32_t top[OR_MAXV];
    or_slot* slots;
    uint64_t n_slots;
    uint64_t* hidden;
    /* last plan */
    uint32_t n_last;
    uint32_t last_sess[OR_MAXV];
    double last_view[OR_MAXV][6];
    int planned_once;
};

static uint32_t rd32(const uint8_t* p) {
    uint32_t v;
    memcpy(&v, p, 4);
    return v;
}

/* camera.js:61-77: orthonormal basis in double, then float32. */
void or_camera_uniform(const double* pos, const double* dir, double fov, float* out) {
    double f[3], r[3], u[3], wu[3];
    double n = sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
    if (n == 0.0) n = 1.0;
    for (int a = 0; a < 3; ++a) f[a] = dir[a] / n;
    if (fabs(f[1]) > 0.999) {
        wu[0] = 1.0; wu[1] = 0.0; wu[2] = 0.0;
    } else {
        wu[0] = 0.0; wu[1] = 1.0; wu[2] = 0.0;
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
    const double thf = tan(fov * 0.5);
    const double v[16] = {pos[0], pos[1], pos[2], thf, f[0], f[1], f[2], 0.0,
                          r[0],   r[1],   r[2],   0.0, u[0], u[1], u[2], 0.0};
    for (int i = 0; i < 16; ++i) out[i] = (float)v[i];
}

/* Planning constants shared with the device server (host side there too). */
void or_serve_constants(uint32_t W, uint32_t H, double fov, uint32_t cone, uint32_t b, double* focal,
                        double* cos_half, double* radius) {
    const double screen = (double)(W < H ? W : H);
    *focal = (screen / 2.0) / tan(fov / 2.0);              /* camera.js:114 */
    if (cone == 0) {
        *cos_half = cos(fov / 2.0);                         /* culling.js:132 */
    } else {
        const double a = (double)W / (double)H;
        *cos_half = cos(atan(tan(fov / 2.0) * sqrt(a * a + 1.0)));
    }
    *radius = sqrt(3.0) * ((double)b / 2.0);                /* culling.js:128 */
}

/* LOD (camera.js:103-137) and cone (culling.js:87-153) of one brick for one view. */
static int brick_in_cone(const or_server* s, const double* c, const double* v) {
    const double tx = c[0] - v[0], ty = c[1] - v[1], tz = c[2] - v[2];
    const double dist = sqrt(tx * tx + ty * ty + tz * tz);
    if (dist < 2.0 * s->radius) return 1;
    const double dot = (tx / dist) * v[3] + (ty / dist) * v[4] + (tz / dist) * v[5];
    const double margin = s->radius / sqrt(s->radius * s->radius + dist * dist);
    return !(dot < s->cos_half - margin);
}

static int has_hidden(const uint64_t* h, uint32_t n, uint64_t v) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        uint32_t mid = (lo + hi) / 2;
        if (h[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    return lo < n && h[lo] == v;
}

or_server* or_serve_new(const uint8_t* img, size_t len, uint32_t W, uint32_t H, double fov, uint32_t cone,
                        uint64_t cache_bytes, const uint64_t* hidden, uint32_t n_hidden) {
    if (!img || len < 152 || rd32(img) != 0x43534244u) return NULL;
    or_server* s = (or_server*)calloc(1, sizeof *s);
    s->nb = rd32(img + 8);
    s->b = rd32(img + 12);
    s->max_lod = 0;
    while ((1u << s->max_lod) < s->b) ++s->max_lod;
    s->W = W;
    s->H = H;
    s->fov = fov;
    s->cone = cone;
    for (int i = 0; i < 16; ++i) {
        s->freq[i] = rd32(img + 24 + 4 * i);
        s->cum[i] = rd32(img + 88 + 4 * i);
    }
    or_serve_constants(W, H, fov, cone, s->b, &s->focal, &s->cos_half, &s->radius);
    s->half = (double)s->b / 2.0;
    s->n_hidden = n_hidden;
    s->hidden = (uint64_t*)malloc(sizeof(uint64_t) * (n_hidden ? n_hidden : 1));
    if (n_hidden) memcpy(s->hidden, hidden, sizeof(uint64_t) * n_hidden);
    const uint32_t nb = s->nb;
    s->id = (uint32_t*)calloc(nb + 1, 4);
    s->has = (uint8_t*)calloc(nb + 1, 1);
    s->uni = (uint8_t*)calloc(nb + 1, 1);
    s->pal0 = (uint64_t*)calloc(nb + 1, 8);
    s->enc = (const uint8_t**)calloc(nb + 1, sizeof(void*));
    s->pal = (const uint64_t**)calloc(nb + 1, sizeof(void*));
    s->E = (uint32_t*)calloc(nb + 1, 4);
    s->nsym = (uint32_t*)calloc(nb + 1, 4);
    s->P = (uint32_t*)calloc(nb + 1, 4);
    s->res_lod = (uint8_t*)malloc(nb + 1);
    memset(s->res_lod, OR_NONE, nb + 1);
    s->res_off = (uint64_t*)calloc(nb + 1, 8);
    size_t o = 152;
    uint32_t maxc = 0;
    for (uint32_t i = 0; i < nb; ++i) {
        s->id[i] = rd32(img + o);
        s->P[i] = rd32(img + o + 4);
        s->pal[i] = (const uint64_t*)(img + o + 8);
        o += 8 + 8ull * s->P[i];
        s->E[i] = rd32(img + o);
        s->enc[i] = img + o + 4;
        o += 4 + s->E[i];
        s->nsym[i] = rd32(img + o);
        o += 4;
        uint64_t p0;
        memcpy(&p0, s->pal[i], 8);
        s->pal0[i] = p0;
        for (uint32_t k = 0; k < s->P[i]; ++k) {
            uint64_t v;
            memcpy(&v, (const uint8_t*)s->pal[i] + 8ull * k, 8);
            if (v != 0 && !has_hidden(s->hidden, n_hidden, v)) {
                s->has[i] = 1;
                break;
            }
        }
        if (s->E[i] >= 4 && s->nsym[i] >= 1) {
            uint8_t nib = 0;
            or_rans_decode(s->freq, s->cum, 4096, s->enc[i], s->E[i], 1, &nib);
            s->uni[i] = (uint8_t)((nib >> 4) & 1u);
        }
        uint32_t x, y, z;
        or_demorton3(s->id[i], &x, &y, &z);
        if (x > maxc) maxc = x;
        if (y > maxc) maxc = y;
        if (z > maxc) maxc = z;
    }
    (void)len;
    s->bpa = maxc + 1;
    uint32_t p2 = 1;
    while (p2 < s->bpa) p2 <<= 1;
    s->n_slots = (uint64_t)p2 * p2 * p2;
    s->slots = (or_slot*)calloc(s->n_slots, sizeof(or_slot));
    for (uint64_t m = 0; m < s->n_slots; ++m) s->slots[m].flags = 1u;
    const uint64_t total = cache_bytes / 8;
    s->pal_region = ((uint64_t)nb + 31) & ~31ull;
    s->cap = total > s->pal_region ? total - s->pal_region : 0;
    s->cache = (uint64_t*)calloc(total ? total : 1, 8);
    for (uint32_t i = 0; i < nb; ++i) s->cache[i] = s->pal0[i];
    for (uint32_t l = 0; l < OR_MAXV; ++l) s->stack[l] = (uint64_t*)calloc(nb + 1, 8);
    return s;
}

void or_serve_free(or_server* s) {
    if (!s) return;
    free(s->id); free(s->has); free(s->uni); free(s->pal0); free(s->enc); free(s->pal); free(s->E);
    free(s->nsym); free(s->P); free(s->res_lod); free(s->res_off); free(s->cache); free(s->slots); free(s->hidden);
    for (uint32_t l = 0; l < OR_MAXV; ++l) free(s->stack[l]);
    free(s);
}

uint64_t or_serve_n_slots(const or_server* s) { return s->n_slots; }
uint32_t or_serve_bricks_per_axis(const or_server* s) { return s->bpa; }
const or_slot* or_serve_slots(const or_server* s) { return s->slots; }
const uint64_t* or_serve_cache(const or_server* s) { return s->cache; }

/* culling.js:22-56 over the views of a step. */
static int views_moved(const or_server* s, const uint32_t* sess, const double* views, uint32_t n) {
    if (!s->planned_once || n != s->n_last) return 1;
    const double cos_rot = cos(0.05);
    for (uint32_t k = 0; k < n; ++k) {
        if (sess[k] != s->last_sess[k]) return 1;
        const double* v = views + 6 * k;
        const double* p = s->last_view[k];
        const double dx = v[0] - p[0], dy = v[1] - p[1], dz = v[2] - p[2];
        const double moved = dx * dx + dy * dy + dz * dz;
        const double dot = v[3] * p[3] + v[4] * p[4] + v[5] * p[5];
        if (moved > 0.5 * 0.5 || dot < cos_rot) return 1;
    }
    return 0;
}

static void decode_into(or_server* s, uint32_t i, uint32_t lod, uint64_t* dst) {
    const uint32_t ns = s->nsym[i];
    uint8_t* nib = (uint8_t*)calloc(ns / 2 + 2, 1);
    if (s->E[i] >= 4 && ns >= 1) or_rans_decode(s->freq, s->cum, 4096, s->enc[i], s->E[i], ns, nib);
    uint64_t* pal = (uint64_t*)malloc(8ull * s->P[i]);
    memcpy(pal, s->pal[i], 8ull * s->P[i]);
    or_decode_brick(pal, s->P[i], nib, (ns + 1) / 2, s->b, lod, dst);
    free(pal);
    free(nib);
}

int or_serve_step(or_server* s, const uint32_t* sess, const double* views_in, uint32_t n, uint64_t* out_label,
                  float* out_depth, uint32_t* stats) {
    if (n == 0 || n > OR_MAXV) return -1;
    const uint32_t nb = s->nb, b = s->b;
    memset(stats, 0, sizeof(uint32_t) * OR_SERVE_STATS);
    /* directions normalised as the view's forward (camera.js:63) */
    double views[OR_MAXV * 6];
    for (uint32_t k = 0; k < n; ++k) {
        const double* v = views_in + 6 * k;
        double len = sqrt(v[3] * v[3] + v[4] * v[4] + v[5] * v[5]);
        if (len == 0.0) len = 1.0;
        views[6 * k + 0] = v[0];
        views[6 * k + 1] = v[1];
        views[6 * k + 2] = v[2];
        views[6 * k + 3] = v[3] / len;
        views[6 * k + 4] = v[4] / len;
        views[6 * k + 5] = v[5] / len;
    }
    const int plan = views_moved(s, sess, views, n);
    if (plan) {
        s->planned_once = 1;
        s->n_last = n;
        for (uint32_t k = 0; k < n; ++k) {
            s->last_sess[k] = sess[k];
            memcpy(s->last_view[k], views + 6 * k, sizeof(double) * 6);
        }
        uint8_t* want = (uint8_t*)malloc(nb + 1);
        uint32_t A[OR_MAXV] = {0}, Wn[OR_MAXV] = {0};
        for (uint32_t i = 0; i < nb; ++i) {
            uint8_t w = OR_NONE;
            if (s->has[i]) {
                uint32_t x, y, z;
                or_demorton3(s->id[i], &x, &y, &z);
                const double c[3] = {(double)x * (double)b + s->half, (double)y * (double)b + s->half,
                                     (double)z * (double)b + s->half};
                for (uint32_t k = 0; k < n; ++k) {
                    if (!brick_in_cone(s, c, views + 6 * k)) continue;
                    const uint32_t l = or_brick_lod(c, (double)b, views + 6 * k, s->focal, s->max_lod);
                    if (w == OR_NONE || l > w) w = (uint8_t)l;
                }
            }
            want[i] = w;
            if (w != OR_NONE) stats[OR_ST_VISIBLE]++;
            const int cached = w != OR_NONE && w > 0 && !s->uni[i];
            const int keep = cached && s->res_lod[i] == w;
            if (s->res_lod[i] != OR_NONE && !keep) { /* free: push in brick order */
                const uint32_t l = s->res_lod[i];
                s->stack[l][s->top[l]++] = s->res_off[i];
                s->res_lod[i] = OR_NONE;
                stats[OR_ST_FREED]++;
            }
            if (cached && !keep) A[w]++;
            if (cached) Wn[w]++;
        }
        uint64_t need = 0;
        for (uint32_t l = 1; l <= s->max_lod; ++l)
            if (A[l] > s->top[l]) need += (uint64_t)(A[l] - s->top[l]) << (3 * l);
        uint32_t* admitted = (uint32_t*)malloc(sizeof(uint32_t) * (nb + 1));
        uint32_t n_adm = 0;
        if (s->bump + need <= s->cap) {
            for (uint32_t l = 1; l <= s->max_lod; ++l)
                for (uint32_t i = 0; i < nb; ++i) {
                    const int cached = want[i] == l && !s->uni[i];
                    if (!cached || s->res_lod[i] == l) continue;
                    uint64_t off;
                    if (s->top[l] > 0) off = s->stack[l][--s->top[l]];
                    else {
                        off = s->bump;
                        s->bump += 1ull << (3 * l);
                    }
                    s->res_lod[i] = (uint8_t)l;
                    s->res_off[i] = off;
                    admitted[n_adm++] = i;
                }
        } else {
            stats[OR_ST_REBUILT] = 1;
            for (uint32_t i = 0; i < nb; ++i) s->res_lod[i] = OR_NONE;
            for (uint32_t l = 0; l < OR_MAXV; ++l) s->top[l] = 0;
            s->bump = 0;
            for (uint32_t l = 1; l <= s->max_lod; ++l)
                for (uint32_t i = 0; i < nb; ++i) {
                    if (want[i] != l || s->uni[i]) continue;
                    const uint64_t sz = 1ull << (3 * l);
                    if (s->bump + sz > s->cap) continue;
                    s->res_lod[i] = (uint8_t)l;
                    s->res_off[i] = s->bump;
                    s->bump += sz;
                    admitted[n_adm++] = i;
                }
        }
        uint64_t vox = 0;
        for (uint32_t k = 0; k < n_adm; ++k) {
            const uint32_t i = admitted[k];
            decode_into(s, i, s->res_lod[i], s->cache + s->pal_region + s->res_off[i]);
            vox += 1ull << (3 * s->res_lod[i]);
        }
        stats[OR_ST_DECODED] = n_adm;
        stats[OR_ST_VOX_LO] = (uint32_t)vox;
        stats[OR_ST_VOX_HI] = (uint32_t)(vox >> 32);
        /* slot table */
        for (uint32_t i = 0; i < nb; ++i) {
            or_slot sl = {0, 0, 0};
            if (!s->has[i]) sl.flags = 1u;
            else if (s->res_lod[i] != OR_NONE) {
                sl.offset = s->pal_region + s->res_off[i];
                sl.lod = s->res_lod[i];
            } else if (s->uni[i] || want[i] == 0) {
                sl.offset = i;
            } else sl.flags = 2u;
            s->slots[s->id[i]] = sl;
        }
        free(admitted);
        free(want);
        stats[OR_ST_PLANNED] = 1;
    }
    for (uint32_t i = 0; i < nb; ++i) stats[OR_ST_RESIDENT] += s->res_lod[i] != OR_NONE;
    /* render every view; request words as brickRequests, union over the views */
    uint32_t* req = (uint32_t*)calloc(s->n_slots, 4);
    const size_t px = (size_t)s->W * s->H;
    for (uint32_t k = 0; k < n; ++k) {
        float cam[16];
        or_camera_uniform(views_in + 6 * k, views_in + 6 * k + 3, s->fov, cam);
        or_render_rows(cam, s->W, s->H, 0, 1, (float)(s->bpa * b), b, s->bpa, s->slots, s->n_slots, s->cache,
                       s->hidden, s->n_hidden, out_label + k * px, out_depth + k * px, NULL, req);
    }
    for (uint64_t m = 0; m < s->n_slots; ++m) {
        if (req[m]) stats[OR_ST_ENTERED]++;
        if (req[m] == 3u) stats[OR_ST_MISSING]++;
    }
    free(req);
    return 0;
}
