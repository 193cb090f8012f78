/* csv_oracle_serve.c -- CPU restatement of the viewer's frame loop: plan,
 * cache policy, decode of the admitted bricks, render.  Test infrastructure
 * only: it is the checker the device server is compared with, slot table for
 * slot table and pixel for pixel.
 *
 * Follows, per frame (renderLoop.js:208-340 with LOD_UPDATE_INTERVAL 1):
 *   - the camera-moved test (culling.js:22-56): a view is re-planned only when
 *     its camera moved more than 0.5 units or turned more than 0.05 rad since
 *     the view its plan used;
 *   - the LOD of every brick (camera.js:103-137, screen size min(W, H),
 *     renderLoop.js:374) and the cone test (culling.js:87-153), with the
 *     transfer-function test (culling.js:162-171) as a per-brick flag;
 *   - the cache (cacheManager.js:10-246, cacheProcessing.js:99-232): per-LOD
 *     free stacks of blocks of 8^lod labels, a bump pointer, eviction of the
 *     blocks no view needs, a rebuild when an allocation fails;
 *   - the decode of the newly admitted (brick, LOD) blocks and the label/depth
 *     render of every view that submitted a frame (or_render_rows).
 *
 * Several sessions (viewers) share one cache.  Each keeps its own LODs and its
 * own slot table, so a session's image does not depend on which other
 * sessions are open (given room in the cache): a block is keyed by (brick,
 * LOD), and a brick two sessions see at different LODs holds two blocks.
 * With one session this is the reference's loop.
 *
 * Where the reference leaves an order or a corner case open, this file fixes
 * it, and the device server follows the same rules:
 *   - frees are pushed in brick (file) order; admissions are served LOD by
 *     LOD (coarse first), in brick order within a LOD, each popping its LOD's
 *     stack (last pushed first) and taking fresh space from the bump pointer
 *     once the stack is empty;
 *   - when the frame's fresh space does not fit, the cache is rebuilt: every
 *     block is dropped and every needed block is placed again, LOD by LOD
 *     (coarse first) in brick order, while space remains (the blocks that do
 *     not fit stay missing for this frame);
 *   - LOD-0 bricks and uniform bricks (root stop bit: the whole brick is
 *     palette[0]) take no block: their slot reads palette[0] from a table at
 *     the start of the cache (rayTrace.wgsl:167-178 reads palette[0] for LOD 0;
 *     a uniform brick decodes to palette[0] at every LOD, so the image is the
 *     one a decoded copy would give);
 *   - admission by rays (or_serve_set_admit 1): the path the reference wrote
 *     and left switched off (cacheProcessing.js:134-164, useGPUCulling; the
 *     marcher's brickRequests words, rayTrace.wgsl:682-686).  A brick a session
 *     needs by the cone and LOD tests is kept or admitted only if that
 *     session's rays entered it in its last render; a session with no render
 *     since the last plan (a new session) keeps the cone plan, the reference's
 *     fallback while no requests are ready.  The plan consumes the words.  In
 *     this mode a step also re-plans when an open session rendered since the
 *     last plan (the requests change while the camera stands still, as bricks
 *     arrive and hide the ones behind them);
 *   - compaction (or_serve_compact, CacheState.compact(), cacheManager.js:
 *     170-211): every resident block is kept and placed again from offset 0,
 *     LOD by LOD (coarse first) in brick order, the free stacks are
 *     emptied and fresh space starts after the last block; the blocks' labels
 *     are those they held (decoded again into their new place);
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
#define OR_LODS 8

struct or_server {
    uint32_t nb, b, max_lod, bpa, W, H, cone, n_hidden;
    double fov, focal, cos_half, radius, half;
    uint32_t freq[16], cum[16];
    /* per brick */
    uint32_t* id;
    uint8_t* has;      /* a palette entry is neither 0 nor hidden */
    uint8_t* uni;      /* uniform brick */
    const uint8_t** enc;
    uint32_t* E;
    uint32_t* nsym;
    const uint8_t* pal_bytes;
    size_t* pal_at;
    uint32_t* P;
    uint8_t* res;      /* bit l: a block at LOD l is resident */
    uint64_t* off;     /* [brick][OR_LODS] block offsets */
    uint8_t* want[OR_MAX_SESSIONS]; /* per session and brick: its LOD, OR_NONE when it does not need the brick */
    /* cache */
    uint64_t pal_region, cap, bump;
    uint64_t* cache;
    uint64_t* stack[OR_LODS]; /* per LOD, nb entries */
    uint32_t top[OR_LODS];
    or_slot* slots[OR_MAX_SESSIONS];
    uint64_t n_slots;
    uint64_t* hidden;
    /* plan bookkeeping */
    uint8_t planned[OR_MAX_SESSIONS];     /* the session has a planned view */
    double pview[OR_MAX_SESSIONS][6];     /* the view its plan used */
    uint8_t last_open[OR_MAX_SESSIONS];   /* open at the last plan */
    /* admission by rays */
    uint32_t admit;                       /* 0: cone plan, 1: rays' requests */
    uint32_t* req[OR_MAX_SESSIONS];       /* request words of the session's last render, by Morton slot */
    uint8_t ready[OR_MAX_SESSIONS];       /* the session rendered since the last plan */
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

/* culling.js:87-153 for one brick centre and one view (position, unit direction). */
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

static uint64_t pal_entry(const or_server* s, uint32_t i, uint32_t k) {
    uint64_t v;
    memcpy(&v, s->pal_bytes + s->pal_at[i] + 8ull * k, 8);
    return v;
}

or_server* or_serve_new(const uint8_t* img, size_t len, uint32_t W, uint32_t H, double fov, uint32_t cone,
                        uint64_t cache_bytes, const uint64_t* hidden, uint32_t n_hidden) {
    if (!img || len < 152 || rd32(img) != 0x43534244u) return NULL;
    or_server* s = (or_server*)calloc(1, sizeof *s);
    s->nb = rd32(img + 8);
    s->b = rd32(img + 12);
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
    s->enc = (const uint8_t**)calloc(nb + 1, sizeof(void*));
    s->pal_at = (size_t*)calloc(nb + 1, sizeof(size_t));
    s->E = (uint32_t*)calloc(nb + 1, 4);
    s->nsym = (uint32_t*)calloc(nb + 1, 4);
    s->P = (uint32_t*)calloc(nb + 1, 4);
    s->res = (uint8_t*)calloc(nb + 1, 1);
    s->off = (uint64_t*)calloc((size_t)(nb + 1) * OR_LODS, 8);
    for (int k = 0; k < OR_MAX_SESSIONS; ++k) {
        s->want[k] = (uint8_t*)malloc(nb + 1);
        memset(s->want[k], OR_NONE, nb + 1);
    }
    s->pal_bytes = img;
    size_t o = 152;
    uint32_t maxc = 0;
    for (uint32_t i = 0; i < nb; ++i) {
        s->id[i] = rd32(img + o);
        s->P[i] = rd32(img + o + 4);
        s->pal_at[i] = o + 8;
        o += 8 + 8ull * s->P[i];
        s->E[i] = rd32(img + o);
        s->enc[i] = img + o + 4;
        o += 4 + s->E[i];
        s->nsym[i] = rd32(img + o);
        o += 4;
        for (uint32_t k = 0; k < s->P[i]; ++k) {
            const uint64_t v = pal_entry(s, i, k);
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
    s->bpa = maxc + 1;
    uint32_t p2 = 1;
    while (p2 < s->bpa) p2 <<= 1;
    s->n_slots = (uint64_t)p2 * p2 * p2;
    for (int k = 0; k < OR_MAX_SESSIONS; ++k) {
        s->slots[k] = (or_slot*)calloc(s->n_slots, sizeof(or_slot));
        for (uint64_t m = 0; m < s->n_slots; ++m) s->slots[k][m].flags = 1u;
        s->req[k] = (uint32_t*)calloc(s->n_slots, 4);
    }
    const uint64_t total = cache_bytes / 8;
    s->pal_region = ((uint64_t)nb + 31) & ~31ull;
    s->cap = total > s->pal_region ? total - s->pal_region : 0;
    s->cache = (uint64_t*)calloc(total ? total : 1, 8);
    for (uint32_t i = 0; i < nb && i < total; ++i) s->cache[i] = s->P[i] ? pal_entry(s, i, 0) : 0;
    for (uint32_t l = 0; l < OR_LODS; ++l) s->stack[l] = (uint64_t*)calloc(nb + 1, 8);
    return s;
}

void or_serve_free(or_server* s) {
    if (!s) return;
    free(s->id); free(s->has); free(s->uni); free(s->enc); free(s->pal_at); free(s->E);
    free(s->nsym); free(s->P); free(s->res); free(s->off); free(s->cache); free(s->hidden);
    for (int k = 0; k < OR_MAX_SESSIONS; ++k) {
        free(s->want[k]);
        free(s->slots[k]);
        free(s->req[k]);
    }
    for (uint32_t l = 0; l < OR_LODS; ++l) free(s->stack[l]);
    free(s);
}

void or_serve_set_admit(or_server* s, uint32_t admit) { s->admit = admit; }

uint64_t or_serve_n_slots(const or_server* s) { return s->n_slots; }
uint32_t or_serve_bricks_per_axis(const or_server* s) { return s->bpa; }
const or_slot* or_serve_slots(const or_server* s, uint32_t session) {
    return session < OR_MAX_SESSIONS ? s->slots[session] : NULL;
}
const uint64_t* or_serve_cache(const or_server* s) { return s->cache; }

/* culling.js:22-56: moved more than 0.5 units or turned more than 0.05 rad. */
static int view_moved(const double* v, const double* p) {
    const double dx = v[0] - p[0], dy = v[1] - p[1], dz = v[2] - p[2];
    const double moved = dx * dx + dy * dy + dz * dz;
    const double dot = v[3] * p[3] + v[4] * p[4] + v[5] * p[5];
    return moved > 0.5 * 0.5 || dot < cos(0.05);
}

static void decode_into(or_server* s, uint32_t i, uint32_t lod, uint64_t* dst) {
    const uint32_t ns = s->nsym[i];
    uint8_t* nib = (uint8_t*)calloc(ns / 2 + 2, 1);
    if (s->E[i] >= 4 && ns >= 1) or_rans_decode(s->freq, s->cum, 4096, s->enc[i], s->E[i], ns, nib);
    uint64_t* pal = (uint64_t*)malloc(8ull * (s->P[i] ? s->P[i] : 1));
    for (uint32_t k = 0; k < s->P[i]; ++k) pal[k] = pal_entry(s, i, k);
    or_decode_brick(pal, s->P[i], nib, (ns + 1) / 2, s->b, lod, dst);
    free(pal);
    free(nib);
}

static uint8_t need_mask(const or_server* s, uint32_t i, const uint8_t* open) {
    uint8_t m = 0;
    if (s->uni[i]) return 0;
    for (int k = 0; k < OR_MAX_SESSIONS; ++k) {
        if (!open[k]) continue;
        const uint8_t w = s->want[k][i];
        if (w != OR_NONE && w > 0) m |= (uint8_t)(1u << w);
    }
    return m;
}

static void plan(or_server* s, const uint8_t* open, uint32_t* stats) {
    const uint32_t nb = s->nb, b = s->b;
    /* wants of every open session with its planned view */
    for (int k = 0; k < OR_MAX_SESSIONS; ++k) {
        if (!open[k]) {
            memset(s->want[k], OR_NONE, nb + 1);
            continue;
        }
        for (uint32_t i = 0; i < nb; ++i) {
            uint8_t w = OR_NONE;
            if (s->has[i]) {
                uint32_t x, y, z;
                or_demorton3(s->id[i], &x, &y, &z);
                const double c[3] = {(double)x * (double)b + s->half, (double)y * (double)b + s->half,
                                     (double)z * (double)b + s->half};
                if (brick_in_cone(s, c, s->pview[k]))
                    w = (uint8_t)or_brick_lod(c, (double)b, s->pview[k], s->focal, s->max_lod);
                /* admission by rays: only the bricks the session's last render entered */
                if (s->admit && s->ready[k] && s->req[k][s->id[i]] == 0) w = OR_NONE;
            }
            s->want[k][i] = w;
        }
        if (s->admit && s->ready[k]) { /* the plan consumes the requests */
            memset(s->req[k], 0, s->n_slots * 4);
            s->ready[k] = 0;
        }
    }
    uint32_t A[OR_LODS] = {0};
    for (uint32_t i = 0; i < nb; ++i) {
        int vis = 0;
        for (int k = 0; k < OR_MAX_SESSIONS; ++k) vis |= open[k] && s->want[k][i] != OR_NONE;
        stats[OR_ST_VISIBLE] += vis;
        const uint8_t need = need_mask(s, i, open);
        const uint8_t fr = s->res[i] & (uint8_t)~need;
        for (uint32_t l = 1; l <= s->max_lod; ++l) /* frees: pushed in brick order */
            if (fr & (1u << l)) {
                s->stack[l][s->top[l]++] = s->off[(size_t)i * OR_LODS + l];
                stats[OR_ST_FREED]++;
            }
        s->res[i] &= need;
        const uint8_t al = need & (uint8_t)~s->res[i];
        for (uint32_t l = 1; l <= s->max_lod; ++l) A[l] += (al >> l) & 1u;
    }
    uint64_t fresh = 0;
    for (uint32_t l = 1; l <= s->max_lod; ++l)
        if (A[l] > s->top[l]) fresh += (uint64_t)(A[l] - s->top[l]) << (3 * l);
    uint32_t* adm = (uint32_t*)malloc(sizeof(uint32_t) * ((size_t)nb * OR_LODS + 1));
    uint32_t n_adm = 0;
    if (s->bump + fresh <= s->cap) {
        for (uint32_t l = 1; l <= s->max_lod; ++l)
            for (uint32_t i = 0; i < nb; ++i) {
                const uint8_t need = need_mask(s, i, open);
                if (!((need >> l) & 1u) || ((s->res[i] >> l) & 1u)) continue;
                uint64_t o;
                if (s->top[l] > 0) o = s->stack[l][--s->top[l]];
                else {
                    o = s->bump;
                    s->bump += 1ull << (3 * l);
                }
                s->res[i] |= (uint8_t)(1u << l);
                s->off[(size_t)i * OR_LODS + l] = o;
                adm[n_adm++] = i * OR_LODS + l;
            }
    } else {
        stats[OR_ST_REBUILT] = 1;
        memset(s->res, 0, nb + 1);
        for (uint32_t l = 0; l < OR_LODS; ++l) s->top[l] = 0;
        s->bump = 0;
        for (uint32_t l = 1; l <= s->max_lod; ++l)
            for (uint32_t i = 0; i < nb; ++i) {
                if (!((need_mask(s, i, open) >> l) & 1u)) continue;
                const uint64_t sz = 1ull << (3 * l);
                if (s->bump + sz > s->cap) continue;
                s->res[i] |= (uint8_t)(1u << l);
                s->off[(size_t)i * OR_LODS + l] = s->bump;
                s->bump += sz;
                adm[n_adm++] = i * OR_LODS + l;
            }
    }
    uint64_t vox = 0;
    for (uint32_t k = 0; k < n_adm; ++k) {
        const uint32_t i = adm[k] / OR_LODS, l = adm[k] % OR_LODS;
        decode_into(s, i, l, s->cache + s->pal_region + s->off[(size_t)i * OR_LODS + l]);
        vox += 1ull << (3 * l);
    }
    free(adm);
    stats[OR_ST_DECODED] = n_adm;
    stats[OR_ST_VOX_LO] = (uint32_t)vox;
    stats[OR_ST_VOX_HI] = (uint32_t)(vox >> 32);
    /* slot tables of the open sessions */
    for (int k = 0; k < OR_MAX_SESSIONS; ++k) {
        if (!open[k]) continue;
        for (uint32_t i = 0; i < nb; ++i) {
            const uint8_t w = s->want[k][i];
            or_slot sl = {0, 0, 0};
            if (!s->has[i]) sl.flags = 1u;
            else if (s->uni[i] || w == 0) sl.offset = i;
            else if (w != OR_NONE && ((s->res[i] >> w) & 1u)) {
                sl.offset = s->pal_region + s->off[(size_t)i * OR_LODS + w];
                sl.lod = w;
            } else sl.flags = 2u;
            s->slots[k][s->id[i]] = sl;
        }
    }
    stats[OR_ST_PLANNED] = 1;
}

int or_serve_step(or_server* s, const uint32_t* sess, const double* views_in, const uint8_t* render, uint32_t n,
                  uint64_t* out_label, float* out_depth, uint32_t* stats) {
    if (n > OR_MAX_SESSIONS) return -1;
    memset(stats, 0, sizeof(uint32_t) * OR_SERVE_STATS);
    uint8_t open[OR_MAX_SESSIONS] = {0};
    int changed = 0;
    for (uint32_t k = 0; k < n; ++k) {
        const uint32_t id = sess[k];
        if (id >= OR_MAX_SESSIONS || open[id]) return -1;
        open[id] = 1;
        const double* v = views_in + 6 * k;
        double len = sqrt(v[3] * v[3] + v[4] * v[4] + v[5] * v[5]);
        if (len == 0.0) len = 1.0;
        const double u[6] = {v[0], v[1], v[2], v[3] / len, v[4] / len, v[5] / len};
        if (!s->planned[id] || view_moved(u, s->pview[id])) {
            memcpy(s->pview[id], u, sizeof u);
            s->planned[id] = 1;
            changed = 1;
        }
    }
    for (int k = 0; k < OR_MAX_SESSIONS; ++k) {
        if (open[k] != s->last_open[k]) changed = 1;
        if (!open[k]) {
            s->planned[k] = 0;
            if (s->ready[k]) { /* a closed session's requests are dropped */
                memset(s->req[k], 0, s->n_slots * 4);
                s->ready[k] = 0;
            }
        }
    }
    if (s->admit) /* admission by rays: new requests re-plan */
        for (int k = 0; k < OR_MAX_SESSIONS; ++k) changed |= open[k] && s->ready[k];
    if (changed) {
        plan(s, open, stats);
        memcpy(s->last_open, open, sizeof open);
    }
    for (uint32_t i = 0; i < s->nb; ++i)
        for (uint32_t l = 1; l <= s->max_lod; ++l) stats[OR_ST_RESIDENT] += (s->res[i] >> l) & 1u;
    /* render the sessions that submitted a frame; request words as brickRequests (kept for the next plan
       when admission is by rays) */
    uint32_t* tmp = (uint32_t*)calloc(s->n_slots, 4);
    const size_t px = (size_t)s->W * s->H;
    uint32_t j = 0;
    for (uint32_t k = 0; k < n; ++k) {
        if (!render[k]) continue;
        float cam[16];
        or_camera_uniform(views_in + 6 * k, views_in + 6 * k + 3, s->fov, cam);
        uint32_t* req = s->admit ? s->req[sess[k]] : tmp;
        memset(req, 0, s->n_slots * 4);
        if (s->admit) s->ready[sess[k]] = 1;
        or_render_rows(cam, s->W, s->H, 0, 1, (float)(s->bpa * s->b), s->b, s->bpa, s->slots[sess[k]], s->n_slots,
                       s->cache, s->hidden, s->n_hidden, out_label + j * px, out_depth + j * px, NULL, req);
        for (uint64_t m = 0; m < s->n_slots; ++m) {
            if (req[m]) stats[OR_ST_SESSION + 2 * j]++;
            if (req[m] == 3u) stats[OR_ST_SESSION + 2 * j + 1]++;
        }
        ++j;
    }
    free(tmp);
    return 0;
}

/* CacheState.compact() (cacheManager.js:170-211) with the labels moved: every
 * resident block placed again from offset 0, LOD by LOD (coarse first) in brick
 * order; free stacks emptied; fresh space after the last block; the slot tables
 * of the sessions open at the last plan point at the new places. */
int or_serve_compact(or_server* s) {
    const uint32_t nb = s->nb;
    uint64_t* newoff = (uint64_t*)calloc((size_t)(nb + 1) * OR_LODS, 8);
    uint64_t b = 0;
    for (uint32_t l = 1; l <= s->max_lod; ++l)
        for (uint32_t i = 0; i < nb; ++i) {
            if (!((s->res[i] >> l) & 1u)) continue;
            newoff[(size_t)i * OR_LODS + l] = b;
            b += 1ull << (3 * l);
        }
    /* decode into the new places (the labels equal the old block's) */
    for (uint32_t l = 1; l <= s->max_lod; ++l)
        for (uint32_t i = 0; i < nb; ++i)
            if ((s->res[i] >> l) & 1u) {
                s->off[(size_t)i * OR_LODS + l] = newoff[(size_t)i * OR_LODS + l];
                decode_into(s, i, l, s->cache + s->pal_region + newoff[(size_t)i * OR_LODS + l]);
            }
    free(newoff);
    s->bump = b;
    for (uint32_t l = 0; l < OR_LODS; ++l) s->top[l] = 0;
    for (int k = 0; k < OR_MAX_SESSIONS; ++k) {
        if (!s->last_open[k]) continue;
        for (uint32_t i = 0; i < nb; ++i) {
            const uint8_t w = s->want[k][i];
            or_slot* sl = &s->slots[k][s->id[i]];
            if (s->has[i] && !s->uni[i] && w != OR_NONE && w != 0 && ((s->res[i] >> w) & 1u))
                sl->offset = s->pal_region + s->off[(size_t)i * OR_LODS + w];
        }
    }
    return 0;
}
