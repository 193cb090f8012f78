/* csv_oracle.c -- CPU restatement of the reference brick codec.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle).  Loaded by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg, as the checker.
 * The product library never links or calls it.
 *
 * Each function cites the reference lines it restates.  Reference paths are
 * relative to the reference project root.  Parity of this restatement is
 * pinned in tests/test_oracle.py against the reference sources compiled as
 * oracle/_ref/libcsvref.so (encode bytes, full-resolution decode, majority
 * vote, rANS model) and against the shipped compressed_dataset.csbd.
 */
#include "csv_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define EMPTY_LABEL UINT64_MAX /* types.hpp:19 */
#define RANS_L (1u << 23)      /* types.hpp:24-28 */
#define TOT_BITS 12u
#define TOT (1u << TOT_BITS)

enum { OP_RP = 0, OP_RX, OP_RY, OP_RZ, OP_PA, OP_P0, OP_PD }; /* types.hpp:162-171 */

void or_free(void* p) { free(p); }

/* ---------------------------------------------------------------- Morton */
/* utils.cpp:4-21: 10 bits per axis, x in bit 0. */
static uint32_t spread3(uint32_t v) {
    uint32_t r = 0;
    for (int i = 0; i < 10; ++i) r |= ((v >> i) & 1u) << (3 * i);
    return r;
}
uint32_t or_morton3(uint32_t x, uint32_t y, uint32_t z) {
    return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
}
/* utils.cpp:24-43 */
void or_demorton3(uint32_t m, uint32_t* x, uint32_t* y, uint32_t* z) {
    uint32_t a = 0, b = 0, c = 0;
    for (int i = 0; i < 10; ++i) {
        a |= ((m >> (3 * i)) & 1u) << i;
        b |= ((m >> (3 * i + 1)) & 1u) << i;
        c |= ((m >> (3 * i + 2)) & 1u) << i;
    }
    *x = a; *y = b; *z = c;
}

/* ------------------------------------------------------------- majority */
/* majorityVote8 (brick.hpp:24-37): std::max_element over a
 * std::unordered_map<uint64_t,int> filled in child order 0..7.  With GNU
 * libstdc++ the map has 13 buckets for up to 8 keys and the identity hash, so
 * key k sits in bucket k % 13.  A key whose bucket is empty is linked at the
 * front of the iteration list; a key whose bucket is occupied is linked just
 * before that bucket's first key.  Iteration therefore visits bucket groups
 * newest-group-first and, inside a group, newest-key-first; max_element keeps
 * the first maximal count.  Equivalently: among keys with the maximal count,
 * the winner maximises (first-insertion index of its bucket group, its own
 * insertion index). */
uint64_t or_majority8(const uint64_t* v) {
    uint64_t key[8];
    int cnt[8], grp[8], n = 0;
    for (int i = 0; i < 8; ++i) {
        int j;
        for (j = 0; j < n; ++j)
            if (key[j] == v[i]) break;
        if (j < n) { cnt[j]++; continue; }
        key[n] = v[i];
        cnt[n] = 1;
        grp[n] = n;
        for (int k = 0; k < n; ++k)
            if (key[k] % 13u == v[i] % 13u) { grp[n] = grp[k]; break; }
        n++;
    }
    int best = 0;
    for (int j = 1; j < n; ++j) {
        if (cnt[j] > cnt[best] ||
            (cnt[j] == cnt[best] && (grp[j] > grp[best] || (grp[j] == grp[best] && j > best))))
            best = j;
    }
    return key[best];
}

/* -------------------------------------------------------------- pyramid */
/* splitGridIntoBricks (brick.hpp:133-195): brick (bx,by,bz) voxel (dx,dy,dz)
 * reads vol[gx + W*(gy + H*gz)], 0 outside the volume, stored at Morton
 * index of (dx,dy,dz).  Brick::buildLevel (brick.hpp:92-123): parent m has
 * children 8m..8m+7 (utils.cpp:45-68); constant = all 8 children equal the
 * majority and are constant themselves; leaves are constant (brick.hpp:188).
 * Levels are stored coarse-first here: level l at offset (8^l-1)/7. */
static uint32_t levels_of(uint32_t b) {
    uint32_t L = 0;
    while ((1u << L) < b) L++;
    return L + 1; /* std::bit_width(b), brick.hpp:50 */
}
static size_t level_off(uint32_t l) { return (((size_t)1 << (3 * l)) - 1) / 7; }

static void cut_brick(const uint64_t* vol, size_t W, size_t H, size_t D, uint32_t b,
                      size_t bx, size_t by, size_t bz, uint64_t* leaf) {
    for (uint32_t dz = 0; dz < b; ++dz)
        for (uint32_t dy = 0; dy < b; ++dy)
            for (uint32_t dx = 0; dx < b; ++dx) {
                size_t gx = bx * b + dx, gy = by * b + dy, gz = bz * b + dz;
                uint64_t lab = 0;
                if (gx < W && gy < H && gz < D) lab = vol[gx + W * (gy + H * gz)];
                leaf[or_morton3(dx, dy, dz)] = lab;
            }
}

static void build_pyramid(uint32_t b, uint64_t* lab, uint8_t* cst) {
    uint32_t L = levels_of(b);
    size_t nleaf = (size_t)b * b * b;
    memset(cst + level_off(L - 1), 1, nleaf);
    for (int l = (int)L - 2; l >= 0; --l) {
        size_t nn = (size_t)1 << (3 * l);
        uint64_t* P = lab + level_off(l);
        uint8_t* PC = cst + level_off(l);
        const uint64_t* C = lab + level_off(l + 1);
        const uint8_t* CC = cst + level_off(l + 1);
        for (size_t m = 0; m < nn; ++m) {
            uint64_t maj = or_majority8(C + 8 * m);
            int same = 1;
            for (int c = 0; c < 8; ++c) same &= (C[8 * m + c] == maj) && CC[8 * m + c];
            P[m] = maj;
            PC[m] = (uint8_t)same;
        }
    }
}

int or_pyramid(const uint64_t* vol, size_t W, size_t H, size_t D, uint32_t b, uint32_t brick_index,
               uint64_t* labels, uint8_t* constant) {
    size_t nbx = (W + b - 1) / b, nby = (H + b - 1) / b, nbz = (D + b - 1) / b;
    if (brick_index >= nbx * nby * nbz) return -1;
    /* split order: bx outer, bz inner (brick.hpp:152-154) */
    size_t bz = brick_index % nbz, by = (brick_index / nbz) % nby, bx = brick_index / (nbz * nby);
    uint32_t L = levels_of(b);
    cut_brick(vol, W, H, D, b, bx, by, bz, labels + level_off(L - 1));
    build_pyramid(b, labels, constant);
    return 0;
}

/* ------------------------------------------------------------ encoding */
typedef struct { uint8_t* p; size_t n, cap; } buf_t;
static void bput(buf_t* b, const void* src, size_t n) {
    if (b->n + n > b->cap) {
        size_t c = b->cap ? b->cap : 1024;
        while (c < b->n + n) c *= 2;
        b->p = (uint8_t*)realloc(b->p, c);
        b->cap = c;
    }
    memcpy(b->p + b->n, src, n);
    b->n += n;
}
static void bput32(buf_t* b, uint32_t v) { bput(b, &v, 4); }

typedef struct {
    uint64_t* pal; uint32_t np, pcap;
    uint8_t* nib;  uint32_t nn, ncap; /* one nibble per byte while building */
} enc_t;

static void push_nib(enc_t* e, uint8_t v) {
    if (e->nn == e->ncap) { e->ncap = e->ncap ? 2 * e->ncap : 4096; e->nib = (uint8_t*)realloc(e->nib, e->ncap); }
    e->nib[e->nn++] = v & 15;
}
static void push_pal(enc_t* e, uint64_t v) {
    if (e->np == e->pcap) { e->pcap = e->pcap ? 2 * e->pcap : 64; e->pal = (uint64_t*)realloc(e->pal, 8 * e->pcap); }
    e->pal[e->np++] = v;
}

/* Encoding modes (no reference counterpart): mode % 6 orders the neighbour
 * axes, modes >= 6 try the neighbours before the parent; mode 0 is the
 * reference's order (Rp, Rx, Ry, Rz: brickEncoding.hpp:202-203, 277-282). */
static const int AXIS_ORDER[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};

/* bestOperation (brickEncoding.hpp:188-318) for child `n` (Morton) at coarse
 * level lc = l+1 with parent level l, under encoding mode `mode`. */
static int best_op(const uint64_t* lab, uint32_t lc, uint32_t n, uint64_t parent_label, enc_t* e, uint8_t* delta,
                   uint32_t mode) {
    const uint64_t* C = lab + level_off(lc);
    const uint64_t* P = lab + level_off(lc - 1);
    uint64_t L = C[n];
    const int nfirst = mode >= 6;
    if (!nfirst && parent_label == L) return OP_RP; /* :202-203 */
    uint32_t x, y, z;
    or_demorton3(n, &x, &y, &z);
    int size = 1 << lc;
    for (int k = 0; k < 3; ++k) { /* X, Y, Z order in mode 0: :277-282 */
        const int axis = AXIS_ORDER[nfirst ? mode - 6 : mode][k];
        int c[3] = {(int)x, (int)y, (int)z};
        c[axis] += (c[axis] & 1) ? 1 : -1; /* outside the sibling block: :224-240 */
        if (c[axis] < 0 || c[axis] >= size) continue; /* :244-246 */
        uint32_t nm = or_morton3((uint32_t)c[0], (uint32_t)c[1], (uint32_t)c[2]);
        if (nm < n) {
            if (C[nm] == L) return OP_RX + axis; /* :256-261 */
        } else {
            /* neighbor's parent (:265-272); levelIndex = lc > 0 always here */
            if (P[or_morton3((uint32_t)c[0] >> 1, (uint32_t)c[1] >> 1, (uint32_t)c[2] >> 1)] == L)
                return OP_RX + axis;
        }
    }
    if (nfirst && parent_label == L) return OP_RP;
    /* palette reverse find (:288-317) */
    for (int64_t i = (int64_t)e->np - 1; i >= 0; --i) {
        if (e->pal[i] == L) {
            uint32_t last = e->np - 1;
            if ((uint32_t)i == last) return OP_P0;
            uint32_t dist = last - (uint32_t)i - 1;
            if (dist <= 15) { *delta = (uint8_t)dist; return OP_PD; }
            return OP_PA;
        }
    }
    return OP_PA;
}

/* encodeBrick (brickEncoding.hpp:348-447) + packOperationsToNibbles
 * (brickEncoding.cpp:11-91): nibbles in emission order. */
static void encode_brick(uint32_t b, const uint64_t* lab, const uint8_t* cst, enc_t* e, uint32_t mode) {
    uint32_t L = levels_of(b);
    e->np = 0; e->nn = 0;
    push_pal(e, lab[0]);
    push_nib(e, (uint8_t)((OP_PA << 1) | (cst[0] ? 1 : 0))); /* root: :360-367 */
    for (uint32_t l = 0; l + 1 < L; ++l) {
        size_t nn = (size_t)1 << (3 * l);
        const uint64_t* P = lab + level_off(l);
        const uint8_t* PC = cst + level_off(l);
        const uint8_t* CC = cst + level_off(l + 1);
        const uint64_t* C = lab + level_off(l + 1);
        for (size_t m = 0; m < nn; ++m) {
            if (PC[m]) continue; /* :386 */
            for (uint32_t c = 0; c < 8; ++c) {
                uint32_t n = (uint32_t)(8 * m + c); /* child Morton = 8m + c (utils.cpp:45-68) */
                uint8_t delta = 0;
                int op = best_op(lab, l + 1, n, P[m], e, &delta, mode);
                if (op == OP_PA) push_pal(e, C[n]); /* :423 */
                push_nib(e, (uint8_t)((op << 1) | (CC[n] ? 1 : 0)));
                if (op == OP_PD) push_nib(e, delta);
            }
        }
    }
}

/* buildRansModel (brickEncoding.cpp:146-200). */
void or_build_model(const uint64_t* raw16, uint32_t* freq, uint32_t* cum) {
    uint64_t raw_sum = 0, norm = 0;
    for (int i = 0; i < 16; ++i) {
        uint32_t f = (uint32_t)raw16[i]; /* size_t -> uint32_t as in :157 */
        if (f == 0) f = 1;
        freq[i] = f;
        raw_sum += f;
    }
    for (int i = 0; i < 16; ++i) {
        uint64_t s = ((uint64_t)freq[i] * TOT) / raw_sum;
        if (s == 0) s = 1;
        freq[i] = (uint32_t)s;
        norm += s;
    }
    while (norm < TOT) { freq[0]++; norm++; }
    while (norm > TOT) {
        int largest = 0;
        for (int i = 1; i < 16; ++i)
            if (freq[i] > freq[largest]) largest = i;
        if (freq[largest] > 1) { freq[largest]--; norm--; } else break;
    }
    uint32_t acc = 0;
    for (int i = 0; i < 16; ++i) { cum[i] = acc; acc += freq[i]; }
    cum[16] = acc;
}

/* rANS over the packed bytes: ransEncodeSymbol (brickEncoding.cpp:202-219)
 * applied to all 2*bytes nibbles (pad included) in reverse, then ransFlush
 * (brickEncoding.hpp:452-464) little-endian.  Bytes are in emission order. */
static void rans_encode(const uint8_t* nib, uint32_t nn, const uint32_t* freq, const uint32_t* cum, buf_t* out) {
    uint32_t nsym2 = (nn + 1) & ~1u; /* pad nibble (0) when odd */
    uint32_t x = RANS_L;
    for (int64_t i = (int64_t)nsym2 - 1; i >= 0; --i) {
        uint8_t s = (uint32_t)i < nn ? nib[i] : 0;
        uint32_t f = freq[s], st = cum[s];
        while (x >= ((RANS_L >> TOT_BITS) << 8) * f) {
            uint8_t byte = (uint8_t)(x & 0xff);
            bput(out, &byte, 1);
            x >>= 8;
        }
        x = ((x / f) * TOT) + (x % f) + st;
    }
    for (int i = 0; i < 4; ++i) {
        uint8_t byte = (uint8_t)(x & 0xff);
        bput(out, &byte, 1);
        x >>= 8;
    }
}

/* compressDataset (brickEncoding.hpp:466-531) + saveDatasetToFile
 * (fileIO.cpp:15-99). */
int or_encode(const uint64_t* vol, size_t W, size_t H, size_t D, uint32_t b, uint8_t** out, size_t* out_len) {
    return or_encode_sel(vol, W, H, D, b, NULL, NULL, 0, out, out_len);
}

/* The whole encoder with its options: per-brick mode and table (sel: mode |
 * table << 4, or NULL; n_tables > 0 writes version 2 with those tables, freq,
 * n_tables x 16), and the shard of a larger volume this volume is (its first
 * brick at x-brick bx0 and file index index_base: brick IDs and the
 * every-512th sample rule use the whole volume's numbering).  hist_out (or
 * NULL) receives the sample histogram of these bricks; hist_in (or NULL)
 * replaces it when the model is built (the histogram summed over all shards). */
static int encode_core(const uint64_t* vol, size_t W, size_t H, size_t D, uint32_t b, const uint8_t* sel,
                       const uint32_t* tables, uint32_t n_tables, uint32_t bx0, uint32_t index_base,
                       const uint64_t* hist_in, uint64_t* hist_out, uint8_t** out, size_t* out_len) {
    if (b < 2 || (b & (b - 1)) || b > 1024) return -1;
    size_t nbx = (W + b - 1) / b, nby = (H + b - 1) / b, nbz = (D + b - 1) / b;
    size_t nb = nbx * nby * nbz;
    uint32_t L = levels_of(b);
    size_t ntot = level_off(L);
    uint64_t* lab = (uint64_t*)malloc(ntot * 8);
    uint8_t* cst = (uint8_t*)malloc(ntot);
    enc_t e = {0};
    uint64_t hist[16] = {0};
    /* per brick: palette, nibbles, nsym, ID */
    uint64_t** pals = (uint64_t**)calloc(nb, sizeof(void*));
    uint32_t* npal = (uint32_t*)calloc(nb, 4);
    uint8_t** nibs = (uint8_t**)calloc(nb, sizeof(void*));
    uint32_t* nnib = (uint32_t*)calloc(nb, 4);
    uint32_t* ids = (uint32_t*)calloc(nb, 4);
    size_t i = 0;
    for (size_t bx = 0; bx < nbx; ++bx)
        for (size_t by = 0; by < nby; ++by)
            for (size_t bz = 0; bz < nbz; ++bz, ++i) {
                cut_brick(vol, W, H, D, b, bx, by, bz, lab + level_off(L - 1));
                build_pyramid(b, lab, cst);
                encode_brick(b, lab, cst, &e, sel ? (sel[i] & 15u) : 0u);
                ids[i] = or_morton3((uint32_t)bx + bx0, (uint32_t)by, (uint32_t)bz);
                pals[i] = (uint64_t*)malloc(8 * (size_t)e.np);
                memcpy(pals[i], e.pal, 8 * (size_t)e.np);
                npal[i] = e.np;
                nibs[i] = (uint8_t*)malloc(e.nn + 1);
                memcpy(nibs[i], e.nib, e.nn);
                nnib[i] = e.nn;
                if ((index_base + i) % 512 == 0) { /* brickEncoding.hpp:482, brickEncoding.cpp:131-143 */
                    for (uint32_t k = 0; k < e.nn; ++k) hist[e.nib[k]]++;
                    if (e.nn & 1) hist[0]++; /* the pad nibble of the last byte */
                }
            }
    uint32_t tf[16][16], tc[16][17];
    const uint32_t nt = n_tables ? n_tables : 1;
    if (hist_out) memcpy(hist_out, hist, sizeof hist);
    if (n_tables == 0) {
        or_build_model(hist_in ? hist_in : hist, tf[0], tc[0]);
    } else {
        for (uint32_t t = 0; t < n_tables; ++t) {
            uint32_t acc = 0;
            for (int k = 0; k < 16; ++k) {
                tf[t][k] = tables[16 * t + k];
                tc[t][k] = acc;
                acc += tf[t][k];
            }
            tc[t][16] = acc;
        }
    }
    buf_t o = {0};
    bput32(&o, 0x43534244u);
    bput32(&o, n_tables ? 2 : 1);
    bput32(&o, (uint32_t)nb);
    bput32(&o, b); /* the reference stores BRICK_SIZE (fileIO.cpp:28); see DESIGN */
    bput32(&o, 16);
    bput32(&o, TOT);
    if (n_tables) bput32(&o, n_tables);
    for (uint32_t t = 0; t < nt; ++t) {
        bput(&o, tf[t], 64);
        bput(&o, tc[t], 64);
    }
    buf_t r = {0};
    for (i = 0; i < nb; ++i) {
        const uint32_t s = sel ? sel[i] : 0u;
        const uint32_t t = n_tables ? ((s >> 4) & 15u) : 0u;
        r.n = 0;
        rans_encode(nibs[i], nnib[i], tf[t < nt ? t : 0], tc[t < nt ? t : 0], &r);
        bput32(&o, ids[i]);
        if (n_tables) bput32(&o, s & 0xFFu);
        bput32(&o, npal[i]);
        bput(&o, pals[i], 8 * (size_t)npal[i]);
        bput32(&o, (uint32_t)r.n);
        bput(&o, r.p, r.n);
        bput32(&o, nnib[i]);
        free(pals[i]);
        free(nibs[i]);
    }
    free(r.p);
    free(pals); free(npal); free(nibs); free(nnib); free(ids);
    free(e.pal); free(e.nib); free(lab); free(cst);
    *out = o.p;
    *out_len = o.n;
    return 0;
}

int or_encode_sel(const uint64_t* vol, size_t W, size_t H, size_t D, uint32_t b, const uint8_t* sel,
                  const uint32_t* tables, uint32_t n_tables, uint8_t** out, size_t* out_len) {
    return encode_core(vol, W, H, D, b, sel, tables, n_tables, 0, 0, NULL, NULL, out, out_len);
}

/* or_encode with the per-brick work on `threads` threads: the same steps in the
 * same order per brick (split, pyramid, encodeBrick, packing; rANS with the one
 * model of the every-512th sample), so the bytes equal or_encode's.  Phase 1
 * builds each brick's palette and nibbles, the sample histogram is summed in
 * file order, phase 2 runs each brick's rANS, and the records are written in
 * file order. */
typedef struct {
    const uint64_t* vol;
    size_t W, H, D, nby, nbz;
    uint32_t b, L;
    size_t i0, i1;
    uint64_t** pals; uint32_t* npal;
    uint8_t** nibs; uint32_t* nnib;
    uint8_t** rans; uint32_t* nrans;
    const uint32_t* freq; const uint32_t* cum;
    int phase;
} encjob_t;

static void* encode_range(void* arg) {
    encjob_t* j = (encjob_t*)arg;
    if (j->phase == 1) {
        size_t ntot = level_off(j->L);
        uint64_t* lab = (uint64_t*)malloc(ntot * 8);
        uint8_t* cst = (uint8_t*)malloc(ntot);
        enc_t e = {0};
        for (size_t i = j->i0; i < j->i1; ++i) {
            size_t bz = i % j->nbz, by = (i / j->nbz) % j->nby, bx = i / (j->nbz * j->nby);
            cut_brick(j->vol, j->W, j->H, j->D, j->b, bx, by, bz, lab + level_off(j->L - 1));
            build_pyramid(j->b, lab, cst);
            encode_brick(j->b, lab, cst, &e, 0u);
            j->pals[i] = (uint64_t*)malloc(8 * (size_t)e.np);
            memcpy(j->pals[i], e.pal, 8 * (size_t)e.np);
            j->npal[i] = e.np;
            j->nibs[i] = (uint8_t*)malloc(e.nn + 1);
            memcpy(j->nibs[i], e.nib, e.nn);
            j->nnib[i] = e.nn;
        }
        free(e.pal); free(e.nib); free(lab); free(cst);
    } else {
        buf_t r = {0};
        for (size_t i = j->i0; i < j->i1; ++i) {
            r.n = 0;
            rans_encode(j->nibs[i], j->nnib[i], j->freq, j->cum, &r);
            j->rans[i] = (uint8_t*)malloc(r.n ? r.n : 1);
            memcpy(j->rans[i], r.p, r.n);
            j->nrans[i] = (uint32_t)r.n;
        }
        free(r.p);
    }
    return NULL;
}

int or_encode_threads(const uint64_t* vol, size_t W, size_t H, size_t D, uint32_t b, uint32_t threads,
                      uint8_t** out, size_t* out_len) {
    if (b < 2 || (b & (b - 1)) || b > 1024) return -1;
    size_t nbx = (W + b - 1) / b, nby = (H + b - 1) / b, nbz = (D + b - 1) / b;
    size_t nb = nbx * nby * nbz;
    if (threads < 1) threads = 1;
    if (threads > nb) threads = nb ? (uint32_t)nb : 1u;
    encjob_t proto = {0};
    proto.vol = vol; proto.W = W; proto.H = H; proto.D = D; proto.nby = nby; proto.nbz = nbz;
    proto.b = b; proto.L = levels_of(b);
    proto.pals = (uint64_t**)calloc(nb, sizeof(void*));
    proto.npal = (uint32_t*)calloc(nb, 4);
    proto.nibs = (uint8_t**)calloc(nb, sizeof(void*));
    proto.nnib = (uint32_t*)calloc(nb, 4);
    proto.rans = (uint8_t**)calloc(nb, sizeof(void*));
    proto.nrans = (uint32_t*)calloc(nb, 4);
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * threads);
    encjob_t* jobs = (encjob_t*)malloc(sizeof(encjob_t) * threads);
    uint32_t freq[16], cum[17];
    for (int phase = 1; phase <= 2; ++phase) {
        if (phase == 2) {
            uint64_t hist[16] = {0};
            for (size_t i = 0; i < nb; i += 512) { /* brickEncoding.hpp:482 */
                for (uint32_t k = 0; k < proto.nnib[i]; ++k) hist[proto.nibs[i][k]]++;
                if (proto.nnib[i] & 1) hist[0]++;
            }
            or_build_model(hist, freq, cum);
            proto.freq = freq;
            proto.cum = cum;
        }
        for (uint32_t t = 0; t < threads; ++t) {
            jobs[t] = proto;
            jobs[t].phase = phase;
            jobs[t].i0 = nb * t / threads;
            jobs[t].i1 = nb * (t + 1) / threads;
            pthread_create(&th[t], NULL, encode_range, &jobs[t]);
        }
        for (uint32_t t = 0; t < threads; ++t) pthread_join(th[t], NULL);
    }
    buf_t o = {0};
    bput32(&o, 0x43534244u);
    bput32(&o, 1);
    bput32(&o, (uint32_t)nb);
    bput32(&o, b);
    bput32(&o, 16);
    bput32(&o, TOT);
    bput(&o, freq, 64);
    bput(&o, cum, 64);
    size_t i = 0;
    for (size_t bx = 0; bx < nbx; ++bx)
        for (size_t by = 0; by < nby; ++by)
            for (size_t bz = 0; bz < nbz; ++bz, ++i) {
                bput32(&o, or_morton3((uint32_t)bx, (uint32_t)by, (uint32_t)bz));
                bput32(&o, proto.npal[i]);
                bput(&o, proto.pals[i], 8 * (size_t)proto.npal[i]);
                bput32(&o, proto.nrans[i]);
                bput(&o, proto.rans[i], proto.nrans[i]);
                bput32(&o, proto.nnib[i]);
                free(proto.pals[i]); free(proto.nibs[i]); free(proto.rans[i]);
            }
    free(proto.pals); free(proto.npal); free(proto.nibs); free(proto.nnib); free(proto.rans); free(proto.nrans);
    free(th); free(jobs);
    *out = o.p;
    *out_len = o.n;
    return 0;
}

int or_encode_shard(const uint64_t* slab, size_t W, size_t H, size_t D, uint32_t b, uint32_t bx0, uint32_t index_base,
                    const uint64_t* hist_in, uint64_t* hist_out, uint8_t** out, size_t* out_len) {
    return encode_core(slab, W, H, D, b, NULL, NULL, 0, bx0, index_base, hist_in, hist_out, out, out_len);
}

/* ------------------------------------------------------------- decoding */
/* findSymbol (brickDecoding.cpp:126-135) with the loaded 16-entry table. */
static uint32_t find_sym(uint32_t x, const uint32_t* cum16) {
    uint32_t s = 0;
    while (s + 1 < 16 && x >= cum16[s + 1]) ++s;
    return s;
}

/* decodeRansStream + ransDecodeSymbol (brickDecoding.cpp:137-188). */
int or_rans_decode(const uint32_t* freq, const uint32_t* cum, uint32_t total_freq, const uint8_t* enc,
                   uint32_t E, uint32_t nsym, uint8_t* nib_out) {
    if (E < 4 || total_freq != TOT) return -1;
    uint32_t pos = E;
    uint32_t x = ((uint32_t)enc[E - 1] << 24) | ((uint32_t)enc[E - 2] << 16) | ((uint32_t)enc[E - 3] << 8) | enc[E - 4];
    pos -= 4;
    for (uint32_t i = 0; i < nsym; ++i) {
        uint32_t v = x % TOT;
        uint32_t s = find_sym(v, cum);
        x = freq[s] * (x / TOT) + (v - cum[s]);
        while (x < RANS_L && pos > 0) x = (x << 8) | enc[--pos];
        if (i & 1) nib_out[i >> 1] |= (uint8_t)(s & 15);
        else nib_out[i >> 1] = (uint8_t)((s & 15) << 4);
    }
    return 0;
}

/* The chain of decodeRansStream (brickDecoding.cpp:153-188) sampled: the
 * state {x, pos} before symbol k * every, for every k with k * every < nsym,
 * to states[2k], states[2k + 1] (a seek-index sidecar's contents).  Returns
 * the number of states, or -1 for a stream shorter than its header. */
int or_rans_states(const uint32_t* freq, const uint32_t* cum, const uint8_t* enc, uint32_t E, uint32_t nsym,
                   uint32_t every, uint32_t* states) {
    if (E < 4 || every == 0) return -1;
    uint32_t pos = E - 4;
    uint32_t x = ((uint32_t)enc[E - 1] << 24) | ((uint32_t)enc[E - 2] << 16) | ((uint32_t)enc[E - 3] << 8) | enc[E - 4];
    int n = 0;
    for (uint32_t i = 0; i < nsym; ++i) {
        if (i % every == 0) {
            states[2 * n] = x;
            states[2 * n + 1] = pos;
            ++n;
        }
        uint32_t v = x % TOT;
        uint32_t s = find_sym(v, cum);
        x = freq[s] * (x / TOT) + (v - cum[s]);
        while (x < RANS_L && pos > 0) x = (x << 8) | enc[--pos];
    }
    return n;
}

/* decode.wgsl:344-509 in label space (the RGBA transfer function of
 * decode.wgsl:135-172 is not applied), which equals brickDecoding.hpp:174-242
 * at full resolution.  Slot of node m at level l is m << 3(t-l)
 * (coarseNodeToOutputIndex, decode.wgsl:239-245: scaling every coordinate by
 * 2^k shifts the Morton code by 3k).  Differences from the reference, each a
 * defined outcome where the reference has none:
 *   - root stop bit set (the brick is one label): fill with palette[0]; the
 *     C++ decoder throws and the WGSL decoder leaves 8^t-1 voxels EMPTY.
 *   - a palette index past the palette is clamped to P-1 as decode.wgsl:472-485
 *     does (status bit 2); reading past the stream is skipped as
 *     decode.wgsl:449 does (status bit 1); op code 7 yields label 0 as
 *     decode.wgsl:487-489 does (status bit 4).
 * Returns the status bits (0 = clean). */
int or_decode_brick(const uint64_t* palette, uint32_t P, const uint8_t* nib, uint32_t nib_bytes,
                    uint32_t b, uint32_t t, uint64_t* out) {
    uint32_t L = levels_of(b);
    if (t >= L || P == 0) return 8;
    size_t nout = (size_t)1 << (3 * t);
    for (size_t k = 0; k < nout; ++k) out[k] = EMPTY_LABEL;
    out[0] = palette[0];
    int status = 0;
    if (nib_bytes > 0 && (nib[0] >> 4) & 1) {
        for (size_t k = 0; k < nout; ++k) out[k] = palette[0];
        return 0;
    }
    uint32_t pos = 0, hi_next = 0, ip = 0;
#define RDNIB(v)                                                              \
    do {                                                                      \
        uint8_t by_ = nib[pos];                                               \
        if (hi_next) { v = by_ >> 4; hi_next = 0; }                           \
        else { v = by_ & 15; hi_next = 1; pos++; }                            \
    } while (0)
    for (uint32_t l = 0; l < t; ++l) {
        size_t nn = (size_t)1 << (3 * l);
        uint32_t sh_p = 3 * (t - l), sh_c = 3 * (t - l - 1);
        for (size_t m = 0; m < nn; ++m) {
            size_t i = m << sh_p;
            size_t last = (8 * m + 7) << sh_c;
            if (out[last] != EMPTY_LABEL) continue;
            uint64_t parent = out[i];
            for (uint32_t c = 0; c < 8; ++c) {
                uint32_t n = (uint32_t)(8 * m + c);
                size_t j = (size_t)n << sh_c;
                if (pos >= nib_bytes) { status |= 1; continue; }
                uint32_t v, d = 0;
                RDNIB(v);
                uint32_t code = v >> 1, stop = v & 1;
                if (code == OP_PD) {
                    if (pos >= nib_bytes) { status |= 1; d = 0; }
                    else RDNIB(d);
                }
                uint64_t val;
                if (code == OP_RP) {
                    val = parent;
                } else if (code <= OP_RZ) {
                    /* getNeighborValue (decode.wgsl:247-306) */
                    uint32_t x, y, z;
                    or_demorton3(n, &x, &y, &z);
                    int cc[3] = {(int)x, (int)y, (int)z};
                    int a = (int)code - 1;
                    cc[a] += (cc[a] & 1) ? 1 : -1;
                    int maxc = (1 << (l + 1)) - 1;
                    if (cc[0] < 0 || cc[1] < 0 || cc[2] < 0 || cc[0] > maxc || cc[1] > maxc || cc[2] > maxc) {
                        val = out[(size_t)or_morton3(x >> 1, y >> 1, z >> 1) << sh_p];
                    } else {
                        uint32_t nm = or_morton3((uint32_t)cc[0], (uint32_t)cc[1], (uint32_t)cc[2]);
                        if (nm < n) val = out[(size_t)nm << sh_c];
                        else val = out[(size_t)or_morton3((uint32_t)cc[0] >> 1, (uint32_t)cc[1] >> 1, (uint32_t)cc[2] >> 1) << sh_p];
                    }
                } else if (code == OP_PA) {
                    ip += 1;
                    uint32_t k = ip >= P ? (status |= 2, P - 1) : ip;
                    val = palette[k];
                } else if (code == OP_P0) {
                    uint32_t k = ip >= P ? (status |= 2, P - 1) : ip;
                    val = palette[k];
                } else if (code == OP_PD) {
                    uint32_t k = ip - d - 1;
                    if (k >= P) { status |= 2; k = P - 1; }
                    val = palette[k];
                } else {
                    status |= 4;
                    val = 0;
                }
                out[j] = val;
                if (stop) {
                    size_t cnt = (size_t)1 << sh_c;
                    for (size_t q = 0; q < cnt; ++q) out[j + q] = val;
                }
            }
        }
    }
#undef RDNIB
    return status;
}

/* ----------------------------------------------------------- .csbd read */
typedef struct {
    uint32_t nb, b, total, version, n_tables;
    uint32_t freq[16][16], cum[16][16];
    size_t* off;  /* per brick: offset such that P is at off + 4 (after the ID, and the table word of v2) */
    uint8_t* tab; /* each brick's table */
} img_t;

static int parse_fail(img_t* I) {
    free(I->off);
    free(I->tab);
    return -1;
}

static int parse_image(const uint8_t* img, size_t len, img_t* I) {
    /* layout: fileIO.cpp:25-96 (version 1); version 2 adds the table header and a word per brick */
    if (len < 28) return -1;
    uint32_t h[7];
    memcpy(h, img, 28);
    if (h[0] != 0x43534244u || h[4] != 16 || (h[1] != 1 && h[1] != 2)) return -1;
    I->version = h[1]; I->nb = h[2]; I->b = h[3]; I->total = h[5];
    size_t o;
    if (I->version == 1) {
        if (len < 152) return -1;
        I->n_tables = 1;
        memcpy(I->freq[0], img + 24, 64);
        memcpy(I->cum[0], img + 88, 64);
        o = 152;
    } else {
        I->n_tables = h[6];
        if (I->n_tables == 0 || I->n_tables > 16 || len < 28 + 128 * (size_t)I->n_tables) return -1;
        for (uint32_t t = 0; t < I->n_tables; ++t) {
            memcpy(I->freq[t], img + 28 + 128 * t, 64);
            memcpy(I->cum[t], img + 28 + 128 * t + 64, 64);
        }
        o = 28 + 128 * (size_t)I->n_tables;
    }
    I->off = (size_t*)malloc(sizeof(size_t) * (I->nb + 1));
    I->tab = (uint8_t*)calloc(I->nb + 1, 1);
    for (uint32_t i = 0; i < I->nb; ++i) {
        uint32_t P, E;
        if (I->version == 2) {
            uint32_t s;
            if (o + 8 > len) return parse_fail(I);
            memcpy(&s, img + o + 4, 4);
            I->tab[i] = (uint8_t)((s >> 4) & 15u);
            if (I->tab[i] >= I->n_tables) return parse_fail(I);
            o += 4;
        }
        I->off[i] = o;
        if (o + 8 > len) return parse_fail(I);
        memcpy(&P, img + o + 4, 4);
        o += 8 + 8 * (size_t)P;
        if (o + 4 > len) return parse_fail(I);
        memcpy(&E, img + o, 4);
        o += 4 + E + 4;
        if (o > len) return parse_fail(I);
    }
    I->off[I->nb] = o;
    return 0;
}

int or_decode_image(const uint8_t* img, size_t len, uint32_t t, uint64_t* out, uint32_t* status) {
    img_t I;
    if (parse_image(img, len, &I)) return -1;
    size_t per = (size_t)1 << (3 * t);
    for (uint32_t i = 0; i < I.nb; ++i) {
        size_t o = I.off[i];
        uint32_t P, E, ns;
        memcpy(&P, img + o + 4, 4);
        const uint64_t* pal = (const uint64_t*)(const void*)(img + o + 8); /* may be unaligned: copy */
        uint64_t* palc = (uint64_t*)malloc(8 * (size_t)(P ? P : 1));
        memcpy(palc, pal, 8 * (size_t)P);
        o += 8 + 8 * (size_t)P;
        memcpy(&E, img + o, 4);
        const uint8_t* enc = img + o + 4;
        memcpy(&ns, img + o + 4 + E, 4);
        uint32_t nbytes = (ns + 1) / 2;
        uint8_t* nib = (uint8_t*)calloc(nbytes + 1, 1);
        int st = 0;
        if (or_rans_decode(I.freq[I.tab[i]], I.cum[I.tab[i]], I.total, enc, E, ns, nib)) st = 16;
        else st = or_decode_brick(palc, P, nib, nbytes, I.b, t, out + per * i);
        if (status) status[i] = (uint32_t)st;
        free(nib);
        free(palc);
    }
    free(I.off);
    free(I.tab);
    return (int)I.nb;
}

/* ------------------------------------------------------------ seek index */
/* The project's sidecar (no reference counterpart): replaying the decoder's
 * serial rANS pass, record (state, byte position, nibble index, palette
 * index) before every ops_per_ckpt-th op, the op count, and the first op of
 * each level.  Level l+1 holds 8 ops per level-l op with stop bit 0 (8 ops for
 * level 1 unless the root's stop bit is set); this is the decoder's skip rule
 * (decode.wgsl:430-433) stated through stop bits. */
int or_seek_index(const uint32_t* freq, const uint32_t* cum, const uint8_t* enc, uint32_t E, uint32_t nsym,
                  uint32_t P, uint32_t b, uint32_t S, uint32_t* n_ops, uint32_t* level_start,
                  uint32_t* ckpt, uint32_t max_ckpt, uint32_t* n_ckpt) {
    (void)P;
    uint32_t L = levels_of(b);
    for (int k = 0; k < 8; ++k) level_start[k] = 0;
    *n_ops = 0; *n_ckpt = 0;
    if (E < 4 || nsym == 0) return -1;
    uint32_t pos = E - 4;
    uint32_t x = ((uint32_t)enc[E - 1] << 24) | ((uint32_t)enc[E - 2] << 16) | ((uint32_t)enc[E - 3] << 8) | enc[E - 4];
    uint32_t sym_i = 0;
#define DEC(outv)                                                     \
    do {                                                              \
        uint32_t v_ = x % TOT, s_ = find_sym(v_, cum);                \
        x = freq[s_] * (x / TOT) + (v_ - cum[s_]);                    \
        while (x < RANS_L && pos > 0) x = (x << 8) | enc[--pos];      \
        outv = s_;                                                    \
        sym_i++;                                                      \
    } while (0)
    uint32_t root;
    DEC(root);
    if (root & 1) return 0; /* one-label brick: no ops */
    uint32_t ops = 0, ip = 0, need = 8, lvl = 0, active_next = 0, done_in_level = 0;
    int status = 0;
    level_start[0] = 0;
    while (lvl + 1 < L && need > 0) {
        if (ops % S == 0) {
            if (*n_ckpt < max_ckpt) {
                uint32_t* c = ckpt + 4 * (*n_ckpt);
                c[0] = x; c[1] = pos; c[2] = sym_i; c[3] = ip;
            }
            (*n_ckpt)++;
        }
        if (sym_i >= nsym) { status = 1; break; }
        uint32_t v;
        DEC(v);
        uint32_t code = v >> 1, stop = v & 1;
        if (code == OP_PD) {
            if (sym_i >= nsym) { status = 1; ops++; break; }
            uint32_t d;
            DEC(d);
            (void)d;
        }
        if (code == OP_PA) ip++;
        if (!stop) active_next++;
        ops++;
        if (++done_in_level == need) {
            lvl++;
            level_start[lvl] = ops;
            need = 8 * active_next;
            active_next = 0;
            done_in_level = 0;
        }
    }
#undef DEC
    for (uint32_t k = lvl + 1; k < 8; ++k) level_start[k] = ops;
    *n_ops = ops;
    return status;
}

/* ------------------------------------------------------------ LOD rule */
/* calculateBrickLOD (camera.js:103-137), double precision as in JS.  The
 * focal length (screenWidth / 2) / tan(fov / 2) is computed once by the caller
 * (the reference passes min(canvas.width, canvas.height), renderLoop.js:374). */
uint32_t or_brick_lod(const double* c, double brick_size, const double* cam, double focal, uint32_t max_lod) {
    double dx = c[0] - cam[0], dy = c[1] - cam[1], dz = c[2] - cam[2];
    double dist = sqrt(dx * dx + dy * dy + dz * dz);
    double d = dist > 0.1 ? dist : 0.1;
    uint32_t best = 0;
    for (uint32_t lod = 0; lod <= max_lod; ++lod) {
        double voxel = brick_size / (double)(1u << lod);
        double px = (focal * voxel) / d;
        if (px >= 1.0) best = lod;
        else break;
    }
    return best;
}

/* ------------------------------------------------------------ scalar DDA */
/* rayTrace.wgsl:565-906 in label/depth space, every float operation in the
 * shader's order, one rounding per operation (built with -ffp-contract=off).
 * Shading, shadows, gradients and compositing do not change which voxel is hit
 * first and are left out.  A voxel is visible when its label is not 0 and not
 * hidden: every other label maps to alpha >= 0.25 > 0.05 (decode.wgsl:171,
 * rayTrace.wgsl:794), label 0 and hidden labels to alpha 0. */
static float fsgn(float x) { return x > 0.f ? 1.f : (x < 0.f ? -1.f : 0.f); }
static int isgn(float x) { return (x > 0.f ? 1 : 0) + (x < 0.f ? -1 : 0); }
static int hidden_has(const uint64_t* h, uint32_t n, uint64_t v) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        uint32_t mid = (lo + hi) / 2;
        if (h[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    return lo < n && h[lo] == v;
}
static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

void or_render(const float* cam, uint32_t W, uint32_t H, float grid, uint32_t bsz, uint32_t bpa,
               const or_slot* slots, uint64_t n_slots, const uint64_t* labels, const uint64_t* hidden,
               uint32_t n_hidden, uint64_t* out_label, float* out_depth, uint32_t* miss) {
    or_render_rows(cam, W, H, 0, 1, grid, bsz, bpa, slots, n_slots, labels, hidden, n_hidden, out_label, out_depth,
                   miss, NULL);
}

void or_render_rows(const float* cam, uint32_t W, uint32_t H, uint32_t y0, uint32_t ystep, float grid, uint32_t bsz,
                    uint32_t bpa, const or_slot* slots, uint64_t n_slots, const uint64_t* labels,
                    const uint64_t* hidden, uint32_t n_hidden, uint64_t* out_label, float* out_depth, uint32_t* miss,
                    uint32_t* requests) {
    const float o[3] = {cam[0], cam[1], cam[2]};
    const float thf = cam[3];
    const float fw = (float)W, fh = (float)H, aspect = fw / fh;
    const int bs = (int)bsz;
    int lb = 0;
    while ((1 << lb) < bs) ++lb;
    const int numBricks = (int)bpa > 1 ? (int)bpa : 1;
    if (ystep == 0) ystep = 1;
    for (uint32_t py = y0; py < H; py += ystep)
        for (uint32_t px = 0; px < W; ++px) {
            const size_t pix = (size_t)py * W + px;
            out_label[pix] = 0;
            out_depth[pix] = INFINITY;
            if (miss) miss[pix] = 0;
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
            for (int a = 0; a < 3; ++a) inv[a] = fsgn(d[a]) / fmaxf(fabsf(d[a]), 1e-6f);
            /* intersectVolume (:457-471) */
            float t0[3], t1[3];
            for (int a = 0; a < 3; ++a) {
                t0[a] = (0.0f - o[a]) * inv[a];
                t1[a] = (grid - o[a]) * inv[a];
            }
            float tmin = fmaxf(fmaxf(fminf(t0[0], t1[0]), fminf(t0[1], t1[1])), fminf(t0[2], t1[2]));
            float tmax = fminf(fminf(fmaxf(t0[0], t1[0]), fmaxf(t0[1], t1[1])), fmaxf(t0[2], t1[2]));
            if (tmax < 0.0f || tmin > tmax) continue;
            const float tEnter = fmaxf(tmin, 0.0f), tExit = tmax;
            /* initBrickDDA (:519-545) */
            int brick[3], step[3];
            float btMax[3], btDelta[3];
            {
                float eps = fmaxf(tEnter * 1e-6f, 1e-5f), ts = tEnter + eps;
                for (int a = 0; a < 3; ++a) {
                    float pos = o[a] + d[a] * ts;
                    brick[a] = (int)floorf(pos) / bs;
                    step[a] = isgn(d[a]);
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
                if (brick[0] < 0 || brick[1] < 0 || brick[2] < 0 || brick[0] >= numBricks || brick[1] >= numBricks ||
                    brick[2] >= numBricks)
                    break;
                uint32_t m = or_morton3((uint32_t)brick[0], (uint32_t)brick[1], (uint32_t)brick[2]);
                int skip = m >= n_slots;
                or_slot sl = {0, 0, 0};
                if (!skip) {
                    sl = slots[m];
                    if (sl.flags & 1u) skip = 1;
                    else {
                        /* brickRequests (rayTrace.wgsl:684-686): 1 resident, 3 missing */
                        if (requests) requests[m] = (sl.flags & 2u) ? 3u : 1u;
                        if (sl.flags & 2u) {
                            skip = 1;
                            if (miss) miss[pix]++;
                        }
                    }
                }
                if (!skip) {
                    int bmin[3];
                    for (int a = 0; a < 3; ++a) bmin[a] = brick[a] * bs;
                    float tEnterBrick = fmaxf(brickEntryT, tEnter);
                    float tExitBrick = fminf(fminf(btMax[0], btMax[1]), btMax[2]);
                    float exitBias = fmaxf(tExitBrick * 1e-6f, 1e-5f);
                    tExitBrick = fmaxf(tEnterBrick, tExitBrick - exitBias);
                    /* initDDA (:473-499) */
                    int vox[3];
                    float vtMax[3], vtDelta[3];
                    float eps = fmaxf(tEnterBrick * 1e-6f, 1e-5f), ts = tEnterBrick + eps;
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
                    if (stride > 1) { /* :706-731 */
                        for (int a = 0; a < 3; ++a) {
                            int lv = (vox[a] / stride) * stride;
                            vox[a] = clampi(lv, 0, bs - 1);
                            vtDelta[a] = fabsf(inv[a]) * (float)stride;
                            float lw = (float)bmin[a] + (float)vox[a];
                            float nb = d[a] > 0.0f ? lw + (float)stride : lw;
                            vtMax[a] = (nb - o[a]) * inv[a];
                        }
                    } else {
                        for (int a = 0; a < 3; ++a) vox[a] = clampi(vox[a], 0, bs - 1);
                    }
                    int le[3], lx[3];
                    for (int a = 0; a < 3; ++a) {
                        float ve = o[a] + d[a] * tEnterBrick, vx = o[a] + d[a] * tExitBrick;
                        float lef = (ve - (float)bmin[a]) / (float)stride;
                        float lxf = (vx - (float)bmin[a]) / (float)stride;
                        le[a] = (int)floorf(lef);
                        lx[a] = (int)ceilf(lxf);
                    }
                    uint32_t maxSteps = (uint32_t)(abs(lx[0] - le[0]) + abs(lx[1] - le[1]) + abs(lx[2] - le[2])) + 128u;
                    float tcell = tEnterBrick;
                    for (uint32_t vi = 0; vi < maxSteps; ++vi) {
                        int inb = vox[0] >= 0 && vox[1] >= 0 && vox[2] >= 0 && vox[0] < bs && vox[1] < bs && vox[2] < bs;
                        if (inb) {
                            uint64_t lab;
                            if (sl.lod == 0) lab = labels[sl.offset];
                            else {
                                int sh = lb - (int)sl.lod;
                                lab = labels[sl.offset + or_morton3((uint32_t)vox[0] >> sh, (uint32_t)vox[1] >> sh,
                                                                    (uint32_t)vox[2] >> sh)];
                            }
                            if (lab != 0 && !(n_hidden && hidden_has(hidden, n_hidden, lab))) {
                                out_label[pix] = lab;
                                out_depth[pix] = tcell;
                                done = 1;
                                break;
                            }
                        }
                        /* advanceDDA (:501-517) */
                        float t;
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
                /* advanceBrickDDA (:547-563) */
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
}
