/* csv_oracle_select.c -- CPU restatement of the mode / table selector.
 * Test infrastructure only: the checker for selector.cu (statistics,
 * exhaustive choice, features) and for the selector network's forward and
 * backward passes.
 *
 * The network is restated with the device's rounding points: inputs, hidden
 * activations and backpropagated gradients are rounded to bf16 (round to
 * nearest even) where the device stores them as bf16, weights are used as bf16
 * copies of fp32 masters, and every dot product accumulates in fp32 (the
 * device's tensor cores accumulate in another order, so results agree to
 * rounding, not bit for bit).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "csv_oracle.h"

#define NF 32
#define NFP 64
#define NH 256
#define NO 32
#define NMODES 12
#define NTABLES 16

/* ---------------------------------------------------------------- statistics */
/* Per brick (split order) and mode: the 16-bin histogram of the nibbles the
 * rANS coder codes (root, ops, Pd offsets, and the pad of an odd count). */
int or_encode_stats(const uint64_t* vol, size_t W, size_t H, size_t D, uint32_t b, uint32_t* hist) {
    size_t nbx = (W + b - 1) / b, nby = (H + b - 1) / b, nbz = (D + b - 1) / b;
    size_t nb = nbx * nby * nbz;
    uint8_t* sel = (uint8_t*)malloc(nb ? nb : 1);
    for (uint32_t m = 0; m < NMODES; ++m) {
        /* encode every brick with mode m as a version-1 image and read its nibbles back */
        memset(sel, (int)m, nb ? nb : 1);
        uint8_t* img = NULL;
        size_t len = 0;
        if (or_encode_sel(vol, W, H, D, b, sel, NULL, 0, &img, &len)) {
            free(sel);
            return -1;
        }
        uint32_t freq[16], cum[16];
        memcpy(freq, img + 24, 64);
        memcpy(cum, img + 88, 64);
        size_t o = 152;
        for (size_t i = 0; i < nb; ++i) {
            uint32_t P, E, ns;
            memcpy(&P, img + o + 4, 4);
            o += 8 + 8 * (size_t)P;
            memcpy(&E, img + o, 4);
            const uint8_t* enc = img + o + 4;
            o += 4 + E;
            memcpy(&ns, img + o, 4);
            o += 4;
            uint8_t* nib = (uint8_t*)calloc(ns / 2 + 2, 1);
            or_rans_decode(freq, cum, 4096, enc, E, ns, nib);
            uint32_t* h = hist + (i * NMODES + m) * 16;
            memset(h, 0, 64);
            for (uint32_t k = 0; k < ns; ++k) h[(nib[k / 2] >> ((k & 1) ? 0 : 4)) & 15u]++;
            if (ns & 1) h[0]++;
            free(nib);
        }
        free(img);
    }
    free(sel);
    return 0;
}

/* 16.16 fixed-point bits per symbol of a table: -log2(f / 4096). */
void or_table_lengths(const uint32_t* tables, uint32_t n_tables, uint32_t* len) {
    for (uint32_t t = 0; t < n_tables; ++t)
        for (int s = 0; s < 16; ++s)
            len[16 * t + s] = (uint32_t)llround(-log2((double)tables[16 * t + s] / 4096.0) * 65536.0);
}

/* Exhaustive choice (select_kernel): fewest estimated bits, ties to the lower mode, then table. */
void or_select_exhaustive(const uint32_t* hist, uint32_t nb, const uint32_t* tables, uint32_t n_tables, uint8_t* sel,
                          uint64_t* cost) {
    uint32_t len[NTABLES * 16];
    or_table_lengths(tables, n_tables, len);
    for (uint32_t i = 0; i < nb; ++i) {
        uint64_t best = ~0ull;
        uint32_t bm = 0, bt = 0;
        for (uint32_t m = 0; m < NMODES; ++m) {
            const uint32_t* h = hist + ((size_t)i * NMODES + m) * 16;
            for (uint32_t t = 0; t < n_tables; ++t) {
                uint64_t c = 0;
                for (int s = 0; s < 16; ++s) c += (uint64_t)h[s] * len[16 * t + s];
                if (cost) cost[((size_t)i * NMODES + m) * n_tables + t] = c;
                if (c < best) {
                    best = c;
                    bm = m;
                    bt = t;
                }
            }
        }
        sel[i] = (uint8_t)(bm | (bt << 4));
    }
}

/* ---------------------------------------------------------------- features */
static uint64_t vox(const uint64_t* v, size_t W, size_t H, size_t D, size_t x, size_t y, size_t z) {
    return (x < W && y < H && z < D) ? v[x + W * (y + H * z)] : 0;
}
static uint32_t bitlen(uint32_t v) {
    uint32_t n = 0;
    while (v) {
        ++n;
        v >>= 1;
    }
    return n;
}
static int cmp_u64(const void* a, const void* b) {
    const uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
    return x < y ? -1 : (x > y);
}

/* The 8^3 sample encoded as a brick (mode 0): nibble histogram of root, ops and Pd offsets. */
static void mini_ops(const uint64_t* samp_m, uint32_t* nib) {
    uint64_t lab[585];
    uint8_t cst[585];
    memcpy(lab + 73, samp_m, 512 * 8);
    for (int m = 0; m < 512; ++m) cst[73 + m] = 1;
    const size_t off[4] = {0, 1, 9, 73};
    for (int l = 2; l >= 0; --l) {
        for (uint32_t m = 0; m < (1u << (3 * l)); ++m) {
            uint64_t v[8];
            int cc = 1;
            for (int k = 0; k < 8; ++k) {
                v[k] = lab[off[l + 1] + 8 * m + k];
                cc &= cst[off[l + 1] + 8 * m + k] != 0;
            }
            const uint64_t mj = or_majority8(v);
            int same = cc;
            for (int k = 0; k < 8; ++k) same &= v[k] == mj;
            lab[off[l] + m] = mj;
            cst[off[l] + m] = (uint8_t)same;
        }
    }
    uint64_t win[17];
    uint32_t P = 1;
    win[0] = lab[0];
    nib[(4u << 1) | (cst[0] ? 1u : 0u)]++;
    if (cst[0]) return;
    for (uint32_t l = 0; l < 3; ++l) {
        const uint32_t lc = l + 1, lvlmask = (1u << (3 * lc)) - 1u;
        for (uint32_t p = 0; p < (1u << (3 * l)); ++p) {
            if (cst[off[l] + p]) continue;
            const uint64_t plab = lab[off[l] + p];
            for (uint32_t c = 0; c < 8; ++c) {
                const uint32_t n = 8 * p + c;
                const uint64_t Lc = lab[off[lc] + n];
                const uint32_t stop = cst[off[lc] + n] ? 1u : 0u;
                uint32_t code = 7;
                if (plab == Lc) code = 0;
                for (uint32_t a = 0; a < 3 && code == 7; ++a) {
                    const uint32_t mm = (0x09249249u << a) & lvlmask, bit = 1u << a;
                    if (n & bit) {
                        if ((n & mm) == mm) continue;
                        const uint32_t N = (((n | ~mm) + bit) & mm) | (n & ~mm);
                        if (lab[off[lc - 1] + (N >> 3)] == Lc) code = 1 + a;
                    } else {
                        if ((n & mm) == 0) continue;
                        const uint32_t N = (((n & mm) - bit) & mm) | (n & ~mm);
                        if (lab[off[lc] + N] == Lc) code = 1 + a;
                    }
                }
                if (code == 7) {
                    int hit = -1;
                    for (uint32_t k = 0; k < (P < 17 ? P : 17); ++k)
                        if (win[k] == Lc) {
                            hit = (int)k;
                            break;
                        }
                    if (hit == 0) code = 5;
                    else if (hit > 0) {
                        code = 6;
                        nib[hit - 1]++;
                    } else {
                        code = 4;
                        for (int k = 16; k > 0; --k) win[k] = win[k - 1];
                        win[0] = Lc;
                        ++P;
                    }
                }
                nib[(code << 1) | stop]++;
            }
        }
    }
}

/* 32 features per brick (features_kernel in selector.cu). */
int or_brick_features(const uint64_t* vol, size_t W, size_t H, size_t D, uint32_t b, float* feat) {
    if (b < 8 || b > 64 || (b & (b - 1))) return -1;
    size_t nbx = (W + b - 1) / b, nby = (H + b - 1) / b, nbz = (D + b - 1) / b;
    size_t i = 0;
    for (size_t bx = 0; bx < nbx; ++bx)
        for (size_t by = 0; by < nby; ++by)
            for (size_t bz = 0; bz < nbz; ++bz, ++i) {
                const size_t x0 = bx * b, y0 = by * b, z0 = bz * b;
                uint64_t samp[512], sorted[512];
                const uint32_t step = b / 8, off = step / 2;
                for (uint32_t k = 0; k < 512; ++k) {
                    const uint32_t x = k & 7u, y = (k >> 3) & 7u, z = k >> 6;
                    const uint64_t v = vox(vol, W, H, D, x0 + x * step + off, y0 + y * step + off, z0 + z * step + off);
                    samp[or_morton3(x, y, z)] = v;
                    sorted[k] = v;
                }
                uint32_t c[15] = {0};
                /* rows of even y and even z, all x */
                for (uint32_t z = 0; z < b; z += 2)
                    for (uint32_t y = 0; y < b; y += 2) {
                        uint32_t run = 0;
                        for (uint32_t x = 0; x < b; ++x) {
                            const size_t gx = x0 + x, gy = y0 + y, gz = z0 + z;
                            const uint64_t v = vox(vol, W, H, D, gx, gy, gz);
                            if (x + 1 < b) c[0] += v == vox(vol, W, H, D, gx + 1, gy, gz);
                            if (y + 1 < b) c[1] += v == vox(vol, W, H, D, gx, gy + 1, gz);
                            if (z + 1 < b) c[2] += v == vox(vol, W, H, D, gx, gy, gz + 1);
                            if (x + 4 < b) c[3] += v == vox(vol, W, H, D, gx + 4, gy, gz);
                            if (y + 4 < b) c[4] += v == vox(vol, W, H, D, gx, gy + 4, gz);
                            if (z + 4 < b) c[5] += v == vox(vol, W, H, D, gx, gy, gz + 4);
                            c[6] += v == 0;
                            ++run;
                            const int last = x + 1 == b || vox(vol, W, H, D, gx + 1, gy, gz) != v;
                            if (last) {
                                const uint32_t bk = run <= 1    ? 0
                                                    : run == 2  ? 1
                                                    : run <= 4  ? 2
                                                    : run <= 8  ? 3
                                                    : run <= 16 ? 4
                                                    : run <= 32 ? 5
                                                                : 6;
                                c[7 + bk]++;
                                c[14]++;
                                run = 0;
                            }
                        }
                    }
                qsort(sorted, 512, 8, cmp_u64);
                uint32_t distinct = 1;
                for (int k = 1; k < 512; ++k) distinct += sorted[k] != sorted[k - 1];
                uint32_t nib[16] = {0};
                mini_ops(samp, nib);
                float* f = feat + i * NF;
                const float hb = (float)(b / 2), fb = (float)b;
                const float px1 = hb * hb * (fb - 1.0f), px4 = hb * hb * (fb - 4.0f);
                const float pyz1 = hb * hb * fb, pyz4 = (float)((b - 4) / 2) * hb * fb;
                f[0] = (float)bitlen(distinct) / 10.0f;
                f[1] = (float)c[0] / px1;
                f[2] = (float)c[1] / pyz1;
                f[3] = (float)c[2] / pyz1;
                f[4] = (float)c[3] / px4;
                f[5] = (float)c[4] / pyz4;
                f[6] = (float)c[5] / pyz4;
                f[7] = (float)c[6] / (hb * hb * fb);
                const float runs = (float)(c[14] ? c[14] : 1u);
                for (int k = 0; k < 7; ++k) f[8 + k] = (float)c[7 + k] / runs;
                f[15] = (float)bitlen(c[14]) / 20.0f;
                uint32_t tot = 0;
                for (int k = 0; k < 16; ++k) tot += nib[k];
                for (int k = 0; k < 16; ++k) f[16 + k] = (float)nib[k] / (float)(tot ? tot : 1u);
            }
    return 0;
}

/* ---------------------------------------------------------------- network */
static float bf16r(float x) {
    uint32_t u;
    memcpy(&u, &x, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return x; /* inf / nan */
    u += 0x7fffu + ((u >> 16) & 1u);
    u &= 0xffff0000u;
    memcpy(&x, &u, 4);
    return x;
}

enum { P_W1 = 0, P_B1 = P_W1 + NH * NFP, P_W2 = P_B1 + NH, P_B2 = P_W2 + NH * NH, P_W3 = P_B2 + NH,
       P_B3 = P_W3 + NO * NH, P_N = P_B3 + NO };

typedef struct {
    float *X, *H1, *H2, *Z; /* rows x {64, 256, 256, 32}; X, H1, H2 hold bf16 values */
} acts_t;

static void forward(const float* P, const float* feat, uint32_t n, acts_t* A) {
    float* W1 = (float*)malloc(sizeof(float) * NH * NFP);
    float* W2 = (float*)malloc(sizeof(float) * NH * NH);
    float* W3 = (float*)malloc(sizeof(float) * NO * NH);
    for (int k = 0; k < NH * NFP; ++k) W1[k] = bf16r(P[P_W1 + k]);
    for (int k = 0; k < NH * NH; ++k) W2[k] = bf16r(P[P_W2 + k]);
    for (int k = 0; k < NO * NH; ++k) W3[k] = bf16r(P[P_W3 + k]);
    for (uint32_t r = 0; r < n; ++r) {
        float* x = A->X + (size_t)r * NFP;
        for (int c = 0; c < NFP; ++c) x[c] = c < NF ? bf16r(feat[(size_t)r * NF + c]) : 0.0f;
        float* h1 = A->H1 + (size_t)r * NH;
        for (int o = 0; o < NH; ++o) {
            float s = 0.0f;
            for (int c = 0; c < NFP; ++c) s += x[c] * W1[o * NFP + c];
            s += P[P_B1 + o];
            h1[o] = bf16r(s > 0.0f ? s : 0.0f);
        }
        float* h2 = A->H2 + (size_t)r * NH;
        for (int o = 0; o < NH; ++o) {
            float s = 0.0f;
            for (int c = 0; c < NH; ++c) s += h1[c] * W2[o * NH + c];
            s += P[P_B2 + o];
            h2[o] = bf16r(s > 0.0f ? s : 0.0f);
        }
        float* z = A->Z + (size_t)r * NO;
        for (int o = 0; o < NO; ++o) {
            float s = 0.0f;
            for (int c = 0; c < NH; ++c) s += h2[c] * W3[o * NH + c];
            z[o] = s + P[P_B3 + o];
        }
    }
    free(W1);
    free(W2);
    free(W3);
}

/* Logits (n x 32). */
void or_mlp_forward(const float* params, const float* feat, uint32_t n, float* logits) {
    acts_t A;
    A.X = (float*)malloc(sizeof(float) * n * NFP);
    A.H1 = (float*)malloc(sizeof(float) * n * NH);
    A.H2 = (float*)malloc(sizeof(float) * n * NH);
    A.Z = logits;
    forward(params, feat, n, &A);
    free(A.X);
    free(A.H1);
    free(A.H2);
}

/* Mean cross-entropy of both heads and its gradient (CSV_MLP_PARAMS floats). */
float or_mlp_grad(const float* P, const float* feat, const uint8_t* label, uint32_t n, float* G) {
    acts_t A;
    A.X = (float*)malloc(sizeof(float) * n * NFP);
    A.H1 = (float*)malloc(sizeof(float) * n * NH);
    A.H2 = (float*)malloc(sizeof(float) * n * NH);
    A.Z = (float*)malloc(sizeof(float) * n * NO);
    forward(P, feat, n, &A);
    float* dZ = (float*)calloc((size_t)n * NO, sizeof(float));
    float* dH2 = (float*)calloc((size_t)n * NH, sizeof(float));
    float* dH1 = (float*)calloc((size_t)n * NH, sizeof(float));
    float loss = 0.0f;
    for (uint32_t r = 0; r < n; ++r) {
        const float* z = A.Z + (size_t)r * NO;
        const uint32_t y[2] = {label[r] & 15u, (uint32_t)(label[r] >> 4)};
        for (int head = 0; head < 2; ++head) {
            const int b0 = head ? NMODES : 0, cnt = head ? NTABLES : NMODES;
            float mx = -INFINITY;
            for (int k = 0; k < cnt; ++k) mx = fmaxf(mx, z[b0 + k]);
            float se = 0.0f;
            for (int k = 0; k < cnt; ++k) se += expf(z[b0 + k] - mx);
            for (int k = 0; k < cnt; ++k)
                dZ[(size_t)r * NO + b0 + k] =
                    bf16r((expf(z[b0 + k] - mx) / se - ((uint32_t)k == y[head] ? 1.0f : 0.0f)) / (float)n);
            loss += (logf(se) + mx - z[b0 + y[head]]) / (float)n;
        }
    }
    float* W2 = (float*)malloc(sizeof(float) * NH * NH);
    float* W3 = (float*)malloc(sizeof(float) * NO * NH);
    for (int k = 0; k < NH * NH; ++k) W2[k] = bf16r(P[P_W2 + k]);
    for (int k = 0; k < NO * NH; ++k) W3[k] = bf16r(P[P_W3 + k]);
    for (uint32_t r = 0; r < n; ++r)
        for (int c = 0; c < NH; ++c) {
            float s = 0.0f;
            for (int o = 0; o < NO; ++o) s += dZ[(size_t)r * NO + o] * W3[o * NH + c];
            dH2[(size_t)r * NH + c] = A.H2[(size_t)r * NH + c] > 0.0f ? bf16r(s) : 0.0f;
        }
    for (uint32_t r = 0; r < n; ++r)
        for (int c = 0; c < NH; ++c) {
            float s = 0.0f;
            for (int o = 0; o < NH; ++o) s += dH2[(size_t)r * NH + o] * W2[o * NH + c];
            dH1[(size_t)r * NH + c] = A.H1[(size_t)r * NH + c] > 0.0f ? bf16r(s) : 0.0f;
        }
    memset(G, 0, sizeof(float) * P_N);
    for (int o = 0; o < NO; ++o)
        for (int c = 0; c < NH; ++c) {
            float s = 0.0f;
            for (uint32_t r = 0; r < n; ++r) s += dZ[(size_t)r * NO + o] * A.H2[(size_t)r * NH + c];
            G[P_W3 + o * NH + c] = s;
        }
    for (int o = 0; o < NH; ++o)
        for (int c = 0; c < NH; ++c) {
            float s = 0.0f;
            for (uint32_t r = 0; r < n; ++r) s += dH2[(size_t)r * NH + o] * A.H1[(size_t)r * NH + c];
            G[P_W2 + o * NH + c] = s;
        }
    for (int o = 0; o < NH; ++o)
        for (int c = 0; c < NFP; ++c) {
            float s = 0.0f;
            for (uint32_t r = 0; r < n; ++r) s += dH1[(size_t)r * NH + o] * A.X[(size_t)r * NFP + c];
            G[P_W1 + o * NFP + c] = s;
        }
    for (uint32_t r = 0; r < n; ++r) {
        for (int o = 0; o < NO; ++o) G[P_B3 + o] += dZ[(size_t)r * NO + o];
        for (int o = 0; o < NH; ++o) G[P_B2 + o] += dH2[(size_t)r * NH + o];
        for (int o = 0; o < NH; ++o) G[P_B1 + o] += dH1[(size_t)r * NH + o];
    }
    free(W2);
    free(W3);
    free(dZ);
    free(dH2);
    free(dH1);
    free(A.X);
    free(A.H1);
    free(A.H2);
    free(A.Z);
    return loss;
}
