/* csv_oracle_synth.c -- CPU restatement of the seeded synthetic volumes of the
 * native library (csv_synth_volume), and a multi-threaded restatement of the
 * encoder for large volumes.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle).  Used by tests/ and by bench.py's
 * reference arm, which must build its input images without the product
 * library: or_synth_volume gives the same volume as the device generator (the
 * same random draws in the same order, every float operation rounded on its own
 * as the device kernels do), and or_encode_threads gives the same bytes as
 * or_encode (and so as the reference encoder, compressDataset<b>,
 * brickEncoding.hpp:466-531), with the per-brick work spread over threads.
 */
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#include "csv_oracle.h"

/* ------------------------------------------------------------ generator */
typedef struct { uint64_t s; } rng_t;
static uint64_t rng_next(rng_t* r) { /* splitmix64 */
    uint64_t z = (r->s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static double rng_uniform(rng_t* r) { return (rng_next(r) >> 11) * (1.0 / 9007199254740992.0); }
static uint64_t rng_label(rng_t* r) {
    uint64_t v;
    do { v = rng_next(r); } while (v == 0 || v == UINT64_MAX);
    return v;
}

typedef struct { float x, y, z; int idx; } seed_t;

typedef struct {
    float cell;
    int gx, gy, gz;
    uint32_t* start; /* gx*gy*gz + 1 */
    seed_t* pts;
} grid_t;

static int maxi(int a, int b) { return a > b ? a : b; }
static int mini(int a, int b) { return a < b ? a : b; }

static void bucket_seeds(const float* xyz, uint32_t n, uint32_t W, uint32_t H, uint32_t D, grid_t* g) {
    double vol = (double)W * H * D;
    double c = cbrt(vol / (n > 1 ? n : 1));
    g->cell = (float)(c > 1.0 ? c : 1.0);
    g->gx = maxi(1, (int)ceil(W / g->cell));
    g->gy = maxi(1, (int)ceil(H / g->cell));
    g->gz = maxi(1, (int)ceil(D / g->cell));
    size_t nbk = (size_t)g->gx * g->gy * g->gz;
    uint32_t* cnt = (uint32_t*)calloc(nbk + 1, 4);
    uint32_t* bk = (uint32_t*)malloc((size_t)n * 4 + 4);
    for (uint32_t i = 0; i < n; ++i) {
        int bx = mini(g->gx - 1, (int)(xyz[3 * i] / g->cell));
        int by = mini(g->gy - 1, (int)(xyz[3 * i + 1] / g->cell));
        int bz = mini(g->gz - 1, (int)(xyz[3 * i + 2] / g->cell));
        bk[i] = (uint32_t)(bx + (size_t)g->gx * (by + (size_t)g->gy * bz));
        cnt[bk[i] + 1]++;
    }
    for (size_t k = 0; k < nbk; ++k) cnt[k + 1] += cnt[k];
    g->start = cnt;
    g->pts = (seed_t*)malloc(sizeof(seed_t) * (n ? n : 1));
    uint32_t* fill = (uint32_t*)malloc(nbk * 4);
    memcpy(fill, cnt, nbk * 4);
    for (uint32_t i = 0; i < n; ++i) { /* seeds keep index order inside a bucket */
        seed_t p = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], (int)i};
        g->pts[fill[bk[i]]++] = p;
    }
    free(fill);
    free(bk);
}

typedef struct {
    float ax, ay, az, bx, by, bz, r;
    uint32_t tube;
    int lo[3], hi[3];
} piece_t;

typedef struct {
    uint64_t* vol;
    const grid_t* g;
    const uint64_t* ids;
    const uint8_t* zero_cell; /* NULL: none */
    uint32_t W, H, D;
    float nx, ny, nz, thr;
    uint32_t* owner;
    const piece_t* pieces;
    size_t n_pieces;
    const uint64_t* tube_ids;
    uint32_t z0, z1; /* this thread's z range */
} synth_job_t;

static float dot3(float ax, float ay, float az, float bx, float by, float bz) {
    float a = ax * bx, b = ay * by, c = az * bz;
    return (a + b) + c;
}

/* voronoi_kernel: nearest seed to the voxel centre (ties -> lower seed index),
 * bucket shells searched outward until no unsearched bucket can hold a closer
 * seed; the zero slab or zero cells. */
static void* voronoi_rows(void* arg) {
    synth_job_t* j = (synth_job_t*)arg;
    const grid_t* g = j->g;
    for (uint32_t z = j->z0; z < j->z1; ++z)
        for (uint32_t y = 0; y < j->H; ++y)
            for (uint32_t x = 0; x < j->W; ++x) {
                float px = x + 0.5f, py = y + 0.5f, pz = z + 0.5f;
                int bx = mini(g->gx - 1, (int)(px / g->cell)), by = mini(g->gy - 1, (int)(py / g->cell)),
                    bz = mini(g->gz - 1, (int)(pz / g->cell));
                float best = INFINITY;
                int besti = 0x7fffffff;
                int maxr = maxi(g->gx, maxi(g->gy, g->gz));
                for (int rad = 0; rad <= maxr; ++rad) {
                    for (int dz = -rad; dz <= rad; ++dz) {
                        int cz = bz + dz;
                        if (cz < 0 || cz >= g->gz) continue;
                        for (int dy = -rad; dy <= rad; ++dy) {
                            int cy = by + dy;
                            if (cy < 0 || cy >= g->gy) continue;
                            int face = (abs(dz) == rad) || (abs(dy) == rad);
                            for (int dx = -rad; dx <= rad; dx += (face ? 1 : (rad > 0 ? 2 * rad : 1))) {
                                int cx = bx + dx;
                                if (cx < 0 || cx >= g->gx) continue;
                                uint32_t k = (uint32_t)(cx + g->gx * (cy + g->gy * cz));
                                for (uint32_t s = g->start[k]; s < g->start[k + 1]; ++s) {
                                    seed_t q = g->pts[s];
                                    float ddx = q.x - px, ddy = q.y - py, ddz = q.z - pz;
                                    float d2 = (ddx * ddx) + (ddy * ddy);
                                    d2 = d2 + (ddz * ddz);
                                    if (d2 < best || (d2 == best && q.idx < besti)) { best = d2; besti = q.idx; }
                                }
                            }
                        }
                    }
                    float reach = rad * g->cell;
                    if (besti != 0x7fffffff && best < reach * reach) break;
                }
                uint64_t lab = j->ids[besti];
                if (j->zero_cell && j->zero_cell[besti]) lab = 0;
                if (dot3(px, py, pz, j->nx, j->ny, j->nz) >= j->thr) lab = 0;
                j->vol[x + (uint64_t)j->W * (y + (uint64_t)j->H * z)] = lab;
            }
    return NULL;
}

/* tube_kernel + combine_kernel for the z range of this thread: a voxel within
 * r of a piece takes the highest tube number covering it. */
static void* tube_rows(void* arg) {
    synth_job_t* j = (synth_job_t*)arg;
    for (size_t k = 0; k < j->n_pieces; ++k) {
        const piece_t* p = &j->pieces[k];
        int ex = p->hi[0] - p->lo[0], ey = p->hi[1] - p->lo[1], ez = p->hi[2] - p->lo[2];
        if (ex <= 0 || ey <= 0 || ez <= 0) continue;
        int zlo = maxi(p->lo[2], (int)j->z0), zhi = mini(p->hi[2], (int)j->z1);
        if (zlo >= zhi) continue;
        float abx = p->bx - p->ax, aby = p->by - p->ay, abz = p->bz - p->az;
        float den = fmaxf(dot3(abx, aby, abz, abx, aby, abz), 1e-12f);
        float r2 = p->r * p->r;
        for (int z = zlo; z < zhi; ++z)
            for (int y = p->lo[1]; y < p->hi[1]; ++y)
                for (int x = p->lo[0]; x < p->hi[0]; ++x) {
                    float qx = (x + 0.5f) - p->ax, qy = (y + 0.5f) - p->ay, qz = (z + 0.5f) - p->az;
                    float s = dot3(qx, qy, qz, abx, aby, abz) / den;
                    s = fminf(1.f, fmaxf(0.f, s));
                    float dx = qx - s * abx, dy = qy - s * aby, dz = qz - s * abz;
                    if (dot3(dx, dy, dz, dx, dy, dz) < r2) {
                        uint32_t* o = j->owner + x + (uint64_t)j->W * (y + (uint64_t)j->H * z);
                        if (*o < p->tube + 1) *o = p->tube + 1;
                    }
                }
    }
    uint64_t a = (uint64_t)j->W * j->H * j->z0, b = (uint64_t)j->W * j->H * j->z1;
    for (uint64_t i = a; i < b; ++i)
        if (j->owner[i]) j->vol[i] = j->tube_ids[j->owner[i] - 1];
    return NULL;
}

static int cmp_double(const void* a, const void* b) {
    double x = *(const double*)a, y = *(const double*)b;
    return (x > y) - (x < y);
}

static void run_threads(void* (*fn)(void*), synth_job_t* proto, uint32_t D, uint32_t threads) {
    if (threads < 1) threads = 1;
    if (threads > D) threads = D ? D : 1;
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * threads);
    synth_job_t* jobs = (synth_job_t*)malloc(sizeof(synth_job_t) * threads);
    for (uint32_t t = 0; t < threads; ++t) {
        jobs[t] = *proto;
        jobs[t].z0 = (uint32_t)((uint64_t)D * t / threads);
        jobs[t].z1 = (uint32_t)((uint64_t)D * (t + 1) / threads);
        pthread_create(&th[t], NULL, fn, &jobs[t]);
    }
    for (uint32_t t = 0; t < threads; ++t) pthread_join(th[t], NULL);
    free(jobs);
    free(th);
}

/* csv_synth_volume (the native library's workload generator), kinds 0/1/2:
 * 0 Voronoi + zero slab; 1 tubes over Voronoi with zero cells; 2 x < W/2
 * smooth Voronoi, x >= W/2 tubes over the Voronoi background. */
int or_synth_volume(uint64_t* vol, uint32_t W, uint32_t H, uint32_t D, int kind, uint32_t n_cells, uint32_t n_tubes,
                    float r_min, float r_max, float zero_frac, uint64_t seed, uint32_t threads) {
    rng_t rng = {seed * 0x2545F4914F6CDD1Dull + 17};
    if (n_cells == 0) n_cells = 1;
    float* xyz = (float*)malloc(sizeof(float) * 3 * (size_t)n_cells);
    uint64_t* ids = (uint64_t*)malloc(8 * (size_t)n_cells);
    uint8_t* zero_cell = (uint8_t*)calloc(n_cells, 1);
    if (!xyz || !ids || !zero_cell) return -1;
    for (uint32_t i = 0; i < n_cells; ++i) {
        xyz[3 * i] = (float)(rng_uniform(&rng) * W);
        xyz[3 * i + 1] = (float)(rng_uniform(&rng) * H);
        xyz[3 * i + 2] = (float)(rng_uniform(&rng) * D);
        ids[i] = rng_label(&rng);
    }
    grid_t g;
    bucket_seeds(xyz, n_cells, W, H, D, &g);
    synth_job_t J;
    memset(&J, 0, sizeof J);
    J.vol = vol; J.g = &g; J.ids = ids; J.W = W; J.H = H; J.D = D;
    J.thr = INFINITY;
    if (kind == 0 && zero_frac > 0) {
        double nx = rng_uniform(&rng) - 0.5, ny = rng_uniform(&rng) - 0.5, nz = rng_uniform(&rng) - 0.5;
        double nn = sqrt(nx * nx + ny * ny + nz * nz) + 1e-12;
        nx /= nn; ny /= nn; nz /= nn;
        double* d = (double*)malloc(sizeof(double) * 65536);
        for (int k = 0; k < 65536; ++k) {
            double a = rng_uniform(&rng) * W;
            double b = rng_uniform(&rng) * H;
            double c = rng_uniform(&rng) * D;
            d[k] = a * nx + b * ny + c * nz;
        }
        qsort(d, 65536, sizeof(double), cmp_double);
        size_t q = (size_t)((1.0 - zero_frac) * (65536 - 1));
        J.nx = (float)nx; J.ny = (float)ny; J.nz = (float)nz;
        J.thr = (float)d[q];
        free(d);
    } else if (kind != 0 && zero_frac > 0) {
        for (uint32_t i = 0; i < n_cells; ++i) zero_cell[i] = rng_uniform(&rng) < zero_frac ? 1 : 0;
    }
    J.zero_cell = kind != 0 ? zero_cell : NULL;
    run_threads(voronoi_rows, &J, D, threads);

    int rc = 0;
    if (kind != 0 && n_tubes > 0) {
        size_t cap = 1024, np = 0;
        piece_t* pieces = (piece_t*)malloc(sizeof(piece_t) * cap);
        uint64_t* tids = (uint64_t*)malloc(8 * (size_t)n_tubes);
        float xlo = (kind == 2) ? W * 0.5f : 0.f;
        for (uint32_t t = 0; t < n_tubes; ++t) {
            float c[4][3];
            for (int k = 0; k < 4; ++k) {
                c[k][0] = (float)(xlo + rng_uniform(&rng) * (W - xlo));
                c[k][1] = (float)(rng_uniform(&rng) * H);
                c[k][2] = (float)(rng_uniform(&rng) * D);
            }
            float r = (float)(r_min + rng_uniform(&rng) * (r_max - r_min));
            tids[t] = rng_label(&rng);
            /* Catmull-Rom segment between c[1] and c[2] */
            float len = sqrtf((c[2][0] - c[1][0]) * (c[2][0] - c[1][0]) + (c[2][1] - c[1][1]) * (c[2][1] - c[1][1]) +
                              (c[2][2] - c[1][2]) * (c[2][2] - c[1][2]));
            int ns = maxi(2, (int)(len / fmaxf(1.f, r)) + 2);
            float prev[3] = {0, 0, 0};
            for (int k = 0; k <= ns; ++k) {
                float u = (float)k / ns, u2 = u * u, u3 = u2 * u;
                float p[3];
                for (int d = 0; d < 3; ++d)
                    p[d] = 0.5f * (2 * c[1][d] + (-c[0][d] + c[2][d]) * u +
                                   (2 * c[0][d] - 5 * c[1][d] + 4 * c[2][d] - c[3][d]) * u2 +
                                   (-c[0][d] + 3 * c[1][d] - 3 * c[2][d] + c[3][d]) * u3);
                if (k > 0) {
                    piece_t pc;
                    pc.ax = prev[0]; pc.ay = prev[1]; pc.az = prev[2];
                    pc.bx = p[0]; pc.by = p[1]; pc.bz = p[2];
                    pc.r = r;
                    pc.tube = t;
                    uint32_t ext[3] = {W, H, D};
                    for (int d = 0; d < 3; ++d) {
                        float lo = fminf(prev[d], p[d]) - r, hi = fmaxf(prev[d], p[d]) + r;
                        pc.lo[d] = maxi(0, (int)floorf(lo));
                        if (d == 0 && kind == 2) pc.lo[d] = maxi(pc.lo[d], (int)(W / 2));
                        pc.hi[d] = mini((int)ext[d], (int)ceilf(hi) + 1);
                    }
                    if (np == cap) {
                        cap *= 2;
                        pieces = (piece_t*)realloc(pieces, sizeof(piece_t) * cap);
                    }
                    pieces[np++] = pc;
                }
                prev[0] = p[0]; prev[1] = p[1]; prev[2] = p[2];
            }
        }
        uint32_t* owner = (uint32_t*)calloc((size_t)W * H * D, 4);
        if (!owner) {
            rc = -1;
        } else {
            J.owner = owner;
            J.pieces = pieces;
            J.n_pieces = np;
            J.tube_ids = tids;
            run_threads(tube_rows, &J, D, threads);
            free(owner);
        }
        free(pieces);
        free(tids);
    }
    free(g.start);
    free(g.pts);
    free(xyz);
    free(ids);
    free(zero_cell);
    return rc;
}
