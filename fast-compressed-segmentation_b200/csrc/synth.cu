// synth.cu -- seeded synthetic label volumes on the device (workload generator).
//
// The reference's input is a downloaded MICrONS segmentation (dataset/
// dataset_downloader.py), unavailable here; these volumes stand in for it with
// the same dtype and layout (uint64, x fastest, brick.hpp:183).  All random
// choices are made on the host from one 64-bit seed (splitmix64), so a volume
// is a pure function of its arguments.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "csv_internal.h"

namespace csv {

namespace {

struct Rng {
    uint64_t s;
    uint64_t next() {  // splitmix64
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
    uint64_t label() {  // uniform in [1, 2^64 - 2]
        uint64_t v;
        do { v = next(); } while (v == 0 || v == UINT64_MAX);
        return v;
    }
};

struct Grid {
    float cell;                 // bucket edge in voxels
    int gx, gy, gz;             // buckets per axis
    std::vector<uint32_t> start;  // gx*gy*gz + 1
    std::vector<float4> pts;    // x, y, z, bit-cast seed index
};

Grid bucket_seeds(const std::vector<float>& xyz, uint32_t n, uint32_t W, uint32_t H, uint32_t D) {
    Grid g;
    double vol = (double)W * H * D;
    g.cell = (float)std::max(1.0, cbrt(vol / std::max<uint32_t>(n, 1)));
    g.gx = std::max(1, (int)ceil(W / g.cell));
    g.gy = std::max(1, (int)ceil(H / g.cell));
    g.gz = std::max(1, (int)ceil(D / g.cell));
    size_t nbk = (size_t)g.gx * g.gy * g.gz;
    std::vector<uint32_t> cnt(nbk + 1, 0), bk(n);
    for (uint32_t i = 0; i < n; ++i) {
        int bx = std::min(g.gx - 1, (int)(xyz[3 * i] / g.cell));
        int by = std::min(g.gy - 1, (int)(xyz[3 * i + 1] / g.cell));
        int bz = std::min(g.gz - 1, (int)(xyz[3 * i + 2] / g.cell));
        bk[i] = (uint32_t)(bx + (size_t)g.gx * (by + (size_t)g.gy * bz));
        cnt[bk[i] + 1]++;
    }
    for (size_t k = 0; k < nbk; ++k) cnt[k + 1] += cnt[k];
    g.start = cnt;
    g.pts.resize(n);
    std::vector<uint32_t> fill(cnt.begin(), cnt.end() - 1);
    for (uint32_t i = 0; i < n; ++i) {  // seeds keep index order inside a bucket
        float4 p;
        p.x = xyz[3 * i];
        p.y = xyz[3 * i + 1];
        p.z = xyz[3 * i + 2];
        int iv = (int)i;
        memcpy(&p.w, &iv, 4);
        g.pts[fill[bk[i]]++] = p;
    }
    return g;
}

struct VoronoiArgs {
    const uint32_t* start;
    const float4* pts;
    const uint64_t* ids;
    float cell;
    int gx, gy, gz;
    uint32_t W, H, D;
    uint32_t x0, x1;             // x range written [x0, x1)
    float nx, ny, nz, thr;       // zero slab: p . n >= thr -> 0 (thr = +inf: none)
    const uint8_t* zero_cell;    // per seed: 1 -> label 0 (may be null)
};

// Nearest seed to the voxel centre (ties -> lower seed index), searching bucket
// shells outward until no unsearched bucket can hold a closer seed.
__global__ void voronoi_kernel(uint64_t* __restrict__ vol, VoronoiArgs a) {
    uint64_t n = (uint64_t)(a.x1 - a.x0) * a.H * a.D;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t xs = a.x1 - a.x0;
        uint32_t x = a.x0 + (uint32_t)(i % xs);
        uint64_t r = i / xs;
        uint32_t y = (uint32_t)(r % a.H), z = (uint32_t)(r / a.H);
        float px = x + 0.5f, py = y + 0.5f, pz = z + 0.5f;
        int bx = min(a.gx - 1, (int)(px / a.cell)), by = min(a.gy - 1, (int)(py / a.cell)),
            bz = min(a.gz - 1, (int)(pz / a.cell));
        float best = INFINITY;
        int besti = 0x7fffffff;
        int maxr = max(a.gx, max(a.gy, a.gz));
        for (int rad = 0; rad <= maxr; ++rad) {
            for (int dz = -rad; dz <= rad; ++dz) {
                int cz = bz + dz;
                if (cz < 0 || cz >= a.gz) continue;
                for (int dy = -rad; dy <= rad; ++dy) {
                    int cy = by + dy;
                    if (cy < 0 || cy >= a.gy) continue;
                    bool face = (abs(dz) == rad) || (abs(dy) == rad);
                    for (int dx = -rad; dx <= rad; dx += (face ? 1 : (rad > 0 ? 2 * rad : 1))) {
                        int cx = bx + dx;
                        if (cx < 0 || cx >= a.gx) continue;
                        uint32_t k = (uint32_t)(cx + a.gx * (cy + a.gy * cz));
                        for (uint32_t s = a.start[k]; s < a.start[k + 1]; ++s) {
                            float4 q = a.pts[s];
                            float ddx = q.x - px, ddy = q.y - py, ddz = q.z - pz;
                            float d2 = __fmul_rn(ddx, ddx) + __fmul_rn(ddy, ddy);
                            d2 = __fadd_rn(d2, __fmul_rn(ddz, ddz));
                            int qi = __float_as_int(q.w);
                            if (d2 < best || (d2 == best && qi < besti)) { best = d2; besti = qi; }
                        }
                    }
                }
            }
            // every bucket outside the searched shell is at least rad*cell away
            float reach = rad * a.cell;
            if (besti != 0x7fffffff && best < reach * reach) break;
        }
        uint64_t lab = a.ids[besti];
        if (a.zero_cell && a.zero_cell[besti]) lab = 0;
        if (__fadd_rn(__fadd_rn(__fmul_rn(px, a.nx), __fmul_rn(py, a.ny)), __fmul_rn(pz, a.nz)) >= a.thr) lab = 0;
        vol[x + (uint64_t)a.W * (y + (uint64_t)a.H * z)] = lab;
    }
}

struct Piece {
    float ax, ay, az, bx, by, bz, r;
    uint32_t tube;
    int lo[3], hi[3];
};

__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
    return __fadd_rn(__fadd_rn(__fmul_rn(ax, bx), __fmul_rn(ay, by)), __fmul_rn(az, bz));
}

// One block per straight piece of a tube: voxels within r of the piece get the
// highest tube number that covers them (atomicMax makes overlaps deterministic).
__global__ void tube_kernel(uint32_t* __restrict__ owner, const Piece* __restrict__ pieces, uint32_t W, uint32_t H) {
    Piece p = pieces[blockIdx.x];
    int ex = p.hi[0] - p.lo[0], ey = p.hi[1] - p.lo[1], ez = p.hi[2] - p.lo[2];
    if (ex <= 0 || ey <= 0 || ez <= 0) return;
    // every product and sum rounded on its own (no contracted multiply-adds), so that
    // a CPU restatement with the same operation order gives the same volume
    float abx = p.bx - p.ax, aby = p.by - p.ay, abz = p.bz - p.az;
    float den = fmaxf(dot3(abx, aby, abz, abx, aby, abz), 1e-12f);
    float r2 = __fmul_rn(p.r, p.r);
    uint32_t n = (uint32_t)ex * ey * ez;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        int x = p.lo[0] + (int)(i % ex), y = p.lo[1] + (int)((i / ex) % ey), z = p.lo[2] + (int)(i / (ex * ey));
        float qx = (x + 0.5f) - p.ax, qy = (y + 0.5f) - p.ay, qz = (z + 0.5f) - p.az;
        float s = __fdiv_rn(dot3(qx, qy, qz, abx, aby, abz), den);
        s = fminf(1.f, fmaxf(0.f, s));
        float dx = __fsub_rn(qx, __fmul_rn(s, abx)), dy = __fsub_rn(qy, __fmul_rn(s, aby)),
              dz = __fsub_rn(qz, __fmul_rn(s, abz));
        if (dot3(dx, dy, dz, dx, dy, dz) < r2) atomicMax(owner + x + (uint64_t)W * (y + (uint64_t)H * z), p.tube + 1);
    }
}

__global__ void combine_kernel(uint64_t* __restrict__ vol, const uint32_t* __restrict__ owner,
                               const uint64_t* __restrict__ tube_ids, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t o = owner[i];
        if (o) vol[i] = tube_ids[o - 1];
    }
}

template <class T>
cudaError_t upload(T** d, const std::vector<T>& h) {
    cudaError_t e = cudaMalloc(d, std::max<size_t>(1, h.size()) * sizeof(T));
    if (e != cudaSuccess) return e;
    if (!h.empty()) e = cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
    return e;
}

}  // namespace

// kind 0: Voronoi + zero slab; kind 1: tubes over Voronoi with zero cells;
// kind 2: x < W/2 smooth Voronoi (n_cells), x >= W/2 dense tubes (n_tubes)
// over a Voronoi background of n_cells cells.
cudaError_t synth_volume(uint64_t* d_vol, uint32_t W, uint32_t H, uint32_t D, int kind, uint32_t n_cells,
                         uint32_t n_tubes, float r_min, float r_max, float zero_frac, uint64_t seed,
                         cudaStream_t st) {
    Rng rng{seed * 0x2545F4914F6CDD1Dull + 17};
    if (n_cells == 0) n_cells = 1;
    std::vector<float> xyz(3 * (size_t)n_cells);
    std::vector<uint64_t> ids(n_cells);
    for (uint32_t i = 0; i < n_cells; ++i) {
        xyz[3 * i] = (float)(rng.uniform() * W);
        xyz[3 * i + 1] = (float)(rng.uniform() * H);
        xyz[3 * i + 2] = (float)(rng.uniform() * D);
        ids[i] = rng.label();
    }
    Grid g = bucket_seeds(xyz, n_cells, W, H, D);
    std::vector<uint64_t> pts_ids(n_cells);
    for (uint32_t i = 0; i < n_cells; ++i) pts_ids[i] = ids[i];
    std::vector<uint8_t> zero_cell(n_cells, 0);
    VoronoiArgs a{};
    a.cell = g.cell;
    a.gx = g.gx; a.gy = g.gy; a.gz = g.gz;
    a.W = W; a.H = H; a.D = D;
    a.x0 = 0; a.x1 = W;
    a.thr = INFINITY;
    if (kind == 0 && zero_frac > 0) {
        double nx = rng.uniform() - 0.5, ny = rng.uniform() - 0.5, nz = rng.uniform() - 0.5;
        double nn = sqrt(nx * nx + ny * ny + nz * nz) + 1e-12;
        nx /= nn; ny /= nn; nz /= nn;
        std::vector<double> d(65536);
        for (auto& v : d) {  // the three draws in a fixed order
            const double a = rng.uniform() * W;
            const double b = rng.uniform() * H;
            const double c = rng.uniform() * D;
            v = a * nx + b * ny + c * nz;
        }
        std::sort(d.begin(), d.end());
        size_t q = (size_t)((1.0 - zero_frac) * (d.size() - 1));
        a.nx = (float)nx; a.ny = (float)ny; a.nz = (float)nz;
        a.thr = (float)d[q];
    } else if (kind != 0 && zero_frac > 0) {
        for (uint32_t i = 0; i < n_cells; ++i) zero_cell[i] = rng.uniform() < zero_frac ? 1 : 0;
    }
    uint32_t *d_start = nullptr;
    float4* d_pts = nullptr;
    uint64_t* d_ids = nullptr;
    uint8_t* d_zero = nullptr;
    uint32_t* d_owner = nullptr;
    Piece* d_pieces = nullptr;
    uint64_t* d_tids = nullptr;
    cudaError_t e = upload(&d_start, g.start);
    if (e == cudaSuccess) e = upload(&d_pts, g.pts);
    if (e == cudaSuccess) e = upload(&d_ids, pts_ids);
    if (e == cudaSuccess) e = upload(&d_zero, zero_cell);
    if (e == cudaSuccess) {
        a.start = d_start; a.pts = d_pts; a.ids = d_ids;
        a.zero_cell = (kind != 0) ? d_zero : nullptr;
        uint64_t n = (uint64_t)W * H * D;
        uint32_t blocks = (uint32_t)std::min<uint64_t>((n + 255) / 256, 148ull * 64);
        voronoi_kernel<<<blocks, 256, 0, st>>>(d_vol, a);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && kind != 0 && n_tubes > 0) {
        std::vector<Piece> pieces;
        std::vector<uint64_t> tids(n_tubes);
        float xlo = (kind == 2) ? W * 0.5f : 0.f;
        for (uint32_t t = 0; t < n_tubes; ++t) {
            float c[4][3];
            for (int k = 0; k < 4; ++k) {
                c[k][0] = (float)(xlo + rng.uniform() * (W - xlo));
                c[k][1] = (float)(rng.uniform() * H);
                c[k][2] = (float)(rng.uniform() * D);
            }
            float r = (float)(r_min + rng.uniform() * (r_max - r_min));
            tids[t] = rng.label();
            // Catmull-Rom segment between c[1] and c[2]
            float len = sqrtf((c[2][0] - c[1][0]) * (c[2][0] - c[1][0]) + (c[2][1] - c[1][1]) * (c[2][1] - c[1][1]) +
                              (c[2][2] - c[1][2]) * (c[2][2] - c[1][2]));
            int ns = std::max(2, (int)(len / std::max(1.f, r)) + 2);
            float prev[3] = {0, 0, 0};
            for (int k = 0; k <= ns; ++k) {
                float u = (float)k / ns, u2 = u * u, u3 = u2 * u;
                float p[3];
                for (int d = 0; d < 3; ++d)
                    p[d] = 0.5f * (2 * c[1][d] + (-c[0][d] + c[2][d]) * u +
                                   (2 * c[0][d] - 5 * c[1][d] + 4 * c[2][d] - c[3][d]) * u2 +
                                   (-c[0][d] + 3 * c[1][d] - 3 * c[2][d] + c[3][d]) * u3);
                if (k > 0) {
                    Piece pc;
                    pc.ax = prev[0]; pc.ay = prev[1]; pc.az = prev[2];
                    pc.bx = p[0]; pc.by = p[1]; pc.bz = p[2];
                    pc.r = r;
                    pc.tube = t;
                    uint32_t ext[3] = {W, H, D};
                    for (int d = 0; d < 3; ++d) {
                        float lo = std::min(prev[d], p[d]) - r, hi = std::max(prev[d], p[d]) + r;
                        pc.lo[d] = std::max(0, (int)floorf(lo));
                        if (d == 0 && kind == 2) pc.lo[d] = std::max(pc.lo[d], (int)(W / 2));
                        pc.hi[d] = std::min((int)ext[d], (int)ceilf(hi) + 1);
                    }
                    pieces.push_back(pc);
                }
                prev[0] = p[0]; prev[1] = p[1]; prev[2] = p[2];
            }
        }
        uint64_t n = (uint64_t)W * H * D;
        e = cudaMalloc(&d_owner, n * 4);
        if (e == cudaSuccess) e = cudaMemsetAsync(d_owner, 0, n * 4, st);
        if (e == cudaSuccess) e = upload(&d_pieces, pieces);
        if (e == cudaSuccess) e = upload(&d_tids, tids);
        if (e == cudaSuccess && !pieces.empty()) {
            for (size_t off = 0; off < pieces.size() && e == cudaSuccess; off += 65535) {
                uint32_t cnt = (uint32_t)std::min<size_t>(65535, pieces.size() - off);
                tube_kernel<<<cnt, 256, 0, st>>>(d_owner, d_pieces + off, W, H);
                e = cudaGetLastError();
            }
            uint32_t blocks = (uint32_t)std::min<uint64_t>((n + 255) / 256, 148ull * 64);
            if (e == cudaSuccess) combine_kernel<<<blocks, 256, 0, st>>>(d_vol, d_owner, d_tids, n);
            if (e == cudaSuccess) e = cudaGetLastError();
        }
    }
    cudaError_t e2 = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = e2;
    cudaFree(d_start); cudaFree(d_pts); cudaFree(d_ids); cudaFree(d_zero);
    cudaFree(d_owner); cudaFree(d_pieces); cudaFree(d_tids);
    return e;
}

}  // namespace csv
