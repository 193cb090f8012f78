// example_encode_decode.cpp -- the reference's main.cpp flow (main.cpp:67-130)
// through the C++ host API: volume -> compressDataset -> saveDatasetToFile ->
// loadDatasetFromFile -> decode every brick -> compare with the source.
// Unlike main.cpp (whose comparison is commented out, main.cpp:104-114), the
// comparison here is real and sets the exit code.
//
//   usage: example_encode_decode <W> <H> <D> <brickSize> <out.csbd>
#include <cstdio>
#include <cstdlib>

#include "csv_codec.hpp"

static uint32_t spread(uint32_t v) {
    uint32_t r = 0;
    for (int i = 0; i < 10; ++i) r |= ((v >> i) & 1u) << (3 * i);
    return r;
}

int main(int argc, char** argv) {
    if (argc != 6) {
        std::fprintf(stderr, "usage: %s W H D brickSize out.csbd\n", argv[0]);
        return 2;
    }
    const size_t W = std::strtoul(argv[1], 0, 10), H = std::strtoul(argv[2], 0, 10), D = std::strtoul(argv[3], 0, 10);
    const uint32_t b = (uint32_t)std::strtoul(argv[4], 0, 10);
    csvb200::NpyArray npy;
    npy.shape = {W, H, D};
    npy.data.resize(W * H * D);
    // blocky test pattern: slabs and boxes of a few labels
    for (size_t z = 0; z < D; ++z)
        for (size_t y = 0; y < H; ++y)
            for (size_t x = 0; x < W; ++x) {
                uint64_t v = 1 + ((x / 7) ^ (y / 11) ^ (z / 5)) % 9;
                if ((x / 16 + y / 16 + z / 16) % 5 == 0) v = 0;
                npy.data[x + W * (y + H * z)] = v * 0x9E3779B97F4A7C15ull;
            }
    try {
        auto ds = csvb200::compressDataset(npy, b);
        csvb200::saveDatasetToFile(ds, argv[5]);
        auto loaded = csvb200::loadDatasetFromFile(argv[5]);
        const uint32_t full = __builtin_ctz(b);
        auto labels = csvb200::decodeAll(loaded, full);
        const size_t nbx = (W + b - 1) / b, nby = (H + b - 1) / b, nbz = (D + b - 1) / b, per = (size_t)b * b * b;
        size_t i = 0, bad = 0;
        for (size_t bx = 0; bx < nbx; ++bx)
            for (size_t by = 0; by < nby; ++by)
                for (size_t bz = 0; bz < nbz; ++bz, ++i)
                    for (uint32_t dz = 0; dz < b; ++dz)
                        for (uint32_t dy = 0; dy < b; ++dy)
                            for (uint32_t dx = 0; dx < b; ++dx) {
                                size_t gx = bx * b + dx, gy = by * b + dy, gz = bz * b + dz;
                                uint64_t want = (gx < W && gy < H && gz < D) ? npy.data[gx + W * (gy + H * gz)] : 0;
                                uint32_t m = spread(dx) | (spread(dy) << 1) | (spread(dz) << 2);
                                bad += labels[i * per + m] != want;
                            }
        auto coarse = csvb200::decodeBrick(loaded, 0, full > 2 ? 2 : 0);
        std::printf("bricks=%u bytes=%zu mismatches=%zu coarse=%zu\n", loaded.numBricks(), loaded.bytes.size(), bad,
                    coarse.size());
        return bad == 0 ? 0 : 1;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
}
