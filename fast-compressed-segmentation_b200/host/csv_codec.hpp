// csv_codec.hpp -- C++ host API over the C ABI (include/csv.h), shaped like the
// reference encoder/decoder it replaces (paths relative to the reference root):
//
//   reference                                         here (namespace csvb200)
//   NpyArray (types.hpp:147-151)                      NpyArray
//   splitGridIntoBricks<b> + Encoding::compressDataset compressDataset(npy, brickSize)
//     (brick.hpp:134, brickEncoding.hpp:467)
//   saveDatasetToFile (fileIO.cpp:15)                 saveDatasetToFile(dataset, filename)
//   loadDatasetFromFile (fileIO.cpp:101)              loadDatasetFromFile(filename)
//   decodeRansStream + decodeBrick<b>                 decodeBrick(dataset, brickIndex, targetLOD)
//     (brickDecoding.cpp:153, brickDecoding.hpp:175)
//
// As in the reference, failures throw std::runtime_error.  Unlike the
// reference, decodeBrick is valid at every targetLOD (the reference's C++
// decoder is only valid at full resolution), all bricks of a dataset can be
// decoded in one launch (decodeAll), and all codec work runs on the GPU.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iterator>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/csv.h"

namespace csvb200 {

// shape = {width, height, depth}; data[x + width * (y + height * z)] (brick.hpp:139-141,183).
struct NpyArray {
    std::vector<uint64_t> data;
    std::vector<size_t> shape;
};

// A .csbd v1 image held in host memory, plus its device-resident form once opened.
struct CompressedDataset {
    std::vector<uint8_t> bytes;
    uint32_t numBricks() const { return bytes.size() >= 12 ? rd32(8) : 0; }
    uint32_t brickSize() const { return bytes.size() >= 16 ? rd32(12) : 0; }

  private:
    uint32_t rd32(size_t o) const {
        uint32_t v;
        std::memcpy(&v, bytes.data() + o, 4);
        return v;
    }
};

class Context {
  public:
    explicit Context(int device = 0) {
        if (csv_create(device, &ctx_) != CSV_OK) throw std::runtime_error("csv_create failed (no CUDA device?)");
    }
    ~Context() { csv_destroy(ctx_); }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    csv_ctx* get() const { return ctx_; }
    void check(int rc) const {
        if (rc != CSV_OK) throw std::runtime_error(std::string("csv: ") + csv_last_error(ctx_));
    }

  private:
    csv_ctx* ctx_ = nullptr;
};

inline Context& defaultContext() {
    static Context ctx(0);
    return ctx;
}

// splitGridIntoBricks<b> + compressDataset<b>: the whole volume to one .csbd image.
inline CompressedDataset compressDataset(const NpyArray& array, uint32_t brickSize = 64,
                                         Context& ctx = defaultContext()) {
    if (array.shape.size() != 3) throw std::runtime_error("Expected a 3D array");  // brick.hpp:136-137
    uint8_t* out = nullptr;
    size_t len = 0;
    ctx.check(csv_encode(ctx.get(), array.data.data(), (uint32_t)array.shape[0], (uint32_t)array.shape[1],
                         (uint32_t)array.shape[2], brickSize, &out, &len));
    CompressedDataset ds;
    ds.bytes.assign(out, out + len);
    csv_free(out);
    return ds;
}

inline void saveDatasetToFile(const CompressedDataset& dataset, const std::string& filename) {
    std::ofstream out(filename, std::ios::binary);
    if (!out) throw std::runtime_error("Failed to open file for writing");  // fileIO.cpp:19-20
    out.write(reinterpret_cast<const char*>(dataset.bytes.data()), (std::streamsize)dataset.bytes.size());
}

inline CompressedDataset loadDatasetFromFile(const std::string& filename) {
    std::ifstream in(filename, std::ios::binary);
    if (!in) throw std::runtime_error("Failed to open file");  // fileIO.cpp:104-105
    CompressedDataset ds;
    ds.bytes.assign(std::istreambuf_iterator<char>(in), std::istreambuf_iterator<char>());
    if (ds.bytes.size() < 4 || ds.bytes[0] != 0x44 || ds.bytes[1] != 0x42 || ds.bytes[2] != 0x53 ||
        ds.bytes[3] != 0x43)
        throw std::runtime_error("Invalid file format");  // fileIO.cpp:118-119
    return ds;
}

// Every brick at targetLOD; brick i (file order) at i * 8^targetLOD, Morton order inside.
inline std::vector<uint64_t> decodeAll(const CompressedDataset& ds, uint32_t targetLOD,
                                       Context& ctx = defaultContext()) {
    size_t per = size_t(1) << (3 * targetLOD);
    std::vector<uint64_t> out(per * ds.numBricks());
    ctx.check(csv_decode_image(ctx.get(), ds.bytes.data(), ds.bytes.size(), targetLOD, out.data(), nullptr));
    return out;
}

// One brick at targetLOD (8^targetLOD labels, Morton order).
inline std::vector<uint64_t> decodeBrick(const CompressedDataset& ds, uint32_t brickIndex, uint32_t targetLOD,
                                         Context& ctx = defaultContext()) {
    if (brickIndex >= ds.numBricks()) throw std::runtime_error("brick index out of range");
    std::vector<uint64_t> all = decodeAll(ds, targetLOD, ctx);
    size_t per = size_t(1) << (3 * targetLOD);
    return std::vector<uint64_t>(all.begin() + per * brickIndex, all.begin() + per * (brickIndex + 1));
}

}  // namespace csvb200
