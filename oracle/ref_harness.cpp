// ref_harness.cpp -- C-linkage wrappers around the UNMODIFIED reference encoder /
// decoder sources (encoder/CSVEncoder/src/*.cpp, compiled where they lie by
// oracle/Makefile).  This file is test infrastructure: it is built into
// oracle/_ref/libcsvref.so and is only ever loaded by tests/, by
// __graft_entry__.smoke() and by bench.py's CPU-baseline / reference arm, as the
// checker or the timed CPU reference.  Nothing in the product links it.
//
// Each wrapper cites the reference entry point it drives.  The wrappers add no
// codec arithmetic of their own; they only marshal plain buffers in and out.
#include "brickEncoding.hpp"
#include "brickDecoding.hpp"
#include "fileIO.hpp"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <unistd.h>

namespace {

std::string g_err;

// One main() invocation of the reference starts from zeroed frequency
// globals (brickEncoding.cpp:7-8).  They are never reset by the reference, so a
// long-lived process must reset them before each dataset to mean the same thing.
void reset_globals() {
    Encoding::interiorFreqTable.fill(0);
    Encoding::leafFreqTable.fill(0);
}

std::string temp_path() {
    char buf[] = "/tmp/csvref_XXXXXX";
    int fd = mkstemp(buf);
    if (fd >= 0) close(fd);
    return std::string(buf);
}

bool slurp(const std::string& p, std::vector<uint8_t>& out) {
    std::ifstream in(p, std::ios::binary);
    if (!in) return false;
    in.seekg(0, std::ios::end);
    size_t n = (size_t)in.tellg();
    in.seekg(0);
    out.resize(n);
    in.read(reinterpret_cast<char*>(out.data()), n);
    return true;
}

template <size_t b>
int encode_impl(const uint64_t* vol, size_t W, size_t H, size_t D, uint8_t** out, size_t* out_len,
                double* ms_split, double* ms_compress, double* ms_save) {
    NpyArray npy;
    npy.shape = {W, H, D};
    npy.data.assign(vol, vol + W * H * D);
    reset_globals();
    auto t0 = std::chrono::steady_clock::now();
    auto bricks = splitGridIntoBricks<b>(npy);                      // brick.hpp:134
    auto t1 = std::chrono::steady_clock::now();
    auto compressed = Encoding::compressDataset(bricks);             // brickEncoding.hpp:467
    auto t2 = std::chrono::steady_clock::now();
    std::string path = temp_path();
    saveDatasetToFile(compressed, path);                             // fileIO.cpp:15
    auto t3 = std::chrono::steady_clock::now();
    std::vector<uint8_t> bytes;
    bool ok = slurp(path, bytes);
    std::remove(path.c_str());
    if (!ok) { g_err = "cannot read back the written .csbd"; return -1; }
    // fileIO.cpp:28 always stores BRICK_SIZE (64); a dataset compressed with
    // another brick size gets its real size in that header field.
    if (b != BRICK_SIZE && bytes.size() >= 16) {
        uint32_t bs = (uint32_t)b;
        std::memcpy(bytes.data() + 12, &bs, 4);
    }
    *out = (uint8_t*)std::malloc(bytes.size());
    std::memcpy(*out, bytes.data(), bytes.size());
    *out_len = bytes.size();
    auto ms = [](auto a, auto c) { return std::chrono::duration<double, std::milli>(c - a).count(); };
    if (ms_split) *ms_split = ms(t0, t1);
    if (ms_compress) *ms_compress = ms(t1, t2);
    if (ms_save) *ms_save = ms(t2, t3);
    return 0;
}

// Parse the .csbd image with the reference reader (fileIO.cpp:101).
bool load_image(const uint8_t* csbd, size_t len, Encoding::CompressedDataset& ds) {
    std::string path = temp_path();
    {
        std::ofstream o(path, std::ios::binary);
        o.write(reinterpret_cast<const char*>(csbd), (std::streamsize)len);
    }
    try {
        ds = loadDatasetFromFile(path);
    } catch (const std::exception& e) {
        g_err = e.what();
        std::remove(path.c_str());
        return false;
    }
    std::remove(path.c_str());
    // The reader keeps 16 cumulative entries (fileIO.cpp:131); findSymbol
    // (brickDecoding.cpp:126-135) then tests boundaries 1..15, which selects
    // the same symbol as the 17-entry table the encoder built because x < 4096
    // never reaches cum[16].  The model is used exactly as loaded (main.cpp:99).
    return true;
}

template <size_t b>
int decode_full_impl(const Encoding::CompressedBrick& br, const RansModel& model, uint64_t* out) {
    Encoding::CompressedBrick cb = br;
    cb.encodedData = decodeRansStream(cb, model);                    // brickDecoding.cpp:153
    auto labels = decodeBrick<b>(cb, Brick<b>::Levels - 1);           // brickDecoding.hpp:175
    std::memcpy(out, labels.data(), labels.size() * sizeof(uint64_t));
    return 0;
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

void ref_free(void* p) { std::free(p); }

// splitGridIntoBricks<b> + compressDataset<b> + saveDatasetToFile.
// vol is x-fastest: vol[x + W*(y + H*z)] (brick.hpp:183).
int ref_encode(const uint64_t* vol, size_t W, size_t H, size_t D, int brick_size,
               uint8_t** out, size_t* out_len, double* ms_split, double* ms_compress, double* ms_save) {
    try {
        switch (brick_size) {
        case 8: return encode_impl<8>(vol, W, H, D, out, out_len, ms_split, ms_compress, ms_save);
        case 16: return encode_impl<16>(vol, W, H, D, out, out_len, ms_split, ms_compress, ms_save);
        case 32: return encode_impl<32>(vol, W, H, D, out, out_len, ms_split, ms_compress, ms_save);
        case 64: return encode_impl<64>(vol, W, H, D, out, out_len, ms_split, ms_compress, ms_save);
        default: g_err = "unsupported brick size"; return -1;
        }
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// decodeRansStream + decodeBrick<b>(., Levels-1) for brick `index` (file order).
// out receives b^3 labels in Morton order.  Returns -1 (and sets the error
// text) where the reference throws, e.g. on a uniform brick.
int ref_decode_brick_full(const uint8_t* csbd, size_t len, uint32_t index, uint64_t* out) {
    Encoding::CompressedDataset ds;
    if (!load_image(csbd, len, ds)) return -1;
    if (index >= ds.bricks.size()) { g_err = "brick index out of range"; return -1; }
    uint32_t bs;
    std::memcpy(&bs, csbd + 12, 4);
    try {
        switch (bs) {
        case 8: return decode_full_impl<8>(ds.bricks[index], ds.model, out);
        case 16: return decode_full_impl<16>(ds.bricks[index], ds.model, out);
        case 32: return decode_full_impl<32>(ds.bricks[index], ds.model, out);
        case 64: return decode_full_impl<64>(ds.bricks[index], ds.model, out);
        default: g_err = "unsupported brick size"; return -1;
        }
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// Decode every brick of the image at full resolution (main.cpp:94-118 loop),
// optionally timing it.  out holds numBricks * b^3 labels, brick i at i*b^3.
// status[i] = 0 on success, 1 where the reference threw for that brick.
int ref_decode_all_full(const uint8_t* csbd, size_t len, uint64_t* out, uint32_t* status,
                        uint32_t max_bricks, double* ms_rans, double* ms_replay) {
    Encoding::CompressedDataset ds;
    if (!load_image(csbd, len, ds)) return -1;
    uint32_t bs;
    std::memcpy(&bs, csbd + 12, 4);
    size_t vox = (size_t)bs * bs * bs;
    size_t n = ds.bricks.size();
    if (max_bricks && max_bricks < n) n = max_bricks;
    double tr = 0, tp = 0;
    for (size_t i = 0; i < n; ++i) {
        auto& br = ds.bricks[i];
        try {
            auto t0 = std::chrono::steady_clock::now();
            Encoding::CompressedBrick cb = br;
            cb.encodedData = decodeRansStream(cb, ds.model);
            auto t1 = std::chrono::steady_clock::now();
            std::vector<LabelType> labels;
            switch (bs) {
            case 8: labels = decodeBrick<8>(cb, Brick<8>::Levels - 1); break;
            case 16: labels = decodeBrick<16>(cb, Brick<16>::Levels - 1); break;
            case 32: labels = decodeBrick<32>(cb, Brick<32>::Levels - 1); break;
            case 64: labels = decodeBrick<64>(cb, Brick<64>::Levels - 1); break;
            default: g_err = "unsupported brick size"; return -1;
            }
            auto t2 = std::chrono::steady_clock::now();
            tr += std::chrono::duration<double, std::milli>(t1 - t0).count();
            tp += std::chrono::duration<double, std::milli>(t2 - t1).count();
            if (out) std::memcpy(out + i * vox, labels.data(), vox * sizeof(uint64_t));
            if (status) status[i] = 0;
        } catch (const std::exception& e) {
            if (status) status[i] = 1;
        }
    }
    if (ms_rans) *ms_rans = tr;
    if (ms_replay) *ms_replay = tp;
    return (int)n;
}

// A loaded image for repeated, range-wise decoding (the reference arm decodes
// disjoint brick ranges from several host threads).
struct RefImage {
    Encoding::CompressedDataset ds;
    uint32_t b;
};

void* ref_load(const uint8_t* csbd, size_t len) {
    auto* h = new RefImage();
    if (!load_image(csbd, len, h->ds)) { delete h; return nullptr; }
    std::memcpy(&h->b, csbd + 12, 4);
    return h;
}

void ref_unload(void* h) { delete static_cast<RefImage*>(h); }

// decodeRansStream + decodeBrick<b>(., full) for bricks [start, start+count);
// out (may be null) receives count * b^3 labels.  Returns bricks that threw.
int ref_decode_strided(void* hv, uint32_t start, uint32_t count, uint32_t stride, uint64_t* out);
int ref_decode_range(void* hv, uint32_t start, uint32_t count, uint64_t* out) {
    return ref_decode_strided(hv, start, count, 1, out);
}

// The same over bricks start, start + stride, ... (count of them).
int ref_decode_strided(void* hv, uint32_t start, uint32_t count, uint32_t stride, uint64_t* out) {
    auto* h = static_cast<RefImage*>(hv);
    int bad = 0;
    size_t vox = (size_t)h->b * h->b * h->b;
    if (stride == 0) stride = 1;
    for (uint32_t k = 0; k < count && start + (size_t)k * stride < h->ds.bricks.size(); ++k) {
        try {
            Encoding::CompressedBrick cb = h->ds.bricks[start + (size_t)k * stride];
            cb.encodedData = decodeRansStream(cb, h->ds.model);
            std::vector<LabelType> labels;
            switch (h->b) {
            case 8: labels = decodeBrick<8>(cb, Brick<8>::Levels - 1); break;
            case 16: labels = decodeBrick<16>(cb, Brick<16>::Levels - 1); break;
            case 32: labels = decodeBrick<32>(cb, Brick<32>::Levels - 1); break;
            case 64: labels = decodeBrick<64>(cb, Brick<64>::Levels - 1); break;
            default: return -1;
            }
            if (out) std::memcpy(out + k * vox, labels.data(), vox * sizeof(uint64_t));
        } catch (const std::exception&) {
            ++bad;
        }
    }
    return bad;
}

// The reference's rANS stage alone (brickDecoding.cpp:153): the repacked nibble
// bytes of brick `index`.  out must hold ceil(nSymbols/2) bytes.
int ref_rans_decode(const uint8_t* csbd, size_t len, uint32_t index, uint8_t* out, size_t* out_len) {
    Encoding::CompressedDataset ds;
    if (!load_image(csbd, len, ds)) return -1;
    if (index >= ds.bricks.size()) { g_err = "brick index out of range"; return -1; }
    auto nib = decodeRansStream(ds.bricks[index], ds.model);
    std::memcpy(out, nib.data(), nib.size());
    *out_len = nib.size();
    return 0;
}

// majorityVote8 (brick.hpp:24-37) as compiled here (libstdc++ unordered_map).
uint64_t ref_majority8(const uint64_t* labels) { return majorityVote8(labels); }

// buildRansModel (brickEncoding.cpp:146-200) on a raw 16-bin histogram.
void ref_build_model(const uint64_t* raw16, uint32_t* freq16, uint32_t* cum17) {
    Encoding::FrequencyTable t{};
    for (int i = 0; i < 16; ++i) t[i] = (size_t)raw16[i];
    auto m = Encoding::buildRansModel(t);
    for (int i = 0; i < 16; ++i) freq16[i] = m.freq[i];
    for (int i = 0; i < 17; ++i) cum17[i] = m.cumulativeFreq[i];
}

// Brick<b>::build (brick.hpp:78-123) for one brick cut from the volume:
// levels_out receives all levels finest-first, each in Morton order, as
// (label, constantChildren) pairs: label array then a byte array of flags.
int ref_build_pyramid64(const uint64_t* vol, size_t W, size_t H, size_t D, uint32_t brick_index,
                        uint64_t* labels_out, uint8_t* const_out) {
    NpyArray npy;
    npy.shape = {W, H, D};
    npy.data.assign(vol, vol + W * H * D);
    auto bricks = splitGridIntoBricks<64>(npy);
    if (brick_index >= bricks.size()) return -1;
    auto& br = bricks[brick_index];
    br.build();
    size_t o = 0;
    for (size_t l = 0; l < Brick<64>::Levels; ++l)
        for (auto& n : br.level(l)) {
            labels_out[o] = n.label;
            const_out[o] = n.constantChildren ? 1 : 0;
            ++o;
        }
    return (int)o;
}

}  // extern "C"
