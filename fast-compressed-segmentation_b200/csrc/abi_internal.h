// abi_internal.h -- the opaque handles of include/csv.h and the host helpers the
// C-ABI translation units (abi.cu, serve.cu) share.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "csv_internal.h"

struct csv_ctx {
    int device = 0;
    std::string err;
    csv::DecodeScratch scr;
    uint32_t scr_b = 0;
    // the second launch of a split graph (outputs of 32^3 and smaller) runs beside the first
    // one's last CTAs, so it has scratch and a queue counter of its own; created on first use
    csv::DecodeScratch scr_small;
    // the 64^3 outputs of bricks with 255 or more palette entries, when a split graph gives the
    // others to the 8-bit variant: a third launch, beside the first; created on first use
    csv::DecodeScratch scr_wide;
    cudaMemPool_t pool = nullptr;  // stream-ordered temporaries of opens (keeps freed memory)
    uint32_t scr_wide_b = 0;
    csv::EncoderState* enc = nullptr;
    // csv_decode_image's pipeline: two chunk buffers (decode one while the
    // other drains to the host), its streams and events; created on first use
    uint64_t* chunk_buf[2] = {nullptr, nullptr};
    size_t chunk_bytes = 0;
    cudaStream_t pipe_stream[2] = {nullptr, nullptr};  // decode, copy
    cudaEvent_t pipe_event[4] = {nullptr, nullptr, nullptr, nullptr};  // decoded[2], drained[2]
};

struct csv_dataset {
    csv_ctx* ctx = nullptr;
    csv::DeviceDataset d;
};

namespace csv {

// Record `msg` as the context's last error and return `code`.
int abi_fail(csv_ctx* ctx, int code, const std::string& msg);
int abi_cuda_fail(csv_ctx* ctx, cudaError_t e, const char* where);
// Size the context's decode scratch for bricks of edge b (grows, never shrinks).
int abi_ensure_scratch(csv_ctx* ctx, uint32_t b);
// Allocate the context's scratch for the small variant's part of a split schedule.
int abi_ensure_scratch_small(csv_ctx* ctx);
int abi_ensure_scratch_wide(csv_ctx* ctx, uint32_t b);
// buildTransferFunctionBuffers (webgpuSetup.js:389-465) on a dataset: its distinct
// non-zero palette labels ascending and their RGBA8, hidden labels transparent.
cudaError_t transfer_function(const DeviceDataset& d, const uint64_t* hidden, uint32_t n_hidden,
                              std::vector<uint64_t>& keys, std::vector<uint32_t>& rgba);

// Makes `dev` current for the scope and restores the caller's device after.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace csv
