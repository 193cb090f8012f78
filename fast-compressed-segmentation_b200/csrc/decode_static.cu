// decode_static.cu -- the batched brick decoder for callers that cannot allocate.
//
// csv_decode_batch sizes its per-CTA scratch on first use with cudaMalloc.  Some
// callers cannot call cudaMalloc at that point: a render loop that must not
// stall (cudaMalloc can synchronize the device), or a host program that runs
// every allocation through its own arena and forbids the driver's allocator
// after start-up.  csv_decode_batch_static runs the same decode kernel with its
// scratch (op records, active-node lists, the work-queue counter) taken from
// the file-scope device array below instead, so it allocates nothing.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <string>

#include "csv_internal.h"

namespace csv {

// Reserved in every GPU that loads this library, until the process exits.
static __device__ __align__(256) uint8_t g_static_scratch[CSV_STATIC_SCRATCH_BYTES];

namespace {

constexpr size_t kQueueBytes = 256;  // the work-queue counter, at the start of the array
std::mutex g_mu;
uint8_t* g_addr[64] = {nullptr};     // device address of g_static_scratch, per device

// Host code cannot use g_static_scratch as a pointer: here it names a host-side
// stand-in.  The device address is looked up once per device, with that device
// current.
cudaError_t static_scratch(int device, uint8_t** out) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
    if (!g_addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return e;
        g_addr[device] = static_cast<uint8_t*>(p);
    }
    *out = g_addr[device];
    return cudaSuccess;
}

}  // namespace

int decode_batch_static(int device, const DeviceDataset& ds, const csv_request* d_reqs, uint32_t n, uint64_t* d_out,
                        uint32_t* d_status, cudaStream_t st, std::string& err) {
    const size_t per = decode_scratch_per_cta(ds.b);
    if (per > CSV_STATIC_SCRATCH_BYTES - kQueueBytes) {
        err = "brick size " + std::to_string(ds.b) + " needs " + std::to_string(per) +
              " bytes of decode scratch per CTA; the static array holds " +
              std::to_string((size_t)CSV_STATIC_SCRATCH_BYTES - kQueueBytes);
        return CSV_ERANGE;
    }
    uint8_t* base = nullptr;
    cudaError_t e = static_scratch(device, &base);
    if (e != cudaSuccess) {
        err = std::string("static scratch address: ") + cudaGetErrorString(e);
        return CSV_ECUDA;
    }
    DecodeScratch scr;
    scr.d_queue = reinterpret_cast<uint32_t*>(base);  // cleared by launch_decode before the kernel
    scr.base = base + kQueueBytes;
    scr.per_cta = per;
    scr.ctas = (uint32_t)((CSV_STATIC_SCRATCH_BYTES - kQueueBytes) / per);
    scr.bytes = CSV_STATIC_SCRATCH_BYTES - kQueueBytes;
    e = launch_decode(ds, d_reqs, n, d_out, d_status, scr, st);
    if (e != cudaSuccess) {
        err = std::string("decode launch: ") + cudaGetErrorString(e);
        return CSV_ECUDA;
    }
    return CSV_OK;
}

}  // namespace csv
