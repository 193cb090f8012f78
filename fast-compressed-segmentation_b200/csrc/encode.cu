// encode.cu -- sm_100a brick encoder.
#include <cuda_runtime.h>
#include <stdint.h>

#include "csv_internal.h"

namespace csv {

struct EncoderState {
    int unused = 0;
};

void encoder_state_free(EncoderState* s) { delete s; }

}  // namespace csv

extern "C" {

int csv_encode(csv_ctx*, const uint64_t*, uint32_t, uint32_t, uint32_t, uint32_t, uint8_t**, size_t*) {
    return CSV_EINVAL;
}
int csv_encode_device(csv_ctx*, const uint64_t*, uint32_t, uint32_t, uint32_t, uint32_t, void*, size_t*) {
    return CSV_EINVAL;
}
int csv_encoded_image(csv_ctx*, const uint8_t**, size_t*) { return CSV_EINVAL; }
int csv_open_encoded(csv_ctx*, csv_dataset**) { return CSV_EINVAL; }

}
