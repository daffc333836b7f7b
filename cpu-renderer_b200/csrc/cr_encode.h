// Device-side output encoding of a linear RGB film (cr_encode.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace crg {

// Encodes width*height RGB float triples at dFilm (device memory of the current device) on
// stream s into one of the cr_encode_format layouts. Returns the encoded size in bytes; the
// bytes are copied to `out` (host memory) when out is not NULL and capacity suffices,
// otherwise nothing is copied. Throws crh::Error with the reference's validation messages.
uint64_t encode_film(const float* dFilm, int width, int height, int format, float exposure,
                     cudaStream_t s, void* out, uint64_t capacity);

}  // namespace crg
