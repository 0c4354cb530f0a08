// Device-side workload generation (host side declarations).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "field.cuh"

namespace modlin {

cudaError_t gen_uniform_device(uint64_t p, uint64_t seed, uint64_t* d_out, uint64_t count, cudaStream_t st,
                               uint64_t* launches);
cudaError_t reduce_device(const FieldParams& fp, uint64_t* d_x, uint64_t count, cudaStream_t st);

}  // namespace modlin
