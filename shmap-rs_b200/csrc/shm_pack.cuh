// Reads packed on the device (see shm_pack.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace shm {

// nb ASCII bytes at seq (device; 16 readable bytes past seq + nb) to codes
// (2 * (nb / 32 + 3) words) and mask (nb / 32 + 3 words), device memory:
// the layout of host/pack.hpp.
void pack_reads_device(const uint8_t* seq, int64_t nb, uint32_t* codes, uint32_t* mask, cudaStream_t s);

}  // namespace shm
