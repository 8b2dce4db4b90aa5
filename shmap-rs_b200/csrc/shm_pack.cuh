// Reads packed on the device (see shm_pack.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace shm {

// nb ASCII bytes at seq (device; 16 readable bytes past seq + nb) to codes
// (2 * (nb / 32 + 3) words) and mask (nb / 32 + 3 words), device memory:
// the layout of host/pack.hpp.
void pack_reads_device(const uint8_t* seq, int64_t nb, uint32_t* codes, uint32_t* mask, cudaStream_t s);

// Exactly n_groups whole groups of 32 bytes at seq (device, 16-byte aligned)
// to codes[0, 2 n_groups) and mask[0, n_groups): no spare groups, nothing
// past them written. Returns the launch's error instead of throwing (it is
// called from host packing threads).
cudaError_t pack_groups_device(const uint8_t* seq, int64_t n_groups, uint32_t* codes, uint32_t* mask,
                               cudaStream_t s);

}  // namespace shm
