// Device-wide primitives written for this path: an exclusive scan and a
// stable LSD radix sort of (u64 key, u32 value) pairs. Temporaries come from
// a stream-ordered pool per device that keeps its memory.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace shm {

// out[0..n] = exclusive prefix sums of in[0..n), out[n] = total.
void exclusive_scan_u32(const uint32_t* in, uint32_t* out, size_t n, cudaStream_t s);
void exclusive_scan_u64(const uint64_t* in, uint64_t* out, size_t n, cudaStream_t s);

// Stable sort by key bits [0, key_bits). Sorts (k0,v0) using (k1,v1) as the
// ping-pong buffer; returns true if the result ended in (k1,v1).
bool radix_sort_pairs(uint64_t* k0, uint32_t* v0, uint64_t* k1, uint32_t* v1, size_t n, int key_bits,
                      cudaStream_t s);

// Kernels this process launched (every launch site of the library bumps it).
int64_t kernel_launches();
void count_launch(int64_t n = 1);

// Grid size for grid-stride kernels: a multiple of the SM count.
int grid_for(size_t work, int block, int max_blocks_per_sm = 8);

}  // namespace shm
