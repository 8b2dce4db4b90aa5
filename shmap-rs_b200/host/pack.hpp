// Host packing of reads into 2-bit codes and a non-ACGT mask (see pack.cpp).
#pragma once
#include <cstddef>
#include <cstdint>

namespace shm {

// Packs nb bytes; codes needs packed_code_words(nb) words, mask
// packed_mask_words(nb) (the spare words past the end hold code 0, masked).
void pack_reads_host(const uint8_t* seq, int64_t nb, uint32_t* codes, uint32_t* mask);
// The same on the host threads in the background with the mask in sparse
// form: start returns at once; wait returns when the packing is complete,
// writing the nonzero mask words as (word index, word) pairs, at most cap of
// them (never more than packed_mask_words(nb)), and returns their number.
// One packing at a time: a thread's start waits for another thread's packing
// to be waited for. The work is cut into tasks of task_groups 32-byte groups
// (rounded down to an even number), or, for task_groups <= 0, into four tasks
// a thread of at least 1 MiB each.
void pack_reads_host_start(const uint8_t* seq, int64_t nb, uint32_t* codes, int64_t task_groups = 0);
size_t pack_reads_host_wait(uint32_t* pairs, size_t cap);
// Ends a packing that will not be waited for (an error in between): the
// packing calls of other threads may start again.
void pack_reads_host_release();
size_t packed_code_words(int64_t nb);
size_t packed_mask_words(int64_t nb);

}  // namespace shm
