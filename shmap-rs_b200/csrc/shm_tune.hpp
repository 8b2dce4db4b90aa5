// Measured launch and batch shapes (see shm_tune.cu).
#pragma once
#include <stdint.h>

namespace shm {

struct Tuning {
    int64_t dev_batch_reads = 1 << 17;          // reads a batch of a device-resident call holds
    int64_t dev_batch_bases = (int64_t)1 << 31;  // bases a batch of a device-resident call holds
    int64_t dev_first_batch_reads = 1 << 14;     // the first, small: the device starts while the host plans
    int64_t host_batch_reads = 1 << 15;          // the same for calls from host buffers
    int64_t host_batch_bases = 1 << 28;
    int64_t host_first_batch_reads = 1 << 12;
    int64_t sketch_ctas_per_sm = 8;   // packed-read sketch: resident CTAs a grid fills per SM
    int64_t wide_ctas_per_sm = 8;     // bucket kernels that read their counts on the device
    int64_t refine_warps_per_sm = 64; // refinement warps in flight per SM (global-table path)
    int64_t device_pack = 0;          // reads in device memory: 1 = packed there and sketched from codes,
                                      // 0 = sketched from their bytes
    int64_t bt_fast_slots = 512;      // bucket-table slots a read (a power of two) when a batch is queued
                                      // without waiting for its sizes; fuller tables take a second table
    int64_t host_raw_share = 0;       // reads in pinned host memory: the percent of batches sent up as
                                      // ASCII by the copy engine instead of packed on the host threads
    int64_t host_pack_task_kib = 1024;  // host packing: KiB of reads a task of the packing threads takes
                                        // (0: four tasks a thread, at least 1 MiB each)
    int64_t host_stream = 1;            // host reads: one packing stream per call, its chunks sent from
                                        // one pinned buffer (1) or each piece sent by its packing thread
                                        // from a ring of small pinned buffers (2); or host batches packed
                                        // and sent whole, one after another (0)
    int64_t host_stream_piece_kib = 2048;  // host_stream 2: KiB of reads a piece (a packing task)
    int64_t host_stream_ring = 4;          // host_stream 2: piece buffers a packing thread cycles through
    int64_t host_stream_raw_share = 0;     // host_stream 2, reads in pinned memory: percent of the pieces
                                           // sent up as bytes and packed on the device
    int64_t plan_mapped = 1;               // a batch's plan read by a kernel through its pinned block's
                                           // device mapping (1) instead of copied by the copy engine (0)
    int64_t host_stream_bases = (int64_t)1 << 32;  // bases a packing stream covers at most (a longer
                                                   // call is streamed in parts)
    int64_t host_stream_chunk_kib = 16384;  // KiB of reads a chunk of the stream: sent up as soon as
                                            // all its tasks are packed
    int64_t host_stream_first_kib = 32768;  // KiB of reads the first device batch of a stream maps;
                                            // the batches double from there and halve at the end
    int64_t host_stream_last_kib = 262144;  // ... down to about this many KiB
};

// The settings in force (read once per process, then as set).
Tuning tuning();

}  // namespace shm
