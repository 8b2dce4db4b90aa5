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
};

// The settings in force (read once per process, then as set).
Tuning tuning();

}  // namespace shm
