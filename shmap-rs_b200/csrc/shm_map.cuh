// Batched mapping on the device (see shm_map.cu).
#pragma once
#include <string>
#include <cstdlib>
#include <cstdio>
#include <chrono>
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../../include/shmap_gpu.h"
#include "shm_internal.hpp"

namespace shm {

// One slot of a read's bucket hash table: a bucket (segm_id, b) and its
// content after seeding (src/buckets.rs:64-73).
struct BSlot {
    unsigned long long key;  // (u64)segm_id << 32 | b, EMPTY_KEY when free
    unsigned long long mc;   // matches << 32 plus codir (signed), summed by one 64-bit atomic add
    int32_t rmin, rmax;
};

// A bucket taken past seeding: extended by the seed heuristic, then (if it
// can still clear a threshold) refined.
struct BucketJob {
    int32_t read, seg, bb, m0;            // location, matches after seeding (the sort key)
    int32_t matches, codir, rmin, rmax;   // content after extension
    double sh;                            // final seed-heuristic score (1.0 when pruning is off)
    int32_t is_cand, pad0;
    double score;                         // refinement result
    int32_t t_l, t_r, inter, same, s_sz, pad1;
    double support;                       // rarity-weighted support of the scored window (0 without rarity)
};

struct MapScratch;  // grow-only device buffers owned by a context
struct PafScratch;  // those of the PAF formatting (shm_paf.cu)
struct StreamSink;  // pinned piece buffers and copy streams of the host packing threads

// Stages timed with CUDA events on the context's stream when timing is on.
enum Stage { STG_SKETCH, STG_SEEDPREP, STG_CONTRIB, STG_BSCAN, STG_EXTEND, STG_REFINE, STG_SWEEP, STG_AUX, N_STAGES };
extern const char* const STAGE_NAMES[N_STAGES];

// Work done, accumulated over every batch of a context: the units the
// roofline's algorithmic bytes are counted in, and the bytes copied between
// host and device.
enum Work { W_READS, W_BASES, W_KMERS, W_DISTINCT, W_PROC_SEEDS, W_HITS, W_BUCKETS, W_JOBS, W_EXT_SEEDS, W_CANDS,
            W_REFINE_KMERS, W_H2D_BYTES, W_D2H_BYTES, W_REFINED, W_BT2_READS, N_WORK };
extern const char* const WORK_NAMES[N_WORK];

// Host-side phase clock, printed per batch when SHMAP_HOSTPROF is set.
struct HostClock {
    bool on;
    std::chrono::steady_clock::time_point t0, last;
    std::string line;
    HostClock() : on(std::getenv("SHMAP_HOSTPROF") != nullptr) {
        if (on) t0 = last = std::chrono::steady_clock::now();
    }
    void mark(const char* what) {
        if (!on) return;
        auto now = std::chrono::steady_clock::now();
        char b[64];
        std::snprintf(b, sizeof b, " %s=%.3f", what, std::chrono::duration<double, std::milli>(now - last).count());
        line += b;
        last = now;
    }
    void print(const char* tag, int32_t n) {
        if (!on) return;
        std::fprintf(stderr, "[shmap-host] %s n=%d total=%.3f%s\n", tag, n,
                     std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count(),
                     line.c_str());
    }
};

struct MapCtx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;  // host-to-device copies of the next batch
    cudaEvent_t copied[2] = {nullptr, nullptr};
    cudaEvent_t sketched[2] = {nullptr, nullptr};  // the sketch of the batch in each buffer has read it
    // host-form batches sent up as bytes: their own stream and two buffers, so
    // their copies run beside the packed batches' without waiting in line
    cudaStream_t raw_stream = nullptr;
    cudaEvent_t raw_copied[2] = {nullptr, nullptr};
    cudaEvent_t raw_sketched[2] = {nullptr, nullptr};
    std::vector<cudaEvent_t> up_ev;  // the streamed host form: one per chunk uploaded in a call
    StreamSink* sink = nullptr;      // the streamed host form with pieces sent by the packing threads
    cudaEvent_t sketch_done = nullptr;             // recorded by run_batch after its sketch when set
    cudaStream_t side_stream = nullptr;  // seed preparation of the few reads with large sketches
    cudaEvent_t fork = nullptr, join = nullptr;
    MapScratch* scr = nullptr;
    PafScratch* paf = nullptr;
    size_t hbm_budget = 0;
    int64_t launches = 0;
    // host staging (pinned): the plan of the batch in flight, small readbacks
    uint8_t* h_pinned = nullptr;
    size_t h_pinned_cap = 0;
    void* h_slots = nullptr;  // per-call batch results
    size_t h_slots_cap = 0;
    uint8_t* h_pack = nullptr;  // two slots of packed reads (codes, mask) on their way up
    size_t h_pack_cap = 0;
    // work counters (always on): see WORK_NAMES
    int64_t work[16] = {};
    int seed_smem_set = 0;   // dynamic shared memory the seed kernels have been allowed so far
    int rchip_smem_set = 0;  // k_refine_chip's dynamic shared memory allowed
    int refine_smem_set = 0; // k_refine's
    int seedc_smem_set = 0;
    // stage timing
    bool timing = false;
    double stage_ms[N_STAGES] = {};
    int64_t stage_calls[N_STAGES] = {};
    std::vector<cudaEvent_t> ev_pool;
};

MapCtx* mapctx_create(int device, size_t hbm_budget);
void mapctx_destroy(MapCtx* c);

// Maps reads [0, n) whose bytes are at d_seq (device) with host offsets
// h_offs[0..n] (h_offs[0] may be nonzero: bytes are relative to d_seq - h_offs[0]).
// Writes n records to d_out (device). plain = one read per launch sequence.
void map_device(MapCtx* c, const IndexStorage* ix, const shm_params& p, const uint8_t* d_seq, const int64_t* h_offs,
                int32_t n, shm_map_record* d_out, bool plain);

// Takes each batch's records while they are still on the device: batch(i, j,
// d_rec, s) is called, in batch order, right after reads [i, j) are mapped,
// with their records at d_rec (device) valid for work queued on stream s.
struct BatchSink {
    virtual void batch(int32_t i, int32_t j, const shm_map_record* d_rec, cudaStream_t s) = 0;
    // called between batches: work that waits for earlier batches, without blocking
    virtual void poll() {}
    virtual ~BatchSink() = default;
};

// Host-buffer form: copies each batch in, maps it, copies records out. With a
// sink, returns true when some records changed after the sink had taken them
// (a batch mapped again with exact sizes, or reads retried); out then holds
// the final records.
bool map_host(MapCtx* c, const IndexStorage* ix, const shm_params& p, const uint8_t* seqs, const int64_t* offs,
              int32_t n, shm_map_record* out, bool plain, BatchSink* sink = nullptr);

}  // namespace shm
