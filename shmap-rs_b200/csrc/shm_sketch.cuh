// Device FracMinHash sketching (see shm_sketch.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace shm {

enum SketchMode { SK_APPEND = 0, SK_COUNT = 1, SK_WRITE = 2 };

// Sequences are concatenated in `seq` (device, padded by 16 bytes, 16-byte
// aligned base) with seq_off[n_seq+1]. chunk_off[n_seq+1] is the prefix of
// ceil(windows / SKETCH_WIN) per sequence.
//  - SK_APPEND: unordered output per sequence into [kmer_off[q], kmer_off[q+1]),
//    counted in kmer_cnt[q] (which may exceed the capacity: caller checks).
//  - SK_COUNT: chunk_cnt[c] = selected windows of chunk c.
//  - SK_WRITE: writes chunk c's selections in order from chunk_out[c].
struct SketchArgs {
    const uint8_t* seq;
    const int64_t* seq_off;
    const uint64_t* chunk_off;
    int32_t n_seq;
    uint64_t n_chunks;
    int32_t k;
    uint64_t thr;
    int32_t r_offset;  // added to every r (sketch_slice_into's `offset`)
    // SK_APPEND
    const uint64_t* kmer_off;
    uint32_t* kmer_cnt;
    // SK_COUNT / SK_WRITE
    uint32_t* chunk_cnt;
    const uint32_t* chunk_out;  // n_chunks+1 exclusive offsets (total < 2^32)
    // outputs
    uint64_t* out_h;
    uint32_t* out_rs;  // r << 1 | strand
    // SK_APPEND only: when set, the reads come as 2-bit codes and a non-ACGT
    // mask instead of `seq` (the layout of host/pack.hpp: base p, relative to
    // the batch, is bits 2(p & 15) of pk_codes[p >> 4], masked when bit p & 31
    // of pk_mask[p >> 5] is set; two spare groups of 32 past the end)
    const uint32_t* pk_codes;
    const uint32_t* pk_mask;
    uint64_t pk_words;  // code words readable at pk_codes (those past it read as 0)
};

// The five lookup tables of src/sketch.rs:50-97 for one k, in device memory
// (owned by the caller, released with cudaFree).
struct SketchLuts;
SketchLuts* create_device_luts(int32_t k, cudaStream_t s);
void launch_sketch(int mode, const SketchArgs& a, const SketchLuts* luts, cudaStream_t s);

// Builds the tables on the device into caller-provided device memory of
// sketch_luts_bytes() bytes (8-byte aligned); no host copy, no allocation.
size_t sketch_luts_bytes();
void launch_fill_luts(SketchLuts* d, int32_t k, cudaStream_t s);

}  // namespace shm
