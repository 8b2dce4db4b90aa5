// Host-side objects behind the C ABI (context, index, batch scratch).
#pragma once
#include <cuda_runtime.h>
#include <cstdio>
#include <cstdlib>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/shmap_gpu.h"
#include "shm_common.cuh"
#include "shm_sketch.cuh"

namespace shm {

uint64_t h_thres(double h_frac);  // src/sketch.rs:126-132

// Sets the message shm_last_error() returns on this thread.
void set_last_error(const std::string& m);

// A device buffer that only grows; released by the destructor.
template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t cap = 0;  // elements
    // Grows (never shrinks). Queued work may still use the old buffer, so a
    // growth waits for the device first; a buffer that grows again takes a
    // quarter more than asked, so that batches of varying size (a server's)
    // stop growing it soon.
    void reserve(size_t n) {
        if (n <= cap && p) return;
        if (p) {
            SHM_CUDA(cudaDeviceSynchronize());
            SHM_CUDA(cudaFree(p));
            n += n / 4;
        }
        if (std::getenv("SHMAP_HOSTPROF"))
            std::fprintf(stderr, "[shmap-host] grow %zu -> %zu bytes\n", cap * sizeof(T), n * sizeof(T));
        p = nullptr;
        size_t want = n < 16 ? 16 : n;
        SHM_CUDA(cudaMalloc(&p, want * sizeof(T)));
        cap = want;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    ~DevBuf() { release(); }
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
};

struct IndexStorage {
    DevIndex dev{};
    DevBuf<uint32_t> seg_off, key_off, hits, hit_fw, dir, ref_rs;
    DevBuf<int32_t> seg_sz;
    DevBuf<uint64_t> ref_h, keys;
    DevBuf<uint4> btab;
    std::vector<std::string> names;
    std::vector<int32_t> seg_len;        // bases
    std::vector<uint32_t> h_seg_off;     // k-mer offsets (n_seg+1)
    shm_index_stats stats{};
    int32_t k = 0;
    double h_frac = 0;
    int32_t max_matches = -1;
    int device = 0;
    uint32_t max_list = 0;  // longest hit list of the index
};

// An index written to a file and read back (shm_index.cu); failures throw
// IndexFileError with a message.
struct IndexFileError {
    std::string what;
};
void save_index(const IndexStorage* ix, const char* path);
IndexStorage* load_index(const char* path, cudaStream_t s);
// The checks load_index makes, on the host alone (no device is touched).
void check_index_file(const char* path);

// The segments' bases are read from h_seq (host) or, when d_seq is given,
// from device memory (d_seq + seg_off[i], 32 readable bytes past the end).
IndexStorage* build_index(const uint8_t* h_seq, const int64_t* seg_off, int32_t n_seg,
                          const std::vector<std::string>& names, int32_t k, double h_frac, int32_t max_matches,
                          cudaStream_t s, const uint8_t* d_seq = nullptr);

}  // namespace shm

// The opaque handles of the C ABI.
struct shm_index {
    shm::IndexStorage* s;
};
