// Shared definitions of the B200 mapping path: the device index layout, the
// per-batch buffers and small device helpers. Everything here is integer
// except the f64 scores, which use explicit round-to-nearest intrinsics so the
// compiler can never contract them (the reference computes them in plain
// IEEE f64: src/shmap/pruning.rs:10-13, src/shmap/scoring.rs:172-178).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>

#define SHM_CUDA(call)                                                                    \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            std::fprintf(stderr, "shmap-b200: CUDA error %s at %s:%d: %s\n", #call,      \
                         __FILE__, __LINE__, cudaGetErrorString(e_));                     \
            throw shm_cuda_error(e_);                                                     \
        }                                                                                 \
    } while (0)

struct shm_cuda_error {
    cudaError_t err;
    explicit shm_cuda_error(cudaError_t e) : err(e) {}
};

namespace shm {

constexpr int SKETCH_WIN = 128;          // windows rolled by one thread
constexpr int MIN_HALFLEN = 5;           // src/buckets.rs:15
constexpr uint64_t EMPTY_KEY = ~0ULL;    // empty slot of the per-read hash tables
constexpr int SEED_SMEM_MAX = 4096;      // largest sketch sorted in shared memory

// Per-read status codes written into the output record.
enum ReadStatus : int32_t {
    ST_MAPPED = 0,
    ST_UNMAPPED = 1,          // nothing cleared the threshold
    ST_SHORT_SKETCH = 2,      // sketch below MIN_HALFLEN (src/shmap/mod.rs:750-783)
    ST_OVERFLOW = 3,          // a per-read capacity was exceeded; the host retries
};

// The reference index on the device (replaces the 8 FxHashMap shards of
// src/index.rs:104-125). Reference k-mers are stored once, in (segment, tpos)
// order, so a hit is just its global k-mer id `gidx`; ordering hits by gidx
// is ordering by (segm_id, r), the order of src/index.rs:300.
struct DevIndex {
    int32_t k;
    int32_t n_seg;
    uint64_t thr;             // FracMinHash::h_thres (src/sketch.rs:126-132)
    const uint32_t* seg_off;  // n_seg+1: first gidx of each segment's sketch
    const int32_t* seg_sz;    // n_seg: segment length in bases
    const uint64_t* ref_h;    // n_kmers: canonical hash of each reference k-mer
    const uint32_t* ref_rs;   // n_kmers: r << 1 | strand
    const uint64_t* keys;     // n_keys: distinct hashes, ascending
    const uint32_t* key_off;  // n_keys+1: start of each hash's hit list in `hits`
    const uint32_t* hits;     // n_hits: gidx, ascending within a list
    const uint32_t* hit_fw;   // n_hits+1: prefix count of forward-strand hits
    const uint32_t* dir;      // (1 << dir_bits) + 1: first key of each hash range
    int32_t dir_bits;
    uint64_t dir_mul;         // range of h: __umul64hi(h, dir_mul), monotone, < 2^dir_bits for h <= thr
    // Bucket table (null when thr is all ones): 1 << btab_bits buckets of two
    // uint4, bucket __umul64hi(h, btab_mul) holding the first two keys of its
    // hash range in key order, {key0, key1} then {a0, cnt0, a1, cnt1 | more << 31};
    // an empty slot has key ~0 (no hash <= thr) and count 0, and `more` says
    // the range has further keys (all above key1), found through dir.
    const uint4* btab;
    int32_t btab_bits;
    uint64_t btab_mul;
    uint32_t n_keys, n_kmers, n_hits;
};

// Mapping parameters as the device sees them (src/params.rs:20-186).
struct DevParams {
    int32_t k;
    uint64_t thr;
    double theta, min_diff, max_overlap;
    double theta_low;  // fl(theta * fl(1 - min_diff)): lowest threshold either sweep can use
    int32_t metric;    // 0 Containment, 1 Jaccard, 2 bucket_SH
    int32_t nbp, os, ap;
    // slot_mul[b] = min(2^64 - 1, floor(2^(64+b) / (thr + 1))): __umul64hi(h, slot_mul[b])
    // maps h <= thr monotonically onto [0, 2^b)
    uint64_t slot_mul[16];
    // rarity (src/shmap/mod.rs:694-723, scoring.rs:214-281, 409-481): when on,
    // a seed of c hits weighs wtab[c] = max(c, 1)^-alpha (the host's pow;
    // c < wtab_n), and refinement reports each bucket's weighted support
    int32_t rarity;     // a rarity flag is on
    int32_t rw_score;   // --rarity-weight: the score is the weighted containment
    double tiebreak;    // --rarity-tiebreak band (0 = off)
    const double* wtab;
    uint32_t wtab_n;
};

// The last i in [0, n) with off[i] <= key (off[0] = 0 <= key), by one warp:
// each step tests 32 evenly spaced places at once, so n = 2^17 sequences
// take four dependent loads instead of seventeen.
__device__ __forceinline__ int32_t warp_last_le(const uint64_t* __restrict__ off, int32_t n, uint64_t key, int lane) {
    int32_t lo = 0, hi = n;  // the answer lies in [lo, hi)
    while (hi - lo > 1) {
        const int32_t step = (hi - lo + 31) / 32;
        const int32_t i = lo + lane * step;
        const unsigned b = __ballot_sync(0xffffffffu, i < hi && __ldg(off + i) <= key);  // bit 0 is set
        lo += (31 - __clz(b)) * step;
        hi = min(hi, lo + step);
    }
    return lo;
}

__device__ __forceinline__ uint64_t rotl64(uint64_t x, uint32_t n) {
    n &= 63;
    return n ? (x << n) | (x >> (64 - n)) : x;
}
__device__ __forceinline__ uint64_t rotr64(uint64_t x, uint32_t n) {
    n &= 63;
    return n ? (x >> n) | (x << (64 - n)) : x;
}
__device__ __forceinline__ uint64_t mix64(uint64_t h) {
    h ^= h >> 31;
    h *= 0x7fb5d329728ea185ULL;
    h ^= h >> 27;
    h *= 0x81dadef4bc2dd44dULL;
    return h ^ (h >> 33);
}

// Segment of a reference k-mer id (upper_bound over seg_off).
__device__ __forceinline__ int32_t seg_of(const DevIndex& I, uint32_t g) {
    int32_t lo = 0, hi = I.n_seg;  // seg_off[lo] <= g < seg_off[hi]
    while (hi - lo > 1) {
        int32_t mid = (lo + hi) >> 1;
        if (__ldg(I.seg_off + mid) <= g) lo = mid;
        else hi = mid;
    }
    return lo;
}

// The same over a copy of seg_off (for instance in shared memory).
__device__ __forceinline__ int32_t seg_of_in(const uint32_t* seg_off, int32_t n_seg, uint32_t g) {
    int32_t lo = 0, hi = n_seg;
    while (hi - lo > 1) {
        int32_t mid = (lo + hi) >> 1;
        if (seg_off[mid] <= g) lo = mid;
        else hi = mid;
    }
    return lo;
}

// The hash-range search of idx_lookup, through the directory and the keys.
__device__ __forceinline__ bool idx_lookup_dir(const DevIndex& I, uint64_t h, uint32_t& a, uint32_t& cnt) {
    uint32_t b = (uint32_t)__umul64hi(h, I.dir_mul);
    uint32_t lo = __ldg(I.dir + b), hi = __ldg(I.dir + b + 1);
    while (hi - lo > 8) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(I.keys + mid) <= h) lo = mid;
        else hi = mid;
    }
    for (uint32_t i = lo; i < hi; i++) {
        uint64_t kk = __ldg(I.keys + i);
        if (kk == h) {
            a = __ldg(I.key_off + i);
            cnt = __ldg(I.key_off + i + 1) - a;
            return true;
        }
        if (kk > h) break;
    }
    return false;
}

// The bucket of h in the bucket table (I.btab non-null, h <= thr).
__device__ __forceinline__ const uint4* btab_bucket(const DevIndex& I, uint64_t h) {
    return I.btab + 2 * (size_t)__umul64hi(h, I.btab_mul);
}

// Looks h up among a bucket's two keys k = {key0, key1}: returns the slot
// (0 or 1) holding h, 2 when h may be among the range's further keys (key1
// is present and below h: the slot's `more` flag decides), -1 when absent.
__device__ __forceinline__ int btab_slot(uint4 k, uint64_t h) {
    const uint64_t k0 = ((uint64_t)k.y << 32) | k.x, k1 = ((uint64_t)k.w << 32) | k.z;
    if (k0 == h) return 0;
    if (k1 == h) return 1;
    return (k1 != ~0ULL && h > k1) ? 2 : -1;
}

// SketchIndex::count + hit-list lookup (src/index.rs:192-213): the bucket
// table first (one 32-byte sector), the directory for the rest of a crowded
// range.
__device__ __forceinline__ bool idx_lookup(const DevIndex& I, uint64_t h, uint32_t& a, uint32_t& cnt) {
    cnt = 0;
    a = 0;
    if (h > I.thr || I.n_keys == 0) return false;
    if (I.btab) {
        const uint4* p = btab_bucket(I, h);
        const int sl = btab_slot(__ldg(p), h);
        if (sl < 0) return false;
        const uint4 ac = __ldg(p + 1);
        if (sl == 0) {
            a = ac.x;
            cnt = ac.y;
            return true;
        }
        if (sl == 1) {
            a = ac.z;
            cnt = ac.w & 0x7fffffffu;
            return true;
        }
        if (!(ac.w >> 31)) return false;
    }
    return idx_lookup_dir(I, h, a, cnt);
}

// First index in hits[a, a+n) with hits[i] >= v.
__device__ __forceinline__ uint32_t hits_lower_bound(const uint32_t* __restrict__ hits, uint32_t a, uint32_t n,
                                                     uint32_t v) {
    uint32_t lo = a, len = n;
    while (len > 0) {
        uint32_t half = len >> 1;
        if (__ldg(hits + lo + half) < v) {
            lo += half + 1;
            len -= half + 1;
        } else {
            len = half;
        }
    }
    return lo;
}

// hseed (src/shmap/pruning.rs:10-13): 1 - (seeds - matches) / p in IEEE f64.
__device__ __forceinline__ double hseed(int32_t p, int32_t seeds, int32_t matches) {
    return __dsub_rn(1.0, __ddiv_rn((double)(seeds - matches), (double)p));
}

template <class T>
__device__ __forceinline__ T warp_inclusive_scan(T v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T n = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += n;
    }
    return v;
}

}  // namespace shm
