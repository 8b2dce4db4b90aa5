// Exclusive scan (reduce / scan-of-sums / apply, recursive) and the stable LSD
// radix sort used to build the reference index on the device.
#include <algorithm>
#include <atomic>
#include <cstdio>

#include "shm_common.cuh"
#include "shm_prims.cuh"

#include <mutex>

namespace shm {

// Temporaries of the primitives come from one stream-ordered pool per device
// that keeps its memory (release threshold: never), so that a call after a
// synchronize does not map the pool's memory again.
static cudaMemPool_t prim_pool() {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    int dev = 0;
    SHM_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> g(mu);
    if (dev < 0 || dev >= 64) throw shm_cuda_error(cudaErrorInvalidDevice);
    if (!pools[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        SHM_CUDA(cudaMemPoolCreate(&pools[dev], &props));
        uint64_t keep = UINT64_MAX;
        SHM_CUDA(cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep));
    }
    return pools[dev];
}

template <class T>
static void pool_alloc(T** p, size_t bytes, cudaStream_t s) {
    SHM_CUDA(cudaMallocFromPoolAsync((void**)p, bytes, prim_pool(), s));
}


static int g_num_sms = 0;
static std::atomic<int64_t> g_launches{0};

int64_t kernel_launches() { return g_launches.load(); }
void count_launch(int64_t n) { g_launches.fetch_add(n); }

int grid_for(size_t work, int block, int max_blocks_per_sm) {
    if (g_num_sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
        if (g_num_sms <= 0) g_num_sms = 148;
    }
    size_t want = (work + (size_t)block - 1) / (size_t)block;
    size_t cap = (size_t)g_num_sms * (size_t)max_blocks_per_sm;
    size_t g = std::min(std::max<size_t>(want, 1), cap);
    return (int)g;
}

// ------------------------------------------------------------------ scan
constexpr int SCAN_THREADS = 512;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

template <class T>
__device__ T block_exclusive_scan(T v, T* warp_tot, T* total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    T inc = warp_inclusive_scan(v);
    if (lane == 31) warp_tot[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        T w = (lane < (SCAN_THREADS >> 5)) ? warp_tot[lane] : T(0);
        T wi = warp_inclusive_scan(w);
        if (lane < (SCAN_THREADS >> 5)) warp_tot[lane] = wi - w;
        if (lane == (SCAN_THREADS >> 5) - 1) *total = wi;
    }
    __syncthreads();
    T r = warp_tot[wid] + inc - v;
    __syncthreads();
    return r;
}

template <class T>
__global__ void k_scan_reduce(const T* __restrict__ in, size_t n, T* __restrict__ sums) {
    __shared__ T wt[32];
    __shared__ T tot;
    size_t base = (size_t)blockIdx.x * SCAN_TILE + (size_t)threadIdx.x * SCAN_ITEMS;
    T s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++)
        if (base + i < n) s += in[base + i];
    block_exclusive_scan<T>(s, wt, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

template <class T>
__global__ void k_scan_apply(const T* __restrict__ in, size_t n, const T* __restrict__ block_off, T* __restrict__ out,
                             bool write_total) {
    __shared__ T wt[32];
    __shared__ T tot;
    size_t base = (size_t)blockIdx.x * SCAN_TILE + (size_t)threadIdx.x * SCAN_ITEMS;
    T loc[SCAN_ITEMS];
    T s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        loc[i] = (base + i < n) ? in[base + i] : T(0);
        s += loc[i];
    }
    T ex = block_exclusive_scan<T>(s, wt, &tot);
    T off = (block_off ? block_off[blockIdx.x] : T(0)) + ex;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        if (base + i < n) out[base + i] = off;
        off += loc[i];
    }
    if (write_total && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) {
        T t = (block_off ? block_off[blockIdx.x] : T(0)) + tot;
        out[n] = t;
    }
}

template <class T>
static void exclusive_scan_impl(const T* in, T* out, size_t n, cudaStream_t s) {
    if (n == 0) {
        SHM_CUDA(cudaMemsetAsync(out, 0, sizeof(T), s));
        return;
    }
    size_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (nb == 1) {
        k_scan_apply<T><<<1, SCAN_THREADS, 0, s>>>(in, n, nullptr, out, true);
        SHM_CUDA(cudaGetLastError());
        count_launch();
        return;
    }
    T* sums = nullptr;
    pool_alloc(&sums, sizeof(T) * (nb + 1), s);
    k_scan_reduce<T><<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, n, sums);
    SHM_CUDA(cudaGetLastError());
    exclusive_scan_impl<T>(sums, sums, nb, s);  // in-place is safe: each level reads before it writes per tile
    k_scan_apply<T><<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, n, sums, out, true);
    SHM_CUDA(cudaGetLastError());
    count_launch(2);
    SHM_CUDA(cudaFreeAsync(sums, s));
}

void exclusive_scan_u32(const uint32_t* in, uint32_t* out, size_t n, cudaStream_t s) {
    exclusive_scan_impl<uint32_t>(in, out, n, s);
}
void exclusive_scan_u64(const uint64_t* in, uint64_t* out, size_t n, cudaStream_t s) {
    exclusive_scan_impl<uint64_t>(in, out, n, s);
}

// ------------------------------------------------------------------ radix sort
constexpr int RS_THREADS = 256;                 // 8 warps
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_STEPS = 8;                     // 32-element steps per warp
constexpr int RS_TILE = RS_THREADS * RS_STEPS;  // 2048 elements per block
constexpr int RS_BINS = 256;

__global__ void k_rs_hist(const uint64_t* __restrict__ keys, size_t n, int shift, uint32_t* __restrict__ hist,
                          uint32_t nblocks) {
    __shared__ uint32_t h[RS_BINS];
    for (int i = threadIdx.x; i < RS_BINS; i += blockDim.x) h[i] = 0;
    __syncthreads();
    size_t base = (size_t)blockIdx.x * RS_TILE;
    for (int i = threadIdx.x; i < RS_TILE; i += blockDim.x) {
        size_t j = base + (size_t)i;
        if (j < n) atomicAdd(&h[(keys[j] >> shift) & 0xff], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < RS_BINS; d += blockDim.x) hist[(size_t)d * nblocks + blockIdx.x] = h[d];
}

// Stable scatter: warp w ranks its 8 consecutive 32-element steps in order
// (match_any gives the rank among equal digits inside a step), then warps are
// ordered by a per-digit prefix over the block.
__global__ void k_rs_scatter(const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin, size_t n, int shift,
                             const uint32_t* __restrict__ off, uint32_t nblocks, uint64_t* __restrict__ kout,
                             uint32_t* __restrict__ vout) {
    __shared__ uint32_t cnt[RS_WARPS][RS_BINS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int i = lane; i < RS_BINS; i += 32) cnt[w][i] = 0;
    __syncwarp();
    const size_t base = (size_t)blockIdx.x * RS_TILE + (size_t)w * (RS_STEPS * 32);
    uint64_t key[RS_STEPS];
    uint32_t val[RS_STEPS], rank[RS_STEPS];
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int s = 0; s < RS_STEPS; s++) {
        size_t j = base + (size_t)s * 32 + lane;
        bool valid = j < n;
        unsigned vmask = __ballot_sync(0xffffffffu, valid);
        key[s] = valid ? kin[j] : 0;
        val[s] = valid ? vin[j] : 0;
        uint32_t d = (uint32_t)((key[s] >> shift) & 0xff);
        rank[s] = 0;
        if (valid) {
            unsigned peers = __match_any_sync(vmask, d);
            uint32_t before = cnt[w][d];
            rank[s] = before + __popc(peers & lt);
            __syncwarp(vmask);
            if ((peers & lt) == 0) cnt[w][d] = before + __popc(peers);
        }
        __syncwarp();
    }
    __syncthreads();
    // exclusive prefix of counts over warps, per digit
    for (int d = threadIdx.x; d < RS_BINS; d += blockDim.x) {
        uint32_t acc = 0;
        for (int ww = 0; ww < RS_WARPS; ww++) {
            uint32_t c = cnt[ww][d];
            cnt[ww][d] = acc;
            acc += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < RS_STEPS; s++) {
        size_t j = base + (size_t)s * 32 + lane;
        if (j < n) {
            uint32_t d = (uint32_t)((key[s] >> shift) & 0xff);
            uint32_t dst = off[(size_t)d * nblocks + blockIdx.x] + cnt[w][d] + rank[s];
            kout[dst] = key[s];
            vout[dst] = val[s];
        }
    }
}

bool radix_sort_pairs(uint64_t* k0, uint32_t* v0, uint64_t* k1, uint32_t* v1, size_t n, int key_bits,
                      cudaStream_t s) {
    if (n <= 1 || key_bits <= 0) return false;
    if (n >= (size_t)UINT32_MAX) {
        std::fprintf(stderr, "shmap-b200: radix sort of %zu elements exceeds 32-bit offsets\n", n);
        throw shm_cuda_error(cudaErrorInvalidValue);
    }
    const uint32_t nb = (uint32_t)((n + RS_TILE - 1) / RS_TILE);
    uint32_t *hist = nullptr, *off = nullptr;
    pool_alloc(&hist, sizeof(uint32_t) * (size_t)RS_BINS * nb, s);
    pool_alloc(&off, sizeof(uint32_t) * ((size_t)RS_BINS * nb + 1), s);
    bool flipped = false;
    for (int shift = 0; shift < key_bits; shift += 8) {
        uint64_t* ki = flipped ? k1 : k0;
        uint32_t* vi = flipped ? v1 : v0;
        uint64_t* ko = flipped ? k0 : k1;
        uint32_t* vo = flipped ? v0 : v1;
        k_rs_hist<<<nb, RS_THREADS, 0, s>>>(ki, n, shift, hist, nb);
        SHM_CUDA(cudaGetLastError());
        exclusive_scan_u32(hist, off, (size_t)RS_BINS * nb, s);
        k_rs_scatter<<<nb, RS_THREADS, 0, s>>>(ki, vi, n, shift, off, nb, ko, vo);
        SHM_CUDA(cudaGetLastError());
        count_launch(2);
        flipped = !flipped;
    }
    SHM_CUDA(cudaFreeAsync(hist, s));
    SHM_CUDA(cudaFreeAsync(off, s));
    return flipped;
}

}  // namespace shm
