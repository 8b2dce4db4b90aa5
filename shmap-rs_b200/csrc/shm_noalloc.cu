// shm_sketch_device_noalloc: FracMinHash sketching of one device-resident
// sequence that allocates no memory at all.
//
// Who needs it: callers that must not allocate device memory on this path —
// for example a host program whose device memory is fully reserved by its own
// pool allocator (a cudaMalloc here would fail or escape that pool's
// accounting), or a latency-critical loop that cannot afford cudaMalloc /
// cudaFree, which may synchronize the whole device. Such a caller passes its
// own input and output buffers; every temporary this call needs lives in the
// file-scope array below.
//
// The array is static device memory: every GPU that loads this library holds
// its NOALLOC_SCRATCH_BYTES (about 0.5 MiB) from load until process exit.
// Every call shares it and it keeps the last call's contents; calls that
// overlap on the GPU (on different streams, or from several host threads)
// race on it and must be serialized by the caller.
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/shmap_gpu.h"
#include "shm_common.cuh"
#include "shm_internal.hpp"
#include "shm_prims.cuh"
#include "shm_sketch.cuh"

namespace {

// Largest input: NOALLOC_MAX_CHUNKS runs of SKETCH_WIN windows.
constexpr int64_t NOALLOC_MAX_CHUNKS = 1 << 16;
constexpr int64_t NOALLOC_MAX_WINDOWS = 4194304;
static_assert(NOALLOC_MAX_WINDOWS <= NOALLOC_MAX_CHUNKS * shm::SKETCH_WIN, "scratch holds every run of the limit");
constexpr size_t NOALLOC_LUT_BYTES = 5 * 256 * 8;                              // the five lookup tables
constexpr size_t NOALLOC_OFF_BYTES = 64;                                       // seq_off[2], chunk_off[2]
constexpr size_t NOALLOC_SCRATCH_BYTES =
    NOALLOC_LUT_BYTES + NOALLOC_OFF_BYTES + 4 * NOALLOC_MAX_CHUNKS + 4 * (NOALLOC_MAX_CHUNKS + 16);

// The scratch: lookup tables | offsets | per-run counts | per-run output offsets (+ total).
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// In host code `g_noalloc_scratch` names a host-side shadow, not device
// memory: its device address comes from cudaGetSymbolAddress, taken once per
// device (with that device current) on the first call there.
std::mutex g_mu;
void* g_addr[64] = {};

int fail(int code, const std::string& m) {
    shm::set_last_error(m);
    return code;
}

__global__ void k_noalloc_offsets(int64_t* seq_off, uint64_t* chunk_off, int64_t len, uint64_t n_chunks) {
    if (threadIdx.x == 0) {
        seq_off[0] = 0;
        seq_off[1] = len;
        chunk_off[0] = 0;
        chunk_off[1] = n_chunks;
    }
}

// Exclusive scan of at most NOALLOC_MAX_CHUNKS counts in one block; out[n] = total.
__global__ void __launch_bounds__(1024) k_noalloc_scan(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                       uint32_t n) {
    __shared__ uint32_t wsum[32];
    const uint32_t per = (n + blockDim.x - 1) / blockDim.x;
    const uint32_t a = min(n, threadIdx.x * per), b = min(n, a + per);
    uint32_t s = 0;
    for (uint32_t i = a; i < b; i++) s += in[i];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t inc = shm::warp_inclusive_scan(s);
    if (lane == 31) wsum[w] = inc;
    __syncthreads();
    if (w == 0) {
        uint32_t x = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0;
        uint32_t xi = shm::warp_inclusive_scan(x);
        wsum[lane] = xi - x;
        if (lane == 31) out[n] = xi;
    }
    __syncthreads();
    uint32_t run = wsum[w] + inc - s;
    for (uint32_t i = a; i < b; i++) {
        out[i] = run;
        run += in[i];
    }
}

}  // namespace

extern "C" int shm_sketch_device_noalloc(const uint8_t* d_seq, int64_t len, int32_t k, double h_frac,
                                         int32_t offset, uint64_t* d_h, uint32_t* d_rs, int64_t cap,
                                         int64_t* n_out, void* stream) {
    if (!n_out) return fail(SHM_ERR_INVALID, "n_out is null");
    *n_out = 0;
    if (k <= 0) return fail(SHM_ERR_INVALID, "K-mer length (-k) should be positive.");
    if (len < 0 || (len > 0 && !d_seq)) return fail(SHM_ERR_INVALID, "bad input sequence");
    if (((uintptr_t)d_seq & 15) != 0) return fail(SHM_ERR_INVALID, "d_seq must be 16-byte aligned");
    if (len < k) return SHM_OK;
    const int64_t nw = len - k + 1;
    if (nw > NOALLOC_MAX_WINDOWS)
        return fail(SHM_ERR_INVALID, "sequence too long for shm_sketch_device_noalloc: " + std::to_string(nw) +
                                         " windows, the limit is " + std::to_string(NOALLOC_MAX_WINDOWS) +
                                         " (length " + std::to_string(NOALLOC_MAX_WINDOWS + k - 1) + ")");
    if (cap > 0 && (!d_h || !d_rs)) return fail(SHM_ERR_INVALID, "output buffers are null");
    if (shm::sketch_luts_bytes() != NOALLOC_LUT_BYTES) return fail(SHM_ERR_INVALID, "lookup table layout changed");
    cudaStream_t s = (cudaStream_t)stream;
    try {
        int dev = 0;
        SHM_CUDA(cudaGetDevice(&dev));
        if (dev < 0 || dev >= 64) return fail(SHM_ERR_INVALID, "device index out of range");
        unsigned char* base;
        {
            std::lock_guard<std::mutex> lk(g_mu);
            if (!g_addr[dev]) {
                void* p = nullptr;
                cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
                if (e != cudaSuccess || !p)
                    return fail(SHM_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
                g_addr[dev] = p;
            }
            base = (unsigned char*)g_addr[dev];
        }
        auto* luts = (shm::SketchLuts*)base;
        auto* seq_off = (int64_t*)(base + NOALLOC_LUT_BYTES);
        auto* chunk_off = (uint64_t*)(base + NOALLOC_LUT_BYTES + 16);
        auto* cnt = (uint32_t*)(base + NOALLOC_LUT_BYTES + NOALLOC_OFF_BYTES);
        auto* outo = cnt + NOALLOC_MAX_CHUNKS;
        const uint64_t n_chunks = (uint64_t)((nw + shm::SKETCH_WIN - 1) / shm::SKETCH_WIN);
        // nothing here has to start at zero: every slot read below is written first in this call
        shm::launch_fill_luts(luts, k, s);
        k_noalloc_offsets<<<1, 32, 0, s>>>(seq_off, chunk_off, len, n_chunks);
        SHM_CUDA(cudaGetLastError());
        shm::SketchArgs a{};
        a.seq = d_seq;
        a.seq_off = seq_off;
        a.chunk_off = chunk_off;
        a.n_seq = 1;
        a.n_chunks = n_chunks;
        a.k = k;
        a.thr = shm::h_thres(h_frac);
        a.r_offset = offset;
        a.chunk_cnt = cnt;
        shm::launch_sketch(shm::SK_COUNT, a, luts, s);
        k_noalloc_scan<<<1, 1024, 0, s>>>(cnt, outo, (uint32_t)n_chunks);
        SHM_CUDA(cudaGetLastError());
        uint32_t total = 0;
        SHM_CUDA(cudaMemcpyAsync(&total, outo + n_chunks, sizeof total, cudaMemcpyDeviceToHost, s));
        SHM_CUDA(cudaStreamSynchronize(s));
        *n_out = total;
        if ((int64_t)total > cap) return fail(SHM_ERR_CAPACITY, "output capacity too small");
        a.chunk_out = outo;
        a.out_h = d_h;
        a.out_rs = d_rs;
        shm::launch_sketch(shm::SK_WRITE, a, luts, s);
        SHM_CUDA(cudaStreamSynchronize(s));
        return SHM_OK;
    } catch (const shm_cuda_error& e) {
        return fail(SHM_ERR_CUDA, cudaGetErrorString(e.err));
    }
}
