// FracMinHash sketching on the device: FracMinHash::sketch_slice_into
// (src/sketch.rs:167-209) split into runs of SKETCH_WIN windows, one run per
// thread. A run starts from the directly computed hash of its first window
// (the definition the reference pins in tests/nthash_equivalence.rs:31-61) and
// rolls the rest, so the concatenated runs equal the serial sketch
// (src/sketch.rs:232-270 pins exactly that property for any split).
//
// Bytes are read through 16-byte aligned vector loads into a small register
// window; the five pre-rotated lookup tables of src/sketch.rs:50-97 live in
// shared memory, indexed by the raw byte (so case and non-ACGT bytes behave as
// in the reference: lower/upper case alike, every other byte hashes to 0).
#include "shm_common.cuh"
#include "shm_prims.cuh"
#include "shm_sketch.cuh"

namespace shm {

struct SketchLuts {
    uint64_t fw[256], rc[256], fw_k[256], rc_r1[256], rc_k1[256];
};

// Built on the host once per (k) exactly as src/sketch.rs:58-108 does.
void build_luts(int32_t k, SketchLuts* L) {
    const uint64_t A = 0x3c8bfbb395c60474ULL, C = 0x3193c18562a02b4cULL, G = 0x20323ed082572324ULL,
                   T = 0x295549f54be24456ULL;
    for (int c = 0; c < 256; c++) L->fw[c] = L->rc[c] = 0;
    const unsigned char lo[4] = {'a', 'c', 'g', 't'}, up[4] = {'A', 'C', 'G', 'T'};
    const uint64_t v[4] = {A, C, G, T};
    for (int i = 0; i < 4; i++) L->fw[lo[i]] = L->fw[up[i]] = v[i];
    for (int i = 0; i < 4; i++) L->rc[lo[i]] = L->rc[up[i]] = v[3 - i];  // complement: A<->T, C<->G
    auto rl = [](uint64_t x, uint32_t n) { n &= 63; return n ? (x << n) | (x >> (64 - n)) : x; };
    auto rr = [](uint64_t x, uint32_t n) { n &= 63; return n ? (x >> n) | (x << (64 - n)) : x; };
    for (int c = 0; c < 256; c++) {
        L->fw_k[c] = rl(L->fw[c], (uint32_t)k);
        L->rc_r1[c] = rr(L->rc[c], 1);
        L->rc_k1[c] = rl(L->rc[c], (uint32_t)(k - 1));
    }
}

// Fixed 64-bit rotates by one (two funnel shifts each).
__device__ __forceinline__ uint64_t rotl1(uint64_t x) {
    uint32_t lo = (uint32_t)x, hi = (uint32_t)(x >> 32);
    return ((uint64_t)__funnelshift_l(lo, hi, 1) << 32) | __funnelshift_l(hi, lo, 1);
}
__device__ __forceinline__ uint64_t rotr1(uint64_t x) {
    uint32_t lo = (uint32_t)x, hi = (uint32_t)(x >> 32);
    return ((uint64_t)__funnelshift_r(hi, lo, 1) << 32) | __funnelshift_r(lo, hi, 1);
}

// One selected window: record it by the kernel's mode.
template <int MODE>
__device__ __forceinline__ void emit_kmer(const SketchArgs& a, int32_t q, uint64_t h, uint32_t rs, uint64_t out_base,
                                          uint32_t out_cap, uint32_t& n_sel) {
    if (MODE == SK_COUNT) {
        n_sel++;
    } else if (MODE == SK_WRITE) {
        a.out_h[out_base + n_sel] = h;
        a.out_rs[out_base + n_sel] = rs;
        n_sel++;
    } else {
        uint32_t slot = atomicAdd(a.kmer_cnt + q, 1u);
        if (slot < out_cap) {
            a.out_h[out_base + slot] = h;
            a.out_rs[out_base + slot] = rs;
        }
    }
}

template <int MODE>
__global__ void __launch_bounds__(256) k_sketch(SketchArgs a, const SketchLuts* __restrict__ luts) {
    __shared__ SketchLuts L;
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        L.fw[i] = luts->fw[i];
        L.rc[i] = luts->rc[i];
        L.fw_k[i] = luts->fw_k[i];
        L.rc_r1[i] = luts->rc_r1[i];
        L.rc_k1[i] = luts->rc_k1[i];
    }
    __syncthreads();
    const int k = a.k;
    const uint64_t thr = a.thr;
    const uint64_t n_chunks = a.n_chunks;
    for (uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n_chunks;
         c += (uint64_t)gridDim.x * blockDim.x) {
        // sequence of this chunk: upper_bound over chunk_off
        int32_t lo = 0, hi = a.n_seq;
        while (hi - lo > 1) {
            int32_t mid = (lo + hi) >> 1;
            if (__ldg(a.chunk_off + mid) <= c) lo = mid;
            else hi = mid;
        }
        const int32_t q = lo;
        const int64_t s0 = __ldg(a.seq_off + q), L_ = __ldg(a.seq_off + q + 1) - s0;
        const int64_t nw = L_ - k + 1;
        const int64_t w0 = (int64_t)(c - __ldg(a.chunk_off + q)) * SKETCH_WIN;
        const int32_t cnt = (int32_t)(min(w0 + (int64_t)SKETCH_WIN, nw) - w0);  // windows of this run
        if (cnt <= 0) continue;
        uint64_t out_base = 0;
        uint32_t out_cap = 0;
        uint32_t n_sel = 0;
        if (MODE == SK_WRITE) out_base = a.chunk_out[c];
        if (MODE == SK_APPEND) {
            out_base = a.kmer_off[q];
            out_cap = (uint32_t)(a.kmer_off[q + 1] - out_base);
        }
        const uint8_t* p = a.seq + (s0 + w0);
        const int32_t r0 = (int32_t)(w0 + k - 1) + a.r_offset;  // r of the run's first window
        // first window, by definition (tests/nthash_equivalence.rs:31-61)
        uint64_t fw = 0, rc = 0;
        for (int i = 0; i < k; i++) {
            uint32_t b = __ldg(p + i);
            fw ^= rotl64(L.fw[b], (uint32_t)(k - 1 - i));
            rc ^= rotl64(L.rc[b], (uint32_t)i);
        }
        {
            const uint64_t h = fw ^ rc;
            if (h <= thr) emit_kmer<MODE>(a, q, h, ((uint32_t)r0 << 1) | (fw > rc ? 1u : 0u), out_base, out_cap, n_sel);
        }
        // rolling: window t takes base p[t + k - 1] in and drops p[t - 1]; both byte
        // streams are read as aligned 32-bit words realigned by one funnel shift
        const uintptr_t ai = (uintptr_t)(p + k), ao = (uintptr_t)p;
        const uint32_t shi = (uint32_t)(ai & 3) * 8, sho = (uint32_t)(ao & 3) * 8;
        const uint32_t* wi = (const uint32_t*)(ai & ~(uintptr_t)3);
        const uint32_t* wo = (const uint32_t*)(ao & ~(uintptr_t)3);
        uint32_t li = __ldg(wi), lo_ = __ldg(wo);
        for (int32_t t = 1; t < cnt; t += 4) {
            const uint32_t hi_i = __ldg(++wi), hi_o = __ldg(++wo);
            const uint32_t ib4 = __funnelshift_r(li, hi_i, shi), ob4 = __funnelshift_r(lo_, hi_o, sho);
            li = hi_i;
            lo_ = hi_o;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                if (t + j < cnt) {
                    const uint32_t ib = (ib4 >> (8 * j)) & 0xffu, ob = (ob4 >> (8 * j)) & 0xffu;
                    fw = rotl1(fw) ^ L.fw_k[ob] ^ L.fw[ib];
                    rc = rotr1(rc) ^ L.rc_r1[ob] ^ L.rc_k1[ib];
                    const uint64_t h = fw ^ rc;
                    if (h <= thr)
                        emit_kmer<MODE>(a, q, h, ((uint32_t)(r0 + t + j) << 1) | (fw > rc ? 1u : 0u), out_base,
                                        out_cap, n_sel);
                }
            }
        }
        if (MODE == SK_COUNT) a.chunk_cnt[c] = n_sel;
    }
}

SketchLuts* create_device_luts(int32_t k, cudaStream_t s) {
    SketchLuts h;
    build_luts(k, &h);
    SketchLuts* d = nullptr;
    SHM_CUDA(cudaMalloc(&d, sizeof(SketchLuts)));
    SHM_CUDA(cudaMemcpyAsync(d, &h, sizeof h, cudaMemcpyHostToDevice, s));
    SHM_CUDA(cudaStreamSynchronize(s));
    return d;
}

void launch_sketch(int mode, const SketchArgs& a, const SketchLuts* L, cudaStream_t s) {
    if (a.n_chunks == 0) return;
    int grid = grid_for(a.n_chunks, 256, 8);
    if (mode == SK_COUNT) k_sketch<SK_COUNT><<<grid, 256, 0, s>>>(a, L);
    else if (mode == SK_WRITE) k_sketch<SK_WRITE><<<grid, 256, 0, s>>>(a, L);
    else k_sketch<SK_APPEND><<<grid, 256, 0, s>>>(a, L);
    SHM_CUDA(cudaGetLastError());
    count_launch();
}

}  // namespace shm

namespace shm {

// The same five tables as build_luts, computed on the device (for callers
// that may not copy from the host or allocate).
__global__ void k_fill_luts(SketchLuts* L, int32_t k) {
    const uint64_t v[4] = {0x3c8bfbb395c60474ULL, 0x3193c18562a02b4cULL, 0x20323ed082572324ULL,
                           0x295549f54be24456ULL};
    for (int c = threadIdx.x; c < 256; c += blockDim.x) {
        int fi = -1;
        switch (c) {
            case 'A': case 'a': fi = 0; break;
            case 'C': case 'c': fi = 1; break;
            case 'G': case 'g': fi = 2; break;
            case 'T': case 't': fi = 3; break;
        }
        uint64_t fw = fi >= 0 ? v[fi] : 0, rc = fi >= 0 ? v[3 - fi] : 0;
        L->fw[c] = fw;
        L->rc[c] = rc;
        L->fw_k[c] = rotl64(fw, (uint32_t)k);
        L->rc_r1[c] = rotr64(rc, 1);
        L->rc_k1[c] = rotl64(rc, (uint32_t)(k - 1));
    }
}

size_t sketch_luts_bytes() { return sizeof(SketchLuts); }

void launch_fill_luts(SketchLuts* d, int32_t k, cudaStream_t s) {
    k_fill_luts<<<1, 256, 0, s>>>(d, k);
    SHM_CUDA(cudaGetLastError());
    count_launch();
}

}  // namespace shm
