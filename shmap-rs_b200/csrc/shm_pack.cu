// Reads packed on the device: ASCII bases in device memory to the 2-bit codes
// and non-ACGT mask of host/pack.hpp (the layout the host-buffer path
// uploads), so reads parsed or kept on the device are sketched from codes too.
// Codes: a byte b of ACGT in either case has code (b >> 1) & 3 (A 0, C 1,
// T 2, G 3); base p is bits 2(p & 15) of codes[p >> 4]. Mask: bit p & 31 of
// mask[p >> 5] is set for every other byte (those hash to 0 on both strands,
// src/sketch.rs:58-97) and for positions past the end.
//
// A byte is ACGT iff its upper-cased value equals the letter its code names,
// 0x41 + 2c (+ 15 for c = 2, T); four bytes of a word are tested at once
// with byte-wise integer arithmetic that never carries between bytes.
#include "shm_common.cuh"
#include "shm_pack.cuh"
#include "shm_prims.cuh"

namespace shm {

namespace {

// Codes of the word's four bytes (8 bits, byte 0 in bits 0-1) and its
// non-ACGT bits (bit i for byte i).
__device__ __forceinline__ void pack_word(uint32_t w, uint32_t& code8, uint32_t& bad4) {
    const uint32_t c = (w >> 1) & 0x03030303u;
    const uint32_t is_t = (c >> 1) & ~c & 0x01010101u;  // code 2 (T)
    const uint32_t want = 0x41414141u + c + c + (is_t << 4) - is_t;
    const uint32_t d = (w & 0xdfdfdfdfu) ^ want;  // zero bytes: ACGT
    // bit 7 of a byte set iff the byte is nonzero (no carry leaves a byte)
    const uint32_t nz = (((d & 0x7f7f7f7fu) + 0x7f7f7f7fu) | d) & 0x80808080u;
    bad4 = ((nz >> 7) * 0x01020408u) >> 24;
    const uint32_t x = c | (c >> 6);
    code8 = (x | (x >> 12)) & 0xffu;
}

// Group g of 32 bases: bytes [32g, 32g + 32) of seq (nb bytes; seq + nb has
// 16 readable bytes). Past nb: code 0, masked. SW = (seq & 15) >> 2, the
// whole words the start lies past a 16-byte boundary (the same for every
// group, since groups are 32 bytes apart).
template <int SW>
__global__ void __launch_bounds__(256) k_pack_ascii(const uint8_t* __restrict__ seq, int64_t nb, int64_t n_groups,
                                                   uint32_t* __restrict__ codes, uint32_t* __restrict__ mask) {
    const uintptr_t mis = (uintptr_t)seq & 15u;
    const uint8_t* A = seq - mis;  // 16-byte aligned
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n_groups; g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b0 = 32 * g;
        uint32_t w[8];
        if (b0 + 32 <= nb) {
            // bytes [mis + b0, mis + b0 + 32) of A: three aligned 16-byte loads
            // (the third stays inside the 16 readable bytes past the end)
            const uint4* v = (const uint4*)(A + mis + b0 - ((mis + b0) & 15));
            const uint4 u0 = __ldg(v), u1 = __ldg(v + 1);
            const uint4 u2 = ((mis + b0) & 15) ? __ldg(v + 2) : make_uint4(0, 0, 0, 0);
            const uint32_t a[12] = {u0.x, u0.y, u0.z, u0.w, u1.x, u1.y, u1.z, u1.w, u2.x, u2.y, u2.z, u2.w};
            const uint32_t sb = (uint32_t)(mis & 3) * 8;
#pragma unroll
            for (int i = 0; i < 8; i++) w[i] = __funnelshift_r(a[i + SW], a[i + SW + 1], sb);
        } else {
#pragma unroll
            for (int i = 0; i < 8; i++) {
                uint32_t x = 0;
                for (int j = 0; j < 4; j++) {
                    const int64_t p = b0 + 4 * i + j;
                    x |= (p < nb ? (uint32_t)seq[p] : 0u) << (8 * j);
                }
                w[i] = x;
            }
        }
        uint32_t c0 = 0, c1 = 0, m = 0;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            uint32_t c8, b4;
            pack_word(w[i], c8, b4);
            if (i < 4) c0 |= c8 << (8 * i);
            else c1 |= c8 << (8 * (i - 4));
            m |= b4 << (4 * i);
        }
        if (b0 + 32 > nb) {  // positions past the end are masked, code 0
            const int64_t valid = nb > b0 ? nb - b0 : 0;
            const uint32_t keep = valid >= 32 ? ~0u : (valid <= 0 ? 0u : ((1u << valid) - 1u));
            m = (m & keep) | ~keep;
            const uint64_t ck = valid >= 32 ? ~0ull : (valid <= 0 ? 0ull : ((1ull << (2 * valid)) - 1ull));
            c0 &= (uint32_t)ck;
            c1 &= (uint32_t)(ck >> 32);
        }
        codes[2 * g] = c0;
        codes[2 * g + 1] = c1;
        mask[g] = m;
    }
}

}  // namespace

void pack_reads_device(const uint8_t* seq, int64_t nb, uint32_t* codes, uint32_t* mask, cudaStream_t s) {
    const int64_t n_groups = nb / 32 + 3;  // packed_mask_words(nb): two spare groups past the end
    const int grid = grid_for((size_t)n_groups, 256, 8);
    switch (((uintptr_t)seq & 15u) >> 2) {
        case 0: k_pack_ascii<0><<<grid, 256, 0, s>>>(seq, nb, n_groups, codes, mask); break;
        case 1: k_pack_ascii<1><<<grid, 256, 0, s>>>(seq, nb, n_groups, codes, mask); break;
        case 2: k_pack_ascii<2><<<grid, 256, 0, s>>>(seq, nb, n_groups, codes, mask); break;
        default: k_pack_ascii<3><<<grid, 256, 0, s>>>(seq, nb, n_groups, codes, mask); break;
    }
    SHM_CUDA(cudaGetLastError());
    count_launch();
}

cudaError_t pack_groups_device(const uint8_t* seq, int64_t n_groups, uint32_t* codes, uint32_t* mask,
                               cudaStream_t s) {
    if (n_groups <= 0) return cudaSuccess;
    if (((uintptr_t)seq & 15u) != 0) return cudaErrorInvalidValue;
    k_pack_ascii<0><<<grid_for((size_t)n_groups, 256, 8), 256, 0, s>>>(seq, 32 * n_groups, n_groups, codes, mask);
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) count_launch();
    return e;
}

}  // namespace shm

// Test hook (not part of the C ABI of include/shmap_gpu.h): nb bytes of host
// memory packed on `device` into caller buffers of packed_code_words(nb) and
// packed_mask_words(nb) words (host memory).
#include <vector>

extern "C" int shm_internal_pack_reads_device(int device, const uint8_t* seq, int64_t nb, uint32_t* codes,
                                              uint32_t* mask) {
    if (nb < 0 || (nb > 0 && !seq) || !codes || !mask) return -1;
    uint8_t* d_seq = nullptr;
    uint32_t *d_c = nullptr, *d_m = nullptr;
    const size_t ng = (size_t)(nb / 32 + 3);
    int rc = 0;
    try {
        SHM_CUDA(cudaSetDevice(device));
        // an odd start, so the unaligned loads are exercised
        SHM_CUDA(cudaMalloc(&d_seq, (size_t)nb + 64));
        SHM_CUDA(cudaMemset(d_seq, 0x55, (size_t)nb + 64));
        if (nb) SHM_CUDA(cudaMemcpy(d_seq + 3, seq, (size_t)nb, cudaMemcpyHostToDevice));
        SHM_CUDA(cudaMalloc(&d_c, 8 * ng));
        SHM_CUDA(cudaMalloc(&d_m, 4 * ng));
        shm::pack_reads_device(d_seq + 3, nb, d_c, d_m, nullptr);
        SHM_CUDA(cudaDeviceSynchronize());
        SHM_CUDA(cudaMemcpy(codes, d_c, 8 * ng, cudaMemcpyDeviceToHost));
        SHM_CUDA(cudaMemcpy(mask, d_m, 4 * ng, cudaMemcpyDeviceToHost));
    } catch (const shm_cuda_error&) {
        rc = -2;
    }
    cudaFree(d_seq);
    cudaFree(d_c);
    cudaFree(d_m);
    return rc;
}
