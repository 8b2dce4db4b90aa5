// The reference index built on the device (SketchIndex::build_index,
// src/index.rs:384-663).
//
// 1. Every segment is sketched in order (count, scan, write) so reference
//    k-mer ids (gidx) run in (segment file order, tpos) order.
// 2. (hash, gidx) pairs are radix-sorted stably by hash: each hash's hits come
//    out in gidx order = (segm_id, r) order, the order finalize_shard gives its
//    multi-hit lists (src/index.rs:295-315).
// 3. Runs of equal hashes become a CSR (keys, key_off, hits). With -M, the
//    reference keeps the first min(n, M+2) hits of a hash (insert_hit's cap,
//    src/index.rs:286-288, plus the migrated single hit) and then erases every
//    list longer than M (src/index.rs:360-376): a hash survives iff n <= M.
// 4. hit_fw is the prefix count of forward-strand hits (codirection sums of a
//    hit range in O(1)); dir maps the top bits of a hash to its first key.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "shm_common.cuh"
#include "shm_internal.hpp"
#include "shm_prims.cuh"
#include "shm_sketch.cuh"

namespace shm {

uint64_t h_thres(double h_frac) {
    if (h_frac < 1.0) {
        double x = h_frac * (double)UINT64_MAX;
        if (std::isnan(x) || x <= 0.0) return 0;
        if (x >= 18446744073709551616.0) return UINT64_MAX;
        return (uint64_t)x;
    }
    return UINT64_MAX;
}

__global__ void k_iota(uint32_t* v, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        v[i] = (uint32_t)i;
}

__global__ void k_seg_offsets(const uint64_t* __restrict__ chunk_off, const uint32_t* __restrict__ chunk_out,
                              int32_t n_seg, uint32_t* __restrict__ seg_off) {
    for (int32_t s = blockIdx.x * blockDim.x + threadIdx.x; s <= n_seg; s += gridDim.x * blockDim.x)
        seg_off[s] = chunk_out[chunk_off[s]];
}

__global__ void k_key_flags(const uint64_t* __restrict__ ks, size_t n, uint32_t* __restrict__ flag) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        flag[i] = (i == 0 || ks[i] != ks[i - 1]) ? 1u : 0u;
}

__global__ void k_key_emit(const uint64_t* __restrict__ ks, size_t n, const uint32_t* __restrict__ fscan,
                           uint64_t* __restrict__ keys, uint32_t* __restrict__ key_off) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        if (i == 0 || ks[i] != ks[i - 1]) {
            uint32_t j = fscan[i];
            keys[j] = ks[i];
            key_off[j] = (uint32_t)i;
        }
    }
}

struct IdxStatsDev {
    unsigned long long indexed_hits, blacklisted_kmers, blacklisted_hits, kept_keys, kept_hits;
    unsigned int highest;
};

// Per-key cap/erase decision and statistics (src/index.rs:264-291, 343-376).
__global__ void k_key_keep(const uint32_t* __restrict__ key_off, uint32_t n_keys, int32_t max_matches,
                           uint32_t* __restrict__ keep, uint32_t* __restrict__ keep_hits, IdxStatsDev* st) {
    unsigned long long ih = 0, bk = 0, bh = 0;
    unsigned int hi = 0;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n_keys; j += gridDim.x * blockDim.x) {
        uint32_t len = key_off[j + 1] - key_off[j];
        uint32_t capped = len;
        bool kept = true;
        if (max_matches >= 0) {
            uint32_t cap = (uint32_t)max_matches + 2u;
            capped = len < cap ? len : cap;
            kept = len <= (uint32_t)max_matches;
        }
        ih += capped;
        hi = capped > hi ? capped : hi;
        if (!kept) {
            bk += 1;
            bh += capped;
        }
        keep[j] = kept ? 1u : 0u;
        keep_hits[j] = kept ? len : 0u;
    }
    atomicAdd(&st->indexed_hits, ih);
    atomicAdd(&st->blacklisted_kmers, bk);
    atomicAdd(&st->blacklisted_hits, bh);
    atomicMax(&st->highest, hi);
}

// Moves the kept keys and their hit lists to their compacted places.
__global__ void k_compact_keys(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ key_off,
                               uint32_t n_keys, const uint32_t* __restrict__ keep_scan,
                               const uint32_t* __restrict__ hits_scan, uint64_t* __restrict__ nkeys,
                               uint32_t* __restrict__ nkey_off) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n_keys; j += gridDim.x * blockDim.x) {
        if (keep_scan[j + 1] != keep_scan[j]) {
            nkeys[keep_scan[j]] = keys[j];
            nkey_off[keep_scan[j]] = hits_scan[j];
        }
    }
}

// Per hit: its key id (from the inclusive flag scan) and its compacted place.
__global__ void k_compact_hits(const uint32_t* __restrict__ vals, size_t n, const uint32_t* __restrict__ fscan,
                               const uint32_t* __restrict__ flag, const uint32_t* __restrict__ key_off,
                               const uint32_t* __restrict__ keep_scan, const uint32_t* __restrict__ hits_scan,
                               uint32_t* __restrict__ nhits) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        uint32_t kid = fscan[i] + flag[i] - 1u;
        if (keep_scan[kid + 1] != keep_scan[kid]) nhits[hits_scan[kid] + ((uint32_t)i - key_off[kid])] = vals[i];
    }
}

__global__ void k_fw_flags(const uint32_t* __restrict__ hits, size_t n, const uint32_t* __restrict__ ref_rs,
                           uint32_t* __restrict__ f) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        f[i] = (ref_rs[hits[i]] & 1u) ? 0u : 1u;
}

__device__ __forceinline__ int64_t dir_bucket(uint64_t h, uint64_t mul) { return (int64_t)__umul64hi(h, mul); }

// dir[b] = first key whose range is >= b; the ranges past the last key point at n_keys.
__global__ void k_dir_fill(const uint64_t* __restrict__ keys, uint32_t n_keys, uint32_t* __restrict__ dir,
                           int64_t nb, uint64_t mul) {
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, nthreads = (int64_t)gridDim.x * blockDim.x;
    const int64_t blast = n_keys ? dir_bucket(keys[n_keys - 1], mul) : -1;
    for (int64_t b = blast + 1 + tid; b <= nb; b += nthreads) dir[b] = n_keys;
    for (int64_t i = tid; i < (int64_t)n_keys; i += nthreads) {
        int64_t bi = dir_bucket(keys[i], mul);
        int64_t bp = i > 0 ? dir_bucket(keys[i - 1], mul) : -1;
        for (int64_t b = bp + 1; b <= bi; b++) dir[b] = (uint32_t)i;
    }
}

// The bucket table (DevIndex::btab) over the sorted keys: every key finds its
// rank in its bucket from its two predecessors (the keys are sorted and the
// bucket map is monotone), so each slot has one writer.
__global__ void k_btab_clear(uint4* __restrict__ bt, int64_t nb) {
    for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += (int64_t)gridDim.x * blockDim.x) {
        bt[2 * b] = make_uint4(~0u, ~0u, ~0u, ~0u);
        bt[2 * b + 1] = make_uint4(0u, 0u, 0u, 0u);
    }
}
__global__ void k_btab_fill(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ key_off, uint32_t n_keys,
                            uint4* __restrict__ bt, uint64_t mul) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (int64_t)n_keys;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t h = keys[i];
        const uint64_t b = __umul64hi(h, mul);
        const bool p1 = i > 0 && __umul64hi(keys[i - 1], mul) == b;
        if (p1 && i > 1 && __umul64hi(keys[i - 2], mul) == b) continue;  // third or later: through dir
        const uint32_t a = key_off[i], c = key_off[i + 1] - a;
        uint32_t* q0 = (uint32_t*)(bt + 2 * b);
        uint32_t* q1 = (uint32_t*)(bt + 2 * b + 1);
        if (!p1) {
            q0[0] = (uint32_t)h;
            q0[1] = (uint32_t)(h >> 32);
            q1[0] = a;
            q1[1] = c;
        } else {
            const bool more = i + 1 < (int64_t)n_keys && __umul64hi(keys[i + 1], mul) == b;
            q0[2] = (uint32_t)h;
            q0[3] = (uint32_t)(h >> 32);
            q1[2] = a;
            q1[3] = c | (more ? 0x80000000u : 0u);
        }
    }
}

// The arrays derived from the reference k-mers and the CSR (forward-strand
// prefix of the hits, hash directory, bucket table) and the device view;
// build_index and load_index end here. ix holds k, the segments, ref_h,
// ref_rs, keys[n_kept], key_off[n_kept+1] and hits[n_hits] on the device.
static void finish_index(IndexStorage* ix, uint64_t thr, uint32_t n_kept, uint32_t n_kmers, uint32_t n_hits,
                         uint32_t highest, cudaStream_t s) {
    DevBuf<uint32_t> flag;
    flag.reserve((size_t)n_hits + 1);
    ix->hit_fw.reserve((size_t)n_hits + 1);
    k_fw_flags<<<grid_for(n_hits, 256), 256, 0, s>>>(ix->hits.p, n_hits, ix->ref_rs.p, flag.p);
    SHM_CUDA(cudaGetLastError());
    exclusive_scan_u32(flag.p, ix->hit_fw.p, n_hits, s);
    int bits = 1;
    while (bits < 30 && (1u << bits) < n_kept) bits++;
    const int64_t nb = (int64_t)1 << bits;
    // mul = floor(2^64 * nb / (thr + 1)): h <= thr maps monotonically onto [0, nb)
    unsigned __int128 m128 = ((unsigned __int128)nb << 64) / ((unsigned __int128)thr + 1);
    const uint64_t mul = m128 > (unsigned __int128)UINT64_MAX ? UINT64_MAX : (uint64_t)m128;
    ix->dir.reserve((size_t)nb + 1);
    k_dir_fill<<<grid_for((size_t)std::max<int64_t>(nb, (int64_t)n_kept), 256), 256, 0, s>>>(ix->keys.p, n_kept,
                                                                                           ix->dir.p, nb, mul);
    SHM_CUDA(cudaGetLastError());
    // the bucket table: two buckets per key (at most 2^28), when no hash is
    // all ones (thr below the maximum) and every count fits in 31 bits
    int tbits = 0;
    uint64_t tmul = 0;
    if (thr != UINT64_MAX && n_kept > 0 && highest < (1u << 31)) {
        tbits = std::min(bits + 1, 28);
        const int64_t nt = (int64_t)1 << tbits;
        unsigned __int128 t128 = ((unsigned __int128)nt << 64) / ((unsigned __int128)thr + 1);
        tmul = t128 > (unsigned __int128)UINT64_MAX ? UINT64_MAX : (uint64_t)t128;
        ix->btab.reserve(2 * (size_t)nt);
        k_btab_clear<<<grid_for((size_t)nt, 256), 256, 0, s>>>(ix->btab.p, nt);
        SHM_CUDA(cudaGetLastError());
        k_btab_fill<<<grid_for((size_t)n_kept, 256), 256, 0, s>>>(ix->keys.p, ix->key_off.p, n_kept, ix->btab.p,
                                                                 tmul);
        SHM_CUDA(cudaGetLastError());
    }
    SHM_CUDA(cudaStreamSynchronize(s));

    DevIndex& d = ix->dev;
    d.k = ix->k;
    d.n_seg = (int32_t)ix->seg_len.size();
    d.thr = thr;
    d.seg_off = ix->seg_off.p;
    d.seg_sz = ix->seg_sz.p;
    d.ref_h = ix->ref_h.p;
    d.ref_rs = ix->ref_rs.p;
    d.keys = ix->keys.p;
    d.key_off = ix->key_off.p;
    d.hits = ix->hits.p;
    d.hit_fw = ix->hit_fw.p;
    d.dir = ix->dir.p;
    d.dir_bits = bits;
    d.dir_mul = mul;
    d.btab = tbits ? ix->btab.p : nullptr;
    d.btab_bits = tbits;
    d.btab_mul = tmul;
    d.n_keys = n_kept;
    d.n_kmers = n_kmers;
    d.n_hits = n_hits;
}

IndexStorage* build_index(const uint8_t* h_seq, const int64_t* seg_off_b, int32_t n_seg,
                          const std::vector<std::string>& names, int32_t k, double h_frac, int32_t max_matches,
                          cudaStream_t s, const uint8_t* d_seq_in) {
    auto* ix = new IndexStorage();
    try {
        SHM_CUDA(cudaGetDevice(&ix->device));
        ix->k = k;
        ix->h_frac = h_frac;
        ix->max_matches = max_matches;
        ix->names = names;
        const uint64_t thr = h_thres(h_frac);
        const int64_t total_bases = seg_off_b[n_seg] - seg_off_b[0];

        // chunk layout per segment (host)
        std::vector<uint64_t> chunk_off((size_t)n_seg + 1, 0);
        std::vector<int64_t> soff((size_t)n_seg + 1, 0);
        for (int32_t i = 0; i < n_seg; i++) {
            int64_t L = seg_off_b[i + 1] - seg_off_b[i];
            soff[(size_t)i + 1] = soff[(size_t)i] + L;
            ix->seg_len.push_back((int32_t)L);
            int64_t nw = L - k + 1;
            uint64_t ch = nw > 0 ? (uint64_t)((nw + SKETCH_WIN - 1) / SKETCH_WIN) : 0;
            chunk_off[(size_t)i + 1] = chunk_off[(size_t)i] + ch;
        }
        const uint64_t n_chunks = chunk_off[(size_t)n_seg];

        DevBuf<uint8_t> d_seq;
        DevBuf<int64_t> d_soff;
        DevBuf<uint64_t> d_chunk_off;
        DevBuf<uint32_t> d_ccnt, d_cout;
        if (!d_seq_in) {
            d_seq.reserve((size_t)total_bases + 32);
            SHM_CUDA(cudaMemsetAsync(d_seq.p + total_bases, 0, 32, s));
            SHM_CUDA(cudaMemcpyAsync(d_seq.p, h_seq + seg_off_b[0], (size_t)total_bases, cudaMemcpyHostToDevice, s));
        }
        d_soff.reserve((size_t)n_seg + 1);
        SHM_CUDA(cudaMemcpyAsync(d_soff.p, soff.data(), sizeof(int64_t) * ((size_t)n_seg + 1), cudaMemcpyHostToDevice, s));
        d_chunk_off.reserve((size_t)n_seg + 1);
        SHM_CUDA(cudaMemcpyAsync(d_chunk_off.p, chunk_off.data(), sizeof(uint64_t) * ((size_t)n_seg + 1),
                                 cudaMemcpyHostToDevice, s));
        d_ccnt.reserve(n_chunks + 1);
        d_cout.reserve(n_chunks + 1);

        SketchLuts* luts = create_device_luts(k, s);
        SketchArgs a{};
        a.seq = d_seq_in ? d_seq_in + seg_off_b[0] : d_seq.p;
        a.seq_off = d_soff.p;
        a.chunk_off = d_chunk_off.p;
        a.n_seq = n_seg;
        a.n_chunks = n_chunks;
        a.k = k;
        a.thr = thr;
        a.r_offset = 0;
        a.chunk_cnt = d_ccnt.p;
        launch_sketch(SK_COUNT, a, luts, s);
        exclusive_scan_u32(d_ccnt.p, d_cout.p, n_chunks, s);
        uint32_t n_kmers = 0;
        SHM_CUDA(cudaMemcpyAsync(&n_kmers, d_cout.p + n_chunks, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        SHM_CUDA(cudaStreamSynchronize(s));
        ix->ref_h.reserve((size_t)n_kmers + 1);
        ix->ref_rs.reserve((size_t)n_kmers + 1);
        a.chunk_out = d_cout.p;
        a.out_h = ix->ref_h.p;
        a.out_rs = ix->ref_rs.p;
        launch_sketch(SK_WRITE, a, luts, s);
        ix->seg_off.reserve((size_t)n_seg + 1);
        k_seg_offsets<<<grid_for((size_t)n_seg + 1, 128), 128, 0, s>>>(d_chunk_off.p, d_cout.p, n_seg, ix->seg_off.p);
        SHM_CUDA(cudaGetLastError());
        SHM_CUDA(cudaFree(luts));
        d_seq.release();
        d_ccnt.release();
        d_cout.release();
        ix->h_seg_off.resize((size_t)n_seg + 1);
        SHM_CUDA(cudaMemcpyAsync(ix->h_seg_off.data(), ix->seg_off.p, sizeof(uint32_t) * ((size_t)n_seg + 1),
                                 cudaMemcpyDeviceToHost, s));
        ix->seg_sz.reserve((size_t)n_seg + 1);
        SHM_CUDA(cudaMemcpyAsync(ix->seg_sz.p, ix->seg_len.data(), sizeof(int32_t) * (size_t)n_seg,
                                 cudaMemcpyHostToDevice, s));

        // 2. stable sort of (hash, gidx) by hash
        const size_t n = n_kmers;
        DevBuf<uint64_t> k0, k1;
        DevBuf<uint32_t> v0, v1;
        k0.reserve(n + 1);
        k1.reserve(n + 1);
        v0.reserve(n + 1);
        v1.reserve(n + 1);
        SHM_CUDA(cudaMemcpyAsync(k0.p, ix->ref_h.p, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, s));
        k_iota<<<grid_for(n, 256), 256, 0, s>>>(v0.p, n);
        SHM_CUDA(cudaGetLastError());
        int key_bits = thr == 0 ? 0 : 64 - __builtin_clzll(thr);
        bool flipped = radix_sort_pairs(k0.p, v0.p, k1.p, v1.p, n, key_bits, s);
        uint64_t* ks = flipped ? k1.p : k0.p;
        uint32_t* vals = flipped ? v1.p : v0.p;

        // 3. CSR over runs of equal hashes
        DevBuf<uint32_t> flag, fscan;
        flag.reserve(n + 1);
        fscan.reserve(n + 1);
        k_key_flags<<<grid_for(n, 256), 256, 0, s>>>(ks, n, flag.p);
        SHM_CUDA(cudaGetLastError());
        exclusive_scan_u32(flag.p, fscan.p, n, s);
        uint32_t n_keys = 0;
        SHM_CUDA(cudaMemcpyAsync(&n_keys, fscan.p + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        SHM_CUDA(cudaStreamSynchronize(s));
        DevBuf<uint64_t> keys_all;
        DevBuf<uint32_t> key_off_all;
        keys_all.reserve((size_t)n_keys + 1);
        key_off_all.reserve((size_t)n_keys + 1);
        k_key_emit<<<grid_for(n, 256), 256, 0, s>>>(ks, n, fscan.p, keys_all.p, key_off_all.p);
        SHM_CUDA(cudaGetLastError());
        uint32_t nn = (uint32_t)n;
        SHM_CUDA(cudaMemcpyAsync(key_off_all.p + n_keys, &nn, sizeof(uint32_t), cudaMemcpyHostToDevice, s));

        IdxStatsDev* dst = nullptr;
        SHM_CUDA(cudaMallocAsync(&dst, sizeof(IdxStatsDev), s));
        SHM_CUDA(cudaMemsetAsync(dst, 0, sizeof(IdxStatsDev), s));
        DevBuf<uint32_t> keep, keep_hits, keep_scan, hits_scan;
        keep.reserve((size_t)n_keys + 1);
        keep_hits.reserve((size_t)n_keys + 1);
        keep_scan.reserve((size_t)n_keys + 1);
        hits_scan.reserve((size_t)n_keys + 1);
        k_key_keep<<<grid_for(n_keys, 256), 256, 0, s>>>(key_off_all.p, n_keys, max_matches, keep.p, keep_hits.p, dst);
        SHM_CUDA(cudaGetLastError());
        IdxStatsDev hst{};
        SHM_CUDA(cudaMemcpyAsync(&hst, dst, sizeof hst, cudaMemcpyDeviceToHost, s));
        SHM_CUDA(cudaFreeAsync(dst, s));
        exclusive_scan_u32(keep.p, keep_scan.p, n_keys, s);
        exclusive_scan_u32(keep_hits.p, hits_scan.p, n_keys, s);
        uint32_t n_kept = 0, n_hits = 0;
        SHM_CUDA(cudaMemcpyAsync(&n_kept, keep_scan.p + n_keys, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        SHM_CUDA(cudaMemcpyAsync(&n_hits, hits_scan.p + n_keys, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        SHM_CUDA(cudaStreamSynchronize(s));

        ix->keys.reserve((size_t)n_kept + 1);
        ix->key_off.reserve((size_t)n_kept + 1);
        ix->hits.reserve((size_t)n_hits + 1);
        k_compact_keys<<<grid_for(n_keys, 256), 256, 0, s>>>(keys_all.p, key_off_all.p, n_keys, keep_scan.p,
                                                             hits_scan.p, ix->keys.p, ix->key_off.p);
        SHM_CUDA(cudaGetLastError());
        SHM_CUDA(cudaMemcpyAsync(ix->key_off.p + n_kept, &n_hits, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
        k_compact_hits<<<grid_for(n, 256), 256, 0, s>>>(vals, n, fscan.p, flag.p, key_off_all.p, keep_scan.p,
                                                        hits_scan.p, ix->hits.p);
        SHM_CUDA(cudaGetLastError());

        // 4. forward-strand prefix, hash directory, bucket table, device view
        // the longest hit list kept: -M erases every list longer than M
        ix->max_list = max_matches > 0 ? std::min<uint32_t>(hst.highest, (uint32_t)max_matches) : hst.highest;
        finish_index(ix, thr, n_kept, n_kmers, n_hits, hst.highest, s);

        shm_index_stats& st = ix->stats;
        st.segments = n_seg;
        st.total_nucls = total_bases;
        st.indexed_hits = (int64_t)hst.indexed_hits;
        st.indexed_kmers = n_keys;
        st.highest_freq_kmer = hst.highest;
        st.blacklisted_kmers = (int64_t)hst.blacklisted_kmers;
        st.blacklisted_hits = (int64_t)hst.blacklisted_hits;
        st.sketched_kmers = n_kmers;
        return ix;
    } catch (...) {
        delete ix;
        throw;
    }
}

// ------------------------------------------------------------------ index files
// A built index written to a file and read back, so that a service can start
// mapping without the reference's sequence and without rebuilding (the
// reference itself sketches and indexes on every run, src/main.rs:45-57).
// The file holds what the index answers from: the segments, every reference
// k-mer and the CSR over distinct hashes; the derived arrays (forward-strand
// prefix, directory, bucket table) are rebuilt on load by finish_index.
// Layout, little endian, no padding:
//   "SHMAPIX1", u32 version = 2, i32 k, f64 h_frac, i32 max_matches,
//   i32 n_seg, u32 n_keys, u32 n_kmers, u32 n_hits, shm_index_stats (8 i64);
//   per segment: u32 name length, the name's bytes, i32 length in bases;
//   u32 seg_off[n_seg+1], u64 ref_h[n_kmers], u32 ref_rs[n_kmers],
//   u64 keys[n_keys], u32 key_off[n_keys+1], u32 hits[n_hits];
//   u64 byte count of everything before it (a truncation check), u64
//   checksum of those bytes (IdxSum).
// Reading checks every section on the host before any of it reaches the
// device, so a damaged or hand-made file is refused instead of steering a
// kernel outside its arrays: the checksum, then segment offsets ascending,
// every reference k-mer's hash at most the threshold and its position inside
// its segment and after the previous one, keys strictly ascending and at most
// the threshold, hit-list offsets strictly ascending from 0 to n_hits, and
// every hit a reference k-mer id, ascending within its list.
static const char IDX_MAGIC[8] = {'S', 'H', 'M', 'A', 'P', 'I', 'X', '1'};
static const uint32_t IDX_VERSION = 2;

namespace {

// A 64-bit checksum of a byte stream fed in pieces of any size: 8-byte words
// go round-robin into four multiply-rotate lanes (independent, so the host
// overlaps them), the tail and the length close it.
struct IdxSum {
    uint64_t lane[4] = {0x9e3779b97f4a7c15ULL, 0xbf58476d1ce4e5b9ULL, 0x94d049bb133111ebULL, 0x2545f4914f6cdd1dULL};
    uint64_t part = 0, words = 0, bytes = 0;
    unsigned np = 0;
    static uint64_t rotl(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }
    void word(uint64_t w) {
        uint64_t& h = lane[words & 3];
        h = rotl(h ^ (w * 0xff51afd7ed558ccdULL), 29) * 0xc4ceb9fe1a85ec53ULL;
        words++;
    }
    void add(const void* data, size_t n) {
        const uint8_t* p = (const uint8_t*)data;
        bytes += n;
        while (np && n) {  // finish a word begun by an earlier piece
            part |= (uint64_t)*p++ << (8 * np);
            n--;
            if (++np == 8) {
                word(part);
                part = 0;
                np = 0;
            }
        }
        for (; n >= 8; p += 8, n -= 8) {
            uint64_t w;
            std::memcpy(&w, p, 8);
            word(w);
        }
        for (; n; n--) part |= (uint64_t)*p++ << (8 * np++);
    }
    uint64_t value() const {
        IdxSum t = *this;
        t.word(t.part ^ ((uint64_t)t.np << 56));
        t.word(t.bytes);
        uint64_t h = t.lane[0];
        for (int i = 1; i < 4; i++) h = rotl(h, 17) ^ (t.lane[i] * 0x9e3779b97f4a7c15ULL);
        return h ^ (h >> 31);
    }
};

struct FileW {
    std::FILE* f;
    uint64_t n = 0;
    IdxSum sum;
    void put(const void* p, size_t bytes) {
        if (bytes && std::fwrite(p, 1, bytes, f) != bytes) throw IndexFileError{"write failed"};
        sum.add(p, bytes);
        n += bytes;
    }
    template <class T>
    void val(const T& v) {
        put(&v, sizeof v);
    }
    template <class T>
    void dev(const T* d, size_t count) {  // a device array, in slices through host memory
        std::vector<T> h(std::min<size_t>(count, (size_t)1 << 24));
        for (size_t i = 0; i < count; i += h.size()) {
            const size_t c = std::min(h.size(), count - i);
            SHM_CUDA(cudaMemcpy(h.data(), d + i, sizeof(T) * c, cudaMemcpyDeviceToHost));
            put(h.data(), sizeof(T) * c);
        }
    }
};

struct FileR {
    std::FILE* f;
    uint64_t n = 0;
    IdxSum sum;
    void get(void* p, size_t bytes) {
        if (bytes && std::fread(p, 1, bytes, f) != bytes) throw IndexFileError{"truncated or unreadable index file"};
        sum.add(p, bytes);
        n += bytes;
    }
    template <class T>
    T val() {
        T v;
        get(&v, sizeof v);
        return v;
    }
};

[[noreturn]] void corrupt(const char* what) { throw IndexFileError{std::string("corrupt index file (") + what + ")"}; }

// Where the checked sections go: device buffers on load, nowhere on a check.
struct IdxUpload {
    IndexStorage* ix;  // null: check only
    template <class T>
    void slice(DevBuf<T>* d, size_t at, const T* h, size_t c) {
        if (ix && c) SHM_CUDA(cudaMemcpy(d->p + at, h, sizeof(T) * c, cudaMemcpyHostToDevice));
    }
    template <class T>
    void reserve(DevBuf<T>* d, size_t n) {
        if (ix) d->reserve(n);
    }
};

// Reads the file at path, checking every section (see the layout above), into
// ix when up.ix is set. Throws IndexFileError on any failure.
void read_index_file(const char* path, IndexStorage& hx, IdxUpload up) {
    std::FILE* f = std::fopen(path, "rb");
    if (!f) throw IndexFileError{std::string("cannot open index file: ") + path};
    FileR r{f};
    try {
        // the checksum first: a damaged file is refused before any array is examined
        {
            if (std::fseek(f, 0, SEEK_END) != 0) throw IndexFileError{"unreadable index file"};
            const long size = std::ftell(f);
            if (size < 16 + 8) throw IndexFileError{"truncated or unreadable index file"};
            std::rewind(f);
            IdxSum s;
            std::vector<uint8_t> buf((size_t)1 << 22);
            uint64_t left = (uint64_t)size - 16;
            while (left) {
                const size_t c = (size_t)std::min<uint64_t>(left, buf.size());
                if (std::fread(buf.data(), 1, c, f) != c) throw IndexFileError{"truncated or unreadable index file"};
                if (left == (uint64_t)size - 16 && c >= 12) {  // the magic and version decide the message
                    if (std::memcmp(buf.data(), IDX_MAGIC, 8) != 0) throw IndexFileError{"not a shmap-b200 index file"};
                    uint32_t v;
                    std::memcpy(&v, buf.data() + 8, 4);
                    if (v != IDX_VERSION) throw IndexFileError{"unsupported index file version"};
                }
                s.add(buf.data(), c);
                left -= c;
            }
            uint64_t tail[2];
            if (std::fread(tail, 1, 16, f) != 16) throw IndexFileError{"truncated or unreadable index file"};
            if (tail[0] != (uint64_t)size - 16) throw IndexFileError{"corrupt or truncated index file"};
            if (tail[1] != s.value()) throw IndexFileError{"corrupt index file (checksum)"};
            std::rewind(f);
        }
        char magic[8];
        r.get(magic, 8);
        if (std::memcmp(magic, IDX_MAGIC, 8) != 0) throw IndexFileError{"not a shmap-b200 index file"};
        if (r.val<uint32_t>() != IDX_VERSION) throw IndexFileError{"unsupported index file version"};
        hx.k = r.val<int32_t>();
        hx.h_frac = r.val<double>();
        hx.max_matches = r.val<int32_t>();
        const int32_t n_seg = r.val<int32_t>();
        const uint32_t n_keys = r.val<uint32_t>(), n_kmers = r.val<uint32_t>(), n_hits = r.val<uint32_t>();
        if (hx.k <= 0 || !(hx.h_frac > 0.0) || hx.h_frac > 1.0 || n_seg < 0 || n_keys > n_kmers ||
            n_hits > n_kmers || n_keys > n_hits || hx.max_matches < -1)
            throw IndexFileError{"corrupt index file header"};
        const uint64_t thr = h_thres(hx.h_frac);
        hx.stats = r.val<shm_index_stats>();
        for (int32_t i = 0; i < n_seg; i++) {
            const uint32_t len = r.val<uint32_t>();
            if (len > (1u << 20)) corrupt("segment name");
            std::string nm(len, '\0');
            r.get(&nm[0], len);
            hx.names.push_back(std::move(nm));
            const int32_t sl = r.val<int32_t>();
            if (sl < 0) corrupt("segment length");
            hx.seg_len.push_back(sl);
        }
        hx.h_seg_off.resize((size_t)n_seg + 1);
        r.get(hx.h_seg_off.data(), sizeof(uint32_t) * ((size_t)n_seg + 1));
        if (hx.h_seg_off[0] != 0 || hx.h_seg_off[(size_t)n_seg] != n_kmers) corrupt("segment offsets");
        for (int32_t i = 0; i < n_seg; i++) {
            const uint32_t c = hx.h_seg_off[(size_t)i + 1] - hx.h_seg_off[(size_t)i];
            if (hx.h_seg_off[(size_t)i + 1] < hx.h_seg_off[(size_t)i] ||
                (int64_t)c > std::max<int64_t>(0, (int64_t)hx.seg_len[(size_t)i] - hx.k + 1))
                corrupt("segment offsets");
        }
        IndexStorage* ix = up.ix;
        if (ix) {
            ix->seg_off.reserve((size_t)n_seg + 1);
            SHM_CUDA(cudaMemcpy(ix->seg_off.p, hx.h_seg_off.data(), sizeof(uint32_t) * ((size_t)n_seg + 1),
                                cudaMemcpyHostToDevice));
            ix->seg_sz.reserve((size_t)n_seg + 1);
            if (n_seg)
                SHM_CUDA(cudaMemcpy(ix->seg_sz.p, hx.seg_len.data(), sizeof(int32_t) * (size_t)n_seg,
                                    cudaMemcpyHostToDevice));
        }
        const size_t SL = (size_t)1 << 24;  // elements a slice
        // reference k-mers: hashes at most the threshold
        {
            std::vector<uint64_t> h(std::min<size_t>(std::max<size_t>(n_kmers, 1), SL));
            up.reserve(ix ? &ix->ref_h : nullptr, (size_t)n_kmers + 1);
            for (size_t i = 0; i < n_kmers; i += h.size()) {
                const size_t c = std::min(h.size(), (size_t)n_kmers - i);
                r.get(h.data(), 8 * c);
                for (size_t j = 0; j < c; j++)
                    if (h[j] > thr) corrupt("reference k-mer hash above the threshold");
                up.slice(ix ? &ix->ref_h : nullptr, i, h.data(), c);
            }
        }
        // r << 1 | strand: inside the segment, after the previous k-mer of the segment
        {
            std::vector<uint32_t> v(std::min<size_t>(std::max<size_t>(n_kmers, 1), SL));
            up.reserve(ix ? &ix->ref_rs : nullptr, (size_t)n_kmers + 1);
            int32_t g = 0;
            int64_t prev = -1;
            for (size_t i = 0; i < n_kmers; i += v.size()) {
                const size_t c = std::min(v.size(), (size_t)n_kmers - i);
                r.get(v.data(), 4 * c);
                for (size_t j = 0; j < c; j++) {
                    const uint64_t gi = i + j;
                    while (g < n_seg && gi >= hx.h_seg_off[(size_t)g + 1]) {
                        g++;
                        prev = -1;
                    }
                    const int64_t pos = (int64_t)(v[j] >> 1);
                    if (g >= n_seg || pos < hx.k - 1 || pos >= hx.seg_len[(size_t)g] || pos <= prev)
                        corrupt("reference k-mer position");
                    prev = pos;
                }
                up.slice(ix ? &ix->ref_rs : nullptr, i, v.data(), c);
            }
        }
        // keys: strictly ascending, at most the threshold
        {
            std::vector<uint64_t> h(std::min<size_t>(std::max<size_t>(n_keys, 1), SL));
            up.reserve(ix ? &ix->keys : nullptr, (size_t)n_keys + 1);
            bool first = true;
            uint64_t prev = 0;
            for (size_t i = 0; i < n_keys; i += h.size()) {
                const size_t c = std::min(h.size(), (size_t)n_keys - i);
                r.get(h.data(), 8 * c);
                for (size_t j = 0; j < c; j++) {
                    if (h[j] > thr || (!first && h[j] <= prev)) corrupt("keys");
                    prev = h[j];
                    first = false;
                }
                up.slice(ix ? &ix->keys : nullptr, i, h.data(), c);
            }
        }
        // hit-list offsets: 0, strictly ascending, n_hits (kept on the host for the hits' check)
        std::vector<uint32_t> ko((size_t)n_keys + 1);
        r.get(ko.data(), 4 * ko.size());
        if (ko[0] != 0 || ko[(size_t)n_keys] != n_hits) corrupt("hit-list offsets");
        for (size_t i = 0; i < n_keys; i++) {
            if (ko[i + 1] <= ko[i]) corrupt("hit-list offsets");
            hx.max_list = std::max(hx.max_list, ko[i + 1] - ko[i]);
        }
        up.reserve(ix ? &ix->key_off : nullptr, (size_t)n_keys + 1);
        up.slice(ix ? &ix->key_off : nullptr, 0, ko.data(), ko.size());
        // hits: reference k-mer ids, ascending within each list
        {
            std::vector<uint32_t> v(std::min<size_t>(std::max<size_t>(n_hits, 1), SL));
            up.reserve(ix ? &ix->hits : nullptr, (size_t)n_hits + 1);
            size_t key = 0;
            uint32_t prev = 0;
            for (size_t i = 0; i < n_hits; i += v.size()) {
                const size_t c = std::min(v.size(), (size_t)n_hits - i);
                r.get(v.data(), 4 * c);
                for (size_t j = 0; j < c; j++) {
                    const size_t gi = i + j;
                    while (gi >= ko[key + 1]) key++;
                    if (v[j] >= n_kmers || (gi > ko[key] && v[j] <= prev)) corrupt("hits");
                    prev = v[j];
                }
                up.slice(ix ? &ix->hits : nullptr, i, v.data(), c);
            }
        }
        const uint64_t expect = r.n;
        if (r.val<uint64_t>() != expect) throw IndexFileError{"corrupt or truncated index file"};
        std::fclose(f);
        f = nullptr;
        hx.dev.n_keys = n_keys;
        hx.dev.n_kmers = n_kmers;
        hx.dev.n_hits = n_hits;
    } catch (...) {
        if (f) std::fclose(f);
        throw;
    }
}

}  // namespace

void save_index(const IndexStorage* ix, const char* path) {
    std::FILE* f = std::fopen(path, "wb");
    if (!f) throw IndexFileError{std::string("cannot open for writing: ") + path};
    FileW w{f};
    try {
        const DevIndex& d = ix->dev;
        const int32_t n_seg = (int32_t)ix->seg_len.size();
        w.put(IDX_MAGIC, 8);
        w.val(IDX_VERSION);
        w.val((int32_t)ix->k);
        w.val(ix->h_frac);
        w.val((int32_t)ix->max_matches);
        w.val(n_seg);
        w.val(d.n_keys);
        w.val(d.n_kmers);
        w.val(d.n_hits);
        w.val(ix->stats);
        for (int32_t i = 0; i < n_seg; i++) {
            const std::string& nm = ix->names[(size_t)i];
            w.val((uint32_t)nm.size());
            w.put(nm.data(), nm.size());
            w.val(ix->seg_len[(size_t)i]);
        }
        w.put(ix->h_seg_off.data(), sizeof(uint32_t) * ((size_t)n_seg + 1));
        w.dev(ix->ref_h.p, d.n_kmers);
        w.dev(ix->ref_rs.p, d.n_kmers);
        w.dev(ix->keys.p, d.n_keys);
        w.dev(ix->key_off.p, (size_t)d.n_keys + 1);
        w.dev(ix->hits.p, d.n_hits);
        const uint64_t total = w.n, sum = w.sum.value();  // both cover the bytes before them
        w.val(total);
        w.val(sum);
    } catch (...) {
        std::fclose(f);
        throw;
    }
    if (std::fclose(f) != 0) throw IndexFileError{"write failed"};
}

void check_index_file(const char* path) {
    IndexStorage hx;
    read_index_file(path, hx, IdxUpload{nullptr});
}

IndexStorage* load_index(const char* path, cudaStream_t s) {
    auto* ix = new IndexStorage();
    try {
        SHM_CUDA(cudaGetDevice(&ix->device));
        read_index_file(path, *ix, IdxUpload{ix});
        finish_index(ix, h_thres(ix->h_frac), ix->dev.n_keys, ix->dev.n_kmers, ix->dev.n_hits, ix->max_list, s);
        return ix;
    } catch (...) {
        delete ix;
        throw;
    }
}

}  // namespace shm
