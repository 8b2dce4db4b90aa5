// The per-read mapping path (SHMapper::map_read, src/shmap/mod.rs:653-971)
// as a sequence of batch-wide kernels over thousands of reads:
//
//  K1 sketch        reads -> k-mers                       (src/sketch.rs:167-209)
//  K2 seedprep      group by hash, count() probes, rarest-first order, S and
//                   the seeding prefix; p_ht               (seeding.rs:26-77, mod.rs:682-748)
//  K3 contrib       every hit of every processed seed -> bucket contributions
//                   into a per-read hash table             (seeding.rs:98-212, buckets.rs:642-674)
//  K4 bscan         distinct buckets; which ones can still clear a threshold
//  K5 extend        seed-heuristic extension, one warp per bucket (pruning.rs:10-119)
//  K6 cidx          candidates grouped per read
//  K7 refine        sliding-window Containment/Jaccard, one warp per candidate
//                   (scoring.rs:189-291)
//  K8 sweep         the two ordered sweeps of match_rest and the record
//                   (scoring.rs:367-489, mod.rs:816-943)
//
// Exactness of the reformulation (why the parallel stages reproduce the
// sequential sweep bit for bit):
//  * sh = 1 - (seeds - matches)/m never increases as seeds are added (each
//    seed adds occs to seeds and at most occs to matches), so
//    seed_heuristic_pass(thr) keeps a bucket iff its sh after ALL seeds
//    (sh_final) is >= thr, and then reports sh_final. The in-place pruning
//    state only changes how far the CPU had to look, not the outcome.
//  * pass 1 admits only scores > thr >= theta, so pass 2's threshold
//    best*(1-d) is >= fl(theta*fl(1-d)) = theta_low. Extending every bucket
//    until sh < theta_low therefore decides every survival test of both
//    passes, and refining the buckets with sh_final >= theta_low covers every
//    bucket either pass scores. The sweeps then run on those results in the
//    reference's order (matches desc, (segm_id, b) asc).
//  * a seed's contribution to bucket (g, b) is the aggregate over its hits
//    with pos in [b*h, (b+2)*h) of segment g: exactly what match_seeds'
//    two-slot stream flushes (matches clamped to occs). Hit lists are sorted,
//    so that aggregate is a range found by binary search, and every touched
//    bucket is emitted once, by the first hit of its first run.
//  * best_fixed_length's multiset intersection over window [l, r(l)) is
//    sum_s min(c_s, occs_s): position j counts for window l iff l <= j < r(l)
//    and the occs-th previous occurrence of its seed lies before l. Each j
//    therefore adds 1 on an interval of l, and the per-l intersection is a
//    prefix sum; the first l with the maximal score wins, as the strict `>`
//    of the sequential loop does.
// All scores use explicit round-to-nearest f64 intrinsics.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <mutex>
#include <string>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <tuple>
#include <vector>

#include "shm_common.cuh"
#include "shm_map.cuh"
#include "shm_pack.cuh"
#include "shm_tune.hpp"
#include "shm_paf.hpp"
#include "../host/pack.hpp"
#include "shm_prims.cuh"
#include "shm_sketch.cuh"

namespace shm {

// Candidates refined through the global tables are taken from a queue in
// cost order, the dearest first (a warp's cost grows with the window region,
// twice the bucket half-length): half-lengths above FAR_EDGE0, above
// FAR_EDGE1, the rest.
constexpr int FAR_BINS = 3;
constexpr int32_t FAR_EDGE0 = 1024, FAR_EDGE1 = 512;
__host__ __device__ __forceinline__ int far_bin_of(int32_t half) {
    return half > FAR_EDGE0 ? 0 : (half > FAR_EDGE1 ? 1 : 2);
}

struct BatchMax {
    unsigned int m_max, nu_max, half_max, n_overflow;
    unsigned long long kmers, distinct, proc_seeds, hits, buckets, ext_seeds, refine_kmers;
    unsigned int refine_next[2];  // next candidate chunk k_refine_chip takes, per refinement pass
    unsigned int n_far;        // candidates refined by k_refine (listed in cfar)
    unsigned int lcs_next;     // next candidate k_refine takes under bucket_LCS
    unsigned int far_bin[FAR_BINS];  // candidates of cfar by cost bin (their read's bucket half-length)
    unsigned int far_cur[FAR_BINS];  // placing them, binned, into cfar_q
    unsigned int far_next[2];        // next candidate of cfar_q a refinement warp takes, per pass
    unsigned long long refined;      // candidates refined (the reads' leads and those that can still score)
    unsigned long long bt2_next;     // spare bucket-table slots handed out (second tables)
    unsigned int bt2_n;              // reads given a second table (listed in bt2_list)
};

// Small device-to-host reads of a batch, landing in pinned memory.
struct HostReads {
    uint64_t totals[2];  // hit words, bucket-table slots
    BatchMax hm;         // after seed preparation
    uint32_t nj, nc;     // bucket jobs, candidates
    uint32_t nbk;        // distinct buckets of every read (synchronous sizing)
    BatchMax fin;        // after the sweep
};

// A seed of a read, in rarest-first order: its hit-list start and length in
// the index, occurrences << 1 | strand of its smallest r, and the offset of
// its occurrences among all of the read's (one 16-byte load for every reader).
struct __align__(16) SeedRec {
    uint32_t a, cnt, os, ooff;
};

struct BatchView {
    int32_t n;
    DevParams P;
    DevIndex I;
    double theta2;
    const uint8_t* seq;
    const int64_t* roff;
    const uint64_t* kcap_off;
    uint32_t* kcnt;
    uint64_t* km_h;
    uint32_t* km_rs;
    SeedRec* sd;        // per read, its seeds in rarest-first order
    uint64_t* sd_h;     // per read, the hash of each seed (reads refined on chip only)
    uint32_t* sd_hpre;  // hit words before each processed seed
    const uint64_t* pht_off;
    uint64_t* pht_key;
    uint32_t* pht_val;
    int32_t *r_status, *r_m, *r_nu, *r_nproc, *r_S, *r_S0, *r_half, *r_maxseed;
    int64_t* r_smatch;
    uint32_t* r_seeded;
    uint64_t *hw, *hw_off, *bt_size, *bt_off;
    BSlot* bt;
    ulonglong2* bt_tab; // per read: its bucket table's first slot and slot mask (k_bt_init, k_bt_second)
    uint32_t* bt_list;  // per read, the slots of its distinct buckets (r_seeded[q] of them)
    uint64_t bt_pool;   // slots of the first tables; bt2_spare more follow for second tables
    uint64_t bt2_spare;
    uint32_t* bt2_list; // the reads given a second table
    uint64_t* bt2_off;  // their first runs of hit work items for k_contrib2 (exclusive prefix, nl + 1)
    uint64_t bt_cap;    // most slots a read's bucket table gets (a power of two >= 16)
    uint64_t* r_eb;     // per read: the bound on its distinct buckets (0 until its seeds are prepared)
    uint64_t ext_total; // reference k-mers (bases under -F): a read's buckets are at most ext_total / half + 2 n_seg + 2
    uint32_t* r_flags;  // per read: nonzero when its bucket table passed its load limit
    BucketJob* jobs;
    uint32_t* n_jobs;
    uint32_t job_cap;
    uint32_t *ccnt, *coff, *ccur, *cidx;
    uint32_t* cfar;    // the jobs of the candidates not refined on chip (mx->n_far of them)
    uint32_t* cfar_q;  // the same jobs by cost bin, dearest bin first: the refinement queue
    uint32_t* r_lead;  // per read: its lead candidate's job (refined first), UINT32_MAX for none
    int32_t lead_on;   // candidates refined in two passes (the leads, then those that can still score)
    uint32_t* ovf_list;
    BatchMax* mx;
    shm_map_record* out;
    uint32_t* lcs_pos;  // bucket_LCS: each seed's read positions, decreasing (at kb + its ooff)
    double* r_mw;       // rarity: per read, the weighted total of its k-mers (m_weight)
};

// ------------------------------------------------------------------ helpers
__device__ __forceinline__ uint64_t pow2_ceil(uint64_t x) {
    if (x <= 1) return 1;
    return 1ULL << (64 - __clzll((long long)(x - 1)));
}

template <class T>
__device__ T block_scan_excl(T v, T* sh_warp, T* total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    T inc = warp_inclusive_scan(v);
    if (lane == 31) sh_warp[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        T w = lane < nw ? sh_warp[lane] : T(0);
        T wi = warp_inclusive_scan(w);
        if (lane < nw) sh_warp[lane] = wi - w;
        if (lane == nw - 1) *total = wi;
    }
    __syncthreads();
    T r = sh_warp[wid] + inc - v;
    __syncthreads();
    return r;
}

// Block-wide sum; sh_tot must be shared memory (every thread reads it back).
template <class T>
__device__ T block_reduce_sum(T v, T* sh_warp, T* sh_tot) {
    block_scan_excl<T>(v, sh_warp, sh_tot);
    T tot = *sh_tot;
    __syncthreads();
    return tot;
}

__device__ uint32_t block_reduce_max(uint32_t v, uint32_t* sh_warp) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (lane == 0) sh_warp[wid] = v;
    __syncthreads();
    uint32_t r = 0;
    for (int i = 0; i < nw; i++) r = max(r, sh_warp[i]);
    __syncthreads();
    return r;
}

// Bitonic sort of (A,B) pairs ascending by (A, B), P a power of two.
__device__ void bitonic_ab(uint64_t* A, uint32_t* B, uint32_t P) {
    for (uint32_t k = 2; k <= P; k <<= 1)
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t t = threadIdx.x; t < P / 2; t += blockDim.x) {
                uint32_t i = ((t & ~(j - 1)) << 1) | (t & (j - 1)), l = i + j;  // j is a power of two
                bool asc = (i & k) == 0;
                uint64_t ai = A[i], al = A[l];
                uint32_t bi = B[i], bl = B[l];
                bool gt = ai > al || (ai == al && bi > bl);
                if (gt == asc) {
                    A[i] = al;
                    A[l] = ai;
                    B[i] = bl;
                    B[l] = bi;
                }
            }
            __syncthreads();
        }
}

__device__ void bitonic_u64(uint64_t* A, uint32_t P) {
    for (uint32_t k = 2; k <= P; k <<= 1)
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t t = threadIdx.x; t < P / 2; t += blockDim.x) {
                uint32_t i = ((t & ~(j - 1)) << 1) | (t & (j - 1)), l = i + j;  // j is a power of two
                bool asc = (i & k) == 0;
                uint64_t ai = A[i], al = A[l];
                if ((ai > al) == asc) {
                    A[i] = al;
                    A[l] = ai;
                }
            }
            __syncthreads();
        }
}

// Metrics (src/types.rs:299-322). The bucket metrics report a bucket's own
// content (position range, matches, codirection) rather than a refined
// window: bucket_SH scores it by its seed heuristic, bucket_LCS by the
// longest common subsequence of read and window positions.
constexpr int32_t MET_BUCKET_SH = 2;  // bucket_LCS is 3
__device__ __forceinline__ bool bucket_metric(const DevParams& P) { return P.metric >= MET_BUCKET_SH; }

// Reads refined on chip (k_refine_chip): Containment or Jaccard without
// absolute positions, m and the bucket half-length at most RCHIP_M, so that
// the read's seed table, per-seed state and a window's difference array fit
// a warp's shared slice. Their seed preparation writes the seed hashes
// (sd_h) instead of the global probe table; every other read keeps the
// global table and k_refine.
constexpr int RCHIP_M = 248;
__device__ __forceinline__ bool refine_on_chip(const DevParams& P, uint32_t m, int32_t halflen) {
    return !P.ap && !bucket_metric(P) && !P.rarity && m <= (uint32_t)RCHIP_M && halflen <= RCHIP_M;
}

// The sketch hashes are uniform in [0, thr], so their low bits pick the slot.
__device__ __forceinline__ void pht_insert(const BatchView& v, int32_t q, uint64_t h, uint32_t idx) {
    const uint64_t base = v.pht_off[q];
    const uint64_t mask = v.pht_off[q + 1] - base - 1;
    uint64_t i = h & mask;
    for (;;) {
        if (atomicCAS(v.pht_val + base + i, 0xffffffffu, idx) == 0xffffffffu) {
            v.pht_key[base + i] = h;
            return;
        }
        i = (i + 1) & mask;
    }
}

// Upper bound on the buckets one processed seed contributes to (and so on its
// emissions in k_contrib): a single hit touches 2; a list spanning gidx range
// [first, last] over n segments touches at most (last-first)/h + 3 per
// segment spanned, and never more than 2 per hit. Sizes the bucket tables.
__device__ __forceinline__ uint64_t seed_bucket_bound(const BatchView& v, uint32_t a, uint32_t cnt, int64_t h) {
    if (cnt == 0) return 0;
    if (cnt == 1 || v.P.ap) return 2ULL * cnt;
    const uint32_t g0 = __ldg(v.I.hits + a), g1 = __ldg(v.I.hits + a + cnt - 1);
    const int32_t s0 = seg_of(v.I, g0), s1 = seg_of(v.I, g1);
    const uint64_t span = (uint64_t)(g1 - g0) / (uint64_t)h + 1 + 3ULL * (uint64_t)(s1 - s0 + 1);
    return min((uint64_t)(2ULL * cnt), span);
}

// Slots of a read's bucket table: twice the bound on its distinct buckets
// (a power of two, at least 16), capped at v.bt_cap. A capped table that
// fills past its load limit marks the read, which is then mapped again with
// the full bound.
// The bound on a read's distinct buckets, no more than the genome has for
// its half-length (every bucket b of a segment of e k-mers has b <= (e-1)/h).
__device__ __forceinline__ uint64_t genome_bucket_cap(const BatchView& v, uint64_t ebound, int64_t h) {
    const uint64_t cap = v.ext_total / (uint64_t)max(h, (int64_t)1) + 2ULL * (uint64_t)v.I.n_seg + 2ULL;
    return min(ebound, cap);
}

__device__ __forceinline__ uint64_t bt_slots(const BatchView& v, uint64_t ebound) {
    return min(max((uint64_t)16, pow2_ceil(2 * ebound)), v.bt_cap);
}

// ------------------------------------------------------------------ K2 seedprep
// The per-read fields every seed-preparation form starts from; false when
// the read stops here (overflow or a sketch below MIN_HALFLEN).
__device__ __forceinline__ bool seed_prologue(const BatchView& v, int32_t q, uint32_t P, bool leader, uint32_t& m,
                                              uint64_t& kb, int32_t& S, int32_t& halflen) {
    const int64_t read_len = v.roff[q + 1] - v.roff[q];
    kb = v.kcap_off[q];
    const uint32_t cap = (uint32_t)(v.kcap_off[q + 1] - kb);
    m = v.kcnt[q];
    if (leader) {
        v.hw[q] = 0;
        v.bt_size[q] = 0;
        v.r_nproc[q] = 0;
        v.r_nu[q] = 0;
        v.r_S0[q] = 0;
        v.r_smatch[q] = 0;
        v.r_maxseed[q] = 0;
        v.r_m[q] = (int32_t)m;
        v.r_half[q] = 0;
    }
    if (m > cap || m > P) {
        if (leader) v.r_status[q] = ST_OVERFLOW;
        return false;
    }
    S = __double2int_rz(__dmul_rn(__dsub_rn(1.0, v.theta2), (double)m)) + 1;
    halflen = v.P.ap ? (int32_t)read_len : (int32_t)m;
    if (halflen < MIN_HALFLEN) {
        if (leader) {
            v.r_status[q] = ST_SHORT_SKETCH;
            v.r_S[q] = S;
        }
        return false;
    }
    return true;
}

// One CTA per read. Arrays (P = power of two >= the read's k-mer capacity):
// A/B element keys, GA/GB group hash and occs<<1|strand, GF first index then
// count(), GD hit-list start, E rarest-first sort keys. A and B are dead once
// the groups are formed, so E lives in A's place and GD in B's: 28 bytes an
// element, two CTAs an SM at P = 4096.
struct SeedArrays {
    uint64_t *A, *GA, *E;
    uint32_t *B, *GB, *GF, *GD;
};

__device__ SeedArrays carve(uint8_t* base, uint32_t P) {
    SeedArrays s;
    s.A = (uint64_t*)base;
    s.GA = s.A + P;
    s.E = s.A;
    s.B = (uint32_t*)(s.GA + P);
    s.GB = s.B + P;
    s.GF = s.GB + P;
    s.GD = s.B;
    return s;
}
constexpr size_t SEED_BYTES_PER_ELEM = 2 * 8 + 3 * 4;

__device__ void seedprep_one(const BatchView& v, int32_t q, uint32_t P, const SeedArrays& S_) {
    __shared__ uint64_t sw64[32];
    __shared__ uint32_t sw32[32];
    __shared__ uint64_t t64;
    __shared__ uint32_t t32;
    const int tid = threadIdx.x, nt = blockDim.x;
    uint32_t m;
    uint64_t kb;
    int32_t S, halflen;
    if (!seed_prologue(v, q, P, tid == 0, m, kb, S, halflen)) return;
    const uint32_t Pm = (uint32_t)pow2_ceil(m);
    for (uint32_t i = tid; i < Pm; i += nt) {
        if (i < m) {
            S_.A[i] = v.km_h[kb + i];
            uint32_t rs = v.km_rs[kb + i];
            S_.B[i] = ((0x3fffffffu - (rs >> 1)) << 1) | (rs & 1u);
        } else {
            S_.A[i] = ~0ULL;
            S_.B[i] = 0xffffffffu;
        }
    }
    __syncthreads();
    bitonic_ab(S_.A, S_.B, Pm);  // (h asc, r desc): src/shmap/seeding.rs:28-34

    // groups of equal hashes (src/shmap/seeding.rs:45-67)
    const uint32_t per = (m + nt - 1) / nt;
    const uint32_t i0 = min(m, (uint32_t)tid * per), i1 = min(m, i0 + per);
    uint32_t nf = 0;
    for (uint32_t i = i0; i < i1; i++) nf += (i == 0 || S_.A[i] != S_.A[i - 1]) ? 1u : 0u;
    uint32_t gbase = block_scan_excl<uint32_t>(nf, sw32, &t32);
    const uint32_t n_u = t32;
    {
        uint32_t c = gbase;
        for (uint32_t i = i0; i < i1; i++)
            if (i == 0 || S_.A[i] != S_.A[i - 1]) {
                S_.GF[c] = i;
                S_.GA[c] = S_.A[i];
                c++;
            }
    }
    __syncthreads();
    {
        uint32_t c = gbase;
        for (uint32_t i = i0; i < i1; i++) {
            if (i == 0 || S_.A[i] != S_.A[i - 1]) c++;
            if (i + 1 == m || S_.A[i + 1] != S_.A[i]) {
                uint32_t g = c - 1;
                uint32_t occs = i - S_.GF[g] + 1;
                S_.GB[g] = (occs << 1) | (S_.B[i] & 1u);  // representative: smallest r (seeding.rs:56)
            }
        }
    }
    __syncthreads();
    if (v.P.os) S = (int32_t)n_u;  // mod.rs:732-736
    // count() probes (index.rs:204-213) and the hit-list start of each group
    for (uint32_t g = tid; g < n_u; g += nt) {
        uint32_t a, cnt;
        idx_lookup(v.I, S_.GA[g], a, cnt);
        S_.GD[g] = a;
        S_.GF[g] = cnt;
    }
    __syncthreads();
    // rarest first, stable over hash order (seeding.rs:71): key (hits_in_t, group)
    const uint32_t Pu = (uint32_t)pow2_ceil(n_u);
    for (uint32_t g = tid; g < Pu; g += nt) S_.E[g] = g < n_u ? (((uint64_t)S_.GF[g] << 32) | g) : ~0ULL;
    __syncthreads();
    bitonic_u64(S_.E, Pu);

    // seeding prefix: seed i is processed iff sum(occs before i) < S (seeding.rs:101)
    const uint32_t per2 = (n_u + nt - 1) / nt;
    const uint32_t j0 = min(n_u, (uint32_t)tid * per2), j1 = min(n_u, j0 + per2);
    uint32_t so = 0;
    uint64_t sc = 0;
    for (uint32_t i = j0; i < j1; i++) {
        uint32_t g = (uint32_t)(S_.E[i] & 0xffffffffu);
        so += S_.GB[g] >> 1;
        sc += S_.E[i] >> 32;
    }
    uint32_t po = block_scan_excl<uint32_t>(so, sw32, &t32);
    uint64_t pc = block_scan_excl<uint64_t>(sc, sw64, &t64);
    const bool pht = v.P.metric != MET_BUCKET_SH;  // bucket_SH looks nothing up (these reads are never on chip)
    if (pht) {  // the read's probe table starts empty
        const uint64_t pb = v.pht_off[q], pe = v.pht_off[q + 1];
        for (uint64_t i = pb + tid; i < pe; i += nt) v.pht_val[i] = 0xffffffffu;
        __syncthreads();
    }
    uint32_t l_np = 0, l_s0 = 0, l_max = 0;
    uint64_t l_sm = 0, l_eb = 0;
    for (uint32_t i = j0; i < j1; i++) {
        const uint64_t e = S_.E[i];
        const uint32_t g = (uint32_t)(e & 0xffffffffu), cnt = (uint32_t)(e >> 32);
        const uint32_t os = S_.GB[g], occs = os >> 1;
        v.sd[kb + i] = SeedRec{S_.GD[g], cnt, os, po};
        if ((int64_t)po < (int64_t)S) {
            v.sd_hpre[kb + i] = (uint32_t)pc;
            l_np++;
            l_s0 += occs;
            l_sm += cnt;
            l_max = max(l_max, cnt);
            l_eb += seed_bucket_bound(v, S_.GD[g], cnt, halflen);
        }
        if (pht) pht_insert(v, q, S_.GA[g], i);
        po += occs;
        pc += cnt;
    }
    const uint32_t n_proc = block_reduce_sum<uint32_t>(l_np, sw32, &t32);
    const uint32_t S0 = block_reduce_sum<uint32_t>(l_s0, sw32, &t32);
    const uint64_t smatch = block_reduce_sum<uint64_t>(l_sm, sw64, &t64);
    const uint64_t ebound = block_reduce_sum<uint64_t>(l_eb, sw64, &t64);
    const uint32_t mxs = block_reduce_max(l_max, sw32);
    if (tid == 0) {
        v.r_status[q] = ST_UNMAPPED;
        v.r_nu[q] = (int32_t)n_u;
        v.r_nproc[q] = (int32_t)n_proc;
        v.r_S[q] = S;
        v.r_S0[q] = (int32_t)S0;
        v.r_smatch[q] = (int64_t)smatch;
        v.r_maxseed[q] = (int32_t)mxs;
        v.r_half[q] = halflen;
        if (smatch >= 0xffffffffULL) {
            v.r_status[q] = ST_OVERFLOW;
        } else {
            v.hw[q] = smatch;
            const uint64_t eb = genome_bucket_cap(v, ebound, halflen);
            v.r_eb[q] = eb;
            v.bt_size[q] = smatch ? bt_slots(v, eb) : 0;
        }
        atomicMax(&v.mx->m_max, m);
        atomicMax(&v.mx->nu_max, n_u);
        atomicMax(&v.mx->half_max, (uint32_t)halflen);
        atomicAdd(&v.mx->kmers, (unsigned long long)m);
        atomicAdd(&v.mx->distinct, (unsigned long long)n_u);
        atomicAdd(&v.mx->proc_seeds, (unsigned long long)n_proc);
        atomicAdd(&v.mx->hits, (unsigned long long)smatch);
    }
}

constexpr int SEEDP_THREADS = 512;  // a CTA per read: two CTAs an SM (112 KB of shared memory each at P = 4096)
template <bool GLOBAL>
__global__ void __launch_bounds__(SEEDP_THREADS) k_seedprep(BatchView v, const int32_t* __restrict__ list,
                                                  const uint32_t* __restrict__ n_list_d, uint32_t P, uint8_t* gscr,
                                                  size_t gscr_per_cta) {
    extern __shared__ __align__(16) uint8_t smem[];
    uint8_t* base = GLOBAL ? gscr + (size_t)blockIdx.x * gscr_per_cta : smem;
    SeedArrays S_ = carve(base, P);
    const int32_t n_list = (int32_t)*n_list_d;
    for (int32_t li = blockIdx.x; li < n_list; li += gridDim.x) {
        seedprep_one(v, list[li], P, S_);
        __syncthreads();
    }
}

// Seed-preparation bins by the actual sketch size m of each read (reads past
// their k-mer capacity go to bin 0, whose prologue marks them overflowed):
// m <= 256, 512 and 1024 the counting form (a warp per read), m <= 4096 a
// CTA per read in shared memory, larger a CTA with global scratch.
constexpr int N_SEED_BINS = 5;
__global__ void k_seed_bins(BatchView v, int32_t* __restrict__ lists, uint32_t* __restrict__ bin_cnt) {
    const int lane = threadIdx.x & 31;
    for (int32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < v.n; base += gridDim.x * blockDim.x) {
        const int32_t q = base + lane;
        int b = -1;
        if (q < v.n) {
            const uint32_t m = v.kcnt[q];
            const uint32_t cap = (uint32_t)(v.kcap_off[q + 1] - v.kcap_off[q]);
            b = m > cap ? 0 : m <= 256 ? 0 : m <= 512 ? 1 : m <= 1024 ? 2 : m <= 4096 ? 3 : 4;
        }
        const unsigned same = __match_any_sync(0xffffffffu, b);
        const int leader = __ffs(same) - 1;
        uint32_t at = 0;
        if (lane == leader && b >= 0) at = atomicAdd(bin_cnt + b, (uint32_t)__popc(same));
        at = __shfl_sync(0xffffffffu, at, leader);
        if (b >= 0) lists[(size_t)b * v.n + at + __popc(same & ((1u << lane) - 1u))] = q;
    }
}

// count() probes for U hashes of one lane at once (index.rs:204-213): the
// bucket-table sectors of the U probes are loaded together (one round; the
// hit-list start and count of a found key come from the same sector), and
// the few probes that land in a crowded range finish through the directory.
template <int U>
__device__ __forceinline__ void idx_lookup_u(const DevIndex& I, const uint64_t (&h)[U], const bool (&on)[U],
                                             uint32_t (&a)[U], uint32_t (&cnt)[U]) {
    if (!I.btab) {
#pragma unroll
        for (int u = 0; u < U; u++) {
            a[u] = cnt[u] = 0;
            if (on[u]) idx_lookup(I, h[u], a[u], cnt[u]);
        }
        return;
    }
    uint4 k[U];
    bool live[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
        a[u] = 0;
        cnt[u] = 0;
        live[u] = on[u] && h[u] <= I.thr && I.n_keys != 0;
        k[u] = live[u] ? __ldg(btab_bucket(I, h[u])) : make_uint4(~0u, ~0u, ~0u, ~0u);
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
        const int sl = live[u] ? btab_slot(k[u], h[u]) : -1;
        if (sl < 0) continue;
        const uint4 ac = __ldg(btab_bucket(I, h[u]) + 1);  // the same sector
        if (sl == 0) {
            a[u] = ac.x;
            cnt[u] = ac.y;
        } else if (sl == 1) {
            a[u] = ac.z;
            cnt[u] = ac.w & 0x7fffffffu;
        } else if (ac.w >> 31) {
            idx_lookup_dir(I, h[u], a[u], cnt[u]);
        }
    }
}

// pht_insert for U seeds of one lane; the compare-and-swaps of the U probes
// are issued together.
template <int U>
__device__ __forceinline__ void pht_insert_u(const BatchView& v, int32_t q, const uint64_t (&h)[U],
                                             const uint32_t (&idx)[U], const bool (&on)[U]) {
    const uint64_t base = v.pht_off[q];
    const uint64_t mask = v.pht_off[q + 1] - base - 1;
    uint64_t i[U];
    bool pend[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
        i[u] = h[u] & mask;
        pend[u] = on[u];
    }
    for (;;) {  // the table has at least twice as many slots as seeds: every insert ends
        bool more = false;
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (!pend[u]) continue;
            if (atomicCAS(v.pht_val + base + i[u], 0xffffffffu, idx[u]) == 0xffffffffu) {
                v.pht_key[base + i[u]] = h[u];
                pend[u] = false;
            } else {
                i[u] = (i[u] + 1) & mask;
                more = true;
            }
        }
        if (!more) break;
    }
}

// seed_bucket_bound summed over U seeds of one lane (those with on[u]); the
// hit-list ends of the U seeds are loaded together, and their segments found
// in `segs`, a copy of seg_off.
template <int U>
__device__ __forceinline__ uint64_t seed_bucket_bound_u(const BatchView& v, const uint32_t (&a)[U],
                                                        const uint32_t (&cnt)[U], const bool (&on)[U], int64_t h,
                                                        const uint32_t* segs) {
    uint32_t g0[U], g1[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
        g0[u] = g1[u] = 0;
        if (on[u] && cnt[u] > 1 && !v.P.ap) {
            g0[u] = __ldg(v.I.hits + a[u]);
            g1[u] = __ldg(v.I.hits + a[u] + cnt[u] - 1);
        }
    }
    uint64_t sum = 0;
#pragma unroll
    for (int u = 0; u < U; u++) {
        if (!on[u] || cnt[u] == 0) continue;
        if (cnt[u] == 1 || v.P.ap) {
            sum += 2ULL * cnt[u];
            continue;
        }
        const int32_t s0 = seg_of_in(segs, v.I.n_seg, g0[u]), s1 = seg_of_in(segs, v.I.n_seg, g1[u]);
        const uint64_t span = (uint64_t)(g1[u] - g0[u]) / (uint64_t)h + 1 + 3ULL * (uint64_t)(s1 - s0 + 1);
        sum += min((uint64_t)(2ULL * cnt[u]), span);
    }
    return sum;
}

// ------------------------------------------------------------------ K2 counting form
// Seed preparation with one warp per read and work linear in m: the k-mers
// are bucketed by a counting sort on h -> h * Ht / (thr + 1) (order
// preserving, about one k-mer per bucket for Ht >= m), each bucket is put in
// hash order by insertion, equal hashes are grouped in place, and the groups
// are put rarest first by a stable least-significant-digit radix sort on
// their hit counts, which keeps hash order among equal counts: the order of
// src/shmap/seeding.rs:28-71. Shared memory per warp, for capacity C:
//   Sh (8C), Srs (4C): the bucketed k-mers, then the groups in place (hash,
//                      then occs << 1 | strand of the smallest r)
//   Rc (4C): bucket offsets, then each group's count() hit count
//   Ra (4C): each group's hit-list start
//   P0, P1 (2C each): radix permutations (16-bit group indices)
//   RH (128 words): digit offsets of the 7-bit radix digits
// followed, once per CTA, by seg_off when the reference has at most
// SEEDC_SEGS segments (seedc_seg_bytes).
constexpr int SEEDC_DIGIT = 7;
__host__ __device__ constexpr size_t seedc_bytes(uint32_t C) { return 24 * (size_t)C + 4 * (1u << SEEDC_DIGIT); }
constexpr int SEEDC_U = 4;       // groups a lane probes at once
constexpr int SEEDC_SEGS = 1024;  // references with at most this many segments keep seg_off in shared memory
static_assert(1024 <= 65536, "group indices of the largest bin fit 16 bits");
inline size_t seedc_seg_bytes(int32_t n_seg) {
    return n_seg <= SEEDC_SEGS ? (4 * (size_t)(n_seg + 1) + 15) / 16 * 16 : 0;
}

// Exclusive scan, in place, of the n (a multiple of 32) words X[0..n): lane l
// owns n/32 consecutive words.
__device__ __forceinline__ void warp_scan_words(uint32_t* X, uint32_t n, int lane) {
    const uint32_t per = n >> 5, b0 = (uint32_t)lane * per;
    uint32_t sum = 0;
    for (uint32_t j = 0; j < per; j++) sum += X[b0 + j];
    uint32_t run = warp_inclusive_scan(sum) - sum;
    for (uint32_t j = 0; j < per; j++) {
        const uint32_t c = X[b0 + j];
        X[b0 + j] = run;
        run += c;
    }
}

__device__ void seedprep_count(const BatchView& v, int32_t q, uint32_t C, uint8_t* base, const uint32_t* segs) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u, le = lt | (1u << lane);
    uint32_t m;
    uint64_t kb;
    int32_t S, halflen;
    if (!seed_prologue(v, q, C, lane == 0, m, kb, S, halflen)) return;
    uint64_t* Sh = (uint64_t*)base;
    uint32_t* Srs = (uint32_t*)(Sh + C);
    uint32_t* Rc = Srs + C;
    uint32_t* Ra = Rc + C;
    uint16_t* P0 = (uint16_t*)(Ra + C);
    uint16_t* P1 = P0 + C;
    uint32_t* RH = (uint32_t*)(P1 + C);

    // counting sort by bucket: Ht = power of two in [32, C], >= m
    const uint32_t Ht = max((uint32_t)32, (uint32_t)pow2_ceil(m));
    const uint64_t mul = v.P.slot_mul[31 - __clz(Ht)];
    for (uint32_t i = lane; i < Ht; i += 32) Rc[i] = 0;
    __syncwarp();
#pragma unroll 4
    for (uint32_t i = lane; i < m; i += 32) atomicAdd(&Rc[(uint32_t)__umul64hi(v.km_h[kb + i], mul)], 1u);
    __syncwarp();
    warp_scan_words(Rc, Ht, lane);
    __syncwarp();
#pragma unroll 4
    for (uint32_t i = lane; i < m; i += 32) {
        const uint64_t h = v.km_h[kb + i];
        const uint32_t pos = atomicAdd(&Rc[(uint32_t)__umul64hi(h, mul)], 1u);
        Sh[pos] = h;
        Srs[pos] = v.km_rs[kb + i];
    }
    __syncwarp();
    // bucket b now spans [Rc[b-1], Rc[b]); insertion by hash (equal hashes stay put)
    {
        const uint32_t per = Ht >> 5, b0 = (uint32_t)lane * per;
        uint32_t s0 = b0 ? Rc[b0 - 1] : 0u;
        for (uint32_t j = 0; j < per; j++) {
            const uint32_t e1 = Rc[b0 + j];
            for (uint32_t x = s0 + 1; x < e1; x++) {
                const uint64_t hx = Sh[x];
                const uint32_t rx = Srs[x];
                uint32_t y = x;
                while (y > s0 && Sh[y - 1] > hx) {
                    Sh[y] = Sh[y - 1];
                    Srs[y] = Srs[y - 1];
                    y--;
                }
                Sh[y] = hx;
                Srs[y] = rx;
            }
            s0 = e1;
        }
    }
    __syncwarp();

    // groups of equal hashes, compacted in place (src/shmap/seeding.rs:45-67);
    // Srs[g] keeps the group's smallest r << 1 | strand until its last element
    // writes occs << 1 | that strand (the representative: seeding.rs:56)
    uint32_t n_u = 0, open_start = 0;
    uint64_t carry_h = 0;
    for (uint32_t c0 = 0; c0 < m; c0 += 32) {
        const uint32_t e = c0 + lane;
        const bool valid = e < m;
        const uint64_t h = valid ? Sh[e] : 0;
        const uint32_t rs = valid ? Srs[e] : 0;
        const uint64_t hn = (e + 1 < m) ? Sh[e + 1] : 0;
        uint64_t hp = __shfl_up_sync(0xffffffffu, h, 1);
        if (lane == 0) hp = carry_h;
        const bool first = valid && (e == 0 || h != hp);
        const bool last = valid && (e + 1 == m || hn != h);
        const unsigned fmask = __ballot_sync(0xffffffffu, first);
        const unsigned fle = fmask & le;
        const uint32_t gid = n_u + __popc(fle) - 1;
        const uint32_t start = fle ? (c0 + 31 - __clz(fle)) : open_start;
        __syncwarp();  // this chunk is read before anything is written at gid <= e
        if (first) {
            Sh[gid] = h;
            Srs[gid] = rs;
        }
        __syncwarp();
        if (valid && !first) atomicMin(&Srs[gid], rs);
        __syncwarp();
        if (last) Srs[gid] = ((e - start + 1) << 1) | (Srs[gid] & 1u);
        n_u += __popc(fmask);
        open_start = __shfl_sync(0xffffffffu, start, 31);
        carry_h = __shfl_sync(0xffffffffu, h, 31);
        __syncwarp();
    }
    if (v.P.os) S = (int32_t)n_u;  // mod.rs:732-736

    // count() probes (index.rs:204-213), SEEDC_U groups a lane at once
    uint32_t maxc = 0;
    for (uint32_t g0 = 0; g0 < n_u; g0 += 32 * SEEDC_U) {
        uint64_t hh[SEEDC_U];
        bool on[SEEDC_U];
        uint32_t a[SEEDC_U], cnt[SEEDC_U];
#pragma unroll
        for (int u = 0; u < SEEDC_U; u++) {
            const uint32_t g = g0 + 32 * u + lane;
            on[u] = g < n_u;
            hh[u] = on[u] ? Sh[g] : 0;
        }
        idx_lookup_u<SEEDC_U>(v.I, hh, on, a, cnt);
#pragma unroll
        for (int u = 0; u < SEEDC_U; u++) {
            const uint32_t g = g0 + 32 * u + lane;
            if (on[u]) {
                Rc[g] = cnt[u];
                Ra[g] = a[u];
                maxc = max(maxc, cnt[u]);
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) maxc = max(maxc, __shfl_xor_sync(0xffffffffu, maxc, o));
    __syncwarp();

    // rarest first, stable over hash order (seeding.rs:71): LSD radix on the
    // count, SEEDC_DIGIT bits a pass, as many passes as the largest count needs
    constexpr uint32_t ND = 1u << SEEDC_DIGIT;
    const uint16_t* ord = nullptr;  // null: identity
    uint16_t* pout = P0;
    for (int sh = 0; sh < 32 && (maxc >> sh) != 0; sh += SEEDC_DIGIT) {
        for (uint32_t i = lane; i < ND; i += 32) RH[i] = 0;
        __syncwarp();
        for (uint32_t i = lane; i < n_u; i += 32) {
            const uint32_t g = ord ? ord[i] : i;
            atomicAdd(&RH[(Rc[g] >> sh) & (ND - 1)], 1u);
        }
        __syncwarp();
        warp_scan_words(RH, ND, lane);
        __syncwarp();
        for (uint32_t c0 = 0; c0 < n_u; c0 += 32) {
            const uint32_t i = c0 + lane;
            const bool valid = i < n_u;
            const uint32_t g = valid ? (ord ? ord[i] : i) : 0u;
            const uint32_t d = valid ? (Rc[g] >> sh) & (ND - 1) : ND + (uint32_t)lane;
            const unsigned peers = __match_any_sync(0xffffffffu, d);
            const int leader = __ffs(peers) - 1;
            uint32_t at = (valid && lane == leader) ? RH[d] : 0u;
            at = __shfl_sync(0xffffffffu, at, leader);
            if (valid) pout[at + __popc(peers & lt)] = (uint16_t)g;
            __syncwarp();
            if (valid && lane == leader) RH[d] = at + __popc(peers);
            __syncwarp();
        }
        ord = pout;
        pout = pout == P0 ? P1 : P0;
    }

    // seeding prefix: seed i is processed iff sum(occs before i) < S
    // (seeding.rs:101); the processed seeds are a prefix of the order
    const bool chip = refine_on_chip(v.P, m, halflen);
    const bool pht = !chip && v.P.metric != MET_BUCKET_SH;  // bucket_SH looks nothing up
    if (pht) {  // the read's probe table starts empty (written before the inserts below)
        const uint64_t pb = v.pht_off[q], pe = v.pht_off[q + 1];
        for (uint64_t i = pb + lane; i < pe; i += 32) v.pht_val[i] = 0xffffffffu;
        __syncwarp();
    }
    uint32_t po_carry = 0, l_np = 0, l_s0 = 0, l_max = 0;
    uint64_t pc_carry = 0, l_sm = 0, l_eb = 0;
    for (uint32_t c0 = 0; c0 < n_u; c0 += 32) {
        const uint32_t i = c0 + lane;
        const bool valid = i < n_u;
        const uint32_t g = valid ? (ord ? ord[i] : i) : 0u;
        const uint32_t cnt = valid ? Rc[g] : 0u;
        const uint32_t os = valid ? Srs[g] : 0u, occs = os >> 1;
        const uint32_t oi = warp_inclusive_scan(occs);
        const uint64_t ci = warp_inclusive_scan((uint64_t)cnt);
        const uint32_t po = po_carry + oi - occs;
        const uint64_t pc = pc_carry + ci - cnt;
        if (valid) {
            v.sd[kb + i] = SeedRec{Ra[g], cnt, os, po};
            if (chip) v.sd_h[kb + i] = Sh[g];
            if ((int64_t)po < (int64_t)S) {
                v.sd_hpre[kb + i] = (uint32_t)pc;
                l_np++;
                l_s0 += occs;
                l_sm += cnt;
                l_max = max(l_max, cnt);
            }
        }
        po_carry += __shfl_sync(0xffffffffu, oi, 31);
        pc_carry += __shfl_sync(0xffffffffu, ci, 31);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        l_np += __shfl_xor_sync(0xffffffffu, l_np, o);
        l_s0 += __shfl_xor_sync(0xffffffffu, l_s0, o);
        l_sm += __shfl_xor_sync(0xffffffffu, l_sm, o);
        l_max = max(l_max, __shfl_xor_sync(0xffffffffu, l_max, o));
    }
    // bucket bounds of the processed seeds and the probe table, SEEDC_U seeds a
    // lane at once (both are independent of the order they are done in)
    for (uint32_t c0 = 0; c0 < n_u; c0 += 32 * SEEDC_U) {
        uint64_t hh[SEEDC_U];
        uint32_t a[SEEDC_U], cnt[SEEDC_U], ii[SEEDC_U];
        bool on[SEEDC_U], proc[SEEDC_U];
#pragma unroll
        for (int u = 0; u < SEEDC_U; u++) {
            ii[u] = c0 + 32 * u + lane;
            on[u] = ii[u] < n_u;
            proc[u] = ii[u] < l_np;
            const uint32_t g = on[u] ? (ord ? ord[ii[u]] : ii[u]) : 0u;
            hh[u] = on[u] ? Sh[g] : 0;
            a[u] = on[u] ? Ra[g] : 0u;
            cnt[u] = on[u] ? Rc[g] : 0u;
        }
        l_eb += seed_bucket_bound_u<SEEDC_U>(v, a, cnt, proc, halflen, segs);
        if (pht) pht_insert_u<SEEDC_U>(v, q, hh, ii, on);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l_eb += __shfl_xor_sync(0xffffffffu, l_eb, o);
    if (lane == 0) {
        v.r_status[q] = ST_UNMAPPED;
        v.r_nu[q] = (int32_t)n_u;
        v.r_nproc[q] = (int32_t)l_np;
        v.r_S[q] = S;
        v.r_S0[q] = (int32_t)l_s0;
        v.r_smatch[q] = (int64_t)l_sm;
        v.r_maxseed[q] = (int32_t)l_max;
        v.r_half[q] = halflen;
        if (l_sm >= 0xffffffffULL) {
            v.r_status[q] = ST_OVERFLOW;
        } else {
            v.hw[q] = l_sm;
            const uint64_t eb = genome_bucket_cap(v, l_eb, halflen);
            v.r_eb[q] = eb;
            v.bt_size[q] = l_sm ? bt_slots(v, eb) : 0;
        }
        atomicMax(&v.mx->m_max, m);
        atomicMax(&v.mx->nu_max, n_u);
        atomicMax(&v.mx->half_max, (uint32_t)halflen);
        atomicAdd(&v.mx->kmers, (unsigned long long)m);
        atomicAdd(&v.mx->distinct, (unsigned long long)n_u);
        atomicAdd(&v.mx->proc_seeds, (unsigned long long)l_np);
        atomicAdd(&v.mx->hits, (unsigned long long)l_sm);
    }
}

template <uint32_t C, int W>
__global__ void __launch_bounds__(W * 32, 4) k_seedprep_c(BatchView v, const int32_t* __restrict__ list,
                                                       const uint32_t* __restrict__ n_list) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int wib = threadIdx.x >> 5;
    uint8_t* base = smem + (size_t)wib * seedc_bytes(C);
    uint32_t* s_seg = (uint32_t*)(smem + (size_t)W * seedc_bytes(C));  // seg_off (seedc_seg_bytes)
    const int32_t n = (int32_t)*n_list;
    const bool staged = v.I.n_seg <= SEEDC_SEGS;
    if (staged)
        for (int i = threadIdx.x; i <= v.I.n_seg; i += blockDim.x) s_seg[i] = __ldg(v.I.seg_off + i);
    __syncthreads();
    const uint32_t* segs = staged ? s_seg : v.I.seg_off;
    for (int32_t li = blockIdx.x * W + wib; li < n; li += gridDim.x * W) {
        seedprep_count(v, list[li], C, base, segs);
        __syncwarp();
    }
}

// ------------------------------------------------------------------ K3 contributions
__device__ __forceinline__ int64_t hit_pos(const DevIndex& I, uint32_t g, int32_t seg, bool ap) {
    return ap ? (int64_t)(__ldg(I.ref_rs + g) >> 1) : (int64_t)(g - __ldg(I.seg_off + seg));
}

// First index in [lo, end) whose hit is >= v, or end, when every hit before lo
// is below v: probes lo, lo+1, lo+3, lo+7, ... then a binary search in the
// last gap, so a range of c hits costs about 2 log2(c) + 1 loads (one when
// the next hit is already past v).
__device__ __forceinline__ uint32_t hits_gallop(const uint32_t* __restrict__ hits, uint32_t lo, uint32_t end,
                                                uint32_t v) {
    uint32_t step = 1;
    while (lo < end) {
        const uint32_t pr = min(lo + step, end) - 1;
        if (__ldg(hits + pr) >= v) {
            end = pr;
            break;
        }
        lo = pr + 1;
        step <<= 1;
    }
    return hits_lower_bound(hits, lo, end - lo, v);
}

// Hits of one seed's list [a, a+cnt) in segment g with pos in [lo, hi): returns [A, B).
__device__ __forceinline__ void seed_range(const DevIndex& I, uint32_t a, uint32_t cnt, int32_t g, int64_t lo,
                                           int64_t hi, bool ap, uint32_t& A, uint32_t& B) {
    const uint32_t s_lo = __ldg(I.seg_off + g), s_hi = __ldg(I.seg_off + g + 1);
    if (!ap) {
        uint64_t glo = (uint64_t)s_lo + (uint64_t)max(lo, (int64_t)0);
        uint64_t ghi = min((uint64_t)s_lo + (uint64_t)max(hi, (int64_t)0), (uint64_t)s_hi);
        glo = min(glo, (uint64_t)s_hi);
        A = hits_lower_bound(I.hits, a, cnt, (uint32_t)glo);
        // the range spans two half-lengths, which few hits of a list fall in:
        // its end is galloped to from A rather than searched for from a
        B = ghi > glo ? hits_gallop(I.hits, A, a + cnt, (uint32_t)ghi) : A;
        return;
    }
    uint32_t sA = hits_lower_bound(I.hits, a, cnt, s_lo), sB = hits_lower_bound(I.hits, a, cnt, s_hi);
    auto lb_r = [&](int64_t rv) {
        uint32_t l = sA, len = sB - sA;
        while (len > 0) {
            uint32_t half = len >> 1;
            if ((int64_t)(__ldg(I.ref_rs + __ldg(I.hits + l + half)) >> 1) < rv) {
                l += half + 1;
                len -= half + 1;
            } else {
                len = half;
            }
        }
        return l;
    };
    A = lb_r(lo);
    B = lb_r(hi);
    if (B < A) B = A;
}

struct Agg {
    int32_t count, codir, rmin, rmax;
};

// The hits [A, B) of a seed: their count and, when `full`, their
// codirection and position range (only the bucket metrics report those:
// Containment and Jaccard leave them unread).
__device__ __forceinline__ Agg range_agg(const DevIndex& I, uint32_t A, uint32_t B, uint32_t seed_strand,
                                         bool full = true) {
    Agg r;
    r.count = (int32_t)(B - A);
    if (r.count <= 0 || !full) {
        r.count = max(r.count, 0);
        r.codir = 0;
        r.rmin = INT32_MAX;
        r.rmax = -1;
        return r;
    }
    int32_t fw = (int32_t)(__ldg(I.hit_fw + B) - __ldg(I.hit_fw + A));
    int32_t same = seed_strand ? r.count - fw : fw;
    r.codir = 2 * same - r.count;
    r.rmin = (int32_t)(__ldg(I.ref_rs + __ldg(I.hits + A)) >> 1);
    r.rmax = (int32_t)(__ldg(I.ref_rs + __ldg(I.hits + B - 1)) >> 1);
    return r;
}

// A bucket's matches and codirection sum in one 64-bit word: the sum of
// packed values is matches_sum << 32 plus codir_sum (two's complement), and
// both sums stay below 2^31 in magnitude, so the low half is codir_sum and
// the rest is matches_sum.
__device__ __forceinline__ unsigned long long bt_pack(int32_t matches, int32_t codir) {
    return ((unsigned long long)(uint32_t)matches << 32) + (unsigned long long)(long long)codir;
}
__device__ __forceinline__ void bt_unpack(unsigned long long mc, int32_t& matches, int32_t& codir) {
    codir = (int32_t)(uint32_t)mc;
    matches = (int32_t)((mc - (unsigned long long)(long long)codir) >> 32);
}

__device__ __forceinline__ void bt_add(const BatchView& v, int32_t q, int32_t seg, int64_t bb, int32_t matches,
                                       int32_t codir, int32_t rmin, int32_t rmax) {
    if (v.r_flags[q]) return;  // the read is mapped again, or given a second table first
    const ulonglong2 tb = v.bt_tab[q];
    const uint64_t base = tb.x, mask = tb.y;
    const unsigned long long key = ((unsigned long long)(uint32_t)seg << 32) | (uint32_t)bb;
    uint64_t i = mix64(key) & mask;
    BSlot* s;
    for (uint64_t probe = 0;; probe++) {
        if (probe > mask) {  // every slot taken by other buckets
            atomicOr(v.r_flags + q, 1u);
            return;
        }
        s = v.bt + base + i;
        unsigned long long prev = atomicCAS(&s->key, EMPTY_KEY, key);
        if (prev == EMPTY_KEY) {  // a new bucket: list it for k_bscan (seeded_buckets, mod.rs:794)
            const uint32_t at = atomicAdd(v.r_seeded + q, 1u);  // < slots: every listed bucket holds a slot
            v.bt_list[base + at] = (uint32_t)i;
            if ((uint64_t)at + 1 > ((mask + 1) >> 1) + ((mask + 1) >> 2)) atomicOr(v.r_flags + q, 1u);  // load > 3/4
            break;
        }
        if (prev == key) break;
        i = (i + 1) & mask;
    }
    atomicAdd(&s->mc, bt_pack(matches, codir));
    if (bucket_metric(v.P)) {  // the position range is read by the bucket metrics only
        atomicMin(&s->rmin, rmin);
        atomicMax(&s->rmax, rmax);
    }
}

__device__ __forceinline__ uint32_t ub_u64(const uint64_t* a, uint32_t n, uint64_t x) {  // first index with a[i] > x
    uint32_t lo = 0, len = n;
    while (len > 0) {
        uint32_t half = len >> 1;
        if (a[lo + half] <= x) {
            lo += half + 1;
            len -= half + 1;
        } else {
            len = half;
        }
    }
    return lo;
}
__device__ __forceinline__ uint32_t ub_u32(const uint32_t* a, uint32_t n, uint32_t x) {
    uint32_t lo = 0, len = n;
    while (len > 0) {
        uint32_t half = len >> 1;
        if (a[lo + half] <= x) {
            lo += half + 1;
            len -= half + 1;
        } else {
            len = half;
        }
    }
    return lo;
}

// Each thread takes CONTRIB_RUN consecutive hit words: the first word's read
// and seed come from two binary searches, the rest by stepping through the
// seed's hit list (sorted by gidx) and on to the next seed or read. The
// previous hit's bucket and the current segment's bounds are carried along.
constexpr int CONTRIB_RUN = 8;

__device__ __forceinline__ int32_t seg_step(const DevIndex& I, uint32_t g, int32_t seg, uint32_t& s_lo,
                                            uint32_t& s_hi) {
    if (seg >= 0 && g >= s_lo && g < s_hi) return seg;
    seg = seg_of(I, g);
    s_lo = __ldg(I.seg_off + seg);
    s_hi = __ldg(I.seg_off + seg + 1);
    return seg;
}

// The hit work items [w, wend) (of one read or of consecutive reads, the
// first of them read q), added to their reads' bucket tables.
__device__ __forceinline__ void contrib_span(const BatchView& v, uint64_t w, const uint64_t wend, int32_t q) {
    const bool ap = v.P.ap != 0;
    const bool sh_out = bucket_metric(v.P);  // codirection and positions are reported (bucket metrics)
    const DevIndex& I = v.I;
    uint64_t kb = v.kcap_off[q];
    uint32_t np = (uint32_t)v.r_nproc[q];
    uint32_t h = (uint32_t)v.r_half[q];
    uint32_t j = ub_u32(v.sd_hpre + kb, np, (uint32_t)(w - v.hw_off[q])) - 1;
    uint32_t t = (uint32_t)(w - v.hw_off[q]) - v.sd_hpre[kb + j];
    SeedRec sr = v.sd[kb + j];
    uint32_t a = sr.a, cnt = sr.cnt, os = sr.os;
    int32_t seg = -1;
    uint32_t s_lo = 0, s_hi = 0;
    int32_t seg_p = -1;  // bucket of the seed's previous hit (seg_p < 0: none)
    uint32_t b_p = 0;
    if (t > 0) {
        const uint32_t g_p = __ldg(I.hits + a + t - 1);
        seg_p = seg = seg_step(I, g_p, seg, s_lo, s_hi);
        b_p = (ap ? (__ldg(I.ref_rs + g_p) >> 1) : g_p - s_lo) / h;
    }
    for (;;) {
        const uint32_t occs = os >> 1, sstr = os & 1u;
        const uint32_t g_t = __ldg(I.hits + a + t);
        seg = seg_step(I, g_t, seg, s_lo, s_hi);
        const uint32_t b_t = (ap ? (__ldg(I.ref_rs + g_t) >> 1) : g_t - s_lo) / h;
        const bool first = !(seg_p == seg && b_p == b_t);
        const bool prev_is_bm1 = seg_p == seg && b_p + 1 == b_t;
        if (first) {
            if (cnt == 1) {
                const uint32_t rs = sh_out ? __ldg(I.ref_rs + g_t) : 0u;
                const int32_t cd = ((rs & 1u) == sstr) ? 1 : -1, r = (int32_t)(rs >> 1);
                bt_add(v, q, seg, b_t, 1, cd, r, r);  // add_to_pos (buckets.rs:642-662)
                if (b_t > 0) bt_add(v, q, seg, (int64_t)b_t - 1, 1, cd, r, r);
            } else if (!ap) {
                // streamed multi-hit seed: one clamped contribution per bucket
                // (seeding.rs:113-205). Both of this hit's ranges, buckets b_t
                // and b_t - 1 (the latter unless the previous hit is in it),
                // start at this hit: the previous hit lies in a lower bucket
                // (below b_t - 1 when b_t - 1 is added) or an earlier segment.
                // Their ends are found by galloping forward.
                const uint32_t A = a + t, E = a + cnt;
                const uint64_t up1 = (uint64_t)s_lo + (uint64_t)(b_t + 1) * h, up0 = up1 + h;
                const uint32_t B1 = hits_gallop(I.hits, A + 1, E, (uint32_t)min(up1, (uint64_t)s_hi));
                const uint32_t B0 = hits_gallop(I.hits, B1, E, (uint32_t)min(up0, (uint64_t)s_hi));
                if (!sh_out) {  // matches only
                    bt_add(v, q, seg, b_t, min((int32_t)(B0 - A), (int32_t)occs), 0, 0, 0);
                    if (b_t > 0 && !prev_is_bm1)
                        bt_add(v, q, seg, (int64_t)b_t - 1, min((int32_t)(B1 - A), (int32_t)occs), 0, 0, 0);
                } else {
                    const int32_t r0 = (int32_t)(__ldg(I.ref_rs + g_t) >> 1);
                    const uint32_t fwA = __ldg(I.hit_fw + A);
                    {
                        const int32_t c = (int32_t)(B0 - A), fw = (int32_t)(__ldg(I.hit_fw + B0) - fwA);
                        const int32_t same = sstr ? c - fw : fw;
                        const int32_t r1 = (int32_t)(__ldg(I.ref_rs + __ldg(I.hits + B0 - 1)) >> 1);
                        bt_add(v, q, seg, b_t, min(c, (int32_t)occs), 2 * same - c, r0, r1);
                    }
                    if (b_t > 0 && !prev_is_bm1) {
                        const int32_t c = (int32_t)(B1 - A), fw = (int32_t)(__ldg(I.hit_fw + B1) - fwA);
                        const int32_t same = sstr ? c - fw : fw;
                        const int32_t r1 = (int32_t)(__ldg(I.ref_rs + __ldg(I.hits + B1 - 1)) >> 1);
                        bt_add(v, q, seg, (int64_t)b_t - 1, min(c, (int32_t)occs), 2 * same - c, r0, r1);
                    }
                }
            } else {
                // streamed multi-hit seed, absolute positions: the ranges by search
                for (int e = 0; e < 2; e++) {
                    const int64_t bb = (int64_t)b_t - e;
                    if (bb < 0) break;
                    if (e == 1 && prev_is_bm1) break;
                    uint32_t A, B;
                    seed_range(I, a, cnt, seg, bb * (int64_t)h, (bb + 2) * (int64_t)h, ap, A, B);
                    Agg g = range_agg(I, A, B, sstr, sh_out);
                    bt_add(v, q, seg, bb, min(g.count, (int32_t)occs), g.codir, g.rmin, g.rmax);
                }
            }
        }
        if (++w >= wend) break;
        seg_p = seg;
        b_p = b_t;
        if (++t == cnt) {  // next seed of the read, or the next read with hits
            t = 0;
            seg_p = -1;
            if (++j == np) {
                do {
                    q++;
                } while (v.hw_off[q + 1] <= w);
                kb = v.kcap_off[q];
                np = (uint32_t)v.r_nproc[q];
                h = (uint32_t)v.r_half[q];
                j = ub_u32(v.sd_hpre + kb, np, 0u) - 1;  // past the seeds without hits
            }
            sr = v.sd[kb + j];
            a = sr.a;
            cnt = sr.cnt;
            os = sr.os;
        }
    }
}

__global__ void __launch_bounds__(256) k_contrib(BatchView v) {
    const uint64_t total = v.hw_off[v.n];
    const uint64_t nrun = (total + CONTRIB_RUN - 1) / CONTRIB_RUN;
    const int lane = threadIdx.x & 31;
    // a warp takes 32 consecutive runs: the read of its first by a 32-way
    // search, each lane's own by walking on from there (runs of one warp
    // rarely cross more than a read or two)
    for (uint64_t r0 = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); r0 < nrun;
         r0 += (uint64_t)gridDim.x * blockDim.x) {
        int32_t q = warp_last_le(v.hw_off, v.n + 1, r0 * CONTRIB_RUN, lane);
        const uint64_t rn = r0 + (uint64_t)lane;
        if (rn >= nrun) continue;
        const uint64_t w = rn * CONTRIB_RUN;
        while (v.hw_off[q + 1] <= w) q++;
        contrib_span(v, w, min(w + CONTRIB_RUN, total), q);
    }
}

// The runs of CONTRIB_RUN hit work items of the reads given a second bucket
// table (k_bt_second), as an exclusive prefix over the list (one CTA; the
// list is short unless many reads filled their tables).
__global__ void __launch_bounds__(1024) k_bt2_scan(BatchView v) {
    __shared__ unsigned long long wsum[32];
    __shared__ unsigned long long carry;
    const uint32_t nl = v.mx->bt2_n;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t c0 = 0; c0 < nl; c0 += 1024) {
        const uint32_t i = c0 + threadIdx.x;
        unsigned long long x = 0;
        if (i < nl) {
            const int32_t q = (int32_t)v.bt2_list[i];
            x = (v.hw_off[q + 1] - v.hw_off[q] + CONTRIB_RUN - 1) / CONTRIB_RUN;
        }
        unsigned long long inc = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane == 31) wsum[wid] = inc;
        __syncthreads();
        if (wid == 0) {
            unsigned long long t = wsum[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            wsum[lane] = t;  // inclusive over warps
        }
        __syncthreads();
        const unsigned long long before = carry + (wid ? wsum[wid - 1] : 0ULL) + inc - x;
        if (i < nl) v.bt2_off[i] = before;
        __syncthreads();
        if (threadIdx.x == 0) carry += wsum[31];
        __syncthreads();
    }
    if (threadIdx.x == 0) v.bt2_off[nl] = carry;
}

// Those runs over the whole grid: each finds its read in the list by the
// prefix and contributes into the read's second table.
__global__ void __launch_bounds__(256) k_contrib2(BatchView v) {
    const uint32_t nl = v.mx->bt2_n;
    if (nl == 0) return;
    const uint64_t nrun = v.bt2_off[nl];
    for (uint64_t rn = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; rn < nrun;
         rn += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = nl;  // the last list entry whose first run is <= rn
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (v.bt2_off[mid] <= rn) lo = mid;
            else hi = mid;
        }
        const int32_t q = (int32_t)v.bt2_list[lo];
        const uint64_t w = v.hw_off[q] + (rn - v.bt2_off[lo]) * CONTRIB_RUN;
        contrib_span(v, w, min(w + CONTRIB_RUN, v.hw_off[q + 1]), q);
    }
}

// Empties the first *total slots (the total is read on the device).
// Clears the batch's bucket tables, the first `pool` slots at most: a read
// whose table would end past the pool is flagged (mapped again) before any
// kernel touches it.
__global__ void k_bt_init(BSlot* bt, const uint64_t* __restrict__ bt_off, int32_t n_reads, uint64_t pool,
                          uint32_t* __restrict__ r_flags, ulonglong2* __restrict__ bt_tab) {
    const uint64_t n = min(bt_off[n_reads], pool);
    for (int32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n_reads; q += gridDim.x * blockDim.x) {
        const uint64_t b = bt_off[q], e = bt_off[q + 1];
        bt_tab[q] = make_ulonglong2(b, e - b - 1);
        if (e > pool) r_flags[q] = 1u;
    }
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        BSlot s;
        s.key = EMPTY_KEY;
        s.mc = 0;
        s.rmin = INT32_MAX;
        s.rmax = -1;
        bt[i] = s;
    }
}

// Second tables (a batch mapped without waiting for its sizes): a read whose
// bucket table filled up, or lay past the pool, gets a table of twice the
// bound on its distinct buckets (a power of two, at most BT2_MAX slots) from
// the spare slots after the pool, emptied here, and is listed for k_contrib2
// to contribute again; a read that finds no room stays flagged and is mapped
// again by the host. A warp takes 32 reads, each flagged one in turn.
constexpr uint64_t BT2_MAX = 4096;  // (a read needing more climbs the host's ladder)
__global__ void __launch_bounds__(256) k_bt_second(BatchView v) {
    const int lane = threadIdx.x & 31;
    const int32_t nwarps = (int32_t)((gridDim.x * blockDim.x) >> 5);
    for (int32_t q0 = (int32_t)((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; q0 < v.n; q0 += nwarps * 32) {
        const int32_t q = q0 + lane;
        const bool fl = q < v.n && v.r_flags[q] != 0 && v.r_status[q] != ST_OVERFLOW;
        for (unsigned bal = __ballot_sync(0xffffffffu, fl); bal; bal &= bal - 1) {
            const int src = __ffs(bal) - 1;
            const int32_t r = q0 + src;
            const uint64_t slots = min(max((uint64_t)16, pow2_ceil(2 * max(v.r_eb[r], (uint64_t)1))), BT2_MAX);
            unsigned long long off = 0;
            if (lane == 0) off = atomicAdd(&v.mx->bt2_next, (unsigned long long)slots);
            off = __shfl_sync(0xffffffffu, off, 0);
            if (off + slots > v.bt2_spare) continue;  // no room: the host maps it again
            const uint64_t base = v.bt_pool + off;
            for (uint64_t i = lane; i < slots; i += 32) {
                BSlot e;
                e.key = EMPTY_KEY;
                e.mc = 0;
                e.rmin = INT32_MAX;
                e.rmax = -1;
                v.bt[base + i] = e;
            }
            if (lane == 0) {
                v.bt_tab[r] = make_ulonglong2(base, slots - 1);
                v.r_seeded[r] = 0;
                v.r_flags[r] = 0;
                v.bt2_list[atomicAdd(&v.mx->bt2_n, 1u)] = (uint32_t)r;
            }
        }
    }
}

// ------------------------------------------------------------------ K4 distinct buckets
__global__ void __launch_bounds__(256) k_bscan(BatchView v) {
    const int lane = threadIdx.x & 31;
    const int32_t wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int32_t q = wid; q < v.n; q += nwarps) {
        const uint32_t nb = v.r_seeded[q];
        if (v.r_flags[q]) {  // its capped bucket table filled up, or lay past the pool: mapped again
            if (lane == 0) v.r_status[q] = ST_OVERFLOW;
            continue;
        }
        if (nb == 0) continue;
        const uint64_t base = v.bt_tab[q].x;
        if (lane == 0) atomicAdd(&v.mx->buckets, (unsigned long long)nb);
        for (uint32_t j = lane; j < nb; j += 32) {
            const BSlot s = v.bt[base + v.bt_list[base + j]];
            BucketJob jb;
            jb.read = q;
            jb.seg = (int32_t)(s.key >> 32);
            jb.bb = (int32_t)(s.key & 0xffffffffu);
            int32_t s_matches, s_codir;
            bt_unpack(s.mc, s_matches, s_codir);
            jb.m0 = s_matches;
            jb.matches = s_matches;
            jb.codir = s_codir;
            jb.rmin = s.rmin;
            jb.rmax = s.rmax;
            jb.pad0 = jb.pad1 = 0;
            jb.score = -1.0;
            jb.support = 0.0;
            jb.t_l = jb.t_r = jb.inter = jb.same = jb.s_sz = -1;
            if (v.P.nbp) {
                jb.sh = 1.0;  // seed_heuristic_pass does nothing under NBP (pruning.rs:351)
                jb.is_cand = 1;
            } else {
                const double sh0 = hseed(v.r_m[q], v.r_S0[q], s_matches);
                if (sh0 < v.P.theta_low) continue;
                jb.sh = sh0;
                jb.is_cand = 0;
            }
            uint32_t ji = atomicAdd(v.n_jobs, 1u);
            if (ji < v.job_cap) {
                v.jobs[ji] = jb;
                if (jb.is_cand) atomicAdd(v.ccnt + q, 1u);
            }
        }
    }
}

// ------------------------------------------------------------------ K5 extension
// One warp per bucket; 32 remaining seeds per step, matches_in_bucket for each
// (pruning.rs:18-80), then an inclusive scan of (seeds, matches) finds the
// first prefix whose sh drops below theta_low.
__global__ void __launch_bounds__(256) k_extend(BatchView v) {
    const int lane = threadIdx.x & 31;
    const uint32_t njobs = min(*v.n_jobs, v.job_cap);
    const uint32_t wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    const bool ap = v.P.ap != 0;
    for (uint32_t ji = wid; ji < njobs; ji += nwarps) {
        BucketJob* J = v.jobs + ji;
        const int32_t q = J->read, seg = J->seg, bb = J->bb;
        const int32_t m = v.r_m[q], n_u = v.r_nu[q], np = v.r_nproc[q];
        const int64_t h = v.r_half[q];
        const uint64_t kb = v.kcap_off[q];
        int32_t seeds = v.r_S0[q], matches = J->matches, codir = J->codir, rmin = J->rmin, rmax = J->rmax;
        bool stopped = false;
        int32_t examined = 0;
        for (int32_t i0 = np; i0 < n_u; i0 += 32) {
            examined += min(32, n_u - i0);
            const int32_t i = i0 + lane;
            const bool valid = i < n_u;
            int32_t ds = 0, dm = 0, dc = 0, rmn = INT32_MAX, rmx = -1;
            if (valid) {
                const SeedRec sr = v.sd[kb + i];
                const uint32_t os = sr.os, cnt = sr.cnt;
                ds = (int32_t)(os >> 1);
                if (cnt > 0) {
                    uint32_t A, B;
                    seed_range(v.I, sr.a, cnt, seg, (int64_t)bb * h, ((int64_t)bb + 2) * h, ap, A, B);
                    Agg g = range_agg(v.I, A, B, os & 1u, bucket_metric(v.P));
                    dm = min(g.count, ds);
                    dc = g.codir;
                    rmn = g.rmin;
                    rmx = g.rmax;
                }
            }
            const int32_t ps = warp_inclusive_scan(ds), pm = warp_inclusive_scan(dm);
            const bool low = valid && hseed(m, seeds + ps, matches + pm) < v.P.theta_low;
            if (__any_sync(0xffffffffu, low)) {
                stopped = true;
                break;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                dc += __shfl_xor_sync(0xffffffffu, dc, o);
                rmn = min(rmn, __shfl_xor_sync(0xffffffffu, rmn, o));
                rmx = max(rmx, __shfl_xor_sync(0xffffffffu, rmx, o));
            }
            seeds += __shfl_sync(0xffffffffu, ps, 31);
            matches += __shfl_sync(0xffffffffu, pm, 31);
            codir += dc;
            rmin = min(rmin, rmn);
            rmax = max(rmax, rmx);
        }
        if (lane == 0) atomicAdd(&v.mx->ext_seeds, (unsigned long long)examined);
        if (lane == 0 && !stopped) {
            J->sh = hseed(m, seeds, matches);
            J->matches = matches;
            J->codir = codir;
            J->rmin = rmin;
            J->rmax = rmax;
            J->is_cand = 1;
            atomicAdd(v.ccnt + q, 1u);
        }
    }
}

// ------------------------------------------------------------------ K6 candidates per read
// Also lists the candidates k_refine takes (those not refined on chip), one
// counter update per warp.
__global__ void k_cidx(BatchView v) {
    const uint32_t njobs = min(*v.n_jobs, v.job_cap);
    const int lane = threadIdx.x & 31;
    for (uint32_t b = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); b < njobs; b += gridDim.x * blockDim.x) {
        const uint32_t ji = b + (uint32_t)lane;
        bool far = false;
        if (ji < njobs && v.jobs[ji].is_cand) {
            const int32_t q = v.jobs[ji].read;
            v.cidx[v.coff[q] + atomicAdd(v.ccur + q, 1u)] = ji;
            far = !refine_on_chip(v.P, (uint32_t)v.r_m[q], v.r_half[q]);
        }
        const unsigned fm = __ballot_sync(0xffffffffu, far);
        if (fm) {
            const int leader = __ffs(fm) - 1;
            uint32_t at = 0;
            if (lane == leader) at = atomicAdd(&v.mx->n_far, (uint32_t)__popc(fm));
            at = __shfl_sync(0xffffffffu, at, leader);
            if (far) v.cfar[at + __popc(fm & ((1u << lane) - 1u))] = ji;
            const int bin = far ? far_bin_of(v.r_half[v.jobs[ji].read]) : -1;
#pragma unroll
            for (int b2 = 0; b2 < FAR_BINS; b2++) {
                const unsigned bm = __ballot_sync(0xffffffffu, bin == b2);
                if (bm && lane == __ffs(bm) - 1) atomicAdd(&v.mx->far_bin[b2], (uint32_t)__popc(bm));
            }
        }
    }
}

// The refinement queue: cfar's candidates placed by cost bin, the dearest
// bin first, so the longest refinements start first and the short ones fill
// the end (within a bin, in any order).
__global__ void k_far_bins(BatchView v) {
    const uint32_t nfar = v.mx->n_far;
    const int lane = threadIdx.x & 31;
    uint32_t base[FAR_BINS];
    base[0] = 0;
    for (int b = 1; b < FAR_BINS; b++) base[b] = base[b - 1] + v.mx->far_bin[b - 1];
    for (uint32_t i0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); i0 < nfar; i0 += gridDim.x * blockDim.x) {
        const uint32_t i = i0 + (uint32_t)lane;
        const uint32_t ji = i < nfar ? v.cfar[i] : 0u;
        const int bin = i < nfar ? far_bin_of(v.r_half[v.jobs[ji].read]) : -1;
#pragma unroll
        for (int b = 0; b < FAR_BINS; b++) {
            const unsigned bm = __ballot_sync(0xffffffffu, bin == b);
            if (!bm) continue;
            const int leader = __ffs(bm) - 1;
            uint32_t at = 0;
            if (lane == leader) at = atomicAdd(&v.mx->far_cur[b], (uint32_t)__popc(bm));
            at = __shfl_sync(0xffffffffu, at, leader);
            if (bin == b) v.cfar_q[base[b] + at + __popc(bm & ((1u << lane) - 1u))] = ji;
        }
    }
}

// The next candidate of the refinement queue for this warp (UINT32_MAX when
// the queue is empty).
__device__ __forceinline__ uint32_t next_far(const BatchView& v, int lane, int pass = 0) {
    uint32_t ci = 0;
    if (lane == 0) ci = atomicAdd(&v.mx->far_next[pass], 1u);
    ci = __shfl_sync(0xffffffffu, ci, 0);
    return ci < v.mx->n_far ? v.cfar_q[ci] : UINT32_MAX;
}

// ------------------------------------------------------------------ which candidates are refined
// Under Containment with bucket pruning, the sweep (k_sweep, as
// match_rest) scores a candidate only while its sh is at least the running
// threshold. The first candidate of a read's sweep order whose sh is at
// least theta (its lead) is always scored; after it the threshold of pass 1
// is at least T1 = max(theta, s1) when the lead's score s1 clears theta's
// admission bar (else theta), and pass 2 starts from best * (1 - d), where
// best clears the admission bar of a threshold >= T1. So every candidate
// either pass scores has sh >= L = admit(T1) * (1 - d), rounded as the sweep
// rounds (both roundings are monotone), and a read with no lead scores none.
// The leads are refined first (pass 0), then the other candidates with sh >=
// L (pass 1); the rest are never consulted. Without the two passes
// (lead_on = 0) pass 0 refines every candidate.
__global__ void k_lead(BatchView v) {
    const int lane = threadIdx.x & 31;
    const int32_t nwarps = (int32_t)((gridDim.x * blockDim.x) >> 5);
    const double theta = v.P.theta;
    for (int32_t q = (int32_t)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); q < v.n; q += nwarps) {
        const uint32_t c0 = v.coff[q], nc = v.coff[q + 1] - c0;
        // the first in sweep order (m0 desc, then (seg, bb) asc) with sh >= theta
        int32_t bm = INT32_MIN, bs = INT32_MAX, bb = INT32_MAX;
        uint32_t bj = UINT32_MAX;
        for (uint32_t i = lane; i < nc; i += 32) {
            const uint32_t ji = v.cidx[c0 + i];
            const BucketJob& J = v.jobs[ji];
            if (!(J.sh >= theta)) continue;
            if (J.m0 > bm || (J.m0 == bm && (J.seg < bs || (J.seg == bs && J.bb < bb)))) {
                bm = J.m0;
                bs = J.seg;
                bb = J.bb;
                bj = ji;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const int32_t om = __shfl_xor_sync(0xffffffffu, bm, o), os = __shfl_xor_sync(0xffffffffu, bs, o),
                          ob = __shfl_xor_sync(0xffffffffu, bb, o);
            const uint32_t oj = __shfl_xor_sync(0xffffffffu, bj, o);
            if (om > bm || (om == bm && (os < bs || (os == bs && ob < bb)))) {
                bm = om;
                bs = os;
                bb = ob;
                bj = oj;
            }
        }
        if (lane == 0) v.r_lead[q] = bj;
    }
}

// Whether candidate ji (job J) is refined in refinement pass `pass`.
__device__ __forceinline__ bool refined_in(const BatchView& v, const BucketJob& J, uint32_t ji, int pass) {
    if (!v.lead_on) return pass == 0;
    const uint32_t ld = v.r_lead[J.read];
    if (pass == 0) return ji == ld;
    if (ld == UINT32_MAX || ji == ld) return false;
    const double theta = v.P.theta, tb = v.P.tiebreak, s1 = v.jobs[ld].score;
    auto admit_of = [&](double t) { return tb > 0.0 ? __dsub_rn(t, __dmul_rn(tb, fabs(t))) : t; };
    const double T1 = s1 > admit_of(theta) ? fmax(theta, s1) : theta;
    const double L = __dmul_rn(admit_of(T1), __dsub_rn(1.0, v.P.min_diff));
    // one ulp of slack below L (a candidate more is harmless)
    const long long b = __double_as_longlong(L);
    const double Ls = L > 0.0 ? __longlong_as_double(b - 1) : (L < 0.0 ? __longlong_as_double(b + 1) : -4.9e-324);
    return J.sh >= Ls;
}

// ------------------------------------------------------------------ K7 refinement
struct RefScratch {
    int32_t* base;
    size_t per_warp;  // ints
    uint32_t nu_max, wmax;
    uint32_t ring_n;  // ints of the occurrence rings (m_max + 1)
    size_t wt_at;     // rarity: ints from a warp's base to its f64 weights (even)
};

// pht_lookup for U hashes of one lane, the probes issued together; s[u] =
// the seed index, or -1 when absent (or !on[u]).
template <int U>
__device__ __forceinline__ void pht_lookup_u(const BatchView& v, int32_t q, const uint64_t (&h)[U], const bool (&on)[U],
                                             int32_t (&s)[U]) {
    const uint64_t base = v.pht_off[q];
    const uint64_t mask = v.pht_off[q + 1] - base - 1;
    uint64_t i[U];
    bool pend[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
        i[u] = h[u] & mask;
        pend[u] = on[u];
        s[u] = -1;
    }
    for (;;) {  // the table keeps empty slots (at least twice as many slots as seeds): every probe ends
        uint32_t val[U];
        uint64_t key[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            val[u] = pend[u] ? v.pht_val[base + i[u]] : 0xffffffffu;
            key[u] = pend[u] ? v.pht_key[base + i[u]] : 0;
        }
        bool more = false;
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (!pend[u]) continue;
            if (val[u] == 0xffffffffu) {
                pend[u] = false;
            } else if (key[u] == h[u]) {
                s[u] = (int32_t)val[u];
                pend[u] = false;
            } else {
                i[u] = (i[u] + 1) & mask;
                more = true;
            }
        }
        if (!more) break;
    }
}

constexpr int REFINE_WARPS = 8;
constexpr int REFINE_U = 2;  // position chunks whose seeds are fetched together

// ------------------------------------------------------------------ bucket_LCS
// Each seed's read positions in decreasing order (its pmatches,
// src/shmap/seeding.rs:28-56), stored at the seed's occurrence offset:
// pos[kb + ooff + j] is the j-th largest r among the read's k-mers with the
// seed's hash. One CTA per read; reads that stopped before their seeds were
// laid out, or that are mapped again, are skipped.
__global__ void __launch_bounds__(256) k_lcs_occ(BatchView v, uint32_t* __restrict__ pos, uint32_t* __restrict__ cnt) {
    for (int32_t q = blockIdx.x; q < v.n; q += gridDim.x) {
        const int32_t n_u = v.r_nu[q], m = v.r_m[q];
        if (n_u == 0 || v.r_status[q] == ST_OVERFLOW) continue;  // the same for every thread
        const uint64_t kb = v.kcap_off[q];
        for (int32_t i = threadIdx.x; i < n_u; i += blockDim.x) cnt[kb + i] = 0;
        __syncthreads();
        for (int32_t j = threadIdx.x; j < m; j += blockDim.x) {
            const uint64_t h[1] = {v.km_h[kb + j]};
            const bool on[1] = {true};
            int32_t sx[1];
            pht_lookup_u<1>(v, q, h, on, sx);
            if (sx[0] < 0) continue;  // every sketch hash is a seed's: not taken
            const uint32_t at = v.sd[kb + sx[0]].ooff + atomicAdd(cnt + kb + sx[0], 1u);
            pos[kb + at] = v.km_rs[kb + j] >> 1;
        }
        __syncthreads();
        for (int32_t i = threadIdx.x; i < n_u; i += blockDim.x) {  // each seed's positions, decreasing
            const SeedRec sr = v.sd[kb + i];
            const uint32_t occ = sr.os >> 1;
            uint32_t* a = pos + kb + sr.ooff;
            for (uint32_t x = 1; x < occ; x++) {
                const uint32_t val = a[x];
                uint32_t y = x;
                for (; y > 0 && a[y - 1] < val; y--) a[y] = a[y - 1];
                a[y] = val;
            }
        }
        __syncthreads();
    }
}

// Places of x in sorted Ti[0, li) and of y in sorted Td[0, ld) (the first
// index whose value is >= the key), found together: lanes 0-15 search Ti,
// lanes 16-31 Td. At each level a half's lane 15 compares the range's last
// value and lanes 0-14 the first values of 15 pieces; the ballot settles the
// place (past the last value, or at the first) or leaves the rest of the
// piece after the last first value below the key. A key beyond either end
// of its range, the common case when read and window are collinear, takes
// one level.
__device__ __forceinline__ void half_warp_places(const int32_t* Ti, int32_t li, int32_t x, const int32_t* Td,
                                                 int32_t ld, int32_t y, int lane, int32_t& pi, int32_t& pd) {
    const int hf = lane >> 4, hl = lane & 15;
    const int32_t* T = hf ? Td : Ti;
    const int32_t key = hf ? y : x;
    int32_t lo = 0, hi = hf ? ld : li;  // the place lies in [lo, hi]; T[lo, hi) is still unread
    while (__any_sync(0xffffffffu, lo < hi)) {
        const bool act = lo < hi;
        const int32_t step = (hi - lo + 14) / 15;
        bool below = false;
        if (act) {
            if (hl == 15) {
                below = T[hi - 1] < key;
            } else {
                const int32_t st = lo + hl * step;
                below = st < hi && T[st] < key;
            }
        }
        const unsigned bits = (__ballot_sync(0xffffffffu, below) >> (hf * 16)) & 0xffffu;
        if (act) {
            const int32_t nb = __popc(bits & 0x7fffu);
            if (bits & 0x8000u) {
                lo = hi;
            } else if (nb == 0) {
                hi = lo;
            } else {  // after piece nb-1's first value, before piece nb's first and the last value
                const int32_t first = lo + (nb - 1) * step;
                hi = min(lo + nb * step, hi - 1);
                lo = first + 1;
            }
        }
    }
    pi = __shfl_sync(0xffffffffu, lo, 0);
    pd = __shfl_sync(0xffffffffu, lo, 16);
}

// First index of sorted T[0, len) whose value is >= x, by one lane.
__device__ __forceinline__ int32_t lane_lower_bound(const int32_t* T, int32_t len, int32_t x) {
    int32_t lo = 0;
    while (len > 0) {
        const int32_t half = len >> 1;
        if (T[lo + half] < x) {
            lo += half + 1;
            len -= half + 1;
        } else {
            len = half;
        }
    }
    return lo;
}

__device__ __forceinline__ int32_t warp_inclusive_max(int32_t x) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x = max(x, y);
    }
    return x;
}

// bucket_LCS for one candidate (src/shmap/scoring.rs:114-170, 326-344): the
// read positions of every window k-mer found among the read's seeds, each
// seed's in decreasing order, are fed in window order to two patience-sorting
// tail arrays at once, Ti for the longest strictly increasing subsequence of
// the list and Td (values negated) for that of its reverse, the longest
// strictly decreasing one. Tails hold distinct read positions: at most m
// each. The record takes the bucket's own content, as bucket_SH's does.
//
// A seed with one read position is placed by half_warp_places. The
// positions of a seed with several are placed 32 at a time, each lane
// searching for its own, which gives the sequential result because
//  * in Ti the group's values decrease, so none can extend a tail another
//    one of the group set: each value's place is its place among the tails
//    before the group, places do not increase along the group, and of the
//    values that share a place the last (smallest) stays;
//  * in Td the group's values increase, and value t's place is the first
//    one past value t-1's: p_t = max(q_t, p_(t-1) + 1) with q_t its place
//    among the tails before it, a running maximum of q_j - j.
__device__ __forceinline__ void lcs_one(const BatchView& v, BucketJob* J, int32_t q, int32_t* Ti, int32_t* Td,
                                        int lane) {
    const DevIndex& I = v.I;
    const int32_t m = v.r_m[q];
    const int64_t h = v.r_half[q];
    const uint64_t kb = v.kcap_off[q];
    const uint32_t G0 = __ldg(I.seg_off + J->seg), Gend = __ldg(I.seg_off + J->seg + 1);
    const int64_t from = (int64_t)J->bb * h;
    const int64_t end = min(((int64_t)J->bb + 2) * h, (int64_t)(Gend - G0));
    const int32_t W = (int32_t)max(end - from, (int64_t)0);
    if (lane == 0 && W > 0) atomicAdd(&v.mx->refine_kmers, (unsigned long long)W);
    int32_t li = 0, ld = 0;
    for (int32_t c0 = 0; c0 < W; c0 += 32) {
        const int32_t x = c0 + lane;
        const bool on[1] = {x < W};
        const uint64_t hx[1] = {on[0] ? __ldg(I.ref_h + G0 + (uint32_t)(from + x)) : 0};
        int32_t sx[1];
        pht_lookup_u<1>(v, q, hx, on, sx);
        uint32_t occ = 0, ooff = 0;
        if (sx[0] >= 0) {
            const SeedRec sr = v.sd[kb + sx[0]];
            occ = sr.os >> 1;
            ooff = sr.ooff;
        }
        for (unsigned mk = __ballot_sync(0xffffffffu, occ > 0); mk; mk &= mk - 1) {
            const int src = __ffs(mk) - 1;
            const uint32_t o = __shfl_sync(0xffffffffu, occ, src), off = __shfl_sync(0xffffffffu, ooff, src);
            if (o == 1) {
                const int32_t val = (int32_t)v.lcs_pos[kb + off];
                int32_t pi, pd;
                half_warp_places(Ti, li, val, Td, ld, -val, lane, pi, pd);
                if (lane == 0) Ti[pi] = val;
                if (lane == 16) Td[pd] = -val;
                li += pi == li;
                ld += pd == ld;
                __syncwarp();
                continue;
            }
            int32_t cd = -1;  // Td place of the group's previous value
            for (uint32_t c0 = 0; c0 < o; c0 += 32) {
                const uint32_t idx = c0 + (uint32_t)lane;
                const bool valid = idx < o;
                const int32_t val = valid ? (int32_t)v.lcs_pos[kb + off + idx] : 0;
                const int32_t qi = valid ? lane_lower_bound(Ti, li, val) : 0;
                const int32_t qd = valid ? lane_lower_bound(Td, ld, -val) : 0;
                const int32_t qn = __shfl_down_sync(0xffffffffu, qi, 1);
                const bool run_end = idx + 1 == o || lane == 31 || qn != qi;
                const int32_t pd = lane + max(cd + 1, warp_inclusive_max(valid ? qd - lane : INT32_MIN));
                __syncwarp();  // every search has read the tails
                if (valid && run_end) Ti[qi] = val;
                if (valid) Td[pd] = -val;
                li = max(li, __shfl_sync(0xffffffffu, qi, 0) + 1);
                cd = __shfl_sync(0xffffffffu, pd, (int)min(31u, o - 1 - c0));
                ld = max(ld, cd + 1);
                __syncwarp();
            }
        }
    }
    if (lane == 0) {
        J->score = __ddiv_rn((double)max(li, ld), (double)m);
        J->t_l = J->rmin;
        J->t_r = J->rmax;
        J->inter = J->matches;
        J->same = J->codir;
        J->s_sz = J->rmax - J->rmin;
    }
}

// One candidate window (best_fixed_length, src/shmap/scoring.rs:189-291).
// cntA (per seed: occurrences seen), ring (per seed: positions of its last
// occs occurrences), the difference array D and the strand prefix PC come
// from the warp's shared slice when the read is small enough (16-bit counts,
// positions and prefix: all below 2^15 there), else from its global scratch.
template <class CT, class PT>
__device__ __forceinline__ void refine_one(const BatchView& v, BucketJob* J, int32_t q, CT* cntA, int32_t* D, PT* PC,
                                           CT* ring, int lane, unsigned lt) {
    const bool ap = v.P.ap != 0;
    const DevIndex& I = v.I;
    const int32_t m = v.r_m[q], n_u = v.r_nu[q];
    const int64_t h = v.r_half[q];
    const uint64_t kb = v.kcap_off[q];
    const int32_t seg = J->seg;
    const uint32_t G0 = __ldg(I.seg_off + seg), Gend = __ldg(I.seg_off + seg + 1);
    const int64_t seglen = (int64_t)(Gend - G0);
    const int64_t from = (int64_t)J->bb * h;
    const int64_t end = min(((int64_t)J->bb + 2) * h, seglen);
    const int32_t W = (int32_t)(end - from);
    if (lane == 0 && W > 0) atomicAdd(&v.mx->refine_kmers, (unsigned long long)W);
    for (int32_t i = lane; i < n_u; i += 32) cntA[i] = 0;
    for (int32_t i = lane; i <= W; i += 32) D[i] = 0;
    __syncwarp();
    // phase 1: seed of every position, its occurrence interval of windows,
    // and the prefix PC of strand agreement (+1 same strand, -1 opposite).
    // REFINE_U chunks of 32 positions at a time: their reference k-mers,
    // probe lookups and seed records are fetched together, then the chunks
    // are folded in order.
    int32_t pc_carry = 0;
    if (lane == 0) PC[0] = 0;
    for (int32_t c00 = 0; c00 < W; c00 += 32 * REFINE_U) {
        uint64_t hx[REFINE_U];
        uint32_t rsx[REFINE_U], osx[REFINE_U], ooffx[REFINE_U];
        bool on[REFINE_U];
        int32_t sx[REFINE_U];
#pragma unroll
        for (int u = 0; u < REFINE_U; u++) {
            const int32_t x = c00 + 32 * u + lane;
            on[u] = x < W;
            const uint32_t gid = G0 + (uint32_t)(from + (on[u] ? x : 0));
            hx[u] = on[u] ? __ldg(I.ref_h + gid) : 0;
            rsx[u] = on[u] ? __ldg(I.ref_rs + gid) : 0;
        }
        pht_lookup_u<REFINE_U>(v, q, hx, on, sx);
#pragma unroll
        for (int u = 0; u < REFINE_U; u++) {
            const SeedRec sr = sx[u] >= 0 ? v.sd[kb + sx[u]] : SeedRec{0u, 0u, 0u, 0u};
            osx[u] = sr.os;
            ooffx[u] = sr.ooff;
        }
#pragma unroll
        for (int u = 0; u < REFINE_U; u++) {
            const int32_t c0 = c00 + 32 * u;
            if (c0 >= W) break;  // warp-uniform
            const int32_t x = c0 + lane;
            const bool valid = on[u];
            const int32_t s = sx[u];
            const uint32_t os = osx[u], rs = rsx[u];
            {
                const int32_t cv = (valid && s >= 0) ? (((os & 1u) == (rs & 1u)) ? 1 : -1) : 0;
                const int32_t inc = warp_inclusive_scan(cv);
                if (valid) PC[x + 1] = (PT)(pc_carry + inc);
                pc_carry += __shfl_sync(0xffffffffu, inc, 31);
            }
            const unsigned peers = __match_any_sync(0xffffffffu, s);
            int32_t t = 0, occ = 1, rho = 0, gsz = 0;
            const uint32_t ooff = ooffx[u];
            if (s >= 0) {
                occ = (int32_t)(os >> 1);
                rho = __popc(peers & lt);
                gsz = __popc(peers);
                t = (int32_t)cntA[s] + rho;
                int32_t p = -1;  // position (relative) of the occ-th previous occurrence, -1 = none
                // (positions, r and m are below 2^31: 32-bit arithmetic throughout)
                if (t >= occ) {
                    if (rho >= occ)  // in this chunk: the peer occ places before this lane
                        p = c0 + (occ == 1 ? 31 - __clz(peers & lt) : (int32_t)__fns(peers, 0, rho - occ + 1));
                    else
                        p = (int32_t)ring[ooff + (occ == 1 ? 0u : (uint32_t)(t % occ))];
                }
                int32_t Lj;
                if (!ap) {
                    Lj = x - m + 1;
                } else {  // first l with R[l] > R[x] - m
                    const int32_t rv = (int32_t)(rs >> 1) - m;
                    int32_t lo = 0, len = x;
                    while (len > 0) {
                        int32_t half = len >> 1;
                        if ((int32_t)(__ldg(I.ref_rs + G0 + from + lo + half) >> 1) <= rv) {
                            lo += half + 1;
                            len -= half + 1;
                        } else {
                            len = half;
                        }
                    }
                    Lj = lo;
                }
                const int32_t st = max(max(p + 1, Lj), 0);
                if (st <= x) {
                    atomicAdd(D + st, 1);
                    atomicAdd(D + x + 1, -1);
                }
            }
            __syncwarp();
            if (s >= 0) {
                if (rho >= gsz - occ) ring[ooff + (occ == 1 ? 0u : (uint32_t)(t % occ))] = (CT)x;
                if (rho == gsz - 1) cntA[s] = (CT)(t + 1);
            }
            __syncwarp();
        }
    }
    __syncwarp();
    // phase 2: intersection per window start, score, first maximum. Under
    // Containment every score is I / m for the same m, and distinct I < 2^31
    // give distinct quotients, so the first maximum of I is the first
    // maximum of the score: the division is done once, for the winner.
    const bool jac = v.P.metric == 1;
    double best = -1.0;
    int32_t bl = -1, bI = -1, bS = 0, br = 0;
    int32_t icarry = 0;
    for (int32_t c0 = 0; c0 < W; c0 += 32) {
        const int32_t x = c0 + lane;
        int32_t dv = x < W ? D[x] : 0;
        int32_t inc = warp_inclusive_scan(dv) + icarry;
        icarry = __shfl_sync(0xffffffffu, inc, 31);
        if (x < W) {
            int32_t r;
            if (!ap) {
                r = min(x + m, W);
            } else {
                const int32_t lim = (int32_t)(__ldg(I.ref_rs + G0 + from + x) >> 1) + m;
                int32_t lo = x, len = W - x;
                while (len > 0) {
                    int32_t half = len >> 1;
                    if ((int32_t)(__ldg(I.ref_rs + G0 + from + lo + half) >> 1) < lim) {
                        lo += half + 1;
                        len -= half + 1;
                    } else {
                        len = half;
                    }
                }
                r = lo;
            }
            const int32_t I_ = inc, sk = r - x;
            bool better;
            if (jac) {
                const double score = __ddiv_rn((double)I_, (double)(m + sk - I_));
                better = score > best;
                if (better) best = score;
            } else {
                better = I_ > bI;
            }
            if (better) {
                bl = x;
                bI = I_;
                bS = (int32_t)PC[r] - (int32_t)PC[x];
                br = r;
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double ob = __shfl_xor_sync(0xffffffffu, best, o);
        int32_t obl = __shfl_xor_sync(0xffffffffu, bl, o);
        int32_t obI = __shfl_xor_sync(0xffffffffu, bI, o);
        int32_t obS = __shfl_xor_sync(0xffffffffu, bS, o);
        int32_t obr = __shfl_xor_sync(0xffffffffu, br, o);
        const bool take = jac ? (ob > best || (ob == best && obl >= 0 && (bl < 0 || obl < bl)))
                              : (obI > bI || (obI == bI && obl >= 0 && (bl < 0 || obl < bl)));
        if (take) {
            best = ob;
            bl = obl;
            bI = obI;
            bS = obS;
            br = obr;
        }
    }
    if (!jac && bl >= 0) best = __ddiv_rn((double)bI, (double)m);
    if (lane == 0) {
        J->score = best;
        if (bl >= 0) {
            const int32_t tl = (int32_t)(__ldg(I.ref_rs + G0 + from + bl) >> 1);
            const int32_t tr = (int32_t)(__ldg(I.ref_rs + G0 + from + br - 1) >> 1);
            J->t_l = tl;
            J->t_r = tr;
            J->inter = bI;
            J->same = bS;
            J->s_sz = tr - tl + 1;
        }
    }
}

// Each warp's shared slice (REFINE_SLICE bytes, 16-bit counts, positions and
// strand prefix) holds, for reads of at most REFINE_SM k-mers whose window
// region has at most 2 REFINE_SM + 2 k-mers, all of a candidate's state: the
// rings and counts, the difference array and the strand prefix, so only the
// reference k-mers, the probe table and the seed records come from global
// memory. For larger reads (up to REFINE_SLICE / 4 k-mers) it holds the
// rings and counts, and the rest stays in the warp's global scratch; the
// largest reads keep everything there. Four CTAs of REFINE_WARPS warps fit
// an SM.
constexpr int REFINE_SM = 384;
constexpr int REFINE_WA = 2 * REFINE_SM + 2;  // window positions of the all-on-chip layout
constexpr size_t REFINE_OFF_CNT = 2 * (size_t)REFINE_SM;
constexpr size_t REFINE_OFF_D = 4 * (size_t)REFINE_SM;
constexpr size_t REFINE_OFF_PC = REFINE_OFF_D + 4 * (size_t)REFINE_WA;
constexpr size_t REFINE_SLICE = (REFINE_OFF_PC + 2 * (size_t)REFINE_WA + 15) / 16 * 16;
static_assert(REFINE_OFF_D % 4 == 0 && REFINE_OFF_PC % 2 == 0, "slice alignment");
static_assert(REFINE_WARPS * REFINE_SLICE * 4 + 4 * 1024 <= 228 * 1024, "four CTAs per SM");

__global__ void __launch_bounds__(REFINE_WARPS * 32, 4) k_refine(BatchView v, RefScratch rsc, int pass) {
    extern __shared__ __align__(16) uint8_t rf_dyn[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const uint32_t wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int32_t* const cntA = rsc.base + (size_t)wid * rsc.per_warp;
    int32_t* const D = cntA + rsc.nu_max;
    int32_t* const PC = D + rsc.wmax + 1;
    int32_t* const ring = PC + rsc.wmax + 1;
    uint8_t* const slice = rf_dyn + (size_t)wib * REFINE_SLICE;
    for (uint32_t jq; (jq = next_far(v, lane, pass)) != UINT32_MAX;) {
        BucketJob* J = v.jobs + jq;
        if (!refined_in(v, *J, jq, pass)) continue;
        if (lane == 0) atomicAdd(&v.mx->refined, 1ULL);
        const int32_t q = J->read;
        if (v.P.metric == MET_BUCKET_SH) {  // bucket_SH (scoring.rs:311-325)
            if (lane == 0) {
                J->score = J->sh;
                J->t_l = J->rmin;
                J->t_r = J->rmax;
                J->inter = J->matches;
                J->same = J->codir;
                J->s_sz = J->rmax - J->rmin;
            }
            continue;
        }
        // the candidate's window region (as refine_one forms it): its size picks the layout
        const int32_t m = v.r_m[q];
        const int64_t h = v.r_half[q];
        const int64_t seglen = (int64_t)(__ldg(v.I.seg_off + J->seg + 1) - __ldg(v.I.seg_off + J->seg));
        const int64_t W = min(((int64_t)J->bb + 2) * h, seglen) - (int64_t)J->bb * h;
        if (m <= REFINE_SM && W <= REFINE_WA - 1)  // n_u <= m: counts and rings fit
            refine_one<uint16_t, int16_t>(v, J, q, (uint16_t*)(slice + REFINE_OFF_CNT), (int32_t*)(slice + REFINE_OFF_D),
                                          (int16_t*)(slice + REFINE_OFF_PC), (uint16_t*)slice, lane, lt);
        else if (4 * (size_t)m <= REFINE_SLICE && W < 32768)
            refine_one<uint16_t, int32_t>(v, J, q, (uint16_t*)(slice + 2 * (size_t)m), D, PC, (uint16_t*)slice, lane,
                                          lt);
        else
            refine_one<int32_t, int32_t>(v, J, q, cntA, D, PC, ring, lane, lt);
        __syncwarp();
    }
}

// ------------------------------------------------------------------ rarity
// m_weight of each read (src/shmap/mod.rs:712-722): the sum over its seeds,
// in rarest-first order, of weight * occurrences, one f64 addition at a time
// in that order, as the reference adds them.
__global__ void k_rarity_mw(BatchView v) {
    for (int32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < v.n; q += gridDim.x * blockDim.x) {
        const uint64_t kb = v.kcap_off[q];
        const int32_t n_u = v.r_nu[q];
        double mw = 0.0;
        for (int32_t i = 0; i < n_u; i++) {
            const SeedRec sr = v.sd[kb + i];
            const uint32_t c = min(sr.cnt, v.P.wtab_n - 1u);
            mw = __dadd_rn(mw, __dmul_rn(v.P.wtab[c], (double)(sr.os >> 1)));
        }
        v.r_mw[q] = mw;
    }
}

// best_fixed_length with its rarity-weighted support (src/shmap/scoring.rs:
// 189-291). The reference keeps the support as one running f64 sum, adding a
// position's weight when it enters the window and counts (its seed's count in
// the window is still within the seed's occurrences) and subtracting a
// position's weight when it leaves the window while it counts; rounding makes
// that sum depend on the order of those operations, so it is replayed in
// that order by one lane. Which operations happen is decided in parallel
// first, from the same per-seed occurrence rings as refine_one:
//   enters counting: the seed's occs-th previous occurrence p lies before the
//     window start at which the position enters;
//   leaves counting: the seed's occs-th next occurrence (the position x whose
//     p is this one) lies at or past the window end.
// Without --rarity-weight the window is the one refine_one's arithmetic
// picks, and the replay runs up to it; with it, the score of every window is
// the weighted containment clamp(support / m_weight, 0, 1) and the replay
// takes its first maximum.
constexpr int RAR_ADD = 1, RAR_SUB = 2;

struct RarScratch {
    int32_t *cntA, *D, *PC, *ring, *nxt, *flag;
    double* wt;
};

__device__ __forceinline__ int32_t window_end(const DevIndex& I, uint32_t G0, int64_t from, int32_t x, int32_t W,
                                              int32_t m, bool ap) {
    if (!ap) return min(x + m, W);
    const int32_t lim = (int32_t)(__ldg(I.ref_rs + G0 + from + x) >> 1) + m;
    int32_t lo = x, len = W - x;
    while (len > 0) {
        const int32_t half = len >> 1;
        if ((int32_t)(__ldg(I.ref_rs + G0 + from + lo + half) >> 1) < lim) {
            lo += half + 1;
            len -= half + 1;
        } else {
            len = half;
        }
    }
    return lo;
}

__device__ void refine_rarity_one(const BatchView& v, BucketJob* J, int32_t q, const RarScratch& R, int lane,
                                  unsigned lt) {
    const bool ap = v.P.ap != 0;
    const DevIndex& I = v.I;
    const int32_t m = v.r_m[q], n_u = v.r_nu[q];
    const int64_t h = v.r_half[q];
    const uint64_t kb = v.kcap_off[q];
    const int32_t seg = J->seg;
    const uint32_t G0 = __ldg(I.seg_off + seg), Gend = __ldg(I.seg_off + seg + 1);
    const int64_t seglen = (int64_t)(Gend - G0);
    const int64_t from = (int64_t)J->bb * h;
    const int64_t end = min(((int64_t)J->bb + 2) * h, seglen);
    const int32_t W = (int32_t)(end - from);
    if (lane == 0 && W > 0) atomicAdd(&v.mx->refine_kmers, (unsigned long long)W);
    for (int32_t i = lane; i < n_u; i += 32) R.cntA[i] = 0;
    for (int32_t i = lane; i <= W; i += 32) {
        R.D[i] = 0;
        R.nxt[i] = INT32_MAX;
    }
    __syncwarp();
    int32_t pc_carry = 0;
    if (lane == 0) R.PC[0] = 0;
    for (int32_t c0 = 0; c0 < W; c0 += 32) {
        const int32_t x = c0 + lane;
        const bool valid = x < W;
        const uint32_t gid = G0 + (uint32_t)(from + (valid ? x : 0));
        uint64_t hx[1] = {valid ? __ldg(I.ref_h + gid) : 0};
        const uint32_t rs = valid ? __ldg(I.ref_rs + gid) : 0;
        bool on[1] = {valid};
        int32_t sx[1];
        pht_lookup_u<1>(v, q, hx, on, sx);
        const int32_t s = sx[0];
        const SeedRec sr = s >= 0 ? v.sd[kb + s] : SeedRec{0u, 0u, 0u, 0u};
        {
            const int32_t cv = (valid && s >= 0) ? (((sr.os & 1u) == (rs & 1u)) ? 1 : -1) : 0;
            const int32_t inc = warp_inclusive_scan(cv);
            if (valid) R.PC[x + 1] = pc_carry + inc;
            pc_carry += __shfl_sync(0xffffffffu, inc, 31);
        }
        const unsigned peers = __match_any_sync(0xffffffffu, s);
        int32_t t = 0, occ = 1, rho = 0, gsz = 0;
        int32_t fl = 0;
        if (s >= 0) {
            occ = (int32_t)(sr.os >> 1);
            rho = __popc(peers & lt);
            gsz = __popc(peers);
            t = R.cntA[s] + rho;
            int32_t p = -1;  // the occ-th previous occurrence in the window region, -1 = none
            if (t >= occ) {
                if (rho >= occ)
                    p = c0 + (occ == 1 ? 31 - __clz(peers & lt) : (int32_t)__fns(peers, 0, rho - occ + 1));
                else
                    p = R.ring[sr.ooff + (occ == 1 ? 0u : (uint32_t)(t % occ))];
            }
            int32_t Lj;
            if (!ap) {
                Lj = x - m + 1;
            } else {  // first l with R[l] > R[x] - m
                const int32_t rv = (int32_t)(rs >> 1) - m;
                int32_t lo = 0, len = x;
                while (len > 0) {
                    int32_t half = len >> 1;
                    if ((int32_t)(__ldg(I.ref_rs + G0 + from + lo + half) >> 1) <= rv) {
                        lo += half + 1;
                        len -= half + 1;
                    } else {
                        len = half;
                    }
                }
                Lj = lo;
            }
            const int32_t lin = max(Lj, 0);  // the window start at which x enters
            const int32_t st = max(p + 1, lin);
            if (st <= x) {
                atomicAdd(R.D + st, 1);
                atomicAdd(R.D + x + 1, -1);
            }
            if (p < lin) fl |= RAR_ADD;
            if (p >= 0) R.nxt[p] = x;  // x is p's occs-th next occurrence
            R.wt[x] = v.P.wtab[min(sr.cnt, v.P.wtab_n - 1u)];
        }
        if (valid) R.flag[x] = s >= 0 ? fl : -1;
        __syncwarp();
        if (s >= 0) {
            if (rho >= gsz - occ) R.ring[sr.ooff + (occ == 1 ? 0u : (uint32_t)(t % occ))] = x;
            if (rho == gsz - 1) R.cntA[s] = t + 1;
        }
        __syncwarp();
    }
    // leaves counting: its occs-th next occurrence at or past the window end
    for (int32_t x = lane; x < W; x += 32) {
        const int32_t f = R.flag[x];
        if (f >= 0 && R.nxt[x] >= window_end(I, G0, from, x, W, m, ap)) R.flag[x] = f | RAR_SUB;
    }
    // intersection per window start (prefix of D, kept in D) and, without
    // --rarity-weight, the window refine_one's arithmetic picks
    const bool jac = v.P.metric == 1;
    const bool rw = v.P.rw_score != 0;
    double best = -1.0;
    int32_t bl = -1, bI = -1;
    int32_t icarry = 0;
    for (int32_t c0 = 0; c0 < W; c0 += 32) {
        const int32_t x = c0 + lane;
        int32_t dv = x < W ? R.D[x] : 0;
        int32_t inc = warp_inclusive_scan(dv) + icarry;
        icarry = __shfl_sync(0xffffffffu, inc, 31);
        if (x < W) {
            R.D[x] = inc;
            if (!rw) {
                const int32_t r = window_end(I, G0, from, x, W, m, ap);
                bool better;
                if (jac) {
                    const double score = __ddiv_rn((double)inc, (double)(m + (r - x) - inc));
                    better = score > best;
                    if (better) best = score;
                } else {
                    better = inc > bI;
                }
                if (better) {
                    bl = x;
                    bI = inc;
                }
            }
        }
    }
    if (!rw) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            double ob = __shfl_xor_sync(0xffffffffu, best, o);
            int32_t obl = __shfl_xor_sync(0xffffffffu, bl, o);
            int32_t obI = __shfl_xor_sync(0xffffffffu, bI, o);
            const bool take = jac ? (ob > best || (ob == best && obl >= 0 && (bl < 0 || obl < bl)))
                                  : (obI > bI || (obI == bI && obl >= 0 && (bl < 0 || obl < bl)));
            if (take) {
                best = ob;
                bl = obl;
                bI = obI;
            }
        }
        if (!jac && bl >= 0) best = __ddiv_rn((double)bI, (double)m);
    }
    __syncwarp();
    if (lane == 0) {
        // the reference's running sum, in its order, up to the chosen window
        // (or over every window, taking the first maximum of the weighted score)
        const double mw = rw ? v.r_mw[q] : 0.0;
        const bool mono = mw > 0.0 && mw < INFINITY;
        double w = 0.0, wbest = 0.0;
        int32_t r = 0;
        if (rw) {
            best = -1.0;
            bl = -1;
        }
        double w_at_best = 0.0;
        const int32_t last = rw ? W - 1 : bl;
        for (int32_t l = 0; l <= last; l++) {
            const int32_t rl = window_end(I, G0, from, l, W, m, ap);
            for (; r < rl; r++)
                if (R.flag[r] > 0 && (R.flag[r] & RAR_ADD)) w = __dadd_rn(w, R.wt[r]);
            if (rw) {
                // the score is monotone in w (for a positive finite m_weight):
                // a window can beat the best only with more support
                if (!mono || bl < 0 || w > w_at_best) {
                    double sc = __ddiv_rn(w, mw);  // min(max(x, 0), 1), NaN kept, as clamp does
                    sc = sc < 0.0 ? 0.0 : sc;
                    sc = 1.0 < sc ? 1.0 : sc;
                    if (sc > best) {
                        best = sc;
                        bl = l;
                        w_at_best = w;
                    }
                }
            } else if (l == bl) {
                wbest = w;
            }
            if (R.flag[l] > 0 && (R.flag[l] & RAR_SUB)) w = __dsub_rn(w, R.wt[l]);
        }
        if (rw) wbest = w_at_best;
        J->score = best;
        J->support = wbest;
        if (bl >= 0) {
            const int32_t br = window_end(I, G0, from, bl, W, m, ap);
            const int32_t tl = (int32_t)(__ldg(I.ref_rs + G0 + from + bl) >> 1);
            const int32_t tr = (int32_t)(__ldg(I.ref_rs + G0 + from + br - 1) >> 1);
            J->t_l = tl;
            J->t_r = tr;
            J->inter = R.D[bl];
            J->same = R.PC[br] - R.PC[bl];
            J->s_sz = tr - tl + 1;
        }
    }
}

__global__ void __launch_bounds__(REFINE_WARPS * 32, 4) k_refine_rarity(BatchView v, RefScratch rsc) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const uint32_t wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t nfar = v.mx->n_far;
    int32_t* const base = rsc.base + (size_t)wid * rsc.per_warp;
    RarScratch R;
    R.cntA = base;
    R.D = R.cntA + rsc.nu_max;
    R.PC = R.D + rsc.wmax + 1;
    R.ring = R.PC + rsc.wmax + 1;
    R.nxt = R.ring + rsc.ring_n;
    R.flag = R.nxt + rsc.wmax + 1;
    R.wt = (double*)(base + rsc.wt_at);
    (void)nfar;
    (void)nwarps;
    for (uint32_t jq; (jq = next_far(v, lane)) != UINT32_MAX;) {
        BucketJob* J = v.jobs + jq;
        refine_rarity_one(v, J, J->read, R, lane, lt);
        __syncwarp();
    }
}

// bucket_LCS over the candidates in cfar, a warp at a time, taken from a
// queue (their costs differ by orders of magnitude: a window in a tandem
// repeat feeds each seed's many read positions once per k-mer). The two tail
// arrays of a read of at most LCS_SM k-mers are in the warp's shared slice,
// those of larger reads in its global scratch.
constexpr int LCS_WARPS = 8;
constexpr int LCS_SM = 512;
__global__ void __launch_bounds__(LCS_WARPS * 32, 5) k_refine_lcs(BatchView v, RefScratch rsc) {
    __shared__ int32_t s_tails[LCS_WARPS][2 * LCS_SM];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const uint32_t wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nfar = v.mx->n_far;
    int32_t* const D = rsc.base + (size_t)wid * rsc.per_warp + rsc.nu_max;
    for (;;) {
        uint32_t ci = 0;
        if (lane == 0) ci = atomicAdd(&v.mx->lcs_next, 1u);
        ci = __shfl_sync(0xffffffffu, ci, 0);
        if (ci >= nfar) break;
        BucketJob* J = v.jobs + v.cfar[ci];
        const int32_t q = J->read, m = v.r_m[q];
        if (m <= LCS_SM)
            lcs_one(v, J, q, s_tails[wib], s_tails[wib] + LCS_SM, lane);
        else
            lcs_one(v, J, q, D, D + m, lane);
        __syncwarp();
    }
}

// ------------------------------------------------------------------ K7 refinement on chip
// Candidates of the reads refine_on_chip selects, a warp at a time: the
// read's seed table is built in the warp's shared slice from its seed hashes
// and records, then its candidate windows are refined against it, with the
// per-seed counts and rings and the window's difference array on chip too.
// Only the reference k-mers of the windows are read from global memory.
// Per-warp slice (7 KB, so that four 8-warp CTAs fit an SM):
//   tslot  u16[RCHIP_T]      probe table: seed index + 1, or 0 (empty)
//   shash  u64[RCHIP_M]      each seed's hash
//   sinfo  u32[RCHIP_M]      occs << 1 | strand, ring offset << 16
//   D      i32[2 RCHIP_M]    difference array over window starts
//   cntA   u16[RCHIP_M]      occurrences seen per seed
//   ring   u16[RCHIP_M]      positions of each seed's last occs occurrences
//   smask  u32[2 RCHIP_M/16] per 32 positions: ballots of same / opposite strand
constexpr int RCHIP_WARPS = 8;
constexpr int RCHIP_CHUNK = 8;  // candidates a warp takes at once (<= 32)
constexpr int RCHIP_T = 512;    // a power of two >= 2 RCHIP_M
constexpr size_t RCHIP_OFF_HASH = 2 * (size_t)RCHIP_T;
constexpr size_t RCHIP_OFF_INFO = RCHIP_OFF_HASH + 8 * (size_t)RCHIP_M;
constexpr size_t RCHIP_OFF_D = RCHIP_OFF_INFO + 4 * (size_t)RCHIP_M;
constexpr size_t RCHIP_OFF_CNT = RCHIP_OFF_D + 4 * 2 * (size_t)RCHIP_M;
constexpr size_t RCHIP_OFF_RING = RCHIP_OFF_CNT + 2 * (size_t)RCHIP_M;
constexpr size_t RCHIP_OFF_MASK = RCHIP_OFF_RING + 2 * (size_t)RCHIP_M;
constexpr size_t RCHIP_SLICE = (RCHIP_OFF_MASK + 4 * 2 * ((2 * (size_t)RCHIP_M + 31) / 32) + 15) / 16 * 16;
static_assert(RCHIP_T >= 2 * RCHIP_M && (RCHIP_T & (RCHIP_T - 1)) == 0, "probe table size");
static_assert(RCHIP_OFF_HASH % 8 == 0 && RCHIP_OFF_D % 4 == 0 && RCHIP_OFF_MASK % 4 == 0, "slice alignment");
static_assert(RCHIP_SLICE <= 7168, "four CTAs of RCHIP_WARPS warps per SM");

// Seed of hash x in the on-chip table, or -1 (the table keeps empty slots).
__device__ __forceinline__ int32_t chip_lookup(const uint16_t* tslot, const uint64_t* shash, uint32_t T, uint64_t x) {
    uint32_t sl = (uint32_t)x & (T - 1);
    for (;;) {
        const uint32_t t = tslot[sl];
        if (t == 0) return -1;
        if (shash[t - 1] == x) return (int32_t)t - 1;
        sl = (sl + 1) & (T - 1);
    }
}

// Inserts seed i (hash hs) into the table: a compare-and-swap on the word
// that holds the slot.
__device__ __forceinline__ void chip_insert(uint16_t* tslot, uint32_t T, uint64_t hs, uint32_t i) {
    uint32_t sl = (uint32_t)hs & (T - 1);
    for (;;) {
        uint32_t* w = (uint32_t*)tslot + (sl >> 1);
        const uint32_t sh = (sl & 1u) * 16u;
        uint32_t old = *(volatile uint32_t*)w;
        while (((old >> sh) & 0xffffu) == 0) {
            const uint32_t got = atomicCAS(w, old, old | ((i + 1u) << sh));
            if (got == old) return;
            old = got;  // the other slot of the word changed: look again
        }
        sl = (sl + 1) & (T - 1);
    }
}

// best_fixed_length (src/shmap/scoring.rs:189-291) for one candidate window,
// the arithmetic of refine_one with every per-read array on chip; the strand
// agreement of the winning window is counted from the ballots.
__device__ __forceinline__ void refine_chip_one(const BatchView& v, BucketJob* J, int32_t m, int32_t n_u, int64_t h,
                                                uint32_t T, const uint16_t* tslot, const uint64_t* shash,
                                                const uint32_t* sinfo, uint16_t* cntA, uint16_t* ring, int32_t* D,
                                                uint32_t* smask, int lane, unsigned lt) {
    const DevIndex& I = v.I;
    const int32_t seg = J->seg;
    const uint32_t G0 = __ldg(I.seg_off + seg), Gend = __ldg(I.seg_off + seg + 1);
    const int64_t seglen = (int64_t)(Gend - G0);
    const int64_t from = (int64_t)J->bb * h;
    const int64_t end = min(((int64_t)J->bb + 2) * h, seglen);
    const int32_t W = (int32_t)(end - from);  // <= 2 h <= 2 RCHIP_M
    if (lane == 0 && W > 0) atomicAdd(&v.mx->refine_kmers, (unsigned long long)W);
    for (int32_t i = lane; i < n_u; i += 32) cntA[i] = 0;
    for (int32_t i = lane; i < W; i += 32) D[i] = 0;
    __syncwarp();
    // the reference k-mers of REFINE_U chunks of 32 positions; the next
    // chunks' are loaded while these are folded
    uint64_t hx[REFINE_U];
    uint32_t rsx[REFINE_U];
#pragma unroll
    for (int u = 0; u < REFINE_U; u++) {
        const int32_t x = 32 * u + lane;
        const uint32_t gid = G0 + (uint32_t)(from + (x < W ? x : 0));
        hx[u] = x < W ? __ldg(I.ref_h + gid) : 0;
        rsx[u] = x < W ? __ldg(I.ref_rs + gid) : 0;
    }
    for (int32_t c00 = 0; c00 < W; c00 += 32 * REFINE_U) {
        uint64_t hy[REFINE_U];
        uint32_t ry[REFINE_U];
        int32_t sx[REFINE_U];
        uint32_t sxi[REFINE_U];
#pragma unroll
        for (int u = 0; u < REFINE_U; u++) {
            const int32_t y = c00 + 32 * (REFINE_U + u) + lane;
            const uint32_t gid = G0 + (uint32_t)(from + (y < W ? y : 0));
            hy[u] = y < W ? __ldg(I.ref_h + gid) : 0;
            ry[u] = y < W ? __ldg(I.ref_rs + gid) : 0;
        }
#pragma unroll
        for (int u = 0; u < REFINE_U; u++)  // the chunks' lookups together
            sx[u] = c00 + 32 * u + lane < W ? chip_lookup(tslot, shash, T, hx[u]) : -1;
#pragma unroll
        for (int u = 0; u < REFINE_U; u++) sxi[u] = sx[u] >= 0 ? sinfo[sx[u]] : 0u;
#pragma unroll
        for (int u = 0; u < REFINE_U; u++) {
            const int32_t c0 = c00 + 32 * u;
            if (c0 >= W) break;  // warp-uniform
            const int32_t x = c0 + lane;
            const int32_t s = sx[u];
            const uint32_t os = sxi[u] & 0xffffu, ooff = sxi[u] >> 16;
            {
                const bool same = s >= 0 && ((os ^ rsx[u]) & 1u) == 0;
                const unsigned bs = __ballot_sync(0xffffffffu, same);
                const unsigned bo = __ballot_sync(0xffffffffu, s >= 0 && !same);
                if (lane == 0) {
                    smask[2 * (c0 >> 5)] = bs;
                    smask[2 * (c0 >> 5) + 1] = bo;
                }
            }
            const unsigned peers = __match_any_sync(0xffffffffu, s);
            int32_t t = 0, occ = 1, rho = 0, gsz = 0;
            if (s >= 0) {
                occ = (int32_t)(os >> 1);
                rho = __popc(peers & lt);
                gsz = __popc(peers);
                t = (int32_t)cntA[s] + rho;
                int32_t p = -1;  // position of the occ-th previous occurrence, -1 = none
                if (t >= occ) {
                    if (rho >= occ)  // in this chunk: the peer occ places before this lane
                        p = c0 + (occ == 1 ? 31 - __clz(peers & lt) : (int32_t)__fns(peers, 0, rho - occ + 1));
                    else
                        p = ring[ooff + (occ == 1 ? 0u : (uint32_t)(t % occ))];
                }
                const int32_t st = max(max(p + 1, x - m + 1), 0);
                if (st <= x) {
                    atomicAdd(D + st, 1);
                    if (x + 1 < W) atomicAdd(D + x + 1, -1);  // D[W] is never read
                }
            }
            __syncwarp();
            if (s >= 0) {
                if (rho >= gsz - occ) ring[ooff + (occ == 1 ? 0u : (uint32_t)(t % occ))] = (uint16_t)x;
                if (rho == gsz - 1) cntA[s] = (uint16_t)(t + 1);
            }
            __syncwarp();
        }
#pragma unroll
        for (int u = 0; u < REFINE_U; u++) {
            hx[u] = hy[u];
            rsx[u] = ry[u];
        }
    }
    __syncwarp();
    // intersection per window start, score, first maximum (as refine_one)
    const bool jac = v.P.metric == 1;
    double best = -1.0;
    int32_t bl = -1, bI = -1, br = 0;
    int32_t icarry = 0;
    for (int32_t c0 = 0; c0 < W; c0 += 32) {
        const int32_t x = c0 + lane;
        const int32_t dv = x < W ? D[x] : 0;
        const int32_t inc = warp_inclusive_scan(dv) + icarry;
        icarry = __shfl_sync(0xffffffffu, inc, 31);
        if (x < W) {
            const int32_t r = min(x + m, W);
            const int32_t I_ = inc, sk = r - x;
            bool better;
            if (jac) {
                const double score = __ddiv_rn((double)I_, (double)(m + sk - I_));
                better = score > best;
                if (better) best = score;
            } else {
                better = I_ > bI;
            }
            if (better) {
                bl = x;
                bI = I_;
                br = r;
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double ob = __shfl_xor_sync(0xffffffffu, best, o);
        int32_t obl = __shfl_xor_sync(0xffffffffu, bl, o);
        int32_t obI = __shfl_xor_sync(0xffffffffu, bI, o);
        int32_t obr = __shfl_xor_sync(0xffffffffu, br, o);
        const bool take = jac ? (ob > best || (ob == best && obl >= 0 && (bl < 0 || obl < bl)))
                              : (obI > bI || (obI == bI && obl >= 0 && (bl < 0 || obl < bl)));
        if (take) {
            best = ob;
            bl = obl;
            bI = obI;
            br = obr;
        }
    }
    if (!jac && bl >= 0) best = __ddiv_rn((double)bI, (double)m);
    // every lane holds the winner: the strand agreement over [bl, br) from
    // the ballots, a lane per 32 positions
    int32_t same = 0;
    if (bl >= 0) {
        const int32_t j = (bl >> 5) + lane, jl = (br - 1) >> 5;
        if (j <= jl) {
            uint32_t keep = 0xffffffffu;
            if (j == (bl >> 5)) keep &= 0xffffffffu << (bl & 31);
            if (j == jl) keep &= 0xffffffffu >> (31 - ((br - 1) & 31));
            same = __popc(smask[2 * j] & keep) - __popc(smask[2 * j + 1] & keep);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) same += __shfl_xor_sync(0xffffffffu, same, o);
    }
    if (lane == 0) {
        J->score = best;
        if (bl >= 0) {
            const int32_t tl = (int32_t)(__ldg(I.ref_rs + G0 + from + bl) >> 1);
            const int32_t tr = (int32_t)(__ldg(I.ref_rs + G0 + from + br - 1) >> 1);
            J->t_l = tl;
            J->t_r = tr;
            J->inter = bI;
            J->same = same;
            J->s_sz = tr - tl + 1;
        }
    }
}

__global__ void __launch_bounds__(RCHIP_WARPS * 32, 4) k_refine_chip(BatchView v, int pass) {
    extern __shared__ __align__(16) uint8_t rc_smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    uint8_t* base = rc_smem + (size_t)wib * RCHIP_SLICE;
    uint16_t* tslot = (uint16_t*)base;
    uint64_t* shash = (uint64_t*)(base + RCHIP_OFF_HASH);
    uint32_t* sinfo = (uint32_t*)(base + RCHIP_OFF_INFO);
    int32_t* D = (int32_t*)(base + RCHIP_OFF_D);
    uint16_t* cntA = (uint16_t*)(base + RCHIP_OFF_CNT);
    uint16_t* ring = (uint16_t*)(base + RCHIP_OFF_RING);
    uint32_t* smask = (uint32_t*)(base + RCHIP_OFF_MASK);
    // work comes in chunks of RCHIP_CHUNK consecutive candidates (a read's
    // candidates are consecutive) from a batch counter, the next chunk's
    // number fetched while this one is refined; the seed table is rebuilt
    // only when the read changes
    const uint32_t ncand = v.coff[v.n];
    uint32_t nxt = 0;
    if (lane == 0) nxt = atomicAdd(&v.mx->refine_next[pass], 1u);
    int32_t cur = -1;  // the read whose table is staged
    uint32_t T = 32;
    for (;;) {
        const uint32_t ci0 = __shfl_sync(0xffffffffu, nxt, 0) * (uint32_t)RCHIP_CHUNK;
        if (ci0 >= ncand) break;
        if (lane == 0) nxt = atomicAdd(&v.mx->refine_next[pass], 1u);
        int32_t ql = -1;
        bool onl = false;
        if (lane < RCHIP_CHUNK && ci0 + lane < ncand) {
            const uint32_t ji = v.cidx[ci0 + lane];
            const BucketJob& Jl = v.jobs[ji];
            ql = Jl.read;
            onl = refine_on_chip(v.P, (uint32_t)v.r_m[ql], v.r_half[ql]) && refined_in(v, Jl, ji, pass);
        }
        const unsigned on_mask = __ballot_sync(0xffffffffu, onl);
        if (lane == 0 && on_mask) atomicAdd(&v.mx->refined, (unsigned long long)__popc(on_mask));
        const uint32_t nc = min((uint32_t)RCHIP_CHUNK, ncand - ci0);
        for (uint32_t j = 0; j < nc; j++) {
            const int32_t q = __shfl_sync(0xffffffffu, ql, (int)j);
            if (!__shfl_sync(0xffffffffu, onl, (int)j)) continue;  // k_refine's, or not refined in this pass
            const int32_t m = v.r_m[q], n_u = v.r_nu[q];  // n_u <= m <= RCHIP_M
            if (q != cur) {
                const uint64_t kb = v.kcap_off[q];
                T = max(32u, (uint32_t)pow2_ceil(2ULL * (uint64_t)n_u));  // <= RCHIP_T
                for (uint32_t i = lane; i < T / 2; i += 32) ((uint32_t*)tslot)[i] = 0u;
#pragma unroll 4
                for (int32_t i = lane; i < n_u; i += 32) {
                    const SeedRec sr = v.sd[kb + i];
                    shash[i] = v.sd_h[kb + i];
                    sinfo[i] = sr.os | (sr.ooff << 16);
                }
                __syncwarp();
                for (int32_t i = lane; i < n_u; i += 32) chip_insert(tslot, T, shash[i], (uint32_t)i);
                __syncwarp();
                cur = q;
            }
            refine_chip_one(v, v.jobs + v.cidx[ci0 + j], m, n_u, (int64_t)v.r_half[q], T, tslot, shash, sinfo, cntA,
                            ring, D, smask, lane, lt);
            __syncwarp();
        }
    }
}

// ------------------------------------------------------------------ K8 sweeps and record
// Per read (one warp): the candidates in the reference's bucket order, then
// the two sweeps on their precomputed results. Small candidate sets are
// staged in shared memory and rank-sorted; large ones are bitonic-sorted in a
// global scratch region by the same warp.
constexpr int SWEEP_WARPS = 4;
constexpr int SWEEP_CAP = 64;

struct SweepCand {
    double sh, score;
    int32_t seg, bb, m0, t_l, t_r, job;
};

__device__ __forceinline__ bool sc_less(const SweepCand& a, const SweepCand& b) {
    if (a.m0 != b.m0) return a.m0 > b.m0;  // get_sorted_buckets: matches desc (buckets.rs:697-704)
    if (a.seg != b.seg) return a.seg < b.seg;
    return a.bb < b.bb;
}

__device__ __forceinline__ SweepCand load_cand(const BucketJob& j, uint32_t ji) {
    SweepCand c;
    c.sh = j.sh;
    c.score = j.score;
    c.seg = j.seg;
    c.bb = j.bb;
    c.m0 = j.m0;
    c.t_l = j.t_l;
    c.t_r = j.t_r;
    c.job = (int32_t)ji;
    return c;
}

__device__ double overlap_of(const SweepCand& a, const SweepCand& b) {  // mapping.rs:412-420
    if (a.seg != b.seg) return -0.0;
    int32_t cap = max(0, min(a.t_r, b.t_r) - max(a.t_l, b.t_l));
    int32_t cup = max(a.t_r, b.t_r) - min(a.t_l, b.t_l);
    return __ddiv_rn((double)cap, (double)cup);
}

__global__ void __launch_bounds__(SWEEP_WARPS * 32) k_sweep(BatchView v, SweepCand* __restrict__ big_scr) {
    __shared__ SweepCand sm[SWEEP_WARPS][SWEEP_CAP];
    __shared__ SweepCand srt[SWEEP_WARPS][SWEEP_CAP];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int32_t gw = blockIdx.x * SWEEP_WARPS + w, nwarps = gridDim.x * SWEEP_WARPS;
    for (int32_t q = gw; q < v.n; q += nwarps) {
        const uint32_t c0 = v.coff[q], nc = v.coff[q + 1] - c0;
        const SweepCand* L;
        if (nc <= SWEEP_CAP) {
            for (uint32_t i = lane; i < nc; i += 32) {
                uint32_t ji = v.cidx[c0 + i];
                sm[w][i] = load_cand(v.jobs[ji], ji);
            }
            __syncwarp();
            for (uint32_t i = lane; i < nc; i += 32) {
                const SweepCand me = sm[w][i];
                uint32_t rank = 0;
                for (uint32_t k = 0; k < nc; k++) rank += sc_less(sm[w][k], me) ? 1u : 0u;
                srt[w][rank] = me;
            }
            __syncwarp();
            L = srt[w];
        } else {
            // regions of 2*nc slots at 2*c0 hold a power of two >= nc
            SweepCand* G = big_scr + 2 * (size_t)c0;
            uint32_t P = 1;
            while (P < nc) P <<= 1;
            for (uint32_t i = lane; i < P; i += 32) {
                if (i < nc) {
                    uint32_t ji = v.cidx[c0 + i];
                    G[i] = load_cand(v.jobs[ji], ji);
                } else {
                    G[i].m0 = INT32_MIN;  // sorts after every real candidate
                    G[i].seg = INT32_MAX;
                    G[i].bb = INT32_MAX;
                    G[i].job = -1;
                }
            }
            __syncwarp();
            for (uint32_t k = 2; k <= P; k <<= 1)
                for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                    for (uint32_t t = lane; t < P / 2; t += 32) {
                        uint32_t i = ((t & ~(j - 1)) << 1) | (t & (j - 1)), l = i + j;  // j is a power of two
                        bool asc = (i & k) == 0;
                        SweepCand a = G[i], b = G[l];
                        if (sc_less(b, a) == asc) {
                            G[i] = b;
                            G[l] = a;
                        }
                    }
                    __syncwarp();
                }
            L = G;
        }
        if (lane == 0) {
            const int32_t st = v.r_status[q];
            shm_map_record rec;
            memset(&rec, 0, sizeof rec);
            rec.read_len = (int32_t)(v.roff[q + 1] - v.roff[q]);
            rec.sketch_size = v.r_m[q];
            rec.seeds = v.r_S[q];
            rec.total_matches = (int32_t)v.r_smatch[q];
            rec.seed_matches = (int32_t)v.r_smatch[q];
            rec.max_seed_matches = v.r_maxseed[q];
            rec.seeded_buckets = (int32_t)v.r_seeded[q];
            rec.bucket_seg = rec.bucket_b = rec.bucket2_seg = rec.bucket2_b = -1;
            rec.intersection2 = -1;
            rec.score2 = -1.0;
            rec.status = st;
            if (st == ST_UNMAPPED) {
                const bool nbp = v.P.nbp != 0;
                int32_t fb = 0;
                // the rarity tie-break (scoring.rs:409-416, 453-481): a bucket is
                // admitted above thr - band * |thr|, and one within the band of the
                // incumbent's score takes over only with more rarity support
                const double tb = v.P.tiebreak;
                auto admit_of = [&](double t) { return tb > 0.0 ? __dsub_rn(t, __dmul_rn(tb, fabs(t))) : t; };
                auto takes = [&](const SweepCand& c, const SweepCand& cur) {
                    if (tb > 0.0 && fabs(__dsub_rn(c.score, cur.score)) <= __dmul_rn(tb, fabs(cur.score)))
                        return v.jobs[c.job].support > v.jobs[cur.job].support;
                    return c.score > cur.score;
                };
                // pass 1 (mod.rs:816-832): thr = theta, no forbidden region
                double thr = v.P.theta;
                int32_t b1 = -1;
                for (uint32_t i = 0; i < nc; i++) {
                    const SweepCand& c = L[i];
                    if (!nbp && !(c.sh >= thr)) continue;
                    if (c.score > admit_of(thr)) {
                        fb++;
                        if (b1 < 0 || takes(c, L[b1])) {
                            thr = fmax(thr, c.score);
                            b1 = (int32_t)i;
                        }
                    }
                }
                int32_t b2 = -1;
                if (b1 >= 0) {
                    // pass 2 (mod.rs:835-859): thr = best * (1 - d), best forbidden
                    const SweepCand B1 = L[b1];
                    thr = __dmul_rn(B1.score, __dsub_rn(1.0, v.P.min_diff));
                    for (uint32_t i = 0; i < nc; i++) {
                        const SweepCand& c = L[i];
                        if (!nbp && !(c.sh >= thr)) continue;
                        if (c.score > admit_of(thr)) {
                            fb++;
                            if (overlap_of(c, B1) < v.P.max_overlap) {
                                if (b2 < 0 || takes(c, L[b2])) {
                                    thr = fmax(thr, c.score);
                                    b2 = (int32_t)i;
                                }
                            }
                        }
                    }
                }
                rec.final_buckets = fb;
                if (b1 >= 0) {
                    const BucketJob& B = v.jobs[L[b1].job];
                    rec.status = ST_MAPPED;
                    rec.score = B.score;
                    rec.sh = B.sh;
                    rec.p_start = 0;
                    rec.p_end = bucket_metric(v.P) ? rec.read_len - 1 : rec.read_len - v.P.k - 1;
                    rec.segm_id = B.seg;
                    rec.t_l = B.t_l;
                    rec.t_r = B.t_r;
                    rec.same_strand = B.same;
                    rec.intersection = B.inter;
                    rec.s_sz = B.s_sz;
                    rec.bucket_seg = B.seg;
                    rec.bucket_b = B.bb;
                    if (b2 >= 0) {
                        const BucketJob& C2 = v.jobs[L[b2].job];
                        rec.has_second = 1;
                        rec.intersection2 = C2.inter;
                        rec.score2 = C2.score;
                        rec.bucket2_seg = C2.seg;
                        rec.bucket2_b = C2.bb;
                    }
                }
            } else if (st == ST_OVERFLOW) {
                uint32_t k = atomicAdd(&v.mx->n_overflow, 1u);
                const uint64_t eb = v.r_eb[q];
                v.ovf_list[4 * (size_t)k] = (uint32_t)q;
                v.ovf_list[4 * (size_t)k + 1] = v.kcnt[q];
                v.ovf_list[4 * (size_t)k + 2] = (uint32_t)eb;
                v.ovf_list[4 * (size_t)k + 3] = (uint32_t)(eb >> 32);
            }
            v.out[q] = rec;
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------------ host side
// A host<->device copy on stream s, counted in the context's work counters.
static void copy_async(MapCtx* c, void* dst, const void* src, size_t bytes, cudaMemcpyKind kind, cudaStream_t s) {
    SHM_CUDA(cudaMemcpyAsync(dst, src, bytes, kind, s));
    if (kind == cudaMemcpyHostToDevice) c->work[W_H2D_BYTES] += (int64_t)bytes;
    else if (kind == cudaMemcpyDeviceToHost) c->work[W_D2H_BYTES] += (int64_t)bytes;
}

const char* const STAGE_NAMES[N_STAGES] = {"sketch", "seedprep", "contrib", "bscan", "extend", "refine", "sweep", "aux"};
const char* const WORK_NAMES[N_WORK] = {"reads", "bases", "kmers", "distinct_seeds", "processed_seeds",
                                        "seed_hits", "buckets", "bucket_jobs", "extension_seeds", "candidates",
                                        "refine_kmers", "h2d_bytes", "d2h_bytes", "refined_candidates",
                                        "second_tables"};


// Event pairs around each stage of a batch, read back once the batch is done.
struct StageTimer {
    MapCtx* c;
    size_t used = 0;
    int cur = 0;
    cudaEvent_t a = nullptr;
    std::vector<std::tuple<int, cudaEvent_t, cudaEvent_t>> rec;
    explicit StageTimer(MapCtx* cc) : c(cc) {}
    cudaEvent_t get() {
        if (used < c->ev_pool.size()) return c->ev_pool[used++];
        cudaEvent_t e;
        SHM_CUDA(cudaEventCreate(&e));
        c->ev_pool.push_back(e);
        used++;
        return e;
    }
    // counts = the launch that follows is not counted by a helper of its own
    void begin(int st, bool counts = true) {
        if (counts) count_launch();
        if (!c->timing) return;
        cur = st;
        a = get();
        SHM_CUDA(cudaEventRecord(a, c->stream));
    }
    void end() {
        if (!c->timing) return;
        cudaEvent_t b = get();
        SHM_CUDA(cudaEventRecord(b, c->stream));
        rec.emplace_back(cur, a, b);
    }
    void collect() {  // after the stream is synchronized
        for (auto& r : rec) {
            float ms = 0;
            SHM_CUDA(cudaEventElapsedTime(&ms, std::get<1>(r), std::get<2>(r)));
            c->stage_ms[std::get<0>(r)] += ms;
            c->stage_calls[std::get<0>(r)] += 1;
        }
        rec.clear();
        used = 0;
    }
};

struct MapScratch {
    DevBuf<uint8_t> seqb[2];  // host-form batches: one mapped, the next arriving
    DevBuf<uint8_t> plan;  // BatchPlan's arrays on the device
    DevBuf<int32_t> seed_lists;  // N_SEED_BINS lists of n reads
    DevBuf<uint32_t> bin_cnt;
    DevBuf<uint8_t> retry_seq;  // reads mapped again with exact bounds
    DevBuf<shm_map_record> retry_out;
    DevBuf<int64_t> retry_list;
    DevBuf<int32_t> retry_idx;
    DevBuf<uint64_t> km_h, pht_key, hw, hw_off, bt_size, bt_off;
    DevBuf<SeedRec> sd;
    DevBuf<uint32_t> pk_codes[2], pk_mask[2];  // host-buffer batches, packed (host/pack.hpp)
    DevBuf<uint32_t> pk_list[2];               // their nonzero mask words as uploaded (index, word)
    DevBuf<uint32_t> dpk_codes, dpk_mask;      // device-resident batches, packed on the device
    DevBuf<uint64_t> sd_h;
    DevBuf<uint32_t> kcnt, km_rs, sd_hpre, pht_val, r_seeded, n_jobs, ccnt, coff, ccur,
        cidx, cfar, cfar_q, sort_scr, ovf_list, r_flags;
    DevBuf<uint32_t> lcs_pos, lcs_cnt;  // bucket_LCS only
    DevBuf<uint32_t> r_lead;
    DevBuf<int32_t> r_i32, ref_scr;
    DevBuf<int64_t> r_smatch;
    DevBuf<uint64_t> r_eb;
    DevBuf<BSlot> bt;
    DevBuf<uint32_t> bt_list, bt2_list;
    DevBuf<ulonglong2> bt_tab;
    DevBuf<uint64_t> bt2_off;
    DevBuf<BucketJob> jobs;
    DevBuf<BatchMax> mx;
    DevBuf<SweepCand> sweep_scr;
    DevBuf<uint8_t> seed_gscr;
    DevBuf<shm_map_record> out;
    SketchLuts* luts = nullptr;
    int32_t luts_k = -1;
    // rarity weights max(c, 1)^-alpha for one (index, alpha), and per-read m_weight
    DevBuf<double> wtab, r_mw;
    double wtab_alpha = 0.0;
    const IndexStorage* wtab_ix = nullptr;
    uint32_t wtab_n = 0;
};

static void free_stream_sink(StreamSink* u);  // (defined with StreamSink below)

MapCtx* mapctx_create(int device, size_t hbm_budget) {
    SHM_CUDA(cudaSetDevice(device));
    auto* c = new MapCtx();
    c->device = device;
    c->hbm_budget = hbm_budget;
    SHM_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    SHM_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    SHM_CUDA(cudaStreamCreateWithFlags(&c->side_stream, cudaStreamNonBlocking));
    SHM_CUDA(cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming));
    SHM_CUDA(cudaEventCreateWithFlags(&c->join, cudaEventDisableTiming));
    for (auto& e : c->copied) SHM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (auto& e : c->sketched) SHM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    SHM_CUDA(cudaStreamCreateWithFlags(&c->raw_stream, cudaStreamNonBlocking));
    for (auto& e : c->raw_copied) SHM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (auto& e : c->raw_sketched) SHM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    c->scr = new MapScratch();
    return c;
}

void mapctx_destroy(MapCtx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->scr) {
        if (c->scr->luts) cudaFree(c->scr->luts);
        delete c->scr;
    }
    paf_scratch_free(c->paf);
    if (c->h_pinned) cudaFreeHost(c->h_pinned);
    if (c->h_slots) cudaFreeHost(c->h_slots);
    if (c->h_pack) cudaFreeHost(c->h_pack);
    if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
    for (auto& e : c->copied)
        if (e) cudaEventDestroy(e);
    for (auto& e : c->sketched)
        if (e) cudaEventDestroy(e);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->raw_stream) {
        cudaStreamSynchronize(c->raw_stream);
        cudaStreamDestroy(c->raw_stream);
    }
    for (auto& e : c->raw_copied)
        if (e) cudaEventDestroy(e);
    for (auto& e : c->raw_sketched)
        if (e) cudaEventDestroy(e);
    for (auto& e : c->up_ev) cudaEventDestroy(e);
    free_stream_sink(c->sink);
    if (c->side_stream) {
        cudaStreamSynchronize(c->side_stream);
        cudaStreamDestroy(c->side_stream);
    }
    if (c->fork) cudaEventDestroy(c->fork);
    if (c->join) cudaEventDestroy(c->join);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

static uint64_t pow2_host(uint64_t x) {  // smallest power of two >= x (1 for x <= 1)
    return x <= 1 ? 1 : (uint64_t)1 << (64 - __builtin_clzll(x - 1));
}

// k-mer capacity of a read of nw windows: the reference's own estimate
// mean + 6 sigma + 16 (src/sketch.rs:143-146), raised to twice the mean + 16.
// The binomial estimate holds for unique sequence, but a read from a tandem
// array selects each of its few k-mers once per copy: on human-like
// references about 0.2% of long reads reach 1.5-2x the mean. Reads that beat
// the capacity are retried with the count the first pass found.
static uint64_t kmer_cap(int64_t nw, double h_frac) {
    if (nw <= 0) return 0;
    if (h_frac >= 1.0) return (uint64_t)nw;
    double mean = std::max(0.0, (double)nw * h_frac);
    uint64_t c = std::max((uint64_t)(mean + 6.0 * std::sqrt(mean)), (uint64_t)(2.0 * mean)) + 16;
    return std::min<uint64_t>(c, (uint64_t)nw);
}

// A batch's per-read plan, written by the host straight into pinned memory
// and sent up in one copy: offsets of the reads, of their sketch runs, of
// their k-mer capacities and of their probe tables.
struct BatchPlan {
    int64_t* roff;         // n+1
    uint64_t* chunk_off;   // n+1
    uint64_t* kcap_off;    // n+1
    uint64_t* pht_off;     // n+1
    uint32_t n_cap_512 = 0, n_cap_1024 = 0, n_cap_4096 = 0;  // reads whose capacity exceeds 512 / 1024 / 4096
    uint32_t P_g = 0;                          // power of two >= every capacity above 4096
    uint64_t max_cap = 0;                      // largest k-mer capacity of a read
    int64_t max_len = 0;                       // longest read
    size_t bytes = 0;
    static size_t layout(int32_t n) { return 4 * ((size_t)n + 1) * 8; }
    void carve(uint8_t* base, int32_t n) {
        const size_t a = ((size_t)n + 1) * 8;
        bytes = layout(n);
        roff = (int64_t*)base;
        chunk_off = (uint64_t*)(base + a);
        kcap_off = (uint64_t*)(base + 2 * a);
        pht_off = (uint64_t*)(base + 3 * a);
    }
};

// Grow-only pinned host staging of a context (the plan of the batch in flight).
static uint8_t* pinned_stage(MapCtx* c, size_t bytes) {
    if (bytes > c->h_pinned_cap) {
        if (c->h_pinned) SHM_CUDA(cudaFreeHost(c->h_pinned));
        c->h_pinned = nullptr;
        c->h_pinned_cap = 0;
        const size_t want = std::max<size_t>(bytes + bytes / 4, (size_t)1 << 20);
        SHM_CUDA(cudaHostAlloc((void**)&c->h_pinned, want, cudaHostAllocDefault));
        c->h_pinned_cap = want;
    }
    return c->h_pinned;
}

// Written into pinned memory at h_plan (BatchPlan::layout(n) bytes). caps =
// null: capacities from the estimate; else caps[i] k-mers for read i (the
// counts a previous pass found).
// words [0, n) of src (device-accessible, e.g. a mapped pinned block) to dst.
__global__ void k_copy_words(uint32_t* __restrict__ dst, const uint32_t* __restrict__ src, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

// roff starts at base0: the batch's first base in the buffer its sketch reads
// (only differences of roff are read elsewhere).
static void plan_batch(uint8_t* h_plan, const int64_t* h_offs, int32_t n, int32_t k, double h_frac,
                       const uint32_t* caps, BatchPlan& bp, int64_t base0 = 0) {
    bp.carve(h_plan, n);
    bp.P_g = 0;
    bp.max_cap = 0;
    bp.max_len = 0;
    bp.n_cap_512 = bp.n_cap_1024 = bp.n_cap_4096 = 0;
    bp.roff[0] = base0;
    bp.chunk_off[0] = 0;
    bp.kcap_off[0] = 0;
    bp.pht_off[0] = 0;
    for (int32_t i = 0; i < n; i++) {
        const int64_t L = h_offs[i + 1] - h_offs[i];
        bp.roff[i + 1] = bp.roff[i] + L;
        const int64_t nw = L - k + 1;
        bp.chunk_off[i + 1] = bp.chunk_off[i] + (nw > 0 ? (uint64_t)((nw + SKETCH_WIN - 1) / SKETCH_WIN) : 0);
        const uint64_t cap = caps ? (uint64_t)caps[i] : kmer_cap(nw, h_frac);
        bp.kcap_off[i + 1] = bp.kcap_off[i] + cap;
        bp.max_cap = std::max(bp.max_cap, cap);
        bp.max_len = std::max(bp.max_len, L);
        bp.pht_off[i + 1] = bp.pht_off[i] + std::max<uint64_t>(16, pow2_host(2 * cap));
        if (cap > 512) bp.n_cap_512++;
        if (cap > 1024) bp.n_cap_1024++;
        if (cap > 4096) {
            bp.n_cap_4096++;
            bp.P_g = std::max<uint32_t>(bp.P_g, (uint32_t)pow2_host(cap));
        }
    }
}

// A read that overflowed a capacity, with its sketch size.
struct Overflow {
    int32_t read;
    uint32_t m;   // its counted k-mers (the capacity it is mapped again with)
    uint64_t eb;  // the bound on its distinct buckets (0: its seeds were not prepared)
};

// Where a batch's results land on the host (pinned): the small reads, then
// its overflow list (up to n pairs read, m).
struct BatchSlot {
    HostReads* R;
    uint32_t* ovf;
    int32_t i0, n;
    int64_t bases;
    uint32_t job_cap;  // set by run_batch: more jobs than this and the batch is mapped again
};

// The bucket tables of a batch mapped without waiting for its sizes get at
// most bt_fast_slots slots a read (twice the bound on the read's distinct
// buckets, as in exact sizing, when that is less), laid out in read order in
// a pool of that many slots a read; a read whose table fills up gets a second table from
// spare slots after the pool (k_bt_second), and is mapped again by the host
// only when that fills up too or finds no room. A batch has at most 64
// bucket jobs a read on average (a batch with more is mapped again). The
// environment variables SHMAP_BT_FAST_SLOTS (the pool and per-read limit, a
// power of two >= 16), SHMAP_BT_FAST_READ (a larger per-read limit, so that
// tables can run past the pool), SHMAP_BT_SPARE_SLOTS and SHMAP_FAST_JOB_CAP
// lower them, so that tests reach every fallback.
static uint64_t env_pow2(const char* name, uint64_t lo, uint64_t hi) {
    const char* e = std::getenv(name);
    const uint64_t v = e ? std::strtoull(e, nullptr, 10) : 0;
    return (v >= lo && (v & (v - 1)) == 0 && v <= hi) ? v : 0;
}
static uint64_t fast_bt_slots() {
    const uint64_t v = env_pow2("SHMAP_BT_FAST_SLOTS", 16, 512);
    if (v) return v;
    const uint64_t t = (uint64_t)tuning().bt_fast_slots;  // a power of two in [16, 512] (rounded down)
    return (uint64_t)1 << (63 - __builtin_clzll(t));
}
static uint64_t fast_bt_read_cap() {
    const uint64_t r = env_pow2("SHMAP_BT_FAST_READ", 16, 4096);
    return r ? r : fast_bt_slots();
}
// Spare slots for second tables: 1,024 a read and a million more, room for
// a full-size second table for a quarter of a batch (at r = 0.10 a fifth of
// the reads, those from satellite arrays, fill their first table); the spare
// is only written where a second table is handed out
// (SHMAP_BT_SPARE_SLOTS sets the number; 0 turns second tables off).
static uint64_t bt_spare_slots(int32_t n) {
    const char* e = std::getenv("SHMAP_BT_SPARE_SLOTS");
    if (e) return std::strtoull(e, nullptr, 10);
    return 1024 * (uint64_t)n + ((uint64_t)1 << 20);
}
static uint32_t fast_job_cap(int32_t n) {
    const char* e = std::getenv("SHMAP_FAST_JOB_CAP");
    const uint64_t v = e ? std::strtoull(e, nullptr, 10) : 0;
    const uint64_t cap = std::min<uint64_t>(std::max<uint64_t>(fast_bt_slots(), 512) * (uint64_t)n + 1,
                                            64 * (uint64_t)n + (1u << 20));
    return (uint32_t)(v >= 1 ? std::min(v, cap) : cap);
}

// Pinned per-call result slots for batches of the given sizes.
static std::vector<BatchSlot> batch_slots(MapCtx* c, const std::vector<std::pair<int32_t, int32_t>>& b,
                                          const int64_t* offs) {
    size_t bytes = 0;
    for (auto [i, j] : b) bytes += (sizeof(HostReads) + 63) / 64 * 64 + (16 * (size_t)(j - i) + 63) / 64 * 64;
    if (bytes > c->h_slots_cap) {
        if (c->h_slots) SHM_CUDA(cudaFreeHost(c->h_slots));
        c->h_slots = nullptr;
        c->h_slots_cap = 0;
        const size_t want = std::max<size_t>(bytes + bytes / 4, (size_t)1 << 16);
        SHM_CUDA(cudaHostAlloc(&c->h_slots, want, cudaHostAllocDefault));
        c->h_slots_cap = want;
    }
    std::vector<BatchSlot> out;
    uint8_t* at = (uint8_t*)c->h_slots;
    for (auto [i, j] : b) {
        BatchSlot sl;
        sl.R = (HostReads*)at;
        at += (sizeof(HostReads) + 63) / 64 * 64;
        sl.ovf = (uint32_t*)at;
        at += (16 * (size_t)(j - i) + 63) / 64 * 64;
        sl.i0 = i;
        sl.n = j - i;
        sl.bases = offs[j] - offs[i];
        out.push_back(sl);
    }
    return out;
}

// After the stream has drained: a batch's work counters and its overflowed
// reads (indices offset by the batch's first read), appended to `ovf`.
static void collect_batch(MapCtx* c, const BatchSlot& sl, std::vector<Overflow>& ovf) {
    const HostReads& R = *sl.R;
    const BatchMax& fin = R.fin;
    c->work[W_READS] += sl.n;
    c->work[W_BASES] += sl.bases;
    c->work[W_KMERS] += (int64_t)fin.kmers;
    c->work[W_DISTINCT] += (int64_t)fin.distinct;
    c->work[W_PROC_SEEDS] += (int64_t)fin.proc_seeds;
    c->work[W_HITS] += (int64_t)fin.hits;
    c->work[W_BUCKETS] += (int64_t)fin.buckets;
    c->work[W_JOBS] += R.nj;
    c->work[W_EXT_SEEDS] += (int64_t)fin.ext_seeds;
    c->work[W_CANDS] += R.nc;
    c->work[W_REFINE_KMERS] += (int64_t)fin.refine_kmers;
    c->work[W_REFINED] += (int64_t)fin.refined;
    c->work[W_BT2_READS] += (int64_t)fin.bt2_n;
    const size_t at = ovf.size();
    for (uint32_t i = 0; i < fin.n_overflow && i < (uint32_t)sl.n; i++)
        ovf.push_back(Overflow{sl.i0 + (int32_t)sl.ovf[4 * i], sl.ovf[4 * i + 1],
                               (uint64_t)sl.ovf[4 * i + 2] | ((uint64_t)sl.ovf[4 * i + 3] << 32)});
    std::sort(ovf.begin() + at, ovf.end(), [](const Overflow& x, const Overflow& y) { return x.read < y.read; });
}

// Enqueues the mapping of one batch whose bytes are already on the device at
// d_seq (relative offsets h_offs[i] - h_offs[0]), or packed (pk_codes,
// pk_mask: host/pack.hpp) when those are set; caps as for plan_batch.
// The host waits once, for the sizes of the bucket tables; everything after
// is queued, and the batch's results reach `sl` when the stream drains
// (collect_batch then lists the reads that overflowed a capacity).
// exact: sizes are read back as the batch goes (tables of at most bt_lim
// slots a read, 0 = no limit; the bucket jobs counted before they are
// allocated), which costs two synchronizations; else host-known caps, with
// the batch mapped again when its jobs exceed them.
static void run_batch(MapCtx* c, const IndexStorage* ix, const shm_params& p, const uint8_t* d_seq,
                      const int64_t* h_offs, int32_t n, shm_map_record* d_out, const uint32_t* caps, bool exact,
                      uint8_t* h_plan, StageTimer& T, BatchSlot& sl, const uint32_t* pk_codes = nullptr,
                      const uint32_t* pk_mask = nullptr, uint64_t bt_lim = 0, int32_t pk_base = 0,
                      uint64_t pk_words = 0) {
    cudaStream_t s = c->stream;
    MapScratch& S = *c->scr;
    HostClock H;
    BatchPlan bp;
    // packed reads: the batch's first base is base pk_base (0..31) of pk_codes
    // / pk_mask, and pk_words code words are readable there (0: the batch's own)
    plan_batch(h_plan, h_offs, n, p.k, p.h_frac, caps, bp, pk_codes ? pk_base : 0);
    H.mark("plan");
    if (!S.luts || S.luts_k != p.k) {
        if (S.luts) SHM_CUDA(cudaFree(S.luts));
        S.luts = create_device_luts(p.k, s);
        S.luts_k = p.k;
    }
    const uint64_t kcap = bp.kcap_off[(size_t)n], phtn = bp.pht_off[(size_t)n];
    // the plan goes up in one copy from its own pinned block, by the copy
    // engine, or (plan_mapped) by a kernel reading the block through its
    // device mapping: then it does not queue behind the other host-to-device
    // copies of the copy engine (the packing threads' pieces)
    S.plan.reserve(bp.bytes + 64);
    void* d_src = nullptr;
    if (tuning().plan_mapped && cudaHostGetDevicePointer(&d_src, h_plan, 0) == cudaSuccess) {
        const size_t words = (bp.bytes + 3) / 4;  // the block is padded to 64 bytes
        k_copy_words<<<grid_for(words, 256, 4), 256, 0, s>>>((uint32_t*)S.plan.p, (const uint32_t*)d_src, words);
        SHM_CUDA(cudaGetLastError());
        count_launch();
        c->work[W_H2D_BYTES] += (int64_t)bp.bytes;
    } else {
        cudaGetLastError();
        copy_async(c, S.plan.p, h_plan, bp.bytes, cudaMemcpyHostToDevice, s);
    }
    BatchPlan dp;
    dp.carve(S.plan.p, n);
    S.kcnt.reserve((size_t)n);
    S.km_h.reserve(kcap + 1);
    S.km_rs.reserve(kcap + 1);
    S.sd.reserve(kcap + 1);
    S.sd_h.reserve(kcap + 1);
    S.sd_hpre.reserve(kcap + 1);
    S.pht_key.reserve(phtn);
    S.pht_val.reserve(phtn);
    S.r_i32.reserve((size_t)n * 8);
    S.r_smatch.reserve((size_t)n);
    S.r_seeded.reserve((size_t)n);
    S.r_flags.reserve((size_t)n);
    S.hw.reserve((size_t)n);
    S.hw_off.reserve((size_t)n + 1);
    S.bt_size.reserve((size_t)n);
    S.bt_off.reserve((size_t)n + 1);
    S.ccnt.reserve((size_t)n);
    S.coff.reserve((size_t)n + 1);
    S.ccur.reserve((size_t)n);
    S.ovf_list.reserve(4 * (size_t)n);
    S.r_eb.reserve((size_t)n);
    S.n_jobs.reserve(1);
    S.mx.reserve(1);
    SHM_CUDA(cudaMemsetAsync(S.kcnt.p, 0, sizeof(uint32_t) * (size_t)n, s));
    SHM_CUDA(cudaMemsetAsync(S.r_seeded.p, 0, sizeof(uint32_t) * (size_t)n, s));
    SHM_CUDA(cudaMemsetAsync(S.r_flags.p, 0, sizeof(uint32_t) * (size_t)n, s));
    SHM_CUDA(cudaMemsetAsync(S.r_eb.p, 0, sizeof(uint64_t) * (size_t)n, s));
    SHM_CUDA(cudaMemsetAsync(S.ccnt.p, 0, sizeof(uint32_t) * (size_t)n, s));
    SHM_CUDA(cudaMemsetAsync(S.ccur.p, 0, sizeof(uint32_t) * (size_t)n, s));
    SHM_CUDA(cudaMemsetAsync(S.n_jobs.p, 0, sizeof(uint32_t), s));
    SHM_CUDA(cudaMemsetAsync(S.mx.p, 0, sizeof(BatchMax), s));
    SHM_CUDA(cudaMemsetAsync(S.r_i32.p, 0, sizeof(int32_t) * (size_t)n * 8, s));
    SHM_CUDA(cudaMemsetAsync(S.hw.p, 0, sizeof(uint64_t) * (size_t)n, s));
    SHM_CUDA(cudaMemsetAsync(S.bt_size.p, 0, sizeof(uint64_t) * (size_t)n, s));
    H.mark("upload");

    BatchView v{};
    v.n = n;
    v.I = ix->dev;
    v.P.k = p.k;
    v.P.thr = ix->dev.thr;
    v.P.theta = p.theta;
    v.P.min_diff = p.min_diff;
    v.P.max_overlap = p.max_overlap;
    v.P.theta_low = p.theta * (1.0 - p.min_diff);
    v.P.metric = p.metric;
    v.P.nbp = p.no_bucket_pruning;
    v.P.os = p.one_sweep;
    v.P.ap = p.abs_pos;
    {
        // rarity (src/shmap/mod.rs:694-723): alpha follows --rarity-alpha, else
        // --rarity-weight, else 1 when only the tie-break is on
        const double alpha = p.rarity_alpha > 0.0    ? p.rarity_alpha
                             : p.rarity_weight > 0.0 ? p.rarity_weight
                             : p.rarity_tiebreak > 0.0 ? 1.0
                                                       : 0.0;
        v.P.tiebreak = p.rarity_tiebreak > 0.0 ? p.rarity_tiebreak : 0.0;
        v.P.rarity = alpha > 0.0 && p.metric <= SHM_JACCARD;  // the bucket metrics report no support
        v.P.rw_score = v.P.rarity && p.rarity_weight > 0.0;
        if (v.P.rarity) {
            // a seed's hit count is at most the longest hit list of the index
            const uint32_t n_w = ix->max_list + 1;
            if (S.wtab_ix != ix || S.wtab_alpha != alpha || S.wtab_n != n_w) {
                std::vector<double> w(n_w);
                for (uint32_t c2 = 0; c2 < n_w; c2++) w[c2] = std::pow((double)std::max<uint32_t>(c2, 1u), -alpha);
                S.wtab.reserve(n_w);
                SHM_CUDA(cudaMemcpy(S.wtab.p, w.data(), sizeof(double) * n_w, cudaMemcpyHostToDevice));
                S.wtab_ix = ix;
                S.wtab_alpha = alpha;
                S.wtab_n = n_w;
            }
            v.P.wtab = S.wtab.p;
            v.P.wtab_n = n_w;
        }
        if (v.P.tiebreak > 0.0) {
            // the band admits scores below thr: pass 2's threshold can go down to
            // fl(fl(theta - fl(band * theta)) * fl(1 - d)), so candidates reach that low
            const double adm = p.theta - v.P.tiebreak * std::fabs(p.theta);
            v.P.theta_low = std::min(v.P.theta_low, adm * (1.0 - p.min_diff));
        }
    }
    for (int b = 0; b < 16; b++) {
        const unsigned __int128 num = (unsigned __int128)1 << (64 + b);
        const unsigned __int128 den = (unsigned __int128)ix->dev.thr + 1;
        const unsigned __int128 q128 = num / den;
        v.P.slot_mul[b] = q128 > (unsigned __int128)UINT64_MAX ? UINT64_MAX : (uint64_t)q128;
    }
    v.theta2 = p.theta - p.min_diff;
    v.seq = d_seq;
    v.roff = dp.roff;
    v.kcap_off = dp.kcap_off;
    v.kcnt = S.kcnt.p;
    v.km_h = S.km_h.p;
    v.km_rs = S.km_rs.p;
    v.sd = S.sd.p;
    v.sd_h = S.sd_h.p;
    v.sd_hpre = S.sd_hpre.p;
    v.pht_off = dp.pht_off;
    v.pht_key = S.pht_key.p;
    v.pht_val = S.pht_val.p;
    int32_t* ri = S.r_i32.p;
    v.r_status = ri;
    v.r_m = ri + n;
    v.r_nu = ri + 2 * (size_t)n;
    v.r_nproc = ri + 3 * (size_t)n;
    v.r_S = ri + 4 * (size_t)n;
    v.r_S0 = ri + 5 * (size_t)n;
    v.r_half = ri + 6 * (size_t)n;
    v.r_maxseed = ri + 7 * (size_t)n;
    v.r_smatch = S.r_smatch.p;
    v.r_seeded = S.r_seeded.p;
    v.r_flags = S.r_flags.p;
    // synchronous sizing: tables of at most bt_lim slots a read (0: the full bound);
    // queued sizing: at most fast_bt_read_cap() a read, from a pool of fast_bt_slots() a read
    v.bt_cap = exact ? (bt_lim ? bt_lim : ((uint64_t)1 << 62)) : fast_bt_read_cap();
    v.r_eb = S.r_eb.p;
    v.ext_total = p.abs_pos ? (uint64_t)ix->stats.total_nucls : (uint64_t)ix->dev.n_kmers;
    v.hw = S.hw.p;
    v.hw_off = S.hw_off.p;
    v.bt_size = S.bt_size.p;
    v.bt_off = S.bt_off.p;
    v.n_jobs = S.n_jobs.p;
    v.ccnt = S.ccnt.p;
    v.coff = S.coff.p;
    v.ccur = S.ccur.p;
    v.ovf_list = S.ovf_list.p;
    v.mx = S.mx.p;
    v.out = d_out;

    // K1
    SketchArgs a{};
    a.seq = d_seq;
    a.seq_off = dp.roff;
    a.chunk_off = dp.chunk_off;
    a.n_seq = n;
    a.n_chunks = bp.chunk_off[(size_t)n];
    a.k = p.k;
    a.thr = ix->dev.thr;
    a.r_offset = 0;
    a.kmer_off = dp.kcap_off;
    a.kmer_cnt = S.kcnt.p;
    a.out_h = S.km_h.p;
    a.out_rs = S.km_rs.p;
    const int64_t batch_bytes = h_offs[n] - h_offs[0];
    static const bool letters = std::getenv("SHMAP_SKETCH_LETTERS") != nullptr;
    if (!pk_codes && d_seq && !letters && tuning().device_pack) {  // reads in device memory packed there first
        S.dpk_codes.reserve(packed_code_words(batch_bytes));
        S.dpk_mask.reserve(packed_mask_words(batch_bytes));
        T.begin(STG_SKETCH, false);
        pack_reads_device(d_seq, batch_bytes, S.dpk_codes.p, S.dpk_mask.p, s);
        T.end();
        pk_codes = S.dpk_codes.p;
        pk_mask = S.dpk_mask.p;
    }
    a.pk_codes = pk_codes;  // packed reads instead of d_seq when set
    a.pk_mask = pk_mask;
    a.pk_words = pk_codes ? (pk_words ? pk_words : packed_code_words(batch_bytes)) : 0;
    T.begin(STG_SKETCH, false);
    launch_sketch(SK_APPEND, a, S.luts, s);
    T.end();
    if (c->sketch_done) SHM_CUDA(cudaEventRecord(c->sketch_done, s));  // the batch's bytes are free again

    // K2: bins by the actual sketch sizes, then one launch per bin (each
    // reads its own count on the device; empty bins return at once)
    S.bin_cnt.reserve(N_SEED_BINS);
    S.seed_lists.reserve((size_t)N_SEED_BINS * (size_t)n);
    SHM_CUDA(cudaMemsetAsync(S.bin_cnt.p, 0, sizeof(uint32_t) * N_SEED_BINS, s));
    const int32_t* LB = S.seed_lists.p;
    const uint32_t* NB = S.bin_cnt.p;
    T.begin(STG_SEEDPREP);  // one span: bins, the side stream's large bins, the join
    k_seed_bins<<<grid_for((size_t)n, 256, 8), 256, 0, s>>>(v, S.seed_lists.p, S.bin_cnt.p);
    SHM_CUDA(cudaGetLastError());
    // the few reads with large sketches go on the side stream, so that their
    // long per-read latency overlaps the bulk of the reads on the main stream
    // (a read of bin b has capacity >= m, which bounds each bin's size on the host)
    const bool side = bp.n_cap_512 > 0;
    if (side) {
        SHM_CUDA(cudaEventRecord(c->fork, s));
        SHM_CUDA(cudaStreamWaitEvent(c->side_stream, c->fork, 0));
    }
    cudaStream_t s2 = c->side_stream;
    if (bp.P_g) {  // m > 4096: CTA per read, global scratch
        const size_t bytes = SEED_BYTES_PER_ELEM * bp.P_g;
        const int grid = (int)std::min<size_t>(bp.n_cap_4096, 296);
        S.seed_gscr.reserve(bytes * (size_t)grid);
        k_seedprep<true><<<grid, 256, 0, s2>>>(v, LB + 4 * (size_t)n, NB + 4, bp.P_g, S.seed_gscr.p, bytes);
        SHM_CUDA(cudaGetLastError());
        count_launch();
    }
    if (bp.n_cap_1024) {  // 1024 < m <= 4096: CTA per read
        const uint32_t P = 4096;
        const size_t bytes = SEED_BYTES_PER_ELEM * P;
        if ((int)bytes > c->seed_smem_set) {
            SHM_CUDA(cudaFuncSetAttribute(k_seedprep<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
            c->seed_smem_set = (int)bytes;
        }
        k_seedprep<false><<<grid_for((size_t)bp.n_cap_1024 * SEEDP_THREADS, SEEDP_THREADS, 2), SEEDP_THREADS, bytes,
                            s2>>>(v, LB + 3 * (size_t)n,
                                                                                               NB + 3, P, nullptr, 0);
        SHM_CUDA(cudaGetLastError());
        count_launch();
    }
    const size_t sgb = seedc_seg_bytes(v.I.n_seg);
    if (!c->seedc_smem_set) {
        const int sg = (int)seedc_seg_bytes(SEEDC_SEGS);
        SHM_CUDA(cudaFuncSetAttribute(k_seedprep_c<256, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(8 * seedc_bytes(256)) + sg));
        SHM_CUDA(cudaFuncSetAttribute(k_seedprep_c<512, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(4 * seedc_bytes(512)) + sg));
        SHM_CUDA(cudaFuncSetAttribute(k_seedprep_c<1024, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(4 * seedc_bytes(1024)) + sg));
        c->seedc_smem_set = 1;
    }
    if (bp.n_cap_512) {  // 512 < m <= 1024
        k_seedprep_c<1024, 4><<<grid_for((size_t)bp.n_cap_512 * 32, 128, 1), 128, 4 * seedc_bytes(1024) + sgb, s2>>>(
            v, LB + 2 * (size_t)n, NB + 2);
        SHM_CUDA(cudaGetLastError());
        count_launch();
    }
    if (side) SHM_CUDA(cudaEventRecord(c->join, s2));
    {
        k_seedprep_c<256, 8><<<grid_for((size_t)n * 32, 256, 4), 256, 8 * seedc_bytes(256) + sgb, s>>>(v, LB, NB);
        SHM_CUDA(cudaGetLastError());
        count_launch();
        k_seedprep_c<512, 4><<<grid_for((size_t)n * 32, 128, 4), 128, 4 * seedc_bytes(512) + sgb, s>>>(v, LB + n,
                                                                                                      NB + 1);
        SHM_CUDA(cudaGetLastError());
        count_launch();
    }
    if (side) SHM_CUDA(cudaStreamWaitEvent(s, c->join, 0));
    T.end();

    exclusive_scan_u64(S.hw.p, S.hw_off.p, (size_t)n, s);
    exclusive_scan_u64(S.bt_size.p, S.bt_off.p, (size_t)n, s);
    HostReads& R = *sl.R;
    const bool debug = std::getenv("SHMAP_DEBUG") != nullptr;
    // Sizes after seeding. Exact mode: wait for the bucket tables' total and
    // the batch maxima. Otherwise bounds the host knows: capped tables, the
    // largest capacity and read.
    uint64_t bt_slots_alloc;
    uint32_t job_cap, m_max, nu_max, half_max;
    if (exact || debug) {
        copy_async(c, &R.totals[0], S.hw_off.p + n, sizeof(uint64_t), cudaMemcpyDeviceToHost, s);
        copy_async(c, &R.totals[1], S.bt_off.p + n, sizeof(uint64_t), cudaMemcpyDeviceToHost, s);
        copy_async(c, &R.hm, S.mx.p, sizeof(BatchMax), cudaMemcpyDeviceToHost, s);
        H.mark("enq1");
        SHM_CUDA(cudaStreamSynchronize(s));
        H.mark("sync1");
        if (debug) {
            std::fprintf(stderr,
                         "[shmap] batch n=%d kcap=%llu hw_total=%llu bt_total=%llu m_max=%u nu_max=%u half_max=%u\n", n,
                         (unsigned long long)kcap, (unsigned long long)R.totals[0], (unsigned long long)R.totals[1],
                         R.hm.m_max, R.hm.nu_max, R.hm.half_max);
            if (n <= 8) {
                std::vector<int32_t> ri((size_t)n * 8);
                std::vector<uint32_t> kc((size_t)n);
                std::vector<uint64_t> hw((size_t)n), bs((size_t)n);
                SHM_CUDA(cudaMemcpy(ri.data(), S.r_i32.p, sizeof(int32_t) * ri.size(), cudaMemcpyDeviceToHost));
                SHM_CUDA(cudaMemcpy(kc.data(), S.kcnt.p, sizeof(uint32_t) * kc.size(), cudaMemcpyDeviceToHost));
                SHM_CUDA(cudaMemcpy(hw.data(), S.hw.p, sizeof(uint64_t) * hw.size(), cudaMemcpyDeviceToHost));
                SHM_CUDA(cudaMemcpy(bs.data(), S.bt_size.p, sizeof(uint64_t) * bs.size(), cudaMemcpyDeviceToHost));
                for (int32_t q = 0; q < n; q++)
                    std::fprintf(stderr,
                                 "[shmap]  read %d kcnt=%u status=%d m=%d nu=%d nproc=%d S=%d S0=%d half=%d maxseed=%d "
                                 "hw=%llu bt=%llu\n",
                                 q, kc[q], ri[q], ri[n + q], ri[2 * n + q], ri[3 * n + q], ri[4 * n + q], ri[5 * n + q],
                                 ri[6 * n + q], ri[7 * n + q], (unsigned long long)hw[q], (unsigned long long)bs[q]);
            }
        }
    }
    if (exact) {
        bt_slots_alloc = R.totals[1];
        job_cap = 0;  // counted after the contributions: a job per distinct bucket at most
        m_max = R.hm.m_max;
        nu_max = R.hm.nu_max;
        half_max = R.hm.half_max;
    } else {
        bt_slots_alloc = fast_bt_slots() * (uint64_t)n;
        job_cap = fast_job_cap(n);
        m_max = nu_max = (uint32_t)bp.max_cap;  // m <= capacity, distinct seeds <= m
        half_max = p.abs_pos ? (uint32_t)bp.max_len : (uint32_t)bp.max_cap;
    }
    sl.job_cap = job_cap;
    const Tuning tu = tuning();
    // a full grid for kernels that read their counts on the device
    const int wide = grid_for((size_t)1 << 40, 256, (int)tu.wide_ctas_per_sm);

    H.mark("sizes");
    // spare slots after the pool for second tables (queued sizing only)
    const uint64_t spare = exact ? 0 : bt_spare_slots(n);
    S.bt.reserve(bt_slots_alloc + spare + 1);
    S.bt_list.reserve(bt_slots_alloc + spare + 1);
    S.bt_tab.reserve((size_t)n);
    S.bt2_list.reserve((size_t)n);
    S.bt2_off.reserve((size_t)n + 1);
    H.mark("bt_res");
    v.bt = S.bt.p;
    v.bt_list = S.bt_list.p;
    v.bt_tab = S.bt_tab.p;
    v.bt2_list = S.bt2_list.p;
    v.bt2_off = S.bt2_off.p;
    v.bt_pool = bt_slots_alloc;
    v.bt2_spare = spare;
    T.begin(STG_AUX);
    k_bt_init<<<wide, 256, 0, s>>>(S.bt.p, S.bt_off.p, n, bt_slots_alloc, S.r_flags.p, S.bt_tab.p);
    SHM_CUDA(cudaGetLastError());
    T.end();
    T.begin(STG_CONTRIB);
    k_contrib<<<wide, 256, 0, s>>>(v);
    SHM_CUDA(cudaGetLastError());
    T.end();
    if (spare) {  // reads whose table filled up: a second table and their contributions again
        T.begin(STG_CONTRIB);
        k_bt_second<<<wide, 256, 0, s>>>(v);
        SHM_CUDA(cudaGetLastError());
        T.end();
        T.begin(STG_CONTRIB);
        k_bt2_scan<<<1, 1024, 0, s>>>(v);
        SHM_CUDA(cudaGetLastError());
        T.end();
        T.begin(STG_CONTRIB);
        k_contrib2<<<wide, 256, 0, s>>>(v);
        SHM_CUDA(cudaGetLastError());
        T.end();
    }
    H.mark("contrib");
    if (exact) {  // the distinct buckets of every read, counted: they bound the jobs
        S.sort_scr.reserve((size_t)n + 1);
        exclusive_scan_u32(S.r_seeded.p, S.sort_scr.p, (size_t)n, s);
        copy_async(c, &R.nbk, S.sort_scr.p + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
        SHM_CUDA(cudaStreamSynchronize(s));
        job_cap = R.nbk + 1;
        sl.job_cap = job_cap;
    }
    S.jobs.reserve(job_cap);
    H.mark("jobs_res");
    v.jobs = S.jobs.p;
    v.job_cap = job_cap;
    T.begin(STG_BSCAN);
    k_bscan<<<grid_for((size_t)n * 32, 256, 8), 256, 0, s>>>(v);
    SHM_CUDA(cudaGetLastError());
    T.end();
    if (!p.no_bucket_pruning) {
        T.begin(STG_EXTEND);
        k_extend<<<wide, 256, 0, s>>>(v);
        SHM_CUDA(cudaGetLastError());
        T.end();
    }
    H.mark("extend");
    exclusive_scan_u32(S.ccnt.p, S.coff.p, (size_t)n, s);
    H.mark("scan");
    S.cidx.reserve((size_t)job_cap + 1);
    S.cfar.reserve((size_t)job_cap + 1);
    S.sweep_scr.reserve(2 * (size_t)job_cap + 2);
    H.mark("cidx_res");
    v.cidx = S.cidx.p;
    v.cfar = S.cfar.p;
    S.cfar_q.reserve((size_t)job_cap + 1);
    v.cfar_q = S.cfar_q.p;
    // two refinement passes (the reads' leads, then the candidates that can
    // still be scored) where the sweep's thresholds bound what it scores
    // (Containment only: a Jaccard score sits well below the sh of its bucket,
    // so its bound prunes little and the second pass only adds a tail)
    v.lead_on = p.metric == SHM_CONTAINMENT && !p.no_bucket_pruning && !v.P.rarity;
    S.r_lead.reserve((size_t)n);
    v.r_lead = S.r_lead.p;
    T.begin(STG_AUX);
    k_cidx<<<wide, 256, 0, s>>>(v);
    SHM_CUDA(cudaGetLastError());
    k_far_bins<<<wide, 256, 0, s>>>(v);
    SHM_CUDA(cudaGetLastError());
    count_launch();
    if (v.lead_on) {
        k_lead<<<grid_for((size_t)n * 32, 256, 8), 256, 0, s>>>(v);
        SHM_CUDA(cudaGetLastError());
        count_launch();
    }
    T.end();

    RefScratch rsc{};
    rsc.nu_max = nu_max + 1;
    rsc.wmax = 2 * half_max + 2;
    rsc.ring_n = m_max + 1;
    rsc.per_warp = (size_t)rsc.nu_max + 2 * ((size_t)rsc.wmax + 1) + (size_t)m_max + 1;
    if (v.P.rarity) {  // + nxt, flag, and the f64 weights at an even offset (every warp base 8-byte aligned)
        rsc.wt_at = (rsc.per_warp + 2 * ((size_t)rsc.wmax + 1) + 1) & ~(size_t)1;
        rsc.per_warp = rsc.wt_at + 2 * ((size_t)rsc.wmax + 1);
    }
    size_t warps = (size_t)grid_for((size_t)1 << 40, 1, (int)tu.refine_warps_per_sm);  // SMs x warps per SM
    const size_t budget_ints = (size_t)1 << 28;  // 1 GiB of refinement scratch at most
    while (warps >= 16 && warps * rsc.per_warp > budget_ints) warps /= 2;  // stays >= 8: a block's worth
    S.ref_scr.reserve(warps * rsc.per_warp);
    H.mark("ref_res");
    rsc.base = S.ref_scr.p;
    T.begin(STG_REFINE);
    if (p.metric == SHM_BUCKET_LCS) {
        S.lcs_pos.reserve(kcap + 1);
        S.lcs_cnt.reserve(kcap + 1);
        v.lcs_pos = S.lcs_pos.p;
        k_lcs_occ<<<grid_for((size_t)n * 256, 256, 8), 256, 0, s>>>(v, S.lcs_pos.p, S.lcs_cnt.p);
        SHM_CUDA(cudaGetLastError());
        count_launch();
    }
    if (!c->rchip_smem_set) {
        SHM_CUDA(cudaFuncSetAttribute(k_refine_chip, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(RCHIP_WARPS * RCHIP_SLICE)));
        c->rchip_smem_set = 1;
    }
    if (p.metric == SHM_BUCKET_LCS) {  // no read is refined on chip under the bucket metrics
        k_refine_lcs<<<(unsigned)std::max<size_t>(1, warps / LCS_WARPS), LCS_WARPS * 32, 0, s>>>(v, rsc);
        SHM_CUDA(cudaGetLastError());
    } else if (v.P.rarity) {  // every candidate through the global path, with its rarity support
        if (v.P.rw_score) {
            S.r_mw.reserve((size_t)n);
            v.r_mw = S.r_mw.p;
            k_rarity_mw<<<grid_for((size_t)n, 128, 8), 128, 0, s>>>(v);
            SHM_CUDA(cudaGetLastError());
            count_launch();
        }
        k_refine_rarity<<<(unsigned)std::max<size_t>(1, warps / REFINE_WARPS), REFINE_WARPS * 32, 0, s>>>(v, rsc);
        SHM_CUDA(cudaGetLastError());
    } else {
        if (!c->refine_smem_set) {
            SHM_CUDA(cudaFuncSetAttribute(k_refine, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)(REFINE_WARPS * REFINE_SLICE)));
            c->refine_smem_set = 1;
        }
        for (int pass = 0; pass < (v.lead_on ? 2 : 1); pass++) {
            if (p.metric != SHM_BUCKET_SH) {
                k_refine_chip<<<grid_for((size_t)n * 32, RCHIP_WARPS * 32, 4), RCHIP_WARPS * 32,
                                RCHIP_WARPS * RCHIP_SLICE, s>>>(v, pass);
                SHM_CUDA(cudaGetLastError());
                count_launch();
            }
            k_refine<<<(unsigned)std::max<size_t>(1, warps / REFINE_WARPS), REFINE_WARPS * 32,
                       REFINE_WARPS * REFINE_SLICE, s>>>(v, rsc, pass);
            SHM_CUDA(cudaGetLastError());
            if (pass == 0 && v.lead_on) count_launch();  // the last launch is counted by the stage timer
        }
    }
    T.end();
    T.begin(STG_SWEEP);
    k_sweep<<<grid_for((size_t)n * 32, SWEEP_WARPS * 32, 16), SWEEP_WARPS * 32, 0, s>>>(v, S.sweep_scr.p);
    SHM_CUDA(cudaGetLastError());
    T.end();

    copy_async(c, &R.fin, S.mx.p, sizeof(BatchMax), cudaMemcpyDeviceToHost, s);
    copy_async(c, &R.nj, S.n_jobs.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    copy_async(c, &R.nc, S.coff.p + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    copy_async(c, sl.ovf, S.ovf_list.p, 4 * sizeof(uint32_t) * (size_t)n, cudaMemcpyDeviceToHost, s);
    H.mark("enq_rest");
    if (debug) {
        SHM_CUDA(cudaStreamSynchronize(s));
        std::fprintf(stderr, "[shmap] jobs=%u (cap %u) candidates=%u overflow=%u\n", R.nj, job_cap, R.nc,
                     R.fin.n_overflow);
        if (R.nj && R.nj <= 16) {
            std::vector<BucketJob> jb(R.nj);
            SHM_CUDA(cudaMemcpy(jb.data(), S.jobs.p, sizeof(BucketJob) * R.nj, cudaMemcpyDeviceToHost));
            for (auto& j : jb)
                std::fprintf(stderr,
                             "[shmap]  job read=%d seg=%d bb=%d m0=%d matches=%d codir=%d r=[%d,%d] sh=%.6f cand=%d "
                             "score=%.6f t=[%d,%d] I=%d same=%d\n",
                             j.read, j.seg, j.bb, j.m0, j.matches, j.codir, j.rmin, j.rmax, j.sh, j.is_cand, j.score,
                             j.t_l, j.t_r, j.inter, j.same);
        }
    }
    H.print(exact ? "exact-batch" : "batch", n);
}

// Batch limits: device-resident reads in few large batches; host reads in
// smaller ones so that copying batch b+1 overlaps mapping batch b.
// Batch sizes come from the measured settings (shm_tune.hpp): device-resident
// calls cut batches of dev_batch_reads / dev_batch_bases, the first of them
// smaller (dev_first_batch_reads) so the device starts while the host plans
// the next (about 5 ns a read); calls from host buffers cut host_batch_*, the
// first small too, since its packing on the host is what nothing overlaps.

__global__ void k_scatter_records(const shm_map_record* __restrict__ src, const int32_t* __restrict__ idx, int32_t n,
                                  shm_map_record* __restrict__ dst) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[idx[i]] = src[i];
}

// Copies read i of a list (bytes [src[3i], src[3i] + src[3i+2]) of `base`) to
// staged + src[3i+1]; one block per read.
__global__ void k_gather_reads(const uint8_t* __restrict__ base, const int64_t* __restrict__ list, int32_t n,
                               uint8_t* __restrict__ staged) {
    for (int32_t i = blockIdx.x; i < n; i += gridDim.x) {
        const int64_t from = list[3 * (size_t)i], to = list[3 * (size_t)i + 1], len = list[3 * (size_t)i + 2];
        for (int64_t j = threadIdx.x; j < len; j += blockDim.x) staged[to + j] = base[from + j];
    }
}

// Where retried reads come from and where their records go: device memory
// (read g at d_seq + offs[g] - offs[0], record g at d_out[g]) or host memory
// (read g at h_seq + offs[g], record g at h_out[g]).
struct RetryIO {
    const uint8_t* d_seq;
    shm_map_record* d_out;
    const uint8_t* h_seq;
    shm_map_record* h_out;
};

// One group of reads mapped again (exact: synchronous sizing, bucket tables
// of at most bt_lim slots a read, 0 = the full bound): their bytes gathered
// into one batch, their records scattered back to their places; the reads
// that overflow again go to *again (with their read indices in the call).
static void retry_group(MapCtx* c, const IndexStorage* ix, const shm_params& p, const std::vector<Overflow>& ovf,
                        const int64_t* offs, const RetryIO& io, bool exact, uint64_t bt_lim,
                        std::vector<Overflow>* again_out) {
    cudaStream_t s = c->stream;
    MapScratch& S = *c->scr;
    const int32_t n = (int32_t)ovf.size();
    std::vector<int64_t> o((size_t)n + 1, 0);
    std::vector<uint32_t> caps((size_t)n);
    for (int32_t i = 0; i < n; i++) {
        o[(size_t)i + 1] = o[(size_t)i] + (offs[ovf[i].read + 1] - offs[ovf[i].read]);
        caps[(size_t)i] = ovf[i].m;
    }
    const int64_t nb = o.back();
    // one pinned block: the gather list or the reads' bytes, the plan, the record slots
    const size_t list_bytes = io.d_seq ? 24 * (size_t)n : (size_t)nb;
    const size_t plan_at = (list_bytes + 63) / 64 * 64;
    const size_t idx_at = plan_at + (BatchPlan::layout(n) + 63) / 64 * 64;
    uint8_t* pin = pinned_stage(c, idx_at + sizeof(int32_t) * (size_t)n);
    S.retry_seq.reserve((size_t)nb + 32);
    SHM_CUDA(cudaMemsetAsync(S.retry_seq.p + nb, 0, 32, s));
    if (io.d_seq) {  // device reads: one gather kernel
        int64_t* lst = (int64_t*)pin;
        for (int32_t i = 0; i < n; i++) {
            lst[3 * (size_t)i] = offs[ovf[i].read] - offs[0];
            lst[3 * (size_t)i + 1] = o[(size_t)i];
            lst[3 * (size_t)i + 2] = o[(size_t)i + 1] - o[(size_t)i];
        }
        S.retry_list.reserve(3 * (size_t)n);
        copy_async(c, S.retry_list.p, lst, 24 * (size_t)n, cudaMemcpyHostToDevice, s);
        k_gather_reads<<<(unsigned)std::min<int32_t>(n, 1184), 256, 0, s>>>(io.d_seq, S.retry_list.p, n,
                                                                           S.retry_seq.p);
        SHM_CUDA(cudaGetLastError());
        count_launch();
    } else {  // host reads: gathered into pinned memory, one copy
        for (int32_t i = 0; i < n; i++)
            std::memcpy(pin + o[(size_t)i], io.h_seq + offs[ovf[i].read], (size_t)(o[(size_t)i + 1] - o[(size_t)i]));
        copy_async(c, S.retry_seq.p, pin, (size_t)nb, cudaMemcpyHostToDevice, s);
    }
    S.retry_out.reserve((size_t)n);
    StageTimer T(c);
    const std::vector<std::pair<int32_t, int32_t>> one{{0, n}};
    std::vector<BatchSlot> sl = batch_slots(c, one, o.data());
    run_batch(c, ix, p, S.retry_seq.p, o.data(), n, S.retry_out.p, caps.data(), exact, pin + plan_at, T, sl[0],
              nullptr, nullptr, bt_lim);
    SHM_CUDA(cudaStreamSynchronize(s));
    if (!exact && sl[0].R->nj > sl[0].job_cap) {  // too many bucket jobs for the queued sizes: counted this time
        run_batch(c, ix, p, S.retry_seq.p, o.data(), n, S.retry_out.p, caps.data(), true, pin + plan_at, T, sl[0],
                  nullptr, nullptr, fast_bt_read_cap());
        SHM_CUDA(cudaStreamSynchronize(s));
    }
    T.collect();
    std::vector<Overflow> again;
    collect_batch(c, sl[0], again);
    if (io.d_out) {  // records to their slots on the device
        int32_t* h_idx = (int32_t*)(pin + idx_at);
        for (int32_t i = 0; i < n; i++) h_idx[i] = ovf[i].read;
        S.retry_idx.reserve((size_t)n);
        copy_async(c, S.retry_idx.p, h_idx, sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, s);
        k_scatter_records<<<grid_for((size_t)n, 256), 256, 0, s>>>(S.retry_out.p, S.retry_idx.p, n, io.d_out);
        SHM_CUDA(cudaGetLastError());
        count_launch();
        SHM_CUDA(cudaStreamSynchronize(s));
    } else {  // records to their slots on the host, through pinned memory
        shm_map_record* h_rec = (shm_map_record*)pinned_stage(c, sizeof(shm_map_record) * (size_t)n);
        copy_async(c, h_rec, S.retry_out.p, sizeof(shm_map_record) * (size_t)n, cudaMemcpyDeviceToHost, s);
        SHM_CUDA(cudaStreamSynchronize(s));
        for (int32_t i = 0; i < n; i++) io.h_out[ovf[i].read] = h_rec[i];
    }
    for (const Overflow& a : again) again_out->push_back(Overflow{ovf[a.read].read, a.m, a.eb});
}

// The retry ladder's bucket-table limits, in slots a read: a read whose table
// filled up is mapped again with eight times the slots (never more than its
// bound), and the last step takes its full bound.
static const uint64_t RETRY_BT[] = {4096, 32768, 262144, 0};
constexpr int RETRY_STEPS = (int)(sizeof(RETRY_BT) / sizeof(RETRY_BT[0]));

// Reads that overflowed a capacity are mapped again. Those that beat their
// k-mer capacity estimate (their seeds never prepared) go first as a queued
// batch with their counts as capacities. Those whose bucket table filled up
// climb the ladder, each step synchronous and cut into groups whose tables
// and per-read buffers fit a share of the device's free memory, so that many
// reads of huge bucket counts (reads from tandem arrays at high -r) never ask
// for all their memory at once.
static void retry_overflows(MapCtx* c, const IndexStorage* ix, const shm_params& p, const std::vector<Overflow>& ovf,
                            const int64_t* offs, const RetryIO& io, int step = -1) {
    if (ovf.empty()) return;
    std::vector<Overflow> next;
    if (step < 0) {  // k-mer capacity overflows: one queued batch; table overflows climb from the first step
        std::vector<Overflow> kmer;
        for (const Overflow& o : ovf) (o.eb == 0 ? kmer : next).push_back(o);
        if (!kmer.empty()) retry_group(c, ix, p, kmer, offs, io, false, 0, &next);
        retry_overflows(c, ix, p, next, offs, io, 0);
        return;
    }
    if (step >= RETRY_STEPS) {
        std::fprintf(stderr, "shmap-b200: read %d exceeds a device capacity even with exact bounds\n", ovf[0].read);
        throw shm_cuda_error(cudaErrorMemoryAllocation);
    }
    const uint64_t lim = RETRY_BT[step];
    size_t free_b = 0, total_b = 0;
    SHM_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const uint64_t budget = std::max<uint64_t>((uint64_t)1 << 29, free_b / 3);
    std::vector<Overflow> group;
    uint64_t used = 0;
    auto flush = [&]() {
        if (group.empty()) return;
        retry_group(c, ix, p, group, offs, io, true, lim, &next);
        group.clear();
        used = 0;
    };
    for (const Overflow& o : ovf) {
        const uint64_t full = std::max<uint64_t>(16, pow2_host(2 * std::max<uint64_t>(o.eb, 1)));
        const uint64_t slots = lim ? std::min(lim, full) : full;
        // the table (slot, list entry), a job and its lists and sweep scratch per slot,
        // the k-mer, seed and probe arrays per k-mer of capacity
        const uint64_t bytes = slots * (sizeof(BSlot) + 4 + sizeof(BucketJob) + 12 + 2 * 48) +
                               (uint64_t)o.m * 160 + ((uint64_t)offs[o.read + 1] - (uint64_t)offs[o.read]) + 4096;
        if (!group.empty() && used + bytes > budget) flush();
        group.push_back(o);
        used += bytes;
    }
    flush();
    retry_overflows(c, ix, p, next, offs, io, step + 1);
}

// The nonzero mask words of a packed batch into its zeroed mask.
__global__ void k_mask_scatter(const uint32_t* __restrict__ pairs, uint32_t n, uint32_t* __restrict__ mask) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        mask[pairs[2 * i]] = pairs[2 * i + 1];
}

// Batches of at most max_reads reads and max_bases bases (one read at a time
// in the plain form).
static std::vector<std::pair<int32_t, int32_t>> cut_batches(const int64_t* offs, int32_t n, bool plain,
                                                            int32_t max_reads, int64_t max_bases,
                                                            int32_t first_max_reads = 0, bool taper = false) {
    std::vector<std::pair<int32_t, int32_t>> b;
    int32_t i = 0;
    int64_t lim_b = max_bases;
    while (i < n) {
        int32_t j = i + 1;
        const int32_t lim = (i == 0 && first_max_reads > 0) ? first_max_reads : max_reads;
        // taper: the rest, once it fits one batch, in about four (the last
        // batch's upload and mapping are what nothing overlaps)
        if (taper && lim_b == max_bases && offs[n] - offs[i] <= max_bases)
            lim_b = std::max<int64_t>((offs[n] - offs[i]) / 4 + 1, (int64_t)1 << 24);
        if (!plain)
            while (j < n && j - i < lim && offs[j + 1] - offs[i] <= lim_b) j++;
        b.emplace_back(i, j);
        i = j;
    }
    return b;
}

// Pinned plan blocks for every batch of a call (batches are queued without
// waiting, so each keeps its own until the stream drains).
static std::vector<uint8_t*> plan_blocks(MapCtx* c, const std::vector<std::pair<int32_t, int32_t>>& b) {
    size_t total = 0;
    for (auto [i, j] : b) total += (BatchPlan::layout(j - i) + 63) / 64 * 64;
    uint8_t* base = pinned_stage(c, total);
    std::vector<uint8_t*> out;
    for (auto [i, j] : b) {
        out.push_back(base);
        base += (BatchPlan::layout(j - i) + 63) / 64 * 64;
    }
    return out;
}

void map_device(MapCtx* c, const IndexStorage* ix, const shm_params& p, const uint8_t* d_seq, const int64_t* h_offs,
                int32_t n, shm_map_record* d_out, bool plain) {
    SHM_CUDA(cudaSetDevice(c->device));
    const Tuning tu = tuning();
    const auto batches = cut_batches(h_offs, n, plain, (int32_t)tu.dev_batch_reads, tu.dev_batch_bases,
                                     (int32_t)tu.dev_first_batch_reads);
    std::vector<BatchSlot> slots = batch_slots(c, batches, h_offs);
    const std::vector<uint8_t*> plans = plan_blocks(c, batches);
    StageTimer T(c);
    // every batch is queued without a wait; the sketch reads exactly the
    // batch's bytes, at any alignment
    for (size_t b = 0; b < batches.size(); b++) {
        const auto [i, j] = batches[b];
        run_batch(c, ix, p, d_seq + (h_offs[i] - h_offs[0]), h_offs + i, j - i, d_out + i, nullptr, false, plans[b], T,
                  slots[b]);
    }
    SHM_CUDA(cudaStreamSynchronize(c->stream));
    // a batch with more bucket jobs than its capacity is mapped again, its jobs counted first
    for (size_t b = 0; b < batches.size(); b++) {
        if (slots[b].R->nj <= slots[b].job_cap) continue;
        const auto [i, j] = batches[b];
        run_batch(c, ix, p, d_seq + (h_offs[i] - h_offs[0]), h_offs + i, j - i, d_out + i, nullptr, true, plans[b], T,
                  slots[b], nullptr, nullptr, fast_bt_read_cap());
        SHM_CUDA(cudaStreamSynchronize(c->stream));
    }
    T.collect();
    std::vector<Overflow> ovf_all;
    for (const BatchSlot& sl : slots) collect_batch(c, sl, ovf_all);
    HostClock H;
    retry_overflows(c, ix, p, ovf_all, h_offs, RetryIO{d_seq, d_out, nullptr, nullptr});
    H.mark("retry");
    H.print("retries", (int32_t)ovf_all.size());
}

// Pieces of a packing stream sent by the threads that pack them. Each thread
// packs a piece into one of its own pinned buffers with plain stores and
// queues the piece's copy into the stream's device codes at once, on its own
// copy stream, while the piece is still in that core's cache (the copy
// engine's reads then come from the cache instead of the codes making a round
// trip through host memory). A buffer is packed again once its last copy has
// completed. Errors on a packing thread are kept and raised by the next call
// of the thread that holds the packing.
struct StreamSink final : PackSink {
    struct Worker {
        cudaStream_t st = nullptr;
        std::vector<cudaEvent_t> ev;  // the last copy out of each buffer
        cudaEvent_t mark = nullptr;   // every copy queued so far (join)
        uint32_t* buf = nullptr;      // ring * piece_words words of the pinned block
        uint32_t next = 0;
    };
    int device = 0, ring = 0;
    size_t piece_words = 0;
    uint32_t* pinned = nullptr;
    std::vector<Worker> w;
    uint32_t* dst = nullptr;       // the device codes of the stream in flight
    uint32_t* mask_dst = nullptr;  // its device mask (raw pieces write their words there)
    uint8_t* d_raw = nullptr;      // raw pieces: ring * piece bytes a thread, device memory
    bool raw_ok = false;           // raw pieces taken in this stream
    cudaEvent_t zeroed = nullptr;  // the stream's device mask is cleared
    std::atomic<int64_t> bytes{0};
    std::atomic<bool> failed{false};
    cudaError_t err = cudaSuccess;
    std::mutex err_mu;

    void fail(cudaError_t e) {
        std::lock_guard<std::mutex> g(err_mu);
        if (failed.load()) return;
        std::fprintf(stderr, "shmap-b200: CUDA error on a packing thread: %s\n", cudaGetErrorString(e));
        err = e;
        failed.store(true);
    }
    uint32_t* piece_buffer(int wi) override {
        if (failed.load() || wi < 0 || wi >= (int)w.size()) {
            if (!failed.load()) fail(cudaErrorInvalidValue);
            return nullptr;
        }
        Worker& x = w[(size_t)wi];
        cudaError_t e = cudaSetDevice(device);
        if (e == cudaSuccess) e = cudaEventSynchronize(x.ev[x.next % ring]);
        if (e != cudaSuccess) {
            fail(e);
            return nullptr;
        }
        return x.buf + (size_t)(x.next % ring) * piece_words;
    }
    void piece_done(int wi, uint32_t* b, size_t first, size_t words) override {
        Worker& x = w[(size_t)wi];
        cudaError_t e = cudaMemcpyAsync(dst + first, b, 4 * words, cudaMemcpyHostToDevice, x.st);
        if (e == cudaSuccess) e = cudaEventRecord(x.ev[x.next % ring], x.st);
        if (e != cudaSuccess) fail(e);
        x.next++;
        bytes += (int64_t)(4 * words);
    }
    // A raw piece: its bytes copied into the thread's device slot, packed
    // there into the stream's codes and mask words (the same layout).
    bool piece_raw(int wi, const uint8_t* src, size_t g0, size_t ng) override {
        if (!raw_ok || !d_raw || failed.load() || wi < 0 || wi >= (int)w.size() || ng == 0 ||
            32 * ng > 16 * piece_words)
            return false;
        Worker& x = w[(size_t)wi];
        const uint32_t sl = x.next % ring;
        uint8_t* d = d_raw + ((size_t)wi * (size_t)ring + sl) * 16 * piece_words;
        cudaError_t e = cudaSetDevice(device);
        if (e == cudaSuccess) e = cudaEventSynchronize(x.ev[sl]);  // the slot's last use is done
        if (e == cudaSuccess) e = cudaMemcpyAsync(d, src, 32 * ng, cudaMemcpyHostToDevice, x.st);
        if (e == cudaSuccess) e = pack_groups_device(d, (int64_t)ng, dst + 2 * g0, mask_dst + g0, x.st);
        if (e == cudaSuccess) e = cudaEventRecord(x.ev[sl], x.st);
        if (e != cudaSuccess) fail(e);  // the call fails at check(); the piece counts as taken
        x.next++;
        bytes += (int64_t)(32 * ng);
        return true;
    }
    void check() {
        if (failed.load()) throw shm_cuda_error(err);
    }
    // (thread holding the packing, no task running) every copy stream waits for e
    void gate(cudaEvent_t e) {
        for (Worker& x : w) SHM_CUDA(cudaStreamWaitEvent(x.st, e, 0));
    }
    // stream s waits for every copy queued so far
    void join(cudaStream_t s) {
        check();
        for (Worker& x : w) {
            SHM_CUDA(cudaEventRecord(x.mark, x.st));
            SHM_CUDA(cudaStreamWaitEvent(s, x.mark, 0));
        }
    }
    ~StreamSink() override {
        cudaSetDevice(device);
        for (Worker& x : w) {
            if (x.st) cudaStreamSynchronize(x.st);
            for (cudaEvent_t e : x.ev)
                if (e) cudaEventDestroy(e);
            if (x.mark) cudaEventDestroy(x.mark);
            if (x.st) cudaStreamDestroy(x.st);
        }
        if (zeroed) cudaEventDestroy(zeroed);
        if (pinned) cudaFreeHost(pinned);
        if (d_raw) cudaFree(d_raw);
    }
};

static void free_stream_sink(StreamSink* u) { delete u; }

// The context's stream sink for pieces of piece_words code words and `ring`
// buffers a packing thread (made again when the settings changed).
static StreamSink* stream_sink(MapCtx* c, size_t piece_words, int ring, bool raw) {
    const int nw = pack_workers();
    if (c->sink && c->sink->piece_words == piece_words && c->sink->ring == ring && (int)c->sink->w.size() == nw &&
        !c->sink->failed.load()) {
        if (raw && !c->sink->d_raw)
            SHM_CUDA(cudaMalloc((void**)&c->sink->d_raw, 16 * piece_words * (size_t)ring * (size_t)nw));
        return c->sink;
    }
    delete c->sink;
    c->sink = nullptr;
    auto* u = new StreamSink();
    u->device = c->device;
    u->ring = ring;
    u->piece_words = piece_words;
    c->sink = u;  // released with the context even if a step below fails
    SHM_CUDA(cudaHostAlloc((void**)&u->pinned, 4 * piece_words * (size_t)ring * (size_t)nw, cudaHostAllocDefault));
    if (raw) SHM_CUDA(cudaMalloc((void**)&u->d_raw, 16 * piece_words * (size_t)ring * (size_t)nw));
    SHM_CUDA(cudaEventCreateWithFlags(&u->zeroed, cudaEventDisableTiming));
    u->w.resize((size_t)nw);
    for (int i = 0; i < nw; i++) {
        StreamSink::Worker& x = u->w[(size_t)i];
        x.buf = u->pinned + piece_words * (size_t)ring * (size_t)i;
        SHM_CUDA(cudaStreamCreateWithFlags(&x.st, cudaStreamNonBlocking));
        x.ev.assign((size_t)ring, nullptr);
        for (auto& e : x.ev) SHM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        SHM_CUDA(cudaEventCreateWithFlags(&x.mark, cudaEventDisableTiming));
    }
    return u;
}

// Device batches over one packing stream: the first of about first_bases,
// each next twice the one before (at most max_reads reads and max_bases
// bases), and once the rest fits two of the current size, halves of the rest
// down to last_bases: the device starts early, maps most of the stream in
// large batches and ends soon after the packing does; a rest below
// last_bases joins the batch before it. (A batch has a fixed device cost,
// about 0.7 ms on the hifi workload, so batches below a few hundred MB would
// map slower than the host packs the next one.)
static std::vector<std::pair<int32_t, int32_t>> cut_stream_batches(const int64_t* offs, int32_t r0, int32_t r1,
                                                                   int64_t first_bases, int64_t last_bases,
                                                                   int64_t max_bases, int32_t max_reads) {
    std::vector<std::pair<int32_t, int32_t>> b;
    int64_t tgt = std::max<int64_t>(1, first_bases);
    for (int32_t i = r0; i < r1;) {
        const int64_t rest = offs[r1] - offs[i];
        int64_t lim = rest <= 2 * tgt ? std::max(rest / 2, last_bases) : tgt;
        if (rest - lim < last_bases) lim = rest;  // no last batch smaller than last_bases (its fixed cost)
        int32_t j = i + 1;
        while (j < r1 && j - i < max_reads && offs[j + 1] - offs[i] <= lim) j++;
        b.emplace_back(i, j);
        i = j;
        tgt = std::min(2 * tgt, max_bases);
    }
    return b;
}

// Host-buffer form, streamed. The reads of a call (in parts of at most
// host_stream_bases) are packed in order by the host threads into one pinned
// buffer, in tasks of host_pack_task_kib with no wait between batches; each
// chunk of host_stream_chunk_kib goes up on the copy stream as soon as all
// its tasks are done (codes, then its nonzero mask words scattered into the
// zeroed device mask). The device maps batches over the packed copy
// (cut_stream_batches), each once the chunk holding its last base is up: a
// batch starts at any base of the stream, its sketch reading the codes from
// the batch's first 32-base group with the base offset in its plan. The
// calling thread uploads chunks, queues batches and packs tasks in between.
static bool map_host_stream(MapCtx* c, const IndexStorage* ix, const shm_params& p, const uint8_t* seqs,
                            const int64_t* offs, int32_t n, shm_map_record* out, BatchSink* sink) {
    MapScratch& S = *c->scr;
    cudaStream_t s = c->stream, cs = c->copy_stream;
    const Tuning tu = tuning();
    const bool by_piece = tu.host_stream == 2;  // pieces sent by the packing threads
    const int64_t task_kib = by_piece ? tu.host_stream_piece_kib : (tu.host_pack_task_kib > 0 ? tu.host_pack_task_kib : 256);
    const int64_t task_groups = std::max<int64_t>(2, (task_kib * 1024 / 32) & ~(int64_t)1);
    const int chunk_tasks = (int)std::max<int64_t>(1, tu.host_stream_chunk_kib * 1024 / 32 / task_groups);
    const int64_t chunk_groups = task_groups * chunk_tasks;
    const int LIST_SLOTS = 8;
    // the parts: whole reads, at most host_stream_bases each (a longer read alone)
    std::vector<std::pair<int32_t, int32_t>> parts;
    for (int32_t i = 0; i < n;) {
        int32_t j = i + 1;
        while (j < n && offs[j + 1] - offs[i] <= tu.host_stream_bases) j++;
        parts.emplace_back(i, j);
        i = j;
    }
    // every device batch of the call, part by part (their plans and result slots)
    std::vector<std::pair<int32_t, int32_t>> batches;
    std::vector<size_t> part_first;
    for (auto [r0, r1] : parts) {
        part_first.push_back(batches.size());
        auto b = cut_stream_batches(offs, r0, r1, tu.host_stream_first_kib * 1024, tu.host_stream_last_kib * 1024,
                                    tu.dev_batch_bases, (int32_t)tu.dev_batch_reads);
        batches.insert(batches.end(), b.begin(), b.end());
    }
    part_first.push_back(batches.size());
    int64_t max_nb = 0;
    int32_t max_n = 1;
    for (auto [r0, r1] : parts) max_nb = std::max<int64_t>(max_nb, offs[r1] - offs[r0]);
    for (auto [i, j] : batches) max_n = std::max(max_n, j - i);
    const size_t cwords = packed_code_words(max_nb), mwords = packed_mask_words(max_nb);
    const size_t list_cap = (size_t)chunk_groups + 3;  // mask words of a chunk at most (the last: + tail)
    // pinned: the codes of a part, then LIST_SLOTS chunk lists (pairs)
    // (by piece, the codes go up from the packing threads' own buffers: only the six tail words stay here)
    const size_t codes_bytes = by_piece ? 64 : (4 * cwords + 63) / 64 * 64, list_bytes = (8 * list_cap + 63) / 64 * 64;
    const size_t need = codes_bytes + LIST_SLOTS * list_bytes;
    if (need > c->h_pack_cap) {
        if (c->h_pack) SHM_CUDA(cudaFreeHost(c->h_pack));
        c->h_pack = nullptr;
        c->h_pack_cap = 0;
        SHM_CUDA(cudaHostAlloc(&c->h_pack, need, cudaHostAllocDefault));
        c->h_pack_cap = need;
    }
    uint32_t* h_codes = (uint32_t*)c->h_pack;
    auto h_list = [&](int slot) { return (uint32_t*)(c->h_pack + codes_bytes + (size_t)slot * list_bytes); };
    S.pk_codes[0].reserve(cwords);
    S.pk_mask[0].reserve(mwords);
    S.pk_list[0].reserve(2 * list_cap * LIST_SLOTS);
    S.out.reserve((size_t)max_n);
    // a share of the pieces (host_stream_raw_share percent) goes up as bytes
    // from the caller's buffer, when that is pinned, and is packed on the device
    int raw_pct = by_piece ? (int)tu.host_stream_raw_share : 0;
    if (raw_pct > 0) {
        cudaPointerAttributes pa{};
        if (cudaPointerGetAttributes(&pa, seqs) != cudaSuccess || pa.type != cudaMemoryTypeHost) {
            cudaGetLastError();
            raw_pct = 0;
        }
    }
    StreamSink* sink_up =
        by_piece ? stream_sink(c, 2 * (size_t)task_groups, (int)tu.host_stream_ring, raw_pct > 0) : nullptr;
    if (sink_up) {
        sink_up->dst = S.pk_codes[0].p;
        sink_up->mask_dst = S.pk_mask[0].p;
        sink_up->raw_ok = raw_pct > 0;
    }
    std::vector<BatchSlot> slots = batch_slots(c, batches, offs);
    const std::vector<uint8_t*> plans = plan_blocks(c, batches);
    StageTimer T(c);
    HostClock H;
    // per-batch timeline (SHMAP_HOSTPROF): when each batch was queued, and its device span
    struct Tl {
        double run0 = 0;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
    };
    std::vector<Tl> tl(H.on ? batches.size() : 0);
    cudaEvent_t tl0 = nullptr;
    if (H.on) {
        SHM_CUDA(cudaEventCreate(&tl0));
        SHM_CUDA(cudaEventRecord(tl0, s));
        for (auto& t : tl) {
            SHM_CUDA(cudaEventCreate(&t.e0));
            SHM_CUDA(cudaEventCreate(&t.e1));
        }
    }
    struct StreamEnd {  // a packing started and never finished (an error) is ended
        bool on = false;
        ~StreamEnd() {
            if (on) pack_stream_finish();
        }
    } stream_end;
    for (size_t pi = 0; pi < parts.size(); pi++) {
        const auto [r0, r1] = parts[pi];
        const int64_t nb = offs[r1] - offs[r0];
        const size_t pw = packed_code_words(nb);
        // the pinned codes and lists are free once the part before is up; the
        // device buffers once its last sketch has read them
        if (pi > 0) SHM_CUDA(cudaStreamSynchronize(cs));
        SHM_CUDA(cudaStreamWaitEvent(cs, c->sketched[0], 0));
        SHM_CUDA(cudaMemsetAsync(S.pk_mask[0].p, 0, 4 * packed_mask_words(nb), cs));
        if (sink_up) {  // the threads' copies go after the last sketch of the buffers and the mask's clearing
            SHM_CUDA(cudaEventRecord(sink_up->zeroed, cs));
            sink_up->gate(c->sketched[0]);
            sink_up->gate(sink_up->zeroed);
        }
        stream_end.on = true;
        const int chunks =
            pack_stream_start(seqs + offs[r0], nb, h_codes, task_groups, chunk_tasks, sink_up, raw_pct);
        while (c->up_ev.size() < (size_t)chunks) {
            cudaEvent_t e;
            SHM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            c->up_ev.push_back(e);
        }
        auto chunk_of = [&](int64_t g) { return (int)std::min<int64_t>(chunks - 1, g / chunk_groups); };
        auto upload = [&](int ch) {  // chunk ch's codes and mask words, on the copy stream
            const size_t w0 = 2 * (size_t)ch * (size_t)chunk_groups;
            const size_t w1 = ch + 1 == chunks ? pw : std::min(pw, 2 * (size_t)(ch + 1) * (size_t)chunk_groups);
            const int sl = ch % LIST_SLOTS;
            if (ch >= LIST_SLOTS) SHM_CUDA(cudaEventSynchronize(c->up_ev[(size_t)(ch - LIST_SLOTS)]));
            const size_t nl = pack_stream_chunk_list(ch, h_list(sl), list_cap);
            if (nl > list_cap) throw shm_cuda_error(cudaErrorInvalidValue);  // cannot happen: a word a group
            if (sink_up) {  // the pieces went up from the packing threads; the tail words from here
                if (ch + 1 == chunks)
                    copy_async(c, S.pk_codes[0].p + 2 * (size_t)(nb / 32), h_codes, 4 * 6, cudaMemcpyHostToDevice, cs);
            } else if (w1 > w0) {
                copy_async(c, S.pk_codes[0].p + w0, h_codes + w0, 4 * (w1 - w0), cudaMemcpyHostToDevice, cs);
            }
            if (nl) {
                uint32_t* dl = S.pk_list[0].p + 2 * list_cap * (size_t)sl;
                copy_async(c, dl, h_list(sl), 8 * nl, cudaMemcpyHostToDevice, cs);
                k_mask_scatter<<<grid_for(nl, 256, 4), 256, 0, cs>>>(dl, (uint32_t)nl, S.pk_mask[0].p);
                SHM_CUDA(cudaGetLastError());
                count_launch();
            }
            SHM_CUDA(cudaEventRecord(c->up_ev[(size_t)ch], cs));
        };
        int up_next = 0;
        for (size_t b = part_first[pi]; b < part_first[pi + 1];) {
            while (up_next < chunks && pack_stream_chunk_ready(up_next)) upload(up_next++);
            const auto [i, j] = batches[b];
            const int64_t o = offs[i] - offs[r0], e = offs[j] - offs[r0];
            const int need_ch = chunk_of(std::max<int64_t>(0, e - 1) / 32);
            if (need_ch >= up_next) {  // its last chunk is not up yet: pack a task meanwhile
                if (!pack_stream_help()) std::this_thread::yield();
                continue;
            }
            SHM_CUDA(cudaStreamWaitEvent(s, c->up_ev[(size_t)need_ch], 0));
            if (sink_up) sink_up->join(s);  // every piece queued so far (those of its chunks among them)
            c->sketch_done = c->sketched[0];
            if (!tl.empty()) {
                tl[b].run0 = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - H.t0).count();
                SHM_CUDA(cudaEventRecord(tl[b].e0, s));
            }
            const int64_t g0 = o / 32;
            run_batch(c, ix, p, nullptr, offs + i, j - i, S.out.p, nullptr, false, plans[b], T, slots[b],
                      S.pk_codes[0].p + 2 * g0, S.pk_mask[0].p + g0, 0, (int32_t)(o - 32 * g0), pw - 2 * (size_t)g0);
            c->sketch_done = nullptr;
            if (sink) sink->batch(i, j, S.out.p, s);
            copy_async(c, out + i, S.out.p, sizeof(shm_map_record) * (size_t)(j - i), cudaMemcpyDeviceToHost, s);
            if (!tl.empty()) SHM_CUDA(cudaEventRecord(tl[b].e1, s));
            if (sink) sink->poll();
            b++;
        }
        stream_end.on = false;
        pack_stream_finish();
        if (sink_up) sink_up->check();
    }
    if (sink_up) c->work[W_H2D_BYTES] += sink_up->bytes.exchange(0);
    H.mark("enqueue");
    SHM_CUDA(cudaStreamSynchronize(s));
    H.mark("drain");
    if (!tl.empty()) {
        for (size_t b = 0; b < tl.size(); b++) {
            float d0 = 0, d1 = 0;
            SHM_CUDA(cudaEventElapsedTime(&d0, tl0, tl[b].e0));
            SHM_CUDA(cudaEventElapsedTime(&d1, tl0, tl[b].e1));
            std::fprintf(stderr, "[shmap-host] stream batch %zu reads %d MB %.0f: queued %.2f device %.2f-%.2f\n", b,
                         batches[b].second - batches[b].first,
                         (offs[batches[b].second] - offs[batches[b].first]) / 1e6, tl[b].run0, d0, d1);
            cudaEventDestroy(tl[b].e0);
            cudaEventDestroy(tl[b].e1);
        }
        cudaEventDestroy(tl0);
    }
    // a batch with more bucket jobs than its capacity is mapped again, its jobs counted first
    bool changed = false;
    for (size_t b = 0; b < batches.size(); b++) {
        if (slots[b].R->nj <= slots[b].job_cap) continue;
        changed = true;
        const auto [i, j] = batches[b];
        const int64_t nb = offs[j] - offs[i];
        S.seqb[0].reserve((size_t)nb + 32);
        SHM_CUDA(cudaMemsetAsync(S.seqb[0].p + nb, 0, 32, s));
        copy_async(c, S.seqb[0].p, seqs + offs[i], (size_t)nb, cudaMemcpyHostToDevice, s);
        run_batch(c, ix, p, S.seqb[0].p, offs + i, j - i, S.out.p, nullptr, true, plans[b], T, slots[b], nullptr,
                  nullptr, fast_bt_read_cap());
        copy_async(c, out + i, S.out.p, sizeof(shm_map_record) * (size_t)(j - i), cudaMemcpyDeviceToHost, s);
        SHM_CUDA(cudaStreamSynchronize(s));
    }
    T.collect();
    std::vector<Overflow> ovf_all;
    for (const BatchSlot& sl : slots) collect_batch(c, sl, ovf_all);
    retry_overflows(c, ix, p, ovf_all, offs, RetryIO{nullptr, nullptr, seqs, out});
    H.mark("retry");
    H.print("host-stream", n);
    return changed || !ovf_all.empty();
}

// Host-buffer form. Batch b+1's bytes go up on the copy stream while batch b
// is mapped (two device buffers, each reused once the sketch of the batch
// before has read it), so the transfer of the reads overlaps the mapping when
// `seqs` is pinned; records come back batch by batch.
bool map_host(MapCtx* c, const IndexStorage* ix, const shm_params& p, const uint8_t* seqs, const int64_t* offs,
              int32_t n, shm_map_record* out, bool plain, BatchSink* sink) {
    SHM_CUDA(cudaSetDevice(c->device));
    if (!plain && n > 0 && tuning().host_stream && tuning().host_raw_share == 0)
        return map_host_stream(c, ix, p, seqs, offs, n, out, sink);
    MapScratch& S = *c->scr;
    cudaStream_t s = c->stream;
    const auto batches =
        cut_batches(offs, n, plain, (int32_t)tuning().host_batch_reads, tuning().host_batch_bases,
                    (int32_t)tuning().host_first_batch_reads, true);
    int64_t max_nb = 0;
    int32_t max_n = 0;
    for (auto [i, j] : batches) {
        max_nb = std::max<int64_t>(max_nb, offs[j] - offs[i]);
        max_n = std::max(max_n, j - i);
    }
    // reads go up packed: two pinned slots on the host (codes, then the
    // nonzero mask words as pairs), two device buffers
    const size_t cwords = packed_code_words(max_nb), mwords = packed_mask_words(max_nb);
    const size_t slot_bytes = (4 * (cwords + 2 * mwords) + 63) / 64 * 64;  // slots and their code words 64-byte aligned
    if (2 * slot_bytes > c->h_pack_cap) {
        if (c->h_pack) SHM_CUDA(cudaFreeHost(c->h_pack));
        c->h_pack = nullptr;
        c->h_pack_cap = 0;
        SHM_CUDA(cudaHostAlloc(&c->h_pack, 2 * slot_bytes, cudaHostAllocDefault));
        c->h_pack_cap = 2 * slot_bytes;
    }
    for (int k = 0; k < 2; k++) {
        S.pk_codes[k].reserve(cwords);
        S.pk_mask[k].reserve(mwords);
        S.pk_list[k].reserve(2 * mwords);
    }
    S.out.reserve((size_t)std::max(max_n, 1));
    // a share of the batches (host_raw_share percent, spread evenly) goes up as
    // ASCII straight from the caller's buffer when that is pinned: the copy
    // engine reads 1 byte a base where packing reads 1, writes 1/4 and the
    // copy engine reads that 1/4, so moving a share off the host threads eases
    // the host's memory bandwidth while the link takes more bytes
    int64_t raw_pct = tuning().host_raw_share;
    if (raw_pct > 0) {
        cudaPointerAttributes pa{};
        if (cudaPointerGetAttributes(&pa, seqs) != cudaSuccess || pa.type != cudaMemoryTypeHost) {
            cudaGetLastError();
            raw_pct = 0;
        }
    }
    std::vector<char> raw(batches.size(), 0);
    for (size_t b = 0; b < batches.size(); b++)
        raw[b] = ((int64_t)(b + 1) * raw_pct / 100) > ((int64_t)b * raw_pct / 100);
    for (int k = 0; k < 2 && raw_pct > 0; k++) S.seqb[k].reserve((size_t)max_nb + 32);
    // the packed batches and the raw ones, each in order; a batch's buffers
    // (host slot and device buffer) alternate within its own kind
    std::vector<size_t> pk_list, raw_list;
    std::vector<int> slot(batches.size(), 0), kind_pos(batches.size(), 0);
    for (size_t b = 0; b < batches.size(); b++) {
        std::vector<size_t>& L = raw[b] ? raw_list : pk_list;
        kind_pos[b] = (int)L.size();
        slot[b] = (int)(L.size() & 1);
        L.push_back(b);
    }
    auto h_codes = [&](size_t b) { return (uint32_t*)(c->h_pack + (size_t)slot[b] * slot_bytes); };
    auto h_list = [&](size_t b) { return (uint32_t*)(c->h_pack + (size_t)slot[b] * slot_bytes + 4 * cwords); };
    HostClock H;
    // per-batch timeline (SHMAP_HOSTPROF): host phases, and device events around each batch's mapping
    struct Tl {
        double pack0 = 0, wait0 = 0, wait1 = 0, run0 = 0, run1 = 0;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
    };
    std::vector<Tl> tl(H.on ? batches.size() : 0);
    cudaEvent_t tl0 = nullptr;
    auto ms_now = [&] {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - H.t0).count();
    };
    if (H.on) {
        SHM_CUDA(cudaEventCreate(&tl0));
        SHM_CUDA(cudaEventRecord(tl0, s));
        for (auto& t : tl) {
            SHM_CUDA(cudaEventCreate(&t.e0));
            SHM_CUDA(cudaEventCreate(&t.e1));
        }
    }
    const int64_t task_groups = tuning().host_pack_task_kib * 1024 / 32;
    auto pack = [&](size_t b) {  // on the host threads in the background, once the slot's previous upload left
        const auto [i, j] = batches[b];
        SHM_CUDA(cudaEventSynchronize(c->copied[slot[b]]));
        if (!tl.empty()) tl[b].pack0 = ms_now();
        pack_reads_host_start(seqs + offs[i], offs[j] - offs[i], h_codes(b), task_groups);
    };
    size_t n_list = 0;  // nonzero mask words of the packing just waited for
    auto wait = [&](size_t b) {
        const auto [i, j] = batches[b];
        if (!tl.empty()) tl[b].wait0 = ms_now();
        n_list = pack_reads_host_wait(h_list(b), packed_mask_words(offs[j] - offs[i]));
        if (!tl.empty()) tl[b].wait1 = ms_now();
    };
    auto send = [&](size_t b) {  // on the copy stream, after the sketch that last read the buffers
        const auto [i, j] = batches[b];
        const int64_t nb = offs[j] - offs[i];
        const int sl = slot[b];
        cudaStream_t cs = c->copy_stream;
        SHM_CUDA(cudaStreamWaitEvent(cs, c->sketched[sl], 0));
        copy_async(c, S.pk_codes[sl].p, h_codes(b), 4 * packed_code_words(nb), cudaMemcpyHostToDevice, cs);
        SHM_CUDA(cudaMemsetAsync(S.pk_mask[sl].p, 0, 4 * packed_mask_words(nb), cs));
        if (n_list) {  // the nonzero mask words into the zeroed mask
            copy_async(c, S.pk_list[sl].p, h_list(b), 8 * n_list, cudaMemcpyHostToDevice, cs);
            k_mask_scatter<<<grid_for(n_list, 256, 4), 256, 0, cs>>>(S.pk_list[sl].p, (uint32_t)n_list,
                                                                    S.pk_mask[sl].p);
            SHM_CUDA(cudaGetLastError());
            count_launch();
        }
        SHM_CUDA(cudaEventRecord(c->copied[sl], cs));
    };
    // a raw batch's bytes as they are, and the zero pad the sketch reads past
    // the end, on the raw stream once the sketch of the raw batch two before
    // it (the same buffer) has read that buffer, and no earlier than RAW_LEAD
    // batches before its own: the copy runs while the batches before it are
    // packed, without taking the link from the first batches' uploads
    constexpr size_t RAW_LEAD = 3;
    size_t raw_sent = 0;
    auto send_raw_ready = [&](size_t mapped_upto) {  // batches [0, mapped_upto) are queued
        while (raw_sent < raw_list.size() && raw_list[raw_sent] <= mapped_upto + RAW_LEAD &&
               (raw_sent < 2 || raw_list[raw_sent - 2] < mapped_upto)) {
            const size_t b = raw_list[raw_sent++];
            const auto [i, j] = batches[b];
            const int64_t nb = offs[j] - offs[i];
            const int sl = slot[b];
            cudaStream_t rs = c->raw_stream;
            SHM_CUDA(cudaStreamWaitEvent(rs, c->raw_sketched[sl], 0));
            copy_async(c, S.seqb[sl].p, seqs + offs[i], (size_t)nb, cudaMemcpyHostToDevice, rs);
            SHM_CUDA(cudaMemsetAsync(S.seqb[sl].p + nb, 0, 32, rs));
            SHM_CUDA(cudaEventRecord(c->raw_copied[sl], rs));
        }
    };
    std::vector<BatchSlot> slots = batch_slots(c, batches, offs);
    const std::vector<uint8_t*> plans = plan_blocks(c, batches);
    StageTimer T(c);
    struct PackRelease {  // a packing started and never waited for (an error) is ended
        ~PackRelease() { pack_reads_host_release(); }
    } pack_release;
    // the packed batches: k + 1 is packed on the host threads while k is
    // queued, k - 1 maps and k goes up
    size_t pk_next = 0;  // the next packed batch to wait for and send
    send_raw_ready(0);
    if (!pk_list.empty()) {
        pack(pk_list[0]);
        wait(pk_list[0]);
        send(pk_list[0]);
        pk_next = 1;
        if (pk_list.size() > 1) pack(pk_list[1]);
    }
    for (size_t b = 0; b < batches.size(); b++) {
        const auto [i, j] = batches[b];
        const int sl = slot[b];
        if (!raw[b] && kind_pos[b] >= (int)pk_next) {  // not sent yet (a raw batch came before it)
            wait(b);
            send(b);
            pk_next = (size_t)kind_pos[b] + 1;
            if (pk_next < pk_list.size()) pack(pk_list[pk_next]);
        }
        SHM_CUDA(cudaStreamWaitEvent(s, raw[b] ? c->raw_copied[sl] : c->copied[sl], 0));
        c->sketch_done = raw[b] ? c->raw_sketched[sl] : c->sketched[sl];
        if (!tl.empty()) {
            tl[b].run0 = ms_now();
            SHM_CUDA(cudaEventRecord(tl[b].e0, s));
        }
        if (raw[b])
            run_batch(c, ix, p, S.seqb[sl].p, offs + i, j - i, S.out.p, nullptr, false, plans[b], T, slots[b]);
        else
            run_batch(c, ix, p, nullptr, offs + i, j - i, S.out.p, nullptr, false, plans[b], T, slots[b],
                      S.pk_codes[sl].p, S.pk_mask[sl].p);
        c->sketch_done = nullptr;
        if (sink) sink->batch(i, j, S.out.p, s);
        copy_async(c, out + i, S.out.p, sizeof(shm_map_record) * (size_t)(j - i), cudaMemcpyDeviceToHost,
                                 s);
        if (!tl.empty()) {
            SHM_CUDA(cudaEventRecord(tl[b].e1, s));
            tl[b].run1 = ms_now();
        }
        send_raw_ready(b + 1);
        // the next packed batch, when it maps next: wait for its packing, send it, start the one after
        if (b + 1 < batches.size() && !raw[b + 1] && pk_next < pk_list.size() && pk_list[pk_next] == b + 1) {
            wait(b + 1);
            send(b + 1);
            pk_next++;
            if (pk_next < pk_list.size()) pack(pk_list[pk_next]);
        }
        if (sink) sink->poll();
    }
    H.mark("enqueue");
    SHM_CUDA(cudaStreamSynchronize(s));
    H.mark("drain");
    if (!tl.empty()) {
        for (size_t b = 0; b < tl.size(); b++) {
            float d0 = 0, d1 = 0;
            SHM_CUDA(cudaEventElapsedTime(&d0, tl0, tl[b].e0));
            SHM_CUDA(cudaEventElapsedTime(&d1, tl0, tl[b].e1));
            std::fprintf(stderr,
                         "[shmap-host] batch %zu reads %d MB %.0f%s: pack %.2f wait %.2f-%.2f run %.2f-%.2f "
                         "device %.2f-%.2f\n",
                         b, batches[b].second - batches[b].first,
                         (offs[batches[b].second] - offs[batches[b].first]) / 1e6, raw[b] ? " raw" : "", tl[b].pack0,
                         tl[b].wait0, tl[b].wait1, tl[b].run0, tl[b].run1, d0, d1);
            cudaEventDestroy(tl[b].e0);
            cudaEventDestroy(tl[b].e1);
        }
        cudaEventDestroy(tl0);
    }
    // a batch with more bucket jobs than its capacity is mapped again, its jobs counted first
    bool changed = false;
    for (size_t b = 0; b < batches.size(); b++) {
        if (slots[b].R->nj <= slots[b].job_cap) continue;
        changed = true;
        const auto [i, j] = batches[b];
        const int64_t nb = offs[j] - offs[i];
        S.seqb[0].reserve((size_t)nb + 32);
        SHM_CUDA(cudaMemsetAsync(S.seqb[0].p + nb, 0, 32, s));
        copy_async(c, S.seqb[0].p, seqs + offs[i], (size_t)nb, cudaMemcpyHostToDevice, s);
        run_batch(c, ix, p, S.seqb[0].p, offs + i, j - i, S.out.p, nullptr, true, plans[b], T, slots[b], nullptr,
                  nullptr, fast_bt_read_cap());
        copy_async(c, out + i, S.out.p, sizeof(shm_map_record) * (size_t)(j - i), cudaMemcpyDeviceToHost,
                                 s);
        SHM_CUDA(cudaStreamSynchronize(s));
    }
    T.collect();
    std::vector<Overflow> ovf_all;
    for (const BatchSlot& sl : slots) collect_batch(c, sl, ovf_all);
    retry_overflows(c, ix, p, ovf_all, offs, RetryIO{nullptr, nullptr, seqs, out});
    H.mark("retry");
    H.print("host-form", n);
    return changed || !ovf_all.empty();
}

}  // namespace shm

// Test hook (not part of the C ABI of include/shmap_gpu.h): the device batches
// cut_stream_batches makes of reads [0, n) with offsets offs[0..n]; writes up
// to cap (first, end) read-index pairs to out and returns their number.
extern "C" int shm_internal_cut_stream(const int64_t* offs, int32_t n, int64_t first_bases, int64_t last_bases,
                                       int64_t max_bases, int32_t max_reads, int32_t* out, int32_t cap) {
    if (n < 0 || (n > 0 && !offs) || first_bases <= 0 || last_bases <= 0 || max_bases <= 0 || max_reads <= 0)
        return -1;
    const auto b = shm::cut_stream_batches(offs, 0, n, first_bases, last_bases, max_bases, max_reads);
    for (size_t i = 0; i < b.size() && (int32_t)i < cap; i++) {
        out[2 * i] = b[i].first;
        out[2 * i + 1] = b[i].second;
    }
    return (int)b.size();
}
