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
#include "shm_tune.hpp"

#include <cstdlib>
#include <mutex>
#include <vector>

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

// Lookup tables as the rolling step reads them: the entering base's pair
// {fw, rc rotated left by k-1} and the leaving base's pair {fw rotated left
// by k, rc rotated right by 1}, one 16-byte shared load each.
struct __align__(16) LutPair {
    uint64_t a, b;
};

constexpr int SK_THREADS = 256;                                  // one run of SKETCH_WIN windows per thread
constexpr int SK_TILE_CAP = SK_THREADS * SKETCH_WIN + 1024;       // bytes a CTA stages per tile
// + slack for the words past the last byte: the rotated-frame runs read up to
// 36 bytes past it (their last group of 32 windows, and the word after)
constexpr int SK_TILE_WORDS = SK_TILE_CAP / 4 + 16;
constexpr int SK_TILE_PWORDS = SK_TILE_WORDS + SK_TILE_WORDS / 32 + 1;
constexpr int SK_TILE_BYTES = (SK_TILE_PWORDS * 4 + 15) / 16 * 16; // the tile, rounded to 16 bytes

// Staged bytes carry one pad word after every 32 words: the runs of
// neighbouring threads start SKETCH_WIN bytes apart, so without the pad every
// lane of a warp would read the same bank.
__device__ __forceinline__ int pword(int w) { return w + (w >> 5); }

// The bytes of a tile, staged in shared memory (offsets relative to the tile).
struct StagedBytes {
    const uint32_t* tile;
    __device__ __forceinline__ uint32_t word(int w) const { return tile[pword(w)]; }
};

// The same bytes read from global memory (a tile too large to stage): bytes
// of `base` outside [first, lim) read as 0.
struct GlobalBytes {
    const uint8_t* base;
    int64_t first, lim;
    __device__ __forceinline__ uint32_t word(int64_t w) const {
        uint32_t v = 0;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int64_t x = 4 * w + j;
            if (x >= first && x < lim) v |= (uint32_t)__ldg(base + x) << (8 * j);
        }
        return v;
    }
};

constexpr int SK_LB = 16;  // selections a thread holds per run (append mode)

// The same bytes from packed reads (codes and mask of base B0 + x): ACGT
// letters (upper case) and 'N' for a masked base, 0 outside [first, lim).
struct GlobalPacked {
    const uint32_t* codes;
    const uint32_t* mask;
    int64_t B0, first, lim;
    __device__ __forceinline__ uint32_t word(int64_t w) const {
        uint32_t v = 0;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int64_t x = 4 * w + j;
            if (x >= first && x < lim) {
                const int64_t p = B0 + x;
                const uint32_t c = (__ldg(codes + (p >> 4)) >> (2 * (p & 15))) & 3u;
                const bool m = (__ldg(mask + (p >> 5)) >> (p & 31)) & 1u;
                v |= (m ? 0x4eu : (uint32_t)"ACTG"[c]) << (8 * j);
            }
        }
        return v;
    }
};

// Where a thread's selections go: its count, and (write mode) the run's
// output range from chunk_out[c]. Append
// mode holds the run's first SK_LB selections in thread-local slots (cached
// local memory), moved to the read's list after the run with one counter
// update per read and warp; selections past SK_LB take a slot of the list
// one at a time.
struct Emit {
    uint64_t out_base;
    uint32_t out_cap, n_sel;
    uint64_t bh[SK_LB];
    uint32_t br[SK_LB];
};

// One selection, recorded by the kernel's mode. The bodies stay short (no
// loops, no waits on results): they sit in the rolling loop's rarely taken
// branch, and anything larger there slows every window.
template <int MODE>
__device__ __forceinline__ void emit_kmer(const SketchArgs& a, int32_t q, uint64_t h, uint32_t rs, Emit& e) {
    if (MODE == SK_COUNT) {
        e.n_sel++;
    } else if (MODE == SK_WRITE) {
        a.out_h[e.out_base + e.n_sel] = h;
        a.out_rs[e.out_base + e.n_sel] = rs;
        e.n_sel++;
    } else if (e.n_sel < (uint32_t)SK_LB) {
        e.bh[e.n_sel] = h;
        e.br[e.n_sel] = rs;
        e.n_sel++;
    } else {
        const uint32_t slot = atomicAdd(a.kmer_cnt + q, 1u);
        if (slot < e.out_cap) {
            a.out_h[e.out_base + slot] = h;
            a.out_rs[e.out_base + slot] = rs;
        }
    }
}

// Byte j of a word, as a table index (one byte permute).
__device__ __forceinline__ uint32_t byte_of(uint32_t w, int j) { return __byte_perm(w, 0u, 0x4440u + (uint32_t)j); }

// One rolling step: byte ib enters, byte ob leaves.
__device__ __forceinline__ void roll(uint64_t& fw, uint64_t& rc, const LutPair* __restrict__ Lin,
                                     const LutPair* __restrict__ Lout, uint32_t ib, uint32_t ob) {
    const LutPair pi = Lin[ib], po = Lout[ob];
    fw = rotl1(fw) ^ po.a ^ pi.a;
    rc = rotr1(rc) ^ po.b ^ pi.b;
}

// Window selection: h = fw ^ rc <= thr. The high words decide all but about
// one window in a hundred (for thr near 1% of the range); the full compare
// runs only for those.
template <int MODE>
__device__ __forceinline__ void check(const SketchArgs& a, uint64_t fw, uint64_t rc, uint32_t thr_hi, uint64_t thr,
                                      int32_t q, int32_t r, Emit& e) {
    const uint32_t hh = (uint32_t)(fw >> 32) ^ (uint32_t)(rc >> 32);
    if (hh <= thr_hi) {
        const uint64_t h = fw ^ rc;
        if (h <= thr) emit_kmer<MODE>(a, q, h, ((uint32_t)r << 1) | (fw > rc ? 1u : 0u), e);
    }
}

// The windows [0, cnt) of one run whose first byte is at offset x of `src`.
// Window 0 is reached by rolling its k bytes in from the all-zero state: a
// window of k non-ACGT bytes hashes to 0 on both strands, and the leaving
// bytes of those steps are such bytes. Window t > 0 takes byte x+t+k-1 in and
// drops byte x+t-1.
template <int MODE, class Src, class Idx>
__device__ __forceinline__ void sketch_run(const SketchArgs& a, const LutPair* __restrict__ Lin,
                                           const LutPair* __restrict__ Lout, const Src& src, Idx x, int32_t cnt,
                                           int k, uint64_t thr, int32_t q, int32_t r0, Emit& e) {
    if (cnt <= 0) return;
    const uint32_t thr_hi = (uint32_t)(thr >> 32);
    uint64_t fw = 0, rc = 0;
    {  // bytes x .. x+k-1, four per word read (bytes past x+k-1 are read, not used)
        const uint32_t sh = (uint32_t)(x & 3) * 8;
        Idx w = x >> 2;
        uint32_t lw = src.word(w);
        for (int i = 0; i < k; i += 4) {
            const uint32_t hw = src.word(++w);
            const uint32_t b4 = __funnelshift_r(lw, hw, sh);
            lw = hw;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                if (i + j < k) {
                    const LutPair pi = Lin[byte_of(b4, j)];
                    fw = rotl1(fw) ^ pi.a;
                    rc = rotr1(rc) ^ pi.b;
                }
            }
        }
    }
    check<MODE>(a, fw, rc, thr_hi, thr, q, r0, e);
    const Idx xi = x + k, xo = x;
    const uint32_t shi = (uint32_t)(xi & 3) * 8, sho = (uint32_t)(xo & 3) * 8;
    Idx wi = xi >> 2, wo = xo >> 2;
    uint32_t li = src.word(wi), lo_ = src.word(wo);
    int32_t t = 1;
    for (; t + 3 < cnt; t += 4) {
        const uint32_t hi_i = src.word(++wi), hi_o = src.word(++wo);
        const uint32_t ib4 = __funnelshift_r(li, hi_i, shi), ob4 = __funnelshift_r(lo_, hi_o, sho);
        li = hi_i;
        lo_ = hi_o;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            roll(fw, rc, Lin, Lout, byte_of(ib4, j), byte_of(ob4, j));
            check<MODE>(a, fw, rc, thr_hi, thr, q, r0 + t + j, e);
        }
    }
    if (t < cnt) {
        const uint32_t hi_i = src.word(++wi), hi_o = src.word(++wo);
        const uint32_t ib4 = __funnelshift_r(li, hi_i, shi), ob4 = __funnelshift_r(lo_, hi_o, sho);
#pragma unroll
        for (int j = 0; j < 3; j++) {
            if (t + j < cnt) {
                roll(fw, rc, Lin, Lout, byte_of(ib4, j), byte_of(ob4, j));
                check<MODE>(a, fw, rc, thr_hi, thr, q, r0 + t + j, e);
            }
        }
    }
}

// ------------------------------------------------------------------ packed reads
// The sketch of reads packed as 2-bit codes (A, C, T, G = 0..3) with a
// non-ACGT mask, rolled without rotating the state. With X_t and Y_t the
// table values window t XORs in (forward: fw of the entering base and fw<<k
// of the leaving one; reverse: rc<<(k-1) of the entering base and rc>>1 of
// the leaving one), the rolling step is F_t = rotl1(F_{t-1}) ^ X_t and
// R_t = rotr1(R_{t-1}) ^ Y_t. In the frame F~_t = rotr(F_t, t),
// R~_t = rotl(R_t, t) the step is a plain XOR: F~_t = F~_{t-1} ^ rotr(X_t, t),
// R~_t = R~_{t-1} ^ rotl(Y_t, t), and the tables hold the rotated values for
// every entering/leaving code pair. Rotation by 32 swaps a value's halves,
// so the state is kept half-swapped during every other group of 32 windows
// and the tables need 32 rows: row jj holds rotr(X, jj) and rotl(Y, jj).
// The selection test needs only the high word of h_t = F_t ^ R_t, two funnel
// shifts of the stored state by jj; the full hash and the strand are formed
// for the rare windows that pass it. A run starts from the hash of the
// window one base before its first (warm-up, four bases a step), so the
// leaving base of its first window is read like every other.
struct PkTables {
    uint2 pf[32][16];  // [jj][ci * 4 + co]: rotr(fw[ci] ^ fw_k[co], jj), as (lo, hi)
    uint2 pr[32][16];  // rotl(rc_k1[ci] ^ rc_r1[co], jj)
    uint4 w4[256];     // four bases c0..c3 (c0 the earliest, bits 0-1): rolled-in (F, R) as (Flo, Fhi, Rlo, Rhi)
    uint4 w1[4];       // one base: (fw, rc_k1)
};

__device__ __forceinline__ uint64_t u64_of(uint32_t lo, uint32_t hi) { return ((uint64_t)hi << 32) | lo; }

__device__ void build_pk_tables(PkTables& P, const SketchLuts* __restrict__ L) {
    const unsigned char let[4] = {'A', 'C', 'T', 'G'};
    for (int e = threadIdx.x; e < 32 * 16; e += blockDim.x) {
        const int jj = e >> 4, ci = (e >> 2) & 3, co = e & 3;
        const uint64_t x = L->fw[let[ci]] ^ L->fw_k[let[co]];
        const uint64_t y = L->rc_k1[let[ci]] ^ L->rc_r1[let[co]];
        const uint64_t rx = rotr64(x, (uint32_t)jj), ly = rotl64(y, (uint32_t)jj);
        P.pf[jj][ci * 4 + co] = make_uint2((uint32_t)rx, (uint32_t)(rx >> 32));
        P.pr[jj][ci * 4 + co] = make_uint2((uint32_t)ly, (uint32_t)(ly >> 32));
    }
    for (int idx = threadIdx.x; idx < 256; idx += blockDim.x) {
        uint64_t f = 0, r = 0;
        for (int i = 0; i < 4; i++) {
            const unsigned char c = let[(idx >> (2 * i)) & 3];
            f ^= rotl64(L->fw[c], (uint32_t)(3 - i));
            r ^= rotr64(L->rc_k1[c], (uint32_t)(3 - i));
        }
        P.w4[idx] = make_uint4((uint32_t)f, (uint32_t)(f >> 32), (uint32_t)r, (uint32_t)(r >> 32));
    }
    if (threadIdx.x < 4) {
        const unsigned char c = let[threadIdx.x];
        const uint64_t f = L->fw[c], r = L->rc_k1[c];
        P.w1[threadIdx.x] = make_uint4((uint32_t)f, (uint32_t)(f >> 32), (uint32_t)r, (uint32_t)(r >> 32));
    }
}

// ------------------------------------------------------------------ staged letters in the rotated frame
// The windows of a run whose bytes are all A, C, G or T (either case) roll
// in the frame of k_sketch_pk: each letter's code is (byte >> 1) & 3 (A, C,
// T, G = 0..3), so four windows' table offsets (entering code * 32 + leaving
// code * 8) come from one entering and one leaving word with two shifts and
// masks, and a window is one byte permute, two 8-byte table loads, four
// XORs and the high-word test. A window that passes the test keeps its
// state in a thread-local buffer; the full hash, strand and selection are
// formed for those after the run, once every byte the run read is known to
// be a letter. A run with any other byte (or more than FR_CAP such windows)
// returns false having selected nothing, and rolls through the byte tables
// instead. The window before the run's first (which includes the byte
// before it, whatever it holds) is the warm-up's: that byte enters and
// leaves through the same code, so it cancels.
constexpr int FR_CAP = 32;

// Code byte of four letters (the earliest in bits 0-1): the codes sit at
// bits 0-1 of each byte after the shift and mask; the multiply gathers byte
// i's code at bits 24 + 2i with no carry into them from the other products.
__device__ __forceinline__ uint32_t codes4(uint32_t w) { return (((w >> 1) & 0x03030303u) * 0x01041040u) >> 24; }

// Nonzero unless the four bytes of w are letters A, C, G, T of either case:
// the byte that a letter of the same code would be (A, C, T, G = 0x41 +
// 2c, plus 15 for c = 2), against the byte with its case bit cleared.
__device__ __forceinline__ uint32_t not_acgt4(uint32_t w) {
    const uint32_t d = w & 0x06060606u;                        // 2c per byte
    const uint32_t t = (d >> 2) & ~(d >> 1) & 0x01010101u;      // c == 2
    const uint32_t want = t * 15u + d + 0x41414141u;            // no carries between bytes
    return (w & 0xdfdfdfdfu) ^ want;
}

// Tile word w (words before the tile read as 0: only the byte before a run
// at the tile's first byte reaches them, and that byte cancels).
__device__ __forceinline__ uint32_t tile_word(const uint32_t* tile, int w) { return w < 0 ? 0u : tile[pword(w)]; }

template <int MODE>
__device__ __forceinline__ bool sketch_run_frame(const SketchArgs& a, const PkTables& P, const uint32_t* tile, int x,
                                                 int32_t cnt, int k, uint64_t thr, int32_t q, int32_t r0, Emit& e) {
    uint32_t bad = 0;
    // warm-up: the window of bytes [x - 1, x + k - 1), four letters a step
    uint64_t F = 0, R = 0;
    {
        const int b = x - 1;
        const uint32_t sh = (uint32_t)(b & 3) * 8;
        int w = b >> 2;  // -1 for b = -1
        uint32_t lw = tile_word(tile, w);
        int i = 0;
        for (; i + 4 <= k; i += 4) {
            const uint32_t hw = tile_word(tile, ++w);
            const uint32_t b4 = __funnelshift_r(lw, hw, sh);
            lw = hw;
            // the byte before the run is not checked (it cancels); the rest are
            bad |= i == 0 ? (not_acgt4(b4) & 0xffffff00u) : not_acgt4(b4);
            const uint4 t = P.w4[codes4(b4)];
            F = rotl64(F, 4) ^ u64_of(t.x, t.y);
            R = rotr64(R, 4) ^ u64_of(t.z, t.w);
        }
        if (i < k) {
            const uint32_t hw = tile_word(tile, ++w);
            const uint32_t b4 = __funnelshift_r(lw, hw, sh);
            const int rem = k - i;  // 1..3 bytes
            const uint32_t keep = (1u << (8 * rem)) - 1u;
            bad |= (i == 0 ? (not_acgt4(b4) & 0xffffff00u) : not_acgt4(b4)) & keep;
            for (int u = 0; u < rem; u++) {
                const uint4 t = P.w1[(b4 >> (8 * u + 1)) & 3u];
                F = rotl64(F, 1) ^ u64_of(t.x, t.y);
                R = rotr64(R, 1) ^ u64_of(t.z, t.w);
            }
        }
    }
    F = rotl64(F, 1);  // the frame at t = -1
    R = rotr64(R, 1);
    // the frame state as one register quad (F~ low, high; R~ low, high): a
    // passing window stores it with one 16-byte store, no moves
    uint4 st = make_uint4((uint32_t)F, (uint32_t)(F >> 32), (uint32_t)R, (uint32_t)(R >> 32));
    const uint32_t thr_hi = (uint32_t)(thr >> 32);
    // entering bytes from x + k - 1, leaving bytes from x - 1
    const int bi = x + k - 1, bo = x - 1;
    const uint32_t shi = (uint32_t)(bi & 3) * 8, sho = (uint32_t)(bo & 3) * 8;
    int wi = bi >> 2, wo = bo >> 2;
    uint32_t li = tile_word(tile, wi), lo_ = tile_word(tile, wo);
    uint4 buf[FR_CAP];
    uint32_t n = 0, m0 = 0, m1 = 0, m2 = 0, m3 = 0;  // passing windows of the last four groups (m0 the latest)
    int32_t groups = 0;
#pragma unroll 1
    for (int32_t t0 = 0; t0 < cnt; t0 += 32) {
        uint32_t mg = 0;
#pragma unroll
        for (int s4 = 0; s4 < 8; s4++) {
            const uint32_t hi_i = tile[pword(++wi)], hi_o = tile[pword(++wo)];  // wo >= -1 before the increment
            const uint32_t win = __funnelshift_r(li, hi_i, shi), wout = __funnelshift_r(lo_, hi_o, sho);
            li = hi_i;
            lo_ = hi_o;
            bad |= not_acgt4(win);
            // byte j: entering code * 32 + leaving code * 8, the entry's offset in its row
            const uint32_t comb = ((win << 4) & 0x60606060u) | ((wout << 2) & 0x18181818u);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int jj = 4 * s4 + j;
                const uint32_t off = __byte_perm(comb, 0u, 0x4440u + (uint32_t)j);
                const uint2 ef = *(const uint2*)((const char*)&P.pf[jj][0] + off);
                const uint2 er = *(const uint2*)((const char*)&P.pr[jj][0] + off);
                st.x ^= ef.x;
                st.y ^= ef.y;
                st.z ^= er.x;
                st.w ^= er.y;
                const uint32_t hh = __funnelshift_l(st.x, st.y, jj) ^ __funnelshift_r(st.w, st.z, jj);
                if (hh <= thr_hi) {
                    buf[n & (FR_CAP - 1)] = st;
                    n++;
                    mg |= 1u << jj;
                }
            }
        }
        m3 = m2;
        m2 = m1;
        m1 = m0;
        m0 = mg;
        groups++;
        st = make_uint4(st.y, st.x, st.w, st.z);  // rotation by 32: the next group's rows apply to the swapped halves
    }
    if (bad != 0 || n > (uint32_t)FR_CAP) return false;
    // the passing windows in order: group g's mask is m_(groups - 1 - g)
    // (windows past the run's last one, rolled in its last group, are skipped)
    uint32_t at = 0;
    for (int32_t g = 0; g < groups; g++) {
        const int back = groups - 1 - g;
        uint32_t mk = back == 0 ? m0 : back == 1 ? m1 : back == 2 ? m2 : m3;
        if (32 * g + 32 > cnt) mk &= (1u << (cnt - 32 * g)) - 1u;  // cnt - 32g in 1..31 here
        while (mk) {
            const uint32_t jj = (uint32_t)__ffs(mk) - 1;
            mk &= mk - 1;
            const uint4 st = buf[at++];
            const uint64_t Fv = rotl64(u64_of(st.x, st.y), jj), Rv = rotr64(u64_of(st.z, st.w), jj);
            const uint64_t h = Fv ^ Rv;
            if (h <= thr) emit_kmer<MODE>(a, q, h, ((uint32_t)(r0 + 32 * g + (int32_t)jj) << 1) | (Fv > Rv ? 1u : 0u), e);
        }
    }
    return true;
}

// Dynamic shared memory of a k_sketch CTA: the staged tile.
constexpr size_t sk_dyn_bytes(int) { return (size_t)SK_TILE_BYTES; }

// Each CTA takes tiles of SK_THREADS consecutive runs. Runs are laid out in
// sequence order, so a tile's bytes are one contiguous range of `seq`: it is
// staged in shared memory with coalesced 16-byte loads and the runs roll out
// of shared memory. A tile whose range does not fit (many sequences shorter
// than k between its runs) rolls from global memory instead.
//
// PK: the tile is staged from packed reads instead, each code word unpacked
// to four words of letters (a 256-entry table of four letters per code byte)
// and masked bases set to 'N', so the rolling below sees the bytes that the
// same read's upper-cased ASCII would give — the same hashes.
template <int MODE, bool PK>
__global__ void __launch_bounds__(SK_THREADS) k_sketch(SketchArgs a, const SketchLuts* __restrict__ luts) {
    __shared__ LutPair Lin[256], Lout[256];
    __shared__ PkTables P;
    __shared__ uint32_t s_unpack[PK ? 256 : 1];
    __shared__ int64_t s_lo, s_hi;
    __shared__ int32_t s_q[2];
    extern __shared__ __align__(16) uint8_t sk_dyn[];
    uint32_t* tile = (uint32_t*)sk_dyn;
    build_pk_tables(P, luts);
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        Lin[i] = LutPair{luts->fw[i], luts->rc_k1[i]};
        Lout[i] = LutPair{luts->fw_k[i], luts->rc_r1[i]};
        if (PK) {
            uint32_t w = 0;
            for (int j = 0; j < 4; j++) w |= (uint32_t)"ACTG"[(i >> (2 * j)) & 3] << (8 * j);
            s_unpack[i] = w;
        }
    }
    Emit e;
    const int lane = threadIdx.x & 31;
    const int k = a.k;
    const uint64_t thr = a.thr;
    const uint64_t n_chunks = a.n_chunks;
    const uint64_t n_tiles = (n_chunks + SK_THREADS - 1) / SK_THREADS;
    for (uint64_t tl = blockIdx.x; tl < n_tiles; tl += gridDim.x) {
        const uint64_t c0 = tl * SK_THREADS, c = c0 + threadIdx.x;
        const uint64_t c_last = min(c0 + SK_THREADS, n_chunks) - 1;
        if (threadIdx.x < 64) {  // sequences of the tile's first and last runs: warps 0 and 1
            const int32_t lo = warp_last_le(a.chunk_off, a.n_seq, threadIdx.x < 32 ? c0 : c_last, lane);
            if (lane == 0) s_q[threadIdx.x < 32 ? 0 : 1] = lo;
        }
        __syncthreads();
        int32_t q = 0, cnt = 0;
        int64_t start = 0, w0 = 0;  // byte offset of the run in `seq`, its first window in the sequence
        if (c < n_chunks) {
            // the run's sequence lies between those of the tile's first and last runs
            int32_t lo = s_q[0], hi = s_q[1] + 1;
            while (hi - lo > 1) {
                const int32_t mid = (lo + hi) >> 1;
                if (__ldg(a.chunk_off + mid) <= c) lo = mid;
                else hi = mid;
            }
            q = lo;
            const int64_t s0 = __ldg(a.seq_off + q), nw = __ldg(a.seq_off + q + 1) - s0 - k + 1;
            w0 = (int64_t)(c - __ldg(a.chunk_off + q)) * SKETCH_WIN;
            cnt = (int32_t)(min(w0 + (int64_t)SKETCH_WIN, nw) - w0);
            start = s0 + w0;
            if (c == c0) s_lo = start;
            if (c == c_last) s_hi = start + cnt + k - 1;
        }
        __syncthreads();  // s_lo/s_hi written; the previous tile's readers are done
        const int64_t lo_b = s_lo, hi_b = s_hi;
        // the tile's bytes are [first, lim) from A0 (ASCII) or from base B0 (packed), both 16-aligned
        const uint8_t* A0 = PK ? nullptr : (const uint8_t*)((uintptr_t)(a.seq + lo_b) & ~(uintptr_t)15);
        const int64_t B0 = lo_b & ~(int64_t)15;
        const int64_t lim = PK ? hi_b - B0 : (int64_t)((a.seq + hi_b) - A0);
        const int64_t first = PK ? lo_b - B0 : (int64_t)((a.seq + lo_b) - A0);
        const bool staged = lim <= (int64_t)SK_TILE_CAP;
        if (PK && staged) {
            const int nv = (int)((lim + 15) >> 4);
            for (int v = threadIdx.x; v < nv; v += SK_THREADS) {
                const int64_t cwi = (B0 >> 4) + v;  // code word of bases B0 + 16v ..
                const uint32_t cw = __ldg(a.pk_codes + cwi);
                const uint32_t m16 = (__ldg(a.pk_mask + (cwi >> 1)) >> (16 * (cwi & 1))) & 0xffffu;
#pragma unroll
                for (int m = 0; m < 4; m++) {
                    uint32_t w = s_unpack[(cw >> (8 * m)) & 0xffu];
                    const uint32_t nib = (m16 >> (4 * m)) & 15u;
                    if (nib) {  // masked bases: 'N' (byte j of M is 0xff for bit j of nib)
                        const uint32_t M = ((nib * 0x00204081u) & 0x01010101u) * 0xffu;
                        w = (w & ~M) | (0x4e4e4e4eu & M);
                    }
                    tile[pword(4 * v + m)] = w;
                }
            }
        } else if (staged) {
            const int nv = (int)((lim + 15) >> 4);
            for (int v = threadIdx.x; v < nv; v += SK_THREADS) {
                uint32_t wv[4];
                if (16 * v >= first && 16 * v + 16 <= lim) {
                    const uint4 u = __ldg((const uint4*)(A0 + 16 * v));
                    wv[0] = u.x;
                    wv[1] = u.y;
                    wv[2] = u.z;
                    wv[3] = u.w;
                } else {
#pragma unroll
                    for (int m = 0; m < 4; m++) {
                        uint32_t w = 0;
                        for (int j = 0; j < 4; j++) {
                            const int64_t xx = 16 * v + 4 * m + j;
                            if (xx >= first && xx < lim) w |= (uint32_t)__ldg(A0 + xx) << (8 * j);
                        }
                        wv[m] = w;
                    }
                }
#pragma unroll
                for (int m = 0; m < 4; m++) tile[pword(4 * v + m)] = wv[m];
            }
        }
        __syncthreads();
        e.n_sel = 0;
        e.out_base = 0;
        e.out_cap = 0;
        if (cnt > 0) {
            if (MODE == SK_WRITE) e.out_base = a.chunk_out[c];
            if (MODE == SK_APPEND) {
                e.out_base = a.kmer_off[q];
                e.out_cap = (uint32_t)(a.kmer_off[q + 1] - e.out_base);
            }
        }
        const int64_t x = PK ? start - B0 : (int64_t)((a.seq + start) - A0);  // the run's first byte in the tile
        const int32_t r0 = (int32_t)(w0 + k - 1) + a.r_offset;              // r of the run's first window
        if (staged) {
            if (cnt > 0 && !sketch_run_frame<MODE>(a, P, tile, (int)x, cnt, k, thr, q, r0, e))
                sketch_run<MODE>(a, Lin, Lout, StagedBytes{tile}, (int)x, cnt, k, thr, q, r0, e);
        } else if (PK)
            sketch_run<MODE>(a, Lin, Lout, GlobalPacked{a.pk_codes, a.pk_mask, B0, first, lim}, x, cnt, k, thr, q, r0,
                             e);
        else
            sketch_run<MODE>(a, Lin, Lout, GlobalBytes{A0, first, lim}, x, cnt, k, thr, q, r0, e);
        if (MODE == SK_COUNT && c < n_chunks) a.chunk_cnt[c] = e.n_sel;
        if (MODE == SK_APPEND) {
            // the held selections go to the read's list: a warp's runs are
            // consecutive, so the lanes of one read are contiguous and take one
            // range of the list between them
            const uint32_t nb = e.n_sel;
            uint32_t incl = nb;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            const unsigned peers = __match_any_sync(0xffffffffu, cnt > 0 ? q : -1);
            const int leader = __ffs(peers) - 1, last = 31 - __clz(peers);
            const uint32_t g0 = __shfl_sync(0xffffffffu, incl - nb, leader);
            const uint32_t gtot = __shfl_sync(0xffffffffu, incl, last) - g0;
            uint32_t base = 0;
            if (lane == leader && cnt > 0 && gtot) base = atomicAdd(a.kmer_cnt + q, gtot);
            base = __shfl_sync(0xffffffffu, base, leader) + (incl - nb) - g0;
            for (uint32_t j = 0; j < nb; j++) {
                if (base + j < e.out_cap) {
                    a.out_h[e.out_base + base + j] = e.bh[j];
                    a.out_rs[e.out_base + base + j] = e.br[j];
                }
            }
        }
        __syncthreads();  // the tile is free for the next one
    }
}

// Code word wi of the batch; words before the batch and past its padding read as 0.
__device__ __forceinline__ uint32_t pk_word(const uint32_t* __restrict__ codes, int64_t wi, uint64_t n_words) {
    return (wi >= 0 && (uint64_t)wi < n_words) ? __ldg(codes + wi) : 0u;
}

// True when bases [b, e) of the batch hold no masked (non-ACGT) base.
__device__ __forceinline__ bool pk_unmasked(const uint32_t* __restrict__ mask, int64_t b, int64_t e) {
    if (e <= b) return true;
    const int64_t w0 = b >> 5, w1 = (e - 1) >> 5;
    uint32_t acc = 0;
    for (int64_t w = w0; w <= w1; w++) {
        uint32_t m = __ldg(mask + w);
        if (w == w0) m &= ~0u << (b & 31);
        if (w == w1) m &= ~0u >> (31 - ((e - 1) & 31));
        acc |= m;
    }
    return acc == 0;
}

// One group of 32 windows, t = t0 + jj: in and out hold the entering and
// leaving bases' codes (32 each, the earliest in bits 0-1 of the low word).
template <int MODE>
__device__ __forceinline__ void pk_group(const SketchArgs& a, const PkTables& P, uint2 in, uint2 out,
                                         uint32_t& Flo, uint32_t& Fhi, uint32_t& Rlo, uint32_t& Rhi,
                                         uint32_t thr_hi, uint64_t thr, int32_t q, int32_t r_t0, int32_t lim,
                                         Emit& e) {
#pragma unroll
    for (int jj = 0; jj < 32; jj++) {
        const uint32_t xi = jj < 16 ? in.x : in.y, xo = jj < 16 ? out.x : out.y;
        const int s = 2 * (jj & 15);
        // entering code * 32 + leaving code * 8: the byte offset in row jj
        const uint32_t ci32 = (s >= 5 ? (xi >> (s - 5)) : (xi << (5 - s))) & 0x60u;
        const uint32_t co8 = (s >= 3 ? (xo >> (s - 3)) : (xo << (3 - s))) & 0x18u;
        const uint32_t off = ci32 | co8;
        const uint2 ef = *(const uint2*)((const char*)&P.pf[jj][0] + off);
        const uint2 er = *(const uint2*)((const char*)&P.pr[jj][0] + off);
        Flo ^= ef.x;
        Fhi ^= ef.y;
        Rlo ^= er.x;
        Rhi ^= er.y;
        const uint32_t hh = __funnelshift_l(Flo, Fhi, jj) ^ __funnelshift_r(Rhi, Rlo, jj);
        if (hh <= thr_hi) {
            const uint64_t F = rotl64(u64_of(Flo, Fhi), (uint32_t)jj), R = rotr64(u64_of(Rlo, Rhi), (uint32_t)jj);
            const uint64_t h = F ^ R;
            if (h <= thr && jj < lim) emit_kmer<MODE>(a, q, h, ((uint32_t)(r_t0 + jj) << 1) | (F > R ? 1u : 0u), e);
        }
    }
}

// The windows [0, cnt) (cnt <= SKETCH_WIN) of the run whose first window
// starts at base p0 of the batch, all of whose bases are unmasked.
template <int MODE>
__device__ __forceinline__ void pk_run(const SketchArgs& a, const PkTables& P, int64_t p0, int32_t cnt, int k,
                                       uint64_t thr, int32_t q, int32_t r0, Emit& e) {
    const uint32_t* __restrict__ codes = a.pk_codes;
    const uint64_t nw = a.pk_words;
    // warm-up: the window of bases [p0 - 1, p0 + k - 1), four bases a step
    uint64_t F = 0, R = 0;
    {
        const int64_t b = p0 - 1;
        int64_t wi = b >> 4;  // arithmetic: -1 for b = -1
        const uint32_t sh = (uint32_t)(b & 15) * 2;
        uint32_t w0 = pk_word(codes, wi, nw), w1 = pk_word(codes, wi + 1, nw);
        int i = 0;
        for (; i + 16 <= k; i += 16) {
            const uint32_t c16 = __funnelshift_r(w0, w1, sh);  // 16 codes from base b + i
            w0 = w1;
            w1 = pk_word(codes, wi + 2 + (i >> 4), nw);
#pragma unroll
            for (int g = 0; g < 4; g++) {
                const uint4 t = P.w4[__byte_perm(c16, 0u, 0x4440u + (uint32_t)g)];
                F = rotl64(F, 4) ^ u64_of(t.x, t.y);
                R = rotr64(R, 4) ^ u64_of(t.z, t.w);
            }
        }
        if (i < k) {  // the last k - i < 16 bases
            const uint32_t c16 = __funnelshift_r(w0, w1, sh);
            int j = 0;
            for (; i + 4 <= k; i += 4, j++) {
                const uint4 t = P.w4[__byte_perm(c16, 0u, 0x4440u + (uint32_t)j)];
                F = rotl64(F, 4) ^ u64_of(t.x, t.y);
                R = rotr64(R, 4) ^ u64_of(t.z, t.w);
            }
            for (int u = 4 * j; i < k; i++, u++) {
                const uint4 t = P.w1[(c16 >> (2 * u)) & 3u];
                F = rotl64(F, 1) ^ u64_of(t.x, t.y);
                R = rotr64(R, 1) ^ u64_of(t.z, t.w);
            }
        }
    }
    // the frame at t = -1: F~ = rotl1(F), R~ = rotr1(R)
    F = rotl64(F, 1);
    R = rotr64(R, 1);
    uint32_t Flo = (uint32_t)F, Fhi = (uint32_t)(F >> 32), Rlo = (uint32_t)R, Rhi = (uint32_t)(R >> 32);
    const uint32_t thr_hi = (uint32_t)(thr >> 32);
    // entering bases from p0 + k - 1, leaving bases from p0 - 1; 32 of each a group
    const int64_t bi = p0 + k - 1, bo = p0 - 1;
    int64_t wi = bi >> 4, wo = bo >> 4;
    const uint32_t shi = (uint32_t)(bi & 15) * 2, sho = (uint32_t)(bo & 15) * 2;
    uint32_t i0 = pk_word(codes, wi, nw), i1 = pk_word(codes, wi + 1, nw), i2 = pk_word(codes, wi + 2, nw);
    uint32_t o0 = pk_word(codes, wo, nw), o1 = pk_word(codes, wo + 1, nw), o2 = pk_word(codes, wo + 2, nw);
    // one group body (32 windows) in the loop: after each group the state's
    // halves are swapped (rotation by 32), so the next group's rows apply as
    // they are; a single body keeps the kernel's code within the instruction cache
#pragma unroll 1
    for (int t0 = 0; t0 < cnt; t0 += 32) {
        // the next group's words, loaded while this one rolls
        const uint32_t i3 = pk_word(codes, wi + 3, nw), i4 = pk_word(codes, wi + 4, nw);
        const uint32_t o3 = pk_word(codes, wo + 3, nw), o4 = pk_word(codes, wo + 4, nw);
        const uint2 in = make_uint2(__funnelshift_r(i0, i1, shi), __funnelshift_r(i1, i2, shi));
        const uint2 out = make_uint2(__funnelshift_r(o0, o1, sho), __funnelshift_r(o1, o2, sho));
        pk_group<MODE>(a, P, in, out, Flo, Fhi, Rlo, Rhi, thr_hi, thr, q, r0 + t0, cnt - t0, e);
        uint32_t x = Flo;
        Flo = Fhi;
        Fhi = x;
        x = Rlo;
        Rlo = Rhi;
        Rhi = x;
        i0 = i2;
        i1 = i3;
        i2 = i4;
        o0 = o2;
        o1 = o3;
        o2 = o4;
        wi += 2;
        wo += 2;
    }
}

// Each thread one run of SKETCH_WIN windows of packed reads (tiles of
// SK_THREADS consecutive runs a CTA, as k_sketch). A run with a masked base
// among its bases rolls through the letter tables instead (GlobalPacked).
template <int MODE>
__global__ void __launch_bounds__(SK_THREADS) k_sketch_pk(SketchArgs a, const SketchLuts* __restrict__ luts) {
    __shared__ PkTables P;
    __shared__ LutPair Lin[256], Lout[256];
    __shared__ int32_t s_q[2];
    build_pk_tables(P, luts);
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        Lin[i] = LutPair{luts->fw[i], luts->rc_k1[i]};
        Lout[i] = LutPair{luts->fw_k[i], luts->rc_r1[i]};
    }
    Emit e;
    const int lane = threadIdx.x & 31;
    const int k = a.k;
    const uint64_t thr = a.thr;
    const uint64_t n_chunks = a.n_chunks;
    const uint64_t n_tiles = (n_chunks + SK_THREADS - 1) / SK_THREADS;
    for (uint64_t tl = blockIdx.x; tl < n_tiles; tl += gridDim.x) {
        const uint64_t c0 = tl * SK_THREADS, c = c0 + threadIdx.x;
        const uint64_t c_last = min(c0 + SK_THREADS, n_chunks) - 1;
        if (threadIdx.x < 64) {  // sequences of the tile's first and last runs: warps 0 and 1
            const int32_t lo = warp_last_le(a.chunk_off, a.n_seq, threadIdx.x < 32 ? c0 : c_last, lane);
            if (lane == 0) s_q[threadIdx.x < 32 ? 0 : 1] = lo;
        }
        __syncthreads();  // also: the tables are built
        int32_t q = 0, cnt = 0;
        int64_t p0 = 0, w0 = 0;
        if (c < n_chunks) {
            int32_t lo = s_q[0], hi = s_q[1] + 1;
            while (hi - lo > 1) {
                const int32_t mid = (lo + hi) >> 1;
                if (__ldg(a.chunk_off + mid) <= c) lo = mid;
                else hi = mid;
            }
            q = lo;
            const int64_t s0 = __ldg(a.seq_off + q), nwin = __ldg(a.seq_off + q + 1) - s0 - k + 1;
            w0 = (int64_t)(c - __ldg(a.chunk_off + q)) * SKETCH_WIN;
            cnt = (int32_t)(min(w0 + (int64_t)SKETCH_WIN, nwin) - w0);
            p0 = s0 + w0;
        }
        __syncthreads();  // s_q read by every thread before the next tile writes it
        e.n_sel = 0;
        e.out_base = 0;
        e.out_cap = 0;
        if (cnt > 0) {
            if (MODE == SK_WRITE) e.out_base = a.chunk_out[c];
            if (MODE == SK_APPEND) {
                e.out_base = a.kmer_off[q];
                e.out_cap = (uint32_t)(a.kmer_off[q + 1] - e.out_base);
            }
        }
        const int32_t r0 = (int32_t)(w0 + k - 1) + a.r_offset;
        const bool fast = cnt > 0 && pk_unmasked(a.pk_mask, p0, p0 + cnt + k - 1);
        if (fast)
            pk_run<MODE>(a, P, p0, cnt, k, thr, q, r0, e);
        else if (cnt > 0)
            sketch_run<MODE>(a, Lin, Lout, GlobalPacked{a.pk_codes, a.pk_mask, 0, p0, p0 + cnt + k - 1}, p0, cnt, k,
                             thr, q, r0, e);
        if (MODE == SK_COUNT && c < n_chunks) a.chunk_cnt[c] = e.n_sel;
        if (MODE == SK_APPEND) {
            const uint32_t nb = e.n_sel;
            uint32_t incl = nb;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            const unsigned peers = __match_any_sync(0xffffffffu, cnt > 0 ? q : -1);
            const int leader = __ffs(peers) - 1, last = 31 - __clz(peers);
            const uint32_t g0 = __shfl_sync(0xffffffffu, incl - nb, leader);
            const uint32_t gtot = __shfl_sync(0xffffffffu, incl, last) - g0;
            uint32_t base = 0;
            if (lane == leader && cnt > 0 && gtot) base = atomicAdd(a.kmer_cnt + q, gtot);
            base = __shfl_sync(0xffffffffu, base, leader) + (incl - nb) - g0;
            for (uint32_t j = 0; j < nb && j < (uint32_t)SK_LB; j++) {
                if (base + j < e.out_cap) {
                    a.out_h[e.out_base + base + j] = e.bh[j];
                    a.out_rs[e.out_base + base + j] = e.br[j];
                }
            }
        }
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
    const bool pk = a.pk_codes != nullptr;
    if (pk && mode != SK_APPEND) throw shm_cuda_error(cudaErrorInvalidValue);
    // packed reads roll in the rotated frame (k_sketch_pk); SHMAP_SKETCH_LETTERS=1
    // rolls them through the letter tables instead (the same selections)
    static const bool letters = std::getenv("SHMAP_SKETCH_LETTERS") != nullptr;
    if (pk && !letters) {
        const uint64_t n_tiles = (a.n_chunks + SK_THREADS - 1) / SK_THREADS;
        k_sketch_pk<SK_APPEND><<<grid_for(n_tiles, 1, (int)tuning().sketch_ctas_per_sm), SK_THREADS, 0, s>>>(a, L);
        SHM_CUDA(cudaGetLastError());
        count_launch();
        return;
    }
    const uint64_t n_tiles = (a.n_chunks + SK_THREADS - 1) / SK_THREADS;
    const int grid = grid_for(n_tiles, 1, 4);  // tiles, at most 4 resident CTAs per SM (shared memory)
    const size_t dyn = sk_dyn_bytes(mode);
    {  // the dynamic shared memory limit, once per device and kernel
        static std::mutex mu;
        static bool done[4][64] = {};
        int dev = 0;
        SHM_CUDA(cudaGetDevice(&dev));
        const int kk = pk ? 3 : mode;
        std::lock_guard<std::mutex> g(mu);
        if (dev >= 0 && dev < 64 && !done[kk][dev]) {
            if (pk)
                SHM_CUDA(cudaFuncSetAttribute(k_sketch<SK_APPEND, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)dyn));
            else if (mode == SK_COUNT)
                SHM_CUDA(cudaFuncSetAttribute(k_sketch<SK_COUNT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)dyn));
            else if (mode == SK_WRITE)
                SHM_CUDA(cudaFuncSetAttribute(k_sketch<SK_WRITE, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)dyn));
            else
                SHM_CUDA(cudaFuncSetAttribute(k_sketch<SK_APPEND, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)dyn));
            done[kk][dev] = true;
        }
    }
    if (pk) k_sketch<SK_APPEND, true><<<grid, SK_THREADS, dyn, s>>>(a, L);
    else if (mode == SK_COUNT) k_sketch<SK_COUNT, false><<<grid, SK_THREADS, dyn, s>>>(a, L);
    else if (mode == SK_WRITE) k_sketch<SK_WRITE, false><<<grid, SK_THREADS, dyn, s>>>(a, L);
    else k_sketch<SK_APPEND, false><<<grid, SK_THREADS, dyn, s>>>(a, L);
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

// Test hook (not part of the C ABI of include/shmap_gpu.h): the read sketch
// of the mapping path (SK_APPEND) for n host reads on `device`, from the
// reads packed on the host (packed != 0, the host-buffer path's layout) or
// from their bytes. Read i's k-mers go unordered to out_h/out_rs from
// cap_off[i] (at most cap_off[i+1] - cap_off[i] of them); out_cnt[i] gets
// their number. Allocates its own device buffers.
#include "../host/pack.hpp"
#include "shm_internal.hpp"

extern "C" int shm_internal_sketch_reads(int device, const uint8_t* seqs, const int64_t* offs, int32_t n, int32_t k,
                                         double h_frac, int packed, const uint64_t* cap_off, uint64_t* out_h,
                                         uint32_t* out_rs, uint32_t* out_cnt) {
    using namespace shm;
    if (n < 0 || k <= 0 || !offs || (n > 0 && (!seqs || !cap_off || !out_cnt))) return -1;
    std::vector<void*> bufs;
    auto dalloc = [&](size_t bytes) {
        void* p = nullptr;
        SHM_CUDA(cudaMalloc(&p, bytes < 16 ? 16 : bytes));
        bufs.push_back(p);
        return p;
    };
    try {
        SHM_CUDA(cudaSetDevice(device));
        const int64_t nb = offs[n] - offs[0];
        std::vector<int64_t> so((size_t)n + 1);
        std::vector<uint64_t> co((size_t)n + 1, 0);
        for (int32_t i = 0; i <= n; i++) so[(size_t)i] = offs[i] - offs[0];
        for (int32_t i = 0; i < n; i++) {
            const int64_t nw = so[(size_t)i + 1] - so[(size_t)i] - k + 1;
            co[(size_t)i + 1] = co[(size_t)i] + (nw > 0 ? (uint64_t)((nw + SKETCH_WIN - 1) / SKETCH_WIN) : 0);
        }
        SketchArgs a{};
        a.n_seq = n;
        a.n_chunks = co[(size_t)n];
        a.k = k;
        a.thr = h_thres(h_frac);
        auto* d_so = (int64_t*)dalloc(8 * so.size());
        auto* d_co = (uint64_t*)dalloc(8 * co.size());
        auto* d_ko = (uint64_t*)dalloc(8 * ((size_t)n + 1));
        auto* d_kc = (uint32_t*)dalloc(4 * (size_t)std::max(n, 1));
        const uint64_t total = cap_off[n];
        auto* d_h = (uint64_t*)dalloc(8 * (size_t)total);
        auto* d_rs = (uint32_t*)dalloc(4 * (size_t)total);
        SHM_CUDA(cudaMemcpy(d_so, so.data(), 8 * so.size(), cudaMemcpyHostToDevice));
        SHM_CUDA(cudaMemcpy(d_co, co.data(), 8 * co.size(), cudaMemcpyHostToDevice));
        SHM_CUDA(cudaMemcpy(d_ko, cap_off, 8 * ((size_t)n + 1), cudaMemcpyHostToDevice));
        SHM_CUDA(cudaMemset(d_kc, 0, 4 * (size_t)std::max(n, 1)));
        if (packed) {
            std::vector<uint32_t> cw(packed_code_words(nb)), mw(packed_mask_words(nb));
            pack_reads_host(seqs + offs[0], nb, cw.data(), mw.data());
            auto* d_cw = (uint32_t*)dalloc(4 * cw.size());
            auto* d_mw = (uint32_t*)dalloc(4 * mw.size());
            SHM_CUDA(cudaMemcpy(d_cw, cw.data(), 4 * cw.size(), cudaMemcpyHostToDevice));
            SHM_CUDA(cudaMemcpy(d_mw, mw.data(), 4 * mw.size(), cudaMemcpyHostToDevice));
            a.pk_codes = d_cw;
            a.pk_mask = d_mw;
            a.pk_words = cw.size();
        } else {
            auto* d_seq = (uint8_t*)dalloc((size_t)nb + 32);
            SHM_CUDA(cudaMemset(d_seq, 0, (size_t)nb + 32));
            if (nb) SHM_CUDA(cudaMemcpy(d_seq, seqs + offs[0], (size_t)nb, cudaMemcpyHostToDevice));
            a.seq = d_seq;
        }
        a.seq_off = d_so;
        a.chunk_off = d_co;
        a.kmer_off = d_ko;
        a.kmer_cnt = d_kc;
        a.out_h = d_h;
        a.out_rs = d_rs;
        SketchLuts* L = create_device_luts(k, nullptr);
        bufs.push_back(L);
        launch_sketch(SK_APPEND, a, L, nullptr);
        SHM_CUDA(cudaDeviceSynchronize());
        SHM_CUDA(cudaMemcpy(out_cnt, d_kc, 4 * (size_t)n, cudaMemcpyDeviceToHost));
        if (total) {
            SHM_CUDA(cudaMemcpy(out_h, d_h, 8 * (size_t)total, cudaMemcpyDeviceToHost));
            SHM_CUDA(cudaMemcpy(out_rs, d_rs, 4 * (size_t)total, cudaMemcpyDeviceToHost));
        }
    } catch (const shm_cuda_error&) {
        for (void* p : bufs) cudaFree(p);
        return -2;
    }
    for (void* p : bufs) cudaFree(p);
    return 0;
}
