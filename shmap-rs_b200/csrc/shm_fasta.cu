// FASTA parsed on the device. The reference reads its inputs with needletail
// (src/io/mod.rs:383-427): a record per '>' header, the id cut at the first
// space or tab, the sequence the record's lines joined without their line
// ends. The command line's host reader (host/shmap_cli.cpp read_fastx) states
// those byte rules, and this parser keeps them exactly. Lines end at '\n'.
// One '\r' right before a line's end is dropped. A line whose first byte is
// '>' is a header, and every other line after the first header belongs to
// the current record, empty lines included. It declines a FASTA file that
// has a line starting with '@' or a non-empty line before the first header
// (which the host reader reports as an error), so such files go to the host
// reader. A file whose first byte is '@' is FASTQ: records of four lines
// (header, sequence, '+', quality), parsed by line index (see the FASTQ
// passes below).
//
// The file's bytes are processed in chunks of CHUNK bytes, one CTA per chunk,
// each thread taking a contiguous run of the chunk (staged in shared memory):
//  1. per chunk: its last line start, whether it starts a header, the flags;
//  2. one block scans those over the chunks: the line start in effect and
//     whether a header was seen, at each chunk's start;
//  3. per chunk: the bytes kept and the headers, counted;
//  4. both counts scanned over the chunks;
//  5. per chunk: the kept bytes compacted through shared memory and stored
//     coalesced at their place; each header's position and the number of
//     sequence bytes before it;
//  6. per header: its name's length, then (after a scan) the name itself.
#include <cstring>
#include <string>
#include <vector>

#include "shm_common.cuh"
#include "shm_fasta.hpp"
#include "shm_internal.hpp"
#include "../host/utf8.hpp"
#include "shm_prims.cuh"

namespace shm {

namespace {

constexpr int FA_THREADS = 256;
constexpr int FA_PER_THREAD = 64;
constexpr int64_t CHUNK = (int64_t)FA_THREADS * FA_PER_THREAD;  // 16 KiB: the write pass stages two

enum : uint32_t { FA_FASTQ = 1u, FA_TEXT_BEFORE_HEADER = 2u };

struct FaView {
    const uint8_t* d;  // the file's bytes
    int64_t len;
    int64_t n_chunks;
};

__device__ __forceinline__ bool line_start(const FaView& v, const uint8_t* sm, int64_t c0, int64_t i) {
    if (i == 0) return true;
    const uint8_t prev = i - 1 >= c0 ? sm[i - 1 - c0] : v.d[i - 1];
    return prev == '\n';
}

// Byte i is the one '\r' dropped before its line's end.
__device__ __forceinline__ bool dropped_cr(const FaView& v, const uint8_t* sm, int64_t c0, int64_t cend, int64_t i) {
    if (sm[i - c0] != '\r') return false;
    if (i + 1 == v.len) return true;
    const uint8_t nx = i + 1 < cend ? sm[i + 1 - c0] : v.d[i + 1];
    return nx == '\n';
}

__device__ void stage_chunk(const FaView& v, int64_t c0, int64_t cend, uint8_t* sm) {
    for (int64_t i = c0 + threadIdx.x; i < cend; i += blockDim.x) sm[i - c0] = v.d[i];
    __syncthreads();
}

template <class T, class Op>
__device__ T block_scan_excl_op(T x, T ident, Op op, T* sh, T* total) {
    // exclusive scan with an associative op over the block's threads (in order)
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    T inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc = op(inc, y);
    }
    if (lane == 31) sh[w] = inc;
    __syncthreads();
    if (w == 0) {
        T t = lane < nw ? sh[lane] : ident;
        T ti = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const T y = __shfl_up_sync(0xffffffffu, ti, o);
            if (lane >= o) ti = op(ti, y);
        }
        if (lane < nw) sh[lane] = ti;  // inclusive over warps
        if (lane == nw - 1) *total = ti;
    }
    __syncthreads();
    const T before_warp = w ? sh[w - 1] : ident;
    T excl = __shfl_up_sync(0xffffffffu, inc, 1);
    excl = lane ? op(before_warp, excl) : before_warp;
    __syncthreads();
    return excl;
}

struct MaxOp {
    __device__ int64_t operator()(int64_t a, int64_t b) const { return a > b ? a : b; }
};
struct SumOp {
    __device__ int64_t operator()(int64_t a, int64_t b) const { return a + b; }
};

// Pass 1: per chunk, its last line start (-1 if none), whether a header
// starts in it, and the flags of line starts with '@'.
__global__ void __launch_bounds__(FA_THREADS) k_fa_marks(FaView v, int64_t* __restrict__ last_ls,
                                                       uint8_t* __restrict__ any_hdr, uint32_t* __restrict__ flags) {
    __shared__ uint8_t sm[CHUNK];
    __shared__ int64_t sh[32];
    __shared__ int64_t tot;
    for (int64_t c = blockIdx.x; c < v.n_chunks; c += gridDim.x) {
        const int64_t c0 = c * CHUNK, cend = min(c0 + CHUNK, v.len);
        stage_chunk(v, c0, cend, sm);
        const int64_t a = c0 + (int64_t)threadIdx.x * FA_PER_THREAD, b = min(a + FA_PER_THREAD, cend);
        int64_t ls = -1, hdr = 0;
        uint32_t fl = 0;
        for (int64_t i = a; i < b; i++) {
            if (!line_start(v, sm, c0, i)) continue;
            ls = i;
            const uint8_t ch = sm[i - c0];
            hdr |= ch == '>';
            if (ch == '@') fl |= FA_FASTQ;
        }
        block_scan_excl_op<int64_t>(ls, -1, MaxOp(), sh, &tot);
        const int64_t cls = tot;
        block_scan_excl_op<int64_t>(hdr, 0, SumOp(), sh, &tot);
        const int64_t chdr = tot;
        if (fl) atomicOr(flags, fl);
        if (threadIdx.x == 0) {
            last_ls[c] = cls;
            any_hdr[c] = chdr > 0;
        }
        __syncthreads();
    }
}

// Pass 2 (one block): at each chunk's start, the line start in effect and
// whether a header was seen before it.
__global__ void __launch_bounds__(1024) k_fa_carry(int64_t n_chunks, const int64_t* __restrict__ last_ls,
                                                   const uint8_t* __restrict__ any_hdr, int64_t* __restrict__ carry_ls,
                                                   uint8_t* __restrict__ carry_open) {
    __shared__ int64_t sh[32];
    __shared__ int64_t tot;
    const int64_t per = (n_chunks + blockDim.x - 1) / blockDim.x;
    const int64_t a = min((int64_t)threadIdx.x * per, n_chunks), b = min(a + per, n_chunks);
    int64_t m = -1, o = 0;
    for (int64_t c = a; c < b; c++) {
        m = max(m, last_ls[c]);
        o |= any_hdr[c];
    }
    int64_t em = block_scan_excl_op<int64_t>(m, -1, MaxOp(), sh, &tot);
    int64_t eo = block_scan_excl_op<int64_t>(o, 0, MaxOp(), sh, &tot);
    for (int64_t c = a; c < b; c++) {
        carry_ls[c] = em;
        carry_open[c] = (uint8_t)eo;
        em = max(em, last_ls[c]);
        eo |= any_hdr[c];
    }
}

// A thread's state at the start of its run: the line start in effect (and
// so whether its line is a header) and whether any header started before.
struct RunState {
    int64_t ls;
    bool hdr, open;
};

__device__ RunState run_state(const FaView& v, const uint8_t* sm, int64_t c0, int64_t a, int64_t b, int64_t carry_ls,
                              bool carry_open, int64_t* sh, int64_t* tot) {
    int64_t ls = -1, h = 0;
    for (int64_t i = a; i < b; i++)
        if (line_start(v, sm, c0, i)) {
            ls = i;
            h |= sm[i - c0] == '>';
        }
    const int64_t els = block_scan_excl_op<int64_t>(ls, -1, MaxOp(), sh, tot);
    const int64_t eh = block_scan_excl_op<int64_t>(h, 0, MaxOp(), sh, tot);
    RunState st;
    st.ls = max(carry_ls, els);
    st.hdr = st.ls >= 0 && (st.ls >= c0 ? sm[st.ls - c0] : v.d[st.ls]) == '>';
    st.open = carry_open || eh != 0;
    return st;
}

// Classifies byte i, advancing the state: 1 = a sequence byte kept, 2 = the
// first byte of a header line, 0 = neither. *bad is set for content before
// the first header.
__device__ __forceinline__ int classify(const FaView& v, const uint8_t* sm, int64_t c0, int64_t cend, int64_t i,
                                        RunState& st, bool* bad) {
    const uint8_t ch = sm[i - c0];
    int r = 0;
    if (line_start(v, sm, c0, i)) {
        st.ls = i;
        st.hdr = ch == '>';
        if (st.hdr) {
            st.open = true;
            r = 2;
        }
    }
    if (st.hdr || ch == '\n' || dropped_cr(v, sm, c0, cend, i)) return r;
    if (!st.open) {
        *bad = true;
        return 0;
    }
    return 1;
}

// Pass 3: per chunk, kept bytes and headers.
__global__ void __launch_bounds__(FA_THREADS) k_fa_count(FaView v, const int64_t* __restrict__ carry_ls,
                                                       const uint8_t* __restrict__ carry_open,
                                                       uint64_t* __restrict__ nkeep, uint32_t* __restrict__ nhdr,
                                                       uint32_t* __restrict__ flags) {
    __shared__ uint8_t sm[CHUNK];
    __shared__ int64_t sh[32];
    __shared__ int64_t tot;
    for (int64_t c = blockIdx.x; c < v.n_chunks; c += gridDim.x) {
        const int64_t c0 = c * CHUNK, cend = min(c0 + CHUNK, v.len);
        stage_chunk(v, c0, cend, sm);
        const int64_t a = c0 + (int64_t)threadIdx.x * FA_PER_THREAD, b = min(a + FA_PER_THREAD, cend);
        RunState st = run_state(v, sm, c0, a, b, carry_ls[c], carry_open[c] != 0, sh, &tot);
        int64_t k = 0, h = 0;
        bool bad = false;
        for (int64_t i = a; i < b; i++) {
            const int r = classify(v, sm, c0, cend, i, st, &bad);
            k += r == 1;
            h += r == 2;
        }
        if (bad) atomicOr(flags, (uint32_t)FA_TEXT_BEFORE_HEADER);
        block_scan_excl_op<int64_t>(k, 0, SumOp(), sh, &tot);
        const int64_t ck = tot;
        block_scan_excl_op<int64_t>(h, 0, SumOp(), sh, &tot);
        if (threadIdx.x == 0) {
            nkeep[c] = (uint64_t)ck;
            nhdr[c] = (uint32_t)tot;
        }
        __syncthreads();
    }
}

// Pass 5: the kept bytes at their place; each header's position and the
// sequence bytes before it.
__global__ void __launch_bounds__(FA_THREADS) k_fa_write(FaView v, const int64_t* __restrict__ carry_ls,
                                                       const uint8_t* __restrict__ carry_open,
                                                       const uint64_t* __restrict__ keep_off,
                                                       const uint32_t* __restrict__ hdr_off, uint8_t* __restrict__ out,
                                                       int64_t* __restrict__ hdr_pos, int64_t* __restrict__ hdr_seq) {
    __shared__ uint8_t sm[CHUNK];
    __shared__ uint8_t so[CHUNK];
    __shared__ int64_t sh[32];
    __shared__ int64_t tot;
    for (int64_t c = blockIdx.x; c < v.n_chunks; c += gridDim.x) {
        const int64_t c0 = c * CHUNK, cend = min(c0 + CHUNK, v.len);
        stage_chunk(v, c0, cend, sm);
        const int64_t a = c0 + (int64_t)threadIdx.x * FA_PER_THREAD, b = min(a + FA_PER_THREAD, cend);
        const RunState st0 = run_state(v, sm, c0, a, b, carry_ls[c], carry_open[c] != 0, sh, &tot);
        RunState st = st0;
        int64_t k = 0, h = 0;
        bool bad = false;
        for (int64_t i = a; i < b; i++) {
            const int r = classify(v, sm, c0, cend, i, st, &bad);
            k += r == 1;
            h += r == 2;
        }
        const int64_t kb = block_scan_excl_op<int64_t>(k, 0, SumOp(), sh, &tot);
        const int64_t ck = tot;
        const int64_t hb = block_scan_excl_op<int64_t>(h, 0, SumOp(), sh, &tot);
        st = st0;
        int64_t kk = kb, hh = (int64_t)hdr_off[c] + hb;
        for (int64_t i = a; i < b; i++) {
            const int r = classify(v, sm, c0, cend, i, st, &bad);
            if (r == 1) {
                so[kk++] = sm[i - c0];
            } else if (r == 2) {
                hdr_pos[hh] = i;
                hdr_seq[hh] = (int64_t)keep_off[c] + kk;
                hh++;
            }
        }
        __syncthreads();
        uint8_t* dst = out + keep_off[c];
        for (int64_t j = threadIdx.x; j < ck; j += blockDim.x) dst[j] = so[j];
        __syncthreads();
    }
}

// Pass 6: a header's name: after '>' up to the first space or tab, within
// the line without its dropped '\r'.
__device__ void name_span(const FaView& v, int64_t h, int64_t* s, int64_t* e) {
    int64_t i = h + 1;
    while (i < v.len && v.d[i] != '\n') i++;
    int64_t end = i;  // the line's end
    if (end > h + 1 && v.d[end - 1] == '\r') end--;
    int64_t j = h + 1;
    while (j < end && v.d[j] != ' ' && v.d[j] != '\t') j++;
    *s = h + 1;
    *e = j;
}

__global__ void k_fa_name_len(FaView v, const int64_t* __restrict__ hdr_pos, int64_t n, uint64_t* __restrict__ len) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        int64_t s, e;
        name_span(v, hdr_pos[r], &s, &e);
        len[r] = (uint64_t)(e - s + 1);  // with its '\n' separator
    }
}

__global__ void k_fa_name_write(FaView v, const int64_t* __restrict__ hdr_pos, int64_t n,
                                const uint64_t* __restrict__ off, char* __restrict__ names) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        int64_t s, e;
        name_span(v, hdr_pos[r], &s, &e);
        char* o = names + off[r];
        for (int64_t i = s; i < e; i++) *o++ = (char)v.d[i];
        *o = r + 1 < n ? '\n' : '\0';
    }
}

// ---------------------------------------------------------------- FASTQ
// Records of four lines (needletail's FASTQ, src/io/mod.rs:383-427): '@'
// header, sequence, '+' line, quality. A byte's role follows from the index
// of its line, counted from the file's start: the lines are counted per
// chunk, scanned over the chunks, and within a chunk over the threads' runs.
// A line 4r must start with '@' and a line 4r+2 with '+' (when not empty),
// else the file is refused and read on the host. Blank lines at the file's
// end are dropped first; a last record left without its quality (it was
// empty) or its '+' line reads as the host reader reads it: an empty or
// missing line.
enum : uint32_t { FQ_BAD = 4u };

// Pass 1: newlines per chunk.
__global__ void __launch_bounds__(FA_THREADS) k_fq_lines(FaView v, uint64_t* __restrict__ nl) {
    __shared__ uint8_t sm[CHUNK];
    __shared__ int64_t sh[32];
    __shared__ int64_t tot;
    for (int64_t c = blockIdx.x; c < v.n_chunks; c += gridDim.x) {
        const int64_t c0 = c * CHUNK, cend = min(c0 + CHUNK, v.len);
        stage_chunk(v, c0, cend, sm);
        const int64_t a = c0 + (int64_t)threadIdx.x * FA_PER_THREAD, b = min(a + FA_PER_THREAD, cend);
        int64_t k = 0;
        for (int64_t i = a; i < b; i++) k += sm[i - c0] == '\n';
        block_scan_excl_op<int64_t>(k, 0, SumOp(), sh, &tot);
        if (threadIdx.x == 0) nl[c] = (uint64_t)tot;
        __syncthreads();
    }
}

// The index of the line a thread's run starts in (from the chunk's first
// line's index and the newlines of the runs before it in the chunk).
__device__ int64_t fq_run_line(const uint8_t* sm, int64_t c0, int64_t a, int64_t b, uint64_t chunk_line, int64_t* sh,
                               int64_t* tot) {
    int64_t k = 0;
    for (int64_t i = a; i < b; i++) k += sm[i - c0] == '\n';
    return (int64_t)chunk_line + block_scan_excl_op<int64_t>(k, 0, SumOp(), sh, tot);
}

// Byte i of line `line`: 1 = a sequence byte kept, 2 = the first byte of a
// header line, 0 = neither; *bad for a line that breaks the record layout.
__device__ __forceinline__ int fq_classify(const FaView& v, const uint8_t* sm, int64_t c0, int64_t cend, int64_t i,
                                           int64_t& line, bool* bad) {
    const uint8_t ch = sm[i - c0];
    int r = 0;
    if (ch == '\n') {
        line++;
        return 0;
    }
    const int role = (int)(line & 3);
    if (line_start(v, sm, c0, i)) {
        if (role == 0) {
            if (ch == '@') r = 2;
            else *bad = true;
        } else if (role == 2 && ch != '+') {
            *bad = true;
        }
    }
    if (role == 1 && !dropped_cr(v, sm, c0, cend, i)) return 1;
    return r;
}

// Pass 2: kept bytes and headers per chunk.
__global__ void __launch_bounds__(FA_THREADS) k_fq_count(FaView v, const uint64_t* __restrict__ nl_off,
                                                       uint64_t* __restrict__ nkeep, uint32_t* __restrict__ nhdr,
                                                       uint32_t* __restrict__ flags) {
    __shared__ uint8_t sm[CHUNK];
    __shared__ int64_t sh[32];
    __shared__ int64_t tot;
    for (int64_t c = blockIdx.x; c < v.n_chunks; c += gridDim.x) {
        const int64_t c0 = c * CHUNK, cend = min(c0 + CHUNK, v.len);
        stage_chunk(v, c0, cend, sm);
        const int64_t a = c0 + (int64_t)threadIdx.x * FA_PER_THREAD, b = min(a + FA_PER_THREAD, cend);
        int64_t line = fq_run_line(sm, c0, a, b, nl_off[c], sh, &tot);
        int64_t k = 0, h = 0;
        bool bad = false;
        for (int64_t i = a; i < b; i++) {
            const int r = fq_classify(v, sm, c0, cend, i, line, &bad);
            k += r == 1;
            h += r == 2;
        }
        if (bad) atomicOr(flags, (uint32_t)FQ_BAD);
        block_scan_excl_op<int64_t>(k, 0, SumOp(), sh, &tot);
        const int64_t ck = tot;
        block_scan_excl_op<int64_t>(h, 0, SumOp(), sh, &tot);
        if (threadIdx.x == 0) {
            nkeep[c] = (uint64_t)ck;
            nhdr[c] = (uint32_t)tot;
        }
        __syncthreads();
    }
}

// Pass 3: the kept bytes at their place; each header's position and the
// sequence bytes before it.
__global__ void __launch_bounds__(FA_THREADS) k_fq_write(FaView v, const uint64_t* __restrict__ nl_off,
                                                       const uint64_t* __restrict__ keep_off,
                                                       const uint32_t* __restrict__ hdr_off, uint8_t* __restrict__ out,
                                                       int64_t* __restrict__ hdr_pos, int64_t* __restrict__ hdr_seq) {
    __shared__ uint8_t sm[CHUNK];
    __shared__ uint8_t so[CHUNK];
    __shared__ int64_t sh[32];
    __shared__ int64_t tot;
    for (int64_t c = blockIdx.x; c < v.n_chunks; c += gridDim.x) {
        const int64_t c0 = c * CHUNK, cend = min(c0 + CHUNK, v.len);
        stage_chunk(v, c0, cend, sm);
        const int64_t a = c0 + (int64_t)threadIdx.x * FA_PER_THREAD, b = min(a + FA_PER_THREAD, cend);
        const int64_t line0 = fq_run_line(sm, c0, a, b, nl_off[c], sh, &tot);
        int64_t line = line0, k = 0, h = 0;
        bool bad = false;
        for (int64_t i = a; i < b; i++) {
            const int r = fq_classify(v, sm, c0, cend, i, line, &bad);
            k += r == 1;
            h += r == 2;
        }
        const int64_t kb = block_scan_excl_op<int64_t>(k, 0, SumOp(), sh, &tot);
        const int64_t ck = tot;
        const int64_t hb = block_scan_excl_op<int64_t>(h, 0, SumOp(), sh, &tot);
        line = line0;
        int64_t kk = kb, hh = (int64_t)hdr_off[c] + hb;
        for (int64_t i = a; i < b; i++) {
            const int r = fq_classify(v, sm, c0, cend, i, line, &bad);
            if (r == 1) {
                so[kk++] = sm[i - c0];
            } else if (r == 2) {
                hdr_pos[hh] = i;
                hdr_seq[hh] = (int64_t)keep_off[c] + kk;
                hh++;
            }
        }
        __syncthreads();
        uint8_t* dst = out + keep_off[c];
        for (int64_t j = threadIdx.x; j < ck; j += blockDim.x) dst[j] = so[j];
        __syncthreads();
    }
}

}  // namespace

FastaDev* fasta_parse_device(int device, cudaStream_t s, const uint8_t* file, int64_t len, std::string* why) {
    SHM_CUDA(cudaSetDevice(device));
    auto* F = new FastaDev();
    try {
        FaView v{};
        // FASTQ when the file starts with '@'; its blank lines at the end are
        // not part of any record
        const bool fastq = len > 0 && file[0] == '@';
        if (fastq)
            while (len > 0 && (file[len - 1] == '\n' || file[len - 1] == '\r')) len--;
        DevBuf<uint8_t> raw;
        raw.reserve((size_t)len + 1);
        if (len) SHM_CUDA(cudaMemcpyAsync(raw.p, file, (size_t)len, cudaMemcpyHostToDevice, s));
        v.d = raw.p;
        v.len = len;
        v.n_chunks = (len + CHUNK - 1) / CHUNK;
        const int64_t nc = v.n_chunks;
        DevBuf<int64_t> last_ls, carry_ls;
        DevBuf<uint8_t> any_hdr, carry_open;
        DevBuf<uint64_t> nkeep, keep_off;
        DevBuf<uint32_t> nhdr, hdr_off, flags;
        last_ls.reserve((size_t)nc + 1);
        carry_ls.reserve((size_t)nc + 1);
        any_hdr.reserve((size_t)nc + 1);
        carry_open.reserve((size_t)nc + 1);
        nkeep.reserve((size_t)nc + 1);
        keep_off.reserve((size_t)nc + 1);
        nhdr.reserve((size_t)nc + 1);
        hdr_off.reserve((size_t)nc + 1);
        flags.reserve(1);
        SHM_CUDA(cudaMemsetAsync(flags.p, 0, sizeof(uint32_t), s));
        const int grid = grid_for((size_t)std::max<int64_t>(nc, 1), 1, 4);
        uint64_t total = 0;
        uint32_t n_rec = 0, fl = 0;
        DevBuf<uint64_t> nl, nl_off;
        if (fastq) {
            nl.reserve((size_t)nc + 1);
            nl_off.reserve((size_t)nc + 1);
            uint64_t lines = 0;
            k_fq_lines<<<grid, FA_THREADS, 0, s>>>(v, nl.p);
            SHM_CUDA(cudaGetLastError());
            exclusive_scan_u64(nl.p, nl_off.p, (size_t)nc, s);
            k_fq_count<<<grid, FA_THREADS, 0, s>>>(v, nl_off.p, nkeep.p, nhdr.p, flags.p);
            SHM_CUDA(cudaGetLastError());
            exclusive_scan_u64(nkeep.p, keep_off.p, (size_t)nc, s);
            exclusive_scan_u32(nhdr.p, hdr_off.p, (size_t)nc, s);
            count_launch(2);
            SHM_CUDA(cudaMemcpyAsync(&lines, nl_off.p + nc, sizeof lines, cudaMemcpyDeviceToHost, s));
            SHM_CUDA(cudaMemcpyAsync(&total, keep_off.p + nc, sizeof total, cudaMemcpyDeviceToHost, s));
            SHM_CUDA(cudaMemcpyAsync(&n_rec, hdr_off.p + nc, sizeof n_rec, cudaMemcpyDeviceToHost, s));
            SHM_CUDA(cudaMemcpyAsync(&fl, flags.p, sizeof fl, cudaMemcpyDeviceToHost, s));
            SHM_CUDA(cudaStreamSynchronize(s));
            (void)lines;  // a last record may end early (an empty quality line looks like a trailing blank)
            if (fl & FQ_BAD) {
                *why = "not FASTQ records of four lines";
                delete F;
                return nullptr;
            }
        } else if (nc) {
            k_fa_marks<<<grid, FA_THREADS, 0, s>>>(v, last_ls.p, any_hdr.p, flags.p);
            SHM_CUDA(cudaGetLastError());
            k_fa_carry<<<1, 1024, 0, s>>>(nc, last_ls.p, any_hdr.p, carry_ls.p, carry_open.p);
            SHM_CUDA(cudaGetLastError());
            k_fa_count<<<grid, FA_THREADS, 0, s>>>(v, carry_ls.p, carry_open.p, nkeep.p, nhdr.p, flags.p);
            SHM_CUDA(cudaGetLastError());
            exclusive_scan_u64(nkeep.p, keep_off.p, (size_t)nc, s);
            exclusive_scan_u32(nhdr.p, hdr_off.p, (size_t)nc, s);
            count_launch(3);
            SHM_CUDA(cudaMemcpyAsync(&total, keep_off.p + nc, sizeof total, cudaMemcpyDeviceToHost, s));
            SHM_CUDA(cudaMemcpyAsync(&n_rec, hdr_off.p + nc, sizeof n_rec, cudaMemcpyDeviceToHost, s));
            SHM_CUDA(cudaMemcpyAsync(&fl, flags.p, sizeof fl, cudaMemcpyDeviceToHost, s));
            SHM_CUDA(cudaStreamSynchronize(s));
        }
        if (fl & FA_FASTQ) {
            *why = "a line starts with '@' (FASTQ records are read on the host)";
            delete F;
            return nullptr;
        }
        if (fl & FA_TEXT_BEFORE_HEADER) {
            *why = "text before the first '>' header";
            delete F;
            return nullptr;
        }
        F->device = device;
        F->seq.reserve((size_t)total + 32);
        SHM_CUDA(cudaMemsetAsync(F->seq.p + total, 0, 32, s));
        F->offs.assign((size_t)n_rec + 1, (int64_t)total);
        if (n_rec) {
            DevBuf<int64_t> hdr_pos, hdr_seq;
            hdr_pos.reserve(n_rec);
            hdr_seq.reserve(n_rec);
            if (fastq)
                k_fq_write<<<grid, FA_THREADS, 0, s>>>(v, nl_off.p, keep_off.p, hdr_off.p, F->seq.p, hdr_pos.p,
                                                       hdr_seq.p);
            else
                k_fa_write<<<grid, FA_THREADS, 0, s>>>(v, carry_ls.p, carry_open.p, keep_off.p, hdr_off.p, F->seq.p,
                                                       hdr_pos.p, hdr_seq.p);
            SHM_CUDA(cudaGetLastError());
            DevBuf<uint64_t> nlen, noff;
            nlen.reserve(n_rec);
            noff.reserve((size_t)n_rec + 1);
            const int g2 = grid_for(n_rec, 128, 8);
            k_fa_name_len<<<g2, 128, 0, s>>>(v, hdr_pos.p, n_rec, nlen.p);
            SHM_CUDA(cudaGetLastError());
            exclusive_scan_u64(nlen.p, noff.p, n_rec, s);
            uint64_t nbytes = 0;
            SHM_CUDA(cudaMemcpyAsync(&nbytes, noff.p + n_rec, sizeof nbytes, cudaMemcpyDeviceToHost, s));
            SHM_CUDA(cudaStreamSynchronize(s));
            DevBuf<char> names;
            names.reserve((size_t)nbytes + 1);
            k_fa_name_write<<<g2, 128, 0, s>>>(v, hdr_pos.p, n_rec, noff.p, names.p);
            SHM_CUDA(cudaGetLastError());
            count_launch(3);
            F->names.resize((size_t)nbytes);
            SHM_CUDA(cudaMemcpyAsync(&F->names[0], names.p, (size_t)nbytes, cudaMemcpyDeviceToHost, s));
            SHM_CUDA(cudaMemcpyAsync(F->offs.data(), hdr_seq.p, sizeof(int64_t) * n_rec, cudaMemcpyDeviceToHost, s));
            SHM_CUDA(cudaStreamSynchronize(s));
            if (!F->names.empty()) F->names.pop_back();  // the last name's terminator
            // names as String::from_utf8_lossy gives them (src/io/mod.rs:408-410)
            bool ascii = true;
            for (char ch : F->names) ascii = ascii && (unsigned char)ch < 0x80;
            if (!ascii) F->names = utf8_lossy(F->names);
        }
        F->n = (int32_t)n_rec;
        return F;
    } catch (...) {
        delete F;
        throw;
    }
}

}  // namespace shm
