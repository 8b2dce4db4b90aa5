// PAF text on the device: the same bytes as shm_format_paf (host/paf.cpp),
// which restates the reference's MappingPaf / LocalMappingStats /
// GlobalMappingStats Display impls (src/mapping.rs:87-107, 161-182, 228-247)
// and the set_second_best / calc_mapq / set_global_stats post-processing
// (src/mapping.rs:329-408). One thread per read renders its line twice: once
// to measure it, then, after a scan of the lengths, into its place in the
// output. Unmapped reads print nothing.
//
// Fixed-point f64 ({:.N}, N = 3 or 5) is exact, rounding half to even like
// the host's printf: x = m 2^e, so x 10^N = m 5^N 2^(e+N), an integer
// times a power of two. For e + N < 0 it is shifted right in 128-bit integer
// arithmetic and rounded on the bits shifted out; for e + N >= 0 it is the
// integer m 5^N 2^(e+N), and values too large for 128 bits are printed from
// a multi-word integer.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>
#include <thread>
#include <functional>
#include <exception>

#include "shm_common.cuh"
#include "shm_internal.hpp"
#include "shm_map.cuh"
#include "shm_paf.hpp"
#include "shm_prims.cuh"

namespace shm {

namespace {

typedef unsigned __int128 u128;

// Appends to the line, or only counts when p is null.
struct Out {
    char* p;
    int64_t n;
    __device__ void c(char ch) {
        if (p) p[n] = ch;
        n++;
    }
    __device__ void s(const char* z) {
        while (*z) c(*z++);
    }
    __device__ void mem(const char* a, int64_t len) {
        for (int64_t i = 0; i < len; i++) c(a[i]);
    }
};

// Decimal digits with the narrowest arithmetic the value allows (a digit of
// a 128-bit value costs a software division).
__device__ void put_u128(Out& o, u128 v) {
    char d[40];
    int k = 0;
    while (v >> 64) {
        d[k++] = (char)('0' + (int)(v % 10));
        v /= 10;
    }
    uint64_t w = (uint64_t)v;
    while (w >> 32) {
        d[k++] = (char)('0' + (int)(w % 10));
        w /= 10;
    }
    uint32_t x = (uint32_t)w;
    do {
        d[k++] = (char)('0' + x % 10);
        x /= 10;
    } while (x);
    while (k) o.c(d[--k]);
}

__device__ void put_i(Out& o, int64_t v) {
    if (v < 0) {
        o.c('-');
        put_u128(o, (u128)(-(v + 1)) + 1);
    } else {
        put_u128(o, (u128)v);
    }
}

// m 2^e (e >= 0) in decimal, for values of 2^127 and more: 32-bit words,
// divided by 10^9 repeatedly.
__device__ void put_big(Out& o, uint64_t m, int e) {
    uint32_t w[36];
    int nw = 0;
    for (int i = 0; i < 36; i++) w[i] = 0;
    const int ws = e >> 5, bs = e & 31;
    const u128 sh = (u128)m << bs;  // at most 53 + 31 bits
    w[ws] = (uint32_t)sh;
    w[ws + 1] = (uint32_t)(sh >> 32);
    w[ws + 2] = (uint32_t)(sh >> 64);
    nw = ws + 3;
    uint32_t chunk[40];
    int nc = 0;
    while (nw > 0) {
        uint64_t rem = 0;
        for (int i = nw - 1; i >= 0; i--) {
            const uint64_t cur = (rem << 32) | w[i];
            w[i] = (uint32_t)(cur / 1000000000u);
            rem = cur % 1000000000u;
        }
        chunk[nc++] = (uint32_t)rem;
        while (nw > 0 && w[nw - 1] == 0) nw--;
    }
    put_u128(o, chunk[nc - 1]);
    for (int i = nc - 2; i >= 0; i--) {
        char d[9];
        uint32_t v = chunk[i];
        for (int j = 8; j >= 0; j--) {
            d[j] = (char)('0' + v % 10);
            v /= 10;
        }
        o.mem(d, 9);
    }
}

// Rust {:.prec} / printf %.*f of x (prec 3 or 5): NaN, inf and -inf as
// the host prints them; otherwise exactly rounded, half to even.
__device__ void put_f(Out& o, double x, int prec) {
    if (isnan(x)) {
        o.s("NaN");
        return;
    }
    if (isinf(x)) {
        o.s(x > 0 ? "inf" : "-inf");
        return;
    }
    const uint64_t bits = (uint64_t)__double_as_longlong(x);
    if (bits >> 63) o.c('-');
    const int E = (int)((bits >> 52) & 0x7ff);
    const uint64_t F = bits & ((1ULL << 52) - 1);
    const uint64_t m = E ? (F | (1ULL << 52)) : F;
    const int e = E ? E - 1075 : -1074;
    const uint64_t p5 = prec == 3 ? 125u : 3125u;
    const uint64_t p10 = prec == 3 ? 1000u : 100000u;
    if (e > 56) {  // an integer of 2^109 or more: beyond the 128-bit form below
        put_big(o, m, e);
        o.c('.');
        for (int i = 0; i < prec; i++) o.c('0');
        return;
    }
    const u128 M = (u128)m * p5;  // x 10^prec = M 2^s
    const int s = e + prec;
    u128 N;
    if (s >= 0) {
        N = M << s;  // M < 2^65 and s <= 61: below 2^126
    } else if (-s >= 127) {
        N = 0;  // x 10^prec < 2^65 2^-127: below one half
    } else {
        const int r = -s;
        N = M >> r;
        const u128 rem = M & (((u128)1 << r) - 1), half = (u128)1 << (r - 1);
        if (rem > half || (rem == half && (N & 1))) N += 1;
    }
    uint32_t f;
    if (N >> 64) {
        put_u128(o, N / p10);
        f = (uint32_t)(N % p10);
    } else {
        const uint64_t n64 = (uint64_t)N;
        put_u128(o, n64 / p10);
        f = (uint32_t)(n64 % p10);
    }
    o.c('.');
    char d[5];
    for (int j = prec - 1; j >= 0; j--) {
        d[j] = (char)('0' + f % 10);
        f /= 10;
    }
    o.mem(d, prec);
}

struct PafView {
    const shm_map_record* rec;
    int32_t n;
    const char* qnames;      // joined query names
    const int64_t* qse;      // name i is qnames[qse[2i], qse[2i+1])
    const char* snames;      // joined segment names
    const int64_t* soff;     // n_seg+1, likewise
    const int32_t* slen;     // segment lengths
    const double* map_time;  // per read, or null (0.0)
    int32_t k;
    double theta, min_diff;
};

// One read's line (host/paf.cpp render, in the same order and arithmetic).
__device__ void render(Out& o, const PafView& v, int32_t i) {
    const shm_map_record r = v.rec[i];
    if (r.status != 0) return;
    double j2 = -1.0, sigmas = -1.0;
    int32_t i2 = -1, b2s = -1, b2b = -1;
    if (r.has_second) {
        j2 = r.score2;
        i2 = r.intersection2;
        b2s = r.bucket2_seg;
        b2b = r.bucket2_b;
        const double x = (double)(i2 == -1 ? 0 : i2), y = (double)(r.intersection == -1 ? 0 : r.intersection);
        sigmas = __ddiv_rn(fabs(__dsub_rn(x, y)), __dsqrt_rn(__dadd_rn(x, y)));  // mapping.rs:329-333
    }
    const double theta2 = __dsub_rn(v.theta, v.min_diff);  // calc_mapq (mapping.rs:341-354)
    if (j2 < theta2) j2 = theta2;
    const double frac = __dsub_rn(1.0, __ddiv_rn(j2, r.score));
    const int32_t mapq_strand = abs(r.same_strand) < r.intersection / 2 ? 5 : 60;
    const int mapq = frac > v.min_diff ? (mapq_strand < 60 ? mapq_strand : 60) : 0;
    o.mem(v.qnames + v.qse[2 * i], v.qse[2 * i + 1] - v.qse[2 * i]);
    o.c('\t');
    put_i(o, r.read_len);
    o.c('\t');
    put_i(o, r.p_start);
    o.c('\t');
    put_i(o, r.p_end);
    o.c('\t');
    o.c(r.same_strand > 0 ? '+' : '-');
    o.c('\t');
    o.mem(v.snames + v.soff[r.segm_id], v.soff[r.segm_id + 1] - v.soff[r.segm_id]);
    o.c('\t');
    put_i(o, v.slen[r.segm_id]);
    o.c('\t');
    put_i(o, r.t_l);
    o.c('\t');
    put_i(o, r.t_r);
    o.c('\t');
    put_i(o, r.read_len);
    o.c('\t');
    put_i(o, r.read_len);
    o.c('\t');
    put_i(o, mapq);
    o.s("\tp:i:");
    put_i(o, r.sketch_size);
    o.s("\ts:i:");
    put_i(o, r.s_sz);
    o.s("\tI:i:");
    put_i(o, r.intersection);
    o.s("\tI2:i:");
    put_i(o, i2);
    o.s("\tIdiff:i:");
    put_i(o, (int32_t)(r.intersection - i2));
    o.s("\tIsdiff:f:");
    put_f(o, sigmas, 5);
    o.s("\tJ:f:");
    put_f(o, r.score, 5);
    o.s("\tJ2:f:");
    put_f(o, j2, 5);
    o.s("\tJdiff:f:");
    put_f(o, __dsub_rn(r.score, j2), 5);
    o.s("\tsh:f:");
    put_f(o, r.sh, 5);
    o.s("\tstrand:i:");
    put_i(o, r.same_strand);
    o.s("\tt:f:");
    put_f(o, v.map_time ? v.map_time[i] : 0.0, 5);
    o.s("\tb:s:(");
    put_i(o, r.bucket_seg);
    o.c(',');
    put_i(o, r.bucket_b);
    o.s(")\tb2:s:(");
    put_i(o, b2s);
    o.c(',');
    put_i(o, b2b);
    o.s(")\tk:i:");
    put_i(o, v.k);
    o.s("\tgt_J:f:-1.000\tgt_C:f:-1.000\tgt_C_bucket:f:-1.000\tseeds:i:");
    put_i(o, r.seeds);
    o.s("\tmax_seed_matches:i:");
    put_i(o, r.max_seed_matches);
    o.s("\tseed_matches:i:");
    put_i(o, r.seed_matches);
    o.s("\ttotal_matches:i:");
    put_i(o, r.total_matches);
    o.s("\tmatch_inefficiency:f:");
    put_f(o, __ddiv_rn((double)r.total_matches, (double)r.intersection), 3);
    o.s("\tseeded_buckets:i:");
    put_i(o, r.seeded_buckets);
    o.s("\tfinal_buckets:i:");
    put_i(o, r.final_buckets);
    o.s("\tFPTP:f:-1.000\n");
}

__global__ void k_paf_len(PafView v, uint64_t* __restrict__ len) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < v.n; i += gridDim.x * blockDim.x) {
        Out o{nullptr, 0};
        render(o, v, i);
        len[i] = (uint64_t)o.n;
    }
}

__global__ void k_paf_write(PafView v, const uint64_t* __restrict__ off, char* __restrict__ text) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < v.n; i += gridDim.x * blockDim.x) {
        Out o{text + off[i], 0};
        render(o, v, i);
    }
}

// Lines of a batch at their places in one text buffer: line i at base +
// off[i], where base (device) is the length of the batches' text before this
// one. A line that would end past cap is not written; *overflow is set.
__global__ void k_paf_write_at(PafView v, const uint64_t* __restrict__ off, const uint64_t* __restrict__ base,
                               char* __restrict__ text, uint64_t cap, uint32_t* __restrict__ overflow) {
    const uint64_t b0 = *base;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < v.n; i += gridDim.x * blockDim.x) {
        const uint64_t at = b0 + off[i], end = b0 + off[i + 1];
        if (end == at) continue;
        if (end > cap) {
            atomicOr(overflow, 1u);
            continue;
        }
        Out o{text + at, 0};
        render(o, v, i);
    }
}

// The text of the batch just written moves the base past it.
__global__ void k_paf_advance(uint64_t* __restrict__ base, const uint64_t* __restrict__ off, int32_t n,
                              uint64_t* __restrict__ range) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const uint64_t a = *base;
        *base = a + off[n];
        if (range) {  // the batch's text span
            range[0] = a;
            range[1] = a + off[n];
        }
    }
}


}  // namespace

struct PafScratch {
    DevBuf<shm_map_record> rec;
    DevBuf<char> q, sn, text;
    DevBuf<int64_t> qse, soff;
    DevBuf<int32_t> slen;
    DevBuf<double> mt;
    DevBuf<uint64_t> len, off, base;
    DevBuf<uint32_t> flag;
    shm_map_record* h_rec = nullptr;  // pinned records of shm_map_paf calls that pass none
    size_t h_rec_cap = 0;
    uint64_t* h_small = nullptr;  // pinned readback: text length, overflow flag
    DevBuf<uint64_t> ranges;      // per batch of a shm_map_paf call: its text span
    cudaStream_t ns = nullptr;    // the names' upload of a shm_map_paf call, beside its first batch
    cudaEvent_t nev = nullptr;
    int64_t names_h2d = 0;        // bytes of the last names upload
    uint64_t* h_ranges = nullptr; // the text spans, pinned, read once the batch's event completes
    size_t h_ranges_cap = 0;      // (pairs)
    std::vector<cudaEvent_t> evs; // one per batch in flight
    cudaStream_t ts = nullptr;    // the text's copies to the caller's buffer, batch by batch
    ~PafScratch() {
        if (h_rec) cudaFreeHost(h_rec);
        if (h_small) cudaFreeHost(h_small);
        if (ts) {
            cudaStreamSynchronize(ts);
            cudaStreamDestroy(ts);
        }
        for (cudaEvent_t e : evs) cudaEventDestroy(e);
        if (h_ranges) cudaFreeHost(h_ranges);
        if (ns) {
            cudaStreamSynchronize(ns);
            cudaStreamDestroy(ns);
        }
        if (nev) cudaEventDestroy(nev);
    }
};

void paf_scratch_free(PafScratch* p) { delete p; }

static PafScratch& paf_scratch(MapCtx* c) {
    if (!c->paf) c->paf = new PafScratch();
    return *c->paf;
}

// Query names split on '\n' as shm_format_paf does (name i is q[qse[2i],
// qse[2i+1])), the segment names joined with their offsets. names_view
// sizes the device buffers and returns the view of them (records, count and
// map times unset); names_upload fills them on stream s (the host work: a
// scan of the names and pageable copies), from any host thread.
static PafView names_view(PafScratch& P, const IndexStorage& ix, const shm_params& p, int32_t n, size_t qlen) {
    size_t sn = 0;
    for (const std::string& x : ix.names) sn += x.size();
    P.q.reserve(qlen + 1);
    P.sn.reserve(sn + 1);
    P.qse.reserve(2 * (size_t)n + 1);
    P.soff.reserve(ix.names.size() + 1);
    P.slen.reserve(ix.seg_len.size() + 1);
    P.len.reserve((size_t)n + 1);
    P.off.reserve((size_t)n + 1);
    PafView v{};
    v.qnames = P.q.p;
    v.qse = P.qse.p;
    v.snames = P.sn.p;
    v.soff = P.soff.p;
    v.slen = P.slen.p;
    v.k = p.k;
    v.theta = p.theta;
    v.min_diff = p.min_diff;
    return v;
}

static void names_upload(MapCtx* c, PafScratch& P, const IndexStorage& ix, int32_t n, const char* names, size_t qlen,
                         cudaStream_t s) {
    const char* q = names ? names : "";
    std::vector<int64_t> qse(2 * (size_t)n + 1, 0);
    for (size_t i = 0, at = 0; i < (size_t)n; i++) {
        const char* e = (const char*)std::memchr(q + at, '\n', qlen - at);
        const size_t end = e ? (size_t)(e - q) : qlen;
        qse[2 * i] = (int64_t)at;
        qse[2 * i + 1] = (int64_t)end;
        at = e ? end + 1 : end;
    }
    std::string sn;
    std::vector<int64_t> soff(1, 0);
    for (const std::string& x : ix.names) {
        sn += x;
        soff.push_back((int64_t)sn.size());
    }
    if (qlen) SHM_CUDA(cudaMemcpyAsync(P.q.p, q, qlen, cudaMemcpyHostToDevice, s));
    if (!sn.empty()) SHM_CUDA(cudaMemcpyAsync(P.sn.p, sn.data(), sn.size(), cudaMemcpyHostToDevice, s));
    SHM_CUDA(cudaMemcpyAsync(P.qse.p, qse.data(), sizeof(int64_t) * qse.size(), cudaMemcpyHostToDevice, s));
    SHM_CUDA(cudaMemcpyAsync(P.soff.p, soff.data(), sizeof(int64_t) * soff.size(), cudaMemcpyHostToDevice, s));
    if (!ix.seg_len.empty())
        SHM_CUDA(cudaMemcpyAsync(P.slen.p, ix.seg_len.data(), sizeof(int32_t) * ix.seg_len.size(),
                                 cudaMemcpyHostToDevice, s));
    // the query and segment names and their offset tables (counted by the caller's thread)
    P.names_h2d = (int64_t)(qlen + sn.size() + sizeof(int64_t) * (qse.size() + soff.size()) +
                            sizeof(int32_t) * ix.seg_len.size());
}

// Both, on stream s.
static PafView upload_names(MapCtx* c, PafScratch& P, const IndexStorage& ix, const shm_params& p, int32_t n,
                            const char* names, cudaStream_t s) {
    const size_t qlen = std::strlen(names ? names : "");
    PafView v = names_view(P, ix, p, n, qlen);
    names_upload(c, P, ix, n, names, qlen, s);
    c->work[W_H2D_BYTES] += P.names_h2d;
    return v;
}

int64_t format_paf_device(MapCtx* c, const IndexStorage& ix, const shm_params& p, const shm_map_record* rec,
                          int32_t n, const char* names, const double* map_time, char* buf, int64_t cap) {
    SHM_CUDA(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    PafScratch& P = paf_scratch(c);
    P.rec.reserve((size_t)std::max(n, 1));
    if (map_time && n) P.mt.reserve((size_t)n);
    PafView v = upload_names(c, P, ix, p, n, names, s);
    if (n) SHM_CUDA(cudaMemcpyAsync(P.rec.p, rec, sizeof(shm_map_record) * (size_t)n, cudaMemcpyHostToDevice, s));
    if (map_time && n)
        SHM_CUDA(cudaMemcpyAsync(P.mt.p, map_time, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, s));
    c->work[W_H2D_BYTES] += (int64_t)((sizeof(shm_map_record) + (map_time ? sizeof(double) : 0)) * (size_t)n);
    v.rec = P.rec.p;
    v.n = n;
    v.map_time = map_time && n ? P.mt.p : nullptr;
    int64_t total = 0;
    if (n) {
        k_paf_len<<<grid_for((size_t)n, 128, 8), 128, 0, s>>>(v, P.len.p);
        SHM_CUDA(cudaGetLastError());
        count_launch();
        exclusive_scan_u64(P.len.p, P.off.p, (size_t)n, s);
        uint64_t tot = 0;
        SHM_CUDA(cudaMemcpyAsync(&tot, P.off.p + n, sizeof tot, cudaMemcpyDeviceToHost, s));
        SHM_CUDA(cudaStreamSynchronize(s));
        total = (int64_t)tot;
    }
    if (buf && cap > 0 && total > 0) {
        P.text.reserve((size_t)total);
        k_paf_write<<<grid_for((size_t)n, 128, 8), 128, 0, s>>>(v, P.off.p, P.text.p);
        SHM_CUDA(cudaGetLastError());
        count_launch();
        const int64_t take = std::min(cap, total);
        SHM_CUDA(cudaMemcpyAsync(buf, P.text.p, (size_t)take, cudaMemcpyDeviceToHost, s));
        c->work[W_D2H_BYTES] += take;
        SHM_CUDA(cudaStreamSynchronize(s));
    }
    return total;
}

namespace {

// Renders each batch's lines as soon as its records are on the device, into
// one text buffer, in read order.
struct PafSink : BatchSink {
    MapCtx* c;
    PafScratch* P;
    PafView v0;
    uint64_t cap;
    char* hbuf = nullptr;  // the caller's buffer when it is pinned (each batch's text copied as it is done)
    uint64_t hcap = 0;
    int32_t nb = 0;        // batches rendered
    int32_t ncopied = 0;   // batches whose text copy is queued
    std::function<void()> names_ready;  // waits for the names' upload (once, before the first kernel)
    void batch(int32_t i, int32_t j, const shm_map_record* d_rec, cudaStream_t s) override {
        const int32_t n = j - i;
        if (n <= 0) return;
        if (names_ready) {
            names_ready();
            names_ready = nullptr;
        }
        PafView v = v0;
        v.rec = d_rec;
        v.n = n;
        v.qse = P->qse.p + 2 * (size_t)i;
        k_paf_len<<<grid_for((size_t)n, 128, 8), 128, 0, s>>>(v, P->len.p);
        SHM_CUDA(cudaGetLastError());
        count_launch();
        exclusive_scan_u64(P->len.p, P->off.p, (size_t)n, s);
        k_paf_write_at<<<grid_for((size_t)n, 128, 8), 128, 0, s>>>(v, P->off.p, P->base.p, P->text.p, cap,
                                                                   P->flag.p);
        SHM_CUDA(cudaGetLastError());
        count_launch();
        uint64_t* range = hbuf ? P->ranges.p + 2 * (size_t)nb : nullptr;
        k_paf_advance<<<1, 32, 0, s>>>(P->base.p, P->off.p, n, range);
        SHM_CUDA(cudaGetLastError());
        count_launch();
        if (hbuf) {  // the batch's text span, read back; its copy is queued by poll() once known
            SHM_CUDA(cudaMemcpyAsync(P->h_ranges + 2 * (size_t)nb, range, 2 * sizeof(uint64_t),
                                     cudaMemcpyDeviceToHost, s));
            if ((size_t)nb >= P->evs.size()) {
                cudaEvent_t e;
                SHM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
                P->evs.push_back(e);
            }
            SHM_CUDA(cudaEventRecord(P->evs[(size_t)nb], s));
        }
        nb++;
    }
    // the text of every finished batch to the caller's buffer, on the text
    // stream (the copy engine, beside the uploads of later batches)
    void copy_batch(int32_t b) {
        const uint64_t a = P->h_ranges[2 * (size_t)b], e = std::min(P->h_ranges[2 * (size_t)b + 1], hcap);
        if (e > a) SHM_CUDA(cudaMemcpyAsync(hbuf + a, P->text.p + a, (size_t)(e - a), cudaMemcpyDeviceToHost, P->ts));
    }
    void poll() override {
        while (hbuf && ncopied < nb) {
            const cudaError_t q = cudaEventQuery(P->evs[(size_t)ncopied]);
            if (q == cudaErrorNotReady) return;
            SHM_CUDA(q);
            copy_batch(ncopied++);
        }
    }
    void finish() {
        while (hbuf && ncopied < nb) {
            SHM_CUDA(cudaEventSynchronize(P->evs[(size_t)ncopied]));
            copy_batch(ncopied++);
        }
        if (hbuf) SHM_CUDA(cudaStreamSynchronize(P->ts));
    }
    ~PafSink() override {  // no copy into the caller's buffer outlives the call (an error path)
        if (hbuf) cudaStreamSynchronize(P->ts);
    }
};

// True for a pinned (page-locked) host buffer, which copies can fill
// asynchronously.
bool pinned_host(const char* buf) {
    if (!buf) return false;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, buf) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

}  // namespace

int64_t map_paf_host(MapCtx* c, const IndexStorage& ix, const shm_params& p, const uint8_t* seqs,
                     const int64_t* offs, int32_t n, const char* names, shm_map_record* out, char* buf,
                     int64_t cap) {
    SHM_CUDA(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    PafScratch& P = paf_scratch(c);
    shm_map_record* rec = out;
    if (!rec) {  // records land in pinned memory, so that their copies stay asynchronous
        if (P.h_rec_cap < (size_t)n || !P.h_rec) {
            if (P.h_rec) SHM_CUDA(cudaFreeHost(P.h_rec));
            P.h_rec = nullptr;
            P.h_rec_cap = 0;
            SHM_CUDA(cudaHostAlloc(&P.h_rec, sizeof(shm_map_record) * (size_t)std::max(n, 1), cudaHostAllocDefault));
            P.h_rec_cap = (size_t)std::max(n, 1);
        }
        rec = P.h_rec;
    }
    if (!P.h_small) SHM_CUDA(cudaHostAlloc(&P.h_small, 2 * sizeof(uint64_t), cudaHostAllocDefault));
    HostClock H;
    // the names go up from a helper thread on their own stream while the
    // first batch is packed; the sink joins it before its first kernel
    const size_t qlen = std::strlen(names ? names : "");
    PafView v = names_view(P, ix, p, n, qlen);
    if (!P.ns) SHM_CUDA(cudaStreamCreateWithFlags(&P.ns, cudaStreamNonBlocking));
    if (!P.nev) SHM_CUDA(cudaEventCreateWithFlags(&P.nev, cudaEventDisableTiming));
    std::exception_ptr names_err;
    std::thread names_th([&] {
        try {
            SHM_CUDA(cudaSetDevice(c->device));
            names_upload(c, P, ix, n, names, qlen, P.ns);
            SHM_CUDA(cudaEventRecord(P.nev, P.ns));
        } catch (...) {
            names_err = std::current_exception();
        }
    });
    struct Join {  // joined on every path out of this function
        std::thread& t;
        ~Join() {
            if (t.joinable()) t.join();
        }
    } names_join{names_th};
    auto names_ready = [&] {
        if (names_th.joinable()) names_th.join();
        if (names_err) std::rethrow_exception(names_err);
        SHM_CUDA(cudaStreamWaitEvent(s, P.nev, 0));
    };
    H.mark("names");
    v.map_time = nullptr;
    // room for every line: a line is its query name, a segment name and at
    // most about 700 bytes of numbers and tags (t:f: is 0 here); a line that
    // would not fit sends the call to the two-pass path below
    size_t seg_name = 0;
    for (const std::string& x : ix.names) seg_name = std::max(seg_name, x.size());
    const uint64_t tcap = (uint64_t)std::strlen(names ? names : "") + (uint64_t)n * (seg_name + 1024) + 64;
    P.text.reserve((size_t)tcap);
    P.base.reserve(1);
    P.flag.reserve(1);
    SHM_CUDA(cudaMemsetAsync(P.base.p, 0, sizeof(uint64_t), s));
    SHM_CUDA(cudaMemsetAsync(P.flag.p, 0, sizeof(uint32_t), s));
    PafSink sink;
    sink.c = c;
    sink.P = &P;
    sink.v0 = v;
    sink.cap = tcap;
    sink.names_ready = names_ready;
    // a pinned caller buffer takes each batch's text as soon as it is written
    sink.hbuf = cap > 0 && pinned_host(buf) ? buf : nullptr;
    sink.hcap = sink.hbuf ? (uint64_t)cap : 0;
    if (sink.hbuf) {
        if (!P.ts) SHM_CUDA(cudaStreamCreateWithFlags(&P.ts, cudaStreamNonBlocking));
        P.ranges.reserve(2 * ((size_t)n + 1));
        if (P.h_ranges_cap < (size_t)n + 1) {
            if (P.h_ranges) SHM_CUDA(cudaFreeHost(P.h_ranges));
            P.h_ranges = nullptr;
            P.h_ranges_cap = 0;
            SHM_CUDA(cudaHostAlloc((void**)&P.h_ranges, 2 * sizeof(uint64_t) * ((size_t)n + 1), cudaHostAllocDefault));
            P.h_ranges_cap = (size_t)n + 1;
        }
    }
    const bool changed = map_host(c, &ix, p, seqs, offs, n, rec, false, &sink);
    names_ready();  // (no batch: n = 0)
    c->work[W_H2D_BYTES] += P.names_h2d;
    H.mark("map");
    sink.finish();  // (a fallback below writes buf again)
    if (changed)  // records replaced after their batch's text was written: render from the final records
        return format_paf_device(c, ix, p, rec, n, names, nullptr, buf, cap);
    SHM_CUDA(cudaMemcpyAsync(P.h_small, P.base.p, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    SHM_CUDA(cudaMemcpyAsync(P.h_small + 1, P.flag.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    SHM_CUDA(cudaStreamSynchronize(s));
    H.mark("sync");
    if ((uint32_t)P.h_small[1] != 0) return format_paf_device(c, ix, p, rec, n, names, nullptr, buf, cap);
    const int64_t total = (int64_t)P.h_small[0];
    if (buf && cap > 0 && total > 0) {
        const int64_t take = std::min(cap, total);
        if (!sink.hbuf) {
            SHM_CUDA(cudaMemcpyAsync(buf, P.text.p, (size_t)take, cudaMemcpyDeviceToHost, s));
            SHM_CUDA(cudaStreamSynchronize(s));
        }
        c->work[W_D2H_BYTES] += take;
    }
    H.mark("text");
    H.print("paf", n);
    return total;
}

}  // namespace shm
