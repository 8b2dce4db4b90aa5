// TEST INFRASTRUCTURE ONLY: C entry points of the CPU oracle for the Python
// tests and bench.py's CPU baseline (ctypes). Not part of the product.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <string>
#include <vector>

#include "oracle.hpp"

using namespace oracle;

extern "C" {

// Same field set as the device path's per-read record, declared here on its
// own so the oracle does not depend on the product's headers.
struct orc_record {
    double score, sh, score2;
    int32_t status;  // 0 mapped, 1 nothing above the threshold, 2 sketch below MIN_HALFLEN
    int32_t read_len, sketch_size, seeds;
    int32_t p_start, p_end, segm_id, t_l, t_r;
    int32_t same_strand, intersection, s_sz;
    int32_t bucket_seg, bucket_b;
    int32_t has_second, intersection2, bucket2_seg, bucket2_b;
    int32_t total_matches, max_seed_matches, seed_matches, seeded_buckets, final_buckets;
    int32_t reserved;
};

struct orc_params {
    int32_t k;
    double h_frac;
    int32_t max_matches;
    double theta, min_diff, max_overlap;
    int32_t metric;  // 0 Containment, 1 Jaccard, 2 bucket_SH, 3 bucket_LCS
    int32_t no_bucket_pruning, one_sweep, abs_pos;
    double rarity_weight, rarity_tiebreak, rarity_alpha;  // params.rs:76-112
};

static Params to_params(const orc_params* p) {
    Params q;
    q.k = p->k;
    q.h_frac = p->h_frac;
    q.max_matches = p->max_matches;
    q.theta = p->theta;
    q.min_diff = p->min_diff;
    q.max_overlap = p->max_overlap;
    q.metric = (Metric)p->metric;
    q.no_bucket_pruning = p->no_bucket_pruning != 0;
    q.one_sweep = p->one_sweep != 0;
    q.abs_pos = p->abs_pos != 0;
    q.rarity_weight = p->rarity_weight;
    q.rarity_tiebreak = p->rarity_tiebreak;
    q.rarity_alpha = p->rarity_alpha;
    return q;
}

static std::vector<std::string> split_names(const char* joined, int32_t n) {
    std::vector<std::string> v;
    const char* s = joined ? joined : "";
    for (int32_t i = 0; i < n; i++) {
        const char* e = std::strchr(s, '\n');
        if (!e) e = s + std::strlen(s);
        v.emplace_back(s, (size_t)(e - s));
        s = *e ? e + 1 : e;
    }
    return v;
}

struct OrcIndex {
    SketchIndex idx;
    FracMinHash sk;
    OrcIndex(int32_t k, double f) : sk(k, f) {}
};

int64_t orc_sketch(const uint8_t* seq, int64_t len, int32_t k, double h_frac, int32_t offset, int32_t* r,
                   uint64_t* h, uint8_t* strand, int64_t cap) {
    FracMinHash sk(k, h_frac);
    std::vector<Kmer> v;
    sk.sketch_slice_into(seq, (size_t)len, offset, v);
    for (size_t i = 0; i < v.size() && (int64_t)i < cap; i++) {
        r[i] = v[i].r;
        h[i] = v[i].h;
        strand[i] = v[i].strand ? 1 : 0;
    }
    return (int64_t)v.size();
}

// bucket_LCS's count over window [bgn, end) of the sketch (t_r, t_h); seed i
// has hash seed_h[i] and positions pos[pos_off[i] .. pos_off[i + 1]).
int32_t orc_lcs(const int32_t* t_r, const uint64_t* t_h, int32_t n_t, int32_t bgn, int32_t end, const uint64_t* seed_h,
                const int32_t* pos_off, const int32_t* pos, int32_t n_seeds) {
    std::vector<Kmer> t((size_t)n_t);
    for (int32_t i = 0; i < n_t; i++) t[(size_t)i] = Kmer{t_r[i], t_h[i], false};
    std::vector<Hash> sh(seed_h, seed_h + n_seeds);
    std::vector<std::vector<QPos>> sp((size_t)n_seeds);
    for (int32_t i = 0; i < n_seeds; i++) sp[(size_t)i].assign(pos + pos_off[i], pos + pos_off[i + 1]);
    return lcs_window(t, bgn, end, sh, sp);
}

uint64_t orc_h_thres(int32_t k, double h_frac) { return FracMinHash(k, h_frac).h_thres(); }

void* orc_index_build(const uint8_t* seq, const int64_t* seg_off, int32_t n_seg, const char* names_joined,
                      int32_t k, double h_frac, int32_t max_matches, int32_t threads) {
    auto* o = new OrcIndex(k, h_frac);
    std::vector<const uint8_t*> seqs;
    std::vector<size_t> lens;
    for (int32_t i = 0; i < n_seg; i++) {
        seqs.push_back(seq + seg_off[i]);
        lens.push_back((size_t)(seg_off[i + 1] - seg_off[i]));
    }
    o->idx.build_index(split_names(names_joined, n_seg), seqs, lens, o->sk, max_matches, threads);
    return o;
}

void orc_index_free(void* p) { delete (OrcIndex*)p; }

// segments, total_nucls, indexed_hits, indexed_kmers, highest_freq, blacklisted_kmers, blacklisted_hits, sketched_kmers
void orc_index_stats(void* p, int64_t* out) {
    const IndexCounters& c = ((OrcIndex*)p)->idx.counters;
    out[0] = c.segments;
    out[1] = c.total_nucls;
    out[2] = c.indexed_hits;
    out[3] = c.indexed_kmers;
    out[4] = c.indexed_highest_freq_kmer;
    out[5] = c.blacklisted_kmers;
    out[6] = c.blacklisted_hits;
    out[7] = c.sketched_kmers;
}

void orc_index_count(void* p, const uint64_t* h, int64_t n, int32_t* out) {
    const SketchIndex& idx = ((OrcIndex*)p)->idx;
    for (int64_t i = 0; i < n; i++) out[i] = idx.count(h[i]);
}

// Hit list of one hash in the reference's order (segm_id, r); returns its length.
int64_t orc_index_hits(void* p, uint64_t h, int32_t* seg, int32_t* tpos, int32_t* r, uint8_t* strand, int64_t cap) {
    const SketchIndex& idx = ((OrcIndex*)p)->idx;
    int32_t c = idx.count(h);
    if (c == 0) return 0;
    std::vector<Hit> v;
    if (c == 1) v.push_back(idx.single_hit(h));
    else v = idx.multi_hits(h);
    for (size_t i = 0; i < v.size() && (int64_t)i < cap; i++) {
        seg[i] = v[i].segm_id;
        tpos[i] = v[i].tpos;
        r[i] = v[i].r;
        strand[i] = v[i].strand;
    }
    return (int64_t)v.size();
}

// Reference sketch of one segment (r, h, strand in tpos order); returns its length.
int64_t orc_segment_sketch(void* p, int32_t seg, int32_t* r, uint64_t* h, uint8_t* strand, int64_t cap) {
    const auto& km = ((OrcIndex*)p)->idx.segments[(size_t)seg].kmers;
    for (size_t i = 0; i < km.size() && (int64_t)i < cap; i++) {
        r[i] = km[i].r;
        h[i] = km[i].h;
        strand[i] = km[i].strand;
    }
    return (int64_t)km.size();
}

static void fill(orc_record& o, const ReadResult& rr) {
    std::memset(&o, 0, sizeof o);
    o.status = rr.unmappable_short_sketch ? 2 : (rr.mapped ? 0 : 1);
    o.read_len = rr.read_len;
    o.sketch_size = rr.m;
    o.seeds = rr.s;
    o.total_matches = (int32_t)rr.total_matches;
    o.max_seed_matches = (int32_t)rr.max_seed_matches;
    o.seed_matches = (int32_t)rr.seed_matches;
    o.seeded_buckets = (int32_t)rr.seeded_buckets;
    o.final_buckets = (int32_t)rr.final_buckets;
    o.bucket_seg = o.bucket_b = o.bucket2_seg = o.bucket2_b = -1;
    o.intersection2 = -1;
    o.score2 = -1.0;
    if (!rr.mapped) return;
    const Mapping& b = rr.best;
    o.score = b.j;
    o.sh = b.sh;
    o.p_start = b.p_start;
    o.p_end = b.p_end;
    o.segm_id = b.segm_id;
    o.t_l = b.t_l;
    o.t_r = b.t_r;
    o.same_strand = b.same_strand_seeds;
    o.intersection = b.intersection;
    o.s_sz = b.s_sz;
    o.bucket_seg = b.bucket.segm_id;
    o.bucket_b = b.bucket.b;
    if (rr.has2) {
        o.has_second = 1;
        o.intersection2 = rr.best2.intersection;
        o.score2 = rr.best2.j;
        o.bucket2_seg = rr.best2.bucket.segm_id;
        o.bucket2_b = rr.best2.bucket.b;
    }
}

int32_t orc_map(void* p, const orc_params* prm, const uint8_t* seqs, const int64_t* offs, int32_t n, int32_t threads,
                orc_record* out) {
    OrcIndex* o = (OrcIndex*)p;
    Params q = to_params(prm);
    std::vector<const uint8_t*> s;
    std::vector<size_t> l;
    for (int32_t i = 0; i < n; i++) {
        s.push_back(seqs + offs[i]);
        l.push_back((size_t)(offs[i + 1] - offs[i]));
    }
    auto res = map_reads(o->idx, o->sk, q, s, l, threads);
    for (int32_t i = 0; i < n; i++) fill(out[i], res[(size_t)i]);
    return 0;
}

// Maps and renders the stdout PAF text (mapped reads only, one line each,
// t:f: printed as 0). Returns the byte length needed; writes up to cap bytes.
int64_t orc_paf(void* p, const orc_params* prm, const uint8_t* seqs, const int64_t* offs, const char* names_joined,
                int32_t n, int32_t threads, char* buf, int64_t cap) {
    OrcIndex* o = (OrcIndex*)p;
    Params q = to_params(prm);
    std::vector<const uint8_t*> s;
    std::vector<size_t> l;
    for (int32_t i = 0; i < n; i++) {
        s.push_back(seqs + offs[i]);
        l.push_back((size_t)(offs[i + 1] - offs[i]));
    }
    auto names = split_names(names_joined, n);
    auto res = map_reads(o->idx, o->sk, q, s, l, threads);
    std::string text;
    for (int32_t i = 0; i < n; i++)
        if (res[(size_t)i].mapped) text += render_paf(res[(size_t)i], names[(size_t)i], q, 0.0) + "\n";
    if (buf && cap > 0) std::memcpy(buf, text.data(), (size_t)std::min<int64_t>(cap, (int64_t)text.size()));
    return (int64_t)text.size();
}

// Maps n reads with `threads` host threads and renders their PAF text in input
// order (mapped reads only, t:f: as 0), timed from the first read taken to the
// joined text: records to out[n] (may be NULL), the text's length to
// *text_len. Returns the wall-clock seconds. The text stays in this file's
// buffer until orc_take_text copies it out (bench.py's CPU baseline and its
// full-size parity check).
static std::string g_text;
double orc_map_paf(void* p, const orc_params* prm, const uint8_t* seqs, const int64_t* offs, const char* names_joined,
                   int32_t n, int32_t threads, orc_record* out, int64_t* text_len) {
    OrcIndex* o = (OrcIndex*)p;
    Params q = to_params(prm);
    std::vector<const uint8_t*> s;
    std::vector<size_t> l;
    for (int32_t i = 0; i < n; i++) {
        s.push_back(seqs + offs[i]);
        l.push_back((size_t)(offs[i + 1] - offs[i]));
    }
    auto names = split_names(names_joined, n);
    std::vector<ReadResult> res;
    auto t0 = std::chrono::steady_clock::now();
    map_reads_paf(o->idx, o->sk, q, s, l, names, threads, res, g_text);
    auto t1 = std::chrono::steady_clock::now();
    if (out)
        for (int32_t i = 0; i < n; i++) fill(out[i], res[(size_t)i]);
    if (text_len) *text_len = (int64_t)g_text.size();
    return std::chrono::duration<double>(t1 - t0).count();
}

// Copies the text of the last orc_map_paf (up to cap bytes) and releases it.
int64_t orc_take_text(char* buf, int64_t cap) {
    const int64_t n = std::min<int64_t>(cap, (int64_t)g_text.size());
    if (buf && n > 0) std::memcpy(buf, g_text.data(), (size_t)n);
    std::string().swap(g_text);
    return n;
}

// Wall-clock seconds to map a sample with `threads` host threads (bench.py's CPU baseline).
double orc_time_map(void* p, const orc_params* prm, const uint8_t* seqs, const int64_t* offs, int32_t n,
                    int32_t threads) {
    OrcIndex* o = (OrcIndex*)p;
    Params q = to_params(prm);
    std::vector<const uint8_t*> s;
    std::vector<size_t> l;
    for (int32_t i = 0; i < n; i++) {
        s.push_back(seqs + offs[i]);
        l.push_back((size_t)(offs[i + 1] - offs[i]));
    }
    auto t0 = std::chrono::steady_clock::now();
    auto res = map_reads(o->idx, o->sk, q, s, l, threads);
    auto t1 = std::chrono::steady_clock::now();
    volatile int64_t sink = 0;
    for (auto& r : res) sink += r.mapped;
    (void)sink;
    return std::chrono::duration<double>(t1 - t0).count();
}

}  // extern "C"
