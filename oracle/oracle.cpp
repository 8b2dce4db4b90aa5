// TEST INFRASTRUCTURE ONLY: the CPU oracle (see oracle.hpp). Restates
// shmap-rs v1.4.3 (crate `shmap`), file by file; citations are paths inside
// that project.
#include "oracle.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <thread>

namespace oracle {

static inline uint64_t rotl(uint64_t x, uint32_t n) {
    n &= 63;
    return n == 0 ? x : (x << n) | (x >> (64 - n));
}
static inline uint64_t rotr(uint64_t x, uint32_t n) {
    n &= 63;
    return n == 0 ? x : (x >> n) | (x << (64 - n));
}

// Rust `f64 as i32`: truncation toward zero, saturating, NaN -> 0.
static int32_t f64_as_i32(double x) {
    if (std::isnan(x)) return 0;
    if (x >= 2147483647.0) return INT32_MAX;
    if (x <= -2147483648.0) return INT32_MIN;
    return (int32_t)x;
}
// Rust `f64 as u64`: truncation toward zero, saturating, NaN -> 0.
static uint64_t f64_as_u64(double x) {
    if (std::isnan(x) || x <= 0.0) return 0;
    if (x >= 18446744073709551616.0) return UINT64_MAX;
    return (uint64_t)x;
}

// ---------------------------------------------------------------- sketch.rs
// src/sketch.rs:58-108
FracMinHash::FracMinHash(int32_t k_, double h_frac_) : k(k_), h_frac(h_frac_) {
    const Hash A = 0x3c8bfbb395c60474ULL, C = 0x3193c18562a02b4cULL,
               G = 0x20323ed082572324ULL, T = 0x295549f54be24456ULL;
    std::memset(lut_fw, 0, sizeof lut_fw);
    std::memset(lut_rc, 0, sizeof lut_rc);
    const struct { uint8_t lo, up; Hash v; } fw[4] = {{'a', 'A', A}, {'c', 'C', C}, {'g', 'G', G}, {'t', 'T', T}};
    for (auto& e : fw) lut_fw[e.lo] = lut_fw[e.up] = e.v;
    const struct { uint8_t lo, up, comp; } rc[4] = {{'a', 'A', 'T'}, {'c', 'C', 'G'}, {'g', 'G', 'C'}, {'t', 'T', 'A'}};
    for (auto& e : rc) lut_rc[e.lo] = lut_rc[e.up] = lut_fw[e.comp];
    for (int c = 0; c < 256; c++) {
        lut_fw_k[c] = rotl(lut_fw[c], (uint32_t)k);
        lut_rc_r1[c] = rotr(lut_rc[c], 1);
        lut_rc_k1[c] = rotl(lut_rc[c], (uint32_t)(k - 1));
    }
}

// src/sketch.rs:126-132
Hash FracMinHash::h_thres() const {
    if (h_frac < 1.0) return f64_as_u64(h_frac * (double)UINT64_MAX);
    return UINT64_MAX;
}

// src/sketch.rs:167-209 and emit() at 213-219
void FracMinHash::sketch_slice_into(const uint8_t* s, size_t n, RPos offset, std::vector<Kmer>& out) const {
    out.clear();
    if ((int64_t)n < (int64_t)k || k <= 0) return;
    const size_t ks = (size_t)k;
    const Hash thr = h_thres();
    Hash fw = 0, rc = 0;
    for (size_t i = 0; i < ks; i++) {
        fw ^= rotl(lut_fw[s[i]], (uint32_t)(ks - i - 1));
        rc ^= rotl(lut_rc[s[i]], (uint32_t)i);
    }
    RPos r = k - 1 + offset;
    auto emit = [&](RPos rr, Hash f, Hash c) {
        Hash h = c ^ f;
        if (h <= thr) out.push_back(Kmer{rr, h, f > c});
    };
    emit(r, fw, rc);
    for (size_t j = ks; j < n; j++) {
        const uint8_t in_c = s[j], out_c = s[j - ks];
        fw = rotl(fw, 1) ^ lut_fw_k[out_c] ^ lut_fw[in_c];
        rc = rotr(rc, 1) ^ lut_rc_r1[out_c] ^ lut_rc_k1[in_c];
        r += 1;
        emit(r, fw, rc);
    }
}

// ---------------------------------------------------------------- HashMap
template <class V> void HashMap<V>::reserve(size_t n) {
    size_t cap = 16;
    while (cap < n * 2) cap <<= 1;
    if (cap <= keys_.size()) return;
    std::vector<Hash> ok;
    std::vector<uint8_t> ou;
    std::vector<V> ov;
    ok.swap(keys_);
    ou.swap(used_);
    ov.swap(vals_);
    keys_.assign(cap, 0);
    used_.assign(cap, 0);
    vals_.resize(cap);
    n_ = 0;
    for (size_t i = 0; i < ok.size(); i++)
        if (ou[i]) {
            bool ins;
            get_or_insert(ok[i], &ins) = std::move(ov[i]);
        }
}
template <class V> void HashMap<V>::grow() { reserve(std::max<size_t>(16, n_ + 1)); }
template <class V> V* HashMap<V>::get(Hash h) {
    if (keys_.empty()) return nullptr;
    size_t mask = keys_.size() - 1, i = mix(h) & mask;
    while (used_[i]) {
        if (keys_[i] == h) return &vals_[i];
        i = (i + 1) & mask;
    }
    return nullptr;
}
template <class V> const V* HashMap<V>::get(Hash h) const { return const_cast<HashMap*>(this)->get(h); }
template <class V> V& HashMap<V>::get_or_insert(Hash h, bool* inserted) {
    if ((n_ + 1) * 2 > keys_.size()) reserve(std::max<size_t>(16, (n_ + 1) * 2));
    size_t mask = keys_.size() - 1, i = mix(h) & mask;
    while (used_[i]) {
        if (keys_[i] == h) {
            *inserted = false;
            return vals_[i];
        }
        i = (i + 1) & mask;
    }
    used_[i] = 1;
    keys_[i] = h;
    vals_[i] = V();
    n_++;
    *inserted = true;
    return vals_[i];
}
// Linear-probing deletion by backward shift (keeps every remaining key reachable).
template <class V> bool HashMap<V>::erase(Hash h) {
    if (keys_.empty()) return false;
    size_t mask = keys_.size() - 1, i = mix(h) & mask;
    while (used_[i] && keys_[i] != h) i = (i + 1) & mask;
    if (!used_[i]) return false;
    size_t j = i;
    for (;;) {
        j = (j + 1) & mask;
        if (!used_[j]) break;
        size_t home = mix(keys_[j]) & mask;
        // move j into the hole at i if its home is not in the cyclic range (i, j]
        bool in_range = (i <= j) ? (i < home && home <= j) : (i < home || home <= j);
        if (!in_range) {
            keys_[i] = keys_[j];
            vals_[i] = std::move(vals_[j]);
            i = j;
        }
    }
    used_[i] = 0;
    vals_[i] = V();
    n_--;
    return true;
}
template <class V> template <class F> void HashMap<V>::for_each(F f) {
    for (size_t i = 0; i < keys_.size(); i++)
        if (used_[i]) f(keys_[i], vals_[i]);
}

// ---------------------------------------------------------------- index.rs
static inline int shard_of(Hash h) { return (int)(h & (SketchIndex::N_SHARDS - 1)); }  // index.rs:97-99

// src/index.rs:264-291
static void insert_hit(Shard& shard, const Kmer& kmer, RPos tpos, SegmId segm_id, int32_t max_matches) {
    Hit hit{kmer.r, tpos, kmer.strand, segm_id};
    bool ins;
    Hit& single = shard.h2single.get_or_insert(kmer.h, &ins);
    if (ins) {
        single = hit;
        return;
    }
    std::vector<Hit>& multi = shard.h2multi.get_or_insert(kmer.h, &ins);
    if (max_matches < 0 || (int32_t)multi.size() < max_matches + 1) multi.push_back(hit);
}

// src/index.rs:295-315
static void finalize_shard(Shard& shard) {
    shard.h2multi.for_each([&](Hash h, std::vector<Hit>& hits) {
        if (Hit* s = shard.h2single.get(h)) {
            hits.push_back(*s);
            shard.h2single.erase(h);
        }
        std::stable_sort(hits.begin(), hits.end(), [](const Hit& a, const Hit& b) {
            return a.segm_id != b.segm_id ? a.segm_id < b.segm_id : a.r < b.r;
        });
    });
}

// src/index.rs:384-663: segments sketched and applied in file order; the
// shard fill (index.rs:233-261) is split by shard across threads, which the
// reference shows is output-identical to the serial fill.
void SketchIndex::build_index(const std::vector<std::string>& names, const std::vector<const uint8_t*>& seqs,
                              const std::vector<size_t>& lens, const FracMinHash& sk, int32_t max_matches,
                              int threads) {
    const size_t nseg = names.size();
    segments.resize(nseg);
    threads = std::max(1, threads);
    {
        std::atomic<size_t> next{0};
        auto work = [&]() {
            for (size_t i; (i = next.fetch_add(1)) < nseg;) {
                RefSegment& s = segments[i];
                sk.sketch_slice_into(seqs[i], lens[i], 0, s.kmers);
                s.name = names[i];
                s.sz = (RPos)lens[i];
                s.id = (int32_t)i;
            }
        };
        std::vector<std::thread> ts;
        for (int t = 0; t < threads; t++) ts.emplace_back(work);
        for (auto& t : ts) t.join();
    }
    for (auto& s : segments) {
        counters.segments += 1;
        counters.total_nucls += s.sz;
        counters.sketched_kmers += (int64_t)s.kmers.size();
    }
    // populate (index.rs:233-261): each thread owns whole shards and scans every
    // segment in file order and every k-mer in tpos order.
    {
        std::vector<std::thread> ts;
        int nt = std::min(threads, N_SHARDS);
        for (int t = 0; t < nt; t++)
            ts.emplace_back([&, t]() {
                for (int s = t; s < N_SHARDS; s += nt) {
                    size_t est = 0;
                    for (auto& seg : segments) est += seg.kmers.size() / N_SHARDS;
                    shards[s].h2single.reserve(est / 2 + 16);
                }
                for (size_t sid = 0; sid < segments.size(); sid++) {
                    const auto& km = segments[sid].kmers;
                    for (size_t tpos = 0; tpos < km.size(); tpos++) {
                        int s = shard_of(km[tpos].h);
                        if (s % nt != t) continue;
                        insert_hit(shards[s], km[tpos], (RPos)tpos, (SegmId)sid, max_matches);
                    }
                }
                for (int s = t; s < N_SHARDS; s += nt) finalize_shard(shards[s]);
            });
        for (auto& t : ts) t.join();
    }
    // get_kmer_stats (index.rs:343-358)
    for (auto& sh : shards) {
        counters.indexed_hits += (int64_t)sh.h2single.size();
        counters.indexed_kmers += (int64_t)sh.h2single.size();
        sh.h2multi.for_each([&](Hash, std::vector<Hit>& hits) {
            counters.indexed_hits += (int64_t)hits.size();
            counters.indexed_kmers += 1;
            counters.indexed_highest_freq_kmer = std::max<int64_t>(counters.indexed_highest_freq_kmer, (int64_t)hits.size());
        });
    }
    // erase_frequent_kmers (index.rs:360-376)
    if (max_matches >= 0) {
        for (auto& sh : shards) {
            std::vector<Hash> black;
            sh.h2multi.for_each([&](Hash h, std::vector<Hit>& hits) {
                if ((int32_t)hits.size() > max_matches) {
                    counters.blacklisted_kmers += 1;
                    counters.blacklisted_hits += (int64_t)hits.size();
                    black.push_back(h);
                }
            });
            for (Hash h : black) sh.h2multi.erase(h);
        }
    }
}

RPos SketchIndex::count(Hash h) const {
    const Shard& s = shards[shard_of(h)];
    if (s.h2single.get(h)) return 1;
    if (const auto* v = s.h2multi.get(h)) return (RPos)v->size();
    return 0;
}
Hit SketchIndex::single_hit(Hash h) const { return *shards[shard_of(h)].h2single.get(h); }
const std::vector<Hit>& SketchIndex::multi_hits(Hash h) const { return *shards[shard_of(h)].h2multi.get(h); }

// ---------------------------------------------------------------- buckets.rs
static const QPos MIN_HALFLEN = 5;                 // buckets.rs:15
static const size_t MAX_DENSE_SLOTS = 2u << 20;    // buckets.rs:62

struct Entry {
    BucketLoc loc;
    QPos matches;
    int32_t codirection;
    RPos r_min, r_max;
    void merge(const Entry& o) {  // buckets.rs:133-138
        matches += o.matches;
        codirection += o.codirection;
        r_min = std::min(r_min, o.r_min);
        r_max = std::max(r_max, o.r_max);
    }
};
struct Slot {
    QPos matches = 0;
    int32_t codirection = 0;
    RPos r_min = INT32_MAX, r_max = -1;
};

// src/buckets.rs:241-725 (dense accumulator with the sparse fallback; the
// sparse fallback's LSD radix sort is replaced by an equivalent comparison
// sort, the reference's own dense==sparse test pins that both orders agree).
class Buckets {
public:
    Buckets(const SketchIndex& t, bool ap) : tidx(t), AP(ap) {}
    const SketchIndex& tidx;
    bool AP;
    QPos halflen = -1;
    int32_t i = 0;
    QPos seeds = 0;

    void clear() {  // buckets.rs:331-343
        i = 0;
        seeds = 0;
        entries.clear();
        prop_i = -1;
        prop_seeds = 0;
        merged = true;
    }
    bool dense_on = false;  // the dense accumulator is in use (read by the tests)

    bool set_halflen(QPos h) {  // buckets.rs:348-356
        halflen = h;
        if (halflen < MIN_HALFLEN) {
            dense_on = false;
            return false;
        }
        plan_dense();
        return true;
    }
    RPos begin(const BucketLoc& b) const { return b.b * halflen; }
    RPos end(const BucketLoc& b) const { return (b.b + 2) * halflen; }

    void add_to_pos(const Hit& hit, const BucketContent& c) {  // buckets.rs:642-662
        RPos b = (AP ? hit.r : hit.tpos) / halflen;
        merged = false;
        if (dense_on) {
            size_t g = seg_base[hit.segm_id] + (size_t)b;
            dense_add(g, c);
            if (b > 0) dense_add(g - 1, c);
            return;
        }
        entries.push_back(Entry{BucketLoc{hit.segm_id, b}, c.matches, c.codirection, c.r_min, c.r_max});
        if (b > 0) entries.push_back(Entry{BucketLoc{hit.segm_id, b - 1}, c.matches, c.codirection, c.r_min, c.r_max});
    }
    void add_to_bucket(BucketLoc b, const BucketContent& c) {  // buckets.rs:664-674
        merged = false;
        if (dense_on) {
            dense_add(seg_base[b.segm_id] + (size_t)b.b, c);
            return;
        }
        entries.push_back(Entry{b, c.matches, c.codirection, c.r_min, c.r_max});
    }
    void propagate_seeds_to_buckets() {  // buckets.rs:634-640
        merge_entries();
        prop_i = i;
        prop_seeds = seeds;
    }
    std::vector<std::pair<BucketLoc, BucketContent>> get_sorted_buckets() {  // buckets.rs:685-724
        merge_entries();
        order.clear();
        for (size_t idx = 0; idx < entries.size(); idx++)
            order.push_back(((uint64_t)(UINT32_MAX - (uint32_t)entries[idx].matches) << 32) | (uint64_t)idx);
        std::sort(order.begin(), order.end());
        std::vector<std::pair<BucketLoc, BucketContent>> out;
        out.reserve(order.size());
        for (uint64_t key : order) {
            const Entry& e = entries[key & 0xffffffffu];
            BucketContent c;
            c.i = prop_i;
            c.seeds = prop_seeds;
            c.matches = e.matches;
            c.codirection = e.codirection;
            c.r_min = e.r_min;
            c.r_max = e.r_max;
            out.emplace_back(e.loc, c);
        }
        return out;
    }

private:
    std::vector<Entry> entries;
    bool merged = true;
    int32_t prop_i = -1;
    QPos prop_seeds = 0;
    std::vector<Slot> dense;
    std::vector<uint32_t> seg_base;
    std::vector<uint32_t> touched;
    size_t dense_slots = 0;
    bool dense_dirty = false;
    std::vector<uint64_t> order;

    void retire_dense_slots() {  // buckets.rs:384-392
        if (dense_dirty) {
            for (uint32_t g : touched) dense[g] = Slot();
            dense_dirty = false;
        }
        touched.clear();
    }
    void plan_dense() {  // buckets.rs:394-425
        retire_dense_slots();
        const int64_t hl = halflen;
        seg_base.clear();
        int64_t total = 0;
        for (const auto& seg : tidx.segments) {
            seg_base.push_back((uint32_t)total);
            int64_t extent = AP ? (int64_t)seg.sz : (int64_t)seg.kmers.size();
            total += (std::max<int64_t>(extent, 1) - 1) / hl + 2;
            if (total > (int64_t)MAX_DENSE_SLOTS) {
                seg_base.clear();
                dense.clear();
                dense.shrink_to_fit();
                dense_on = false;
                return;
            }
        }
        if (dense.size() < (size_t)total) dense.resize((size_t)total);
        dense_slots = (size_t)total;
        dense_on = true;
        dense_dirty = true;
    }
    void dense_add(size_t g, const BucketContent& c) {  // buckets.rs:430-436
        Slot& s = dense[g];
        if (s.matches == 0) touched.push_back((uint32_t)g);
        s.matches += c.matches;
        s.codirection += c.codirection;
        s.r_min = std::min(s.r_min, c.r_min);
        s.r_max = std::max(s.r_max, c.r_max);
    }
    void extract_dense() {  // buckets.rs:454-510 (the sorted-touched-list walk)
        entries.clear();
        std::sort(touched.begin(), touched.end());
        size_t sid = 0;
        for (uint32_t g : touched) {
            while (sid + 1 < seg_base.size() && seg_base[sid + 1] <= g) sid++;
            Slot s = dense[g];
            dense[g] = Slot();
            entries.push_back(Entry{BucketLoc{(SegmId)sid, (RPos)(g - seg_base[sid])}, s.matches, s.codirection, s.r_min, s.r_max});
        }
        touched.clear();
        dense_dirty = false;
    }
    void merge_entries() {  // buckets.rs:608-632
        if (merged) return;
        merged = true;
        if (dense_on) {
            extract_dense();
            return;
        }
        if (entries.empty()) return;
        std::stable_sort(entries.begin(), entries.end(), [](const Entry& a, const Entry& b) {
            return a.loc.segm_id != b.loc.segm_id ? a.loc.segm_id < b.loc.segm_id : a.loc.b < b.loc.b;
        });
        size_t w = 0;
        for (size_t r = 1; r < entries.size(); r++) {
            if (entries[r].loc == entries[w].loc) entries[w].merge(entries[r]);
            else entries[++w] = entries[r];
        }
        entries.resize(w + 1);
    }
};

// ---------------------------------------------------------------- mapping.rs
void Mapping::update(QPos ps, QPos pe, RPos tl, RPos tr, const RefSegment& sg, QPos inter, double new_score,
                     int32_t same, RPos sz) {
    if (new_score > score()) {
        p_start = ps;
        p_end = pe;
        strand = same > 0 ? '+' : '-';
        segm = &sg;
        segm_id = sg.id;
        t_l = tl;
        t_r = tr;
        mapq = 255;
        read_len = -1;
        s_sz = sz;
        same_strand_seeds = same;
        intersection = inter;
        j = new_score;
    }
}
static double sigmas_diff_fn(QPos x, QPos y) {  // mapping.rs:329-333
    double fx = (double)(x == -1 ? 0 : x), fy = (double)(y == -1 ? 0 : y);
    return std::fabs(fx - fy) / std::sqrt(fx + fy);
}
uint8_t Mapping::calc_mapq(double theta2, double min_diff) {
    if (j2 < theta2) j2 = theta2;
    double frac = 1.0 - j2 / j;
    int32_t mapq_strand = std::abs(same_strand_seeds) < intersection / 2 ? 5 : 60;
    return frac > min_diff ? (uint8_t)std::min(60, mapq_strand) : 0;
}
void Mapping::set_second_best(const Mapping& m2) {
    bucket2 = m2.bucket;
    intersection2 = m2.intersection;
    j2 = m2.score();
    sigmas_diff = sigmas_diff_fn(intersection2, intersection);
}
double Mapping::overlap(const Mapping& a, const Mapping& b) {
    if (a.segm_id != b.segm_id) return -0.0;
    RPos cap = std::max(0, std::min(a.t_r, b.t_r) - std::max(a.t_l, b.t_l));
    RPos cup = std::max(a.t_r, b.t_r) - std::min(a.t_l, b.t_l);
    return (double)cap / (double)cup;
}

// Rust `{:.N}` on f64: correctly rounded fixed notation, NaN as "NaN".
static std::string ff(double x, int prec) {
    if (std::isnan(x)) return "NaN";
    if (std::isinf(x)) return x > 0 ? "inf" : "-inf";
    char buf[512];
    std::snprintf(buf, sizeof buf, "%.*f", prec, x);
    return buf;
}

// String building without iostreams (this library is loaded next to other
// copies of the C++ runtime, and their stream locales must not meet).
struct Out {
    std::string s;
    Out& operator<<(const std::string& v) {
        s += v;
        return *this;
    }
    Out& operator<<(const char* v) {
        s += v;
        return *this;
    }
    Out& operator<<(char v) {
        s += v;
        return *this;
    }
    Out& operator<<(long long v) {
        char b[32];
        std::snprintf(b, sizeof b, "%lld", v);
        s += b;
        return *this;
    }
    Out& operator<<(int32_t v) { return *this << (long long)v; }
};

std::string Mapping::paf(const std::string& query_id) const {
    Out o;
    o << query_id << '\t' << read_len << '\t' << p_start << '\t' << p_end << '\t' << strand << '\t'
      << (segm ? segm->name : std::string()) << '\t' << (segm ? segm->sz : -1) << '\t' << t_l << '\t' << t_r << '\t'
      << read_len << '\t' << read_len << '\t' << (int32_t)mapq;
    o << "\tp:i:" << p_sz << "\ts:i:" << s_sz << "\tI:i:" << intersection << "\tI2:i:" << intersection2
      << "\tIdiff:i:" << (int32_t)(intersection - intersection2) << "\tIsdiff:f:" << ff(sigmas_diff, 5)
      << "\tJ:f:" << ff(j, 5) << "\tJ2:f:" << ff(j2, 5) << "\tJdiff:f:" << ff(j - j2, 5) << "\tsh:f:" << ff(sh, 5)
      << "\tstrand:i:" << same_strand_seeds << "\tt:f:" << ff(map_time, 5) << "\tb:s:(" << bucket.segm_id << ','
      << bucket.b << ")\tb2:s:(" << bucket2.segm_id << ',' << bucket2.b << ')';
    if (has_global)
        o << "\tk:i:" << g_k << "\tgt_J:f:" << ff(-1.0, 3) << "\tgt_C:f:" << ff(-1.0, 3) << "\tgt_C_bucket:f:"
          << ff(-1.0, 3) << "\tseeds:i:" << g_seeds << "\tmax_seed_matches:i:" << max_seed_matches
          << "\tseed_matches:i:" << seed_matches << "\ttotal_matches:i:" << total_matches
          << "\tmatch_inefficiency:f:" << ff(match_inefficiency, 3) << "\tseeded_buckets:i:" << seeded_buckets
          << "\tfinal_buckets:i:" << final_buckets << "\tFPTP:f:" << ff(fptp, 3);
    return o.s;
}

std::string unmapped_line(const std::string& query_id, QPos read_len) {
    Out o;
    o << query_id << '\t' << read_len << "\t0\t0\t*\t*\t0\t0\t0\t0\t0\t0";
    return o.s;
}

// ---------------------------------------------------------------- shmap/*.rs
namespace {

struct Ctx {
    const SketchIndex& tidx;
    const Params& p;
    int64_t total_matches = 0, seed_matches = 0, max_seed_matches = 0, final_buckets = 0;
    // rarity weights of the read's seeds by seed_num and their total over its
    // k-mers (src/shmap/mod.rs:341-352, 694-723); empty when no rarity flag is on
    std::vector<double> rarity;
    double m_weight = 0.0;
};

// p_ht: hash -> index into p_unique (the reference stores a Seed clone; same content)
using PHt = HashMap<int32_t>;

// src/shmap/seeding.rs:26-77
std::vector<Seed> unique_elements_with_info(Ctx& cx, std::vector<Kmer>& p) {
    std::sort(p.begin(), p.end(), [](const Kmer& a, const Kmer& b) { return a.h != b.h ? a.h < b.h : b.r < a.r; });
    std::vector<Seed> u;
    u.reserve(p.size());
    size_t group_start = 0;
    for (size_t ppos = 0; ppos < p.size(); ppos++) {
        if (ppos + 1 == p.size() || p[ppos].h != p[ppos + 1].h) {
            QPos strike = (QPos)(ppos + 1 - group_start);
            RPos hits = cx.tidx.count(p[ppos].h);
            u.push_back(Seed{p[ppos], hits, strike, (QPos)u.size()});
            group_start = ppos + 1;
        }
    }
    std::stable_sort(u.begin(), u.end(), [](const Seed& a, const Seed& b) { return a.hits_in_t < b.hits_in_t; });
    return u;
}

// src/shmap/seeding.rs:11-20
inline void flush_slot(Buckets& bk, SegmId sid, RPos bb, const BucketContent& acc, QPos occs) {
    BucketContent c;
    c.matches = std::min(acc.matches, occs);
    c.seeds = 0;
    c.codirection = acc.codirection;
    c.r_min = acc.r_min;
    c.r_max = acc.r_max;
    bk.add_to_bucket(BucketLoc{sid, bb}, c);
}

// src/shmap/seeding.rs:98-212
void match_seeds(Ctx& cx, const std::vector<Seed>& pu, Buckets& bk, QPos s) {
    int64_t seed_matches = 0;
    const QPos halflen = bk.halflen;
    while ((size_t)bk.i < pu.size() && bk.seeds < s) {
        const Seed& seed = pu[(size_t)bk.i];
        if (seed.hits_in_t > 0) {
            seed_matches += seed.hits_in_t;
            cx.max_seed_matches = std::max<int64_t>(cx.max_seed_matches, seed.hits_in_t);
            if (seed.hits_in_t == 1) {
                Hit hit = cx.tidx.single_hit(seed.kmer.h);
                BucketContent c;
                c.matches = 1;
                c.codirection = hit.strand == seed.kmer.strand ? 1 : -1;
                c.r_min = c.r_max = hit.r;
                bk.add_to_pos(hit, c);
            } else {
                const QPos occs = seed.occs_in_p;
                SegmId cur_sid = -1;
                RPos b = 0, b_hi = 0, base = 0;
                BucketContent acc[2];
                for (const Hit& hit : cx.tidx.multi_hits(seed.kmer.h)) {
                    RPos pos = cx.p.abs_pos ? hit.r : hit.tpos;
                    BucketContent content;
                    content.matches = 1;
                    content.codirection = hit.strand == seed.kmer.strand ? 1 : -1;
                    content.r_min = content.r_max = hit.r;
                    if (hit.segm_id != cur_sid) {
                        for (int j = 0; j < 2; j++)
                            if (acc[j].matches > 0) {
                                flush_slot(bk, cur_sid, base + j, acc[j], occs);
                                acc[j] = BucketContent();
                            }
                        cur_sid = hit.segm_id;
                        b = pos / halflen;
                        b_hi = (b + 1) * halflen;
                        base = std::max(b - 1, 0);
                    } else {
                        while (pos >= b_hi) {
                            b += 1;
                            b_hi += halflen;
                        }
                        RPos new_base = std::max(b - 1, 0);
                        if (new_base > base) {
                            if (acc[0].matches > 0) flush_slot(bk, cur_sid, base, acc[0], occs);
                            if (new_base == base + 1) {
                                acc[0] = acc[1];
                            } else {
                                if (acc[1].matches > 0) flush_slot(bk, cur_sid, base + 1, acc[1], occs);
                                acc[0] = BucketContent();
                            }
                            acc[1] = BucketContent();
                            base = new_base;
                        }
                    }
                    acc[b - base].add(content);
                    if (b > 0) acc[b - 1 - base].add(content);
                }
                for (int j = 0; j < 2; j++)
                    if (acc[j].matches > 0) flush_slot(bk, cur_sid, base + j, acc[j], occs);
            }
        }
        bk.seeds += seed.occs_in_p;
        bk.i += 1;
    }
    cx.seed_matches += seed_matches;
    cx.total_matches += seed_matches;
}

// src/shmap/pruning.rs:10-13
inline double hseed(QPos p, QPos seeds, QPos matches) { return 1.0 - (double)(seeds - matches) / (double)p; }

// src/shmap/pruning.rs:18-80
void matches_in_bucket(Ctx& cx, const Buckets& bk, const BucketLoc& b, BucketContent& bucket, const Seed& s) {
    const bool AP = cx.p.abs_pos;
    bucket.seeds += s.occs_in_p;
    if (s.hits_in_t == 0) {
    } else if (s.hits_in_t == 1) {
        Hit hit = cx.tidx.single_hit(s.kmer.h);
        RPos pos = AP ? hit.r : hit.tpos;
        bool in_range = hit.segm_id == b.segm_id && bk.begin(b) <= pos && pos < bk.end(b);
        if (in_range) {
            bucket.matches += 1;
            bucket.codirection += hit.strand == s.kmer.strand ? 1 : -1;
            bucket.r_min = std::min(bucket.r_min, hit.r);
            bucket.r_max = std::max(bucket.r_max, hit.r);
        }
    } else {
        const auto& hits = cx.tidx.multi_hits(s.kmer.h);
        const RPos bgn = bk.begin(b), end = bk.end(b);
        auto start = std::partition_point(hits.begin(), hits.end(), [&](const Hit& h) {
            if (h.segm_id != b.segm_id) return h.segm_id < b.segm_id;
            return (AP ? h.r : h.tpos) < bgn;
        });
        RPos matches = 0;
        for (auto it = start; it != hits.end(); ++it) {
            if (!(it->segm_id == b.segm_id && (AP ? it->r : it->tpos) < end)) break;
            matches += 1;
            bucket.codirection += it->strand == s.kmer.strand ? 1 : -1;
            bucket.r_min = std::min(bucket.r_min, it->r);
            bucket.r_max = std::max(bucket.r_max, it->r);
        }
        bucket.matches += std::min(matches, s.occs_in_p);
    }
}

// src/shmap/pruning.rs:95-119
bool seed_heuristic_pass(Ctx& cx, const Buckets& bk, const std::vector<Seed>& pu, QPos m, const BucketLoc& b,
                         BucketContent& bucket, double& sh, double thr) {
    if (!cx.p.no_bucket_pruning) {
        for (;;) {
            sh = hseed(m, bucket.seeds, bucket.matches);
            if (sh < thr) return false;
            if ((size_t)bucket.i >= pu.size()) break;
            matches_in_bucket(cx, bk, b, bucket, pu[(size_t)bucket.i]);
            bucket.i += 1;
        }
    }
    return true;
}

// src/shmap/scoring.rs:172-178
inline double mapping_score(QPos inter, QPos m, QPos s_sz, Metric metric) {
    if (metric == Metric::Jaccard) return (double)inter / (double)(m + s_sz - inter);
    return (double)inter / (double)m;
}

// src/shmap/scoring.rs:189-291; the rarity-weighted support runs beside
// the count (scoring.rs:214-217, 240, 259, 280) and, under --rarity-weight,
// is the score
Mapping best_fixed_length(Ctx& cx, const RefSegment& segm, RPos from, RPos to, const PHt& p_ht,
                          const std::vector<Seed>& pu, std::vector<QPos>& diff_hist, QPos p_sz, QPos m,
                          Metric metric) {
    const auto& t = segm.kmers;
    RPos l = std::max(from, 0), r = l;
    const RPos end = std::min((RPos)t.size(), to);
    QPos inter = 0;
    int32_t same = 0;
    Mapping best;
    const bool weighted = !cx.rarity.empty();
    const bool score_weighted = weighted && cx.p.rarity_weight > 0.0;
    double w_inter = 0.0;
    while (l < end) {
        const Kmer& tl = t[(size_t)l];
        while (r < end) {
            const Kmer& tr = t[(size_t)r];
            bool in_window = cx.p.abs_pos ? tr.r < tl.r + m : r < l + m;
            if (!in_window) break;
            if (const int32_t* si = p_ht.get(tr.h)) {
                const Seed& seed = pu[(size_t)*si];
                same += seed.kmer.strand == tr.strand ? 1 : -1;
                QPos& cnt = diff_hist[(size_t)seed.seed_num];
                cnt -= 1;
                if (cnt >= 0) {
                    inter += 1;
                    if (weighted) w_inter += cx.rarity[(size_t)seed.seed_num];
                }
            }
            r += 1;
        }
        QPos s_kmers = r - l;
        double score = score_weighted ? std::min(std::max(w_inter / cx.m_weight, 0.0), 1.0)
                                      : mapping_score(inter, m, s_kmers, metric);
        if (l < r && score > best.score()) {
            best.rarity_support = w_inter;
            best.update(0, p_sz - 1, t[(size_t)l].r, t[(size_t)(r - 1)].r, segm, inter, score, same,
                        t[(size_t)(r - 1)].r - t[(size_t)l].r + 1);
        }
        if (const int32_t* si = p_ht.get(tl.h)) {
            const Seed& seed = pu[(size_t)*si];
            same -= seed.kmer.strand == tl.strand ? 1 : -1;
            QPos& cnt = diff_hist[(size_t)seed.seed_num];
            cnt += 1;
            if (cnt >= 1) {
                inter -= 1;
                if (weighted) w_inter -= cx.rarity[(size_t)seed.seed_num];
            }
        }
        l += 1;
    }
    return best;
}

// src/shmap/scoring.rs:114-170 (bucket_LCS): the read positions of every
// window k-mer found in p_ht (each seed's in decreasing order), then the
// longest strictly increasing subsequence of that list and of its reverse.
QPos lcs(const std::vector<Kmer>& t, RPos bgn, RPos bucket_end, const PHt& p_ht, const std::vector<Seed>& pu,
         const std::vector<std::vector<QPos>>& pmatches) {
    std::vector<QPos> pp;
    RPos end = std::min((RPos)t.size(), bucket_end);
    for (RPos l = bgn; l < end; l++)
        if (const int32_t* si = p_ht.get(t[(size_t)l].h))
            for (QPos q : pmatches[(size_t)pu[(size_t)*si].seed_num]) pp.push_back(q);
    auto lis = [](const std::vector<QPos>& v) {
        std::vector<QPos> s;
        for (QPos x : v) {
            auto it = std::lower_bound(s.begin(), s.end(), x);
            if (it == s.end()) s.push_back(x);
            else *it = x;
        }
        return s.size();
    };
    size_t fwd = lis(pp);
    std::reverse(pp.begin(), pp.end());
    size_t rev = lis(pp);
    return (QPos)std::max(fwd, rev);
}

// src/shmap/scoring.rs:38-109
struct RefineCache {
    enum Mode { Off, Record, Replay } mode = Off;
    std::vector<std::pair<uint32_t, Mapping>> entries;
    size_t cursor = 0;
    void start_recording() {
        entries.clear();
        cursor = 0;
        mode = Record;
    }
    void start_replay() {
        cursor = 0;
        mode = Replay;
    }
    long lookup(uint32_t idx) {
        if (mode != Replay) return -1;
        while (cursor < entries.size() && entries[cursor].first < idx) cursor++;
        if (cursor < entries.size() && entries[cursor].first == idx) return (long)cursor;
        return -1;
    }
    void record(uint32_t idx, const Mapping& m) {
        if (mode == Record) entries.emplace_back(idx, m);
    }
};

struct ReadState {
    const std::vector<Seed>& pu;
    const PHt& p_ht;
    std::vector<QPos>& diff_hist;
    const std::vector<std::vector<QPos>>& pmatches;
};

// src/shmap/scoring.rs:296-359
Mapping find_best_mapping(Ctx& cx, const Buckets& bk, BucketLoc b, const BucketContent& content, ReadState& rs,
                          QPos p_sz, QPos m, QPos lmax, double sh, Metric metric, QPos k) {
    Mapping mp;
    const RefSegment& segm = cx.tidx.segments[(size_t)b.segm_id];
    if (metric == Metric::BucketSh) {
        mp.update(0, p_sz - 1, content.r_min, content.r_max, segm, content.matches, sh, content.codirection,
                  content.r_max - content.r_min);
    } else if (metric == Metric::BucketLcs) {
        QPos c = lcs(segm.kmers, bk.begin(b), bk.end(b), rs.p_ht, rs.pu, rs.pmatches);
        mp.update(0, p_sz - 1, content.r_min, content.r_max, segm, content.matches, (double)c / (double)m,
                  content.codirection, content.r_max - content.r_min);
    } else {
        mp = best_fixed_length(cx, segm, bk.begin(b), bk.end(b), rs.p_ht, rs.pu, rs.diff_hist, p_sz - k, lmax, metric);
    }
    mp.bucket = b;
    mp.sh = sh;
    return mp;
}

// src/shmap/scoring.rs:367-489 (no rarity tie-break: admit == thr)
bool match_rest(Ctx& cx, QPos p_sz, QPos m, QPos lmax, const Buckets& bk,
                std::vector<std::pair<BucketLoc, BucketContent>>& sorted, ReadState& rs, double thr,
                const Mapping* forbidden, double max_overlap, Metric metric, QPos k, RefineCache& cache,
                Mapping& best) {
    bool have = false;
    const bool memoizable = metric == Metric::Containment || metric == Metric::Jaccard;
    for (size_t idx = 0; idx < sorted.size(); idx++) {
        BucketLoc b = sorted[idx].first;
        BucketContent& content = sorted[idx].second;
        double sh = 1.0;
        if (!seed_heuristic_pass(cx, bk, rs.pu, m, b, content, sh, thr)) continue;
        // scoring.rs:412-416: under a tie-break band a bucket slightly below
        // the incumbent is still scored
        const double tb = cx.p.rarity_tiebreak;
        const double admit = tb > 0.0 ? thr - tb * std::fabs(thr) : thr;
        long memo = memoizable ? cache.lookup((uint32_t)idx) : -1;
        bool got = false;
        Mapping bib;
        if (memo >= 0) {
            if (cache.entries[(size_t)memo].second.score() > admit) {
                bib = cache.entries[(size_t)memo].second;
                bib.sh = sh;
                got = true;
            }
        } else {
            Mapping scored = find_best_mapping(cx, bk, b, content, rs, p_sz, m, lmax, sh, metric, k);
            if (memoizable) cache.record((uint32_t)idx, scored);
            if (scored.score() > admit) {
                bib = scored;
                got = true;
            }
        }
        if (got) {
            cx.final_buckets += 1;
            if (!forbidden || Mapping::overlap(bib, *forbidden) < max_overlap) {
                bool take = !have;
                if (have) {  // scoring.rs:453-470: scores within the band are decided by rarity support
                    const bool tied = tb > 0.0 && std::fabs(bib.score() - best.score()) <= tb * std::fabs(best.score());
                    take = tied ? bib.rarity_support > best.rarity_support : bib.score() > best.score();
                }
                if (take) {
                    thr = std::max(thr, bib.score());
                    best = bib;
                    have = true;
                }
            }
        }
    }
    return have;
}

}  // namespace

QPos lcs_window(const std::vector<Kmer>& t, RPos bgn, RPos end, const std::vector<Hash>& seed_h,
                const std::vector<std::vector<QPos>>& seed_pos) {
    PHt p_ht;
    std::vector<Seed> pu(seed_h.size());
    for (size_t i = 0; i < seed_h.size(); i++) {
        bool ins;
        p_ht.get_or_insert(seed_h[i], &ins) = (int32_t)i;
        pu[i].seed_num = (QPos)i;
    }
    return lcs(t, bgn, end, p_ht, pu, seed_pos);
}

// The positions of each run of equal hashes of a sketch sorted by
// (h asc, r desc), by seed_num: the pmatches of src/shmap/seeding.rs:45-56.
static std::vector<std::vector<QPos>> group_positions(const std::vector<Kmer>& pk, size_t n_groups) {
    std::vector<std::vector<QPos>> pm(n_groups);
    size_t gs = 0, gi = 0;
    for (size_t ppos = 0; ppos < pk.size(); ppos++)
        if (ppos + 1 == pk.size() || pk[ppos].h != pk[ppos + 1].h) {
            for (size_t q = gs; q <= ppos; q++) pm[gi].push_back(pk[q].r);
            gi++;
            gs = ppos + 1;
        }
    return pm;
}

// src/shmap/mod.rs:653-971
ReadResult map_read(const SketchIndex& tidx, const FracMinHash& sk, const Params& p, const uint8_t* seq, size_t len,
                    Buckets& bk) {
    ReadResult rr;
    Ctx cx{tidx, p, 0, 0, 0, 0, {}, 0.0};
    bk.clear();
    std::vector<Kmer> pk = sk.sketch(seq, len);
    const QPos m = (QPos)pk.size();
    rr.read_len = (int32_t)len;
    rr.m = m;
    // pmatches (positions of each distinct hash, decreasing) for bucket_LCS only
    std::vector<std::vector<QPos>> pmatches;
    std::vector<Seed> pu = unique_elements_with_info(cx, pk);
    if (p.metric == Metric::BucketLcs) pmatches = group_positions(pk, pu.size());
    PHt p_ht;
    p_ht.reserve(pu.size());
    std::vector<QPos> diff_hist(pu.size(), 0);
    for (size_t i = 0; i < pu.size(); i++) {
        bool ins;
        p_ht.get_or_insert(pu[i].kmer.h, &ins) = (int32_t)i;
        diff_hist[(size_t)pu[i].seed_num] = pu[i].occs_in_p;
    }
    // src/shmap/mod.rs:694-723: rarity weights 1 / max(hits, 1)^alpha, in
    // rarest-first seed order; alpha follows --rarity-alpha, else
    // --rarity-weight, else 1 when only the tie-break is on
    const double alpha = p.rarity_alpha > 0.0    ? p.rarity_alpha
                         : p.rarity_weight > 0.0 ? p.rarity_weight
                         : p.rarity_tiebreak > 0.0 ? 1.0
                                                   : 0.0;
    if (alpha > 0.0) {
        cx.rarity.assign(pu.size(), 0.0);
        for (const Seed& sd : pu) {
            const double w = std::pow((double)std::max<RPos>(sd.hits_in_t, 1), -alpha);
            cx.rarity[(size_t)sd.seed_num] = w;
            cx.m_weight += w * (double)sd.occs_in_p;
        }
    }
    const QPos lmax = m;
    const double theta = p.theta;
    const double theta2 = theta - p.min_diff;
    const QPos s = p.one_sweep ? (QPos)pu.size() : f64_as_i32((1.0 - theta2) * (double)m) + 1;
    rr.s = s;
    const bool bucketable = bk.set_halflen(p.abs_pos ? (QPos)len : m);
    if (!bucketable) {
        rr.unmappable_short_sketch = true;
        return rr;
    }
    match_seeds(cx, pu, bk, s);
    bk.propagate_seeds_to_buckets();
    auto sorted = bk.get_sorted_buckets();
    rr.seeded_buckets = (int64_t)sorted.size();

    ReadState rs{pu, p_ht, diff_hist, pmatches};
    RefineCache cache;
    cache.start_recording();
    Mapping best, best2;
    bool have = match_rest(cx, (QPos)len, m, lmax, bk, sorted, rs, theta, nullptr, p.max_overlap, p.metric, p.k,
                           cache, best);
    bool have2 = false;
    if (have) {
        double thr2 = best.score() * (1.0 - p.min_diff);
        cache.start_replay();
        have2 = match_rest(cx, (QPos)len, m, lmax, bk, sorted, rs, thr2, &best, p.max_overlap, p.metric, p.k, cache,
                           best2);
    }
    rr.total_matches = cx.total_matches;
    rr.seed_matches = cx.seed_matches;
    rr.max_seed_matches = cx.max_seed_matches;
    rr.final_buckets = cx.final_buckets;
    rr.mapped = have;
    rr.best = best;
    rr.has2 = have2;
    rr.best2 = best2;
    return rr;
}

ReadResult map_read(const SketchIndex& tidx, const FracMinHash& sk, const Params& p, const uint8_t* seq,
                    size_t len) {
    Buckets bk(tidx, p.abs_pos);
    return map_read(tidx, sk, p, seq, len, bk);
}

std::vector<ReadResult> map_reads(const SketchIndex& tidx, const FracMinHash& sk, const Params& p,
                                  const std::vector<const uint8_t*>& seqs, const std::vector<size_t>& lens,
                                  int threads) {
    std::vector<ReadResult> out(seqs.size());
    std::atomic<size_t> next{0};
    threads = std::max(1, threads);
    auto work = [&]() {
        Buckets bk(tidx, p.abs_pos);  // one per worker, reused across reads (mod.rs:484-485)
        for (size_t i; (i = next.fetch_add(1)) < seqs.size();) out[i] = map_read(tidx, sk, p, seqs[i], lens[i], bk);
    };
    std::vector<std::thread> ts;
    for (int t = 0; t < threads; t++) ts.emplace_back(work);
    for (auto& t : ts) t.join();
    return out;
}

// src/shmap/mod.rs:374-650 with the collector's output (mod.rs:868-963): the
// workers map reads and render each mapped read's PAF line (t:f: printed as
// map_time = 0); the lines are then joined in input order, as the in-order
// collector writes them. Results keep the state before render_paf's
// post-processing (second best, mapq) in `res`; `lines` get the text.
void map_reads_paf(const SketchIndex& tidx, const FracMinHash& sk, const Params& p,
                   const std::vector<const uint8_t*>& seqs, const std::vector<size_t>& lens,
                   const std::vector<std::string>& names, int threads, std::vector<ReadResult>& res,
                   std::string& text) {
    res.assign(seqs.size(), ReadResult());
    std::vector<std::string> lines(seqs.size());
    std::atomic<size_t> next{0};
    threads = std::max(1, threads);
    auto work = [&]() {
        Buckets bk(tidx, p.abs_pos);
        for (size_t i; (i = next.fetch_add(1)) < seqs.size();) {
            res[i] = map_read(tidx, sk, p, seqs[i], lens[i], bk);
            if (res[i].mapped) {
                ReadResult copy = res[i];
                lines[i] = render_paf(copy, names[i], p, 0.0);
                lines[i] += '\n';
            }
        }
    };
    std::vector<std::thread> ts;
    for (int t = 0; t < threads; t++) ts.emplace_back(work);
    for (auto& t : ts) t.join();
    size_t total = 0;
    for (auto& l : lines) total += l.size();
    text.clear();
    text.reserve(total);
    for (auto& l : lines) text += l;
}

// src/shmap/mod.rs:871-943 with mapping.rs:356-408
std::string render_paf(ReadResult& rr, const std::string& query_id, const Params& p, double map_time) {
    Mapping& best = rr.best;
    if (rr.has2) best.set_second_best(rr.best2);
    const double theta2 = p.theta - p.min_diff;
    best.read_len = rr.read_len;
    best.mapq = best.calc_mapq(theta2, p.min_diff);
    best.p_sz = rr.m;
    best.map_time = map_time;
    best.has_global = true;
    best.g_k = p.k;
    best.g_seeds = rr.s;
    best.total_matches = (RPos)rr.total_matches;
    best.max_seed_matches = (RPos)rr.max_seed_matches;
    best.seed_matches = (RPos)rr.seed_matches;
    best.seeded_buckets = (RPos)rr.seeded_buckets;
    best.final_buckets = (RPos)rr.final_buckets;
    best.fptp = -1.0;
    best.match_inefficiency = (double)best.total_matches / (double)best.intersection;
    return best.paf(query_id);
}

// ---------------------------------------------------------------- io
// String::from_utf8_lossy, which src/io/mod.rs:408-410 applies to every
// record id: each maximal subpart of an ill-formed UTF-8 sequence becomes one
// U+FFFD, per the Unicode standard's well-formed byte sequence table.
static std::string from_utf8_lossy(const std::string& s) {
    std::string out;
    size_t i = 0;
    const size_t n = s.size();
    while (i < n) {
        const unsigned char c = (unsigned char)s[i];
        if (c < 0x80) {
            out.push_back((char)c);
            i++;
            continue;
        }
        int len = 0;
        unsigned char first_lo = 0x80, first_hi = 0xbf;
        if (c >= 0xc2 && c <= 0xdf) {
            len = 2;
        } else if (c >= 0xe0 && c <= 0xef) {
            len = 3;
            if (c == 0xe0) first_lo = 0xa0;
            if (c == 0xed) first_hi = 0x9f;
        } else if (c >= 0xf0 && c <= 0xf4) {
            len = 4;
            if (c == 0xf0) first_lo = 0x90;
            if (c == 0xf4) first_hi = 0x8f;
        }
        size_t k = 1;
        if (len) {
            for (; k < (size_t)len && i + k < n; k++) {
                const unsigned char d = (unsigned char)s[i + k];
                const unsigned char lo = k == 1 ? first_lo : 0x80, hi = k == 1 ? first_hi : 0xbf;
                if (d < lo || d > hi) break;
            }
        }
        if (len && k == (size_t)len) out.append(s, i, k);
        else out += "\xef\xbf\xbd";
        i += k;
    }
    return out;
}

bool read_fasta(const std::string& path, std::vector<FastaRecord>& out, std::string* err) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) {
        if (err) *err = "failed to open " + path;
        return false;
    }
    std::string data;
    char chunk[1 << 16];
    for (size_t got; (got = std::fread(chunk, 1, sizeof chunk, f)) > 0;) data.append(chunk, got);
    std::fclose(f);
    size_t pos = 0, n = data.size();
    FastaRecord* cur = nullptr;
    while (pos < n) {
        size_t e = data.find('\n', pos);
        if (e == std::string::npos) e = n;
        size_t le = e;
        if (le > pos && data[le - 1] == '\r') le--;
        if (le > pos && data[pos] == '>') {
            std::string hdr = data.substr(pos + 1, le - pos - 1);
            size_t cut = hdr.find_first_of(" \t");
            out.push_back(FastaRecord{from_utf8_lossy(cut == std::string::npos ? hdr : hdr.substr(0, cut)),
                                      std::string()});
            cur = &out.back();
        } else if (cur) {
            cur->seq.append(data, pos, le - pos);
        } else if (le > pos) {
            if (err) *err = "invalid FASTA record in " + path;
            return false;
        }
        pos = e + 1;
    }
    return true;
}

}  // namespace oracle

// Test hooks (test infrastructure): the bucket accumulator, Mapping and the
// seed grouping driven directly, for the reference's own unit tests of them
// (src/buckets.rs:748-957, src/mapping.rs:445-495, src/shmap/seeding.rs:221-245).
namespace {
struct OrcBuckets {
    oracle::SketchIndex idx;
    oracle::Buckets b;
    OrcBuckets(int32_t sz, int32_t n_kmers, bool ap) : b(idx, ap) {
        oracle::RefSegment sg;
        sg.kmers.assign((size_t)n_kmers, oracle::Kmer{0, 0, false});
        sg.name = "seg0";
        sg.sz = sz;
        sg.id = 0;
        idx.segments.push_back(std::move(sg));
    }
};
struct OrcMapping {
    oracle::Mapping m;
    std::vector<std::unique_ptr<oracle::RefSegment>> segs;
};
}  // namespace

extern "C" {
void* orc_buckets_new(int32_t seg_sz, int32_t n_kmers, int32_t ap) { return new OrcBuckets(seg_sz, n_kmers, ap != 0); }
void orc_buckets_free(void* p) { delete (OrcBuckets*)p; }
int32_t orc_buckets_set_halflen(void* p, int32_t h) { return ((OrcBuckets*)p)->b.set_halflen(h) ? 1 : 0; }
int32_t orc_buckets_dense_on(void* p) { return ((OrcBuckets*)p)->b.dense_on ? 1 : 0; }
int32_t orc_buckets_begin(void* p, int32_t segm, int32_t bb) {
    return ((OrcBuckets*)p)->b.begin(oracle::BucketLoc{segm, bb});
}
int32_t orc_buckets_end(void* p, int32_t segm, int32_t bb) { return ((OrcBuckets*)p)->b.end(oracle::BucketLoc{segm, bb}); }
void orc_buckets_add_to_pos(void* p, int32_t r, int32_t tpos, int32_t segm, int32_t matches, int32_t seeds,
                            int32_t codir, int32_t rmin, int32_t rmax) {
    oracle::BucketContent c;
    c.matches = matches;
    c.seeds = seeds;
    c.codirection = codir;
    c.r_min = rmin;
    c.r_max = rmax;
    ((OrcBuckets*)p)->b.add_to_pos(oracle::Hit{r, tpos, false, segm}, c);
}
void orc_buckets_propagate(void* p) { ((OrcBuckets*)p)->b.propagate_seeds_to_buckets(); }
void orc_buckets_clear(void* p) { ((OrcBuckets*)p)->b.clear(); }
// Sorted buckets as 6 ints each: segm_id, b, matches, codirection, r_min, r_max.
int64_t orc_buckets_sorted(void* p, int32_t* out, int64_t cap) {
    auto v = ((OrcBuckets*)p)->b.get_sorted_buckets();
    for (size_t i = 0; i < v.size() && (int64_t)i < cap; i++) {
        const auto& [loc, c] = v[i];
        int32_t* o = out + 6 * i;
        o[0] = loc.segm_id;
        o[1] = loc.b;
        o[2] = c.matches;
        o[3] = c.codirection;
        o[4] = c.r_min;
        o[5] = c.r_max;
    }
    return (int64_t)v.size();
}

void* orc_mapping_new(void) { return new OrcMapping(); }
void orc_mapping_free(void* p) { delete (OrcMapping*)p; }
void orc_mapping_update(void* p, int32_t ps, int32_t pe, int32_t tl, int32_t tr, int32_t seg_id, int32_t seg_sz,
                        int32_t inter, double score, int32_t same, int32_t sz) {
    auto* o = (OrcMapping*)p;
    auto sg = std::make_unique<oracle::RefSegment>();
    sg->name = "chr" + std::to_string(seg_id + 1);
    sg->sz = seg_sz;
    sg->id = seg_id;
    o->m.update(ps, pe, tl, tr, *sg, inter, score, same, sz);
    o->segs.push_back(std::move(sg));
}
void orc_mapping_get(void* p, double* score, int32_t* t_l, char* strand) {
    auto* o = (OrcMapping*)p;
    *score = o->m.score();
    *t_l = o->m.t_l;
    *strand = o->m.strand;
}
double orc_mapping_overlap(void* a, void* b) { return oracle::Mapping::overlap(((OrcMapping*)a)->m, ((OrcMapping*)b)->m); }
int32_t orc_mapping_calc_mapq(void* p, double theta2, double min_diff) {
    return ((OrcMapping*)p)->m.calc_mapq(theta2, min_diff);
}
// Seeds of a sketch (r, h, strand) against an empty index, in the order
// unique_elements_with_info returns them: hash, occurrences and pmatches
// (pm[pm_off[i] .. pm_off[i + 1])). Returns the number of seeds.
int64_t orc_seed_groups(const int32_t* r, const uint64_t* h, const uint8_t* strand, int32_t n, uint64_t* out_h,
                        int32_t* out_occ, int32_t* pm_off, int32_t* pm) {
    oracle::SketchIndex idx;
    oracle::Params prm;
    oracle::Ctx cx{idx, prm, 0, 0, 0, 0, {}, 0.0};
    std::vector<oracle::Kmer> pk((size_t)n);
    for (int32_t i = 0; i < n; i++) pk[(size_t)i] = oracle::Kmer{r[i], h[i], strand[i] != 0};
    std::vector<oracle::Seed> pu = oracle::unique_elements_with_info(cx, pk);
    std::vector<std::vector<oracle::QPos>> pmv = oracle::group_positions(pk, pu.size());
    int32_t at = 0;
    for (size_t i = 0; i < pu.size(); i++) {
        out_h[i] = pu[i].kmer.h;
        out_occ[i] = pu[i].occs_in_p;
        pm_off[i] = at;
        for (oracle::QPos q : pmv[(size_t)pu[i].seed_num]) pm[at++] = q;
    }
    pm_off[pu.size()] = at;
    return (int64_t)pu.size();
}
// read_fasta (src/io/mod.rs:383-427) of a file: *n records, *name_bytes
// bytes of '\n'-joined names, *seq_bytes bases; with buffers given, also the
// names, the bases back to back and n+1 offsets. Returns 0, or -1 with the
// message in names (when it fits) on a read error.
int32_t orc_read_fasta(const char* path, int64_t* n, int64_t* name_bytes, int64_t* seq_bytes, char* names,
                       uint8_t* seq, int64_t* offs) {
    std::vector<oracle::FastaRecord> recs;
    std::string err;
    if (!oracle::read_fasta(path, recs, &err)) return -1;
    std::string joined;
    int64_t total = 0;
    for (size_t i = 0; i < recs.size(); i++) {
        if (i) joined += '\n';
        joined += recs[i].name;
        total += (int64_t)recs[i].seq.size();
    }
    *n = (int64_t)recs.size();
    *name_bytes = (int64_t)joined.size();
    *seq_bytes = total;
    if (names) std::memcpy(names, joined.data(), joined.size());
    if (seq && offs) {
        int64_t at = 0;
        offs[0] = 0;
        for (size_t i = 0; i < recs.size(); i++) {
            std::memcpy(seq + at, recs[i].seq.data(), recs[i].seq.size());
            at += (int64_t)recs[i].seq.size();
            offs[i + 1] = at;
        }
    }
    return 0;
}
}  // extern "C"
