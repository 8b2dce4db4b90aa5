// TEST INFRASTRUCTURE ONLY. This is the CPU oracle: a sequential C++ restatement
// of shmap-rs v1.4.3's long-read mapping path, used by tests/, by smoke() and by
// bench.py's cpu_baseline / reference arm as the checker and the timed CPU
// baseline. The product (shmap-rs_b200/) never links, loads or calls it.
//
// It follows the reference one function at a time, in the reference's own
// shape (sequential per read, in-place pruning state, a RefineCache memo), so
// that it checks the GPU path's reformulations instead of sharing them.
// Every function cites the reference file:line it restates. Parity of the
// oracle itself is pinned by the reference's golden PAF and known-answer tests
// (tests/golden/, tests/test_oracle_golden.py).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace oracle {

using Hash = uint64_t;
using RPos = int32_t;
using QPos = int32_t;
using SegmId = int32_t;

// src/types.rs:23-33
struct Kmer {
    RPos r;
    Hash h;
    bool strand;
};

// src/types.rs:43-61
struct Hit {
    RPos r;
    RPos tpos;
    bool strand;
    SegmId segm_id;
};

// src/types.rs:131-151 (pmatches kept as a vector; only its length is used here)
struct Seed {
    Kmer kmer;
    RPos hits_in_t;
    QPos occs_in_p;
    QPos seed_num;
};

// src/types.rs:203-226
struct BucketLoc {
    SegmId segm_id = -1;
    RPos b = -1;
    bool operator==(const BucketLoc& o) const { return segm_id == o.segm_id && b == o.b; }
};

// src/types.rs:236-281
struct BucketContent {
    int32_t i = -1;
    QPos seeds = 0;
    QPos matches = 0;
    int32_t codirection = 0;
    RPos r_min = INT32_MAX;
    RPos r_max = -1;
    void add(const BucketContent& o) {
        matches += o.matches;
        seeds += o.seeds;
        codirection += o.codirection;
        if (o.r_min < r_min) r_min = o.r_min;
        if (o.r_max > r_max) r_max = o.r_max;
    }
};

// src/types.rs:299-322
enum class Metric : int32_t { Containment = 0, Jaccard = 1, BucketSh = 2, BucketLcs = 3 };

// src/sketch.rs:34-219
class FracMinHash {
public:
    FracMinHash(int32_t k, double h_frac);
    Hash h_thres() const;                                         // sketch.rs:126-132
    void sketch_slice_into(const uint8_t* s, size_t n, RPos offset,
                           std::vector<Kmer>& out) const;          // sketch.rs:167-209
    std::vector<Kmer> sketch(const uint8_t* s, size_t n) const {  // sketch.rs:113-122
        std::vector<Kmer> v;
        sketch_slice_into(s, n, 0, v);
        return v;
    }
    int32_t k;
    double h_frac;

private:
    Hash lut_fw[256], lut_rc[256], lut_fw_k[256], lut_rc_r1[256], lut_rc_k1[256];
};

// src/sketch.rs:16-27
struct RefSegment {
    std::vector<Kmer> kmers;
    std::string name;
    RPos sz;
    int32_t id;
};

// A FxHashMap<Hash, V> stand-in: open addressing, power-of-two capacity.
// Only lookups are made by hash, never iteration in an output-affecting order.
template <class V>
class HashMap {
public:
    void reserve(size_t n);
    V* get(Hash h);
    const V* get(Hash h) const;
    V& get_or_insert(Hash h, bool* inserted);
    bool erase(Hash h);  // tombstone-free: used only before any further inserts
    template <class F> void for_each(F f);
    size_t size() const { return n_; }

private:
    static uint64_t mix(Hash h) { return (h ^ (h >> 29)) * 0xbf58476d1ce4e5b9ULL; }
    void grow();
    std::vector<Hash> keys_;
    std::vector<uint8_t> used_;
    std::vector<V> vals_;
    size_t n_ = 0;
};

// src/index.rs:104-110
struct Shard {
    HashMap<Hit> h2single;
    HashMap<std::vector<Hit>> h2multi;
};

struct IndexCounters {
    int64_t segments = 0, total_nucls = 0, indexed_hits = 0, indexed_kmers = 0,
            indexed_highest_freq_kmer = 0, blacklisted_kmers = 0, blacklisted_hits = 0,
            sketched_kmers = 0;
};

// src/index.rs:112-125 (8 hash shards by the low 3 bits, index.rs:73-99)
class SketchIndex {
public:
    static constexpr int N_SHARDS = 8;
    std::vector<RefSegment> segments;
    Shard shards[N_SHARDS];
    IndexCounters counters;

    // src/index.rs:384-663, with the sequence already read: segments in file order.
    void build_index(const std::vector<std::string>& names, const std::vector<const uint8_t*>& seqs,
                     const std::vector<size_t>& lens, const FracMinHash& sk, int32_t max_matches,
                     int threads);
    RPos count(Hash h) const;                         // index.rs:204-213
    Hit single_hit(Hash h) const;                     // index.rs:192-194
    const std::vector<Hit>& multi_hits(Hash h) const; // index.rs:199-201
};

// src/params.rs:20-186 (the fields the mapping path reads)
struct Params {
    int32_t k = 15;
    double h_frac = 0.05;
    int32_t max_matches = -1;  // -M; -1 = None
    double theta = 0.9;
    double min_diff = 0.02;
    double max_overlap = 0.5;
    Metric metric = Metric::Containment;
    bool no_bucket_pruning = false;  // -P (NBP)
    bool one_sweep = false;          // -B (OS)
    bool abs_pos = false;            // -F (AP)
    double rarity_weight = 0.0;      // --rarity-weight (params.rs:76-77)
    double rarity_tiebreak = 0.0;    // --rarity-tiebreak (params.rs:95-96)
    double rarity_alpha = 0.0;       // --rarity-alpha (params.rs:111-112)
    int threads = 1;
};

// src/mapping.rs:12-27, 110-136, 185-207, 253-257 folded into one record.
struct Mapping {
    // MappingPaf
    QPos p_start = -1, p_end = -1;
    char strand = '?';
    const RefSegment* segm = nullptr;
    SegmId segm_id = -1;
    RPos t_l = -1, t_r = -1;
    uint8_t mapq = 255;
    QPos read_len = -1;
    // LocalMappingStats
    RPos s_sz = -1;
    QPos intersection = -1;
    double map_time = -1.0;
    int32_t same_strand_seeds = -1;
    double j = -1.0, j2 = -1.0, sh = -1.0;
    QPos p_sz = -1;
    BucketLoc bucket, bucket2;
    QPos intersection2 = -1;
    double sigmas_diff = -1.0;
    double rarity_support = 0.0;  // mapping.rs:124-128 (never printed)
    // GlobalMappingStats
    bool has_global = false;
    QPos g_k = -1, g_seeds = -1;
    RPos max_seed_matches = -1, seed_matches = -1, total_matches = -1;
    double match_inefficiency = -1.0;
    RPos seeded_buckets = -1, final_buckets = -1;
    double fptp = -1.0;

    double score() const { return j; }
    void update(QPos p_start, QPos p_end, RPos t_l, RPos t_r, const RefSegment& segm,
                QPos intersection, double new_score, int32_t same_strand_seeds, RPos sz);  // mapping.rs:299-327
    uint8_t calc_mapq(double theta2, double min_diff);                                      // mapping.rs:341-354
    void set_second_best(const Mapping& m2);                                                // mapping.rs:356-361
    static double overlap(const Mapping& a, const Mapping& b);                              // mapping.rs:412-420
    std::string paf(const std::string& query_id) const;                                     // mapping.rs:87-107,161-182,228-247
};

// One read's outcome, flattened for comparison with the device path's records.
struct ReadResult {
    bool mapped = false;
    bool unmappable_short_sketch = false;
    Mapping best;
    bool has2 = false;
    Mapping best2;
    int32_t read_len = 0, m = 0, s = 0;
    int64_t total_matches = 0, max_seed_matches = 0, seed_matches = 0, seeded_buckets = 0,
            final_buckets = 0;
};

// src/shmap/mod.rs:653-971 for one read (no wall-clock work inside).
ReadResult map_read(const SketchIndex& tidx, const FracMinHash& sk, const Params& p,
                    const uint8_t* seq, size_t len);

// src/shmap/mod.rs:374-650: map every read, results in input order, -@ threads.
std::vector<ReadResult> map_reads(const SketchIndex& tidx, const FracMinHash& sk, const Params& p,
                                  const std::vector<const uint8_t*>& seqs,
                                  const std::vector<size_t>& lens, int threads);

// map_reads plus the collector's in-order PAF text (mod.rs:374-650, 868-963):
// every mapped read's line, t:f: printed as 0, joined in input order.
void map_reads_paf(const SketchIndex& tidx, const FracMinHash& sk, const Params& p,
                   const std::vector<const uint8_t*>& seqs, const std::vector<size_t>& lens,
                   const std::vector<std::string>& names, int threads, std::vector<ReadResult>& res,
                   std::string& text);

// Fills the global stats and renders the reference's PAF line (mod.rs:871-943).
std::string render_paf(ReadResult& rr, const std::string& query_id, const Params& p, double map_time);

// src/mapping.rs:82-84
std::string unmapped_line(const std::string& query_id, QPos read_len);

// needletail-compatible FASTA reading (src/io/mod.rs:383-427): id cut at the
// first space or tab, sequence lines joined with \n and \r removed.
struct FastaRecord {
    std::string name;
    std::string seq;
};
bool read_fasta(const std::string& path, std::vector<FastaRecord>& out, std::string* err);

// bucket_LCS's count for the window [bgn, end) of a reference sketch t, with
// the read's seeds given as hashes and their positions (scoring.rs:114-170).
QPos lcs_window(const std::vector<Kmer>& t, RPos bgn, RPos end, const std::vector<Hash>& seed_h,
                const std::vector<std::vector<QPos>>& seed_pos);

}  // namespace oracle
