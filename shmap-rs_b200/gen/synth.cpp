// Seeded synthetic references and long reads with the shapes of the benchmark
// workloads (uniform contigs; a human-scale genome with tandem satellite arrays
// and interspersed repeats; HiFi/ONT-like reads with sub/ins/del errors).
//
// Every base is a pure function of (seed, position) through a counter-based
// generator, so a genome can be filled by any number of threads and always
// comes out the same. Read headers follow `S<i>_1!<chr>!<start>!<end>!<strand>`,
// the convention of the reference's read simulator (simulate/simulate_reads.py).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace {

inline uint64_t splitmix(uint64_t x) {
    x += 0x9e3779b97f4a7c15ULL;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}
inline uint64_t h3(uint64_t a, uint64_t b, uint64_t c) { return splitmix(splitmix(splitmix(a) ^ b) ^ c); }
inline double u01(uint64_t x) { return (double)(x >> 11) * (1.0 / 9007199254740992.0); }

const char BASES[4] = {'A', 'C', 'G', 'T'};

struct Rng {  // sequential stream for planning and for read errors
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed) {}
    uint64_t next() { return splitmix(s += 0x632be59bd9b4e019ULL); }
    double uni() { return u01(next()); }
    uint64_t below(uint64_t n) { return n ? next() % n : 0; }
    double normal() {
        double u1 = std::max(uni(), 1e-300), u2 = uni();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

// A stretch of a contig copied from a consensus with per-copy substitutions.
struct Feature {
    int64_t start, len;   // in contig coordinates
    int32_t family;       // index into consensus list
    int32_t period;       // tandem period (monomer length); 0 = single copy of a repeat
    double divergence;    // per-base substitution rate against the consensus
    uint64_t key;         // per-feature hash key
};

}  // namespace

extern "C" {

struct synth_ref_cfg {
    uint64_t seed;
    int64_t total_bases;     // sum of contig lengths
    int32_t n_contigs;
    int64_t min_contig;      // every contig is at least this long
    double satellite_frac;   // fraction of bases in tandem satellite arrays
    double repeat_frac;      // fraction of bases in interspersed repeats
    int32_t repeat_len;      // interspersed repeat length (6 kb)
    double repeat_div;       // their divergence (0.10)
    double sat_div_lo, sat_div_hi;  // satellite copy divergence range (0.01..0.03)
    int64_t sat_array_lo, sat_array_hi;  // satellite array length range
};

struct synth_read_cfg {
    uint64_t seed;
    int32_t n_reads;
    double len_mean, len_sd;      // lognormal; sd 0 = fixed length
    int64_t len_min, len_max;     // clipping
    double err_rate;              // per-base error probability
    double sub_w, ins_w, del_w;   // split of errors
    double satellite_read_frac;   // fraction of reads started inside a satellite array
};

}  // extern "C"

namespace {

struct Genome {
    synth_ref_cfg cfg;
    std::vector<int64_t> contig_len, contig_off;
    std::vector<std::string> names;
    std::vector<std::vector<Feature>> features;  // per contig, sorted by start, disjoint
    std::vector<std::string> consensus;          // families: satellites then repeats
    std::vector<std::pair<int32_t, size_t>> sat_arrays;  // (contig, feature index)
    int64_t total = 0;
};

inline char random_base(uint64_t seed, int32_t contig, int64_t pos) {
    uint64_t w = h3(seed, (uint64_t)contig + 1, (uint64_t)(pos >> 5));
    return BASES[(w >> (2 * (pos & 31))) & 3];
}

inline char feature_base(const Genome& g, const Feature& f, int64_t pos) {
    const std::string& cons = g.consensus[(size_t)f.family];
    int64_t off = pos - f.start;
    int64_t ci = f.period > 0 ? off % f.period : off % (int64_t)cons.size();
    char b = cons[(size_t)ci];
    uint64_t x = h3(f.key, (uint64_t)off, 0x5bd1e995ULL);
    if (u01(x) < f.divergence) {
        int bi = (int)(std::find(BASES, BASES + 4, b) - BASES);
        b = BASES[(bi + 1 + (int)((x >> 8) % 3)) & 3];
    }
    return b;
}

void plan_genome(Genome& g) {
    const synth_ref_cfg& c = g.cfg;
    Rng rng(splitmix(c.seed ^ 0x1111));
    const int32_t n = std::max(1, c.n_contigs);
    std::vector<double> w((size_t)n);
    double sw = 0;
    for (auto& x : w) sw += (x = 0.2 + rng.uni());
    int64_t spare = c.total_bases - (int64_t)n * c.min_contig;
    if (spare < 0) spare = 0;
    int64_t acc = 0;
    for (int32_t i = 0; i < n; i++) {
        int64_t L = c.min_contig + (int64_t)std::floor((double)spare * w[(size_t)i] / sw);
        if (i == n - 1) L = c.total_bases - acc;
        g.contig_off.push_back(acc);
        g.contig_len.push_back(L);
        acc += L;
        char nm[32];
        std::snprintf(nm, sizeof nm, "chr%d", i + 1);
        g.names.push_back(nm);
    }
    g.total = acc;
    g.features.assign((size_t)n, {});
    auto rand_seq = [&](int64_t len) {
        std::string s((size_t)len, 'A');
        for (auto& ch : s) ch = BASES[rng.below(4)];
        return s;
    };
    // occupancy check against features already placed in a contig
    auto fits = [&](int32_t ci, int64_t s, int64_t len) {
        if (s < 0 || s + len > g.contig_len[(size_t)ci]) return false;
        for (const Feature& f : g.features[(size_t)ci])
            if (s < f.start + f.len && f.start < s + len) return false;
        return true;
    };
    auto pick_contig = [&]() {
        uint64_t x = rng.below((uint64_t)g.total);
        return (int32_t)(std::upper_bound(g.contig_off.begin(), g.contig_off.end(), (int64_t)x) - g.contig_off.begin() - 1);
    };
    // tandem satellite arrays: each array has its own monomer family (171 bp or 2 kb)
    int64_t sat_target = (int64_t)(c.satellite_frac * (double)g.total);
    int64_t placed = 0;
    int guard = 0;
    while (placed < sat_target && guard++ < 1000000) {
        int32_t period = rng.uni() < 0.5 ? 171 : 2000;
        int64_t len = c.sat_array_lo + (int64_t)rng.below((uint64_t)std::max<int64_t>(1, c.sat_array_hi - c.sat_array_lo));
        len = std::min(len, sat_target - placed + period);
        len = std::max<int64_t>(len, 2 * period);
        int32_t ci = pick_contig();
        int64_t maxs = g.contig_len[(size_t)ci] - len;
        if (maxs <= 0) continue;
        int64_t s = (int64_t)rng.below((uint64_t)maxs);
        if (!fits(ci, s, len)) continue;
        int32_t fam = (int32_t)g.consensus.size();
        g.consensus.push_back(rand_seq(period));
        double div = c.sat_div_lo + (c.sat_div_hi - c.sat_div_lo) * rng.uni();
        g.features[(size_t)ci].push_back(Feature{s, len, fam, period, div, rng.next()});
        placed += len;
    }
    // interspersed repeats: a few families of repeat_len, copies at repeat_div
    int64_t rep_target = (int64_t)(c.repeat_frac * (double)g.total);
    const int n_fam = 16;
    int32_t fam0 = (int32_t)g.consensus.size();
    if (rep_target > 0 && c.repeat_len > 0)
        for (int i = 0; i < n_fam; i++) g.consensus.push_back(rand_seq(c.repeat_len));
    placed = 0;
    guard = 0;
    while (rep_target > 0 && c.repeat_len > 0 && placed < rep_target && guard++ < 10000000) {
        int32_t ci = pick_contig();
        int64_t maxs = g.contig_len[(size_t)ci] - c.repeat_len;
        if (maxs <= 0) continue;
        int64_t s = (int64_t)rng.below((uint64_t)maxs);
        // only check the nearest neighbours after sorting lazily: keep it simple, check all on small counts
        bool ok = true;
        auto& fv = g.features[(size_t)ci];
        if (fv.size() < 64) ok = fits(ci, s, c.repeat_len);
        else {
            // fv is kept sorted once it grows; binary search the neighbourhood
            auto it = std::lower_bound(fv.begin(), fv.end(), s, [](const Feature& f, int64_t v) { return f.start < v; });
            if (it != fv.end() && it->start < s + c.repeat_len) ok = false;
            if (it != fv.begin() && (it - 1)->start + (it - 1)->len > s) ok = false;
        }
        if (!ok) continue;
        Feature f{s, c.repeat_len, fam0 + (int32_t)rng.below(n_fam), 0, c.repeat_div, rng.next()};
        if (fv.size() < 64) {
            fv.push_back(f);
            if (fv.size() == 64)
                std::sort(fv.begin(), fv.end(), [](const Feature& a, const Feature& b) { return a.start < b.start; });
        } else {
            auto it = std::lower_bound(fv.begin(), fv.end(), s, [](const Feature& x, int64_t v) { return x.start < v; });
            fv.insert(it, f);
        }
        placed += c.repeat_len;
    }
    for (size_t ci = 0; ci < g.features.size(); ci++) {
        auto& fv = g.features[ci];
        std::sort(fv.begin(), fv.end(), [](const Feature& a, const Feature& b) { return a.start < b.start; });
        for (size_t fi = 0; fi < fv.size(); fi++)
            if (fv[fi].period > 0) g.sat_arrays.emplace_back((int32_t)ci, fi);
    }
}

void fill_contig_range(const Genome& g, int32_t ci, int64_t a, int64_t b, uint8_t* out) {
    const auto& fv = g.features[(size_t)ci];
    auto it = std::upper_bound(fv.begin(), fv.end(), a, [](int64_t v, const Feature& f) { return v < f.start; });
    size_t fi = (it == fv.begin()) ? 0 : (size_t)(it - fv.begin() - 1);
    for (int64_t p = a; p < b; p++) {
        while (fi < fv.size() && fv[fi].start + fv[fi].len <= p) fi++;
        if (fi < fv.size() && fv[fi].start <= p) out[p - a] = (uint8_t)feature_base(g, fv[fi], p);
        else out[p - a] = (uint8_t)random_base(g.cfg.seed, ci, p);
    }
}

struct ReadPlan {
    int32_t contig;
    int64_t start, len;  // reference span
    bool rev;
    uint64_t key;
};

struct ReadSet {
    synth_read_cfg cfg;
    std::vector<ReadPlan> plan;
    std::vector<int64_t> out_len;  // filled by the first fill pass (lengths after indels)
};

}  // namespace

extern "C" {

void* synth_ref_create(const synth_ref_cfg* cfg) {
    auto* g = new Genome();
    g->cfg = *cfg;
    plan_genome(*g);
    return g;
}
void synth_ref_free(void* p) { delete (Genome*)p; }
int64_t synth_ref_total(void* p) { return ((Genome*)p)->total; }
int32_t synth_ref_nseg(void* p) { return (int32_t)((Genome*)p)->contig_len.size(); }
int64_t synth_ref_num_sat_arrays(void* p) { return (int64_t)((Genome*)p)->sat_arrays.size(); }

// seg_off: n_seg+1 entries. names: '\n'-joined into a buffer of names_cap bytes.
void synth_ref_segments(void* p, int64_t* seg_off, char* names, int64_t names_cap) {
    Genome* g = (Genome*)p;
    std::string joined;
    for (size_t i = 0; i < g->contig_len.size(); i++) {
        seg_off[i] = g->contig_off[i];
        if (i) joined += '\n';
        joined += g->names[i];
    }
    seg_off[g->contig_len.size()] = g->total;
    if (names && names_cap > 0) {
        size_t n = std::min((size_t)names_cap - 1, joined.size());
        std::memcpy(names, joined.data(), n);
        names[n] = 0;
    }
}

// Fills all bases of the genome (concatenated in contig order) with `threads` threads.
void synth_ref_fill(void* p, uint8_t* out, int32_t threads) {
    Genome* g = (Genome*)p;
    const int64_t CH = 1 << 22;
    std::vector<std::pair<int32_t, int64_t>> jobs;
    for (size_t ci = 0; ci < g->contig_len.size(); ci++)
        for (int64_t a = 0; a < g->contig_len[ci]; a += CH) jobs.emplace_back((int32_t)ci, a);
    std::atomic<size_t> next{0};
    auto work = [&]() {
        for (size_t j; (j = next.fetch_add(1)) < jobs.size();) {
            int32_t ci = jobs[j].first;
            int64_t a = jobs[j].second, b = std::min(a + CH, g->contig_len[(size_t)ci]);
            fill_contig_range(*g, ci, a, b, out + g->contig_off[(size_t)ci] + a);
        }
    };
    std::vector<std::thread> ts;
    for (int t = 0; t < std::max(1, threads); t++) ts.emplace_back(work);
    for (auto& t : ts) t.join();
}

void* synth_reads_create(void* refp, const synth_read_cfg* cfg) {
    Genome* g = (Genome*)refp;
    auto* rs = new ReadSet();
    rs->cfg = *cfg;
    Rng rng(splitmix(cfg->seed ^ 0x2222));
    double mu = cfg->len_mean, sd = cfg->len_sd;
    double s2 = sd > 0 ? std::log(1.0 + sd * sd / (mu * mu)) : 0.0;
    double m = std::log(mu) - s2 / 2;
    for (int32_t i = 0; i < cfg->n_reads; i++) {
        int64_t L = sd > 0 ? (int64_t)std::llround(std::exp(m + std::sqrt(s2) * rng.normal())) : (int64_t)mu;
        L = std::max(cfg->len_min, std::min(cfg->len_max, L));
        ReadPlan rp{};
        bool placed = false;
        if (cfg->satellite_read_frac > 0 && !g->sat_arrays.empty() && rng.uni() < cfg->satellite_read_frac) {
            auto sa = g->sat_arrays[(size_t)rng.below(g->sat_arrays.size())];
            const Feature& f = g->features[(size_t)sa.first][sa.second];
            int64_t lo = f.start, hi = f.start + f.len;
            rp.contig = sa.first;
            int64_t clen = g->contig_len[(size_t)sa.first];
            L = std::min(L, clen);
            int64_t s0 = std::max<int64_t>(0, std::min(lo + (int64_t)rng.below((uint64_t)std::max<int64_t>(1, hi - lo)), clen - L));
            rp.start = s0;
            placed = true;
        }
        if (!placed) {
            for (int tries = 0; tries < 1000; tries++) {
                uint64_t x = rng.below((uint64_t)g->total);
                int32_t ci = (int32_t)(std::upper_bound(g->contig_off.begin(), g->contig_off.end(), (int64_t)x) -
                                       g->contig_off.begin() - 1);
                int64_t clen = g->contig_len[(size_t)ci];
                if (clen < L) continue;
                rp.contig = ci;
                rp.start = (int64_t)rng.below((uint64_t)(clen - L + 1));
                placed = true;
                break;
            }
            if (!placed) {
                rp.contig = 0;
                L = std::min(L, g->contig_len[0]);
                rp.start = 0;
            }
        }
        rp.len = L;
        rp.rev = rng.uni() < 0.5;
        rp.key = rng.next();
        rs->plan.push_back(rp);
    }
    rs->out_len.assign(rs->plan.size(), -1);
    return rs;
}
void synth_reads_free(void* p) { delete (ReadSet*)p; }

static char comp(char b) {
    switch (b) {
        case 'A': return 'T';
        case 'C': return 'G';
        case 'G': return 'C';
        case 'T': return 'A';
        default: return 'N';
    }
}

// Builds read i (reference span with errors, reverse-complemented if on '-').
static void build_read(const Genome& g, const ReadSet& rs, size_t i, const uint8_t* ref, std::string& out) {
    const ReadPlan& rp = rs.plan[i];
    const synth_read_cfg& c = rs.cfg;
    const uint8_t* src = ref + g.contig_off[(size_t)rp.contig] + rp.start;
    std::string span((const char*)src, (size_t)rp.len);
    if (rp.rev) {
        std::reverse(span.begin(), span.end());
        for (auto& ch : span) ch = comp(ch);
    }
    out.clear();
    out.reserve(span.size() + span.size() / 16 + 16);
    Rng rng(rp.key);
    double tw = c.sub_w + c.ins_w + c.del_w;
    double ps = tw > 0 ? c.sub_w / tw : 0, pi = tw > 0 ? c.ins_w / tw : 0;
    for (size_t j = 0; j < span.size(); j++) {
        if (c.err_rate > 0 && rng.uni() < c.err_rate) {
            double u = rng.uni();
            if (u < ps) {
                char b = span[j];
                int bi = (int)(std::find(BASES, BASES + 4, b) - BASES);
                out.push_back(BASES[(bi + 1 + (int)rng.below(3)) & 3]);
            } else if (u < ps + pi) {
                out.push_back(BASES[rng.below(4)]);
                out.push_back(span[j]);
            }  // else deletion: drop span[j]
        } else {
            out.push_back(span[j]);
        }
    }
}

// Total bases of all reads (runs the error model once; cached per read).
int64_t synth_reads_total(void* refp, void* rsp, const uint8_t* ref, int32_t threads) {
    Genome* g = (Genome*)refp;
    ReadSet* rs = (ReadSet*)rsp;
    std::atomic<size_t> next{0};
    auto work = [&]() {
        std::string s;
        for (size_t i; (i = next.fetch_add(1)) < rs->plan.size();) {
            build_read(*g, *rs, i, ref, s);
            rs->out_len[i] = (int64_t)s.size();
        }
    };
    std::vector<std::thread> ts;
    for (int t = 0; t < std::max(1, threads); t++) ts.emplace_back(work);
    for (auto& t : ts) t.join();
    int64_t tot = 0;
    for (int64_t l : rs->out_len) tot += l;
    return tot;
}

// Fills the concatenated read bases and offsets (n_reads+1). Call synth_reads_total first.
void synth_reads_fill(void* refp, void* rsp, const uint8_t* ref, uint8_t* out, int64_t* offs, int32_t threads) {
    Genome* g = (Genome*)refp;
    ReadSet* rs = (ReadSet*)rsp;
    int64_t acc = 0;
    for (size_t i = 0; i < rs->plan.size(); i++) {
        offs[i] = acc;
        acc += rs->out_len[i];
    }
    offs[rs->plan.size()] = acc;
    std::atomic<size_t> next{0};
    auto work = [&]() {
        std::string s;
        for (size_t i; (i = next.fetch_add(1)) < rs->plan.size();) {
            build_read(*g, *rs, i, ref, s);
            std::memcpy(out + offs[i], s.data(), s.size());
        }
    };
    std::vector<std::thread> ts;
    for (int t = 0; t < std::max(1, threads); t++) ts.emplace_back(work);
    for (auto& t : ts) t.join();
}

// Header of read i: S<i>_1!<chr>!<start>!<end>!<strand> (written NUL-terminated).
void synth_read_name(void* refp, void* rsp, int32_t i, char* buf, int32_t cap) {
    Genome* g = (Genome*)refp;
    ReadSet* rs = (ReadSet*)rsp;
    const ReadPlan& rp = rs->plan[(size_t)i];
    std::snprintf(buf, (size_t)cap, "S%d_1!%s!%lld!%lld!%c", i + 1, g->names[(size_t)rp.contig].c_str(),
                  (long long)rp.start, (long long)(rp.start + rp.len), rp.rev ? '-' : '+');
}

}  // extern "C"
