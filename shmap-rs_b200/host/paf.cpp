// PAF text of a mapped read, byte for byte as the reference prints it
// (MappingPaf / LocalMappingStats / GlobalMappingStats Display impls,
// src/mapping.rs:87-107, 161-182, 228-247), from a device record. The
// record carries the raw best/second-best results; the mapq, J2 and sigma
// post-processing of set_second_best/set_global_stats/calc_mapq
// (src/mapping.rs:329-408) happens here, on the host, in plain IEEE f64.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/shmap_gpu.h"
#include "../csrc/shm_internal.hpp"

namespace {

// Rust `{:.N}` on f64: the exactly rounded fixed form; NaN prints as "NaN".
void put_f(std::string& o, double x, int prec) {
    if (std::isnan(x)) {
        o += "NaN";
        return;
    }
    if (std::isinf(x)) {
        o += x > 0 ? "inf" : "-inf";
        return;
    }
    char b[400];
    std::snprintf(b, sizeof b, "%.*f", prec, x);
    o += b;
}
void put_i(std::string& o, long long v) {
    char b[32];
    std::snprintf(b, sizeof b, "%lld", v);
    o += b;
}

void render(std::string& o, const shm::IndexStorage& ix, const shm_params& p, const shm_map_record& r,
            const std::string& qid, double map_time) {
    // set_second_best (mapping.rs:356-361) runs only when a second best exists
    double j2 = -1.0, sigmas = -1.0;
    int32_t i2 = -1, b2s = -1, b2b = -1;
    if (r.has_second) {
        j2 = r.score2;
        i2 = r.intersection2;
        b2s = r.bucket2_seg;
        b2b = r.bucket2_b;
        double x = (double)(i2 == -1 ? 0 : i2), y = (double)(r.intersection == -1 ? 0 : r.intersection);
        sigmas = std::fabs(x - y) / std::sqrt(x + y);  // mapping.rs:329-333
    }
    // calc_mapq (mapping.rs:341-354), which also lifts J2 to theta2
    const double theta2 = p.theta - p.min_diff;
    if (j2 < theta2) j2 = theta2;
    const double frac = 1.0 - j2 / r.score;
    const int32_t mapq_strand = std::abs(r.same_strand) < r.intersection / 2 ? 5 : 60;
    const int mapq = frac > p.min_diff ? (mapq_strand < 60 ? mapq_strand : 60) : 0;
    const std::string& sname = ix.names[(size_t)r.segm_id];
    const int32_t ssz = ix.seg_len[(size_t)r.segm_id];

    o += qid;
    o += '\t';
    put_i(o, r.read_len);
    o += '\t';
    put_i(o, r.p_start);
    o += '\t';
    put_i(o, r.p_end);
    o += '\t';
    o += r.same_strand > 0 ? '+' : '-';
    o += '\t';
    o += sname;
    o += '\t';
    put_i(o, ssz);
    o += '\t';
    put_i(o, r.t_l);
    o += '\t';
    put_i(o, r.t_r);
    o += '\t';
    put_i(o, r.read_len);
    o += '\t';
    put_i(o, r.read_len);
    o += '\t';
    put_i(o, mapq);
    o += "\tp:i:";
    put_i(o, r.sketch_size);
    o += "\ts:i:";
    put_i(o, r.s_sz);
    o += "\tI:i:";
    put_i(o, r.intersection);
    o += "\tI2:i:";
    put_i(o, i2);
    o += "\tIdiff:i:";
    put_i(o, (int32_t)(r.intersection - i2));
    o += "\tIsdiff:f:";
    put_f(o, sigmas, 5);
    o += "\tJ:f:";
    put_f(o, r.score, 5);
    o += "\tJ2:f:";
    put_f(o, j2, 5);
    o += "\tJdiff:f:";
    put_f(o, r.score - j2, 5);
    o += "\tsh:f:";
    put_f(o, r.sh, 5);
    o += "\tstrand:i:";
    put_i(o, r.same_strand);
    o += "\tt:f:";
    put_f(o, map_time, 5);
    o += "\tb:s:(";
    put_i(o, r.bucket_seg);
    o += ',';
    put_i(o, r.bucket_b);
    o += ")\tb2:s:(";
    put_i(o, b2s);
    o += ',';
    put_i(o, b2b);
    o += ")\tk:i:";
    put_i(o, p.k);
    o += "\tgt_J:f:-1.000\tgt_C:f:-1.000\tgt_C_bucket:f:-1.000\tseeds:i:";
    put_i(o, r.seeds);
    o += "\tmax_seed_matches:i:";
    put_i(o, r.max_seed_matches);
    o += "\tseed_matches:i:";
    put_i(o, r.seed_matches);
    o += "\ttotal_matches:i:";
    put_i(o, r.total_matches);
    o += "\tmatch_inefficiency:f:";
    put_f(o, (double)r.total_matches / (double)r.intersection, 3);
    o += "\tseeded_buckets:i:";
    put_i(o, r.seeded_buckets);
    o += "\tfinal_buckets:i:";
    put_i(o, r.final_buckets);
    o += "\tFPTP:f:-1.000\n";
}

}  // namespace

extern "C" int shm_format_paf(const shm_index* idx, const shm_params* p, const shm_map_record* rec, int32_t n,
                              const char* names, const double* map_time, char* buf, int64_t cap, int64_t* n_out) {
    if (!idx || !p || !n_out || (n > 0 && !rec)) return SHM_ERR_INVALID;
    std::string o;
    const char* s = names ? names : "";
    for (int32_t i = 0; i < n; i++) {
        const char* e = std::strchr(s, '\n');
        if (!e) e = s + std::strlen(s);
        std::string qid(s, (size_t)(e - s));
        s = *e ? e + 1 : e;
        if (rec[i].status != 0) continue;
        render(o, *idx->s, *p, rec[i], qid, map_time ? map_time[i] : 0.0);
    }
    *n_out = (int64_t)o.size();
    if (buf && cap > 0) std::memcpy(buf, o.data(), (size_t)std::min<int64_t>(cap, (int64_t)o.size()));
    return (int64_t)o.size() > cap && buf ? SHM_ERR_CAPACITY : SHM_OK;
}
