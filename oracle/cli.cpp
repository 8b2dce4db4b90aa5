// TEST INFRASTRUCTURE ONLY: `shmap_oracle`, the oracle behind the reference's
// command line (src/main.rs:16-70, src/params.rs:20-263). Used by the tests to
// check the oracle against the reference's golden PAF and CLI tests.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "oracle.hpp"

using namespace oracle;

static void die(const std::string& m) {
    std::fprintf(stderr, "ERROR: %s\n", m.c_str());
    std::exit(1);
}

int main(int argc, char** argv) {
    Params p;
    std::string t_file, p_file, z_file;
    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        auto val = [&]() -> std::string {
            if (i + 1 >= argc) die("missing value for " + a);
            return argv[++i];
        };
        if (a == "-s" || a == "--text") t_file = val();
        else if (a == "-p" || a == "--pattern") p_file = val();
        else if (a == "-k" || a == "--ksize") p.k = std::atoi(val().c_str());
        else if (a == "-r" || a == "--hashratio") p.h_frac = std::atof(val().c_str());
        else if (a == "-t" || a == "--threshold") p.theta = std::atof(val().c_str());
        else if (a == "-d" || a == "--min_diff") p.min_diff = std::atof(val().c_str());
        else if (a == "-o" || a == "--max_overlap") p.max_overlap = std::atof(val().c_str());
        else if (a == "-M" || a == "--max_matches") p.max_matches = std::atoi(val().c_str());
        else if (a == "-@" || a == "--threads") p.threads = std::atoi(val().c_str());
        else if (a == "-z" || a == "--params") z_file = val();
        else if (a == "-P" || a == "--no_bucket_pruning") p.no_bucket_pruning = true;
        else if (a == "-B" || a == "--one_sweep") p.one_sweep = true;
        else if (a == "-F" || a == "--abs_pos") p.abs_pos = true;
        else if (a == "--rarity-weight") p.rarity_weight = std::atof(val().c_str());
        else if (a == "--rarity-tiebreak") p.rarity_tiebreak = std::atof(val().c_str());
        else if (a == "--rarity-alpha") p.rarity_alpha = std::atof(val().c_str());
        else if (a == "-m" || a == "--metric") {
            std::string m = val();
            if (m == "Containment") p.metric = Metric::Containment;
            else if (m == "Jaccard") p.metric = Metric::Jaccard;
            else if (m == "bucket_SH") p.metric = Metric::BucketSh;
            else if (m == "bucket_LCS") p.metric = Metric::BucketLcs;
            else die("invalid metric " + m);
        } else die("unknown argument " + a);
    }
    // src/params.rs:191-263
    if (p.k <= 0) die("K-mer length (-k) should be positive. You provided " + std::to_string(p.k) + ".");
    if (p.h_frac <= 0.0 || p.h_frac > 1.0) die("Given hash ratio (-r) should be between 0 and 1.");
    if (p.max_matches != -1 && p.max_matches <= 0) die("The number of seed matches (-M) should be positive.");
    if (p.theta < 0.0 || p.theta > 1.0) die("The threshold (-t) should be between 0 and 1.");
    if (p.min_diff < 0.0) die("The minimum difference (-d) should be >= 0.");
    if (p.rarity_weight < 0.0 || p.rarity_weight > 4.0)
        die("The rarity weight (--rarity-weight) should be between 0 and 4.");
    if (p.rarity_weight > 0.0 && p.metric != Metric::Containment)
        die("--rarity-weight is only defined for -m Containment.");
    if (p.max_overlap < 0.0 || p.max_overlap > 1.0) die("The maximum overlap (-o) should be between 0 and 1.");
    if (p.threads <= 0) die("The number of threads (-@) should be positive.");
    if (t_file.empty() || p_file.empty()) die("both -s and -p are required");

    std::vector<FastaRecord> ref, reads;
    std::string err;
    if (!read_fasta(t_file, ref, &err)) die(err);
    if (!read_fasta(p_file, reads, &err)) die(err);
    FracMinHash sk(p.k, p.h_frac);
    SketchIndex idx;
    std::vector<std::string> names;
    std::vector<const uint8_t*> seqs;
    std::vector<size_t> lens;
    for (auto& r : ref) {
        names.push_back(r.name);
        seqs.push_back((const uint8_t*)r.seq.data());
        lens.push_back(r.seq.size());
    }
    idx.build_index(names, seqs, lens, sk, p.max_matches, p.threads);
    std::vector<const uint8_t*> rs;
    std::vector<size_t> rl;
    for (auto& r : reads) {
        rs.push_back((const uint8_t*)r.seq.data());
        rl.push_back(r.seq.size());
    }
    auto t0 = std::chrono::steady_clock::now();
    auto res = map_reads(idx, sk, p, rs, rl, p.threads);
    double per_read = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() /
                      (reads.empty() ? 1.0 : (double)reads.size());
    FILE* unm = nullptr;
    if (!z_file.empty()) unm = std::fopen((z_file + ".unmapped.paf").c_str(), "w");
    std::string out;
    for (size_t i = 0; i < reads.size(); i++) {
        if (res[i].mapped) out += render_paf(res[i], reads[i].name, p, per_read) + "\n";
        else if (unm) std::fprintf(unm, "%s\n", unmapped_line(reads[i].name, (QPos)reads[i].seq.size()).c_str());
    }
    std::fwrite(out.data(), 1, out.size(), stdout);
    if (unm) std::fclose(unm);
    return 0;
}
