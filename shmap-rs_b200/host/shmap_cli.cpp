// `shmap`: the reference's command line (src/main.rs:16-70, src/params.rs:20-263)
// over the B200 path. Reads the reference and the reads (FASTA/FASTQ, as the
// reference's needletail reader does: id cut at the first space or tab, line
// ends and '\r' removed), builds the index on the device, maps the reads in
// batches and writes PAF to stdout in input order; with -z, unmapped reads go
// to <z>.unmapped.paf (src/shmap/mod.rs:388-394, src/mapping.rs:82-84).
// Options the reference does not have: --index-out FILE writes the built
// index to FILE; --index-in FILE takes the index from FILE instead of -s, and
// its k, -r and -M replace those given on the command line; --host-fasta
// parses FASTA on the host (by default the device parses it and keeps the
// sequences; FASTQ is always read on the host).
#include "utf8.hpp"
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "../../include/shmap_gpu.h"

namespace {

struct Records {
    std::vector<std::string> names;
    std::string seq;              // all sequences back to back
    std::vector<int64_t> off{0};  // n+1
};

[[noreturn]] void die(const std::string& m) {
    std::fprintf(stderr, "ERROR: %s\n", m.c_str());
    std::exit(1);
}

bool read_file(const std::string& path, std::string& data, std::string& err) {
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        err = "failed to open " + path;
        return false;
    }
    data.assign((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    return true;
}

bool parse_fastx(const std::string& data, const std::string& path, Records& out, std::string& err) {
    size_t pos = 0, n = data.size();
    auto line = [&](size_t& a, size_t& b) {  // next line [a, b) without '\n' / trailing '\r'
        a = pos;
        size_t e = data.find('\n', pos);
        if (e == std::string::npos) e = n;
        b = e;
        if (b > a && data[b - 1] == '\r') b--;
        pos = e + 1;
    };
    auto add_name = [&](size_t a, size_t b) {
        std::string h = data.substr(a, b - a);
        size_t cut = h.find_first_of(" \t");
        out.names.push_back(shm::utf8_lossy(cut == std::string::npos ? h : h.substr(0, cut)));
    };
    bool open = false;
    while (pos < n) {
        size_t a, b;
        line(a, b);
        if (b > a && data[a] == '>') {
            if (open) out.off.push_back((int64_t)out.seq.size());
            add_name(a + 1, b);
            open = true;
        } else if (b > a && data[a] == '@' && (!open || out.off.size() == out.names.size())) {
            // FASTQ record: header, sequence, '+', quality
            if (open) out.off.push_back((int64_t)out.seq.size());
            add_name(a + 1, b);
            size_t sa, sb, pa, pb, qa, qb;
            line(sa, sb);
            out.seq.append(data, sa, sb - sa);
            line(pa, pb);
            line(qa, qb);
            out.off.push_back((int64_t)out.seq.size());
            open = false;
        } else if (open) {
            out.seq.append(data, a, b - a);
        } else if (b > a) {
            err = "invalid FASTA record in " + path;
            return false;
        }
    }
    if (open) out.off.push_back((int64_t)out.seq.size());
    return true;
}

std::string join(const std::vector<std::string>& v, size_t a, size_t b) {
    std::string s;
    for (size_t i = a; i < b; i++) {
        if (i > a) s += '\n';
        s += v[i];
    }
    return s;
}

}  // namespace

int main(int argc, char** argv) {
    shm_params p;
    shm_params_default(&p);
    std::string t_file, p_file, z_file, ix_in, ix_out;
    int threads = 1, verbose = 0, device = 0;
    bool host_fasta = false;
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
        else if (a == "-S" || a == "--max_seeds") (void)val();  // accepted and inert (params.rs:37-45)
        else if (a == "-@" || a == "--threads") threads = std::atoi(val().c_str());
        else if (a == "-z" || a == "--params") z_file = val();
        else if (a == "-v" || a == "--verbose") verbose = std::atoi(val().c_str());
        else if (a == "-n" || a == "--normalize") {
        } else if (a == "-P" || a == "--no_bucket_pruning") p.no_bucket_pruning = 1;
        else if (a == "-B" || a == "--one_sweep") p.one_sweep = 1;
        else if (a == "-F" || a == "--abs_pos") p.abs_pos = 1;
        else if (a == "--rarity-weight") p.rarity_weight = std::atof(val().c_str());
        else if (a == "--rarity-tiebreak") p.rarity_tiebreak = std::atof(val().c_str());
        else if (a == "--rarity-alpha") p.rarity_alpha = std::atof(val().c_str());
        else if (a == "--device") device = std::atoi(val().c_str());
        // index files (not flags of the reference): write the built index, or
        // start from one instead of -s (its k, -r and -M then apply)
        else if (a == "--index-out") ix_out = val();
        else if (a == "--index-in") ix_in = val();
        else if (a == "--host-fasta") host_fasta = true;  // parse FASTA on the host (same records)
        else if (a == "-m" || a == "--metric") {
            std::string m = val();
            if (m == "Containment") p.metric = SHM_CONTAINMENT;
            else if (m == "Jaccard") p.metric = SHM_JACCARD;
            else if (m == "bucket_SH") p.metric = SHM_BUCKET_SH;
            else if (m == "bucket_LCS") p.metric = SHM_BUCKET_LCS;
            else die("invalid value '" + m + "' for '--metric <METRIC>'");
        } else die("unexpected argument '" + a + "'");
    }
    if ((t_file.empty() && ix_in.empty()) || p_file.empty()) {
        std::string miss = p_file.empty() ? "--pattern" : "";
        if (t_file.empty() && ix_in.empty()) miss += std::string(miss.empty() ? "" : ", ") + "--text";
        die("the following required arguments were not provided: " + miss);
    }
    if (shm_params_validate(&p) != SHM_OK) die(shm_last_error());
    if (threads <= 0) die("The number of threads (-@) should be positive. You provided " + std::to_string(threads) + ".");
    if (verbose < 0 || verbose > 2) die("--verbose (-v) should be 0, 1, or 2.");

    Records ref, reads;
    std::string err, t_data, p_data;
    if (ix_in.empty() && !read_file(t_file, t_data, err)) die(err);
    if (!read_file(p_file, p_data, err)) die(err);
    shm_ctx* ctx = nullptr;
    if (shm_ctx_create(device, 0, &ctx) != SHM_OK) die(std::string("CUDA: ") + shm_last_error());
    // FASTA is parsed on the device, its sequences left there; FASTQ (and
    // files the host reader rejects) go through the host reader
    auto parse = [&](const std::string& data, const std::string& path, Records& rec) -> shm_fasta* {
        shm_fasta* fa = nullptr;
        if (!host_fasta && shm_fasta_parse_device(ctx, (const uint8_t*)data.data(), (int64_t)data.size(), &fa) ==
                               SHM_OK) {
            int32_t nr = 0;
            const int64_t* offs = nullptr;
            const char* names = nullptr;
            shm_fasta_records(fa, &nr, &offs, &names);
            rec.off.assign(offs, offs + nr + 1);
            const char* q = names;
            for (int32_t i = 0; i < nr; i++) {
                const char* e = std::strchr(q, '\n');
                if (!e) e = q + std::strlen(q);
                rec.names.emplace_back(q, (size_t)(e - q));
                q = *e ? e + 1 : e;
            }
            return fa;
        }
        if (!parse_fastx(data, path, rec, err)) die(err);
        return nullptr;
    };
    shm_index* idx = nullptr;
    if (!ix_in.empty()) {
        if (shm_index_load(ctx, ix_in.c_str(), &idx) != SHM_OK)
            die(std::string("failed to load index from ") + ix_in + ": " + shm_last_error());
        shm_index_info(idx, &p.k, &p.h_frac, &p.max_matches);
    } else {
        shm_fasta* tfa = parse(t_data, t_file, ref);
        std::string().swap(t_data);
        int rc;
        if (tfa) {
            rc = shm_index_build_fasta(ctx, tfa, p.k, p.h_frac, p.max_matches, &idx);
        } else {
            std::string rnames = join(ref.names, 0, ref.names.size());
            rc = shm_index_build(ctx, (const uint8_t*)ref.seq.data(), ref.off.data(), (int32_t)ref.names.size(),
                                 rnames.c_str(), p.k, p.h_frac, p.max_matches, &idx);
        }
        shm_fasta_destroy(tfa);
        if (rc != SHM_OK) die(std::string("failed to build index from ") + t_file + ": " + shm_last_error());
    }
    shm_fasta* pfa = parse(p_data, p_file, reads);
    std::string().swap(p_data);
    if (!ix_out.empty() && shm_index_save(idx, ix_out.c_str()) != SHM_OK)
        die(std::string("failed to write index to ") + ix_out + ": " + shm_last_error());

    FILE* unm = nullptr;
    if (!z_file.empty()) {
        unm = std::fopen((z_file + ".unmapped.paf").c_str(), "w");
        if (!unm) die("cannot create " + z_file + ".unmapped.paf");
    }
    const size_t n = reads.names.size();
    const size_t CH = 1 << 17;  // reads per call; output stays in input order
    std::vector<shm_map_record> rec;
    std::vector<double> tms;
    std::string buf;
    for (size_t a = 0; a < n; a += CH) {
        size_t b = std::min(n, a + CH);
        rec.resize(b - a);
        auto t0 = std::chrono::steady_clock::now();
        std::vector<int64_t> off(reads.off.begin() + (long)a, reads.off.begin() + (long)b + 1);
        const int rc = pfa ? shm_map_fasta(ctx, idx, &p, pfa, (int32_t)a, (int32_t)(b - a), rec.data())
                           : shm_map_batch(ctx, idx, &p, (const uint8_t*)reads.seq.data(), off.data(),
                                           (int32_t)(b - a), rec.data());
        if (rc != SHM_OK) die(std::string("failed while mapping reads from ") + p_file + ": " + shm_last_error());
        double per = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() / (double)(b - a);
        tms.assign(b - a, per);
        std::string names = join(reads.names, a, b);
        int64_t need = 0;
        // the PAF text is rendered on the device, byte for byte shm_format_paf's
        if (shm_format_paf_device(ctx, idx, &p, rec.data(), (int32_t)(b - a), names.c_str(), tms.data(), nullptr, 0,
                                  &need) != SHM_OK)
            die(std::string("failed to format PAF: ") + shm_last_error());
        buf.resize((size_t)need);
        if (need && shm_format_paf_device(ctx, idx, &p, rec.data(), (int32_t)(b - a), names.c_str(), tms.data(),
                                          buf.data(), need, &need) != SHM_OK)
            die(std::string("failed to format PAF: ") + shm_last_error());
        std::fwrite(buf.data(), 1, buf.size(), stdout);
        if (unm)
            for (size_t i = a; i < b; i++)
                if (rec[i - a].status != 0)
                    std::fprintf(unm, "%s\t%lld\t0\t0\t*\t*\t0\t0\t0\t0\t0\t0\n", reads.names[i].c_str(),
                                 (long long)(reads.off[i + 1] - reads.off[i]));
    }
    if (unm) std::fclose(unm);
    shm_fasta_destroy(pfa);
    shm_index_destroy(idx);
    shm_ctx_destroy(ctx);
    return 0;
}
