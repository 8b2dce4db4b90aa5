// Launch and batch shapes that are chosen by measurement rather than fixed in
// the code: the project's autotuner (shmap_b200/autotune.py) sweeps them on a
// workload and writes tuning.conf, which the library reads once per process
// (from $SHMAP_TUNING, else tuning.conf in the directory above the library's
// own). None of them changes a result, only how the work is cut and spread.
#include <dlfcn.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/shmap_gpu.h"
#include "shm_internal.hpp"
#include "shm_tune.hpp"

namespace shm {

namespace {

struct Knob {
    const char* name;
    int64_t Tuning::*field;
    int64_t lo, hi;
};

const Knob KNOBS[] = {
    {"dev_batch_reads", &Tuning::dev_batch_reads, 1024, 1 << 22},
    {"dev_batch_bases", &Tuning::dev_batch_bases, 1 << 20, (int64_t)1 << 34},
    {"dev_first_batch_reads", &Tuning::dev_first_batch_reads, 64, 1 << 22},
    {"host_batch_reads", &Tuning::host_batch_reads, 1024, 1 << 22},
    {"host_batch_bases", &Tuning::host_batch_bases, 1 << 20, (int64_t)1 << 32},
    {"host_first_batch_reads", &Tuning::host_first_batch_reads, 64, 1 << 22},
    {"sketch_ctas_per_sm", &Tuning::sketch_ctas_per_sm, 1, 8},
    {"wide_ctas_per_sm", &Tuning::wide_ctas_per_sm, 1, 8},
    {"refine_warps_per_sm", &Tuning::refine_warps_per_sm, 8, 64},
    {"device_pack", &Tuning::device_pack, 0, 1},
    {"host_raw_share", &Tuning::host_raw_share, 0, 100},
    {"bt_fast_slots", &Tuning::bt_fast_slots, 16, 512},
    {"host_pack_task_kib", &Tuning::host_pack_task_kib, 0, 1 << 20},
    {"host_stream", &Tuning::host_stream, 0, 2},
    {"host_stream_piece_kib", &Tuning::host_stream_piece_kib, 64, 1 << 16},
    {"host_stream_ring", &Tuning::host_stream_ring, 2, 16},
    {"host_stream_raw_share", &Tuning::host_stream_raw_share, 0, 100},
    {"plan_mapped", &Tuning::plan_mapped, 0, 1},
    {"host_stream_bases", &Tuning::host_stream_bases, 1 << 24, (int64_t)1 << 36},
    {"host_stream_chunk_kib", &Tuning::host_stream_chunk_kib, 256, 1 << 20},
    {"host_stream_first_kib", &Tuning::host_stream_first_kib, 256, 1 << 22},
    {"host_stream_last_kib", &Tuning::host_stream_last_kib, 256, 1 << 22},
};

std::mutex g_mu;
Tuning g_t;
bool g_loaded = false;
std::string g_source = "built-in defaults";

const Knob* find(const char* key) {
    for (const Knob& k : KNOBS)
        if (key && std::strcmp(k.name, key) == 0) return &k;
    return nullptr;
}

// key = value lines, '#' comments; returns an error message or "".
std::string load_file(const char* path, Tuning& t) {
    std::FILE* f = std::fopen(path, "r");
    if (!f) return std::string("cannot open ") + path;
    char line[512];
    int no = 0;
    std::string err;
    while (err.empty() && std::fgets(line, sizeof line, f)) {
        no++;
        char* h = std::strchr(line, '#');
        if (h) *h = 0;
        char key[128];
        long long v;
        char extra;
        if (std::sscanf(line, " %127[a-z_0-9] = %lld %c", key, &v, &extra) == 2) {
            const Knob* k = find(key);
            if (!k) err = std::string(path) + ":" + std::to_string(no) + ": unknown setting " + key;
            else if (v < k->lo || v > k->hi)
                err = std::string(path) + ":" + std::to_string(no) + ": " + key + " out of range";
            else t.*(k->field) = v;
        } else {
            for (char* c = line; *c; c++)
                if (*c != ' ' && *c != '\t' && *c != '\n' && *c != '\r') {
                    err = std::string(path) + ":" + std::to_string(no) + ": not a 'key = value' line";
                    break;
                }
        }
    }
    std::fclose(f);
    return err;
}

std::string default_path() {
    if (const char* e = std::getenv("SHMAP_TUNING")) return e;
    Dl_info info;
    if (dladdr((void*)&default_path, &info) && info.dli_fname) {
        std::string p = info.dli_fname;
        const size_t s1 = p.rfind('/');
        if (s1 != std::string::npos) {
            const size_t s2 = p.rfind('/', s1 ? s1 - 1 : 0);
            if (s2 != std::string::npos) return p.substr(0, s2) + "/tuning.conf";
        }
    }
    return "tuning.conf";
}

void ensure_loaded() {
    if (g_loaded) return;
    g_loaded = true;
    const std::string p = default_path();
    std::FILE* f = std::fopen(p.c_str(), "r");
    if (!f) return;  // no file: the built-in defaults
    std::fclose(f);
    Tuning t;
    const std::string err = load_file(p.c_str(), t);
    if (err.empty()) {
        g_t = t;
        g_source = p;
    } else {
        std::fprintf(stderr, "shmap-b200: ignoring %s\n", err.c_str());
    }
}

}  // namespace

Tuning tuning() {
    std::lock_guard<std::mutex> g(g_mu);
    ensure_loaded();
    return g_t;
}

}  // namespace shm

extern "C" int shm_tuning_get(const char* key, int64_t* value) {
    const shm::Knob* k = shm::find(key);
    if (!k || !value) {
        shm::set_last_error(std::string("unknown tuning setting ") + (key ? key : "(null)"));
        return SHM_ERR_INVALID;
    }
    std::lock_guard<std::mutex> g(shm::g_mu);
    shm::ensure_loaded();
    *value = shm::g_t.*(k->field);
    return SHM_OK;
}

extern "C" int shm_tuning_set(const char* key, int64_t value) {
    const shm::Knob* k = shm::find(key);
    if (!k) {
        shm::set_last_error(std::string("unknown tuning setting ") + (key ? key : "(null)"));
        return SHM_ERR_INVALID;
    }
    if (value < k->lo || value > k->hi) {
        shm::set_last_error(std::string(k->name) + " must be between " + std::to_string(k->lo) + " and " +
                            std::to_string(k->hi));
        return SHM_ERR_INVALID;
    }
    std::lock_guard<std::mutex> g(shm::g_mu);
    shm::ensure_loaded();
    shm::g_t.*(k->field) = value;
    return SHM_OK;
}

extern "C" int shm_tuning_load(const char* path) {
    std::lock_guard<std::mutex> g(shm::g_mu);
    shm::g_loaded = true;
    shm::Tuning t;
    const std::string p = path ? std::string(path) : shm::default_path();
    const std::string err = shm::load_file(p.c_str(), t);
    if (!err.empty()) {
        shm::set_last_error(err);
        return SHM_ERR_INVALID;
    }
    shm::g_t = t;
    shm::g_source = p;
    return SHM_OK;
}

extern "C" const char* shm_tuning_source(void) {
    std::lock_guard<std::mutex> g(shm::g_mu);
    shm::ensure_loaded();
    return shm::g_source.c_str();
}
