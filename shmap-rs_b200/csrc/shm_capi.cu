// The C ABI of include/shmap_gpu.h. Every entry point catches CUDA and host
// errors and turns them into status codes; nothing here falls back to the CPU.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/shmap_gpu.h"
#include "shm_common.cuh"
#include "shm_fasta.hpp"
#include "shm_internal.hpp"
#include "shm_map.cuh"
#include "shm_paf.hpp"
#include "shm_prims.cuh"
#include "shm_serve.hpp"
#include "shm_sketch.cuh"

struct shm_ctx {
    shm::MapCtx* m = nullptr;
};

static thread_local std::string g_err;

static int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

namespace shm {
void set_last_error(const std::string& m) { g_err = m; }
}  // namespace shm

#define SHM_GUARD_BEGIN try {
#define SHM_GUARD_END                                                                                   \
    }                                                                                                   \
    catch (const shm_cuda_error& e) {                                                                   \
        if (e.err == cudaErrorMemoryAllocation) return fail(SHM_ERR_NOMEM, cudaGetErrorString(e.err)); \
        return fail(SHM_ERR_CUDA, cudaGetErrorString(e.err));                                         \
    }                                                                                                   \
    catch (const std::bad_alloc&) {                                                                     \
        return fail(SHM_ERR_NOMEM, "host allocation failed");                                           \
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

extern "C" {

const char* shm_last_error(void) { return g_err.c_str(); }

void shm_params_default(shm_params* p) {
    p->k = 15;
    p->h_frac = 0.05;
    p->max_matches = -1;
    p->theta = 0.9;
    p->min_diff = 0.02;
    p->max_overlap = 0.5;
    p->metric = SHM_CONTAINMENT;
    p->no_bucket_pruning = 0;
    p->one_sweep = 0;
    p->abs_pos = 0;
    p->rarity_weight = 0.0;
    p->rarity_tiebreak = 0.0;
    p->rarity_alpha = 0.0;
}

static const char* metric_name(int32_t m) {  // Metric's Display (src/types.rs:312-321)
    switch (m) {
        case SHM_CONTAINMENT: return "Containment";
        case SHM_JACCARD: return "Jaccard";
        case SHM_BUCKET_SH: return "bucket_SH";
        default: return "bucket_LCS";
    }
}

static std::string fmt_g(double x) {  // Rust `{}` for an f64 that needs no exponent
    char b[64];
    std::snprintf(b, sizeof b, "%.17g", x);
    // shortest representation that round-trips
    for (int prec = 1; prec <= 17; prec++) {
        std::snprintf(b, sizeof b, "%.*g", prec, x);
        if (std::strtod(b, nullptr) == x) break;
    }
    return b;
}

int shm_params_validate(const shm_params* p) {
    if (!p) return fail(SHM_ERR_INVALID, "null params");
    if (p->k <= 0) return fail(SHM_ERR_INVALID, "K-mer length (-k) should be positive. You provided " + std::to_string(p->k) + ".");
    if (!(p->h_frac > 0.0) || p->h_frac > 1.0)
        return fail(SHM_ERR_INVALID, "Given hash ratio (-r) should be between 0 and 1. You provided " + fmt_g(p->h_frac) + ".");
    if (p->max_matches != -1 && p->max_matches <= 0)
        return fail(SHM_ERR_INVALID, "The number of seed matches (-M) should be positive. You provided " + std::to_string(p->max_matches) + ".");
    if (p->theta < 0.0 || p->theta > 1.0)
        return fail(SHM_ERR_INVALID, "The threshold (-t) should be between 0 and 1. You provided " + fmt_g(p->theta) + ".");
    if (p->min_diff < 0.0)
        return fail(SHM_ERR_INVALID, "The minimum difference (-d) should be >= 0. You provided " + fmt_g(p->min_diff) + ".");
    if (p->metric < SHM_CONTAINMENT || p->metric > SHM_BUCKET_LCS)
        return fail(SHM_ERR_INVALID, "unknown metric " + std::to_string(p->metric));
    if (p->rarity_weight < 0.0 || p->rarity_weight > 4.0)
        return fail(SHM_ERR_INVALID, "The rarity weight (--rarity-weight) should be between 0 and 4. You provided " +
                                         fmt_g(p->rarity_weight) + ".");
    if (p->rarity_weight > 0.0 && p->metric != SHM_CONTAINMENT)
        return fail(SHM_ERR_INVALID, std::string("--rarity-weight is only defined for -m Containment (got ") +
                                         metric_name(p->metric) +
                                         "). Jaccard's denominator includes reference k-mers absent from the read, "
                                         "which have no frequency to weight by.");
    if (p->max_overlap < 0.0 || p->max_overlap > 1.0)
        return fail(SHM_ERR_INVALID, "The maximum overlap (-o) should be between 0 and 1. You provided " + fmt_g(p->max_overlap) + ".");
    return SHM_OK;
}

uint64_t shm_h_thres(double h_frac) { return shm::h_thres(h_frac); }

int shm_ctx_create(int device, size_t hbm_budget, shm_ctx** out) {
    if (!out) return fail(SHM_ERR_INVALID, "null out");
    SHM_GUARD_BEGIN
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return fail(SHM_ERR_CUDA, "no CUDA device available");
    if (device < 0 || device >= n) return fail(SHM_ERR_INVALID, "device index out of range");
    auto* c = new shm_ctx();
    c->m = shm::mapctx_create(device, hbm_budget);
    *out = c;
    return SHM_OK;
    SHM_GUARD_END
}

int shm_ctx_destroy(shm_ctx* ctx) {
    if (!ctx) return SHM_OK;
    shm::mapctx_destroy(ctx->m);
    delete ctx;
    return SHM_OK;
}

int64_t shm_ctx_launches(const shm_ctx* ctx) {
    (void)ctx;
    return shm::kernel_launches();
}

void* shm_ctx_stream(const shm_ctx* ctx) { return ctx && ctx->m ? (void*)ctx->m->stream : nullptr; }

int shm_ctx_set_timing(shm_ctx* ctx, int on) {
    if (!ctx) return fail(SHM_ERR_INVALID, "null ctx");
    ctx->m->timing = on != 0;
    if (!on) {
        for (int i = 0; i < shm::N_STAGES; i++) {
            ctx->m->stage_ms[i] = 0;
            ctx->m->stage_calls[i] = 0;
        }
        for (int i = 0; i < shm::N_WORK; i++) ctx->m->work[i] = 0;
    }
    return SHM_OK;
}

int shm_ctx_stage_times(const shm_ctx* ctx, double* ms, int64_t* launches, int n) {
    if (!ctx) return fail(SHM_ERR_INVALID, "null ctx");
    for (int i = 0; i < shm::N_STAGES && i < n; i++) {
        if (ms) ms[i] = ctx->m->stage_ms[i];
        if (launches) launches[i] = ctx->m->stage_calls[i];
    }
    return shm::N_STAGES;
}

const char* shm_stage_name(int i) { return i >= 0 && i < shm::N_STAGES ? shm::STAGE_NAMES[i] : ""; }

int shm_ctx_work_stats(const shm_ctx* ctx, int64_t* out, int n) {
    if (!ctx) return fail(SHM_ERR_INVALID, "null ctx");
    for (int i = 0; i < shm::N_WORK && i < n; i++) out[i] = ctx->m->work[i];
    return shm::N_WORK;
}

const char* shm_work_stat_name(int i) { return i >= 0 && i < shm::N_WORK ? shm::WORK_NAMES[i] : ""; }

int shm_sketch(shm_ctx* ctx, const uint8_t* seq, int64_t len, int32_t k, double h_frac, int32_t offset, int32_t* r,
               uint64_t* h, uint8_t* strand, int64_t cap, int64_t* n_out) {
    if (!ctx || !n_out || (len > 0 && !seq)) return fail(SHM_ERR_INVALID, "null argument");
    if (k <= 0) return fail(SHM_ERR_INVALID, "K-mer length (-k) should be positive.");
    SHM_GUARD_BEGIN
    SHM_CUDA(cudaSetDevice(ctx->m->device));
    cudaStream_t s = ctx->m->stream;
    *n_out = 0;
    if (len < k) return SHM_OK;
    const int64_t nw = len - k + 1;
    const uint64_t n_chunks = (uint64_t)((nw + shm::SKETCH_WIN - 1) / shm::SKETCH_WIN);
    shm::DevBuf<uint8_t> d_seq;
    shm::DevBuf<int64_t> d_off;
    shm::DevBuf<uint64_t> d_coff, d_h;
    shm::DevBuf<uint32_t> d_cnt, d_out, d_rs;
    d_seq.reserve((size_t)len + 32);
    SHM_CUDA(cudaMemsetAsync(d_seq.p + len, 0, 32, s));
    SHM_CUDA(cudaMemcpyAsync(d_seq.p, seq, (size_t)len, cudaMemcpyHostToDevice, s));
    int64_t off[2] = {0, len};
    uint64_t coff[2] = {0, n_chunks};
    d_off.reserve(2);
    d_coff.reserve(2);
    SHM_CUDA(cudaMemcpyAsync(d_off.p, off, sizeof off, cudaMemcpyHostToDevice, s));
    SHM_CUDA(cudaMemcpyAsync(d_coff.p, coff, sizeof coff, cudaMemcpyHostToDevice, s));
    d_cnt.reserve(n_chunks + 1);
    d_out.reserve(n_chunks + 1);
    shm::SketchLuts* L = shm::create_device_luts(k, s);
    shm::SketchArgs a{};
    a.seq = d_seq.p;
    a.seq_off = d_off.p;
    a.chunk_off = d_coff.p;
    a.n_seq = 1;
    a.n_chunks = n_chunks;
    a.k = k;
    a.thr = shm::h_thres(h_frac);
    a.r_offset = offset;
    a.chunk_cnt = d_cnt.p;
    shm::launch_sketch(shm::SK_COUNT, a, L, s);
    shm::exclusive_scan_u32(d_cnt.p, d_out.p, n_chunks, s);
    uint32_t total = 0;
    SHM_CUDA(cudaMemcpyAsync(&total, d_out.p + n_chunks, sizeof total, cudaMemcpyDeviceToHost, s));
    SHM_CUDA(cudaStreamSynchronize(s));
    d_h.reserve((size_t)total + 1);
    d_rs.reserve((size_t)total + 1);
    a.chunk_out = d_out.p;
    a.out_h = d_h.p;
    a.out_rs = d_rs.p;
    shm::launch_sketch(shm::SK_WRITE, a, L, s);
    ctx->m->launches += 3;
    std::vector<uint64_t> hh(total);
    std::vector<uint32_t> rs(total);
    SHM_CUDA(cudaMemcpyAsync(hh.data(), d_h.p, sizeof(uint64_t) * total, cudaMemcpyDeviceToHost, s));
    SHM_CUDA(cudaMemcpyAsync(rs.data(), d_rs.p, sizeof(uint32_t) * total, cudaMemcpyDeviceToHost, s));
    SHM_CUDA(cudaStreamSynchronize(s));
    SHM_CUDA(cudaFree(L));
    *n_out = total;
    if ((int64_t)total > cap) return fail(SHM_ERR_CAPACITY, "output capacity too small");
    for (uint32_t i = 0; i < total; i++) {
        if (r) r[i] = (int32_t)(rs[i] >> 1);
        if (h) h[i] = hh[i];
        if (strand) strand[i] = (uint8_t)(rs[i] & 1u);
    }
    return SHM_OK;
    SHM_GUARD_END
}

static int check_index_args(const int64_t* seg_off, int32_t n_seg, int32_t k, double h_frac, int32_t max_matches);

int shm_index_build(shm_ctx* ctx, const uint8_t* seq, const int64_t* seg_off, int32_t n_seg, const char* names,
                    int32_t k, double h_frac, int32_t max_matches, shm_index** out) {
    if (!ctx || !out || !seg_off || n_seg < 0) return fail(SHM_ERR_INVALID, "null argument");
    const int v = check_index_args(seg_off, n_seg, k, h_frac, max_matches);
    if (v != SHM_OK) return v;
    SHM_GUARD_BEGIN
    SHM_CUDA(cudaSetDevice(ctx->m->device));
    auto* ix = new shm_index();
    ix->s = shm::build_index(seq, seg_off, n_seg, split_names(names, n_seg), k, h_frac, max_matches, ctx->m->stream);
    ctx->m->launches += 40;
    *out = ix;
    return SHM_OK;
    SHM_GUARD_END
}

static int check_index_args(const int64_t* seg_off, int32_t n_seg, int32_t k, double h_frac, int32_t max_matches) {
    if (k <= 0) return fail(SHM_ERR_INVALID, "K-mer length (-k) should be positive.");
    if (!(h_frac > 0.0) || h_frac > 1.0) return fail(SHM_ERR_INVALID, "Given hash ratio (-r) should be between 0 and 1.");
    if (max_matches != -1 && max_matches <= 0) return fail(SHM_ERR_INVALID, "The number of seed matches (-M) should be positive.");
    uint64_t windows = 0;
    for (int32_t i = 0; i < n_seg; i++) {
        int64_t L = seg_off[i + 1] - seg_off[i];
        if (L < 0 || L > INT32_MAX) return fail(SHM_ERR_INVALID, "segment length out of range (0 .. 2^31-1)");
        if (L >= k) windows += (uint64_t)(L - k + 1);
    }
    if (windows >= 0xfffffff0ULL) return fail(SHM_ERR_INVALID, "more than 2^32 reference windows");
    return SHM_OK;
}

struct shm_fasta {
    shm::FastaDev* f = nullptr;
};

int shm_fasta_parse_device(shm_ctx* ctx, const uint8_t* file, int64_t len, shm_fasta** out) {
    if (!ctx || !out || len < 0 || (len > 0 && !file)) return fail(SHM_ERR_INVALID, "null argument");
    *out = nullptr;
    SHM_GUARD_BEGIN
    std::string why;
    shm::FastaDev* f = shm::fasta_parse_device(ctx->m->device, ctx->m->stream, file, len, &why);
    if (!f) return fail(SHM_ERR_INVALID, "not parsed on the device: " + why);
    auto* h = new shm_fasta();
    h->f = f;
    *out = h;
    return SHM_OK;
    SHM_GUARD_END
}

int shm_fasta_records(const shm_fasta* fa, int32_t* n, const int64_t** offs, const char** names) {
    if (!fa) return fail(SHM_ERR_INVALID, "null argument");
    if (n) *n = fa->f->n;
    if (offs) *offs = fa->f->offs.data();
    if (names) *names = fa->f->names.c_str();
    return SHM_OK;
}

int shm_fasta_copy_seq(const shm_fasta* fa, uint8_t* dst) {
    if (!fa || !dst) return fail(SHM_ERR_INVALID, "null argument");
    SHM_GUARD_BEGIN
    SHM_CUDA(cudaSetDevice(fa->f->device));
    const int64_t total = fa->f->offs.back();
    if (total) SHM_CUDA(cudaMemcpy(dst, fa->f->seq.p, (size_t)total, cudaMemcpyDeviceToHost));
    return SHM_OK;
    SHM_GUARD_END
}

int shm_fasta_destroy(shm_fasta* fa) {
    if (!fa) return SHM_OK;
    cudaSetDevice(fa->f->device);
    delete fa->f;
    delete fa;
    return SHM_OK;
}

int shm_index_build_fasta(shm_ctx* ctx, const shm_fasta* fa, int32_t k, double h_frac, int32_t max_matches,
                          shm_index** out) {
    if (!ctx || !fa || !out) return fail(SHM_ERR_INVALID, "null argument");
    if (fa->f->device != ctx->m->device) return fail(SHM_ERR_INVALID, "the FASTA is on another device");
    const int v = check_index_args(fa->f->offs.data(), fa->f->n, k, h_frac, max_matches);
    if (v != SHM_OK) return v;
    SHM_GUARD_BEGIN
    SHM_CUDA(cudaSetDevice(ctx->m->device));
    auto* ix = new shm_index();
    ix->s = shm::build_index(nullptr, fa->f->offs.data(), fa->f->n, split_names(fa->f->names.c_str(), fa->f->n), k,
                             h_frac, max_matches, ctx->m->stream, fa->f->seq.p);
    ctx->m->launches += 40;
    *out = ix;
    return SHM_OK;
    SHM_GUARD_END
}

int shm_index_destroy(shm_index* idx) {
    if (!idx) return SHM_OK;
    if (idx->s) {
        cudaSetDevice(idx->s->device);
        delete idx->s;
    }
    delete idx;
    return SHM_OK;
}

int shm_index_save(const shm_index* idx, const char* path) {
    if (!idx || !path) return fail(SHM_ERR_INVALID, "null argument");
    SHM_GUARD_BEGIN
    SHM_CUDA(cudaSetDevice(idx->s->device));
    try {
        shm::save_index(idx->s, path);
    } catch (const shm::IndexFileError& e) {
        return fail(SHM_ERR_INVALID, e.what);
    }
    return SHM_OK;
    SHM_GUARD_END
}

int shm_index_load(shm_ctx* ctx, const char* path, shm_index** out) {
    if (!ctx || !path || !out) return fail(SHM_ERR_INVALID, "null argument");
    SHM_GUARD_BEGIN
    SHM_CUDA(cudaSetDevice(ctx->m->device));
    shm::IndexStorage* s = nullptr;
    try {
        s = shm::load_index(path, ctx->m->stream);
    } catch (const shm::IndexFileError& e) {
        return fail(SHM_ERR_INVALID, e.what);
    }
    ctx->m->launches += 8;
    auto* ix = new shm_index();
    ix->s = s;
    *out = ix;
    return SHM_OK;
    SHM_GUARD_END
}

int shm_index_file_check(const char* path) {
    if (!path) return fail(SHM_ERR_INVALID, "null argument");
    try {
        shm::check_index_file(path);
    } catch (const shm::IndexFileError& e) {
        return fail(SHM_ERR_INVALID, e.what);
    } catch (const std::exception& e) {
        return fail(SHM_ERR_INVALID, e.what());
    }
    return SHM_OK;
}

int shm_index_info(const shm_index* idx, int32_t* k, double* h_frac, int32_t* max_matches) {
    if (!idx) return fail(SHM_ERR_INVALID, "null argument");
    if (k) *k = idx->s->k;
    if (h_frac) *h_frac = idx->s->h_frac;
    if (max_matches) *max_matches = idx->s->max_matches;
    return SHM_OK;
}

int shm_index_stats_get(const shm_index* idx, shm_index_stats* out) {
    if (!idx || !out) return fail(SHM_ERR_INVALID, "null argument");
    *out = idx->s->stats;
    return SHM_OK;
}

__global__ void k_count(shm::DevIndex I, const uint64_t* h, int64_t n, int32_t* out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t a, c;
        shm::idx_lookup(I, h[i], a, c);
        out[i] = (int32_t)c;
    }
}

__global__ void k_one_list(shm::DevIndex I, uint64_t h, uint32_t* ac) {
    uint32_t a, c;
    shm::idx_lookup(I, h, a, c);
    ac[0] = a;
    ac[1] = c;
}

int shm_index_count(shm_ctx* ctx, const shm_index* idx, const uint64_t* h, int64_t n, int32_t* out) {
    if (!ctx || !idx || (n > 0 && (!h || !out))) return fail(SHM_ERR_INVALID, "null argument");
    SHM_GUARD_BEGIN
    SHM_CUDA(cudaSetDevice(ctx->m->device));
    if (n == 0) return SHM_OK;
    cudaStream_t s = ctx->m->stream;
    shm::DevBuf<uint64_t> dh;
    shm::DevBuf<int32_t> dout;
    dh.reserve((size_t)n);
    dout.reserve((size_t)n);
    SHM_CUDA(cudaMemcpyAsync(dh.p, h, sizeof(uint64_t) * (size_t)n, cudaMemcpyHostToDevice, s));
    k_count<<<shm::grid_for((size_t)n, 256), 256, 0, s>>>(idx->s->dev, dh.p, n, dout.p);
    SHM_CUDA(cudaGetLastError());
    ctx->m->launches++;
    SHM_CUDA(cudaMemcpyAsync(out, dout.p, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost, s));
    SHM_CUDA(cudaStreamSynchronize(s));
    return SHM_OK;
    SHM_GUARD_END
}

int shm_index_hits(shm_ctx* ctx, const shm_index* idx, uint64_t h, int32_t* segm_id, int32_t* tpos, int32_t* r,
                   uint8_t* strand, int64_t cap, int64_t* n_out) {
    if (!ctx || !idx || !n_out) return fail(SHM_ERR_INVALID, "null argument");
    SHM_GUARD_BEGIN
    SHM_CUDA(cudaSetDevice(ctx->m->device));
    cudaStream_t s = ctx->m->stream;
    const shm::IndexStorage* ix = idx->s;
    shm::DevBuf<uint32_t> ac;
    ac.reserve(2);
    k_one_list<<<1, 1, 0, s>>>(ix->dev, h, ac.p);
    SHM_CUDA(cudaGetLastError());
    ctx->m->launches++;
    uint32_t hac[2];
    SHM_CUDA(cudaMemcpyAsync(hac, ac.p, sizeof hac, cudaMemcpyDeviceToHost, s));
    SHM_CUDA(cudaStreamSynchronize(s));
    *n_out = hac[1];
    if ((int64_t)hac[1] > cap) return fail(SHM_ERR_CAPACITY, "output capacity too small");
    std::vector<uint32_t> g(hac[1]), rs(hac[1]);
    if (hac[1]) {
        SHM_CUDA(cudaMemcpy(g.data(), ix->hits.p + hac[0], sizeof(uint32_t) * hac[1], cudaMemcpyDeviceToHost));
        for (uint32_t i = 0; i < hac[1]; i++)
            SHM_CUDA(cudaMemcpy(&rs[i], ix->ref_rs.p + g[i], sizeof(uint32_t), cudaMemcpyDeviceToHost));
    }
    for (uint32_t i = 0; i < hac[1]; i++) {
        int32_t sg = (int32_t)(std::upper_bound(ix->h_seg_off.begin(), ix->h_seg_off.end(), g[i]) - ix->h_seg_off.begin()) - 1;
        // a segment with no k-mers shares its offset with the next one: take the last segment starting at or before g
        if (segm_id) segm_id[i] = sg;
        if (tpos) tpos[i] = (int32_t)(g[i] - ix->h_seg_off[(size_t)sg]);
        if (r) r[i] = (int32_t)(rs[i] >> 1);
        if (strand) strand[i] = (uint8_t)(rs[i] & 1u);
    }
    return SHM_OK;
    SHM_GUARD_END
}

int shm_index_segment(shm_ctx* ctx, const shm_index* idx, int32_t seg, int32_t* r, uint64_t* h, uint8_t* strand,
                      int64_t cap, int64_t* n_out, char* name, int32_t name_cap, int32_t* seg_len) {
    if (!ctx || !idx || !n_out) return fail(SHM_ERR_INVALID, "null argument");
    const shm::IndexStorage* ix = idx->s;
    if (seg < 0 || seg >= (int32_t)ix->names.size()) return fail(SHM_ERR_INVALID, "segment out of range");
    SHM_GUARD_BEGIN
    SHM_CUDA(cudaSetDevice(ctx->m->device));
    const uint32_t a = ix->h_seg_off[(size_t)seg], b = ix->h_seg_off[(size_t)seg + 1];
    *n_out = b - a;
    if (seg_len) *seg_len = ix->seg_len[(size_t)seg];
    if (name && name_cap > 0) {
        std::snprintf(name, (size_t)name_cap, "%s", ix->names[(size_t)seg].c_str());
    }
    if ((int64_t)(b - a) > cap) return fail(SHM_ERR_CAPACITY, "output capacity too small");
    std::vector<uint64_t> hh(b - a);
    std::vector<uint32_t> rs(b - a);
    if (b > a) {
        SHM_CUDA(cudaMemcpy(hh.data(), ix->ref_h.p + a, sizeof(uint64_t) * (b - a), cudaMemcpyDeviceToHost));
        SHM_CUDA(cudaMemcpy(rs.data(), ix->ref_rs.p + a, sizeof(uint32_t) * (b - a), cudaMemcpyDeviceToHost));
    }
    for (uint32_t i = 0; i < b - a; i++) {
        if (r) r[i] = (int32_t)(rs[i] >> 1);
        if (h) h[i] = hh[i];
        if (strand) strand[i] = (uint8_t)(rs[i] & 1u);
    }
    return SHM_OK;
    SHM_GUARD_END
}

static int check_map_args(shm_ctx* ctx, const shm_index* idx, const shm_params* p, int32_t n) {
    if (!ctx || !idx || !p || n < 0) return fail(SHM_ERR_INVALID, "null argument");
    int v = shm_params_validate(p);
    if (v != SHM_OK) return v;
    if (p->k != idx->s->k) return fail(SHM_ERR_INVALID, "params.k differs from the index's k");
    if (p->h_frac != idx->s->h_frac) return fail(SHM_ERR_INVALID, "params.h_frac differs from the index's h_frac");
    return SHM_OK;
}

static int check_reads(const int64_t* offs, int32_t n) {
    for (int32_t i = 0; i < n; i++) {
        int64_t L = offs[i + 1] - offs[i];
        if (L < 0 || L >= ((int64_t)1 << 30)) return fail(SHM_ERR_INVALID, "read length out of range (0 .. 2^30-1)");
    }
    return SHM_OK;
}

int shm_map_batch(shm_ctx* ctx, const shm_index* idx, const shm_params* p, const uint8_t* seqs, const int64_t* offs,
                  int32_t n, shm_map_record* out) {
    int v = check_map_args(ctx, idx, p, n);
    if (v != SHM_OK) return v;
    if (n > 0 && (!seqs || !offs || !out)) return fail(SHM_ERR_INVALID, "null argument");
    if ((v = check_reads(offs, n)) != SHM_OK) return v;
    SHM_GUARD_BEGIN
    shm::map_host(ctx->m, idx->s, *p, seqs, offs, n, out, false);
    return SHM_OK;
    SHM_GUARD_END
}

int shm_map_multi(shm_ctx* const* ctxs, const shm_index* const* idxs, int32_t n_dev, const shm_params* p,
                  const uint8_t* seqs, const int64_t* offs, int32_t n, shm_map_record* out, int32_t* shares) {
    if (!ctxs || !idxs || n_dev <= 0 || !p || n < 0) return fail(SHM_ERR_INVALID, "null argument");
    if (n > 0 && (!seqs || !offs || !out)) return fail(SHM_ERR_INVALID, "null argument");
    for (int32_t d = 0; d < n_dev; d++) {
        int v = check_map_args(ctxs[d], idxs[d], p, n);
        if (v != SHM_OK) return v;
        if (idxs[d]->s->device != ctxs[d]->m->device)
            return fail(SHM_ERR_INVALID, "index " + std::to_string(d) + " is not on its context's device");
        for (int32_t e = 0; e < d; e++)
            if (ctxs[e] == ctxs[d]) return fail(SHM_ERR_INVALID, "a context appears twice");
    }
    int v = check_reads(offs, n);
    if (v != SHM_OK) return v;
    // contiguous shares of about equal bases, in read order
    std::vector<int32_t> cut((size_t)n_dev + 1, 0);
    cut[(size_t)n_dev] = n;
    const int64_t total = n ? offs[n] - offs[0] : 0;
    for (int32_t d = 1; d < n_dev; d++) {
        const int64_t want = offs[0] + total * d / n_dev;
        int32_t lo = cut[(size_t)d - 1], hi = n;  // first read starting at or after want
        while (lo < hi) {
            const int32_t mid = lo + (hi - lo) / 2;
            if (offs[mid] < want) lo = mid + 1;
            else hi = mid;
        }
        cut[(size_t)d] = lo;
    }
    if (shares)
        for (int32_t d = 0; d < n_dev; d++) shares[d] = cut[(size_t)d + 1] - cut[(size_t)d];
    std::vector<int> rc((size_t)n_dev, SHM_OK);
    std::vector<std::string> msg((size_t)n_dev);
    auto work = [&](int32_t d) {
        const int32_t a = cut[(size_t)d], b = cut[(size_t)d + 1];
        if (a == b) return;
        rc[(size_t)d] = shm_map_batch(ctxs[d], idxs[d], p, seqs, offs + a, b - a, out + a);
        if (rc[(size_t)d] != SHM_OK) msg[(size_t)d] = shm_last_error();
    };
    std::vector<std::thread> th;
    for (int32_t d = 1; d < n_dev; d++) th.emplace_back(work, d);
    work(0);
    for (auto& t : th) t.join();
    for (int32_t d = 0; d < n_dev; d++)
        if (rc[(size_t)d] != SHM_OK) return fail(rc[(size_t)d], "device share " + std::to_string(d) + ": " + msg[(size_t)d]);
    return SHM_OK;
}

int shm_map_plain(shm_ctx* ctx, const shm_index* idx, const shm_params* p, const uint8_t* seqs, const int64_t* offs,
                  int32_t n, shm_map_record* out) {
    int v = check_map_args(ctx, idx, p, n);
    if (v != SHM_OK) return v;
    if (n > 0 && (!seqs || !offs || !out)) return fail(SHM_ERR_INVALID, "null argument");
    if ((v = check_reads(offs, n)) != SHM_OK) return v;
    SHM_GUARD_BEGIN
    shm::map_host(ctx->m, idx->s, *p, seqs, offs, n, out, true);
    return SHM_OK;
    SHM_GUARD_END
}

int shm_format_paf_device(shm_ctx* ctx, const shm_index* idx, const shm_params* p, const shm_map_record* rec,
                          int32_t n, const char* names, const double* map_time, char* buf, int64_t cap,
                          int64_t* n_out) {
    if (!ctx || !idx || !p || !n_out || n < 0 || (n > 0 && !rec)) return fail(SHM_ERR_INVALID, "null argument");
    for (int32_t i = 0; i < n; i++)
        if (rec[i].status == 0 && (rec[i].segm_id < 0 || (size_t)rec[i].segm_id >= idx->s->names.size()))
            return fail(SHM_ERR_INVALID, "record with a segment the index does not have");
    SHM_GUARD_BEGIN
    const int64_t total = shm::format_paf_device(ctx->m, *idx->s, *p, rec, n, names, map_time, buf, cap);
    *n_out = total;
    if (buf && total > cap) return fail(SHM_ERR_CAPACITY, "output buffer too small");
    return SHM_OK;
    SHM_GUARD_END
}

int shm_map_paf(shm_ctx* ctx, const shm_index* idx, const shm_params* p, const uint8_t* seqs, const int64_t* offs,
                int32_t n, const char* names, shm_map_record* out, char* buf, int64_t cap, int64_t* n_out) {
    int v = check_map_args(ctx, idx, p, n);
    if (v != SHM_OK) return v;
    if (!n_out || cap < 0) return fail(SHM_ERR_INVALID, "null argument");
    if (n > 0 && (!seqs || !offs)) return fail(SHM_ERR_INVALID, "null argument");
    if ((v = check_reads(offs, n)) != SHM_OK) return v;
    SHM_GUARD_BEGIN
    const int64_t total = shm::map_paf_host(ctx->m, *idx->s, *p, seqs, offs, n, names, out, buf, cap);
    *n_out = total;
    if (buf && total > cap) return fail(SHM_ERR_CAPACITY, "output buffer too small");
    return SHM_OK;
    SHM_GUARD_END
}

void shm_server_config_default(shm_server_config* cfg) {
    if (!cfg) return;
    cfg->slots = 2;
    cfg->max_batch_reads = 16384;
    cfg->max_batch_bases = (int64_t)1 << 28;
    cfg->hbm_budget = 0;
}

struct shm_server {
    shm::Server* s = nullptr;
    int32_t k = 0;
};

int shm_server_create(shm_ctx* ctx, const shm_index* idx, const shm_params* p, const shm_server_config* cfg,
                      shm_server** out) {
    if (!out) return fail(SHM_ERR_INVALID, "null out");
    *out = nullptr;
    int v = check_map_args(ctx, idx, p, 0);
    if (v != SHM_OK) return v;
    shm_server_config c;
    shm_server_config_default(&c);
    if (cfg) c = *cfg;
    if (c.slots < 1 || c.slots > 64 || c.max_batch_reads < 1 || c.max_batch_bases < 1)
        return fail(SHM_ERR_INVALID, "server config out of range");
    SHM_GUARD_BEGIN
    auto* h = new shm_server();
    h->s = shm::server_create(ctx->m->device, idx->s, *p,
                              shm::ServeConfig{c.slots, c.max_batch_reads, c.max_batch_bases, c.hbm_budget});
    *out = h;
    return SHM_OK;
    SHM_GUARD_END
}

int shm_submit(shm_server* srv, const uint8_t* seqs, const int64_t* offs, int32_t n, shm_map_record* out,
               uint64_t* ticket) {
    if (!srv || !ticket || n < 0) return fail(SHM_ERR_INVALID, "null argument");
    if (n > 0 && (!seqs || !offs || !out)) return fail(SHM_ERR_INVALID, "null argument");
    int v = check_reads(offs, n);
    if (v != SHM_OK) return v;
    const int64_t mb = shm::server_max_bases(srv->s);
    for (int32_t i = 0; i < n; i++)
        if (offs[i + 1] - offs[i] > mb)
            return fail(SHM_ERR_INVALID, "read " + std::to_string(i) + " has " + std::to_string(offs[i + 1] - offs[i]) +
                                             " bases, more than a server batch holds (" + std::to_string(mb) + ")");
    SHM_GUARD_BEGIN
    *ticket = shm::server_submit(srv->s, seqs, offs, n, out);
    return SHM_OK;
    SHM_GUARD_END
}

int shm_poll(shm_server* srv, uint64_t ticket, int32_t wait_ms, shm_request_stats* st) {
    if (!srv) return fail(SHM_ERR_INVALID, "null argument");
    shm::ServeStats s{};
    std::string err;
    const int r = shm::server_poll(srv->s, ticket, wait_ms, st ? &s : nullptr, &err);
    if (st && r != SHM_ERR_INVALID && r != SHM_ERR_TIMEOUT) {
        st->status = s.status;
        st->reads = s.reads;
        st->batch_reads = s.batch_reads;
        st->batch_requests = s.batch_requests;
        st->queued_ms = s.queued_ms;
        st->mapped_ms = s.mapped_ms;
        st->total_ms = s.total_ms;
    }
    if (r == SHM_ERR_TIMEOUT) return fail(r, "not done yet");
    if (r != SHM_OK) return fail(r, err);
    return SHM_OK;
}

int shm_server_destroy(shm_server* srv) {
    if (!srv) return SHM_OK;
    SHM_GUARD_BEGIN
    shm::server_destroy(srv->s);
    delete srv;
    return SHM_OK;
    SHM_GUARD_END
}

// Test hook: the admission rule of a server slot (how many of the queued
// requests one batch takes whole, and how many reads of the front request
// when it alone is too large), with no device involved.
int64_t shm_internal_serve_admit(const int64_t* reads, const int64_t* bases, int64_t n, const int64_t* front_lens,
                                 int64_t max_reads, int64_t max_bases, int64_t* part) {
    return (int64_t)shm::admit_parts(reads, bases, (size_t)n, front_lens, max_reads, max_bases, part);
}

int shm_map_fasta(shm_ctx* ctx, const shm_index* idx, const shm_params* p, const shm_fasta* fa, int32_t first,
                  int32_t n, shm_map_record* out) {
    int v = check_map_args(ctx, idx, p, n);
    if (v != SHM_OK) return v;
    if (!fa || (n > 0 && !out) || first < 0 || (int64_t)first + n > fa->f->n)
        return fail(SHM_ERR_INVALID, "null argument or records out of range");
    if (fa->f->device != ctx->m->device) return fail(SHM_ERR_INVALID, "the FASTA is on another device");
    const int64_t* offs = fa->f->offs.data() + first;
    if ((v = check_reads(offs, n)) != SHM_OK) return v;
    if (n == 0) return SHM_OK;
    SHM_GUARD_BEGIN
    shm::FastaDev* f = fa->f;
    f->rec.reserve((size_t)n);
    shm::map_device(ctx->m, idx->s, *p, f->seq.p + offs[0], offs, n, f->rec.p, false);
    SHM_CUDA(cudaMemcpyAsync(out, f->rec.p, sizeof(shm_map_record) * (size_t)n, cudaMemcpyDeviceToHost,
                             ctx->m->stream));
    SHM_CUDA(cudaStreamSynchronize(ctx->m->stream));
    return SHM_OK;
    SHM_GUARD_END
}

int shm_map_batch_device(shm_ctx* ctx, const shm_index* idx, const shm_params* p, const uint8_t* d_seqs,
                         const int64_t* d_offs, const int64_t* h_offs, int32_t n, shm_map_record* d_out) {
    (void)d_offs;
    int v = check_map_args(ctx, idx, p, n);
    if (v != SHM_OK) return v;
    if (n > 0 && (!d_seqs || !h_offs || !d_out)) return fail(SHM_ERR_INVALID, "null argument");
    if ((v = check_reads(h_offs, n)) != SHM_OK) return v;
    SHM_GUARD_BEGIN
    shm::map_device(ctx->m, idx->s, *p, d_seqs, h_offs, n, d_out, false);
    return SHM_OK;
    SHM_GUARD_END
}

}  // extern "C"
