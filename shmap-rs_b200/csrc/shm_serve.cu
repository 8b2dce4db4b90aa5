// Serving with continuous batching: a server keeps one index resident on the
// device and maps read requests that callers submit at any time, from any
// thread.
//
// The reference maps one file per run (src/shmap/mod.rs:458-636: a reader
// thread, N mapping workers over a shared immutable index, an in-order
// collector). Here the unit of work is a request (a caller's reads), and the
// mapping workers are device slots. Each slot owns a device context of its own
// (stream, scratch, pinned staging), so the slots' batches run on the device
// at the same time. A free slot takes the queued requests in arrival order,
// as many as fit its limits: at most max_batch_reads reads and, in bases, its
// share of the HBM budget divided by the device bytes a base costs at the
// index's hash ratio. A request larger than those limits is taken in parts,
// each the longest run of its next reads that fits (a single read longer than
// the base limit is refused when submitted), so no batch exceeds the budget.
// Requests that arrive while the slots are busy wait in the queue and join
// the next batch a slot takes.
//
// Each request of a batch is copied from the caller's memory straight to its
// place in the slot's device buffer (one copy a request, direct from pinned
// memory), the batch is mapped by the device-resident path (the same kernels
// and batch logic as every other entry point, so a read's record does not
// depend on the batch it travels in), and its records are copied back into
// each request's own output. A batch that fails reports its error to every
// request in it; the slot carries on. A slot's buffers are sized for a full
// batch when the server starts.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <exception>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "shm_common.cuh"
#include "shm_internal.hpp"
#include "shm_map.cuh"
#include "shm_serve.hpp"

namespace shm {

using Clock = std::chrono::steady_clock;

static double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

size_t admit_parts(const int64_t* reads, const int64_t* bases, size_t n, const int64_t* front_lens,
                   int64_t max_reads, int64_t max_bases, int64_t* part) {
    *part = 0;
    size_t k = 0;
    int64_t r = 0, b = 0;
    for (; k < n; k++) {
        if (r + reads[k] > max_reads || b + bases[k] > max_bases) break;
        r += reads[k];
        b += bases[k];
    }
    if (k == 0 && n > 0) {  // the front request alone is larger than a batch: its first reads that fit
        int64_t c = 0, cb = 0;
        while (c < reads[0] && c < max_reads && cb + front_lens[c] <= max_bases) cb += front_lens[c++];
        *part = std::max<int64_t>(c, 1);
    }
    return k;
}

struct Request {
    const uint8_t* seqs;
    const int64_t* offs;
    int32_t n;
    shm_map_record* out;
    Clock::time_point t_submit, t_start, t_done;
    int32_t taken = 0;    // reads handed to slots so far (a request larger than a batch goes in parts)
    int32_t written = 0;  // reads whose records are in out
    bool started = false, done = false;
    int status = 0;
    std::string err;
    int32_t batch_reads = 0, batch_requests = 0;
    int64_t bases_from(int32_t i) const { return n ? offs[n] - offs[i] : 0; }
};

// Reads [first, first + count) of a request, mapped in one batch.
struct Part {
    Request* r;
    int32_t first, count;
    int64_t bases() const { return r->offs[first + count] - r->offs[first]; }
};

struct Slot {
    MapCtx* c = nullptr;
    shm_map_record* h_out = nullptr;  // pinned records of a batch
    size_t h_out_cap = 0;
    DevBuf<uint8_t> d_seq;
    DevBuf<shm_map_record> d_out;
    std::vector<int64_t> offs;
    std::thread th;
};

struct Server {
    const IndexStorage* ix;
    shm_params p;
    int device;
    int32_t max_reads;
    int64_t max_bases;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request*> queue;
    std::unordered_map<uint64_t, Request*> reqs;
    uint64_t next_ticket = 1;
    bool stop = false;
    std::vector<Slot> slots;
};

static void grow_pinned(void** p, size_t* cap, size_t want) {
    if (want <= *cap && *p) return;
    if (*p) SHM_CUDA(cudaFreeHost(*p));
    *p = nullptr;
    *cap = 0;
    want = std::max<size_t>(want + want / 4, 1 << 20);
    SHM_CUDA(cudaHostAlloc(p, want, cudaHostAllocDefault));
    *cap = want;
}

static void run_slot(Server* S, Slot* sl) {
    cudaSetDevice(S->device);
    std::vector<Part> batch;
    std::vector<int64_t> rq_reads, rq_bases, front_lens;
    for (;;) {
        batch.clear();
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv_work.wait(lk, [&] { return S->stop || !S->queue.empty(); });
            if (S->queue.empty()) return;  // stopping, and nothing left to map
            rq_reads.clear();
            rq_bases.clear();
            for (Request* r : S->queue) {
                rq_reads.push_back(r->n - r->taken);
                rq_bases.push_back(r->bases_from(r->taken));
                if ((int64_t)rq_reads.size() > S->max_reads) break;  // enough to decide
            }
            Request* f = S->queue.front();
            front_lens.clear();
            if (rq_reads[0] > S->max_reads || rq_bases[0] > S->max_bases)
                for (int32_t i = f->taken; i < f->n && (int64_t)front_lens.size() < S->max_reads; i++)
                    front_lens.push_back(f->offs[i + 1] - f->offs[i]);
            int64_t part = 0;
            const size_t k = admit_parts(rq_reads.data(), rq_bases.data(), rq_reads.size(), front_lens.data(),
                                         S->max_reads, S->max_bases, &part);
            const auto now = Clock::now();
            auto start = [&](Request* r) {
                if (!r->started) r->t_start = now;
                r->started = true;
            };
            for (size_t i = 0; i < k; i++) {
                Request* r = S->queue.front();
                S->queue.pop_front();
                start(r);
                batch.push_back(Part{r, r->taken, r->n - r->taken});
                r->taken = r->n;
            }
            if (part > 0) {
                start(f);
                batch.push_back(Part{f, f->taken, (int32_t)part});
                f->taken += (int32_t)part;
                if (f->taken == f->n) S->queue.pop_front();
            }
        }
        int64_t nreads = 0, nbases = 0;
        for (const Part& q : batch) {
            nreads += q.count;
            nbases += q.bases();
        }
        int status = SHM_OK;
        std::string err;
        try {
            MapCtx* c = sl->c;
            grow_pinned((void**)&sl->h_out, &sl->h_out_cap, sizeof(shm_map_record) * (size_t)std::max<int64_t>(nreads, 1));
            sl->d_seq.reserve((size_t)nbases + 32);
            sl->d_out.reserve((size_t)std::max<int64_t>(nreads, 1));
            sl->offs.assign(1, 0);
            int64_t at = 0;
            for (const Part& q : batch) {  // each part's reads to their place in the batch
                const Request* r = q.r;
                const int64_t b = q.bases(), o0 = r->offs[q.first];
                if (b)
                    SHM_CUDA(cudaMemcpyAsync(sl->d_seq.p + at, r->seqs + o0, (size_t)b, cudaMemcpyHostToDevice,
                                             c->stream));
                for (int32_t i = q.first; i < q.first + q.count; i++) sl->offs.push_back(at + (r->offs[i + 1] - o0));
                at += b;
            }
            SHM_CUDA(cudaMemsetAsync(sl->d_seq.p + at, 0, 32, c->stream));
            c->work[W_H2D_BYTES] += nbases;
            map_device(c, S->ix, S->p, sl->d_seq.p, sl->offs.data(), (int32_t)nreads, sl->d_out.p, false);
            SHM_CUDA(cudaMemcpyAsync(sl->h_out, sl->d_out.p, sizeof(shm_map_record) * (size_t)nreads,
                                     cudaMemcpyDeviceToHost, c->stream));
            c->work[W_D2H_BYTES] += (int64_t)sizeof(shm_map_record) * nreads;
            SHM_CUDA(cudaStreamSynchronize(c->stream));
            int64_t pos = 0;
            for (const Part& q : batch) {  // scatter: each part's records into its request's output
                if (q.count)
                    std::memcpy(q.r->out + q.first, sl->h_out + pos, sizeof(shm_map_record) * (size_t)q.count);
                pos += q.count;
            }
        } catch (const shm_cuda_error& e) {
            status = e.err == cudaErrorMemoryAllocation ? SHM_ERR_NOMEM : SHM_ERR_CUDA;
            err = cudaGetErrorString(e.err);
            cudaGetLastError();
        } catch (const std::bad_alloc&) {
            status = SHM_ERR_NOMEM;
            err = "host allocation failed";
        } catch (const std::exception& e) {  // reported to the batch's requests; the slot carries on
            status = SHM_ERR_CUDA;
            err = std::string("internal error: ") + e.what();
        }
        {
            std::lock_guard<std::mutex> lk(S->mu);
            const auto now = Clock::now();
            for (const Part& q : batch) {
                Request* r = q.r;
                if (status != SHM_OK && r->status == SHM_OK) {
                    r->status = status;
                    r->err = err;
                }
                r->batch_reads = (int32_t)nreads;
                r->batch_requests = (int32_t)batch.size();
                r->written += q.count;
                if (r->written == r->n) {
                    r->t_done = now;
                    r->done = true;
                }
            }
        }
        S->cv_done.notify_all();
    }
}

Server* server_create(int device, const IndexStorage* ix, const shm_params& p, const ServeConfig& cfg) {
    auto* S = new Server();
    S->ix = ix;
    S->p = p;
    S->device = device;
    const int nslots = std::max(1, cfg.slots);
    size_t budget = cfg.hbm_budget;
    try {
        SHM_CUDA(cudaSetDevice(device));
        if (budget == 0) {
            size_t fr = 0, tot = 0;
            SHM_CUDA(cudaMemGetInfo(&fr, &tot));
            budget = fr / 2;
        }
        // device bytes a batch costs per base: the read itself plus, per
        // sketched k-mer (h_frac of the bases), its sketch entry, seed record,
        // probe-table slots, bucket slots and jobs (128 bytes bounds them)
        const double per_base = 1.0 + 128.0 * p.h_frac;
        const int64_t by_budget = (int64_t)((double)(budget / (size_t)nslots) / per_base);
        S->max_reads = std::max(1, cfg.max_batch_reads);
        S->max_bases = std::max<int64_t>(1, std::min<int64_t>(cfg.max_batch_bases, by_budget));
        S->slots = std::vector<Slot>((size_t)nslots);
        for (Slot& sl : S->slots) {
            sl.c = mapctx_create(device, budget / (size_t)nslots);
            sl.d_seq.reserve((size_t)S->max_bases + 32);
            sl.d_out.reserve((size_t)S->max_reads);
            grow_pinned((void**)&sl.h_out, &sl.h_out_cap, sizeof(shm_map_record) * (size_t)S->max_reads);
        }
        for (Slot& sl : S->slots) sl.th = std::thread(run_slot, S, &sl);
    } catch (...) {
        server_destroy(S);
        throw;
    }
    return S;
}

int64_t server_max_bases(const Server* S) { return S->max_bases; }

uint64_t server_submit(Server* S, const uint8_t* seqs, const int64_t* offs, int32_t n, shm_map_record* out) {
    auto* r = new Request();
    r->seqs = seqs;
    r->offs = offs;
    r->n = n;
    r->out = out;
    r->t_submit = Clock::now();
    uint64_t t;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        t = S->next_ticket++;
        S->reqs[t] = r;
        if (n == 0) {  // nothing to map
            r->t_start = r->t_done = r->t_submit;
            r->done = true;
        } else {
            S->queue.push_back(r);
        }
    }
    if (n) S->cv_work.notify_one();
    return t;
}

int server_poll(Server* S, uint64_t ticket, int32_t wait_ms, ServeStats* st, std::string* err) {
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end()) {
        *err = "unknown ticket";
        return SHM_ERR_INVALID;
    }
    Request* r = it->second;
    if (!r->done) {
        if (wait_ms < 0)
            S->cv_done.wait(lk, [&] { return r->done; });
        else if (wait_ms > 0)
            S->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return r->done; });
        if (!r->done) return SHM_ERR_TIMEOUT;
    }
    if (st) {
        st->status = r->status;
        st->reads = r->n;
        st->batch_reads = r->batch_reads;
        st->batch_requests = r->batch_requests;
        st->queued_ms = ms_between(r->t_submit, r->t_start);
        st->mapped_ms = ms_between(r->t_start, r->t_done);
        st->total_ms = ms_between(r->t_submit, r->t_done);
    }
    const int status = r->status;
    *err = r->err;
    S->reqs.erase(it);
    delete r;
    return status;
}

void server_destroy(Server* S) {
    if (!S) return;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cv_work.notify_all();
    for (Slot& sl : S->slots)
        if (sl.th.joinable()) sl.th.join();  // each slot drains the queue before it stops
    for (Slot& sl : S->slots) {
        if (sl.h_out) cudaFreeHost(sl.h_out);
        sl.d_seq.release();
        sl.d_out.release();
        mapctx_destroy(sl.c);
    }
    for (auto& kv : S->reqs) delete kv.second;  // tickets never polled
    delete S;
}

}  // namespace shm
