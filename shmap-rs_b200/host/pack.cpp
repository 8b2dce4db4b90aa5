// Host packing of reads into 2-bit codes and a non-ACGT mask, the form the
// host-buffer path uploads (a quarter of the ASCII bytes, plus an eighth for
// the mask). Codes: a byte b of ACGT in either case has code (b >> 1) & 3
// (A 0, C 1, T 2, G 3); base p is bits 2(p & 15) of codes[p >> 4]. Mask: bit
// p & 31 of mask[p >> 5] is set for every other byte (those hash to 0 on
// both strands, src/sketch.rs:58-97) and for positions past the end.
//
// A byte is ACGT iff its upper-cased value equals the letter its code names:
// 0x41 + 2c, plus 15 for c = 2 (T is 0x54); the AVX2 form tests 32 bytes at
// once. The work is split over a persistent pool of host threads.
#include "pack.hpp"

#include <immintrin.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace shm {
namespace {

// 32 bytes at s: codes of bases 0..31 (two words) and their mask word.
inline void pack32_scalar(const uint8_t* s, uint32_t* codes, uint32_t* mask, int n) {
    uint32_t c0 = 0, c1 = 0, m = 0;
    for (int i = 0; i < 32; i++) {
        uint32_t c = 0, bad = 1;
        if (i < n) {
            const uint32_t b = s[i];
            c = (b >> 1) & 3u;
            const uint32_t want = 0x41u + 2u * c + (c == 2 ? 15u : 0u);
            bad = (b & 0xdfu) == want ? 0u : 1u;
        }
        if (i < 16) c0 |= c << (2 * i);
        else c1 |= c << (2 * (i - 16));
        m |= bad << i;
    }
    codes[0] = c0;
    codes[1] = c1;
    mask[0] = m;
}

// Nonzero mask words (group index, word) of the sparse form, one list per task.
using MaskList = std::vector<std::pair<uint32_t, uint32_t>>;

template <bool SPARSE>
__attribute__((target("avx2"))) void pack_range_avx2(const uint8_t* s, int64_t n32, uint32_t* codes, uint32_t* mask,
                                                     int64_t g_base, MaskList* list) {
    const __m256i k3 = _mm256_set1_epi8(3), kdf = _mm256_set1_epi8((char)0xdf), k41 = _mm256_set1_epi8(0x41),
                  k15 = _mm256_set1_epi8(15), k2 = _mm256_set1_epi8(2);
    const __m256i m1 = _mm256_set1_epi16(0x0401), m2 = _mm256_set1_epi32(0x00100001);
    // the low byte of every 32-bit lane (4 codes each) to the front of each 128-bit half
    const __m256i gather = _mm256_setr_epi8(0, 4, 8, 12, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, 0, 4, 8,
                                            12, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1);
    for (int64_t g = 0; g < n32; g++) {
        const __m256i v = _mm256_loadu_si256((const __m256i*)(s + 32 * g));
        const __m256i c = _mm256_and_si256(_mm256_srli_epi16(v, 1), k3);
        const __m256i u = _mm256_and_si256(v, kdf);
        const __m256i is2 = _mm256_cmpeq_epi8(c, k2);
        const __m256i want = _mm256_add_epi8(_mm256_add_epi8(k41, _mm256_add_epi8(c, c)), _mm256_and_si256(is2, k15));
        const uint32_t good = (uint32_t)_mm256_movemask_epi8(_mm256_cmpeq_epi8(u, want));
        // byte pairs c0 + 4 c1, then pairs of those + 16x: 8 code bits per 32-bit lane
        const __m256i p = _mm256_madd_epi16(_mm256_maddubs_epi16(c, m1), m2);
        const __m256i q = _mm256_shuffle_epi8(p, gather);
        // streaming stores: the output is read next by the copy engine, and
        // plain stores would first read every output line into the cache
        const uint64_t cw = (uint64_t)(uint32_t)_mm256_extract_epi32(q, 0) |
                            ((uint64_t)(uint32_t)_mm256_extract_epi32(q, 4) << 32);
        _mm_stream_si64((long long*)(codes + 2 * g), (long long)cw);
        if (SPARSE) {
            if (~good) list->emplace_back((uint32_t)(g_base + g), ~good);
        } else {
            _mm_stream_si32((int*)(mask + g), (int)~good);
        }
    }
    _mm_sfence();
}

// AVX-512 (BW, VBMI): 64 bytes a step, groups g and g + 1. A byte is ACGT
// (either case) iff its value with the case bit cleared equals the letter its
// code names (a 16-byte table indexed by the code, one byte shuffle, one
// compare into a mask register; a byte with the top bit set never matches).
// The codes of four bases gather into one byte of a 32-bit lane by two
// multiply-adds (c0 + 4 c1, then + 16 (c2 + 4 c3)); one byte permute brings
// the sixteen lanes' low bytes together: the 64 bases' 16 bytes of codes.
// n32 is even; codes + 2 g0 is 16-byte aligned when `aligned` (streaming
// stores), else plain stores are used.
template <bool SPARSE>
__attribute__((target("avx512f,avx512bw,avx512vbmi"))) void pack_range_avx512(const uint8_t* s, int64_t n32,
                                                                              uint32_t* codes, uint32_t* mask,
                                                                              int64_t g_base, MaskList* list,
                                                                              bool aligned) {
    const __m512i k3 = _mm512_set1_epi8(3), kdf = _mm512_set1_epi8((char)0xdf);
    const __m512i m1 = _mm512_set1_epi16(0x0401), m2 = _mm512_set1_epi32(0x00100001);
    // the letter of code c (A, C, T, G) at byte c of every 128-bit lane
    const __m512i letter = _mm512_broadcast_i32x4(_mm_setr_epi8(0x41, 0x43, 0x54, 0x47, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                                                                0, 0, 0));
    alignas(64) uint8_t low_bytes[64];
    for (int i = 0; i < 64; i++) low_bytes[i] = (uint8_t)((4 * i) & 63);  // byte 0 of lane i first
    const __m512i gather = _mm512_load_si512((const void*)low_bytes);
    for (int64_t g = 0; g < n32; g += 2) {
        const __m512i v = _mm512_loadu_si512((const void*)(s + 32 * g));
        const __m512i c = _mm512_and_si512(_mm512_srli_epi16(v, 1), k3);
        const uint64_t good = _mm512_cmpeq_epi8_mask(_mm512_and_si512(v, kdf), _mm512_shuffle_epi8(letter, c));
        const __m512i p = _mm512_madd_epi16(_mm512_maddubs_epi16(c, m1), m2);
        const __m128i q = _mm512_castsi512_si128(_mm512_permutexvar_epi8(gather, p));
        if (aligned) _mm_stream_si128((__m128i*)(codes + 2 * g), q);
        else _mm_storeu_si128((__m128i*)(codes + 2 * g), q);
        const uint64_t bad = ~good;
        if (SPARSE) {
            if (bad) {
                if ((uint32_t)bad) list->emplace_back((uint32_t)(g_base + g), (uint32_t)bad);
                if ((uint32_t)(bad >> 32)) list->emplace_back((uint32_t)(g_base + g + 1), (uint32_t)(bad >> 32));
            }
        } else {
            _mm_stream_si64((long long*)(mask + g), (long long)bad);
        }
    }
    _mm_sfence();
}

bool have_avx512() {
    static const bool v = __builtin_cpu_supports("avx512f") && __builtin_cpu_supports("avx512bw") &&
                          __builtin_cpu_supports("avx512vbmi");
    return v;
}

template <bool SPARSE>
void pack_range_scalar(const uint8_t* s, int64_t n32, uint32_t* codes, uint32_t* mask, int64_t g_base,
                       MaskList* list) {
    for (int64_t g = 0; g < n32; g++) {
        uint32_t m = 0;
        pack32_scalar(s + 32 * g, codes + 2 * g, SPARSE ? &m : mask + g, 32);
        if (SPARSE && m) list->emplace_back((uint32_t)(g_base + g), m);
    }
}

bool have_avx2() {
    static const bool v = __builtin_cpu_supports("avx2");
    return v;
}

// Index of the calling thread among the packing threads: 0 for the thread
// that holds the packing (one at a time), 1.. for the pool's own.
thread_local int t_worker = 0;

// Persistent workers. start(n, f) has them call f(0..n-1) and returns at
// once; finish() waits until every call has returned and no worker holds
// the job; run(n, f) does both, the caller working too. One job at a time.
class Pool {
  public:
    Pool() {
        const unsigned hc = std::max(1u, std::thread::hardware_concurrency());
        for (unsigned i = 1; i < hc; i++)
            th_.emplace_back([this, i] {
                t_worker = (int)i;
                loop();
            });
    }
    ~Pool() {
        finish();
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : th_) t.join();
    }
    void start(int n, std::function<void(int)> f) {
        finish();
        {
            std::lock_guard<std::mutex> g(mu_);
            job_.f = std::move(f);
            job_.n = n;
            job_.next.store(0);
            job_.done = 0;
            cur_ = &job_;
            gen_++;
        }
        cv_.notify_all();
    }
    void finish() {
        std::unique_lock<std::mutex> g(mu_);
        if (!cur_) return;
        done_cv_.wait(g, [&] { return job_.done == job_.n && active_ == 0; });
        cur_ = nullptr;
    }
    void run(int n, std::function<void(int)> f) {
        start(n, std::move(f));
        work(job_);
        finish();
    }
    // finish(), the caller taking tasks of the job in flight first
    void help_finish() {
        bool have;
        {
            std::lock_guard<std::mutex> g(mu_);
            have = cur_ != nullptr;
        }
        if (have) work(job_);
        finish();
    }
    int size() const { return (int)th_.size() + 1; }
    // One task of the job in flight on the calling thread; false when none is left to take.
    bool help_one() {
        {
            std::lock_guard<std::mutex> g(mu_);
            if (!cur_) return false;
        }
        const int i = job_.next.fetch_add(1);
        if (i >= job_.n) return false;
        job_.f(i);
        std::lock_guard<std::mutex> g(mu_);
        if (++job_.done == job_.n) done_cv_.notify_all();
        return true;
    }

  private:
    struct Job {
        std::function<void(int)> f;
        int n = 0;
        std::atomic<int> next{0};
        int done = 0;  // under mu_
    };
    void work(Job& j) {
        for (;;) {
            const int i = j.next.fetch_add(1);
            if (i >= j.n) return;
            j.f(i);
            std::lock_guard<std::mutex> g(mu_);
            if (++j.done == j.n) done_cv_.notify_all();
        }
    }
    void loop() {
        uint64_t seen = 0;
        for (;;) {
            Job* j = nullptr;
            {
                std::unique_lock<std::mutex> g(mu_);
                cv_.wait(g, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
                j = cur_;
                if (j) active_++;
            }
            if (!j) continue;
            work(*j);
            std::lock_guard<std::mutex> g(mu_);
            if (--active_ == 0) done_cv_.notify_all();
        }
    }
    std::vector<std::thread> th_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    Job job_;
    Job* cur_ = nullptr;
    int active_ = 0;
    uint64_t gen_ = 0;
    bool stop_ = false;
};

Pool& pool() {
    static Pool p;
    return p;
}

// The whole 32-byte groups as pool tasks; the tail and two spare groups
// (codes 0, every position masked) by the caller.
template <bool SPARSE>
// (tail: the six code words of groups n32 .. n32 + 2; mask_tail their three
// mask words, or the list)
static void pack_tail(const uint8_t* seq, int64_t nb, uint32_t* tail, uint32_t* mask_tail, MaskList* list) {
    const int64_t n32 = nb / 32;
    uint32_t m = 0;
    pack32_scalar(seq + 32 * n32, tail, SPARSE ? &m : mask_tail, (int)(nb - 32 * n32));
    if (SPARSE && m) list->emplace_back((uint32_t)n32, m);
    for (int64_t g = 1; g < 3; g++) {
        tail[2 * g] = tail[2 * g + 1] = 0;
        if (SPARSE) list->emplace_back((uint32_t)(n32 + g), ~0u);
        else mask_tail[g] = ~0u;
    }
}

static std::vector<MaskList>& task_lists() {
    static std::vector<MaskList> v;
    return v;
}

template <bool SPARSE>
static std::function<void(int)> pack_tasks(const uint8_t* seq, int64_t nb, uint32_t* codes, uint32_t* mask,
                                           int& tasks, int64_t task_groups) {
    const int64_t n32 = nb / 32;
    // an even number of groups a task (the AVX-512 form takes two at a time):
    // task_groups, else a quarter of a thread's share (at least 1 MiB)
    const int64_t per =
        task_groups > 0
            ? std::max<int64_t>(2, task_groups & ~1LL)
            : (std::max<int64_t>(1 << 15, (n32 + 4 * pool().size() - 1) / (4 * pool().size())) + 1) & ~1LL;
    tasks = (int)((n32 + per - 1) / per);
    const bool avx2 = have_avx2(), avx512 = have_avx512() && !std::getenv("SHMAP_PACK_AVX2");
    const bool aligned = ((uintptr_t)codes & 15) == 0;
    std::vector<MaskList>& lists = task_lists();
    if (SPARSE) {
        if ((int)lists.size() < tasks + 1) lists.resize(tasks + 1);
        for (auto& l : lists) l.clear();
    }
    MaskList* L = lists.data();
    return [=](int t) {
        const int64_t g0 = per * t, g1 = std::min(n32, g0 + per);
        if (avx512) {
            const int64_t ge = g0 + ((g1 - g0) & ~1LL);  // pairs of groups; an odd last one by AVX2
            pack_range_avx512<SPARSE>(seq + 32 * g0, ge - g0, codes + 2 * g0, SPARSE ? nullptr : mask + g0, g0,
                                      SPARSE ? L + t : nullptr, aligned);
            if (ge < g1)
                pack_range_avx2<SPARSE>(seq + 32 * ge, g1 - ge, codes + 2 * ge, SPARSE ? nullptr : mask + ge, ge,
                                        SPARSE ? L + t : nullptr);
        } else if (avx2)
            pack_range_avx2<SPARSE>(seq + 32 * g0, g1 - g0, codes + 2 * g0, SPARSE ? nullptr : mask + g0, g0,
                                    SPARSE ? L + t : nullptr);
        else
            pack_range_scalar<SPARSE>(seq + 32 * g0, g1 - g0, codes + 2 * g0, SPARSE ? nullptr : mask + g0, g0,
                                      SPARSE ? L + t : nullptr);
    };
}

// The streamed form with a sink: a task is one piece of `per` groups, packed
// with plain stores into the buffer the sink hands the packing thread (so the
// piece is still in that core's cache when the sink sends it on) and handed
// back with its place among the stream's code words.
static std::function<void(int)> pack_tasks_sink(const uint8_t* seq, int64_t nb, PackSink* sink, int64_t per,
                                                int& tasks, int raw_pct) {
    const int64_t n32 = nb / 32;
    per = std::max<int64_t>(2, per & ~1LL);
    tasks = (int)((n32 + per - 1) / per);
    const bool avx2 = have_avx2(), avx512 = have_avx512() && !std::getenv("SHMAP_PACK_AVX2");
    std::vector<MaskList>& lists = task_lists();
    if ((int)lists.size() < tasks + 1) lists.resize(tasks + 1);
    for (auto& l : lists) l.clear();
    MaskList* L = lists.data();
    return [=](int t) {
        const int64_t g0 = per * t, g1 = std::min(n32, g0 + per);
        const int w = t_worker;
        if (raw_pct > 0 && (int64_t)(t + 1) * raw_pct / 100 > (int64_t)t * raw_pct / 100 &&
            sink->piece_raw(w, seq + 32 * g0, (size_t)g0, (size_t)(g1 - g0)))
            return;
        uint32_t* buf = sink->piece_buffer(w);
        if (!buf) return;  // the sink failed; it reports that itself
        if (avx512) {
            const int64_t ge = g0 + ((g1 - g0) & ~1LL);
            pack_range_avx512<true>(seq + 32 * g0, ge - g0, buf, nullptr, g0, L + t, false);
            if (ge < g1) pack_range_avx2<true>(seq + 32 * ge, g1 - ge, buf + 2 * (ge - g0), nullptr, ge, L + t);
        } else if (avx2)
            pack_range_avx2<true>(seq + 32 * g0, g1 - g0, buf, nullptr, g0, L + t);
        else
            pack_range_scalar<true>(seq + 32 * g0, g1 - g0, buf, nullptr, g0, L + t);
        sink->piece_done(w, buf, (size_t)(2 * g0), (size_t)(2 * (g1 - g0)));
    };
}

int g_sparse_tasks = 0;  // task lists of the sparse packing in flight (the tail's is the last)

// The streamed packing in flight: its tasks in order, chunk_tasks a chunk,
// and how many tasks of each chunk are still to finish.
struct Stream {
    int tasks = 0, chunk_tasks = 1, chunks = 0;
    std::unique_ptr<std::atomic<int>[]> left;
};
Stream g_stream;

}  // namespace

// The pool and the task lists serve one packing at a time: a thread holds
// this lock from pack_reads_host_start to pack_reads_host_wait (or
// pack_reads_host_release), or for the whole of pack_reads_host, so calls
// from several host threads (one per device, say) take turns.
static std::mutex g_pack_mu;
static thread_local bool t_pack_held = false;

void pack_reads_host(const uint8_t* seq, int64_t nb, uint32_t* codes, uint32_t* mask) {
    const bool own = !t_pack_held;
    if (own) g_pack_mu.lock();
    int tasks = 0;
    auto f = pack_tasks<false>(seq, nb, codes, mask, tasks, 0);
    if (tasks > 0) pool().run(tasks, std::move(f));
    pack_tail<false>(seq, nb, codes + 2 * (nb / 32), mask + nb / 32, nullptr);
    if (own) g_pack_mu.unlock();
}

void pack_reads_host_start(const uint8_t* seq, int64_t nb, uint32_t* codes, int64_t task_groups) {
    if (!t_pack_held) {
        g_pack_mu.lock();
        t_pack_held = true;
    }
    pool().finish();
    int tasks = 0;
    auto f = pack_tasks<true>(seq, nb, codes, nullptr, tasks, task_groups);
    pack_tail<true>(seq, nb, codes + 2 * (nb / 32), nullptr, &task_lists()[tasks]);
    g_sparse_tasks = tasks;
    if (tasks > 0) pool().start(tasks, std::move(f));
}

int pack_stream_start(const uint8_t* seq, int64_t nb, uint32_t* codes, int64_t task_groups, int chunk_tasks,
                      PackSink* sink, int raw_pct) {
    if (!t_pack_held) {
        g_pack_mu.lock();
        t_pack_held = true;
    }
    pool().finish();
    int tasks = 0;
    std::function<void(int)> f = sink ? pack_tasks_sink(seq, nb, sink, std::max<int64_t>(2, task_groups), tasks, raw_pct)
                                      : pack_tasks<true>(seq, nb, codes, nullptr, tasks, std::max<int64_t>(2, task_groups));
    Stream& S = g_stream;
    S.tasks = tasks;
    S.chunk_tasks = std::max(1, chunk_tasks);
    S.chunks = std::max(1, (tasks + S.chunk_tasks - 1) / S.chunk_tasks);
    S.left.reset(new std::atomic<int>[(size_t)S.chunks]);
    for (int c = 0; c < S.chunks; c++)
        S.left[(size_t)c].store(std::min(S.chunk_tasks, std::max(0, tasks - c * S.chunk_tasks)));
    // the tail's list joins the last chunk's (with a sink, codes holds only the tail's six words)
    pack_tail<true>(seq, nb, sink ? codes : codes + 2 * (nb / 32), nullptr, &task_lists()[tasks]);
    g_sparse_tasks = tasks;
    if (tasks > 0) {
        std::atomic<int>* left = S.left.get();
        const int ct = S.chunk_tasks;
        pool().start(tasks, [f = std::move(f), left, ct](int t) {
            f(t);
            left[t / ct].fetch_sub(1, std::memory_order_release);
        });
    }
    return S.chunks;
}

bool pack_stream_chunk_ready(int c) {
    return c >= 0 && c < g_stream.chunks && g_stream.left[(size_t)c].load(std::memory_order_acquire) == 0;
}

bool pack_stream_help() { return pool().help_one(); }

int pack_workers() { return pool().size(); }

size_t pack_stream_chunk_list(int c, uint32_t* pairs, size_t cap) {
    const Stream& S = g_stream;
    const int t0 = c * S.chunk_tasks, t1 = (c + 1 == S.chunks) ? S.tasks + 1 : std::min(S.tasks, t0 + S.chunk_tasks);
    size_t n = 0;
    for (int t = t0; t < t1; t++)
        for (const auto& e : task_lists()[(size_t)t]) {
            if (n < cap) {
                pairs[2 * n] = e.first;
                pairs[2 * n + 1] = e.second;
            }
            n++;
        }
    return n;
}

void pack_stream_finish() {
    pool().help_finish();
    g_stream.chunks = 0;
    if (t_pack_held) {
        t_pack_held = false;
        g_pack_mu.unlock();
    }
}

size_t pack_reads_host_wait(uint32_t* pairs, size_t cap) {
    pool().help_finish();  // the caller packs too while it waits
    size_t n = 0;
    for (int t = 0; t <= g_sparse_tasks; t++)
        for (const auto& e : task_lists()[t]) {
            if (n < cap) {
                pairs[2 * n] = e.first;
                pairs[2 * n + 1] = e.second;
            }
            n++;
        }
    if (t_pack_held) {
        t_pack_held = false;
        g_pack_mu.unlock();
    }
    return n;
}

void pack_reads_host_release() {
    if (!t_pack_held) return;
    pool().finish();
    t_pack_held = false;
    g_pack_mu.unlock();
}

size_t packed_code_words(int64_t nb) { return 2 * (size_t)(nb / 32 + 3); }
size_t packed_mask_words(int64_t nb) { return (size_t)(nb / 32 + 3); }

}  // namespace shm

// Test hook (not part of the C ABI of include/shmap_gpu.h): the packing of
// `nb` bytes into caller buffers of packed_code_words / packed_mask_words.
extern "C" int shm_internal_pack_reads(const uint8_t* seq, int64_t nb, uint32_t* codes, uint32_t* mask,
                                       int force_scalar) {
    if (nb < 0 || (nb > 0 && (!seq || !codes || !mask))) return -1;
    if (force_scalar) {
        const int64_t n32 = nb / 32;
        for (int64_t g = 0; g < n32; g++) shm::pack32_scalar(seq + 32 * g, codes + 2 * g, mask + g, 32);
        shm::pack32_scalar(seq + 32 * n32, codes + 2 * n32, mask + n32, (int)(nb - 32 * n32));
        for (int64_t g = n32 + 1; g < n32 + 3; g++) {
            codes[2 * g] = codes[2 * g + 1] = 0;
            mask[g] = ~0u;
        }
        return 0;
    }
    shm::pack_reads_host(seq, nb, codes, mask);
    return 0;
}

// Test hook (not part of the C ABI of include/shmap_gpu.h): the streamed
// packing of `nb` bytes as the host-buffer path runs it (tasks of task_groups
// groups, chunk_tasks a chunk, chunks taken in order as they finish), its
// mask words gathered from the chunks' lists into a dense mask. Returns the
// number of chunks.
extern "C" int shm_internal_pack_stream(const uint8_t* seq, int64_t nb, uint32_t* codes, uint32_t* mask,
                                        int64_t task_groups, int chunk_tasks) {
    if (nb < 0 || (nb > 0 && (!seq || !codes || !mask))) return -1;
    const size_t mw = shm::packed_mask_words(nb);
    for (size_t i = 0; i < mw; i++) mask[i] = 0;
    const int chunks = shm::pack_stream_start(seq, nb, codes, task_groups, chunk_tasks, nullptr);
    std::vector<uint32_t> pairs(2 * (mw + 4));
    for (int c = 0; c < chunks; c++) {
        while (!shm::pack_stream_chunk_ready(c))
            if (!shm::pack_stream_help()) std::this_thread::yield();
        const size_t n = shm::pack_stream_chunk_list(c, pairs.data(), mw + 4);
        for (size_t i = 0; i < n && i < mw + 4; i++) mask[pairs[2 * i]] = pairs[2 * i + 1];
    }
    shm::pack_stream_finish();
    return chunks;
}
