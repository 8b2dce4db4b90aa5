/*
 * shmap-b200: C ABI of the B200 long-read mapping path (libshmapgpu.so).
 *
 * The reference (shmap-rs v1.4.3, crate `shmap`) exposes this path through its
 * Rust API and the `shmap -s -p -k -r -t -m` command line; it has no FFI of its
 * own. These entry points are what a Rust (or any C-ABI) host binds to replace
 * that API one call for one call. Each declaration names the reference
 * function it stands in for.
 *
 * Conventions: every call returns an int status (SHM_OK = 0, negative on
 * error). Host buffers are caller-owned; device buffers are owned by the
 * context or the index. A context serves one host thread at a time.
 * Sequences are raw ASCII bytes exactly as the reference's FASTA reader hands
 * them to FracMinHash::sketch (any case; bytes other than ACGTacgt hash as 0).
 */
#ifndef SHMAP_GPU_H
#define SHMAP_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    SHM_OK = 0,
    SHM_ERR_INVALID = -1,   /* bad argument (message via shm_last_error) */
    SHM_ERR_CUDA = -2,      /* CUDA runtime error */
    SHM_ERR_NOMEM = -3,     /* device allocation failed / over the HBM budget */
    SHM_ERR_CAPACITY = -4,  /* an output buffer is too small */
    SHM_ERR_TIMEOUT = -5    /* a bounded device wait ran out */
};

/* Metric (src/types.rs:299-322). */
enum { SHM_CONTAINMENT = 0, SHM_JACCARD = 1, SHM_BUCKET_SH = 2, SHM_BUCKET_LCS = 3 };

/* Mapping parameters: the fields of Params (src/params.rs:20-186) that the
 * mapping path reads. Defaults are the CLI defaults (shm_params_default). */
typedef struct shm_params {
    int32_t k;              /* -k */
    double h_frac;          /* -r */
    int32_t max_matches;    /* -M, -1 = none */
    double theta;           /* -t */
    double min_diff;        /* -d */
    double max_overlap;     /* -o */
    int32_t metric;         /* -m */
    int32_t no_bucket_pruning; /* -P (NBP) */
    int32_t one_sweep;      /* -B (OS) */
    int32_t abs_pos;        /* -F (AP) */
    double rarity_weight;   /* --rarity-weight: score = rarity-weighted containment (0 = off) */
    double rarity_tiebreak; /* --rarity-tiebreak: band of scores decided by rarity support (0 = off) */
    double rarity_alpha;    /* --rarity-alpha: weights 1 / max(hits, 1)^alpha (0 = follow the others) */
} shm_params;

/* One read's outcome: everything the reference's PAF line is made of
 * (src/mapping.rs:87-107, 161-182, 228-247; src/shmap/mod.rs:871-943).
 * status: 0 mapped, 1 nothing cleared -t, 2 sketch below MIN_HALFLEN
 * (src/shmap/mod.rs:750-783), 3 internal capacity exceeded (retried). */
typedef struct shm_map_record {
    double score, sh, score2;
    int32_t status;
    int32_t read_len, sketch_size, seeds;
    int32_t p_start, p_end, segm_id, t_l, t_r;
    int32_t same_strand, intersection, s_sz;
    int32_t bucket_seg, bucket_b;
    int32_t has_second, intersection2, bucket2_seg, bucket2_b;
    int32_t total_matches, max_seed_matches, seed_matches, seeded_buckets, final_buckets;
    int32_t reserved;
} shm_map_record;
#ifdef __cplusplus
static_assert(sizeof(shm_map_record) == 120, "shm_map_record layout is part of the ABI");
#endif

/* SketchIndex statistics (src/index.rs:343-376, printed by index.rs:665-700). */
typedef struct shm_index_stats {
    int64_t segments, total_nucls, indexed_hits, indexed_kmers, highest_freq_kmer;
    int64_t blacklisted_kmers, blacklisted_hits, sketched_kmers;
} shm_index_stats;

typedef struct shm_ctx shm_ctx;
typedef struct shm_index shm_index;

/* Last error message of this thread (static storage). */
const char* shm_last_error(void);

/* Fills the CLI defaults of src/params.rs:29-116. */
void shm_params_default(shm_params* p);

/* Params::validate (src/params.rs:191-263): SHM_OK or SHM_ERR_INVALID with the
 * reference's message in shm_last_error(). */
int shm_params_validate(const shm_params* p);

/* A device context: one CUDA device, one stream, grow-only scratch.
 * hbm_budget bytes (0 = no limit) bounds the scratch the context keeps. */
int shm_ctx_create(int device, size_t hbm_budget, shm_ctx** out);
int shm_ctx_destroy(shm_ctx* ctx);

/* FracMinHash::sketch_slice_into (src/sketch.rs:167-209) for one host
 * sequence: writes up to cap k-mers (r, h, strand) in sequence order and the
 * total count to *n_out (SHM_ERR_CAPACITY if it exceeds cap). */
int shm_sketch(shm_ctx* ctx, const uint8_t* seq, int64_t len, int32_t k, double h_frac, int32_t offset,
               int32_t* r, uint64_t* h, uint8_t* strand, int64_t cap, int64_t* n_out);

/* FracMinHash::h_thres (src/sketch.rs:126-132). */
uint64_t shm_h_thres(double h_frac);

/* SketchIndex::build_index (src/index.rs:384-663) from segments already read:
 * `seq` holds every segment's bases back to back, seg_off[n_seg+1] are byte
 * offsets, names are '\n'-joined (file order = segm_id order). */
int shm_index_build(shm_ctx* ctx, const uint8_t* seq, const int64_t* seg_off, int32_t n_seg, const char* names,
                    int32_t k, double h_frac, int32_t max_matches, shm_index** out);
int shm_index_destroy(shm_index* idx);
int shm_index_stats_get(const shm_index* idx, shm_index_stats* out);

/* No counterpart in the reference, which sketches and indexes the reference on
 * every run (src/main.rs:45-57): a built index written to a file, and read
 * back onto the device of ctx, so that a service starts mapping without the
 * reference's sequence or a rebuild. The file holds the segments, every
 * reference k-mer and the hash CSR (about 20 bytes per reference k-mer plus
 * the names, and a checksum); the derived tables are rebuilt on load. Load
 * checks every section on the host before any of it reaches the device and
 * answers SHM_ERR_INVALID, with a message, for a file that is missing, of
 * another kind or version, truncated, fails its checksum, or holds arrays an
 * index cannot have (offsets out of order, hashes above the threshold,
 * positions outside their segment, hits that are no reference k-mer).
 * shm_index_file_check makes the same checks on the host alone (no device
 * needed). shm_index_info gives the k, hash ratio and -M (-1 = none) the
 * index was built with. */
int shm_index_save(const shm_index* idx, const char* path);
int shm_index_load(shm_ctx* ctx, const char* path, shm_index** out);
int shm_index_file_check(const char* path);
int shm_index_info(const shm_index* idx, int32_t* k, double* h_frac, int32_t* max_matches);

/* SketchIndex::count (src/index.rs:204-213) for n hashes. */
int shm_index_count(shm_ctx* ctx, const shm_index* idx, const uint64_t* h, int64_t n, int32_t* out);

/* SketchIndex::single_hit / multi_hits (src/index.rs:192-201): the hit list of
 * one hash in (segm_id, r) order; *n_out = its length. */
int shm_index_hits(shm_ctx* ctx, const shm_index* idx, uint64_t h, int32_t* segm_id, int32_t* tpos, int32_t* r,
                   uint8_t* strand, int64_t cap, int64_t* n_out);

/* RefSegment::kmers of one segment (src/sketch.rs:16-27). */
int shm_index_segment(shm_ctx* ctx, const shm_index* idx, int32_t seg, int32_t* r, uint64_t* h, uint8_t* strand,
                      int64_t cap, int64_t* n_out, char* name, int32_t name_cap, int32_t* seg_len);

/* Mapper::map_reads / SHMapper::map_read (src/mapper.rs:15-17,
 * src/shmap/mod.rs:374-971) for n host reads: seqs holds the reads back to
 * back with offs[n+1] byte offsets. One record per read, in input order.
 * Reads are cut into device batches; host<->device copies are inside. */
int shm_map_batch(shm_ctx* ctx, const shm_index* idx, const shm_params* p, const uint8_t* seqs, const int64_t* offs,
                  int32_t n, shm_map_record* out);

/* The same for reads already in device memory (d_seqs 16-byte aligned with 16
 * readable bytes past the end; d_offs device, h_offs the same offsets on the
 * host); d_out is device memory. Used to time the device path alone. */
int shm_map_batch_device(shm_ctx* ctx, const shm_index* idx, const shm_params* p, const uint8_t* d_seqs,
                         const int64_t* d_offs, const int64_t* h_offs, int32_t n, shm_map_record* d_out);

/* Mapper::map_reads over several GPUs of one process (src/shmap/mod.rs:458-636:
 * mapping workers over one shared immutable index, output in input order).
 * ctxs[d] and idxs[d] (d < n_dev) are a context and an index replica on the
 * same device (built there, or loaded from one index file); the reads are cut
 * into n_dev contiguous shares of about equal bases, each mapped by
 * shm_map_batch on its device, all at the same time (one host thread each),
 * and every record lands in out at its read's place. shares (may be NULL)
 * gets each share's read count. Nothing crosses between devices. An error
 * of any share is returned (with its share named) once all have finished. */
int shm_map_multi(shm_ctx* const* ctxs, const shm_index* const* idxs, int32_t n_dev, const shm_params* p,
                  const uint8_t* seqs, const int64_t* offs, int32_t n, shm_map_record* out, int32_t* shares);

/* One read per call, every stage launched for that read alone: the plain
 * one-read-per-launch GPU form the batched path is compared against. */
int shm_map_plain(shm_ctx* ctx, const shm_index* idx, const shm_params* p, const uint8_t* seqs, const int64_t* offs,
                  int32_t n, shm_map_record* out);

/* PAF text of the mapped reads (src/mapping.rs:87-107, 161-182, 228-247;
 * src/shmap/mod.rs:871-943): one line per record with status 0, t:f: from
 * map_time[i] (NULL = 0). names are '\n'-joined. Returns the bytes needed in
 * *n_out; writes at most cap bytes. */
int shm_format_paf(const shm_index* idx, const shm_params* p, const shm_map_record* rec, int32_t n, const char* names,
                   const double* map_time, char* buf, int64_t cap, int64_t* n_out);
/* The same text, byte for byte, rendered on ctx's device (one thread per
 * read; f64 fields rounded exactly, half to even). Same arguments, all in
 * host memory; buf = NULL only measures. SHM_ERR_CAPACITY when the text
 * exceeds cap (its first cap bytes are written). */
int shm_format_paf_device(shm_ctx* ctx, const shm_index* idx, const shm_params* p, const shm_map_record* rec,
                          int32_t n, const char* names, const double* map_time, char* buf, int64_t cap,
                          int64_t* n_out);

/* Mapper::map_reads as the command line runs it (src/mapper.rs:15-17,
 * src/shmap/mod.rs:374-650 with the in-order collector's output,
 * mod.rs:868-963): n host reads in (seqs/offs as in shm_map_batch, names
 * '\n'-joined), the PAF text of the mapped reads out, in input order: the
 * bytes shm_format_paf gives for the same records, t:f: printed as 0 (the
 * batched path keeps no per-read wall clock). The text of each device batch
 * is rendered on the device as soon as the batch is mapped, so it overlaps
 * the next batches. out (may be NULL) gets the records too. *n_out = the
 * text's length; at most cap bytes go to buf (NULL only measures, after
 * mapping everything); SHM_ERR_CAPACITY when the text exceeds cap. Pinned
 * seqs, out and buf keep every copy asynchronous: a pinned buf receives each
 * batch's text while later batches map, and pinned seqs let a share of the
 * batches go up as bytes (the host_raw_share setting). The names are split
 * and uploaded by a helper thread while the first batch is packed. */
int shm_map_paf(shm_ctx* ctx, const shm_index* idx, const shm_params* p, const uint8_t* seqs, const int64_t* offs,
                int32_t n, const char* names, shm_map_record* out, char* buf, int64_t cap, int64_t* n_out);

/* Kernel launches this library issued so far in this process (the bench
 * reports the count inside its timed region). */
int64_t shm_ctx_launches(const shm_ctx* ctx);

/* The CUDA stream (cudaStream_t) every call of this context runs on, so a
 * caller can bracket calls with its own events on the same stream. */
void* shm_ctx_stream(const shm_ctx* ctx);

/* Per-stage device timing with CUDA events on the context's stream (off by
 * default). shm_ctx_stage_times fills up to n stages: accumulated
 * milliseconds and number of timed launches; returns the number of stages.
 * shm_stage_name(i) names stage i. on = 0 also clears the totals. */
int shm_ctx_set_timing(shm_ctx* ctx, int on);
int shm_ctx_stage_times(const shm_ctx* ctx, double* ms, int64_t* launches, int n);
const char* shm_stage_name(int i);

/* Work counters of every mapping call of this context (reads, bases,
 * sketched k-mers, distinct seeds, processed seeds, seed hits gathered,
 * buckets, bucket jobs, extension seeds, candidates, refined reference
 * k-mers); cleared with shm_ctx_set_timing(ctx, 0). Returns the count. */
int shm_ctx_work_stats(const shm_ctx* ctx, int64_t* out, int n);
const char* shm_work_stat_name(int i);

/* No counterpart in the reference. The sketch of shm_sketch, for one sequence
 * already in device memory, for callers that must not allocate device memory
 * here: a host whose device memory is fully reserved by its own pool
 * allocator, or a latency-critical loop that cannot pay for cudaMalloc /
 * cudaFree (which may synchronize the device). It allocates nothing: the
 * caller passes d_seq (16-byte aligned, 16 readable bytes past the end) and
 * the outputs d_h[cap] (hashes) and d_rs[cap] (r << 1 | strand), in sequence
 * order; *n_out gets the count (SHM_ERR_CAPACITY if it exceeds cap). Its
 * temporaries live in a static device array of about 0.5 MiB that every GPU
 * loading the library holds until exit, shared by all calls: calls that
 * overlap on the GPU race and must be serialized by the caller. Inputs longer
 * than 4,194,304 windows (4,194,304 + k - 1 bases) are rejected with
 * SHM_ERR_INVALID. The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress) with that device current; make that first
 * call before any stream capture. Every call synchronizes `stream` before it
 * returns: it reads the k-mer count back to the host between its counting
 * and its writing pass. stream = NULL runs on the default stream. */
int shm_sketch_device_noalloc(const uint8_t* d_seq, int64_t len, int32_t k, double h_frac, int32_t offset,
                              uint64_t* d_h, uint32_t* d_rs, int64_t cap, int64_t* n_out, void* stream);

/* No counterpart in the reference: the launch and batch shapes the project's
 * autotuner measures (shmap_b200/autotune.py) instead of fixing them in the
 * code: dev_batch_reads, dev_batch_bases, dev_first_batch_reads,
 * host_batch_reads, host_batch_bases, host_first_batch_reads,
 * sketch_ctas_per_sm, wide_ctas_per_sm, refine_warps_per_sm, device_pack
 * (reads in device memory packed there before sketching: 1, or sketched
 * from their bytes: 0), bt_fast_slots, host_raw_share (reads in pinned host
 * memory: the percent of host batches sent up as bytes on their own stream
 * instead of packed on the host threads), host_pack_task_kib (KiB of reads
 * a packing task takes; 0: four tasks a thread), host_stream (host reads as
 * one packing stream a call: 1 = chunks sent from one pinned buffer, 2 =
 * pieces sent by the packing threads; 0 = host batches one after another),
 * host_stream_bases, host_stream_chunk_kib, host_stream_first_kib,
 * host_stream_last_kib (the device batches of a stream grow from the first
 * size and shrink to the last), host_stream_piece_kib, host_stream_ring and
 * host_stream_raw_share (percent of the pieces sent up as bytes and packed on
 * the device) and plan_mapped (a batch's plan read by a kernel through its
 * pinned block's device mapping instead of copied by the copy engine). None
 * of them
 * changes a result. They are read once per process from the file named by
 * $SHMAP_TUNING, else tuning.conf in the directory above the library's
 * (key = value lines, '#' comments), else built-in defaults;
 * shm_tuning_set changes one for later calls, shm_tuning_load (path NULL =
 * the default place) reads a file again, shm_tuning_source names where the
 * settings came from. Unknown keys and values out of range are
 * SHM_ERR_INVALID. */
int shm_tuning_get(const char* key, int64_t* value);
int shm_tuning_set(const char* key, int64_t value);
int shm_tuning_load(const char* path);
const char* shm_tuning_source(void);

/* FASTA parsed on the device: the reference reads its inputs with
 * needletail (src/io/mod.rs:383-427, src/index.rs:384-393). The file's bytes
 * (host memory) go up once and are parsed on ctx's device: a record per '>'
 * header line, its name the header up to the first space or tab, its
 * sequence its lines joined without '\n' and without one '\r' before a line's
 * end. A file whose first byte is '@' is FASTQ: records of four lines ('@'
 * header, sequence, '+' line, quality; blank lines only at the file's end,
 * which are dropped, so a last record may lack its empty quality line).
 * The sequences stay in device memory, for shm_index_build_fasta and
 * shm_map_fasta. A FASTA file with a line starting with '@' or text before the
 * first header, and a FASTQ file whose line 4r does not start with '@' or
 * line 4r+2 with '+', are refused with SHM_ERR_INVALID: read those on the
 * host. */
typedef struct shm_fasta shm_fasta;
int shm_fasta_parse_device(shm_ctx* ctx, const uint8_t* file, int64_t len, shm_fasta** out);
/* n records; offs (n+1 entries) and names ('\n'-joined) stay owned by fa. */
int shm_fasta_records(const shm_fasta* fa, int32_t* n, const int64_t** offs, const char** names);
/* All records' bases, back to back (offs[n] bytes), to host memory. */
int shm_fasta_copy_seq(const shm_fasta* fa, uint8_t* dst);
int shm_fasta_destroy(shm_fasta* fa);
/* shm_index_build over the parsed records (segments in file order). */
int shm_index_build_fasta(shm_ctx* ctx, const shm_fasta* fa, int32_t k, double h_frac, int32_t max_matches,
                          shm_index** out);
/* shm_map_batch over records [first, first + n) of the parsed reads, from
 * device memory; out (host) gets their records. */
int shm_map_fasta(shm_ctx* ctx, const shm_index* idx, const shm_params* p, const shm_fasta* fa, int32_t first,
                  int32_t n, shm_map_record* out);

/* Serving with continuous batching. The reference maps one file per run
 * through Mapper::map_reads (src/mapper.rs:15-17; src/shmap/mod.rs:458-636:
 * mapping workers over the shared immutable index, output in input order);
 * a server keeps the index resident and maps requests (a caller's reads)
 * submitted at any time from any thread, each request's records in its
 * input order. Its slots, each a device context with its own stream, take
 * the queued requests in arrival order, as many as fit max_batch_reads reads
 * and, in bases, the slot's share of hbm_budget, and map them as one batch (a
 * request larger than that is mapped in parts, so no batch exceeds the
 * budget; shm_submit refuses a single read longer than a batch holds);
 * requests that arrive meanwhile join the next batch a slot takes, and the
 * slots' batches run on the device at the same time. A read's record does
 * not depend on the requests it is batched with. */
typedef struct shm_server shm_server;

typedef struct shm_server_config {
    int32_t slots;            /* device slots (default 2) */
    int32_t max_batch_reads;  /* most reads a slot takes at once (default 16384) */
    int64_t max_batch_bases;  /* most bases a slot takes at once (default 2^28) */
    size_t hbm_budget;        /* device bytes the slots may use together; 0 = half the free memory */
} shm_server_config;

typedef struct shm_request_stats {
    int32_t status;          /* SHM_OK, or the error of the batch that carried the request */
    int32_t reads;           /* reads of the request */
    int32_t batch_reads;     /* reads of the batch it was mapped in */
    int32_t batch_requests;  /* requests of that batch */
    double queued_ms;        /* submitted -> taken by a slot */
    double mapped_ms;        /* taken -> records written */
    double total_ms;         /* submitted -> records written */
} shm_request_stats;

void shm_server_config_default(shm_server_config* cfg);
/* The server maps on ctx's device with idx (built or loaded there) and p; ctx
 * and idx must outlive it. cfg = NULL takes the defaults. */
int shm_server_create(shm_ctx* ctx, const shm_index* idx, const shm_params* p, const shm_server_config* cfg,
                      shm_server** out);
/* Queues n reads (seqs/offs as in shm_map_batch; host memory, pinned or
 * not). seqs, offs and out must stay valid until shm_poll reports the
 * request done; out[0..n) is written then. */
int shm_submit(shm_server* srv, const uint8_t* seqs, const int64_t* offs, int32_t n, shm_map_record* out,
               uint64_t* ticket);
/* Waits up to wait_ms (< 0: until done) for a request. Done: returns its
 * status (SHM_OK or its batch's error), fills st (may be NULL) and releases
 * the ticket. Not done yet: SHM_ERR_TIMEOUT. Unknown ticket: SHM_ERR_INVALID. */
int shm_poll(shm_server* srv, uint64_t ticket, int32_t wait_ms, shm_request_stats* st);
/* Maps every request still queued, then stops. Unpolled tickets are dropped. */
int shm_server_destroy(shm_server* srv);

#ifdef __cplusplus
}
#endif
#endif /* SHMAP_GPU_H */
