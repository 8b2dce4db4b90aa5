// Host packing of reads into 2-bit codes and a non-ACGT mask (see pack.cpp).
#pragma once
#include <cstddef>
#include <cstdint>

namespace shm {

// Packs nb bytes; codes needs packed_code_words(nb) words, mask
// packed_mask_words(nb) (the spare words past the end hold code 0, masked).
void pack_reads_host(const uint8_t* seq, int64_t nb, uint32_t* codes, uint32_t* mask);
// The same on the host threads in the background with the mask in sparse
// form: start returns at once; wait returns when the packing is complete,
// writing the nonzero mask words as (word index, word) pairs, at most cap of
// them (never more than packed_mask_words(nb)), and returns their number.
// One packing at a time: a thread's start waits for another thread's packing
// to be waited for. The work is cut into tasks of task_groups 32-byte groups
// (rounded down to an even number), or, for task_groups <= 0, into four tasks
// a thread of at least 1 MiB each.
void pack_reads_host_start(const uint8_t* seq, int64_t nb, uint32_t* codes, int64_t task_groups = 0);
size_t pack_reads_host_wait(uint32_t* pairs, size_t cap);
// Receives the code words of a streamed packing piece by piece. A packing
// thread (worker 0 .. pack_workers() - 1; 0 is the thread that holds the
// packing) asks for a buffer of at least 2 * task_groups words, packs one
// task into it with plain stores and hands it back with the task's first code
// word in the stream and its word count. Called concurrently for different
// workers; a sink that cannot go on returns NULL from piece_buffer (the task
// is skipped) and reports the failure itself.
struct PackSink {
    virtual uint32_t* piece_buffer(int worker) = 0;
    virtual void piece_done(int worker, uint32_t* buf, size_t first_word, size_t words) = 0;
    // A task left to the sink as bytes (groups [first_group, first_group +
    // groups) at src): true when the sink took it (no codes, no mask words
    // from the host for those groups), false to have it packed here.
    virtual bool piece_raw(int worker, const uint8_t* src, size_t first_group, size_t groups) { return false; }
    virtual ~PackSink() = default;
};
// The number of packing threads (the pool's and the one holding the packing).
int pack_workers();

// Streamed packing of one call's bytes into codes (packed_code_words(nb)
// words, as pack_reads_host_start lays them out): tasks of task_groups 32-byte
// groups in order, chunk_tasks consecutive tasks a chunk, packed by the
// pool's threads in the background. Returns the number of chunks; the caller
// polls pack_stream_chunk_ready(c), may pack one task itself with
// pack_stream_help() (false when none is left to take), and takes a finished
// chunk's nonzero mask words with pack_stream_chunk_list (as in
// pack_reads_host_wait; the last chunk's include the tail groups'). Chunk c
// covers groups [c * chunk_tasks * task_groups, ...) of the codes, the last
// chunk also the tail. pack_stream_finish waits for every task and ends the
// packing (on every path: it also releases the packing lock).
// With a sink, each task's code words go to the sink instead, and codes
// receives only the six tail words (groups nb / 32 .. nb / 32 + 2).
// raw_pct percent of the tasks (spread evenly) are offered to the sink as
// bytes first (PackSink::piece_raw).
int pack_stream_start(const uint8_t* seq, int64_t nb, uint32_t* codes, int64_t task_groups, int chunk_tasks,
                      PackSink* sink = nullptr, int raw_pct = 0);
bool pack_stream_chunk_ready(int c);
bool pack_stream_help();
size_t pack_stream_chunk_list(int c, uint32_t* pairs, size_t cap);
void pack_stream_finish();
// Ends a packing that will not be waited for (an error in between): the
// packing calls of other threads may start again.
void pack_reads_host_release();
size_t packed_code_words(int64_t nb);
size_t packed_mask_words(int64_t nb);

}  // namespace shm
