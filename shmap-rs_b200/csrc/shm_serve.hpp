// Serving with continuous batching (see shm_serve.cu).
#pragma once
#include <stddef.h>
#include <stdint.h>

#include <string>

#include "../../include/shmap_gpu.h"

namespace shm {

struct IndexStorage;

struct ServeConfig {
    int slots;
    int32_t max_batch_reads;
    int64_t max_batch_bases;
    size_t hbm_budget;
};

struct ServeStats {
    int32_t status, reads, batch_reads, batch_requests;
    double queued_ms, mapped_ms, total_ms;
};

struct Server;

// One batch's share of a queue whose requests hold reads[i] reads and
// bases[i] bases (what is left of them): whole requests from the front, in
// order, while both totals stay within the limits (the count is returned).
// When the front request alone does not fit, none is taken whole and *part
// gets the number of its first reads (lengths front_lens[], at least
// min(reads[0], max_reads) of them) that fit, at least one; else *part = 0.
size_t admit_parts(const int64_t* reads, const int64_t* bases, size_t n, const int64_t* front_lens,
                   int64_t max_reads, int64_t max_bases, int64_t* part);
// The longest read, in bases, a request may hold.
int64_t server_max_bases(const Server* s);

Server* server_create(int device, const IndexStorage* ix, const shm_params& p, const ServeConfig& cfg);
uint64_t server_submit(Server* s, const uint8_t* seqs, const int64_t* offs, int32_t n, shm_map_record* out);
// SHM_OK (or the request's error) once it is done, then the ticket is
// released; SHM_ERR_TIMEOUT while it is not; SHM_ERR_INVALID for an unknown
// ticket. wait_ms < 0 waits until it is done.
int server_poll(Server* s, uint64_t ticket, int32_t wait_ms, ServeStats* st, std::string* err);
// Maps what is still queued, then stops the slots.
void server_destroy(Server* s);

}  // namespace shm
