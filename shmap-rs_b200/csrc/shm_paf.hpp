// PAF text on the device (see shm_paf.cu).
#pragma once
#include <stdint.h>

#include "../../include/shmap_gpu.h"

namespace shm {

struct MapCtx;
struct IndexStorage;
struct PafScratch;  // device buffers of the formatting, owned by a context

void paf_scratch_free(PafScratch* p);

// The PAF lines of records rec[0..n) (host memory) for the reads named by
// `names` ('\n'-separated), rendered on the context's device: the same bytes
// as shm_format_paf. Returns the text's length; when buf is not null, its
// first min(cap, length) bytes are written there.
int64_t format_paf_device(MapCtx* c, const IndexStorage& ix, const shm_params& p, const shm_map_record* rec,
                          int32_t n, const char* names, const double* map_time, char* buf, int64_t cap);

// Maps n host reads (map_host) and renders the PAF text of each batch on the
// device as soon as its records are there, so the text of batch b is written
// while the next batches are packed, copied and mapped: the same bytes as
// format_paf_device over the call's records, with t:f: 0. Records go to out
// (host; null = internal pinned memory). Returns the text's length; when buf
// is not null, its first min(cap, length) bytes are written there.
int64_t map_paf_host(MapCtx* c, const IndexStorage& ix, const shm_params& p, const uint8_t* seqs,
                     const int64_t* offs, int32_t n, const char* names, shm_map_record* out, char* buf,
                     int64_t cap);

}  // namespace shm
