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

}  // namespace shm
