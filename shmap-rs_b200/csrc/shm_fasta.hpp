// FASTA parsed on the device (see shm_fasta.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/shmap_gpu.h"
#include "shm_internal.hpp"

namespace shm {

// A FASTA file's records with their sequences resident on one device.
struct FastaDev {
    int device = 0;
    int32_t n = 0;
    DevBuf<uint8_t> seq;         // every record's bases back to back, 32 zero bytes past the end
    std::vector<int64_t> offs;   // n+1: record i is seq[offs[i], offs[i+1])
    std::string names;           // '\n'-joined record names
    DevBuf<shm_map_record> rec;  // records of the reads mapped from it
};

// Parses the file's bytes (host memory) on the device: FASTA, or FASTQ when
// the first byte is '@'. Returns null, with the reason in *why, for files the
// host reader handles instead: a FASTA file with a line starting with '@' or
// text before the first header, a FASTQ file not made of four-line records.
FastaDev* fasta_parse_device(int device, cudaStream_t s, const uint8_t* file, int64_t len, std::string* why);

}  // namespace shm
