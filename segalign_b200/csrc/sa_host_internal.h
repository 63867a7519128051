// sa_host_internal.h — host-side pieces shared by the seeder pipeline
// (sa_host.cpp) and the FASTA ingest driver (sa_ingest.cpp).
#pragma once

#include <cstdint>
#include <utility>
#include <vector>

#include "../../include/segalign_b200.h"
#include "../../include/segalign_b200_host.h"

// One SeedAndFilter call of a seeder: strand 0 seeds query positions
// [j0, j1) of the block, strand 1 the same positions of its reverse
// complement (src/seeder.cpp:47-121).
struct SaHostCall {
    int strand;
    uint32_t j0, j1;
};

// A call's output: header + HSPs as sa_seed_and_filter returned them
// (p == nullptr for a call without seeds); n = HSPs without the header.
struct SaHostCallOut {
    sa_segment* p = nullptr;
    uint64_t n = 0;
};

struct SaHostRunStats {
    uint64_t num_seeds = 0, num_hits = 0, num_hsps = 0;
    double seed_seconds = 0, call_seconds = 0;
};

// Runs `calls` on `nthreads` host threads: seed words of each chunk
// (src/seeder.cpp:57-74) and sa_seed_and_filter on query buffer `buffer`.
// A chunk without seed words is not called (src/seeder.cpp:76).  On error
// every output is freed and the status is returned.
int sa_host_run_calls(const std::vector<SaHostCall>& calls, const char* query, const char* rctext, uint32_t buffer,
                      int nthreads, std::vector<SaHostCallOut>& res, SaHostRunStats* st);

// Seed size and K of the host shape (sa_host_set_shape).
int sa_host_seed_size();
int sa_host_kmer_size();

// Repeat-masker coverage runs of one interval on the GPU (sa_coverage.cu,
// repeat_masker_src/seeder.cpp:151-186): hsps = (query_start, len) pairs,
// block-relative; runs = (start, len) of the stretches with uint8 coverage
// >= M, in position order, without a run still open at block_len.
int sa_device_coverage_runs(const std::vector<std::pair<uint32_t, uint32_t>>& hsps, uint32_t block_len, uint32_t M,
                            std::vector<std::pair<uint32_t, uint32_t>>& runs);

// sa_format_segments_gpu into a pinned host buffer of the caller (*pinned,
// *cap bytes, reallocated with cudaMallocHost when the text is longer): plus
// lines at [0, plus_len), minus lines at [plus_len, plus_len + minus_len).
// Release the buffer with cudaFreeHost.
int sa_format_segments_pinned(const sa_chrom_table* ref, uint64_t ref_block_start, const sa_chrom_table* query,
                              uint64_t query_block_start, uint32_t query_block_len, const sa_segment* fw,
                              uint64_t n_fw, const sa_segment* rc, uint64_t n_rc, char** pinned, uint64_t* cap,
                              uint64_t* plus_len, uint64_t* minus_len);

// Error state of the API layer (sa_last_error), defined in sa_api.cu.
void sa_set_error(int code, const char* fmt, ...);
