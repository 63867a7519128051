// segalign_b200_shim.hpp — drop-in replacement of the reference's seed-filter
// translation units (src/seed_filter.cu, common/seed_filter_interface.cu,
// common/seed_pos_table.cu) for an unchanged reference host build.
//
// Include this header in exactly ONE C++ translation unit of the host
// program, after the reference's own headers that declare the interface:
//
//     #include "seed_filter.h"             // src/seed_filter.h:4-14 (plain mode)
//     #include "seed_filter_interface.h"   // common/seed_filter_interface.h:3-11
//     #include "ntcoding.h"                // common/ntcoding.h:9 (GenerateSeedPosTable)
//     #include "store.h"                   // src/store.h (query_DRAM)
//     #define SEGALIGN_B200_SHIM_PLAIN     // or SEGALIGN_B200_SHIM_REPEAT_MASKER
//     #include "segalign_b200_shim.hpp"
//
// and link with -lsegalign_b200.  It defines the function-pointer globals the
// reference's seeder and driver call (g_InitializeProcessor, g_SeedAndFilter,
// ... src/seed_filter.cu:892-896, common/seed_filter_interface.cu:115-117)
// plus GenerateSeedPosTable and SendSeedPosTable, with the reference's
// signatures and types (segmentPair, std::vector).  The reference aborts with
// exit() on CUDA errors (common/cuda_utils.h:4-37); the shim does the same
// with the library's message, so callers see the same behaviour.
#pragma once

#include <cstdio>
#include <cstdlib>
#include <vector>

#include "segalign_b200.h"

namespace segalign_b200_shim {

inline void check(int r, const char* what) {
    if (r < 0) {
        std::fprintf(stderr, "Error: %s failed: %s\n", what, sa_last_error());
        std::exit(r == SA_ERR_NO_DEVICE ? 1 : r == SA_ERR_TOO_MANY_GPUS ? 10 : 13);
    }
}

// sa_segment and segmentPair share their layout (src/graph.h:25-30).
static_assert(sizeof(segmentPair) == sizeof(sa_segment), "segmentPair layout");

inline std::vector<segmentPair> to_vector(sa_segment* p, uint64_t n) {
    std::vector<segmentPair> v(n);
    for (uint64_t i = 0; i < n; ++i) {
        v[i].ref_start = p[i].ref_start;
        v[i].query_start = p[i].query_start;
        v[i].len = p[i].len;
        v[i].score = p[i].score;
    }
    sa_free_segments(p);
    return v;
}

// common/seed_filter_interface.cu:49-117
inline int InitializeInterface(int num_gpu) {
    int n = sa_initialize_interface(num_gpu);
    check(n, "InitializeInterface");
    return n;
}
inline void SendRefWriteRequest(char* seq, size_t start_addr, uint32_t len) {
    check(sa_send_ref_write_request(seq, start_addr, len), "SendRefWriteRequest");
}
inline void ClearRef() { check(sa_clear_ref(), "ClearRef"); }

}  // namespace segalign_b200_shim

InitializeInterface_ptr g_InitializeInterface = segalign_b200_shim::InitializeInterface;
SendRefWriteRequest_ptr g_SendRefWriteRequest = segalign_b200_shim::SendRefWriteRequest;
ClearRef_ptr g_ClearRef = segalign_b200_shim::ClearRef;

// common/seed_pos_table.cu:33-47 and :49-109
void SendSeedPosTable(uint32_t* index_table, uint32_t index_table_size, uint32_t* pos_table, uint32_t num_index) {
    segalign_b200_shim::check(sa_send_seed_pos_table(index_table, index_table_size, pos_table, num_index),
                              "SendSeedPosTable");
}
void GenerateSeedPosTable(char* ref_str, size_t start_addr, uint32_t ref_length, uint32_t step, int shape_size,
                          int kmer_size) {
    segalign_b200_shim::check(
        sa_generate_seed_pos_table(ref_str, start_addr, ref_length, step, shape_size, kmer_size),
        "GenerateSeedPosTable");
}

#if defined(SEGALIGN_B200_SHIM_PLAIN)
namespace segalign_b200_shim {
// src/seed_filter.cu:780-896
inline void InitializeProcessor(bool transition, uint32_t WGA_CHUNK, uint32_t seed_size, int* sub_mat, int xdrop,
                                int hspthresh, bool noentropy) {
    check(sa_initialize_processor(transition, WGA_CHUNK, seed_size, sub_mat, xdrop, hspthresh, noentropy),
          "InitializeProcessor");
}
inline void SendQueryWriteRequest(size_t start_addr, uint32_t len, uint32_t buffer) {
    check(sa_send_query_write_request(query_DRAM->buffer, start_addr, len, buffer), "SendQueryWriteRequest");
}
inline std::vector<segmentPair> SeedAndFilter(std::vector<uint64_t> seeds, bool rev, uint32_t buffer) {
    sa_segment* out = nullptr;
    uint64_t n = 0;
    check(sa_seed_and_filter(seeds.data(), (uint32_t)seeds.size(), rev, buffer, &out, &n), "SeedAndFilter");
    return to_vector(out, n);
}
inline void ClearQuery(uint32_t buffer) { check(sa_clear_query(buffer), "ClearQuery"); }
inline void ShutdownProcessor() { check(sa_shutdown_processor(), "ShutdownProcessor"); }
}  // namespace segalign_b200_shim
InitializeProcessor_ptr g_InitializeProcessor = segalign_b200_shim::InitializeProcessor;
SendQueryWriteRequest_ptr g_SendQueryWriteRequest = segalign_b200_shim::SendQueryWriteRequest;
SeedAndFilter_ptr g_SeedAndFilter = segalign_b200_shim::SeedAndFilter;
ClearQuery_ptr g_ClearQuery = segalign_b200_shim::ClearQuery;
ShutdownProcessor_ptr g_ShutdownProcessor = segalign_b200_shim::ShutdownProcessor;

#elif defined(SEGALIGN_B200_SHIM_REPEAT_MASKER)
namespace segalign_b200_shim {
// repeat_masker_src/seed_filter.cu:723-961
inline void InitializeProcessor(bool transition, uint32_t WGA_CHUNK, uint32_t seed_size, int* sub_mat, int xdrop,
                                int hspthresh, bool noentropy) {
    check(sa_initialize_processor(transition, WGA_CHUNK, seed_size, sub_mat, xdrop, hspthresh, noentropy),
          "InitializeProcessor");
}
inline void SendQueryWriteRequest() { check(sa_rm_send_query_write_request(), "SendQueryWriteRequest"); }
inline std::vector<segmentPair> SeedAndFilter(std::vector<uint64_t> seeds, bool rev, uint32_t ref_start,
                                              uint32_t ref_end) {
    sa_segment* out = nullptr;
    uint64_t n = 0;
    check(sa_rm_seed_and_filter(seeds.data(), (uint32_t)seeds.size(), rev, ref_start, ref_end, &out, &n),
          "SeedAndFilter");
    return to_vector(out, n);
}
inline void ClearQuery() { check(sa_rm_clear_query(), "ClearQuery"); }
inline void ShutdownProcessor() { check(sa_shutdown_processor(), "ShutdownProcessor"); }
}  // namespace segalign_b200_shim
InitializeProcessor_ptr g_InitializeProcessor = segalign_b200_shim::InitializeProcessor;
SendQueryWriteRequest_ptr g_SendQueryWriteRequest = segalign_b200_shim::SendQueryWriteRequest;
SeedAndFilter_ptr g_SeedAndFilter = segalign_b200_shim::SeedAndFilter;
ClearQuery_ptr g_ClearQuery = segalign_b200_shim::ClearQuery;
ShutdownProcessor_ptr g_ShutdownProcessor = segalign_b200_shim::ShutdownProcessor;
#else
#error "define SEGALIGN_B200_SHIM_PLAIN or SEGALIGN_B200_SHIM_REPEAT_MASKER before including segalign_b200_shim.hpp"
#endif
