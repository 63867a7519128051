// Harness that runs the reference's own seed-filter code (compiled unmodified
// from the reference tree by `make -C oracle ref_kernels`) on one GPU.
//
// TEST INFRASTRUCTURE ONLY.  It pins the CPU oracle against the reference's
// kernels (find_num_hits, find_hits, find_hsps, compress_output and the thrust
// sort/unique chain of src/seed_filter.cu:654-778, or of
// repeat_masker_src/seed_filter.cu:723-855 when built with -DREF_RM), and it
// times them as an unranked baseline.  Nothing in segalign_b200 links it.
//
// The reference is driven through its own function-pointer API (g_* globals,
// src/seed_filter.cu:892-896, common/seed_filter_interface.cu:115-117) plus the
// direct GenerateSeedPosTable call, in src/main.cpp's order.
//
// Input file (little-endian):
//   char[8] "SAREFIN1"
//   u32 mode (0 plain, 1 repeat-masker), u32 transition, u32 noentropy,
//   i32 xdrop, i32 hspthresh, u32 wga_chunk, u32 step, u32 records
//   i64 max_hits (0 keeps the value InitializeProcessor computes)
//   u32 shape_len, char shape[shape_len]          (T/0 form, src/main.cpp:152-171)
//   i32 sub_mat[64]
//   u64 target_len, char target[target_len]
//   u64 query_len,  char query[query_len]         (0 in repeat-masker mode)
//   u32 ncalls, then per call:
//     u32 rev, u32 a, u32 b    plain: a = query buffer; rm: [a, b] = ref window
//     u32 kind                 0: u64 n, u64 seeds[n]; 1: u32 j0, u32 j1 and the
//                              seeds are made here as src/seeder.cpp:57-74 does,
//                              from the query (or its reverse complement)
// Output file: char[8] "SAREFOUT", u32 ncalls, then per call:
//   u64 n_records (header included), u64 num_seeds, f64 seconds of the
//   SeedAndFilter call, u32 header.len, i32 header.score, then the n_records-1
//   body records (16 B each) when `records` is set.
//
// Safety preconditions, checked before any call (exit code 3 when violated):
//   * no code >= 4 (lowercase, N, X, '&') occurs in both sequences, so the
//     reference's count[]/count_del[] arrays are only ever indexed with 0..3
//     (src/seed_filter.cu:235-236,416-422,567-573 index them with r_chr);
//   * every seed, and every table position of its bucket, leaves 32 in-range
//     bases to its right, so no lane of a warp's first tile skips its character load and
//     compares an uninitialised r_chr/q_chr (src/seed_filter.cu:237-238,309-313);
//   * 1 <= seeds per call <= MAX_SEEDS (a call with 0 seeds would read
//     d_hit_num_array[-1], src/seed_filter.cu:684), no seed bucket larger than
//     MAX_HITS (src/seed_filter.cu:690-697 would produce pos = -1) and at most
//     the hit capacity InitializeProcessor allocated per call.
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "DRAM.h"
#include "ntcoding.h"
#include "seed_filter.h"
#include "seed_filter_interface.h"
#include "store.h"
#include "store_gpu.h"

// Globals the reference's host program (src/main.cpp, repeat_masker_src/main.cpp)
// defines and its seed-filter files read.
#ifdef REF_RM
DRAM* seq_DRAM = nullptr;
DRAM* seq_rc_DRAM = nullptr;
#else
DRAM* ref_DRAM = nullptr;
DRAM* query_DRAM = nullptr;
DRAM* query_rc_DRAM = nullptr;
#endif
DRAM::DRAM() : buffer(nullptr), size(0), seqSize(0), bufferPosition(0) {}
DRAM::~DRAM() {}

extern int MAX_HITS;
extern int MAX_SEEDS;

namespace {

struct Reader {
    FILE* f;
    template <typename T>
    T get() {
        T v;
        if (fread(&v, sizeof(T), 1, f) != 1) die("truncated input");
        return v;
    }
    void bytes(void* p, size_t n) {
        if (n && fread(p, 1, n, f) != n) die("truncated input");
    }
    [[noreturn]] static void die(const char* m) {
        fprintf(stderr, "ref_harness: %s\n", m);
        exit(2);
    }
};

[[noreturn]] void refuse(const std::string& m) {
    fprintf(stderr, "ref_harness: precondition failed: %s\n", m.c_str());
    exit(3);
}

// Code of a text character as compress_string assigns it
// (common/seed_filter_interface.cu:28-46).
int code_of(char ch) {
    switch (ch) {
        case 'A': return 0;
        case 'C': return 1;
        case 'G': return 2;
        case 'T': return 3;
        case 'a': case 'c': case 'g': case 't': return 4;
        case 'n': case 'N': return 5;
        case '&': return 7;
        default: return 6;
    }
}

unsigned codes_present(const std::string& s) {
    unsigned m = 0;
    for (char ch : s) m |= 1u << code_of(ch);
    return m;
}

// The seeder's words for positions [j0, j1) of `text` (src/seeder.cpp:57-74).
std::vector<uint64_t> make_seeds(std::string& text, uint32_t j0, uint32_t j1, int seed_size, int kmer_size,
                                 bool transition) {
    std::vector<uint64_t> v;
    for (uint32_t j = j0; j < j1; ++j) {
        uint64_t k = GetKmerIndexAtPos(&text[0], j, seed_size);
        if (k == ((uint32_t)1 << 31)) continue;
        v.push_back((k << 32) + j);
        if (transition)
            for (int t = 0; t < kmer_size; ++t)
                if (IsTransitionAtPos(t) == 1) v.push_back(((k ^ ((uint64_t)TRANSITION_MASK << (2 * t))) << 32) + j);
    }
    return v;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 3) {
        fprintf(stderr, "usage: %s <input> <output>\n", argv[0]);
        return 2;
    }
    FILE* fi = fopen(argv[1], "rb");
    if (!fi) Reader::die("cannot open input");
    Reader r{fi};
    char magic[8];
    r.bytes(magic, 8);
    if (memcmp(magic, "SAREFIN1", 8) != 0) Reader::die("bad magic");
    const uint32_t mode = r.get<uint32_t>();
    const bool transition = r.get<uint32_t>() != 0;
    const bool noentropy = r.get<uint32_t>() != 0;
    const int xdrop = r.get<int32_t>();
    const int hspthresh = r.get<int32_t>();
    const uint32_t wga_chunk = r.get<uint32_t>();
    const uint32_t step = r.get<uint32_t>();
    const bool records = r.get<uint32_t>() != 0;
    const int64_t max_hits = r.get<int64_t>();
    std::string shape(r.get<uint32_t>(), '\0');
    r.bytes(&shape[0], shape.size());
    int sub_mat[64];
    r.bytes(sub_mat, sizeof(sub_mat));
    std::string target(r.get<uint64_t>(), '\0');
    r.bytes(&target[0], target.size());
    std::string query(r.get<uint64_t>(), '\0');
    r.bytes(&query[0], query.size());
#ifdef REF_RM
    if (mode != 1) Reader::die("this build runs the repeat-masker variant only");
#else
    if (mode != 0) Reader::die("this build runs the plain variant only");
#endif
    const int seed_size = (int)shape.size();
    const int kmer_size = GenerateShapePos(shape);

    // --- preconditions on the sequences -----------------------------------
    const std::string& qtext = mode == 1 ? target : query;
    if (mode == 1) {
        if (codes_present(target) & ~0xFu) refuse("repeat-masker sequence holds codes other than ACGT");
    } else if (codes_present(target) & codes_present(query) & ~0xFu) {
        refuse("target and query share a code >= 4");
    }
    if (target.size() < (size_t)seed_size + 64 || qtext.size() < (size_t)seed_size + 64)
        refuse("sequence too short");
    // Keys of the table positions that lie within 32 bases of the target end:
    // a seed with one of them would give a hit whose first tile runs past it.
    std::vector<uint32_t> tail_keys;
    for (size_t p = target.size() - seed_size - 31; p + seed_size <= target.size(); ++p) {
        uint32_t k = GetKmerIndexAtPos(&target[0], p, seed_size);
        if (k != ((uint32_t)1 << 31)) tail_keys.push_back(k);
    }

    // --- reference set-up, in src/main.cpp's order ---------------------------
    if (g_InitializeInterface(1) != 1) Reader::die("InitializeInterface");
    g_SendRefWriteRequest(&target[0], 0, (uint32_t)target.size());
    g_InitializeProcessor(transition, wga_chunk, seed_size, sub_mat, xdrop, hspthresh, noentropy);
    const int64_t hit_capacity = MAX_HITS;  // per-iteration buffers were sized with this
    if (max_hits > 0 && max_hits < MAX_HITS) MAX_HITS = (int)max_hits;
    GenerateSeedPosTable(&target[0], 0, (uint32_t)target.size(), step, seed_size, kmer_size);

    std::vector<uint32_t> index((size_t)1 << (2 * kmer_size));
    if (cudaMemcpy(index.data(), d_index_table[0], index.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        Reader::die("index read-back");

#ifdef REF_RM
    std::string rc_text(target.size(), '\0');
    RevComp(&rc_text[0], &target[0], 0, 0, target.size());
    g_SendQueryWriteRequest();
#else
    query_DRAM = new DRAM();
    query_DRAM->buffer = &query[0];
    std::string rc_text(query.size(), '\0');
    RevComp(&rc_text[0], &query[0], 0, 0, query.size());
    g_SendQueryWriteRequest(0, (uint32_t)query.size(), 0);
#endif

    FILE* fo = fopen(argv[2], "wb");
    if (!fo) Reader::die("cannot open output");
    const uint32_t ncalls = r.get<uint32_t>();
    fwrite("SAREFOUT", 1, 8, fo);
    fwrite(&ncalls, 4, 1, fo);
    for (uint32_t c = 0; c < ncalls; ++c) {
        const bool rev = r.get<uint32_t>() != 0;
        const uint32_t a = r.get<uint32_t>(), b = r.get<uint32_t>();
        const uint32_t kind = r.get<uint32_t>();
        std::vector<uint64_t> seeds;
        if (kind == 0) {
            seeds.resize(r.get<uint64_t>());
            r.bytes(seeds.data(), seeds.size() * 8);
        } else {
            const uint32_t j0 = r.get<uint32_t>(), j1 = r.get<uint32_t>();
            if (j1 < j0 || (size_t)j1 + seed_size > qtext.size()) refuse("seed range outside the query");
            seeds = make_seeds(rev ? rc_text : const_cast<std::string&>(qtext), j0, j1, seed_size, kmer_size,
                               transition);
        }
        // --- per-call preconditions ------------------------------------------
        if (seeds.empty() || seeds.size() > (size_t)MAX_SEEDS) refuse("seed count outside [1, MAX_SEEDS]");
        uint64_t total = 0;
        for (uint64_t w : seeds) {
            const uint32_t key = (uint32_t)(w >> 32), j = (uint32_t)w;
            if (key >= index.size()) refuse("seed key outside the table");
            for (uint32_t tk : tail_keys)
                if (key == tk) refuse("seed key occurs within 32 bases of the target end");
            if ((size_t)j + seed_size + 32 > qtext.size()) refuse("seed within 32 bases of the query end");
            const uint64_t n = index[key] - (key ? index[key - 1] : 0);
            if (n > (uint64_t)MAX_HITS) refuse("one seed has more than MAX_HITS hits");
            total += n;
        }
        if (total > (uint64_t)hit_capacity || total >= (1ull << 32)) refuse("hits beyond the allocated capacity");
#ifndef REF_RM
        if (a != 0) refuse("only query buffer 0 is loaded");
#else
        if (b + 32 >= target.size()) refuse("window end within 32 bases of the sequence end");
#endif
        auto t0 = std::chrono::steady_clock::now();
#ifdef REF_RM
        std::vector<segmentPair> out = g_SeedAndFilter(seeds, rev, a, b);
#else
        std::vector<segmentPair> out = g_SeedAndFilter(seeds, rev, a);
#endif
        auto t1 = std::chrono::steady_clock::now();
        const double secs = std::chrono::duration<double>(t1 - t0).count();
        const uint64_t n = out.size(), ns = seeds.size();
        fwrite(&n, 8, 1, fo);
        fwrite(&ns, 8, 1, fo);
        fwrite(&secs, 8, 1, fo);
        // The header's ref_start/query_start are never set by the reference
        // (src/seed_filter.cu:756-759); only len and score are written out.
        fwrite(&out[0].len, 4, 1, fo);
        fwrite(&out[0].score, 4, 1, fo);
        if (records && n > 1) fwrite(&out[1], sizeof(segmentPair), n - 1, fo);
    }
    fclose(fo);
    fclose(fi);
#ifdef REF_RM
    g_ClearQuery();
#else
    g_ClearQuery(0);
#endif
    g_ShutdownProcessor();
    return 0;
}
