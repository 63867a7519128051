/*
 * sa_oracle.h — CPU oracle for the SegAlign seed-filter hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain CPU restatement of the
 * reference's semantics (thiagogenez/SegAlign, commit 8b63a0fe).  It is used
 * by tests/, by __graft_entry__.smoke() and by bench.py's cpu_baseline /
 * --impl reference leg, always as the checker or the timed CPU baseline,
 * never as the product path.
 *
 * Pinning: the reference ships no tests or golden vectors, so both halves are
 * pinned against the reference's own code, compiled from its sources where
 * they lie (oracle/Makefile, outputs in oracle/_ref/).  The seeding half
 * (character coding, shape parsing, k-mer keys, host reverse complement) is
 * checked against its common/ntcoding.cpp ("make ref").  The table /
 * extension / compaction / dedup half is checked against its SeedAndFilter
 * (src/seed_filter.cu, repeat_masker_src/seed_filter.cu and the interface
 * files, built for sm_100a with "make ref_kernels" and driven by
 * ref_harness.cu): live on a GPU, and through the reference outputs recorded
 * in tests/golden/ref_calls.npz on the CPU.
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 16-byte HSP record, identical layout to segmentPair (src/graph.h:25-30). */
typedef struct {
    uint32_t ref_start;
    uint32_t query_start;
    uint32_t len;
    int32_t score;
} or_segment;

/* Filter parameters (src/seed_filter.cu:20-27, InitializeProcessor :780-796). */
typedef struct {
    int32_t sub_mat[64];      /* row = target code, column = query code      */
    int32_t xdrop;
    int32_t hspthresh;
    int32_t noentropy;
    int32_t seed_size;        /* shape span, 19 for 12of19                   */
    int32_t kmer_size;        /* number of T/1 positions, 12 for 12of19      */
    int32_t shape_pos[32];    /* kmer index -> offset in the shape           */
    int32_t transition;       /* 1 = emit the 1-transition seed variants     */
    int32_t rm_exclude_diag;  /* rm mode: drop forward HSPs on the main diagonal */
    uint64_t max_hits;        /* MAX_HITS (dedup scope = MAX_HITS iteration) */
} or_params;

/* Per-call statistics. */
typedef struct {
    uint64_t num_seeds;
    uint64_t num_hits;        /* "ungapped extensions", header score field   */
    uint64_t hits_extended;   /* rm mode: hits inside the reference window    */
    uint64_t tiles_right;     /* 32-base tiles the reference scans, right     */
    uint64_t tiles_left;      /* 32-base tiles the reference scans, left      */
    uint64_t survivors;       /* records kept before dedup                    */
    uint64_t num_hsps;        /* records after dedup (body length)            */
    uint64_t unpinned;        /* entropy-branch HSPs touching reference UB    */
    uint64_t base_steps;      /* bases scored (right + left)                  */
    int32_t  num_iter;
    int32_t  pad;
} or_stats;

/* ---- coding (A.1) ---- */
void or_encode(const char* text, uint64_t len, uint8_t* codes);
void or_encode_rc(const char* text, uint64_t len, uint8_t* rc_codes);
void or_rc_codes(const uint8_t* codes, uint64_t len, uint8_t* rc_codes);
/* host text reverse complement, ntcoding.cpp:63-105 (skips unknown chars); returns chars written */
uint64_t or_revcomp_text(char* dst, const char* src, uint64_t len);

/* ---- scoring table (A.3) ---- */
int or_build_sub_mat(int xdrop, const char* ambiguous, int32_t* sub_mat);

/* ---- shape & keys (A.4, A.5) ---- */
int or_parse_shape(const char* seed_name, or_params* p);
uint32_t or_kmer_index(const char* text, uint64_t pos, const or_params* p);

/* ---- target table (A.6) ---- */
uint64_t or_table_count(const char* text, uint32_t len, uint32_t step, const or_params* p);
int or_build_table(const char* text, uint32_t len, uint32_t step, const or_params* p,
                   uint32_t* index_table, uint32_t* pos_table, uint64_t pos_cap,
                   uint64_t* num_index);

/* ---- query seeds (A.7) ---- */
uint64_t or_chunk_seeds(const char* text, uint32_t j0, uint32_t j1, const or_params* p,
                        uint64_t* out, uint64_t cap);

/* ---- SeedAndFilter (A.8 - A.18) ----
 * Returns 0 on success, <0 on error.  *out receives a malloc'd array of
 * *out_len records: element 0 is the header {0, 0, total_anchors, num_hits},
 * then each MAX_HITS iteration's sorted, deduplicated list.
 * mode 0 = plain, 1 = repeat-masker (rm_ref_start/rm_ref_end window). */
int or_seed_and_filter(const or_params* p,
                       const uint8_t* ref_codes, uint32_t ref_len,
                       const uint8_t* query_codes, uint32_t query_len,
                       const uint32_t* index_table, const uint32_t* pos_table,
                       const uint64_t* seeds, uint64_t num_seeds,
                       int rev, int mode, uint32_t rm_ref_start, uint32_t rm_ref_end,
                       or_segment** out, uint64_t* out_len, or_stats* stats);
void or_free(void* ptr);

/* Single-hit extension, exposed for known-answer tests. */
typedef struct {
    int32_t right_best, right_pos, left_best, left_pos;
    int32_t total, keep, score, entropy_branch;
    double entropy;
    uint32_t tiles_right, tiles_left;
    int32_t unpinned;
    int32_t pad;
} or_hit_result;
void or_extend_hit(const or_params* p, const uint8_t* ref_codes, uint32_t ref_len,
                   const uint8_t* query_codes, uint32_t query_len,
                   uint32_t ref_loc, uint32_t query_loc, or_hit_result* r);

/* ---- seeder pipeline (src/seeder.cpp:47-121) over one query block ----
 * Runs every interval/chunk/strand of one query block against one target
 * block with nthreads std::threads.  Returns 0 on success.  HSP bodies are
 * concatenated per strand in seeder order. */
typedef struct {
    uint32_t interval_size;   /* 10,000,000 (src/graph.h:11)   */
    uint32_t interval_overlap;/* 0 in the reference            */
    uint32_t chunk_size;      /* 250,000 (src/graph.h:12)      */
    int32_t  strand;          /* 1 plus, 2 minus, 3 both       */
    int32_t  nthreads;
    uint32_t max_chunks;      /* 0 = all; else a bounded sample */
} or_pipeline_cfg;

int or_pipeline(const or_params* p, const or_pipeline_cfg* cfg,
                const char* ref_text, uint32_t ref_len,
                const char* query_text, uint32_t query_len,
                const uint32_t* index_table, const uint32_t* pos_table,
                or_segment** fw, uint64_t* fw_len, or_segment** rc, uint64_t* rc_len,
                or_stats* stats);

/* rm interval coverage (repeat_masker_src/seeder.cpp:151-186). */
uint64_t or_rm_intervals(const or_segment* hsps, uint64_t n, uint32_t block_len, uint32_t M,
                         uint32_t* starts, uint32_t* lens, uint64_t cap, uint8_t* scratch_counts);

// repeat_masker_src/main.cpp:319-428: blocks (with neighbour overlap) and
// intervals with their target windows.  Row i of out (cap rows): block,
// block_start (low 32 bits), block_len, start, end, ref_start, ref_end.
// Returns the number of intervals.
uint64_t or_rm_plan(uint64_t seq_len, uint32_t interval_size, uint32_t block_size, float prop_neigh,
                    uint32_t seed_size, uint32_t* out, uint64_t cap);

#ifdef __cplusplus
}
#endif
