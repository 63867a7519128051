/*
 * segalign_b200_host.h — host-side C++ of the seed-filter path behind a C ABI:
 * query seeding, the scoring table and the multi-threaded seeder pipeline.
 */
#ifndef SEGALIGN_B200_HOST_H
#define SEGALIGN_B200_HOST_H

#include <stdint.h>
#include "segalign_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Host copy of the seed shape and transition flag used by the seeder
 * (src/main.cpp:78-80,152-173 with common/ntcoding.cpp:21-37).  Returns K. */
int sa_host_set_shape(const char* shape, int transition);

/* Seed words of query positions [j0, j1) of `text`, src/seeder.cpp:57-74:
 * (key << 32) + j for every valid 19-mer window, followed by its K
 * transition variants when transitions are on.  Writes at most cap words,
 * returns the full count (call with cap = 0 to size the array). */
uint64_t sa_host_chunk_seeds(const char* text, uint32_t j0, uint32_t j1, uint64_t* out, uint64_t cap);

/* RevComp, common/ntcoding.cpp:63-105 (characters other than ACGTacgtnN& are
 * skipped, as in the reference).  Returns the number of characters written. */
uint64_t sa_host_revcomp(char* dst, const char* src, uint64_t len);

/* Scoring table of src/main.cpp:180-261 (no --scoring file). */
int sa_build_sub_mat(int xdrop, const char* ambiguous, int* sub_mat);

/* Seeder pipeline over one query block already sent to `buffer`
 * (src/main.cpp:373-386 intervals of interval_size from 0 to Lq - seed_size;
 * src/seeder.cpp:47-121 chunks of chunk_size per strand). */
typedef struct {
    uint32_t interval_size;    /* 10,000,000 (src/graph.h:11)          */
    uint32_t interval_overlap; /* extra bases seeded past each interval; 0 in the reference */
    uint32_t chunk_size;       /* 250,000 (src/graph.h:12)             */
    int32_t strand;            /* 1 plus, 2 minus, 3 both              */
    int32_t num_threads;       /* concurrent seeder calls              */
    uint32_t buffer;           /* query buffer id                      */
    uint32_t max_chunks;       /* 0 = every chunk; else a bounded sample */
    uint32_t pad;
} sa_seeder_cfg;

typedef struct {
    uint64_t num_seeds;
    uint64_t num_hits;
    uint64_t num_hsps;
    uint64_t num_calls;
    double seconds;
    double seed_seconds;  /* summed over threads: host seeding           */
    double call_seconds;  /* summed over threads: sa_seed_and_filter     */
    double copy_seconds;  /* summed over threads and the final assembly: HSP copies */
} sa_seeder_stats;

int sa_seeder_run(const sa_seeder_cfg* cfg, const char* query_block, uint32_t query_len, sa_segment** fw,
                  uint64_t* fw_len, sa_segment** rc, uint64_t* rc_len, sa_seeder_stats* stats);

/* Repeat-masker self-alignment driver over a whole sequence
 * (repeat_masker_src/main.cpp:318-426 blocks and intervals with neighbour
 * windows; repeat_masker_src/seeder.cpp:40-186 per-interval chunks on both
 * strands through the rm SeedAndFilter, uint8 coverage of the HSPs' query
 * ranges, runs with coverage >= M).  For every block it sends the block as the
 * resident target (SendRefWriteRequest, rm SendQueryWriteRequest,
 * GenerateSeedPosTable), so it replaces any resident target.  Runs are
 * block-relative, in interval order; a run still open at the block end is not
 * reported, as in the reference. */
typedef struct {
    uint32_t lastz_interval_size;  /* 0 = 10,000,000 (repeat_masker_src/graph.h:11) */
    uint32_t seq_block_size;       /* 0 = 1e9 rounded down to a multiple of the interval */
    float prop_neigh_interval;     /* 0 = 0.2                                  */
    uint32_t M;                    /* 0 = 1: minimum coverage of a reported run */
    uint32_t chunk_size;           /* 0 = the WGA chunk of InitializeProcessor  */
    int32_t strand;                /* 1 plus, 2 minus, 3 both (0 = both)        */
    int32_t num_threads;           /* intervals processed concurrently          */
    uint32_t max_intervals;        /* 0 = every interval; else the first ones   */
    uint32_t step;                 /* seed table step; 0 = 1                    */
    uint32_t pad;
} sa_rm_seeder_cfg;

typedef struct {
    uint32_t block;        /* block index                                 */
    uint32_t interval;     /* interval index over all blocks              */
    uint32_t query_start;  /* block-relative start of the run             */
    uint32_t len;
} sa_rm_run;

typedef struct {
    uint64_t num_seeds;
    uint64_t num_hits;       /* hits looked up (every window)              */
    uint64_t num_hsps;
    uint64_t num_calls;
    uint64_t num_intervals;
    uint64_t num_blocks;
    double seconds;
} sa_rm_seeder_stats;

int sa_rm_seeder_run(const sa_rm_seeder_cfg* cfg, const char* seq, uint64_t seq_len, sa_rm_run** runs,
                     uint64_t* n_runs, sa_rm_seeder_stats* stats);
/* Frees the runs array of sa_rm_seeder_run. */
void sa_free_rm_runs(sa_rm_run* runs);

/* Chromosome table of a concatenated sequence text: chromosome i is
 * starts[i] .. starts[i] + lens[i] (global positions, ascending). */
typedef struct {
    const char* const* names;
    const uint64_t* starts;
    const uint32_t* lens;
    uint32_t count;
    uint32_t pad;
} sa_chrom_table;

/* Segment writer, src/segment_printer.cpp:51-147: the lastz --segments lines
 * of one SeedAndFilter interval's HSP lists, "rchr rstart rend qchr qstart
 * qend +|- score" with 1-based starts and chromosome-relative coordinates.
 * Plus-strand lines follow fw in order; minus-strand lines follow rc in
 * reverse order, with query chromosomes placed in the reverse complement of
 * the query block (start 2*block_start + block_len - start - len).  `query`
 * is the whole query's table; the block is [query_block_start,
 * query_block_start + query_block_len).  Texts are malloc'd (sa_free_text). */
int sa_format_segments(const sa_chrom_table* ref, uint64_t ref_block_start, const sa_chrom_table* query,
                       uint64_t query_block_start, uint32_t query_block_len, const sa_segment* fw, uint64_t n_fw,
                       const sa_segment* rc, uint64_t n_rc, char** plus_text, uint64_t* plus_len, char** minus_text,
                       uint64_t* minus_len);

/* The same writer on the current GPU: the same arguments and the same text,
 * byte for byte (one line per HSP formatted by its own thread).  Returns
 * SA_ERR_CUDA when the device work fails. */
int sa_format_segments_gpu(const sa_chrom_table* ref, uint64_t ref_block_start, const sa_chrom_table* query,
                           uint64_t query_block_start, uint32_t query_block_len, const sa_segment* fw, uint64_t n_fw,
                           const sa_segment* rc, uint64_t n_rc, char** plus_text, uint64_t* plus_len,
                           char** minus_text, uint64_t* minus_len);

/* Interval writer of the repeat masker, repeat_masker_src/segment_printer.cpp:24-62:
 * "chr start end" per run (start 0-based, end = start + len + 1 as the
 * reference prints it), and an end-of-file marker line when markend. */
int sa_format_rm_intervals(const sa_chrom_table* chroms, uint64_t block_start, const sa_rm_run* runs, uint64_t n,
                           int markend, char** text, uint64_t* len);

void sa_free_text(char* text);

/* ---- FASTA ingest and the whole-file driver (src/main.cpp:297-730) ---- */

/* A FASTA file joined into sequence blocks as src/main.cpp:336-455 (query)
 * and :486-528 (target) join it: records are concatenated with '&' after
 * each; a block closes after the record that takes its length above
 * seq_block_size (that record gets no '&'); the last block's length excludes
 * its trailing '&'.  Chromosome starts and block starts are offsets into
 * text.  Records are read with kseq's rules (common/kseq.h): name up to the
 * first white space, sequence lines up to the next '>'/'@'/'+' line, empty
 * lines skipped, trailing '\r' dropped; gzip or plain. */
typedef struct {
    const char* text;
    uint64_t text_len;
    uint32_t num_chroms;
    uint32_t num_blocks;
    const char* const* names;
    const uint64_t* chrom_start;
    const uint32_t* chrom_len;
    const uint64_t* block_start;
    const uint32_t* block_len;
    void* impl;
} sa_seq_set;

/* Reads `path` (seq_block_size 0 = 500,000,000, src/graph.h:10).  Free with sa_seq_set_free. */
int sa_fasta_load(const char* path, uint32_t seq_block_size, sa_seq_set* out);
void sa_seq_set_free(sa_seq_set* s);

/* One target file against one query file, src/main.cpp:297-730: every target
 * block is sent and its seed table built; the query blocks stream through the
 * two query buffers (BUFFER_DEPTH = 2): block k is written into buffer k % 2
 * by a loader thread once block k - 2 has finished, while the seeders work on
 * block k - 1 from the other buffer.  Each query block is cut into intervals
 * of interval_size over [0, len - seed_size) and each interval into chunk_size
 * SeedAndFilter calls per strand (src/seeder.cpp:47-121).  Per interval, the
 * lastz --segments lines of its HSPs (plus strand, then minus; the text
 * sa_format_segments gives, written by the GPU segment writer) go to
 * segments_path, and its HSP records to hsp_path as
 * {u32 target block, u32 query block, u32 interval, u32 strand, sa_segment};
 * a writer thread puts out interval i while the seeders run interval i + 1. 
 * Needs sa_initialize_interface, sa_generate_shape_pos, sa_host_set_shape and
 * sa_initialize_processor first; replaces the resident target and query
 * buffers 0 and 1. */
typedef struct {
    const char* target_path;
    const char* query_path;
    const char* segments_path;  /* NULL: no segments file           */
    const char* hsp_path;       /* NULL: no HSP record file         */
    uint32_t seq_block_size;    /* 0 = 500,000,000                  */
    uint32_t interval_size;     /* 0 = 10,000,000                   */
    uint32_t interval_overlap;  /* extra bases seeded past each interval; 0 as in the reference */
    uint32_t chunk_size;        /* 0 = 250,000                      */
    int32_t strand;             /* 0 or 3 both, 1 plus, 2 minus     */
    int32_t num_threads;        /* concurrent seeder calls; 0 = 16  */
    uint32_t step;              /* seed table step; 0 = 1           */
    uint32_t pad;
} sa_align_cfg;

typedef struct {
    uint64_t ref_blocks;
    uint64_t query_blocks;
    uint64_t intervals;
    uint64_t num_seeds;
    uint64_t num_hits;
    uint64_t num_hsps;
    double seconds;              /* whole call                                   */
    double read_seconds;         /* FASTA parsing and block assembly             */
    double table_seconds;        /* target uploads and seed-table builds         */
    double query_write_seconds;  /* query block uploads (loader thread)          */
    double overlap_seconds;      /* of those, while the seeders ran the other buffer */
    double calls_seconds;        /* seeding and SeedAndFilter calls, interval by interval */
    double output_seconds;       /* HSP records and segment lines (writer thread, overlaps the calls) */
} sa_align_stats;

int sa_align_fasta(const sa_align_cfg* cfg, sa_align_stats* stats);

#ifdef __cplusplus
}
#endif
#endif
