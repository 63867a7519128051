/*
 * segalign_b200.h — C ABI of the B200 seed-filter path (drop-in for
 * SegAlign's seed_filter_interface).
 *
 * Every entry point mirrors one reference interface (file:line in
 * thiagogenez/SegAlign) with these deliberate differences:
 *   - status returns (0 = SA_OK, negative = error, message from
 *     sa_last_error()) instead of exit()/assert (common/cuda_utils.h:4-37,
 *     src/seed_filter.cu:660);
 *   - explicit host pointers instead of the query_DRAM global
 *     (src/seed_filter.cu:860);
 *   - results in library-allocated arrays released with sa_free_segments()
 *     instead of a std::vector returned by value;
 *   - concurrent sa_seed_and_filter() calls from several host threads each
 *     take a slot (stream + workspace) from a per-GPU pool, where the
 *     reference takes a whole GPU (src/seed_filter.cu:667-674).
 * Records keep the reference layout: sa_segment == segmentPair
 * (src/graph.h:25-30), element 0 of every SeedAndFilter result is the header
 * {0, 0, total HSPs, num_hits}.
 */
#ifndef SEGALIGN_B200_H
#define SEGALIGN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    uint32_t ref_start;
    uint32_t query_start;
    uint32_t len;
    int32_t score;
} sa_segment;

#define SA_OK 0
#define SA_ERR_ARG -1          /* invalid argument                           */
#define SA_ERR_STATE -2        /* call order (e.g. no target / table / query)  */
#define SA_ERR_CUDA -3         /* CUDA runtime error                          */
#define SA_ERR_NOMEM -4        /* device or host allocation failed            */
#define SA_ERR_MAX_SEEDS -5    /* more seeds than MAX_SEEDS (ref: assert)      */
#define SA_ERR_BAD_SEED -6     /* seed key outside the 4^K table              */
#define SA_ERR_MAX_HITS -7     /* one seed holds >= MAX_HITS hits (ref: UB)   */
#define SA_ERR_CAPACITY -8     /* survivor workspace exceeded                 */
#define SA_ERR_NO_DEVICE -9    /* no CUDA device (ref: exit(1))               */
#define SA_ERR_TOO_MANY_GPUS -10 /* more GPUs requested than present (ref: exit(10)) */

/* ---- device registry and target (common/seed_filter_interface.cu) ---- */

/* InitializeInterface(int num_gpu), common/seed_filter_interface.cu:49-80.
 * num_gpu = -1 uses every visible GPU.  Returns the GPU count or an error. */
int sa_initialize_interface(int num_gpu);

/* SendRefWriteRequest(char* seq, size_t start_addr, uint32_t len),
 * common/seed_filter_interface.cu:82-101: encodes seq[start_addr, +len) and
 * keeps it resident on every GPU (nibble-packed). */
int sa_send_ref_write_request(const char* seq, size_t start_addr, uint32_t len);

/* ClearRef(), common/seed_filter_interface.cu:103-113: frees the target and its table. */
int sa_clear_ref(void);

/* ---- seeds and the target seed-position table ---- */

/* GenerateShapePos(std::string shape), common/ntcoding.cpp:21-37, together
 * with the shape-name handling of src/main.cpp:152-171: accepts "12of19",
 * "14of22" or a pattern of 1/0 (or T/0) characters.  Returns K (the number
 * of sampled positions) or an error.  Default shape: 12of19. */
int sa_generate_shape_pos(const char* shape);

/* GenerateSeedPosTable(char* ref_str, size_t start_addr, uint32_t ref_length,
 * uint32_t step, int shape_size, int kmer_size), common/seed_pos_table.cu:49-109.
 * Built on the GPU from the resident target when (ref_str, start_addr,
 * ref_length) is what sa_send_ref_write_request() received, else from
 * ref_str uploaded for the build.  Buckets hold positions in ascending order
 * (the reference's order inside a bucket is an atomic-add order). */
int sa_generate_seed_pos_table(const char* ref_str, size_t start_addr, uint32_t ref_length, uint32_t step,
                               int shape_size, int kmer_size);

/* SendSeedPosTable(uint32_t* index_table, uint32_t index_table_size,
 * uint32_t* pos_table, uint32_t num_index), common/seed_pos_table.cu:33-47:
 * uploads a host-built table (index_table[k] = positions with key <= k). */
int sa_send_seed_pos_table(const uint32_t* index_table, uint32_t index_table_size, const uint32_t* pos_table,
                           uint32_t num_index);

/* Copy of the resident table of GPU 0 (no reference counterpart; for checks). */
int sa_get_seed_pos_table(uint32_t* index_table, uint64_t index_cap, uint32_t* pos_table, uint64_t pos_cap,
                          uint64_t* index_table_size, uint64_t* num_index);

/* ---- seed filter, plain mode (src/seed_filter.cu) ---- */

/* InitializeProcessor(bool transition, uint32_t WGA_CHUNK, uint32_t
 * input_seed_size, int* sub_mat, int input_xdrop, int input_hspthresh, bool
 * input_noentropy), src/seed_filter.cu:780-847.  sub_mat is the 8x8 table
 * (row = target code, column = query code) of src/main.cpp:180-261.
 * MAX_SEEDS = 13*WGA_CHUNK with transitions else WGA_CHUNK; MAX_HITS as the
 * reference computes it from the GPU's memory (override: sa_set_max_hits). */
int sa_initialize_processor(int transition, uint32_t wga_chunk, uint32_t seed_size, const int* sub_mat, int xdrop,
                            int hspthresh, int noentropy);

/* SendQueryWriteRequest(size_t start_addr, uint32_t len, uint32_t buffer),
 * src/seed_filter.cu:849-869.  The reference reads the global
 * query_DRAM->buffer; here the host block is passed as query_buffer.
 * Keeps the forward and reverse-complement query of `buffer` resident. */
int sa_send_query_write_request(const char* query_buffer, size_t start_addr, uint32_t len, uint32_t buffer);

/* SeedAndFilter(std::vector<uint64_t> seed_offset_vector, bool rev, uint32_t
 * buffer), src/seed_filter.cu:654-778.  seeds are (key << 32) | j words
 * (src/seeder.cpp:57-74).  *out receives header + HSPs (num_anchors+1
 * records); free with sa_free_segments().  Thread safe. */
int sa_seed_and_filter(const uint64_t* seeds, uint32_t num_seeds, int rev, uint32_t buffer, sa_segment** out,
                       uint64_t* out_len);

/* ClearQuery(uint32_t buffer), src/seed_filter.cu:871-880. */
int sa_clear_query(uint32_t buffer);

/* ShutdownProcessor(), src/seed_filter.cu:882-890.  Frees every device
 * buffer of the library (the reference calls cudaDeviceReset). */
int sa_shutdown_processor(void);

/* ---- seed filter, repeat-masker mode (repeat_masker_src/seed_filter.cu) ---- */

/* SendQueryWriteRequest(), repeat_masker_src/seed_filter.cu:925-935: the
 * query is the resident target; builds its reverse complement. */
int sa_rm_send_query_write_request(void);

/* SeedAndFilter(seeds, bool rev, uint32_t ref_start, uint32_t ref_end),
 * repeat_masker_src/seed_filter.cu:723-855.  Hits whose ref_loc is outside
 * [ref_start, ref_end] are counted but not extended. */
int sa_rm_seed_and_filter(const uint64_t* seeds, uint32_t num_seeds, int rev, uint32_t ref_start, uint32_t ref_end,
                          sa_segment** out, uint64_t* out_len);

/* ClearQuery(), repeat_masker_src/seed_filter.cu:937-946. */
int sa_rm_clear_query(void);

/* No counterpart in the reference.  SeedAndFilter for callers that cannot
 * let the library allocate device memory while they run (a host program
 * that owns all device memory through its own fixed-budget pool, or a
 * latency-bound loop that cannot take the device-wide synchronisation of
 * cudaMalloc/cudaFree).  Same output as sa_seed_and_filter(), written to the
 * caller's buffer out[0 .. out_cap); *out_len gets the record count (also
 * when the buffer is too small, which returns SA_ERR_CAPACITY).  Per-call
 * scratch lives in one fixed ~40 MB device array that every GPU using the
 * library holds until exit; at most 262,144 seed words and 262,144 distinct
 * HSPs per call, else SA_ERR_CAPACITY.  The first
 * call on a device looks up that array's address: make it before any stream
 * capture.  Calls share the array and run one at a time; calls that
 * overlapped on the GPU would race.  Needs the resident target, table and
 * query of the normal set-up calls. */
int sa_seed_and_filter_noalloc(const uint64_t* seeds, uint32_t num_seeds, int rev, uint32_t buffer, sa_segment* out,
                               uint64_t out_cap, uint64_t* out_len);

/* ---- batched form (no single reference counterpart) ---- */

/* One unit = one SeedAndFilter call of the reference on the seed words the
 * host seeder builds for query positions [start, end) of `buffer` on strand
 * `rev` (src/seeder.cpp:47-121): its output equals sa_seed_and_filter() on
 * those seeds.  Seeds are generated on the GPU from the resident query. */
typedef struct {
    uint32_t buffer;
    int32_t rev;
    uint32_t start;
    uint32_t end;
} sa_unit;

/* Runs n_units units in as few device passes as the workspace allows.
 * Unit u's records (header + HSPs) are out[offsets[u] .. offsets[u+1]);
 * offsets must hold n_units + 1 entries.  With out == NULL and out_len ==
 * NULL the HSPs stay on the device and only sa_last_call_stats() is filled. */
int sa_seed_and_filter_batch(const sa_unit* units, uint32_t n_units, sa_segment** out, uint64_t* out_len,
                             uint64_t* offsets);

/* Device seeding of a resident query buffer (no reference counterpart; it
 * replaces the host loop of src/seeder.cpp:57-74 for the batched form): the
 * per-position 12-mer keys of both strands are computed on the GPU now.  The
 * batched form otherwise computes them on first use after each query write
 * and keeps them while the query stays. */
int sa_refresh_query_keys(uint32_t buffer);

/* ---- serving form (no reference counterpart) ----
 * A request loop over the resident target and seed table.  A request is one
 * query sequence; it is cut into units exactly as the seeder cuts a query
 * block (src/main.cpp:373-386 intervals, src/seeder.cpp:47-121 chunks and
 * strands), so its result equals sa_seeder_run() on that query alone: one
 * HSP list per strand, the units' lists concatenated in interval/chunk order
 * (no per-unit headers).  Requests are admitted while their device buffers
 * fit in a budget of free HBM taken at sa_serve_start (minus hbm_reserve);
 * admitted requests' units are batched into device passes as they arrive, so
 * a request that arrives while others are on the GPU joins the next pass and
 * its buffers are built while the current pass runs. */
typedef struct {
    uint32_t interval_size;    /* query positions per interval; 0 = 10,000,000 */
    uint32_t interval_overlap; /* positions shared with the next interval      */
    uint32_t chunk_size;       /* positions per unit; 0 = the WGA chunk        */
    int32_t strands;           /* 1 = plus, 2 = minus, 3 = both                */
    uint64_t pass_slots;       /* seed slots per device pass; 0 = 2^25         */
    uint64_t hbm_reserve;      /* free HBM admission leaves unused; 0 = 2 GiB  */
} sa_serve_cfg;

typedef struct {
    double submit_s;           /* seconds since sa_serve_start: submitted      */
    double admit_s;            /* device buffers built                         */
    double done_s;             /* HSP lists complete on the host               */
    uint64_t num_units;
    uint64_t num_passes;       /* device passes the request took part in       */
    uint64_t num_hits;         /* ungapped extensions                          */
    uint64_t num_hsps;
    uint64_t device_bytes;     /* device memory the request held               */
} sa_serve_request_stats;

#define SA_PENDING 1           /* sa_serve_wait: not finished within the timeout */

/* Starts the request loop (one at a time per process); needs a resident
 * target and seed table and an initialised processor. */
int sa_serve_start(const sa_serve_cfg* cfg);
/* Queues a copy of query[0, len); *request_id identifies it. */
int sa_serve_submit(const char* query, uint32_t len, uint64_t* request_id);
/* Waits up to timeout_ms (< 0: no limit) for a request.  SA_OK: *fw / *rc
 * hold its plus / minus HSP lists (free with sa_free_segments) and the
 * request is forgotten; SA_PENDING: not finished yet; < 0: it failed. */
int sa_serve_wait(uint64_t request_id, int timeout_ms, sa_segment** fw, uint64_t* fw_len, sa_segment** rc,
                  uint64_t* rc_len, sa_serve_request_stats* stats);
/* Stops the loop; unfinished requests fail with SA_ERR_STATE. */
int sa_serve_stop(void);

/* ---- results, configuration, diagnostics (no reference counterpart) ---- */

/* Releases an array the library returned.  The two largest batched outputs
 * freed (64 MiB or more each) are kept for the next batched calls' outputs,
 * which then skip the page faults of a fresh allocation (a caller may hold one
 * call's lists while the next call runs); sa_shutdown_processor() frees them. */
void sa_free_segments(sa_segment* segments);

/* MAX_HITS override (src/seed_filter.cu:18,784-791); 0 restores the default. */
int sa_set_max_hits(uint64_t max_hits);

/* Repeat-masker self alignment: drop forward-strand HSPs on the main
 * diagonal (ref_start == query_start).  Off by default (the reference never
 * excludes it). */
int sa_set_rm_exclude_diagonal(int on);

typedef struct {
    uint64_t num_seeds;
    uint64_t num_hits;       /* ungapped extensions (header score)            */
    uint64_t hits_extended;  /* hits actually extended (rm window)            */
    uint64_t seeds_with_hits;
    uint64_t survivors;      /* HSPs kept before dedup                        */
    uint64_t num_hsps;       /* after dedup                                   */
    uint64_t long_hits;      /* hits finished by the warp-per-hit kernel       */
    uint64_t tiles;          /* 32-base tiles the reference would scan          */
    uint32_t num_iter;       /* MAX_HITS iterations                            */
    uint32_t batch_calls;    /* calls that shared the device pass (call coalescing);
                              * above 1, hits_extended, seeds_with_hits, survivors,
                              * long_hits, tiles and the ms_* times are the pass's */
    /* device time of the call's phases (CUDA events on the call's stream),
     * filled when sa_set_timing(1) is on */
    double ms_total, ms_lookup, ms_extend_lane, ms_extend_warp, ms_dedup, ms_copy;
} sa_call_stats;

/* Statistics of the calling thread's last sa_*seed_and_filter* call. */
int sa_last_call_stats(sa_call_stats* stats);

/* Per-phase device timing of the following calls (CUDA events); off by default. */
int sa_set_timing(int on);

/* Number of kernels this library has launched since it was loaded. */
uint64_t sa_kernel_launches(void);

/* Message of the calling thread's last error. */
const char* sa_last_error(void);

/* Tuning knobs of the extension kernels: bases per direction a lane scans
 * before a hit moves to the warp-per-hit queue, threads per CTA, CTAs per SM,
 * hits per warp tile.  -1 keeps a value. */
int sa_set_tuning(int lane_cap, int ext_block, int ext_ctas_per_sm, int tile_hits);

/* Phase timing state set by sa_set_timing. */
int sa_get_timing(void);

/* Autotuner (no reference counterpart).  Times the batched path on `units`
 * under candidate settings of the named tuning parameters (coordinate
 * descent from the current setting; each candidate must reproduce the
 * starting setting's HSP lists exactly, else it is rejected), applies the
 * fastest and records it in cache_path (JSON lines keyed by GPU name and
 * workload signature).  With a cache hit and refresh == 0 the cached setting
 * is applied without timing anything. */
typedef struct {
    const char* cache_path;  /* NULL: no cache                          */
    int32_t repeats;         /* timed runs per candidate (best); 0 = 2   */
    int32_t quick;           /* 1: fewer candidates, one round           */
    int32_t refresh;         /* 1: ignore a cached entry                 */
    int32_t pad;
} sa_autotune_cfg;

typedef struct {
    int32_t ext_ctas_per_sm, step_bases, tile_hits, lane_cap, range_ctas, substeps, switch_now;
    int32_t candidates;      /* settings timed                           */
    int32_t rejected;        /* settings that failed or changed results  */
    int32_t from_cache;
    double ms_start;         /* device ms of the batch at the start       */
    double ms_best;          /* device ms with the chosen setting         */
} sa_autotune_result;

int sa_autotune(const sa_unit* units, uint32_t n_units, const sa_autotune_cfg* cfg, sa_autotune_result* out);

/* Named tuning parameters: "lane_cap", "ext_ctas_per_sm" (2..4), "tile_hits" (32..1024),
 * "substeps" (1..8 steps a lane may take per iteration of the lane kernel),
 * "step_bases" (8, 16 or 32 bases scored per lane step), "range_ctas" (CTAs of the
 * lookup/sort kernels of a batched pass), "call_range_ctas" (the same for one plain or
 * rm call), "call_lane_ctas" (CTAs of one plain call's lane kernel; 0 = half of
 * the batched grid, so that concurrent calls share the GPU), "switch_now" (0/1: a lane
 * starts a hit's left side in the iteration its right side ends), and for the lane
 * kernel of one rm call "rm_lane_ctas" (0 = the batched grid), "rm_substeps" (1..8),
 * "rm_switch_now" (0/1).  Results never depend on them.  Returns SA_OK or SA_ERR_ARG;
 * sa_get_tuning_param returns the current value. */
int sa_set_tuning_param(const char* name, int value);
int sa_get_tuning_param(const char* name);

#ifdef __cplusplus
}
#endif
#endif
