// sa_launch.h — host-side launchers of the device kernels (internal).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>
#include <vector>

#include "sa_internal.cuh"

// Per-call device descriptor, read by every kernel of one call so that the
// whole chain can be launched without host-side sizes.
struct SaCallDesc {
    uint64_t num_seeds;     // seed words (plain) or seed slots (batched)
    uint64_t max_hits;      // MAX_HITS (dedup iteration size)
    uint32_t num_units;
    uint32_t num_scopes_max;
    uint32_t rm_exclude_diag;
    uint32_t pad;
};

#define SA_BATCH_ITERS 16

// Batched unit: either a query window [q_start, q_end) of one packed query,
// seeded on the device from its per-position keys (S slots per position), or
// (seeds != null) the explicit seed words of one plain call, one slot per
// word, words [q_start, q_end) of `seeds`.
struct SaBatchUnit {
    uint64_t slot_begin;    // first seed slot of the unit in the flattened slot space
    uint32_t q_start, q_end;// seed positions j (or word indices) in [q_start, q_end)
    const uint32_t* keys;   // per-position seed keys of the unit's query strand
    const uint64_t* seeds;  // explicit seed words (key << 32 | j), or null
    uint32_t unit;          // index into the SaUnit table
    uint32_t pad;
};

// A batched unit resolved to device pointers (library query buffer or a
// serving request's own buffers), or a plain call's seed words on the device.
struct SaResolvedUnit {
    const uint32_t* keys;      // per-position seed keys of this strand
    const uint32_t* q_packed;  // packed strand (forward or reverse complement)
    uint32_t q_len;
    uint32_t start, end;       // seed positions [start, end) (word indices with seeds)
    int32_t rev;
    const uint64_t* seeds = nullptr;  // explicit seed words (device), or null
};

// Seed slots of a resolved unit: S per position, one per explicit word.
inline uint64_t sa_unit_slots(const SaResolvedUnit& u, uint64_t S) {
    return (uint64_t)(u.end - u.start) * (u.seeds ? 1 : S);
}

// Receives the output of one completed device group of a batched run:
// units [u0, u0 + n) of the run's non-empty units, in order, their HSP
// records back to back in recs (cnt[i] each) and their hit counts.  Groups
// arrive in unit order, a group possibly in several consecutive parts.  recs
// is valid only during the call.  expect() announces the records of the
// parts that follow (so that a sink can size its storage once).
struct SaBatchSink {
    virtual ~SaBatchSink() = default;
    virtual int expect(uint64_t records) { (void)records; return 0; }
    virtual int put(uint32_t u0, uint32_t n, const SaRec* recs, const uint32_t* cnt, const uint64_t* hits) = 0;
};

struct SaRunResult {
    // per unit: HSP records (body) and hits; recs stays empty when sink is set
    std::vector<std::vector<SaRec>>* recs;
    std::vector<uint64_t>* hits;
    SaCounters tot;
    double ms_total, ms_lookup, ms_extend_lane, ms_extend_warp, ms_dedup, ms_copy;
    SaBatchSink* sink;  // optional: records go here as groups complete
};

// Runs resolved units on GPU 0's batch workspace (one batch at a time).
int sa_run_units(const SaResolvedUnit* units, uint32_t n, bool want_out, SaRunResult* res);

// Workspace of one slot (one in-flight call).  Sizes are capacities.
struct SaWork {
    // seeds
    uint64_t* seeds;        // [seed_cap]
    uint32_t* s_lo;         // [seed_cap] bucket start per seed
    uint32_t* s_cnt;        // [seed_cap] bucket size per seed
    uint64_t* s_P;          // [seed_cap] inclusive hit prefix per seed
    SaSeedList cs;          // compacted seeds [seed_cap + 1]
    uint64_t seed_cap;
    // per-CTA partials (range-partitioned kernels)
    unsigned long long* cta_a;  // [SA_MAX_CTAS]
    unsigned long long* cta_b;  // [SA_MAX_CTAS]
    // MAX_HITS iteration limits (seed indices) [SA_MAX_ITERS]
    uint64_t* limits;
    // long queue
    SaLongHit* long_q;
    uint64_t long_cap;
    // survivors (ping-pong) and dedup output
    SaRec* rec[2];
    uint32_t* scope[2];
    uint32_t* flags;        // [surv_cap]
    uint64_t surv_cap;
    SaHashSet hset;         // [2 * surv_cap] slots: distinct HSPs of the call; used list aliases rec[1]
    bool hash_clean;        // host: every slot of hset is empty (no full clear needed)
    SaRec* out;             // [surv_cap] deduplicated records (device)
    uint32_t* out_scope;
    uint32_t* scope_count;  // [SA_MAX_SCOPES]
    uint32_t* scope_flags;  // [SA_MAX_SCOPES] bit0 = rev (rm diagonal exclusion)
    // sort state
    unsigned int* sort_hist;      // [SA_SORT_MAX_DIGITS * 256] global histograms
    unsigned int* sort_cta_hist;  // [256 * SA_MAX_CTAS]
    int* sort_in_buf;             // [SA_SORT_MAX_DIGITS + 1] input buffer per pass, final at [D]
    // counters + descriptor
    SaCounters* ctr;
    SaCallDesc* desc;
    // units
    SaUnit* units;          // [SA_MAX_UNITS]
    SaBatchUnit* bunits;    // [SA_MAX_UNITS]
    // batched calls
    unsigned long long* unit_hit_base;  // [SA_MAX_UNITS]
    unsigned long long* unit_hit_end;   // [SA_MAX_UNITS]
    unsigned long long* bounds;         // [SA_MAX_UNITS * SA_BATCH_ITERS]
    uint32_t* unit_iters;               // [SA_MAX_UNITS]
};

#define SA_MAX_CTAS 1024
#define SA_MAX_ITERS 256
#define SA_MAX_SCOPES 65536
#define SA_MAX_UNITS 65536
#define SA_SORT_MAX_DIGITS 20

struct SaTuning {
    int lane_cap;        // bases per direction handled lane-per-hit before a hit moves to the long queue
    int ext_block;       // threads per CTA of the lane-per-hit kernel
    int ext_ctas_per_sm;
    int long_block;      // threads per CTA of the warp-per-hit kernel
    int range_ctas;      // CTAs of the range-partitioned kernels
    int tile_hits;       // hits per warp tile
    int step_bases;      // bases a lane scores per step of the lane-per-hit kernel (8, 16 or 32)
    int substeps;        // steps a lane may take per iteration of the lane-per-hit kernel
    int switch_now;      // 1: a lane whose right side ends starts its left side in the same
                         // iteration (with substeps > 1) instead of at the next one
    int call_range_ctas; // CTAs of the range-partitioned kernels of a plain or rm call (at most
                         // MAX_SEEDS seed words: fewer CTAs than a batch needs)
    int call_lane_ctas;  // CTAs of a plain call's lane kernel; 0: half of the batched
                         // grid, so that concurrent calls' kernels share the SMs and fill
                         // each other's ramp-up and tail instead of queueing
    // a repeat-masker call's lane kernel (its hits are windowed and its calls
    // large): CTAs (0: the batched grid), steps per iteration, switch_now
    int rm_lane_ctas, rm_substeps, rm_switch_now;
};

// ---- sa_pack.cu ----
void sa_launch_pack_text(const char* d_text, uint64_t len, uint32_t* packed, cudaStream_t st);
// out = in reversed (complement: reverse complement); out needs (len + 7) / 8 words.
void sa_launch_reverse_packed(const uint32_t* in, uint64_t len, uint32_t* out, bool complement, cudaStream_t st);
void sa_launch_pad_fill(uint32_t* packed_base, uint64_t nwords_with_pad, cudaStream_t st);
// Table build: keys of target positions, ordered compaction of valid ones.
void sa_launch_table_keys(const uint32_t* ref, uint32_t start, uint64_t num_steps, uint32_t step,
                          const SaParams& p, uint32_t* keys, uint32_t* vals,
                          unsigned long long* cta_a, unsigned long long* cta_b,
                          unsigned long long* d_total, int G, cudaStream_t st);
void sa_launch_table_index(const uint32_t* sorted_keys, const unsigned long long* d_n,
                           uint32_t* index, uint64_t nbuckets, cudaStream_t st);
// Plain (key, value) radix sort by the low `bits` bits of the key.
void sa_launch_sort_kv(uint32_t* keys, uint32_t* vals, uint32_t* keys_tmp, uint32_t* vals_tmp,
                       const unsigned long long* d_n, int bits, unsigned int* cta_hist,
                       int G, cudaStream_t st, int* result_in_tmp);

// ---- sa_lookup.cu ----
void sa_launch_lookup_seeds(SaWork& w, const uint32_t* index, uint32_t nbuckets,
                            const SaParams& p, int G, cudaStream_t st);
void sa_launch_lookup_batch(SaWork& w, const uint32_t* index, uint32_t nbuckets, uint32_t n_bunits,
                            const SaParams& p, int G, cudaStream_t st);

// ---- sa_extend.cu ----
struct SaExtendArgs {
    const uint32_t* ref;
    uint32_t ref_len;
    const uint32_t* pos_table;
    uint32_t seed_size;
    int32_t xdrop, hspthresh, noentropy;
    // 1: units may restrict their hits to a target window (repeat-masker
    // calls); the lane kernel drops the others when it expands a tile
    int32_t windowed = 0;
};
// Phase A (lane per hit) and phase B (warp per long hit); B must follow A.
// grid: CTAs of the persistent launch (0: num_sms x ext_ctas_per_sm).
void sa_launch_extend_lane(SaWork& w, const SaExtendArgs& a, const SaParams& p, const SaTuning& t,
                           int num_sms, cudaStream_t st, int grid = 0);
void sa_launch_extend_warp(SaWork& w, const SaExtendArgs& a, const SaParams& p, const SaTuning& t,
                           int num_sms, cudaStream_t st);

// ---- sa_sort.cu ----
// Sizes the call's HSP set from its hit count (<= 2 * surv_cap slots) and empties it.
// Sizes the call's HSP set (device side, from the hit count); `full` also
// empties every slot.  sa_launch_hash_clear only empties every slot.
void sa_launch_hash_init(SaWork& w, bool full, cudaStream_t st);
void sa_launch_hash_clear(SaWork& w, cudaStream_t st);
// Kernel attributes of the lane kernel, set once per device outside stream capture.
void sa_prepare_extend_lane(const SaParams& p, const SaTuning& t);
// After the host has read a call's counters: whether the HSP set was left empty.
void sa_note_hash_state(SaWork& w, const SaCounters& c);
// mode 0 = plain dedup; 1 = rm (adds diagonal sort/unique and final sort).
// scope_shift: records are counted per (scope >> scope_shift) and flags are
// looked up the same way (0 for single calls, 4 for batches: scope = unit<<4 | iteration).
void sa_launch_dedup(SaWork& w, int mode, int scope_shift, int G, cudaStream_t st);
// ---- sa_pack.cu (batched seeding) ----
void sa_launch_query_keys(const uint32_t* packed, uint64_t len, const SaParams& p, uint32_t* keys, cudaStream_t st);

// Read-only view of the resident state of GPU 0 (sa_api.cu), for entry points
// that live in other files.  Returns SA_OK (0) when target, table and the
// processor are ready.
struct SaResidentView {
    int dev;
    int num_sms;
    const uint32_t* ref;
    uint32_t ref_len;
    const uint32_t* index;
    uint64_t nbuckets;
    const uint32_t* pos;
    const uint32_t* q_packed[2];  // forward, reverse complement of the requested buffer
    uint32_t q_len;
    uint64_t max_seeds;
    uint64_t max_hits;
    uint32_t wga_chunk;           // InitializeProcessor's WGA_CHUNK
    SaParams params;
    SaTuning tuning;
};
int sa_resident_view(uint32_t buffer, SaResidentView* v);

// Grids and lane-kernel settings of one plain (mode 0) or repeat-masker
// (mode 1) call: CTAs of the range-partitioned kernels (lookup, dedup), CTAs of
// the lane kernel, and the tuning the lane kernel runs with.
struct SaCallGrids {
    int range_ctas;
    int lane_ctas;
    SaTuning lane_tuning;
};
SaCallGrids sa_call_grids(const SaTuning& t, int num_sms, int mode);

// Status code (and sa_last_error message) of a device-detected error code
// of SaCounters::error.
int sa_map_device_error(unsigned long long e);

// Counts kernel launches of this library (reported by sa_kernel_launches()).
void sa_note_launch();

// Hand-off of a failed CUDA call to the API layer's error state.
void sa_set_error(int code, const char* fmt, ...);
