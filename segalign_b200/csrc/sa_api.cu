// sa_api.cu — C ABI of the B200 seed-filter path: device registry, resident
// target / table / query buffers, the slot pool and the per-call pipeline.
//
// Reference interfaces (file:line) are cited at each entry point and in
// include/segalign_b200.h.  Differences from the reference: status codes in
// place of exit(); a pool of slots (stream + workspace) per GPU in place of
// one lock per GPU; host pointers in place of the query_DRAM global.
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <shared_mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/segalign_b200.h"
#include "sa_launch.h"
#include "sa_slot_pool.h"

// ---------------------------------------------------------------------------
// Errors
// ---------------------------------------------------------------------------
static thread_local std::string t_err;
// A slot's CUDA-graph capture (shared) against device-wide work from other
// threads (exclusive): cudaDeviceSynchronize, cudaMalloc and cudaFree may not
// run while any stream of the device is capturing, so query and target
// uploads, table builds, key computation and frees wait for captures to end.
static std::shared_mutex g_capture_mu;
static thread_local sa_call_stats t_stats;
static std::atomic<unsigned long long> g_launches{0};
static std::atomic<int> g_timing{0};

void sa_note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
// Generation of everything a captured call graph bakes in (tuning, timing,
// parameters, resident target and table); bumped by every change of them.
static std::atomic<uint64_t> g_graph_gen{1};
static void invalidate_graphs() { g_graph_gen.fetch_add(1); }

void sa_set_error(int, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    t_err = buf;
}

int sa_cuda_fail(cudaError_t e, const char* what, const char* file, int line) {
    sa_set_error(SA_ERR_CUDA, "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
    return e == cudaErrorMemoryAllocation ? SA_ERR_NOMEM : SA_ERR_CUDA;
}

#define SA_TRY(expr)                   \
    do {                               \
        int _r = (expr);               \
        if (_r != SA_OK) return _r;    \
    } while (0)

// ---------------------------------------------------------------------------
// State
// ---------------------------------------------------------------------------
namespace {

constexpr int kMaxBuffers = 8;

struct Packed {
    uint32_t* base = nullptr;  // allocation (with padding)
    uint32_t* data = nullptr;  // word 0
    uint64_t len = 0;
    void release() {
        if (base) cudaFree(base);
        base = data = nullptr;
        len = 0;
    }
};

struct Slot;

struct DevState {
    int dev = 0;
    int num_sms = 148;
    uint64_t total_mem = 0;
    Packed ref, ref_rc;
    uint32_t* index = nullptr;
    uint64_t nbuckets = 0;
    uint32_t* pos = nullptr;
    uint64_t num_index = 0;
    Packed qf[kMaxBuffers], qr[kMaxBuffers];
    uint32_t* qkeys[kMaxBuffers][2] = {};  // per-position seed keys (batched seeding)
    uint64_t qkeys_cap[kMaxBuffers][2] = {};  // bytes allocated for qkeys
    bool qkeys_ok[kMaxBuffers][2] = {};       // qkeys hold the keys of the resident query
    char* stage = nullptr;                 // text staging of uploads (grow-only)
    uint64_t stage_cap = 0;
    std::vector<Slot*> slots;
    Slot* batch = nullptr;                 // workspace of batched calls
};

struct Slot {
    int dev_idx = 0;
    cudaStream_t stream = nullptr;
    SaWork w{};
    void* arena = nullptr;  // one device allocation carved into the workspace
    SaCounters* h_ctr = nullptr;
    SaCallDesc* h_desc = nullptr;
    SaUnit* h_units = nullptr;
    uint32_t* h_scope_flags = nullptr;
    uint32_t* h_scope_count = nullptr;
    SaRec* h_out = nullptr;
    uint64_t h_out_cap = 0;
    cudaEvent_t ev[6] = {};
    cudaEvent_t part_ev[4] = {};  // batched output copied back in parts (created on first use)
    // CUDA graph of the per-call device chain (run_chain), valid for graph_key
    cudaGraphExec_t graph = nullptr;
    uint64_t graph_key = 0;
    uint64_t graph_kernels = 0;
    bool graph_off = false;  // capture failed once: launch directly
    uint32_t max_units = 64;  // units per batched pass (batched kinds)
};

// A queued plain call (call coalescing): its inputs, then its result.
struct CallReq {
    const uint64_t* seeds = nullptr;  // the caller's words, copied to `staged` before queueing
    uint64_t* staged = nullptr;       // pinned copy of the words
    uint32_t n = 0;
    int rev = 0;
    uint32_t buffer = 0;
    bool taken = false, done = false;  // taken into a pass; result ready (both under Global::mu)
    int status = SA_OK;
    std::string err;
    sa_segment* out = nullptr;
    uint64_t out_len = 0;
    sa_call_stats stats{};
};

// Phase timing with CUDA events on the slot stream (enabled by sa_set_timing).
struct PhaseTimer {
    Slot* s;
    bool on;
    PhaseTimer(Slot* slot) : s(slot), on(g_timing.load() != 0) {}
    void mark(int i) {
        if (on) cudaEventRecord(s->ev[i], s->stream);
    }
    // after the stream is synchronized
    void collect(sa_call_stats& st) {
        if (!on) return;
        float a = 0, b = 0, b2 = 0, c = 0, d = 0;
        cudaEventElapsedTime(&a, s->ev[0], s->ev[1]);
        cudaEventElapsedTime(&b, s->ev[1], s->ev[2]);
        cudaEventElapsedTime(&b2, s->ev[2], s->ev[3]);
        cudaEventElapsedTime(&c, s->ev[3], s->ev[4]);
        cudaEventElapsedTime(&d, s->ev[4], s->ev[5]);
        st.ms_lookup += a;
        st.ms_extend_lane += b;
        st.ms_extend_warp += b2;
        st.ms_dedup += c;
        st.ms_copy += d;
        st.ms_total += a + b + b2 + c + d;
    }
};

struct Global {
    std::mutex mu;
    std::mutex batch_mu;  // one batched call at a time
    std::condition_variable cv;
    std::deque<Slot*> free_slots;
    std::vector<DevState> devs;
    bool interface_ready = false;
    bool processor_ready = false;
    // shape (common/ntcoding.cpp globals)
    SaParams params{};
    bool shape_set = false;
    // processor configuration
    uint32_t wga_chunk = 250000;
    uint64_t max_seeds = 0;
    uint64_t max_hits_override = 0;
    uint64_t max_hits_default = 0;
    int rm_exclude_diag = 0;
    SaTuning tuning{8192, 256, 3, 256, 592, 160, 32, 3, 1, 148, 0, 0, 2, 0};  // autotuned on the genome-scale batch
    // last target upload (to reuse it for the table build)
    const char* last_ref_ptr = nullptr;
    size_t last_ref_start = 0;
    uint32_t last_ref_len = 0;
    uint32_t ref_len = 0;
    uint64_t surv_cap = 0;
    uint64_t long_cap = 0;
    uint64_t batch_slot_cap = 0;
    uint64_t batch_surv_cap = 0;
    // call coalescing: calls per pass (0 = every call runs alone), queued calls,
    // and pinned staging buffers of max_seeds words for the callers' seeds
    uint32_t coalesce_calls = 0;
    std::deque<CallReq*> pending;
    std::mutex pinned_mu;
    std::vector<uint64_t*> pinned_free, pinned_all;
};

Global& G() {
    static Global g;
    return g;
}

uint64_t env_u64(const char* name, uint64_t dflt) {
    const char* v = getenv(name);
    if (!v || !*v) return dflt;
    return strtoull(v, nullptr, 10);
}

// Default 12of19 shape (src/main.cpp:153-156).
void set_shape_positions(SaParams& p, const std::string& shape) {
    int k = 0;
    for (size_t i = 0; i < shape.size(); ++i)
        if (shape[i] == '1' || shape[i] == 'T') p.shape_pos[k++] = (int)i;
    p.kmer_size = k;
    p.seed_size = (int)shape.size();
}

// Allocates a packed sequence of len bases followed by its reversed copy
// (sa_rev_words), all words E-filled.
// A packed sequence of the same word count reuses its allocation (a new
// query block of the same size is written in place); the device is first
// synchronized, as cudaFree would, so no earlier work still reads it.
int alloc_packed(Packed& pk, uint64_t len) {
    const uint64_t nw = sa_rev_words(len);
    if (pk.base && sa_rev_words(pk.len) == nw) {
        SA_CUDA_OK(cudaDeviceSynchronize());
        pk.len = len;
        sa_launch_pad_fill(pk.base, 2 * nw, 0);
        return SA_OK;
    }
    pk.release();
    SA_CUDA_OK(cudaMalloc(&pk.base, 2 * nw * sizeof(uint32_t)));
    pk.data = pk.base + SA_PADW;
    pk.len = len;
    sa_launch_pad_fill(pk.base, 2 * nw, 0);
    return SA_OK;
}

// Writes the reversed copy of pk once its forward words are in place.
void finish_packed(Packed& pk) { sa_launch_reverse_packed(pk.data, pk.len, pk.data + sa_rev_words(pk.len), false, 0); }

// rc = reverse complement of pk (both allocated by alloc_packed), with its reversed copy.
void make_rc_packed(const Packed& pk, Packed& rc) {
    sa_launch_reverse_packed(pk.data, pk.len, rc.data, true, 0);
    finish_packed(rc);
}

// Uploads text[0, len) and packs it into pk (and its reverse complement into rc if given).
int upload_pack(DevState& d, const char* text, uint64_t len, Packed& pk, Packed* rc) {
    std::unique_lock<std::shared_mutex> dev_wide(g_capture_mu);
    SA_CUDA_OK(cudaSetDevice(d.dev));
    SA_TRY(alloc_packed(pk, len));
    if (rc) SA_TRY(alloc_packed(*rc, len));
    const uint64_t chunk = 1ull << 28;  // 256 MiB text per round
    const uint64_t need = std::min<uint64_t>(len ? len : 1, chunk) + 16;
    if (d.stage_cap < need) {
        if (d.stage) cudaFree(d.stage);
        d.stage = nullptr;
        d.stage_cap = 0;
        SA_CUDA_OK(cudaMalloc(&d.stage, need));
        d.stage_cap = need;
    }
    char* d_text = d.stage;
    for (uint64_t off = 0; off < len; off += chunk) {
        uint64_t n = std::min(chunk, len - off);
        cudaError_t e = cudaMemcpy(d_text, text + off, n, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return sa_cuda_fail(e, "cudaMemcpy(text)", __FILE__, __LINE__);
        // chunk is a multiple of 8 bases, so word boundaries line up
        sa_launch_pack_text(d_text, n, pk.data + off / 8, 0);
    }
    finish_packed(pk);
    if (rc) make_rc_packed(pk, *rc);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return sa_cuda_fail(e, "pack", __FILE__, __LINE__);
    return SA_OK;
}

void free_slot(Slot* s) {
    if (!s) return;
    cudaSetDevice(s->dev_idx >= 0 ? G().devs[s->dev_idx].dev : 0);
    if (s->graph) cudaGraphExecDestroy(s->graph);
    if (s->arena) cudaFree(s->arena);
    if (s->stream) cudaStreamDestroy(s->stream);
    if (s->h_ctr) cudaFreeHost(s->h_ctr);
    if (s->h_desc) cudaFreeHost(s->h_desc);
    if (s->h_units) cudaFreeHost(s->h_units);
    if (s->h_scope_flags) cudaFreeHost(s->h_scope_flags);
    if (s->h_scope_count) cudaFreeHost(s->h_scope_count);
    if (s->h_out) cudaFreeHost(s->h_out);
    for (auto& e : s->ev)
        if (e) cudaEventDestroy(e);
    for (auto& e : s->part_ev)
        if (e) cudaEventDestroy(e);
    delete s;
}

// Carves one slot workspace out of a single device allocation.
// Workspace kinds: plain calls (host seed words), batched passes (device
// seeding over query windows), or both (passes of coalesced plain calls, and
// plain calls one at a time), with at most `units` units per pass.
enum SlotKind { kSlotPlain = 0, kSlotBatch = 1, kSlotBoth = 2 };

int make_slot(int dev_idx, uint64_t seed_cap, uint64_t surv_cap, uint64_t long_cap, Slot** out,
              SlotKind kind = kSlotPlain, uint64_t units = SA_MAX_UNITS) {
    const bool batch = kind != kSlotPlain, host_seeds = kind != kSlotBatch;
    DevState& d = G().devs[dev_idx];
    SA_CUDA_OK(cudaSetDevice(d.dev));
    Slot* s = new Slot();
    s->dev_idx = dev_idx;
    struct Part {
        void** ptr;
        uint64_t bytes;
    };
    SaWork& w = s->w;
    w.seed_cap = seed_cap;
    w.surv_cap = surv_cap;
    w.long_cap = long_cap;
    const uint64_t nunits = batch ? std::max<uint64_t>(64, std::min<uint64_t>(units, SA_MAX_UNITS)) : 64;
    s->max_units = (uint32_t)nunits;
    std::vector<Part> parts = {
        {(void**)&w.seeds, host_seeds ? 8 * seed_cap : 0},
        {(void**)&w.s_lo, 4 * seed_cap},
        {(void**)&w.s_cnt, 4 * seed_cap},
        {(void**)&w.s_P, host_seeds ? 8 * seed_cap : 0},
        {(void**)&w.cs.E, 8 * (seed_cap + 1)},
        {(void**)&w.cs.lo, 4 * (seed_cap + 1)},
        {(void**)&w.cs.qpos, 4 * (seed_cap + 1)},
        {(void**)&w.cs.scope, 4 * (seed_cap + 1)},
        {(void**)&w.cs.unit, 4 * (seed_cap + 1)},
        {(void**)&w.cta_a, 8 * SA_MAX_CTAS},
        {(void**)&w.cta_b, 8 * SA_MAX_CTAS},
        {(void**)&w.limits, 8 * SA_MAX_ITERS},
        {(void**)&w.long_q, sizeof(SaLongHit) * long_cap},
        {(void**)&w.rec[0], sizeof(SaRec) * surv_cap},
        {(void**)&w.rec[1], sizeof(SaRec) * surv_cap},
        {(void**)&w.scope[0], 4 * surv_cap},
        {(void**)&w.scope[1], 4 * surv_cap},
        {(void**)&w.hset.keys, 16 * 2 * surv_cap},
        {(void**)&w.hset.score, 4 * 2 * surv_cap},
        {(void**)&w.out, sizeof(SaRec) * surv_cap},
        {(void**)&w.out_scope, 4 * surv_cap},
        {(void**)&w.scope_count, 4 * SA_MAX_SCOPES},
        {(void**)&w.scope_flags, 4 * SA_MAX_SCOPES},
        {(void**)&w.sort_hist, 4 * 256 * SA_SORT_MAX_DIGITS},
        {(void**)&w.sort_cta_hist, 4 * 256 * (uint64_t)SA_MAX_CTAS + 4 * 64},
        {(void**)&w.sort_in_buf, 4 * (SA_SORT_MAX_DIGITS + 2)},
        {(void**)&w.ctr, sizeof(SaCounters)},
        {(void**)&w.desc, sizeof(SaCallDesc)},
        {(void**)&w.units, sizeof(SaUnit) * nunits},
        {(void**)&w.bunits, batch ? sizeof(SaBatchUnit) * nunits : 0},
        {(void**)&w.unit_hit_base, batch ? 8 * nunits : 0},
        {(void**)&w.unit_hit_end, batch ? 8 * nunits : 0},
        {(void**)&w.bounds, batch ? 8 * nunits * SA_BATCH_ITERS : 0},
        {(void**)&w.unit_iters, batch ? 4 * nunits : 0},
    };
    w.flags = nullptr;
    uint64_t total = 0;
    for (auto& p : parts) total += (p.bytes + 255) & ~255ull;
    cudaError_t e = cudaMalloc(&s->arena, total);
    if (e != cudaSuccess) {
        delete s;
        return sa_cuda_fail(e, "cudaMalloc(slot workspace)", __FILE__, __LINE__);
    }
    char* at = (char*)s->arena;
    for (auto& p : parts) {
        *p.ptr = at;
        at += (p.bytes + 255) & ~255ull;
    }
    // the HSP set's list of claimed slots lives in rec[1], free until the sort
    w.hset.used = reinterpret_cast<unsigned long long*>(w.rec[1]);
    w.hset.used_cap = surv_cap;
    w.hash_clean = false;
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMallocHost(&s->h_ctr, sizeof(SaCounters)) != cudaSuccess ||
        cudaMallocHost(&s->h_desc, sizeof(SaCallDesc)) != cudaSuccess ||
        cudaMallocHost(&s->h_units, sizeof(SaUnit) * nunits) != cudaSuccess ||
        cudaMallocHost(&s->h_scope_flags, 4 * SA_MAX_ITERS) != cudaSuccess ||
        cudaMallocHost(&s->h_scope_count, 4 * SA_MAX_ITERS) != cudaSuccess ||
        cudaEventCreate(&s->ev[0]) != cudaSuccess || cudaEventCreate(&s->ev[1]) != cudaSuccess ||
        cudaEventCreate(&s->ev[2]) != cudaSuccess || cudaEventCreate(&s->ev[3]) != cudaSuccess ||
        cudaEventCreate(&s->ev[4]) != cudaSuccess || cudaEventCreate(&s->ev[5]) != cudaSuccess) {
        free_slot(s);
        sa_set_error(SA_ERR_NOMEM, "pinned host allocation failed");
        return SA_ERR_NOMEM;
    }
    *out = s;
    return SA_OK;
}

// Takes a free slot (g.mu held): the first one of the device with the most
// free slots (sa_slot_pool.h).
Slot* take_free_slot_locked() {
    Global& g = G();
    std::vector<int> dev(g.free_slots.size());
    for (size_t i = 0; i < dev.size(); ++i) dev[i] = g.free_slots[i]->dev_idx;
    const size_t k = sa_pick_free_slot(dev, (int)g.devs.size());
    Slot* s = g.free_slots[k];
    g.free_slots.erase(g.free_slots.begin() + (std::ptrdiff_t)k);
    return s;
}

Slot* acquire_slot() {
    Global& g = G();
    std::unique_lock<std::mutex> lk(g.mu);
    g.cv.wait(lk, [&] { return !g.free_slots.empty(); });
    return take_free_slot_locked();
}

void release_slot(Slot* s) {
    Global& g = G();
    {
        std::lock_guard<std::mutex> lk(g.mu);
        g.free_slots.push_back(s);
    }
    g.cv.notify_all();  // waiters for a slot and coalesced callers share the condition
}

int map_device_error(unsigned long long e) { return sa_map_device_error(e); }

uint64_t max_hits_now();

}  // namespace

int sa_map_device_error(unsigned long long e) {
    switch (e) {
        case 0: return SA_OK;
        case 1: sa_set_error(SA_ERR_BAD_SEED, "seed key outside the 4^K seed table"); return SA_ERR_BAD_SEED;
        case 2: sa_set_error(SA_ERR_MAX_HITS, "a single seed has at least MAX_HITS hits"); return SA_ERR_MAX_HITS;
        case 3: sa_set_error(SA_ERR_MAX_HITS, "more than %d MAX_HITS iterations", SA_MAX_ITERS); return SA_ERR_MAX_HITS;
        case 4: sa_set_error(SA_ERR_CAPACITY, "survivor workspace exceeded (raise SA_SURV_CAP)"); return SA_ERR_CAPACITY;
        case 5: sa_set_error(SA_ERR_BAD_SEED, "hit coordinates past the end of the target or query"); return SA_ERR_BAD_SEED;
        default: sa_set_error(SA_ERR_CUDA, "device error %llu", e); return SA_ERR_CUDA;
    }
}

SaCallGrids sa_call_grids(const SaTuning& t, int num_sms, int mode) {
    SaCallGrids c;
    c.range_ctas = std::min(t.call_range_ctas, SA_MAX_CTAS);
    c.lane_tuning = t;
    c.lane_ctas = t.call_lane_ctas > 0 ? t.call_lane_ctas : std::max(1, num_sms * t.ext_ctas_per_sm / 2);
    if (mode == 1) {  // repeat-masker call
        c.lane_tuning.substeps = t.rm_substeps;
        c.lane_tuning.switch_now = t.rm_switch_now;
        c.lane_ctas = t.rm_lane_ctas > 0 ? t.rm_lane_ctas : num_sms * t.ext_ctas_per_sm;
    }
    return c;
}

namespace {

uint64_t max_hits_now() {
    Global& g = G();
    return g.max_hits_override ? g.max_hits_override : g.max_hits_default;
}

// One SeedAndFilter call on a slot: seeds -> hits -> X-drop -> dedup -> host.
// mode 0 = plain, 1 = repeat masker.
// Device work of one plain (mode 0) or rm (mode 1) call once its seed words
// are on the device: descriptor uploads from the slot's pinned buffers,
// counters reset, lookup, extension, dedup and the counters' copy back.
// Every size is read on the device, so one capture serves every call.
int launch_call_chain(Slot* s, int mode, PhaseTimer& tm) {
    Global& g = G();
    DevState& d = g.devs[s->dev_idx];
    SaWork& w = s->w;
    cudaStream_t st = s->stream;
    const SaCallGrids cg = sa_call_grids(g.tuning, d.num_sms, mode);
    const int Gr = cg.range_ctas;
    SA_CUDA_OK(cudaMemcpyAsync(w.desc, s->h_desc, sizeof(SaCallDesc), cudaMemcpyHostToDevice, st));
    SA_CUDA_OK(cudaMemcpyAsync(w.units, s->h_units, sizeof(SaUnit), cudaMemcpyHostToDevice, st));
    SA_CUDA_OK(cudaMemcpyAsync(w.scope_flags, s->h_scope_flags, 4 * SA_MAX_ITERS, cudaMemcpyHostToDevice, st));
    SA_CUDA_OK(cudaMemsetAsync(w.ctr, 0, sizeof(SaCounters), st));
    sa_launch_lookup_seeds(w, d.index, (uint32_t)d.nbuckets, g.params, Gr, st);
    sa_launch_hash_init(w, false, st);
    tm.mark(1);
    SaExtendArgs xa;
    xa.ref = d.ref.data;
    xa.ref_len = (uint32_t)d.ref.len;
    xa.pos_table = d.pos;
    xa.seed_size = (uint32_t)g.params.seed_size;
    xa.xdrop = g.params.xdrop;
    xa.hspthresh = g.params.hspthresh;
    xa.noentropy = g.params.noentropy;
    xa.windowed = mode == 1 ? 1 : 0;
    sa_launch_extend_lane(w, xa, g.params, cg.lane_tuning, d.num_sms, st, cg.lane_ctas);
    tm.mark(2);
    sa_launch_extend_warp(w, xa, g.params, g.tuning, d.num_sms, st);
    tm.mark(3);
    sa_launch_dedup(w, mode, 0, Gr, st);
    tm.mark(4);
    SA_CUDA_OK(cudaGetLastError());
    SA_CUDA_OK(cudaMemcpyAsync(s->h_ctr, w.ctr, sizeof(SaCounters), cudaMemcpyDeviceToHost, st));
    return SA_OK;
}

bool graphs_enabled() {
    static const bool on = env_u64("SA_GRAPHS", 1) != 0;
    return on;
}

// Runs the call chain: replays the slot's CUDA graph, capturing it first when
// the chain changed (mode, or anything invalidate_graphs covers).
int run_chain(Slot* s, int mode, PhaseTimer& tm) {
    // phase timing (a diagnostic mode) records events between the kernels: direct launches
    if (!graphs_enabled() || s->graph_off || tm.on) return launch_call_chain(s, mode, tm);
    Global& g = G();
    cudaStream_t st = s->stream;
    const uint64_t key = (g_graph_gen.load() << 1) | (uint64_t)mode;
    if (!s->graph || s->graph_key != key) {
        if (s->graph) cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
        sa_prepare_extend_lane(g.params, g.tuning);  // kernel attributes are not set during capture
        const unsigned long long l0 = g_launches.load();
        std::shared_lock<std::shared_mutex> capturing(g_capture_mu);
        SA_CUDA_OK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        const int r = launch_call_chain(s, mode, tm);
        cudaGraph_t graph = nullptr;
        const cudaError_t e = cudaStreamEndCapture(st, &graph);
        const unsigned long long captured = g_launches.load() - l0;
        g_launches.fetch_sub(captured);  // counted again at each replay
        cudaError_t ei = cudaErrorUnknown;
        if (r == SA_OK && e == cudaSuccess && graph) ei = cudaGraphInstantiate(&s->graph, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (ei != cudaSuccess) {
            // capture not possible here: direct launches from now on
            s->graph = nullptr;
            s->graph_off = true;
            cudaGetLastError();
            return launch_call_chain(s, mode, tm);
        }
        s->graph_key = key;
        s->graph_kernels = captured;
    }
    SA_CUDA_OK(cudaGraphLaunch(s->graph, st));
    g_launches.fetch_add(s->graph_kernels);
    return SA_OK;
}

// One SeedAndFilter call on a slot: seeds -> hits -> X-drop -> dedup -> host.
// mode 0 = plain, 1 = repeat masker.
int run_call(Slot* s, const uint64_t* seeds, uint32_t n, int rev, const Packed& q, int mode, uint32_t rm_lo,
             uint32_t rm_hi, sa_segment** out, uint64_t* out_len) {
    Global& g = G();
    DevState& d = g.devs[s->dev_idx];
    SaWork& w = s->w;
    cudaStream_t st = s->stream;
    SA_CUDA_OK(cudaSetDevice(d.dev));
    // descriptor, unit, scope flags
    SaCallDesc* hd = s->h_desc;
    hd->num_seeds = n;
    hd->max_hits = max_hits_now();
    hd->num_units = 1;
    hd->num_scopes_max = SA_MAX_ITERS;
    hd->rm_exclude_diag = (uint32_t)g.rm_exclude_diag;
    SaUnit* u = s->h_units;
    u[0].q_packed = q.data;
    u[0].q_len = (uint32_t)q.len;
    u[0].rm_lo = rm_lo;
    u[0].rm_hi = rm_hi;
    u[0].flags = mode == 1 ? (1u | (rev ? 2u : 0u)) : 0u;
    for (int i = 0; i < SA_MAX_ITERS; ++i)
        s->h_scope_flags[i] = (rev ? 1u : 0u) | ((mode == 1 && g.rm_exclude_diag) ? 2u : 0u);
    PhaseTimer tm(s);
    tm.mark(0);
    SA_CUDA_OK(cudaMemcpyAsync(w.seeds, seeds, 8ull * n, cudaMemcpyHostToDevice, st));
    if (!w.hash_clean) sa_launch_hash_clear(w, st);
    w.hash_clean = false;  // until this call is seen to complete
    SA_TRY(run_chain(s, mode, tm));
    SA_CUDA_OK(cudaStreamSynchronize(st));
    SaCounters c = *s->h_ctr;
    sa_note_hash_state(w, c);
    std::memset(&t_stats, 0, sizeof t_stats);
    t_stats.num_seeds = n;
    t_stats.num_hits = c.num_hits;
    t_stats.hits_extended = c.extended;
    t_stats.seeds_with_hits = c.nnz;
    t_stats.survivors = c.surv_count;
    t_stats.num_hsps = c.uniq_count;
    t_stats.long_hits = c.long_count;
    t_stats.tiles = c.base_steps;
    t_stats.num_iter = (uint32_t)c.num_iter;
    t_stats.batch_calls = 1;
    if (c.error) return map_device_error(c.error);
    const uint64_t nh = c.uniq_count;
    if (nh + 1 > s->h_out_cap) {
        if (s->h_out) cudaFreeHost(s->h_out);
        s->h_out = nullptr;
        uint64_t cap = std::max<uint64_t>(nh + 1, 1 << 16);
        cap = std::max(cap, s->h_out_cap * 2);
        SA_CUDA_OK(cudaMallocHost(&s->h_out, cap * sizeof(SaRec)));
        s->h_out_cap = cap;
    }
    if (nh) SA_CUDA_OK(cudaMemcpyAsync(s->h_out + 1, w.out, nh * sizeof(SaRec), cudaMemcpyDeviceToHost, st));
    tm.mark(5);
    SA_CUDA_OK(cudaStreamSynchronize(st));
    tm.collect(t_stats);
    // header (src/seed_filter.cu:756-759): len = total anchors, score = num_hits
    s->h_out[0].ref_start = 0;
    s->h_out[0].query_start = 0;
    s->h_out[0].len = (uint32_t)nh;
    s->h_out[0].score = (int32_t)(uint32_t)c.num_hits;
    sa_segment* res = (sa_segment*)malloc((nh + 1) * sizeof(sa_segment));
    if (!res) {
        sa_set_error(SA_ERR_NOMEM, "host allocation of %llu records failed", (unsigned long long)(nh + 1));
        return SA_ERR_NOMEM;
    }
    std::memcpy(res, s->h_out, (nh + 1) * sizeof(sa_segment));
    *out = res;
    *out_len = nh + 1;
    return SA_OK;
}

int check_ready(bool need_query) {
    Global& g = G();
    if (!g.interface_ready) {
        sa_set_error(SA_ERR_STATE, "sa_initialize_interface() has not been called");
        return SA_ERR_STATE;
    }
    if (!g.processor_ready) {
        sa_set_error(SA_ERR_STATE, "sa_initialize_processor() has not been called");
        return SA_ERR_STATE;
    }
    for (auto& d : g.devs) {
        if (!d.ref.data || !d.index || !d.pos) {
            sa_set_error(SA_ERR_STATE, "no resident target and seed table");
            return SA_ERR_STATE;
        }
    }
    (void)need_query;
    return SA_OK;
}


// ---------------------------------------------------------------------------
// Batched calls: many (query window, strand) units in one launch sequence,
// seeded on the device from the resident query.  Each unit's output equals
// what sa_seed_and_filter() returns for the seed words the host seeder would
// build for that window (src/seeder.cpp:57-74).
// ---------------------------------------------------------------------------
int ensure_keys(DevState& d, uint32_t buffer, int rev) {
    Global& g = G();
    if (d.qkeys[buffer][rev] && d.qkeys_ok[buffer][rev]) return SA_OK;
    std::unique_lock<std::shared_mutex> dev_wide(g_capture_mu);
    const Packed& q = rev ? d.qr[buffer] : d.qf[buffer];
    if (!q.data) {
        sa_set_error(SA_ERR_STATE, "query buffer %u is not resident", buffer);
        return SA_ERR_STATE;
    }
    SA_CUDA_OK(cudaSetDevice(d.dev));
    const uint64_t need = 4 * (q.len ? q.len : 1);
    if (d.qkeys_cap[buffer][rev] < need) {  // a new query of the same size reuses the array
        if (d.qkeys[buffer][rev]) cudaFree(d.qkeys[buffer][rev]);
        d.qkeys[buffer][rev] = nullptr;
        d.qkeys_cap[buffer][rev] = 0;
        SA_CUDA_OK(cudaMalloc(&d.qkeys[buffer][rev], need));
        d.qkeys_cap[buffer][rev] = need;
    }
    sa_launch_query_keys(q.data, q.len, g.params, d.qkeys[buffer][rev], 0);
    SA_CUDA_OK(cudaDeviceSynchronize());
    d.qkeys_ok[buffer][rev] = true;
    return SA_OK;
}

// Keys of a buffer whose query is rewritten: recomputed on next use, in place.
void invalidate_keys(DevState& d, uint32_t buffer) {
    for (int r = 0; r < 2; ++r) d.qkeys_ok[buffer][r] = false;
}

void drop_keys(DevState& d, uint32_t buffer) {
    for (int r = 0; r < 2; ++r) {
        if (d.qkeys[buffer][r]) {
            cudaFree(d.qkeys[buffer][r]);
            d.qkeys[buffer][r] = nullptr;
        }
        d.qkeys_cap[buffer][r] = 0;
        d.qkeys_ok[buffer][r] = false;
    }
}

struct BatchResult {
    std::vector<std::vector<SaRec>> recs;  // per unit (body only), unless sink is set
    std::vector<uint64_t> hits;            // per unit
    std::vector<uint32_t> iters;           // per unit: MAX_HITS iterations
    SaCounters tot{};
    sa_call_stats timing{};
    SaBatchSink* sink = nullptr;  // records go here instead of recs
};

// Runs units [u0, u1) in one device pass.  Returns SA_ERR_CAPACITY when the
// survivors do not fit (the caller splits the range).
int run_batch_group(DevState& d, Slot* s, const SaResolvedUnit* units, uint32_t u0, uint32_t u1, bool want_out,
                    BatchResult& res) {
    Global& g = G();
    SaWork& w = s->w;
    cudaStream_t st = s->stream;
    SA_CUDA_OK(cudaSetDevice(d.dev));
    const int S = g.params.transition ? 1 + g.params.kmer_size : 1;
    const uint32_t n = u1 - u0;
    std::vector<SaBatchUnit> bu(n);
    SaUnit* hu = s->h_units;
    uint64_t slots = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const SaResolvedUnit& u = units[u0 + i];
        bu[i].slot_begin = slots;
        bu[i].q_start = u.start;
        bu[i].q_end = u.end;
        bu[i].keys = u.keys;
        bu[i].seeds = u.seeds;
        bu[i].unit = i;
        bu[i].pad = 0;
        hu[i].q_packed = u.q_packed;
        hu[i].q_len = u.q_len;
        hu[i].rm_lo = hu[i].rm_hi = 0;
        hu[i].flags = 0;
        slots += sa_unit_slots(u, S);
    }
    SaCallDesc* hd = s->h_desc;
    hd->num_seeds = slots;
    hd->max_hits = max_hits_now();
    hd->num_units = n;
    hd->num_scopes_max = n;
    hd->rm_exclude_diag = 0;
    const int Gr = std::min(g.tuning.range_ctas, SA_MAX_CTAS);
    PhaseTimer tm(s);
    tm.mark(0);
    SA_CUDA_OK(cudaMemcpyAsync(w.bunits, bu.data(), sizeof(SaBatchUnit) * n, cudaMemcpyHostToDevice, st));
    SA_CUDA_OK(cudaMemcpyAsync(w.units, hu, sizeof(SaUnit) * n, cudaMemcpyHostToDevice, st));
    SA_CUDA_OK(cudaMemcpyAsync(w.desc, hd, sizeof(SaCallDesc), cudaMemcpyHostToDevice, st));
    SA_CUDA_OK(cudaMemsetAsync(w.scope_flags, 0, 4 * n, st));
    SA_CUDA_OK(cudaMemsetAsync(w.ctr, 0, sizeof(SaCounters), st));
    sa_launch_lookup_batch(w, d.index, (uint32_t)d.nbuckets, n, g.params, Gr, st);
    if (!w.hash_clean) sa_launch_hash_clear(w, st);
    w.hash_clean = false;  // until this group is seen to complete
    sa_launch_hash_init(w, false, st);
    tm.mark(1);
    SaExtendArgs xa;
    xa.ref = d.ref.data;
    xa.ref_len = (uint32_t)d.ref.len;
    xa.pos_table = d.pos;
    xa.seed_size = (uint32_t)g.params.seed_size;
    xa.xdrop = g.params.xdrop;
    xa.hspthresh = g.params.hspthresh;
    xa.noentropy = g.params.noentropy;
    sa_launch_extend_lane(w, xa, g.params, g.tuning, d.num_sms, st);
    tm.mark(2);
    sa_launch_extend_warp(w, xa, g.params, g.tuning, d.num_sms, st);
    tm.mark(3);
    sa_launch_dedup(w, 0, 4, Gr, st);
    tm.mark(4);
    SA_CUDA_OK(cudaGetLastError());
    SA_CUDA_OK(cudaMemcpyAsync(s->h_ctr, w.ctr, sizeof(SaCounters), cudaMemcpyDeviceToHost, st));
    SA_CUDA_OK(cudaStreamSynchronize(st));
    SaCounters c = *s->h_ctr;
    sa_note_hash_state(w, c);
    if (c.hash_overflow || c.error == 4) return SA_ERR_CAPACITY;
    if (c.error) return map_device_error(c.error);
    res.tot.num_hits += c.num_hits;
    res.tot.extended += c.extended;
    res.tot.nnz += c.nnz;
    res.tot.surv_count += c.surv_count;
    res.tot.uniq_count += c.uniq_count;
    res.tot.long_count += c.long_count;
    res.tot.base_steps += c.base_steps;
    std::vector<unsigned long long> hb(n), he(n);
    std::vector<uint32_t> cnt(n);
    if (res.iters.size() >= u1)
        SA_CUDA_OK(cudaMemcpyAsync(res.iters.data() + u0, w.unit_iters, 4ull * n, cudaMemcpyDeviceToHost, st));
    SA_CUDA_OK(cudaMemcpyAsync(hb.data(), w.unit_hit_base, 8ull * n, cudaMemcpyDeviceToHost, st));
    SA_CUDA_OK(cudaMemcpyAsync(he.data(), w.unit_hit_end, 8ull * n, cudaMemcpyDeviceToHost, st));
    SA_CUDA_OK(cudaMemcpyAsync(cnt.data(), w.scope_count, 4ull * n, cudaMemcpyDeviceToHost, st));
    const uint64_t nh = c.uniq_count;
    if (want_out && nh + 1 > s->h_out_cap) {
        SA_CUDA_OK(cudaStreamSynchronize(st));
        if (s->h_out) cudaFreeHost(s->h_out);
        s->h_out = nullptr;
        uint64_t cap = std::max<uint64_t>(nh + 1, std::max<uint64_t>(1 << 16, s->h_out_cap * 2));
        SA_CUDA_OK(cudaMallocHost(&s->h_out, cap * sizeof(SaRec)));
        s->h_out_cap = cap;
    }
    // A large output for a sink comes back in parts of whole units; the sink
    // copies part k while part k + 1 is in flight.
    // (SA_OUT_PARTS_MIN: the smallest output, in records, copied in parts)
    constexpr int kParts = 4;
    static const uint64_t parts_min = env_u64("SA_OUT_PARTS_MIN", 1ull << 20);
    const bool parts = want_out && res.sink && nh >= std::max<uint64_t>(parts_min, 1);
    if (parts) {
        SA_CUDA_OK(cudaStreamSynchronize(st));  // the per-unit counts split the records
        for (auto& e : s->part_ev)
            if (!e) SA_CUDA_OK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    uint32_t part_u[kParts + 1] = {0};
    uint64_t part_r[kParts + 1] = {0};
    if (parts) {
        uint32_t u = 0;
        uint64_t r = 0;
        for (int k = 0; k < kParts; ++k) {
            const uint64_t goal = nh * (uint64_t)(k + 1) / kParts;
            while (u < n && (r < goal || k + 1 == kParts)) r += cnt[u++];
            part_u[k + 1] = u;
            part_r[k + 1] = r;
            if (r > part_r[k])
                SA_CUDA_OK(cudaMemcpyAsync(s->h_out + part_r[k], w.out + part_r[k], (r - part_r[k]) * sizeof(SaRec),
                                           cudaMemcpyDeviceToHost, st));
            SA_CUDA_OK(cudaEventRecord(s->part_ev[k], st));
        }
    } else if (want_out && nh) {
        SA_CUDA_OK(cudaMemcpyAsync(s->h_out, w.out, nh * sizeof(SaRec), cudaMemcpyDeviceToHost, st));
    }
    tm.mark(5);
    for (uint32_t i = 0; i < n; ++i) res.hits[u0 + i] = he[i] - hb[i];
    if (parts) {
        if (const int r = res.sink->expect(nh); r != SA_OK) {
            cudaStreamSynchronize(st);
            return r;
        }
        for (int k = 0; k < kParts; ++k) {
            SA_CUDA_OK(cudaEventSynchronize(s->part_ev[k]));
            const uint32_t a = part_u[k], b = part_u[k + 1];
            const int r = b > a ? res.sink->put(u0 + a, b - a, s->h_out + part_r[k], cnt.data() + a,
                                                 res.hits.data() + u0 + a)
                                : SA_OK;
            if (r != SA_OK) {
                cudaStreamSynchronize(st);  // no copy into h_out outlives the call
                return r;
            }
        }
        SA_CUDA_OK(cudaStreamSynchronize(st));
        tm.collect(res.timing);
        return SA_OK;
    }
    SA_CUDA_OK(cudaStreamSynchronize(st));
    tm.collect(res.timing);
    if (want_out && res.sink) return res.sink->put(u0, n, s->h_out, cnt.data(), res.hits.data() + u0);
    uint64_t at = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (want_out) res.recs[u0 + i].assign(s->h_out + at, s->h_out + at + cnt[i]);
        at += cnt[i];
    }
    return SA_OK;
}

int run_batch_range(DevState& d, Slot* s, const SaResolvedUnit* units, uint32_t u0, uint32_t u1, bool want_out,
                    BatchResult& res) {
    Global& g = G();
    const uint64_t S = g.params.transition ? 1 + g.params.kmer_size : 1;
    // split by seed-slot capacity and unit count
    uint32_t a = u0;
    while (a < u1) {
        uint32_t b = a;
        uint64_t slots = 0;
        while (b < u1 && b - a < SA_MAX_UNITS) {
            uint64_t add = sa_unit_slots(units[b], S);
            if (b > a && slots + add > s->w.seed_cap) break;
            if (add > s->w.seed_cap) {
                sa_set_error(SA_ERR_CAPACITY, "one unit needs %llu seed slots (capacity %llu, SA_BATCH_SLOT_CAP)",
                             (unsigned long long)add, (unsigned long long)s->w.seed_cap);
                return SA_ERR_CAPACITY;
            }
            slots += add;
            ++b;
        }
        int r = run_batch_group(d, s, units, a, b, want_out, res);
        if (r == SA_ERR_CAPACITY) {
            if (b - a == 1) {
                sa_set_error(SA_ERR_CAPACITY, "survivors of one unit exceed SA_BATCH_SURV_CAP");
                return r;
            }
            uint32_t m = a + (b - a) / 2;
            SA_TRY(run_batch_range(d, s, units, a, m, want_out, res));
            SA_TRY(run_batch_range(d, s, units, m, b, want_out, res));
        } else if (r != SA_OK) {
            return r;
        }
        a = b;
    }
    return SA_OK;
}

// Units with an empty window are not run; the rest go through the batch slot.
int run_resolved(const SaResolvedUnit* units, uint32_t n, bool want_out, BatchResult& res,
                 std::vector<int64_t>& map) {
    Global& g = G();
    DevState& d = g.devs[0];
    if (!d.batch) {
        Slot* s = nullptr;
        SA_TRY(make_slot(0, g.batch_slot_cap, g.batch_surv_cap, g.long_cap, &s, kSlotBatch));
        d.batch = s;
    }
    std::vector<SaResolvedUnit> live;
    map.assign(n, -1);
    for (uint32_t i = 0; i < n; ++i)
        if (units[i].end > units[i].start) {
            map[i] = (int64_t)live.size();
            live.push_back(units[i]);
        }
    if (!res.sink) res.recs.resize(live.size());
    res.hits.assign(live.size(), 0);
    res.iters.assign(live.size(), 0);
    return run_batch_range(d, d.batch, live.data(), 0, (uint32_t)live.size(), want_out, res);
}

// ---------------------------------------------------------------------------
// Call coalescing.  Concurrent sa_seed_and_filter calls on one GPU share
// device passes: a caller stages its seed words in pinned memory and queues
// its call; then either another caller's pass takes it, or the caller gets a
// free slot and runs every queued call (its own among them, oldest first, up
// to the slot's unit and seed capacity) as the units of one batched pass with
// explicit seed words.  The batched path gives each unit exactly the HSP list
// of a plain call on the same words (per-unit MAX_HITS iterations and dedup
// scopes), so a call's result does not depend on its neighbours.  A pass that
// reports a device error (bad key, MAX_HITS, coordinates) re-runs its calls
// one at a time on the plain path, so each call gets its own status.
// ---------------------------------------------------------------------------
void free_staging() {
    Global& g = G();
    std::lock_guard<std::mutex> lk(g.pinned_mu);
    for (uint64_t* p : g.pinned_all) cudaFreeHost(p);
    g.pinned_all.clear();
    g.pinned_free.clear();
}

uint64_t* take_staging() {
    Global& g = G();
    {
        std::lock_guard<std::mutex> lk(g.pinned_mu);
        if (!g.pinned_free.empty()) {
            uint64_t* p = g.pinned_free.back();
            g.pinned_free.pop_back();
            return p;
        }
    }
    uint64_t* p = nullptr;
    if (cudaMallocHost(&p, 8 * std::max<uint64_t>(g.max_seeds, 1)) != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> lk(g.pinned_mu);
    g.pinned_all.push_back(p);
    return p;
}

void give_staging(uint64_t* p) {
    Global& g = G();
    std::lock_guard<std::mutex> lk(g.pinned_mu);
    g.pinned_free.push_back(p);
}

// Hands each live call of a completed group its output: header {0, 0, HSPs,
// hits} (src/seed_filter.cu:756-759) then its HSPs.
struct CallSink : SaBatchSink {
    const std::vector<CallReq*>& live;
    explicit CallSink(const std::vector<CallReq*>& l) : live(l) {}
    int put(uint32_t u0, uint32_t n, const SaRec* recs, const uint32_t* cnt, const uint64_t* hits) override {
        uint64_t at = 0;
        for (uint32_t i = 0; i < n; ++i) {
            CallReq& c = *live[u0 + i];
            sa_segment* o = (sa_segment*)malloc(sizeof(sa_segment) * (cnt[i] + 1ull));
            if (!o) {
                sa_set_error(SA_ERR_NOMEM, "host allocation of %u records failed", cnt[i] + 1);
                return SA_ERR_NOMEM;
            }
            o[0] = sa_segment{0, 0, cnt[i], (int32_t)(uint32_t)hits[i]};
            if (cnt[i]) std::memcpy(o + 1, recs + at, cnt[i] * sizeof(sa_segment));
            at += cnt[i];
            c.out = o;
            c.out_len = cnt[i] + 1ull;
            c.stats.num_hits = hits[i];
            c.stats.num_hsps = cnt[i];
        }
        return SA_OK;
    }
};

// The plain path for one queued call on slot s (a pass's fallback).
void run_call_alone(Slot* s, CallReq& c) {
    Global& g = G();
    DevState& d = g.devs[s->dev_idx];
    const Packed& q = c.rev ? d.qr[c.buffer] : d.qf[c.buffer];
    const sa_call_stats keep = t_stats;
    c.status = run_call(s, c.staged, c.n, c.rev, q, 0, 0, 0, &c.out, &c.out_len);
    c.stats = t_stats;
    c.stats.batch_calls = 1;
    if (c.status != SA_OK) c.err = t_err;
    t_stats = keep;
}

// One pass over queued calls on slot s (results and statuses into the calls).
void run_coalesced(Slot* s, const std::vector<CallReq*>& calls) {
    Global& g = G();
    DevState& d = g.devs[s->dev_idx];
    SaWork& w = s->w;
    std::vector<CallReq*> live;
    std::vector<SaResolvedUnit> ru;
    uint64_t off = 0;
    int r = cudaSetDevice(d.dev) == cudaSuccess ? SA_OK : SA_ERR_CUDA;
    for (CallReq* c : calls) {
        const Packed& q = c->rev ? d.qr[c->buffer] : d.qf[c->buffer];
        if (!q.data) {
            c->status = SA_ERR_STATE;
            c->err = "query buffer " + std::to_string(c->buffer) + " is not resident";
            continue;
        }
        if (c->n == 0) {  // no seeds: header only (src/seed_filter.cu:736-777 with num_hits = 0)
            c->out = (sa_segment*)malloc(sizeof(sa_segment));
            if (!c->out) {
                c->status = SA_ERR_NOMEM;
                c->err = "host allocation failed";
                continue;
            }
            c->out[0] = sa_segment{0, 0, 0, 0};
            c->out_len = 1;
            c->stats.batch_calls = 1;
            continue;
        }
        if (r == SA_OK &&
            cudaMemcpyAsync(w.seeds + off, c->staged, 8ull * c->n, cudaMemcpyHostToDevice, s->stream) != cudaSuccess)
            r = SA_ERR_CUDA;
        SaResolvedUnit u{nullptr, q.data, (uint32_t)q.len, 0, c->n, c->rev};
        u.seeds = w.seeds + off;
        ru.push_back(u);
        live.push_back(c);
        off += c->n;
    }
    if (live.empty()) return;
    if (r != SA_OK) {
        for (CallReq* c : live) {
            c->status = SA_ERR_CUDA;
            c->err = "seed upload failed";
        }
        return;
    }
    BatchResult res;
    CallSink sink(live);
    res.sink = &sink;
    res.hits.assign(live.size(), 0);
    res.iters.assign(live.size(), 0);
    r = run_batch_range(d, s, ru.data(), 0, (uint32_t)ru.size(), true, res);
    if (r == SA_OK) {
        for (size_t i = 0; i < live.size(); ++i) {
            sa_call_stats& st = live[i]->stats;
            st.num_seeds = live[i]->n;
            st.num_iter = res.iters[i];
            st.batch_calls = (uint32_t)live.size();
            // totals of the pass (the call's own when it ran alone)
            st.hits_extended = res.tot.extended;
            st.seeds_with_hits = res.tot.nnz;
            st.survivors = res.tot.surv_count;
            st.long_hits = res.tot.long_count;
            st.tiles = res.tot.base_steps;
            st.ms_total = res.timing.ms_total;
            st.ms_lookup = res.timing.ms_lookup;
            st.ms_extend_lane = res.timing.ms_extend_lane;
            st.ms_extend_warp = res.timing.ms_extend_warp;
            st.ms_dedup = res.timing.ms_dedup;
            st.ms_copy = res.timing.ms_copy;
        }
        return;
    }
    // a device error or a failed allocation: each call alone on the plain path
    for (CallReq* c : live) {
        free(c->out);
        c->out = nullptr;
        c->out_len = 0;
        c->stats = sa_call_stats{};
        run_call_alone(s, *c);
    }
}

// sa_seed_and_filter with coalescing (SA_COALESCE > 1).
int seed_and_filter_coalesced(const uint64_t* seeds, uint32_t num_seeds, int rev, uint32_t buffer,
                              sa_segment** out, uint64_t* out_len) {
    Global& g = G();
    CallReq c;
    c.seeds = seeds;
    c.n = num_seeds;
    c.rev = rev ? 1 : 0;
    c.buffer = buffer;
    c.staged = take_staging();
    if (!c.staged) {
        sa_set_error(SA_ERR_NOMEM, "pinned staging allocation failed");
        return SA_ERR_NOMEM;
    }
    if (num_seeds) std::memcpy(c.staged, seeds, 8ull * num_seeds);
    {
        std::unique_lock<std::mutex> lk(g.mu);
        g.pending.push_back(&c);
        while (true) {
            g.cv.wait(lk, [&] { return c.done || (!c.taken && !g.free_slots.empty()); });
            if (c.done) break;
            Slot* s = take_free_slot_locked();
            std::vector<CallReq*> pass;
            uint64_t words = 0;
            while (!g.pending.empty() && pass.size() < std::min<uint32_t>(g.coalesce_calls, s->max_units)) {
                CallReq* r = g.pending.front();
                if (!pass.empty() && words + r->n > s->w.seed_cap) break;
                g.pending.pop_front();
                r->taken = true;
                pass.push_back(r);
                words += r->n;
            }
            lk.unlock();
            run_coalesced(s, pass);
            lk.lock();
            for (CallReq* r : pass) r->done = true;
            g.free_slots.push_back(s);
            g.cv.notify_all();
        }
    }
    give_staging(c.staged);
    t_stats = c.stats;
    if (c.status != SA_OK) {
        sa_set_error(c.status, "%s", c.err.c_str());
        return c.status;
    }
    *out = c.out;
    *out_len = c.out_len;
    return SA_OK;
}

// Output of sa_seed_and_filter_batch, written as groups complete: per unit a
// header record {0, 0, HSP count, hit count} then its HSPs; a unit with an
// empty window gets its header only.  One malloc'd block (grown by realloc,
// which remaps rather than copies at these sizes), freed by sa_free_segments.
// Batched outputs of at least kKeepBytes are remembered, and the two largest
// the caller has freed are kept for the next batched outputs that fit: a fresh
// array of hundreds of MB pays a page fault per 4 KiB page at its first write.
constexpr uint64_t kKeepBytes = 64ull << 20;
struct OutKeep {
    std::mutex mu;
    std::vector<std::pair<void*, uint64_t>> live;  // batched outputs handed out (pointer, bytes)
    std::vector<std::pair<void*, uint64_t>> kept;  // freed ones kept for reuse (at most kKeepArrays)
};
// Two: a caller that holds one call's lists while the next call runs (a
// steady loop over batches) then never allocates.
constexpr size_t kKeepArrays = 2;
OutKeep& out_keep() {
    static OutKeep k;
    return k;
}

// Allocation of a batched output array of `bytes` (or more, when a kept one fits).
void* out_alloc(uint64_t bytes, uint64_t* got) {
    OutKeep& k = out_keep();
    std::lock_guard<std::mutex> lk(k.mu);
    void* p = nullptr;
    size_t best = k.kept.size();
    for (size_t i = 0; i < k.kept.size(); ++i)  // the smallest kept array that fits
        if (k.kept[i].second >= bytes && (best == k.kept.size() || k.kept[i].second < k.kept[best].second)) best = i;
    if (best < k.kept.size()) {
        p = k.kept[best].first;
        *got = k.kept[best].second;
        k.kept.erase(k.kept.begin() + (std::ptrdiff_t)best);
    } else {
        p = malloc(bytes);
        *got = bytes;
    }
    if (p && *got >= kKeepBytes) k.live.emplace_back(p, *got);
    return p;
}

void out_forget(void* p) {
    OutKeep& k = out_keep();
    for (size_t i = 0; i < k.live.size(); ++i)
        if (k.live[i].first == p) {
            k.live.erase(k.live.begin() + (std::ptrdiff_t)i);
            return;
        }
}

// Returns true when p was a remembered batched output (kept or freed here).
bool out_release(void* p) {
    OutKeep& k = out_keep();
    std::lock_guard<std::mutex> lk(k.mu);
    for (size_t i = 0; i < k.live.size(); ++i)
        if (k.live[i].first == p) {
            k.kept.push_back(k.live[i]);
            k.live.erase(k.live.begin() + (std::ptrdiff_t)i);
            if (k.kept.size() > kKeepArrays) {  // free the smallest
                size_t s = 0;
                for (size_t j = 1; j < k.kept.size(); ++j)
                    if (k.kept[j].second < k.kept[s].second) s = j;
                free(k.kept[s].first);
                k.kept.erase(k.kept.begin() + (std::ptrdiff_t)s);
            }
            return true;
        }
    return false;
}

void out_drop_kept() {
    OutKeep& k = out_keep();
    std::lock_guard<std::mutex> lk(k.mu);
    for (auto& e : k.kept) free(e.first);
    k.kept.clear();
}

struct SegmentWriter : SaBatchSink {
    const uint64_t n_units;
    uint64_t* offsets;
    std::vector<uint32_t> orig;  // live unit -> unit index
    sa_segment* o = nullptr;
    uint64_t cap = 0, at = 0;
    uint32_t next = 0;  // next unit to get a header

    SegmentWriter(const sa_unit* units, uint32_t n, uint64_t* offs) : n_units(n), offsets(offs) {
        for (uint32_t i = 0; i < n; ++i)
            if (units[i].end > units[i].start) orig.push_back(i);
    }
    ~SegmentWriter() override {
        if (o && !out_release(o)) free(o);
    }

    sa_segment* release() {
        sa_segment* p = o;
        o = nullptr;
        return p;
    }

    int reserve(uint64_t need) {
        if (need <= cap) return SA_OK;
        uint64_t c = std::max<uint64_t>(need, cap + cap / 2);
        void* p = nullptr;
        if (!o) {
            uint64_t got = 0;
            p = out_alloc(sizeof(sa_segment) * c, &got);
            c = got / sizeof(sa_segment);
        } else {
            {
                std::lock_guard<std::mutex> lk(out_keep().mu);
                out_forget(o);
            }
            p = realloc(o, sizeof(sa_segment) * c);
            if (p && sizeof(sa_segment) * c >= kKeepBytes) {
                std::lock_guard<std::mutex> lk(out_keep().mu);
                out_keep().live.emplace_back(p, sizeof(sa_segment) * c);
            }
        }
        if (!p) {
            sa_set_error(SA_ERR_NOMEM, "cannot hold %llu HSP records", (unsigned long long)c);
            return SA_ERR_NOMEM;
        }
        o = (sa_segment*)p;
        cap = c;
        return SA_OK;
    }

    void header(uint32_t nb, uint64_t hits) {
        offsets[next++] = at;
        o[at++] = sa_segment{0, 0, nb, (int32_t)(uint32_t)hits};
    }

    int expect(uint64_t records) override { return reserve(at + records + (n_units - next) + 1); }

    int put(uint32_t u0, uint32_t n, const SaRec* recs, const uint32_t* cnt, const uint64_t* hits) override {
        if (!n) return SA_OK;
        uint64_t body = 0;
        for (uint32_t i = 0; i < n; ++i) body += cnt[i];
        // this group's records plus a header for every unit not yet written,
        // so that finish() does not grow the array
        SA_TRY(reserve(at + body + (n_units - next) + 1));
        std::vector<uint64_t> dst(n), src(n);
        uint64_t s = 0;
        for (uint32_t i = 0; i < n; ++i) {
            while (next < orig[u0 + i]) header(0, 0);
            header(cnt[i], hits[i]);
            dst[i] = at;
            src[i] = s;
            at += cnt[i];
            s += cnt[i];
        }
        // copy the bodies, units split over up to 8 threads by record count
        auto copy = [&](uint32_t a, uint32_t b) {
            for (uint32_t i = a; i < b; ++i)
                if (cnt[i]) std::memcpy(o + dst[i], recs + src[i], cnt[i] * sizeof(sa_segment));
        };
        const uint64_t kPer = 1u << 19;  // records per thread, at least
        const uint32_t nt = (uint32_t)std::min<uint64_t>({8, n, body / kPer});
        if (nt < 2) {
            copy(0, n);
            return SA_OK;
        }
        std::vector<uint32_t> cut(nt + 1, n);
        cut[0] = 0;
        for (uint32_t i = 0, t = 1; i < n && t < nt; ++i)
            if (src[i] + cnt[i] >= body * t / nt) cut[t++] = i + 1;
        std::vector<std::thread> th;
        for (uint32_t t = 1; t < nt; ++t) th.emplace_back(copy, cut[t], cut[t + 1]);
        copy(cut[0], cut[1]);
        for (auto& x : th) x.join();
        return SA_OK;
    }

    int finish() {
        SA_TRY(reserve(at + (n_units - next) + 1));
        while (next < n_units) header(0, 0);
        offsets[n_units] = at;
        return SA_OK;
    }
};

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char* sa_last_error(void) { return t_err.c_str(); }

int sa_last_call_stats(sa_call_stats* s) {
    if (!s) return SA_ERR_ARG;
    *s = t_stats;
    return SA_OK;
}

// common/seed_filter_interface.cu:49-80
int sa_initialize_interface(int num_gpu) {
    Global& g = G();
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        sa_set_error(SA_ERR_NO_DEVICE, "no GPU device found");
        return SA_ERR_NO_DEVICE;
    }
    int use = num_gpu == -1 ? n : num_gpu;
    if (use < 1) {
        sa_set_error(SA_ERR_ARG, "num_gpu must be -1 or >= 1");
        return SA_ERR_ARG;
    }
    if (use > n) {
        sa_set_error(SA_ERR_TOO_MANY_GPUS, "requested %d GPUs, %d available", use, n);
        return SA_ERR_TOO_MANY_GPUS;
    }
    if (g.interface_ready) sa_shutdown_processor();
    int cur = 0;
    cudaGetDevice(&cur);
    g.devs.assign(use, DevState());
    for (int i = 0; i < use; ++i) {
        // with one GPU in use, keep the caller's current device
        g.devs[i].dev = use == 1 ? cur : i;
        cudaDeviceProp prop;
        SA_CUDA_OK(cudaGetDeviceProperties(&prop, g.devs[i].dev));
        g.devs[i].num_sms = prop.multiProcessorCount;
        g.devs[i].total_mem = prop.totalGlobalMem;
    }
    if (!g.shape_set) {
        set_shape_positions(g.params, "TTT0T00TT00T0T0TTTT");
        g.shape_set = true;
    }
    g.interface_ready = true;
    return use;
}

// common/ntcoding.cpp:21-37 + src/main.cpp:152-171
int sa_generate_shape_pos(const char* shape) {
    if (!shape) return SA_ERR_ARG;
    std::string name = shape, pat;
    if (name == "12of19") pat = "TTT0T00TT00T0T0TTTT";
    else if (name == "14of22") pat = "TTT0T0TT00TT00T0T0TTTT";
    else {
        pat = name;
        for (auto& c : pat) c = (c == '1' || c == 'T') ? 'T' : '0';
    }
    int k = 0;
    for (char c : pat) k += c == 'T';
    if (k > 15 || k <= 3 || pat.size() > 32) {
        sa_set_error(SA_ERR_ARG, "shape must have 4..15 sampled positions and span <= 32 (got K=%d, span=%zu)", k,
                     pat.size());
        return SA_ERR_ARG;
    }
    Global& g = G();
    set_shape_positions(g.params, pat);
    g.shape_set = true;
    return k;
}

// common/seed_filter_interface.cu:82-101
int sa_send_ref_write_request(const char* seq, size_t start_addr, uint32_t len) {
    invalidate_graphs();
    Global& g = G();
    if (!g.interface_ready) {
        sa_set_error(SA_ERR_STATE, "sa_initialize_interface() has not been called");
        return SA_ERR_STATE;
    }
    if (!seq) return SA_ERR_ARG;
    for (auto& d : g.devs) SA_TRY(upload_pack(d, seq + start_addr, len, d.ref, nullptr));
    g.last_ref_ptr = seq;
    g.last_ref_start = start_addr;
    g.last_ref_len = len;
    g.ref_len = len;
    return SA_OK;
}

// common/seed_filter_interface.cu:103-113
int sa_clear_ref(void) {
    invalidate_graphs();
    std::unique_lock<std::shared_mutex> dev_wide(g_capture_mu);
    Global& g = G();
    for (auto& d : g.devs) {
        cudaSetDevice(d.dev);
        d.ref.release();
        d.ref_rc.release();
        if (d.index) cudaFree(d.index);
        if (d.pos) cudaFree(d.pos);
        d.index = d.pos = nullptr;
        d.nbuckets = d.num_index = 0;
    }
    g.last_ref_ptr = nullptr;
    return SA_OK;
}

static int build_table_on(DevState& d, const Packed& ref, uint32_t step) {
    std::unique_lock<std::shared_mutex> dev_wide(g_capture_mu);
    Global& g = G();
    SA_CUDA_OK(cudaSetDevice(d.dev));
    const SaParams& p = g.params;
    // common/seed_pos_table.cu:58-64: offset, start, num_steps
    uint32_t offset = (uint32_t)(p.seed_size + 1) % step;
    uint32_t start = step - offset;
    int64_t span = (int64_t)ref.len - p.seed_size + offset;
    uint64_t num_steps = span > 0 ? (uint64_t)span / step : 0;
    uint64_t nb = 1ull << (2 * p.kmer_size);
    uint64_t cap = num_steps ? num_steps : 1;
    uint32_t *keys = nullptr, *vals = nullptr, *keys2 = nullptr, *vals2 = nullptr;
    unsigned long long* scratch = nullptr;
    unsigned int* hist = nullptr;
    auto cleanup = [&]() {
        if (keys) cudaFree(keys);
        if (vals) cudaFree(vals);
        if (keys2) cudaFree(keys2);
        if (vals2) cudaFree(vals2);
        if (scratch) cudaFree(scratch);
        if (hist) cudaFree(hist);
    };
    cudaError_t e = cudaSuccess;
    if ((e = cudaMalloc(&keys, 4 * cap)) != cudaSuccess || (e = cudaMalloc(&vals, 4 * cap)) != cudaSuccess ||
        (e = cudaMalloc(&keys2, 4 * cap)) != cudaSuccess || (e = cudaMalloc(&vals2, 4 * cap)) != cudaSuccess ||
        (e = cudaMalloc(&scratch, 8 * (2 * SA_MAX_CTAS + 4))) != cudaSuccess ||
        (e = cudaMalloc(&hist, 4 * (256 * (uint64_t)SA_MAX_CTAS + 64))) != cudaSuccess) {
        cleanup();
        return sa_cuda_fail(e, "cudaMalloc(table build)", __FILE__, __LINE__);
    }
    const int Gr = std::min(g.tuning.range_ctas, SA_MAX_CTAS);
    unsigned long long* cta_a = scratch;
    unsigned long long* cta_b = scratch + SA_MAX_CTAS;
    unsigned long long* d_total = scratch + 2 * SA_MAX_CTAS;
    cudaMemset(d_total, 0, 8);
    sa_launch_table_keys(ref.data, start, num_steps, step, p, keys, vals, cta_a, cta_b, d_total, Gr, 0);
    int in_tmp = 0;
    sa_launch_sort_kv(keys, vals, keys2, vals2, d_total, 2 * p.kmer_size, hist, Gr, 0, &in_tmp);
    unsigned long long n_valid = 0;
    e = cudaMemcpy(&n_valid, d_total, 8, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        cleanup();
        return sa_cuda_fail(e, "table build", __FILE__, __LINE__);
    }
    if (d.index) cudaFree(d.index);
    if (d.pos) cudaFree(d.pos);
    d.index = d.pos = nullptr;
    if ((e = cudaMalloc(&d.index, 4 * nb)) != cudaSuccess) {
        cleanup();
        return sa_cuda_fail(e, "cudaMalloc(index table)", __FILE__, __LINE__);
    }
    uint32_t* sk = in_tmp ? keys2 : keys;
    uint32_t* sv = in_tmp ? vals2 : vals;
    sa_launch_table_index(sk, d_total, d.index, nb, 0);
    // keep the sorted positions as the position table; free the rest
    d.pos = sv;
    if (sv == vals) vals = nullptr;
    else vals2 = nullptr;
    e = cudaDeviceSynchronize();
    cleanup();
    if (e != cudaSuccess) return sa_cuda_fail(e, "table build", __FILE__, __LINE__);
    d.nbuckets = nb;
    d.num_index = n_valid;
    return SA_OK;
}

// common/seed_pos_table.cu:49-109
int sa_generate_seed_pos_table(const char* ref_str, size_t start_addr, uint32_t ref_length, uint32_t step,
                               int shape_size, int kmer_size) {
    invalidate_graphs();
    Global& g = G();
    if (!g.interface_ready) {
        sa_set_error(SA_ERR_STATE, "sa_initialize_interface() has not been called");
        return SA_ERR_STATE;
    }
    if (step == 0 || shape_size != g.params.seed_size || kmer_size != g.params.kmer_size) {
        sa_set_error(SA_ERR_ARG, "step must be >= 1 and shape_size/kmer_size must match the shape (%d/%d)",
                     g.params.seed_size, g.params.kmer_size);
        return SA_ERR_ARG;
    }
    const bool resident = ref_str == g.last_ref_ptr && start_addr == g.last_ref_start &&
                          ref_length == g.last_ref_len && g.last_ref_ptr;
    for (auto& d : g.devs) {
        if (resident && d.ref.data) {
            SA_TRY(build_table_on(d, d.ref, step));
        } else {
            if (!ref_str) return SA_ERR_ARG;
            Packed tmp;
            SA_TRY(upload_pack(d, ref_str + start_addr, ref_length, tmp, nullptr));
            int r = build_table_on(d, tmp, step);
            tmp.release();
            if (r != SA_OK) return r;
        }
    }
    return SA_OK;
}

// common/seed_pos_table.cu:33-47
int sa_send_seed_pos_table(const uint32_t* index_table, uint32_t index_table_size, const uint32_t* pos_table,
                           uint32_t num_index) {
    invalidate_graphs();
    Global& g = G();
    if (!g.interface_ready) return SA_ERR_STATE;
    if (!index_table || (num_index && !pos_table)) return SA_ERR_ARG;
    if (index_table_size != (1ull << (2 * g.params.kmer_size)) || index_table[index_table_size - 1] != num_index) {
        sa_set_error(SA_ERR_ARG, "index table must have 4^K = %llu entries ending at num_index",
                     1ull << (2 * g.params.kmer_size));
        return SA_ERR_ARG;
    }
    for (uint32_t i = 0; i < num_index; ++i)
        if ((uint64_t)pos_table[i] + (uint64_t)g.params.seed_size > g.ref_len) {
            sa_set_error(SA_ERR_ARG, "position %u of the table lies past the target end", pos_table[i]);
            return SA_ERR_ARG;
        }
    for (auto& d : g.devs) {
        SA_CUDA_OK(cudaSetDevice(d.dev));
        if (d.index) cudaFree(d.index);
        if (d.pos) cudaFree(d.pos);
        d.index = d.pos = nullptr;
        SA_CUDA_OK(cudaMalloc(&d.index, 4ull * index_table_size));
        SA_CUDA_OK(cudaMemcpy(d.index, index_table, 4ull * index_table_size, cudaMemcpyHostToDevice));
        SA_CUDA_OK(cudaMalloc(&d.pos, 4ull * (num_index ? num_index : 1)));
        if (num_index) SA_CUDA_OK(cudaMemcpy(d.pos, pos_table, 4ull * num_index, cudaMemcpyHostToDevice));
        d.nbuckets = index_table_size;
        d.num_index = num_index;
    }
    return SA_OK;
}

int sa_get_seed_pos_table(uint32_t* index_table, uint64_t index_cap, uint32_t* pos_table, uint64_t pos_cap,
                          uint64_t* index_table_size, uint64_t* num_index) {
    Global& g = G();
    if (g.devs.empty() || !g.devs[0].index) return SA_ERR_STATE;
    DevState& d = g.devs[0];
    if (index_table_size) *index_table_size = d.nbuckets;
    if (num_index) *num_index = d.num_index;
    SA_CUDA_OK(cudaSetDevice(d.dev));
    if (index_table && index_cap >= d.nbuckets)
        SA_CUDA_OK(cudaMemcpy(index_table, d.index, 4 * d.nbuckets, cudaMemcpyDeviceToHost));
    if (pos_table && pos_cap >= d.num_index && d.num_index)
        SA_CUDA_OK(cudaMemcpy(pos_table, d.pos, 4 * d.num_index, cudaMemcpyDeviceToHost));
    return SA_OK;
}

// src/seed_filter.cu:780-847
int sa_initialize_processor(int transition, uint32_t wga_chunk, uint32_t seed_size, const int* sub_mat, int xdrop,
                            int hspthresh, int noentropy) {
    invalidate_graphs();
    Global& g = G();
    if (!g.interface_ready) {
        sa_set_error(SA_ERR_STATE, "sa_initialize_interface() has not been called");
        return SA_ERR_STATE;
    }
    if (!sub_mat || wga_chunk == 0 || (int)seed_size != g.params.seed_size) {
        sa_set_error(SA_ERR_ARG, "sub_mat required, wga_chunk > 0, seed_size must equal the shape span (%d)",
                     g.params.seed_size);
        return SA_ERR_ARG;
    }
    // release old slots
    free_staging();
    {
        std::lock_guard<std::mutex> lk(g.mu);
        for (auto* s : g.free_slots) free_slot(s);
        g.free_slots.clear();
        for (auto& d : g.devs) {
            d.slots.clear();
            if (d.batch) free_slot(d.batch);
            d.batch = nullptr;
            for (int b = 0; b < kMaxBuffers; ++b) drop_keys(d, b);
        }
    }
    for (int i = 0; i < 64; ++i) g.params.sub_mat[i] = sub_mat[i];
    g.params.xdrop = xdrop;
    g.params.hspthresh = hspthresh;
    g.params.noentropy = noentropy ? 1 : 0;
    g.params.transition = transition ? 1 : 0;
    g.wga_chunk = wga_chunk;
    g.max_seeds = transition ? 13ull * wga_chunk : wga_chunk;  // :786-789
    // MAX_HITS = MAX_HITS_PER_GB * (float)(totalGlobalMem / 1 GiB) (:784, :791)
    float gb = (float)(g.devs[0].total_mem / 1073741824.0f);
    g.max_hits_default = (uint64_t)(int)(4194304 * gb);
    auto pow2_floor = [](uint64_t v) {
        uint64_t p = 1;
        while (p * 2 <= v) p <<= 1;
        return p;
    };
    g.surv_cap = pow2_floor(env_u64("SA_SURV_CAP", 1ull << 25));
    g.long_cap = env_u64("SA_LONG_CAP", 1ull << 24);
    g.batch_slot_cap = env_u64("SA_BATCH_SLOT_CAP", 1ull << 28);
    g.batch_surv_cap = pow2_floor(env_u64("SA_BATCH_SURV_CAP", 1ull << 29));
    const int per_gpu = (int)env_u64("SA_SLOTS_PER_GPU", 2);
    // call coalescing (opt-in): up to SA_COALESCE calls (and SA_COALESCE_SEEDS
    // words) per pass.  Off by default: with free slots the passes stay small,
    // and on a 16-core host the per-call graphs on 12 slots measured faster
    // (genome scale, 16 seeder threads: 0.373 s per step against 0.43-0.52 s).
    g.coalesce_calls = (uint32_t)std::min<uint64_t>(env_u64("SA_COALESCE", 0), 1024);
    const uint64_t pass_seeds =
        std::max<uint64_t>(g.max_seeds, std::min<uint64_t>((uint64_t)g.coalesce_calls * g.max_seeds,
                                                           env_u64("SA_COALESCE_SEEDS", 1ull << 23)));
    for (size_t di = 0; di < g.devs.size(); ++di) {
        for (int k = 0; k < per_gpu; ++k) {
            Slot* s = nullptr;
            if (g.coalesce_calls > 1)
                SA_TRY(make_slot((int)di, pass_seeds, g.surv_cap, g.long_cap, &s, kSlotBoth, g.coalesce_calls));
            else
                SA_TRY(make_slot((int)di, g.max_seeds, g.surv_cap, g.long_cap, &s));
            std::lock_guard<std::mutex> lk(g.mu);
            g.devs[di].slots.push_back(s);
            g.free_slots.push_back(s);
        }
    }
    g.processor_ready = true;
    return SA_OK;
}

// src/seed_filter.cu:849-869
int sa_send_query_write_request(const char* query_buffer, size_t start_addr, uint32_t len, uint32_t buffer) {
    Global& g = G();
    if (!g.interface_ready) return SA_ERR_STATE;
    if (!query_buffer || buffer >= (uint32_t)kMaxBuffers) {
        sa_set_error(SA_ERR_ARG, "query buffer pointer required and buffer < %d", kMaxBuffers);
        return SA_ERR_ARG;
    }
    for (auto& d : g.devs) {
        invalidate_keys(d, buffer);
        SA_TRY(upload_pack(d, query_buffer + start_addr, len, d.qf[buffer], &d.qr[buffer]));
    }
    return SA_OK;
}

// src/seed_filter.cu:654-778
int sa_seed_and_filter(const uint64_t* seeds, uint32_t num_seeds, int rev, uint32_t buffer, sa_segment** out,
                       uint64_t* out_len) {
    SA_TRY(check_ready(true));
    Global& g = G();
    if (!out || !out_len || (num_seeds && !seeds) || buffer >= (uint32_t)kMaxBuffers) return SA_ERR_ARG;
    if (num_seeds > g.max_seeds) {
        sa_set_error(SA_ERR_MAX_SEEDS, "%u seeds exceed MAX_SEEDS = %llu", num_seeds,
                     (unsigned long long)g.max_seeds);
        return SA_ERR_MAX_SEEDS;
    }
    if (g.coalesce_calls > 1) return seed_and_filter_coalesced(seeds, num_seeds, rev, buffer, out, out_len);
    Slot* s = acquire_slot();
    DevState& d = g.devs[s->dev_idx];
    const Packed& q = rev ? d.qr[buffer] : d.qf[buffer];
    int r;
    if (!q.data) {
        sa_set_error(SA_ERR_STATE, "query buffer %u is not resident", buffer);
        r = SA_ERR_STATE;
    } else {
        r = run_call(s, seeds, num_seeds, rev, q, 0, 0, 0, out, out_len);
    }
    release_slot(s);
    return r;
}

// src/seed_filter.cu:871-880
int sa_clear_query(uint32_t buffer) {
    Global& g = G();
    if (buffer >= (uint32_t)kMaxBuffers) return SA_ERR_ARG;
    std::unique_lock<std::shared_mutex> dev_wide(g_capture_mu);
    for (auto& d : g.devs) {
        cudaSetDevice(d.dev);
        d.qf[buffer].release();
        d.qr[buffer].release();
        drop_keys(d, buffer);
    }
    return SA_OK;
}

// repeat_masker_src/seed_filter.cu:925-935
int sa_rm_send_query_write_request(void) {
    invalidate_graphs();
    Global& g = G();
    for (auto& d : g.devs) {
        if (!d.ref.data) {
            sa_set_error(SA_ERR_STATE, "no resident target");
            return SA_ERR_STATE;
        }
        std::unique_lock<std::shared_mutex> dev_wide(g_capture_mu);
        SA_CUDA_OK(cudaSetDevice(d.dev));
        SA_TRY(alloc_packed(d.ref_rc, d.ref.len));
        make_rc_packed(d.ref, d.ref_rc);
        SA_CUDA_OK(cudaDeviceSynchronize());
    }
    return SA_OK;
}

// repeat_masker_src/seed_filter.cu:723-855
int sa_rm_seed_and_filter(const uint64_t* seeds, uint32_t num_seeds, int rev, uint32_t ref_start, uint32_t ref_end,
                          sa_segment** out, uint64_t* out_len) {
    SA_TRY(check_ready(false));
    Global& g = G();
    if (!out || !out_len || (num_seeds && !seeds)) return SA_ERR_ARG;
    if (num_seeds > g.max_seeds) {
        sa_set_error(SA_ERR_MAX_SEEDS, "%u seeds exceed MAX_SEEDS", num_seeds);
        return SA_ERR_MAX_SEEDS;
    }
    Slot* s = acquire_slot();
    DevState& d = g.devs[s->dev_idx];
    const Packed& q = rev ? d.ref_rc : d.ref;
    int r;
    if (!q.data) {
        sa_set_error(SA_ERR_STATE, "sa_rm_send_query_write_request() has not been called");
        r = SA_ERR_STATE;
    } else {
        r = run_call(s, seeds, num_seeds, rev, q, 1, ref_start, ref_end, out, out_len);
    }
    release_slot(s);
    return r;
}

// repeat_masker_src/seed_filter.cu:937-946
int sa_rm_clear_query(void) {
    Global& g = G();
    for (auto& d : g.devs) {
        cudaSetDevice(d.dev);
        d.ref_rc.release();
    }
    return SA_OK;
}

// src/seed_filter.cu:882-890 (without cudaDeviceReset: only this library's buffers are freed)
int sa_shutdown_processor(void) {
    Global& g = G();
    free_staging();
    out_drop_kept();
    {
        std::lock_guard<std::mutex> lk(g.mu);
        for (auto& d : g.devs)
            for (auto* s : d.slots) free_slot(s);
        g.free_slots.clear();
        for (auto& d : g.devs) {
            d.slots.clear();
            if (d.batch) free_slot(d.batch);
            d.batch = nullptr;
        }
    }
    for (auto& d : g.devs) {
        cudaSetDevice(d.dev);
        for (int b = 0; b < kMaxBuffers; ++b) {
            d.qf[b].release();
            d.qr[b].release();
            drop_keys(d, b);
        }
        if (d.stage) cudaFree(d.stage);
        d.stage = nullptr;
        d.stage_cap = 0;
    }
    sa_clear_ref();
    g.processor_ready = false;
    return SA_OK;
}


int sa_refresh_query_keys(uint32_t buffer) {
    SA_TRY(check_ready(true));
    Global& g = G();
    if (buffer >= (uint32_t)kMaxBuffers) return SA_ERR_ARG;
    std::lock_guard<std::mutex> lk(g.batch_mu);
    for (auto& d : g.devs)
        for (int rev = 0; rev < 2; ++rev) {
            d.qkeys_ok[buffer][rev] = false;
            SA_TRY(ensure_keys(d, buffer, rev));
        }
    return SA_OK;
}

// Batched SeedAndFilter (no single reference counterpart; each unit reproduces
// one src/seed_filter.cu:654-778 call on the seeds of src/seeder.cpp:57-74).
int sa_seed_and_filter_batch(const sa_unit* units, uint32_t n_units, sa_segment** out, uint64_t* out_len,
                             uint64_t* offsets) {
    SA_TRY(check_ready(true));
    Global& g = G();
    if (!units && n_units) return SA_ERR_ARG;
    if ((out == nullptr) != (out_len == nullptr) || (out && !offsets)) return SA_ERR_ARG;
    DevState& d = g.devs[0];
    for (uint32_t i = 0; i < n_units; ++i) {
        const sa_unit& u = units[i];
        if (u.buffer >= (uint32_t)kMaxBuffers || u.start > u.end) {
            sa_set_error(SA_ERR_ARG, "unit %u: buffer < %d and start <= end required", i, kMaxBuffers);
            return SA_ERR_ARG;
        }
        const Packed& q = u.rev ? d.qr[u.buffer] : d.qf[u.buffer];
        if (!q.data || u.end > q.len) {
            sa_set_error(SA_ERR_STATE, "unit %u: query buffer %u not resident or window past its end", i, u.buffer);
            return SA_ERR_STATE;
        }
    }
    std::lock_guard<std::mutex> lk(g.batch_mu);
    std::vector<SaResolvedUnit> ru(n_units);
    for (uint32_t i = 0; i < n_units; ++i) {
        const int rev = units[i].rev ? 1 : 0;
        SA_TRY(ensure_keys(d, units[i].buffer, rev));
        const Packed& q = rev ? d.qr[units[i].buffer] : d.qf[units[i].buffer];
        ru[i] = SaResolvedUnit{d.qkeys[units[i].buffer][rev], q.data, (uint32_t)q.len, units[i].start, units[i].end,
                               rev};
    }
    BatchResult res;
    std::vector<int64_t> map;
    SegmentWriter wr(units, n_units, offsets);
    if (out) res.sink = &wr;
    SA_TRY(run_resolved(ru.data(), n_units, out != nullptr, res, map));
    std::memset(&t_stats, 0, sizeof t_stats);
    t_stats.num_hits = res.tot.num_hits;
    t_stats.hits_extended = res.tot.extended;
    t_stats.seeds_with_hits = res.tot.nnz;
    t_stats.survivors = res.tot.surv_count;
    t_stats.num_hsps = res.tot.uniq_count;
    t_stats.long_hits = res.tot.long_count;
    t_stats.tiles = res.tot.base_steps;
    t_stats.num_iter = 1;
    t_stats.ms_total = res.timing.ms_total;
    t_stats.ms_lookup = res.timing.ms_lookup;
    t_stats.ms_extend_lane = res.timing.ms_extend_lane;
    t_stats.ms_extend_warp = res.timing.ms_extend_warp;
    t_stats.ms_dedup = res.timing.ms_dedup;
    t_stats.ms_copy = res.timing.ms_copy;
    if (!out) return SA_OK;
    SA_TRY(wr.finish());
    *out_len = wr.at;
    *out = wr.release();
    return SA_OK;
}

void sa_free_segments(sa_segment* p) {
    if (p && !out_release(p)) free(p);
}

int sa_set_timing(int on) {
    invalidate_graphs();
    g_timing = on ? 1 : 0;
    return SA_OK;
}

int sa_get_timing(void) { return g_timing.load(); }

uint64_t sa_kernel_launches(void) { return g_launches.load(); }

}  // extern "C"

int sa_run_units(const SaResolvedUnit* units, uint32_t n, bool want_out, SaRunResult* out) {
    int r = check_ready(true);
    if (r != SA_OK) return r;
    Global& g = G();
    std::lock_guard<std::mutex> lk(g.batch_mu);
    BatchResult res;
    res.sink = out->sink;
    std::vector<int64_t> map;
    r = run_resolved(units, n, want_out, res, map);
    if (r != SA_OK) return r;
    if (!out->sink) out->recs->assign(n, {});
    out->hits->assign(n, 0);
    for (uint32_t i = 0; i < n; ++i)
        if (map[i] >= 0) {
            (*out->hits)[i] = res.hits[map[i]];
            if (want_out && !out->sink) (*out->recs)[i] = std::move(res.recs[map[i]]);
        }
    out->tot = res.tot;
    out->ms_total = res.timing.ms_total;
    out->ms_lookup = res.timing.ms_lookup;
    out->ms_extend_lane = res.timing.ms_extend_lane;
    out->ms_extend_warp = res.timing.ms_extend_warp;
    out->ms_dedup = res.timing.ms_dedup;
    out->ms_copy = res.timing.ms_copy;
    return SA_OK;
}

int sa_resident_view(uint32_t buffer, SaResidentView* v) {
    int r = check_ready(true);
    if (r != SA_OK) return r;
    Global& g = G();
    if (buffer >= (uint32_t)kMaxBuffers) return SA_ERR_ARG;
    const DevState& d = g.devs[0];
    v->dev = d.dev;
    v->num_sms = d.num_sms;
    v->ref = d.ref.data;
    v->ref_len = (uint32_t)d.ref.len;
    v->index = d.index;
    v->nbuckets = d.nbuckets;
    v->pos = d.pos;
    v->q_packed[0] = d.qf[buffer].data;
    v->q_packed[1] = d.qr[buffer].data;
    v->q_len = (uint32_t)d.qf[buffer].len;
    v->max_seeds = g.max_seeds;
    v->max_hits = max_hits_now();
    v->wga_chunk = g.wga_chunk;
    v->params = g.params;
    v->tuning = g.tuning;
    return SA_OK;
}

extern "C" {

int sa_set_max_hits(uint64_t max_hits) {
    invalidate_graphs();
    G().max_hits_override = max_hits;
    return SA_OK;
}

int sa_set_rm_exclude_diagonal(int on) {
    invalidate_graphs();
    G().rm_exclude_diag = on ? 1 : 0;
    return SA_OK;
}

int sa_set_tuning_param(const char* name, int value) {
    invalidate_graphs();
    if (!name) return SA_ERR_ARG;
    SaTuning& t = G().tuning;
    const std::string n = name;
    if (n == "lane_cap") return sa_set_tuning(value, -1, -1, -1);
    if (n == "ext_ctas_per_sm") return sa_set_tuning(-1, -1, value, -1);
    if (n == "tile_hits") return sa_set_tuning(-1, -1, -1, value);
    if (n == "step_bases") {
        if (value != 8 && value != 16 && value != 32) {
            sa_set_error(SA_ERR_ARG, "step_bases must be 8, 16 or 32 (got %d)", value);
            return SA_ERR_ARG;
        }
        t.step_bases = value;
        return SA_OK;
    }
    if (n == "range_ctas" || n == "call_range_ctas") {
        if (value < 1 || value > SA_MAX_CTAS) {
            sa_set_error(SA_ERR_ARG, "%s must be 1..%d (got %d)", name, SA_MAX_CTAS, value);
            return SA_ERR_ARG;
        }
        (n == "range_ctas" ? t.range_ctas : t.call_range_ctas) = value;
        return SA_OK;
    }
    if (n == "switch_now" || n == "rm_switch_now") {
        if (value != 0 && value != 1) {
            sa_set_error(SA_ERR_ARG, "%s must be 0 or 1 (got %d)", name, value);
            return SA_ERR_ARG;
        }
        (n == "switch_now" ? t.switch_now : t.rm_switch_now) = value;
        return SA_OK;
    }
    if (n == "rm_substeps") {
        if (value < 1 || value > 8) {
            sa_set_error(SA_ERR_ARG, "rm_substeps must be 1..8 (got %d)", value);
            return SA_ERR_ARG;
        }
        t.rm_substeps = value;
        return SA_OK;
    }
    if (n == "rm_lane_ctas") {
        if (value < 0 || value > 8 * SA_MAX_CTAS) {
            sa_set_error(SA_ERR_ARG, "rm_lane_ctas must be 0 (the batched grid) .. %d (got %d)", 8 * SA_MAX_CTAS,
                         value);
            return SA_ERR_ARG;
        }
        t.rm_lane_ctas = value;
        return SA_OK;
    }
    if (n == "call_lane_ctas") {
        if (value < 0 || value > 8 * SA_MAX_CTAS) {
            sa_set_error(SA_ERR_ARG, "call_lane_ctas must be 0 (half the batched grid) .. %d (got %d)",
                         8 * SA_MAX_CTAS, value);
            return SA_ERR_ARG;
        }
        t.call_lane_ctas = value;
        return SA_OK;
    }
    if (n == "substeps") {
        if (value < 1 || value > 8) {
            sa_set_error(SA_ERR_ARG, "substeps must be 1..8 (got %d)", value);
            return SA_ERR_ARG;
        }
        t.substeps = value;
        return SA_OK;
    }
    sa_set_error(SA_ERR_ARG, "unknown tuning parameter %s", name);
    return SA_ERR_ARG;
}

int sa_get_tuning_param(const char* name) {
    if (!name) return SA_ERR_ARG;
    const SaTuning& t = G().tuning;
    const std::string n = name;
    if (n == "lane_cap") return t.lane_cap;
    if (n == "ext_ctas_per_sm") return t.ext_ctas_per_sm;
    if (n == "tile_hits") return t.tile_hits;
    if (n == "step_bases") return t.step_bases;
    if (n == "substeps") return t.substeps;
    if (n == "range_ctas") return t.range_ctas;
    if (n == "call_range_ctas") return t.call_range_ctas;
    if (n == "call_lane_ctas") return t.call_lane_ctas;
    if (n == "switch_now") return t.switch_now;
    if (n == "rm_switch_now") return t.rm_switch_now;

    if (n == "rm_substeps") return t.rm_substeps;
    if (n == "rm_lane_ctas") return t.rm_lane_ctas;
    return SA_ERR_ARG;
}

int sa_set_tuning(int lane_cap, int ext_block, int ext_ctas_per_sm, int tile_hits) {
    invalidate_graphs();
    SaTuning& t = G().tuning;
    if (lane_cap >= 0 && (lane_cap % 8 || lane_cap < 8)) {
        sa_set_error(SA_ERR_ARG, "lane_cap must be a positive multiple of 8 (got %d)", lane_cap);
        return SA_ERR_ARG;
    }
    if (ext_block >= 0 && ext_block != 256) {
        sa_set_error(SA_ERR_ARG, "ext_block must be 256: the lane kernel is compiled for 256 threads");
        return SA_ERR_ARG;
    }
    if (ext_ctas_per_sm >= 0 && (ext_ctas_per_sm < 2 || ext_ctas_per_sm > 4)) {
        sa_set_error(SA_ERR_ARG, "ext_ctas_per_sm must be 2, 3 or 4 (got %d)", ext_ctas_per_sm);
        return SA_ERR_ARG;
    }
    if (tile_hits >= 0 && (tile_hits < 32 || tile_hits > 1024)) {
        // the lane kernel keeps 8 warp tiles of 24 bytes per hit in shared memory
        sa_set_error(SA_ERR_ARG, "tile_hits must be in [32, 1024] (got %d)", tile_hits);
        return SA_ERR_ARG;
    }
    if (lane_cap >= 0) t.lane_cap = lane_cap;
    if (ext_block >= 0) t.ext_block = ext_block;
    if (ext_ctas_per_sm >= 0) t.ext_ctas_per_sm = ext_ctas_per_sm;
    if (tile_hits >= 0) t.tile_hits = tile_hits;
    return SA_OK;
}

}  // extern "C"
