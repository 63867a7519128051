// sa_noalloc.cu — SeedAndFilter without any memory allocation per call.
//
// Some callers of this library cannot let it allocate device memory while
// they run: a host program that owns all device memory through its own pool
// (a caching allocator with a fixed budget, where a library's private
// cudaMalloc fragments or overruns that budget), or a latency-bound loop that
// cannot afford the device-wide synchronisation cudaMalloc and cudaFree may
// perform while other streams are busy.  sa_seed_and_filter_noalloc() serves
// them: its per-call scratch (seed words, bucket bounds, hit prefixes, the
// compacted seed list, the long-extension queue, the set of distinct HSPs,
// sort buffers, counters) is carved out of one file-scope __device__ array of fixed size,
// SA_NOALLOC_BYTES, which every GPU that loads the library holds until the
// process exits.  The result is copied into a buffer the caller provides.
//
// Set-up: the first call on a device looks up the array's device address
// with cudaGetSymbolAddress while that device is current; make that first
// call before any stream capture.  Limits: at most SA_NOALLOC_MAX_SEEDS seed
// words and SA_NOALLOC_MAX_SURVIVORS distinct HSPs per call; larger calls are
// rejected with SA_ERR_CAPACITY.  All calls share the
// array and it keeps the last call's contents: each call clears its counters
// first, and calls run one at a time in this process (a host lock; each call
// finishes on the GPU before it returns).  Calls that overlapped on the GPU
// would race on the shared array.
#include <cstring>
#include <mutex>

#include "../../include/segalign_b200.h"
#include "sa_launch.h"

#define SA_NOALLOC_MAX_SEEDS (1u << 18)
#define SA_NOALLOC_MAX_SURVIVORS (1u << 18)
#define SA_NOALLOC_LONG_CAP (1u << 16)
#define SA_NOALLOC_UNITS 64

namespace {

constexpr uint64_t al(uint64_t b) { return (b + 255) & ~255ull; }
constexpr uint64_t kSeeds = SA_NOALLOC_MAX_SEEDS, kSurv = SA_NOALLOC_MAX_SURVIVORS;
// Byte sizes of the carved parts, in carving order.
constexpr uint64_t kParts[] = {
    8 * kSeeds,                                          // seeds
    4 * kSeeds, 4 * kSeeds, 8 * kSeeds,                  // s_lo, s_cnt, s_P
    8 * (kSeeds + 1), 4 * (kSeeds + 1), 4 * (kSeeds + 1), 4 * (kSeeds + 1), 4 * (kSeeds + 1),  // cs
    8 * SA_MAX_CTAS, 8 * SA_MAX_CTAS, 8 * SA_MAX_ITERS,  // cta_a, cta_b, limits
    sizeof(SaLongHit) * SA_NOALLOC_LONG_CAP,             // long queue
    sizeof(SaRec) * kSurv, sizeof(SaRec) * kSurv, 4 * kSurv, 4 * kSurv,  // rec[2], scope[2]
    16 * 2 * kSurv, 4 * 2 * kSurv,                       // HSP set: keys, scores
    sizeof(SaRec) * kSurv, 4 * kSurv,                    // out, out_scope
    4 * SA_MAX_SCOPES, 4 * SA_MAX_SCOPES,                // scope_count, scope_flags
    4 * 256 * SA_SORT_MAX_DIGITS, 4 * 256 * (uint64_t)SA_MAX_CTAS + 4 * 64, 4 * (SA_SORT_MAX_DIGITS + 2),
    sizeof(SaCounters), sizeof(SaCallDesc), sizeof(SaUnit) * SA_NOALLOC_UNITS,
};
constexpr uint64_t total_bytes() {
    uint64_t t = 0;
    for (uint64_t b : kParts) t += al(b);
    return t;
}

}  // namespace

#define SA_NOALLOC_BYTES (total_bytes())

// The scratch array.  In host code this name is only a host-side stand-in:
// the device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char sa_noalloc_scratch[SA_NOALLOC_BYTES];

namespace {

std::mutex g_noalloc_mu;
constexpr int kMaxDevices = 64;
void* g_scratch_ptr[kMaxDevices] = {};
bool g_hash_clean[kMaxDevices] = {};  // the array's HSP set is known to be empty

// Per-device set-up, with `dev` current: the device address of the array.
int scratch_address(int dev, void** ptr) {
    if (dev < 0 || dev >= kMaxDevices) return SA_ERR_ARG;
    if (!g_scratch_ptr[dev]) {
        cudaError_t e = cudaGetSymbolAddress(&g_scratch_ptr[dev], sa_noalloc_scratch);
        if (e != cudaSuccess) {
            g_scratch_ptr[dev] = nullptr;
            return sa_cuda_fail(e, "cudaGetSymbolAddress(sa_noalloc_scratch)", __FILE__, __LINE__);
        }
    }
    *ptr = g_scratch_ptr[dev];
    return SA_OK;
}

void carve(void* base, SaWork& w) {
    char* at = (char*)base;
    int i = 0;
    auto take = [&](void** p) {
        *p = at;
        at += al(kParts[i++]);
    };
    std::memset(&w, 0, sizeof w);
    take((void**)&w.seeds);
    take((void**)&w.s_lo);
    take((void**)&w.s_cnt);
    take((void**)&w.s_P);
    take((void**)&w.cs.E);
    take((void**)&w.cs.lo);
    take((void**)&w.cs.qpos);
    take((void**)&w.cs.scope);
    take((void**)&w.cs.unit);
    take((void**)&w.cta_a);
    take((void**)&w.cta_b);
    take((void**)&w.limits);
    take((void**)&w.long_q);
    take((void**)&w.rec[0]);
    take((void**)&w.rec[1]);
    take((void**)&w.scope[0]);
    take((void**)&w.scope[1]);
    take((void**)&w.hset.keys);
    take((void**)&w.hset.score);
    take((void**)&w.out);
    take((void**)&w.out_scope);
    take((void**)&w.scope_count);
    take((void**)&w.scope_flags);
    take((void**)&w.sort_hist);
    take((void**)&w.sort_cta_hist);
    take((void**)&w.sort_in_buf);
    take((void**)&w.ctr);
    take((void**)&w.desc);
    take((void**)&w.units);
    w.seed_cap = kSeeds;
    w.surv_cap = kSurv;
    w.long_cap = SA_NOALLOC_LONG_CAP;
    // the HSP set's list of claimed slots lives in rec[1], free until the sort
    w.hset.used = reinterpret_cast<unsigned long long*>(w.rec[1]);
    w.hset.used_cap = kSurv;
}

}  // namespace

extern "C" {

// No counterpart in the reference: SeedAndFilter (src/seed_filter.cu:654-778
// semantics, same output as sa_seed_and_filter) with no allocation per call.
int sa_seed_and_filter_noalloc(const uint64_t* seeds, uint32_t num_seeds, int rev, uint32_t buffer, sa_segment* out,
                               uint64_t out_cap, uint64_t* out_len) {
    if (!out_len || (num_seeds && !seeds) || (!out && out_cap)) return SA_ERR_ARG;
    SaResidentView v;
    int r = sa_resident_view(buffer, &v);
    if (r != SA_OK) return r;
    const uint32_t* q = v.q_packed[rev ? 1 : 0];
    if (!q) {
        sa_set_error(SA_ERR_STATE, "query buffer %u is not resident", buffer);
        return SA_ERR_STATE;
    }
    if (num_seeds > v.max_seeds) {
        sa_set_error(SA_ERR_MAX_SEEDS, "%u seeds exceed MAX_SEEDS = %llu", num_seeds, (unsigned long long)v.max_seeds);
        return SA_ERR_MAX_SEEDS;
    }
    if (num_seeds > SA_NOALLOC_MAX_SEEDS) {
        sa_set_error(SA_ERR_CAPACITY, "%u seeds exceed the no-allocation limit of %u seeds per call", num_seeds,
                     SA_NOALLOC_MAX_SEEDS);
        return SA_ERR_CAPACITY;
    }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    SA_CUDA_OK(cudaSetDevice(v.dev));
    void* base = nullptr;
    r = scratch_address(v.dev, &base);
    if (r != SA_OK) return r;
    SaWork w;
    carve(base, w);
    w.hash_clean = g_hash_clean[v.dev];
    g_hash_clean[v.dev] = false;  // set again once this call is seen to complete
    cudaStream_t st = cudaStreamPerThread;
    SaCallDesc desc{};
    desc.num_seeds = num_seeds;
    desc.max_hits = v.max_hits;
    desc.num_units = 1;
    desc.num_scopes_max = SA_MAX_ITERS;
    SaUnit unit{};
    unit.q_packed = q;
    unit.q_len = v.q_len;
    uint32_t flags[SA_MAX_ITERS];
    for (int i = 0; i < SA_MAX_ITERS; ++i) flags[i] = rev ? 1u : 0u;
    SA_CUDA_OK(cudaMemsetAsync(w.ctr, 0, sizeof(SaCounters), st));
    SA_CUDA_OK(cudaMemcpyAsync(w.seeds, seeds, 8ull * num_seeds, cudaMemcpyHostToDevice, st));
    SA_CUDA_OK(cudaMemcpyAsync(w.desc, &desc, sizeof desc, cudaMemcpyHostToDevice, st));
    SA_CUDA_OK(cudaMemcpyAsync(w.units, &unit, sizeof unit, cudaMemcpyHostToDevice, st));
    SA_CUDA_OK(cudaMemcpyAsync(w.scope_flags, flags, sizeof flags, cudaMemcpyHostToDevice, st));
    // the grids and lane-kernel settings of a plain call (sa_seed_and_filter)
    const SaCallGrids cg = sa_call_grids(v.tuning, v.num_sms, 0);
    const int G = cg.range_ctas;
    sa_launch_lookup_seeds(w, v.index, (uint32_t)v.nbuckets, v.params, G, st);
    if (!w.hash_clean) sa_launch_hash_clear(w, st);
    w.hash_clean = false;
    sa_launch_hash_init(w, false, st);
    SaExtendArgs xa;
    xa.ref = v.ref;
    xa.ref_len = v.ref_len;
    xa.pos_table = v.pos;
    xa.seed_size = (uint32_t)v.params.seed_size;
    xa.xdrop = v.params.xdrop;
    xa.hspthresh = v.params.hspthresh;
    xa.noentropy = v.params.noentropy;
    sa_launch_extend_lane(w, xa, v.params, cg.lane_tuning, v.num_sms, st, cg.lane_ctas);
    sa_launch_extend_warp(w, xa, v.params, v.tuning, v.num_sms, st);
    sa_launch_dedup(w, 0, 0, G, st);
    SA_CUDA_OK(cudaGetLastError());
    SaCounters c;
    SA_CUDA_OK(cudaMemcpyAsync(&c, w.ctr, sizeof c, cudaMemcpyDeviceToHost, st));
    SA_CUDA_OK(cudaStreamSynchronize(st));
    sa_note_hash_state(w, c);
    g_hash_clean[v.dev] = w.hash_clean;
    if (c.hash_overflow || c.error == 4) {
        sa_set_error(SA_ERR_CAPACITY, "more than %u distinct HSPs (no-allocation limit)", SA_NOALLOC_MAX_SURVIVORS);
        return SA_ERR_CAPACITY;
    }
    if (c.error) return sa_map_device_error(c.error);
    const uint64_t nh = c.uniq_count;
    *out_len = nh + 1;
    if (nh + 1 > out_cap) {
        sa_set_error(SA_ERR_CAPACITY, "output needs %llu records, buffer holds %llu", (unsigned long long)(nh + 1),
                     (unsigned long long)out_cap);
        return SA_ERR_CAPACITY;
    }
    if (nh) SA_CUDA_OK(cudaMemcpyAsync(out + 1, w.out, nh * sizeof(SaRec), cudaMemcpyDeviceToHost, st));
    SA_CUDA_OK(cudaStreamSynchronize(st));
    out[0].ref_start = 0;
    out[0].query_start = 0;
    out[0].len = (uint32_t)nh;
    out[0].score = (int32_t)(uint32_t)c.num_hits;
    return SA_OK;
}

}  // extern "C"
