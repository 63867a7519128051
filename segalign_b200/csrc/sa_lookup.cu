// sa_lookup.cu — seed lookup: bucket bounds per seed, hit prefix, compaction
// of seeds that have hits, and the MAX_HITS iteration split.
//
// Reference behaviour restated here:
//   find_num_hits + inclusive_scan + num_hits D2H   src/seed_filter.cu:129-154, 680-684
//   MAX_HITS split (lower_bound loop)              src/seed_filter.cu:686-697
//   find_hits hit records {pos+seed_size, j+seed_size}   src/seed_filter.cu:156-202
// The reference materialises one 16-byte record per hit; here only seeds with
// hits are compacted (E = exclusive hit prefix, lo = bucket start, j), and the
// extension kernel expands hits on the fly from that list.
#include "sa_launch.h"
#include "sa_radix.cuh"

// Error codes raised on the device (SaCounters::error).
#define SA_DERR_BAD_KEY 1        // seed key outside the 4^K table
#define SA_DERR_MAX_HITS 2       // one seed holds >= MAX_HITS hits (reference UB)
#define SA_DERR_ITERS 3          // more MAX_HITS iterations than supported

__global__ void __launch_bounds__(256)
sa_k_lookup_count(const uint64_t* __restrict__ seeds, const SaCallDesc* __restrict__ desc,
                  const uint32_t* __restrict__ index, uint32_t nbuckets, uint32_t* __restrict__ s_lo,
                  uint32_t* __restrict__ s_cnt, unsigned long long* cta_a, unsigned long long* cta_b,
                  SaCounters* ctr) {
    uint64_t a, b;
    sa_cta_range(desc->num_seeds, a, b);
    unsigned long long hits = 0, nz = 0;
    for (uint64_t i = a + threadIdx.x; i < b; i += 256) {
        uint32_t key = (uint32_t)(seeds[i] >> 32);
        uint32_t lo = 0, cnt = 0;
        if (key < nbuckets) {
            uint32_t hi = __ldg(index + key);
            lo = key ? __ldg(index + key - 1) : 0u;
            cnt = hi - lo;
        } else {
            atomicCAS(&ctr->error, 0ull, (unsigned long long)SA_DERR_BAD_KEY);
        }
        s_lo[i] = lo;
        s_cnt[i] = cnt;
        hits += cnt;
        nz += cnt != 0;
    }
    __shared__ unsigned long long ws[9];
    unsigned long long tot;
    sa_block_excl_sum<unsigned long long, 256>(hits, ws, &tot);
    if (threadIdx.x == 0) cta_a[blockIdx.x] = tot;
    sa_block_excl_sum<unsigned long long, 256>(nz, ws, &tot);
    if (threadIdx.x == 0) cta_b[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(256)
sa_k_lookup_emit(const uint64_t* __restrict__ seeds, const SaCallDesc* __restrict__ desc,
                 const uint32_t* __restrict__ s_lo, const uint32_t* __restrict__ s_cnt,
                 uint64_t* __restrict__ s_P, SaSeedList cs, const unsigned long long* cta_a,
                 const unsigned long long* cta_b, SaCounters* ctr) {
    const uint64_t n = desc->num_seeds;
    uint64_t a, b;
    sa_cta_range(n, a, b);
    unsigned long long hbase = cta_a[blockIdx.x], cbase = cta_b[blockIdx.x];
    __shared__ unsigned long long ws[9];
    for (uint64_t r = a; r < b; r += 256) {
        uint64_t i = r + threadIdx.x;
        uint32_t cnt = i < b ? s_cnt[i] : 0u;
        unsigned long long th, tc;
        unsigned long long eh = sa_block_excl_sum<unsigned long long, 256>(cnt, ws, &th);
        unsigned long long ec = sa_block_excl_sum<unsigned long long, 256>(cnt != 0, ws, &tc);
        if (i < b) {
            s_P[i] = hbase + eh + cnt;  // inclusive prefix (thrust::inclusive_scan, :682)
            if (cnt) {
                uint64_t c = cbase + ec;
                cs.E[c] = hbase + eh;
                cs.lo[c] = s_lo[i];
                cs.qpos[c] = (uint32_t)(seeds[i] & 0xffffffffu);
                cs.scope[c] = (uint32_t)i;  // seed index; turned into the iteration by sa_k_scope
                cs.unit[c] = 0;
            }
        }
        hbase += th;
        cbase += tc;
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) cs.E[ctr->nnz] = ctr->num_hits;
}

// MAX_HITS iterations (src/seed_filter.cu:686-697): num_iter = num_hits/MAX_HITS + 1;
// limit[i] = lower_bound(P, lim) - 1, lim = P[limit[i]] + MAX_HITS, last limit = n-1.
__global__ void sa_k_groups(const uint64_t* __restrict__ P, const SaCallDesc* desc, uint64_t* limits,
                            SaCounters* ctr) {
    const uint64_t n = desc->num_seeds, MH = desc->max_hits, H = ctr->num_hits;
    uint64_t num_iter = MH ? H / MH + 1 : 1;
    if (num_iter > SA_MAX_ITERS) {
        atomicCAS(&ctr->error, 0ull, (unsigned long long)SA_DERR_ITERS);
        num_iter = 1;
    }
    ctr->num_iter = num_iter;
    uint64_t lim = MH;
    int64_t prev = -1;
    for (uint64_t it = 0; it + 1 < num_iter; ++it) {
        uint64_t lo = 0, hi = n;  // first index with P >= lim
        while (lo < hi) {
            uint64_t mid = (lo + hi) >> 1;
            if (P[mid] < lim) lo = mid + 1;
            else hi = mid;
        }
        int64_t pos = (int64_t)lo - 1;
        if (pos <= prev) {
            atomicCAS(&ctr->error, 0ull, (unsigned long long)SA_DERR_MAX_HITS);
            pos = prev + 1;
        }
        limits[it] = (uint64_t)pos;
        lim = P[pos] + MH;
        prev = pos;
    }
    limits[num_iter - 1] = n ? n - 1 : 0;
}

// Seed index -> iteration: the first iteration whose limit is >= the seed index.
__global__ void sa_k_scope(SaSeedList cs, const uint64_t* __restrict__ limits, SaCounters* ctr) {
    const uint64_t nnz = ctr->nnz, it = ctr->num_iter;
    for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < nnz; c += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t s = cs.scope[c];
        uint32_t g = 0;
        while (g + 1 < it && (uint64_t)s > limits[g]) ++g;
        cs.scope[c] = g;
    }
}

void sa_launch_lookup_seeds(SaWork& w, const uint32_t* index, uint32_t nbuckets, const SaParams& p, int G,
                            cudaStream_t st) {
    sa_k_lookup_count<<<G, 256, 0, st>>>(w.seeds, w.desc, index, nbuckets, w.s_lo, w.s_cnt, w.cta_a, w.cta_b, w.ctr);
    sa_note_launch();
    sa_k_scan_partials<<<1, 1024, 0, st>>>(w.cta_a, w.cta_b, G, &w.ctr->num_hits, &w.ctr->nnz);
    sa_note_launch();
    sa_k_lookup_emit<<<G, 256, 0, st>>>(w.seeds, w.desc, w.s_lo, w.s_cnt, w.s_P, w.cs, w.cta_a, w.cta_b, w.ctr);
    sa_note_launch();
    sa_k_groups<<<1, 1, 0, st>>>(w.s_P, w.desc, w.limits, w.ctr);
    sa_note_launch();
    sa_k_scope<<<148 * 4, 256, 0, st>>>(w.cs, w.limits, w.ctr);
    sa_note_launch();
}

// ---------------------------------------------------------------------------
// Batched lookup over "seed slots".  Unit u covers query positions
// [q_start, q_end) of one strand; each position owns S = 1 (+K with
// transitions) consecutive slots in the order the host seeder emits seed
// words (key, then key ^ (2 << 2t), t = 0..K-1).  Positions whose window is
// not all uppercase ACGT produce no seed in the reference; here their slots
// simply have no hits, which leaves every hit and its MAX_HITS iteration
// unchanged (iterations are defined by the hit prefix only).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t sa_find_unit(const SaBatchUnit* __restrict__ bu, uint32_t n, uint64_t slot) {
    uint32_t lo = 0, hi = n;  // last unit with slot_begin <= slot
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (bu[mid].slot_begin <= slot) lo = mid;
        else hi = mid;
    }
    return lo;
}

// The unit holding slot s, kept per thread: a thread's slots only increase,
// so the binary search runs only when s passes the current unit's end.
struct SaUnitCursor {
    uint32_t u = 0;
    uint64_t end = 0;  // one past the unit's last slot (0: not located yet)
    SaBatchUnit B{};
    __device__ __forceinline__ void seek(const SaBatchUnit* __restrict__ bu, uint32_t nu, uint64_t n, uint64_t s) {
        if (s < end) return;
        u = sa_find_unit(bu, nu, s);
        B = bu[u];
        end = (u + 1 < nu) ? bu[u + 1].slot_begin : n;
    }
};

// Per CTA: hits and hit-bearing slots of its range.  A thread takes
// SA_COUNT_ITEMS slots 256 apart per round and issues all their key loads,
// then all their bucket-bound loads, then the stores (the loads of one round
// are in flight together).
#define SA_COUNT_ITEMS 4
__global__ void __launch_bounds__(256)
sa_k_blookup_count(const SaBatchUnit* __restrict__ bu, const SaCallDesc* __restrict__ desc,
                   const uint32_t* __restrict__ index, uint32_t nbuckets, int S,
                   uint32_t* __restrict__ s_lo, uint32_t* __restrict__ s_cnt, unsigned long long* cta_a,
                   unsigned long long* cta_b, SaCounters* ctr) {
    constexpr int J = SA_COUNT_ITEMS;
    const uint64_t n = desc->num_seeds;
    uint64_t a, b;
    sa_cta_range(n, a, b);
    const uint32_t nu = desc->num_units;
    unsigned long long hits = 0, nz = 0;
    bool bad_key = false;
    SaUnitCursor cur;
    for (uint64_t s0 = a + threadIdx.x; s0 < b; s0 += 256 * J) {
        uint32_t key[J];
#pragma unroll
        for (int j = 0; j < J; ++j) {
            const uint64_t s = s0 + 256ull * j;
            key[j] = SA_INVALID_KEY;
            if (s < b) {
                cur.seek(bu, nu, n, s);
                const SaBatchUnit& B = cur.B;
                const uint64_t off = s - B.slot_begin;
                // find_num_hits (src/seed_filter.cu:129-154) on a call's own words; a key
                // outside the table is reported (a plain call's SA_ERR_BAD_SEED), never read
                if (B.seeds) {
                    const uint32_t k = (uint32_t)(__ldg(reinterpret_cast<const unsigned long long*>(B.seeds) +
                                                        B.q_start + off) >> 32);
                    if (k >= nbuckets) bad_key = true;
                    else key[j] = k;
                } else {
                    const uint32_t v = (uint32_t)(off % S);
                    const uint32_t k = __ldg(B.keys + B.q_start + (uint32_t)(off / S));
                    key[j] = (k == SA_INVALID_KEY || !v) ? k : k ^ (2u << (2 * (v - 1)));
                }
            }
        }
        uint32_t lo[J], hi[J];
#pragma unroll
        for (int j = 0; j < J; ++j) {
            lo[j] = hi[j] = 0;
            if (key[j] < nbuckets) {
                hi[j] = __ldg(index + key[j]);
                lo[j] = key[j] ? __ldg(index + key[j] - 1) : 0u;
            }
        }
#pragma unroll
        for (int j = 0; j < J; ++j) {
            const uint64_t s = s0 + 256ull * j;
            if (s < b) {
                const uint32_t c = hi[j] - lo[j];
                s_lo[s] = lo[j];
                s_cnt[s] = c;
                hits += c;
                nz += c != 0;
            }
        }
    }
    if (bad_key) atomicCAS(&ctr->error, 0ull, (unsigned long long)SA_DERR_BAD_KEY);
    __shared__ unsigned long long ws[9];
    unsigned long long tot;
    sa_block_excl_sum<unsigned long long, 256>(hits, ws, &tot);
    if (threadIdx.x == 0) cta_a[blockIdx.x] = tot;
    sa_block_excl_sum<unsigned long long, 256>(nz, ws, &tot);
    if (threadIdx.x == 0) cta_b[blockIdx.x] = tot;
}

// Compaction of hit-bearing slots; also records each unit's hit range
// [unit_hit_base, unit_hit_end) in the global hit prefix.  A round covers
// 256 x SA_EMIT_ITEMS consecutive slots, SA_EMIT_ITEMS per thread, with one
// block scan of the packed (hits << 16 | hit-bearing slots) per round (a
// round has at most 2^12 hit-bearing slots, so the low field never carries).
#define SA_EMIT_ITEMS 4
__global__ void __launch_bounds__(256)
sa_k_blookup_emit(const SaBatchUnit* __restrict__ bu, const SaCallDesc* __restrict__ desc, int S,
                  const uint32_t* __restrict__ s_lo, const uint32_t* __restrict__ s_cnt, SaSeedList cs,
                  const unsigned long long* cta_a, const unsigned long long* cta_b, unsigned long long* unit_hit_base,
                  unsigned long long* unit_hit_end, SaCounters* ctr) {
    static_assert(256 * SA_EMIT_ITEMS < (1 << 16), "packed scan field");
    const uint64_t n = desc->num_seeds;
    const uint32_t nu = desc->num_units;
    uint64_t a, b;
    sa_cta_range(n, a, b);
    unsigned long long hbase = cta_a[blockIdx.x], cbase = cta_b[blockIdx.x];
    __shared__ unsigned long long ws[9];
    SaUnitCursor cur;
    // each round's counts and bucket starts are loaded during the round before
    uint32_t cnt[SA_EMIT_ITEMS], lo[SA_EMIT_ITEMS];
    auto fetch = [&](uint64_t r, uint32_t* c, uint32_t* l) {
        const uint64_t s0 = r + (uint64_t)threadIdx.x * SA_EMIT_ITEMS;
#pragma unroll
        for (int k = 0; k < SA_EMIT_ITEMS; ++k) {
            const bool in = s0 + k < b;
            c[k] = in ? s_cnt[s0 + k] : 0u;
            l[k] = in ? s_lo[s0 + k] : 0u;
        }
    };
    fetch(a, cnt, lo);
    for (uint64_t r = a; r < b; r += 256 * SA_EMIT_ITEMS) {
        const uint64_t s0 = r + (uint64_t)threadIdx.x * SA_EMIT_ITEMS;
        uint32_t ncnt[SA_EMIT_ITEMS], nlo[SA_EMIT_ITEMS];
        fetch(r + 256 * SA_EMIT_ITEMS, ncnt, nlo);
        unsigned long long mine = 0;
#pragma unroll
        for (int k = 0; k < SA_EMIT_ITEMS; ++k) mine += ((unsigned long long)cnt[k] << 16) | (cnt[k] != 0);
        unsigned long long tot;
        const unsigned long long e = sa_block_excl_sum<unsigned long long, 256>(mine, ws, &tot);
        unsigned long long eh = hbase + (e >> 16), ec = cbase + (e & 0xffffu);
#pragma unroll
        for (int k = 0; k < SA_EMIT_ITEMS; ++k) {
            const uint64_t s = s0 + k;
            if (s < b) {
                cur.seek(bu, nu, n, s);
                const SaBatchUnit& B = cur.B;
                if (s == B.slot_begin) unit_hit_base[cur.u] = eh;
                if (s + 1 == cur.end) unit_hit_end[cur.u] = eh + cnt[k];
                if (cnt[k]) {
                    cs.E[ec] = eh;
                    cs.lo[ec] = lo[k];
                    cs.qpos[ec] = B.seeds ? (uint32_t)__ldg(reinterpret_cast<const unsigned long long*>(B.seeds) +
                                                            B.q_start + (s - B.slot_begin))
                                          : B.q_start + (uint32_t)((s - B.slot_begin) / S);
                    cs.unit[ec] = B.unit;
                    cs.scope[ec] = cur.u << 4;  // (batch unit, iteration 0); sa_k_bscope sets later iterations
                    ++ec;
                }
                eh += cnt[k];
            }
        }
        hbase += tot >> 16;
        cbase += tot & 0xffffu;
#pragma unroll
        for (int k = 0; k < SA_EMIT_ITEMS; ++k) {
            cnt[k] = ncnt[k];
            lo[k] = nlo[k];
        }
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) cs.E[ctr->nnz] = ctr->num_hits;
}

// Per unit: MAX_HITS iteration boundaries in hit space (relative to the unit's
// first hit).  The reference's limit_pos[i] = lower_bound(P, lim) - 1 selects
// the last seed whose inclusive prefix is < lim; its prefix is the boundary.
__global__ void sa_k_bgroups(const SaCallDesc* __restrict__ desc, SaSeedList cs,
                             const unsigned long long* __restrict__ unit_hit_base,
                             const unsigned long long* __restrict__ unit_hit_end, unsigned long long* bounds,
                             uint32_t* unit_iters, SaCounters* ctr) {
    const uint32_t nu = desc->num_units;
    const uint64_t MH = desc->max_hits, nnz = ctr->nnz;
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < nu; u += gridDim.x * blockDim.x) {
        const uint64_t base = unit_hit_base[u], H = unit_hit_end[u] - base;
        uint64_t it = MH ? H / MH + 1 : 1;
        if (it > SA_BATCH_ITERS) {
            atomicCAS(&ctr->error, 0ull, 3ull);
            it = 1;
        }
        unit_iters[u] = (uint32_t)it;
        unsigned long long* B = bounds + (uint64_t)u * SA_BATCH_ITERS;
        if (it > 1) {
            // compacted seeds of the unit: c with base <= E[c] < base + H
            uint64_t lo = 0, hi = nnz;
            while (lo < hi) {
                uint64_t m = (lo + hi) >> 1;
                if (cs.E[m] < base) lo = m + 1;
                else hi = m;
            }
            const uint64_t c0 = lo;
            hi = nnz;
            while (lo < hi) {
                uint64_t m = (lo + hi) >> 1;
                if (cs.E[m] < base + H) lo = m + 1;
                else hi = m;
            }
            const uint64_t c1 = lo;
            uint64_t lim = MH, prev_bound = 0;
            for (uint64_t i = 0; i + 1 < it; ++i) {
                // last c in [c0, c1) with inclusive prefix E[c+1] - base < lim
                uint64_t l = c0, h = c1;
                while (l < h) {
                    uint64_t m = (l + h) >> 1;
                    if (cs.E[m + 1] - base < lim) l = m + 1;
                    else h = m;
                }
                uint64_t bnd = (l > c0) ? cs.E[l] - base : 0;  // prefix of the last qualifying seed
                if (l == c0 || bnd <= prev_bound) {
                    if (i > 0 || l == c0) atomicCAS(&ctr->error, 0ull, 2ull);
                }
                B[i] = bnd;
                prev_bound = bnd;
                lim = bnd + MH;
            }
        }
        B[it - 1] = ~0ull;
    }
}

// Compacted seed -> scope = (batch unit << 4) | iteration, for the units with
// more than one MAX_HITS iteration (the emit wrote iteration 0).  One CTA per
// such unit: its compacted seeds are those with E in [base, base + H).
__global__ void __launch_bounds__(256)
sa_k_bscope(const SaCallDesc* __restrict__ desc, SaSeedList cs, const unsigned long long* __restrict__ unit_hit_base,
            const unsigned long long* __restrict__ unit_hit_end, const unsigned long long* __restrict__ bounds,
            const uint32_t* __restrict__ unit_iters, SaCounters* ctr) {
    const uint32_t nu = desc->num_units;
    const uint64_t nnz = ctr->nnz;
    for (uint32_t u = blockIdx.x; u < nu; u += gridDim.x) {
        const uint32_t it = unit_iters[u];
        if (it <= 1) continue;
        const uint64_t base = unit_hit_base[u], H = unit_hit_end[u] - base;
        uint64_t lo = 0, hi = nnz;
        while (lo < hi) {
            const uint64_t m = (lo + hi) >> 1;
            if (cs.E[m] < base) lo = m + 1;
            else hi = m;
        }
        const uint64_t c0 = lo;
        hi = nnz;
        while (lo < hi) {
            const uint64_t m = (lo + hi) >> 1;
            if (cs.E[m] < base + H) lo = m + 1;
            else hi = m;
        }
        const unsigned long long* B = bounds + (uint64_t)u * SA_BATCH_ITERS;
        for (uint64_t c = c0 + threadIdx.x; c < lo; c += blockDim.x) {
            const uint64_t p = cs.E[c + 1] - base;
            uint32_t g = 0;
            while (g + 1 < it && p > B[g]) ++g;
            cs.scope[c] = (u << 4) | g;
        }
    }
}

void sa_launch_lookup_batch(SaWork& w, const uint32_t* index, uint32_t nbuckets, uint32_t n_bunits, const SaParams& p,
                            int G, cudaStream_t st) {
    const int S = p.transition ? 1 + p.kmer_size : 1;
    // a unit without slots (an empty window) gets the empty hit range [0, 0)
    cudaMemsetAsync(w.unit_hit_base, 0, 8ull * n_bunits, st);
    cudaMemsetAsync(w.unit_hit_end, 0, 8ull * n_bunits, st);
    sa_k_blookup_count<<<G, 256, 0, st>>>(w.bunits, w.desc, index, nbuckets, S, w.s_lo, w.s_cnt, w.cta_a, w.cta_b,
                                          w.ctr);
    sa_note_launch();
    sa_k_scan_partials<<<1, 1024, 0, st>>>(w.cta_a, w.cta_b, G, &w.ctr->num_hits, &w.ctr->nnz);
    sa_note_launch();
    sa_k_blookup_emit<<<G, 256, 0, st>>>(w.bunits, w.desc, S, w.s_lo, w.s_cnt, w.cs, w.cta_a, w.cta_b,
                                         w.unit_hit_base, w.unit_hit_end, w.ctr);
    sa_note_launch();
    const int ub = (int)std::min<uint32_t>((n_bunits + 255) / 256, 1024u);
    sa_k_bgroups<<<ub > 0 ? ub : 1, 256, 0, st>>>(w.desc, w.cs, w.unit_hit_base, w.unit_hit_end, w.bounds,
                                                  w.unit_iters, w.ctr);
    sa_note_launch();
    sa_k_bscope<<<(int)std::min<uint32_t>(std::max<uint32_t>(n_bunits, 1u), 1024u), 256, 0, st>>>(w.desc, w.cs, w.unit_hit_base, w.unit_hit_end,
                                                                      w.bounds, w.unit_iters, w.ctr);
    sa_note_launch();
}
