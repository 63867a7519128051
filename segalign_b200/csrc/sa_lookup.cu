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
    sa_k_scan_partials<<<1, 1024, 0, st>>>(w.cta_a, w.cta_b, G, &w.ctr->num_hits, &w.ctr->nnz);
    sa_k_lookup_emit<<<G, 256, 0, st>>>(w.seeds, w.desc, w.s_lo, w.s_cnt, w.s_P, w.cs, w.cta_a, w.cta_b, w.ctr);
    sa_k_groups<<<1, 1, 0, st>>>(w.s_P, w.desc, w.limits, w.ctr);
    sa_k_scope<<<148 * 4, 256, 0, st>>>(w.cs, w.limits, w.ctr);
}
