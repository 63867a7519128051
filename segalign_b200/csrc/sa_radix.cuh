// sa_radix.cuh — stable LSD radix sort (8-bit digits) with device-resident
// item counts, plus the block/warp scan helpers used by the range-partitioned
// kernels.
//
// Every kernel here is range-partitioned: CTA c of a G-CTA grid owns items
// [n*c/G, n*(c+1)/G), with n read from device memory, so a whole call can be
// launched without host round trips.  The sort passes use only the first
// A = min(G, ceil(n / SA_RADIX_MIN_ITEMS)) CTAs, so small sorts scan small
// histograms.  One pass = up-sweep (per-CTA digit histogram), a single-CTA
// exclusive scan of the bin-major histogram [256][A], and a stable down-sweep
// scatter that ranks equal digits inside a warp with __match_any_sync and
// across warps with a per-round shared-memory prefix.
// A pass whose input buffer is recorded as -1 is skipped (all items share
// that digit), which is how the fixed-layout HSP keys avoid scattering
// constant bytes.
#pragma once
#include <cstdint>
#include "sa_internal.cuh"

#define SA_RADIX_BLOCK 256
#define SA_RADIX_MIN_ITEMS 512  // items per active CTA of a sort pass (at least)

__device__ __forceinline__ void sa_cta_range(uint64_t n, uint64_t& a, uint64_t& b) {
    const uint64_t G = gridDim.x, c = blockIdx.x;
    a = (n * c) / G;
    b = (n * (c + 1)) / G;
}

// Active CTAs of a sort pass over n items on a G-CTA grid.
__host__ __device__ __forceinline__ uint32_t sa_radix_active(uint64_t n, uint32_t G) {
    const uint64_t want = (n + SA_RADIX_MIN_ITEMS - 1) / SA_RADIX_MIN_ITEMS;
    return want == 0 ? 1u : (want < G ? (uint32_t)want : G);
}

// Range of CTA blockIdx.x among the A active CTAs (empty for the others).
__device__ __forceinline__ void sa_radix_range(uint64_t n, uint32_t A, uint64_t& a, uint64_t& b) {
    const uint64_t c = blockIdx.x;
    if (c >= A) {
        a = b = 0;
        return;
    }
    a = (n * c) / A;
    b = (n * (c + 1)) / A;
}

// Inclusive warp scan (sum).
template <class T>
__device__ __forceinline__ T sa_warp_incl_sum(T v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Exclusive block scan (sum) for blockDim.x == NT (multiple of 32, <= 1024).
// `ws` must hold NT/32 + 1 elements.  Returns the exclusive prefix; *total gets the sum.
template <class T, int NT>
__device__ __forceinline__ T sa_block_excl_sum(T v, T* ws, T* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = NT / 32;
    T incl = sa_warp_incl_sum(v);
    if (lane == 31) ws[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        T x = lane < NW ? ws[lane] : T(0);
        T xi = sa_warp_incl_sum(x);
        if (lane < NW) ws[lane] = xi - x;
        if (lane == NW - 1) ws[NW] = xi;
    }
    __syncthreads();
    T r = ws[warp] + incl - v;
    *total = ws[NW];
    __syncthreads();
    return r;
}

// Exclusive scan of per-CTA partials a[G], b[G] (G <= 1024) in place by one
// CTA of 1024 threads; totals are written to *ta, *tb.
__global__ void sa_k_scan_partials(unsigned long long* a, unsigned long long* b, int G,
                                   unsigned long long* ta, unsigned long long* tb);

// Exclusive scan of the bin-major histogram [256][A] in place (one CTA of
// 1024), A = sa_radix_active(*d_n, G).
__global__ void sa_k_radix_scan(unsigned int* hist, int G, const int* in_buf, int pass,
                                const unsigned long long* d_n);

struct SaRadixCtl {
    const unsigned long long* d_n;  // item count
    const int* in_buf;              // [passes]: input buffer of each pass, -1 = skip
};

// Ops must provide:
//   struct Ctx;  struct Item;  (one item: its key and payload)
//   struct Pass;  (what selects the digit of one pass, resolved once per kernel)
//   static __device__ Pass pass_of(const Ctx&, int pass);
//   static __device__ Item load(const Ctx&, int buf, uint64_t i);
//   static __device__ uint32_t digit_of(const Pass&, const Item&);
//   static __device__ void store(const Ctx&, int buf, const Item&, uint32_t dst);  (into buffer buf ^ 1)
template <class Ops>
__global__ void __launch_bounds__(SA_RADIX_BLOCK)
sa_k_radix_up(typename Ops::Ctx ctx, int pass, SaRadixCtl ctl, unsigned int* hist) {
    const int buf = ctl.in_buf[pass];
    if (buf < 0) return;
    const uint64_t n = *ctl.d_n;
    const uint32_t A = sa_radix_active(n, gridDim.x);
    if (blockIdx.x >= A) return;
    __shared__ unsigned int h[256];
    const int t = threadIdx.x;
    h[t] = 0;
    __syncthreads();
    uint64_t a, b;
    sa_radix_range(n, A, a, b);
    const typename Ops::Pass P = Ops::pass_of(ctx, pass);
    for (uint64_t i = a + t; i < b; i += SA_RADIX_BLOCK) atomicAdd(&h[Ops::digit_of(P, Ops::load(ctx, buf, i))], 1u);
    __syncthreads();
    hist[(uint64_t)t * A + blockIdx.x] = h[t];
}

// Down-sweep: tiles of SA_RADIX_TILE = 256 x SA_RADIX_ITEMS items.  Warp w
// ranks the tile's items [w * 32 * ITEMS, (w + 1) * 32 * ITEMS) row by row
// (coalesced loads, __match_any_sync within a row, a per-warp digit count
// carried across rows); per-digit warp prefixes and the tile's digit starts
// then place every item in digit order in shared memory, and the tile is
// written back in that order, so items of one digit leave as runs of
// consecutive addresses.  Items keep their input order within a digit
// (stable).
#ifndef SA_RADIX_ITEMS
#define SA_RADIX_ITEMS 4
#endif
#define SA_RADIX_TILE (SA_RADIX_BLOCK * SA_RADIX_ITEMS)

template <class Ops>
__global__ void __launch_bounds__(SA_RADIX_BLOCK)
sa_k_radix_down(typename Ops::Ctx ctx, int pass, SaRadixCtl ctl, const unsigned int* hist) {
    constexpr int NWARP = SA_RADIX_BLOCK / 32;
    constexpr int K = SA_RADIX_ITEMS;
    using Item = typename Ops::Item;
    const int buf = ctl.in_buf[pass];
    if (buf < 0) return;
    const uint64_t n = *ctl.d_n;
    const uint32_t A = sa_radix_active(n, gridDim.x);
    if (blockIdx.x >= A) return;
    __shared__ unsigned int offs[256];           // next output index of each digit (this CTA)
    __shared__ unsigned int wcnt[NWARP][256];    // per-warp digit counts, then their exclusive prefixes
    __shared__ unsigned int tstart[256];         // tile-local start of each digit
    __shared__ unsigned int ws[NWARP + 1];
    __shared__ Item stage[SA_RADIX_TILE];
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    offs[t] = hist[(uint64_t)t * A + blockIdx.x];
    uint64_t a, b;
    sa_radix_range(n, A, a, b);
    const uint32_t lt = sa_lanemask_lt();
    const typename Ops::Pass P = Ops::pass_of(ctx, pass);
    for (uint64_t base = a; base < b; base += SA_RADIX_TILE) {
#pragma unroll
        for (int w = 0; w < NWARP; ++w) wcnt[w][t] = 0;
        __syncthreads();
        Item it[K];
        uint32_t d[K], r[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const uint64_t i = base + (uint64_t)warp * 32 * K + (uint64_t)k * 32 + lane;
            const bool valid = i < b;
            if (valid) it[k] = Ops::load(ctx, buf, i);
            d[k] = valid ? Ops::digit_of(P, it[k]) : 256u;
        }
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const uint32_t peers = __match_any_sync(0xffffffffu, d[k]);
            const uint32_t rank = __popc(peers & lt);
            const bool valid = d[k] < 256u;
            r[k] = valid ? wcnt[warp][d[k]] + rank : 0u;
            __syncwarp();
            if (valid && rank == 0) wcnt[warp][d[k]] += __popc(peers);
            __syncwarp();
        }
        __syncthreads();
        // digit t: prefixes over the warps, the tile's count, and its start in the tile
        unsigned int run = 0;
#pragma unroll
        for (int w = 0; w < NWARP; ++w) {
            const unsigned int c = wcnt[w][t];
            wcnt[w][t] = run;
            run += c;
        }
        unsigned int tot;
        tstart[t] = sa_block_excl_sum<unsigned int, SA_RADIX_BLOCK>(run, ws, &tot);
        __syncthreads();
#pragma unroll
        for (int k = 0; k < K; ++k)
            if (d[k] < 256u) stage[tstart[d[k]] + wcnt[warp][d[k]] + r[k]] = it[k];
        __syncthreads();
        const uint32_t tile_n = (uint32_t)min((uint64_t)SA_RADIX_TILE, b - base);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const uint32_t s = (uint32_t)k * SA_RADIX_BLOCK + t;
            if (s < tile_n) {
                const Item x = stage[s];
                const uint32_t dd = Ops::digit_of(P, x);
                Ops::store(ctx, buf, x, offs[dd] + (s - tstart[dd]));
            }
        }
        __syncthreads();
        offs[t] += run;
    }
}
