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
//   static __device__ uint32_t digit(const Ctx&, int buf, uint64_t i, int pass);
//   static __device__ Item load(const Ctx&, int buf, uint64_t i);
//   static __device__ uint32_t digit_of(const Ctx&, const Item&, int pass);
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
    for (uint64_t i = a + t; i < b; i += SA_RADIX_BLOCK) atomicAdd(&h[Ops::digit(ctx, buf, i, pass)], 1u);
    __syncthreads();
    hist[(uint64_t)t * A + blockIdx.x] = h[t];
}

template <class Ops>
__global__ void __launch_bounds__(SA_RADIX_BLOCK)
sa_k_radix_down(typename Ops::Ctx ctx, int pass, SaRadixCtl ctl, const unsigned int* hist) {
    const int buf = ctl.in_buf[pass];
    if (buf < 0) return;
    const uint64_t n = *ctl.d_n;
    const uint32_t A = sa_radix_active(n, gridDim.x);
    if (blockIdx.x >= A) return;
    __shared__ unsigned int offs[256];
    __shared__ unsigned int wcnt[SA_RADIX_BLOCK / 32][256];
    const int t = threadIdx.x, warp = t >> 5;
    offs[t] = hist[(uint64_t)t * A + blockIdx.x];
#pragma unroll
    for (int w = 0; w < SA_RADIX_BLOCK / 32; ++w) wcnt[w][t] = 0;
    __syncthreads();
    uint64_t a, b;
    sa_radix_range(n, A, a, b);
    const uint32_t lt = sa_lanemask_lt();
    // Items are loaded one round ahead, so that the load of round r + 1
    // overlaps the ranking and scatter of round r.
    typename Ops::Item cur{}, nxt{};
    if (a + t < b) cur = Ops::load(ctx, buf, a + t);
    for (uint64_t base = a; base < b; base += SA_RADIX_BLOCK) {
        const uint64_t i = base + t;
        const bool valid = i < b;
        if (i + SA_RADIX_BLOCK < b) nxt = Ops::load(ctx, buf, i + SA_RADIX_BLOCK);
        const uint32_t d = valid ? Ops::digit_of(ctx, cur, pass) : 256u;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t rank = __popc(peers & lt);
        if (valid && rank == 0) wcnt[warp][d] = __popc(peers);
        __syncthreads();
        uint32_t run = offs[t];
#pragma unroll
        for (int w = 0; w < SA_RADIX_BLOCK / 32; ++w) {
            uint32_t c = wcnt[w][t];
            wcnt[w][t] = run;
            run += c;
        }
        offs[t] = run;
        __syncthreads();
        if (valid) Ops::store(ctx, buf, cur, wcnt[warp][d] + rank);
        cur = nxt;
        __syncthreads();
#pragma unroll
        for (int w = 0; w < SA_RADIX_BLOCK / 32; ++w) wcnt[w][t] = 0;
        __syncthreads();
    }
}
