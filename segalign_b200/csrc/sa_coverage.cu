// sa_coverage.cu — repeat-masker coverage runs on the GPU.
//
// Reference: repeat_masker_src/seeder.cpp:151-186.  For each interval, every
// HSP adds one to a uint8 count at block positions query_start ..
// query_start + len - 1 (counts wrap at 256); the interval's runs are the
// maximal stretches of positions with count >= M; a run still open at the
// block end is not reported (the reference only closes a run in its else
// branch).
//
// Here the counts over the span the HSPs cover are a prefix sum of a
// difference array: +1 at each HSP start, -1 at each end (atomics), then a
// two-level scan (per-CTA sums, one CTA scans the sums, each CTA rescans its
// tile with its prefix).  The pass that rescans marks run boundaries, the
// positions where (count & 255) >= M changes, and appends them to a list;
// the host sorts that list and pairs it into runs.  Positions outside the
// span have count 0, so they are never in a run when M >= 1.
#include <algorithm>
#include <mutex>
#include <vector>

#include "sa_host_internal.h"
#include "sa_launch.h"

namespace {

constexpr int kCovThreads = 1024;
constexpr int kCovPer = 8;                          // positions per thread
constexpr int kCovTile = kCovThreads * kCovPer;     // positions per CTA

// Exclusive prefix sum over the CTA (1024 threads); *total = CTA sum.
__device__ int sa_cta_excl_scan(int v, int* total) {
    __shared__ int warp_sums[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_sums[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int s = warp_sums[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += t;
        }
        warp_sums[lane] = s;  // inclusive over warps
    }
    __syncthreads();
    const int before = wid ? warp_sums[wid - 1] : 0;
    *total = warp_sums[31];
    __syncthreads();
    return before + incl - v;
}

__global__ void sa_k_cov_diff(const uint2* __restrict__ hsp, uint64_t n, uint32_t lo, uint64_t span,
                              int* __restrict__ diff) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint2 h = hsp[i];  // (query_start, len)
        if (h.y == 0) continue;  // covers no position
        atomicAdd(&diff[h.x - lo], 1);
        const uint64_t e = (uint64_t)h.x + h.y - lo;
        if (e < span) atomicAdd(&diff[e], -1);
    }
}

__global__ void __launch_bounds__(kCovThreads) sa_k_cov_tile_sums(const int* __restrict__ diff, uint64_t span,
                                                                  int* __restrict__ sums) {
    const uint64_t base = (uint64_t)blockIdx.x * kCovTile + (uint64_t)threadIdx.x * kCovPer;
    int s = 0;
#pragma unroll
    for (int k = 0; k < kCovPer; ++k)
        if (base + k < span) s += diff[base + k];
    int total;
    sa_cta_excl_scan(s, &total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// One CTA: exclusive prefix of the tile sums, in place.
__global__ void __launch_bounds__(kCovThreads) sa_k_cov_scan_sums(int* __restrict__ sums, uint32_t n) {
    const uint32_t per = (n + kCovThreads - 1) / kCovThreads;
    const uint32_t a = threadIdx.x * per, b = min(n, a + per);
    int s = 0;
    for (uint32_t i = a; i < b; ++i) s += sums[i];
    int total;
    int run = sa_cta_excl_scan(s, &total);
    for (uint32_t i = a; i < b; ++i) {
        const int v = sums[i];
        sums[i] = run;
        run += v;
    }
}

__global__ void __launch_bounds__(kCovThreads) sa_k_cov_bounds(const int* __restrict__ diff, uint64_t span,
                                                               const int* __restrict__ prefix, uint32_t lo, uint32_t M,
                                                               uint32_t* __restrict__ bnd,
                                                               unsigned long long* __restrict__ n_bnd, uint64_t cap) {
    const uint64_t base = (uint64_t)blockIdx.x * kCovTile + (uint64_t)threadIdx.x * kCovPer;
    int d[kCovPer];
    int s = 0;
#pragma unroll
    for (int k = 0; k < kCovPer; ++k) {
        d[k] = base + k < span ? diff[base + k] : 0;
        s += d[k];
    }
    int total;
    int count = prefix[blockIdx.x] + sa_cta_excl_scan(s, &total);  // count before this thread's first position
    // position lo - 1 (or any position before the span) has count 0: in a run iff M == 0
    bool prev = ((uint32_t)(count & 255) >= M);
    if (base == 0) prev = (M == 0);
#pragma unroll
    for (int k = 0; k < kCovPer; ++k) {
        if (base + k >= span) break;
        count += d[k];
        const bool in = (uint32_t)(count & 255) >= M;
        if (in != prev) {
            const unsigned long long i = atomicAdd(n_bnd, 1ull);
            if (i < cap) bnd[i] = lo + (uint32_t)(base + k);
        }
        prev = in;
    }
}

struct CovState {
    std::mutex mu;
    int dev = -1;
    cudaStream_t st = nullptr;
    int* diff = nullptr;
    uint64_t diff_cap = 0;
    int* sums = nullptr;
    uint64_t sums_cap = 0;
    uint2* hsp = nullptr;
    uint64_t hsp_cap = 0;
    uint32_t* bnd = nullptr;
    uint64_t bnd_cap = 0;
    unsigned long long* n_bnd = nullptr;
    uint2* h_hsp = nullptr;  // pinned staging
    uint64_t h_hsp_cap = 0;
};

CovState g_cov[64];

template <typename T>
int grow(T** p, uint64_t* cap, uint64_t need) {
    if (*cap >= need) return SA_OK;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    const uint64_t n = std::max<uint64_t>(need, 1024);
    SA_CUDA_OK(cudaMalloc(p, n * sizeof(T)));
    *cap = n;
    return SA_OK;
}

}  // namespace

int sa_device_coverage_runs(const std::vector<std::pair<uint32_t, uint32_t>>& hsps, uint32_t block_len, uint32_t M,
                            std::vector<std::pair<uint32_t, uint32_t>>& runs) {
    runs.clear();
    if (M == 0 || hsps.empty()) return SA_OK;  // M == 0: one run open at the block end, never reported
    uint32_t lo = UINT32_MAX;
    uint64_t hi = 0;
    for (const auto& h : hsps) {
        if (!h.second) continue;
        lo = std::min(lo, h.first);
        hi = std::max<uint64_t>(hi, (uint64_t)h.first + h.second);
    }
    if (hi == 0) return SA_OK;
    hi = std::min<uint64_t>(hi, block_len);
    if (lo >= hi) return SA_OK;
    // positions lo .. hi; position hi (count 0) closes the last run unless it is the block end
    const uint64_t span = (hi < block_len ? hi + 1 : hi) - lo;
    int dev = 0;
    SA_CUDA_OK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return SA_ERR_ARG;
    CovState& c = g_cov[dev];
    std::lock_guard<std::mutex> lk(c.mu);
    if (!c.st) {
        SA_CUDA_OK(cudaStreamCreateWithFlags(&c.st, cudaStreamNonBlocking));
        SA_CUDA_OK(cudaMalloc(&c.n_bnd, sizeof(unsigned long long)));
    }
    const uint64_t n = hsps.size();
    const uint32_t tiles = (uint32_t)((span + kCovTile - 1) / kCovTile);
    int r = grow(&c.diff, &c.diff_cap, span);
    if (r == SA_OK) r = grow(&c.sums, &c.sums_cap, tiles);
    if (r == SA_OK) r = grow(&c.hsp, &c.hsp_cap, n);
    if (r == SA_OK) r = grow(&c.bnd, &c.bnd_cap, 2 * n + 2);  // each HSP adds at most two boundaries
    if (r != SA_OK) return r;
    if (c.h_hsp_cap < n) {
        if (c.h_hsp) cudaFreeHost(c.h_hsp);
        c.h_hsp = nullptr;
        c.h_hsp_cap = 0;
        SA_CUDA_OK(cudaMallocHost(&c.h_hsp, std::max<uint64_t>(n, 1024) * sizeof(uint2)));
        c.h_hsp_cap = std::max<uint64_t>(n, 1024);
    }
    for (uint64_t i = 0; i < n; ++i) c.h_hsp[i] = make_uint2(hsps[i].first, hsps[i].second);
    SA_CUDA_OK(cudaMemcpyAsync(c.hsp, c.h_hsp, n * sizeof(uint2), cudaMemcpyHostToDevice, c.st));
    SA_CUDA_OK(cudaMemsetAsync(c.diff, 0, span * sizeof(int), c.st));
    SA_CUDA_OK(cudaMemsetAsync(c.n_bnd, 0, sizeof(unsigned long long), c.st));
    const int g = (int)std::min<uint64_t>((n + 255) / 256, 4096);
    sa_k_cov_diff<<<g, 256, 0, c.st>>>(c.hsp, n, lo, span, c.diff);
    sa_k_cov_tile_sums<<<tiles, kCovThreads, 0, c.st>>>(c.diff, span, c.sums);
    sa_k_cov_scan_sums<<<1, kCovThreads, 0, c.st>>>(c.sums, tiles);
    sa_k_cov_bounds<<<tiles, kCovThreads, 0, c.st>>>(c.diff, span, c.sums, lo, M, c.bnd, c.n_bnd, c.bnd_cap);
    for (int k = 0; k < 4; ++k) sa_note_launch();
    SA_CUDA_OK(cudaGetLastError());
    unsigned long long nb = 0;
    SA_CUDA_OK(cudaMemcpyAsync(&nb, c.n_bnd, sizeof nb, cudaMemcpyDeviceToHost, c.st));
    SA_CUDA_OK(cudaStreamSynchronize(c.st));
    if (nb > c.bnd_cap) {
        sa_set_error(SA_ERR_CAPACITY, "coverage boundaries exceed their list");
        return SA_ERR_CAPACITY;
    }
    std::vector<uint32_t> b(nb);
    if (nb) SA_CUDA_OK(cudaMemcpyAsync(b.data(), c.bnd, nb * sizeof(uint32_t), cudaMemcpyDeviceToHost, c.st));
    SA_CUDA_OK(cudaStreamSynchronize(c.st));
    std::sort(b.begin(), b.end());
    for (size_t i = 0; i + 1 < b.size(); i += 2) runs.emplace_back(b[i], b[i + 1] - b[i]);
    return SA_OK;  // an unpaired last boundary is a run open at the block end
}
