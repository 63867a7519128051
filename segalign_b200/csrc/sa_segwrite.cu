// sa_segwrite.cu — the segment writer on the GPU.
//
// Reference: src/segment_printer.cpp:51-147 (one line per HSP, "rchr rstart
// rend qchr qstart qend +|- score", 1-based chromosome-relative starts; the
// minus strand's lines in reverse HSP order, its query chromosomes placed in
// the reverse complement of the query block, src/main.cpp:355-362).  The
// output is the same text, byte for byte, as the host writer
// (sa_format_segments in sa_host.cpp).
//
// Three kernels over the lines (plus lines first, then minus lines): the
// length of every line summed per CTA range, one CTA scanning the range sums,
// and a pass that rescans each range in rounds of 256 lines to place and
// write every line.  A line's fields are recomputed in each pass (two
// chromosome binary searches and the decimal digits) instead of being
// stored.  Device memory is stream-ordered (cudaMallocAsync on the writer's
// own stream), so the writer never synchronises the whole device.
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/segalign_b200_host.h"
#include "sa_host_internal.h"
#include "sa_launch.h"
#include "sa_radix.cuh"

namespace {

constexpr int kSegThreads = 256;
constexpr int kSegMaxCtas = 1024;

// A chromosome table on the device: starts ascending; name k of row i is
// names[off[k] .. off[k] + len[k]) with k = idx ? idx[i] : i.
struct SegTab {
    const uint64_t* starts;
    const uint32_t* idx;
    const uint32_t* off;
    const uint32_t* len;
    uint32_t n;
};

struct SegArgs {
    const sa_segment* fw;
    const sa_segment* rc;
    uint64_t n_fw, n_rc;
    uint64_t ref_block_start, query_block_start;
    SegTab ref, qry, qrc;
    const char* names;
};

struct SegLine {
    uint32_t rname, qname;  // name index
    uint64_t rs, re, qs, qe;
    int32_t score;
    char strand;
};

// Row of the last start <= x (row 0 when x precedes every start), as
// std::upper_bound - 1 in the host writer.
__device__ __forceinline__ uint32_t sa_chrom_row(const uint64_t* __restrict__ s, uint32_t n, uint64_t x) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (s[mid] <= x) lo = mid + 1;
        else hi = mid;
    }
    return lo ? lo - 1 : 0u;
}

__device__ __forceinline__ uint32_t sa_ndigits(uint64_t v) {
    uint32_t d = 1;
    while (v >= 10) {
        v /= 10;
        ++d;
    }
    return d;
}

__device__ __forceinline__ char* sa_put_u64(char* p, uint64_t v) {
    const uint32_t d = sa_ndigits(v);
    for (int i = (int)d - 1; i >= 0; --i) {
        p[i] = (char)('0' + (int)(v % 10));
        v /= 10;
    }
    return p + d;
}

__device__ __forceinline__ SegLine sa_seg_line(const SegArgs& a, uint64_t i) {
    const bool minus = i >= a.n_fw;
    const sa_segment e = minus ? a.rc[a.n_rc - 1 - (i - a.n_fw)] : a.fw[i];
    SegLine L;
    const uint64_t sr = a.ref_block_start + e.ref_start;
    const uint32_t r = sa_chrom_row(a.ref.starts, a.ref.n, sr);
    L.rname = r;
    L.rs = sr + 1 - a.ref.starts[r];
    L.re = sr + e.len + 1 - a.ref.starts[r];
    const uint64_t sq = a.query_block_start + e.query_start;
    const SegTab& q = minus ? a.qrc : a.qry;
    const uint32_t j = sa_chrom_row(q.starts, q.n, sq);
    L.qname = q.idx ? q.idx[j] : j;
    L.qs = sq + 1 - q.starts[j];
    L.qe = sq + e.len + 1 - q.starts[j];
    L.score = e.score;
    L.strand = minus ? '-' : '+';
    return L;
}

__device__ __forceinline__ uint64_t sa_seg_len(const SegArgs& a, const SegLine& L) {
    const uint64_t mag = L.score < 0 ? (uint64_t)(-(int64_t)L.score) : (uint64_t)L.score;
    return (uint64_t)a.ref.len[L.rname] + sa_ndigits(L.rs) + sa_ndigits(L.re) + a.qry.len[L.qname] +
           sa_ndigits(L.qs) + sa_ndigits(L.qe) + (L.score < 0 ? 1u : 0u) + sa_ndigits(mag) + 9u;
}

__device__ __forceinline__ void sa_seg_write(const SegArgs& a, const SegLine& L, char* p) {
    const uint32_t rl = a.ref.len[L.rname], ql = a.qry.len[L.qname];
    const char* rn = a.names + a.ref.off[L.rname];
    const char* qn = a.names + a.qry.off[L.qname];
    for (uint32_t k = 0; k < rl; ++k) *p++ = rn[k];
    *p++ = '\t';
    p = sa_put_u64(p, L.rs);
    *p++ = '\t';
    p = sa_put_u64(p, L.re);
    *p++ = '\t';
    for (uint32_t k = 0; k < ql; ++k) *p++ = qn[k];
    *p++ = '\t';
    p = sa_put_u64(p, L.qs);
    *p++ = '\t';
    p = sa_put_u64(p, L.qe);
    *p++ = '\t';
    *p++ = L.strand;
    *p++ = '\t';
    if (L.score < 0) *p++ = '-';
    p = sa_put_u64(p, L.score < 0 ? (uint64_t)(-(int64_t)L.score) : (uint64_t)L.score);
    *p = '\n';
}

__global__ void __launch_bounds__(kSegThreads) sa_k_seg_sums(SegArgs a, unsigned long long* cta_sum) {
    const uint64_t n = a.n_fw + a.n_rc;
    uint64_t lo, hi;
    sa_cta_range(n, lo, hi);
    unsigned long long s = 0;
    for (uint64_t i = lo + threadIdx.x; i < hi; i += kSegThreads) s += sa_seg_len(a, sa_seg_line(a, i));
    __shared__ unsigned long long ws[kSegThreads / 32 + 1];
    unsigned long long tot;
    sa_block_excl_sum<unsigned long long, kSegThreads>(s, ws, &tot);
    if (threadIdx.x == 0) cta_sum[blockIdx.x] = tot;
}

// Exclusive scan of the G (<= 1024) range sums in place; total[0] = the sum.
__global__ void __launch_bounds__(1024) sa_k_seg_scan(unsigned long long* cta_sum, int G, unsigned long long* total) {
    const unsigned long long v = threadIdx.x < (unsigned)G ? cta_sum[threadIdx.x] : 0ull;
    __shared__ unsigned long long ws[1024 / 32 + 1];
    unsigned long long tot;
    const unsigned long long ex = sa_block_excl_sum<unsigned long long, 1024>(v, ws, &tot);
    if (threadIdx.x < (unsigned)G) cta_sum[threadIdx.x] = ex;
    if (threadIdx.x == 0) *total = tot;
}

// Writes every line; split[0] = the offset of the first minus line.
__global__ void __launch_bounds__(kSegThreads)
sa_k_seg_write(SegArgs a, const unsigned long long* cta_base, char* text, unsigned long long* split) {
    const uint64_t n = a.n_fw + a.n_rc;
    uint64_t lo, hi;
    sa_cta_range(n, lo, hi);
    unsigned long long base = cta_base[blockIdx.x];
    __shared__ unsigned long long ws[kSegThreads / 32 + 1];
    for (uint64_t r = lo; r < hi; r += kSegThreads) {
        const uint64_t i = r + threadIdx.x;
        SegLine L{};
        unsigned long long len = 0;
        if (i < hi) {
            L = sa_seg_line(a, i);
            len = sa_seg_len(a, L);
        }
        unsigned long long tot;
        const unsigned long long at = base + sa_block_excl_sum<unsigned long long, kSegThreads>(len, ws, &tot);
        if (i < hi) {
            sa_seg_write(a, L, text + at);
            if (i == a.n_fw) *split = at;
        }
        base += tot;
    }
}

// One table's rows for the device: starts, name index per row, and the
// names (appended to a shared blob) with their offsets and lengths.
struct HostTab {
    std::vector<uint64_t> starts;
    std::vector<uint32_t> idx, off, len;
};

void add_names(const sa_chrom_table* t, std::string& blob, HostTab& h) {
    for (uint32_t k = 0; k < t->count; ++k) {
        const char* s = t->names[k] ? t->names[k] : "";
        h.off.push_back((uint32_t)blob.size());
        h.len.push_back((uint32_t)std::strlen(s));
        blob += s;
    }
}

std::mutex g_seg_mu;           // one writer at a time per process (its stream)
cudaStream_t g_seg_st = nullptr;

template <class T>
int dev_copy(const T* src, uint64_t n, T** dst, cudaStream_t st) {
    *dst = nullptr;
    if (!n) return SA_OK;
    SA_CUDA_OK(cudaMallocAsync(dst, n * sizeof(T), st));
    SA_CUDA_OK(cudaMemcpyAsync(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice, st));
    return SA_OK;
}

}  // namespace

// The writer.  With `pin` the text (plus lines, then minus lines) goes into
// the caller's pinned buffer *pin, reallocated when it holds fewer than the
// text's bytes (*pin_cap), and plus_text / minus_text are not set; without
// it, into two malloc'd strings.
static int seg_format(const sa_chrom_table* ref, uint64_t ref_block_start, const sa_chrom_table* query,
                      uint64_t query_block_start, uint32_t query_block_len, const sa_segment* fw, uint64_t n_fw,
                      const sa_segment* rc, uint64_t n_rc, char** plus_text, uint64_t* plus_len, char** minus_text,
                      uint64_t* minus_len, char** pin, uint64_t* pin_cap) {
    if (!ref || !query || !ref->count || !query->count || (n_fw && !fw) || (n_rc && !rc) || !plus_len ||
        !minus_len || (pin ? !pin_cap : (!plus_text || !minus_text)))
        return SA_ERR_ARG;
    // reverse-complement chromosome table of the block (src/main.cpp:355-362),
    // as the host writer builds it
    HostTab hr, hq, hc;
    std::string blob;
    hr.starts.assign(ref->starts, ref->starts + ref->count);
    add_names(ref, blob, hr);
    hq.starts.assign(query->starts, query->starts + query->count);
    add_names(query, blob, hq);
    for (uint32_t i = query->count; i-- > 0;) {
        const uint64_t st = query->starts[i];
        if (st < query_block_start || st >= query_block_start + query_block_len) continue;
        hc.starts.push_back(2 * query_block_start + query_block_len - st - query->lens[i]);
        hc.idx.push_back(i);
    }
    if (hc.starts.empty()) return SA_ERR_ARG;
    *plus_len = *minus_len = 0;
    const uint64_t n = n_fw + n_rc;
    if (pin && n == 0) return SA_OK;
    if (!pin) *plus_text = *minus_text = nullptr;
    if (n == 0) {
        *plus_text = (char*)calloc(1, 1);
        *minus_text = (char*)calloc(1, 1);
        if (!*plus_text || !*minus_text) {
            free(*plus_text);
            free(*minus_text);
            *plus_text = *minus_text = nullptr;
            return SA_ERR_NOMEM;
        }
        return SA_OK;
    }

    std::lock_guard<std::mutex> lk(g_seg_mu);
    if (!g_seg_st) SA_CUDA_OK(cudaStreamCreateWithFlags(&g_seg_st, cudaStreamNonBlocking));
    cudaStream_t st = g_seg_st;
    std::vector<void*> owned;
    int rcode = SA_OK;
    char* text_h = nullptr;
    do {
        SegArgs a{};
        sa_segment *dfw = nullptr, *drc = nullptr;
        uint64_t *rs = nullptr, *qs = nullptr, *cs = nullptr;
        uint32_t *roff = nullptr, *rlen = nullptr, *qoff = nullptr, *qlen = nullptr, *cidx = nullptr;
        char* names = nullptr;
        if ((rcode = dev_copy(fw, n_fw, &dfw, st)) != SA_OK) break;
        owned.push_back(dfw);
        if ((rcode = dev_copy(rc, n_rc, &drc, st)) != SA_OK) break;
        owned.push_back(drc);
        if ((rcode = dev_copy(hr.starts.data(), hr.starts.size(), &rs, st)) != SA_OK) break;
        owned.push_back(rs);
        if ((rcode = dev_copy(hr.off.data(), hr.off.size(), &roff, st)) != SA_OK) break;
        owned.push_back(roff);
        if ((rcode = dev_copy(hr.len.data(), hr.len.size(), &rlen, st)) != SA_OK) break;
        owned.push_back(rlen);
        if ((rcode = dev_copy(hq.starts.data(), hq.starts.size(), &qs, st)) != SA_OK) break;
        owned.push_back(qs);
        if ((rcode = dev_copy(hq.off.data(), hq.off.size(), &qoff, st)) != SA_OK) break;
        owned.push_back(qoff);
        if ((rcode = dev_copy(hq.len.data(), hq.len.size(), &qlen, st)) != SA_OK) break;
        owned.push_back(qlen);
        if ((rcode = dev_copy(hc.starts.data(), hc.starts.size(), &cs, st)) != SA_OK) break;
        owned.push_back(cs);
        if ((rcode = dev_copy(hc.idx.data(), hc.idx.size(), &cidx, st)) != SA_OK) break;
        owned.push_back(cidx);
        if ((rcode = dev_copy(blob.data(), blob.size() + 1, &names, st)) != SA_OK) break;
        owned.push_back(names);
        a.fw = dfw;
        a.rc = drc;
        a.n_fw = n_fw;
        a.n_rc = n_rc;
        a.ref_block_start = ref_block_start;
        a.query_block_start = query_block_start;
        a.ref = SegTab{rs, nullptr, roff, rlen, ref->count};
        a.qry = SegTab{qs, nullptr, qoff, qlen, query->count};
        a.qrc = SegTab{cs, cidx, qoff, qlen, (uint32_t)hc.starts.size()};
        a.names = names;

        const int G = (int)std::min<uint64_t>((n + 4 * kSegThreads - 1) / (4 * kSegThreads), kSegMaxCtas);
        unsigned long long* scan = nullptr;  // [G] range sums, then [G] total, [G + 1] split
        if ((rcode = [&]() {
                 SA_CUDA_OK(cudaMallocAsync(&scan, (G + 2) * sizeof(unsigned long long), st));
                 return SA_OK;
             }()) != SA_OK)
            break;
        owned.push_back(scan);
        sa_k_seg_sums<<<G, kSegThreads, 0, st>>>(a, scan);
        sa_k_seg_scan<<<1, 1024, 0, st>>>(scan, G, scan + G);
        unsigned long long h[2] = {0, 0};
        if (cudaMemcpyAsync(h, scan + G, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            rcode = SA_ERR_CUDA;
            break;
        }
        const unsigned long long total = h[0];
        char* text = nullptr;
        if (cudaMallocAsync(&text, total ? total : 1, st) != cudaSuccess) {
            rcode = SA_ERR_CUDA;
            break;
        }
        owned.push_back(text);
        // the split defaults to the end (no minus lines)
        if (cudaMemcpyAsync(scan + G + 1, &total, sizeof total, cudaMemcpyHostToDevice, st) != cudaSuccess) {
            rcode = SA_ERR_CUDA;
            break;
        }
        sa_k_seg_write<<<G, kSegThreads, 0, st>>>(a, scan, text, scan + G + 1);
        unsigned long long split = 0;
        if (cudaMemcpyAsync(&split, scan + G + 1, sizeof split, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            rcode = SA_ERR_CUDA;
            break;
        }
        if (pin) {
            if (*pin_cap < total) {
                if (*pin) cudaFreeHost(*pin);
                *pin = nullptr;
                *pin_cap = 0;
                if (cudaMallocHost(pin, total) != cudaSuccess) {
                    cudaGetLastError();  // an allocation failure is reported, not left pending
                    *pin = nullptr;
                    rcode = SA_ERR_NOMEM;
                    break;
                }
                *pin_cap = total;
            }
            if (cudaMemcpyAsync(*pin, text, total, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess) {
                rcode = SA_ERR_CUDA;
                break;
            }
            *plus_len = split;
            *minus_len = total - split;
            break;
        }
        text_h = (char*)malloc(total + 1);
        char* minus_h = (char*)malloc(total - split + 1);
        if (!text_h || !minus_h) {
            free(minus_h);
            rcode = SA_ERR_NOMEM;
            break;
        }
        if (cudaMemcpyAsync(text_h, text, split, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaMemcpyAsync(minus_h, text + split, total - split, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            free(minus_h);
            rcode = SA_ERR_CUDA;
            break;
        }
        text_h[split] = 0;
        minus_h[total - split] = 0;
        *plus_text = text_h;
        *plus_len = split;
        *minus_text = minus_h;
        *minus_len = total - split;
        text_h = nullptr;
    } while (false);
    free(text_h);
    for (void* p : owned)
        if (p) cudaFreeAsync(p, st);
    cudaStreamSynchronize(st);
    if (rcode == SA_ERR_CUDA) sa_set_error(SA_ERR_CUDA, "segment writer: %s", cudaGetErrorString(cudaGetLastError()));
    if (rcode == SA_ERR_NOMEM) sa_set_error(SA_ERR_NOMEM, "segment writer: host allocation failed");
    return rcode;
}

extern "C" int sa_format_segments_gpu(const sa_chrom_table* ref, uint64_t ref_block_start,
                                      const sa_chrom_table* query, uint64_t query_block_start,
                                      uint32_t query_block_len, const sa_segment* fw, uint64_t n_fw,
                                      const sa_segment* rc, uint64_t n_rc, char** plus_text, uint64_t* plus_len,
                                      char** minus_text, uint64_t* minus_len) {
    return seg_format(ref, ref_block_start, query, query_block_start, query_block_len, fw, n_fw, rc, n_rc, plus_text,
                      plus_len, minus_text, minus_len, nullptr, nullptr);
}

int sa_format_segments_pinned(const sa_chrom_table* ref, uint64_t ref_block_start, const sa_chrom_table* query,
                              uint64_t query_block_start, uint32_t query_block_len, const sa_segment* fw,
                              uint64_t n_fw, const sa_segment* rc, uint64_t n_rc, char** pinned, uint64_t* cap,
                              uint64_t* plus_len, uint64_t* minus_len) {
    return seg_format(ref, ref_block_start, query, query_block_start, query_block_len, fw, n_fw, rc, n_rc, nullptr,
                      plus_len, nullptr, minus_len, pinned, cap);
}
