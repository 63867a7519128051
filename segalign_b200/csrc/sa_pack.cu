// sa_pack.cu — sequence packing, reverse complement, target seed-position
// table build on the device, and the shared scan kernels.
//
// Reference behaviour restated here:
//   compress_string            common/seed_filter_interface.cu:18-47
//   compress_string_rev_comp   src/seed_filter.cu:82-127
//   rev_comp_string (rm)       repeat_masker_src/seed_filter.cu:137-167
//   GenerateSeedPosTable       common/seed_pos_table.cu:49-109 (CPU in the reference)
#include <cstdio>

#include "sa_launch.h"
#include "sa_radix.cuh"

// ---------------------------------------------------------------------------
// Scans shared by the range-partitioned kernels
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024)
sa_k_scan_partials(unsigned long long* a, unsigned long long* b, int G, unsigned long long* ta,
                   unsigned long long* tb) {
    __shared__ unsigned long long ws[33];
    const int t = threadIdx.x;
    unsigned long long va = t < G ? a[t] : 0ull, vb = t < G ? b[t] : 0ull, tot;
    unsigned long long ea = sa_block_excl_sum<unsigned long long, 1024>(va, ws, &tot);
    if (t == 0 && ta) *ta = tot;
    unsigned long long eb = sa_block_excl_sum<unsigned long long, 1024>(vb, ws, &tot);
    if (t == 0 && tb) *tb = tot;
    if (t < G) {
        a[t] = ea;
        b[t] = eb;
    }
}

__global__ void __launch_bounds__(1024)
sa_k_radix_scan(unsigned int* hist, int G, const int* in_buf, int pass, const unsigned long long* d_n) {
    if (in_buf && in_buf[pass] < 0) return;
    constexpr int PER = 8, TILE = 1024 * PER;
    __shared__ unsigned int tile[TILE];
    __shared__ unsigned int ws[33];
    const int t = threadIdx.x;
    const uint32_t n = 256u * sa_radix_active(*d_n, (uint32_t)G);
    unsigned int carry = 0;
    for (uint32_t base = 0; base < n; base += TILE) {
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const uint32_t i = base + k * 1024 + t;
            tile[k * 1024 + t] = i < n ? hist[i] : 0u;
        }
        __syncthreads();
        unsigned int v[PER], s = 0;
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            v[k] = tile[t * PER + k];
            s += v[k];
        }
        unsigned int tot;
        unsigned int run = sa_block_excl_sum<unsigned int, 1024>(s, ws, &tot) + carry;
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            tile[t * PER + k] = run;
            run += v[k];
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const uint32_t i = base + k * 1024 + t;
            if (i < n) hist[i] = tile[k * 1024 + t];
        }
        carry += tot;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Packing
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t sa_char_code(uint8_t ch) {
    // common/seed_filter_interface.cu:28-46
    switch (ch) {
        case 'A': return 0;
        case 'C': return 1;
        case 'G': return 2;
        case 'T': return 3;
        case 'a': case 'c': case 'g': case 't': return 4;
        case 'n': case 'N': return 5;
        case '&': return 7;
        default: return 6;
    }
}

// One thread per output word: 8 text bytes -> 8 nibbles; bases past `len` are E.
__global__ void sa_k_pack_text(const uint8_t* __restrict__ text, uint64_t len, uint32_t* __restrict__ out,
                               uint64_t nwords) {
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < nwords;
         w += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t b = w * 8;
        uint32_t word = 0;
        if (b + 8 <= len) {
            uint2 v = *reinterpret_cast<const uint2*>(text + b);
#pragma unroll
            for (int k = 0; k < 4; ++k) word |= sa_char_code((v.x >> (8 * k)) & 0xff) << (4 * k);
#pragma unroll
            for (int k = 0; k < 4; ++k) word |= sa_char_code((v.y >> (8 * k)) & 0xff) << (4 * (k + 4));
        } else {
#pragma unroll
            for (int k = 0; k < 8; ++k) word |= (b + k < len ? sa_char_code(text[b + k]) : 7u) << (4 * k);
        }
        out[w] = word;
    }
}

// Reversed copy of a packed sequence: out[i] = in[len-1-i]; with COMP the
// codes 0..3 are complemented as well (reverse complement, A<->T, C<->G;
// L/N/X/E unchanged; src/seed_filter.cu:96-125).  Bases past len are E.
template <bool COMP>
__global__ void sa_k_reverse_packed(const uint32_t* __restrict__ in, uint64_t len, uint32_t* __restrict__ out,
                                    uint64_t nwords) {
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < nwords;
         w += (uint64_t)gridDim.x * blockDim.x) {
        // output bases 8w..8w+7 come from in[len-1-8w-k]; load in[len-8w-8 .. len-8w)
        int64_t p = (int64_t)len - (int64_t)(8 * w) - 8;
        uint32_t x = sa_load8(in, p);
        // reverse nibble order
        x = __byte_perm(x, 0, 0x0123);
        x = ((x >> 4) & 0x0f0f0f0fu) | ((x & 0x0f0f0f0fu) << 4);
        if (COMP) {
            // complement codes 0..3 (bit 2 clear) by xor 3
            uint32_t m = (~(x >> 2)) & 0x11111111u;
            x ^= m * 3u;
        }
        uint64_t b = w * 8;
        if (b + 8 > len) {
#pragma unroll
            for (int k = 0; k < 8; ++k)
                if (b + k >= len) x = (x & ~(0xfu << (4 * k))) | (7u << (4 * k));
        }
        out[w] = x;
    }
}

__global__ void sa_k_fill_u32(uint32_t* p, uint64_t n, uint32_t v) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        p[i] = v;
}

void sa_launch_pack_text(const char* d_text, uint64_t len, uint32_t* packed, cudaStream_t st) {
    uint64_t nwords = (len + 7) / 8;
    if (!nwords) return;
    int blocks = (int)std::min<uint64_t>((nwords + 255) / 256, 148ull * 16);
    sa_k_pack_text<<<blocks, 256, 0, st>>>((const uint8_t*)d_text, len, packed, nwords);
    sa_note_launch();
}

void sa_launch_reverse_packed(const uint32_t* in, uint64_t len, uint32_t* out, bool complement, cudaStream_t st) {
    uint64_t nwords = (len + 7) / 8;
    if (!nwords) return;
    int blocks = (int)std::min<uint64_t>((nwords + 255) / 256, 148ull * 16);
    if (complement) sa_k_reverse_packed<true><<<blocks, 256, 0, st>>>(in, len, out, nwords);
    else sa_k_reverse_packed<false><<<blocks, 256, 0, st>>>(in, len, out, nwords);
    sa_note_launch();
}

void sa_launch_pad_fill(uint32_t* base, uint64_t n, cudaStream_t st) {
    if (!n) return;
    int blocks = (int)std::min<uint64_t>((n + 255) / 256, 148ull * 16);
    sa_k_fill_u32<<<blocks, 256, 0, st>>>(base, n, 0x77777777u);
    sa_note_launch();
}

// ---------------------------------------------------------------------------
// Spaced-seed key of the window starting at base p (common/ntcoding.cpp:43-61):
// invalid unless all seed_size codes are 0..3 (uppercase ACGT); the key folds
// the shape positions in order, first position most significant.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t sa_key_at(const uint32_t* __restrict__ packed, int64_t p,
                                              const SaParams& P) {
    uint32_t w[4];
    w[0] = sa_load8(packed, p);
    w[1] = sa_load8(packed, p + 8);
    w[2] = sa_load8(packed, p + 16);
    w[3] = sa_load8(packed, p + 24);
    uint32_t bad = 0;
    const int ss = P.seed_size;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        int n = ss - 8 * i;
        uint32_t m = n >= 8 ? 0x44444444u : (n <= 0 ? 0u : (0x44444444u & ((1u << (4 * n)) - 1u)));
        bad |= w[i] & m;
    }
    if (bad) return SA_INVALID_KEY;
    uint32_t key = 0;
    for (int i = 0; i < P.kmer_size; ++i) {
        int sp = P.shape_pos[i];
        key = (key << 2) | ((w[sp >> 3] >> (4 * (sp & 7))) & 3u);
    }
    return key;
}

// Table keys, pass 1: per-CTA count of valid positions p = start + i*step.
__global__ void __launch_bounds__(256)
sa_k_table_count(const uint32_t* __restrict__ ref, uint32_t start, uint64_t n, uint32_t step, SaParams P,
                 unsigned long long* cta_a) {
    uint64_t a, b;
    sa_cta_range(n, a, b);
    unsigned long long c = 0;
    for (uint64_t i = a + threadIdx.x; i < b; i += 256)
        c += sa_key_at(ref, (int64_t)start + (int64_t)i * step, P) != SA_INVALID_KEY;
    __shared__ unsigned long long ws[9];
    unsigned long long tot;
    sa_block_excl_sum<unsigned long long, 256>(c, ws, &tot);
    if (threadIdx.x == 0) cta_a[blockIdx.x] = tot;
}

// Table keys, pass 2: ordered compaction of (key, position) pairs.
__global__ void __launch_bounds__(256)
sa_k_table_emit(const uint32_t* __restrict__ ref, uint32_t start, uint64_t n, uint32_t step, SaParams P,
                const unsigned long long* cta_a, uint32_t* keys, uint32_t* vals) {
    uint64_t a, b;
    sa_cta_range(n, a, b);
    unsigned long long base = cta_a[blockIdx.x];
    __shared__ unsigned long long ws[9];
    for (uint64_t r = a; r < b; r += 256) {
        uint64_t i = r + threadIdx.x;
        uint32_t key = SA_INVALID_KEY;
        uint32_t pos = start + (uint32_t)(i * step);
        if (i < b) key = sa_key_at(ref, (int64_t)start + (int64_t)i * step, P);
        unsigned long long v = key != SA_INVALID_KEY, tot;
        unsigned long long e = sa_block_excl_sum<unsigned long long, 256>(v, ws, &tot);
        if (v) {
            keys[base + e] = key;
            vals[base + e] = pos;
        }
        base += tot;
    }
}

void sa_launch_table_keys(const uint32_t* ref, uint32_t start, uint64_t num_steps, uint32_t step,
                          const SaParams& p, uint32_t* keys, uint32_t* vals, unsigned long long* cta_a,
                          unsigned long long* cta_b, unsigned long long* d_total, int G, cudaStream_t st) {
    sa_k_table_count<<<G, 256, 0, st>>>(ref, start, num_steps, step, p, cta_a);
    sa_note_launch();
    sa_k_scan_partials<<<1, 1024, 0, st>>>(cta_a, cta_b, G, d_total, nullptr);
    sa_note_launch();
    sa_k_table_emit<<<G, 256, 0, st>>>(ref, start, num_steps, step, p, cta_a, keys, vals);
    sa_note_launch();
}

// index[k] = number of valid positions with key <= k (the shifted inclusive
// table the reference ships, common/seed_pos_table.cu:83,103): each sorted item
// i fills buckets [key_i, key_{i+1}) with i+1.  `index` must be zeroed first.
__global__ void sa_k_table_index(const uint32_t* __restrict__ keys, const unsigned long long* d_n,
                                 uint32_t* __restrict__ index, uint64_t nbuckets) {
    const uint64_t n = *d_n;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t k = keys[i];
        uint64_t nx = (i + 1 < n) ? keys[i + 1] : nbuckets;
        for (uint64_t bkt = k; bkt < nx; ++bkt) index[bkt] = (uint32_t)(i + 1);
    }
}

void sa_launch_table_index(const uint32_t* sorted_keys, const unsigned long long* d_n, uint32_t* index,
                           uint64_t nbuckets, cudaStream_t st) {
    cudaMemsetAsync(index, 0, nbuckets * sizeof(uint32_t), st);
    sa_k_table_index<<<148 * 8, 256, 0, st>>>(sorted_keys, d_n, index, nbuckets);
    sa_note_launch();
}

// ---------------------------------------------------------------------------
// (key, value) radix sort
// ---------------------------------------------------------------------------
struct SaKvOps {
    struct Ctx {
        uint32_t* k[2];
        uint32_t* v[2];
    };
    struct Pass {
        uint32_t shift;
    };
    static __device__ __forceinline__ Pass pass_of(const Ctx&, int pass) { return {8u * (uint32_t)pass}; }
    struct Item {
        uint32_t k, v;
    };
    static __device__ __forceinline__ Item load(const Ctx& c, int buf, uint64_t i) { return {c.k[buf][i], c.v[buf][i]}; }
    static __device__ __forceinline__ uint32_t digit_of(const Pass& p, const Item& x) { return (x.k >> p.shift) & 0xffu; }
    static __device__ __forceinline__ void store(const Ctx& c, int buf, const Item& x, uint32_t dst) {
        c.k[buf ^ 1][dst] = x.k;
        c.v[buf ^ 1][dst] = x.v;
    }
};

__global__ void sa_k_plan_noskip(int* in_buf, int passes) {
    for (int p = 0; p <= passes; ++p) in_buf[p] = p & 1;
}

void sa_launch_sort_kv(uint32_t* keys, uint32_t* vals, uint32_t* keys_tmp, uint32_t* vals_tmp,
                       const unsigned long long* d_n, int bits, unsigned int* cta_hist, int G,
                       cudaStream_t st, int* result_in_tmp) {
    int passes = (bits + 7) / 8;
    // in_buf lives right after the histogram workspace
    int* in_buf = reinterpret_cast<int*>(cta_hist + 256 * (uint64_t)SA_MAX_CTAS);
    sa_k_plan_noskip<<<1, 1, 0, st>>>(in_buf, passes);
    sa_note_launch();
    SaKvOps::Ctx c;
    c.k[0] = keys;
    c.k[1] = keys_tmp;
    c.v[0] = vals;
    c.v[1] = vals_tmp;
    SaRadixCtl ctl{d_n, in_buf};
    for (int p = 0; p < passes; ++p) {
        sa_k_radix_up<SaKvOps><<<G, SA_RADIX_BLOCK, 0, st>>>(c, p, ctl, cta_hist);
        sa_note_launch();
        sa_k_radix_scan<<<1, 1024, 0, st>>>(cta_hist, G, in_buf, p, d_n);
        sa_note_launch();
        sa_k_radix_down<SaKvOps><<<G, SA_RADIX_BLOCK, 0, st>>>(c, p, ctl, cta_hist);
        sa_note_launch();
    }
    *result_in_tmp = passes & 1;
}

// ---------------------------------------------------------------------------
// Spaced-seed key of every query position (device-side seeding, the work of
// src/seeder.cpp:57-74 without the host loop): keys[j] = key of the window at
// j, SA_INVALID_KEY unless all seed_size bases are uppercase ACGT.
// ---------------------------------------------------------------------------
//
// One thread takes the 8 positions of one packed word, p0 = 8g .. 8g + 7, and
// the five words from word g on, which hold every base their windows reach
// (seed_size <= 32 bases, padding after the last word).  Validity: a 40-bit
// mask of the windows' non-ACGT bases (code bit 2), tested against the
// seed_size bits from each position.  Keys: for each shape position s in
// increasing order (the shape's order, common/ntcoding.cpp:21-37), the word
// of bases p0 + s .. p0 + s + 7 gives the next 2-bit code of all 8 keys at once.
__device__ __forceinline__ uint32_t sa_nonacgt8(uint32_t w) {
    uint32_t t = (w >> 2) & 0x11111111u;  // bit 4k = code bit 2 of base k
    t = (t | (t >> 3)) & 0x03030303u;
    t = (t | (t >> 6)) & 0x000f000fu;
    return (t | (t >> 12)) & 0xffu;
}

__global__ void __launch_bounds__(256)
sa_k_query_keys(const uint32_t* __restrict__ packed, uint64_t len, SaParams P, uint32_t* __restrict__ keys) {
    uint64_t smask = 0;  // bit s set: shape position s is a care position
#pragma unroll
    for (int i = 0; i < 32; ++i)
        if (i < P.kmer_size) smask |= 1ull << P.shape_pos[i];
    const uint32_t ss = (uint32_t)P.seed_size;
    const uint64_t wmask = ss >= 64 ? ~0ull : (1ull << ss) - 1;
    const uint64_t ngroups = (len + 7) / 8;
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < ngroups;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t* pw = packed + g;
        const uint32_t W0 = __ldg(pw), W1 = __ldg(pw + 1), W2 = __ldg(pw + 2), W3 = __ldg(pw + 3), W4 = __ldg(pw + 4);
        const uint64_t bad = (uint64_t)sa_nonacgt8(W0) | ((uint64_t)sa_nonacgt8(W1) << 8) |
                             ((uint64_t)sa_nonacgt8(W2) << 16) | ((uint64_t)sa_nonacgt8(W3) << 24) |
                             ((uint64_t)sa_nonacgt8(W4) << 32);
        uint32_t key[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) key[k] = 0;
        for (uint64_t m = smask; m; m &= m - 1) {
            const uint32_t sp = (uint32_t)(__ffsll((long long)m) - 1);
            const uint32_t q = sp >> 3;
            const uint32_t a = q == 0 ? W0 : q == 1 ? W1 : q == 2 ? W2 : W3;
            const uint32_t b = q == 0 ? W1 : q == 1 ? W2 : q == 2 ? W3 : W4;
            const uint32_t win = __funnelshift_r(a, b, 4u * (sp & 7u));
#pragma unroll
            for (int k = 0; k < 8; ++k) key[k] = (key[k] << 2) | ((win >> (4 * k)) & 3u);
        }
        const uint64_t p0 = 8 * g;
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (p0 + k < len) keys[p0 + k] = ((bad >> k) & wmask) ? SA_INVALID_KEY : key[k];
    }
}

void sa_launch_query_keys(const uint32_t* packed, uint64_t len, const SaParams& p, uint32_t* keys, cudaStream_t st) {
    if (!len) return;
    const uint64_t groups = (len + 7) / 8;
    int blocks = (int)std::min<uint64_t>((groups + 255) / 256, 148ull * 16);
    sa_k_query_keys<<<blocks, 256, 0, st>>>(packed, len, p, keys);
    sa_note_launch();
}
