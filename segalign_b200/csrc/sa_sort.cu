// sa_sort.cu — per-scope ordering and deduplication of surviving HSPs.
//
// Reference (per SeedAndFilter call and MAX_HITS iteration):
//   plain: thrust::stable_sort(hspComp) + unique_copy(hspEqual)
//          src/seed_filter.cu:47-80, 728-732
//   rm:    then stable_sort(hspDiagComp) + unique_copy(hspDiagEqual) +
//          stable_sort(hspFinalComp)   repeat_masker_src/seed_filter.cu:45-107, 797-811
// unique_copy on the CUDA backend keeps element i iff i == 0 or
// !pred(x[i-1], x[i]) with x[i-1] the input predecessor (CUB FlagHeads), which
// matters for the non-transitive hspDiagEqual.
//
// Keys.  Records of one scope come from one (query, target) pair, so the HSP
// score is a function of (ref_start, query_start, len): total is the sum of
// substitution scores over the segment and the entropy factor depends only on
// the segment's base counts.  hspComp therefore orders a scope totally by
// (query_start asc, len desc, ref_start asc); equal keys are equal records.
// The rm sorts are stable on their input, so hspDiagComp needs (diag, ref_start,
// score desc) [query_start follows from diag and ref_start] and hspFinalComp
// needs (query_start, score desc, ref_start desc); ties keep the earlier order
// exactly as thrust's stable sort does.  The scope is the most significant key.
#include "sa_launch.h"
#include "sa_radix.cuh"

#define SA_DERR_SURV_OVERFLOW 4

enum : uint8_t { F_RS = 0, F_QS = 1, F_LEN = 2, F_SCORE = 3, F_SCOPE = 4, F_DIAG = 5 };

struct SaSortSpec {
    int npass;
    uint8_t field[SA_SORT_MAX_DIGITS];
    uint8_t byte[SA_SORT_MAX_DIGITS];
    uint8_t inv[SA_SORT_MAX_DIGITS];
};

struct SaRecOps {
    struct Ctx {
        SaRec* rec[2];
        uint32_t* scope[2];
        SaSortSpec spec;
    };
    static __device__ __forceinline__ uint32_t field_value(const SaRec& r, uint32_t scope, int f) {
        switch (f) {
            case F_RS: return r.ref_start;
            case F_QS: return r.query_start;
            case F_LEN: return r.len;
            case F_SCORE: return (uint32_t)r.score ^ 0x80000000u;  // signed ascending
            case F_SCOPE: return scope;
            default: return r.ref_start - r.query_start;      // uint32 diagonal
        }
    }
    struct Pass {
        uint32_t field, shift, inv;
    };
    static __device__ __forceinline__ Pass pass_of(const Ctx& c, int pass) {
        return {c.spec.field[pass], 8u * c.spec.byte[pass], c.spec.inv[pass] ? ~0u : 0u};
    }
    struct Item {
        SaRec r;
        uint32_t scope;
    };
    static __device__ __forceinline__ Item load(const Ctx& c, int buf, uint64_t i) {
        return {c.rec[buf][i], c.scope[buf][i]};
    }
    static __device__ __forceinline__ uint32_t digit_of(const Pass& p, const Item& x) {
        return ((field_value(x.r, x.scope, (int)p.field) ^ p.inv) >> p.shift) & 0xffu;
    }
    static __device__ __forceinline__ void store(const Ctx& c, int buf, const Item& x, uint32_t dst) {
        c.rec[buf ^ 1][dst] = x.r;
        c.scope[buf ^ 1][dst] = x.scope;
    }
};

// Histograms of every digit of the spec in one read (pre-pass).
__global__ void __launch_bounds__(256)
sa_k_sort_hist_all(SaRecOps::Ctx c, const unsigned long long* d_n, const int* st, unsigned int* ghist) {
    __shared__ unsigned int h[SA_SORT_MAX_DIGITS][256];
    const int np = c.spec.npass, t = threadIdx.x;
    for (int p = 0; p < np; ++p) h[p][t] = 0;
    __syncthreads();
    const int buf = st[0];
    uint64_t a, b;
    sa_cta_range(*d_n, a, b);
    for (uint64_t i = a + t; i < b; i += 256) {
        const SaRec r = c.rec[buf][i];
        const uint32_t sc = c.scope[buf][i];
        for (int p = 0; p < np; ++p) {
            uint32_t v = SaRecOps::field_value(r, sc, c.spec.field[p]);
            if (c.spec.inv[p]) v = ~v;
            atomicAdd(&h[p][(v >> (8 * c.spec.byte[p])) & 0xffu], 1u);
        }
    }
    __syncthreads();
    for (int p = 0; p < np; ++p)
        if (h[p][t]) atomicAdd(&ghist[p * 256 + t], h[p][t]);
}

// Pass plan: a pass whose digit is the same for all items is skipped.
// in_buf[p] = input buffer of pass p (-1 = skip); in_buf[np] = final buffer.
__global__ void sa_k_sort_plan(const unsigned int* ghist, int np, const unsigned long long* d_n, int* st) {
    __shared__ int skip[SA_SORT_MAX_DIGITS];
    const int t = threadIdx.x;
    const unsigned long long n = *d_n;
    if (t < np) skip[t] = (n <= 1);
    __syncthreads();
    for (int p = 0; p < np; ++p)
        if (ghist[p * 256 + t] == n) skip[p] = 1;
    __syncthreads();
    if (t == 0) {
        int cur = st[0];
        for (int p = 0; p < np; ++p) {
            st[1 + p] = skip[p] ? -1 : cur;
            if (!skip[p]) cur ^= 1;
        }
        st[1 + np] = cur;
    }
}

static void sa_radix_sort_recs(SaWork& w, const SaSortSpec& spec, const unsigned long long* d_n, int* st, int G,
                               cudaStream_t s) {
    SaRecOps::Ctx c;
    c.rec[0] = w.rec[0];
    c.rec[1] = w.rec[1];
    c.scope[0] = w.scope[0];
    c.scope[1] = w.scope[1];
    c.spec = spec;
    cudaMemsetAsync(w.sort_hist, 0, sizeof(unsigned int) * 256 * SA_SORT_MAX_DIGITS, s);
    sa_k_sort_hist_all<<<G, 256, 0, s>>>(c, d_n, st, w.sort_hist);
    sa_note_launch();
    sa_k_sort_plan<<<1, 256, 0, s>>>(w.sort_hist, spec.npass, d_n, st);
    sa_note_launch();
    SaRadixCtl ctl{d_n, st + 1};
    for (int p = 0; p < spec.npass; ++p) {
        sa_k_radix_up<SaRecOps><<<G, SA_RADIX_BLOCK, 0, s>>>(c, p, ctl, w.sort_cta_hist);
        sa_note_launch();
        sa_k_radix_scan<<<1, 1024, 0, s>>>(w.sort_cta_hist, G, st + 1, p, d_n);
        sa_note_launch();
        sa_k_radix_down<SaRecOps><<<G, SA_RADIX_BLOCK, 0, s>>>(c, p, ctl, w.sort_cta_hist);
        sa_note_launch();
    }
}

// ---------------------------------------------------------------------------
// Predecessor-adjacent unique + ordered compaction
// ---------------------------------------------------------------------------
struct SaUniqArgs {
    SaRec* rec[2];
    uint32_t* scope[2];
    const uint32_t* scope_flags;
    SaRec* out_rec;             // null: write to the other ping-pong buffer
    uint32_t* out_scope;
    uint32_t* scope_count;      // null: no per-scope counts
    int mode;                   // 0 = hspEqual, 1 = hspDiagEqual + diagonal exclusion, 2 = keep all (copy)
    int scope_shift;            // counts and flags are indexed by scope >> scope_shift
};

__device__ __forceinline__ bool sa_rec_equal(const SaRec& x, const SaRec& y) {
    return x.ref_start == y.ref_start && x.query_start == y.query_start && x.len == y.len && x.score == y.score;
}

// hspDiagEqual (repeat_masker_src/seed_filter.cu:45-50).
__device__ __forceinline__ bool sa_rec_diag_equal(const SaRec& x, const SaRec& y) {
    if ((uint32_t)(x.ref_start - x.query_start) != (uint32_t)(y.ref_start - y.query_start)) return false;
    const bool xin = x.ref_start >= y.ref_start && (uint32_t)(x.ref_start + x.len) <= (uint32_t)(y.ref_start + y.len);
    const bool yin = y.ref_start >= x.ref_start && (uint32_t)(y.ref_start + y.len) <= (uint32_t)(x.ref_start + x.len);
    return xin || yin;
}

__device__ __forceinline__ bool sa_uniq_keep(const SaUniqArgs& u, int buf, uint64_t i) {
    const SaRec r = u.rec[buf][i];
    const uint32_t sc = u.scope[buf][i];
    bool keep = true;
    if (u.mode != 2 && i > 0) {
        const SaRec pr = u.rec[buf][i - 1];
        const uint32_t ps = u.scope[buf][i - 1];
        if (ps == sc) keep = u.mode == 0 ? !sa_rec_equal(pr, r) : !sa_rec_diag_equal(pr, r);
    }
    // Main-diagonal exclusion for the repeat-masker self alignment: scope
    // flags bit1 = exclusion requested, bit0 = minus strand (never excluded).
    if (u.mode == 1 && (u.scope_flags[sc >> u.scope_shift] & 3u) == 2u && r.ref_start == r.query_start) keep = false;
    return keep;
}

__global__ void __launch_bounds__(256)
sa_k_uniq_count(SaUniqArgs u, const unsigned long long* d_n, const int* src_buf, unsigned long long* cta_a) {
    const int buf = *src_buf;
    uint64_t a, b;
    sa_cta_range(*d_n, a, b);
    unsigned long long c = 0;
    for (uint64_t i = a + threadIdx.x; i < b; i += 256) c += sa_uniq_keep(u, buf, i);
    __shared__ unsigned long long ws[9];
    unsigned long long tot;
    sa_block_excl_sum<unsigned long long, 256>(c, ws, &tot);
    if (threadIdx.x == 0) cta_a[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(256)
sa_k_uniq_emit(SaUniqArgs u, const unsigned long long* d_n, const int* src_buf, const unsigned long long* cta_a) {
    const int buf = *src_buf;
    uint64_t a, b;
    sa_cta_range(*d_n, a, b);
    unsigned long long base = cta_a[blockIdx.x];
    SaRec* dr = u.out_rec ? u.out_rec : u.rec[buf ^ 1];
    uint32_t* ds = u.out_scope ? u.out_scope : u.scope[buf ^ 1];
    __shared__ unsigned long long ws[9];
    for (uint64_t r0 = a; r0 < b; r0 += 256) {
        const uint64_t i = r0 + threadIdx.x;
        const bool k = i < b && sa_uniq_keep(u, buf, i);
        unsigned long long tot;
        const unsigned long long e = sa_block_excl_sum<unsigned long long, 256>((unsigned long long)k, ws, &tot);
        if (k) {
            const uint32_t sc = u.scope[buf][i];
            dr[base + e] = u.rec[buf][i];
            ds[base + e] = sc;
            if (u.scope_count) atomicAdd(&u.scope_count[sc >> u.scope_shift], 1u);
        }
        base += tot;
    }
}

// Plain-mode output.  The records of a plain sort are the distinct keys
// (scope, ref_start, query_start, len) of the HSP set, and within a scope the
// score is a function of the key, so no two records of a scope are equal:
// unique_copy(hspEqual) keeps every record.  The sorted records are copied
// to the output as they are, and each count[s] (s = scope >> shift, counts
// zeroed beforehand) gets end(s) - start(s) from the two records at its
// boundaries: count[s] -= first index, count[s] += one past the last (the
// counts wrap through unsigned arithmetic), two atomics per count.
__global__ void __launch_bounds__(256)
sa_k_out_copy(SaUniqArgs u, const unsigned long long* d_n, const int* src_buf, unsigned long long* d_out_n) {
    const unsigned long long n = *d_n;
    const int buf = *src_buf;
    const SaRec* __restrict__ rec = u.rec[buf];
    const uint32_t* __restrict__ sc = u.scope[buf];
    if (blockIdx.x == 0 && threadIdx.x == 0) *d_out_n = n;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const uint32_t s = sc[i];
        u.out_rec[i] = rec[i];
        u.out_scope[i] = s;
        const uint32_t g = s >> u.scope_shift;
        const uint32_t gp = i > 0 ? sc[i - 1] >> u.scope_shift : ~0u;
        if (g != gp) {
            atomicSub(&u.scope_count[g], (uint32_t)i);
            if (i > 0) atomicAdd(&u.scope_count[gp], (uint32_t)i);
        }
        if (i + 1 == n) atomicAdd(&u.scope_count[g], (uint32_t)n);
    }
}

// st[0] <- 1 - final buffer of the last sort (the buffer the unique step wrote).
__global__ void sa_k_flip_cur(int* st, int np) { st[0] = st[1 + np] ^ 1; }

// Sizes the call's HSP set: the smallest power of two >= 2 * hits (at least
// 1024), at most `max_slots` (a power of two, the whole table).  With `full`
// every slot of the table is marked empty; otherwise the table is known to be
// empty already (the previous call's compaction emptied the slots it used).
__global__ void sa_k_hash_init(SaHashSet hs, SaCounters* ctr, unsigned long long max_slots, int full) {
    unsigned long long want = 2 * ctr->num_hits;
    if (want < 1024) want = 1024;
    unsigned long long slots = 1;
    while (slots < want && slots < max_slots) slots <<= 1;
    if (blockIdx.x == 0 && threadIdx.x == 0) ctr->hash_mask = slots - 1;
    if (!full) return;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < 2 * max_slots;
         i += (unsigned long long)gridDim.x * blockDim.x)
        hs.keys[i] = ~0ull;
}

// Distinct HSPs out of the set into rec/scope, in claim order (the sort that
// follows is total), emptying their slots.  *n_out = slots claimed; more than
// `cap` is a capacity error (sa_k_dedup_prep).  A thread gathers
// SA_COMPACT_ITEMS slots before it writes any (the slots of the list are
// distinct), so their scattered loads are in flight together.
#define SA_COMPACT_ITEMS 4
__global__ void __launch_bounds__(256)
sa_k_hash_compact(SaHashSet hs, SaCounters* ctr, SaRec* rec, uint32_t* scope, uint64_t cap, unsigned long long* n_out) {
    constexpr int J = SA_COMPACT_ITEMS;
    const unsigned long long used = ctr->hash_used;
    unsigned long long n = used < hs.used_cap ? used : hs.used_cap;
    if (n > cap) n = cap;
    if (blockIdx.x == 0 && threadIdx.x == 0) *n_out = used;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long i0 = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i0 < n; i0 += J * stride) {
        unsigned long long h[J];
        ulonglong2 k[J];
        int32_t sc[J];
#pragma unroll
        for (int j = 0; j < J; ++j) {
            const unsigned long long i = i0 + j * stride;
            h[j] = i < n ? hs.used[i] : ~0ull;
        }
#pragma unroll
        for (int j = 0; j < J; ++j)
            if (h[j] != ~0ull) {
                k[j] = *reinterpret_cast<const ulonglong2*>(hs.keys + 2 * h[j]);
                sc[j] = hs.score[h[j]];
            }
#pragma unroll
        for (int j = 0; j < J; ++j)
            if (h[j] != ~0ull) {
                const unsigned long long i = i0 + j * stride;
                SaRec r;
                r.ref_start = (uint32_t)k[j].x;
                r.query_start = (uint32_t)(k[j].y >> 32);
                r.len = (uint32_t)k[j].y;
                r.score = sc[j];
                rec[i] = r;
                scope[i] = (uint32_t)(k[j].x >> 32);
                *reinterpret_cast<ulonglong2*>(hs.keys + 2 * h[j]) = make_ulonglong2(~0ull, ~0ull);
            }
    }
}

__global__ void sa_k_dedup_prep(SaCounters* ctr, uint64_t cap, unsigned long long* n0, int* st) {
    if (ctr->hash_overflow || *n0 > cap) atomicCAS(&ctr->error, 0ull, (unsigned long long)SA_DERR_SURV_OVERFLOW);
    if (*n0 > cap) *n0 = cap;
    st[0] = 0;
}

static unsigned long long sa_hash_max_slots(const SaWork& w) {
    unsigned long long max_slots = 1;
    while (max_slots * 2 <= 2 * w.surv_cap) max_slots <<= 1;
    return max_slots;
}

void sa_launch_hash_init(SaWork& w, bool full, cudaStream_t st) {
    sa_k_hash_init<<<148 * 8, 256, 0, st>>>(w.hset, w.ctr, sa_hash_max_slots(w), full ? 1 : 0);
    sa_note_launch();
}

__global__ void sa_k_hash_clear(unsigned long long* keys, unsigned long long n) {
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x)
        keys[i] = ~0ull;
}

void sa_launch_hash_clear(SaWork& w, cudaStream_t st) {
    sa_k_hash_clear<<<148 * 8, 256, 0, st>>>(w.hset.keys, 2 * sa_hash_max_slots(w));
    sa_note_launch();
}

void sa_note_hash_state(SaWork& w, const SaCounters& c) {
    w.hash_clean = c.error == 0 && c.hash_used <= w.hset.used_cap && c.hash_used <= w.surv_cap;
}

__global__ void sa_k_copy_u64(unsigned long long* dst, const unsigned long long* src) { *dst = *src; }

static void sa_uniq(SaWork& w, SaUniqArgs u, const unsigned long long* d_n, const int* src_buf,
                    unsigned long long* d_out_n, int G, cudaStream_t s) {
    sa_k_uniq_count<<<G, 256, 0, s>>>(u, d_n, src_buf, w.cta_a);
    sa_note_launch();
    sa_k_scan_partials<<<1, 1024, 0, s>>>(w.cta_a, w.cta_b, G, d_out_n, nullptr);
    sa_note_launch();
    sa_k_uniq_emit<<<G, 256, 0, s>>>(u, d_n, src_buf, w.cta_a);
    sa_note_launch();
}

struct SaSortField {
    uint8_t field, inv, bytes;  // bytes: low-order byte digits that can vary (the rest are zero)
};

static SaSortSpec spec_of(std::initializer_list<SaSortField> fields_lsd_first) {
    // each field expands to its byte digits, least significant first
    SaSortSpec sp{};
    int n = 0;
    for (auto& f : fields_lsd_first)
        for (int byte = 0; byte < f.bytes; ++byte) {
            sp.field[n] = f.field;
            sp.byte[n] = (uint8_t)byte;
            sp.inv[n] = f.inv;
            ++n;
        }
    sp.npass = n;
    return sp;
}

void sa_launch_dedup(SaWork& w, int mode, int scope_shift, int G, cudaStream_t s) {
    // Device-side counts live in the spare counter slots.
    unsigned long long* n0 = &w.ctr->pad[0];
    unsigned long long* n1 = &w.ctr->pad[1];
    unsigned long long* n2 = &w.ctr->pad[2];
    int* st = w.sort_in_buf;
    sa_k_hash_compact<<<148 * 8, 256, 0, s>>>(w.hset, w.ctr, w.rec[0], w.scope[0], w.surv_cap, n0);
    sa_note_launch();
    sa_k_dedup_prep<<<1, 1, 0, s>>>(w.ctr, w.surv_cap, n0, st);
    sa_note_launch();
    cudaMemsetAsync(w.scope_count, 0, sizeof(uint32_t) * SA_MAX_SCOPES, s);

    // Scopes are MAX_HITS iterations (< SA_MAX_ITERS = 256: one byte) in a
    // call, (unit << 4) | iteration (< SA_MAX_UNITS << 4 = 2^20: three bytes)
    // in a batch; their high digits are never sorted on.  Every digit pass
    // costs three launches even when the device plan skips it.
    static_assert(SA_MAX_ITERS <= 256 && SA_MAX_UNITS <= (1 << 20), "scope digit counts");
    const uint8_t sb = scope_shift ? 3 : 1;
    // hspComp order: (scope, query_start asc, len desc, ref_start asc).
    const SaSortSpec plain = spec_of({{F_RS, 0, 4}, {F_LEN, 1, 4}, {F_QS, 0, 4}, {F_SCOPE, 0, sb}});
    sa_radix_sort_recs(w, plain, n0, st, G, s);
    SaUniqArgs u{};
    u.rec[0] = w.rec[0];
    u.rec[1] = w.rec[1];
    u.scope[0] = w.scope[0];
    u.scope[1] = w.scope[1];
    u.scope_flags = w.scope_flags;
    u.scope_shift = scope_shift;
    if (mode == 0) {
        u.mode = 0;
        u.out_rec = w.out;
        u.out_scope = w.out_scope;
        u.scope_count = w.scope_count;
        sa_k_out_copy<<<148 * 8, 256, 0, s>>>(u, n0, st + 1 + plain.npass, &w.ctr->uniq_count);
        sa_note_launch();
        return;
    }
    // rm: unique(hspEqual) into the other buffer
    u.mode = 0;
    sa_uniq(w, u, n0, st + 1 + plain.npass, n1, G, s);
    sa_k_flip_cur<<<1, 1, 0, s>>>(st, plain.npass);
    sa_note_launch();
    // hspDiagComp: (scope, diag asc, ref_start asc, score desc), stable
    const SaSortSpec diag = spec_of({{F_SCORE, 1, 4}, {F_RS, 0, 4}, {F_DIAG, 0, 4}, {F_SCOPE, 0, sb}});
    sa_radix_sort_recs(w, diag, n1, st, G, s);
    u.mode = 1;
    sa_uniq(w, u, n1, st + 1 + diag.npass, n2, G, s);
    sa_k_flip_cur<<<1, 1, 0, s>>>(st, diag.npass);
    sa_note_launch();
    // hspFinalComp: (scope, query_start asc, score desc, ref_start desc), stable
    const SaSortSpec fin = spec_of({{F_RS, 1, 4}, {F_SCORE, 1, 4}, {F_QS, 0, 4}, {F_SCOPE, 0, sb}});
    sa_radix_sort_recs(w, fin, n2, st, G, s);
    u.mode = 2;
    u.out_rec = w.out;
    u.out_scope = w.out_scope;
    u.scope_count = w.scope_count;
    sa_uniq(w, u, n2, st + 1 + fin.npass, &w.ctr->uniq_count, G, s);
}
