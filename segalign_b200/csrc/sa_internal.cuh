// sa_internal.cuh — shared types and device helpers of the B200 seed-filter path.
//
// Sequence layout in HBM: one 4-bit code per base, 8 bases per uint32 word
// ("nibble-packed"), base i in bits [4*(i&7), 4*(i&7)+4) of word i>>3.  Codes
// are the reference's (common/parameters.h:4-11): A0 C1 G2 T3 L4 N5 X6 E7.
// Every packed array carries SA_PADW words of padding on both sides (filled
// with E codes) so that 8-base windows next to either end can be loaded
// without bounds checks; scoring itself never reads past the sequence.
// Every packed sequence of the library is followed, in the same allocation,
// by its reversed copy (base i = base len-1-i of the sequence, with its own
// padding): word 0 of the copy lies sa_rev_words(len) words after word 0 of
// the sequence.  A leftward extension from position p is a rightward scan of
// the copy from position len - p.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define SA_PADW 16  // padding words on each side of a packed sequence (>= the lane kernel's read-ahead)
#define SA_NUC 8
#define SA_WARP 32
#define SA_INVALID_KEY 0xffffffffu

// Words from word 0 of a packed sequence of `len` bases to word 0 of its
// reversed copy: a multiple of 4, so that word 0 of both copies starts a
// 16-byte chunk.
__host__ __device__ __forceinline__ uint64_t sa_rev_words(uint64_t len) {
    return ((len + 7) / 8 + 2 * SA_PADW + 3) & ~3ull;
}

// Filter parameters (src/seed_filter.cu:20-27; InitializeProcessor :780-796).
struct SaParams {
    int32_t sub_mat[64];   // row = target code, column = query code
    int32_t xdrop;
    int32_t hspthresh;
    int32_t noentropy;
    int32_t seed_size;     // shape span (19 for 12of19)
    int32_t kmer_size;     // K
    int32_t transition;
    int32_t shape_pos[32];
};

// A query (or target-as-query) view used by one extension unit.
struct SaSeqView {
    const uint32_t* packed;  // points at word 0 (padding precedes it)
    uint32_t len;
};

// Per compacted seed (seed with >= 1 hit), struct-of-arrays in the workspace.
//   E[c]     exclusive prefix of hits (uint64), E[nnz] = total hits
//   lo[c]    first bucket entry in the position table
//   qpos[c]  query position j (seed word low 32 bits)
//   scope[c] dedup scope (MAX_HITS iteration, or unit/iteration in batches)
//   unit[c]  extension unit (query view, strand, rm window)
struct SaSeedList {
    uint64_t* E;
    uint32_t* lo;
    uint32_t* qpos;
    uint32_t* scope;
    uint32_t* unit;
};

// Extension unit: what a hit needs besides its two coordinates.
struct SaUnit {
    const uint32_t* q_packed;
    uint32_t q_len;
    uint32_t rm_lo, rm_hi;   // rm window on ref_loc, inclusive
    uint32_t flags;          // bit0 = rm mode, bit1 = rev (rm coordinate flip)
};

// Survivor record (segmentPair, src/graph.h:25-30) + dedup scope.
struct SaRec {
    uint32_t ref_start;
    uint32_t query_start;
    uint32_t len;
    int32_t score;
};

// Long-extension queue entry (hits whose X-drop ran past the lane-per-hit cap).
struct SaLongHit {
    uint32_t ref_loc;
    uint32_t query_loc;
    uint32_t unit;
    uint32_t scope;
};

// Device-side counters of one call.
struct SaCounters {
    unsigned long long num_hits;       // total hits (ungapped extensions)
    unsigned long long nnz;            // seeds with >= 1 hit
    unsigned long long hit_cursor;     // extension work counter
    unsigned long long long_count;     // hits in the long queue
    unsigned long long long_cursor;
    unsigned long long surv_count;     // survivors appended
    unsigned long long extended;       // hits actually extended (rm window)
    unsigned long long base_steps;     // bases scored
    unsigned long long long_overflow;  // long-queue pushes refused (handled in place)
    unsigned long long surv_overflow;  // survivor appends refused -> error
    unsigned long long uniq_count;     // records after dedup
    unsigned long long num_iter;       // MAX_HITS iterations
    unsigned long long error;          // nonzero = device-side error code
    unsigned long long hash_mask;      // slots - 1 of this call's HSP hash set
    unsigned long long hash_overflow;  // inserts that found no free slot
    unsigned long long hash_used;      // slots claimed in the HSP set (entries of its used list)
    unsigned long long pad[3];         // device-side counts of the dedup stages
};

// Open-addressing set of distinct HSPs of one call: slot = 16-byte key
// {(scope << 32) | ref_start, (query_start << 32) | len} claimed with a
// 128-bit compare-and-swap (all ones = empty), plus the score.  Within one
// scope the score is a function of the key (sum of substitution scores over
// the segment, entropy of its base counts), so equal keys are equal records.
// Every claimed slot is also appended to `used`; the compaction reads the
// distinct HSPs from that list and empties those slots again, so the set is
// left empty for the next call without clearing the whole table.
struct SaHashSet {
    unsigned long long* keys;  // [2 * slots]
    int32_t* score;            // [slots]
    unsigned long long* used;  // [used_cap] claimed slots, in claim order
    unsigned long long used_cap;
};

#define SA_HASH_MAX_PROBES 4096

__device__ __forceinline__ void sa_cas128(unsigned long long* p, unsigned long long c0, unsigned long long c1,
                                          unsigned long long v0, unsigned long long v1, unsigned long long& o0,
                                          unsigned long long& o1) {
    asm volatile(
        "{\n\t.reg .b128 d, b, c;\n\t"
        "mov.b128 b, {%2, %3};\n\t"
        "mov.b128 c, {%4, %5};\n\t"
        "atom.global.cas.b128 d, [%6], b, c;\n\t"
        "mov.b128 {%0, %1}, d;\n\t}"
        : "=l"(o0), "=l"(o1)
        : "l"(c0), "l"(c1), "l"(v0), "l"(v1), "l"(p)
        : "memory");
}

__device__ __forceinline__ unsigned long long sa_hash_mix(unsigned long long a, unsigned long long b) {
    unsigned long long x = a * 0x9e3779b97f4a7c15ull ^ (b + 0x632be59bd9b4e019ull + (a << 6) + (a >> 2));
    x ^= x >> 31;
    x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 29;
    return x;
}

// Inserts one HSP; returns the slot it claimed when it was new, else ~0.
// Counts an overflow when no slot was found within SA_HASH_MAX_PROBES (the
// set is too small).  The caller records claimed slots (sa_hash_note_used).
__device__ __forceinline__ unsigned long long sa_hash_insert(const SaHashSet& hs, unsigned long long mask,
                                                             uint32_t scope, uint32_t rs, uint32_t qs, uint32_t len,
                                                             int32_t score, unsigned long long* overflow) {
    const unsigned long long k0 = ((unsigned long long)scope << 32) | rs;
    const unsigned long long k1 = ((unsigned long long)qs << 32) | len;
    unsigned long long h = sa_hash_mix(k0, k1) & mask;
    for (int probe = 0; probe < SA_HASH_MAX_PROBES; ++probe) {
        unsigned long long o0, o1;
        sa_cas128(hs.keys + 2 * h, ~0ull, ~0ull, k0, k1, o0, o1);
        if (o0 == ~0ull && o1 == ~0ull) {
            hs.score[h] = score;
            return h;
        }
        if (o0 == k0 && o1 == k1) return ~0ull;
        h = (h + 1) & mask;
    }
    atomicAdd(overflow, 1ull);
    return ~0ull;
}

#define SA_HASH_LOOKUP_PROBES 64

// Whether the set already holds the key (scope, rs, qs, len).  Read-only and
// conservative.  Slots are read from L2 (.cg: no line from an earlier call can
// answer), a key never changes once its 128-bit CAS has written it, and a
// slot seen empty or half-written ends the search with false, as does a long
// probe chain.  A true answer therefore means an HSP with exactly this key was
// kept by this call; false only sends the caller down the full insert path.
__device__ __forceinline__ bool sa_hash_contains(const SaHashSet& hs, unsigned long long mask, uint32_t scope,
                                                 uint32_t rs, uint32_t qs, uint32_t len) {
    const unsigned long long k0 = ((unsigned long long)scope << 32) | rs;
    const unsigned long long k1 = ((unsigned long long)qs << 32) | len;
    unsigned long long h = sa_hash_mix(k0, k1) & mask;
    for (int probe = 0; probe < SA_HASH_LOOKUP_PROBES; ++probe) {
        unsigned long long s0, s1;
        asm volatile("ld.global.cg.v2.u64 {%0, %1}, [%2];" : "=l"(s0), "=l"(s1) : "l"(hs.keys + 2 * h));
        if (s0 == k0 && s1 == k1) return true;
        if (s0 == ~0ull || s1 == ~0ull) return false;
        h = (h + 1) & mask;
    }
    return false;
}

__device__ __forceinline__ uint32_t sa_lanemask_lt();

// Appends the slots claimed by the lanes of a warp (slot != ~0) to the set's
// used list; called by all 32 lanes together.
__device__ __forceinline__ void sa_hash_note_used(const SaHashSet& hs, unsigned long long* hash_used,
                                                  unsigned long long slot) {
    const bool c = slot != ~0ull;
    const uint32_t m = __ballot_sync(0xffffffffu, c);
    if (!m) return;
    const int leader = __ffs(m) - 1;
    unsigned long long base = 0;
    if ((int)(threadIdx.x & 31) == leader) base = atomicAdd(hash_used, (unsigned long long)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (c) {
        const unsigned long long i = base + __popc(m & sa_lanemask_lt());
        if (i < hs.used_cap) hs.used[i] = slot;
    }
}

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t sa_lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// 8 consecutive codes starting at base position p (may be negative down to
// -8*SA_PADW): nibble k of the result is the code of base p+k.
__device__ __forceinline__ uint32_t sa_load8(const uint32_t* __restrict__ packed, int64_t p) {
    int64_t w = p >> 3;  // floor division (arithmetic shift)
    uint32_t sh = (uint32_t)(p & 7) * 4u;
    uint32_t lo = __ldg(packed + w);
    uint32_t hi = __ldg(packed + w + 1);
    return __funnelshift_r(lo, hi, sh);
}

// Per-base match counts over nb >= 1 consecutive positions from rp (target
// R) and qp (query Q): c[b] += #positions whose codes are equal and == b, for
// b in 0..3 (the A/C/G/T counts of src/seed_filter.cu:580-598).  One new word
// per sequence per 8 bases; the counts come from bit planes of the target
// codes at the matching nibbles (code bit 0, bit 1, both).
__device__ __forceinline__ void sa_count_matches_span(const uint32_t* __restrict__ R, int64_t rp,
                                                      const uint32_t* __restrict__ Q, int64_t qp, int64_t nb,
                                                      int* c) {
    const uint32_t* pr = R + (rp >> 3);
    const uint32_t* pq = Q + (qp >> 3);
    const uint32_t shr = (uint32_t)(rp & 7) * 4u, shq = (uint32_t)(qp & 7) * 4u;
    uint32_t r0 = __ldg(pr), q0 = __ldg(pq);
    int n = 0, n0 = 0, n1 = 0, n01 = 0;
    for (int64_t i = 0; i < nb; i += 8) {
        ++pr;
        ++pq;
        const uint32_t r1 = __ldg(pr), q1 = __ldg(pq);
        const uint32_t rw = __funnelshift_r(r0, r1, shr), qw = __funnelshift_r(q0, q1, shq);
        r0 = r1;
        q0 = q1;
        uint32_t d = rw ^ qw;
        d |= d >> 1;
        d |= d >> 2;  // bit 4k set: codes of base k differ
        uint32_t v = ~(d | (rw >> 2) | (rw >> 3)) & 0x11111111u;  // equal codes in 0..3
        if (nb - i < 8) v &= (1u << (4u * (uint32_t)(nb - i))) - 1u;
        const uint32_t b0 = rw & v, b1 = (rw >> 1) & v;
        n += __popc(v);
        n0 += __popc(b0);
        n1 += __popc(b1);
        n01 += __popc(b0 & b1);
    }
    c[0] += n - n0 - n1 + n01;
    c[1] += n0 - n01;
    c[2] += n1 - n01;
    c[3] += n01;
}

__device__ __forceinline__ uint32_t sa_code_at(const uint32_t* __restrict__ packed, int64_t p) {
    return (__ldg(packed + (p >> 3)) >> ((uint32_t)(p & 7) * 4u)) & 0xfu;
}

// Per-base match counts (R == Q == b, b in 0..3) over 8 packed bases, only for
// the nibbles selected by `nmask` (one bit per nibble, bit k = base k).
__device__ __forceinline__ void sa_count_matches8(uint32_t rw, uint32_t qw, uint32_t nmask,
                                                  int* c) {
    uint32_t eq = ~(rw ^ qw);
    eq = eq & (eq >> 1) & (eq >> 2) & (eq >> 3) & 0x11111111u;  // nibble equal -> bit 0 set
    uint32_t sel = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) sel |= ((nmask >> k) & 1u) << (4 * k);
    eq &= sel;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        uint32_t t = ~(rw ^ (0x11111111u * (uint32_t)b));
        t = t & (t >> 1) & (t >> 2) & (t >> 3) & 0x11111111u;
        c[b] += __popc(eq & t);
    }
}

#define SA_CUDA_OK(expr)                                   \
    do {                                                   \
        cudaError_t _e = (expr);                           \
        if (_e != cudaSuccess) return sa_cuda_fail(_e, #expr, __FILE__, __LINE__); \
    } while (0)

int sa_cuda_fail(cudaError_t e, const char* what, const char* file, int line);
