// sa_extend.cu — ungapped X-drop extension of every seed hit, HSP keep/score
// (entropy adjustment) and survivor compaction.
//
// Reference: find_hsps (src/seed_filter.cu:204-624; repeat-masker variant
// repeat_masker_src/seed_filter.cu:249-688) and compress_output (:626-652;
// rm :690-721).  The reference runs one warp per hit over 32-base tiles with
// four shuffle scans per tile.  Its result does not depend on the tile width.
// For each direction it is defined per position:
//   S(o) = running score, M(o) = max(0, max S up to o),
//   stop at the first o with M(o) - S(o) > xdrop or at the sequence edge,
//   best = max over o < stop, pos = first o reaching best (right: -1 if
//   best == 0; left: 0).
// This file computes the same quantities in two phases:
//   phase A (sa_k_extend_lane): one hit per lane.  A warp keeps its 32 lanes
//     busy by handing out the next hits of its tile, in order, to lanes that
//     finish.  Hits are expanded on the fly from the compacted seed
//     list.  The short random-hit extensions that dominate the hit count
//     finish here in a few steps.
//   phase B (sa_k_extend_warp): hits whose extension passes `lane_cap` bases in
//     one direction move to a queue and are redone by one warp per hit,
//     256 bases per step.  Each lane scans 8 bases; warp scans carry the
//     running sum and maximum.
// Kept HSPs, with their dedup scope, go into the call's set of distinct HSPs
// (SaHashSet), which the dedup stage compacts and sorts.
#include <algorithm>
#include <climits>
#include <mutex>

#include "sa_launch.h"
#include "sa_radix.cuh"

#define SA_FULL 0xffffffffu
#define SA_LANE_TABLES 256  // lane kernel: the 64-entry score table

struct SaExtK {
    const uint32_t* ref;
    uint32_t ref_len;
    const uint32_t* pos_table;
    SaSeedList cs;
    const SaUnit* units;
    SaCounters* ctr;
    SaLongHit* long_q;
    uint64_t long_cap;
    SaHashSet hset;
    uint32_t seed_size;
    int32_t xdrop, hspthresh, noentropy;
    uint32_t lane_cap;
    uint32_t tile_hits;
    uint32_t substeps;  // steps per lane-kernel iteration (at most)
    uint32_t switch_now;  // 1: a lane starts its left side in the step after its right side ends
    uint32_t windowed;    // 1: hits outside their unit's rm window are dropped from the tiles
};

// Reverse the order of the 8 nibbles of a word.
__device__ __forceinline__ uint32_t sa_rev_nibbles(uint32_t x) {
    x = __byte_perm(x, 0, 0x0123);
    return ((x >> 4) & 0x0f0f0f0fu) | ((x & 0x0f0f0f0fu) << 4);
}

// Largest compacted seed c in [0, nnz) with E[c] <= h (E strictly increasing,
// E[0] == 0 <= h).  Warp-cooperative 32-ary search; all lanes get the result.
__device__ __forceinline__ uint64_t sa_warp_find_seed(const uint64_t* __restrict__ E, uint64_t nnz, uint64_t h) {
    const int lane = threadIdx.x & 31;
    uint64_t lo = 0, hi = nnz;
    while (hi - lo > 32) {
        uint64_t step = (hi - lo + 31) / 32;
        uint64_t probe = lo + (uint64_t)lane * step;
        bool ok = probe < hi && E[probe] <= h;
        uint32_t m = __ballot_sync(SA_FULL, ok);
        uint64_t k = 31 - __clz(m);
        uint64_t nlo = lo + k * step;
        hi = (nlo + step < hi) ? nlo + step : hi;
        lo = nlo;
    }
    uint64_t probe = lo + lane;
    bool ok = probe < hi && E[probe] <= h;
    uint32_t m = __ballot_sync(SA_FULL, ok);
    return lo + (31 - __clz(m));
}

// Entropy factor and keep/score of one HSP (src/seed_filter.cu:580-621).
// c[] are the match counts per base over the HSP, already summed.
__device__ __forceinline__ void sa_keep_score(int total, int ext, const int* cnt, bool entropy_branch,
                                              int hspthresh, int* keep, int* score) {
    if (!entropy_branch) {
        // E = 1.0: (int)((double)(float)total * 1.0) == (int)(float)total, score == total
        *keep = (int)(float)total >= hspthresh;
        *score = total;
        return;
    }
    double E = 1.0;  // entropy[warp_id] = 1.0f
    {
        short c0 = (short)cnt[0], c1 = (short)cnt[1], c2 = (short)cnt[2], c3 = (short)cnt[3];
        if ((int)c0 + (int)c1 + (int)c2 + (int)c3 >= 20) {
            double n = (double)(ext + 1);
            double e = 0.0;
            // one log at a time (same accumulation order): keeps the register peak low
#pragma unroll 1
            for (int b = 0; b < 4; ++b) {
                const short cb = b == 0 ? c0 : b == 1 ? c1 : b == 2 ? c2 : c3;
                double q = (double)cb / n;
                double lg = (cb != 0) ? log((double)cb / n) : 0.0;
                e = fma(q, lg, e);
            }
            E = -e / (double)logf(4.0f);
        }
    }
    *keep = (int)(((double)(float)total) * E) >= hspthresh;
    *score = E > 0 ? (int)((double)total * E) : 0;
}

__device__ __forceinline__ bool sa_entropy_branch(const SaExtK& a, int total) {
    return !a.noentropy && total >= a.hspthresh && total <= 3 * a.hspthresh;
}

// ---------------------------------------------------------------------------
// Phase A: one hit per lane.
//
// A warp takes tiles of consecutive hits from a global counter and expands
// each tile once into shared memory ({ref_loc, query_loc, scope, unit} per
// hit).  At the top of every iteration the lanes without a hit take the next
// records of the tile, in order, and start them in the same iteration.
// Both directions of a hit run the same rightward scan: the left
// extension from (rl, ql) is the right extension from (ref_len - rl,
// qlen - ql) in the reversed copies that follow every packed sequence, so
// lanes in different directions execute the same instructions.  A step
// scores STEP bases as 8-base windows; the target and query words of the
// next step are loaded while the current one is scored.
//
// Fast scoring form.  Inside a step, scores are kept relative to the best
// score at the step start and packed with the base index k (0..STEP-1):
//     P(k) = SCALE * (S(k) - best_in) + (STEP - 1 - k),   SCALE = 2 * STEP,
// so a running max over P yields the best score together with the FIRST base
// that reached it; the best carried in from earlier steps enters as
// STEP, which no base of the step ties.  The X-drop stop test runs once
// per 8-base window: with m = the window's minimum score and b = the best
// score at the window's end, a base of the window stops the scan iff
// b - m > xdrop, provided 7 * max(0, max_sub) <= xdrop (max_sub = largest
// substitution score).  If b was reached at or before the minimum's base,
// that base itself has best - S = b - m; otherwise b - m is a climb over at
// most 7 bases, <= xdrop, and no base has best - S above b - m.  The same
// bound shows that no base after a stop in the window can raise the best
// (that takes a climb of more than xdrop), so the window's best is the best
// at the stop.  Bases past the sequence end score -(xdrop + 1): the first of
// them stops the scan.  The test runs on the packed values themselves:
// with B = SCALE * b + i (i in 0..STEP) and min = SCALE * m + j (j in
// 0..STEP-1), b - m > xdrop  <=>  B - min > SCALE * xdrop + STEP.
// Parameters outside the bound use the exact form, which tests every base.
// ---------------------------------------------------------------------------
// Byte b of lo (hi) = byte offset ((q << 3) | r) * 4 of the score of base 2b
// (2b+1) in a 64-entry int table; codes are 0..7, so a byte never carries.
__device__ __forceinline__ void sa_merge8(uint32_t rw, uint32_t qw, uint32_t& lo, uint32_t& hi) {
    lo = ((qw & 0x07070707u) << 5) | ((rw & 0x07070707u) << 2);
    hi = (((qw >> 4) & 0x07070707u) << 5) | (((rw >> 4) & 0x07070707u) << 2);
}

__device__ __forceinline__ int sa_tbl(const char* tblb, uint32_t lo, uint32_t hi, int kk) {
    const uint32_t byte = __byte_perm((kk & 1) ? hi : lo, 0, 0x4440 | (kk >> 1));
    return *reinterpret_cast<const int*>(tblb + byte);
}

// Fast form, one 8-base window.  P = packed running score, B = packed
// running best; `at` takes B at the end of each window up to and including
// the one that stops; `stop` is set by that window.  EDGE: bases at
// off0 + k >= avail score `neg`.
template <bool EDGE>
__device__ __forceinline__ void sa_window_fast(const char* tblb, uint32_t lo, uint32_t hi, uint32_t off0,
                                               uint32_t avail, int neg, uint32_t T, int& P, int& B, int& at,
                                               bool& stop) {
    int mn = INT_MAX;
    // Bases in pairs: the running best and minimum take both prefixes of a
    // pair with one 3-input max / min (DPX on sm_90 and later).
#pragma unroll
    for (int kk = 0; kk < 8; kk += 2) {
        int t0 = sa_tbl(tblb, lo, hi, kk);
        int t1 = sa_tbl(tblb, lo, hi, kk + 1);
        if (EDGE && off0 + kk >= avail) t0 = neg;
        if (EDGE && off0 + kk + 1 >= avail) t1 = neg;
        const int P0 = P + t0;
        P = P0 + t1;
        B = __vimax3_s32(B, P0, P);
        mn = __vimin3_s32(mn, P0, P);
    }
    if (!stop) at = B;
    stop = stop || (uint32_t)(B - mn) > T;
}

// Exact form, one 8-base window at step-relative indices k0..k0+7: S =
// running score, best = running maximum (from 0), pk = step-relative index
// of the last strict increase of best, alive cleared at the first base with
// best - S > xdrop or (EDGE) at off0 + k >= avail.
template <bool EDGE>
__device__ __forceinline__ void sa_window_exact(const char* tblb, uint32_t lo, uint32_t hi, int k0, uint32_t off0,
                                                uint32_t avail, int xdrop, int& S, int& best, int& pk, bool& alive) {
#pragma unroll
    for (int kk = 0; kk < 8; ++kk) {
        const int sc = sa_tbl(tblb, lo, hi, kk);
        if (EDGE && off0 + kk >= avail) alive = false;
        S += sc;
        const bool up = alive && S > best;
        best = up ? S : best;
        pk = up ? k0 + kk : pk;
        alive = alive && (best - S <= xdrop);
    }
}

// Keep test of `n` (<= 32) ring candidates from slot `head` on, one per lane:
// entropy factor from the per-base match counts over the HSP when the total
// is in the entropy range (src/seed_filter.cu:580-621), then insertion of the
// kept ones into the call's set of distinct HSPs (rm: query start flipped on
// the reverse strand, repeat_masker_src/seed_filter.cu:704-707).  Called by
// the whole warp; leaves the slots free for reuse.
__device__ __forceinline__ void sa_flush_candidates(const SaExtK& a, const uint4* s_em, const uint2* s_ex,
                                                    uint32_t head, uint32_t n) {
    const int lane = threadIdx.x & 31;
    const bool on = (uint32_t)lane < n;
    uint4 r = make_uint4(0, 0, 0, 0);
    uint2 x = make_uint2(0, 0);
    if (on) {
        const uint32_t slot = (head + lane) & 63u;
        r = s_em[slot];
        x = s_ex[slot];
    }
    __syncwarp();  // slots are rewritten by later appends
    int keep = 0, score = 0;
    bool known = false;
    uint32_t qs = 0;
    if (on) {
        const SaUnit U = a.units[x.y];
        const int total = (int)x.x, ext = (int)r.z;
        qs = r.y;
        if (U.flags & 2u) qs = a.ref_len - 1 - (qs + r.z);
        // A candidate whose key the set already holds was kept with this same
        // key (the scope fixes the unit, so the same bases): it is a survivor,
        // and its match counts, logs and insertion are skipped.
        known = sa_hash_contains(a.hset, a.ctr->hash_mask, r.w, r.x, qs, r.z);
        if (known) {
            keep = 1;
        } else {
            int cnt[4] = {0, 0, 0, 0};
            const bool eb = sa_entropy_branch(a, total);
            if (eb) sa_count_matches_span(a.ref, r.x, U.q_packed, r.y, (int64_t)ext + 1, cnt);
            sa_keep_score(total, ext, cnt, eb, a.hspthresh, &keep, &score);
        }
    }
    const uint32_t km = __ballot_sync(SA_FULL, keep != 0);
    if (lane == 0 && km) atomicAdd(&a.ctr->surv_count, (unsigned long long)__popc(km));
    unsigned long long claimed = ~0ull;
    if (keep && !known)
        claimed = sa_hash_insert(a.hset, a.ctr->hash_mask, r.w, r.x, qs, r.z, score, &a.ctr->hash_overflow);
    sa_hash_note_used(a.hset, &a.ctr->hash_used, claimed);
}

// Dynamic shared memory of the lane kernel for `tile` hits per warp tile.
static size_t sa_lane_smem(uint32_t tile) {
    return SA_LANE_TABLES + 8 * (size_t)tile * 16 + 8 * (size_t)(tile + 1) * 8 + 8 * 64 * 16 + 8 * 64 * 8;
}

template <int MIN_CTAS, int STEP, bool EXACT>
__global__ void __launch_bounds__(256, MIN_CTAS)
sa_k_extend_lane(SaExtK a, SaParams P) {
    constexpr int NW = STEP / 8;                  // 8-base windows per step
    constexpr int SCALE = 2 * STEP;               // packed score scale (fast form)
    constexpr int SH = STEP == 8 ? 4 : STEP == 16 ? 5 : 6;  // log2(SCALE)
    static_assert(STEP == 8 || STEP == 16 || STEP == 32, "8-, 16- or 32-base steps");
    // Read-ahead: the last step reads up to 2 * NW + 1 words past the last base.
    static_assert(2 * NW + 2 <= SA_PADW, "padding shorter than the read-ahead");
    // Shared memory: score table (64 ints), then per warp: tile records,
    // tile E window, and a 64-entry ring of candidate HSPs awaiting the keep
    // test and insertion.
    extern __shared__ __align__(16) unsigned char sa_smem[];
    const uint32_t TILE = a.tile_hits;
    // entry (q << 3) | r: target code r vs query code q.  Codes 0..3 use
    // entries 0..27 only, one per bank: lookups of A/C/G/T pairs never conflict.
    int* tbl = reinterpret_cast<int*>(sa_smem);
    if (threadIdx.x < 64) {
        const int sc = P.sub_mat[(threadIdx.x & 7) * 8 + (threadIdx.x >> 3)];
        tbl[threadIdx.x] = EXACT ? sc : sc * SCALE - 1;
    }
    __syncthreads();
    const char* tblb = reinterpret_cast<const char*>(tbl);
    if (a.ctr->error) return;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t lt = sa_lanemask_lt();
    uint4* const s_hits = reinterpret_cast<uint4*>(sa_smem + SA_LANE_TABLES) + wid * TILE;
    unsigned long long* const s_E =
        reinterpret_cast<unsigned long long*>(sa_smem + SA_LANE_TABLES + 128 * (size_t)TILE) + wid * (TILE + 1);
    unsigned char* const em_base = sa_smem + SA_LANE_TABLES + 128 * (size_t)TILE + 64 * (size_t)(TILE + 1);
    uint4* const s_em = reinterpret_cast<uint4*>(em_base) + wid * 64;
    uint2* const s_ex = reinterpret_cast<uint2*>(em_base + 8 * 64 * 16) + wid * 64;

    // H, nnz, ref_len, seed_size and xdrop are read where used (registers
    // are the lane kernel's limit)
    const uint32_t* __restrict__ ref = a.ref;

    uint32_t tile_pos = 0, tile_n = 0;
    bool exhausted = false;
    uint32_t em_head = 0, em_tail = 0;  // ring of kept HSPs (warp-uniform cursors)

    // current hit
    bool has = false, nocap = false, setup = false;
    uint32_t rl = 0, ql = 0, scope = 0, unit_id = 0;
    int dir = 0;
    // scan of the current direction: offset, bases available, word shifts,
    // words w[0..NW] of the coming step, next word addresses
    uint32_t o = 0, avail = 0, sh_r = 0, sh_q = 0;
    uint32_t w_r[NW + 1], w_q[NW + 1];
#pragma unroll
    for (int j = 0; j <= NW; ++j) w_r[j] = w_q[j] = 0;
    const uint32_t* __restrict__ pr = ref;
    const uint32_t* __restrict__ pq = ref;
    // running score, best, offset of the first base reaching best
    int S = 0, best = 0, bpos = 0, Rbest = 0, Rpos = -1;
    uint32_t tiles = 0, tiles_acc = 0, ext_acc = 0;  // per-lane statistics (32-bit per lane)

    // Start of a direction of the current hit (dir 0: right of the hit; 1:
    // left, read rightwards in the reversed copies): offsets, bases
    // available, word shifts and the first NW + 1 words of both sequences.
    auto begin_dir = [&](const uint32_t* __restrict__ qp, uint32_t qlen) {
        const uint32_t ref_len = a.ref_len;
        const uint32_t sr = dir ? ref_len - rl : rl, sq = dir ? qlen - ql : ql;
        avail = min(ref_len - sr, qlen - sq);
        sh_r = (sr & 7u) * 4u;
        sh_q = (sq & 7u) * 4u;
        pr = (dir ? ref + sa_rev_words(ref_len) : ref) + (sr >> 3);
        pq = (dir ? qp + sa_rev_words(qlen) : qp) + (sq >> 3);
#pragma unroll
        for (int j = 0; j <= NW; ++j) {
            w_r[j] = __ldg(pr + j);
            w_q[j] = __ldg(pq + j);
        }
        pr += NW + 1;
        pq += NW + 1;
        o = 0;
        S = 0;
        best = 0;
        bpos = 0;
    };

    while (true) {
        // ---- idle lanes take the next hits of the warp tile, in order ----
        const uint32_t idle = __ballot_sync(SA_FULL, !has);
        bool fresh = false;
        if (idle && !(exhausted && tile_pos >= tile_n)) {
            if (tile_pos >= tile_n) {
                // Take the next tile of hits and expand it: the hits of the
                // tile span at most TILE consecutive hit-bearing seeds from the
                // one holding its first hit, so E over that window locates each
                // hit's seed by binary search.
                unsigned long long t0 = 0;
                if (lane == 0) t0 = atomicAdd(&a.ctr->hit_cursor, (unsigned long long)TILE);
                t0 = __shfl_sync(SA_FULL, t0, 0);
                const uint64_t H = a.ctr->num_hits, nnz = a.ctr->nnz;
                if (t0 >= H) {
                    exhausted = true;
                    tile_n = tile_pos = 0;
                } else {
                    uint32_t n = (uint32_t)min((unsigned long long)TILE, H - t0);
                    const uint64_t c0 = sa_warp_find_seed(a.cs.E, nnz, t0);
                    const uint32_t nw = (uint32_t)min((uint64_t)n, nnz - c0);  // seeds of the window
                    for (uint32_t i = lane; i <= nw; i += 32) s_E[i] = a.cs.E[c0 + i];  // E[nnz] == H
                    __syncwarp();
                    // record of hit t0 + i: its seed by binary search in the E window
                    auto record = [&](uint32_t i) {
                        const unsigned long long h = t0 + i;
                        uint32_t lo = 0, hi = nw;  // last k in [0, nw) with E[c0+k] <= h
                        while (hi - lo > 1) {
                            const uint32_t mid = (lo + hi) >> 1;
                            if (s_E[mid] <= h) lo = mid;
                            else hi = mid;
                        }
                        const uint64_t c = c0 + lo;
                        uint4 r;
                        r.x = __ldg(a.pos_table + a.cs.lo[c] + (uint32_t)(h - s_E[lo])) + a.seed_size;  // find_hits :192
                        r.y = a.cs.qpos[c] + a.seed_size;                                                 // find_hits :176
                        r.z = a.cs.scope[c];
                        r.w = a.cs.unit[c];
                        return r;
                    };
                    if (!a.windowed) {
                        for (uint32_t i = lane; i < n; i += 32) s_hits[i] = record(i);
                    } else {
                        // rm: hits outside [ref_start, ref_end] are never extended
                        // (repeat_masker_src/seed_filter.cu:237-243, 304-333); the
                        // tile keeps only the others, in order, so that no lane is
                        // handed a hit it would skip.  Coordinates past either
                        // sequence end are rejected here too.
                        uint32_t kept = 0;
                        for (uint32_t i0 = 0; i0 < n; i0 += 32) {
                            bool live = false;
                            uint4 r = make_uint4(0, 0, 0, 0);
                            if (i0 + lane < n) {
                                r = record(i0 + lane);
                                const SaUnit U = a.units[r.w];
                                live = !(U.flags & 1u) || (r.x >= U.rm_lo && r.x <= U.rm_hi);
                                if (!live && (r.x > a.ref_len || r.y > U.q_len)) atomicCAS(&a.ctr->error, 0ull, 5ull);
                            }
                            const uint32_t m = __ballot_sync(SA_FULL, live);
                            if (live) s_hits[kept + __popc(m & lt)] = r;
                            kept += __popc(m);
                        }
                        n = kept;
                    }
                    __syncwarp();
                    tile_n = n;
                    tile_pos = 0;
                }
            }
            if (tile_pos < tile_n) {
                const uint32_t m = min((uint32_t)__popc(idle), tile_n - tile_pos);
                const uint32_t rank = __popc(idle & lt);
                if (!has && rank < m) {
                    const uint4 r = s_hits[tile_pos + rank];
                    rl = r.x;
                    ql = r.y;
                    scope = r.z;
                    unit_id = r.w;
                    fresh = true;
                }
                tile_pos += m;
            }
        }

        // ---- start of a direction: a fresh hit (right), or the left side of
        // the current hit after its right end ----
        if (fresh || setup) {
            const SaUnit U = a.units[unit_id];
            if (fresh) {
                // rm: hits outside [ref_start, ref_end] are never extended
                // (repeat_masker_src/seed_filter.cu:237-243, 304-333).
                bool skip = (U.flags & 1u) && !(rl >= U.rm_lo && rl <= U.rm_hi);
                // Coordinates past either sequence end (a caller-supplied table or
                // seed beyond the sequences) are rejected, not read.
                if (rl > a.ref_len || ql > U.q_len) {
                    atomicCAS(&a.ctr->error, 0ull, 5ull);
                    skip = true;
                }
                if (!skip) {
                    has = true;
                    nocap = false;
                    setup = true;
                    dir = 0;
                    tiles = 0;
                    ++ext_acc;
                }
            }
            if (setup) {
                setup = false;
                begin_dir(U.q_packed, U.q_len);
            }
        }
        const bool done = !__any_sync(SA_FULL, has) && exhausted && tile_pos >= tile_n;

        // ---- up to `substeps` STEP-base steps per busy lane: the lanes still
        // scanning go on while any lane of the warp does; a lane stops for
        // this iteration when its direction ends or it goes to the long queue ----
        bool finished = false, to_long = false;
        int Lpos = 0, total = 0;
        bool scanning = has;
#pragma unroll 1
        for (uint32_t sub = 0; sub < a.substeps; ++sub) {
            if (!__any_sync(SA_FULL, scanning)) break;
            if (scanning) {
                uint32_t rwin[NW], qwin[NW];
    #pragma unroll
                for (int j = 0; j < NW; ++j) {
                    rwin[j] = __funnelshift_r(w_r[j], w_r[j + 1], sh_r);
                    qwin[j] = __funnelshift_r(w_q[j], w_q[j + 1], sh_q);
                }
                w_r[0] = w_r[NW];
                w_q[0] = w_q[NW];
    #pragma unroll
                for (int j = 1; j <= NW; ++j) {
                    w_r[j] = __ldg(pr + j - 1);
                    w_q[j] = __ldg(pq + j - 1);
                }
                pr += NW;
                pq += NW;
                const bool edge = o + STEP > avail;
                bool stop = false;
                uint32_t lo, hi;
                if (EXACT) {
                    bool alive = true;
                    int pk = 0;
                    const int best_in = best;
                    if (!edge) {
    #pragma unroll
                        for (int j = 0; j < NW; ++j) {
                            sa_merge8(rwin[j], qwin[j], lo, hi);
                            sa_window_exact<false>(tblb, lo, hi, 8 * j, o + 8 * j, avail, a.xdrop, S, best, pk, alive);
                        }
                    } else {
    #pragma unroll
                        for (int j = 0; j < NW; ++j) {
                            sa_merge8(rwin[j], qwin[j], lo, hi);
                            sa_window_exact<true>(tblb, lo, hi, 8 * j, o + 8 * j, avail, a.xdrop, S, best, pk, alive);
                        }
                    }
                    if (best != best_in) bpos = (int)o + pk;
                    stop = !alive;
                } else {
                    // B - min > SCALE * xdrop + STEP  <=>  (B >> SH) - (min >> SH) > xdrop, because
                    // the low parts of B (0..STEP) and min (0..STEP-1) differ by less than SCALE
                    const uint32_t T = (uint32_t)a.xdrop * SCALE + STEP;
                    int Pk = ((S - best) << SH) + STEP, B = STEP, at = 0;
                    if (!edge) {
    #pragma unroll
                        for (int j = 0; j < NW; ++j) {
                            sa_merge8(rwin[j], qwin[j], lo, hi);
                            sa_window_fast<false>(tblb, lo, hi, o + 8 * j, avail, 0, T, Pk, B, at, stop);
                        }
                    } else {
    #pragma unroll
                        for (int j = 0; j < NW; ++j) {
                            sa_merge8(rwin[j], qwin[j], lo, hi);
                            // a base past the sequence end scores -(xdrop + 1)
                            sa_window_fast<true>(tblb, lo, hi, o + 8 * j, avail, -(a.xdrop + 1) * SCALE - 1, T, Pk,
                                                 B, at, stop);
                        }
                    }
                    const int low = at & (SCALE - 1);
                    if (low != STEP) bpos = (int)o + (STEP - 1 - low);
                    const int best_in = best;
                    best = best_in + (at >> SH);
                    S = best_in + (Pk >> SH);  // exact after a full step without a stop
                }
                if (stop) {
                    // Steps start at multiples of STEP (8, 16 or 32), so the stop offset
                    // lies in 32-base tile o >> 5 whichever base of the step it is.
                    tiles += (o >> 5) + 1;
                    if (dir == 0) {
                        Rbest = best;
                        Rpos = best > 0 ? bpos : -1;  // -1 when no positive score
                        dir = 1;
                        setup = true;
                    } else {
                        finished = true;
                    }
                    scanning = false;
                } else {
                    o += STEP;
                    if (o >= a.lane_cap && !nocap) {
                        to_long = true;
                        scanning = false;
                    }
                }
                if (finished) {
                    Lpos = best > 0 ? bpos + 1 : 0;  // left offsets are 1-based
                    total = Rbest + best;
                    tiles_acc += tiles;
                    has = false;
                }
            }
            // switch_now: a lane whose right side ended in this step starts
            // its left side at once and scans in the iteration's remaining
            // steps instead of idling until the next iteration
            if (a.switch_now && sub + 1 < a.substeps && __any_sync(SA_FULL, setup)) {
                if (setup) {
                    setup = false;
                    const SaUnit U = a.units[unit_id];
                    begin_dir(U.q_packed, U.q_len);
                    scanning = true;
                }
            }
        }

        // ---- long queue pushes (warp-aggregated) ----
        {
            const uint32_t lm = __ballot_sync(SA_FULL, to_long);
            if (lm) {
                const int leader = __ffs(lm) - 1;
                unsigned long long base = 0;
                if (lane == leader) base = atomicAdd(&a.ctr->long_count, (unsigned long long)__popc(lm));
                base = __shfl_sync(SA_FULL, base, leader);
                if (to_long) {
                    const unsigned long long idx = base + __popc(lm & lt);
                    if (idx < a.long_cap) {
                        SaLongHit e;
                        e.ref_loc = rl;
                        e.query_loc = ql;
                        e.unit = unit_id;
                        e.scope = scope;
                        a.long_q[idx] = e;
                        has = false;
                    } else {
                        nocap = true;  // queue full: finish this hit in the lane
                        atomicAdd(&a.ctr->long_overflow, 1ull);
                    }
                }
            }
        }
        // ---- candidate HSPs (total >= hspthresh; the entropy factor is at
        // most 1, so lower totals are never kept) into the warp's ring ----
        {
            const bool emit = finished && (int)(float)total >= a.hspthresh;
            const uint32_t em = __ballot_sync(SA_FULL, emit);
            if (emit) {
                const uint32_t slot = (em_tail + __popc(em & lt)) & 63u;
                // {ref_start, query_start (before the rm flip), len, scope}, {total, unit} (:606-608)
                s_em[slot] = make_uint4(rl - (uint32_t)Lpos, ql - (uint32_t)Lpos, (uint32_t)(Rpos + Lpos), scope);
                s_ex[slot] = make_uint2((uint32_t)total, unit_id);
            }
            em_tail += __popc(em);
            // full batches of 32; at the end, whatever is left
            while (em_tail - em_head >= 32 || (done && em_tail != em_head)) {
                const uint32_t n = min(em_tail - em_head, 32u);
                __syncwarp();
                sa_flush_candidates(a, s_em, s_ex, em_head, n);
                em_head += n;
            }
        }
        if (done) break;
    }
    // flush statistics
    unsigned long long t = tiles_acc, e = ext_acc;
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) {
        t += __shfl_xor_sync(SA_FULL, t, s);
        e += __shfl_xor_sync(SA_FULL, e, s);
    }
    if (lane == 0) {
        atomicAdd(&a.ctr->base_steps, t);
        atomicAdd(&a.ctr->extended, e);
    }
}

// ---------------------------------------------------------------------------
// Phase B: one warp per long hit, 256 bases per step.
// ---------------------------------------------------------------------------
struct SaDirResult {
    int best;
    int pos;
    uint32_t tiles;
};

__device__ __forceinline__ int sa_warp_incl_max(int v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(SA_FULL, v, o);
        if (lane >= o) v = max(v, t);
    }
    return v;
}

// (value, index) arg-max over the warp: larger value wins, ties go to the smaller index.
__device__ __forceinline__ void sa_warp_argmax(int& v, uint32_t& idx) {
    long long key = ((long long)v << 32) | (long long)(uint32_t)(~idx);
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) {
        long long o = __shfl_xor_sync(SA_FULL, key, s);
        key = o > key ? o : key;
    }
    v = (int)(key >> 32);
    idx = ~(uint32_t)(key & 0xffffffffll);
}

__device__ SaDirResult sa_warp_xdrop(const int* sub, const uint32_t* __restrict__ ref, const uint32_t* __restrict__ qp,
                                     uint32_t rl, uint32_t ql, uint32_t avail, int dir, int xdrop) {
    const int lane = threadIdx.x & 31;
    int S_prev = 0, best = 0, bpos = dir ? 0 : -1;
    uint32_t o = 0;
    SaDirResult res;
    while (true) {
        const uint32_t loff = o + 8u * lane;
        const int cnt_in = (avail > loff) ? (int)min(avail - loff, 8u) : 0;
        uint32_t rw = 0, qw = 0;
        if (cnt_in > 0) {
            if (dir == 0) {
                rw = sa_load8(ref, (int64_t)rl + loff);
                qw = sa_load8(qp, (int64_t)ql + loff);
            } else {
                rw = sa_rev_nibbles(sa_load8(ref, (int64_t)rl - loff - 8));
                qw = sa_rev_nibbles(sa_load8(qp, (int64_t)ql - loff - 8));
            }
        }
        int ps[8];
        int p = 0, lmax = INT_MIN, lmax_k = 0, lmin = INT_MAX;
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) {
            int s = (kk < cnt_in) ? sub[(((rw >> (4 * kk)) & 7u) << 3) | ((qw >> (4 * kk)) & 7u)] : 0;
            p += s;
            ps[kk] = p;
            if (kk < cnt_in) {
                if (p > lmax) {
                    lmax = p;
                    lmax_k = kk;
                }
                lmin = min(lmin, p);
            }
        }
        const int incl = sa_warp_incl_sum(p);
        const int pre = incl - p;
        const int step_total = __shfl_sync(SA_FULL, incl, 31);
        const int base = S_prev + pre;
        const int amax = cnt_in > 0 ? base + lmax : INT_MIN;
        const int im = sa_warp_incl_max(amax);
        int excl = __shfl_up_sync(SA_FULL, im, 1);
        if (lane == 0) excl = INT_MIN;
        const int Mbefore = max(best, excl);
        int stop_k = -1, bmax = INT_MIN, bmax_k = 0;
        const bool possible = (cnt_in < 8) || (max(Mbefore, amax) - (base + lmin) > xdrop);
        if (possible) {
            int M = Mbefore;
#pragma unroll
            for (int kk = 0; kk < 8; ++kk) {
                if (stop_k < 0) {
                    if (kk >= cnt_in) {
                        stop_k = kk;
                    } else {
                        const int Sv = base + ps[kk];
                        M = max(M, Sv);
                        if (M - Sv > xdrop) stop_k = kk;
                        else if (Sv > bmax) {
                            bmax = Sv;
                            bmax_k = kk;
                        }
                    }
                }
            }
        }
        const uint32_t sm = __ballot_sync(SA_FULL, stop_k >= 0);
        int cv;
        uint32_t ci;
        if (sm) {
            const int f = __ffs(sm) - 1;
            if (lane < f) {
                cv = amax;
                ci = loff + lmax_k;
            } else if (lane == f) {
                cv = bmax;
                ci = loff + bmax_k;
            } else {
                cv = INT_MIN;
                ci = 0xffffffffu;
            }
            sa_warp_argmax(cv, ci);
            if (cv > best) {
                best = cv;
                bpos = (int)ci + dir;
            }
            const uint32_t stop_idx = __shfl_sync(SA_FULL, loff + (uint32_t)stop_k, f);
            res.tiles = (stop_idx >> 5) + 1;
            break;
        }
        cv = amax;
        ci = loff + lmax_k;
        sa_warp_argmax(cv, ci);
        if (cv > best) {
            best = cv;
            bpos = (int)ci + dir;
        }
        S_prev += step_total;
        o += 256;
    }
    res.best = best;
    res.pos = bpos;
    return res;
}

__global__ void __launch_bounds__(256)
sa_k_extend_warp(SaExtK a, SaParams P) {
    __shared__ int sub[64];
    if (threadIdx.x < 64) sub[threadIdx.x] = P.sub_mat[threadIdx.x];
    __syncthreads();
    if (a.ctr->error) return;
    const int lane = threadIdx.x & 31;
    const unsigned long long nlong = min(a.ctr->long_count, (unsigned long long)a.long_cap);
    unsigned long long tiles_acc = 0;
    while (true) {
        unsigned long long idx = 0;
        if (lane == 0) idx = atomicAdd(&a.ctr->long_cursor, 1ull);
        idx = __shfl_sync(SA_FULL, idx, 0);
        if (idx >= nlong) break;
        const SaLongHit L = a.long_q[idx];
        const SaUnit U = a.units[L.unit];
        const uint32_t rl = L.ref_loc, ql = L.query_loc;
        const uint32_t avail_r = (rl < a.ref_len && ql < U.q_len) ? min(a.ref_len - rl, U.q_len - ql) : 0u;
        const SaDirResult R = sa_warp_xdrop(sub, a.ref, U.q_packed, rl, ql, avail_r, 0, a.xdrop);
        const SaDirResult Lr = sa_warp_xdrop(sub, a.ref, U.q_packed, rl, ql, min(rl, ql), 1, a.xdrop);
        tiles_acc += R.tiles + Lr.tiles;
        const int total = R.best + Lr.best;
        const int ext = R.pos + Lr.pos;
        int cnt[4] = {0, 0, 0, 0};
        const bool eb = sa_entropy_branch(a, total);
        if (eb) {
            const int64_t r0 = (int64_t)rl - Lr.pos, q0 = (int64_t)ql - Lr.pos, nb = (int64_t)ext + 1;
            for (int64_t i = 8 * lane; i < nb; i += 256) {
                uint32_t nm = (nb - i >= 8) ? 0xffu : ((1u << (uint32_t)(nb - i)) - 1u);
                sa_count_matches8(sa_load8(a.ref, r0 + i), sa_load8(U.q_packed, q0 + i), nm, cnt);
            }
#pragma unroll
            for (int b = 0; b < 4; ++b)
#pragma unroll
                for (int s = 16; s >= 1; s >>= 1) cnt[b] += __shfl_xor_sync(SA_FULL, cnt[b], s);
        }
        if (lane == 0) {
            int keep, score;
            sa_keep_score(total, ext, cnt, eb, a.hspthresh, &keep, &score);
            if (keep) {
                atomicAdd(&a.ctr->surv_count, 1ull);
                const uint32_t rs = rl - (uint32_t)Lr.pos;
                uint32_t qs = ql - (uint32_t)Lr.pos;
                const uint32_t len = (uint32_t)ext;
                if (U.flags & 2u) qs = a.ref_len - 1 - (qs + len);
                const unsigned long long cl =
                    sa_hash_insert(a.hset, a.ctr->hash_mask, L.scope, rs, qs, len, score, &a.ctr->hash_overflow);
                if (cl != ~0ull) {
                    const unsigned long long i = atomicAdd(&a.ctr->hash_used, 1ull);
                    if (i < a.hset.used_cap) a.hset.used[i] = cl;
                }
            }
        }
    }
    if (lane == 0) atomicAdd(&a.ctr->base_steps, tiles_acc);
}

static SaExtK sa_ext_args(SaWork& w, const SaExtendArgs& x, const SaTuning& t) {
    SaExtK a;
    a.ref = x.ref;
    a.ref_len = x.ref_len;
    a.pos_table = x.pos_table;
    a.cs = w.cs;
    a.units = w.units;
    a.ctr = w.ctr;
    a.long_q = w.long_q;
    a.long_cap = w.long_cap;
    a.hset = w.hset;
    a.seed_size = x.seed_size;
    a.xdrop = x.xdrop;
    a.hspthresh = x.hspthresh;
    a.noentropy = x.noentropy;
    a.lane_cap = (uint32_t)t.lane_cap;
    a.tile_hits = (uint32_t)t.tile_hits;
    a.substeps = (uint32_t)t.substeps;
    a.switch_now = t.switch_now ? 1u : 0u;
    a.windowed = x.windowed ? 1u : 0u;
    return a;
}

// The fast scoring form holds when 7 * max(0, max_sub) <= xdrop (see the
// phase A notes) and its packed scores stay inside 31 bits: a step starts at
// >= -xdrop * SCALE and adds STEP scores of >= min_sub * SCALE - 1 (or
// -(xdrop + 1) * SCALE - 1 past a sequence end).
static bool sa_lane_fast_form(const SaParams& p, int step) {
    long long mx = 0, mn = 0;
    for (int i = 0; i < 64; ++i) {
        mx = std::max<long long>(mx, p.sub_mat[i]);
        mn = std::min<long long>(mn, p.sub_mat[i]);
    }
    const long long scale = 2ll * step, x = p.xdrop;
    const long long low = std::min(mn, -(x + 1)) * scale - 1;
    return x >= 0 && 7 * mx <= x && x * scale - low * step < (1ll << 31) && mx * scale * step < (1ll << 31);
}

template <int C, int STEP, bool EXACT>
static void sa_lane_launch(const SaExtK& a, const SaParams& p, int grid, size_t smem, cudaStream_t st) {
    if (grid > 0) sa_k_extend_lane<C, STEP, EXACT><<<grid, 256, smem, st>>>(a, p);
    else cudaFuncSetAttribute(sa_k_extend_lane<C, STEP, EXACT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

template <int C>
static void sa_lane_dispatch(const SaExtK& a, const SaParams& p, int step, bool exact, int grid, size_t smem,
                             cudaStream_t st) {
    if (step == 32) {
        if (exact) sa_lane_launch<C, 32, true>(a, p, grid, smem, st);
        else sa_lane_launch<C, 32, false>(a, p, grid, smem, st);
    } else if (step == 16) {
        if (exact) sa_lane_launch<C, 16, true>(a, p, grid, smem, st);
        else sa_lane_launch<C, 16, false>(a, p, grid, smem, st);
    } else {
        if (exact) sa_lane_launch<C, 8, true>(a, p, grid, smem, st);
        else sa_lane_launch<C, 8, false>(a, p, grid, smem, st);
    }
}

// Allows every lane-kernel instance the largest tile's shared memory, once
// per device (kernel attributes cannot be set while a stream is captured).
void sa_prepare_extend_lane(const SaParams& p, const SaTuning& t) {
    (void)t;
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    if (dev < 0 || dev >= 64 || done[dev]) return;
    const size_t smem = sa_lane_smem(1024);
    SaExtK none{};
    for (int step : {8, 16, 32})
        for (bool exact : {false, true}) {
            sa_lane_dispatch<2>(none, p, step, exact, 0, smem, 0);
            sa_lane_dispatch<3>(none, p, step, exact, 0, smem, 0);
            sa_lane_dispatch<4>(none, p, step, exact, 0, smem, 0);
        }
    done[dev] = true;
}

void sa_launch_extend_lane(SaWork& w, const SaExtendArgs& x, const SaParams& p, const SaTuning& t, int num_sms,
                           cudaStream_t st, int grid_ctas) {
    sa_prepare_extend_lane(p, t);
    // Register budget follows the CTAs per SM: 4 -> <= 64 registers, 3 -> <= 85, 2 -> <= 128.
    const SaExtK a = sa_ext_args(w, x, t);
    const int grid = grid_ctas > 0 ? grid_ctas : num_sms * t.ext_ctas_per_sm;
    const size_t smem = sa_lane_smem(a.tile_hits);
    const bool exact = !sa_lane_fast_form(p, t.step_bases);
    if (t.ext_ctas_per_sm >= 4) sa_lane_dispatch<4>(a, p, t.step_bases, exact, grid, smem, st);
    else if (t.ext_ctas_per_sm == 3) sa_lane_dispatch<3>(a, p, t.step_bases, exact, grid, smem, st);
    else sa_lane_dispatch<2>(a, p, t.step_bases, exact, grid, smem, st);
    sa_note_launch();
}

void sa_launch_extend_warp(SaWork& w, const SaExtendArgs& x, const SaParams& p, const SaTuning& t, int num_sms,
                           cudaStream_t st) {
    sa_k_extend_warp<<<num_sms * 4, t.long_block, 0, st>>>(sa_ext_args(w, x, t), p);
    sa_note_launch();
}
