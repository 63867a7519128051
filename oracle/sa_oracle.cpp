// sa_oracle.cpp — CPU oracle (test infrastructure only) for the SegAlign
// seed-filter hot path.  Every function restates the reference semantics and
// cites the reference file:line it follows.  See sa_oracle.h for the pinning
// status.  Build: oracle/Makefile (g++ -O2 -std=c++17 -shared).
#include "sa_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

// Codes (common/parameters.h:4-11).
enum : uint8_t { A_NT = 0, C_NT = 1, G_NT = 2, T_NT = 3, L_NT = 4, N_NT = 5, X_NT = 6, E_NT = 7 };
constexpr uint32_t INVALID_KMER = 1u << 31;  // common/ntcoding.h:1

// common/seed_filter_interface.cu:28-46 and src/seed_filter.cu:92-123.
inline uint8_t code_of(char ch) {
    switch (ch) {
        case 'A': return A_NT;
        case 'C': return C_NT;
        case 'G': return G_NT;
        case 'T': return T_NT;
        case 'a': case 'c': case 'g': case 't': return L_NT;
        case 'n': case 'N': return N_NT;
        case '&': return E_NT;
        default: return X_NT;
    }
}

// Complement of a code (src/seed_filter.cu:96-125; rm seed_filter.cu:147-166):
// A<->T, C<->G, everything else unchanged.
inline uint8_t comp_code(uint8_t c) { return c < 4 ? (uint8_t)(3 - c) : c; }

// NtChar2Int + validity test (common/ntcoding.cpp:10-19, 47-52): only
// uppercase ACGT are valid seed characters.
inline int nt_valid(char ch, uint32_t* v) {
    switch (ch) {
        case 'A': *v = 0; return 1;
        case 'C': *v = 1; return 1;
        case 'G': *v = 2; return 1;
        case 'T': *v = 3; return 1;
        default: return 0;
    }
}

// hspComp (src/seed_filter.cu:54-80): query_start asc, len desc, ref_start asc, score desc.
inline bool hsp_comp(const or_segment& x, const or_segment& y) {
    if (x.query_start != y.query_start) return x.query_start < y.query_start;
    if (x.len != y.len) return x.len > y.len;
    if (x.ref_start != y.ref_start) return x.ref_start < y.ref_start;
    return x.score > y.score;
}
// hspEqual (src/seed_filter.cu:47-52).
inline bool hsp_equal(const or_segment& x, const or_segment& y) {
    return x.ref_start == y.ref_start && x.query_start == y.query_start && x.len == y.len &&
           x.score == y.score;
}
// hspDiagComp (repeat_masker_src/seed_filter.cu:52-78); the diagonal is uint32 arithmetic.
inline bool hsp_diag_comp(const or_segment& x, const or_segment& y) {
    uint32_t dx = x.ref_start - x.query_start, dy = y.ref_start - y.query_start;
    if (dx != dy) return dx < dy;
    if (x.ref_start != y.ref_start) return x.ref_start < y.ref_start;
    if (x.query_start != y.query_start) return x.query_start < y.query_start;
    return x.score > y.score;
}
// hspDiagEqual (repeat_masker_src/seed_filter.cu:45-50): same diagonal and one
// ref span [start, start+len] contains the other.  Not transitive.
inline bool hsp_diag_equal(const or_segment& x, const or_segment& y) {
    uint32_t dx = x.ref_start - x.query_start, dy = y.ref_start - y.query_start;
    if (dx != dy) return false;
    bool xin = x.ref_start >= y.ref_start && (uint32_t)(x.ref_start + x.len) <= (uint32_t)(y.ref_start + y.len);
    bool yin = y.ref_start >= x.ref_start && (uint32_t)(y.ref_start + y.len) <= (uint32_t)(x.ref_start + x.len);
    return xin || yin;
}
// hspFinalComp (repeat_masker_src/seed_filter.cu:87-107): query_start asc, score desc, ref_start desc.
inline bool hsp_final_comp(const or_segment& x, const or_segment& y) {
    if (x.query_start != y.query_start) return x.query_start < y.query_start;
    if (x.score != y.score) return x.score > y.score;
    return x.ref_start > y.ref_start;
}

// thrust::unique_copy on the CUDA backend keeps element i iff i == 0 or
// !pred(x[i-1], x[i]) with x[i-1] the *input* predecessor (CUB
// BlockDiscontinuity::FlagHeads with the tile predecessor).
template <class Pred>
void unique_pred_adjacent(std::vector<or_segment>& v, Pred pred) {
    if (v.empty()) return;
    std::vector<or_segment> out;
    out.reserve(v.size());
    out.push_back(v[0]);
    for (size_t i = 1; i < v.size(); ++i)
        if (!pred(v[i - 1], v[i])) out.push_back(v[i]);
    v.swap(out);
}

struct Scan {
    int best;       // R* / L*
    int pos;        // Rpos (or -1) / Lpos (or 0)
    uint32_t tiles; // 32-base tiles the reference kernel scans
    bool oob_in_tiles;
};

// Right pass (src/seed_filter.cu:298-425), restated per position (A.9):
// s(o) = sub[R[rl+o]][Q[ql+o]] while both are in bounds; S = running sum;
// M = max(0, running max of S); stop at the first o with M - S > xdrop or at
// the first out-of-bounds offset; best = M over o < stop; pos = first o with
// S(o) == best > 0, else -1.
inline Scan scan_right(const int32_t* sub, const uint8_t* R, uint32_t rlen, const uint8_t* Q,
                       uint32_t qlen, uint32_t rl, uint32_t ql, int xdrop, uint64_t* steps) {
    int S = 0, best = 0, bpos = -1;
    uint64_t avail_r = rl < rlen ? (uint64_t)(rlen - rl) : 0;
    uint64_t avail_q = ql < qlen ? (uint64_t)(qlen - ql) : 0;
    uint64_t avail = std::min(avail_r, avail_q);
    uint64_t o = 0;
    for (; o < avail; ++o) {
        S += sub[R[rl + o] * 8 + Q[ql + o]];
        if (S > best) { best = S; bpos = (int)o; }
        if (best - S > xdrop) break;
    }
    *steps += (o < avail) ? o + 1 : o;
    Scan r;
    r.best = best;
    r.pos = bpos;
    // Tile containing the stop offset (xdrop position or first OOB offset);
    // the reference's lane-31 edge test gives exactly o_stop >> 5.
    r.tiles = (uint32_t)(o >> 5) + 1;
    r.oob_in_tiles = ((uint64_t)r.tiles * 32 > avail);
    return r;
}

// Left pass (src/seed_filter.cu:450-576), A.10: offsets o = 1, 2, ...,
// in bounds while o <= rl and o <= ql; pos = first o with S(o) == best > 0, else 0.
inline Scan scan_left(const int32_t* sub, const uint8_t* R, const uint8_t* Q, uint32_t rl,
                      uint32_t ql, int xdrop, uint64_t* steps) {
    int S = 0, best = 0, bpos = 0;
    uint64_t avail = std::min(rl, ql);
    uint64_t o = 1;
    for (; o <= avail; ++o) {
        S += sub[R[rl - o] * 8 + Q[ql - o]];
        if (S > best) { best = S; bpos = (int)o; }
        if (best - S > xdrop) break;
    }
    *steps += (o <= avail) ? o : avail;
    Scan r;
    r.best = best;
    r.pos = bpos;
    r.tiles = (uint32_t)((o - 1) >> 5) + 1;  // tile of offsets [32t+1, 32t+32]
    r.oob_in_tiles = ((uint64_t)r.tiles * 32 > avail);
    return r;
}

// Keep/score of one hit (src/seed_filter.cu:580-621), A.11-A.13.
void extend_hit(const or_params* p, const uint8_t* R, uint32_t rlen, const uint8_t* Q,
                uint32_t qlen, uint32_t rl, uint32_t ql, or_hit_result* out, uint64_t* steps) {
    Scan rs = scan_right(p->sub_mat, R, rlen, Q, qlen, rl, ql, p->xdrop, steps);
    Scan ls = scan_left(p->sub_mat, R, Q, rl, ql, p->xdrop, steps);
    int total = rs.best + ls.best;
    int ext = rs.pos + ls.pos;  // extent = Rpos + Lpos
    double entropy = 1.0;       // entropy[warp_id] = 1.0f (:279)
    int branch = 0, unpinned = 0;
    if (total >= p->hspthresh && total <= 3 * p->hspthresh && !p->noentropy) {
        branch = 1;
        // Matches per base over right offsets 0..Rpos and left offsets 1..Lpos
        // (count/count_del, :286-293, 408-423, 559-574), stored in short.
        int cnt[4] = {0, 0, 0, 0};
        int64_t lo = (int64_t)rl - ls.pos, hi = (int64_t)rl + rs.pos;  // ref span, inclusive
        int64_t qlo = (int64_t)ql - ls.pos;
        for (int64_t r = lo; r <= hi; ++r) {
            uint8_t a = R[r], b = Q[qlo + (r - lo)];
            if (a == b && a < 4) cnt[a]++;
        }
        int16_t c[4];
        for (int b = 0; b < 4; ++b) c[b] = (int16_t)cnt[b];
        // Reference UB (A.12): equal pairs with code >= 4 in scanned tiles, or
        // stale per-lane characters in out-of-bounds lanes, index count_del
        // out of bounds.  The oracle ignores them and reports the HSP as unpinned.
        {
            bool ub = rs.oob_in_tiles || ls.oob_in_tiles;
            uint64_t rend = std::min<uint64_t>((uint64_t)rs.tiles * 32, std::min<uint64_t>(rlen - std::min(rl, rlen), qlen - std::min(ql, qlen)));
            for (uint64_t o = 0; !ub && o < rend; ++o) {
                uint8_t a = R[rl + o], b = Q[ql + o];
                if (a == b && a >= 4) ub = true;
            }
            uint64_t lend = std::min<uint64_t>((uint64_t)ls.tiles * 32, std::min(rl, ql));
            for (uint64_t o = 1; !ub && o <= lend; ++o) {
                uint8_t a = R[rl - o], b = Q[ql - o];
                if (a == b && a >= 4) ub = true;
            }
            unpinned = ub ? 1 : 0;
        }
        if ((int)c[0] + (int)c[1] + (int)c[2] + (int)c[3] >= 20) {
            // :591-595.  nvcc contracts `e += a * b` into an FMA (default
            // --fmad=true); log(4.0f) resolves to the float overload.
            double n = (double)(ext + 1);
            double e = 0.0;
            for (int b = 0; b < 4; ++b) {
                double q = (double)c[b] / n;
                double lg = (c[b] != 0) ? std::log((double)c[b] / n) : 0.0;
                e = std::fma(q, lg, e);
            }
            entropy = -e / (double)logf(4.0f);
        }
    }
    int keep = (int)(((double)(float)total) * entropy) >= p->hspthresh;  // :605
    int score = 0;
    if (entropy > 0) score = (int)((double)total * entropy);  // :609-610
    out->right_best = rs.best;
    out->right_pos = rs.pos;
    out->left_best = ls.best;
    out->left_pos = ls.pos;
    out->total = total;
    out->keep = keep;
    out->score = score;
    out->entropy_branch = branch;
    out->entropy = entropy;
    out->tiles_right = rs.tiles;
    out->tiles_left = ls.tiles;
    out->unpinned = unpinned;
}

}  // namespace

extern "C" {

void or_encode(const char* text, uint64_t len, uint8_t* codes) {
    for (uint64_t i = 0; i < len; ++i) codes[i] = code_of(text[i]);
}

// Device rc of the query text (src/seed_filter.cu:82-127): rc[len-1-i] = comp(code(text[i])).
void or_encode_rc(const char* text, uint64_t len, uint8_t* rc) {
    for (uint64_t i = 0; i < len; ++i) rc[len - 1 - i] = comp_code(code_of(text[i]));
}

// rm mode rc of an encoded block (repeat_masker_src/seed_filter.cu:137-167).
void or_rc_codes(const uint8_t* codes, uint64_t len, uint8_t* rc) {
    for (uint64_t i = 0; i < len; ++i) rc[len - 1 - i] = comp_code(codes[i]);
}

// common/ntcoding.cpp:63-105: reverse complement of host text; characters
// outside ACGTacgtnN& are skipped (the reference prints "Bad Nt char").
uint64_t or_revcomp_text(char* dst, const char* src, uint64_t len) {
    uint64_t r = 0;
    for (uint64_t i = len; i > 0; --i) {
        char c = src[i - 1], o;
        switch (c) {
            case 'a': o = 't'; break;
            case 'A': o = 'T'; break;
            case 'c': o = 'g'; break;
            case 'C': o = 'G'; break;
            case 'g': o = 'c'; break;
            case 'G': o = 'C'; break;
            case 't': o = 'a'; break;
            case 'T': o = 'A'; break;
            case 'n': o = 'n'; break;
            case 'N': o = 'N'; break;
            case '&': o = '&'; break;
            default: continue;
        }
        dst[r++] = o;
    }
    return r;
}

// src/main.cpp:180-261 (no --scoring file).  ambiguous: "" / "n" / "iupac" /
// "x,reward,penalty" style (fields.size()==3).  Returns 0, or -1 when the
// ambiguous string cannot be parsed.
int or_build_sub_mat(int xdrop, const char* ambiguous, int32_t* m) {
    int ambiguous_reward = -100, ambiguous_penalty = -100;
    const int fill_score = -100, bad_score = -1000;
    std::string amb = ambiguous ? ambiguous : "";
    std::vector<std::string> fields;
    {
        size_t s = 0;
        while (true) {
            size_t k = amb.find(',', s);
            fields.push_back(amb.substr(s, k == std::string::npos ? std::string::npos : k - s));
            if (k == std::string::npos) break;
            s = k + 1;
        }
    }
    std::string field = fields[0];
    if (fields.size() == 3) {
        try {
            ambiguous_reward = std::stoi(fields[1]);
            ambiguous_penalty = -1 * std::stoi(fields[2]);
        } catch (...) {
            return -1;
        }
    } else if (amb == "n" || amb == "iupac") {
        ambiguous_reward = 0;
        ambiguous_penalty = 0;
    }
    static const int hoxd70[4][4] = {{91, -114, -31, -123},
                                     {-114, 100, -125, -31},
                                     {-31, -125, 100, -114},
                                     {-123, -31, -114, 91}};
    for (int i = 0; i < 64; ++i) m[i] = 0;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) m[i * 8 + j] = hoxd70[i][j];
    for (int i = 0; i < L_NT; ++i) {
        m[i * 8 + L_NT] = bad_score;
        m[L_NT * 8 + i] = bad_score;
    }
    m[L_NT * 8 + L_NT] = bad_score;
    if (field == "n" || field == "iupac") {
        for (int i = 0; i < N_NT; ++i) {
            m[i * 8 + N_NT] = ambiguous_penalty;
            m[N_NT * 8 + i] = ambiguous_penalty;
        }
        m[N_NT * 8 + N_NT] = ambiguous_reward;
    } else {
        for (int i = 0; i < N_NT; ++i) {
            m[i * 8 + N_NT] = bad_score;
            m[N_NT * 8 + i] = bad_score;
        }
        m[N_NT * 8 + N_NT] = bad_score;
    }
    if (field == "iupac") {
        for (int i = 0; i < X_NT; ++i) {
            m[i * 8 + X_NT] = ambiguous_penalty;
            m[X_NT * 8 + i] = ambiguous_penalty;
        }
        m[X_NT * 8 + X_NT] = ambiguous_reward;
    } else {
        for (int i = 0; i < L_NT; ++i) {
            m[i * 8 + X_NT] = fill_score;
            m[X_NT * 8 + i] = fill_score;
        }
        for (int i = L_NT; i < X_NT; ++i) {
            m[i * 8 + X_NT] = bad_score;
            m[X_NT * 8 + i] = bad_score;
        }
        m[X_NT * 8 + X_NT] = fill_score;
    }
    for (int i = 0; i < E_NT; ++i) {
        m[i * 8 + E_NT] = -10 * xdrop;
        m[E_NT * 8 + i] = -10 * xdrop;
    }
    m[E_NT * 8 + E_NT] = -10 * xdrop;
    return 0;
}

// src/main.cpp:152-173 + common/ntcoding.cpp:21-37.  Accepts "12of19",
// "14of22" or an explicit pattern of 1/0/T characters.  Returns kmer_size or -1.
int or_parse_shape(const char* seed_name, or_params* p) {
    std::string name = seed_name ? seed_name : "12of19";
    std::string shape;
    if (name == "12of19") shape = "TTT0T00TT00T0T0TTTT";
    else if (name == "14of22") shape = "TTT0T0TT00TT00T0T0TTTT";
    else {
        shape = name;
        for (auto& c : shape) c = (c == '1') ? 'T' : '0';
    }
    int k = 0;
    for (size_t i = 0; i < shape.size(); ++i) {
        if (shape[i] == '1' || shape[i] == 'T') {
            if (k >= 32) return -1;
            p->shape_pos[k++] = (int)i;
        }
    }
    if (k > 15 || k <= 3) return -1;  // common/seed_pos_table.cu:51-52
    p->seed_size = (int)shape.size();
    p->kmer_size = k;
    return k;
}

// common/ntcoding.cpp:43-61: INVALID_KMER unless all seed_size characters are
// uppercase ACGT; key folds the shape positions in order, first = most significant.
uint32_t or_kmer_index(const char* text, uint64_t pos, const or_params* p) {
    uint32_t nt[64];
    for (int i = 0; i < p->seed_size; ++i)
        if (!nt_valid(text[pos + i], &nt[i])) return INVALID_KMER;
    uint32_t k = 0;
    for (int i = 0; i < p->kmer_size; ++i) k = (k << 2) + nt[p->shape_pos[i]];
    return k;
}

// common/seed_pos_table.cu:49-109 positions: p = start + i*step, i < num_steps.
static void table_geometry(uint32_t len, uint32_t step, const or_params* p, uint32_t* start,
                           uint64_t* num_steps) {
    uint32_t offset = (uint32_t)(p->seed_size + 1) % step;
    *start = step - offset;
    int64_t span = (int64_t)len - p->seed_size + offset;
    *num_steps = span > 0 ? (uint64_t)(span / step) : 0;
}

// Keys of all table positions, computed with std::threads (the reference
// uses a TBB parallel_for, common/seed_pos_table.cu:69-81).
static void table_keys(const char* text, uint32_t len, uint32_t step, const or_params* p,
                       std::vector<uint32_t>& keys, uint32_t* start_out) {
    uint32_t start;
    uint64_t n;
    table_geometry(len, step, p, &start, &n);
    *start_out = start;
    keys.resize(n);
    unsigned nt = std::max(1u, std::thread::hardware_concurrency());
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t)
        th.emplace_back([&, t]() {
            uint64_t a = n * t / nt, b = n * (t + 1) / nt;
            for (uint64_t i = a; i < b; ++i) keys[i] = or_kmer_index(text, start + i * step, p);
        });
    for (auto& x : th) x.join();
}

uint64_t or_table_count(const char* text, uint32_t len, uint32_t step, const or_params* p) {
    std::vector<uint32_t> keys;
    uint32_t start;
    table_keys(text, len, step, p, keys, &start);
    uint64_t c = 0;
    for (uint32_t k : keys) c += k != INVALID_KMER;
    return c;
}

// index_table[k] = number of valid positions with key <= k (the shipped,
// shifted table, :83, :103); pos_table grouped by key.  The reference's order
// inside a bucket is an atomic-fetch-add order; the oracle uses ascending
// positions (results do not depend on bucket order).
int or_build_table(const char* text, uint32_t len, uint32_t step, const or_params* p,
                   uint32_t* index_table, uint32_t* pos_table, uint64_t pos_cap,
                   uint64_t* num_index) {
    uint32_t start;
    std::vector<uint32_t> keys;
    table_keys(text, len, step, p, keys, &start);
    const uint64_t n = keys.size();
    const uint64_t nb = 1ull << (2 * p->kmer_size);
    std::vector<uint64_t> cnt(nb + 1, 0);
    for (uint64_t i = 0; i < n; ++i)
        if (keys[i] != INVALID_KMER) cnt[keys[i] + 1]++;
    for (uint64_t k = 1; k <= nb; ++k) cnt[k] += cnt[k - 1];
    uint64_t total = cnt[nb];
    *num_index = total;
    if (total > pos_cap) return -1;
    for (uint64_t k = 0; k < nb; ++k) index_table[k] = (uint32_t)cnt[k + 1];
    std::vector<uint64_t> fill(cnt.begin(), cnt.end() - 1);
    for (uint64_t i = 0; i < n; ++i)
        if (keys[i] != INVALID_KMER) pos_table[fill[keys[i]]++] = (uint32_t)(start + i * step);
    return 0;
}

// src/seeder.cpp:57-74: positions j0..j1-1 in order; word (key<<32)+j, then
// the transition variants key ^ (2 << 2t) for t = 0..K-1.
uint64_t or_chunk_seeds(const char* text, uint32_t j0, uint32_t j1, const or_params* p,
                        uint64_t* out, uint64_t cap) {
    uint64_t n = 0;
    for (uint32_t j = j0; j < j1; ++j) {
        uint32_t k = or_kmer_index(text, j, p);
        if (k == INVALID_KMER) continue;
        if (n < cap) out[n] = ((uint64_t)k << 32) + j;
        ++n;
        if (p->transition) {
            for (int t = 0; t < p->kmer_size; ++t) {
                uint64_t tk = (uint64_t)(k ^ (2u << (2 * t)));
                if (n < cap) out[n] = (tk << 32) + j;
                ++n;
            }
        }
    }
    return n;
}

void or_extend_hit(const or_params* p, const uint8_t* R, uint32_t rlen, const uint8_t* Q,
                   uint32_t qlen, uint32_t rl, uint32_t ql, or_hit_result* r) {
    uint64_t steps = 0;
    extend_hit(p, R, rlen, Q, qlen, rl, ql, r, &steps);
}

// src/seed_filter.cu:654-778 (plain) and repeat_masker_src/seed_filter.cu:723-855 (rm).
int or_seed_and_filter(const or_params* p, const uint8_t* R, uint32_t rlen, const uint8_t* Q,
                       uint32_t qlen, const uint32_t* index_table, const uint32_t* pos_table,
                       const uint64_t* seeds, uint64_t n, int rev, int mode,
                       uint32_t rm_ref_start, uint32_t rm_ref_end, or_segment** out,
                       uint64_t* out_len, or_stats* st) {
    or_stats s;
    std::memset(&s, 0, sizeof(s));
    s.num_seeds = n;
    const uint32_t seed_size = (uint32_t)p->seed_size;
    // find_num_hits + inclusive_scan (:129-154, :680-684).
    std::vector<uint64_t> P(n);
    std::vector<uint32_t> lo(n);
    uint64_t acc = 0;
    for (uint64_t i = 0; i < n; ++i) {
        uint32_t key = (uint32_t)(seeds[i] >> 32);
        uint32_t end = index_table[key];
        uint32_t beg = key > 0 ? index_table[key - 1] : 0;
        lo[i] = beg;
        acc += (uint64_t)(end - beg);
        P[i] = acc;
    }
    uint64_t num_hits = acc;
    s.num_hits = num_hits;
    // MAX_HITS split (:686-697), A.16.
    const uint64_t MH = p->max_hits;
    if (MH == 0) return -2;
    uint64_t num_iter = num_hits / MH + 1;
    std::vector<int64_t> limit(num_iter);
    {
        uint64_t lim = MH;
        int64_t prev = -1;
        for (uint64_t i = 0; i + 1 < num_iter; ++i) {
            int64_t pos = (int64_t)(std::lower_bound(P.begin(), P.end(), lim) - P.begin()) - 1;
            if (pos <= prev) return -3;  // a single seed holds >= MAX_HITS hits: reference UB
            lim = P[pos] + MH;
            limit[i] = pos;
            prev = pos;
        }
        limit[num_iter - 1] = (int64_t)n - 1;
    }
    s.num_iter = (int32_t)num_iter;
    std::vector<or_segment> result;
    result.push_back(or_segment{0, 0, 0, 0});
    uint64_t total_anchors = 0;
    if (num_hits > 0) {
        int64_t start_seed = 0;
        for (uint64_t it = 0; it < num_iter; ++it) {
            std::vector<or_segment> surv;
            for (int64_t sd = start_seed; sd <= limit[it]; ++sd) {
                uint32_t key = (uint32_t)(seeds[sd] >> 32);
                uint32_t end = index_table[key];
                uint32_t query_loc = (uint32_t)(seeds[sd] & 0xffffffffu) + seed_size;  // find_hits :176
                for (uint32_t t = lo[sd]; t < end; ++t) {
                    uint32_t ref_loc = pos_table[t] + seed_size;  // :192
                    if (mode == 1 && !(ref_loc >= rm_ref_start && ref_loc <= rm_ref_end))
                        continue;  // rm find_hits :237-243, find_hsps :304-333
                    s.hits_extended++;
                    or_hit_result h;
                    extend_hit(p, R, rlen, Q, qlen, ref_loc, query_loc, &h, &s.base_steps);
                    s.tiles_right += h.tiles_right;
                    s.tiles_left += h.tiles_left;
                    if (h.keep) {
                        if (h.unpinned) s.unpinned++;
                        or_segment g;
                        g.ref_start = ref_loc - (uint32_t)h.left_pos;  // :606-608
                        g.query_start = query_loc - (uint32_t)h.left_pos;
                        g.len = (uint32_t)(h.right_pos + h.left_pos);
                        g.score = h.score;
                        if (mode == 1 && rev)  // rm compress_output :704-707
                            g.query_start = rlen - 1 - (g.query_start + g.len);
                        surv.push_back(g);
                    }
                }
            }
            s.survivors += surv.size();
            // stable_sort(hspComp) + unique_copy(hspEqual) (:728-732).
            std::stable_sort(surv.begin(), surv.end(), hsp_comp);
            unique_pred_adjacent(surv, hsp_equal);
            if (mode == 1) {
                // rm :803-809.
                std::stable_sort(surv.begin(), surv.end(), hsp_diag_comp);
                unique_pred_adjacent(surv, hsp_diag_equal);
                if (p->rm_exclude_diag && !rev) {
                    std::vector<or_segment> keep;
                    keep.reserve(surv.size());
                    for (auto& g : surv)
                        if (g.ref_start != g.query_start) keep.push_back(g);
                    surv.swap(keep);
                }
                std::stable_sort(surv.begin(), surv.end(), hsp_final_comp);
            }
            total_anchors += surv.size();
            result.insert(result.end(), surv.begin(), surv.end());
            start_seed = limit[it] + 1;
        }
    }
    // Header (:756-759): len = total anchors, score = num_hits (uint32 -> int).
    result[0].len = (uint32_t)total_anchors;
    result[0].score = (int32_t)(uint32_t)num_hits;
    s.num_hsps = total_anchors;
    or_segment* o = (or_segment*)std::malloc(sizeof(or_segment) * result.size());
    if (!o) return -4;
    std::memcpy(o, result.data(), sizeof(or_segment) * result.size());
    *out = o;
    *out_len = result.size();
    if (st) *st = s;
    return 0;
}

void or_free(void* ptr) { std::free(ptr); }

// src/seeder.cpp:47-121 over every interval of one query block
// (src/main.cpp:373-386 intervals, :707 q_len = Lq - seed_size).
int or_pipeline(const or_params* p, const or_pipeline_cfg* cfg, const char* ref_text,
                uint32_t ref_len, const char* query_text, uint32_t query_len,
                const uint32_t* index_table, const uint32_t* pos_table, or_segment** fw,
                uint64_t* fw_len, or_segment** rc, uint64_t* rc_len, or_stats* stats) {
    std::vector<uint8_t> R(ref_len), Q(query_len), QR(query_len);
    or_encode(ref_text, ref_len, R.data());
    or_encode(query_text, query_len, Q.data());
    or_encode_rc(query_text, query_len, QR.data());
    std::vector<char> rctext(query_len);
    uint64_t wrote = or_revcomp_text(rctext.data(), query_text, query_len);
    if (wrote != query_len) return -5;  // characters outside ACGTacgtnN&: reference rc buffer shifts
    struct Call {
        int strand;
        uint32_t j0, j1;
        uint64_t order;
    };
    std::vector<Call> calls;
    if (query_len < (uint32_t)p->seed_size) return -6;
    const uint32_t qlen_s = query_len - (uint32_t)p->seed_size;  // curr_block.q_len
    std::vector<std::pair<uint32_t, uint32_t>> intervals;
    for (uint32_t cur = 0; cur < qlen_s; cur += cfg->interval_size) {
        uint64_t e = std::min<uint64_t>(qlen_s, (uint64_t)cur + cfg->interval_size + cfg->interval_overlap);
        intervals.push_back({cur, (uint32_t)e});
        if ((uint64_t)cur + cfg->interval_size >= qlen_s) break;
    }
    uint64_t ord = 0;
    for (auto& iv : intervals) {
        if (cfg->strand & 1)
            for (uint32_t i = iv.first; i < iv.second; i += cfg->chunk_size)
                calls.push_back({0, i, std::min(i + cfg->chunk_size, iv.second), ord++});
        if (cfg->strand & 2) {
            uint32_t rs = qlen_s - iv.second, re = qlen_s - iv.first;
            for (uint32_t i = rs; i < re; i += cfg->chunk_size)
                calls.push_back({1, i, std::min(i + cfg->chunk_size, re), ord++});
        }
    }
    if (cfg->max_chunks && calls.size() > cfg->max_chunks) calls.resize(cfg->max_chunks);
    std::vector<std::vector<or_segment>> results(calls.size());
    std::vector<or_stats> cstats(calls.size());
    std::atomic<uint64_t> next{0};
    std::atomic<int> err{0};
    auto worker = [&]() {
        std::vector<uint64_t> seeds;
        while (true) {
            uint64_t c = next.fetch_add(1);
            if (c >= calls.size()) break;
            const Call& cl = calls[c];
            const char* txt = cl.strand ? rctext.data() : query_text;
            uint64_t need = or_chunk_seeds(txt, cl.j0, cl.j1, p, nullptr, 0);
            seeds.resize(need);
            or_chunk_seeds(txt, cl.j0, cl.j1, p, seeds.data(), need);
            std::memset(&cstats[c], 0, sizeof(or_stats));
            if (need == 0) continue;  // seeder.cpp:190 skips empty seed vectors
            or_segment* o = nullptr;
            uint64_t ol = 0;
            int rcode = or_seed_and_filter(p, R.data(), ref_len, cl.strand ? QR.data() : Q.data(),
                                           query_len, index_table, pos_table, seeds.data(), need,
                                           cl.strand, 0, 0, 0, &o, &ol, &cstats[c]);
            if (rcode) {
                err = rcode;
                continue;
            }
            results[c].assign(o + 1, o + ol);
            std::free(o);
        }
    };
    int nt = cfg->nthreads > 0 ? cfg->nthreads : 1;
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t) th.emplace_back(worker);
    for (auto& t : th) t.join();
    if (err) return err;
    std::vector<or_segment> F, Rv;
    or_stats tot;
    std::memset(&tot, 0, sizeof(tot));
    for (size_t c = 0; c < calls.size(); ++c) {
        auto& dst = calls[c].strand ? Rv : F;
        dst.insert(dst.end(), results[c].begin(), results[c].end());
        tot.num_seeds += cstats[c].num_seeds;
        tot.num_hits += cstats[c].num_hits;
        tot.hits_extended += cstats[c].hits_extended;
        tot.tiles_right += cstats[c].tiles_right;
        tot.tiles_left += cstats[c].tiles_left;
        tot.survivors += cstats[c].survivors;
        tot.num_hsps += cstats[c].num_hsps;
        tot.unpinned += cstats[c].unpinned;
        tot.base_steps += cstats[c].base_steps;
    }
    auto dup = [](const std::vector<or_segment>& v, or_segment** o, uint64_t* l) {
        *l = v.size();
        *o = (or_segment*)std::malloc(sizeof(or_segment) * (v.size() ? v.size() : 1));
        if (!v.empty()) std::memcpy(*o, v.data(), sizeof(or_segment) * v.size());
    };
    dup(F, fw, fw_len);
    dup(Rv, rc, rc_len);
    if (stats) *stats = tot;
    return 0;
}

// repeat_masker_src/main.cpp:319-428.  Interval counts use float ceil as the
// reference does; all window arithmetic is uint32.
uint64_t or_rm_plan(uint64_t seq_len, uint32_t interval_size, uint32_t block_size, float prop_neigh,
                    uint32_t seed_size, uint32_t* out, uint64_t cap) {
    const uint32_t total = (uint32_t)std::ceil((float)seq_len / interval_size);
    const uint32_t neigh = (uint32_t)std::ceil((float)prop_neigh * total);
    const uint32_t left_iv = (uint32_t)std::ceil((float)(neigh - 1) / 2);
    const uint32_t right_iv = neigh - 1 - left_iv;
    const uint32_t left_overlap = left_iv * interval_size;
    const uint32_t right_overlap = right_iv * interval_size;
    const uint32_t max_len = left_overlap + interval_size + right_overlap;
    uint64_t k = 0;
    uint32_t block = 0;
    for (uint64_t l = 0; l < seq_len; l += block_size, ++block) {
        uint64_t bstart = (l < left_overlap) ? l : l - left_overlap;
        uint32_t blen;
        if (l + block_size + right_overlap > seq_len) blen = (uint32_t)(seq_len - bstart);
        else blen = (uint32_t)(l - bstart + block_size) + right_overlap;
        uint32_t start_pos = (uint32_t)(l - bstart), end_pos;
        if (blen < block_size) end_pos = start_pos + blen - (uint32_t)(l - bstart) - seed_size;
        else end_pos = start_pos + block_size - seed_size;
        while (start_pos < end_pos) {
            const uint32_t is = start_pos, ie = std::min(end_pos, is + interval_size);
            uint32_t rs, re;
            const bool ll = is < left_overlap, rl = (ie + right_overlap) > blen;
            if (ll) {
                rs = 0;
                re = rl ? blen : (max_len > blen ? blen : max_len);
            } else if (rl) {
                re = blen;
                rs = blen < max_len ? 0 : blen - max_len;
            } else {
                rs = is - left_overlap;
                re = ie + right_overlap;
            }
            if (k < cap) {
                uint32_t* row = out + 7 * k;
                row[0] = block;
                row[1] = (uint32_t)bstart;
                row[2] = blen;
                row[3] = is;
                row[4] = ie;
                row[5] = rs;
                row[6] = re;
            }
            ++k;
            start_pos += interval_size;
        }
    }
    return k;
}

// repeat_masker_src/seeder.cpp:151-186: uint8 coverage over [qs, qs+len) of
// every HSP, then runs with count >= M; a run still open at the block end is
// not emitted (the loop only closes runs in its else branch).
uint64_t or_rm_intervals(const or_segment* h, uint64_t n, uint32_t block_len, uint32_t M,
                         uint32_t* starts, uint32_t* lens, uint64_t cap, uint8_t* cnt) {
    std::memset(cnt, 0, block_len);
    for (uint64_t i = 0; i < n; ++i)
        for (uint64_t j = h[i].query_start; j < (uint64_t)h[i].query_start + h[i].len && j < block_len; ++j)
            cnt[j]++;
    uint64_t k = 0;
    int run = 0;
    uint32_t qs = 0, len = 0;
    for (uint32_t i = 0; i < block_len; ++i) {
        if (cnt[i] >= M) {
            if (!run) { run = 1; qs = i; }
            len++;
        } else {
            if (run) {
                run = 0;
                if (k < cap) { starts[k] = qs; lens[k] = len; }
                ++k;
            }
            qs = 0;
            len = 0;
        }
    }
    return k;
}

}  // extern "C"
