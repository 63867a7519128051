// sa_host.cpp — host side of the seed-filter path, in C++ as in the
// reference: query seeding (src/seeder.cpp), the scoring table
// (src/main.cpp:180-261), host reverse complement (common/ntcoding.cpp:63-105)
// and the seeder pipeline that cuts a query block into intervals and chunks
// and calls sa_seed_and_filter() from several host threads, in the way the
// reference's TBB flow graph does (src/main.cpp:546-566, src/seeder.cpp:12-127).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/segalign_b200.h"
#include "../../include/segalign_b200_host.h"
#include "sa_host_internal.h"

namespace {

struct HostShape {
    int seed_size = 19;
    int kmer_size = 12;
    int pos[32] = {0, 1, 2, 4, 7, 8, 11, 13, 15, 16, 17, 18};
    int transition = 0;
    // Key extraction from a rolling window of 2-bit codes (newest base in the
    // low bits): key = OR over b of part[b][byte b of the window].
    uint32_t part[8][256];
    int nbytes = 5;
};
HostShape g_shape;

// Code of each character: 0..3 for A, C, G, T; 4 for every other character
// (lowercase, N, '&', IUPAC: invalid in a seed, common/ntcoding.cpp:10-19).
struct CodeTable {
    uint8_t c[256];
    CodeTable() {
        std::memset(c, 4, sizeof c);
        c[(uint8_t)'A'] = 0;
        c[(uint8_t)'C'] = 1;
        c[(uint8_t)'G'] = 2;
        c[(uint8_t)'T'] = 3;
    }
};
const CodeTable g_codes;

// Key of the window whose first base is at window offset 0: shape position
// p_i (i = 0..K-1, the first one most significant, common/ntcoding.cpp:43-61)
// lies 2 * (S - 1 - p_i) bits up the window; byte b of the window contributes
// the key bits of the shape positions it holds.
void build_parts(HostShape& h) {
    const int S = h.seed_size, K = h.kmer_size;
    h.nbytes = (2 * S + 7) / 8;
    for (int b = 0; b < 8; ++b)
        for (int v = 0; v < 256; ++v) {
            uint32_t key = 0;
            for (int i = 0; i < K; ++i) {
                const int bit = 2 * (S - 1 - h.pos[i]);  // position of the base's code in the window
                if (bit / 8 != b) continue;
                const uint32_t code = (uint32_t)(v >> (bit % 8)) & 3u;
                key |= code << (2 * (K - 1 - i));
            }
            h.part[b][v] = key;
        }
}

struct PartsInit {
    PartsInit() { build_parts(g_shape); }
} g_parts_init;

// Seed words of positions [j0, j1): the first `cap` go to out (out may be
// NULL with cap 0); returns the count.  One pass: rolling window of 2-bit
// codes and the position of the last invalid base.
uint64_t chunk_seeds(const HostShape& h, const char* text, uint32_t j0, uint32_t j1, uint64_t* out, uint64_t cap) {
    const int S = h.seed_size, K = h.kmer_size;
    const uint64_t wmask = (S >= 32) ? ~0ull : ((1ull << (2 * S)) - 1);
    uint64_t w = 0, n = 0;
    int64_t last_bad = (int64_t)j0 - 1;
    // prime the window with bases j0 .. j0+S-2
    for (int i = 0; i + 1 < S; ++i) {
        const uint32_t c = g_codes.c[(uint8_t)text[j0 + i]];
        if (c > 3) last_bad = (int64_t)j0 + i;
        w = ((w << 2) | (c & 3u)) & wmask;
    }
    for (uint32_t j = j0; j < j1; ++j) {
        const uint64_t p = (uint64_t)j + (uint64_t)(S - 1);  // newest base of window j
        const uint32_t c = g_codes.c[(uint8_t)text[p]];
        if (c > 3) last_bad = (int64_t)p;
        w = ((w << 2) | (c & 3u)) & wmask;
        if (last_bad >= (int64_t)j) continue;  // window has a non-ACGT base
        uint32_t key = 0;
        for (int b = 0; b < h.nbytes; ++b) key |= h.part[b][(w >> (8 * b)) & 0xff];
        if (n < cap) out[n] = ((uint64_t)key << 32) + j;
        ++n;
        if (h.transition)
            for (int t = 0; t < K; ++t) {
                if (n < cap) out[n] = ((uint64_t)(key ^ (2u << (2 * t))) << 32) + j;
                ++n;
            }
    }
    return n;
}

}  // namespace

extern "C" {

int sa_host_set_shape(const char* shape, int transition) {
    std::string name = shape ? shape : "12of19", pat;
    if (name == "12of19") pat = "TTT0T00TT00T0T0TTTT";
    else if (name == "14of22") pat = "TTT0T0TT00TT00T0T0TTTT";
    else {
        pat = name;
        for (auto& c : pat) c = (c == '1' || c == 'T') ? 'T' : '0';
    }
    HostShape h;
    int k = 0;
    for (size_t i = 0; i < pat.size() && k < 32; ++i)
        if (pat[i] == 'T') h.pos[k++] = (int)i;
    if (k > 15 || k <= 3 || pat.size() > 32) return SA_ERR_ARG;
    h.kmer_size = k;
    h.seed_size = (int)pat.size();
    h.transition = transition ? 1 : 0;
    if (h.seed_size != g_shape.seed_size || h.kmer_size != g_shape.kmer_size || h.transition != g_shape.transition ||
        !std::equal(h.pos, h.pos + k, g_shape.pos)) {
        build_parts(h);
        g_shape = h;
    }
    return k;
}

// src/seeder.cpp:57-74: for j in [j0, j1): word (key << 32) + j, followed by
// the transition variants key ^ (2 << 2t), t = 0..K-1, when transitions are on.
// With out == NULL (or cap too small) only the count is returned.
uint64_t sa_host_chunk_seeds(const char* text, uint32_t j0, uint32_t j1, uint64_t* out, uint64_t cap) {
    if (j1 <= j0) return 0;
    return chunk_seeds(g_shape, text, j0, j1, out, out ? cap : 0);
}

// common/ntcoding.cpp:63-105; characters other than ACGTacgtnN& are skipped.
// Large inputs are split into blocks on several threads: each block's count
// of kept characters gives, by a suffix sum, where its output starts.
uint64_t sa_host_revcomp(char* dst, const char* src, uint64_t len) {
    static const struct CompTable {
        char c[256];
        CompTable() {
            std::memset(c, 0, sizeof c);
            const char* from = "aAcCgGtTnN&";
            const char* to = "tTgGcCaAnN&";
            for (int i = 0; from[i]; ++i) c[(uint8_t)from[i]] = to[i];
        }
    } comp;
    unsigned hw = std::thread::hardware_concurrency();
    const int nb = len >= (1u << 22) ? (int)std::min<unsigned>(16, hw ? hw : 1) : 1;
    std::vector<uint64_t> lo(nb + 1), cnt(nb, 0), start(nb + 1, 0);
    for (int b = 0; b <= nb; ++b) lo[b] = len * (uint64_t)b / (uint64_t)nb;
    auto count = [&](int b) {
        uint64_t k = 0;
        for (uint64_t i = lo[b]; i < lo[b + 1]; ++i) k += comp.c[(uint8_t)src[i]] != 0;
        cnt[b] = k;
    };
    auto write = [&](int b) {
        char* o = dst + start[b + 1];  // kept characters of the blocks after b come first
        for (uint64_t i = lo[b + 1]; i > lo[b]; --i) {
            const char c = comp.c[(uint8_t)src[i - 1]];
            if (c) *o++ = c;
        }
    };
    auto run = [&](auto&& f) {
        if (nb == 1) return f(0);
        std::vector<std::thread> th;
        for (int b = 0; b < nb; ++b) th.emplace_back(f, b);
        for (auto& t : th) t.join();
    };
    run(count);
    for (int b = nb - 1; b >= 0; --b) start[b] = start[b + 1] + cnt[b];  // kept in blocks b..nb-1
    run(write);
    return start[0];
}

// src/main.cpp:180-261 (no --scoring file): HOXD70 plus the lowercase, N,
// other-IUPAC and separator rows.  ambiguous: NULL/"" , "n", "iupac", or
// "<field>,<reward>,<penalty>".
int sa_build_sub_mat(int xdrop, const char* ambiguous, int* m) {
    int reward = -100, penalty = -100;
    const int fill = -100, bad = -1000;
    std::string amb = ambiguous ? ambiguous : "";
    std::vector<std::string> f;
    size_t s = 0;
    while (true) {
        size_t k = amb.find(',', s);
        f.push_back(amb.substr(s, k == std::string::npos ? std::string::npos : k - s));
        if (k == std::string::npos) break;
        s = k + 1;
    }
    const std::string field = f[0];
    if (f.size() == 3) {
        char* e1 = nullptr;
        char* e2 = nullptr;
        long r = strtol(f[1].c_str(), &e1, 10), p = strtol(f[2].c_str(), &e2, 10);
        if (f[1].empty() || f[2].empty() || *e1 || *e2) return SA_ERR_ARG;
        reward = (int)r;
        penalty = -(int)p;
    } else if (amb == "n" || amb == "iupac") {
        reward = 0;
        penalty = 0;
    }
    static const int hoxd70[4][4] = {{91, -114, -31, -123}, {-114, 100, -125, -31}, {-31, -125, 100, -114}, {-123, -31, -114, 91}};
    for (int i = 0; i < 64; ++i) m[i] = 0;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) m[i * 8 + j] = hoxd70[i][j];
    for (int i = 0; i < 4; ++i) m[i * 8 + 4] = m[4 * 8 + i] = bad;
    m[4 * 8 + 4] = bad;
    const bool nmode = field == "n" || field == "iupac";
    for (int i = 0; i < 5; ++i) m[i * 8 + 5] = m[5 * 8 + i] = nmode ? penalty : bad;
    m[5 * 8 + 5] = nmode ? reward : bad;
    if (field == "iupac") {
        for (int i = 0; i < 6; ++i) m[i * 8 + 6] = m[6 * 8 + i] = penalty;
        m[6 * 8 + 6] = reward;
    } else {
        for (int i = 0; i < 4; ++i) m[i * 8 + 6] = m[6 * 8 + i] = fill;
        for (int i = 4; i < 6; ++i) m[i * 8 + 6] = m[6 * 8 + i] = bad;
        m[6 * 8 + 6] = fill;
    }
    for (int i = 0; i < 7; ++i) m[i * 8 + 7] = m[7 * 8 + i] = -10 * xdrop;
    m[7 * 8 + 7] = -10 * xdrop;
    return SA_OK;
}

}  // extern "C"

int sa_host_seed_size() { return g_shape.seed_size; }
int sa_host_kmer_size() { return g_shape.kmer_size; }

int sa_host_run_calls(const std::vector<SaHostCall>& calls, const char* query, const char* rctext, uint32_t buffer,
                      int nthreads, std::vector<SaHostCallOut>& res, SaHostRunStats* st) {
    res.assign(calls.size(), SaHostCallOut());
    std::atomic<uint64_t> next{0}, nseeds{0}, nhits{0}, nhsps{0};
    std::atomic<uint64_t> ns_seed{0}, ns_call{0};
    std::atomic<int> err{0};
    std::mutex err_mu;
    std::string err_msg;  // the first failing worker's sa_last_error() text
    using SClock = std::chrono::steady_clock;
    auto ns_since = [](SClock::time_point t) {
        return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(SClock::now() - t).count();
    };
    auto worker = [&]() {
        std::vector<uint64_t> seeds;
        while (!err) {
            uint64_t c = next.fetch_add(1);
            if (c >= calls.size()) break;
            const SaHostCall& cl = calls[c];
            const char* txt = cl.strand ? rctext : query;
            const uint64_t per = 1 + (g_shape.transition ? (uint64_t)g_shape.kmer_size : 0);
            auto t_seed = SClock::now();
            seeds.resize((uint64_t)(cl.j1 - cl.j0) * per);
            const uint64_t need = chunk_seeds(g_shape, txt, cl.j0, cl.j1, seeds.data(), seeds.size());
            ns_seed += ns_since(t_seed);
            if (need == 0) continue;  // src/seeder.cpp:76
            sa_segment* out = nullptr;
            uint64_t ol = 0;
            auto t_call = SClock::now();
            int r = sa_seed_and_filter(seeds.data(), (uint32_t)need, cl.strand, buffer, &out, &ol);
            ns_call += ns_since(t_call);
            if (r != SA_OK) {
                std::lock_guard<std::mutex> lk(err_mu);
                if (!err) {
                    err_msg = sa_last_error();
                    err = r;
                }
                break;
            }
            sa_call_stats cs;
            sa_last_call_stats(&cs);
            nseeds += need;
            nhits += cs.num_hits;
            nhsps += ol - 1;
            res[c].p = out;
            res[c].n = ol - 1;
        }
    };
    std::vector<std::thread> th;
    for (int t = 0; t < std::max(1, nthreads); ++t) th.emplace_back(worker);
    for (auto& t : th) t.join();
    if (err) {
        for (auto& r : res) sa_free_segments(r.p);
        res.clear();
        sa_set_error(err, "%s", err_msg.c_str());  // the worker's message, in the calling thread
        return err;
    }
    if (st) {
        st->num_seeds = nseeds;
        st->num_hits = nhits;
        st->num_hsps = nhsps;
        st->seed_seconds = ns_seed * 1e-9;
        st->call_seconds = ns_call * 1e-9;
    }
    return SA_OK;
}

extern "C" {

// Seeder pipeline over one query block (src/main.cpp:373-386 intervals,
// :707 q_len = Lq - seed_size; src/seeder.cpp:47-121 chunks and strands).
// Calls run on cfg->num_threads host threads; results are concatenated per
// strand in interval/chunk order.
int sa_seeder_run(const sa_seeder_cfg* cfg, const char* query, uint32_t query_len, sa_segment** fw,
                  uint64_t* fw_len, sa_segment** rc, uint64_t* rc_len, sa_seeder_stats* stats) {
    if (!cfg || !query || !fw || !fw_len || !rc || !rc_len || cfg->chunk_size == 0 || cfg->interval_size == 0)
        return SA_ERR_ARG;
    auto t0 = std::chrono::steady_clock::now();
    if (query_len < (uint32_t)g_shape.seed_size) return SA_ERR_ARG;
    std::unique_ptr<char[]> rcbuf;
    if (cfg->strand & 2) {
        rcbuf.reset(new char[query_len]);
        if (sa_host_revcomp(rcbuf.get(), query, query_len) != query_len) return SA_ERR_ARG;
    }
    const char* rctext = rcbuf.get();
    const uint32_t qlen_s = query_len - (uint32_t)g_shape.seed_size;
    std::vector<SaHostCall> calls;
    for (uint64_t cur = 0; cur < qlen_s; cur += cfg->interval_size) {
        uint32_t s = (uint32_t)cur;
        uint32_t e = (uint32_t)std::min<uint64_t>(qlen_s, cur + cfg->interval_size + cfg->interval_overlap);
        if (cfg->strand & 1)
            for (uint64_t i = s; i < e; i += cfg->chunk_size)
                calls.push_back({0, (uint32_t)i, (uint32_t)std::min<uint64_t>(i + cfg->chunk_size, e)});
        if (cfg->strand & 2) {
            uint32_t rs = qlen_s - e, re = qlen_s - s;
            for (uint64_t i = rs; i < re; i += cfg->chunk_size)
                calls.push_back({1, (uint32_t)i, (uint32_t)std::min<uint64_t>(i + cfg->chunk_size, re)});
        }
    }
    if (cfg->max_chunks && calls.size() > cfg->max_chunks) calls.resize(cfg->max_chunks);
    std::vector<SaHostCallOut> res;
    SaHostRunStats rs;
    const int nt = std::max(1, cfg->num_threads);
    using SClock = std::chrono::steady_clock;
    int err = sa_host_run_calls(calls, query, rctext, cfg->buffer, nt, res, &rs);
    if (err) return err;
    auto t_asm = SClock::now();
    auto free_all = [&]() {
        for (auto& r : res) sa_free_segments(r.p);
    };
    // per strand, the calls' HSP lists concatenated in call order: offsets
    // first, then the copies spread over the worker threads
    uint64_t nf = 0, nr = 0;
    std::vector<uint64_t> at(calls.size());
    for (size_t c = 0; c < calls.size(); ++c) {
        uint64_t& n = calls[c].strand ? nr : nf;
        at[c] = n;
        n += res[c].n;
    }
    *fw = (sa_segment*)malloc(sizeof(sa_segment) * (nf ? nf : 1));
    *rc = (sa_segment*)malloc(sizeof(sa_segment) * (nr ? nr : 1));
    if (!*fw || !*rc) {
        free(*fw);
        free(*rc);
        free_all();
        return SA_ERR_NOMEM;
    }
    {
        std::atomic<size_t> nc{0};
        auto copier = [&]() {
            for (size_t c; (c = nc.fetch_add(1)) < calls.size();) {
                if (res[c].n)
                    std::memcpy((calls[c].strand ? *rc : *fw) + at[c], res[c].p + 1, res[c].n * sizeof(sa_segment));
                sa_free_segments(res[c].p);
                res[c].p = nullptr;
            }
        };
        std::vector<std::thread> th;
        for (int t = 0; t < nt; ++t) th.emplace_back(copier);
        for (auto& t : th) t.join();
    }
    *fw_len = nf;
    *rc_len = nr;
    if (stats) {
        stats->num_seeds = rs.num_seeds;
        stats->num_hits = rs.num_hits;
        stats->num_hsps = rs.num_hsps;
        stats->num_calls = calls.size();
        stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        stats->seed_seconds = rs.seed_seconds;
        stats->call_seconds = rs.call_seconds;
        stats->copy_seconds = std::chrono::duration<double>(SClock::now() - t_asm).count();
    }
    return SA_OK;
}

}  // extern "C"

namespace {

// Index of the chromosome holding global position x: the last with start <= x
// (std::upper_bound - 1, as src/segment_printer.cpp does); 0 before the first.
uint32_t chrom_of(const uint64_t* starts, uint32_t n, uint64_t x) {
    const uint64_t* it = std::upper_bound(starts, starts + n, x);
    return it == starts ? 0u : (uint32_t)(it - starts - 1);
}

char* dup_text(const std::string& t, uint64_t* len) {
    char* p = (char*)malloc(t.size() + 1);
    if (!p) return nullptr;
    std::memcpy(p, t.data(), t.size());
    p[t.size()] = 0;
    *len = t.size();
    return p;
}

}  // namespace

extern "C" {

void sa_free_text(char* text) { free(text); }

int sa_format_segments(const sa_chrom_table* ref, uint64_t ref_block_start, const sa_chrom_table* query,
                       uint64_t query_block_start, uint32_t query_block_len, const sa_segment* fw, uint64_t n_fw,
                       const sa_segment* rc, uint64_t n_rc, char** plus_text, uint64_t* plus_len, char** minus_text,
                       uint64_t* minus_len) {
    if (!ref || !query || !ref->count || !query->count || (n_fw && !fw) || (n_rc && !rc) || !plus_text ||
        !plus_len || !minus_text || !minus_len)
        return SA_ERR_ARG;
    // reverse-complement chromosome table of the block (src/main.cpp:355-362):
    // the block's chromosomes in reverse order
    std::vector<uint64_t> rs;
    std::vector<uint32_t> rl, ri;
    for (uint32_t i = query->count; i-- > 0;) {
        const uint64_t st = query->starts[i];
        if (st < query_block_start || st >= query_block_start + query_block_len) continue;
        rs.push_back(2 * query_block_start + query_block_len - st - query->lens[i]);
        rl.push_back(query->lens[i]);
        ri.push_back(i);
    }
    if (rs.empty()) return SA_ERR_ARG;
    // "rchr rstart rend qchr " of one HSP
    auto ref_part = [&](std::string& out, const sa_segment& e, const char* qname) {
        const uint64_t sr = e.ref_start + ref_block_start;
        const uint32_t r = chrom_of(ref->starts, ref->count, sr);
        char buf[64];
        out += ref->names[r];
        std::snprintf(buf, sizeof buf, "\t%llu\t%llu\t", (unsigned long long)(sr + 1 - ref->starts[r]),
                      (unsigned long long)(sr + e.len + 1 - ref->starts[r]));
        out += buf;
        out += qname;
    };
    std::string plus, minus;
    for (uint64_t k = 0; k < n_fw; ++k) {
        const sa_segment& e = fw[k];
        const uint64_t sq = query_block_start + e.query_start;
        const uint32_t q = chrom_of(query->starts, query->count, sq);
        ref_part(plus, e, query->names[q]);
        char buf[96];
        std::snprintf(buf, sizeof buf, "\t%llu\t%llu\t+\t%d\n", (unsigned long long)(sq + 1 - query->starts[q]),
                      (unsigned long long)(sq + e.len + 1 - query->starts[q]), e.score);
        plus += buf;
    }
    for (uint64_t k = n_rc; k-- > 0;) {
        const sa_segment& e = rc[k];
        const uint64_t sq = query_block_start + e.query_start;
        const uint32_t j = chrom_of(rs.data(), (uint32_t)rs.size(), sq);
        ref_part(minus, e, query->names[ri[j]]);
        char buf[96];
        std::snprintf(buf, sizeof buf, "\t%llu\t%llu\t-\t%d\n", (unsigned long long)(sq + 1 - rs[j]),
                      (unsigned long long)(sq + e.len + 1 - rs[j]), e.score);
        minus += buf;
    }
    *plus_text = dup_text(plus, plus_len);
    *minus_text = dup_text(minus, minus_len);
    if (!*plus_text || !*minus_text) {
        free(*plus_text);
        free(*minus_text);
        return SA_ERR_NOMEM;
    }
    return SA_OK;
}

int sa_format_rm_intervals(const sa_chrom_table* chroms, uint64_t block_start, const sa_rm_run* runs, uint64_t n,
                           int markend, char** text, uint64_t* len) {
    if (!chroms || !chroms->count || (n && !runs) || !text || !len) return SA_ERR_ARG;
    std::string out;
    char buf[64];
    for (uint64_t k = 0; k < n; ++k) {
        const uint64_t sq = block_start + runs[k].query_start;
        const uint32_t c = chrom_of(chroms->starts, chroms->count, sq);
        out += chroms->names[c];
        std::snprintf(buf, sizeof buf, "\t%llu\t%llu\n", (unsigned long long)(sq - chroms->starts[c]),
                      (unsigned long long)(sq + runs[k].len + 1 - chroms->starts[c]));
        out += buf;
    }
    if (n && markend) out += "# segalign_repeat_masker end-of-file\n";
    *text = dup_text(out, len);
    return *text ? SA_OK : SA_ERR_NOMEM;
}

}  // extern "C"

namespace {

struct RmInterval {
    uint32_t block, start, end, ref_start, ref_end;
};

}  // namespace

extern "C" {

void sa_free_rm_runs(sa_rm_run* runs) { free(runs); }

int sa_rm_seeder_run(const sa_rm_seeder_cfg* cfg, const char* seq, uint64_t seq_len, sa_rm_run** runs,
                     uint64_t* n_runs, sa_rm_seeder_stats* stats) {
    if (!cfg || !seq || !runs || !n_runs || seq_len == 0 || seq_len > 0xffffffffull) return SA_ERR_ARG;
    auto t0 = std::chrono::steady_clock::now();
    const uint32_t isz = cfg->lastz_interval_size ? cfg->lastz_interval_size : 10000000u;
    uint32_t bsz = cfg->seq_block_size;
    if (!bsz) bsz = 1000000000u - 1000000000u % isz;  // repeat_masker_src/main.cpp:255-258
    const float prop = cfg->prop_neigh_interval > 0 ? cfg->prop_neigh_interval : 0.2f;
    const uint32_t M = cfg->M ? cfg->M : 1;
    const uint32_t chunk = cfg->chunk_size ? cfg->chunk_size : 250000u;
    const int strand = cfg->strand ? cfg->strand : 3;
    const uint32_t step = cfg->step ? cfg->step : 1;
    const uint32_t S = (uint32_t)g_shape.seed_size;
    // intervals and neighbour windows (repeat_masker_src/main.cpp:319-428)
    uint32_t total_iv = (uint32_t)std::ceil((float)seq_len / isz);
    const uint32_t num_neigh = (uint32_t)std::ceil(prop * total_iv);
    const uint32_t left_iv = (uint32_t)std::ceil((float)(num_neigh - 1) / 2);
    const uint32_t right_iv = num_neigh - 1 - left_iv;
    const uint32_t left_ov = left_iv * isz, right_ov = right_iv * isz;
    const uint32_t max_iv_len = left_ov + isz + right_ov;
    std::vector<uint64_t> bstart;
    std::vector<uint32_t> blen;
    std::vector<RmInterval> ivs;
    for (uint64_t l = 0; l < seq_len; l += bsz) {
        const uint64_t b0 = l < left_ov ? l : l - left_ov;
        const uint32_t bl = (l + bsz + right_ov > seq_len) ? (uint32_t)(seq_len - b0)
                                                             : (uint32_t)(l - b0 + bsz) + right_ov;
        const uint32_t blk = (uint32_t)bstart.size();
        bstart.push_back(b0);
        blen.push_back(bl);
        uint32_t start_pos = (uint32_t)(l - b0), end_pos;
        if (bl < bsz) end_pos = start_pos + bl - (uint32_t)(l - b0) - S;
        else end_pos = start_pos + bsz - S;
        while (start_pos < end_pos) {
            RmInterval iv{blk, start_pos, std::min(end_pos, start_pos + isz), 0, 0};
            const bool lim_l = iv.start < left_ov, lim_r = iv.end + right_ov > bl;
            if (lim_l) {
                iv.ref_start = 0;
                iv.ref_end = lim_r ? bl : (max_iv_len > bl ? bl : max_iv_len);
            } else if (lim_r) {
                iv.ref_end = bl;
                iv.ref_start = bl < max_iv_len ? 0 : bl - max_iv_len;
            } else {
                iv.ref_start = iv.start - left_ov;
                iv.ref_end = iv.end + right_ov;
            }
            ivs.push_back(iv);
            start_pos += isz;
        }
    }
    if (cfg->max_intervals && ivs.size() > cfg->max_intervals) ivs.resize(cfg->max_intervals);
    // reverse complement of the whole sequence, padded past its end with N
    // (minus-strand seeds near a block end read past it, as in the reference)
    std::unique_ptr<char[]> rc(new char[seq_len + 64]);
    if (sa_host_revcomp(rc.get(), seq, seq_len) != seq_len) return SA_ERR_ARG;
    std::memset(rc.get() + seq_len, 'N', 64);
    std::vector<std::vector<sa_rm_run>> out(ivs.size());
    std::atomic<uint64_t> nseeds{0}, nhits{0}, nhsps{0}, ncalls{0};
    std::atomic<int> err{0};
    const int nt = std::max(1, cfg->num_threads);
    size_t first = 0;
    uint32_t blocks_run = 0;
    while (first < ivs.size() && !err) {
        const uint32_t blk = ivs[first].block;
        size_t last = first;
        while (last < ivs.size() && ivs[last].block == blk) ++last;
        const uint64_t b0 = bstart[blk];
        const uint32_t bl = blen[blk];
        int r = sa_send_ref_write_request(seq, b0, bl);
        if (r == SA_OK) r = sa_rm_send_query_write_request();
        if (r == SA_OK) r = sa_generate_seed_pos_table(seq, b0, bl, step, (int)S, g_shape.kmer_size);
        if (r != SA_OK) return r;
        ++blocks_run;
        const char* text = seq + b0;
        const char* rctext = rc.get() + (seq_len - b0 - bl);  // repeat_masker_src/seeder.cpp:49
        std::atomic<size_t> next{first};
        auto worker = [&]() {
            const uint64_t per = 1 + (g_shape.transition ? (uint64_t)g_shape.kmer_size : 0);
            std::vector<uint64_t> seeds;
            std::vector<std::pair<uint32_t, uint32_t>> ev, cov;  // HSP (query_start, len); runs (start, len)
            while (!err) {
                const size_t k = next.fetch_add(1);
                if (k >= last) break;
                const RmInterval& iv = ivs[k];
                const uint32_t end_rc = bl - 1 - iv.start;
                ev.clear();
                auto call = [&](const char* t, uint32_t a, uint32_t b, int rev) -> int {
                    if (b <= a) return SA_OK;
                    seeds.resize((uint64_t)(b - a) * per);
                    const uint64_t n = chunk_seeds(g_shape, t, a, b, seeds.data(), seeds.size());
                    if (!n) return SA_OK;
                    sa_segment* o = nullptr;
                    uint64_t ol = 0;
                    const int rr = sa_rm_seed_and_filter(seeds.data(), (uint32_t)n, rev, iv.ref_start, iv.ref_end, &o, &ol);
                    if (rr != SA_OK) return rr;
                    nseeds += n;
                    nhits += (uint32_t)o[0].score;
                    nhsps += ol - 1;
                    ++ncalls;
                    for (uint64_t h = 1; h < ol; ++h) ev.emplace_back(o[h].query_start, o[h].len);
                    sa_free_segments(o);
                    return SA_OK;
                };
                for (uint32_t i = iv.start; i < iv.end && !err; i += chunk) {
                    const uint32_t e = std::min(i + chunk, iv.end);
                    int rr = SA_OK;
                    if (strand & 1) rr = call(text, i, e, 0);
                    if (rr == SA_OK && (strand & 2)) {
                        const uint32_t ms = bl - 1 - e;  // repeat_masker_src/seeder.cpp:115-117
                        rr = call(rctext, ms, std::min(ms + chunk, end_rc), 1);
                    }
                    if (rr != SA_OK) err = rr;
                }
                if (!err) {
                    // uint8 coverage counts and runs >= M on the GPU (repeat_masker_src/seeder.cpp:151-186)
                    const int rr = sa_device_coverage_runs(ev, bl, M, cov);
                    if (rr != SA_OK) err = rr;
                    for (const auto& r : cov) out[k].push_back({blk, (uint32_t)k, r.first, r.second});
                }
            }
        };
        std::vector<std::thread> th;
        for (int t = 0; t < nt; ++t) th.emplace_back(worker);
        for (auto& t : th) t.join();
        first = last;
    }
    if (err) return err;
    uint64_t total = 0;
    for (auto& v : out) total += v.size();
    *runs = (sa_rm_run*)malloc(sizeof(sa_rm_run) * (total ? total : 1));
    if (!*runs) return SA_ERR_NOMEM;
    uint64_t at = 0;
    for (auto& v : out)
        for (auto& x : v) (*runs)[at++] = x;
    *n_runs = total;
    if (stats) {
        stats->num_seeds = nseeds;
        stats->num_hits = nhits;
        stats->num_hsps = nhsps;
        stats->num_calls = ncalls;
        stats->num_intervals = ivs.size();
        stats->num_blocks = blocks_run;
        stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    return SA_OK;
}

}  // extern "C"
