// synth.cpp — seeded synthetic genomes for the benchmark workloads.
//
// Stand-ins for the UCSC assembly pairs the reference runs on (no dataset is
// available offline).  Each workload reproduces the shapes of one named
// configuration: sequence lengths, chromosome counts, GC content, inserted
// homologous segments at a stated substitution divergence, inversions,
// interspersed/tandem repeat families, soft-masked (lowercase) runs and N runs.
// Output is the reference's block text: chromosomes joined by '&', no
// trailing separator (src/main.cpp:400-408, 520-529).
//
// The RNG is std::mt19937_64 with explicit integer->range mappings (no
// std::*_distribution), so a seed gives the same bytes on every machine.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <string>
#include <vector>

namespace {

struct Rng {
    std::mt19937_64 g;
    explicit Rng(uint64_t s) : g(s) {}
    uint64_t u64() { return g(); }
    // uniform integer in [a, b]
    uint64_t range(uint64_t a, uint64_t b) {
        unsigned __int128 m = (unsigned __int128)u64() * (unsigned __int128)(b - a + 1);
        return a + (uint64_t)(m >> 64);
    }
    double unit() { return (double)(u64() >> 11) * (1.0 / 9007199254740992.0); }
    double loguniform(double lo, double hi) { return std::exp(std::log(lo) + unit() * (std::log(hi) - std::log(lo))); }
};

const char kACGT[4] = {'A', 'C', 'G', 'T'};

// i.i.d. bases with P(C)=P(G)=gc/2 (4 bases per 64-bit draw).
void random_bases(Rng& r, char* dst, uint64_t n, double gc) {
    uint32_t tA = (uint32_t)((1.0 - gc) / 2 * 65536.0);
    uint32_t tC = tA + (uint32_t)(gc / 2 * 65536.0);
    uint32_t tG = tC + (uint32_t)(gc / 2 * 65536.0);
    uint64_t i = 0;
    while (i < n) {
        uint64_t x = r.u64();
        for (int k = 0; k < 4 && i < n; ++k, ++i) {
            uint32_t v = (uint32_t)(x >> (16 * k)) & 0xffff;
            dst[i] = v < tA ? 'A' : v < tC ? 'C' : v < tG ? 'G' : 'T';
        }
    }
}

char comp(char c) {
    switch (c) {
        case 'A': return 'T';
        case 'C': return 'G';
        case 'G': return 'C';
        case 'T': return 'A';
        case 'a': return 't';
        case 'c': return 'g';
        case 'g': return 'c';
        case 't': return 'a';
        default: return c;
    }
}

void revcomp(std::string& s) {
    std::reverse(s.begin(), s.end());
    for (auto& c : s) c = comp(c);
}

// Substitute each base with probability p, uniformly among the other three.
void mutate(Rng& r, std::string& s, double p) {
    uint64_t thr = (uint64_t)(p * 18446744073709551615.0);
    for (auto& c : s) {
        if (r.u64() < thr) {
            int b = c == 'A' ? 0 : c == 'C' ? 1 : c == 'G' ? 2 : 3;
            int nb = (b + 1 + (int)r.range(0, 2)) & 3;
            c = kACGT[nb];
        }
    }
}

// Runs of length U[lo,hi] at random positions until `frac` of the sequence is covered.
template <class F>
void apply_runs(Rng& r, std::string& s, double frac, uint64_t lo, uint64_t hi, F f) {
    if (s.empty()) return;
    uint64_t target = (uint64_t)(frac * (double)s.size()), covered = 0;
    while (covered < target) {
        uint64_t len = r.range(lo, hi);
        uint64_t at = r.range(0, s.size() - 1);
        uint64_t e = std::min<uint64_t>(s.size(), at + len);
        for (uint64_t i = at; i < e; ++i) s[i] = f(s[i]);
        covered += e - at;
    }
}

char to_lower(char c) { return (c >= 'A' && c <= 'Z') ? (char)(c + 32) : c; }

struct Genome {
    std::vector<std::string> chroms;
};

struct Workload {
    std::string target, query;  // block texts
    std::vector<uint64_t> tstart, tlen, qstart, qlen;
};

std::string join_block(const std::vector<std::string>& chroms, std::vector<uint64_t>& st,
                       std::vector<uint64_t>& ln) {
    std::string out;
    size_t tot = 0;
    for (auto& c : chroms) tot += c.size() + 1;
    out.reserve(tot);
    for (size_t i = 0; i < chroms.size(); ++i) {
        st.push_back(out.size());
        ln.push_back(chroms[i].size());
        out += chroms[i];
        if (i + 1 < chroms.size()) out += '&';
    }
    return out;
}

// Plain method, small: 1 Mbp x 1 Mbp, 200 inserted target segments
// (U[300,5000] bp, 25% substitutions, half reverse-complemented), 2% lowercase
// runs U[50,500], 0.1% N runs U[10,100] in both sequences.
Workload make_small(uint64_t seed, double scale, int nseg) {
    Rng r(seed);
    uint64_t L = (uint64_t)(1000000 * scale);
    std::string T(L, 'A'), Q(L, 'A');
    random_bases(r, &T[0], L, 0.36);
    random_bases(r, &Q[0], L, 0.36);
    std::vector<uint8_t> used(L, 0);
    for (int k = 0; k < nseg; ++k) {
        uint64_t len = std::min<uint64_t>(r.range(300, 5000), L / 4);
        uint64_t src = r.range(0, L - len);
        std::string seg = T.substr(src, len);
        mutate(r, seg, 0.25);
        if (k & 1) revcomp(seg);
        for (int tries = 0; tries < 1000; ++tries) {
            uint64_t at = r.range(0, L - len);
            bool ok = true;
            for (uint64_t i = at; i < at + len && ok; ++i) ok = !used[i];
            if (!ok) continue;
            for (uint64_t i = 0; i < len; ++i) {
                Q[at + i] = seg[i];
                used[at + i] = 1;
            }
            break;
        }
    }
    for (std::string* s : {&T, &Q}) {
        apply_runs(r, *s, 0.02, 50, 500, to_lower);
        apply_runs(r, *s, 0.001, 10, 100, [](char) { return 'N'; });
    }
    Workload w;
    w.target = join_block({T}, w.tstart, w.tlen);
    w.query = join_block({Q}, w.qstart, w.qlen);
    return w;
}

// Repeat families shared by target and query: motif U[10,300] bp, U[50,2000]
// copies, each copy diverged by U[5%,20%] substitutions, random orientation;
// half the families are interspersed (single copies), half tandem (arrays of
// 2-10 adjacent copies).  Families are added until `frac` of the bases are covered.
void add_repeats(Rng& r, std::vector<std::string*> seqs, double frac, double gc) {
    uint64_t total = 0;
    for (auto* s : seqs) total += s->size();
    if (total == 0) return;
    uint64_t target = (uint64_t)(frac * (double)total), covered = 0;
    while (covered < target) {
        uint64_t m = r.range(10, 300);
        uint64_t copies = r.range(50, 2000);
        bool tandem = r.range(0, 1);
        std::string motif(m, 'A');
        random_bases(r, &motif[0], m, gc);
        uint64_t placed = 0;
        while (placed < copies && covered < target) {
            uint64_t arr = tandem ? r.range(2, 10) : 1;
            // pick a sequence weighted by length
            uint64_t pick = r.range(0, total - 1), acc = 0;
            std::string* s = seqs[0];
            for (auto* q : seqs) {
                acc += q->size();
                if (pick < acc) { s = q; break; }
            }
            if (s->size() < m * arr + 1) { placed += arr; continue; }
            uint64_t at = r.range(0, s->size() - m * arr);
            bool rc = r.range(0, 1);
            for (uint64_t a = 0; a < arr; ++a) {
                std::string c = motif;
                mutate(r, c, 0.05 + 0.15 * r.unit());
                if (rc) revcomp(c);
                std::memcpy(&(*s)[at + a * m], c.data(), m);
            }
            placed += arr;
            covered += m * arr;
        }
    }
}

// A query of QL bases: pieces of U[1,50] kbp, each with probability hom_frac
// a copy of a random stretch of a target chromosome at U[div_lo,div_hi]
// divergence (5% reverse-complemented), else random bases.
std::string draw_query(Rng& r, const std::vector<std::string>& chroms, uint64_t QL, double gc, double hom_frac,
                       double div_lo, double div_hi) {
    std::string Q;
    Q.reserve(QL + 60000);
    const int nchr = (int)chroms.size();
    while (Q.size() < QL) {
        uint64_t len = r.range(1000, 50000);
        if (r.unit() < hom_frac) {
            int c = (int)r.range(0, nchr - 1);
            auto& ch = chroms[c];
            if (ch.size() <= len) continue;
            uint64_t src = r.range(0, ch.size() - len);
            std::string b = ch.substr(src, len);
            mutate(r, b, div_lo + (div_hi - div_lo) * r.unit());
            if (r.unit() < 0.05) revcomp(b);
            Q += b;
        } else {
            std::string b(len, 'A');
            random_bases(r, &b[0], len, gc);
            Q += b;
        }
    }
    Q.resize(QL);
    return Q;
}

// Plain method, genome scale: 100 Mbp target in 6 chromosomes (U[15,21] Mbp
// rescaled) vs a 108 Mbp query, GC 36%.  ~60% of the query is target blocks of
// U[1,50] kbp at U[15%,35%] divergence (5% of blocks inverted), the rest random;
// 12% repeats; 8% soft-masking in runs of U[50,2000].
// Query block b > 0 of the same job: the same final target (block 0's bytes),
// and a query drawn the same way from that target with its own random stream,
// soft-masked the same way (its repeats are the copies it draws from the
// target; no repeat families are added to it).
Workload make_genome(uint64_t seed, double scale, uint64_t tlen_full, int nchr, uint64_t qlen_full,
                     double gc, double rep_frac, double mask_frac, double hom_frac,
                     double div_lo, double div_hi, uint32_t block) {
    Rng r(seed);
    uint64_t TL = (uint64_t)(tlen_full * scale), QL = (uint64_t)(qlen_full * scale);
    std::vector<double> w(nchr);
    double ws = 0;
    for (auto& x : w) { x = 15.0 + 6.0 * r.unit(); ws += x; }
    Genome tg;
    uint64_t acc = 0;
    for (int i = 0; i < nchr; ++i) {
        uint64_t l = (i + 1 == nchr) ? TL - acc : (uint64_t)(w[i] / ws * (double)TL);
        acc += l;
        tg.chroms.emplace_back(l, 'A');
        random_bases(r, &tg.chroms.back()[0], l, gc);
    }
    std::string Q = draw_query(r, tg.chroms, QL, gc, hom_frac, div_lo, div_hi);
    std::vector<std::string*> all;
    for (auto& c : tg.chroms) all.push_back(&c);
    all.push_back(&Q);
    add_repeats(r, all, rep_frac, gc);
    for (auto* s : all) apply_runs(r, *s, mask_frac, 50, 2000, to_lower);
    if (block > 0) {
        Rng rb(seed * 0x9E3779B97F4A7C15ull + block);
        Q = draw_query(rb, tg.chroms, QL, gc, hom_frac, div_lo, div_hi);
        apply_runs(rb, Q, mask_frac, 50, 2000, to_lower);
    }
    Workload wl;
    wl.target = join_block(tg.chroms, wl.tstart, wl.tlen);
    wl.query = join_block({Q}, wl.qstart, wl.qlen);
    return wl;
}

}  // namespace

extern "C" {

// config: 1 = plain small (1 Mbp x 1 Mbp), 2 = genome scale (100 x 108 Mbp,
// 6 chromosomes), 4 = large (600 x 600 Mbp, 12 chromosomes, GC 41%, 45% repeats).
// scale multiplies the sequence lengths (1.0 = the named sizes).
// block: query block of the job (0 = the workload's own query; b > 0 = another
// query against the same target, genome configs only).
void* synth_make_block(int config, uint64_t seed, double scale, uint32_t block) {
    if (config == 1 && block > 0) return nullptr;
    Workload* w = new Workload();
    if (config == 1) *w = make_small(seed, scale, std::max(1, (int)(200 * std::min(1.0, scale))));
    else if (config == 2) *w = make_genome(seed, scale, 100000000ull, 6, 108000000ull, 0.36, 0.12, 0.08, 0.60, 0.15, 0.35, block);
    else if (config == 4) *w = make_genome(seed, scale, 600000000ull, 12, 600000000ull, 0.41, 0.45, 0.08, 0.60, 0.10, 0.30, block);
    else { delete w; return nullptr; }
    return w;
}

void* synth_make(int config, uint64_t seed, double scale) { return synth_make_block(config, seed, scale, 0); }

uint64_t synth_len(void* h, int which) {
    Workload* w = (Workload*)h;
    return which == 0 ? w->target.size() : w->query.size();
}

void synth_copy(void* h, int which, char* dst) {
    Workload* w = (Workload*)h;
    const std::string& s = which == 0 ? w->target : w->query;
    std::memcpy(dst, s.data(), s.size());
}

uint32_t synth_nchr(void* h, int which) {
    Workload* w = (Workload*)h;
    return (uint32_t)(which == 0 ? w->tstart.size() : w->qstart.size());
}

void synth_chr(void* h, int which, uint64_t* starts, uint64_t* lens) {
    Workload* w = (Workload*)h;
    auto& st = which == 0 ? w->tstart : w->qstart;
    auto& ln = which == 0 ? w->tlen : w->qlen;
    for (size_t i = 0; i < st.size(); ++i) { starts[i] = st[i]; lens[i] = ln[i]; }
}

void synth_free(void* h) { delete (Workload*)h; }

// Log-uniform chunk boundaries over [0, len): lengths in [lo, hi].
uint32_t synth_chunks(uint64_t seed, uint64_t len, double lo, double hi, uint64_t* bounds, uint32_t cap) {
    Rng r(seed);
    uint64_t at = 0;
    uint32_t n = 0;
    while (at < len) {
        uint64_t l = (uint64_t)r.loguniform(lo, hi);
        if (l == 0) l = 1;
        uint64_t e = std::min<uint64_t>(len, at + l);
        if (n < cap) { bounds[2 * n] = at; bounds[2 * n + 1] = e; }
        ++n;
        at = e;
    }
    return n;
}

}  // extern "C"
