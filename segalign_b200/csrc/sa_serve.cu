// sa_serve.cu — serving form: a request loop over the resident target table.
//
// A request is one query sequence.  Two host threads run the loop:
//   admitter  takes queued requests in arrival order while their device
//             buffers fit in the HBM budget, and builds them on its own
//             stream with stream-ordered allocations: the packed query and
//             its reverse complement (each with its reversed copy) and the
//             per-position seed keys of both strands.
//   runner    forms each device pass from the units of all admitted requests
//             that have not run yet, oldest request first, up to pass_slots
//             seed slots, runs it through the batched path (sa_run_units)
//             and hands each finished request its HSP lists.
// A request that arrives while a pass is on the GPU is built concurrently and
// joins the next pass (continuous batching).  Units are cut as the seeder
// cuts a query block (src/main.cpp:373-386, src/seeder.cpp:47-121), and the
// batched path gives each unit the same HSP list as a plain SeedAndFilter
// call, so a request's result does not depend on what it was batched with.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/segalign_b200.h"
#include "sa_launch.h"

namespace {

using Clock = std::chrono::steady_clock;

struct ServeUnit {
    int strand;
    uint32_t j0, j1;
};

// One strand's HSP list of a request: a malloc'd array grown as the request's
// units complete (in unit order), handed to the caller as is.
struct SegBuf {
    sa_segment* p = nullptr;
    uint64_t n = 0, cap = 0;
    SegBuf() = default;
    SegBuf(const SegBuf&) = delete;
    SegBuf& operator=(const SegBuf&) = delete;
    ~SegBuf() { free(p); }
    bool append(const SaRec* r, uint64_t k) {
        if (n + k > cap) {
            const uint64_t c = std::max<uint64_t>(n + k, std::max<uint64_t>(1024, cap + cap / 2));
            void* q = realloc(p, c * sizeof(sa_segment));
            if (!q) return false;
            p = (sa_segment*)q;
            cap = c;
        }
        if (k) std::memcpy(p + n, r, k * sizeof(sa_segment));
        n += k;
        return true;
    }
};

struct Request {
    uint64_t id = 0;
    std::vector<char> text;  // until admitted
    uint32_t len = 0;
    double t_submit = 0, t_admit = 0, t_done = 0;
    void* dmem = nullptr;  // one stream-ordered allocation
    uint64_t dbytes = 0;
    const uint32_t* packed[2] = {};
    const uint32_t* keys[2] = {};
    std::vector<ServeUnit> units;
    size_t next_unit = 0;   // first unit not yet given to a pass
    size_t done_units = 0;
    uint64_t hits = 0, passes = 0, hsps = 0;
    int status = SA_OK;
    bool done = false;
    SegBuf out[2];  // per strand; written by the runner only, read once done
};

struct Server {
    sa_serve_cfg cfg{};
    SaResidentView view{};
    Clock::time_point t0;
    std::mutex mu;
    std::condition_variable cv_admit, cv_run, cv_done;
    bool stop = false;
    uint64_t next_id = 1;
    uint64_t budget = 0, in_use = 0;
    std::deque<std::shared_ptr<Request>> queued;   // submitted, not admitted
    std::deque<std::shared_ptr<Request>> active;   // admitted, units left to run or in flight
    std::map<uint64_t, std::shared_ptr<Request>> all;
    cudaStream_t admit_stream = nullptr, free_stream = nullptr;
    std::thread admitter, runner;
    bool trace = false;  // SA_SERVE_TRACE=1: one stderr line per pass and per request build

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

std::mutex g_serve_mu;  // start / stop, and the current server pointer
std::shared_ptr<Server> g_server;

// The running server, kept alive for the caller even if sa_serve_stop runs meanwhile.
std::shared_ptr<Server> current_server() {
    std::lock_guard<std::mutex> g(g_serve_mu);
    return g_server;
}

uint64_t align256(uint64_t b) { return (b + 255) & ~255ull; }

// Device bytes of a request: per strand the packed sequence with its reversed
// copy, and one key per position; plus the text staging area.
uint64_t request_bytes(uint32_t len, int strands) {
    const uint64_t packed = align256(8ull * sa_rev_words(len));
    const uint64_t keys = align256(4ull * (len ? len : 1));
    const int ns = (strands & 1) + ((strands >> 1) & 1);
    return (uint64_t)ns * (packed + keys) + packed /* forward copy for the rc */ + align256(len ? len : 1);
}

// Units of a query of `len` bases in seeder order (src/main.cpp:373-386 plus
// the interval overlap; src/seeder.cpp:47-121): per interval, its plus-strand
// chunks then its minus-strand chunks.
std::vector<ServeUnit> cut_units(uint32_t len, const sa_serve_cfg& c, uint32_t seed_size) {
    std::vector<ServeUnit> u;
    if (len <= seed_size) return u;
    const uint64_t L = len - seed_size;
    for (uint64_t cur = 0; cur < L; cur += c.interval_size) {
        const uint64_t s = cur, e = std::min<uint64_t>(L, cur + c.interval_size + c.interval_overlap);
        if (c.strands & 1)
            for (uint64_t i = s; i < e; i += c.chunk_size)
                u.push_back({0, (uint32_t)i, (uint32_t)std::min<uint64_t>(i + c.chunk_size, e)});
        if (c.strands & 2)
            for (uint64_t i = L - e; i < L - s; i += c.chunk_size)
                u.push_back({1, (uint32_t)i, (uint32_t)std::min<uint64_t>(i + c.chunk_size, L - s)});
    }
    return u;
}

// Builds a request's device buffers on the admitter stream.
int build_request(Server& sv, Request& r) {
    cudaStream_t st = sv.admit_stream;
    const uint32_t len = r.len;
    const uint64_t pw = sa_rev_words(len);
    const uint64_t packed = align256(8ull * pw), keys = align256(4ull * (len ? len : 1));
    SA_CUDA_OK(cudaMallocAsync(&r.dmem, r.dbytes, st));
    char* at = (char*)r.dmem;
    uint32_t* fwd = (uint32_t*)at;  // forward packed (+ reversed copy)
    at += packed;
    uint32_t* rc = nullptr;
    if (sv.cfg.strands & 2) {
        rc = (uint32_t*)at;
        at += packed;
    }
    uint32_t* kf = nullptr;
    uint32_t* kr = nullptr;
    if (sv.cfg.strands & 1) {
        kf = (uint32_t*)at;
        at += keys;
    }
    if (sv.cfg.strands & 2) {
        kr = (uint32_t*)at;
        at += keys;
    }
    char* d_text = at;
    SA_CUDA_OK(cudaMemcpyAsync(d_text, r.text.data(), len, cudaMemcpyHostToDevice, st));
    uint32_t* fwd0 = fwd + SA_PADW;  // word 0 of the forward sequence
    sa_launch_pad_fill(fwd, 2 * pw, st);
    sa_launch_pack_text(d_text, len, fwd0, st);
    sa_launch_reverse_packed(fwd0, len, fwd0 + pw, false, st);
    r.packed[0] = fwd0;
    if (rc) {
        uint32_t* rc0 = rc + SA_PADW;
        sa_launch_pad_fill(rc, 2 * pw, st);
        sa_launch_reverse_packed(fwd0, len, rc0, true, st);
        sa_launch_reverse_packed(rc0, len, rc0 + pw, false, st);
        r.packed[1] = rc0;
    }
    if (kf) sa_launch_query_keys(fwd0, len, sv.view.params, kf, st);
    if (kr) sa_launch_query_keys(r.packed[1], len, sv.view.params, kr, st);
    r.keys[0] = kf;
    r.keys[1] = kr;
    SA_CUDA_OK(cudaGetLastError());
    SA_CUDA_OK(cudaStreamSynchronize(st));
    return SA_OK;
}

// Completes a request (lock held): device buffers released.
void finish(Server& sv, Request& r, int status) {
    if (r.dmem) {
        cudaFreeAsync(r.dmem, sv.free_stream);
        r.dmem = nullptr;
    }
    sv.in_use -= r.dbytes;
    r.status = status;
    r.done = true;
    r.t_done = sv.now();
}

void admitter_loop(Server& sv) {
    cudaSetDevice(sv.view.dev);
    std::unique_lock<std::mutex> lk(sv.mu);
    while (true) {
        sv.cv_admit.wait(lk, [&] {
            return sv.stop || (!sv.queued.empty() && sv.in_use + sv.queued.front()->dbytes <= sv.budget);
        });
        if (sv.stop) return;
        std::shared_ptr<Request> r = sv.queued.front();
        sv.queued.pop_front();
        sv.in_use += r->dbytes;
        lk.unlock();
        const double t_build = sv.now();
        int st = build_request(sv, *r);
        if (sv.trace)
            std::fprintf(stderr, "[sa_serve] build %.4f-%.4f s: request %llu, %u bases, status %d\n", t_build, sv.now(),
                         (unsigned long long)r->id, r->len, st);
        lk.lock();
        r->text.clear();
        r->text.shrink_to_fit();
        r->t_admit = sv.now();
        if (st != SA_OK) {
            finish(sv, *r, st);
            sv.cv_done.notify_all();
            sv.cv_admit.notify_all();
            continue;
        }
        sv.active.push_back(r);
        sv.cv_run.notify_all();
    }
}

// Appends each unit's HSPs of a completed device group to its request's
// strand list (units of a request run in order, so the lists stay in seeder
// order); called on the runner thread.
struct PassSink : SaBatchSink {
    const std::vector<std::pair<std::shared_ptr<Request>, size_t>>& owner;
    explicit PassSink(const std::vector<std::pair<std::shared_ptr<Request>, size_t>>& o) : owner(o) {}
    int put(uint32_t u0, uint32_t n, const SaRec* recs, const uint32_t* cnt, const uint64_t*) override {
        uint64_t at = 0;
        for (uint32_t i = 0; i < n; ++i) {
            Request& r = *owner[u0 + i].first;
            if (!r.out[r.units[owner[u0 + i].second].strand].append(recs + at, cnt[i])) {
                sa_set_error(SA_ERR_NOMEM, "cannot hold the HSP list of request %llu", (unsigned long long)r.id);
                return SA_ERR_NOMEM;
            }
            r.hsps += cnt[i];
            at += cnt[i];
        }
        return SA_OK;
    }
};

void runner_loop(Server& sv) {
    cudaSetDevice(sv.view.dev);
    const uint64_t per = sv.view.params.transition ? 1 + (uint64_t)sv.view.params.kmer_size : 1;
    std::unique_lock<std::mutex> lk(sv.mu);
    while (true) {
        sv.cv_run.wait(lk, [&] {
            if (sv.stop) return true;
            for (auto& r : sv.active)
                if (r->next_unit < r->units.size()) return true;
            return false;
        });
        if (sv.stop) return;
        // the pass: units not yet run, oldest request first
        std::vector<SaResolvedUnit> units;
        std::vector<std::pair<std::shared_ptr<Request>, size_t>> owner;
        uint64_t slots = 0;
        bool full = false;
        for (auto& r : sv.active) {
            bool in_pass = false;
            while (r->next_unit < r->units.size()) {
                const ServeUnit& u = r->units[r->next_unit];
                const uint64_t add = (uint64_t)(u.j1 - u.j0) * per;
                if (!units.empty() && (slots + add > sv.cfg.pass_slots || units.size() >= SA_MAX_UNITS)) {
                    full = true;
                    break;
                }
                units.push_back(SaResolvedUnit{r->keys[u.strand], r->packed[u.strand], r->len, u.j0, u.j1, u.strand});
                owner.emplace_back(r, r->next_unit);
                slots += add;
                ++r->next_unit;
                in_pass = true;
            }
            if (in_pass) ++r->passes;
            if (full) break;
        }
        lk.unlock();
        // every unit is non-empty (cut_units), so the batched path's group
        // indices are indices into `units` and `owner`
        std::vector<uint64_t> hits;
        PassSink sink(owner);
        SaRunResult res{};
        res.hits = &hits;
        res.sink = &sink;
        const double t_pass = sv.now();
        const int st = sa_run_units(units.data(), (uint32_t)units.size(), true, &res);
        if (sv.trace)
            std::fprintf(stderr, "[sa_serve] pass %.4f-%.4f s: %zu units, %llu slots, %llu hits, device %.2f ms, status %d\n",
                         t_pass, sv.now(), units.size(), (unsigned long long)slots,
                         (unsigned long long)res.tot.num_hits, res.ms_total, st);
        lk.lock();
        for (size_t i = 0; i < owner.size(); ++i) {
            Request& r = *owner[i].first;
            if (r.done) continue;
            if (st != SA_OK) {
                finish(sv, r, st);
                continue;
            }
            r.hits += hits[i];
            if (++r.done_units == r.units.size()) finish(sv, r, SA_OK);
        }
        for (auto it = sv.active.begin(); it != sv.active.end();)
            it = (*it)->done ? sv.active.erase(it) : it + 1;
        sv.cv_done.notify_all();
        sv.cv_admit.notify_all();
    }
}

}  // namespace

extern "C" {

int sa_serve_start(const sa_serve_cfg* cfg) {
    std::lock_guard<std::mutex> g(g_serve_mu);
    if (g_server) {
        sa_set_error(SA_ERR_STATE, "the request loop is already running");
        return SA_ERR_STATE;
    }
    auto sv = std::make_shared<Server>();
    int r = sa_resident_view(0, &sv->view);
    if (r != SA_OK) return r;
    sv->cfg = cfg ? *cfg : sa_serve_cfg{};
    if (!sv->cfg.interval_size) sv->cfg.interval_size = 10000000;
    if (!sv->cfg.chunk_size) sv->cfg.chunk_size = sv->view.wga_chunk;
    if (!sv->cfg.strands) sv->cfg.strands = 3;
    if (!sv->cfg.pass_slots) sv->cfg.pass_slots = 1ull << 25;
    if (!sv->cfg.hbm_reserve) sv->cfg.hbm_reserve = 2ull << 30;
    if (sv->cfg.strands < 1 || sv->cfg.strands > 3 || sv->cfg.chunk_size > sv->view.max_seeds) {
        sa_set_error(SA_ERR_ARG, "strands must be 1..3 and chunk_size at most the WGA chunk");
        return SA_ERR_ARG;
    }
    SA_CUDA_OK(cudaSetDevice(sv->view.dev));
    size_t free_b = 0, total_b = 0;
    SA_CUDA_OK(cudaMemGetInfo(&free_b, &total_b));
    sv->budget = free_b > sv->cfg.hbm_reserve ? free_b - sv->cfg.hbm_reserve : 0;
    SA_CUDA_OK(cudaStreamCreateWithFlags(&sv->admit_stream, cudaStreamNonBlocking));
    SA_CUDA_OK(cudaStreamCreateWithFlags(&sv->free_stream, cudaStreamNonBlocking));
    const char* tr = std::getenv("SA_SERVE_TRACE");
    sv->trace = tr && *tr && *tr != '0';
    sv->t0 = Clock::now();
    Server* p = sv.get();
    sv->admitter = std::thread(admitter_loop, std::ref(*p));
    sv->runner = std::thread(runner_loop, std::ref(*p));
    g_server = sv;
    return SA_OK;
}

int sa_serve_submit(const char* query, uint32_t len, uint64_t* request_id) {
    if ((!query && len) || !request_id) return SA_ERR_ARG;
    std::shared_ptr<Server> sv = current_server();
    if (!sv) {
        sa_set_error(SA_ERR_STATE, "the request loop is not running (sa_serve_start)");
        return SA_ERR_STATE;
    }
    auto r = std::make_shared<Request>();
    r->len = len;
    r->text.assign(query, query + len);
    r->units = cut_units(len, sv->cfg, (uint32_t)sv->view.params.seed_size);
    r->dbytes = request_bytes(len, sv->cfg.strands);
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->stop) return SA_ERR_STATE;
    r->id = sv->next_id++;
    r->t_submit = sv->now();
    *request_id = r->id;
    sv->all[r->id] = r;
    if (r->dbytes > sv->budget) {
        sa_set_error(SA_ERR_CAPACITY, "request of %u bases needs %llu device bytes, budget %llu", len,
                     (unsigned long long)r->dbytes, (unsigned long long)sv->budget);
        r->t_admit = r->t_submit;
        r->dbytes = 0;
        finish(*sv, *r, SA_ERR_CAPACITY);
        return SA_OK;  // the failure is reported by sa_serve_wait
    }
    if (r->units.empty()) {  // shorter than a seed: empty lists, no device work
        r->t_admit = r->t_submit;
        r->dbytes = 0;
        finish(*sv, *r, SA_OK);
        return SA_OK;
    }
    sv->queued.push_back(r);
    sv->cv_admit.notify_all();
    return SA_OK;
}

int sa_serve_wait(uint64_t request_id, int timeout_ms, sa_segment** fw, uint64_t* fw_len, sa_segment** rc,
                  uint64_t* rc_len, sa_serve_request_stats* stats) {
    if (!fw || !fw_len || !rc || !rc_len) return SA_ERR_ARG;
    std::shared_ptr<Server> sv = current_server();
    if (!sv) {
        sa_set_error(SA_ERR_STATE, "the request loop is not running (sa_serve_start)");
        return SA_ERR_STATE;
    }
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->all.find(request_id);
    if (it == sv->all.end()) {
        sa_set_error(SA_ERR_ARG, "no request %llu", (unsigned long long)request_id);
        return SA_ERR_ARG;
    }
    std::shared_ptr<Request> r = it->second;
    auto ready = [&] { return r->done || sv->stop; };
    if (timeout_ms < 0) sv->cv_done.wait(lk, ready);
    else if (!sv->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) return SA_PENDING;
    if (!r->done) return SA_ERR_STATE;
    sv->all.erase(request_id);
    if (stats) {
        stats->submit_s = r->t_submit;
        stats->admit_s = r->t_admit;
        stats->done_s = r->t_done;
        stats->num_units = r->units.size();
        stats->num_passes = r->passes;
        stats->num_hits = r->hits;
        stats->num_hsps = r->hsps;
        stats->device_bytes = r->dbytes;
    }
    if (r->status != SA_OK) {
        sa_set_error(r->status, "request %llu failed", (unsigned long long)request_id);
        return r->status;
    }
    // the lists are handed over without a copy (freed by sa_free_segments)
    for (int s = 0; s < 2; ++s)
        if (!r->out[s].p && !(r->out[s].p = (sa_segment*)malloc(sizeof(sa_segment)))) return SA_ERR_NOMEM;
    *fw = r->out[0].p;
    *fw_len = r->out[0].n;
    *rc = r->out[1].p;
    *rc_len = r->out[1].n;
    for (int s = 0; s < 2; ++s) {
        r->out[s].p = nullptr;
        r->out[s].n = r->out[s].cap = 0;
    }
    return SA_OK;
}

int sa_serve_stop(void) {
    std::lock_guard<std::mutex> g(g_serve_mu);
    if (!g_server) return SA_OK;
    Server& sv = *g_server;
    {
        std::lock_guard<std::mutex> lk(sv.mu);
        sv.stop = true;
    }
    sv.cv_admit.notify_all();
    sv.cv_run.notify_all();
    sv.cv_done.notify_all();
    if (sv.admitter.joinable()) sv.admitter.join();
    if (sv.runner.joinable()) sv.runner.join();
    cudaSetDevice(sv.view.dev);
    {
        std::lock_guard<std::mutex> lk(sv.mu);
        for (auto& kv : sv.all)
            if (!kv.second->done) finish(sv, *kv.second, SA_ERR_STATE);
    }
    cudaStreamSynchronize(sv.free_stream);
    cudaStreamDestroy(sv.admit_stream);
    cudaStreamDestroy(sv.free_stream);
    g_server.reset();
    return SA_OK;
}

}  // extern "C"
