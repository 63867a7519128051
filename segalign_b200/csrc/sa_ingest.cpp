// sa_ingest.cpp — FASTA ingest, sequence blocks and the whole-file driver
// with double-buffered query blocks.
//
// Reference: src/main.cpp:297-534 reads the query and the target with kseq
// (common/kseq.h), concatenates their records with '&' into blocks of
// DEFAULT_SEQ_BLOCK_SIZE (src/graph.h:10), and cuts every query block into
// intervals; src/main.cpp:594-730 then sends each target block, and streams
// the query blocks through BUFFER_DEPTH = 2 device buffers: a block is written
// into a buffer once the seeders have finished every interval of the block
// that used it, while the seeders work on the other buffer.  Segments of each
// interval go out in lastz --segments form (src/segment_printer.cpp:51-147).
//
// The FASTA reader follows kseq's published parsing rules:
//   * a record starts at '>' (or '@'); its name runs up to the first white
//     space, the rest of the header line is a comment;
//   * sequence lines follow until a line starting with '>', '+' or '@';
//     empty lines are skipped; every other character is kept as is; a line's
//     trailing '\r' is dropped once the sequence holds more than one
//     character;
//   * after a '+' line (FASTQ) quality lines are read until they are as long
//     as the sequence; a missing or mismatched quality ends the input;
//   * gzip-compressed and plain files are read alike (zlib).
#include <cuda_runtime.h>
#include <sys/stat.h>
#include <zlib.h>

#include <algorithm>
#include <cctype>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/segalign_b200.h"
#include "../../include/segalign_b200_host.h"
#include "sa_host_internal.h"

namespace {

class FastaReader {
  public:
    explicit FastaReader(const char* path) : f_(gzopen(path, "r")), buf_(new char[kBuf]) {}
    ~FastaReader() {
        if (f_) gzclose(f_);
    }
    bool ok() const { return f_ != nullptr; }

    // Next record: its name, and its sequence appended to `out`; false at the
    // end of the input (or on a truncated FASTQ record, whose bases are then
    // taken off `out` again).
    bool next(std::string& name, std::string& out) {
        const size_t st = out.size();
        int c;
        if (!pending_) {  // skip to the next header character
            while ((c = getc()) >= 0 && c != '>' && c != '@') {
            }
            if (c < 0) return false;
        }
        pending_ = false;
        name.clear();
        // name: up to the first white space
        bool any = false;
        while ((c = getc()) >= 0 && !std::isspace(c)) {
            name.push_back((char)c);
            any = true;
        }
        if (c < 0 && !any) return false;
        if (c >= 0 && c != '\n')  // comment: the rest of the header line
            while ((c = getc()) >= 0 && c != '\n') {
            }
        // sequence lines
        while ((c = getc()) >= 0 && c != '>' && c != '+' && c != '@') {
            if (c == '\n') continue;
            out.push_back((char)c);
            append_line(out);
            if (out.size() - st > 1 && out.back() == '\r') out.pop_back();
        }
        if (c == '>' || c == '@') pending_ = true;
        if (c != '+') return true;
        // FASTQ quality: skip the '+' line, then quality lines up to the sequence length
        const size_t n = out.size() - st;
        while ((c = getc()) >= 0 && c != '\n') {
        }
        size_t ql = 0;
        if (c >= 0) {
            while (ql < n) {
                size_t line = 0;
                int d;
                bool got = false;
                while ((d = getc()) >= 0 && d != '\n') {
                    ++line;
                    got = true;
                }
                if (!got && d < 0) break;
                ql += line;
                if (d < 0) break;
            }
        }
        if (c >= 0 && ql == n) return true;
        out.resize(st);
        return false;
    }

  private:
    bool refill() {
        if (eof_) return false;
        int n = gzread(f_, buf_.get(), kBuf);
        if (n <= 0) {
            eof_ = true;
            return false;
        }
        len_ = n;
        pos_ = 0;
        return true;
    }
    int getc() {
        if (pos_ >= len_ && !refill()) return -1;
        return (unsigned char)buf_[pos_++];
    }
    // Appends the rest of the current line to s and consumes its '\n' (the
    // same characters as reading them one at a time, a buffer span at a time).
    void append_line(std::string& s) {
        while (pos_ < len_ || refill()) {
            const char* b = buf_.get() + pos_;
            const char* e = static_cast<const char*>(std::memchr(b, '\n', (size_t)(len_ - pos_)));
            if (e) {
                s.append(b, (size_t)(e - b));
                pos_ += (int)(e - b) + 1;
                return;
            }
            s.append(b, (size_t)(len_ - pos_));
            pos_ = len_;
        }
    }
    static constexpr unsigned kBuf = 1u << 20;
    gzFile f_;
    std::unique_ptr<char[]> buf_;
    int pos_ = 0, len_ = 0;
    bool eof_ = false, pending_ = false;
};

struct SeqSetImpl {
    std::string text;
    std::vector<std::string> names;
    std::vector<const char*> name_ptrs;
    std::vector<uint64_t> chrom_start;
    std::vector<uint32_t> chrom_len;
    std::vector<uint64_t> block_start;
    std::vector<uint32_t> block_len;
};

// Records joined into blocks as src/main.cpp:336-455 (query) and :486-528
// (target) join them: each record is appended at the running position; a
// block closes after the record that takes its length above block_size (no
// '&' after that record), otherwise a '&' follows the record; the last block
// drops its trailing '&' from its length.
int load_fasta(const char* path, uint64_t block_size, SeqSetImpl& s) {
    FastaReader rd(path);
    if (!rd.ok()) {
        sa_set_error(SA_ERR_ARG, "cannot open FASTA file %s", path);
        return SA_ERR_ARG;
    }
    {
        struct stat sb;
        if (stat(path, &sb) == 0 && sb.st_size > 0) s.text.reserve((size_t)sb.st_size + 16);
    }
    std::string name;
    uint64_t blk_len = 0;
    s.block_start.push_back(0);
    while (true) {
        const size_t at = s.text.size();
        if (!rd.next(name, s.text)) break;  // records are read straight into the joined text
        const uint64_t len = s.text.size() - at;
        s.names.push_back(name);
        s.chrom_start.push_back(at);
        s.chrom_len.push_back((uint32_t)len);
        blk_len += len;
        if (blk_len > block_size) {
            s.block_len.push_back((uint32_t)blk_len);
            s.block_start.push_back(s.text.size());
            blk_len = 0;
        } else {
            s.text.push_back('&');
            blk_len += 1;
        }
    }
    if (blk_len > 0) {
        s.block_len.push_back((uint32_t)(blk_len - 1));
    } else {
        s.block_start.pop_back();  // the last record closed a block: no open block follows
    }
    for (auto& n : s.names) s.name_ptrs.push_back(n.c_str());
    return SA_OK;
}

void fill_view(SeqSetImpl* impl, sa_seq_set* out) {
    out->text = impl->text.data();
    out->text_len = impl->text.size();
    out->num_chroms = (uint32_t)impl->names.size();
    out->num_blocks = (uint32_t)impl->block_len.size();
    out->names = impl->name_ptrs.data();
    out->chrom_start = impl->chrom_start.data();
    out->chrom_len = impl->chrom_len.data();
    out->block_start = impl->block_start.data();
    out->block_len = impl->block_len.data();
    out->impl = impl;
}

sa_chrom_table table_of(const SeqSetImpl& s) {
    sa_chrom_table t;
    t.names = s.name_ptrs.data();
    t.starts = s.chrom_start.data();
    t.lens = s.chrom_len.data();
    t.count = (uint32_t)s.names.size();
    t.pad = 0;
    return t;
}

double secs_since(std::chrono::steady_clock::time_point t) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t).count();
}

// Puts out the finished intervals of one query block on a thread of its own,
// in interval order, while the seeders run the next interval: per interval
// its HSP records {target block, query block, interval, strand, sa_segment}
// (plus strand first) and the lastz --segments lines of both strands from the
// GPU segment writer.  The lines come back into one of two pinned buffers,
// and a file thread writes a buffer out while the next interval is formatted
// into the other.  Takes ownership of each interval's call outputs.
class IntervalWriter {
  public:
    IntervalWriter(FILE* seg, FILE* hsp, const sa_chrom_table* ttab, uint64_t rstart, const sa_chrom_table* qtab,
                   uint64_t qs, uint32_t ql, uint32_t rb, uint32_t qb)
        : seg_(seg), hsp_(hsp), ttab_(ttab), qtab_(qtab), rstart_(rstart), qs_(qs), ql_(ql), rb_(rb), qb_(qb),
          file_th_([this] { file_run(); }), th_([this] { run(); }) {}
    ~IntervalWriter() { finish(nullptr); }

    // Queues interval iv; returns the writer's first error, if it failed.
    int push(uint32_t iv, std::vector<SaHostCall>&& calls, std::vector<SaHostCallOut>&& res) {
        std::lock_guard<std::mutex> lk(mu_);
        q_.push_back(Item{iv, std::move(calls), std::move(res)});
        cv_.notify_all();
        return err_;
    }

    // Waits until every queued interval is out; returns the first error (its
    // message becomes the calling thread's sa_last_error()).
    int finish(double* seconds) {
        {
            std::lock_guard<std::mutex> lk(mu_);
            closed_ = true;
        }
        cv_.notify_all();
        if (th_.joinable()) {
            th_.join();
            {
                std::lock_guard<std::mutex> lk(fmu_);
                fclosed_ = true;
            }
            fcv_.notify_all();
            file_th_.join();
            for (char* b : pbuf_)
                if (b) cudaFreeHost(b);
            if (err_ == SA_OK && ferr_ != SA_OK) {
                err_ = ferr_;
                msg_ = "writing the segments file failed";
            }
            if (err_ != SA_OK) sa_set_error(err_, "%s", msg_.c_str());
            if (seconds) *seconds += busy_;
        }
        return err_;
    }

  private:
    struct Item {
        uint32_t iv = 0;
        std::vector<SaHostCall> calls;
        std::vector<SaHostCallOut> res;
    };

    void run() {
        while (true) {
            Item it;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return closed_ || !q_.empty(); });
                if (q_.empty()) return;
                it = std::move(q_.front());
                q_.pop_front();
            }
            const auto t0 = std::chrono::steady_clock::now();
            const int e = err_ == SA_OK ? write(it) : err_;  // after a failure the rest is only freed
            for (auto& x : it.res) sa_free_segments(x.p);
            busy_ += secs_since(t0);
            if (e != SA_OK && err_ == SA_OK) {
                msg_ = sa_last_error();
                std::lock_guard<std::mutex> lk(mu_);
                err_ = e;
            }
        }
    }

    int write(const Item& it) {
        std::vector<sa_segment> fw, rc;
        for (size_t c = 0; c < it.calls.size(); ++c) {
            if (!it.res[c].p) continue;
            auto& dst = it.calls[c].strand ? rc : fw;
            dst.insert(dst.end(), it.res[c].p + 1, it.res[c].p + 1 + it.res[c].n);
        }
        if (hsp_) {
            struct Rec {
                uint32_t key[4];
                sa_segment h;
            };
            static_assert(sizeof(Rec) == 32, "HSP record layout");
            std::vector<Rec> out;
            out.reserve(fw.size() + rc.size());
            for (int sd = 0; sd < 2; ++sd)
                for (const sa_segment& h : sd ? rc : fw) out.push_back(Rec{{rb_, qb_, it.iv, (uint32_t)sd}, h});
            if (!out.empty() && fwrite(out.data(), sizeof(Rec), out.size(), hsp_) != out.size()) {
                sa_set_error(SA_ERR_ARG, "writing the HSP record file failed");
                return SA_ERR_ARG;
            }
        }
        if (seg_ && (fw.size() || rc.size())) {
            const int b = next_;
            next_ ^= 1;
            {
                std::unique_lock<std::mutex> lk(fmu_);
                fcv_.wait(lk, [&] { return !pbusy_[b]; });  // its previous text is on file
                if (ferr_ != SA_OK) return SA_OK;            // finish() reports the file error
            }
            uint64_t pl = 0, ml = 0;
            const int f = sa_format_segments_pinned(ttab_, rstart_, qtab_, qs_, ql_, fw.data(), fw.size(), rc.data(),
                                                    rc.size(), &pbuf_[b], &pcap_[b], &pl, &ml);
            if (f == SA_ERR_NOMEM) return write_unpinned(fw, rc);
            if (f != SA_OK) return f;
            std::lock_guard<std::mutex> lk(fmu_);
            pbusy_[b] = true;
            fq_.push_back({b, pl + ml});
            fcv_.notify_all();
        }
        return SA_OK;
    }

    // An interval whose text does not fit in pinned memory: formatted into
    // ordinary host memory and written here, after the queued buffers.
    int write_unpinned(const std::vector<sa_segment>& fw, const std::vector<sa_segment>& rc) {
        {
            std::unique_lock<std::mutex> lk(fmu_);
            fcv_.wait(lk, [&] { return fq_.empty() && !pbusy_[0] && !pbusy_[1]; });
            if (ferr_ != SA_OK) return SA_OK;  // finish() reports the file error
        }
        char *pt = nullptr, *mt = nullptr;
        uint64_t pl = 0, ml = 0;
        const int f = sa_format_segments_gpu(ttab_, rstart_, qtab_, qs_, ql_, fw.data(), fw.size(), rc.data(), rc.size(),
                                             &pt, &pl, &mt, &ml);
        const bool ok = f == SA_OK && fwrite(pt, 1, pl, seg_) == pl && fwrite(mt, 1, ml, seg_) == ml;
        sa_free_text(pt);
        sa_free_text(mt);
        if (f != SA_OK) return f;
        if (!ok) {
            sa_set_error(SA_ERR_ARG, "writing the segments file failed");
            return SA_ERR_ARG;
        }
        return SA_OK;
    }

    // File thread: writes the formatted buffers in the order they were queued.
    void file_run() {
        while (true) {
            std::pair<int, uint64_t> job;
            {
                std::unique_lock<std::mutex> lk(fmu_);
                fcv_.wait(lk, [&] { return fclosed_ || !fq_.empty(); });
                if (fq_.empty()) return;
                job = fq_.front();
                fq_.pop_front();
            }
            const bool ok = ferr_ == SA_OK && fwrite(pbuf_[job.first], 1, job.second, seg_) == job.second;
            std::lock_guard<std::mutex> lk(fmu_);
            if (!ok && ferr_ == SA_OK) ferr_ = SA_ERR_ARG;
            pbusy_[job.first] = false;
            fcv_.notify_all();
        }
    }

    FILE* seg_;
    FILE* hsp_;
    const sa_chrom_table* ttab_;
    const sa_chrom_table* qtab_;
    uint64_t rstart_, qs_;
    uint32_t ql_, rb_, qb_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<Item> q_;
    bool closed_ = false;
    int err_ = SA_OK;
    std::string msg_;
    double busy_ = 0;
    // pinned text buffers and the file thread's queue of (buffer, bytes)
    char* pbuf_[2] = {nullptr, nullptr};
    uint64_t pcap_[2] = {0, 0};
    bool pbusy_[2] = {false, false};
    int next_ = 0;
    std::mutex fmu_;
    std::condition_variable fcv_;
    std::deque<std::pair<int, uint64_t>> fq_;
    bool fclosed_ = false;
    int ferr_ = SA_OK;
    std::thread file_th_;
    std::thread th_;  // last: starts once the members above are set
};

}  // namespace

extern "C" {

int sa_fasta_load(const char* path, uint32_t seq_block_size, sa_seq_set* out) {
    if (!path || !out) return SA_ERR_ARG;
    auto* impl = new SeqSetImpl();
    int r = load_fasta(path, seq_block_size ? seq_block_size : 500000000u, *impl);
    if (r != SA_OK) {
        delete impl;
        return r;
    }
    fill_view(impl, out);
    return SA_OK;
}

void sa_seq_set_free(sa_seq_set* s) {
    if (!s) return;
    delete static_cast<SeqSetImpl*>(s->impl);
    std::memset(s, 0, sizeof *s);
}

// src/main.cpp:297-730 for one target file and one query file, processor
// already initialised (sa_initialize_interface, sa_generate_shape_pos,
// sa_initialize_processor).
int sa_align_fasta(const sa_align_cfg* cfg_in, sa_align_stats* stats) {
    if (!cfg_in || !cfg_in->target_path || !cfg_in->query_path) return SA_ERR_ARG;
    auto t_all = std::chrono::steady_clock::now();
    sa_align_cfg cfg = *cfg_in;
    if (!cfg.seq_block_size) cfg.seq_block_size = 500000000u;
    if (!cfg.interval_size) cfg.interval_size = 10000000u;
    if (!cfg.chunk_size) cfg.chunk_size = 250000u;
    if (!cfg.strand) cfg.strand = 3;
    if (!cfg.num_threads) cfg.num_threads = 16;
    if (!cfg.step) cfg.step = 1;
    const int seed_size = sa_host_seed_size();
    sa_align_stats st{};

    // query first, then target (src/main.cpp:297-534)
    SeqSetImpl Q, T;
    auto t_read = std::chrono::steady_clock::now();
    int r = load_fasta(cfg.query_path, cfg.seq_block_size, Q);
    if (r == SA_OK) r = load_fasta(cfg.target_path, cfg.seq_block_size, T);
    if (r != SA_OK) return r;
    st.read_seconds = secs_since(t_read);
    st.ref_blocks = T.block_len.size();
    st.query_blocks = Q.block_len.size();
    const sa_chrom_table ttab = table_of(T), qtab = table_of(Q);

    FILE* seg = nullptr;
    FILE* hsp = nullptr;
    if (cfg.segments_path && !(seg = fopen(cfg.segments_path, "wb"))) {
        sa_set_error(SA_ERR_ARG, "cannot open %s", cfg.segments_path);
        return SA_ERR_ARG;
    }
    if (cfg.hsp_path && !(hsp = fopen(cfg.hsp_path, "wb"))) {
        if (seg) fclose(seg);
        sa_set_error(SA_ERR_ARG, "cannot open %s", cfg.hsp_path);
        return SA_ERR_ARG;
    }
    const uint32_t nq = (uint32_t)Q.block_len.size();
    for (uint32_t rb = 0; rb < T.block_len.size() && r == SA_OK; ++rb) {
        const char* rtext = T.text.data();
        const uint64_t rstart = T.block_start[rb];
        const uint32_t rlen = T.block_len[rb];
        auto t_tab = std::chrono::steady_clock::now();
        if (rb > 0) sa_clear_ref();
        r = sa_send_ref_write_request(rtext, rstart, rlen);
        if (r == SA_OK) r = sa_generate_seed_pos_table(rtext, rstart, rlen, cfg.step, seed_size, sa_host_kmer_size());
        st.table_seconds += secs_since(t_tab);
        if (r != SA_OK) break;

        // The loader writes query block k into buffer k % 2 once the seeders
        // have released that buffer (block k - 2 done), while the seeders run
        // block k - 1 from the other buffer.
        std::mutex mu;
        std::condition_variable cv;
        std::vector<int> loaded(nq, 0);  // 1 loaded, -1 failed
        int load_err = SA_OK;
        std::string load_msg;             // the loader's sa_last_error() text
        int done_upto = -1;               // blocks [0, done_upto] finished seeding
        bool abort = false;
        std::string rc_text[2];
        double write_s = 0, overlap_s = 0;
        std::thread loader([&]() {
            for (uint32_t k = 0; k < nq; ++k) {
                {
                    std::unique_lock<std::mutex> lk(mu);
                    cv.wait(lk, [&] { return abort || (int)k - 2 <= done_upto; });
                    if (abort) return;
                }
                const uint32_t b = k & 1;
                const uint64_t qs = Q.block_start[k];
                const uint32_t ql = Q.block_len[k];
                auto t0 = std::chrono::steady_clock::now();
                const bool busy = (int)k - 1 > done_upto;  // the seeders are still on the other buffer
                rc_text[b].resize(ql);
                sa_host_revcomp(&rc_text[b][0], Q.text.data() + qs, ql);
                int w = sa_send_query_write_request(Q.text.data(), qs, ql, b);
                const double dt = secs_since(t0);
                {
                    std::lock_guard<std::mutex> lk(mu);
                    write_s += dt;
                    if (busy) overlap_s += dt;
                    loaded[k] = w == SA_OK ? 1 : -1;
                    if (w != SA_OK) {
                        load_err = w;
                        load_msg = sa_last_error();
                    }
                }
                cv.notify_all();
                if (w != SA_OK) return;
            }
        });
        for (uint32_t k = 0; k < nq && r == SA_OK; ++k) {
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return loaded[k] != 0; });
                if (loaded[k] < 0) {
                    r = load_err;
                    sa_set_error(r, "query block %u: %s", k, load_msg.c_str());
                    break;
                }
            }
            const uint32_t b = k & 1;
            const uint64_t qs = Q.block_start[k];
            const uint32_t ql = Q.block_len[k];
            if (ql > (uint32_t)seed_size) {
                // intervals over [0, Lq - seed_size) (src/main.cpp:373-386, :707),
                // each with its plus-strand then its minus-strand calls
                const uint32_t qlen_s = ql - (uint32_t)seed_size;
                std::vector<std::vector<SaHostCall>> iv_calls;
                for (uint64_t cur = 0; cur < qlen_s; cur += cfg.interval_size) {
                    const uint32_t s = (uint32_t)cur;
                    const uint32_t e = (uint32_t)std::min<uint64_t>(qlen_s, cur + cfg.interval_size + cfg.interval_overlap);
                    std::vector<SaHostCall> calls;
                    if (cfg.strand & 1)
                        for (uint64_t i = s; i < e; i += cfg.chunk_size)
                            calls.push_back({0, (uint32_t)i, (uint32_t)std::min<uint64_t>(i + cfg.chunk_size, e)});
                    if (cfg.strand & 2) {
                        const uint32_t rs = qlen_s - e, re = qlen_s - s;
                        for (uint64_t i = rs; i < re; i += cfg.chunk_size)
                            calls.push_back({1, (uint32_t)i, (uint32_t)std::min<uint64_t>(i + cfg.chunk_size, re)});
                    }
                    iv_calls.push_back(std::move(calls));
                }
                // The seeders run interval i + 1 while the writer thread puts
                // out interval i: its HSP records, then its segment lines
                // (plus strand, then minus), in interval order.
                IntervalWriter wr(seg, hsp, &ttab, rstart, &qtab, qs, ql, rb, k);
                for (uint32_t iv = 0; iv < iv_calls.size() && r == SA_OK; ++iv) {
                    std::vector<SaHostCallOut> res;
                    SaHostRunStats rs;
                    auto t_calls = std::chrono::steady_clock::now();
                    r = sa_host_run_calls(iv_calls[iv], Q.text.data() + qs, rc_text[b].data(), b, cfg.num_threads, res,
                                          &rs);
                    st.calls_seconds += secs_since(t_calls);
                    if (r != SA_OK) break;
                    st.num_seeds += rs.num_seeds;
                    st.num_hits += rs.num_hits;
                    st.num_hsps += rs.num_hsps;
                    r = wr.push(iv, std::move(iv_calls[iv]), std::move(res));
                }
                const int w_r = wr.finish(&st.output_seconds);
                if (r == SA_OK) r = w_r;
                st.intervals += iv_calls.size();
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                done_upto = (int)k;
                if (r != SA_OK) abort = true;
            }
            cv.notify_all();
        }
        {
            std::lock_guard<std::mutex> lk(mu);
            abort = true;  // no further blocks for this target block
        }
        cv.notify_all();
        loader.join();
        st.query_write_seconds += write_s;
        st.overlap_seconds += overlap_s;
    }
    if (seg) fclose(seg);
    if (hsp) fclose(hsp);
    st.seconds = secs_since(t_all);
    if (stats) *stats = st;
    return r;
}

}  // extern "C"
