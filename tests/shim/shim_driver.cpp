// Drives the reference's unchanged seeder (src/seeder.cpp: seeder_body) over
// segalign_b200 through the drop-in shim, the way src/main.cpp does for one
// target block and one query block: InitializeInterface, SendRefWriteRequest,
// InitializeProcessor, GenerateSeedPosTable, SendQueryWriteRequest, then one
// seeder_body call per interval.  Writes the per-strand HSP lists the seeder
// returns.  Test program only.
//
// usage: shim_seeder <target.txt> <query.txt> <out.bin> [interval_size]
// out.bin: u64 n_fw, u64 n_rc, u64 seed_hits, u64 seeds, then n_fw + n_rc
// segmentPair records (plus strand first).
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "DRAM.h"
#include "graph.h"
#include "ntcoding.h"
#include "seed_filter.h"
#include "seed_filter_interface.h"
#include "store.h"

// Globals src/main.cpp defines and the seeder reads.
Configuration cfg;
DRAM* ref_DRAM = nullptr;
DRAM* query_DRAM = nullptr;
DRAM* query_rc_DRAM = nullptr;

static std::string slurp(const char* path) {
    std::string s;
    FILE* f = fopen(path, "rb");
    if (!f) return s;
    char buf[1 << 16];
    size_t n;
    while ((n = fread(buf, 1, sizeof buf, f)) > 0) s.append(buf, n);
    fclose(f);
    return s;
}

// src/main.cpp:180-261 with the default options (no --scoring, no --ambiguous):
// HOXD70, lowercase/N penalties, X fill, E rows -10 * xdrop.
static void default_scoring(int* m, int xdrop) {
    const int hoxd70[4][4] = {{91, -114, -31, -123}, {-114, 100, -125, -31}, {-31, -125, 100, -114},
                              {-123, -31, -114, 91}};
    for (int i = 0; i < NUC; ++i)
        for (int j = 0; j < NUC; ++j) {
            int v;
            if (i < 4 && j < 4) v = hoxd70[i][j];
            else if (i == E_NT || j == E_NT) v = -10 * xdrop;
            else if (i == L_NT || j == L_NT || i == N_NT || j == N_NT) v = -1000;
            else v = -100;  // X against A/C/G/T and X
            m[i * NUC + j] = v;
        }
    // X against L or N is -1000 (already set by the L/N branch)
}

int main(int argc, char** argv) {
    if (argc < 4) {
        fprintf(stderr, "usage: %s <target.txt> <query.txt> <out.bin> [interval_size]\n", argv[0]);
        return 2;
    }
    std::string target = slurp(argv[1]), query = slurp(argv[2]);
    if (target.empty() || query.empty()) return 2;
    const uint32_t interval = argc > 4 ? (uint32_t)strtoul(argv[4], nullptr, 10) : DEFAULT_LASTZ_INTERVAL;

    cfg.strand = "both";
    cfg.seed_shape = "12of19";
    cfg.seed.shape = "TTT0T00TT00T0T0TTTT";  // src/main.cpp:152-171
    cfg.seed.size = 19;
    cfg.seed.transition = false;
    cfg.step = 1;
    cfg.xdrop = 910;
    cfg.hspthresh = 3000;
    cfg.noentropy = false;
    cfg.wga_chunk_size = DEFAULT_WGA_CHUNK;
    cfg.lastz_interval_size = interval;
    cfg.num_gpu = 1;
    cfg.seed.kmer_size = GenerateShapePos(cfg.seed.shape);
    default_scoring(cfg.sub_mat, cfg.xdrop);

    ref_DRAM = new DRAM();
    query_DRAM = new DRAM();
    query_rc_DRAM = new DRAM();
    memcpy(ref_DRAM->buffer, target.data(), target.size());
    memcpy(query_DRAM->buffer, query.data(), query.size());
    RevComp(query_rc_DRAM->buffer, query_DRAM->buffer, 0, 0, query.size());  // common/ntcoding.cpp:63-105

    if (g_InitializeInterface(cfg.num_gpu) != 1) return 3;
    g_SendRefWriteRequest(ref_DRAM->buffer, 0, (uint32_t)target.size());
    g_InitializeProcessor(cfg.seed.transition, cfg.wga_chunk_size, cfg.seed.size, cfg.sub_mat, cfg.xdrop,
                          cfg.hspthresh, cfg.noentropy);
    GenerateSeedPosTable(ref_DRAM->buffer, 0, (uint32_t)target.size(), cfg.step, cfg.seed.size, cfg.seed.kmer_size);
    g_SendQueryWriteRequest(0, (uint32_t)query.size(), 0);

    // Intervals over [0, len - seed_size) as src/main.cpp:373-386 cuts them.
    const uint32_t qlen = (uint32_t)query.size();
    const uint32_t last = qlen - cfg.seed.size;
    std::vector<segmentPair> fw, rc;
    uint32_t k = 0, nint = (last + interval - 1) / interval;
    for (uint32_t s = 0; s < last; s += interval, ++k) {
        seq_block b{0, 0, 0, 0, (uint32_t)target.size(), qlen};
        seed_interval iv{s, std::min(s + interval, last), k, nint, 0};
        seeder_input in(seeder_payload(b, iv), (size_t)k);
        printer_input out = seeder_body()(in);
        auto& f = std::get<1>(std::get<0>(out));
        auto& r = std::get<2>(std::get<0>(out));
        fw.insert(fw.end(), f.begin(), f.end());
        rc.insert(rc.end(), r.begin(), r.end());
    }
    g_ClearQuery(0);
    g_ShutdownProcessor();

    FILE* fo = fopen(argv[3], "wb");
    if (!fo) return 2;
    const uint64_t hdr[4] = {fw.size(), rc.size(), (uint64_t)seeder_body::num_seed_hits.load(),
                             (uint64_t)seeder_body::num_seeds.load()};
    fwrite(hdr, 8, 4, fo);
    if (!fw.empty()) fwrite(fw.data(), sizeof(segmentPair), fw.size(), fo);
    if (!rc.empty()) fwrite(rc.data(), sizeof(segmentPair), rc.size(), fo);
    fclose(fo);
    printf("shim seeder: %zu + %zu HSPs, %llu seed hits\n", fw.size(), rc.size(),
           (unsigned long long)seeder_body::num_seed_hits.load());
    return 0;
}
