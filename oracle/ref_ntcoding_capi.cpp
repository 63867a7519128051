// C-ABI shim over the reference's common/ntcoding.cpp (compiled from the
// reference tree by oracle/Makefile `ref`).  Test infrastructure only: it lets
// the oracle's seeding half be checked against the reference's own functions.
#include <cstddef>
#include <cstdint>
#include <string>
#include "ntcoding.h"

extern "C" {
// common/ntcoding.cpp:21-37 (expects the T/0 shape form built in src/main.cpp:152-171)
int ref_generate_shape_pos(const char* shape) { return GenerateShapePos(std::string(shape)); }
// common/ntcoding.cpp:39-41
int ref_is_transition_at_pos(int t) { return IsTransitionAtPos(t); }
// common/ntcoding.cpp:43-61
uint32_t ref_get_kmer_index_at_pos(char* seq, size_t pos, uint32_t seed_size) {
    return GetKmerIndexAtPos(seq, pos, seed_size);
}
// common/ntcoding.cpp:63-105
void ref_revcomp(char* dst, char* src, size_t rc_start, size_t start, size_t len) {
    RevComp(dst, src, rc_start, start, len);
}
}
