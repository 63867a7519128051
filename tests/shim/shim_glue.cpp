// The glue file INTEGRATION.md describes, verbatim: the reference's own
// interface headers followed by include/segalign_b200_shim.hpp.  Linked with
// the reference's unchanged src/seeder.cpp by tests/shim/Makefile.
#include "seed_filter.h"            // src/seed_filter.h:4-14 (typedefs, segmentPair)
#include "seed_filter_interface.h"  // common/seed_filter_interface.h:3-11
#include "ntcoding.h"               // GenerateSeedPosTable declaration
#include "store.h"                  // query_DRAM (read by SendQueryWriteRequest)
#define SEGALIGN_B200_SHIM_PLAIN
#include "segalign_b200_shim.hpp"
