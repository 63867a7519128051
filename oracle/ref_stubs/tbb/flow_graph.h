// Stand-in for the parts of TBB's flow-graph header that the reference's
// src/graph.h and repeat_masker_src/graph.h name in type declarations
// (tbb::flow::tuple, multifunction_node<...>::output_ports_type).  The
// reference's seed-filter translation units only need the types to exist;
// no flow graph is built by the harness that links them.  Test infrastructure.
#pragma once
#include <cstddef>
#include <tuple>

namespace tbb {
namespace flow {
using std::get;
using std::tuple;

template <typename Input, typename Output>
struct multifunction_node {
    struct output_ports_type {};
};
}  // namespace flow
}  // namespace tbb
