// Match-order planner without heap storage, compilable for the host and the
// device (one query per thread): the same plan as the host planner
// (gva_plan.cpp, itself a restatement of src/genMatchOrderCPU.cpp:670-983)
// for every query it accepts, DV mode.
//
// Where the host planner sorts with std::sort, this sorts with a stable
// insertion sort, which is what libstdc++'s std::sort does for 16 entries or
// fewer; a query whose edge, neighbour or back-edge lists grow longer, or
// that exceeds a fixed capacity below, is answered with DPLAN_HOST and left
// to the host planner, as is one whose automorphism search grows past fixed
// bounds (so that a call's time is bounded).  Restrictions are gathered
// while automorphisms are enumerated: an automorphism contributes only at the
// first vertex (in plan order) that it moves, so none has to be stored.
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define GVA_HD __host__ __device__
#else
#define GVA_HD
#endif

namespace gva {
constexpr uint32_t kDpNone = 0xffffffffu;
constexpr int kDpV = 32;          // query vertices
constexpr int kDpLines = 64;      // edge lines of the query
constexpr int kDpPhases = 96;     // E phases <= vertices, R phases <= edges
constexpr int kDpPairs = 256;     // vertex ids over all phases
constexpr int kDpKeys = 256;      // (edge label, vertex label) keys
constexpr int kDpSort = 16;       // longest list sorted as std::sort would
constexpr uint64_t kDpMaxAut = 1u << 20;    // automorphisms enumerated at most
constexpr uint64_t kDpMaxSearch = 1u << 22;  // partial maps tried at most (bounds the search's time)


// The planner proper is in gva_dplan_body.inc, written against the capacity
// constants above; a caller may include it again in a namespace of its own
// with smaller capacities (gva_dplan.cu does, for the device, where every
// thread's frame holds the planner's arrays).  Capacities only decide which
// queries are answered with DPLAN_HOST; the plans of the others are the same.
#include "gva_dplan_body.inc"

}  // namespace gva
