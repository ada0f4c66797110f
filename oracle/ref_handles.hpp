// Test infrastructure: the handles oracle/ref_capi.cpp hands to ctypes (one
// reference Basis or PairList each), shared with oracle/b200_shim.cpp so the
// shim can be driven with the same reference objects.
#pragma once
#include <memory>
#include <lightspeed/basis.hpp>
#include <lightspeed/pair_list.hpp>

namespace oracle_ref {
struct RefBasis { std::shared_ptr<lightspeed::Basis> b; };
struct RefPairs { std::shared_ptr<lightspeed::PairList> p; };
} // namespace oracle_ref
