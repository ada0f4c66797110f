// Instantiates the J kernels of one bra Hermite class (compiled once per
// LSJK_LB = 0..2 kLmax + 1 by the build) against every ket Hermite class.
#include "jkernel.cuh"

#ifndef LSJK_LB
#error "compile with -DLSJK_LB=<bra Hermite class>"
#endif

namespace lsjk {
template void launch_j<LSJK_LB, 0>(Context*, const JArgs&, int, int);
template void launch_j<LSJK_LB, 1>(Context*, const JArgs&, int, int);
template void launch_j<LSJK_LB, 2>(Context*, const JArgs&, int, int);
template void launch_j<LSJK_LB, 3>(Context*, const JArgs&, int, int);
template void launch_j<LSJK_LB, 4>(Context*, const JArgs&, int, int);
template void launch_j<LSJK_LB, 5>(Context*, const JArgs&, int, int);
template void launch_j<LSJK_LB, 6>(Context*, const JArgs&, int, int);
} // namespace lsjk
