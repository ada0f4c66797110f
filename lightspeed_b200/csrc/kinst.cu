// Instantiates the K kernels whose partner/indexed classes are (L1, L2) on the
// bra side (compiled once per LSJK_L1, LSJK_L2 in 0..2 by the build).
#ifndef LSJK_L1
#error "compile with -DLSJK_L1=<L> -DLSJK_L2=<L>"
#endif
#define LSJK_STR2(x) #x
#define LSJK_STR(x) LSJK_STR2(x)
#define LSJK_KHDR(a, b) LSJK_STR(generated/kquartets_##a##b.cuh)
#define LSJK_KHDR2(a, b) LSJK_KHDR(a, b)
#include LSJK_KHDR2(LSJK_L1, LSJK_L2)
#include "kkernel.cuh"

namespace lsjk {
template void launch_k<LSJK_L1, LSJK_L2, 0, 0>(Context*, const KArgs&, long, bool);
template void launch_k<LSJK_L1, LSJK_L2, 0, 1>(Context*, const KArgs&, long, bool);
template void launch_k<LSJK_L1, LSJK_L2, 0, 2>(Context*, const KArgs&, long, bool);
template void launch_k<LSJK_L1, LSJK_L2, 1, 0>(Context*, const KArgs&, long, bool);
template void launch_k<LSJK_L1, LSJK_L2, 1, 1>(Context*, const KArgs&, long, bool);
template void launch_k<LSJK_L1, LSJK_L2, 1, 2>(Context*, const KArgs&, long, bool);
template void launch_k<LSJK_L1, LSJK_L2, 2, 0>(Context*, const KArgs&, long, bool);
template void launch_k<LSJK_L1, LSJK_L2, 2, 1>(Context*, const KArgs&, long, bool);
template void launch_k<LSJK_L1, LSJK_L2, 2, 2>(Context*, const KArgs&, long, bool);
} // namespace lsjk
