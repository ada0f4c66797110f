// Instantiates the K kernels whose partner/indexed classes are (L1, L2) on the
// bra side (compiled once per LSJK_L1, LSJK_L2 in 0..kLmax by the build). The
// generated header holds the straight-line quartet code of the classes it
// emits; the others take the loop form (quartet_loops.cuh).
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
#define LSJK_K_ROW(L3)                                                                   \
    template void launch_k<LSJK_L1, LSJK_L2, L3, 0>(Context*, const KArgs&, long, bool); \
    template void launch_k<LSJK_L1, LSJK_L2, L3, 1>(Context*, const KArgs&, long, bool); \
    template void launch_k<LSJK_L1, LSJK_L2, L3, 2>(Context*, const KArgs&, long, bool); \
    template void launch_k<LSJK_L1, LSJK_L2, L3, 3>(Context*, const KArgs&, long, bool);
LSJK_K_ROW(0)
LSJK_K_ROW(1)
LSJK_K_ROW(2)
LSJK_K_ROW(3)
} // namespace lsjk
