// Arguments of the J kernel and the declaration of its per-class launcher
// (defined in jkernel.cuh, instantiated in jinst.cu).
#pragma once
#include "engine.cuh"

namespace lsjk {

constexpr int kJThreads = 128;   // bra pairs per CTA (one per thread)
constexpr int kJChunk = 512;     // default ket pairs per CTA (the autotuner may pick another)
constexpr int kJBatch = kJBatchMax;   // densities sharing one pass over the quartets

struct JArgs {
    const double* bgeom;      // bra: n x 4 (p, P)
    const float* bbound;
    const int* nbra;          // device count after truncation
    double* jbra;             // n x HB accumulators
    const double* krec;       // ket records (q, Q, D_u...)
    const float* kbound;
    const int* nket;
    const double* boys;       // Boys table of order LB+LK
    const float* krec32;      // FP32 copy of the ket records (mixed precision)
    const float* boys32;      // FP32 Boys table of order LB+LK
    int* status;
    unsigned long long* qcount;     // FP64 quartets of this class
    unsigned long long* qcount32;   // FP32 quartets of this class
    int mixed;                // 1: quartets with estimate < thredp run in FP32
    float thredp;
    int chunk;                // ket pairs per CTA (grid.y = ceil(nket / chunk))
    int ng;                   // densities of the build (1..kMaxDens); CTA z covers NG of them
    int slots;                // density blocks per ket record (= ng)
    long jbra_stride;         // distance between the densities' bra accumulators
    int nterm;
    double alpha[4], omega[4];
    float thresp;
};

template <int LB, int LK>
void launch_j(Context* ctx, const JArgs& A, int nbra_full, int nket_full);

} // namespace lsjk
