// Arguments of the K kernel and the declaration of its per-class launcher
// (defined in kkernel.cuh, instantiated in kinst.cu once per (L1, L2)).
#pragma once
#include "engine.cuh"

namespace lsjk {

constexpr int kKThreads = 128;
constexpr int kKWarps = kKThreads / 32;

struct KTask {
    int i2, i4;
    double dmax;
};

// Thresholds that depend on max|D24| (exchange.cpp:48-71), kept on the device
// so the build needs no host round trip.
struct KScalars {
    unsigned long long dmax_bits;   // max |D24| as the bits of a non-negative double
    float thre12, thre34;
};

struct KArgs {
    const KTask* tasks;
    const int* ntask;
    unsigned* queue;
    const int* r12s;
    const int* r12l;
    const int* r34s;
    const int* r34l;
    const double *kab12, *e12, *x12, *y12, *z12;
    const int* cart12;
    const float* b12;
    const double *kab34, *e34, *x34, *y34, *z34;
    const int* cart34;
    const float* b34;
    BasisView b2, b4;
    const double* Dc;
    int ld4;
    double* Kc;
    int ld3;
    int flip;
    float thresp;
    const KScalars* sc;
    const double* rys;     // table block of this rule
    const double* asym_t;
    const double* asym_w;
    int nbin;
    double tmax;
    int* status;
    unsigned long long* qcount;     // FP64 quartets of this class
    unsigned long long* qcount32;   // FP32 quartets of this class
    const float* rys32;             // FP32 copy of the table block
    const float* asym_t32;
    const float* asym_w32;
    int mixed;                      // 1: estimate < thredp runs in FP32
    float thredp;
    int nterm;
    double alpha[4], omega[4];
};

template <int L1, int L2, int L3, int L4>
void launch_k(Context* ctx, const KArgs& A, long cap);

} // namespace lsjk
