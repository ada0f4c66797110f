// Arguments of the K kernel and the declaration of its per-class launcher
// (defined in kkernel.cuh, instantiated in kinst.cu once per (L1, L2)).
#pragma once
#include "engine.cuh"

namespace lsjk {

constexpr int kKThreads = 128;
constexpr int kKWarps = kKThreads / 32;
constexpr int kKBatch = 4;        // densities of a group (one task list, screened with their largest |D|)

// One (prim2, prim4) task of a density group: the K-invert rows of prim2
// (partners 1) and prim4 (partners 3) and the largest |D24| over the pair's
// Cartesian block and the group's densities (primitive indices < 65536).
struct KTask {
    int i2;
    unsigned short i4, grp;
    double dmax;
};

// Thresholds that depend on max|D24| (exchange.cpp:48-71), kept on the device
// so the build needs no host round trip.
struct KScalars {
    unsigned long long dmax_bits;   // max |D24| as the bits of a non-negative double
    float thre12, thre34;
};

// K-invert partner data of one pair list, in one precision (w0, w1: the
// partner's weights in its two output targets).
template <typename R>
struct KRows {
    const R *kab, *p, *ip, *px, *py, *pz, *ax, *ay, *az, *w0, *w1;
};

struct KArgs {
    const KTask* tasks;
    const int* ntask;
    unsigned* queue;             // work-queue counters, one per kernel launch of the pass
    const int* r12s;          // rows of prim2 in class (L2 indexed, L1 partner)
    const int* r12l;
    const int* r34s;          // rows of prim4 in class (L4, L3)
    const int* r34l;
    KRows<double> d12, d34;
    KRows<float> f12, f34;
    // partner output targets: first (t0) and second (t1, -1 if none) Cartesian
    // offsets, and the target group that delimits a partner-1 segment
    const int* cart12;
    const int* t1_12;
    const int* seg12;
    const float* b12;
    const int* cart34;
    const int* t1_34;
    const double* w0_34;      // partner-3 weights in FP64 (applied when a segment is flushed)
    const double* w1_34;
    const float* b34;
    BasisView b2, b4;         // indexed primitives (centres, cartIdx)
    const double* Dc[kMaxDens];  // D24 of each density of the build (Cartesian, ld4)
    int ld4;
    double* Kc[kMaxDens];        // K13 of each density (Cartesian output space of bases 1 and 3, ld3)
    int ld3;
    int ng;                      // densities of the build, in groups of kKBatch (the tasks' grp)
    int nsub;                    // densities of a group / NG of the launch, rounded up: the launch
                                 // runs its tasks nsub times (task index t + sub * ntask), sub-slot
                                 // `sub` taking densities grp * kKBatch + sub * NG + [0, NG)
    int flip;
    int gc;                      // partners may carry two output targets (merged twins): the kernel
                                 // variant with two target blocks for s-type partners
    // this pass computes quartets with thr_lo <= estimate < thr_hi
    float thr_lo, thr_hi;
    const KScalars* sc;
    const void* rys;          // table block of this rule, in the pass precision
    const void* asym_t;
    const void* asym_w;
    // FP64 table block and asymptotic nodes of this rule in global memory: the
    // FP32 pass evaluates the roots and weights in FP64 from the last table bin on
    const double* rys64g;
    const double* asym64_t;
    const double* asym64_w;
    int nbin;
    double tmax;
    int* status;
    unsigned long long* qcount;
    int nterm;
    double alpha[4], omega[4];
    int stripes;                 // k_exchange_warp: partner-3 stripes per task (work units per task)
    int split_hi;                // this is the FP64 pass of a mixed build (estimate >= thredp only)
};

// Launch the FP64 (fp32 = false) or FP32 (fp32 = true) pass of one class.
template <int L1, int L2, int L3, int L4>
void launch_k(Context* ctx, const KArgs& A, long cap, bool fp32);

// Arguments of the K gradient kernel (kgrad.cu): the K build's task list and
// bound-ordered partner rows of one exact pair list, with each partner's
// exponent and atom, one D13 and one D24 (Cartesian), and G (natom x 3).
struct KGradArgs {
    const KTask* tasks;
    const int* ntask;
    unsigned* queue;
    const int *r12s, *r12l, *r34s, *r34l;
    const float *b12, *b34;
    const double *kab12, *p12, *ip12, *px12, *py12, *pz12, *ax12, *ay12, *az12, *pe12;
    const int *cart12, *atom12, *pidx12;
    const double *kab34, *p34, *ip34, *px34, *py34, *pz34, *ax34, *ay34, *az34, *pe34;
    const int *cart34, *atom34, *pidx34;
    BasisView b2, b4;
    const double* D13;
    int ld13;
    const double* D24;
    int ld24;
    double* G;
    const KScalars* sc;
    float thr_lo;               // thresp: quartets with bound12 bound34 max|D24 block| >= thresp
    // canon != 0: the reference's fully symmetric gradient, whose screen reads the
    // D block of (max(prim1, prim2), max(prim3, prim4)) for every quartet: dblk holds
    // max|D block| per primitive pair (nprim x nprim), and the tasks carry the global max
    const double* dblk;
    int nprim;
    int canon;
    // pairsym != 0 (D13 and D24 both symmetric): the tasks have prim2 <= prim4 and
    // a task with prim2 < prim4 stands for itself and its mirror (1,2,3,4) <-> (3,4,1,2),
    // whose terms are equal: its D24 block enters doubled
    int pairsym;
    int stripes;                // k_exchange_grad_warp: partner-3 stripes per task
    const double* rys;          // FP64 Rys table block of the rule one quantum up
    const double* asym_t;
    const double* asym_w;
    int nbin;
    double tmax;
    int nterm;
    double alpha[4], omega[4];
};

// One (L1 L2|L3 L4) class of the K gradient (cap: the class's task capacity);
// launch_k_grad_l1<L1> holds the classes of one partner-1 shell.
void launch_k_grad(Context* ctx, const KGradArgs& A, long cap, int L1, int L2, int L3, int L4);
template <int L1>
void launch_k_grad_l1(Context* ctx, const KGradArgs& A, long cap, int L2, int L3, int L4);

} // namespace lsjk
