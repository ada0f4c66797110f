/*
 * lsjk.h -- C ABI of the B200 Coulomb/exchange (J/K) engine.
 *
 * This is the boundary the Lightspeed IntBox J/K path binds to. It replaces the
 * closed TeraChem library behind IntBox::coulombTC / exchangeTC
 * (src/cpp/intbox/tc/coulomb.cpp:14-63, tc/exchange.cpp:14-77 in the reference)
 * and is called from the C++ IntBox::coulomb / IntBox::exchange shim in
 * lightspeed_b200/csrc/host/lightspeed.cpp, which keeps the reference signatures
 * (src/lightspeed/intbox.hpp:761-771 and :817-828).
 *
 * Conventions
 *  - Plain C types only; every function returns 0 on success and a nonzero
 *    LSJK_E* code on failure, with a message from lsjk_last_error() (per
 *    thread). No entry point falls back to the CPU.
 *  - Matrices are dense row-major double arrays in the basis' AO ("pure")
 *    representation, exactly the Lightspeed Tensor layout (src/lightspeed/
 *    tensor.hpp:19-320). Results are ACCUMULATED into the caller's arrays, as
 *    IntBox::coulomb/exchange do when J12/K13 is passed in.
 *  - Host-pointer entry points copy in and out on the context's stream and
 *    return after the result is in host memory. The *_device entry points take
 *    device pointers and only enqueue work on the context's stream.
 *  - A context is not reentrant: one caller thread at a time (the reference's
 *    TCIntBox session has the same rule, tc/tcintbox/tcintbox.cpp:75-78).
 */
#ifndef LSJK_H
#define LSJK_H

#ifdef __cplusplus
extern "C" {
#endif

#define LSJK_OK            0
#define LSJK_EINVAL        1   /* bad argument / shape / unsupported basis    */
#define LSJK_ECUDA         2   /* CUDA runtime error                          */
#define LSJK_ENOMEM        3   /* device allocation failed                    */
#define LSJK_EKERNEL       4   /* a kernel reported an error status           */
#define LSJK_ENOTSUPP      5   /* angular momentum beyond the built kernels   */

/* Precision policy (reference semantics, src/lightspeed/intbox.hpp:730-740):
 * quartets whose estimate is >= thredp run in FP64, those in [thresp, thredp)
 * in FP32 (LSJK_PREC_MIXED); LSJK_PREC_FP64 runs every quartet >= thresp in
 * FP64, like the reference CPU path. Accumulation is always FP64. */
#define LSJK_PREC_MIXED 0
#define LSJK_PREC_FP64  1

typedef struct lsjk_context  lsjk_context;
typedef struct lsjk_basis    lsjk_basis;
typedef struct lsjk_pairlist lsjk_pairlist;

/* Work counters accumulated since the context was created or last reset.
 * Quartets are primitive quartets that passed the screen (counted once per
 * quartet, whatever the number of Ewald terms); flops are algorithmic flops
 * per quartet class x quartets (one Ewald term). */
typedef struct lsjk_stats {
    double quartets_fp64;      /* primitive quartets evaluated in FP64 (J + K) */
    double quartets_fp32;      /* ... in FP32                                  */
    double j_quartets;         /* J quartets (both precisions)                 */
    double k_quartets;         /* K quartets (both precisions)                 */
    double ms_j;               /* reserved (0)                                 */
    double ms_k;               /* reserved (0)                                 */
    double flops_j;            /* algorithmic flops of the J quartets          */
    double flops_k;            /* algorithmic flops of the K quartets          */
    long   kernel_launches;    /* kernels launched (host count)                */
} lsjk_stats;

/* Last error message of the calling thread ("" if none). */
const char* lsjk_last_error(void);

/* Library version string. */
const char* lsjk_version(void);

/* Number of device allocations (cudaMalloc) the library has made since it was
 * loaded, over all contexts: a caller can check that a call allocated nothing
 * by reading it before and after. No counterpart in the reference. */
long lsjk_device_allocations(void);

/* ---- context: one per device; owns the stream, tables and scratch memory.
 * Replaces the TCIntBox session (tc/tcintbox/tcintbox.cpp:20-50). */
int lsjk_context_create(int device, lsjk_context** out);
int lsjk_context_destroy(lsjk_context* ctx);
int lsjk_context_set_precision(lsjk_context* ctx, int mode);
/* Merge mode for K (on = 1; off, the default). Some basis sets (cc-pVXZ, ANO)
 * repeat one s exponent of an atom in several contracted shells; the
 * reference treats every copy as a primitive of its own
 * (src/cpp/core/pair_list.cpp:29-177). In merge mode each basis carries a
 * twin with one primitive per distinct (atom, s exponent); K builds compute
 * each of its integrals once and contract it into every shell that shares
 * it, screening with bounds that cover every copy, so every quartet the
 * reference keeps is kept (plus copies just below thresp): K equals the
 * reference's within the size of those sub-threshold quartets (~1e-11 on
 * C10H22-C40H82 / cc-pVDZ at thresp 1e-14, ~2e-12 on a small molecule), with
 * fewer quartets computed. Off: K runs over the primitives as given, the
 * reference's exact quartet set (the counters then equal the reference's
 * count). J always runs over the primitives as given. No counterpart in the
 * reference. */
int lsjk_context_set_merge(lsjk_context* ctx, int on);
/* The CUDA stream (cudaStream_t) the context enqueues on, as void*. */
void* lsjk_context_stream(lsjk_context* ctx);
int lsjk_context_stats(lsjk_context* ctx, lsjk_stats* out);
int lsjk_context_reset_stats(lsjk_context* ctx);
/* Largest shell the kernels take (f) and the class counts it gives: J classes
 * (LB, LK) with Hermite orders LB, LK = 0..2 LSJK_LMAX, K classes (L1,L2,L3,L4)
 * with L = 0..LSJK_LMAX. */
#define LSJK_LMAX 3
#define LSJK_NJCLASS ((2 * LSJK_LMAX + 1) * (2 * LSJK_LMAX + 1))
#define LSJK_NKCLASS ((LSJK_LMAX + 1) * (LSJK_LMAX + 1) * (LSJK_LMAX + 1) * (LSJK_LMAX + 1))
/* Raw per-class quartet counters: [precision FP64, FP32][J classes
 * LB*(2 LSJK_LMAX+1)+LK, K classes ((L1*n+L2)*n+L3)*n+L4 with n = LSJK_LMAX+1];
 * n must be >= 2*(LSJK_NJCLASS+LSJK_NKCLASS). */
int lsjk_context_counters(lsjk_context* ctx, unsigned long long* out, int n);
/* Algorithmic flops of the quartets counted since the last reset, split by
 * precision: out[0] J in FP64, out[1] J in FP32, out[2] K in FP64, out[3] K
 * in FP32 (the per-class flop counts of lsjk_stats, by precision). For the
 * mixed-precision roofline sum_prec flops_prec / peak_prec. No counterpart in
 * the reference. */
int lsjk_context_flops_split(lsjk_context* ctx, double* out4);

/* Autotuner. While on, every J/K build first times candidate launch schedules
 * of each class it meets (J: ket pairs per CTA; K: CTAs per SM of each pass)
 * on scratch outputs and keeps the fastest in the context's table; builds
 * then use the table. The table (LSJK_TUNE_INTS ints: J chunk per (LB,LK),
 * then K CTAs/SM per pass and class; 0 = default) can be saved and restored
 * (set = 0: read, 1: write) so a workload is tuned once. */
#define LSJK_TUNE_INTS (LSJK_NJCLASS + 2 * LSJK_NKCLASS)
int lsjk_context_set_autotune(lsjk_context* ctx, int on);
int lsjk_context_tune_table(lsjk_context* ctx, int* table, int n, int set);
/* Copy the device status word of the context's kernels (0 = no error). */
int lsjk_context_status(lsjk_context* ctx, int* status);
/* Measured FMA throughput of the device (fp64 = 1: FP64 pipe, 0: FP32),
 * TFLOP/s; the roofline denominator of the J/K kernels. */
int lsjk_measure_fma_peak(lsjk_context* ctx, int fp64, double* tflops);

/* ---- basis: primitive shells exactly as lightspeed::Primitive
 * (src/lightspeed/basis.hpp:143-172); xyz is nprim x 3. Dense primIdx,
 * aoIdx, cartIdx, shellIdx and atomIdx are validated as in the Basis
 * constructor (basis.hpp:433-470). */
int lsjk_basis_create(lsjk_context* ctx, int nprim,
                      const double* c, const double* e, const double* xyz,
                      const int* L, const int* is_pure, const int* aoIdx,
                      const int* cartIdx, const int* primIdx, const int* shellIdx,
                      const int* atomIdx, lsjk_basis** out);
int lsjk_basis_destroy(lsjk_basis* basis);
int lsjk_basis_nao(const lsjk_basis* basis);
int lsjk_basis_ncart(const lsjk_basis* basis);

/* Cartesian -> pure coefficients of one shell of angular momentum L (0..6):
 * coef is (2L+1) x ncart(L), pure order m = 0, +1, -1, +2, -2, ..., Cartesian
 * order CCA lexical; the transform the engine applies to D, J and K (the
 * reference's AngularMomentum coefficients, src/cpp/core/am.cpp:74-220).
 * Host only; needs no GPU. */
int lsjk_solid_harmonics(int L, double* coef);

/* ---- pair list: PairList::build_schwarz (src/cpp/core/pair_list.cpp:29-177)
 * built on the device: Schwarz bounds of all primitive pairs (pair_list.cpp:
 * 15-27), pairs with bound > thre kept (lower triangle if symmetric), grouped
 * by (L1, L2) and sorted by bound descending, then prim1, prim2 ascending
 * (pair_list_util.cpp:12-20). */
int lsjk_pairlist_build_schwarz(lsjk_context* ctx, const lsjk_basis* basis1,
                                const lsjk_basis* basis2, int is_symmetric, float thre,
                                lsjk_pairlist** out);
int lsjk_pairlist_destroy(lsjk_pairlist* pl);
long lsjk_pairlist_size(const lsjk_pairlist* pl);
/* Copy the pairs out in class order (L1-major, then L2) and sorted order. */
int lsjk_pairlist_export(const lsjk_pairlist* pl, int* L1, int* L2, int* prim1,
                         int* prim2, float* bound);

/* ---- J: J12 += sum_rs (pq|rs) D34_rs for the Ewald operator
 * O(r) = sum_i scales[i] erf(omegas[i] r)/r (omega = -1: 1/r), ndens densities
 * at once. IntBox::coulomb (src/lightspeed/intbox.hpp:761-771,
 * src/cpp/intbox/intbox.cpp:213-250). D34[k] is (nao3, nao4), J12[k] is
 * (nao1, nao2), host memory. Up to 64 densities go through one build: one
 * kernel launch per class for all of them (more are taken 64 at a time). */
int lsjk_coulomb(lsjk_context* ctx, int nterm, const double* scales, const double* omegas,
                 const lsjk_pairlist* pl12, const lsjk_pairlist* pl34, int ndens,
                 const double* const* D34, float thresp, float thredp, double* const* J12);

/* ---- K: K13 += sum_qs (pq|rs) D24_qs with the reference's density-screened
 * K-invert ordering. IntBox::exchange (src/lightspeed/intbox.hpp:817-828,
 * src/cpp/intbox/intbox.cpp:290-330). D24symm requires basis 2 == basis 4
 * (LSJK_EINVAL otherwise, like src/cpp/intbox/cpu/exchange.cpp:74-76).
 * Up to 64 densities go through one build: groups of four share a task list
 * screened with their largest |D24|, and one kernel launch per class and
 * precision pass serves every group (more are taken 64 at a time). */
int lsjk_exchange(lsjk_context* ctx, int nterm, const double* scales, const double* omegas,
                  const lsjk_pairlist* pl12, const lsjk_pairlist* pl34, int ndens,
                  const double* const* D24, int D24symm, float thresp, float thredp,
                  double* const* K13);

/* Device-resident variants: D and J/K are device pointers (same layout); the
 * work is only enqueued on the context stream. Used when the caller keeps its
 * matrices in HBM across SCF iterations. */
int lsjk_coulomb_device(lsjk_context* ctx, int nterm, const double* scales, const double* omegas,
                        const lsjk_pairlist* pl12, const lsjk_pairlist* pl34, int ndens,
                        const double* const* D34_dev, float thresp, float thredp,
                        double* const* J12_dev);
int lsjk_exchange_device(lsjk_context* ctx, int nterm, const double* scales, const double* omegas,
                         const lsjk_pairlist* pl12, const lsjk_pairlist* pl34, int ndens,
                         const double* const* D24_dev, int D24symm, float thresp, float thredp,
                         double* const* K13_dev);

/* J12_dev += J[D34_dev] for one density (device pointers, like
 * lsjk_coulomb_device), allocating no device memory. No counterpart in the
 * reference: it is for callers that may not call cudaMalloc/cudaFree while
 * they run -- a host framework that owns all of the GPU's memory and forbids
 * allocation after start-up, or a latency-bound loop that cannot take the
 * device-wide synchronisation an allocation or free can cause. Every
 * intermediate buffer of the build comes from one static device array of
 * LSJK_NOALLOC_SCRATCH_BYTES that each GPU loading this library holds until
 * the process exits; a build that needs more is rejected with LSJK_ENOMEM
 * (and a message naming the limit) before anything is written to J12_dev.
 * The first call on a device (and again after a device reset replaced its
 * CUDA context) looks up the array's device address: make that first call
 * before any stream capture. All calls on a device share the
 * array, which keeps the previous call's contents (the build clears what must
 * start at zero), so calls whose GPU work overlaps -- on different streams or
 * contexts of the same device -- race. */
#define LSJK_NOALLOC_SCRATCH_BYTES (32u << 20)
int lsjk_coulomb_device_noalloc(lsjk_context* ctx, int nterm, const double* scales, const double* omegas,
                                const lsjk_pairlist* pl12, const lsjk_pairlist* pl34,
                                const double* D34_dev, float thresp, float thredp, double* J12_dev);

/* Two-electron integrals in an MO basis through J builds: for host
 * coefficient blocks C1 (nao1 x n1), C2 (nao2 x n2), C3 (nao3 x n3),
 * C4 (nao4 x n4), row-major, with nao1/nao2 the bases of pl12 and nao3/nao4
 * those of pl34, writes (overwrites) I[i][j][k][l] = (C1_i C2_j | C3_k C4_l)
 * (host, n1*n2*n3*n4 doubles). Replaces IntBox::eriJ
 * (src/cpp/intbox/mo_eri.cpp:10-157): one J build per (i, j), with i >= j
 * when sym12, of the density C1[:,i] C2[:,j]^T over pl34's pairs (bra pl34,
 * ket pl12, mo_eri.cpp:74-118), then I[i][j] = C3^T J C4. Here the densities
 * are formed on the device and go through the batched J path 64 at a time;
 * J never leaves the device. The flags stand for the reference's
 * pointer-identity tests and select its symmetrisations (mo_eri.cpp:121-155):
 * sym12 for C1 == C2, sym34 for C3 == C4, sym1234 for C1 == C3 and C2 == C4.
 * n3 is at most 65535 (LSJK_EINVAL above). */
int lsjk_eri_j(lsjk_context* ctx, int nterm, const double* scales, const double* omegas,
               const lsjk_pairlist* pl12, const lsjk_pairlist* pl34, int n1, int n2, int n3, int n4,
               const double* C1, const double* C2, const double* C3, const double* C4, int sym12, int sym34,
               int sym1234, float thresp, float thredp, double* I);

/* J nuclear gradient, replaces IntBox::coulombGrad (src/lightspeed/intbox.hpp:998-1008,
 * src/cpp/intbox/intbox.cpp:423-491; CPU kernels src/cpp/intbox/cpu/coulomb_grad.cpp):
 * G (natom x 3, row-major, host) += sum_{pqrs} D12_pq d(pq|rs)/dR D34_rs over a
 * symmetric pair list; D12, D34 are host nao x nao matrices (the same pointer
 * for D12 == D34, the reference's symmetric branch). FP64 throughout (thredp
 * is ignored, as on the reference's CPU path); quartets screened like J
 * (B_pq B_rs max|D34 block| >= thresp). LSJK_EINVAL for a non-symmetric list. */
int lsjk_coulomb_grad(lsjk_context* ctx, int nterm, const double* scales, const double* omegas,
                      const lsjk_pairlist* pl, const double* D12, const double* D34, float thresp, float thredp,
                      double* G);

/* One-electron integrals on the device, replacing IntBox::overlapCPU,
 * kineticCPU and potentialCPU (src/lightspeed/intbox.hpp overlap/kinetic/
 * potential; CPU kernels src/cpp/intbox/cpu/overlap.cpp, kinetic.cpp,
 * potential.cpp): out (host, nao1 x nao2 of the pair list's bases, row-major)
 * += S, T, or V = sum_C -Z_C <a| O(r - C) |b> for natom point charges xyzc
 * (natom x 4: x, y, z, Z) under the Ewald operator. Every primitive pair of
 * the list contributes (no further screening), as in the reference. */
int lsjk_overlap(lsjk_context* ctx, const lsjk_pairlist* pl, double* out);
int lsjk_kinetic(lsjk_context* ctx, const lsjk_pairlist* pl, double* out);
int lsjk_potential(lsjk_context* ctx, int nterm, const double* scales, const double* omegas, const lsjk_pairlist* pl,
                   int natom, const double* xyzc, double* out);

/* K nuclear gradient, replaces IntBox::exchangeGrad (src/lightspeed/intbox.hpp:1095-1160,
 * src/cpp/intbox/intbox.cpp:519-588; CPU kernels src/cpp/intbox/cpu/exchange_grad.cpp):
 * G (natom x 3, row-major, host) += sum_{pqrs} D13_pr d(pq|rs)/dR D24_qs over a
 * symmetric pair list; D13, D24 are host nao x nao matrices. D13symm, D24symm
 * and Dsame are the reference's promises (symmetric D13, symmetric D24, D13 ==
 * D24): with D13symm and D24symm the engine computes each pair of equal terms
 * (12|34), (34|12) once and doubles it; all three select the reference's fully
 * symmetric routine, whose screen (and result near thresp) the engine
 * reproduces, reading D13 alone. A false promise gives a wrong gradient, as in
 * the reference. FP64
 * throughout (thredp is ignored, as on the reference's CPU path); quartets
 * screened like K (B_12 B_34 max|D24 block| >= thresp). LSJK_EINVAL for a
 * non-symmetric list. */
int lsjk_exchange_grad(lsjk_context* ctx, int nterm, const double* scales, const double* omegas,
                       const lsjk_pairlist* pl, const double* D13, const double* D24, int D13symm, int D24symm,
                       int Dsame, float thresp, float thredp, double* G);

/* ---- CUDA graphs: capture the builds issued through the *_device entry
 * points between lsjk_graph_begin and lsjk_graph_end on the context stream,
 * then replay them with one lsjk_graph_launch (an SCF iteration's J+K as one
 * graph). Each captured call must have run once before with the same pair
 * lists, densities and sizes (one-time set-up and scratch growth happen
 * outside capture). No reference counterpart: the reference re-enters
 * TeraChem per call (tc/coulomb.cpp:30-55). */
typedef struct lsjk_graph lsjk_graph;
int lsjk_graph_begin(lsjk_context* ctx);
int lsjk_graph_end(lsjk_context* ctx, lsjk_graph** out);
int lsjk_graph_launch(lsjk_graph* graph);
int lsjk_graph_destroy(lsjk_graph* graph);

#ifdef __cplusplus
}
#endif

#endif /* LSJK_H */
