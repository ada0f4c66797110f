// Internal data structures of the B200 J/K engine (not part of the C ABI).
//
// Device memory layout (all arrays in HBM, one allocation each):
//  * Basis: per-primitive SoA (c, e, x, y, z, L, cartIdx, ...), plus the
//    pure<->Cartesian maps of its shells as CSR rows.
//  * PairList: the Schwarz-screened primitive pairs sorted exactly like the
//    reference PairList (class (L1,L2), bound desc, prim1 asc, prim2 asc).
//    Two derived views are kept next to it:
//      - JBra: pairs merged by Hermite angular momentum L1+L2 and re-sorted by
//        bound, with the Gaussian-product geometry (p, P) precomputed;
//      - KInv: the reference's K-invert lists (src/cpp/core/kvec.cpp:31-232):
//        for every "indexed" primitive, its partners sorted by bound desc, as
//        CSR rows per (L_indexed, L_partner) class, with the partner data
//        (K_ab prefactor, exponent, centre, cartIdx, bound) in SoA.
#pragma once
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>
#include <memory>
#include <stdexcept>
#include <cuda_runtime.h>
#include "../../include/lsjk.h"

namespace lsjk {

constexpr int kLmax = LSJK_LMAX;               // s, p, d, f shells
constexpr int kNL = kLmax + 1;
constexpr int kNHerm = 2 * kLmax + 1;          // Hermite classes L1+L2 = 0..6
constexpr int kGenLmax = 2;                    // largest shell of the straight-line quartet code

inline int ncart_count(int L) { return (L + 1) * (L + 2) / 2; }

// Layout of the context's device counters: quartets per class, per precision.
constexpr int kNJClass = kNHerm * kNHerm;            // (LB, LK)
constexpr int kNKClass = kNL * kNL * kNL * kNL;      // (L1, L2, L3, L4)
constexpr int kNCounters = 2 * (kNJClass + kNKClass); // [prec][J classes, K classes]
static_assert(kNJClass == LSJK_NJCLASS && kNKClass == LSJK_NKCLASS, "class counts of the C ABI");

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define LSJK_CUDA(call)                                                                    \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            throw ::lsjk::Error(LSJK_ECUDA, std::string(#call " failed: ") +              \
                                               cudaGetErrorString(e_));                    \
    } while (0)

// Device allocations the library has made since it was loaded (every
// cudaMalloc goes through DBuf::alloc); read by lsjk_device_allocations().
inline std::atomic<long> g_device_allocations{0};

// Device buffer owned by RAII (freed with the context's stream-ordered pool).
template <typename T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DBuf& operator=(DBuf&& o) noexcept { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; return *this; }
    ~DBuf() { release(); }
    void alloc(size_t count) {
        release();
        n = count;
        if (count == 0) return;
        g_device_allocations.fetch_add(1, std::memory_order_relaxed);
        cudaError_t e = cudaMalloc(&p, sizeof(T) * count);
        if (e != cudaSuccess) {
            p = nullptr;
            throw Error(LSJK_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
        }
    }
    void upload(const std::vector<T>& h, cudaStream_t s) {
        alloc(h.size());
        if (!h.empty()) LSJK_CUDA(cudaMemcpyAsync(p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, s));
    }
    void release() { if (p) cudaFree(p); p = nullptr; n = 0; }
};

struct Context;

// Primitive data on the device (SoA). For the K kernels each primitive also
// names where its contributions go in the output (Cartesian) matrix: up to two
// target shells t0, t1 (Cartesian offsets; t1 = -1 if none) with weights w0,
// w1, and `seg`, the id of the group of primitives that share those targets.
// For a basis as given: t0 = cartIdx, t1 = -1, w0 = 1, seg = shellIdx. For a
// merged basis (see Basis::twin) one primitive stands for the copies of an s
// exponent that several contracted shells of an atom share.
struct BasisView {
    int nprim, nao, ncart;
    const double *c, *e, *x, *y, *z;
    const int *L, *cart, *ao;
    const int *t0, *t1, *seg;
    const double *w0, *w1;
    const int* atom;
};

struct Basis {
    Context* ctx = nullptr;
    int nprim = 0, nao = 0, ncart = 0, nshell = 0, natom = 0, maxL = 0;
    bool has_pure = false;
    // host copies
    std::vector<double> c, e, x, y, z;
    std::vector<int> L, pure, ao, cart, prim, shell, atom;
    // output targets of each primitive (see BasisView)
    std::vector<int> t0, t1, seg;
    std::vector<double> w0, w1;
    // device copies
    DBuf<double> dc, de, dx, dy, dz;
    DBuf<int> dL, dcart, dao;
    DBuf<int> dt0, dt1, dseg, datom;
    DBuf<double> dw0, dw1;
    // pure <-> cart maps: cart row -> (pure index, coef) and pure row -> (cart index, coef)
    DBuf<int> c2p_off, c2p_idx, p2c_off, p2c_idx;
    DBuf<double> c2p_w, p2c_w;
    // per Cartesian slot of a twin: the Cartesian functions of the original basis
    // it stands for (second -1 if none) and their weights (screening densities)
    DBuf<int> uc_t0, uc_t1;
    DBuf<double> uc_w0, uc_w1;
    // The merged twin (null when no exponent is shared): one primitive per
    // distinct (atom, s exponent), with c = the largest |c| of its copies,
    // its own Cartesian slot, and pure <-> cart maps into THIS basis' AO
    // space that carry the copies' contraction weights c_copy / c. J and K
    // built over the twin equal the builds over this basis: every copy's
    // integral is the twin primitive's times its weight.
    std::unique_ptr<Basis> twin;
    bool is_twin = false;   // this basis is a merged twin (some s primitives carry two targets)
    BasisView view() const {
        return BasisView{nprim, nao, ncart, dc.p, de.p, dx.p, dy.p, dz.p, dL.p, dcart.p, dao.p,
                         dt0.p, dt1.p, dseg.p, dw0.p, dw1.p, datom.p};
    }
    bool equivalent(const Basis& o) const;
};

// One Hermite class (L1+L2 = LH) of a pair list, merged over (L1, L2) and
// sorted by bound desc (prim1, prim2 asc): the bra side of J.
struct JBraClass {
    int n = 0;                       // pairs in the class
    DBuf<int> p1, p2;                // primitive indices
    DBuf<float> bound;
    DBuf<double> geom;               // n x 4: p, Px, Py, Pz
};

// K-invert rows of one (L_indexed, L_partner) class: for every primitive of
// the indexed basis, the [start, start+len) slice of the partner arrays.
struct KInvClass {
    int nent = 0;
    DBuf<int> row_start, row_len;    // per indexed primitive (len 0: no partners)
};

// Partner entries of all K-invert rows (SoA). Each row (class, indexed prim)
// holds the partners grouped by contracted shell ("segments": same K target
// block), segments ordered by their largest bound, entries inside a segment
// by bound desc, partner asc. The quartet set does not depend on this order
// (every screen is a per-quartet test); the grouping lets the K kernel sum a
// segment in registers before one atomic update.
// Pair data are stored relative to the indexed primitive's centre R_i:
//   P_rel = P - R_i, A_rel = R_partner - R_i
// so FP32 arithmetic on them has no cancellation.
struct KInvData {
    long nent = 0;
    DBuf<double> kab, p, ip, px, py, pz, ax, ay, az;        // FP64 pair data; kab = K_ab / p
    DBuf<float> kab32, p32, ip32, px32, py32, pz32, ax32, ay32, az32;  // FP32 copies
    DBuf<int> pcart;                   // partner's first output target (t0; its cartIdx unless merged)
    DBuf<float> pbound;                // Schwarz bound of the pair
    DBuf<int> pt1, pseg;               // partner's second target (-1: none) and target group
    DBuf<double> pw0, pw1;             // partner's weights in its targets
    DBuf<float> pw0_32, pw1_32;
    DBuf<double> pe;                   // partner's exponent (the K gradient's derivatives)
    DBuf<int> patom;                   // partner's atom
    DBuf<int> pidx;                    // partner's primitive index
};

struct PairList {
    Context* ctx = nullptr;
    const Basis* b1 = nullptr;
    const Basis* b2 = nullptr;
    bool symm = false;
    float thre = 0.f;
    long npair = 0;
    // sorted pairs (reference order)
    DBuf<int> p1, p2;
    DBuf<float> bound;
    std::vector<int> cls_L1, cls_L2;   // class list in order
    std::vector<long> cls_off;         // offsets into the sorted arrays (size nclass+1)
    std::vector<float> cls_max;        // first (largest) bound of each class
    double max_bound = 0.0;            // PairListUtil::max_bound
    // J bra view per Hermite class
    JBraClass jb[kNHerm];
    // K-invert rows: [L_indexed][L_partner]
    KInvClass kinv[kNL][kNL];
    KInvData kdat;     // rows grouped by contracted shell (segments): the partner-1 side of K
    KInvData kdat_b;   // the same rows, entries by bound only: the partner-3 side of K
    bool kinv_built = false;
    // the same list over the merged twins of b1 and b2 (null when neither has one)
    std::unique_ptr<PairList> twin;
};

// Launch schedules picked by the autotuner (0 = built-in default).
struct Tune {
    int j_chunk[kNHerm][kNHerm] = {};              // ket pairs per J CTA, per (LB, LK)
    int k_ctas_per_sm[2][kNL][kNL][kNL][kNL] = {}; // K grid size, per pass (FP64, FP32) and class
};
constexpr int kTuneInts = kNHerm * kNHerm + 2 * kNL * kNL * kNL * kNL;

struct Context {
    int device = 0;
    Tune tune;
    bool tuning = false;            // time candidate schedules on the next builds
    DBuf<unsigned long long> tune_sink;  // counters written by timing launches
    cudaStream_t stream = nullptr;
    int precision = LSJK_PREC_MIXED;
    DBuf<double> boys64, rys64;     // quadrature tables (FP64)
    DBuf<float> boys32, rys32;      // FP32 copies for the mixed path
    DBuf<double> rys_asym64;
    DBuf<float> rys_asym32;
    DBuf<int> status;               // kernel error word
    DBuf<unsigned long long> counters;  // quartet counters and work queues
    lsjk_stats stats{};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
    // auxiliary streams: the per-class J and K kernels of one build are spread
    // over them (fork after the shared set-up, join before the back
    // transforms), so one class's tail overlaps the next class's start
    static constexpr int kAux = 8;
    cudaStream_t aux[kAux] = {};
    cudaEvent_t fork_ev = nullptr;
    cudaEvent_t join_ev[kAux] = {};
    // scratch buffers reused across calls (grown on demand)
    std::vector<std::unique_ptr<DBuf<char>>> scratch;
    size_t scratch_used = 0;
    bool scratch_fixed = false;     // scratch is a caller-independent fixed block: never grow
    char* scratch_take(size_t bytes);
    void scratch_reset() { scratch_used = 0; }
    int smem_optin = 0;
    int nsm = 148;                  // multiprocessors of the device
    // build K over the merged twins of the bases (shared s exponents computed
    // once); off (the default): over the primitives as given, the reference's
    // exact quartet set. J always runs over the primitives as given.
    bool merge = false;
};

// Stream-ordered scratch: a bump allocator over a few large blocks, reset at
// the start of every build (all kernels of one build run on one stream).
inline char* Context::scratch_take(size_t bytes)
{
    bytes = (bytes + 255) & ~size_t(255);
    size_t used = 0;
    for (auto& blk : scratch) {
        if (scratch_used < used + blk->n) {
            size_t off = scratch_used - used;
            if (off + bytes <= blk->n) {
                scratch_used += bytes;
                return blk->p + off;
            }
            // skip the rest of this block
            scratch_used = used + blk->n;
        }
        used += blk->n;
    }
    if (scratch_fixed) throw Error(LSJK_ENOMEM, "fixed scratch block exhausted");
    size_t sz = std::max(bytes, size_t(64) << 20);
    scratch.emplace_back(new DBuf<char>());
    scratch.back()->alloc(sz);
    scratch_used = used + bytes;
    return scratch.back()->p;
}

// Make the auxiliary streams wait for the work enqueued so far on ctx->stream.
inline void fork_aux(Context* ctx)
{
    LSJK_CUDA(cudaEventRecord(ctx->fork_ev, ctx->stream));
    for (int i = 0; i < Context::kAux; ++i) LSJK_CUDA(cudaStreamWaitEvent(ctx->aux[i], ctx->fork_ev, 0));
}

// Make ctx->stream wait for everything enqueued on the auxiliary streams.
inline void join_aux(Context* ctx)
{
    for (int i = 0; i < Context::kAux; ++i) {
        LSJK_CUDA(cudaEventRecord(ctx->join_ev[i], ctx->aux[i]));
        LSJK_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->join_ev[i], 0));
    }
}

// While alive, ctx->stream is auxiliary stream i (the launchers enqueue on
// ctx->stream); restores the main stream on exit.
struct OnAux {
    Context* ctx;
    cudaStream_t main;
    OnAux(Context* c, int i) : ctx(c), main(c->stream) { c->stream = c->aux[i % Context::kAux]; }
    ~OnAux() { ctx->stream = main; }
};

template <typename T>
inline T* take(Context* ctx, size_t n) { return reinterpret_cast<T*>(ctx->scratch_take(sizeof(T) * (n ? n : 1))); }

// Build steps (basis.cu, pairs.cu, jbuild.cu, kbuild.cu)
void basis_init(Context* ctx, Basis* B);
// Build B->twin (left null when B shares no exponent between shells).
void basis_build_twin(Context* ctx, Basis* B);
double j_quartet_flops(int LB, int LK);
double k_quartet_flops(int L1, int L2, int L3, int L4);
void build_pairlist(Context* ctx, PairList* pl);
void build_kinv(Context* ctx, PairList* pl);
void pure_to_cart(Context* ctx, const Basis* b1, const Basis* b2, const double* Dpure, double* Dcart);
// Screening density of twins u1 x u2 (u1/u2 may be plain bases) from the
// Cartesian density Dorig of the bases they stand for (leading dimension ld):
//   Dscr[a, b] = max over the copies (i of a, j of b) of |w_i w_j| |Dorig[i, j]|,
// an upper bound of every copy's |D| weighted as the reference's screens see
// it, so screens over twins keep every quartet the reference keeps.
void screen_density(Context* ctx, const Basis* u1, const Basis* u2, const double* Dorig, int ld, double* Dscr);
void cart_to_pure_acc(Context* ctx, const Basis* b1, const Basis* b2, const double* Xcart, double* Xpure);

struct Ewald {
    std::vector<double> alpha, omega;   // terms with alpha != 0 and omega != 0
};

// One-electron integrals over a pair list (oneint.cu), added into the device
// Cartesian matrix Xcart (ncart1 x ncart2): kind 0 overlap, 1 kinetic, 2 the
// nuclear potential of natom charges xyzc (x, y, z, Z) under the operator ew.
void one_electron(Context* ctx, int kind, const PairList* pl, const Ewald* ew, const double* xyzc, int natom,
                  double* Xcart);

// densities whose quartets one J thread or K lane evaluates together (one
// quadrature, several contractions)
constexpr int kJBatchMax = 4;
// densities per J or K build: one launch per class and pass serves all of them
// (K: groups of kJBatchMax densities share a task list; J: grid.z over groups)
constexpr int kMaxDens = 64;

// J for ng (1..4) densities at once; batched densities share the quartets
// (screened with the largest |D| of the batch).
void coulomb_build(Context* ctx, const Ewald& ew, const PairList* pl12, const PairList* pl34,
                   const double* const* Dcart, double* const* Jcart, int ng, float thresp, float thredp);
// J nuclear gradient (FP64): G[atom][xyz] += sum D12 d(12|34) D34 over a symmetric
// pair list, Cartesian densities in, device G (natom x 3) accumulated. `same`:
// D12 and D34 are the same matrix (one bra-derivative pass, doubled).
void coulomb_grad(Context* ctx, const Ewald& ew, const PairList* pl, const double* D12cart, const double* D34cart,
                  bool same, double* G, float thresp);
// K for ng (1..4) densities sharing one task list (screened with the largest
// |D24| of the batch) and the quartet integrals.
// Dscr: the densities the screens read (Dcart itself when null, or screening
// densities of the same layout when the pair lists are twins).
// Kcart is laid out in the Cartesian spaces of kb1 x kb3, the bases the
// partner primitives' output targets point into (pl12->b1 and pl34->b1
// themselves, or the bases they are the twins of).
void exchange_build(Context* ctx, const Ewald& ew, const PairList* pl12, const PairList* pl34,
                    const double* const* Dcart, const double* const* Dscr, double* const* Kcart, int ng,
                    bool d24symm, bool flip_ok, float thresp, float thredp, const Basis* kb1, const Basis* kb3);
// K nuclear gradient (FP64): G[atom][xyz] += sum D13 d(12|34)/dR D24 over the
// K-invert quartets of a symmetric pair list (K-invert rows built), Cartesian
// densities in, device G (natom x 3) accumulated. pairsym: D13 and D24 are both
// symmetric (each term computed once for itself and its mirror); canon: the
// quartet screen of the reference's fully symmetric routine (D13 == D24 symmetric).
void exchange_grad(Context* ctx, const Ewald& ew, const PairList* pl, const double* D13cart, const double* D24cart,
                   bool pairsym, bool canon, double* G, float thresp);

} // namespace lsjk
