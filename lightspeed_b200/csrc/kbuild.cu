// Exchange (K) build on the device: the reference's exchangeCPU
// (src/cpp/intbox/cpu/exchange.cpp:17-355) re-laid out for the B200.
//
// The reference loops over (prim2, prim4) pairs -- rows of its K-invert lists
// -- and inside over partners 1 of prim2 and 3 of prim4, both sorted by bound,
// breaking as soon as bound12 * bound34 * max|D24 block| < thresp
// (exchange.cpp:124-343). The computed quartet set is exactly
//   { (1,2,3,4) : bound12 >= thre12, bound34 >= thre34,
//                 double(float(bound12*bound34)) * Dmax(2,4) >= thresp },
// with prim2 <= prim4 and the transposed write when D24 is symmetric.
// Here:
//  1. one device pass over all (prim2, prim4) pairs drops those whose first
//     quartet already fails and appends the rest to per-class task lists;
//  2. one kernel per class (L1 L2|L3 L4): each warp takes (prim2, prim4) tasks
//     from a device work queue, keeps the D24 block in registers, walks the
//     partner rows (prim1 uniform across the warp, prim3 across lanes), runs
//     the Rys quadrature (tables staged in shared memory by a bulk copy) and
//     contracts with D24 in registers, then scatters the K13 block with FP64
//     atomics. No ERI is stored.
#include <algorithm>
#include <optional>
#include "engine.cuh"
#include "lsjk_device.cuh"
#include "kargs.cuh"

namespace lsjk {

namespace {


inline unsigned nblk(long n, int t) { return (unsigned) ((n + t - 1) / t); }

__host__ __device__ inline int combo_index(int L1, int L2, int L3, int L4) { return ((L1 * kNL + L2) * kNL + L3) * kNL + L4; }
constexpr int kNCombo = kNL * kNL * kNL * kNL;





// K = K + K^T in place (square ld x ld): the transposed half of the symmetric
// D24 contributions, which the class kernels do not write.
__global__ void k_symmetrize(double* __restrict__ K, int n)
{
    const long total = (long) n * n;
    for (long k = blockIdx.x * (long) blockDim.x + threadIdx.x; k < total; k += (long) gridDim.x * blockDim.x) {
        const int i = (int) (k / n), j = (int) (k % n);
        if (i > j) continue;
        if (i == j) {
            K[k] *= 2.0;
        } else {
            const double v = K[k] + K[(long) j * n + i];
            K[k] = v;
            K[(long) j * n + i] = v;
        }
    }
}

__global__ void k_absmax(const double* __restrict__ X, long n, unsigned long long* __restrict__ out)
{
    double m = 0.0;
    for (long k = blockIdx.x * (long) blockDim.x + threadIdx.x; k < n; k += (long) gridDim.x * blockDim.x)
        m = fmax(m, fabs(X[k]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long) __double_as_longlong(m));
}

// out[i * nprim + j] = max |D| over the Cartesian block of primitives (i, j).
__global__ void k_prim_blockmax(const double* __restrict__ D, int ld, BasisView b, double* __restrict__ out)
{
    const long k = blockIdx.x * (long) blockDim.x + threadIdx.x;
    if (k >= (long) b.nprim * b.nprim) return;
    const int i = (int) (k / b.nprim), j = (int) (k % b.nprim);
    const int ci = b.cart[i], cj = b.cart[j], ni = ncart_of(b.L[i]), nj = ncart_of(b.L[j]);
    double m = 0.0;
    for (int a = 0; a < ni; ++a)
        for (int c = 0; c < nj; ++c) m = fmax(m, fabs(D[(long) (ci + a) * ld + cj + c]));
    out[k] = m;
}

// thre12 = thresp / (max_bound(pl34) * D24max), thre34 likewise (exchange.cpp:54-71)
__global__ void k_kscalars(KScalars* S, float thresp, double maxb12, double maxb34)
{
    double d = __longlong_as_double((long long) S->dmax_bits);
    S->thre12 = (float) ((double) thresp / (maxb34 * d));
    S->thre34 = (float) ((double) thresp / (maxb12 * d));
}

struct KRowTables {
    const int* start[kNL][kNL];   // [L_indexed][L_partner]
    const int* len[kNL][kNL];
};

struct TaskGenArgs {
    BasisView b2, b4;
    KRowTables r12, r34;
    const float* pb12;
    const float* pb34;
    const double* Dc[kMaxDens];    // screening densities of the build; CTA z = group of kKBatch
    int ng;
    int ld4;
    int d24symm;
    float thresp;
    const KScalars* sc;
    KTask* tasks;                  // per-combo regions (all groups' tasks of a class in one region)
    long cap_off[kNCombo];         // region offsets (by value: graph-capturable)
    int* ntask;                    // per-combo counts
    // mixed precision: tasks whose first quartet reaches thredp, the only ones the FP64 pass can use
    KTask* tasks_hi;
    int* ntask_hi;
    float thredp;
    int split;
    int global_dmax;               // tasks carry the global max|D| (sc) instead of their block's
};

// Append one task per lane that wants one to the list of its class c: the
// lanes of the warp with the same class take consecutive slots from one
// atomic (the leader's), so the per-class counters see one atomic per warp
// and class instead of one per task.
__device__ __forceinline__ void append_task(unsigned want_mask, int c, long off, int* __restrict__ count,
                                            KTask* __restrict__ list, const KTask& t)
{
    const int lane = threadIdx.x & 31;
    const unsigned peers = __match_any_sync(want_mask, c);
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(&count[c], __popc(peers));
    base = __shfl_sync(peers, base, leader);
    list[off + base + __popc(peers & ((1u << lane) - 1u))] = t;
}

__global__ void k_task_gen(TaskGenArgs A)
{
    const int i2 = blockIdx.x;
    const int i4 = blockIdx.y * blockDim.x + threadIdx.x;
    const int grp = blockIdx.z;   // densities grp * kKBatch .. + kKBatch - 1
    const int g0 = grp * kKBatch, g1 = min(A.ng, g0 + kKBatch);
    // exchange.cpp:137-139 (prim2 <= prim4 for a symmetric D24); lanes out of
    // range stay for the warp-wide votes below
    const bool valid = i4 < A.b4.nprim && !(A.d24symm && i2 > i4);
    if (!__any_sync(0xffffffffu, valid)) return;
    const float thre12 = A.sc->thre12, thre34 = A.sc->thre34;
    const int L2 = A.b2.L[i2];
    const int L4 = valid ? A.b4.L[i4] : 0;
    // largest |D24| over the pair's block and the batch's densities
    double dmax = 0.0;
    if (A.global_dmax) {
        dmax = __longlong_as_double((long long) A.sc->dmax_bits);
    } else if (valid) {
        const int c2 = A.b2.cart[i2], c4 = A.b4.cart[i4];
        const int n2 = ncart_of(L2), n4 = ncart_of(L4);
        for (int g = g0; g < g1; ++g)
            for (int a = 0; a < n2; ++a)
                for (int b = 0; b < n4; ++b) dmax = fmax(dmax, fabs(A.Dc[g][(long) (c2 + a) * A.ld4 + c4 + b]));
    }
    for (int L1 = 0; L1 < kNL; ++L1) {
        const int* rl12 = A.r12.len[L2][L1];
        // uniform over the block (i2 and L2 are)
        if (!rl12) continue;
        const int len12 = rl12[i2];
        if (!len12) continue;
        const float b12 = A.pb12[A.r12.start[L2][L1][i2]];
        if (b12 < thre12) continue;
        for (int L3 = 0; L3 < kNL; ++L3) {
            bool want = false;
            float b34 = 0.0f;
            if (valid) {
                const int* rl34 = A.r34.len[L4][L3];
                if (rl34 && rl34[i4]) {
                    b34 = A.pb34[A.r34.start[L4][L3][i4]];
                    want = b34 >= thre34 && (double) (b12 * b34) * dmax >= (double) A.thresp;
                }
            }
            const int c = combo_index(L1, L2, L3, L4);
            const KTask t{i2, (unsigned short) i4, (unsigned short) grp, dmax};
            const unsigned wm = __ballot_sync(0xffffffffu, want);
            if (want) append_task(wm, c, A.cap_off[c], A.ntask, A.tasks, t);
            const bool hi = want && A.split && (double) (b12 * b34) * dmax >= (double) A.thredp;
            const unsigned hm = __ballot_sync(0xffffffffu, hi);
            if (hi) append_task(hm, c, A.cap_off[c], A.ntask_hi, A.tasks_hi, t);
        }
    }
}

// Runtime (L1,L2,L3,L4) -> template dispatch.
template <int L1, int L2, int L3>
void launch_k4(Context* ctx, const KArgs& A, long cap, int L4, bool fp32)
{
    switch (L4) {
    case 0: launch_k<L1, L2, L3, 0>(ctx, A, cap, fp32); break;
    case 1: launch_k<L1, L2, L3, 1>(ctx, A, cap, fp32); break;
    case 2: launch_k<L1, L2, L3, 2>(ctx, A, cap, fp32); break;
    case 3: launch_k<L1, L2, L3, 3>(ctx, A, cap, fp32); break;
    default: throw Error(LSJK_ENOTSUPP, "K: shell above f");
    }
}
template <int L1, int L2>
void launch_k3(Context* ctx, const KArgs& A, long cap, int L3, int L4, bool fp32)
{
    switch (L3) {
    case 0: launch_k4<L1, L2, 0>(ctx, A, cap, L4, fp32); break;
    case 1: launch_k4<L1, L2, 1>(ctx, A, cap, L4, fp32); break;
    case 2: launch_k4<L1, L2, 2>(ctx, A, cap, L4, fp32); break;
    case 3: launch_k4<L1, L2, 3>(ctx, A, cap, L4, fp32); break;
    default: throw Error(LSJK_ENOTSUPP, "K: shell above f");
    }
}
template <int L1>
void launch_k2(Context* ctx, const KArgs& A, long cap, int L2, int L3, int L4, bool fp32)
{
    switch (L2) {
    case 0: launch_k3<L1, 0>(ctx, A, cap, L3, L4, fp32); break;
    case 1: launch_k3<L1, 1>(ctx, A, cap, L3, L4, fp32); break;
    case 2: launch_k3<L1, 2>(ctx, A, cap, L3, L4, fp32); break;
    case 3: launch_k3<L1, 3>(ctx, A, cap, L3, L4, fp32); break;
    default: throw Error(LSJK_ENOTSUPP, "K: shell above f");
    }
}
void launch_k1(Context* ctx, const KArgs& A, long cap, int L1, int L2, int L3, int L4, bool fp32)
{
    switch (L1) {
    case 0: launch_k2<0>(ctx, A, cap, L2, L3, L4, fp32); break;
    case 1: launch_k2<1>(ctx, A, cap, L2, L3, L4, fp32); break;
    case 2: launch_k2<2>(ctx, A, cap, L2, L3, L4, fp32); break;
    case 3: launch_k2<3>(ctx, A, cap, L2, L3, L4, fp32); break;
    default: throw Error(LSJK_ENOTSUPP, "K: shell above f");
    }
}

} // namespace

// Algorithmic flops of one K quartet of class (L1 L2|L3 L4) for one Ewald
// term: geometry/prefactor 40, per root 16 (Rys tables) + 12 (recursion
// coefficients) + 3 flops per 1-D integral entry over the three directions,
// and 4 flops per (a,b,c,d) component product-and-contract.
double k_quartet_flops(int L1, int L2, int L3, int L4)
{
    int nr = (L1 + L2 + L3 + L4) / 2 + 1;
    double n1d = 3.0 * (L1 + L2 + 1) * (L3 + L4 + 1) + 3.0 * (L1 + 1) * (L2 + 1) * (L3 + 1) * (L4 + 1);
    double nc = (double) ncart_of(L1) * ncart_of(L2) * ncart_of(L3) * ncart_of(L4);
    return 40.0 + nr * (28.0 + 2.0 * n1d + 4.0 * nc);
}

void exchange_build(Context* ctx, const Ewald& ew, const PairList* pl12, const PairList* pl34,
                    const double* const* Dcart, const double* const* Dscr_in, double* const* Kcart, int ng,
                    bool d24symm, bool flip_ok, float thresp, float thredp, const Basis* kb1, const Basis* kb3)
{
    // screens read Dscr (max|D24| estimates); the integrals contract with Dcart
    const double* const* Dscr = Dscr_in ? Dscr_in : Dcart;
    if (ng < 1 || ng > kMaxDens) throw Error(LSJK_EINVAL, "exchange_build: 1..64 densities per build");
    const int ngroup = (ng + kKBatch - 1) / kKBatch;
    cudaStream_t s = ctx->stream;
    const int b1c = kb1->ncart;   // K13 lives in the output spaces of bases 1 and 3
    const Basis *b2 = pl12->b2, *b3 = kb3, *b4 = pl34->b2;
    // global max |D24| (exchange.cpp:48-52) and the K-invert thresholds
    KScalars* sc = take<KScalars>(ctx, 1);
    LSJK_CUDA(cudaMemsetAsync(sc, 0, sizeof(KScalars), s));
    long nd = (long) pl12->b2->ncart * b4->ncart;
    for (int g = 0; g < ng && nd; ++g) {
        k_absmax<<<std::min<long>(nblk(nd, 256), 1184), 256, 0, s>>>(Dscr[g], nd, &sc->dmax_bits);
        ctx->stats.kernel_launches++;
    }
    k_kscalars<<<1, 1, 0, s>>>(sc, thresp, pl12->max_bound, pl34->max_bound);
    LSJK_CUDA(cudaGetLastError());
    ctx->stats.kernel_launches++;

    // per-combo task regions: capacity = prims of L2 in basis2 x prims of L4 in basis4,
    // none where basis 1 has no partner of L1 or basis 3 none of L3 (no task can name it)
    int cnt1[kNL] = {0}, cnt2[kNL] = {0}, cnt3[kNL] = {0}, cnt4[kNL] = {0};
    for (int L : pl12->b1->L) cnt1[L]++;
    for (int L : b2->L) cnt2[L]++;
    for (int L : pl34->b1->L) cnt3[L]++;
    for (int L : b4->L) cnt4[L]++;
    std::vector<long> off(kNCombo + 1, 0);
    for (int L1 = 0; L1 < kNL; ++L1)
        for (int L2 = 0; L2 < kNL; ++L2)
            for (int L3 = 0; L3 < kNL; ++L3)
                for (int L4 = 0; L4 < kNL; ++L4) {
                    int c = combo_index(L1, L2, L3, L4);
                    off[c + 1] = (cnt1[L1] && cnt3[L3]) ? (long) cnt2[L2] * cnt4[L4] * ngroup : 0L;
                }
    for (int c = 0; c < kNCombo; ++c) off[c + 1] += off[c];
    const bool mixed = ctx->precision == LSJK_PREC_MIXED && thredp > thresp;
    KTask* tasks = take<KTask>(ctx, off[kNCombo]);
    int* ntask = take<int>(ctx, 2 * kNCombo);   // all tasks, then the FP64-pass tasks
    KTask* tasks_hi = mixed ? take<KTask>(ctx, off[kNCombo]) : nullptr;
    unsigned* queue = take<unsigned>(ctx, 2 * kNCombo);   // per class and pass (one launch each)
    unsigned long long* qcnt = ctx->counters.p + kNJClass;                          // FP64 K classes
    unsigned long long* qcnt32 = ctx->counters.p + kNJClass + kNKClass + kNJClass;  // FP32 K classes
    LSJK_CUDA(cudaMemsetAsync(ntask, 0, sizeof(int) * 2 * kNCombo, s));
    LSJK_CUDA(cudaMemsetAsync(queue, 0, sizeof(unsigned) * 2 * kNCombo, s));

    TaskGenArgs G{};
    G.b2 = b2->view();
    G.b4 = b4->view();
    for (int a = 0; a < kNL; ++a)
        for (int b = 0; b < kNL; ++b) {
            G.r12.start[a][b] = pl12->kinv[a][b].row_start.p;
            G.r12.len[a][b] = pl12->kinv[a][b].row_len.p;
            G.r34.start[a][b] = pl34->kinv[a][b].row_start.p;
            G.r34.len[a][b] = pl34->kinv[a][b].row_len.p;
        }
    G.pb12 = pl12->kdat.pbound.p;
    G.pb34 = pl34->kdat.pbound.p;
    for (int g = 0; g < ng; ++g) G.Dc[g] = Dscr[g];
    G.ng = ng;
    G.ld4 = b4->ncart;
    G.d24symm = d24symm ? 1 : 0;
    G.thresp = thresp;
    G.sc = sc;
    G.tasks = tasks;
    for (int c = 0; c < kNCombo; ++c) G.cap_off[c] = off[c];
    G.ntask = ntask;
    G.tasks_hi = tasks_hi;
    G.ntask_hi = ntask + kNCombo;
    G.thredp = thredp;
    G.split = mixed ? 1 : 0;
    if (b2->nprim && b4->nprim && pl12->kdat.nent && pl34->kdat.nent) {
        // prim2 varies fastest over the blocks, so the lists interleave prim2 rows: warps taking
        // neighbouring tasks then mostly add into different K13 rows
        dim3 grid(b2->nprim, nblk(b4->nprim, 128), ngroup);
        k_task_gen<<<grid, 128, 0, s>>>(G);
        LSJK_CUDA(cudaGetLastError());
        ctx->stats.kernel_launches++;
    } else {
        return;
    }

    // class kernels go round-robin to the auxiliary streams (not while the
    // autotuner times them one by one)
    const bool par = !ctx->tuning;
    if (par) fork_aux(ctx);
    int lane = 0;
    for (int L1 = 0; L1 < kNL; ++L1)
        for (int L2 = 0; L2 < kNL; ++L2)
            for (int L3 = 0; L3 < kNL; ++L3)
                for (int L4 = 0; L4 < kNL; ++L4) {
                    int c = combo_index(L1, L2, L3, L4);
                    long cap = off[c + 1] - off[c];
                    if (!cap) continue;
                    if (!pl12->kinv[L2][L1].row_len.p || !pl34->kinv[L4][L3].row_len.p) continue;
                    int NR = (L1 + L2 + L3 + L4) / 2 + 1;
                    KArgs A{};
                    A.tasks = tasks + off[c];
                    A.ntask = ntask + c;
                    A.r12s = pl12->kinv[L2][L1].row_start.p;
                    A.r12l = pl12->kinv[L2][L1].row_len.p;
                    A.r34s = pl34->kinv[L4][L3].row_start.p;
                    A.r34l = pl34->kinv[L4][L3].row_len.p;
                    const KInvData& d12 = pl12->kdat;     // partner 1: shell segments
                    const KInvData& d34 = pl34->kdat_b;   // partner 3: by bound
                    A.d12 = KRows<double>{d12.kab.p, d12.p.p, d12.ip.p, d12.px.p, d12.py.p, d12.pz.p,
                                          d12.ax.p, d12.ay.p, d12.az.p, d12.pw0.p, d12.pw1.p};
                    A.d34 = KRows<double>{d34.kab.p, d34.p.p, d34.ip.p, d34.px.p, d34.py.p, d34.pz.p,
                                          d34.ax.p, d34.ay.p, d34.az.p, d34.pw0.p, d34.pw1.p};
                    A.f12 = KRows<float>{d12.kab32.p, d12.p32.p, d12.ip32.p, d12.px32.p, d12.py32.p,
                                         d12.pz32.p, d12.ax32.p, d12.ay32.p, d12.az32.p, d12.pw0_32.p,
                                         d12.pw1_32.p};
                    A.f34 = KRows<float>{d34.kab32.p, d34.p32.p, d34.ip32.p, d34.px32.p, d34.py32.p,
                                         d34.pz32.p, d34.ax32.p, d34.ay32.p, d34.az32.p, d34.pw0_32.p,
                                         d34.pw1_32.p};
                    A.cart12 = d12.pcart.p;
                    A.t1_12 = d12.pt1.p;
                    A.seg12 = d12.pseg.p;
                    A.b12 = d12.pbound.p;
                    A.cart34 = d34.pcart.p;
                    A.t1_34 = d34.pt1.p;
                    A.w0_34 = d34.pw0.p;
                    A.w1_34 = d34.pw1.p;
                    A.b34 = d34.pbound.p;
                    A.b2 = b2->view();
                    A.b4 = b4->view();
                    for (int g = 0; g < ng; ++g) {
                        A.Dc[g] = Dcart[g];
                        A.Kc[g] = Kcart[g];
                    }
                    A.ng = ng;
                    A.ld4 = b4->ncart;
                    A.ld3 = b3->ncart;
                    A.flip = flip_ok ? 1 : 0;
                    A.gc = (pl12->b1->is_twin || pl34->b1->is_twin) ? 1 : 0;
                    A.sc = sc;
                    A.nbin = kRysNbin[NR];
                    A.tmax = kRysTmax[NR];
                    A.status = ctx->status.p;
                    A.nterm = (int) ew.alpha.size();
                    for (int t = 0; t < A.nterm; ++t) {
                        A.alpha[t] = ew.alpha[t];
                        A.omega[t] = ew.omega[t];
                    }
                    const float inf = __builtin_huge_valf();
                    // classes above the straight-line quartet code (an f shell) run in FP64 only:
                    // one pass over all tasks (their FP32 loop form is no faster than FP64)
                    const bool two_pass = mixed && std::max(std::max(L1, L2), std::max(L3, L4)) <= kGenLmax;
                    // FP64 pass: estimate >= thredp (mixed) or >= thresp (FP64 mode)
                    A.queue = queue + c;
                    if (two_pass) {
                        // FP64 pass: only the tasks that can reach thredp
                        A.tasks = tasks_hi + off[c];
                        A.ntask = ntask + kNCombo + c;
                    }
                    A.thr_lo = two_pass ? thredp : thresp;
                    A.thr_hi = inf;
                    A.split_hi = two_pass ? 1 : 0;
                    A.rys = ctx->rys64.p + kRysOffset[NR];
                    A.asym_t = ctx->rys_asym64.p + NR * LSJK_RYS_NMAX;
                    A.asym_w = ctx->rys_asym64.p + (LSJK_RYS_NMAX + 1) * LSJK_RYS_NMAX + NR * LSJK_RYS_NMAX;
                    A.rys64g = ctx->rys64.p + kRysOffset[NR];
                    A.asym64_t = ctx->rys_asym64.p + NR * LSJK_RYS_NMAX;
                    A.asym64_w = ctx->rys_asym64.p + (LSJK_RYS_NMAX + 1) * LSJK_RYS_NMAX + NR * LSJK_RYS_NMAX;
                    A.qcount = qcnt + c;
                    auto tune = [&](const KArgs& X, bool fp32) {
                        // autotuner: time candidate grid sizes on scratch outputs
                        static const int cand[] = {2, 4, 8, 16, 32};
                        KArgs T = X;
                        for (int g = 0; g < X.ng; ++g) T.Kc[g] = take<double>(ctx, (size_t) b1c * b3->ncart);
                        T.qcount = ctx->tune_sink.p;
                        int& slot = ctx->tune.k_ctas_per_sm[fp32 ? 1 : 0][L1][L2][L3][L4];
                        float best = 1e30f;
                        int bestc = 16;
                        for (int cnd : cand) {
                            slot = cnd;
                            float ms = 1e30f;
                            for (int rep = 0; rep < 2; ++rep) {
                                LSJK_CUDA(cudaMemsetAsync(T.queue, 0, sizeof(unsigned), s));
                                LSJK_CUDA(cudaEventRecord(ctx->ev0, s));
                                launch_k1(ctx, T, cap, L1, L2, L3, L4, fp32);
                                LSJK_CUDA(cudaEventRecord(ctx->ev1, s));
                                LSJK_CUDA(cudaEventSynchronize(ctx->ev1));
                                float t = 0.f;
                                LSJK_CUDA(cudaEventElapsedTime(&t, ctx->ev0, ctx->ev1));
                                ms = std::min(ms, t);
                            }
                            if (ms < best) {
                                best = ms;
                                bestc = cnd;
                            }
                        }
                        slot = bestc;
                        LSJK_CUDA(cudaMemsetAsync(X.queue, 0, sizeof(unsigned), s));
                    };
                    if (ctx->tuning) tune(A, false);
                    {
                        std::optional<OnAux> on;
                        if (par) on.emplace(ctx, lane++);
                        launch_k1(ctx, A, cap, L1, L2, L3, L4, false);
                    }
                    if (two_pass) {
                        // FP32 pass: thresp <= estimate < thredp, over all tasks
                        A.tasks = tasks + off[c];
                        A.ntask = ntask + c;
                        A.queue = queue + kNCombo + c;
                        A.thr_lo = thresp;
                        A.thr_hi = thredp;
                        A.split_hi = 0;
                        A.rys = ctx->rys32.p + kRysOffset[NR];
                        A.asym_t = ctx->rys_asym32.p + NR * LSJK_RYS_NMAX;
                        A.asym_w = ctx->rys_asym32.p + (LSJK_RYS_NMAX + 1) * LSJK_RYS_NMAX + NR * LSJK_RYS_NMAX;
                        A.qcount = qcnt32 + c;
                        if (ctx->tuning) tune(A, true);
                        std::optional<OnAux> on;
                        if (par) on.emplace(ctx, lane++);
                        launch_k1(ctx, A, cap, L1, L2, L3, L4, true);
                    }
                }
    if (par) join_aux(ctx);
    if (flip_ok) {
        // basis 1 == basis 3 here, so each K13 is square
        const int n = b3->ncart;
        for (int g = 0; g < ng; ++g) {
            k_symmetrize<<<std::min<long>(nblk((long) n * n, 256), 1184), 256, 0, s>>>(Kcart[g], n);
            LSJK_CUDA(cudaGetLastError());
            ctx->stats.kernel_launches++;
        }
    }
}

// The K gradient over the K build's quartet set (exchange_grad.cpp:523-760:
// bound12 >= thre12, bound34 >= thre34, bound12 bound34 max|D24 block| >=
// thresp), every (prim2, prim4) pair and every partner pair -- the D13/D24
// symmetry flags of the reference's general routine only choose which equal
// terms it skips and doubles, so the sum is the same without them. `canon`:
// the reference's fully symmetric routine (D13symm, D24symm and Dsame;
// exchange_grad.cpp:17-470), which computes one representative per set of
// equal terms and screens all of them with the representative's D block;
// the same sum over the same quartets here. `pairsym` (D13 and D24 both
// symmetric, the reference's D13symm and D24symm): the terms of (1,2,3,4) and
// (3,4,1,2) are equal, screens included, so only tasks with prim2 <= prim4 run
// and those with prim2 < prim4 count twice.
void exchange_grad(Context* ctx, const Ewald& ew, const PairList* pl, const double* D13cart, const double* D24cart,
                   bool pairsym, bool canon, double* G, float thresp)
{
    if (ew.alpha.size() > 4) throw Error(LSJK_EINVAL, "exchange_grad: at most 4 Ewald terms");
    cudaStream_t s = ctx->stream;
    const Basis* b = pl->b1;
    if (!b->nprim || !pl->kdat.nent) return;
    KScalars* sc = take<KScalars>(ctx, 1);
    LSJK_CUDA(cudaMemsetAsync(sc, 0, sizeof(KScalars), s));
    const long nd = (long) b->ncart * b->ncart;
    k_absmax<<<std::min<long>(nblk(nd, 256), 1184), 256, 0, s>>>(D24cart, nd, &sc->dmax_bits);
    k_kscalars<<<1, 1, 0, s>>>(sc, thresp, pl->max_bound, pl->max_bound);
    LSJK_CUDA(cudaGetLastError());
    ctx->stats.kernel_launches += 2;

    int cnt[kNL] = {0};
    for (int L : b->L) cnt[L]++;
    std::vector<long> off(kNCombo + 1, 0);
    for (int L1 = 0; L1 < kNL; ++L1)
        for (int L2 = 0; L2 < kNL; ++L2)
            for (int L3 = 0; L3 < kNL; ++L3)
                for (int L4 = 0; L4 < kNL; ++L4)
                    off[combo_index(L1, L2, L3, L4) + 1] = (cnt[L1] && cnt[L3]) ? (long) cnt[L2] * cnt[L4] : 0L;
    for (int c = 0; c < kNCombo; ++c) off[c + 1] += off[c];
    KTask* tasks = take<KTask>(ctx, off[kNCombo]);
    int* ntask = take<int>(ctx, kNCombo);
    unsigned* queue = take<unsigned>(ctx, kNCombo);
    LSJK_CUDA(cudaMemsetAsync(ntask, 0, sizeof(int) * kNCombo, s));
    LSJK_CUDA(cudaMemsetAsync(queue, 0, sizeof(unsigned) * kNCombo, s));

    TaskGenArgs T{};
    T.b2 = b->view();
    T.b4 = b->view();
    for (int a = 0; a < kNL; ++a)
        for (int c = 0; c < kNL; ++c) {
            T.r12.start[a][c] = T.r34.start[a][c] = pl->kinv[a][c].row_start.p;
            T.r12.len[a][c] = T.r34.len[a][c] = pl->kinv[a][c].row_len.p;
        }
    T.pb12 = T.pb34 = pl->kdat_b.pbound.p;
    T.Dc[0] = D24cart;
    T.ng = 1;
    T.ld4 = b->ncart;
    T.d24symm = pairsym ? 1 : 0;   // prim2 <= prim4 when each task also stands for its mirror
    T.thresp = thresp;
    T.sc = sc;
    T.tasks = tasks;
    for (int c = 0; c < kNCombo; ++c) T.cap_off[c] = off[c];
    T.ntask = ntask;
    T.global_dmax = canon ? 1 : 0;
    double* dblk = nullptr;
    if (canon) {
        const long np2 = (long) b->nprim * b->nprim;
        dblk = take<double>(ctx, np2);
        k_prim_blockmax<<<nblk(np2, 256), 256, 0, s>>>(D24cart, b->ncart, b->view(), dblk);
        LSJK_CUDA(cudaGetLastError());
        ctx->stats.kernel_launches++;
    }
    dim3 grid(b->nprim, nblk(b->nprim, 128));
    k_task_gen<<<grid, 128, 0, s>>>(T);
    LSJK_CUDA(cudaGetLastError());
    ctx->stats.kernel_launches++;

    const KInvData& d = pl->kdat_b;   // partners 1 and 3 both in bound order
    for (int L1 = 0; L1 < kNL; ++L1)
        for (int L2 = 0; L2 < kNL; ++L2)
            for (int L3 = 0; L3 < kNL; ++L3)
                for (int L4 = 0; L4 < kNL; ++L4) {
                    const int c = combo_index(L1, L2, L3, L4);
                    const long cap = off[c + 1] - off[c];
                    if (!cap || !pl->kinv[L2][L1].row_len.p || !pl->kinv[L4][L3].row_len.p) continue;
                    const int NR = (L1 + L2 + L3 + L4 + 1) / 2 + 1;   // one quantum up
                    KGradArgs A{};
                    A.tasks = tasks + off[c];
                    A.ntask = ntask + c;
                    A.queue = queue + c;
                    A.r12s = pl->kinv[L2][L1].row_start.p;
                    A.r12l = pl->kinv[L2][L1].row_len.p;
                    A.r34s = pl->kinv[L4][L3].row_start.p;
                    A.r34l = pl->kinv[L4][L3].row_len.p;
                    A.b12 = A.b34 = d.pbound.p;
                    A.kab12 = A.kab34 = d.kab.p;
                    A.p12 = A.p34 = d.p.p;
                    A.ip12 = A.ip34 = d.ip.p;
                    A.px12 = A.px34 = d.px.p;
                    A.py12 = A.py34 = d.py.p;
                    A.pz12 = A.pz34 = d.pz.p;
                    A.ax12 = A.ax34 = d.ax.p;
                    A.ay12 = A.ay34 = d.ay.p;
                    A.az12 = A.az34 = d.az.p;
                    A.pe12 = A.pe34 = d.pe.p;
                    A.cart12 = A.cart34 = d.pcart.p;
                    A.atom12 = A.atom34 = d.patom.p;
                    A.pidx12 = A.pidx34 = d.pidx.p;
                    A.dblk = dblk;
                    A.nprim = b->nprim;
                    A.canon = canon ? 1 : 0;
                    A.pairsym = pairsym ? 1 : 0;
                    A.b2 = A.b4 = b->view();
                    A.D13 = D13cart;
                    A.ld13 = b->ncart;
                    A.D24 = D24cart;
                    A.ld24 = b->ncart;
                    A.G = G;
                    A.sc = sc;
                    A.thr_lo = thresp;
                    A.rys = ctx->rys64.p + kRysOffset[NR];
                    A.asym_t = ctx->rys_asym64.p + NR * LSJK_RYS_NMAX;
                    A.asym_w = ctx->rys_asym64.p + (LSJK_RYS_NMAX + 1) * LSJK_RYS_NMAX + NR * LSJK_RYS_NMAX;
                    A.nbin = kRysNbin[NR];
                    A.tmax = kRysTmax[NR];
                    A.nterm = (int) ew.alpha.size();
                    for (int t = 0; t < A.nterm; ++t) {
                        A.alpha[t] = ew.alpha[t];
                        A.omega[t] = ew.omega[t];
                    }
                    launch_k_grad(ctx, A, cap, L1, L2, L3, L4);
                }
}

} // namespace lsjk
