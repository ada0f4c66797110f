// Coulomb (J) build on the device: the reference's coulombCPU pipeline
// (src/cpp/intbox/cpu/coulomb.cpp:14-196) re-laid out for the B200.
//
//  1. ket screening: B34' = B34 * max|D_cart block| (truncate_ket,
//     src/cpp/core/pair_list_util.cpp:60-123), kept if > thresp/max12, and a
//     radix sort by B34' descending per Hermite class L3+L4;
//  2. bra truncation: bound >= thresp/max34 (truncate_bra, :32-59) -- a
//     binary search on the bound-sorted bra list, on the device;
//  3. ket Hermite densities D_u = (-1)^|u| K_cd/q sum_cd E^cd_u D'_cd
//     (cart_to_herm with phases, src/cpp/core/hermite.cpp:9-206);
//  4. the J kernel per Hermite class pair (LB|LK): one thread per bra pair,
//     ket pairs streamed in bound order by the whole CTA, quartets kept iff
//     B12 * B34' >= thresp (coulomb.cpp:113-115), Boys table staged in shared
//     memory by a bulk (TMA) copy, Hermite integrals + density contraction in
//     registers, FP64 accumulation; no ERI is stored;
//  5. bra Hermite -> Cartesian (herm_to_cart, hermite.cpp:207-411) with the
//     symmetric-list double write and 1/2 on diagonal primitive pairs.
#include <algorithm>
#include <cub/device/device_radix_sort.cuh>
#include <optional>
#include <type_traits>
#include "engine.cuh"
#include "hermite.cuh"
#include "jargs.cuh"
#include "lsjk_device.cuh"

namespace lsjk {

namespace {

constexpr double kTwoPi52 = 34.986836655249725693;   // 2 pi^(5/2)

inline unsigned nblk(long n, int t) { return (unsigned) ((n + t - 1) / t); }

// ---- 1. ket screening -------------------------------------------------------

// The densities of one build (1..kMaxDens), passed by value.
struct DSet {
    const double* d[kMaxDens];
    int n;       // densities present
    int slots;   // record slots (= n)
};

__global__ void k_ket_screen(const int* __restrict__ p1, const int* __restrict__ p2,
                             const float* __restrict__ bound, int n, BasisView b3, BasisView b4,
                             int symm, DSet D, float thre,
                             unsigned* __restrict__ key, int* __restrict__ val,
                             int* __restrict__ nkept, unsigned* __restrict__ maxbits)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int i = p1[k], j = p2[k];
    int a1 = b3.cart[i], a2 = b4.cart[j];
    int c1 = ncart_of(b3.L[i]), c2 = ncart_of(b4.L[j]);
    int ld = b4.ncart;
    // max |D| over the pair block (both triangles if symmetric) and, for a
    // batched launch, over its densities: the batch screens with the union
    double v = 0.0;
    for (int g = 0; g < D.n; ++g) {
        const double* Dc = D.d[g];
        for (int x = 0; x < c1; ++x)
            for (int y = 0; y < c2; ++y) v = fmax(v, fabs(Dc[(long) (a1 + x) * ld + a2 + y]));
        if (symm)
            for (int x = 0; x < c1; ++x)
                for (int y = 0; y < c2; ++y) v = fmax(v, fabs(Dc[(long) (a2 + y) * ld + a1 + x]));
    }
    float B2 = (float) (v * (double) bound[k]);
    bool keep = B2 > thre;
    key[k] = keep ? ~__float_as_uint(B2) : 0xffffffffu;
    val[k] = k;
    if (keep) {
        atomicAdd(nkept, 1);
        atomicMax(maxbits, __float_as_uint(B2));
    }
}

// Bra class tables passed by value (no host->device copy, so a build can be
// captured in a CUDA graph).
struct BraTables {
    const float* bound[kNHerm];
    int n[kNHerm];
};

// thre_bra = thresp / max34 (float), then count bra pairs with bound >= thre_bra.
__global__ void k_bra_count(const unsigned* __restrict__ maxbits, float thresp, BraTables T,
                            int* __restrict__ nbra)
{
    int c = threadIdx.x;
    if (c >= kNHerm) return;
    unsigned mb = 0;
    for (int k = 0; k < kNHerm; ++k) mb = max(mb, maxbits[k]);
    float max34 = __uint_as_float(mb);
    float thre = (float) ((double) thresp / (double) max34);   // inf when max34 == 0
    int n = T.n[c];
    const float* b = T.bound[c];
    int lo = 0, hi = n;                 // first index with b < thre
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (b[mid] >= thre) lo = mid + 1; else hi = mid;
    }
    nbra[c] = lo;
}

// The (L1, LB - L1) split of a pair of Hermite class LB whose first shell has
// angular momentum l1, as a compile-time constant: calls f(integral_constant<L1>)
// for the one split with L1 == l1 (shells up to kLmax on either side).
template <int LB, int L1 = (LB > kLmax ? LB - kLmax : 0), typename F>
__device__ __forceinline__ void with_split(int l1, F&& f)
{
    if constexpr (L1 < kLmax && L1 < LB) {
        if (l1 == L1)
            f(std::integral_constant<int, L1>{});
        else
            with_split<LB, L1 + 1>(l1, f);
    } else {
        f(std::integral_constant<int, L1>{});
    }
}

// ---- 3. ket Hermite densities -------------------------------------------------

// Hermite expansion of one pair block of one density: out[t] for t < H.
// Kept out of line so the (runtime) loop over the densities of a batch wraps
// a call instead of the fully unrolled expansion.
template <int L3, int L4>
__device__ __noinline__ void ket_herm_block(const ECoef<L3, L4>& E, const double* __restrict__ Dc, int a1, int a2,
                                            int ld, bool symm, double scale, double pre, double* __restrict__ out)
{
    constexpr int N3 = ncart_of(L3), N4 = ncart_of(L4), H = nherm_of(L3 + L4);
    double Dp[N3][N4];
#pragma unroll
    for (int x = 0; x < N3; ++x)
#pragma unroll
        for (int y = 0; y < N4; ++y) {
            double v = Dc[(long) (a1 + x) * ld + a2 + y];
            if (symm) v += Dc[(long) (a2 + y) * ld + a1 + x];
            Dp[x][y] = v * scale;
        }
#pragma unroll
    for (int t = 0; t < H; ++t) {
        const int tx = herm_tx(t), ty = herm_ty(t), tz = herm_tz(t);
        double s = 0.0;
#pragma unroll
        for (int x = 0; x < N3; ++x)
#pragma unroll
            for (int y = 0; y < N4; ++y) {
                s += E.v[0][cart_lx(L3, x)][cart_lx(L4, y)][tx] * E.v[1][cart_ly(L3, x)][cart_ly(L4, y)][ty] *
                     E.v[2][cart_lz(L3, x)][cart_lz(L4, y)][tz] * Dp[x][y];
            }
        out[t] = ((tx + ty + tz) & 1 ? -pre : pre) * s;
    }
}

template <int L3, int L4>
__device__ void ket_record(int i, int j, BasisView b3, BasisView b4, bool symm, const DSet& DS,
                           const double* __restrict__ geom, double* __restrict__ rec)
{
    constexpr int H = nherm_of(L3 + L4);
    const double q = geom[0];
    const double Q[3] = {geom[1], geom[2], geom[3]};
    const double A[3] = {b3.x[i], b3.y[i], b3.z[i]};
    const double B[3] = {b4.x[j], b4.y[j], b4.z[j]};
    double QA[3], QB[3];
    double R2 = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        QA[d] = Q[d] - A[d];
        QB[d] = Q[d] - B[d];
        R2 += (A[d] - B[d]) * (A[d] - B[d]);
    }
    const double e1 = b3.e[i], e2 = b4.e[j];
    const double Kab = b3.c[i] * b4.c[j] * exp(-e1 * e2 / q * R2);
    ECoef<L3, L4> E;
    build_E<L3, L4>(q, QA, QB, E);
    const int a1 = b3.cart[i], a2 = b4.cart[j], ld = b4.ncart;
    const double scale = (symm && i == j) ? 0.5 : 1.0;
    const double pre = Kab / q;
    rec[0] = q;
    rec[1] = Q[0];
    rec[2] = Q[1];
    rec[3] = Q[2];
#pragma unroll 1
    for (int g = 0; g < DS.slots; ++g) {
        double* out = rec + 4 + g * H;
        if (g < DS.n)
            ket_herm_block<L3, L4>(E, DS.d[g], a1, a2, ld, symm, scale, pre, out);
        else
            for (int t = 0; t < H; ++t) out[t] = 0.0;   // unused slot of a partial batch
    }
}

template <int LK>
__global__ void k_ket_herm(const int* __restrict__ perm, const int* __restrict__ nkept,
                           const int* __restrict__ p1, const int* __restrict__ p2,
                           const float* __restrict__ bound, const double* __restrict__ geom,
                           BasisView b3, BasisView b4, int symm, DSet Dc,
                           double* __restrict__ rec, float* __restrict__ rec32)
{
    const int S = 4 + Dc.slots * nherm_of(LK);
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= *nkept) return;
    int src = perm[k];
    int i = p1[src], j = p2[src];
    int L3 = b3.L[i], L4 = b4.L[j];
    double* r = rec + (long) k * S;
    const double* g = geom + 4L * src;
    // L3 + L4 == LK
    with_split<LK>(L3, [&](auto c) {
        constexpr int A3 = decltype(c)::value;
        ket_record<A3, LK - A3>(i, j, b3, b4, symm, Dc, g, r);
    });
    (void) L4;
    if (rec32) {
        float* r32 = rec32 + (long) k * S;
#pragma unroll
        for (int t = 0; t < S; ++t) r32[t] = (float) r[t];   // S is runtime: plain loop
    }
}

// kbound of the sorted ket: recomputed from the sort keys
__global__ void k_ket_bounds(const unsigned* __restrict__ keys_sorted, const int* __restrict__ nkept,
                             float* __restrict__ kbound)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= *nkept) return;
    kbound[k] = __uint_as_float(~keys_sorted[k]);
}

// ---- 5. bra Hermite -> Cartesian --------------------------------------------

// Hermite index t -> (tx, ty, tz) as a compile-time table (so unrolled loops
// index registers, not memory).
constexpr int kHermTab = nherm_of(2 * kLmax + 1);   // Hermite orders up to the gradients' bra classes
struct HermTab {
    int x[kHermTab], y[kHermTab], z[kHermTab];
};
__host__ __device__ constexpr HermTab make_herm_tab()
{
    HermTab T{};
    for (int t = 0; t < kHermTab; ++t) {
        T.x[t] = herm_tx(t);
        T.y[t] = herm_ty(t);
        T.z[t] = herm_tz(t);
    }
    return T;
}

// Cartesian exponents (lx, ly, lz) of component k of a shell of angular
// momentum L <= kLmax, as a compile-time table.
struct CartTab {
    int x[kNL][ncart_of(kLmax)], y[kNL][ncart_of(kLmax)], z[kNL][ncart_of(kLmax)];
};
__host__ __device__ constexpr CartTab make_cart_tab()
{
    CartTab T{};
    for (int L = 0; L <= kLmax; ++L)
        for (int k = 0; k < ncart_of(L); ++k) {
            T.x[L][k] = cart_lx(L, k);
            T.y[L][k] = cart_ly(L, k);
            T.z[L][k] = cart_lz(L, k);
        }
    return T;
}

template <int L1, int L2>
__device__ void bra_to_cart(int i, int j, BasisView b1, BasisView b2, bool symm, const double* __restrict__ geom,
                            const double* __restrict__ jt, double* __restrict__ Jc)
{
    constexpr int N1 = ncart_of(L1), N2 = ncart_of(L2), H = nherm_of(L1 + L2);
    const double p = geom[0];
    const double P[3] = {geom[1], geom[2], geom[3]};
    const double A[3] = {b1.x[i], b1.y[i], b1.z[i]};
    const double B[3] = {b2.x[j], b2.y[j], b2.z[j]};
    double PA[3], PB[3];
    double R2 = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        PA[d] = P[d] - A[d];
        PB[d] = P[d] - B[d];
        R2 += (A[d] - B[d]) * (A[d] - B[d]);
    }
    const double e1 = b1.e[i], e2 = b2.e[j];
    double pre = kTwoPi52 / p * b1.c[i] * b2.c[j] * exp(-e1 * e2 / p * R2);
    if (symm && i == j) pre *= 0.5;
    ECoef<L1, L2> E;
    build_E<L1, L2>(p, PA, PB, E);
    const int a1 = b1.cart[i], a2 = b2.cart[j], ld = b2.ncart;
#pragma unroll
    for (int x = 0; x < N1; ++x)
#pragma unroll
        for (int y = 0; y < N2; ++y) {
            constexpr HermTab ht = make_herm_tab();
            constexpr CartTab ct = make_cart_tab();
            double s = 0.0;
#pragma unroll
            for (int t = 0; t < H; ++t)
                s += E.v[0][ct.x[L1][x]][ct.x[L2][y]][ht.x[t]] *
                     E.v[1][ct.y[L1][x]][ct.y[L2][y]][ht.y[t]] *
                     E.v[2][ct.z[L1][x]][ct.z[L2][y]][ht.z[t]] * jt[t];
            s *= pre;
            atomicAdd(&Jc[(long) (a1 + x) * ld + a2 + y], s);
            if (symm) atomicAdd(&Jc[(long) (a2 + y) * ld + a1 + x], s);
        }
}

template <int LB>
__global__ void k_herm_to_cart(const int* __restrict__ nbra, const int* __restrict__ p1,
                               const int* __restrict__ p2, const double* __restrict__ geom,
                               BasisView b1, BasisView b2, int symm, const double* __restrict__ jbra,
                               double* __restrict__ Jc)
{
    constexpr int H = nherm_of(LB);
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= *nbra) return;
    int i = p1[k], j = p2[k];
    int L1 = b1.L[i];
    const double* g = geom + 4L * k;
    const double* jt = jbra + (long) k * H;
    with_split<LB>(L1, [&](auto c) {
        constexpr int A1 = decltype(c)::value;
        bra_to_cart<A1, LB - A1>(i, j, b1, b2, symm, g, jt, Jc);
    });
}

// The same transform for the high bra classes (LB >= 3), a warp per bra
// pair: lane o (and o + 32) owns the Cartesian output (x, y) = (o / N2, o % N2)
// and raises its three 1-D coefficient vectors E^{l1,l2}_t in registers by the
// recursion of build_E (first in the exponent on A, then on B), so no
// coefficient table goes to local memory (one thread per pair needs the whole
// (LA+1)(LB+1)(LA+LB+1) table per direction).
template <int LB>
__global__ void k_herm_to_cart_warp(const int* __restrict__ nbra, const int* __restrict__ p1,
                                    const int* __restrict__ p2, const double* __restrict__ geom,
                                    BasisView b1, BasisView b2, int symm, const double* __restrict__ jbra,
                                    double* __restrict__ Jc)
{
    constexpr int H = nherm_of(LB), V = LB + 1;
    const int lane = threadIdx.x & 31;
    const long k = ((long) blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (k >= *nbra) return;   // whole warps leave together
    const int i = p1[k], j = p2[k];
    const int L1 = b1.L[i], L2 = LB - L1;
    const int N1 = ncart_of(L1), N2 = ncart_of(L2);
    const double* g = geom + 4L * k;
    const double p = g[0];
    const double A[3] = {b1.x[i], b1.y[i], b1.z[i]};
    const double B[3] = {b2.x[j], b2.y[j], b2.z[j]};
    double PA[3], PB[3];
    double R2 = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        PA[d] = g[1 + d] - A[d];
        PB[d] = g[1 + d] - B[d];
        R2 += (A[d] - B[d]) * (A[d] - B[d]);
    }
    double pre = kTwoPi52 / p * b1.c[i] * b2.c[j] * exp(-b1.e[i] * b2.e[j] / p * R2);
    if (symm && i == j) pre *= 0.5;
    const double h = 0.5 / p;
    const double* jt = jbra + k * H;
    const int a1 = b1.cart[i], a2 = b2.cart[j], ld = b2.ncart;
    struct Ev {
        double v[V];
    };
    // E^{l1,l2}_t of one direction: raised n1 times on A, then n2 times on B,
    // each step E'_t = X E_t + h E_{t-1} + (t+1) E_{t+1}
    auto vec = [h](int n1, int n2, double XA, double XB) {
        Ev e;
#pragma unroll
        for (int t = 0; t < V; ++t) e.v[t] = t == 0 ? 1.0 : 0.0;
#pragma unroll
        for (int r = 0; r < LB; ++r) {
            if (r >= n1 + n2) break;
            const double X = r < n1 ? XA : XB;
            Ev n;
#pragma unroll
            for (int t = 0; t < V; ++t) {
                double s = X * e.v[t];
                if (t > 0) s += h * e.v[t - 1];
                if (t + 1 < V) s += (t + 1) * e.v[t + 1];
                n.v[t] = s;
            }
            e = n;
        }
        return e;
    };
    for (int o = lane; o < N1 * N2; o += 32) {
        const int x = o / N2, y = o - x * N2;
        const Ev ex = vec(cart_lx(L1, x), cart_lx(L2, y), PA[0], PB[0]);
        const Ev ey = vec(cart_ly(L1, x), cart_ly(L2, y), PA[1], PB[1]);
        const Ev ez = vec(cart_lz(L1, x), cart_lz(L2, y), PA[2], PB[2]);
        constexpr HermTab ht = make_herm_tab();
        double s = 0.0;
#pragma unroll
        for (int t = 0; t < H; ++t) s += ex.v[ht.x[t]] * ey.v[ht.y[t]] * ez.v[ht.z[t]] * jt[t];
        s *= pre;
        atomicAdd(&Jc[(long) (a1 + x) * ld + a2 + y], s);
        if (symm) atomicAdd(&Jc[(long) (a2 + y) * ld + a1 + x], s);
    }
}

template <int LB>
void launch_j_row(Context* ctx, const JArgs& A, int LK, int nbra_full, int nket_full)
{
    switch (LK) {
    case 0: launch_j<LB, 0>(ctx, A, nbra_full, nket_full); break;
    case 1: launch_j<LB, 1>(ctx, A, nbra_full, nket_full); break;
    case 2: launch_j<LB, 2>(ctx, A, nbra_full, nket_full); break;
    case 3: launch_j<LB, 3>(ctx, A, nbra_full, nket_full); break;
    case 4: launch_j<LB, 4>(ctx, A, nbra_full, nket_full); break;
    case 5: launch_j<LB, 5>(ctx, A, nbra_full, nket_full); break;
    case 6: launch_j<LB, 6>(ctx, A, nbra_full, nket_full); break;
    default: throw Error(LSJK_ENOTSUPP, "J: ket Hermite class above 6");
    }
}

} // namespace

// ---- J nuclear gradient: bra derivatives ---------------------------------------
//
// With the Hermite potential V_t of the ket density at a bra pair one order
// above the pair's class (the J kernel run with bra class L1+L2+1), every
// Cartesian integral of the pair and of its shifted partners is
// pre * sum_t E^{ij}_t V_t. The derivative of a primitive Gaussian,
//   d/dA_x phi_i = 2 alpha phi_{i+1x} - i_x phi_{i-1x},
// then gives the pair's share of dE/dA and dE/dB, E = sum D_bra (ij|ket):
//   dE/dA_x = pre sum_ij D_ij (2 alpha (i+1x, j|) - i_x (i-1x, j|)), and in j for B.
template <int L1, int L2>
__device__ void bra_grad(int i, int j, BasisView b1, BasisView b2, bool symm, const double* __restrict__ geom,
                         const double* __restrict__ vt, const double* __restrict__ Dc, double scale,
                         double* __restrict__ G)
{
    constexpr int N1 = ncart_of(L1), N2 = ncart_of(L2), H = nherm_of(L1 + L2 + 1);
    constexpr HermTab ht = make_herm_tab();
    constexpr CartTab ct = make_cart_tab();
    const double p = geom[0];
    const double P[3] = {geom[1], geom[2], geom[3]};
    const double A[3] = {b1.x[i], b1.y[i], b1.z[i]};
    const double B[3] = {b2.x[j], b2.y[j], b2.z[j]};
    double PA[3], PB[3];
    double R2 = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        PA[d] = P[d] - A[d];
        PB[d] = P[d] - B[d];
        R2 += (A[d] - B[d]) * (A[d] - B[d]);
    }
    const double e1 = b1.e[i], e2 = b2.e[j];
    double pre = scale * kTwoPi52 / p * b1.c[i] * b2.c[j] * exp(-e1 * e2 / p * R2);
    if (symm && i == j) pre *= 0.5;
    ECoef<L1 + 1, L2 + 1> E;
    build_E<L1 + 1, L2 + 1>(p, PA, PB, E);
    auto I = [&](int lx, int ly, int lz, int mx, int my, int mz) {
        double s = 0.0;
#pragma unroll
        for (int t = 0; t < H; ++t)
            s += E.v[0][lx][mx][ht.x[t]] * E.v[1][ly][my][ht.y[t]] * E.v[2][lz][mz][ht.z[t]] * vt[t];
        return s;
    };
    const int a1 = b1.cart[i], a2 = b2.cart[j], ld = b2.ncart;
    double gA[3] = {0.0, 0.0, 0.0}, gB[3] = {0.0, 0.0, 0.0};
#pragma unroll 1
    for (int x = 0; x < N1; ++x)
#pragma unroll 1
        for (int y = 0; y < N2; ++y) {
            double dxy = Dc[(long) (a1 + x) * ld + a2 + y];
            if (symm) dxy += Dc[(long) (a2 + y) * ld + a1 + x];
            if (dxy == 0.0) continue;
            const int l[3] = {ct.x[L1][x], ct.y[L1][x], ct.z[L1][x]};
            const int m[3] = {ct.x[L2][y], ct.y[L2][y], ct.z[L2][y]};
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const int ux = d == 0, uy = d == 1, uz = d == 2;
                double ga = 2.0 * e1 * I(l[0] + ux, l[1] + uy, l[2] + uz, m[0], m[1], m[2]);
                if (l[d] > 0) ga -= l[d] * I(l[0] - ux, l[1] - uy, l[2] - uz, m[0], m[1], m[2]);
                double gb = 2.0 * e2 * I(l[0], l[1], l[2], m[0] + ux, m[1] + uy, m[2] + uz);
                if (m[d] > 0) gb -= m[d] * I(l[0], l[1], l[2], m[0] - ux, m[1] - uy, m[2] - uz);
                gA[d] += dxy * ga;
                gB[d] += dxy * gb;
            }
        }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        atomicAdd(&G[3 * b1.atom[i] + d], pre * gA[d]);
        atomicAdd(&G[3 * b2.atom[j] + d], pre * gB[d]);
    }
}

template <int LB>
__global__ void k_bra_grad(const int* __restrict__ nbra, const int* __restrict__ p1, const int* __restrict__ p2,
                           const double* __restrict__ geom, BasisView b1, BasisView b2, int symm,
                           const double* __restrict__ vbra, const double* __restrict__ Dc, double scale,
                           double* __restrict__ G)
{
    constexpr int H = nherm_of(LB + 1);
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= *nbra) return;
    int i = p1[k], j = p2[k];
    int L1 = b1.L[i];
    const double* g = geom + 4L * k;
    const double* vt = vbra + (long) k * H;
    with_split<LB>(L1, [&](auto c) {
        constexpr int A1 = decltype(c)::value;
        bra_grad<A1, LB - A1>(i, j, b1, b2, symm, g, vt, Dc, scale, G);
    });
}

// Algorithmic FP64/FP32 flops of one J quartet of Hermite class (LB|LK):
// prefactor/geometry 16, Boys (table 8 FMA + L recursion steps + exp),
// Hermite recursion (one FMA per R^{(n)}_{tuv}) and the contraction (2 flops
// per (t,u)); counted once per Ewald term.
double j_quartet_flops(int LB, int LK)
{
    int L = LB + LK;
    double nR = 0;
    for (int n = 0; n <= L; ++n) nR += nherm_of(L - n);
    return 16.0 + (16.0 + 3.0 * L + 1.0) + 2.0 * nR + 2.0 * nherm_of(LB) * nherm_of(LK);
}

namespace {

// Ket side of a J build and the bra truncation (stages 1 and 2), shared by the
// J build and the J gradient: per ket Hermite class the screened, bound-sorted
// ket records, and the device counts of kets and of bras that can pass.
struct KetSet {
    int* nket = nullptr;              // [kNHerm] kets kept per class (device)
    int* nbra = nullptr;              // [kNHerm] bra pairs that can pass per class (device)
    double* krec[kNHerm] = {};
    float* krec32[kNHerm] = {};
    float* kbound[kNHerm] = {};
};

KetSet prepare_kets(Context* ctx, const PairList* pl12, const PairList* pl34, const DSet& DS, float thresp,
                    bool mixed)
{
    cudaStream_t s = ctx->stream;
    const Basis *b3 = pl34->b1, *b4 = pl34->b2;
    // thresp / max12 (truncate_ket threshold), float as in the reference call
    const float thre_ket = (float) ((double) thresp / pl12->max_bound);
    int* counts = take<int>(ctx, 4 * kNHerm);          // nket[5], nbra[5]
    unsigned* maxbits = take<unsigned>(ctx, kNHerm);
    LSJK_CUDA(cudaMemsetAsync(counts, 0, sizeof(int) * 4 * kNHerm, s));
    LSJK_CUDA(cudaMemsetAsync(maxbits, 0, sizeof(unsigned) * kNHerm, s));
    KetSet K;
    K.nket = counts;
    K.nbra = counts + kNHerm;

    // 1. ket screening + sort per Hermite class
    for (int LK = 0; LK < kNHerm; ++LK) {
        const JBraClass& jk = pl34->jb[LK];
        int n = jk.n;
        if (n == 0) continue;
        unsigned* key = take<unsigned>(ctx, n);
        unsigned* keys = take<unsigned>(ctx, n);
        int* val = take<int>(ctx, n);
        int* perm = take<int>(ctx, n);
        k_ket_screen<<<nblk(n, 256), 256, 0, s>>>(jk.p1.p, jk.p2.p, jk.bound.p, n, b3->view(), b4->view(),
                                                 pl34->symm ? 1 : 0, DS, thre_ket, key, val, K.nket + LK,
                                                 maxbits + LK);
        size_t tmp = 0;
        LSJK_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, key, keys, val, perm, n, 0, 32, s));
        void* t = ctx->scratch_take(tmp);
        LSJK_CUDA(cub::DeviceRadixSort::SortPairs(t, tmp, key, keys, val, perm, n, 0, 32, s));
        double*& krec = K.krec[LK];
        float*& krec32 = K.krec32[LK];
        krec = take<double>(ctx, (long) n * (4 + DS.slots * nherm_of(LK)));
        if (mixed) krec32 = take<float>(ctx, (long) n * (4 + DS.slots * nherm_of(LK)));
        K.kbound[LK] = take<float>(ctx, n);
        k_ket_bounds<<<nblk(n, 256), 256, 0, s>>>(keys, K.nket + LK, K.kbound[LK]);
        int* nk = K.nket + LK;
        switch (LK) {
        case 0: k_ket_herm<0><<<nblk(n, 128), 128, 0, s>>>(perm, nk, jk.p1.p, jk.p2.p, jk.bound.p, jk.geom.p, b3->view(), b4->view(), pl34->symm, DS, krec, krec32); break;
        case 1: k_ket_herm<1><<<nblk(n, 128), 128, 0, s>>>(perm, nk, jk.p1.p, jk.p2.p, jk.bound.p, jk.geom.p, b3->view(), b4->view(), pl34->symm, DS, krec, krec32); break;
        case 2: k_ket_herm<2><<<nblk(n, 128), 128, 0, s>>>(perm, nk, jk.p1.p, jk.p2.p, jk.bound.p, jk.geom.p, b3->view(), b4->view(), pl34->symm, DS, krec, krec32); break;
        case 3: k_ket_herm<3><<<nblk(n, 128), 128, 0, s>>>(perm, nk, jk.p1.p, jk.p2.p, jk.bound.p, jk.geom.p, b3->view(), b4->view(), pl34->symm, DS, krec, krec32); break;
        case 4: k_ket_herm<4><<<nblk(n, 128), 128, 0, s>>>(perm, nk, jk.p1.p, jk.p2.p, jk.bound.p, jk.geom.p, b3->view(), b4->view(), pl34->symm, DS, krec, krec32); break;
        case 5: k_ket_herm<5><<<nblk(n, 128), 128, 0, s>>>(perm, nk, jk.p1.p, jk.p2.p, jk.bound.p, jk.geom.p, b3->view(), b4->view(), pl34->symm, DS, krec, krec32); break;
        case 6: k_ket_herm<6><<<nblk(n, 128), 128, 0, s>>>(perm, nk, jk.p1.p, jk.p2.p, jk.bound.p, jk.geom.p, b3->view(), b4->view(), pl34->symm, DS, krec, krec32); break;
        default: throw Error(LSJK_ENOTSUPP, "J: ket Hermite class above 6");
        }
        LSJK_CUDA(cudaGetLastError());
        ctx->stats.kernel_launches += 7;
    }

    // 2. bra truncation counts
    BraTables T{};
    for (int c = 0; c < kNHerm; ++c) {
        T.bound[c] = pl12->jb[c].bound.p;
        T.n[c] = pl12->jb[c].n;
    }
    k_bra_count<<<1, 32, 0, s>>>(maxbits, thresp, T, K.nbra);
    LSJK_CUDA(cudaGetLastError());
    ctx->stats.kernel_launches++;
    return K;
}

} // namespace

void coulomb_build(Context* ctx, const Ewald& ew, const PairList* pl12, const PairList* pl34,
                   const double* const* Dcart, double* const* Jcart, int ng, float thresp, float thredp)
{
    if (ng < 1 || ng > kMaxDens) throw Error(LSJK_EINVAL, "coulomb_build: 1..64 densities per build");
    DSet DS{};
    for (int g = 0; g < ng; ++g) DS.d[g] = Dcart[g];
    DS.n = ng;
    DS.slots = ng;
    cudaStream_t s = ctx->stream;
    const Basis *b1 = pl12->b1, *b2 = pl12->b2;
    unsigned long long* qcnt = ctx->counters.p;                          // FP64 J classes
    unsigned long long* qcnt32 = ctx->counters.p + kNJClass + kNKClass;  // FP32 J classes
    const bool mixed = ctx->precision == LSJK_PREC_MIXED && thredp > thresp;
    const KetSet KS = prepare_kets(ctx, pl12, pl34, DS, thresp, mixed);
    const int* nket = KS.nket;
    int* nbra = KS.nbra;
    double* const* krec = KS.krec;
    float* const* krec32 = KS.krec32;
    float* const* kbound = KS.kbound;

    // 3./4. J kernels
    double* jbra[kNHerm] = {};
    for (int LB = 0; LB < kNHerm; ++LB) {
        int n = pl12->jb[LB].n;
        if (!n) continue;
        jbra[LB] = take<double>(ctx, (long) DS.slots * n * nherm_of(LB));
        LSJK_CUDA(cudaMemsetAsync(jbra[LB], 0, sizeof(double) * DS.slots * n * nherm_of(LB), s));
    }
    // class kernels go round-robin to the auxiliary streams (not while the
    // autotuner times them one by one)
    const bool par = !ctx->tuning;
    if (par) fork_aux(ctx);
    int lane = 0;
    for (int LB = 0; LB < kNHerm; ++LB) {
        const JBraClass& jb = pl12->jb[LB];
        if (!jb.n) continue;
        for (int LK = 0; LK < kNHerm; ++LK) {
            const JBraClass& jk = pl34->jb[LK];
            if (!jk.n) continue;
            JArgs A{};
            A.bgeom = jb.geom.p;
            A.bbound = jb.bound.p;
            A.nbra = nbra + LB;
            A.jbra = jbra[LB];
            A.krec = krec[LK];
            A.kbound = kbound[LK];
            A.nket = nket + LK;
            A.boys = ctx->boys64.p + (long) (LB + LK) * LSJK_BOYS_NBIN * 8;
            A.status = ctx->status.p;
            A.qcount = qcnt + LB * kNHerm + LK;
            A.qcount32 = qcnt32 + LB * kNHerm + LK;
            A.krec32 = krec32[LK];
            A.boys32 = ctx->boys32.p + (long) (LB + LK) * LSJK_BOYS_NBIN * 8;
            A.mixed = mixed ? 1 : 0;
            A.thredp = thredp;
            if (ctx->tune.j_chunk[LB][LK] > 0) {
                A.chunk = ctx->tune.j_chunk[LB][LK];
            } else {
                // default: kJChunk kets per CTA, halved (down to 64) while the grid would not
                // give every multiprocessor two CTAs -- small molecules need the parallelism
                const long tiles = (jb.n + kJThreads - 1) / kJThreads;
                int chunk = kJChunk;
                while (chunk > 64 && tiles * ((jk.n + chunk - 1) / chunk) < 2L * ctx->nsm) chunk >>= 1;
                A.chunk = chunk;
            }
            A.ng = ng;
            A.slots = DS.slots;
            A.jbra_stride = (long) jb.n * nherm_of(LB);
            A.nterm = (int) ew.alpha.size();
            for (int t = 0; t < A.nterm; ++t) {
                A.alpha[t] = ew.alpha[t];
                A.omega[t] = ew.omega[t];
            }
            A.thresp = thresp;
            auto launch = [&](const JArgs& X) {
                switch (LB) {
                case 0: launch_j_row<0>(ctx, X, LK, jb.n, jk.n); break;
                case 1: launch_j_row<1>(ctx, X, LK, jb.n, jk.n); break;
                case 2: launch_j_row<2>(ctx, X, LK, jb.n, jk.n); break;
                case 3: launch_j_row<3>(ctx, X, LK, jb.n, jk.n); break;
                case 4: launch_j_row<4>(ctx, X, LK, jb.n, jk.n); break;
                case 5: launch_j_row<5>(ctx, X, LK, jb.n, jk.n); break;
                case 6: launch_j_row<6>(ctx, X, LK, jb.n, jk.n); break;
                default: throw Error(LSJK_ENOTSUPP, "J: bra Hermite class above 6");
                }
            };
            if (ctx->tuning) {
                // autotuner: time the candidate ket chunk sizes on scratch outputs
                static const int cand[] = {128, 256, 512, 1024, 2048, 4096};
                JArgs T = A;
                T.jbra = take<double>(ctx, (long) DS.slots * jb.n * nherm_of(LB));
                T.qcount = T.qcount32 = ctx->tune_sink.p;
                float best = 1e30f;
                for (int c : cand) {
                    T.chunk = c;
                    float ms = 1e30f;
                    for (int rep = 0; rep < 2; ++rep) {
                        LSJK_CUDA(cudaEventRecord(ctx->ev0, s));
                        launch(T);
                        LSJK_CUDA(cudaEventRecord(ctx->ev1, s));
                        LSJK_CUDA(cudaEventSynchronize(ctx->ev1));
                        float t = 0.f;
                        LSJK_CUDA(cudaEventElapsedTime(&t, ctx->ev0, ctx->ev1));
                        ms = std::min(ms, t);
                    }
                    if (ms < best) {
                        best = ms;
                        ctx->tune.j_chunk[LB][LK] = c;
                    }
                }
                A.chunk = ctx->tune.j_chunk[LB][LK];
            }
            std::optional<OnAux> on;
            if (par) on.emplace(ctx, lane++);
            launch(A);
        }
    }
    if (par) join_aux(ctx);

    // 5. back to Cartesian, per density
    for (int g = 0; g < ng; ++g)
        for (int LB = 0; LB < kNHerm; ++LB) {
            const JBraClass& jb = pl12->jb[LB];
            if (!jb.n) continue;
            unsigned gr = nblk(jb.n, 128);
            const double* jt = jbra[LB] + (long) g * jb.n * nherm_of(LB);
            double* Jc = Jcart[g];
            switch (LB) {
            case 0: k_herm_to_cart<0><<<gr, 128, 0, s>>>(nbra + LB, jb.p1.p, jb.p2.p, jb.geom.p, b1->view(), b2->view(), pl12->symm, jt, Jc); break;
            case 1: k_herm_to_cart<1><<<gr, 128, 0, s>>>(nbra + LB, jb.p1.p, jb.p2.p, jb.geom.p, b1->view(), b2->view(), pl12->symm, jt, Jc); break;
            case 2: k_herm_to_cart<2><<<gr, 128, 0, s>>>(nbra + LB, jb.p1.p, jb.p2.p, jb.geom.p, b1->view(), b2->view(), pl12->symm, jt, Jc); break;
            case 3: k_herm_to_cart_warp<3><<<nblk(jb.n, 4), 128, 0, s>>>(nbra + LB, jb.p1.p, jb.p2.p, jb.geom.p, b1->view(), b2->view(), pl12->symm, jt, Jc); break;
            case 4: k_herm_to_cart_warp<4><<<nblk(jb.n, 4), 128, 0, s>>>(nbra + LB, jb.p1.p, jb.p2.p, jb.geom.p, b1->view(), b2->view(), pl12->symm, jt, Jc); break;
            case 5: k_herm_to_cart_warp<5><<<nblk(jb.n, 4), 128, 0, s>>>(nbra + LB, jb.p1.p, jb.p2.p, jb.geom.p, b1->view(), b2->view(), pl12->symm, jt, Jc); break;
            case 6: k_herm_to_cart_warp<6><<<nblk(jb.n, 4), 128, 0, s>>>(nbra + LB, jb.p1.p, jb.p2.p, jb.geom.p, b1->view(), b2->view(), pl12->symm, jt, Jc); break;
            default: throw Error(LSJK_ENOTSUPP, "J: bra Hermite class above 6");
            }
            LSJK_CUDA(cudaGetLastError());
            ctx->stats.kernel_launches++;
        }
}

// One bra-derivative pass of the J gradient: kets from Dket, bra pairs
// contracted with Dbra, derivatives at the bra centres into G.
static void coulomb_grad_bra(Context* ctx, const Ewald& ew, const PairList* pl, const double* Dbra,
                             const double* Dket, double scale, double* G, float thresp)
{
    cudaStream_t s = ctx->stream;
    DSet DS{};
    DS.d[0] = Dket;
    DS.n = 1;
    DS.slots = 1;
    const KetSet KS = prepare_kets(ctx, pl, pl, DS, thresp, false);
    for (int LB = 0; LB < kNHerm; ++LB) {
        const JBraClass& jb = pl->jb[LB];
        if (!jb.n) continue;
        const int H1 = nherm_of(LB + 1);
        double* vbra = take<double>(ctx, (long) jb.n * H1);
        LSJK_CUDA(cudaMemsetAsync(vbra, 0, sizeof(double) * jb.n * H1, s));
        for (int LK = 0; LK < kNHerm; ++LK) {
            const JBraClass& jk = pl->jb[LK];
            if (!jk.n) continue;
            // the J kernel of bra class LB + 1 over the class-LB pairs: the Hermite potential
            // of the ket density one order above the pairs' own class
            JArgs A{};
            A.bgeom = jb.geom.p;
            A.bbound = jb.bound.p;
            A.nbra = KS.nbra + LB;
            A.jbra = vbra;
            A.krec = KS.krec[LK];
            A.kbound = KS.kbound[LK];
            A.nket = KS.nket + LK;
            A.boys = ctx->boys64.p + (long) (LB + 1 + LK) * LSJK_BOYS_NBIN * 8;
            A.status = ctx->status.p;
            A.qcount = A.qcount32 = ctx->tune_sink.p;
            A.mixed = 0;
            A.thredp = thresp;
            int chunk = kJChunk;
            const long tiles = (jb.n + kJThreads - 1) / kJThreads;
            while (chunk > 64 && tiles * ((jk.n + chunk - 1) / chunk) < 2L * ctx->nsm) chunk >>= 1;
            A.chunk = chunk;
            A.ng = 1;
            A.slots = 1;
            A.jbra_stride = (long) jb.n * H1;
            A.nterm = (int) ew.alpha.size();
            for (int t = 0; t < A.nterm; ++t) {
                A.alpha[t] = ew.alpha[t];
                A.omega[t] = ew.omega[t];
            }
            A.thresp = thresp;
            switch (LB + 1) {
            case 1: launch_j_row<1>(ctx, A, LK, jb.n, jk.n); break;
            case 2: launch_j_row<2>(ctx, A, LK, jb.n, jk.n); break;
            case 3: launch_j_row<3>(ctx, A, LK, jb.n, jk.n); break;
            case 4: launch_j_row<4>(ctx, A, LK, jb.n, jk.n); break;
            case 5: launch_j_row<5>(ctx, A, LK, jb.n, jk.n); break;
            case 6: launch_j_row<6>(ctx, A, LK, jb.n, jk.n); break;
            case 7: launch_j_row<7>(ctx, A, LK, jb.n, jk.n); break;
            default: throw Error(LSJK_ENOTSUPP, "J gradient: bra Hermite class above 7");
            }
        }
        const BasisView v1 = pl->b1->view(), v2 = pl->b2->view();
        const unsigned gr = nblk(jb.n, 64);
        switch (LB) {
        case 0: k_bra_grad<0><<<gr, 64, 0, s>>>(KS.nbra + LB, jb.p1.p, jb.p2.p, jb.geom.p, v1, v2, pl->symm, vbra, Dbra, scale, G); break;
        case 1: k_bra_grad<1><<<gr, 64, 0, s>>>(KS.nbra + LB, jb.p1.p, jb.p2.p, jb.geom.p, v1, v2, pl->symm, vbra, Dbra, scale, G); break;
        case 2: k_bra_grad<2><<<gr, 64, 0, s>>>(KS.nbra + LB, jb.p1.p, jb.p2.p, jb.geom.p, v1, v2, pl->symm, vbra, Dbra, scale, G); break;
        case 3: k_bra_grad<3><<<gr, 64, 0, s>>>(KS.nbra + LB, jb.p1.p, jb.p2.p, jb.geom.p, v1, v2, pl->symm, vbra, Dbra, scale, G); break;
        case 4: k_bra_grad<4><<<gr, 64, 0, s>>>(KS.nbra + LB, jb.p1.p, jb.p2.p, jb.geom.p, v1, v2, pl->symm, vbra, Dbra, scale, G); break;
        case 5: k_bra_grad<5><<<gr, 64, 0, s>>>(KS.nbra + LB, jb.p1.p, jb.p2.p, jb.geom.p, v1, v2, pl->symm, vbra, Dbra, scale, G); break;
        case 6: k_bra_grad<6><<<gr, 64, 0, s>>>(KS.nbra + LB, jb.p1.p, jb.p2.p, jb.geom.p, v1, v2, pl->symm, vbra, Dbra, scale, G); break;
        default: throw Error(LSJK_ENOTSUPP, "J gradient: bra Hermite class above 6");
        }
        LSJK_CUDA(cudaGetLastError());
        ctx->stats.kernel_launches++;
    }
}

// E = sum D12 (12|34) D34 moves with all four centres: its gradient is the
// bra-centre derivative with D12 on the bra and D34 on the ket, plus the same
// with the roles exchanged ((12|34) = (34|12)).
void coulomb_grad(Context* ctx, const Ewald& ew, const PairList* pl, const double* D12cart, const double* D34cart,
                  bool same, double* G, float thresp)
{
    if (!pl->symm) throw Error(LSJK_EINVAL, "IntBox::coulombGrad: pairlist must be symmetric");
    if (ew.alpha.empty() || !pl->npair) return;
    if (same) {
        coulomb_grad_bra(ctx, ew, pl, D12cart, D34cart, 2.0, G, thresp);   // both halves are this pass
    } else {
        coulomb_grad_bra(ctx, ew, pl, D12cart, D34cart, 1.0, G, thresp);
        coulomb_grad_bra(ctx, ew, pl, D34cart, D12cart, 1.0, G, thresp);
    }
}

} // namespace lsjk
