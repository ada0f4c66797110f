// Nuclear gradient of the exchange energy on the device: the reference's
// IntBox::exchangeGrad (src/lightspeed/intbox.hpp:1147-1160,
// src/cpp/intbox/intbox.cpp:519-607; CPU kernels src/cpp/intbox/cpu/exchange_grad.cpp)
//
//   G[atom] += sum_{1234} D13 d(12|34)/dR D24
//
// over the K-invert quartets of the K build (kbuild.cu): the same task list of
// (prim2, prim4) pairs and the same partner rows, here both in bound order.
// A warp takes a task, its lanes take 32 partners 3 at a time and walk the
// partners 1 together. Each quartet's derivatives come from the Rys
// quadrature one quantum higher: the 2-D integrals of the vertical recursion
//   I(a+1,0) = C00 I(a,0) + a B10 I(a-1,0)
//   I(a,c+1) = D00 I(a,c) + c B01 I(a,c-1) + a B00 I(a-1,c)
// and the horizontal transfers to centres 2 and 4, then for each Cartesian
// component d/dA_x (ab|cd) = 2 alpha (a+1x b|cd) - a_x (a-1x b|cd) (likewise at
// B and C; D by translational invariance). FP64 throughout, plain loops over
// small local arrays: this is not the hot path. Contributions collect per atom
// in registers (partner-1 atom: warp-uniform; prim2 and prim4: per task;
// partner-3: per lane) and reach G with few atomics.
#include <atomic>
#include "engine.cuh"
#include "kargs.cuh"
#include "lsjk_device.cuh"
#include "hermite.cuh"   // cart_lx/ly/lz

#ifndef LSJK_KG_L1
#error "compile with -DLSJK_KG_L1=<partner-1 shell>"
#endif

namespace lsjk {

namespace {

constexpr double kTwoPi52G = 34.986836655249725693;   // 2 pi^(5/2)
constexpr int kGradStripes3 = 32;      // partner-3 stripes of a task in the warp kernel, at most
constexpr int kGradStripesMax = 256;  // work units per task, at most (beyond 32: partner-1 stripes too)

// Smallest float x with double(x) * dmax >= thr (as in the K kernel).
__device__ __forceinline__ float grad_threshold(double thr, double dmax)
{
    if (!(thr > 0.0)) return 0.0f;
    if (!(dmax > 0.0)) return __int_as_float(0x7f800000);
    float x = (float) (thr / dmax);
    for (int it = 0; it < 8 && (double) x * dmax < thr; ++it) x = nextafterf(x, __int_as_float(0x7f800000));
    for (int it = 0; it < 8 && x > 0.0f && (double) nextafterf(x, 0.0f) * dmax >= thr; ++it) x = nextafterf(x, 0.0f);
    return x;
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Light classes (small 1-D integral tables and few Cartesian combinations):
// one lane per quartet with every loop unrolled into registers.
template <int L1, int L2, int L3, int L4>
__host__ __device__ constexpr bool kgrad_flat()
{
    return (L1 + 2) * (L2 + 2) * (L3 + 2) * (L4 + 1) <= 27 &&
           ncart_of(L1) * ncart_of(L2) * ncart_of(L3) * ncart_of(L4) <= 27;
}

// Every class that is not light runs one quartet per warp with the tables in
// shared memory (with work units of partner-3 stripes this measured faster than a
// quartet per lane for every such class); the light ones one quartet per lane.
template <int L1, int L2, int L3, int L4>
__host__ __device__ constexpr bool kgrad_warp()
{
    return !kgrad_flat<L1, L2, L3, L4>();
}

// One quartet's derivatives at centres 1, 2 and 3 contracted with the D13 and
// D24 blocks, added into gA, gB, gC.
template <int L1, int L2, int L3, int L4>
__device__ void kgrad_quartet(const KGradArgs& A, double alpha, double beta, double gamma, double kab12, double p,
                              double ip, const double P[3], const double Ar[3], double kab34, double q, double iq,
                              const double Qs[3], const double QC[3], const double Cr[3],
                              const double* __restrict__ D13, const double* __restrict__ D24, double gA[3],
                              double gB[3], double gC[3])
{
    constexpr int NR = (L1 + L2 + L3 + L4 + 1) / 2 + 1;
    constexpr int MA = L1 + L2 + 2, MC = L3 + L4 + 1;   // vertical-recursion extents (one quantum up)
    constexpr int XA = L1 + 2, XB = L2 + 2, XC = L3 + 2, XE = L4 + 1;
    constexpr int N1 = ncart_of(L1), N2 = ncart_of(L2), N3 = ncart_of(L3), N4 = ncart_of(L4);
    // light classes: every loop unrolled, so the 1-D integral tables live in
    // registers with compile-time indices; the others keep runtime loops over
    // local arrays (their tables are too large for registers)
    constexpr bool kFlat = kgrad_flat<L1, L2, L3, L4>();
    constexpr int U3 = kFlat ? 3 : 1, U1 = kFlat ? N1 : 1, U2 = kFlat ? N2 : 1, U3c = kFlat ? N3 : 1,
                  U4 = kFlat ? N4 : 1, UR = kFlat ? NR : 1;
    double PQ[3], PA[3];
    double RR = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        PQ[d] = P[d] + Qs[d];   // (P - R2) - (Q - R4) + (R2 - R4)
        PA[d] = P[d] - Ar[d];
        RR += PQ[d] * PQ[d];
    }
    const double rs = rsqrt(p + q);
    const double ipq = rs * rs;
    const double rho = p * q * ipq;
    // kab fields hold K_ab / p per pair
    const double pref = kTwoPi52G * (kab12 * kab34) * rs;
#pragma unroll 1
    for (int tm = 0; tm < A.nterm; ++tm) {
        double d2 = 1.0, f = A.alpha[tm] * pref;
        if (A.omega[tm] != -1.0) {
            const double w2 = A.omega[tm] * A.omega[tm];
            d2 = w2 / (rho + w2);
            f *= sqrt(d2);
        }
        double t2[NR], w[NR];
        rys_eval<NR, double>(rho * d2 * RR, A.rys, A.nbin, A.tmax, A.asym_t, A.asym_w, t2, w);
#pragma unroll (UR)
        for (int r = 0; r < NR; ++r) {
            const double u = t2[r] * d2 * ipq;
            const double b00 = 0.5 * u, b10 = 0.5 * ip * (1.0 - q * u), b01 = 0.5 * iq * (1.0 - p * u);
            // 1-D integrals X[d][a][b][c][e], a <= L1+1, b <= L2+1, c <= L3+1, e <= L4
            // (the entries with a+b+c+e above L+1 are not exact for this rule and not used)
            double X[3][XA][XB][XC][XE];
#pragma unroll (U3)
            for (int d = 0; d < 3; ++d) {
                const double c00 = PA[d] - q * u * PQ[d], d00 = QC[d] + p * u * PQ[d];
                double I[MA + 1][MC + 1];
                I[0][0] = d == 2 ? f * w[r] : 1.0;
#pragma unroll
                for (int a = 0; a < MA; ++a) I[a + 1][0] = c00 * I[a][0] + (a ? a * b10 * I[a - 1][0] : 0.0);
#pragma unroll
                for (int c = 0; c < MC; ++c)
#pragma unroll
                    for (int a = 0; a <= MA; ++a) {
                        double v = d00 * I[a][c];
                        if (c) v += c * b01 * I[a][c - 1];
                        if (a) v += a * b00 * I[a - 1][c];
                        I[a][c + 1] = v;
                    }
                // transfer to centre 2, in place over a: H(a, b+1) = H(a+1, b) + (A - B) H(a, b);
                // after step b, row a holds H(a, b) for a <= MA - b
                double Hb[XB][XA][MC + 1];
#pragma unroll
                for (int a = 0; a < XA; ++a)
#pragma unroll
                    for (int c = 0; c <= MC; ++c) Hb[0][a][c] = I[a][c];
#pragma unroll
                for (int b = 0; b + 1 < XB; ++b) {
#pragma unroll
                    for (int a = 0; a + 1 <= MA - b; ++a)
#pragma unroll
                        for (int c = 0; c <= MC; ++c) I[a][c] = I[a + 1][c] + Ar[d] * I[a][c];
#pragma unroll
                    for (int a = 0; a < XA && a <= MA - b - 1; ++a)
#pragma unroll
                        for (int c = 0; c <= MC; ++c) Hb[b + 1][a][c] = I[a][c];
                }
                // and to centre 4: (c, e+1) = (c+1, e) + (C - D) (c, e)
#pragma unroll
                for (int a = 0; a < XA; ++a)
#pragma unroll
                    for (int b = 0; b < XB; ++b) {
                        if (a + b > MA) continue;
                        double Hd[MC + 1];
#pragma unroll
                        for (int c = 0; c <= MC; ++c) Hd[c] = Hb[b][a][c];
#pragma unroll
                        for (int c = 0; c < XC; ++c) X[d][a][b][c][0] = Hd[c];
#pragma unroll
                        for (int e = 0; e + 1 < XE; ++e) {
#pragma unroll
                            for (int c = 0; c + 1 <= MC - e; ++c) Hd[c] = Hd[c + 1] + Cr[d] * Hd[c];
#pragma unroll
                            for (int c = 0; c < XC && c <= MC - e - 1; ++c) X[d][a][b][c][e + 1] = Hd[c];
                        }
                    }
            }
            // contraction with D13[i1, i3] D24[i2, i4]
#pragma unroll (U1)
            for (int i1 = 0; i1 < N1; ++i1) {
                const int a[3] = {cart_lx(L1, i1), cart_ly(L1, i1), cart_lz(L1, i1)};
#pragma unroll (U3c)
                for (int i3 = 0; i3 < N3; ++i3) {
                    const double d13 = D13[i1 * N3 + i3];
                    if (d13 == 0.0) continue;
                    const int c[3] = {cart_lx(L3, i3), cart_ly(L3, i3), cart_lz(L3, i3)};
#pragma unroll (U2)
                    for (int i2 = 0; i2 < N2; ++i2) {
                        const int b[3] = {cart_lx(L2, i2), cart_ly(L2, i2), cart_lz(L2, i2)};
#pragma unroll (U4)
                        for (int i4 = 0; i4 < N4; ++i4) {
                            const double W = d13 * D24[i2 * N4 + i4];
                            if (W == 0.0) continue;
                            const int e[3] = {cart_lx(L4, i4), cart_ly(L4, i4), cart_lz(L4, i4)};
                            double v[3], da[3], db[3], dc[3];
#pragma unroll
                            for (int d = 0; d < 3; ++d) {
                                const int ad = a[d], bd = b[d], cd = c[d], ed = e[d];
                                v[d] = X[d][ad][bd][cd][ed];
                                da[d] = 2.0 * alpha * X[d][ad + 1][bd][cd][ed];
                                if (ad) da[d] -= ad * X[d][ad - 1][bd][cd][ed];
                                db[d] = 2.0 * beta * X[d][ad][bd + 1][cd][ed];
                                if (bd) db[d] -= bd * X[d][ad][bd - 1][cd][ed];
                                dc[d] = 2.0 * gamma * X[d][ad][bd][cd + 1][ed];
                                if (cd) dc[d] -= cd * X[d][ad][bd][cd - 1][ed];
                            }
                            const double yz = W * v[1] * v[2], xz = W * v[0] * v[2], xy = W * v[0] * v[1];
                            gA[0] += da[0] * yz;
                            gA[1] += da[1] * xz;
                            gA[2] += da[2] * xy;
                            gB[0] += db[0] * yz;
                            gB[1] += db[1] * xz;
                            gB[2] += db[2] * xy;
                            gC[0] += dc[0] * yz;
                            gC[1] += dc[1] * xz;
                            gC[2] += dc[2] * xy;
                        }
                    }
                }
            }
        }
    }
}

template <int L1, int L2, int L3, int L4>
__global__ void __launch_bounds__(128) k_exchange_grad(const __grid_constant__ KGradArgs A)
{
    constexpr int N1 = ncart_of(L1), N2 = ncart_of(L2), N3 = ncart_of(L3), N4 = ncart_of(L4);
    const int ntask = *A.ntask;
    const int lane = threadIdx.x & 31;
    const float thre12 = A.sc->thre12, thre34 = A.sc->thre34;
    for (;;) {
        int t = 0;
        if (lane == 0) t = (int) atomicAdd(A.queue, 1u);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= ntask) break;
        const KTask T = A.tasks[t];
        const int i2 = T.i2, i4 = T.i4;
        const float tlo = grad_threshold((double) A.thr_lo, T.dmax);
        const double dR[3] = {A.b2.x[i2] - A.b4.x[i4], A.b2.y[i2] - A.b4.y[i4], A.b2.z[i2] - A.b4.z[i4]};
        const double beta = A.b2.e[i2];
        const int c2 = A.b2.cart[i2], c4 = A.b4.cart[i4];
        const double w24 = (A.pairsym && i2 != i4) ? 2.0 : 1.0;   // a task and its mirror
        double D24[N2 * N4];
        for (int a = 0; a < N2; ++a)
            for (int b = 0; b < N4; ++b) D24[a * N4 + b] = w24 * A.D24[(long) (c2 + a) * A.ld24 + c4 + b];
        const int s12 = A.r12s[i2], n12 = A.r12l[i2], s34 = A.r34s[i4], n34 = A.r34l[i4];
        double gB[3] = {0, 0, 0}, gD[3] = {0, 0, 0};
        for (int cs = 0; cs < n34; cs += 32) {
            const int k3 = s34 + cs + lane;
            const bool in3 = cs + lane < n34;
            float b34 = 0.0f;
            double kab34 = 0, q = 1, iq = 1, gamma = 0, Qs[3] = {0, 0, 0}, QC[3] = {0, 0, 0}, Cr[3] = {0, 0, 0};
            int c3 = 0, atomC = 0, K3 = 0;
            if (in3) {
                b34 = A.b34[k3];
                kab34 = A.kab34[k3];
                q = A.p34[k3];
                iq = A.ip34[k3];
                gamma = A.pe34[k3];
                const double Q[3] = {A.px34[k3], A.py34[k3], A.pz34[k3]};
                Cr[0] = A.ax34[k3];
                Cr[1] = A.ay34[k3];
                Cr[2] = A.az34[k3];
                for (int d = 0; d < 3; ++d) {
                    QC[d] = Q[d] - Cr[d];
                    Qs[d] = dR[d] - Q[d];
                }
                c3 = A.cart34[k3];
                atomC = A.atom34[k3];
                K3 = A.pidx34[k3];
            }
            const bool v3 = in3 && b34 >= thre34;
            float bmax34 = v3 ? b34 : 0.0f;
            for (int o = 16; o > 0; o >>= 1) bmax34 = fmaxf(bmax34, __shfl_xor_sync(0xffffffffu, bmax34, o));
            if (bmax34 == 0.0f || A.b12[s12] * bmax34 < tlo) break;   // rows in bound order
            double gA[3] = {0, 0, 0}, gC[3] = {0, 0, 0};
            int atomA = -1;
            for (int j = 0; j < n12; ++j) {
                const int e = s12 + j;
                const float b12 = A.b12[e];
                if (b12 < thre12 || b12 * bmax34 < tlo) break;   // bound order: nothing later passes
                const int aj = A.atom12[e];
                if (aj != atomA) {
                    if (atomA >= 0)
                        for (int d = 0; d < 3; ++d) {
                            const double s = warp_sum(gA[d]);
                            if (lane == 0 && s != 0.0) atomicAdd(&A.G[3 * atomA + d], s);
                            gA[d] = 0.0;
                        }
                    atomA = aj;
                }
                bool pass = v3 && b12 * b34 >= tlo;
                if (pass && A.canon) {
                    // the fully symmetric routine screens each quartet with the D block
                    // of its representative's primitives 2 and 4 (exchange_grad.cpp:137-217):
                    // (max(prim1, prim2), max(prim3, prim4)) for a symmetric D
                    const int K1 = A.pidx12[e];
                    const int r2 = K1 > i2 ? K1 : i2, r4 = K3 > i4 ? K3 : i4;
                    pass = (double) (b12 * b34) * A.dblk[(long) r2 * A.nprim + r4] >= (double) A.thr_lo;
                }
                if (!pass) continue;
                const double P[3] = {A.px12[e], A.py12[e], A.pz12[e]};
                const double Ar[3] = {A.ax12[e], A.ay12[e], A.az12[e]};
                const int c1 = A.cart12[e];
                double D13[N1 * N3];
                for (int a = 0; a < N1; ++a)
                    for (int c = 0; c < N3; ++c) D13[a * N3 + c] = A.D13[(long) (c1 + a) * A.ld13 + c3 + c];
                double qa[3] = {0, 0, 0}, qb[3] = {0, 0, 0}, qc[3] = {0, 0, 0};
                kgrad_quartet<L1, L2, L3, L4>(A, A.pe12[e], beta, gamma, A.kab12[e], A.p12[e], A.ip12[e], P, Ar, kab34,
                                              q, iq, Qs, QC, Cr, D13, D24, qa, qb, qc);
                for (int d = 0; d < 3; ++d) {
                    gA[d] += qa[d];
                    gB[d] += qb[d];
                    gC[d] += qc[d];
                    gD[d] -= qa[d] + qb[d] + qc[d];   // translational invariance
                }
            }
            if (atomA >= 0)
                for (int d = 0; d < 3; ++d) {
                    const double s = warp_sum(gA[d]);
                    if (lane == 0 && s != 0.0) atomicAdd(&A.G[3 * atomA + d], s);
                }
            if (in3)
                for (int d = 0; d < 3; ++d)
                    if (gC[d] != 0.0) atomicAdd(&A.G[3 * atomC + d], gC[d]);
        }
        for (int d = 0; d < 3; ++d) {
            const double sb = warp_sum(gB[d]), sd = warp_sum(gD[d]);
            if (lane == 0) {
                if (sb != 0.0) atomicAdd(&A.G[3 * A.b2.atom[i2] + d], sb);
                if (sd != 0.0) atomicAdd(&A.G[3 * A.b4.atom[i4] + d], sd);
            }
        }
    }
}

// Per-warp shared tables of the warp-cooperative quartet.
template <int L1, int L2, int L3, int L4>
struct KGradWarpTables {
    static constexpr int MA = L1 + L2 + 2, MC = L3 + L4 + 1, XA = L1 + 2, XB = L2 + 2, XC = L3 + 2, XE = L4 + 1;
    double X[3][XA][XB][XC][XE];      // 1-D integrals (as in kgrad_quartet)
    double I[3][MA + 1][MC + 1];      // vertical recursion, per direction
    double Hb[3][XB][XA][MC + 1];     // after the transfer to centre 2
    double D13[ncart_of(L1) * ncart_of(L3)];
    double D24[ncart_of(L2) * ncart_of(L4)];
    // per (a <= L1, b <= L2, c <= L3, e <= L4) and direction: the 1-D integral and its
    // derivatives at centres 1, 2 and 3 (2 alpha X(a+1) - a X(a-1), likewise in b, c)
    static constexpr int SG = (L1 + 1) * (L2 + 1) * (L3 + 1) * (L4 + 1);
    double T4[3][SG][4];
};

// One quartet of a heavy class, computed by the whole warp: lanes 0-2 run the
// vertical recursion and the transfer to centre 2 of one direction each, the
// lanes share the transfers to centre 4 (one (direction, a, b) row each) and
// the Cartesian combinations of the contraction; the tables live in shared
// memory. Each lane returns its part of the derivative sums.
template <int L1, int L2, int L3, int L4>
__device__ void kgrad_quartet_warp(const KGradArgs& A, KGradWarpTables<L1, L2, L3, L4>& S, int lane, double alpha,
                                   double beta, double gamma, double kab12, double p, double ip, const double P[3],
                                   const double Ar[3], double kab34, double q, double iq, const double Qs[3],
                                   const double QC[3], const double Cr[3], double gA[3], double gB[3], double gC[3])
{
    using Tab = KGradWarpTables<L1, L2, L3, L4>;
    constexpr int NR = (L1 + L2 + L3 + L4 + 1) / 2 + 1;
    constexpr int MA = Tab::MA, MC = Tab::MC, XA = Tab::XA, XB = Tab::XB, XC = Tab::XC, XE = Tab::XE;
    constexpr int N1 = ncart_of(L1), N2 = ncart_of(L2), N3 = ncart_of(L3), N4 = ncart_of(L4);
    // contraction jobs: element (i1, i3) of D13, split over P ranges of i2 when there are
    // fewer elements than lanes
    constexpr int NO = N1 * N3, NPART = NO >= 32 ? 1 : (N2 < 32 / NO ? N2 : 32 / NO);
    constexpr int NJOB = NO * NPART, NJL = (NJOB + 31) / 32;
    double PQ[3], PA[3];
    double RR = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        PQ[d] = P[d] + Qs[d];
        PA[d] = P[d] - Ar[d];
        RR += PQ[d] * PQ[d];
    }
    const double rs = rsqrt(p + q);
    const double ipq = rs * rs;
    const double rho = p * q * ipq;
    const double pref = kTwoPi52G * (kab12 * kab34) * rs;
    // this lane's direction in the recursions (lanes 0-2)
    const int dl = lane < 3 ? lane : 0;
    const double PAd = dl == 0 ? PA[0] : (dl == 1 ? PA[1] : PA[2]);
    const double PQd = dl == 0 ? PQ[0] : (dl == 1 ? PQ[1] : PQ[2]);
    const double QCd = dl == 0 ? QC[0] : (dl == 1 ? QC[1] : QC[2]);
    const double ABd = dl == 0 ? Ar[0] : (dl == 1 ? Ar[1] : Ar[2]);
#pragma unroll 1
    for (int tm = 0; tm < A.nterm; ++tm) {
        double d2 = 1.0, f = A.alpha[tm] * pref;
        if (A.omega[tm] != -1.0) {
            const double w2 = A.omega[tm] * A.omega[tm];
            d2 = w2 / (rho + w2);
            f *= sqrt(d2);
        }
        double t2[NR], w[NR];
        rys_eval<NR, double>(rho * d2 * RR, A.rys, A.nbin, A.tmax, A.asym_t, A.asym_w, t2, w);
#pragma unroll 1
        for (int r = 0; r < NR; ++r) {
            const double u = t2[r] * d2 * ipq;
            const double b00 = 0.5 * u, b10 = 0.5 * ip * (1.0 - q * u), b01 = 0.5 * iq * (1.0 - p * u);
            if (lane < 3) {
                // vertical recursion and transfer to centre 2 of direction dl
                double (*I)[MC + 1] = S.I[dl];
                const double c00 = PAd - q * u * PQd, d00 = QCd + p * u * PQd;
                I[0][0] = dl == 2 ? f * w[r] : 1.0;
#pragma unroll
                for (int a = 0; a < MA; ++a) I[a + 1][0] = c00 * I[a][0] + (a ? a * b10 * I[a - 1][0] : 0.0);
#pragma unroll
                for (int c = 0; c < MC; ++c)
#pragma unroll
                    for (int a = 0; a <= MA; ++a) {
                        double v = d00 * I[a][c];
                        if (c) v += c * b01 * I[a][c - 1];
                        if (a) v += a * b00 * I[a - 1][c];
                        I[a][c + 1] = v;
                    }
#pragma unroll
                for (int a = 0; a < XA; ++a)
#pragma unroll
                    for (int c = 0; c <= MC; ++c) S.Hb[dl][0][a][c] = I[a][c];
#pragma unroll
                for (int b = 0; b + 1 < XB; ++b) {
#pragma unroll
                    for (int a = 0; a + 1 <= MA - b; ++a)
#pragma unroll
                        for (int c = 0; c <= MC; ++c) I[a][c] = I[a + 1][c] + ABd * I[a][c];
#pragma unroll
                    for (int a = 0; a < XA && a <= MA - b - 1; ++a)
#pragma unroll
                        for (int c = 0; c <= MC; ++c) S.Hb[dl][b + 1][a][c] = I[a][c];
                }
            }
            __syncwarp();
            // transfers to centre 4, one (direction, a, b) row per lane
            for (int job = lane; job < 3 * XA * XB; job += 32) {
                const int d = job / (XA * XB), a = (job / XB) % XA, b = job % XB;
                if (a + b > MA) continue;
                const double CD = d == 0 ? Cr[0] : (d == 1 ? Cr[1] : Cr[2]);
                double Hd[MC + 1];
#pragma unroll
                for (int c = 0; c <= MC; ++c) Hd[c] = S.Hb[d][b][a][c];
#pragma unroll
                for (int c = 0; c < XC; ++c) S.X[d][a][b][c][0] = Hd[c];
#pragma unroll
                for (int e = 0; e + 1 < XE; ++e) {
#pragma unroll
                    for (int c = 0; c + 1 <= MC - e; ++c) Hd[c] = Hd[c + 1] + CD * Hd[c];
#pragma unroll
                    for (int c = 0; c < XC && c <= MC - e - 1; ++c) S.X[d][a][b][c][e + 1] = Hd[c];
                }
            }
            __syncwarp();
            // the integrals and their derivatives at the (a, b, c, e) of the contraction
            constexpr int SG = Tab::SG, S2 = L2 + 1, S3 = L3 + 1, S4 = L4 + 1;
            for (int idx = lane; idx < 3 * SG; idx += 32) {
                const int d = idx / SG, rr = idx - d * SG;
                const int e = rr % S4, c = (rr / S4) % S3, b = (rr / (S4 * S3)) % S2, a = rr / (S4 * S3 * S2);
                double da = 2.0 * alpha * S.X[d][a + 1][b][c][e];
                if (a) da -= a * S.X[d][a - 1][b][c][e];
                double db = 2.0 * beta * S.X[d][a][b + 1][c][e];
                if (b) db -= b * S.X[d][a][b - 1][c][e];
                double dc = 2.0 * gamma * S.X[d][a][b][c + 1][e];
                if (c) dc -= c * S.X[d][a][b][c - 1][e];
                double* o = S.T4[d][rr];
                o[0] = S.X[d][a][b][c][e];
                o[1] = da;
                o[2] = db;
                o[3] = dc;
            }
            __syncwarp();
            // the contraction: jobs (i1, i3, a range of i2) over the lanes, i4 innermost
#pragma unroll 1
            for (int k = 0; k < NJL; ++k) {
                const int job = lane + 32 * k;
                if (job >= NJOB) break;
                const int o13 = job / NPART, part = job % NPART;
                const double d13 = S.D13[o13];
                if (d13 == 0.0) continue;
                const int i1 = o13 / N3, i3 = o13 - (o13 / N3) * N3;
                const int x1 = cart_lx(L1, i1), y1 = cart_ly(L1, i1), z1 = cart_lz(L1, i1);
                const int x3 = cart_lx(L3, i3), y3 = cart_ly(L3, i3), z3 = cart_lz(L3, i3);
#pragma unroll 1
                for (int i2 = part * N2 / NPART; i2 < (part + 1) * N2 / NPART; ++i2) {
                    const int x2 = cart_lx(L2, i2), y2 = cart_ly(L2, i2), z2 = cart_lz(L2, i2);
                    const double(*tx)[4] = &S.T4[0][((x1 * S2 + x2) * S3 + x3) * S4];
                    const double(*ty)[4] = &S.T4[1][((y1 * S2 + y2) * S3 + y3) * S4];
                    const double(*tz)[4] = &S.T4[2][((z1 * S2 + z2) * S3 + z3) * S4];
                    const double* D24r = &S.D24[i2 * N4];
                    int i4 = 0;
#pragma unroll
                    for (int j4 = 0; j4 <= L4; ++j4)
#pragma unroll
                        for (int z4 = 0; z4 <= j4; ++z4, ++i4) {
                            const double W = d13 * D24r[i4];
                            const double* X4 = tx[L4 - j4];
                            const double* Y4 = ty[j4 - z4];
                            const double* Z4 = tz[z4];
                            const double yz = W * Y4[0] * Z4[0], xz = W * X4[0] * Z4[0], xy = W * X4[0] * Y4[0];
                            gA[0] = fma(X4[1], yz, gA[0]);
                            gA[1] = fma(Y4[1], xz, gA[1]);
                            gA[2] = fma(Z4[1], xy, gA[2]);
                            gB[0] = fma(X4[2], yz, gB[0]);
                            gB[1] = fma(Y4[2], xz, gB[1]);
                            gB[2] = fma(Z4[2], xy, gB[2]);
                            gC[0] = fma(X4[3], yz, gC[0]);
                            gC[1] = fma(Y4[3], xz, gC[1]);
                            gC[2] = fma(Z4[3], xy, gC[2]);
                        }
                }
            }
            __syncwarp();
        }
    }
}

// Heavy classes: the warp walks the task's passing (partner 1, partner 3)
// quartets one at a time (partners 3 outer, both rows in bound order, the same
// screens as k_exchange_grad) and computes each with kgrad_quartet_warp.
template <int L1, int L2, int L3, int L4>
__global__ void __launch_bounds__(128) k_exchange_grad_warp(const __grid_constant__ KGradArgs A)
{
    constexpr int N1 = ncart_of(L1), N2 = ncart_of(L2), N3 = ncart_of(L3), N4 = ncart_of(L4);
    // four warps' tables (dynamic: the f classes need more than 48 KB)
    extern __shared__ __align__(16) unsigned char kgrad_smem[];
    auto* tabs = reinterpret_cast<KGradWarpTables<L1, L2, L3, L4>*>(kgrad_smem);
    KGradWarpTables<L1, L2, L3, L4>& S = tabs[threadIdx.x >> 5];
    const int ntask = *A.ntask;
    const int lane = threadIdx.x & 31;
    const float thre12 = A.sc->thre12, thre34 = A.sc->thre34;
    for (;;) {
        // work unit: a task and one of A.stripes stripes of its partners 3
        int unit = 0;
        if (lane == 0) unit = (int) atomicAdd(A.queue, 1u);
        unit = __shfl_sync(0xffffffffu, unit, 0);
        if (unit >= ntask * A.stripes) break;
        const int t = unit / A.stripes, su = unit - t * A.stripes;
        const int ns3 = A.stripes < kGradStripes3 ? A.stripes : kGradStripes3, ns1 = A.stripes / ns3;
        const int stripe = su % ns3, stripe1 = su / ns3;   // partner-3 stripe, partner-1 stripe
        const KTask T = A.tasks[t];
        const int i2 = T.i2, i4 = T.i4;
        const float tlo = grad_threshold((double) A.thr_lo, T.dmax);
        const double dR[3] = {A.b2.x[i2] - A.b4.x[i4], A.b2.y[i2] - A.b4.y[i4], A.b2.z[i2] - A.b4.z[i4]};
        const double beta = A.b2.e[i2];
        const int c2 = A.b2.cart[i2], c4 = A.b4.cart[i4];
        const double w24 = (A.pairsym && i2 != i4) ? 2.0 : 1.0;   // a task and its mirror
        __syncwarp();   // the previous task's tables have been read
        for (int idx = lane; idx < N2 * N4; idx += 32)
            S.D24[idx] = w24 * A.D24[(long) (c2 + idx / N4) * A.ld24 + c4 + idx % N4];
        const int s12 = A.r12s[i2], n12 = A.r12l[i2], s34 = A.r34s[i4], n34 = A.r34l[i4];
        const float b12max = A.b12[s12];
        double gB[3] = {0, 0, 0}, gD[3] = {0, 0, 0};
        for (int k = stripe; k < n34; k += ns3) {
            const int k3 = s34 + k;
            const float b34 = A.b34[k3];
            if (b34 < thre34 || b12max * b34 < tlo) break;   // bound order: nothing later passes
            const double kab34 = A.kab34[k3], q = A.p34[k3], iq = A.ip34[k3], gamma = A.pe34[k3];
            const double Q[3] = {A.px34[k3], A.py34[k3], A.pz34[k3]};
            const double Cr[3] = {A.ax34[k3], A.ay34[k3], A.az34[k3]};
            double QC[3], Qs[3];
            for (int d = 0; d < 3; ++d) {
                QC[d] = Q[d] - Cr[d];
                Qs[d] = dR[d] - Q[d];
            }
            const int c3 = A.cart34[k3], atomC = A.atom34[k3], K3 = A.pidx34[k3];
            double gC[3] = {0, 0, 0};
            for (int j = stripe1; j < n12; j += ns1) {
                const int e = s12 + j;
                const float b12 = A.b12[e];
                if (b12 < thre12 || b12 * b34 < tlo) break;
                if (A.canon) {
                    const int K1 = A.pidx12[e];
                    const int r2 = K1 > i2 ? K1 : i2, r4 = K3 > i4 ? K3 : i4;
                    if ((double) (b12 * b34) * A.dblk[(long) r2 * A.nprim + r4] < (double) A.thr_lo) continue;
                }
                const double P[3] = {A.px12[e], A.py12[e], A.pz12[e]};
                const double Ar[3] = {A.ax12[e], A.ay12[e], A.az12[e]};
                const int c1 = A.cart12[e];
                __syncwarp();   // the previous quartet's D13 has been read
                for (int idx = lane; idx < N1 * N3; idx += 32)
                    S.D13[idx] = A.D13[(long) (c1 + idx / N3) * A.ld13 + c3 + idx % N3];
                __syncwarp();
                double qa[3] = {0, 0, 0}, qb[3] = {0, 0, 0}, qc[3] = {0, 0, 0};
                kgrad_quartet_warp<L1, L2, L3, L4>(A, S, lane, A.pe12[e], beta, gamma, A.kab12[e], A.p12[e],
                                                   A.ip12[e], P, Ar, kab34, q, iq, Qs, QC, Cr, qa, qb, qc);
                const int atomA = A.atom12[e];
                for (int d = 0; d < 3; ++d) {
                    const double sa = warp_sum(qa[d]);
                    if (lane == 0 && sa != 0.0) atomicAdd(&A.G[3 * atomA + d], sa);
                    gB[d] += qb[d];
                    gC[d] += qc[d];
                    gD[d] -= qa[d] + qb[d] + qc[d];   // translational invariance
                }
            }
            for (int d = 0; d < 3; ++d) {
                const double sc = warp_sum(gC[d]);
                if (lane == 0 && sc != 0.0) atomicAdd(&A.G[3 * atomC + d], sc);
            }
        }
        for (int d = 0; d < 3; ++d) {
            const double sb = warp_sum(gB[d]), sd = warp_sum(gD[d]);
            if (lane == 0) {
                if (sb != 0.0) atomicAdd(&A.G[3 * A.b2.atom[i2] + d], sb);
                if (sd != 0.0) atomicAdd(&A.G[3 * A.b4.atom[i4] + d], sd);
            }
        }
    }
}

template <int L1, int L2, int L3, int L4>
void launch_one(Context* ctx, const KGradArgs& A, long cap)
{
    const unsigned grid = (unsigned) std::min<long>((cap + 3) / 4, (long) ctx->nsm * 8);
    if constexpr (kgrad_warp<L1, L2, L3, L4>()) {
        constexpr size_t smem = 4 * sizeof(KGradWarpTables<L1, L2, L3, L4>);
        auto kern = k_exchange_grad_warp<L1, L2, L3, L4>;
        if constexpr (smem > 48 * 1024) {
            // the opt-in is a per-device function attribute: set it once per device
            static std::atomic<unsigned long long> devices{0};
            const unsigned long long bit = 1ull << (ctx->device & 63);
            if (!(devices.load(std::memory_order_acquire) & bit)) {
                LSJK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
                devices.fetch_or(bit, std::memory_order_acq_rel);
            }
        }
        // work units per task: at least 8 partner-3 stripes (long rows split for the load
        // balance), up to about 64 units per SM when the class has few tasks (up to 32
        // partner-3 stripes, then partner-1 stripes as well)
        KGradArgs B = A;
        const long want = 64L * ctx->nsm;
        B.stripes = (int) std::max<long>(8, std::min<long>(kGradStripesMax, (want + cap - 1) / std::max(1L, cap)));
        if (B.stripes > kGradStripes3) B.stripes -= B.stripes % kGradStripes3;   // whole partner-1 stripes
        const unsigned gw = (unsigned) std::min<long>((cap * B.stripes + 3) / 4, (long) ctx->nsm * 16);
        kern<<<gw, 128, smem, ctx->stream>>>(B);
    } else
        k_exchange_grad<L1, L2, L3, L4><<<grid, 128, 0, ctx->stream>>>(A);
    LSJK_CUDA(cudaGetLastError());
    ctx->stats.kernel_launches++;
}

template <int L1, int L2, int L3>
void launch4(Context* ctx, const KGradArgs& A, long cap, int L4)
{
    switch (L4) {
    case 0: launch_one<L1, L2, L3, 0>(ctx, A, cap); break;
    case 1: launch_one<L1, L2, L3, 1>(ctx, A, cap); break;
    case 2: launch_one<L1, L2, L3, 2>(ctx, A, cap); break;
    case 3: launch_one<L1, L2, L3, 3>(ctx, A, cap); break;
    default: throw Error(LSJK_ENOTSUPP, "K gradient: shell above f");
    }
}
template <int L1, int L2>
void launch3(Context* ctx, const KGradArgs& A, long cap, int L3, int L4)
{
    switch (L3) {
    case 0: launch4<L1, L2, 0>(ctx, A, cap, L4); break;
    case 1: launch4<L1, L2, 1>(ctx, A, cap, L4); break;
    case 2: launch4<L1, L2, 2>(ctx, A, cap, L4); break;
    case 3: launch4<L1, L2, 3>(ctx, A, cap, L4); break;
    default: throw Error(LSJK_ENOTSUPP, "K gradient: shell above f");
    }
}
template <int L1>
void launch2(Context* ctx, const KGradArgs& A, long cap, int L2, int L3, int L4)
{
    switch (L2) {
    case 0: launch3<L1, 0>(ctx, A, cap, L3, L4); break;
    case 1: launch3<L1, 1>(ctx, A, cap, L3, L4); break;
    case 2: launch3<L1, 2>(ctx, A, cap, L3, L4); break;
    case 3: launch3<L1, 3>(ctx, A, cap, L3, L4); break;
    default: throw Error(LSJK_ENOTSUPP, "K gradient: shell above f");
    }
}

} // namespace

// This unit holds the classes with partner-1 shell LSJK_KG_L1 (the build compiles
// it once per shell, so the classes compile in parallel).
template <int L1>
void launch_k_grad_l1(Context* ctx, const KGradArgs& A, long cap, int L2, int L3, int L4)
{
    launch2<L1>(ctx, A, cap, L2, L3, L4);
}
template void launch_k_grad_l1<LSJK_KG_L1>(Context*, const KGradArgs&, long, int, int, int);

#if LSJK_KG_L1 == 0
void launch_k_grad(Context* ctx, const KGradArgs& A, long cap, int L1, int L2, int L3, int L4)
{
    if (cap == 0) return;
    switch (L1) {
    case 0: launch_k_grad_l1<0>(ctx, A, cap, L2, L3, L4); break;
    case 1: launch_k_grad_l1<1>(ctx, A, cap, L2, L3, L4); break;
    case 2: launch_k_grad_l1<2>(ctx, A, cap, L2, L3, L4); break;
    case 3: launch_k_grad_l1<3>(ctx, A, cap, L2, L3, L4); break;
    default: throw Error(LSJK_ENOTSUPP, "K gradient: shell above f");
    }
}
#endif

} // namespace lsjk
