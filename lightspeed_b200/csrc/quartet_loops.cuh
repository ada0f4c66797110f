// Loop forms of the per-quartet integral code, for the classes the generator
// does not emit as straight-line code (the largest classes with an f shell; see
// gen_kernels.py). The J kernel of those classes builds the same table per warp
// (k_coulomb_warp); the K ones mostly run k_exchange_warp.
// They compute the same quantities with the same recursions as the generated
// functions (gen_kernels.py), over index loops into per-thread arrays, so a
// class of any angular momentum compiles to a compact kernel:
//
//  * JQLoop<LB, LK>: Hermite integrals R_tuv of order LB + LK from the scaled
//    Boys values a_n by the downward recursion in n, one shell of (t, u, v) at
//    a time, top shell first, in place:
//        R^{(n)}_{t,u,v} = (t-1) R^{(n+1)}_{t-2,u,v} + X R^{(n+1)}_{t-1,u,v}
//    (in y, z likewise when t = 0), then jp[t] += sum_u R_{t+u} dk[u];
//  * KQLoop<L1, L2, L3, L4>: one Rys root of a quartet: the 2-D integrals by the
//    vertical recursion, the transfer to centre 2 and then to centre 4, and the
//    contraction K[i1, i3] += sum_{i2, i4} Ix Iy Iz D[i2, i4].
#pragma once
#include "lsjk_device.cuh"

namespace lsjk {

// Position of the Hermite function (t, u, v) in shell-major lexical order.
__host__ __device__ constexpr int herm_pos(int t, int u, int v)
{
    const int N = t + u + v, i = u + v;
    return nherm_of(N - 1) + i * (i + 1) / 2 + v;
}

template <int LB, int LK>
struct JQLoop {
    static constexpr bool loop = true;   // the class has no straight-line code
    template <typename R>
    __device__ static void run(const R* __restrict__ a, R X, R Y, R Z, const R* __restrict__ dk,
                               R* __restrict__ jp)
    {
        constexpr int L = LB + LK;
        R buf[nherm_of(L)];
        buf[0] = a[L];
#pragma unroll 1
        for (int m = L - 1; m >= 0; --m) {
            // level m from level m + 1: shells N = L - m .. 1 read shells N - 1, N - 2,
            // which still hold level m + 1 when the top shell goes first
#pragma unroll 1
            for (int N = L - m; N >= 1; --N) {
                int k = nherm_of(N - 1);
#pragma unroll 1
                for (int i = 0; i <= N; ++i)
#pragma unroll 1
                    for (int v = 0; v <= i; ++v, ++k) {
                        const int t = N - i, u = i - v;
                        R s;
                        if (t > 0) {
                            s = X * buf[herm_pos(t - 1, u, v)];
                            if (t > 1) s = fma(R(t - 1), buf[herm_pos(t - 2, u, v)], s);
                        } else if (u > 0) {
                            s = Y * buf[herm_pos(t, u - 1, v)];
                            if (u > 1) s = fma(R(u - 1), buf[herm_pos(t, u - 2, v)], s);
                        } else {
                            s = Z * buf[herm_pos(t, u, v - 1)];
                            if (v > 1) s = fma(R(v - 1), buf[herm_pos(t, u, v - 2)], s);
                        }
                        buf[k] = s;
                    }
            }
            buf[0] = a[m];
        }
        int tb = 0;
#pragma unroll 1
        for (int NB = 0; NB <= LB; ++NB)
#pragma unroll 1
            for (int ib = 0; ib <= NB; ++ib)
#pragma unroll 1
                for (int vb = 0; vb <= ib; ++vb, ++tb) {
                    const int xb = NB - ib, yb = ib - vb;
                    R s = jp[tb];
                    int uk = 0;
#pragma unroll 1
                    for (int NK = 0; NK <= LK; ++NK)
#pragma unroll 1
                        for (int ik = 0; ik <= NK; ++ik)
#pragma unroll 1
                            for (int vk = 0; vk <= ik; ++vk, ++uk)
                                s = fma(buf[herm_pos(xb + NK - ik, yb + ik - vk, vb + vk)], dk[uk], s);
                    jp[tb] = s;
                }
    }
};

template <int L1, int L2, int L3, int L4>
struct KQLoop {
    template <typename R>
    __device__ static void run(R c00x, R c00y, R c00z, R d00x, R d00y, R d00z, R b00, R b10, R b01, R abx, R aby,
                               R abz, R cdx, R cdy, R cdz, R wz, const R* __restrict__ D, R* __restrict__ K)
    {
        constexpr int LA = L1 + L2, LC = L3 + L4;
        constexpr int S2 = L2 + 1, S3 = L3 + 1, S4 = L4 + 1, SG = (L1 + 1) * S2 * S3 * S4;
        constexpr int NC = LC + 1;
        constexpr int N2 = ncart_of(L2), N3 = ncart_of(L3), N4 = ncart_of(L4);
        R G[3][SG];
#pragma unroll 1
        for (int d = 0; d < 3; ++d) {
            const R c00 = d == 0 ? c00x : (d == 1 ? c00y : c00z);
            const R d00 = d == 0 ? d00x : (d == 1 ? d00y : d00z);
            const R ab = d == 0 ? abx : (d == 1 ? aby : abz);
            const R cd = d == 0 ? cdx : (d == 1 ? cdy : cdz);
            // H[b][a][c]: the 2-D integrals I(a, c) (b = 0), then moved to centre 2
            R H[L2 + 1][LA + 1][NC];
            H[0][0][0] = d == 2 ? wz : R(1);
#pragma unroll 1
            for (int a = 1; a <= LA; ++a) {
                R s = c00 * H[0][a - 1][0];
                if (a > 1) s = fma(R(a - 1) * b10, H[0][a - 2][0], s);
                H[0][a][0] = s;
            }
#pragma unroll 1
            for (int c = 1; c <= LC; ++c)
#pragma unroll 1
                for (int a = 0; a <= LA; ++a) {
                    R s = d00 * H[0][a][c - 1];
                    if (c > 1) s = fma(R(c - 1) * b01, H[0][a][c - 2], s);
                    if (a > 0) s = fma(R(a) * b00, H[0][a - 1][c - 1], s);
                    H[0][a][c] = s;
                }
#pragma unroll 1
            for (int b = 1; b <= L2; ++b)
#pragma unroll 1
                for (int a = 0; a <= LA - b; ++a)
#pragma unroll 1
                    for (int c = 0; c <= LC; ++c) H[b][a][c] = fma(ab, H[b - 1][a][c], H[b - 1][a + 1][c]);
            // then to centre 4, for each (a <= L1, b <= L2)
#pragma unroll 1
            for (int a = 0; a <= L1; ++a)
#pragma unroll 1
                for (int b = 0; b <= L2; ++b) {
                    R T[L4 + 1][NC];
#pragma unroll 1
                    for (int c = 0; c <= LC; ++c) T[0][c] = H[b][a][c];
#pragma unroll 1
                    for (int e = 1; e <= L4; ++e)
#pragma unroll 1
                        for (int c = 0; c <= LC - e; ++c) T[e][c] = fma(cd, T[e - 1][c], T[e - 1][c + 1]);
#pragma unroll 1
                    for (int c = 0; c <= L3; ++c)
#pragma unroll 1
                        for (int e = 0; e <= L4; ++e) G[d][((a * S2 + b) * S3 + c) * S4 + e] = T[e][c];
                }
        }
        // K[i1, i3] += sum_{i2, i4} Gx Gy Gz D[i2, i4] (Cartesian components in CCA order)
        int i1 = 0;
#pragma unroll 1
        for (int j1 = 0; j1 <= L1; ++j1)
#pragma unroll 1
            for (int z1 = 0; z1 <= j1; ++z1, ++i1) {
                const int x1 = L1 - j1, y1 = j1 - z1;
                int i3 = 0;
#pragma unroll 1
                for (int j3 = 0; j3 <= L3; ++j3)
#pragma unroll 1
                    for (int z3 = 0; z3 <= j3; ++z3, ++i3) {
                        const int x3 = L3 - j3, y3 = j3 - z3;
                        R s = K[i1 * N3 + i3];
                        int i2 = 0;
#pragma unroll 1
                        for (int j2 = 0; j2 <= L2; ++j2)
#pragma unroll 1
                            for (int z2 = 0; z2 <= j2; ++z2, ++i2) {
                                const int x2 = L2 - j2, y2 = j2 - z2;
                                const int gx = (x1 * S2 + x2) * S3 + x3, gy = (y1 * S2 + y2) * S3 + y3,
                                          gz = (z1 * S2 + z2) * S3 + z3;
                                int i4 = 0;
#pragma unroll 1
                                for (int j4 = 0; j4 <= L4; ++j4)
#pragma unroll 1
                                    for (int z4 = 0; z4 <= j4; ++z4, ++i4) {
                                        const int x4 = L4 - j4, y4 = j4 - z4;
                                        const R v = G[0][gx * S4 + x4] * G[1][gy * S4 + y4] * G[2][gz * S4 + z4];
                                        s = fma(v, D[i2 * N4 + i4], s);
                                    }
                            }
                        K[i1 * N3 + i3] = s;
                    }
            }
        (void) N2;
    }
};

} // namespace lsjk
