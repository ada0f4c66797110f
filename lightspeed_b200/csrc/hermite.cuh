// McMurchie-Davidson Hermite expansion coefficients of a primitive pair and
// the transforms between a Cartesian pair block and its Hermite coefficients.
//
//   E^{i+1,j}_t = E^{ij}_{t-1}/(2p) + X_PA E^{ij}_t + (t+1) E^{ij}_{t+1}
//   E^{i,j+1}_t = E^{ij}_{t-1}/(2p) + X_PB E^{ij}_t + (t+1) E^{ij}_{t+1}
//   E^{00}_0 = 1
// The reference evaluates the same coefficients by Gauss-Hermite quadrature
// (src/cpp/core/hermite.cpp:84-134); the recursion is exact.
#pragma once
#include "lsjk_device.cuh"

namespace lsjk {

template <int LA, int LB>
struct ECoef {
    static constexpr int V = LA + LB + 1;
    double v[3][LA + 1][LB + 1][V];
};

template <int LA, int LB>
__device__ __forceinline__ void build_E(double p, const double PA[3], const double PB[3], ECoef<LA, LB>& E)
{
    constexpr int V = LA + LB + 1;
    const double h = 0.5 / p;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
#pragma unroll
        for (int i = 0; i <= LA; ++i)
#pragma unroll
            for (int j = 0; j <= LB; ++j)
#pragma unroll
                for (int t = 0; t < V; ++t) E.v[d][i][j][t] = 0.0;
        E.v[d][0][0][0] = 1.0;
#pragma unroll
        for (int i = 0; i < LA; ++i)
#pragma unroll
            for (int t = 0; t <= i + 1; ++t) {
                double s = PA[d] * E.v[d][i][0][t];
                if (t > 0) s += h * E.v[d][i][0][t - 1];
                if (t + 1 <= i) s += (t + 1) * E.v[d][i][0][t + 1];
                E.v[d][i + 1][0][t] = s;
            }
#pragma unroll
        for (int j = 0; j < LB; ++j)
#pragma unroll
            for (int i = 0; i <= LA; ++i)
#pragma unroll
                for (int t = 0; t <= i + j + 1; ++t) {
                    double s = PB[d] * E.v[d][i][j][t];
                    if (t > 0) s += h * E.v[d][i][j][t - 1];
                    if (t + 1 <= i + j) s += (t + 1) * E.v[d][i][j][t + 1];
                    E.v[d][i][j + 1][t] = s;
                }
    }
}

// Cartesian exponents of component k of a shell (CCA lexical order).
__host__ __device__ constexpr int cart_lx(int L, int k)
{
    int i = 0;
    while ((i + 1) * (i + 2) / 2 <= k) ++i;
    return L - i;
}
__host__ __device__ constexpr int cart_lz(int L, int k)
{
    int i = 0;
    while ((i + 1) * (i + 2) / 2 <= k) ++i;
    return k - i * (i + 1) / 2;
}
__host__ __device__ constexpr int cart_ly(int L, int k) { return L - cart_lx(L, k) - cart_lz(L, k); }

// Hermite index t -> (tx, ty, tz) in shell-major lexical order.
__host__ __device__ constexpr int herm_shell(int t)
{
    int L = 0;
    while ((L + 1) * (L + 2) * (L + 3) / 6 <= t) ++L;
    return L;
}
__host__ __device__ constexpr int herm_tx(int t)
{
    return cart_lx(herm_shell(t), t - herm_shell(t) * (herm_shell(t) + 1) * (herm_shell(t) + 2) / 6);
}
__host__ __device__ constexpr int herm_ty(int t)
{
    return cart_ly(herm_shell(t), t - herm_shell(t) * (herm_shell(t) + 1) * (herm_shell(t) + 2) / 6);
}
__host__ __device__ constexpr int herm_tz(int t)
{
    return cart_lz(herm_shell(t), t - herm_shell(t) * (herm_shell(t) + 1) * (herm_shell(t) + 2) / 6);
}

} // namespace lsjk
