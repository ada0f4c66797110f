// The J kernel: one template per Hermite class pair (LB|LK), instantiated in
// jinst.cu (compiled once per LB) so the classes build in parallel.
#pragma once
#include "engine.cuh"
#include "lsjk_device.cuh"
#include "generated/jquartets.cuh"
#include "jargs.cuh"

namespace lsjk {




template <int LB, int LK>
__global__ void __launch_bounds__(kJThreads) k_coulomb(JArgs A)
{
    constexpr int L = LB + LK, HB = nherm_of(LB), S = 4 + nherm_of(LK);
    __shared__ __align__(128) double tab[LSJK_BOYS_NBIN * 8];
    __shared__ __align__(8) uint64_t mbar;
    const int nb = *A.nbra, nk = *A.nket;
    const int i0 = blockIdx.x * kJThreads;
    const int j0 = blockIdx.y * kJChunk;
    if (i0 >= nb || j0 >= nk) return;
    const float B0 = A.bbound[i0];
    if (B0 * A.kbound[j0] < A.thresp) return;
    if (!stage_bulk(tab, A.boys, sizeof(tab), &mbar, A.status)) return;

    const int i = i0 + threadIdx.x;
    const bool act = i < nb;
    double p = 1.0, Px = 0.0, Py = 0.0, Pz = 0.0;
    float Bi = 0.0f;
    if (act) {
        p = A.bgeom[4L * i];
        Px = A.bgeom[4L * i + 1];
        Py = A.bgeom[4L * i + 2];
        Pz = A.bgeom[4L * i + 3];
        Bi = A.bbound[i];
    }
    double jp[HB];
#pragma unroll
    for (int t = 0; t < HB; ++t) jp[t] = 0.0;
    long nq = 0;
    const int j1 = min(j0 + kJChunk, nk);
    for (int j = j0; j < j1; ++j) {
        const float Bj = A.kbound[j];
        if (B0 * Bj < A.thresp) break;
        if (!act || Bi * Bj < A.thresp) continue;
        ++nq;
        const double* r = A.krec + (long) j * S;
        const double q = r[0];
        const double X = Px - r[1], Y = Py - r[2], Z = Pz - r[3];
        const double R2 = X * X + Y * Y + Z * Z;
        const double rs = rsqrt(p + q);
        const double rho = p * q * (rs * rs);
        for (int tm = 0; tm < A.nterm; ++tm) {
            const double om = A.omega[tm];
            double d2 = 1.0, f = A.alpha[tm] * rs;
            if (om != -1.0) {
                const double w2 = om * om;
                d2 = w2 / (rho + w2);
                f *= sqrt(d2);
            }
            const double rhoe = rho * d2;
            double F[L + 1];
            boys_eval<L, double>(rhoe * R2, tab, F);
            double a[L + 1];
            const double m2r = -2.0 * rhoe;
            double pw = f;
#pragma unroll
            for (int n = 0; n <= L; ++n) {
                a[n] = pw * F[n];
                pw *= m2r;
            }
            jq_dispatch<LB, LK>(a, X, Y, Z, r + 4, jp);
        }
    }
    if (act) {
#pragma unroll
        for (int t = 0; t < HB; ++t)
            if (jp[t] != 0.0) atomicAdd(&A.jbra[(long) i * HB + t], jp[t]);
    }
    // quartet count for the statistics
    for (int o = 16; o > 0; o >>= 1) nq += __shfl_xor_sync(0xffffffffu, nq, o);
    if ((threadIdx.x & 31) == 0 && nq) atomicAdd(A.qcount, (unsigned long long) nq);
}


template <int LB, int LK>
void launch_j(Context* ctx, const JArgs& A, int nbra_full, int nket_full)
{
    if (nbra_full == 0 || nket_full == 0) return;
    dim3 grid((nbra_full + kJThreads - 1) / kJThreads, (nket_full + kJChunk - 1) / kJChunk);
    k_coulomb<LB, LK><<<grid, kJThreads, 0, ctx->stream>>>(A);
    LSJK_CUDA(cudaGetLastError());
    ctx->stats.kernel_launches++;
}


} // namespace lsjk
