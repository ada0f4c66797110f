// The J kernel: one template per Hermite class pair (LB|LK), instantiated in
// jinst.cu (compiled once per LB) so the classes build in parallel.
#pragma once
#include "engine.cuh"
#include "lsjk_device.cuh"
#include "generated/jquartets.cuh"
#include "jargs.cuh"

namespace lsjk {




// One J quartet (bra pair in registers, ket record r whose header q, Q the
// caller has already loaded) accumulated into jp, for the NG densities of the
// record (the Hermite integrals R_tuv are shared).
template <int LB, int LK, int NG>
__device__ __forceinline__ void j_quartet64(const JArgs& A, int g0, const double* tab, double p, double Px, double Py,
                                            double Pz, double q, double Qx, double Qy, double Qz,
                                            const double* __restrict__ r, double (*jp)[nherm_of(LB)])
{
    constexpr int L = LB + LK, HK = nherm_of(LK);
    const double X = Px - Qx, Y = Py - Qy, Z = Pz - Qz;
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
#pragma unroll
        for (int g = 0; g < NG; ++g)
            if (g0 + g < A.ng) jq_dispatch<LB, LK>(a, X, Y, Z, r + 4 + (g0 + g) * HK, jp[g]);
    }
}

// Densities per CTA for a bra class: the batched kernel keeps NG x HB FP64
// accumulators per thread (and as many FP32 ones), so the heavy bra classes
// take fewer densities per CTA (more CTA z-slices over the same ket records)
// instead of spilling.
template <int LB>
__host__ __device__ constexpr int j_batch() { return nherm_of(LB) <= 4 ? kJBatch : (nherm_of(LB) <= 10 ? 2 : 1); }

// Start of the last bin of the Boys table: from here on (the bin next to the
// switch to the asymptotic form, and the asymptotic region itself) the FP32
// path evaluates the Boys function in FP64 by its asymptotic form.
constexpr float kBoysSwitch32 = (float) (LSJK_BOYS_TMAX - LSJK_BOYS_TMAX / LSJK_BOYS_NBIN);

// The same quartet in FP32 (geometry differences formed in FP64, everything
// else in FP32 except the Boys function at T >= kBoysSwitch32, which is
// evaluated in FP64 by its asymptotic form), added to the FP64 accumulators.
template <int LB, int LK, int NG>
__device__ __forceinline__ void j_quartet32(const JArgs& A, int g0, const float* tab, float p,
                                            double Px, double Py, double Pz, double qd, double Qx, double Qy,
                                            double Qz, const float* __restrict__ r32, double (*jp)[nherm_of(LB)])
{
    constexpr int L = LB + LK, HB = nherm_of(LB), HK = nherm_of(LK);
    const float q = (float) qd;   // the FP32 record's q is this rounding
    const double Xd = Px - Qx, Yd = Py - Qy, Zd = Pz - Qz;
    const float X = (float) Xd, Y = (float) Yd, Z = (float) Zd;
    const float R2 = X * X + Y * Y + Z * Z;
    const float rs = rsqrtf(p + q);
    const float rho = p * q * (rs * rs);
    float jq[NG][HB];
#pragma unroll
    for (int g = 0; g < NG; ++g)
#pragma unroll
        for (int t = 0; t < HB; ++t) jq[g][t] = 0.0f;
    for (int tm = 0; tm < A.nterm; ++tm) {
        const float om = (float) A.omega[tm];
        float d2 = 1.0f, f = (float) A.alpha[tm] * rs;
        if (A.omega[tm] != -1.0) {
            const float w2 = om * om;
            d2 = w2 / (rho + w2);
            f *= sqrtf(d2);
        }
        const float rhoe = rho * d2;
        float F[L + 1];
        const float T = rhoe * R2;
        if (T < kBoysSwitch32) {
            boys_eval<L, float>(T, tab, F);
        } else {
            boys_asym_f64_to_f32<L>((double) rhoe * (Xd * Xd + Yd * Yd + Zd * Zd), F);
        }
        float a[L + 1];
        const float m2r = -2.0f * rhoe;
        float pw = f;
#pragma unroll
        for (int n = 0; n <= L; ++n) {
            a[n] = pw * F[n];
            pw *= m2r;
        }
#pragma unroll
        for (int g = 0; g < NG; ++g)
            if (g0 + g < A.ng) jq_dispatch<LB, LK>(a, X, Y, Z, r32 + 4 + (g0 + g) * HK, jq[g]);
    }
#pragma unroll
    for (int g = 0; g < NG; ++g)
#pragma unroll
        for (int t = 0; t < HB; ++t) jp[g][t] += (double) jq[g][t];
}

template <int LB, int LK, int NG>
__global__ void __launch_bounds__(kJThreads) k_coulomb(JArgs A)
{
    constexpr int HB = nherm_of(LB), HK = nherm_of(LK);
    const int S = 4 + A.slots * HK;              // doubles (floats) per ket record
    __shared__ __align__(128) double tab[LSJK_BOYS_NBIN * 8];
    __shared__ __align__(128) float tab32[LSJK_BOYS_NBIN * 8];
    __shared__ __align__(8) uint64_t mbar[2];
    const int nb = *A.nbra, nk = *A.nket;
    const int g0 = blockIdx.z * NG;   // the densities g0 .. g0 + NG - 1 of the build
    const int i0 = blockIdx.x * kJThreads;
    const int j0 = blockIdx.y * A.chunk;
    if (i0 >= nb || j0 >= nk) return;
    const float B0 = A.bbound[i0];
    if (B0 * A.kbound[j0] < A.thresp) return;
    if (!stage_bulk(tab, A.boys, sizeof(tab), &mbar[0], A.status)) return;
    if (A.mixed && !stage_bulk(tab32, A.boys32, sizeof(tab32), &mbar[1], A.status)) return;

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
    const float p32 = (float) p;
    const float thr_dp = A.mixed ? A.thredp : 0.0f;
    double jp[NG][HB];
#pragma unroll
    for (int g = 0; g < NG; ++g)
#pragma unroll
        for (int t = 0; t < HB; ++t) jp[g][t] = 0.0;
    long nq = 0, nq32 = 0;
    const int nd = min(NG, A.ng - g0);   // statistics count density-quartets
    const int j1 = min(j0 + A.chunk, nk);
    // the next ket's bound and record header are loaded one iteration ahead, so
    // their latency overlaps the current quartet (all lanes read the same ket)
    float Bn = A.kbound[j0];
    double qn, Qxn, Qyn, Qzn;
    {
        const double* r = A.krec + (long) j0 * S;
        qn = r[0];
        Qxn = r[1];
        Qyn = r[2];
        Qzn = r[3];
    }
    for (int j = j0; j < j1; ++j) {
        const float Bj = Bn;
        const double qk = qn, Qx = Qxn, Qy = Qyn, Qz = Qzn;
        if (B0 * Bj < A.thresp) break;
        if (j + 1 < j1) {
            const double* rn = A.krec + (long) (j + 1) * S;
            Bn = A.kbound[j + 1];
            qn = rn[0];
            Qxn = rn[1];
            Qyn = rn[2];
            Qzn = rn[3];
        }
        const float est = Bi * Bj;
        const bool pass = act && est >= A.thresp;
        // one precision per warp and ket: FP64 while any lane's estimate reaches thredp
        // (those lanes need it; the others get FP64 too rather than a second, FP32
        // pass of the warp over the same ket), FP32 after. The kets are in bound
        // order, so the warp switches once.
        const bool dp = __any_sync(0xffffffffu, pass && est >= thr_dp);
        const double* r = A.krec + (long) j * S;
        if (dp) {
            if (pass) {
                nq += nd;
                j_quartet64<LB, LK, NG>(A, g0, tab, p, Px, Py, Pz, qk, Qx, Qy, Qz, r, jp);
            }
        } else if (__any_sync(0xffffffffu, pass)) {
            if (pass) {
                nq32 += nd;
                j_quartet32<LB, LK, NG>(A, g0, tab32, p32, Px, Py, Pz, qk, Qx, Qy, Qz, A.krec32 + (long) j * S,
                                        jp);
            }
        }
    }
    if (act) {
#pragma unroll
        for (int g = 0; g < NG; ++g)
#pragma unroll
            for (int t = 0; t < HB; ++t) {
                const double v = jp[g][t];
                if (v != 0.0 && g0 + g < A.ng) atomicAdd(&A.jbra[(g0 + g) * A.jbra_stride + (long) i * HB + t], v);
            }
    }
    // quartet counts for the statistics
    for (int o = 16; o > 0; o >>= 1) {
        nq += __shfl_xor_sync(0xffffffffu, nq, o);
        nq32 += __shfl_xor_sync(0xffffffffu, nq32, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (nq) atomicAdd(A.qcount, (unsigned long long) nq);
        if (nq32) atomicAdd(A.qcount32, (unsigned long long) nq32);
    }
}

// The classes without straight-line code (the largest f classes): a bra pair per
// warp, FP64. For each ket (bound order, all lanes) the lanes build the Hermite
// integrals R_tuv in a per-warp shared table -- one shell of (t, u, v) at a time,
// top shell first, in place, as JQLoop does per thread -- and then each lane
// contracts its bra components t: jp[t] += sum_u R_{t+u} D_u. A thread-per-pair
// kernel needs the whole table and the accumulators per thread (several KB),
// which overflow L1 for 128 threads per CTA.
constexpr int kJWarpPairs = kJThreads / 32;   // bra pairs per CTA

template <int LB, int LK>
__global__ void __launch_bounds__(kJThreads) k_coulomb_warp(JArgs A)
{
    constexpr int L = LB + LK, HB = nherm_of(LB), HK = nherm_of(LK), NT = (HB + 31) / 32;
    const int S = 4 + A.slots * HK;
    __shared__ __align__(128) double tab[LSJK_BOYS_NBIN * 8];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ double Rall[kJWarpPairs][nherm_of(L)];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nb = *A.nbra, nk = *A.nket;
    const int g = blockIdx.z;   // the density (one per CTA z)
    const int ib = blockIdx.x * kJWarpPairs;
    const int j0 = blockIdx.y * A.chunk;
    if (ib >= nb || j0 >= nk) return;
    if (A.bbound[ib] * A.kbound[j0] < A.thresp) return;
    if (!stage_bulk(tab, A.boys, sizeof(tab), &mbar, A.status)) return;
    const int i = ib + warp;
    if (i >= nb) return;   // (after the CTA-wide staging)
    double* Rb = Rall[warp];
    const double p = A.bgeom[4L * i], Px = A.bgeom[4L * i + 1], Py = A.bgeom[4L * i + 2], Pz = A.bgeom[4L * i + 3];
    const float Bi = A.bbound[i];
    // this lane's bra components t = lane + 32 k
    int tx[NT], ty[NT], tz[NT];
    double jp[NT];
#pragma unroll
    for (int k = 0; k < NT; ++k) {
        const int t = lane + 32 * k < HB ? lane + 32 * k : 0;
        int N = 0;
        while (nherm_of(N) <= t) ++N;
        int r = t - nherm_of(N - 1), ii = 0;
        while ((ii + 1) * (ii + 2) / 2 <= r) ++ii;
        tz[k] = r - ii * (ii + 1) / 2;
        ty[k] = ii - tz[k];
        tx[k] = N - ii;
        jp[k] = 0.0;
    }
    long nq = 0;
    const int j1 = min(j0 + A.chunk, nk);
    for (int j = j0; j < j1; ++j) {
        if (Bi * A.kbound[j] < A.thresp) break;   // kets in bound order
        const double* r = A.krec + (long) j * S;
        const double q = r[0];
        const double X = Px - r[1], Y = Py - r[2], Z = Pz - r[3];
        const double R2 = X * X + Y * Y + Z * Z;
        const double rs = rsqrt(p + q);
        const double rho = p * q * (rs * rs);
        const double* dk = r + 4 + g * HK;
        ++nq;
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
            if (lane == 0) Rb[0] = a[L];
            __syncwarp();
#pragma unroll 1
            for (int m = L - 1; m >= 0; --m) {
#pragma unroll 1
                for (int N = L - m; N >= 1; --N) {
                    for (int k = lane; k < (N + 1) * (N + 2) / 2; k += 32) {
                        int ii = 0;
                        while ((ii + 1) * (ii + 2) / 2 <= k) ++ii;
                        const int v = k - ii * (ii + 1) / 2, u = ii - v, t = N - ii;
                        double sv;
                        if (t > 0) {
                            sv = X * Rb[herm_pos(t - 1, u, v)];
                            if (t > 1) sv = fma(double(t - 1), Rb[herm_pos(t - 2, u, v)], sv);
                        } else if (u > 0) {
                            sv = Y * Rb[herm_pos(t, u - 1, v)];
                            if (u > 1) sv = fma(double(u - 1), Rb[herm_pos(t, u - 2, v)], sv);
                        } else {
                            sv = Z * Rb[herm_pos(t, u, v - 1)];
                            if (v > 1) sv = fma(double(v - 1), Rb[herm_pos(t, u, v - 2)], sv);
                        }
                        Rb[nherm_of(N - 1) + k] = sv;
                    }
                    __syncwarp();
                }
                if (lane == 0) Rb[0] = a[m];
                __syncwarp();
            }
#pragma unroll
            for (int k = 0; k < NT; ++k) {
                if (lane + 32 * k >= HB) break;
                double sv = jp[k];
                int uk = 0;
#pragma unroll 1
                for (int NK = 0; NK <= LK; ++NK)
#pragma unroll 1
                    for (int ik = 0; ik <= NK; ++ik)
#pragma unroll 1
                        for (int vk = 0; vk <= ik; ++vk, ++uk)
                            sv = fma(Rb[herm_pos(tx[k] + NK - ik, ty[k] + ik - vk, tz[k] + vk)], dk[uk], sv);
                jp[k] = sv;
            }
            __syncwarp();   // the table is rebuilt for the next term or ket
        }
    }
#pragma unroll
    for (int k = 0; k < NT; ++k) {
        const int t = lane + 32 * k;
        if (t < HB && jp[k] != 0.0) atomicAdd(&A.jbra[g * A.jbra_stride + (long) i * HB + t], jp[k]);
    }
    if (lane == 0 && nq) atomicAdd(A.qcount, (unsigned long long) nq);
}

template <int LB, int LK>
void launch_j(Context* ctx, const JArgs& A, int nbra_full, int nket_full)
{
    if (nbra_full == 0 || nket_full == 0) return;
    if constexpr (JQ<LB, LK>::loop) {
        // classes without straight-line code: a bra pair per warp, FP64, a density per CTA z
        dim3 grid((nbra_full + kJWarpPairs - 1) / kJWarpPairs, (nket_full + A.chunk - 1) / A.chunk, A.ng);
        k_coulomb_warp<LB, LK><<<grid, kJThreads, 0, ctx->stream>>>(A);
        LSJK_CUDA(cudaGetLastError());
        ctx->stats.kernel_launches++;
        return;
    }
    // one launch for all densities: CTA z takes NG of them over the same ket
    // records (NG = the class's batch when there are that many, else 1)
    constexpr int NGB = j_batch<LB>();
    const bool batched = NGB > 1 && A.ng >= NGB;
    const int NG = batched ? NGB : 1;
    dim3 grid((nbra_full + kJThreads - 1) / kJThreads, (nket_full + A.chunk - 1) / A.chunk, (A.ng + NG - 1) / NG);
    if (batched)
        k_coulomb<LB, LK, NGB><<<grid, kJThreads, 0, ctx->stream>>>(A);
    else
        k_coulomb<LB, LK, 1><<<grid, kJThreads, 0, ctx->stream>>>(A);
    LSJK_CUDA(cudaGetLastError());
    ctx->stats.kernel_launches++;
}


} // namespace lsjk
