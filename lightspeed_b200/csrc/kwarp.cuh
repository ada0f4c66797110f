// The K kernel of the heavy classes with an f shell: one quartet per warp.
// Included by kkernel.cuh.
//
// A lane-per-quartet kernel needs, for (ff|ff), about 1.5 K doubles of 1-D
// integral tables per lane: 32 lanes' tables no longer fit the SM's L1 and
// the loop-form quartet runs out of L2. Here the warp shares one set of
// tables in shared memory and splits each quartet:
//   * the Rys roots and weights: every lane (the same values);
//   * per root, lanes 0-2 run the vertical recursion and the transfer to
//     centre 2 of one direction each; the transfers to centre 4 go one
//     (direction, a, b) row per lane;
//   * the contraction K[i1, i3] += sum_{i2, i4} Ix Iy Iz D[i2, i4] is split
//     into jobs (i1, i3, a range of i2) over the lanes; each lane keeps its
//     jobs' sums in registers over the partner-1 entries of a shell segment,
//     and at the segment's end the parts of an element are added in shared
//     memory and reach K with one atomic per element.
// Work order and screens are those of k_exchange (a (prim2, prim4) task per
// warp, here split into stripes of its partners 3; partners 3 outer, partners 1
// of each partner 3 in segment order), FP64 only, one density per task and
// sub-slot, partners with one output target.
#pragma once
#include "hermite.cuh"   // cart_lx/ly/lz

namespace lsjk {

// Classes that take this kernel: an f shell and at least 100 Cartesian
// combinations (below, a lane's tables still fit L1), and the classes of at
// least 600 ((dd|dd), (dd|dp) and the like: their straight-line FP64 quartets
// spill 5-29 KB per lane; from 324 on the FP64 build measured slower).
template <int L1, int L2, int L3, int L4>
__host__ __device__ constexpr bool k_warp_class()
{
    constexpr int nc = ncart_of(L1) * ncart_of(L2) * ncart_of(L3) * ncart_of(L4);
    return ((L1 > 2 || L2 > 2 || L3 > 2 || L4 > 2) && nc >= 100) || nc >= 600;
}

// The heavy classes without an f shell (at least 324 combinations) take it for the
// FP64 pass of a mixed build, whose few tasks (those that reach thredp) a quartet
// per lane spreads too thinly; their full FP64 builds stay a quartet per lane.
template <int L1, int L2, int L3, int L4>
__host__ __device__ constexpr bool k_warp_class_hi()
{
    return ncart_of(L1) * ncart_of(L2) * ncart_of(L3) * ncart_of(L4) >= 324;
}

constexpr int kKWarpStripes3 = 32;     // partner-3 stripes of a task, at most
constexpr int kKWarpStripesMax = 256;  // work units per task, at most (beyond 32: partner-1 segment stripes too)

template <int L1, int L2, int L3, int L4>
struct KWarpShape {
    static constexpr int LA = L1 + L2, LC = L3 + L4;
    static constexpr int S2 = L2 + 1, S3 = L3 + 1, S4 = L4 + 1, SG = (L1 + 1) * S2 * S3 * S4;
    static constexpr int N1 = ncart_of(L1), N2 = ncart_of(L2), N3 = ncart_of(L3), N4 = ncart_of(L4);
    static constexpr int NO = N1 * N3;                                      // output elements
    static constexpr int P = NO >= 32 ? 1 : (N2 < 32 / NO ? N2 : 32 / NO);   // i2 parts per element
    static constexpr int NJOB = NO * P, NJL = (NJOB + 31) / 32;             // jobs, jobs per lane
};

template <int L1, int L2, int L3, int L4>
struct KWarpTab {
    using S = KWarpShape<L1, L2, L3, L4>;
    double G[3][S::SG];                            // 1-D integrals of the current root
    double H[3][L2 + 1][S::LA + 1][S::LC + 1];     // after the transfer to centre 2
    double D[S::N2 * S::N4];                       // the task's D24 block
    double red[S::NJOB];                           // job sums at a segment flush
};

template <int L1, int L2, int L3, int L4>
__global__ void __launch_bounds__(kKThreads) k_exchange_warp(const __grid_constant__ KArgs A)
{
    using Sh = KWarpShape<L1, L2, L3, L4>;
    constexpr int NR = (L1 + L2 + L3 + L4) / 2 + 1;
    constexpr int LA = Sh::LA, LC = Sh::LC, S2 = Sh::S2, S3 = Sh::S3, S4 = Sh::S4;
    constexpr int N2 = Sh::N2, N3 = Sh::N3, N4 = Sh::N4, NO = Sh::NO, P = Sh::P, NJOB = Sh::NJOB,
                  NJL = Sh::NJL;
    extern __shared__ __align__(16) unsigned char kwarp_smem[];
    KWarpTab<L1, L2, L3, L4>& S = reinterpret_cast<KWarpTab<L1, L2, L3, L4>*>(kwarp_smem)[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int ntask1 = *A.ntask;
    const int ntask = ntask1 * A.nsub;
    const int nstripe = A.stripes;
    const int ns3 = nstripe < kKWarpStripes3 ? nstripe : kKWarpStripes3, ns1 = nstripe / ns3;
    const double* tab = static_cast<const double*>(A.rys);
    const double* asym_t = static_cast<const double*>(A.asym_t);
    const double* asym_w = static_cast<const double*>(A.asym_w);
    const float thre12 = A.sc->thre12, thre34 = A.sc->thre34;
    const double thr_lo = (double) A.thr_lo, thr_hi = (double) A.thr_hi;

    // this lane's jobs: element o = job / P (i1 = o / N3, i3 = o % N3), i2 range part = job % P
    int jx[NJL][2], jy[NJL][2], jz[NJL][2];   // Cartesian exponents of shells 1 and 3
    int j2lo[NJL], j2hi[NJL];
#pragma unroll
    for (int k = 0; k < NJL; ++k) {
        const int job = lane + 32 * k;
        const int o = job < NJOB ? job / P : 0, part = job < NJOB ? job % P : 0;
        const int i1 = o / N3, i3 = o % N3;
        jx[k][0] = cart_lx(L1, i1); jy[k][0] = cart_ly(L1, i1); jz[k][0] = cart_lz(L1, i1);
        jx[k][1] = cart_lx(L3, i3); jy[k][1] = cart_ly(L3, i3); jz[k][1] = cart_lz(L3, i3);
        j2lo[k] = job < NJOB ? part * N2 / P : 0;
        j2hi[k] = job < NJOB ? (part + 1) * N2 / P : 0;
    }
    long nq = 0;
    for (;;) {
        // work unit: a task and one of A.stripes stripes of its partners 3 (the small
        // f-class task lists of a small molecule still fill the GPU)
        int unit = 0;
        if (lane == 0) unit = (int) atomicAdd(A.queue, 1u);
        unit = __shfl_sync(0xffffffffu, unit, 0);
        if (unit >= ntask * nstripe) break;
        const int tv = unit / nstripe, su = unit - tv * nstripe;
        const int stripe = su % ns3, stripe1 = su / ns3;   // partner-3 stripe, partner-1 segment stripe
        const int sub = tv / ntask1;
        const KTask T = A.tasks[tv - sub * ntask1];
        const int dens = T.grp * kKBatch + sub;
        if (dens >= A.ng || dens >= (T.grp + 1) * kKBatch) continue;   // a sub-slot past the group's densities
        const int i2 = T.i2, i4 = T.i4;
        const double dRx = A.b2.x[i2] - A.b4.x[i4], dRy = A.b2.y[i2] - A.b4.y[i4], dRz = A.b2.z[i2] - A.b4.z[i4];
        const int s12 = A.r12s[i2], n12 = A.r12l[i2], s34 = A.r34s[i4], n34 = A.r34l[i4];
        const int c2 = A.b2.cart[i2], c4 = A.b4.cart[i4];
        const float tlo = float_threshold(thr_lo, T.dmax), thi = float_threshold(thr_hi, T.dmax);
        const double wsym = (A.flip && i2 == i4) ? 0.5 : 1.0;
        const float b12max = A.b12[s12];
        __syncwarp();   // the previous task's tables have been read
        for (int t = lane; t < N2 * N4; t += 32)
            S.D[t] = A.Dc[dens][(long) (c2 + t / N4) * A.ld4 + c4 + t % N4];
        __syncwarp();
        double* Kc = A.Kc[dens];
        for (int k3i = stripe; k3i < n34; k3i += ns3) {
            const int k3 = s34 + k3i;
            const float b34 = A.b34[k3];
            if (b34 < thre34 || b12max * b34 < tlo) break;   // the row (and the stripe) is in bound order
            const double kab34 = A.d34.kab[k3], q = A.d34.p[k3], iq = A.d34.ip[k3];
            const double Qx = A.d34.px[k3], Qy = A.d34.py[k3], Qz = A.d34.pz[k3];
            const double Cx = A.d34.ax[k3], Cy = A.d34.ay[k3], Cz = A.d34.az[k3];
            const int c3 = A.cart34[k3];
            const double QC[3] = {Qx - Cx, Qy - Cy, Qz - Cz};
            const double Sx = dRx - Qx, Sy = dRy - Qy, Sz = dRz - Qz;
            double acc[NJL];
#pragma unroll
            for (int k = 0; k < NJL; ++k) acc[k] = 0.0;
            bool any = false;
            int prev_seg = -1, prev_c1 = 0;
            auto flush = [&]() {
                if (any) {
#pragma unroll
                    for (int k = 0; k < NJL; ++k)
                        if (lane + 32 * k < NJOB) S.red[lane + 32 * k] = acc[k];
                    __syncwarp();
                    for (int o = lane; o < NO; o += 32) {
                        double v = 0.0;
#pragma unroll
                        for (int pp = 0; pp < P; ++pp) v += S.red[o * P + pp];
                        const int a = o / N3, c = o % N3;
                        atomicAdd(Kc + (long) (prev_c1 + a) * A.ld3 + c3 + c, wsym * v);
                    }
                    __syncwarp();
#pragma unroll
                    for (int k = 0; k < NJL; ++k) acc[k] = 0.0;
                }
                any = false;
            };
            for (int j = 0; j < n12; ++j) {
                const int e = s12 + j;
                const float b12 = A.b12[e];
                const int sg = A.seg12[e];
                if (ns1 > 1 && sg % ns1 != stripe1) continue;   // another unit's segment
                const float est = b12 * b34;
                const bool can = b12 >= thre12 && est >= tlo;
                if (sg != prev_seg) {
                    flush();
                    prev_seg = sg;
                    prev_c1 = A.cart12[e];
                    if (!can) break;   // segments are ordered by their largest bound
                } else if (!can) {
                    continue;          // entries of a segment are ordered by bound
                }
                if (est >= thi) continue;   // the other pass's quartet
                ++nq;
                any = true;
                const double p = A.d12.p[e], ip = A.d12.ip[e];
                const double ex = A.d12.px[e], ey = A.d12.py[e], ez = A.d12.pz[e];
                const double AB[3] = {A.d12.ax[e], A.d12.ay[e], A.d12.az[e]};
                const double PQ[3] = {ex + Sx, ey + Sy, ez + Sz};
                const double PA[3] = {ex - AB[0], ey - AB[1], ez - AB[2]};
                const double CD[3] = {Cx, Cy, Cz};
                const double RR = PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2];
                const double rs = rsqrt(p + q);
                const double ipq = rs * rs;
                const double rho = p * q * ipq;
                const double pref = kTwoPi52K * (A.d12.kab[e] * kab34) * rs;
                for (int tm = 0; tm < A.nterm; ++tm) {
                    double d2 = 1.0, f = A.alpha[tm] * pref;
                    if (A.omega[tm] != -1.0) {
                        const double w2 = A.omega[tm] * A.omega[tm];
                        d2 = w2 / (rho + w2);
                        f *= sqrt(d2);
                    }
                    double t2[NR], w[NR];
                    rys_eval<NR, double>(rho * d2 * RR, tab, A.nbin, A.tmax, asym_t, asym_w, t2, w);
#pragma unroll 1
                    for (int r = 0; r < NR; ++r) {
                        const double u = t2[r] * d2 * ipq;
                        const double qu = q * u, pu = p * u;
                        const double b00 = 0.5 * u, b10 = 0.5 * ip * (1.0 - qu), b01 = 0.5 * iq * (1.0 - pu);
                        if (lane < 3) {
                            // 2-D integrals I(a, c) of direction `lane`, then moved to centre 2
                            const int d = lane;
                            const double c00 = PA[d] - qu * PQ[d], d00 = QC[d] + pu * PQ[d], ab = AB[d];
                            auto& H = S.H[d];
                            H[0][0][0] = d == 2 ? f * w[r] : 1.0;
                            for (int a = 1; a <= LA; ++a) {
                                double s = c00 * H[0][a - 1][0];
                                if (a > 1) s = fma((a - 1) * b10, H[0][a - 2][0], s);
                                H[0][a][0] = s;
                            }
                            for (int c = 1; c <= LC; ++c)
                                for (int a = 0; a <= LA; ++a) {
                                    double s = d00 * H[0][a][c - 1];
                                    if (c > 1) s = fma((c - 1) * b01, H[0][a][c - 2], s);
                                    if (a > 0) s = fma(a * b00, H[0][a - 1][c - 1], s);
                                    H[0][a][c] = s;
                                }
                            for (int b = 1; b <= L2; ++b)
                                for (int a = 0; a <= LA - b; ++a)
                                    for (int c = 0; c <= LC; ++c) H[b][a][c] = fma(ab, H[b - 1][a][c], H[b - 1][a + 1][c]);
                        }
                        __syncwarp();
                        // to centre 4: one (direction, a, b) row per lane
                        for (int row = lane; row < 3 * (L1 + 1) * S2; row += 32) {
                            const int d = row / ((L1 + 1) * S2), a = (row / S2) % (L1 + 1), b = row % S2;
                            double Tr[L4 + 1][LC + 1];
#pragma unroll
                            for (int c = 0; c <= LC; ++c) Tr[0][c] = S.H[d][b][a][c];
#pragma unroll
                            for (int e4 = 1; e4 <= L4; ++e4)
#pragma unroll
                                for (int c = 0; c <= LC - e4; ++c) Tr[e4][c] = fma(CD[d], Tr[e4 - 1][c], Tr[e4 - 1][c + 1]);
#pragma unroll
                            for (int c = 0; c <= L3; ++c)
#pragma unroll
                                for (int e4 = 0; e4 <= L4; ++e4) S.G[d][((a * S2 + b) * S3 + c) * S4 + e4] = Tr[e4][c];
                        }
                        __syncwarp();
                        // the contraction jobs of this lane
#pragma unroll
                        for (int k = 0; k < NJL; ++k) {
                            double s = acc[k];
                            const int x1 = jx[k][0], y1 = jy[k][0], z1 = jz[k][0];
                            const int x3 = jx[k][1], y3 = jy[k][1], z3 = jz[k][1];
#pragma unroll 1
                            for (int i2c = j2lo[k]; i2c < j2hi[k]; ++i2c) {
                                const int x2 = cart_lx(L2, i2c), y2 = cart_ly(L2, i2c), z2 = cart_lz(L2, i2c);
                                const double* gx = &S.G[0][((x1 * S2 + x2) * S3 + x3) * S4];
                                const double* gy = &S.G[1][((y1 * S2 + y2) * S3 + y3) * S4];
                                const double* gz = &S.G[2][((z1 * S2 + z2) * S3 + z3) * S4];
                                const double* Drow = &S.D[i2c * N4];
                                int i4 = 0;
#pragma unroll
                                for (int j4 = 0; j4 <= L4; ++j4)
#pragma unroll
                                    for (int z4 = 0; z4 <= j4; ++z4, ++i4)
                                        s = fma(gx[L4 - j4] * gy[j4 - z4] * gz[z4], Drow[i4], s);
                            }
                            acc[k] = s;
                        }
                        __syncwarp();   // the tables are rewritten by the next root
                    }
                }
            }
            flush();
        }
    }
    if (lane == 0 && nq) atomicAdd(A.qcount, (unsigned long long) nq);
}

template <int L1, int L2, int L3, int L4>
void launch_k_warp(Context* ctx, const KArgs& A0, long units, int per_sm)
{
    // work units per task: at least 8 partner-3 stripes (long rows split for the load
    // balance), up to about 64 units per SM when the class has few tasks (the capacity
    // bounds the task count from above; the screens keep a part of it): up to 32
    // partner-3 stripes, then partner-1 segment stripes as well
    KArgs A = A0;
    const long want = 64L * ctx->nsm;
    A.stripes = (int) std::max<long>(8, std::min<long>(kKWarpStripesMax, (want + units - 1) / std::max(1L, units)));
    if (A.stripes > kKWarpStripes3) A.stripes -= A.stripes % kKWarpStripes3;   // whole partner-1 stripes
    unsigned grid = (unsigned) std::min<long>((units * A.stripes + kKWarps - 1) / kKWarps,
                                              (long) ctx->nsm * (per_sm > 0 ? per_sm : 16));
    constexpr size_t smem = (size_t) kKWarps * sizeof(KWarpTab<L1, L2, L3, L4>);
    auto kern = k_exchange_warp<L1, L2, L3, L4>;
    static std::atomic<unsigned long long> attr_devices{0};
    const unsigned long long bit = 1ull << (ctx->device & 63);
    if (smem > 48 * 1024 && !(attr_devices.load(std::memory_order_acquire) & bit)) {
        LSJK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
        attr_devices.fetch_or(bit, std::memory_order_acq_rel);
    }
    kern<<<grid, kKThreads, smem, ctx->stream>>>(A);
    LSJK_CUDA(cudaGetLastError());
    ctx->stats.kernel_launches++;
}

} // namespace lsjk
