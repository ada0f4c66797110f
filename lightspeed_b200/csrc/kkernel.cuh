// The K kernel: one template per class (L1 L2|L3 L4). Included only by
// kinst.cu, which is compiled once per (L1, L2) with the matching generated
// quartet header so the 81 classes build in parallel.
#pragma once
#include <algorithm>
#include "kargs.cuh"
#include "lsjk_device.cuh"

namespace lsjk {

constexpr double kTwoPi52K = 34.986836655249725693;   // 2 pi^(5/2)

template <int L1, int L2, int L3, int L4>
__global__ void __launch_bounds__(kKThreads) k_exchange(KArgs A)
{
    constexpr int NR = (L1 + L2 + L3 + L4) / 2 + 1;
    constexpr int N1 = ncart_of(L1), N2 = ncart_of(L2), N3 = ncart_of(L3), N4 = ncart_of(L4);
    extern __shared__ __align__(128) double tab[];
    __shared__ __align__(8) uint64_t mbar;
    const int ntask = *A.ntask;
    if (ntask == 0) return;
    const unsigned bytes = (unsigned) (2 * NR * A.nbin * 8 * sizeof(double));
    if (!stage_bulk(tab, A.rys, bytes, &mbar, A.status)) return;

    const int lane = threadIdx.x & 31;
    const float thre12 = A.sc->thre12, thre34 = A.sc->thre34;
    long nq = 0;
    for (;;) {
        int task = 0;
        if (lane == 0) task = (int) atomicAdd(A.queue, 1u);
        task = __shfl_sync(0xffffffffu, task, 0);
        if (task >= ntask) break;
        const KTask T = A.tasks[task];
        const int i2 = T.i2, i4 = T.i4;
        const double dmax = T.dmax;
        const double e2 = A.b2.e[i2], Bx = A.b2.x[i2], By = A.b2.y[i2], Bz = A.b2.z[i2];
        const double e4 = A.b4.e[i4], Dx = A.b4.x[i4], Dy = A.b4.y[i4], Dz = A.b4.z[i4];
        const int c2 = A.b2.cart[i2], c4 = A.b4.cart[i4];
        double Dblk[N2 * N4];
#pragma unroll
        for (int a = 0; a < N2; ++a)
#pragma unroll
            for (int b = 0; b < N4; ++b) Dblk[a * N4 + b] = A.Dc[(long) (c2 + a) * A.ld4 + c4 + b];
        const int s12 = A.r12s[i2], n12 = A.r12l[i2];
        const int s34 = A.r34s[i4], n34 = A.r34l[i4];
        const float b34_0 = A.b34[s34];
        for (int k1 = 0; k1 < n12; ++k1) {
            const float b12 = A.b12[s12 + k1];
            if (b12 < thre12) break;
            if ((double) (b12 * b34_0) * dmax < (double) A.thresp) break;
            const double kab12 = A.kab12[s12 + k1], e1 = A.e12[s12 + k1];
            const double Ax = A.x12[s12 + k1], Ay = A.y12[s12 + k1], Az = A.z12[s12 + k1];
            const int c1 = A.cart12[s12 + k1];
            const double p = e1 + e2, ip = 1.0 / p;
            const double Px = (e1 * Ax + e2 * Bx) * ip, Py = (e1 * Ay + e2 * By) * ip, Pz = (e1 * Az + e2 * Bz) * ip;
            for (int k3 = lane; k3 < n34; k3 += 32) {
                const float b34 = A.b34[s34 + k3];
                if (b34 < thre34) break;
                if ((double) (b12 * b34) * dmax < (double) A.thresp) break;
                ++nq;
                const double kab34 = A.kab34[s34 + k3], e3 = A.e34[s34 + k3];
                const double Cx = A.x34[s34 + k3], Cy = A.y34[s34 + k3], Cz = A.z34[s34 + k3];
                const int c3 = A.cart34[s34 + k3];
                const double q = e3 + e4, iq = 1.0 / q;
                const double Qx = (e3 * Cx + e4 * Dx) * iq, Qy = (e3 * Cy + e4 * Dy) * iq, Qz = (e3 * Cz + e4 * Dz) * iq;
                const double ipq = 1.0 / (p + q);
                const double rho = p * q * ipq;
                const double PQx = Px - Qx, PQy = Py - Qy, PQz = Pz - Qz;
                const double R2 = PQx * PQx + PQy * PQy + PQz * PQz;
                const double pref = kTwoPi52K * kab12 * kab34 * ip * iq * sqrt(ipq);
                double KV[N1 * N3];
#pragma unroll
                for (int t = 0; t < N1 * N3; ++t) KV[t] = 0.0;
                for (int tm = 0; tm < A.nterm; ++tm) {
                    const double om = A.omega[tm];
                    double d2 = 1.0, f = A.alpha[tm] * pref;
                    if (om != -1.0) {
                        const double w2 = om * om;
                        d2 = w2 / (rho + w2);
                        f *= sqrt(d2);
                    }
                    double t2[NR], w[NR];
                    rys_eval<NR, double>(rho * d2 * R2, tab, A.nbin, A.tmax, A.asym_t, A.asym_w, t2, w);
#pragma unroll
                    for (int r = 0; r < NR; ++r) {
                        const double te = t2[r] * d2;
                        const double u = te * ipq;
                        const double b00 = 0.5 * u;
                        const double b10 = 0.5 * ip * (1.0 - q * u);
                        const double b01 = 0.5 * iq * (1.0 - p * u);
                        const double qu = q * u, pu = p * u;
                        kq_dispatch<L1, L2, L3, L4>(
                            (Px - Ax) - qu * PQx, (Py - Ay) - qu * PQy, (Pz - Az) - qu * PQz,
                            (Qx - Cx) + pu * PQx, (Qy - Cy) + pu * PQy, (Qz - Cz) + pu * PQz,
                            b00, b10, b01, Ax - Bx, Ay - By, Az - Bz, Cx - Dx, Cy - Dy, Cz - Dz,
                            f * w[r], Dblk, KV);
                    }
                }
#pragma unroll
                for (int a = 0; a < N1; ++a)
#pragma unroll
                    for (int c = 0; c < N3; ++c) {
                        const double v = KV[a * N3 + c];
                        atomicAdd(&A.Kc[(long) (c1 + a) * A.ld3 + c3 + c], v);
                        if (A.flip && i2 != i4) atomicAdd(&A.Kc[(long) (c3 + c) * A.ld3 + c1 + a], v);
                    }
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) nq += __shfl_xor_sync(0xffffffffu, nq, o);
    if (lane == 0 && nq) atomicAdd(A.qcount, (unsigned long long) nq);
}

template <int L1, int L2, int L3, int L4>
void launch_k(Context* ctx, const KArgs& A, long cap)
{
    if (cap == 0) return;
    constexpr int NR = (L1 + L2 + L3 + L4) / 2 + 1;
    size_t smem = (size_t) 2 * NR * A.nbin * 8 * sizeof(double);
    static bool attr_set = false;
    if (!attr_set) {
        LSJK_CUDA(cudaFuncSetAttribute(k_exchange<L1, L2, L3, L4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int) smem));
        attr_set = true;
    }
    long want = (cap + kKWarps - 1) / kKWarps;
    unsigned grid = (unsigned) std::min<long>(want, 148L * 16);
    k_exchange<L1, L2, L3, L4><<<grid, kKThreads, smem, ctx->stream>>>(A);
    LSJK_CUDA(cudaGetLastError());
    ctx->stats.kernel_launches++;
}


} // namespace lsjk
