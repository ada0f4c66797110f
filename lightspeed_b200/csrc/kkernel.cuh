// The K kernel: one template per class (L1 L2|L3 L4). Included only by
// kinst.cu, which is compiled once per (L1, L2) with the matching generated
// quartet header so the 81 classes build in parallel.
#pragma once
#include <algorithm>
#include "kargs.cuh"
#include "lsjk_device.cuh"

namespace lsjk {

constexpr double kTwoPi52K = 34.986836655249725693;   // 2 pi^(5/2)

// Geometry of one K quartet, shared by both precisions (FP64).
struct KGeom {
    double p, q, ip, iq, Px, Py, Pz, Qx, Qy, Qz, Ax, Ay, Az, Bx, By, Bz, Cx, Cy, Cz, Dx, Dy, Dz, kab;
};

template <int L1, int L2, int L3, int L4>
__device__ __forceinline__ void k_quartet64(const KArgs& A, const double* tab, const KGeom& g,
                                            const double* Dblk, double* KV)
{
    constexpr int NR = (L1 + L2 + L3 + L4) / 2 + 1;
    const double p = g.p, q = g.q, ip = g.ip, iq = g.iq;
    const double ipq = 1.0 / (p + q);
    const double rho = p * q * ipq;
    const double PQx = g.Px - g.Qx, PQy = g.Py - g.Qy, PQz = g.Pz - g.Qz;
    const double R2 = PQx * PQx + PQy * PQy + PQz * PQz;
    const double pref = kTwoPi52K * g.kab * ip * iq * sqrt(ipq);
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
            const double u = t2[r] * d2 * ipq;
            const double qu = q * u, pu = p * u;
            kq_dispatch<L1, L2, L3, L4>(
                (g.Px - g.Ax) - qu * PQx, (g.Py - g.Ay) - qu * PQy, (g.Pz - g.Az) - qu * PQz,
                (g.Qx - g.Cx) + pu * PQx, (g.Qy - g.Cy) + pu * PQy, (g.Qz - g.Cz) + pu * PQz,
                0.5 * u, 0.5 * ip * (1.0 - qu), 0.5 * iq * (1.0 - pu),
                g.Ax - g.Bx, g.Ay - g.By, g.Az - g.Bz, g.Cx - g.Dx, g.Cy - g.Dy, g.Cz - g.Dz,
                f * w[r], Dblk, KV);
        }
    }
}

// FP32 quartet: geometry differences formed in FP64, the rest in FP32.
template <int L1, int L2, int L3, int L4>
__device__ __forceinline__ void k_quartet32(const KArgs& A, const float* tab, const KGeom& g,
                                            const float* Dblk, float* KV)
{
    constexpr int NR = (L1 + L2 + L3 + L4) / 2 + 1;
    const float p = (float) g.p, q = (float) g.q, ip = (float) g.ip, iq = (float) g.iq;
    const float ipq = 1.0f / (p + q);
    const float rho = p * q * ipq;
    const float PQx = (float) (g.Px - g.Qx), PQy = (float) (g.Py - g.Qy), PQz = (float) (g.Pz - g.Qz);
    const float PAx = (float) (g.Px - g.Ax), PAy = (float) (g.Py - g.Ay), PAz = (float) (g.Pz - g.Az);
    const float QCx = (float) (g.Qx - g.Cx), QCy = (float) (g.Qy - g.Cy), QCz = (float) (g.Qz - g.Cz);
    const float ABx = (float) (g.Ax - g.Bx), ABy = (float) (g.Ay - g.By), ABz = (float) (g.Az - g.Bz);
    const float CDx = (float) (g.Cx - g.Dx), CDy = (float) (g.Cy - g.Dy), CDz = (float) (g.Cz - g.Dz);
    const float R2 = PQx * PQx + PQy * PQy + PQz * PQz;
    const float pref = (float) (kTwoPi52K * g.kab) * ip * iq * sqrtf(ipq);
    for (int tm = 0; tm < A.nterm; ++tm) {
        const float om = (float) A.omega[tm];
        float d2 = 1.0f, f = (float) A.alpha[tm] * pref;
        if (A.omega[tm] != -1.0) {
            const float w2 = om * om;
            d2 = w2 / (rho + w2);
            f *= sqrtf(d2);
        }
        float t2[NR], w[NR];
        rys_eval<NR, float>(rho * d2 * R2, tab, A.nbin, (float) A.tmax, A.asym_t32, A.asym_w32, t2, w);
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            const float u = t2[r] * d2 * ipq;
            const float qu = q * u, pu = p * u;
            kq_dispatch<L1, L2, L3, L4>(PAx - qu * PQx, PAy - qu * PQy, PAz - qu * PQz,
                                        QCx + pu * PQx, QCy + pu * PQy, QCz + pu * PQz,
                                        0.5f * u, 0.5f * ip * (1.0f - qu), 0.5f * iq * (1.0f - pu),
                                        ABx, ABy, ABz, CDx, CDy, CDz, f * w[r], Dblk, KV);
        }
    }
}

template <int L1, int L2, int L3, int L4>
__global__ void __launch_bounds__(kKThreads) k_exchange(KArgs A)
{
    constexpr int NR = (L1 + L2 + L3 + L4) / 2 + 1;
    constexpr int N1 = ncart_of(L1), N2 = ncart_of(L2), N3 = ncart_of(L3), N4 = ncart_of(L4);
    extern __shared__ __align__(128) double tab[];
    __shared__ __align__(8) uint64_t mbar[2];
    const int ntask = *A.ntask;
    if (ntask == 0) return;
    const unsigned nco = (unsigned) (2 * NR * A.nbin * 8);
    float* tab32 = reinterpret_cast<float*>(tab + nco);
    if (!stage_bulk(tab, A.rys, nco * (unsigned) sizeof(double), &mbar[0], A.status)) return;
    if (A.mixed && !stage_bulk(tab32, A.rys32, nco * (unsigned) sizeof(float), &mbar[1], A.status)) return;

    const int lane = threadIdx.x & 31;
    const float thre12 = A.sc->thre12, thre34 = A.sc->thre34;
    const double thr_dp = A.mixed ? (double) A.thredp : 0.0;
    long nq = 0, nq32 = 0;
    for (;;) {
        int task = 0;
        if (lane == 0) task = (int) atomicAdd(A.queue, 1u);
        task = __shfl_sync(0xffffffffu, task, 0);
        if (task >= ntask) break;
        const KTask T = A.tasks[task];
        const int i2 = T.i2, i4 = T.i4;
        const double dmax = T.dmax;
        KGeom g;
        const double e2 = A.b2.e[i2], e4 = A.b4.e[i4];
        g.Bx = A.b2.x[i2]; g.By = A.b2.y[i2]; g.Bz = A.b2.z[i2];
        g.Dx = A.b4.x[i4]; g.Dy = A.b4.y[i4]; g.Dz = A.b4.z[i4];
        const int c2 = A.b2.cart[i2], c4 = A.b4.cart[i4];
        double Dblk[N2 * N4];
        float Dblk32[N2 * N4];
#pragma unroll
        for (int a = 0; a < N2; ++a)
#pragma unroll
            for (int b = 0; b < N4; ++b) {
                Dblk[a * N4 + b] = A.Dc[(long) (c2 + a) * A.ld4 + c4 + b];
                Dblk32[a * N4 + b] = (float) Dblk[a * N4 + b];
            }
        const int s12 = A.r12s[i2], n12 = A.r12l[i2];
        const int s34 = A.r34s[i4], n34 = A.r34l[i4];
        const float b34_0 = A.b34[s34];
        for (int k1 = 0; k1 < n12; ++k1) {
            const float b12 = A.b12[s12 + k1];
            if (b12 < thre12) break;
            if ((double) (b12 * b34_0) * dmax < (double) A.thresp) break;
            const double kab12 = A.kab12[s12 + k1], e1 = A.e12[s12 + k1];
            g.Ax = A.x12[s12 + k1]; g.Ay = A.y12[s12 + k1]; g.Az = A.z12[s12 + k1];
            const int c1 = A.cart12[s12 + k1];
            g.p = e1 + e2;
            g.ip = 1.0 / g.p;
            g.Px = (e1 * g.Ax + e2 * g.Bx) * g.ip;
            g.Py = (e1 * g.Ay + e2 * g.By) * g.ip;
            g.Pz = (e1 * g.Az + e2 * g.Bz) * g.ip;
            for (int k3 = lane; k3 < n34; k3 += 32) {
                const float b34 = A.b34[s34 + k3];
                if (b34 < thre34) break;
                const double est = (double) (b12 * b34) * dmax;
                if (est < (double) A.thresp) break;
                const double e3 = A.e34[s34 + k3];
                g.Cx = A.x34[s34 + k3]; g.Cy = A.y34[s34 + k3]; g.Cz = A.z34[s34 + k3];
                const int c3 = A.cart34[s34 + k3];
                g.kab = kab12 * A.kab34[s34 + k3];
                g.q = e3 + e4;
                g.iq = 1.0 / g.q;
                g.Qx = (e3 * g.Cx + e4 * g.Dx) * g.iq;
                g.Qy = (e3 * g.Cy + e4 * g.Dy) * g.iq;
                g.Qz = (e3 * g.Cz + e4 * g.Dz) * g.iq;
                double KV[N1 * N3];
                if (est >= thr_dp) {
                    ++nq;
#pragma unroll
                    for (int t = 0; t < N1 * N3; ++t) KV[t] = 0.0;
                    k_quartet64<L1, L2, L3, L4>(A, tab, g, Dblk, KV);
                } else {
                    ++nq32;
                    float KV32[N1 * N3];
#pragma unroll
                    for (int t = 0; t < N1 * N3; ++t) KV32[t] = 0.0f;
                    k_quartet32<L1, L2, L3, L4>(A, tab32, g, Dblk32, KV32);
#pragma unroll
                    for (int t = 0; t < N1 * N3; ++t) KV[t] = (double) KV32[t];
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
    for (int o = 16; o > 0; o >>= 1) {
        nq += __shfl_xor_sync(0xffffffffu, nq, o);
        nq32 += __shfl_xor_sync(0xffffffffu, nq32, o);
    }
    if (lane == 0) {
        if (nq) atomicAdd(A.qcount, (unsigned long long) nq);
        if (nq32) atomicAdd(A.qcount32, (unsigned long long) nq32);
    }
}

template <int L1, int L2, int L3, int L4>
void launch_k(Context* ctx, const KArgs& A, long cap)
{
    if (cap == 0) return;
    constexpr int NR = (L1 + L2 + L3 + L4) / 2 + 1;
    size_t smem = (size_t) 2 * NR * A.nbin * 8 * (sizeof(double) + sizeof(float));
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
