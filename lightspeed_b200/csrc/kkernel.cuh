// The K kernel: one template per class (L1 L2|L3 L4) and precision. Included
// only by kinst.cu, which is compiled once per (L1, L2) with the matching
// generated quartet header so the classes build in parallel.
//
// Work unit: one (prim2, prim4) task, taken by a warp from a device queue.
// The 32 lanes own 32 consecutive partners 3 of prim4, taken from a copy of
// the rows ordered by bound alone (their pair data stay in registers while
// the chunk is processed); the warp walks the partners 1 of prim2,
// which are staged 32 at a time into a per-warp shared-memory ring by
// cp.async (the next 32 are in flight while the current 32 are used) and read
// as broadcasts. Partners 1 come grouped by contracted shell, so a lane sums
// the quartets of one shell segment -- same K13 target block -- in registers
// and issues one FP64 atomic per element when the segment ends (for a
// symmetric D24 only the untransposed one: the build symmetrises K13 after
// the class kernels).
// Up to k_batch densities share a lane: the integrals of a quartet are
// formed once and contracted with each density's D24 block; one launch per
// class and pass serves every density of the build (groups of kKBatch with
// their own task lists, each run once per sub-slot of k_batch densities).
// Screens (per quartet, exactly the reference's set):
//   bound12 >= thre12, bound34 >= thre34,
//   thr_lo <= double(float(bound12*bound34)) * max|D24 block| < thr_hi
// where [thr_lo, thr_hi) is [thresp, inf) in FP64 mode and splits at thredp
// into an FP64 pass and an FP32 pass in mixed mode.
#pragma once
#include <algorithm>
#include <atomic>
#include <type_traits>
#include "kargs.cuh"
#include "lsjk_device.cuh"

namespace lsjk {

constexpr double kTwoPi52K = 34.986836655249725693;   // 2 pi^(5/2)

// Smallest float x with double(x) * dmax >= thr. For non-negative float
// products b = float(bound12 * bound34) the reference's screen
// double(b) * dmax >= thr is then exactly b >= x (the map x -> double(x)*dmax
// is monotone), so each quartet is screened with one float compare.
__device__ __forceinline__ float float_threshold(double thr, double dmax)
{
    if (!(thr > 0.0)) return 0.0f;
    if (!(dmax > 0.0)) return __int_as_float(0x7f800000);   // +inf: nothing passes
    float x = (float) (thr / dmax);
    for (int it = 0; it < 8 && (double) x * dmax < thr; ++it) x = nextafterf(x, __int_as_float(0x7f800000));
    for (int it = 0; it < 8 && x > 0.0f && (double) nextafterf(x, 0.0f) * dmax >= thr; ++it) x = nextafterf(x, 0.0f);
    return x;
}

// One partner-1 entry as staged in shared memory (112 / 64 bytes): pair data,
// the partner's weights in its two output targets, the bound, the first and
// second target (Cartesian offsets, t1 = -1 if none) and the target group.
template <typename R>
struct alignas(16) KEnt {
    R kab, p, ip, px, py, pz, ax, ay, az, w0, w1;
    float b;
    int c, t1, seg;
};

// Tasks a warp takes from the queue at once (at most; fewer when the class
// has few tasks per warp, so the queue still balances the load).
constexpr int kKGrab = 16;

// Everything a task needs before its partner rows, prepared by one lane per
// task of a grab (the loads of all the grab's tasks overlap) and read by the
// warp as shared-memory broadcasts (64 bytes).
struct alignas(16) KHdr {
    double dRx, dRy, dRz;   // R2 - R4 (pair data are relative to these centres)
    int s12, n12, s34, n34; // K-invert rows of prim2 (partners 1) and prim4 (partners 3; n34: the
                            // prefix of the row that can pass the screens)
    int c2, c4;             // Cartesian offsets of prim2 and prim4
    float tlo, thi;         // float thresholds on bound12 * bound34 for this task's max|D24|
    float b12max;           // largest bound of the partner-1 row
    float wsym;             // 1/2 for a diagonal task of a symmetric D24, else 1
    int dbase, dn;          // densities dbase .. dbase + dn - 1 of the build (the task's sub-slot)
};

// Lane l copies entry kb + l of the row (if it exists) into dst[l].
template <typename R>
__device__ __forceinline__ void stage_ent(KEnt<R>* dst, const KRows<R>& d, const float* __restrict__ b,
                                          const int* __restrict__ cart, const int* __restrict__ t1,
                                          const int* __restrict__ seg, int s12, int kb, int n12, int lane)
{
    if (kb + lane >= n12) return;
    const int e = s12 + kb + lane;
    KEnt<R>* o = dst + lane;
    if constexpr (sizeof(R) == 8) {
        cp_async8(&o->kab, d.kab + e);
        cp_async8(&o->p, d.p + e);
        cp_async8(&o->ip, d.ip + e);
        cp_async8(&o->px, d.px + e);
        cp_async8(&o->py, d.py + e);
        cp_async8(&o->pz, d.pz + e);
        cp_async8(&o->ax, d.ax + e);
        cp_async8(&o->ay, d.ay + e);
        cp_async8(&o->az, d.az + e);
        cp_async8(&o->w0, d.w0 + e);
        cp_async8(&o->w1, d.w1 + e);
    } else {
        cp_async4(&o->kab, d.kab + e);
        cp_async4(&o->p, d.p + e);
        cp_async4(&o->ip, d.ip + e);
        cp_async4(&o->px, d.px + e);
        cp_async4(&o->py, d.py + e);
        cp_async4(&o->pz, d.pz + e);
        cp_async4(&o->ax, d.ax + e);
        cp_async4(&o->ay, d.ay + e);
        cp_async4(&o->az, d.az + e);
        cp_async4(&o->w0, d.w0 + e);
        cp_async4(&o->w1, d.w1 + e);
    }
    cp_async4(&o->b, b + e);
    cp_async4(&o->c, cart + e);
    cp_async4(&o->t1, t1 + e);
    cp_async4(&o->seg, seg + e);
}

// Densities per lane for a class: up to kKBatch while a per-density
// register weight, N1*N3*(2+w) + N2*N4*w with w the 32-bit registers of one R
// (the segment accumulators and D24 block, with headroom for the
// accumulation's temporaries; chosen by measurement), stays within 64; 1 above.
template <int L1, int L2, int L3, int L4, typename R>
__host__ __device__ constexpr int k_batch()
{
    constexpr int w = sizeof(R) / 4;
    constexpr int per = ncart_of(L1) * ncart_of(L3) * (2 + w) + ncart_of(L2) * ncart_of(L4) * w;
    return 4 * per <= 64 ? 4 : (2 * per <= 64 ? 2 : 1);
}

// One quartet (partner 1 from the staged entry e, partner 3 from registers)
// contracted with the NG densities' D24 blocks and added straight into the
// lane's shell-segment accumulators (type R: the FP32 pass sums the at most
// one contracted shell's worth of quartets of a segment in FP32, and the sum
// enters K in FP64 when the segment is flushed). The Rys roots, weights and
// 1-D integrals are shared by the densities (the NG inlined contractions see
// identical integral inputs).
template <int L1, int L2, int L3, int L4, typename R, int NG>
__device__ __forceinline__ void k_quartet(const KArgs& A, const R* __restrict__ tab, R tmax,
                                          const R* __restrict__ asym_t, const R* __restrict__ asym_w,
                                          const KEnt<R>& e, R kab34, R q, R iq, R Sx, R Sy, R Sz, R QCx,
                                          R QCy, R QCz, R Cx, R Cy, R Cz, const R (*Dblk)[ncart_of(L2) * ncart_of(L4)],
                                          R (*acc)[ncart_of(L1) * ncart_of(L3)])
{
    constexpr int NR = (L1 + L2 + L3 + L4) / 2 + 1;
    constexpr int N1 = ncart_of(L1), N3 = ncart_of(L3);
    const R p = e.p, ip = e.ip;
    // PQ = (P - R2) - (Q - R4) + (R2 - R4)
    const R PQx = e.px + Sx, PQy = e.py + Sy, PQz = e.pz + Sz;
    const R PAx = e.px - e.ax, PAy = e.py - e.ay, PAz = e.pz - e.az;
    const R RR = PQx * PQx + PQy * PQy + PQz * PQz;
    const R rs = drsqrt(p + q);
    const R ipq = rs * rs;
    const R rho = p * q * ipq;
    // kab fields hold K_ab / p per pair
    const R pref = (R) kTwoPi52K * (e.kab * kab34) * rs;
    for (int tm = 0; tm < A.nterm; ++tm) {
        R d2 = R(1), f = (R) A.alpha[tm] * pref;
        if (A.omega[tm] != -1.0) {
            const R w2 = (R) (A.omega[tm] * A.omega[tm]);
            d2 = w2 / (rho + w2);
            f *= sqrt(d2);
        }
        R t2[NR], w[NR];
        if constexpr (sizeof(R) == 4) {
            // FP32 pass: from the last table bin on (the bin next to the switch to the
            // asymptotic form, and the asymptotic region) the roots and weights are the
            // FP64 asymptotic form t = s / sqrt(T), w = h / sqrt(T), which over the last
            // bin already agrees with the exact rule to ~1e-13 relative
            const R T = rho * d2 * RR;
            if (T < tmax - tmax / (R) A.nbin) {
                rys_eval<NR, R>(T, tab, A.nbin, tmax, asym_t, asym_w, t2, w);
            } else {
                const double r = rsqrt_f64_newton((double) rho * (double) d2 * (double) RR);
#pragma unroll
                for (int i = 0; i < NR; ++i) {
                    const double t = c_rys_asym_t[NR * LSJK_RYS_NMAX + i] * r;
                    t2[i] = (R) (t * t);
                    w[i] = (R) (c_rys_asym_w[NR * LSJK_RYS_NMAX + i] * r);
                }
            }
        } else {
            rys_eval<NR, R>(rho * d2 * RR, tab, A.nbin, tmax, asym_t, asym_w, t2, w);
        }
        auto root = [&](int r) {
            const R u = t2[r] * d2 * ipq;
            const R qu = q * u, pu = p * u;
            const R c00x = PAx - qu * PQx, c00y = PAy - qu * PQy, c00z = PAz - qu * PQz;
            const R d00x = QCx + pu * PQx, d00y = QCy + pu * PQy, d00z = QCz + pu * PQz;
            const R b00 = R(0.5) * u, b10 = R(0.5) * ip * (R(1) - qu), b01 = R(0.5) * iq * (R(1) - pu);
#pragma unroll
            for (int g = 0; g < NG; ++g)
                kq_dispatch<L1, L2, L3, L4>(c00x, c00y, c00z, d00x, d00y, d00z, b00, b10, b01, e.ax, e.ay, e.az,
                                            Cx, Cy, Cz, f * w[r], Dblk[g], acc[g]);
        };
        if constexpr (sizeof(R) == 4) {
            // FP32: roots one after another (fewer live registers, more resident warps);
            // the root in use is always slot 0 and the rest shift down, so the
            // arrays keep static indices and stay in registers
#pragma unroll 1
            for (int r = 0; r < NR; ++r) {
                root(0);
#pragma unroll
                for (int i = 0; i + 1 < NR; ++i) {
                    t2[i] = t2[i + 1];
                    w[i] = w[i + 1];
                }
            }
        } else {
#pragma unroll
            for (int r = 0; r < NR; ++r) root(r);
        }
    }
}

template <int L1, int L2, int L3, int L4, typename R, int NG, bool GC>
__global__ void __launch_bounds__(kKThreads) k_exchange(const __grid_constant__ KArgs A)
{
    constexpr int NR = (L1 + L2 + L3 + L4) / 2 + 1;
    constexpr int N1 = ncart_of(L1), N2 = ncart_of(L2), N3 = ncart_of(L3), N4 = ncart_of(L4);
    constexpr bool FP64 = std::is_same<R, double>::value;
    // over merged twins s-type partners may stand for two contracted shells:
    // two target blocks per segment (partner 1) or per lane (partner 3)
    constexpr int G1 = (GC && L1 == 0) ? 2 : 1;
    constexpr int G3 = (GC && L3 == 0) ? 2 : 1;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    R* tab = reinterpret_cast<R*>(smem_raw);
    __shared__ __align__(8) uint64_t mbar;
    __shared__ KEnt<R> ring_all[kKWarps][2][32];
    __shared__ KHdr hdr_all[kKWarps][kKGrab];
    const int ntask1 = *A.ntask;
    const int ntask = ntask1 * A.nsub;   // the task list once per density sub-slot
    // the grid is sized for the class's task capacity; CTAs whose warps cannot
    // get a task leave before staging the quadrature table
    if ((long) blockIdx.x * kKWarps >= ntask) return;
    const unsigned bytes = (unsigned) (2 * NR * A.nbin * 8 * sizeof(R));
    if (!stage_bulk(tab, A.rys, bytes, &mbar, A.status)) return;
    const R* asym_t = static_cast<const R*>(A.asym_t);
    const R* asym_w = static_cast<const R*>(A.asym_w);
    const R tmax = (R) A.tmax;

    const KRows<R> d12 = [&] { if constexpr (FP64) return A.d12; else return A.f12; }();
    const KRows<R> d34 = [&] { if constexpr (FP64) return A.d34; else return A.f34; }();
    const int lane = threadIdx.x & 31;
    KEnt<R>* ring = &ring_all[threadIdx.x >> 5][0][0];
    KHdr* hdr = &hdr_all[threadIdx.x >> 5][0];
    const float thre12 = A.sc->thre12, thre34 = A.sc->thre34;
    const double thr_lo = (double) A.thr_lo, thr_hi = (double) A.thr_hi;   // (float -> double exact)
    // guided self-scheduling: a grab takes about a quarter of this warp's share of
    // the tasks left after its previous grab (1..kKGrab), so grabs shrink to
    // single tasks as the queue drains
    const int nwarp4 = 4 * (int) gridDim.x * kKWarps;
    int t0 = 0;
    long nq = 0;
    for (;;) {
        const int left = ntask - t0;
        const int grab = left >= kKGrab * nwarp4 ? kKGrab : (left >= 2 * nwarp4 ? left / nwarp4 : 1);
        if (lane == 0) t0 = (int) atomicAdd(A.queue, (unsigned) grab);
        t0 = __shfl_sync(0xffffffffu, t0, 0);
        if (t0 >= ntask) break;
        const int nt = min(grab, ntask - t0);
        __syncwarp();   // the previous grab's headers have been read
        if (lane < nt) {
            const int tv = t0 + lane;
            const int sub = tv / ntask1;
            const KTask T = A.tasks[tv - sub * ntask1];
            const int i2 = T.i2, i4 = T.i4;
            KHdr h;
            h.dbase = T.grp * kKBatch + sub * NG;
            h.dn = max(0, min(NG, min(A.ng, (T.grp + 1) * kKBatch) - h.dbase));
            h.dRx = A.b2.x[i2] - A.b4.x[i4];
            h.dRy = A.b2.y[i2] - A.b4.y[i4];
            h.dRz = A.b2.z[i2] - A.b4.z[i4];
            h.s12 = A.r12s[i2];
            h.n12 = A.r12l[i2];
            h.s34 = A.r34s[i4];
            h.n34 = A.r34l[i4];
            h.c2 = A.b2.cart[i2];
            h.c4 = A.b4.cart[i4];
            // per-task float thresholds on the bound product (exactly the double screens);
            // T.dmax is the largest |D24 block| over the densities of the batch
            h.tlo = float_threshold(thr_lo, T.dmax);
            h.thi = float_threshold(thr_hi, T.dmax);
            h.b12max = A.b12[h.s12];   // first segment's first entry: the row maximum
            // partners 3 that can pass with the row's largest partner-1 bound: a prefix of
            // the bound-ordered row (b34 >= thre34 and b12max * b34 >= tlo, both monotone)
            {
                int lo = 0, hi = h.n34;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    const float b = A.b34[h.s34 + mid];
                    if (b >= thre34 && h.b12max * b >= h.tlo) lo = mid + 1; else hi = mid;
                }
                h.n34 = h.dn > 0 ? lo : 0;   // a sub-slot past the group's densities: no work
            }
            // symmetric D24 (A.flip): the transposed contribution of a task with i2 != i4 is
            // not written here; the build adds K13 to its transpose afterwards, and tasks with
            // i2 == i4 (whose contribution is symmetric) enter with weight 1/2
            h.wsym = (A.flip && i2 == i4) ? 0.5f : 1.0f;
            hdr[lane] = h;
        }
        __syncwarp();
        // Packs: the lanes of the warp take partners 3 of one or more consecutive tasks of
        // the grab that share prim2 (hence the same partner-1 row), a lane each, so short
        // partner-3 rows (p and d partners) and the tail of a long row fill the warp
        // together; each lane keeps its own task's thresholds, D24 block and centres.
        int pos = 0, koff = 0;
#pragma unroll 1
        for (;;) {
            while (pos < nt && hdr[pos].n34 == 0) ++pos;
            if (pos >= nt) break;
            const int s12 = hdr[pos].s12, n12 = hdr[pos].n12, c2 = hdr[pos].c2;
            // the pack's densities (its tasks share prim2 and the density sub-slot)
            const int dbase = hdr[pos].dbase, dn = hdr[pos].dn;
            int my_task = -1, my_k = 0;
            {
                int filled = 0, at = pos, k0 = koff;
                while (filled < 32 && at < nt && hdr[at].s12 == s12 && hdr[at].dbase == dbase) {
                    const int n = hdr[at].n34;
                    const int len = min(n - k0, 32 - filled);
                    if (lane >= filled && lane < filled + len) {
                        my_task = at;
                        my_k = k0 + lane - filled;
                    }
                    filled += len;
                    k0 += len;
                    if (k0 < n) break;   // this task goes on in the next pack
                    ++at;
                    k0 = 0;
                }
                pos = at;
                koff = k0;
            }
            const bool in3 = my_task >= 0;
            float tlo = __int_as_float(0x7f800000), thi = 0.0f;
            double wsym = 1.0;
            R dRx = 0, dRy = 0, dRz = 0;
            int k3 = 0, c4 = 0;
            if (in3) {
                const KHdr& H = hdr[my_task];
                tlo = H.tlo;
                thi = H.thi;
                wsym = (double) H.wsym;
                dRx = (R) H.dRx;
                dRy = (R) H.dRy;
                dRz = (R) H.dRz;
                k3 = H.s34 + my_k;
                c4 = H.c4;
            }
            R Dblk[NG][N2 * N4];
#pragma unroll
            for (int g = 0; g < NG; ++g)
#pragma unroll
                for (int a = 0; a < N2; ++a)
#pragma unroll
                    for (int b = 0; b < N4; ++b)
                        Dblk[g][a * N4 + b] = in3 && (NG == 1 || g < dn)
                                                  ? (R) A.Dc[dbase + g][(long) (c2 + a) * A.ld4 + c4 + b] : R(0);
            {
                // partner 3 of this lane (all loads of the entry issue together)
                float b34 = 0.0f;
                R kab34 = 0, q = 1, iq = 1, Qx = 0, Qy = 0, Qz = 0, Cx = 0, Cy = 0, Cz = 0;
                int c3 = 0, c3b = -1;
                double w30 = 1.0, w31 = 0.0;
                if (in3) {
                    b34 = A.b34[k3];
                    kab34 = d34.kab[k3]; q = d34.p[k3]; iq = d34.ip[k3];
                    Qx = d34.px[k3]; Qy = d34.py[k3]; Qz = d34.pz[k3];
                    Cx = d34.ax[k3]; Cy = d34.ay[k3]; Cz = d34.az[k3];
                    c3 = A.cart34[k3];
                    if constexpr (G3 == 2) {
                        c3b = A.t1_34[k3];
                        w30 = A.w0_34[k3];
                        w31 = A.w1_34[k3];
                    }
                }
                // (every lane of a pack passes thre34 and the row's first partner 1)
                const bool v3 = in3;
                const R QCx = Qx - Cx, QCy = Qy - Cy, QCz = Qz - Cz;
                // ket side of PQ: (Q - R4) with the task's centre shift folded in
                const R Sx = dRx - Qx, Sy = dRy - Qy, Sz = dRz - Qz;
                // segment accumulators: acc for the segment's first target, accb for its
                // second (s-type partners 1 may stand for two contracted shells)
                R acc[NG][N1 * N3];
                R accb[NG][G1 == 2 ? N1 * N3 : 1];
#pragma unroll
                for (int g = 0; g < NG; ++g) {
#pragma unroll
                    for (int t = 0; t < N1 * N3; ++t) acc[g][t] = R(0);
#pragma unroll
                    for (int t = 0; t < (G1 == 2 ? N1 * N3 : 1); ++t) accb[g][t] = R(0);
                }
                bool any = false;
                int prev_seg = -1, prev_c1 = 0, prev_c1b = -1;
                // flush the finished shell segment of partner 1: one atomic per element, density
                // and target pair (fire-and-forget reductions; a segmented shuffle sum over the
                // lanes of one shell 3 before them measured slower)
                auto flush = [&]() {
                    if (any) {
#pragma unroll
                        for (int g = 0; g < NG; ++g) {
                            if (NG > 1 && g >= dn) break;   // (a pack of one density always has it)
                            double* Kc = A.Kc[dbase + g];
#pragma unroll
                            for (int a = 0; a < N1; ++a)
#pragma unroll
                                for (int c = 0; c < N3; ++c) {
                                    const double v = wsym * (double) acc[g][a * N3 + c];
                                    double* row = Kc + (long) (prev_c1 + a) * A.ld3;
                                    if constexpr (G3 == 2) {
                                        atomicAdd(row + c3 + c, w30 * v);
                                        if (c3b >= 0) atomicAdd(row + c3b + c, w31 * v);
                                    } else {
                                        atomicAdd(row + c3 + c, v);
                                    }
                                    acc[g][a * N3 + c] = R(0);
                                    if constexpr (G1 == 2) {
                                        if (prev_c1b >= 0) {
                                            const double vb = wsym * (double) accb[g][a * N3 + c];
                                            double* rowb = Kc + (long) (prev_c1b + a) * A.ld3;
                                            if constexpr (G3 == 2) {
                                                atomicAdd(rowb + c3 + c, w30 * vb);
                                                if (c3b >= 0) atomicAdd(rowb + c3b + c, w31 * vb);
                                            } else {
                                                atomicAdd(rowb + c3 + c, vb);
                                            }
                                        }
                                        accb[g][a * N3 + c] = R(0);
                                    }
                                }
                        }
                    }
                    any = false;
                };
                stage_ent(ring, d12, A.b12, A.cart12, A.t1_12, A.seg12, s12, 0, n12, lane);
                cp_async_commit();
                bool stop = false;
                for (int kb = 0; kb < n12 && !stop; kb += 32) {
                    const KEnt<R>* cur = ring + ((kb >> 5) & 1) * 32;
                    if (kb + 32 < n12)
                        stage_ent(ring + (((kb >> 5) + 1) & 1) * 32, d12, A.b12, A.cart12, A.t1_12, A.seg12, s12,
                                  kb + 32, n12, lane);
                    cp_async_commit();
                    cp_async_wait<1>();
                    __syncwarp();
                    const int kend = min(32, n12 - kb);
                    // chg bit l: entry l of the chunk starts a new shell segment (l >= 1)
                    const int cl = lane < kend ? cur[lane].seg : -1;
                    const int cl_prev = __shfl_up_sync(0xffffffffu, cl, 1);
                    const unsigned chg = __ballot_sync(0xffffffffu, lane >= 1 && lane < kend && cl != cl_prev);
                    for (int j = 0; j < kend; ++j) {
                        const float b12 = cur[j].b;
                        const int sg = cur[j].seg;
                        // can this lane's quartet reach its lower threshold (or any later one of the
                        // segment / of later segments, whose bounds are not larger)?
                        const float est = b12 * b34;
                        const bool can = v3 && est >= tlo;
                        const bool any_can = b12 >= thre12 && __any_sync(0xffffffffu, can);
                        if (sg != prev_seg) {
                            flush();
                            prev_seg = sg;
                            prev_c1 = cur[j].c;
                            if constexpr (G1 == 2) prev_c1b = cur[j].t1;
                            // segments are ordered by their largest bound: nothing later passes
                            if (!any_can) {
                                stop = true;
                                break;
                            }
                        } else if (!any_can) {
                            // entries of a segment are ordered by bound: skip the rest of this
                            // segment within the chunk (to the next segment start, or the chunk end)
                            const unsigned nxt = j == 31 ? 0u : (chg & ~((2u << j) - 1u));
                            j = (nxt ? __ffs(nxt) - 1 : kend) - 1;
                            continue;
                        }
                        const bool pass = can && est < thi;
                        if (!__any_sync(0xffffffffu, pass)) continue;
                        if (!pass) continue;
                        const KEnt<R> e = cur[j];
                        nq += dn;   // statistics count density-quartets
                        any = true;
                        if constexpr (G1 == 2) {
                            // one integral, added to both targets with the entry's weights
                            R tmp[NG][N1 * N3];
#pragma unroll
                            for (int g = 0; g < NG; ++g)
#pragma unroll
                                for (int t = 0; t < N1 * N3; ++t) tmp[g][t] = R(0);
                            k_quartet<L1, L2, L3, L4, R, NG>(A, tab, tmax, asym_t, asym_w, e, kab34, q, iq, Sx, Sy,
                                                             Sz, QCx, QCy, QCz, Cx, Cy, Cz, Dblk, tmp);
#pragma unroll
                            for (int g = 0; g < NG; ++g)
#pragma unroll
                                for (int t = 0; t < N1 * N3; ++t) {
                                    acc[g][t] = fma(e.w0, tmp[g][t], acc[g][t]);
                                    accb[g][t] = fma(e.w1, tmp[g][t], accb[g][t]);
                                }
                        } else {
                            k_quartet<L1, L2, L3, L4, R, NG>(A, tab, tmax, asym_t, asym_w, e, kab34, q, iq, Sx, Sy,
                                                             Sz, QCx, QCy, QCz, Cx, Cy, Cz, Dblk, acc);
                        }
                    }
                    __syncwarp();   // the next chunk's prefetch refills this slot
                }
                cp_async_wait<0>();
                __syncwarp();
                flush();
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) nq += __shfl_xor_sync(0xffffffffu, nq, o);
    if (lane == 0 && nq) atomicAdd(A.qcount, (unsigned long long) nq);
}

} // namespace lsjk

#include "kwarp.cuh"

namespace lsjk {

template <int L1, int L2, int L3, int L4, typename R, int NG, bool GC>
void launch_k_one(Context* ctx, const KArgs& A, unsigned grid)
{
    constexpr int NR = (L1 + L2 + L3 + L4) / 2 + 1;
    const size_t smem = (size_t) 2 * NR * A.nbin * 8 * sizeof(R);
    // the shared-memory opt-in is a per-device function attribute: set it once per
    // device, and read how many CTAs of this kernel fit on a multiprocessor
    static std::atomic<unsigned long long> attr_devices{0};
    static std::atomic<int> resident[64];
    const int dev = ctx->device & 63;
    const unsigned long long bit = 1ull << dev;
    auto kern = k_exchange<L1, L2, L3, L4, R, NG, GC>;
    if (!(attr_devices.load(std::memory_order_acquire) & bit)) {
        LSJK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
        int occ = 0;
        LSJK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kKThreads, smem));
        resident[dev].store(occ > 0 ? occ : 1, std::memory_order_relaxed);
        attr_devices.fetch_or(bit, std::memory_order_acq_rel);
    }
    // warps take tasks from the queue until it is empty, so CTAs beyond one
    // resident wave would only start, find no work and leave
    grid = std::min<unsigned>(grid, (unsigned) (ctx->nsm * resident[dev].load(std::memory_order_relaxed)));
    kern<<<grid, kKThreads, smem, ctx->stream>>>(A);
    LSJK_CUDA(cudaGetLastError());
    ctx->stats.kernel_launches++;
}

// The two-target variant only where an s-type partner can carry two targets.
template <int L1, int L2, int L3, int L4, typename R, int NG>
void launch_k_gc(Context* ctx, const KArgs& A, unsigned grid)
{
    if constexpr (L1 == 0 || L3 == 0) {
        if (A.gc) {
            launch_k_one<L1, L2, L3, L4, R, NG, true>(ctx, A, grid);
            return;
        }
    }
    launch_k_one<L1, L2, L3, L4, R, NG, false>(ctx, A, grid);
}

// One class, one precision pass, all A.ng densities in one launch: NG =
// k_batch densities per lane when a group holds that many, else 1, and the
// task list run once per sub-slot of NG densities of the groups.
template <int L1, int L2, int L3, int L4>
void launch_k(Context* ctx, const KArgs& A, long cap, bool fp32)
{
    if (cap == 0 || A.ng < 1) return;
    const int per_group = std::min(A.ng, kKBatch);
    int per_sm = ctx->tune.k_ctas_per_sm[fp32 ? 1 : 0][L1][L2][L3][L4];
    auto grid_for = [&](int nsub) {
        const long want = (cap * nsub + kKWarps - 1) / kKWarps;
        return (unsigned) std::min<long>(want, (long) ctx->nsm * (per_sm > 0 ? per_sm : 16));
    };
    KArgs B = A;
    if (fp32) {
        constexpr int NGf = k_batch<L1, L2, L3, L4, float>();
        if (NGf > 1 && per_group >= NGf) {
            B.nsub = (per_group + NGf - 1) / NGf;
            launch_k_gc<L1, L2, L3, L4, float, NGf>(ctx, B, grid_for(B.nsub));
        } else {
            B.nsub = per_group;
            launch_k_gc<L1, L2, L3, L4, float, 1>(ctx, B, grid_for(B.nsub));
        }
    } else {
        if constexpr (k_warp_class<L1, L2, L3, L4>() || k_warp_class_hi<L1, L2, L3, L4>()) {
            // heavy classes: a quartet per warp (partners with one output target; over
            // merged twins only s-type partners can carry two)
            if ((k_warp_class<L1, L2, L3, L4>() || A.split_hi) && (!A.gc || (L1 != 0 && L3 != 0))) {
                B.nsub = per_group;
                launch_k_warp<L1, L2, L3, L4>(ctx, B, cap * B.nsub, per_sm);
                return;
            }
        }
        constexpr int NGd = k_batch<L1, L2, L3, L4, double>();
        if (NGd > 1 && per_group >= NGd) {
            B.nsub = (per_group + NGd - 1) / NGd;
            launch_k_gc<L1, L2, L3, L4, double, NGd>(ctx, B, grid_for(B.nsub));
        } else {
            B.nsub = per_group;
            launch_k_gc<L1, L2, L3, L4, double, 1>(ctx, B, grid_for(B.nsub));
        }
    }
}

} // namespace lsjk
