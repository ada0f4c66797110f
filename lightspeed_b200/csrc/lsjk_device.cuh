// Device helpers shared by the J and K kernels: quadrature table evaluation,
// shared-memory staging of tables with the Blackwell bulk-copy engine (TMA,
// cp.async.bulk, no multicast), and the bounded-wait error protocol.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "tables/quad_tables.inc"

namespace lsjk {

// Error bits a kernel may set in its status word (read back by the host).
enum : int {
    kErrBulkTimeout = 1,   // a bulk copy into shared memory did not complete in time
    kErrBadClass    = 2,   // a kernel met an angular momentum class it was not built for
};

// Every spin-wait gives up after this many try_wait polls (each poll itself
// suspends for a hardware-chosen interval), so a lost copy ends the kernel
// with an error status instead of hanging the GPU.
constexpr long kMaxPolls = 1L << 22;

__device__ __forceinline__ unsigned smem_u32(const void* p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* mbar, unsigned parity)
{
    unsigned addr = smem_u32(mbar);
    for (long it = 0; it < kMaxPolls; ++it) {
        unsigned done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done) : "r"(addr), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

// Copy `bytes` (multiple of 16, both addresses 16-byte aligned) from global to
// shared memory with cp.async.bulk, completing on an mbarrier. Must be called
// by all threads of the CTA. Returns false (and sets kErrBulkTimeout in
// *status) if the copy did not land within the poll budget; callers then exit.
__device__ __forceinline__ bool stage_bulk(void* smem_dst, const void* gsrc, unsigned bytes,
                                           uint64_t* mbar, int* status)
{
    if (threadIdx.x == 0) {
        unsigned a = smem_u32(mbar);
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" :: "r"(a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n"
                     :: "r"(a), "r"(bytes) : "memory");
        const unsigned kChunk = 32768u;
        for (unsigned off = 0; off < bytes; off += kChunk) {
            unsigned n = (bytes - off < kChunk) ? (bytes - off) : kChunk;
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                :: "r"(smem_u32(static_cast<char*>(smem_dst) + off)),
                   "l"(static_cast<const char*>(gsrc) + off), "r"(n), "r"(a)
                : "memory");
        }
    }
    __syncthreads();
    bool ok = mbar_wait_bounded(mbar, 0);
    if (!ok) {
        atomicOr(status, kErrBulkTimeout);
        // the copy may still be in flight: wait once more (bounded) before the
        // CTA releases its shared memory
        mbar_wait_bounded(mbar, 0);
    }
    __syncthreads();
    return ok;
}

// Horner evaluation of the degree-7 per-bin polynomial from its 8 monomial
// coefficients. The coefficient blocks of the quadrature tables start on
// 32-byte (float) / 64-byte (double) boundaries, so they are fetched with
// 16-byte vector loads. (Estrin's scheme, three operations deep instead of
// seven, measured no faster in K and slower in J, whose quartets are bound by
// the FP64 pipe rather than by latency.)
__device__ __forceinline__ float horner8(const float* __restrict__ c, float x)
{
    const float4 lo = reinterpret_cast<const float4*>(c)[0];
    const float4 hi = reinterpret_cast<const float4*>(c)[1];
    float f = hi.w;
    f = fmaf(f, x, hi.z);
    f = fmaf(f, x, hi.y);
    f = fmaf(f, x, hi.x);
    f = fmaf(f, x, lo.w);
    f = fmaf(f, x, lo.z);
    f = fmaf(f, x, lo.y);
    f = fmaf(f, x, lo.x);
    return f;
}
__device__ __forceinline__ double horner8(const double* __restrict__ c, double x)
{
    const double2 c01 = reinterpret_cast<const double2*>(c)[0];
    const double2 c23 = reinterpret_cast<const double2*>(c)[1];
    const double2 c45 = reinterpret_cast<const double2*>(c)[2];
    const double2 c67 = reinterpret_cast<const double2*>(c)[3];
    double f = c67.y;
    f = fma(f, x, c67.x);
    f = fma(f, x, c45.y);
    f = fma(f, x, c45.x);
    f = fma(f, x, c23.y);
    f = fma(f, x, c23.x);
    f = fma(f, x, c01.y);
    f = fma(f, x, c01.x);
    return f;
}

// Ampere-style asynchronous global -> shared copies of 4 / 8 bytes (one
// thread each), grouped with commit/wait.
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem)
{
    const unsigned s = (unsigned) __cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem)
{
    const unsigned s = (unsigned) __cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Half-range Gauss-Hermite nodes and weights of the asymptotic Rys rules,
// [nrys][root], in constant memory (read with uniform indices).
static __constant__ double c_rys_asym_t[(LSJK_RYS_NMAX + 1) * LSJK_RYS_NMAX] = {LSJK_RYS_ASYM_T_LIST};
static __constant__ double c_rys_asym_w[(LSJK_RYS_NMAX + 1) * LSJK_RYS_NMAX] = {LSJK_RYS_ASYM_W_LIST};

// 1/sqrt(T) in FP64 for T > 0: the FP32 estimate refined by two Newton steps
// r <- r (3 - T r^2) / 2 (relative error ~1e-16; the FP32 paths' switch
// region never sees T near 0 or beyond the float range).
__device__ __forceinline__ double rsqrt_f64_newton(double T)
{
    double r = (double) rsqrtf((float) T);
    const double hT = 0.5 * T;
    r = r * fma(-hT * r, r, 1.5);
    r = r * fma(-hT * r, r, 1.5);
    return r;
}

__device__ __forceinline__ double dexp(double x) { return exp(x); }
__device__ __forceinline__ float dexp(float x) { return __expf(x); }
__device__ __forceinline__ double drsqrt(double x) { return rsqrt(x); }
__device__ __forceinline__ float drsqrt(float x) { return rsqrtf(x); }

// Boys functions F_0..F_L at T. `tab` holds the [bin][8] polynomial table of
// F_L on [0, LSJK_BOYS_TMAX). Below the table edge F_L comes from the table
// and the lower orders from the (stable) downward recursion
//   F_m = (2T F_{m+1} + e^{-T}) / (2m+1);
// above it F_0 = sqrt(pi/T)/2 and the upward recursion
//   F_{m+1} = ((2m+1) F_m - e^{-T}) / (2T)  (stable for T > L).
template <int L, typename R>
__device__ __forceinline__ void boys_eval(R T, const R* __restrict__ tab, R* __restrict__ F)
{
    const R tmax = R(LSJK_BOYS_TMAX);
    if (T < tmax) {
        const R u = T * R(LSJK_BOYS_NBIN / LSJK_BOYS_TMAX);
        int b = static_cast<int>(u);
        b = b < LSJK_BOYS_NBIN - 1 ? b : LSJK_BOYS_NBIN - 1;
        const R x = R(2) * (u - R(b)) - R(1);
        F[L] = horner8(tab + 8 * b, x);
        if (L > 0) {
            const R e = dexp(-T);
            const R T2 = T + T;
#pragma unroll
            for (int m = L - 1; m >= 0; --m) F[m] = fma(T2, F[m + 1], e) * (R(1) / R(2 * m + 1));
        }
    } else {
        const R r = drsqrt(T);
        F[0] = R(0.88622692545275801364908374167057259) * r;   // sqrt(pi)/2
        if (L > 0) {
            const R e = dexp(-T);
            const R h = R(0.5) * r * r;
#pragma unroll
            for (int m = 0; m < L; ++m) F[m + 1] = (R(2 * m + 1) * F[m] - e) * h;
        }
    }
}

// Rys roots (returned as t^2) and weights of the N-point rule at T. `tab` is the
// per-rule block [2N][nbin][8] (roots t, then ln w; for N = 1 the weight
// w = F_0(T) itself, so the one-root classes need no exponential);
// `asym_t/asym_w` hold the half-range Gauss-Hermite limit used for T >= tmax.
template <int N, typename R>
__device__ __forceinline__ void rys_eval(R T, const R* __restrict__ tab, int nbin, R tmax,
                                         const R* __restrict__ asym_t, const R* __restrict__ asym_w,
                                         R* __restrict__ t2, R* __restrict__ w)
{
    if (T < tmax) {
        const R u = T * (R(nbin) / tmax);
        int b = static_cast<int>(u);
        b = b < nbin - 1 ? b : nbin - 1;
        const R x = R(2) * (u - R(b)) - R(1);
#pragma unroll
        for (int i = 0; i < N; ++i) {
            const R t = horner8(tab + 8 * (i * nbin + b), x);
            t2[i] = t * t;
            const R lw = horner8(tab + 8 * ((N + i) * nbin + b), x);
            w[i] = N == 1 ? lw : dexp(lw);
        }
    } else {
        const R r = drsqrt(T);
#pragma unroll
        for (int i = 0; i < N; ++i) {
            const R t = asym_t[i] * r;
            t2[i] = t * t;
            w[i] = asym_w[i] * r;
        }
    }
}

// Boys values F_0..F_L at T >= LSJK_BOYS_TMAX - (one bin) by the FP64
// asymptotic form F_0 = sqrt(pi/T)/2 and the upward recursion with the exp(-T)
// term, rounded to FP32 (the FP32 J path from the last table bin on: over that
// bin the form already agrees with the exact function to ~1e-16 relative).
template <int L>
__device__ __forceinline__ void boys_asym_f64_to_f32(double T, float* __restrict__ F)
{
    const double r = rsqrt_f64_newton(T);
    double f = 0.88622692545275801364908374167057259 * r;   // sqrt(pi)/2 / sqrt(T)
    F[0] = (float) f;
    if (L > 0) {
        // exp(-T) <= 3e-16 here: its relative size in F_m is below 1e-10, so its own
        // FP32 rounding changes F_m by less than 1e-17 relative
        const double e = (double) __expf(-(float) T);
        const double h = 0.5 * r * r;
#pragma unroll
        for (int m = 0; m < L; ++m) {
            f = (double(2 * m + 1) * f - e) * h;
            F[m + 1] = (float) f;
        }
    }
}

// Cartesian component count of a shell and Hermite count of a pair.
__host__ __device__ constexpr int ncart_of(int L) { return (L + 1) * (L + 2) / 2; }
__host__ __device__ constexpr int nherm_of(int L) { return (L + 1) * (L + 2) * (L + 3) / 6; }

} // namespace lsjk
