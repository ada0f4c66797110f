// One-electron integrals on the device: the reference's IntBox::overlapCPU,
// kineticCPU and potentialCPU (src/cpp/intbox/cpu/overlap.cpp, kinetic.cpp,
// potential.cpp) over the same primitive pair lists, re-laid out as one
// thread per primitive pair and class.
//
// Each thread builds the McMurchie-Davidson expansion coefficients E^{ij}_t of
// its pair (hermite.cuh) and forms its Cartesian block:
//   S_ab = K_ab (pi/p)^{3/2} E^x_0 E^y_0 E^z_0
//   T_ab = sum_d T^d S^{d'} S^{d''},  T^d_{ij} = -2b^2 S_{i,j+2} + b(2j+1) S_ij - j(j-1)/2 S_{i,j-2}
//   V_ab = sum_C -Z_C sum_w a_w f_w 2 pi/p K_ab sum_tuv E^x_t E^y_u E^z_v R_tuv(p d2_w, P - C)
// (d2_w = w^2/(p + w^2), f_w = sqrt(d2_w) for an erf-attenuated term), and
// adds it with FP64 atomics into the Cartesian matrix (both triangles for a
// symmetric list, 1/2 on a primitive's pair with itself, as the reference's
// symmetric pair-list consumers). The pure transform follows on the device.
#include "engine.cuh"
#include "hermite.cuh"
#include "quartet_loops.cuh"   // herm_pos

namespace lsjk {

namespace {

enum OneKind { kOneS = 0, kOneT = 1, kOneV = 2 };

constexpr double kPi = 3.14159265358979323846;

struct OneArgs {
    const int* p1;
    const int* p2;
    long off, n;          // the class's slice of the sorted pair arrays
    BasisView b1, b2;
    int symm;
    double* X;            // Cartesian output, ncart1 x ncart2 (ld)
    int ld;
    const double* xyzc;   // potential: natom x (x, y, z, Z)
    int natom;
    int nterm;
    double alpha[4], omega[4];
    const double* boys;   // FP64 Boys table of order LA + LB
};

// Hermite Coulomb integrals R_tuv (t + u + v <= L) of exponent a at (X, Y, Z)
// from the Boys values F_0..F_L, by the downward recursion in n of
//   R^n_{t+1,u,v} = t R^{n+1}_{t-1,u,v} + X R^{n+1}_{t,u,v}   (likewise u, v),
//   R^n_{000} = (-2a)^n F_n,
// in place over one array in shell-major order (herm_pos): level n from level
// n + 1, top shell first, so the shells a step reads still hold level n + 1.
template <int L>
__device__ void hermite_R(double a, double X, double Y, double Z, const double* F, double* R)
{
    double f[L + 1];
    double pw = 1.0;
    for (int n = 0; n <= L; ++n) {
        f[n] = pw * F[n];
        pw *= -2.0 * a;
    }
    R[0] = f[L];
    for (int m = L - 1; m >= 0; --m) {
        for (int N = L - m; N >= 1; --N) {
            int k = nherm_of(N - 1);
            for (int i = 0; i <= N; ++i)
                for (int v = 0; v <= i; ++v, ++k) {
                    const int t = N - i, u = i - v;
                    double s;
                    if (t > 0) {
                        s = X * R[herm_pos(t - 1, u, v)];
                        if (t > 1) s += (t - 1) * R[herm_pos(t - 2, u, v)];
                    } else if (u > 0) {
                        s = Y * R[herm_pos(t, u - 1, v)];
                        if (u > 1) s += (u - 1) * R[herm_pos(t, u - 2, v)];
                    } else {
                        s = Z * R[herm_pos(t, u, v - 1)];
                        if (v > 1) s += (v - 1) * R[herm_pos(t, u, v - 2)];
                    }
                    R[k] = s;
                }
        }
        R[0] = f[m];
    }
}

template <int LA, int LB, int KIND>
__global__ void __launch_bounds__(128) k_oneint(const __grid_constant__ OneArgs A)
{
    constexpr int LBX = KIND == kOneT ? LB + 2 : LB;
    constexpr int NA = ncart_of(LA), NB = ncart_of(LB);
    const long k = blockIdx.x * (long) blockDim.x + threadIdx.x;
    if (k >= A.n) return;
    const int ia = A.p1[A.off + k], ib = A.p2[A.off + k];
    const double ea = A.b1.e[ia], eb = A.b2.e[ib];
    const double Ra[3] = {A.b1.x[ia], A.b1.y[ia], A.b1.z[ia]};
    const double Rb[3] = {A.b2.x[ib], A.b2.y[ib], A.b2.z[ib]};
    const double p = ea + eb, ip = 1.0 / p;
    double P[3], PA[3], PB[3], AB2 = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        P[d] = (ea * Ra[d] + eb * Rb[d]) * ip;
        PA[d] = P[d] - Ra[d];
        PB[d] = P[d] - Rb[d];
        AB2 += (Ra[d] - Rb[d]) * (Ra[d] - Rb[d]);
    }
    const double Kab = A.b1.c[ia] * A.b2.c[ib] * exp(-ea * eb * ip * AB2);
    ECoef<LA, LBX> E;
    build_E<LA, LBX>(p, PA, PB, E);
    const double scale = (A.symm && ia == ib) ? 0.5 : 1.0;
    double out[NA][NB];
    if (KIND == kOneS || KIND == kOneT) {
        const double s1 = sqrt(kPi * ip);
        auto S1 = [&](int d, int i, int j) { return j < 0 ? 0.0 : E.v[d][i][j][0] * s1; };
#pragma unroll
        for (int i = 0; i < NA; ++i)
#pragma unroll
            for (int j = 0; j < NB; ++j) {
                const int a[3] = {cart_lx(LA, i), cart_ly(LA, i), cart_lz(LA, i)};
                const int b[3] = {cart_lx(LB, j), cart_ly(LB, j), cart_lz(LB, j)};
                double s[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) s[d] = S1(d, a[d], b[d]);
                if (KIND == kOneS) {
                    out[i][j] = s[0] * s[1] * s[2];
                } else {
                    double t[3];
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        const int bj = b[d];
                        double v = -2.0 * eb * eb * S1(d, a[d], bj + 2) + eb * (2 * bj + 1) * s[d];
                        if (bj >= 2) v -= 0.5 * bj * (bj - 1) * S1(d, a[d], bj - 2);
                        t[d] = v;
                    }
                    out[i][j] = t[0] * s[1] * s[2] + s[0] * t[1] * s[2] + s[0] * s[1] * t[2];
                }
            }
    } else {
        constexpr int L = LA + LB, H = nherm_of(L);
        double Rs[H];
        for (int k = 0; k < H; ++k) Rs[k] = 0.0;
        double R[H];
        double F[L + 1];
        for (int C = 0; C < A.natom; ++C) {
            const double Zc = A.xyzc[4 * C + 3];
            if (Zc == 0.0) continue;
            const double X = P[0] - A.xyzc[4 * C], Y = P[1] - A.xyzc[4 * C + 1], Z = P[2] - A.xyzc[4 * C + 2];
            const double R2 = X * X + Y * Y + Z * Z;
            for (int w = 0; w < A.nterm; ++w) {
                const double al = A.alpha[w], om = A.omega[w];
                if (al == 0.0 || om == 0.0) continue;
                double d2 = 1.0, f = 1.0;
                if (om != -1.0) {
                    d2 = om * om / (p + om * om);
                    f = sqrt(d2);
                }
                boys_eval<L, double>(p * d2 * R2, A.boys, F);
                hermite_R<L>(p * d2, X, Y, Z, F, R);
                const double c = -Zc * al * f * 2.0 * kPi * ip;
                for (int k = 0; k < H; ++k) Rs[k] += c * R[k];
            }
        }
#pragma unroll
        for (int i = 0; i < NA; ++i)
#pragma unroll
            for (int j = 0; j < NB; ++j) {
                const int ax = cart_lx(LA, i), ay = cart_ly(LA, i), az = cart_lz(LA, i);
                const int bx = cart_lx(LB, j), by = cart_ly(LB, j), bz = cart_lz(LB, j);
                double v = 0.0;
                for (int t = 0; t <= ax + bx; ++t)
                    for (int u = 0; u <= ay + by; ++u)
                        for (int w = 0; w <= az + bz; ++w)
                            v += E.v[0][ax][bx][t] * E.v[1][ay][by][u] * E.v[2][az][bz][w] * Rs[herm_pos(t, u, w)];
                out[i][j] = v;
            }
    }
    const int ca = A.b1.cart[ia], cb = A.b2.cart[ib];
    const double fac = Kab * scale;
#pragma unroll
    for (int i = 0; i < NA; ++i)
#pragma unroll
        for (int j = 0; j < NB; ++j) {
            const double v = out[i][j] * fac;
            atomicAdd(&A.X[(long) (ca + i) * A.ld + cb + j], v);
            if (A.symm) atomicAdd(&A.X[(long) (cb + j) * A.ld + ca + i], v);
        }
}

template <int KIND>
void launch_one(Context* ctx, const OneArgs& A, int LA, int LB)
{
    const unsigned grid = (unsigned) ((A.n + 127) / 128);
    cudaStream_t s = ctx->stream;
#define LSJK_ONE(a, b)                                                     \
    if (LA == a && LB == b) {                                              \
        k_oneint<a, b, KIND><<<grid, 128, 0, s>>>(A);                      \
    }
#define LSJK_ONE_ROW(a) LSJK_ONE(a, 0) else LSJK_ONE(a, 1) else LSJK_ONE(a, 2) else LSJK_ONE(a, 3)
    LSJK_ONE_ROW(0) else LSJK_ONE_ROW(1) else LSJK_ONE_ROW(2) else LSJK_ONE_ROW(3) else
        throw Error(LSJK_ENOTSUPP, "one-electron integrals: shell above f");
#undef LSJK_ONE_ROW
#undef LSJK_ONE
    LSJK_CUDA(cudaGetLastError());
    ctx->stats.kernel_launches++;
}

} // namespace

void one_electron(Context* ctx, int kind, const PairList* pl, const Ewald* ew, const double* xyzc, int natom,
                  double* Xcart)
{
    if (ew && ew->alpha.size() > 4) throw Error(LSJK_EINVAL, "IntBox::potential: at most 4 Ewald terms");
    for (size_t c = 0; c + 1 < pl->cls_off.size(); ++c) {
        OneArgs A{};
        A.p1 = pl->p1.p;
        A.p2 = pl->p2.p;
        A.off = pl->cls_off[c];
        A.n = pl->cls_off[c + 1] - pl->cls_off[c];
        if (A.n == 0) continue;
        A.b1 = pl->b1->view();
        A.b2 = pl->b2->view();
        A.symm = pl->symm ? 1 : 0;
        A.X = Xcart;
        A.ld = pl->b2->ncart;
        const int LA = pl->cls_L1[c], LB = pl->cls_L2[c];
        if (kind == kOneV) {
            A.xyzc = xyzc;
            A.natom = natom;
            A.nterm = (int) ew->alpha.size();
            for (int t = 0; t < A.nterm; ++t) {
                A.alpha[t] = ew->alpha[t];
                A.omega[t] = ew->omega[t];
            }
            A.boys = ctx->boys64.p + (long) (LA + LB) * LSJK_BOYS_NBIN * 8;
            launch_one<kOneV>(ctx, A, LA, LB);
        } else if (kind == kOneT) {
            launch_one<kOneT>(ctx, A, LA, LB);
        } else {
            launch_one<kOneS>(ctx, A, LA, LB);
        }
    }
}

} // namespace lsjk
