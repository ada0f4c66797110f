/*
 * Test infrastructure only -- the oracle's CPU restatement of the reference
 * J/K path (Lightspeed IntBox::coulombCPU / exchangeCPU). Built by
 * oracle/Makefile into oracle/_ref/libjk_port.so; called from oracle/port.py
 * by the tests and never by the product.
 *
 * Screening and quartet sets follow the reference exactly:
 *   J (src/cpp/intbox/cpu/coulomb.cpp:14-196):
 *     max12 = max bra bound (pair_list_util.cpp:22-31);
 *     ket bound B34' = float(max|D_cart block| * B34), kept if > float(thresp/max12)
 *       (truncate_ket, pair_list_util.cpp:60-123, both triangles if symmetric);
 *     bra kept if bound >= float(thresp/max34) (truncate_bra, :32-59);
 *     quartet computed iff B12 * B34' >= thresp in float (coulomb.cpp:113-115);
 *     ket density symmetrised with 1/2 on diagonal primitive pairs and (-1)^t
 *     Hermite phases (hermite.cpp:146-154, :194-200); bra back-transform writes
 *     both triangles for symmetric lists (hermite.cpp:390-400).
 *   K (src/cpp/intbox/cpu/exchange.cpp:17-355, kvec.cpp:31-232):
 *     partners of prim2 from pl12 with bound >= float(thresp/(max34*D24max)),
 *     both orientations for symmetric lists (diagonal once);
 *     quartet computed iff double(float(b12*b34)) * max|D24 block| >= thresp;
 *     D24symm (and basis1 == basis3): prim2 <= prim4 only, transposed write.
 * The integrals themselves are McMurchie-Davidson Hermite integrals with Boys
 * functions (power series / asymptotic + recursions), which evaluate the same
 * quantities the reference's Rys quadratures do.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define LMAXP 4   /* per shell */
#define HMAX 1000

typedef struct {
    int nprim;
    const double *c, *e, *xyz;
    const int *L, *cart;
    int ncart;
} PBasis;

static int ncart_of(int L) { return (L + 1) * (L + 2) / 2; }

static void cart_exps(int L, int* lx, int* ly, int* lz)
{
    int k = 0;
    for (int i = 0; i <= L; ++i)
        for (int j = 0; j <= i; ++j) {
            lx[k] = L - i;
            ly[k] = i - j;
            lz[k] = j;
            ++k;
        }
}

/* Boys functions F_0..F_m(T) */
static void boys(int m, double T, double* F)
{
    double e = exp(-T);
    if (T < 30.0) {
        double term = 1.0 / (2 * m + 1), sum = term;
        for (int k = 1; k < 500; ++k) {
            term *= 2.0 * T / (2 * m + 2 * k + 1);
            sum += term;
            if (term < 1e-18 * sum) break;
        }
        F[m] = e * sum;
        for (int n = m - 1; n >= 0; --n) F[n] = (2.0 * T * F[n + 1] + e) / (2 * n + 1);
    } else {
        F[0] = 0.5 * sqrt(M_PI / T);
        for (int n = 0; n < m; ++n) F[n + 1] = ((2 * n + 1) * F[n] - e) / (2.0 * T);
    }
}

/* E[d][i][j][t], i <= la, j <= lb, t <= i + j */
#define EI(i, j, t) (((i) * (LMAXP + 1) + (j)) * (2 * LMAXP + 1) + (t))
static void hermite_E(int la, int lb, double p, const double* PA, const double* PB, double* E /* 3 x ... */)
{
    const int sz = (LMAXP + 1) * (LMAXP + 1) * (2 * LMAXP + 1);
    memset(E, 0, sizeof(double) * 3 * sz);
    double h = 0.5 / p;
    for (int d = 0; d < 3; ++d) {
        double* Ed = E + d * sz;
        Ed[EI(0, 0, 0)] = 1.0;
        for (int i = 0; i < la; ++i)
            for (int t = 0; t <= i + 1; ++t) {
                double s = PA[d] * Ed[EI(i, 0, t)];
                if (t > 0) s += h * Ed[EI(i, 0, t - 1)];
                if (t + 1 <= i) s += (t + 1) * Ed[EI(i, 0, t + 1)];
                Ed[EI(i + 1, 0, t)] = s;
            }
        for (int j = 0; j < lb; ++j)
            for (int i = 0; i <= la; ++i)
                for (int t = 0; t <= i + j + 1; ++t) {
                    double s = PB[d] * Ed[EI(i, j, t)];
                    if (t > 0) s += h * Ed[EI(i, j, t - 1)];
                    if (t + 1 <= i + j) s += (t + 1) * Ed[EI(i, j, t + 1)];
                    Ed[EI(i, j + 1, t)] = s;
                }
    }
}

/* R_{tuv} (n = 0) for t+u+v <= L into R[(t*V+u)*V+v], V = L+1; includes the
 * factor f and the scaled exponent a. */
static void hermite_R(int L, double a, double X, double Y, double Z, double f, double T, double* R)
{
    int V = L + 1;
    static __thread double Rn[(2 * 2 * LMAXP + 1) * 17 * 17 * 17];
    double F[4 * LMAXP + 2];
    boys(L, T, F);
    double pw = f;
    for (int n = 0; n <= L; ++n) {
        Rn[((n * V + 0) * V + 0) * V + 0] = pw * F[n];
        pw *= -2.0 * a;
    }
    for (int n = L - 1; n >= 0; --n) {
        int top = L - n;
        for (int t = 0; t <= top; ++t)
            for (int u = 0; u + t <= top; ++u)
                for (int v = 0; v + u + t <= top; ++v) {
                    if (t + u + v == 0) continue;
                    double s;
#define RN(nn, tt, uu, vv) Rn[((((nn) * V + (tt)) * V + (uu)) * V) + (vv)]
                    if (t > 0) {
                        s = X * RN(n + 1, t - 1, u, v);
                        if (t > 1) s += (t - 1) * RN(n + 1, t - 2, u, v);
                    } else if (u > 0) {
                        s = Y * RN(n + 1, t, u - 1, v);
                        if (u > 1) s += (u - 1) * RN(n + 1, t, u - 2, v);
                    } else {
                        s = Z * RN(n + 1, t, u, v - 1);
                        if (v > 1) s += (v - 1) * RN(n + 1, t, u, v - 2);
                    }
                    RN(n, t, u, v) = s;
                }
    }
    for (int t = 0; t <= L; ++t)
        for (int u = 0; u + t <= L; ++u)
            for (int v = 0; v + u + t <= L; ++v) R[(t * V + u) * V + v] = RN(0, t, u, v);
#undef RN
}

static double max_bound(long n, const float* b)
{
    double m = 0.0;
    for (long k = 0; k < n; ++k)
        if (b[k] > m) m = b[k];
    return m;
}

/* ---------------------------------------------------------------------- J */

/* Hermite coefficients of a pair block: out[t] (t over |t| <= L1+L2 in
 * shell-major lexical order) = pre * sum_ab E_t^{ab} X[a][b]. */
static int herm_index(int tx, int ty, int tz)
{
    int L = tx + ty + tz;
    int base = L * (L + 1) * (L + 2) / 6;
    int i = L - tx;            /* CCA position within shell L */
    return base + i * (i + 1) / 2 + tz;
}

int port_coulomb(const PBasis* b1, const PBasis* b2, long n12, const int* p12a, const int* p12b,
                 const float* bnd12, int symm12, const PBasis* b3, const PBasis* b4, long n34,
                 const int* p34a, const int* p34b, const float* bnd34, int symm34, const double* D34c,
                 int nterm, const double* scales, const double* omegas, float thresp, double* J12c)
{
    const double max12 = max_bound(n12, bnd12);
    const float thre_ket = (float) ((double) thresp / max12);
    float* B34 = (float*) malloc(sizeof(float) * (n34 ? n34 : 1));
    int* keep34 = (int*) malloc(sizeof(int) * (n34 ? n34 : 1));
    double max34 = 0.0;
    const int ld4 = b4->ncart;
    for (long k = 0; k < n34; ++k) {
        int i = p34a[k], j = p34b[k];
        int a1 = b3->cart[i], a2 = b4->cart[j], c1 = ncart_of(b3->L[i]), c2 = ncart_of(b4->L[j]);
        double v = 0.0;
        for (int x = 0; x < c1; ++x)
            for (int y = 0; y < c2; ++y) {
                double d = fabs(D34c[(long) (a1 + x) * ld4 + a2 + y]);
                if (d > v) v = d;
                if (symm34) {
                    d = fabs(D34c[(long) (a2 + y) * ld4 + a1 + x]);
                    if (d > v) v = d;
                }
            }
        B34[k] = (float) (v * (double) bnd34[k]);
        keep34[k] = B34[k] > thre_ket;
        if (keep34[k] && B34[k] > max34) max34 = B34[k];
    }
    const float thre_bra = (float) ((double) thresp / max34);
    /* ket Hermite densities */
    const int HK = 35;
    double* dk = (double*) calloc((size_t) (n34 ? n34 : 1) * HK, sizeof(double));
    double* kg = (double*) calloc((size_t) (n34 ? n34 : 1) * 4, sizeof(double));
    for (long k = 0; k < n34; ++k) {
        if (!keep34[k]) continue;
        int i = p34a[k], j = p34b[k], la = b3->L[i], lb = b4->L[j];
        double e1 = b3->e[i], e2 = b4->e[j], q = e1 + e2;
        const double *A = b3->xyz + 3 * i, *B = b4->xyz + 3 * j;
        double Q[3], QA[3], QB[3], R2 = 0.0;
        for (int d = 0; d < 3; ++d) {
            Q[d] = (e1 * A[d] + e2 * B[d]) / q;
            QA[d] = Q[d] - A[d];
            QB[d] = Q[d] - B[d];
            R2 += (A[d] - B[d]) * (A[d] - B[d]);
        }
        double Kab = b3->c[i] * b4->c[j] * exp(-e1 * e2 / q * R2);
        double E[3 * (LMAXP + 1) * (LMAXP + 1) * (2 * LMAXP + 1)];
        const int sz = (LMAXP + 1) * (LMAXP + 1) * (2 * LMAXP + 1);
        hermite_E(la, lb, q, QA, QB, E);
        int lx1[15], ly1[15], lz1[15], lx2[15], ly2[15], lz2[15];
        cart_exps(la, lx1, ly1, lz1);
        cart_exps(lb, lx2, ly2, lz2);
        int a1 = b3->cart[i], a2 = b4->cart[j];
        double scale = (symm34 && i == j) ? 0.5 : 1.0;
        for (int x = 0; x < ncart_of(la); ++x)
            for (int y = 0; y < ncart_of(lb); ++y) {
                double Dv = D34c[(long) (a1 + x) * ld4 + a2 + y];
                if (symm34) Dv += D34c[(long) (a2 + y) * ld4 + a1 + x];
                Dv *= scale;
                for (int tx = 0; tx <= lx1[x] + lx2[y]; ++tx)
                    for (int ty = 0; ty <= ly1[x] + ly2[y]; ++ty)
                        for (int tz = 0; tz <= lz1[x] + lz2[y]; ++tz) {
                            double sign = ((tx + ty + tz) & 1) ? -1.0 : 1.0;
                            dk[k * HK + herm_index(tx, ty, tz)] += sign * Kab * E[EI(lx1[x], lx2[y], tx)] *
                                E[sz + EI(ly1[x], ly2[y], ty)] * E[2 * sz + EI(lz1[x], lz2[y], tz)] * Dv;
                        }
            }
        kg[4 * k] = q;
        kg[4 * k + 1] = Q[0];
        kg[4 * k + 2] = Q[1];
        kg[4 * k + 3] = Q[2];
    }
    const int ld2 = b2->ncart;
#pragma omp parallel for schedule(dynamic, 16)
    for (long k12 = 0; k12 < n12; ++k12) {
        if (bnd12[k12] < thre_bra) continue;
        int i = p12a[k12], j = p12b[k12], la = b1->L[i], lb = b2->L[j], LB = la + lb;
        double e1 = b1->e[i], e2 = b2->e[j], p = e1 + e2;
        const double *A = b1->xyz + 3 * i, *B = b2->xyz + 3 * j;
        double P[3], PA[3], PB[3], R2 = 0.0;
        for (int d = 0; d < 3; ++d) {
            P[d] = (e1 * A[d] + e2 * B[d]) / p;
            PA[d] = P[d] - A[d];
            PB[d] = P[d] - B[d];
            R2 += (A[d] - B[d]) * (A[d] - B[d]);
        }
        double jp[35];
        memset(jp, 0, sizeof jp);
        double R[17 * 17 * 17];
        for (long k34 = 0; k34 < n34; ++k34) {
            if (!keep34[k34]) continue;
            if (bnd12[k12] * B34[k34] < thresp) continue;
            int LK = b3->L[p34a[k34]] + b4->L[p34b[k34]], L = LB + LK, V = L + 1;
            double q = kg[4 * k34];
            double X = P[0] - kg[4 * k34 + 1], Y = P[1] - kg[4 * k34 + 2], Z = P[2] - kg[4 * k34 + 3];
            double rho = p * q / (p + q), PQ2 = X * X + Y * Y + Z * Z;
            for (int w = 0; w < nterm; ++w) {
                double al = scales[w], om = omegas[w];
                if (al == 0.0 || om == 0.0) continue;
                double d2 = 1.0, f = al * 2.0 * pow(M_PI, 2.5) / (p * q * sqrt(p + q));
                if (om != -1.0) {
                    d2 = om * om / (rho + om * om);
                    f *= sqrt(d2);
                }
                hermite_R(L, rho * d2, X, Y, Z, f, rho * d2 * PQ2, R);
                for (int tx = 0; tx <= LB; ++tx)
                    for (int ty = 0; tx + ty <= LB; ++ty)
                        for (int tz = 0; tx + ty + tz <= LB; ++tz) {
                            double s = 0.0;
                            for (int ux = 0; ux <= LK; ++ux)
                                for (int uy = 0; ux + uy <= LK; ++uy)
                                    for (int uz = 0; ux + uy + uz <= LK; ++uz)
                                        s += R[((tx + ux) * V + ty + uy) * V + tz + uz] *
                                             dk[k34 * HK + herm_index(ux, uy, uz)];
                            jp[herm_index(tx, ty, tz)] += s;
                        }
            }
        }
        /* bra back-transform */
        double Kab = b1->c[i] * b2->c[j] * exp(-e1 * e2 / p * R2);
        double E[3 * (LMAXP + 1) * (LMAXP + 1) * (2 * LMAXP + 1)];
        const int sz = (LMAXP + 1) * (LMAXP + 1) * (2 * LMAXP + 1);
        hermite_E(la, lb, p, PA, PB, E);
        int lx1[15], ly1[15], lz1[15], lx2[15], ly2[15], lz2[15];
        cart_exps(la, lx1, ly1, lz1);
        cart_exps(lb, lx2, ly2, lz2);
        int a1 = b1->cart[i], a2 = b2->cart[j];
        double scale = (symm12 && i == j) ? 0.5 : 1.0;
        for (int x = 0; x < ncart_of(la); ++x)
            for (int y = 0; y < ncart_of(lb); ++y) {
                double v = 0.0;
                for (int tx = 0; tx <= lx1[x] + lx2[y]; ++tx)
                    for (int ty = 0; ty <= ly1[x] + ly2[y]; ++ty)
                        for (int tz = 0; tz <= lz1[x] + lz2[y]; ++tz)
                            v += E[EI(lx1[x], lx2[y], tx)] * E[sz + EI(ly1[x], ly2[y], ty)] *
                                 E[2 * sz + EI(lz1[x], lz2[y], tz)] * jp[herm_index(tx, ty, tz)];
                v *= Kab * scale;
#pragma omp atomic
                J12c[(long) (a1 + x) * ld2 + a2 + y] += v;
                if (symm12) {
#pragma omp atomic
                    J12c[(long) (a2 + y) * ld2 + a1 + x] += v;
                }
            }
    }
    free(B34);
    free(keep34);
    free(dk);
    free(kg);
    return 0;
}

/* ---------------------------------------------------------------------- K */

typedef struct {
    int idx, part;
    float b;
} KEnt;

/* partner rows: for every primitive of the indexed basis, its partners sorted
 * by bound desc, partner asc (kvec.cpp:17-27), with bound >= thre. */
static int cmp_kent(const void* x, const void* y)
{
    const KEnt *a = (const KEnt*) x, *b = (const KEnt*) y;
    if (a->idx != b->idx) return a->idx < b->idx ? -1 : 1;
    if (a->b != b->b) return a->b > b->b ? -1 : 1;
    return a->part < b->part ? -1 : (a->part > b->part);
}

static KEnt* kinv(long n, const int* pa, const int* pb, const float* bnd, int symm, float thre, long* nent)
{
    KEnt* e = (KEnt*) malloc(sizeof(KEnt) * (2 * n + 1));
    long m = 0;
    for (long k = 0; k < n; ++k) {
        if (bnd[k] < thre) continue;
        e[m].idx = pb[k]; e[m].part = pa[k]; e[m].b = bnd[k]; ++m;
        if (symm && pa[k] != pb[k]) { e[m].idx = pa[k]; e[m].part = pb[k]; e[m].b = bnd[k]; ++m; }
    }
    qsort(e, m, sizeof(KEnt), cmp_kent);
    *nent = m;
    return e;
}

/* full primitive ERI block (ab|cd), row-major [a][b][c][d] */
static void eri_block(const PBasis* B1, int i1, const PBasis* B2, int i2, const PBasis* B3, int i3,
                      const PBasis* B4, int i4, int nterm, const double* scales, const double* omegas, double* out)
{
    int l1 = B1->L[i1], l2 = B2->L[i2], l3 = B3->L[i3], l4 = B4->L[i4];
    int n1 = ncart_of(l1), n2 = ncart_of(l2), n3 = ncart_of(l3), n4 = ncart_of(l4);
    double e1 = B1->e[i1], e2 = B2->e[i2], e3 = B3->e[i3], e4 = B4->e[i4];
    const double *A = B1->xyz + 3 * i1, *Bc = B2->xyz + 3 * i2, *C = B3->xyz + 3 * i3, *D = B4->xyz + 3 * i4;
    double p = e1 + e2, q = e3 + e4, P[3], Q[3], PA[3], PB[3], QC[3], QD[3], AB2 = 0, CD2 = 0;
    for (int d = 0; d < 3; ++d) {
        P[d] = (e1 * A[d] + e2 * Bc[d]) / p;
        Q[d] = (e3 * C[d] + e4 * D[d]) / q;
        PA[d] = P[d] - A[d]; PB[d] = P[d] - Bc[d]; QC[d] = Q[d] - C[d]; QD[d] = Q[d] - D[d];
        AB2 += (A[d] - Bc[d]) * (A[d] - Bc[d]);
        CD2 += (C[d] - D[d]) * (C[d] - D[d]);
    }
    double Kab = B1->c[i1] * B2->c[i2] * exp(-e1 * e2 / p * AB2);
    double Kcd = B3->c[i3] * B4->c[i4] * exp(-e3 * e4 / q * CD2);
    const int sz = (LMAXP + 1) * (LMAXP + 1) * (2 * LMAXP + 1);
    double Eab[3 * (LMAXP + 1) * (LMAXP + 1) * (2 * LMAXP + 1)], Ecd[3 * (LMAXP + 1) * (LMAXP + 1) * (2 * LMAXP + 1)];
    hermite_E(l1, l2, p, PA, PB, Eab);
    hermite_E(l3, l4, q, QC, QD, Ecd);
    int L = l1 + l2 + l3 + l4, V = L + 1;
    double X = P[0] - Q[0], Y = P[1] - Q[1], Z = P[2] - Q[2], rho = p * q / (p + q), PQ2 = X * X + Y * Y + Z * Z;
    double R[17 * 17 * 17], Rs[17 * 17 * 17];
    memset(Rs, 0, sizeof(double) * V * V * V);
    for (int w = 0; w < nterm; ++w) {
        double al = scales[w], om = omegas[w];
        if (al == 0.0 || om == 0.0) continue;
        double d2 = 1.0, f = al * 2.0 * pow(M_PI, 2.5) / (p * q * sqrt(p + q)) * Kab * Kcd;
        if (om != -1.0) {
            d2 = om * om / (rho + om * om);
            f *= sqrt(d2);
        }
        hermite_R(L, rho * d2, X, Y, Z, f, rho * d2 * PQ2, R);
        for (int t = 0; t < V * V * V; ++t) Rs[t] += R[t];
    }
    int lx1[15], ly1[15], lz1[15], lx2[15], ly2[15], lz2[15], lx3[15], ly3[15], lz3[15], lx4[15], ly4[15], lz4[15];
    cart_exps(l1, lx1, ly1, lz1); cart_exps(l2, lx2, ly2, lz2);
    cart_exps(l3, lx3, ly3, lz3); cart_exps(l4, lx4, ly4, lz4);
    for (int a = 0; a < n1; ++a)
        for (int b = 0; b < n2; ++b)
            for (int c = 0; c < n3; ++c)
                for (int d = 0; d < n4; ++d) {
                    double s = 0.0;
                    for (int tx = 0; tx <= lx1[a] + lx2[b]; ++tx)
                        for (int ty = 0; ty <= ly1[a] + ly2[b]; ++ty)
                            for (int tz = 0; tz <= lz1[a] + lz2[b]; ++tz) {
                                double et = Eab[EI(lx1[a], lx2[b], tx)] * Eab[sz + EI(ly1[a], ly2[b], ty)] *
                                            Eab[2 * sz + EI(lz1[a], lz2[b], tz)];
                                for (int ux = 0; ux <= lx3[c] + lx4[d]; ++ux)
                                    for (int uy = 0; uy <= ly3[c] + ly4[d]; ++uy)
                                        for (int uz = 0; uz <= lz3[c] + lz4[d]; ++uz) {
                                            double sign = ((ux + uy + uz) & 1) ? -1.0 : 1.0;
                                            s += et * sign * Ecd[EI(lx3[c], lx4[d], ux)] *
                                                 Ecd[sz + EI(ly3[c], ly4[d], uy)] * Ecd[2 * sz + EI(lz3[c], lz4[d], uz)] *
                                                 Rs[((tx + ux) * V + ty + uy) * V + tz + uz];
                                        }
                            }
                    out[((a * n2 + b) * n3 + c) * n4 + d] = s;
                }
}

int port_exchange(const PBasis* b1, const PBasis* b2, long n12, const int* p12a, const int* p12b,
                  const float* bnd12, int symm12, const PBasis* b3, const PBasis* b4, long n34,
                  const int* p34a, const int* p34b, const float* bnd34, int symm34, const double* D24c,
                  int d24symm, int nterm, const double* scales, const double* omegas, float thresp,
                  double* K13c)
{
    const long nD = (long) b2->ncart * b4->ncart;
    double dmax = 0.0;
    for (long k = 0; k < nD; ++k)
        if (fabs(D24c[k]) > dmax) dmax = fabs(D24c[k]);
    const float thre12 = (float) ((double) thresp / (max_bound(n34, bnd34) * dmax));
    const float thre34 = (float) ((double) thresp / (max_bound(n12, bnd12) * dmax));
    long m12, m34;
    KEnt* e12 = kinv(n12, p12a, p12b, bnd12, symm12, thre12, &m12);
    KEnt* e34 = kinv(n34, p34a, p34b, bnd34, symm34, thre34, &m34);
    /* row starts per indexed primitive */
    long* r12 = (long*) calloc(b2->nprim + 1, sizeof(long));
    long* r34 = (long*) calloc(b4->nprim + 1, sizeof(long));
    for (long k = 0; k < m12; ++k) r12[e12[k].idx + 1]++;
    for (long k = 0; k < m34; ++k) r34[e34[k].idx + 1]++;
    for (int k = 0; k < b2->nprim; ++k) r12[k + 1] += r12[k];
    for (int k = 0; k < b4->nprim; ++k) r34[k + 1] += r34[k];
    const int ld4 = b4->ncart, ld3 = b3->ncart;
#pragma omp parallel for schedule(dynamic)
    for (long t = 0; t < (long) b2->nprim * b4->nprim; ++t) {
        int i2 = (int) (t / b4->nprim), i4 = (int) (t % b4->nprim);
        if (d24symm && i2 > i4) continue;
        int flip = d24symm && i2 != i4;
        int l2 = b2->L[i2], l4 = b4->L[i4], n2 = ncart_of(l2), n4 = ncart_of(l4);
        int c2 = b2->cart[i2], c4 = b4->cart[i4];
        double Dv = 0.0;
        for (int a = 0; a < n2; ++a)
            for (int b = 0; b < n4; ++b)
                if (fabs(D24c[(long) (c2 + a) * ld4 + c4 + b]) > Dv) Dv = fabs(D24c[(long) (c2 + a) * ld4 + c4 + b]);
        double eri[6 * 6 * 6 * 6];
        for (long k1 = r12[i2]; k1 < r12[i2 + 1]; ++k1) {
            for (long k3 = r34[i4]; k3 < r34[i4 + 1]; ++k3) {
                if ((double) (e12[k1].b * e34[k3].b) * Dv < (double) thresp) continue;
                int i1 = e12[k1].part, i3 = e34[k3].part;
                int n1 = ncart_of(b1->L[i1]), n3 = ncart_of(b3->L[i3]);
                eri_block(b1, i1, b2, i2, b3, i3, b4, i4, nterm, scales, omegas, eri);
                int c1 = b1->cart[i1], c3 = b3->cart[i3];
                for (int a = 0; a < n1; ++a)
                    for (int c = 0; c < n3; ++c) {
                        double s = 0.0;
                        for (int b = 0; b < n2; ++b)
                            for (int d = 0; d < n4; ++d)
                                s += eri[((a * n2 + b) * n3 + c) * n4 + d] * D24c[(long) (c2 + b) * ld4 + c4 + d];
#pragma omp atomic
                        K13c[(long) (c1 + a) * ld3 + c3 + c] += s;
                        if (flip) {
#pragma omp atomic
                            K13c[(long) (c3 + c) * ld3 + c1 + a] += s;
                        }
                    }
            }
        }
    }
    free(e12);
    free(e34);
    free(r12);
    free(r34);
    return 0;
}

/* ---------------------------------------------------------------- pairs */

/* Schwarz bound of a primitive pair (pair_list.cpp:15-27), same operation order. */
float port_schwarz(double c1, double e1, const double* r1, double c2, double e2, const double* r2)
{
    double R2 = 0.0;
    R2 += pow(r1[0] - r2[0], 2);
    R2 += pow(r1[1] - r2[1], 2);
    R2 += pow(r1[2] - r2[2], 2);
    return (float) (fabs(c1 * c2) * exp(-e1 * e2 / (e1 + e2) * R2) * pow(2.0, 0.25) * pow(M_PI / (e1 + e2), 1.25));
}

/* All primitive pairs with bound > thre (prim2 <= prim1 if symmetric), in
 * row-major (prim1, prim2) order; returns the count. Arrays need n1*n2 room. */
long port_pairs(const PBasis* b1, const PBasis* b2, int symm, float thre, int* pa, int* pb, float* bnd)
{
    long m = 0;
    for (int i = 0; i < b1->nprim; ++i)
        for (int j = 0; j < b2->nprim; ++j) {
            if (symm && j > i) continue;
            float b = port_schwarz(b1->c[i], b1->e[i], b1->xyz + 3 * i, b2->c[j], b2->e[j], b2->xyz + 3 * j);
            if (b > thre) {
                pa[m] = i;
                pb[m] = j;
                bnd[m] = b;
                ++m;
            }
        }
    return m;
}

/* ------------------------------------------------------- quartet counts */

/* Number of primitive quartets the reference J and K evaluate for these pair
 * lists, density (Cartesian) and thresholds -- the same screening as
 * port_coulomb / port_exchange, without the integrals. Bra/ket loops use the
 * bound ordering (binary search over the float-product condition, which is
 * monotone), so this stays cheap at 1e5 pairs. */
static int cmp_float_desc(const void* x, const void* y)
{
    float a = *(const float*) x, b = *(const float*) y;
    return a > b ? -1 : (a < b);
}

/* count of leading entries v[k] (sorted desc) with (double)(float(b*v[k]))*s >= thr */
static long count_prefix(const float* v, long n, float b, double s, float thr)
{
    long lo = 0, hi = n;
    while (lo < hi) {
        long mid = (lo + hi) / 2;
        if ((double) (b * v[mid]) * s >= (double) thr) lo = mid + 1; else hi = mid;
    }
    return lo;
}

double port_count_j(const PBasis* b1, const PBasis* b2, long n12, const int* p12a, const int* p12b,
                    const float* bnd12, int symm12, const PBasis* b3, const PBasis* b4, long n34,
                    const int* p34a, const int* p34b, const float* bnd34, int symm34, const double* D34c,
                    float thresp)
{
    (void) b1; (void) b2; (void) p12a; (void) p12b; (void) symm12;
    const double max12 = max_bound(n12, bnd12);
    const float thre_ket = (float) ((double) thresp / max12);
    float* B34 = (float*) malloc(sizeof(float) * (n34 ? n34 : 1));
    long nk = 0;
    double max34 = 0.0;
    const int ld4 = b4->ncart;
    for (long k = 0; k < n34; ++k) {
        int i = p34a[k], j = p34b[k];
        int a1 = b3->cart[i], a2 = b4->cart[j], c1 = ncart_of(b3->L[i]), c2 = ncart_of(b4->L[j]);
        double v = 0.0;
        for (int x = 0; x < c1; ++x)
            for (int y = 0; y < c2; ++y) {
                double d = fabs(D34c[(long) (a1 + x) * ld4 + a2 + y]);
                if (d > v) v = d;
                if (symm34) {
                    d = fabs(D34c[(long) (a2 + y) * ld4 + a1 + x]);
                    if (d > v) v = d;
                }
            }
        float B2 = (float) (v * (double) bnd34[k]);
        if (B2 > thre_ket) {
            B34[nk++] = B2;
            if (B2 > max34) max34 = B2;
        }
    }
    qsort(B34, nk, sizeof(float), cmp_float_desc);
    const float thre_bra = (float) ((double) thresp / max34);
    double total = 0.0;
    for (long k = 0; k < n12; ++k) {
        if (bnd12[k] < thre_bra) continue;
        /* B12 * B34 >= thresp in float */
        long lo = 0, hi = nk;
        while (lo < hi) {
            long mid = (lo + hi) / 2;
            if (bnd12[k] * B34[mid] >= thresp) lo = mid + 1; else hi = mid;
        }
        total += (double) lo;
    }
    free(B34);
    return total;
}

double port_count_k(const PBasis* b1, const PBasis* b2, long n12, const int* p12a, const int* p12b,
                    const float* bnd12, int symm12, const PBasis* b3, const PBasis* b4, long n34,
                    const int* p34a, const int* p34b, const float* bnd34, int symm34, const double* D24c,
                    int d24symm, float thresp)
{
    (void) b1; (void) b3;
    const long nD = (long) b2->ncart * b4->ncart;
    double dmax = 0.0;
    for (long k = 0; k < nD; ++k)
        if (fabs(D24c[k]) > dmax) dmax = fabs(D24c[k]);
    const float thre12 = (float) ((double) thresp / (max_bound(n34, bnd34) * dmax));
    const float thre34 = (float) ((double) thresp / (max_bound(n12, bnd12) * dmax));
    long m12, m34;
    KEnt* e12 = kinv(n12, p12a, p12b, bnd12, symm12, thre12, &m12);
    KEnt* e34 = kinv(n34, p34a, p34b, bnd34, symm34, thre34, &m34);
    long* r12 = (long*) calloc(b2->nprim + 1, sizeof(long));
    long* r34 = (long*) calloc(b4->nprim + 1, sizeof(long));
    for (long k = 0; k < m12; ++k) r12[e12[k].idx + 1]++;
    for (long k = 0; k < m34; ++k) r34[e34[k].idx + 1]++;
    for (int k = 0; k < b2->nprim; ++k) r12[k + 1] += r12[k];
    for (int k = 0; k < b4->nprim; ++k) r34[k + 1] += r34[k];
    float* b34s = (float*) malloc(sizeof(float) * (m34 ? m34 : 1));
    for (long k = 0; k < m34; ++k) b34s[k] = e34[k].b;
    const int ld4 = b4->ncart;
    double total = 0.0;
#pragma omp parallel for schedule(dynamic) reduction(+ : total)
    for (long t = 0; t < (long) b2->nprim * b4->nprim; ++t) {
        int i2 = (int) (t / b4->nprim), i4 = (int) (t % b4->nprim);
        if (d24symm && i2 > i4) continue;
        int n2 = ncart_of(b2->L[i2]), n4 = ncart_of(b4->L[i4]);
        int c2 = b2->cart[i2], c4 = b4->cart[i4];
        double Dv = 0.0;
        for (int a = 0; a < n2; ++a)
            for (int b = 0; b < n4; ++b)
                if (fabs(D24c[(long) (c2 + a) * ld4 + c4 + b]) > Dv) Dv = fabs(D24c[(long) (c2 + a) * ld4 + c4 + b]);
        /* partners of each class are mixed in a row here: count per partner */
        for (long k1 = r12[i2]; k1 < r12[i2 + 1]; ++k1) {
            long n = 0;
            for (long k3 = r34[i4]; k3 < r34[i4 + 1]; ++k3)
                if ((double) (e12[k1].b * b34s[k3]) * Dv >= (double) thresp) ++n;
            total += (double) n;
        }
    }
    free(e12); free(e34); free(r12); free(r34); free(b34s);
    return total;
}
