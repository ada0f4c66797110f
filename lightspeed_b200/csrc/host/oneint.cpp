// One-electron integrals S, T, V for the SCF drivers around the J/K path.
// These are not on the J/K hot path (they are computed once per geometry);
// the reference computes them on the CPU too (src/cpp/intbox/cpu/overlap.cpp,
// kinetic.cpp, potential.cpp). Here they are McMurchie-Davidson integrals over
// the same primitive pair lists, Cartesian first, then the pure transform of
// the basis.
#include <cmath>
#include <cstring>
#include <vector>
#include "lightspeed.hpp"
#include "oneint.hpp"

extern "C" int lsjk_solid_harmonics(int L, double* coef);

namespace lightspeed {

namespace {

// Hermite expansion coefficients E^{ij}_t of one Cartesian direction.
void hermite_E(int la, int lb, double p, double PA, double PB, std::vector<double>& E, int V)
{
    // E[(i*(lb+1)+j)*V + t]
    E.assign((size_t) (la + 1) * (lb + 1) * V, 0.0);
    auto at = [&](int i, int j, int t) -> double& { return E[((size_t) i * (lb + 1) + j) * V + t]; };
    at(0, 0, 0) = 1.0;
    double h = 0.5 / p;
    for (int i = 0; i < la; ++i)
        for (int t = 0; t <= i + 1; ++t) {
            double s = PA * at(i, 0, t);
            if (t > 0) s += h * at(i, 0, t - 1);
            if (t + 1 <= i) s += (t + 1) * at(i, 0, t + 1);
            at(i + 1, 0, t) = s;
        }
    for (int j = 0; j < lb; ++j)
        for (int i = 0; i <= la; ++i)
            for (int t = 0; t <= i + j + 1; ++t) {
                double s = PB * at(i, j, t);
                if (t > 0) s += h * at(i, j, t - 1);
                if (t + 1 <= i + j) s += (t + 1) * at(i, j, t + 1);
                at(i, j + 1, t) = s;
            }
}

void cart_exps(int L, std::vector<int>& lx, std::vector<int>& ly, std::vector<int>& lz)
{
    lx.clear(); ly.clear(); lz.clear();
    for (int i = 0; i <= L; ++i)
        for (int j = 0; j <= i; ++j) {
            lx.push_back(L - i);
            ly.push_back(i - j);
            lz.push_back(j);
        }
}

// Boys functions F_0..F_m(T): power series below T = 30 (summed until the
// terms vanish), downward recursion; asymptotic form with the exact upward
// recursion above.
void boys(int m, double T, double* F)
{
    if (T < 30.0) {
        double e = std::exp(-T);
        double term = 1.0 / (2 * m + 1), sum = term;
        for (int k = 1; k < 400; ++k) {
            term *= 2.0 * T / (2 * m + 2 * k + 1);
            sum += term;
            if (term < 1e-18 * sum) break;
        }
        F[m] = e * sum;
        for (int n = m - 1; n >= 0; --n) F[n] = (2.0 * T * F[n + 1] + e) / (2 * n + 1);
    } else {
        double e = std::exp(-T);
        F[0] = 0.5 * std::sqrt(M_PI / T);
        for (int n = 0; n < m; ++n) F[n + 1] = ((2 * n + 1) * F[n] - e) / (2.0 * T);
    }
}

// Hermite Coulomb integrals R_{tuv} (n = 0) for |tuv| <= L, indexed [t][u][v].
void hermite_R(int L, double alpha, double X, double Y, double Z, const double* Fs, std::vector<double>& R)
{
    int V = L + 1;
    std::vector<double> Rn((size_t) (L + 1) * V * V * V, 0.0);
    auto at = [&](int n, int t, int u, int v) -> double& { return Rn[(((size_t) n * V + t) * V + u) * V + v]; };
    double m2a = -2.0 * alpha, pw = 1.0;
    for (int n = 0; n <= L; ++n) {
        at(n, 0, 0, 0) = pw * Fs[n];
        pw *= m2a;
    }
    for (int n = L - 1; n >= 0; --n) {
        int top = L - n;
        for (int t = 0; t <= top; ++t)
            for (int u = 0; u + t <= top; ++u)
                for (int v = 0; v + u + t <= top; ++v) {
                    if (t + u + v == 0) continue;
                    double s;
                    if (t > 0) {
                        s = X * at(n + 1, t - 1, u, v);
                        if (t > 1) s += (t - 1) * at(n + 1, t - 2, u, v);
                    } else if (u > 0) {
                        s = Y * at(n + 1, t, u - 1, v);
                        if (u > 1) s += (u - 1) * at(n + 1, t, u - 2, v);
                    } else {
                        s = Z * at(n + 1, t, u, v - 1);
                        if (v > 1) s += (v - 1) * at(n + 1, t, u, v - 2);
                    }
                    at(n, t, u, v) = s;
                }
    }
    R.assign((size_t) V * V * V, 0.0);
    for (int t = 0; t <= L; ++t)
        for (int u = 0; u + t <= L; ++u)
            for (int v = 0; v + u + t <= L; ++v) R[((size_t) t * V + u) * V + v] = at(0, t, u, v);
}

enum Kind { kOverlap, kKinetic, kPotential };

// Cartesian integrals accumulated over the pair list (both triangles for a
// symmetric list, 1/2 on diagonal primitive pairs like the reference's pair
// list consumers).
std::vector<double> cart_ints(const std::shared_ptr<PairList>& pl, Kind kind, const Ewald* ewald,
                              const std::vector<double>& xyzc)
{
    auto b1 = pl->basis1(), b2 = pl->basis2();
    size_t n1 = b1->ncart(), n2 = b2->ncart();
    std::vector<double> out(n1 * n2, 0.0);
    std::vector<const Pair*> pairs;
    for (const auto& l : pl->pairlists())
        for (const auto& p : l.pairs()) pairs.push_back(&p);
    bool symm = pl->is_symmetric();
    size_t natom = xyzc.size() / 4;
#pragma omp parallel
    {
        std::vector<double> loc(n1 * n2, 0.0);
        std::vector<double> Ex, Ey, Ez, R;
        std::vector<int> lx1, ly1, lz1, lx2, ly2, lz2;
        double Fs[64];
#pragma omp for schedule(dynamic, 64)
        for (long k = 0; k < (long) pairs.size(); ++k) {
            const Primitive& a = pairs[k]->prim1();
            const Primitive& b = pairs[k]->prim2();
            int la = a.L(), lb = b.L();
            int extra = (kind == kKinetic) ? 2 : 0;
            int V = la + lb + extra + 1;
            double p = a.e() + b.e();
            double P[3] = {(a.e() * a.x() + b.e() * b.x()) / p, (a.e() * a.y() + b.e() * b.y()) / p,
                           (a.e() * a.z() + b.e() * b.z()) / p};
            double AB2 = (a.x() - b.x()) * (a.x() - b.x()) + (a.y() - b.y()) * (a.y() - b.y()) +
                         (a.z() - b.z()) * (a.z() - b.z());
            double Kab = a.c() * b.c() * std::exp(-a.e() * b.e() / p * AB2);
            hermite_E(la, lb + extra, p, P[0] - a.x(), P[0] - b.x(), Ex, V);
            hermite_E(la, lb + extra, p, P[1] - a.y(), P[1] - b.y(), Ey, V);
            hermite_E(la, lb + extra, p, P[2] - a.z(), P[2] - b.z(), Ez, V);
            int lbe = lb + extra;
            auto E = [&](const std::vector<double>& Ed, int i, int j, int t) {
                return Ed[((size_t) i * (lbe + 1) + j) * V + t];
            };
            cart_exps(la, lx1, ly1, lz1);
            cart_exps(lb, lx2, ly2, lz2);
            double scale = (symm && a.primIdx() == b.primIdx()) ? 0.5 : 1.0;
            double s1 = std::sqrt(M_PI / p);
            // 1-D overlap and kinetic factors
            auto S1 = [&](const std::vector<double>& Ed, int i, int j) { return j < 0 ? 0.0 : E(Ed, i, j, 0) * s1; };
            auto T1 = [&](const std::vector<double>& Ed, int i, int j) {
                double be = b.e();
                double v = -2.0 * be * be * S1(Ed, i, j + 2) + be * (2 * j + 1) * S1(Ed, i, j);
                if (j >= 2) v -= 0.5 * j * (j - 1) * S1(Ed, i, j - 2);
                return v;
            };
            std::vector<double> Rsum;
            if (kind == kPotential) {
                int L = la + lb, VV = L + 1;
                Rsum.assign((size_t) VV * VV * VV, 0.0);
                for (size_t C = 0; C < natom; ++C) {
                    double Z = xyzc[4 * C + 3];
                    if (Z == 0.0) continue;
                    double X = P[0] - xyzc[4 * C], Y = P[1] - xyzc[4 * C + 1], Zc = P[2] - xyzc[4 * C + 2];
                    double R2 = X * X + Y * Y + Zc * Zc;
                    for (size_t w = 0; w < ewald->scales().size(); ++w) {
                        double al = ewald->scales()[w], om = ewald->omegas()[w];
                        if (al == 0.0 || om == 0.0) continue;
                        double d2 = 1.0, f = 1.0;
                        if (om != -1.0) {
                            d2 = om * om / (p + om * om);
                            f = std::sqrt(d2);
                        }
                        boys(L, p * d2 * R2, Fs);
                        hermite_R(L, p * d2, X, Y, Zc, Fs, R);
                        double c = -Z * al * f * 2.0 * M_PI / p;
                        for (size_t q = 0; q < R.size(); ++q) Rsum[q] += c * R[q];
                    }
                }
            }
            int a0 = a.cartIdx(), b0 = b.cartIdx();
            for (size_t i = 0; i < lx1.size(); ++i)
                for (size_t j = 0; j < lx2.size(); ++j) {
                    double v = 0.0;
                    if (kind == kOverlap) {
                        v = S1(Ex, lx1[i], lx2[j]) * S1(Ey, ly1[i], ly2[j]) * S1(Ez, lz1[i], lz2[j]);
                    } else if (kind == kKinetic) {
                        double sx = S1(Ex, lx1[i], lx2[j]), sy = S1(Ey, ly1[i], ly2[j]), sz = S1(Ez, lz1[i], lz2[j]);
                        v = T1(Ex, lx1[i], lx2[j]) * sy * sz + sx * T1(Ey, ly1[i], ly2[j]) * sz +
                            sx * sy * T1(Ez, lz1[i], lz2[j]);
                    } else {
                        int L = la + lb, VV = L + 1;
                        for (int t = 0; t <= lx1[i] + lx2[j]; ++t)
                            for (int u = 0; u <= ly1[i] + ly2[j]; ++u)
                                for (int w = 0; w <= lz1[i] + lz2[j]; ++w)
                                    v += E(Ex, lx1[i], lx2[j], t) * E(Ey, ly1[i], ly2[j], u) *
                                         E(Ez, lz1[i], lz2[j], w) * Rsum[((size_t) t * VV + u) * VV + w];
                    }
                    v *= Kab * scale;
                    loc[(a0 + i) * n2 + b0 + j] += v;
                    if (symm) loc[(b0 + j) * n2 + a0 + i] += v;
                }
        }
#pragma omp critical
        for (size_t q = 0; q < out.size(); ++q) out[q] += loc[q];
    }
    return out;
}

// Pure transform: X = C1 Xc C2^T per shell pair, using the solid-harmonic
// coefficients of the engine.
std::shared_ptr<Tensor> to_pure(const std::shared_ptr<Basis>& b1, const std::shared_ptr<Basis>& b2,
                                const std::vector<double>& Xc, const std::shared_ptr<Tensor>& out, const char* name)
{
    size_t n1 = b1->nao(), n2 = b2->nao(), c2n = b2->ncart();
    auto T = out ? out : std::make_shared<Tensor>(std::vector<size_t>{n1, n2}, name);
    T->shape_error({n1, n2});
    auto rows = [](const std::shared_ptr<Basis>& b) {
        // per cart index: list of (ao index, coef)
        std::vector<std::vector<std::pair<int, double>>> m(b->ncart());
        std::vector<double> coef;
        const auto& P = b->primitives();
        for (size_t k = 0; k < P.size(); ++k) {
            if (k && P[k].shellIdx() == P[k - 1].shellIdx()) continue;
            int L = P[k].L(), nc = P[k].ncart();
            if (!P[k].is_pure()) {
                for (int c = 0; c < nc; ++c) m[P[k].cartIdx() + c].push_back({P[k].aoIdx() + c, 1.0});
            } else {
                coef.assign((size_t) (2 * L + 1) * nc, 0.0);
                check_rc(lsjk_solid_harmonics(L, coef.data()), "solid harmonics");
                for (int pp = 0; pp < 2 * L + 1; ++pp)
                    for (int c = 0; c < nc; ++c)
                        if (coef[pp * nc + c] != 0.0)
                            m[P[k].cartIdx() + c].push_back({P[k].aoIdx() + pp, coef[pp * nc + c]});
            }
        }
        return m;
    };
    auto m1 = rows(b1), m2 = rows(b2);
    std::vector<double> tmp(b1->ncart() * n2, 0.0);
    for (size_t c1 = 0; c1 < b1->ncart(); ++c1)
        for (size_t c2 = 0; c2 < c2n; ++c2)
            for (const auto& e : m2[c2]) tmp[c1 * n2 + e.first] += e.second * Xc[c1 * c2n + c2];
    double* d = T->data().data();
    for (size_t c1 = 0; c1 < b1->ncart(); ++c1)
        for (const auto& e : m1[c1])
            for (size_t q = 0; q < n2; ++q) d[e.first * n2 + q] += e.second * tmp[c1 * n2 + q];
    return T;
}

} // namespace

std::shared_ptr<Tensor> OneInt::overlap(const std::shared_ptr<PairList>& pl, const std::shared_ptr<Tensor>& S)
{
    return to_pure(pl->basis1(), pl->basis2(), cart_ints(pl, kOverlap, nullptr, {}), S, "S");
}

std::shared_ptr<Tensor> OneInt::kinetic(const std::shared_ptr<PairList>& pl, const std::shared_ptr<Tensor>& T)
{
    return to_pure(pl->basis1(), pl->basis2(), cart_ints(pl, kKinetic, nullptr, {}), T, "T");
}

std::shared_ptr<Tensor> OneInt::potential(const std::shared_ptr<Ewald>& ewald, const std::shared_ptr<PairList>& pl,
                                          const std::shared_ptr<Tensor>& xyzc, const std::shared_ptr<Tensor>& V)
{
    xyzc->ndim_error(2);
    if (xyzc->shape()[1] != 4) throw std::runtime_error("IntBox::potential: xyzc must be (natom, 4)");
    return to_pure(pl->basis1(), pl->basis2(), cart_ints(pl, kPotential, ewald.get(), xyzc->data()), V, "V");
}

} // namespace lightspeed
