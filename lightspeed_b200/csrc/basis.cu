// Basis handling: validation of the primitive arrays (the dense-index rules of
// the Lightspeed Basis constructor, src/lightspeed/basis.hpp:433-470), the
// real-solid-harmonic coefficients that map Cartesian to pure shells, and the
// device kernels that apply them to whole matrices.
#include <algorithm>
#include <cmath>
#include <map>
#include <tuple>
#include "engine.cuh"

namespace lsjk {

namespace {

// Monomial polynomial in x, y, z: (lx, ly, lz) -> coefficient.
using Poly = std::map<std::tuple<int, int, int>, double>;

void axpy(Poly& y, double a, const Poly& x, int dx, int dy, int dz)
{
    for (const auto& kv : x) {
        auto k = std::make_tuple(std::get<0>(kv.first) + dx, std::get<1>(kv.first) + dy,
                                 std::get<2>(kv.first) + dz);
        y[k] += a * kv.second;
    }
}

void prune(Poly& p)
{
    for (auto it = p.begin(); it != p.end();) {
        if (std::fabs(it->second) <= 1.0e-15) it = p.erase(it); else ++it;
    }
}

} // namespace

// Real solid harmonics S_{L,m} as Cartesian polynomials, built with the
// recursions of Helgaker, Jorgensen & Olsen, "Molecular Electronic-Structure
// Theory", eqs. 6.4.70-6.4.73 (the same construction the reference uses,
// src/cpp/core/am.cpp:74-220):
//   S_{00} = 1
//   S_{l+1,l+1}  = sqrt(2^{d_l0} (2l+1)/(2l+2)) (x S_{ll} - (1-d_l0) y S_{l,-l})
//   S_{l+1,-l-1} = sqrt(2^{d_l0} (2l+1)/(2l+2)) (y S_{ll} + (1-d_l0) x S_{l,-l})
//   S_{l+1,m} = ((2l+1) z S_{lm} - sqrt((l+m)(l-m)) r^2 S_{l-1,m}) / sqrt((l+m+1)(l-m+1))
// Pure functions are ordered m = 0, +1, -1, +2, -2, ... and Cartesian
// components in CCA lexical order. Returns coef[pure][cart] (dense).
std::vector<std::vector<double>> solid_harmonics(int L)
{
    const int ncart = (L + 1) * (L + 2) / 2;
    std::vector<Poly> Sc(L + 1), Ss(L + 1);   // diagonal S_{l,+l}, S_{l,-l}
    Sc[0][std::make_tuple(0, 0, 0)] = 1.0;
    for (int l = 0; l < L; ++l) {
        double Nc = std::sqrt((l == 0 ? 2.0 : 1.0) * (2.0 * l + 1.0) / (2.0 * l + 2.0));
        double Ns = (l == 0 ? 0.0 : Nc);
        Poly c, s;
        axpy(c, Nc, Sc[l], 1, 0, 0);
        axpy(s, Nc, Sc[l], 0, 1, 0);
        axpy(c, -Ns, Ss[l], 0, 1, 0);
        axpy(s, Ns, Ss[l], 1, 0, 0);
        prune(c);
        prune(s);
        Sc[l + 1] = c;
        Ss[l + 1] = s;
    }
    std::vector<Poly> out(2 * L + 1);
    for (int m = 0; m <= L; ++m) {
        Poly cur_c = Sc[m], cur_s = Ss[m], prev_c, prev_s;
        for (int l = m; l < L; ++l) {
            double a = (2.0 * l + 1.0) / std::sqrt((l + m + 1.0) * (l - m + 1.0));
            double b = std::sqrt(((l + m) * double(l - m)) / ((l + m + 1.0) * (l - m + 1.0)));
            Poly nc, ns;
            axpy(nc, a, cur_c, 0, 0, 1);
            axpy(ns, a, cur_s, 0, 0, 1);
            for (int d = 0; d < 3; ++d) {
                axpy(nc, -b, prev_c, d == 0 ? 2 : 0, d == 1 ? 2 : 0, d == 2 ? 2 : 0);
                axpy(ns, -b, prev_s, d == 0 ? 2 : 0, d == 1 ? 2 : 0, d == 2 ? 2 : 0);
            }
            prune(nc);
            prune(ns);
            prev_c = cur_c;
            prev_s = cur_s;
            cur_c = nc;
            cur_s = ns;
        }
        if (m == 0) {
            out[0] = cur_c;
        } else {
            out[2 * m - 1] = cur_c;
            out[2 * m] = cur_s;
        }
    }
    std::vector<std::vector<double>> coef(2 * L + 1, std::vector<double>(ncart, 0.0));
    for (int p = 0; p < 2 * L + 1; ++p) {
        for (const auto& kv : out[p]) {
            int lx, ly, lz;
            std::tie(lx, ly, lz) = kv.first;
            // CCA index of (lx, ly, lz): i = L - lx, j = lz
            int i = L - lx, j = lz;
            int idx = i * (i + 1) / 2 + j;
            coef[p][idx] += kv.second;
        }
    }
    return coef;
}

namespace {

void upload_prims(Context* ctx, Basis* B)
{
    cudaStream_t s = ctx->stream;
    B->dc.upload(B->c, s);
    B->de.upload(B->e, s);
    B->dx.upload(B->x, s);
    B->dy.upload(B->y, s);
    B->dz.upload(B->z, s);
    B->dL.upload(B->L, s);
    B->dcart.upload(B->cart, s);
    B->dao.upload(B->ao, s);
    B->dt0.upload(B->t0, s);
    B->dt1.upload(B->t1, s);
    B->dseg.upload(B->seg, s);
    B->dw0.upload(B->w0, s);
    B->dw1.upload(B->w1, s);
    B->datom.upload(B->atom, s);
}

void upload_maps(Context* ctx, Basis* B, const std::vector<std::vector<std::pair<int, double>>>& c2p,
                 const std::vector<std::vector<std::pair<int, double>>>& p2c)
{
    cudaStream_t s = ctx->stream;
    auto flatten = [&](const std::vector<std::vector<std::pair<int, double>>>& m, DBuf<int>& off,
                       DBuf<int>& idx, DBuf<double>& w) {
        std::vector<int> o(1, 0), ii;
        std::vector<double> ww;
        for (const auto& row : m) {
            for (const auto& e : row) { ii.push_back(e.first); ww.push_back(e.second); }
            o.push_back((int) ii.size());
        }
        off.upload(o, s);
        idx.upload(ii, s);
        w.upload(ww, s);
    };
    flatten(c2p, B->c2p_off, B->c2p_idx, B->c2p_w);
    flatten(p2c, B->p2c_off, B->p2c_idx, B->p2c_w);
    LSJK_CUDA(cudaStreamSynchronize(s));
}

} // namespace

bool Basis::equivalent(const Basis& o) const
{
    if (this == &o) return true;
    if (nprim != o.nprim || nao != o.nao || ncart != o.ncart || nshell != o.nshell || natom != o.natom)
        return false;
    return c == o.c && e == o.e && x == o.x && y == o.y && z == o.z && L == o.L && pure == o.pure &&
           ao == o.ao && cart == o.cart && prim == o.prim && shell == o.shell && atom == o.atom;
}

// Validate and upload; builds the pure <-> cart maps per shell.
void basis_init(Context* ctx, Basis* B)
{
    const int n = B->nprim;
    for (int P = 0; P < n; ++P) {
        if (B->prim[P] != P) throw Error(LSJK_EINVAL, "Basis: primIdx field is not dense");
        if (B->L[P] < 0) throw Error(LSJK_EINVAL, "Basis: negative angular momentum");
        int nao_p = B->pure[P] ? 2 * B->L[P] + 1 : ncart_count(B->L[P]);
        (void)nao_p;
        if (P == 0) {
            if (B->ao[0] || B->cart[0] || B->shell[0] || B->atom[0])
                throw Error(LSJK_EINVAL, "Basis: index fields are not dense");
        } else {
            int q = P - 1;
            int nao_q = B->pure[q] ? 2 * B->L[q] + 1 : ncart_count(B->L[q]);
            if (B->shell[q] == B->shell[P]) {
                if (B->ao[q] != B->ao[P] || B->cart[q] != B->cart[P] || B->atom[q] != B->atom[P])
                    throw Error(LSJK_EINVAL, "Basis: index fields are not dense");
                if (B->L[q] != B->L[P] || B->pure[q] != B->pure[P])
                    throw Error(LSJK_EINVAL, "Basis: shell with mixed L or purity");
            } else if (B->shell[q] + 1 == B->shell[P]) {
                if (B->ao[q] + nao_q != B->ao[P] || B->cart[q] + ncart_count(B->L[q]) != B->cart[P])
                    throw Error(LSJK_EINVAL, "Basis: aoIdx/cartIdx field is not dense");
                if (B->atom[q] != B->atom[P] && B->atom[q] + 1 != B->atom[P])
                    throw Error(LSJK_EINVAL, "Basis: atomIdx field is not dense");
            } else {
                throw Error(LSJK_EINVAL, "Basis: shellIdx field is not dense");
            }
        }
    }
    B->nao = B->ncart = B->nshell = B->natom = B->maxL = 0;
    B->has_pure = false;
    if (n) {
        int q = n - 1;
        B->nao = B->ao[q] + (B->pure[q] ? 2 * B->L[q] + 1 : ncart_count(B->L[q]));
        B->ncart = B->cart[q] + ncart_count(B->L[q]);
        B->nshell = B->shell[q] + 1;
        B->natom = B->atom[q] + 1;
        for (int P = 0; P < n; ++P) {
            B->maxL = std::max(B->maxL, B->L[P]);
            B->has_pure = B->has_pure || B->pure[P];
        }
    }
    // as given, a primitive's contributions go to its own shell, weight 1
    B->t0 = B->cart;
    B->t1.assign(n, -1);
    B->seg = B->shell;
    B->w0.assign(n, 1.0);
    B->w1.assign(n, 0.0);
    upload_prims(ctx, B);
    {
        std::vector<int> t0(B->ncart), t1(B->ncart, -1);
        for (int k = 0; k < B->ncart; ++k) t0[k] = k;
        B->uc_t0.upload(t0, ctx->stream);
        B->uc_t1.upload(t1, ctx->stream);
        B->uc_w0.upload(std::vector<double>(B->ncart, 1.0), ctx->stream);
        B->uc_w1.upload(std::vector<double>(B->ncart, 0.0), ctx->stream);
    }

    // pure <-> cart maps, one shell at a time (first primitive of each shell)
    std::vector<std::vector<std::pair<int, double>>> c2p(B->ncart), p2c(B->nao);
    std::map<int, std::vector<std::vector<double>>> sh;
    for (int P = 0; P < n; ++P) {
        if (P > 0 && B->shell[P] == B->shell[P - 1]) continue;
        int Lp = B->L[P], ao = B->ao[P], ca = B->cart[P];
        int nc = ncart_count(Lp);
        if (!B->pure[P]) {
            for (int k = 0; k < nc; ++k) {
                c2p[ca + k].push_back({ao + k, 1.0});
                p2c[ao + k].push_back({ca + k, 1.0});
            }
        } else {
            if (!sh.count(Lp)) sh[Lp] = solid_harmonics(Lp);
            const auto& C = sh[Lp];
            for (int p = 0; p < 2 * Lp + 1; ++p) {
                for (int k = 0; k < nc; ++k) {
                    if (C[p][k] == 0.0) continue;
                    c2p[ca + k].push_back({ao + p, C[p][k]});
                    p2c[ao + p].push_back({ca + k, C[p][k]});
                }
            }
        }
    }
    upload_maps(ctx, B, c2p, p2c);
}

// One primitive of a merged twin: the copies (original primitive indices) it
// stands for, at most two, all s type on one atom with one exponent.
namespace {
struct TwinPrim {
    int first;                 // original primitive the twin primitive takes its data from
    std::vector<int> copies;   // original primitives merged into it (1 or 2)
};
}

void basis_build_twin(Context* ctx, Basis* B)
{
    B->twin.reset();
    const int n = B->nprim;
    // copies of an s exponent on one atom, in primitive order
    std::map<std::pair<int, double>, std::vector<int>> groups;
    for (int P = 0; P < n; ++P)
        if (B->L[P] == 0) groups[{B->atom[P], B->e[P]}].push_back(P);
    // a twin primitive per chunk of two copies (a third copy starts another)
    std::vector<int> owner(n, -1);   // original primitive -> twin primitive
    std::vector<TwinPrim> tp;
    bool any = false;
    for (int P = 0; P < n; ++P) {
        if (owner[P] >= 0) continue;
        std::vector<int> copies{P};
        if (B->L[P] == 0) {
            const auto& g = groups[{B->atom[P], B->e[P]}];
            for (int Q : g)
                if (Q > P && owner[Q] < 0 && copies.size() < 2 && B->shell[Q] != B->shell[P]) copies.push_back(Q);
        }
        any = any || copies.size() > 1;
        for (int Q : copies) owner[Q] = (int) tp.size();
        tp.push_back(TwinPrim{P, copies});
    }
    if (!any) return;

    auto T = std::make_unique<Basis>();
    T->ctx = ctx;
    T->is_twin = true;
    // Cartesian slots: unmerged primitives keep sharing their shell's block
    // (a contracted shell stays one block); a merged primitive gets its own
    std::map<int, int> shell_slot;
    int ncart = 0;
    std::map<std::pair<int, int>, int> seg_of;   // (t0, t1) -> target group id
    for (const TwinPrim& u : tp) {
        const int P = u.first;
        int slot;
        if (u.copies.size() == 1) {
            auto it = shell_slot.find(B->shell[P]);
            if (it == shell_slot.end()) {
                slot = ncart;
                ncart += ncart_count(B->L[P]);
                shell_slot[B->shell[P]] = slot;
            } else {
                slot = it->second;
            }
        } else {
            slot = ncart;
            ncart += 1;
        }
        double cu;
        int t0 = B->cart[u.copies[0]], t1 = -1;
        double w0 = 1.0, w1 = 0.0;
        if (u.copies.size() == 1) {
            cu = B->c[P];   // as given: weight exactly 1
        } else {
            const int Q = u.copies[1];
            // the larger |c| of the copies: the pair bounds of the twin then bound
            // every copy's pair, so the twin's screens keep what the copies' keep
            cu = std::max(std::fabs(B->c[P]), std::fabs(B->c[Q]));
            w0 = B->c[P] / cu;
            w1 = B->c[Q] / cu;
            t1 = B->cart[Q];
        }
        auto sk = seg_of.emplace(std::make_pair(t0, t1), (int) seg_of.size()).first->second;
        T->c.push_back(cu);
        T->e.push_back(B->e[P]);
        T->x.push_back(B->x[P]);
        T->y.push_back(B->y[P]);
        T->z.push_back(B->z[P]);
        T->L.push_back(B->L[P]);
        T->pure.push_back(0);
        T->cart.push_back(slot);
        T->ao.push_back(slot);
        T->prim.push_back((int) T->prim.size());
        T->shell.push_back(sk);
        T->atom.push_back(B->atom[P]);
        T->t0.push_back(t0);
        T->t1.push_back(t1);
        T->seg.push_back(sk);
        T->w0.push_back(w0);
        T->w1.push_back(w1);
    }
    T->nprim = (int) tp.size();
    T->nao = B->nao;   // the maps lead into B's AO space
    T->ncart = ncart;
    T->nshell = (int) seg_of.size();
    T->natom = B->natom;
    T->maxL = B->maxL;
    T->has_pure = B->has_pure;
    upload_prims(ctx, T.get());

    // maps between the twin's Cartesian slots and B's AO functions: a slot
    // stands for sum_copies w_copy * (the copy's shell), so
    //   D_twin = M D_cart M^T and X_pure = C (M^T X_twin M) C^T
    // with M the weights and C the solid harmonics of B's shells
    std::vector<std::vector<std::pair<int, double>>> c2p(ncart), p2c(B->nao);
    std::map<int, std::vector<std::vector<double>>> sh;
    std::vector<char> done_shell_slot(ncart, 0);
    for (size_t k = 0; k < tp.size(); ++k) {
        const TwinPrim& u = tp[k];
        const int slot = T->cart[k];
        const double ws[2] = {T->w0[k], T->w1[k]};
        if (u.copies.size() == 1) {
            if (done_shell_slot[slot]) continue;   // one map entry per shared shell block
            done_shell_slot[slot] = 1;
        }
        for (size_t g = 0; g < u.copies.size(); ++g) {
            const int P = u.copies[g];
            const int Lp = B->L[P], ao = B->ao[P], nc = ncart_count(Lp);
            const double w = ws[g];
            if (!B->pure[P]) {
                for (int q = 0; q < nc; ++q) {
                    c2p[slot + q].push_back({ao + q, w});
                    p2c[ao + q].push_back({slot + q, w});
                }
            } else {
                if (!sh.count(Lp)) sh[Lp] = solid_harmonics(Lp);
                const auto& C = sh[Lp];
                for (int m = 0; m < 2 * Lp + 1; ++m)
                    for (int q = 0; q < nc; ++q) {
                        if (C[m][q] == 0.0) continue;
                        c2p[slot + q].push_back({ao + m, w * C[m][q]});
                        p2c[ao + m].push_back({slot + q, w * C[m][q]});
                    }
            }
        }
    }
    upload_maps(ctx, T.get(), c2p, p2c);
    // the original Cartesian functions behind each slot, for screening densities
    std::vector<int> ut0(ncart), ut1(ncart, -1);
    std::vector<double> uw0(ncart, 1.0), uw1(ncart, 0.0);
    for (int k = 0; k < T->nprim; ++k) {
        const int nc = ncart_count(T->L[k]);
        for (int q = 0; q < nc; ++q) {
            ut0[T->cart[k] + q] = T->t0[k] + q;
            ut1[T->cart[k] + q] = T->t1[k] >= 0 ? T->t1[k] + q : -1;
            uw0[T->cart[k] + q] = T->w0[k];
            uw1[T->cart[k] + q] = T->w1[k];
        }
    }
    T->uc_t0.upload(ut0, ctx->stream);
    T->uc_t1.upload(ut1, ctx->stream);
    T->uc_w0.upload(uw0, ctx->stream);
    T->uc_w1.upload(uw1, ctx->stream);
    LSJK_CUDA(cudaStreamSynchronize(ctx->stream));
    B->twin = std::move(T);
}

namespace {

// Dcart[c1,c2] = sum_{p1,p2} C1[p1,c1] C2[p2,c2] Dpure[p1,p2]   (pureToCart2)
__global__ void k_pure_to_cart(int nc1, int nc2, int np2, const int* __restrict__ o1,
                               const int* __restrict__ i1, const double* __restrict__ w1,
                               const int* __restrict__ o2, const int* __restrict__ i2,
                               const double* __restrict__ w2, const double* __restrict__ Dp,
                               double* __restrict__ Dc)
{
    long idx = blockIdx.x * (long) blockDim.x + threadIdx.x;
    if (idx >= (long) nc1 * nc2) return;
    int c1 = (int) (idx / nc2), c2 = (int) (idx % nc2);
    double acc = 0.0;
    for (int a = o1[c1]; a < o1[c1 + 1]; ++a) {
        double s = 0.0;
        const double* row = Dp + (long) i1[a] * np2;
        for (int b = o2[c2]; b < o2[c2 + 1]; ++b) s = fma(w2[b], row[i2[b]], s);
        acc = fma(w1[a], s, acc);
    }
    Dc[idx] = acc;
}

// Xpure[p1,p2] += sum_{c1,c2} C1[p1,c1] C2[p2,c2] Xcart[c1,c2]   (cartToPure2)
__global__ void k_cart_to_pure_acc(int np1, int np2, int nc2, const int* __restrict__ o1,
                                   const int* __restrict__ i1, const double* __restrict__ w1,
                                   const int* __restrict__ o2, const int* __restrict__ i2,
                                   const double* __restrict__ w2, const double* __restrict__ Xc,
                                   double* __restrict__ Xp)
{
    long idx = blockIdx.x * (long) blockDim.x + threadIdx.x;
    if (idx >= (long) np1 * np2) return;
    int p1 = (int) (idx / np2), p2 = (int) (idx % np2);
    double acc = 0.0;
    for (int a = o1[p1]; a < o1[p1 + 1]; ++a) {
        double s = 0.0;
        const double* row = Xc + (long) i1[a] * nc2;
        for (int b = o2[p2]; b < o2[p2 + 1]; ++b) s = fma(w2[b], row[i2[b]], s);
        acc = fma(w1[a], s, acc);
    }
    Xp[idx] += acc;
}

__global__ void k_screen_density(int n1, int n2, int ld, const int* __restrict__ t0a, const int* __restrict__ t1a,
                                 const double* __restrict__ w0a, const double* __restrict__ w1a,
                                 const int* __restrict__ t0b, const int* __restrict__ t1b,
                                 const double* __restrict__ w0b, const double* __restrict__ w1b,
                                 const double* __restrict__ D, double* __restrict__ S)
{
    long idx = blockIdx.x * (long) blockDim.x + threadIdx.x;
    if (idx >= (long) n1 * n2) return;
    const int a = (int) (idx / n2), b = (int) (idx % n2);
    const int ia[2] = {t0a[a], t1a[a]}, ib[2] = {t0b[b], t1b[b]};
    const double wa[2] = {fabs(w0a[a]), fabs(w1a[a])}, wb[2] = {fabs(w0b[b]), fabs(w1b[b])};
    double v = 0.0;
#pragma unroll
    for (int x = 0; x < 2; ++x)
#pragma unroll
        for (int y = 0; y < 2; ++y)
            if (ia[x] >= 0 && ib[y] >= 0) v = fmax(v, wa[x] * wb[y] * fabs(D[(long) ia[x] * ld + ib[y]]));
    S[idx] = v;
}

} // namespace

void screen_density(Context* ctx, const Basis* u1, const Basis* u2, const double* Dorig, int ld, double* Dscr)
{
    long n = (long) u1->ncart * u2->ncart;
    if (n == 0) return;
    k_screen_density<<<(unsigned) ((n + 255) / 256), 256, 0, ctx->stream>>>(
        u1->ncart, u2->ncart, ld, u1->uc_t0.p, u1->uc_t1.p, u1->uc_w0.p, u1->uc_w1.p, u2->uc_t0.p, u2->uc_t1.p,
        u2->uc_w0.p, u2->uc_w1.p, Dorig, Dscr);
    LSJK_CUDA(cudaGetLastError());
    ctx->stats.kernel_launches++;
}

void pure_to_cart(Context* ctx, const Basis* b1, const Basis* b2, const double* Dpure, double* Dcart)
{
    long n = (long) b1->ncart * b2->ncart;
    if (n == 0) return;
    k_pure_to_cart<<<(unsigned) ((n + 255) / 256), 256, 0, ctx->stream>>>(
        b1->ncart, b2->ncart, b2->nao, b1->c2p_off.p, b1->c2p_idx.p, b1->c2p_w.p, b2->c2p_off.p,
        b2->c2p_idx.p, b2->c2p_w.p, Dpure, Dcart);
    LSJK_CUDA(cudaGetLastError());
    ctx->stats.kernel_launches++;
}

void cart_to_pure_acc(Context* ctx, const Basis* b1, const Basis* b2, const double* Xcart, double* Xpure)
{
    long n = (long) b1->nao * b2->nao;
    if (n == 0) return;
    k_cart_to_pure_acc<<<(unsigned) ((n + 255) / 256), 256, 0, ctx->stream>>>(
        b1->nao, b2->nao, b2->ncart, b1->p2c_off.p, b1->p2c_idx.p, b1->p2c_w.p, b2->p2c_off.p,
        b2->p2c_idx.p, b2->p2c_w.p, Xcart, Xpure);
    LSJK_CUDA(cudaGetLastError());
    ctx->stats.kernel_launches++;
}

} // namespace lsjk
