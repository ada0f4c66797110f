// Test infrastructure only: a flat C interface over the reference Lightspeed
// CPU IntBox, compiled from the reference sources by oracle/Makefile into
// oracle/_ref/libls_ref.so. Nothing in the product links or loads this file;
// tests, smoke() and the CPU-baseline leg of bench.py call it through ctypes.
//
// Reference entry points wrapped here (paths inside the reference project):
//   IntBox::coulombCPU   src/cpp/intbox/cpu/coulomb.cpp:14-196
//   IntBox::exchangeCPU  src/cpp/intbox/cpu/exchange.cpp:17-355
//   IntBox::coulombGrad / exchangeGrad dispatch  src/cpp/intbox/intbox.cpp:423-630, restated
//     over the CPU routines it selects (coulombGradSymmCPU / coulombGradAdvCPU,
//     exchangeGradSymmCPU / exchangeGradAdvCPU in src/cpp/intbox/cpu/*_grad.cpp)
//   PairList::build_schwarz src/cpp/core/pair_list.cpp:29-177
//   IntBox::overlapCPU / kineticCPU / potentialCPU  src/cpp/intbox/cpu/*.cpp
//   Rys::compute_t / compute_w  src/cpp/quad/rys.cpp:28-80
#include <lightspeed/basis.hpp>
#include <lightspeed/pair_list.hpp>
#include <lightspeed/intbox.hpp>
#include <lightspeed/tensor.hpp>
#include <lightspeed/resource_list.hpp>
#include <lightspeed/ewald.hpp>
#include <lightspeed/rys.hpp>
#include <cstring>
#include <memory>
#include <string>
#include <vector>
#include <exception>
#include "ref_handles.hpp"

using namespace lightspeed;
using oracle_ref::RefBasis;
using oracle_ref::RefPairs;

namespace {
thread_local std::string g_err;

std::shared_ptr<ResourceList> resources(int nthread)
{
    auto r = ResourceList::build_cpu();
    if (nthread > 0) {
        std::vector<std::shared_ptr<GPUContext>> none;
        r = std::make_shared<ResourceList>(nthread, none);
    }
    return r;
}

std::shared_ptr<Tensor> wrap(const double* p, size_t n1, size_t n2)
{
    auto t = std::make_shared<Tensor>(std::vector<size_t>{n1, n2});
    if (p) std::memcpy(t->data().data(), p, sizeof(double) * n1 * n2);
    return t;
}
} // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

void* ref_basis_new(int nprim, const double* c, const double* e, const double* xyz,
                    const double* c0, const int* L, const int* pure, const int* aoIdx,
                    const int* cartIdx, const int* primIdx, const int* shellIdx,
                    const int* atomIdx)
{
    try {
        std::vector<Primitive> prims;
        for (int i = 0; i < nprim; i++) {
            prims.push_back(Primitive(c[i], e[i], xyz[3*i], xyz[3*i+1], xyz[3*i+2], c0[i],
                L[i], pure[i] != 0, aoIdx[i], cartIdx[i], primIdx[i], shellIdx[i], atomIdx[i]));
        }
        return new RefBasis{std::make_shared<Basis>("ref", prims)};
    } catch (std::exception& ex) { g_err = ex.what(); return nullptr; }
}

void ref_basis_free(void* b) { delete static_cast<RefBasis*>(b); }

int ref_basis_nao(void* b) { return (int) static_cast<RefBasis*>(b)->b->nao(); }
int ref_basis_ncart(void* b) { return (int) static_cast<RefBasis*>(b)->b->ncart(); }

void* ref_pairlist_new(void* b1, void* b2, int symm, float thre)
{
    try {
        auto p = PairList::build_schwarz(static_cast<RefBasis*>(b1)->b,
                                         static_cast<RefBasis*>(b2)->b, symm != 0, thre);
        return new RefPairs{p};
    } catch (std::exception& ex) { g_err = ex.what(); return nullptr; }
}

void ref_pairlist_free(void* p) { delete static_cast<RefPairs*>(p); }

long ref_pairlist_count(void* p)
{
    long n = 0;
    for (const auto& pl : static_cast<RefPairs*>(p)->p->pairlists()) n += (long) pl.pairs().size();
    return n;
}

// Flattened in the reference's own class order, pairs in their sorted order.
void ref_pairlist_export(void* p, int* L1, int* L2, int* prim1, int* prim2, float* bound)
{
    long k = 0;
    for (const auto& pl : static_cast<RefPairs*>(p)->p->pairlists()) {
        for (const auto& pr : pl.pairs()) {
            L1[k] = pl.L1(); L2[k] = pl.L2();
            prim1[k] = pr.prim1().primIdx(); prim2[k] = pr.prim2().primIdx();
            bound[k] = pr.bound();
            k++;
        }
    }
}

// J12 (n1 x n2, pure/nao basis) is accumulated in place.
int ref_coulomb(void* pl12, void* pl34, int nterm, const double* scales, const double* omegas,
                const double* D34, float thresp, float thredp, double* J12, int nthread)
{
    try {
        auto p12 = static_cast<RefPairs*>(pl12)->p;
        auto p34 = static_cast<RefPairs*>(pl34)->p;
        auto ew = std::make_shared<Ewald>(std::vector<double>(scales, scales + nterm),
                                          std::vector<double>(omegas, omegas + nterm));
        size_t n1 = p12->basis1()->nao(), n2 = p12->basis2()->nao();
        size_t n3 = p34->basis1()->nao(), n4 = p34->basis2()->nao();
        auto D = wrap(D34, n3, n4);
        auto J = wrap(J12, n1, n2);
        auto R = IntBox::coulombCPU(resources(nthread), ew, p12, p34, D, thresp, thredp, J);
        std::memcpy(J12, R->data().data(), sizeof(double) * n1 * n2);
        return 0;
    } catch (std::exception& ex) { g_err = ex.what(); return 1; }
}

// K13 (n1 x n3) is accumulated in place.
int ref_exchange(void* pl12, void* pl34, int nterm, const double* scales, const double* omegas,
                 const double* D24, int D24symm, float thresp, float thredp, double* K13,
                 int nthread)
{
    try {
        auto p12 = static_cast<RefPairs*>(pl12)->p;
        auto p34 = static_cast<RefPairs*>(pl34)->p;
        auto ew = std::make_shared<Ewald>(std::vector<double>(scales, scales + nterm),
                                          std::vector<double>(omegas, omegas + nterm));
        size_t n1 = p12->basis1()->nao(), n2 = p12->basis2()->nao();
        size_t n3 = p34->basis1()->nao(), n4 = p34->basis2()->nao();
        auto D = wrap(D24, n2, n4);
        auto K = wrap(K13, n1, n3);
        auto R = IntBox::exchangeCPU(resources(nthread), ew, p12, p34, D, D24symm != 0,
                                     thresp, thredp, K);
        std::memcpy(K13, R->data().data(), sizeof(double) * n1 * n3);
        return 0;
    } catch (std::exception& ex) { g_err = ex.what(); return 1; }
}

// G (natom x 3) += the J gradient sum D12 d(12|34) D34 (IntBox::coulombGrad;
// `same` stands for the reference's test D12 == D34, an object identity).
int ref_coulomb_grad(void* pl, int nterm, const double* scales, const double* omegas, const double* D12,
                     const double* D34, int same, float thresp, float thredp, double* G, int nthread)
{
    try {
        auto p = static_cast<RefPairs*>(pl)->p;
        auto ew = std::make_shared<Ewald>(std::vector<double>(scales, scales + nterm),
                                          std::vector<double>(omegas, omegas + nterm));
        size_t n = p->basis1()->nao(), natom = p->basis1()->natom();
        auto A = wrap(D12, n, n);
        auto B = same ? A : wrap(D34, n, n);
        auto Gt = wrap(G, natom, 3);
        if (same) {
            Gt = IntBox::coulombGradSymmCPU(resources(nthread), ew, p, A, thresp, thredp, Gt);
        } else {
            auto parts = IntBox::coulombGradAdvCPU(resources(nthread), ew, p, p, A, B, thresp, thredp,
                                                   std::vector<std::shared_ptr<Tensor>>());
            for (auto& t : parts)
                for (size_t i = 0; i < Gt->size(); ++i) Gt->data()[i] += t->data()[i];
        }
        std::memcpy(G, Gt->data().data(), sizeof(double) * natom * 3);
        return 0;
    } catch (std::exception& ex) { g_err = ex.what(); return 1; }
}

// G (natom x 3) += the K gradient sum D13 d(12|34) D24 (IntBox::exchangeGrad).
int ref_exchange_grad(void* pl, int nterm, const double* scales, const double* omegas, const double* D13,
                      const double* D24, int D13symm, int D24symm, int Dsame, float thresp, float thredp,
                      double* G, int nthread)
{
    try {
        auto p = static_cast<RefPairs*>(pl)->p;
        auto ew = std::make_shared<Ewald>(std::vector<double>(scales, scales + nterm),
                                          std::vector<double>(omegas, omegas + nterm));
        size_t n = p->basis1()->nao(), natom = p->basis1()->natom();
        auto A = wrap(D13, n, n);
        auto B = Dsame ? A : wrap(D24, n, n);
        auto Gt = wrap(G, natom, 3);
        if (D13symm && D24symm && Dsame) {
            Gt = IntBox::exchangeGradSymmCPU(resources(nthread), ew, p, A, thresp, thredp, Gt);
        } else {
            auto parts = IntBox::exchangeGradAdvCPU(resources(nthread), ew, p, p, A, B, D13symm != 0,
                                                    D24symm != 0, Dsame != 0, thresp, thredp,
                                                    std::vector<std::shared_ptr<Tensor>>());
            for (auto& t : parts)
                for (size_t i = 0; i < Gt->size(); ++i) Gt->data()[i] += t->data()[i];
        }
        std::memcpy(G, Gt->data().data(), sizeof(double) * natom * 3);
        return 0;
    } catch (std::exception& ex) { g_err = ex.what(); return 1; }
}

int ref_overlap(void* pl, double* S, int nthread)
{
    try {
        auto p = static_cast<RefPairs*>(pl)->p;
        auto T = IntBox::overlapCPU(resources(nthread), p);
        std::memcpy(S, T->data().data(), sizeof(double) * T->size());
        return 0;
    } catch (std::exception& ex) { g_err = ex.what(); return 1; }
}

int ref_kinetic(void* pl, double* Tk, int nthread)
{
    try {
        auto p = static_cast<RefPairs*>(pl)->p;
        auto T = IntBox::kineticCPU(resources(nthread), p);
        std::memcpy(Tk, T->data().data(), sizeof(double) * T->size());
        return 0;
    } catch (std::exception& ex) { g_err = ex.what(); return 1; }
}

// xyzc: natom x 4 (x, y, z, Z); V accumulates -Z/r style nuclear potential.
int ref_potential(void* pl, int nterm, const double* scales, const double* omegas,
                  int natom, const double* xyzc, double* V, int nthread)
{
    try {
        auto p = static_cast<RefPairs*>(pl)->p;
        auto ew = std::make_shared<Ewald>(std::vector<double>(scales, scales + nterm),
                                          std::vector<double>(omegas, omegas + nterm));
        auto X = wrap(xyzc, natom, 4);
        auto T = IntBox::potentialCPU(resources(nthread), ew, p, X);
        std::memcpy(V, T->data().data(), sizeof(double) * T->size());
        return 0;
    } catch (std::exception& ex) { g_err = ex.what(); return 1; }
}

// Rys roots and weights of the reference tables: t and w are npoint x nrys.
int ref_rys(int nrys, int npoint, const double* T, double* t, double* w)
{
    try {
        auto Tt = std::make_shared<Tensor>(std::vector<size_t>{(size_t) npoint});
        std::memcpy(Tt->data().data(), T, sizeof(double) * npoint);
        auto tt = Rys::compute_t(nrys, Tt);
        auto ww = Rys::compute_w(nrys, Tt);
        std::memcpy(t, tt->data().data(), sizeof(double) * npoint * nrys);
        std::memcpy(w, ww->data().data(), sizeof(double) * npoint * nrys);
        return 0;
    } catch (std::exception& ex) { g_err = ex.what(); return 1; }
}

} // extern "C"
