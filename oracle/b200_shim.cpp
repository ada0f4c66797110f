// The reference-side binding of the B200 engine: what a Lightspeed maintainer
// adds to the reference so that IntBox::coulomb / IntBox::exchange
// (src/lightspeed/intbox.hpp:761-771, :817-828) and their nuclear gradients
// coulombGrad / exchangeGrad (:998-1008, :1147-1160) run on liblsjk.so, written
// against the reference's own headers and types (Tensor, Basis, PairList,
// Ewald, ResourceList) and compiled from them by oracle/Makefile (target
// shim) into oracle/_ref/libls_b200shim.so. In the reference it would replace
// the TeraChem branch of the dispatch (src/cpp/intbox/intbox.cpp:224-236,
// :302-315); here a flat C wrapper over the oracle's reference objects lets
// the tests call it with reference Basis/PairList/Tensor objects and check
// the reference's golden vectors. Test infrastructure: the product never
// links it.
#include <lightspeed/basis.hpp>
#include <lightspeed/ewald.hpp>
#include <lightspeed/pair_list.hpp>
#include <lightspeed/resource_list.hpp>
#include <lightspeed/tensor.hpp>
#include <lsjk.h>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#include "ref_handles.hpp"

namespace lightspeed {
namespace b200 {

namespace {

void check(int rc)
{
    if (rc) throw std::runtime_error(lsjk_last_error());
}

// one engine session per process, like the reference's TCIntBox::instance
lsjk_context* ctx()
{
    static lsjk_context* c = nullptr;
    if (!c) check(lsjk_context_create(0, &c));
    return c;
}

// device copies cached per reference object (as TCIntBox::set_basis caches
// by basis), dropped and rebuilt when the reference object has gone
template <typename T, typename H>
struct Cache {
    std::map<const T*, std::pair<std::weak_ptr<T>, H*>> m;
    H* find(const std::shared_ptr<T>& key)
    {
        auto it = m.find(key.get());
        if (it == m.end()) return nullptr;
        if (it->second.first.expired()) {
            m.erase(it);
            return nullptr;
        }
        return it->second.second;
    }
};

lsjk_basis* dev(const std::shared_ptr<Basis>& b)
{
    static Cache<Basis, lsjk_basis> cache;
    if (lsjk_basis* h = cache.find(b)) return h;
    const std::vector<Primitive>& P = b->primitives();
    const int n = (int) P.size();
    std::vector<double> c(n), e(n), xyz(3 * n);
    std::vector<int> L(n), pure(n), ao(n), cart(n), prim(n), shell(n), atom(n);
    for (int i = 0; i < n; ++i) {
        c[i] = P[i].c();
        e[i] = P[i].e();
        xyz[3 * i] = P[i].x();
        xyz[3 * i + 1] = P[i].y();
        xyz[3 * i + 2] = P[i].z();
        L[i] = P[i].L();
        pure[i] = P[i].is_pure() ? 1 : 0;
        ao[i] = P[i].aoIdx();
        cart[i] = P[i].cartIdx();
        prim[i] = P[i].primIdx();
        shell[i] = P[i].shellIdx();
        atom[i] = P[i].atomIdx();
    }
    lsjk_basis* h = nullptr;
    check(lsjk_basis_create(ctx(), n, c.data(), e.data(), xyz.data(), L.data(), pure.data(), ao.data(), cart.data(),
                            prim.data(), shell.data(), atom.data(), &h));
    cache.m[b.get()] = {b, h};
    return h;
}

// the engine rebuilds the same pair list on the device from the same bases
// and threshold (PairList::build_schwarz, src/cpp/core/pair_list.cpp:29-177)
lsjk_pairlist* dev(const std::shared_ptr<PairList>& pl)
{
    static Cache<PairList, lsjk_pairlist> cache;
    if (lsjk_pairlist* h = cache.find(pl)) return h;
    lsjk_pairlist* h = nullptr;
    check(lsjk_pairlist_build_schwarz(ctx(), dev(pl->basis1()), dev(pl->basis2()), pl->is_symmetric() ? 1 : 0,
                                      pl->thre(), &h));
    cache.m[pl.get()] = {pl, h};
    return h;
}

} // namespace

// IntBox::coulomb's signature and semantics: J12 (nao1 x nao2) accumulates
// J[D34]; a new zeroed tensor when none is passed.
std::shared_ptr<Tensor> coulomb(const std::shared_ptr<ResourceList>&, const std::shared_ptr<Ewald>& ewald,
                                const std::shared_ptr<PairList>& pl12, const std::shared_ptr<PairList>& pl34,
                                const std::shared_ptr<Tensor>& D34, float thresp, float thredp,
                                const std::shared_ptr<Tensor>& J12 = std::shared_ptr<Tensor>())
{
    const size_t n1 = pl12->basis1()->nao(), n2 = pl12->basis2()->nao();
    D34->shape_error({pl34->basis1()->nao(), pl34->basis2()->nao()});
    std::shared_ptr<Tensor> J = J12 ? J12 : std::make_shared<Tensor>(std::vector<size_t>{n1, n2});
    J->shape_error({n1, n2});
    const double* d = D34->data().data();
    double* j = J->data().data();
    check(lsjk_coulomb(ctx(), (int) ewald->scales().size(), ewald->scales().data(), ewald->omegas().data(),
                       dev(pl12), dev(pl34), 1, &d, thresp, thredp, &j));
    return J;
}

// IntBox::exchange's signature and semantics: K13 (nao1 x nao3) accumulates
// K[D24]; D24symm needs equivalent bases 2 and 4 (the engine checks and
// raises the reference's message).
std::shared_ptr<Tensor> exchange(const std::shared_ptr<ResourceList>&, const std::shared_ptr<Ewald>& ewald,
                                 const std::shared_ptr<PairList>& pl12, const std::shared_ptr<PairList>& pl34,
                                 const std::shared_ptr<Tensor>& D24, bool D24symm, float thresp, float thredp,
                                 const std::shared_ptr<Tensor>& K13 = std::shared_ptr<Tensor>())
{
    const size_t n1 = pl12->basis1()->nao(), n3 = pl34->basis1()->nao();
    D24->shape_error({pl12->basis2()->nao(), pl34->basis2()->nao()});
    std::shared_ptr<Tensor> K = K13 ? K13 : std::make_shared<Tensor>(std::vector<size_t>{n1, n3});
    K->shape_error({n1, n3});
    const double* d = D24->data().data();
    double* k = K->data().data();
    check(lsjk_exchange(ctx(), (int) ewald->scales().size(), ewald->scales().data(), ewald->omegas().data(),
                        dev(pl12), dev(pl34), 1, &d, D24symm ? 1 : 0, thresp, thredp, &k));
    return K;
}

// IntBox::coulombGrad's signature (src/lightspeed/intbox.hpp:998-1008): G
// (natom x 3) accumulates; D12 and D34 the same object is the reference's
// symmetric branch (one pointer passed on).
std::shared_ptr<Tensor> coulombGrad(const std::shared_ptr<ResourceList>&, const std::shared_ptr<Ewald>& ewald,
                                    const std::shared_ptr<PairList>& pl, const std::shared_ptr<Tensor>& D12,
                                    const std::shared_ptr<Tensor>& D34, float thresp, float thredp,
                                    const std::shared_ptr<Tensor>& G = std::shared_ptr<Tensor>())
{
    const size_t n = pl->basis1()->nao(), natom = pl->basis1()->natom();
    D12->shape_error({n, n});
    D34->shape_error({n, n});
    std::shared_ptr<Tensor> out = G ? G : std::make_shared<Tensor>(std::vector<size_t>{natom, 3});
    out->shape_error({natom, 3});
    const double* a = D12->data().data();
    const double* b = D12 == D34 ? a : D34->data().data();
    check(lsjk_coulomb_grad(ctx(), (int) ewald->scales().size(), ewald->scales().data(), ewald->omegas().data(),
                            dev(pl), a, b, thresp, thredp, out->data().data()));
    return out;
}

// IntBox::exchangeGrad's signature (src/lightspeed/intbox.hpp:1147-1160): the
// three flags pass through (all three select the reference's fully symmetric
// routine, which reads D13 alone).
std::shared_ptr<Tensor> exchangeGrad(const std::shared_ptr<ResourceList>&, const std::shared_ptr<Ewald>& ewald,
                                     const std::shared_ptr<PairList>& pl, const std::shared_ptr<Tensor>& D13,
                                     const std::shared_ptr<Tensor>& D24, bool D13symm, bool D24symm, bool Dsame,
                                     float thresp, float thredp,
                                     const std::shared_ptr<Tensor>& G = std::shared_ptr<Tensor>())
{
    const size_t n = pl->basis1()->nao(), natom = pl->basis1()->natom();
    D13->shape_error({n, n});
    D24->shape_error({n, n});
    std::shared_ptr<Tensor> out = G ? G : std::make_shared<Tensor>(std::vector<size_t>{natom, 3});
    out->shape_error({natom, 3});
    check(lsjk_exchange_grad(ctx(), (int) ewald->scales().size(), ewald->scales().data(), ewald->omegas().data(),
                             dev(pl), D13->data().data(), D24->data().data(), D13symm ? 1 : 0, D24symm ? 1 : 0,
                             Dsame ? 1 : 0, thresp, thredp, out->data().data()));
    return out;
}

} // namespace b200
} // namespace lightspeed

// ---- flat wrapper for the tests (reference objects made by oracle/ref_capi.cpp)
namespace {
thread_local std::string g_err;
}

extern "C" {

const char* shim_last_error() { return g_err.c_str(); }

// J or K through the reference-signature functions above. D (row-major) and
// out are host arrays; out is passed as the accumulating J12/K13 tensor when
// accumulate != 0, else a new tensor is made and copied to out.
int shim_jk(int which, void* pl12, void* pl34, int nterm, const double* scales, const double* omegas,
            const double* D, int d24symm, float thresp, float thredp, int accumulate, double* out)
{
    using namespace lightspeed;
    try {
        auto p12 = static_cast<oracle_ref::RefPairs*>(pl12)->p;
        auto p34 = static_cast<oracle_ref::RefPairs*>(pl34)->p;
        auto ew = std::make_shared<Ewald>(std::vector<double>(scales, scales + nterm),
                                          std::vector<double>(omegas, omegas + nterm));
        auto res = ResourceList::build_cpu();
        // D34 (nao3 x nao4) for J, D24 (nao2 x nao4) for K
        const size_t dr = which ? p12->basis2()->nao() : p34->basis1()->nao();
        const size_t dc = p34->basis2()->nao();
        auto Dt = std::make_shared<Tensor>(std::vector<size_t>{dr, dc});
        std::memcpy(Dt->data().data(), D, sizeof(double) * dr * dc);
        const size_t o1 = p12->basis1()->nao(), o2 = which ? p34->basis1()->nao() : p12->basis2()->nao();
        std::shared_ptr<Tensor> O;
        if (accumulate) {
            O = std::make_shared<Tensor>(std::vector<size_t>{o1, o2});
            std::memcpy(O->data().data(), out, sizeof(double) * o1 * o2);
        }
        std::shared_ptr<Tensor> R = which ? b200::exchange(res, ew, p12, p34, Dt, d24symm != 0, thresp, thredp, O)
                                          : b200::coulomb(res, ew, p12, p34, Dt, thresp, thredp, O);
        if (accumulate && R != O) throw std::runtime_error("the accumulating tensor was not returned");
        std::memcpy(out, R->data().data(), sizeof(double) * o1 * o2);
        return 0;
    } catch (std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// coulombGrad (which 0) or exchangeGrad (which 1) through the functions above:
// D1, D2 host (nao x nao) arrays (the same pointer: the same reference
// Tensor), G host (natom x 3), accumulated.
int shim_grad(int which, void* pl, int nterm, const double* scales, const double* omegas, const double* D1,
              const double* D2, int D13symm, int D24symm, int Dsame, float thresp, float thredp, double* G)
{
    using namespace lightspeed;
    try {
        auto p = static_cast<oracle_ref::RefPairs*>(pl)->p;
        auto ew = std::make_shared<Ewald>(std::vector<double>(scales, scales + nterm),
                                          std::vector<double>(omegas, omegas + nterm));
        auto res = ResourceList::build_cpu();
        const size_t n = p->basis1()->nao(), natom = p->basis1()->natom();
        auto A = std::make_shared<Tensor>(std::vector<size_t>{n, n});
        std::memcpy(A->data().data(), D1, sizeof(double) * n * n);
        std::shared_ptr<Tensor> B = A;
        if (D2 != D1) {
            B = std::make_shared<Tensor>(std::vector<size_t>{n, n});
            std::memcpy(B->data().data(), D2, sizeof(double) * n * n);
        }
        auto Gt = std::make_shared<Tensor>(std::vector<size_t>{natom, 3});
        std::memcpy(Gt->data().data(), G, sizeof(double) * natom * 3);
        auto R = which ? b200::exchangeGrad(res, ew, p, A, B, D13symm != 0, D24symm != 0, Dsame != 0, thresp,
                                            thredp, Gt)
                       : b200::coulombGrad(res, ew, p, A, B, thresp, thredp, Gt);
        if (R != Gt) throw std::runtime_error("the accumulating tensor was not returned");
        std::memcpy(G, R->data().data(), sizeof(double) * natom * 3);
        return 0;
    } catch (std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

} // extern "C"
