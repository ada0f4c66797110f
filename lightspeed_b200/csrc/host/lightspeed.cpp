// Implementation of the host API in lightspeed.hpp.
#include "lightspeed.hpp"
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <sstream>

namespace lightspeed {

void check_rc(int rc, const char* what)
{
    if (rc != LSJK_OK) {
        std::string msg = std::string(what) + ": " + lsjk_last_error();
        throw std::runtime_error(msg);
    }
}

// ---- Tensor -------------------------------------------------------------------

Tensor::Tensor(const std::vector<size_t>& shape, const std::string& name) : shape_(shape), name_(name)
{
    size_t n = 1;
    for (size_t s : shape) n *= s;
    data_.assign(n, 0.0);
}

void Tensor::shape_error(const std::vector<size_t>& shape) const
{
    if (shape != shape_) {
        std::ostringstream os;
        os << "Tensor::shape_error: " << name_ << " has shape (";
        for (size_t k = 0; k < shape_.size(); ++k) os << (k ? "," : "") << shape_[k];
        os << "), expected (";
        for (size_t k = 0; k < shape.size(); ++k) os << (k ? "," : "") << shape[k];
        os << ")";
        throw std::runtime_error(os.str());
    }
}

void Tensor::ndim_error(size_t ndim) const
{
    if (ndim != shape_.size()) throw std::runtime_error("Tensor::ndim_error: " + name_ + " has the wrong rank");
}

std::shared_ptr<Tensor> Tensor::clone() const
{
    auto t = std::make_shared<Tensor>(shape_, name_);
    t->data_ = data_;
    return t;
}

void Tensor::zero() { std::fill(data_.begin(), data_.end(), 0.0); }

std::string Tensor::string() const
{
    std::ostringstream os;
    os << "Tensor: " << name_ << " shape (";
    for (size_t k = 0; k < shape_.size(); ++k) os << (k ? "," : "") << shape_[k];
    os << ")";
    return os.str();
}

// ---- Primitive / Basis ---------------------------------------------------------

bool Primitive::operator==(const Primitive& o) const
{
    return c_ == o.c_ && e_ == o.e_ && x_ == o.x_ && y_ == o.y_ && z_ == o.z_ && c0_ == o.c0_ && L_ == o.L_ &&
           is_pure_ == o.is_pure_ && aoIdx_ == o.aoIdx_ && cartIdx_ == o.cartIdx_ && primIdx_ == o.primIdx_ &&
           shellIdx_ == o.shellIdx_ && atomIdx_ == o.atomIdx_;
}

Basis::Basis(const std::string& name, const std::vector<Primitive>& prims) : name_(name), primitives_(prims)
{
    for (size_t P = 0; P < prims.size(); ++P) {
        const Primitive& p = prims[P];
        if (p.primIdx() != (int) P) throw std::runtime_error("Basis: primIdx field is not dense");
        if (P == 0) {
            if (p.aoIdx() || p.cartIdx() || p.shellIdx() || p.atomIdx())
                throw std::runtime_error("Basis: index fields are not dense");
        } else {
            const Primitive& q = prims[P - 1];
            if (q.shellIdx() == p.shellIdx()) {
                if (q.aoIdx() != p.aoIdx() || q.cartIdx() != p.cartIdx() || q.atomIdx() != p.atomIdx())
                    throw std::runtime_error("Basis: index fields are not dense");
            } else if (q.shellIdx() + 1 == p.shellIdx()) {
                if (q.aoIdx() + q.nao() != p.aoIdx()) throw std::runtime_error("Basis: aoIdx field is not dense");
                if (q.cartIdx() + q.ncart() != p.cartIdx()) throw std::runtime_error("Basis: cartIdx field is not dense");
                if (q.atomIdx() != p.atomIdx() && q.atomIdx() + 1 != p.atomIdx())
                    throw std::runtime_error("Basis: atomIdx field is not dense");
            } else {
                throw std::runtime_error("Basis: shellIdx field is not dense");
            }
        }
    }
    if (!prims.empty()) {
        const Primitive& p = prims.back();
        nao_ = p.aoIdx() + p.nao();
        ncart_ = p.cartIdx() + p.ncart();
        nshell_ = p.shellIdx() + 1;
        natom_ = p.atomIdx() + 1;
    }
}

Basis::~Basis()
{
    if (handle_) lsjk_basis_destroy(handle_);
}

int Basis::max_L() const
{
    int m = 0;
    for (const auto& p : primitives_) m = std::max(m, p.L());
    return m;
}

bool Basis::has_pure() const
{
    for (const auto& p : primitives_)
        if (p.is_pure()) return true;
    return false;
}

bool Basis::equivalent(const std::shared_ptr<Basis>& a, const std::shared_ptr<Basis>& b)
{
    if (a->nao() != b->nao() || a->ncart() != b->ncart() || a->nprim() != b->nprim() ||
        a->nshell() != b->nshell() || a->natom() != b->natom())
        return false;
    return a->primitives() == b->primitives();
}

std::shared_ptr<Basis> Basis::concatenate(const std::vector<std::shared_ptr<Basis>>& bases)
{
    std::vector<Primitive> out;
    int ao = 0, cart = 0, prim = 0, shell = 0, atom = 0;
    std::string name;
    for (const auto& b : bases) {
        name += (name.empty() ? "" : "+") + b->name();
        for (const auto& p : b->primitives())
            out.emplace_back(p.c(), p.e(), p.x(), p.y(), p.z(), p.c0(), p.L(), p.is_pure(), p.aoIdx() + ao,
                             p.cartIdx() + cart, p.primIdx() + prim, p.shellIdx() + shell, p.atomIdx() + atom);
        ao += (int) b->nao();
        cart += (int) b->ncart();
        prim += (int) b->nprim();
        shell += (int) b->nshell();
        atom += (int) b->natom();
    }
    return std::make_shared<Basis>(name, out);
}

lsjk_basis* Basis::device_handle() const
{
    if (handle_) return handle_;
    size_t n = primitives_.size();
    std::vector<double> c(n), e(n), xyz(3 * n);
    std::vector<int> L(n), pu(n), ao(n), ca(n), pr(n), sh(n), at(n);
    for (size_t i = 0; i < n; ++i) {
        const Primitive& p = primitives_[i];
        c[i] = p.c(); e[i] = p.e();
        xyz[3 * i] = p.x(); xyz[3 * i + 1] = p.y(); xyz[3 * i + 2] = p.z();
        L[i] = p.L(); pu[i] = p.is_pure(); ao[i] = p.aoIdx(); ca[i] = p.cartIdx();
        pr[i] = p.primIdx(); sh[i] = p.shellIdx(); at[i] = p.atomIdx();
    }
    check_rc(lsjk_basis_create(Engine::instance().ctx(), (int) n, c.data(), e.data(), xyz.data(), L.data(),
                               pu.data(), ao.data(), ca.data(), pr.data(), sh.data(), at.data(), &handle_),
             "Basis");
    return handle_;
}

std::string Basis::string() const
{
    char buf[512];
    snprintf(buf, sizeof buf,
             "Basis: %s\n  nao     = %5zu\n  ncart   = %5zu\n  nprim   = %5zu\n  nshell  = %5zu\n"
             "  natom   = %5zu\n  pure?   = %5s\n  max L   = %5d\n",
             name_.c_str(), nao_, ncart_, nprim(), nshell_, natom_, has_pure() ? "Yes" : "No", max_L());
    return buf;
}

// ---- PairList --------------------------------------------------------------------

std::shared_ptr<PairList> PairList::build_schwarz(const std::shared_ptr<Basis>& basis1,
                                                  const std::shared_ptr<Basis>& basis2, bool is_symmetric,
                                                  float threpq)
{
    if (is_symmetric && (basis1->nprim() != basis2->nprim() || basis1->natom() != basis2->natom()))
        throw std::runtime_error("PairList::build_schwarz: basis sets are not symmetric");
    std::shared_ptr<PairList> pl(new PairList());
    pl->b1_ = basis1;
    pl->b2_ = basis2;
    pl->symm_ = is_symmetric;
    pl->thre_ = threpq;
    check_rc(lsjk_pairlist_build_schwarz(Engine::instance().ctx(), basis1->device_handle(),
                                         basis2->device_handle(), is_symmetric ? 1 : 0, threpq, &pl->handle_),
             "PairList::build_schwarz");
    long n = lsjk_pairlist_size(pl->handle_);
    std::vector<int> L1(n), L2(n), p1(n), p2(n);
    std::vector<float> b(n);
    check_rc(lsjk_pairlist_export(pl->handle_, L1.data(), L2.data(), p1.data(), p2.data(), b.data()),
             "PairList::build_schwarz");
    const auto& P1 = basis1->primitives();
    const auto& P2 = basis2->primitives();
    long k = 0;
    while (k < n) {
        long e = k;
        std::vector<Pair> pairs;
        while (e < n && L1[e] == L1[k] && L2[e] == L2[k]) {
            pairs.emplace_back(&P1[p1[e]], &P2[p2[e]], b[e]);
            ++e;
        }
        pl->pairlists_.emplace_back(is_symmetric, L1[k], L2[k], pairs);
        k = e;
    }
    return pl;
}

PairList::~PairList()
{
    if (handle_) lsjk_pairlist_destroy(handle_);
}

std::string PairList::string() const
{
    size_t n = 0;
    for (const auto& l : pairlists_) n += l.pairs().size();
    char buf[256];
    snprintf(buf, sizeof buf, "PairList:\n  symm? = %11s\n  thre  = %11.3E\n  npair = %11zu\n",
             symm_ ? "Yes" : "No", thre_, n);
    return buf;
}

// ---- Ewald / Engine / ResourceList -------------------------------------------------

Ewald::Ewald(const std::vector<double>& scales, const std::vector<double>& omegas) : scales_(scales), omegas_(omegas)
{
    if (scales.size() != omegas.size()) throw std::runtime_error("Ewald: scales and omegas must be same size.");
    if (scales.empty()) throw std::runtime_error("Ewald: scales/omegas must have >= 1 elements.");
}

Engine::Engine()
{
    const char* d = std::getenv("LSJK_DEVICE");
    device_ = d ? std::atoi(d) : 0;
    check_rc(lsjk_context_create(device_, &ctx_), "Engine");
}

Engine& Engine::instance()
{
    static Engine* e = new Engine();   // lives until process exit
    return *e;
}

void Engine::set_precision(int mode)
{
    check_rc(lsjk_context_set_precision(ctx_, mode), "Engine::set_precision");
    precision_ = mode;
}

void Engine::set_merge(bool on)
{
    check_rc(lsjk_context_set_merge(ctx_, on ? 1 : 0), "Engine::set_merge");
    merge_ = on;
}

std::shared_ptr<ResourceList> ResourceList::build(size_t, size_t)
{
    Engine::instance();
    return std::make_shared<ResourceList>(1, 1);
}

std::shared_ptr<ResourceList> ResourceList::build_cpu()
{
    // the J/K engine has no CPU path; a CPU-only resource list still routes
    // J/K to the GPU engine (there is nothing else to route to)
    return std::make_shared<ResourceList>(1, 0);
}

std::string ResourceList::string() const
{
    char buf[128];
    snprintf(buf, sizeof buf, "ResourceList:\n  CPU threads:  %3d\n  GPU contexts: %3d\n", nthread_, ngpu_);
    return buf;
}

// ---- IntBox -------------------------------------------------------------------------

namespace {

std::shared_ptr<Tensor> out_tensor(const std::shared_ptr<Tensor>& T, size_t n1, size_t n2, const char* name)
{
    if (T) {
        T->shape_error({n1, n2});
        return T;
    }
    return std::make_shared<Tensor>(std::vector<size_t>{n1, n2}, name);
}

} // namespace

std::shared_ptr<Tensor> IntBox::coulomb(const std::shared_ptr<ResourceList>& resources,
                                        const std::shared_ptr<Ewald>& ewald,
                                        const std::shared_ptr<PairList>& pl12, const std::shared_ptr<PairList>& pl34,
                                        const std::shared_ptr<Tensor>& D34, float thresp, float thredp,
                                        const std::shared_ptr<Tensor>& J12)
{
    return coulombMulti(resources, ewald, pl12, pl34, {D34}, thresp, thredp,
                        J12 ? std::vector<std::shared_ptr<Tensor>>{J12} : std::vector<std::shared_ptr<Tensor>>{})[0];
}

std::shared_ptr<Tensor> IntBox::coulombGrad(const std::shared_ptr<ResourceList>&, const std::shared_ptr<Ewald>& ewald,
                                            const std::shared_ptr<PairList>& pl, const std::shared_ptr<Tensor>& D12,
                                            const std::shared_ptr<Tensor>& D34, float thresp, float thredp,
                                            const std::shared_ptr<Tensor>& G)
{
    const size_t n = pl->basis1()->nao();
    D12->shape_error({n, n});
    D34->shape_error({n, n});
    auto out = out_tensor(G, pl->basis1()->natom(), 3, "G");
    // D12 == D34 (one object) is the reference's symmetric branch: pass one pointer
    const double* d12 = D12->data().data();
    const double* d34 = D12 == D34 ? d12 : D34->data().data();
    check_rc(lsjk_coulomb_grad(Engine::instance().ctx(), (int) ewald->scales().size(), ewald->scales().data(),
                               ewald->omegas().data(), pl->device_handle(), d12, d34, thresp, thredp,
                               out->data().data()),
             "IntBox::coulombGrad");
    return out;
}

std::shared_ptr<Tensor> IntBox::exchangeGrad(const std::shared_ptr<ResourceList>&, const std::shared_ptr<Ewald>& ewald,
                                             const std::shared_ptr<PairList>& pl, const std::shared_ptr<Tensor>& D13,
                                             const std::shared_ptr<Tensor>& D24, bool D13symm, bool D24symm,
                                             bool Dsame, float thresp, float thredp,
                                             const std::shared_ptr<Tensor>& G)
{
    const size_t n = pl->basis1()->nao();
    D13->shape_error({n, n});
    D24->shape_error({n, n});
    auto out = out_tensor(G, pl->basis1()->natom(), 3, "G");
    const double* d13 = D13->data().data();
    const double* d24 = D13 == D24 ? d13 : D24->data().data();
    check_rc(lsjk_exchange_grad(Engine::instance().ctx(), (int) ewald->scales().size(), ewald->scales().data(),
                                ewald->omegas().data(), pl->device_handle(), d13, d24, D13symm, D24symm, Dsame,
                                thresp, thredp, out->data().data()),
             "IntBox::exchangeGrad");
    return out;
}

std::shared_ptr<Tensor> IntBox::exchange(const std::shared_ptr<ResourceList>& resources,
                                         const std::shared_ptr<Ewald>& ewald,
                                         const std::shared_ptr<PairList>& pl12, const std::shared_ptr<PairList>& pl34,
                                         const std::shared_ptr<Tensor>& D24, bool D24symm, float thresp,
                                         float thredp, const std::shared_ptr<Tensor>& K13)
{
    return exchangeMulti(resources, ewald, pl12, pl34, {D24}, D24symm, thresp, thredp,
                         K13 ? std::vector<std::shared_ptr<Tensor>>{K13} : std::vector<std::shared_ptr<Tensor>>{})[0];
}

std::vector<std::shared_ptr<Tensor>> IntBox::coulombMulti(
    const std::shared_ptr<ResourceList>&, const std::shared_ptr<Ewald>& ewald,
    const std::shared_ptr<PairList>& pl12, const std::shared_ptr<PairList>& pl34,
    const std::vector<std::shared_ptr<Tensor>>& D34, float thresp, float thredp,
    const std::vector<std::shared_ptr<Tensor>>& J12)
{
    if (!J12.empty() && J12.size() != D34.size()) throw std::runtime_error("IntBox::coulomb: D/J count mismatch");
    size_t n1 = pl12->basis1()->nao(), n2 = pl12->basis2()->nao();
    size_t n3 = pl34->basis1()->nao(), n4 = pl34->basis2()->nao();
    std::vector<std::shared_ptr<Tensor>> out;
    std::vector<const double*> dp;
    std::vector<double*> jp;
    for (size_t k = 0; k < D34.size(); ++k) {
        D34[k]->shape_error({n3, n4});
        out.push_back(out_tensor(J12.empty() ? nullptr : J12[k], n1, n2, "J"));
        dp.push_back(D34[k]->data().data());
        jp.push_back(out.back()->data().data());
    }
    check_rc(lsjk_coulomb(Engine::instance().ctx(), (int) ewald->scales().size(), ewald->scales().data(),
                          ewald->omegas().data(), pl12->device_handle(), pl34->device_handle(), (int) D34.size(),
                          dp.data(), thresp, thredp, jp.data()),
             "IntBox::coulomb");
    return out;
}

std::vector<std::shared_ptr<Tensor>> IntBox::exchangeMulti(
    const std::shared_ptr<ResourceList>&, const std::shared_ptr<Ewald>& ewald,
    const std::shared_ptr<PairList>& pl12, const std::shared_ptr<PairList>& pl34,
    const std::vector<std::shared_ptr<Tensor>>& D24, bool D24symm, float thresp, float thredp,
    const std::vector<std::shared_ptr<Tensor>>& K13)
{
    if (!K13.empty() && K13.size() != D24.size()) throw std::runtime_error("IntBox::exchange: D/K count mismatch");
    size_t n1 = pl12->basis1()->nao(), n2 = pl12->basis2()->nao();
    size_t n3 = pl34->basis1()->nao(), n4 = pl34->basis2()->nao();
    std::vector<std::shared_ptr<Tensor>> out;
    std::vector<const double*> dp;
    std::vector<double*> kp;
    for (size_t k = 0; k < D24.size(); ++k) {
        D24[k]->shape_error({n2, n4});
        out.push_back(out_tensor(K13.empty() ? nullptr : K13[k], n1, n3, "K"));
        dp.push_back(D24[k]->data().data());
        kp.push_back(out.back()->data().data());
    }
    check_rc(lsjk_exchange(Engine::instance().ctx(), (int) ewald->scales().size(), ewald->scales().data(),
                           ewald->omegas().data(), pl12->device_handle(), pl34->device_handle(), (int) D24.size(),
                           dp.data(), D24symm ? 1 : 0, thresp, thredp, kp.data()),
             "IntBox::exchange");
    return out;
}

std::shared_ptr<Tensor> IntBox::eriJ(const std::shared_ptr<ResourceList>&, const std::shared_ptr<Ewald>& ewald,
                                     const std::shared_ptr<PairList>& pl12, const std::shared_ptr<PairList>& pl34,
                                     const std::shared_ptr<Tensor>& C1, const std::shared_ptr<Tensor>& C2,
                                     const std::shared_ptr<Tensor>& C3, const std::shared_ptr<Tensor>& C4,
                                     float thresp, float thredp, const std::shared_ptr<Tensor>& I)
{
    const std::shared_ptr<Tensor>* C[4] = {&C1, &C2, &C3, &C4};
    const size_t nao[4] = {pl12->basis1()->nao(), pl12->basis2()->nao(), pl34->basis1()->nao(),
                           pl34->basis2()->nao()};
    size_t n[4];
    for (int a = 0; a < 4; ++a) {
        if (!*C[a]) throw std::runtime_error("IntBox::eriJ: null coefficient tensor");
        (*C[a])->ndim_error(2);
        n[a] = (*C[a])->shape()[1];
        (*C[a])->shape_error({nao[a], n[a]});
    }
    std::shared_ptr<Tensor> out = I;
    if (out)
        out->shape_error({n[0], n[1], n[2], n[3]});
    else
        out = std::make_shared<Tensor>(std::vector<size_t>{n[0], n[1], n[2], n[3]}, "I");
    check_rc(lsjk_eri_j(Engine::instance().ctx(), (int) ewald->scales().size(), ewald->scales().data(),
                        ewald->omegas().data(), pl12->device_handle(), pl34->device_handle(), (int) n[0], (int) n[1],
                        (int) n[2], (int) n[3], C1->data().data(), C2->data().data(), C3->data().data(),
                        C4->data().data(), C1 == C2 ? 1 : 0, C3 == C4 ? 1 : 0, (C1 == C3 && C2 == C4) ? 1 : 0,
                        thresp, thredp, out->data().data()),
             "IntBox::eriJ");
    return out;
}

} // namespace lightspeed
