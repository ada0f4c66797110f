// One-electron integrals S, T, V for the SCF drivers around the J/K path:
// IntBox::overlap / kinetic / potential (src/lightspeed/intbox.hpp; CPU
// kernels src/cpp/intbox/cpu/overlap.cpp, kinetic.cpp, potential.cpp),
// computed on the device through the C ABI (lsjk_overlap, lsjk_kinetic,
// lsjk_potential) over the same primitive pair lists, accumulated into the
// given tensor or a new zeroed one.
#include <stdexcept>
#include "lightspeed.hpp"
#include "oneint.hpp"

namespace lightspeed {

namespace {

std::shared_ptr<Tensor> out_for(const std::shared_ptr<PairList>& pl, const std::shared_ptr<Tensor>& out,
                                const char* name)
{
    const size_t n1 = pl->basis1()->nao(), n2 = pl->basis2()->nao();
    auto T = out ? out : std::make_shared<Tensor>(std::vector<size_t>{n1, n2}, name);
    T->shape_error({n1, n2});
    return T;
}

} // namespace

std::shared_ptr<Tensor> OneInt::overlap(const std::shared_ptr<PairList>& pl, const std::shared_ptr<Tensor>& S)
{
    auto T = out_for(pl, S, "S");
    check_rc(lsjk_overlap(Engine::instance().ctx(), pl->device_handle(), T->data().data()), "IntBox::overlap");
    return T;
}

std::shared_ptr<Tensor> OneInt::kinetic(const std::shared_ptr<PairList>& pl, const std::shared_ptr<Tensor>& T)
{
    auto X = out_for(pl, T, "T");
    check_rc(lsjk_kinetic(Engine::instance().ctx(), pl->device_handle(), X->data().data()), "IntBox::kinetic");
    return X;
}

std::shared_ptr<Tensor> OneInt::potential(const std::shared_ptr<Ewald>& ewald, const std::shared_ptr<PairList>& pl,
                                          const std::shared_ptr<Tensor>& xyzc, const std::shared_ptr<Tensor>& V)
{
    xyzc->ndim_error(2);
    if (xyzc->shape()[1] != 4) throw std::runtime_error("IntBox::potential: xyzc must be (natom, 4)");
    auto X = out_for(pl, V, "V");
    check_rc(lsjk_potential(Engine::instance().ctx(), (int) ewald->scales().size(), ewald->scales().data(),
                            ewald->omegas().data(), pl->device_handle(), (int) xyzc->shape()[0],
                            xyzc->data().data(), X->data().data()),
             "IntBox::potential");
    return X;
}

} // namespace lightspeed
