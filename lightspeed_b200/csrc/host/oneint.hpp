// One-electron integrals (S, T, V) used by the SCF drivers of the J/K path.
#pragma once
#include <memory>
#include "lightspeed.hpp"

namespace lightspeed {

struct OneInt {
    static std::shared_ptr<Tensor> overlap(const std::shared_ptr<PairList>& pl, const std::shared_ptr<Tensor>& S);
    static std::shared_ptr<Tensor> kinetic(const std::shared_ptr<PairList>& pl, const std::shared_ptr<Tensor>& T);
    static std::shared_ptr<Tensor> potential(const std::shared_ptr<Ewald>& ewald, const std::shared_ptr<PairList>& pl,
                                             const std::shared_ptr<Tensor>& xyzc, const std::shared_ptr<Tensor>& V);
};

} // namespace lightspeed
