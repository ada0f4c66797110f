// Host-side C++ API of the J/K path, with the names, argument meanings and
// error behaviour of the reference Lightspeed classes it stands in for:
//   Tensor        src/lightspeed/tensor.hpp:19-320   (row-major double)
//   Primitive     src/lightspeed/basis.hpp:143-172
//   Basis         src/lightspeed/basis.hpp:404-614
//   Pair/PairListL/PairList   src/lightspeed/pair_list.hpp:25-288
//   Ewald         src/lightspeed/ewald.hpp:25-109
//   ResourceList  src/lightspeed/resource_list.hpp:25-73
//   IntBox::coulomb/exchange  src/lightspeed/intbox.hpp:761-771, 817-828
//   IntBox::eriJ  src/lightspeed/intbox.hpp:1349, src/cpp/intbox/mo_eri.cpp:10-157
// The integral work goes through the C ABI in include/lsjk.h (liblsjk.so);
// nothing here computes J or K on the CPU.
#pragma once
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#include "lsjk.h"

namespace lightspeed {

class Tensor {
public:
    explicit Tensor(const std::vector<size_t>& shape, const std::string& name = "T");
    const std::vector<size_t>& shape() const { return shape_; }
    size_t ndim() const { return shape_.size(); }
    size_t size() const { return data_.size(); }
    const std::string& name() const { return name_; }
    std::vector<double>& data() { return data_; }
    const std::vector<double>& data() const { return data_; }
    // throws std::runtime_error if the shape differs (Tensor::shape_error)
    void shape_error(const std::vector<size_t>& shape) const;
    void ndim_error(size_t ndim) const;
    std::shared_ptr<Tensor> clone() const;
    void zero();
    std::string string() const;

private:
    std::vector<size_t> shape_;
    std::string name_;
    std::vector<double> data_;
};

class Primitive {
public:
    Primitive(double c, double e, double x, double y, double z, double c0, int L, bool is_pure,
              int aoIdx, int cartIdx, int primIdx, int shellIdx, int atomIdx)
        : c_(c), e_(e), x_(x), y_(y), z_(z), c0_(c0), L_(L), is_pure_(is_pure), aoIdx_(aoIdx),
          cartIdx_(cartIdx), primIdx_(primIdx), shellIdx_(shellIdx), atomIdx_(atomIdx) {}
    double c() const { return c_; }
    double e() const { return e_; }
    double x() const { return x_; }
    double y() const { return y_; }
    double z() const { return z_; }
    double c0() const { return c0_; }
    int L() const { return L_; }
    bool is_pure() const { return is_pure_; }
    int aoIdx() const { return aoIdx_; }
    int cartIdx() const { return cartIdx_; }
    int primIdx() const { return primIdx_; }
    int shellIdx() const { return shellIdx_; }
    int atomIdx() const { return atomIdx_; }
    int ncart() const { return (L_ + 1) * (L_ + 2) / 2; }
    int npure() const { return 2 * L_ + 1; }
    int nao() const { return is_pure_ ? npure() : ncart(); }
    bool operator==(const Primitive& o) const;
    bool operator!=(const Primitive& o) const { return !(*this == o); }

private:
    double c_, e_, x_, y_, z_, c0_;
    int L_;
    bool is_pure_;
    int aoIdx_, cartIdx_, primIdx_, shellIdx_, atomIdx_;
};

class Engine;

class Basis {
public:
    Basis(const std::string& name, const std::vector<Primitive>& primitives);
    ~Basis();
    const std::string& name() const { return name_; }
    const std::vector<Primitive>& primitives() const { return primitives_; }
    size_t nao() const { return nao_; }
    size_t ncart() const { return ncart_; }
    size_t nprim() const { return primitives_.size(); }
    size_t nshell() const { return nshell_; }
    size_t natom() const { return natom_; }
    int max_L() const;
    bool has_pure() const;
    static bool equivalent(const std::shared_ptr<Basis>& a, const std::shared_ptr<Basis>& b);
    static std::shared_ptr<Basis> concatenate(const std::vector<std::shared_ptr<Basis>>& bases);
    // the engine's device copy (created on first use)
    lsjk_basis* device_handle() const;
    std::string string() const;

private:
    std::string name_;
    std::vector<Primitive> primitives_;
    size_t nao_ = 0, ncart_ = 0, nshell_ = 0, natom_ = 0;
    mutable lsjk_basis* handle_ = nullptr;
};

class Pair {
public:
    Pair(const Primitive* p1, const Primitive* p2, float bound) : p1_(p1), p2_(p2), bound_(bound) {}
    const Primitive& prim1() const { return *p1_; }
    const Primitive& prim2() const { return *p2_; }
    float bound() const { return bound_; }

private:
    const Primitive* p1_;
    const Primitive* p2_;
    float bound_;
};

class PairListL {
public:
    PairListL(bool is_symmetric, int L1, int L2, const std::vector<Pair>& pairs)
        : symm_(is_symmetric), L1_(L1), L2_(L2), pairs_(pairs) {}
    bool is_symmetric() const { return symm_; }
    int L1() const { return L1_; }
    int L2() const { return L2_; }
    const std::vector<Pair>& pairs() const { return pairs_; }

private:
    bool symm_;
    int L1_, L2_;
    std::vector<Pair> pairs_;
};

class PairList {
public:
    // Built on the device (include/lsjk.h: lsjk_pairlist_build_schwarz).
    static std::shared_ptr<PairList> build_schwarz(const std::shared_ptr<Basis>& basis1,
                                                   const std::shared_ptr<Basis>& basis2,
                                                   bool is_symmetric, float threpq);
    ~PairList();
    std::shared_ptr<Basis> basis1() const { return b1_; }
    std::shared_ptr<Basis> basis2() const { return b2_; }
    bool is_symmetric() const { return symm_; }
    float thre() const { return thre_; }
    const std::vector<PairListL>& pairlists() const { return pairlists_; }
    lsjk_pairlist* device_handle() const { return handle_; }
    std::string string() const;

private:
    PairList() = default;
    std::shared_ptr<Basis> b1_, b2_;
    bool symm_ = false;
    float thre_ = 0.f;
    std::vector<PairListL> pairlists_;
    lsjk_pairlist* handle_ = nullptr;
};

class Ewald {
public:
    Ewald(const std::vector<double>& scales, const std::vector<double>& omegas);
    static std::shared_ptr<Ewald> coulomb() { return std::make_shared<Ewald>(std::vector<double>{1.0}, std::vector<double>{-1.0}); }
    const std::vector<double>& scales() const { return scales_; }
    const std::vector<double>& omegas() const { return omegas_; }
    bool is_coulomb() const { return omegas_.size() == 1 && omegas_[0] == -1.0; }

private:
    std::vector<double> scales_, omegas_;
};

// The process-wide engine session on one GPU (the reference keeps one
// TCIntBox session per process, tc/tcintbox/tcintbox.cpp:18-27).
class Engine {
public:
    static Engine& instance();
    lsjk_context* ctx() const { return ctx_; }
    int device() const { return device_; }
    void set_precision(int mode);
    int precision() const { return precision_; }
    void set_merge(bool on);
    bool merge() const { return merge_; }

private:
    Engine();
    lsjk_context* ctx_ = nullptr;
    int device_ = 0;
    int precision_ = LSJK_PREC_MIXED;
    bool merge_ = false;
};

class ResourceList {
public:
    ResourceList(int nthread, int ngpu) : nthread_(nthread), ngpu_(ngpu) {}
    static std::shared_ptr<ResourceList> build(size_t cpu_memory = 1024, size_t gpu_memory = 1024);
    static std::shared_ptr<ResourceList> build_cpu();
    int nthread() const { return nthread_; }
    int ngpu() const { return ngpu_; }
    std::string string() const;

private:
    int nthread_, ngpu_;
};

class IntBox {
public:
    static std::shared_ptr<Tensor> coulomb(const std::shared_ptr<ResourceList>& resources,
                                           const std::shared_ptr<Ewald>& ewald,
                                           const std::shared_ptr<PairList>& pairlist12,
                                           const std::shared_ptr<PairList>& pairlist34,
                                           const std::shared_ptr<Tensor>& D34, float thresp, float thredp,
                                           const std::shared_ptr<Tensor>& J12 = std::shared_ptr<Tensor>());
    // J nuclear gradient (src/lightspeed/intbox.hpp:998-1008): G (natom, 3) +=
    // sum D12 d(12|34) D34 over a symmetric pair list; D12 and D34 the same
    // object selects the symmetric branch, as in the reference.
    static std::shared_ptr<Tensor> coulombGrad(const std::shared_ptr<ResourceList>& resources,
                                               const std::shared_ptr<Ewald>& ewald,
                                               const std::shared_ptr<PairList>& pairlist,
                                               const std::shared_ptr<Tensor>& D12,
                                               const std::shared_ptr<Tensor>& D34, float thresp, float thredp,
                                               const std::shared_ptr<Tensor>& G = std::shared_ptr<Tensor>());
    // K nuclear gradient (src/lightspeed/intbox.hpp:1095-1160): G (natom, 3) +=
    // sum D13 d(12|34) D24 over a symmetric pair list. D13symm, D24symm, Dsame
    // are the reference's promises: D13symm and D24symm let each pair of equal terms
    // be computed once; all three select the reference's fully symmetric routine.
    static std::shared_ptr<Tensor> exchangeGrad(const std::shared_ptr<ResourceList>& resources,
                                                const std::shared_ptr<Ewald>& ewald,
                                                const std::shared_ptr<PairList>& pairlist,
                                                const std::shared_ptr<Tensor>& D13,
                                                const std::shared_ptr<Tensor>& D24, bool D13symm, bool D24symm,
                                                bool Dsame, float thresp, float thredp,
                                                const std::shared_ptr<Tensor>& G = std::shared_ptr<Tensor>());
    static std::shared_ptr<Tensor> exchange(const std::shared_ptr<ResourceList>& resources,
                                            const std::shared_ptr<Ewald>& ewald,
                                            const std::shared_ptr<PairList>& pairlist12,
                                            const std::shared_ptr<PairList>& pairlist34,
                                            const std::shared_ptr<Tensor>& D24, bool D24symm, float thresp,
                                            float thredp,
                                            const std::shared_ptr<Tensor>& K13 = std::shared_ptr<Tensor>());
    // Batched forms: many densities through one engine call (no reference
    // counterpart; the reference loops IntBox calls per density in est/cis.py).
    static std::vector<std::shared_ptr<Tensor>> coulombMulti(
        const std::shared_ptr<ResourceList>& resources, const std::shared_ptr<Ewald>& ewald,
        const std::shared_ptr<PairList>& pairlist12, const std::shared_ptr<PairList>& pairlist34,
        const std::vector<std::shared_ptr<Tensor>>& D34, float thresp, float thredp,
        const std::vector<std::shared_ptr<Tensor>>& J12 = {});
    static std::vector<std::shared_ptr<Tensor>> exchangeMulti(
        const std::shared_ptr<ResourceList>& resources, const std::shared_ptr<Ewald>& ewald,
        const std::shared_ptr<PairList>& pairlist12, const std::shared_ptr<PairList>& pairlist34,
        const std::vector<std::shared_ptr<Tensor>>& D24, bool D24symm, float thresp, float thredp,
        const std::vector<std::shared_ptr<Tensor>>& K13 = {});
    // (C1_i C2_j | C3_k C4_l) through J builds (mo_eri.cpp:10-157); the
    // symmetrisations follow the reference's tests of object identity
    // (C1 is C2, C3 is C4, C1 is C3 and C2 is C4).
    static std::shared_ptr<Tensor> eriJ(const std::shared_ptr<ResourceList>& resources,
                                        const std::shared_ptr<Ewald>& ewald,
                                        const std::shared_ptr<PairList>& pairlist12,
                                        const std::shared_ptr<PairList>& pairlist34,
                                        const std::shared_ptr<Tensor>& C1, const std::shared_ptr<Tensor>& C2,
                                        const std::shared_ptr<Tensor>& C3, const std::shared_ptr<Tensor>& C4,
                                        float thresp, float thredp,
                                        const std::shared_ptr<Tensor>& I = std::shared_ptr<Tensor>());
};

// Raise std::runtime_error with the engine's message when rc != 0.
void check_rc(int rc, const char* what);

} // namespace lightspeed
