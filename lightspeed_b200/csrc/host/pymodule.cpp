// Python binding of the host API (module lightspeed_b200._lightspeed), with
// the class and method names of the reference's Boost.Python module
// (src/python/export_intbox.cpp:127-158, export_core.cpp:241-309,
// export_env.cpp:19-66, export_tensor.cpp:8-24).
#include <pybind11/pybind11.h>
#include <pybind11/numpy.h>
#include <pybind11/stl.h>
#include "lightspeed.hpp"
#include "oneint.hpp"

namespace py = pybind11;
using namespace lightspeed;

namespace {

py::array tensor_view(const std::shared_ptr<Tensor>& t)
{
    std::vector<py::ssize_t> shape(t->shape().begin(), t->shape().end());
    std::vector<py::ssize_t> strides(shape.size());
    py::ssize_t s = sizeof(double);
    for (int k = (int) shape.size() - 1; k >= 0; --k) {
        strides[k] = s;
        s *= shape[k];
    }
    // the numpy array keeps the Tensor alive through its base object
    py::object owner = py::cast(t);
    return py::array(py::dtype::of<double>(), shape, strides, t->data().data(), owner);
}

std::shared_ptr<Tensor> tensor_from_array(py::array_t<double, py::array::c_style | py::array::forcecast> a,
                                          const std::string& name)
{
    std::vector<size_t> shape(a.shape(), a.shape() + a.ndim());
    auto t = std::make_shared<Tensor>(shape, name);
    std::copy(a.data(), a.data() + a.size(), t->data().begin());
    return t;
}

py::dict stats_dict_of(lsjk_context* ctx)
{
    lsjk_stats st{};
    check_rc(lsjk_context_stats(ctx, &st), "stats");
    py::dict d;
    d["quartets_fp64"] = st.quartets_fp64;
    d["quartets_fp32"] = st.quartets_fp32;
    d["j_quartets"] = st.j_quartets;
    d["k_quartets"] = st.k_quartets;
    d["flops_j"] = st.flops_j;
    d["flops_k"] = st.flops_k;
    d["kernel_launches"] = st.kernel_launches;
    return d;
}

py::dict stats_dict() { return stats_dict_of(Engine::instance().ctx()); }

} // namespace

PYBIND11_MODULE(_lightspeed, m)
{
    m.doc() = "B200 J/K engine: host API mirroring the Lightspeed IntBox J/K path";

    py::class_<Tensor, std::shared_ptr<Tensor>>(m, "Tensor", py::buffer_protocol())
        .def(py::init<const std::vector<size_t>&, const std::string&>(), py::arg("shape"), py::arg("name") = "T")
        .def_property_readonly("shape", [](const Tensor& t) { return py::tuple(py::cast(t.shape())); })
        .def_property_readonly("ndim", &Tensor::ndim)
        .def_property_readonly("size", &Tensor::size)
        .def_property_readonly("name", &Tensor::name)
        .def_property_readonly("np", [](const std::shared_ptr<Tensor>& t) { return tensor_view(t); })
        .def("clone", &Tensor::clone)
        .def("zero", &Tensor::zero)
        .def("shape_error", &Tensor::shape_error)
        .def("__str__", &Tensor::string)
        .def_static("array", &tensor_from_array, py::arg("array"), py::arg("name") = "T")
        .def_static("zeros", [](const std::vector<size_t>& shape, const std::string& name) {
            return std::make_shared<Tensor>(shape, name);
        }, py::arg("shape"), py::arg("name") = "T")
        .def_buffer([](Tensor& t) -> py::buffer_info {
            std::vector<py::ssize_t> shape(t.shape().begin(), t.shape().end());
            std::vector<py::ssize_t> strides(shape.size());
            py::ssize_t s = sizeof(double);
            for (int k = (int) shape.size() - 1; k >= 0; --k) {
                strides[k] = s;
                s *= shape[k];
            }
            return py::buffer_info(t.data().data(), sizeof(double), py::format_descriptor<double>::format(),
                                   (py::ssize_t) shape.size(), shape, strides);
        });

    py::class_<Primitive>(m, "Primitive")
        .def(py::init<double, double, double, double, double, double, int, bool, int, int, int, int, int>(),
             py::arg("c"), py::arg("e"), py::arg("x"), py::arg("y"), py::arg("z"), py::arg("c0"), py::arg("L"),
             py::arg("is_pure"), py::arg("aoIdx"), py::arg("cartIdx"), py::arg("primIdx"), py::arg("shellIdx"),
             py::arg("atomIdx"))
        .def_property_readonly("c", &Primitive::c)
        .def_property_readonly("e", &Primitive::e)
        .def_property_readonly("x", &Primitive::x)
        .def_property_readonly("y", &Primitive::y)
        .def_property_readonly("z", &Primitive::z)
        .def_property_readonly("c0", &Primitive::c0)
        .def_property_readonly("L", &Primitive::L)
        .def_property_readonly("is_pure", &Primitive::is_pure)
        .def_property_readonly("aoIdx", &Primitive::aoIdx)
        .def_property_readonly("cartIdx", &Primitive::cartIdx)
        .def_property_readonly("primIdx", &Primitive::primIdx)
        .def_property_readonly("shellIdx", &Primitive::shellIdx)
        .def_property_readonly("atomIdx", &Primitive::atomIdx)
        .def_property_readonly("ncart", &Primitive::ncart)
        .def_property_readonly("npure", &Primitive::npure)
        .def_property_readonly("nao", &Primitive::nao)
        .def("__eq__", &Primitive::operator==);

    py::class_<Basis, std::shared_ptr<Basis>>(m, "Basis")
        .def(py::init<const std::string&, const std::vector<Primitive>&>(), py::arg("name"), py::arg("primitives"))
        .def_property_readonly("name", &Basis::name)
        .def_property_readonly("primitives", &Basis::primitives)
        .def_property_readonly("nao", &Basis::nao)
        .def_property_readonly("ncart", &Basis::ncart)
        .def_property_readonly("nprim", &Basis::nprim)
        .def_property_readonly("nshell", &Basis::nshell)
        .def_property_readonly("natom", &Basis::natom)
        .def_property_readonly("max_L", &Basis::max_L)
        .def_property_readonly("has_pure", &Basis::has_pure)
        .def_static("equivalent", &Basis::equivalent)
        .def_static("concatenate", &Basis::concatenate)
        .def("__str__", &Basis::string);

    py::class_<Pair>(m, "Pair")
        .def_property_readonly("prim1", &Pair::prim1, py::return_value_policy::reference_internal)
        .def_property_readonly("prim2", &Pair::prim2, py::return_value_policy::reference_internal)
        .def_property_readonly("bound", &Pair::bound);

    py::class_<PairListL>(m, "PairListL")
        .def_property_readonly("is_symmetric", &PairListL::is_symmetric)
        .def_property_readonly("L1", &PairListL::L1)
        .def_property_readonly("L2", &PairListL::L2)
        .def_property_readonly("pairs", &PairListL::pairs, py::return_value_policy::reference_internal);

    py::class_<PairList, std::shared_ptr<PairList>>(m, "PairList")
        .def_static("build_schwarz", &PairList::build_schwarz, py::arg("basis1"), py::arg("basis2"),
                    py::arg("is_symmetric"), py::arg("thre"))
        .def_property_readonly("basis1", &PairList::basis1)
        .def_property_readonly("basis2", &PairList::basis2)
        .def_property_readonly("is_symmetric", &PairList::is_symmetric)
        .def_property_readonly("thre", &PairList::thre)
        .def_property_readonly("pairlists", &PairList::pairlists, py::return_value_policy::reference_internal)
        .def("__str__", &PairList::string);

    py::class_<Ewald, std::shared_ptr<Ewald>>(m, "Ewald")
        .def(py::init<const std::vector<double>&, const std::vector<double>&>(), py::arg("scales"),
             py::arg("omegas"))
        .def_static("coulomb", &Ewald::coulomb)
        .def_property_readonly("scales", &Ewald::scales)
        .def_property_readonly("omegas", &Ewald::omegas)
        .def_property_readonly("is_coulomb", &Ewald::is_coulomb);

    py::class_<ResourceList, std::shared_ptr<ResourceList>>(m, "ResourceList")
        .def_static("build", &ResourceList::build, py::arg("cpu_memory") = 1024, py::arg("gpu_memory") = 1024)
        .def_static("build_cpu", &ResourceList::build_cpu)
        .def_property_readonly("nthread", &ResourceList::nthread)
        .def_property_readonly("ngpu", &ResourceList::ngpu)
        .def("__str__", &ResourceList::string);

    py::class_<IntBox>(m, "IntBox")
        .def_static("coulomb", &IntBox::coulomb, py::arg("resources"), py::arg("ewald"), py::arg("pairlist12"),
                    py::arg("pairlist34"), py::arg("D34"), py::arg("thresp"), py::arg("thredp"),
                    py::arg("J12") = std::shared_ptr<Tensor>(), py::call_guard<py::gil_scoped_release>())
        .def_static("coulombGrad", &IntBox::coulombGrad, py::arg("resources"), py::arg("ewald"), py::arg("pairlist"),
                    py::arg("D12"), py::arg("D34"), py::arg("thresp"), py::arg("thredp"),
                    py::arg("G") = std::shared_ptr<Tensor>(), py::call_guard<py::gil_scoped_release>())
        .def_static("exchangeGrad", &IntBox::exchangeGrad, py::arg("resources"), py::arg("ewald"),
                    py::arg("pairlist"), py::arg("D13"), py::arg("D24"), py::arg("D13symm"), py::arg("D24symm"),
                    py::arg("Dsame"), py::arg("thresp"), py::arg("thredp"), py::arg("G") = std::shared_ptr<Tensor>(),
                    py::call_guard<py::gil_scoped_release>())
        .def_static("exchange", &IntBox::exchange, py::arg("resources"), py::arg("ewald"), py::arg("pairlist12"),
                    py::arg("pairlist34"), py::arg("D24"), py::arg("D24symm"), py::arg("thresp"),
                    py::arg("thredp"), py::arg("K13") = std::shared_ptr<Tensor>(),
                    py::call_guard<py::gil_scoped_release>())
        .def_static("coulombMulti", &IntBox::coulombMulti, py::arg("resources"), py::arg("ewald"),
                    py::arg("pairlist12"), py::arg("pairlist34"), py::arg("D34"), py::arg("thresp"),
                    py::arg("thredp"), py::arg("J12") = std::vector<std::shared_ptr<Tensor>>(),
                    py::call_guard<py::gil_scoped_release>())
        .def_static("exchangeMulti", &IntBox::exchangeMulti, py::arg("resources"), py::arg("ewald"),
                    py::arg("pairlist12"), py::arg("pairlist34"), py::arg("D24"), py::arg("D24symm"),
                    py::arg("thresp"), py::arg("thredp"), py::arg("K13") = std::vector<std::shared_ptr<Tensor>>(),
                    py::call_guard<py::gil_scoped_release>())
        .def_static("eriJ", &IntBox::eriJ, py::arg("resources"), py::arg("ewald"), py::arg("pairlist12"),
                    py::arg("pairlist34"), py::arg("C1"), py::arg("C2"), py::arg("C3"), py::arg("C4"),
                    py::arg("thresp"), py::arg("thredp"), py::arg("I") = std::shared_ptr<Tensor>(),
                    py::call_guard<py::gil_scoped_release>())
        // one-electron integrals for the SCF drivers (device kernels, oneint.cu)
        .def_static("overlap", [](const std::shared_ptr<ResourceList>&, const std::shared_ptr<PairList>& pl,
                                  const std::shared_ptr<Tensor>& S) { return OneInt::overlap(pl, S); },
                    py::arg("resources"), py::arg("pairlist"), py::arg("S") = std::shared_ptr<Tensor>(),
                    py::call_guard<py::gil_scoped_release>())
        .def_static("kinetic", [](const std::shared_ptr<ResourceList>&, const std::shared_ptr<PairList>& pl,
                                  const std::shared_ptr<Tensor>& T) { return OneInt::kinetic(pl, T); },
                    py::arg("resources"), py::arg("pairlist"), py::arg("T") = std::shared_ptr<Tensor>(),
                    py::call_guard<py::gil_scoped_release>())
        .def_static("potential", [](const std::shared_ptr<ResourceList>&, const std::shared_ptr<Ewald>& ew,
                                    const std::shared_ptr<PairList>& pl, const std::shared_ptr<Tensor>& xyzc,
                                    const std::shared_ptr<Tensor>& V) { return OneInt::potential(ew, pl, xyzc, V); },
                    py::arg("resources"), py::arg("ewald"), py::arg("pairlist"), py::arg("xyzc"),
                    py::arg("V") = std::shared_ptr<Tensor>(), py::call_guard<py::gil_scoped_release>());

    m.attr("PREC_MIXED") = LSJK_PREC_MIXED;
    m.attr("PREC_FP64") = LSJK_PREC_FP64;
    m.def("set_precision", [](int mode) { Engine::instance().set_precision(mode); });
    m.def("set_merge", [](bool on) { Engine::instance().set_merge(on); },
          "K over merged twins of the bases (shared s exponents computed once) or, the default, over the "
          "primitives as given (the reference's exact quartet set); J always runs over the primitives as given");
    m.def("get_merge", []() { return Engine::instance().merge(); });
    m.def("get_precision", []() { return Engine::instance().precision(); });
    m.def("stats", &stats_dict);
    m.def("flops_split", []() {
        double f[4];
        check_rc(lsjk_context_flops_split(Engine::instance().ctx(), f), "flops_split");
        py::dict d;
        d["j_fp64"] = f[0];
        d["j_fp32"] = f[1];
        d["k_fp64"] = f[2];
        d["k_fp32"] = f[3];
        return d;
    }, "algorithmic flops since the last reset_stats, by J/K and precision");
    m.def("class_counts", []() {
        // quartets per class: {"fp64"|"fp32": {"J": {(LB,LK): n}, "K": {(L1,L2,L3,L4): n}}}
        constexpr int NH = 2 * LSJK_LMAX + 1, NL = LSJK_LMAX + 1, NJ = LSJK_NJCLASS, NK = LSJK_NKCLASS;
        std::vector<unsigned long long> h(2 * (NJ + NK));
        check_rc(lsjk_context_counters(Engine::instance().ctx(), h.data(), (int) h.size()), "class_counts");
        py::dict out;
        for (int prec = 0; prec < 2; ++prec) {
            py::dict j, k;
            const unsigned long long* b = h.data() + prec * (NJ + NK);
            for (int LB = 0; LB < NH; ++LB)
                for (int LK = 0; LK < NH; ++LK)
                    if (b[LB * NH + LK]) j[py::make_tuple(LB, LK)] = b[LB * NH + LK];
            for (int c = 0; c < NK; ++c)
                if (b[NJ + c])
                    k[py::make_tuple(c / (NL * NL * NL), (c / (NL * NL)) % NL, (c / NL) % NL, c % NL)] = b[NJ + c];
            py::dict d;
            d["J"] = j;
            d["K"] = k;
            out[prec ? "fp32" : "fp64"] = d;
        }
        return out;
    });
    m.def("reset_stats", []() { check_rc(lsjk_context_reset_stats(Engine::instance().ctx()), "reset_stats"); });
    m.def("engine_version", []() { return std::string(lsjk_version()); });
    // CUDA-graph capture of device-API builds (see include/lsjk.h)
    struct Graph {
        lsjk_graph* g = nullptr;
        ~Graph() { if (g) lsjk_graph_destroy(g); }
    };
    py::class_<Graph, std::shared_ptr<Graph>>(m, "Graph")
        .def("launch", [](Graph& g) { check_rc(lsjk_graph_launch(g.g), "graph launch"); },
             py::call_guard<py::gil_scoped_release>());
    m.def("graph_begin", []() { check_rc(lsjk_graph_begin(Engine::instance().ctx()), "graph_begin"); });
    m.def("graph_end", []() {
        auto g = std::make_shared<Graph>();
        check_rc(lsjk_graph_end(Engine::instance().ctx(), &g->g), "graph_end");
        return g;
    });
    m.def("set_autotune", [](bool on) { check_rc(lsjk_context_set_autotune(Engine::instance().ctx(), on ? 1 : 0),
                                                 "set_autotune"); });
    m.def("get_tune_table", []() {
        std::vector<int> t(LSJK_TUNE_INTS);
        check_rc(lsjk_context_tune_table(Engine::instance().ctx(), t.data(), (int) t.size(), 0), "tune table");
        return t;
    });
    m.def("set_tune_table", [](std::vector<int> t) {
        if (t.size() != LSJK_TUNE_INTS) throw std::runtime_error("tune table: wrong size");
        check_rc(lsjk_context_tune_table(Engine::instance().ctx(), t.data(), (int) t.size(), 1), "tune table");
    });
    m.def("stream_handle", []() { return (uintptr_t) lsjk_context_stream(Engine::instance().ctx()); },
          "cudaStream_t of the engine context, as an integer");
    m.def("fma_peak_tflops", [](bool fp64) {
        double t = 0.0;
        check_rc(lsjk_measure_fma_peak(Engine::instance().ctx(), fp64 ? 1 : 0, &t), "fma_peak");
        return t;
    }, py::arg("fp64") = true);
    // An additional engine context with its own CUDA stream, scratch and
    // counters, for running independent builds concurrently (e.g. the J/K of
    // different molecules): pair lists and bases are shared with the main
    // context; calls on one Stream are ordered, different Streams overlap.
    struct ExtraContext {
        lsjk_context* c = nullptr;
        explicit ExtraContext(int device)
        {
            check_rc(lsjk_context_create(device, &c), "Stream");
            check_rc(lsjk_context_set_precision(c, Engine::instance().precision()), "Stream");
            check_rc(lsjk_context_set_merge(c, Engine::instance().merge() ? 1 : 0), "Stream");
        }
        ~ExtraContext() { if (c) lsjk_context_destroy(c); }
    };
    py::class_<ExtraContext, std::shared_ptr<ExtraContext>>(m, "Stream")
        .def(py::init([]() { return std::make_shared<ExtraContext>(Engine::instance().device()); }))
        .def("set_precision", [](ExtraContext& x, int mode) { check_rc(lsjk_context_set_precision(x.c, mode),
                                                                       "Stream.set_precision"); })
        .def("set_merge", [](ExtraContext& x, bool on) { check_rc(lsjk_context_set_merge(x.c, on ? 1 : 0),
                                                                   "Stream.set_merge"); })
        .def("stream_handle", [](ExtraContext& x) { return (uintptr_t) lsjk_context_stream(x.c); })
        .def("stats", [](ExtraContext& x) { return stats_dict_of(x.c); })
        .def("reset_stats", [](ExtraContext& x) { check_rc(lsjk_context_reset_stats(x.c), "Stream.reset_stats"); })
        .def("coulomb_device", [](ExtraContext& x, const std::shared_ptr<Ewald>& ew,
                                  const std::shared_ptr<PairList>& pl12, const std::shared_ptr<PairList>& pl34,
                                  const std::vector<uintptr_t>& D, const std::vector<uintptr_t>& J, float thresp,
                                  float thredp) {
            if (D.size() != J.size()) throw std::runtime_error("coulomb_device: D/J count mismatch");
            std::vector<const double*> dp;
            std::vector<double*> jp;
            for (size_t k = 0; k < D.size(); ++k) {
                dp.push_back(reinterpret_cast<const double*>(D[k]));
                jp.push_back(reinterpret_cast<double*>(J[k]));
            }
            check_rc(lsjk_coulomb_device(x.c, (int) ew->scales().size(), ew->scales().data(), ew->omegas().data(),
                                         pl12->device_handle(), pl34->device_handle(), (int) dp.size(), dp.data(),
                                         thresp, thredp, jp.data()),
                     "Stream.coulomb_device");
        }, py::call_guard<py::gil_scoped_release>())
        .def("exchange_device", [](ExtraContext& x, const std::shared_ptr<Ewald>& ew,
                                   const std::shared_ptr<PairList>& pl12, const std::shared_ptr<PairList>& pl34,
                                   const std::vector<uintptr_t>& D, bool D24symm, const std::vector<uintptr_t>& K,
                                   float thresp, float thredp) {
            if (D.size() != K.size()) throw std::runtime_error("exchange_device: D/K count mismatch");
            std::vector<const double*> dp;
            std::vector<double*> kp;
            for (size_t k = 0; k < D.size(); ++k) {
                dp.push_back(reinterpret_cast<const double*>(D[k]));
                kp.push_back(reinterpret_cast<double*>(K[k]));
            }
            check_rc(lsjk_exchange_device(x.c, (int) ew->scales().size(), ew->scales().data(), ew->omegas().data(),
                                          pl12->device_handle(), pl34->device_handle(), (int) dp.size(), dp.data(),
                                          D24symm ? 1 : 0, thresp, thredp, kp.data()),
                     "Stream.exchange_device");
        }, py::call_guard<py::gil_scoped_release>());
    // Device-resident J/K: D and J/K are device addresses (e.g. torch
    // tensor.data_ptr()); the work is enqueued on the engine stream only.
    m.def("coulomb_device", [](const std::shared_ptr<Ewald>& ew, const std::shared_ptr<PairList>& pl12,
                               const std::shared_ptr<PairList>& pl34, const std::vector<uintptr_t>& D,
                               const std::vector<uintptr_t>& J, float thresp, float thredp) {
        if (D.size() != J.size()) throw std::runtime_error("coulomb_device: D/J count mismatch");
        std::vector<const double*> dp;
        std::vector<double*> jp;
        for (size_t k = 0; k < D.size(); ++k) {
            dp.push_back(reinterpret_cast<const double*>(D[k]));
            jp.push_back(reinterpret_cast<double*>(J[k]));
        }
        check_rc(lsjk_coulomb_device(Engine::instance().ctx(), (int) ew->scales().size(), ew->scales().data(),
                                     ew->omegas().data(), pl12->device_handle(), pl34->device_handle(),
                                     (int) dp.size(), dp.data(), thresp, thredp, jp.data()),
                 "coulomb_device");
    }, py::call_guard<py::gil_scoped_release>());
    m.def("exchange_device", [](const std::shared_ptr<Ewald>& ew, const std::shared_ptr<PairList>& pl12,
                                const std::shared_ptr<PairList>& pl34, const std::vector<uintptr_t>& D,
                                bool D24symm, const std::vector<uintptr_t>& K, float thresp, float thredp) {
        if (D.size() != K.size()) throw std::runtime_error("exchange_device: D/K count mismatch");
        std::vector<const double*> dp;
        std::vector<double*> kp;
        for (size_t k = 0; k < D.size(); ++k) {
            dp.push_back(reinterpret_cast<const double*>(D[k]));
            kp.push_back(reinterpret_cast<double*>(K[k]));
        }
        check_rc(lsjk_exchange_device(Engine::instance().ctx(), (int) ew->scales().size(), ew->scales().data(),
                                      ew->omegas().data(), pl12->device_handle(), pl34->device_handle(),
                                      (int) dp.size(), dp.data(), D24symm ? 1 : 0, thresp, thredp, kp.data()),
                 "exchange_device");
    }, py::call_guard<py::gil_scoped_release>());
}
