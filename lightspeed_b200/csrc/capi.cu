// extern "C" entry points of liblsjk.so (declared in include/lsjk.h).
#include <algorithm>
#include <cstring>
#include <dlfcn.h>
#include <memory>
#include <mutex>
#include <string>
#include <vector>
#include "engine.cuh"
#include "lsjk_device.cuh"

// Page-locked host staging for the host-pointer entry points (grow-only).
struct PinnedBuf {
    double* p = nullptr;
    size_t n = 0;
    PinnedBuf() = default;
    PinnedBuf(const PinnedBuf&) = delete;
    PinnedBuf& operator=(const PinnedBuf&) = delete;
    ~PinnedBuf() { if (p) cudaFreeHost(p); }
    double* ensure(size_t count)
    {
        if (count > n) {
            if (p) cudaFreeHost(p);
            p = nullptr;
            n = 0;
            LSJK_CUDA(cudaMallocHost((void**) &p, sizeof(double) * count));
            n = count;
        }
        return p;
    }
};

// The context plus the device and pinned host buffers the host-pointer entry
// points (lsjk_coulomb, lsjk_exchange) stage D and J/K through; both grow to
// the largest call and are reused, so repeated calls allocate nothing.
struct lsjk_context {
    lsjk::Context c;
    lsjk::DBuf<double> io_dev;
    PinnedBuf io_host;
    double* dev(size_t count)
    {
        if (count > io_dev.n) io_dev.alloc(count);
        return io_dev.p;
    }
};
struct lsjk_basis { lsjk::Basis b; };
struct lsjk_pairlist { lsjk::PairList p; };
struct lsjk_graph {
    lsjk::Context* ctx = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace lsjk {
void basis_init(Context* ctx, Basis* B);
std::vector<std::vector<double>> solid_harmonics(int L);
}

namespace {

thread_local std::string g_err;

template <typename F>
int guard(F&& f)
{
    try {
        f();
        g_err.clear();
        return LSJK_OK;
    } catch (const lsjk::Error& e) {
        g_err = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_err = e.what();
        return LSJK_EINVAL;
    }
}

void set_device(const lsjk::Context& c) { LSJK_CUDA(cudaSetDevice(c.device)); }

lsjk::Ewald make_ewald(int nterm, const double* scales, const double* omegas)
{
    if (nterm < 1 || !scales || !omegas) throw lsjk::Error(LSJK_EINVAL, "Ewald: need >= 1 term");
    lsjk::Ewald ew;
    for (int t = 0; t < nterm; ++t) {
        // terms with zero scale or zero omega contribute nothing (coulomb.cpp:72-73)
        if (scales[t] == 0.0 || omegas[t] == 0.0) continue;
        ew.alpha.push_back(scales[t]);
        ew.omega.push_back(omegas[t]);
    }
    if (ew.alpha.size() > 4) throw lsjk::Error(LSJK_EINVAL, "Ewald: at most 4 nonzero terms are supported");
    return ew;
}

void check_kernels(lsjk::Context* ctx)
{
    int st = 0;
    LSJK_CUDA(cudaMemcpyAsync(&st, ctx->status.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    LSJK_CUDA(cudaStreamSynchronize(ctx->stream));
    if (st) {
        LSJK_CUDA(cudaMemsetAsync(ctx->status.p, 0, sizeof(int), ctx->stream));
        throw lsjk::Error(LSJK_EKERNEL, "a J/K kernel reported error status " + std::to_string(st));
    }
}

void check_lmax(const lsjk::PairList* pl)
{
    if (pl->b1->maxL > lsjk::kLmax || pl->b2->maxL > lsjk::kLmax)
        throw lsjk::Error(LSJK_ENOTSUPP, "J/K: angular momentum above f is not supported by the GPU kernels");
}

// The pair list a K build runs over: its merged twin (shared s exponents of a
// basis computed once) unless the context builds over the primitives as given.
// J builds always run over the primitives as given: merging their screens
// moves J by up to ~1e-10 on the largest workload, while merged K stays within
// ~2e-11 of the reference's quartet set.
const lsjk::PairList* effective(const lsjk::Context* ctx, const lsjk::PairList* pl)
{
    return (ctx->merge && pl->twin) ? pl->twin.get() : pl;
}

// Screening densities for a K build over twins (u3 x u4, standing for the
// caller's bases o3 x o4): the density in the caller's Cartesian layout,
// then per twin slot the largest weighted |D| of its copies. Null when
// neither side is a twin (the screens then read the density itself).
void screening_densities(lsjk::Context* ctx, const lsjk::Basis* o3, const lsjk::Basis* o4, const lsjk::Basis* u3,
                         const lsjk::Basis* u4, const double* const* Dpure, int ng, double** Dscr)
{
    for (int g = 0; g < ng; ++g) Dscr[g] = nullptr;
    if (u3 == o3 && u4 == o4) return;
    double* Dorig = lsjk::take<double>(ctx, (size_t) o3->ncart * o4->ncart);
    for (int g = 0; g < ng; ++g) {
        Dscr[g] = lsjk::take<double>(ctx, (size_t) u3->ncart * u4->ncart);
        lsjk::pure_to_cart(ctx, o3, o4, Dpure[g], Dorig);
        lsjk::screen_density(ctx, u3, u4, Dorig, o4->ncart, Dscr[g]);
    }
}

// One J build for ng (1..kMaxDens) densities (one launch per class for all of
// them), device pointers in and out.
void coulomb_group(lsjk::Context* ctx, const lsjk::Ewald& ew, const lsjk::PairList* pl12,
                   const lsjk::PairList* pl34, const double* const* Dpure, double* const* Jpure, int ng,
                   float thresp, float thredp)
{
    ctx->scratch_reset();
    const lsjk::Basis *b1 = pl12->b1, *b2 = pl12->b2, *b3 = pl34->b1, *b4 = pl34->b2;
    double* Dc[lsjk::kMaxDens];
    double* Jc[lsjk::kMaxDens];
    for (int g = 0; g < ng; ++g) {
        Dc[g] = lsjk::take<double>(ctx, (size_t) b3->ncart * b4->ncart);
        Jc[g] = lsjk::take<double>(ctx, (size_t) b1->ncart * b2->ncart);
        lsjk::pure_to_cart(ctx, b3, b4, Dpure[g], Dc[g]);
        LSJK_CUDA(cudaMemsetAsync(Jc[g], 0, sizeof(double) * b1->ncart * b2->ncart, ctx->stream));
    }
    if (!ew.alpha.empty() && pl12->npair && pl34->npair)
        lsjk::coulomb_build(ctx, ew, pl12, pl34, Dc, Jc, ng, thresp, thredp);
    for (int g = 0; g < ng; ++g) lsjk::cart_to_pure_acc(ctx, b1, b2, Jc[g], Jpure[g]);
}

// One K build for ng (1..kMaxDens) densities (groups of four share task lists
// and quartet integrals; one launch per class and pass), device pointers in
// and out. Over twins D24 lives in the twins' slots of bases 2
// and 4, while K13 is accumulated straight into the Cartesian spaces of the
// caller's bases 1 and 3 (each partner primitive carries its output targets).
void exchange_group(lsjk::Context* ctx, const lsjk::Ewald& ew, const lsjk::PairList* pl12_in,
                    const lsjk::PairList* pl34_in, const double* const* Dpure, bool d24symm, bool flip_ok,
                    double* const* Kpure, int ng, float thresp, float thredp)
{
    const lsjk::PairList* pl12 = effective(ctx, pl12_in);
    const lsjk::PairList* pl34 = effective(ctx, pl34_in);
    ctx->scratch_reset();
    const lsjk::Basis *b1 = pl12_in->b1, *b2 = pl12->b2, *b3 = pl34_in->b1, *b4 = pl34->b2;
    double* Dc[lsjk::kMaxDens];
    double* Kc[lsjk::kMaxDens];
    for (int g = 0; g < ng; ++g) {
        Dc[g] = lsjk::take<double>(ctx, (size_t) b2->ncart * b4->ncart);
        Kc[g] = lsjk::take<double>(ctx, (size_t) b1->ncart * b3->ncart);
        lsjk::pure_to_cart(ctx, b2, b4, Dpure[g], Dc[g]);
        LSJK_CUDA(cudaMemsetAsync(Kc[g], 0, sizeof(double) * b1->ncart * b3->ncart, ctx->stream));
    }
    double* Ds[lsjk::kMaxDens];
    screening_densities(ctx, pl12_in->b2, pl34_in->b2, b2, b4, Dpure, ng, Ds);
    if (!ew.alpha.empty() && pl12->npair && pl34->npair)
        lsjk::exchange_build(ctx, ew, pl12, pl34, Dc, Ds[0] ? Ds : nullptr, Kc, ng, d24symm, flip_ok, thresp,
                             thredp, b1, b3);
    for (int g = 0; g < ng; ++g) lsjk::cart_to_pure_acc(ctx, b1, b3, Kc[g], Kpure[g]);
}

void exchange_prepare(lsjk::Context* ctx, lsjk::PairList* pl12, lsjk::PairList* pl34, int D24symm,
                      bool* d24, bool* flip)
{
    check_lmax(pl12);
    check_lmax(pl34);
    bool symm = D24symm != 0;
    if (symm && !pl12->b2->equivalent(*pl34->b2))
        throw lsjk::Error(LSJK_EINVAL,
                          "IntBox::exchange: D24symm implied, but basis sets 2 and 4 not the same");
    *d24 = symm;
    // the transposed write needs basis 1 == basis 3 as well (exchange.cpp:79-81)
    *flip = symm && pl12->b1->equivalent(*pl34->b1);
    *d24 = *flip;
    lsjk::PairList* e12 = const_cast<lsjk::PairList*>(effective(ctx, pl12));
    lsjk::PairList* e34 = const_cast<lsjk::PairList*>(effective(ctx, pl34));
    lsjk::build_kinv(ctx, e12);
    if (e34 != e12) lsjk::build_kinv(ctx, e34);
}

// FMA throughput probe: 8 independent dependency chains per thread so the
// pipe, not latency, limits; every thread does 16 * iters flops.
template <typename R>
__global__ void k_fma_peak(R* out, int iters, R m, R c)
{
    R a0 = R(threadIdx.x) * R(1e-3), a1 = a0 + R(1), a2 = a0 + R(2), a3 = a0 + R(3);
    R a4 = a0 + R(4), a5 = a0 + R(5), a6 = a0 + R(6), a7 = a0 + R(7);
    for (int i = 0; i < iters; ++i) {
        a0 = fma(a0, m, c); a1 = fma(a1, m, c); a2 = fma(a2, m, c); a3 = fma(a3, m, c);
        a4 = fma(a4, m, c); a5 = fma(a5, m, c); a6 = fma(a6, m, c); a7 = fma(a7, m, c);
    }
    R s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == R(-12345.678)) out[threadIdx.x] = s;   // keeps the chains alive
}

} // namespace

extern "C" {

int lsjk_measure_fma_peak(lsjk_context* ctx, int fp64, double* tflops)
{
    return guard([&] {
        if (!ctx || !tflops) throw lsjk::Error(LSJK_EINVAL, "null argument");
        lsjk::Context& c = ctx->c;
        set_device(c);
        int nsm = 0;
        LSJK_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c.device));
        const int threads = 256, blocks = nsm * 8, iters = 1 << 14;
        lsjk::DBuf<double> out;
        out.alloc(threads);
        float best = 1e30f;
        for (int rep = 0; rep < 5; ++rep) {
            LSJK_CUDA(cudaEventRecord(c.ev0, c.stream));
            if (fp64)
                k_fma_peak<double><<<blocks, threads, 0, c.stream>>>(out.p, iters, 0.999999, 1e-7);
            else
                k_fma_peak<float><<<blocks, threads, 0, c.stream>>>((float*) out.p, iters, 0.999999f, 1e-7f);
            LSJK_CUDA(cudaGetLastError());
            LSJK_CUDA(cudaEventRecord(c.ev1, c.stream));
            LSJK_CUDA(cudaEventSynchronize(c.ev1));
            float ms = 0.f;
            LSJK_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
            if (rep > 0) best = std::min(best, ms);
        }
        double flops = 16.0 * iters * (double) threads * blocks;
        *tflops = flops / (best * 1e-3) / 1e12;
    });
}

const char* lsjk_last_error(void) { return g_err.c_str(); }

long lsjk_device_allocations(void) { return lsjk::g_device_allocations.load(std::memory_order_relaxed); }

const char* lsjk_version(void) { return "lsjk 0.1 (sm_100a)"; }

int lsjk_context_create(int device, lsjk_context** out)
{
    return guard([&] {
        if (!out) throw lsjk::Error(LSJK_EINVAL, "null output");
        auto* h = new lsjk_context();
        lsjk::Context& c = h->c;
        try {
            c.device = device;
            LSJK_CUDA(cudaSetDevice(device));
            LSJK_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
            LSJK_CUDA(cudaDeviceGetAttribute(&c.nsm, cudaDevAttrMultiProcessorCount, device));
            std::vector<double> boys(kBoysCoef, kBoysCoef + sizeof(kBoysCoef) / sizeof(double));
            std::vector<double> rys(kRysCoef, kRysCoef + sizeof(kRysCoef) / sizeof(double));
            std::vector<double> asym(kRysAsymT, kRysAsymT + sizeof(kRysAsymT) / sizeof(double));
            asym.insert(asym.end(), kRysAsymW, kRysAsymW + sizeof(kRysAsymW) / sizeof(double));
            c.boys64.upload(boys, c.stream);
            c.rys64.upload(rys, c.stream);
            c.rys_asym64.upload(asym, c.stream);
            c.boys32.upload(std::vector<float>(boys.begin(), boys.end()), c.stream);
            c.rys32.upload(std::vector<float>(rys.begin(), rys.end()), c.stream);
            c.rys_asym32.upload(std::vector<float>(asym.begin(), asym.end()), c.stream);
            c.status.alloc(1);
            LSJK_CUDA(cudaMemsetAsync(c.status.p, 0, sizeof(int), c.stream));
            c.counters.alloc(lsjk::kNCounters);
            c.tune_sink.alloc(lsjk::kNCounters);
            LSJK_CUDA(cudaMemsetAsync(c.counters.p, 0, sizeof(unsigned long long) * lsjk::kNCounters, c.stream));
            LSJK_CUDA(cudaEventCreate(&c.ev0));
            LSJK_CUDA(cudaEventCreate(&c.ev1));
            LSJK_CUDA(cudaEventCreate(&c.ev2));
            for (int i = 0; i < lsjk::Context::kAux; ++i) {
                LSJK_CUDA(cudaStreamCreateWithFlags(&c.aux[i], cudaStreamNonBlocking));
                LSJK_CUDA(cudaEventCreateWithFlags(&c.join_ev[i], cudaEventDisableTiming));
            }
            LSJK_CUDA(cudaEventCreateWithFlags(&c.fork_ev, cudaEventDisableTiming));
            LSJK_CUDA(cudaStreamSynchronize(c.stream));
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int lsjk_context_destroy(lsjk_context* ctx)
{
    return guard([&] {
        if (!ctx) return;
        cudaSetDevice(ctx->c.device);
        cudaStreamSynchronize(ctx->c.stream);
        if (ctx->c.ev0) cudaEventDestroy(ctx->c.ev0);
        if (ctx->c.ev1) cudaEventDestroy(ctx->c.ev1);
        if (ctx->c.ev2) cudaEventDestroy(ctx->c.ev2);
        for (int i = 0; i < lsjk::Context::kAux; ++i) {
            if (ctx->c.aux[i]) {
                cudaStreamSynchronize(ctx->c.aux[i]);
                cudaStreamDestroy(ctx->c.aux[i]);
            }
            if (ctx->c.join_ev[i]) cudaEventDestroy(ctx->c.join_ev[i]);
        }
        if (ctx->c.fork_ev) cudaEventDestroy(ctx->c.fork_ev);
        cudaStream_t s = ctx->c.stream;
        delete ctx;
        if (s) cudaStreamDestroy(s);
    });
}

int lsjk_context_set_merge(lsjk_context* ctx, int on)
{
    return guard([&] {
        if (!ctx) throw lsjk::Error(LSJK_EINVAL, "null context");
        ctx->c.merge = on != 0;
    });
}

int lsjk_context_set_precision(lsjk_context* ctx, int mode)
{
    return guard([&] {
        if (!ctx || (mode != LSJK_PREC_MIXED && mode != LSJK_PREC_FP64))
            throw lsjk::Error(LSJK_EINVAL, "bad precision mode");
        ctx->c.precision = mode;
    });
}

void* lsjk_context_stream(lsjk_context* ctx) { return ctx ? (void*) ctx->c.stream : nullptr; }

int lsjk_context_stats(lsjk_context* ctx, lsjk_stats* out)
{
    return guard([&] {
        if (!ctx || !out) throw lsjk::Error(LSJK_EINVAL, "null argument");
        lsjk::Context& c = ctx->c;
        set_device(c);
        std::vector<unsigned long long> h(lsjk::kNCounters);
        LSJK_CUDA(cudaMemcpyAsync(h.data(), c.counters.p, sizeof(unsigned long long) * h.size(),
                                  cudaMemcpyDeviceToHost, c.stream));
        LSJK_CUDA(cudaStreamSynchronize(c.stream));
        lsjk_stats st = c.stats;
        st.quartets_fp64 = st.quartets_fp32 = st.j_quartets = st.k_quartets = st.flops_j = st.flops_k = 0.0;
        for (int prec = 0; prec < 2; ++prec) {
            const unsigned long long* b = h.data() + prec * (lsjk::kNJClass + lsjk::kNKClass);
            for (int LB = 0; LB < lsjk::kNHerm; ++LB)
                for (int LK = 0; LK < lsjk::kNHerm; ++LK) {
                    double n = (double) b[LB * lsjk::kNHerm + LK];
                    st.j_quartets += n;
                    (prec ? st.quartets_fp32 : st.quartets_fp64) += n;
                    st.flops_j += n * lsjk::j_quartet_flops(LB, LK);
                }
            for (int L1 = 0; L1 < lsjk::kNL; ++L1)
                for (int L2 = 0; L2 < lsjk::kNL; ++L2)
                    for (int L3 = 0; L3 < lsjk::kNL; ++L3)
                        for (int L4 = 0; L4 < lsjk::kNL; ++L4) {
                            int ci = ((L1 * lsjk::kNL + L2) * lsjk::kNL + L3) * lsjk::kNL + L4;
                            double n = (double) b[lsjk::kNJClass + ci];
                            st.k_quartets += n;
                            (prec ? st.quartets_fp32 : st.quartets_fp64) += n;
                            st.flops_k += n * lsjk::k_quartet_flops(L1, L2, L3, L4);
                        }
        }
        *out = st;
    });
}

int lsjk_context_flops_split(lsjk_context* ctx, double* out4)
{
    return guard([&] {
        if (!ctx || !out4) throw lsjk::Error(LSJK_EINVAL, "null argument");
        lsjk::Context& c = ctx->c;
        set_device(c);
        std::vector<unsigned long long> h(lsjk::kNCounters);
        LSJK_CUDA(cudaMemcpyAsync(h.data(), c.counters.p, sizeof(unsigned long long) * h.size(),
                                  cudaMemcpyDeviceToHost, c.stream));
        LSJK_CUDA(cudaStreamSynchronize(c.stream));
        for (int k = 0; k < 4; ++k) out4[k] = 0.0;
        for (int prec = 0; prec < 2; ++prec) {
            const unsigned long long* b = h.data() + prec * (lsjk::kNJClass + lsjk::kNKClass);
            for (int LB = 0; LB < lsjk::kNHerm; ++LB)
                for (int LK = 0; LK < lsjk::kNHerm; ++LK)
                    out4[prec] += (double) b[LB * lsjk::kNHerm + LK] * lsjk::j_quartet_flops(LB, LK);
            for (int L1 = 0; L1 < lsjk::kNL; ++L1)
                for (int L2 = 0; L2 < lsjk::kNL; ++L2)
                    for (int L3 = 0; L3 < lsjk::kNL; ++L3)
                        for (int L4 = 0; L4 < lsjk::kNL; ++L4) {
                            int ci = ((L1 * lsjk::kNL + L2) * lsjk::kNL + L3) * lsjk::kNL + L4;
                            out4[2 + prec] += (double) b[lsjk::kNJClass + ci] * lsjk::k_quartet_flops(L1, L2, L3, L4);
                        }
        }
    });
}

int lsjk_context_counters(lsjk_context* ctx, unsigned long long* out, int n)
{
    return guard([&] {
        if (!ctx || !out || n < lsjk::kNCounters) throw lsjk::Error(LSJK_EINVAL, "bad counters buffer");
        set_device(ctx->c);
        LSJK_CUDA(cudaMemcpyAsync(out, ctx->c.counters.p, sizeof(unsigned long long) * lsjk::kNCounters,
                                  cudaMemcpyDeviceToHost, ctx->c.stream));
        LSJK_CUDA(cudaStreamSynchronize(ctx->c.stream));
    });
}

int lsjk_context_set_autotune(lsjk_context* ctx, int on)
{
    return guard([&] {
        if (!ctx) throw lsjk::Error(LSJK_EINVAL, "null context");
        ctx->c.tuning = on != 0;
    });
}

int lsjk_context_tune_table(lsjk_context* ctx, int* table, int n, int set)
{
    return guard([&] {
        if (!ctx || !table || n < lsjk::kTuneInts) throw lsjk::Error(LSJK_EINVAL, "bad tune table");
        int* t = reinterpret_cast<int*>(&ctx->c.tune);
        static_assert(sizeof(lsjk::Tune) == sizeof(int) * lsjk::kTuneInts, "Tune layout");
        if (set)
            std::copy(table, table + lsjk::kTuneInts, t);
        else
            std::copy(t, t + lsjk::kTuneInts, table);
    });
}

int lsjk_context_reset_stats(lsjk_context* ctx)
{
    return guard([&] {
        if (!ctx) throw lsjk::Error(LSJK_EINVAL, "null argument");
        set_device(ctx->c);
        LSJK_CUDA(cudaMemsetAsync(ctx->c.counters.p, 0, sizeof(unsigned long long) * lsjk::kNCounters,
                                  ctx->c.stream));
        LSJK_CUDA(cudaStreamSynchronize(ctx->c.stream));
        ctx->c.stats = lsjk_stats{};
    });
}

int lsjk_context_status(lsjk_context* ctx, int* status)
{
    return guard([&] {
        if (!ctx || !status) throw lsjk::Error(LSJK_EINVAL, "null argument");
        set_device(ctx->c);
        LSJK_CUDA(cudaMemcpyAsync(status, ctx->c.status.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->c.stream));
        LSJK_CUDA(cudaStreamSynchronize(ctx->c.stream));
    });
}

int lsjk_basis_create(lsjk_context* ctx, int nprim, const double* c, const double* e, const double* xyz,
                      const int* L, const int* is_pure, const int* aoIdx, const int* cartIdx,
                      const int* primIdx, const int* shellIdx, const int* atomIdx, lsjk_basis** out)
{
    return guard([&] {
        if (!ctx || !out || nprim < 0) throw lsjk::Error(LSJK_EINVAL, "bad basis arguments");
        if (nprim > 0 && (!c || !e || !xyz || !L || !is_pure || !aoIdx || !cartIdx || !primIdx ||
                          !shellIdx || !atomIdx))
            throw lsjk::Error(LSJK_EINVAL, "null basis array");
        set_device(ctx->c);
        auto* h = new lsjk_basis();
        lsjk::Basis& B = h->b;
        B.ctx = &ctx->c;
        B.nprim = nprim;
        B.c.assign(c, c + nprim);
        B.e.assign(e, e + nprim);
        for (int i = 0; i < nprim; ++i) {
            B.x.push_back(xyz[3 * i]);
            B.y.push_back(xyz[3 * i + 1]);
            B.z.push_back(xyz[3 * i + 2]);
        }
        B.L.assign(L, L + nprim);
        B.pure.assign(is_pure, is_pure + nprim);
        B.ao.assign(aoIdx, aoIdx + nprim);
        B.cart.assign(cartIdx, cartIdx + nprim);
        B.prim.assign(primIdx, primIdx + nprim);
        B.shell.assign(shellIdx, shellIdx + nprim);
        B.atom.assign(atomIdx, atomIdx + nprim);
        try {
            lsjk::basis_init(&ctx->c, &B);
            lsjk::basis_build_twin(&ctx->c, &B);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int lsjk_basis_destroy(lsjk_basis* basis)
{
    return guard([&] { delete basis; });
}

int lsjk_basis_nao(const lsjk_basis* basis) { return basis ? basis->b.nao : -1; }

int lsjk_solid_harmonics(int L, double* coef)
{
    return guard([&] {
        if (L < 0 || L > 6 || !coef) throw lsjk::Error(LSJK_EINVAL, "solid_harmonics: L must be 0..6");
        auto C = lsjk::solid_harmonics(L);
        int nc = (L + 1) * (L + 2) / 2;
        for (int p = 0; p < 2 * L + 1; ++p)
            for (int k = 0; k < nc; ++k) coef[p * nc + k] = C[p][k];
    });
}
int lsjk_basis_ncart(const lsjk_basis* basis) { return basis ? basis->b.ncart : -1; }

int lsjk_pairlist_build_schwarz(lsjk_context* ctx, const lsjk_basis* basis1, const lsjk_basis* basis2,
                                int is_symmetric, float thre, lsjk_pairlist** out)
{
    return guard([&] {
        if (!ctx || !basis1 || !basis2 || !out) throw lsjk::Error(LSJK_EINVAL, "null argument");
        set_device(ctx->c);
        auto* h = new lsjk_pairlist();
        lsjk::PairList& P = h->p;
        P.ctx = &ctx->c;
        P.b1 = &basis1->b;
        P.b2 = &basis2->b;
        P.symm = is_symmetric != 0;
        P.thre = thre;
        try {
            lsjk::build_pairlist(&ctx->c, &P);
            // the same list over the merged twins, for builds in merge mode
            if (P.b1->twin || P.b2->twin) {
                P.twin.reset(new lsjk::PairList());
                lsjk::PairList& T = *P.twin;
                T.ctx = &ctx->c;
                T.b1 = P.b1->twin ? P.b1->twin.get() : P.b1;
                T.b2 = P.b2->twin ? P.b2->twin.get() : P.b2;
                T.symm = P.symm;
                T.thre = P.thre;
                lsjk::build_pairlist(&ctx->c, &T);
            }
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int lsjk_pairlist_destroy(lsjk_pairlist* pl)
{
    return guard([&] { delete pl; });
}

long lsjk_pairlist_size(const lsjk_pairlist* pl) { return pl ? pl->p.npair : -1; }

int lsjk_pairlist_export(const lsjk_pairlist* pl, int* L1, int* L2, int* prim1, int* prim2, float* bound)
{
    return guard([&] {
        if (!pl) throw lsjk::Error(LSJK_EINVAL, "null pair list");
        const lsjk::PairList& P = pl->p;
        long n = P.npair;
        if (!n) return;
        lsjk::Context* ctx = P.ctx;
        set_device(*ctx);
        if (prim1) LSJK_CUDA(cudaMemcpyAsync(prim1, P.p1.p, sizeof(int) * n, cudaMemcpyDeviceToHost, ctx->stream));
        if (prim2) LSJK_CUDA(cudaMemcpyAsync(prim2, P.p2.p, sizeof(int) * n, cudaMemcpyDeviceToHost, ctx->stream));
        if (bound) LSJK_CUDA(cudaMemcpyAsync(bound, P.bound.p, sizeof(float) * n, cudaMemcpyDeviceToHost, ctx->stream));
        LSJK_CUDA(cudaStreamSynchronize(ctx->stream));
        for (size_t c = 0; c + 1 < P.cls_off.size(); ++c)
            for (long k = P.cls_off[c]; k < P.cls_off[c + 1]; ++k) {
                if (L1) L1[k] = P.cls_L1[c];
                if (L2) L2[k] = P.cls_L2[c];
            }
    });
}

int lsjk_coulomb_device(lsjk_context* ctx, int nterm, const double* scales, const double* omegas,
                        const lsjk_pairlist* pl12, const lsjk_pairlist* pl34, int ndens,
                        const double* const* D34, float thresp, float thredp, double* const* J12)
{
    return guard([&] {
        if (!ctx || !pl12 || !pl34 || ndens < 0 || (ndens && (!D34 || !J12)))
            throw lsjk::Error(LSJK_EINVAL, "null argument");
        set_device(ctx->c);
        lsjk::Ewald ew = make_ewald(nterm, scales, omegas);
        check_lmax(&pl12->p);
        check_lmax(&pl34->p);
        for (int k0 = 0; k0 < ndens; k0 += lsjk::kMaxDens)
            coulomb_group(&ctx->c, ew, &pl12->p, &pl34->p, D34 + k0, J12 + k0,
                          std::min(lsjk::kMaxDens, ndens - k0), thresp, thredp);
    });
}

int lsjk_exchange_device(lsjk_context* ctx, int nterm, const double* scales, const double* omegas,
                         const lsjk_pairlist* pl12, const lsjk_pairlist* pl34, int ndens,
                         const double* const* D24, int D24symm, float thresp, float thredp,
                         double* const* K13)
{
    return guard([&] {
        if (!ctx || !pl12 || !pl34 || ndens < 0 || (ndens && (!D24 || !K13)))
            throw lsjk::Error(LSJK_EINVAL, "null argument");
        set_device(ctx->c);
        lsjk::Ewald ew = make_ewald(nterm, scales, omegas);
        bool d24 = false, flip = false;
        exchange_prepare(&ctx->c, const_cast<lsjk::PairList*>(&pl12->p), const_cast<lsjk::PairList*>(&pl34->p),
                         D24symm, &d24, &flip);
        for (int k0 = 0; k0 < ndens; k0 += lsjk::kMaxDens)
            exchange_group(&ctx->c, ew, &pl12->p, &pl34->p, D24 + k0, d24, flip, K13 + k0,
                           std::min(lsjk::kMaxDens, ndens - k0), thresp, thredp);
    });
}

int lsjk_coulomb(lsjk_context* ctx, int nterm, const double* scales, const double* omegas,
                 const lsjk_pairlist* pl12, const lsjk_pairlist* pl34, int ndens,
                 const double* const* D34, float thresp, float thredp, double* const* J12)
{
    return guard([&] {
        if (!ctx || !pl12 || !pl34 || ndens < 0 || (ndens && (!D34 || !J12)))
            throw lsjk::Error(LSJK_EINVAL, "null argument");
        lsjk::Context* c = &ctx->c;
        set_device(*c);
        lsjk::Ewald ew = make_ewald(nterm, scales, omegas);
        check_lmax(&pl12->p);
        check_lmax(&pl34->p);
        const size_t nD = (size_t) pl34->p.b1->nao * pl34->p.b2->nao;
        const size_t nJ = (size_t) pl12->p.b1->nao * pl12->p.b2->nao;
        const int G = std::max(1, std::min(lsjk::kMaxDens, ndens));
        double* dD = ctx->dev((nD + nJ) * G);
        double* dJ = dD + nD * G;
        double* hD = ctx->io_host.ensure((nD + nJ) * G);
        double* hJ = hD + nD * G;
        for (int k0 = 0; k0 < ndens; k0 += G) {
            const int ng = std::min(G, ndens - k0);
            const double* dp[lsjk::kMaxDens];
            double* jp[lsjk::kMaxDens];
            for (int g = 0; g < ng; ++g) {
                dp[g] = dD + g * nD;
                jp[g] = dJ + g * nJ;
                if (nD) std::memcpy(hD + g * nD, D34[k0 + g], sizeof(double) * nD);
            }
            if (nD) LSJK_CUDA(cudaMemcpyAsync(dD, hD, sizeof(double) * nD * ng, cudaMemcpyHostToDevice, c->stream));
            if (nJ) LSJK_CUDA(cudaMemsetAsync(dJ, 0, sizeof(double) * nJ * ng, c->stream));
            coulomb_group(c, ew, &pl12->p, &pl34->p, dp, jp, ng, thresp, thredp);
            if (nJ) LSJK_CUDA(cudaMemcpyAsync(hJ, dJ, sizeof(double) * nJ * ng, cudaMemcpyDeviceToHost, c->stream));
            check_kernels(c);
            for (int g = 0; g < ng; ++g)
                for (size_t i = 0; i < nJ; ++i) J12[k0 + g][i] += hJ[g * nJ + i];
        }
    });
}

int lsjk_exchange(lsjk_context* ctx, int nterm, const double* scales, const double* omegas,
                  const lsjk_pairlist* pl12, const lsjk_pairlist* pl34, int ndens,
                  const double* const* D24, int D24symm, float thresp, float thredp, double* const* K13)
{
    return guard([&] {
        if (!ctx || !pl12 || !pl34 || ndens < 0 || (ndens && (!D24 || !K13)))
            throw lsjk::Error(LSJK_EINVAL, "null argument");
        lsjk::Context* c = &ctx->c;
        set_device(*c);
        lsjk::Ewald ew = make_ewald(nterm, scales, omegas);
        bool d24 = false, flip = false;
        exchange_prepare(c, const_cast<lsjk::PairList*>(&pl12->p), const_cast<lsjk::PairList*>(&pl34->p), D24symm,
                         &d24, &flip);
        const size_t nD = (size_t) pl12->p.b2->nao * pl34->p.b2->nao;
        const size_t nK = (size_t) pl12->p.b1->nao * pl34->p.b1->nao;
        const int G = std::max(1, std::min(lsjk::kMaxDens, ndens));
        double* dD = ctx->dev((nD + nK) * G);
        double* dK = dD + nD * G;
        double* hD = ctx->io_host.ensure((nD + nK) * G);
        double* hK = hD + nD * G;
        for (int k0 = 0; k0 < ndens; k0 += G) {
            const int ng = std::min(G, ndens - k0);
            const double* dp[lsjk::kMaxDens];
            double* kp[lsjk::kMaxDens];
            for (int g = 0; g < ng; ++g) {
                dp[g] = dD + g * nD;
                kp[g] = dK + g * nK;
                if (nD) std::memcpy(hD + g * nD, D24[k0 + g], sizeof(double) * nD);
            }
            if (nD) LSJK_CUDA(cudaMemcpyAsync(dD, hD, sizeof(double) * nD * ng, cudaMemcpyHostToDevice, c->stream));
            if (nK) LSJK_CUDA(cudaMemsetAsync(dK, 0, sizeof(double) * nK * ng, c->stream));
            exchange_group(c, ew, &pl12->p, &pl34->p, dp, d24, flip, kp, ng, thresp, thredp);
            if (nK) LSJK_CUDA(cudaMemcpyAsync(hK, dK, sizeof(double) * nK * ng, cudaMemcpyDeviceToHost, c->stream));
            check_kernels(c);
            for (int g = 0; g < ng; ++g)
                for (size_t i = 0; i < nK; ++i) K13[k0 + g][i] += hK[g * nK + i];
        }
    });
}

int lsjk_coulomb_grad(lsjk_context* ctx, int nterm, const double* scales, const double* omegas,
                      const lsjk_pairlist* pl, const double* D12, const double* D34, float thresp, float thredp,
                      double* G)
{
    (void) thredp;   // FP64 throughout, as the reference's CPU gradient
    return guard([&] {
        if (!ctx || !pl || !D12 || !D34 || !G) throw lsjk::Error(LSJK_EINVAL, "null argument");
        lsjk::Context* c = &ctx->c;
        set_device(*c);
        lsjk::Ewald ew = make_ewald(nterm, scales, omegas);
        const lsjk::PairList* p = &pl->p;
        check_lmax(p);
        if (!p->symm) throw lsjk::Error(LSJK_EINVAL, "IntBox::coulombGrad: pairlist must be symmetric");
        const lsjk::Basis* b = p->b1;
        const size_t nD = (size_t) b->nao * b->nao, nG = (size_t) b->natom * 3;
        const bool same = D12 == D34;
        c->scratch_reset();
        double* dD = ctx->dev(2 * nD + nG);
        double* dG = dD + 2 * nD;
        double* h = ctx->io_host.ensure(2 * nD + nG);
        std::memcpy(h, D12, sizeof(double) * nD);
        std::memcpy(h + nD, D34, sizeof(double) * nD);
        LSJK_CUDA(cudaMemcpyAsync(dD, h, sizeof(double) * 2 * nD, cudaMemcpyHostToDevice, c->stream));
        LSJK_CUDA(cudaMemsetAsync(dG, 0, sizeof(double) * nG, c->stream));
        double* D12c = lsjk::take<double>(c, (size_t) b->ncart * b->ncart);
        double* D34c = same ? D12c : lsjk::take<double>(c, (size_t) b->ncart * b->ncart);
        lsjk::pure_to_cart(c, b, b, dD, D12c);
        if (!same) lsjk::pure_to_cart(c, b, b, dD + nD, D34c);
        lsjk::coulomb_grad(c, ew, p, D12c, D34c, same, dG, thresp);
        LSJK_CUDA(cudaMemcpyAsync(h, dG, sizeof(double) * nG, cudaMemcpyDeviceToHost, c->stream));
        check_kernels(c);
        for (size_t i = 0; i < nG; ++i) G[i] += h[i];
    });
}

namespace {

void one_electron_host(lsjk_context* ctx, int kind, const lsjk_pairlist* pl, const lsjk::Ewald* ew, int natom,
                       const double* xyzc, double* out)
{
    if (!ctx || !pl || !out || (kind == 2 && natom > 0 && !xyzc)) throw lsjk::Error(LSJK_EINVAL, "null argument");
    if (natom < 0) throw lsjk::Error(LSJK_EINVAL, "natom < 0");
    lsjk::Context* c = &ctx->c;
    set_device(*c);
    const lsjk::PairList* p = &pl->p;
    check_lmax(p);
    const lsjk::Basis *b1 = p->b1, *b2 = p->b2;
    const size_t nX = (size_t) b1->nao * b2->nao, nC = (size_t) b1->ncart * b2->ncart;
    const size_t nq = kind == 2 ? (size_t) 4 * natom : 0;
    c->scratch_reset();
    double* dX = ctx->dev(nX + nq);
    double* dq = dX + nX;
    double* h = ctx->io_host.ensure(nX + nq);
    if (nq) {
        std::memcpy(h + nX, xyzc, sizeof(double) * nq);
        LSJK_CUDA(cudaMemcpyAsync(dq, h + nX, sizeof(double) * nq, cudaMemcpyHostToDevice, c->stream));
    }
    double* Xc = lsjk::take<double>(c, nC);
    LSJK_CUDA(cudaMemsetAsync(Xc, 0, sizeof(double) * nC, c->stream));
    LSJK_CUDA(cudaMemsetAsync(dX, 0, sizeof(double) * nX, c->stream));
    lsjk::one_electron(c, kind, p, ew, dq, natom, Xc);
    lsjk::cart_to_pure_acc(c, b1, b2, Xc, dX);
    LSJK_CUDA(cudaMemcpyAsync(h, dX, sizeof(double) * nX, cudaMemcpyDeviceToHost, c->stream));
    check_kernels(c);
    for (size_t i = 0; i < nX; ++i) out[i] += h[i];
}

} // namespace

int lsjk_overlap(lsjk_context* ctx, const lsjk_pairlist* pl, double* out)
{
    return guard([&] { one_electron_host(ctx, 0, pl, nullptr, 0, nullptr, out); });
}

int lsjk_kinetic(lsjk_context* ctx, const lsjk_pairlist* pl, double* out)
{
    return guard([&] { one_electron_host(ctx, 1, pl, nullptr, 0, nullptr, out); });
}

int lsjk_potential(lsjk_context* ctx, int nterm, const double* scales, const double* omegas, const lsjk_pairlist* pl,
                   int natom, const double* xyzc, double* out)
{
    return guard([&] {
        lsjk::Ewald ew = make_ewald(nterm, scales, omegas);
        one_electron_host(ctx, 2, pl, &ew, natom, xyzc, out);
    });
}

int lsjk_exchange_grad(lsjk_context* ctx, int nterm, const double* scales, const double* omegas,
                       const lsjk_pairlist* pl, const double* D13, const double* D24, int D13symm, int D24symm,
                       int Dsame, float thresp, float thredp, double* G)
{
    (void) thredp;   // FP64 throughout, as the reference's CPU gradient
    return guard([&] {
        if (!ctx || !pl || !D13 || !D24 || !G) throw lsjk::Error(LSJK_EINVAL, "null argument");
        lsjk::Context* c = &ctx->c;
        set_device(*c);
        lsjk::Ewald ew = make_ewald(nterm, scales, omegas);
        lsjk::PairList* p = const_cast<lsjk::PairList*>(&pl->p);
        check_lmax(p);
        if (!p->symm) throw lsjk::Error(LSJK_EINVAL, "IntBox::exchangeGrad: pairlist must be symmetric");
        lsjk::build_kinv(c, p);   // the exact list's rows (merged twins are a K-build option only)
        const lsjk::Basis* b = p->b1;
        const size_t nD = (size_t) b->nao * b->nao, nG = (size_t) b->natom * 3;
        // all three promises: the reference's fully symmetric routine, which reads D13 alone
        // (intbox.cpp:553-564); otherwise its general routine over D13 and D24
        const bool canon = D13symm && D24symm && Dsame;
        const bool same = canon || D13 == D24;
        c->scratch_reset();
        double* dD = ctx->dev(2 * nD + nG);
        double* dG = dD + 2 * nD;
        double* h = ctx->io_host.ensure(2 * nD + nG);
        std::memcpy(h, D13, sizeof(double) * nD);
        if (!same) std::memcpy(h + nD, D24, sizeof(double) * nD);
        LSJK_CUDA(cudaMemcpyAsync(dD, h, sizeof(double) * 2 * nD, cudaMemcpyHostToDevice, c->stream));
        LSJK_CUDA(cudaMemsetAsync(dG, 0, sizeof(double) * nG, c->stream));
        double* D13c = lsjk::take<double>(c, (size_t) b->ncart * b->ncart);
        double* D24c = same ? D13c : lsjk::take<double>(c, (size_t) b->ncart * b->ncart);
        lsjk::pure_to_cart(c, b, b, dD, D13c);
        if (!same) lsjk::pure_to_cart(c, b, b, dD + nD, D24c);
        lsjk::exchange_grad(c, ew, p, D13c, D24c, D13symm && D24symm, canon, dG, thresp);
        LSJK_CUDA(cudaMemcpyAsync(h, dG, sizeof(double) * nG, cudaMemcpyDeviceToHost, c->stream));
        check_kernels(c);
        for (size_t i = 0; i < nG; ++i) G[i] += h[i];
    });
}

int lsjk_graph_begin(lsjk_context* ctx)
{
    return guard([&] {
        if (!ctx) throw lsjk::Error(LSJK_EINVAL, "null context");
        set_device(ctx->c);
        LSJK_CUDA(cudaStreamBeginCapture(ctx->c.stream, cudaStreamCaptureModeThreadLocal));
    });
}

int lsjk_graph_end(lsjk_context* ctx, lsjk_graph** out)
{
    return guard([&] {
        if (!ctx || !out) throw lsjk::Error(LSJK_EINVAL, "null argument");
        set_device(ctx->c);
        auto* g = new lsjk_graph();
        g->ctx = &ctx->c;
        cudaError_t e = cudaStreamEndCapture(ctx->c.stream, &g->graph);
        if (e != cudaSuccess) {
            delete g;
            throw lsjk::Error(LSJK_ECUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
        }
        e = cudaGraphInstantiate(&g->exec, g->graph, 0);
        if (e != cudaSuccess) {
            cudaGraphDestroy(g->graph);
            delete g;
            throw lsjk::Error(LSJK_ECUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
        }
        *out = g;
    });
}

int lsjk_graph_launch(lsjk_graph* graph)
{
    return guard([&] {
        if (!graph) throw lsjk::Error(LSJK_EINVAL, "null graph");
        set_device(*graph->ctx);
        LSJK_CUDA(cudaGraphLaunch(graph->exec, graph->ctx->stream));
    });
}

int lsjk_graph_destroy(lsjk_graph* graph)
{
    return guard([&] {
        if (!graph) return;
        if (graph->exec) cudaGraphExecDestroy(graph->exec);
        if (graph->graph) cudaGraphDestroy(graph->graph);
        delete graph;
    });
}

} // extern "C"

// ---- J build without device allocation -------------------------------------
//
// Some callers may not allocate device memory while they run: a host framework
// that hands out all of the GPU's memory itself and forbids cudaMalloc after
// start-up, or a latency-bound loop that cannot afford the device-wide
// synchronisation cudaMalloc/cudaFree can cause. lsjk_coulomb_device_noalloc
// serves them: every intermediate buffer of the J build (Cartesian D and J,
// ket records, sort keys and sort workspace, bra accumulators, counters) is
// carved from the fixed array below instead of the context's growable scratch.
//
// The array is a file-scope __device__ object, so every GPU that loads this
// library holds its LSJK_NOALLOC_SCRATCH_BYTES until the process exits. All
// calls on a device share it and it keeps the last call's contents; the build
// clears what must start at zero (counters, accumulators) on every call. Two
// calls whose work overlaps on the GPU (different streams or contexts on the
// same device) race on it.
static __device__ __align__(256) unsigned char g_noalloc_scratch[LSJK_NOALLOC_SCRATCH_BYTES];

namespace {

// The CUDA context current on this thread (the driver's cuCtxGetCurrent,
// found in the driver library the runtime has already loaded), or null if
// it cannot be read.
void* current_cuda_context()
{
    using Fn = int (*)(void**);
    static Fn fn = [] {
        void* h = dlopen("libcuda.so.1", RTLD_LAZY | RTLD_NOLOAD);
        return h ? reinterpret_cast<Fn>(dlsym(h, "cuCtxGetCurrent")) : nullptr;
    }();
    void* c = nullptr;
    if (fn && fn(&c) != 0) c = nullptr;
    return c;
}

// Device address of g_noalloc_scratch, looked up once per device and CUDA
// context (a device reset makes a new context, and the address is looked up
// again). In host code the name g_noalloc_scratch is only a host-side
// stand-in for the device object; a kernel given it would fault (or, where
// the GPU can reach host memory, silently use the wrong memory), so kernels
// get this address.
char* noalloc_scratch_address(int device)
{
    struct Entry {
        int device;
        void* context;
        char* addr;
    };
    static std::mutex mu;
    static std::vector<Entry> cache;
    std::lock_guard<std::mutex> lock(mu);
    if (device < 0) throw lsjk::Error(LSJK_EINVAL, "noalloc: bad device");
    // the caller made `device` current (set_device), so its context is current too
    void* context = current_cuda_context();
    for (const Entry& e : cache)
        if (e.device == device && e.context == context) return e.addr;
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
        throw lsjk::Error(LSJK_ECUDA, std::string("noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    for (Entry& x : cache)
        if (x.device == device) {   // the device's earlier context is gone
            x.context = context;
            x.addr = static_cast<char*>(p);
            return x.addr;
        }
    cache.push_back(Entry{device, context, static_cast<char*>(p)});
    return static_cast<char*>(p);
}

// Points the context's scratch allocator at the static array for the lifetime
// of this object and restores the context's own blocks afterwards (also when
// the build throws). With scratch_fixed set, a request that does not fit
// raises LSJK_ENOMEM instead of growing.
struct StaticScratch {
    lsjk::Context* ctx;
    std::vector<std::unique_ptr<lsjk::DBuf<char>>> saved;
    StaticScratch(lsjk::Context* c, char* base) : ctx(c)
    {
        saved.swap(ctx->scratch);
        ctx->scratch.emplace_back(new lsjk::DBuf<char>());
        ctx->scratch.back()->p = base;    // not owned: never freed
        ctx->scratch.back()->n = LSJK_NOALLOC_SCRATCH_BYTES;
        ctx->scratch_used = 0;
        ctx->scratch_fixed = true;
    }
    ~StaticScratch()
    {
        ctx->scratch.back()->p = nullptr;
        ctx->scratch.back()->n = 0;
        ctx->scratch.swap(saved);
        ctx->scratch_used = 0;
        ctx->scratch_fixed = false;
    }
};

} // namespace

extern "C" int lsjk_coulomb_device_noalloc(lsjk_context* ctx, int nterm, const double* scales, const double* omegas,
                                           const lsjk_pairlist* pl12, const lsjk_pairlist* pl34,
                                           const double* D34_dev, float thresp, float thredp, double* J12_dev)
{
    return guard([&] {
        if (!ctx || !pl12 || !pl34 || !D34_dev || !J12_dev) throw lsjk::Error(LSJK_EINVAL, "null argument");
        lsjk::Context* c = &ctx->c;
        set_device(*c);
        lsjk::Ewald ew = make_ewald(nterm, scales, omegas);
        check_lmax(&pl12->p);
        check_lmax(&pl34->p);
        // the Cartesian D and J alone must fit; the rest is checked as the
        // build takes it, always before the first write to J12
        const size_t need = ((sizeof(double) * pl34->p.b1->ncart * pl34->p.b2->ncart + 255) & ~size_t(255)) +
                            ((sizeof(double) * pl12->p.b1->ncart * pl12->p.b2->ncart + 255) & ~size_t(255));
        if (need > LSJK_NOALLOC_SCRATCH_BYTES)
            throw lsjk::Error(LSJK_ENOMEM, "lsjk_coulomb_device_noalloc: the basis is too large for the " +
                                               std::to_string(LSJK_NOALLOC_SCRATCH_BYTES >> 20) +
                                               " MiB static scratch; use lsjk_coulomb_device");
        char* base = noalloc_scratch_address(c->device);
        StaticScratch arena(c, base);
        const double* d[1] = {D34_dev};
        double* j[1] = {J12_dev};
        try {
            coulomb_group(c, ew, &pl12->p, &pl34->p, d, j, 1, thresp, thredp);
        } catch (const lsjk::Error& e) {
            if (e.code == LSJK_ENOMEM)
                throw lsjk::Error(LSJK_ENOMEM, "lsjk_coulomb_device_noalloc: this J build needs more than the " +
                                                   std::to_string(LSJK_NOALLOC_SCRATCH_BYTES >> 20) +
                                                   " MiB static scratch; use lsjk_coulomb_device");
            throw;
        }
    });
}

// ---- MO-basis integrals through J builds (IntBox::eriJ, src/cpp/intbox/mo_eri.cpp:10-157)

namespace {

constexpr int kEriBatch = lsjk::kMaxDens;   // (i, j) densities per J build

struct EriPairs {
    int i[kEriBatch], j[kEriBatch];
};

// D[g] = C1[:, i_g] C2[:, j_g]^T (nao1 x nao2, row-major; mo_eri.cpp:75-86)
__global__ void k_eri_density(EriPairs P, int ng, const double* __restrict__ C1, int n1,
                              const double* __restrict__ C2, int n2, int nao1, int nao2, double* __restrict__ D)
{
    const long per = (long) nao1 * nao2, total = per * ng;
    for (long t = blockIdx.x * (long) blockDim.x + threadIdx.x; t < total; t += (long) gridDim.x * blockDim.x) {
        const int g = (int) (t / per);
        const long pq = t - g * per;
        const int p = (int) (pq / nao2), q = (int) (pq - (long) p * nao2);
        D[t] = C1[(long) p * n1 + P.i[g]] * C2[(long) q * n2 + P.j[g]];
    }
}

// T[g][k][s] = sum_r C3[r][k] J[g][r][s]; grid (s blocks, k, g)
__global__ void k_eri_left(int nao3, int nao4, int n3, const double* __restrict__ C3, const double* __restrict__ J,
                           double* __restrict__ T)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y, g = blockIdx.z;
    if (s >= nao4) return;
    const double* Jg = J + (long) g * nao3 * nao4;
    double acc = 0.0;
    for (int r = 0; r < nao3; ++r) acc += C3[(long) r * n3 + k] * Jg[(long) r * nao4 + s];
    T[((long) g * n3 + k) * nao4 + s] = acc;
}

// I[i_g][j_g][k][l] = sum_s T[g][k][s] C4[s][l], also stored at I[j_g][i_g] for
// a symmetric pair (mo_eri.cpp:112-116)
__global__ void k_eri_right(EriPairs P, int ng, int n2, int n3, int n4, int nao4, const double* __restrict__ T,
                            const double* __restrict__ C4, int sym12, double* __restrict__ I)
{
    const long n34 = (long) n3 * n4, total = ng * n34;
    for (long t = blockIdx.x * (long) blockDim.x + threadIdx.x; t < total; t += (long) gridDim.x * blockDim.x) {
        const int g = (int) (t / n34);
        const int kl = (int) (t - g * n34);
        const int k = kl / n4, l = kl - k * n4;
        const double* Tk = T + ((long) g * n3 + k) * nao4;
        double acc = 0.0;
        for (int s = 0; s < nao4; ++s) acc += Tk[s] * C4[(long) s * n4 + l];
        I[((long) P.i[g] * n2 + P.j[g]) * n34 + kl] = acc;
        if (sym12 && P.i[g] != P.j[g]) I[((long) P.j[g] * n2 + P.i[g]) * n34 + kl] = acc;
    }
}

void upload(lsjk::DBuf<double>& d, const double* h, size_t n, cudaStream_t s)
{
    d.alloc(n);
    if (n) LSJK_CUDA(cudaMemcpyAsync(d.p, h, sizeof(double) * n, cudaMemcpyHostToDevice, s));
}

} // namespace

extern "C" int lsjk_eri_j(lsjk_context* ctx, int nterm, const double* scales, const double* omegas,
                          const lsjk_pairlist* pl12, const lsjk_pairlist* pl34, int n1, int n2, int n3, int n4,
                          const double* C1, const double* C2, const double* C3, const double* C4, int sym12,
                          int sym34, int sym1234, float thresp, float thredp, double* I)
{
    return guard([&] {
        // the orbital counts are checked first: they need no device
        if (n1 < 0 || n2 < 0 || n3 < 0 || n4 < 0) throw lsjk::Error(LSJK_EINVAL, "negative orbital count");
        if ((sym12 && n1 != n2) || (sym34 && n3 != n4) || (sym1234 && (n1 != n3 || n2 != n4)))
            throw lsjk::Error(LSJK_EINVAL, "a symmetry flag needs equal orbital counts");
        if (n3 > 65535) throw lsjk::Error(LSJK_EINVAL, "lsjk_eri_j: at most 65535 orbitals in C3");
        if (!ctx || !pl12 || !pl34) throw lsjk::Error(LSJK_EINVAL, "null argument");
        const size_t nI = (size_t) n1 * n2 * n3 * n4;
        if (nI && (!C1 || !C2 || !C3 || !C4 || !I)) throw lsjk::Error(LSJK_EINVAL, "null argument");
        lsjk::Context* c = &ctx->c;
        set_device(*c);
        lsjk::Ewald ew = make_ewald(nterm, scales, omegas);
        check_lmax(&pl12->p);
        check_lmax(&pl34->p);
        if (!nI) return;
        const int nao1 = pl12->p.b1->nao, nao2 = pl12->p.b2->nao;
        const int nao3 = pl34->p.b1->nao, nao4 = pl34->p.b2->nao;
        cudaStream_t s = c->stream;
        lsjk::DBuf<double> dC1, dC2, dC3, dC4, dD, dJ, dT, dI;
        upload(dC1, C1, (size_t) nao1 * n1, s);
        upload(dC2, C2, (size_t) nao2 * n2, s);
        upload(dC3, C3, (size_t) nao3 * n3, s);
        upload(dC4, C4, (size_t) nao4 * n4, s);
        const size_t n12 = (size_t) nao1 * nao2, n34 = (size_t) nao3 * nao4;
        dD.alloc(n12 * kEriBatch);
        dJ.alloc(n34 * kEriBatch);
        dT.alloc((size_t) kEriBatch * n3 * nao4);
        dI.alloc(nI);
        // the (i, j) densities, i >= j when the bra is symmetric (mo_eri.cpp:71-74)
        std::vector<std::pair<int, int>> ij;
        for (int i = 0; i < n1; ++i)
            for (int j = 0; j < n2; ++j)
                if (!(sym12 && i < j)) ij.emplace_back(i, j);
        for (size_t b0 = 0; b0 < ij.size(); b0 += kEriBatch) {
            const int ng = (int) std::min<size_t>(kEriBatch, ij.size() - b0);
            EriPairs P{};
            for (int g = 0; g < ng; ++g) {
                P.i[g] = ij[b0 + g].first;
                P.j[g] = ij[b0 + g].second;
            }
            if (n12) {
                const long tot = (long) n12 * ng;
                k_eri_density<<<(unsigned) std::min<long>((tot + 255) / 256, 4096), 256, 0, s>>>(
                    P, ng, dC1.p, n1, dC2.p, n2, nao1, nao2, dD.p);
                LSJK_CUDA(cudaGetLastError());
            }
            if (n34) LSJK_CUDA(cudaMemsetAsync(dJ.p, 0, sizeof(double) * n34 * ng, s));
            // J over pl34's pairs of each density on pl12's bases (bra pl34, ket pl12: mo_eri.cpp:88-95)
            {
                static_assert(kEriBatch <= lsjk::kMaxDens, "one J build per batch of densities");
                const double* dp[kEriBatch];
                double* jp[kEriBatch];
                for (int g = 0; g < ng; ++g) {
                    dp[g] = dD.p + g * n12;
                    jp[g] = dJ.p + g * n34;
                }
                coulomb_group(c, ew, &pl34->p, &pl12->p, dp, jp, ng, thresp, thredp);
            }
            // L = C3^T J C4 (mo_eri.cpp:96-110)
            if (nao4 > 0 && nao3 > 0) {
                k_eri_left<<<dim3((unsigned) ((nao4 + 127) / 128), (unsigned) n3, (unsigned) ng), 128, 0, s>>>(
                    nao3, nao4, n3, dC3.p, dJ.p, dT.p);
                LSJK_CUDA(cudaGetLastError());
            } else if (nao4 > 0) {
                LSJK_CUDA(cudaMemsetAsync(dT.p, 0, sizeof(double) * ng * n3 * (size_t) nao4, s));
            }
            const long tot = (long) ng * n3 * n4;
            k_eri_right<<<(unsigned) std::min<long>((tot + 127) / 128, 4096), 128, 0, s>>>(
                P, ng, n2, n3, n4, nao4, dT.p, dC4.p, sym12, dI.p);
            LSJK_CUDA(cudaGetLastError());
        }
        LSJK_CUDA(cudaMemcpyAsync(I, dI.p, sizeof(double) * nI, cudaMemcpyDeviceToHost, s));
        check_kernels(c);
        // the reference's symmetrisations, in its order (mo_eri.cpp:121-155)
        const size_t s234 = (size_t) n2 * n3 * n4, s34 = (size_t) n3 * n4;
        if (sym12)
            for (size_t rs = 0; rs < s34; ++rs)
                for (int p = 0; p < n1; ++p)
                    for (int q = 0; q < p; ++q) {
                        double& a = I[p * s234 + q * s34 + rs];
                        double& b = I[q * s234 + p * s34 + rs];
                        a = b = 0.5 * (a + b);
                    }
        if (sym34)
            for (size_t pq = 0; pq < (size_t) n1 * n2; ++pq) {
                double* Ip = I + pq * s34;
                for (int r = 0; r < n3; ++r)
                    for (int t = 0; t < r; ++t) {
                        double& a = Ip[r * n4 + t];
                        double& b = Ip[t * n4 + r];
                        a = b = 0.5 * (a + b);
                    }
            }
        if (sym1234)
            for (size_t pq = 0; pq < (size_t) n1 * n2; ++pq)
                for (size_t rs = 0; rs < pq; ++rs) {
                    double& a = I[pq * s34 + rs];
                    double& b = I[rs * s34 + pq];
                    a = b = 0.5 * (a + b);
                }
    });
}
