// Primitive pair lists built on the device.
//
//  * Schwarz bound of every primitive pair (src/cpp/core/pair_list.cpp:15-27),
//    evaluated with the reference's operation order and explicit IEEE
//    roundings so the float bounds come out the same;
//  * compaction of pairs with bound > thre (lower triangle for symmetric
//    lists, pair_list.cpp:99-143);
//  * order: class (L1, L2), bound descending, prim1, prim2 ascending
//    (pair_list_util.cpp:12-20) -- two stable LSD radix passes;
//  * the J bra view (classes merged by L1+L2) and the K-invert rows
//    (src/cpp/core/kvec.cpp:31-232).
#include <algorithm>
#include <cub/device/device_radix_sort.cuh>
#include "engine.cuh"
#include "lsjk_device.cuh"

namespace lsjk {

namespace {

struct PairTmp {
    int i, j;
    float b;
    int cls;
};

__device__ __forceinline__ float schwarz_bound(double c1, double e1, double x1, double y1, double z1,
                                               double c2, double e2, double x2, double y2, double z2)
{
    // R2 = pow(dx,2) + pow(dy,2) + pow(dz,2), no contraction
    double dx = __dsub_rn(x1, x2), dy = __dsub_rn(y1, y2), dz = __dsub_rn(z1, z2);
    double R2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
    double p = __dadd_rn(e1, e2);
    double ex = __dmul_rn(__ddiv_rn(__dmul_rn(-e1, e2), p), R2);
    double v = __dmul_rn(fabs(__dmul_rn(c1, c2)), exp(ex));
    v = __dmul_rn(v, 1.18920711500272106672);               // pow(2.0, 0.25)
    v = __dmul_rn(v, pow(__ddiv_rn(3.14159265358979323846, p), 1.25));
    return (float) v;
}

__global__ void k_pair_bounds(BasisView b1, BasisView b2, int symm, float thre, int nL2,
                              PairTmp* __restrict__ out, unsigned long long* __restrict__ count)
{
    int i = blockIdx.y;
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    bool keep = false;
    PairTmp t;
    if (j < b2.nprim && !(symm && j > i)) {
        float b = schwarz_bound(b1.c[i], b1.e[i], b1.x[i], b1.y[i], b1.z[i],
                                b2.c[j], b2.e[j], b2.x[j], b2.y[j], b2.z[j]);
        if (b > thre) {
            keep = true;
            t = PairTmp{i, j, b, b1.L[i] * nL2 + b2.L[j]};
        }
    }
    // warp-aggregated append
    unsigned mask = __ballot_sync(0xffffffffu, keep);
    if (!mask) return;
    int lane = threadIdx.x & 31;
    unsigned long long base = 0;
    if (lane == __ffs(mask) - 1) base = atomicAdd(count, (unsigned long long) __popc(mask));
    base = __shfl_sync(0xffffffffu, base, __ffs(mask) - 1);
    if (keep) out[base + __popc(mask & ((1u << lane) - 1))] = t;
}

__global__ void k_keys_ij(const PairTmp* __restrict__ in, long n, unsigned* __restrict__ key,
                          int* __restrict__ val)
{
    long k = blockIdx.x * (long) blockDim.x + threadIdx.x;
    if (k >= n) return;
    key[k] = ((unsigned) in[k].i << 16) | (unsigned) in[k].j;
    val[k] = (int) k;
}

// key = (class << 32) | ~bits(bound): ascending order = class asc, bound desc.
__global__ void k_keys_cls_bound(const PairTmp* __restrict__ in, const int* __restrict__ perm, long n,
                                 int herm, unsigned long long* __restrict__ key)
{
    long k = blockIdx.x * (long) blockDim.x + threadIdx.x;
    if (k >= n) return;
    const PairTmp& t = in[perm[k]];
    unsigned cls = (unsigned) t.cls;
    if (herm) cls = (unsigned) herm - 1;   // filled below for the Hermite view
    key[k] = ((unsigned long long) cls << 32) | (unsigned long long) (~__float_as_uint(t.b));
}

__global__ void k_keys_herm(const PairTmp* __restrict__ in, const int* __restrict__ perm, long n,
                            const int* __restrict__ L1, const int* __restrict__ L2,
                            unsigned long long* __restrict__ key)
{
    long k = blockIdx.x * (long) blockDim.x + threadIdx.x;
    if (k >= n) return;
    const PairTmp& t = in[perm[k]];
    unsigned cls = (unsigned) (L1[t.i] + L2[t.j]);
    key[k] = ((unsigned long long) cls << 32) | (unsigned long long) (~__float_as_uint(t.b));
}

__global__ void k_gather_pairs(const PairTmp* __restrict__ in, const int* __restrict__ perm, long n,
                               int* __restrict__ p1, int* __restrict__ p2, float* __restrict__ b)
{
    long k = blockIdx.x * (long) blockDim.x + threadIdx.x;
    if (k >= n) return;
    const PairTmp& t = in[perm[k]];
    p1[k] = t.i;
    p2[k] = t.j;
    b[k] = t.b;
}

// Gaussian product geometry of a pair: p = e1 + e2, P = (e1 A + e2 B) / p.
__global__ void k_pair_geom(BasisView b1, BasisView b2, const int* __restrict__ p1,
                            const int* __restrict__ p2, int n, double* __restrict__ geom)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int i = p1[k], j = p2[k];
    double e1 = b1.e[i], e2 = b2.e[j];
    double p = e1 + e2, ip = 1.0 / p;
    geom[4 * k + 0] = p;
    geom[4 * k + 1] = (e1 * b1.x[i] + e2 * b2.x[j]) * ip;
    geom[4 * k + 2] = (e1 * b1.y[i] + e2 * b2.y[j]) * ip;
    geom[4 * k + 3] = (e1 * b1.z[i] + e2 * b2.z[j]) * ip;
}

template <typename K, typename V>
void radix_sort_pairs(Context* ctx, const K* kin, K* kout, const V* vin, V* vout, long n, int end_bit)
{
    size_t tmp = 0;
    LSJK_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, kin, kout, vin, vout, (int) n, 0, end_bit,
                                              ctx->stream));
    void* t = ctx->scratch_take(tmp);
    LSJK_CUDA(cub::DeviceRadixSort::SortPairs(t, tmp, kin, kout, vin, vout, (int) n, 0, end_bit,
                                              ctx->stream));
    ctx->stats.kernel_launches += 4;
}

inline unsigned nblk(long n, int t) { return (unsigned) ((n + t - 1) / t); }

// ---- K-invert -------------------------------------------------------------

struct KEnt {
    int idx;      // indexed primitive (the "2" of K13 += (12|34) D24)
    int part;     // partner primitive (the "1")
    float b;
    int cls;      // L_idx * kNL + L_part
};

__global__ void k_kinv_entries(const int* __restrict__ p1, const int* __restrict__ p2,
                               const float* __restrict__ b, long n, int symm,
                               const int* __restrict__ L1, const int* __restrict__ L2,
                               KEnt* __restrict__ out, unsigned long long* __restrict__ count)
{
    long k = blockIdx.x * (long) blockDim.x + threadIdx.x;
    if (k >= n) return;
    int i = p1[k], j = p2[k];
    // build21 (kvec.cpp:128-168): indexed = prim2, partner = prim1
    unsigned long long s = atomicAdd(count, 1ull);
    out[s] = KEnt{j, i, b[k], L2[j] * kNL + L1[i]};
    // build_symmetric (kvec.cpp:169-232): both orientations, diagonal once
    if (symm && i != j) {
        s = atomicAdd(count, 1ull);
        out[s] = KEnt{i, j, b[k], L1[i] * kNL + L2[j]};
    }
}

// pass A key: bound desc, partner asc
__global__ void k_kinv_key1(const KEnt* __restrict__ e, long n, unsigned long long* __restrict__ key,
                            int* __restrict__ val)
{
    long k = blockIdx.x * (long) blockDim.x + threadIdx.x;
    if (k >= n) return;
    key[k] = ((unsigned long long) (~__float_as_uint(e[k].b)) << 16) | (unsigned) e[k].part;
    val[k] = (int) k;
}

// pass B key: (class, indexed, partner target group) -- the group names the
// output block(s) the partner's contributions go to (its contracted shell)
__global__ void k_kinv_key2(const KEnt* __restrict__ e, const int* __restrict__ perm, long n,
                            const int* __restrict__ pseg, unsigned long long* __restrict__ key)
{
    long k = blockIdx.x * (long) blockDim.x + threadIdx.x;
    if (k >= n) return;
    const KEnt& t = e[perm[k]];
    key[k] = ((unsigned long long) t.cls << 48) | ((unsigned long long) t.idx << 32) | (unsigned) pseg[t.part];
}

// row key (class, indexed): a stable pass over the bound order gives each row
// its entries by bound alone (the partner-3 copy of the rows)
__global__ void k_kinv_keyrow(const KEnt* __restrict__ e, const int* __restrict__ perm, long n,
                              unsigned long long* __restrict__ key)
{
    long k = blockIdx.x * (long) blockDim.x + threadIdx.x;
    if (k >= n) return;
    const KEnt& t = e[perm[k]];
    key[k] = ((unsigned long long) t.cls << 32) | (unsigned) t.idx;
}

// pass C key: (class, indexed, segment max bound desc); the segment max is the
// bound of the segment's first entry after pass B.
__global__ void k_kinv_key3(const KEnt* __restrict__ e, const int* __restrict__ perm,
                            const unsigned long long* __restrict__ key2s, long n,
                            unsigned long long* __restrict__ key)
{
    long k = blockIdx.x * (long) blockDim.x + threadIdx.x;
    if (k >= n) return;
    long h = k;
    while (h > 0 && key2s[h - 1] == key2s[k]) --h;   // segments are short (<= shell length)
    const KEnt& t = e[perm[k]];
    const KEnt& head = e[perm[h]];
    key[k] = ((unsigned long long) t.cls << 48) | ((unsigned long long) t.idx << 32) |
             (unsigned long long) (~__float_as_uint(head.b));
}

__global__ void k_kinv_fill(const KEnt* __restrict__ e, const int* __restrict__ perm, long n,
                            BasisView bidx, BasisView bpart, KInvData* __restrict__ out_unused,
                            double* __restrict__ kab, double* __restrict__ pp, double* __restrict__ ipp,
                            double* __restrict__ px, double* __restrict__ py, double* __restrict__ pz,
                            double* __restrict__ ax, double* __restrict__ ay, double* __restrict__ az,
                            float* __restrict__ kab32, float* __restrict__ pp32, float* __restrict__ ipp32,
                            float* __restrict__ px32, float* __restrict__ py32, float* __restrict__ pz32,
                            float* __restrict__ ax32, float* __restrict__ ay32, float* __restrict__ az32,
                            int* __restrict__ pcart, float* __restrict__ pb, int* __restrict__ pt1,
                            int* __restrict__ pseg, double* __restrict__ pw0, double* __restrict__ pw1,
                            float* __restrict__ pw0_32, float* __restrict__ pw1_32, double* __restrict__ pe,
                            int* __restrict__ patom, int* __restrict__ pidx, int* __restrict__ rstart,
                            int* __restrict__ rlen, int nrow)
{
    long k = blockIdx.x * (long) blockDim.x + threadIdx.x;
    if (k >= n) return;
    const KEnt& t = e[perm[k]];
    int i = t.idx, j = t.part;
    double ei = bidx.e[i], ej = bpart.e[j];
    double Ax = bpart.x[j] - bidx.x[i], Ay = bpart.y[j] - bidx.y[i], Az = bpart.z[j] - bidx.z[i];
    double p = ei + ej, ip = 1.0 / p;
    // K_ab = c_a c_b exp(-e_a e_b / (e_a + e_b) |AB|^2)  (kvec.cpp:66-70)
    double K = bidx.c[i] * bpart.c[j] * exp(-ei * ej * ip * (Ax * Ax + Ay * Ay + Az * Az));
    double Px = ej * Ax * ip, Py = ej * Ay * ip, Pz = ej * Az * ip;   // P - R_i
    kab[k] = K * ip; pp[k] = p; ipp[k] = ip;   // K_ab / p: the pair's share of the ERI prefactor
    px[k] = Px; py[k] = Py; pz[k] = Pz; ax[k] = Ax; ay[k] = Ay; az[k] = Az;
    kab32[k] = (float) (K * ip); pp32[k] = (float) p; ipp32[k] = (float) ip;
    px32[k] = (float) Px; py32[k] = (float) Py; pz32[k] = (float) Pz;
    ax32[k] = (float) Ax; ay32[k] = (float) Ay; az32[k] = (float) Az;
    pcart[k] = bpart.t0[j];
    pt1[k] = bpart.t1[j];
    pseg[k] = bpart.seg[j];
    pw0[k] = bpart.w0[j];
    pw1[k] = bpart.w1[j];
    pw0_32[k] = (float) bpart.w0[j];
    pw1_32[k] = (float) bpart.w1[j];
    pe[k] = ej;
    patom[k] = bpart.atom[j];
    pidx[k] = j;
    pb[k] = t.b;
    long r = (long) t.cls * nrow + i;
    bool first = (k == 0);
    if (!first) {
        const KEnt& u = e[perm[k - 1]];
        first = (u.cls != t.cls) || (u.idx != t.idx);
    }
    if (first) rstart[r] = (int) k;
    atomicAdd(&rlen[r], 1);
}

} // namespace

void build_pairlist(Context* ctx, PairList* pl)
{
    const Basis* b1 = pl->b1;
    const Basis* b2 = pl->b2;
    if (b1->nprim >= 65536 || b2->nprim >= 65536)
        throw Error(LSJK_EINVAL, "PairList: more than 65535 primitives per basis is not supported");
    if (pl->symm && (b1->nprim != b2->nprim || b1->natom != b2->natom))
        throw Error(LSJK_EINVAL, "PairList::build_schwarz: basis sets are not symmetric");
    cudaStream_t s = ctx->stream;
    ctx->scratch_reset();
    long cap = (long) b1->nprim * b2->nprim;
    int nL2 = b2->maxL + 1;
    PairTmp* tmp = take<PairTmp>(ctx, cap);
    unsigned long long* cnt = take<unsigned long long>(ctx, 1);
    LSJK_CUDA(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), s));
    if (cap > 0) {
        dim3 grid(nblk(b2->nprim, 128), b1->nprim);
        k_pair_bounds<<<grid, 128, 0, s>>>(b1->view(), b2->view(), pl->symm ? 1 : 0, pl->thre, nL2, tmp, cnt);
        LSJK_CUDA(cudaGetLastError());
    }
    unsigned long long hn = 0;
    LSJK_CUDA(cudaMemcpyAsync(&hn, cnt, sizeof(hn), cudaMemcpyDeviceToHost, s));
    LSJK_CUDA(cudaStreamSynchronize(s));
    long n = (long) hn;
    pl->npair = n;
    pl->p1.alloc(n);
    pl->p2.alloc(n);
    pl->bound.alloc(n);
    pl->cls_L1.clear();
    pl->cls_L2.clear();
    pl->cls_off.assign(1, 0);
    pl->cls_max.clear();
    pl->max_bound = 0.0;
    for (int h = 0; h < kNHerm; ++h) pl->jb[h].n = 0;
    if (n == 0) return;

    // pass 1: (prim1, prim2) ascending
    unsigned* k1 = take<unsigned>(ctx, n);
    unsigned* k1s = take<unsigned>(ctx, n);
    int* v1 = take<int>(ctx, n);
    int* perm1 = take<int>(ctx, n);
    k_keys_ij<<<nblk(n, 256), 256, 0, s>>>(tmp, n, k1, v1);
    radix_sort_pairs(ctx, k1, k1s, v1, perm1, n, 32);
    // pass 2 (stable): class asc, bound desc
    unsigned long long* k2 = take<unsigned long long>(ctx, n);
    unsigned long long* k2s = take<unsigned long long>(ctx, n);
    int* perm = take<int>(ctx, n);
    k_keys_cls_bound<<<nblk(n, 256), 256, 0, s>>>(tmp, perm1, n, 0, k2);
    radix_sort_pairs(ctx, k2, k2s, perm1, perm, n, 40);
    k_gather_pairs<<<nblk(n, 256), 256, 0, s>>>(tmp, perm, n, pl->p1.p, pl->p2.p, pl->bound.p);
    LSJK_CUDA(cudaGetLastError());

    // class offsets and the leading (largest) bound of each class
    std::vector<unsigned long long> hk(n);
    LSJK_CUDA(cudaMemcpyAsync(hk.data(), k2s, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost, s));
    LSJK_CUDA(cudaStreamSynchronize(s));
    for (long k = 0; k < n; ++k) {
        unsigned cls = (unsigned) (hk[k] >> 32);
        if (k == 0 || cls != (unsigned) (hk[k - 1] >> 32)) {
            if (k > 0) pl->cls_off.push_back(k);
            pl->cls_L1.push_back((int) cls / nL2);
            pl->cls_L2.push_back((int) cls % nL2);
            unsigned bits = ~(unsigned) (hk[k] & 0xffffffffu);
            float b;
            memcpy(&b, &bits, sizeof(b));
            pl->cls_max.push_back(b);
            pl->max_bound = std::max(pl->max_bound, (double) b);
        }
    }
    pl->cls_off.push_back(n);

    // J bra view: stable re-sort of pass-1 order by (L1+L2, bound desc)
    int* perm_h = take<int>(ctx, n);
    k_keys_herm<<<nblk(n, 256), 256, 0, s>>>(tmp, perm1, n, b1->dL.p, b2->dL.p, k2);
    radix_sort_pairs(ctx, k2, k2s, perm1, perm_h, n, 40);
    std::vector<unsigned long long> hh(n);
    LSJK_CUDA(cudaMemcpyAsync(hh.data(), k2s, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost, s));
    LSJK_CUDA(cudaStreamSynchronize(s));
    long start = 0;
    for (int h = 0; h < kNHerm + 4; ++h) {
        long end = start;
        while (end < n && (int) (hh[end] >> 32) == h) ++end;
        long cnth = end - start;
        if (h < kNHerm) {
            JBraClass& jb = pl->jb[h];
            jb.n = (int) cnth;
            jb.p1.alloc(cnth);
            jb.p2.alloc(cnth);
            jb.bound.alloc(cnth);
            jb.geom.alloc(4 * cnth);
            if (cnth) {
                k_gather_pairs<<<nblk(cnth, 256), 256, 0, s>>>(tmp, perm_h + start, cnth, jb.p1.p, jb.p2.p,
                                                               jb.bound.p);
                k_pair_geom<<<nblk(cnth, 256), 256, 0, s>>>(b1->view(), b2->view(), jb.p1.p, jb.p2.p,
                                                            (int) cnth, jb.geom.p);
            }
        } else if (cnth) {
            throw Error(LSJK_ENOTSUPP, "PairList: angular momentum above d is not supported by the GPU J/K kernels");
        }
        start = end;
    }
    LSJK_CUDA(cudaGetLastError());
    LSJK_CUDA(cudaStreamSynchronize(s));
    ctx->stats.kernel_launches += 8;
}

void build_kinv(Context* ctx, PairList* pl)
{
    if (pl->kinv_built) return;
    cudaStream_t s = ctx->stream;
    ctx->scratch_reset();
    const Basis* bidx = pl->b2;   // indexed primitives live in basis 2 (basis 1 if symmetric)
    const Basis* bpart = pl->b1;
    long n = pl->npair;
    long cap = pl->symm ? 2 * n : n;
    int nrow = bidx->nprim;
    KInvData& kd = pl->kdat;
    for (int a = 0; a < kNL; ++a)
        for (int b = 0; b < kNL; ++b) {
            pl->kinv[a][b].row_start.alloc(nrow);
            pl->kinv[a][b].row_len.alloc(nrow);
            pl->kinv[a][b].nent = 0;
        }
    if (n == 0) { kd.nent = 0; pl->kinv_built = true; return; }
    KEnt* ent = take<KEnt>(ctx, cap);
    unsigned long long* cnt = take<unsigned long long>(ctx, 1);
    LSJK_CUDA(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), s));
    k_kinv_entries<<<nblk(n, 256), 256, 0, s>>>(pl->p1.p, pl->p2.p, pl->bound.p, n, pl->symm ? 1 : 0,
                                               pl->b1->dL.p, pl->b2->dL.p, ent, cnt);
    unsigned long long hn = 0;
    LSJK_CUDA(cudaMemcpyAsync(&hn, cnt, sizeof(hn), cudaMemcpyDeviceToHost, s));
    LSJK_CUDA(cudaStreamSynchronize(s));
    long m = (long) hn;
    kd.nent = m;
    kd.kab.alloc(m); kd.p.alloc(m); kd.ip.alloc(m); kd.px.alloc(m); kd.py.alloc(m); kd.pz.alloc(m);
    kd.ax.alloc(m); kd.ay.alloc(m); kd.az.alloc(m);
    kd.kab32.alloc(m); kd.p32.alloc(m); kd.ip32.alloc(m); kd.px32.alloc(m); kd.py32.alloc(m);
    kd.pz32.alloc(m); kd.ax32.alloc(m); kd.ay32.alloc(m); kd.az32.alloc(m);
    kd.pcart.alloc(m); kd.pbound.alloc(m);
    kd.pt1.alloc(m); kd.pseg.alloc(m); kd.pw0.alloc(m); kd.pw1.alloc(m); kd.pw0_32.alloc(m); kd.pw1_32.alloc(m);
    kd.pe.alloc(m); kd.patom.alloc(m); kd.pidx.alloc(m);
    unsigned long long* ka = take<unsigned long long>(ctx, m);
    unsigned long long* kas = take<unsigned long long>(ctx, m);
    int* va = take<int>(ctx, m);
    int* pa = take<int>(ctx, m);
    k_kinv_key1<<<nblk(m, 256), 256, 0, s>>>(ent, m, ka, va);
    radix_sort_pairs(ctx, ka, kas, va, pa, m, 48);
    unsigned long long* kr = take<unsigned long long>(ctx, m);
    unsigned long long* krs = take<unsigned long long>(ctx, m);
    int* perm_b = take<int>(ctx, m);
    k_kinv_keyrow<<<nblk(m, 256), 256, 0, s>>>(ent, pa, m, kr);
    radix_sort_pairs(ctx, kr, krs, pa, perm_b, m, 36);
    unsigned long long* kb = take<unsigned long long>(ctx, m);
    unsigned long long* kbs = take<unsigned long long>(ctx, m);
    int* pb2 = take<int>(ctx, m);
    k_kinv_key2<<<nblk(m, 256), 256, 0, s>>>(ent, pa, m, bpart->dseg.p, kb);
    radix_sort_pairs(ctx, kb, kbs, pa, pb2, m, 52);
    unsigned long long* kc = take<unsigned long long>(ctx, m);
    unsigned long long* kcs = take<unsigned long long>(ctx, m);
    int* perm = take<int>(ctx, m);
    k_kinv_key3<<<nblk(m, 256), 256, 0, s>>>(ent, pb2, kbs, m, kc);
    radix_sort_pairs(ctx, kc, kcs, pb2, perm, m, 52);
    // row tables live in one [class][row] block per class
    int* rstart = take<int>(ctx, (long) kNL * kNL * nrow);
    int* rlen = take<int>(ctx, (long) kNL * kNL * nrow);
    LSJK_CUDA(cudaMemsetAsync(rstart, 0, sizeof(int) * kNL * kNL * nrow, s));
    LSJK_CUDA(cudaMemsetAsync(rlen, 0, sizeof(int) * kNL * kNL * nrow, s));
    k_kinv_fill<<<nblk(m, 256), 256, 0, s>>>(ent, perm, m, bidx->view(), bpart->view(), nullptr, kd.kab.p, kd.p.p,
                                            kd.ip.p, kd.px.p, kd.py.p, kd.pz.p, kd.ax.p, kd.ay.p, kd.az.p,
                                            kd.kab32.p, kd.p32.p, kd.ip32.p, kd.px32.p, kd.py32.p, kd.pz32.p,
                                            kd.ax32.p, kd.ay32.p, kd.az32.p, kd.pcart.p, kd.pbound.p, kd.pt1.p,
                                            kd.pseg.p, kd.pw0.p, kd.pw1.p, kd.pw0_32.p, kd.pw1_32.p, kd.pe.p,
                                            kd.patom.p, kd.pidx.p, rstart, rlen, nrow);
    LSJK_CUDA(cudaGetLastError());
    // the bound-ordered copy (same rows, so the same row tables)
    KInvData& kb_ = pl->kdat_b;
    kb_.nent = m;
    kb_.kab.alloc(m); kb_.p.alloc(m); kb_.ip.alloc(m); kb_.px.alloc(m); kb_.py.alloc(m); kb_.pz.alloc(m);
    kb_.ax.alloc(m); kb_.ay.alloc(m); kb_.az.alloc(m);
    kb_.kab32.alloc(m); kb_.p32.alloc(m); kb_.ip32.alloc(m); kb_.px32.alloc(m); kb_.py32.alloc(m);
    kb_.pz32.alloc(m); kb_.ax32.alloc(m); kb_.ay32.alloc(m); kb_.az32.alloc(m);
    kb_.pcart.alloc(m); kb_.pbound.alloc(m);
    kb_.pt1.alloc(m); kb_.pseg.alloc(m); kb_.pw0.alloc(m); kb_.pw1.alloc(m); kb_.pw0_32.alloc(m);
    kb_.pw1_32.alloc(m); kb_.pe.alloc(m); kb_.patom.alloc(m); kb_.pidx.alloc(m);
    int* rstart_b = take<int>(ctx, (long) kNL * kNL * nrow);
    int* rlen_b = take<int>(ctx, (long) kNL * kNL * nrow);
    LSJK_CUDA(cudaMemsetAsync(rstart_b, 0, sizeof(int) * kNL * kNL * nrow, s));
    LSJK_CUDA(cudaMemsetAsync(rlen_b, 0, sizeof(int) * kNL * kNL * nrow, s));
    k_kinv_fill<<<nblk(m, 256), 256, 0, s>>>(ent, perm_b, m, bidx->view(), bpart->view(), nullptr, kb_.kab.p,
                                            kb_.p.p, kb_.ip.p, kb_.px.p, kb_.py.p, kb_.pz.p, kb_.ax.p, kb_.ay.p,
                                            kb_.az.p, kb_.kab32.p, kb_.p32.p, kb_.ip32.p, kb_.px32.p, kb_.py32.p,
                                            kb_.pz32.p, kb_.ax32.p, kb_.ay32.p, kb_.az32.p, kb_.pcart.p,
                                            kb_.pbound.p, kb_.pt1.p, kb_.pseg.p, kb_.pw0.p, kb_.pw1.p, kb_.pw0_32.p,
                                            kb_.pw1_32.p, kb_.pe.p, kb_.patom.p, kb_.pidx.p, rstart_b, rlen_b, nrow);
    LSJK_CUDA(cudaGetLastError());
    for (int a = 0; a < kNL; ++a)
        for (int b = 0; b < kNL; ++b) {
            long off = (long) (a * kNL + b) * nrow;
            LSJK_CUDA(cudaMemcpyAsync(pl->kinv[a][b].row_start.p, rstart + off, sizeof(int) * nrow,
                                      cudaMemcpyDeviceToDevice, s));
            LSJK_CUDA(cudaMemcpyAsync(pl->kinv[a][b].row_len.p, rlen + off, sizeof(int) * nrow,
                                      cudaMemcpyDeviceToDevice, s));
        }
    LSJK_CUDA(cudaStreamSynchronize(s));
    pl->kinv_built = true;
    ctx->stats.kernel_launches += 20;
}

} // namespace lsjk
