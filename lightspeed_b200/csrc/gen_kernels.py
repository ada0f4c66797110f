"""Emit the straight-line per-quartet integral code for the J and K kernels.

Writes lightspeed_b200/csrc/generated/{jquartets,kquartets_*}.cuh with, for the
angular momentum classes up to LMAX per shell (every class up to d; above d the
ones below a size limit, see j_emitted / k_emitted):

* jq_B<LB>_K<LK>: McMurchie-Davidson Hermite integrals R_{tuv} built from the
  scaled Boys values a_n = f (-2 rho)^n F_n(T) by the recursion
      R^{(n)}_{t+1,u,v} = t R^{(n+1)}_{t-1,u,v} + X_PQ R^{(n+1)}_{t,u,v}
  (and likewise in y, z), contracted with the ket Hermite density:
      jp[t] += sum_u R_{t+u} dk[u].
  This is the J inner loop of the reference (src/cpp/intbox/cpu/coulomb.cpp:
  137-171) written as Boys + Hermite recursion instead of per-root Rys sums;
  both evaluate the same Hermite Coulomb integrals.

* kq_<L1><L2><L3><L4>: one Rys root of a primitive quartet (12|34): the 2-D
  integrals from the standard Rys vertical recursion
      I(a+1,0) = C00 I(a,0) + a B10 I(a-1,0)
      I(a,c+1) = D00 I(a,c) + c B01 I(a,c-1) + a B00 I(a-1,c)
  then horizontal transfer to centres 2 and 4, assembled into the 6-D integral
  and contracted with the density block:  K[i1,i3] += sum_{i2,i4} I D[i2,i4].
  This replaces the 2-D Gauss-Hermite evaluation of the reference K kernel
  (src/cpp/intbox/cpu/exchange.cpp:228-322); both compute the same integrals.

All functions are templates on the arithmetic type so the FP64 and FP32 paths
share one source.  Run:  python lightspeed_b200/csrc/gen_kernels.py [LMAX]
"""
import os
import sys


def cart_list(L):
    """Cartesian components of a shell of angular momentum L in CCA lexical
    order (x^L first), the order used for AO indices."""
    out = []
    for i in range(L + 1):
        l = L - i
        for j in range(i + 1):
            out.append((l, i - j, j))
    return out


def herm_list(L):
    """Hermite functions t=(tx,ty,tz) with |t| <= L in shell-major lexical order."""
    out = []
    for LL in range(L + 1):
        out.extend(cart_list(LL))
    return out


class Emitter:
    def __init__(self):
        self.lines = []
        self.names = {}

    def emit(self, s):
        self.lines.append("    " + s)


# --------------------------------------------------------------------- J ----

def gen_j(LB, LK):
    L = LB + LK
    em = Emitter()
    memo = {}

    def R(n, t, u, v):
        key = (n, t, u, v)
        if key in memo:
            return memo[key]
        if t == 0 and u == 0 and v == 0:
            name = "a[%d]" % n
            memo[key] = name
            return name
        if t > 0:
            d, c, lo = "X", t, (n + 1, t - 2, u, v)
            hi = (n + 1, t - 1, u, v)
            cnt = t - 1
        elif u > 0:
            d, c, lo = "Y", u, (n + 1, t, u - 2, v)
            hi = (n + 1, t, u - 1, v)
            cnt = u - 1
        else:
            d, c, lo = "Z", v, (n + 1, t, u, v - 2)
            hi = (n + 1, t, u, v - 1)
            cnt = v - 1
        h = R(*hi)
        name = "r%d_%d_%d_%d" % key
        if cnt > 0:
            l = R(*lo)
            em.emit("const R %s = fma(%s, %s, R(%d) * %s);" % (name, d, h, cnt, l))
        else:
            em.emit("const R %s = %s * %s;" % (name, d, h))
        memo[key] = name
        return name

    bra = herm_list(LB)
    ket = herm_list(LK)
    body_rs = {}
    for t in bra:
        for u in ket:
            tu = (t[0] + u[0], t[1] + u[1], t[2] + u[2])
            if tu not in body_rs:
                body_rs[tu] = R(0, *tu)
    for ti, t in enumerate(bra):
        em.emit("{ R s = jp[%d];" % ti)
        for ui, u in enumerate(ket):
            tu = (t[0] + u[0], t[1] + u[1], t[2] + u[2])
            em.emit("  s = fma(%s, dk[%d], s);" % (body_rs[tu], ui))
        em.emit("  jp[%d] = s; }" % ti)
    head = ("template <typename R>\n__device__ __forceinline__ void jq_B%d_K%d("
            "const R* __restrict__ a, R X, R Y, R Z, const R* __restrict__ dk, R* __restrict__ jp)\n{\n" % (LB, LK))
    return head + "\n".join(em.lines) + "\n}\n"


# --------------------------------------------------------------------- K ----

def gen_k(L1, L2, L3, L4):
    em = Emitter()
    LA, LC = L1 + L2, L3 + L4
    c1, c2, c3, c4 = cart_list(L1), cart_list(L2), cart_list(L3), cart_list(L4)
    N1, N2, N3, N4 = len(c1), len(c2), len(c3), len(c4)

    def dimfuncs(dim):
        memoI = {}
        memoG = {}
        base = "wz" if dim == "z" else None

        def I(a, c):
            key = (a, c)
            if key in memoI:
                return memoI[key]
            if a == 0 and c == 0:
                memoI[key] = base  # None means the constant 1
                return base
            terms = []
            if c == 0:
                p = I(a - 1, 0)
                terms.append(("c00" + dim, p))
                if a - 1 > 0:
                    terms.append(("R(%d) * b10" % (a - 1), I(a - 2, 0)))
            else:
                p = I(a, c - 1)
                terms.append(("d00" + dim, p))
                if c - 1 > 0:
                    terms.append(("R(%d) * b01" % (c - 1), I(a, c - 2)))
                if a > 0:
                    terms.append(("R(%d) * b00" % a, I(a - 1, c - 1)))
            name = "i%s_%d_%d" % (dim, a, c)
            expr = None
            for coef, src in terms:
                t = coef if src is None else "%s * %s" % (coef, src)
                if expr is None:
                    expr = t
                else:
                    if src is None:
                        expr = "(%s) + %s" % (expr, coef)
                    else:
                        expr = "fma(%s, %s, %s)" % (coef, src, expr)
            em.emit("const R %s = %s;" % (name, expr))
            memoI[key] = name
            return name

        def G(a, b, c, d):
            key = (a, b, c, d)
            if key in memoG:
                return memoG[key]
            if d > 0:
                hi = G(a, b, c + 1, d - 1)
                lo = G(a, b, c, d - 1)
                dd = "cd" + dim
            elif b > 0:
                hi = G(a + 1, b - 1, c, d)
                lo = G(a, b - 1, c, d)
                dd = "ab" + dim
            else:
                name = I(a, c)
                memoG[key] = name
                return name
            name = "g%s_%d_%d_%d_%d" % (dim, a, b, c, d)
            if lo is None:
                em.emit("const R %s = %s + %s;" % (name, hi, dd))
            elif hi is None:
                em.emit("const R %s = fma(%s, %s, R(1));" % (name, dd, lo))
            else:
                em.emit("const R %s = fma(%s, %s, %s);" % (name, dd, lo, hi))
            memoG[key] = name
            return name

        return G

    Gx, Gy, Gz = dimfuncs("x"), dimfuncs("y"), dimfuncs("z")

    def mul(a, b):
        if a is None:
            return b
        if b is None:
            return a
        return "%s * %s" % (a, b)

    # emit all needed 1-D factors first
    need = {}
    for a in c1:
        for b in c2:
            for c in c3:
                for d in c4:
                    need[(a, b, c, d)] = (Gx(a[0], b[0], c[0], d[0]),
                                          Gy(a[1], b[1], c[1], d[1]),
                                          Gz(a[2], b[2], c[2], d[2]))
    for i1, a in enumerate(c1):
        for i3, c in enumerate(c3):
            em.emit("{ R s = K[%d];" % (i1 * N3 + i3))
            for i2, b in enumerate(c2):
                for i4, d in enumerate(c4):
                    gx, gy, gz = need[(a, b, c, d)]
                    xy = mul(gx, gy)
                    em.emit("  s = fma(%s, %s, s);" % (mul(xy, gz) if xy else gz, "D[%d]" % (i2 * N4 + i4)))
            em.emit("  K[%d] = s; }" % (i1 * N3 + i3))
    head = ("template <typename R>\n__device__ __forceinline__ void kq_%d%d%d%d("
            "R c00x, R c00y, R c00z, R d00x, R d00y, R d00z, R b00, R b10, R b01, "
            "R abx, R aby, R abz, R cdx, R cdy, R cdz, R wz, "
            "const R* __restrict__ D, R* __restrict__ K)\n{\n" % (L1, L2, L3, L4))
    # silence unused-parameter warnings for low-L classes
    pre = "    (void)c00x; (void)c00y; (void)c00z; (void)d00x; (void)d00y; (void)d00z;\n" \
          "    (void)b00; (void)b10; (void)b01; (void)abx; (void)aby; (void)abz;\n" \
          "    (void)cdx; (void)cdy; (void)cdz;\n"
    return head + pre + "\n".join(em.lines) + "\n}\n"


def nherm(L):
    return (L + 1) * (L + 2) * (L + 3) // 6


def ncart(L):
    return (L + 1) * (L + 2) // 2


# Every class with shells up to d is emitted. Above d (f shells) a class is emitted
# while its code stays small enough to compile and schedule well: J up to J_TERMS
# (t, u) contraction terms, K below K_COMBOS Cartesian combinations (the larger K
# classes run the quartet-per-warp kernel). The rest take the loop form, and their
# J kernel is k_coulomb_warp (a bra pair per warp). Emitted J classes of 4700 terms
# and more compiled to 32 registers and 38-97 KB of stack per thread; between 1600
# and 3200 terms the emitted and the warp form measured the same.
GEN_D = 2
J_TERMS = 1600
K_COMBOS = 100


def j_emitted(LB, LK):
    return (LB <= 2 * GEN_D + 1 and LK <= 2 * GEN_D) or nherm(LB) * nherm(LK) <= J_TERMS


def k_emitted(L1, L2, L3, L4):
    return max(L1, L2, L3, L4) <= GEN_D or ncart(L1) * ncart(L2) * ncart(L3) * ncart(L4) < K_COMBOS


def main():
    lmax = int(sys.argv[1]) if len(sys.argv) > 1 else 3
    out_dir = os.path.join(os.path.dirname(os.path.abspath(__file__)), "generated")
    os.makedirs(out_dir, exist_ok=True)
    head = ["// Generated by lightspeed_b200/csrc/gen_kernels.py -- do not edit.", "#pragma once",
            "#define LSJK_GEN_LMAX %d" % lmax, ""]
    # J: Hermite classes 0..2*lmax, and bra classes one higher (2*lmax+1) for the
    # nuclear gradients (the Hermite potential at a bra pair one order above its class)
    jcls = [(LB, LK) for LB in range(2 * lmax + 2) for LK in range(2 * lmax + 1) if j_emitted(LB, LK)]
    jparts = list(head)
    for LB, LK in jcls:
        jparts.append(gen_j(LB, LK))
    # classes not emitted here take the loop form
    jparts.append('#include "quartet_loops.cuh"')
    jparts.append("template <int LB, int LK> struct JQ : lsjk::JQLoop<LB, LK> {};")
    for LB, LK in jcls:
        jparts.append("template <> struct JQ<%d, %d> { static constexpr bool loop = false; "
                      "template <typename R> __device__ __forceinline__ static void "
                      "run(const R* a, R X, R Y, R Z, const R* dk, R* jp) { jq_B%d_K%d<R>(a, X, Y, Z, dk, jp); } };"
                      % (LB, LK, LB, LK))
    jparts.append("template <int LB, int LK, typename R> __device__ __forceinline__ void jq_dispatch("
                  "const R* a, R X, R Y, R Z, const R* dk, R* jp) { JQ<LB, LK>::run(a, X, Y, Z, dk, jp); }")
    with open(os.path.join(out_dir, "jquartets.cuh"), "w") as fh:
        fh.write("\n".join(jparts) + "\n")
    # K: one header per (L1, L2) so each instantiation unit parses only its classes
    args = ("R c00x, R c00y, R c00z, R d00x, R d00y, R d00z, R b00, R b10, R b01, R abx, R aby, R abz, "
            "R cdx, R cdy, R cdz, R wz, const R* D, R* K")
    call = "c00x, c00y, c00z, d00x, d00y, d00z, b00, b10, b01, abx, aby, abz, cdx, cdy, cdz, wz, D, K"
    kfwd = list(head)
    kfwd.append('#include "quartet_loops.cuh"')
    kfwd.append("template <int L1, int L2, int L3, int L4> struct KQ : lsjk::KQLoop<L1, L2, L3, L4> {};")
    kfwd.append("template <int L1, int L2, int L3, int L4, typename R> __device__ __forceinline__ void kq_dispatch(%s) "
                "{ KQ<L1, L2, L3, L4>::run(%s); }" % (args, call))
    with open(os.path.join(out_dir, "kquartets_fwd.cuh"), "w") as fh:
        fh.write("\n".join(kfwd) + "\n")
    for L1 in range(lmax + 1):
        for L2 in range(lmax + 1):
            kparts = list(head) + ['#include "kquartets_fwd.cuh"', ""]
            for L3 in range(lmax + 1):
                for L4 in range(lmax + 1):
                    if not k_emitted(L1, L2, L3, L4):
                        continue
                    kparts.append(gen_k(L1, L2, L3, L4))
                    kparts.append("template <> struct KQ<%d, %d, %d, %d> { template <typename R> __device__ "
                                  "__forceinline__ static void run(%s) { kq_%d%d%d%d<R>(%s); } };"
                                  % (L1, L2, L3, L4, args, L1, L2, L3, L4, call))
            with open(os.path.join(out_dir, "kquartets_%d%d.cuh" % (L1, L2)), "w") as fh:
                fh.write("\n".join(kparts) + "\n")
    print("wrote", out_dir)


if __name__ == "__main__":
    main()
