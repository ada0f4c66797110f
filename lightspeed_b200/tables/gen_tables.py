"""Generate the Rys quadrature and Boys function interpolation tables used by the
device kernels (written to lightspeed_b200/csrc/tables/quad_tables.inc).

The tables are built here from first principles, not taken from any other code:

* Rys roots/weights for the measure exp(-T t^2) dt on t in [0, 1] come from the
  Golub-Welsch procedure: the measure is discretised with the 512 positive nodes of
  a 1024-point Gauss-Legendre rule (exact for the polynomial part, converged for the
  Gaussian factor up to T ~ 100), the Jacobi matrix is obtained by Lanczos with
  full re-orthogonalisation, and its eigen-decomposition gives roots x_i = t_i^2
  and weights.  Above T_asym(n) the roots/weights follow the half-range
  Gauss-Hermite limit t_i = s_i / sqrt(T), w_i = h_i / sqrt(T), where s_i, h_i are
  the positive nodes and weights of the 2n-point Gauss-Hermite rule.
* Boys functions F_m(T) = int_0^1 t^{2m} exp(-T t^2) dt come from mpmath's
  regularised incomplete gamma function at 30 digits.  Above T_boys the device
  uses F_0 = sqrt(pi/T)/2 and the upward recursion with the exp(-T) term.

Each interval [0, T_asym) is split into uniform bins; in every bin each function
(t_i, ln w_i for Rys -- for the one-point rule w_1 = F_0(T) itself, smooth and
of modest range, so the device needs no exponential there; F_m for Boys) is
interpolated by a degree-7 Chebyshev
series that is then rewritten as a monomial polynomial in the local variable
x in [-1, 1] so the device can evaluate it with 8 fused multiply-adds (Horner).
Interpolating ln w (then exponentiating) keeps small weights relatively
accurate, as the reference's Rys tables also do (src/lightspeed/rys.hpp:109-153).

Run:  python lightspeed_b200/tables/gen_tables.py   (takes ~10 s)
"""
import os
import sys
import numpy as np
from numpy.polynomial import legendre, hermite, chebyshev

NMAX_RYS = 9            # roots 1..9 (total angular momentum up to 16)
MMAX_BOYS = 16          # Boys orders 0..16
DEG = 7                 # polynomial degree per bin (8 coefficients)
NCOEF = DEG + 1

# Discretised Rys measure: positive half of a 1024-point Gauss-Legendre rule.
_gx, _gw = legendre.leggauss(1024)
_TK = _gx[_gx > 0]
_VK = _gw[_gx > 0]
_XK = _TK ** 2


def rys_exact(n, T):
    """Roots t_i (ascending) and weights w_i of the n-point Rys rule at T."""
    w = _VK * np.exp(-T * _XK)
    q = np.sqrt(w)
    mu0 = q @ q
    q = q / np.sqrt(mu0)
    basis = [q]
    alpha, beta = [], []
    qprev = np.zeros_like(q)
    b = 0.0
    for _ in range(n):
        v = _XK * basis[-1]
        a = basis[-1] @ v
        alpha.append(a)
        v = v - a * basis[-1] - b * qprev
        for _rep in range(2):
            for qq in basis:
                v -= (qq @ v) * qq
        b = np.sqrt(v @ v)
        beta.append(b)
        qprev = basis[-1]
        basis.append(v / b)
    J = np.diag(alpha) + np.diag(beta[: n - 1], 1) + np.diag(beta[: n - 1], -1)
    ev, V = np.linalg.eigh(J)
    return np.sqrt(ev), mu0 * V[0, :] ** 2


def rys_asym(n):
    s, h = hermite.hermgauss(2 * n)
    pos = s > 0
    order = np.argsort(s[pos])
    return s[pos][order], h[pos][order]


def boys_exact(mmax, T):
    import mpmath as mp
    mp.mp.dps = 30
    out = np.zeros(mmax + 1)
    for m in range(mmax + 1):
        if T == 0.0:
            out[m] = 1.0 / (2 * m + 1)
        else:
            a = mp.mpf(m) + mp.mpf(1) / 2
            Tm = mp.mpf(T)
            out[m] = float(mp.gammainc(a, 0, Tm) / (2 * Tm ** a))
    return out


def _fit_bins(func, nfun, tmax, nbin):
    """Degree-DEG Chebyshev interpolation per bin, returned as monomial
    coefficients c[fun][bin][k] of sum_k c_k x^k, x in [-1, 1]."""
    h = tmax / nbin
    xs = np.cos(np.pi * (np.arange(NCOEF) + 0.5) / NCOEF)  # Chebyshev nodes
    coefs = np.zeros((nfun, nbin, NCOEF))
    for b in range(nbin):
        T0 = b * h
        vals = np.array([func(T0 + 0.5 * h * (x + 1.0)) for x in xs])  # (NCOEF, nfun)
        for f in range(nfun):
            ch = chebyshev.chebfit(xs, vals[:, f], DEG)
            coefs[f, b, :] = chebyshev.cheb2poly(ch)
    return coefs


def _eval_bins(coefs, tmax, nbin, T):
    h = tmax / nbin
    b = min(int(T / h), nbin - 1)
    x = 2.0 * (T / h - b) - 1.0
    out = []
    for f in range(coefs.shape[0]):
        c = coefs[f, b]
        acc = c[-1]
        for k in range(NCOEF - 2, -1, -1):
            acc = acc * x + c[k]
        out.append(acc)
    return np.array(out)


def choose_rys_tasym(n, eps=2e-15):
    s, h = rys_asym(n)
    T = 20.0
    while True:
        ok = True
        for TT in np.arange(T, T + 20.0, 0.5):
            t, w = rys_exact(n, TT)
            if np.max(np.abs(t - s / np.sqrt(TT))) > eps or np.max(np.abs(w - h / np.sqrt(TT))) > eps:
                ok = False
                break
        if ok:
            return T
        T += 1.0


def build_rys(n, width):
    tasym = choose_rys_tasym(n)
    nbin = int(np.ceil(tasym / width))
    tmax = nbin * width

    def func(T):
        t, w = rys_exact(n, T)
        return np.concatenate([t, w if n == 1 else np.log(w)])

    coefs = _fit_bins(func, 2 * n, tmax, nbin)
    # accuracy check on random points
    rng = np.random.default_rng(n)
    errt = errw = 0.0
    for T in rng.uniform(0.0, tmax, 300):
        t, w = rys_exact(n, T)
        v = _eval_bins(coefs, tmax, nbin, T)
        errt = max(errt, np.max(np.abs(v[:n] - t)))
        errw = max(errw, np.max(np.abs((v[n:] if n == 1 else np.exp(v[n:])) - w)))
    return dict(n=n, tmax=tmax, nbin=nbin, coefs=coefs, asym=rys_asym(n), errt=errt, errw=errw)


def build_boys(width=0.25, tmax=36.0):
    nbin = int(np.ceil(tmax / width))
    tmax = nbin * width
    cache = {}

    def func(T):
        if T not in cache:
            cache[T] = boys_exact(MMAX_BOYS, T)
        return cache[T]

    coefs = _fit_bins(func, MMAX_BOYS + 1, tmax, nbin)
    rng = np.random.default_rng(7)
    err = 0.0
    for T in rng.uniform(0.0, tmax, 200):
        ex = boys_exact(MMAX_BOYS, T)
        v = _eval_bins(coefs, tmax, nbin, T)
        err = max(err, np.max(np.abs(v - ex)))
    return dict(tmax=tmax, nbin=nbin, coefs=coefs, err=err)


def _fmt(a):
    return ",\n".join(", ".join("%.17e" % v for v in a[i:i + 4]) for i in range(0, len(a), 4))


def write_inc(path, rys_list, boys):
    lines = ["// Generated by lightspeed_b200/tables/gen_tables.py -- do not edit.",
             "// Rys: per nrys, [root][bin][coef] for t, then [root][bin][coef] for ln w",
             "// (for nrys = 1 the weight w itself),",
             "// monomial coefficients c0..c7 of the local variable x in [-1,1].",
             "// Boys: [m][bin][coef] for F_m on [0, BOYS_TMAX).",
             "#pragma once", ""]
    lines.append("#define LSJK_RYS_NMAX %d" % NMAX_RYS)
    lines.append("#define LSJK_BOYS_MMAX %d" % MMAX_BOYS)
    lines.append("#define LSJK_TAB_NCOEF %d" % NCOEF)
    lines.append("static const int    kRysNbin[%d] = {0, %s};" % (NMAX_RYS + 1, ", ".join(str(r["nbin"]) for r in rys_list)))
    lines.append("static const double kRysTmax[%d] = {0.0, %s};" % (NMAX_RYS + 1, ", ".join("%.17e" % r["tmax"] for r in rys_list)))
    off = [0]
    for r in rys_list:
        off.append(off[-1] + 2 * r["n"] * r["nbin"] * NCOEF)
    lines.append("static const long   kRysOffset[%d] = {0, %s};" % (NMAX_RYS + 2, ", ".join(str(o) for o in off)))
    allc = np.concatenate([np.concatenate([r["coefs"][:r["n"]].ravel(), r["coefs"][r["n"]:].ravel()]) for r in rys_list])
    lines.append("static const double kRysCoef[%d] = {\n%s};" % (len(allc), _fmt(allc)))
    asym_t = np.zeros((NMAX_RYS + 1, NMAX_RYS))
    asym_w = np.zeros((NMAX_RYS + 1, NMAX_RYS))
    for r in rys_list:
        s, h = r["asym"]
        asym_t[r["n"], :r["n"]] = s
        asym_w[r["n"], :r["n"]] = h
    lines.append("static const double kRysAsymT[%d] = {\n%s};" % (asym_t.size, _fmt(asym_t.ravel())))
    lines.append("static const double kRysAsymW[%d] = {\n%s};" % (asym_w.size, _fmt(asym_w.ravel())))
    # the same nodes as initializer lists, for constant-memory copies in device code
    lines.append("#define LSJK_RYS_ASYM_T_LIST \\\n%s" % " \\\n".join(
        ", ".join("%.17e" % v for v in asym_t.ravel()[i:i + 4]) + ("," if i + 4 < asym_t.size else "")
        for i in range(0, asym_t.size, 4)))
    lines.append("#define LSJK_RYS_ASYM_W_LIST \\\n%s" % " \\\n".join(
        ", ".join("%.17e" % v for v in asym_w.ravel()[i:i + 4]) + ("," if i + 4 < asym_w.size else "")
        for i in range(0, asym_w.size, 4)))
    lines.append("#define LSJK_BOYS_NBIN %d" % boys["nbin"])
    lines.append("#define LSJK_BOYS_TMAX %.17e" % boys["tmax"])
    lines.append("static const double kBoysCoef[%d] = {\n%s};" % (boys["coefs"].size, _fmt(boys["coefs"].ravel())))
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def main():
    out = os.path.join(os.path.dirname(__file__), "..", "csrc", "tables", "quad_tables.inc")
    os.makedirs(os.path.dirname(out), exist_ok=True)
    rys_list = []
    for n in range(1, NMAX_RYS + 1):
        # bin width per rule: the one- and two-point rules vary fastest
        r = build_rys(n, 0.4 if n <= 2 else 0.6)
        print("rys n=%d tasym=%.1f nbin=%d err_t=%.2e err_w=%.2e" % (n, r["tmax"], r["nbin"], r["errt"], r["errw"]))
        sys.stdout.flush()
        rys_list.append(r)
    boys = build_boys()
    print("boys nbin=%d tmax=%.1f err=%.2e" % (boys["nbin"], boys["tmax"], boys["err"]))
    write_inc(out, rys_list, boys)
    print("wrote", os.path.normpath(out))


if __name__ == "__main__":
    main()
