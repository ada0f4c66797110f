"""Accuracy of the device quadrature tables (lightspeed_b200/csrc/tables/
quad_tables.inc, written by lightspeed_b200/tables/gen_tables.py), evaluated
on the CPU exactly the way lsjk_device.cuh evaluates them: bin index
floor(T * nbin / tmax) clamped to the last bin, local variable
x = 2 (u - bin) - 1, Horner over the 8 monomial coefficients, exp of the
interpolated ln w (the one-point rule tabulates w = F_0 itself); the
half-range Gauss-Hermite form at T >= tmax.

* Rys roots and weights against the reference's own tables,
  Rys::compute_t / compute_w (src/lightspeed/rys.hpp:56-153, through
  oracle/_ref), for every rule the kernels use (1..5 roots, classes up to
  (dd|dd)), over [0, 1.3 tmax] including the bin edges.
* The FP32 path's switch: from the last table bin on it uses the FP64
  asymptotic form, which must agree with the reference there.
* Boys F_0..F_16 against mpmath's incomplete gamma function at 30 digits
  (the definition F_m(T) = int_0^1 t^2m exp(-T t^2) dt), over the table range
  and the asymptotic range with the upward recursion.
"""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "lightspeed_b200", "csrc", "tables", "quad_tables.inc")


def _tables():
    if not os.path.exists(INC):
        pytest.skip("quadrature tables not generated (run the build)")
    txt = open(INC).read()

    def arr(name):
        m = re.search(r"%s\[\d+\] = \{(.*?)\};" % name, txt, re.S)
        return np.array([float(v) for v in m.group(1).replace("\n", " ").split(",") if v.strip()])

    def define(name):
        return float(re.search(r"#define %s (\S+)" % name, txt).group(1))

    return {"nbin": arr("kRysNbin").astype(int), "tmax": arr("kRysTmax"), "off": arr("kRysOffset").astype(int),
            "coef": arr("kRysCoef"), "asym_t": arr("kRysAsymT").reshape(10, 9),
            "asym_w": arr("kRysAsymW").reshape(10, 9), "boys": arr("kBoysCoef"),
            "boys_nbin": int(define("LSJK_BOYS_NBIN")), "boys_tmax": define("LSJK_BOYS_TMAX")}


def _horner(c, x):
    f = c[..., 7]
    for k in range(6, -1, -1):
        f = f * x + c[..., k]
    return f


def _bin(T, nbin, tmax):
    u = T * (nbin / tmax)
    b = np.minimum(u.astype(int), nbin - 1)
    return b, 2.0 * (u - b) - 1.0


def rys_device(tab, n, T):
    """(t, w) of the n-point rule as the FP64 device path computes them."""
    nbin, tmax = tab["nbin"][n], tab["tmax"][n]
    blk = tab["coef"][tab["off"][n]:tab["off"][n + 1]].reshape(2 * n, nbin, 8)
    t = np.zeros((len(T), n))
    w = np.zeros((len(T), n))
    lo = T < tmax
    b, x = _bin(T[lo], nbin, tmax)
    for i in range(n):
        t[lo, i] = _horner(blk[i, b], x)
        lw = _horner(blk[n + i, b], x)
        w[lo, i] = lw if n == 1 else np.exp(lw)   # the one-point rule tabulates w itself
    r = 1.0 / np.sqrt(T[~lo])
    t[~lo] = tab["asym_t"][n, :n] * r[:, None]
    w[~lo] = tab["asym_w"][n, :n] * r[:, None]
    return t, w


def _sample(tmax, nbin):
    edges = np.arange(nbin + 1) * (tmax / nbin)
    rng = np.random.default_rng(3)
    return np.unique(np.concatenate([[0.0, 1e-12, 1e-6], edges, edges + 1e-9, rng.uniform(0, 1.3 * tmax, 400),
                                     [1.3 * tmax, 200.0, 1e4]]))


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5])
def test_rys_tables_match_reference(n):
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref (reference CPU IntBox) not built")
    tab = _tables()
    T = _sample(tab["tmax"][n], tab["nbin"][n])
    t, w = rys_device(tab, n, T)
    tr, wr = ref.rys(n, T)
    # roots are in (0, 1); weights sum to F_0(T) <= 1: compare absolutely and relatively
    assert np.max(np.abs(t - tr)) < 5e-13
    assert np.max(np.abs(w - wr) / np.maximum(wr, 1e-300)) < 5e-12
    assert np.max(np.abs(w - wr)) < 5e-14


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5])
def test_rys_fp32_switch_region_is_fp64_asymptote(n):
    """From the start of the last bin the FP32 pass uses the FP64 asymptotic
    form (kkernel.cuh); there it must agree with the reference's rule to far
    better than FP32 resolution."""
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref (reference CPU IntBox) not built")
    tab = _tables()
    nbin, tmax = tab["nbin"][n], tab["tmax"][n]
    T = np.linspace(tmax - tmax / nbin, 2.0 * tmax, 97)
    r = 1.0 / np.sqrt(T)
    t = tab["asym_t"][n, :n] * r[:, None]
    w = tab["asym_w"][n, :n] * r[:, None]
    tr, wr = ref.rys(n, T)
    assert np.max(np.abs(t - tr) / tr) < 1e-11
    assert np.max(np.abs(w - wr) / wr) < 1e-11


def test_rys_fp32_tables_below_switch():
    """The FP32 copy of the tables, evaluated in FP32 below the last bin,
    stays within FP32 resolution of the reference."""
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref (reference CPU IntBox) not built")
    tab = _tables()
    for n in range(1, 6):
        nbin, tmax = tab["nbin"][n], tab["tmax"][n]
        blk = tab["coef"][tab["off"][n]:tab["off"][n + 1]].reshape(2 * n, nbin, 8).astype(np.float32)
        T = np.linspace(0.0, tmax - tmax / nbin, 301, endpoint=False).astype(np.float32)
        u = T * np.float32(nbin / np.float32(tmax))
        b = np.minimum(u.astype(int), nbin - 1)
        x = (np.float32(2) * (u - b.astype(np.float32)) - np.float32(1)).astype(np.float32)
        tr, wr = ref.rys(n, T.astype(np.float64))
        for i in range(n):
            t = _horner(blk[i, b], x).astype(np.float32)
            lw = _horner(blk[n + i, b], x).astype(np.float32)
            w = lw if n == 1 else np.exp(lw)
            assert np.max(np.abs(t - tr[:, i])) < 2e-6
            assert np.max(np.abs(w - wr[:, i]) / wr[:, i]) < 2e-5


def _boys_exact(mmax, T):
    import mpmath as mp
    mp.mp.dps = 30
    out = np.zeros(mmax + 1)
    for m in range(mmax + 1):
        if T == 0.0:
            out[m] = 1.0 / (2 * m + 1)
        else:
            a = mp.mpf(m) + mp.mpf(1) / 2
            out[m] = float(mp.gammainc(a, 0, mp.mpf(T)) / (2 * mp.mpf(T) ** a))
    return out


def boys_device(tab, L, T):
    """F_0..F_L as boys_eval<L, double> computes them."""
    nbin, tmax = tab["boys_nbin"], tab["boys_tmax"]
    F = np.zeros(L + 1)
    if T < tmax:
        b, x = _bin(np.array([T]), nbin, tmax)
        F[L] = _horner(tab["boys"].reshape(-1, nbin, 8)[L, b[0]], x[0])
        e = np.exp(-T)
        for m in range(L - 1, -1, -1):
            F[m] = (2 * T * F[m + 1] + e) * (1.0 / (2 * m + 1))
    else:
        r = 1.0 / np.sqrt(T)
        F[0] = 0.88622692545275801364908374167057259 * r
        e = np.exp(-T)
        for m in range(L):
            F[m + 1] = ((2 * m + 1) * F[m] - e) * 0.5 * r * r
    return F


def test_boys_tables_match_mpmath():
    pytest.importorskip("mpmath")
    tab = _tables()
    rng = np.random.default_rng(11)
    Ts = np.concatenate([[0.0, 1e-9, tab["boys_tmax"] - 1e-9, tab["boys_tmax"]], rng.uniform(0, 36, 40),
                         rng.uniform(36, 120, 10)])
    worst = 0.0
    for T in Ts:
        ex = _boys_exact(8, T)
        for L in (0, 1, 2, 4, 8):
            F = boys_device(tab, L, T)
            worst = max(worst, float(np.max(np.abs(F - ex[:L + 1]) / ex[:L + 1])))
    # relative accuracy of the FP64 path, the J kernels' Boys values (L <= 8)
    assert worst < 5e-14, worst
