"""Batched densities: IntBox.coulombMulti / exchangeMulti with several
densities in one call against one call per density.

A batched J launch shares its quartet loop between up to four densities and
screens with the largest |D| of the batch, so it evaluates a superset of each
density's quartets: results agree with the per-density builds to the size of
the quartets the single-density screen drops. At thresp = 1e-14 that is far
below the 1e-10 elementwise FP64 tolerance. In mixed precision the batch also
moves some quartets from FP32 to FP64 (the estimate uses the batch's largest
|D|), so there the check is the mixed-precision tolerance (1e-6 against the
FP64 result) of the other mixed tests. The densities are non-symmetric rank-3
products (the shape of response trial vectors); the bare Coulomb operator and
erf-attenuated interactions (omega = 0.3) are both covered."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _system(ls):
    from lightspeed_b200.geometry import water_cluster
    bas = ls.Basis.from_gbs_file(water_cluster(4, seed=3), "6-31gs")
    pl = ls.PairList.build_schwarz(bas, bas, True, 1e-14)
    return bas, pl


def _densities(n, nao, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        X = rng.standard_normal((nao, 3)) / np.sqrt(nao)
        Y = rng.standard_normal((nao, 3)) / np.sqrt(nao)
        out.append(X @ Y.T)
    return out


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("ndens", [1, 3, 6])
@pytest.mark.parametrize("ewald", [([1.0], [-1.0]), ([1.0], [0.3])])
def test_multi_matches_single(ls, prec, ndens, ewald):
    ls.set_precision(ls.PREC_FP64 if prec == "fp64" else ls.PREC_MIXED)
    try:
        bas, pl = _system(ls)
        res = ls.ResourceList.build()
        ew = ls.Ewald(*ewald)
        Ds = [ls.Tensor.array(D) for D in _densities(ndens, bas.nao, 7 + ndens)]
        thresp = 1e-14
        thredp = thresp if prec == "fp64" else 1e-5
        tol = 1e-10 if prec == "fp64" else 1e-6
        Jm = ls.IntBox.coulombMulti(res, ew, pl, pl, Ds, thresp, thredp)
        Km = ls.IntBox.exchangeMulti(res, ew, pl, pl, Ds, False, thresp, thredp)
        assert len(Jm) == ndens and len(Km) == ndens
        ls.set_precision(ls.PREC_FP64)
        for D, J, K in zip(Ds, Jm, Km):
            J1 = ls.IntBox.coulomb(res, ew, pl, pl, D, thresp, thresp)
            K1 = ls.IntBox.exchange(res, ew, pl, pl, D, False, thresp, thresp)
            assert np.max(abs(J.np - J1.np)) < tol
            assert np.max(abs(K.np - K1.np)) < tol
    finally:
        ls.set_precision(ls.PREC_MIXED)


def test_multi_fp64_vs_oracle(ls):
    """Four densities batched in FP64 against the oracle, one density at a time."""
    from oracle import ref
    if not ref.available():
        pytest.skip("reference CPU IntBox not built")
    ls.set_precision(ls.PREC_FP64)
    try:
        bas, pl = _system(ls)
        res = ls.ResourceList.build()
        ew = ls.Ewald([1.0], [-1.0])
        Dn = _densities(4, bas.nao, 11)
        Jm = ls.IntBox.coulombMulti(res, ew, pl, pl, [ls.Tensor.array(D) for D in Dn], 1e-14, 1e-14)
        rb = ref.RefBasis(ref.prim_arrays(bas))
        rp = ref.RefPairs(rb, rb, True, 1e-14)
        for D, J in zip(Dn, Jm):
            Jr = ref.coulomb(rp, rp, D, 1e-14, 1e-14)
            assert np.max(abs(J.np - Jr)) < 1e-10
    finally:
        ls.set_precision(ls.PREC_MIXED)
