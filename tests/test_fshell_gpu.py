"""f shells: classes with an f shell run the loop form of the quartet code
(quartet_loops.cuh) inside the same J/K kernels, one-electron kernels and
gradients as the lighter classes. Checked against the oracle (the reference CPU
IntBox, which takes any angular momentum) on a water dimer in cc-pVTZ
(spherical f on oxygen, d on hydrogen) and in a Cartesian copy of it:

* pair list identical, J, symmetric and non-symmetric K elementwise 1e-10
  (FP64), 1e-6 in mixed precision at thredp 1e-6;
* range-separated J and K (erf-attenuated and a two-term operator) at 1e-10;
* S, T at 1e-12 and V at 1e-10;
* the J and K gradients at 1e-9 (K: the fully symmetric routine, the mirror
  halving of two symmetric densities, and the unpromised path);
* non-symmetric pair lists between cc-pVTZ and cc-pVDZ at 1e-10, and K over
  merged s exponents within 1e-9 of the exact K;
* six densities in one build and IntBox.eriJ at 1e-10."""
import numpy as np
import pytest

from oracle import ref

pytestmark = pytest.mark.gpu


def _dimer(ls, spherical=None):
    from lightspeed_b200.geometry import water_cluster
    mol = water_cluster(2, seed=1)
    bas = ls.Basis.from_gbs_file(mol, "cc-pvtz", spherical=spherical)
    return mol, bas


def _densities(bas, seed):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((bas.nao, 10)) / np.sqrt(bas.nao)
    Y = rng.standard_normal((bas.nao, 10)) / np.sqrt(bas.nao)
    D = X @ X.T
    Dn = D + 0.05 * (X @ Y.T)
    return D, Dn


@pytest.fixture(scope="module")
def oracle_ok():
    if not ref.available():
        pytest.skip("oracle/_ref not built")


@pytest.mark.parametrize("spherical", [None, False])
def test_fshell_jk_vs_oracle(ls, oracle_ok, spherical):
    mol, bas = _dimer(ls, spherical)
    assert max(p.L for p in bas.primitives) == 3
    res = ls.ResourceList.build()
    ew = ls.Ewald.coulomb()
    pl = ls.PairList.build_schwarz(bas, bas, True, 1e-14)
    rb = ref.RefBasis(ref.prim_arrays(bas))
    rp = ref.RefPairs(rb, rb, True, 1e-14)
    got = [(l.L1, l.L2, p.prim1.primIdx, p.prim2.primIdx, p.bound) for l in pl.pairlists for p in l.pairs]
    L1, L2, p1, p2, b = rp.export()
    assert np.array_equal(np.array([x[:4] for x in got]), np.stack([L1, L2, p1, p2], 1))
    gb = np.array([x[4] for x in got], np.float32)
    assert np.all(np.abs(gb.view(np.int32) - b.view(np.int32)) <= 1)
    D, Dn = _densities(bas, 7)
    J = ls.IntBox.coulomb(res, ew, pl, pl, ls.Tensor.array(D), 1e-14, 1e-14).np
    Jr = ref.coulomb(rp, rp, D, 1e-14, 1e-14)
    assert np.max(np.abs(Jr)) > 1.0
    assert np.max(np.abs(J - Jr)) < 1e-10
    K = ls.IntBox.exchange(res, ew, pl, pl, ls.Tensor.array(D), True, 1e-14, 1e-14).np
    assert np.max(np.abs(K - ref.exchange(rp, rp, D, True, 1e-14, 1e-14))) < 1e-10
    Kn = ls.IntBox.exchange(res, ew, pl, pl, ls.Tensor.array(Dn), False, 1e-14, 1e-14).np
    assert np.max(np.abs(Kn - ref.exchange(rp, rp, Dn, False, 1e-14, 1e-14))) < 1e-10
    # mixed precision: FP32 below thredp, FP64 accumulation
    Jm = ls.IntBox.coulomb(res, ew, pl, pl, ls.Tensor.array(D), 1e-14, 1e-6).np
    Km = ls.IntBox.exchange(res, ew, pl, pl, ls.Tensor.array(D), True, 1e-14, 1e-6).np
    assert np.max(np.abs(Jm - Jr)) < 1e-6
    assert np.max(np.abs(Km - K)) < 1e-6


def test_fshell_range_separated(ls, oracle_ok):
    mol, bas = _dimer(ls)
    res = ls.ResourceList.build()
    pl = ls.PairList.build_schwarz(bas, bas, True, 1e-14)
    rb = ref.RefBasis(ref.prim_arrays(bas))
    rp = ref.RefPairs(rb, rb, True, 1e-14)
    D, _ = _densities(bas, 8)
    for sc, om in (([1.0], [0.4]), ([0.6, 0.4], [-1.0, 0.3])):
        ew = ls.Ewald(sc, om)
        J = ls.IntBox.coulomb(res, ew, pl, pl, ls.Tensor.array(D), 1e-14, 1e-14).np
        assert np.max(np.abs(J - ref.coulomb(rp, rp, D, 1e-14, 1e-14, sc, om))) < 1e-10
        K = ls.IntBox.exchange(res, ew, pl, pl, ls.Tensor.array(D), True, 1e-14, 1e-14).np
        assert np.max(np.abs(K - ref.exchange(rp, rp, D, True, 1e-14, 1e-14, sc, om))) < 1e-10


def test_fshell_one_electron(ls, oracle_ok):
    mol, bas = _dimer(ls)
    res = ls.ResourceList.build()
    pl = ls.PairList.build_schwarz(bas, bas, True, 1e-14)
    rb = ref.RefBasis(ref.prim_arrays(bas))
    rp = ref.RefPairs(rb, rb, True, 1e-14)
    assert np.max(np.abs(ls.IntBox.overlap(res, pl).np - ref.overlap(rp))) < 1e-12
    assert np.max(np.abs(ls.IntBox.kinetic(res, pl).np - ref.kinetic(rp))) < 1e-12
    V = ls.IntBox.potential(res, ls.Ewald.coulomb(), pl, ls.Tensor.array(mol.xyzZ)).np
    assert np.max(np.abs(V - ref.potential(rp, mol.xyzZ))) < 1e-10


def test_fshell_coulomb_grad(ls, oracle_ok):
    mol, bas = _dimer(ls)
    res = ls.ResourceList.build()
    pl = ls.PairList.build_schwarz(bas, bas, True, 1e-14)
    rb = ref.RefBasis(ref.prim_arrays(bas))
    rp = ref.RefPairs(rb, rb, True, 1e-14)
    D, _ = _densities(bas, 9)
    _, Db = _densities(bas, 10)
    Db = 0.5 * (Db + Db.T)
    A, B = ls.Tensor.array(D), ls.Tensor.array(Db)
    G = ls.IntBox.coulombGrad(res, ls.Ewald.coulomb(), pl, A, B, 1e-14, 1e-14).np
    Gr = ref.coulomb_grad(rp, D, Db, 1e-14, 1e-14)
    assert np.max(np.abs(Gr)) > 1e-3
    assert np.max(np.abs(G - Gr)) < 1e-9


def test_fshell_exchange_grad(ls, oracle_ok):
    mol, bas = _dimer(ls)
    res = ls.ResourceList.build()
    ew = ls.Ewald.coulomb()
    pl = ls.PairList.build_schwarz(bas, bas, True, 1e-14)
    rb = ref.RefBasis(ref.prim_arrays(bas))
    rp = ref.RefPairs(rb, rb, True, 1e-14)
    Da, _ = _densities(bas, 11)
    Db, _ = _densities(bas, 12)
    A, B = ls.Tensor.array(Da), ls.Tensor.array(Db)
    G_same = ls.IntBox.exchangeGrad(res, ew, pl, A, A, True, True, True, 1e-14, 1e-14).np
    Gr_same = ref.exchange_grad(rp, Da, None, True, True, 1e-14, 1e-14)
    assert np.max(np.abs(Gr_same)) > 1e-3
    assert np.max(np.abs(G_same - Gr_same)) < 1e-9
    G_ab = ls.IntBox.exchangeGrad(res, ew, pl, A, B, True, True, False, 1e-14, 1e-14).np
    Gr_ab = ref.exchange_grad(rp, Da, Db, True, True, 1e-14, 1e-14)
    assert np.max(np.abs(G_ab - Gr_ab)) < 1e-9
    G_nosym = ls.IntBox.exchangeGrad(res, ew, pl, A, B, False, False, False, 1e-14, 1e-14).np
    assert np.max(np.abs(G_nosym - Gr_ab)) < 1e-9


def test_fshell_mixed_basis(ls, oracle_ok):
    """Non-symmetric pair lists between cc-pVTZ (f) and cc-pVDZ on the same dimer:
    J and K with a rectangular and a symmetric density against the oracle."""
    from lightspeed_b200.geometry import water_cluster
    mol = water_cluster(2, seed=1)
    b1 = ls.Basis.from_gbs_file(mol, "cc-pvtz")
    b2 = ls.Basis.from_gbs_file(mol, "cc-pvdz")
    res = ls.ResourceList.build()
    ew = ls.Ewald.coulomb()
    p11 = ls.PairList.build_schwarz(b1, b1, True, 1e-14)
    p12 = ls.PairList.build_schwarz(b1, b2, False, 1e-14)
    r1, r2 = ref.RefBasis(ref.prim_arrays(b1)), ref.RefBasis(ref.prim_arrays(b2))
    rp11 = ref.RefPairs(r1, r1, True, 1e-14)
    rp12 = ref.RefPairs(r1, r2, False, 1e-14)
    rng = np.random.default_rng(13)
    X = rng.standard_normal((b1.nao, 8)) / np.sqrt(b1.nao)
    Y = rng.standard_normal((b2.nao, 8)) / np.sqrt(b2.nao)
    D12 = X @ Y.T
    J = ls.IntBox.coulomb(res, ew, p11, p12, ls.Tensor.array(D12), 1e-14, 1e-14).np
    assert np.max(np.abs(J - ref.coulomb(rp11, rp12, D12, 1e-14, 1e-14))) < 1e-10
    D22 = Y @ Y.T
    K = ls.IntBox.exchange(res, ew, p12, p12, ls.Tensor.array(D22), True, 1e-14, 1e-14).np
    assert np.max(np.abs(K - ref.exchange(rp12, rp12, D22, True, 1e-14, 1e-14))) < 1e-10


def test_fshell_merged_exponents(ls, oracle_ok):
    """K over merged s exponents (cc-pVTZ repeats s exponents across contracted
    shells; the twin classes with an f shell run the two-target kernels): within
    1e-9 of the oracle's exact K, symmetric and non-symmetric."""
    mol, bas = _dimer(ls)
    res = ls.ResourceList.build()
    ew = ls.Ewald.coulomb()
    pl = ls.PairList.build_schwarz(bas, bas, True, 1e-14)
    rb = ref.RefBasis(ref.prim_arrays(bas))
    rp = ref.RefPairs(rb, rb, True, 1e-14)
    D, Dn = _densities(bas, 14)
    ls.set_merge(True)
    try:
        K = ls.IntBox.exchange(res, ew, pl, pl, ls.Tensor.array(D), True, 1e-14, 1e-14).np
        Kn = ls.IntBox.exchange(res, ew, pl, pl, ls.Tensor.array(Dn), False, 1e-14, 1e-14).np
    finally:
        ls.set_merge(False)
    assert np.max(np.abs(K - ref.exchange(rp, rp, D, True, 1e-14, 1e-14))) < 1e-9
    assert np.max(np.abs(Kn - ref.exchange(rp, rp, Dn, False, 1e-14, 1e-14))) < 1e-9


def test_fshell_multi_density_and_eriJ(ls, oracle_ok):
    """Six non-symmetric densities in one build (J: CTA z-slices; K: density groups
    and sub-slots, the warp kernel included) and IntBox.eriJ over the same basis,
    against the oracle."""
    mol, bas = _dimer(ls)
    res = ls.ResourceList.build()
    ew = ls.Ewald.coulomb()
    pl = ls.PairList.build_schwarz(bas, bas, True, 1e-14)
    rb = ref.RefBasis(ref.prim_arrays(bas))
    rp = ref.RefPairs(rb, rb, True, 1e-14)
    rng = np.random.default_rng(21)
    Dn = []
    for _ in range(6):
        X = rng.standard_normal((bas.nao, 4)) / np.sqrt(bas.nao)
        Y = rng.standard_normal((bas.nao, 4)) / np.sqrt(bas.nao)
        Dn.append(X @ Y.T)
    ls.set_precision(ls.PREC_FP64)
    try:
        Ds = [ls.Tensor.array(D) for D in Dn]
        Jm = ls.IntBox.coulombMulti(res, ew, pl, pl, Ds, 1e-14, 1e-14)
        Km = ls.IntBox.exchangeMulti(res, ew, pl, pl, Ds, False, 1e-14, 1e-14)
        C = rng.standard_normal((bas.nao, 3)) / np.sqrt(bas.nao)
        A = ls.Tensor.array(C)
        I = ls.IntBox.eriJ(res, ew, pl, pl, A, A, A, A, 1e-14, 1e-14).np.copy()
    finally:
        ls.set_precision(ls.PREC_MIXED)
    for D, J, K in zip(Dn, Jm, Km):
        assert np.max(np.abs(J.np - ref.coulomb(rp, rp, D, 1e-14, 1e-14))) < 1e-10
        assert np.max(np.abs(K.np - ref.exchange(rp, rp, D, False, 1e-14, 1e-14))) < 1e-10
    Iref = ref.eri_j(rp, rp, C, C, C, C, 1e-14, 1e-14, True, True, True)
    assert np.max(np.abs(I - Iref)) < 1e-10
