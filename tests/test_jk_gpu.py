"""Parity of the sm_100a J/K path with the oracle (the reference CPU IntBox)
and the reference's own golden vectors. All calls go through the product API
(lightspeed_b200 -> liblsjk.so C ABI). FP64 mode: elementwise tolerance 1e-10
against the oracle on the same pair list and thresholds; the reference's own
test tolerances (1e-9 prop, 1e-12 Ewald/mixed-basis) on its golden vectors."""
import os

import numpy as np
import pytest

from oracle import ref

pytestmark = pytest.mark.gpu

EWALD = {"LR": ([1.0], [0.3]), "LR2": ([0.7, 0.7, 0.7], [0.2, 0.1, 0.05]), "SR": ([-0.7, 0.7], [0.3, -1.0]),
         "SR2": ([-0.7, 0.7], [-1.0, -1.0]), "MIX": ([0.8, 0.2], [0.2, -1.0])}


@pytest.fixture(scope="module", autouse=True)
def fp64(ls):
    ls.set_precision(ls.PREC_FP64)
    yield
    ls.set_precision(ls.PREC_MIXED)


def _h2o(ls, golden_dir, basis):
    mol = ls.Molecule.from_xyz_file(os.path.join(golden_dir, "h2o.xyz"))
    return ls.Basis.from_gbs_file(mol, basis)


@pytest.mark.parametrize("basis", ["sto-3g", "6-31gs", "cc-pvdz"])
@pytest.mark.parametrize("symm", [True, False])
def test_pairlist_matches_reference(ls, golden_dir, basis, symm):
    bas = _h2o(ls, golden_dir, basis)
    pl = ls.PairList.build_schwarz(bas, bas, symm, 1e-14)
    got = [(l.L1, l.L2, p.prim1.primIdx, p.prim2.primIdx, p.bound) for l in pl.pairlists for p in l.pairs]
    if ref.available():
        rb = ref.RefBasis(ref.prim_arrays(bas))
        L1, L2, p1, p2, b = ref.RefPairs(rb, rb, symm, 1e-14).export()
        assert len(got) == len(L1)
        g = np.array([x[:4] for x in got])
        assert np.array_equal(g, np.stack([L1, L2, p1, p2], 1))
        gb = np.array([x[4] for x in got], np.float32)
        # float bounds agree to the last bit except where exp/pow round differently (<= 1 ulp)
        assert np.all(np.abs(gb.view(np.int32) - b.view(np.int32)) <= 1)


@pytest.mark.parametrize("basis", ["sto-3g", "6-31gs", "cc-pvdz"])
@pytest.mark.parametrize("symm", [True, False])
def test_prop_golden(ls, golden_dir, basis, symm):
    bas = _h2o(ls, golden_dir, basis)
    z = np.load(os.path.join(golden_dir, "ref_prop_h2o_%s.npz" % basis))
    res = ls.ResourceList.build()
    ew = ls.Ewald([1.0], [-1.0])
    pl = ls.PairList.build_schwarz(bas, bas, symm, 1e-14)
    D, D2 = ls.Tensor.array(z["D"]), ls.Tensor.array(z["D2"])
    J = ls.IntBox.coulomb(res, ew, pl, pl, D, 1e-14, 1e-14)
    assert np.max(abs(J.np - z["J"])) < 1e-9
    # accumulate into the passed tensor (same object returned)
    J2 = ls.IntBox.coulomb(res, ew, pl, pl, D, 1e-14, 1e-14, J)
    assert J2 is J or np.shares_memory(J2.np, J.np)
    assert np.max(abs(J.np - 2 * z["J"])) < 2e-9
    assert np.max(abs(ls.IntBox.coulomb(res, ew, pl, pl, D2, 1e-14, 1e-14).np - z["J2"])) < 1e-9
    assert np.max(abs(ls.IntBox.exchange(res, ew, pl, pl, D, True, 1e-14, 1e-14).np - z["K"])) < 1e-9
    assert np.max(abs(ls.IntBox.exchange(res, ew, pl, pl, D2, False, 1e-14, 1e-14).np - z["K2"])) < 1e-9


@pytest.mark.parametrize("basis", ["sto-3g", "6-31gs", "cc-pvdz"])
@pytest.mark.parametrize("symm", [True, False])
def test_ewald_golden(ls, golden_dir, basis, symm):
    bas = _h2o(ls, golden_dir, basis)
    z = np.load(os.path.join(golden_dir, "ref_ewald_h2o_%s.npz" % basis))
    res = ls.ResourceList.build()
    pl = ls.PairList.build_schwarz(bas, bas, symm, 1e-14)
    for name, (s, o) in EWALD.items():
        ew = ls.Ewald(s, o)
        for dk, jk, kk, symmD in (("D_", "J_", "K_", True), ("D2_", "J2_", "K2_", False)):
            D = ls.Tensor.array(z[dk + name])
            J = ls.IntBox.coulomb(res, ew, pl, pl, D, 1e-14, 1e-14)
            K = ls.IntBox.exchange(res, ew, pl, pl, D, symmD, 1e-14, 1e-14)
            assert np.max(abs(J.np - z[jk + name])) < 1e-12, (name, jk)
            assert np.max(abs(K.np - z[kk + name])) < 1e-12, (name, kk)


def test_mixed_basis_golden(ls, golden_dir):
    """Different bases on bra and ket, non-symmetric pair lists (mix_basis.py)."""
    res = ls.ResourceList.build()
    ew = ls.Ewald([1.0], [-1.0])
    z = np.load(os.path.join(golden_dir, "ref_mix_h2o_nh3.npz"))
    m1 = ls.Molecule.from_xyz_file(os.path.join(golden_dir, "h2o.xyz"))
    m2 = ls.Molecule.from_xyz_file(os.path.join(golden_dir, "nh3.xyz"))
    for a, b in (("sto-3g", "6-31gs"), ("6-31gs", "cc-pvdz")):
        b1 = ls.Basis.from_gbs_file(m1, a)
        b2 = ls.Basis.from_gbs_file(m2, b)
        N1 = b1.nao
        p11 = ls.PairList.build_schwarz(b1, b1, True, 1e-14)
        p12 = ls.PairList.build_schwarz(b1, b2, False, 1e-14)
        p21 = ls.PairList.build_schwarz(b2, b1, False, 1e-14)
        p22 = ls.PairList.build_schwarz(b2, b2, True, 1e-14)
        suf = "_" + a.upper() + "_" + b.upper()
        D12 = ls.Tensor.array(z["D0" + suf][:N1, N1:])
        J0 = z["J0" + suf]
        assert np.max(abs(ls.IntBox.coulomb(res, ew, p11, p12, D12, 1e-14, 1e-14).np - J0[:N1, :N1])) < 1e-12
        assert np.max(abs(ls.IntBox.coulomb(res, ew, p21, p12, D12, 1e-14, 1e-14).np - J0[N1:, :N1])) < 1e-12
        K0 = z["K0" + suf]
        assert np.max(abs(ls.IntBox.exchange(res, ew, p11, p12, D12, False, 1e-14, 1e-14).np - K0[:N1, :N1])) < 1e-12
        assert np.max(abs(ls.IntBox.exchange(res, ew, p21, p22, D12, False, 1e-14, 1e-14).np - K0[N1:, N1:])) < 1e-12
        D22 = ls.Tensor.array(z["D1" + suf][N1:, N1:])
        K1 = z["K1" + suf]
        assert np.max(abs(ls.IntBox.exchange(res, ew, p12, p22, D22, True, 1e-14, 1e-14).np - K1[:N1, N1:])) < 1e-12


def test_water8_vs_oracle_fixture(ls, golden_dir):
    """8 H2O / 6-31G*, Schwarz 1e-12: elementwise 1e-10 against the oracle."""
    from lightspeed_b200.geometry import water_cluster
    z = np.load(os.path.join(golden_dir, "oracle_w8.npz"))
    mol = water_cluster(8, seed=0)
    assert np.allclose(mol.xyz, z["xyz"], atol=0, rtol=0)
    bas = ls.Basis.from_gbs_file(mol, "6-31gs")
    res = ls.ResourceList.build()
    ew = ls.Ewald.coulomb()
    pl = ls.PairList.build_schwarz(bas, bas, True, 1e-12)
    D = ls.Tensor.array(z["D"])
    J = ls.IntBox.coulomb(res, ew, pl, pl, D, 1e-12, 1e-12)
    K = ls.IntBox.exchange(res, ew, pl, pl, D, True, 1e-12, 1e-12)
    assert np.max(abs(J.np - z["J"])) < 1e-10
    assert np.max(abs(K.np - z["K"])) < 1e-10


def test_propane_ccpvdz_vs_reference(ls):
    """C3H8 / cc-pVDZ (spherical d on carbon, long contracted s shells): J and K
    of a SAD-like symmetric density elementwise 1e-10 against the reference
    CPU IntBox, symmetric and non-symmetric K."""
    from lightspeed_b200.geometry import alkane
    if not ref.available():
        pytest.skip("reference CPU IntBox not built")
    bas = ls.Basis.from_gbs_file(alkane(3), "cc-pvdz")
    rng = np.random.default_rng(3)
    X = rng.standard_normal((bas.nao, 13)) / np.sqrt(bas.nao)
    D = X @ X.T
    res = ls.ResourceList.build()
    pl = ls.PairList.build_schwarz(bas, bas, True, 1e-14)
    rb = ref.RefBasis(ref.prim_arrays(bas))
    rp = ref.RefPairs(rb, rb, True, 1e-14)
    J = ls.IntBox.coulomb(res, ls.Ewald.coulomb(), pl, pl, ls.Tensor.array(D), 1e-14, 1e-14).np
    assert np.max(abs(J - ref.coulomb(rp, rp, D, 1e-14, 1e-14))) < 1e-10
    K = ls.IntBox.exchange(res, ls.Ewald.coulomb(), pl, pl, ls.Tensor.array(D), True, 1e-14, 1e-14).np
    assert np.max(abs(K - ref.exchange(rp, rp, D, True, 1e-14, 1e-14))) < 1e-10
    Dn = D + 0.05 * np.triu(X @ X[::-1].T)
    Kn = ls.IntBox.exchange(res, ls.Ewald.coulomb(), pl, pl, ls.Tensor.array(Dn), False, 1e-14, 1e-14).np
    assert np.max(abs(Kn - ref.exchange(rp, rp, Dn, False, 1e-14, 1e-14))) < 1e-10


def test_d24symm_requires_equivalent_bases(ls, golden_dir):
    b1 = _h2o(ls, golden_dir, "sto-3g")
    b2 = _h2o(ls, golden_dir, "6-31gs")
    res = ls.ResourceList.build()
    p12 = ls.PairList.build_schwarz(b1, b2, False, 1e-14)
    p11 = ls.PairList.build_schwarz(b1, b1, True, 1e-14)
    D = ls.Tensor.zeros((b2.nao, b1.nao))
    with pytest.raises(RuntimeError, match="D24symm"):
        ls.IntBox.exchange(res, ls.Ewald.coulomb(), p12, p11, D, True, 1e-14, 1e-14)


def test_shape_errors(ls, golden_dir):
    bas = _h2o(ls, golden_dir, "sto-3g")
    res = ls.ResourceList.build()
    pl = ls.PairList.build_schwarz(bas, bas, True, 1e-14)
    with pytest.raises(RuntimeError, match="shape"):
        ls.IntBox.coulomb(res, ls.Ewald.coulomb(), pl, pl, ls.Tensor.zeros((3, 3)), 1e-14, 1e-14)


def test_quartet_sets_equal_reference(ls, golden_dir):
    """The GPU evaluates exactly the reference's quartet set: its per-build
    quartet counters equal the oracle's count of quartets passing the
    reference screening (ket/bra truncation, K-invert thresholds, D24 symmetry)."""
    from lightspeed_b200.geometry import water_cluster
    from oracle import port
    z = np.load(os.path.join(golden_dir, "oracle_w8.npz"))
    bas = ls.Basis.from_gbs_file(water_cluster(8, seed=0), "6-31gs")
    pb = port.Basis(bas.primitives)
    ppl = port.Pairs(pb, pb, True, 1e-12)
    for D, symm in ((z["D"], True), (z["D"] + 0.01 * np.tril(z["D"]), False)):
        nj, nk = port.count_quartets(ppl, ppl, D, D, symm, 1e-12)
        res = ls.ResourceList.build()
        pl = ls.PairList.build_schwarz(bas, bas, True, 1e-12)
        ls.reset_stats()
        ls.IntBox.coulomb(res, ls.Ewald.coulomb(), pl, pl, ls.Tensor.array(D), 1e-12, 1e-12)
        ls.IntBox.exchange(res, ls.Ewald.coulomb(), pl, pl, ls.Tensor.array(D), symm, 1e-12, 1e-12)
        st = ls.stats()
        assert st["j_quartets"] == nj
        assert st["k_quartets"] == nk
