"""Nuclear gradients of the J and K energies on the GPU (IntBox.coulombGrad,
IntBox.exchangeGrad) against the reference: its golden vectors
(tests/coverage/prop_int.py:142-214, keys Jgr..Jgr4 and Kgr..Kgr4 -- equal
and different densities, symmetric and not, tolerance 1e-9) and the oracle's
coulombGrad / exchangeGrad (the reference CPU code, oracle/_ref) on 8 H2O /
6-31G* and propane / cc-pVDZ (spherical d), with accumulation into a passed G."""
import os

import numpy as np
import pytest

from oracle import ref

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _fp64(ls):
    ls.set_precision(ls.PREC_FP64)
    yield
    ls.set_precision(ls.PREC_MIXED)


@pytest.mark.parametrize("basis", ["sto-3g", "6-31gs", "cc-pvdz"])
def test_coulomb_grad_golden(ls, golden_dir, basis):
    mol = ls.Molecule.from_xyz_file(os.path.join(golden_dir, "h2o.xyz"))
    bas = ls.Basis.from_gbs_file(mol, basis)
    z = np.load(os.path.join(golden_dir, "ref_prop_h2o_%s.npz" % basis))
    res = ls.ResourceList.build()
    ew = ls.Ewald.coulomb()
    pl = ls.PairList.build_schwarz(bas, bas, True, 1e-14)
    D, D2 = ls.Tensor.array(z["D"]), ls.Tensor.array(z["D2"])
    G = ls.IntBox.coulombGrad(res, ew, pl, D, D, 1e-14, 1e-14)
    assert G.shape == (3, 3)
    assert np.max(np.abs(G.np - z["Jgr"])) < 1e-9
    # accumulates into the passed G
    G2 = ls.IntBox.coulombGrad(res, ew, pl, D, D, 1e-14, 1e-14, G)
    assert np.max(np.abs(G2.np - 2.0 * z["Jgr"])) < 2e-9
    assert np.max(np.abs(ls.IntBox.coulombGrad(res, ew, pl, D2, D2, 1e-14, 1e-14).np - z["Jgr2"])) < 1e-9
    assert np.max(np.abs(ls.IntBox.coulombGrad(res, ew, pl, D, D2, 1e-14, 1e-14).np - z["Jgr3"])) < 1e-9
    assert np.max(np.abs(ls.IntBox.coulombGrad(res, ew, pl, D2, D, 1e-14, 1e-14).np - z["Jgr4"])) < 1e-9


def _oracle_case(ls, mol, basis, seed):
    bas = ls.Basis.from_gbs_file(mol, basis)
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((bas.nao, 8)) / np.sqrt(bas.nao)
    Y = rng.standard_normal((bas.nao, 8)) / np.sqrt(bas.nao)
    return bas, X @ X.T, Y @ Y.T


@pytest.mark.parametrize("case", ["water8", "propane"])
def test_coulomb_grad_vs_oracle(ls, case):
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    from lightspeed_b200.geometry import alkane, water_cluster
    if case == "water8":
        bas, Da, Db = _oracle_case(ls, water_cluster(8, seed=0), "6-31gs", 3)
        thre = 1e-12
    else:
        bas, Da, Db = _oracle_case(ls, alkane(3), "cc-pvdz", 4)
        thre = 1e-14
    res = ls.ResourceList.build()
    ew = ls.Ewald.coulomb()
    pl = ls.PairList.build_schwarz(bas, bas, True, thre)
    rb = ref.RefBasis(ref.prim_arrays(bas))
    rp = ref.RefPairs(rb, rb, True, thre)
    A, B = ls.Tensor.array(Da), ls.Tensor.array(Db)
    G_same = ls.IntBox.coulombGrad(res, ew, pl, A, A, thre, thre).np
    G_ab = ls.IntBox.coulombGrad(res, ew, pl, A, B, thre, thre).np
    Gr_same = ref.coulomb_grad(rp, Da, None, thre, thre)
    Gr_ab = ref.coulomb_grad(rp, Da, Db, thre, thre)
    assert np.max(np.abs(Gr_same)) > 1e-3
    assert np.max(np.abs(G_same - Gr_same)) < 1e-9
    assert np.max(np.abs(G_ab - Gr_ab)) < 1e-9
    # translational invariance of the energy: the gradient sums to zero
    assert np.max(np.abs(G_ab.sum(axis=0))) < 1e-9


def test_coulomb_grad_range_separated(ls, golden_dir):
    """erf-attenuated operator (omega = 0.3) against the oracle."""
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    mol = ls.Molecule.from_xyz_file(os.path.join(golden_dir, "h2o.xyz"))
    bas = ls.Basis.from_gbs_file(mol, "cc-pvdz")
    z = np.load(os.path.join(golden_dir, "ref_prop_h2o_cc-pvdz.npz"))
    res = ls.ResourceList.build()
    ew = ls.Ewald([1.0], [0.3])
    pl = ls.PairList.build_schwarz(bas, bas, True, 1e-14)
    rb = ref.RefBasis(ref.prim_arrays(bas))
    rp = ref.RefPairs(rb, rb, True, 1e-14)
    G = ls.IntBox.coulombGrad(res, ew, pl, ls.Tensor.array(z["D"]), ls.Tensor.array(z["D2"]), 1e-14, 1e-14).np
    Gr = ref.coulomb_grad(rp, z["D"], z["D2"], 1e-14, 1e-14, [1.0], [0.3])
    assert np.max(np.abs(G - Gr)) < 1e-9


def test_coulomb_grad_needs_symmetric_pairlist(ls, golden_dir):
    mol = ls.Molecule.from_xyz_file(os.path.join(golden_dir, "h2o.xyz"))
    bas = ls.Basis.from_gbs_file(mol, "sto-3g")
    res = ls.ResourceList.build()
    pl = ls.PairList.build_schwarz(bas, bas, False, 1e-14)
    D = ls.Tensor.array(np.eye(bas.nao))
    with pytest.raises(RuntimeError, match="symmetric"):
        ls.IntBox.coulombGrad(res, ls.Ewald.coulomb(), pl, D, D, 1e-14, 1e-14)


@pytest.mark.parametrize("basis", ["sto-3g", "6-31gs", "cc-pvdz"])
def test_exchange_grad_golden(ls, golden_dir, basis):
    mol = ls.Molecule.from_xyz_file(os.path.join(golden_dir, "h2o.xyz"))
    bas = ls.Basis.from_gbs_file(mol, basis)
    z = np.load(os.path.join(golden_dir, "ref_prop_h2o_%s.npz" % basis))
    res = ls.ResourceList.build()
    ew = ls.Ewald.coulomb()
    pl = ls.PairList.build_schwarz(bas, bas, True, 1e-14)
    D, D2 = ls.Tensor.array(z["D"]), ls.Tensor.array(z["D2"])
    # the reference's four calls (prop_int.py:178-211)
    G = ls.IntBox.exchangeGrad(res, ew, pl, D, D, True, True, True, 1e-14, 1e-14)
    assert G.shape == (3, 3)
    assert np.max(np.abs(G.np - z["Kgr"])) < 1e-9
    G2 = ls.IntBox.exchangeGrad(res, ew, pl, D, D, True, True, True, 1e-14, 1e-14, G)
    assert np.max(np.abs(G2.np - 2.0 * z["Kgr"])) < 2e-9
    G = ls.IntBox.exchangeGrad(res, ew, pl, D2, D2, False, False, True, 1e-14, 1e-14)
    assert np.max(np.abs(G.np - z["Kgr2"])) < 1e-9
    G = ls.IntBox.exchangeGrad(res, ew, pl, D, D2, True, False, False, 1e-14, 1e-14)
    assert np.max(np.abs(G.np - z["Kgr3"])) < 1e-9
    G = ls.IntBox.exchangeGrad(res, ew, pl, D2, D, False, True, False, 1e-14, 1e-14)
    assert np.max(np.abs(G.np - z["Kgr4"])) < 1e-9


@pytest.mark.parametrize("case", ["water8", "propane"])
def test_exchange_grad_vs_oracle(ls, case):
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    from lightspeed_b200.geometry import alkane, water_cluster
    if case == "water8":
        bas, Da, Db = _oracle_case(ls, water_cluster(8, seed=0), "6-31gs", 5)
        thre = 1e-12
    else:
        bas, Da, Db = _oracle_case(ls, alkane(3), "cc-pvdz", 6)
        thre = 1e-14
    res = ls.ResourceList.build()
    ew = ls.Ewald.coulomb()
    pl = ls.PairList.build_schwarz(bas, bas, True, thre)
    rb = ref.RefBasis(ref.prim_arrays(bas))
    rp = ref.RefPairs(rb, rb, True, thre)
    A, B = ls.Tensor.array(Da), ls.Tensor.array(Db)
    G_same = ls.IntBox.exchangeGrad(res, ew, pl, A, A, True, True, True, thre, thre).np
    G_ab = ls.IntBox.exchangeGrad(res, ew, pl, A, B, True, True, False, thre, thre).np
    Gr_same = ref.exchange_grad(rp, Da, None, True, True, thre, thre)
    Gr_ab = ref.exchange_grad(rp, Da, Db, True, True, thre, thre)
    assert np.max(np.abs(Gr_same)) > 1e-3
    assert np.max(np.abs(G_same - Gr_same)) < 1e-9
    assert np.max(np.abs(G_ab - Gr_ab)) < 1e-9
    assert np.max(np.abs(G_ab.sum(axis=0))) < 1e-9
    # without the symmetry promises every ordered quartet runs (no mirror halving): same sum
    G_nosym = ls.IntBox.exchangeGrad(res, ew, pl, A, B, False, False, False, thre, thre).np
    assert np.max(np.abs(G_nosym - Gr_ab)) < 1e-9


def test_exchange_grad_range_separated(ls, golden_dir):
    """erf-attenuated and two-term operators against the oracle."""
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    mol = ls.Molecule.from_xyz_file(os.path.join(golden_dir, "h2o.xyz"))
    bas = ls.Basis.from_gbs_file(mol, "cc-pvdz")
    z = np.load(os.path.join(golden_dir, "ref_prop_h2o_cc-pvdz.npz"))
    res = ls.ResourceList.build()
    pl = ls.PairList.build_schwarz(bas, bas, True, 1e-14)
    rb = ref.RefBasis(ref.prim_arrays(bas))
    rp = ref.RefPairs(rb, rb, True, 1e-14)
    for sc, om in (([1.0], [0.3]), ([-0.7, 0.7], [0.3, -1.0])):
        G = ls.IntBox.exchangeGrad(res, ls.Ewald(sc, om), pl, ls.Tensor.array(z["D2"]), ls.Tensor.array(z["D"]),
                                   False, True, False, 1e-14, 1e-14).np
        Gr = ref.exchange_grad(rp, z["D2"], z["D"], False, True, 1e-14, 1e-14, sc, om)
        assert np.max(np.abs(G - Gr)) < 1e-9


def test_exchange_grad_needs_symmetric_pairlist(ls, golden_dir):
    mol = ls.Molecule.from_xyz_file(os.path.join(golden_dir, "h2o.xyz"))
    bas = ls.Basis.from_gbs_file(mol, "sto-3g")
    res = ls.ResourceList.build()
    pl = ls.PairList.build_schwarz(bas, bas, False, 1e-14)
    D = ls.Tensor.array(np.eye(bas.nao))
    with pytest.raises(RuntimeError, match="symmetric"):
        ls.IntBox.exchangeGrad(res, ls.Ewald.coulomb(), pl, D, D, True, True, True, 1e-14, 1e-14)
