"""The oracle's C restatement (oracle/jk_port.c) pinned against the reference's
golden vectors and, where the reference build is present, against the
reference CPU IntBox itself on the same inputs (1e-12)."""
import os

import numpy as np
import pytest

from oracle import port, ref

pytestmark = pytest.mark.skipif(not port.available(), reason="oracle/_ref/libjk_port.so not built")

EWALD = {"LR": ([1.0], [0.3]), "SR": ([-0.7, 0.7], [0.3, -1.0]), "MIX": ([0.8, 0.2], [0.2, -1.0])}


@pytest.mark.parametrize("basis", ["sto-3g", "6-31gs", "cc-pvdz"])
@pytest.mark.parametrize("symm", [True, False])
def test_port_prop_golden(ls, golden_dir, basis, symm):
    mol = ls.Molecule.from_xyz_file(os.path.join(golden_dir, "h2o.xyz"))
    pb = port.Basis(ls.Basis.from_gbs_file(mol, basis).primitives)
    z = np.load(os.path.join(golden_dir, "ref_prop_h2o_%s.npz" % basis))
    pl = port.Pairs(pb, pb, symm, 1e-14)
    assert np.max(abs(port.coulomb(pl, pl, z["D"], 1e-14) - z["J"])) < 1e-9
    assert np.max(abs(port.coulomb(pl, pl, z["D2"], 1e-14) - z["J2"])) < 1e-9
    assert np.max(abs(port.exchange(pl, pl, z["D"], True, 1e-14) - z["K"])) < 1e-9
    assert np.max(abs(port.exchange(pl, pl, z["D2"], False, 1e-14) - z["K2"])) < 1e-9


@pytest.mark.parametrize("basis", ["6-31gs", "cc-pvdz"])
def test_port_ewald_golden(ls, golden_dir, basis):
    mol = ls.Molecule.from_xyz_file(os.path.join(golden_dir, "h2o.xyz"))
    pb = port.Basis(ls.Basis.from_gbs_file(mol, basis).primitives)
    z = np.load(os.path.join(golden_dir, "ref_ewald_h2o_%s.npz" % basis))
    pl = port.Pairs(pb, pb, True, 1e-14)
    for name, (s, o) in EWALD.items():
        assert np.max(abs(port.coulomb(pl, pl, z["D_" + name], 1e-14, s, o) - z["J_" + name])) < 1e-12
        assert np.max(abs(port.exchange(pl, pl, z["D2_" + name], False, 1e-14, s, o) - z["K2_" + name])) < 1e-12


def test_port_pairlist_matches_reference(ls, golden_dir):
    if not ref.available():
        pytest.skip("reference build absent")
    from lightspeed_b200.geometry import water_cluster
    bas = ls.Basis.from_gbs_file(water_cluster(3, seed=2), "cc-pvdz")
    pb = port.Basis(bas.primitives)
    rb = ref.RefBasis(ref.prim_arrays(bas))
    for symm in (True, False):
        pl = port.Pairs(pb, pb, symm, 1e-12)
        L1, L2, p1, p2, b = ref.RefPairs(rb, rb, symm, 1e-12).export()
        assert np.array_equal(pl.pa, p1) and np.array_equal(pl.pb, p2) and np.array_equal(pl.bound, b)


def test_port_matches_reference_water3(ls):
    """Thresholds that bite (1e-10): the restated screening gives the same J/K."""
    if not ref.available():
        pytest.skip("reference build absent")
    from lightspeed_b200.geometry import water_cluster
    bas = ls.Basis.from_gbs_file(water_cluster(3, seed=2), "6-31gs")
    pb = port.Basis(bas.primitives)
    rb = ref.RefBasis(ref.prim_arrays(bas))
    rng = np.random.default_rng(3)
    D = rng.normal(size=(bas.nao, bas.nao)) * 0.05
    Ds = D + D.T
    for thre in (1e-10, 1e-14):
        pl = port.Pairs(pb, pb, True, thre)
        rp = ref.RefPairs(rb, rb, True, thre)
        assert np.max(abs(port.coulomb(pl, pl, Ds, thre) - ref.coulomb(rp, rp, Ds, thre, thre))) < 1e-12
        assert np.max(abs(port.exchange(pl, pl, Ds, True, thre) - ref.exchange(rp, rp, Ds, True, thre, thre))) < 1e-12
        assert np.max(abs(port.exchange(pl, pl, D, False, thre) - ref.exchange(rp, rp, D, False, thre, thre))) < 1e-12
