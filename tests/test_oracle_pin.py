"""The oracle (reference CPU IntBox built from its own sources, oracle/_ref)
pinned against the reference's known-answer vectors for the J/K path
(tests/coverage/prop_int.py:68-108, ewald_int.py:33-108 and mix_basis.py in the
reference), at the tolerances those tests use (1e-9, 1e-12)."""
import os

import numpy as np
import pytest

from oracle import ref

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")

EWALD = {"LR": ([1.0], [0.3]), "LR2": ([0.7, 0.7, 0.7], [0.2, 0.1, 0.05]), "SR": ([-0.7, 0.7], [0.3, -1.0]),
         "SR2": ([-0.7, 0.7], [-1.0, -1.0]), "MIX": ([0.8, 0.2], [0.2, -1.0])}


def _ref_basis(ls, golden_dir, basis, xyz="h2o"):
    mol = ls.Molecule.from_xyz_file(os.path.join(golden_dir, xyz + ".xyz"))
    bas = ls.Basis.from_gbs_file(mol, basis)
    return bas, ref.RefBasis(ref.prim_arrays(bas))


@pytest.mark.parametrize("basis", ["sto-3g", "6-31gs", "cc-pvdz"])
@pytest.mark.parametrize("symm", [True, False])
def test_oracle_prop(ls, golden_dir, basis, symm):
    _, rb = _ref_basis(ls, golden_dir, basis)
    z = np.load(os.path.join(golden_dir, "ref_prop_h2o_%s.npz" % basis))
    pl = ref.RefPairs(rb, rb, symm, 1e-14)
    assert np.max(abs(ref.coulomb(pl, pl, z["D"], 1e-14, 1e-14) - z["J"])) < 1e-9
    assert np.max(abs(ref.coulomb(pl, pl, z["D2"], 1e-14, 1e-14) - z["J2"])) < 1e-9
    assert np.max(abs(ref.exchange(pl, pl, z["D"], True, 1e-14, 1e-14) - z["K"])) < 1e-9
    assert np.max(abs(ref.exchange(pl, pl, z["D2"], False, 1e-14, 1e-14) - z["K2"])) < 1e-9


@pytest.mark.parametrize("basis", ["sto-3g", "6-31gs", "cc-pvdz"])
def test_oracle_ewald(ls, golden_dir, basis):
    _, rb = _ref_basis(ls, golden_dir, basis)
    z = np.load(os.path.join(golden_dir, "ref_ewald_h2o_%s.npz" % basis))
    pl = ref.RefPairs(rb, rb, True, 1e-14)
    for name, (s, o) in EWALD.items():
        D, D2 = z["D_" + name], z["D2_" + name]
        assert np.max(abs(ref.coulomb(pl, pl, D, 1e-14, 1e-14, s, o) - z["J_" + name])) < 1e-12
        assert np.max(abs(ref.exchange(pl, pl, D2, False, 1e-14, 1e-14, s, o) - z["K2_" + name])) < 1e-12


@pytest.mark.parametrize("basis", ["sto-3g", "6-31gs", "cc-pvdz"])
def test_oracle_gradients(ls, golden_dir, basis):
    """IntBox::coulombGrad / exchangeGrad of the reference build against the
    reference's gradient vectors (prop_int.py:142-214, tolerance 1e-9): the
    symmetric and the general (D12 != D34, D13/D24 symmetry flags) branches."""
    _, rb = _ref_basis(ls, golden_dir, basis)
    z = np.load(os.path.join(golden_dir, "ref_prop_h2o_%s.npz" % basis))
    pl = ref.RefPairs(rb, rb, True, 1e-14)
    D, D2 = z["D"], z["D2"]
    assert np.max(abs(ref.coulomb_grad(pl, D) - z["Jgr"])) < 1e-9
    assert np.max(abs(ref.coulomb_grad(pl, D2) - z["Jgr2"])) < 1e-9
    assert np.max(abs(ref.coulomb_grad(pl, D, D2) - z["Jgr3"])) < 1e-9
    assert np.max(abs(ref.coulomb_grad(pl, D2, D) - z["Jgr4"])) < 1e-9
    assert np.max(abs(ref.exchange_grad(pl, D) - z["Kgr"])) < 1e-9
    assert np.max(abs(ref.exchange_grad(pl, D2, None, False, False) - z["Kgr2"])) < 1e-9
    assert np.max(abs(ref.exchange_grad(pl, D, D2, True, False) - z["Kgr3"])) < 1e-9
    assert np.max(abs(ref.exchange_grad(pl, D2, D, False, True) - z["Kgr4"])) < 1e-9
