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
