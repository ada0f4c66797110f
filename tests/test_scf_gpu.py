"""One-electron integrals (device kernels, oneint.cu) and the RHF energy
around the GPU J/K path, against the oracle (reference CPU IntBox): S/T/V
elementwise 1e-12 (symmetric, mixed-basis and range-separated cases,
accumulation into a passed tensor), and the converged
RHF energy of 8 H2O / 6-31G* (Schwarz 1e-12, SCF to gradient 1e-8) equal to
the energy of the same SCF driven by the oracle's J/K to 1e-9 Eh."""
import os

import numpy as np
import pytest

from oracle import ref

pytestmark = pytest.mark.gpu


def test_one_electron_vs_oracle(ls, golden_dir):
    mol = ls.Molecule.from_xyz_file(os.path.join(golden_dir, "h2o.xyz"))
    res = ls.ResourceList.build()
    for basis in ("sto-3g", "6-31gs", "cc-pvdz"):
        bas = ls.Basis.from_gbs_file(mol, basis)
        pl = ls.PairList.build_schwarz(bas, bas, True, 1e-14)
        rb = ref.RefBasis(ref.prim_arrays(bas))
        rp = ref.RefPairs(rb, rb, True, 1e-14)
        S = ls.IntBox.overlap(res, pl).np
        T = ls.IntBox.kinetic(res, pl).np
        V = ls.IntBox.potential(res, ls.Ewald.coulomb(), pl, ls.Tensor.array(mol.xyzZ)).np
        assert np.max(abs(S - ref.overlap(rp))) < 1e-12
        assert np.max(abs(T - ref.kinetic(rp))) < 1e-12
        assert np.max(abs(V - ref.potential(rp, mol.xyzZ))) < 1e-11


def test_one_electron_mixed_basis_and_ewald(ls, golden_dir):
    """Non-symmetric pair lists between two bases, an erf-attenuated and a
    two-term potential, propane / cc-pVDZ, and accumulation into a given tensor."""
    from lightspeed_b200.geometry import alkane
    res = ls.ResourceList.build()
    h2o = ls.Molecule.from_xyz_file(os.path.join(golden_dir, "h2o.xyz"))
    ba = ls.Basis.from_gbs_file(h2o, "6-31gs")
    bb = ls.Basis.from_gbs_file(h2o, "cc-pvdz")
    pl = ls.PairList.build_schwarz(ba, bb, False, 1e-14)
    rp = ref.RefPairs(ref.RefBasis(ref.prim_arrays(ba)), ref.RefBasis(ref.prim_arrays(bb)), False, 1e-14)
    assert np.max(abs(ls.IntBox.overlap(res, pl).np - ref.overlap(rp))) < 1e-12
    assert np.max(abs(ls.IntBox.kinetic(res, pl).np - ref.kinetic(rp))) < 1e-12
    for sc, om in (([1.0], [0.3]), ([0.7, 0.3], [-1.0, 0.5])):
        V = ls.IntBox.potential(res, ls.Ewald(sc, om), pl, ls.Tensor.array(h2o.xyzZ)).np
        assert np.max(abs(V - ref.potential(rp, h2o.xyzZ, sc, om))) < 1e-11
    mol = alkane(3)
    bas = ls.Basis.from_gbs_file(mol, "cc-pvdz")
    pl = ls.PairList.build_schwarz(bas, bas, True, 1e-14)
    rb = ref.RefBasis(ref.prim_arrays(bas))
    rp = ref.RefPairs(rb, rb, True, 1e-14)
    S = ls.IntBox.overlap(res, pl)
    S2 = ls.IntBox.overlap(res, pl, S)
    assert S2 is S or np.shares_memory(S2.np, S.np)
    Sr = ref.overlap(rp)
    assert np.max(abs(S2.np - 2.0 * Sr)) < 2e-12
    assert np.max(abs(ls.IntBox.kinetic(res, pl).np - ref.kinetic(rp))) < 1e-12
    V = ls.IntBox.potential(res, ls.Ewald.coulomb(), pl, ls.Tensor.array(mol.xyzZ)).np
    assert np.max(abs(V - ref.potential(rp, mol.xyzZ))) < 1e-10


def test_rhf_energy_water8(ls):
    from lightspeed_b200.geometry import water_cluster
    from lightspeed_b200.scf import RHF, loewdin_density
    ls.set_precision(ls.PREC_FP64)
    mol = water_cluster(8, seed=0)
    bas = ls.Basis.from_gbs_file(mol, "6-31gs")
    scf = RHF(ls, mol, bas, thre_pq=1e-12, thre_sp=1e-12, thre_dp=1e-12)
    D0 = loewdin_density(scf.S, scf.nocc, seed=1)
    E_gpu = scf.compute(D0=D0, g_conv=1e-8)
    assert scf.converged
    # the same SCF with the oracle's J and K
    rb = ref.RefBasis(ref.prim_arrays(bas))
    rp = ref.RefPairs(rb, rb, True, 1e-12)
    oracle_scf = RHF(ls, mol, bas, thre_pq=1e-12, thre_sp=1e-12, thre_dp=1e-12)
    oracle_scf.jk = lambda D: (ref.coulomb(rp, rp, D, 1e-12, 1e-12), ref.exchange(rp, rp, D, True, 1e-12, 1e-12))
    E_ref = oracle_scf.compute(D0=D0, g_conv=1e-8)
    assert abs(E_gpu - E_ref) < 1e-9, (E_gpu, E_ref)
    ls.set_precision(ls.PREC_MIXED)
