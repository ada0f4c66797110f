"""The oracle's eriJ restatement (oracle/ref.py: eri_j, after
src/cpp/intbox/mo_eri.cpp:10-157) on the CPU, over the reference's own
coulomb: with every symmetry flag set (the CASCI call) the result has the
8-fold permutation symmetry of (ij|kl) exactly, and the symmetrised values
differ from the unsymmetrised composition only at the screening level
(1e-11); (ij|kl) also equals the trace of D_ij with J[D_kl] built
independently."""
import numpy as np
import pytest

from oracle import ref

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref/libls_ref.so not built")


def _pairs(ls):
    from lightspeed_b200.geometry import water_cluster
    bas = ls.Basis.from_gbs_file(water_cluster(2, seed=3), "6-31gs")
    rb = ref.RefBasis(ref.prim_arrays(bas))
    return bas, rb, ref.RefPairs(rb, rb, True, 1e-14)


def test_eri_j_oracle_symmetry_and_definition(ls):
    bas, _, rp = _pairs(ls)
    C = np.random.default_rng(2).standard_normal((bas.nao, 3)) / np.sqrt(bas.nao)
    I = ref.eri_j(rp, rp, C, C, C, C, 1e-14, 1e-14, True, True, True)
    for perm in ((1, 0, 2, 3), (0, 1, 3, 2), (2, 3, 0, 1)):
        assert np.array_equal(I, I.transpose(perm))
    I0 = ref.eri_j(rp, rp, C, C, C, C, 1e-14, 1e-14, False, False, False)
    assert np.max(np.abs(I - I0)) < 1e-11
    # (01|21) = sum_pq D_01[p,q] J[D_21][p,q]
    D01 = np.outer(C[:, 0], C[:, 1])
    J21 = ref.coulomb(rp, rp, np.outer(C[:, 2], C[:, 1]), 1e-14, 1e-14)
    assert abs(np.sum(D01 * J21) - I0[0, 1, 2, 1]) < 1e-11
