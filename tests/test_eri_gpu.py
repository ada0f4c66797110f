"""IntBox.eriJ (MO-basis integrals through J builds) against the reference's
IntBox::eriJ restated over the reference's own CPU coulomb (oracle/ref.py:
eri_j, after src/cpp/intbox/mo_eri.cpp:10-157).

Cases: the CASCI use (one active-orbital block passed as all four
coefficient tensors: every symmetrisation applies), a symmetric bra and ket
with different blocks, and four different blocks (no symmetry), bare and
erf-attenuated operators. FP64 mode; tolerance 1e-10 elementwise (the J
builds agree with the reference to ~1e-13; the contractions differ only in
summation order). Repeated calls agree to 1e-13, not bit for bit: J sums
with FP64 atomics in no fixed order."""
import numpy as np
import pytest

from oracle import ref

pytestmark = pytest.mark.gpu


def _setup(ls):
    from lightspeed_b200.geometry import water_cluster
    if not ref.available():
        pytest.skip("reference build (oracle/_ref) not present")
    mol = water_cluster(2, seed=3)
    bas = ls.Basis.from_gbs_file(mol, "6-31gs")
    pl = ls.PairList.build_schwarz(bas, bas, True, 1e-14)
    rb = ref.RefBasis(ref.prim_arrays(bas))
    rp = ref.RefPairs(rb, rb, True, 1e-14)
    return bas, pl, rp


@pytest.mark.parametrize("operator", ["coulomb", "erf"])
@pytest.mark.parametrize("case", ["casci", "sym_pairs", "general"])
def test_eriJ_matches_reference(ls, case, operator):
    bas, pl, rp = _setup(ls)
    rng = np.random.default_rng(11)
    nao = bas.nao
    blocks = [rng.standard_normal((nao, n)) / np.sqrt(nao) for n in (4, 3, 5, 2)]
    if case == "casci":
        A = ls.Tensor.array(blocks[0])
        T = [A, A, A, A]
        flags = (True, True, True)
    elif case == "sym_pairs":
        A, B = ls.Tensor.array(blocks[0]), ls.Tensor.array(blocks[2])
        T = [A, A, B, B]
        flags = (True, True, False)
    else:
        T = [ls.Tensor.array(b) for b in blocks]
        flags = (False, False, False)
    if operator == "coulomb":
        ew, scales, omegas = ls.Ewald.coulomb(), (1.0,), (-1.0,)
    else:
        scales, omegas = (1.0, -0.7), (-1.0, 0.3)
        ew = ls.Ewald(list(scales), list(omegas))
    ls.set_precision(ls.PREC_FP64)
    try:
        res = ls.ResourceList.build()
        I = ls.IntBox.eriJ(res, ew, pl, pl, T[0], T[1], T[2], T[3], 1e-14, 1e-14).np.copy()
        I2 = ls.IntBox.eriJ(res, ew, pl, pl, T[0], T[1], T[2], T[3], 1e-14, 1e-14).np.copy()
    finally:
        ls.set_precision(ls.PREC_MIXED)
    C = [t.np for t in T]
    Iref = ref.eri_j(rp, rp, C[0], C[1], C[2], C[3], 1e-14, 1e-14, *flags, scales=scales, omegas=omegas)
    assert I.shape == Iref.shape
    assert np.max(np.abs(I - Iref)) < 1e-10
    # a second call agrees up to the order of the J builds' FP64 atomic sums
    assert np.max(np.abs(I - I2)) < 1e-13
    if case == "casci":
        # (ij|kl) = (ji|kl) = (ij|lk) = (kl|ij)
        for perm in ((1, 0, 2, 3), (0, 1, 3, 2), (2, 3, 0, 1)):
            assert np.max(np.abs(I - I.transpose(perm))) < 1e-13


def test_eriJ_shape_errors(ls):
    bas, pl, _ = _setup(ls)
    res = ls.ResourceList.build()
    A = ls.Tensor.array(np.zeros((bas.nao + 1, 2)))
    with pytest.raises(Exception):
        ls.IntBox.eriJ(res, ls.Ewald.coulomb(), pl, pl, A, A, A, A, 1e-14, 1e-14)
