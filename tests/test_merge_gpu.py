"""Merged s exponents in K (the opt-in build mode ls.set_merge(True)).

cc-pVDZ repeats the eight tight s exponents of C, N, O, ... in the 1s and 2s
contracted shells; the reference treats each copy as a primitive of its own.
In merge mode the engine builds K over a twin basis with one primitive per
distinct (atom, s exponent) and contracts each integral into every shell
that shares it (J always runs over the primitives as given). The screens of
the merged build bound every copy, so it keeps every quartet the reference
keeps plus copies just below thresp: K must equal the reference's
(oracle/_ref) elementwise within the FP64 tolerance 1e-10 at the workloads'
threshold 1e-14, with fewer K quartets computed; with merging off the
quartet counters equal the oracle's count of the reference quartet set
exactly. Propane in cc-pVDZ (spherical d, all shells of C and H) and a mixed
cc-pVDZ / 6-31G* pair of bases cover merged and unmerged primitives side by
side.
"""
import numpy as np
import pytest

from oracle import port, ref

pytestmark = pytest.mark.gpu

THRE = 1.0e-14


@pytest.fixture(autouse=True)
def _modes(ls):
    ls.set_precision(ls.PREC_FP64)
    ls.set_merge(True)
    yield
    ls.set_merge(False)
    ls.set_precision(ls.PREC_MIXED)


def _propane(ls):
    from lightspeed_b200.geometry import alkane
    mol = alkane(3)
    return mol, ls.Basis.from_gbs_file(mol, "cc-pvdz")


def _density(nao, seed, symm=True):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((nao, 12)) / np.sqrt(nao)
    if symm:
        return X @ X.T
    Y = rng.standard_normal((nao, 12)) / np.sqrt(nao)
    return X @ Y.T


def _ref_pairs(bas, thre=THRE):
    rb = ref.RefBasis(ref.prim_arrays(bas))
    return ref.RefPairs(rb, rb, True, thre)


def _need_ref():
    if not (ref.available() and port.available()):
        pytest.skip("oracle/_ref not built")


@pytest.mark.parametrize("ewald", [([1.0], [-1.0]), ([1.0], [0.3]), ([-0.7, 0.7], [0.3, -1.0])])
def test_merged_jk_match_reference(ls, ewald):
    _need_ref()
    _, bas = _propane(ls)
    res = ls.ResourceList.build()
    ew = ls.Ewald(*ewald)
    pl = ls.PairList.build_schwarz(bas, bas, True, THRE)
    rp = _ref_pairs(bas)
    assert ls.get_merge()
    for seed, symm in ((1, True), (2, False)):
        D = _density(bas.nao, seed, symm)
        J = ls.IntBox.coulomb(res, ew, pl, pl, ls.Tensor.array(D), THRE, THRE).np
        K = ls.IntBox.exchange(res, ew, pl, pl, ls.Tensor.array(D), symm, THRE, THRE).np
        assert np.max(np.abs(J - ref.coulomb(rp, rp, D, THRE, THRE, *ewald))) < 1e-10
        assert np.max(np.abs(K - ref.exchange(rp, rp, D, symm, THRE, THRE, *ewald))) < 1e-10


def test_merged_computes_fewer_quartets_exact_mode_counts_reference_set(ls):
    _need_ref()
    _, bas = _propane(ls)
    res = ls.ResourceList.build()
    ew = ls.Ewald.coulomb()
    pl = ls.PairList.build_schwarz(bas, bas, True, THRE)
    D = _density(bas.nao, 3)
    pb = port.Basis(bas.primitives)
    ppl = port.Pairs(pb, pb, True, THRE)
    nj, nk = port.count_quartets(ppl, ppl, D, D, True, THRE)
    out = {}
    for merge in (False, True):
        ls.set_merge(merge)
        ls.reset_stats()
        J = ls.IntBox.coulomb(res, ew, pl, pl, ls.Tensor.array(D), THRE, THRE).np.copy()
        K = ls.IntBox.exchange(res, ew, pl, pl, ls.Tensor.array(D), True, THRE, THRE).np.copy()
        out[merge] = (J, K, ls.stats())
    st = out[False][2]
    assert st["j_quartets"] == nj and st["k_quartets"] == nk
    sm = out[True][2]
    # J is never merged; in K eight of the nine s exponents of carbon are shared by two shells
    assert sm["j_quartets"] == nj
    assert sm["k_quartets"] < 0.8 * nk
    assert np.max(np.abs(out[True][0] - out[False][0])) < 1e-12
    assert np.max(np.abs(out[True][1] - out[False][1])) < 1e-10


def test_merged_mixed_bases(ls):
    """Bra and ket pair lists over different bases (one with shared
    exponents, one without), J and non-symmetric K, against the reference."""
    _need_ref()
    mol, b1 = _propane(ls)
    b2 = ls.Basis.from_gbs_file(mol, "6-31gs")
    res = ls.ResourceList.build()
    ew = ls.Ewald.coulomb()
    p11 = ls.PairList.build_schwarz(b1, b1, True, THRE)
    p12 = ls.PairList.build_schwarz(b1, b2, False, THRE)
    p22 = ls.PairList.build_schwarz(b2, b2, True, THRE)
    r1 = ref.RefBasis(ref.prim_arrays(b1))
    r2 = ref.RefBasis(ref.prim_arrays(b2))
    rp11 = ref.RefPairs(r1, r1, True, THRE)
    rp12 = ref.RefPairs(r1, r2, False, THRE)
    rp22 = ref.RefPairs(r2, r2, True, THRE)
    D22 = _density(b2.nao, 4)
    J11 = ls.IntBox.coulomb(res, ew, p11, p22, ls.Tensor.array(D22), THRE, THRE).np
    assert np.max(np.abs(J11 - ref.coulomb(rp11, rp22, D22, THRE, THRE))) < 1e-10
    rng = np.random.default_rng(5)
    # K13 (cc-pVDZ x cc-pVDZ) from D24 over the 6-31G* functions of both pair lists
    D24 = rng.standard_normal((b2.nao, b2.nao)) * 0.05
    K13 = ls.IntBox.exchange(res, ew, p12, p12, ls.Tensor.array(D24), False, THRE, THRE).np
    assert np.max(np.abs(K13 - ref.exchange(rp12, rp12, D24, False, THRE, THRE))) < 1e-10


def test_merged_batched_k_matches_single(ls):
    _need_ref()
    _, bas = _propane(ls)
    res = ls.ResourceList.build()
    ew = ls.Ewald.coulomb()
    pl = ls.PairList.build_schwarz(bas, bas, True, THRE)
    Ds = [_density(bas.nao, 10 + k, symm=False) for k in range(4)]
    Km = ls.IntBox.exchangeMulti(res, ew, pl, pl, [ls.Tensor.array(D) for D in Ds], False, THRE, THRE)
    rp = _ref_pairs(bas)
    for D, K in zip(Ds, Km):
        assert np.max(np.abs(K.np - ref.exchange(rp, rp, D, False, THRE, THRE))) < 1e-10


def test_merged_mixed_precision(ls):
    """Mixed precision over the merged twin: within 1e-6 of the reference."""
    _need_ref()
    _, bas = _propane(ls)
    res = ls.ResourceList.build()
    ew = ls.Ewald.coulomb()
    pl = ls.PairList.build_schwarz(bas, bas, True, THRE)
    D = _density(bas.nao, 6)
    ls.set_precision(ls.PREC_MIXED)
    ls.reset_stats()
    J = ls.IntBox.coulomb(res, ew, pl, pl, ls.Tensor.array(D), THRE, 1e-5).np
    K = ls.IntBox.exchange(res, ew, pl, pl, ls.Tensor.array(D), True, THRE, 1e-5).np
    assert ls.stats()["quartets_fp32"] > 0
    rp = _ref_pairs(bas)
    assert np.max(np.abs(J - ref.coulomb(rp, rp, D, THRE, THRE))) < 1e-6
    assert np.max(np.abs(K - ref.exchange(rp, rp, D, True, THRE, THRE))) < 1e-6
