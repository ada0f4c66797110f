"""Mixed precision (the reference's thredp semantics, src/lightspeed/intbox.hpp:
730-740): quartets with estimate >= thredp in FP64, [thresp, thredp) in FP32,
FP64 accumulation. Checked against the FP64 path and the oracle: the same
quartet set, a nonzero FP32 share, elementwise J/K error <= 1e-6 and an
energy error at fixed density <= 1e-6 Eh."""
import os

import numpy as np
import pytest

from oracle import ref

pytestmark = pytest.mark.gpu


def _water8(ls, golden_dir):
    from lightspeed_b200.geometry import water_cluster
    z = np.load(os.path.join(golden_dir, "oracle_w8.npz"))
    bas = ls.Basis.from_gbs_file(water_cluster(8, seed=0), "6-31gs")
    return bas, z


def test_mixed_matches_fp64_within_tolerance(ls, golden_dir):
    bas, z = _water8(ls, golden_dir)
    res = ls.ResourceList.build()
    ew = ls.Ewald.coulomb()
    pl = ls.PairList.build_schwarz(bas, bas, True, 1e-12)
    D = ls.Tensor.array(z["D"])
    out = {}
    for mode in (ls.PREC_FP64, ls.PREC_MIXED):
        ls.set_precision(mode)
        ls.reset_stats()
        J = ls.IntBox.coulomb(res, ew, pl, pl, D, 1e-12, 1e-6).np.copy()
        K = ls.IntBox.exchange(res, ew, pl, pl, D, True, 1e-12, 1e-6).np.copy()
        out[mode] = (J, K, ls.stats())
    ls.set_precision(ls.PREC_MIXED)
    J64, K64, s64 = out[ls.PREC_FP64]
    J32, K32, s32 = out[ls.PREC_MIXED]
    assert s64["quartets_fp32"] == 0
    assert s32["quartets_fp32"] > 0.5 * (s32["quartets_fp32"] + s32["quartets_fp64"])
    assert s32["j_quartets"] == s64["j_quartets"] and s32["k_quartets"] == s64["k_quartets"]
    assert np.max(abs(J64 - z["J"])) < 1e-10 and np.max(abs(K64 - z["K"])) < 1e-10
    assert np.max(abs(J32 - z["J"])) < 1e-6
    assert np.max(abs(K32 - z["K"])) < 1e-6
    Dn = z["D"]
    dE = np.sum(Dn * (2.0 * (J32 - z["J"]) - (K32 - z["K"])))
    assert abs(dE) < 1e-6


def test_mixed_with_equal_thresholds_is_fp64(ls, golden_dir):
    bas, z = _water8(ls, golden_dir)
    res = ls.ResourceList.build()
    pl = ls.PairList.build_schwarz(bas, bas, True, 1e-12)
    ls.set_precision(ls.PREC_MIXED)
    ls.reset_stats()
    J = ls.IntBox.coulomb(res, ls.Ewald.coulomb(), pl, pl, ls.Tensor.array(z["D"]), 1e-12, 1e-12).np
    assert ls.stats()["quartets_fp32"] == 0
    assert np.max(abs(J - z["J"])) < 1e-10


def test_mixed_ewald_range_separated(ls, golden_dir):
    """erf-attenuated operator (omega = 0.3) through the FP32 path."""
    bas, z = _water8(ls, golden_dir)
    res = ls.ResourceList.build()
    pl = ls.PairList.build_schwarz(bas, bas, True, 1e-12)
    ew = ls.Ewald([1.0], [0.3])
    D = ls.Tensor.array(z["D"])
    ls.set_precision(ls.PREC_FP64)
    J64 = ls.IntBox.coulomb(res, ew, pl, pl, D, 1e-12, 1e-6).np.copy()
    K64 = ls.IntBox.exchange(res, ew, pl, pl, D, True, 1e-12, 1e-6).np.copy()
    ls.set_precision(ls.PREC_MIXED)
    J32 = ls.IntBox.coulomb(res, ew, pl, pl, D, 1e-12, 1e-6).np
    K32 = ls.IntBox.exchange(res, ew, pl, pl, D, True, 1e-12, 1e-6).np
    if ref.available():
        rb = ref.RefBasis(ref.prim_arrays(bas))
        rp = ref.RefPairs(rb, rb, True, 1e-12)
        assert np.max(abs(J64 - ref.coulomb(rp, rp, z["D"], 1e-12, 1e-12, [1.0], [0.3]))) < 1e-10
    assert np.max(abs(J32 - J64)) < 1e-6 and np.max(abs(K32 - K64)) < 1e-6
