"""The drop-in boundary exercised from the reference's side.

oracle/b200_shim.cpp is the binding a Lightspeed maintainer adds so that
IntBox::coulomb / IntBox::exchange (and the gradients coulombGrad /
exchangeGrad) run on liblsjk.so: functions with the
reference's signatures, written against the reference's own headers and
types (Tensor, Basis, PairList, Ewald, ResourceList) and compiled from them
(oracle/Makefile, target shim). These tests call them with reference Basis
and PairList objects (built by the reference's own PairList::build_schwarz)
and check the reference's golden vectors at the reference's tolerances
(prop_int.py 1e-9, ewald_int.py and mix_basis.py 1e-12), the
accumulate-into-J12 contract, that a D24symm misuse raises the
reference's error through the shim, and the J/K nuclear gradients
(coulombGrad / exchangeGrad) against the Jgr*/Kgr* goldens."""
import ctypes
import os

import numpy as np
import pytest

from oracle import ref

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "oracle", "_ref", "libls_b200shim.so")
EWALD = {"LR": ([1.0], [0.3]), "LR2": ([0.7, 0.7, 0.7], [0.2, 0.1, 0.05]), "SR": ([-0.7, 0.7], [0.3, -1.0]),
         "SR2": ([-0.7, 0.7], [-1.0, -1.0]), "MIX": ([0.8, 0.2], [0.2, -1.0])}


@pytest.fixture(scope="module")
def shim():
    if not (os.path.exists(SHIM) and ref.available()):
        pytest.skip("oracle/_ref/libls_b200shim.so not built")
    ref.lib()   # the reference objects' library first (the shim links it)
    lib = ctypes.CDLL(SHIM)
    lib.shim_last_error.restype = ctypes.c_char_p
    vp, ip, fp = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
    # typed arguments: an untyped Python int would go through as a 32-bit C int
    lib.shim_jk.argtypes = [ip, vp, vp, ip, vp, vp, vp, ip, fp, fp, ip, vp]
    lib.shim_grad.argtypes = [ip, vp, ip, vp, vp, vp, vp, ip, ip, ip, fp, fp, vp]
    return lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _jk(shim, which, p12, p34, D, symm=False, ewald=([1.0], [-1.0]), thre=1e-14, out=None):
    s = np.ascontiguousarray(ewald[0], np.float64)
    o = np.ascontiguousarray(ewald[1], np.float64)
    D = np.ascontiguousarray(D, np.float64)
    n1 = p12.b1.nao
    n2 = p34.b1.nao if which else p12.b2.nao
    acc = out is not None
    O = np.ascontiguousarray(out if acc else np.zeros((n1, n2)), np.float64)
    rc = shim.shim_jk(which, p12.h, p34.h, len(s), _p(s), _p(o), _p(D), int(symm), ctypes.c_float(thre),
                      ctypes.c_float(thre), int(acc), _p(O))
    if rc:
        raise RuntimeError(shim.shim_last_error().decode())
    return O


def _refbasis(ls, xyzfile, name):
    mol = ls.Molecule.from_xyz_file(os.path.join(ROOT, "tests", "golden", xyzfile))
    return ref.RefBasis(ref.prim_arrays(ls.Basis.from_gbs_file(mol, name)))


@pytest.mark.parametrize("basis", ["sto-3g", "6-31gs", "cc-pvdz"])
def test_prop_golden_through_reference_types(ls, shim, basis):
    z = np.load(os.path.join(ROOT, "tests", "golden", "ref_prop_h2o_%s.npz" % basis))
    rb = _refbasis(ls, "h2o.xyz", basis)
    for symm in (True, False):
        pl = ref.RefPairs(rb, rb, symm, 1e-14)
        J = _jk(shim, 0, pl, pl, z["D"])
        assert np.max(np.abs(J - z["J"])) < 1e-9
        # accumulates into the passed J12 (the reference's contract)
        J2 = _jk(shim, 0, pl, pl, z["D"], out=J)
        assert np.max(np.abs(J2 - 2.0 * z["J"])) < 2e-9
        assert np.max(np.abs(_jk(shim, 0, pl, pl, z["D2"]) - z["J2"])) < 1e-9
        assert np.max(np.abs(_jk(shim, 1, pl, pl, z["D"], symm=True) - z["K"])) < 1e-9
        assert np.max(np.abs(_jk(shim, 1, pl, pl, z["D2"]) - z["K2"])) < 1e-9


@pytest.mark.parametrize("basis", ["sto-3g", "6-31gs", "cc-pvdz"])
def test_ewald_golden_through_reference_types(ls, shim, basis):
    z = np.load(os.path.join(ROOT, "tests", "golden", "ref_ewald_h2o_%s.npz" % basis))
    rb = _refbasis(ls, "h2o.xyz", basis)
    pl = ref.RefPairs(rb, rb, True, 1e-14)
    for name, ew in EWALD.items():
        for dk, jk, kk, symmD in (("D_", "J_", "K_", True), ("D2_", "J2_", "K2_", False)):
            D = z[dk + name]
            assert np.max(np.abs(_jk(shim, 0, pl, pl, D, ewald=ew) - z[jk + name])) < 1e-12, (name, jk)
            assert np.max(np.abs(_jk(shim, 1, pl, pl, D, symm=symmD, ewald=ew) - z[kk + name])) < 1e-12


def test_mixed_basis_golden_through_reference_types(ls, shim):
    z = np.load(os.path.join(ROOT, "tests", "golden", "ref_mix_h2o_nh3.npz"))
    for a, b in (("sto-3g", "6-31gs"), ("6-31gs", "cc-pvdz")):
        b1 = _refbasis(ls, "h2o.xyz", a)
        b2 = _refbasis(ls, "nh3.xyz", b)
        N1 = b1.nao
        p11 = ref.RefPairs(b1, b1, True, 1e-14)
        p12 = ref.RefPairs(b1, b2, False, 1e-14)
        p21 = ref.RefPairs(b2, b1, False, 1e-14)
        p22 = ref.RefPairs(b2, b2, True, 1e-14)
        suf = "_" + a.upper() + "_" + b.upper()
        D12 = z["D0" + suf][:N1, N1:]
        J0, K0 = z["J0" + suf], z["K0" + suf]
        assert np.max(np.abs(_jk(shim, 0, p11, p12, D12) - J0[:N1, :N1])) < 1e-12
        assert np.max(np.abs(_jk(shim, 0, p21, p12, D12) - J0[N1:, :N1])) < 1e-12
        assert np.max(np.abs(_jk(shim, 1, p11, p12, D12) - K0[:N1, :N1])) < 1e-12
        assert np.max(np.abs(_jk(shim, 1, p21, p22, D12) - K0[N1:, N1:])) < 1e-12
        D22 = z["D1" + suf][N1:, N1:]
        assert np.max(np.abs(_jk(shim, 1, p12, p22, D22, symm=True) - z["K1" + suf][:N1, N1:])) < 1e-12


def test_d24symm_misuse_raises_reference_error(ls, shim):
    b1 = _refbasis(ls, "h2o.xyz", "sto-3g")
    b2 = _refbasis(ls, "h2o.xyz", "6-31gs")
    p12 = ref.RefPairs(b1, b2, False, 1e-14)
    p11 = ref.RefPairs(b1, b1, True, 1e-14)
    with pytest.raises(RuntimeError, match="D24symm"):
        _jk(shim, 1, p12, p11, np.zeros((b2.nao, b1.nao)), symm=True)


def _grad(shim, which, pl, D1, D2, flags=(1, 1, 1), thre=1e-14, G=None):
    s = np.ascontiguousarray([1.0], np.float64)
    o = np.ascontiguousarray([-1.0], np.float64)
    A = np.ascontiguousarray(D1, np.float64)
    B = A if D2 is None else np.ascontiguousarray(D2, np.float64)
    natom = int(pl.b1.arrs["atom"][-1]) + 1
    out = np.zeros((natom, 3)) if G is None else np.array(G, np.float64, copy=True)
    rc = shim.shim_grad(which, pl.h, 1, _p(s), _p(o), _p(A), _p(B), flags[0], flags[1], flags[2],
                        ctypes.c_float(thre), ctypes.c_float(thre), _p(out))
    if rc:
        raise RuntimeError(shim.shim_last_error().decode())
    return out


@pytest.mark.parametrize("basis", ["sto-3g", "6-31gs", "cc-pvdz"])
def test_gradient_golden_through_reference_types(ls, shim, basis):
    """coulombGrad / exchangeGrad with the reference's signatures and types
    (the prop_int.py:142-211 calls) against its Jgr*/Kgr* golden vectors."""
    z = np.load(os.path.join(ROOT, "tests", "golden", "ref_prop_h2o_%s.npz" % basis))
    rb = _refbasis(ls, "h2o.xyz", basis)
    pl = ref.RefPairs(rb, rb, True, 1e-14)
    D, D2 = z["D"], z["D2"]
    G = _grad(shim, 0, pl, D, None)
    assert np.max(np.abs(G - z["Jgr"])) < 1e-9
    assert np.max(np.abs(_grad(shim, 0, pl, D, None, G=G) - 2.0 * z["Jgr"])) < 2e-9
    assert np.max(np.abs(_grad(shim, 0, pl, D, D2) - z["Jgr3"])) < 1e-9
    assert np.max(np.abs(_grad(shim, 1, pl, D, None, (1, 1, 1)) - z["Kgr"])) < 1e-9
    assert np.max(np.abs(_grad(shim, 1, pl, D2, None, (0, 0, 1)) - z["Kgr2"])) < 1e-9
    assert np.max(np.abs(_grad(shim, 1, pl, D, D2, (1, 0, 0)) - z["Kgr3"])) < 1e-9
    assert np.max(np.abs(_grad(shim, 1, pl, D2, D, (0, 1, 0)) - z["Kgr4"])) < 1e-9
