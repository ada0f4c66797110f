"""CPU-only checks of the boundary: the C-ABI library loads, exports every
entry point include/lsjk.h declares, and fails loudly (error code + message,
no CPU fallback) when no GPU is usable."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in ("lsjk.h", "lsmlp.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        names |= set(re.findall(r"\b(ls(?:jk|mlp)_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_header_symbols_exported(ls):
    lib = ctypes.CDLL(ls.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 26
    for n in names:
        assert hasattr(lib, n), n


def test_version_and_error_string(ls):
    lib = ctypes.CDLL(ls.LIB_PATH)
    lib.lsjk_version.restype = ctypes.c_char_p
    lib.lsjk_last_error.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.lsjk_version()
    assert isinstance(lib.lsjk_last_error(), bytes)


def test_null_arguments_rejected(ls):
    lib = ctypes.CDLL(ls.LIB_PATH)
    lib.lsjk_last_error.restype = ctypes.c_char_p
    assert lib.lsjk_context_create(0, None) == 1          # LSJK_EINVAL
    assert lib.lsjk_coulomb(None, 1, None, None, None, None, 0, None, ctypes.c_float(0), ctypes.c_float(0), None) == 1
    assert lib.lsjk_last_error() != b""


def test_no_gpu_fails_loudly(ls):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    mol = ls.Molecule.from_xyz_file(os.path.join(ROOT, "tests", "golden", "h2o.xyz"))
    bas = ls.Basis.from_gbs_file(mol, "sto-3g")
    with pytest.raises(RuntimeError):
        ls.PairList.build_schwarz(bas, bas, True, 1e-14)


def test_basis_sizes_and_density_checks(ls):
    mol = ls.Molecule.from_xyz_file(os.path.join(ROOT, "tests", "golden", "h2o.xyz"))
    for name, nao, ncart in (("sto-3g", 7, 7), ("6-31gs", 19, 19), ("cc-pvdz", 24, 25)):
        b = ls.Basis.from_gbs_file(mol, name)
        assert (b.nao, b.ncart) == (nao, ncart)
    p = ls.Primitive(1.0, 1.0, 0.0, 0.0, 0.0, 1.0, 0, False, 0, 0, 1, 0, 0)
    with pytest.raises(Exception, match="primIdx"):
        ls.Basis("bad", [p])


def test_tensor_numpy_view(ls):
    t = ls.Tensor.array(np.arange(12.0).reshape(3, 4))
    assert t.shape == (3, 4)
    v = t.np
    v[1, 2] = -5.0
    assert t.np[1, 2] == -5.0
    assert np.asarray(t).shape == (3, 4)


def test_eri_j_rejects_more_than_65535_c3_orbitals(ls):
    """lsjk_eri_j's C3 count is the grid height of its left contraction kernel:
    65536 orbitals are refused before any device work, with LSJK_EINVAL."""
    lib = ctypes.CDLL(ls.LIB_PATH)
    lib.lsjk_last_error.restype = ctypes.c_char_p
    f = ctypes.c_float(1e-14)
    rc = lib.lsjk_eri_j(None, 1, None, None, None, None, 1, 1, 65536, 1, None, None, None, None, 0, 0, 0, f, f,
                        None)
    assert rc == 1   # LSJK_EINVAL
    assert b"65535" in lib.lsjk_last_error()
    rc = lib.lsjk_eri_j(None, 1, None, None, None, None, 1, 1, 65535, 1, None, None, None, None, 0, 0, 0, f, f,
                        None)
    assert rc == 1 and b"null argument" in lib.lsjk_last_error()
