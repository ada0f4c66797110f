"""ctypes access to the reference Lightspeed CPU IntBox built by oracle/Makefile
(oracle/_ref/libls_ref.so). Test infrastructure only: tests, smoke() and the
CPU-baseline leg of bench.py use it as the checker; the product never does.
"""
import ctypes
import os
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libls_ref.so")

_lib = None


def available():
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(LIB)
        vp, ip, dp, fp = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_float
        _lib.ref_basis_new.restype = vp
        _lib.ref_pairlist_new.restype = vp
        _lib.ref_pairlist_new.argtypes = [vp, vp, ip, fp]
        _lib.ref_pairlist_count.restype = ctypes.c_long
        _lib.ref_pairlist_count.argtypes = [vp]
        _lib.ref_pairlist_export.argtypes = [vp] + [vp] * 5
        _lib.ref_basis_free.argtypes = [vp]
        _lib.ref_pairlist_free.argtypes = [vp]
        _lib.ref_last_error.restype = ctypes.c_char_p
        _lib.ref_coulomb.argtypes = [vp, vp, ip, vp, vp, vp, fp, fp, vp, ip]
        _lib.ref_exchange.argtypes = [vp, vp, ip, vp, vp, vp, ip, fp, fp, vp, ip]
        _lib.ref_overlap.argtypes = [vp, vp, ip]
        _lib.ref_kinetic.argtypes = [vp, vp, ip]
        _lib.ref_potential.argtypes = [vp, ip, vp, vp, ip, vp, vp, ip]
        _lib.ref_rys.argtypes = [ip, ip, vp, vp, vp]
        # every handle and pointer argument typed: an untyped Python int goes through
        # ctypes as a 32-bit C int, which cuts a 64-bit handle short
        _lib.ref_basis_nao.argtypes = [vp]
        _lib.ref_basis_ncart.argtypes = [vp]
        _lib.ref_coulomb_grad.argtypes = [vp, ip, vp, vp, vp, vp, ip, fp, fp, vp, ip]
        _lib.ref_exchange_grad.argtypes = [vp, ip, vp, vp, vp, vp, ip, ip, ip, fp, fp, vp, ip]
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _check(rc):
    if rc != 0:
        raise RuntimeError("reference IntBox: " + lib().ref_last_error().decode())


class RefBasis:
    """A reference lightspeed::Basis built from primitive arrays (see prim_arrays)."""

    def __init__(self, arrs):
        self.arrs = {k: np.ascontiguousarray(v) for k, v in arrs.items()}
        a = self.arrs
        n = len(a["c"])
        self.h = lib().ref_basis_new(n, _p(a["c"]), _p(a["e"]), _p(a["xyz"]), _p(a["c0"]), _p(a["L"]),
                                     _p(a["pure"]), _p(a["ao"]), _p(a["cart"]), _p(a["prim"]), _p(a["shell"]),
                                     _p(a["atom"]))
        if not self.h:
            _check(1)
        self.nao = lib().ref_basis_nao(self.h)
        self.ncart = lib().ref_basis_ncart(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            lib().ref_basis_free(self.h)


class RefPairs:
    def __init__(self, b1, b2, symm, thre):
        self.b1, self.b2 = b1, b2
        self.h = lib().ref_pairlist_new(b1.h, b2.h, 1 if symm else 0, thre)
        if not self.h:
            _check(1)

    def export(self):
        n = lib().ref_pairlist_count(self.h)
        L1, L2, p1, p2 = (np.zeros(n, np.int32) for _ in range(4))
        b = np.zeros(n, np.float32)
        lib().ref_pairlist_export(self.h, _p(L1), _p(L2), _p(p1), _p(p2), _p(b))
        return L1, L2, p1, p2, b

    def __del__(self):
        if getattr(self, "h", None):
            lib().ref_pairlist_free(self.h)


def prim_arrays(basis):
    """Primitive arrays of an ls.Basis (lightspeed_b200) for the reference."""
    P = basis.primitives
    return dict(c=np.array([p.c for p in P]), e=np.array([p.e for p in P]),
                xyz=np.array([[p.x, p.y, p.z] for p in P]).reshape(-1, 3), c0=np.array([p.c0 for p in P]),
                L=np.array([p.L for p in P], np.int32), pure=np.array([int(p.is_pure) for p in P], np.int32),
                ao=np.array([p.aoIdx for p in P], np.int32), cart=np.array([p.cartIdx for p in P], np.int32),
                prim=np.array([p.primIdx for p in P], np.int32), shell=np.array([p.shellIdx for p in P], np.int32),
                atom=np.array([p.atomIdx for p in P], np.int32))


def _ewald(scales, omegas):
    return np.ascontiguousarray(scales, np.float64), np.ascontiguousarray(omegas, np.float64)


def coulomb(pl12, pl34, D, thresp, thredp, scales=(1.0,), omegas=(-1.0,), J=None, nthread=0):
    s, o = _ewald(scales, omegas)
    D = np.ascontiguousarray(D, np.float64)
    out = np.zeros((pl12.b1.nao, pl12.b2.nao)) if J is None else np.array(J, np.float64, copy=True)
    _check(lib().ref_coulomb(pl12.h, pl34.h, len(s), _p(s), _p(o), _p(D), thresp, thredp, _p(out), nthread))
    return out


def exchange(pl12, pl34, D, symm, thresp, thredp, scales=(1.0,), omegas=(-1.0,), K=None, nthread=0):
    s, o = _ewald(scales, omegas)
    D = np.ascontiguousarray(D, np.float64)
    out = np.zeros((pl12.b1.nao, pl34.b1.nao)) if K is None else np.array(K, np.float64, copy=True)
    _check(lib().ref_exchange(pl12.h, pl34.h, len(s), _p(s), _p(o), _p(D), 1 if symm else 0, thresp, thredp,
                              _p(out), nthread))
    return out


def overlap(pl, nthread=0):
    out = np.zeros((pl.b1.nao, pl.b2.nao))
    _check(lib().ref_overlap(pl.h, _p(out), nthread))
    return out


def kinetic(pl, nthread=0):
    out = np.zeros((pl.b1.nao, pl.b2.nao))
    _check(lib().ref_kinetic(pl.h, _p(out), nthread))
    return out


def potential(pl, xyzZ, scales=(1.0,), omegas=(-1.0,), nthread=0):
    s, o = _ewald(scales, omegas)
    X = np.ascontiguousarray(xyzZ, np.float64)
    out = np.zeros((pl.b1.nao, pl.b2.nao))
    _check(lib().ref_potential(pl.h, len(s), _p(s), _p(o), X.shape[0], _p(X), _p(out), nthread))
    return out


def coulomb_grad(pl, D12, D34=None, thresp=1e-14, thredp=1e-14, scales=(1.0,), omegas=(-1.0,), G=None,
                 nthread=0):
    """IntBox::coulombGrad: G (natom x 3) += sum D12 d(12|34) D34 (D34 None: the
    same matrix, the reference's D12 == D34 branch)."""
    s, o = _ewald(scales, omegas)
    A = np.ascontiguousarray(D12, np.float64)
    B = A if D34 is None else np.ascontiguousarray(D34, np.float64)
    natom = int(pl.b1.arrs["atom"][-1]) + 1
    out = np.zeros((natom, 3)) if G is None else np.array(G, np.float64, copy=True)
    _check(lib().ref_coulomb_grad(pl.h, len(s), _p(s), _p(o), _p(A), _p(B), int(D34 is None), ctypes.c_float(thresp),
                                  ctypes.c_float(thredp), _p(out), nthread))
    return out


def exchange_grad(pl, D13, D24=None, D13symm=True, D24symm=True, thresp=1e-14, thredp=1e-14, scales=(1.0,),
                  omegas=(-1.0,), G=None, nthread=0):
    """IntBox::exchangeGrad: G (natom x 3) += sum D13 d(12|34) D24 (D24 None: the
    same matrix, Dsame)."""
    s, o = _ewald(scales, omegas)
    A = np.ascontiguousarray(D13, np.float64)
    B = A if D24 is None else np.ascontiguousarray(D24, np.float64)
    natom = int(pl.b1.arrs["atom"][-1]) + 1
    out = np.zeros((natom, 3)) if G is None else np.array(G, np.float64, copy=True)
    _check(lib().ref_exchange_grad(pl.h, len(s), _p(s), _p(o), _p(A), _p(B), int(D13symm), int(D24symm),
                                   int(D24 is None), ctypes.c_float(thresp), ctypes.c_float(thredp), _p(out), nthread))
    return out


def rys(nrys, T):
    T = np.ascontiguousarray(T, np.float64)
    t = np.zeros((len(T), nrys))
    w = np.zeros((len(T), nrys))
    _check(lib().ref_rys(nrys, len(T), _p(T), _p(t), _p(w)))
    return t, w


def eri_j(pl12, pl34, C1, C2, C3, C4, thresp, thredp, sym12, sym34, sym1234, scales=(1.0,), omegas=(-1.0,)):
    """IntBox::eriJ restated over the reference's own CPU coulomb
    (src/cpp/intbox/mo_eri.cpp:10-157): one J build per (i, j) (i >= j when
    sym12) of D = C1[:, i] C2[:, j]^T with bra pl34 and ket pl12 (:74-95),
    I[i, j] = C3^T J C4 (:96-118), then the symmetrisations of :121-155 in
    that order; the flags stand for its object-identity tests."""
    n1, n2, n3, n4 = C1.shape[1], C2.shape[1], C3.shape[1], C4.shape[1]
    I = np.zeros((n1, n2, n3, n4))
    for i in range(n1):
        for j in range(n2):
            if sym12 and i < j:
                continue
            D = np.outer(C1[:, i], C2[:, j])
            J = coulomb(pl34, pl12, D, thresp, thredp, scales, omegas)
            L = C3.T @ J @ C4
            I[i, j] = L
            if sym12 and i != j:
                I[j, i] = L
    if sym12:
        for p in range(n1):
            for q in range(p):
                I[p, q] = I[q, p] = 0.5 * (I[p, q] + I[q, p])
    if sym34:
        for r in range(n3):
            for s in range(r):
                I[:, :, r, s] = I[:, :, s, r] = 0.5 * (I[:, :, r, s] + I[:, :, s, r])
    if sym1234:
        M = I.reshape(n1 * n2, n3 * n4)
        for pq in range(n1 * n2):
            for rs in range(pq):
                M[pq, rs] = M[rs, pq] = 0.5 * (M[pq, rs] + M[rs, pq])
    return I
