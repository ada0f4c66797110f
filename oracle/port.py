"""numpy/ctypes front end of the oracle's C restatement (oracle/jk_port.c,
built into oracle/_ref/libjk_port.so). Test infrastructure only.

Pure <-> Cartesian transforms use real solid harmonics rebuilt here from the
published recursion (Helgaker, Jorgensen & Olsen eqs. 6.4.70-6.4.73, the
construction of the reference's src/cpp/core/am.cpp:74-220), so the oracle
shares no code with the product.
"""
import ctypes
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libjk_port.so")
_lib = None


def available():
    return os.path.exists(LIB)


class PBasis(ctypes.Structure):
    _fields_ = [("nprim", ctypes.c_int), ("c", ctypes.c_void_p), ("e", ctypes.c_void_p), ("xyz", ctypes.c_void_p),
                ("L", ctypes.c_void_p), ("cart", ctypes.c_void_p), ("ncart", ctypes.c_int)]


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(LIB)
        _lib.port_pairs.restype = ctypes.c_long
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def solid_harmonics(L):
    """coef[pure m = 0,+1,-1,+2,-2,..][cart CCA lexical]"""
    def add(dst, a, src, dx, dy, dz):
        for (lx, ly, lz), v in src.items():
            k = (lx + dx, ly + dy, lz + dz)
            dst[k] = dst.get(k, 0.0) + a * v

    def prune(p):
        return {k: v for k, v in p.items() if abs(v) > 1e-15}

    Sc = [dict() for _ in range(L + 1)]
    Ss = [dict() for _ in range(L + 1)]
    Sc[0][(0, 0, 0)] = 1.0
    for l in range(L):
        Nc = math.sqrt((2.0 if l == 0 else 1.0) * (2 * l + 1) / (2 * l + 2))
        Ns = 0.0 if l == 0 else Nc
        c, s = {}, {}
        add(c, Nc, Sc[l], 1, 0, 0)
        add(s, Nc, Sc[l], 0, 1, 0)
        add(c, -Ns, Ss[l], 0, 1, 0)
        add(s, Ns, Ss[l], 1, 0, 0)
        Sc[l + 1], Ss[l + 1] = prune(c), prune(s)
    out = [None] * (2 * L + 1)
    for m in range(L + 1):
        cc, cs, pc, ps = Sc[m], Ss[m], {}, {}
        for l in range(m, L):
            a = (2 * l + 1) / math.sqrt((l + m + 1.0) * (l - m + 1.0))
            b = math.sqrt(((l + m) * float(l - m)) / ((l + m + 1.0) * (l - m + 1.0)))
            nc, ns = {}, {}
            add(nc, a, cc, 0, 0, 1)
            add(ns, a, cs, 0, 0, 1)
            for d in range(3):
                sh = [2 if d == q else 0 for q in range(3)]
                add(nc, -b, pc, *sh)
                add(ns, -b, ps, *sh)
            pc, ps, cc, cs = cc, cs, prune(nc), prune(ns)
        if m == 0:
            out[0] = cc
        else:
            out[2 * m - 1], out[2 * m] = cc, cs
    ncart = (L + 1) * (L + 2) // 2
    C = np.zeros((2 * L + 1, ncart))
    for p in range(2 * L + 1):
        for (lx, ly, lz), v in out[p].items():
            i = L - lx
            C[p, i * (i + 1) // 2 + lz] += v
    return C


class Basis:
    """Primitive arrays of a basis (from any object with .primitives) plus the
    pure<-cart matrix T (nao x ncart): X_pure = T X_cart T^T, D_cart = T^T D T."""

    def __init__(self, prims):
        self.c = np.array([p.c for p in prims])
        self.e = np.array([p.e for p in prims])
        self.xyz = np.ascontiguousarray(np.array([[p.x, p.y, p.z] for p in prims]).reshape(-1, 3))
        self.L = np.array([p.L for p in prims], np.int32)
        self.cart = np.array([p.cartIdx for p in prims], np.int32)
        if np.any(self.L > 2):
            raise ValueError("oracle port supports s, p, d shells")
        last = prims[-1]
        self.nao = last.aoIdx + last.nao
        self.ncart = last.cartIdx + last.ncart
        self.T = np.zeros((self.nao, self.ncart))
        for k, p in enumerate(prims):
            if k and p.shellIdx == prims[k - 1].shellIdx:
                continue
            if p.is_pure:
                self.T[p.aoIdx:p.aoIdx + p.nao, p.cartIdx:p.cartIdx + p.ncart] = solid_harmonics(p.L)
            else:
                self.T[p.aoIdx:p.aoIdx + p.nao, p.cartIdx:p.cartIdx + p.ncart] = np.eye(p.ncart)
        self.s = PBasis(len(prims), _p(self.c), _p(self.e), _p(self.xyz), _p(self.L), _p(self.cart), self.ncart)


class Pairs:
    """Schwarz pair list sorted like the reference: class (L1, L2), bound desc,
    prim1 asc, prim2 asc (pair_list_util.cpp:12-20)."""

    def __init__(self, b1, b2, symm, thre):
        n = len(b1.c) * len(b2.c)
        pa, pb = np.zeros(n, np.int32), np.zeros(n, np.int32)
        bd = np.zeros(n, np.float32)
        m = lib().port_pairs(ctypes.byref(b1.s), ctypes.byref(b2.s), int(symm), ctypes.c_float(thre), _p(pa), _p(pb),
                             _p(bd))
        pa, pb, bd = pa[:m], pb[:m], bd[:m]
        cls = b1.L[pa] * 16 + b2.L[pb]
        order = np.lexsort((pb, pa, -bd.astype(np.float64), cls))
        self.b1, self.b2, self.symm = b1, b2, bool(symm)
        self.pa = np.ascontiguousarray(pa[order])
        self.pb = np.ascontiguousarray(pb[order])
        self.bound = np.ascontiguousarray(bd[order])
        self.L1 = b1.L[self.pa]
        self.L2 = b2.L[self.pb]


def _ew(scales, omegas):
    return np.ascontiguousarray(scales, np.float64), np.ascontiguousarray(omegas, np.float64)


def coulomb(pl12, pl34, D, thresp, scales=(1.0,), omegas=(-1.0,)):
    """J12 (pure) for D34 (pure), one build."""
    s, o = _ew(scales, omegas)
    Dc = np.ascontiguousarray(pl34.b1.T.T @ D @ pl34.b2.T)
    Jc = np.zeros((pl12.b1.ncart, pl12.b2.ncart))
    lib().port_coulomb(ctypes.byref(pl12.b1.s), ctypes.byref(pl12.b2.s), ctypes.c_long(len(pl12.pa)), _p(pl12.pa),
                       _p(pl12.pb), _p(pl12.bound), int(pl12.symm), ctypes.byref(pl34.b1.s), ctypes.byref(pl34.b2.s),
                       ctypes.c_long(len(pl34.pa)), _p(pl34.pa), _p(pl34.pb), _p(pl34.bound), int(pl34.symm), _p(Dc),
                       len(s), _p(s), _p(o), ctypes.c_float(thresp), _p(Jc))
    return pl12.b1.T @ Jc @ pl12.b2.T.T


def exchange(pl12, pl34, D, D24symm, thresp, scales=(1.0,), omegas=(-1.0,), equivalent13=None):
    """K13 (pure) for D24 (pure), one build. D24symm needs basis2 == basis4;
    the transposed write is used only if basis1 == basis3 too."""
    s, o = _ew(scales, omegas)
    Dc = np.ascontiguousarray(pl12.b2.T.T @ D @ pl34.b2.T)
    Kc = np.zeros((pl12.b1.ncart, pl34.b1.ncart))
    eq13 = equivalent13 if equivalent13 is not None else (pl12.b1 is pl34.b1)
    lib().port_exchange(ctypes.byref(pl12.b1.s), ctypes.byref(pl12.b2.s), ctypes.c_long(len(pl12.pa)), _p(pl12.pa),
                        _p(pl12.pb), _p(pl12.bound), int(pl12.symm), ctypes.byref(pl34.b1.s), ctypes.byref(pl34.b2.s),
                        ctypes.c_long(len(pl34.pa)), _p(pl34.pa), _p(pl34.pb), _p(pl34.bound), int(pl34.symm), _p(Dc),
                        int(bool(D24symm) and eq13), len(s), _p(s), _p(o), ctypes.c_float(thresp), _p(Kc))
    return pl12.b1.T @ Kc @ pl34.b1.T.T


def count_quartets(pl12, pl34, DJ, DK, DK_symm, thresp, equivalent13=None):
    """(J quartets, K quartets) the reference evaluates for J with D34 = DJ
    and K with D24 = DK (pure matrices) -- the shared counting routine that
    turns a measured time into quartets/s for the CPU and the GPU alike."""
    lib().port_count_j.restype = ctypes.c_double
    lib().port_count_k.restype = ctypes.c_double
    DJc = np.ascontiguousarray(pl34.b1.T.T @ DJ @ pl34.b2.T)
    DKc = np.ascontiguousarray(pl12.b2.T.T @ DK @ pl34.b2.T)
    eq13 = equivalent13 if equivalent13 is not None else (pl12.b1 is pl34.b1)
    args = (ctypes.byref(pl12.b1.s), ctypes.byref(pl12.b2.s), ctypes.c_long(len(pl12.pa)), _p(pl12.pa),
            _p(pl12.pb), _p(pl12.bound), int(pl12.symm), ctypes.byref(pl34.b1.s), ctypes.byref(pl34.b2.s),
            ctypes.c_long(len(pl34.pa)), _p(pl34.pa), _p(pl34.pb), _p(pl34.bound), int(pl34.symm))
    nj = lib().port_count_j(*args, _p(DJc), ctypes.c_float(thresp))
    nk = lib().port_count_k(*args, _p(DKc), int(bool(DK_symm) and eq13), ctypes.c_float(thresp))
    return nj, nk
