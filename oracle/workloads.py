"""Benchmark inputs restated for the oracle side (test infrastructure): the
all-trans alkane geometry and Gaussian basis sets from GBS files, built here
without the product package so the reference CPU IntBox (oracle/_ref) can be
driven on its own -- the reference arm of bench.py and the fixture scripts
use only this module, oracle/ref.py and oracle/port.py.

* alkane(n): all-trans CnH(2n+2), C-C 1.54 A, C-H 1.09 A, tetrahedral
  angles, zig-zag in the xz plane (Bohr, 0.52917720859 A per Bohr, the value
  of the reference's src/python/util.py:3).
* basis(symbols, xyz, gbs_path): the primitive arrays ref.RefBasis takes,
  normalised like the reference's Basis.from_gbs_file
  (src/python/core.py:265-548): each contraction coefficient times
  sqrt(2^L (2e)^(L+3/2) / (pi^(3/2) (2L-1)!!)) and the contracted shell
  rescaled to norm N, dense aoIdx / cartIdx / primIdx / shellIdx / atomIdx.
"""
import math
import os
import re

import numpy as np

ANG_PER_BOHR = 0.52917720859
Z = {"H": 1, "HE": 2, "LI": 3, "BE": 4, "B": 5, "C": 6, "N": 7, "O": 8, "F": 9, "NE": 10}
_SHELL_L = {"S": 0, "P": 1, "D": 2, "F": 3, "G": 4}
BASIS_DIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "lightspeed_b200", "data",
                         "basis")


def alkane(n_carbon):
    """(symbols, xyz in Bohr) of all-trans CnH(2n+2)."""
    tet = math.acos(-1.0 / 3.0)
    half = tet / 2.0
    cc, ch = 1.54, 1.09
    dx, dz = cc * math.sin(half), cc * math.cos(half)
    carbons = [np.array([k * dx, 0.0, (k % 2) * dz]) for k in range(n_carbon)]
    symbols = ["C"] * n_carbon
    xyz = list(carbons)
    for k, c in enumerate(carbons):
        up = 1.0 if k % 2 else -1.0
        b = np.array([0.0, 0.0, up])
        for sgn in (1.0, -1.0):
            symbols.append("H")
            xyz.append(c + ch * (math.cos(half) * b + math.sin(half) * np.array([0.0, sgn, 0.0])))
    for k, sgn in ((0, -1.0), (n_carbon - 1, 1.0)):
        up = 1.0 if k % 2 else -1.0
        d = np.array([sgn * math.sin(half), 0.0, -up * math.cos(half)])
        symbols.append("H")
        xyz.append(carbons[k] + ch * d / np.linalg.norm(d))
    return symbols, np.array(xyz) * (1.0 / ANG_PER_BOHR)


def nuclear_charge(symbols):
    return sum(Z[s.upper()] for s in symbols)


def nuclear_repulsion(symbols, xyz):
    e = 0.0
    for a in range(len(symbols)):
        for b in range(a):
            e += Z[symbols[a].upper()] * Z[symbols[b].upper()] / np.linalg.norm(xyz[a] - xyz[b])
    return e


def _parse_gbs(path):
    lines = [l for l in open(path) if l.strip() and not l.lstrip().startswith("!")]
    spherical = lines[0].strip().lower() == "spherical"
    atoms, cur, sym, i = {}, None, None, 1
    while i < len(lines):
        s = lines[i].split()
        if s[0] == "****":
            cur, sym = None, None
            i += 1
            continue
        if cur is None:
            sym, cur = s[0].upper(), []
            atoms[sym] = cur
            i += 1
            continue
        kind, nprim, norm = s[0].upper(), int(s[1]), float(s[2])
        rows = [re.sub(r"[Dd]", "E", lines[i + 1 + q]).split() for q in range(nprim)]
        es = [float(r[0]) for r in rows]
        if kind in ("SP", "SPD"):
            for col in range(len(kind)):
                cur.append((col, norm, [float(r[1 + col]) for r in rows], es))
        else:
            cur.append((_SHELL_L[kind], norm, [float(r[1]) for r in rows], es))
        i += 1 + nprim
    return spherical, atoms


def _normalized(L, N, ws, es):
    dfact = 1
    for l in range(1, L + 1):
        dfact *= 2 * l - 1
    pi32 = math.pow(math.pi, 1.5)
    cs = [w * math.sqrt(math.pow(2, L) * math.pow(e + e, L + 1.5) / (pi32 * dfact)) for w, e in zip(ws, es)]
    V = 0.0
    for a in range(len(ws)):
        for b in range(len(ws)):
            V += math.pow(math.sqrt(4 * es[a] * es[b]) / (es[a] + es[b]), L + 1.5) * ws[a] * ws[b]
    V = math.sqrt(N) * math.pow(V, -0.5)
    return [V * c for c in cs]


class Prim:
    """One primitive with the attribute names oracle/port.py reads."""

    def __init__(self, **kw):
        self.__dict__.update(kw)


def basis(symbols, xyz, name):
    """-> (arrays for ref.RefBasis, [Prim] for port.Basis, nao)."""
    spherical, shells = _parse_gbs(os.path.join(BASIS_DIR, name + ".gbs"))
    prims = []
    nao = ncart = nshell = 0
    for A, sym in enumerate(symbols):
        for (L, N, ws, es) in shells[sym.upper()]:
            nfun = 2 * L + 1 if spherical else (L + 1) * (L + 2) // 2
            nc = (L + 1) * (L + 2) // 2
            for c, e, w in zip(_normalized(L, N, ws, es), es, ws):
                prims.append(Prim(c=c, e=e, x=xyz[A][0], y=xyz[A][1], z=xyz[A][2], c0=w, L=L, is_pure=spherical,
                                  aoIdx=nao, cartIdx=ncart, primIdx=len(prims), shellIdx=nshell, atomIdx=A,
                                  nao=nfun, ncart=nc))
            nao += nfun
            ncart += nc
            nshell += 1
    arrays = dict(c=np.array([p.c for p in prims]), e=np.array([p.e for p in prims]),
                  xyz=np.array([[p.x, p.y, p.z] for p in prims]).reshape(-1, 3),
                  c0=np.array([p.c0 for p in prims]), L=np.array([p.L for p in prims], np.int32),
                  pure=np.array([int(p.is_pure) for p in prims], np.int32),
                  ao=np.array([p.aoIdx for p in prims], np.int32), cart=np.array([p.cartIdx for p in prims], np.int32),
                  prim=np.array([p.primIdx for p in prims], np.int32),
                  shell=np.array([p.shellIdx for p in prims], np.int32),
                  atom=np.array([p.atomIdx for p in prims], np.int32))
    return arrays, prims, nao
