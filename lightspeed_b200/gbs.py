"""Gaussian basis sets from GBS files, normalised the Lightspeed way.

Reads the Gaussian-94 style .gbs format (first line 'cartesian' or
'spherical', atoms separated by '****', shells 'S/P/D/.. K N' or 'SP'/'SPD')
and builds the primitive list of a Basis exactly as the reference's
Basis.from_gbs_file does (src/python/core.py:265-548): contraction
coefficients are multiplied by the primitive normalisation
  sqrt(2^L (2e)^(L+3/2) / (pi^(3/2) (2L-1)!!))
and the contracted shell is rescaled to norm N (the third field of the shell
line); primitives carry dense aoIdx / cartIdx / primIdx / shellIdx / atomIdx.
"""
import math
import os
import re

_SHELL_L = {"S": 0, "P": 1, "D": 2, "F": 3, "G": 4, "H": 5, "I": 6}

BASIS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "basis")


def _normalized(am, N, ws, es):
    pi32 = math.pow(math.pi, 1.5)
    twoL = math.pow(2, am)
    dfact = 1
    for l in range(1, am + 1):
        dfact *= 2 * l - 1
    cs = [w * math.sqrt(twoL * math.pow(e + e, am + 1.5) / (pi32 * dfact)) for w, e in zip(ws, es)]
    V = 0.0
    for k1 in range(len(ws)):
        for k2 in range(len(ws)):
            V += math.pow(math.sqrt(4 * es[k1] * es[k2]) / (es[k1] + es[k2]), am + 1.5) * ws[k1] * ws[k2]
    V = math.sqrt(N) * math.pow(V, -0.5)
    return [V * c for c in cs]


def parse_gbs_lines(lines):
    """-> (spherical flag, {SYMBOL: [shell, ...]}) with shell = (L, N, [w], [e])."""
    body = [l for l in lines if not re.match(r"^\s*$", l) and not re.match(r"^\s*!", l)]
    if re.match(r"^\s*cartesian\s*$", body[0], re.IGNORECASE):
        spherical = False
    elif re.match(r"^\s*spherical\s*$", body[0], re.IGNORECASE):
        spherical = True
    else:
        raise ValueError("GBS file: where is the cartesian/spherical line?")
    body = body[1:]
    stars = [0] + [k for k, l in enumerate(body) if re.match(r"^\s*\*\*\*\*\s*$", l)] + [len(body)]
    atoms = {}
    for k in range(len(stars) - 1):
        i1, i2 = stars[k] + 1, stars[k + 1]
        if i2 - i1 <= 0:
            continue
        m = re.match(r"^\s*(\S+)\s+(\d+)\s*$", body[i1])
        if m is None:
            raise ValueError("GBS file: where is the ID V line?")
        if m.group(2) != "0":
            continue
        symbol = m.group(1).upper()
        block = body[i1 + 1:i2]
        shells = []
        ind = 0
        while ind < len(block):
            m = re.match(r"^\s*(\S+)\s+(\d+)\s+(\S+)\s*$", block[ind])
            if m is None:
                raise ValueError("GBS file: where is the L K N line?")
            ID, K, N = m.group(1).upper(), int(m.group(2)), float(m.group(3))
            ind += 1
            rows = [re.sub(r"[Dd]", "E", block[ind + q]).split() for q in range(K)]
            es = [float(r[0]) for r in rows]
            if ID in ("SP", "SPD"):
                for col, L in enumerate(range(len(ID))):
                    shells.append((L, N, [float(r[1 + col]) for r in rows], es))
            else:
                shells.append((_SHELL_L[ID], N, [float(r[1]) for r in rows], es))
            ind += K
        atoms[symbol] = shells
    return spherical, atoms


def basis_from_gbs_lines(ls, molecule, lines, name="bas", normalize=True, spherical=None):
    sph_file, atom_shells = parse_gbs_lines(lines)
    if spherical is None:
        spherical = sph_file
    prims = []
    nao = ncart = nprim = nshell = 0
    for A, atom in enumerate(molecule.atoms):
        if atom.symbol not in atom_shells:
            raise ValueError("basis %s has no entry for %s" % (name, atom.symbol))
        for (L, N, ws, es) in atom_shells[atom.symbol]:
            cs = _normalized(L, N, ws, es) if normalize else list(ws)
            nfun = (2 * L + 1) if spherical else (L + 1) * (L + 2) // 2
            for c, e, w in zip(cs, es, ws):
                prims.append(ls.Primitive(c, e, atom.x, atom.y, atom.z, w, L, spherical, nao, ncart, nprim,
                                          nshell, A))
                nprim += 1
            nao += nfun
            ncart += (L + 1) * (L + 2) // 2
            nshell += 1
    return ls.Basis(name, prims)


def basis_from_gbs_file(ls, molecule, filename, normalize=True, spherical=None):
    if len(filename) >= 4 and filename[-4:] != ".gbs":
        filename += ".gbs"
    if not os.path.isfile(filename):
        filename = os.path.join(BASIS_DIR, filename)
    if not os.path.isfile(filename):
        raise ValueError("Could not find GBS file: %s" % filename)
    with open(filename) as fh:
        lines = fh.readlines()
    name = os.path.basename(filename)[:-4]
    return basis_from_gbs_lines(ls, molecule, lines, name=name, normalize=normalize, spherical=spherical)
