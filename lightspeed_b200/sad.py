"""Superposition-of-atomic-densities (SAD) SCF guess.

Follows the reference's SAD (src/cpp/sad/sad.cpp:17-163,
src/lightspeed/sad.hpp:15-40): the fully contracted core + valence orbitals
of the cc-pVDZ "MinAO" basis are occupied fractionally -- core orbitals with
one electron pair, the valence pairs of the neutral atom spread evenly over
the valence orbitals -- and projected into the target basis atom by atom:

    A = S12^T C1,  M = A^T S22^-1 A,  C2 = S22^-1 A M^-1/2,
    Csad[:, i] = C2[:, i] sqrt(nocc_i),  D = Csad Csad^T

(S12: MinAO x target overlap of one atom, S22: target overlap of that atom,
C1 = identity). Each atom's block depends only on its element (the
projection of a free atom is translation and rotation invariant for these
spherically averaged occupations), so the block is computed once per element
and basis and placed on the diagonal.
"""
import numpy as np

# Valence layout of the MinAO basis (the reference's convention,
# data/basis/cc-pvdz-minao.gbs header): [frozen][valence] per row of the table.
_CORE_FUNCS = {1: 0, 2: 0, 3: 1, 4: 1, 5: 1, 6: 1, 7: 1, 8: 1, 9: 1, 10: 1}


def minao_nocc(Z, nfunc):
    """Electron-pair occupations of the MinAO functions of a neutral atom."""
    ncore = _CORE_FUNCS[Z]
    nval = nfunc - ncore
    pairs = 0.5 * Z - ncore
    return np.array([1.0] * ncore + [pairs / nval] * nval)


def _atom_blocks(basis):
    """(atom index, first AO, AO count) per atom, in AO order."""
    lo, hi = {}, {}
    for p in basis.primitives:
        n = (2 * p.L + 1) if p.is_pure else (p.L + 1) * (p.L + 2) // 2
        a = p.atomIdx
        lo[a] = min(lo.get(a, p.aoIdx), p.aoIdx)
        hi[a] = max(hi.get(a, p.aoIdx + n), p.aoIdx + n)
    return [(a, lo[a], hi[a] - lo[a]) for a in sorted(lo)]


class SAD:
    """SAD densities for molecules in one target basis (blocks cached per element)."""

    def __init__(self, ls, basis_name, minao_name="cc-pvdz-minao", thre_pow=1.0e-12):
        self.ls = ls
        self.basis_name = basis_name
        self.minao_name = minao_name
        self.thre_pow = thre_pow
        self._blocks = {}

    def _power(self, M, p):
        w, U = np.linalg.eigh(0.5 * (M + M.T))
        keep = w > self.thre_pow * max(w.max(), 1.0)
        return (U[:, keep] * w[keep] ** p) @ U[:, keep].T

    def atom_block(self, symbol, Z):
        key = symbol.upper()
        if key in self._blocks:
            return self._blocks[key]
        ls = self.ls
        mol = ls.Molecule.from_arrays([symbol], np.zeros((1, 3)), name="atom_" + symbol)
        b1 = ls.Basis.from_gbs_file(mol, self.minao_name)
        b2 = ls.Basis.from_gbs_file(mol, self.basis_name)
        res = ls.ResourceList.build()
        S12 = ls.IntBox.overlap(res, ls.PairList.build_schwarz(b1, b2, False, 1.0e-14)).np.copy()
        S22 = ls.IntBox.overlap(res, ls.PairList.build_schwarz(b2, b2, True, 1.0e-14)).np.copy()
        C1 = np.eye(b1.nao)
        S22inv = self._power(S22, -1.0)
        A = S12.T @ C1
        M = A.T @ S22inv @ A
        C2 = S22inv @ A @ self._power(M, -0.5)
        C = C2 * np.sqrt(minao_nocc(Z, b1.nao))[None, :]
        D = C @ C.T
        self._blocks[key] = D
        return D

    def density(self, mol, basis):
        """SAD density (electron pairs: tr(D S) = N/2 for a neutral molecule)."""
        D = np.zeros((basis.nao, basis.nao))
        atoms = mol.atoms
        for a, lo, n in _atom_blocks(basis):
            at = atoms[a]
            blk = self.atom_block(at.symbol, int(round(at.Z)))
            if blk.shape[0] != n:
                raise RuntimeError("SAD: atom %d block size %d != %d" % (a, blk.shape[0], n))
            D[lo:lo + n, lo:lo + n] = blk
        return D
