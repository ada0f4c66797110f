"""Atoms and molecules (Bohr), with the reference's xyz-file conventions.

Mirrors lightspeed.Atom / lightspeed.Molecule as used by the J/K callers:
Molecule.from_xyz_file / from_xyz_str (src/python/core.py:100-161),
xyz, xyzZ, Z and Molecule.concatenate. Coordinates in xyz files are Angstrom
and are scaled by 1/0.52917720859 (src/python/util.py:3, the PSI4 value).
"""
import os
import re
import numpy as np

units = {"ang_per_bohr": 0.52917720859}
units["bohr_per_ang"] = 1.0 / units["ang_per_bohr"]

_SYMBOLS = ["X", "H", "HE", "LI", "BE", "B", "C", "N", "O", "F", "NE", "NA", "MG", "AL", "SI", "P", "S",
            "CL", "AR", "K", "CA"]
ATOMIC_NUMBERS = {s: i for i, s in enumerate(_SYMBOLS)}

_atom_re = re.compile(r"^\s*([a-z]+)(\d*)\s+(\S+)\s+(\S+)\s+(\S+)\s*$", re.IGNORECASE)
_ghost_re = re.compile(r"^\s*(Gh)\(([a-z]+)(\d*)\)\s+(\S+)\s+(\S+)\s+(\S+)\s*$", re.IGNORECASE)


class Atom:
    def __init__(self, label, symbol, N, x, y, z, Z, atomIdx):
        self.label, self.symbol, self.N = label, symbol, N
        self.x, self.y, self.z, self.Z = float(x), float(y), float(z), float(Z)
        self.atomIdx = atomIdx

    @staticmethod
    def from_xyz_line(line, scale=units["bohr_per_ang"]):
        m = _atom_re.match(line)
        if m:
            sym = m.group(1).upper()
            if sym not in ATOMIC_NUMBERS:
                raise ValueError("XYZ Line has unrecognized atomic symbol:\n%s" % line)
            N = ATOMIC_NUMBERS[sym]
            return Atom(m.group(1) + m.group(2), sym, N, float(m.group(3)) * scale,
                        float(m.group(4)) * scale, float(m.group(5)) * scale, float(N), 0)
        m = _ghost_re.match(line)
        if m:
            sym = m.group(2).upper()
            if sym not in ATOMIC_NUMBERS:
                raise ValueError("XYZ Line has unrecognized atomic symbol:\n%s" % line)
            return Atom("Gh(%s%s)" % (m.group(2), m.group(3)), sym, ATOMIC_NUMBERS[sym],
                        float(m.group(4)) * scale, float(m.group(5)) * scale, float(m.group(6)) * scale, 0.0, 0)
        raise ValueError("XYZ Line is malformed:\n%s" % line)


class Molecule:
    def __init__(self, name, atoms, charge=0.0, multiplicity=1.0):
        self.name = name
        self.atoms = [Atom(a.label, a.symbol, a.N, a.x, a.y, a.z, a.Z, k) for k, a in enumerate(atoms)]
        self.charge = float(charge)
        self.multiplicity = float(multiplicity)

    @property
    def natom(self):
        return len(self.atoms)

    @property
    def xyz(self):
        return np.array([[a.x, a.y, a.z] for a in self.atoms]).reshape(-1, 3)

    @property
    def Z(self):
        return np.array([a.Z for a in self.atoms])

    @property
    def xyzZ(self):
        return np.array([[a.x, a.y, a.z, a.Z] for a in self.atoms]).reshape(-1, 4)

    @property
    def nuclear_charge(self):
        return float(np.sum(self.Z))

    def nuclear_repulsion_energy(self):
        X = self.xyz
        Z = self.Z
        E = 0.0
        for A in range(len(Z)):
            for B in range(A):
                E += Z[A] * Z[B] / np.linalg.norm(X[A] - X[B])
        return E

    @staticmethod
    def from_xyz_str(strval, scale=units["bohr_per_ang"], name="mol"):
        lines = [l for l in strval.split("\n") if len(l) and not l.isspace()]
        if not lines:
            raise ValueError("No lines in molecule: %s" % name)
        if re.match(r"^\s*(\d+)\s*$", lines[0]):
            lines = lines[1:]
        Q, M = 0.0, 1.0
        m = re.match(r"^\s*(-?\d+)\s+(\d+)\s*$", lines[0])
        if m:
            Q, M = float(m.group(1)), float(m.group(2))
            lines = lines[1:]
        elif not _atom_re.match(lines[0]) and not _ghost_re.match(lines[0]):
            lines = lines[1:]
        return Molecule(name, [Atom.from_xyz_line(l, scale) for l in lines], Q, M)

    @staticmethod
    def from_xyz_file(filename, scale=units["bohr_per_ang"], name=None):
        with open(filename) as fh:
            s = fh.read()
        if name is None:
            name = os.path.splitext(os.path.basename(filename))[0]
        return Molecule.from_xyz_str(s, scale=scale, name=name)

    @staticmethod
    def from_arrays(symbols, xyz_bohr, name="mol", charge=0.0, multiplicity=1.0):
        atoms = []
        for k, (s, r) in enumerate(zip(symbols, xyz_bohr)):
            s = s.upper()
            N = ATOMIC_NUMBERS[s]
            atoms.append(Atom(s, s, N, r[0], r[1], r[2], float(N), k))
        return Molecule(name, atoms, charge, multiplicity)

    @staticmethod
    def concatenate(mols, charge, multiplicity):
        atoms = [a for m in mols for a in m.atoms]
        return Molecule("+".join(m.name for m in mols), atoms, charge, multiplicity)
