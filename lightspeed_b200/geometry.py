"""Seeded synthetic molecules for the J/K workloads (all coordinates in Bohr).

* water_cluster(n, seed): n rigid waters (O-H 0.96 A, H-O-H 104.5 deg) with
  uniformly random orientations (random unit quaternions) and O positions
  uniform in a cube of side (n * 30 A^3)^(1/3) (liquid-water density),
  redrawn until every O-O distance is >= 2.8 A.
* alkane(n_carbon): all-trans linear alkane CnH(2n+2) with C-C 1.54 A,
  C-H 1.09 A and tetrahedral angles.
* distorted(mol, seed, dr, dtheta): bond-length and angle noise for waters.
"""
import math
import numpy as np

from .molecule import Molecule, units

ANG = units["bohr_per_ang"]
ROH = 0.96
HOH = math.radians(104.5)
TET = math.acos(-1.0 / 3.0)


def _random_rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def _water_frame(roh1=ROH, roh2=ROH, theta=HOH):
    return np.array([
        [0.0, 0.0, 0.0],
        [roh1 * math.sin(theta / 2), 0.0, roh1 * math.cos(theta / 2)],
        [-roh2 * math.sin(theta / 2), 0.0, roh2 * math.cos(theta / 2)],
    ])


def water_cluster(n, seed=0, side=None, min_oo=2.8, noise=None):
    """Seeded cluster of n waters; returns a Molecule (Bohr). `noise` =
    (dr_ang, dtheta_deg) applies uniform bond/angle noise per water."""
    rng = np.random.default_rng(seed)
    if side is None:
        side = (n * 30.0) ** (1.0 / 3.0)
    centers = []
    tries = 0
    while len(centers) < n:
        tries += 1
        if tries > 100000 * n:
            raise RuntimeError("water_cluster: could not place %d waters in a %.2f A box" % (n, side))
        c = rng.uniform(0.0, side, size=3)
        if all(np.linalg.norm(c - o) >= min_oo for o in centers):
            centers.append(c)
    symbols, xyz = [], []
    for c in centers:
        if noise:
            dr, dth = noise
            frame = _water_frame(ROH + rng.uniform(-dr, dr), ROH + rng.uniform(-dr, dr),
                                 HOH + math.radians(rng.uniform(-dth, dth)))
        else:
            frame = _water_frame()
        R = _random_rotation(rng)
        for s, r in zip("OHH", frame):
            symbols.append(s)
            xyz.append((R @ r + c) * ANG)
    return Molecule.from_arrays(symbols, np.array(xyz), name="w%d_s%d" % (n, seed))


def alkane(n_carbon=40):
    """All-trans CnH(2n+2) in the xz plane zig-zag, Bohr."""
    cc, ch = 1.54, 1.09
    half = TET / 2.0
    dx = cc * math.sin(half)
    dz = cc * math.cos(half)
    C = [np.array([k * dx, 0.0, (k % 2) * dz]) for k in range(n_carbon)]
    symbols, xyz = [], []
    for k, c in enumerate(C):
        symbols.append("C")
        xyz.append(c)
    # two H per carbon in the plane perpendicular to the local C-C-C bisector
    for k, c in enumerate(C):
        up = 1.0 if k % 2 else -1.0       # pointing away from the backbone
        b = np.array([0.0, 0.0, up])      # bisector direction (outward)
        # tetrahedral: H-C-H angle 109.47, both in the plane spanned by b and y
        for sgn in (1.0, -1.0):
            d = math.cos(half) * b + math.sin(half) * np.array([0.0, sgn, 0.0])
            symbols.append("H")
            xyz.append(c + ch * d)
    # terminal hydrogens along the chain axis
    for k, sgn in ((0, -1.0), (n_carbon - 1, 1.0)):
        c = C[k]
        up = 1.0 if k % 2 else -1.0
        d = np.array([sgn * math.sin(half), 0.0, -up * math.cos(half)])
        symbols.append("H")
        xyz.append(c + ch * d / np.linalg.norm(d))
    return Molecule.from_arrays(symbols, np.array(xyz) * ANG, name="C%dH%d" % (n_carbon, 2 * n_carbon + 2))
