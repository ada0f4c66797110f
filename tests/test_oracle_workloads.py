"""The benchmark inputs restated on the oracle side (oracle/workloads.py) equal
the product's (lightspeed_b200.geometry.alkane, Basis.from_gbs_file) bit for
bit, and the reference arm of bench.py builds its sample without loading the
product package."""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("ncarbon", [1, 3, 8, 40])
def test_alkane_and_basis_match_product(ls, ncarbon):
    from lightspeed_b200.geometry import alkane
    from oracle import workloads
    symbols, xyz = workloads.alkane(ncarbon)
    mol = alkane(ncarbon)
    assert [a.symbol for a in mol.atoms] == symbols
    assert np.array_equal(xyz, mol.xyz)
    assert workloads.nuclear_charge(symbols) == int(round(mol.nuclear_charge))
    assert abs(workloads.nuclear_repulsion(symbols, xyz) - mol.nuclear_repulsion_energy()) < 1e-9
    for name in ("cc-pvdz", "6-31gs"):
        arrays, prims, nao = workloads.basis(symbols, xyz, name)
        bas = ls.Basis.from_gbs_file(mol, name)
        assert nao == bas.nao and len(prims) == bas.nprim
        P = bas.primitives
        assert np.array_equal(arrays["c"], np.array([p.c for p in P]))
        assert np.array_equal(arrays["e"], np.array([p.e for p in P]))
        assert np.array_equal(arrays["xyz"], np.array([[p.x, p.y, p.z] for p in P]).reshape(-1, 3))
        for key, attr in (("L", "L"), ("ao", "aoIdx"), ("cart", "cartIdx"), ("shell", "shellIdx"),
                          ("atom", "atomIdx")):
            assert np.array_equal(arrays[key], np.array([getattr(p, attr) for p in P]))


def test_reference_sample_loads_no_product_code():
    from oracle import port, ref
    fixture = os.path.join(ROOT, "tests", "golden", "c8h18_ccpvdz_cocc.npz")
    if not (ref.available() and port.available() and os.path.exists(fixture)):
        pytest.skip("oracle/_ref or the density fixture is missing")
    code = ("import sys; sys.path.insert(0, %r); import bench; rp, D, nq, desc = bench.cpu_sample(); "
            "mods = [m for m in sys.modules if m.startswith('lightspeed_b200')]; "
            "print(len(mods), nq > 0, abs(D - D.T).max() < 1e-12)" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    assert out.stdout.split() == ["0", "True", "True"]
