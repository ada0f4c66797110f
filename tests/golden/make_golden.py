"""Make the golden fixtures in tests/golden/ (run in a container that has the
reference tree and oracle/_ref built; the fixtures are committed).

1. ref_<case>.npz: the reference's own known-answer vectors for the J/K path,
   copied from its test data (tests/coverage/data/{prop,ewald,mix}_*.npz,
   checked by tests/coverage/prop_int.py:68-108, ewald_int.py:33-108 and
   mix_basis.py:101-225 in the reference) -- only the density/J/K keys and
   the J/K nuclear gradients (Jgr..Jgr4, Kgr..Kgr4 of prop_int.py:142-214).
2. oracle_w8.npz: J and K of the reference CPU IntBox (oracle/_ref) for an
   8-water 6-31G* cluster (seed 0) at thresp = 1e-12 with the density
   D = C C^T of 40 seeded Gaussian columns Loewdin-orthonormalised in the
   reference overlap metric; plus the pair list of that basis.

  python tests/golden/make_golden.py [REFERENCE_ROOT]   (default: $REFROOT, else /root/reference)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def copy_reference_vectors(ref_root):
    data = os.path.join(ref_root, "tests", "coverage", "data")
    for basis in ("sto-3g", "6-31gs", "cc-pvdz"):
        z = np.load(os.path.join(data, "prop_h2o_%s.npz" % basis))
        np.savez_compressed(os.path.join(HERE, "ref_prop_h2o_%s.npz" % basis),
                            **{k: z[k] for k in ("D", "D2", "J", "J2", "K", "K2", "Jgr", "Jgr2", "Jgr3", "Jgr4",
                                                  "Kgr", "Kgr2", "Kgr3", "Kgr4")})
        z = np.load(os.path.join(data, "ewald_h2o_%s.npz" % basis))
        keep = [k for k in z.files if k.split("_")[0] in ("D", "D2", "J", "J2", "K", "K2")]
        np.savez_compressed(os.path.join(HERE, "ref_ewald_h2o_%s.npz" % basis), **{k: z[k] for k in keep})
    z = np.load(os.path.join(data, "mix_h2o_nh3.npz"))
    keep = [k for k in z.files if k[0] in "DJK"]
    np.savez_compressed(os.path.join(HERE, "ref_mix_h2o_nh3.npz"), **{k: z[k] for k in keep})
    for xyz in ("h2o", "nh3"):
        with open(os.path.join(data, xyz + ".xyz")) as fh, open(os.path.join(HERE, xyz + ".xyz"), "w") as out:
            out.write(fh.read())


def loewdin_density(S, nocc, seed):
    rng = np.random.default_rng(seed)
    C = rng.normal(size=(S.shape[0], nocc))
    M = C.T @ S @ C
    w, V = np.linalg.eigh(M)
    C = C @ (V @ np.diag(w ** -0.5) @ V.T)
    return C @ C.T


def oracle_water8():
    import lightspeed_b200 as ls
    from lightspeed_b200.geometry import water_cluster
    from oracle import ref
    mol = water_cluster(8, seed=0)
    bas = ls.Basis.from_gbs_file(mol, "6-31gs")
    rb = ref.RefBasis(ref.prim_arrays(bas))
    pl = ref.RefPairs(rb, rb, True, 1.0e-12)
    S = ref.overlap(pl)
    D = loewdin_density(S, 40, seed=1)
    J = ref.coulomb(pl, pl, D, 1.0e-12, 1.0e-12)
    K = ref.exchange(pl, pl, D, True, 1.0e-12, 1.0e-12)
    L1, L2, p1, p2, b = pl.export()
    np.savez_compressed(os.path.join(HERE, "oracle_w8.npz"), D=D, J=J, K=K, S=S, L1=L1, L2=L2, p1=p1, p2=p2,
                        bound=b, xyz=mol.xyz)


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REFROOT", "/root/reference")
    copy_reference_vectors(ref_root)
    oracle_water8()
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
