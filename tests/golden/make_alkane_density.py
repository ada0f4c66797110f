"""Make tests/golden/c8h18_ccpvdz_cocc.npz: the occupied RHF orbitals of
all-trans C8H18 in cc-pVDZ, converged with the reference CPU IntBox alone
(oracle/_ref: S, T, V, J and K of the reference), so the reference arm of
bench.py can time the reference's J/K at a converged density without running
any code of the product. Thresholds as in the alkane workload (Schwarz and
thresp 1e-14); core-Hamiltonian start, DIIS on F D S - S D F, full J/K every
iteration, converged to an rms orbital gradient of 1e-7 (orthogonal basis).

  python tests/golden/make_alkane_density.py [n_carbon]   (default 8; needs oracle/_ref)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref, workloads  # noqa: E402

THRE = 1.0e-14


def main(ncarbon=8):
    symbols, xyz = workloads.alkane(ncarbon)
    arrays, _, nao = workloads.basis(symbols, xyz, "cc-pvdz")
    rb = ref.RefBasis(arrays)
    rp = ref.RefPairs(rb, rb, True, THRE)
    xyzZ = np.hstack([xyz, np.array([[workloads.Z[s]] for s in symbols], float)])
    S = ref.overlap(rp)
    H = ref.kinetic(rp) + ref.potential(rp, xyzZ)
    s, U = np.linalg.eigh(S)
    X = U[:, s > 1e-7] / np.sqrt(s[s > 1e-7])
    nocc = workloads.nuclear_charge(symbols) // 2
    Enuc = workloads.nuclear_repulsion(symbols, xyz)

    def orbitals(F):
        e, C = np.linalg.eigh(X.T @ F @ X)
        return X @ C[:, :nocc]

    Cocc = orbitals(H)
    Fs, Es = [], []
    E = 0.0
    for it in range(100):
        D = Cocc @ Cocc.T
        J = ref.coulomb(rp, rp, D, THRE, THRE)
        K = ref.exchange(rp, rp, D, True, THRE, THRE)
        F = H + 2.0 * J - K
        E = float(np.sum(D * (H + F))) + Enuc
        G = X.T @ (F @ D @ S - S @ D @ F) @ X
        g = float(np.sqrt(np.mean(G * G)))
        print("%3d %20.12f %10.3e" % (it, E, g), flush=True)
        if g < 1e-7:
            break
        Fs.append(F)
        Es.append(G)
        Fs, Es = Fs[-8:], Es[-8:]
        n = len(Fs)
        B = -np.ones((n + 1, n + 1))
        B[n, n] = 0.0
        for a in range(n):
            for b in range(n):
                B[a, b] = np.sum(Es[a] * Es[b])
        rhs = np.zeros(n + 1)
        rhs[n] = -1.0
        c = np.linalg.solve(B, rhs)[:n]
        Cocc = orbitals(sum(ci * Fi for ci, Fi in zip(c, Fs)))
    out = os.path.join(HERE, "c%dh%d_ccpvdz_cocc.npz" % (ncarbon, 2 * ncarbon + 2))
    np.savez_compressed(out, Cocc=Cocc, E=E, gnorm=g)
    print("wrote", out, "E =", E)


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else 8)
