"""Make tests/golden/c40h82_ccpvdz_kref.npz: the reference CPU IntBox's K (and J
energy) for C40H82 / cc-pVDZ (all-trans, oracle/workloads.alkane) at thre_pq =
thresp = 1e-14, FP64, at a converged RHF density.

The density comes in as an npz with key D (nao x nao), e.g. saved from the
engine's FP64 SCF; its occupied factor Cocc (D = Cocc Cocc^T, from the
eigenvectors of D with non-zero eigenvalues) is stored, and the reference J and
K are computed at Cocc Cocc^T. Stored: Cocc, four rows of K, the traces
E_J = sum D J and E_K = sum D K, and the seconds and threads the reference took.

    REFROOT=/path/to/lightspeed python tests/golden/make_c40_kref.py density.npz
(runs the reference CPU IntBox built by `make -C oracle ref`; ~17 minutes on 8 cores)."""
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import ref, workloads  # noqa: E402

ROWS = (0, 100, 500, 969)


def main(path):
    D0 = np.load(path)["D"]
    w, U = np.linalg.eigh(0.5 * (D0 + D0.T))
    keep = w > 1e-8
    C = U[:, keep] * np.sqrt(w[keep])
    D = C @ C.T
    syms, xyz = workloads.alkane(40)
    arr, prims, nao = workloads.basis(syms, xyz, "cc-pvdz")
    assert D.shape == (nao, nao)
    rb = ref.RefBasis(arr)
    rp = ref.RefPairs(rb, rb, True, 1e-14)
    nt = os.cpu_count() or 1
    t0 = time.time()
    J = ref.coulomb(rp, rp, D, 1e-14, 1e-14, nthread=nt)
    t1 = time.time()
    K = ref.exchange(rp, rp, D, True, 1e-14, 1e-14, nthread=nt)
    t2 = time.time()
    out = os.path.join(ROOT, "tests", "golden", "c40h82_ccpvdz_kref.npz")
    np.savez_compressed(out, Cocc=C, rows=np.array(ROWS), K_rows=K[list(ROWS)], E_J=np.sum(D * J),
                        E_K=np.sum(D * K), seconds_J=t1 - t0, seconds_K=t2 - t1, threads=nt)
    print(json.dumps({"out": out, "seconds_J": t1 - t0, "seconds_K": t2 - t1, "threads": nt,
                      "E_J": float(np.sum(D * J)), "E_K": float(np.sum(D * K))}))


if __name__ == "__main__":
    main(sys.argv[1])
