"""Restricted Hartree-Fock around the GPU J/K path.

The SCF linear algebra stays on the host in FP64 (as in the reference's
est/rhf.py); every J and K goes through ls.IntBox.coulomb / exchange. The
iteration follows est/rhf.py:583-660: incremental Fock builds with the
difference density dD = D - D_old, a full rebuild every `incremental_niter`
iterations, DIIS on the orbital gradient F D S - S D F.
"""
import time

import numpy as np


class RHF:
    def __init__(self, ls, molecule, basis, thre_pq=1.0e-14, thre_sp=1.0e-14, thre_dp=1.0e-6,
                 incremental_niter=8, ewald=None, resources=None):
        self.ls = ls
        self.mol = molecule
        self.basis = basis
        self.res = resources or ls.ResourceList.build()
        self.ewald = ewald or ls.Ewald.coulomb()
        self.thre_sp = thre_sp
        self.thre_dp = thre_dp
        self.incremental_niter = incremental_niter
        self.pairs = ls.PairList.build_schwarz(basis, basis, True, thre_pq)
        nel = int(round(molecule.nuclear_charge - molecule.charge))
        if nel % 2:
            raise ValueError("RHF needs an even electron count")
        self.nocc = nel // 2
        xyzc = ls.Tensor.array(molecule.xyzZ)
        self.S = ls.IntBox.overlap(self.res, self.pairs).np.copy()
        self.T = ls.IntBox.kinetic(self.res, self.pairs).np.copy()
        self.V = ls.IntBox.potential(self.res, ls.Ewald.coulomb(), self.pairs, xyzc).np.copy()
        self.H = self.T + self.V
        self.Enuc = molecule.nuclear_repulsion_energy()
        s, U = np.linalg.eigh(self.S)
        keep = s > 1.0e-7
        self.X = U[:, keep] / np.sqrt(s[keep])        # canonical orthogonalisation
        self.trace = []

    # -- Fock pieces -------------------------------------------------------------
    def jk(self, D):
        ls = self.ls
        Dt = ls.Tensor.array(D)
        J = ls.IntBox.coulomb(self.res, self.ewald, self.pairs, self.pairs, Dt, self.thre_sp, self.thre_dp)
        K = ls.IntBox.exchange(self.res, self.ewald, self.pairs, self.pairs, Dt, True, self.thre_sp, self.thre_dp)
        return J.np.copy(), K.np.copy()

    def density(self, F):
        Fo = self.X.T @ F @ self.X
        eps, Co = np.linalg.eigh(Fo)
        C = self.X @ Co
        Cocc = C[:, :self.nocc]
        return Cocc @ Cocc.T, eps, C

    def energy(self, D, J, K):
        F = self.H + 2.0 * J - K
        return float(np.sum(D * (self.H + F))) + self.Enuc, F

    def core_guess(self):
        return self.density(self.H)[0]

    # -- iterations --------------------------------------------------------------
    def compute(self, D0=None, maxiter=60, g_conv=1.0e-8, e_conv=1.0e-10, ndiis=8, verbose=False):
        D = self.core_guess() if D0 is None else np.array(D0, copy=True)
        Dold = np.zeros_like(D)
        J = np.zeros_like(D)
        K = np.zeros_like(D)
        diis_F, diis_E = [], []
        E_old = 0.0
        self.trace = []
        t_start = time.time()
        for it in range(maxiter):
            if it % self.incremental_niter == 0:
                J[...] = 0.0
                K[...] = 0.0
                Dold[...] = 0.0
            t0 = time.time()
            dJ, dK = self.jk(D - Dold)
            t_jk = time.time() - t0
            J += dJ
            K += dK
            Dold = D.copy()
            E, F = self.energy(D, J, K)
            G = F @ D @ self.S - self.S @ D @ F
            Go = self.X.T @ G @ self.X
            gnorm = float(np.sqrt(np.mean(Go * Go)))
            dE = E - E_old
            E_old = E
            self.trace.append(dict(iter=it, E=E, dE=dE, gnorm=gnorm, t_jk=t_jk))
            if verbose:
                print("  %3d %24.16f %11.3e %11.3e %8.3f s" % (it, E, dE, gnorm, t_jk), flush=True)
            if gnorm < g_conv and abs(dE) < max(e_conv, 1e-14):
                break
            diis_F.append(F.copy())
            diis_E.append(Go.copy())
            if len(diis_F) > ndiis:
                diis_F.pop(0)
                diis_E.pop(0)
            n = len(diis_F)
            B = -np.ones((n + 1, n + 1))
            B[n, n] = 0.0
            for a in range(n):
                for b in range(n):
                    B[a, b] = np.sum(diis_E[a] * diis_E[b])
            rhs = np.zeros(n + 1)
            rhs[n] = -1.0
            try:
                c = np.linalg.solve(B, rhs)[:n]
            except np.linalg.LinAlgError:
                c = np.zeros(n)
                c[-1] = 1.0
            Fd = sum(ci * Fi for ci, Fi in zip(c, diis_F))
            D = self.density(Fd)[0]
        self.E = E
        self.D = D
        self.J, self.K = J, K
        self.wall = time.time() - t_start
        self.converged = gnorm < g_conv
        return E


def loewdin_density(S, nocc, seed):
    """D = C C^T for nocc seeded Gaussian columns Loewdin-orthonormalised in
    the metric S (the first density of the 8-water workload)."""
    rng = np.random.default_rng(seed)
    C = rng.normal(size=(S.shape[0], nocc))
    w, V = np.linalg.eigh(C.T @ S @ C)
    C = C @ (V @ np.diag(w ** -0.5) @ V.T)
    return C @ C.T
