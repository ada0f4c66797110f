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
    def compute(self, D0=None, maxiter=60, g_conv=1.0e-8, e_conv=None, ndiis=8, verbose=False):
        """Converge until the orbital gradient (rms, orthogonal basis) is below
        g_conv on a Fock matrix from a full (not incremental) J/K build: when an
        incremental build reaches g_conv, the same density is rebuilt in full
        and tested again, so the final energy carries no accumulated
        difference-density screening error. e_conv, if given, also bounds the
        last energy change."""
        st = SCFStepper(self, D0, g_conv=g_conv, e_conv=e_conv, ndiis=ndiis)
        t_start = time.time()
        for it in range(maxiter):
            dD = st.build_density()
            t0 = time.time()
            dJ, dK = self.jk(dD)
            st.t_jk = time.time() - t0
            done = st.update(dJ, dK)
            if verbose:
                tr = self.trace[-1]
                print("  %3d %24.16f %11.3e %11.3e %8.3f s%s" % (it, tr["E"], tr["dE"], tr["gnorm"], st.t_jk,
                                                                  "" if tr["full"] else " (incr)"), flush=True)
            if done:
                break
        st.finish()
        self.wall = time.time() - t_start
        return self.E


class SCFStepper:
    """One RHF's iterations as explicit steps, so a driver can build the J/K
    of many molecules together: build_density() gives the (difference)
    density to build, update(dJ, dK) consumes the result and returns True once
    converged. The iteration follows est/rhf.py:583-660: incremental Fock
    builds with dD = D - D_old and a full rebuild every `incremental_niter`
    iterations, DIIS on F D S - S D F, convergence confirmed on a full build."""

    def __init__(self, rhf, D0=None, g_conv=1.0e-8, e_conv=None, ndiis=8):
        self.r = rhf
        self.D = rhf.core_guess() if D0 is None else np.array(D0, copy=True)
        self.Dold = np.zeros_like(self.D)
        self.J = np.zeros_like(self.D)
        self.K = np.zeros_like(self.D)
        self.diis_F, self.diis_E = [], []
        self.E_old = 0.0
        self.g_conv, self.e_conv, self.ndiis = g_conv, e_conv, ndiis
        self.force_full = False
        self.n_full = 0
        self.full = True
        self.gnorm = np.inf
        self.E = None
        self.t_jk = 0.0
        self.converged = False
        rhf.trace = []

    def build_density(self):
        self.full = self.force_full or self.n_full % self.r.incremental_niter == 0
        self.force_full = False
        if self.full:
            self.n_full = 0
            self.J[...] = 0.0
            self.K[...] = 0.0
            self.Dold[...] = 0.0
        self.n_full += 1
        return self.D - self.Dold

    def update(self, dJ, dK):
        r = self.r
        self.J += dJ
        self.K += dK
        self.Dold = self.D.copy()
        E, F = r.energy(self.D, self.J, self.K)
        G = F @ self.D @ r.S - r.S @ self.D @ F
        Go = r.X.T @ G @ r.X
        self.gnorm = float(np.sqrt(np.mean(Go * Go)))
        dE = E - self.E_old
        self.E_old = E
        self.E = E
        r.trace.append(dict(iter=len(r.trace), E=E, dE=dE, gnorm=self.gnorm, t_jk=self.t_jk, full=self.full))
        if self.gnorm < self.g_conv and (self.e_conv is None or abs(dE) < self.e_conv):
            if self.full:
                self.converged = True
                return True
            self.force_full = True     # confirm on a full build of the same density
            return False
        self.diis_F.append(F.copy())
        self.diis_E.append(Go.copy())
        if len(self.diis_F) > self.ndiis:
            self.diis_F.pop(0)
            self.diis_E.pop(0)
        n = len(self.diis_F)
        B = -np.ones((n + 1, n + 1))
        B[n, n] = 0.0
        for a in range(n):
            for b in range(n):
                B[a, b] = np.sum(self.diis_E[a] * self.diis_E[b])
        rhs = np.zeros(n + 1)
        rhs[n] = -1.0
        try:
            c = np.linalg.solve(B, rhs)[:n]
        except np.linalg.LinAlgError:
            c = np.zeros(n)
            c[-1] = 1.0
        Fd = sum(ci * Fi for ci, Fi in zip(c, self.diis_F))
        self.D = r.density(Fd)[0]
        return False

    def finish(self):
        r = self.r
        r.E = self.E
        r.D = self.D
        r.J, r.K = self.J, self.K
        r.converged = self.converged


def loewdin_density(S, nocc, seed):
    """D = C C^T for nocc seeded Gaussian columns Loewdin-orthonormalised in
    the metric S (the first density of the 8-water workload)."""
    rng = np.random.default_rng(seed)
    C = rng.normal(size=(S.shape[0], nocc))
    w, V = np.linalg.eigh(C.T @ S @ C)
    C = C @ (V @ np.diag(w ** -0.5) @ V.T)
    return C @ C.T
