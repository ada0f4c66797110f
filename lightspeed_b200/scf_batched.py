"""Lockstep RHF for many molecules with every matrix on the GPU.

The same iteration as scf.SCFStepper (est/rhf.py:583-660: incremental Fock
builds from the difference density with a full rebuild every
`incremental_niter` iterations, DIIS on F D S - S D F, convergence confirmed
on a full build), carried out for all molecules of equal size at once with
batched FP64 tensor algebra (torch is the container and the batched
eigensolver here; J and K come from the engine's device entry points, which
read and write the same tensors in place). Molecules are grouped by basis
size; a molecule stops iterating when it has converged.
"""
import numpy as np


class BatchedRHF:
    def __init__(self, ls, systems, device, incremental_niter=8, ndiis=8):
        """systems: list of scf.RHF objects (their S, H, X, nocc, Enuc and pair lists are used)."""
        import torch
        self.torch = torch
        self.ls = ls
        self.dev = device
        self.systems = systems
        self.incremental_niter = incremental_niter
        self.ndiis = ndiis
        by_n = {}
        for k, r in enumerate(systems):
            by_n.setdefault((r.S.shape[0], r.X.shape[1], r.nocc), []).append(k)
        f64 = dict(dtype=torch.float64, device=device)
        self.groups = []
        for (n, m, nocc), idx in sorted(by_n.items()):
            grp = {
                "idx": idx, "n": n, "nocc": nocc,
                "S": torch.tensor(np.stack([systems[k].S for k in idx]), **f64),
                "H": torch.tensor(np.stack([systems[k].H for k in idx]), **f64),
                "X": torch.tensor(np.stack([systems[k].X for k in idx]), **f64),
                "Enuc": torch.tensor([systems[k].Enuc for k in idx], **f64),
            }
            B = len(idx)
            for key in ("D", "Dold", "dD", "J", "K", "dJ", "dK"):
                grp[key] = torch.zeros(B, n, n, **f64)
            grp["Fh"] = torch.zeros(ndiis, B, n, n, **f64)
            grp["Eh"] = torch.zeros(ndiis, B, m, m, **f64)
            grp["nh"] = 0
            grp["E"] = torch.zeros(B, **f64)
            grp["gnorm"] = torch.full((B,), float("inf"), **f64)
            grp["done"] = torch.zeros(B, dtype=torch.bool, device=device)
            grp["full_pending"] = torch.zeros(B, dtype=torch.bool, device=device)
            self.groups.append(grp)
        self.iteration = 0

    def set_guess(self, densities):
        """densities: list of numpy arrays (one per system, in the systems' order)."""
        torch = self.torch
        for grp in self.groups:
            grp["D"].copy_(torch.tensor(np.stack([densities[k] for k in grp["idx"]]), device=self.dev))

    def active(self):
        """(group index, slot) of every molecule still iterating."""
        out = []
        for gi, grp in enumerate(self.groups):
            for b in range(len(grp["idx"])):
                if not bool(grp["done"][b]):
                    out.append((gi, b))
        return out

    def prepare(self):
        """Difference densities for this iteration (full rebuild every
        incremental_niter iterations or when a molecule must confirm)."""
        full_all = self.iteration % self.incremental_niter == 0
        for grp in self.groups:
            full = grp["full_pending"] | full_all
            f = full.view(-1, 1, 1)
            grp["J"].masked_fill_(f, 0.0)
            grp["K"].masked_fill_(f, 0.0)
            grp["Dold"].masked_fill_(f, 0.0)
            grp["dD"].copy_(grp["D"] - grp["Dold"])
            grp["dJ"].zero_()
            grp["dK"].zero_()
            grp["was_full"] = full.clone()
            grp["full_pending"].zero_()

    def targets(self, gi, b):
        """Device pointers (dD, dJ, dK) of one molecule for the J/K builds."""
        grp = self.groups[gi]
        return grp["dD"][b].data_ptr(), grp["dJ"][b].data_ptr(), grp["dK"][b].data_ptr()

    def update(self, g_conv):
        """Consume the builds: energies, gradients, convergence, DIIS, new densities."""
        torch = self.torch
        self.iteration += 1
        for grp in self.groups:
            act = ~grp["done"]
            if not bool(act.any()):
                continue
            a = act.view(-1, 1, 1)
            grp["J"] += torch.where(a, grp["dJ"], torch.zeros_like(grp["dJ"]))
            grp["K"] += torch.where(a, grp["dK"], torch.zeros_like(grp["dK"]))
            grp["Dold"].copy_(torch.where(a, grp["D"], grp["Dold"]))
            H, S, X, D = grp["H"], grp["S"], grp["X"], grp["D"]
            F = H + 2.0 * grp["J"] - grp["K"]
            E = (D * (H + F)).sum(dim=(1, 2)) + grp["Enuc"]
            G = F @ D @ S - S @ D @ F
            Go = X.transpose(1, 2) @ G @ X
            gn = torch.sqrt((Go * Go).mean(dim=(1, 2)))
            grp["E"] = torch.where(act, E, grp["E"])
            grp["gnorm"] = torch.where(act, gn, grp["gnorm"])
            below = act & (gn < g_conv)
            grp["done"] |= below & grp["was_full"]
            grp["full_pending"] |= below & ~grp["was_full"]
            # DIIS over the last ndiis iterations (shared history slots; done molecules are frozen)
            k = grp["nh"] % self.ndiis
            grp["Fh"][k] = F
            grp["Eh"][k] = Go
            grp["nh"] += 1
            m = min(grp["nh"], self.ndiis)
            Fh, Eh = grp["Fh"][:m], grp["Eh"][:m]
            Bm = torch.einsum("ibxy,jbxy->bij", Eh, Eh)
            nb = Bm.shape[0]
            A = -torch.ones(nb, m + 1, m + 1, dtype=Bm.dtype, device=self.dev)
            A[:, :m, :m] = Bm
            A[:, m, m] = 0.0
            rhs = torch.zeros(nb, m + 1, dtype=Bm.dtype, device=self.dev)
            rhs[:, m] = -1.0
            c = torch.linalg.lstsq(A, rhs.unsqueeze(-1)).solution.squeeze(-1)[:, :m]
            Fd = torch.einsum("bi,ibxy->bxy", c, Fh)
            Fo = X.transpose(1, 2) @ Fd @ X
            _, Co = torch.linalg.eigh(Fo)
            C = X @ Co[:, :, :grp["nocc"]]
            Dn = C @ C.transpose(1, 2)
            # molecules that converged or confirm on a full build keep their density
            keep = (grp["done"] | grp["full_pending"] | ~act).view(-1, 1, 1)
            grp["D"] = torch.where(keep, D, Dn)

    def finished(self):
        return all(bool(grp["done"].all()) for grp in self.groups)

    def energies(self):
        out = np.zeros(len(self.systems))
        for grp in self.groups:
            e = grp["E"].cpu().numpy()
            for b, k in enumerate(grp["idx"]):
                out[k] = e[b]
        return out

    def converged(self):
        out = np.zeros(len(self.systems), dtype=bool)
        for grp in self.groups:
            d = grp["done"].cpu().numpy()
            for b, k in enumerate(grp["idx"]):
                out[k] = d[b]
        return out
