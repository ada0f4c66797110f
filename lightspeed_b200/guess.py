"""Learned SCF starting guess for water clusters (BF16 multilayer perceptron).

No counterpart in the reference, whose SCF starts from SAD (est/rhf.py:401-421).
A three-layer, 256-wide MLP maps a description of an atom pair (I, J) to that
pair's block of the converged RHF density. To make one network serve every
orientation, blocks are predicted in local frames: each atom carries the
frame of its water (origin O, e1 along the HOH bisector, e3 normal to the
molecular plane, e2 = e3 x e1), and the global block is

    D_IJ = A_I^T D'_IJ A_J,

where A_I maps atom I's Cartesian Gaussian components from global to local
axes (the action of the frame rotation on monomials x^a y^b z^c; components
of a shell share one normalisation, so monomials transform like the basis
functions). The inputs are rotation invariant: the pair type, 16 Gaussian
radial shells of the distance, J's position in I's frame and I's in J's,
the relative orientation F_I F_J^T, and per atom 16-shell radial symmetry
functions (Behler type, cutoff 6 Angstrom) for H and O neighbours plus the
positions, in the atom's frame, of its three nearest O and three nearest H
atoms of other waters.

The network's weights, activations and gradients are bfloat16 and every
product accumulates in FP32 (kernels: lsmlp_* in liblsjk.so); master weights
are FP32 (Adam). The guess is used only through `LearnedGuess.guess`, which
assembles the blocks, projects onto the nearest idempotent density with the
right electron count (natural orbitals in the S metric) and falls back to
the SAD guess when the projected guess misses the electron count or
idempotency by more than 1e-3, or is not finite. The SCF then converges as
always, so the final energy does not depend on the guess.
"""
import ctypes

import numpy as np

ANG_PER_BOHR = 0.52917720859
N_RADIAL = 16
R_CUT = 6.0                     # Angstrom
MU = np.linspace(0.5, R_CUT, N_RADIAL)
ETA = 1.0 / (2.0 * (MU[1] - MU[0]) ** 2)
PAIR_TYPES = ("O*", "H*", "OO", "OH", "HH")   # self blocks, then I < J pairs (O before H)
N_NEIGH = 3                     # nearest O and nearest H of other waters, per atom
N_ENV = 2 * N_NEIGH * 3         # their positions in the atom's frame
N_FEAT = len(PAIR_TYPES) + N_RADIAL + 3 + 3 + 9 + 2 * (2 * N_RADIAL + N_ENV)
WIDTH = 256
N_OUT = 15 * 15


# ---- geometry -----------------------------------------------------------------

def _cutoff(r):
    return np.where(r < R_CUT, 0.5 * (np.cos(np.pi * r / R_CUT) + 1.0), 0.0)


def atom_descriptors(xyz_ang, symbols):
    """(natom, 32): radial symmetry functions of H and O neighbours."""
    n = len(symbols)
    d = np.linalg.norm(xyz_ang[:, None, :] - xyz_ang[None, :, :], axis=2)
    G = np.zeros((n, 2 * N_RADIAL))
    isO = np.array([s.upper() == "O" for s in symbols])
    w = np.exp(-ETA * (d[:, :, None] - MU[None, None, :]) ** 2) * _cutoff(d)[:, :, None]
    w[np.arange(n), np.arange(n), :] = 0.0
    G[:, :N_RADIAL] = w[:, ~isO, :].sum(axis=1)
    G[:, N_RADIAL:] = w[:, isO, :].sum(axis=1)
    return G


def water_frames(xyz, symbols):
    """(natom, 3, 3) rows = local axes of each atom's water (atoms in O, H, H order)."""
    n = len(symbols)
    if n % 3 or any(symbols[k].upper() != "OHH"[k % 3] for k in range(n)):
        raise ValueError("learned guess: atoms must come as O, H, H per water")
    F = np.zeros((n, 3, 3))
    for w in range(n // 3):
        O, H1, H2 = xyz[3 * w], xyz[3 * w + 1], xyz[3 * w + 2]
        e1 = (H1 - O) + (H2 - O)
        e1 /= np.linalg.norm(e1)
        e3 = np.cross(H1 - O, H2 - O)
        e3 /= np.linalg.norm(e3)
        e2 = np.cross(e3, e1)
        F[3 * w:3 * w + 3] = np.stack([e1, e2, e3])
    return F


def _cart_components(L):
    """(lx, ly, lz) of a Cartesian shell in CCA order (xx, xy, xz, yy, yz, zz for d)."""
    return [(lx, ly, L - lx - ly) for lx in range(L, -1, -1) for ly in range(L - lx, -1, -1)]


def monomial_map(F, L):
    """A with m(F r) = A m(r) for the Cartesian monomials m of degree L (CCA order)."""
    comps = _cart_components(L)
    rng = np.random.default_rng(1234)
    pts = rng.standard_normal((4 * len(comps) + 4, 3))
    def mono(P):
        return np.stack([P[:, 0] ** a * P[:, 1] ** b * P[:, 2] ** c for a, b, c in comps], axis=1)
    M = mono(pts)
    Mr = mono(pts @ F.T)
    A_T, *_ = np.linalg.lstsq(M, Mr, rcond=None)
    return A_T.T


def atom_shells(basis):
    """Per atom: list of (L, first AO) of its shells, in AO order."""
    shells = {}
    seen = set()
    for p in basis.primitives:
        if p.is_pure and p.L > 1:
            raise ValueError("learned guess: Cartesian basis sets only")
        key = (p.atomIdx, p.shellIdx)
        if key in seen:
            continue
        seen.add(key)
        shells.setdefault(p.atomIdx, []).append((p.L, p.aoIdx))
    return [sorted(shells[a], key=lambda s: s[1]) for a in sorted(shells)]


def atom_maps(basis, F):
    """Per atom: (first AO, size, A) with A the block-diagonal monomial map of its shells."""
    out = []
    for a, shells in enumerate(atom_shells(basis)):
        lo = shells[0][1]
        size = sum((L + 1) * (L + 2) // 2 for L, _ in shells)
        A = np.zeros((size, size))
        off = 0
        for L, _ in shells:
            n = (L + 1) * (L + 2) // 2
            A[off:off + n, off:off + n] = monomial_map(F[a], L)
            off += n
        out.append((lo, size, A))
    return out


def pair_list(xyz_ang, symbols):
    """Atom pairs (I, J) predicted: self pairs, and I != J within the cutoff with
    O before H (for O-H) or I < J; returns (I, J, type index)."""
    n = len(symbols)
    isO = [s.upper() == "O" for s in symbols]
    d = np.linalg.norm(xyz_ang[:, None, :] - xyz_ang[None, :, :], axis=2)
    pairs = []
    for i in range(n):
        pairs.append((i, i, 0 if isO[i] else 1))
        for j in range(n):
            if j == i or d[i, j] >= R_CUT:
                continue
            if isO[i] and not isO[j]:
                pairs.append((i, j, 3))
            elif isO[i] == isO[j] and i < j:
                pairs.append((i, j, 2 if isO[i] else 4))
    return pairs


def atom_environments(xyz_ang, symbols, F):
    """(natom, N_ENV): for each atom, the N_NEIGH nearest O and H atoms of other
    waters, as positions in the atom's frame scaled by the cutoff function
    (zero padded), nearest first."""
    n = len(symbols)
    isO = np.array([s.upper() == "O" for s in symbols])
    water = np.arange(n) // 3
    E = np.zeros((n, N_ENV))
    for i in range(n):
        v = xyz_ang - xyz_ang[i]
        d = np.linalg.norm(v, axis=1)
        other = (water != water[i]) & (d < R_CUT)
        for s_idx, sel in enumerate((isO, ~isO)):
            cand = np.nonzero(other & sel)[0]
            cand = cand[np.argsort(d[cand])][:N_NEIGH]
            for k, j in enumerate(cand):
                off = (s_idx * N_NEIGH + k) * 3
                E[i, off:off + 3] = (F[i] @ v[j]) * _cutoff(d[j])
    return E


def pair_features(xyz_bohr, symbols, pairs, F, G, Env):
    xyz = xyz_bohr * ANG_PER_BOHR
    P = np.array(pairs, dtype=np.int64).reshape(-1, 3)
    I, J, T = P[:, 0], P[:, 1], P[:, 2]
    v = xyz[J] - xyz[I]
    r = np.linalg.norm(v, axis=1)
    X = np.concatenate([
        np.eye(len(PAIR_TYPES))[T],
        np.exp(-ETA * (r[:, None] - MU[None, :]) ** 2),
        np.einsum("pab,pb->pa", F[I], v),
        np.einsum("pab,pb->pa", F[J], -v),
        np.einsum("pab,pcb->pac", F[I], F[J]).reshape(-1, 9),
        G[I], Env[I], G[J], Env[J]], axis=1)
    return X.astype(np.float32)


def local_targets(D, pairs, maps):
    """(npair, 225) local-frame blocks D'_IJ = A_I^-T D_IJ A_J^-1 (zero padded) and mask."""
    Y = np.zeros((len(pairs), N_OUT), np.float32)
    W = np.zeros((len(pairs), N_OUT), np.float32)
    inv = [np.linalg.inv(A) for _, _, A in maps]
    for k, (i, j, _) in enumerate(pairs):
        li, ni, _ = maps[i]
        lj, nj, _ = maps[j]
        blk = inv[i].T @ D[li:li + ni, lj:lj + nj] @ inv[j]
        Y[k, :ni * nj] = blk.ravel()
        W[k, :ni * nj] = 1.0
    return Y, W


def assemble(nao, pairs, maps, Yp):
    """Global density from predicted local blocks (zero beyond the cutoff)."""
    D = np.zeros((nao, nao))
    for k, (i, j, _) in enumerate(pairs):
        li, ni, Ai = maps[i]
        lj, nj, Aj = maps[j]
        blk = Ai.T @ Yp[k, :ni * nj].reshape(ni, nj).astype(np.float64) @ Aj
        D[li:li + ni, lj:lj + nj] = blk
        if i != j:
            D[lj:lj + nj, li:li + ni] = blk.T
    return D


def project_idempotent(D, S, nocc):
    """Nearest density with nocc doubly occupied natural orbitals in the S metric."""
    w, U = np.linalg.eigh(S)
    Sh = (U * np.sqrt(w)) @ U.T
    Smh = (U / np.sqrt(w)) @ U.T
    Dt = Sh @ (0.5 * (D + D.T)) @ Sh
    e, V = np.linalg.eigh(Dt)
    C = Smh @ V[:, -nocc:]
    return C @ C.T


def guess_errors(D, S, nocc):
    """(|tr(DS) - nocc| / nocc, ||DSD - D||_F / ||D||_F)."""
    DS = D @ S
    tr = abs(np.trace(DS) - nocc) / nocc
    idem = np.linalg.norm(DS @ D - D) / max(np.linalg.norm(D), 1e-300)
    return tr, idem


# ---- network (device, BF16 kernels) --------------------------------------------

class _Lib:
    def __init__(self, ls):
        lib = ctypes.CDLL(ls.LIB_PATH)
        lib.lsmlp_last_error.restype = ctypes.c_char_p
        P, I, L, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_long, ctypes.c_float
        lib.lsmlp_gemm_bf16.argtypes = [P, P, P, I, I, I, I, I, I, I, I, I, P]
        lib.lsmlp_bias_act.argtypes = [P, P, P, I, I, I, P]
        lib.lsmlp_act_grad.argtypes = [P, P, P, L, I, P]
        lib.lsmlp_mse.argtypes = [P, P, P, P, L, F, P, P]
        lib.lsmlp_colsum.argtypes = [P, P, I, I, P]
        lib.lsmlp_adam.argtypes = [P, P, P, P, P, L, F, F, F, F, I, F, P]
        lib.lsmlp_to_bf16.argtypes = [P, P, L, P]
        self.lib = lib

    def __call__(self, name, *args):
        rc = getattr(self.lib, name)(*args)
        if rc:
            raise RuntimeError("%s: %s" % (name, self.lib.lsmlp_last_error().decode()))


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


class MLP:
    """3 x 256 SiLU MLP: N_FEAT -> 256 -> 256 -> N_OUT (BF16 compute, FP32 masters)."""

    def __init__(self, ls, seed=0, device="cuda"):
        import torch
        self.torch = torch
        self.k = _Lib(ls)
        self.dev = torch.device(device)
        g = torch.Generator().manual_seed(seed)
        dims = [N_FEAT, WIDTH, WIDTH, N_OUT]
        self.W, self.b = [], []
        for a, b in zip(dims[:-1], dims[1:]):
            self.W.append((torch.randn(a, b, generator=g) * (1.0 / np.sqrt(a))).to(self.dev))
            self.b.append(torch.zeros(b, device=self.dev))
        self.Wb = [w.to(torch.bfloat16) for w in self.W]
        self.mom = [(torch.zeros_like(w), torch.zeros_like(w)) for w in self.W + self.b]
        self.step = 0
        self.x_mean = torch.zeros(N_FEAT, device=self.dev)
        self.x_std = torch.ones(N_FEAT, device=self.dev)
        # targets are standardised per pair type and output element
        self.y_mean = torch.zeros(len(PAIR_TYPES), N_OUT, device=self.dev)
        self.y_std = torch.ones(len(PAIR_TYPES), N_OUT, device=self.dev)

    def stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)

    def _prep(self, X):
        torch = self.torch
        X = torch.as_tensor(X, device=self.dev, dtype=torch.float32)
        return ((X - self.x_mean) / self.x_std).to(torch.bfloat16).contiguous()

    def forward(self, Xb, keep=False):
        """Xb: (B, N_FEAT) bf16 -> Y (B, N_OUT) FP32 (scaled targets)."""
        torch, k, s = self.torch, self.k, self.stream()
        B = Xb.shape[0]
        H = Xb
        Zs, Hs = [], [Xb]
        for li, (Wb, b) in enumerate(zip(self.Wb, self.b)):
            n_in, n_out = Wb.shape
            Z = torch.empty(B, n_out, device=self.dev, dtype=torch.float32)
            k("lsmlp_gemm_bf16", _p(H), _p(Wb), _p(Z), B, n_out, n_in, n_in, n_out, n_out, 0, 0, 0, s)
            last = li == len(self.Wb) - 1
            Hn = None if last else torch.empty(B, n_out, device=self.dev, dtype=torch.bfloat16)
            k("lsmlp_bias_act", _p(Z), _p(b), _p(Hn), B, n_out, 0 if last else 1, s)
            Zs.append(Z)
            if not last:
                Hs.append(Hn)
                H = Hn
        if keep:
            self._cache = (Zs, Hs)
        return Zs[-1]

    def backward(self, dY):
        """dY: (B, N_OUT) bf16 gradient of the loss w.r.t. the output; returns FP32 grads."""
        torch, k, s = self.torch, self.k, self.stream()
        Zs, Hs = self._cache
        B = dY.shape[0]
        gW = [None] * len(self.W)
        gb = [None] * len(self.b)
        dZ = dY
        for li in range(len(self.W) - 1, -1, -1):
            n_in, n_out = self.W[li].shape
            gW[li] = torch.empty(n_in, n_out, device=self.dev, dtype=torch.float32)
            # dW = H^T dZ
            k("lsmlp_gemm_bf16", _p(Hs[li]), _p(dZ), _p(gW[li]), n_in, n_out, B, n_in, n_out, n_out, 1, 0, 0, s)
            gb[li] = torch.empty(n_out, device=self.dev, dtype=torch.float32)
            k("lsmlp_colsum", _p(dZ), _p(gb[li]), B, n_out, s)
            if li == 0:
                break
            dH = torch.empty(B, n_in, device=self.dev, dtype=torch.float32)
            # dH = dZ W^T
            k("lsmlp_gemm_bf16", _p(dZ), _p(self.Wb[li]), _p(dH), B, n_in, n_out, n_out, n_out, n_in, 0, 1, 0, s)
            dZn = torch.empty(B, n_in, device=self.dev, dtype=torch.bfloat16)
            k("lsmlp_act_grad", _p(dH), _p(Zs[li - 1]), _p(dZn), B * n_in, 1, s)
            dZ = dZn
        return gW, gb

    def loss_grad(self, Y, T, Wm):
        """Masked MSE (mean over unmasked values) and its bf16 gradient."""
        torch, k, s = self.torch, self.k, self.stream()
        n = Y.numel()
        norm = float(Wm.sum().item())
        loss = torch.zeros(1, device=self.dev, dtype=torch.float32)
        dY = torch.empty_like(Y, dtype=torch.bfloat16)
        k("lsmlp_mse", _p(Y), _p(T), _p(Wm), _p(dY), n, 1.0 / max(norm, 1.0), _p(loss), s)
        return loss, dY

    def adam(self, gW, gb, lr, wd=0.0):
        k, s = self.k, self.stream()
        self.step += 1
        params = self.W + self.b
        grads = gW + gb
        for idx, (w, g) in enumerate(zip(params, grads)):
            m, v = self.mom[idx]
            wb = self.Wb[idx] if idx < len(self.W) else None
            k("lsmlp_adam", _p(w), _p(g), _p(m), _p(v), _p(wb), w.numel(), lr, 0.9, 0.999, 1e-8, self.step,
              wd if idx < len(self.W) else 0.0, s)

    def fit(self, X, Y, Wm, epochs=40, batch=2048, lr=2e-3, seed=0, log=None, norm="element"):
        """Train on features X, targets Y with mask Wm. norm = "element": targets
        standardised per pair type and block element; "type": centred per
        element but scaled by one spread per pair type (the loss then weights
        elements by their own spread, i.e. absolute error within a type)."""
        torch = self.torch
        X = torch.as_tensor(X, device=self.dev, dtype=torch.float32)
        self.x_mean = X.mean(0)
        self.x_std = X.std(0).clamp_min(1e-3)
        Yt = torch.as_tensor(Y, device=self.dev, dtype=torch.float32)
        Wt = torch.as_tensor(Wm, device=self.dev, dtype=torch.float32)
        ptype = X[:, :len(PAIR_TYPES)].argmax(1)
        for t in range(len(PAIR_TYPES)):
            sel = ptype == t
            if int(sel.sum()) == 0:
                continue
            w = Wt[sel]
            cnt = w.sum(0).clamp_min(1.0)
            mu = (Yt[sel] * w).sum(0) / cnt
            var = (((Yt[sel] - mu) ** 2) * w).sum(0) / cnt
            self.y_mean[t] = mu
            if norm == "type":
                tot = float((((Yt[sel] - mu) ** 2) * w).sum().item() / max(float(w.sum().item()), 1.0))
                self.y_std[t] = max(tot, 1e-8) ** 0.5
            else:
                self.y_std[t] = var.sqrt().clamp_min(1e-4)
        Yt = (Yt - self.y_mean[ptype]) / self.y_std[ptype] * Wt
        Xb = self._prep(X)
        n = X.shape[0]
        g = torch.Generator(device=self.dev).manual_seed(seed)
        hist = []
        for ep in range(epochs):
            perm = torch.randperm(n, device=self.dev, generator=g)
            lr_ep = lr * 0.5 * (1.0 + np.cos(np.pi * ep / epochs))
            tot = 0.0
            for s0 in range(0, n, batch):
                idx = perm[s0:s0 + batch]
                Yp = self.forward(Xb[idx].contiguous(), keep=True)
                loss, dY = self.loss_grad(Yp, Yt[idx].contiguous(), Wt[idx].contiguous())
                gW, gb = self.backward(dY)
                self.adam(gW, gb, lr_ep)
                tot += float(loss.item()) * idx.numel()
            hist.append(tot / n)
            if log:
                log(ep, hist[-1])
        return hist

    def predict(self, X):
        torch = self.torch
        Xt = torch.as_tensor(X, device=self.dev, dtype=torch.float32)
        ptype = Xt[:, :len(PAIR_TYPES)].argmax(1)
        Yp = self.forward(self._prep(Xt))
        return (Yp * self.y_std[ptype] + self.y_mean[ptype]).cpu().numpy()


# ---- the guess -------------------------------------------------------------------

def water_pairs_data(mol, basis):
    """(pairs, features, per-atom maps) of one water cluster."""
    symbols = [a.symbol for a in mol.atoms]
    xyz = np.array(mol.xyz)
    F = water_frames(xyz, symbols)
    G = atom_descriptors(xyz * ANG_PER_BOHR, symbols)
    Env = atom_environments(xyz * ANG_PER_BOHR, symbols, F)
    pairs = pair_list(xyz * ANG_PER_BOHR, symbols)
    X = pair_features(xyz, symbols, pairs, F, G, Env)
    maps = atom_maps(basis, F)
    return pairs, X, maps


class LearnedGuess:
    THRESHOLD = 1.0e-3

    def __init__(self, mlp, sad):
        self.mlp = mlp
        self.sad = sad

    def guess(self, mol, basis, S, nocc):
        """(D, source, (trace error, idempotency error)); source 'mlp' or 'sad'."""
        pairs, X, maps = water_pairs_data(mol, basis)
        Yp = self.mlp.predict(X)
        D = assemble(basis.nao, pairs, maps, Yp)
        if np.all(np.isfinite(D)):
            Dp = project_idempotent(D, S, nocc)
            err = guess_errors(Dp, S, nocc)
            if max(err) <= self.THRESHOLD and np.all(np.isfinite(Dp)):
                return Dp, "mlp", err
        else:
            err = (np.inf, np.inf)
        return self.sad.density(mol, basis), "sad", err


# ---- data, training and evaluation on seeded water clusters ----------------------

def converged_cluster(ls, n, seed, noise, basis_name="6-31gs", thre=1.0e-12, g_conv=1.0e-6, D0=None, sad=None):
    """(mol, basis, RHF) of one seeded water cluster converged from SAD (or D0)."""
    from .geometry import water_cluster
    from .scf import RHF
    mol = water_cluster(n, seed=seed, noise=noise)
    bas = ls.Basis.from_gbs_file(mol, basis_name)
    scf = RHF(ls, mol, bas, thre_pq=thre, thre_sp=thre, thre_dp=thre)
    if D0 is None and sad is not None:
        D0 = sad.density(mol, bas)
    scf.compute(D0=D0, g_conv=g_conv, maxiter=100)
    return mol, bas, scf


def training_set(ls, specs, sad, noise=(0.05, 5.0), g_conv=1.0e-6, log=None):
    """Features, local-frame targets and masks from converged clusters.
    specs: iterable of (n_water, seed)."""
    Xs, Ys, Ws = [], [], []
    for k, (n, seed) in enumerate(specs):
        mol, bas, scf = converged_cluster(ls, n, seed, noise, g_conv=g_conv, sad=sad)
        pairs, X, maps = water_pairs_data(mol, bas)
        Y, W = local_targets(scf.D, pairs, maps)
        Xs.append(X)
        Ys.append(Y)
        Ws.append(W)
        if log:
            log(k, n, seed, len(scf.trace))
    return np.concatenate(Xs), np.concatenate(Ys), np.concatenate(Ws)


def compare_guesses(ls, guess, specs, noise=(0.05, 5.0), g_conv=1.0e-8, repeats=1):
    """SCF from SAD vs from the learned guess on each cluster: iterations, wall
    time (guess construction included; the fastest of `repeats` runs) and
    final energies."""
    import time
    from .geometry import water_cluster
    from .scf import RHF
    rows = []
    for n, seed in specs:
        mol = water_cluster(n, seed=seed, noise=noise)
        bas = ls.Basis.from_gbs_file(mol, "6-31gs")
        out = {"n_water": n, "seed": seed}
        for name in ("sad", "mlp"):
            best = None
            for _ in range(repeats):
                scf = RHF(ls, mol, bas, thre_pq=1.0e-12, thre_sp=1.0e-12, thre_dp=1.0e-12)
                t0 = time.time()
                if name == "sad":
                    D0, src, err = guess.sad.density(mol, bas), "sad", None
                else:
                    D0, src, err = guess.guess(mol, bas, scf.S, scf.nocc)
                t_guess = time.time() - t0
                E = scf.compute(D0=D0, g_conv=g_conv, maxiter=100)
                wall = time.time() - t0
                if best is None or wall < best:
                    best = wall
            out[name] = {"iterations": len(scf.trace), "seconds": best, "guess_seconds": t_guess,
                         "energy": E, "converged": bool(scf.converged), "source": src,
                         "E_first": scf.trace[0]["E"],
                         "guess_errors": None if err is None else [float(e) for e in err]}
        out["dE"] = out["mlp"]["energy"] - out["sad"]["energy"]
        rows.append(out)
    return rows
