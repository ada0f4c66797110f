"""Learned SCF guess: BF16 kernels against the CPU oracle (oracle/mlp_ref.py),
the SAD guess, the local-frame block transforms, and a small end-to-end
check that a network trained on converged densities starts the SCF closer to
the answer than SAD and converges to the same energy.

Tolerances: the BF16 tensor-core GEMM is compared with float64 sums of the
same bf16 inputs at 1e-5 relative (FP32 accumulation of up to 256 terms), in
all four transposes and accumulating; the
network's output and gradients at 2e-2 of their largest value, since an
accumulation-order difference can flip one bf16 rounding of a hidden value."""
import numpy as np
import pytest

from oracle import mlp_ref

pytestmark = pytest.mark.gpu


def _bf16_tensor(torch, a):
    return torch.tensor(mlp_ref.bf16(a), device="cuda").to(torch.bfloat16)


@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_gemm_bf16_matches_float64(ls, ta, tb):
    import torch
    from lightspeed_b200.guess import _Lib, _p
    k = _Lib(ls)
    rng = np.random.default_rng(ta * 2 + tb)
    M, N, K = 77, 130, 93
    A = rng.standard_normal((K, M) if ta else (M, K)).astype(np.float32)
    B = rng.standard_normal((N, K) if tb else (K, N)).astype(np.float32)
    Ab, Bb = mlp_ref.bf16(A), mlp_ref.bf16(B)
    ref = (Ab.T if ta else Ab).astype(np.float64) @ (Bb.T if tb else Bb).astype(np.float64)
    C = torch.zeros(M, N, device="cuda")
    At, Bt = _bf16_tensor(torch, A), _bf16_tensor(torch, B)   # keep the inputs alive over the launch
    torch.cuda.synchronize()
    k("lsmlp_gemm_bf16", _p(At), _p(Bt), _p(C), M, N, K, M if ta else K, K if tb else N, N, ta, tb, 0, None)
    torch.cuda.synchronize()
    assert np.max(np.abs(C.cpu().numpy() - ref)) <= 1e-5 * np.max(np.abs(ref))
    # accumulate into C (the tensor-core tiles add to what is there)
    k("lsmlp_gemm_bf16", _p(At), _p(Bt), _p(C), M, N, K, M if ta else K, K if tb else N, N, ta, tb, 1, None)
    torch.cuda.synchronize()
    assert np.max(np.abs(C.cpu().numpy() - 2.0 * ref)) <= 2e-5 * np.max(np.abs(ref))


def test_mlp_forward_and_gradients_match_oracle(ls):
    import torch
    from lightspeed_b200.guess import MLP, N_FEAT, N_OUT
    net = MLP(ls, seed=3)
    rng = np.random.default_rng(5)
    B = 300
    X = mlp_ref.bf16(rng.standard_normal((B, N_FEAT)).astype(np.float32))
    T = rng.standard_normal((B, N_OUT)).astype(np.float32) * 0.1
    Wm = (rng.random((B, N_OUT)) < 0.7).astype(np.float32)
    Xb = torch.tensor(X, device="cuda").to(torch.bfloat16)
    Y = net.forward(Xb, keep=True)
    loss, dY = net.loss_grad(Y, torch.tensor(T, device="cuda"), torch.tensor(Wm, device="cuda"))
    gW, gb = net.backward(dY)
    torch.cuda.synchronize()
    Wb = [w.float().cpu().numpy() for w in net.Wb]
    bb = [b.cpu().numpy() for b in net.b]
    Yr, Zs, Hs = mlp_ref.forward(X, Wb, bb)
    assert np.max(np.abs(Y.cpu().numpy() - Yr)) <= 2e-2 * np.max(np.abs(Yr))
    lr, dYr = mlp_ref.mse_grad(Y.cpu().numpy(), T, Wm)   # same output: isolates the backward pass
    assert abs(float(loss.item()) - lr) <= 1e-4 * lr
    gWr, gbr = mlp_ref.backward(dY.float().cpu().numpy(), Wb, Zs, Hs)
    for g, r in zip(gW + gb, gWr + gbr):
        assert np.max(np.abs(g.cpu().numpy() - r)) <= 2e-2 * np.max(np.abs(r))


def test_sad_guess_electron_count(ls):
    from lightspeed_b200.geometry import water_cluster
    from lightspeed_b200.sad import SAD
    mol = water_cluster(3, seed=2)
    bas = ls.Basis.from_gbs_file(mol, "6-31gs")
    res = ls.ResourceList.build()
    S = ls.IntBox.overlap(res, ls.PairList.build_schwarz(bas, bas, True, 1e-14)).np
    D = SAD(ls, "6-31gs").density(mol, bas)
    assert abs(np.sum(D * S) - 15.0) < 1e-8      # 3 waters: 15 electron pairs
    assert np.allclose(D, D.T)


def test_local_frame_blocks_round_trip(ls):
    """A converged density mapped to local-frame blocks and back is unchanged
    on every predicted pair block, and the local blocks of a rigidly rotated copy of
    the cluster equal the original ones (the frames carry the rotation)."""
    from lightspeed_b200 import guess as g
    from lightspeed_b200.geometry import water_cluster
    from lightspeed_b200.molecule import Molecule
    from lightspeed_b200.sad import SAD
    from lightspeed_b200.scf import RHF
    ls.set_precision(ls.PREC_FP64)
    try:
        mol = water_cluster(2, seed=4)
        Rm = np.linalg.qr(np.random.default_rng(9).standard_normal((3, 3)))[0]
        if np.linalg.det(Rm) < 0:
            Rm[:, 0] *= -1
        mol_r = Molecule.from_arrays([a.symbol for a in mol.atoms], np.array(mol.xyz) @ Rm.T)
        blocks = []
        for m in (mol, mol_r):
            bas = ls.Basis.from_gbs_file(m, "6-31gs")
            scf = RHF(ls, m, bas, thre_pq=1e-14, thre_sp=1e-14, thre_dp=1e-14)
            scf.compute(D0=SAD(ls, "6-31gs").density(m, bas), g_conv=1e-9)
            pairs, X, maps = g.water_pairs_data(m, bas)
            Y, W = g.local_targets(scf.D, pairs, maps)
            D2 = g.assemble(bas.nao, pairs, maps, Y)
            for i, j, _ in pairs:
                li, ni, _ = maps[i]
                lj, nj, _ = maps[j]
                assert np.max(np.abs(D2[li:li + ni, lj:lj + nj] - scf.D[li:li + ni, lj:lj + nj])) < 1e-5
            blocks.append((Y, X))
        assert np.max(np.abs(blocks[0][0] - blocks[1][0])) < 1e-5
        assert np.max(np.abs(blocks[0][1] - blocks[1][1])) < 1e-4
    finally:
        ls.set_precision(ls.PREC_MIXED)


def test_learned_guess_beats_sad_small(ls):
    """Train on 48 converged 2-4 water clusters; on held-out 5-water clusters
    the learned guess starts the SCF at a lower energy than SAD, needs no more
    iterations, and reaches the same energy (1e-8 Eh)."""
    from lightspeed_b200 import guess as g
    from lightspeed_b200.sad import SAD
    ls.set_precision(ls.PREC_FP64)
    try:
        sad = SAD(ls, "6-31gs")
        specs = [(2 + (s % 3), 1000 + s) for s in range(48)]
        X, Y, W = g.training_set(ls, specs, sad)
        net = g.MLP(ls, seed=0)
        hist = net.fit(X, Y, W, epochs=60, batch=512, lr=2e-3)
        assert hist[-1] < 0.5 * hist[0]   # standardised targets: the loss starts near 1
        rows = g.compare_guesses(ls, g.LearnedGuess(net, sad), [(5, 5000), (5, 5001)])
        for r in rows:
            assert r["mlp"]["source"] == "mlp"
            assert abs(r["dE"]) < 1e-8
            assert r["mlp"]["E_first"] < r["sad"]["E_first"]
            assert r["mlp"]["iterations"] <= r["sad"]["iterations"]
    finally:
        ls.set_precision(ls.PREC_MIXED)
