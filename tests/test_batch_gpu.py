"""Batched densities: IntBox.coulombMulti / exchangeMulti with several
densities in one call against one call per density.

A batched build serves all its densities with one launch per class (J: CTA
z-slices of up to four densities; K: task lists per group of four densities,
run once per sub-slot), shares each quartet between up to four densities and
screens with the largest |D| of the group, so it evaluates a superset of each
density's quartets: results agree with the per-density builds to the size of
the quartets the single-density screen drops. At thresp = 1e-14 that is far
below the 1e-10 elementwise FP64 tolerance. In mixed precision the batch also
moves some quartets from FP32 to FP64 (the estimate uses the batch's largest
|D|), so there the check is the mixed-precision tolerance (1e-6 against the
FP64 result) of the other mixed tests. The densities are non-symmetric rank-3
products (the shape of response trial vectors); the bare Coulomb operator and
erf-attenuated interactions (omega = 0.3) are both covered."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _system(ls):
    from lightspeed_b200.geometry import water_cluster
    bas = ls.Basis.from_gbs_file(water_cluster(4, seed=3), "6-31gs")
    pl = ls.PairList.build_schwarz(bas, bas, True, 1e-14)
    return bas, pl


def _densities(n, nao, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        X = rng.standard_normal((nao, 3)) / np.sqrt(nao)
        Y = rng.standard_normal((nao, 3)) / np.sqrt(nao)
        out.append(X @ Y.T)
    return out


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("ndens", [1, 3, 6])
@pytest.mark.parametrize("ewald", [([1.0], [-1.0]), ([1.0], [0.3])])
def test_multi_matches_single(ls, prec, ndens, ewald):
    ls.set_precision(ls.PREC_FP64 if prec == "fp64" else ls.PREC_MIXED)
    try:
        bas, pl = _system(ls)
        res = ls.ResourceList.build()
        ew = ls.Ewald(*ewald)
        Ds = [ls.Tensor.array(D) for D in _densities(ndens, bas.nao, 7 + ndens)]
        thresp = 1e-14
        thredp = thresp if prec == "fp64" else 1e-5
        tol = 1e-10 if prec == "fp64" else 1e-6
        Jm = ls.IntBox.coulombMulti(res, ew, pl, pl, Ds, thresp, thredp)
        Km = ls.IntBox.exchangeMulti(res, ew, pl, pl, Ds, False, thresp, thredp)
        assert len(Jm) == ndens and len(Km) == ndens
        ls.set_precision(ls.PREC_FP64)
        for D, J, K in zip(Ds, Jm, Km):
            J1 = ls.IntBox.coulomb(res, ew, pl, pl, D, thresp, thresp)
            K1 = ls.IntBox.exchange(res, ew, pl, pl, D, False, thresp, thresp)
            assert np.max(abs(J.np - J1.np)) < tol
            assert np.max(abs(K.np - K1.np)) < tol
    finally:
        ls.set_precision(ls.PREC_MIXED)


def test_multi_fp64_vs_oracle(ls):
    """Four densities batched in FP64 against the oracle, one density at a time."""
    from oracle import ref
    if not ref.available():
        pytest.skip("reference CPU IntBox not built")
    ls.set_precision(ls.PREC_FP64)
    try:
        bas, pl = _system(ls)
        res = ls.ResourceList.build()
        ew = ls.Ewald([1.0], [-1.0])
        Dn = _densities(4, bas.nao, 11)
        Jm = ls.IntBox.coulombMulti(res, ew, pl, pl, [ls.Tensor.array(D) for D in Dn], 1e-14, 1e-14)
        rb = ref.RefBasis(ref.prim_arrays(bas))
        rp = ref.RefPairs(rb, rb, True, 1e-14)
        for D, J in zip(Dn, Jm):
            Jr = ref.coulomb(rp, rp, D, 1e-14, 1e-14)
            assert np.max(abs(J.np - Jr)) < 1e-10
    finally:
        ls.set_precision(ls.PREC_MIXED)


def test_thirteen_densities_one_build_vs_oracle(ls):
    """Thirteen densities in one build (four density groups, the last one
    partial: every class kernel runs once over all groups and sub-slots)
    against the oracle one density at a time, J and K, FP64."""
    from oracle import ref
    if not ref.available():
        pytest.skip("reference CPU IntBox not built")
    ls.set_precision(ls.PREC_FP64)
    try:
        bas, pl = _system(ls)
        res = ls.ResourceList.build()
        ew = ls.Ewald([1.0], [-1.0])
        Dn = _densities(13, bas.nao, 23)
        Ds = [ls.Tensor.array(D) for D in Dn]
        Jm = ls.IntBox.coulombMulti(res, ew, pl, pl, Ds, 1e-14, 1e-14)
        Km = ls.IntBox.exchangeMulti(res, ew, pl, pl, Ds, False, 1e-14, 1e-14)
        rb = ref.RefBasis(ref.prim_arrays(bas))
        rp = ref.RefPairs(rb, rb, True, 1e-14)
        for D, J, K in zip(Dn, Jm, Km):
            assert np.max(abs(J.np - ref.coulomb(rp, rp, D, 1e-14, 1e-14))) < 1e-10
            assert np.max(abs(K.np - ref.exchange(rp, rp, D, False, 1e-14, 1e-14))) < 1e-10
    finally:
        ls.set_precision(ls.PREC_MIXED)


def test_concurrent_streams_match_engine(ls):
    """Builds enqueued on two extra engine contexts (ls.Stream, own CUDA
    streams and scratch) for two different molecules at once equal the main
    context's builds (1e-10): the contexts share pair lists but nothing else."""
    import torch
    from lightspeed_b200.geometry import water_cluster
    ls.set_precision(ls.PREC_FP64)
    try:
        res = ls.ResourceList.build()
        ew = ls.Ewald.coulomb()
        mols = []
        for n, seed in ((3, 21), (4, 22)):
            bas = ls.Basis.from_gbs_file(water_cluster(n, seed=seed), "6-31gs")
            pl = ls.PairList.build_schwarz(bas, bas, True, 1e-14)
            D = _densities(1, bas.nao, seed)[0]
            D = D + D.T
            J1 = ls.IntBox.coulomb(res, ew, pl, pl, ls.Tensor.array(D), 1e-14, 1e-14).np
            K1 = ls.IntBox.exchange(res, ew, pl, pl, ls.Tensor.array(D), True, 1e-14, 1e-14).np
            mols.append((pl, D, J1, K1))
        streams = [ls.Stream(), ls.Stream()]
        out = []
        for (pl, D, _, _), st in zip(mols, streams):
            Dd = torch.tensor(D, device="cuda")
            Jd = torch.zeros_like(Dd)
            Kd = torch.zeros_like(Dd)
            out.append((Dd, Jd, Kd))
        torch.cuda.synchronize()
        for (pl, _, _, _), st, (Dd, Jd, Kd) in zip(mols, streams, out):
            st.coulomb_device(ew, pl, pl, [Dd.data_ptr()], [Jd.data_ptr()], 1e-14, 1e-14)
            st.exchange_device(ew, pl, pl, [Dd.data_ptr()], True, [Kd.data_ptr()], 1e-14, 1e-14)
        for st in streams:
            torch.cuda.ExternalStream(st.stream_handle()).synchronize()
        for (_, _, J1, K1), (_, Jd, Kd) in zip(mols, out):
            assert np.max(np.abs(Jd.cpu().numpy() - J1)) < 1e-10
            assert np.max(np.abs(Kd.cpu().numpy() - K1)) < 1e-10
    finally:
        ls.set_precision(ls.PREC_MIXED)


def test_batched_scf_matches_single(ls):
    """The GPU-resident lockstep SCF (scf_batched.BatchedRHF, molecules grouped
    by size, J/K through the device entry points into its own tensors)
    converges every molecule to the energy of a separate RHF.compute (1e-8 Eh)."""
    import torch
    from lightspeed_b200.geometry import water_cluster
    from lightspeed_b200.sad import SAD
    from lightspeed_b200.scf import RHF
    from lightspeed_b200.scf_batched import BatchedRHF
    ls.set_precision(ls.PREC_FP64)
    try:
        sad = SAD(ls, "6-31gs")
        mols = [water_cluster(n, seed=s) for n, s in ((1, 31), (2, 32), (2, 33), (3, 34))]
        rhfs = [RHF(ls, m, ls.Basis.from_gbs_file(m, "6-31gs"), thre_pq=1e-12, thre_sp=1e-12, thre_dp=1e-12)
                for m in mols]
        ref = []
        for m, r in zip(mols, rhfs):
            ref.append(r.compute(D0=sad.density(m, r.basis), g_conv=1e-8, maxiter=100))
        dev = torch.device("cuda", 0)
        stream = torch.cuda.ExternalStream(ls.stream_handle(), device=dev)
        bat = BatchedRHF(ls, rhfs, dev)
        bat.set_guess([sad.density(m, r.basis) for m, r in zip(mols, rhfs)])
        ew = ls.Ewald.coulomb()
        while not bat.finished() and bat.iteration < 100:
            bat.prepare()
            torch.cuda.synchronize()
            for gi, b in bat.active():
                d, j, k = bat.targets(gi, b)
                pl = rhfs[bat.groups[gi]["idx"][b]].pairs
                ls.coulomb_device(ew, pl, pl, [d], [j], 1e-12, 1e-12)
                ls.exchange_device(ew, pl, pl, [d], True, [k], 1e-12, 1e-12)
            stream.synchronize()
            bat.update(1e-8)
        assert bat.converged().all()
        assert np.max(np.abs(bat.energies() - np.array(ref))) < 1e-8
    finally:
        ls.set_precision(ls.PREC_MIXED)
