"""CUDA-graph capture of the device builds and the schedule autotuner.

Graph: the J and K builds of a water cluster are captured once and replayed;
the replay reads the density buffer's current contents, so two replays with
two different densities must equal direct builds of those densities. The
autotuner times candidate schedules on scratch outputs and keeps the
fastest: builds made while it tunes, and after, equal the untuned ones, and
its table can be read and restored. Tolerance: 1e-10 elementwise (FP64).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(ls, n=4, seed=8):
    from lightspeed_b200.geometry import water_cluster
    bas = ls.Basis.from_gbs_file(water_cluster(n, seed=seed), "6-31gs")
    pl = ls.PairList.build_schwarz(bas, bas, True, 1e-14)
    return bas, pl


def _density(nao, seed):
    X = np.random.default_rng(seed).standard_normal((nao, 8)) / np.sqrt(nao)
    return X @ X.T


def _direct(ls, pl, D):
    res = ls.ResourceList.build()
    ew = ls.Ewald.coulomb()
    J = ls.IntBox.coulomb(res, ew, pl, pl, ls.Tensor.array(D), 1e-14, 1e-14).np.copy()
    K = ls.IntBox.exchange(res, ew, pl, pl, ls.Tensor.array(D), True, 1e-14, 1e-14).np.copy()
    return J, K


def test_graph_replay_matches_direct(ls):
    import torch
    ls.set_precision(ls.PREC_FP64)
    try:
        bas, pl = _setup(ls)
        ew = ls.Ewald.coulomb()
        dev = torch.device("cuda", 0)
        stream = torch.cuda.ExternalStream(ls.stream_handle(), device=dev)
        D1, D2 = _density(bas.nao, 1), _density(bas.nao, 2)
        Dd = torch.tensor(D1, device=dev)
        Jd = torch.zeros_like(Dd)
        Kd = torch.zeros_like(Dd)
        torch.cuda.synchronize()

        def build():
            ls.coulomb_device(ew, pl, pl, [Dd.data_ptr()], [Jd.data_ptr()], 1e-14, 1e-14)
            ls.exchange_device(ew, pl, pl, [Dd.data_ptr()], True, [Kd.data_ptr()], 1e-14, 1e-14)

        build()                     # the first build does the one-time set-up outside the capture
        stream.synchronize()
        ls.graph_begin()
        build()
        g = ls.graph_end()
        for D in (D1, D2):
            with torch.cuda.stream(stream):
                Dd.copy_(torch.tensor(D, device=dev))
                Jd.zero_()
                Kd.zero_()
            g.launch()
            stream.synchronize()
            J, K = _direct(ls, pl, D)
            assert np.max(np.abs(Jd.cpu().numpy() - J)) < 1e-10
            assert np.max(np.abs(Kd.cpu().numpy() - K)) < 1e-10
        del g
    finally:
        ls.set_precision(ls.PREC_MIXED)


def test_autotuner_keeps_results(ls):
    ls.set_precision(ls.PREC_FP64)
    saved = ls.get_tune_table()
    try:
        bas, pl = _setup(ls, n=5, seed=9)
        D = _density(bas.nao, 3)
        J0, K0 = _direct(ls, pl, D)
        ls.set_autotune(True)
        J1, K1 = _direct(ls, pl, D)      # built while candidate schedules are timed
        ls.set_autotune(False)
        J2, K2 = _direct(ls, pl, D)      # built with the chosen schedules
        for J, K in ((J1, K1), (J2, K2)):
            assert np.max(np.abs(J - J0)) < 1e-10
            assert np.max(np.abs(K - K0)) < 1e-10
        table = ls.get_tune_table()
        assert any(v > 0 for v in table)
        ls.set_tune_table(saved)
        assert list(ls.get_tune_table()) == list(saved)
    finally:
        ls.set_autotune(False)
        ls.set_tune_table(saved)
        ls.set_precision(ls.PREC_MIXED)
