"""lsjk_coulomb_device_noalloc: the J build for callers that may not
allocate device memory during a call (a host framework that owns the GPU's
memory and forbids cudaMalloc after start-up, or a latency-bound loop that
cannot take the device-wide synchronisation of cudaMalloc/cudaFree).

The entry point takes its intermediate buffers from a fixed static device
array instead of the context's growable scratch. These tests call it through
the C ABI (ctypes on liblsjk.so, device buffers from torch) and compare it
with lsjk_coulomb_device on the same context, pair list and density, for two
calls in a row (the static array keeps the previous call's contents, so the
second call shows that nothing stale leaks in), at the 1e-10 elementwise
tolerance of the other J/K parity tests. The first of these calls is the
first build on a fresh context, and the library's count of device
allocations (lsjk_device_allocations) does not move over the two calls. A
basis whose Cartesian D and J alone do not fit the array, and one whose D and
J fit but whose whole build does not, are rejected with LSJK_ENOMEM and a
message, leave J unchanged, and leave the context usable.

This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LSJK_ENOMEM = 3
LSJK_PREC_FP64 = 1


def _lib(ls):
    lib = ctypes.CDLL(ls.LIB_PATH)
    lib.lsjk_last_error.restype = ctypes.c_char_p
    lib.lsjk_device_allocations.restype = ctypes.c_long
    return lib


def _basis_arrays(bas):
    P = bas.primitives
    f64 = lambda v: np.ascontiguousarray(np.array(v, np.float64))
    i32 = lambda v: np.ascontiguousarray(np.array(v, np.int32))
    return dict(c=f64([p.c for p in P]), e=f64([p.e for p in P]), xyz=f64([[p.x, p.y, p.z] for p in P]),
                L=i32([p.L for p in P]), pure=i32([int(p.is_pure) for p in P]), ao=i32([p.aoIdx for p in P]),
                cart=i32([p.cartIdx for p in P]), prim=i32([p.primIdx for p in P]),
                shell=i32([p.shellIdx for p in P]), atom=i32([p.atomIdx for p in P]))


class CApi:
    """Context, basis and pair list created through the C ABI."""

    def __init__(self, ls, bas, thre):
        self.lib = lib = _lib(ls)
        self.ctx = ctypes.c_void_p()
        self._ok(lib.lsjk_context_create(0, ctypes.byref(self.ctx)))
        self._ok(lib.lsjk_context_set_precision(self.ctx, LSJK_PREC_FP64))
        a = self.arrays = _basis_arrays(bas)
        ptr = lambda x: x.ctypes.data_as(ctypes.c_void_p)
        self.bas = ctypes.c_void_p()
        self._ok(lib.lsjk_basis_create(self.ctx, len(a["c"]), ptr(a["c"]), ptr(a["e"]), ptr(a["xyz"]), ptr(a["L"]),
                                       ptr(a["pure"]), ptr(a["ao"]), ptr(a["cart"]), ptr(a["prim"]),
                                       ptr(a["shell"]), ptr(a["atom"]), ctypes.byref(self.bas)))
        self.pl = ctypes.c_void_p()
        self._ok(lib.lsjk_pairlist_build_schwarz(self.ctx, self.bas, self.bas, 1, ctypes.c_float(thre),
                                                 ctypes.byref(self.pl)))
        self.scales = (ctypes.c_double * 1)(1.0)
        self.omegas = (ctypes.c_double * 1)(-1.0)

    def _ok(self, rc):
        assert rc == 0, self.lib.lsjk_last_error()

    def coulomb_device(self, D, J, thre):
        dp = (ctypes.c_void_p * 1)(D.data_ptr())
        jp = (ctypes.c_void_p * 1)(J.data_ptr())
        return self.lib.lsjk_coulomb_device(self.ctx, 1, self.scales, self.omegas, self.pl, self.pl, 1, dp,
                                            ctypes.c_float(thre), ctypes.c_float(thre), jp)

    def coulomb_noalloc(self, D, J, thre):
        return self.lib.lsjk_coulomb_device_noalloc(self.ctx, 1, self.scales, self.omegas, self.pl, self.pl,
                                                    ctypes.c_void_p(D.data_ptr()), ctypes.c_float(thre),
                                                    ctypes.c_float(thre), ctypes.c_void_p(J.data_ptr()))

    def sync(self):
        import torch
        torch.cuda.synchronize()

    def close(self):
        self.sync()
        self.lib.lsjk_pairlist_destroy(self.pl)
        self.lib.lsjk_basis_destroy(self.bas)
        self.lib.lsjk_context_destroy(self.ctx)


def _density(nao, seed):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((nao, 6)) / np.sqrt(nao)
    return X @ X.T


def test_noalloc_matches_device_entry_two_calls(ls):
    import torch
    from lightspeed_b200.geometry import water_cluster
    bas = ls.Basis.from_gbs_file(water_cluster(4, seed=5), "6-31gs")
    api = CApi(ls, bas, 1e-12)
    try:
        n = bas.nao
        Ds = [torch.tensor(_density(n, seed), device="cuda") for seed in (1, 2)]
        J_new = [torch.zeros((n, n), dtype=torch.float64, device="cuda") for _ in Ds]
        api.sync()   # torch filled the buffers on its own stream
        # the two no-alloc calls first: the first J build of this fresh context
        allocs = api.lib.lsjk_device_allocations()
        for D, J in zip(Ds, J_new):
            api._ok(api.coulomb_noalloc(D, J, 1e-12))
        api.sync()
        assert api.lib.lsjk_device_allocations() == allocs, "a no-alloc call allocated device memory"
        for call, (D, J) in enumerate(zip(Ds, J_new)):
            J_ref = torch.zeros((n, n), dtype=torch.float64, device="cuda")
            api.sync()
            api._ok(api.coulomb_device(D, J_ref, 1e-12))
            api.sync()
            diff = (J - J_ref).abs().max().item()
            assert J_ref.abs().max().item() > 1e-3, "empty reference J"
            assert diff < 1e-10, "call %d: max |dJ| = %.3e" % (call + 1, diff)
    finally:
        api.close()


def test_noalloc_rejects_too_large(ls):
    import torch
    from lightspeed_b200.geometry import water_cluster
    bas = ls.Basis.from_gbs_file(water_cluster(64, seed=1), "6-31gs")
    api = CApi(ls, bas, 1e-12)
    try:
        n = bas.nao
        D = torch.tensor(_density(n, 3), device="cuda")
        J = torch.full((n, n), 7.0, dtype=torch.float64, device="cuda")
        api.sync()
        rc = api.coulomb_noalloc(D, J, 1e-12)
        api.sync()
        assert rc == LSJK_ENOMEM
        assert b"static scratch" in api.lib.lsjk_last_error()
        assert bool((J == 7.0).all().item()), "a rejected call wrote to J"
    finally:
        api.close()


def test_noalloc_rejects_a_build_that_outgrows_the_array(ls):
    """D and J (2 x 1368^2 doubles, 30 MB) fit the 32 MiB array, the ket
    records and sort space of the build do not: the build itself refuses,
    before anything reaches J, and the context's own scratch is back in place
    for the next ordinary call."""
    import torch
    from lightspeed_b200.geometry import water_cluster
    bas = ls.Basis.from_gbs_file(water_cluster(72, seed=2), "6-31gs")
    assert 2 * bas.ncart ** 2 * 8 < (32 << 20)
    api = CApi(ls, bas, 1e-12)
    try:
        n = bas.nao
        D = torch.tensor(_density(n, 4), device="cuda")
        J = torch.full((n, n), 7.0, dtype=torch.float64, device="cuda")
        api.sync()
        rc = api.coulomb_noalloc(D, J, 1e-12)
        api.sync()
        assert rc == LSJK_ENOMEM
        msg = api.lib.lsjk_last_error()
        assert b"static scratch" in msg and b"this J build" in msg
        assert bool((J == 7.0).all().item()), "a rejected call wrote to J"
        J2 = torch.zeros((n, n), dtype=torch.float64, device="cuda")
        api.sync()
        api._ok(api.coulomb_device(D, J2, 1e-12))
        api.sync()
        assert J2.abs().max().item() > 1e-3
    finally:
        api.close()
