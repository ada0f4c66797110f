"""The quartet-code generator (lightspeed_b200/csrc/gen_kernels.py): which
classes get straight-line code, and the order conventions the loop forms and
the warp kernels rely on (quartet_loops.cuh: herm_pos; kwarp.cuh / kgrad.cu:
Cartesian components in CCA order)."""
import importlib.util
import os

HERE = os.path.dirname(os.path.abspath(__file__))
GEN = os.path.join(HERE, "..", "lightspeed_b200", "csrc", "gen_kernels.py")


def _gen():
    spec = importlib.util.spec_from_file_location("gen_kernels", GEN)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_every_class_up_to_d_is_emitted():
    g = _gen()
    for LB in range(6):
        for LK in range(5):
            assert g.j_emitted(LB, LK)
    for L1 in range(3):
        for L2 in range(3):
            for L3 in range(3):
                for L4 in range(3):
                    assert g.k_emitted(L1, L2, L3, L4)


def test_f_class_limits():
    g = _gen()
    # J: emitted up to J_TERMS contraction terms, the largest f classes in the loop form
    assert g.j_emitted(6, 0) and g.j_emitted(3, 5)
    assert not g.j_emitted(6, 6) and not g.j_emitted(7, 4) and not g.j_emitted(5, 5)
    # K: f classes emitted below K_COMBOS Cartesian combinations (the warp kernel takes the rest)
    assert g.k_emitted(3, 0, 0, 0) and g.k_emitted(0, 1, 3, 1)
    assert not g.k_emitted(3, 3, 0, 0) and not g.k_emitted(1, 3, 3, 3)


def test_herm_pos_matches_generator_order():
    """herm_pos(t, u, v) = nherm(N-1) + i(i+1)/2 + v with N = t+u+v, i = u+v is the
    index of (t, u, v) in herm_list (shell-major, CCA order within a shell)."""
    g = _gen()
    for L in range(14):
        for k, (t, u, v) in enumerate(g.herm_list(L)):
            N, i = t + u + v, u + v
            assert k == (g.nherm(N - 1) if N > 0 else 0) + i * (i + 1) // 2 + v


def test_cartesian_order():
    """Component k of a shell of angular momentum L: (L - j, j - z, z) over
    j = 0..L, z = 0..j, the loop order of the warp kernels' job tables."""
    g = _gen()
    for L in range(5):
        order = [(L - j, j - z, z) for j in range(L + 1) for z in range(j + 1)]
        assert order == g.cart_list(L)
        assert len(order) == g.ncart(L)
