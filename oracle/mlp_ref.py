"""CPU oracle of the learned-guess network (test infrastructure only).

A numpy restatement of the BF16 multilayer perceptron that
lightspeed_b200/guess.py runs on the GPU kernels of include/lsmlp.h: the same
rounding points (bfloat16 inputs, weights, hidden activations and
back-propagated gradients, round to nearest even), with every product summed
in float64 here instead of FP32 there. The GPU forward pass and gradients are
checked against it in tests/test_guess_gpu.py.
"""
import numpy as np


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    b = np.ascontiguousarray(np.asarray(x, np.float32)).view(np.uint32)
    r = ((b >> 16) & 1) + np.uint32(0x7FFF)
    return ((b + r) & np.uint32(0xFFFF0000)).view(np.float32)


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(Xb, Wb, b):
    """Xb (B, n0) bf16 values; Wb list of bf16 weight matrices; b list of FP32 biases.
    Returns (Y, Zs, Hs) with Zs the FP32 pre-activations and Hs the bf16 layer inputs."""
    H = Xb.astype(np.float64)
    Zs, Hs = [], [Xb]
    for li, (W, bias) in enumerate(zip(Wb, b)):
        Z = (H @ W.astype(np.float64)).astype(np.float32) + bias.astype(np.float32)
        Zs.append(Z)
        if li < len(Wb) - 1:
            Hn = bf16(silu(Z.astype(np.float64)).astype(np.float32))
            Hs.append(Hn)
            H = Hn.astype(np.float64)
    return Zs[-1], Zs, Hs


def mse_grad(Y, T, Wm):
    norm = max(float(Wm.sum()), 1.0)
    d = Y.astype(np.float64) - T
    loss = float(np.sum(Wm * d * d) / norm)
    return loss, bf16((2.0 * Wm * d / norm).astype(np.float32))


def backward(dY, Wb, Zs, Hs):
    """Gradients (FP32 values) of all weights and biases for the bf16 output gradient dY."""
    n = len(Wb)
    gW, gb = [None] * n, [None] * n
    dZ = dY.astype(np.float64)
    for li in range(n - 1, -1, -1):
        gW[li] = (Hs[li].astype(np.float64).T @ dZ).astype(np.float32)
        gb[li] = dZ.sum(axis=0).astype(np.float32)
        if li == 0:
            break
        dH = (dZ @ Wb[li].astype(np.float64).T).astype(np.float32)
        dZ = bf16((dH.astype(np.float64) * silu_grad(Zs[li - 1].astype(np.float64))).astype(np.float32))
        dZ = dZ.astype(np.float64)
    return gW, gb
