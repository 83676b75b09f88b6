"""CPU oracle of the per-cage-vertex MLP (test infrastructure only): the
forward pass, mean-squared-error loss and gradients in float64 numpy, with the
GELU tanh form of Hendrycks & Gimpel, "Gaussian Error Linear Units" (2016):
gelu(x) = x/2 (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))).

Inputs are the BF16 values the GPU sees (weights and features rounded to
BF16 by the caller), so the oracle checks the tensor-core kernels' FP32
accumulation and the backward algebra, not the rounding of the inputs.
"""
import numpy as np

C0 = np.sqrt(2.0 / np.pi)


def bf16_round(x):
    """Round-to-nearest-even to bfloat16, returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(C0 * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    t = np.tanh(C0 * (x + 0.044715 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * C0 * (1.0 + 3 * 0.044715 * x * x)


def forward(X, Ws, bs):
    """Returns Y and the pre-activations Z and layer inputs H."""
    H, Z = [np.asarray(X, np.float64)], []
    for l in range(len(Ws) - 1):
        Z.append(H[-1] @ Ws[l].T + bs[l])
        H.append(gelu(Z[-1]))
    return H[-1] @ Ws[-1].T + bs[-1], Z, H


def loss_and_grads(X, Ws, bs, T):
    """Mean squared error over all outputs and its gradients (dW, db)."""
    Y, Z, H = forward(X, Ws, bs)
    m, n = T.shape
    dZ = 2.0 * (Y - T) / (m * n)
    loss = float(((Y - T) ** 2).mean())
    gW, gb = [None] * len(Ws), [None] * len(Ws)
    for l in range(len(Ws) - 1, -1, -1):
        gW[l] = dZ.T @ H[l]
        gb[l] = dZ.sum(0)
        if l > 0:
            dZ = (dZ @ Ws[l]) * gelu_grad(Z[l - 1])
    return loss, Y, gW, gb
