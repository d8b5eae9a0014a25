"""FP64 CPU reference of the warm-start MLP (test infrastructure only).

Only tests/ import this module; the product never does.  It restates the
network that fmm3dbie_b200/csrc/cuda/mlp.cu trains and runs: 10 -> 256 ->
256 -> 256 -> 256 -> 2 with tanh on the hidden layers and a mean squared
error loss, in float64 with numpy.  The reference (fmm3dbie) has no learned
component -- its solvers start GMRES from zero (helm_comb_dir.f:2222 calls
zgmres_guru, gmres_routs.f90:13) -- so this module is pinned against its own
central finite differences (tests/test_mlp_oracle.py), not against reference
output.

With ``emulate_bf16=True`` the weights and every stored activation and
activation gradient are rounded to bfloat16 where the CUDA kernels store
them in bfloat16, so the comparison with the device gradient measures the
kernels' arithmetic, not the storage format.
"""
from __future__ import annotations

import numpy as np

N_IN, WIDTH, N_OUT = 10, 256, 2
# flat parameter layout (float32 on the device)
OFF_W = [0, 2560, 2560 + 65536, 2560 + 2 * 65536, 2560 + 3 * 65536]
SHAPE_W = [(WIDTH, N_IN), (WIDTH, WIDTH), (WIDTH, WIDTH), (WIDTH, WIDTH), (N_OUT, WIDTH)]
NW = OFF_W[4] + N_OUT * WIDTH
OFF_B = [NW, NW + 256, NW + 512, NW + 768, NW + 1024]
SHAPE_B = [WIDTH, WIDTH, WIDTH, WIDTH, N_OUT]
NPARAMS = OFF_B[4] + N_OUT


def bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, np.float64).astype(np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, np.float64)
    W = [p[o:o + a * b].reshape(a, b) for o, (a, b) in zip(OFF_W, SHAPE_W)]
    b = [p[o:o + n] for o, n in zip(OFF_B, SHAPE_B)]
    return W, b


def pack(W, b):
    p = np.zeros(NPARAMS)
    for o, w in zip(OFF_W, W):
        p[o:o + w.size] = w.ravel()
    for o, v in zip(OFF_B, b):
        p[o:o + v.size] = v
    return p


def forward(p, X, emulate_bf16=False):
    W, b = unpack(p)
    r = bf16 if emulate_bf16 else (lambda v: v)
    W = [r(w) for w in W]
    h = np.asarray(X, np.float64)
    H = []
    for layer in range(4):
        h = r(np.tanh(h @ W[layer].T + b[layer]))
        H.append(h)
    return h @ W[4].T + b[4], H


def loss_and_grad(p, X, T, emulate_bf16=False):
    """Mean over rows of |Y - T|^2 and its gradient (flat, parameter layout)."""
    W, b = unpack(p)
    r = bf16 if emulate_bf16 else (lambda v: v)
    Wr = [r(w) for w in W]
    X = np.asarray(X, np.float64)
    Y, H = forward(p, X, emulate_bf16)
    m = X.shape[0]
    D = Y - np.asarray(T, np.float64)
    loss = float(np.sum(D * D) / m)
    dY = 2.0 * D / m
    gW = [None] * 5
    gb = [None] * 5
    gW[4] = dY.T @ H[3]
    gb[4] = dY.sum(0)
    dZ = r((dY @ Wr[4]) * (1.0 - H[3] ** 2))
    for layer in (3, 2, 1):
        gW[layer] = dZ.T @ H[layer - 1]
        gb[layer] = dZ.sum(0)
        dZ = r((dZ @ Wr[layer]) * (1.0 - H[layer - 1] ** 2))
    gW[0] = dZ.T @ X
    gb[0] = dZ.sum(0)
    return loss, pack(gW, gb)
