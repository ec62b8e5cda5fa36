"""CPU oracle of the learned radiance cache (test infrastructure only).

numpy restatement of the network the device kernels evaluate and train:
the multi-resolution hash-grid encoding (Muller et al. 2022: per-level
resolution floor(base * b^l), dense indexing where (res+1)^3 fits the table,
else (x * 1) ^ (y * 2654435761) ^ (z * 805459861) mod T, trilinear fp32
interpolation of fp16 feature pairs), the 4 x 64 ReLU MLP without biases, the
relative L2 loss sum_c (y_c - t_c)^2 / (y_c^2 + 0.01) with the denominator
held constant, its backward pass, and Adam (Kingma & Ba 2015).

The reference (VoxelEngine3.0) has no learned cache; this module pins the
device implementation against the mathematics, and its own backward pass is
checked against central finite differences in tests.  ``bf16=True`` rounds
weights, activations and gradients to bf16 exactly where the device kernels
store bf16 operand tiles, so device and oracle agree to f32-accumulation
order; ``bf16=False`` is the plain float64 network used for the finite
difference check.
"""
from __future__ import annotations

import math

import numpy as np

LEVELS = 16
WIDTH = 64
LAYERS = 5
OUT = 3
PRIMES = (1, 2654435761, 805459861)


def bf16(x):
    """Round to bf16 (nearest even), returned as float32 values."""
    x = np.ascontiguousarray(np.asarray(x, np.float32))
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32).reshape(x.shape)


def make_grid(log2_table=19, base=16, max_res=2048):
    b = math.exp((math.log(max_res) - math.log(base)) / (LEVELS - 1))
    T = 1 << log2_table
    res, dense = [], []
    for lv in range(LEVELS):
        r = max(int(math.floor(base * b ** lv + 1e-9)), 1)
        res.append(r)
        dense.append((r + 1) ** 3 <= T)
    return {"res": res, "dense": dense, "log2T": log2_table}


def oct_encode(v):
    """Octahedral map of unit vectors to [-1, 1]^2 (Cigolle et al. 2014)."""
    v = np.asarray(v, np.float64)
    p = v / np.abs(v).sum(axis=-1, keepdims=True)
    x, y, z = p[..., 0], p[..., 1], p[..., 2]
    neg = z < 0
    ox = np.where(neg, (1 - np.abs(y)) * np.where(x >= 0, 1.0, -1.0), x)
    oy = np.where(neg, (1 - np.abs(x)) * np.where(y >= 0, 1.0, -1.0), y)
    return np.stack([ox, oy], -1).astype(np.float32)


def level_corners(grid, lv, pos):
    """Corner indices (n, 8) and trilinear weights (n, 8), in the device's f32
    operation order."""
    R = grid["res"][lv]
    s = np.float32(R)
    p = np.asarray(pos, np.float32)
    x = p * s
    f0 = np.floor(x)
    i = np.minimum(np.maximum(f0, np.float32(0)).astype(np.int64), R - 1)
    f = (x - i.astype(np.float32)).astype(np.float32)
    T = 1 << grid["log2T"]
    idx = np.zeros((p.shape[0], 8), np.int64)
    w = np.zeros((p.shape[0], 8), np.float32)
    one = np.float32(1)
    for c in range(8):
        cx = i[:, 0] + (c & 1)
        cy = i[:, 1] + ((c >> 1) & 1)
        cz = i[:, 2] + ((c >> 2) & 1)
        if grid["dense"][lv]:
            R1 = R + 1
            idx[:, c] = cx + R1 * (cy + R1 * cz)
        else:
            h = (cx.astype(np.uint64) * PRIMES[0]) ^ (cy.astype(np.uint64) * PRIMES[1] & 0xFFFFFFFF) ^ \
                (cz.astype(np.uint64) * PRIMES[2] & 0xFFFFFFFF)
            idx[:, c] = (h & (T - 1)).astype(np.int64)
        wx = f[:, 0] if c & 1 else one - f[:, 0]
        wy = f[:, 1] if c & 2 else one - f[:, 1]
        wz = f[:, 2] if c & 4 else one - f[:, 2]
        w[:, c] = (wx * wy).astype(np.float32) * wz
    return idx, w


def encode(grid, table, inputs, bf16_round=True):
    """inputs: (n, 8) float32 rows [px, py, pz, reserved, nx, ny, vx, vy];
    table: (levels, T, 2) parameters.  Returns the (n, 64) input matrix."""
    inputs = np.asarray(inputs, np.float32)
    n = inputs.shape[0]
    pos = inputs[:, 0:3]
    if bf16_round:
        tab = np.asarray(table, np.float32).astype(np.float16).astype(np.float32)
    else:
        tab = np.asarray(table, np.float64)
    X = np.zeros((n, WIDTH), np.float64)
    for lv in range(LEVELS):
        idx, w = level_corners(grid, lv, pos)
        if bf16_round:
            f0 = np.zeros(n, np.float32)
            f1 = np.zeros(n, np.float32)
            for c in range(8):
                f0 = (f0 + w[:, c] * tab[lv, idx[:, c], 0]).astype(np.float32)
                f1 = (f1 + w[:, c] * tab[lv, idx[:, c], 1]).astype(np.float32)
        else:
            w64 = w.astype(np.float64)
            f0 = (w64 * tab[lv][idx][..., 0].astype(np.float64)).sum(1)
            f1 = (w64 * tab[lv][idx][..., 1].astype(np.float64)).sum(1)
        X[:, 2 * lv] = f0
        X[:, 2 * lv + 1] = f1
    X[:, 32:34] = inputs[:, 4:6]
    X[:, 34:36] = inputs[:, 6:8]
    X[:, 36] = 1.0
    return bf16(X).astype(np.float64) if bf16_round else X


def forward(grid, weights, table, inputs, bf16_round=True):
    """Returns (y (n, 3), cache) for backward."""
    W = np.asarray(weights, np.float64).reshape(LAYERS, WIDTH, WIDTH).copy()
    W[LAYERS - 1, OUT:] = 0.0
    if bf16_round:
        W = bf16(W).astype(np.float64)
    H = [encode(grid, table, inputs, bf16_round)]
    for lv in range(LAYERS - 1):
        Z = H[-1] @ W[lv].T
        Hn = np.maximum(Z, 0.0)
        H.append(bf16(Hn).astype(np.float64) if bf16_round else Hn)
    Y = H[-1] @ W[LAYERS - 1].T
    return Y[:, :OUT], {"W": W, "H": H, "inputs": np.asarray(inputs, np.float32)}


def loss_and_grad(y, target, norm=None):
    """Mean relative L2 loss over samples and channels; dL/dy with the
    denominator held constant."""
    y = np.asarray(y, np.float64)
    t = np.asarray(target, np.float64)
    den = y * y + 0.01
    diff = y - t
    n = y.shape[0]
    norm = 3.0 * n if norm is None else norm
    loss = float((diff * diff / den).sum() / norm)
    dy = 2.0 * diff / den / norm
    return loss, dy


def backward(grid, table_shape, cache, dy, bf16_round=True):
    """Gradients of the loss w.r.t. the f32 weights (5, 64, 64) and the table
    (levels, T, 2)."""
    W, H = cache["W"], cache["H"]
    n = dy.shape[0]
    G = np.zeros((n, WIDTH))
    G[:, :OUT] = dy
    if bf16_round:
        G = bf16(G).astype(np.float64)
    dW = np.zeros((LAYERS, WIDTH, WIDTH))
    for lv in range(LAYERS - 1, -1, -1):
        dW[lv] = G.T @ H[lv]
        dH = G @ W[lv]
        if lv > 0:
            G = dH * (H[lv] > 0)
            if bf16_round:
                G = bf16(G).astype(np.float64)
        else:
            dX = dH
    dW[LAYERS - 1, OUT:] = 0.0
    dT = np.zeros(table_shape)
    pos = cache["inputs"][:, 0:3]
    for lv in range(LEVELS):
        idx, w = level_corners(grid, lv, pos)
        for f in range(2):
            contrib = w.astype(np.float64) * dX[:, 2 * lv + f][:, None]
            np.add.at(dT[lv, :, f], idx.reshape(-1), contrib.reshape(-1))
    return dW, dT


def adam(p, m, v, g, step, lr=1e-2, b1=0.9, b2=0.99, eps=1e-8):
    """One Adam step in float32 (in place on copies); returns (p, m, v)."""
    p = np.asarray(p, np.float32).copy()
    m = np.float32(b1) * np.asarray(m, np.float32) + np.float32(1 - b1) * np.asarray(g, np.float32)
    v = np.float32(b2) * np.asarray(v, np.float32) + np.float32(1 - b2) * np.asarray(g, np.float32) ** 2
    bc1 = np.float32(1 - b1 ** step)
    bc2 = np.float32(1 - b2 ** step)
    p -= np.float32(lr) * (m / bc1) / (np.sqrt(v / bc2) + np.float32(eps))
    return p, m, v


def init_params(log2_table, seed=0, table_scale=1e-4):
    rng = np.random.default_rng(seed)
    W = np.zeros((LAYERS, WIDTH, WIDTH), np.float32)
    lim = math.sqrt(6.0 / WIDTH)
    for lv in range(LAYERS):
        rows = WIDTH if lv < LAYERS - 1 else OUT
        W[lv, :rows] = rng.uniform(-lim, lim, (rows, WIDTH)) * (1.0 if lv < LAYERS - 1 else 0.1)
    T = 1 << log2_table
    table = rng.uniform(-table_scale, table_scale, (LEVELS, T, 2)).astype(np.float32)
    return W, table
