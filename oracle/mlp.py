"""CPU restatement of the return-map surrogate MLP (7 -> 64 -> 64 -> 3, SiLU) -- test infrastructure.

The checker for the device kernels in ``baking_b200/csrc/bk_mlp.cu``: the forward pass with the
tensor-core rounding (inputs as two BF16 terms, BF16 weights and hidden activations; FP32
accumulation and biases),
the gradient of the mean-squared loss through that forward (rounding treated as identity), one
Adam step and the packed operand layout. The reference has no learned component, so there is no
reference call site to pin this against: it is pinned by float64 finite differences of its own
loss (tests/test_mlp_oracle.py).
"""
from __future__ import annotations

import numpy as np

FEATURES, HIDDEN, OUTPUTS = 7, 64, 3
P_W1 = 0
P_B1 = P_W1 + FEATURES * HIDDEN
P_W2 = P_B1 + HIDDEN
P_B2 = P_W2 + HIDDEN * HIDDEN
P_W3 = P_B2 + HIDDEN
P_B3 = P_W3 + HIDDEN * OUTPUTS
PARAMS = P_B3 + OUTPUTS
PACKED_BYTES = 12864


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    rounded = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return rounded.astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(params):
    p = np.asarray(params)
    if p.dtype != np.float64:
        p = p.astype(np.float32)
    return (p[P_W1:P_B1].reshape(FEATURES, HIDDEN), p[P_B1:P_W2], p[P_W2:P_B2].reshape(HIDDEN, HIDDEN),
            p[P_B2:P_W3], p[P_W3:P_B3].reshape(HIDDEN, OUTPUTS), p[P_B3:PARAMS])


def init_params(seed=0):
    """He-style initialisation for SiLU layers, zero biases."""
    rng = np.random.default_rng(seed)
    p = np.zeros(PARAMS, np.float32)
    p[P_W1:P_B1] = (rng.standard_normal(FEATURES * HIDDEN) * np.sqrt(2.0 / FEATURES)).astype(np.float32)
    p[P_W2:P_B2] = (rng.standard_normal(HIDDEN * HIDDEN) * np.sqrt(2.0 / HIDDEN)).astype(np.float32)
    p[P_W3:P_B3] = (rng.standard_normal(HIDDEN * OUTPUTS) * np.sqrt(1.0 / HIDDEN)).astype(np.float32)
    return p


def _silu(z):
    return z / (1.0 + np.exp(-z))


def normalise(features, in_mean, in_scale):
    f = np.asarray(features, np.float32)[:, :FEATURES]
    return ((f - np.asarray(in_mean, np.float32)[:FEATURES]) / np.asarray(in_scale, np.float32)[:FEATURES]).astype(np.float32)


def two_term(x):
    """The layer-1 input as the tensor cores see it: bf16(x) + bf16(x - bf16(x)) (the inputs and
    their BF16 remainders share the first layer's weights)."""
    x = np.asarray(x, np.float32)
    hi = bf16(x)
    return hi.astype(np.float64) + bf16((x - hi).astype(np.float32)).astype(np.float64)


def forward(params, x, keep=False, exact=False):
    """Network outputs (in units of out_scale) for normalised inputs x[n, 7]. ``exact`` skips the
    BF16 rounding (float64 throughout), for checking the gradient formulas by finite differences."""
    W1, b1, W2, b2, W3, b3 = unpack(params)
    r = (lambda a: np.asarray(a, np.float64)) if exact else (lambda a: bf16(np.asarray(a, np.float32)).astype(np.float64))
    xb = np.asarray(x, np.float64) if exact else two_term(x)
    z1 = xb @ r(W1) + b1
    h1 = r(_silu(z1))
    z2 = h1 @ r(W2) + b2
    h2 = r(_silu(z2))
    y = h2 @ r(W3) + b3
    if keep:
        return y, (xb, z1, h1, z2, h2)
    return y


def loss_and_gradient(params, x, target, exact=False):
    """Mean over samples and outputs of (y - target)^2 (target in units of out_scale), its gradient
    (the BF16 rounding of the forward is treated as the identity)."""
    W1, b1, W2, b2, W3, b3 = unpack(params)
    r = (lambda a: np.asarray(a, np.float64)) if exact else (lambda a: bf16(np.asarray(a, np.float32)).astype(np.float64))
    y, (xb, z1, h1, z2, h2) = forward(params, x, keep=True, exact=exact)
    n = x.shape[0]
    d = y - target
    loss = float((d * d).sum() / (n * OUTPUTS))
    dy = 2.0 * d / (n * OUTPUTS)

    def dsilu(z):
        s = 1.0 / (1.0 + np.exp(-z))
        return s * (1.0 + z * (1.0 - s))

    g = np.zeros(PARAMS, np.float64)
    g[P_W3:P_B3] = (h2.T @ dy).ravel()
    g[P_B3:PARAMS] = dy.sum(0)
    dz2 = (dy @ r(W3).T) * dsilu(z2)
    g[P_W2:P_B2] = (h1.T @ dz2).ravel()
    g[P_B2:P_W3] = dz2.sum(0)
    dz1 = (dz2 @ r(W2).T) * dsilu(z1)
    g[P_W1:P_B1] = (xb.T @ dz1).ravel()
    g[P_B1:P_W2] = dz1.sum(0)
    return loss, g


def adam(params, grads, m, v, step, lr, beta1=0.9, beta2=0.999, eps=1e-8):
    m = beta1 * m + (1 - beta1) * grads
    v = beta2 * v + (1 - beta2) * grads * grads
    c1, c2 = 1 - beta1 ** step, 1 - beta2 ** step
    return params - lr * (m / c1) / (np.sqrt(v / c2) + eps), m, v


def operand_offset(row, k, K):
    return (row // 8) * (K * 16) + (k // 8) * 128 + (row % 8) * 16 + (k % 8) * 2


def pack(params):
    """Bytes of the packed operands (see include/baking_b200.h, bk_mlp_pack)."""
    W1, b1, W2, b2, W3, b3 = unpack(params)
    blob = np.zeros(PACKED_BYTES, np.uint8)
    half = lambda x: (bf16(np.float32(x)).view(np.uint32) >> 16).astype(np.uint16)  # noqa: E731

    def put(off, value):
        blob[off:off + 2] = np.frombuffer(half(value).tobytes(), np.uint8)

    for n in range(HIDDEN):
        for k in range(16):
            f = k if k < FEATURES else (k - 8 if 8 <= k < 8 + FEATURES else -1)
            put(operand_offset(n, k, 16), W1[f, n] if f >= 0 else 0.0)
        for k in range(HIDDEN):
            put(2048 + operand_offset(n, k, HIDDEN), W2[k, n])
    for n in range(16):
        for k in range(HIDDEN):
            put(10240 + operand_offset(n, k, HIDDEN), W3[k, n] if n < OUTPUTS else 0.0)
    biases = np.zeros(144, np.float32)
    biases[:64], biases[64:128], biases[128:131] = b1, b2, b3
    blob[12288:] = np.frombuffer(biases.tobytes(), np.uint8)
    return blob
