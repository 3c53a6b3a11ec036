"""The surrogate MLP's CPU oracle (oracle/mlp.py): its gradient formulas against float64 central
differences, its BF16 rounding against the definition, and its packed layout against the header."""
import re
from pathlib import Path

import numpy as np

from oracle import mlp

ROOT = Path(__file__).resolve().parents[1]


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    params = mlp.init_params(1).astype(np.float64)
    params[mlp.P_B1:mlp.P_W2] = 0.1 * rng.standard_normal(64)
    x = rng.standard_normal((32, 7))
    target = rng.standard_normal((32, 3))
    _, g = mlp.loss_and_gradient(params, x, target, exact=True)
    for k in rng.choice(mlp.PARAMS, 60, replace=False):
        h = 1e-6
        p1, p2 = params.copy(), params.copy()
        p1[k] += h
        p2[k] -= h
        l1, _ = mlp.loss_and_gradient(p1, x, target, exact=True)
        l2, _ = mlp.loss_and_gradient(p2, x, target, exact=True)
        np.testing.assert_allclose(g[k], (l1 - l2) / (2 * h), rtol=1e-5, atol=1e-10)


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 3.14159265], np.float32)
    r = mlp.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == 1.0
    np.testing.assert_allclose(r[4:], [-2.5, 3.140625])
    bits = r.view(np.uint32)
    assert np.all(bits & 0xFFFF == 0)


def test_layout_constants_match_header():
    text = (ROOT / "include" / "baking_b200.h").read_text()
    assert int(re.search(r"#define BK_MLP_PARAMS (\d+)", text).group(1)) == mlp.PARAMS
    assert int(re.search(r"#define BK_MLP_PACKED_BYTES (\d+)", text).group(1)) == mlp.PACKED_BYTES
    blob = mlp.pack(mlp.init_params(0))
    assert blob.size == mlp.PACKED_BYTES
    # every core-matrix slot of W2^T is used exactly once
    offs = {mlp.operand_offset(n, k, 64) for n in range(64) for k in range(64)}
    assert len(offs) == 64 * 64 and max(offs) == 64 * 64 * 2 - 2
