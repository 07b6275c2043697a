"""The preconditioner's CPU oracle: its hand-written backward equals torch
autograd of the FP32 network, and its BF16 rounding stays close to FP32."""
import numpy as np
import pytest

from oracle.precond_oracle import NetOracle, autograd_reference, layer_table
from tests.conftest import rel_l2


def seeded_params(widths=(16, 32, 64, 64), seed=0):
    layers, n = layer_table(widths)
    rng = np.random.default_rng(seed)
    p = np.zeros(n, np.float32)
    for ci, co, wo, bo in layers[:-1]:
        lim = np.sqrt(6.0 / (9 * ci))
        p[wo:wo + co * 9 * ci] = rng.uniform(-lim, lim, co * 9 * ci)
        p[bo:bo + co] = rng.uniform(-0.05, 0.05, co)
    ci, _, wo, bo = layers[-1]
    p[wo:wo + ci] = rng.uniform(-0.25, 0.25, ci)
    p[bo] = 0.01
    return p


def test_layer_table_counts():
    layers, n = layer_table()
    assert len(layers) == 15
    # 3x3 convs: 16->16->16, 16->32->32, 32->64->64, 64->64->64,
    # 128->64->64, 96->32->32, 48->16->16; 1x1 16->1
    convs = sum(co * 9 * ci + co for ci, co, _, _ in layers[:-1])
    assert n == convs + 17
    assert 290_000 < n < 320_000


@pytest.mark.parametrize("N,H,W", [(1, 16, 24), (2, 8, 16)])
def test_backward_matches_autograd_fp32(N, H, W):
    rng = np.random.default_rng(1)
    p = seeded_params()
    x = rng.standard_normal((N, H, W, 3)).astype(np.float32)
    t = rng.standard_normal((N, H, W)).astype(np.float32)
    o = NetOracle(p, bf16=False)
    y = o.forward(x)
    loss, g = o.backward(t)
    loss_ref, y_ref, g_ref = autograd_reference(p, x, t)
    assert rel_l2(y, y_ref) < 1e-5
    assert abs(loss - loss_ref) <= 1e-5 * abs(loss_ref)
    assert rel_l2(g, g_ref) < 1e-4
    for ci, co, wo, bo in layer_table()[0]:
        assert rel_l2(g[wo:bo], g_ref[wo:bo]) < 1e-3


def test_bf16_rounding_close_to_fp32():
    rng = np.random.default_rng(2)
    p = seeded_params()
    x = rng.standard_normal((1, 16, 16, 3)).astype(np.float32)
    t = rng.standard_normal((1, 16, 16)).astype(np.float32)
    a = NetOracle(p, bf16=True)
    b = NetOracle(p, bf16=False)
    ya, yb = a.forward(x), b.forward(x)
    assert 1e-5 < rel_l2(ya, yb) < 5e-2
    _, ga = a.backward(t)
    _, gb = b.backward(t)
    # BF16 activations and gradients through 14 layers: a few percent
    assert rel_l2(ga, gb) < 0.15
