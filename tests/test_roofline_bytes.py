"""Algorithmic byte counts of the fused substep kernels (baking_b200/roofline.py) that bench.py's
roofline fractions divide by: the G2P + return kernel with and without the next substep's
transport scatter, and the P2G kernel per mode. Host arithmetic only."""
from types import SimpleNamespace

from baking_b200 import roofline


def engine(transport=True, gas=True, ding=True, n=1000, prescatter=True):
    return SimpleNamespace(n=n, transport=transport, gas=gas, is_ding=ding,
                           prescatter_allowed=lambda: prescatter and transport)


def test_g2p_return_bytes_follow_the_scatter_ahead():
    e = engine()
    plain = roofline.fused_bytes("g2p_return", e, 10)
    ahead = roofline.fused_bytes("g2p_return", e, 10, scatter_ahead=True)
    # x F read, x v C F written, Ding Fe n gel T read and Fe tau n gel written: 276 B per particle
    assert plain == 276 * 1000 + 16 * 10
    # the scatter ahead adds V0, capacity and water per particle and four node fields
    assert ahead == 296 * 1000 + 48 * 10
    # an engine that cannot scatter ahead (no transport, or a surrogate) counts the plain form
    assert roofline.fused_bytes("g2p_return", engine(prescatter=False), 10, scatter_ahead=True) == plain


def test_p2g_and_transport_scatter_bytes():
    e = engine()
    assert roofline.fused_bytes("p2g", e, 10) == 200 * 1000 + 32 * 10
    assert roofline.fused_bytes("transport_scatter", e, 10) == 76 * 1000 + 32 * 10
    elastic = engine(transport=False, gas=False, ding=False)
    # x v C F V0 read, mass read; node (p, m) written
    assert roofline.fused_bytes("p2g", elastic, 10) == 104 * 1000 + 16 * 10
