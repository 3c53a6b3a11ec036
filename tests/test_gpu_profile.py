"""The library's per-kernel CUDA-event timing (KernelTimer over bk_profile_*) that bench.py's
roofline uses: every kernel of the fused substep, or only the selected one."""
import pytest

pytestmark = pytest.mark.gpu


def test_kernel_timer_all_and_selected():
    from baking_b200 import _lib
    from tests.scenes import build_transport
    sim = build_transport("cuda", gas=True)
    sim.scatter_ahead = True
    sim.AdvanceUnchecked(1)
    every = _lib.KernelTimer()
    with every:
        sim.AdvanceUnchecked(2)
    names = every.summary()
    for kernel in ("p2g", "g2p_return", "diffuse", "grid_update"):
        assert names[kernel]["count"] == 2 and names[kernel]["mean_s"] > 0.0, kernel
    # the second substep of the call finds its transport fields scattered ahead by the first
    assert names["transport_scatter"]["count"] == 1
    only = _lib.KernelTimer(only="g2p_return")
    with only:
        sim.AdvanceUnchecked(3)
    selected = only.summary()
    assert set(selected) == {"g2p_return"} and selected["g2p_return"]["count"] == 3
    again = _lib.KernelTimer()  # the selection ends with its timer
    with again:
        sim.AdvanceUnchecked(1)
    assert "p2g" in again.summary()
