"""Settling (rest) diagnostics (the reference's ``physics/quasistatic.py:11-21``).

Max particle speed, max norm of sym(C), and max relative plastic-gradient rate,
max-reduced on the device into a 3-float array.
"""

from __future__ import annotations

from .. import _lib, arrays


def SettlingMetrics(velocities, affine, old_plastic, new_plastic, metrics, time_step):
    n = velocities.shape[0]
    pitch = arrays.common_pitch(velocities, affine, old_plastic, new_plastic)
    _lib.call("bk_settling_metrics", n, pitch, arrays.ptr(velocities), arrays.ptr(affine), arrays.ptr(old_plastic),
              arrays.ptr(new_plastic), metrics.data_ptr(), time_step, _lib.stream_handle())
