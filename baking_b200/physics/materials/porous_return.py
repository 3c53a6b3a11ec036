"""End-state porosity consistency solve (the reference's ``physics/materials/porous_return.py:11-100``).

The solve runs inside the return-map kernel; these wrappers evaluate the same
device functions on arrays of inputs (the reference's tests call them from a
one-thread Warp kernel).
"""

from __future__ import annotations

import math

import torch

from ... import _lib


def pressure_coefficient64(porosity):
    """a(n) in float64 (host helper)."""
    return 0.0 if porosity <= 0 else 9.0 / (4.0 * math.log(1.0 / porosity) ** 2 * (3.5 * porosity + 1.0))


def SolvePorosity(q_value, p_value, dev_factor, mean_scale, exponent, plastic_volume, initial_porosity):
    """Vectorised ``solve_porosity`` on the device; returns (porosity float32, prediction float64)."""
    dev = _lib.require_cuda()
    cols = [torch.as_tensor(v, dtype=torch.float32, device=dev).reshape(-1).contiguous()
            for v in (q_value, p_value, dev_factor, mean_scale, exponent)]
    vp = torch.as_tensor(plastic_volume, dtype=torch.float64, device=dev).reshape(-1).contiguous()
    n = vp.shape[0]
    out = torch.empty(n, dtype=torch.float32, device=dev)
    pred = torch.empty(n, dtype=torch.float64, device=dev)
    _lib.call("bk_solve_porosity", n, *[c.data_ptr() for c in cols], vp.data_ptr(), initial_porosity,
              out.data_ptr(), pred.data_ptr(), _lib.stream_handle())
    return out, pred


def PorosityCoefficients(porosities):
    dev = _lib.require_cuda()
    por = torch.as_tensor(porosities, dtype=torch.float32, device=dev).reshape(-1).contiguous()
    out = torch.empty_like(por)
    _lib.call("bk_porosity_coefficient", por.shape[0], por.data_ptr(), out.data_ptr(), _lib.stream_handle())
    return out
