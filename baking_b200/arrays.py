"""Device arrays in the structure-of-arrays layout the kernels read.

A per-particle vec3 is stored as 3 planes and a mat33 as 9 planes (row-major
component order), each plane ``pitch`` elements long, with ``pitch`` a multiple
of 64 so every plane starts 256-byte aligned. Callers see ordinary torch views
of shape (n, 3) and (n, 3, 3) -- the shapes of the reference's ``wp.vec3`` and
``wp.mat33`` arrays -- whose strides walk the planes; ``.cpu().numpy()`` on a
view gives the reference's array-of-structures values.
"""

from __future__ import annotations

import numpy as np
import torch

ALIGN = 64

_TORCH = {"f4": torch.float32, "f8": torch.float64, "i4": torch.int32}


def pitch_for(n):
    return max(ALIGN, (int(n) + ALIGN - 1) // ALIGN * ALIGN)


def _planes(components, n, dtype, device, pitch=None):
    pitch = pitch_for(n) if pitch is None else pitch
    storage = torch.zeros(components, pitch, dtype=dtype, device=device)
    return storage, pitch


def scalars(n, dtype=torch.float32, device="cuda", pitch=None, fill=0):
    storage, _ = _planes(1, n, dtype, device, pitch)
    if fill:
        storage.fill_(fill)
    return storage[0, :n]


def vec3s(n, dtype=torch.float32, device="cuda", pitch=None):
    storage, _ = _planes(3, n, dtype, device, pitch)
    return storage.t()[:n]


def mat33s(n, dtype=torch.float32, device="cuda", pitch=None):
    storage, pitch = _planes(9, n, dtype, device, pitch)
    if n > 0:
        return storage.t()[:n].view(n, 3, 3)
    return storage.as_strided((0, 3, 3), (1, 3 * pitch, pitch))  # empty, with the plane strides


def layout_pitch(t):
    """Plane pitch of a tensor made by this module (or of any equivalent strided view)."""
    if t.dim() == 1:
        return None  # scalars fit any pitch
    if t.dim() == 2:
        if t.stride(0) != 1 and t.shape[0] > 1:
            raise ValueError("vec3 array is not in plane layout")
        return t.stride(1)
    if t.dim() == 3:
        if (t.stride(0) != 1 and t.shape[0] > 1) or t.stride(1) != 3 * t.stride(2):
            raise ValueError("mat33 array is not in plane layout")
        return t.stride(2)
    raise ValueError("unsupported array rank")


def like(t, n=None):
    """New zeroed array with the layout, dtype and device of ``t``."""
    n = t.shape[0] if n is None else n
    pitch = layout_pitch(t)
    if t.dim() == 1:
        return scalars(n, t.dtype, t.device)
    if t.dim() == 2:
        return vec3s(n, t.dtype, t.device, pitch if n == t.shape[0] else None)
    return mat33s(n, t.dtype, t.device, pitch if n == t.shape[0] else None)


def from_numpy(values, kind, device="cuda", pitch=None):
    """Upload numpy values; (n,), (n, 3) and (n, 3, 3) shapes map to scalars, vec3 and mat33 planes."""
    a = np.asarray(values)
    dtype = _TORCH[kind]
    n = a.shape[0]
    if a.ndim == 1:
        out = scalars(n, dtype, device, pitch)
    elif a.ndim == 2 and a.shape[1] == 3:
        out = vec3s(n, dtype, device, pitch)
    elif a.ndim == 3 and a.shape[1:] == (3, 3):
        out = mat33s(n, dtype, device, pitch)
    else:
        raise ValueError(f"unsupported shape {a.shape}")
    out.copy_(torch.as_tensor(np.ascontiguousarray(a)).to(dtype))
    return out


def to_numpy(t):
    return t.detach().cpu().numpy()


def assign(t, values):
    """In-place upload of numpy values into a device array (the reference's ``array.assign``)."""
    t.copy_(torch.as_tensor(np.asarray(values)).to(t.dtype).reshape(t.shape))
    return t


def ptr(t):
    """Device pointer of a plane-layout array (its first plane)."""
    return t.data_ptr() if t is not None else None


def common_pitch(*arrays):
    """The single pitch shared by the given plane-layout arrays (scalars accept any)."""
    pitch = None
    n = None
    for t in arrays:
        if t is None:
            continue
        n = t.shape[0] if n is None else n
        p = layout_pitch(t)
        if p is None:
            continue
        if pitch is None:
            pitch = p
        elif p != pitch:
            raise ValueError("particle arrays of one call must share a plane pitch")
    return pitch if pitch is not None else max(n or 1, 1)
