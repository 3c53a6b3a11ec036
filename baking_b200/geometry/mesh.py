"""Tetrahedral meshes: validation, the built-in cube and sphere meshes, NPZ/meshio loading.

Host-side set-up that runs once per scene. It reproduces the behaviour of the
reference's ``geometry/mesh_validation.py:18-47`` (``TetMesh``,
``ComputeSignedVolumes``, ``ValidateTetMesh``) and ``geometry/mesh_loader.py:6-79``
(``LoadTetMesh``, ``CreateDemoMesh``, ``CreateSphereMesh``): same checks and
messages, positively oriented tets, the 0.3 m demo cube at (0.35, 0.45, 0.35).
"""

from __future__ import annotations

from dataclasses import dataclass
from itertools import permutations
from pathlib import Path

import numpy as np


@dataclass(frozen=True)
class TetMesh:
    vertex_positions: np.ndarray  # (V, 3) float64
    tet_indices: np.ndarray       # (T, 4) int32, positively oriented
    reference_volumes: np.ndarray  # (T,) float64, |signed volume|


def ComputeSignedVolumes(vertex_positions, tet_indices):
    corners = np.asarray(vertex_positions)[np.asarray(tet_indices)]
    edges = corners[:, 1:] - corners[:, :1]
    return np.linalg.det(edges) / 6.0


def ValidateTetMesh(vertex_positions, tet_indices):
    """Check a tet mesh and return it with every tet positively oriented."""
    vertices = np.asarray(vertex_positions, dtype=np.float64)
    raw = np.asarray(tet_indices)
    if vertices.ndim != 2 or vertices.shape[1] != 3:
        raise ValueError("vertices must have shape (vertex_count, 3)")
    if raw.ndim != 2 or raw.shape[1] != 4 or len(raw) == 0:
        raise ValueError("tetrahedra must have nonempty shape (tet_count, 4)")
    if not np.issubdtype(raw.dtype, np.integer):
        raise ValueError("tetrahedron indices must be integers (zero based)")
    if len(vertices) < 4 or not np.isfinite(vertices).all():
        raise ValueError("vertices must be finite and contain at least four entries")
    if raw.min() < 0 or raw.max() >= len(vertices):
        raise ValueError("tetrahedron index outside vertex array")
    tets = raw.astype(np.int32, copy=True)
    ordered = np.sort(tets, axis=1)
    if np.any(ordered[:, 1:] == ordered[:, :-1]):
        raise ValueError("tetrahedron contains repeated vertex indices")
    if len(np.unique(ordered, axis=0)) != len(tets):
        raise ValueError("duplicate tetrahedra detected")
    volumes = ComputeSignedVolumes(vertices, tets)
    corners = vertices[tets]
    longest_edge = np.linalg.norm(corners[:, :, None] - corners[:, None, :], axis=-1).max(axis=(1, 2))
    if np.any(np.abs(volumes) <= 1.0e-12 * longest_edge ** 3):
        raise ValueError("zero-volume or nearly degenerate tetrahedron detected")
    flip = volumes < 0.0
    tets[flip, 0], tets[flip, 1] = tets[flip, 1].copy(), tets[flip, 0].copy()
    return TetMesh(vertices.copy(), tets, np.abs(volumes))


def _kuhn_tets():
    """Six tets of the unit cube sharing the (0,0,0)-(1,1,1) diagonal.

    Each tet follows one monotone lattice path from corner 0 to corner 7, one
    per ordering of the three axes; corner index = x + 2y + 4z.
    """
    tets = []
    for order in permutations(range(3)):
        corner, path = 0, [0]
        for axis in order:
            corner += 1 << axis
            path.append(corner)
        tets.append(path)
    return np.asarray(tets, dtype=np.int64)


def VoxelTetMesh(occupied, origin, voxel_size):
    """Tet mesh of the occupied voxels of a boolean (nx, ny, nz) array, six tets per voxel.

    Vertices are the voxel corners that some occupied voxel uses, numbered in
    x-major lattice order; tets are listed voxel by voxel in x-major order.
    """
    occupied = np.asarray(occupied, dtype=bool)
    shape = np.array(occupied.shape)
    lattice = tuple(shape + 1)
    voxels = np.argwhere(occupied)
    if len(voxels) == 0:
        raise ValueError("no occupied voxels")
    corner_offsets = np.array([[(c >> 0) & 1, (c >> 1) & 1, (c >> 2) & 1] for c in range(8)])
    corners = voxels[:, None, :] + corner_offsets[None, :, :]           # (n, 8, 3)
    corner_ids = np.ravel_multi_index(corners.reshape(-1, 3).T, lattice).reshape(-1, 8)
    tet_ids = corner_ids[:, _kuhn_tets()].reshape(-1, 4)
    used, compact = np.unique(tet_ids, return_inverse=True)
    coords = np.stack(np.unravel_index(used, lattice), axis=1).astype(np.float64)
    vertices = np.asarray(origin, dtype=np.float64) + coords * voxel_size
    return ValidateTetMesh(vertices, compact.reshape(-1, 4))


def CreateDemoMesh(subdivision_count=6):
    """A 0.3 m cube whose lower corner is at (0.35, 0.45, 0.35); six tets per voxel."""
    if subdivision_count < 1:
        raise ValueError("subdivision_count must be positive")
    s = int(subdivision_count)
    return VoxelTetMesh(np.ones((s, s, s), dtype=bool), (0.35, 0.45, 0.35), 0.3 / s)


def CreateSphereMesh(radius=0.1, subdivision_count=12):
    """Structured cube mesh mapped onto a ball of ``radius`` centred at the origin.

    Uses the volume-filling cube-to-ball map
    x' = x sqrt(1 - y^2/2 - z^2/2 + y^2 z^2/3) (and cyclic), which puts the
    cube's boundary vertices exactly on the sphere and keeps the connectivity.
    """
    cube = CreateDemoMesh(subdivision_count)
    low = cube.vertex_positions.min(axis=0)
    extent = cube.vertex_positions.max(axis=0) - low
    unit = 2.0 * (cube.vertex_positions - low) / extent - 1.0
    sq = unit ** 2
    mapped = np.empty_like(unit)
    for axis in range(3):
        a, b = sq[:, (axis + 1) % 3], sq[:, (axis + 2) % 3]
        mapped[:, axis] = radius * unit[:, axis] * np.sqrt(1.0 - a / 2.0 - b / 2.0 + a * b / 3.0)
    return ValidateTetMesh(mapped, cube.tet_indices)


def LoadTetMesh(mesh_path, mesh_scale=1.0, mesh_translation=(0.0, 0.0, 0.0)):
    """Read an NPZ (``vertices``, ``tetrahedra``) or, when meshio is installed, a meshio format."""
    mesh_path = Path(mesh_path)
    if not np.isfinite(mesh_scale) or mesh_scale <= 0.0:
        raise ValueError("mesh_scale must be positive and finite")
    translation = np.asarray(mesh_translation, dtype=np.float64)
    if translation.shape != (3,) or not np.isfinite(translation).all():
        raise ValueError("mesh_translation must contain three finite values")
    if mesh_path.suffix.lower() == ".npz":
        with np.load(mesh_path, allow_pickle=False) as data:
            vertices, tets = data["vertices"], data["tetrahedra"]
    else:
        import meshio  # optional dependency, as in the reference
        mesh = meshio.read(mesh_path)
        if any(block.type.startswith("tetra") and block.type != "tetra" for block in mesh.cells):
            raise ValueError("higher-order tetrahedra are unsupported; export linear tetrahedra")
        blocks = [block.data for block in mesh.cells if block.type == "tetra"]
        if not blocks:
            raise ValueError("input contains no linear tetrahedra")
        tets, vertices = np.concatenate(blocks), mesh.points
    vertices = np.asarray(vertices, dtype=np.float64) * mesh_scale + translation
    return ValidateTetMesh(vertices, tets)
