"""Particle samples inside a tet mesh, and the host-side index tables built from them.

* ``SampleParticles`` follows ``geometry/particle_sampling.py:13-53`` of the
  reference: four points per tet from the symmetric degree-2 quadrature rule
  (barycentric weights (5+3*sqrt5)/20 and (5-sqrt5)/20), the centroid for one
  point, otherwise seeded Dirichlet(1,1,1,1) points drawn tet by tet.
* ``BoundaryFaces`` follows ``physics/thermal_water.py:51-74``: faces used by
  exactly one tet, wound so the normal points out of the tet, owned by the
  particle of that tet closest to the face centre.
* ``MeshBindingTables`` follows ``geometry/mesh_tracking.py:42-75``: the CSR
  vertex -> (particle, weight, reference offset) table used to rebuild mesh
  vertices from particle positions and deformation gradients.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class ParticleSamples:
    particle_positions: np.ndarray  # (N, 3) float64
    reference_volumes: np.ndarray   # (N,) float64
    particle_masses: np.ndarray     # (N,) float64
    source_tets: np.ndarray         # (N,) int


def _symmetric_rule():
    off = (5.0 - np.sqrt(5.0)) / 20.0
    weights = np.full((4, 4), off)
    np.fill_diagonal(weights, (5.0 + 3.0 * np.sqrt(5.0)) / 20.0)
    return weights


def SampleParticles(tet_mesh, density, particles_per_tet=0, target_volume=None,
                    random_seed=42, max_particles=500000):
    if not np.isfinite(density) or density <= 0.0:
        raise ValueError("density must be positive and finite")
    if particles_per_tet < 0:
        raise ValueError("particles_per_tet must be nonnegative")
    tet_count = len(tet_mesh.tet_indices)
    if particles_per_tet == 0:
        if target_volume is None or not np.isfinite(target_volume) or target_volume <= 0.0:
            raise ValueError("automatic sampling needs a positive target_volume")
        wanted = np.maximum(4.0, np.ceil(tet_mesh.reference_volumes / target_volume))
        if wanted.sum() > max_particles:
            raise ValueError("sampling exceeds max_particles; coarsen the input mesh or sampling")
        counts = wanted.astype(np.int64)
    else:
        counts = np.full(tet_count, particles_per_tet, dtype=np.int64)
    if counts.sum() > max_particles:
        raise ValueError("sampling exceeds max_particles")
    source_tets = np.repeat(np.arange(tet_count), counts)
    volumes = np.repeat(tet_mesh.reference_volumes / counts, counts)
    corners = tet_mesh.vertex_positions[tet_mesh.tet_indices]  # (T, 4, 3)
    positions = np.empty((len(source_tets), 3), dtype=np.float64)
    rng = np.random.default_rng(random_seed)
    symmetric = _symmetric_rule()
    start = 0
    for tet, count in enumerate(counts):
        if count == 4:
            bary = symmetric
        elif count == 1:
            bary = np.full((1, 4), 0.25)
        else:
            bary = rng.dirichlet(np.ones(4), size=count)
        positions[start:start + count] = bary @ corners[tet]
        start += count
    return ParticleSamples(positions, volumes, density * volumes, source_tets)


def _tet_particle_lists(source_tets, tet_count):
    order = np.argsort(source_tets, kind="stable")
    starts = np.concatenate(([0], np.cumsum(np.bincount(source_tets, minlength=tet_count))))
    return order, starts


def BoundaryFaces(tet_mesh, samples):
    """Outward-wound boundary triangles (F, 3) int32 and their owner particles (F,) int32."""
    tets = np.asarray(tet_mesh.tet_indices, dtype=np.int64)
    vertices = tet_mesh.vertex_positions
    tet_count = len(tets)
    # Face k of a tet omits local vertex k; faces are enumerated tet-major.
    keep = np.array([[1, 2, 3], [0, 2, 3], [0, 1, 3], [0, 1, 2]])
    faces = tets[:, keep].reshape(-1, 3)
    opposite = tets.reshape(-1)
    owner_tet = np.repeat(np.arange(tet_count), 4)
    keys = np.sort(faces, axis=1)
    _, inverse, counts = np.unique(keys, axis=0, return_inverse=True, return_counts=True)
    boundary = np.flatnonzero(counts[inverse.reshape(-1)] == 1)
    faces = faces[boundary].copy()
    opposite = opposite[boundary]
    owner_tet = owner_tet[boundary]
    p = vertices[faces]
    normal = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
    inward = np.einsum("ij,ij->i", normal, vertices[opposite] - p[:, 0]) > 0
    faces[inward, 1], faces[inward, 2] = faces[inward, 2].copy(), faces[inward, 1].copy()
    order, starts = _tet_particle_lists(np.asarray(samples.source_tets), tet_count)
    centres = vertices[faces].mean(axis=1)
    owners = np.empty(len(faces), dtype=np.int64)
    for f, tet in enumerate(owner_tet):
        members = order[starts[tet]:starts[tet + 1]]
        if len(members) == 0:
            raise ValueError("every tetrahedron must contain particles for mesh reconstruction")
        distance = np.linalg.norm(samples.particle_positions[members] - centres[f], axis=1)
        owners[f] = members[np.argmin(distance)]
    return faces.astype(np.int32), owners.astype(np.int32)


@dataclass(frozen=True)
class MeshBindingTables:
    binding_offsets: np.ndarray    # (V+1,) int32
    binding_particles: np.ndarray  # (B,) int32
    binding_weights: np.ndarray    # (B,) float64, reference-volume weights, sum 1 per vertex
    reference_offsets: np.ndarray  # (B, 3) float64, X_vertex - X_particle
    unmapped_vertex_count: int


def MeshBindingTables_build(tet_mesh, samples):
    vertex_count = len(tet_mesh.vertex_positions)
    particle_count = len(samples.particle_positions)
    source_tets = np.asarray(samples.source_tets)
    volumes = np.asarray(samples.reference_volumes, dtype=np.float64)
    if source_tets.shape != (particle_count,) or not np.issubdtype(source_tets.dtype, np.integer):
        raise ValueError("source_tets must contain one integer tet index per particle")
    if particle_count == 0 or source_tets.min() < 0 or source_tets.max() >= len(tet_mesh.tet_indices):
        raise ValueError("invalid particle source tetrahedra")
    if volumes.shape != (particle_count,) or not np.isfinite(volumes).all() or np.any(volumes <= 0.0):
        raise ValueError("particle reference volumes must be positive and finite")
    if np.any(np.bincount(source_tets, minlength=len(tet_mesh.tet_indices)) == 0):
        raise ValueError("every tetrahedron must contain particles for mesh reconstruction")
    # Each particle binds to the four corners of its tet; group bindings by vertex,
    # keeping particle order inside a vertex (the first binding is the anchor).
    vertex_of = np.asarray(tet_mesh.tet_indices)[source_tets].reshape(-1)
    particle_of = np.repeat(np.arange(particle_count, dtype=np.int64), 4)
    order = np.argsort(vertex_of, kind="stable")
    vertex_of, particle_of = vertex_of[order], particle_of[order]
    counts = np.bincount(vertex_of, minlength=vertex_count)
    offsets = np.concatenate(([0], np.cumsum(counts))).astype(np.int32)
    weights = volumes[particle_of]
    weights = weights / np.bincount(vertex_of, weights=weights, minlength=vertex_count)[vertex_of]
    ref_offsets = tet_mesh.vertex_positions[vertex_of] - samples.particle_positions[particle_of]
    return MeshBindingTables(offsets, particle_of.astype(np.int32), weights, ref_offsets,
                             int(np.count_nonzero(counts == 0)))
