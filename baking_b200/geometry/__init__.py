"""Scene set-up (tet meshes, particle samples, index tables) and device mesh reconstruction.

``ParticleMeshBinding`` (device) is imported from ``geometry.mesh_tracking`` on demand so that
the host-only helpers here import without CUDA.
"""
from .mesh import (TetMesh, ComputeSignedVolumes, ValidateTetMesh, VoxelTetMesh, CreateDemoMesh,
                   CreateSphereMesh, LoadTetMesh)
from .sampling import (ParticleSamples, SampleParticles, BoundaryFaces, MeshBindingTables,
                       MeshBindingTables_build)

__all__ = ["TetMesh", "ComputeSignedVolumes", "ValidateTetMesh", "VoxelTetMesh", "CreateDemoMesh",
           "CreateSphereMesh", "LoadTetMesh", "ParticleSamples", "SampleParticles", "BoundaryFaces",
           "MeshBindingTables", "MeshBindingTables_build"]
