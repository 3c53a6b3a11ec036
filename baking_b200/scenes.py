"""Seeded synthetic baking scenes (no dataset is involved; all inputs are generated).

``box_loaf``: a box of dough resting 0.1 mm above the floor wall of a unit-cube
grid, filled with jittered particles (equal reference volumes) emitted cell by
cell in Morton order of their grid cell, and a voxel tet mesh (six tets per
voxel) whose boundary faces carry the transport's surface terms. Particles are
assigned to tets by point location, so every tet owns particles.

``jittered_sphere``: a ball of dough sampled with k x k x k jittered points per
grid cell inside the ball, meshed with the voxels that the ball covers.
"""

from __future__ import annotations

from dataclasses import dataclass, fields, replace

import numpy as np

from .config import DingConfig, MaterialConfig, SimulationConfig, TransportConfig
from .geometry import ParticleSamples, VoxelTetMesh


@dataclass
class Scene:
    name: str
    tet_mesh: object
    samples: ParticleSamples
    simulation: SimulationConfig
    material: MaterialConfig
    ding: DingConfig
    transport: TransportConfig
    gas_source_rates: np.ndarray | None = None
    initial_velocity: tuple = (0.0, 0.0, 0.0)
    # Initial elastic stretch (principal log strains along x, y, z) applied to F and Fe of every
    # particle: a shaped, pre-stressed crumb. Zero for a stress-free start.
    initial_log_strain: tuple = (0.0, 0.0, 0.0)

    @property
    def particle_count(self):
        return len(self.samples.particle_positions)


def _morton3(ix, iy, iz):
    def spread(v):
        v = v.astype(np.uint64) & np.uint64(0x1FFFFF)
        v = (v | (v << np.uint64(32))) & np.uint64(0x1F00000000FFFF)
        v = (v | (v << np.uint64(16))) & np.uint64(0x1F0000FF0000FF)
        v = (v | (v << np.uint64(8))) & np.uint64(0x100F00F00F00F00F)
        v = (v | (v << np.uint64(4))) & np.uint64(0x10C30C30C30C30C3)
        v = (v | (v << np.uint64(2))) & np.uint64(0x1249249249249249)
        return v
    return spread(ix) | (spread(iy) << np.uint64(1)) | (spread(iz) << np.uint64(2))


def stencil_order(points, spacing, origin=(0.0, 0.0, 0.0)):
    """Permutation that groups particles by quadratic stencil base floor(x/dx - 0.5), Morton order.

    Particles sharing a base scatter to the same 27 nodes, so the device scatter sums them in
    registers and shared memory before touching the grid.
    """
    base = np.floor((np.asarray(points) - np.asarray(origin)) / spacing - 0.5).astype(np.int64)
    base -= base.min(axis=0)
    return np.argsort(_morton3(base[:, 0], base[:, 1], base[:, 2]), kind="stable")


def _kuhn_index(local):
    """Index (in VoxelTetMesh's tet order) of the Kuhn tet containing unit-voxel coordinates ``local``."""
    from itertools import permutations
    order = np.argsort(-local, axis=1, kind="stable")          # axes by descending coordinate
    table = {p: k for k, p in enumerate(permutations(range(3)))}
    codes = order[:, 0] * 9 + order[:, 1] * 3 + order[:, 2]
    lut = np.zeros(27, dtype=np.int64)
    for p, k in table.items():
        lut[p[0] * 9 + p[1] * 3 + p[2]] = k
    return lut[codes]


def _locate(points, origin, voxel, shape):
    rel = (points - origin) / voxel
    cell = np.clip(np.floor(rel).astype(np.int64), 0, np.asarray(shape) - 1)
    voxel_id = np.ravel_multi_index(cell.T, shape)
    return voxel_id * 6 + _kuhn_index(rel - cell)


def box_loaf(resolution=128, particle_count=1_000_000, seed=0, size=(0.4, 0.15, 0.2), gas=True,
             time_step=5e-5, gas_rate_max=1e-3, initial_temperature=None, prestrain=0.0):
    """Box loaf (x length, y height, z width) on the floor, ``particle_count`` jittered particles.
    ``initial_temperature`` (K) starts the crumb part-baked (default: the transport default, 293.15 K;
    at 318 K the temperature tables lower the yield stress to 0.425 of its base value).
    ``prestrain`` a > 0 starts every particle with the isochoric elastic stretch
    diag(exp(a/2), exp(-a), exp(a/2)) (compressed in y), which yields from the first substep."""
    dx = 1.0 / resolution
    voxel = 2 * dx
    nvox = np.maximum(1, np.round(np.asarray(size) / voxel).astype(np.int64))
    extent = nvox * voxel
    boundary_cells = 3
    floor = (boundary_cells - 1) * dx
    origin = np.array([0.5 - extent[0] / 2, floor + 1e-4, 0.5 - extent[2] / 2])
    origin[[0, 2]] = np.round(origin[[0, 2]] / dx) * dx
    mesh = VoxelTetMesh(np.ones(tuple(nvox), dtype=bool), origin, voxel)
    # Cells of size dx inside the box, visited in Morton order; counts as even as possible.
    ncell = nvox * 2
    cells = np.stack(np.meshgrid(*[np.arange(c) for c in ncell], indexing="ij"), -1).reshape(-1, 3)
    cells = cells[np.argsort(_morton3(cells[:, 0], cells[:, 1], cells[:, 2]), kind="stable")]
    per = np.full(len(cells), particle_count // len(cells), dtype=np.int64)
    per[: particle_count - per.sum()] += 1
    rng = np.random.default_rng(seed)
    corner = np.repeat(cells, per, axis=0).astype(np.float64)
    points = origin + (corner + rng.random((particle_count, 3))) * dx
    points = points[stencil_order(points, dx)]
    source_tets = _locate(points, origin, voxel, tuple(nvox))
    if np.any(np.bincount(source_tets, minlength=len(mesh.tet_indices)) == 0):
        raise ValueError("a tet received no particle; use more particles")
    density = 1000.0
    volumes = np.full(particle_count, float(np.prod(extent)) / particle_count)
    samples = ParticleSamples(points, volumes, density * volumes, source_tets)
    sim = replace(SimulationConfig(), grid_resolution=resolution, grid_spacing=dx, time_step=time_step,
                  gravity=(0.0, -9.8, 0.0), boundary_cells=boundary_cells, device_name="cuda:0")
    material = MaterialConfig(density=density, model="ding2019")
    ding = DingConfig(porosity=0.2 if gas else 0.0, temperature_enabled=True, gas_enabled=gas)
    transport = TransportConfig(enabled=True) if initial_temperature is None else \
        TransportConfig(enabled=True, initial_temperature_k=float(initial_temperature))
    rates = rng.uniform(0.0, gas_rate_max, particle_count).astype(np.float32) if gas else None
    strain = (0.5 * prestrain, -prestrain, 0.5 * prestrain)
    return Scene("box_loaf", mesh, samples, sim, material, ding, transport, rates, initial_log_strain=strain)


def jittered_sphere(resolution=64, per_axis=2, radius=0.1, center=(0.5, 0.5, 0.3), seed=0, time_step=1e-4):
    """Sphere of dough, ``per_axis``^3 jittered particles per cell, Ding defaults, transport on, gas off."""
    dx = 1.0 / resolution
    sub = dx / per_axis
    lo = np.floor((np.asarray(center) - radius) / dx).astype(int)
    hi = np.ceil((np.asarray(center) + radius) / dx).astype(int)
    axes = [np.arange(lo[a] * per_axis, hi[a] * per_axis) for a in range(3)]
    grid = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 3)
    rng = np.random.default_rng(seed)
    points = (grid + 0.5 + rng.uniform(-0.5, 0.5, grid.shape)) * sub
    points = points[np.linalg.norm(points - np.asarray(center), axis=1) <= radius]
    points = points[stencil_order(points, dx)]
    # Mesh: the voxels (size dx) that hold particles.
    vox_lo = np.floor(points.min(axis=0) / dx).astype(int)
    vcell = np.floor(points / dx).astype(np.int64) - vox_lo
    shape = tuple(vcell.max(axis=0) + 1)
    occupied = np.zeros(shape, dtype=bool)
    occupied[tuple(vcell.T)] = True
    mesh = VoxelTetMesh(occupied, vox_lo * dx, dx)
    # Tet ids of VoxelTetMesh follow the occupied voxels in x-major order.
    voxel_rank = np.cumsum(occupied.reshape(-1)) - 1
    local = points / dx - np.floor(points / dx)
    source_tets = voxel_rank[np.ravel_multi_index(vcell.T, shape)] * 6 + _kuhn_index(local)
    counts = np.bincount(source_tets, minlength=len(mesh.tet_indices))
    keep_tets = counts > 0
    if not keep_tets.all():
        # Drop tets without particles (reference binding needs every tet sampled).
        remap = np.cumsum(keep_tets) - 1
        from .geometry import ValidateTetMesh
        mesh = ValidateTetMesh(mesh.vertex_positions, mesh.tet_indices[keep_tets])
        source_tets = remap[source_tets]
        used = np.unique(mesh.tet_indices)
        vmap = np.full(len(mesh.vertex_positions), -1)
        vmap[used] = np.arange(len(used))
        mesh = ValidateTetMesh(mesh.vertex_positions[used], vmap[mesh.tet_indices])
    density = 1000.0
    volumes = np.full(len(points), sub ** 3)
    samples = ParticleSamples(points, volumes, density * volumes, source_tets)
    sim = replace(SimulationConfig(), grid_resolution=resolution, grid_spacing=dx, time_step=time_step,
                  gravity=(0.0, -9.8, 0.0), device_name="cuda:0")
    return Scene("jittered_sphere", mesh, samples, sim, MaterialConfig(model="ding2019"), DingConfig(),
                 TransportConfig(enabled=True, initial_temperature_k=298.15, oven_temperature_k=453.15,
                                 tray_temperature_k=453.15, initial_saturation=0.4))


def permuted(scene, order):
    """The same scene with its particles listed in another order (``order[k]`` is the sample that
    goes to position k): every per-particle sample array and per-particle gas source rate."""
    order = np.asarray(order)
    n = len(scene.samples.particle_positions)
    if sorted(order.tolist()) != list(range(n)):
        raise ValueError("order must be a permutation of the particle indices")
    s = scene.samples
    samples = replace(s, **{f.name: np.asarray(getattr(s, f.name))[order] for f in fields(s)
                            if np.ndim(getattr(s, f.name)) >= 1 and len(getattr(s, f.name)) == n})
    rates = scene.gas_source_rates
    if rates is not None and np.ndim(rates) >= 1 and len(rates) == n:
        rates = np.asarray(rates)[order]
    return replace(scene, samples=samples, gas_source_rates=rates)


def make_simulator(scene, engine="cuda", **kwargs):
    """Build the device ``MpmSimulator`` (or, for tests, another engine class) for a scene."""
    if engine == "cuda":
        from .physics.mpm import MpmSimulator
        cls = MpmSimulator
    else:
        cls = engine
    sim_cfg = scene.simulation if engine == "cuda" else replace(scene.simulation, device_name="cpu")
    sim = cls(scene.tet_mesh, scene.samples, sim_cfg, scene.material, scene.initial_velocity,
              ding_config=scene.ding, transport_config=scene.transport, **kwargs)
    if scene.gas_source_rates is not None:
        sim.SetGasSourceRates(scene.gas_source_rates)
    if any(scene.initial_log_strain):
        stretch = np.diag(np.exp(np.asarray(scene.initial_log_strain, np.float64))).astype(np.float32)
        st = sim.current_state
        for target in (st.deformation_gradients, getattr(st.material_state, "elastic_gradients", None)):
            if target is None:
                continue
            if isinstance(target, np.ndarray):
                target[...] = stretch
            else:
                import torch
                target.copy_(torch.as_tensor(stretch, device=target.device).expand(target.shape))
    return sim


def dough_ball(resolution, particle_count, seed=0, oven_temperature=453.15, initial_temperature=318.15,
               prestrain=0.0, time_step=5e-5, gas_rate_max=1e-3):
    """A sphere of the box loaf's dough (Ding with temperature tables, porosity 0.2, gas, thermal-water
    transport) centred in the unit cube with about ``particle_count`` jittered particles: the radius
    and the particles per cell axis (2..8) are chosen so that the sphere fits within 0.3 of the centre."""
    from dataclasses import replace as _replace
    dx = 1.0 / resolution
    per_axis, radius = 2, None
    for per_axis in range(2, 9):
        radius = (3.0 * particle_count / (4.0 * np.pi)) ** (1.0 / 3.0) / (resolution * per_axis)
        if radius <= 0.3:
            break
    radius = min(radius, 0.3)
    base = jittered_sphere(resolution, per_axis, radius, (0.5, 0.5, 0.5), seed, time_step)
    rng = np.random.default_rng(seed + 7919)
    n = len(base.samples.particle_positions)
    transport = _replace(base.transport, oven_temperature_k=float(oven_temperature),
                         tray_temperature_k=float(oven_temperature), initial_temperature_k=float(initial_temperature))
    ding = DingConfig(porosity=0.2, temperature_enabled=True, gas_enabled=True)
    rates = rng.uniform(0.0, gas_rate_max, n).astype(np.float32)
    del dx
    return _replace(base, name="dough_ball", ding=ding, transport=transport, gas_source_rates=rates,
                    initial_log_strain=(0.5 * prestrain, -prestrain, 0.5 * prestrain))


def dough_batch(count=64, seed=0, particles=(5_000, 200_000), resolutions=(32, 48, 64, 96),
                oven_celsius=(150.0, 220.0), prestrain=(0.0, 0.0)):
    """``count`` independent dough balls drawn from ``seed``: particle count uniform in ``particles``,
    grid resolution from ``resolutions``, oven temperature uniform in ``oven_celsius``, isochoric
    prestrain uniform in ``prestrain``."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        out.append(dough_ball(int(rng.choice(resolutions)), int(rng.integers(particles[0], particles[1] + 1)),
                              seed=seed * 1000 + k, oven_temperature=273.15 + rng.uniform(*oven_celsius),
                              prestrain=float(rng.uniform(*prestrain))))
    return out
