"""Algorithmic HBM bytes per launch of each kernel, for the roofline fraction.

A kernel's algorithmic traffic counts every array it must read and every array it
must write exactly once, at the stored precision, and nothing else: no re-reads,
no atomics traffic beyond one write per touched grid node. Per-particle figures
multiply the particle count; per-node figures multiply the number of active grid
nodes (nodes with mass); per-binding / per-face figures multiply the mesh tables.
"""

from __future__ import annotations

# kernel -> (bytes per particle, bytes per active node)
PER_KERNEL = {
    # x 12, v 12, C 36, tau 36, m 4, V0 4 read; node (p, m) 16 written
    "bk_particle_to_grid": (104, 16),
    # node (p, m) 16 read, node v 16 written
    "bk_update_grid": (0, 32),
    # x 12, F 36 read, x v C F 96 written; node v 16 read
    "bk_grid_to_particle": (144, 16),
    # Fe 36, n 4, gelled 4, F 36, C 36, T 4 read; Fe Fp tau 108, 7 scalars 28 written
    "bk_update_ding": (256, 0),
    # tau_s 36, F 36, n 4, N 8, T 4, rho 4 read; tau 36 written
    "bk_combine_gas_stress": (128, 0),
    # N 8, F 36, n 4, T 4 read; N 8, p 8 written
    "bk_refresh_gas": (68, 0),
    # x 12, F 36, V0 4, cap 8, T 8, W 8, exposed 8, contact 8 read; heat, loss 16 written; 7 node fields
    "bk_scalar_to_grid": (108, 56),
    # 4 node fields read, T and s written
    "bk_grid_fields": (0, 48),
    # 8 node fields read, dT and dW written
    "bk_diffuse_grid": (0, 80),
    # x 12, T W loss exch dry 40, V0 4, F 36, heat loss 16 read; 8 outputs 52 written; 3 node fields
    "bk_scalar_to_particles": (160, 24),
    # N 8, T_old 8, T_new 8, F 36, n 4, alpha 4 read; N 8, p 8 written
    "bk_local_gas": (84, 0),
    # F 36, s 8, tau 36 read; tau 36 written
    "bk_water_stress": (116, 0),
    # W 8, V0 4, F 36 read; s 8 written
    "bk_saturations": (56, 0),
    # v 12, C 36, Fp_old 36, Fp_new 36 read
    "bk_settling_metrics": (120, 0),
}


def fused_bytes(kernel, engine, active_nodes, scatter_ahead=False):
    """Bytes per launch of the kernels inside ``bk_substep`` for the engine's mode; ``scatter_ahead``:
    the G2P kernel also scatters the next substep's transport fields."""
    n, tr, gas = engine.n, engine.transport, engine.gas
    ding = engine.is_ding
    if kernel == "surface_vertices":
        # per binding: particle index 4, weight 4, offset 12, particle x 12 and F 36; per vertex 12 written
        return 68 * engine.surface_bindings + 12 * engine.surface.vertex_count
    if kernel == "surface_owners":
        # per owner: x 12, F 36, V0 4, T 8, W 8 read, heat/loss 16 written; per owned face 3 vertices 36 + ids 12
        return 84 * engine.surface.owner_count + 48 * engine.owned_faces
    if kernel == "transport_scatter":
        return 76 * n + 32 * active_nodes          # x F V0 cap T W; 4 node fields written
    if kernel == "diffuse":
        return 72 * active_nodes                   # 7 node fields read, (dT, ratio) written
    if kernel == "clear_previous":
        return 32 * active_nodes                   # node (p, m) and v zeroed
    if kernel == "p2g":
        per = 12 + 12 + 36 + 36 + 4                # x v C F V0
        per += 36 + 4 if ding else 0               # tau, porosity
        per += (8 + 8 + 8 + 8 + 8) if tr else 4    # T W dry read, T W written | mass
        per += (8 + 4 + 8) if gas else 0           # N, alpha read, N written
        return per * n + (16 + 16 if tr else 16) * active_nodes
    if kernel == "grid_update":
        return (32 + (56 if tr else 0)) * active_nodes
    if kernel == "g2p_return":
        per = 48 + 96                               # x F read; x v C F written
        if ding:
            per += 36 + 4 + 4 + (8 if tr else 4)    # Fe, porosity, gelled, temperature read
            per += 36 + 36 + 4 + 4                  # Fe, tau, porosity, gelled written
        node = 16
        if scatter_ahead and engine.prescatter_allowed():
            # Inside an Advance call the kernel also scatters the next substep's transport fields:
            # V0 4, capacity 8, water 8 read (temperature counted above); 4 node fields written.
            per += 4 + 8 + 8
            node += 32
        return per * n + node * active_nodes
    return None


def algorithmic_bytes(kernel, simulator, active_nodes):
    n = simulator.particle_data.particle_count
    engine = getattr(simulator, "_engine", None)
    if engine is not None:
        fused = fused_bytes(kernel, engine, active_nodes, getattr(simulator, "scatter_ahead", False))
        if fused is not None:
            return fused
    if kernel in PER_KERNEL:
        per_particle, per_node = PER_KERNEL[kernel]
        return per_particle * n + per_node * active_nodes
    if kernel == "bk_reconstruct_mesh_vertices":
        binding = simulator.mesh_binding
        return 68 * int(binding.binding_particles.shape[0]) + 12 * binding.vertex_count
    if kernel == "bk_surface_areas" and simulator.transport is not None:
        return 60 * int(simulator.transport.faces.shape[0])
    return None
