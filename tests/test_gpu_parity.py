"""Device substep against the CPU oracle on the same seeded scenes (parity gate).

Tolerances follow the stated bar: grid mass and momentum within 1e-5 relative per
substep; particle x within 1e-4*dx and F/T/water/gas within 1e-4 relative
(atomic accumulation order and CUDA-vs-libm rounding are the only differences).
"""
import numpy as np
import pytest

from tests.scenes import baking_cube, build_gas, build_transport, set_velocity_field, to_np

pytestmark = pytest.mark.gpu


def _pair(builder, *args, **kwargs):
    out = []
    for engine in ("oracle", "cuda"):
        sim = builder(engine, *args, **kwargs)
        out.append(sim[0] if isinstance(sim, tuple) else sim)
    return out


def _compare_state(ref, dev, dx, steps, rtol=1e-4):
    a, b = ref.current_state, dev.current_state
    np.testing.assert_allclose(to_np(b.particle_positions), a.particle_positions, rtol=0, atol=1e-4 * dx)
    np.testing.assert_allclose(to_np(b.deformation_gradients), a.deformation_gradients, rtol=rtol, atol=rtol)
    if a.transport_state is not None:
        np.testing.assert_allclose(to_np(b.transport_state.temperatures), a.transport_state.temperatures, rtol=rtol)
        np.testing.assert_allclose(to_np(b.transport_state.water_masses), a.transport_state.water_masses, rtol=rtol)
    if a.material_state is not None:
        ms, md = a.material_state, b.material_state
        np.testing.assert_allclose(to_np(md.gas_moles), ms.gas_moles, rtol=rtol, atol=1e-12)
        np.testing.assert_allclose(to_np(md.porosities), ms.porosities, rtol=rtol, atol=1e-7)
        np.testing.assert_allclose(to_np(md.elastic_gradients), ms.elastic_gradients, rtol=rtol, atol=rtol)


def test_baking_cube_matches_oracle_per_substep():
    ref, rates = baking_cube("oracle")
    dev, _ = baking_cube("cuda")
    set_velocity_field(ref, rates)
    set_velocity_field(dev, rates)
    dx = ref.simulation_config.grid_spacing
    for step in range(20):
        ref.Step()
        dev.Step()
        m_ref, m_dev = ref.grid_masses.astype(np.float64), to_np(dev.grid_state.node_masses).astype(np.float64)
        np.testing.assert_allclose(m_dev.sum(), m_ref.sum(), rtol=1e-5)
        np.testing.assert_allclose(m_dev, m_ref, rtol=1e-5, atol=1e-5 * m_ref.max())
        p_ref = ref.grid_momenta.astype(np.float64)
        p_dev = to_np(dev.grid_state.node_momenta).astype(np.float64)
        np.testing.assert_allclose(p_dev, p_ref, rtol=1e-5, atol=1e-5 * np.abs(p_ref).max())
    _compare_state(ref, dev, dx, 20)


def test_gas_scene_matches_oracle_after_many_substeps():
    ref, dev = _pair(build_gas)
    ref.Advance(60)
    dev.Advance(60)
    _compare_state(ref, dev, ref.simulation_config.grid_spacing, 60)


def test_transport_scene_matches_oracle():
    ref, dev = _pair(build_transport, gas=True)
    ref.Advance(10)
    dev.Advance(10)
    _compare_state(ref, dev, ref.simulation_config.grid_spacing, 10)


@pytest.mark.parametrize("diagnostics", ["lean", "full"])
def test_box_loaf_matches_oracle(diagnostics):
    """The benchmark workload at reduced size (48^3 grid, 20k particles), both diagnostics modes."""
    from baking_b200.scenes import box_loaf, make_simulator
    from oracle.sim import OracleSimulator
    scene = box_loaf(resolution=48, particle_count=20000, seed=3, time_step=1e-4)
    ref = make_simulator(scene, engine=OracleSimulator)
    dev = make_simulator(scene, diagnostics=diagnostics)
    for _ in range(15):
        ref.Step()
    dev.Advance(15)
    dx = scene.simulation.grid_spacing
    _compare_state(ref, dev, dx, 15)
    a, b = ref.current_state, dev.current_state
    for name in ("temperatures", "yield_stresses", "viscosities", "reference_densities"):
        np.testing.assert_allclose(to_np(getattr(b.material_state, name)), getattr(a.material_state, name), rtol=1e-4,
                                   err_msg=name)
    np.testing.assert_allclose(to_np(b.material_state.plastic_gradients), a.material_state.plastic_gradients,
                               rtol=1e-4, atol=1e-4)
    np.testing.assert_allclose(to_np(b.material_state.gas_pressures), a.material_state.gas_pressures, rtol=1e-4)
    np.testing.assert_allclose(to_np(b.transport_state.saturations), a.transport_state.saturations, rtol=1e-4)
    np.testing.assert_allclose(to_np(b.transport_state.particle_masses), a.transport_state.particle_masses, rtol=1e-6)
    np.testing.assert_allclose(to_np(b.transport_state.water_losses), a.transport_state.water_losses, rtol=1e-4,
                               atol=1e-15)
    np.testing.assert_allclose(to_np(b.transport_state.heat_exchanges), a.transport_state.heat_exchanges, rtol=1e-4,
                               atol=1e-12)
    np.testing.assert_allclose(to_np(dev.grid_state.node_masses), ref.grid_masses, rtol=1e-5,
                               atol=1e-5 * ref.grid_masses.max())


def test_prescattered_transport_matches_substep_by_substep():
    """Inside one AdvanceUnchecked call each substep's G2P scatters the next substep's transport
    fields (volume, capacity, energy, water) ahead; Step() scatters them at the start of every
    substep. Both give the same state, up to float summation order."""
    from baking_b200.scenes import box_loaf, make_simulator
    scene = box_loaf(resolution=48, particle_count=20000, seed=4, time_step=1e-4)
    a = make_simulator(scene)
    b = make_simulator(scene)
    b.scatter_ahead = True
    for _ in range(12):
        a.Step()
    b.AdvanceUnchecked(12)
    b.CheckState()
    sa, sb = a.current_state, b.current_state
    dx = scene.simulation.grid_spacing
    np.testing.assert_allclose(to_np(sb.particle_positions), to_np(sa.particle_positions), rtol=0, atol=1e-5 * dx)
    np.testing.assert_allclose(to_np(sb.deformation_gradients), to_np(sa.deformation_gradients), rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(to_np(sb.transport_state.temperatures), to_np(sa.transport_state.temperatures),
                               rtol=1e-9)
    np.testing.assert_allclose(to_np(sb.transport_state.water_masses), to_np(sa.transport_state.water_masses),
                               rtol=1e-9)
    np.testing.assert_allclose(to_np(sb.material_state.gas_moles), to_np(sa.material_state.gas_moles), rtol=1e-9,
                               atol=1e-15)
    # Step() advances the surface accumulators after its checks (bk_surface_accumulate); the
    # unchecked call advances them in the surface kernel. The rates go through the saturation
    # W / (rho_w V0 det F), so they follow F's summation-order differences (1e-8 relative).
    for name in ("water_losses", "heat_exchanges"):
        acc_a, acc_b = to_np(getattr(sa.transport_state, name)), to_np(getattr(sb.transport_state, name))
        assert np.count_nonzero(acc_a) > 100, name
        np.testing.assert_allclose(acc_b, acc_a, rtol=1e-6, atol=1e-12 * np.abs(acc_a).max(), err_msg=name)
    m_a, m_b = to_np(a.grid_state.node_masses), to_np(b.grid_state.node_masses)
    np.testing.assert_allclose(m_b, m_a, rtol=1e-5, atol=1e-6 * m_a.max())
