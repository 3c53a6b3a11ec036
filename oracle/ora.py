"""ctypes binding of the CPU oracle (``baking_oracle.c``) -- test infrastructure only.

Every wrapper takes numpy arrays in the reference's layouts (vec3 as (N, 3),
mat33 as (N, 3, 3) row-major, both float32; float64 scalars where the reference
uses ``wp.float64``) and calls the C restatement of one reference kernel.
"""

from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libbaking_oracle.so"


def build(force=False):
    """Compile the oracle with its Makefile (gcc only)."""
    source = HERE / "baking_oracle.c"
    if force or not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < source.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(str(LIB_PATH))
        _declare(_lib)
    return _lib


class DingParams(C.Structure):
    _fields_ = [("coupled_porosity", C.c_int), ("temperature_enabled", C.c_int), ("mu", C.c_float),
                ("lam", C.c_float), ("yield_stress", C.c_float), ("initial_porosity", C.c_float),
                ("dt", C.c_float), ("knots", C.c_float * 4), ("yield_factors", C.c_float * 4),
                ("viscosity_factors", C.c_float * 4)]


class ScalarParams(C.Structure):
    _fields_ = [("oven_temperature", C.c_float), ("tray_temperature", C.c_float), ("tray_transfer", C.c_float),
                ("surface_loss", C.c_float), ("water_density", C.c_float), ("latent_heat", C.c_float),
                ("water_enabled", C.c_int), ("origin", C.c_float * 3), ("dx", C.c_float), ("R", C.c_int)]


P = C.c_void_p
I32, I64, F32, F64 = C.c_int, C.c_int64, C.c_float, C.c_double


def _declare(L):
    sig = {
        "ora_set_threads": (None, [I32]),
        "ora_get_max_threads": (I32, []),
        "ora_svd3": (None, [P, P, P, P]),
        "ora_quadratic_weight": (F32, [F32, I32]),
        "ora_particle_to_grid": (None, [I32, P, P, P, P, P, P, P, P, P, F32, I32, F32, P]),
        "ora_update_grid": (None, [I64, P, P, P, I32, I32, P, F32]),
        "ora_grid_to_particle": (None, [I32, P, P, P, P, P, P, P, P, F32, I32, F32, P]),
        "ora_compute_elastic_stress": (None, [I32, P, P, F32, F32, P]),
        "ora_temperature_factor": (F32, [F32, P, P]),
        "ora_porosity_coefficient": (F32, [F32]),
        "ora_solve_overstress": (F32, [F32, F32, F32, F32]),
        "ora_pressure_coefficient64": (F64, [F64]),
        "ora_overstress64": (F64, [F64, F64, F64, F64]),
        "ora_porosity_prediction": (F64, [F64, F32, F32, F32, F32, F32, F64, F32]),
        "ora_solve_porosity": (F32, [F32, F32, F32, F32, F32, F64, F32]),
        "ora_ding_return": (None, [P, F32, F32, F32, F32, F32, F32, P, P, P, P, P, P]),
        "ora_update_ding": (None, [I32, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P]),
        "ora_gas_pressure": (F64, [F64, F32, F32, F32]),
        "ora_combine_gas_stress": (None, [I32, P, P, P, P, P, P, P, F32, F32, P, F32, F32, F32, F32]),
        "ora_refresh_gas": (None, [I32, P, P, P, P, P, P]),
        "ora_surface_areas": (None, [I32, P, P, P, P, P, F32, F32]),
        "ora_scalar_to_grid": (None, [I32] + [P] * 10 + [P] * 9 + [P]),
        "ora_grid_fields": (None, [I64, P, P, P, P, P, P, F32]),
        "ora_diffuse_grid": (None, [I64] + [P] * 11 + [F32, F32, F32, I32, F32, I32, F32]),
        "ora_scalar_to_particles": (None, [I32] + [P] * 21 + [F32, P, F32, I32, F32, P]),
        "ora_local_gas": (None, [I32, P, P, P, P, P, P, P, P, I32, F32, F32, F32, F32, I32]),
        "ora_water_stress": (None, [I32, P, P, P, P, F32, F32]),
        "ora_saturations": (None, [I32, P, P, P, P, F32]),
        "ora_reconstruct_mesh_vertices": (None, [I32, P, P, P, P, P, P, P, P]),
        "ora_settling_metrics": (None, [I32, P, P, P, P, P, F32]),
    }
    for name, (restype, argtypes) in sig.items():
        fn = getattr(L, name)
        fn.restype = restype
        fn.argtypes = argtypes


_DT = {"f4": np.float32, "f8": np.float64, "i4": np.int32}


def ptr(array, kind):
    """Pointer to a C-contiguous numpy array of the required dtype (no silent copies)."""
    if array is None:
        return None
    if not isinstance(array, np.ndarray) or array.dtype != _DT[kind] or not array.flags.c_contiguous:
        raise TypeError(f"oracle expects a C-contiguous {_DT[kind].__name__} array")
    return array.ctypes.data


def f32(*shape):
    return np.zeros(shape, dtype=np.float32)


def f64(*shape):
    return np.zeros(shape, dtype=np.float64)


def i32(*shape):
    return np.zeros(shape, dtype=np.int32)


def vec(values, dtype=np.float32):
    return np.ascontiguousarray(np.asarray(values, dtype=dtype))


def set_threads(n):
    lib().ora_set_threads(int(n))


def max_threads():
    return lib().ora_get_max_threads()


# ----------------------------------------------------------------- kernels
def svd3(matrix):
    a = vec(matrix, np.float64).reshape(9)
    u, s, v = f64(9), f64(3), f64(9)
    lib().ora_svd3(ptr(a, "f8"), ptr(u, "f8"), ptr(s, "f8"), ptr(v, "f8"))
    return u.reshape(3, 3), s, v.reshape(3, 3)


def particle_to_grid(x, v, Cm, tau, mass, V0, node_m, node_p, origin, dx, R, dt, flags):
    lib().ora_particle_to_grid(len(x), ptr(x, "f4"), ptr(v, "f4"), ptr(Cm, "f4"), ptr(tau, "f4"), ptr(mass, "f4"),
                               ptr(V0, "f4"), ptr(node_m, "f4"), ptr(node_p, "f4"), ptr(vec(origin), "f4"),
                               dx, R, dt, ptr(flags, "i4"))


def update_grid(node_m, node_p, node_v, R, boundary_cells, gravity, dt):
    lib().ora_update_grid(len(node_m), ptr(node_m, "f4"), ptr(node_p, "f4"), ptr(node_v, "f4"), R,
                          boundary_cells, ptr(vec(gravity), "f4"), dt)


def grid_to_particle(x, F, node_v, x_out, v_out, C_out, F_out, origin, dx, R, dt, flags):
    lib().ora_grid_to_particle(len(x), ptr(x, "f4"), ptr(F, "f4"), ptr(node_v, "f4"), ptr(x_out, "f4"),
                               ptr(v_out, "f4"), ptr(C_out, "f4"), ptr(F_out, "f4"), ptr(vec(origin), "f4"),
                               dx, R, dt, ptr(flags, "i4"))


def compute_elastic_stress(F, tau, mu, lam, flags):
    lib().ora_compute_elastic_stress(len(F), ptr(F, "f4"), ptr(tau, "f4"), mu, lam, ptr(flags, "i4"))


def temperature_factor(T, knots, factors):
    return lib().ora_temperature_factor(T, ptr(vec(knots), "f4"), ptr(vec(factors), "f4"))


def porosity_coefficient(n):
    return lib().ora_porosity_coefficient(n)


def solve_overstress(q2, p2, d, h):
    return lib().ora_solve_overstress(q2, p2, d, h)


def pressure_coefficient64(n):
    return lib().ora_pressure_coefficient64(n)


def overstress64(q, p, d, h):
    return lib().ora_overstress64(q, p, d, h)


def porosity_prediction(n, q, p, d, h, e, Vp, n0):
    return lib().ora_porosity_prediction(n, q, p, d, h, e, Vp, n0)


def solve_porosity(q, p, d, h, e, Vp, n0):
    return lib().ora_solve_porosity(q, p, d, h, e, Vp, n0)


def ding_return(trial, mu, lam, ty, eta, a, dt):
    t = vec(trial).reshape(9)
    fe, tau, res = f32(9), f32(9), np.zeros(1, np.float32)
    lib().ora_ding_return(ptr(t, "f4"), mu, lam, ty, eta, a, dt, None, None, None, ptr(fe, "f4"), ptr(tau, "f4"),
                          ptr(res, "f4"))
    return fe.reshape(3, 3), tau.reshape(3, 3), float(res[0])


def ding_params(coupled, temperature_enabled, mu, lam, yield_stress, n0, dt, knots, yf, vf):
    p = DingParams()
    p.coupled_porosity, p.temperature_enabled = int(coupled), int(temperature_enabled)
    p.mu, p.lam, p.yield_stress, p.initial_porosity, p.dt = mu, lam, yield_stress, n0, dt
    p.knots[:] = list(knots)
    p.yield_factors[:] = list(yf)
    p.viscosity_factors[:] = list(vf)
    return p


def update_ding(Fe_old, n_old, gel_old, F_tot, C_new, Fe_new, Fp_new, tau_new, residuals, n_new, T_out,
                gel_new, yield_out, visc_out, viscosity_parameter, flags, por_res, params, T_local):
    lib().ora_update_ding(len(Fe_old), ptr(Fe_old, "f4"), ptr(n_old, "f4"), ptr(gel_old, "i4"), ptr(F_tot, "f4"),
                          ptr(C_new, "f4"), ptr(Fe_new, "f4"), ptr(Fp_new, "f4"), ptr(tau_new, "f4"),
                          ptr(residuals, "f4"), ptr(n_new, "f4"), ptr(T_out, "f4"), ptr(gel_new, "i4"),
                          ptr(yield_out, "f4"), ptr(visc_out, "f4"), ptr(viscosity_parameter, "f4"),
                          ptr(flags, "i4"), ptr(por_res, "f4"), C.addressof(params), ptr(T_local, "f4"))


def gas_pressure(moles, T, J, n):
    return lib().ora_gas_pressure(moles, T, J, n)


def combine_gas_stress(tau_s, F, por, moles, T, tau_t, flags, ambient, n0, density, K, dt, dx, cfl):
    lib().ora_combine_gas_stress(len(F), ptr(tau_s, "f4"), ptr(F, "f4"), ptr(por, "f4"), ptr(moles, "f8"),
                                 ptr(T, "f4"), ptr(tau_t, "f4"), ptr(flags, "i4"), ambient, n0,
                                 ptr(density, "f4"), K, dt, dx, cfl)


def refresh_gas(old_moles, new_moles, F, por, pressures, T):
    lib().ora_refresh_gas(len(F), ptr(old_moles, "f8"), ptr(new_moles, "f8"), ptr(F, "f4"), ptr(por, "f4"),
                          ptr(pressures, "f8"), ptr(T, "f4"))


def surface_areas(vertices, faces, owners, exposed, contact, floor, contact_distance):
    lib().ora_surface_areas(len(faces), ptr(vertices, "f4"), ptr(faces, "i4"), ptr(owners, "i4"),
                            ptr(exposed, "f8"), ptr(contact, "f8"), floor, contact_distance)


def scalar_params(oven, tray, tray_transfer, surface_loss, water_density, latent, water_enabled, origin, dx, R):
    p = ScalarParams()
    p.oven_temperature, p.tray_temperature, p.tray_transfer = oven, tray, tray_transfer
    p.surface_loss, p.water_density, p.latent_heat = surface_loss, water_density, latent
    p.water_enabled = int(water_enabled)
    p.origin[:] = list(origin)
    p.dx, p.R = dx, R
    return p


def scalar_to_grid(x, F, V0, cap, T, W, exposed, contact, heat_parameter, params, g, p_heat, p_loss, flags):
    lib().ora_scalar_to_grid(len(x), ptr(x, "f4"), ptr(F, "f4"), ptr(V0, "f4"), ptr(cap, "f8"), ptr(T, "f8"),
                             ptr(W, "f8"), ptr(exposed, "f8"), ptr(contact, "f8"), ptr(heat_parameter, "f4"),
                             C.addressof(params), ptr(g["volumes"], "f8"), ptr(g["capacities"], "f8"),
                             ptr(g["energy"], "f8"), ptr(g["water"], "f8"), ptr(g["heat"], "f8"),
                             ptr(g["loss"], "f8"), ptr(g["exchange"], "f8"), ptr(p_heat, "f8"),
                             ptr(p_loss, "f8"), ptr(flags, "i4"))


def grid_fields(vol, cap, energy, water, T, s, water_density):
    lib().ora_grid_fields(len(vol), ptr(vol, "f8"), ptr(cap, "f8"), ptr(energy, "f8"), ptr(water, "f8"),
                          ptr(T, "f8"), ptr(s, "f8"), water_density)


def diffuse_grid(vol, cap, T, s, water, heat, loss, exch, dT, dW, errors, conductivity, diffusivity,
                 water_density, water_enabled, dx, R, dt):
    lib().ora_diffuse_grid(len(vol), ptr(vol, "f8"), ptr(cap, "f8"), ptr(T, "f8"), ptr(s, "f8"), ptr(water, "f8"),
                           ptr(heat, "f8"), ptr(loss, "f8"), ptr(exch, "f8"), ptr(dT, "f8"), ptr(dW, "f8"),
                           ptr(errors, "i4"), conductivity, diffusivity, water_density, int(water_enabled), dx, R,
                           dt)


def scalar_to_particles(x, T_old, W_old, loss_old, exch_old, dry, V0, F, n_water, n_dT, n_dW, p_heat, p_loss,
                        T_new, T_mat, W_new, loss_new, exch_new, mass_new, dens_new, sat_new, water_density,
                        origin, dx, R, dt, flags):
    lib().ora_scalar_to_particles(
        len(x), ptr(x, "f4"), ptr(T_old, "f8"), ptr(W_old, "f8"), ptr(loss_old, "f8"), ptr(exch_old, "f8"),
        ptr(dry, "f8"), ptr(V0, "f4"), ptr(F, "f4"), ptr(n_water, "f8"), ptr(n_dT, "f8"), ptr(n_dW, "f8"),
        ptr(p_heat, "f8"), ptr(p_loss, "f8"), ptr(T_new, "f8"), ptr(T_mat, "f4"), ptr(W_new, "f8"),
        ptr(loss_new, "f8"), ptr(exch_new, "f8"), ptr(mass_new, "f4"), ptr(dens_new, "f4"), ptr(sat_new, "f8"),
        water_density, ptr(vec(origin), "f4"), dx, R, dt, ptr(flags, "i4"))


def local_gas(old_moles, T_old, T_new, new_moles, pressures, F, por, parameter, density, peak, width, dt, produce):
    per_particle = int(len(parameter) == len(old_moles) and len(old_moles) > 1)
    lib().ora_local_gas(len(old_moles), ptr(old_moles, "f8"), ptr(T_old, "f8"), ptr(T_new, "f8"),
                        ptr(new_moles, "f8"), ptr(pressures, "f8"), ptr(F, "f4"), ptr(por, "f4"),
                        ptr(parameter, "f4"), per_particle, density, peak, width, dt, int(produce))


def water_stress(F, sat, tau_old, tau_new, s0, stiffness):
    lib().ora_water_stress(len(F), ptr(F, "f4"), ptr(sat, "f8"), ptr(tau_old, "f4"), ptr(tau_new, "f4"), s0,
                           stiffness)


def saturations(W, V0, F, sat, density):
    lib().ora_saturations(len(W), ptr(W, "f8"), ptr(V0, "f4"), ptr(F, "f4"), ptr(sat, "f8"), density)


def reconstruct_mesh_vertices(x, F, ref_vertices, offsets, particles, weights, ref_offsets, out):
    lib().ora_reconstruct_mesh_vertices(len(out), ptr(x, "f4"), ptr(F, "f4"), ptr(ref_vertices, "f4"),
                                        ptr(offsets, "i4"), ptr(particles, "i4"), ptr(weights, "f4"),
                                        ptr(ref_offsets, "f4"), ptr(out, "f4"))


def settling_metrics(v, Cm, Fp_old, Fp_new, metrics, dt):
    lib().ora_settling_metrics(len(v), ptr(v, "f4"), ptr(Cm, "f4"), ptr(Fp_old, "f4"), ptr(Fp_new, "f4"),
                               ptr(metrics, "f4"), dt)
