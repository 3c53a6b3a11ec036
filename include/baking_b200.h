/*
 * baking_b200 -- C ABI of the B200 (sm_100a) MLS-MPM baking substep.
 *
 * One entry point per reference Warp kernel (same argument order as the kernel,
 * arrays passed as device pointers), plus the fused whole-substep entry points
 * the simulator uses. Conventions shared by every call:
 *
 *  - Device memory is owned by the caller; nothing here allocates or frees it.
 *  - Per-particle arrays are structure-of-arrays "planes": a vec3 is 3 planes and
 *    a mat33 is 9 planes (row-major component order), each plane `pitch`
 *    elements long, so component c of particle i lives at base[c * pitch + i].
 *    Scalars are one plane. Every particle array in one call shares `pitch`.
 *  - Grid nodes are indexed (i * R + j) * R + k like the reference
 *    (physics/transfer.py:31-33). Mechanics nodes are packed float4:
 *    node_pm = {px, py, pz, m} (momentum, mass), node_v = {vx, vy, vz, 0}.
 *  - `stream` is a cudaStream_t passed as void*; every call is asynchronous on it.
 *  - Return value: 0 on success, BK_ERR_* (< 0) on an invalid argument or a
 *    launch failure; bk_last_error() describes the most recent failure of the
 *    calling thread. No call aborts the process.
 *  - Physical failures (inverted J, stencil outside the grid, porosity domain,
 *    gas CFL, transport stability) are reported exactly as in the reference:
 *    int flags on the device set to 1, read by the host afterwards.
 */
#ifndef BAKING_B200_H
#define BAKING_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define BK_API __attribute__((visibility("default")))
#else
#define BK_API
#endif

#define BK_OK 0
#define BK_ERR_ARGUMENT (-1)
#define BK_ERR_LAUNCH (-2)
#define BK_ERR_UNSUPPORTED (-3)

typedef struct BkDingParams {
    int32_t coupled_porosity;    /* gas mode: end-state porosity solve */
    int32_t temperature_enabled;
    float shear_modulus, lame_lambda, yield_stress, initial_porosity, time_step;
    float temperature_knots[4], yield_factors[4], viscosity_factors[4];
} BkDingParams;

typedef struct BkScalarParams {
    float oven_temperature, tray_temperature, tray_transfer, surface_loss, water_density, latent_heat;
    int32_t water_enabled;
    float origin[3];
    float spacing;
    int32_t resolution;
} BkScalarParams;

/* Library version (major * 10000 + minor * 100 + patch). */
BK_API int bk_version(void);
/* Message of the last failed call on this thread ("" if none). */
BK_API const char *bk_last_error(void);

/* ---- mechanics: physics/transfer.py, physics/grid.py ------------------- */

/* ParticleToGrid, physics/transfer.py:36-70. Adds w*m and w*(m v + A (x_i - x_p)) into node_pm. */
BK_API int bk_particle_to_grid(int64_t n, int64_t pitch, const float *x, const float *v, const float *C,
                        const float *tau, const float *mass, const float *V0, float *node_pm,
                        const float *origin, float spacing, int32_t resolution, float time_step,
                        int32_t *flags, void *stream);

/* UpdateGrid, physics/grid.py:20-38. v = p/m + dt g with unilateral walls, where m > 0. */
BK_API int bk_update_grid(int32_t resolution, const float *node_pm, float *node_v, int32_t boundary_cells,
                   const float *gravity, float time_step, void *stream);

/* GridToParticle, physics/transfer.py:73-109. */
BK_API int bk_grid_to_particle(int64_t n, int64_t pitch, const float *x_in, const float *F_in, const float *node_v,
                        float *x_out, float *v_out, float *C_out, float *F_out, const float *origin,
                        float spacing, int32_t resolution, float time_step, int32_t *flags, void *stream);

/* ---- materials: physics/materials/{elastic,ding,gas}.py ------------------ */

/* ComputeElasticStress, physics/materials/elastic.py:13-26. */
BK_API int bk_compute_elastic_stress(int64_t n, int64_t pitch, const float *F, float *tau, float shear_modulus,
                              float lame_lambda, int32_t *flags, void *stream);

/* UpdateDing, physics/materials/ding.py:140-221 (ding_return :103-137, solve_porosity
   physics/materials/porous_return.py:43-61). flags has 3 entries (ding.py:232). */
BK_API int bk_update_ding(int64_t n, int64_t pitch, const float *Fe_old, const float *porosity_old,
                   const int32_t *gelled_old, const float *F_total, const float *C_new, float *Fe_new,
                   float *Fp_new, float *tau_new, float *residuals, float *porosity_new, float *temperature_out,
                   int32_t *gelled_new, float *yield_out, float *viscosity_out, const float *viscosity_parameter,
                   int32_t *flags, float *porosity_residuals, const BkDingParams *params,
                   const float *temperature_local, void *stream);

/* CombineGasStress, physics/materials/gas.py:16-35. */
BK_API int bk_combine_gas_stress(int64_t n, int64_t pitch, const float *tau_solid, const float *F, const float *porosity,
                          const double *moles, const float *temperature, float *tau_total, int32_t *flags,
                          float ambient_pressure, float initial_porosity, const float *density,
                          float elastic_modulus, float time_step, float spacing, float cfl_limit, void *stream);

/* RefreshGas, physics/materials/gas.py:38-45. */
BK_API int bk_refresh_gas(int64_t n, int64_t pitch, const double *old_moles, double *new_moles, const float *F,
                   const float *porosity, double *pressures, const float *temperature, void *stream);

/* ---- transport: physics/thermal_water.py, geometry/mesh_tracking.py ---- */

/* ReconstructMeshVertices, geometry/mesh_tracking.py:13-38. Vertex arrays use `vertex_pitch`;
   reference_offsets are 3 planes of `binding_pitch` (one entry per binding). */
BK_API int bk_reconstruct_mesh_vertices(int64_t vertex_count, int64_t pitch, const float *x, const float *F,
                                 int64_t vertex_pitch, const float *reference_vertices, const int32_t *offsets,
                                 const int32_t *particles, const float *weights, int64_t binding_pitch,
                                 const float *reference_offsets, float *out_vertices, void *stream);

/* SurfaceAreas, physics/thermal_water.py:77-92. faces: face_count x 3 int32 (row-major). */
BK_API int bk_surface_areas(int64_t face_count, int64_t vertex_pitch, const float *vertices, const int32_t *faces,
                     const int32_t *owners, double *exposed, double *contact, float floor_height,
                     float contact_distance, void *stream);

/* ScalarToGrid, physics/thermal_water.py:95-137. node_fields: 7 arrays of R^3 doubles in the order
   volumes, capacities, energy, water, heat, loss, exchange. */
BK_API int bk_scalar_to_grid(int64_t n, int64_t pitch, const float *x, const float *F, const float *V0,
                      const double *capacities, const double *temperatures, const double *water,
                      const double *exposed, const double *contact, const float *heat_parameter,
                      const BkScalarParams *params, double *const *node_fields, double *particle_heat,
                      double *particle_loss, int32_t *flags, void *stream);

/* GridFields, physics/thermal_water.py:140-147. */
BK_API int bk_grid_fields(int64_t node_count, const double *volumes, const double *capacities, const double *energy,
                   const double *water, double *temperatures, double *saturations, float water_density,
                   void *stream);

/* DiffuseGrid, physics/thermal_water.py:150-190 (7-point finite-volume stencil). */
BK_API int bk_diffuse_grid(int64_t node_count, const double *volumes, const double *capacities,
                    const double *temperatures, const double *saturations, const double *water,
                    const double *boundary_heat, const double *boundary_loss, const double *boundary_exchange,
                    double *temperature_changes, double *water_changes, int32_t *errors, float conductivity,
                    float diffusivity, float water_density, int32_t water_enabled, float spacing,
                    int32_t resolution, float time_step, void *stream);

/* ScalarToParticles, physics/thermal_water.py:193-229. */
BK_API int bk_scalar_to_particles(int64_t n, int64_t pitch, const float *x, const double *T_old, const double *W_old,
                           const double *loss_old, const double *exchange_old, const double *dry_masses,
                           const float *V0, const float *F, const double *node_water, const double *node_dT,
                           const double *node_dW, const double *particle_heat, const double *particle_loss,
                           double *T_new, float *T_material, double *W_new, double *loss_new, double *exchange_new,
                           float *mass_new, float *density_new, double *saturation_new, float water_density,
                           const float *origin, float spacing, int32_t resolution, float time_step,
                           int32_t *flags, void *stream);

/* LocalGas, physics/thermal_water.py:232-245. parameter has n entries when per_particle != 0
   (per-particle source rate), else 1. */
BK_API int bk_local_gas(int64_t n, int64_t pitch, const double *old_moles, const double *T_old, const double *T_new,
                 double *new_moles, double *pressures, const float *F, const float *porosity,
                 const float *parameter, int32_t per_particle, float density, float peak, float width,
                 float time_step, int32_t produce, void *stream);

/* WaterStress, physics/thermal_water.py:248-253. */
BK_API int bk_water_stress(int64_t n, int64_t pitch, const float *F, const double *saturations, const float *tau_old,
                    float *tau_new, float initial_saturation, float stiffness, void *stream);

/* Saturations, physics/thermal_water.py:256-260. */
BK_API int bk_saturations(int64_t n, int64_t pitch, const double *water, const float *V0, const float *F,
                   double *saturations, float density, void *stream);

/* SettlingMetrics, physics/quasistatic.py:11-21. metrics: 3 floats, max-reduced. */
BK_API int bk_settling_metrics(int64_t n, int64_t pitch, const float *v, const float *C, const float *Fp_old,
                        const float *Fp_new, float *metrics, float time_step, void *stream);


/* Device evaluation of the float64 end-state porosity solve, one problem per entry:
   solve_porosity (physics/materials/porous_return.py:43-61) into porosity[i] and
   porosity_prediction (:34-40) of that result into prediction[i]. */
BK_API int bk_solve_porosity(int64_t n, const float *q, const float *p, const float *dev_factor,
                             const float *mean_scale, const float *exponent, const double *plastic_volume,
                             float initial_porosity, float *porosity, double *prediction, void *stream);

/* Device evaluation of porosity_coefficient (physics/materials/ding.py:68-74) per entry. */
BK_API int bk_porosity_coefficient(int64_t n, const float *porosity, float *coefficient, void *stream);

/* ---- fused substep (the simulator's hot path) ----------------------------- */

/* One particle state (ping-pong buffer). Planes share BkSubstepParams.pitch. */
typedef struct BkState {
    float *x, *v, *C, *F;          /* 3, 3, 9, 9 planes */
    float *Fe, *tau;               /* Ding elastic gradient and Kirchhoff stress (9 planes); NULL if neo-Hookean */
    float *porosity;               /* Ding */
    int32_t *gelled;               /* Ding */
    float *material_temperature;   /* Ding temperature when transport is off (read) */
    double *temperature, *water;   /* transport; NULL when off */
    double *gas_moles;             /* gas mode; NULL when off */
} BkState;

/* Per-particle constants and device-resident scalar parameters. */
typedef struct BkConstants {
    const float *volume;           /* reference volume V0 */
    const float *mass;             /* particle mass (used when transport is off) */
    const double *capacity;        /* rho c V0 (transport) */
    const double *dry_mass;        /* (rho - rho_w s0) V0 (transport) */
    const float *gas_rate;         /* alpha: 1 value, or one per particle */
    int32_t gas_rate_per_particle;
    const float *viscosity_parameter;  /* 1 value */
    const float *heat_parameter;       /* 1 value (zero while settling) */
} BkConstants;

/* Dense R^3 grid; only the active box of the current particles is touched per substep. */
typedef struct BkGrid {
    float *node_pm;                /* R^3 float4 (px, py, pz, m); the last substep's values, zero elsewhere */
    float *node_v;                 /* R^3 float4 (vx, vy, vz, 0); the last substep's values, zero elsewhere */
    double *fields[7];             /* volumes, capacities, energy, water, heat, loss, exchange -- zero between substeps */
    double *node_dT_ratio;         /* R^3 x 2 doubles: temperature change, water change / node water */
    int32_t *bounds;               /* 12 ints (device): lo[3], hi[3] of the active node box being built,
                                      then lo[3], hi[3] of the last substep's box. Start as
                                      {INT_MAX x3, INT_MIN x3, INT_MAX x3, INT_MIN x3} on a zero grid.
                                      18 ints with the transport prescatter: then the box of the
                                      fields scattered ahead for the next substep. */
} BkGrid;

/* Surface terms: the boundary-face vertices and the particles that own boundary faces. */
typedef struct BkSurface {
    int64_t vertex_count;          /* surface vertices to rebuild */
    const int32_t *vertex_ids;     /* mesh vertex index of each */
    const int32_t *binding_offsets;/* mesh vertex -> binding range (CSR over all mesh vertices) */
    const int32_t *binding_particles;
    const float *binding_weights;
    int64_t binding_pitch;
    const float *reference_offsets;/* 3 planes of binding_pitch */
    int64_t vertex_pitch;
    float *vertices;               /* 3 planes of vertex_pitch (surface entries rebuilt) */
    const float *reference_vertices;   /* 3 planes of vertex_pitch (used for unbound vertices) */
    int64_t owner_count;           /* particles that own boundary faces */
    const int32_t *owners;
    const int32_t *owner_face_offsets; /* owner -> face range */
    const int32_t *faces;          /* 3 vertex ids per face, grouped by owner */
    double *owner_heat, *owner_loss;   /* per owner, this substep */
    float floor_height, contact_distance;
    int64_t binding_count;         /* total bindings of the vertex_ids vertices, a launch-size hint
                                      (0: unknown, one warp per vertex) */
    double *accumulate_water_losses, *accumulate_heat_exchanges;  /* optional (NULL: not here): the
                                      surface kernel of bk_substep also advances the owners'
                                      accumulators by accumulate_time_step * their rates, which
                                      bk_surface_accumulate does otherwise after the substep */
    float accumulate_time_step;
} BkSurface;

/* Optional full per-particle outputs of the reference kernels (NULL pointers are skipped). */
typedef struct BkDiagnostics {
    float *plastic_gradients;      /* Fp, 9 planes */
    float *return_residuals, *porosity_residuals;
    float *max_residuals;          /* device [2]: max return residual, max porosity residual (always) */
} BkDiagnostics;

typedef struct BkFlags {
    int32_t *simulation;           /* [2]: J, stencil (physics/mpm.py:145) */
    int32_t *ding;                 /* [3]: porosity domain, porosity solve, gas CFL (ding.py:232) */
    int32_t *transport;            /* [2]: heat bound, water bound (thermal_water.py:279) */
} BkFlags;

typedef struct BkMlpNorm {
    float in_mean[8], in_scale[8];  /* network input k = (feature k - in_mean[k]) / in_scale[k], k < 7 */
    float out_scale[4];             /* prediction k = network output k * out_scale[k], k < 3 */
} BkMlpNorm;

/* Learned return-map surrogate for the Ding model (no counterpart in the reference). Features of a
   particle: the trial elastic gradient's log singular values (descending), the temperature after
   the gelation latch, water saturation, gas content and log(1 - n0 + n); targets: the change of the
   three log principal strains made by the return (before volume corrections), same order.
   - packed != NULL: the surrogate replaces the return for yielding particles whose features lie in
     [in_low, in_high]; elastic and out-of-range particles keep the exact map.
   - packed == NULL, samples != NULL: exact map; yielding particles with index % sample_stride ==
     sample_offset append rows of 12 floats (7 features, 3 targets, 2 zero) while
     *sample_count < sample_capacity (*sample_count keeps counting past it).
   judge_error (device, may be NULL): max |surrogate - exact| of the log strains over the particles
   with (index / 32) % judge_stride == 0 (whole warps, so the exact map's cost stays on those). path_counts (device [3], may be NULL): += particles that took the
   elastic, surrogate and exact-yielding paths. */
typedef struct BkReturnSurrogate {
    const void *packed;            /* bk_mlp_pack output (16-byte aligned) */
    BkMlpNorm norm;
    float in_low[8], in_high[8];
    float *samples;
    int32_t *sample_count;
    int32_t sample_capacity, sample_stride, sample_offset;
    float *judge_error;
    int32_t judge_stride;
    int32_t *path_counts;
} BkReturnSurrogate;

typedef struct BkSubstepParams {
    int64_t n, pitch;
    int32_t resolution, boundary_cells;
    float origin[3], spacing, time_step, gravity[3];
    int32_t material;              /* 0 neo-Hookean, 1 Ding */
    BkDingParams ding;
    int32_t transport, gas, settling;
    BkScalarParams scalar;
    float conductivity, diffusivity, initial_saturation, water_stress;
    float gas_ambient_pressure, density, elastic_modulus, cfl_limit, gas_peak, gas_width;
    const BkReturnSurrogate *surrogate;  /* NULL: exact return map */
    int32_t keep_transport_fields;  /* 1: the grid update leaves the transport node fields in place
                                       (for bk_transport_adjoint, which clears them) */
    int32_t transport_prescattered; /* 1: this substep's transport node fields (volume, capacity,
                                       energy, water) and their node box (bounds[12..17]) were built by
                                       the previous substep's G2P with transport_prescatter_next; the
                                       scalar P2G kernel is skipped */
    int32_t transport_prescatter_next; /* 1: the G2P kernel also scatters the next substep's transport
                                       node fields from the state it writes, with their box in
                                       bounds[12..17] (grid bounds of 18 ints). Valid only for a next
                                       substep that starts from this output with nothing changed in
                                       between; needs the exact return map (no surrogate). */
    int32_t transport_prescatter_stale; /* 1 with transport_prescattered = 0: fields an earlier G2P
                                       scattered ahead (box in bounds[12..17]) are still on the grid
                                       and are cleared before this substep's scalar P2G */
    int32_t *status;                /* optional (device, 1 int, may be NULL): set to 1 when a kernel gave
                                       up a bounded wait (a bulk copy into shared memory or a
                                       tensor-core completion) and left its particles unprocessed */
} BkSubstepParams;

#define BK_PHASE_TRANSPORT 1       /* surface terms, scalar P2G, diffusion */
#define BK_PHASE_MECHANICS 2       /* scalar G2P + gas/water stress + P2G, grid update, G2P + return map */

/* The fused substep of physics/mpm.py:163-225: reads `in`, writes `out`, uses `grid` as scratch. */
BK_API int bk_substep(const BkSubstepParams *params, const BkState *in, BkState *out, const BkConstants *constants,
                      BkGrid *grid, BkSurface *surface, BkDiagnostics *diagnostics, BkFlags *flags,
                      int32_t phases, void *stream);

/* bk_substep's mechanics phase with the grid held in a fixed array inside this library, for
   callers that must not allocate device memory (code inside an allocator hook, a real-time or
   signal-safe path, or a process that forbids device allocation after start-up): the call
   allocates and frees nothing. It has no counterpart in the reference. Limits: neo-Hookean or
   Ding without transport or gas, grid resolution 4..48 (48^3 nodes, about 3.4 MB held on every
   GPU that loads the library until exit); larger grids return BK_ERR_ARGUMENT with a message.
   Every call looks up the array's device address in the current CUDA context, primary or not.
   Under lazy module loading (the default since CUDA 12.2) the first call in each context loads
   the module, which reserves the array's memory: make that first call at start-up, before any
   stream capture, so that no later call allocates. All calls on a device share the array and
   each call clears it first, so calls that overlap on the GPU race and must be serialised by the
   caller. */
BK_API int bk_substep_static_grid(const BkSubstepParams *params, const BkState *in, BkState *out,
                                  const BkConstants *constants, BkDiagnostics *diagnostics, BkFlags *flags,
                                  void *stream);

/* ---- Batched substeps over an instance table (no counterpart in the reference) ----
   Many independent simulators (own particles, grids, parameters) advanced by ONE launch per stage
   of bk_substep instead of one per stage and simulator: each block of a batched launch finds its
   instance in a device table and runs the plain kernel's body on it. An instance gets the blocks
   its own launch would use (particles, surface vertices, face owners) and, for the node-box passes,
   about one block per 2048 particles. Each instance holds its two ping-pong states: parity 0 steps
   states[0] -> states[1], parity 1 steps states[1] -> states[0]. Instances with transport need
   18-int grid bounds (the transport prescatter) and the surface accumulators of both states, which
   bk_batch_substep advances in its surface kernel (the instances' own accumulate_* fields are
   ignored). An instance
   whose params carry a surrogate runs the surrogate G2P kernel, the others the exact one. The
   transport_prescattered/_next/_stale fields and the phases are ignored in `params`: the flags of
   bk_batch_substep apply to every transport instance without a surrogate, and an instance's
   fields must not be left scattered ahead by an earlier bk_substep (the batch never clears them). */
typedef struct BkBatchInstance {
    BkSubstepParams params;
    BkState states[2];
    double *water_losses[2], *heat_exchanges[2];   /* surface accumulators of states[k] (transport) */
    BkConstants constants;
    BkGrid grid;
    BkSurface surface;
    BkDiagnostics diagnostics;
    BkFlags flags;
} BkBatchInstance;

typedef struct BkBatch BkBatch;

/* Checks every instance as bk_substep would (both parities) and uploads the table (about 1 KB per
   instance and parity, allocated on the current device; the call synchronises). The device
   arrays named by the instances must outlive the batch. */
BK_API int bk_batch_create(const BkBatchInstance *instances, int32_t count, BkBatch **batch);
/* One substep of every instance, 8-10 launches on `stream` (capturable in a CUDA graph). */
BK_API int bk_batch_substep(BkBatch *batch, int32_t parity, int32_t phases, int32_t prescattered,
                            int32_t prescatter_next, void *stream);
BK_API int bk_batch_destroy(BkBatch *batch);

/* Per-kernel timing of the fused entry points with CUDA events on the launching stream.
   bk_profile_start clears old records and starts recording; bk_profile_stop stops;
   bk_profile_report waits for the events and writes, per kernel name (name_capacity bytes each),
   the total milliseconds and launch count. */
BK_API int bk_profile_start(void);
BK_API int bk_profile_stop(void);
/* Record only the kernel named `name` (NULL or "": every kernel). Each recorded launch adds two
   event records to its stream, a few microseconds between kernels. */
BK_API int bk_profile_select(const char *name);
BK_API int bk_profile_report(int32_t max_kernels, char *names, int32_t name_capacity, double *total_ms,
                             int32_t *counts, int32_t *kernel_count);

/* Water-loss and heat-exchange accumulators of the face-owning particles after an accepted substep
   (physics/thermal_water.py:225-226): += time_step * the owner rates bk_substep stored in `surface`. */
BK_API int bk_surface_accumulate(const BkSurface *surface, float time_step, double *water_losses,
                                 double *heat_exchanges, void *stream);

/* Recompute the derivable reference outputs of a state from its primary arrays: plastic gradients
   Fp = Fe^-1 F, material temperature, reference density, yield stress, viscosity, gas pressure,
   saturation and particle mass (any output pointer may be NULL). */
BK_API int bk_materialize(const BkSubstepParams *params, const BkState *state, const BkConstants *constants,
                          float *plastic_gradients, float *material_temperature, float *reference_density,
                          float *yield_stress, float *viscosity, double *gas_pressure, double *saturation,
                          float *particle_mass, void *stream);

/* Adjoint (reverse-mode derivative) of one state of the mechanics substep, in the plane layout of
   BkState. Ding fields may be NULL for the neo-Hookean model. `temperature` is the adjoint of the
   per-particle material temperature, which is constant without transport: the call adds this
   substep's contribution to the incoming value. */
typedef struct BkAdjointState {
    float *x, *v, *C, *F;          /* 3, 3, 9, 9 planes */
    float *Fe, *tau;               /* Ding, 9 planes; with transport tau is dL/d(the stress P2G used) */
    float *porosity;               /* Ding */
    float *temperature;            /* Ding material temperature: accumulated over substeps without
                                      transport; with transport, dL/d(this substep's T_mat), written */
    float *mass;                   /* may be NULL: dL/d(particle mass P2G used), written */
} BkAdjointState;

/* Reverse sweep of one mechanics substep (P2G, grid update, G2P, neo-Hookean stress or the
   Ding return map with its uncoupled or coupled (gas mode) porosity; physics/mpm.py:163-205 with
   transfer.py:37-105, grid.py:20-38, elastic.py:4-26, ding.py:103-221, porous_return.py:43-100). The reference gets these derivatives from Warp's tape replaying
   its kernels' generated adjoints; this entry point replaces that replay for one substep.
   Inputs: the substep's input state `in`, the grid that bk_substep left after running from `in`
   (node_pm, node_v: R^3 float4), and `out_adjoint` = dL/d(output state). Writes
   `in_adjoint` = dL/d(input state); `in_adjoint` may be the same arrays as `out_adjoint`.
   `node_v_adjoint` and `node_pm_adjoint` are R^3 float4 scratch arrays. `node_box` (device, may be
   NULL): that substep's active node box, BkGrid.bounds + 6 after bk_substep returned (inclusive
   lo[3], hi[3]); with it only the box is visited and node_v_adjoint is left zero, so it must be
   zero before the first call; without it node_v_adjoint is cleared and the whole grid visited. `parameter_adjoint`
   (device, float64, may be NULL) accumulates dL/d(shear modulus), dL/d(Lame lambda) and
   dL/d(viscosity parameter). The coupled porosity solve is reversed through its converged
   consistency equation (the derivative of the reference's SolvePorosityGradient). On a transport
   substep `in` carries the stress and material temperature, and `constants` the particle mass,
   that bk_transport_adjoint_prepare produced; `in_adjoint->mass` receives dL/d(particle mass) and
   `in_adjoint->temperature` dL/d(material temperature); bk_transport_adjoint then finishes the
   substep. */
BK_API int bk_substep_adjoint(const BkSubstepParams *params, const BkState *in, const BkConstants *constants,
                              const float *node_pm, const float *node_v, const int32_t *node_box,
                              const BkAdjointState *out_adjoint, BkAdjointState *in_adjoint, float *node_v_adjoint,
                              float *node_pm_adjoint, double *parameter_adjoint, void *stream);

/* ---- Return-map surrogate MLP (7 -> 64 -> 64 -> 3, SiLU; BF16 weights, FP32 accumulation) ----
   The reference has no learned component; these entry points serve the surrogate that may replace
   the Ding return map (ding.py:103-137 with porous_return.py:43-61) for in-distribution particles.
   Parameters are an FP32 vector of BK_MLP_PARAMS values: W1[7][64], b1[64], W2[64][64], b2[64],
   W3[64][3], b3[3] (input x output, row-major). Inference reads them packed by bk_mlp_pack into
   BK_MLP_PACKED_BYTES bytes (16-byte aligned): BF16 tensor-core operands plus FP32 biases. */
#define BK_MLP_PARAMS 4867
#define BK_MLP_PACKED_BYTES 12864

/* BkMlpNorm is declared with BkReturnSurrogate above. */

/* outputs[i*4 + k] (k < 3) for the raw features[i*8 + k] (k < 7), on the tensor cores. *status
   (device) is set to 1 if a tensor-core completion wait gave up. */
BK_API int bk_mlp_infer(int64_t n, const float *features, const BkMlpNorm *norm, const void *packed,
                        float *outputs, int32_t *status, void *stream);
/* grads += dL/dparams of L = mean over the batch and the 3 outputs of (prediction/out_scale -
   target/out_scale)^2, with the forward rounded like inference (BF16 inputs, weights and hidden
   activations; FP32 accumulation); *loss_sum (device, may be NULL) += sum of squared errors. */
BK_API int bk_mlp_gradient(int64_t batch, const float *features, const float *targets, const BkMlpNorm *norm,
                           const float *params, float *grads, double *loss_sum, void *stream);
/* One Adam step (bias-corrected, `step` >= 1) on the parameter vector. */
BK_API int bk_mlp_adam(const float *grads, float *params, float *first_moment, float *second_moment, int32_t step,
                       float learning_rate, float beta1, float beta2, float epsilon, void *stream);
/* FP32 parameters -> packed BF16 operands + FP32 biases for bk_mlp_infer and the fused substep. */
BK_API int bk_mlp_pack(const float *params, void *packed, void *stream);

/* Transport half of the reverse sweep of one substep (Ding with thermal-water transport, with or
   without gas): the surface heat/loss terms with their face areas, the scalar P2G, the diffusion
   stencil, the scalar G2P, the water stress and the water-dependent mass
   (physics/thermal_water.py:77-253) and, with gas, the local gas source and the gas-pressure
   stress (thermal_water.py:232-245, physics/materials/gas.py:16-35), reversed. Node arrays are R^3
   (node_dT_ratio: double2); all start at zero and are left at zero; vertices: 3 planes of the
   surface's vertex_pitch, zero on entry, left zero. */
typedef struct BkAdjointTransport {
    const double *temperature_out, *water_out;  /* dL/d(T', W') of the substep's output */
    double *temperature_in, *water_in;          /* dL/d(T, W) of its input (may alias the above) */
    double *node_dT_ratio;                      /* node adjoint scratch of (dT, dW/W) */
    double *node_fields[6];                     /* node adjoint scratch: volume, capacity, energy, water,
                                                   heat, loss */
    double *vertices;                           /* surface-vertex adjoint scratch */
    double *heat_parameter;                     /* device [1], may be NULL: += dL/d(heat transfer) */
    const double *gas_moles_out;                /* gas mode: dL/dN' of the substep's output */
    double *gas_moles_in;                       /* gas mode: dL/dN of its input (may alias the above) */
    double *gas_rate;                           /* gas mode, may be NULL: += dL/d(gas source rate), one
                                                   entry per entry of BkConstants.gas_rate */
} BkAdjointTransport;

/* Before bk_substep_adjoint on a transport substep: the material temperature T + sum w dT, the
   particle mass dry + W', and the stress tau + J (p_amb - p_gas) I - J c (s - s0) I (the gas term
   in gas mode) that the forward P2G and return map used, from the substep's input state and node
   (dT, dW/W) (n entries; stress: 9 planes). */
BK_API int bk_transport_adjoint_prepare(const BkSubstepParams *params, const BkState *in,
                                        const BkConstants *constants, const double *node_dT_ratio,
                                        float *material_temperature, float *mass, float *stress, void *stream);
/* After bk_substep_adjoint (whose tau, mass and temperature outputs are `mechanics`' inputs here,
   and whose x and F outputs receive the transport terms): `grid` is the substep's forward grid run
   with keep_transport_fields = 1, whose transport fields this call clears over the box in
   grid->bounds + 6; `surface` the BkSurface of that substep, whose `vertices` this call rewrites
   with the substep's mesh vertex positions (as the forward transport phase computed them). */
BK_API int bk_transport_adjoint(const BkSubstepParams *params, const BkState *in, const BkConstants *constants,
                                const BkGrid *grid, const BkSurface *surface, const BkAdjointState *mechanics,
                                BkAdjointTransport *adjoint, void *stream);

/* The recorder's per-step measurements (experiments/recording.py:46-112, SimulationRecorder.Measure)
   as one device reduction over the particles, mesh vertices and tets, in place of pulling every
   array to the host. Arrays are in plane layout with `pitch` (vertices: `vertex_pitch`); groups
   whose pointers are NULL are skipped and their slots left 0. `regions` marks particles: bit 0 a
   surface-face owner, bit 1 the initial core. */
typedef struct BkMeasureInputs {
    int64_t n, pitch;
    const float *F;                              /* 9 planes */
    const float *reference_volume;               /* n */
    const float *material_temperature, *porosity; /* Ding */
    const int32_t *gelled;                       /* Ding */
    const double *gas_moles, *gas_pressure;      /* gas mode */
    const double *temperature, *water, *saturation, *water_losses, *heat_exchanges, *capacity; /* transport */
    const uint8_t *regions;                      /* transport */
    int64_t vertex_count, vertex_pitch;
    const float *vertices;                       /* 3 planes */
    int64_t tet_count;
    const int32_t *tets;                         /* tet_count x 4 */
} BkMeasureInputs;

/* Slots of bk_measure_state's output (float64). */
enum {
    BK_MEASURE_PARTICLE_VOLUME = 0,  /* sum V0 det F */
    BK_MEASURE_INVALID_PARTICLES,    /* count det F <= 0 */
    BK_MEASURE_NONFINITE,            /* count of particles or vertices with a nonfinite F or position */
    BK_MEASURE_MATERIAL_T_SUM,       /* Ding: sum of the material temperatures */
    BK_MEASURE_POROSITY_SUM, BK_MEASURE_POROSITY_MIN, BK_MEASURE_POROSITY_MAX,
    BK_MEASURE_GELLED,               /* count of gelled particles */
    BK_MEASURE_GAS_TOTAL,            /* sum V0 N */
    BK_MEASURE_PRESSURE_SUM, BK_MEASURE_PRESSURE_MIN, BK_MEASURE_PRESSURE_MAX,
    BK_MEASURE_PORE_VOLUME,          /* sum V0 det F n */
    BK_MEASURE_T_MIN, BK_MEASURE_T_MAX,
    BK_MEASURE_ENERGY,               /* sum c T */
    BK_MEASURE_CAPACITY,             /* sum c */
    BK_MEASURE_SURFACE_T_SUM, BK_MEASURE_SURFACE_COUNT, BK_MEASURE_CORE_T_SUM, BK_MEASURE_CORE_COUNT,
    BK_MEASURE_WATER, BK_MEASURE_WATER_LOST, BK_MEASURE_HEAT_EXCHANGE,
    BK_MEASURE_SATURATION_SUM, BK_MEASURE_SATURATION_MIN, BK_MEASURE_SATURATION_MAX,
    BK_MEASURE_X_MIN, BK_MEASURE_Y_MIN, BK_MEASURE_Z_MIN, BK_MEASURE_X_MAX, BK_MEASURE_Y_MAX, BK_MEASURE_Z_MAX,
    BK_MEASURE_MESH_VOLUME,          /* sum |signed tet volume| */
    BK_MEASURE_INVERTED_TETS,        /* count signed volume <= 0 */
    BK_MEASURE_SLOTS
};
#define BK_MEASURE_BLOCKS 296        /* partial results per slot held in `scratch` */

/* out: BK_MEASURE_SLOTS doubles (device); scratch: BK_MEASURE_BLOCKS * BK_MEASURE_SLOTS doubles
   (device). Deterministic: fixed grid, per-block partials reduced in a fixed order. */
BK_API int bk_measure_state(const BkMeasureInputs *in, double *out, double *scratch, void *stream);

/* A substep's result for a caller that reads one back per step (no counterpart in the reference,
   whose callers pull whole arrays): out[0] = grid mass of the last substep (node masses over the
   active box in grid->bounds + 6), out[1] = particle kinetic energy sum 1/2 m |v|^2 of `state`
   (m = dry + W with transport, else constants->mass). out: 2 doubles, scratch: 2 *
   BK_MEASURE_BLOCKS doubles (device). Deterministic. */
BK_API int bk_step_summary(const BkSubstepParams *params, const BkState *state, const BkConstants *constants,
                           const BkGrid *grid, double *out, double *scratch, void *stream);

/* ---- particle order (no counterpart in the reference, whose Warp kernels read particles in
   sample order) ---- */

/* Device bytes of `scratch` that bk_sort_by_cell needs for n particles on an R^3 grid; -1 with
   an error message on bad arguments. Host call, no launch. */
BK_API int64_t bk_sort_by_cell_scratch_bytes(int64_t n, int32_t resolution);

/* order[k] = index of the particle that goes to position k: particles grouped by quadratic stencil
   base floor((x - origin)/dx - 0.5), the bases in Morton order, particles of one base in their
   current relative order (stable); particles whose stencil leaves the grid go last. x: 3 planes
   of `pitch`; origin: 3 floats in HOST memory; order: n int32 (device); scratch: device, 256-byte
   aligned, at least bk_sort_by_cell_scratch_bytes(n, resolution) bytes. */
BK_API int bk_sort_by_cell(int64_t n, int64_t pitch, const float *x, const float *origin, float dx,
                           int32_t resolution, int32_t *order, void *scratch, int64_t scratch_bytes, void *stream);

/* CheckState (physics/mpm.py:243-308 with physics/materials/ding.py:294-301) as one device
   reduction: the particle-state checks, the inputs of the CFL estimate and the values CheckState
   returns, plus copies of the simulation, Ding and transport flag words, in BK_CHECK_SLOTS doubles. The host
   raises the reference's messages from them after one small device-to-host copy. */
enum {
    BK_CHECK_SIM_FLAG0 = 0, BK_CHECK_SIM_FLAG1,      /* simulation flags [0] (J), [1] (stencil) */
    BK_CHECK_DING_FLAG0, BK_CHECK_DING_FLAG1, BK_CHECK_DING_FLAG2,  /* Ding flags (porosity, return, gas CFL) */
    BK_CHECK_TRANSPORT_FLAG0, BK_CHECK_TRANSPORT_FLAG1,             /* transport flags (heat, water stability) */
    BK_CHECK_NONFINITE_STATE,        /* particles with a nonfinite x, v, F or C */
    BK_CHECK_J_MIN, BK_CHECK_J_MAX,  /* det F in float64 */
    BK_CHECK_OUTSIDE_STENCIL,        /* particles with a grid coordinate < 0.5 or >= R - 1.5 */
    BK_CHECK_SPEED_MAX,              /* max |v| */
    BK_CHECK_GAS_WAVE_MAX,           /* gas mode: max sqrt((K + p (1 + (1 - n0 + n) / n)) J / rho_ref) */
    BK_CHECK_WATER_WAVE2_MAX,        /* transport with water: max water_stress s J / rho_ref */
    BK_CHECK_NONFINITE_DING,         /* Ding: particles with a nonfinite Fe or Fp = Fe^-1 F */
    BK_CHECK_RESIDUAL_MAX,           /* Ding: largest return residual */
    BK_CHECK_PARTICLE_VOLUME,        /* sum V0 det F */
    BK_CHECK_TOTAL_MASS,             /* sum of particle masses */
    BK_CHECK_KINETIC_ENERGY,         /* sum 1/2 m |v|^2 */
    BK_CHECK_GRID_MASS,              /* node masses of the last substep's active box */
    BK_CHECK_NONFINITE_VERTICES,     /* mesh vertices with a nonfinite coordinate */
    BK_CHECK_INVERTED_TETS,          /* tets with signed volume <= 0 (or a vertex index out of range) */
    BK_CHECK_SUBSTEP_STATUS,         /* BkSubstepParams.status (a bounded wait gave up) */
    BK_CHECK_SLOTS
};

typedef struct {
    int64_t n, pitch;
    const float *x, *v, *F, *C;           /* state planes (device) */
    const float *reference_volume;        /* V0 */
    const float *mass;                    /* particle masses without transport, else NULL */
    const double *dry_mass, *water;       /* transport: mass = dry + W, rho_ref = mass / V0 */
    const double *temperature;            /* transport temperatures (gas pressure), else NULL */
    const float *material_temperature;    /* Ding without transport (gas pressure), else NULL */
    const float *Fe;                      /* Ding elastic gradients, else NULL */
    const float *porosity;                /* gas mode, else NULL */
    const double *gas_moles;              /* gas mode, else NULL */
    const float *return_residuals;        /* per-particle residuals, or NULL */
    const float *max_residuals;           /* the substep's max residual (1 float), or NULL */
    const int32_t *sim_flags;             /* 2 ints */
    const int32_t *ding_flags;            /* 3 ints, or NULL */
    const int32_t *transport_flags;       /* 2 ints, or NULL */
    float origin[3], spacing;
    int32_t resolution;
    int32_t water_enabled;
    float density, water_density, water_stress, gas_modulus, initial_porosity;  /* gas_modulus = lambda + 2 mu */
    const float *node_pm;                 /* grid (px, py, pz, m) float4 nodes, or NULL */
    const int32_t *box;                   /* the last substep's active box (6 ints: lo, hi) */
    int64_t vertex_count, vertex_pitch;
    const float *vertices;                /* 3 planes of vertex_pitch floats */
    int64_t tet_count;
    const int32_t *tets;                  /* tet_count x 4 vertex ids */
    const int32_t *substep_status;        /* BkSubstepParams.status, or NULL */
} BkCheckInputs;

/* out: BK_CHECK_SLOTS doubles (device); scratch: BK_MEASURE_BLOCKS * BK_CHECK_SLOTS doubles (device).
   Two launches (block partials, then a fixed-order finish), deterministic. */
BK_API int bk_check_state(const BkCheckInputs *in, double *out, double *scratch, void *stream);

/* One per-particle array for bk_permute_particles: `planes` planes of n elements of
   `element_bytes` (4 or 8) bytes, `pitch` elements apart, starting at `data` (device). */
typedef struct {
    void *data;
    int64_t pitch;
    int32_t planes;
    int32_t element_bytes;
} BkParticleArray;

/* In place, for every array: element k of each plane becomes the element order[k] had. `arrays`
   is a HOST table of `array_count` entries, each array aligned to its element size; order: n
   int32 (device), a permutation, so n <= INT32_MAX; scratch: device, 256-byte aligned, at least
   planes * n * element_bytes bytes of the largest array. Arrays must not overlap one another.
   Consecutive arrays are permuted in groups whose slices (each rounded up to 256 bytes) fit the
   scratch buffer: one gather launch and one copy-back launch per group, in order on `stream`, so
   a scratch buffer as large as all the arrays together takes two launches in all. */
BK_API int bk_permute_particles(int64_t n, const int32_t *order, int32_t array_count, const BkParticleArray *arrays,
                                void *scratch, int64_t scratch_bytes, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* BAKING_B200_H */
