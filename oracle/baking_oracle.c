/*
 * CPU ORACLE for the MLS-MPM baking substep -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of every Warp kernel on the reference's substep path,
 * written op by op in the reference's precisions (float32 where the Warp kernel
 * uses `float`, float64 where it uses `wp.float64`) and in its layouts
 * (vec3 = 3 floats, mat33 = 9 floats row-major, array-of-structures).
 * Each function cites the reference file:line it restates.
 *
 * Only the tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg call
 * this library, and only as the checker. The product (baking_b200/) never loads it.
 *
 * Pinning: the reference cannot run here (its Warp dependency is absent), so this
 * restatement is pinned against the known answers held by the reference's own
 * tests (tests/test_mpm.py, test_ding.py, test_ding_thermal.py, test_transport.py,
 * test_gas.py, test_elastic_material.py, test_mesh_reconstruction.py), restated in
 * tests/test_oracle_*.py. Bit-level agreement with Warp's own svd3 and its
 * float32 transcendental builtins is not pinned: the 3x3 SVD below is our own
 * one-sided Jacobi method (Hestenes 1958), and the math functions are the C
 * library's.
 *
 * Particle loops run in index order when ora_set_threads(1) (the parity mode, the
 * order a single-threaded CPU launch uses); with more threads the scatters use
 * OpenMP atomics, which is how the CPU baseline is timed.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORA_API __attribute__((visibility("default")))

static int g_threads = 1;

ORA_API void ora_set_threads(int threads) {
    g_threads = threads < 1 ? 1 : threads;
#ifdef _OPENMP
    omp_set_num_threads(g_threads);
#endif
}

ORA_API int ora_get_max_threads(void) {
#ifdef _OPENMP
    return omp_get_num_procs();
#else
    return 1;
#endif
}

#define PAR_FOR _Pragma("omp parallel for schedule(static) if(g_threads > 1)")
#define ATOMIC _Pragma("omp atomic")

static inline void flag_set(int *flags, int index) {
#pragma omp atomic write
    flags[index] = 1;
}

/* ---------------------------------------------------------------- helpers */

static inline float det3f(const float *m) {
    return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6])
         + m[2] * (m[3] * m[7] - m[4] * m[6]);
}

static inline double det3d(const double *m) {
    return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6])
         + m[2] * (m[3] * m[7] - m[4] * m[6]);
}

static inline void matmul3f(const float *a, const float *b, float *out) {
    float r[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            r[3 * i + j] = a[3 * i] * b[j] + a[3 * i + 1] * b[3 + j] + a[3 * i + 2] * b[6 + j];
    memcpy(out, r, sizeof r);
}

/* Inverse by adjugate / determinant (float32). */
static inline void inverse3f(const float *m, float *out) {
    float d = det3f(m);
    float inv = 1.0f / d;
    float r[9];
    r[0] = (m[4] * m[8] - m[5] * m[7]) * inv;
    r[1] = (m[2] * m[7] - m[1] * m[8]) * inv;
    r[2] = (m[1] * m[5] - m[2] * m[4]) * inv;
    r[3] = (m[5] * m[6] - m[3] * m[8]) * inv;
    r[4] = (m[0] * m[8] - m[2] * m[6]) * inv;
    r[5] = (m[2] * m[3] - m[0] * m[5]) * inv;
    r[6] = (m[3] * m[7] - m[4] * m[6]) * inv;
    r[7] = (m[1] * m[6] - m[0] * m[7]) * inv;
    r[8] = (m[0] * m[4] - m[1] * m[3]) * inv;
    memcpy(out, r, sizeof r);
}

/*
 * 3x3 SVD A = U diag(s) V^T in float64 by one-sided Jacobi rotations
 * (Hestenes 1958): plane rotations applied on the right orthogonalise the
 * columns of A; the column norms are the singular values. s >= 0; U and V are
 * orthogonal. Used where the reference calls wp.svd3 on a mat33d
 * (physics/materials/ding.py:106,179). The return map only uses U f(s) V^T and
 * U g(s) U^T, which do not depend on the SVD's ordering or sign conventions.
 */
ORA_API void ora_svd3(const double *A, double *U, double *s, double *V) {
    double b[9];
    memcpy(b, A, sizeof b);
    double v[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    static const int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
    for (int sweep = 0; sweep < 40; ++sweep) {
        int rotated = 0;
        for (int k = 0; k < 3; ++k) {
            int p = pairs[k][0], q = pairs[k][1];
            double alpha = 0, beta = 0, gamma = 0;
            for (int r = 0; r < 3; ++r) {
                alpha += b[3 * r + p] * b[3 * r + p];
                beta += b[3 * r + q] * b[3 * r + q];
                gamma += b[3 * r + p] * b[3 * r + q];
            }
            if (gamma == 0.0 || fabs(gamma) <= 1e-15 * sqrt(alpha * beta)) continue;
            rotated = 1;
            double zeta = (beta - alpha) / (2.0 * gamma);
            double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
            double c = 1.0 / sqrt(1.0 + t * t);
            double sn = c * t;
            for (int r = 0; r < 3; ++r) {
                double bp = b[3 * r + p], bq = b[3 * r + q];
                b[3 * r + p] = c * bp - sn * bq;
                b[3 * r + q] = sn * bp + c * bq;
                double vp = v[3 * r + p], vq = v[3 * r + q];
                v[3 * r + p] = c * vp - sn * vq;
                v[3 * r + q] = sn * vp + c * vq;
            }
        }
        if (!rotated) break;
    }
    int zero[3];
    for (int c = 0; c < 3; ++c) {
        double n = sqrt(b[c] * b[c] + b[3 + c] * b[3 + c] + b[6 + c] * b[6 + c]);
        s[c] = n;
        zero[c] = !(n > 1e-300);
        for (int r = 0; r < 3; ++r) U[3 * r + c] = zero[c] ? 0.0 : b[3 * r + c] / n;
    }
    /* Complete U for rank-deficient input so it stays orthogonal. */
    for (int c = 0; c < 3; ++c) {
        if (!zero[c]) continue;
        int a = (c + 1) % 3, d = (c + 2) % 3;
        double ua[3] = {U[a], U[3 + a], U[6 + a]}, ud[3] = {U[d], U[3 + d], U[6 + d]};
        if (zero[a]) { ua[0] = (fabs(ud[0]) < 0.9) ? 1 : 0; ua[1] = 1 - ua[0]; ua[2] = 0;
            double dp = ua[0] * ud[0] + ua[1] * ud[1] + ua[2] * ud[2];
            for (int r = 0; r < 3; ++r) ua[r] -= dp * ud[r];
            double n = sqrt(ua[0] * ua[0] + ua[1] * ua[1] + ua[2] * ua[2]);
            for (int r = 0; r < 3; ++r) { ua[r] /= n; U[3 * r + a] = ua[r]; }
            zero[a] = 0; }
        double cr[3] = {ua[1] * ud[2] - ua[2] * ud[1], ua[2] * ud[0] - ua[0] * ud[2], ua[0] * ud[1] - ua[1] * ud[0]};
        for (int r = 0; r < 3; ++r) U[3 * r + c] = cr[r];
        zero[c] = 0;
    }
    memcpy(V, v, sizeof v);
}

/* ------------------------------------------------- physics/transfer.py:4-33 */

ORA_API float ora_quadratic_weight(float l, int i) {
    if (i == 0) return 0.5f * (1.5f - l) * (1.5f - l);
    if (i == 1) return 0.75f - (l - 1.0f) * (l - 1.0f);
    return 0.5f * (l - 0.5f) * (l - 0.5f);
}

static inline void stencil_base(const float *g, int *b) {
    for (int a = 0; a < 3; ++a) b[a] = (int)floorf(g[a] - 0.5f);
}

static inline int valid_stencil(const int *b, int R) {
    return b[0] >= 0 && b[1] >= 0 && b[2] >= 0 && b[0] + 2 < R && b[1] + 2 < R && b[2] + 2 < R;
}

static inline int64_t flatten_node(int i, int j, int k, int R) {
    return ((int64_t)i * R + j) * R + k;
}

/* --------------------------------------- physics/transfer.py:36-70 (P2G) */
ORA_API void ora_particle_to_grid(int n, const float *x, const float *v, const float *C, const float *tau,
                                  const float *mass, const float *V0, float *node_m, float *node_p,
                                  const float *origin, float dx, int R, float dt, int *flags) {
    PAR_FOR
    for (int i = 0; i < n; ++i) {
        float g[3];
        for (int a = 0; a < 3; ++a) g[a] = (x[3 * i + a] - origin[a]) / dx;
        int b[3];
        stencil_base(g, b);
        if (!valid_stencil(b, R)) { flag_set(flags, 1); continue; }
        float l[3] = {g[0] - (float)b[0], g[1] - (float)b[1], g[2] - (float)b[2]};
        float m = mass[i];
        float scale = dt * V0[i] * 4.0f / (dx * dx);
        float A[9];
        for (int e = 0; e < 9; ++e) A[e] = m * C[9 * i + e] - scale * tau[9 * i + e];
        for (int ox = 0; ox < 3; ++ox)
            for (int oy = 0; oy < 3; ++oy)
                for (int oz = 0; oz < 3; ++oz) {
                    float w = ora_quadratic_weight(l[0], ox) * ora_quadratic_weight(l[1], oy)
                            * ora_quadratic_weight(l[2], oz);
                    int64_t node = flatten_node(b[0] + ox, b[1] + oy, b[2] + oz, R);
                    float d[3] = {((float)ox - l[0]) * dx, ((float)oy - l[1]) * dx, ((float)oz - l[2]) * dx};
                    float mom[3];
                    for (int r = 0; r < 3; ++r)
                        mom[r] = w * (m * v[3 * i + r] + (A[3 * r] * d[0] + A[3 * r + 1] * d[1] + A[3 * r + 2] * d[2]));
                    float wm = w * m;
                    ATOMIC node_m[node] += wm;
                    ATOMIC node_p[3 * node + 0] += mom[0];
                    ATOMIC node_p[3 * node + 1] += mom[1];
                    ATOMIC node_p[3 * node + 2] += mom[2];
                }
    }
}

/* ------------------------------------------------ physics/grid.py:20-38 */
ORA_API void ora_update_grid(int64_t node_count, const float *node_m, const float *node_p, float *node_v,
                             int R, int boundary_cells, const float *gravity, float dt) {
    PAR_FOR
    for (int64_t i = 0; i < node_count; ++i) {
        if (!(node_m[i] > 0.0f)) continue;
        float vel[3];
        for (int a = 0; a < 3; ++a) vel[a] = node_p[3 * i + a] / node_m[i] + dt * gravity[a];
        int c[3] = {(int)(i / ((int64_t)R * R)), (int)((i / R) % R), (int)(i % R)};
        for (int a = 0; a < 3; ++a) {
            if (c[a] < boundary_cells && vel[a] < 0.0f) vel[a] = 0.0f;
            if (c[a] >= R - boundary_cells && vel[a] > 0.0f) vel[a] = 0.0f;
        }
        for (int a = 0; a < 3; ++a) node_v[3 * i + a] = vel[a];
    }
}

/* -------------------------------------- physics/transfer.py:73-109 (G2P) */
ORA_API void ora_grid_to_particle(int n, const float *x_in, const float *F_in, const float *node_v,
                                  float *x_out, float *v_out, float *C_out, float *F_out,
                                  const float *origin, float dx, int R, float dt, int *flags) {
    PAR_FOR
    for (int i = 0; i < n; ++i) {
        float g[3];
        for (int a = 0; a < 3; ++a) g[a] = (x_in[3 * i + a] - origin[a]) / dx;
        int b[3];
        stencil_base(g, b);
        if (!valid_stencil(b, R)) { flag_set(flags, 1); continue; }
        float l[3] = {g[0] - (float)b[0], g[1] - (float)b[1], g[2] - (float)b[2]};
        float nv[3] = {0, 0, 0}, nc[9] = {0};
        float k = 4.0f / (dx * dx);
        for (int ox = 0; ox < 3; ++ox)
            for (int oy = 0; oy < 3; ++oy)
                for (int oz = 0; oz < 3; ++oz) {
                    float w = ora_quadratic_weight(l[0], ox) * ora_quadratic_weight(l[1], oy)
                            * ora_quadratic_weight(l[2], oz);
                    int64_t node = flatten_node(b[0] + ox, b[1] + oy, b[2] + oz, R);
                    float d[3] = {((float)ox - l[0]) * dx, ((float)oy - l[1]) * dx, ((float)oz - l[2]) * dx};
                    const float *u = node_v + 3 * node;
                    for (int r = 0; r < 3; ++r) nv[r] = nv[r] + w * u[r];
                    float kw = k * w;
                    for (int r = 0; r < 3; ++r)
                        for (int c = 0; c < 3; ++c) nc[3 * r + c] = nc[3 * r + c] + kw * (u[r] * d[c]);
                }
        float xin[3] = {x_in[3 * i], x_in[3 * i + 1], x_in[3 * i + 2]};
        float Fi[9];
        memcpy(Fi, F_in + 9 * i, sizeof Fi);
        for (int r = 0; r < 3; ++r) v_out[3 * i + r] = nv[r];
        memcpy(C_out + 9 * i, nc, sizeof nc);
        for (int r = 0; r < 3; ++r) x_out[3 * i + r] = xin[r] + dt * nv[r];
        float G[9];
        for (int e = 0; e < 9; ++e) G[e] = dt * nc[e] + ((e % 4) == 0 ? 1.0f : 0.0f);
        matmul3f(G, Fi, F_out + 9 * i);
    }
}

/* ------------------------------- physics/materials/elastic.py:4-26 */
ORA_API void ora_compute_elastic_stress(int n, const float *F, float *tau, float mu, float lam, int *flags) {
    PAR_FOR
    for (int i = 0; i < n; ++i) {
        const float *f = F + 9 * i;
        float J = det3f(f);
        if (!isfinite(J) || J <= 0.0f) {
            flag_set(flags, 0);
            for (int e = 0; e < 9; ++e) tau[9 * i + e] = 0.0f;
            continue;
        }
        float logJ = logf(J);
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                float ffT = f[3 * r] * f[3 * c] + f[3 * r + 1] * f[3 * c + 1] + f[3 * r + 2] * f[3 * c + 2];
                float id = r == c ? 1.0f : 0.0f;
                tau[9 * i + 3 * r + c] = mu * (ffT - id) + lam * logJ * id;
            }
    }
}

/* ------------------------------- physics/materials/ding.py:56-100 */
ORA_API float ora_temperature_factor(float T, const float *knots, const float *factors) {
    float f = factors[0];
    for (int k = 0; k < 3; ++k) {
        if (T >= knots[k]) {
            float frac = fminf((T - knots[k]) / (knots[k + 1] - knots[k]), 1.0f);
            f = (1.0f - frac) * factors[k] + frac * factors[k + 1];
        }
    }
    return f;
}

ORA_API float ora_porosity_coefficient(float n) {
    float c = 0.0f;
    if (n > 0.0f) c = 9.0f / (4.0f * powf(logf(1.0f / n), 2.0f) * (3.5f * n + 1.0f));
    return c;
}

ORA_API float ora_solve_overstress(float q2, float p2, float d, float h) {
    float r = 0.0f;
    if (q2 + p2 > 1.0f) {
        for (int it = 0; it < 32; ++it) {
            float dd = 1.0f + d * r, md = 1.0f + h * r;
            float res = r + 1.0f - q2 / powf(dd, 2.0f) - p2 / powf(md, 2.0f);
            float der = 1.0f + 2.0f * d * q2 / powf(dd, 3.0f) + 2.0f * h * p2 / powf(md, 3.0f);
            r = r - res / der;
        }
    }
    return r;
}

/* ---------------------------- physics/materials/porous_return.py:11-61 */
ORA_API double ora_pressure_coefficient64(double n) {
    double c = 0.0;
    if (n > 0.0) c = 9.0 / (4.0 * pow(log(1.0 / n), 2.0) * (3.5 * n + 1.0));
    return c;
}

ORA_API double ora_overstress64(double q, double p, double d, double h) {
    double r = 0.0;
    if (q + p > 1.0) {
        for (int it = 0; it < 48; ++it) {
            double u = 1.0 + d * r, v = 1.0 + h * r;
            double res = r + 1.0 - q / (u * u) - p / (v * v);
            double der = 1.0 + 2.0 * d * q / pow(u, 3.0) + 2.0 * h * p / pow(v, 3.0);
            r -= res / der;
            if (fabs(res) < 1.0e-12) break;
        }
    }
    return r;
}

ORA_API double ora_porosity_prediction(double n, float q, float p, float d, float h, float e, double Vp,
                                       float n0) {
    double a = ora_pressure_coefficient64(n);
    double r = ora_overstress64((double)q, a * (double)p, (double)d, (double)h * a);
    double den = 1.0 + (double)h * a * r;
    return Vp * exp((double)e * (1.0 - 1.0 / den)) - 1.0 + (double)n0;
}

ORA_API float ora_solve_porosity(float q, float p, float d, float h, float e, double Vp, float n0) {
    double trial = Vp - 1.0 + (double)n0;
    if (trial > 0.0 && trial < 1.0) {
        double a = ora_pressure_coefficient64(trial);
        if ((double)q + a * (double)p <= 1.0) return (float)trial;
    }
    double lo = 0.0, hi = 1.0 - 1.0e-9;
    for (int it = 0; it < 64; ++it) {
        double mid = (lo + hi) * 0.5;
        double pred = ora_porosity_prediction(mid, q, p, d, h, e, Vp, n0);
        if (mid < pred) lo = mid; else hi = mid;
    }
    return (float)((lo + hi) * 0.5);
}

/* ------------------------------- physics/materials/ding.py:103-137 */
ORA_API void ora_ding_return(const float *trial, float mu, float lam, float ty, float eta, float a, float dt,
                             const double *svd_U, const double *svd_s, const double *svd_V,
                             float *Fe_out, float *tau_out, float *residual_out) {
    double Ud[9], sd[3], Vd[9];
    if (svd_U) { memcpy(Ud, svd_U, sizeof Ud); memcpy(sd, svd_s, sizeof sd); memcpy(Vd, svd_V, sizeof Vd); }
    else {
        double Ad[9];
        for (int e = 0; e < 9; ++e) Ad[e] = (double)trial[e];
        ora_svd3(Ad, Ud, sd, Vd);
    }
    float U[9], V[9], s[3];
    for (int e = 0; e < 9; ++e) { U[e] = (float)Ud[e]; V[e] = (float)Vd[e]; }
    for (int k = 0; k < 3; ++k) s[k] = (float)sd[k];
    float eps[3] = {logf(s[0]), logf(s[1]), logf(s[2])};
    float tr = eps[0] + eps[1] + eps[2];
    float ts[3];
    for (int k = 0; k < 3; ++k) ts[k] = 2.0f * mu * eps[k] + lam * tr * 1.0f;
    float mean = (ts[0] + ts[1] + ts[2]) / 3.0f;
    float dev[3] = {ts[0] - mean, ts[1] - mean, ts[2] - mean};
    float q2 = 1.5f * (dev[0] * dev[0] + dev[1] * dev[1] + dev[2] * dev[2]) / (ty * ty);
    float p2 = a * mean * mean / (ty * ty);
    float df = 6.0f * mu * dt * ty * ty / eta;
    float mf = 2.0f * a / 3.0f * (2.0f * mu + 3.0f * lam) * dt * ty * ty / eta;
    float r = ora_solve_overstress(q2, p2, df, mf);
    float cs[3];
    for (int k = 0; k < 3; ++k) cs[k] = dev[k] / (1.0f + df * r) + mean / (1.0f + mf * r) * 1.0f;
    float cm = (cs[0] + cs[1] + cs[2]) / 3.0f;
    float ce[3];
    for (int k = 0; k < 3; ++k) ce[k] = (cs[k] - cm) / (2.0f * mu) + cm / (2.0f * mu + 3.0f * lam) * 1.0f;
    float ex[3] = {expf(ce[0]), expf(ce[1]), expf(ce[2])};
    float Fe[9], tau[9];
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) {
            Fe[3 * i + k] = (U[3 * i] * ex[0]) * V[3 * k] + (U[3 * i + 1] * ex[1]) * V[3 * k + 1]
                          + (U[3 * i + 2] * ex[2]) * V[3 * k + 2];
            tau[3 * i + k] = (U[3 * i] * cs[0]) * U[3 * k] + (U[3 * i + 1] * cs[1]) * U[3 * k + 1]
                           + (U[3 * i + 2] * cs[2]) * U[3 * k + 2];
        }
    if (a == 0.0f) {
        float scale = powf(det3f(trial) / det3f(Fe), 1.0f / 3.0f);
        for (int e = 0; e < 9; ++e) Fe[e] = Fe[e] * scale;
    }
    float res = 0.0f;
    if (q2 + p2 > 1.0f)
        res = fabsf(r + 1.0f - q2 / powf(1.0f + df * r, 2.0f) - p2 / powf(1.0f + mf * r, 2.0f));
    memcpy(Fe_out, Fe, sizeof Fe);
    memcpy(tau_out, tau, sizeof tau);
    *residual_out = res;
}

/* ------------------------------- physics/materials/ding.py:140-221 */
typedef struct {
    int coupled_porosity, temperature_enabled;
    float mu, lam, yield_stress, initial_porosity, dt;
    float knots[4], yield_factors[4], viscosity_factors[4];
} OraDingParams;

ORA_API void ora_update_ding(int n, const float *Fe_old, const float *n_old, const int *gelled_old,
                             const float *F_tot, const float *C_new, float *Fe_new, float *Fp_new,
                             float *tau_new, float *residuals, float *n_new, float *T_out, int *gelled_new,
                             float *yield_out, float *visc_out, const float *viscosity_parameter,
                             int *flags, float *porosity_residuals, const OraDingParams *P,
                             const float *T_local) {
    PAR_FOR
    for (int i = 0; i < n; ++i) {
        float por = n_old[i];
        if (!isfinite(por) || por < 0.0f || por >= 1.0f) { flag_set(flags, 0); continue; }
        int gel = gelled_old[i];
        float T = T_local[i];
        int reached = T >= P->knots[3];
        float Teff = T;
        float ty = P->yield_stress;
        float eta = viscosity_parameter[0];
        if (P->temperature_enabled) {
            if (reached) gel = 1;
            if (gel) Teff = P->knots[3];
            ty = P->yield_stress * ora_temperature_factor(Teff, P->knots, P->yield_factors);
            eta = viscosity_parameter[0] * ora_temperature_factor(Teff, P->knots, P->viscosity_factors);
        }
        float G[9], trial[9];
        for (int e = 0; e < 9; ++e) G[e] = P->dt * C_new[9 * i + e] + ((e % 4) == 0 ? 1.0f : 0.0f);
        matmul3f(G, Fe_old + 9 * i, trial);
        float ret_por = por, consistency = 0.0f;
        double Ud[9], sd[3], Vd[9];
        int have_svd = 0;
        float mu = P->mu, lam = P->lam, dt = P->dt, n0 = P->initial_porosity;
        if (P->coupled_porosity) {
            double Ad[9];
            for (int e = 0; e < 9; ++e) Ad[e] = (double)trial[e];
            ora_svd3(Ad, Ud, sd, Vd);
            have_svd = 1;
            float st[3] = {logf((float)sd[0]), logf((float)sd[1]), logf((float)sd[2])};
            float tr = st[0] + st[1] + st[2];
            float ts[3];
            for (int k = 0; k < 3; ++k) ts[k] = 2.0f * mu * st[k] + lam * tr * 1.0f;
            float mean = (ts[0] + ts[1] + ts[2]) / 3.0f;
            float dev[3] = {ts[0] - mean, ts[1] - mean, ts[2] - mean};
            float qv = 1.5f * (dev[0] * dev[0] + dev[1] * dev[1] + dev[2] * dev[2]) / (ty * ty);
            float pv = mean * mean / (ty * ty);
            float df = 6.0f * mu * dt * ty * ty / eta;
            float ms = 2.0f / 3.0f * (2.0f * mu + 3.0f * lam) * dt * ty * ty / eta;
            float ex = 3.0f * mean / (2.0f * mu + 3.0f * lam);
            double Vp = 1.0 - (double)n0 + (double)por;
            ret_por = ora_solve_porosity(qv, pv, df, ms, ex, Vp, n0);
            double pred = ora_porosity_prediction((double)ret_por, qv, pv, df, ms, ex, Vp, n0);
            consistency = (float)fabs((double)ret_por - pred);
            if (consistency > 1.0e-6f || ret_por <= 0.0f || ret_por >= 1.0f) flag_set(flags, 1);
        }
        float Fe[9], tau[9], res;
        ora_ding_return(trial, mu, lam, ty, eta, ora_porosity_coefficient(ret_por), dt,
                        have_svd ? Ud : NULL, sd, Vd, Fe, tau, &res);
        if (P->coupled_porosity) {
            double target = 1.0 - (double)n0 + (double)ret_por;
            double Fd[9], Fed[9];
            for (int e = 0; e < 9; ++e) { Fd[e] = (double)F_tot[9 * i + e]; Fed[e] = (double)Fe[e]; }
            double vs = det3d(Fd) / (target * det3d(Fed));
            float scale = (float)pow(vs, 1.0 / 3.0);
            for (int e = 0; e < 9; ++e) Fe[e] = Fe[e] * scale;
        }
        float Fp[9], inv[9];
        inverse3f(Fe, inv);
        matmul3f(inv, F_tot + 9 * i, Fp);
        float npor = det3f(Fp) - 1.0f + n0;
        if (P->coupled_porosity) npor = ret_por;
        if (n0 == 0.0f && por == 0.0f) npor = 0.0f;
        if (!isfinite(npor) || npor < 0.0f || npor >= 1.0f) flag_set(flags, 0);
        memcpy(Fe_new + 9 * i, Fe, sizeof Fe);
        memcpy(Fp_new + 9 * i, Fp, sizeof Fp);
        memcpy(tau_new + 9 * i, tau, sizeof tau);
        residuals[i] = res;
        porosity_residuals[i] = consistency;
        n_new[i] = npor;
        T_out[i] = T;
        gelled_new[i] = gel;
        yield_out[i] = ty;
        visc_out[i] = eta;
    }
}

/* ------------------------------------ physics/materials/gas.py:7-45 */
#define GAS_CONSTANT 8.31446261815324

ORA_API double ora_gas_pressure(double moles, float T, float J, float n) {
    return moles * GAS_CONSTANT * (double)T / ((double)J * (double)n);
}

ORA_API void ora_combine_gas_stress(int n, const float *tau_solid, const float *F, const float *por,
                                    const double *moles, const float *T, float *tau_total, int *flags,
                                    float ambient, float n0, const float *density, float elastic_modulus,
                                    float dt, float dx, float cfl) {
    PAR_FOR
    for (int i = 0; i < n; ++i) {
        float J = det3f(F + 9 * i);
        float ni = por[i];
        if (ni <= 0.0f || ni >= 1.0f || !isfinite(ni) || J <= 0.0f) { flag_set(flags, 0); continue; }
        float p = (float)ora_gas_pressure(moles[i], T[i], J, ni);
        float iso = J * (ambient - p);
        for (int e = 0; e < 9; ++e) tau_total[9 * i + e] = tau_solid[9 * i + e] + ((e % 4) == 0 ? iso : iso * 0.0f);
        float bulk = p * (1.0f + (1.0f - n0 + ni) / ni);
        float wave = sqrtf((elastic_modulus + bulk) * J / density[i]);
        if (!isfinite(p) || wave * dt / dx > cfl) flag_set(flags, 2);
    }
}

ORA_API void ora_refresh_gas(int n, const double *old_moles, double *new_moles, const float *F, const float *por,
                             double *pressures, const float *T) {
    PAR_FOR
    for (int i = 0; i < n; ++i) {
        new_moles[i] = old_moles[i];
        if (por[i] > 0.0f && por[i] < 1.0f)
            pressures[i] = ora_gas_pressure(old_moles[i], T[i], det3f(F + 9 * i), por[i]);
    }
}

/* ------------------------------- physics/thermal_water.py:77-92 */
ORA_API void ora_surface_areas(int nf, const float *vertices, const int *faces, const int *owners,
                               double *exposed, double *contact, float floor_height, float contact_distance) {
    for (int f = 0; f < nf; ++f) {
        double p[3][3];
        for (int k = 0; k < 3; ++k)
            for (int a = 0; a < 3; ++a) p[k][a] = (double)vertices[3 * faces[3 * f + k] + a];
        double e1[3] = {p[1][0] - p[0][0], p[1][1] - p[0][1], p[1][2] - p[0][2]};
        double e2[3] = {p[2][0] - p[0][0], p[2][1] - p[0][1], p[2][2] - p[0][2]};
        double nrm[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
        double len = sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
        double area = 0.5 * len;
        double cy = (p[0][1] + p[1][1] + p[2][1]) / 3.0;
        if (cy <= (double)(floor_height + contact_distance) && nrm[1] < -0.2 * len) contact[owners[f]] += area;
        else exposed[owners[f]] += area;
    }
}

/* ------------------------------- physics/thermal_water.py:95-137 */
typedef struct {
    float oven_temperature, tray_temperature, tray_transfer, surface_loss, water_density, latent_heat;
    int water_enabled;
    float origin[3];
    float dx;
    int R;
} OraScalarParams;

ORA_API void ora_scalar_to_grid(int n, const float *x, const float *F, const float *V0, const double *cap,
                                const double *T, const double *W, const double *exposed, const double *contact,
                                const float *heat_parameter, const OraScalarParams *P, double *n_vol,
                                double *n_cap, double *n_energy, double *n_water, double *n_heat,
                                double *n_loss, double *n_exch, double *p_heat, double *p_loss, int *flags) {
    PAR_FOR
    for (int i = 0; i < n; ++i) {
        double vol = (double)V0[i] * (double)det3f(F + 9 * i);
        double Ti = T[i];
        double sat = W[i] / ((double)P->water_density * vol);
        double loss = 0.0;
        if (P->water_enabled) loss = (double)P->surface_loss * Ti * sat * exposed[i];
        double h = (double)heat_parameter[0];
        double heat = h * exposed[i] * ((double)P->oven_temperature - Ti)
                    + (double)P->tray_transfer * contact[i] * ((double)P->tray_temperature - Ti)
                    - (double)P->latent_heat * loss;
        double exch = h * exposed[i] + (double)P->tray_transfer * contact[i];
        if (P->water_enabled) exch += (double)(P->latent_heat * P->surface_loss) * sat * exposed[i];
        p_heat[i] = heat;
        p_loss[i] = loss;
        float g[3];
        for (int a = 0; a < 3; ++a) g[a] = (x[3 * i + a] - P->origin[a]) / P->dx;
        int b[3];
        stencil_base(g, b);
        /* The reference does not range-check here; an out-of-grid stencil is
           reported through the P2G flag instead of writing out of bounds. */
        if (!valid_stencil(b, P->R)) { flag_set(flags, 1); continue; }
        float l[3] = {g[0] - (float)b[0], g[1] - (float)b[1], g[2] - (float)b[2]};
        for (int ox = 0; ox < 3; ++ox)
            for (int oy = 0; oy < 3; ++oy)
                for (int oz = 0; oz < 3; ++oz) {
                    double w = (double)(ora_quadratic_weight(l[0], ox) * ora_quadratic_weight(l[1], oy)
                                        * ora_quadratic_weight(l[2], oz));
                    int64_t node = flatten_node(b[0] + ox, b[1] + oy, b[2] + oz, P->R);
                    double wv = w * vol, wc = w * cap[i], we = w * cap[i] * Ti, ww = w * W[i];
                    double wh = w * heat, wl = w * loss, wx = w * exch;
                    ATOMIC n_vol[node] += wv;
                    ATOMIC n_cap[node] += wc;
                    ATOMIC n_energy[node] += we;
                    ATOMIC n_water[node] += ww;
                    ATOMIC n_heat[node] += wh;
                    ATOMIC n_loss[node] += wl;
                    ATOMIC n_exch[node] += wx;
                }
    }
}

/* ------------------------------- physics/thermal_water.py:140-147 */
ORA_API void ora_grid_fields(int64_t nn, const double *vol, const double *cap, const double *energy,
                             const double *water, double *T, double *s, float water_density) {
    PAR_FOR
    for (int64_t i = 0; i < nn; ++i) {
        if (cap[i] > 0.0) {
            T[i] = energy[i] / cap[i];
            s[i] = water[i] / ((double)water_density * vol[i]);
        }
    }
}

/* ------------------------------- physics/thermal_water.py:150-190 */
ORA_API void ora_diffuse_grid(int64_t nn, const double *vol, const double *cap, const double *T, const double *s,
                              const double *water, const double *b_heat, const double *b_loss,
                              const double *b_exch, double *dT, double *dW, int *errors, float conductivity,
                              float diffusivity, float water_density, int water_enabled, float dx, int R,
                              float dt) {
    PAR_FOR
    for (int64_t i = 0; i < nn; ++i) {
        if (cap[i] <= 0.0) continue;
        int c[3] = {(int)(i / ((int64_t)R * R)), (int)((i / R) % R), (int)(i % R)};
        double heat_rate = b_heat[i];
        double water_rate = -b_loss[i];
        double heat_diag = b_exch[i];
        double water_diag = 0.0;
        for (int axis = 0; axis < 3; ++axis)
            for (int side = 0; side < 2; ++side) {
                int o[3] = {c[0], c[1], c[2]};
                o[axis] += 2 * side - 1;
                if (o[axis] < 0 || o[axis] >= R) continue;
                int64_t j = flatten_node(o[0], o[1], o[2], R);
                if (!(cap[j] > 0.0)) continue;
                double fill = 2.0 * vol[i] * vol[j] / (vol[i] + vol[j]) / (double)(dx * dx * dx);
                double hc = (double)(conductivity * dx) * fill;
                heat_rate += hc * (T[j] - T[i]);
                heat_diag += hc;
                if (water_enabled) {
                    double mob = (double)(diffusivity * water_density * dx) * fill * 0.5 * (T[i] + T[j])
                               * 0.5 * (s[i] + s[j]);
                    water_rate += mob * (s[j] - s[i]);
                    water_diag += mob / ((double)water_density * vol[i]);
                }
            }
        if ((double)dt * heat_diag > cap[i]) flag_set(errors, 0);
        double change = (double)dt * water_rate;
        if (water[i] + change < 0.0 || (double)dt * water_diag > 1.0) flag_set(errors, 1);
        dT[i] = (double)dt * heat_rate / cap[i];
        dW[i] = change;
    }
}

/* ------------------------------- physics/thermal_water.py:193-229 */
ORA_API void ora_scalar_to_particles(int n, const float *x, const double *T_old, const double *W_old,
                                     const double *loss_old, const double *exch_old, const double *dry,
                                     const float *V0, const float *F, const double *n_water, const double *n_dT,
                                     const double *n_dW, const double *p_heat, const double *p_loss,
                                     double *T_new, float *T_material, double *W_new, double *loss_new,
                                     double *exch_new, float *mass_new, float *density_new, double *sat_new,
                                     float water_density, const float *origin, float dx, int R, float dt,
                                     int *flags) {
    PAR_FOR
    for (int i = 0; i < n; ++i) {
        float g[3];
        for (int a = 0; a < 3; ++a) g[a] = (x[3 * i + a] - origin[a]) / dx;
        int b[3];
        stencil_base(g, b);
        if (!valid_stencil(b, R)) { flag_set(flags, 1); continue; }
        float l[3] = {g[0] - (float)b[0], g[1] - (float)b[1], g[2] - (float)b[2]};
        double dTp = 0.0, ratio = 0.0;
        for (int ox = 0; ox < 3; ++ox)
            for (int oy = 0; oy < 3; ++oy)
                for (int oz = 0; oz < 3; ++oz) {
                    double w = (double)(ora_quadratic_weight(l[0], ox) * ora_quadratic_weight(l[1], oy)
                                        * ora_quadratic_weight(l[2], oz));
                    int64_t node = flatten_node(b[0] + ox, b[1] + oy, b[2] + oz, R);
                    dTp += w * n_dT[node];
                    if (n_water[node] > 0.0) ratio += w * n_dW[node] / n_water[node];
                }
        double Tn = T_old[i] + dTp;
        double Wn = W_old[i] * (1.0 + ratio);
        T_new[i] = Tn;
        T_material[i] = (float)Tn;
        W_new[i] = Wn;
        loss_new[i] = loss_old[i] + (double)dt * p_loss[i];
        exch_new[i] = exch_old[i] + (double)dt * p_heat[i];
        mass_new[i] = (float)(dry[i] + Wn);
        density_new[i] = (float)((dry[i] + Wn) / (double)V0[i]);
        sat_new[i] = Wn / ((double)water_density * (double)V0[i] * (double)det3f(F + 9 * i));
    }
}

/* ------------------------------- physics/thermal_water.py:232-260 */
ORA_API void ora_local_gas(int n, const double *old_moles, const double *T_old, const double *T_new,
                           double *new_moles, double *pressures, const float *F, const float *por,
                           const float *parameter, int per_particle, float density, float peak, float width,
                           float dt, int produce) {
    PAR_FOR
    for (int i = 0; i < n; ++i) {
        double moles = old_moles[i];
        if (produce) {
            double Tm = 0.5 * (T_old[i] + T_new[i]);
            double alpha = (double)parameter[per_particle ? i : 0];
            moles += (double)(dt * density) * alpha * exp(-pow((Tm - (double)peak) / (double)width, 2.0));
        }
        new_moles[i] = moles;
        if (por[i] > 0.0f) pressures[i] = ora_gas_pressure(moles, (float)T_new[i], det3f(F + 9 * i), por[i]);
    }
}

ORA_API void ora_water_stress(int n, const float *F, const double *sat, const float *tau_old, float *tau_new,
                              float s0, float stiffness) {
    PAR_FOR
    for (int i = 0; i < n; ++i) {
        float iso = det3f(F + 9 * i) * stiffness * ((float)sat[i] - s0);
        for (int e = 0; e < 9; ++e) tau_new[9 * i + e] = tau_old[9 * i + e] - ((e % 4) == 0 ? iso : iso * 0.0f);
    }
}

ORA_API void ora_saturations(int n, const double *W, const float *V0, const float *F, double *sat, float density) {
    PAR_FOR
    for (int i = 0; i < n; ++i)
        sat[i] = W[i] / ((double)density * (double)V0[i] * (double)det3f(F + 9 * i));
}

/* ------------------------------- geometry/mesh_tracking.py:13-38 */
ORA_API void ora_reconstruct_mesh_vertices(int nv, const float *x, const float *F, const float *ref_vertices,
                                           const int *offsets, const int *particles, const float *weights,
                                           const float *ref_offsets, float *out) {
    PAR_FOR
    for (int v = 0; v < nv; ++v) {
        int b0 = offsets[v], b1 = offsets[v + 1];
        if (b0 == b1) { for (int a = 0; a < 3; ++a) out[3 * v + a] = ref_vertices[3 * v + a]; continue; }
        int ap = particles[b0];
        float anchor[3];
        for (int r = 0; r < 3; ++r) {
            const float *f = F + 9 * ap, *o = ref_offsets + 3 * b0;
            anchor[r] = x[3 * ap + r] + (f[3 * r] * o[0] + f[3 * r + 1] * o[1] + f[3 * r + 2] * o[2]);
        }
        float disp[3] = {0, 0, 0};
        for (int b = b0; b < b1; ++b) {
            int p = particles[b];
            const float *f = F + 9 * p, *o = ref_offsets + 3 * b;
            for (int r = 0; r < 3; ++r) {
                float pred = x[3 * p + r] + (f[3 * r] * o[0] + f[3 * r + 1] * o[1] + f[3 * r + 2] * o[2]);
                disp[r] = disp[r] + weights[b] * (pred - anchor[r]);
            }
        }
        for (int r = 0; r < 3; ++r) out[3 * v + r] = anchor[r] + disp[r];
    }
}

/* ------------------------------- physics/quasistatic.py:11-21 */
ORA_API void ora_settling_metrics(int n, const float *v, const float *C, const float *Fp_old, const float *Fp_new,
                                  float *metrics, float dt) {
    for (int i = 0; i < n; ++i) {
        const float *a = C + 9 * i, *po = Fp_old + 9 * i, *pn = Fp_new + 9 * i;
        float sym2 = 0, ch2 = 0, pn2 = 0;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                float s = 0.5f * (a[3 * r + c] + a[3 * c + r]);
                sym2 += s * s;
                float d = pn[3 * r + c] - po[3 * r + c];
                ch2 += d * d;
                pn2 += po[3 * r + c] * po[3 * r + c];
            }
        float speed = sqrtf(v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2]);
        float rate = sqrtf(ch2) / (dt * sqrtf(pn2));
        if (speed > metrics[0]) metrics[0] = speed;
        if (sqrtf(sym2) > metrics[1]) metrics[1] = sqrtf(sym2);
        if (rate > metrics[2]) metrics[2] = rate;
    }
}
