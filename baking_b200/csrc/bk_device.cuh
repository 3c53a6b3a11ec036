// Device-side math shared by the baking_b200 kernels (sm_100a).
//
// Per-particle physics of the reference kernels as __device__ functions, so the
// one-kernel-per-reference-kernel entry points and the fused substep kernels run
// the same arithmetic. Precision follows the reference: float32 where its Warp
// kernel uses `float`, float64 where it uses `wp.float64`.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define BK_DEV __device__ __forceinline__

namespace bk {

struct M3 { float m[9]; };
struct M3d { double m[9]; };
struct V3 { float v[3]; };

// Two independent float32 fused multiply-adds in one instruction (sm_100's packed fma.rn.f32x2):
// each half is rounded exactly like fmaf, so a loop of paired accumulators gives the bits of the
// same loop written with fmaf, at half the issue slots.
BK_DEV float2 ffma2(float2 a, float2 b, float2 c) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\tmov.b64 rc, {%6, %7};\n\t"
        "fma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return d;
}

// ------------------------------------------------------------- SoA access
BK_DEV V3 load_v3(const float* __restrict__ p, int64_t i, int64_t pitch) {
    V3 r;
#pragma unroll
    for (int c = 0; c < 3; ++c) r.v[c] = __ldg(p + c * pitch + i);
    return r;
}
BK_DEV void store_v3(float* __restrict__ p, int64_t i, int64_t pitch, const V3& a) {
#pragma unroll
    for (int c = 0; c < 3; ++c) p[c * pitch + i] = a.v[c];
}
BK_DEV M3 load_m3(const float* __restrict__ p, int64_t i, int64_t pitch) {
    M3 r;
#pragma unroll
    for (int c = 0; c < 9; ++c) r.m[c] = __ldg(p + c * pitch + i);
    return r;
}
BK_DEV void store_m3(float* __restrict__ p, int64_t i, int64_t pitch, const M3& a) {
#pragma unroll
    for (int c = 0; c < 9; ++c) p[c * pitch + i] = a.m[c];
}

// ------------------------------------------------------------- 3x3 algebra
BK_DEV float det3(const M3& a) {
    const float* m = a.m;
    return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6])
         + m[2] * (m[3] * m[7] - m[4] * m[6]);
}
BK_DEV double det3(const M3d& a) {
    const double* m = a.m;
    return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6])
         + m[2] * (m[3] * m[7] - m[4] * m[6]);
}
BK_DEV M3 matmul(const M3& a, const M3& b) {
    M3 r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            r.m[3 * i + j] = a.m[3 * i] * b.m[j] + a.m[3 * i + 1] * b.m[3 + j] + a.m[3 * i + 2] * b.m[6 + j];
    return r;
}
// Adjugate / determinant.
BK_DEV M3 inverse3(const M3& a) {
    const float* m = a.m;
    float inv = 1.0f / det3(a);
    M3 r;
    r.m[0] = (m[4] * m[8] - m[5] * m[7]) * inv;
    r.m[1] = (m[2] * m[7] - m[1] * m[8]) * inv;
    r.m[2] = (m[1] * m[5] - m[2] * m[4]) * inv;
    r.m[3] = (m[5] * m[6] - m[3] * m[8]) * inv;
    r.m[4] = (m[0] * m[8] - m[2] * m[6]) * inv;
    r.m[5] = (m[2] * m[3] - m[0] * m[5]) * inv;
    r.m[6] = (m[3] * m[7] - m[4] * m[6]) * inv;
    r.m[7] = (m[1] * m[6] - m[0] * m[7]) * inv;
    r.m[8] = (m[0] * m[4] - m[1] * m[3]) * inv;
    return r;
}

// 3x3 SVD A = U diag(s) V^T in float64 by one-sided Jacobi (Hestenes 1958): right
// plane rotations orthogonalise A's columns; column norms are the singular values.
// Out of line: the hot kernels reach it only for rank-deficient input, and inlining it there would
// put its code between their hot instructions.
static __device__ __noinline__ void svd3(const M3d& A, M3d& U, double s[3], M3d& V) {
    double b[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) b[e] = A.m[e];
    double v[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    for (int sweep = 0; sweep < 40; ++sweep) {
        bool rotated = false;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int p = k == 2 ? 1 : 0;
            const int q = k == 0 ? 1 : 2;
            double alpha = 0, beta = 0, gamma = 0;
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                alpha += b[3 * r + p] * b[3 * r + p];
                beta += b[3 * r + q] * b[3 * r + q];
                gamma += b[3 * r + p] * b[3 * r + q];
            }
            if (gamma == 0.0 || fabs(gamma) <= 1e-15 * sqrt(alpha * beta)) continue;
            rotated = true;
            double zeta = (beta - alpha) / (2.0 * gamma);
            double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
            double c = rsqrt(1.0 + t * t);
            double sn = c * t;
#pragma unroll
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
    bool zero[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double n = sqrt(b[c] * b[c] + b[3 + c] * b[3 + c] + b[6 + c] * b[6 + c]);
        s[c] = n;
        zero[c] = !(n > 1e-300);
        double inv = zero[c] ? 0.0 : 1.0 / n;
#pragma unroll
        for (int r = 0; r < 3; ++r) U.m[3 * r + c] = b[3 * r + c] * inv;
    }
    if (zero[0] || zero[1] || zero[2]) {
        // Rank-deficient input: complete U to an orthonormal basis.
        for (int c = 0; c < 3; ++c) {
            if (!zero[c]) continue;
            int a = (c + 1) % 3, d = (c + 2) % 3;
            double ua[3] = {U.m[a], U.m[3 + a], U.m[6 + a]}, ud[3] = {U.m[d], U.m[3 + d], U.m[6 + d]};
            if (zero[a]) {
                ua[0] = fabs(ud[0]) < 0.9 ? 1.0 : 0.0;
                ua[1] = 1.0 - ua[0];
                ua[2] = 0.0;
                double dp = ua[0] * ud[0] + ua[1] * ud[1] + ua[2] * ud[2];
                for (int r = 0; r < 3; ++r) ua[r] -= dp * ud[r];
                double n = sqrt(ua[0] * ua[0] + ua[1] * ua[1] + ua[2] * ua[2]);
                for (int r = 0; r < 3; ++r) { ua[r] /= n; U.m[3 * r + a] = ua[r]; }
                zero[a] = false;
            }
            U.m[c] = ua[1] * ud[2] - ua[2] * ud[1];
            U.m[3 + c] = ua[2] * ud[0] - ua[0] * ud[2];
            U.m[6 + c] = ua[0] * ud[1] - ua[1] * ud[0];
            zero[c] = false;
        }
    }
#pragma unroll
    for (int e = 0; e < 9; ++e) V.m[e] = v[e];
}

// Fast 3x3 SVD with the same float64 accuracy as svd3: a float32 cyclic Jacobi eigen-solve of
// A^T A (four sweeps, Jacobi 1846 / Golub-Van Loan 8.4) gives approximate right singular vectors;
// after re-orthonormalising them in float64, the one-sided float64 Jacobi iteration of svd3
// continues from B = A V, whose columns are already nearly orthogonal, so it usually converges in
// one sweep instead of four to six.
BK_DEV void svd3_fast(const M3d& A, M3d& U, double s[3], M3d& V) {
    // float32 warm start on S = A^T A.
    float S[3][3], a32[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) a32[e] = (float)A.m[e];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) S[i][j] = a32[i] * a32[j] + a32[3 + i] * a32[3 + j] + a32[6 + i] * a32[6 + j];
    float v[3][3] = {{1.f, 0.f, 0.f}, {0.f, 1.f, 0.f}, {0.f, 0.f, 1.f}};
#pragma unroll
    for (int sweep = 0; sweep < 4; ++sweep) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int p = k == 2 ? 1 : 0;
            const int q = k == 0 ? 1 : 2;
            const int r = 3 - p - q;
            float apq = S[p][q];
            if (fabsf(apq) <= 1e-30f) continue;
            float theta = (S[q][q] - S[p][p]) / (2.0f * apq);
            float t = copysignf(1.0f, theta) / (fabsf(theta) + sqrtf(theta * theta + 1.0f));
            float c = rsqrtf(t * t + 1.0f);
            float sn = t * c;
            S[p][p] -= t * apq;
            S[q][q] += t * apq;
            S[p][q] = S[q][p] = 0.0f;
            float arp = S[r][p], arq = S[r][q];
            S[r][p] = S[p][r] = c * arp - sn * arq;
            S[r][q] = S[q][r] = sn * arp + c * arq;
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                float vp = v[i][p], vq = v[i][q];
                v[i][p] = c * vp - sn * vq;
                v[i][q] = sn * vp + c * vq;
            }
        }
    }
    // Re-orthonormalise in float64 (Gram-Schmidt on columns 0, 1; column 2 = c0 x c1).
    double c0[3] = {v[0][0], v[1][0], v[2][0]}, c1[3] = {v[0][1], v[1][1], v[2][1]};
    double n0 = rsqrt(c0[0] * c0[0] + c0[1] * c0[1] + c0[2] * c0[2]);
#pragma unroll
    for (int i = 0; i < 3; ++i) c0[i] *= n0;
    double d01 = c0[0] * c1[0] + c0[1] * c1[1] + c0[2] * c1[2];
#pragma unroll
    for (int i = 0; i < 3; ++i) c1[i] -= d01 * c0[i];
    double n1 = rsqrt(c1[0] * c1[0] + c1[1] * c1[1] + c1[2] * c1[2]);
#pragma unroll
    for (int i = 0; i < 3; ++i) c1[i] *= n1;
    double c2[3] = {c0[1] * c1[2] - c0[2] * c1[1], c0[2] * c1[0] - c0[0] * c1[2], c0[0] * c1[1] - c0[1] * c1[0]};
    double vv[9] = {c0[0], c1[0], c2[0], c0[1], c1[1], c2[1], c0[2], c1[2], c2[2]};
    // B = A V; one-sided float64 Jacobi on B's columns, V accumulating the rotations.
    double b[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            b[3 * i + j] = A.m[3 * i] * vv[j] + A.m[3 * i + 1] * vv[3 + j] + A.m[3 * i + 2] * vv[6 + j];
    for (int sweep = 0; sweep < 12; ++sweep) {
        bool rotated = false;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int p = k == 2 ? 1 : 0;
            const int q = k == 0 ? 1 : 2;
            double alpha = 0, beta = 0, gamma = 0;
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                alpha += b[3 * r + p] * b[3 * r + p];
                beta += b[3 * r + q] * b[3 * r + q];
                gamma += b[3 * r + p] * b[3 * r + q];
            }
            if (gamma * gamma <= 1e-30 * alpha * beta) continue;
            rotated = true;
            double zeta = (beta - alpha) / (2.0 * gamma);
            double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
            double c = rsqrt(1.0 + t * t);
            double sn = c * t;
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                double bp = b[3 * r + p], bq = b[3 * r + q];
                b[3 * r + p] = c * bp - sn * bq;
                b[3 * r + q] = sn * bp + c * bq;
                double vp = vv[3 * r + p], vq = vv[3 * r + q];
                vv[3 * r + p] = c * vp - sn * vq;
                vv[3 * r + q] = sn * vp + c * vq;
            }
        }
        if (!rotated) break;
    }
    bool zero[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double n = sqrt(b[c] * b[c] + b[3 + c] * b[3 + c] + b[6 + c] * b[6 + c]);
        s[c] = n;
        zero[c] = !(n > 1e-300);
        double inv = zero[c] ? 0.0 : 1.0 / n;
#pragma unroll
        for (int r = 0; r < 3; ++r) U.m[3 * r + c] = b[3 * r + c] * inv;
    }
#pragma unroll
    for (int e = 0; e < 9; ++e) V.m[e] = vv[e];
    if (zero[0] || zero[1] || zero[2]) {
        // Rank-deficient input: fall back to the reference-path solver, which completes U.
        svd3(A, U, s, V);
    }
}

// 3x3 SVD A = U diag(s) V^T in float32 by one-sided Jacobi (Hestenes 1958), iterated to float32
// convergence. The reference computes its SVD in float64 and rounds U, s and V to float32 before
// using them (physics/materials/ding.py:106-109); a converged float32 Jacobi SVD carries errors of
// the same few-ulp size, with a third of the registers and latency of the float64 solve.
// Rank-deficient input (a zero singular value) falls back to the float64 solver. e = log(s), the
// principal log stretches, as the reference takes the log of its rounded singular values.
// kPolish = false stops after the float32 sweeps (columns orthogonal to ~2e-7): the factors then
// reproduce A to float32 rounding, but nearly equal singular values leave their singular vectors
// mixed by ~2^-24 / gap, so U, s and V no longer round like the reference's. The surrogate return
// (an approximation to ~1e-3 by construction) takes that form.
template <bool kPolish = true>
BK_DEV void svd3f(const M3& A, M3& U, float s[3], M3& V, float e[3]) {
    float b[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) b[e] = A.m[e];
    float v[9] = {1.f, 0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, 1.f};
    for (int sweep = 0; sweep < 6; ++sweep) {
        bool rotated = false;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int p = k == 2 ? 1 : 0;
            const int q = k == 0 ? 1 : 2;
            float alpha = 0.f, beta = 0.f, gamma = 0.f;
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                alpha = fmaf(b[3 * r + p], b[3 * r + p], alpha);
                beta = fmaf(b[3 * r + q], b[3 * r + q], beta);
                gamma = fmaf(b[3 * r + p], b[3 * r + q], gamma);
            }
            // Columns orthogonal to 1e-6 (|gamma| <= 1e-6 sqrt(alpha beta)) are enough when the
            // float64 sweep below takes the off-diagonal terms from there to ~1e-12 / gap; without
            // it the sweeps go on to ~2e-7, the float32 rounding level.
            if (gamma * gamma <= (kPolish ? 1e-12f : 4e-14f) * alpha * beta) continue;
            rotated = true;
            float zeta = (beta - alpha) / (2.0f * gamma);
            float t = fabsf(zeta) > 1e18f ? 0.5f / zeta
                                           : copysignf(1.0f, zeta) / (fabsf(zeta) + sqrtf(fmaf(zeta, zeta, 1.0f)));
            float c = rsqrtf(fmaf(t, t, 1.0f));
            float sn = c * t;
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                float bp = b[3 * r + p], bq = b[3 * r + q];
                b[3 * r + p] = c * bp - sn * bq;
                b[3 * r + q] = sn * bp + c * bq;
                float vp = v[3 * r + p], vq = v[3 * r + q];
                v[3 * r + p] = c * vp - sn * vq;
                v[3 * r + q] = sn * vp + c * vq;
            }
        }
        if (!rotated) break;
    }
    if constexpr (!kPolish) {
        bool degenerate = false;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float n2 = b[c] * b[c] + b[3 + c] * b[3 + c] + b[6 + c] * b[6 + c];
            degenerate |= !(n2 > 1e-30f);
            const float inv = rsqrtf(n2);
            s[c] = n2 * inv;
#pragma unroll
            for (int r = 0; r < 3; ++r) U.m[3 * r + c] = b[3 * r + c] * inv;
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) V.m[k] = v[k];
        if (degenerate) {
            M3d Ad, Ud, Vd;
            double sd[3];
#pragma unroll
            for (int k = 0; k < 9; ++k) Ad.m[k] = (double)A.m[k];
            svd3(Ad, Ud, sd, Vd);
#pragma unroll
            for (int k = 0; k < 9; ++k) { U.m[k] = (float)Ud.m[k]; V.m[k] = (float)Vd.m[k]; }
#pragma unroll
            for (int k = 0; k < 3; ++k) s[k] = (float)sd[k];
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) e[k] = logf(s[k]);
        return;
    }
    // Finish in float64. The float32 rotations leave the columns of B = A V orthogonal to ~2^-24,
    // but nearly equal singular values (small elastic strains) make float32 mix their singular
    // vectors by ~2^-24 / gap. One float64 Jacobi sweep from this start reduces the off-diagonal
    // terms to ~2^-48 / gap (Jacobi's quadratic convergence), after which s = |B_i| and U = B / s
    // agree with the float64 SVD to float32 rounding.
    // The accumulated float32 rotations are orthonormal only to ~1e-7, which would scale s by as
    // much; re-orthonormalise them in float64 first (Gram-Schmidt, third column = cross product).
    double vv[9], bb[9];
    {
        double c0[3] = {v[0], v[3], v[6]}, c1[3] = {v[1], v[4], v[7]};
        double n0 = rsqrt(c0[0] * c0[0] + c0[1] * c0[1] + c0[2] * c0[2]);
#pragma unroll
        for (int i = 0; i < 3; ++i) c0[i] *= n0;
        double d01 = c0[0] * c1[0] + c0[1] * c1[1] + c0[2] * c1[2];
#pragma unroll
        for (int i = 0; i < 3; ++i) c1[i] -= d01 * c0[i];
        double n1 = rsqrt(c1[0] * c1[0] + c1[1] * c1[1] + c1[2] * c1[2]);
#pragma unroll
        for (int i = 0; i < 3; ++i) c1[i] *= n1;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            vv[3 * i] = c0[i];
            vv[3 * i + 1] = c1[i];
        }
        vv[2] = c0[1] * c1[2] - c0[2] * c1[1];
        vv[5] = c0[2] * c1[0] - c0[0] * c1[2];
        vv[8] = c0[0] * c1[1] - c0[1] * c1[0];
    }
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            bb[3 * r + c] = (double)A.m[3 * r] * vv[c] + (double)A.m[3 * r + 1] * vv[3 + c] +
                            (double)A.m[3 * r + 2] * vv[6 + c];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int p = k == 2 ? 1 : 0;
        const int q = k == 0 ? 1 : 2;
        double alpha = 0, beta = 0, gamma = 0;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            alpha += bb[3 * r + p] * bb[3 * r + p];
            beta += bb[3 * r + q] * bb[3 * r + q];
            gamma += bb[3 * r + p] * bb[3 * r + q];
        }
        if (gamma * gamma <= 1e-30 * alpha * beta) continue;
        // tan of the rotation angle, t = 2 gamma sign(d) / (|d| + sqrt(d^2 + 4 gamma^2)), d = beta - alpha.
        double d = beta - alpha;
        double t = 2.0 * gamma / (d >= 0.0 ? d + sqrt(d * d + 4.0 * gamma * gamma) : d - sqrt(d * d + 4.0 * gamma * gamma));
        double c = rsqrt(1.0 + t * t);
        double sn = c * t;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            double bp = bb[3 * r + p], bq = bb[3 * r + q];
            bb[3 * r + p] = c * bp - sn * bq;
            bb[3 * r + q] = sn * bp + c * bq;
            double vp = vv[3 * r + p], vq = vv[3 * r + q];
            vv[3 * r + p] = c * vp - sn * vq;
            vv[3 * r + q] = sn * vp + c * vq;
        }
    }
    bool degenerate = false;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double n2 = bb[c] * bb[c] + bb[3 + c] * bb[3 + c] + bb[6 + c] * bb[6 + c];
        degenerate |= !(n2 > 1e-30);
        double inv = rsqrt(n2);
        s[c] = (float)(n2 * inv);
#pragma unroll
        for (int r = 0; r < 3; ++r) U.m[3 * r + c] = (float)(bb[3 * r + c] * inv);
    }
#pragma unroll
    for (int e = 0; e < 9; ++e) V.m[e] = (float)vv[e];
    if (degenerate) {
        M3d Ad, Ud, Vd;
        double sd[3];
#pragma unroll
        for (int e = 0; e < 9; ++e) Ad.m[e] = (double)A.m[e];
        svd3(Ad, Ud, sd, Vd);
#pragma unroll
        for (int e = 0; e < 9; ++e) { U.m[e] = (float)Ud.m[e]; V.m[e] = (float)Vd.m[e]; }
#pragma unroll
        for (int k = 0; k < 3; ++k) s[k] = (float)sd[k];
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) e[k] = logf(s[k]);
}

// ------------------------------------------------- physics/transfer.py:4-28
BK_DEV float qweight(float l, int i) {
    if (i == 0) return 0.5f * (1.5f - l) * (1.5f - l);
    if (i == 1) return 0.75f - (l - 1.0f) * (l - 1.0f);
    return 0.5f * (l - 0.5f) * (l - 0.5f);
}

struct Stencil {
    int b[3];
    float l[3];
    float w[3][3];  // w[axis][offset]
    bool valid;
};

BK_DEV Stencil make_stencil(const V3& x, const float* origin, float dx, int R) {
    Stencil s;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float g = (x.v[a] - origin[a]) / dx;
        s.b[a] = (int)floorf(g - 0.5f);
        s.l[a] = g - (float)s.b[a];
    }
    s.valid = s.b[0] >= 0 && s.b[1] >= 0 && s.b[2] >= 0 && s.b[0] + 2 < R && s.b[1] + 2 < R && s.b[2] + 2 < R;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int o = 0; o < 3; ++o) s.w[a][o] = qweight(s.l[a], o);
    return s;
}

BK_DEV int64_t node_index(int i, int j, int k, int R) { return ((int64_t)i * R + j) * R + k; }

// flags may be NULL (a re-evaluation whose flags are not reported).
BK_DEV void set_flag(int32_t* flags, int index) {
    if (flags && flags[index] == 0) atomicMax(flags + index, 1);
}

// ------------------------------------------------------- ding.py:56-100
BK_DEV float temperature_factor(float T, const float* knots, const float* factors) {
    float f = factors[0];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (T >= knots[k]) {
            float frac = fminf((T - knots[k]) / (knots[k + 1] - knots[k]), 1.0f);
            f = (1.0f - frac) * factors[k] + frac * factors[k + 1];
        }
    }
    return f;
}

BK_DEV float porosity_coefficient(float n) {
    float c = 0.0f;
    if (n > 0.0f) {
        float lg = logf(1.0f / n);
        c = 9.0f / (4.0f * (lg * lg) * (3.5f * n + 1.0f));
    }
    return c;
}

// Scalar overstress Newton solve (ding.py:77-87): up to 32 steps from r = 0 in float32.
// Iterates of this concave increasing residual approach the root monotonically from below;
// once a step moves r by no more than a few float32 ulps the iteration has converged and the
// reference's remaining steps only toggle the last bit, so it stops there.
BK_DEV float solve_overstress(float q2, float p2, float d, float h, float r0 = 0.0f) {
    // r0 > 0 warm-starts the iteration (a root of a nearby problem); the same stopping test applies.
    float r = r0 > 0.0f ? r0 : 0.0f;
    if (q2 + p2 > 1.0f) {
        for (int it = 0; it < 32; ++it) {
            float dd = 1.0f + d * r, md = 1.0f + h * r;
            float dd2 = dd * dd, md2 = md * md;
            float res = r + 1.0f - q2 / dd2 - p2 / md2;
            float der = 1.0f + 2.0f * d * q2 / (dd2 * dd) + 2.0f * h * p2 / (md2 * md);
            float rn = r - res / der;
            if (rn < 0.0f) { r = 0.0f; continue; }  // see overstress64
            bool done = fabsf(rn - r) <= 2.4e-7f * fabsf(rn);
            r = rn;
            if (done) break;
        }
    }
    return r;
}

// --------------------------------------- porous_return.py:11-61 (float64)
BK_DEV double pressure_coefficient64(double n) {
    double c = 0.0;
    if (n > 0.0) {
        double lg = log(1.0 / n);
        c = 9.0 / (4.0 * (lg * lg) * (3.5 * n + 1.0));
    }
    return c;
}

// `warm` (may be NULL): in, a root of a nearby problem to start from (0 starts at r = 0 like the
// reference); out, this problem's root. Newton on this concave increasing residual converges to the
// same root from either side, to the same |residual| < 1e-12 test.
BK_DEV double overstress64(double q, double p, double d, double h, double* warm = nullptr) {
    double r = (warm && *warm > 0.0) ? *warm : 0.0;
    if (!(q + p > 1.0)) r = 0.0;
    if (q + p > 1.0) {
        for (int it = 0; it < 48; ++it) {
            double u = 1.0 + d * r, v = 1.0 + h * r;
            double u2 = u * u, v2 = v * v;
            double res = r + 1.0 - q / u2 - p / v2;
            double der = 1.0 + 2.0 * d * q / (u2 * u) + 2.0 * h * p / (v2 * v);
            r -= res / der;
            // From a warm start above the root a step can pass zero; restart from r = 0 (the
            // iterates from 0 increase monotonically and never get here).
            if (r < 0.0) { r = 0.0; continue; }
            if (fabs(res) < 1.0e-12) break;
        }
    }
    if (warm) *warm = r;
    return r;
}

BK_DEV double porosity_prediction(double n, float q, float p, float d, float h, float e, double Vp, float n0,
                                  double* warm = nullptr) {
    double a = pressure_coefficient64(n);
    double r = overstress64((double)q, a * (double)p, (double)d, (double)h * a, warm);
    if (r == 0.0) return Vp - 1.0 + (double)n0;  // no overstress: exp(e (1 - 1/1)) = exp(0) = 1 exactly
    double den = 1.0 + (double)h * a * r;
    return Vp * exp((double)e * (1.0 - 1.0 / den)) - 1.0 + (double)n0;
}

// prediction(n) and its derivative in n. The overstress root r(n) is the reference's 48-step Newton
// solve; dr/dn follows from the implicit function theorem on its residual
// R = r + 1 - q/(1+dr)^2 - a p/(1+h a r)^2 with a = a(n) (the derivatives the reference's
// SolvePorosityGradient uses, porous_return.py:68-92).
BK_DEV double porosity_prediction_slope(double n, float qf, float pf, float df, float hf, float ef, double Vp,
                                        float n0, double& slope, double* warm = nullptr) {
    const double q = qf, p = pf, d = df, h = hf, e = ef;
    double a = pressure_coefficient64(n);
    double r = overstress64(q, a * p, d, h * a, warm);
    double v = 1.0 + h * a * r;
    double core = Vp * exp(e * (1.0 - 1.0 / v));
    double da = 0.0;
    if (n > 0.0) {
        double lg = log(1.0 / n);
        da = a * (2.0 / (n * lg) - 3.5 / (3.5 * n + 1.0));
    }
    double dr = 0.0;
    if (q + a * p > 1.0) {
        double u = 1.0 + d * r;
        double Rr = 1.0 + 2.0 * d * q / (u * u * u) + 2.0 * h * a * a * p / (v * v * v);
        dr = p * (1.0 - h * a * r) / (Rr * v * v * v) * da;
    }
    slope = core * e * h * (da * r + a * dr) / (v * v);
    return core - 1.0 + (double)n0;
}

// The reference's 64-step bisection of n -> prediction(n) on [0, 1 - 1e-9] (porous_return.py:51-61).
static __device__ __noinline__ float solve_porosity_bisection(float q, float p, float d, float h, float e, double Vp, float n0,
                                      double* warm = nullptr) {
    double lo = 0.0, hi = 1.0 - 1.0e-9;
    for (int it = 0; it < 64; ++it) {
        double mid = (lo + hi) * 0.5;
        double pred = porosity_prediction(mid, q, p, d, h, e, Vp, n0, warm);
        if (mid < pred) lo = mid; else hi = mid;
    }
    return (float)((lo + hi) * 0.5);
}

// End-state porosity (porous_return.py:43-61): the elastic early exit, then the root of
// g(n) = n - prediction(n) on the reference's bracket [0, 1 - 1e-9] with the reference's test
// (n lies below the root when n < prediction(n)). Safeguarded Newton steps replace the 64
// bisection steps: a step that leaves the current bracket becomes a bisection step, so the
// iteration cannot escape the bracket and converges in a few evaluations. When the bracket's
// lower end is not below the root (g(0+) >= 0) the reference's bisection runs unchanged. The root
// is resolved to ~1e-14 relative, far below the float32 rounding of the returned porosity.
// Each evaluation's overstress root starts from the previous one (`warm`, which also returns the
// last root to the caller); the roots are the reference's to its |residual| < 1e-12 test.
//
// The elastic early exit (q + a(trial) p <= 1) is first decided in float32 where that is certain:
// a float32 a(n) is within 1e-6 (2/ln(1/n) + 1) relative of the float64 one, so when
// q + a p <= 1 - 4e-6 (2/ln(1/n) + 1) a p the float64 test passes as well, both at the float64
// trial and at its float32 rounding (which moves ln n by at most 2^-24). `elastic_exit` (may be
// NULL) reports that certain case; there prediction(float(trial)) has no overstress and equals
// trial, so the caller can skip that evaluation. Every other case takes the float64 test.
BK_DEV float solve_porosity(float q, float p, float d, float h, float e, double Vp, float n0,
                            double* warm = nullptr, bool* elastic_exit = nullptr) {
    double r_local = 0.0;
    if (!warm) warm = &r_local;
    if (elastic_exit) *elastic_exit = false;
    double trial = Vp - 1.0 + (double)n0;
    if (trial > 0.0 && trial < 1.0) {
        const float nf = (float)trial;
        const float lgf = logf(1.0f / nf);
        const float af = 9.0f / (4.0f * (lgf * lgf) * (3.5f * nf + 1.0f));
        const double ap = (double)af * (double)p;
        const double bound = 4.0e-6 * (2.0 / (double)lgf + 1.0) * ap;
        if (nf >= 1.0e-30f && lgf > 0.0f && (double)q + ap <= 1.0 - bound) {
            if (elastic_exit) *elastic_exit = true;
            return nf;
        }
        double a = pressure_coefficient64(trial);
        if ((double)q + a * (double)p <= 1.0) return (float)trial;
    }
    double lo = 0.0, hi = 1.0 - 1.0e-9;
    // g(0+) = -trial: the root lies above zero only when the elastic prediction is positive.
    if (!(trial > 0.0)) return solve_porosity_bisection(q, p, d, h, e, Vp, n0, warm);
    double n = trial < hi ? trial : 0.5 * (lo + hi);
    for (int it = 0; it < 100; ++it) {
        double slope;
        double pred = porosity_prediction_slope(n, q, p, d, h, e, Vp, n0, slope, warm);
        double g = n - pred;
        if (g == 0.0) break;  // n is the root
        if (n < pred) lo = n; else hi = n;
        double dg = 1.0 - slope;
        double next = n - g / dg;
        // A converged Newton step ends the solve before the bracket test: when the root sits on
        // the end of the bracket that n just became (g at the float64 rounding level, as when the
        // mean stress vanishes), the step falls on that end, and treating it as a bracket escape
        // would bisect all the way back to it.
        if (fabs(next - n) <= 1e-14 * fabs(n)) {
            if (next > lo && next < hi) n = next;
            break;
        }
        if (!(next > lo && next < hi)) next = 0.5 * (lo + hi);
        n = next;
        if (hi - lo <= 1e-15 * hi) break;
    }
    return (float)n;
}

struct DingOut {
    M3 Fe, tau;
    float residual;
    float e[3];     // returned log principal strains before the isochoric correction (exponents of Fe)
    bool yielded;   // q^2 + p^2 > 1: the overstress solve ran
};

// Ding return map (ding.py:103-137) given the SVD of the trial gradient (float32 factors) and its
// principal log stretches log_s (svd3f).
BK_DEV DingOut ding_return(float det_trial, const M3& Um, const float* log_s, const M3& Vm, float mu, float lam,
                           float ty, float eta, float a, float dt, float r0 = 0.0f) {
    const float* U = Um.m;
    const float* V = Vm.m;
    float eps[3] = {log_s[0], log_s[1], log_s[2]};
    float tr = eps[0] + eps[1] + eps[2];
    float ts[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) ts[k] = 2.0f * mu * eps[k] + lam * tr;
    float mean = (ts[0] + ts[1] + ts[2]) / 3.0f;
    float dev[3] = {ts[0] - mean, ts[1] - mean, ts[2] - mean};
    float ty2 = ty * ty;
    float q2 = 1.5f * (dev[0] * dev[0] + dev[1] * dev[1] + dev[2] * dev[2]) / ty2;
    float p2 = a * mean * mean / ty2;
    float df = 6.0f * mu * dt * ty * ty / eta;
    float mf = 2.0f * a / 3.0f * (2.0f * mu + 3.0f * lam) * dt * ty * ty / eta;
    float r = solve_overstress(q2, p2, df, mf, r0);
    float cs[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) cs[k] = dev[k] / (1.0f + df * r) + mean / (1.0f + mf * r);
    float cm = (cs[0] + cs[1] + cs[2]) / 3.0f;
    float ex[3];
    DingOut o;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        o.e[k] = (cs[k] - cm) / (2.0f * mu) + cm / (2.0f * mu + 3.0f * lam);
        ex[k] = expf(o.e[k]);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            o.Fe.m[3 * i + k] = (U[3 * i] * ex[0]) * V[3 * k] + (U[3 * i + 1] * ex[1]) * V[3 * k + 1]
                              + (U[3 * i + 2] * ex[2]) * V[3 * k + 2];
            o.tau.m[3 * i + k] = (U[3 * i] * cs[0]) * U[3 * k] + (U[3 * i + 1] * cs[1]) * U[3 * k + 1]
                               + (U[3 * i + 2] * cs[2]) * U[3 * k + 2];
        }
    if (a == 0.0f) {
        // pow(x, 1/3) of the reference; cube root of the same argument.
        float scale = cbrtf(det_trial / det3(o.Fe));
#pragma unroll
        for (int e = 0; e < 9; ++e) o.Fe.m[e] *= scale;
    }
    o.residual = 0.0f;
    o.yielded = q2 + p2 > 1.0f;
    if (o.yielded) {
        float u = 1.0f + df * r, w = 1.0f + mf * r;
        o.residual = fabsf(r + 1.0f - q2 / (u * u) - p2 / (w * w));
    }
    return o;
}

struct DingParamsDev {
    int coupled_porosity, temperature_enabled;
    float mu, lam, yield_stress, initial_porosity, dt;
    float knots[4], yield_factors[4], viscosity_factors[4];
};

struct DingParticleOut {
    M3 Fe, Fp, tau;
    float residual, porosity, porosity_residual, yield_stress, viscosity;
    int gelled;
    float e[3];     // returned log principal strains, before volume corrections (SVD order)
    bool yielded;
};

// The part of UpdateDing (ding.py:154-180) before the return: gelation latch, temperature tables,
// trial gradient and its SVD.
struct DingPrelude {
    M3 U, V;
    float det_trial;   // det of the trial elastic gradient (the isochoric correction's numerator)
    float s[3], e[3];  // singular values and their logs (svd3f)
    float ty, eta, T_eff;
    int gel;
};

template <bool kPolish = true>
BK_DEV bool ding_prelude(const DingParamsDev& P, const M3& Fe_old, float por, int gel, const M3& C_new, float T,
                         float eta_base, int32_t* flags, DingPrelude& d) {
    if (!isfinite(por) || por < 0.0f || por >= 1.0f) { set_flag(flags, 0); return false; }
    int reached = T >= P.knots[3];
    float Teff = T;
    float ty = P.yield_stress;
    float eta = eta_base;
    if (P.temperature_enabled) {
        if (reached) gel = 1;
        if (gel) Teff = P.knots[3];
        ty = P.yield_stress * temperature_factor(Teff, P.knots, P.yield_factors);
        eta = eta_base * temperature_factor(Teff, P.knots, P.viscosity_factors);
    }
    M3 G;
#pragma unroll
    for (int e = 0; e < 9; ++e) G.m[e] = P.dt * C_new.m[e] + ((e % 4) == 0 ? 1.0f : 0.0f);
    const M3 trial = matmul(G, Fe_old);
    d.det_trial = det3(trial);
    svd3f<kPolish>(trial, d.U, d.s, d.V, d.e);
    d.ty = ty;
    d.eta = eta;
    d.T_eff = Teff;
    d.gel = gel;
    return true;
}

// Where ding_close reads the total gradient F' from: a matrix the caller holds (FInRegs), or the F'
// this thread stored earlier in the same kernel (FStored), read back with plain loads only where
// the close needs it, so that it is not held in registers through the return map.
struct FInRegs {
    const M3& m;
    BK_DEV M3 get() const { return m; }
};
struct FStored {
    const float* p;  // not the read-only path: the data were written during this kernel
    int64_t i, pitch;
    BK_DEV M3 get() const {
        M3 r;
#pragma unroll
        for (int c = 0; c < 9; ++c) r.m[c] = p[c * pitch + i];
        return r;
    }
};

// The float32 rounding of the cube root of v, for the volume corrections, whose ratios lie within
// ~1e-6 of 1 (they undo spectral reconstruction roundoff). Near 1 it sums the binomial series
// (1 + d)^(1/3) = 1 + d/3 - d^2/9 + 5 d^3/81 - 10 d^4/243 + ...; for |d| < 2^-10 the omitted terms
// are below 3e-17, so the rounded result is that of the float64 cube root unless the root lies
// within ~2e-16 (relative) of a float32 rounding boundary. Elsewhere it calls cbrt.
BK_DEV float cbrt_near_one(double v) {
    const double d = v - 1.0;
    if (fabs(d) < 0x1p-10) return (float)(1.0 + d * (1.0 / 3.0 + d * (-1.0 / 9.0 + d * (5.0 / 81.0 - d * (10.0 / 243.0)))));
    return (float)cbrt(v);
}

// Volume correction (gas mode), plastic gradient and porosity update shared by the exact and the
// surrogate returns (ding.py:200-221).
template <class FSrc>
BK_DEV void ding_close(const DingParamsDev& P, float por, const FSrc& F_src, float ret_por, M3 Fe, int32_t* flags,
                       DingParticleOut& out, bool need_fp) {
    const float n0 = P.initial_porosity;
    const M3 F_tot = F_src.get();
    if (P.coupled_porosity) {
        double target = 1.0 - (double)n0 + (double)ret_por;
        M3d Fd, Fed;
#pragma unroll
        for (int e = 0; e < 9; ++e) { Fd.m[e] = (double)F_tot.m[e]; Fed.m[e] = (double)Fe.m[e]; }
        double vs = det3(Fd) / (target * det3(Fed));
        float scale = cbrt_near_one(vs);  // pow(vs, 1/3) in the reference
#pragma unroll
        for (int e = 0; e < 9; ++e) Fe.m[e] *= scale;
    }
    M3 Fp;
    float npor;
    if (P.coupled_porosity) {
        npor = ret_por;
        if (need_fp) Fp = matmul(inverse3(Fe), F_tot);
    } else {
        Fp = matmul(inverse3(Fe), F_tot);
        npor = det3(Fp) - 1.0f + n0;
    }
    if (n0 == 0.0f && por == 0.0f) npor = 0.0f;
    if (!isfinite(npor) || npor < 0.0f || npor >= 1.0f) set_flag(flags, 0);
    out.Fe = Fe;
    out.Fp = Fp;
    out.porosity = npor;
}

// The exact return of UpdateDing after the prelude (ding.py:181-221).
template <class FSrc>
BK_DEV void ding_exact(const DingParamsDev& P, const DingPrelude& d, float por, const FSrc& F_tot, int32_t* flags,
                       DingParticleOut& out, bool need_fp) {
    const float dt = P.dt, mu = P.mu, lam = P.lam, n0 = P.initial_porosity;
    const float ty = d.ty, eta = d.eta;
    float ret_por = por, consistency = 0.0f;
    double r_warm = 0.0;  // overstress root carried from one solve to the next
    if (P.coupled_porosity) {
        const float* st = d.e;
        float tr = st[0] + st[1] + st[2];
        float ts[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) ts[k] = 2.0f * mu * st[k] + lam * tr;
        float mean = (ts[0] + ts[1] + ts[2]) / 3.0f;
        float dev[3] = {ts[0] - mean, ts[1] - mean, ts[2] - mean};
        float ty2 = ty * ty;
        float qv = 1.5f * (dev[0] * dev[0] + dev[1] * dev[1] + dev[2] * dev[2]) / ty2;
        float pv = mean * mean / ty2;
        float df = 6.0f * mu * dt * ty * ty / eta;
        float ms = 2.0f / 3.0f * (2.0f * mu + 3.0f * lam) * dt * ty * ty / eta;
        float ex = 3.0f * mean / (2.0f * mu + 3.0f * lam);
        double Vp = 1.0 - (double)n0 + (double)por;
        bool elastic_exit;
        ret_por = solve_porosity(qv, pv, df, ms, ex, Vp, n0, &r_warm, &elastic_exit);
        // Certain elastic exit: prediction(ret_por) has r = 0 and returns Vp - 1 + n0 exactly.
        double pred = elastic_exit ? Vp - 1.0 + (double)n0
                                   : porosity_prediction((double)ret_por, qv, pv, df, ms, ex, Vp, n0, &r_warm);
        consistency = (float)fabs((double)ret_por - pred);
        if (consistency > 1.0e-6f || ret_por <= 0.0f || ret_por >= 1.0f) set_flag(flags, 1);
    }
    DingOut r = ding_return(d.det_trial, d.U, d.e, d.V, mu, lam, ty, eta, porosity_coefficient(ret_por), dt,
                            (float)r_warm);
    ding_close(P, por, F_tot, ret_por, r.Fe, flags, out, need_fp);
    out.tau = r.tau;
    out.residual = r.residual;
    out.porosity_residual = consistency;
    out.yield_stress = ty;
    out.viscosity = eta;
    out.gelled = d.gel;
#pragma unroll
    for (int k = 0; k < 3; ++k) out.e[k] = r.e[k];
    out.yielded = r.yielded;
}

// UpdateDing for one particle (ding.py:154-221). Returns false when the old porosity is
// outside [0, 1) (flag 0 set, nothing written, as in the reference). Fp = Fe^-1 F is formed
// only when `need_fp` or when the porosity update needs it (uncoupled mode).
BK_DEV bool update_ding_particle(const DingParamsDev& P, const M3& Fe_old, float por, int gel, const M3& F_tot,
                                 const M3& C_new, float T, float eta_base, int32_t* flags, DingParticleOut& out,
                                 bool need_fp = true) {
    DingPrelude d;
    if (!ding_prelude(P, Fe_old, por, gel, C_new, T, eta_base, flags, d)) return false;
    ding_exact(P, d, por, FInRegs{F_tot}, flags, out, need_fp);
    return true;
}

// --------------------------------------------------- gas.py:7-13
constexpr double kGasConstant = 8.31446261815324;

BK_DEV double gas_pressure(double moles, float T, float J, float n) {
    return moles * kGasConstant * (double)T / ((double)J * (double)n);
}

// Threads per vertex block for surface vertices with `bindings` particle bindings in total: a
// block's worth of gathers in flight for vertices binding thousands of particles (large bodies),
// one warp for vertices binding tens (small bodies, or an unknown count).
inline int vertex_block_threads(int64_t vertices, int64_t bindings) {
    const int64_t mean = vertices > 0 ? bindings / vertices : 0;
    return mean >= 1024 ? 256 : (mean >= 128 ? 128 : 32);
}

// ------------------------------------------- geometry/mesh_tracking.py:13-38
// One mesh vertex reconstructed by a whole block of kBlock threads: anchor + sum_b w_b (pred_b -
// anchor) over its bindings b0..b1, pred_b = x_p + F_p o_b (o_b: the binding's reference offset,
// 3 planes of `bp`), the anchor being the first binding's prediction; a vertex without bindings
// keeps its reference position. Every thread of the block must call it (it synchronises the block);
// threads 0, 1, 2 get components x, y, z.
template <int kBlock>
BK_DEV float vertex_block(const int* __restrict__ offsets, const int* __restrict__ particles,
                          const float* __restrict__ weights, const float* __restrict__ ref_offsets, int64_t bp,
                          const float* __restrict__ ref_vertices, int64_t vp, const float* __restrict__ x,
                          const float* __restrict__ F, int64_t pitch, int vid) {
    __shared__ float s_part[3][kBlock / 32];
    const int b0 = offsets[vid], b1 = offsets[vid + 1];
    const int t = threadIdx.x;
    if (b0 == b1) return t < 3 ? ref_vertices[t * vp + vid] : 0.0f;  // the same branch for the whole block
    auto predict = [&](int b, float* r) {
        const int p = particles[b];
        const M3 f = load_m3(F, p, pitch);
        const V3 xp = load_v3(x, p, pitch);
        const float o[3] = {ref_offsets[b], ref_offsets[bp + b], ref_offsets[2 * bp + b]};
#pragma unroll
        for (int a = 0; a < 3; ++a) r[a] = xp.v[a] + (f.m[3 * a] * o[0] + f.m[3 * a + 1] * o[1] + f.m[3 * a + 2] * o[2]);
    };
    float anchor[3];
    predict(b0, anchor);
    float disp[3] = {0.f, 0.f, 0.f};
#pragma unroll 4
    for (int b = b0 + t; b < b1; b += kBlock) {  // unrolled: several bindings' gathers in flight
        float pr[3];
        predict(b, pr);
        const float w = weights[b];
#pragma unroll
        for (int a = 0; a < 3; ++a) disp[a] += w * (pr[a] - anchor[a]);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) disp[a] += __shfl_xor_sync(0xffffffffu, disp[a], o);
    if ((t & 31) == 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) s_part[a][t >> 5] = disp[a];
    }
    __syncthreads();
    float out = 0.0f;
    if (t < 3) {
        float sum = 0.0f;
        for (int w = 0; w < kBlock / 32; ++w) sum += s_part[t][w];
        out = anchor[t] + sum;
    }
    return out;
}

// The same reconstruction by one warp (lanes stride over the bindings) for vertices binding a few
// tens of particles (a fine mesh), so that a block can hold several vertices; no block barrier.
// Lane a < 3 returns coordinate a. The warp's sum is lane 0's butterfly result, as in vertex_block
// with one warp, so both give the same bits.
BK_DEV float vertex_warp(const int* __restrict__ offsets, const int* __restrict__ particles,
                         const float* __restrict__ weights, const float* __restrict__ ref_offsets, int64_t bp,
                         const float* __restrict__ ref_vertices, int64_t vp, const float* __restrict__ x,
                         const float* __restrict__ F, int64_t pitch, int vid) {
    const int b0 = offsets[vid], b1 = offsets[vid + 1];
    const int lane = threadIdx.x & 31;
    if (b0 == b1) return lane < 3 ? ref_vertices[lane * vp + vid] : 0.0f;  // the same branch for the warp
    auto predict = [&](int b, float* r) {
        const int p = particles[b];
        const M3 f = load_m3(F, p, pitch);
        const V3 xp = load_v3(x, p, pitch);
        const float o[3] = {ref_offsets[b], ref_offsets[bp + b], ref_offsets[2 * bp + b]};
#pragma unroll
        for (int a = 0; a < 3; ++a) r[a] = xp.v[a] + (f.m[3 * a] * o[0] + f.m[3 * a + 1] * o[1] + f.m[3 * a + 2] * o[2]);
    };
    float anchor[3];
    predict(b0, anchor);
    float disp[3] = {0.f, 0.f, 0.f};
#pragma unroll 4
    for (int b = b0 + lane; b < b1; b += 32) {
        float pr[3];
        predict(b, pr);
        const float w = weights[b];
#pragma unroll
        for (int a = 0; a < 3; ++a) disp[a] += w * (pr[a] - anchor[a]);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) disp[a] += __shfl_xor_sync(0xffffffffu, disp[a], o);
        disp[a] = __shfl_sync(0xffffffffu, disp[a], 0);
    }
    float out = 0.0f;
#pragma unroll
    for (int a = 0; a < 3; ++a)
        if (lane == a) out = anchor[a] + disp[a];
    return out;
}

}  // namespace bk
