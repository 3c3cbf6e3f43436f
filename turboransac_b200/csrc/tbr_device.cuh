// Device building blocks of the absolute-pose engine (sm_100a).
//
//  * Philox4x32-10 counter-based sampler and the without-replacement triple draw
//  * FP64 Lambda-Twist-type P3P, following the reference's p3p.cuh:9-222 and
//    p3p_utils.cuh:192-422 branch for branch (same eps constants, same
//    solution order) so that replayed samples give the reference's hypotheses
//  * FP64 quaternion helpers (pose_utils.cuh:13-188)
//  * packed FP32x2 arithmetic (Blackwell fma/mul/add .f32x2) for the scoring pass
//  * bulk-copy (TMA, 1-D) + mbarrier helpers with bounded waits
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tbr {

// ------------------------------------------------------------------ Philox --
// Philox4x32 with 10 rounds (Salmon, Moraes, Dror, Shaw, SC'11): published
// round multipliers and Weyl key increments.
__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
        c[1] = (uint32_t)p1;
        c[3] = (uint32_t)p0;
        c[0] = n0;
        c[2] = n2;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

__host__ __device__ __forceinline__ uint32_t mulhi_range(uint32_t r, uint32_t n) {
    return (uint32_t)(((uint64_t)r * n) >> 32);
}

// Sample `sample` of the stream keyed by `seed`: an ordered triple of distinct
// indices in [0, n), drawn without replacement in one shot (no rejection loop,
// so no unbounded retry for small n).
__host__ __device__ __forceinline__ void draw_triple(uint64_t seed, uint64_t sample, uint32_t n,
                                                     int32_t out[3]) {
    uint32_t c[4] = {(uint32_t)sample, (uint32_t)(sample >> 32), 0u, 0u};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    uint32_t i0 = mulhi_range(c[0], n);
    uint32_t i1 = mulhi_range(c[1], n - 1);
    if (i1 >= i0) ++i1;
    uint32_t i2 = mulhi_range(c[2], n - 2);
    const uint32_t lo = i0 < i1 ? i0 : i1, hi = i0 < i1 ? i1 : i0;
    if (i2 >= lo) ++i2;
    if (i2 >= hi) ++i2;
    out[0] = (int32_t)i0;
    out[1] = (int32_t)i1;
    out[2] = (int32_t)i2;
}

// PROSAC ordered triple (Chum & Matas, CVPR 2005) of sample `sample` (0-based;
// iteration t = sample + 1) over points sorted by quality. Tp[k-3] = T'_k for
// k = 3..n (growth table). With g = #{k in 3..n-1 : T'_k <= t} and m = 3 + g,
// the triple is two distinct indices of the first m-1 points and point m-1;
// once m = n and T'_n < t it is the uniform triple of draw_triple.
__device__ __forceinline__ void prosac_triple(uint64_t seed, uint64_t sample, uint32_t n, const int64_t *Tp,
                                              int32_t out[3]) {
    const int64_t t = (int64_t)sample + 1;
    int64_t lo = 0, hi = (int64_t)n - 3;  // first entry of Tp[0, n-3) above t
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (Tp[mid] <= t) lo = mid + 1;
        else hi = mid;
    }
    const uint32_t m = 3u + (uint32_t)lo;
    if (m >= n && Tp[n - 3] < t) {
        draw_triple(seed, sample, n, out);
        return;
    }
    uint32_t c[4] = {(uint32_t)sample, (uint32_t)(sample >> 32), 0u, 0u};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    uint32_t i0 = mulhi_range(c[0], m - 1);
    uint32_t i1 = mulhi_range(c[1], m - 2);
    if (i1 >= i0) ++i1;
    out[0] = (int32_t)i0;
    out[1] = (int32_t)i1;
    out[2] = (int32_t)(m - 1);
}

// ------------------------------------------------------------- FP64 math ----
struct d3 {
    double x, y, z;
};
__device__ __forceinline__ d3 d3sub(d3 a, d3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ d3 d3neg(d3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ double d3dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ d3 d3cross(d3 a, d3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// Bearing (x, y, 1)/||.|| of a normalized image point (ransac.cuh:196-200).
__device__ __forceinline__ d3 bearing(double x, double y) {
    const double z = x * x + y * y + 1.0;
    if (z > 0.0) {
        const double nrm = sqrt(z);
        return {x / nrm, y / nrm, 1.0 / nrm};
    }
    return {x, y, 1.0};
}

// The reference's eps constants are float literals cast to double (config.h:4,20-22).
#define TBR_EPS_ROOT2REAL ((double)1e-6f)
#define TBR_EPS_REFINE ((double)1e-6f)

// Cubic x^3 + c2 x^2 + c1 x + c0: one real root; true only in the Cardano
// branch (p3p_utils.cuh:393-422).
__device__ __forceinline__ bool cubic_one_root(double c2, double c1, double c0, double &root) {
    double a = c1 - c2 * c2 / 3.0;
    double b = (2.0 * c2 * c2 * c2 - 9.0 * c2 * c1) / 27.0 + c0;
    double c = b * b / 4.0 + a * a * a / 27.0;
    if (c != 0.0) {
        if (c > 0.0) {
            c = sqrt(c);
            b *= -0.5;
            root = cbrt(b + c) + cbrt(b - c) - c2 / 3.0;
            return true;
        }
        c = 3.0 * b / (2.0 * a) * sqrt(-3.0 / a);
        root = 2.0 * sqrt(-a / 3.0) * cos(acos(c) / 3.0) - c2 / 3.0;
    } else {
        root = -c2 / 3.0 + ((a != 0.0) ? (3.0 * b / a) : 0.0);
    }
    return false;
}

// Real roots of x^2 + b x + c (p3p_utils.cuh:295-327).
__device__ __forceinline__ bool quad_roots(double b, double c, double &r1, double &r2) {
    const double v = b * b - 4.0 * c;
    if (v < TBR_EPS_ROOT2REAL) {
        r1 = r2 = -0.5 * b;
        return false;
    }
    const double y = sqrt(v);
    if (b < 0.0) {
        r1 = 0.5 * (-b + y);
        r2 = 0.5 * (-b - y);
    } else {
        r1 = 2.0 * c / (-b + y);
        r2 = 2.0 * c / (-b - y);
    }
    return true;
}

// Gauss-Newton polish of the three depths (p3p_utils.cuh:329-360).
__device__ __forceinline__ void polish_depths(double &d0, double &d1, double &d2, double a01,
                                              double a02, double a12, double m01, double m02,
                                              double m12) {
    for (int it = 0; it < 5; ++it) {
        const double l1 = d0, l2 = d1, l3 = d2;
        const double r1 = l1 * l1 - 2.0 * l1 * l2 * m01 + l2 * l2 - a01;
        const double r2 = l1 * l1 - 2.0 * l1 * l3 * m02 + l3 * l3 - a02;
        const double r3 = l2 * l2 - 2.0 * l2 * l3 * m12 + l3 * l3 - a12;
        if (fabs(r1) + fabs(r2) + fabs(r3) < TBR_EPS_REFINE) return;
        const double x11 = l1 - l2 * m01, x12 = l2 - l1 * m01;
        const double x21 = l1 - l3 * m02, x23 = l3 - l1 * m02;
        const double x32 = l2 - l3 * m12, x33 = l3 - l2 * m12;
        const double detJ = 0.5 / (x11 * x23 * x32 + x12 * x21 * x33);
        d0 += (-x23 * x32 * r1 - x12 * x33 * r2 + x12 * x23 * r3) * detJ;
        d1 += (-x21 * x33 * r1 + x11 * x33 * r2 - x11 * x23 * r3) * detJ;
        d2 += (x21 * x32 * r1 - x11 * x32 * r2 - x12 * x21 * r3) * detJ;
    }
}

// Pose from three bearings x[], world points X[] and depths (p3p.cuh:155-172):
// R = [v1 v2 v1xv2] * inv([X01 X02 X01xX02]), t = d0 x0 - R X0. P: [R | t] row-major.
__device__ __forceinline__ void pose_from_depths(const d3 x[3], const d3 &X0, double d0, double d1,
                                                 double d2, const double *Mi, double *P) {
    const d3 v1 = {d0 * x[0].x - d1 * x[1].x, d0 * x[0].y - d1 * x[1].y, d0 * x[0].z - d1 * x[1].z};
    const d3 v2 = {d0 * x[0].x - d2 * x[2].x, d0 * x[0].y - d2 * x[2].y, d0 * x[0].z - d2 * x[2].z};
    const d3 v3 = d3cross(v1, v2);
    const double Y[9] = {v1.x, v2.x, v3.x, v1.y, v2.y, v3.y, v1.z, v2.z, v3.z};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < 3; ++k) s += Y[i * 3 + k] * Mi[k * 3 + j];
            P[i * 4 + j] = s;
        }
    }
    const double dx[3] = {d0 * x[0].x, d0 * x[0].y, d0 * x[0].z};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        double s = 0.0;
        s += P[i * 4 + 0] * X0.x;
        s += P[i * 4 + 1] * X0.y;
        s += P[i * 4 + 2] * X0.z;
        P[i * 4 + 3] = dx[i] - s;
    }
}

// What every candidate of one P3P sample needs after the root filters: the
// reordered bearings and first world point, inv([X01 X02 X01xX02]) and the
// squared distances / bearing cosines of the depth polish.
struct P3PCtx {
    d3 x[3];
    d3 X0;
    double Mi[9];
    double a01, a02, a12, m01, m02, m12;
};

// P3P for three unit bearings and world points, up to the candidates: the
// depth triples that pass the root filters, in the order p3p.cuh:9-222 visits
// them (line 0 then 1, root 0 then 1, the same early exit after line 0),
// written to dep[3*k]; returns their number. Same reorder, conic split and
// root filters as there.
__device__ int p3p_candidates(const d3 xin[3], const d3 Xin[3], P3PCtx &c, double *dep) {
    d3 x[3] = {xin[0], xin[1], xin[2]};
    d3 X[3] = {Xin[0], Xin[1], Xin[2]};
    d3 X01 = d3sub(X[0], X[1]);
    d3 X02 = d3sub(X[0], X[2]);
    const d3 X12 = d3sub(X[1], X[2]);
    double a01 = d3dot(X01, X01), a02 = d3dot(X02, X02), a12 = d3dot(X12, X12);
    if (a01 > a02) {
        if (a01 > a12) {
            d3 tx = x[0]; x[0] = x[2]; x[2] = tx;
            d3 tX = X[0]; X[0] = X[2]; X[2] = tX;
            double ta = a01; a01 = a12; a12 = ta;
            X01 = d3neg(X12);
            X02 = d3neg(X02);
        }
    } else if (a02 > a12) {
        d3 tx = x[0]; x[0] = x[1]; x[1] = tx;
        d3 tX = X[0]; X[0] = X[1]; X[1] = tX;
        double ta = a02; a02 = a12; a12 = ta;
        X01 = d3neg(X01);
        X02 = X12;
    }
    const double a12_inv = 1.0 / a12;
    const double a = a01 * a12_inv;
    const double b = a02 * a12_inv;
    const double m01 = d3dot(x[0], x[1]);
    const double m02 = d3dot(x[0], x[2]);
    const double m12 = d3dot(x[1], x[2]);
    const double m12sq = -m12 * m12 + 1.0;
    const double m02sq = -1.0 + m02 * m02;
    const double m01sq = -1.0 + m01 * m01;
    const double ab = a * b, bsq = b * b, asq = a * a;
    const double m013 = -2.0 + 2.0 * m01 * m02 * m12;
    const double bsqm12sq = bsq * m12sq, asqm12sq = asq * m12sq, abm12sq = 2.0 * ab * m12sq;
    const double k3_inv = 1.0 / (bsqm12sq + b * m02sq);
    const double k2 = k3_inv * ((-1.0 + a) * m02sq + abm12sq + bsqm12sq + b * m013);
    const double k1 = k3_inv * (asqm12sq + abm12sq + a * m013 + (-1.0 + b) * m01sq);
    const double k0 = k3_inv * (asqm12sq + a * m01sq);
    double s;
    const bool G = cubic_one_root(k2, k1, k0, s);

    // Degenerate conic C and its split into two lines p, q (p3p_utils.cuh:192-241).
    const double C00 = -a + s * (1.0 - b), C01 = -m02 * s, C02 = a * m12 + b * m12 * s;
    const double C11 = s + 1.0, C12 = -m01, C22 = -a - b * s + 1.0;
    const double A00 = C12 * C12 - C11 * C22;
    const double A11 = C02 * C02 - C00 * C22;
    const double A22 = C01 * C01 - C00 * C11;
    const double A01 = C01 * C22 - C02 * C12;
    const double A02 = C02 * C11 - C01 * C12;
    const double A12 = C00 * C12 - C02 * C01;
    double v0, v1, v2;
    {
        int col;
        if (A00 > A11) col = (A00 > A22) ? 0 : 2;
        else col = (A11 > A22) ? 1 : 2;
        const double c0 = col == 0 ? A00 : (col == 1 ? A01 : A02);
        const double c1 = col == 0 ? A01 : (col == 1 ? A11 : A12);
        const double c2 = col == 0 ? A02 : (col == 1 ? A12 : A22);
        const double sq = sqrt(col == 0 ? A00 : (col == 1 ? A11 : A22));
        v0 = c0 / sq; v1 = c1 / sq; v2 = c2 / sq;
    }
    const double M01 = C01 - v2, M02 = C02 + v1, M10 = C01 + v2, M20 = C02 - v1;
    const double pq[2][3] = {{C00, M10, M20}, {C00, M01, M02}};

    // inv([X01 X02 X01xX02]) (p3p_utils.cuh:259-293; identity if singular).
    const d3 c3 = d3cross(X01, X02);
    const double m[9] = {X01.x, X02.x, c3.x, X01.y, X02.y, c3.y, X01.z, X02.z, c3.z};
    double Mi[9];
    {
        const double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                           m[2] * (m[3] * m[7] - m[4] * m[6]);
        if (det == 0.0) {
#pragma unroll
            for (int i = 0; i < 9; ++i) Mi[i] = (i % 4 == 0) ? 1.0 : 0.0;
        } else {
            Mi[0] = (m[4] * m[8] - m[5] * m[7]) / det;
            Mi[1] = -(m[1] * m[8] - m[2] * m[7]) / det;
            Mi[2] = (m[1] * m[5] - m[2] * m[4]) / det;
            Mi[3] = -(m[3] * m[8] - m[5] * m[6]) / det;
            Mi[4] = (m[0] * m[8] - m[2] * m[6]) / det;
            Mi[5] = -(m[0] * m[5] - m[2] * m[3]) / det;
            Mi[6] = (m[3] * m[7] - m[4] * m[6]) / det;
            Mi[7] = -(m[0] * m[7] - m[1] * m[6]) / det;
            Mi[8] = (m[0] * m[4] - m[1] * m[3]) / det;
        }
    }

    for (int k = 0; k < 3; ++k) c.x[k] = x[k];
    c.X0 = X[0];
    for (int k = 0; k < 9; ++k) c.Mi[k] = Mi[k];
    c.a01 = a01, c.a02 = a02, c.a12 = a12, c.m01 = m01, c.m02 = m02, c.m12 = m12;
    int n_sols = 0;
    for (int i = 0; i < 2; ++i) {
        const double p0 = pq[i][0], p1 = pq[i][1], p2 = pq[i][2];
        if (fabs(p0) <= fabs(p1)) {
            const double w0 = -p0 / p1, w1 = -p2 / p1;
            const double ca = 1.0 / (w1 * w1 - b);
            const double cb = 2.0 * (b * m12 - m02 * w1 + w0 * w1) * ca;
            const double cc = (w0 * w0 - 2.0 * m02 * w0 - b + 1.0) * ca;
            double taus[2];
            if (!quad_roots(cb, cc, taus[0], taus[1])) continue;
            for (int k = 0; k < 2; ++k) {
                const double tau = taus[k];
                if (tau <= 0) continue;
                double d2 = sqrt(a12 / (tau * (tau - 2.0 * m12) + 1.0));
                double d1 = tau * d2;
                double d0 = (w0 * d2 + w1 * d1);
                if (d0 < 0) continue;
                dep[3 * n_sols] = d0, dep[3 * n_sols + 1] = d1, dep[3 * n_sols + 2] = d2;
                ++n_sols;
            }
        } else {
            const double w0 = -p1 / p0, w1 = -p2 / p0;
            const double ca = 1.0 / (-a * w1 * w1 + 2.0 * a * m12 * w1 - a + 1.0);
            const double cb = 2.0 * (a * m12 * w0 - m01 - a * w0 * w1) * ca;
            const double cc = (1.0 - a * w0 * w0) * ca;
            double taus[2];
            if (!quad_roots(cb, cc, taus[0], taus[1])) continue;
            for (int k = 0; k < 2; ++k) {
                const double tau = taus[k];
                if (tau <= 0.0) continue;
                double d0 = sqrt(a01 / (tau * (tau - 2.0 * m01) + 1.0));
                double d1 = tau * d0;
                double d2 = w0 * d0 + w1 * d1;
                if (d2 < 0.0) continue;
                dep[3 * n_sols] = d0, dep[3 * n_sols + 1] = d1, dep[3 * n_sols + 2] = d2;
                ++n_sols;
            }
        }
        if (n_sols > 0 && G) break;
    }
    return n_sols;
}

// One candidate of p3p_candidates to its pose (12 doubles, row-major [R | t]):
// the depth polish, then the pose from the depths (p3p.cuh's inner loop).
__device__ __forceinline__ void p3p_finish(const P3PCtx &c, double d0, double d1, double d2, double *P) {
    polish_depths(d0, d1, d2, c.a01, c.a02, c.a12, c.m01, c.m02, c.m12);
    pose_from_depths(c.x, c.X0, d0, d1, d2, c.Mi, P);
}

// P3P for three unit bearings and world points; up to 4 poses written to
// out[12*k]; returns their number (p3p.cuh:9-222).
__device__ __forceinline__ int p3p_solve(const d3 xin[3], const d3 Xin[3], double *out) {
    P3PCtx c;
    double dep[12];
    const int n = p3p_candidates(xin, Xin, c, dep);
    for (int k = 0; k < n; ++k) p3p_finish(c, dep[3 * k], dep[3 * k + 1], dep[3 * k + 2], out + 12 * k);
    return n;
}

// ---------------------------------------------------------- quaternions -----
// R (row-major) -> unit quaternion (w, x, y, z), Shepperd branches then
// normalisation (pose_utils.cuh:13-58).
__host__ __device__ __forceinline__ void rotmat_to_quat(const double *R, double q[4]) {
    const double trace = R[0] + R[4] + R[8];
    if (trace > 0.0) {
        const double s = 0.5 / sqrt(trace + 1.0);
        q[0] = 0.25 / s;
        q[1] = (R[7] - R[5]) * s;
        q[2] = (R[2] - R[6]) * s;
        q[3] = (R[3] - R[1]) * s;
    } else if (R[0] > R[4] && R[0] > R[8]) {
        const double s = 2.0 * sqrt(1.0 + R[0] - R[4] - R[8]);
        q[0] = (R[7] - R[5]) / s;
        q[1] = 0.25 * s;
        q[2] = (R[1] + R[3]) / s;
        q[3] = (R[2] + R[6]) / s;
    } else if (R[4] > R[8]) {
        const double s = 2.0 * sqrt(1.0 + R[4] - R[0] - R[8]);
        q[0] = (R[2] - R[6]) / s;
        q[1] = (R[1] + R[3]) / s;
        q[2] = 0.25 * s;
        q[3] = (R[5] + R[7]) / s;
    } else {
        const double s = 2.0 * sqrt(1.0 + R[8] - R[0] - R[4]);
        q[0] = (R[3] - R[1]) / s;
        q[1] = (R[2] + R[6]) / s;
        q[2] = (R[5] + R[7]) / s;
        q[3] = 0.25 * s;
    }
    const double z = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
    if (z > 0.0) {
        const double nrm = sqrt(z);
        q[0] /= nrm; q[1] /= nrm; q[2] /= nrm; q[3] /= nrm;
    }
}

// pose_utils.cuh:60-82
__host__ __device__ __forceinline__ void quat_to_rotmat(const double q[4], double *R) {
    const double w = q[0], x = q[1], y = q[2], z = q[3];
    R[0] = 1.0 - 2.0 * (y * y + z * z);
    R[1] = 2.0 * (x * y - z * w);
    R[2] = 2.0 * (x * z + y * w);
    R[3] = 2.0 * (x * y + z * w);
    R[4] = 1.0 - 2.0 * (x * x + z * z);
    R[5] = 2.0 * (y * z - x * w);
    R[6] = 2.0 * (x * z - y * w);
    R[7] = 2.0 * (y * z + x * w);
    R[8] = 1.0 - 2.0 * (x * x + y * y);
}

// pose_utils.cuh:107-131
__device__ __forceinline__ void quat_rotate(const double *q, double p1, double p2, double p3,
                                            double *out) {
    const double q1 = q[0], q2 = q[1], q3 = q[2], q4 = q[3];
    const double px1 = -p1 * q2 - p2 * q3 - p3 * q4;
    const double px2 = p1 * q1 - p2 * q4 + p3 * q3;
    const double px3 = p2 * q1 + p1 * q4 - p3 * q2;
    const double px4 = p2 * q2 - p1 * q3 + p3 * q1;
    out[0] = px2 * q1 - px1 * q2 - px3 * q4 + px4 * q3;
    out[1] = px3 * q1 - px1 * q3 + px2 * q4 - px4 * q2;
    out[2] = px3 * q2 - px2 * q3 - px1 * q4 + px4 * q1;
}

// q <- q * exp(w) (quat_step_post with quat_exp's Taylor branch, pose_utils.cuh:138-188).
__device__ __forceinline__ void quat_step_post(const double *q, const double *w, double *out) {
    const double theta2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
    const double theta = sqrt(theta2);
    const double th = 0.5 * theta;
    double re, im;
    if (theta > 1e-6) {
        re = cos(th);
        im = sin(th) / theta;
    } else {
        const double theta4 = theta2 * theta2;
        re = 1.0 - (1.0 / 8.0) * theta2 + (1.0 / 384.0) * theta4;
        im = 0.5 - (1.0 / 48.0) * theta2 + (1.0 / 3840.0) * theta4;
        const double s = sqrt(re * re + im * im * theta2);
        re /= s;
        im /= s;
    }
    const double b[4] = {re, im * w[0], im * w[1], im * w[2]};
    out[0] = q[0] * b[0] - q[1] * b[1] - q[2] * b[2] - q[3] * b[3];
    out[1] = q[0] * b[1] + q[1] * b[0] + q[2] * b[3] - q[3] * b[2];
    out[2] = q[0] * b[2] + q[2] * b[0] - q[1] * b[3] + q[3] * b[1];
    out[3] = q[0] * b[3] + q[1] * b[2] - q[2] * b[1] + q[3] * b[0];
}

// -------------------------------------------------------- packed FP32x2 -----
// Two FP32 lanes in one 64-bit register: low half = first value.
__device__ __forceinline__ uint64_t f2pack(float lo, float hi) {
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void f2unpack(uint64_t v, float &lo, float &hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ uint64_t f2fma(uint64_t a, uint64_t b, uint64_t c) {
    uint64_t d;
    asm("fma.rn.ftz.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ uint64_t f2mul(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("mul.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ uint64_t f2add(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("add.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
// rn(a*b + c) clamped to [0, 1] (NaN becomes 0).
__device__ __forceinline__ float fma_sat(float a, float b, float c) {
    float d;
    asm("fma.rn.ftz.sat.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// ----------------------------------------------- bulk copy + mbarrier (TMA) --
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// One arrival that also expects `bytes` of transaction, then the copy itself.
__device__ __forceinline__ void bulk_load(void *dst_smem, const void *src_gmem, uint32_t bytes,
                                          uint64_t *bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst_smem)),
        "l"(src_gmem), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
// Bounded wait on phase `parity`; returns false if it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t max_polls) {
    const uint32_t a = smem_addr(bar);
    for (uint32_t i = 0; i < max_polls; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Ordered-integer encodings so that atomicMin/atomicMax work on doubles.
__device__ __forceinline__ unsigned long long dbl_to_ordered(double v) {
    const unsigned long long u = (unsigned long long)__double_as_longlong(v);
    return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}
__host__ __device__ __forceinline__ double ordered_to_dbl(unsigned long long o) {
    const unsigned long long u = (o & 0x8000000000000000ull) ? (o & 0x7fffffffffffffffull) : ~o;
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)u);
#else
    double d;
    __builtin_memcpy(&d, &u, 8);
    return d;
#endif
}

}  // namespace tbr
