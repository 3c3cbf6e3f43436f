// FP64 CPU oracle (TEST INFRASTRUCTURE) -- see tbr_oracle.h for the contract.
//
// Every function restates the reference algorithm step by step in plain
// arrays (no Eigen). Expressions keep the reference's association order so
// that, compiled without FMA contraction, results agree with the reference's
// own host-compiled headers to the last bit wherever libm agrees.
// Paths cited are inside the reference project (Module/TbrCudaPnP/...).

#include "tbr_oracle.h"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

namespace {

// ---------------------------------------------------------------- Philox ----
// Philox4x32 with 10 rounds: multipliers and Weyl key increments are the
// published constants of Salmon, Moraes, Dror and Shaw, "Parallel random
// numbers: as easy as 1, 2, 3" (SC'11).
constexpr uint32_t kPhiloxM0 = 0xD2511F53u;
constexpr uint32_t kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u;
constexpr uint32_t kPhiloxW1 = 0xBB67AE85u;

inline void philox(uint32_t c[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)kPhiloxM0 * c[0];
        uint64_t p1 = (uint64_t)kPhiloxM1 * c[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c[1] ^ k0;
        uint32_t n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
        k0 += kPhiloxW0; k1 += kPhiloxW1;
    }
}

inline uint32_t mulhi_range(uint32_t r, uint32_t n) { return (uint32_t)(((uint64_t)r * n) >> 32); }

// Ordered triple of distinct indices, drawn without replacement in one shot:
// i0 uniform on n values, i1 on the n-1 others, i2 on the n-2 others.
inline void triple_from_sample(uint64_t seed, uint64_t sample, uint32_t n, int32_t out[3]) {
    uint32_t c[4] = {(uint32_t)sample, (uint32_t)(sample >> 32), 0u, 0u};
    philox(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    uint32_t i0 = mulhi_range(c[0], n);
    uint32_t i1 = mulhi_range(c[1], n - 1);
    if (i1 >= i0) ++i1;
    uint32_t i2 = mulhi_range(c[2], n - 2);
    uint32_t lo = i0 < i1 ? i0 : i1, hi = i0 < i1 ? i1 : i0;
    if (i2 >= lo) ++i2;
    if (i2 >= hi) ++i2;
    out[0] = (int32_t)i0; out[1] = (int32_t)i1; out[2] = (int32_t)i2;
}

// ------------------------------------------------------------ small math ----
struct V3 { double v[3]; double &operator[](int i) { return v[i]; } double operator[](int i) const { return v[i]; } };

inline V3 sub(const V3 &a, const V3 &b) { return {{a[0] - b[0], a[1] - b[1], a[2] - b[2]}}; }
inline V3 neg(const V3 &a) { return {{-a[0], -a[1], -a[2]}}; }
inline double dot(const V3 &a, const V3 &b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline double sqnorm(const V3 &a) { return a[0] * a[0] + a[1] * a[1] + a[2] * a[2]; }
// cross3, p3p_utils.cuh:182-190
inline V3 cross(const V3 &a, const V3 &b) {
    return {{a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]}};
}

// 3x3 row-major helpers; sums start from 0 as in matmul3x3 / matmul3x1
// (p3p_utils.cuh:117-179).
inline void mat3_mul(const double *A, const double *B, double *C) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += A[i * 3 + k] * B[k * 3 + j];
            C[i * 3 + j] = s;
        }
}
inline V3 mat3_vec(const double *A, const V3 &v) {
    V3 r;
    for (int i = 0; i < 3; ++i) {
        double s = 0.0;
        for (int j = 0; j < 3; ++j) s += A[i * 3 + j] * v[j];
        r[i] = s;
    }
    return r;
}

// inverse3x3, p3p_utils.cuh:259-293 (identity when det == 0).
inline void inverse3(const double *m, double *inv) {
    auto M = [&](int r, int c) { return m[r * 3 + c]; };
    double det = M(0, 0) * (M(1, 1) * M(2, 2) - M(1, 2) * M(2, 1)) -
                 M(0, 1) * (M(1, 0) * M(2, 2) - M(1, 2) * M(2, 0)) +
                 M(0, 2) * (M(1, 0) * M(2, 1) - M(1, 1) * M(2, 0));
    if (det == 0.0) {
        for (int i = 0; i < 9; ++i) inv[i] = (i % 4 == 0) ? 1.0 : 0.0;
        return;
    }
    double a[9];
    a[0] = (M(1, 1) * M(2, 2) - M(1, 2) * M(2, 1));
    a[1] = -(M(0, 1) * M(2, 2) - M(0, 2) * M(2, 1));
    a[2] = (M(0, 1) * M(1, 2) - M(0, 2) * M(1, 1));
    a[3] = -(M(1, 0) * M(2, 2) - M(1, 2) * M(2, 0));
    a[4] = (M(0, 0) * M(2, 2) - M(0, 2) * M(2, 0));
    a[5] = -(M(0, 0) * M(1, 2) - M(0, 2) * M(1, 0));
    a[6] = (M(1, 0) * M(2, 1) - M(1, 1) * M(2, 0));
    a[7] = -(M(0, 0) * M(2, 1) - M(0, 1) * M(2, 0));
    a[8] = (M(0, 0) * M(1, 1) - M(0, 1) * M(1, 0));
    for (int i = 0; i < 9; ++i) inv[i] = a[i] / det;
}

// The reference's eps constants are float literals (config.h:4,20-22) cast to T.
const double kEpsRoot2Real = (double)1e-6f;
const double kEpsRefine = (double)1e-6f;

// solve_cubic_single_real_cuda, p3p_utils.cuh:393-422. Returns true only in the
// one-real-root (Cardano) branch.
inline bool cubic_single_real(double c2, double c1, double c0, double &root) {
    double a = c1 - c2 * c2 / 3.0;
    double b = (2.0 * c2 * c2 * c2 - 9.0 * c2 * c1) / 27.0 + c0;
    double c = b * b / 4.0 + a * a * a / 27.0;
    if (c != 0.0) {
        if (c > 0.0) {
            c = std::sqrt(c);
            b *= -0.5;
            root = std::cbrt(b + c) + std::cbrt(b - c) - c2 / 3.0;
            return true;
        } else {
            c = 3.0 * b / (2.0 * a) * std::sqrt(-3.0 / a);
            root = 2.0 * std::sqrt(-a / 3.0) * std::cos(std::acos(c) / 3.0) - c2 / 3.0;
        }
    } else {
        root = -c2 / 3.0 + ((a != 0.0) ? (3.0 * b / a) : 0.0);
    }
    return false;
}

// root2real_cuda, p3p_utils.cuh:295-327 (the second branch is unreachable but kept).
inline bool root2real(double b, double c, double &r1, double &r2) {
    const double thr = kEpsRoot2Real;
    double v = b * b - 4.0 * c;
    if (v < thr) {
        r1 = r2 = -0.5 * b;
        return false;
    }
    if (v > thr && v < 0.0) {
        r1 = -0.5 * b;
        r2 = -2.0;
        return true;
    }
    double y = std::sqrt(v);
    if (b < 0.0) {
        r1 = 0.5 * (-b + y);
        r2 = 0.5 * (-b - y);
    } else {
        r1 = 2.0 * c / (-b + y);
        r2 = 2.0 * c / (-b - y);
    }
    return true;
}

// refine_lambda_cuda, p3p_utils.cuh:329-360: five Gauss-Newton steps on the depths.
inline void refine_lambda(double &l1o, double &l2o, double &l3o, double a12, double a13,
                          double a23, double b12, double b13, double b23) {
    for (int it = 0; it < 5; ++it) {
        double l1 = l1o, l2 = l2o, l3 = l3o;
        double r1 = l1 * l1 - 2.0 * l1 * l2 * b12 + l2 * l2 - a12;
        double r2 = l1 * l1 - 2.0 * l1 * l3 * b13 + l3 * l3 - a13;
        double r3 = l2 * l2 - 2.0 * l2 * l3 * b23 + l3 * l3 - a23;
        if (std::fabs(r1) + std::fabs(r2) + std::fabs(r3) < kEpsRefine) return;
        double x11 = l1 - l2 * b12;
        double x12 = l2 - l1 * b12;
        double x21 = l1 - l3 * b13;
        double x23 = l3 - l1 * b13;
        double x32 = l2 - l3 * b23;
        double x33 = l3 - l2 * b23;
        double detJ = 0.5 / (x11 * x23 * x32 + x12 * x21 * x33);
        l1o += (-x23 * x32 * r1 - x12 * x33 * r2 + x12 * x23 * r3) * detJ;
        l2o += (-x21 * x33 * r1 + x11 * x33 * r2 - x11 * x23 * r3) * detJ;
        l3o += (x21 * x32 * r1 - x11 * x32 * r2 - x12 * x21 * r3) * detJ;
    }
}

// compute_pq_cuda, p3p_utils.cuh:192-241: split the degenerate conic C into two lines.
inline void compute_pq(const double *C, V3 &p, V3 &q) {
    auto c = [&](int r, int k) { return C[r * 3 + k]; };
    double A[9];
    A[0] = c(1, 2) * c(2, 1) - c(1, 1) * c(2, 2);
    A[4] = c(0, 2) * c(2, 0) - c(0, 0) * c(2, 2);
    A[8] = c(0, 1) * c(1, 0) - c(0, 0) * c(1, 1);
    A[1] = c(0, 1) * c(2, 2) - c(0, 2) * c(2, 1);
    A[2] = c(0, 2) * c(1, 1) - c(0, 1) * c(1, 2);
    A[3] = A[1];
    A[5] = c(0, 0) * c(1, 2) - c(0, 2) * c(1, 0);
    A[6] = A[2];
    A[7] = A[5];
    int col;
    if (A[0] > A[4]) col = (A[0] > A[8]) ? 0 : 2;
    else col = (A[4] > A[8]) ? 1 : 2;
    double s = std::sqrt(A[col * 3 + col]);
    V3 v = {{A[0 * 3 + col] / s, A[1 * 3 + col] / s, A[2 * 3 + col] / s}};
    double M[9];
    std::memcpy(M, C, sizeof(M));
    M[1] -= v[2];
    M[2] += v[1];
    M[5] -= v[0];
    M[3] += v[2];
    M[6] -= v[1];
    M[7] += v[0];
    p = {{M[0], M[3], M[6]}};  // column 0
    q = {{M[0], M[1], M[2]}};  // row 0
}

// The pose assembled for one depth triple (p3p.cuh:155-172 / 197-212).
inline void p3p_emit(const V3 x[3], const V3 X[3], double d0, double d1, double d2,
                     const double *XXinv, double *out) {
    V3 v1 = {{d0 * x[0][0] - d1 * x[1][0], d0 * x[0][1] - d1 * x[1][1], d0 * x[0][2] - d1 * x[1][2]}};
    V3 v2 = {{d0 * x[0][0] - d2 * x[2][0], d0 * x[0][1] - d2 * x[2][1], d0 * x[0][2] - d2 * x[2][2]}};
    V3 v3 = cross(v1, v2);
    double YY[9] = {v1[0], v2[0], v3[0], v1[1], v2[1], v3[1], v1[2], v2[2], v3[2]};
    double R[9];
    mat3_mul(YY, XXinv, R);
    V3 dx = {{d0 * x[0][0], d0 * x[0][1], d0 * x[0][2]}};
    V3 RX = mat3_vec(R, X[0]);
    for (int r = 0; r < 3; ++r) {
        out[r * 4 + 0] = R[r * 3 + 0];
        out[r * 4 + 1] = R[r * 3 + 1];
        out[r * 4 + 2] = R[r * 3 + 2];
        out[r * 4 + 3] = dx[r] - RX[r];
    }
}

// p3p<double>, p3p.cuh:9-222.
int p3p_impl(const double *xin, const double *Xin, double *out) {
    V3 X[3], x[3];
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) { X[i][k] = Xin[i * 3 + k]; x[i][k] = xin[i * 3 + k]; }
    V3 X01 = sub(X[0], X[1]);
    V3 X02 = sub(X[0], X[2]);
    V3 X12 = sub(X[1], X[2]);
    double a01 = sqnorm(X01), a02 = sqnorm(X02), a12 = sqnorm(X12);

    // Reorder so that the pair (1,2) spans the largest side (p3p.cuh:34-53).
    if (a01 > a02) {
        if (a01 > a12) {
            std::swap(x[0], x[2]);
            std::swap(X[0], X[2]);
            std::swap(a01, a12);
            X01 = neg(X12);
            X02 = neg(X02);
        }
    } else if (a02 > a12) {
        std::swap(x[0], x[1]);
        std::swap(X[0], X[1]);
        std::swap(a02, a12);
        X01 = neg(X01);
        X02 = X12;
    }

    const double a12_inv = 1.0 / a12;
    const double a = a01 * a12_inv;
    const double b = a02 * a12_inv;
    const double m01 = dot(x[0], x[1]);
    const double m02 = dot(x[0], x[2]);
    const double m12 = dot(x[1], x[2]);
    const double m12sq = -m12 * m12 + 1.0;
    const double m02sq = -1.0 + m02 * m02;
    const double m01sq = -1.0 + m01 * m01;
    const double ab = a * b;
    const double bsq = b * b;
    const double asq = a * a;
    const double m013 = -2.0 + 2.0 * m01 * m02 * m12;
    const double bsqm12sq = bsq * m12sq;
    const double asqm12sq = asq * m12sq;
    const double abm12sq = 2.0 * ab * m12sq;
    const double k3_inv = 1.0 / (bsqm12sq + b * m02sq);
    const double k2 = k3_inv * ((-1.0 + a) * m02sq + abm12sq + bsqm12sq + b * m013);
    const double k1 = k3_inv * (asqm12sq + abm12sq + a * m013 + (-1.0 + b) * m01sq);
    const double k0 = k3_inv * (asqm12sq + a * m01sq);

    double s;
    bool G = cubic_single_real(k2, k1, k0, s);

    double C[9];
    C[0] = -a + s * (1.0 - b);
    C[1] = -m02 * s;
    C[2] = a * m12 + b * m12 * s;
    C[3] = C[1];
    C[4] = s + 1.0;
    C[5] = -m01;
    C[6] = C[2];
    C[7] = C[5];
    C[8] = -a - b * s + 1.0;
    V3 pq[2];
    compute_pq(C, pq[0], pq[1]);

    V3 c3 = cross(X01, X02);
    double XX[9] = {X01[0], X02[0], c3[0], X01[1], X02[1], c3[1], X01[2], X02[2], c3[2]};
    double XXinv[9];
    inverse3(XX, XXinv);

    int n_sols = 0;
    for (int i = 0; i < 2; ++i) {
        double p0 = pq[i][0], p1 = pq[i][1], p2 = pq[i][2];
        bool switch_12 = std::fabs(p0) <= std::fabs(p1);
        if (switch_12) {
            double w0 = -p0 / p1;
            double w1 = -p2 / p1;
            double ca = 1.0 / (w1 * w1 - b);
            double cb = 2.0 * (b * m12 - m02 * w1 + w0 * w1) * ca;
            double cc = (w0 * w0 - 2.0 * m02 * w0 - b + 1.0) * ca;
            double taus[2];
            if (!root2real(cb, cc, taus[0], taus[1])) continue;
            for (double tau : taus) {
                if (tau <= 0) continue;
                double d2 = std::sqrt(a12 / (tau * (tau - 2.0 * m12) + 1.0));
                double d1 = tau * d2;
                double d0 = (w0 * d2 + w1 * d1);
                if (d0 < 0) continue;
                refine_lambda(d0, d1, d2, a01, a02, a12, m01, m02, m12);
                p3p_emit(x, X, d0, d1, d2, XXinv, out + 12 * n_sols);
                ++n_sols;
            }
        } else {
            double w0 = -p1 / p0;
            double w1 = -p2 / p0;
            double ca = 1.0 / (-a * w1 * w1 + 2.0 * a * m12 * w1 - a + 1.0);
            double cb = 2.0 * (a * m12 * w0 - m01 - a * w0 * w1) * ca;
            double cc = (1.0 - a * w0 * w0) * ca;
            double taus[2];
            if (!root2real(cb, cc, taus[0], taus[1])) continue;
            for (double tau : taus) {
                if (tau <= 0.0) continue;
                double d0 = std::sqrt(a01 / (tau * (tau - 2.0 * m01) + 1.0));
                double d1 = tau * d0;
                double d2 = w0 * d0 + w1 * d1;
                if (d2 < 0.0) continue;
                refine_lambda(d0, d1, d2, a01, a02, a12, m01, m02, m12);
                p3p_emit(x, X, d0, d1, d2, XXinv, out + 12 * n_sols);
                ++n_sols;
            }
        }
        if (n_sols > 0 && G) break;
    }
    return n_sols;
}

// compute_msac_scores per point (msac.cuh:18-56) summed over all points.
inline void msac_impl(const double *xn, const double *X, int64_t n, const double *P, double sq_thr,
                      double &score, int64_t &count) {
    double s = 0.0;
    int64_t c = 0;
    for (int64_t i = 0; i < n; ++i) {
        const double X0 = X[3 * i], X1 = X[3 * i + 1], X2 = X[3 * i + 2];
        const double z0 = P[0] * X0 + P[1] * X1 + P[2] * X2 + P[3];
        const double z1 = P[4] * X0 + P[5] * X1 + P[6] * X2 + P[7];
        const double z2 = P[8] * X0 + P[9] * X1 + P[10] * X2 + P[11];
        const double inv_z2 = 1.0 / z2;
        const double r0 = z0 * inv_z2 - xn[2 * i];
        const double r1 = z1 * inv_z2 - xn[2 * i + 1];
        const double r_sq = r0 * r0 + r1 * r1;
        if (r_sq < sq_thr && z2 > 0.0) {
            s += r_sq;
            ++c;
        }
    }
    score = s + (double)(n - c) * sq_thr;  // ransac.cuh:322
    count = c;
}

// ------------------------------------------------------------ quaternions --
// rotmat_to_quat, pose_utils.cuh:13-58 (Shepperd branches, then normalize()).
void rotmat_to_quat_impl(const double *R, double q[4]) {
    auto r = [&](int i, int j) { return R[i * 3 + j]; };
    double trace = r(0, 0) + r(1, 1) + r(2, 2);
    if (trace > 0.0) {
        double s = 0.5 / std::sqrt(trace + 1.0);
        q[0] = 0.25 / s;
        q[1] = (r(2, 1) - r(1, 2)) * s;
        q[2] = (r(0, 2) - r(2, 0)) * s;
        q[3] = (r(1, 0) - r(0, 1)) * s;
    } else if (r(0, 0) > r(1, 1) && r(0, 0) > r(2, 2)) {
        double s = 2.0 * std::sqrt(1.0 + r(0, 0) - r(1, 1) - r(2, 2));
        q[0] = (r(2, 1) - r(1, 2)) / s;
        q[1] = 0.25 * s;
        q[2] = (r(0, 1) + r(1, 0)) / s;
        q[3] = (r(0, 2) + r(2, 0)) / s;
    } else if (r(1, 1) > r(2, 2)) {
        double s = 2.0 * std::sqrt(1.0 + r(1, 1) - r(0, 0) - r(2, 2));
        q[0] = (r(0, 2) - r(2, 0)) / s;
        q[1] = (r(0, 1) + r(1, 0)) / s;
        q[2] = 0.25 * s;
        q[3] = (r(1, 2) + r(2, 1)) / s;
    } else {
        double s = 2.0 * std::sqrt(1.0 + r(2, 2) - r(0, 0) - r(1, 1));
        q[0] = (r(1, 0) - r(0, 1)) / s;
        q[1] = (r(0, 2) + r(2, 0)) / s;
        q[2] = (r(1, 2) + r(2, 1)) / s;
        q[3] = 0.25 * s;
    }
    double z = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
    if (z > 0.0) {
        double nrm = std::sqrt(z);
        for (int i = 0; i < 4; ++i) q[i] /= nrm;
    }
}

// quat_to_rotmat, pose_utils.cuh:60-82.
void quat_to_rotmat_impl(const double q[4], double *R) {
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

// quat_multiply, pose_utils.cuh:84-105.
inline void quat_mul(const double *a, const double *b, double *r) {
    r[0] = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
    r[1] = a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2];
    r[2] = a[0] * b[2] + a[2] * b[0] - a[1] * b[3] + a[3] * b[1];
    r[3] = a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0];
}

// quat_rotate, pose_utils.cuh:107-131.
inline void quat_rot(const double *q, const double *p, double *out) {
    const double q1 = q[0], q2 = q[1], q3 = q[2], q4 = q[3];
    const double p1 = p[0], p2 = p[1], p3 = p[2];
    const double px1 = -p1 * q2 - p2 * q3 - p3 * q4;
    const double px2 = p1 * q1 - p2 * q4 + p3 * q3;
    const double px3 = p2 * q1 + p1 * q4 - p3 * q2;
    const double px4 = p2 * q2 - p1 * q3 + p3 * q1;
    out[0] = px2 * q1 - px1 * q2 - px3 * q4 + px4 * q3;
    out[1] = px3 * q1 - px1 * q3 + px2 * q4 - px4 * q2;
    out[2] = px3 * q2 - px2 * q3 - px1 * q4 + px4 * q1;
}

// quat_exp, pose_utils.cuh:138-174 (Taylor branch below 1e-6 rad).
inline void quat_exp(const double *w, double *q) {
    const double theta2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
    const double theta = std::sqrt(theta2);
    const double theta_half = 0.5 * theta;
    double re, im;
    if (theta > 1e-6) {
        re = std::cos(theta_half);
        im = std::sin(theta_half) / theta;
    } else {
        const double theta4 = theta2 * theta2;
        re = 1.0 - (1.0 / 8.0) * theta2 + (1.0 / 384.0) * theta4;
        im = 0.5 - (1.0 / 48.0) * theta2 + (1.0 / 3840.0) * theta4;
        const double s = std::sqrt(re * re + im * im * theta2);
        re /= s;
        im /= s;
    }
    q[0] = re;
    q[1] = im * w[0];
    q[2] = im * w[1];
    q[3] = im * w[2];
}

// ---------------------------------------------------------------- LM -------
struct LMProblem {
    const double *x, *X;
    int64_t n;
    double fx, fy, cx, cy;
    double inv_sq_thr;  // CauchyLoss_cuda, robust_loss.cuh:24-38
    int loss = 0;                    // 0 Cauchy, 1 truncated, 2 Huber, 3 trivial
    const double *w8 = nullptr;      // per-point multipliers (NULL: 1.0, jaco.cuh's uniform weight)
    double thr = 1.0, sq_thr = 1.0;  // loss scale and its square

    double pw(int64_t i) const { return w8 ? w8[i] : 1.0; }
    // loss(r2): CauchyLoss_cuda / TruncatedLoss_cuda (robust_loss.cuh:10-38); Huber
    // and trivial as the published PoseLib losses the option enum names.
    double loss_of(double r2) const {
        switch (loss) {
            case 1: return std::fmin(r2, sq_thr);
            case 2: return r2 <= sq_thr ? r2 : 2.0 * thr * std::sqrt(r2) - sq_thr;
            case 3: return r2;
            default: return std::log1p(r2 * inv_sq_thr);
        }
    }
    double weight_of(double r2) const {
        switch (loss) {
            case 1: return r2 < sq_thr ? 1.0 : 0.0;
            case 2: return r2 <= sq_thr ? 1.0 : thr / std::sqrt(r2);
            case 3: return 1.0;
            default: return std::fmax(DBL_MIN, inv_sq_thr / (1.0 + r2 * inv_sq_thr));
        }
    }

    // residual(), jaco.cuh:31-104: Cauchy cost, points behind the camera dropped.
    double residual(const double *q, const double *t) const {
        double cost = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            double Z[3];
            quat_rot(q, X + 3 * i, Z);
            Z[0] += t[0]; Z[1] += t[1]; Z[2] += t[2];
            const bool valid = Z[2] >= 0.0;
            const double inv_z = valid ? 1.0 / Z[2] : 0.0;
            double p0 = Z[0] * inv_z, p1 = Z[1] * inv_z;
            p0 = fx * p0 + cx;
            p1 = fy * p1 + cy;
            const double r0 = p0 - x[2 * i], r1 = p1 - x[2 * i + 1];
            const double r_squared = r0 * r0 + r1 * r1;
            cost += valid ? pw(i) * loss_of(r_squared) : 0.0;
        }
        return cost;
    }

    // accumulate(), jaco.cuh:106-286: lower triangle of J^T W J and J^T W r.
    void accumulate(const double *q, const double *t, double JtJ[36], double Jtr[6]) const {
        double R[9];
        quat_to_rotmat_impl(q, R);
        for (int k = 0; k < 36; ++k) JtJ[k] = 0.0;
        for (int k = 0; k < 6; ++k) Jtr[k] = 0.0;
        auto J = [&](int i, int j) -> double & { return JtJ[i * 6 + j]; };
        for (int64_t i = 0; i < n; ++i) {
            const double X0 = X[3 * i], X1 = X[3 * i + 1], X2 = X[3 * i + 2];
            V3 Xv = {{X0, X1, X2}};
            V3 RX = mat3_vec(R, Xv);
            const double Z[3] = {RX[0] + t[0], RX[1] + t[1], RX[2] + t[2]};
            const double z0 = Z[0] / Z[2], z1 = Z[1] / Z[2];
            const double zp0 = fx * z0 + cx, zp1 = fy * z1 + cy;
            double r0 = zp0 - x[2 * i], r1 = zp1 - x[2 * i + 1];
            const double r_squared = r0 * r0 + r1 * r1;
            const double weight = pw(i) * weight_of(r_squared);
            const double Z_valid = (Z[2] >= 0.0) ? 1.0 : 0.0;
            const double W_valid = (weight != 0.0) ? 1.0 : 0.0;
            const double valid = Z_valid * W_valid;
            const double w = valid * weight;

            // dZ = (1/Z2) * [Jcam | -Jcam z] * R   (jaco.cuh:163-167)
            double d[2][3];
            d[0][0] = fx; d[0][1] = 0.0;
            d[1][0] = 0.0; d[1][1] = fy;
            d[0][2] = -((0.0 + fx * z0) + 0.0 * z1);
            d[1][2] = -((0.0 + 0.0 * z0) + fy * z1);
            const double iz = 1.0 / Z[2];
            for (int r = 0; r < 2; ++r)
                for (int c = 0; c < 3; ++c) d[r][c] = iz * d[r][c];
            double dZ[2][3];
            for (int r = 0; r < 2; ++r)
                for (int c = 0; c < 3; ++c) {
                    double s = 0.0;
                    for (int k = 0; k < 3; ++k) s += d[r][k] * R[k * 3 + c];
                    dZ[r][c] = s;
                }
            auto cd = [&](int a, int b) { return dZ[0][a] * dZ[0][b] + dZ[1][a] * dZ[1][b]; };
            const double d00 = w * cd(0, 0), d10 = w * cd(1, 0), d11 = w * cd(1, 1);
            const double d20 = w * cd(2, 0), d21 = w * cd(2, 1), d22 = w * cd(2, 2);

            J(0, 0) += X2 * (X2 * d11 - X1 * d21) + X1 * (X1 * d22 - X2 * d21);
            J(1, 0) += -X2 * (X2 * d10 - X0 * d21) - X1 * (X0 * d22 - X2 * d20);
            J(2, 0) += X1 * (X0 * d21 - X1 * d20) - X2 * (X0 * d11 - X1 * d10);
            J(3, 0) += X1 * d20 - X2 * d10;
            J(4, 0) += X1 * d21 - X2 * d11;
            J(5, 0) += X1 * d22 - X2 * d21;
            J(1, 1) += X2 * (X2 * d00 - X0 * d20) + X0 * (X0 * d22 - X2 * d20);
            J(2, 1) += -X2 * (X1 * d00 - X0 * d10) - X0 * (X0 * d21 - X1 * d20);
            J(3, 1) += X2 * d00 - X0 * d20;
            J(4, 1) += X2 * d10 - X0 * d21;
            J(5, 1) += X2 * d20 - X0 * d22;
            J(2, 2) += X1 * (X1 * d00 - X0 * d10) + X0 * (X0 * d11 - X1 * d10);
            J(3, 2) += X0 * d10 - X1 * d00;
            J(4, 2) += X0 * d11 - X1 * d10;
            J(5, 2) += X0 * d21 - X1 * d20;
            J(3, 3) += d00;
            J(4, 3) += d10;
            J(5, 3) += d20;
            J(4, 4) += d11;
            J(5, 4) += d21;
            J(5, 5) += d22;

            r0 *= w;
            r1 *= w;
            Jtr[0] += (r0 * (X1 * dZ[0][2] - X2 * dZ[0][1]) + r1 * (X1 * dZ[1][2] - X2 * dZ[1][1]));
            Jtr[1] += (-r0 * (X0 * dZ[0][2] - X2 * dZ[0][0]) - r1 * (X0 * dZ[1][2] - X2 * dZ[1][0]));
            Jtr[2] += (r0 * (X0 * dZ[0][1] - X1 * dZ[0][0]) + r1 * (X0 * dZ[1][1] - X1 * dZ[1][0]));
            Jtr[3] += (dZ[0][0] * r0 + dZ[1][0] * r1);
            Jtr[4] += (dZ[0][1] * r0 + dZ[1][1] * r1);
            Jtr[5] += (dZ[0][2] * r0 + dZ[1][2] * r1);
        }
    }
};

// choleskyDecompose / forward / backward substitution, lm_utils.cuh:14-100.
void cholesky_solve6(const double A[36], const double b[6], double x[6]) {
    double L[36] = {0};
    const double kEpsilon = 1e-15;
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j <= i; ++j) {
            double sum = 0.0;
            for (int k = 0; k < j; ++k) sum += L[i * 6 + k] * L[j * 6 + k];
            if (i == j) {
                double val = A[i * 6 + i] - sum;
                if (val <= 0.0) val = kEpsilon;
                L[i * 6 + j] = std::sqrt(val);
            } else {
                L[i * 6 + j] = (A[i * 6 + j] - sum) / L[j * 6 + j];
            }
        }
    double y[6];
    for (int i = 0; i < 6; ++i) {
        double sum = 0.0;
        for (int j = 0; j < i; ++j) sum += L[i * 6 + j] * y[j];
        y[i] = (b[i] - sum) / L[i * 6 + i];
    }
    for (int i = 5; i >= 0; --i) {
        double sum = 0.0;
        for (int j = i + 1; j < 6; ++j) sum += L[j * 6 + i] * x[j];
        x[i] = (y[i] - sum) / L[i * 6 + i];
    }
}

inline double norm6(const double *v) {
    double s = 0.0;
    for (int i = 0; i < 6; ++i) s += v[i] * v[i];
    return std::sqrt(s);
}

// lm_impl, lm.cuh:15-171, as one thread.
void lm_impl(const LMProblem &pb, double *q, double *t, const orc_lm_opts &opt, orc_lm_stats &st) {
    double JtJ[36], Jtr[6];
    st.cost = pb.residual(q, t);
    st.initial_cost = st.cost;
    st.grad_norm = -1;
    st.step_norm = -1;
    st.invalid_steps = 0;
    st.lambda = opt.initial_lambda;
    st.iterations = 0;
    bool recompute = true;
    for (int64_t it = 0; it < opt.max_iterations; ++it) {
        bool brk = false;
        if (recompute) {
            pb.accumulate(q, t, JtJ, Jtr);
            st.grad_norm = norm6(Jtr);
            if (st.grad_norm < opt.gradient_tol) brk = true;
        }
        for (int k = 0; k < 6; ++k) JtJ[k * 7] += st.lambda;
        double sol[6];
        cholesky_solve6(JtJ, Jtr, sol);
        for (int k = 0; k < 6; ++k) sol[k] = -1 * sol[k];
        st.step_norm = norm6(sol);
        if (st.step_norm < opt.step_tol) brk = true;
        // step(), jaco.cuh:288-299: R <- R * exp([w]x), t <- t + R * dt
        double qn[4], tn[3], e[4], dt[3];
        quat_exp(sol, e);
        quat_mul(q, e, qn);
        quat_rot(q, sol + 3, dt);
        tn[0] = t[0] + dt[0]; tn[1] = t[1] + dt[1]; tn[2] = t[2] + dt[2];
        if (brk) break;
        double cost_new = pb.residual(qn, tn);
        if (cost_new < st.cost) {
            std::memcpy(q, qn, sizeof(qn));
            std::memcpy(t, tn, sizeof(tn));
            st.lambda = std::max(opt.min_lambda, st.lambda / 10);
            st.cost = cost_new;
            recompute = true;
        } else {
            st.invalid_steps++;
            for (int k = 0; k < 6; ++k) JtJ[k * 7] -= st.lambda;
            st.lambda = std::min(opt.max_lambda, st.lambda * 10);
            recompute = false;
        }
        ++st.iterations;
    }
}

// Adaptive-termination sample count (turbo_ransac.cu:223-231). Beyond the int
// range the reference's double->int assignment is undefined; quirk = 1 gives
// what x86's conversion instruction returns (INT_MIN, which ends the loop),
// quirk = 0 saturates (no inlier or K >= INT_MAX: keep sampling to the cap).
inline int64_t needed_samples(int64_t inliers, int64_t n, double success_prob, double mult, int quirk) {
    double log_prob_missing_model = std::log(1.0 - success_prob);
    double inlier_ratio = (double)inliers / (double)n;
    double prob_outlier = 1.0 - std::pow(inlier_ratio, 3);
    double v = std::ceil(log_prob_missing_model / std::log(prob_outlier) * mult);
    if (quirk) {
        if (!(v >= -2147483648.0 && v < 2147483648.0)) return (int64_t)INT_MIN;
        return (int64_t)(int)v;
    }
    if (inliers <= 0 || !(v == v) || v >= 2147483647.0) return (int64_t)INT_MAX;
    if (v <= -2147483648.0) return (int64_t)INT_MIN;
    return (int64_t)v;
}

template <class F>
void parallel_for(int64_t count, int threads, F &&f) {
    if (threads <= 1 || count <= 1) {
        for (int64_t i = 0; i < count; ++i) f(i);
        return;
    }
    std::atomic<int64_t> next{0};
    std::vector<std::thread> pool;
    const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(16, count / (8 * (int64_t)threads)));
    for (int w = 0; w < threads; ++w)
        pool.emplace_back([&] {
            for (;;) {
                int64_t b = next.fetch_add(chunk);
                if (b >= count) break;
                int64_t e = std::min(count, b + chunk);
                for (int64_t i = b; i < e; ++i) f(i);
            }
        });
    for (auto &th : pool) th.join();
}

struct SampleResult {
    int nsol;
    double P[4][12];
    double score[4];
    int64_t count[4];
};

void run_sample(const double *xn, const double *X, int64_t n, double sq_thr, const int32_t idx[3],
                SampleResult &sr) {
    double xb[9], Xs[9];
    for (int k = 0; k < 3; ++k) {
        orc_bearing(xn[2 * idx[k]], xn[2 * idx[k] + 1], xb + 3 * k);
        Xs[3 * k] = X[3 * idx[k]];
        Xs[3 * k + 1] = X[3 * idx[k] + 1];
        Xs[3 * k + 2] = X[3 * idx[k] + 2];
    }
    sr.nsol = p3p_impl(xb, Xs, &sr.P[0][0]);
    for (int s = 0; s < sr.nsol; ++s) msac_impl(xn, X, n, sr.P[s], sq_thr, sr.score[s], sr.count[s]);
}

}  // namespace

// ================================================================ C API ====
extern "C" {

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
    philox(c, key[0], key[1]);
    for (int i = 0; i < 4; ++i) out[i] = c[i];
}

void orc_sample_triples(uint64_t seed, int64_t first_sample, int64_t count, int64_t n,
                        int32_t *idx_out) {
    for (int64_t s = 0; s < count; ++s)
        triple_from_sample(seed, (uint64_t)(first_sample + s), (uint32_t)n, idx_out + 3 * s);
}

void orc_prosac_table(int64_t n, double TN, int64_t *Tp) {
    auto T = [&](int64_t k) {
        return ((TN * ((double)k / (double)n)) * ((double)(k - 1) / (double)(n - 1))) *
               ((double)(k - 2) / (double)(n - 2));
    };
    Tp[0] = 1;
    for (int64_t k = 3; k < n; ++k) Tp[k - 2] = Tp[k - 3] + (int64_t)std::ceil(T(k + 1) - T(k));
}

void orc_prosac_triple(uint64_t seed, int64_t sample, int64_t n, const int64_t *Tp, int32_t out[3]) {
    const int64_t t = sample + 1;
    const int64_t g = std::upper_bound(Tp, Tp + (n - 3), t) - Tp;  // growths so far
    const int64_t m = 3 + g;
    if (m >= n && Tp[n - 3] < t) {
        triple_from_sample(seed, (uint64_t)sample, (uint32_t)n, out);
        return;
    }
    uint32_t c[4] = {(uint32_t)sample, (uint32_t)((uint64_t)sample >> 32), 0u, 0u};
    philox(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    uint32_t i0 = mulhi_range(c[0], (uint32_t)(m - 1));
    uint32_t i1 = mulhi_range(c[1], (uint32_t)(m - 2));
    if (i1 >= i0) ++i1;
    out[0] = (int32_t)i0; out[1] = (int32_t)i1; out[2] = (int32_t)(m - 1);
}

int orc_p3p(const double *x, const double *X, double *poses_out) { return p3p_impl(x, X, poses_out); }

void orc_bearing(double x, double y, double out[3]) {
    double v0 = x, v1 = y, v2 = 1.0;
    double z = v0 * v0 + v1 * v1 + v2 * v2;
    if (z > 0.0) {
        double nrm = std::sqrt(z);
        v0 /= nrm; v1 /= nrm; v2 /= nrm;
    }
    out[0] = v0; out[1] = v1; out[2] = v2;
}

void orc_msac(const double *xn, const double *X, int64_t n, const double *P, double sq_thr,
              double *score, int64_t *count) {
    msac_impl(xn, X, n, P, sq_thr, *score, *count);
}

void orc_rotmat_to_quat(const double *R, double q[4]) { rotmat_to_quat_impl(R, q); }
void orc_quat_to_rotmat(const double q[4], double *R) { quat_to_rotmat_impl(q, R); }

int64_t orc_get_inliers(const double q[4], const double t[3], const double *xn, const double *X,
                        int64_t n, double sq_thr, uint8_t *inliers) {
    double R[9];
    quat_to_rotmat_impl(q, R);
    int64_t cnt = 0;
    for (int64_t k = 0; k < n; ++k) {
        V3 Xv = {{X[3 * k], X[3 * k + 1], X[3 * k + 2]}};
        V3 RX = mat3_vec(R, Xv);
        const double Z0 = RX[0] + t[0], Z1 = RX[1] + t[1], Z2 = RX[2] + t[2];
        const double h0 = Z0 / Z2 - xn[2 * k], h1 = Z1 / Z2 - xn[2 * k + 1];
        const double r2 = h0 * h0 + h1 * h1;
        const uint8_t in = (r2 < sq_thr && Z2 > 0.0) ? 1 : 0;
        if (inliers) inliers[k] = in;
        cnt += in;
    }
    return cnt;
}

int orc_ransac(const double *xn, const double *X, int64_t n, double sq_thr,
               const orc_ransac_cfg *cfg, orc_ransac_out *out, double *hyp_scores,
               int64_t *hyp_counts, int64_t *hyp_ids, double *hyp_poses, int64_t hyp_cap) {
    if (n < 3 || cfg->samples_per_round < 1) return -1;
    const int64_t B = cfg->samples_per_round;
    const bool forced = cfg->force_samples > 0;
    std::memset(out, 0, sizeof(*out));
    for (int i = 0; i < 12; ++i) out->P[i] = (i % 5 == 0) ? 1.0 : 0.0;
    out->score = DBL_MAX;
    out->best_sample = -1;
    out->best_sol = -1;

    std::vector<SampleResult> res;
    std::vector<int32_t> idx;
    std::vector<int64_t> prosac_tp;
    int64_t done = 0, nhyp = 0, rounds = 0;
    bool stop = false;
    // Round loop, turbo_ransac.cu:151-259: at least one round, stop once the
    // samples drawn exceed the adaptive bound or reach the hard cap.
    while (!stop) {
        int64_t cnt = forced ? cfg->force_samples : B;
        if (!forced && done >= cfg->max_total_samples) break;
        idx.resize(cnt * 3);
        if (cfg->replay) {
            if (done + cnt > cfg->replay_count) return -2;
            std::memcpy(idx.data(), cfg->replay + 3 * done, sizeof(int32_t) * 3 * cnt);
        } else if (cfg->prosac) {
            if (prosac_tp.empty()) {
                prosac_tp.resize(n - 2);
                orc_prosac_table(n, cfg->prosac_TN, prosac_tp.data());
            }
            for (int64_t s = 0; s < cnt; ++s) orc_prosac_triple(cfg->seed, done + s, n, prosac_tp.data(), &idx[3 * s]);
        } else {
            orc_sample_triples(cfg->seed, done, cnt, n, idx.data());
        }
        res.resize(cnt);
        parallel_for(cnt, cfg->threads,
                     [&](int64_t s) { run_sample(xn, X, n, sq_thr, &idx[3 * s], res[s]); });
        // Per sample keep the first solution with the lowest score (ransac.cuh:323);
        // across samples the earliest sample wins ties (merge + argmin +
        // strict host update, ransac.cuh:62,79; turbo_ransac.cu:235).
        for (int64_t s = 0; s < cnt; ++s) {
            const SampleResult &sr = res[s];
            int bi = -1;
            double bs = DBL_MAX;
            for (int k = 0; k < sr.nsol; ++k) {
                if (hyp_scores && nhyp < hyp_cap) {
                    hyp_scores[nhyp] = sr.score[k];
                    if (hyp_counts) hyp_counts[nhyp] = sr.count[k];
                    if (hyp_ids) hyp_ids[nhyp] = (done + s) * 4 + k;
                    if (hyp_poses) std::memcpy(hyp_poses + 12 * nhyp, sr.P[k], sizeof(double) * 12);
                }
                ++nhyp;
                if (sr.score[k] < bs) { bs = sr.score[k]; bi = k; }
            }
            if (bi >= 0 && bs < out->score) {
                out->score = bs;
                out->count = sr.count[bi];
                out->best_sample = done + s;
                out->best_sol = bi;
                out->found = 1;
                std::memcpy(out->P, sr.P[bi], sizeof(out->P));
            }
        }
        done += cnt;
        ++rounds;
        if (forced) break;
        int64_t need = needed_samples(out->found ? out->count : 0, n, cfg->success_prob, cfg->trials_mult,
                                      cfg->quirk);
        if (done > need && done >= cfg->min_samples) stop = true;
    }
    out->samples = done;
    out->rounds = rounds;
    out->hypotheses = nhyp;
    return 0;
}

void orc_lm(const double *x, const double *X, int64_t n, const double cam[4], double q[4],
            double t[3], const orc_lm_opts *opt, orc_lm_stats *stats) {
    LMProblem pb{x, X, n, cam[0], cam[1], cam[2], cam[3], 1.0 / (opt->loss_scale * opt->loss_scale)};
    pb.loss = opt->loss;
    pb.w8 = opt->weights;
    pb.thr = opt->loss_scale;
    pb.sq_thr = opt->loss_scale * opt->loss_scale;
    orc_lm_stats st;
    lm_impl(pb, q, t, *opt, st);
    if (stats) *stats = st;
}

int orc_estimate(const double *uv, const double *X, int64_t n, const double K[4],
                 double max_reproj_error, const orc_ransac_cfg *cfg, int skip_refine, double q[4],
                 double t[3], uint8_t *inliers, orc_estimate_info *info) {
    if (n < 3) return -1;
    const double fx = K[0], fy = K[1], cx = K[2], cy = K[3];
    // Camera_cuda::unproject and focal(), camera.cuh:51-67; threshold scaling entry.cu:48-49.
    std::vector<double> xn(2 * n);
    for (int64_t k = 0; k < n; ++k) {
        xn[2 * k] = (uv[2 * k] - cx) / fx;
        xn[2 * k + 1] = (uv[2 * k + 1] - cy) / fy;
    }
    const double focal = 0.5 * (fx + fy);
    const double thr = max_reproj_error / focal;
    const double sq_thr = thr * thr;

    orc_estimate_info local;
    orc_estimate_info &inf = info ? *info : local;
    std::memset(&inf, 0, sizeof(inf));
    int rc = orc_ransac(xn.data(), X, n, sq_thr, cfg, &inf.ransac, nullptr, nullptr, nullptr, nullptr, 0);
    if (rc) return rc;

    // entry.cu:79-83: pose from the 4x4 (R -> quaternion), inliers with it.
    double R[9], tt[3];
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) R[r * 3 + c] = inf.ransac.P[r * 4 + c];
        tt[r] = inf.ransac.P[r * 4 + 3];
    }
    double qq[4];
    rotmat_to_quat_impl(R, qq);
    std::vector<uint8_t> mask(n);
    inf.num_inliers = orc_get_inliers(qq, tt, xn.data(), X, n, sq_thr, mask.data());
    if (inliers) std::memcpy(inliers, mask.data(), n);

    // entry.cu:87-132: LM on the inliers in pixel/f units with a default
    // BundleOptions whose loss scale is 1/f (a 1 px Cauchy).
    std::memcpy(q, qq, sizeof(qq));
    std::memcpy(t, tt, sizeof(tt));
    if (!skip_refine) {
        const double scale = 1.0 / focal;
        std::vector<double> xi, Xi;
        xi.reserve(2 * inf.num_inliers);
        Xi.reserve(3 * inf.num_inliers);
        for (int64_t k = 0; k < n; ++k) {
            if (!mask[k]) continue;
            xi.push_back(uv[2 * k] * scale);
            xi.push_back(uv[2 * k + 1] * scale);
            Xi.push_back(X[3 * k]);
            Xi.push_back(X[3 * k + 1]);
            Xi.push_back(X[3 * k + 2]);
        }
        const double cam[4] = {fx * scale, fy * scale, cx * scale, cy * scale};
        orc_lm_opts lo{100, 1.0 * scale, 1e-10, 1e-8, 1e-3, 1e-10, 1e10};
        orc_lm(xi.data(), Xi.data(), (int64_t)(xi.size() / 2), cam, q, t, &lo, &inf.lm);
    }
    return 0;
}

int orc_estimate_batch(const double *uv, const double *X, const int64_t *offsets,
                       const double *K, const uint64_t *seeds, int n_frames,
                       double max_reproj_error, int64_t samples_per_round, int threads,
                       double *q_out, double *t_out, int64_t *samples_out) {
    std::atomic<int> err{0};
    parallel_for(n_frames, threads, [&](int64_t f) {
        orc_ransac_cfg cfg{};
        cfg.samples_per_round = samples_per_round;
        cfg.max_total_samples = 100000;
        cfg.success_prob = 0.9999;
        cfg.trials_mult = 3.0;
        cfg.seed = seeds[f];
        cfg.threads = 1;
        orc_estimate_info info;
        const int64_t b = offsets[f], e = offsets[f + 1];
        int rc = orc_estimate(uv + 2 * b, X + 3 * b, e - b, K + 4 * f, max_reproj_error, &cfg, 0,
                              q_out + 4 * f, t_out + 3 * f, nullptr, &info);
        if (rc) err = rc;
        if (samples_out) samples_out[f] = info.ransac.samples;
    });
    return err.load();
}

}  // extern "C"
