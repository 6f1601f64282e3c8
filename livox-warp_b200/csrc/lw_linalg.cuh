// Small dense float64 linear algebra for the on-device Gauss-Newton solve and the per-voxel shape analysis:
// cyclic Jacobi eigendecomposition of symmetric matrices (Golub & Van Loan, Matrix Computations, 4th ed.,
// Alg. 8.5.2 with the 2x2 symmetric Schur step of Alg. 8.5.1), LU with partial pivoting, and the SO(3)
// exponential / logarithm through unit quaternions (the rotation-vector conversions of
// scipy.spatial.transform.Rotation that odom.py uses: odom.py:400, 405, 414, 420, 716).
#pragma once
#include <math.h>

namespace lw {

// Eigen-decomposition of the symmetric N x N matrix A (row major, destroyed): ev[k] with eigenvector column
// k of V (V[i*N+k]). Eigenvalues come in diagonal order, not sorted. Cyclic sweeps until the off-diagonal
// mass is below 1e-30 of the total (at most 24 sweeps).
template <int N>
__device__ __forceinline__ void jacobi_eig(double* A, double* ev, double* V) {
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) V[i * N + j] = (i == j) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 24; ++sweep) {
        double off = 0.0, tot = 0.0;
#pragma unroll
        for (int i = 0; i < N; ++i)
#pragma unroll
            for (int j = 0; j < N; ++j) {
                double a2 = A[i * N + j] * A[i * N + j];
                tot += a2;
                if (i != j) off += a2;
            }
        if (off <= 1e-30 * tot || off == 0.0) break;
        // the rotations unrolled: every index is then a constant and A, V stay in registers
#pragma unroll
        for (int p = 0; p < N - 1; ++p) {
#pragma unroll
            for (int q = p + 1; q < N; ++q) {
                double apq = A[p * N + q];
                if (apq == 0.0) continue;
                double tau = (A[q * N + q] - A[p * N + p]) / (2.0 * apq);
                double t = (tau >= 0.0) ? 1.0 / (tau + sqrt(1.0 + tau * tau)) : -1.0 / (-tau + sqrt(1.0 + tau * tau));
                double c = 1.0 / sqrt(1.0 + t * t);
                double s = t * c;
                // A <- J^T A J with J the rotation in the (p, q) plane
#pragma unroll
                for (int k = 0; k < N; ++k) {
                    double akp = A[k * N + p], akq = A[k * N + q];
                    A[k * N + p] = c * akp - s * akq;
                    A[k * N + q] = s * akp + c * akq;
                }
#pragma unroll
                for (int k = 0; k < N; ++k) {
                    double apk = A[p * N + k], aqk = A[q * N + k];
                    A[p * N + k] = c * apk - s * aqk;
                    A[q * N + k] = s * apk + c * aqk;
                }
#pragma unroll
                for (int k = 0; k < N; ++k) {
                    double vkp = V[k * N + p], vkq = V[k * N + q];
                    V[k * N + p] = c * vkp - s * vkq;
                    V[k * N + q] = s * vkp + c * vkq;
                }
            }
        }
    }
#pragma unroll
    for (int i = 0; i < N; ++i) ev[i] = A[i * N + i];
}

// Solve A x = b (A row major N x N, copied) by LU with partial pivoting; false when a pivot is exactly zero
// (numpy.linalg.solve raises LinAlgError there).
template <int N>
__device__ __forceinline__ bool lu_solve(const double* A_in, const double* b, double* x, int n = N) {
    double A[N * N], y[N];
    for (int i = 0; i < n; ++i) {
        y[i] = b[i];
        for (int j = 0; j < n; ++j) A[i * N + j] = A_in[i * N + j];
    }
    for (int k = 0; k < n; ++k) {
        int piv = k;
        double best = fabs(A[k * N + k]);
        for (int i = k + 1; i < n; ++i) {
            double v = fabs(A[i * N + k]);
            if (v > best) {
                best = v;
                piv = i;
            }
        }
        if (best == 0.0) return false;
        if (piv != k) {
            for (int j = 0; j < n; ++j) {
                double tmp = A[k * N + j];
                A[k * N + j] = A[piv * N + j];
                A[piv * N + j] = tmp;
            }
            double tmp = y[k];
            y[k] = y[piv];
            y[piv] = tmp;
        }
        for (int i = k + 1; i < n; ++i) {
            double f = A[i * N + k] / A[k * N + k];
            for (int j = k; j < n; ++j) A[i * N + j] -= f * A[k * N + j];
            y[i] -= f * y[k];
        }
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = y[i];
        for (int j = i + 1; j < n; ++j) s -= A[i * N + j] * x[j];
        x[i] = s / A[i * N + i];
    }
    return true;
}

// ---- SO(3) / SE(3), row-major 3x3 and 4x4 ------------------------------------------------------------------

// Rotation matrix of a rotation vector: unit quaternion (axis sin(a/2), cos(a/2)) with the series for small
// angles, then the quaternion's matrix.
__device__ __forceinline__ void rotvec_to_mat(const double* rv, double* R) {
    double a2 = rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2];
    double a = sqrt(a2);
    double scale, w;
    if (a <= 1e-3) {
        scale = 0.5 - a2 / 48.0 + a2 * a2 / 3840.0;
        w = cos(0.5 * a);
    } else {
        scale = sin(0.5 * a) / a;
        w = cos(0.5 * a);
    }
    double x = rv[0] * scale, y = rv[1] * scale, z = rv[2] * scale;
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

// Rotation vector of a rotation matrix: quaternion by the largest of (trace, diagonal) (Shepperd's method),
// sign chosen so w >= 0, then angle = 2 atan2(|v|, w).
__device__ __forceinline__ void mat_to_rotvec(const double* R, double* rv) {
    double tr = R[0] + R[4] + R[8];
    double q[4];  // x, y, z, w
    int k = 3;
    double best = tr;
    if (R[0] > best) { best = R[0]; k = 0; }
    if (R[4] > best) { best = R[4]; k = 1; }
    if (R[8] > best) { best = R[8]; k = 2; }
    if (k == 3) {
        q[3] = 1.0 + tr;
        q[0] = R[7] - R[5];
        q[1] = R[2] - R[6];
        q[2] = R[3] - R[1];
    } else {
        int i = k, j = (k + 1) % 3, l = (k + 2) % 3;
        q[i] = 1.0 - tr + 2.0 * R[i * 4];
        q[j] = R[j * 3 + i] + R[i * 3 + j];
        q[l] = R[l * 3 + i] + R[i * 3 + l];
        q[3] = R[l * 3 + j] - R[j * 3 + l];
    }
    double nrm = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    for (int c = 0; c < 4; ++c) q[c] /= nrm;
    if (q[3] < 0.0)
        for (int c = 0; c < 4; ++c) q[c] = -q[c];
    double vn = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
    double ang = 2.0 * atan2(vn, q[3]);
    double scale;
    if (ang <= 1e-3) {
        double a2 = ang * ang;
        scale = 2.0 + a2 / 12.0 + 7.0 * a2 * a2 / 2880.0;
    } else {
        scale = ang / sin(0.5 * ang);
    }
    rv[0] = scale * q[0];
    rv[1] = scale * q[1];
    rv[2] = scale * q[2];
}

__device__ __forceinline__ void mat44_mul(const double* A, const double* B, double* C) {
    double t[16];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            double s = 0.0;
            for (int k = 0; k < 4; ++k) s += A[i * 4 + k] * B[k * 4 + j];
            t[i * 4 + j] = s;
        }
    for (int i = 0; i < 16; ++i) C[i] = t[i];
}

// Inverse of a rigid transform [R t; 0 1]: [R^T, -R^T t].
__device__ __forceinline__ void mat44_inv_rigid(const double* T, double* O) {
    double t[16];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) t[i * 4 + j] = T[j * 4 + i];
    for (int i = 0; i < 3; ++i) t[i * 4 + 3] = -(t[i * 4 + 0] * T[3] + t[i * 4 + 1] * T[7] + t[i * 4 + 2] * T[11]);
    t[12] = t[13] = t[14] = 0.0;
    t[15] = 1.0;
    for (int i = 0; i < 16; ++i) O[i] = t[i];
}

__device__ __forceinline__ void mat44_eye(double* T) {
    for (int i = 0; i < 16; ++i) T[i] = (i % 5 == 0) ? 1.0 : 0.0;
}

__device__ __forceinline__ void mat44_rot(const double* T, double* R) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) R[i * 3 + j] = T[i * 4 + j];
}

// (translation, rotation vector) of a 4x4 motion: odom.py _body_twist (:412-414) in float64.
__device__ __forceinline__ void body_twist(const double* D, double* xi) {
    double R[9];
    mat44_rot(D, R);
    xi[0] = D[3];
    xi[1] = D[7];
    xi[2] = D[11];
    mat_to_rotvec(R, xi + 3);
}

// exp(xi) as a 4x4 with translation xi[:3] (odom.py _twist_matrix :417-422).
__device__ __forceinline__ void twist_matrix(const double* xi, double* D) {
    double R[9];
    rotvec_to_mat(xi + 3, R);
    mat44_eye(D);
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) D[i * 4 + j] = R[i * 3 + j];
        D[i * 4 + 3] = xi[i];
    }
}

// T <- exp_left(delta) T (odom.py _apply_twist :404-409).
__device__ __forceinline__ void apply_twist(double* T, const double* delta) {
    double Rz[9];
    rotvec_to_mat(delta + 3, Rz);
    double o[12];
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) o[i * 4 + j] = Rz[i * 3 + 0] * T[0 * 4 + j] + Rz[i * 3 + 1] * T[1 * 4 + j] + Rz[i * 3 + 2] * T[2 * 4 + j];
        o[i * 4 + 3] = Rz[i * 3 + 0] * T[3] + Rz[i * 3 + 1] * T[7] + Rz[i * 3 + 2] * T[11] + delta[i];
    }
    for (int i = 0; i < 12; ++i) T[i] = o[i];
}

}  // namespace lw
