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

// The same eigen-decomposition for a symmetric 6x6 by one warp (every lane calls it), on shared memory: the 15
// rotations of a sweep run as 5 rounds of 3 disjoint (p, q) pairs (the round-robin ordering of parallel Jacobi,
// Golub & Van Loan Sec. 8.5.5). Within a round lanes 0-2 form the three rotations, then 21 lanes rewrite the
// upper triangle of J^T A J (each rotated pair's own element set to zero) and the lanes rewrite V J. A is
// destroyed; ev[k] is A's k-th diagonal element at the end, V's column k its vector (V may be null when VEC is
// false); rot holds 6 doubles of scratch. With v_given, V already holds an orthogonal basis Q and A is Q^T M Q:
// the rotations accumulate onto Q, so V ends as M's eigenvectors. One thread running the unrolled cyclic form spends most of its time
// fetching instructions; this form keeps the code small and the rotations of a round side by side, and forms
// each rotation with jac_rotation (no divide or correctly rounded square root). Same stopping rule as jacobi_eig.
// 1/sqrt(x) and 1/x in float64 for x in [1, 8]: the float32 hardware approximation (relative error below
// 2^-22) refined by two Newton-Raphson steps, y <- y (3 - x y^2) / 2 and y <- y (2 - x y), each of which squares
// the relative error (2^-22 -> 2^-44 -> below the float64 rounding). A few dependent multiply-adds instead of the
// long dependent chains of a correctly rounded divide or square root; the result is within a few ulp.
__device__ __forceinline__ double rsqrt_nr(double x) {
    float yf;
    asm("rsqrt.approx.f32 %0, %1;" : "=f"(yf) : "f"((float)x));
    double y = (double)yf;
    y = y * (1.5 - 0.5 * x * y * y);
    y = y * (1.5 - 0.5 * x * y * y);
    return y;
}

__device__ __forceinline__ double rcp_nr(double x) {
    float yf;
    asm("rcp.approx.f32 %0, %1;" : "=f"(yf) : "f"((float)x));
    double y = (double)yf;
    y = y + y * (1.0 - x * y);
    y = y + y * (1.0 - x * y);
    return y;
}

// The Jacobi rotation (c, s) that annihilates apq (Golub & Van Loan Alg. 8.5.1): t = sign(tau) / (|tau| +
// sqrt(1 + tau^2)) with tau = (aqq - app) / (2 apq), c = 1 / sqrt(1 + t^2), s = t c. Written as
// t = sign(tau) |2 apq| / (|d| + sqrt(d^2 + 4 apq^2)) with d = aqq - app, both scaled by the same power of two so
// the larger has magnitude in [1, 2): every square root and reciprocal then sees an argument in [1, 8] (no
// overflow for any tau). Same sign convention as jacobi_eig (tau = 0 counts as positive).
__device__ __forceinline__ void jac_rotation(double app, double aqq, double apq, double& c, double& sn) {
    c = 1.0;
    sn = 0.0;
    const double d = aqq - app, p2 = 2.0 * apq;
    const double m = fmax(fabs(d), fabs(p2));
    if (!(m >= 1e-290 && m <= 1e290)) return;  // a zero or absurd element: no rotation
    const int e = (int)((__double_as_longlong(m) >> 52) & 0x7ff) - 1023;
    const double sc = __longlong_as_double((long long)(1023 - e) << 52);  // 2^-e, exact
    const double dd = d * sc, pp = p2 * sc;
    const double h = dd * dd + pp * pp;
    const double r = h * rsqrt_nr(h);
    const bool pos = d == 0.0 || ((d > 0.0) == (p2 > 0.0));
    const double t = (pos ? 1.0 : -1.0) * fabs(pp) * rcp_nr(fabs(dd) + r);
    c = rsqrt_nr(1.0 + t * t);
    sn = t * c;
}

template <bool VEC>
__device__ void jacobi6_warp(double* A, double* V, double* ev, double* rot, bool v_given) {
    // round r's three pairs, one byte each (p in the high nibble): (0,5)(1,4)(2,3) / (0,4)(3,5)(1,2) /
    // (0,3)(2,4)(1,5) / (0,2)(1,3)(4,5) / (0,1)(2,5)(3,4) -- every pair once per sweep
    constexpr unsigned PAIRS[5] = {0x231405u, 0x123504u, 0x152403u, 0x451302u, 0x342501u};
    // the same rounds seen from each index x (6 bits at 6x): slot | (x is q) << 2 | partner << 3
    constexpr unsigned long long IDX[5] = {0x00010d59a868ULL, 0x000744a4e4a0ULL, 0x000395121a98ULL,
                                           0x0009aa344650ULL, 0x00055e8a9108ULL};
    const int lane = threadIdx.x & 31;
    // this lane's upper-triangle element (lanes 0-20; lanes 21-31 compute a copy of element 20 and store nothing)
    int ui = 0, uj;
    {
        int e = lane < 21 ? lane : 20;
        while (e >= 6 - ui) {
            e -= 6 - ui;
            ++ui;
        }
        uj = ui + e;
    }
    // this lane's elements of V: lane, and lane + 32 for lanes 0-3 (the others compute a copy of element 35)
    const int k0 = lane / 6, j0 = lane % 6;
    const int e1 = lane < 4 ? lane + 32 : 35;
    const int k1 = e1 / 6, j1 = e1 % 6;
    if (VEC && !v_given) {
        V[lane] = (lane % 7 == 0) ? 1.0 : 0.0;
        if (lane < 4) V[lane + 32] = (lane == 3) ? 1.0 : 0.0;
    }
    __syncwarp();
    for (int sweep = 0; sweep < 24; ++sweep) {
        double a0 = A[lane], a1 = lane < 4 ? A[lane + 32] : 0.0;
        double tot = a0 * a0 + a1 * a1;
        double off = (lane % 7 != 0 ? a0 * a0 : 0.0) + (lane < 3 ? a1 * a1 : 0.0);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            tot += __shfl_xor_sync(0xffffffffu, tot, o);
            off += __shfl_xor_sync(0xffffffffu, off, o);
        }
        if (off <= 1e-30 * tot || off == 0.0) break;
#pragma unroll
        for (int r = 0; r < 5; ++r) {
            if (lane < 3) {
                const unsigned pq = (PAIRS[r] >> (8 * lane)) & 0xffu;
                const int p = (int)(pq >> 4), q = (int)(pq & 15u);
                double c, sn;
                jac_rotation(A[p * 6 + p], A[q * 6 + q], A[p * 6 + q], c, sn);
                rot[2 * lane] = c;
                rot[2 * lane + 1] = sn;
            }
            __syncwarp();
            // index x sits in one pair (p, q) of this round: new_x = ca * old_p + cb * old_q
            auto lookup = [&](int x, int& p, int& q, double& ca, double& cb, int& slot) {
                const int en = (int)((IDX[r] >> (6 * x)) & 63ULL);
                slot = en & 3;
                const int partner = en >> 3;
                const bool is_q = (en & 4) != 0;
                const double c = rot[2 * slot], sn = rot[2 * slot + 1];
                p = is_q ? partner : x;
                q = is_q ? x : partner;
                ca = is_q ? sn : c;
                cb = is_q ? c : -sn;
            };
            int pi, qi, si, pj, qj, sj;
            double ai, bi, aj, bj;
            lookup(ui, pi, qi, ai, bi, si);
            lookup(uj, pj, qj, aj, bj, sj);
            double na = ai * (aj * A[pi * 6 + pj] + bj * A[pi * 6 + qj]) + bi * (aj * A[qi * 6 + pj] + bj * A[qi * 6 + qj]);
            if (ui != uj && si == sj) na = 0.0;  // the rotated pair's own element
            double nv0 = 0.0, nv1 = 0.0;
            if (VEC) {
                int p0, q0, s0, p1, q1, s1;
                double ca0, cb0, ca1, cb1;
                lookup(j0, p0, q0, ca0, cb0, s0);
                lookup(j1, p1, q1, ca1, cb1, s1);
                nv0 = ca0 * V[k0 * 6 + p0] + cb0 * V[k0 * 6 + q0];
                nv1 = ca1 * V[k1 * 6 + p1] + cb1 * V[k1 * 6 + q1];
            }
            __syncwarp();
            if (lane < 21) {
                A[ui * 6 + uj] = na;
                A[uj * 6 + ui] = na;
            }
            if (VEC) {
                V[lane] = nv0;
                if (lane < 4) V[lane + 32] = nv1;
            }
            __syncwarp();
        }
    }
    if (lane < 6) ev[lane] = A[lane * 7];
    __syncwarp();
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
    double scale, w;
    if (a2 <= 1e-2) {
        // angles up to 0.1 rad (every Gauss-Newton step): the Maclaurin series of sin(a/2)/a and cos(a/2) in a^2,
        // truncated where the next term is below 1e-20 -- no square root, sine or cosine on the step's chain
        scale = fma(a2, fma(a2, fma(a2, fma(a2, 1.0 / 185794560.0, -1.0 / 645120.0), 1.0 / 3840.0), -1.0 / 48.0), 0.5);
        w = fma(a2, fma(a2, fma(a2, fma(a2, fma(a2, -1.0 / 3715891200.0, 1.0 / 10321920.0), -1.0 / 46080.0),
                                1.0 / 384.0), -1.0 / 8.0), 1.0);
    } else {
        const double a = sqrt(a2);
        scale = sin(0.5 * a) / a;
        w = cos(0.5 * a);
    }
    double x = rv[0] * scale, y = rv[1] * scale, z = rv[2] * scale;
    R[0] = fma(-2.0, fma(y, y, z * z), 1.0);
    R[1] = 2.0 * fma(x, y, -z * w);
    R[2] = 2.0 * fma(x, z, y * w);
    R[3] = 2.0 * fma(x, y, z * w);
    R[4] = fma(-2.0, fma(x, x, z * z), 1.0);
    R[5] = 2.0 * fma(y, z, -x * w);
    R[6] = 2.0 * fma(x, z, -y * w);
    R[7] = 2.0 * fma(y, z, x * w);
    R[8] = fma(-2.0, fma(x, x, y * y), 1.0);
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
        for (int j = 0; j < 3; ++j)
            o[i * 4 + j] = fma(Rz[i * 3 + 0], T[0 * 4 + j], fma(Rz[i * 3 + 1], T[1 * 4 + j], Rz[i * 3 + 2] * T[2 * 4 + j]));
        o[i * 4 + 3] = fma(Rz[i * 3 + 0], T[3], fma(Rz[i * 3 + 1], T[7], fma(Rz[i * 3 + 2], T[11], delta[i])));
    }
    for (int i = 0; i < 12; ++i) T[i] = o[i];
}

}  // namespace lw
