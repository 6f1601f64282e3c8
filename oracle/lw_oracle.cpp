// lw_oracle.cpp -- CPU restatement of the livox-warp per-frame hot path. TEST INFRASTRUCTURE ONLY: it is the
// checker the GPU path is compared against (tests/, the smoke check and the CPU baseline of bench.py); no
// product code links or calls it.
//
// It follows the reference's Warp kernels (python/livox_warp in nhaumann/livox-warp) as a serial program:
//   keys / hash / probing      gpu.py:231-265          deskew              gpu.py:268-283, odom.py:163-178
//   thinning                   odom.py:126-160         registration insert odom.py:186-230
//   ICP accumulation           odom.py:233-375         integration insert  gpu.py:373-412
//   carving + local_plane      gpu.py:415-593          map classification  gpu.py:286-299, 596-634, 699-747
//   ground grid                perception.py:29-111    clusters            perception.py:114-271
//   prior grid + nearest_point mapgrid.py:35-194       batched ICP + eval  localize.py:126-205, 517-565
//   prior-map voxel means      prior_map.py:57-123     PCA normals         prior_map.py:126-166
// The reference's nondeterministic choices are fixed the way the GPU build fixes them: the lowest point index
// claims a thinning voxel, per-voxel sums are exact int64 fixed point (the units of include/livox_b200.h),
// and 4096-point caps keep the first points in index order. Float expressions are written in the evaluation
// order the GPU kernels use and compiled with -ffp-contract=off, so integer outputs match bit for bit.
// Parity of this restatement against the reference itself is unpinned: the reference needs NVIDIA Warp,
// which is not installed, and ships no golden vectors for these kernels.
#include <math.h>
#include <cmath>
#include <stdint.h>
#include <string.h>
#include <algorithm>
#include <array>
#include <functional>
#include <unordered_map>
#include <vector>

namespace {

constexpr int64_t BIAS = 1LL << 20;
constexpr int64_t KMASK = (1LL << 21) - 1;
constexpr uint64_t MULT = 0x9E3779B97F4A7C15ULL;
constexpr int PROBES = 64;
constexpr double FIX_R = 4294967296.0, FIX_RR = 1099511627776.0, FIX_W = 1048576.0;
constexpr int REG_CAP = 4096, MAP_CAP = 4096, REC = 20, POSE_SLOTS = 65536;

inline int64_t key_ijk(int ix, int iy, int iz) {
    int64_t x = ((int64_t)ix + BIAS) & KMASK, y = ((int64_t)iy + BIAS) & KMASK, z = ((int64_t)iz + BIAS) & KMASK;
    return x | (y << 21) | (z << 42);
}
inline int slot_hash(int64_t k) {
    int64_t h = (int64_t)((uint64_t)k * MULT);
    h = h ^ (h >> 29);
    return (int)(h & 0x7FFFFFFFLL);
}
inline int ifloor(float v) { return (int)floorf(v); }
inline float len3(float x, float y, float z) { return sqrtf(x * x + y * y + z * z); }
inline int refl_of(uint32_t a) { return (int)(a & 255u); }
inline int tag_of(uint32_t a) { return (int)((a >> 8) & 255u); }
inline int ret_of(uint32_t a) { return (int)((a >> 16) & 255u); }

int find_slot(int64_t key, const int64_t* keys, int mask) {
    int h = slot_hash(key) & mask;
    for (int p = 0; p < PROBES; ++p) {
        int s = (h + p) & mask;
        if (keys[s] == key) return s;
        if (keys[s] == -1) return -1;
    }
    return -1;
}
// serial claim: returns the slot and whether it was empty, -1 when the window is full
int claim(int64_t key, int64_t* keys, int mask, bool* claimed) {
    int h = slot_hash(key) & mask;
    *claimed = false;
    for (int p = 0; p < PROBES; ++p) {
        int s = (h + p) & mask;
        if (keys[s] == key) return s;
        if (keys[s] == -1) {
            keys[s] = key;
            *claimed = true;
            return s;
        }
    }
    return -1;
}

// Cyclic Jacobi for a symmetric N x N matrix (Golub & Van Loan Alg. 8.5.2 / 8.5.1), the same sweep order and
// stopping rule as the device solver so the two agree bit for bit.
template <int N>
void jacobi(double* A, double* ev, double* V) {
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) V[i * N + j] = (i == j) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 24; ++sweep) {
        double off = 0.0, tot = 0.0;
        for (int i = 0; i < N; ++i)
            for (int j = 0; j < N; ++j) {
                double a2 = A[i * N + j] * A[i * N + j];
                tot += a2;
                if (i != j) off += a2;
            }
        if (off <= 1e-30 * tot || off == 0.0) break;
        for (int p = 0; p < N - 1; ++p)
            for (int q = p + 1; q < N; ++q) {
                double apq = A[p * N + q];
                if (apq == 0.0) continue;
                double tau = (A[q * N + q] - A[p * N + p]) / (2.0 * apq);
                double t = (tau >= 0.0) ? 1.0 / (tau + sqrt(1.0 + tau * tau)) : -1.0 / (-tau + sqrt(1.0 + tau * tau));
                double c = 1.0 / sqrt(1.0 + t * t), s = t * c;
                for (int k = 0; k < N; ++k) {
                    double akp = A[k * N + p], akq = A[k * N + q];
                    A[k * N + p] = c * akp - s * akq;
                    A[k * N + q] = s * akp + c * akq;
                }
                for (int k = 0; k < N; ++k) {
                    double apk = A[p * N + k], aqk = A[q * N + k];
                    A[p * N + k] = c * apk - s * aqk;
                    A[q * N + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < N; ++k) {
                    double vkp = V[k * N + p], vkq = V[k * N + q];
                    V[k * N + p] = c * vkp - s * vkq;
                    V[k * N + q] = s * vkp + c * vkq;
                }
            }
    }
    for (int i = 0; i < N; ++i) ev[i] = A[i * N + i];
}

inline void xform(const float* T, float x, float y, float z, float& ox, float& oy, float& oz) {
    ox = T[0] * x + T[1] * y + T[2] * z + T[3];
    oy = T[4] * x + T[5] * y + T[6] * z + T[7];
    oz = T[8] * x + T[9] * y + T[10] * z + T[11];
}

}  // namespace

extern "C" {

// ---- primitives -----------------------------------------------------------------------------------------
int64_t or_key_ijk(int ix, int iy, int iz) { return key_ijk(ix, iy, iz); }
int or_slot_hash(int64_t k) { return slot_hash(k); }

void or_voxel_keys(const float* xyz, int64_t n, float inv, int64_t* out) {
    for (int64_t i = 0; i < n; ++i)
        out[i] = key_ijk(ifloor(xyz[3 * i] * inv), ifloor(xyz[3 * i + 1] * inv), ifloor(xyz[3 * i + 2] * inv));
}

// ---- deskew (odom.py:163-178, gpu.py:268-283); raw/out are [m*4] (x, y, z, t) -----------------------------
// deskew (gpu.py:268-283) by a fraction s of the frame's motion tw = (rho, theta): rotation in float64, rounded once
static void deskew_s(float x, float y, float z, float s, const float* tw, float* out) {
    float rx = tw[3] * s, ry = tw[4] * s, rz = tw[5] * s;
    float a = len3(rx, ry, rz);
    float ox = x, oy = y, oz = z;
    if (!(a < 1.0e-9f)) {
        double ad = a;
        double ux = rx / ad, uy = ry / ad, uz = rz / ad;
        double sh = sin(0.5 * ad), w = cos(0.5 * ad);
        double vx = ux * sh, vy = uy * sh, vz = uz * sh;
        double px = x, py = y, pz = z;
        double tx = 2.0 * (vy * pz - vz * py), ty = 2.0 * (vz * px - vx * pz), tz = 2.0 * (vx * py - vy * px);
        ox = (float)(px + w * tx + (vy * tz - vz * ty));
        oy = (float)(py + w * ty + (vz * tx - vx * tz));
        oz = (float)(pz + w * tz + (vx * ty - vy * tx));
    }
    out[0] = ox + tw[0] * s;
    out[1] = oy + tw[1] * s;
    out[2] = oz + tw[2] * s;
}

void or_deskew(const float* raw, int64_t m, float t_mid, float inv_dt, const float* tw, float* out) {
    for (int64_t i = 0; i < m; ++i) {
        const float* p = raw + 4 * i;
        float s = fminf(fmaxf((p[3] - t_mid) * inv_dt, -1.0f), 1.0f);
        deskew_s(p[0], p[1], p[2], s, tw, out + 4 * i);
        out[4 * i + 3] = p[3];
    }
}

// ---- thinning (odom.py:126-160): the first point (in index order) of each half-voxel; out [*4] x,y,z,range --
int64_t or_thin(const float* xyz4, const uint32_t* attr, int64_t m, float inv_v, float min_range, float max_range,
                int ret_mask, float* out4) {
    std::unordered_map<int64_t, char> seen;
    seen.reserve((size_t)m * 2);
    int64_t k = 0;
    for (int64_t i = 0; i < m; ++i) {
        const float* p = xyz4 + 4 * i;
        float r = len3(p[0], p[1], p[2]);
        if (r < min_range || r > max_range) continue;
        if (tag_of(attr[i]) != 0 || ((1 << ret_of(attr[i])) & ret_mask) == 0) continue;
        int64_t key = key_ijk(ifloor(p[0] * inv_v), ifloor(p[1] * inv_v), ifloor(p[2] * inv_v));
        if (!seen.emplace(key, 1).second) continue;
        out4[4 * k + 0] = p[0];
        out4[4 * k + 1] = p[1];
        out4[4 * k + 2] = p[2];
        out4[4 * k + 3] = r;
        ++k;
    }
    return k;
}

// ---- registration map (odom.py:186-230): serial insert in point order ----------------------------------
// T is a float row-major 3x4. Tables: keys [cap], cnt [cap], sum [cap*3], outer [cap*6], stats [2].
void or_reg_insert(const float* xyz4, const uint32_t* attr, int64_t n, const float* T, float inv_v, float voxel,
                   float max_range, int ret_mask, int64_t cap, int64_t* keys, int32_t* cnt, int64_t* sum,
                   int64_t* outer, int32_t* stats) {
    const int mask = (int)(cap - 1);
    for (int64_t i = 0; i < n; ++i) {
        const float* p = xyz4 + 4 * i;
        if (len3(p[0], p[1], p[2]) > max_range || tag_of(attr[i]) != 0 || ((1 << ret_of(attr[i])) & ret_mask) == 0)
            continue;
        float wx, wy, wz;
        xform(T, p[0], p[1], p[2], wx, wy, wz);
        int ix = ifloor(wx * inv_v), iy = ifloor(wy * inv_v), iz = ifloor(wz * inv_v);
        float rx = wx - ((float)ix + 0.5f) * voxel, ry = wy - ((float)iy + 0.5f) * voxel, rz = wz - ((float)iz + 0.5f) * voxel;
        bool claimed;
        int s = claim(key_ijk(ix, iy, iz), keys, mask, &claimed);
        if (claimed) stats[0] += 1;
        if (s < 0) {
            stats[1] += 1;
            continue;
        }
        if (cnt[s] < REG_CAP) {
            const float FR = (float)FIX_R, FRR = (float)FIX_RR;
            sum[3 * s + 0] += llrintf(rx * FR);
            sum[3 * s + 1] += llrintf(ry * FR);
            sum[3 * s + 2] += llrintf(rz * FR);
            outer[6 * s + 0] += llrintf(rx * rx * FRR);
            outer[6 * s + 1] += llrintf(rx * ry * FRR);
            outer[6 * s + 2] += llrintf(rx * rz * FRR);
            outer[6 * s + 3] += llrintf(ry * ry * FRR);
            outer[6 * s + 4] += llrintf(ry * rz * FRR);
            outer[6 * s + 5] += llrintf(rz * rz * FRR);
            cnt[s] += 1;
        }
    }
}

// The per-voxel record the ICP reads: mean, precision M, surface-normal precision Mg, rms direction
// (odom.py:325-368, evaluated in float64 from the exact sums). rec [cap*20].
void or_reg_records(int64_t cap, const int64_t* keys, const int32_t* cnt, const int64_t* sum, const int64_t* outer,
                    float voxel, float tight2f, float noise2f, float alphaf, float* rec) {
    for (int64_t s = 0; s < cap; ++s) {
        float* out = rec + s * REC;
        int c = cnt[s];
        if (keys[s] == -1 || c <= 0) {
            for (int k = 0; k < REC; ++k) out[k] = 0.0f;
            continue;
        }
        int64_t key = keys[s];
        int ix = (int)(key & KMASK) - (int)BIAS, iy = (int)((key >> 21) & KMASK) - (int)BIAS,
            iz = (int)((key >> 42) & KMASK) - (int)BIAS;
        double cf = c, mr[3], C[9];
        for (int k = 0; k < 3; ++k) mr[k] = (double)sum[3 * s + k] / (cf * FIX_R);
        const int up[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) C[i * 3 + j] = (double)outer[6 * s + up[i * 3 + j]] / (cf * FIX_RR) - mr[i] * mr[j];
        double vox = voxel;
        out[0] = (float)(((double)ix + 0.5) * vox + mr[0]);
        out[1] = (float)(((double)iy + 0.5) * vox + mr[1]);
        out[2] = (float)(((double)iz + 0.5) * vox + mr[2]);
        out[3] = (float)c;
        double ev[3], Q[9];
        jacobi<3>(C, ev, Q);
        double tight2 = tight2f, noise2 = noise2f, alpha = alphaf;
        int nt = 0;
        for (int k = 0; k < 3; ++k) nt += ev[k] < tight2 ? 1 : 0;
        double M[6] = {0, 0, 0, 0, 0, 0}, Mg[6] = {0, 0, 0, 0, 0, 0}, q[3] = {0, 0, 0};
        float surf = 0.0f;
        if (c >= 5 && nt <= 1) {
            int kmin = 0;
            if (ev[1] < ev[kmin]) kmin = 1;
            if (ev[2] < ev[kmin]) kmin = 2;
            for (int k = 0; k < 3; ++k) {
                double qa[3] = {Q[k], Q[3 + k], Q[6 + k]};
                double e = fmax(ev[k], 0.0) + noise2, wa = 1.0 / e;
                bool tight = !(ev[k] >= tight2);
                if (!tight) wa = alpha / e;
                double o6[6] = {qa[0] * qa[0], qa[0] * qa[1], qa[0] * qa[2], qa[1] * qa[1], qa[1] * qa[2], qa[2] * qa[2]};
                for (int j = 0; j < 6; ++j) {
                    M[j] += wa * o6[j];
                    if (tight) Mg[j] += wa * o6[j];
                }
                if (k == kmin) {
                    q[0] = qa[0];
                    q[1] = qa[1];
                    q[2] = qa[2];
                }
            }
            surf = 1.0f;
        } else {
            double wa = alpha / (0.25 * vox * vox + noise2);
            M[0] = M[3] = M[5] = wa;
        }
        for (int j = 0; j < 6; ++j) {
            out[4 + j] = (float)M[j];
            out[10 + j] = (float)Mg[j];
        }
        out[16] = (float)q[0];
        out[17] = (float)q[1];
        out[18] = (float)q[2];
        out[19] = surf;
    }
}

// ---- one Gauss-Newton accumulation (odom.py:233-375, k_reduce :378-384) in float64 --------------------
// T64 row-major 4x4 (float64). The correspondence search follows the reference: closest voxel mean among the
// (2 reach + 1)^3 voxels, first strictly smaller distance in (dx, dy, dz) order, within max_d2. out[64].
// Points are split over `threads` OpenMP threads in contiguous ranges; partial sums are added in thread order.
void or_icp_accumulate(const float* ds4, int64_t n, const double* T64, int64_t cap, const int64_t* keys,
                       const float* rec, double inv_v, int reach, double max_d2, double kappa, int threads,
                       double* out) {
    const int mask = (int)(cap - 1);
    if (threads < 1) threads = 1;
    std::vector<double> part((size_t)threads * 64, 0.0);
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int th = 0; th < threads; ++th) {
        double* a = part.data() + (size_t)th * 64;
        int64_t lo = n * th / threads, hi = n * (th + 1) / threads;
        for (int64_t i = lo; i < hi; ++i) {
            const float* p = ds4 + 4 * i;
            double px = p[0], py = p[1], pz = p[2];
            double w[3];
            for (int r = 0; r < 3; ++r) w[r] = T64[r * 4 + 0] * px + T64[r * 4 + 1] * py + T64[r * 4 + 2] * pz + T64[r * 4 + 3];
            int bx = (int)floor(w[0] * inv_v), by = (int)floor(w[1] * inv_v), bz = (int)floor(w[2] * inv_v);
            double best_d2 = max_d2;
            int best_s = -1;
            for (int dx = -reach; dx <= reach; ++dx)
                for (int dy = -reach; dy <= reach; ++dy)
                    for (int dz = -reach; dz <= reach; ++dz) {
                        int s = find_slot(key_ijk(bx + dx, by + dy, bz + dz), keys, mask);
                        if (s < 0) continue;
                        const float* rr = rec + (int64_t)s * REC;
                        if (!(rr[3] > 0.0f)) continue;
                        double ex = w[0] - rr[0], ey = w[1] - rr[1], ez = w[2] - rr[2];
                        double d2 = ex * ex + ey * ey + ez * ez;
                        if (d2 < best_d2) {
                            best_d2 = d2;
                            best_s = s;
                        }
                    }
            if (best_s < 0) continue;
            const float* rr = rec + (int64_t)best_s * REC;
            double r[3] = {w[0] - rr[0], w[1] - rr[1], w[2] - rr[2]};
            const int up[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
            double M[9], G[9];
            for (int k = 0; k < 9; ++k) {
                M[k] = rr[4 + up[k]];
                G[k] = rr[10 + up[k]];
            }
            double Mr[3];
            for (int k = 0; k < 3; ++k) Mr[k] = M[k * 3] * r[0] + M[k * 3 + 1] * r[1] + M[k * 3 + 2] * r[2];
            double d2 = r[0] * Mr[0] + r[1] * Mr[1] + r[2] * Mr[2];
            double wgt = 1.0 / (1.0 + d2 / (kappa * kappa));
            wgt = wgt * wgt;
            double rn = rr[19] > 0.5f ? r[0] * rr[16] + r[1] * rr[17] + r[2] * rr[18] : sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
            double J[3][6] = {{1, 0, 0, 0, w[2], -w[1]}, {0, 1, 0, -w[2], 0, w[0]}, {0, 0, 1, w[1], -w[0], 0}};
            int idx = 0;
            for (int pp = 0; pp < 6; ++pp)
                for (int qq = pp; qq < 6; ++qq) {
                    double v = 0.0, vg = 0.0;
                    for (int aa = 0; aa < 3; ++aa)
                        for (int bb = 0; bb < 3; ++bb) {
                            v += M[aa * 3 + bb] * J[aa][pp] * J[bb][qq];
                            vg += G[aa * 3 + bb] * J[aa][pp] * J[bb][qq];
                        }
                    a[0 + idx] += wgt * v;
                    a[32 + idx] += wgt * vg;
                    ++idx;
                }
            for (int pp = 0; pp < 6; ++pp) a[21 + pp] += wgt * (Mr[0] * J[0][pp] + Mr[1] * J[1][pp] + Mr[2] * J[2][pp]);
            a[27] += 1.0;
            a[28] += wgt * d2;
            a[29] += wgt * rn * rn;
            a[30] += wgt;
            a[31] += p[3];
        }
    }
    for (int k = 0; k < 64; ++k) out[k] = 0.0;
    for (int th = 0; th < threads; ++th)
        for (int k = 0; k < 64; ++k) out[k] += part[(size_t)th * 64 + k];
}

// ---- integration map (gpu.py:155-167 keep_raw, :373-412) -----------------------------------------------
struct View {
    float now, persist, min_range, max_range;
    int32_t min_refl, noise_mask, ret_mask, crop_on;
    float crop_lo[3], crop_hi[3];
    float inv_frame_dt;
    int32_t epoch;
    float inv_voxel;
    int32_t map_mask, dyn_on;
    float dyn_settle;
    int32_t carve_on;
    float carve_ratio;
    int32_t carve_min;
    float carve_stale;
};

static bool keep_raw(float x, float y, float z, uint32_t a, const View& v) {
    float r = len3(x, y, z);
    if (r < v.min_range || r > v.max_range) return false;
    if (refl_of(a) < v.min_refl) return false;
    if (((v.noise_mask >> (tag_of(a) & 3)) & 1) == 0) return false;
    if (((v.ret_mask >> (ret_of(a) & 3)) & 1) == 0) return false;
    return true;
}

// xyz [n*stride]; poses [65536*16] float; map arrays as lw_map.
void or_map_insert(const float* xyz, int stride, const uint32_t* attr, const float* t, const int32_t* frame, int64_t n,
                   const float* poses, const View* v, float inv_voxel, int64_t cap, int64_t* keys, int32_t* cnt,
                   int64_t* acc, float* last, float* first, int32_t* stats) {
    const int mask = (int)(cap - 1);
    for (int64_t i = 0; i < n; ++i) {
        float x = xyz[i * stride], y = xyz[i * stride + 1], z = xyz[i * stride + 2];
        if (!keep_raw(x, y, z, attr[i], *v)) continue;
        const float* T = poses + (int64_t)(frame[i] & (POSE_SLOTS - 1)) * 16;
        float wx, wy, wz;
        xform(T, x, y, z, wx, wy, wz);
        bool claimed;
        int s = claim(key_ijk(ifloor(wx * inv_voxel), ifloor(wy * inv_voxel), ifloor(wz * inv_voxel)), keys, mask, &claimed);
        if (claimed) stats[0] += 1;
        if (s < 0) {
            stats[1] += 1;
            continue;
        }
        int old = cnt[s]++;
        if (old < MAP_CAP) {
            const float FW = (float)FIX_W;
            acc[4 * s + 0] += llrintf(wx * FW);
            acc[4 * s + 1] += llrintf(wy * FW);
            acc[4 * s + 2] += llrintf(wz * FW);
            acc[4 * s + 3] += refl_of(attr[i]);
        }
        last[s] = std::max(last[s], t[i]);
        first[s] = std::min(first[s], t[i]);
    }
}

// ---- carving (gpu.py:415-593) -------------------------------------------------------------------------
struct MapView {
    const int64_t* keys;
    const int32_t* cnt;
    const int64_t* acc;
    int mask;
};

static void centroid(const MapView& m, int s, float& x, float& y, float& z) {
    int c = m.cnt[s];
    double n = (double)(c < MAP_CAP ? c : MAP_CAP) * FIX_W;
    x = (float)((double)m.acc[4 * (int64_t)s + 0] / n);
    y = (float)((double)m.acc[4 * (int64_t)s + 1] / n);
    z = (float)((double)m.acc[4 * (int64_t)s + 2] / n);
}

static void local_plane(int ix, int iy, int iz, float ox, float oy, float oz, const MapView& m, float out[4]) {
    double cs[3] = {0, 0, 0}, cc[6] = {0, 0, 0, 0, 0, 0};
    int cn = 0;
    for (int gx = -1; gx <= 1; ++gx)
        for (int gy = -1; gy <= 1; ++gy)
            for (int gz = -1; gz <= 1; ++gz) {
                int sn = find_slot(key_ijk(ix + gx, iy + gy, iz + gz), m.keys, m.mask);
                if (sn < 0 || m.cnt[sn] <= 0) continue;
                float cx, cy, cz;
                centroid(m, sn, cx, cy, cz);
                double qx = (double)(cx - ox), qy = (double)(cy - oy), qz = (double)(cz - oz);
                cs[0] += qx;
                cs[1] += qy;
                cs[2] += qz;
                cc[0] += qx * qx;
                cc[1] += qx * qy;
                cc[2] += qx * qz;
                cc[3] += qy * qy;
                cc[4] += qy * qz;
                cc[5] += qz * qz;
                ++cn;
            }
    if (cn < 4) {
        out[0] = 0.0f;
        out[1] = 0.0f;
        out[2] = 1.0f;
        out[3] = 0.0f;
        return;
    }
    double inv = 1.0 / (double)cn;
    double mu[3] = {cs[0] * inv, cs[1] * inv, cs[2] * inv}, C[9];
    const int up[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C[i * 3 + j] = cc[up[i * 3 + j]] * inv - mu[i] * mu[j];
    double ev[3], Q[9];
    jacobi<3>(C, ev, Q);
    int k = 0;
    if (ev[1] < ev[k]) k = 1;
    if (ev[2] < ev[k]) k = 2;
    int j = (k + 1) % 3, j2 = (k + 2) % 3;
    double mid = fmin(ev[j], ev[j2]);
    out[0] = (float)Q[k];
    out[1] = (float)Q[3 + k];
    out[2] = (float)Q[6 + k];
    out[3] = ev[k] < 0.25 * mid ? 2.0f : 1.0f;
}

void or_carve(const float* xyz, int stride, const uint32_t* attr, const int32_t* frame, int64_t n, const float* poses,
              int every, float inv_voxel, float max_range, int max_steps, int64_t cap, const int64_t* keys,
              const int32_t* cnt, const int64_t* acc, int32_t* miss, int threads) {
    MapView m{keys, cnt, acc, (int)(cap - 1)};
    if (every < 1) every = 1;
    const int64_t nrays = (n + every - 1) / every;
    if (threads < 1) threads = 1;
#pragma omp parallel for num_threads(threads) schedule(dynamic, 256)
    for (int64_t ray = 0; ray < nrays; ++ray) {
        int64_t i = ray * every;
        if (tag_of(attr[i]) != 0) continue;
        const float* T = poses + (int64_t)(frame[i] & (POSE_SLOTS - 1)) * 16;
        float ox = T[3], oy = T[7], oz = T[11];
        float wx, wy, wz;
        xform(T, xyz[i * stride], xyz[i * stride + 1], xyz[i * stride + 2], wx, wy, wz);
        float dx = wx - ox, dy = wy - oy, dz = wz - oz;
        float L = len3(dx, dy, dz);
        if (L < 0.05f || L > max_range) continue;
        dx = dx / L;
        dy = dy / L;
        dz = dz / L;
        float voxel = 1.0f / inv_voxel;
        float margin = fmaxf(3.0f * voxel, 0.03f * L);
        float pe[4];
        local_plane(ifloor(wx * inv_voxel), ifloor(wy * inv_voxel), ifloor(wz * inv_voxel), wx, wy, wz, m, pe);
        if (pe[3] > 0.5f) {
            float cosine = fabsf(pe[0] * dx + pe[1] * dy + pe[2] * dz);
            margin = fmaxf(margin, 1.5f * voxel / fmaxf(cosine, 0.05f));
        }
        float stop = (L - margin) * inv_voxel;
        if (stop <= 1.0f) continue;
        float posx = ox * inv_voxel, posy = oy * inv_voxel, posz = oz * inv_voxel;
        int ix = ifloor(posx), iy = ifloor(posy), iz = ifloor(posz);
        int sx = 1, sy = 1, sz = 1;
        float tmx = 1.0e30f, tmy = 1.0e30f, tmz = 1.0e30f, tdx = 1.0e30f, tdy = 1.0e30f, tdz = 1.0e30f;
        if (dx > 1.0e-9f) { tmx = ((float)(ix + 1) - posx) / dx; tdx = 1.0f / dx; }
        else if (dx < -1.0e-9f) { sx = -1; tmx = (posx - (float)ix) / (-dx); tdx = -1.0f / dx; }
        if (dy > 1.0e-9f) { tmy = ((float)(iy + 1) - posy) / dy; tdy = 1.0f / dy; }
        else if (dy < -1.0e-9f) { sy = -1; tmy = (posy - (float)iy) / (-dy); tdy = -1.0f / dy; }
        if (dz > 1.0e-9f) { tmz = ((float)(iz + 1) - posz) / dz; tdz = 1.0f / dz; }
        else if (dz < -1.0e-9f) { sz = -1; tmz = (posz - (float)iz) / (-dz); tdz = -1.0f / dz; }
        for (int step = 0; step < max_steps; ++step) {
            float tt;
            if (tmx < tmy && tmx < tmz) { tt = tmx; ix += sx; tmx += tdx; }
            else if (tmy < tmz) { tt = tmy; iy += sy; tmy += tdy; }
            else { tt = tmz; iz += sz; tmz += tdz; }
            if (tt >= stop) break;
            int s = find_slot(key_ijk(ix, iy, iz), keys, m.mask);
            if (s < 0 || cnt[s] <= 0) continue;
            float cx, cy, cz;
            centroid(m, s, cx, cy, cz);
            float rx = cx - ox, ry = cy - oy, rz = cz - oz;
            bool pierced = false;
            float pl[4];
            local_plane(ix, iy, iz, cx, cy, cz, m, pl);
            if (pl[3] > 1.5f) {
                float dn = dx * pl[0] + dy * pl[1] + dz * pl[2];
                if (fabsf(dn) > 1.0e-4f) {
                    float f = (rx * pl[0] + ry * pl[1] + rz * pl[2]) / dn;
                    float xx = dx * f - rx, xy = dy * f - ry, xz = dz * f - rz;
                    if (len3(xx, xy, xz) < 0.6f * voxel) pierced = true;
                }
            } else {
                float g = rx * dx + ry * dy + rz * dz;
                float qx = rx - g * dx, qy = ry - g * dy, qz = rz - g * dz;
                if (len3(qx, qy, qz) < 0.5f * voxel) pierced = true;
            }
            if (pierced) {
#pragma omp atomic
                miss[s] += every;
            }
        }
    }
}

// ---- visible set of the map (gpu.py:286-299, 596-634, 699-747), in slot order ---------------------------
static int transient(int c, int miss, const View& v) {
    if (miss < v.carve_min) return 0;
    return (float)miss > v.carve_ratio * (float)c ? 1 : 0;
}

int64_t or_map_build(int64_t cap, const int64_t* keys, const int32_t* cnt, const int64_t* acc, const float* last,
                     const float* first, const int32_t* miss, const View* vp, int min_count, float* out_xyz,
                     uint32_t* out_attr, float* out_t, int32_t* out_dyn) {
    const View& v = *vp;
    MapView m{keys, cnt, acc, (int)(cap - 1)};
    int64_t k = 0;
    for (int64_t s = 0; s < cap; ++s) {
        if (keys[s] == -1) continue;
        int c = cnt[s];
        if (c < min_count) continue;
        if (v.persist > 0.0f && v.now - last[s] > v.persist) continue;
        int gh = (v.now - last[s] < v.carve_stale) ? 0 : transient(c, miss[s], v);
        if (v.carve_on != 0 && gh != 0) continue;
        if (c <= 0) continue;
        float wx, wy, wz;
        centroid(m, (int)s, wx, wy, wz);
        if (v.crop_on != 0) {
            if (wx < v.crop_lo[0] || wy < v.crop_lo[1] || wz < v.crop_lo[2]) continue;
            if (wx > v.crop_hi[0] || wy > v.crop_hi[1] || wz > v.crop_hi[2]) continue;
        }
        int nn = c < MAP_CAP ? c : MAP_CAP;
        int refl = (int)((double)acc[4 * s + 3] / (double)nn + 0.5);
        if (refl > 255) refl = 255;
        out_xyz[3 * k] = wx;
        out_xyz[3 * k + 1] = wy;
        out_xyz[3 * k + 2] = wz;
        out_attr[k] = (uint32_t)refl;
        out_t[k] = last[s];
        int dyn = 0;
        if (transient(c, miss[s], v)) {
            dyn = 1;
        } else {
            int ix = ifloor(wx * v.inv_voxel), iy = ifloor(wy * v.inv_voxel), iz = ifloor(wz * v.inv_voxel);
            int settled = 0;
            for (int nb = 0; nb < 7 && !settled; ++nb) {
                int jx = ix, jy = iy, jz = iz;
                if (nb == 1) jx = ix - 1;
                else if (nb == 2) jx = ix + 1;
                else if (nb == 3) jy = iy - 1;
                else if (nb == 4) jy = iy + 1;
                else if (nb == 5) jz = iz - 1;
                else if (nb == 6) jz = iz + 1;
                int sn = find_slot(key_ijk(jx, jy, jz), keys, v.map_mask);
                if (sn >= 0) {
                    float age = v.now - first[sn];
                    if (age < 0.0f) age = 1.0e9f;
                    if (age >= v.dyn_settle && transient(cnt[sn], miss[sn], v) == 0) settled = 1;
                }
            }
            dyn = settled ? 0 : 1;
        }
        out_dyn[k] = dyn;
        ++k;
    }
    return k;
}

// ---- live ring visible set (k_classify_live gpu.py:637-697, Pipeline.build live mode :1466-1504) ---------------
// ring_xyz [cap*3]; poses [65536*16], tw [65536*6], owner_frame / owner_epoch [65536]; map arrays as lw_map (for
// the Motion label). Writes the drawn points in ring order and returns their count.
int64_t or_live_build(const float* ring_xyz, const uint32_t* ring_attr, const float* ring_t, const int32_t* ring_frame,
                      int64_t cap, int64_t filled, const float* poses, const float* tw, const int32_t* owner_frame,
                      const int32_t* owner_epoch, const View* vp, const int64_t* keys, const int32_t* cnt,
                      const float* first, const int32_t* miss, float* out_xyz, uint32_t* out_attr, float* out_t,
                      int32_t* out_dyn) {
    const View& v = *vp;
    int64_t k = 0;
    const int64_t nf = std::min(filled, cap);
    for (int64_t i = 0; i < nf; ++i) {
        const float t = ring_t[i];
        if (v.persist > 0.0f && v.now - t > v.persist) continue;
        float p[3] = {ring_xyz[3 * i], ring_xyz[3 * i + 1], ring_xyz[3 * i + 2]};
        const uint32_t a = ring_attr[i];
        if (!keep_raw(p[0], p[1], p[2], a, v)) continue;
        const int fid = ring_frame[i];
        const int f = fid & (POSE_SLOTS - 1);
        if (v.inv_frame_dt > 0.0f) {
            if (owner_frame[f] != fid || owner_epoch[f] != v.epoch) continue;
            const float xf = t * v.inv_frame_dt;
            const float frac = xf - floorf(xf) - 0.5f;
            float q[3];
            deskew_s(p[0], p[1], p[2], frac, tw + 6 * (int64_t)f, q);
            p[0] = q[0];
            p[1] = q[1];
            p[2] = q[2];
        }
        float wx, wy, wz;
        xform(poses + 16 * (int64_t)f, p[0], p[1], p[2], wx, wy, wz);
        if (v.crop_on != 0) {
            if (wx < v.crop_lo[0] || wy < v.crop_lo[1] || wz < v.crop_lo[2]) continue;
            if (wx > v.crop_hi[0] || wy > v.crop_hi[1] || wz > v.crop_hi[2]) continue;
        }
        out_xyz[3 * k] = wx;
        out_xyz[3 * k + 1] = wy;
        out_xyz[3 * k + 2] = wz;
        out_attr[k] = a;
        out_t[k] = t;
        int dyn = 0;
        if (v.dyn_on != 0) {
            const int ix = ifloor(wx * v.inv_voxel), iy = ifloor(wy * v.inv_voxel), iz = ifloor(wz * v.inv_voxel);
            int settled = 0;
            for (int nb = 0; nb < 7 && !settled; ++nb) {  // settled_near, gpu.py:596-634
                int jx = ix, jy = iy, jz = iz;
                if (nb == 1) jx = ix - 1;
                else if (nb == 2) jx = ix + 1;
                else if (nb == 3) jy = iy - 1;
                else if (nb == 4) jy = iy + 1;
                else if (nb == 5) jz = iz - 1;
                else if (nb == 6) jz = iz + 1;
                const int sn = find_slot(key_ijk(jx, jy, jz), keys, v.map_mask);
                if (sn >= 0) {
                    float age = v.now - first[sn];
                    if (age < 0.0f) age = 1.0e9f;
                    if (age >= v.dyn_settle && transient(cnt[sn], miss[sn], v) == 0) settled = 1;
                }
            }
            dyn = 1 - settled;
        }
        out_dyn[k] = dyn;
        ++k;
    }
    return k;
}


// ---- ground (perception.py:29-111, Perception.ground :458-483) -------------------------------------------------
// xyz [n*stride]; nrm [n*3] or null. The grid starts cleared on every call (the GPU keeps it cleared between calls).
void or_ground(const float* xyz, int stride, const float* nrm, int64_t n, float cell, float thick, int min_sup,
               float thresh, float slope_step, int use_normals, float nz_min, int32_t* out_gnd, float* out_hag) {
    const int G = 2048;
    const float inv = 1.0f / fmaxf(cell, 0.05f);
    std::vector<float> cmin((size_t)G * G, 1.0e30f);
    std::vector<int32_t> csup((size_t)G * G, 0);
    auto cell_of = [&](float x, float y) { return (ifloor(y * inv) & (G - 1)) * G + (ifloor(x * inv) & (G - 1)); };
    for (int64_t i = 0; i < n; ++i) {
        int c = cell_of(xyz[i * stride], xyz[i * stride + 1]);
        cmin[c] = std::min(cmin[c], xyz[i * stride + 2]);
    }
    for (int64_t i = 0; i < n; ++i) {
        int c = cell_of(xyz[i * stride], xyz[i * stride + 1]);
        if (xyz[i * stride + 2] - cmin[c] < thick) csup[c] += 1;
    }
    for (int64_t i = 0; i < n; ++i) {
        float x = xyz[i * stride], y = xyz[i * stride + 1], z = xyz[i * stride + 2];
        int cx = ifloor(x * inv), cy = ifloor(y * inv);
        float g = 1.0e30f, g_floor = 1.0e30f;
        for (int dy = -2; dy <= 2; ++dy)
            for (int dx = -2; dx <= 2; ++dx) {
                int c = ((cy + dy) & (G - 1)) * G + ((cx + dx) & (G - 1));
                if (csup[c] >= min_sup) {
                    float cand = cmin[c] + slope_step * (float)std::max(std::abs(dx), std::abs(dy));
                    if (cand < g) {
                        g = cand;
                        g_floor = cmin[c];
                    }
                }
            }
        if (g > 1.0e29f) {
            out_gnd[i] = 0;
            out_hag[i] = 0.0f;
            continue;
        }
        float h = z - g;
        int is_gnd = 0;
        if (h < thresh) {
            is_gnd = 1;
            if (use_normals && h > 0.2f * thresh && fabsf(nrm[i * 3 + 2]) < nz_min) is_gnd = 0;
        }
        out_gnd[i] = is_gnd;
        out_hag[i] = is_gnd ? h : z - g_floor;
    }
}

// ---- clusters (perception.py:114-271, 487-567) --------------------------------------------------------------
// Nodes are the occupied voxels in the order of their first point; components label a node by the smallest node
// index linked to it (what min-label propagation converges to); clusters are the roots with >= min_pts points,
// numbered in node order (at most max_out). Outputs: cid [n], labels [m] (returned count m via *m_out), cluster
// stats cnt [max_out], cen/lo/hi [max_out*3]; returns the number of clusters (before the cap) in *k_all.
int64_t or_cluster(const float* xyz, int stride, const int32_t* gnd, int use_ground, int64_t n, float voxel,
                   float connect, float min_pts, int max_out, int32_t* out_cid, int32_t* labels, int64_t* m_out,
                   float* out_cnt, float* out_cen, float* out_lo, float* out_hi, int64_t* k_all) {
    const float inv = 1.0f / fmaxf(voxel, 0.01f);
    const float FW = (float)FIX_W;
    std::unordered_map<int64_t, int> node_of;
    std::vector<int64_t> nkey;
    std::vector<std::array<int64_t, 4>> nacc;
    std::vector<int> pt_node(n, -1);
    for (int64_t i = 0; i < n; ++i) {
        if (use_ground && gnd[i] != 0) continue;
        float x = xyz[i * stride], y = xyz[i * stride + 1], z = xyz[i * stride + 2];
        int64_t key = key_ijk(ifloor(x * inv), ifloor(y * inv), ifloor(z * inv));
        auto it = node_of.find(key);
        int j;
        if (it == node_of.end()) {
            j = (int)nkey.size();
            node_of.emplace(key, j);
            nkey.push_back(key);
            nacc.push_back({0, 0, 0, 0});
        } else {
            j = it->second;
        }
        nacc[j][0] += llrintf(x * FW);
        nacc[j][1] += llrintf(y * FW);
        nacc[j][2] += llrintf(z * FW);
        nacc[j][3] += 1;
        pt_node[i] = j;
    }
    const int m = (int)nkey.size();
    *m_out = m;
    std::vector<float> cen((size_t)m * 3);
    for (int j = 0; j < m; ++j)
        for (int d = 0; d < 3; ++d) cen[3 * j + d] = (float)((double)nacc[j][d] / ((double)nacc[j][3] * FIX_W));
    int reach = (int)ceilf(connect * inv);
    if (reach < 1) reach = 1;
    const float c2 = connect * connect;
    std::vector<int> parent(m);
    for (int j = 0; j < m; ++j) parent[j] = j;
    std::function<int(int)> find = [&](int x) {
        while (parent[x] != x) {
            parent[x] = parent[parent[x]];
            x = parent[x];
        }
        return x;
    };
    for (int j = 0; j < m; ++j) {
        int64_t key = nkey[j];
        int ix = (int)(key & KMASK) - (int)BIAS, iy = (int)((key >> 21) & KMASK) - (int)BIAS,
            iz = (int)((key >> 42) & KMASK) - (int)BIAS;
        for (int dx = -reach; dx <= reach; ++dx)
            for (int dy = -reach; dy <= reach; ++dy)
                for (int dz = -reach; dz <= reach; ++dz) {
                    if (!dx && !dy && !dz) continue;
                    auto it = node_of.find(key_ijk(ix + dx, iy + dy, iz + dz));
                    if (it == node_of.end()) continue;
                    int k = it->second;
                    float ex = cen[3 * k] - cen[3 * j], ey = cen[3 * k + 1] - cen[3 * j + 1], ez = cen[3 * k + 2] - cen[3 * j + 2];
                    if (ex * ex + ey * ey + ez * ez <= c2) {
                        int a = find(j), b = find(k);
                        if (a != b) parent[std::max(a, b)] = std::min(a, b);
                    }
                }
    }
    for (int j = 0; j < m; ++j) labels[j] = find(j);
    std::vector<std::array<int64_t, 4>> ssum(m, {0, 0, 0, 0});
    std::vector<float> lo((size_t)m * 3, 1.0e30f), hi((size_t)m * 3, -1.0e30f);
    for (int j = 0; j < m; ++j) {
        int r = labels[j];
        for (int d = 0; d < 4; ++d) ssum[r][d] += nacc[j][d];
        for (int d = 0; d < 3; ++d) {
            lo[3 * r + d] = std::min(lo[3 * r + d], cen[3 * j + d]);
            hi[3 * r + d] = std::max(hi[3 * r + d], cen[3 * j + d]);
        }
    }
    std::vector<int> dense(m, -1);
    int64_t k = 0;
    for (int j = 0; j < m; ++j) {
        if (labels[j] != j || (float)ssum[j][3] < min_pts) continue;
        if (k < max_out) {
            dense[j] = (int)k;
            double w = (double)ssum[j][3];
            out_cnt[k] = (float)ssum[j][3];
            for (int d = 0; d < 3; ++d) {
                out_cen[3 * k + d] = (float)((double)ssum[j][d] / (w * FIX_W));
                out_lo[3 * k + d] = lo[3 * j + d];
                out_hi[3 * k + d] = hi[3 * j + d];
            }
        }
        ++k;
    }
    *k_all = k;
    for (int64_t i = 0; i < n; ++i) out_cid[i] = pt_node[i] < 0 ? -1 : dense[labels[pt_node[i]]];
    return k < max_out ? k : max_out;
}


// ---- prior-map grid (mapgrid.py) -----------------------------------------------------------------------------
// The grid geometry, nearest_point and the build follow mapgrid.py:35-170 with two deliberate differences that the
// GPU build shares: the seed key is 64 bits (distance mm << 32 | index; the reference's 32-bit key held 2^23 - 1
// points), and each flood step reads one buffer and writes another (the reference floods in place, so its result
// depends on thread timing).

typedef struct or_grid {
    const float* xyz;
    const float* nrm;
    const float* planar;
    const int32_t* start;
    const int32_t* nn;
    float origin[3];
    float cell, inv_cell;
    int32_t nx, ny, nz, pad_;
} or_grid;

}  // extern "C"

static inline int64_t og_flat(const or_grid& g, int ix, int iy, int iz) {  // grid_flat mapgrid.py:46-50
    if (ix < 0 || iy < 0 || iz < 0 || ix >= g.nx || iy >= g.ny || iz >= g.nz) return -1;
    return ((int64_t)iz * g.ny + iy) * g.nx + ix;
}
static inline void og_centre(const or_grid& g, int64_t c, float& x, float& y, float& z) {  // cell_centre :59-65
    int64_t ix = c % g.nx, r = c / g.nx;
    int64_t iy = r % g.ny, iz = r / g.ny;
    x = g.origin[0] + ((float)ix + 0.5f) * g.cell;
    y = g.origin[1] + ((float)iy + 0.5f) * g.cell;
    z = g.origin[2] + ((float)iz + 0.5f) * g.cell;
}
// nearest_point mapgrid.py:68-102
static int og_nearest(const or_grid& g, float wx, float wy, float wz) {
    int ix = ifloor((wx - g.origin[0]) * g.inv_cell);
    int iy = ifloor((wy - g.origin[1]) * g.inv_cell);
    int iz = ifloor((wz - g.origin[2]) * g.inv_cell);
    int best = -1, seed = -1;
    float bd = g.cell * g.cell, sd = 1.0e30f;
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                int64_t c = og_flat(g, ix + dx, iy + dy, iz + dz);
                if (c < 0) continue;
                for (int k = g.start[c]; k < g.start[c + 1]; ++k) {
                    const float* q = g.xyz + 3 * (int64_t)k;
                    float ex = wx - q[0], ey = wy - q[1], ez = wz - q[2];
                    float d2 = ex * ex + ey * ey + ez * ez;
                    if (d2 < bd) {
                        bd = d2;
                        best = k;
                    }
                }
                if (best < 0) {
                    int s = g.nn[c];
                    if (s >= 0) {
                        const float* q = g.xyz + 3 * (int64_t)s;
                        float ex = wx - q[0], ey = wy - q[1], ez = wz - q[2];
                        float d2 = ex * ex + ey * ey + ez * ez;
                        if (d2 < sd) {
                            sd = d2;
                            seed = s;
                        }
                    }
                }
            }
    return best >= 0 ? best : seed;
}

extern "C" {

// k_seed, k_unpack, k_jfa x JFA_STEPS, k_df (mapgrid.py:105-170, PriorGrid.build :272-296) into nn and df.
void or_grid_build(const or_grid* gp, int64_t n, int32_t* nn, uint8_t* df, int threads) {
    const or_grid& g = *gp;
    const int64_t ncell = (int64_t)g.nx * g.ny * g.nz;
    std::vector<uint64_t> seed(ncell, ~0ULL);
    for (int64_t i = 0; i < n; ++i) {
        const float* p = g.xyz + 3 * i;
        int64_t c = og_flat(g, ifloor((p[0] - g.origin[0]) * g.inv_cell), ifloor((p[1] - g.origin[1]) * g.inv_cell),
                            ifloor((p[2] - g.origin[2]) * g.inv_cell));
        if (c < 0) continue;
        float cx, cy, cz;
        og_centre(g, c, cx, cy, cz);
        int dmm = (int)(len3(p[0] - cx, p[1] - cy, p[2] - cz) * 1000.0f);
        if (dmm > 255) dmm = 255;
        uint64_t key = ((uint64_t)dmm << 32) | (uint64_t)i;
        if (key < seed[c]) seed[c] = key;
    }
    std::vector<int32_t> a(ncell), b(ncell);
    for (int64_t c = 0; c < ncell; ++c) a[c] = seed[c] == ~0ULL ? -1 : (int32_t)(seed[c] & 0xFFFFFFFFULL);
    const int steps[5] = {8, 4, 2, 1, 1};
    for (int st = 0; st < 5; ++st) {
        const int step = steps[st];
#pragma omp parallel for num_threads(threads) schedule(static)
        for (int64_t c = 0; c < ncell; ++c) {
            float px, py, pz;
            og_centre(g, c, px, py, pz);
            int ix = (int)(c % g.nx), iy = (int)((c / g.nx) % g.ny), iz = (int)(c / ((int64_t)g.nx * g.ny));
            int best = a[c];
            float bd = 1.0e30f;
            if (best >= 0) {
                const float* q = g.xyz + 3 * (int64_t)best;
                float ex = px - q[0], ey = py - q[1], ez = pz - q[2];
                bd = ex * ex + ey * ey + ez * ez;
            }
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        int64_t j = og_flat(g, ix + dx * step, iy + dy * step, iz + dz * step);
                        if (j < 0 || j == c) continue;
                        int s = a[j];
                        if (s < 0 || s == best) continue;
                        const float* q = g.xyz + 3 * (int64_t)s;
                        float ex = px - q[0], ey = py - q[1], ez = pz - q[2];
                        float d2 = ex * ex + ey * ey + ez * ez;
                        if (d2 < bd) {
                            bd = d2;
                            best = s;
                        }
                    }
            b[c] = best;
        }
        a.swap(b);
    }
    for (int64_t c = 0; c < ncell; ++c) {
        nn[c] = a[c];
        if (a[c] < 0) {
            df[c] = 255;
            continue;
        }
        float px, py, pz;
        og_centre(g, c, px, py, pz);
        const float* q = g.xyz + 3 * (int64_t)a[c];
        float d = len3(px - q[0], py - q[1], pz - q[2]) * 100.0f;
        int v = (int)(d + 0.5f);
        df[c] = (uint8_t)(v < 255 ? v : 255);
    }
}

// nearest_point for n query points (mapgrid.py:68-102).
void or_nearest(const or_grid* g, const float* w, int64_t n, int32_t* out, int threads) {
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int64_t i = 0; i < n; ++i) out[i] = og_nearest(*g, w[3 * i], w[3 * i + 1], w[3 * i + 2]);
}

// k_changes_T (mapgrid.py:173-194): distance of each point posed by T (float32, as the kernel's mat44) to the map.
void or_prior_distances(const or_grid* g, const float* pts, int64_t n, const double* T, float* out, int threads) {
    float M[12];
    for (int k = 0; k < 12; ++k) M[k] = (float)T[k];
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const float* p = pts + 3 * i;
        float wx = M[0] * p[0] + M[1] * p[1] + M[2] * p[2] + M[3];
        float wy = M[4] * p[0] + M[5] * p[1] + M[6] * p[2] + M[7];
        float wz = M[8] * p[0] + M[9] * p[1] + M[10] * p[2] + M[11];
        int s = og_nearest(*g, wx, wy, wz);
        float d = 1.0e3f;
        if (s >= 0) {
            const float* q = g->xyz + 3 * (int64_t)s;
            d = len3(wx - q[0], wy - q[1], wz - q[2]);
        }
        out[i] = d;
    }
}

}  // extern "C"

// ---- neighbourhoods of the visible points (gpu.py:777-905) --------------------------------------------------------
// The library's definition: points summed into voxels radius / 3 wide (int64 fixed point), each voxel's neighbours
// the voxels whose centroid lies within the radius (found among the 7 x 7 x 7 voxel offsets), their weight,
// weighted offsets and outer products summed in fixed point, the covariance and its eigen-decomposition in float64.
// The reference uses float atomics and a hash-grid query order instead (its sums depend on thread timing).

extern "C" {

void or_neighborhoods(const float* xyz, int stride, int64_t n, float radius, int want_normals, const float* sensor,
                      int32_t* out_cnt, float* out_nrm, float* out_curv, int threads) {
    const float inv_h = 3.0f / radius, r2 = radius * radius;
    const float FW = (float)1048576.0, FD = (float)1048576.0, FDD = (float)1099511627776.0;
    std::unordered_map<int64_t, int> vox;
    std::vector<int64_t> keys, acc;
    std::vector<int> of_pt(n);
    for (int64_t i = 0; i < n; ++i) {
        const float x = xyz[stride * i], y = xyz[stride * i + 1], z = xyz[stride * i + 2];
        const int64_t key = or_key_ijk((int)std::floor(x * inv_h), (int)std::floor(y * inv_h), (int)std::floor(z * inv_h));
        auto it = vox.find(key);
        int v;
        if (it == vox.end()) {
            v = (int)keys.size();
            vox.emplace(key, v);
            keys.push_back(key);
            acc.insert(acc.end(), {0, 0, 0, 0});
        } else {
            v = it->second;
        }
        acc[4 * v + 0] += llrintf(x * FW);
        acc[4 * v + 1] += llrintf(y * FW);
        acc[4 * v + 2] += llrintf(z * FW);
        acc[4 * v + 3] += 1;
        of_pt[i] = v;
    }
    const int m = (int)keys.size();
    std::vector<float> c(3 * (size_t)m), cnt(m), nrm(3 * (size_t)m), curv(m);
    for (int v = 0; v < m; ++v) {
        const double w = (double)acc[4 * v + 3];
        for (int k = 0; k < 3; ++k) c[3 * v + k] = (float)((double)acc[4 * v + k] / (w * 1048576.0));
    }
#pragma omp parallel for num_threads(threads) schedule(dynamic, 64)
    for (int v = 0; v < m; ++v) {
        const int64_t key = keys[v];
        const int ix = (int)(key & 0x1FFFFF) - (1 << 20), iy = (int)((key >> 21) & 0x1FFFFF) - (1 << 20),
                  iz = (int)((key >> 42) & 0x1FFFFF) - (1 << 20);
        const float px = c[3 * v], py = c[3 * v + 1], pz = c[3 * v + 2];
        long long W = 0, s1[3] = {0, 0, 0}, s2[6] = {0, 0, 0, 0, 0, 0};
        for (int dx = -3; dx <= 3; ++dx)
            for (int dy = -3; dy <= 3; ++dy)
                for (int dz = -3; dz <= 3; ++dz) {
                    auto it = vox.find(or_key_ijk(ix + dx, iy + dy, iz + dz));
                    if (it == vox.end()) continue;
                    const int k = it->second;
                    const float ex = c[3 * k] - px, ey = c[3 * k + 1] - py, ez = c[3 * k + 2] - pz;
                    if (ex * ex + ey * ey + ez * ez > r2) continue;
                    const long long wk = acc[4 * k + 3];
                    W += wk;
                    s1[0] += wk * llrintf(ex * FD);
                    s1[1] += wk * llrintf(ey * FD);
                    s1[2] += wk * llrintf(ez * FD);
                    s2[0] += wk * llrintf(ex * ex * FDD);
                    s2[1] += wk * llrintf(ex * ey * FDD);
                    s2[2] += wk * llrintf(ex * ez * FDD);
                    s2[3] += wk * llrintf(ey * ey * FDD);
                    s2[4] += wk * llrintf(ey * ez * FDD);
                    s2[5] += wk * llrintf(ez * ez * FDD);
                }
        cnt[v] = (float)W;
        if (!want_normals) continue;
        double tx = (double)sensor[0] - (double)px, ty = (double)sensor[1] - (double)py, tz = (double)sensor[2] - (double)pz;
        const double tl = std::sqrt(tx * tx + ty * ty + tz * tz);
        if (tl > 0.0) {
            tx /= tl;
            ty /= tl;
            tz /= tl;
        }
        const double inv = 1.0 / std::max((double)W, 1.0);
        const double mu[3] = {(double)s1[0] / 1048576.0 * inv, (double)s1[1] / 1048576.0 * inv,
                              (double)s1[2] / 1048576.0 * inv};
        const int up[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
        double C[9], ev[3], Q[9];
        for (int r = 0; r < 3; ++r)
            for (int q = 0; q < 3; ++q) C[r * 3 + q] = (double)s2[up[r * 3 + q]] / 1099511627776.0 * inv - mu[r] * mu[q];
        jacobi<3>(C, ev, Q);
        int kmin = 0;
        if (ev[1] < ev[kmin]) kmin = 1;
        if (ev[2] < ev[kmin]) kmin = 2;
        double nx = Q[0 * 3 + kmin], ny = Q[1 * 3 + kmin], nz = Q[2 * 3 + kmin];
        const double nl = std::sqrt(nx * nx + ny * ny + nz * nz);
        if (nl > 0.0) {
            nx /= nl;
            ny /= nl;
            nz /= nl;
        }
        if (nx * tx + ny * ty + nz * tz < 0.0) {
            nx = -nx;
            ny = -ny;
            nz = -nz;
        }
        const double tr = ev[0] + ev[1] + ev[2];
        if (tr <= 1.0e-12) {
            nx = tx;
            ny = ty;
            nz = tz;
        }
        nrm[3 * v] = (float)nx;
        nrm[3 * v + 1] = (float)ny;
        nrm[3 * v + 2] = (float)nz;
        curv[v] = (float)(std::max(ev[kmin], 0.0) / std::max(tr, 1.0e-12));
    }
    for (int64_t i = 0; i < n; ++i) {
        const int v = of_pt[i];
        out_cnt[i] = (int)(cnt[v] + 0.5f);
        if (want_normals) {
            for (int k = 0; k < 3; ++k) out_nrm[3 * i + k] = nrm[3 * v + k];
            out_curv[i] = curv[v];
        }
    }
}

}  // extern "C"

// ---- coarse hypothesis scores (localize.py:55-123, k_score_grid / k_score_list) --------------------------------
// Two sums. By default the definition the library computes: the soft count formed exactly from the number of
// points with d < tau and the sum of their d^2 (integers), rounded once. With ref, the reference's own sum: float32
// terms 1 - d*d*inv_t2 added in point order. Both pose the points with the reference's expressions
// (localize.py:89, 117) and the headings' cosines and sines taken in float64 and rounded to float32 (the
// reference's float32 wp.cos / wp.sin may differ from those by an ulp).

static inline int64_t og_at(const or_grid& g, float x, float y, float z) {  // grid_at mapgrid.py:53-56
    return og_flat(g, (int)std::floor((x - g.origin[0]) * g.inv_cell), (int)std::floor((y - g.origin[1]) * g.inv_cell),
                   (int)std::floor((z - g.origin[2]) * g.inv_cell));
}

static inline void og_score_sums(const or_grid& g, const uint8_t* df, const float* pts, int n_pts, float cx, float cy,
                                 float cz, float co, float si, float tau, int& n_in, int& sum_d2) {
    n_in = 0;
    sum_d2 = 0;
    for (int k = 0; k < n_pts; ++k) {
        const float* p = pts + 3 * (int64_t)k;
        const float wx = cx + co * p[0] - si * p[1];
        const float wy = cy + si * p[0] + co * p[1];
        const float wz = cz + p[2];
        const int64_t j = og_at(g, wx, wy, wz);
        if (j >= 0) {
            const int d = df[j];
            if ((float)d < tau) {
                ++n_in;
                sum_d2 += d * d;
            }
        }
    }
}

static inline float og_score_ref(const or_grid& g, const uint8_t* df, const float* pts, int n_pts, float cx, float cy,
                                 float cz, float co, float si, float tau) {
    const float inv_t2 = 1.0f / (tau * tau);
    float s = 0.0f;
    for (int k = 0; k < n_pts; ++k) {
        const float* p = pts + 3 * (int64_t)k;
        const float wx = cx + co * p[0] - si * p[1];
        const float wy = cy + si * p[0] + co * p[1];
        const float wz = cz + p[2];
        const int64_t j = og_at(g, wx, wy, wz);
        if (j >= 0) {
            const float d = (float)df[j];
            if (d < tau) s += 1.0f - d * d * inv_t2;
        }
    }
    return s;
}

extern "C" {

void or_score_grid(const or_grid* gp, const uint8_t* df, const float* pts, int n_pts, const float* pos, int64_t n_pos,
                   int n_yaw, float yaw0, float dyaw, float tau, float free_cm, int ref, float* out, int threads) {
    const or_grid& g = *gp;
    std::vector<float> c(n_yaw), sn(n_yaw);
    for (int j = 0; j < n_yaw; ++j) {
        const float yaw = yaw0 + (float)j * dyaw;
        c[j] = (float)std::cos((double)yaw);
        sn[j] = (float)std::sin((double)yaw);
    }
    const int64_t n_hyp = n_pos * n_yaw;
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int64_t h = 0; h < n_hyp; ++h) {
        const int64_t ip = h / n_yaw;
        const int iyaw = (int)(h - ip * n_yaw);
        const float cx = pos[3 * ip], cy = pos[3 * ip + 1], cz = pos[3 * ip + 2];
        const int64_t cc = og_at(g, cx, cy, cz);
        if (cc < 0 || (float)df[cc] < free_cm) {
            out[h] = -1.0f;
            continue;
        }
        if (ref) {
            out[h] = og_score_ref(g, df, pts, n_pts, cx, cy, cz, c[iyaw], sn[iyaw], tau);
        } else {
            int n_in, sum_d2;
            og_score_sums(g, df, pts, n_pts, cx, cy, cz, c[iyaw], sn[iyaw], tau, n_in, sum_d2);
            out[h] = (float)((double)n_in - (double)sum_d2 / ((double)tau * (double)tau));
        }
    }
}

void or_score_list(const or_grid* gp, const uint8_t* df, const float* pts, int n_pts, const float* hyp, int64_t n_hyp,
                   float tau, int ref, float* out, int threads) {
    const or_grid& g = *gp;
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int64_t h = 0; h < n_hyp; ++h) {
        const float* q = hyp + 4 * h;
        const float co = (float)std::cos((double)q[3]);
        const float si = (float)std::sin((double)q[3]);
        if (ref) {
            out[h] = og_score_ref(g, df, pts, n_pts, q[0], q[1], q[2], co, si, tau);
        } else {
            int n_in, sum_d2;
            og_score_sums(g, df, pts, n_pts, q[0], q[1], q[2], co, si, tau, n_in, sum_d2);
            out[h] = (float)((double)n_in - (double)sum_d2 / ((double)tau * (double)tau));
        }
    }
}

}  // extern "C"

// ---- batched point-to-plane ICP (localize.py) ------------------------------------------------------------------

// solve A x = r by Gaussian elimination with partial pivoting (numpy.linalg.solve); false when A is singular
static bool or_solve6(double A[36], double r[6], double x[6]) {
    int piv[6] = {0, 1, 2, 3, 4, 5};
    for (int c = 0; c < 6; ++c) {
        int p = c;
        for (int k = c + 1; k < 6; ++k)
            if (fabs(A[piv[k] * 6 + c]) > fabs(A[piv[p] * 6 + c])) p = k;
        std::swap(piv[c], piv[p]);
        double d = A[piv[c] * 6 + c];
        if (d == 0.0) return false;
        for (int k = c + 1; k < 6; ++k) {
            double f = A[piv[k] * 6 + c] / d;
            for (int j = c; j < 6; ++j) A[piv[k] * 6 + j] -= f * A[piv[c] * 6 + j];
            r[piv[k]] -= f * r[piv[c]];
        }
    }
    for (int c = 5; c >= 0; --c) {
        double s = r[piv[c]];
        for (int j = c + 1; j < 6; ++j) s -= A[piv[c] * 6 + j] * x[j];
        x[c] = s / A[piv[c] * 6 + c];
    }
    return true;
}

// _twist_apply (localize.py:227-233): T <- [exp(delta_r), delta_t] T, the rotation by Rodrigues' formula.
static void or_twist_apply(double* T, const double* d) {
    double th = sqrt(d[3] * d[3] + d[4] * d[4] + d[5] * d[5]);
    double R[9];
    if (th < 1e-12) {
        const double I[9] = {1, -d[5], d[4], d[5], 1, -d[3], -d[4], d[3], 1};
        for (int k = 0; k < 9; ++k) R[k] = I[k];
    } else {
        double x = d[3] / th, y = d[4] / th, z = d[5] / th, s = sin(th), c = cos(th), v = 1.0 - c;
        const double Q[9] = {c + x * x * v, x * y * v - z * s, x * z * v + y * s,
                             y * x * v + z * s, c + y * y * v, y * z * v - x * s,
                             z * x * v - y * s, z * y * v + x * s, c + z * z * v};
        for (int k = 0; k < 9; ++k) R[k] = Q[k];
    }
    double o[12];
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) o[i * 4 + j] = R[i * 3] * T[j] + R[i * 3 + 1] * T[4 + j] + R[i * 3 + 2] * T[8 + j];
        o[i * 4 + 3] = R[i * 3] * T[3] + R[i * 3 + 1] * T[7] + R[i * 3 + 2] * T[11] + d[i];
    }
    for (int k = 0; k < 12; ++k) T[k] = o[k];
}

static inline void or_posef(const double* T, float* M) {
    for (int k = 0; k < 12; ++k) M[k] = (float)T[k];
}
static inline void or_xform(const float* M, const float* p, float& wx, float& wy, float& wz) {
    wx = M[0] * p[0] + M[1] * p[1] + M[2] * p[2] + M[3];
    wy = M[4] * p[0] + M[5] * p[1] + M[6] * p[2] + M[7];
    wz = M[8] * p[0] + M[9] * p[1] + M[10] * p[2] + M[11];
}

extern "C" {

// GlobalLocalizer._icp (localize.py:517-553) with k_icp_batch / k_reduce_batch (:126-179) in float64: every
// hypothesis h registers pts4[scan_lo[h] .. scan_hi[h]) (x, y, z, unused) from T[16h..] (row-major, updated).
// The correspondences are chosen in float32 as the kernel does (the pose cast to float32, w = T p); the terms
// are formed and summed in float64. max_d2 and c2 are the float32 values the kernel receives.
void or_loc_icp(const or_grid* gp, const float* pts4, const int32_t* scan_lo, const int32_t* scan_hi, int n_hyp,
                double* T, int n_stages, const float* max_d2, const float* c2, const int32_t* iters, float alpha,
                int min_count, int32_t* count, int32_t* iters_run, int threads) {
    const or_grid& g = *gp;
    const float PLANAR_F = 0.5f;
    int run = 0;
    std::vector<double> moved(n_hyp);
    for (int st = 0; st < n_stages; ++st) {
        for (int it = 0; it < iters[st]; ++it) {
            ++run;
#pragma omp parallel for num_threads(threads) schedule(dynamic, 1)
            for (int h = 0; h < n_hyp; ++h) {
                float M[12];
                or_posef(T + 16 * h, M);
                double H[36] = {0}, bv[6] = {0};
                int64_t cnt = 0;
                for (int64_t i = scan_lo[h]; i < scan_hi[h]; ++i) {
                    float wx, wy, wz;
                    or_xform(M, pts4 + 4 * i, wx, wy, wz);
                    int s = og_nearest(g, wx, wy, wz);
                    if (s < 0) continue;
                    const float* q = g.xyz + 3 * (int64_t)s;
                    float rx = wx - q[0], ry = wy - q[1], rz = wz - q[2];
                    if (rx * rx + ry * ry + rz * rz > max_d2[st]) continue;
                    const float* nv = g.nrm + 3 * (int64_t)s;
                    double Mm[9];
                    if (g.planar[s] > PLANAR_F && len3(nv[0], nv[1], nv[2]) > 0.5f) {
                        double a = alpha, b1 = 1.0 - (double)alpha, n3[3] = {nv[0], nv[1], nv[2]};
                        for (int r = 0; r < 3; ++r)
                            for (int c = 0; c < 3; ++c) Mm[r * 3 + c] = n3[r] * n3[c] * b1 + (r == c ? a : 0.0);
                    } else {
                        for (int k = 0; k < 9; ++k) Mm[k] = (k % 4 == 0) ? 4.0 * alpha : 0.0;
                    }
                    double r3[3] = {rx, ry, rz}, Mr[3];
                    for (int r = 0; r < 3; ++r) Mr[r] = Mm[r * 3] * r3[0] + Mm[r * 3 + 1] * r3[1] + Mm[r * 3 + 2] * r3[2];
                    double d2 = r3[0] * Mr[0] + r3[1] * Mr[1] + r3[2] * Mr[2];
                    double wgt = 1.0 / (1.0 + d2 / (double)c2[st]);
                    wgt *= wgt;
                    const double W[3] = {wx, wy, wz};
                    // J = [I | -[w]x] (localize.py:160-162)
                    const double J[3][6] = {{1, 0, 0, 0, W[2], -W[1]}, {0, 1, 0, -W[2], 0, W[0]}, {0, 0, 1, W[1], -W[0], 0}};
                    double MJ[3][6];
                    for (int r = 0; r < 3; ++r)
                        for (int c = 0; c < 6; ++c) MJ[r][c] = Mm[r * 3] * J[0][c] + Mm[r * 3 + 1] * J[1][c] + Mm[r * 3 + 2] * J[2][c];
                    for (int p = 0; p < 6; ++p) {
                        for (int qq = 0; qq < 6; ++qq) H[p * 6 + qq] += wgt * (J[0][p] * MJ[0][qq] + J[1][p] * MJ[1][qq] + J[2][p] * MJ[2][qq]);
                        bv[p] += wgt * (J[0][p] * Mr[0] + J[1][p] * Mr[1] + J[2][p] * Mr[2]);
                    }
                    ++cnt;
                }
                count[h] = (int32_t)cnt;
                moved[h] = 0.0;
                if (cnt < min_count) continue;
                double A[36], rhs[6], delta[6];
                for (int k = 0; k < 36; ++k) A[k] = H[k];
                for (int p = 0; p < 6; ++p) {
                    A[p * 7] += 1e-3 * H[p * 7] + 1e-9;
                    rhs[p] = -bv[p];
                }
                if (!or_solve6(A, rhs, delta)) continue;
                or_twist_apply(T + 16 * h, delta);
                double nt = sqrt(delta[0] * delta[0] + delta[1] * delta[1] + delta[2] * delta[2]);
                double nr = sqrt(delta[3] * delta[3] + delta[4] * delta[4] + delta[5] * delta[5]);
                moved[h] = std::max(nt, 5.0 * nr);
            }
            double mv = 0.0;
            for (int h = 0; h < n_hyp; ++h) mv = std::max(mv, moved[h]);
            if (mv < 2e-4) break;
        }
    }
    *iters_run = run;
}

// k_eval_batch (localize.py:182-205): per hypothesis, the points within radii[k] of their nearest map point.
void or_loc_eval(const or_grid* gp, const float* pts4, const int32_t* scan_lo, const int32_t* scan_hi, int n_hyp,
                 const double* T, const float* radii, int32_t* counts, int threads) {
#pragma omp parallel for num_threads(threads) schedule(dynamic, 1)
    for (int h = 0; h < n_hyp; ++h) {
        float M[12];
        or_posef(T + 16 * h, M);
        int32_t c[3] = {0, 0, 0};
        for (int64_t i = scan_lo[h]; i < scan_hi[h]; ++i) {
            float wx, wy, wz;
            or_xform(M, pts4 + 4 * i, wx, wy, wz);
            int s = og_nearest(*gp, wx, wy, wz);
            if (s < 0) continue;
            const float* q = gp->xyz + 3 * (int64_t)s;
            float d = len3(wx - q[0], wy - q[1], wz - q[2]);
            for (int k = 0; k < 3; ++k) c[k] += d < radii[k];
        }
        for (int k = 0; k < 3; ++k) counts[3 * h + k] = c[k];
    }
}

}  // extern "C"

// ---- prior maps: voxel downsample and PCA normals (prior_map.py:57-219) --------------------------------------------
// The library's definition. Voxel means: offsets from the voxel centre ((i + 0.5) * voxel, float32) summed in int64
// fixed point (2^(30 - e) units per metre, voxel < 2^e), colour and intensity in 2^16 units, the voxels numbered in
// the order of their first point; the mean is centre + sum / (count * units) in float64, rounded once. The reference
// sums float32 offsets with float atomics and emits in hash-slot order. Normals: every point within the radius
// (|q - p|^2 <= r^2 in float32), its offset and the offset's products summed in fixed point (2^20 and 2^40 units
// of the radius' power of two), covariance and Jacobi in float64; the reference sums float32 in query order and
// decomposes with a float32 eig3.

extern "C" {

int64_t or_voxel_downsample(const float* xyz, int64_t n, const float* inten, const float* rgb, float voxel,
                            float* out_xyz, float* out_rgb, float* out_inten, int32_t* out_cnt) {
    const float inv_v = (float)(1.0 / (double)voxel);
    int e = 0;
    frexpf(voxel, &e);
    const float fo = (float)ldexp(1.0, 30 - e), fa = 65536.0f;
    std::unordered_map<int64_t, int64_t> vox;
    std::vector<int64_t> keys, acc;
    for (int64_t i = 0; i < n; ++i) {
        const float x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
        const int ix = ifloor(x * inv_v), iy = ifloor(y * inv_v), iz = ifloor(z * inv_v);
        const int64_t key = key_ijk(ix, iy, iz);
        auto it = vox.find(key);
        int64_t v;
        if (it == vox.end()) {
            v = (int64_t)keys.size();
            vox.emplace(key, v);
            keys.push_back(key);
            acc.insert(acc.end(), 8, 0);
        } else {
            v = it->second;
        }
        int64_t* a = acc.data() + 8 * v;
        a[0] += llrintf((x - ((float)ix + 0.5f) * voxel) * fo);
        a[1] += llrintf((y - ((float)iy + 0.5f) * voxel) * fo);
        a[2] += llrintf((z - ((float)iz + 0.5f) * voxel) * fo);
        if (rgb)
            for (int c = 0; c < 3; ++c) a[3 + c] += llrintf(rgb[3 * i + c] * fa);
        if (inten) a[6] += llrintf(inten[i] * fa);
        a[7] += 1;
    }
    const int64_t m = (int64_t)keys.size();
    for (int64_t j = 0; j < m; ++j) {
        const int64_t key = keys[j];
        const int ix = (int)(key & KMASK) - (int)BIAS, iy = (int)((key >> 21) & KMASK) - (int)BIAS,
                  iz = (int)((key >> 42) & KMASK) - (int)BIAS;
        const int64_t* a = acc.data() + 8 * j;
        const double c = (double)a[7], uo = c * (double)fo, ua = c * 65536.0;
        out_xyz[3 * j + 0] = (float)((double)(((float)ix + 0.5f) * voxel) + (double)a[0] / uo);
        out_xyz[3 * j + 1] = (float)((double)(((float)iy + 0.5f) * voxel) + (double)a[1] / uo);
        out_xyz[3 * j + 2] = (float)((double)(((float)iz + 0.5f) * voxel) + (double)a[2] / uo);
        for (int k = 0; k < 3; ++k) out_rgb[3 * j + k] = (float)((double)a[3 + k] / ua);
        out_inten[j] = (float)((double)a[6] / ua);
        out_cnt[j] = (int32_t)std::min<int64_t>(a[7], 0x7FFFFFFF);
    }
    return m;
}

void or_normals(const float* xyz, int64_t n, float radius, float* out_nrm, float* out_pl, int threads) {
    const float inv_h = (float)(1.0 / ((double)radius * 1.00390625)), r2 = radius * radius;
    int e = 0;
    frexpf(radius, &e);
    const double fd64 = ldexp(1.0, 20 - e), fdd64 = ldexp(1.0, 40 - 2 * e);
    const float fd = (float)fd64, fdd = (float)fdd64;
    std::unordered_map<int64_t, std::vector<int64_t>> cells;
    for (int64_t i = 0; i < n; ++i) {
        const float x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
        const int64_t key = key_ijk(ifloor(x * inv_h), ifloor(y * inv_h), ifloor(z * inv_h));
        cells[key].push_back(i);
    }
#pragma omp parallel for num_threads(threads) schedule(dynamic, 256)
    for (int64_t i = 0; i < n; ++i) {
        const float px = xyz[3 * i], py = xyz[3 * i + 1], pz = xyz[3 * i + 2];
        const int ix = ifloor(px * inv_h), iy = ifloor(py * inv_h), iz = ifloor(pz * inv_h);
        long long cnt = 0, s1[3] = {0, 0, 0}, s2[6] = {0, 0, 0, 0, 0, 0};
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dz = -1; dz <= 1; ++dz) {
                    auto it = cells.find(key_ijk(ix + dx, iy + dy, iz + dz));
                    if (it == cells.end()) continue;
                    for (int64_t k : it->second) {
                        const float ex = xyz[3 * k] - px, ey = xyz[3 * k + 1] - py, ez = xyz[3 * k + 2] - pz;
                        if (ex * ex + ey * ey + ez * ez > r2) continue;
                        ++cnt;
                        s1[0] += llrintf(ex * fd);
                        s1[1] += llrintf(ey * fd);
                        s1[2] += llrintf(ez * fd);
                        s2[0] += llrintf(ex * ex * fdd);
                        s2[1] += llrintf(ex * ey * fdd);
                        s2[2] += llrintf(ex * ez * fdd);
                        s2[3] += llrintf(ey * ey * fdd);
                        s2[4] += llrintf(ey * ez * fdd);
                        s2[5] += llrintf(ez * ez * fdd);
                    }
                }
        if (cnt < 4) {
            out_nrm[3 * i] = out_nrm[3 * i + 1] = out_nrm[3 * i + 2] = 0.0f;
            out_pl[i] = 0.0f;
            continue;
        }
        const double inv = 1.0 / (double)cnt;
        const double mu[3] = {(double)s1[0] / fd64 * inv, (double)s1[1] / fd64 * inv, (double)s1[2] / fd64 * inv};
        const int up[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
        double C[9], ev[3], Q[9];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) C[r * 3 + c] = (double)s2[up[r * 3 + c]] / fdd64 * inv - mu[r] * mu[c];
        jacobi<3>(C, ev, Q);
        int lo = 0, hi = 0;  // prior_map.py:157-164
        for (int a = 1; a < 3; ++a) {
            if (ev[a] < ev[lo]) lo = a;
            if (ev[a] > ev[hi]) hi = a;
        }
        const int mid = lo == hi ? lo : 3 - lo - hi;
        double nx = Q[lo], ny = Q[3 + lo], nz = Q[6 + lo];
        const double nl = std::sqrt(nx * nx + ny * ny + nz * nz);
        if (nl > 0.0) {
            nx /= nl;
            ny /= nl;
            nz /= nl;
        }
        out_nrm[3 * i] = (float)nx;
        out_nrm[3 * i + 1] = (float)ny;
        out_nrm[3 * i + 2] = (float)nz;
        out_pl[i] = (float)((ev[mid] - ev[lo]) / std::max(ev[hi], 1.0e-12));
    }
}

}  // extern "C"
