// Prior-map grid and batched point-to-plane ICP for global localisation, on sm_100a.
//
// Reference: python/livox_warp/mapgrid.py -- Grid / grid_flat / grid_at / cell_centre :35-65, nearest_point :68-102,
// k_seed :105-114, k_unpack :117-125, k_jfa :128-158, k_df :161-170, PriorGrid.build :272-296;
// python/livox_warp/localize.py -- k_icp_batch :126-167, k_reduce_batch :170-179, k_eval_batch :182-205,
// GlobalLocalizer._icp :517-553, _evaluate :555-565.
//
// The grid build seeds each cell with a 64-bit key (distance in mm << 32 | point index) instead of the
// reference's 32-bit (mm << 23 | index), which held at most 2^23 - 1 map points, and floods between two
// buffers instead of in place, so the flood's result does not depend on thread timing.
//
// The batched ICP runs every hypothesis -- each with its own scan, of any length -- in one cooperative launch:
// tiles of one hypothesis' points accumulate float32 terms into float64 tile partials; after a grid barrier
// each hypothesis sums its tiles in a fixed order and solves its 6x6 system (Cholesky, float64); after a second
// barrier every CTA reads the largest step of the iteration and the schedule stage ends when it is below 2e-4
// (localize.py:536-552). The evaluation counts of localize.py:182-205 follow in the same launch.
#include <cmath>
#include <type_traits>

#include "lw_common.cuh"
#include "lw_linalg.cuh"

namespace lw {

// ---- grid geometry (mapgrid.py:35-65) --------------------------------------------------------------------
__device__ __forceinline__ int64_t grid_flat(const lw_prior_grid& g, int ix, int iy, int iz) {
    if (ix < 0 || iy < 0 || iz < 0 || ix >= g.nx || iy >= g.ny || iz >= g.nz) return -1;
    return ((int64_t)iz * g.ny + iy) * g.nx + ix;
}

__device__ __forceinline__ void grid_idx(const lw_prior_grid& g, float x, float y, float z, int& ix, int& iy, int& iz) {
    ix = ifloor((x - g.origin[0]) * g.inv_cell);
    iy = ifloor((y - g.origin[1]) * g.inv_cell);
    iz = ifloor((z - g.origin[2]) * g.inv_cell);
}

__device__ __forceinline__ void cell_centre(const lw_prior_grid& g, int64_t c, float& x, float& y, float& z) {
    int64_t ix = c % g.nx, r = c / g.nx;
    int64_t iy = r % g.ny, iz = r / g.ny;
    x = g.origin[0] + ((float)ix + 0.5f) * g.cell;
    y = g.origin[1] + ((float)iy + 0.5f) * g.cell;
    z = g.origin[2] + ((float)iz + 0.5f) * g.cell;
}

__device__ __forceinline__ float4 ld_pt(const float4* __restrict__ xyzp, int64_t i) { return __ldg(xyzp + i); }

constexpr float BOX_SLACK = 1.0e-4f;  // m: covers the float rounding of cell assignment and of the box offsets

// The map point nearest to w (mapgrid.py:68-102): exact within one cell -- the first point, in the reference's
// scan order (dz, dy, dx, then index), at the smallest distance below one cell -- otherwise the closest of the
// 27 cells' flooded seeds, or -1 beyond the band.
//
// Same result, fewer reads: the own cell is scanned first, and its smallest distance ub bounds the answer; a
// neighbour cell whose box lies farther than ub from w (less BOX_SLACK) holds no point that could be the first
// minimum, so its points are skipped. The seeds are still compared for every cell while nothing within one cell
// has been found, as the reference does. The own cell's contribution in the scan order is its own first minimum.
__device__ int nearest_point(const lw_prior_grid& g, float wx, float wy, float wz) {
    const float4* __restrict__ P = reinterpret_cast<const float4*>(g.xyz);
    int ix, iy, iz;
    grid_idx(g, wx, wy, wz, ix, iy, iz);
    const float cell2 = g.cell * g.cell;
    // w's offsets from its own cell's lower faces
    const float fx = (wx - g.origin[0]) - (float)ix * g.cell;
    const float fy = (wy - g.origin[1]) - (float)iy * g.cell;
    const float fz = (wz - g.origin[2]) - (float)iz * g.cell;
    int own = -1;
    float own_d2 = cell2;
    const int64_t c0 = grid_flat(g, ix, iy, iz);
    if (c0 >= 0) {
        const int k0 = __ldg(g.start + c0), k1 = __ldg(g.start + c0 + 1);
        for (int k = k0; k < k1; ++k) {
            const float4 q = ld_pt(P, k);
            const float ex = wx - q.x, ey = wy - q.y, ez = wz - q.z;
            const float d2 = ex * ex + ey * ey + ez * ez;
            if (d2 < own_d2) {
                own_d2 = d2;
                own = k;
            }
        }
    }
    const float ub = own_d2 * 1.00001f;
    int best = -1;
    float bd = cell2;
    int seed = -1;
    float sd = 1.0e30f;
    for (int dz = -1; dz <= 1; ++dz) {
        const float lz = fmaxf((dz < 0 ? fz : (dz > 0 ? g.cell - fz : 0.0f)) - BOX_SLACK, 0.0f);
        for (int dy = -1; dy <= 1; ++dy) {
            const float ly = fmaxf((dy < 0 ? fy : (dy > 0 ? g.cell - fy : 0.0f)) - BOX_SLACK, 0.0f);
            for (int dx = -1; dx <= 1; ++dx) {
                const int64_t c = grid_flat(g, ix + dx, iy + dy, iz + dz);
                if (c < 0) continue;
                if (dx == 0 && dy == 0 && dz == 0) {
                    if (own >= 0 && own_d2 < bd) {
                        bd = own_d2;
                        best = own;
                    }
                } else {
                    const float lx = fmaxf((dx < 0 ? fx : (dx > 0 ? g.cell - fx : 0.0f)) - BOX_SLACK, 0.0f);
                    if (lx * lx + ly * ly + lz * lz <= ub) {
                        const int k0 = __ldg(g.start + c), k1 = __ldg(g.start + c + 1);
                        for (int k = k0; k < k1; ++k) {
                            const float4 q = ld_pt(P, k);
                            const float ex = wx - q.x, ey = wy - q.y, ez = wz - q.z;
                            const float d2 = ex * ex + ey * ey + ez * ez;
                            if (d2 < bd) {
                                bd = d2;
                                best = k;
                            }
                        }
                    }
                }
                if (best < 0) {
                    const int s = __ldg(g.nn + c);
                    if (s >= 0) {
                        const float4 q = ld_pt(P, s);
                        const float ex = wx - q.x, ey = wy - q.y, ez = wz - q.z;
                        const float d2 = ex * ex + ey * ey + ez * ez;
                        if (d2 < sd) {
                            sd = d2;
                            seed = s;
                        }
                    }
                }
            }
        }
    }
    return best >= 0 ? best : seed;
}

// ---- grid build (mapgrid.py:105-170, 272-296) -------------------------------------------------------------
__global__ void k_seed_clear(lw_prior_grid g) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < g.ncell; c += (int64_t)gridDim.x * blockDim.x)
        g.seed[c] = ~0ULL;
}

__global__ void k_seed(lw_prior_grid g) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += (int64_t)gridDim.x * blockDim.x) {
        const float4 p = ld_pt(reinterpret_cast<const float4*>(g.xyz), i);
        int ix, iy, iz;
        grid_idx(g, p.x, p.y, p.z, ix, iy, iz);
        int64_t c = grid_flat(g, ix, iy, iz);
        if (c < 0) continue;
        float cx, cy, cz;
        cell_centre(g, c, cx, cy, cz);
        int dmm = (int)(len3(p.x - cx, p.y - cy, p.z - cz) * 1000.0f);
        if (dmm > 255) dmm = 255;
        atomicMin((unsigned long long*)(g.seed + c), ((unsigned long long)dmm << 32) | (unsigned long long)i);
    }
}

__global__ void k_unpack(lw_prior_grid g) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < g.ncell; c += (int64_t)gridDim.x * blockDim.x) {
        uint64_t v = g.seed[c];
        g.nn[c] = v == ~0ULL ? -1 : (int32_t)(v & 0xFFFFFFFFULL);
    }
}

// One flood step from `in` to `out`: the nearest of the seeds held `step` cells away in the 26 directions.
__global__ void k_jfa(lw_prior_grid g, const int32_t* __restrict__ in, int32_t* __restrict__ out, int step) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < g.ncell; c += (int64_t)gridDim.x * blockDim.x) {
        float px, py, pz;
        cell_centre(g, c, px, py, pz);
        int ix = (int)(c % g.nx), iy = (int)((c / g.nx) % g.ny), iz = (int)(c / ((int64_t)g.nx * g.ny));
        int best = in[c];
        float bd = 1.0e30f;
        if (best >= 0) {
            const float4 q = ld_pt(reinterpret_cast<const float4*>(g.xyz), best);
            float ex = px - q.x, ey = py - q.y, ez = pz - q.z;
            bd = ex * ex + ey * ey + ez * ez;
        }
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    int64_t j = grid_flat(g, ix + dx * step, iy + dy * step, iz + dz * step);
                    if (j < 0 || j == c) continue;
                    int s = in[j];
                    if (s < 0 || s == best) continue;
                    const float4 q = ld_pt(reinterpret_cast<const float4*>(g.xyz), s);
                    float ex = px - q.x, ey = py - q.y, ez = pz - q.z;
                    float d2 = ex * ex + ey * ey + ez * ez;
                    if (d2 < bd) {
                        bd = d2;
                        best = s;
                    }
                }
        out[c] = best;
    }
}

__global__ void k_df(lw_prior_grid g) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < g.ncell; c += (int64_t)gridDim.x * blockDim.x) {
        int s = g.nn[c];
        if (s < 0) {
            g.df[c] = 255;
            continue;
        }
        float px, py, pz;
        cell_centre(g, c, px, py, pz);
        const float4 q = ld_pt(reinterpret_cast<const float4*>(g.xyz), s);
        float d = len3(px - q.x, py - q.y, pz - q.z) * 100.0f;
        int v = (int)(d + 0.5f);
        g.df[c] = (uint8_t)(v < 255 ? v : 255);
    }
}

// Distance of each point (posed by T) to the nearest map point, 1e3 beyond the band (mapgrid.py:173-194).
struct Pose12 {
    float m[12];
};

__global__ void k_distances(lw_prior_grid g, const float* __restrict__ pts, int64_t n, Pose12 T, float* __restrict__ out) {
    const float* M = T.m;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float wx, wy, wz;
        xform(M, pts[3 * i], pts[3 * i + 1], pts[3 * i + 2], wx, wy, wz);
        int s = nearest_point(g, wx, wy, wz);
        float d = 1.0e3f;
        if (s >= 0) {
            const float4 q = ld_pt(reinterpret_cast<const float4*>(g.xyz), s);
            d = len3(wx - q.x, wy - q.y, wz - q.z);
        }
        out[i] = d;
    }
}

// ---- batched point-to-plane ICP (localize.py:126-205, 517-565) --------------------------------------------

constexpr int LTERMS = 30;  // H 21, b 6, count, err, weight
constexpr float PLANAR = 0.5f;  // mapgrid.py:32

struct LocPose {
    float R[9], tr[3], c[3];
};

// Per-hypothesis float pose, re-centred on the hypothesis' translation (float32 keeps its precision). The poses
// change between iterations of the same launch, so they are read through L2 (__ldcg), never the L1 cache.
__device__ __forceinline__ void loc_pose(const double* T, LocPose& P) {
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) P.R[i * 3 + j] = (float)__ldcg(T + i * 4 + j);
        const double t = __ldcg(T + i * 4 + 3);
        P.c[i] = (float)t;
        P.tr[i] = (float)(t - (double)P.c[i]);
    }
}

// The hypothesis and point range of a tile, checked against the batch: h = -1 for a tile to skip.
__device__ __forceinline__ void tile_range(const lw_loc_batch& b, int tile, int n_hyp, int& h, int& lo, int& hi) {
    h = __ldg(b.tile_hyp + tile);
    lo = __ldg(b.tile_lo + tile);
    if (h < 0 || h >= n_hyp || lo < 0) {
        h = -1;
        lo = hi = 0;
        return;
    }
    hi = (int)min((int64_t)__ldg(b.scan_end + h), b.pts_cap);
}

// One (hypothesis, point) pair's terms (localize.py:144-167) added to a[k * S], k < LTERMS (S = 1: registers;
// S = 32: a warp's per-lane columns in shared memory).
template <int S>
__device__ __forceinline__ void loc_terms(const lw_prior_grid& g, const LocPose& P, float4 p, float max_d2, float c2,
                                          float alpha, float* a) {
    float lx = P.R[0] * p.x + P.R[1] * p.y + P.R[2] * p.z + P.tr[0];
    float ly = P.R[3] * p.x + P.R[4] * p.y + P.R[5] * p.z + P.tr[1];
    float lz = P.R[6] * p.x + P.R[7] * p.y + P.R[8] * p.z + P.tr[2];
    float wx = lx + P.c[0], wy = ly + P.c[1], wz = lz + P.c[2];
    int s = nearest_point(g, wx, wy, wz);
    if (s < 0) return;
    const float4 q = ld_pt(reinterpret_cast<const float4*>(g.xyz), s);
    float r0 = wx - q.x, r1 = wy - q.y, r2 = wz - q.z;
    if (r0 * r0 + r1 * r1 + r2 * r2 > max_d2) return;
    const float3 nv = make_float3(__ldg(g.nrm + 3 * (int64_t)s), __ldg(g.nrm + 3 * (int64_t)s + 1),
                                  __ldg(g.nrm + 3 * (int64_t)s + 2));
    float M[6];
    if (q.w > PLANAR && len3(nv.x, nv.y, nv.z) > 0.5f) {
        // the normal at full weight, along the surface only a little
        float b = 1.0f - alpha;
        M[0] = nv.x * nv.x * b + alpha;
        M[1] = nv.x * nv.y * b;
        M[2] = nv.x * nv.z * b;
        M[3] = nv.y * nv.y * b + alpha;
        M[4] = nv.y * nv.z * b;
        M[5] = nv.z * nv.z * b + alpha;
    } else {
        // an edge or clutter: a weak point-to-point pull
        M[0] = M[3] = M[5] = alpha * 4.0f;
        M[1] = M[2] = M[4] = 0.0f;
    }
    float Mr0 = fmaf(M[0], r0, fmaf(M[1], r1, M[2] * r2));
    float Mr1 = fmaf(M[1], r0, fmaf(M[3], r1, M[4] * r2));
    float Mr2 = fmaf(M[2], r0, fmaf(M[4], r1, M[5] * r2));
    float d2 = fmaf(r0, Mr0, fmaf(r1, Mr1, r2 * Mr2));
    float wgt = 1.0f / (1.0f + d2 / c2);
    wgt = wgt * wgt;  // Geman-McClure
    // J = [I | A] with A = -[l]x, so H = w [[M, M A], [A^T M, A^T M A]] and b = w [M r; A^T M r]
    // (the upper triangle in row-major order, the layout of accumulate(), odom.py:244-259)
    const float A[3][3] = {{0.f, lz, -ly}, {-lz, 0.f, lx}, {ly, -lx, 0.f}};
    const float Ms[3][3] = {{M[0], M[1], M[2]}, {M[1], M[3], M[4]}, {M[2], M[4], M[5]}};
    float MA[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int j = 0; j < 3; ++j) MA[r][j] = fmaf(Ms[r][0], A[0][j], fmaf(Ms[r][1], A[1][j], Ms[r][2] * A[2][j]));
    int idx = 0;
#pragma unroll
    for (int pp = 0; pp < 6; ++pp)
#pragma unroll
        for (int qq = pp; qq < 6; ++qq) {
            float h;
            if (qq < 3)
                h = Ms[pp][qq];
            else if (pp < 3)
                h = MA[pp][qq - 3];
            else
                h = fmaf(A[0][pp - 3], MA[0][qq - 3], fmaf(A[1][pp - 3], MA[1][qq - 3], A[2][pp - 3] * MA[2][qq - 3]));
            a[idx * S] = fmaf(wgt, h, a[idx * S]);
            ++idx;
        }
    a[21 * S] = fmaf(wgt, Mr0, a[21 * S]);
    a[22 * S] = fmaf(wgt, Mr1, a[22 * S]);
    a[23 * S] = fmaf(wgt, Mr2, a[23 * S]);
#pragma unroll
    for (int j = 0; j < 3; ++j)
        a[(24 + j) * S] = fmaf(wgt, fmaf(A[0][j], Mr0, fmaf(A[1][j], Mr1, A[2][j] * Mr2)), a[(24 + j) * S]);
    a[27 * S] += 1.0f;
    a[28 * S] = fmaf(wgt, d2, a[28 * S]);
    a[29 * S] += wgt;
}

// The float64 step of hypothesis h from its summed terms sv (localize.py:537-550) applied to its pose; returns
// the step's size max(|dt|, 5 |dr|), 0 when it is skipped. Kept out of line: it runs on one thread per
// hypothesis per iteration, and inlined its arrays would set the register budget of the whole kernel.
__device__ __noinline__ double loc_solve(const double* sv, double* Th, int min_count) {
    double moved = 0.0;
    if (sv[27] >= (double)min_count) {
        // re-centred sums -> the twist about the world origin: H = A^T Hc A, b = A^T bc
        double c[3] = {(double)(float)__ldcg(Th + 3), (double)(float)__ldcg(Th + 7),
                       (double)(float)__ldcg(Th + 11)};
        double Hc[36], H[36], bc[6], bw[6];
        int idx = 0;
        for (int p = 0; p < 6; ++p)
            for (int q = p; q < 6; ++q) {
                Hc[p * 6 + q] = Hc[q * 6 + p] = sv[idx];
                ++idx;
            }
        for (int p = 0; p < 6; ++p) bc[p] = sv[21 + p];
        const double K[9] = {0.0, c[2], -c[1], -c[2], 0.0, c[0], c[1], -c[0], 0.0};
        double HA[36];
        for (int p = 0; p < 6; ++p)
            for (int q = 0; q < 6; ++q) {
                double x = Hc[p * 6 + q];
                if (q >= 3)
                    for (int k = 0; k < 3; ++k) x += Hc[p * 6 + k] * K[k * 3 + q - 3];
                HA[p * 6 + q] = x;
            }
        for (int p = 0; p < 6; ++p) {
            for (int q = 0; q < 6; ++q) {
                double x = HA[p * 6 + q];
                if (p >= 3)
                    for (int k = 0; k < 3; ++k) x += K[k * 3 + p - 3] * HA[k * 6 + q];
                H[p * 6 + q] = x;
            }
            double x = bc[p];
            if (p >= 3)
                for (int k = 0; k < 3; ++k) x += K[k * 3 + p - 3] * bc[k];
            bw[p] = x;
        }
        // A = H + diag(1e-3 dg + 1e-9), delta = solve(A, -b)
        double Lf[36], rhs[6], delta[6];
        for (int p = 0; p < 6; ++p) {
            H[p * 7] += 1e-3 * H[p * 7] + 1e-9;
            rhs[p] = -bw[p];
        }
        bool ok = true;
        for (int j = 0; j < 6 && ok; ++j) {
            double d = H[j * 6 + j];
            for (int k = 0; k < j; ++k) d -= Lf[j * 6 + k] * Lf[j * 6 + k];
            if (!(d > 0.0)) {
                ok = false;
                break;
            }
            d = sqrt(d);
            Lf[j * 6 + j] = d;
            for (int r = j + 1; r < 6; ++r) {
                double x = H[r * 6 + j];
                for (int k = 0; k < j; ++k) x -= Lf[r * 6 + k] * Lf[j * 6 + k];
                Lf[r * 6 + j] = x / d;
            }
        }
        if (ok) {
            double y[6];
            for (int r = 0; r < 6; ++r) {
                double s = rhs[r];
                for (int k = 0; k < r; ++k) s -= Lf[r * 6 + k] * y[k];
                y[r] = s / Lf[r * 6 + r];
            }
            for (int r = 5; r >= 0; --r) {
                double s = y[r];
                for (int k = r + 1; k < 6; ++k) s -= Lf[k * 6 + r] * delta[k];
                delta[r] = s / Lf[r * 6 + r];
            }
            double T[16];
            for (int k = 0; k < 16; ++k) T[k] = __ldcg(Th + k);
            apply_twist(T, delta);
            for (int k = 0; k < 16; ++k) Th[k] = T[k];
            double nt = sqrt(delta[0] * delta[0] + delta[1] * delta[1] + delta[2] * delta[2]);
            double nr = sqrt(delta[3] * delta[3] + delta[4] * delta[4] + delta[5] * delta[5]);
            moved = fmax(nt, 5.0 * nr);
        }
    }
    return moved;
}

struct LocArgs {
    int n_hyp, n_tiles, n_stages;  // counts, or capacities when b.dims is set
    int tile;                      // points per warp tile
    float max_d2[8], c2[8];
    int iters[8];
    float alpha;
    float radii[3];
    int min_count;  // a hypothesis with fewer matched points skips its update (localize.py:538)
};

constexpr int LOC_BLOCK = 256;
constexpr unsigned FULL = 0xffffffffu;

// Reduce-scatter over a warp: afterwards lane j holds the sum over the 32 lanes of v[j]. Each of the five steps
// hands half of the remaining slots to the partner lane (31 shuffles in all, against 5 per slot for 32 butterfly
// reductions).
__device__ __forceinline__ float warp_reduce_scatter32(float (&v)[32], int lane) {
#pragma unroll
    for (int half = 16; half >= 1; half >>= 1) {
        const bool up = (lane & half) != 0;
#pragma unroll
        for (int k = 0; k < half; ++k) {
            const float send = up ? v[k] : v[k + half];
            const float keep = up ? v[k + half] : v[k];
            v[k] = keep + __shfl_xor_sync(FULL, send, half);
        }
    }
    return v[0];
}

// The next tile of pass `pass` for the calling warp (one atomic per tile, broadcast to the warp).
__device__ __forceinline__ int next_tile(const lw_loc_batch& b, int pass, int lane) {
    int t = 0;
    if (lane == 0) t = atomicAdd(b.next + pass, 1);
    return __shfl_sync(FULL, t, 0);
}

// MINB: CTAs of LOC_BLOCK threads the register budget must let reside per SM. With 2 or 3 the per-lane term
// sums of a tile and the tile's pose live in registers; with 4 to 6 they live in shared memory (a [30][32]
// column block and one pose per warp, 31 KB per CTA), which frees ~47 registers across the nearest-point search
// so that two to three times the 2-CTA warp count stays resident.
template <int MINB>
__global__ void __launch_bounds__(LOC_BLOCK, MINB)
    k_loc_icp(lw_prior_grid g, lw_loc_batch b, LocArgs la) {
    constexpr bool SMEM_ACC = MINB >= 4;
    __shared__ float s_acc[SMEM_ACC ? LOC_BLOCK / 32 : 1][SMEM_ACC ? LTERMS : 1][32];
    __shared__ LocPose s_pose[SMEM_ACC ? LOC_BLOCK / 32 : 1];
    __shared__ double sv[32];
    __shared__ int s_stop;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int n_hyp = b.dims ? min(__ldg(b.dims), la.n_hyp) : la.n_hyp;
    const int n_tiles = b.dims ? min(__ldg(b.dims + 1), la.n_tiles) : la.n_tiles;
    int it_total = 0;
    for (int stage = 0; stage < la.n_stages; ++stage) {
        const float max_d2 = la.max_d2[stage];
        const float c2 = la.c2[stage];
        for (int it = 0; it < la.iters[stage]; ++it, ++it_total) {
            // phase A: warp tiles, handed out in order of arrival, -> float64 tile partials. A tile's partial
            // does not depend on which warp computed it, so the sums of phase B are deterministic.
            for (;;) {
                const int tile = next_tile(b, it_total, lane);
                if (tile >= n_tiles) break;
                int h, lo, hi;
                tile_range(b, tile, n_hyp, h, lo, hi);
                float v[32];
#pragma unroll
                for (int k = 0; k < 32; ++k) v[k] = 0.0f;
                if (h >= 0) {
                    // the tile's pose is the same for the whole warp: with SMEM_ACC it is kept in shared memory
                    // (broadcast reads) instead of 15 registers per lane
                    LocPose Pr;
                    LocPose& P = SMEM_ACC ? s_pose[tid >> 5] : Pr;
                    if (!SMEM_ACC || lane == 0) loc_pose(b.T + 16 * h, P);
                    __syncwarp();
                    const int end = min(hi, lo + la.tile);
                    if constexpr (SMEM_ACC) {
                        float* col = &s_acc[tid >> 5][0][lane];
#pragma unroll
                        for (int k = 0; k < LTERMS; ++k) col[k * 32] = 0.0f;
                        for (int i = lo + lane; i < end; i += 32)
                            loc_terms<32>(g, P, __ldg(reinterpret_cast<const float4*>(b.pts) + i), max_d2, c2,
                                          la.alpha, col);
#pragma unroll
                        for (int k = 0; k < LTERMS; ++k) v[k] = col[k * 32];
                        __syncwarp();  // the pose slot is rewritten by the warp's next tile
                    } else {
                        for (int i = lo + lane; i < end; i += 32)
                            loc_terms<1>(g, P, __ldg(reinterpret_cast<const float4*>(b.pts) + i), max_d2, c2,
                                         la.alpha, v);
                    }
                }
                const float sum = warp_reduce_scatter32(v, lane);
                if (lane < LTERMS) b.tile_part[(int64_t)tile * 32 + lane] = (double)sum;
            }
            if (!grid_barrier(b.bar, b.err, 1)) return;
            // phase B: per hypothesis, sum its tiles in order and solve (localize.py:537-550)
            for (int h = blockIdx.x; h < n_hyp; h += gridDim.x) {
                const int t0 = max(b.hyp_tile[h], 0), t1 = min(b.hyp_tile[h + 1], n_tiles);
                if (tid < LTERMS) {
                    double s = 0.0;
                    for (int t = t0; t < t1; ++t) s += __ldcg(b.tile_part + (int64_t)t * 32 + tid);
                    sv[tid] = s;
                }
                __syncthreads();
                if (tid == 0) {
                    b.count[h] = (int)sv[27];
                    const double moved = loc_solve(sv, b.T + 16 * h, la.min_count);
                    // the largest step of the iteration, as ordered bits of a non-negative float
                    atomicMax(b.moved + it_total, __float_as_int((float)moved));
                }
                __syncthreads();
            }
            if (!grid_barrier(b.bar, b.err, 2)) return;
            if (tid == 0) s_stop = __int_as_float(__ldcg(b.moved + it_total)) < 2e-4f ? 1 : 0;
            __syncthreads();
            if (s_stop) {
                ++it_total;
                break;
            }
        }
    }
    // evaluation (localize.py:182-205): points within each radius of their nearest map point, per hypothesis
    for (;;) {
        const int tile = next_tile(b, it_total, lane);
        if (tile >= n_tiles) break;
        int h, lo, hi;
        tile_range(b, tile, n_hyp, h, lo, hi);
        if (h < 0) continue;
        float M[12];
        for (int k = 0; k < 12; ++k) M[k] = (float)__ldcg(b.T + 16 * h + k);
        int c0 = 0, c1 = 0, c2 = 0;
        const int end = min(hi, lo + la.tile);
        for (int i = lo + lane; i < end; i += 32) {
            float4 p = __ldg(reinterpret_cast<const float4*>(b.pts) + i);
            float wx, wy, wz;
            xform(M, p.x, p.y, p.z, wx, wy, wz);
            int s = nearest_point(g, wx, wy, wz);
            if (s >= 0) {
                const float4 q = ld_pt(reinterpret_cast<const float4*>(g.xyz), s);
                float d = len3(wx - q.x, wy - q.y, wz - q.z);
                c0 += d < la.radii[0];
                c1 += d < la.radii[1];
                c2 += d < la.radii[2];
            }
        }
        c0 = __reduce_add_sync(FULL, c0);
        c1 = __reduce_add_sync(FULL, c1);
        c2 = __reduce_add_sync(FULL, c2);
        if (lane == 0) {
            atomicAdd(b.eval + 3 * h + 0, c0);
            atomicAdd(b.eval + 3 * h + 1, c1);
            atomicAdd(b.eval + 3 * h + 2, c2);
        }
    }
    if (blockIdx.x == 0 && tid == 0) *b.iters_run = it_total;
}

// Clears what the launch accumulates into. The barrier's arrival count is zeroed too: a launch that gave up at a
// barrier may have left it part counted (its generation word needs no reset).
__global__ void k_loc_reset(lw_loc_batch b, int n_hyp, int max_iters) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < max_iters; i += gridDim.x * blockDim.x) b.moved[i] = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= max_iters; i += gridDim.x * blockDim.x) b.next[i] = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 3 * n_hyp; i += gridDim.x * blockDim.x) b.eval[i] = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *b.err = 0;
        b.bar[0] = 0u;
    }
}

}  // namespace lw

using namespace lw;

namespace lw {

// ---- coarse hypothesis scores (localize.py:55-123, k_score_grid / k_score_list) -----------------------------
// A thread per hypothesis, the scan points staged in shared memory in chunks (every thread reads the same point at
// once). The soft count sum over points with d < tau of (1 - d^2 / tau^2) is kept as two integers -- the number of
// such points and the sum of d^2 (d is a whole number of cm) -- and formed once at the end in float64: exact and
// independent of the summation order, where the reference adds float32 terms in point order (the two differ by
// that sum's rounding only). Headings' cosine and sine come from the host (YawTab) so that every implementation
// poses the points with the same float32 values.
constexpr int SC_THREADS = 256;
constexpr int SC_CHUNK = 1024;

struct YawTab {
    float c[LW_SCORE_MAX_YAW], s[LW_SCORE_MAX_YAW];
};

__device__ __forceinline__ void score_chunk(const lw_prior_grid& g, const float* __restrict__ px,
                                            const float* __restrict__ py, const float* __restrict__ pz, int m,
                                            float cx, float cy, float cz, float co, float si, float tau, int& n_in,
                                            int& sum_d2) {
    const uint8_t* __restrict__ df = g.df;
#pragma unroll 4
    for (int k = 0; k < m; ++k) {
        const float wx = cx + co * px[k] - si * py[k];
        const float wy = cy + si * px[k] + co * py[k];
        const float wz = cz + pz[k];
        int ix, iy, iz;
        grid_idx(g, wx, wy, wz, ix, iy, iz);
        const int64_t j = grid_flat(g, ix, iy, iz);
        if (j >= 0) {
            const int d = __ldg(df + j);
            if ((float)d < tau) {
                ++n_in;
                sum_d2 += d * d;
            }
        }
    }
}

__device__ __forceinline__ void stage_pts(const float* __restrict__ pts, int base, int m, float* px, float* py,
                                          float* pz) {
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
        px[k] = pts[3 * (int64_t)(base + k) + 0];
        py[k] = pts[3 * (int64_t)(base + k) + 1];
        pz[k] = pts[3 * (int64_t)(base + k) + 2];
    }
}

__device__ __forceinline__ float soft_count(int n_in, int sum_d2, float tau) {
    return (float)((double)n_in - (double)sum_d2 / ((double)tau * (double)tau));
}

// Thread layout: each thread takes SC_POS consecutive rows of one column, positions ip = c + stride * r with
// r = SC_POS (32 rg + lane) + j, j < SC_POS, at one heading; the warps of a CTA take consecutive headings. When
// positions ip and ip + stride are neighbours along x with the same y and z (stride = ny for a meshgrid with y
// inner), a warp's posed copies of a point differ only in x -- one row of the x-fastest distance field, a few
// cache lines per gather -- and a thread's positions share the rotated offsets, the posed y and z, their cells and
// the row; only the x chain is per position (the kernel is issue-bound, so this removes most of its work). A
// thread whose positions straddle two (y, z) rows (the end of one x run and the start of the next) keeps a second
// row; one with more, or with rows that are not x runs, takes the general path. Each hypothesis' score is the
// same whatever the layout. Two positions per thread and six CTAs per SM: on the office coarse search (28M
// hypotheses x 1024 points) 34.2 ms, against 42.6 / 63.1 ms for four / eight positions at three CTAs per SM and
// 37.3 ms for one position (more resident warps keep more gathers in flight).
constexpr int SC_POS = 2;

template <bool WIDE>
__global__ void __launch_bounds__(SC_THREADS, 6) k_score_grid(lw_prior_grid g, const float* __restrict__ pts, int n_pts,
                                                           const float* __restrict__ pos, int64_t n_pos,
                                                           int64_t stride, int64_t n_rg, int n_yaw,
                                                           const YawTab yt, float tau, int tau_ceil, float free_cm,
                                                           float* __restrict__ out) {
    using idx_t = typename std::conditional<WIDE, int64_t, int32_t>::type;
    __shared__ float px[SC_CHUNK], py[SC_CHUNK], pz[SC_CHUNK];
    const int lane = threadIdx.x & 31;
    const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int iyaw = (int)(wid % n_yaw);
    const int64_t q = wid / n_yaw;
    const int64_t c = q / n_rg, r0 = ((q - c * n_rg) * 32 + lane) * SC_POS;
    const float co = yt.c[iyaw], si = yt.s[iyaw];
    float cx[SC_POS];
    bool live[SC_POS], in_b[SC_POS];
    float ya = 0.f, za = 0.f, yb = 0.f, zb = 0.f;
    int rows = 0;  // distinct (y, z) among the live positions: 0, 1, 2, or 3 for "more"
#pragma unroll
    for (int j = 0; j < SC_POS; ++j) {
        const int64_t ip = c + stride * (r0 + j);
        live[j] = c < stride && ip < n_pos;
        in_b[j] = false;
        cx[j] = 0.f;
        if (live[j]) {
            const float x = pos[3 * ip], y = pos[3 * ip + 1], z = pos[3 * ip + 2];
            int ix, iy, iz;
            grid_idx(g, x, y, z, ix, iy, iz);
            const int64_t cc = grid_flat(g, ix, iy, iz);
            // the sensor outside the grid or inside a mapped surface
            if (cc < 0 || (float)g.df[cc] < free_cm) {
                out[ip * n_yaw + iyaw] = -1.0f;
                live[j] = false;
            } else {
                cx[j] = x;
                if (rows == 0) {
                    ya = y;
                    za = z;
                    rows = 1;
                } else if (y != ya || z != za) {
                    if (rows == 1) {
                        yb = y;
                        zb = z;
                        rows = 2;
                    } else if (y != yb || z != zb) {
                        rows = 3;
                    }
                    in_b[j] = rows == 2 && y == yb && z == zb;
                }
            }
        }
    }
    int n_in[SC_POS], sum_d2[SC_POS];
#pragma unroll
    for (int j = 0; j < SC_POS; ++j) n_in[j] = sum_d2[j] = 0;
    const uint8_t* __restrict__ df = g.df;
    for (int base = 0; base < n_pts; base += SC_CHUNK) {
        const int m = min(SC_CHUNK, n_pts - base);
        __syncthreads();
        stage_pts(pts, base, m, px, py, pz);
        __syncthreads();
        if (rows == 0) continue;
        if (rows <= 2) {
#pragma unroll 2
            for (int k = 0; k < m; ++k) {
                // the reference's expressions (localize.py:89), the shared parts once per row
                const float ax = co * px[k], bx = si * py[k], ey = si * px[k], fy = co * py[k];
                const float wya = ya + ey + fy, wza = za + pz[k];
                const int iya = ifloor((wya - g.origin[1]) * g.inv_cell), iza = ifloor((wza - g.origin[2]) * g.inv_cell);
                const bool oka = iya >= 0 && iza >= 0 && iya < g.ny && iza < g.nz;
                const idx_t rowa = ((idx_t)iza * g.ny + iya) * (idx_t)g.nx;
                idx_t rowb = 0;
                bool okb = false;
                if (rows == 2) {
                    const float wyb = yb + ey + fy, wzb = zb + pz[k];
                    const int iyb = ifloor((wyb - g.origin[1]) * g.inv_cell), izb = ifloor((wzb - g.origin[2]) * g.inv_cell);
                    okb = iyb >= 0 && izb >= 0 && iyb < g.ny && izb < g.nz;
                    rowb = ((idx_t)izb * g.ny + iyb) * (idx_t)g.nx;
                }
#pragma unroll
                for (int j = 0; j < SC_POS; ++j) {
                    const float wx = cx[j] + ax - bx;
                    const int ix = ifloor((wx - g.origin[0]) * g.inv_cell);
                    const bool ok = in_b[j] ? okb : oka;
                    if (live[j] && ok && ix >= 0 && ix < g.nx) {
                        const int d = __ldg(df + (in_b[j] ? rowb : rowa) + ix);
                        if (d < tau_ceil) {  // d < tau for a whole number of cm
                            ++n_in[j];
                            sum_d2[j] += d * d;
                        }
                    }
                }
            }
        } else {
#pragma unroll
            for (int j = 0; j < SC_POS; ++j)
                if (live[j]) {
                    const int64_t ip = c + stride * (r0 + j);
                    score_chunk(g, px, py, pz, m, cx[j], pos[3 * ip + 1], pos[3 * ip + 2], co, si, tau, n_in[j],
                                sum_d2[j]);
                }
        }
    }
#pragma unroll
    for (int j = 0; j < SC_POS; ++j)
        if (live[j]) out[(c + stride * (r0 + j)) * n_yaw + iyaw] = soft_count(n_in[j], sum_d2[j], tau);
}

// Local maxima of the coarse scores (localize.py:450-483, _local_maxima): hypothesis h = ((iz nx + ix) ny + iy)
// n_yaw + iyaw is one when its score is positive, at least min_score, and no less than any of its 26 neighbours in
// (x, y, heading) at its height -- neighbours outside the x / y range are skipped, headings wrap. Survivors are
// appended (index, score) in no particular order; the caller orders them.
__global__ void k_score_maxima(const float* __restrict__ sc, int nz, int nx, int ny, int n_yaw, float min_score,
                               int cap, int64_t* __restrict__ idx, float* __restrict__ val, int* __restrict__ count) {
    const int64_t n = (int64_t)nz * nx * ny * n_yaw;
    for (int64_t h = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; h < n; h += (int64_t)gridDim.x * blockDim.x) {
        const float mine = sc[h];
        if (!(mine > 0.0f) || mine < min_score) continue;
        const int iyaw = (int)(h % n_yaw);
        const int64_t p = h / n_yaw;
        const int iy = (int)(p % ny);
        const int ix = (int)((p / ny) % nx);
        const int64_t base = p - (int64_t)iy - (int64_t)ix * ny;  // iz's first position
        bool best = true;
        for (int ox = -1; ox <= 1 && best; ++ox) {
            const int jx = ix + ox;
            if (jx < 0 || jx >= nx) continue;
            for (int oy = -1; oy <= 1 && best; ++oy) {
                const int jy = iy + oy;
                if (jy < 0 || jy >= ny) continue;
                const int64_t q = (base + (int64_t)jx * ny + jy) * n_yaw;
                for (int oa = -1; oa <= 1; ++oa) {
                    if (ox == 0 && oy == 0 && oa == 0) continue;
                    const int ja = (iyaw + oa + n_yaw) % n_yaw;
                    if (__ldg(sc + q + ja) > mine) {
                        best = false;
                        break;
                    }
                }
            }
        }
        if (!best) continue;
        const int k = atomicAdd(count, 1);
        if (k < cap) {
            idx[k] = h;
            val[k] = mine;
        }
    }
}

__global__ void __launch_bounds__(SC_THREADS) k_score_list(lw_prior_grid g, const float* __restrict__ pts, int n_pts,
                                                           const float4* __restrict__ hyp, int64_t n_hyp, float tau,
                                                           float* __restrict__ out) {
    __shared__ float px[SC_CHUNK], py[SC_CHUNK], pz[SC_CHUNK];
    const int64_t h = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = h < n_hyp;
    float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
    float co = 1.f, si = 0.f;
    if (live) {
        q = hyp[h];
        // cos / sin in float64, rounded once: the heading as the host would pose it
        co = (float)cos((double)q.w);
        si = (float)sin((double)q.w);
    }
    int n_in = 0, sum_d2 = 0;
    for (int base = 0; base < n_pts; base += SC_CHUNK) {
        const int m = min(SC_CHUNK, n_pts - base);
        __syncthreads();
        stage_pts(pts, base, m, px, py, pz);
        __syncthreads();
        if (live) score_chunk(g, px, py, pz, m, q.x, q.y, q.z, co, si, tau, n_in, sum_d2);
    }
    if (live) out[h] = soft_count(n_in, sum_d2, tau);
}

}  // namespace lw

static int check_grid(const lw_prior_grid* g, const char* who) {
    if (!g || !g->xyz || !g->start || !g->nn || g->nx <= 0 || g->ny <= 0 || g->nz <= 0 || g->cell <= 0.0f)
        return set_error(LW_EINVAL, "%s: incomplete prior grid", who);
    if ((int64_t)g->nx * g->ny * g->nz != g->ncell) return set_error(LW_EINVAL, "%s: ncell != nx*ny*nz", who);
    if (((uintptr_t)g->xyz & 15) != 0) return set_error(LW_EINVAL, "%s: xyz must be 16-byte aligned", who);
    if (g->n >= 0x7FFFFFFF) return set_error(LW_ECAPACITY, "%s: %lld map points exceed int32 indices", who, (long long)g->n);
    return LW_OK;
}

extern "C" {

int lw_prior_grid_build(lw_prior_grid* g, void* stream) {
    int r = check_grid(g, "lw_prior_grid_build");
    if (r != LW_OK) return r;
    if (!g->seed || !g->nn2 || !g->df) return set_error(LW_EINVAL, "lw_prior_grid_build: missing build scratch");
    cudaStream_t s = (cudaStream_t)stream;
    int gc = blocks_for(g->ncell, 256, 16 * device_sms());
    int gp = blocks_for(g->n, 256, 16 * device_sms());
    ProfScope prof("grid_build", s);
    k_seed_clear<<<gc, 256, 0, s>>>(*g);
    k_seed<<<gp, 256, 0, s>>>(*g);
    k_unpack<<<gc, 256, 0, s>>>(*g);
    const int steps[5] = {8, 4, 2, 1, 1};  // mapgrid.py:31
    int32_t* a = g->nn;
    int32_t* bbuf = g->nn2;
    for (int k = 0; k < 5; ++k) {
        k_jfa<<<gc, 256, 0, s>>>(*g, a, bbuf, steps[k]);
        int32_t* t = a;
        a = bbuf;
        bbuf = t;
    }
    if (a != g->nn) LW_CUDA(cudaMemcpyAsync(g->nn, a, g->ncell * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
    k_df<<<gc, 256, 0, s>>>(*g);
    LW_LAUNCHED("lw_prior_grid_build");
    count_launches(9);
    return LW_OK;
}

int lw_prior_distances(const lw_prior_grid* g, const float* pts, int64_t n, const double* T_host, float* out,
                       void* stream) {
    int r = check_grid(g, "lw_prior_distances");
    if (r != LW_OK) return r;
    if (!pts || !T_host || !out) return set_error(LW_EINVAL, "lw_prior_distances: null argument");
    if (n <= 0) return LW_OK;
    Pose12 T;
    for (int k = 0; k < 12; ++k) T.m[k] = (float)T_host[k];
    k_distances<<<blocks_for(n, 256, 16 * device_sms()), 256, 0, (cudaStream_t)stream>>>(*g, pts, n, T, out);
    LW_LAUNCHED("lw_prior_distances");
    count_launches(1);
    return LW_OK;
}

int lw_score_grid(const lw_prior_grid* g, const float* pts, int32_t n_pts, const float* pos, int64_t n_pos,
                  int64_t pos_stride, int32_t n_yaw, float yaw0, float dyaw, float tau_cm, float free_cm, float* out,
                  void* stream) {
    int r = check_grid(g, "lw_score_grid");
    if (r != LW_OK) return r;
    if (!g->df || n_pts < 0 || n_pos < 0 || (n_pts > 0 && !pts) || (n_pos > 0 && (!pos || !out)))
        return set_error(LW_EINVAL, "lw_score_grid: bad arguments");
    if (n_yaw < 1 || n_yaw > LW_SCORE_MAX_YAW)
        return set_error(LW_EINVAL, "lw_score_grid: n_yaw %d outside [1, %d]", n_yaw, LW_SCORE_MAX_YAW);
    if (!(tau_cm > 0.0f)) return set_error(LW_EINVAL, "lw_score_grid: tau_cm must be positive");
    if ((int64_t)n_pts * 255 * 255 > 0x7FFFFFFF)
        return set_error(LW_ECAPACITY, "lw_score_grid: %d points overflow the int32 sums", n_pts);
    if (pos_stride < 1) return set_error(LW_EINVAL, "lw_score_grid: pos_stride must be >= 1");
    if (n_pos == 0) return LW_OK;
    const int64_t stride = pos_stride < n_pos ? pos_stride : n_pos;
    const int64_t n_rg = ((n_pos + stride - 1) / stride + 32 * SC_POS - 1) / (32 * SC_POS);  // per column
    const int64_t threads = stride * n_rg * (int64_t)n_yaw * 32;
    YawTab yt;
    lw_score_yaw_table(n_yaw, yaw0, dyaw, yt.c, yt.s);
    const int tau_ceil = tau_cm > 1024.0f ? 1024 : (int)ceilf(tau_cm);  // distances are whole cm in [0, 255]
    const unsigned blocks = (unsigned)((threads + SC_THREADS - 1) / SC_THREADS);
    if (g->ncell < 0x7FFFFFFF)
        k_score_grid<false><<<blocks, SC_THREADS, 0, (cudaStream_t)stream>>>(*g, pts, n_pts, pos, n_pos, stride, n_rg,
                                                                              n_yaw, yt, tau_cm, tau_ceil, free_cm, out);
    else
        k_score_grid<true><<<blocks, SC_THREADS, 0, (cudaStream_t)stream>>>(*g, pts, n_pts, pos, n_pos, stride, n_rg,
                                                                             n_yaw, yt, tau_cm, tau_ceil, free_cm, out);
    LW_LAUNCHED("lw_score_grid");
    count_launches(1);
    return LW_OK;
}

int lw_score_list(const lw_prior_grid* g, const float* pts, int32_t n_pts, const float* hyp, int64_t n_hyp,
                  float tau_cm, float* out, void* stream) {
    int r = check_grid(g, "lw_score_list");
    if (r != LW_OK) return r;
    if (!g->df || n_pts < 0 || n_hyp < 0 || (n_pts > 0 && !pts) || (n_hyp > 0 && (!hyp || !out)))
        return set_error(LW_EINVAL, "lw_score_list: bad arguments");
    if (((uintptr_t)hyp & 15) != 0) return set_error(LW_EINVAL, "lw_score_list: hyp must be 16-byte aligned");
    if (!(tau_cm > 0.0f)) return set_error(LW_EINVAL, "lw_score_list: tau_cm must be positive");
    if ((int64_t)n_pts * 255 * 255 > 0x7FFFFFFF)
        return set_error(LW_ECAPACITY, "lw_score_list: %d points overflow the int32 sums", n_pts);
    if (n_hyp == 0) return LW_OK;
    k_score_list<<<(unsigned)((n_hyp + SC_THREADS - 1) / SC_THREADS), SC_THREADS, 0, (cudaStream_t)stream>>>(
        *g, pts, n_pts, reinterpret_cast<const float4*>(hyp), n_hyp, tau_cm, out);
    LW_LAUNCHED("lw_score_list");
    count_launches(1);
    return LW_OK;
}

int lw_score_maxima(const float* scores, int32_t nz, int32_t nx, int32_t ny, int32_t n_yaw, float min_score,
                    int32_t cap, int64_t* idx, float* val, int32_t* count_dev, void* stream) {
    if (!scores || !idx || !val || !count_dev || nz < 0 || nx < 0 || ny < 0 || n_yaw < 1 || cap < 0)
        return set_error(LW_EINVAL, "lw_score_maxima: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaMemsetAsync(count_dev, 0, sizeof(int32_t), s) != cudaSuccess)
        return set_error(LW_ECUDA, "lw_score_maxima: clearing the count failed");
    const int64_t n = (int64_t)nz * nx * ny * n_yaw;
    if (n == 0) return LW_OK;
    k_score_maxima<<<blocks_for(n, 256, 16 * device_sms()), 256, 0, s>>>(scores, nz, nx, ny, n_yaw, min_score, cap,
                                                                        idx, val, count_dev);
    LW_LAUNCHED("lw_score_maxima");
    count_launches(1);
    return LW_OK;
}

void lw_score_yaw_table(int32_t n_yaw, float yaw0, float dyaw, float* c, float* s) {
    for (int j = 0; j < n_yaw; ++j) {
        const float yaw = yaw0 + (float)j * dyaw;  // float32, as localize.py:82
        c[j] = (float)std::cos((double)yaw);
        s[j] = (float)std::sin((double)yaw);
    }
}

int lw_loc_icp_batch(const lw_prior_grid* g, lw_loc_batch* b, int32_t n_hyp, int32_t n_tiles, int32_t tile,
                     int32_t n_stages, const double* dmax, const int32_t* iters, float alpha, int32_t min_count,
                     int32_t blocks_per_sm, int32_t grid, void* stream) {
    int r = check_grid(g, "lw_loc_icp_batch");
    if (r != LW_OK) return r;
    if (!b || (n_stages > 0 && (!dmax || !iters)) || n_stages < 0 || n_stages > 8 || n_hyp < 1 || n_tiles < 1)
        return set_error(LW_EINVAL, "lw_loc_icp_batch: bad arguments");
    if (!b->pts || !b->scan_end || !b->tile_hyp || !b->tile_lo || !b->hyp_tile || !b->T || !b->tile_part ||
        !b->moved || !b->next || !b->count || !b->eval || !b->bar || !b->err || !b->iters_run || b->pts_cap < 0)
        return set_error(LW_EINVAL, "lw_loc_icp_batch: incomplete batch buffers");
    if (tile < 32 || tile > 2048 || tile % 32 != 0)
        return set_error(LW_EINVAL, "lw_loc_icp_batch: tile must be a multiple of 32 in [32, 2048]");
    if (!g->nrm) return set_error(LW_EINVAL, "lw_loc_icp_batch: the grid needs normals");
    LocArgs la{};
    la.n_hyp = n_hyp;
    la.n_tiles = n_tiles;
    la.n_stages = n_stages;
    la.tile = tile;
    int total_iters = 0;
    for (int k = 0; k < n_stages; ++k) {
        if (iters[k] < 0 || !(dmax[k] > 0.0)) return set_error(LW_EINVAL, "lw_loc_icp_batch: stage %d", k);
        la.max_d2[k] = (float)(dmax[k] * dmax[k]);  // localize.py:541: dmax * dmax
        const double half = dmax[k] * 0.5;
        la.c2[k] = (float)(half * half);  // localize.py:530: (dmax * 0.5) ** 2
        la.iters[k] = iters[k];
        total_iters += iters[k];
    }
    if (total_iters > b->moved_cap) return set_error(LW_ECAPACITY, "lw_loc_icp_batch: %d iterations > moved_cap", total_iters);
    la.alpha = alpha;
    la.radii[0] = 0.03f;  // EVAL_RADII (localize.py:47)
    la.radii[1] = 0.05f;
    la.radii[2] = 0.10f;
    la.min_count = min_count;
    cudaStream_t s = (cudaStream_t)stream;
    int sms = device_sms();
    if (blocks_per_sm == 0) blocks_per_sm = 3;
    if (blocks_per_sm < 2 || blocks_per_sm > 6)
        return set_error(LW_EINVAL, "lw_loc_icp_batch: blocks_per_sm must be 0 or 2..6");
    const void* fn = blocks_per_sm == 2   ? (const void*)k_loc_icp<2>
                     : blocks_per_sm == 3 ? (const void*)k_loc_icp<3>
                     : blocks_per_sm == 4 ? (const void*)k_loc_icp<4>
                     : blocks_per_sm == 5 ? (const void*)k_loc_icp<5>
                                          : (const void*)k_loc_icp<6>;
    int per_sm = 0;
    LW_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, LOC_BLOCK, 0));
    if (per_sm < 1) return set_error(LW_EINVAL, "lw_loc_icp_batch: the kernel does not fit on an SM");
    int max_grid = per_sm * sms;
    if (grid <= 0 || grid > max_grid) grid = max_grid;
    if (grid > b->grid_cap) grid = b->grid_cap;
    ProfScope prof("loc_icp", s);
    k_loc_reset<<<16, 256, 0, s>>>(*b, n_hyp, total_iters);
    // a cooperative launch (every CTA resident: the grid barriers rely on it), made through cudaLaunchKernelEx
    // so that it can also be captured into a CUDA graph
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(LOC_BLOCK);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    switch (blocks_per_sm) {
        case 2: LW_CUDA(cudaLaunchKernelEx(&cfg, k_loc_icp<2>, *g, *b, la)); break;
        case 3: LW_CUDA(cudaLaunchKernelEx(&cfg, k_loc_icp<3>, *g, *b, la)); break;
        case 4: LW_CUDA(cudaLaunchKernelEx(&cfg, k_loc_icp<4>, *g, *b, la)); break;
        case 5: LW_CUDA(cudaLaunchKernelEx(&cfg, k_loc_icp<5>, *g, *b, la)); break;
        default: LW_CUDA(cudaLaunchKernelEx(&cfg, k_loc_icp<6>, *g, *b, la)); break;
    }
    LW_LAUNCHED("lw_loc_icp_batch");
    count_launches(2);
    return LW_OK;
}

}  // extern "C"
