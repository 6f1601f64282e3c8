// Neighbourhood summaries of the visible points on sm_100a: a weighted neighbour count, a PCA normal and the
// curvature per point, from a voxel summary a third of the radius wide.
//
// Reference: python/livox_warp/gpu.py -- k_nb_insert :781-800, k_nb_flag / k_nb_compact :803-826, k_nb_voxel
// :829-876, k_nb_gather :879-904, Pipeline.neighborhoods :1531-1557.
//
// Determinism: the reference adds float coordinates into its voxels with float atomics and sums each voxel's
// neighbours in the order a hash-grid query returns them, so its answers depend on thread timing. Here the voxel
// sums are int64 fixed point (exact), the neighbours of a voxel are the voxels whose centroid lies within the radius
// -- found by probing the 7 x 7 x 7 voxel offsets that can hold one (a centroid lies inside its voxel, so with
// voxels radius / 3 wide no farther voxel qualifies) -- and their weighted offsets and outer products are summed as
// int64 fixed point too; the covariance and its eigen-decomposition are float64. Every point's count, normal and
// curvature is then independent of thread order and of where keys land in the table.
#include "lw_common.cuh"
#include "lw_linalg.cuh"

namespace lw {

constexpr double NB_FIX_D = 1048576.0;         // units per metre of a neighbour offset (2^20)
constexpr double NB_FIX_DD = 1099511627776.0;  // units per m^2 of an offset product (2^40)
constexpr int NB_REACH = 3;                    // voxel offsets probed per axis: radius / (radius / 3)
constexpr int NB_TILE = 1024;

struct NbArgs {
    float inv_h, r2;
    int mask, want_normals;
    double sensor[3];
};

template <int STRIDE>
__device__ __forceinline__ void nb_ld(const float* __restrict__ xyz, int64_t i, float& x, float& y, float& z) {
    x = xyz[STRIDE * i];
    y = xyz[STRIDE * i + 1];
    z = xyz[STRIDE * i + 2];
}

// Each point claims its voxel (key of floor(w * inv_h), gpu.py:243) and adds its coordinates in fixed point.
template <int STRIDE>
__global__ void k_nb_insert(const float* __restrict__ xyz, const int* n_dev, int64_t n_ub, NbArgs a, lw_nbr_buf nb) {
    int64_t n = n_dev ? (int64_t)*n_dev : n_ub;
    if (n > n_ub) n = n_ub;
    const float FW = (float)LW_FIX_W;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float x, y, z;
        nb_ld<STRIDE>(xyz, i, x, y, z);
        const int64_t key = key_ijk(ifloor(x * a.inv_h), ifloor(y * a.inv_h), ifloor(z * a.inv_h));
        bool claimed;
        const int s = claim_slot(key, nb.keys, a.mask, &claimed);
        if (s >= 0) {
            atomic_add_i64(nb.acc + 4 * (int64_t)s + 0, to_fix(x, FW));
            atomic_add_i64(nb.acc + 4 * (int64_t)s + 1, to_fix(y, FW));
            atomic_add_i64(nb.acc + 4 * (int64_t)s + 2, to_fix(z, FW));
            atomic_add_i64(nb.acc + 4 * (int64_t)s + 3, 1);
        }
        nb.slot_of_pt[i] = s;
    }
}

// Occupied slots per tile, then (one CTA) their exclusive scan; the voxels are numbered in slot order.
__global__ void k_nb_count(lw_nbr_buf nb) {
    const int64_t s = (int64_t)blockIdx.x * NB_TILE + threadIdx.x;
    const int f = (s < nb.cap && nb.keys[s] != EMPTY_KEY) ? 1 : 0;
    const int c = __syncthreads_count(f);
    if (threadIdx.x == 0) nb.tiles[blockIdx.x] = c;
}

__global__ void k_nb_scan(lw_nbr_buf nb, int nt) {
    __shared__ int sm[33];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < nt; base += blockDim.x) {
        const int j = base + threadIdx.x;
        const int v = j < nt ? nb.tiles[j] : 0;
        // exclusive prefix of the counts across the CTA: warp scan + warp totals
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        int inc = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += u;
        }
        if (lane == 31) sm[w] = inc;
        __syncthreads();
        if (w == 0) {
            const int nw = blockDim.x >> 5;
            const int x = lane < nw ? sm[lane] : 0;
            int xi = x;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, xi, o);
                if (lane >= o) xi += u;
            }
            if (lane < nw) sm[lane] = xi - x;
            if (lane == 31) sm[32] = xi;
        }
        __syncthreads();
        if (j < nt) nb.tiles[j] = carry + sm[w] + inc - v;
        __syncthreads();
        if (threadIdx.x == 0) carry += sm[32];
        __syncthreads();
    }
    if (threadIdx.x == 0) *nb.m = carry;
}

__global__ void k_nb_scatter(lw_nbr_buf nb) {
    __shared__ int sm[33];
    const int64_t s = (int64_t)blockIdx.x * NB_TILE + threadIdx.x;
    const int f = (s < nb.cap && nb.keys[s] != EMPTY_KEY) ? 1 : 0;
    int tot;
    const int r = block_rank(f, sm, &tot);
    if (!f) return;
    const int j = nb.tiles[blockIdx.x] + r;
    nb.vidx[s] = j;
    nb.v_slot[j] = (int)s;
    const int64_t* acc = nb.acc + 4 * s;
    const double w = (double)acc[3];
    // the voxel's mean, exact from the fixed-point sums (the reference divides float sums, gpu.py:823)
    nb.v_xyz[3 * (int64_t)j + 0] = (float)((double)acc[0] / (w * LW_FIX_W));
    nb.v_xyz[3 * (int64_t)j + 1] = (float)((double)acc[1] / (w * LW_FIX_W));
    nb.v_xyz[3 * (int64_t)j + 2] = (float)((double)acc[2] / (w * LW_FIX_W));
    nb.v_w[j] = (int)acc[3];
}

__device__ __forceinline__ long long warp_sum_ll(long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// A warp per voxel (gpu.py:829-876): its lanes probe the 343 voxel offsets 32 at a time; every voxel whose centroid
// lies within the radius adds its points' weight, weighted offset and weighted outer product in fixed point. Lane 0
// forms the count, and with want_normals the covariance's smallest-eigenvalue vector turned toward the sensor and
// the curvature (smallest eigenvalue / trace).
__global__ void k_nb_voxel(NbArgs a, lw_nbr_buf nb) {
    const int m = *nb.m;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    constexpr int S = 2 * NB_REACH + 1, N = S * S * S;
    for (int j = warp; j < m; j += nwarps) {
        const float px = nb.v_xyz[3 * (int64_t)j], py = nb.v_xyz[3 * (int64_t)j + 1], pz = nb.v_xyz[3 * (int64_t)j + 2];
        const int64_t key = nb.keys[nb.v_slot[j]];
        const int ix = (int)(key & KEY_MASK) - (int)KEY_BIAS;
        const int iy = (int)((key >> 21) & KEY_MASK) - (int)KEY_BIAS;
        const int iz = (int)((key >> 42) & KEY_MASK) - (int)KEY_BIAS;
        long long W = 0, s1[3] = {0, 0, 0}, s2[6] = {0, 0, 0, 0, 0, 0};
        for (int o0 = 0; o0 < N; o0 += 32) {
            const int o = o0 + lane;
            if (o >= N) continue;
            const int dz = o % S - NB_REACH, dy = (o / S) % S - NB_REACH, dx = o / (S * S) - NB_REACH;
            const int s = find_slot(key_ijk(ix + dx, iy + dy, iz + dz), nb.keys, a.mask);
            if (s < 0) continue;
            const int k = nb.vidx[s];
            const float ex = nb.v_xyz[3 * (int64_t)k] - px, ey = nb.v_xyz[3 * (int64_t)k + 1] - py,
                        ez = nb.v_xyz[3 * (int64_t)k + 2] - pz;
            if (ex * ex + ey * ey + ez * ez > a.r2) continue;
            const long long w = nb.v_w[k];
            const float FD = (float)NB_FIX_D, FDD = (float)NB_FIX_DD;
            W += w;
            s1[0] += w * to_fix(ex, FD);
            s1[1] += w * to_fix(ey, FD);
            s1[2] += w * to_fix(ez, FD);
            s2[0] += w * to_fix(ex * ex, FDD);
            s2[1] += w * to_fix(ex * ey, FDD);
            s2[2] += w * to_fix(ex * ez, FDD);
            s2[3] += w * to_fix(ey * ey, FDD);
            s2[4] += w * to_fix(ey * ez, FDD);
            s2[5] += w * to_fix(ez * ez, FDD);
        }
        W = warp_sum_ll(W);
#pragma unroll
        for (int c = 0; c < 3; ++c) s1[c] = warp_sum_ll(s1[c]);
#pragma unroll
        for (int c = 0; c < 6; ++c) s2[c] = warp_sum_ll(s2[c]);
        if (lane != 0) continue;
        nb.v_cnt[j] = (float)W;
        if (a.want_normals == 0) continue;
        // toward the sensor, in float64 from the float coordinates
        double tx = a.sensor[0] - (double)px, ty = a.sensor[1] - (double)py, tz = a.sensor[2] - (double)pz;
        const double tl = sqrt(tx * tx + ty * ty + tz * tz);
        if (tl > 0.0) {
            tx /= tl;
            ty /= tl;
            tz /= tl;
        }
        const double inv = 1.0 / fmax((double)W, 1.0);
        const double mu[3] = {(double)s1[0] / NB_FIX_D * inv, (double)s1[1] / NB_FIX_D * inv,
                              (double)s1[2] / NB_FIX_D * inv};
        const int up[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
        double C[9], ev[3], Q[9];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) C[r * 3 + c] = (double)s2[up[r * 3 + c]] / NB_FIX_DD * inv - mu[r] * mu[c];
        jacobi_eig<3>(C, ev, Q);
        int kmin = 0;
        if (ev[1] < ev[kmin]) kmin = 1;
        if (ev[2] < ev[kmin]) kmin = 2;
        double nx = Q[0 * 3 + kmin], ny = Q[1 * 3 + kmin], nz = Q[2 * 3 + kmin];
        const double nl = sqrt(nx * nx + ny * ny + nz * nz);
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
        if (tr <= 1.0e-12) {  // a lone voxel: no surface to fit
            nx = tx;
            ny = ty;
            nz = tz;
        }
        nb.v_nrm[3 * (int64_t)j + 0] = (float)nx;
        nb.v_nrm[3 * (int64_t)j + 1] = (float)ny;
        nb.v_nrm[3 * (int64_t)j + 2] = (float)nz;
        nb.v_curv[j] = (float)(fmax(ev[kmin], 0.0) / fmax(tr, 1.0e-12));
    }
}

// Each point takes its voxel's answers (gpu.py:879-904); a point whose voxel did not fit in the table reads as
// crowded (count 2^30), flat and facing up, so nothing hides it.
__global__ void k_nb_gather(const int* n_dev, int64_t n_ub, int want_normals, lw_nbr_buf nb, int32_t* __restrict__ cnt,
                            float* __restrict__ nrm, float* __restrict__ curv) {
    int64_t n = n_dev ? (int64_t)*n_dev : n_ub;
    if (n > n_ub) n = n_ub;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int s = nb.slot_of_pt[i];
        if (s < 0) {
            cnt[i] = 1 << 30;
            if (want_normals) {
                nrm[3 * i] = 0.0f;
                nrm[3 * i + 1] = 0.0f;
                nrm[3 * i + 2] = 1.0f;
                curv[i] = 0.0f;
            }
            continue;
        }
        const int v = nb.vidx[s];
        cnt[i] = (int)(nb.v_cnt[v] + 0.5f);
        if (want_normals) {
            nrm[3 * i] = nb.v_nrm[3 * (int64_t)v];
            nrm[3 * i + 1] = nb.v_nrm[3 * (int64_t)v + 1];
            nrm[3 * i + 2] = nb.v_nrm[3 * (int64_t)v + 2];
            curv[i] = nb.v_curv[v];
        }
    }
}

}  // namespace lw

using namespace lw;

extern "C" {

int lw_neighborhoods(const float* xyz, int32_t xyz_stride, const int32_t* n_dev, int64_t n_ub, float radius,
                     int32_t want_normals, const float* sensor, lw_nbr_buf* nb, int32_t* out_cnt, float* out_nrm,
                     float* out_curv, void* stream) {
    if (!nb || !nb->keys || !nb->acc || !nb->vidx || !nb->v_slot || !nb->slot_of_pt || !nb->v_xyz || !nb->v_w ||
        !nb->v_cnt || !nb->v_nrm || !nb->v_curv || !nb->tiles || !nb->m)
        return set_error(LW_EINVAL, "lw_neighborhoods: incomplete buffers");
    if ((nb->cap & (nb->cap - 1)) != 0 || nb->cap <= 0 || nb->cap > (1LL << 30))
        return set_error(LW_EINVAL, "lw_neighborhoods: table capacity must be a power of two");
    if (!(radius > 0.0f) || radius > 4.0f)
        return set_error(LW_EINVAL, "lw_neighborhoods: radius %g outside (0, 4] m", (double)radius);
    if ((xyz_stride != 3 && xyz_stride != 4) || (n_ub > 0 && (!xyz || !out_cnt)) ||
        (want_normals && n_ub > 0 && (!out_nrm || !out_curv || !sensor)))
        return set_error(LW_EINVAL, "lw_neighborhoods: bad arguments");
    if (n_ub > nb->pt_cap)
        return set_error(LW_ECAPACITY, "lw_neighborhoods: %lld points exceed the buffers' %lld", (long long)n_ub,
                         (long long)nb->pt_cap);
    cudaStream_t s = (cudaStream_t)stream;
    NbArgs a{};
    a.inv_h = 3.0f / radius;  // voxels a third of the radius wide (gpu.py:1539)
    a.r2 = radius * radius;
    a.mask = (int)(nb->cap - 1);
    a.want_normals = want_normals ? 1 : 0;
    for (int k = 0; k < 3; ++k) a.sensor[k] = sensor ? (double)sensor[k] : 0.0;
    LW_CUDA(cudaMemsetAsync(nb->keys, 0xFF, sizeof(int64_t) * nb->cap, s));  // EMPTY_KEY is -1
    LW_CUDA(cudaMemsetAsync(nb->acc, 0, sizeof(int64_t) * 4 * nb->cap, s));
    LW_CUDA(cudaMemsetAsync(nb->m, 0, sizeof(int32_t), s));
    if (n_ub <= 0) return LW_OK;
    const int sms = device_sms();
    const int grid = blocks_for(n_ub, 256, 8 * sms);
    if (xyz_stride == 4)
        k_nb_insert<4><<<grid, 256, 0, s>>>(xyz, n_dev, n_ub, a, *nb);
    else
        k_nb_insert<3><<<grid, 256, 0, s>>>(xyz, n_dev, n_ub, a, *nb);
    const int nt = blocks_for(nb->cap, NB_TILE);
    k_nb_count<<<nt, NB_TILE, 0, s>>>(*nb);
    k_nb_scan<<<1, 1024, 0, s>>>(*nb, nt);
    k_nb_scatter<<<nt, NB_TILE, 0, s>>>(*nb);
    // a warp per voxel: at most one voxel per point
    k_nb_voxel<<<blocks_for(n_ub * 32, 256, 16 * sms), 256, 0, s>>>(a, *nb);
    k_nb_gather<<<grid, 256, 0, s>>>(n_dev, n_ub, a.want_normals, *nb, out_cnt, out_nrm, out_curv);
    LW_LAUNCHED("lw_neighborhoods");
    count_launches(6);
    return LW_OK;
}

}  // extern "C"
