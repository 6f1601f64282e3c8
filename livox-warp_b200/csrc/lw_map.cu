// Integration voxel map, free-space carving and the map's visible set on sm_100a.
//
// Reference: python/livox_warp/gpu.py -- keep_raw :155-167, k_map_insert :373-412, map_centroid :415-419,
// local_plane :422-466, k_carve :469-593, transient / ghost :286-299, settled_near :596-634,
// k_classify_map :699-747, the scan + scatter of Pipeline.build :1495-1504, clear_map :1305-1313.
//
// Determinism: the map's sums are exact int64 fixed point and the 4096-hit cap sums the first hits in point
// order, so keys, counts, sums, centroids and therefore every carving decision are independent of thread
// order and agree bit for bit with the CPU oracle.
#include "lw_common.cuh"
#include "lw_linalg.cuh"

namespace lw {


// Carving constants (gpu.py:66-73)
constexpr float CARVE_MIN_RANGE = 0.05f;
constexpr float CARVE_MARGIN_VOXELS = 3.0f;
constexpr float CARVE_MARGIN_FRACTION = 0.03f;
constexpr float CARVE_GRAZING_VOXELS = 1.5f;
constexpr float CARVE_MIN_COSINE = 0.05f;
constexpr float CARVE_PIERCE_PLANE = 0.6f;
constexpr float CARVE_PIERCE_POINT = 0.5f;

__device__ __forceinline__ bool keep_raw(float x, float y, float z, uint32_t a, const lw_view& v) {
    float r = len3(x, y, z);
    if (r < v.min_range || r > v.max_range) return false;
    if (refl_of(a) < v.min_refl) return false;
    if (((v.noise_mask >> (tag_of(a) & 3)) & 1) == 0) return false;
    if (((v.ret_mask >> (ret_of(a) & 3)) & 1) == 0) return false;
    return true;
}

template <int STRIDE>
__device__ __forceinline__ void load_xyz(const float* __restrict__ xyz, int64_t i, float& x, float& y, float& z) {
    if (STRIDE == 4) {
        float4 p = __ldg(reinterpret_cast<const float4*>(xyz) + i);
        x = p.x;
        y = p.y;
        z = p.z;
    } else {
        x = xyz[i * 3 + 0];
        y = xyz[i * 3 + 1];
        z = xyz[i * 3 + 2];
    }
}

struct MapIns {
    float inv_voxel;
    int mask;
};

// =====================================================================================================
// Map insert: A claims and counts, B sums (first LW_MAP_CAP hits in order) and updates the hit times,
// D publishes the counts and resets the scratch.
// =====================================================================================================

template <int STRIDE>
__device__ __forceinline__ bool map_point(const float* __restrict__ xyz, const uint32_t* __restrict__ attr,
                                          const int32_t* __restrict__ frame, const float* __restrict__ poses,
                                          const lw_view& v, int64_t i, float inv, float& wx, float& wy, float& wz) {
    float x, y, z;
    load_xyz<STRIDE>(xyz, i, x, y, z);
    if (!keep_raw(x, y, z, attr[i], v)) return false;
    const float* T = poses + (int64_t)(frame[i] & (LW_POSE_SLOTS - 1)) * 16;
    xform(T, x, y, z, wx, wy, wz);
    return true;
}

template <int STRIDE>
__global__ void k_map_a(const float* __restrict__ xyz, const uint32_t* __restrict__ attr,
                        const int32_t* __restrict__ frame, const int* n_dev, int64_t n_ub,
                        const float* __restrict__ poses, lw_view v, MapIns mi, lw_map map, int* __restrict__ pslot) {
    int64_t n = n_dev ? (int64_t)*n_dev : n_ub;
    if (n > n_ub) n = n_ub;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float wx, wy, wz;
        int s = -1;
        if (map_point<STRIDE>(xyz, attr, frame, poses, v, i, mi.inv_voxel, wx, wy, wz)) {
            int64_t key = key_ijk(ifloor(wx * mi.inv_voxel), ifloor(wy * mi.inv_voxel), ifloor(wz * mi.inv_voxel));
            bool claimed;
            s = claim_slot(key, map.keys, mi.mask, &claimed);
            if (claimed) atomicAdd(map.stats + 0, 1);
            if (s < 0) {
                atomicAdd(map.stats + 1, 1);  // table full along this probe chain
            } else {
                atomicAdd(map.bcnt + s, 1);
                atomicMin(map.lead + s, (int)i);
            }
        }
        pslot[i] = s;
    }
}

__device__ __forceinline__ void map_add(lw_map& map, int s, float wx, float wy, float wz, uint32_t a) {
    const float FW = (float)LW_FIX_W;
    atomic_add_i64(map.acc + 4 * (int64_t)s + 0, to_fix(wx, FW));
    atomic_add_i64(map.acc + 4 * (int64_t)s + 1, to_fix(wy, FW));
    atomic_add_i64(map.acc + 4 * (int64_t)s + 2, to_fix(wz, FW));
    atomic_add_i64(map.acc + 4 * (int64_t)s + 3, (int64_t)refl_of(a));
}

template <int STRIDE>
__global__ void k_map_b(const float* __restrict__ xyz, const uint32_t* __restrict__ attr,
                        const float* __restrict__ t, const int32_t* __restrict__ frame, const int* n_dev, int64_t n_ub,
                        const float* __restrict__ poses, lw_view v, MapIns mi, lw_map map,
                        const int* __restrict__ pslot) {
    int64_t n = n_dev ? (int64_t)*n_dev : n_ub;
    if (n > n_ub) n = n_ub;
    const int lane = threadIdx.x & 31;
    // warp-uniform trip count (blockDim is a multiple of 32): the cap-crossing fill below needs the whole warp
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n;
         base += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = base + lane;
        int s = i < n ? pslot[i] : -1;
        int pre = 0;
        bool lead = false;
        if (s >= 0) {
            float wx, wy, wz;
            map_point<STRIDE>(xyz, attr, frame, poses, v, i, mi.inv_voxel, wx, wy, wz);
            pre = map.cnt[s];
            if (pre + map.bcnt[s] <= LW_MAP_CAP)
                map_add(map, s, wx, wy, wz, attr[i]);
            else
                lead = pre < LW_MAP_CAP && map.lead[s] == (int)i;
            float ti = t[i];
            atomic_max_float(map.last + s, ti);
            atomic_min_float(map.first + s, ti);
        }
        // this batch crosses the cap: the voxel sums its first (cap - pre) hits in index order
        for (unsigned lm = __ballot_sync(0xffffffffu, lead); lm; lm &= lm - 1) {
            int src = __ffs(lm) - 1;
            int sl = __shfl_sync(0xffffffffu, s, src);
            int room = LW_MAP_CAP - __shfl_sync(0xffffffffu, pre, src);
            warp_fill_first(pslot, base + src, n, sl, room, [&](int64_t j) {
                float ux, uy, uz;
                map_point<STRIDE>(xyz, attr, frame, poses, v, j, mi.inv_voxel, ux, uy, uz);
                map_add(map, sl, ux, uy, uz, attr[j]);
            });
        }
    }
}

__global__ void k_map_d(const int* n_dev, int64_t n_ub, lw_map map, const int* __restrict__ pslot) {
    int64_t n = n_dev ? (int64_t)*n_dev : n_ub;
    if (n > n_ub) n = n_ub;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int s = pslot[i];
        if (s < 0 || map.lead[s] != (int)i) continue;
        map.cnt[s] += map.bcnt[s];  // hits keep counting past the cap (carving compares them with misses)
        map.bcnt[s] = 0;
        map.lead[s] = NO_INDEX;
    }
}

// =====================================================================================================
// Carving
// =====================================================================================================

__device__ __forceinline__ void centroid(const lw_map& map, int s, float& x, float& y, float& z) {
    int c = map.cnt[s];
    double n = (double)(c < LW_MAP_CAP ? c : LW_MAP_CAP) * LW_FIX_W;
    x = (float)((double)map.acc[4 * (int64_t)s + 0] / n);
    y = (float)((double)map.acc[4 * (int64_t)s + 1] / n);
    z = (float)((double)map.acc[4 * (int64_t)s + 2] / n);
}

// Normal of the surface through voxel (ix, iy, iz) from a PCA of the occupied 3x3x3 neighbourhood's centroids
// taken relative to `o` (gpu.py:422-466); w = 2 surface, 1 at least 4 occupied but no surface, 0 fewer.
// Find the slots of n keys at once: every first probe is issued before any is waited on; collisions (rare at
// the map's load factor) continue one by one. -1 where the key is absent.
template <int N>
__device__ __forceinline__ void find_slots(const int64_t* key, int* slot, const int64_t* __restrict__ keys, int mask) {
    int h[N];
    int64_t k0[N];
#pragma unroll
    for (int u = 0; u < N; ++u) {
        h[u] = slot_hash(key[u]) & mask;
        k0[u] = __ldg(keys + h[u]);
    }
#pragma unroll
    for (int u = 0; u < N; ++u) {
        if (k0[u] == key[u]) {
            slot[u] = h[u];
        } else if (k0[u] == EMPTY_KEY) {
            slot[u] = -1;
        } else {
            int s = -1;
#pragma unroll 1
            for (int p = 1; p < PROBES; ++p) {
                int t = (h[u] + p) & mask;
                int64_t kk = __ldg(keys + t);
                if (kk == key[u]) {
                    s = t;
                    break;
                }
                if (kk == EMPTY_KEY) break;
            }
            slot[u] = s;
        }
    }
}

// Normal of the surface through voxel (ix, iy, iz) from a PCA of the occupied 3x3x3 neighbourhood's centroids
// taken relative to `o` (gpu.py:422-466); w = 2 surface, 1 at least 4 occupied but no surface, 0 fewer.
// All 27 probes go out together; the occupied neighbours are then summed in the reference's (gx, gy, gz) order.
__device__ float4 local_plane(int ix, int iy, int iz, float ox, float oy, float oz, const lw_map& map, int mask) {
    double cs[3] = {0.0, 0.0, 0.0}, cc[6] = {0, 0, 0, 0, 0, 0};
    int cn = 0;
    int64_t key[27];
    int slot[27];
#pragma unroll
    for (int u = 0; u < 27; ++u) key[u] = key_ijk(ix + u / 9 - 1, iy + (u / 3) % 3 - 1, iz + u % 3 - 1);
    find_slots<27>(key, slot, map.keys, mask);
    int cnt[27];
#pragma unroll
    for (int u = 0; u < 27; ++u) cnt[u] = slot[u] >= 0 ? __ldg(map.cnt + slot[u]) : 0;
    // the occupied neighbours' sums, fetched nine at a time, then taken in order
#pragma unroll 1
    for (int u0 = 0; u0 < 27; u0 += 9) {
        long long ax[9], ay[9], az[9];
#pragma unroll
        for (int v = 0; v < 9; ++v) {
            const int s = slot[u0 + v];
            const bool occ = cnt[u0 + v] > 0;
            const long long* a = reinterpret_cast<const long long*>(map.acc) + 4 * (int64_t)s;
            ax[v] = occ ? __ldg(a + 0) : 0;
            ay[v] = occ ? __ldg(a + 1) : 0;
            az[v] = occ ? __ldg(a + 2) : 0;
        }
#pragma unroll
        for (int v = 0; v < 9; ++v) {
            const int u = u0 + v;
            if (cnt[u] > 0) {
                const int c = cnt[u];
                const double nn = (double)(c < LW_MAP_CAP ? c : LW_MAP_CAP) * LW_FIX_W;
                const float cx = (float)((double)ax[v] / nn), cy = (float)((double)ay[v] / nn);
                const float cz = (float)((double)az[v] / nn);
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
        }
    }
    if (cn < 4) return make_float4(0.0f, 0.0f, 1.0f, 0.0f);
    double inv = 1.0 / (double)cn;
    double mu[3] = {cs[0] * inv, cs[1] * inv, cs[2] * inv};
    double C[9];
    const int up[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C[i * 3 + j] = cc[up[i * 3 + j]] * inv - mu[i] * mu[j];
    double ev[3], Q[9];
    jacobi_eig<3>(C, ev, Q);
    int k = 0;
    if (ev[1] < ev[k]) k = 1;
    if (ev[2] < ev[k]) k = 2;
    int j = (k + 1) % 3, j2 = (k + 2) % 3;
    double mid = fmin(ev[j], ev[j2]);
    float ok = ev[k] < 0.25 * mid ? 2.0f : 1.0f;
    return make_float4((float)Q[0 * 3 + k], (float)Q[1 * 3 + k], (float)Q[2 * 3 + k], ok);
}

// local_plane kept out of line: it runs once per ray and once per occupied voxel a ray meets, and inlined its
// float64 PCA would set the register budget of the whole ray walk
__device__ __noinline__ float4 local_plane_nl(int ix, int iy, int iz, float ox, float oy, float oz, lw_map map,
                                              int mask) {
    return local_plane(ix, iy, iz, ox, oy, oz, map, mask);
}

// A ray of the carving pass: origin and unit direction through its pose; false when it is not carved (a noise
// return, out of range).
template <int STRIDE>
__device__ __forceinline__ bool carve_ray(const float* __restrict__ xyz, const uint32_t* __restrict__ attr,
                                          const int32_t* __restrict__ frame, const float* __restrict__ poses, int64_t i,
                                          float max_range, float& ox, float& oy, float& oz, float& wx, float& wy,
                                          float& wz, float& dx, float& dy, float& dz, float& L) {
    if (tag_of(attr[i]) != 0) return false;
    const float* T = poses + (int64_t)(frame[i] & (LW_POSE_SLOTS - 1)) * 16;
    ox = T[3];
    oy = T[7];
    oz = T[11];
    float px, py, pz;
    load_xyz<STRIDE>(xyz, i, px, py, pz);
    xform(T, px, py, pz, wx, wy, wz);
    dx = wx - ox;
    dy = wy - oy;
    dz = wz - oz;
    L = len3(dx, dy, dz);
    if (L < CARVE_MIN_RANGE || L > max_range) return false;
    dx = dx / L;
    dy = dy / L;
    dz = dz / L;
    return true;
}

// Carving, pass 1 (gpu.py:469-495): one thread per ray finds where the ray stops -- short of its end point by a
// margin that grows at grazing incidence on the end point's local plane -- in voxel units; 0 when not carved.
template <int STRIDE>
__global__ void k_carve_setup(const float* __restrict__ xyz, const uint32_t* __restrict__ attr,
                              const int32_t* __restrict__ frame, const int* n_dev, int64_t n_ub,
                              const float* __restrict__ poses, int every, float inv_voxel, float max_range, lw_map map,
                              float* __restrict__ ray_stop) {
    int64_t n = n_dev ? (int64_t)*n_dev : n_ub;
    if (n > n_ub) n = n_ub;
    const int mask = (int)(map.cap - 1);
    const int64_t nrays = (n + every - 1) / every;
    const float voxel = 1.0f / inv_voxel;
    for (int64_t ray = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; ray < nrays;
         ray += (int64_t)gridDim.x * blockDim.x) {
        float ox, oy, oz, wx, wy, wz, dx, dy, dz, L;
        float stop = 0.0f;
        if (carve_ray<STRIDE>(xyz, attr, frame, poses, ray * every, max_range, ox, oy, oz, wx, wy, wz, dx, dy, dz, L)) {
            float margin = fmaxf(CARVE_MARGIN_VOXELS * voxel, CARVE_MARGIN_FRACTION * L);
            const float4 pe = local_plane(ifloor(wx * inv_voxel), ifloor(wy * inv_voxel), ifloor(wz * inv_voxel), wx,
                                          wy, wz, map, mask);
            if (pe.w > 0.5f) {
                float cosine = fabsf(pe.x * dx + pe.y * dy + pe.z * dz);
                margin = fmaxf(margin, CARVE_GRAZING_VOXELS * voxel / fmaxf(cosine, CARVE_MIN_COSINE));
            }
            stop = (L - margin) * inv_voxel;
        }
        ray_stop[ray] = stop;
    }
}

// Carving, pass 2 (gpu.py:496-593): one warp per ray. Every lane steps the same DDA (identical float operations,
// so the voxel sequence is the single-thread one); lane j takes steps 32c + j of chunk c, probes its voxel and,
// when it is occupied, fits its local plane and tests whether the ray pierces it. The misses are integer atomics,
// so the map gets the same counts in any order.
template <int STRIDE>
__global__ void __launch_bounds__(128) k_carve(const float* __restrict__ xyz, const uint32_t* __restrict__ attr,
                                               const int32_t* __restrict__ frame, const int* n_dev, int64_t n_ub,
                                               const float* __restrict__ poses, int every, float inv_voxel,
                                               float max_range, int max_steps, lw_map map,
                                               const float* __restrict__ ray_stop) {
    int64_t n = n_dev ? (int64_t)*n_dev : n_ub;
    if (n > n_ub) n = n_ub;
    const int mask = (int)(map.cap - 1);
    const int64_t nrays = (n + every - 1) / every;
    const int lane = threadIdx.x & 31;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const float voxel = 1.0f / inv_voxel;
    for (int64_t ray = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; ray < nrays; ray += nwarps) {
        const float stop = ray_stop[ray];
        if (stop <= 1.0f) continue;
        float ox, oy, oz, wx, wy, wz, dx, dy, dz, L;
        carve_ray<STRIDE>(xyz, attr, frame, poses, ray * every, max_range, ox, oy, oz, wx, wy, wz, dx, dy, dz, L);
        float posx = ox * inv_voxel, posy = oy * inv_voxel, posz = oz * inv_voxel;
        int ix = ifloor(posx), iy = ifloor(posy), iz = ifloor(posz);
        int sx = 1, sy = 1, sz = 1;
        float tmx = 1.0e30f, tmy = 1.0e30f, tmz = 1.0e30f, tdx = 1.0e30f, tdy = 1.0e30f, tdz = 1.0e30f;
        if (dx > 1.0e-9f) {
            tmx = ((float)(ix + 1) - posx) / dx;
            tdx = 1.0f / dx;
        } else if (dx < -1.0e-9f) {
            sx = -1;
            tmx = (posx - (float)ix) / (-dx);
            tdx = -1.0f / dx;
        }
        if (dy > 1.0e-9f) {
            tmy = ((float)(iy + 1) - posy) / dy;
            tdy = 1.0f / dy;
        } else if (dy < -1.0e-9f) {
            sy = -1;
            tmy = (posy - (float)iy) / (-dy);
            tdy = -1.0f / dy;
        }
        if (dz > 1.0e-9f) {
            tmz = ((float)(iz + 1) - posz) / dz;
            tdz = 1.0f / dz;
        } else if (dz < -1.0e-9f) {
            sz = -1;
            tmz = (posz - (float)iz) / (-dz);
            tdz = -1.0f / dz;
        }
        bool done = false;
#pragma unroll 1
        for (int c0 = 0; c0 < max_steps && !done; c0 += 32) {
            int vx = 0, vy = 0, vz = 0;
            bool mine = false;
            // every lane takes the same 32 steps (warp-uniform control flow); lane u keeps step c0 + u
#pragma unroll 1
            for (int u = 0; u < 32; ++u) {
                if (c0 + u >= max_steps) {
                    done = true;
                    break;
                }
                float tt;
                if (tmx < tmy && tmx < tmz) {
                    tt = tmx;
                    ix += sx;
                    tmx += tdx;
                } else if (tmy < tmz) {
                    tt = tmy;
                    iy += sy;
                    tmy += tdy;
                } else {
                    tt = tmz;
                    iz += sz;
                    tmz += tdz;
                }
                if (tt >= stop) {
                    done = true;
                    break;
                }
                if (u == lane) {
                    vx = ix;
                    vy = iy;
                    vz = iz;
                    mine = true;
                }
            }
            if (!mine) continue;
            const int s = find_slot(key_ijk(vx, vy, vz), map.keys, mask);
            if (s < 0 || __ldg(map.cnt + s) <= 0) continue;
            float cx, cy, cz;
            centroid(map, s, cx, cy, cz);
            const float rx = cx - ox, ry = cy - oy, rz = cz - oz;
            bool pierced = false;
            const float4 pl = local_plane_nl(vx, vy, vz, cx, cy, cz, map, mask);
            if (pl.w > 1.5f) {
                const float dn = dx * pl.x + dy * pl.y + dz * pl.z;
                if (fabsf(dn) > 1.0e-4f) {
                    const float f = (rx * pl.x + ry * pl.y + rz * pl.z) / dn;
                    const float xx = dx * f - rx, xy = dy * f - ry, xz = dz * f - rz;  // plane crossing rel. to centroid
                    if (len3(xx, xy, xz) < CARVE_PIERCE_PLANE * voxel) pierced = true;
                }
            } else {
                const float g = rx * dx + ry * dy + rz * dz;
                const float qx = rx - g * dx, qy = ry - g * dy, qz = rz - g * dz;
                if (len3(qx, qy, qz) < CARVE_PIERCE_POINT * voxel) pierced = true;
            }
            if (pierced) atomicAdd(map.miss + s, every);
        }
    }
}

// =====================================================================================================
// Visible set of the map (k_classify_map) compacted in slot order.
// =====================================================================================================

__device__ __forceinline__ int transient(int c, int miss, const lw_view& v) {
    if (miss < v.carve_min) return 0;
    return (float)miss > v.carve_ratio * (float)c ? 1 : 0;
}

__device__ __forceinline__ int ghost(int c, int miss, float last, const lw_view& v) {
    if (v.now - last < v.carve_stale) return 0;
    return transient(c, miss, v);
}

__device__ __forceinline__ int in_crop(float x, float y, float z, const lw_view& v) {
    if (v.crop_on == 0) return 1;
    if (x < v.crop_lo[0] || y < v.crop_lo[1] || z < v.crop_lo[2]) return 0;
    if (x > v.crop_hi[0] || y > v.crop_hi[1] || z > v.crop_hi[2]) return 0;
    return 1;
}

__device__ int settled_near(int ix, int iy, int iz, const lw_view& v, const lw_map& map) {
    for (int nb = 0; nb < 7; ++nb) {
        int jx = ix, jy = iy, jz = iz;
        if (nb == 1) jx = ix - 1;
        else if (nb == 2) jx = ix + 1;
        else if (nb == 3) jy = iy - 1;
        else if (nb == 4) jy = iy + 1;
        else if (nb == 5) jz = iz - 1;
        else if (nb == 6) jz = iz + 1;
        int s = find_slot(key_ijk(jx, jy, jz), map.keys, v.map_mask);
        if (s >= 0) {
            float age = v.now - map.first[s];
            if (age < 0.0f) age = 1.0e9f;  // clock restarted: history predates the new clock
            if (age >= v.dyn_settle && transient(map.cnt[s], map.miss[s], v) == 0) return 1;
        }
    }
    return 0;
}

__device__ __forceinline__ bool classify_flag_key(const lw_map& map, int64_t s, int64_t key, const lw_view& v,
                                                  int min_count, float& wx, float& wy, float& wz) {
    if (key == EMPTY_KEY) return false;
    int c = map.cnt[s];
    if (c < min_count) return false;
    float last = map.last[s];
    if (v.persist > 0.0f && v.now - last > v.persist) return false;
    if (v.carve_on != 0 && ghost(c, map.miss[s], last, v) != 0) return false;
    if (c <= 0) return false;
    centroid(map, (int)s, wx, wy, wz);
    return in_crop(wx, wy, wz, v) != 0;
}

// The classification runs in tiles of CL_TILE slots, a CTA per tile and CL_PER consecutive slots per thread (their
// keys in 16-byte loads), so every load of a tile is in flight at once; per-thread counts are scanned across the
// CTA, which keeps the compaction in slot order.
constexpr int CL_PER = 8, CL_THREADS = 512, CL_TILE = CL_PER * CL_THREADS;

__device__ __forceinline__ void load_keys(const lw_map& map, int64_t s0, int64_t* k) {
    if (s0 + CL_PER <= map.cap && (reinterpret_cast<uintptr_t>(map.keys) & 15) == 0) {
        const longlong2* p = reinterpret_cast<const longlong2*>(map.keys + s0);
#pragma unroll
        for (int h = 0; h < CL_PER / 2; ++h) {
            longlong2 x = p[h];
            k[2 * h] = x.x;
            k[2 * h + 1] = x.y;
        }
    } else {
#pragma unroll
        for (int u = 0; u < CL_PER; ++u) k[u] = s0 + u < map.cap ? map.keys[s0 + u] : EMPTY_KEY;
    }
}

__global__ void __launch_bounds__(CL_THREADS) k_classify_count(lw_map map, lw_view v, int min_count,
                                                               int* __restrict__ tiles) {
    __shared__ int sm[33];
    const int64_t s0 = (int64_t)blockIdx.x * CL_TILE + (int64_t)threadIdx.x * CL_PER;
    int64_t k[CL_PER];
    load_keys(map, s0, k);
    int c = 0;
#pragma unroll
    for (int u = 0; u < CL_PER; ++u) {
        float wx, wy, wz;
        if (k[u] != EMPTY_KEY && classify_flag_key(map, s0 + u, k[u], v, min_count, wx, wy, wz)) ++c;
    }
    int tot;
    block_excl(c, sm, &tot);
    if (threadIdx.x == 0) tiles[blockIdx.x] = tot;
}

// In-place exclusive scan of nt tile counts by one CTA; tiles[nt] receives the total.
__global__ void k_scan_tiles(int* tiles, int nt, int* total_out) {
    __shared__ int sm[33];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < nt; base += blockDim.x) {
        int j = base + threadIdx.x;
        int v = j < nt ? tiles[j] : 0;
        // inclusive warp scan, then across warps
        int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        int inc = v;
        for (int o = 1; o < 32; o <<= 1) {
            int u = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += u;
        }
        if (lane == 31) sm[w] = inc;
        __syncthreads();
        if (w == 0) {
            int nw = blockDim.x >> 5;
            int x = lane < nw ? sm[lane] : 0;
            int xi = x;
            for (int o = 1; o < 32; o <<= 1) {
                int u = __shfl_up_sync(0xffffffffu, xi, o);
                if (lane >= o) xi += u;
            }
            if (lane < nw) sm[lane] = xi - x;
            if (lane == 31) sm[32] = xi;
        }
        __syncthreads();
        int excl = carry + sm[w] + inc - v;
        if (j < nt) tiles[j] = excl;
        __syncthreads();
        if (threadIdx.x == 0) carry += sm[32];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        tiles[nt] = carry;
        if (total_out) *total_out = carry;
    }
}

__global__ void __launch_bounds__(CL_THREADS) k_classify_scatter(lw_map map, lw_view v, int min_count,
                                                                 const int* __restrict__ tiles,
                                                                 float* __restrict__ out_xyz,
                                                                 uint32_t* __restrict__ out_attr,
                                                                 float* __restrict__ out_t, int* __restrict__ out_dyn) {
    __shared__ int sm[33];
    const int64_t s0 = (int64_t)blockIdx.x * CL_TILE + (int64_t)threadIdx.x * CL_PER;
    int64_t k[CL_PER];
    load_keys(map, s0, k);
    float wx[CL_PER], wy[CL_PER], wz[CL_PER];
    unsigned flags = 0;
#pragma unroll
    for (int u = 0; u < CL_PER; ++u)
        if (k[u] != EMPTY_KEY && classify_flag_key(map, s0 + u, k[u], v, min_count, wx[u], wy[u], wz[u]))
            flags |= 1u << u;
    int tot;
    int j = tiles[blockIdx.x] + block_excl(__popc(flags), sm, &tot);
#pragma unroll
    for (int u = 0; u < CL_PER; ++u) {
        if (!((flags >> u) & 1u)) continue;
        const int64_t s = s0 + u;
        int c = map.cnt[s];
        int n = c < LW_MAP_CAP ? c : LW_MAP_CAP;
        int refl = (int)((double)map.acc[4 * s + 3] / (double)n + 0.5);
        if (refl > 255) refl = 255;
        out_xyz[3 * (int64_t)j + 0] = wx[u];
        out_xyz[3 * (int64_t)j + 1] = wy[u];
        out_xyz[3 * (int64_t)j + 2] = wz[u];
        out_attr[j] = (uint32_t)refl;  // mean reflectivity only: tag, return and device mean nothing for a voxel
        out_t[j] = map.last[s];
        int dyn = 0;
        if (transient(c, map.miss[s], v) != 0)
            dyn = 1;
        else if (settled_near(ifloor(wx[u] * v.inv_voxel), ifloor(wy[u] * v.inv_voxel), ifloor(wz[u] * v.inv_voxel), v,
                              map) == 0)
            dyn = 1;
        out_dyn[j] = dyn;
        ++j;
    }
}

// =====================================================================================================
// Visible set of the live ring (k_classify_live, gpu.py:637-697) compacted in ring order: a CTA of LV_TILE
// threads per tile of ring slots counts its drawn points, one CTA scans the counts, and the scatter pass
// classifies again and writes each drawn point at its tile's offset plus its rank in the tile.
// =====================================================================================================

constexpr int LV_TILE = 1024;

struct LiveRing {
    const float* xyz;      // [cap*3] sensor-frame points as measured
    const uint32_t* attr;  // [cap]
    const float* t;        // [cap]
    const int32_t* frame;  // [cap] frame ids
    int64_t cap, filled;
};

// Ring slot i posed into the world; false when it is not drawn (gpu.py:664-690).
__device__ __forceinline__ bool live_point(const LiveRing& r, const lw_pose_table& pt, const lw_view& v, int64_t i,
                                           float& wx, float& wy, float& wz) {
    if (i >= r.filled || i >= r.cap) return false;
    const float t = r.t[i];
    if (v.persist > 0.0f && v.now - t > v.persist) return false;
    float x = r.xyz[3 * i], y = r.xyz[3 * i + 1], z = r.xyz[3 * i + 2];
    if (!keep_raw(x, y, z, r.attr[i], v)) return false;
    const int fid = r.frame[i];
    const int f = fid & (LW_POSE_SLOTS - 1);
    if (v.inv_frame_dt > 0.0f) {
        // odometry on: drawn only once the slot holds this frame's pose for the current epoch
        if (pt.owner_frame[f] != fid || pt.owner_epoch[f] != v.epoch) return false;
        const float xf = t * v.inv_frame_dt;
        const float frac = xf - floorf(xf) - 0.5f;  // the point's time from mid-frame, in frames: [-0.5, 0.5)
        deskew_frac(x, y, z, frac, pt.tw + 6 * (int64_t)f, x, y, z);
    }
    xform(pt.poses + 16 * (int64_t)f, x, y, z, wx, wy, wz);
    return in_crop(wx, wy, wz, v) != 0;
}

__global__ void __launch_bounds__(LV_TILE) k_live_count(LiveRing r, lw_pose_table pt, lw_view v,
                                                        int* __restrict__ tiles) {
    const int64_t i = (int64_t)blockIdx.x * LV_TILE + threadIdx.x;
    float wx, wy, wz;
    const int c = __syncthreads_count(live_point(r, pt, v, i, wx, wy, wz) ? 1 : 0);
    if (threadIdx.x == 0) tiles[blockIdx.x] = c;
}

__global__ void __launch_bounds__(LV_TILE) k_live_scatter(LiveRing r, lw_pose_table pt, lw_view v, lw_map map,
                                                          const int* __restrict__ tiles, float* __restrict__ out_xyz,
                                                          uint32_t* __restrict__ out_attr, float* __restrict__ out_t,
                                                          int* __restrict__ out_dyn) {
    __shared__ int sm[33];
    const int64_t i = (int64_t)blockIdx.x * LV_TILE + threadIdx.x;
    float wx = 0.0f, wy = 0.0f, wz = 0.0f;
    const int f = live_point(r, pt, v, i, wx, wy, wz) ? 1 : 0;
    int tot;
    const int rank = block_rank(f, sm, &tot);
    if (!f) return;
    const int64_t j = (int64_t)tiles[blockIdx.x] + rank;
    out_xyz[3 * j + 0] = wx;
    out_xyz[3 * j + 1] = wy;
    out_xyz[3 * j + 2] = wz;
    out_attr[j] = r.attr[i];
    out_t[j] = r.t[i];
    // static when the map voxel it lands in, or one of its 6 neighbours, is old and no ghost (gpu.py:691-697)
    out_dyn[j] = v.dyn_on != 0
                     ? 1 - settled_near(ifloor(wx * v.inv_voxel), ifloor(wy * v.inv_voxel), ifloor(wz * v.inv_voxel), v,
                                        map)
                     : 0;
}

// Frame id of each staged point: floor(max(t, 0) * inv_dt), 0 when inv_dt <= 0 (gpu.py:340-348).
__global__ void k_frame_of(const float* __restrict__ t, int64_t n, float inv_dt, int32_t* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = inv_dt <= 0.0f ? 0 : (int)floorf(fmaxf(t[i], 0.0f) * inv_dt);
}

__global__ void k_map_clear(lw_map map) {
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < map.cap; s += (int64_t)gridDim.x * blockDim.x) {
        map.keys[s] = EMPTY_KEY;
        map.cnt[s] = 0;
        map.acc[4 * s + 0] = map.acc[4 * s + 1] = map.acc[4 * s + 2] = map.acc[4 * s + 3] = 0;
        map.last[s] = 0.0f;
        map.first[s] = 1.0e30f;
        map.miss[s] = 0;
        map.bcnt[s] = 0;
        map.lead[s] = NO_INDEX;
    }
    if (blockIdx.x == 0 && threadIdx.x < 2) map.stats[threadIdx.x] = 0;
}

}  // namespace lw

using namespace lw;

static int check_map(const lw_map* map, const char* who) {
    if (!map || !map->keys || !map->cnt || !map->acc || !map->last || !map->first || !map->miss || !map->bcnt ||
        !map->lead || !map->stats)
        return set_error(LW_EINVAL, "%s: incomplete map", who);
    if (map->cap <= 0 || (map->cap & (map->cap - 1)) != 0)
        return set_error(LW_EINVAL, "%s: map capacity %lld is not a power of two", who, (long long)map->cap);
    return LW_OK;
}

extern "C" {

int lw_map_insert(const float* xyz, int32_t xyz_stride, const uint32_t* attr, const float* t, const int32_t* frame,
                  const int32_t* n_dev, int64_t n_ub, const float* poses, const lw_view* v, float inv_voxel,
                  lw_map* map, int32_t* pslot, void* stream) {
    int r = check_map(map, "lw_map_insert");
    if (r != LW_OK) return r;
    if (!xyz || !attr || !t || !frame || !poses || !v || !pslot || (xyz_stride != 3 && xyz_stride != 4))
        return set_error(LW_EINVAL, "lw_map_insert: bad arguments");
    if (n_ub <= 0) return LW_OK;
    cudaStream_t s = (cudaStream_t)stream;
    MapIns mi{inv_voxel, (int)(map->cap - 1)};
    int grid = blocks_for(n_ub, 256, 8 * device_sms());
    ProfScope prof("map_insert", s);
    if (xyz_stride == 4) {
        k_map_a<4><<<grid, 256, 0, s>>>(xyz, attr, frame, n_dev, n_ub, poses, *v, mi, *map, pslot);
        k_map_b<4><<<grid, 256, 0, s>>>(xyz, attr, t, frame, n_dev, n_ub, poses, *v, mi, *map, pslot);
    } else {
        k_map_a<3><<<grid, 256, 0, s>>>(xyz, attr, frame, n_dev, n_ub, poses, *v, mi, *map, pslot);
        k_map_b<3><<<grid, 256, 0, s>>>(xyz, attr, t, frame, n_dev, n_ub, poses, *v, mi, *map, pslot);
    }
    k_map_d<<<grid, 256, 0, s>>>(n_dev, n_ub, *map, pslot);
    LW_LAUNCHED("lw_map_insert");
    count_launches(3);
    return LW_OK;
}

int lw_carve(const float* xyz, int32_t xyz_stride, const uint32_t* attr, const int32_t* frame, const int32_t* n_dev,
             int64_t n_ub, const float* poses, int32_t every, float inv_voxel, float max_range, int32_t max_steps,
             lw_map* map, float* ray_stop, void* stream) {
    int r = check_map(map, "lw_carve");
    if (r != LW_OK) return r;
    if (!xyz || !attr || !frame || !poses || !ray_stop || (xyz_stride != 3 && xyz_stride != 4))
        return set_error(LW_EINVAL, "lw_carve: bad arguments");
    if (n_ub <= 0) return LW_OK;
    if (every < 1) every = 1;
    cudaStream_t s = (cudaStream_t)stream;
    int64_t rays = (n_ub + every - 1) / every;
    int grid1 = blocks_for(rays, 64, 16 * device_sms());      // a thread per ray
    int grid = blocks_for(rays * 32, 128, 24 * device_sms());  // a warp per ray
    ProfScope prof("carve", s);
    if (xyz_stride == 4) {
        k_carve_setup<4><<<grid1, 64, 0, s>>>(xyz, attr, frame, n_dev, n_ub, poses, every, inv_voxel, max_range, *map,
                                              ray_stop);
        k_carve<4><<<grid, 128, 0, s>>>(xyz, attr, frame, n_dev, n_ub, poses, every, inv_voxel, max_range, max_steps,
                                        *map, ray_stop);
    } else {
        k_carve_setup<3><<<grid1, 64, 0, s>>>(xyz, attr, frame, n_dev, n_ub, poses, every, inv_voxel, max_range, *map,
                                              ray_stop);
        k_carve<3><<<grid, 128, 0, s>>>(xyz, attr, frame, n_dev, n_ub, poses, every, inv_voxel, max_range, max_steps,
                                        *map, ray_stop);
    }
    LW_LAUNCHED("lw_carve");
    count_launches(2);
    return LW_OK;
}

int lw_map_build(const lw_map* map, const lw_view* v, int32_t min_count, float* out_xyz, uint32_t* out_attr,
                 float* out_t, int32_t* out_dyn, int32_t* tiles, int32_t* count_dev, void* stream) {
    int r = check_map(map, "lw_map_build");
    if (r != LW_OK) return r;
    if (!v || !out_xyz || !out_attr || !out_t || !out_dyn || !tiles || !count_dev)
        return set_error(LW_EINVAL, "lw_map_build: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    int nt = blocks_for(map->cap, CL_TILE);  // <= cap / 1024 + 1 tiles: within the caller's buffer
    ProfScope prof("map_build", s);
    k_classify_count<<<nt, CL_THREADS, 0, s>>>(*map, *v, min_count, tiles);
    k_scan_tiles<<<1, 1024, 0, s>>>(tiles, nt, count_dev);
    k_classify_scatter<<<nt, CL_THREADS, 0, s>>>(*map, *v, min_count, tiles, out_xyz, out_attr, out_t, out_dyn);
    LW_LAUNCHED("lw_map_build");
    count_launches(3);
    return LW_OK;
}

int lw_live_build(const float* ring_xyz, const uint32_t* ring_attr, const float* ring_t, const int32_t* ring_frame,
                  int64_t cap, int64_t filled, const lw_pose_table* pt, const lw_view* v, const lw_map* map,
                  float* out_xyz, uint32_t* out_attr, float* out_t, int32_t* out_dyn, int32_t* tiles,
                  int32_t* count_dev, void* stream) {
    int r = check_map(map, "lw_live_build");
    if (r != LW_OK) return r;
    if (!pt || !pt->poses || !pt->tw || !pt->owner_frame || !pt->owner_epoch || !v || !tiles || !count_dev ||
        cap < 0 || cap > (1LL << 30))  // at most 2^20 tiles of 1024 slots
        return set_error(LW_EINVAL, "lw_live_build: bad arguments (ring capacity at most 2^30)");
    if (cap > 0 && (!ring_xyz || !ring_attr || !ring_t || !ring_frame || !out_xyz || !out_attr || !out_t || !out_dyn))
        return set_error(LW_EINVAL, "lw_live_build: missing ring or output buffers");
    if (v->dyn_on != 0 && (v->map_mask < 0 || (int64_t)v->map_mask > map->cap - 1))
        return set_error(LW_EINVAL, "lw_live_build: view map_mask %d does not fit the map's %lld slots", v->map_mask,
                         (long long)map->cap);
    cudaStream_t s = (cudaStream_t)stream;
    LW_CUDA(cudaMemsetAsync(count_dev, 0, sizeof(int32_t), s));
    if (cap == 0 || filled <= 0) return LW_OK;
    LiveRing ring{ring_xyz, ring_attr, ring_t, ring_frame, cap, filled < cap ? filled : cap};
    // only the tiles that hold filled slots: the rest draw nothing
    const int nt = blocks_for(ring.filled, LV_TILE);
    ProfScope prof("live_build", s);
    k_live_count<<<nt, LV_TILE, 0, s>>>(ring, *pt, *v, tiles);
    k_scan_tiles<<<1, 1024, 0, s>>>(tiles, nt, count_dev);
    k_live_scatter<<<nt, LV_TILE, 0, s>>>(ring, *pt, *v, *map, tiles, out_xyz, out_attr, out_t, out_dyn);
    LW_LAUNCHED("lw_live_build");
    count_launches(3);
    return LW_OK;
}

int lw_frame_ids(const float* t, int64_t n, float inv_dt, int32_t* out, void* stream) {
    if (!t || !out) return set_error(LW_EINVAL, "lw_frame_ids: null argument");
    if (n <= 0) return LW_OK;
    k_frame_of<<<blocks_for(n, 256, 8 * device_sms()), 256, 0, (cudaStream_t)stream>>>(t, n, inv_dt, out);
    LW_LAUNCHED("lw_frame_ids");
    count_launches(1);
    return LW_OK;
}

int lw_stage_batch(const float* xyz_host, const uint32_t* attr_host, const float* t_host, int64_t n, float* xyz_dev,
                   uint32_t* attr_dev, float* t_dev, float inv_dt, int32_t* frame_dev, void* stream) {
    if (n < 0) return set_error(LW_EINVAL, "lw_stage_batch: negative point count");
    if (n == 0) return LW_OK;
    if (!xyz_host || !attr_host || !t_host || !xyz_dev || !attr_dev || !t_dev || !frame_dev)
        return set_error(LW_EINVAL, "lw_stage_batch: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    LW_CUDA(cudaMemcpyAsync(xyz_dev, xyz_host, (size_t)n * 3 * sizeof(float), cudaMemcpyHostToDevice, s));
    LW_CUDA(cudaMemcpyAsync(attr_dev, attr_host, (size_t)n * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    LW_CUDA(cudaMemcpyAsync(t_dev, t_host, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, s));
    k_frame_of<<<blocks_for(n, 256, 8 * device_sms()), 256, 0, s>>>(t_dev, n, inv_dt, frame_dev);
    LW_LAUNCHED("lw_stage_batch");
    count_launches(1);
    return LW_OK;
}

int lw_map_clear(lw_map* map, void* stream) {
    int r = check_map(map, "lw_map_clear");
    if (r != LW_OK) return r;
    k_map_clear<<<8 * device_sms(), 256, 0, (cudaStream_t)stream>>>(*map);
    LW_LAUNCHED("lw_map_clear");
    count_launches(1);
    return LW_OK;
}

}  // extern "C"
