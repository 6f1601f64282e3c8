// Ground segmentation and Euclidean clustering of the visible points on sm_100a.
//
// Reference: python/livox_warp/perception.py -- cell_of :32-36, k_gnd_min :39-43, k_gnd_support :46-58,
// k_gnd_label :61-111, Perception.ground :458-483; k_cl_insert :114-139, k_cc_init/step/jump :142-179,
// k_cc_reset/stats/flag/compact/gather :182-271, Perception.cluster / _voxelize / _label / _compact :487-567.
//
// Ground: the same three passes over a toroidal 2048 x 2048 grid; a fourth pass puts back the cells the points
// touched, so the 32 MB grid is cleared once at construction instead of on every call.
// Clusters: the non-ground points go into a voxel hash with exact fixed-point sums; the nodes are the occupied
// voxels in the order of their first point (deterministic); the neighbour graph (centroids within `connect`) is
// built once from the voxel hash instead of a radius query per pass; components come from a lock-free union-find
// that always hooks the larger root under the smaller, so every component is labelled by its smallest node index
// -- the fixed point the reference's min-label propagation converges to -- independent of thread order.
#include "lw_common.cuh"

namespace lw {

constexpr int GRID = 2048;
constexpr int CTILE = 1024;

__device__ __forceinline__ int cell_of(float x, float y, float inv_cell) {
    int cx = ifloor(x * inv_cell) & (GRID - 1);
    int cy = ifloor(y * inv_cell) & (GRID - 1);
    return cy * GRID + cx;
}

struct GroundArgs {
    float inv_cell, thick, thresh, slope_step, nz_min;
    int min_sup, use_nrm;
};

template <int STRIDE>
__device__ __forceinline__ void ld3(const float* __restrict__ p, int64_t i, float& x, float& y, float& z) {
    x = p[i * STRIDE + 0];
    y = p[i * STRIDE + 1];
    z = p[i * STRIDE + 2];
}

template <int STRIDE>
__global__ void k_gnd_min(const float* __restrict__ xyz, const int* n_dev, int64_t n_ub, GroundArgs a,
                          float* __restrict__ cell_min) {
    int64_t n = n_dev ? (int64_t)*n_dev : n_ub;
    if (n > n_ub) n = n_ub;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float x, y, z;
        ld3<STRIDE>(xyz, i, x, y, z);
        atomic_min_float(cell_min + cell_of(x, y, a.inv_cell), z);
    }
}

template <int STRIDE>
__global__ void k_gnd_support(const float* __restrict__ xyz, const int* n_dev, int64_t n_ub, GroundArgs a,
                              const float* __restrict__ cell_min, int* __restrict__ cell_sup) {
    int64_t n = n_dev ? (int64_t)*n_dev : n_ub;
    if (n > n_ub) n = n_ub;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float x, y, z;
        ld3<STRIDE>(xyz, i, x, y, z);
        int c = cell_of(x, y, a.inv_cell);
        if (z - cell_min[c] < a.thick) atomicAdd(cell_sup + c, 1);
    }
}

template <int STRIDE>
__global__ void k_gnd_label(const float* __restrict__ xyz, const float* __restrict__ nrm, const int* n_dev,
                            int64_t n_ub, GroundArgs a, const float* __restrict__ cell_min,
                            const int* __restrict__ cell_sup, int* __restrict__ out_gnd, float* __restrict__ out_hag) {
    int64_t n = n_dev ? (int64_t)*n_dev : n_ub;
    if (n > n_ub) n = n_ub;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float x, y, z;
        ld3<STRIDE>(xyz, i, x, y, z);
        int cx = ifloor(x * a.inv_cell), cy = ifloor(y * a.inv_cell);
        float g = 1.0e30f, g_floor = 1.0e30f;
        for (int dy = -2; dy <= 2; ++dy)
            for (int dx = -2; dx <= 2; ++dx) {
                int c = ((cy + dy) & (GRID - 1)) * GRID + ((cx + dx) & (GRID - 1));
                if (cell_sup[c] >= a.min_sup) {
                    int cheb = max(abs(dx), abs(dy));
                    float cand = cell_min[c] + a.slope_step * (float)cheb;
                    if (cand < g) {
                        g = cand;
                        g_floor = cell_min[c];
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
        if (h < a.thresh) {
            is_gnd = 1;
            // a steep normal within the ground band is the foot of a wall, unless the point is right at ground level
            if (a.use_nrm != 0 && h > 0.2f * a.thresh) {
                if (fabsf(nrm[i * 3 + 2]) < a.nz_min) is_gnd = 0;
            }
        }
        out_gnd[i] = is_gnd;
        out_hag[i] = is_gnd != 0 ? h : z - g_floor;
    }
}

template <int STRIDE>
__global__ void k_gnd_reset(const float* __restrict__ xyz, const int* n_dev, int64_t n_ub, GroundArgs a,
                            float* __restrict__ cell_min, int* __restrict__ cell_sup) {
    int64_t n = n_dev ? (int64_t)*n_dev : n_ub;
    if (n > n_ub) n = n_ub;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float x, y, z;
        ld3<STRIDE>(xyz, i, x, y, z);
        int c = cell_of(x, y, a.inv_cell);
        cell_min[c] = 1.0e30f;
        cell_sup[c] = 0;
    }
}

// =====================================================================================================
// Clusters
// =====================================================================================================

struct ClArgs {
    float inv_v;
    int mask, use_gnd;
    float connect2;
    int reach;
    float min_pts;
    int max_out;
};

// Pass 1: non-ground points claim their voxel and add exact fixed-point sums; the lowest point index per voxel is
// recorded (it orders the nodes).
template <int STRIDE>
__global__ void k_cl_insert(const float* __restrict__ xyz, const int* __restrict__ gnd, const int* n_dev,
                            int64_t n_ub, ClArgs a, lw_cluster_buf cb) {
    int64_t n = n_dev ? (int64_t)*n_dev : n_ub;
    if (n > n_ub) n = n_ub;
    const float FW = (float)LW_FIX_W;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int s = -1;
        if (!(a.use_gnd && gnd[i] != 0)) {
            float x, y, z;
            ld3<STRIDE>(xyz, i, x, y, z);
            int64_t key = key_ijk(ifloor(x * a.inv_v), ifloor(y * a.inv_v), ifloor(z * a.inv_v));
            bool claimed;
            s = claim_slot(key, cb.keys, a.mask, &claimed);
            if (s >= 0) {
                atomic_add_i64(cb.acc + 4 * (int64_t)s + 0, to_fix(x, FW));
                atomic_add_i64(cb.acc + 4 * (int64_t)s + 1, to_fix(y, FW));
                atomic_add_i64(cb.acc + 4 * (int64_t)s + 2, to_fix(z, FW));
                atomic_add_i64(cb.acc + 4 * (int64_t)s + 3, 1);
                atomicMin(cb.first + s, (int)i);
            }
        }
        cb.slot_of_pt[i] = s;
    }
}

// Pass 2/3: the nodes are the voxels in the order of their first point: per-tile counts, then the scatter.
__global__ void k_cl_node_count(const int* n_dev, int64_t n_ub, lw_cluster_buf cb) {
    int64_t n = n_dev ? (int64_t)*n_dev : n_ub;
    if (n > n_ub) n = n_ub;
    int64_t i = (int64_t)blockIdx.x * CTILE + threadIdx.x;
    int f = 0;
    if (i < n) {
        int s = cb.slot_of_pt[i];
        f = (s >= 0 && cb.first[s] == (int)i) ? 1 : 0;
    }
    int c = __syncthreads_count(f);
    if (threadIdx.x == 0) cb.tiles[blockIdx.x] = c;
}

__device__ __forceinline__ int tiles_before(const int* __restrict__ tiles, int b) {
    __shared__ int red[32];
    int s = 0;
    for (int j = threadIdx.x; j < b; j += blockDim.x) s += tiles[j];
    s = warp_sum_i(s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    int tot = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
    __syncthreads();
    return tot;
}

__global__ void k_cl_node_scatter(const int* n_dev, int64_t n_ub, int ntiles_ub, lw_cluster_buf cb) {
    __shared__ int sm[33];
    int64_t n = n_dev ? (int64_t)*n_dev : n_ub;
    if (n > n_ub) n = n_ub;
    int64_t i = (int64_t)blockIdx.x * CTILE + threadIdx.x;
    int f = 0, s = -1;
    if (i < n) {
        s = cb.slot_of_pt[i];
        f = (s >= 0 && cb.first[s] == (int)i) ? 1 : 0;
    }
    int base = tiles_before(cb.tiles, blockIdx.x);
    int tot;
    int r = block_rank(f, sm, &tot);
    if (f) {
        int j = base + r;
        cb.node_slot[j] = s;
        cb.vidx[s] = j;
        const int64_t* acc = cb.acc + 4 * (int64_t)s;
        double w = (double)acc[3];
        cb.v_xyz[3 * (int64_t)j + 0] = (float)((double)acc[0] / (w * LW_FIX_W));
        cb.v_xyz[3 * (int64_t)j + 1] = (float)((double)acc[1] / (w * LW_FIX_W));
        cb.v_xyz[3 * (int64_t)j + 2] = (float)((double)acc[2] / (w * LW_FIX_W));
        cb.v_w[j] = (int)acc[3];
    }
    (void)ntiles_ub;
}

__global__ void k_cl_node_total(const int* tiles, int nt, int* m_dev) {
    int s = 0;
    for (int j = threadIdx.x; j < nt; j += blockDim.x) s += tiles[j];
    s = warp_sum_i(s);
    __shared__ int red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        *m_dev = t;
    }
}

// Neighbours of node j: nodes whose centroid lies within connect, found through the voxel hash within `reach`
// voxels (a centroid lies inside its voxel, so no neighbour is farther). Counted, then written in probe order.
// A warp serves one node: its lanes probe 32 consecutive offsets at a time (independent hash lookups in flight)
// and a ballot ranks the hits, so the edges land in the same ascending probe order a serial walk gives.
template <bool WRITE>
__global__ void k_cl_edges(ClArgs a, lw_cluster_buf cb, int64_t m_ub) {
    int m = *cb.m;
    if (m > m_ub) m = (int)m_ub;
    const int S = 2 * a.reach + 1, N = S * S * S;
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int j = warp; j < m; j += nwarps) {
        float px = cb.v_xyz[3 * j], py = cb.v_xyz[3 * j + 1], pz = cb.v_xyz[3 * j + 2];
        int64_t key = cb.keys[cb.node_slot[j]];
        int ix = (int)(key & KEY_MASK) - (int)KEY_BIAS;
        int iy = (int)((key >> 21) & KEY_MASK) - (int)KEY_BIAS;
        int iz = (int)((key >> 42) & KEY_MASK) - (int)KEY_BIAS;
        int cnt = 0;
        const int out = WRITE ? cb.edge_off[j] : 0;
        for (int o0 = 0; o0 < N; o0 += 32) {
            const int o = o0 + lane;
            int k = -1;
            if (o < N) {
                int dz = o % S - a.reach, dy = (o / S) % S - a.reach, dx = o / (S * S) - a.reach;
                if (dx != 0 || dy != 0 || dz != 0) {
                    int s = find_slot(key_ijk(ix + dx, iy + dy, iz + dz), cb.keys, a.mask);
                    if (s >= 0) {
                        int c = cb.vidx[s];
                        float ex = cb.v_xyz[3 * c] - px, ey = cb.v_xyz[3 * c + 1] - py, ez = cb.v_xyz[3 * c + 2] - pz;
                        if (ex * ex + ey * ey + ez * ez <= a.connect2) k = c;
                    }
                }
            }
            const unsigned hits = __ballot_sync(0xffffffffu, k >= 0);
            if (WRITE && k >= 0) {
                const int e = out + cnt + __popc(hits & below);
                if (e < cb.edge_cap)
                    cb.edges[e] = k;
                else
                    atomicExch(cb.err, 2);  // edge buffer too small: reported, never overrun
            }
            cnt += __popc(hits);
        }
        if (!WRITE && lane == 0) cb.edge_off[j] = cnt;
    }
}

// Exclusive scan of the m per-node edge counts in place (one CTA), edge_off[m] = total.
__global__ void k_cl_scan_edges(lw_cluster_buf cb, int64_t m_ub) {
    __shared__ int sm[33];
    __shared__ int carry;
    int m = *cb.m;
    if (m > m_ub) m = (int)m_ub;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < m; base += blockDim.x) {
        int j = base + threadIdx.x;
        int v = j < m ? cb.edge_off[j] : 0;
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
            int x = lane < nw ? sm[lane] : 0, xi = x;
            for (int o = 1; o < 32; o <<= 1) {
                int u = __shfl_up_sync(0xffffffffu, xi, o);
                if (lane >= o) xi += u;
            }
            if (lane < nw) sm[lane] = xi - x;
            if (lane == 31) sm[32] = xi;
        }
        __syncthreads();
        if (j < m) cb.edge_off[j] = carry + sm[w] + inc - v;
        __syncthreads();
        if (threadIdx.x == 0) carry += sm[32];
        __syncthreads();
    }
    if (threadIdx.x == 0) cb.edge_off[m] = carry;
}

constexpr int UF_SPINS = 1 << 20;

__device__ __forceinline__ int uf_find(int* parent, int x) {
    for (int it = 0; it < UF_SPINS; ++it) {
        int p = parent[x];
        if (p == x) return x;
        int gp = parent[p];
        if (gp != p) atomicMin(parent + x, gp);  // path halving; never raises a parent
        x = p;
    }
    return x;
}

__global__ void k_cl_uf_init(lw_cluster_buf cb, int64_t m_ub) {
    int m = *cb.m;
    if (m > m_ub) m = (int)m_ub;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) cb.label[j] = j;
}

// Hook the larger root under the smaller one for every edge; a CAS that loses a race retries with the new roots.
// Every component ends rooted at its smallest node whatever order the hooks land in, so a warp serves a node
// and its lanes take the node's edges side by side.
__global__ void k_cl_uf_union(lw_cluster_buf cb, int64_t m_ub) {
    int m = *cb.m;
    if (m > m_ub) m = (int)m_ub;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int j = warp; j < m; j += nwarps) {
        int e0 = cb.edge_off[j], e1 = cb.edge_off[j + 1];
        if (e1 > cb.edge_cap) e1 = (int)cb.edge_cap;
        for (int e = e0 + lane; e < e1; e += 32) {
            int k = cb.edges[e];
            if (k <= j) continue;  // every undirected edge once
            int a = j, b = k;
            for (int it = 0; it < UF_SPINS; ++it) {
                a = uf_find(cb.label, a);
                b = uf_find(cb.label, b);
                if (a == b) break;
                if (a < b) {
                    int t = a;
                    a = b;
                    b = t;
                }
                if (atomicCAS(cb.label + a, a, b) == a) break;
                if (it == UF_SPINS - 1) atomicExch(cb.err, 1);
            }
        }
    }
}

__global__ void k_cl_uf_flatten(lw_cluster_buf cb, int64_t m_ub) {
    int m = *cb.m;
    if (m > m_ub) m = (int)m_ub;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x)
        cb.label[j] = uf_find(cb.label, j);
}

// Per-root statistics: exact fixed-point sums and point counts, float min / max of the node centroids.
__global__ void k_cl_stats(lw_cluster_buf cb, int64_t m_ub) {
    int m = *cb.m;
    if (m > m_ub) m = (int)m_ub;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) {
        int r = cb.label[j];
        const int64_t* acc = cb.acc + 4 * (int64_t)cb.node_slot[j];
        atomic_add_i64(cb.st_sum + 4 * (int64_t)r + 0, acc[0]);
        atomic_add_i64(cb.st_sum + 4 * (int64_t)r + 1, acc[1]);
        atomic_add_i64(cb.st_sum + 4 * (int64_t)r + 2, acc[2]);
        atomic_add_i64(cb.st_sum + 4 * (int64_t)r + 3, acc[3]);
        for (int d = 0; d < 3; ++d) {
            float v = cb.v_xyz[3 * j + d];
            atomic_min_float(cb.st_lo + 3 * (int64_t)r + d, v);
            atomic_max_float(cb.st_hi + 3 * (int64_t)r + d, v);
        }
    }
}

// Dense ids for the roots with at least min_pts points, in node order (<= max_out of them).
__global__ void k_cl_flag(lw_cluster_buf cb, ClArgs a, int64_t m_ub) {
    int m = *cb.m;
    if (m > m_ub) m = (int)m_ub;
    int j = blockIdx.x * CTILE + threadIdx.x;
    int f = 0;
    if (j < m) f = (cb.label[j] == j && (float)cb.st_sum[4 * (int64_t)j + 3] >= a.min_pts) ? 1 : 0;
    int c = __syncthreads_count(f);
    if (threadIdx.x == 0) cb.tiles[blockIdx.x] = c;
}

__global__ void k_cl_compact(lw_cluster_buf cb, ClArgs a, int64_t m_ub) {
    __shared__ int sm[33];
    int m = *cb.m;
    if (m > m_ub) m = (int)m_ub;
    int j = blockIdx.x * CTILE + threadIdx.x;
    int f = 0;
    if (j < m) f = (cb.label[j] == j && (float)cb.st_sum[4 * (int64_t)j + 3] >= a.min_pts) ? 1 : 0;
    int base = tiles_before(cb.tiles, blockIdx.x);
    int tot;
    int r = block_rank(f, sm, &tot);
    if (j < m) cb.dense[j] = -1;
    if (f) {
        int d = base + r;
        if (d < a.max_out) {
            cb.dense[j] = d;
            const int64_t* su = cb.st_sum + 4 * (int64_t)j;
            double w = (double)su[3];
            cb.out_cnt[d] = (float)su[3];
            for (int k = 0; k < 3; ++k) {
                cb.out_cen[3 * d + k] = (float)((double)su[k] / (w * LW_FIX_W));
                cb.out_lo[3 * d + k] = cb.st_lo[3 * (int64_t)j + k];
                cb.out_hi[3 * d + k] = cb.st_hi[3 * (int64_t)j + k];
            }
        }
    }
}

__global__ void k_cl_count(lw_cluster_buf cb, int nt, ClArgs a) {
    int s = 0;
    for (int j = threadIdx.x; j < nt; j += blockDim.x) s += cb.tiles[j];
    s = warp_sum_i(s);
    __shared__ int red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        cb.n_clusters[0] = t < a.max_out ? t : a.max_out;
        cb.n_clusters[1] = t;  // before the cap
    }
}

// Per point: its cluster id (or -1), then put the voxel table and the per-root stats back for the next call.
__global__ void k_cl_gather(const int* n_dev, int64_t n_ub, lw_cluster_buf cb, int* __restrict__ out_cid) {
    int64_t n = n_dev ? (int64_t)*n_dev : n_ub;
    if (n > n_ub) n = n_ub;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int s = cb.slot_of_pt[i];
        out_cid[i] = s < 0 ? -1 : cb.dense[cb.label[cb.vidx[s]]];
    }
}

__global__ void k_cl_reset(lw_cluster_buf cb, int64_t m_ub) {
    int m = *cb.m;
    if (m > m_ub) m = (int)m_ub;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) {
        int s = cb.node_slot[j];
        cb.keys[s] = EMPTY_KEY;
        cb.first[s] = NO_INDEX;
        for (int k = 0; k < 4; ++k) cb.acc[4 * (int64_t)s + k] = 0;
        for (int k = 0; k < 4; ++k) cb.st_sum[4 * (int64_t)j + k] = 0;
        for (int k = 0; k < 3; ++k) {
            cb.st_lo[3 * (int64_t)j + k] = 1.0e30f;
            cb.st_hi[3 * (int64_t)j + k] = -1.0e30f;
        }
    }
}

}  // namespace lw

using namespace lw;

extern "C" {

int lw_ground(const float* xyz, int32_t xyz_stride, const float* nrm, const int32_t* n_dev, int64_t n_ub, float cell,
              float thick, int32_t min_sup, float thresh, float slope_step, int32_t use_normals, float nz_min,
              float* cell_min, int32_t* cell_sup, int32_t* out_gnd, float* out_hag, void* stream) {
    if (!xyz || !cell_min || !cell_sup || !out_gnd || !out_hag || (use_normals && !nrm) ||
        (xyz_stride != 3 && xyz_stride != 4))
        return set_error(LW_EINVAL, "lw_ground: bad arguments");
    if (n_ub <= 0) return LW_OK;
    cudaStream_t s = (cudaStream_t)stream;
    GroundArgs a;
    a.inv_cell = 1.0f / fmaxf(cell, 0.05f);
    a.thick = thick;
    a.thresh = thresh;
    a.slope_step = slope_step;
    a.nz_min = nz_min;
    a.min_sup = min_sup;
    a.use_nrm = use_normals ? 1 : 0;
    int grid = blocks_for(n_ub, 256, 8 * device_sms());
    ProfScope prof("ground", s);
    if (xyz_stride == 4) {
        k_gnd_min<4><<<grid, 256, 0, s>>>(xyz, n_dev, n_ub, a, cell_min);
        k_gnd_support<4><<<grid, 256, 0, s>>>(xyz, n_dev, n_ub, a, cell_min, cell_sup);
        k_gnd_label<4><<<grid, 256, 0, s>>>(xyz, nrm, n_dev, n_ub, a, cell_min, cell_sup, out_gnd, out_hag);
        k_gnd_reset<4><<<grid, 256, 0, s>>>(xyz, n_dev, n_ub, a, cell_min, cell_sup);
    } else {
        k_gnd_min<3><<<grid, 256, 0, s>>>(xyz, n_dev, n_ub, a, cell_min);
        k_gnd_support<3><<<grid, 256, 0, s>>>(xyz, n_dev, n_ub, a, cell_min, cell_sup);
        k_gnd_label<3><<<grid, 256, 0, s>>>(xyz, nrm, n_dev, n_ub, a, cell_min, cell_sup, out_gnd, out_hag);
        k_gnd_reset<3><<<grid, 256, 0, s>>>(xyz, n_dev, n_ub, a, cell_min, cell_sup);
    }
    LW_LAUNCHED("lw_ground");
    count_launches(4);
    return LW_OK;
}

int lw_cluster(const float* xyz, int32_t xyz_stride, const int32_t* gnd, int32_t use_ground, const int32_t* n_dev,
               int64_t n_ub, float voxel, float connect, float min_pts, int32_t max_out, lw_cluster_buf* cb,
               int32_t* out_cid, void* stream) {
    if (!xyz || !cb || !out_cid || (use_ground && !gnd) || (xyz_stride != 3 && xyz_stride != 4))
        return set_error(LW_EINVAL, "lw_cluster: bad arguments");
    if ((cb->cap & (cb->cap - 1)) != 0) return set_error(LW_EINVAL, "lw_cluster: table capacity not a power of two");
    if (n_ub > cb->pt_cap) return set_error(LW_ECAPACITY, "lw_cluster: %lld points exceed the buffers' %lld",
                                           (long long)n_ub, (long long)cb->pt_cap);
    if (n_ub <= 0) return LW_OK;
    cudaStream_t s = (cudaStream_t)stream;
    ClArgs a;
    a.inv_v = 1.0f / fmaxf(voxel, 0.01f);
    a.mask = (int)(cb->cap - 1);
    a.use_gnd = use_ground ? 1 : 0;
    a.connect2 = connect * connect;
    a.reach = (int)ceilf(connect * a.inv_v);
    if (a.reach < 1) a.reach = 1;
    if (a.reach > 4) return set_error(LW_EINVAL, "lw_cluster: connect / voxel = %g needs a %d-voxel reach (max 4)",
                                      (double)(connect * a.inv_v), a.reach);
    a.min_pts = min_pts;
    a.max_out = max_out;
    const int64_t m_ub = n_ub;  // at most one node per point
    const int sms = device_sms();
    int grid = blocks_for(n_ub, 256, 8 * sms);
    int gridw = blocks_for(m_ub * 32, 256, 16 * sms);  // a warp per node
    int nt = blocks_for(n_ub, CTILE);
    ProfScope prof("cluster", s);
    if (xyz_stride == 4)
        k_cl_insert<4><<<grid, 256, 0, s>>>(xyz, gnd, n_dev, n_ub, a, *cb);
    else
        k_cl_insert<3><<<grid, 256, 0, s>>>(xyz, gnd, n_dev, n_ub, a, *cb);
    k_cl_node_count<<<nt, CTILE, 0, s>>>(n_dev, n_ub, *cb);
    k_cl_node_scatter<<<nt, CTILE, 0, s>>>(n_dev, n_ub, nt, *cb);
    k_cl_node_total<<<1, 256, 0, s>>>(cb->tiles, nt, cb->m);
    k_cl_edges<false><<<gridw, 256, 0, s>>>(a, *cb, m_ub);
    k_cl_scan_edges<<<1, 1024, 0, s>>>(*cb, m_ub);
    k_cl_edges<true><<<gridw, 256, 0, s>>>(a, *cb, m_ub);
    k_cl_uf_init<<<grid, 256, 0, s>>>(*cb, m_ub);
    k_cl_uf_union<<<gridw, 256, 0, s>>>(*cb, m_ub);
    k_cl_uf_flatten<<<grid, 256, 0, s>>>(*cb, m_ub);
    k_cl_stats<<<grid, 256, 0, s>>>(*cb, m_ub);
    k_cl_flag<<<nt, CTILE, 0, s>>>(*cb, a, m_ub);
    k_cl_compact<<<nt, CTILE, 0, s>>>(*cb, a, m_ub);
    k_cl_count<<<1, 256, 0, s>>>(*cb, nt, a);
    k_cl_gather<<<grid, 256, 0, s>>>(n_dev, n_ub, *cb, out_cid);
    k_cl_reset<<<grid, 256, 0, s>>>(*cb, m_ub);
    LW_LAUNCHED("lw_cluster");
    count_launches(16);
    return LW_OK;
}

}  // extern "C"
