// Odometry hot path on sm_100a: frame cutting, deskew, half-voxel thinning, the registration voxel map with
// per-voxel distribution records, scan-to-map point-to-distribution Gauss-Newton (accumulate on every SM,
// float64 6x6 solve on the device), and the per-frame state machine of odom.py (warm-up, re-deskew,
// keyframes, constant-velocity prediction) -- all without a host round trip.
//
// Reference: python/livox_warp/odom.py (kernels :97-384, host solve :387-455, Odometry :458-803) and the key /
// hash / deskew helpers of python/livox_warp/gpu.py (:231-283).
#include <mutex>
#include "lw_common.cuh"
#include "lw_linalg.cuh"
#include "lw_net.cuh"

namespace lw {

constexpr int TILE = 1024;

// =====================================================================================================
// Frame append (odom.py:97-123): order-preserving compaction of the staged points that belong to the open
// frame. Three launches: per-tile counts, scatter at (count + prefix of tiles), count update.
// =====================================================================================================

__device__ __forceinline__ int frame_of(float t, float inv_dt) { return (int)floorf(fmaxf(t, 0.0f) * inv_dt); }

__global__ void k_append_count(const float* __restrict__ t, int64_t n, float inv_dt, int k_min, int k_open,
                               int* __restrict__ tiles) {
    int64_t i = (int64_t)blockIdx.x * TILE + threadIdx.x;
    int f = 0;
    if (i < n) {
        int k = frame_of(t[i], inv_dt);
        f = (k <= k_open && k >= k_min) ? 1 : 0;
    }
    int c = __syncthreads_count(f);
    if (threadIdx.x == 0) tiles[blockIdx.x] = c;
}

__device__ __forceinline__ int prefix_of_tiles(const int* __restrict__ tiles, int b) {
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

template <int STRIDE>
__global__ void k_append_scatter(const float* __restrict__ xyz, const uint32_t* __restrict__ attr,
                                 const float* __restrict__ t, int64_t n, float inv_dt, int k_min, int k_open,
                                 const int* __restrict__ tiles, lw_frame_buf fb) {
    __shared__ int sm[33];
    int64_t i = (int64_t)blockIdx.x * TILE + threadIdx.x;
    int f = 0;
    float ti = 0.0f;
    if (i < n) {
        ti = t[i];
        int k = frame_of(ti, inv_dt);
        f = (k <= k_open && k >= k_min) ? 1 : 0;
    }
    int base = *fb.count + prefix_of_tiles(tiles, blockIdx.x);
    int tot;
    int r = block_rank(f, sm, &tot);
    if (f) {
        int64_t pos = (int64_t)base + r;
        if (pos < fb.cap) {
            float4 v = make_float4(xyz[i * STRIDE + 0], xyz[i * STRIDE + 1], xyz[i * STRIDE + 2], ti);
            reinterpret_cast<float4*>(fb.f_raw)[pos] = v;
            fb.f_attr[pos] = attr[i];
            fb.f_t[pos] = ti;
            fb.f_frame[pos] = k_open;  // the frame it is deskewed, registered and posed with (odom.py:123)
        }
    }
}

__global__ void k_append_total(const int* __restrict__ tiles, int nt, int* count) {
    int s = 0;
    for (int j = threadIdx.x; j < nt; j += blockDim.x) s += tiles[j];
    s = warp_sum_i(s);
    __shared__ int red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int tot = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
        *count += tot;
    }
}

// =====================================================================================================
// Deskew (odom.py:163-178 with gpu.py:268-283): s = clamp((t - t_mid) / frame_dt, -1, 1), then deskew_frac.
// =====================================================================================================

__device__ __forceinline__ float4 deskew_point(float4 p, float t_mid, float inv_dt, const float* tw) {
    float s = fminf(fmaxf((p.w - t_mid) * inv_dt, -1.0f), 1.0f);
    float ox, oy, oz;
    deskew_frac(p.x, p.y, p.z, s, tw, ox, oy, oz);
    return make_float4(ox, oy, oz, p.w);
}

// =====================================================================================================
// Thinning (odom.py:126-160): keep the lowest-index point of every half-voxel of the (deskewed) sensor frame.
// Pass A (fused with deskew) claims keys and records the lowest index per slot; pass B marks the winners and
// counts them per tile; pass C writes them in point order and clears the table for the next frame.
// =====================================================================================================

struct ThinArgs {
    float inv_v, min_range, max_range;
    int ret_mask;
    int deskew;      // 1: pass A deskews f_raw into f_xyz first
    float t_mid, inv_dt;
};

// The frame's point count and twist come from the state when `st` is set, else from the arguments.
struct Tw6 {
    float v[6];
};

struct RegBegin {
    double T[16];
    double t_mid;
    float tw[6];
    int m;
};

// What a single-frame registration sets up before its first pass (lw_register_frame), done by block 0 of the first
// thinning pass instead of kernels of its own: the registration's start state, and the Gauss-Newton launch's
// fixed-point accumulators and barrier count cleared. With `on`, the pass takes its point count from `m`.
struct ThinBegin {
    lw_odom_state* st;
    long long* part;  // [3 * LW_ACC_STRIDE] to clear
    uint32_t* bar;    // [2] to clear
    RegBegin b;
    int on;
};

__device__ __forceinline__ void reg_begin(lw_odom_state* st, const RegBegin& b) {
    const int t = threadIdx.x;
    if (t < 16) st->T_pred[t] = b.T[t];
    if (t < 6) st->xi_used[t] = b.tw[t];
    if (t < 16) st->T_reg[t] = b.T[t];  // what a registration that gives up leaves: the prediction, not ok
    if (t == 0) {
        st->t_mid = b.t_mid;
        st->m = b.m;
        st->n_ds = 0;
        st->ok = 0;
        st->iters = 0;
        st->corr = 0;
    }
}

__global__ void k_thin_a(lw_frame_buf fb, const int* __restrict__ m_dev, ThinArgs a, const lw_odom_state* st,
                         Tw6 tw_arg, const int* gate_deskew, const int* gate_thin, int thin_on, ThinBegin bg) {
    if (bg.on && blockIdx.x == 0) {
        reg_begin(bg.st, bg.b);
        for (int e = threadIdx.x; e < 3 * LW_ACC_STRIDE; e += blockDim.x) bg.part[e] = 0;
        if (threadIdx.x < 2) bg.bar[threadIdx.x] = 0;
    }
    if (gate_deskew && *gate_deskew == 0) return;
    const bool thin = thin_on && !(gate_thin && *gate_thin == 0);
    int64_t m = bg.on ? (int64_t)bg.b.m : (int64_t)*m_dev;
    if (m > fb.cap) m = fb.cap;
    float tw[6];
    float t_mid = a.t_mid;
    if (st) {
#pragma unroll
        for (int k = 0; k < 6; ++k) tw[k] = st->xi_used[k];
        t_mid = (float)st->t_mid;
    } else {
#pragma unroll
        for (int k = 0; k < 6; ++k) tw[k] = tw_arg.v[k];
    }
    const int mask = (int)(fb.ds_cap - 1);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        float4 p;
        if (a.deskew) {
            p = deskew_point(reinterpret_cast<const float4*>(fb.f_raw)[i], t_mid, a.inv_dt, tw);
            reinterpret_cast<float4*>(fb.f_xyz)[i] = p;
        } else {
            p = reinterpret_cast<const float4*>(fb.f_xyz)[i];
        }
        if (!thin) continue;
        int slot = -1;
        float r = len3(p.x, p.y, p.z);
        uint32_t at = fb.f_attr[i];
        if (!(r < a.min_range || r > a.max_range) && tag_of(at) == 0 && ((1 << ret_of(at)) & a.ret_mask) != 0) {
            int64_t key = key_ijk(ifloor(p.x * a.inv_v), ifloor(p.y * a.inv_v), ifloor(p.z * a.inv_v));
            bool claimed;
            slot = claim_slot(key, fb.ds_keys, mask, &claimed);
            if (slot >= 0) atomicMin(fb.ds_win + slot, (int)i);
        }
        fb.ds_slot[i] = slot;
    }
}

__global__ void k_thin_b(lw_frame_buf fb, const int* __restrict__ m_dev, const int* gate) {
    if (gate && *gate == 0) return;
    int64_t m = *m_dev;
    if (m > fb.cap) m = fb.cap;
    int64_t i = (int64_t)blockIdx.x * TILE + threadIdx.x;
    if ((int64_t)blockIdx.x * TILE >= m) return;  // whole tile past the frame
    int keep = 0;
    if (i < m) {
        int s = fb.ds_slot[i];
        keep = (s >= 0 && fb.ds_win[s] == (int)i) ? 1 : 0;
        if (!keep) fb.ds_slot[i] = -1;
    }
    int c = __syncthreads_count(keep);
    if (threadIdx.x == 0) fb.tiles[blockIdx.x] = c;
}

__global__ void k_thin_c(lw_frame_buf fb, const int* __restrict__ m_dev, int* n_ds, const int* gate) {
    if (gate && *gate == 0) return;
    __shared__ int sm[33];
    int64_t m = *m_dev;
    if (m > fb.cap) m = fb.cap;
    const int ntiles = (int)((m + TILE - 1) / TILE);
    if ((int)blockIdx.x >= ntiles) {
        if (blockIdx.x == gridDim.x - 1 && ntiles == 0 && threadIdx.x == 0) *n_ds = 0;
        return;
    }
    int64_t i = (int64_t)blockIdx.x * TILE + threadIdx.x;
    int s = -1;
    if (i < m) s = fb.ds_slot[i];
    int keep = s >= 0;
    int base = prefix_of_tiles(fb.tiles, blockIdx.x);
    int tot;
    int r = block_rank(keep, sm, &tot);
    if (keep) {
        float4 p = reinterpret_cast<const float4*>(fb.f_xyz)[i];
        reinterpret_cast<float4*>(fb.ds_xyz)[base + r] = make_float4(p.x, p.y, p.z, len3(p.x, p.y, p.z));
        fb.ds_keys[s] = EMPTY_KEY;  // each claimed slot has exactly one winner: it clears the slot
        fb.ds_win[s] = NO_INDEX;
    }
    if ((int)blockIdx.x == ntiles - 1 && threadIdx.x == 0) *n_ds = base + tot;
}

// =====================================================================================================
// Registration map (odom.py:186-230): per voxel the count and exact fixed-point sums of r = w - centre and
// r r^T. Deterministic: the slot content does not depend on thread order, and the 4096-point cap takes the
// first points in index order. Pass D refreshes the record the ICP reads (odom.py:320-368 hoisted out of the
// per-point loop: a voxel's mean and precision only change when it is inserted into).
// =====================================================================================================

struct RegArgs {
    float T[12];  // float row-major 3x4 pose
    float inv_v, voxel, max_range;
    int ret_mask;
};

__device__ __forceinline__ void reg_point(const RegArgs& a, float4 p, int& ix, int& iy, int& iz, float& rx,
                                          float& ry, float& rz) {
    float wx, wy, wz;
    xform(a.T, p.x, p.y, p.z, wx, wy, wz);
    ix = ifloor(wx * a.inv_v);
    iy = ifloor(wy * a.inv_v);
    iz = ifloor(wz * a.inv_v);
    rx = wx - ((float)ix + 0.5f) * a.voxel;
    ry = wy - ((float)iy + 0.5f) * a.voxel;
    rz = wz - ((float)iz + 0.5f) * a.voxel;
}

__device__ __forceinline__ void reg_add(lw_regmap& reg, int s, float rx, float ry, float rz) {
    const float FR = (float)LW_FIX_R, FRR = (float)LW_FIX_RR;
    atomic_add_i64(reg.sum + 3 * s + 0, to_fix(rx, FR));
    atomic_add_i64(reg.sum + 3 * s + 1, to_fix(ry, FR));
    atomic_add_i64(reg.sum + 3 * s + 2, to_fix(rz, FR));
    atomic_add_i64(reg.outer + 6 * s + 0, to_fix(rx * rx, FRR));
    atomic_add_i64(reg.outer + 6 * s + 1, to_fix(rx * ry, FRR));
    atomic_add_i64(reg.outer + 6 * s + 2, to_fix(rx * rz, FRR));
    atomic_add_i64(reg.outer + 6 * s + 3, to_fix(ry * ry, FRR));
    atomic_add_i64(reg.outer + 6 * s + 4, to_fix(ry * rz, FRR));
    atomic_add_i64(reg.outer + 6 * s + 5, to_fix(rz * rz, FRR));
}

// RegArgs from a float64 pose held on the device (the odometry state) or given by the host.
__device__ __forceinline__ void reg_args_pose(RegArgs& a, const double* T_dev) {
    if (T_dev)
        for (int k = 0; k < 12; ++k) a.T[k] = (float)T_dev[k];
}

__device__ __forceinline__ bool reg_keep(float4 p, uint32_t at, const RegArgs& a) {
    return !(len3(p.x, p.y, p.z) > a.max_range || tag_of(at) != 0 || ((1 << ret_of(at)) & a.ret_mask) == 0);
}

__global__ void k_reg_a(const float4* __restrict__ xyz, const uint32_t* __restrict__ attr, const int* n_dev,
                        int64_t n_ub, RegArgs a, const double* T_dev, lw_regmap reg, int* __restrict__ pslot,
                        const int* gate) {
    if (gate && *gate == 0) return;
    reg_args_pose(a, T_dev);
    int64_t n = n_dev ? (int64_t)*n_dev : n_ub;
    if (n > n_ub) n = n_ub;
    const int mask = (int)(reg.cap - 1);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float4 p = xyz[i];
        int s = -1;
        if (reg_keep(p, attr[i], a)) {
            int ix, iy, iz;
            float rx, ry, rz;
            reg_point(a, p, ix, iy, iz, rx, ry, rz);
            bool claimed;
            s = claim_slot(key_ijk(ix, iy, iz), reg.keys, mask, &claimed);
            if (claimed) atomicAdd(reg.stats + 0, 1);
            if (s < 0) {
                atomicAdd(reg.stats + 1, 1);
            } else {
                atomicAdd(reg.bcnt + s, 1);
                atomicMin(reg.first + s, (int)i);
            }
        }
        pslot[i] = s;
    }
}

__global__ void k_reg_b(const float4* __restrict__ xyz, const int* n_dev, int64_t n_ub, RegArgs a, const double* T_dev,
                        lw_regmap reg, const int* __restrict__ pslot, const int* gate) {
    if (gate && *gate == 0) return;
    reg_args_pose(a, T_dev);
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
            pre = reg.cnt[s];
            if (pre + reg.bcnt[s] <= LW_REG_CAP) {
                int ix, iy, iz;
                float rx, ry, rz;
                reg_point(a, xyz[i], ix, iy, iz, rx, ry, rz);
                reg_add(reg, s, rx, ry, rz);
            } else {
                lead = pre < LW_REG_CAP && reg.first[s] == (int)i;
            }
        }
        // this batch crosses the cap: the voxel adds its first (cap - pre) points in index order
        for (unsigned lm = __ballot_sync(0xffffffffu, lead); lm; lm &= lm - 1) {
            int src = __ffs(lm) - 1;
            int sl = __shfl_sync(0xffffffffu, s, src);
            int room = LW_REG_CAP - __shfl_sync(0xffffffffu, pre, src);
            warp_fill_first(pslot, base + src, n, sl, room, [&](int64_t j) {
                int ix, iy, iz;
                float rx, ry, rz;
                reg_point(a, xyz[j], ix, iy, iz, rx, ry, rz);
                reg_add(reg, sl, rx, ry, rz);
            });
        }
    }
}

// The derived record of one voxel (odom.py:325-368): the mean in world coordinates and the precision matrices
// M (all directions) and Mg (surface-normal directions only), plus the direction the metric rms is measured
// along. Evaluated in float64 from the exact sums.
__device__ void reg_record(lw_regmap& reg, int s, const lw_rec_params& rp) {
    float* out = reg.rec + (int64_t)s * LW_REC_FLOATS;
    int c = reg.cnt[s];
    if (c <= 0) {
        for (int k = 0; k < LW_REC_FLOATS; ++k) out[k] = 0.0f;
        return;
    }
    int64_t key = reg.keys[s];
    int ix = (int)(key & KEY_MASK) - (int)KEY_BIAS;
    int iy = (int)((key >> 21) & KEY_MASK) - (int)KEY_BIAS;
    int iz = (int)((key >> 42) & KEY_MASK) - (int)KEY_BIAS;
    double cf = (double)c;
    double mr[3], C[9];
    for (int k = 0; k < 3; ++k) mr[k] = (double)reg.sum[3 * s + k] / (cf * LW_FIX_R);
    const int up[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C[i * 3 + j] = (double)reg.outer[6 * s + up[i * 3 + j]] / (cf * LW_FIX_RR) - mr[i] * mr[j];
    double vox = (double)rp.voxel;
    out[0] = (float)(((double)ix + 0.5) * vox + mr[0]);
    out[1] = (float)(((double)iy + 0.5) * vox + mr[1]);
    out[2] = (float)(((double)iz + 0.5) * vox + mr[2]);
    out[3] = (float)c;
    double ev[3], Q[9];
    jacobi_eig<3>(C, ev, Q);
    double tight2 = rp.tight2, noise2 = rp.noise2, alpha = rp.alpha;
    int nt = 0;
    for (int k = 0; k < 3; ++k) nt += ev[k] < tight2 ? 1 : 0;
    double M[6] = {0, 0, 0, 0, 0, 0}, Mg[6] = {0, 0, 0, 0, 0, 0}, q[3] = {0, 0, 0};
    float surf = 0.0f;
    if (c >= 5 && nt <= 1) {
        int kmin = 0;
        if (ev[1] < ev[kmin]) kmin = 1;
        if (ev[2] < ev[kmin]) kmin = 2;
        for (int k = 0; k < 3; ++k) {
            double qa[3] = {Q[0 * 3 + k], Q[1 * 3 + k], Q[2 * 3 + k]};
            double e = fmax(ev[k], 0.0) + noise2;
            double wa = 1.0 / e;
            bool tight = !(ev[k] >= tight2);
            if (!tight) wa = alpha / e;  // a direction the surface extends along: a weak pull only
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
        double wa = alpha / (0.25 * vox * vox + noise2);  // too few points, or a line / blob: weak isotropic pull
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

__global__ void k_reg_d(const int* n_dev, int64_t n_ub, lw_regmap reg, const int* __restrict__ pslot,
                        lw_rec_params rp, const int* gate) {
    if (gate && *gate == 0) return;
    int64_t n = n_dev ? (int64_t)*n_dev : n_ub;
    if (n > n_ub) n = n_ub;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int s = pslot[i];
        if (s < 0 || reg.first[s] != (int)i) continue;
        int tot = reg.cnt[s] + reg.bcnt[s];
        reg.cnt[s] = tot < LW_REG_CAP ? tot : LW_REG_CAP;
        reg.bcnt[s] = 0;
        reg.first[s] = NO_INDEX;
        reg_record(reg, s, rp);
    }
}

__global__ void k_reg_refresh_all(lw_regmap reg, lw_rec_params rp) {
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < reg.cap; s += (int64_t)gridDim.x * blockDim.x)
        if (reg.keys[s] != EMPTY_KEY) reg_record(reg, (int)s, rp);
}

// =====================================================================================================
// Gauss-Newton accumulation (odom.py:275-375). A group of G = 8 lanes serves one thinned point: the lanes split the
// (2 reach + 1)^3 neighbour voxels between them, B probes in flight per lane (B = 8: two batches of independent
// loads cover the 125 voxels of the wide search; B = 4: one batch the 27 of the narrow one; with 4736 groups a
// frame's points need a single round), reduce to the closest mean in reference order by shuffles, and then split
// the point's 53 weighted terms between them by column pairs of H and Hg (term_slot), from the matched voxel's
// record that every lane reads. The Jacobian is
// taken about a point near the frame (the predicted sensor position) so float32 keeps its precision far from the
// world origin; the float64 reduction maps H, b and Hg back to the reference's twist about the world origin.
// =====================================================================================================

constexpr int GN_THREADS = 256;
constexpr int NTERMS = 53;

struct IcpPose {
    float R[9];   // rotation
    float tr[3];  // translation minus the centre c
    float c[3];   // centre (world)
};

struct IcpConsts {
    float inv_v, max_d2, kappa2, inv_kappa2;
    int reach, mask;
};

// A launch-long memo, in shared memory, of what the first point of each group read from global memory. Within one
// Gauss-Newton launch the map and the thinned points do not change, and a point moves by millimetres between
// iterations. The memo keeps the group's point, the 5 x 5 x 5 window of hash slots and means that its last wide
// search gathered around base voxel `tag`, and the record of its last matched voxel. A wide search from the same
// base voxel, and every narrow search whose 3 x 3 x 3 neighbourhood lies inside the window (base voxel within one of
// the tag's), then reads shared memory instead of making dependent global loads -- the same values, so the sums
// are exactly those of the uncached pass.
constexpr int GN_GROUPS = GN_THREADS / 8;
constexpr int WIN = 128;  // 5^3 = 125 window entries per group, padded
struct IcpCache {
    float4* mean;  // [GN_GROUPS][WIN] means (x, y, z, occupancy weight) of the window's slots
    float4* brec;  // [GN_GROUPS][5] the record of the group's last matched voxel
    float4* pt;    // [GN_GROUPS] the group's first point
    int4* tag;     // [GN_GROUPS] the window's base voxel (x, y, z); w = 0: no window yet
    int* slot;     // [GN_GROUPS][WIN] the window's slots (-1: not in the map), offset (dx + 2) 25 + (dy + 2) 5 + dz + 2
    int* best;     // [GN_GROUPS] the group's last matched slot (-1: none)
    int pt_ok;     // pt holds the points (every pass after the launch's first)
};
constexpr size_t GN_DYN_SMEM = (size_t)(GN_GROUPS * WIN + GN_GROUPS * 5 + GN_GROUPS * 2) * sizeof(float4) +
                               (size_t)(GN_GROUPS * WIN + GN_GROUPS) * sizeof(int);

__device__ __forceinline__ IcpCache icp_cache_carve(float4* base) {
    IcpCache C;
    C.mean = base;
    C.brec = C.mean + GN_GROUPS * WIN;
    C.pt = C.brec + GN_GROUPS * 5;
    C.tag = reinterpret_cast<int4*>(C.pt + GN_GROUPS);
    C.slot = reinterpret_cast<int*>(C.tag + GN_GROUPS);
    C.best = C.slot + GN_GROUPS * WIN;
    C.pt_ok = 0;
    return C;
}

__device__ __forceinline__ int probe_rest(int64_t key, int h, int mask, const int64_t* __restrict__ keys) {
#pragma unroll 1
    for (int p = 1; p < PROBES; ++p) {
        int s = (h + p) & mask;
        int64_t k = __ldg(keys + s);
        if (k == key) return s;
        if (k == EMPTY_KEY) return -1;
    }
    return -1;
}

// Squared distance from w to a voxel mean, one expression wherever candidates are compared (bit-identical d2).
__device__ __forceinline__ float mean_d2(float wx, float wy, float wz, const float4& m) {
    const float dx = wx - m.x, dy = wy - m.y, dz = wz - m.z;
    return dx * dx + dy * dy + dz * dz;
}

// The slot of `key` (hashing to h) and, when it is in the map, its mean: -1 when absent.
__device__ __forceinline__ int lookup_mean(int64_t key, const IcpConsts& k, const int64_t* __restrict__ keys,
                                           const float* __restrict__ rec, float4& hd) {
    const int h = slot_hash(key) & k.mask;
    const int64_t k0 = __ldg(keys + h);
    int s = -1;
    if (k0 == key) s = h;
    else if (k0 != EMPTY_KEY) s = probe_rest(key, h, k.mask, keys);
    if (s >= 0) hd = __ldg(reinterpret_cast<const float4*>(rec + (int64_t)s * LW_REC_FLOATS));
    return s;
}

// Phase A of a search: the closest occupied voxel mean among this lane's share (i = lane_g, lane_g + 8, ...) of the
// 27 voxels around base voxel (bx, by, bz), four lookups in flight per lane. o numbers a voxel as the reference's
// loop visits the reach's whole neighbourhood ((dx + R) (2R + 1)^2 + (dy + R) (2R + 1) + dz + R), which breaks ties.
// ws / wm: the group's memo window, based (ox, oy, oz) voxels from (bx, by, bz); with use, entries come from it (an
// entry not gathered yet, -2, is looked up and then kept); otherwise from the hash table and records, and with store
// they are written to it.
__device__ __forceinline__ void icp_search27(int lane_g, int R, int bx, int by, int bz, float wx, float wy, float wz,
                                             const IcpConsts& k, const int64_t* __restrict__ keys,
                                             const float* __restrict__ rec, int* ws, float4* wm, int ox, int oy,
                                             int oz, bool use, bool store, float& best_d2, int& best_o, int& best_s) {
    constexpr int B = 4;
    const int S = 2 * R + 1;
    int s[B], o[B], w[B];
    int64_t key[B];
    float4 hd[B];
    bool val[B], need[B];
#pragma unroll
    for (int u = 0; u < B; ++u) {
        const int i = lane_g + 8 * u;
        val[u] = i < 27;
        const int dx = i / 9 - 1, dy = (i / 3) % 3 - 1, dz = i % 3 - 1;
        o[u] = (dx + R) * S * S + (dy + R) * S + (dz + R);
        w[u] = (dx + ox + 2) * 25 + (dy + oy + 2) * 5 + (dz + oz + 2);
        s[u] = -1;
        need[u] = val[u];
        if (use && val[u]) {
            s[u] = ws[w[u]];
            need[u] = s[u] == -2;
            if (s[u] >= 0) hd[u] = wm[w[u]];
        }
    }
    // the lookups not served by the window: first every probe's head key, then the records
    int h[B];
    int64_t k0[B];
    if (need[0] || need[1] || need[2] || need[3]) {
#pragma unroll
        for (int u = 0; u < B; ++u)
            if (need[u]) {
                const int i = lane_g + 8 * u;
                key[u] = key_ijk(bx + i / 9 - 1, by + (i / 3) % 3 - 1, bz + i % 3 - 1);
                h[u] = slot_hash(key[u]) & k.mask;
                k0[u] = __ldg(keys + h[u]);
            }
#pragma unroll
        for (int u = 0; u < B; ++u)
            if (need[u]) {
                s[u] = -1;
                if (k0[u] == key[u]) s[u] = h[u];
                else if (k0[u] != EMPTY_KEY) s[u] = probe_rest(key[u], h[u], k.mask, keys);
            }
#pragma unroll
        for (int u = 0; u < B; ++u)
            if (need[u] && s[u] >= 0)
                hd[u] = __ldg(reinterpret_cast<const float4*>(rec + (int64_t)s[u] * LW_REC_FLOATS));
        if (ws && (store || use)) {
#pragma unroll
            for (int u = 0; u < B; ++u)
                if (need[u]) {
                    ws[w[u]] = s[u];
                    if (s[u] >= 0) wm[w[u]] = hd[u];
                }
        }
    }
    // this lane's candidates come in increasing o, so the first of equal distances stays
#pragma unroll
    for (int u = 0; u < B; ++u) {
        if (val[u] && s[u] >= 0 && hd[u].w > 0.0f) {
            const float d2 = mean_d2(wx, wy, wz, hd[u]);
            if (d2 < best_d2) {
                best_d2 = d2;
                best_o = o[u];
                best_s = s[u];
            }
        }
    }
}

// How a group of 8 lanes splits a point's 53 accumulator terms, 7 per lane: lanes 0-2 take column pairs (0, 5),
// (1, 4), (2, 3) of H = sum w J^T M J (1 + 6, 2 + 5, 3 + 4 upper-triangle entries), lanes 3-5 the same of Hg
// (precision Mg), lane 6 b = sum w J^T M r and the count, lane 7 the weighted error, rms, weight and range. Each of
// lanes 0-6 forms its two matrix-vector products W v once and then every Jacobian row against both (J w = (w, w x l)
// at the re-centred point l; odom.py:305-307), and picks its seven.
constexpr int TERM_LANES = 8;
constexpr int TERMS_PER_LANE = 7;

__device__ __forceinline__ int triu6(int p, int q) { return p * 6 - (p * (p - 1)) / 2 + (q - p); }

// (p, q) of the 21 upper-triangle entries of a symmetric 6x6 in row-major order (the accumulator's layout), 3 bits
// each.
__host__ __device__ constexpr uint64_t triu6_code(bool want_q) {
    uint64_t v = 0;
    int t = 0;
    for (int p = 0; p < 6; ++p)
        for (int q = p; q < 6; ++q, ++t) v |= (uint64_t)(want_q ? q : p) << (3 * t);
    return v;
}
constexpr uint64_t TRIU6_P = triu6_code(false);
constexpr uint64_t TRIU6_Q = triu6_code(true);
__host__ __device__ constexpr int triu6c(int i, int j) {
    return i <= j ? i * 6 - (i * (i - 1)) / 2 + (j - i) : j * 6 - (j * (j - 1)) / 2 + (i - j);
}

// Where lane lg of a group keeps its term u in the CTA's term rows (lg * 7 + u), seen from accumulator entry t:
// lanes 0-2 hold H's column pairs (q, 5 - q), lanes 3-5 Hg's, lane 6 b and the count, lane 7 the stats.
__device__ __forceinline__ int term_slot(int t) {
    if (t < LW_ACC_B || (t >= LW_ACC_HG && t < NTERMS)) {
        const int e = t < LW_ACC_B ? t : t - LW_ACC_HG;
        const int p = (int)((TRIU6_P >> (3 * e)) & 7u), q = (int)((TRIU6_Q >> (3 * e)) & 7u);  // p <= q
        const int qa = q < 3 ? q : 5 - q;
        return ((t < LW_ACC_B ? 0 : 3) + qa) * TERMS_PER_LANE + (q == qa ? p : qa + 1 + p);
    }
    if (t <= LW_ACC_COUNT) return 6 * TERMS_PER_LANE + (t - LW_ACC_B);  // b, then the count
    return 7 * TERMS_PER_LANE + (t - LW_ACC_ERR);                       // err, rms, weight, range
}

// Fixed point of the cross-CTA sums of the Gauss-Newton loop: 2^-16 units. The largest term a frame can produce
// (rotation block of H: weight 1 x precision <= 2500 m^-2 x lever arm^2 <= 3600 m^2 x 2^18 points) is 2.4e12, so
// the sum of all CTAs' terms stays below 2^62; a partial that would not fit flags an error instead of wrapping.
constexpr double GN_FIX = 65536.0;
constexpr double GN_FIX_MAX = 4.0e18 / 256.0;  // per-CTA bound: 256 CTAs stay below 2^62

// Phase B of a wide search, for the points whose best mean among their 27 inner voxels is not closer than the outer
// shell of their 5 x 5 x 5 neighbourhood (few: those far from the map's surfaces). The whole CTA splits their outer
// voxels; a voxel whose box (widened by a millimetre, more than the rounding of a mean) is farther than the point's
// current best cannot hold a closer or tying mean and is skipped, and each candidate that may win is folded in by
// an atomic minimum of (d2, o, slot) packed into 64 bits -- the order the reference's loop picks in.
constexpr int SLOT_BITS = 25;  // a registration map of up to 2^25 slots
__device__ __forceinline__ unsigned long long pack_best(float d2, int o, int s) {
    return ((unsigned long long)__float_as_uint(d2) << 32) | ((unsigned long long)(o & 127) << SLOT_BITS) |
           (unsigned long long)(s < 0 ? (1 << SLOT_BITS) - 1 : s);
}

struct NeedyPoint {
    float wx, wy, wz;
    int bx, by, bz;
    int win;  // the group whose memo window is based at (bx, by, bz), or -1: outer entries are read and kept there
};

__device__ void outer_shell(const NeedyPoint* __restrict__ q, unsigned long long* best, int nq, const IcpConsts& k,
                            float voxel, const int64_t* __restrict__ keys, const float* __restrict__ rec,
                            const IcpCache* C) {
    for (int it = threadIdx.x; it < nq * 128; it += blockDim.x) {
        const int qi = it >> 7, o = it & 127;
        const int dx = o / 25 - 2, dy = (o / 5) % 5 - 2, dz = o % 5 - 2;
        if (o >= 125 || (abs(dx) <= 1 && abs(dy) <= 1 && abs(dz) <= 1)) continue;
        const NeedyPoint p = q[qi];
        const float slack = 1e-3f;
        const float lx = (float)(p.bx + dx) * voxel - slack, hx = (float)(p.bx + dx + 1) * voxel + slack;
        const float ly = (float)(p.by + dy) * voxel - slack, hy = (float)(p.by + dy + 1) * voxel + slack;
        const float lz = (float)(p.bz + dz) * voxel - slack, hz = (float)(p.bz + dz + 1) * voxel + slack;
        const float gx = fmaxf(0.0f, fmaxf(lx - p.wx, p.wx - hx));
        const float gy = fmaxf(0.0f, fmaxf(ly - p.wy, p.wy - hy));
        const float gz = fmaxf(0.0f, fmaxf(lz - p.wz, p.wz - hz));
        const float box2 = gx * gx + gy * gy + gz * gz;
        const float cur = __uint_as_float((unsigned)(*(volatile unsigned long long*)(best + qi) >> 32));
        if (box2 > cur) continue;
        float4 hd;
        int s = -2;
        int* ws = nullptr;
        float4* wm = nullptr;
        if (C && p.win >= 0) {  // one thread per (point, voxel): no other thread touches this entry now
            ws = C->slot + p.win * WIN;
            wm = C->mean + p.win * WIN;
            s = ws[o];
            if (s >= 0) hd = wm[o];
        }
        if (s == -2) {
            s = lookup_mean(key_ijk(p.bx + dx, p.by + dy, p.bz + dz), k, keys, rec, hd);
            if (ws) {
                ws[o] = s;
                if (s >= 0) wm[o] = hd;
            }
        }
        if (s < 0 || !(hd.w > 0.0f)) continue;
        const float d2 = mean_d2(p.wx, p.wy, p.wz, hd);
        if (d2 < k.max_d2) atomicMin(best + qi, pack_best(d2, o, s));
    }
}

// One accumulation pass of this CTA over its share of the thinned points, a group of 8 lanes per point; writes the
// CTA's float64 partial (part) or adds it in fixed point (fixed). The rounds over the points are uniform across the
// CTA (a round's phase B needs every thread).
__device__ void icp_pass(const float4* __restrict__ ds, int n, const IcpPose& P, const IcpConsts& k,
                         const int64_t* __restrict__ keys, const float* __restrict__ rec, double* __restrict__ part,
                         long long* __restrict__ fixed = nullptr, int* err = nullptr, const IcpCache* C = nullptr) {
    constexpr int G = 8;
    constexpr int GROUPS = GN_THREADS / G;
    constexpr int TPL = TERMS_PER_LANE;  // terms per lane
    static_assert(G == TERM_LANES, "the terms are split over groups of 8 lanes");
    __shared__ float tacc[GN_THREADS / 32][LW_ACC_STRIDE];
    __shared__ NeedyPoint s_need[2][GROUPS];
    __shared__ unsigned long long s_best[2][GROUPS];
    __shared__ int s_nq[3];
    const int R = k.reach;
    const int lane = threadIdx.x & 31;
    const int lane_g = lane & (G - 1);
    const int gl = threadIdx.x / G;
    const int ngroups = gridDim.x * GROUPS;
    const unsigned gmask = 0xFFu << (lane & ~(G - 1));
    const float voxel = 1.0f / k.inv_v;
    if (R == 2) {
        if (threadIdx.x < 3) s_nq[threadIdx.x] = 0;
        __syncthreads();
    }
    float acc[TPL];
#pragma unroll
    for (int u = 0; u < TPL; ++u) acc[u] = 0.0f;
    int round = 0;
    for (int j0 = blockIdx.x * GROUPS; j0 < n; j0 += ngroups, ++round) {
        const int j = j0 + gl;
        const bool active = j < n;
        const bool memo = C != nullptr && j0 == blockIdx.x * GROUPS;  // the memo serves each group's first point
        float4 p = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (active) p = memo && C->pt_ok ? C->pt[gl] : __ldg(ds + j);
        if (active && memo && !C->pt_ok && lane_g == 0) C->pt[gl] = p;
        const float lx = P.R[0] * p.x + P.R[1] * p.y + P.R[2] * p.z + P.tr[0];
        const float ly = P.R[3] * p.x + P.R[4] * p.y + P.R[5] * p.z + P.tr[1];
        const float lz = P.R[6] * p.x + P.R[7] * p.y + P.R[8] * p.z + P.tr[2];
        const float wx = lx + P.c[0], wy = ly + P.c[1], wz = lz + P.c[2];
        const int bx = ifloor(wx * k.inv_v), by = ifloor(wy * k.inv_v), bz = ifloor(wz * k.inv_v);
        // the window serves the wide search from its own base voxel and the narrow one from within one voxel of it
        bool use = false, store = false;
        int ox = 0, oy = 0, oz = 0;
        if (active && memo) {
            const int4 tg = C->tag[gl];
            ox = bx - tg.x;
            oy = by - tg.y;
            oz = bz - tg.z;
            const int lim = 2 - R;
            use = tg.w != 0 && abs(ox) <= lim && abs(oy) <= lim && abs(oz) <= lim;
            store = !use && R == 2;
            if (!use) ox = oy = oz = 0;
        }
        int* ws = memo ? C->slot + gl * WIN : nullptr;
        float4* wm = memo ? C->mean + gl * WIN : nullptr;
        if (store) {
            __syncwarp(gmask);  // every lane of the group has read the old tag
            // a new window: nothing gathered yet (the search below writes the inner 27)
            int4* w4 = reinterpret_cast<int4*>(ws);
            for (int e = lane_g; e < WIN / 4; e += G) w4[e] = make_int4(-2, -2, -2, -2);
            __syncwarp(gmask);
            if (lane_g == 0) C->tag[gl] = make_int4(bx, by, bz, 1);
        }
        float bd = k.max_d2;
        int bo = 0x7FFFFFFF, bs = -1;
        if (active)
            icp_search27(lane_g, R, bx, by, bz, wx, wy, wz, k, keys, rec, ws, wm, ox, oy, oz, use, store, bd, bo, bs);
#pragma unroll
        for (int off = G / 2; off > 0; off >>= 1) {
            float od = __shfl_xor_sync(gmask, bd, off);
            int oo = __shfl_xor_sync(gmask, bo, off);
            int os = __shfl_xor_sync(gmask, bs, off);
            if (od < bd || (od == bd && oo < bo)) {
                bd = od;
                bo = oo;
                bs = os;
            }
        }
        if (R == 2) {
            // phase B: may a mean in the outer shell be at least as close as the inner best? (the nearest outer
            // voxel is a whole voxel or more away along one axis)
            const float fx = wx * k.inv_v - (float)bx, fy = wy * k.inv_v - (float)by, fz = wz * k.inv_v - (float)bz;
            const float gap = fmaxf(0.0f, fminf(fminf(fminf(2.0f - fx, 1.0f + fx), fminf(2.0f - fy, 1.0f + fy)),
                                                 fminf(2.0f - fz, 1.0f + fz)) * voxel - 2e-3f);
            const bool needy = active && gap * gap <= bd;
            const int buf = round & 1;
            int qi = 0;
            if (needy && lane_g == 0) {
                qi = atomicAdd(&s_nq[round % 3], 1);
                // the group's window is based at this point's voxel when it was gathered or used at reach 2 now
                s_need[buf][qi] = NeedyPoint{wx, wy, wz, bx, by, bz, (use || store) ? gl : -1};
                s_best[buf][qi] = pack_best(bd, bo, bs);
            }
            __syncthreads();
            const int nq = s_nq[round % 3];
            if (threadIdx.x == 0) s_nq[(round + 2) % 3] = 0;  // last used two rounds ago; next used after a barrier
            if (nq > 0) {
                outer_shell(s_need[buf], s_best[buf], nq, k, voxel, keys, rec, C);
                __syncthreads();
                if (needy) {
                    qi = __shfl_sync(gmask, qi, lane & ~(G - 1));
                    const unsigned long long b = s_best[buf][qi];
                    bd = __uint_as_float((unsigned)(b >> 32));
                    bo = (int)((b >> SLOT_BITS) & 127u);
                    bs = (int)(b & ((1u << SLOT_BITS) - 1u));
                    if (bs == (1 << SLOT_BITS) - 1) bs = -1;
                }
            }
        }
        if (!active || bs < 0) continue;  // uniform over the group after the reduction
        // the matched voxel's record (odom.py:335-368, hoisted to the insert): every lane of the group reads it
        float4 h0, h1, h2, h3, h4;
        const bool rec_memo = memo && C->best[gl] == bs;
        if (rec_memo) {
            const float4* cr = C->brec + gl * 5;
            h0 = cr[0];
            h1 = cr[1];
            h2 = cr[2];
            h3 = cr[3];
            h4 = cr[4];
        } else {
            const float* rr = rec + (int64_t)bs * LW_REC_FLOATS;
            h0 = __ldg(reinterpret_cast<const float4*>(rr));
            h1 = __ldg(reinterpret_cast<const float4*>(rr + 4));
            h2 = __ldg(reinterpret_cast<const float4*>(rr + 8));
            h3 = __ldg(reinterpret_cast<const float4*>(rr + 12));
            h4 = __ldg(reinterpret_cast<const float4*>(rr + 16));
            if (memo) {
                __syncwarp(gmask);  // every lane of the group has read the old matched slot
                if (lane_g == 0) {
                    float4* cr = C->brec + gl * 5;
                    cr[0] = h0;
                    cr[1] = h1;
                    cr[2] = h2;
                    cr[3] = h3;
                    cr[4] = h4;
                    C->best[gl] = bs;
                }
            }
        }
        const float M[6] = {h1.x, h1.y, h1.z, h1.w, h2.x, h2.y};
        const float Mg[6] = {h2.z, h2.w, h3.x, h3.y, h3.z, h3.w};
        const float r0 = wx - h0.x, r1 = wy - h0.y, r2 = wz - h0.z;
        const float Mr0 = fmaf(M[0], r0, fmaf(M[1], r1, M[2] * r2));
        const float Mr1 = fmaf(M[1], r0, fmaf(M[3], r1, M[4] * r2));
        const float Mr2 = fmaf(M[2], r0, fmaf(M[4], r1, M[5] * r2));
        const float d2 = fmaf(r0, Mr0, fmaf(r1, Mr1, r2 * Mr2));
        float wgt = __frcp_rn(fmaf(d2, k.inv_kappa2, 1.0f));
        wgt = wgt * wgt;  // Geman-McClure
        const float rn = (h4.w > 0.5f) ? fmaf(r0, h4.x, fmaf(r1, h4.y, r2 * h4.z))
                                       : sqrtf(fmaf(r0, r0, fmaf(r1, r1, r2 * r2)));
        // this lane's two matrix-vector products: W (M for H and b, Mg for Hg) times its two columns' vectors,
        // Jacobian rows qa and qb (the residual r for the b lane); a unit row picks W's column as it is
        const int qa = lane_g % 3;
        const bool hg = lane_g >= 3 && lane_g < 6;
        float W[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) W[i] = hg ? Mg[i] : M[i];
        float wa0 = qa == 0 ? W[0] : (qa == 1 ? W[1] : W[2]);
        float wa1 = qa == 0 ? W[1] : (qa == 1 ? W[3] : W[4]);
        float wa2 = qa == 0 ? W[2] : (qa == 1 ? W[4] : W[5]);
        if (lane_g == 6) {
            wa0 = Mr0;
            wa1 = Mr1;
            wa2 = Mr2;
        }
        // row qb = 5 - qa of J: (0, -lz, ly), (lz, 0, -lx) or (-ly, lx, 0)
        const float xa = qa == 2 ? 0.0f : (qa == 1 ? lz : -ly);
        const float xb = qa == 2 ? -lz : (qa == 1 ? 0.0f : lx);
        const float xc = qa == 2 ? ly : (qa == 1 ? -lx : 0.0f);
        const float wb0 = fmaf(W[0], xa, fmaf(W[1], xb, W[2] * xc));
        const float wb1 = fmaf(W[1], xa, fmaf(W[3], xb, W[4] * xc));
        const float wb2 = fmaf(W[2], xa, fmaf(W[4], xb, W[5] * xc));
        // every Jacobian row against both products: J w = (w, w x l) in the rows' own expressions
        const float A[6] = {wa0, wa1, wa2, fmaf(-lz, wa1, ly * wa2), fmaf(lz, wa0, -lx * wa2),
                            fmaf(-ly, wa0, lx * wa1)};
        const float Bv[6] = {wb0, wb1, wb2, fmaf(-lz, wb1, ly * wb2), fmaf(lz, wb0, -lx * wb2),
                             fmaf(-ly, wb0, lx * wb1)};
#pragma unroll
        for (int u = 0; u < TPL; ++u) {
            // term u: row u against column qa while u <= qa, then rows 0.. against column qb (the b lane: rows
            // against M r, then the count)
            const float b1 = u >= 1 ? Bv[u - 1] : 0.0f, b2 = u >= 2 ? Bv[u - 2] : 0.0f, b3 = u >= 3 ? Bv[u - 3] : 0.0f;
            const float bsel = qa == 0 ? b1 : (qa == 1 ? b2 : b3);
            const float asel = u < 6 ? A[u < 6 ? u : 0] : 0.0f;
            float x = (u <= qa || (lane_g == 6 && u < 6)) ? asel : bsel;
            x *= wgt;
            if (lane_g == 6 && u == 6) x = 1.0f;  // the count
            if (lane_g == 7) x = u == 0 ? wgt * d2 : (u == 1 ? wgt * (rn * rn) : (u == 2 ? wgt : (u == 3 ? p.w : 0.0f)));
            acc[u] += x;
        }
    }
    // the CTA's sums: the groups of a warp by shuffles (a fixed butterfly), then each term over the warps in a
    // fixed order, in float64
#pragma unroll
    for (int u = 0; u < TPL; ++u)
#pragma unroll
        for (int off = G; off < 32; off <<= 1) acc[u] += __shfl_xor_sync(0xffffffffu, acc[u], off);
    const int warp = threadIdx.x >> 5;
    if (lane < G) {
#pragma unroll
        for (int u = 0; u < TPL; ++u) tacc[warp][lane * TPL + u] = acc[u];
    }
    __syncthreads();
    if (threadIdx.x < NTERMS) {
        const int slot = term_slot(threadIdx.x);
        double sum = 0.0;
#pragma unroll
        for (int w = 0; w < GN_THREADS / 32; ++w) sum += (double)tacc[w][slot];
        if (fixed) {
            // integer atomics commute: every CTA reads back the same exact sum, whatever the arrival order
            double q = rint(sum * GN_FIX);
            if (!(fabs(q) < GN_FIX_MAX)) {
                atomicExch(err, 4);
                q = 0.0;
            }
            atomicAdd((unsigned long long*)(fixed + threadIdx.x), (unsigned long long)(long long)q);
        } else {
            part[threadIdx.x] = sum;
        }
    }
    __syncthreads();
}


__device__ __forceinline__ void sym6_from(const double* up, double* H) {
    int idx = 0;
    for (int p = 0; p < 6; ++p)
        for (int q = p; q < 6; ++q) {
            H[p * 6 + q] = up[idx];
            H[q * 6 + p] = up[idx];
            ++idx;
        }
}

// Reduce the CTA partials in a fixed order and map the re-centred sums back to the world-origin twist:
// J_world = J_c A with A = [[I, -[c]x], [0, I]], so H = A^T H_c A and b = A^T b_c.
__device__ void reduce_partials(const double* __restrict__ part, int grid, const double* c, double* v64) {
    __shared__ double vs[LW_ACC_STRIDE];
    if (threadIdx.x < LW_ACC_STRIDE) {
        double s = 0.0;
        if (threadIdx.x < NTERMS)
            for (int b = 0; b < grid; ++b) s += part[(int64_t)b * LW_ACC_STRIDE + threadIdx.x];
        vs[threadIdx.x] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double A[36];
        for (int i = 0; i < 36; ++i) A[i] = (i % 7 == 0) ? 1.0 : 0.0;
        // -[c]x in the upper right block
        A[0 * 6 + 3] = 0.0;   A[0 * 6 + 4] = c[2];  A[0 * 6 + 5] = -c[1];
        A[1 * 6 + 3] = -c[2]; A[1 * 6 + 4] = 0.0;   A[1 * 6 + 5] = c[0];
        A[2 * 6 + 3] = c[1];  A[2 * 6 + 4] = -c[0]; A[2 * 6 + 5] = 0.0;
        for (int t = 0; t < LW_ACC_STRIDE; ++t) v64[t] = vs[t];
        for (int which = 0; which < 2; ++which) {
            int off = which == 0 ? LW_ACC_H : LW_ACC_HG;
            double H[36], AH[36];
            sym6_from(vs + off, H);
            for (int i = 0; i < 6; ++i)
                for (int j = 0; j < 6; ++j) {
                    double s = 0.0;
                    for (int k = 0; k < 6; ++k) s += H[i * 6 + k] * A[k * 6 + j];
                    AH[i * 6 + j] = s;
                }
            int idx = 0;
            for (int p = 0; p < 6; ++p)
                for (int q = p; q < 6; ++q) {
                    double s = 0.0;
                    for (int k = 0; k < 6; ++k) s += A[k * 6 + p] * AH[k * 6 + q];
                    v64[off + idx] = s;
                    ++idx;
                }
        }
        for (int p = 0; p < 6; ++p) {
            double s = 0.0;
            for (int k = 0; k < 6; ++k) s += A[k * 6 + p] * vs[LW_ACC_B + k];
            v64[LW_ACC_B + p] = s;
        }
    }
    __syncthreads();
}

__device__ void make_pose(const double* T, const double* c, IcpPose& P) {
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) P.R[i * 3 + j] = (float)T[i * 4 + j];
        P.tr[i] = (float)(T[i * 4 + 3] - c[i]);
        P.c[i] = (float)c[i];
    }
}

// 6 x 0.7^it, the Geman-McClure scale's decay (odom.py:86, 767), by repeated multiplication at compile time
__host__ __device__ constexpr double kappa_raw(int it) { return it <= 0 ? 6.0 : 0.7 * kappa_raw(it - 1); }

__device__ __forceinline__ void schedule(int it, float voxel, int& reach, float& max_d2, float& kappa) {
    reach = it < 3 ? 2 : 1;  // wide search first, then local refinement (odom.py:765-767)
    float d = ((float)reach + 0.5f) * voxel;
    max_d2 = d * d;
    kappa = it >= 4 ? 2.0f : fmaxf(2.0f, (float)(it == 0 ? kappa_raw(0) : it == 1 ? kappa_raw(1)
                                                 : it == 2 ? kappa_raw(2) : kappa_raw(3)));
}

// ---- the float64 step (odom.py:772-796) ----------------------------------------------------------------

// Sensor basis (odom.py:425-433): SB = [[R, [c]x R / L], [0, R / L]] and its inverse [[R^T, -R^T [c]x], [0, L R^T]].
__device__ void sensor_basis(const double* T, double L, double* SB, double* SBi) {
    double R[9], c[3] = {T[3], T[7], T[11]};
    mat44_rot(T, R);
    double cx[9] = {0.0, -c[2], c[1], c[2], 0.0, -c[0], -c[1], c[0], 0.0};
    for (int i = 0; i < 36; ++i) SB[i] = SBi[i] = 0.0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double cr = 0.0, rc = 0.0;
            for (int k = 0; k < 3; ++k) {
                cr += cx[i * 3 + k] * R[k * 3 + j];
                rc += R[k * 3 + i] * cx[k * 3 + j];  // (R^T [c]x)_ij
            }
            SB[i * 6 + j] = R[i * 3 + j];
            SB[i * 6 + 3 + j] = cr / L;
            SB[(3 + i) * 6 + 3 + j] = R[i * 3 + j] / L;
            SBi[i * 6 + j] = R[j * 3 + i];
            SBi[i * 6 + 3 + j] = -rc;
            SBi[(3 + i) * 6 + 3 + j] = L * R[j * 3 + i];
        }
}

__device__ __forceinline__ void matmul6(const double* A, const double* B, double* C, bool At = false) {
    double t[36];
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            double s = 0.0;
            for (int k = 0; k < 6; ++k) s += (At ? A[k * 6 + i] : A[i * 6 + k]) * B[k * 6 + j];
            t[i * 6 + j] = s;
        }
    for (int i = 0; i < 36; ++i) C[i] = t[i];
}

__device__ __forceinline__ void matvec6(const double* A, const double* x, double* y, bool At = false) {
    double t[6];
    for (int i = 0; i < 6; ++i) {
        double s = 0.0;
        for (int k = 0; k < 6; ++k) s += (At ? A[k * 6 + i] : A[i * 6 + k]) * x[k];
        t[i] = s;
    }
    for (int i = 0; i < 6; ++i) y[i] = t[i];
}

struct StepOut {
    int status;  // 0 continue, 1 converged, 2 too few correspondences, 3 singular
    int corr, degen;
    double rms;
};

// One Gauss-Newton update of T (odom.py:769-796). H (world twist) is returned for the conditioning stat.
__device__ __noinline__ StepOut gn_step(const double* v, double* T, const double* T_pred, const lw_odom_params& prm,
                                        double* H) {
    StepOut o;
    o.corr = (int)v[LW_ACC_COUNT];
    o.degen = 0;
    o.rms = 0.0;
    if (o.corr < prm.min_corr) {
        o.status = 2;
        return o;
    }
    double b[6], Hg[36], A[36], rhs[6];
    sym6_from(v + LW_ACC_H, H);
    sym6_from(v + LW_ACC_HG, Hg);
    for (int k = 0; k < 6; ++k) b[k] = v[LW_ACC_B + k];
    double L = fmax(v[LW_ACC_RANGE] / (double)o.corr, 1.0);
    o.rms = sqrt(fmax(v[LW_ACC_RMS], 0.0) / fmax(v[LW_ACC_WEIGHT], 1e-9));
    double dmean = 0.0;
    for (int k = 0; k < 6; ++k) dmean += H[k * 7];
    dmean /= 6.0;
    for (int i = 0; i < 36; ++i) A[i] = H[i];
    for (int k = 0; k < 6; ++k) {
        A[k * 7] += 1e-9 * dmean + prm.damping * H[k * 7];
        rhs[k] = -b[k];
    }
    // the left twist from T back onto the prediction (odom.py:397-401)
    double Ti[16], Mp[16], xi[6];
    mat44_inv_rigid(T, Ti);
    mat44_mul(T_pred, Ti, Mp);
    body_twist(Mp, xi);
    double SB[36], SBi[36];
    sensor_basis(T, L, SB, SBi);
    if (prm.prior_info > 0.0) {
        double P[36], Pxi[6];
        matmul6(SBi, SBi, P, true);
        for (int i = 0; i < 36; ++i) P[i] *= prm.prior_info;
        matvec6(P, xi, Pxi);
        for (int i = 0; i < 36; ++i) A[i] += P[i];
        for (int k = 0; k < 6; ++k) rhs[k] += Pxi[k];
    }
    double delta[6];
    if (prm.degen_thr > 0.0) {
        // odom.py:436-455: hold the directions the surface normals do not constrain at the prediction
        double G[36], V[36], lam[6], tmp[36];
        matmul6(Hg, SB, tmp);
        matmul6(SB, tmp, G, true);
        jacobi_eig<6>(G, lam, V);
        bool good[6];
        int ng = 0;
        for (int k = 0; k < 6; ++k) {
            good[k] = lam[k] >= prm.degen_thr;
            ng += good[k] ? 1 : 0;
        }
        o.degen = 6 - ng;
        if (ng == 6) {
            if (!lu_solve<6>(A, rhs, delta)) {
                o.status = 3;
                return o;
            }
        } else {
            double z[6], d0[6];
            matvec6(SBi, xi, z);  // solve(J, to_pred)
            for (int i = 0; i < 6; ++i) d0[i] = 0.0;
            for (int k = 0; k < 6; ++k) {
                if (good[k]) continue;
                double pr = 0.0;
                for (int i = 0; i < 6; ++i) pr += V[i * 6 + k] * z[i];
                for (int i = 0; i < 6; ++i) d0[i] += V[i * 6 + k] * pr;
            }
            if (ng > 0) {
                double As[36], Jr[6], Asd[6], g[6], Ag[36], y[6], Vg[36];
                int cols[6], nc = 0;
                for (int k = 0; k < 6; ++k)
                    if (good[k]) cols[nc++] = k;
                matmul6(A, SB, tmp);
                matmul6(SB, tmp, As, true);
                matvec6(SB, rhs, Jr, true);
                matvec6(As, d0, Asd);
                for (int i = 0; i < 6; ++i)
                    for (int a = 0; a < nc; ++a) Vg[i * 6 + a] = V[i * 6 + cols[a]];
                for (int a = 0; a < nc; ++a) {
                    double s = 0.0;
                    for (int i = 0; i < 6; ++i) s += Vg[i * 6 + a] * (Jr[i] - Asd[i]);
                    g[a] = s;
                    for (int c2 = 0; c2 < nc; ++c2) {
                        double s2 = 0.0;
                        for (int i = 0; i < 6; ++i) {
                            double t2 = 0.0;
                            for (int j = 0; j < 6; ++j) t2 += As[i * 6 + j] * Vg[j * 6 + c2];
                            s2 += Vg[i * 6 + a] * t2;
                        }
                        Ag[a * 6 + c2] = s2;
                    }
                }
                if (!lu_solve<6>(Ag, g, y, nc)) {
                    o.status = 3;
                    return o;
                }
                for (int i = 0; i < 6; ++i)
                    for (int a = 0; a < nc; ++a) d0[i] += Vg[i * 6 + a] * y[a];
            }
            matvec6(SB, d0, delta);
        }
    } else if (!lu_solve<6>(A, rhs, delta)) {
        o.status = 3;
        return o;
    }
    apply_twist(T, delta);
    double nt = sqrt(delta[0] * delta[0] + delta[1] * delta[1] + delta[2] * delta[2]);
    double nr = sqrt(delta[3] * delta[3] + delta[4] * delta[4] + delta[5] * delta[5]);
    o.status = (nt < 1e-4 && nr < 1e-4) ? 1 : 0;  // STEP_TOL (odom.py:88)
    return o;
}

// min/max eigenvalue of H normalised by its diagonal (odom.py:797-800)
__device__ __noinline__ double conditioning(const double* H) {
    double dg[6], Hn[36], ev[6], V[36];
    for (int k = 0; k < 6; ++k) dg[k] = sqrt(fmax(H[k * 7], 1e-12));
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) Hn[i * 6 + j] = H[i * 6 + j] / (dg[i] * dg[j]);
    jacobi_eig<6>(Hn, ev, V);
    double lo = ev[0], hi = ev[0];
    for (int k = 1; k < 6; ++k) {
        lo = fmin(lo, ev[k]);
        hi = fmax(hi, ev[k]);
    }
    return fmax(lo, 0.0) / fmax(hi, 1e-12);
}

__device__ __forceinline__ double pow2_below(double p) {  // 2^-e for p = m 2^e, m in [1, 2), p normal and positive
    const int e = ((__double2hiint(p) >> 20) & 0x7FF) - 1023;
    return __hiloint2double((1023 - e) << 20, 0);
}

// ---- the conditioning statistic -------------------------------------------------------------------------------
// How many pivots of the elimination of A - x I (symmetric 6x6, in registers) are negative: by Sylvester's law of
// inertia, the number of A's eigenvalues below x. Each step forms |p| row_i - sign(p) a_ik row_k with |p| scaled
// by a power of two -- a positive multiple of the Schur complement, so its signs are kept -- and no division; a
// zero or non-finite pivot is counted as negative and the elimination goes on from -1.
__device__ __forceinline__ int neg_count6(const double* __restrict__ A, double x) {
    double a[36];
#pragma unroll
    for (int e = 0; e < 36; ++e) a[e] = A[e];
#pragma unroll
    for (int k = 0; k < 6; ++k) a[k * 7] -= x;
    int neg = 0;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        double p = a[k * 7];
        if (!(p > 0.0)) {
            ++neg;
            if (!(p < -1e-290 && p > -1e290)) p = -1.0;
        } else if (!(p > 1e-290 && p < 1e290)) {
            p = 1.0;
        }
        const double ap = fabs(p);
        const double sc = pow2_below(ap);
        const double ps = ap * sc;
        const double sg = p > 0.0 ? sc : -sc;
#pragma unroll
        for (int i = k + 1; i < 6; ++i) {
            const double f = a[k * 6 + i] * sg;
#pragma unroll
            for (int j = i; j < 6; ++j) a[i * 6 + j] = fma(ps, a[i * 6 + j], -(f * a[k * 6 + j]));
        }
    }
    return neg;
}

// min(lambda) / max(lambda) of a positive semi-definite 6x6 with unit diagonal (H normalised by its diagonal,
// odom.py:797-800), on one warp, without an eigen-decomposition: with a unit diagonal lambda_min <= 1 <= lambda_max
// <= 6, and the count of eigenvalues below a shift brackets each end. Every round, lanes 0-15 try 16 shifts on a
// logarithmic grid over lambda_min's bracket (from 2^-46.5 ~ 1e-14 up to 1) and lanes 16-31 16 shifts on a linear
// grid over lambda_max's (1 to 6); each end keeps the sixteenth of its bracket where the count first reaches 1
// (respectively 6). Four rounds leave lambda_max within ~1e-4 and lambda_min within ~5e-4 relative; a lambda_min
// below the grid's floor is taken as 0. Every lane returns the ratio.
__device__ double cond6_warp(const double* __restrict__ A) {
    constexpr float LOG2_FLOOR = -46.5f;
    const int lane = threadIdx.x & 31;
    const bool low = lane < 16;
    const int kk = lane & 15;
    float lo = low ? LOG2_FLOOR : 1.0f, hi = low ? 0.0f : 6.0f;
#pragma unroll 1
    for (int r = 0; r < 4; ++r) {
        const float g = lo + (hi - lo) * (float)(kk + 1) * (1.0f / 16.0f);
        const double x = low ? (double)exp2f(g) : (double)g;
        const int c = neg_count6(A, x);
        const unsigned m = __ballot_sync(0xffffffffu, low ? c >= 1 : c >= 6);
        const unsigned mine = low ? (m & 0xFFFFu) : (m >> 16);
        if (mine == 0u) {
            lo = hi;  // above the bracket's top (rounding): pin it there
        } else {
            const int k = __ffs(mine) - 1;
            const float w = (hi - lo) * (1.0f / 16.0f);
            lo = lo + w * (float)k;
            hi = lo + w;
        }
    }
    const float l0 = __shfl_sync(0xffffffffu, lo, 0), h0 = __shfl_sync(0xffffffffu, hi, 0);
    const float l1 = __shfl_sync(0xffffffffu, lo, 16), h1 = __shfl_sync(0xffffffffu, hi, 16);
    const double lmin = l0 <= LOG2_FLOOR ? 0.0 : (double)exp2f(0.5f * (l0 + h0));
    const double lmax = 0.5 * ((double)l1 + (double)h1);
    return fmax(lmin, 0.0) / fmax(lmax, 1e-12);
}

// ---- the float64 step --------------------------------------------------------------------------------------
// Every CTA of the persistent kernel runs the same step on the same reduced accumulator (so one grid barrier per
// iteration suffices). The step is a chain of dependent float64 operations, so its cost is latency: the 6x6
// products are one element per thread with compile-time indices and no divergent branches, the positive-
// definiteness test and the solve are L D L^T factorisations held in registers on two threads of different warps.
// Only a frame with a degenerate direction takes the eigen-decomposition path (odom.py:436-455).

struct GnSmem {
    double v[LW_ACC_STRIDE];
    double Ac[36];   // [[I, -[c]x], [0, I]]: the re-centred twist's columns in the world-origin twist (per launch)
    double W[36];    // Ac SB0: the sensor basis (without 1/L) seen from the re-centred twist (per iteration)
    double H[36], b[6];
    double A[36], SB[36], SBi[36], P[36], tmp[36], G[36];
    double rhs[6], xi[6], delta[6];
    double EA[36], EV[36], ev[6], rot[6];  // the warp eigen-decomposition (degenerate branch, conditioning)
    double wv[6][6];                        // the degenerate step's vectors
    int have_v, dstat;                      // EV holds an earlier iteration's vectors; the degenerate step's status
    double T[16], Tp[16], c[3];
    double SB0[36], P0[36], P0xi[6];       // from the pose alone, formed while the grid barrier waits
    double L;
    int status, corr, degen;
};

// What the step needs from the current pose alone, formed by one thread while the grid barrier waits: the twist
// from the current pose back to the prediction (odom.py:397-401), the sensor basis without its 1/L scaling,
// SB0 = [[R, C R], [0, R]] (C = [c]x, c the sensor position; odom.py:425-433), the same seen from the twist about
// the pass centre c0, W = [[I, -[c0]x], [0, I]] SB0 = [[R, [c - c0]x R], [0, R]], and the prior's information
// without its L^2 term, P0 = prior_info [[I, -C], [C, C^T C]] (the closed form of SB^-T SB^-1, R R^T = I), with P0 xi.
struct StepPrep {
    GnSmem* S;
    double prior;
    __device__ void operator()() const {
        double Ti[16], Mp[16];
        mat44_inv_rigid(S->T, Ti);
        mat44_mul(S->Tp, Ti, Mp);
        body_twist(Mp, S->xi);
        const double* T = S->T;
        const double c0 = T[3], c1 = T[7], c2 = T[11];
        const double C[9] = {0.0, -c2, c1, c2, 0.0, -c0, -c1, c0, 0.0};
        const double cc = c0 * c0 + c1 * c1 + c2 * c2;
        const double cv[3] = {c0, c1, c2};
        const double d0 = c0 - S->c[0], d1 = c1 - S->c[1], d2 = c2 - S->c[2];
        const double D[9] = {0.0, -d2, d1, d2, 0.0, -d0, -d1, d0, 0.0};
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const double r = T[i * 4 + j];
                const double cr = C[i * 3 + 0] * T[0 * 4 + j] + C[i * 3 + 1] * T[1 * 4 + j] + C[i * 3 + 2] * T[2 * 4 + j];
                const double dr = D[i * 3 + 0] * T[0 * 4 + j] + D[i * 3 + 1] * T[1 * 4 + j] + D[i * 3 + 2] * T[2 * 4 + j];
                S->SB0[i * 6 + j] = r;
                S->SB0[i * 6 + j + 3] = cr;
                S->SB0[(i + 3) * 6 + j] = 0.0;
                S->SB0[(i + 3) * 6 + j + 3] = r;
                S->W[i * 6 + j] = r;
                S->W[i * 6 + j + 3] = dr;
                S->W[(i + 3) * 6 + j] = 0.0;
                S->W[(i + 3) * 6 + j + 3] = r;
                S->P0[i * 6 + j] = i == j ? prior : 0.0;
                S->P0[i * 6 + j + 3] = -prior * C[i * 3 + j];
                S->P0[(i + 3) * 6 + j] = prior * C[i * 3 + j];
                S->P0[(i + 3) * 6 + j + 3] = prior * ((i == j ? cc : 0.0) - cv[i] * cv[j]);
            }
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            double x = 0.0;
#pragma unroll
            for (int k = 0; k < 6; ++k) x += S->P0[i * 6 + k] * S->xi[k];
            S->P0xi[i] = x;
        }
    }
};

// The cross-CTA sums from the fixed-point accumulator (one load per term).
__device__ void gn_reduce_fixed(const long long* __restrict__ fixed, GnSmem& S) {
    const int t = threadIdx.x;
    if (t < LW_ACC_STRIDE) S.v[t] = t < NTERMS ? (double)__ldcg(fixed + t) * (1.0 / GN_FIX) : 0.0;
    __syncthreads();
}

__device__ __forceinline__ int sym_idx(int p, int q) {
    // index of (p, q) in the row-major upper triangle of a 6x6 matrix
    if (p > q) {
        int t = p;
        p = q;
        q = t;
    }
    return p * 6 - (p * (p - 1)) / 2 + (q - p);
}

// -[c]x, the upper-right block of the map from the world-origin twist to the re-centred one
__device__ __forceinline__ double kmat(const double* c, int i, int j) {
    const double K[9] = {0.0, c[2], -c[1], -c[2], 0.0, c[0], c[1], -c[0], 0.0};
    return K[i * 3 + j];
}


// Cholesky of a symmetric 6x6 (row major) shifted by -shift on the diagonal, in registers; false unless it is
// positive definite.
__device__ __forceinline__ bool chol6(const double* M, double shift, double* Lf) {
#pragma unroll
    for (int j = 0; j < 6; ++j) {
        double d = M[j * 6 + j] - shift;
#pragma unroll
        for (int k = 0; k < j; ++k) d -= Lf[j * 6 + k] * Lf[j * 6 + k];
        if (!(d > 0.0)) return false;
        d = sqrt(d);
        Lf[j * 6 + j] = d;
#pragma unroll
        for (int i = j + 1; i < 6; ++i) {
            double x = M[i * 6 + j];
#pragma unroll
            for (int k = 0; k < j; ++k) x -= Lf[i * 6 + k] * Lf[j * 6 + k];
            Lf[i * 6 + j] = x / d;
        }
    }
    return true;
}

__device__ __forceinline__ void chol6_solve(const double* Lf, const double* rhs, double* x) {
    double y[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        double s = rhs[i];
#pragma unroll
        for (int k = 0; k < i; ++k) s -= Lf[i * 6 + k] * y[k];
        y[i] = s / Lf[i * 6 + i];
    }
#pragma unroll
    for (int i = 5; i >= 0; --i) {
        double s = y[i];
#pragma unroll
        for (int k = i + 1; k < 6; ++k) s -= Lf[k * 6 + i] * x[k];
        x[i] = s / Lf[i * 6 + i];
    }
}

// 1 / d for a normal d of moderate size (the caller has checked it) on a chain of dependent operations: the PTX
// approximate reciprocal refined by two Newton-Raphson steps r <- r + r (1 - d r), each of which doubles the number
// of correct bits, to within an ulp or so of the rounded quotient.
__device__ __forceinline__ double rcp_newton_normal(double d) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
    double e = fma(-d, r, 1.0);
    r = fma(r, e, r);
    e = fma(-d, r, 1.0);
    return fma(r, e, r);
}

// Gaussian elimination of a symmetric 6x6 (row major, in registers) shifted by diag(st, st, st, sr, sr, sr), with
// no division on its chain: step k replaces each trailing row by p_k row_i - a_ik row_k, where p_k is the pivot
// times the power of two that brings it to [1, 2) (an exact scaling, so the entries keep their range); the update
// p A - a a^T keeps the trailing block symmetric, so only its upper triangle is formed, and it scales each Schur
// complement by a positive factor, so the pivots carry the signs of the L D L^T pivots. Returns 0 unless every
// pivot is positive (the shifted matrix positive definite). With rhs, the right-hand side is carried along and
// x receives the solution: the six reciprocals are taken together, then the back substitution only multiplies.

__device__ __forceinline__ int elim6(double* a, double st, double sr, double* rhs, double* x) {
#pragma unroll
    for (int k = 0; k < 6; ++k) a[k * 7] -= k < 3 ? st : sr;
    int ok = 1;  // no early exit: a branch per pivot would hold the next steps back
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        double p = a[k * 7];
        const bool good = p > 1e-300 && p < 1e300;
        ok &= good ? 1 : 0;
        p = good ? p : 1.0;  // a failed factor goes on with finite numbers and is discarded
        const double sc = pow2_below(p);
        const double ps = p * sc;
#pragma unroll
        for (int i = k + 1; i < 6; ++i) {
            const double f = a[k * 6 + i] * sc;  // a_ik, by symmetry
#pragma unroll
            for (int j = i; j < 6; ++j) a[i * 6 + j] = fma(ps, a[i * 6 + j], -(f * a[k * 6 + j]));
            if (rhs) rhs[i] = fma(ps, rhs[i], -(f * rhs[k]));
        }
    }
    if (!rhs) return ok;
    double r[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) r[k] = rcp_newton_normal(a[k * 7]);  // the pivots passed the range test
    double acc[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) acc[k] = rhs[k];
#pragma unroll
    for (int k = 5; k >= 0; --k) {
        x[k] = acc[k] * r[k];
#pragma unroll
        for (int i = 0; i < k; ++i) acc[i] = fma(-a[i * 6 + k], x[k], acc[i]);
    }
    return ok;
}

// The degenerate branch of odom.py:436-455 (some direction below degen_thr): with G's eigen-decomposition in
// S.ev / S.EV, hold the weak directions at the prediction and solve for the rest. Warp 0, every lane: the 6x6
// products run one element per lane; the small solve on the kept directions runs on lane 0. Writes S.delta,
// S.degen and S.dstat (0, or 3 when a factorisation fails).
__device__ void gn_degenerate_warp(GnSmem& S, double thr) {
    const int lane = threadIdx.x & 31;
    const double* V = S.EV;
    unsigned gm = 0;
    for (int k = 0; k < 6; ++k)
        if (S.ev[k] >= thr) gm |= 1u << k;
    const int ng = __popc(gm);
    if (lane == 0) {
        S.degen = 6 - ng;
        S.dstat = 0;
    }
    if (ng == 6) {
        if (lane == 0) {
            double Lf[36], d[6];
            if (!chol6(S.A, 0.0, Lf)) {
                S.dstat = 3;
            } else {
                chol6_solve(Lf, S.rhs, d);
                for (int i = 0; i < 6; ++i) S.delta[i] = d[i];
            }
        }
        __syncwarp();
        return;
    }
    double* z = S.wv[0];   // SB^-1 (prediction - current): solve(J, to_pred)
    double* d0 = S.wv[1];  // the step in the sensor basis
    double* Jr = S.wv[2];  // SB^T rhs
    double* pr = S.wv[3];  // weak-direction components of z, then the residual Jr - As d0
    double* gf = S.wv[4];  // V^T (Jr - As d0)
    double* yf = S.wv[5];  // the kept directions' solution (zero on the weak ones)
    double* tmp = S.tmp;   // A SB, then As V
    double* As = S.P;      // SB^T A SB
    double* M = S.EA;      // V^T As V
    if (lane < 6) {
        double t = 0.0;
        for (int k = 0; k < 6; ++k) t += S.SBi[lane * 6 + k] * S.xi[k];
        z[lane] = t;
    } else if (lane >= 8 && lane < 14) {
        const int i = lane - 8;
        double t = 0.0;
        for (int k = 0; k < 6; ++k) t += S.SB[k * 6 + i] * S.rhs[k];
        Jr[i] = t;
    }
    for (int e = lane; e < 36; e += 32) {
        const int i = e / 6, j = e % 6;
        double t = 0.0;
        for (int k = 0; k < 6; ++k) t += S.A[i * 6 + k] * S.SB[k * 6 + j];
        tmp[e] = t;
    }
    __syncwarp();
    if (lane < 6) {
        double t = 0.0;
        if (!((gm >> lane) & 1u))
            for (int i = 0; i < 6; ++i) t += V[i * 6 + lane] * z[i];
        pr[lane] = t;
    }
    for (int e = lane; e < 36; e += 32) {
        const int i = e / 6, j = e % 6;
        double t = 0.0;
        for (int k = 0; k < 6; ++k) t += S.SB[k * 6 + i] * tmp[k * 6 + j];
        As[e] = t;
    }
    __syncwarp();
    if (lane < 6) {
        double t = 0.0;
        for (int k = 0; k < 6; ++k)
            if (!((gm >> k) & 1u)) t += V[lane * 6 + k] * pr[k];
        d0[lane] = t;
    }
    for (int e = lane; e < 36; e += 32) {
        const int i = e / 6, j = e % 6;
        double t = 0.0;
        for (int k = 0; k < 6; ++k) t += As[i * 6 + k] * V[k * 6 + j];
        tmp[e] = t;
    }
    __syncwarp();
    if (ng > 0) {
        if (lane < 6) {
            double t = 0.0;
            for (int k = 0; k < 6; ++k) t += As[lane * 6 + k] * d0[k];
            pr[lane] = Jr[lane] - t;
        }
        for (int e = lane; e < 36; e += 32) {
            const int i = e / 6, j = e % 6;
            double t = 0.0;
            for (int k = 0; k < 6; ++k) t += V[k * 6 + i] * tmp[k * 6 + j];
            M[e] = t;
        }
        __syncwarp();
        if (lane < 6) {
            double t = 0.0;
            for (int i = 0; i < 6; ++i) t += V[i * 6 + lane] * pr[i];
            gf[lane] = t;
        }
        __syncwarp();
        if (lane == 0) {
            int cols[6], nc = 0;
            for (int k = 0; k < 6; ++k)
                if ((gm >> k) & 1u) cols[nc++] = k;
            double Ag[36], g[6], y[6];
            for (int a = 0; a < nc; ++a) {
                g[a] = gf[cols[a]];
                for (int c2 = 0; c2 < nc; ++c2) Ag[a * 6 + c2] = M[cols[a] * 6 + cols[c2]];
            }
            for (int k = 0; k < 6; ++k) yf[k] = 0.0;
            if (!lu_solve<6>(Ag, g, y, nc))
                S.dstat = 3;
            else
                for (int a = 0; a < nc; ++a) yf[cols[a]] = y[a];
        }
        __syncwarp();
        if (lane < 6) {
            double t = d0[lane];
            for (int k = 0; k < 6; ++k)
                if ((gm >> k) & 1u) t += V[lane * 6 + k] * yf[k];
            d0[lane] = t;
        }
        __syncwarp();
    }
    if (lane < 6) {
        double t = 0.0;
        for (int k = 0; k < 6; ++k) t += S.SB[lane * 6 + k] * d0[k];
        S.delta[lane] = t;
    }
    __syncwarp();
}

// -[c]x, entry (k, m), without an indexed local array.
__device__ __forceinline__ double kneg(const double* c, int k, int m) {
    return k == m ? 0.0
                  : (k == 0 ? (m == 1 ? c[2] : -c[1]) : (k == 1 ? (m == 0 ? -c[2] : c[0]) : (m == 0 ? c[1] : -c[0])));
}

__device__ __forceinline__ void pair_sync() { asm volatile("bar.sync 1, 64;" ::: "memory"); }

// u^T M v for a symmetric 6x6 M stored as its packed upper triangle: unrolled, every load of M is a fixed offset and
// the six row sums are independent chains.
__device__ __forceinline__ double sym_bilinear(const double* M, const double (&u)[6], const double (&v)[6]) {
    double r[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        double t = 0.0;
#pragma unroll
        for (int j = 0; j < 6; ++j) t = fma(M[triu6c(i, j)], v[j], t);
        r[i] = u[i] * t;
    }
    return ((r[0] + r[1]) + (r[2] + r[3])) + (r[4] + r[5]);
}

// A = H + LM damping + prior information and rhs = -b + prior (xi) (odom.py:772-785), from the first phase's threads
// plus the 1e-9 mean-diagonal term and the prior's L^2 terms, solved in registers by one thread (elim6); what it
// adds goes back to shared memory for the degenerate branch. 0 when A is not positive definite.
__device__ __forceinline__ int gn_solve_thread(GnSmem& S, const lw_odom_params& prm, double* delta) {
    const double dm = ((S.H[0] + S.H[7]) + (S.H[14] + S.H[21]) + (S.H[28] + S.H[35])) * (1e-9 / 6.0);
    const double pl2 = prm.prior_info > 0.0 ? prm.prior_info * S.L * S.L : 0.0;  // the prior's L^2 term
    double a[36], rhs[6];
#pragma unroll
    for (int p = 0; p < 6; ++p) {
#pragma unroll
        for (int q = p; q < 6; ++q) a[p * 6 + q] = S.A[p * 6 + q];
        rhs[p] = S.rhs[p] + (p >= 3 ? pl2 * S.xi[p] : 0.0);
    }
#pragma unroll
    for (int p = 0; p < 6; ++p) {
        a[p * 7] += dm + (p >= 3 ? pl2 : 0.0);
        S.A[p * 7] = a[p * 7];
    }
#pragma unroll
    for (int p = 3; p < 6; ++p) S.rhs[p] = rhs[p];
    return elim6(a, 0.0, 0.0, rhs, delta);
}

// One Gauss-Newton update of S.T (odom.py:769-796) on warps 0 and 1 (the other warps go straight to the block
// barrier after it). S.status: 0 continue, 1 converged, 2 too few correspondences, 3 singular.
//   1. one output per thread: threads 0-20 the world-origin H = Ac^T Hc Ac (the sums were
//      taken about the pass centre; odom.py's twist is about the origin), 21-41 G0 = W^T Hg_c W, of which the
//      sensor-basis information is G = SB^T Hg SB = diag(s) G0 diag(s) (s = 1, 1, 1, 1/L, 1/L, 1/L), 42-47
//      b = Ac^T b_c, 48 the count and the mean range L (odom.py:769-772); the H threads also form A and the b
//      threads rhs;
//   2. thread 0 solves A delta = rhs (elim6; A and rhs formed in phase 1) while thread 32 tests G for the threshold
//      by the same elimination;
//   3. warp 0 takes the degenerate step if a direction is below the threshold, then applies the twist.
// Named barrier 1 orders the two warps.
__device__ void gn_step_pair(GnSmem& S, const lw_odom_params& prm) {
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    __shared__ int s_g_ok, s_a_ok;
    if (tid < 42) {
        const bool is_h = tid < 21;
        const int u = is_h ? tid : tid - 21;
        const int p = (int)((TRIU6_P >> (3 * u)) & 7u), q = (int)((TRIU6_Q >> (3 * u)) & 7u);
        const double* U = is_h ? S.Ac : S.W;
        double up[6], uq[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            up[i] = U[i * 6 + p];
            uq[i] = U[i * 6 + q];
        }
        const double x = sym_bilinear(S.v + (is_h ? LW_ACC_H : LW_ACC_HG), up, uq);
        double* out = is_h ? S.H : S.G;
        out[p * 6 + q] = x;
        out[q * 6 + p] = x;
        if (is_h) {
            // A = H + LM damping + prior information, but for the 1e-9 mean-diagonal term and the prior's L^2 term
            // (the solve adds those)
            double a = x + S.P0[p * 6 + q];
            if (p == q) a += prm.damping * x;
            S.A[p * 6 + q] = a;
            S.A[q * 6 + p] = a;
        }
    } else if (tid < 48) {
        const int p = tid - 42;
        double x = 0.0;
#pragma unroll
        for (int i = 0; i < 6; ++i) x = fma(S.Ac[i * 6 + p], S.v[LW_ACC_B + i], x);
        S.b[p] = x;
        S.rhs[p] = -x + S.P0xi[p];  // -b + prior (xi), but for the prior's L^2 term
    } else if (tid == 48) {
        S.corr = (int)S.v[LW_ACC_COUNT];
        S.status = S.corr < prm.min_corr ? 2 : 0;
        S.degen = 0;
        S.L = fmax(S.v[LW_ACC_RANGE] / (double)S.corr, 1.0);
    }
    pair_sync();
    if (S.status != 0) return;  // uniform over the two warps
    double delta[6];
    if (tid == 0) s_a_ok = gn_solve_thread(S, prm, delta);
    if (tid == 32) {
        // G = diag(s) G0 diag(s) with s = (1, 1, 1, 1/L, 1/L, 1/L): G - thr I is positive definite exactly when
        // G0 - thr diag(1, 1, 1, L^2, L^2, L^2) is (a congruence), so the test needs no scaling
        int ok = 1;
        if (prm.degen_thr > 0.0) {
            double g[36];
#pragma unroll
            for (int e = 0; e < 36; ++e) g[e] = S.G[e];
            ok = elim6(g, prm.degen_thr, prm.degen_thr * S.L * S.L, nullptr, nullptr);
        }
        s_g_ok = ok;
    }
    pair_sync();
    if (tid >= 32) return;
    const int g_ok = s_g_ok;
    if (!g_ok) {
        // the sensor basis and its inverse, which the degenerate step works in (odom.py:425-433, 436-455), at
        // the current pose's position (not the pass centre S.c, which stays at the prediction)
        const double cT[3] = {S.T[3], S.T[7], S.T[11]};
        const double invL = 1.0 / S.L;
        for (int e = lane; e < 36; e += 32) {
            const int p = e / 6, q = e % 6, i = p % 3, j = q % 3;
            S.G[e] *= (p >= 3 ? invL : 1.0) * (q >= 3 ? invL : 1.0);  // the sensor-basis scaling of G
            S.SB[e] = S.SB0[e] * (q >= 3 ? invL : 1.0);
            double sbi = 0.0;
            if (p < 3 && q < 3) {
                sbi = S.T[j * 4 + i];
            } else if (p < 3) {
                double rc = 0.0;  // (R^T [c]x)[i][j]
                for (int k = 0; k < 3; ++k) rc -= S.T[k * 4 + i] * kneg(cT, k, j);
                sbi = -rc;
            } else if (q >= 3) {
                sbi = S.L * S.T[j * 4 + i];
            }
            S.SBi[e] = sbi;
        }
        __syncwarp();
        const bool warm = S.have_v != 0;
        if (warm) {
            // start from an earlier iteration's vectors: V^T G V is nearly diagonal, so fewer sweeps
            for (int e = lane; e < 36; e += 32) {
                const int i = e / 6, j = e % 6;
                double t = 0.0;
                for (int k = 0; k < 6; ++k) t += S.G[i * 6 + k] * S.EV[k * 6 + j];
                S.tmp[e] = t;
            }
            __syncwarp();
            for (int e = lane; e < 36; e += 32) {
                const int i = e / 6, j = e % 6;
                if (i > j) continue;
                double t = 0.0;
                for (int k = 0; k < 6; ++k) t += S.EV[k * 6 + i] * S.tmp[k * 6 + j];
                S.EA[i * 6 + j] = t;
                S.EA[j * 6 + i] = t;
            }
        } else {
            S.EA[lane] = S.G[lane];
            if (lane < 4) S.EA[lane + 32] = S.G[lane + 32];
        }
        __syncwarp();
        jacobi6_warp<true>(S.EA, S.EV, S.ev, S.rot, warm);
        if (lane == 0) S.have_v = 1;
        gn_degenerate_warp(S, prm.degen_thr);
    }
    if (lane == 0) {
        int st = 0;
        if (!g_ok) {
            st = S.dstat;
            for (int i = 0; i < 6; ++i) delta[i] = S.delta[i];
        } else if (!s_a_ok) {
            st = 3;
        }
        if (st == 0) {
            apply_twist(S.T, delta);
            const double nt = delta[0] * delta[0] + delta[1] * delta[1] + delta[2] * delta[2];
            const double nr = delta[3] * delta[3] + delta[4] * delta[4] + delta[5] * delta[5];
            st = (nt < 1e-8 && nr < 1e-8) ? 1 : 0;  // |step| < STEP_TOL (odom.py:88), squared
        }
        S.status = st;
    }
}

// The frame's deskew and thinning (odom.py:126-178), run by the registration's own launch as its first three
// grid-barrier episodes instead of as three kernels before it. Each CTA takes a contiguous run of the frame's
// points, a thread every 256th of them:
//   A  deskews f_raw into f_xyz and claims each point's half-voxel, keeping the lowest claiming index per slot;
//   B  keeps the points that won their slot and publishes the CTA's count;
//   C  writes the kept points to ds_xyz at the CTA's offset (the counts of the CTAs before it) in point order,
//      and clears the slots for the next frame.
// The result is the kernels' (k_thin_a/b/c): the same points in the same order.
struct GnThin {
    lw_frame_buf fb;
    ThinArgs a;      // a.deskew: deskew f_raw into f_xyz in pass A
    Tw6 tw;          // the deskew twist unless from_state
    RegBegin b;      // begin: the registration's start state and the frame's size
    int on;          // 0: no thinning, the launch registers ds and *n_dev as given
    int from_state;  // 1: twist, t_mid and the point count from the state (the sequence's frames)
    int begin;       // 1: CTA 0 writes b into the state (reg_begin) and the launch starts from b.T
    // a frame read from the host: pass A reads x, y, z [m*3], t [m] and attr [m] through these device pointers of
    // pinned host memory instead of f_raw and f_attr (null: from the frame buffer)
    const float* src3;
    const float* src_t;
    const uint32_t* src_attr;
    // the state and the error flag written to pinned host memory at the end of the launch (null: not)
    lw_odom_state* out_st;
    int32_t* out_err;
};

// Counts out every CTA after its last barrier read; the last one out zeroes the barrier words, so the next launch
// starts from a clean count whether or not this one completed. With th.out_st, the last one out also copies the
// state and the error flag to the caller's pinned host memory: every CTA's writes to them (the state by CTA 0, the
// flag by any CTA that gave up) precede its count by a fence, and the last CTA's fence follows all the counts.
__device__ __forceinline__ void gn_exit(uint32_t* bar, const lw_odom_state* st, const int32_t* err, const GnThin& th) {
    __shared__ int s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        if (th.out_st) __threadfence();
        const uint32_t prev = atomicAdd(bar + 1, 1u);
        const int last = prev == gridDim.x - 1;
        if (last) {
            atomicExch(bar, 0u);
            atomicExch(bar + 1, 0u);
            if (th.out_st) __threadfence();
        }
        s_last = last;
    }
    __syncthreads();
    if (th.out_st && s_last && threadIdx.x < 32) {
        const unsigned long long* a = reinterpret_cast<const unsigned long long*>(st);
        unsigned long long* o = reinterpret_cast<unsigned long long*>(th.out_st);
        constexpr int W = (int)(sizeof(lw_odom_state) / 8);
        for (int e = threadIdx.x; e < W; e += 32) o[e] = *(volatile const unsigned long long*)(a + e);
        if (threadIdx.x == 0 && th.out_err) *th.out_err = *(volatile const int32_t*)err;
    }
}

// Passes A-C; returns the number of thinned points, or -1 when the launch ends here (thinning not gated in, or a
// barrier gave up). `run`: the launch's gate; pass A still deskews without it for the first registration of a
// sequence frame (the frame's map insert reads f_xyz).
__device__ __forceinline__ int gn_thin(const GnThin& th, lw_odom_state* st, const lw_gn_scratch& gn, int which,
                                       bool run, long long budget) {
    const lw_frame_buf& fb = th.fb;
    const bool deskew = th.a.deskew && (run || which != 1);
    if (!deskew && !run) return -1;
    int64_t m = th.from_state ? (int64_t)st->m : (int64_t)th.b.m;
    if (m > fb.cap) m = fb.cap;
    if (m < 0) m = 0;
    float tw[6];
    float t_mid = th.a.t_mid;
    if (th.from_state) {
#pragma unroll
        for (int k = 0; k < 6; ++k) tw[k] = st->xi_used[k];
        t_mid = (float)st->t_mid;
    } else {
#pragma unroll
        for (int k = 0; k < 6; ++k) tw[k] = th.tw.v[k];
    }
    const int G = gridDim.x;
    const int64_t chunk = (m + G - 1) / G;
    const int64_t lo = (int64_t)blockIdx.x * chunk;
    const int64_t hi = lo + chunk < m ? lo + chunk : m;
    const int tid = threadIdx.x;
    const int mask = (int)(fb.ds_cap - 1);
    long long* fixed = reinterpret_cast<long long*>(gn.part);
    int* counts = reinterpret_cast<int*>(fixed + 3 * LW_ACC_STRIDE);  // [G] kept points per CTA
    __shared__ int s_sm[33];
    __shared__ int s_base, s_total;
    if (blockIdx.x == 0) {
        if (th.begin) reg_begin(st, th.b);
        // the fixed-point sums of the first two iterations start at zero (the loop clears the third)
        if (run && tid < 2 * LW_ACC_STRIDE) fixed[tid] = 0;
    }
    // A: deskew, claim; the thread's first point and slot stay in registers for B and C, the rest go to ds_slot. A
    // warp takes 32 consecutive points per round (the rounds are uniform over the warp).
    float4 p0 = make_float4(0.f, 0.f, 0.f, 0.f);
    int slot0 = -1;
    const int lane = tid & 31;
    for (int64_t b0 = lo + (tid & ~31); b0 < hi; b0 += GN_THREADS) {
        const int64_t i = b0 + lane;
        const bool valid = i < hi;
        float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
        uint32_t at = 0;
        if (th.src3) {
            // from pinned host memory, every byte crossing the bus once: the warp's points' x, y, z are 96
            // consecutive floats, read as three coalesced rows and handed to their lanes by shuffles
            float v[3];
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const int64_t e = 3 * b0 + 32 * r + lane;
                v[r] = e < 3 * hi ? th.src3[e] : 0.0f;
            }
            float c[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const int e = 3 * lane + k;
                const float a0 = __shfl_sync(0xffffffffu, v[0], e & 31);
                const float a1 = __shfl_sync(0xffffffffu, v[1], e & 31);
                const float a2 = __shfl_sync(0xffffffffu, v[2], e & 31);
                c[k] = e < 32 ? a0 : (e < 64 ? a1 : a2);
            }
            if (valid) {
                at = th.src_attr[i];
                p = deskew_point(make_float4(c[0], c[1], c[2], th.src_t[i]), t_mid, th.a.inv_dt, tw);
                reinterpret_cast<float4*>(fb.f_xyz)[i] = p;
            }
        } else if (valid) {
            if (deskew) {
                p = deskew_point(reinterpret_cast<const float4*>(fb.f_raw)[i], t_mid, th.a.inv_dt, tw);
                reinterpret_cast<float4*>(fb.f_xyz)[i] = p;
            } else {
                p = reinterpret_cast<const float4*>(fb.f_xyz)[i];
            }
        }
        if (!run || !valid) continue;
        if (!th.src3) at = fb.f_attr[i];
        int slot = -1;
        const float r = len3(p.x, p.y, p.z);
        if (!(r < th.a.min_range || r > th.a.max_range) && tag_of(at) == 0 && ((1 << ret_of(at)) & th.a.ret_mask) != 0) {
            const int64_t key = key_ijk(ifloor(p.x * th.a.inv_v), ifloor(p.y * th.a.inv_v), ifloor(p.z * th.a.inv_v));
            slot = claim_slot_cas(key, fb.ds_keys, mask);
            if (slot >= 0) atomicMin(fb.ds_win + slot, (int)i);
        }
        if (i == lo + tid) {
            p0 = p;
            slot0 = slot;
        } else {
            fb.ds_slot[i] = slot;
        }
    }
    if (!run) return -1;
    // a barrier that gives up leaves the pass unfinished: every CTA then empties the slots its points claimed, so
    // the table is clear for the next frame whichever CTAs got how far (a slot is emptied by each of its claimers)
    auto give_up = [&]() {
        for (int64_t i = lo + tid; i < hi; i += GN_THREADS) {
            const int slot = i == lo + tid ? slot0 : fb.ds_slot[i];
            if (slot >= 0) {
                fb.ds_keys[slot] = EMPTY_KEY;
                fb.ds_win[slot] = NO_INDEX;
            }
        }
        return -1;
    };
    if ((int)blockIdx.x == gn.skip_cta) return give_up();  // injected failure: this CTA never arrives
    if (!grid_sync(gn.bar, (uint32_t)G, gn.err, 1, budget)) return give_up();
    // B: the lowest claiming index of a slot is kept; the CTA's count goes to counts[blockIdx.x]
    int keep0 = 0, kept = 0;
    for (int64_t r0 = lo; r0 < hi; r0 += GN_THREADS) {  // uniform over the CTA
        const int64_t i = r0 + tid;
        int keep = 0;
        if (i < hi) {
            const int slot = r0 == lo ? slot0 : fb.ds_slot[i];
            keep = (slot >= 0 && fb.ds_win[slot] == (int)i) ? 1 : 0;
            if (r0 == lo) keep0 = keep;
        }
        kept += __syncthreads_count(keep);
    }
    if (tid == 0) counts[blockIdx.x] = kept;
    if (!grid_sync(gn.bar, 2u * (uint32_t)G, gn.err, 1, budget)) return give_up();
    // C: this CTA's offset and the total, then the kept points in order. Each kept point empties its slot; a point
    // that is not kept reads an index other than its own there, whether or not the kept point has emptied it yet.
    if (tid < 32) {
        int before = 0, all = 0;
        for (int j = tid; j < G; j += 32) {
            const int c = *(volatile int*)(counts + j);
            all += c;
            if (j < (int)blockIdx.x) before += c;
        }
        before = warp_sum_i(before);
        all = warp_sum_i(all);
        if (tid == 0) {
            s_base = before;
            s_total = all;
        }
    }
    __syncthreads();
    int run_base = s_base;
    const int n = s_total;
    for (int64_t r0 = lo; r0 < hi; r0 += GN_THREADS) {
        const int64_t i = r0 + tid;
        int slot = -1;
        if (i < hi) {
            if (r0 == lo) {
                slot = keep0 ? slot0 : -1;
            } else {
                slot = fb.ds_slot[i];
                if (slot >= 0 && fb.ds_win[slot] != (int)i) slot = -1;
            }
        }
        const int keep = slot >= 0;
        int tot;
        const int rk = block_rank(keep, s_sm, &tot);
        if (keep) {
            const float4 p = r0 == lo ? p0 : reinterpret_cast<const float4*>(fb.f_xyz)[i];
            reinterpret_cast<float4*>(fb.ds_xyz)[run_base + rk] = make_float4(p.x, p.y, p.z, len3(p.x, p.y, p.z));
            fb.ds_keys[slot] = EMPTY_KEY;
            fb.ds_win[slot] = NO_INDEX;
        }
        run_base += tot;
    }
    if (!grid_sync(gn.bar, 3u * (uint32_t)G, gn.err, 1, budget)) return give_up();
    return n;
}

// The whole registration loop (odom.py:752-803) in one cooperative launch, with the frame's thinning before it
// when th.on. Every CTA reduces the partials and computes the same float64 step, so one grid barrier per iteration
// suffices.
__device__ __forceinline__ void gn_run(const float4* __restrict__ ds, const int* __restrict__ n_dev,
                                       const lw_odom_params& prm, lw_odom_state* st, const int64_t* __restrict__ keys,
                                       const float* __restrict__ rec, int mask, const lw_gn_scratch& gn, int which,
                                       const GnThin& th) {
    const int* gate = which == 0 ? &st->run_reg : (which == 1 ? &st->redo : nullptr);
    const bool run = !(gate && *gate == 0);  // uniform: every CTA reads the same flag before any barrier
    const long long budget = gn.spin_budget > 0 ? (long long)gn.spin_budget : BARRIER_SPINS;
    __shared__ GnSmem S;
    __shared__ int s_iters, s_degen, s_corr;
    __shared__ double s_rms_num, s_rms_den;
    extern __shared__ float4 gn_dyn[];
    IcpCache memo = icp_cache_carve(gn_dyn);
    if (threadIdx.x < GN_GROUPS) {
        memo.tag[threadIdx.x] = make_int4(0, 0, 0, 0);
        memo.best[threadIdx.x] = -1;
    }
    // the loop's start state, set up by a thread of the last warp (the one with the least thinning work) while the
    // others thin the frame
    if (threadIdx.x == GN_THREADS - 32) {
        for (int i = 0; i < 16; ++i) S.T[i] = S.Tp[i] = th.on && th.begin ? th.b.T[i] : st->T_pred[i];
        if (gn.trace && blockIdx.x == 0 && run)
            for (int i = 0; i < 12; ++i) gn.trace[i] = S.Tp[i];  // the start pose
        S.c[0] = S.Tp[3];
        S.c[1] = S.Tp[7];
        S.c[2] = S.Tp[11];
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 6; ++j)
                S.Ac[i * 6 + j] = i == j ? 1.0 : (i < 3 && j >= 3 ? kneg(S.c, i, j - 3) : 0.0);
        s_iters = 0;
        s_degen = 0;
        s_corr = 0;
        s_rms_num = 0.0;
        s_rms_den = 1.0;
        for (int i = 0; i < 36; ++i) S.H[i] = (i % 7 == 0) ? 1.0 : 0.0;
        S.have_v = 0;
    }
    int n;
    uint32_t ep0 = 0;  // grid-barrier episodes before the loop's
    if (th.on) {
        n = gn_thin(th, st, gn, which, run, budget);
        if (n < 0) return;
        ep0 = 3;
    } else {
        if (!run) return;
        n = *n_dev;
    }
    __syncthreads();
    if (n < prm.min_corr) {  // odom.py:754-757
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            for (int i = 0; i < 16; ++i) st->T_reg[i] = S.Tp[i];
            st->ok = 0;
            st->n_ds = n;
        }
        return;
    }
    const float voxel = (float)prm.reg_voxel;
    IcpConsts k;
    k.inv_v = (float)(1.0 / prm.reg_voxel);
    k.mask = mask;
    for (int it = 0; it < prm.max_iter; ++it) {
        float kappa;
        schedule(it, voxel, k.reach, k.max_d2, kappa);
        k.kappa2 = kappa * kappa;
        k.inv_kappa2 = 1.0f / k.kappa2;
        IcpPose P;
        make_pose(S.T, S.c, P);
        // cross-CTA sums in fixed point, three buffers in turn: iteration `it` adds into buffer it % 3 before the
        // barrier and reads it after; CTA 0 then clears buffer (it + 2) % 3, which nobody reads any more (its last
        // readers passed this barrier) and nobody adds to before the next barrier
        long long* fixed = reinterpret_cast<long long*>(gn.part) + (it % 3) * LW_ACC_STRIDE;
        memo.pt_ok = it > 0;
        icp_pass(ds, n, P, k, keys, rec, nullptr, fixed, gn.err, &memo);
        if (it == 0 && !th.on && (int)blockIdx.x == gn.skip_cta) return;  // injected failure: never arrives
        // while thread 0 waits, thread 32 prepares what the step needs from the pose alone
        if (!grid_sync(gn.bar, (ep0 + (uint32_t)it + 1u) * gridDim.x, gn.err, 1, budget,
                       StepPrep{&S, prm.prior_info > 0.0 ? prm.prior_info : 0.0}))
            return;
        if (blockIdx.x == 0 && threadIdx.x < LW_ACC_STRIDE)
            reinterpret_cast<long long*>(gn.part)[((it + 2) % 3) * LW_ACC_STRIDE + threadIdx.x] = 0;
        gn_reduce_fixed(fixed, S);
        if (threadIdx.x < 64) gn_step_pair(S, prm);
        __syncthreads();
        if (gn.trace && blockIdx.x == 0 && threadIdx.x < 12 && it + 1 < LW_GN_TRACE)
            gn.trace[(it + 1) * 12 + threadIdx.x] = S.T[threadIdx.x];  // the pose after iteration it
        if (threadIdx.x == 0) {  // read after the loop only (past the barrier below it)
            s_corr = S.corr;
            if (S.status != 2) {  // the rms of the last accumulation with enough matches, taken after the loop
                s_rms_num = S.v[LW_ACC_RMS];
                s_rms_den = S.v[LW_ACC_WEIGHT];
            }
            if (S.status == 0 || S.status == 1) {
                s_iters = it + 1;
                s_degen = S.degen;
            }
        }
        if (S.status != 0) break;  // S.status was written before the block barrier above
    }
    __syncthreads();  // thread 0's last s_corr, s_rms_num / _den, s_iters, s_degen
    if (blockIdx.x == 0 && threadIdx.x < 32 && s_corr >= prm.min_corr) {
        // min/max eigenvalue of H normalised by its diagonal (odom.py:797-800), by warp 0
        for (int e = threadIdx.x; e < 36; e += 32) {
            const int i = e / 6, j = e % 6;
            S.EA[e] = S.H[e] / (sqrt(fmax(S.H[i * 7], 1e-12)) * sqrt(fmax(S.H[j * 7], 1e-12)));
        }
        __syncwarp();
        const double c = cond6_warp(S.EA);
        if (threadIdx.x == 0) S.ev[0] = c;
    }
    __syncthreads();
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        bool ok = s_corr >= prm.min_corr;
        const double cond = ok ? S.ev[0] : st->cond;
        for (int i = 0; i < 16; ++i) st->T_reg[i] = S.T[i];
        st->ok = ok ? 1 : 0;
        st->n_ds = n;
        st->iters = s_iters;
        if (which == 0) st->iters_first = s_iters;
        st->corr = s_corr;
        st->rms = sqrt(fmax(s_rms_num, 0.0) / fmax(s_rms_den, 1e-9));
        st->cond = cond;
        st->degen = s_degen;
        st->weak = (cond < 1e-3 || s_degen > 0) ? 1 : 0;  // WEAK_COND (odom.py:90)
    }
}

__global__ void __launch_bounds__(GN_THREADS, 1)
    k_gn(const float4* __restrict__ ds, const int* __restrict__ n_dev, lw_odom_params prm, lw_odom_state* st,
         const int64_t* __restrict__ keys, const float* __restrict__ rec, int mask, lw_gn_scratch gn, int which,
         GnThin th) {
    gn_run(ds, n_dev, prm, st, keys, rec, mask, gn, which, th);
    gn_exit(gn.bar, st, gn.err, th);
}

// Standalone accumulation at a host pose, for the parity tests and the batched callers.
__global__ void __launch_bounds__(GN_THREADS, 1)
    k_acc_once(const float4* __restrict__ ds, const int* __restrict__ n_dev, int64_t n_ub, IcpPose P, IcpConsts k,
               const int64_t* __restrict__ keys, const float* __restrict__ rec, double* part) {
    int n = n_dev ? *n_dev : (int)n_ub;
    icp_pass(ds, n, P, k, keys, rec, part + (int64_t)blockIdx.x * LW_ACC_STRIDE);
}

__global__ void k_acc_reduce(const double* part, int grid, double c0, double c1, double c2, double* out) {
    __shared__ double v64[LW_ACC_STRIDE];
    double c[3] = {c0, c1, c2};
    reduce_partials(part, grid, c, v64);
    if (threadIdx.x < LW_ACC_STRIDE) out[threadIdx.x] = v64[threadIdx.x];
}

// =====================================================================================================
// Frame state machine (odom.py:642-694, 712-727) on one thread.
// =====================================================================================================

// The Gauss-Newton launch that follows a control kernel needs its fixed-point sums and barrier count at zero; the
// control kernel's threads clear them, so the launch needs no memsets of its own.
__device__ __forceinline__ void clear_gn_sums(long long* part, uint32_t* bar) {
    for (int e = threadIdx.x; e < 3 * LW_ACC_STRIDE; e += blockDim.x) part[e] = 0;
    if (threadIdx.x < 2) bar[threadIdx.x] = 0;
}

__global__ void k_ctl_begin(int k, lw_odom_params prm, lw_odom_state* st, const int* count, long long* part,
                            uint32_t* bar) {
    clear_gn_sums(part, bar);
    if (threadIdx.x != 0) return;
    int m = *count;
    if (m > prm.frame_cap) m = prm.frame_cap;
    st->m = m;
    st->frame_k = k;
    int warm = st->map_frames < prm.warmup;
    st->warm = warm;
    st->t_mid = ((double)k + 0.5) * prm.frame_dt;
    for (int j = 0; j < 6; ++j) st->xi_used[j] = (prm.deskew && !warm) ? st->xi[j] : 0.0f;
    double Ts[16];
    if (warm) {
        for (int i = 0; i < 16; ++i) Ts[i] = st->T[i];
    } else {
        mat44_mul(st->T, st->delta, Ts);  // predict() (odom.py:591-592)
    }
    for (int i = 0; i < 16; ++i) st->T_pred[i] = st->T_reg[i] = Ts[i];
    st->redo = 0;
    st->do_insert = 0;
    st->run_reg = 0;
    st->iters_first = 0;
    if (m < prm.min_points) {
        st->skipped += 1;
        st->ok = 0;
    } else if (warm) {
        st->ok = 1;  // the map is still filling in: assume the sensor holds still
    } else {
        st->run_reg = 1;
    }
}

// After the first registration: deskew again with the frame's own motion when it differs (odom.py:673-679).
__global__ void k_ctl_mid(lw_odom_params prm, lw_odom_state* st, long long* part, uint32_t* bar) {
    clear_gn_sums(part, bar);
    if (threadIdx.x != 0) return;
    st->redo = 0;
    if (!(st->run_reg && st->ok && prm.deskew && prm.redeskew && st->has_prev)) return;
    double Ti[16], D[16], xn[6];
    mat44_inv_rigid(st->T_prev, Ti);
    mat44_mul(Ti, st->T_reg, D);
    body_twist(D, xn);
    float xf[6];
    for (int j = 0; j < 6; ++j) xf[j] = (float)xn[j];
    float dr0 = xf[3] - st->xi_used[3], dr1 = xf[4] - st->xi_used[4], dr2 = xf[5] - st->xi_used[5];
    float dt0 = xf[0] - st->xi_used[0], dt1 = xf[1] - st->xi_used[1], dt2 = xf[2] - st->xi_used[2];
    float nr = sqrtf(dr0 * dr0 + dr1 * dr1 + dr2 * dr2), nt = sqrtf(dt0 * dt0 + dt1 * dt1 + dt2 * dt2);
    if (nr > 2e-3f || nt > 5e-3f) {  // REDESKEW_ROT / REDESKEW_TRANS (odom.py:92-93)
        for (int j = 0; j < 6; ++j) st->xi_used[j] = xf[j];
        for (int i = 0; i < 16; ++i) st->T_pred[i] = st->T_reg[i];
        st->redo = 1;
    }
}

// Keyframe decision, velocity update, pose table and trajectory (odom.py:648-657, 682-694, 712-717).
__global__ void k_ctl_end(lw_odom_params prm, lw_odom_state* st, lw_pose_table pt, int epoch, lw_traj_rec* traj,
                          int64_t traj_cap, const int* gn_err) {
    if (*gn_err != 0) {  // a registration gave up (a bounded wait ran out, or its sums overflowed): not trusted
        st->err = *gn_err;
        st->ok = 0;
    }
    double T[16];
    for (int i = 0; i < 16; ++i) T[i] = st->T_reg[i];
    int warm = st->warm;
    int ins = 0;
    if (st->ok) {
        if (warm || !st->has_key) {
            ins = 1;
        } else {
            double Ki[16], D[16], R[9], rv[3];
            mat44_inv_rigid(st->T_key, Ki);
            mat44_mul(Ki, T, D);
            mat44_rot(D, R);
            mat_to_rotvec(R, rv);
            double ang = sqrt(rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2]) * (180.0 / 3.14159265358979323846);
            double dist = sqrt(D[3] * D[3] + D[7] * D[7] + D[11] * D[11]);
            ins = (dist >= prm.kf_dist || ang >= prm.kf_angle_deg) ? 1 : 0;
        }
    }
    st->do_insert = ins;
    if (ins) {
        st->map_frames += 1;
        for (int i = 0; i < 16; ++i) st->T_key[i] = T[i];
        st->has_key = 1;
        st->keyframes += 1;
    }
    if (st->has_prev && !warm) {
        double Ti[16], D[16];
        mat44_inv_rigid(st->T_prev, Ti);
        mat44_mul(Ti, T, D);
        double jump = sqrt(D[3] * D[3] + D[7] * D[7] + D[11] * D[11]);
        if (jump < 1.5) {  // MAX_FRAME_JUMP (odom.py:94)
            double xd[6];
            body_twist(D, xd);
            for (int j = 0; j < 6; ++j) st->xi[j] = (float)xd[j];
            if (prm.velocity_smooth > 0.0) {
                double a = prm.velocity_smooth;
                for (int j = 0; j < 6; ++j) st->xi_s[j] = a * st->xi_s[j] + (1.0 - a) * (double)st->xi[j];
                twist_matrix(st->xi_s, st->delta);
            } else {
                for (int i = 0; i < 16; ++i) st->delta[i] = D[i];
            }
        } else {  // a failure, not motion: predict rest from here
            mat44_eye(st->delta);
            for (int j = 0; j < 6; ++j) {
                st->xi[j] = 0.0f;
                st->xi_s[j] = 0.0;
            }
        }
    }
    for (int i = 0; i < 16; ++i) st->T_prev[i] = st->T[i] = T[i];
    st->has_prev = 1;
    int k = st->frame_k;
    int j = k & (LW_POSE_SLOTS - 1);
    for (int i = 0; i < 16; ++i) pt.poses[j * 16 + i] = (float)T[i];
    for (int i = 0; i < 6; ++i) pt.tw[j * 6 + i] = st->xi_used[i];
    pt.owner_frame[j] = k;
    pt.owner_epoch[j] = epoch;
    if (traj && traj_cap > 0) {
        lw_traj_rec* r = traj + (st->traj_len % traj_cap);
        for (int i = 0; i < 16; ++i) r->T[i] = T[i];
        r->t_mid = st->t_mid;
        r->k = k;
        r->ok = st->ok;
        r->iters = st->run_reg ? st->iters : 0;
        r->iters_first = st->run_reg ? st->iters_first : 0;
        r->corr = st->run_reg ? st->corr : 0;
    }
    st->traj_len += 1;
    st->frames += 1;
}

__global__ void k_predict_poses(int k0, int k1, int current, const lw_odom_state* st, lw_pose_table pt, int epoch) {
    __shared__ float P[16];
    if (threadIdx.x == 0) {
        double Tp[16];
        if (current & 1) {
            for (int i = 0; i < 16; ++i) Tp[i] = st->T[i];
        } else {
            mat44_mul(st->T, st->delta, Tp);
        }
        for (int i = 0; i < 16; ++i) P[i] = (float)Tp[i];
    }
    __syncthreads();
    if (k1 - k0 > LW_POSE_SLOTS) k0 = k1 - LW_POSE_SLOTS;
    for (int k = k0 + (int)(blockIdx.x * blockDim.x + threadIdx.x); k < k1; k += gridDim.x * blockDim.x) {
        int j = k & (LW_POSE_SLOTS - 1);
        for (int i = 0; i < 16; ++i) pt.poses[j * 16 + i] = P[i];
        for (int i = 0; i < 6; ++i) pt.tw[j * 6 + i] = (current & 2) ? 0.0f : st->xi[i];
        pt.owner_frame[j] = k;
        pt.owner_epoch[j] = epoch;
    }
}

__global__ void k_reset_state(lw_odom_state* st, lw_odom_state init) { *st = init; }

// The start of a single-frame registration (lw_register_frame): the prediction, the frame's point count, its
// mid time and the twist it is deskewed with, into the device state.

__global__ void k_reg_begin(lw_odom_state* st, RegBegin b) { reg_begin(st, b); }

__global__ void k_zero_count(int* c) { *c = 0; }

__global__ void k_restart_clock(lw_odom_state* st) {
    st->has_prev = 0;
    mat44_eye(st->delta);
    for (int j = 0; j < 6; ++j) {
        st->xi[j] = 0.0f;
        st->xi_s[j] = 0.0;
    }
}

__global__ void k_fill_i64(int64_t* a, int64_t n, int64_t v) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) a[i] = v;
}
__global__ void k_fill_i32(int32_t* a, int64_t n, int32_t v) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) a[i] = v;
}

}  // namespace lw

// =========================================================================================================
// C ABI
// =========================================================================================================
using namespace lw;

static int gn_grid(const lw_gn_scratch* gn) {
    int sms = device_sms();
    int g = gn->grid;
    if (g <= 0 || g > sms) g = sms;
    return g;
}

static ThinArgs thin_args(const lw_odom_params* prm) {
    ThinArgs a;
    a.inv_v = (float)(2.0 / prm->reg_voxel);
    a.min_range = (float)prm->min_range;
    a.max_range = (float)prm->max_range;
    a.ret_mask = prm->ret_mask;
    a.deskew = 1;
    a.t_mid = 0.0f;
    a.inv_dt = (float)(1.0 / prm->frame_dt);
    return a;
}

static lw_rec_params rec_params(const lw_odom_params* prm) {
    lw_rec_params rp;
    rp.voxel = (float)prm->reg_voxel;
    double tf = 0.6 * prm->reg_voxel / sqrt(12.0);  // TIGHT_FRACTION (odom.py:89, 761)
    rp.tight2 = (float)(tf * tf);
    rp.noise2 = (float)(prm->noise * prm->noise);
    rp.alpha = (float)prm->alpha;
    return rp;
}

// th: the frame's thinning, done by the launch before its loop (th->on), or nullptr to register ds4 and *n_dev as
// they are. cleared: the fixed-point sums of the first two iterations are already zero (a thinning launch clears
// them itself).
static int launch_gn(const float* ds4, const int32_t* n_dev, const lw_odom_params* prm, lw_odom_state* st,
                     const lw_regmap* reg, lw_gn_scratch* gn, int which, cudaStream_t s, bool cleared = false,
                     const GnThin* th = nullptr) {
    if (reg->cap > (1LL << SLOT_BITS))
        return set_error(LW_EINVAL, "Gauss-Newton: a registration map of %lld slots (at most 2^25)", (long long)reg->cap);
    if (gn->grid < 2)  // the scratch holds 2 * grid accumulators; the loop's sums and the thinning counts need 4
        return set_error(LW_EINVAL, "Gauss-Newton: a scratch of %d CTAs (at least two)", (int)gn->grid);
    int grid = gn_grid(gn);
    lw_gn_scratch g = *gn;
    g.grid = grid;
    const float4* dsp = reinterpret_cast<const float4*>(ds4);
    int mask = (int)(reg->cap - 1);
    const int64_t* keys = reg->keys;
    const float* rec = reg->rec;
    lw_odom_params p = *prm;
    GnThin t{};
    if (th) t = *th;
    void* args[] = {(void*)&dsp, (void*)&n_dev, (void*)&p, (void*)&st, (void*)&keys, (void*)&rec,
                    (void*)&mask, (void*)&g, (void*)&which, (void*)&t};
    // the fixed-point accumulators of the first two iterations start at zero (the kernel clears the rest; a
    // thinning launch clears them all); the barrier words are zero from the previous launch's exit
    if (!cleared && !t.on) {
        LW_CUDA(cudaMemsetAsync(gn->part, 0, 3 * LW_ACC_STRIDE * sizeof(long long), s));
        LW_CUDA(cudaMemsetAsync(gn->bar, 0, 2 * sizeof(uint32_t), s));
    }
    static bool smem_set[64] = {};  // the memo's dynamic shared memory is above the default 48 KB
    int dev = 0;
    LW_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64 || !smem_set[dev]) {
        LW_CUDA(cudaFuncSetAttribute((const void*)k_gn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GN_DYN_SMEM));
        if (dev >= 0 && dev < 64) smem_set[dev] = true;
    }
    LW_CUDA(cudaLaunchCooperativeKernel((const void*)k_gn, dim3(grid), dim3(GN_THREADS), args, GN_DYN_SMEM, s));
    count_launches(1);
    return LW_OK;
}

extern "C" {

int lw_frame_append(const float* xyz, int32_t xyz_stride, const uint32_t* attr, const float* t, int64_t n,
                    double inv_dt, int32_t k_min, int32_t k_open, lw_frame_buf* fb, void* stream) {
    if (n <= 0) return LW_OK;
    if (!xyz || !attr || !t || !fb || (xyz_stride != 3 && xyz_stride != 4))
        return set_error(LW_EINVAL, "lw_frame_append: bad arguments (stride %d)", xyz_stride);
    cudaStream_t s = (cudaStream_t)stream;
    int nt = blocks_for(n, TILE);
    if ((int64_t)nt > fb->cap / TILE + 1 && nt > 1) {
        // the tile scratch holds cap/TILE + 1 counts; a larger batch is appended in frame-sized chunks
        int64_t chunk = (fb->cap / TILE) * TILE;
        if (chunk <= 0) chunk = TILE;
        for (int64_t off = 0; off < n; off += chunk) {
            int64_t c = n - off < chunk ? n - off : chunk;
            int r = lw_frame_append(xyz + off * xyz_stride, xyz_stride, attr + off, t + off, c, inv_dt, k_min, k_open,
                                    fb, stream);
            if (r != LW_OK) return r;
        }
        return LW_OK;
    }
    float idt = (float)inv_dt;
    ProfScope prof("frame_append", s);
    k_append_count<<<nt, TILE, 0, s>>>(t, n, idt, k_min, k_open, fb->tiles);
    if (xyz_stride == 3)
        k_append_scatter<3><<<nt, TILE, 0, s>>>(xyz, attr, t, n, idt, k_min, k_open, fb->tiles, *fb);
    else
        k_append_scatter<4><<<nt, TILE, 0, s>>>(xyz, attr, t, n, idt, k_min, k_open, fb->tiles, *fb);
    k_append_total<<<1, 256, 0, s>>>(fb->tiles, nt, fb->count);
    LW_LAUNCHED("lw_frame_append");
    count_launches(3);
    return LW_OK;
}

int lw_frame_reset(lw_frame_buf* fb, void* stream) {
    k_zero_count<<<1, 1, 0, (cudaStream_t)stream>>>(fb->count);
    LW_LAUNCHED("lw_frame_reset");
    count_launches(1);
    return LW_OK;
}


int lw_deskew(const float* raw, float* out, const int32_t* m_dev, int64_t m_ub, double t_mid, double inv_dt,
              const float* twist6_host, void* stream) {
    if (!raw || !out || !m_dev || !twist6_host) return set_error(LW_EINVAL, "lw_deskew: null argument");
    if (m_ub <= 0) return LW_OK;
    lw_frame_buf fb{};
    fb.f_raw = const_cast<float*>(raw);
    fb.f_xyz = out;
    fb.cap = m_ub;
    ThinArgs a{};
    a.deskew = 1;
    a.t_mid = (float)t_mid;
    a.inv_dt = (float)inv_dt;
    Tw6 tw;
    for (int k = 0; k < 6; ++k) tw.v[k] = twist6_host[k];
    int grid = blocks_for(m_ub, 256, 8 * device_sms());
    k_thin_a<<<grid, 256, 0, (cudaStream_t)stream>>>(fb, m_dev, a, nullptr, tw, nullptr, nullptr, 0, ThinBegin{});
    LW_LAUNCHED("lw_deskew");
    count_launches(1);
    return LW_OK;
}

int lw_thin(lw_frame_buf* fb, const int32_t* m_dev, int64_t m_ub, double inv_v, double min_range, double max_range,
            int32_t ret_mask, int32_t* n_ds_dev, void* stream) {
    if (!fb || !m_dev || !n_ds_dev) return set_error(LW_EINVAL, "lw_thin: null argument");
    if (m_ub > fb->cap) m_ub = fb->cap;
    cudaStream_t s = (cudaStream_t)stream;
    ThinArgs a{};
    a.inv_v = (float)inv_v;
    a.min_range = (float)min_range;
    a.max_range = (float)max_range;
    a.ret_mask = ret_mask;
    a.deskew = 0;
    Tw6 tw{};
    int grid = blocks_for(m_ub, 256, 8 * device_sms());
    int nt = blocks_for(m_ub, TILE);
    k_thin_a<<<grid, 256, 0, s>>>(*fb, m_dev, a, nullptr, tw, nullptr, nullptr, 1, ThinBegin{});
    k_thin_b<<<nt, TILE, 0, s>>>(*fb, m_dev, nullptr);
    k_thin_c<<<nt, TILE, 0, s>>>(*fb, m_dev, n_ds_dev, nullptr);
    LW_LAUNCHED("lw_thin");
    count_launches(3);
    return LW_OK;
}

static RegArgs reg_args(const double* T_host, double reg_voxel, double max_range, int ret_mask) {
    RegArgs a;
    for (int k = 0; k < 12; ++k) a.T[k] = T_host ? (float)T_host[k] : 0.0f;
    a.inv_v = (float)(1.0 / reg_voxel);
    a.voxel = (float)reg_voxel;
    a.max_range = (float)max_range;
    a.ret_mask = ret_mask;
    return a;
}

static int reg_insert_launch(const float* xyz4, const uint32_t* attr, const int32_t* n_dev, int64_t n_ub,
                             const double* T_host, const double* T_dev, double voxel, double max_range,
                             int32_t ret_mask, lw_regmap* reg, const lw_rec_params* rp, int32_t* pslot,
                             const int* gate, cudaStream_t s) {
    RegArgs a = reg_args(T_host, voxel, max_range, ret_mask);
    int grid = blocks_for(n_ub, 256, 8 * device_sms());
    const float4* p4 = reinterpret_cast<const float4*>(xyz4);
    k_reg_a<<<grid, 256, 0, s>>>(p4, attr, n_dev, n_ub, a, T_dev, *reg, pslot, gate);
    k_reg_b<<<grid, 256, 0, s>>>(p4, n_dev, n_ub, a, T_dev, *reg, pslot, gate);
    k_reg_d<<<grid, 256, 0, s>>>(n_dev, n_ub, *reg, pslot, *rp, gate);
    LW_LAUNCHED("reg insert");
    count_launches(3);
    return LW_OK;
}

int lw_reg_insert(const float* xyz4, const uint32_t* attr, const int32_t* n_dev, int64_t n_ub, const double* T_host,
                  double voxel, double max_range, int32_t ret_mask, lw_regmap* reg, const lw_rec_params* rp,
                  int32_t* pslot, void* stream) {
    if (!xyz4 || !attr || !reg || !rp || !pslot || !T_host) return set_error(LW_EINVAL, "lw_reg_insert: null argument");
    if ((reg->cap & (reg->cap - 1)) != 0) return set_error(LW_EINVAL, "lw_reg_insert: capacity not a power of two");
    if (n_ub <= 0) return LW_OK;
    return reg_insert_launch(xyz4, attr, n_dev, n_ub, T_host, nullptr, voxel, max_range, ret_mask, reg, rp, pslot,
                             nullptr, (cudaStream_t)stream);
}

int lw_reg_refresh_all(lw_regmap* reg, const lw_rec_params* rp, void* stream) {
    if (!reg || !rp) return set_error(LW_EINVAL, "lw_reg_refresh_all: null argument");
    k_reg_refresh_all<<<4 * device_sms(), 256, 0, (cudaStream_t)stream>>>(*reg, *rp);
    LW_LAUNCHED("lw_reg_refresh_all");
    count_launches(1);
    return LW_OK;
}

int lw_icp_accumulate(const float* ds4, const int32_t* n_dev, int64_t n_ub, const double* T_host, const lw_regmap* reg,
                      float voxel, int32_t reach, float max_d2, float kappa, lw_gn_scratch* gn, double* out64,
                      void* stream) {
    if (!ds4 || !T_host || !reg || !gn || !out64) return set_error(LW_EINVAL, "lw_icp_accumulate: null argument");
    if (reach != 1 && reach != 2) return set_error(LW_EINVAL, "lw_icp_accumulate: reach must be 1 or 2");
    if (reg->cap > (1LL << SLOT_BITS))
        return set_error(LW_EINVAL, "lw_icp_accumulate: a registration map of %lld slots (at most 2^25)", (long long)reg->cap);
    if (gn->grid < 1) return set_error(LW_EINVAL, "lw_icp_accumulate: a scratch of %d CTAs", (int)gn->grid);
    cudaStream_t s = (cudaStream_t)stream;
    int grid = gn_grid(gn);
    IcpPose P;
    double c[3] = {T_host[3], T_host[7], T_host[11]};
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) P.R[i * 3 + j] = (float)T_host[i * 4 + j];
        P.tr[i] = (float)(T_host[i * 4 + 3] - c[i]);
        P.c[i] = (float)c[i];
    }
    double cf[3] = {(double)P.c[0], (double)P.c[1], (double)P.c[2]};
    IcpConsts k;
    k.inv_v = (float)(1.0 / (double)voxel);
    k.max_d2 = max_d2;
    k.kappa2 = kappa * kappa;
    k.inv_kappa2 = 1.0f / k.kappa2;
    k.reach = reach;
    k.mask = (int)(reg->cap - 1);
    k_acc_once<<<grid, GN_THREADS, 0, s>>>(reinterpret_cast<const float4*>(ds4), n_dev, n_ub, P, k, reg->keys,
                                           reg->rec, gn->part);
    k_acc_reduce<<<1, LW_ACC_STRIDE, 0, s>>>(gn->part, grid, cf[0], cf[1], cf[2], out64);
    LW_LAUNCHED("lw_icp_accumulate");
    count_launches(2);
    return LW_OK;
}

int lw_icp_solve(const float* ds4, const int32_t* n_dev, const lw_odom_params* prm, lw_odom_state* st,
                 const lw_regmap* reg, lw_gn_scratch* gn, void* stream) {
    if (!ds4 || !n_dev || !prm || !st || !reg || !gn) return set_error(LW_EINVAL, "lw_icp_solve: null argument");
    ProfScope prof("gn", (cudaStream_t)stream);
    return launch_gn(ds4, n_dev, prm, st, reg, gn, 2, (cudaStream_t)stream);  // ungated
}

int lw_read_state(const lw_odom_state* st_dev, const int32_t* err_dev, lw_odom_state* st_host, int32_t* err_host,
                  void* stream) {
    if (!st_dev || !st_host) return set_error(LW_EINVAL, "lw_read_state: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    LW_CUDA(cudaMemcpyAsync(st_host, st_dev, sizeof(lw_odom_state), cudaMemcpyDeviceToHost, s));
    if (err_dev && err_host) LW_CUDA(cudaMemcpyAsync(err_host, err_dev, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    LW_CUDA(cudaStreamSynchronize(s));
    return LW_OK;
}

int lw_register_frame(const float* raw4, const uint32_t* attr, int64_t m, double t_mid, const float* twist6_host,
                      const double* T_pred_host, const lw_odom_params* prm, lw_odom_state* st, lw_frame_buf* fb,
                      const lw_regmap* reg, lw_gn_scratch* gn, void* stream) {
    if (!raw4 || !attr || !twist6_host || !T_pred_host || !prm || !st || !fb || !reg || !gn)
        return set_error(LW_EINVAL, "lw_register_frame: null argument");
    if (((uintptr_t)raw4 & 15) != 0) return set_error(LW_EINVAL, "lw_register_frame: raw4 is not 16-byte aligned");
    if (m < 0 || m > fb->cap)
        return set_error(LW_ECAPACITY, "lw_register_frame: %lld points, frame capacity %lld", (long long)m,
                         (long long)fb->cap);
    cudaStream_t s = (cudaStream_t)stream;
    RegBegin b;
    for (int i = 0; i < 16; ++i) b.T[i] = T_pred_host[i];
    for (int i = 0; i < 6; ++i) b.tw[i] = twist6_host[i];
    b.t_mid = t_mid;
    b.m = (int)m;
    // the frame buffer reads the caller's points in place; the launch deskews them into f_xyz and thins them into
    // ds_xyz (its CTA 0 also sets up the registration's state) before the Gauss-Newton loop
    GnThin th{};
    th.fb = *fb;
    th.fb.f_raw = const_cast<float*>(raw4);
    th.fb.f_attr = const_cast<uint32_t*>(attr);
    th.a = thin_args(prm);
    th.a.t_mid = (float)t_mid;
    for (int k = 0; k < 6; ++k) th.tw.v[k] = twist6_host[k];
    th.b = b;
    th.on = 1;
    th.from_state = 0;
    th.begin = 1;
    ProfScope prof("gn", s);
    return launch_gn(fb->ds_xyz, &st->n_ds, prm, st, reg, gn, 2, s, /*cleared=*/true, &th);
}

// A device pointer for pinned host memory (the caller's buffer as the kernel reads or writes it), or null with the
// error set when the memory is not pinned host memory this device can reach.
static void* mapped(const void* host, const char* what) {
    void* dev = nullptr;
    cudaError_t e = cudaHostGetDevicePointer(&dev, const_cast<void*>(host), 0);
    if (e != cudaSuccess || !dev) {
        cudaGetLastError();
        set_error(LW_EINVAL, "lw_register_frame_host: %s is not pinned host memory mapped for the device", what);
        return nullptr;
    }
    return dev;
}

int lw_register_frame_host(const float* xyz3, const float* t, const uint32_t* attr, int64_t m, double t_mid,
                           const float* twist6_host, const double* T_pred_host, const lw_odom_params* prm,
                           lw_odom_state* st, lw_frame_buf* fb, const lw_regmap* reg, lw_gn_scratch* gn,
                           lw_odom_state* st_out, int32_t* err_out, void* stream) {
    if (!xyz3 || !t || !attr || !twist6_host || !T_pred_host || !prm || !st || !fb || !reg || !gn || !st_out || !err_out)
        return set_error(LW_EINVAL, "lw_register_frame_host: null argument");
    if (m < 0 || m > fb->cap)
        return set_error(LW_ECAPACITY, "lw_register_frame_host: %lld points, frame capacity %lld", (long long)m,
                         (long long)fb->cap);
    GnThin th{};
    th.src3 = static_cast<const float*>(mapped(xyz3, "xyz3"));
    th.src_t = static_cast<const float*>(mapped(t, "t"));
    th.src_attr = static_cast<const uint32_t*>(mapped(attr, "attr"));
    th.out_st = static_cast<lw_odom_state*>(mapped(st_out, "st_out"));
    th.out_err = static_cast<int32_t*>(mapped(err_out, "err_out"));
    if (!th.src3 || !th.src_t || !th.src_attr || !th.out_st || !th.out_err) return LW_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    for (int i = 0; i < 16; ++i) th.b.T[i] = T_pred_host[i];
    for (int i = 0; i < 6; ++i) th.b.tw[i] = twist6_host[i];
    th.b.t_mid = t_mid;
    th.b.m = (int)m;
    th.fb = *fb;
    th.a = thin_args(prm);
    th.a.t_mid = (float)t_mid;
    for (int k = 0; k < 6; ++k) th.tw.v[k] = twist6_host[k];
    th.on = 1;
    th.from_state = 0;
    th.begin = 1;
    ProfScope prof("gn", s);
    return launch_gn(fb->ds_xyz, &st->n_ds, prm, st, reg, gn, 2, s, /*cleared=*/true, &th);
}

// The frame's queue of launches; with `net`, the learned start pose replaces the constant-velocity one between
// the first thinning and the first registration.
static int finalize_impl(int32_t k, int64_t m_ub, const lw_odom_params* prm, lw_odom_state* st, lw_frame_buf* fb,
                         lw_regmap* reg, lw_gn_scratch* gn, lw_pose_table* pt, int32_t epoch, lw_traj_rec* traj,
                         int64_t traj_cap, const lw_initnet* net, lw_net_work* work, void* stream) {
    if (!prm || !st || !fb || !reg || !gn || !pt) return set_error(LW_EINVAL, "lw_odom_finalize: null argument");
    if ((reg->cap & (reg->cap - 1)) != 0 || (fb->ds_cap & (fb->ds_cap - 1)) != 0 || fb->ds_cap < fb->cap)
        return set_error(LW_EINVAL, "lw_odom_finalize: table capacities must be powers of two (ds_cap >= cap)");
    if (prm->frame_cap != fb->cap) return set_error(LW_EINVAL, "lw_odom_finalize: frame_cap != frame buffer capacity");
    cudaStream_t s = (cudaStream_t)stream;
    if (m_ub > fb->cap) m_ub = fb->cap;
    if (m_ub < 1) m_ub = 1;
    const int sms = device_sms();
    const int grid = blocks_for(m_ub, 256, 8 * sms);
    const int nt = blocks_for(m_ub, TILE);
    ThinArgs ta = thin_args(prm);
    Tw6 tw{};
    lw_rec_params rp = rec_params(prm);

    {
        ProfScope prof("control", s);
        k_ctl_begin<<<1, 64, 0, s>>>(k, *prm, st, fb->count, reinterpret_cast<long long*>(gn->part), gn->bar);
    }
    // the Gauss-Newton launches deskew and thin the frame themselves (from the state's twist, t_mid and count)
    GnThin th{};
    th.fb = *fb;
    th.a = thin_args(prm);
    th.on = 1;
    th.from_state = 1;
    th.begin = 0;
    int r;
    int nl = 6;  // the three control kernels and the keyframe insert's three passes
    if (net) {
        // first registration: deskew with the predicted motion and thin in kernels of their own, so that the
        // network sees the frame and the map patch around the constant-velocity prediction before the loop starts
        {
            ProfScope prof("thin", s);
            k_thin_a<<<grid, 256, 0, s>>>(*fb, &st->m, ta, st, tw, nullptr, &st->run_reg, 1, ThinBegin{});
            k_thin_b<<<nt, TILE, 0, s>>>(*fb, &st->m, &st->run_reg);
            k_thin_c<<<nt, TILE, 0, s>>>(*fb, &st->m, &st->n_ds, &st->run_reg);
        }
        nl += 3;
        ProfScope prof("net", s);
        r = net_sets_launch(fb->ds_xyz, &st->n_ds, *reg, st->T_pred, work->radius, work->voxel, work->sets,
                            work->cand, work->tiles, work->count, s);
        if (r != LW_OK) return r;
        r = net_forward_launch(*net, work->sets, 1, work->pooled, work->argmax, work->hid, work->step, work->err, s);
        if (r != LW_OK) return r;
        r = net_apply_launch(st, work->step, work->err, s);
        if (r != LW_OK) return r;
    }
    {
        // first registration (after deskewing with the predicted motion and thinning, unless done above)
        ProfScope prof("gn", s);
        r = launch_gn(fb->ds_xyz, &st->n_ds, prm, st, reg, gn, 0, s, /*cleared=*/true, net ? nullptr : &th);
    }
    if (r != LW_OK) return r;
    // re-deskew with the solved motion and register again when it moved enough
    {
        ProfScope prof("control", s);
        k_ctl_mid<<<1, 64, 0, s>>>(*prm, st, reinterpret_cast<long long*>(gn->part), gn->bar);
    }
    {
        ProfScope prof("gn", s);
        r = launch_gn(fb->ds_xyz, &st->n_ds, prm, st, reg, gn, 1, s, /*cleared=*/true, &th);
    }
    if (r != LW_OK) return r;
    // keyframe, velocity, pose table, trajectory
    {
        ProfScope prof("control", s);
        k_ctl_end<<<1, 1, 0, s>>>(*prm, st, *pt, epoch, traj, traj_cap, gn->err);
    }
    // keyframe insert with the frame's final pose (odom.py:719-727), through the state's float64 pose
    RegArgs a = reg_args(nullptr, prm->reg_voxel, prm->max_range, prm->ret_mask);
    const float4* p4 = reinterpret_cast<const float4*>(fb->f_xyz);
    {
        ProfScope prof("reg_insert", s);
        k_reg_a<<<grid, 256, 0, s>>>(p4, fb->f_attr, &st->m, m_ub, a, st->T, *reg, fb->ds_slot, &st->do_insert);
        k_reg_b<<<grid, 256, 0, s>>>(p4, &st->m, m_ub, a, st->T, *reg, fb->ds_slot, &st->do_insert);
        k_reg_d<<<grid, 256, 0, s>>>(&st->m, m_ub, *reg, fb->ds_slot, rp, &st->do_insert);
    }
    LW_LAUNCHED("lw_odom_finalize");
    count_launches(nl);  // plus the two Gauss-Newton launches counted by launch_gn
    return LW_OK;
}

int lw_odom_finalize(int32_t k, int64_t m_ub, const lw_odom_params* prm, lw_odom_state* st, lw_frame_buf* fb,
                     lw_regmap* reg, lw_gn_scratch* gn, lw_pose_table* pt, int32_t epoch, lw_traj_rec* traj,
                     int64_t traj_cap, void* stream) {
    return finalize_impl(k, m_ub, prm, st, fb, reg, gn, pt, epoch, traj, traj_cap, nullptr, nullptr, stream);
}

int lw_odom_finalize_net(int32_t k, int64_t m_ub, const lw_odom_params* prm, lw_odom_state* st, lw_frame_buf* fb,
                         lw_regmap* reg, lw_gn_scratch* gn, lw_pose_table* pt, int32_t epoch, lw_traj_rec* traj,
                         int64_t traj_cap, const lw_initnet* net, lw_net_work* work, void* stream) {
    if (!net || !net->w || !net->out_scale || !work || !work->sets || !work->pooled || !work->argmax || !work->hid ||
        !work->step || !work->err || !work->count || (!(work->voxel > 0.0f) && (!work->cand || !work->tiles)))
        return set_error(LW_EINVAL, "lw_odom_finalize_net: incomplete network or work buffers");
    if (((uintptr_t)net->w & 15) != 0 || ((uintptr_t)work->sets & 15) != 0)
        return set_error(LW_EINVAL, "lw_odom_finalize_net: weights and sets must be 16-byte aligned");
    return finalize_impl(k, m_ub, prm, st, fb, reg, gn, pt, epoch, traj, traj_cap, net, work, stream);
}

int lw_odom_predict_poses(int32_t k0, int32_t k1, int32_t current, const lw_odom_state* st, lw_pose_table* pt,
                          int32_t epoch, void* stream) {
    if (!st || !pt) return set_error(LW_EINVAL, "lw_odom_predict_poses: null argument");
    if (k1 <= k0) return LW_OK;
    int64_t n = (int64_t)k1 - k0;
    if (n > LW_POSE_SLOTS) n = LW_POSE_SLOTS;
    k_predict_poses<<<blocks_for(n, 256, 256), 256, 0, (cudaStream_t)stream>>>(k0, k1, current, st, *pt, epoch);
    LW_LAUNCHED("lw_odom_predict_poses");
    count_launches(1);
    return LW_OK;
}

int lw_odom_reset(const double* T0_host, lw_odom_state* st, lw_regmap* reg, int32_t clear_map, void* stream) {
    if (!T0_host || !st) return set_error(LW_EINVAL, "lw_odom_reset: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    lw_odom_state init;
    memset(&init, 0, sizeof(init));
    for (int i = 0; i < 16; ++i) {
        init.T[i] = T0_host[i];
        double e = (i % 5 == 0) ? 1.0 : 0.0;
        init.delta[i] = e;
        init.T_prev[i] = init.T_key[i] = init.T_pred[i] = init.T_reg[i] = e;
    }
    init.cond = 1.0;
    k_reset_state<<<1, 1, 0, s>>>(st, init);
    if (clear_map && reg) {
        int g = 8 * device_sms();
        k_fill_i64<<<g, 256, 0, s>>>(reg->keys, reg->cap, -1);
        LW_CUDA(cudaMemsetAsync(reg->cnt, 0, reg->cap * sizeof(int32_t), s));
        LW_CUDA(cudaMemsetAsync(reg->sum, 0, reg->cap * 3 * sizeof(int64_t), s));
        LW_CUDA(cudaMemsetAsync(reg->outer, 0, reg->cap * 6 * sizeof(int64_t), s));
        LW_CUDA(cudaMemsetAsync(reg->rec, 0, reg->cap * LW_REC_FLOATS * sizeof(float), s));
        LW_CUDA(cudaMemsetAsync(reg->bcnt, 0, reg->cap * sizeof(int32_t), s));
        k_fill_i32<<<g, 256, 0, s>>>(reg->first, reg->cap, NO_INDEX);
        LW_CUDA(cudaMemsetAsync(reg->stats, 0, 2 * sizeof(int32_t), s));
    }
    LW_LAUNCHED("lw_odom_reset");
    count_launches(clear_map && reg ? 3 : 1);
    return LW_OK;
}

int lw_odom_restart_clock(lw_odom_state* st, void* stream) {
    if (!st) return set_error(LW_EINVAL, "lw_odom_restart_clock: null argument");
    k_restart_clock<<<1, 1, 0, (cudaStream_t)stream>>>(st);
    LW_LAUNCHED("lw_odom_restart_clock");
    count_launches(1);
    return LW_OK;
}

}  // extern "C"

// =========================================================================================================
// Thinning for callers that cannot allocate device memory.
//
// A host that embeds this library inside a real-time sensor thread, or inside a process whose device memory is
// fixed at start-up (a driver callback, a plugin under a memory budget), must not call cudaMalloc on the frame
// path: an allocation can block behind other work on the device and its latency is unbounded. This variant of
// lw_thin takes only the caller's input points and output buffer; its working tables live in one file-scope
// device array that every GPU holds from the moment the library is loaded until the process exits.
// =========================================================================================================

namespace lw {

constexpr int64_t NOALLOC_THIN_MAX = 1 << 16;    // points one call may thin
constexpr int64_t NOALLOC_THIN_SLOTS = 1 << 17;  // hash slots (a power of two >= twice the points)
constexpr int64_t NOALLOC_THIN_TILES = NOALLOC_THIN_MAX / TILE + 2;
// layout (in int64 units): keys [SLOTS] | win [SLOTS/2] | slot [MAX/2] | tiles + m [(TILES + 2)/2]
constexpr int64_t NOALLOC_THIN_WORDS =
    NOALLOC_THIN_SLOTS + NOALLOC_THIN_SLOTS / 2 + NOALLOC_THIN_MAX / 2 + (NOALLOC_THIN_TILES + 2) / 2 + 1;

static __device__ __align__(256) int64_t g_thin_scratch[NOALLOC_THIN_WORDS];  // ~1.8 MB per device

__global__ void k_noalloc_thin_reset(int64_t* keys, int32_t* win, int32_t* m_dev, int32_t m) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < NOALLOC_THIN_SLOTS;
         i += (int64_t)gridDim.x * blockDim.x) {
        keys[i] = EMPTY_KEY;
        win[i] = NO_INDEX;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *m_dev = m;
}

// The array's device address, looked up once per device with that device current (host code may not use
// the symbol itself: on the host it names a stand-in, not device memory). The address is kept for the life of
// the process: after cudaDeviceReset the module loads again and the array may move, so a process that resets a
// device must not call lw_thin_noalloc on it again.
static int noalloc_thin_scratch(int64_t** out) {
    static std::mutex mu;
    static int64_t* addr[256] = {};
    int dev = 0;
    LW_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 256) return set_error(LW_EINVAL, "lw_thin_noalloc: device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> g(mu);
    if (!addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_thin_scratch);
        if (e != cudaSuccess) return check_cuda(e, "lw_thin_noalloc: cudaGetSymbolAddress");
        addr[dev] = (int64_t*)p;
    }
    *out = addr[dev];
    return LW_OK;
}

}  // namespace lw

extern "C" int lw_thin_noalloc(const float* xyz4, const uint32_t* attr, int64_t m, double inv_v, double min_range,
                               double max_range, int32_t ret_mask, float* ds4_out, int32_t* n_ds_dev, void* stream) {
    using namespace lw;
    if (!xyz4 || !attr || !ds4_out || !n_ds_dev) return set_error(LW_EINVAL, "lw_thin_noalloc: null argument");
    // the points are read and written as float4: a misaligned pointer is refused here, not faulted on
    if (((uintptr_t)xyz4 & 15) != 0 || ((uintptr_t)ds4_out & 15) != 0)
        return set_error(LW_EINVAL, "lw_thin_noalloc: xyz4 and ds4_out must be 16-byte aligned");
    if (m < 0 || m > NOALLOC_THIN_MAX)
        return set_error(LW_ECAPACITY, "lw_thin_noalloc: %lld points exceed the fixed maximum of %lld per call",
                         (long long)m, (long long)NOALLOC_THIN_MAX);
    int64_t* base = nullptr;
    int r = noalloc_thin_scratch(&base);
    if (r != LW_OK) return r;
    cudaStream_t s = (cudaStream_t)stream;
    int64_t* keys = base;
    int32_t* win = reinterpret_cast<int32_t*>(base + NOALLOC_THIN_SLOTS);
    int32_t* slot = reinterpret_cast<int32_t*>(base + NOALLOC_THIN_SLOTS + NOALLOC_THIN_SLOTS / 2);
    int32_t* tiles = reinterpret_cast<int32_t*>(base + NOALLOC_THIN_SLOTS + NOALLOC_THIN_SLOTS / 2 + NOALLOC_THIN_MAX / 2);
    int32_t* m_dev = tiles + NOALLOC_THIN_TILES;
    // the array keeps whatever the last call left: start every call from a cleared table
    k_noalloc_thin_reset<<<64, 256, 0, s>>>(keys, win, m_dev, (int32_t)m);
    lw_frame_buf fb{};
    fb.f_xyz = const_cast<float*>(xyz4);
    fb.f_attr = const_cast<uint32_t*>(attr);
    fb.ds_keys = keys;
    fb.ds_win = win;
    fb.ds_slot = slot;
    fb.tiles = tiles;
    fb.ds_xyz = ds4_out;
    fb.cap = m > 0 ? m : 1;
    fb.ds_cap = NOALLOC_THIN_SLOTS;
    ThinArgs a{};
    a.inv_v = (float)inv_v;
    a.min_range = (float)min_range;
    a.max_range = (float)max_range;
    a.ret_mask = ret_mask;
    a.deskew = 0;
    Tw6 tw{};
    int64_t mu = m > 0 ? m : 1;
    int grid = blocks_for(mu, 256, 8 * device_sms());
    int nt = blocks_for(mu, TILE);
    k_thin_a<<<grid, 256, 0, s>>>(fb, m_dev, a, nullptr, tw, nullptr, nullptr, 1, ThinBegin{});
    k_thin_b<<<nt, TILE, 0, s>>>(fb, m_dev, nullptr);
    k_thin_c<<<nt, TILE, 0, s>>>(fb, m_dev, n_ds_dev, nullptr);
    LW_LAUNCHED("lw_thin_noalloc");
    count_launches(4);
    return LW_OK;
}
