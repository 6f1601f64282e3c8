// Prior maps on sm_100a: a point cloud voxel-downsampled to per-voxel means (with the mean colour, intensity and
// point count), then a PCA normal and a planarity for every mean from its neighbours within a radius -- the arrays a
// prior map for global localisation holds.
//
// Reference: python/livox_warp/prior_map.py -- k_vox_insert :57-91, k_vox_flag :94-97, k_vox_emit :100-123,
// k_normals :126-166, voxel_downsample :169-203, normals :206-219, from_points :358-370.
//
// Determinism. The reference adds float32 offsets, colours and intensities into its voxels with float atomics,
// emits the voxels in hash-slot order (for colliding keys that depends on which thread claimed first) and sums a
// point's neighbours in float32 in hash-grid query order. Here every sum is int64 fixed point, the voxels are
// numbered in the order of their first point (the lowest point index that reached each voxel, whichever chunk it
// came in), and the neighbour sums are fixed point too, with the covariance and its eigen-decomposition in float64.
// Every output is then independent of thread timing and of where keys land in the tables.
//
// Layout. Voxel table: keys [cap] int64, acc [cap][8] int64 (offsets x y z, r g b, intensity, count: one 64-byte
// line per voxel), first [cap] int64, order [cap] int32. Normals: the points are counting-sorted by cell into
// `sorted` (16-byte records x, y, z, index) so that a warp's threads, which take consecutive sorted positions,
// walk the same 27 cells and read each cell's records as one contiguous, mostly L1-resident run.
#include "lw_common.cuh"
#include "lw_linalg.cuh"

namespace lw {

constexpr int VX_PROBES = 128;  // open-addressing probes before a point counts as dropped (prior_map.py:36)
constexpr int VX_TILE = 1024;
constexpr float VX_FIX_ATTR = (float)LW_VOX_FIX_ATTR;
constexpr double PC_CELL_PAD = 1.00390625;  // cells 2^-8 wider than the radius: every neighbour lies in the 27

struct VoxArgs {
    float inv_v, voxel, fix_ofs;
    int mask;
    int64_t index0;
};

struct PcaArgs {
    float inv_h, r2, fd, fdd;
    double fd64, fdd64;
    int mask;
};

template <int STRIDE>
__device__ __forceinline__ void ld3(const float* __restrict__ xyz, int64_t i, float& x, float& y, float& z) {
    x = xyz[STRIDE * i];
    y = xyz[STRIDE * i + 1];
    z = xyz[STRIDE * i + 2];
}

// voxel_centre (prior_map.py:53-54): ((i + 0.5) * voxel) in float32
__device__ __forceinline__ float vcentre(int i, float voxel) { return ((float)i + 0.5f) * voxel; }

__device__ __forceinline__ void key_unpack(int64_t key, int& ix, int& iy, int& iz) {  // prior_map.py:41-50
    ix = (int)(key & KEY_MASK) - (int)KEY_BIAS;
    iy = (int)((key >> 21) & KEY_MASK) - (int)KEY_BIAS;
    iz = (int)((key >> 42) & KEY_MASK) - (int)KEY_BIAS;
}

// ---- voxel downsample -------------------------------------------------------------------------------------------

// Each point claims its voxel and adds its offset from the voxel centre, colour, intensity and 1 (k_vox_insert).
template <int STRIDE>
__global__ void k_vox_insert(const float* __restrict__ xyz, const float* __restrict__ inten,
                             const float* __restrict__ rgb, int64_t n, VoxArgs a, lw_vox_buf vb) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float x, y, z;
        ld3<STRIDE>(xyz, i, x, y, z);
        const int ix = ifloor(x * a.inv_v), iy = ifloor(y * a.inv_v), iz = ifloor(z * a.inv_v);
        bool claimed;
        const int s = claim_slot<VX_PROBES>(key_ijk(ix, iy, iz), vb.keys, a.mask, &claimed);
        vb.slot_of_pt[i] = s;
        if (s < 0) {
            atomicAdd((unsigned long long*)(vb.stats + 1), 1ull);
            continue;
        }
        int64_t* acc = vb.acc + 8 * (int64_t)s;
        atomic_add_i64(acc + 0, to_fix(x - vcentre(ix, a.voxel), a.fix_ofs));
        atomic_add_i64(acc + 1, to_fix(y - vcentre(iy, a.voxel), a.fix_ofs));
        atomic_add_i64(acc + 2, to_fix(z - vcentre(iz, a.voxel), a.fix_ofs));
        if (rgb) {
            atomic_add_i64(acc + 3, to_fix(rgb[3 * i], VX_FIX_ATTR));
            atomic_add_i64(acc + 4, to_fix(rgb[3 * i + 1], VX_FIX_ATTR));
            atomic_add_i64(acc + 5, to_fix(rgb[3 * i + 2], VX_FIX_ATTR));
        }
        if (inten) atomic_add_i64(acc + 6, to_fix(inten[i], VX_FIX_ATTR));
        atomic_add_i64(acc + 7, 1);
        atomicMin((unsigned long long*)(vb.first + s), (unsigned long long)(a.index0 + i));
    }
}

// A point opens a voxel when it is the voxel's first point; per tile of the chunk, how many do.
__device__ __forceinline__ int vox_opens(const lw_vox_buf& vb, int64_t i, int64_t n, int64_t index0) {
    if (i >= n) return 0;
    const int s = vb.slot_of_pt[i];
    return s >= 0 && vb.first[s] == index0 + i;
}

__global__ void k_vox_count(int64_t n, int64_t index0, lw_vox_buf vb) {
    const int64_t i = (int64_t)blockIdx.x * VX_TILE + threadIdx.x;
    const int c = __syncthreads_count(vox_opens(vb, i, n, index0));
    if (threadIdx.x == 0) vb.tiles[blockIdx.x] = c;
}

// One CTA: exclusive scan of nt tile counts in place, offset by *counter, which then grows by the total.
template <class T>
__global__ void k_scan_from(int* tiles, int nt, T* counter) {
    __shared__ int sm[33];
    __shared__ long long carry;
    if (threadIdx.x == 0) carry = (long long)*counter;
    __syncthreads();
    for (int base = 0; base < nt; base += blockDim.x) {
        const int j = base + threadIdx.x;
        const int v = j < nt ? tiles[j] : 0;
        int tot;
        const int r = block_excl(v, sm, &tot);
        if (j < nt) tiles[j] = (int)(carry + r);
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) *counter = (T)carry;
}

// The opening points, in index order, append their voxels to `order`.
__global__ void k_vox_scatter(int64_t n, int64_t index0, lw_vox_buf vb) {
    __shared__ int sm[33];
    const int64_t i = (int64_t)blockIdx.x * VX_TILE + threadIdx.x;
    const int f = vox_opens(vb, i, n, index0);
    int tot;
    const int r = block_rank(f, sm, &tot);
    // positions stay below cap when index0 counts the earlier chunks (each voxel opens once); the check keeps a
    // misnumbered call from writing past the array
    const int64_t pos = (int64_t)vb.tiles[blockIdx.x] + r;
    if (f && pos < vb.cap) vb.order[pos] = vb.slot_of_pt[i];
}

// Dense per-voxel means (k_vox_emit): centre + the exact mean offset, rounded once to float32.
__global__ void k_vox_emit(int64_t m_cap, VoxArgs a, lw_vox_buf vb, float* __restrict__ out_xyz,
                           float* __restrict__ out_rgb, float* __restrict__ out_inten, int32_t* __restrict__ out_cnt) {
    const int64_t m = min((int64_t)*vb.stats, m_cap);
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < m; j += (int64_t)gridDim.x * blockDim.x) {
        const int s = vb.order[j];
        int ix, iy, iz;
        key_unpack(vb.keys[s], ix, iy, iz);
        const int64_t* acc = vb.acc + 8 * (int64_t)s;
        const double c = (double)acc[7];
        const double uo = c * (double)a.fix_ofs, ua = c * LW_VOX_FIX_ATTR;
        if (out_xyz) {
            out_xyz[3 * j + 0] = (float)((double)vcentre(ix, a.voxel) + (double)acc[0] / uo);
            out_xyz[3 * j + 1] = (float)((double)vcentre(iy, a.voxel) + (double)acc[1] / uo);
            out_xyz[3 * j + 2] = (float)((double)vcentre(iz, a.voxel) + (double)acc[2] / uo);
        }
        if (out_rgb) {
            out_rgb[3 * j + 0] = (float)((double)acc[3] / ua);
            out_rgb[3 * j + 1] = (float)((double)acc[4] / ua);
            out_rgb[3 * j + 2] = (float)((double)acc[5] / ua);
        }
        if (out_inten) out_inten[j] = (float)((double)acc[6] / ua);
        if (out_cnt) out_cnt[j] = (int32_t)min(acc[7], (int64_t)0x7FFFFFFF);
    }
}

// ---- normals --------------------------------------------------------------------------------------------------

template <int STRIDE>
__global__ void k_pc_insert(const float* __restrict__ xyz, int64_t n, PcaArgs a, lw_pca_buf pb) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float x, y, z;
        ld3<STRIDE>(xyz, i, x, y, z);
        bool claimed;
        const int s = claim_slot<VX_PROBES>(key_ijk(ifloor(x * a.inv_h), ifloor(y * a.inv_h), ifloor(z * a.inv_h)),
                                            pb.keys, a.mask, &claimed);
        pb.slot_of_pt[i] = s;
        if (s < 0) {
            atomicAdd(pb.stats + 1, 1);
            continue;
        }
        pb.rank_of_pt[i] = atomicAdd(pb.cell_cnt + s, 1);
    }
}

// Points per tile of 1024 slots, then (k_scan_from) each tile's first position, then each cell's.
__global__ void k_pc_tiles(lw_pca_buf pb) {
    __shared__ int sm[33];
    const int64_t s = (int64_t)blockIdx.x * VX_TILE + threadIdx.x;
    int tot;
    block_excl(s < pb.cap ? pb.cell_cnt[s] : 0, sm, &tot);
    if (threadIdx.x == 0) pb.tiles[blockIdx.x] = tot;
}

__global__ void k_pc_start(lw_pca_buf pb) {
    __shared__ int sm[33];
    const int64_t s = (int64_t)blockIdx.x * VX_TILE + threadIdx.x;
    const int v = s < pb.cap ? pb.cell_cnt[s] : 0;
    int tot;
    const int r = block_excl(v, sm, &tot);
    if (v > 0) pb.cell_start[s] = pb.tiles[blockIdx.x] + r;
}

template <int STRIDE>
__global__ void k_pc_scatter(const float* __restrict__ xyz, int64_t n, lw_pca_buf pb, float* __restrict__ out_nrm,
                             float* __restrict__ out_pl) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int s = pb.slot_of_pt[i];
        if (s < 0) {  // not placed: no neighbourhood to fit
            out_nrm[3 * i] = out_nrm[3 * i + 1] = out_nrm[3 * i + 2] = 0.0f;
            out_pl[i] = 0.0f;
            continue;
        }
        float x, y, z;
        ld3<STRIDE>(xyz, i, x, y, z);
        const int64_t q = (int64_t)pb.cell_start[s] + pb.rank_of_pt[i];
        reinterpret_cast<float4*>(pb.sorted)[q] = make_float4(x, y, z, __int_as_float((int)i));
    }
}

// A thread per sorted position (k_normals): every point within the radius, found in the 27 cells around the
// point's own, adds 1, its offset and its offset's outer product in fixed point; then the covariance's
// eigen-decomposition in float64, the smallest eigenvalue's vector and (l_mid - l_min) / l_max.
__global__ void __launch_bounds__(256) k_pc_normals(PcaArgs a, lw_pca_buf pb, float* __restrict__ out_nrm,
                                                    float* __restrict__ out_pl) {
    const int m = *pb.stats;
    const float4* __restrict__ pts = reinterpret_cast<const float4*>(pb.sorted);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += gridDim.x * blockDim.x) {
        const float4 P = pts[q];
        const int i = __float_as_int(P.w);
        const int ix = ifloor(P.x * a.inv_h), iy = ifloor(P.y * a.inv_h), iz = ifloor(P.z * a.inv_h);
        int n = 0;
        long long s1[3] = {0, 0, 0}, s2[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll 1
        for (int c = 0; c < 27; ++c) {
            const int s = find_slot<VX_PROBES>(key_ijk(ix + c / 9 - 1, iy + (c / 3) % 3 - 1, iz + c % 3 - 1),
                                               pb.keys, a.mask);
            if (s < 0) continue;
            const int k0 = __ldg(pb.cell_start + s), k1 = k0 + __ldg(pb.cell_cnt + s);
#pragma unroll 1
            for (int k = k0; k < k1; ++k) {
                const float4 Q = __ldg(pts + k);
                const float ex = Q.x - P.x, ey = Q.y - P.y, ez = Q.z - P.z;
                if (ex * ex + ey * ey + ez * ez > a.r2) continue;
                ++n;
                s1[0] += to_fix(ex, a.fd);
                s1[1] += to_fix(ey, a.fd);
                s1[2] += to_fix(ez, a.fd);
                s2[0] += to_fix(ex * ex, a.fdd);
                s2[1] += to_fix(ex * ey, a.fdd);
                s2[2] += to_fix(ex * ez, a.fdd);
                s2[3] += to_fix(ey * ey, a.fdd);
                s2[4] += to_fix(ey * ez, a.fdd);
                s2[5] += to_fix(ez * ez, a.fdd);
            }
        }
        if (n < 4) {  // prior_map.py:151-154
            out_nrm[3 * (int64_t)i] = out_nrm[3 * (int64_t)i + 1] = out_nrm[3 * (int64_t)i + 2] = 0.0f;
            out_pl[i] = 0.0f;
            continue;
        }
        const double inv = 1.0 / (double)n;
        const double mu[3] = {(double)s1[0] / a.fd64 * inv, (double)s1[1] / a.fd64 * inv,
                              (double)s1[2] / a.fd64 * inv};
        const int up[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
        double C[9], ev[3], Qm[9];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) C[r * 3 + c] = (double)s2[up[r * 3 + c]] / a.fdd64 * inv - mu[r] * mu[c];
        jacobi_eig<3>(C, ev, Qm);
        // the eigenvalues' order, as prior_map.py:157-164 picks it
        int lo = 0, hi = 0;
        if (ev[1] < ev[lo]) lo = 1;
        if (ev[1] > ev[hi]) hi = 1;
        if (ev[2] < ev[lo]) lo = 2;
        if (ev[2] > ev[hi]) hi = 2;
        const int mid = lo == hi ? lo : 3 - lo - hi;
        // selects instead of indexing with lo / mid / hi keep ev and Qm in registers
        auto at = [](const double* v, int k) { return k == 0 ? v[0] : (k == 1 ? v[1] : v[2]); };
        double nx = at(Qm, lo), ny = at(Qm + 3, lo), nz = at(Qm + 6, lo);
        const double nl = sqrt(nx * nx + ny * ny + nz * nz);
        if (nl > 0.0) {
            nx /= nl;
            ny /= nl;
            nz /= nl;
        }
        out_nrm[3 * (int64_t)i + 0] = (float)nx;
        out_nrm[3 * (int64_t)i + 1] = (float)ny;
        out_nrm[3 * (int64_t)i + 2] = (float)nz;
        out_pl[i] = (float)((at(ev, mid) - at(ev, lo)) / fmax(at(ev, hi), 1.0e-12));
    }
}

}  // namespace lw

using namespace lw;

namespace {

bool pow2_cap(int64_t cap) { return cap > 0 && cap <= (1LL << 30) && (cap & (cap - 1)) == 0; }

}  // namespace

extern "C" {

double lw_vox_offset_units(float voxel) {
    int e = 0;
    frexpf(voxel, &e);  // voxel = f 2^e, f in [0.5, 1): voxel < 2^e
    return ldexp(1.0, 30 - e);
}

int lw_vox_clear(lw_vox_buf* vb, void* stream) {
    if (!vb || !vb->keys || !vb->acc || !vb->first || !vb->stats || !pow2_cap(vb->cap))
        return set_error(LW_EINVAL, "lw_vox_clear: incomplete buffers or capacity not a power of two");
    cudaStream_t s = (cudaStream_t)stream;
    LW_CUDA(cudaMemsetAsync(vb->keys, 0xFF, sizeof(int64_t) * vb->cap, s));
    LW_CUDA(cudaMemsetAsync(vb->acc, 0, sizeof(int64_t) * 8 * vb->cap, s));
    LW_CUDA(cudaMemsetAsync(vb->first, 0x7F, sizeof(int64_t) * vb->cap, s));
    LW_CUDA(cudaMemsetAsync(vb->stats, 0, sizeof(int64_t) * 2, s));
    return LW_OK;
}

int lw_vox_insert(lw_vox_buf* vb, const float* xyz, int32_t xyz_stride, const float* intensity, const float* rgb,
                  int64_t n, int64_t index0, float voxel, void* stream) {
    if (!vb || !vb->keys || !vb->acc || !vb->first || !vb->order || !vb->slot_of_pt || !vb->tiles || !vb->stats ||
        !pow2_cap(vb->cap))
        return set_error(LW_EINVAL, "lw_vox_insert: incomplete buffers or capacity not a power of two");
    if (!(voxel >= 1.0e-6f && voxel <= 1.0e6f) || (xyz_stride != 3 && xyz_stride != 4) || n < 0 || index0 < 0 ||
        (n > 0 && !xyz))
        return set_error(LW_EINVAL, "lw_vox_insert: bad arguments (voxel must lie in [1e-6, 1e6] m)");
    if (n > vb->pt_cap || vb->pt_cap > (1LL << 30))
        return set_error(LW_ECAPACITY, "lw_vox_insert: %lld points exceed the chunk buffers' %lld", (long long)n,
                         (long long)vb->pt_cap);
    if (n == 0) return LW_OK;
    cudaStream_t s = (cudaStream_t)stream;
    ProfScope prof("lw_vox_insert", s);
    VoxArgs a{};
    a.inv_v = (float)(1.0 / (double)voxel);  // prior_map.py:195, 1.0 / voxel as a float32 kernel argument
    a.voxel = voxel;
    a.fix_ofs = (float)lw_vox_offset_units(voxel);
    a.mask = (int)(vb->cap - 1);
    a.index0 = index0;
    const int sms = device_sms();
    const int grid = blocks_for(n, 256, 16 * sms);
    if (xyz_stride == 4)
        k_vox_insert<4><<<grid, 256, 0, s>>>(xyz, intensity, rgb, n, a, *vb);
    else
        k_vox_insert<3><<<grid, 256, 0, s>>>(xyz, intensity, rgb, n, a, *vb);
    const int nt = blocks_for(n, VX_TILE);
    k_vox_count<<<nt, VX_TILE, 0, s>>>(n, index0, *vb);
    k_scan_from<int64_t><<<1, 1024, 0, s>>>(vb->tiles, nt, vb->stats);
    k_vox_scatter<<<nt, VX_TILE, 0, s>>>(n, index0, *vb);
    LW_LAUNCHED("lw_vox_insert");
    count_launches(4);
    return LW_OK;
}

int lw_vox_emit(const lw_vox_buf* vb, float voxel, int64_t m_cap, float* out_xyz, float* out_rgb,
                float* out_intensity, int32_t* out_cnt, void* stream) {
    if (!vb || !vb->keys || !vb->acc || !vb->order || !vb->stats || !pow2_cap(vb->cap))
        return set_error(LW_EINVAL, "lw_vox_emit: incomplete buffers or capacity not a power of two");
    if (!(voxel >= 1.0e-6f && voxel <= 1.0e6f) || m_cap < 0)
        return set_error(LW_EINVAL, "lw_vox_emit: bad arguments (voxel must lie in [1e-6, 1e6] m)");
    if (m_cap == 0) return LW_OK;
    cudaStream_t s = (cudaStream_t)stream;
    ProfScope prof("lw_vox_emit", s);
    VoxArgs a{};
    a.voxel = voxel;
    a.fix_ofs = (float)lw_vox_offset_units(voxel);
    const int64_t m_ub = m_cap < vb->cap ? m_cap : vb->cap;
    k_vox_emit<<<blocks_for(m_ub, 256, 16 * device_sms()), 256, 0, s>>>(m_ub, a, *vb, out_xyz, out_rgb, out_intensity,
                                                                       out_cnt);
    LW_LAUNCHED("lw_vox_emit");
    count_launches(1);
    return LW_OK;
}

int lw_normals(const float* xyz, int32_t xyz_stride, int64_t n, float radius, lw_pca_buf* pb, float* out_nrm,
               float* out_planarity, void* stream) {
    if (!pb || !pb->keys || !pb->cell_cnt || !pb->cell_start || !pb->slot_of_pt || !pb->rank_of_pt || !pb->sorted ||
        !pb->tiles || !pb->stats || !pow2_cap(pb->cap))
        return set_error(LW_EINVAL, "lw_normals: incomplete buffers or capacity not a power of two");
    if (!(radius >= 1.0e-4f && radius <= 16.0f))
        return set_error(LW_EINVAL, "lw_normals: radius %g outside [1e-4, 16] m", (double)radius);
    if ((xyz_stride != 3 && xyz_stride != 4) || n < 0 || (n > 0 && (!xyz || !out_nrm || !out_planarity)))
        return set_error(LW_EINVAL, "lw_normals: bad arguments");
    if (n > pb->pt_cap || pb->pt_cap > (1LL << 30) || 2 * n > pb->cap)
        return set_error(LW_ECAPACITY, "lw_normals: %lld points need pt_cap >= n and cap >= 2n (%lld, %lld)",
                         (long long)n, (long long)pb->pt_cap, (long long)pb->cap);
    cudaStream_t s = (cudaStream_t)stream;
    LW_CUDA(cudaMemsetAsync(pb->stats, 0, sizeof(int32_t) * 2, s));
    if (n == 0) return LW_OK;
    ProfScope prof("lw_normals", s);
    PcaArgs a{};
    a.inv_h = (float)(1.0 / ((double)radius * PC_CELL_PAD));
    a.r2 = radius * radius;
    int e = 0;
    frexpf(radius, &e);  // radius < 2^e: an offset is below 2^20 units, a product below 2^40
    a.fd64 = ldexp(1.0, 20 - e);
    a.fdd64 = ldexp(1.0, 40 - 2 * e);
    a.fd = (float)a.fd64;
    a.fdd = (float)a.fdd64;
    a.mask = (int)(pb->cap - 1);
    LW_CUDA(cudaMemsetAsync(pb->keys, 0xFF, sizeof(int64_t) * pb->cap, s));
    LW_CUDA(cudaMemsetAsync(pb->cell_cnt, 0, sizeof(int32_t) * pb->cap, s));
    const int sms = device_sms();
    const int grid = blocks_for(n, 256, 16 * sms);
    const int nt = blocks_for(pb->cap, VX_TILE);
    if (xyz_stride == 4)
        k_pc_insert<4><<<grid, 256, 0, s>>>(xyz, n, a, *pb);
    else
        k_pc_insert<3><<<grid, 256, 0, s>>>(xyz, n, a, *pb);
    k_pc_tiles<<<nt, VX_TILE, 0, s>>>(*pb);
    k_scan_from<int32_t><<<1, 1024, 0, s>>>(pb->tiles, nt, pb->stats);
    k_pc_start<<<nt, VX_TILE, 0, s>>>(*pb);
    if (xyz_stride == 4)
        k_pc_scatter<4><<<grid, 256, 0, s>>>(xyz, n, *pb, out_nrm, out_planarity);
    else
        k_pc_scatter<3><<<grid, 256, 0, s>>>(xyz, n, *pb, out_nrm, out_planarity);
    k_pc_normals<<<blocks_for(n, 256, 16 * sms), 256, 0, s>>>(a, *pb, out_nrm, out_planarity);
    LW_LAUNCHED("lw_normals");
    count_launches(6);
    return LW_OK;
}

}  // extern "C"
