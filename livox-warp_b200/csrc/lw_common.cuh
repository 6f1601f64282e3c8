// Device helpers shared by every kernel of the library: voxel keys and the open-addressed hash, float and
// fixed-point atomics, block reductions, a bounded grid barrier and the status plumbing.
//
// The library is compiled with -fmad=false: every float expression below rounds exactly as written, so the
// CPU oracle (compiled with -ffp-contract=off) evaluates the same expressions to the same bits. Where a
// kernel wants fused multiply-adds for speed it asks for them explicitly (fmaf / __fmaf_rn).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include "../../include/livox_b200.h"

namespace lw {

// ---- status -----------------------------------------------------------------------------------------
int set_error(int code, const char* fmt, ...);
int check_cuda(cudaError_t e, const char* what);
#define LW_CUDA(call)                                                   \
    do {                                                                \
        cudaError_t _e = (call);                                        \
        if (_e != cudaSuccess) return ::lw::check_cuda(_e, #call);      \
    } while (0)
#define LW_LAUNCHED(name)                                               \
    do {                                                                \
        cudaError_t _e = cudaGetLastError();                            \
        if (_e != cudaSuccess) return ::lw::check_cuda(_e, name);       \
    } while (0)

int device_sms();

// Kernel launches issued by the entry points since the last lw_launches_reset (a benchmark's claim of how many
// of this library's kernels ran).
void count_launches(int n);

// Brackets the launches issued in its lifetime with CUDA events on `s` when timing is enabled (lw_prof_enable).
class ProfScope {
  public:
    ProfScope(const char* name, cudaStream_t s);
    ~ProfScope();
    ProfScope(const ProfScope&) = delete;
    ProfScope& operator=(const ProfScope&) = delete;

  private:
    const char* name_;
    cudaStream_t s_;
    void* a_;
};

// ---- voxel keys (gpu.py:59-64, 231-265) ----------------------------------------------------------------
constexpr int64_t KEY_BIAS = 1LL << 20;
constexpr int64_t KEY_MASK = (1LL << 21) - 1;
constexpr uint64_t HASH_MULT = 0x9E3779B97F4A7C15ULL;
constexpr int PROBES = 64;
constexpr int64_t EMPTY_KEY = -1;
constexpr int32_t NO_INDEX = 0x7FFFFFFF;

__host__ __device__ __forceinline__ int64_t key_ijk(int ix, int iy, int iz) {
    int64_t x = ((int64_t)ix + KEY_BIAS) & KEY_MASK;
    int64_t y = ((int64_t)iy + KEY_BIAS) & KEY_MASK;
    int64_t z = ((int64_t)iz + KEY_BIAS) & KEY_MASK;
    return x | (y << 21) | (z << 42);
}

// floor(v) as an int, for the voxel index of a coordinate already multiplied by 1/voxel.
__device__ __forceinline__ int ifloor(float v) { return (int)floorf(v); }

__host__ __device__ __forceinline__ int slot_hash(int64_t k) {
    int64_t h = (int64_t)((uint64_t)k * HASH_MULT);  // wrapping 64-bit multiply
    h = h ^ (h >> 29);                                // arithmetic shift of the signed value
    return (int)(h & 0x7FFFFFFFLL);
}

// Slot holding `key`, or -1 (gpu.py:254-265). P probes (the prior-map table takes 128, prior_map.py:36).
template <int P = PROBES>
__device__ __forceinline__ int find_slot(int64_t key, const int64_t* __restrict__ keys, int mask) {
    int h = slot_hash(key) & mask;
#pragma unroll 1
    for (int p = 0; p < P; ++p) {
        int s = (h + p) & mask;
        int64_t k = __ldg(keys + s);
        if (k == key) return s;
        if (k == EMPTY_KEY) return -1;
    }
    return -1;
}

// Find the slot of `key` or claim an empty one. Returns the slot and sets *claimed when this call turned an
// empty slot into `key`; -1 when the probe window of P slots is full (gpu.py:396-412).
template <int P = PROBES>
__device__ __forceinline__ int claim_slot(int64_t key, int64_t* keys, int mask, bool* claimed) {
    int h = slot_hash(key) & mask;
    *claimed = false;
#pragma unroll 1
    for (int p = 0; p < P; ++p) {
        int s = (h + p) & mask;
        int64_t k = *(volatile int64_t*)(keys + s);
        if (k == key) return s;
        if (k == EMPTY_KEY) {
            unsigned long long prev = atomicCAS((unsigned long long*)(keys + s), (unsigned long long)EMPTY_KEY,
                                                (unsigned long long)key);
            if ((int64_t)prev == EMPTY_KEY) {
                *claimed = true;
                return s;
            }
            if ((int64_t)prev == key) return s;
        }
    }
    return -1;
}

// ---- attribute fields (gpu.py:124-141) -----------------------------------------------------------------
__host__ __device__ __forceinline__ int refl_of(uint32_t a) { return (int)(a & 255u); }
__host__ __device__ __forceinline__ int tag_of(uint32_t a) { return (int)((a >> 8) & 255u); }
__host__ __device__ __forceinline__ int ret_of(uint32_t a) { return (int)((a >> 16) & 255u); }

// ---- float helpers ---------------------------------------------------------------------------------------
// |p| evaluated as sqrt((x*x + y*y) + z*z), the order every kernel and the oracle use.
__device__ __forceinline__ float len3(float x, float y, float z) { return sqrtf(x * x + y * y + z * z); }

// Row-major float 4x4 applied to a point: ((m0 x + m1 y) + m2 z) + m3 per row.
__device__ __forceinline__ void xform(const float* __restrict__ T, float x, float y, float z, float& ox,
                                      float& oy, float& oz) {
    ox = T[0] * x + T[1] * y + T[2] * z + T[3];
    oy = T[4] * x + T[5] * y + T[6] * z + T[7];
    oz = T[8] * x + T[9] * y + T[10] * z + T[11];
}

// deskew (gpu.py:268-283): a point measured a fraction s of a frame after mid-frame, moved to the mid-frame sensor
// frame by the frame's body motion tw = (rho, theta): rotation by the rotation vector theta * s, then + rho * s.
// The rotation is evaluated in float64 and rounded once, so the CPU oracle reproduces it exactly.
__device__ __forceinline__ void deskew_frac(float x, float y, float z, float s, const float* tw, float& ox, float& oy,
                                            float& oz) {
    float rx = tw[3] * s, ry = tw[4] * s, rz = tw[5] * s;
    float a = len3(rx, ry, rz);
    ox = x;
    oy = y;
    oz = z;
    if (!(a < 1.0e-9f)) {
        double ad = (double)a;
        double ux = (double)rx / ad, uy = (double)ry / ad, uz = (double)rz / ad;
        double sh = sin(0.5 * ad), w = cos(0.5 * ad);
        double vx = ux * sh, vy = uy * sh, vz = uz * sh;
        double px = x, py = y, pz = z;
        // p' = p + w t + v x t with t = 2 (v x p)
        double tx = 2.0 * (vy * pz - vz * py), ty = 2.0 * (vz * px - vx * pz), tz = 2.0 * (vx * py - vy * px);
        ox = (float)(px + w * tx + (vy * tz - vz * ty));
        oy = (float)(py + w * ty + (vz * tx - vx * tz));
        oz = (float)(pz + w * tz + (vx * ty - vy * tx));
    }
    ox = ox + tw[0] * s;
    oy = oy + tw[1] * s;
    oz = oz + tw[2] * s;
}

__device__ __forceinline__ float atomic_min_float(float* a, float v) {
    return v >= 0.0f ? __int_as_float(atomicMin((int*)a, __float_as_int(v)))
                     : __uint_as_float(atomicMax((unsigned int*)a, __float_as_uint(v)));
}
__device__ __forceinline__ float atomic_max_float(float* a, float v) {
    return v >= 0.0f ? __int_as_float(atomicMax((int*)a, __float_as_int(v)))
                     : __uint_as_float(atomicMin((unsigned int*)a, __float_as_uint(v)));
}
__device__ __forceinline__ void atomic_add_i64(int64_t* a, int64_t v) {
    atomicAdd((unsigned long long*)a, (unsigned long long)v);
}
// float -> int64 fixed point, round to nearest even (llrintf on the host).
__device__ __forceinline__ int64_t to_fix(float v, float scale) { return __float2ll_rn(v * scale); }

// ---- reductions --------------------------------------------------------------------------------------------
// claim_slot with the compare-and-swap as the probe: one atomic round trip per probed slot, where a load first
// costs two for a slot found empty. The same slot results (a key is in at most one slot of its probe sequence:
// a probe stops at the first slot that holds the key or that it turns from empty into the key).
template <int P = PROBES>
__device__ __forceinline__ int claim_slot_cas(int64_t key, int64_t* keys, int mask) {
    int h = slot_hash(key) & mask;
#pragma unroll 1
    for (int p = 0; p < P; ++p) {
        int s = (h + p) & mask;
        unsigned long long prev = atomicCAS((unsigned long long*)(keys + s), (unsigned long long)EMPTY_KEY,
                                            (unsigned long long)key);
        if ((int64_t)prev == EMPTY_KEY || (int64_t)prev == key) return s;
    }
    return -1;
}

__device__ __forceinline__ int warp_sum_i(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Exclusive block scan of 0/1 flags for blockDim.x <= 1024; returns this thread's rank, total in *tot.
__device__ __forceinline__ int block_rank(int flag, int* smem32, int* tot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    unsigned bal = __ballot_sync(0xffffffffu, flag);
    int before = __popc(bal & ((1u << lane) - 1u));
    if (lane == 0) smem32[warp] = __popc(bal);
    __syncthreads();
    if (warp == 0) {
        int v = lane < nw ? smem32[lane] : 0;
        int inc = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int u = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += u;
        }
        if (lane < nw) smem32[lane] = inc - v;
        if (lane == 31) smem32[32] = inc;
    }
    __syncthreads();
    int r = smem32[warp] + before;
    *tot = smem32[32];
    __syncthreads();
    return r;
}

// Exclusive scan of per-thread counts over the CTA (blockDim.x <= 1024); the CTA total in *tot.
__device__ __forceinline__ int block_excl(int v, int* sm, int* tot) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    int inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += u;
    }
    if (lane == 31) sm[w] = inc;
    __syncthreads();
    if (w == 0) {
        int x = lane < nw ? sm[lane] : 0, xi = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int u = __shfl_up_sync(0xffffffffu, xi, o);
            if (lane >= o) xi += u;
        }
        if (lane < nw) sm[lane] = xi - x;
        if (lane == 31) sm[32] = xi;
    }
    __syncthreads();
    int r = sm[w] + inc - v;
    *tot = sm[32];
    __syncthreads();
    return r;
}

// A voxel whose point cap is crossed in this batch sums only its first `room` points in index order: the
// whole warp (every lane active) scans pslot[i0, n) for slot s, 128 entries per round, ranks the hits with
// ballots and calls add(j) for the first `room` of them. Same points as a serial scan from i0; the adds are
// integer atomics, so which lane makes them does not change the sums.
template <class Add>
__device__ __forceinline__ void warp_fill_first(const int* __restrict__ pslot, int64_t i0, int64_t n, int s,
                                                int room, Add add) {
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    for (int64_t j0 = i0; j0 < n && room > 0; j0 += 128) {
        bool hit[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            int64_t j = j0 + 32 * u + lane;
            hit[u] = j < n && pslot[j] == s;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            unsigned m = __ballot_sync(0xffffffffu, hit[u]);
            if (hit[u] && __popc(m & below) < room) add(j0 + 32 * u + lane);
            room -= __popc(m);
        }
    }
}

// ---- bounded grid barrier -------------------------------------------------------------------------------
// bar[0] counts arrivals, bar[1] is the generation. Every CTA of a cooperative launch calls it; a CTA that
// waits longer than the spin budget sets *err and returns false (the kernel then exits), so a fault can
// never leave the GPU spinning. A launch that gave up leaves bar[0] part counted: the launcher zeroes it
// before the next launch.
constexpr long long BARRIER_SPINS = 1LL << 24;  // x ~100 ns sleeps: ~2 s at most

__device__ __forceinline__ bool grid_barrier(uint32_t* bar, int* err, int code, long long budget = BARRIER_SPINS) {
    __shared__ int ok_s;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile uint32_t* gen = bar + 1;
        uint32_t g = *gen;
        __threadfence();
        uint32_t arrived = atomicAdd(bar, 1u);
        int ok = 1;
        if (arrived == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd((uint32_t*)gen, 1u);
        } else {
            long long spins = 0;
            while (*gen == g) {
                if (++spins > budget) {
                    atomicExch(err, code);
                    ok = 0;
                    break;
                }
                if (*(volatile int*)err != 0) {
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        ok_s = ok;
    }
    __syncthreads();
    return ok_s != 0;
}

// An arrival-count grid barrier for kernels that meet many times in one launch. *count only grows during a launch
// (the launcher zeroes it): every CTA adds 1 with release semantics after its writes, and episode e of a grid of G
// CTAs is over once the count reaches (e + 1) G, read with acquire semantics -- no reset, no generation word, so the
// last arrival releases the others with its one atomic. No separate fences: the block barrier orders the CTA's
// writes before thread 0's release add (release is cumulative), and the acquire load that sees the final count
// synchronises with every arrival's release, whose writes the closing block barrier then hands to the whole CTA.
// While thread 0 waits, thread 32 runs side() (work of this CTA that does not depend on the other CTAs). Thread 0
// polls without sleeping (each poll is one L2 round trip, ~0.2 us), so every CTA leaves within a round trip of the
// last arrival. A wait longer than `budget` polls sets *err and returns false; so does a wait during which another
// CTA gave up.
struct NoSide {
    __device__ void operator()() const {}
};

template <class Side = NoSide>
__device__ __forceinline__ bool grid_sync(uint32_t* count, uint32_t target, int* err, int code, long long budget,
                                          const Side& side = Side()) {
    __shared__ int ok_s;
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(count) : "memory");
        int ok = 1;
        long long spins = 0;
        while (true) {
            uint32_t v;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(count) : "memory");
            if ((int32_t)(v - target) >= 0) break;
            if (++spins > budget) {
                atomicExch(err, code);
                ok = 0;
                break;
            }
            if ((spins & 31) == 0 && *(volatile int*)err != 0) {
                ok = 0;
                break;
            }
        }
        ok_s = ok;
    } else if (threadIdx.x == 32) {
        side();
    }
    __syncthreads();
    return ok_s != 0;
}

// ---- grid sizing -----------------------------------------------------------------------------------------
inline int blocks_for(int64_t n, int threads, int cap = 1 << 20) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return (int)b;
}

}  // namespace lw
