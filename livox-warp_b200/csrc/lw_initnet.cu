// The learned start pose of the odometry: a point-set network (shared MLP 3 -> 64 -> 128 -> 256, max over the
// points, 512 -> 128 -> 6) on sm_100a. It has no counterpart in the reference, whose odometry predicts the next
// pose with constant velocity (odom.py:591-592); that prediction stays the network's input frame and fallback.
//
// Forward: one CTA of 128 threads per point set, eight 128-point tiles in turn. Layer 1 (K = 3) runs on the CUDA
// cores; layers 2 and 3 are tcgen05.mma (kind::f16, bf16 operands from shared memory in the canonical K-major
// layout without swizzle, float32 accumulators in TMEM). Layer 2 puts the points on M (D = H1 W2^T, one TMEM
// lane per point), so each thread converts its own point's 128 channels back to bf16 for layer 3. Layer 3 puts
// the channels on M (D = W3 H2^T, two M = 128 halves), so each thread holds one channel across the tile's points
// and the max-pool and its argmax are a per-thread scan of its TMEM lane -- no shuffles, no atomics.
//
// Backward: through the max only each channel's argmax point receives gradient, so it is sparse: one thread per
// (set, channel) recomputes its point's layer-1 and layer-2 activations in float32 and writes the per-row factors
// of the weight gradients; split-K reductions with a fixed order sum them (deterministic).
#include <cuda_bf16.h>

#include "lw_common.cuh"
#include "lw_linalg.cuh"
#include "lw_net.cuh"

namespace lw {

constexpr int NP = LW_NET_P;  // points per set
constexpr int NET_T = 128;    // threads (and points) per forward CTA
constexpr int C1 = 64, C2 = 128, C3 = 256, CH = 128, NOUT = 6;
constexpr long long NET_SPINS = 1LL << 24;

// forward shared memory (bytes)
constexpr uint32_t SM_W2 = 0;                       // [128 out][64 in] bf16, canonical K-major
constexpr uint32_t SM_W3 = SM_W2 + C2 * C1 * 2;     // [256 out][128 in]
constexpr uint32_t SM_H1 = SM_W3 + C3 * C2 * 2;     // [128 points][64]
constexpr uint32_t SM_H2 = SM_H1 + NET_T * C1 * 2;  // [128 points][128]
constexpr uint32_t SM_PAR = SM_H2 + NET_T * C2 * 2; // W1 [192], b1 [64], b2 [128], b3 [256] float
constexpr uint32_t SM_TOTAL = SM_PAR + (192 + 64 + 128 + 256) * 4;
constexpr uint32_t TMEM_COLS = 256;

__device__ __forceinline__ float bf(uint16_t v) { return __uint_as_float((uint32_t)v << 16); }
__device__ __forceinline__ uint16_t to_bf(float x) {
    __nv_bfloat16 b = __float2bfloat16_rn(x);
    return *reinterpret_cast<uint16_t*>(&b);
}
__device__ __forceinline__ float bfr(float x) { return bf(to_bf(x)); }  // rounded to bf16

// byte offset of element (r, k) of a [rows x K] bf16 tile in the canonical K-major layout without swizzle: 8-row
// x 16-byte core matrices, K-chunks of one row group adjacent (LBO = 128 B), row groups K/8 chunks apart (SBO)
__device__ __forceinline__ uint32_t kofs(int r, int k, int K) {
    return (uint32_t)((((r >> 3) * (K >> 3) + (k >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);  // version 1, SWIZZLE_NONE
}

// instruction descriptor of kind::f16: bf16 A and B (K-major), float32 D, M = 128, N = n
__host__ __device__ constexpr uint32_t umma_idesc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void umma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// bounded wait for phase `parity` of the mbarrier; false when it gave up
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (long long i = 0; i < NET_SPINS; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// 32 consecutive float32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// copy a row-major [rows][K] bf16 matrix into shared memory in the canonical layout (16-byte chunks)
__device__ __forceinline__ void load_canonical(const uint16_t* __restrict__ g, uint8_t* smem, int rows, int K) {
    const int chunks = rows * (K >> 3);
    for (int q = threadIdx.x; q < chunks; q += blockDim.x) {
        const int r = q / (K >> 3), kc = q % (K >> 3);
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(g + (size_t)r * K + kc * 8));
        *reinterpret_cast<uint4*>(smem + kofs(r, kc * 8, K)) = v;
    }
}

__global__ void __launch_bounds__(NET_T, 1)
    k_net_mlp(const uint16_t* __restrict__ w, float in_scale, const float4* __restrict__ sets,
              float* __restrict__ pooled, int32_t* __restrict__ argmax, int32_t* err) {
    extern __shared__ __align__(128) uint8_t sm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int set = blockIdx.x;
    const uint32_t bar_a = smem_u32(&bar);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    // weights into shared memory
    load_canonical(w + LW_NET_OFF_W2, sm + SM_W2, C2, C1);
    load_canonical(w + LW_NET_OFF_W3, sm + SM_W3, C3, C2);
    float* par = reinterpret_cast<float*>(sm + SM_PAR);
    float* sW1 = par;
    float* sb1 = par + 192;
    float* sb2 = par + 256;
    float* sb3 = par + 384;
    for (int i = tid; i < 192; i += NET_T) sW1[i] = bf(w[LW_NET_OFF_W1 + i]);
    for (int i = tid; i < C1; i += NET_T) sb1[i] = bf(w[LW_NET_OFF_B1 + i]);
    for (int i = tid; i < C2; i += NET_T) sb2[i] = bf(w[LW_NET_OFF_B2 + i]);
    for (int i = tid; i < C3; i += NET_T) sb3[i] = bf(w[LW_NET_OFF_B3 + i]);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = tmem_slot;
    const uint32_t lane_base = tbase + ((uint32_t)(warp * 32) << 16);
    const uint32_t s_w2 = smem_u32(sm + SM_W2), s_w3 = smem_u32(sm + SM_W3);
    const uint32_t s_h1 = smem_u32(sm + SM_H1), s_h2 = smem_u32(sm + SM_H2);
    float mx0 = -1.0f, mx1 = -1.0f;
    int ag0 = -1, ag1 = -1;
    uint32_t phase = 0;
    int failed = 0;
    const float4* pts = sets + (size_t)set * NP;
    for (int tile = 0; tile < NP / NET_T && !failed; ++tile) {
        // layer 1 on the CUDA cores: this thread's point, 64 channels, bf16 into H1's row
        {
            float4 p = __ldg(pts + tile * NET_T + tid);
            const float x = p.x * in_scale, y = p.y * in_scale, z = p.z * in_scale;
#pragma unroll
            for (int c8 = 0; c8 < C1 / 8; ++c8) {
                uint32_t pk[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    float h[2];
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const int j = c8 * 8 + q * 2 + e;
                        float a = sb1[j];
                        a = fmaf(sW1[3 * j + 0], x, a);
                        a = fmaf(sW1[3 * j + 1], y, a);
                        a = fmaf(sW1[3 * j + 2], z, a);
                        h[e] = fmaxf(a, 0.0f);
                    }
                    pk[q] = (uint32_t)to_bf(h[0]) | ((uint32_t)to_bf(h[1]) << 16);
                }
                *reinterpret_cast<uint4*>(sm + SM_H1 + kofs(tid, c8 * 8, C1)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
            }
        }
        fence_async_smem();
        __syncthreads();
        // layer 2: D[point][out] = H1 W2^T, TMEM columns 0..127
        if (tid == 0) {
            tc_fence_after();
#pragma unroll
            for (int s = 0; s < C1 / 16; ++s)
                umma(tbase, umma_desc(s_h1 + s * 256, 128, (C1 / 8) * 128), umma_desc(s_w2 + s * 256, 128, (C1 / 8) * 128),
                     umma_idesc(C2), s > 0);
            umma_commit(bar_a);
        }
        if (!mbar_wait(bar_a, phase)) failed = 1;
        phase ^= 1;
        if (__syncthreads_or(failed)) {
            failed = 1;
            break;
        }
        tc_fence_after();
        // epilogue 2: this thread's point (TMEM lane), 128 channels + bias, ReLU, bf16 into H2's row
#pragma unroll 1
        for (int c = 0; c < C2 / 32; ++c) {
            float v[32];
            tmem_ld32(lane_base + c * 32, v);
#pragma unroll
            for (int c8 = 0; c8 < 4; ++c8) {
                uint32_t pk[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int j0 = c * 32 + c8 * 8 + q * 2;
                    const float h0 = fmaxf(v[c8 * 8 + q * 2] + sb2[j0], 0.0f);
                    const float h1 = fmaxf(v[c8 * 8 + q * 2 + 1] + sb2[j0 + 1], 0.0f);
                    pk[q] = (uint32_t)to_bf(h0) | ((uint32_t)to_bf(h1) << 16);
                }
                *reinterpret_cast<uint4*>(sm + SM_H2 + kofs(tid, c * 32 + c8 * 8, C2)) =
                    make_uint4(pk[0], pk[1], pk[2], pk[3]);
            }
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        // layer 3: D[channel][point] = W3 H2^T, two halves of 128 channels in TMEM columns 0..255
        if (tid == 0) {
            tc_fence_after();
#pragma unroll
            for (int h = 0; h < 2; ++h)
#pragma unroll
                for (int s = 0; s < C2 / 16; ++s)
                    umma(tbase + h * 128, umma_desc(s_w3 + h * 16 * (C2 / 8) * 128 + s * 256, 128, (C2 / 8) * 128),
                         umma_desc(s_h2 + s * 256, 128, (C2 / 8) * 128), umma_idesc(NET_T), s > 0);
            umma_commit(bar_a);
        }
        if (!mbar_wait(bar_a, phase)) failed = 1;
        phase ^= 1;
        if (__syncthreads_or(failed)) {
            failed = 1;
            break;
        }
        tc_fence_after();
        // epilogue 3: this thread's channel (TMEM lane) over the tile's points: bias, ReLU, running max
#pragma unroll 1
        for (int h = 0; h < 2; ++h) {
            const float b = sb3[h * 128 + tid];
            float m = h ? mx1 : mx0;
            int ag = h ? ag1 : ag0;
#pragma unroll 1
            for (int c = 0; c < NET_T / 32; ++c) {
                float v[32];
                tmem_ld32(lane_base + h * 128 + c * 32, v);
#pragma unroll
                for (int i = 0; i < 32; ++i) {
                    const float zz = fmaxf(v[i] + b, 0.0f);
                    if (zz > m) {
                        m = zz;
                        ag = tile * NET_T + c * 32 + i;
                    }
                }
            }
            if (h) {
                mx1 = m;
                ag1 = ag;
            } else {
                mx0 = m;
                ag0 = ag;
            }
        }
        tc_fence_before();
        __syncthreads();
    }
    if (failed) {
        if (tid == 0) atomicExch(err, 1);
        mx0 = mx1 = 0.0f;
        ag0 = ag1 = -1;
    }
    pooled[(size_t)set * C3 + tid] = mx0;
    pooled[(size_t)set * C3 + 128 + tid] = mx1;
    argmax[(size_t)set * C3 + tid] = ag0;
    argmax[(size_t)set * C3 + 128 + tid] = ag1;
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(TMEM_COLS) : "memory");
    }
}

// The head of sample s: hid = bf16(ReLU(Wh1 bf16(pooled) + bh1)), step = (Wh2 hid + bh2) * out_scale.
__global__ void __launch_bounds__(CH) k_net_head(const uint16_t* __restrict__ w, const float* __restrict__ out_scale,
                                                 const float* __restrict__ pooled, float* __restrict__ hid,
                                                 float* __restrict__ step) {
    __shared__ float x[2 * C3];
    __shared__ float hs[CH];
    const int s = blockIdx.x, j = threadIdx.x;
    for (int k = j; k < 2 * C3; k += CH) x[k] = bfr(pooled[(size_t)s * 2 * C3 + k]);
    __syncthreads();
    float a = bf(w[LW_NET_OFF_BH1 + j]);
    const uint16_t* row = w + LW_NET_OFF_WH1 + (size_t)j * 2 * C3;
    for (int k = 0; k < 2 * C3; ++k) a = fmaf(bf(row[k]), x[k], a);
    const float h = bfr(fmaxf(a, 0.0f));
    hs[j] = h;
    hid[(size_t)s * CH + j] = h;
    __syncthreads();
    if (j < NOUT) {
        float o = bf(w[LW_NET_OFF_BH2 + j]);
        const uint16_t* r2 = w + LW_NET_OFF_WH2 + j * CH;
        for (int k = 0; k < CH; ++k) o = fmaf(bf(r2[k]), hs[k], o);
        step[(size_t)s * NOUT + j] = o * out_scale[j];
    }
}

// ---- backward -------------------------------------------------------------------------------------------------

// The head of sample s: loss, d(out), d(hidden pre-activation), d(pooled).
__global__ void __launch_bounds__(CH) k_net_head_bwd(const uint16_t* __restrict__ w, const float* __restrict__ out_scale,
                                                     const float* __restrict__ hid, const float* __restrict__ step,
                                                     const float* __restrict__ target, const float* __restrict__ wl,
                                                     int n, lw_net_scratch scr) {
    __shared__ float dout[NOUT];
    __shared__ float dz[CH];
    const int s = blockIdx.x, j = threadIdx.x;
    if (j < NOUT) {
        const float sc = out_scale[j];
        const float d = step[(size_t)s * NOUT + j] / sc - target[(size_t)s * NOUT + j] / sc;
        dout[j] = 2.0f * wl[j] * d / (float)n;
        scr.dout[(size_t)s * NOUT + j] = dout[j];
    }
    __syncthreads();
    if (j == 0) {
        float l = 0.0f;
        for (int o = 0; o < NOUT; ++o) {
            const float sc = out_scale[o];
            const float d = step[(size_t)s * NOUT + o] / sc - target[(size_t)s * NOUT + o] / sc;
            l += wl[o] * d * d;
        }
        scr.loss[s] = l / (float)n;
    }
    float dh = 0.0f;
    for (int o = 0; o < NOUT; ++o) dh = fmaf(dout[o], bf(w[LW_NET_OFF_WH2 + o * CH + j]), dh);
    const float z = hid[(size_t)s * CH + j] > 0.0f ? dh : 0.0f;
    dz[j] = z;
    scr.dzh[(size_t)s * CH + j] = z;
    __syncthreads();
    for (int k = j; k < 2 * C3; k += CH) {
        float g = 0.0f;
        for (int q = 0; q < CH; ++q) g = fmaf(dz[q], bf(w[LW_NET_OFF_WH1 + (size_t)q * 2 * C3 + k]), g);
        scr.dpool[(size_t)s * 2 * C3 + k] = g;
    }
}

// One (set, channel): the channel's argmax point gets d(pooled); recompute its layer-1/2 activations and write the
// rows the weight-gradient reductions read (K index = set * 256 + channel).
__global__ void __launch_bounds__(C3) k_net_pt_bwd(const uint16_t* __restrict__ w, float in_scale,
                                                   const float4* __restrict__ sets, const float* __restrict__ pooled,
                                                   const int32_t* __restrict__ argmax, int n_sets, lw_net_scratch scr) {
    const int set = blockIdx.x, c = threadIdx.x;
    const int64_t K = (int64_t)n_sets * C3;
    const int64_t kk = (int64_t)set * C3 + c;
    const int p = argmax[kk];
    const float v = pooled[kk];
    const float g = (p >= 0 && p < NP && v > 0.0f) ? scr.dpool[kk] : 0.0f;
    scr.dz3[kk] = g;
    uint16_t* h2row = scr.h2g + kk * C2;
    if (g == 0.0f) {
        for (int j = 0; j < C2; ++j) {
            h2row[j] = 0;
            scr.d2t[j * K + kk] = 0.0f;
        }
        for (int i = 0; i < C1; ++i) {
            scr.h1t[i * K + kk] = 0.0f;
            scr.d1t[i * K + kk] = 0.0f;
        }
        scr.h1t[C1 * K + kk] = 0.0f;
        for (int d = 0; d < 4; ++d) scr.xt[d * K + kk] = 0.0f;
        return;
    }
    const float4 q = __ldg(sets + (size_t)set * NP + p);
    const float x = q.x * in_scale, y = q.y * in_scale, z = q.z * in_scale;
    float h1[C1];
    bool a1[C1];
#pragma unroll
    for (int j = 0; j < C1; ++j) {
        float a = bf(w[LW_NET_OFF_B1 + j]);
        a = fmaf(bf(w[LW_NET_OFF_W1 + 3 * j + 0]), x, a);
        a = fmaf(bf(w[LW_NET_OFF_W1 + 3 * j + 1]), y, a);
        a = fmaf(bf(w[LW_NET_OFF_W1 + 3 * j + 2]), z, a);
        a1[j] = a > 0.0f;
        h1[j] = bfr(fmaxf(a, 0.0f));
        scr.h1t[j * K + kk] = h1[j];
    }
    scr.h1t[C1 * K + kk] = 1.0f;
    scr.xt[0 * K + kk] = x;
    scr.xt[1 * K + kk] = y;
    scr.xt[2 * K + kk] = z;
    scr.xt[3 * K + kk] = 1.0f;
    float d1[C1];
#pragma unroll
    for (int i = 0; i < C1; ++i) d1[i] = 0.0f;
    const uint16_t* w3row = w + LW_NET_OFF_W3 + (size_t)c * C2;
    for (int j = 0; j < C2; ++j) {
        const uint16_t* w2row = w + LW_NET_OFF_W2 + (size_t)j * C1;
        float a = bf(w[LW_NET_OFF_B2 + j]);
#pragma unroll
        for (int i = 0; i < C1; ++i) a = fmaf(bf(w2row[i]), h1[i], a);
        h2row[j] = to_bf(fmaxf(a, 0.0f));
        const float d2 = a > 0.0f ? g * bf(w3row[j]) : 0.0f;
        scr.d2t[j * K + kk] = d2;
        if (d2 != 0.0f) {
#pragma unroll
            for (int i = 0; i < C1; ++i) d1[i] = fmaf(d2, bf(w2row[i]), d1[i]);
        }
    }
#pragma unroll
    for (int i = 0; i < C1; ++i) scr.d1t[i * K + kk] = a1[i] ? d1[i] : 0.0f;
}

// Split-K partials of C[r][q] = sum_k A[r][k] B[q][k] (rows of length K): chunk `blockIdx.x` of kc columns.
constexpr int DOT_KC = 32;
__global__ void __launch_bounds__(256) k_dot_rows(const float* __restrict__ A, int R, const float* __restrict__ B,
                                                  int Q, int64_t K, int64_t chunk, float* __restrict__ part) {
    __shared__ float sa[128][DOT_KC + 1];
    __shared__ float sb[65][DOT_KC + 1];
    const int t = threadIdx.x;
    const int64_t k0 = (int64_t)blockIdx.x * chunk, k1 = min(K, k0 + chunk);
    const int RQ = R * Q;
    float acc[33];
#pragma unroll
    for (int u = 0; u < 33; ++u) acc[u] = 0.0f;
    for (int64_t kb = k0; kb < k1; kb += DOT_KC) {
        const int kn = (int)min((int64_t)DOT_KC, k1 - kb);
        for (int e = t; e < R * DOT_KC; e += 256) {
            const int r = e / DOT_KC, kx = e % DOT_KC;
            sa[r][kx] = kx < kn ? A[(int64_t)r * K + kb + kx] : 0.0f;
        }
        for (int e = t; e < Q * DOT_KC; e += 256) {
            const int qq = e / DOT_KC, kx = e % DOT_KC;
            sb[qq][kx] = kx < kn ? B[(int64_t)qq * K + kb + kx] : 0.0f;
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 33; ++u) {
            const int o = t + 256 * u;
            if (o < RQ) {
                const int r = o / Q, qq = o % Q;
                float a = acc[u];
#pragma unroll 8
                for (int kx = 0; kx < DOT_KC; ++kx) a = fmaf(sa[r][kx], sb[qq][kx], a);
                acc[u] = a;
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < 33; ++u) {
        const int o = t + 256 * u;
        if (o < RQ) part[(int64_t)blockIdx.x * RQ + o] = acc[u];
    }
}

// out[o] = sum over splits of part[split][o], in split order; scattered into the gradient by `map`.
// mode 0: dW2|db2 from C[128][65]; mode 1: dW1|db1 from C[64][4]
__global__ void k_dot_reduce(const float* __restrict__ part, int splits, int RQ, int mode, float* __restrict__ grad) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= RQ) return;
    float s = 0.0f;
    for (int k = 0; k < splits; ++k) s += part[(int64_t)k * RQ + o];
    if (mode == 0) {
        const int j = o / 65, i = o % 65;
        if (i < 64)
            grad[LW_NET_OFF_W2 + j * 64 + i] = s;
        else
            grad[LW_NET_OFF_B2 + j] = s;
    } else {
        const int i = o / 4, d = o % 4;
        if (d < 3)
            grad[LW_NET_OFF_W1 + i * 3 + d] = s;
        else
            grad[LW_NET_OFF_B1 + i] = s;
    }
}

// dW3[c][k] = sum_set dz3[set][c] h2g[set][c][k], db3[c] = sum_set dz3[set][c]
__global__ void k_net_dw3(const lw_net_scratch scr, int n_sets, float* __restrict__ grad) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= C3 * (C2 + 1)) return;
    const int c = o / (C2 + 1), k = o % (C2 + 1);
    float s = 0.0f;
    for (int set = 0; set < n_sets; ++set) {
        const int64_t kk = (int64_t)set * C3 + c;
        const float g = scr.dz3[kk];
        if (g != 0.0f) s = fmaf(g, k < C2 ? bf(scr.h2g[kk * C2 + k]) : 1.0f, s);
    }
    if (k < C2)
        grad[LW_NET_OFF_W3 + c * C2 + k] = s;
    else
        grad[LW_NET_OFF_B3 + c] = s;
}

// the head's weights: dWh1[j][k] = sum_s dzh[s][j] bf16(pooled)[s][k], dbh1, dWh2[o][j] = sum_s dout[s][o] hid[s][j],
// dbh2
__global__ void k_net_dhead(const lw_net_scratch scr, const float* __restrict__ pooled, const float* __restrict__ hid,
                            int n, float* __restrict__ grad) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    const int n1 = CH * (2 * C3 + 1), n2 = NOUT * (CH + 1);
    if (o < n1) {
        const int j = o / (2 * C3 + 1), k = o % (2 * C3 + 1);
        float s = 0.0f;
        for (int q = 0; q < n; ++q)
            s = fmaf(scr.dzh[(size_t)q * CH + j], k < 2 * C3 ? bfr(pooled[(size_t)q * 2 * C3 + k]) : 1.0f, s);
        if (k < 2 * C3)
            grad[LW_NET_OFF_WH1 + j * 2 * C3 + k] = s;
        else
            grad[LW_NET_OFF_BH1 + j] = s;
    } else if (o < n1 + n2) {
        const int e = o - n1, oo = e / (CH + 1), j = e % (CH + 1);
        float s = 0.0f;
        for (int q = 0; q < n; ++q) s = fmaf(scr.dout[(size_t)q * NOUT + oo], j < CH ? hid[(size_t)q * CH + j] : 1.0f, s);
        if (j < CH)
            grad[LW_NET_OFF_WH2 + oo * CH + j] = s;
        else
            grad[LW_NET_OFF_BH2 + oo] = s;
    }
}

// ---- optimiser and initialisation ------------------------------------------------------------------------------

__global__ void k_net_adam(lw_initnet net, int t, float lr, float b1, float b2, float eps, float wd) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= LW_NET_NPARAM) return;
    if (i >= LW_NET_OFF_BH2 + NOUT) {
        net.w[i] = 0;
        return;
    }
    const float g = net.grad[i];
    const float m = b1 * net.adam_m[i] + (1.0f - b1) * g;
    const float v = b2 * net.adam_v[i] + (1.0f - b2) * g * g;
    net.adam_m[i] = m;
    net.adam_v[i] = v;
    const float mh = m / (1.0f - powf(b1, (float)t));
    const float vh = v / (1.0f - powf(b2, (float)t));
    float x = net.master[i];
    x -= lr * (mh / (sqrtf(vh) + eps) + wd * x);
    net.master[i] = x;
    net.w[i] = to_bf(x);
}

__device__ __forceinline__ float hash_uniform(uint64_t seed, uint64_t i) {  // splitmix64 -> [0, 1)
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (i + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (float)(z >> 40) * (1.0f / 16777216.0f);
}

__global__ void k_net_init(lw_initnet net, uint64_t seed) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= LW_NET_NPARAM) return;
    float lim = 0.0f;  // biases and padding stay zero
    if (i < LW_NET_OFF_B1) lim = sqrtf(6.0f / 3.0f);
    else if (i >= LW_NET_OFF_W2 && i < LW_NET_OFF_B2) lim = sqrtf(6.0f / 64.0f);
    else if (i >= LW_NET_OFF_W3 && i < LW_NET_OFF_B3) lim = sqrtf(6.0f / 128.0f);
    else if (i >= LW_NET_OFF_WH1 && i < LW_NET_OFF_BH1) lim = sqrtf(6.0f / 512.0f);
    else if (i >= LW_NET_OFF_WH2 && i < LW_NET_OFF_BH2) lim = 0.1f * sqrtf(6.0f / 128.0f);
    const float x = lim * (2.0f * hash_uniform(seed, (uint64_t)i) - 1.0f);
    net.master[i] = x;
    net.w[i] = to_bf(x);
    net.adam_m[i] = 0.0f;
    net.adam_v[i] = 0.0f;
    net.grad[i] = 0.0f;
}

// ---- the frame's two point sets ----------------------------------------------------------------------------------

// per 1024-slot tile: occupied registration voxels whose mean lies within radius of T's origin
__device__ __forceinline__ bool map_cand(const lw_regmap& reg, int64_t s, float ox, float oy, float oz, float r2) {
    if (reg.keys[s] == -1) return false;
    const float4 m = __ldg(reinterpret_cast<const float4*>(reg.rec + s * LW_REC_FLOATS));
    if (!(m.w > 0.0f)) return false;
    const float dx = m.x - ox, dy = m.y - oy, dz = m.z - oz;
    return dx * dx + dy * dy + dz * dz <= r2;
}

__global__ void __launch_bounds__(256) k_ns_count(lw_regmap reg, const double* T, float r2, int32_t* tiles) {
    const int64_t base = (int64_t)blockIdx.x * 1024;
    const float ox = (float)T[3], oy = (float)T[7], oz = (float)T[11];
    int c = 0;
    for (int q = 0; q < 4; ++q) {
        const int64_t s = base + threadIdx.x * 4 + q;
        if (s < reg.cap && map_cand(reg, s, ox, oy, oz, r2)) ++c;
    }
    __shared__ int ws[8];
    int v = c;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int k = 0; k < 8; ++k) t += ws[k];
        tiles[blockIdx.x] = t;
    }
}

// exclusive prefix of the tile counts (one CTA), total into count[1]
__global__ void __launch_bounds__(1024) k_ns_scan(int32_t* tiles, int nt, int32_t* count) {
    __shared__ int32_t part[1024];
    const int per = (nt + 1023) / 1024;
    const int t = threadIdx.x;
    int s = 0;
    for (int k = 0; k < per; ++k) {
        const int i = t * per + k;
        if (i < nt) s += tiles[i];
    }
    part[t] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const int v = t >= o ? part[t - o] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int run = t ? part[t - 1] : 0;
    for (int k = 0; k < per; ++k) {
        const int i = t * per + k;
        if (i < nt) {
            const int c = tiles[i];
            tiles[i] = run;
            run += c;
        }
    }
    if (t == 1023) count[1] = part[1023];
}

__global__ void __launch_bounds__(256) k_ns_scatter(lw_regmap reg, const double* T, float r2, const int32_t* tiles,
                                                    int32_t* cand) {
    const int64_t base = (int64_t)blockIdx.x * 1024;
    const float ox = (float)T[3], oy = (float)T[7], oz = (float)T[11];
    bool f[4];
    int c = 0;
    for (int q = 0; q < 4; ++q) {
        const int64_t s = base + threadIdx.x * 4 + q;
        f[q] = s < reg.cap && map_cand(reg, s, ox, oy, oz, r2);
        c += f[q];
    }
    // exclusive prefix of c over the CTA, in thread order
    __shared__ int ws[8];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int v = c;
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
    }
    if (lane == 31) ws[wid] = v;
    __syncthreads();
    int off = tiles[blockIdx.x] + v - c;
    for (int k = 0; k < wid; ++k) off += ws[k];
    for (int q = 0; q < 4; ++q)
        if (f[q]) cand[off++] = (int32_t)(base + threadIdx.x * 4 + q);
}

// The frame set: LW_NET_P thinned frame points at an even stride (sensor frame). The map set: with voxel > 0, for
// each of those points the nearest registration voxel mean among the 27 voxels around it at pose T (the point
// itself when none is occupied) -- the map as the frame should see it; otherwise the patch of candidates (voxel
// means within the radius, in slot order) at an even stride. Both in T's frame.
__global__ void k_ns_fill(const float4* __restrict__ ds, const int32_t* n_ds, lw_regmap reg, const double* T,
                          const int32_t* cand, int32_t* count, float voxel, float4* __restrict__ sets) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NP) return;
    const int nf = *n_ds;
    if (i == 0) count[0] = nf;
    const float4 f = nf > 0 ? ds[(int64_t)i * nf / NP] : make_float4(0.f, 0.f, 0.f, 0.f);
    sets[i] = make_float4(f.x, f.y, f.z, 0.f);
    float mx = 0.f, my = 0.f, mz = 0.f;
    bool have = false;
    if (voxel > 0.0f) {
        if (nf > 0) {
            const double wx = T[0] * f.x + T[1] * f.y + T[2] * f.z + T[3];
            const double wy = T[4] * f.x + T[5] * f.y + T[6] * f.z + T[7];
            const double wz = T[8] * f.x + T[9] * f.y + T[10] * f.z + T[11];
            const float inv = 1.0f / voxel;
            const int ix = ifloor((float)wx * inv), iy = ifloor((float)wy * inv), iz = ifloor((float)wz * inv);
            const int mask = (int)(reg.cap - 1);
            float bd = 1.0e30f;
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        const int sl = find_slot(key_ijk(ix + dx, iy + dy, iz + dz), reg.keys, mask);
                        if (sl < 0) continue;
                        const float4 m = __ldg(reinterpret_cast<const float4*>(reg.rec + (int64_t)sl * LW_REC_FLOATS));
                        if (!(m.w > 0.0f)) continue;
                        const float ex = m.x - (float)wx, ey = m.y - (float)wy, ez = m.z - (float)wz;
                        const float d2 = ex * ex + ey * ey + ez * ez;
                        if (d2 < bd) {
                            bd = d2;
                            mx = m.x;
                            my = m.y;
                            mz = m.z;
                            have = true;
                        }
                    }
        }
    } else {
        const int nm = count[1];
        if (nm > 0) {
            const int sl = cand[(int64_t)i * nm / NP];
            const float4 m = __ldg(reinterpret_cast<const float4*>(reg.rec + (int64_t)sl * LW_REC_FLOATS));
            mx = m.x;
            my = m.y;
            mz = m.z;
            have = true;
        }
    }
    float4 o = voxel > 0.0f ? make_float4(f.x, f.y, f.z, 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
    if (have) {
        const double dx = (double)mx - T[3], dy = (double)my - T[7], dz = (double)mz - T[11];
        o.x = (float)(T[0] * dx + T[4] * dy + T[8] * dz);  // R^T (m - t)
        o.y = (float)(T[1] * dx + T[5] * dy + T[9] * dz);
        o.z = (float)(T[2] * dx + T[6] * dy + T[10] * dz);
    }
    sets[NP + i] = o;
}

int net_sets_launch(const float* ds_xyz, const int32_t* n_ds, const lw_regmap& reg, const double* T, float radius,
                    float voxel, float* sets, int32_t* cand, int32_t* tiles, int32_t* count, cudaStream_t s) {
    int launches = 1;
    if (!(voxel > 0.0f)) {
        const int nt = (int)((reg.cap + 1023) / 1024);
        const float r2 = radius * radius;
        k_ns_count<<<nt, 256, 0, s>>>(reg, T, r2, tiles);
        k_ns_scan<<<1, 1024, 0, s>>>(tiles, nt, count);
        k_ns_scatter<<<nt, 256, 0, s>>>(reg, T, r2, tiles, cand);
        launches += 3;
    }
    k_ns_fill<<<NP / 256, 256, 0, s>>>(reinterpret_cast<const float4*>(ds_xyz), n_ds, reg, T, cand, count, voxel,
                                       reinterpret_cast<float4*>(sets));
    LW_LAUNCHED("lw_net_sets");
    count_launches(launches);
    return LW_OK;
}

int net_forward_launch(const lw_initnet& net, const float* sets, int n, float* pooled, int32_t* argmax, float* hid,
                       float* step, int32_t* err, cudaStream_t s) {
    static bool attr_set[64] = {};
    int dev = 0;
    LW_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64 || !attr_set[dev]) {
        LW_CUDA(cudaFuncSetAttribute(k_net_mlp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM_TOTAL));
        if (dev >= 0 && dev < 64) attr_set[dev] = true;
    }
    k_net_mlp<<<2 * n, NET_T, SM_TOTAL, s>>>(net.w, net.in_scale, reinterpret_cast<const float4*>(sets), pooled,
                                             argmax, err);
    k_net_head<<<n, CH, 0, s>>>(net.w, net.out_scale, pooled, hid, step);
    LW_LAUNCHED("lw_net_forward");
    count_launches(2);
    return LW_OK;
}

// T_pred = T_reg = T_pred * [R(step_r), step_t] when the frame registers and the network ran cleanly
__global__ void k_net_apply(lw_odom_state* st, const float* step, const int32_t* err) {
    if (!st->run_reg || *err != 0) return;
    double d[6];
    for (int j = 0; j < 6; ++j) d[j] = (double)step[j];
    for (int j = 0; j < 6; ++j)
        if (!(fabs(d[j]) < 10.0)) return;  // a non-finite or absurd step keeps the prediction
    double R[9], T[16];
    rotvec_to_mat(d + 3, R);
    for (int i = 0; i < 16; ++i) T[i] = st->T_pred[i];
    double o[16];
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) o[i * 4 + j] = T[i * 4 + 0] * R[j] + T[i * 4 + 1] * R[3 + j] + T[i * 4 + 2] * R[6 + j];
        o[i * 4 + 3] = T[i * 4 + 0] * d[0] + T[i * 4 + 1] * d[1] + T[i * 4 + 2] * d[2] + T[i * 4 + 3];
    }
    o[12] = o[13] = o[14] = 0.0;
    o[15] = 1.0;
    for (int i = 0; i < 16; ++i) st->T_pred[i] = st->T_reg[i] = o[i];
}

int net_apply_launch(lw_odom_state* st, const float* step, const int32_t* err, cudaStream_t s) {
    k_net_apply<<<1, 1, 0, s>>>(st, step, err);
    LW_LAUNCHED("lw_net_apply");
    count_launches(1);
    return LW_OK;
}

}  // namespace lw

using namespace lw;

static int check_net(const lw_initnet* net, const char* who) {
    if (!net || !net->master || !net->w || !net->grad || !net->adam_m || !net->adam_v || !net->out_scale)
        return set_error(LW_EINVAL, "%s: incomplete network", who);
    if (((uintptr_t)net->w & 15) != 0) return set_error(LW_EINVAL, "%s: bf16 weights must be 16-byte aligned", who);
    return LW_OK;
}

extern "C" {

int lw_net_init(lw_initnet* net, uint64_t seed, void* stream) {
    int r = check_net(net, "lw_net_init");
    if (r != LW_OK) return r;
    k_net_init<<<blocks_for(LW_NET_NPARAM, 256), 256, 0, (cudaStream_t)stream>>>(*net, seed);
    LW_LAUNCHED("lw_net_init");
    count_launches(1);
    return LW_OK;
}

int lw_net_forward(const lw_initnet* net, const float* sets, int32_t n, float* pooled, int32_t* argmax, float* hid,
                   float* step, int32_t* err, void* stream) {
    int r = check_net(net, "lw_net_forward");
    if (r != LW_OK) return r;
    if (!sets || !pooled || !argmax || !hid || !step || !err || n < 1 || n > (1 << 20))
        return set_error(LW_EINVAL, "lw_net_forward: bad arguments");
    if (((uintptr_t)sets & 15) != 0) return set_error(LW_EINVAL, "lw_net_forward: sets must be 16-byte aligned");
    ProfScope prof("net_forward", (cudaStream_t)stream);
    return net_forward_launch(*net, sets, n, pooled, argmax, hid, step, err, (cudaStream_t)stream);
}

int lw_net_backward(const lw_initnet* net, const float* sets, int32_t n, const float* pooled, const int32_t* argmax,
                    const float* hid, const float* step, const float* target, const float* w_loss,
                    lw_net_scratch* scr, void* stream) {
    int r = check_net(net, "lw_net_backward");
    if (r != LW_OK) return r;
    if (!sets || !pooled || !argmax || !hid || !step || !target || !w_loss || !scr || n < 1)
        return set_error(LW_EINVAL, "lw_net_backward: bad arguments");
    if (n > scr->n_cap) return set_error(LW_ECAPACITY, "lw_net_backward: %d samples > scratch for %d", n, scr->n_cap);
    cudaStream_t s = (cudaStream_t)stream;
    ProfScope prof("net_backward", s);
    const int n_sets = 2 * n;
    const int64_t K = (int64_t)n_sets * C3;
    k_net_head_bwd<<<n, CH, 0, s>>>(net->w, net->out_scale, hid, step, target, w_loss, n, *scr);
    k_net_pt_bwd<<<n_sets, C3, 0, s>>>(net->w, net->in_scale, reinterpret_cast<const float4*>(sets), pooled, argmax,
                                       n_sets, *scr);
    const int splits = 64;
    const int64_t chunk = ((K + splits - 1) / splits + DOT_KC - 1) / DOT_KC * DOT_KC;
    const int used = (int)((K + chunk - 1) / chunk);
    k_dot_rows<<<used, 256, 0, s>>>(scr->d2t, C2, scr->h1t, C1 + 1, K, chunk, scr->part);
    k_dot_reduce<<<blocks_for(C2 * (C1 + 1), 256), 256, 0, s>>>(scr->part, used, C2 * (C1 + 1), 0, net->grad);
    k_dot_rows<<<used, 256, 0, s>>>(scr->d1t, C1, scr->xt, 4, K, chunk, scr->part);  // after the reduce above
    k_dot_reduce<<<1, 256, 0, s>>>(scr->part, used, C1 * 4, 1, net->grad);
    k_net_dw3<<<blocks_for(C3 * (C2 + 1), 256), 256, 0, s>>>(*scr, n_sets, net->grad);
    k_net_dhead<<<blocks_for(CH * (2 * C3 + 1) + NOUT * (CH + 1), 256), 256, 0, s>>>(*scr, pooled, hid, n, net->grad);
    LW_LAUNCHED("lw_net_backward");
    count_launches(8);
    return LW_OK;
}

int lw_net_adam(lw_initnet* net, int32_t t, float lr, float beta1, float beta2, float eps, float weight_decay,
                void* stream) {
    int r = check_net(net, "lw_net_adam");
    if (r != LW_OK) return r;
    if (t < 1) return set_error(LW_EINVAL, "lw_net_adam: step count starts at 1");
    k_net_adam<<<blocks_for(LW_NET_NPARAM, 256), 256, 0, (cudaStream_t)stream>>>(*net, t, lr, beta1, beta2, eps,
                                                                                 weight_decay);
    LW_LAUNCHED("lw_net_adam");
    count_launches(1);
    return LW_OK;
}

int lw_net_sets(const float* ds_xyz, const int32_t* n_ds, const lw_regmap* reg, const double* T, float radius,
                float voxel, float* sets_out, int32_t* cand, int32_t* tiles, int32_t* count, void* stream) {
    if (!ds_xyz || !n_ds || !reg || !reg->keys || !reg->rec || !T || !sets_out || !count ||
        (!(voxel > 0.0f) && (!cand || !tiles)))
        return set_error(LW_EINVAL, "lw_net_sets: null argument");
    if (voxel > 0.0f && (reg->cap & (reg->cap - 1)) != 0)
        return set_error(LW_EINVAL, "lw_net_sets: the map capacity must be a power of two");
    if (reg->cap <= 0 || reg->cap > (1LL << 30)) return set_error(LW_EINVAL, "lw_net_sets: bad map capacity");
    if (((uintptr_t)ds_xyz & 15) != 0 || ((uintptr_t)sets_out & 15) != 0)
        return set_error(LW_EINVAL, "lw_net_sets: points must be 16-byte aligned");
    return net_sets_launch(ds_xyz, n_ds, *reg, T, radius, voxel, sets_out, cand, tiles, count, (cudaStream_t)stream);
}

}  // extern "C"
