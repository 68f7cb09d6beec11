// surrogate.cu -- learned chemistry for the IRT: track descriptors and a small
// MLP (64 -> 128 -> 128 -> 128 -> 80, GELU) trained and evaluated with
// hand-written tcgen05 kernels: bf16 operands in shared memory (K-major,
// no swizzle), f32 accumulators in tensor memory, one elected thread issuing
// the MMAs, an mbarrier signalled by tcgen05.commit.
//
// Forward: one CTA (4 warps) per tile of 128 tracks; the 4 layers run back to
// back with the activations kept in shared memory.  Warp w owns TMEM lanes
// 32w..32w+31 = rows 32w..32w+31 of the tile, so each thread finishes the
// epilogue (bias, GELU, bf16 rounding) of its own row.
//
// Backward: per tile, layer by layer, the weight gradient dW = D^T H (K = the
// tile's 128 rows) and the input gradient dH = D W (K = the layer's outputs)
// are two MMAs into two TMEM regions; the weight gradients of all tiles are
// summed with f32 atomics.  Loss: mean squared error over the batch and the
// 80 outputs of the standardised G(t) curves.
#include "surrogate.cuh"
#include "common.cuh"

namespace wg {

// ------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t s2u(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long sg_time() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t cnt) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s2u(b)), "r"(cnt) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(s2u(b)), "r"(parity)
        : "memory");
    return ok != 0;
}

// wait for the phase of the given parity, at most lim_ns (0: give up before
// the first poll)
__device__ bool mbar_wait(uint64_t* b, uint32_t parity, unsigned long long lim_ns) {
    if (lim_ns == 0) return false;
    const unsigned long long t0 = sg_time();
    while (!mbar_try(b, parity))
        if (sg_time() - t0 > lim_ns) return false;
    return true;
}

// Wait for the MMAs committed to phase `parity`.  A wait that runs out clears
// *ok (the kernel reports SG_ERR_WAIT) and is followed by a drain wait of at
// most WG_MMA_WAIT_NS, so that tensor memory is not read, reissued or freed
// under an MMA still in flight.
__device__ __forceinline__ void mma_wait(uint64_t* b, uint32_t parity, unsigned long long lim_ns, bool& ok) {
    if (!mbar_wait(b, parity, lim_ns)) {
        ok = false;
        mbar_wait(b, parity, WG_MMA_WAIT_NS);
    }
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {     // one full warp
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(s2u(dst)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {   // the allocating warp
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// all threads: make generic shared-memory writes visible to the tensor cores,
// and order earlier tensor-memory reads before later MMAs
__device__ __forceinline__ void sg_sync() {
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
}

// Shared-memory matrix descriptor: K-major, no swizzle.  Core matrices are
// 8 rows x 16 bytes stored contiguously (128 B); the next core matrix along K
// is LBO bytes on, the next group of 8 rows SBO bytes on; version 1 (bit 46).
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: bf16 A and B (both K-major), f32 D, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// byte offset of element (r, k) of an R x K operand in that layout
__device__ __forceinline__ uint32_t coff(uint32_t r, uint32_t k, uint32_t K) {
    return ((((r >> 3) * (K >> 3)) + (k >> 3)) << 7) + ((r & 7u) << 4) + ((k & 7u) << 1);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t ad, uint64_t bd, uint32_t id, uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(d_tmem), "l"(ad), "l"(bd), "r"(id), "r"(accum), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(s2u(bar))
                 : "memory");
}

// D (TMEM, M x N f32) = A (M x K) * B (N x K)^T, K a multiple of 16; one thread
__device__ __forceinline__ void gemm_issue(uint32_t d_tmem, uint32_t sa, uint32_t sb, int M, int N, int K) {
    const uint32_t id = idesc_bf16(M, N);
    const uint32_t sbo = (uint32_t)(K >> 3) << 7;
    for (int j = 0; j < K / 16; ++j)
        umma_bf16(d_tmem, sdesc(sa + 256u * j, 128u, sbo), sdesc(sb + 256u * j, 128u, sbo), id, j > 0 ? 1u : 0u);
}

// 32 consecutive f32 columns of this warp's 32 TMEM lanes (one row per thread)
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float z) {
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * __expf(-0.5f * z * z);
}

constexpr uint32_t SG_ERR_WAIT = 1u << 6;    // an mbarrier wait gave up

// copy W [R][K] (bf16, row-major) into the canonical layout at dst
__device__ __forceinline__ void load_operand(uint8_t* dst, const __nv_bfloat16* W, int R, int K) {
    const int chunks = K >> 3;
    for (int e = threadIdx.x; e < R * chunks; e += blockDim.x) {
        const int r = e / chunks, c = e - r * chunks;
        *reinterpret_cast<uint4*>(dst + coff(r, 8 * c, K)) = *reinterpret_cast<const uint4*>(W + (size_t)r * K + 8 * c);
    }
}

// ------------------------------------------------------------ forward
__global__ void __launch_bounds__(SG_TILE, 1) k_sg_fwd(SgFwdArgs a) {
    extern __shared__ __align__(1024) uint8_t sm[];
    uint8_t* bufA = sm;                  // activations, 128 x K bf16
    uint8_t* bufB = sm + 32768;          // weights, N x K bf16
    __shared__ uint64_t bar;
    __shared__ uint32_t tbase;
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t r = blockIdx.x * SG_TILE + tid;
    const bool live = r < a.n;
    const uint32_t src = live ? (a.rows ? a.rows[r] : r) : 0u;
    if (warp == 0) tmem_alloc(&tbase, 128);
    if (tid == 0) mbar_init(&bar, 1);
    // input row -> bf16, canonical [128][64]
    for (int c = 0; c < SG_IN / 8; ++c) {
        __align__(16) __nv_bfloat16 h[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            float x = live ? a.X[(size_t)src * SG_IN + 8 * c + j] : 0.0f;
            if (a.xmean && live) x = (x - a.xmean[8 * c + j]) * a.xinv[8 * c + j];
            h[j] = __float2bfloat16_rn(x);
        }
        *reinterpret_cast<uint4*>(bufA + coff(tid, 8 * c, SG_IN)) = *reinterpret_cast<uint4*>(h);
        if (a.H0 && live) *reinterpret_cast<uint4*>(a.H0 + (size_t)r * SG_IN + 8 * c) = *reinterpret_cast<uint4*>(h);
    }
    sg_sync();
    const uint32_t tm = tbase;
    const uint32_t lane_tm = tm + ((uint32_t)(32 * warp) << 16);
    bool ok = true;
    for (int l = 0; l < 4; ++l) {
        const int K = l == 0 ? SG_IN : SG_HID, N = l == 3 ? SG_OUT : SG_HID;
        load_operand(bufB, a.w.W[l], N, K);
        sg_sync();
        if (tid == 0) {
            gemm_issue(tm, s2u(bufA), s2u(bufB), SG_TILE, N, K);
            umma_commit(&bar);
        }
        mma_wait(&bar, (uint32_t)(l & 1), (l == 0 && a.give_up_first) ? 0ull : a.mma_ns, ok);
        tc_after_sync();
        const float* bias = a.w.p + (l == 0 ? SG_OFF_B1 : l == 1 ? SG_OFF_B2 : l == 2 ? SG_OFF_B3 : SG_OFF_B4);
        float* Zs = l == 0 ? a.Z1 : l == 1 ? a.Z2 : l == 2 ? a.Z3 : nullptr;
        __nv_bfloat16* Hs = l == 0 ? a.H1 : l == 1 ? a.H2 : l == 2 ? a.H3 : nullptr;
        for (int c0 = 0; c0 < N; c0 += 32) {
            float v[32];
            tmem_ld32(lane_tm + (uint32_t)c0, v);
            if (l == 3) {
                if (live && a.Y)
                    for (int j = 0; j < 32 && c0 + j < N; ++j) a.Y[(size_t)r * SG_OUT + c0 + j] = v[j] + bias[c0 + j];
                if (a.acc) {
                    // column sums over the tile's rows: each warp reduces its 32
                    // rows, lane 0 adds the warp's partial in f64
                    const float e = live ? (a.E ? a.E[r] : a.E0) : 0.0f;
#pragma unroll 4
                    for (int j = 0; j < 32; ++j) {
                        const int col = c0 + j;
                        if (col >= N) break;
                        float w = live ? ((v[j] + bias[col]) * a.ystd[col] + a.ymean[col]) * e : 0.0f;
#pragma unroll
                        for (int o = 16; o; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
                        if ((tid & 31) == 0) atomicAdd(&a.acc[col], (double)w);
                    }
                    if (c0 == 0) {
                        float w = e;
#pragma unroll
                        for (int o = 16; o; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
                        if ((tid & 31) == 0) atomicAdd(&a.acc[SG_OUT], (double)w);
                    }
                }
                continue;
            }
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                __align__(16) __nv_bfloat16 h[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int col = c0 + 8 * c + j;
                    const float z = v[8 * c + j] + bias[col];
                    if (Zs && live) Zs[(size_t)r * SG_HID + col] = z;
                    h[j] = __float2bfloat16_rn(gelu(z));
                }
                *reinterpret_cast<uint4*>(bufA + coff(tid, c0 + 8 * c, SG_HID)) = *reinterpret_cast<uint4*>(h);
                if (Hs && live) *reinterpret_cast<uint4*>(Hs + (size_t)r * SG_HID + c0 + 8 * c) = *reinterpret_cast<uint4*>(h);
            }
        }
        sg_sync();
    }
    if (warp == 0) tmem_dealloc(tm, 128);
    if (!ok && tid == 0) atomicOr(a.err, SG_ERR_WAIT);
}

// ------------------------------------------------------------ backward
// Writes row `tid` of the gradient D (n_out values in v, f32) into bufG
// (canonical [128][n_out]) and bufGT (canonical [n_out][128]) as bf16, and
// adds it to the bias-gradient partial sums.
__device__ __forceinline__ void put_grad_row(uint8_t* bufG, uint8_t* bufGT, float* sdb, int tid, int c0,
                                             const float* v, int cnt, int n_out) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        if (8 * c >= cnt) break;
        __align__(16) __nv_bfloat16 h[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const float g = v[8 * c + j];
            h[j] = __float2bfloat16_rn(g);
            atomicAdd(&sdb[c0 + 8 * c + j], g);
            *reinterpret_cast<__nv_bfloat16*>(bufGT + coff(c0 + 8 * c + j, tid, SG_TILE)) = h[j];
        }
        *reinterpret_cast<uint4*>(bufG + coff(tid, c0 + 8 * c, n_out)) = *reinterpret_cast<uint4*>(h);
    }
}

__global__ void __launch_bounds__(SG_TILE, 1) k_sg_bwd(SgBwdArgs a) {
    extern __shared__ __align__(1024) uint8_t sm[];
    uint8_t* bufG = sm;                  // D, 128 rows x n_out
    uint8_t* bufGT = sm + 32768;         // D^T, n_out x 128 rows
    uint8_t* bufXT = sm + 65536;         // H^T, n_in x 128 rows
    uint8_t* bufW = sm + 98304;          // W^T, n_in x n_out
    __shared__ float sdb[SG_HID];
    __shared__ uint64_t bar;
    __shared__ uint32_t tbase;
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t r = blockIdx.x * SG_TILE + tid;
    const bool live = r < a.n;
    const uint32_t src = live ? (a.rows ? a.rows[r] : r) : 0u;
    if (warp == 0) tmem_alloc(&tbase, 256);
    if (tid == 0) mbar_init(&bar, 1);
    sdb[tid] = 0.0f;
    __syncthreads();
    // D_3 = dL/dY = 2 (Y - T) / (n * 80); rows past n contribute zeros
    double sse = 0.0;
    const float scale = 2.0f / ((float)a.n * (float)SG_OUT);
    for (int c0 = 0; c0 < SG_OUT; c0 += 32) {
        float v[32];
        const int cnt = min(32, SG_OUT - c0);
        for (int j = 0; j < 32; ++j) {
            float d = 0.0f;
            if (live && j < cnt) {
                d = a.Y[(size_t)r * SG_OUT + c0 + j] - a.T[(size_t)src * SG_OUT + c0 + j];
                sse += (double)d * d;
            }
            v[j] = d * scale;
        }
        put_grad_row(bufG, bufGT, sdb, tid, c0, v, cnt, SG_OUT);
    }
    for (int o = 16; o; o >>= 1) sse += __shfl_xor_sync(0xffffffffu, sse, o);
    if ((tid & 31) == 0 && sse != 0.0) atomicAdd(a.loss, sse);
    const uint32_t tm = tbase;
    const uint32_t lane_tm = tm + ((uint32_t)(32 * warp) << 16);
    bool ok = true;
    for (int l = 3; l >= 0; --l) {
        const int n_out = l == 3 ? SG_OUT : SG_HID, n_in = l == 0 ? SG_IN : SG_HID;
        // H_l^T (the layer's input, rows of this tile) into bufXT
        const __nv_bfloat16* H = l == 0 ? a.H0 : l == 1 ? a.H1 : l == 2 ? a.H2 : a.H3;
        for (int i = 0; i < n_in; ++i) {
            const __nv_bfloat16 h = live ? H[(size_t)r * n_in + i] : __float2bfloat16_rn(0.0f);
            *reinterpret_cast<__nv_bfloat16*>(bufXT + coff(i, tid, SG_TILE)) = h;
        }
        if (l > 0) load_operand(bufW, a.w.WT[l], n_in, n_out);
        sg_sync();
        // bias gradient of this layer
        const int boff = l == 0 ? SG_OFF_B1 : l == 1 ? SG_OFF_B2 : l == 2 ? SG_OFF_B3 : SG_OFF_B4;
        if (tid < n_out) { atomicAdd(&a.grad[boff + tid], sdb[tid]); sdb[tid] = 0.0f; }
        if (tid == 0) {
            if (l == 3) gemm_issue(tm + 128, s2u(bufXT), s2u(bufGT), SG_TILE, SG_OUT, SG_TILE);   // dW^T
            else gemm_issue(tm + 128, s2u(bufGT), s2u(bufXT), SG_TILE, n_in, SG_TILE);            // dW
            if (l > 0) gemm_issue(tm, s2u(bufG), s2u(bufW), SG_TILE, n_in, n_out);              // dH
            umma_commit(&bar);
        }
        mma_wait(&bar, (uint32_t)((3 - l) & 1), (l == 3 && a.give_up_first) ? 0ull : a.mma_ns, ok);
        tc_after_sync();
        // weight gradient: TMEM row tid of D_dW
        const int woff = l == 0 ? SG_OFF_W1 : l == 1 ? SG_OFF_W2 : l == 2 ? SG_OFF_W3 : SG_OFF_W4;
        const int ncol = l == 3 ? SG_OUT : n_in;
        for (int c0 = 0; c0 < ncol; c0 += 32) {
            float v[32];
            tmem_ld32(lane_tm + 128u + (uint32_t)c0, v);
            for (int j = 0; j < 32 && c0 + j < ncol; ++j) {
                // l == 3: row = input i = tid, column = output o; else row = output o = tid, column = input i
                const int idx = l == 3 ? woff + (c0 + j) * SG_HID + tid : woff + tid * n_in + c0 + j;
                if (tid < (l == 3 ? SG_HID : n_out)) atomicAdd(&a.grad[idx], v[j]);
            }
        }
        if (l > 0) {
            // D_{l-1} = dH_l * gelu'(Z_l), written for the next layer
            __syncthreads();       // bufG / bufGT / sdb reads of this layer are done (MMA complete)
            const float* Z = l == 1 ? a.Z1 : l == 2 ? a.Z2 : a.Z3;
            for (int c0 = 0; c0 < SG_HID; c0 += 32) {
                float v[32];
                tmem_ld32(lane_tm + (uint32_t)c0, v);
                for (int j = 0; j < 32; ++j) v[j] = live ? v[j] * gelu_d(Z[(size_t)r * SG_HID + c0 + j]) : 0.0f;
                put_grad_row(bufG, bufGT, sdb, tid, c0, v, 32, SG_HID);
            }
        }
        sg_sync();
    }
    if (warp == 0) tmem_dealloc(tm, 256);
    if (!ok && tid == 0) atomicOr(a.err, SG_ERR_WAIT);
}

// ------------------------------------------------------------ optimiser
__global__ void k_sg_adam(float* p, float* m, float* v, float* g, float lr, float b1t, float b2t) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= SG_NPARAM) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi; v[i] = vi; g[i] = 0.0f;
    const float mh = mi / (1.0f - b1t), vh = vi / (1.0f - b2t);
    p[i] -= lr * mh / (sqrtf(vh) + eps);
}

__global__ void k_sg_convert(const float* p, __nv_bfloat16* W, __nv_bfloat16* WT) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= SG_WTOTAL) return;
    const int woff[4] = {0, SG_HID * SG_IN, SG_HID * SG_IN + SG_HID * SG_HID, SG_HID * SG_IN + 2 * SG_HID * SG_HID};
    int l = 3;
    while (l > 0 && i < woff[l]) --l;
    const int n_in = l == 0 ? SG_IN : SG_HID, n_out = l == 3 ? SG_OUT : SG_HID;
    const int e = i - woff[l], o = e / n_in, in = e - o * n_in;
    const int poff = l == 0 ? SG_OFF_W1 : l == 1 ? SG_OFF_W2 : l == 2 ? SG_OFF_W3 : SG_OFF_W4;
    const __nv_bfloat16 h = __float2bfloat16_rn(p[poff + e]);
    W[i] = h;
    WT[woff[l] + in * n_out + o] = h;
}

__global__ void k_sg_standardise(const float* in, float* out, uint64_t n, int dim, const float* mean,
                                 const float* inv_std) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= n * dim) return;
    const int k = (int)(i % dim);
    out[i] = (in[i] - mean[k]) * inv_std[k];
}

__global__ void k_sg_reduce(const float* Y, uint32_t n, const float* ymean, const float* ystd, const float* E,
                            float E0, double* acc) {
    __shared__ double s[SG_OUT + 1];
    for (int k = threadIdx.x; k <= SG_OUT; k += blockDim.x) s[k] = 0.0;
    __syncthreads();
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const double e = E ? (double)E[r] : (double)E0;
        for (int k = 0; k < SG_OUT; ++k)
            atomicAdd(&s[k], (double)(Y[(size_t)r * SG_OUT + k] * ystd[k] + ymean[k]) * e);
        atomicAdd(&s[SG_OUT], e);
    }
    __syncthreads();
    for (int k = threadIdx.x; k <= SG_OUT; k += blockDim.x) atomicAdd(&acc[k], s[k]);
}

// ------------------------------------------------------------ descriptors
// Per track, from its rad_buf entries in canonical order:
//   0..5   yields per 100 eV of OH, e-aq (codes 1 and 5), H, H3O+, OH-, H2 markers
//   6, 7   log10 E, log10 entries
//   8      log10 radius of gyration (nm)
//   9..24  histogram of log10 |x_i - x_{i-1}| between consecutive entries (16 bins, 0.01-100 nm)
//   25..40 the same for |x_i - x_{i-4}|
//   41..56 the same for |x_i - x_{i-16}|
//   57..62 species fractions of the same six classes
//   63     1
__device__ __forceinline__ int dbin(float d) {
    const float t = (log10f(fmaxf(d, 1e-6f)) + 2.0f) * 4.0f;
    return t < 0.0f ? 0 : t >= 15.0f ? 15 : (int)t;
}

__global__ void __launch_bounds__(128) k_descriptors(DescArgs a) {
    __shared__ float sh[4][64];
    const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
    float* h = sh[wl];
    for (uint32_t p = blockIdx.x * 4 + wl; p < a.nseg; p += gridDim.x * 4) {
        for (int k = lane; k < 64; k += 32) h[k] = 0.0f;
        __syncwarp();
        const unsigned long long s = a.seg_off[p], e = a.seg_off[p + 1];
        double sx = 0, sy = 0, sz = 0, s2 = 0;
        uint32_t cls[6] = {0, 0, 0, 0, 0, 0};
        for (unsigned long long i = s + lane; i < e; i += 32) {
            const float4 q = a.rad[i];
            const int code = (int)rintf(q.w) % 8;
            const int k = code == 0 ? 0 : (code == 1 || code == 5) ? 1 : code == 2 ? 2 : code == 3 ? 3
                        : code == 6 ? 4 : 5;
            cls[k]++;
            sx += q.x; sy += q.y; sz += q.z;
            s2 += (double)q.x * q.x + (double)q.y * q.y + (double)q.z * q.z;
#pragma unroll
            for (int t = 0; t < 3; ++t) {
                const unsigned long long L = t == 0 ? 1 : t == 1 ? 4 : 16;
                if (i >= s + L) {
                    const float4 o = a.rad[i - L];
                    const float dx = q.x - o.x, dy = q.y - o.y, dz = q.z - o.z;
                    atomicAdd(&h[9 + 16 * t + dbin(sqrtf(dx * dx + dy * dy + dz * dz))], 1.0f);
                }
            }
        }
        for (int o = 16; o; o >>= 1) {
            sx += __shfl_xor_sync(0xffffffffu, sx, o); sy += __shfl_xor_sync(0xffffffffu, sy, o);
            sz += __shfl_xor_sync(0xffffffffu, sz, o); s2 += __shfl_xor_sync(0xffffffffu, s2, o);
#pragma unroll
            for (int k = 0; k < 6; ++k) cls[k] += __shfl_xor_sync(0xffffffffu, cls[k], o);
        }
        __syncwarp();
        const uint32_t n = (uint32_t)(e - s);
        const float E = a.E ? a.E[p] : a.E0;
        float* out = a.out + (size_t)p * 64;
        if (lane == 0) {
            const float per100 = E > 0 ? E / 100.0f : 1.0f;
            for (int k = 0; k < 6; ++k) {
                out[k] = (float)cls[k] / per100;
                out[57 + k] = n ? (float)cls[k] / (float)n : 0.0f;
            }
            out[6] = log10f(fmaxf(E, 1.0f));
            out[7] = log10f((float)n + 1.0f);
            double rg2 = 0.0;
            if (n) {
                const double cx = sx / n, cy = sy / n, cz = sz / n;
                rg2 = s2 / n - (cx * cx + cy * cy + cz * cz);
            }
            out[8] = log10f((float)sqrt(fmax(rg2, 0.0)) + 0.01f);
            out[63] = 1.0f;
        }
        for (int t = 0; t < 3; ++t) {
            const uint32_t L = t == 0 ? 1 : t == 1 ? 4 : 16;
            const float norm = n > L ? 1.0f / (float)(n - L) : 0.0f;
            if (lane < 16) out[9 + 16 * t + lane] = h[9 + 16 * t + lane] * norm;
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------ launchers
static int sm_count() {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
}

cudaError_t launch_descriptors(const DescArgs& a, cudaStream_t s) {
    if (a.nseg == 0) return cudaSuccess;
    const uint32_t want = (a.nseg + 3) / 4, cap = (uint32_t)sm_count() * 8;
    const int blocks = (int)(want < cap ? want : cap);
    k_descriptors<<<blocks, 128, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_sg_forward(const SgFwdArgs& a, cudaStream_t s) {
    if (a.n == 0) return cudaSuccess;
    static DeviceOnce attr;
    cudaError_t e = attr.run([] {
        return cudaFuncSetAttribute(k_sg_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, 65536 + 1024);
    });
    if (e != cudaSuccess) return e;
    k_sg_fwd<<<(a.n + SG_TILE - 1) / SG_TILE, SG_TILE, 65536 + 1024, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_sg_backward(const SgBwdArgs& a, cudaStream_t s) {
    if (a.n == 0) return cudaSuccess;
    static DeviceOnce attr;
    cudaError_t e = attr.run([] {
        return cudaFuncSetAttribute(k_sg_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, 131072 + 1024);
    });
    if (e != cudaSuccess) return e;
    k_sg_bwd<<<(a.n + SG_TILE - 1) / SG_TILE, SG_TILE, 131072 + 1024, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_sg_adam(float* p, float* m, float* v, float* grad, float lr, float b1t, float b2t,
                           __nv_bfloat16* Wcat, __nv_bfloat16* WTcat, cudaStream_t s) {
    k_sg_adam<<<(SG_NPARAM + 255) / 256, 256, 0, s>>>(p, m, v, grad, lr, b1t, b2t);
    k_sg_convert<<<(SG_WTOTAL + 255) / 256, 256, 0, s>>>(p, Wcat, WTcat);
    return cudaGetLastError();
}

cudaError_t launch_sg_convert(const float* p, __nv_bfloat16* Wcat, __nv_bfloat16* WTcat, cudaStream_t s) {
    k_sg_convert<<<(SG_WTOTAL + 255) / 256, 256, 0, s>>>(p, Wcat, WTcat);
    return cudaGetLastError();
}

cudaError_t launch_sg_standardise(const float* in, float* out, uint64_t n, int dim, const float* mean,
                                  const float* inv_std, cudaStream_t s) {
    const uint64_t tot = n * (uint64_t)dim;
    if (!tot) return cudaSuccess;
    k_sg_standardise<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(in, out, n, dim, mean, inv_std);
    return cudaGetLastError();
}

cudaError_t launch_sg_reduce(const float* Y, uint32_t n, const float* ymean, const float* ystd, const float* E,
                             float E0, double* acc, cudaStream_t s) {
    { cudaError_t me_ = cudaMemsetAsync(acc, 0, (SG_OUT + 1) * sizeof(double), s); if (me_ != cudaSuccess) return me_; }
    const uint32_t nb = (n + 255) / 256 < 296u ? (n + 255) / 256 : 296u;
    if (n) k_sg_reduce<<<nb, 256, 0, s>>>(Y, n, ymean, ystd, E, E0, acc);
    return cudaGetLastError();
}

}  // namespace wg
