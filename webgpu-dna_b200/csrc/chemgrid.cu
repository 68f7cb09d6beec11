// chemgrid.cu -- the reference's 'gpu' chemistry backend
// (src/shaders/chemistry.wgsl:1-334, driven by src/chemistry/schedule.ts:33-247
// and measure.ts): radicals diffuse in fixed time steps, a spatial hash of
// 1.5 nm cells finds neighbours, and pairs within the reaction radius react
// with a contact probability, each thread claiming both radicals with
// compare-and-swap (so, as in the reference, which of several competing
// pairs reacts depends on thread timing).  The 7-stage schedule (133 steps of
// diffuse / clear / build / react, plus the counts at each checkpoint) is
// captured once into a CUDA graph and replayed with one launch.
//
// Random numbers: Philox4x32-10 with counter (radical, step, 0, 6) and the
// call's key; the f32 Gaussians use this build's own log / sincos
// (dmath.cuh), so the CPU restatement reproduces every displacement.
#include "chemgrid.cuh"
#include "dmath.cuh"

namespace wg {

constexpr uint32_t CG_HASH = CG_HASH_SIZE;       // 2^23 buckets
constexpr float CG_CELL = 1.5f;                  // nm

__device__ __forceinline__ uint32_t cg_hash(int ix, int iy, int iz) {
    const uint32_t h = (uint32_t)(ix * 73856093) ^ (uint32_t)(iy * 19349663) ^ (uint32_t)(iz * 83492791);
    return h % CG_HASH;
}

__device__ __forceinline__ float cg_sigma_react(int a, int b) {
    if (a > b) { int t = a; a = b; b = t; }
    if (a == 0 && b == 0) return 0.44f;
    if (a == 0 && b == 1) return 0.57f;
    if (a == 0 && b == 2) return 0.45f;
    if (a == 1 && b == 1) return 0.54f;
    if (a == 1 && b == 2) return 0.61f;
    if (a == 1 && b == 3) return 0.47f;
    if (a == 2 && b == 2) return 0.34f;
    return 0.0f;
}

__device__ __forceinline__ float cg_pcontact(int a, int b) {
    if (a > b) { int t = a; a = b; b = t; }
    if (a == 0 && b == 0) return 0.376f;
    if (a == 0 && b == 1) return 0.980f;
    if (a == 0 && b == 2) return 0.511f;
    if (a == 1 && b == 1) return 0.125f;
    if (a == 1 && b == 2) return 0.455f;
    if (a == 1 && b == 3) return 0.538f;
    if (a == 2 && b == 2) return 0.216f;
    return 0.0f;
}

// product class: 1 = H2O2, 2 = H2, 3 = the e-aq + H3O+ -> H conversion
__device__ __forceinline__ int cg_product(int a, int b) {
    if (a > b) { int t = a; a = b; b = t; }
    if (a == 0 && b == 0) return 1;
    if (a == 1 && b == 1) return 2;
    if (a == 1 && b == 2) return 2;
    if (a == 1 && b == 3) return 3;
    if (a == 2 && b == 2) return 2;
    return 0;
}

// Box-Muller pair from two uniforms (gauss2, chemistry.wgsl:24-30)
__device__ __forceinline__ float2 cg_gauss2(float u1, float u2) {
    u1 = fmaxf(u1, 1e-10f);
    const float r = sqrtf(-2.0f * logf_pos(u1));
    float s, c;
    sincosf_(6.28318530f * u2, &s, &c);
    return make_float2(r * c, r * s);
}

// sample_init + init_thermal (chemistry.wgsl:92-101, 286-334)
__global__ void k_cg_init(const float4* rad, uint32_t n, uint32_t k0, uint32_t k1, float4* pos, uint32_t* alive) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 r = rad[i];
    int kind = (int)(__float2uint_rn(r.w) % 8u);
    float4 p = make_float4(r.x, r.y, r.z, (float)kind);
    alive[i] = 1u;
    const u4 w = philox(i, 0xffffffffu, 0u, 6u, k0, k1);
    float sigma = 0.0f;
    bool disp = true;
    if (kind == 0) sigma = 0.462f;
    else if (kind == 1) sigma = 1.764f;
    else if (kind == 2) sigma = 1.309f;
    else if (kind == 3) sigma = u01f(w.w) < 0.5f ? 0.462f : 0.0f;
    else if (kind == 5) { kind = 1; sigma = 0.0f; }
    else disp = false;
    if (disp) {
        const float2 g01 = cg_gauss2(u01f(w.x), u01f(w.y));
        const u4 w2 = philox(i, 0xfffffffeu, 0u, 6u, k0, k1);
        const float2 g23 = cg_gauss2(u01f(w2.x), u01f(w2.y));
        p.x = p.x + sigma * g01.x;
        p.y = p.y + sigma * g01.y;
        p.z = p.z + sigma * g23.x;
        p.w = (float)kind;
    }
    pos[i] = p;
}

// diffuse (chemistry.wgsl:32-56)
__global__ void k_cg_diffuse(float4* pos, const uint32_t* alive, uint32_t n, const CgStep* st, uint32_t k0, uint32_t k1) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || alive[i] == 0u) return;
    float4 p = pos[i];
    const int kind = (int)rintf(p.w);
    float D;
    if (kind == 0) D = 2.2f;
    else if (kind == 1) D = 4.9f;
    else if (kind == 2) D = 7.0f;
    else if (kind == 3) D = 9.0f;
    else return;
    const float sigma = sqrtf(2.0f * D * st->dt);
    const u4 w = philox(i, st->step, 0u, 6u, k0, k1);
    const float2 g01 = cg_gauss2(u01f(w.x), u01f(w.y));
    const float2 g23 = cg_gauss2(u01f(w.z), u01f(w.w));
    p.x += sigma * g01.x;
    p.y += sigma * g01.y;
    p.z += sigma * g23.x;
    pos[i] = p;
}

__global__ void k_cg_clear(int* head) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < CG_HASH; i += gridDim.x * blockDim.x) head[i] = -1;
}

__device__ __forceinline__ int cg_cell(float x) { return (int)floorf(x / CG_CELL); }

// build_hash (chemistry.wgsl:111-122)
__global__ void k_cg_build(const float4* pos, const uint32_t* alive, uint32_t n, int* head, int* next) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (alive[i] == 0u) { next[i] = -1; return; }
    const float4 p = pos[i];
    const uint32_t h = cg_hash(cg_cell(p.x), cg_cell(p.y), cg_cell(p.z));
    next[i] = atomicExch(&head[h], (int)i);
}

// react (chemistry.wgsl:194-266): contact within the reaction radius, a
// contact-probability roll from the radical's step stream, claim both
// radicals with compare-and-swap
__global__ void k_cg_react(float4* pos, uint32_t* alive, uint32_t n, const int* head, const int* next,
                           const CgStep* st, uint32_t k0, uint32_t k1, uint32_t* prod) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || alive[i] == 0u) return;
    const float4 pi = pos[i];
    const int ki = (int)rintf(pi.w);
    if (ki < 0 || ki > 3) return;
    const int ix = cg_cell(pi.x), iy = cg_cell(pi.y), iz = cg_cell(pi.z);
    uint32_t draw = 0;
    u4 w = {0, 0, 0, 0};
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                int j = head[cg_hash(ix + dx, iy + dy, iz + dz)];
                for (uint32_t it = 0; it < 1024u && j >= 0; ++it) {
                    const uint32_t ju = (uint32_t)j;
                    const int jn = next[ju];
                    if (ju <= i || alive[ju] == 0u) { j = jn; continue; }
                    const float4 pj = pos[ju];
                    const int kj = (int)rintf(pj.w);
                    if (kj < 0 || kj > 3) { j = jn; continue; }
                    const float R = cg_sigma_react(ki, kj);
                    if (R <= 0.0f) { j = jn; continue; }
                    const float ddx = pi.x - pj.x, ddy = pi.y - pj.y, ddz = pi.z - pj.z;
                    if (ddx * ddx + ddy * ddy + ddz * ddz > R * R) { j = jn; continue; }
                    if ((draw & 3u) == 0u) w = philox(i, st->step, 1u + (draw >> 2), 6u, k0, k1);
                    const uint32_t word = (draw & 3u) == 0u ? w.x : (draw & 3u) == 1u ? w.y : (draw & 3u) == 2u ? w.z : w.w;
                    draw++;
                    if (u01f(word) >= cg_pcontact(ki, kj)) { j = jn; continue; }
                    if (atomicCAS(&alive[i], 1u, 0u) != 1u) return;
                    if (atomicCAS(&alive[ju], 1u, 0u) != 1u) { atomicExch(&alive[i], 1u); j = jn; continue; }
                    const int pr = cg_product(ki, kj);
                    if (pr == 1) atomicAdd(&prod[0], 1u);
                    else if (pr == 2) atomicAdd(&prod[1], 1u);
                    else if (pr == 3) {
                        const uint32_t e = ki == 1 ? i : ju;        // the e-aq becomes an H
                        float4 q = pos[e];
                        q.w = 2.0f;
                        pos[e] = q;
                        atomicExch(&alive[e], 1u);
                    }
                    return;
                }
            }
}

// count_alive (chemistry.wgsl:270-281) into checkpoint slot k: OH, e-aq, H
// alive, then the running H2O2 and H2 product counts
__global__ void k_cg_count(const float4* pos, const uint32_t* alive, uint32_t n, const uint32_t* prod,
                           uint32_t* out) {
    __shared__ uint32_t s[3];
    if (threadIdx.x < 3) s[threadIdx.x] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (alive[i] == 0u) continue;
        const int kind = (int)rintf(pos[i].w);
        if (kind >= 0 && kind <= 2) atomicAdd(&s[kind], 1u);
    }
    __syncthreads();
    if (threadIdx.x < 3 && s[threadIdx.x]) atomicAdd(&out[threadIdx.x], s[threadIdx.x]);
    if (blockIdx.x == 0 && threadIdx.x == 0) { out[3] = prod[0]; out[4] = prod[1]; }
}

__global__ void k_cg_set_step(CgStep* st, float dt, uint32_t step) { st->dt = dt; st->step = step; }

// The schedule of schedule.ts:38-46: [dt ns, steps]
static const float CG_DT[7] = {0.0001f, 0.001f, 0.005f, 0.05f, 0.5f, 3.0f, 30.0f};
static const int CG_NS[7] = {10, 9, 18, 18, 18, 30, 30};

cudaError_t cg_run(const CgArgs& a, cudaStream_t s, cudaGraphExec_t* cache, CgGraphKey* key) {
    const uint32_t n = a.n;
    const unsigned nb = (n + 255) / 256;
    cudaError_t e;
    k_cg_init<<<nb, 256, 0, s>>>(a.rad, n, a.k0, a.k1, a.pos, a.alive);
    { cudaError_t me_ = cudaMemsetAsync(a.counts, 0, 8 * 5 * sizeof(uint32_t), s); if (me_ != cudaSuccess) return me_; }
    { cudaError_t me_ = cudaMemsetAsync(a.prod, 0, 2 * sizeof(uint32_t), s); if (me_ != cudaSuccess) return me_; }
    k_cg_count<<<296, 256, 0, s>>>(a.pos, a.alive, n, a.prod, a.counts);
    // the schedule as one graph; rebuilt when the buffers or sizes change
    const CgGraphKey want{a.pos, a.alive, a.head, a.next, a.prod, a.counts, a.st, n, a.k0, a.k1};
    if (!*cache || memcmp(key, &want, sizeof want) != 0) {
        if (*cache) { cudaGraphExecDestroy(*cache); *cache = nullptr; }
        cudaStream_t cs;
        if ((e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking)) != cudaSuccess) return e;
        cudaGraph_t g;
        if ((e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) { cudaStreamDestroy(cs); return e; }
        uint32_t step = 0;
        for (int stage = 0; stage < 7; ++stage) {
            for (int k = 0; k < CG_NS[stage]; ++k) {
                k_cg_set_step<<<1, 1, 0, cs>>>(a.st, CG_DT[stage], ++step);
                k_cg_diffuse<<<nb, 256, 0, cs>>>(a.pos, a.alive, n, a.st, a.k0, a.k1);
                k_cg_clear<<<2048, 256, 0, cs>>>(a.head);
                k_cg_build<<<nb, 256, 0, cs>>>(a.pos, a.alive, n, a.head, a.next);
                k_cg_react<<<nb, 256, 0, cs>>>(a.pos, a.alive, n, a.head, a.next, a.st, a.k0, a.k1, a.prod);
            }
            k_cg_count<<<296, 256, 0, cs>>>(a.pos, a.alive, n, a.prod, a.counts + 5 * (stage + 1));
        }
        e = cudaStreamEndCapture(cs, &g);
        cudaStreamDestroy(cs);
        if (e != cudaSuccess) return e;
        e = cudaGraphInstantiate(cache, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) { *cache = nullptr; return e; }
        *key = want;
    }
    e = cudaGraphLaunch(*cache, s);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

}  // namespace wg
