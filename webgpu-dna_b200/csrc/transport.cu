// transport.cu -- electron track transport in liquid water (Phase A + B).
//
// Physics follows allaunthefox/webgpu-dna src/shaders/helpers.wgsl:15-186,
// primary.wgsl:41-663 and secondary.wgsl:17-450 (same statements, same f32
// evaluation order); the execution model is new:
//
// * One persistent kernel runs primaries and secondaries together.  Each warp
//   iteration advances every lane's electron by one step (the reference's
//   Phase A loop body for a primary, one Phase B dispatch for a secondary).
//   Lanes whose electron finished refill at once: first from the global
//   secondary queue, then from the primary pool, so warps stay full and the
//   reference's 2000 Phase B dispatches become per-secondary step caps.
// * Every particle owns a Philox4x32-10 stream: key = seed, counter =
//   (block, secondary index, primary id, 1).  Results do not depend on which
//   lane or SM runs a particle, or when.
// * rad_buf entries are staged per warp in shared memory and written out in
//   coalesced bursts with one global atomic per burst; each carries a 64-bit
//   key (pid << 34 | secondary index << 17 | sequence) from which
//   canonicalise() rebuilds a deterministic order.
// * Counters live in shared memory per block; per-lane f64 energy sums.
//
// Compiled with -fmad=false: the only fused multiply-adds are explicit ones.
#include "transport.cuh"
#include "dmath.cuh"

namespace wg {

constexpr int TB = 256;            // threads per block
constexpr int TW = TB / 32;        // warps per block
constexpr int STG = 192;           // staged rad entries per warp
constexpr int STG_FLUSH = 96;      // flushed at this level: + 32 lanes x at most 3 entries per step <= STG
constexpr int STASH = (int)TRANSPORT_STASH;   // secondaries a warp keeps in shared memory

__device__ __forceinline__ unsigned long long gtime() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}


__constant__ float c_SB[5] = {10.79f, 13.39f, 16.05f, 32.30f, 539.0f};
__constant__ float c_EX[5] = {8.22f, 10.00f, 11.24f, 12.61f, 13.77f};
__constant__ float c_DEA_E[14] = {0.0f, 4.2f, 4.3f, 5.8f, 6.0f, 6.2f, 6.4f, 7.0f, 7.5f, 7.7f,
                                  8.4f, 10.2f, 11.2f, 12.3f};
__constant__ float c_DEA_S[14] = {0.0f, 0.0f, 0.0f, 2.5e-5f, 2.8e-4f, 6.0e-4f, 6.7e-4f, 3.7e-4f,
                                  1.09e-4f, 7.0e-5f, 1.4e-4f, 2.0e-5f, 6.0e-5f, 0.0f};
constexpr float NWf = 33.4f;
constexpr float TWO_PI_F = 6.28318530f;
constexpr float PI_F = 3.14159265f;

// counters inside the block's shared block: [0..7] counters, [8..15] sec_stats, [16..23] dbg
enum { C_OH = 0, C_EAQ = 1, C_H = 2, C_H3O = 3, C_DNA = 4, C_H2 = 5,
       SS_CUT = 9, SS_BOUNDS = 10, SS_STEPS = 11, SS_TERT = 12,
       D_IONS = 16, D_EXC = 17, D_ESC = 18, D_PRIM = 19, D_WSUM = 20, D_DOSE = 21 };

struct Particle {
    float px, py, pz, E, dx, dy, dz;
    uint32_t pid, sub, seq, it, nsec;
    uint32_t blk, ri, b0, b1, b2, b3;
    float tpath, ppath, maxr, sx, sy, sz;
    uint32_t nion, nexc;
    bool prim, active;
};

struct Blk {
    const float* T;       // tables in shared memory
    float4* srad;         // this warp's rad_buf staging
    unsigned long long* skey;
    int* sn;
    uint32_t* cnt;        // block counters
    StashRec* stash;      // this warp's secondaries
    int* stn;
};

// One out-of-line copy each of the step's f32 log, exp, pow and sincos: the
// kernel is bound by instruction fetch, and a call is cheaper than another
// inlined copy of the function at every call site.
__device__ __noinline__ float logf_nc(float x) { return logf_pos(x); }
__device__ __noinline__ float expf_nc(float x) { return expf_(x); }
__device__ __noinline__ float powf_nc(float x, float y) { return powf_(x, y); }
__device__ __noinline__ float2 sincosf_nc(float x) { float s, c; sincosf_(x, &s, &c); return make_float2(s, c); }

// Out-of-line Philox block for the transport stream: the generator is drawn
// from many call sites, and one shared copy keeps the kernel's code small
// enough for the instruction cache.
__device__ __noinline__ u4 philox_transport(uint32_t blk, uint32_t sub, uint32_t pid, uint32_t k0, uint32_t k1) {
    return philox(blk, sub, pid, 1u, k0, k1);
}

__device__ __forceinline__ uint32_t rn(Particle& q, uint32_t k0, uint32_t k1) {
    if (q.ri == 4u) {
        u4 o = philox_transport(q.blk, q.sub, q.pid, k0, k1);
        q.blk++;
        q.b0 = o.x; q.b1 = o.y; q.b2 = o.z; q.b3 = o.w;
        q.ri = 0;
    }
    uint32_t v = q.ri == 0 ? q.b0 : q.ri == 1 ? q.b1 : q.ri == 2 ? q.b2 : q.b3;
    q.ri++;
    return v;
}
#define RF() u01f(rn(q, A.k0, A.k1))

__device__ __forceinline__ void put(const TArgs& A, Blk& b, Particle& q, float x, float y, float z, float code) {
    int s = atomicAdd(b.sn, 1);
    b.srad[s] = make_float4(x, y, z, code + __uint2float_rn(q.pid) * 8.0f);
    if (q.seq >= (1u << 17)) atomicOr(&A.st->err, DERR_KEY_RANGE);
    b.skey[s] = ((unsigned long long)(q.pid - A.pid_base) << 34) | ((unsigned long long)q.sub << 17) | q.seq;
    q.seq++;
}

// per-thread deposited energy and number of dose-grid atomics
struct Dep { double e; uint32_t n; };

// voxel of (px, py, pz) in the vc^3 dose grid over +-box, or ~0u outside (out of line: 9 call sites)
__device__ __noinline__ uint32_t dose_voxel(float px, float py, float pz, float box, uint32_t vc) {
    float vs = 2.0f * box / (float)vc;
    int ix = (int)floorf((px + box) / vs);
    int iy = (int)floorf((py + box) / vs);
    int iz = (int)floorf((pz + box) / vs);
    int n = (int)vc;
    if (ix < 0 || ix >= n || iy < 0 || iy >= n || iz < 0 || iz >= n) return ~0u;
    return (uint32_t)((iz * n + iy) * n + ix);
}

__device__ __forceinline__ void deposit(const TArgs& A, Dep& dep, float px, float py, float pz, float d) {
    if (d <= 0.0f) return;                                       // primary.wgsl:103
    dep.e += (double)d;
    uint32_t v = dose_voxel(px, py, pz, A.box, A.vc);
    if (v == ~0u) return;
    atomicAdd(&A.dose[v], (uint32_t)(d * 100.0f));
    dep.n++;
}

// dna_near (primary.wgsl:41-86), out of line (4 call sites)
__device__ __noinline__ uint32_t dna_near_nc(float px, float py, float pz, uint32_t N, float spacing, float x0,
                                             float rise, float r_bb);

__device__ __forceinline__ uint32_t dna_near(const TArgs& A, float px, float py, float pz) {
    if (A.dna_enable == 0u) return 0u;
    return dna_near_nc(px, py, pz, A.dna_grid_n, A.dna_spacing, A.dna_x0, A.dna_rise, A.dna_r_bb);
}

__device__ __noinline__ uint32_t dna_near_nc(float px, float py, float pz, uint32_t N, float spacing, float x0,
                                             float rise, float r_bb) {
    const float r_damage = 0.29f;
    float grid_off = -((float)(N - 1u) * spacing) * 0.5f;
    float inv_s = 1.0f / spacing;
    int fi = (int)rintf((py - grid_off) * inv_s);
    int fj = (int)rintf((pz - grid_off) * inv_s);
    if (fi < 0 || fi >= (int)N || fj < 0 || fj >= (int)N) return 0u;
    float fy = grid_off + (float)fi * spacing;
    float fz = grid_off + (float)fj * spacing;
    float y_rel = py - fy, z_rel = pz - fz;
    float r2 = y_rel * y_rel + z_rel * z_rel;
    float R_reach = r_bb + r_damage;
    if (r2 > R_reach * R_reach) return 0u;
    int bp_est = (int)rintf((px - x0) / rise);
    int b0 = bp_est - 1 > 0 ? bp_est - 1 : 0;
    int b1 = bp_est + 1;
    const float d_phase = (float)(2.0 * 3.14159265 / 10.5);
    for (int bb = b0; bb <= b1; ++bb) {
        float bx = x0 + (float)bb * rise;
        float phi = (float)bb * d_phase;
        float s0z, s0y;
        sincosf_(phi, &s0z, &s0y);
        s0y = r_bb * s0y; s0z = r_bb * s0z;
        float dx = px - bx;
        float dy0 = y_rel - s0y, dz0 = z_rel - s0z;
        if (dx * dx + dy0 * dy0 + dz0 * dz0 < r_damage * r_damage) return 1u;
        float s1z, s1y;
        sincosf_(phi + PI_F, &s1z, &s1y);
        s1y = r_bb * s1y; s1z = r_bb * s1z;
        float dy1 = y_rel - s1y, dz1 = z_rel - s1z;
        if (dx * dx + dy1 * dy1 + dz1 * dz1 < r_damage * r_damage) return 1u;
    }
    return 0u;
}

__device__ __forceinline__ float meesungnoen_sigma(float k) {   // primary.wgsl:90-98
    if (k <= 0.1f) return 0.0f;
    float r = -4.06217193e-08f;
    r = r * k + 3.06848412e-06f; r = r * k - 9.93217814e-05f; r = r * k + 1.80172797e-03f;
    r = r * k - 2.01135480e-02f; r = r * k + 1.42939448e-01f; r = r * k - 6.48348714e-01f;
    r = r * k + 1.85227848e+00f; r = r * k - 3.36450378e+00f; r = r * k + 4.37785068e+00f;
    r = r * k - 4.20557339e+00f; r = r * k + 3.81679083e+00f; r = r * k - 2.34069784e-01f;
    return fmaxf(r, 0.0f) * 0.6267f;
}

// Gaussian 3-D displacement, the mu1..mu4 pattern of primary.wgsl:216-220.
// Out of line (8 call sites); the particle's generator state travels by value.
struct G3 { float x, y, z; uint32_t blk, ri, b0, b1, b2, b3; };

__device__ __noinline__ G3 gauss3_nc(uint32_t blk, uint32_t ri, uint32_t b0, uint32_t b1, uint32_t b2, uint32_t b3,
                                     uint32_t sub, uint32_t pid, uint32_t k0, uint32_t k1, float sigma) {
    // four draws: words ri..3 of the current block, then (unless ri = 0) the
    // first ri words of the next one (all four of it when ri = 4)
    G3 g;
    u4 n = {b0, b1, b2, b3};
    if (ri != 0u) n = philox_transport(blk, sub, pid, k0, k1);
    const uint32_t w[8] = {b0, b1, b2, b3, n.x, n.y, n.z, n.w};
    float u[4];
#pragma unroll
    for (int d = 0; d < 4; ++d) {
        const uint32_t v = ri == 0u ? w[d] : ri == 1u ? w[d + 1] : ri == 2u ? w[d + 2] : ri == 3u ? w[d + 3] : w[d + 4];
        u[d] = u01f(v);
    }
    if (ri == 0u) { g.blk = blk; g.ri = 4u; g.b0 = b0; g.b1 = b1; g.b2 = b2; g.b3 = b3; }
    else { g.blk = blk + 1u; g.ri = ri; g.b0 = n.x; g.b1 = n.y; g.b2 = n.z; g.b3 = n.w; }
    float u1 = fmaxf(u[0], 1e-30f);
    float rr = sqrtf(-2.0f * logf_pos(u1)) * sigma;
    float sn, cs;
    sincosf_(TWO_PI_F * u[1], &sn, &cs);
    g.x = rr * cs; g.y = rr * sn;
    float u3 = fmaxf(u[2], 1e-30f);
    g.z = sqrtf(-2.0f * logf_pos(u3)) * sigma * cosf_(TWO_PI_F * u[3]);
    return g;
}

__device__ __forceinline__ float3 gauss3(const TArgs& A, Particle& q, float sigma) {
    G3 g = gauss3_nc(q.blk, q.ri, q.b0, q.b1, q.b2, q.b3, q.sub, q.pid, A.k0, A.k1, sigma);
    q.blk = g.blk; q.ri = g.ri; q.b0 = g.b0; q.b1 = g.b1; q.b2 = g.b2; q.b3 = g.b3;
    return make_float3(g.x, g.y, g.z);
}

// H2O+ + eaq -> H2Ovib dissociation channels (primary.wgsl:246-276)
__device__ __forceinline__ void h2ovib(const TArgs& A, Blk& b, Particle& q, float x, float y, float z) {
    float r_vd = RF();
    if (r_vd < 0.1365f) {
        atomicAdd(&b.cnt[C_OH], 2u); atomicAdd(&b.cnt[C_H2], 1u);
        put(A, b, q, x, y, z, 0.0f); put(A, b, q, x, y, z, 0.0f); put(A, b, q, x, y, z, 7.0f);
    } else if (r_vd < 0.494f) {
        atomicAdd(&b.cnt[C_OH], 1u); atomicAdd(&b.cnt[C_H], 1u);
        put(A, b, q, x, y, z, 0.0f); put(A, b, q, x, y, z, 2.0f);
    } else if (r_vd < 0.650f) {
        atomicAdd(&b.cnt[C_H], 2u);
        put(A, b, q, x, y, z, 2.0f); put(A, b, q, x, y, z, 2.0f);
    }
}

__device__ __forceinline__ void rotate(float& dx, float& dy, float& dz, float ct, float st, float cp, float sp) {
    if (fabsf(dz) > 0.99999f) {                                  // primary.wgsl:169-170
        float sw = (dz > 0.0f) ? 1.0f : -1.0f;
        dx = st * cp; dy = st * sp * sw; dz = ct * sw;
    } else {
        float qq = sqrtf(1.0f - dz * dz);
        float inv = 1.0f / qq;
        float nx = dx * ct + st * (dx * dz * cp - dy * sp) * inv;
        float ny = dy * ct + st * (dy * dz * cp + dx * sp) * inv;
        float nz = dz * ct - qq * st * cp;
        float len = sqrtf(nx * nx + ny * ny + nz * nz);
        dx = nx / len; dy = ny / len; dz = nz / len;
    }
}

// Born differential CDF: the reference scans breakpoints linearly
// (helpers.wgsl:98-105) for the last j in [0, N_WR-2] whose prefix is <= r.
// Every committed CDF row is non-decreasing, so the index is
// (number of breakpoints <= r) - 1: a guide table in shared memory (every 16th
// breakpoint) picks the 16-wide window, whose (CDF, energy) pairs are then
// fetched together with independent loads.
__device__ __forceinline__ float sample_W_sec(const TArgs& A, const float* T, float E, uint32_t shell, float r) {
    uint32_t lo = 0, hi = NWE_ - 1;                              // helpers.wgsl:88-96
    while (hi - lo > 1u) { uint32_t mid = (lo + hi) / 2u; if (T[S_XWE + mid] <= E) lo = mid; else hi = mid; }
    uint32_t iE = (fabsf(T[S_XWE + hi] - E) < fabsf(T[S_XWE + lo] - E)) ? hi : lo;
    const float* G = T + S_GUIDE + (shell * NWE_ + iE) * GUIDES;
    int M = 0;
#pragma unroll
    for (int m = 0; m < GUIDES; ++m) M += (G[m] <= r) ? 1 : 0;
    int base = 16 * (M - 1);
    const float2* row = A.tab.xcw + (size_t)(shell * NWE_ + iE) * NWR_;
    int cnt = 0;
#pragma unroll
    for (int k = 1; k <= 16; ++k) {
        int idx = base + k;
        if (idx <= NWR_ - 2) cnt += (__ldg(row + idx).x <= r) ? 1 : 0;
    }
    uint32_t jlo = (uint32_t)(base + cnt);
    uint32_t jhi = jlo + 1 < NWR_ - 1 ? jlo + 1 : NWR_ - 1;
    float2 a = __ldg(row + jlo), b = __ldg(row + jhi);
    float c0 = a.x, c1 = b.x, e0 = a.y, e1 = b.y;
    if (c1 <= c0) return e0;
    float f = fminf(fmaxf((r - c0) / (c1 - c0), 0.0f), 1.0f);
    return e0 + (e1 - e0) * f;
}

// Append n stash records to the global queue (one atomic for the batch); the
// consumer spins on the epoch flag written after the payload.  Records beyond
// the queue capacity are dropped and counted, as sec_dropped in the reference.
__device__ void push_global(const TArgs& A, const StashRec* r, int n, int lane_stride) {
    (void)lane_stride;
    unsigned long long base = atomicAdd(&A.st->sec_qtail.v, (uint32_t)n);
    for (int k = 0; k < n; ++k) {
        unsigned long long slot = base + k;
        if (slot >= A.max_sec) { atomicAdd(&A.st->sec_drop, 1u); continue; }
        SecRec* rec = A.secq + slot;
        rec->pe = make_float4(r[k].x, r[k].y, r[k].z, r[k].E);
        rec->dir = make_float4(r[k].dx, r[k].dy, r[k].dz, 0.0f);
        rec->meta.x = r[k].pid;
        rec->meta.y = r[k].sub;
        __threadfence();
        *(volatile uint32_t*)&rec->meta.z = A.pub_epoch;     // publish
    }
}

struct XS {
    float xi, xc, xl, svib, sdea, s_tot, t;
    int grid;        // -1 below the grid, 1 above, 0 inside (t valid)
    uint32_t vbin;
};

// Spurs of interact(): an ionisation whose e-aq thermalises nearby (code 5,
// displaced from the ionisation site), a primary's ionisation with a tracked
// secondary (separation estimated from the secondary's range, no e-aq entry),
// an autoionising excitation (code 1, e-aq displaced from the displaced
// mother site), and a secondary that thermalises below the cutoff (its e-aq
// alone, code 5, secondary.wgsl:100-124).  All share one code path so that a
// warp runs it once.
enum : int { SPUR_NONE = 0, SPUR_LOCAL = 1, SPUR_TRACKED = 2, SPUR_AUTO = 3, SPUR_THERM = 4 };

// the interaction after the move (primary.wgsl:180-649, secondary.wgsl:167-443).
// First each lane takes its branch (ionisation, excitation, vibration, DEA) up
// to the point where it needs a spur; then the lanes that need one run it
// together; then a primary that ionised with W_sec > cutoff emits its
// secondary.  Every lane still draws in the reference's statement order.
__device__ __forceinline__ void interact(const TArgs& A, Blk& b, Particle& q, Dep& dep, const XS& x, bool therm) {
    const float* T = b.T;
    float E = q.E;
    const float px = q.px, py = q.py, pz = q.pz;
    const bool prim = q.prim;
    int spur = SPUR_NONE;
    float W_sec = 0.0f, bind = 0.0f;
    float r_type = therm ? 0.0f : RF() * x.s_tot;
    if (therm) {
        spur = SPUR_THERM;                                       // the lane did not move this step
    } else if (r_type < x.xi && E > c_SB[0]) {
        float sf[5];
        if (x.grid < 0) { for (int k = 0; k < 5; ++k) sf[k] = T[S_XSF + k * XN_]; }
        else if (x.grid > 0) { for (int k = 0; k < 5; ++k) sf[k] = T[S_XSF + k * XN_ + XN_ - 1]; }
        else {
            uint32_t i = (uint32_t)fminf(fmaxf(floorf(x.t), 0.0f), (float)(XN_ - 2));
            float f = x.t - (float)i;
            for (int k = 0; k < 5; ++k) {
                const float* a = T + S_XSF + k * XN_;
                sf[k] = fmaxf(0.0f, a[i] + (a[i + 1] - a[i]) * f);
            }
        }
        float fsum = fmaxf(sf[0] + sf[1] + sf[2] + sf[3] + sf[4], 1e-12f);
        float r_sh = RF() * fsum;
        uint32_t shell;
        if (r_sh < sf[0]) { bind = c_SB[0]; shell = 0; }
        else if (r_sh < sf[0] + sf[1]) { bind = c_SB[1]; shell = 1; }
        else if (r_sh < sf[0] + sf[1] + sf[2]) { bind = c_SB[2]; shell = 2; }
        else if (r_sh < sf[0] + sf[1] + sf[2] + sf[3]) { bind = c_SB[3]; shell = 3; }
        else { bind = c_SB[4]; shell = 4; }
        if (E > bind) {
            float r_w = RF();
            float Wmax = (E + bind) * 0.5f;
            float W = sample_W_sec(A, T, E, shell, r_w);
            W = fminf(fmaxf(W, bind), Wmax);
            W_sec = fmaxf(W - bind, 0.0f);
            E -= W;
            if (prim) {
                q.nion++;
                atomicAdd(&b.cnt[D_WSUM], (uint32_t)(W * 10.0f));
                deposit(A, dep, px, py, pz, bind);
                if (W_sec <= A.ce) deposit(A, dep, px, py, pz, W_sec);
            } else {                                             // secondary.wgsl:192-255
                atomicAdd(&b.cnt[SS_TERT], 1u);
                deposit(A, dep, px, py, pz, W);
            }
            if (dna_near(A, px, py, pz) == 1u) atomicAdd(&b.cnt[C_DNA], 1u);
            spur = (!prim || W_sec <= A.ce) ? SPUR_LOCAL : SPUR_TRACKED;
        }
    } else if (r_type < x.xi + x.xc) {
        float ef[5];
        if (x.grid < 0) { for (int k = 0; k < 5; ++k) ef[k] = T[S_XEF + k * XN_]; }
        else if (x.grid > 0) { for (int k = 0; k < 5; ++k) ef[k] = T[S_XEF + k * XN_ + 85]; }
        else {
            uint32_t i = (uint32_t)fminf(fmaxf(floorf(x.t), 0.0f), (float)(XN_ - 2));
            if (i > 85u) i = 85u;
            float f = (i == 85u) ? 0.0f : x.t - (float)i;
            uint32_t j = i + 1 < 85u ? i + 1 : 85u;
            for (int k = 0; k < 5; ++k) {
                const float* a = T + S_XEF + k * XN_;
                ef[k] = fmaxf(0.0f, a[i] + (a[j] - a[i]) * f);
            }
        }
        float efsum = fmaxf(ef[0] + ef[1] + ef[2] + ef[3] + ef[4], 1e-12f);
        float r_ex = RF() * efsum;
        float exc_E; uint32_t lvl;
        if (r_ex < ef[0]) { exc_E = c_EX[0]; lvl = 0; }
        else if (r_ex < ef[0] + ef[1]) { exc_E = c_EX[1]; lvl = 1; }
        else if (r_ex < ef[0] + ef[1] + ef[2]) { exc_E = c_EX[2]; lvl = 2; }
        else if (r_ex < ef[0] + ef[1] + ef[2] + ef[3]) { exc_E = c_EX[3]; lvl = 3; }
        else { exc_E = c_EX[4]; lvl = 4; }
        float d = fminf(exc_E, E);
        E -= d;
        deposit(A, dep, px, py, pz, d);
        if (prim) q.nexc++;
        float r_ch = RF();
        if (lvl == 0u) {
            if (r_ch < 0.65f) {
                atomicAdd(&b.cnt[C_OH], 1u); atomicAdd(&b.cnt[C_H], 1u);
                put(A, b, q, px, py, pz, 0.0f); put(A, b, q, px, py, pz, 2.0f);
            }
        } else if (lvl == 1u) {
            if (r_ch < 0.175f) {
            } else if (r_ch < 0.2075f) {
                atomicAdd(&b.cnt[C_OH], 2u); atomicAdd(&b.cnt[C_H2], 1u);
                put(A, b, q, px, py, pz, 0.0f); put(A, b, q, px, py, pz, 0.0f); put(A, b, q, px, py, pz, 7.0f);
            } else if (r_ch < 0.7075f) {
                spur = SPUR_AUTO;                                // primary.wgsl:473-536
            } else if (r_ch < 0.961f) {
                atomicAdd(&b.cnt[C_OH], 1u); atomicAdd(&b.cnt[C_H], 1u);
                put(A, b, q, px, py, pz, 0.0f); put(A, b, q, px, py, pz, 2.0f);
            } else {
                atomicAdd(&b.cnt[C_H], 2u);
                put(A, b, q, px, py, pz, 2.0f); put(A, b, q, px, py, pz, 2.0f);
            }
        } else {
            if (r_ch < 0.50f) spur = SPUR_AUTO;                  // primary.wgsl:560-619
        }
        if (dna_near(A, px, py, pz) == 1u) atomicAdd(&b.cnt[C_DNA], 1u);
    } else if (r_type < x.xi + x.xc + x.svib) {
        // sample_vib_mode (helpers.wgsl:148-170) with the bin found by fly()
        float r = RF();
        uint32_t base = x.vbin * 9u;
        float cumsum = 0.0f, cs[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            float frac = (T[S_VIB + k] > E) ? 0.0f : T[S_XVMF + base + k];
            cumsum = cumsum + frac;
            cs[k] = cumsum;
        }
        uint32_t mode = 8u;
        if (cumsum <= 0.0f) mode = 0u;
        else {
            float thr = r * cumsum;
#pragma unroll
            for (int k = 8; k >= 0; --k) if (thr < cs[k]) mode = (uint32_t)k;
        }
        float d = fminf(T[S_VIB + mode], E);
        E -= d;
        deposit(A, dep, px, py, pz, d);
    } else if (r_type < x.xi + x.xc + x.svib + x.sdea) {
        deposit(A, dep, px, py, pz, E);                          // Melton DEA
        atomicAdd(&b.cnt[C_OH], 1u); atomicAdd(&b.cnt[C_H2], 1u);
        put(A, b, q, px, py, pz, 0.0f); put(A, b, q, px, py, pz, 6.0f); put(A, b, q, px, py, pz, 7.0f);
        E = 0.0f;
    }
    if (spur != SPUR_NONE) {
        // mother (H2O+) displacement, then e-aq displacement and Onsager
        // recombination (p = 1 - exp(-0.711 / r)) or the tracked-secondary
        // estimate r = 0.04 W^1.3 + meesungnoen(min(W, 7.4)), then the H2Ovib
        // channels or the OH + [e-aq] + H3O+ entries (primary.wgsl:216-353)
        float mpx = px, mpy = py, mpz = pz;
        if (spur != SPUR_THERM) {
            const float3 m = gauss3(A, q, 1.1547005f);
            mpx = px + m.x; mpy = py + m.y; mpz = pz + m.z;
        }
        float epx = px, epy = py, epz = pz, p_recomb = 0.0f;
        if (spur != SPUR_TRACKED) {
            const bool au = spur == SPUR_AUTO;
            if (au) { epx = mpx; epy = mpy; epz = mpz; }
            const float eaq_s = meesungnoen_sigma(au ? 1.7f : spur == SPUR_THERM ? E : W_sec);
            if (eaq_s > 0.0f) {
                const float3 g = gauss3(A, q, eaq_s);
                epx = epx + g.x; epy = epy + g.y; epz = epz + g.z;
            }
            const float rdx = epx - mpx, rdy = epy - mpy, rdz = epz - mpz;
            const float r_sep = fmaxf(sqrtf(rdx * rdx + rdy * rdy + rdz * rdz), 1e-6f);
            p_recomb = 1.0f - expf_nc(-0.711f / r_sep);
        } else {
            const float r_track = 0.04f * powf_nc(W_sec, 1.3f);
            const float r_tail = meesungnoen_sigma(fminf(W_sec, 7.4f));
            const float r_sep_est = fmaxf(r_track + r_tail, 1e-3f);
            p_recomb = 1.0f - expf_nc(-0.711f / r_sep_est);
        }
        if (spur == SPUR_THERM) {
            put(A, b, q, epx, epy, epz, 5.0f);
        } else if (RF() < p_recomb) {
            h2ovib(A, b, q, mpx, mpy, mpz);
        } else {
            atomicAdd(&b.cnt[C_OH], 1u); atomicAdd(&b.cnt[C_H3O], 1u);
            put(A, b, q, mpx, mpy, mpz, 0.0f);
            if (spur != SPUR_TRACKED) {
                atomicAdd(&b.cnt[C_EAQ], 1u);
                put(A, b, q, epx, epy, epz, spur == SPUR_AUTO ? 1.0f : 5.0f);
            }
            put(A, b, q, mpx, mpy, mpz, 3.0f);
        }
    }
    if (spur == SPUR_TRACKED) {                                  // primary.wgsl:362-413
        // every emission takes a sec_buf index (counters[6]); at or beyond
        // max_sec the secondary is dropped together with its angle draws and
        // the primary's momentum update (:364)
        const uint32_t sec_idx = atomicAdd(&A.st->sec_tail.v, 1u);
        if (sec_idx < A.max_sec) {
            q.nsec++;
            float E_before = E + bind + W_sec;
            float cos_s;
            if (W_sec < 50.0f) {
                cos_s = 2.0f * RF() - 1.0f;
            } else if (W_sec <= 200.0f) {
                if (RF() <= 0.1f) cos_s = 2.0f * RF() - 1.0f;
                else cos_s = RF() * 0.70710678f;
            } else {
                float sin2 = fminf(fmaxf((1.0f - W_sec / E_before) / (1.0f + W_sec / 1022000.0f), 0.0f), 1.0f);
                cos_s = sqrtf(fmaxf(0.0f, 1.0f - sin2));
            }
            float sin_s = sqrtf(fmaxf(0.0f, 1.0f - cos_s * cos_s));
            float sps, cps;
            const float2 sc = sincosf_nc(TWO_PI_F * RF());
            sps = sc.x; cps = sc.y;
            float sdx = q.dx, sdy = q.dy, sdz = q.dz;
            rotate(sdx, sdy, sdz, cos_s, sin_s, cps, sps);
            float p_inc = sqrtf(E_before), p_sec = sqrtf(W_sec);
            float pfx = p_inc * q.dx - p_sec * sdx;
            float pfy = p_inc * q.dy - p_sec * sdy;
            float pfz = p_inc * q.dz - p_sec * sdz;
            float pfl = sqrtf(pfx * pfx + pfy * pfy + pfz * pfz);
            if (pfl > 1e-10f) { q.dx = pfx / pfl; q.dy = pfy / pfl; q.dz = pfz / pfl; }
            if (q.nsec >= (1u << 17)) atomicOr(&A.st->err, DERR_KEY_RANGE);
            StashRec r{px, py, pz, W_sec, sdx, sdy, sdz, q.pid, q.nsec};
            int slot = A.stash_spill ? atomicAdd(b.stn, 1) : STASH;
            if (slot < STASH) b.stash[slot] = r;
            else push_global(A, &r, 1, 0);
        }
    }
    q.E = E;
}

// Cross sections, free flight and elastic deflection (primary.wgsl:155-172)
__device__ __forceinline__ bool fly(const TArgs& A, Blk& b, Particle& q, XS& x, float& dist) {
    const float* T = b.T;
    float E = q.E;
    float lE = logf_nc(E);
    if (E <= T[S_XE]) { x.grid = -1; x.xi = 0.0f; x.xc = 0.0f; x.xl = T[S_XL]; x.t = 0.0f; }
    else if (E >= T[S_XE + XN_ - 1]) {
        x.grid = 1; x.xi = T[S_XI + XN_ - 1]; x.xc = T[S_XC + XN_ - 1]; x.xl = T[S_XL + XN_ - 1]; x.t = 0.0f;
    } else {
        x.grid = 0;
        x.t = (lE - A.tab.log_xe0) * A.tab.inv_log_xe_step;
        uint32_t i = (uint32_t)fminf(fmaxf(floorf(x.t), 0.0f), (float)(XN_ - 2));
        float f = x.t - (float)i;
        x.xi = fmaxf(0.0f, T[S_XI + i] + (T[S_XI + i + 1] - T[S_XI + i]) * f);
        x.xc = fmaxf(0.0f, T[S_XC + i] + (T[S_XC + i + 1] - T[S_XC + i]) * f);
        x.xl = fmaxf(0.0f, T[S_XL + i] + (T[S_XL + i + 1] - T[S_XL + i]) * f);
    }
    x.svib = 0.0f;
    x.vbin = 0;
    if (E >= 2.0f && E < 100.0f) {                               // xs_vib_total
        uint32_t lo = 0, hi = NVIB_ - 1;
        while (hi - lo > 1u) { uint32_t mid = (lo + hi) >> 1; if (T[S_XVE + mid] <= E) lo = mid; else hi = mid; }
        x.vbin = lo;
        float f = (E - T[S_XVE + lo]) / (T[S_XVE + lo + 1] - T[S_XVE + lo]);
        x.svib = fmaxf(0.0f, T[S_XVS + lo] + (T[S_XVS + lo + 1] - T[S_XVS + lo]) * f);
    }
    x.sdea = 0.0f;
    if (E >= 4.0f && E <= 13.0f) {                               // xs_dea
        // rolled: thirteen unrolled copies cost more in instruction fetch than the loop
#pragma unroll 1
        for (int i = 0; i < 13; ++i) {
            if (E >= c_DEA_E[i] && E < c_DEA_E[i + 1]) {
                float f = (E - c_DEA_E[i]) / (c_DEA_E[i + 1] - c_DEA_E[i]);
                x.sdea = fmaxf(0.0f, c_DEA_S[i] + (c_DEA_S[i + 1] - c_DEA_S[i]) * f);
                break;
            }
        }
    }
    x.s_tot = x.xi + x.xc + x.xl + x.svib + x.sdea;
    if (x.s_tot <= 0.0f) return false;
    float lambda = 1.0f / (NWf * x.s_tot);
    dist = -logf_nc(fmaxf(RF(), 1e-10f)) * lambda;
    // xs_el_cos (helpers.wgsl:66-82)
    float r = RF();
    float rr = fminf(fmaxf(r, 0.0f), 1.0f);
    float jf = rr * (float)(NAC_ - 1);
    uint32_t jlo = (uint32_t)floorf(jf);
    uint32_t jhi = jlo + 1 < NAC_ - 1 ? jlo + 1 : NAC_ - 1;
    float fj = jf - (float)jlo;
    float lEa = (E >= T[S_XAE]) ? lE : logf_nc(T[S_XAE]);
    float tE = (lEa - A.tab.log_xae0) * A.tab.inv_log_xae_step;
    uint32_t iE = (uint32_t)fminf(fmaxf(floorf(tE), 0.0f), (float)(NAE_ - 2));
    float fE = fminf(fmaxf(tE - (float)iE, 0.0f), 1.0f);
    const float* a0 = T + S_XAC + iE * NAC_;
    const float* a1 = a0 + NAC_;
    float cE0 = a0[jlo] + (a0[jhi] - a0[jlo]) * fj;
    float cE1 = a1[jlo] + (a1[jhi] - a1[jlo]) * fj;
    float cos_el = fminf(fmaxf(cE0 + (cE1 - cE0) * fE, -1.0f), 1.0f);
    float sin_el = sqrtf(fmaxf(0.0f, 1.0f - cos_el * cos_el));
    const float2 sc = sincosf_nc(TWO_PI_F * RF());
    const float sp = sc.x, cp = sc.y;
    rotate(q.dx, q.dy, q.dz, cos_el, sin_el, cp, sp);
    q.px += q.dx * dist; q.py += q.dy * dist; q.pz += q.dz * dist;
    return true;
}

__device__ __forceinline__ void start_primary(const TArgs& A, Particle& q, uint32_t idx) {
    q.pid = A.pid_base + idx; q.sub = 0; q.seq = 0; q.it = 0; q.nsec = 0;
    q.blk = 0; q.ri = 4;
    q.prim = true; q.active = true;
    q.E = A.E_prim ? A.E_prim[idx] : A.be;
    q.px = 0.0f; q.py = 0.0f; q.pz = 0.0f;
    float sh = A.start_half;
    if (sh > 0.0f) {
        q.px = (RF() * 2.0f - 1.0f) * sh;
        q.py = (RF() * 2.0f - 1.0f) * sh;
        q.pz = (RF() * 2.0f - 1.0f) * sh;
    }
    q.sx = q.px; q.sy = q.py; q.sz = q.pz;
    float u1 = fmaxf(RF(), 1e-10f);
    float u2 = RF();
    float cos_i = 1.0f - 2.0f * u1;
    float sin_i = sqrtf(fmaxf(0.0f, 1.0f - cos_i * cos_i));
    float spi, cpi;
    sincosf_(TWO_PI_F * u2, &spi, &cpi);
    q.dx = sin_i * cpi; q.dy = sin_i * spi; q.dz = cos_i;
    q.tpath = 0.0f; q.ppath = 0.0f; q.maxr = 0.0f; q.nion = 0; q.nexc = 0;
}

__device__ __forceinline__ void finish_primary(const TArgs& A, Blk& b, Particle& q, Dep& dep, uint32_t esc) {
    if (esc == 0u && q.E > 0.0f) deposit(A, dep, q.px, q.py, q.pz, q.E);
    float4* r = reinterpret_cast<float4*>(A.results + 8ull * (q.pid - A.pid_base));
    r[0] = make_float4(q.tpath, q.ppath, q.E, __uint_as_float(q.nion));
    r[1] = make_float4(__uint_as_float(q.nexc), __uint_as_float(esc), q.maxr, 0.0f);
    atomicAdd(&b.cnt[D_IONS], q.nion); atomicAdd(&b.cnt[D_EXC], q.nexc);
    atomicAdd(&b.cnt[D_ESC], esc); atomicAdd(&b.cnt[D_PRIM], 1u);
    q.active = false;
}

// one warp-iteration of a lane's electron.  Primaries and secondaries share
// one fly + interact call site, so a warp holding both kinds runs the step
// code once instead of once per kind; the lanes of `act` (those that entered)
// meet again before the interaction, so its branches run once per warp step.
__device__ __forceinline__ void lane_step(const TArgs& A, Blk& b, Particle& q, Dep& dep,
                                          unsigned long long& nsteps, unsigned act) {
    const float box = A.box;
    const bool prim = q.prim;
    const bool out = fabsf(q.px) >= box || fabsf(q.py) >= box || fabsf(q.pz) >= box;
    bool go = true, therm = false;
    if (prim) {
        if (q.it >= A.ms || q.E < A.ce) { finish_primary(A, b, q, dep, 0u); go = false; }
        else if (out) { finish_primary(A, b, q, dep, 1u); go = false; }
    } else {
        if (q.it >= A.sec_steps) { q.active = false; go = false; }
        else if (q.E < A.ce) {                                   // secondary.wgsl:100-124
            // thermalised: its e-aq is placed in interact()'s spur block
            deposit(A, dep, q.px, q.py, q.pz, q.E);
            atomicAdd(&b.cnt[C_EAQ], 1u);
            atomicAdd(&b.cnt[SS_CUT], 1u);
            therm = true;
            go = false;
        } else if (out) {
            atomicAdd(&b.cnt[SS_BOUNDS], 1u);
            q.active = false;
            go = false;
        }
    }
    XS x;
    if (go) {
        const bool productive = q.E > 12.0f;
        float dist;
        if (!fly(A, b, q, x, dist)) {
            if (prim) finish_primary(A, b, q, dep, 0u);
            else q.active = false;
            go = false;
        } else {
            nsteps++;
            if (prim) {
                q.tpath += dist;
                if (productive) q.ppath += dist;
                float rdx = q.px - q.sx, rdy = q.py - q.sy, rdz = q.pz - q.sz;
                float r = sqrtf(rdx * rdx + rdy * rdy + rdz * rdz);
                if (r > q.maxr) q.maxr = r;
                if (fabsf(q.px) >= box || fabsf(q.py) >= box || fabsf(q.pz) >= box) { finish_primary(A, b, q, dep, 1u); go = false; }
            } else {
                atomicAdd(&b.cnt[SS_STEPS], 1u);
            }
        }
    }
    __syncwarp(act);
    if (go || therm) {
        interact(A, b, q, dep, x, therm);
        if (go) q.it++;
        else q.active = false;
    }
}

__device__ __forceinline__ void flush_staging(const TArgs& A, Blk& b, int lane) {
    __syncwarp();
    int n = *b.sn;
    if (n == 0) return;
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(&A.st->rad_next.v, (unsigned long long)n);
    base = __shfl_sync(0xffffffffu, base, 0);
    int ndrop = 0;
    for (int i = lane; i < n; i += 32) {
        unsigned long long slot = base + (unsigned long long)i;
        if (slot < A.max_rad) { A.rad[slot] = b.srad[i]; A.key[slot] = b.skey[i]; }
        else ndrop++;
    }
    if (ndrop) atomicAdd(&A.st->rad_drop, (unsigned long long)ndrop);
    __syncwarp();
    if (lane == 0) *b.sn = 0;
    __syncwarp();
}

__device__ __forceinline__ void load_secondary(Particle& q, const StashRec& r) {
    q.px = r.x; q.py = r.y; q.pz = r.z; q.E = r.E;
    q.dx = r.dx; q.dy = r.dy; q.dz = r.dz;
    q.pid = r.pid; q.sub = r.sub; q.seq = 0; q.it = 0; q.nsec = 0;
    q.blk = 0; q.ri = 4; q.prim = false; q.active = true;
}

// 2 CTAs per SM: 3 (80 registers, less staging) measured 15 % slower
__global__ void __launch_bounds__(TB, 2) k_transport(TArgs A) {
    extern __shared__ __align__(16) unsigned char smem[];
    float* T = reinterpret_cast<float*>(smem);
    float4* stg_rad = reinterpret_cast<float4*>(smem + S_TOTAL_PAD * 4);
    unsigned long long* stg_key = reinterpret_cast<unsigned long long*>(stg_rad + TW * STG);
    StashRec* stash = reinterpret_cast<StashRec*>(stg_key + TW * STG);
    int* stg_n = reinterpret_cast<int*>(stash + TW * STASH);
    int* stn = stg_n + TW;
    uint32_t* cnt = reinterpret_cast<uint32_t*>(stn + TW);
    for (int i = threadIdx.x; i < S_TOTAL; i += TB) T[i] = A.tab.small[i];
    if (threadIdx.x < TW) { stg_n[threadIdx.x] = 0; stn[threadIdx.x] = 0; }
    if (threadIdx.x < 24) cnt[threadIdx.x] = 0;
    __syncthreads();

    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    Blk b{T, stg_rad + w * STG, stg_key + w * STG, stg_n + w, cnt, stash + w * STASH, stn + w};
    DevState* S = A.st;
    Particle q;
    q.active = false;
    Dep dep{0.0, 0u};
    unsigned long long nsteps = 0;
    bool busy = false;
    unsigned sleep_ns = 64;
    unsigned long long idle_since = 0;

    for (uint32_t it = 0;; ++it) {
        unsigned need = __ballot_sync(0xffffffffu, !q.active);
        // 1) this warp's stash (LIFO)
        if (need) {
            int sn = *(volatile int*)b.stn;
            if (sn > 0) {
                uint32_t take = min((uint32_t)__popc(need), (uint32_t)sn);
                uint32_t rank = __popc(need & lt);
                if (!q.active && rank < take) load_secondary(q, b.stash[sn - 1 - rank]);
                __syncwarp();
                if (lane == 0) *b.stn = sn - (int)take;
                __syncwarp();
                need = __ballot_sync(0xffffffffu, !q.active);
            }
        }
        const bool idle_warp = need == 0xffffffffu;
        const bool poll = idle_warp || (it & A.poll_mask) == 0u;
        // 2) the global queue
        if (need && poll) {
            uint32_t base = 0, got = 0;
            if (lane == 0) {
                uint32_t lim = min(*(volatile uint32_t*)&S->sec_qtail.v, A.max_sec);
                uint32_t h = *(volatile uint32_t*)&S->sec_head.v;
                uint32_t k = __popc(need);
                while (h < lim) {
                    uint32_t take = min(k, lim - h);
                    uint32_t old = atomicCAS(&S->sec_head.v, h, h + take);
                    if (old == h) { base = h; got = take; break; }
                    h = old;
                }
            }
            base = __shfl_sync(0xffffffffu, base, 0);
            got = __shfl_sync(0xffffffffu, got, 0);
            uint32_t rank = __popc(need & lt);
            if (!q.active && rank < got) {
                const SecRec* rec = A.secq + base + rank;
                unsigned long long t0 = gtime();
                bool ok = true;
                // bounded wait for the record's publication; once one wait has
                // run out the run is failed and no lane waits again
                while (*(volatile const uint32_t*)&rec->meta.z != A.epoch) {
                    if ((*(volatile uint32_t*)&S->err & DERR_QUEUE_WAIT) || gtime() - t0 > A.ready_ns) {
                        atomicOr(&S->err, DERR_QUEUE_WAIT);
                        ok = false;
                        break;
                    }
                    __nanosleep(64);
                }
                __threadfence();
                if (ok) {
                    float4 pe = __ldcg(&rec->pe);
                    float4 dr = __ldcg(&rec->dir);
                    uint4 mt = __ldcg(&rec->meta);
                    StashRec r{pe.x, pe.y, pe.z, pe.w, dr.x, dr.y, dr.z, mt.x, mt.y};
                    load_secondary(q, r);
                }
            }
            need = __ballot_sync(0xffffffffu, !q.active);
        }
        // 3) new primaries
        if (need && poll && *(volatile uint32_t*)&S->prim_next.v < A.np) {
            uint32_t pb = 0, pg = 0;
            if (lane == 0) {
                uint32_t take = min((uint32_t)__popc(need), A.prim_take);
                uint32_t old = atomicAdd(&S->prim_next.v, take);
                if (old < A.np) { pg = min(take, A.np - old); pb = old; }
            }
            pb = __shfl_sync(0xffffffffu, pb, 0);
            pg = __shfl_sync(0xffffffffu, pg, 0);
            uint32_t r2 = __popc(need & lt);
            if (!q.active && r2 < pg) start_primary(A, q, pb + r2);
        }
        unsigned act = __ballot_sync(0xffffffffu, q.active);
        if (act && !busy) { busy = true; if (lane == 0) atomicAdd(&S->busy.v, 1u); }
        if (!act) {
            // no lanes and an empty stash: idle
            if (busy) { busy = false; if (lane == 0) atomicSub(&S->busy.v, 1u); idle_since = gtime(); }
            int done = 0;
            if (lane == 0) {
                uint32_t lim = min(*(volatile uint32_t*)&S->sec_qtail.v, A.max_sec);
                done = *(volatile uint32_t*)&S->prim_next.v >= A.np &&
                       *(volatile uint32_t*)&S->sec_head.v >= lim && *(volatile uint32_t*)&S->busy.v == 0u;
            }
            done = __shfl_sync(0xffffffffu, done, 0);
            if (done) break;
            if (idle_since == 0) idle_since = gtime();
            if (gtime() - idle_since > A.idle_ns) { if (lane == 0) atomicOr(&S->err, DERR_IDLE_WAIT); break; }
            __nanosleep(sleep_ns);
            sleep_ns = min(sleep_ns * 2, 8192u);
            continue;
        }
        sleep_ns = 64;
        idle_since = 0;
        if (q.active) lane_step(A, b, q, dep, nsteps, act);
        __syncwarp();
        // stash overflow went straight to the global queue; spill a full stash
        if (lane == 0) {
            int sn = *b.stn;
            if (sn > STASH) sn = STASH;
            if (A.stash_spill && sn >= (int)A.stash_spill) {
                push_global(A, b.stash + A.stash_keep, sn - (int)A.stash_keep, 0);
                sn = (int)A.stash_keep;
            }
            *b.stn = sn;
        }
        __syncwarp();
        if (*b.sn >= STG_FLUSH) flush_staging(A, b, lane);
    }
    flush_staging(A, b, lane);
    for (int o = 16; o; o >>= 1) {
        dep.e += __shfl_xor_sync(0xffffffffu, dep.e, o);
        dep.n += __shfl_xor_sync(0xffffffffu, dep.n, o);
        nsteps += __shfl_xor_sync(0xffffffffu, nsteps, o);
    }
    if (lane == 0) {
        atomicAdd(&S->dep_f64, dep.e);
        atomicAdd(&S->steps, nsteps);
        atomicAdd(&cnt[D_DOSE], dep.n);
    }
    __syncthreads();
    if (threadIdx.x < 24 && cnt[threadIdx.x]) {
        uint32_t v = cnt[threadIdx.x];
        if (threadIdx.x < 8) atomicAdd(&S->counters[threadIdx.x], v);
        else if (threadIdx.x < 16) atomicAdd(&S->sec_stats[threadIdx.x - 8], v);
        else atomicAdd(&S->dbg[threadIdx.x - 16], v);
    }
}

// ---------------------------------------------------------------- canonical order
// Histogram of stored entries per primary.
__global__ void k_pid_hist(const unsigned long long* key, unsigned long long n, uint32_t* cnt) {
    unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
    unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (; i < n; i += stride) atomicAdd(&cnt[(uint32_t)(key[i] >> 34)], 1u);
}

// Exclusive scan of n counts into off[0..n] with one block (chunked per thread).
__global__ void k_scan(const uint32_t* cnt, uint32_t n, unsigned long long* off) {
    __shared__ unsigned long long part[1024];
    uint32_t t = threadIdx.x, per = (n + blockDim.x - 1) / blockDim.x;
    uint32_t lo = min(t * per, n), hi = min(lo + per, n);
    unsigned long long s = 0;
    for (uint32_t i = lo; i < hi; ++i) s += cnt[i];
    part[t] = s;
    __syncthreads();
    if (t == 0) {
        unsigned long long acc = 0;
        for (uint32_t i = 0; i < blockDim.x; ++i) { unsigned long long v = part[i]; part[i] = acc; acc += v; }
        off[n] = acc;
    }
    __syncthreads();
    s = part[t];
    for (uint32_t i = lo; i < hi; ++i) { off[i] = s; s += cnt[i]; }
}

__global__ void k_scatter(const unsigned long long* key, unsigned long long n, const unsigned long long* off,
                          uint32_t* cur, uint32_t* perm) {
    unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
    unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (; i < n; i += stride) {
        uint32_t p = (uint32_t)(key[i] >> 34);
        perm[off[p] + atomicAdd(&cur[p], 1u)] = (uint32_t)i;
    }
}

constexpr int SEG_MAX = 8192;

// One block per primary: sort its entries by key (bitonic, shared memory) and
// write them to the canonical buffer.
__global__ void __launch_bounds__(1024) k_segsort(const unsigned long long* key, const float4* rad,
                                                  const uint32_t* perm, const unsigned long long* off,
                                                  float4* out, uint32_t* err) {
    extern __shared__ __align__(16) unsigned char seg_smem[];
    unsigned long long* sk = reinterpret_cast<unsigned long long*>(seg_smem);
    uint32_t* si = reinterpret_cast<uint32_t*>(sk + SEG_MAX);
    uint32_t p = blockIdx.x;
    unsigned long long s = off[p], e = off[p + 1];
    uint32_t len = (uint32_t)(e - s);
    if (len == 0) return;
    if (len > SEG_MAX) { if (threadIdx.x == 0) atomicOr(err, DERR_SEG_SORT); return; }
    uint32_t n2 = 1;
    while (n2 < len) n2 <<= 1;
    for (uint32_t i = threadIdx.x; i < n2; i += blockDim.x) {
        if (i < len) { uint32_t ix = perm[s + i]; sk[i] = key[ix]; si[i] = ix; }
        else { sk[i] = ~0ull; si[i] = 0; }
    }
    __syncthreads();
    for (uint32_t k = 2; k <= n2; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < n2; i += blockDim.x) {
                uint32_t l = i ^ j;
                if (l > i) {
                    bool up = (i & k) == 0;
                    unsigned long long a = sk[i], c = sk[l];
                    if ((a > c) == up) { sk[i] = c; sk[l] = a; uint32_t t = si[i]; si[i] = si[l]; si[l] = t; }
                }
            }
            __syncthreads();
        }
    }
    for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) out[s + i] = rad[si[i]];
}

// n_therm (non-escaped primaries) and the dose-grid sum
__global__ void k_reduce(const float* results, uint32_t np, const uint32_t* dose, uint32_t nvox,
                         unsigned long long* out) {
    unsigned long long sd = 0;
    uint32_t nt = 0;
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    for (uint32_t v = i; v < nvox; v += stride) sd += dose[v];
    for (uint32_t v = i; v < np; v += stride) nt += (__float_as_uint(results[8ull * v + 5]) == 0u);
    for (int o = 16; o; o >>= 1) {
        sd += __shfl_xor_sync(0xffffffffu, sd, o);
        nt += __shfl_xor_sync(0xffffffffu, nt, o);
    }
    if ((threadIdx.x & 31) == 0) { atomicAdd(&out[0], sd); atomicAdd(&out[1], (unsigned long long)nt); }
}

// ------------------------------------------------------------------ host side
size_t transport_smem_bytes() {
    return S_TOTAL_PAD * 4 + TW * STG * 16 + TW * STG * 8 + TW * STASH * sizeof(StashRec) + 2 * TW * 4 + 24 * 4;
}

// resident CTAs of k_transport on `device` (the current device); the shared
// memory attribute is set on each device the first time
int transport_blocks(int device, uint32_t ctas_per_sm) {
    static DeviceOnce attr;
    attr.run([] {
        return cudaFuncSetAttribute(k_transport, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)transport_smem_bytes());
    });
    int sms = 0, per = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_transport, TB, transport_smem_bytes());
    if (per < 1) per = 1;
    if (ctas_per_sm && (int)ctas_per_sm < per) per = (int)ctas_per_sm;
    return sms * per;
}

cudaError_t launch_transport(const TArgs& a, int blocks, cudaStream_t s) {
    k_transport<<<blocks, TB, transport_smem_bytes(), s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_canon(const unsigned long long* key, const float4* rad, unsigned long long n, uint32_t np,
                         uint32_t* cnt, unsigned long long* off, uint32_t* cur, uint32_t* perm, float4* out,
                         uint32_t* err, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(cnt, 0, (size_t)np * 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(cur, 0, (size_t)np * 4, s);
    if (e != cudaSuccess) return e;
    if (n) k_pid_hist<<<1184, 256, 0, s>>>(key, n, cnt);
    k_scan<<<1, 1024, 0, s>>>(cnt, np, off);
    if (n) {
        k_scatter<<<1184, 256, 0, s>>>(key, n, off, cur, perm);
        static DeviceOnce attr;
        e = attr.run([] {
            return cudaFuncSetAttribute(k_segsort, cudaFuncAttributeMaxDynamicSharedMemorySize, SEG_MAX * 12);
        });
        if (e != cudaSuccess) return e;
        k_segsort<<<np, 1024, SEG_MAX * 12, s>>>(key, rad, perm, off, out, err);
    }
    return cudaGetLastError();
}

cudaError_t launch_scan_u32(const uint32_t* cnt, uint32_t n, unsigned long long* off, cudaStream_t s) {
    k_scan<<<1, 1024, 0, s>>>(cnt, n, off);
    return cudaGetLastError();
}

cudaError_t launch_reduce(const float* results, uint32_t np, const uint32_t* dose, uint32_t nvox,
                          unsigned long long* out, cudaStream_t s) {
    { cudaError_t me_ = cudaMemsetAsync(out, 0, 16, s); if (me_ != cudaSuccess) return me_; }
    k_reduce<<<592, 256, 0, s>>>(results, np, dose, nvox, out);
    return cudaGetLastError();
}

}  // namespace wg
