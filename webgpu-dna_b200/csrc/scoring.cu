// scoring.cu -- SSB / DSB scoring on the B-DNA fibre grid.
//
// Results are bit-identical to src/scoring/ssb-dsb.ts of allaunthefox/webgpu-dna
// (scoreDirectSSB_events :135-217, scoreIndirectSSB :43-121, clusterDSB
// :348-407, makeSsbRng :421-427) evaluated with JavaScript number semantics.
// The reference is a sequential loop; here every entry is scored in parallel:
//
//  1. k_prep: per entry, the adjacent-duplicate link (same xyz as the next
//     entry), the in-reach test and the hit-byte index.  The reference's
//     skip-by-2 walk visits entry i iff (i - start of its run of linked
//     entries) is even.
//  2. k_tiles / k_tilescan: per tile of 1024 entries, the last run start and
//     the number of LCG draws for either parity of an incoming run; one block
//     scans the tiles (run starts by max-scan, draw counts by sum-scan).
//  3. k_apply: per entry, its draw index k; the LCG state after k+1 steps is
//     an affine map (1664525 s + 1013904223 mod 2^32) raised to k+1 by
//     squaring; a draw below p sets the hit byte (atomicOr, counted once).
//
// clusterDSB: one block per fibre collects the strand-0 / strand-1 hit lists
// in order and pairs them greedily; the expected-DSB sum uses the host's pow.
#include "scoring.cuh"

namespace wg {


constexpr int STILE = 1024;

__device__ __forceinline__ double js_round(double x) {
    double f = floor(x);
    return (x - f >= 0.5) ? f + 1.0 : f;
}

// nearest backbone within r_d (ssb-dsb.ts:73-106); returns hit index or -1
__device__ __forceinline__ long long near_backbone(const DnaDev& d, double x, double y, double z,
                                                   double r_d, int* cand) {
    double x_half = ((double)d.n_bp_per - 1) * d.rise * 0.5;
    double rise_inv = 1 / d.rise;
    double grid_off = -(((double)d.grid_N - 1) * d.spacing) * 0.5;
    double inv_sp = 1 / d.spacing;
    *cand = 0;
    if (x < -x_half - r_d || x > x_half + r_d) return -1;
    double fi = js_round((y - grid_off) * inv_sp);
    double fj = js_round((z - grid_off) * inv_sp);
    if (fi < 0 || fi >= d.grid_N || fj < 0 || fj >= d.grid_N) return -1;
    uint32_t fiber = (uint32_t)fi * d.grid_N + (uint32_t)fj;
    double y_rel = y - (double)d.fy[fiber];
    double z_rel = z - (double)d.fz[fiber];
    double r2 = y_rel * y_rel + z_rel * z_rel;
    double outer = d.r_bb + r_d;
    if (r2 > outer * outer) return -1;
    *cand = 1;
    double bp_est = js_round((x + x_half) * rise_inv);
    double b0 = bp_est - 2 > 0 ? bp_est - 2 : 0;
    double b1 = bp_est + 2 < (double)d.n_bp_per - 1 ? bp_est + 2 : (double)d.n_bp_per - 1;
    double best = __longlong_as_double(0x7ff0000000000000ll);
    long long best_bp = -1;
    int best_s = -1;
    for (double bb = b0; bb <= b1; bb += 1) {
        long long b = (long long)bb;
        double dx = x - (d.x0 + bb * d.rise);
        double dy0 = y_rel - (double)d.rbb0[2 * b], dz0 = z_rel - (double)d.rbb0[2 * b + 1];
        double d20 = dx * dx + dy0 * dy0 + dz0 * dz0;
        if (d20 < best) { best = d20; best_bp = b; best_s = 0; }
        double dy1 = y_rel - (double)d.rbb1[2 * b], dz1 = z_rel - (double)d.rbb1[2 * b + 1];
        double d21 = dx * dx + dy1 * dy1 + dz1 * dz1;
        if (d21 < best) { best = d21; best_bp = b; best_s = 1; }
    }
    if (!(best < r_d * r_d)) return -1;
    return (long long)fiber * d.n_bp_per + best_bp + (long long)best_s * d.n_bp;
}

// info word: bit31 run start, bit30 in reach, bit29 candidate (near a fibre
// axis), bits 0..28 hit index.  Candidates are counted by k_apply for the
// entries the reference's walk visits (ssb-dsb.ts:183).
__global__ void k_prep(const float4* rad, const uint32_t* alive, unsigned long long n, DnaDev d,
                       double r_d, int dedupe, uint32_t* info) {
    unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
    if (i < n) {
        float4 e = rad[i];
        uint32_t brk = 1;
        if (dedupe && i > 0) {
            float4 p = rad[i - 1];
            brk = !(p.x == e.x && p.y == e.y && p.z == e.z);
        }
        uint32_t w = brk << 31;
        bool consider = true;
        if (alive) consider = alive[i] != 0 && js_round((double)e.w) == 0.0;   // OH only
        if (consider) {
            int cand;
            long long h = near_backbone(d, e.x, e.y, e.z, r_d, &cand);
            if (cand) w |= 1u << 29;
            if (h >= 0) w |= (1u << 30) | (uint32_t)h;
        }
        info[i] = w;
    }
}

// per tile: last run start (or -1) and draw counts for incoming parity 0 / 1
__global__ void __launch_bounds__(STILE) k_tiles(const uint32_t* info, unsigned long long n,
                                                 long long* last_brk, uint32_t* cnt0, uint32_t* cnt1) {
    __shared__ long long s_last;
    __shared__ uint32_t s_c0, s_c1;
    unsigned long long a = (unsigned long long)blockIdx.x * STILE;
    unsigned long long i = a + threadIdx.x;
    if (threadIdx.x == 0) { s_last = -1; s_c0 = 0; s_c1 = 0; }
    __syncthreads();
    uint32_t w = i < n ? info[i] : 0u;
    bool brk = i < n && (w >> 31);
    if (brk) atomicMax(&s_last, (long long)i);
    __syncthreads();
    // local run start: max brk position <= t within the tile (inclusive max-scan)
    __shared__ int s_cs[STILE];
    s_cs[threadIdx.x] = brk ? (int)threadIdx.x : -1;
    __syncthreads();
    for (int off = 1; off < STILE; off <<= 1) {
        int v = s_cs[threadIdx.x];
        int u = threadIdx.x >= (unsigned)off ? s_cs[threadIdx.x - off] : -1;
        __syncthreads();
        s_cs[threadIdx.x] = max(v, u);
        __syncthreads();
    }
    bool inr = i < n && ((w >> 30) & 1u);
    if (inr) {
        int cs = s_cs[threadIdx.x];
        if (cs >= 0) {
            if (((threadIdx.x - cs) & 1) == 0) { atomicAdd(&s_c0, 1u); atomicAdd(&s_c1, 1u); }
        } else {
            // before the tile's first run start: parity relative to the incoming run
            if ((threadIdx.x & 1) == 0) atomicAdd(&s_c0, 1u); else atomicAdd(&s_c1, 1u);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) { last_brk[blockIdx.x] = s_last; cnt0[blockIdx.x] = s_c0; cnt1[blockIdx.x] = s_c1; }
}

struct Aff { uint32_t a, c; };
__device__ __forceinline__ Aff aff_mul(Aff g, Aff f) { return Aff{g.a * f.a, g.a * f.c + g.c}; }   // g after f
__device__ __forceinline__ uint32_t lcg_jump(uint32_t s, unsigned long long k) {
    Aff r{1u, 0u}, p{1664525u, 1013904223u};
    while (k) {
        if (k & 1ull) r = aff_mul(p, r);
        p = aff_mul(p, p);
        k >>= 1;
    }
    return r.a * s + r.c;
}

// one block: per-tile incoming run start and draw base
__global__ void k_tilescan(const long long* last_brk, const uint32_t* cnt0, const uint32_t* cnt1,
                           uint32_t ntiles, long long* cs_in, unsigned long long* base,
                           unsigned long long* total) {
    __shared__ long long smax[1024];
    __shared__ unsigned long long ssum[1024];
    uint32_t t = threadIdx.x, per = (ntiles + blockDim.x - 1) / blockDim.x;
    uint32_t lo = min(t * per, ntiles), hi = min(lo + per, ntiles);
    long long m = -1;
    for (uint32_t k = lo; k < hi; ++k) m = max(m, last_brk[k]);
    smax[t] = m;
    __syncthreads();
    if (t == 0) {
        long long acc = -1;
        for (uint32_t k = 0; k < blockDim.x; ++k) { long long v = smax[k]; smax[k] = acc; acc = max(acc, v); }
    }
    __syncthreads();
    long long run = smax[t];
    unsigned long long s = 0;
    for (uint32_t k = lo; k < hi; ++k) {
        cs_in[k] = run;
        unsigned long long a = (unsigned long long)k * STILE;
        uint32_t par = (uint32_t)((a - (unsigned long long)run) & 1ull);   // run >= 0 for k >= 1
        s += k == 0 ? cnt0[k] : (par ? cnt1[k] : cnt0[k]);
        run = max(run, last_brk[k]);
    }
    ssum[t] = s;
    __syncthreads();
    if (t == 0) {
        unsigned long long acc = 0;
        for (uint32_t k = 0; k < blockDim.x; ++k) { unsigned long long v = ssum[k]; ssum[k] = acc; acc += v; }
        *total = acc;
    }
    __syncthreads();
    s = ssum[t];
    run = smax[t];
    for (uint32_t k = lo; k < hi; ++k) {
        base[k] = s;
        unsigned long long a = (unsigned long long)k * STILE;
        uint32_t par = (uint32_t)((a - (unsigned long long)run) & 1ull);
        s += k == 0 ? cnt0[k] : (par ? cnt1[k] : cnt0[k]);
        run = max(run, last_brk[k]);
    }
}

// per entry: visited? draw index, LCG value, hit byte
__global__ void __launch_bounds__(STILE) k_apply(const uint32_t* info, unsigned long long n, const long long* cs_in,
                                                 const unsigned long long* base, uint32_t s0, double p,
                                                 uint32_t n_bp, uint32_t* hits_words, unsigned long long* cnt) {
    __shared__ int s_cs[STILE];
    __shared__ uint32_t s_scan[STILE];
    unsigned long long a = (unsigned long long)blockIdx.x * STILE;
    unsigned long long i = a + threadIdx.x;
    uint32_t w = i < n ? info[i] : 0u;
    bool brk = i < n && (w >> 31);
    s_cs[threadIdx.x] = brk ? (int)threadIdx.x : -1;
    __syncthreads();
    for (int off = 1; off < STILE; off <<= 1) {
        int v = s_cs[threadIdx.x];
        int u = threadIdx.x >= (unsigned)off ? s_cs[threadIdx.x - off] : -1;
        __syncthreads();
        s_cs[threadIdx.x] = max(v, u);
        __syncthreads();
    }
    long long cs = s_cs[threadIdx.x] >= 0 ? (long long)(a + s_cs[threadIdx.x]) : cs_in[blockIdx.x];
    bool visited = i < n && (((unsigned long long)((long long)i - cs) & 1ull) == 0);
    bool draw = visited && ((w >> 30) & 1u);
    unsigned cm = __ballot_sync(0xffffffffu, visited && ((w >> 29) & 1u));
    if ((threadIdx.x & 31) == 0 && cm) atomicAdd(&cnt[3], (unsigned long long)__popc(cm));
    // exclusive prefix count of draws in the tile
    s_scan[threadIdx.x] = draw ? 1u : 0u;
    __syncthreads();
    for (int off = 1; off < STILE; off <<= 1) {
        uint32_t v = s_scan[threadIdx.x];
        uint32_t u = threadIdx.x >= (unsigned)off ? s_scan[threadIdx.x - off] : 0u;
        __syncthreads();
        s_scan[threadIdx.x] = v + u;
        __syncthreads();
    }
    if (!draw) return;
    unsigned long long k = base[blockIdx.x] + s_scan[threadIdx.x] - 1;   // 0-based draw index
    uint32_t s = lcg_jump(s0, k + 1);
    double u = s / 4294967296.0;
    if (u < p) {
        uint32_t h = w & 0x1fffffffu;
        uint32_t shift = (h & 3u) * 8u;
        uint32_t old = atomicOr(&hits_words[h >> 2], 1u << shift);
        if (((old >> shift) & 0xffu) == 0u) {
            atomicAdd(&cnt[0], 1ull);
            atomicAdd(&cnt[h >= n_bp ? 2 : 1], 1ull);
        }
    }
}

// clusterDSB, one block per fibre
__global__ void k_cluster(const uint8_t* hits, uint32_t n_per, uint32_t n_bp, uint32_t* out /*3 per fibre*/) {
    extern __shared__ uint32_t lists[];
    uint32_t* s0 = lists;
    uint32_t* s1 = lists + n_per;
    __shared__ uint32_t k0, k1, wcount[2][32];
    const uint8_t* h0 = hits + (size_t)blockIdx.x * n_per;
    const uint8_t* h1 = h0 + n_bp;
    if (threadIdx.x == 0) { k0 = 0; k1 = 0; }
    __syncthreads();
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (uint32_t c = 0; c < n_per; c += blockDim.x) {
        uint32_t b = c + threadIdx.x;
        bool f0 = b < n_per && h0[b] == 1, f1 = b < n_per && h1[b] == 1;
        unsigned m0 = __ballot_sync(0xffffffffu, f0), m1 = __ballot_sync(0xffffffffu, f1);
        if (lane == 0) { wcount[0][wid] = __popc(m0); wcount[1][wid] = __popc(m1); }
        __syncthreads();
        uint32_t o0 = k0, o1 = k1;
        for (int q = 0; q < wid; ++q) { o0 += wcount[0][q]; o1 += wcount[1][q]; }
        unsigned lt = (1u << lane) - 1u;
        if (f0) s0[o0 + __popc(m0 & lt)] = b;
        if (f1) s1[o1 + __popc(m1 & lt)] = b;
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int q = 0; q < nw; ++q) { k0 += wcount[0][q]; k1 += wcount[1][q]; }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const int W = 10;
        uint32_t dsb = 0, jlo = 0;
        // used flags packed in the high bit of s1 entries
        for (uint32_t a = 0; a < k0; ++a) {
            long long b0 = s0[a];
            while (jlo < k1 && (long long)(s1[jlo] & 0x7fffffffu) < b0 - W) jlo++;
            for (uint32_t j = jlo; j < k1 && (long long)(s1[j] & 0x7fffffffu) <= b0 + W; ++j) {
                if (!(s1[j] >> 31)) { s1[j] |= 0x80000000u; dsb++; break; }
            }
        }
        out[3 * blockIdx.x] = dsb;
        out[3 * blockIdx.x + 1] = k0;
        out[3 * blockIdx.x + 2] = k1;
    }
}

// ------------------------------------------------------------------ host side

cudaError_t launch_score(const float4* rad, const uint32_t* alive, unsigned long long n, const DnaDev& d,
                         double r_d, double p, int dedupe, uint32_t s0, uint32_t* hits_words,
                         const ScoreScratch& sc, cudaStream_t s) {
    // the result counters must start at zero: a failed clear would leave the
    // previous call's counts to be read back
    cudaError_t e = cudaMemsetAsync(sc.u64, 0, 8 * sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    if (n == 0) return cudaGetLastError();
    unsigned long long ntiles = (n + STILE - 1) / STILE;
    k_prep<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(rad, alive, n, d, r_d, dedupe, sc.info);
    k_tiles<<<(unsigned)ntiles, STILE, 0, s>>>(sc.info, n, sc.last_brk, sc.cnt0, sc.cnt1);
    k_tilescan<<<1, 1024, 0, s>>>(sc.last_brk, sc.cnt0, sc.cnt1, (uint32_t)ntiles, sc.cs_in, sc.base, sc.u64 + 4);
    k_apply<<<(unsigned)ntiles, STILE, 0, s>>>(sc.info, n, sc.cs_in, sc.base, s0, p, d.n_bp, hits_words, sc.u64);
    return cudaGetLastError();
}

cudaError_t launch_cluster(const uint8_t* hits, const DnaDev& d, uint32_t n_fibers, uint32_t* out, cudaStream_t s) {
    size_t sm = (size_t)d.n_bp_per * 8;
    static DeviceOnce attr;
    cudaError_t e = attr.run([] {
        return cudaFuncSetAttribute(k_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    });
    if (e != cudaSuccess) return e;
    k_cluster<<<n_fibers, 256, sm, s>>>(hits, d.n_bp_per, d.n_bp, out);
    return cudaGetLastError();
}

uint32_t lcg_jump_host(uint32_t s, unsigned long long k) {
    uint32_t ra = 1u, rc = 0u, pa = 1664525u, pc = 1013904223u;
    while (k) {
        if (k & 1ull) { uint32_t na = pa * ra, nc = pa * rc + pc; ra = na; rc = nc; }
        uint32_t na = pa * pa, nc = pa * pc + pc; pa = na; pc = nc;
        k >>= 1;
    }
    return ra * s + rc;
}

}  // namespace wg
