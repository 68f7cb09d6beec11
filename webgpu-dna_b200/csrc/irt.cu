// irt.cu -- Karamitros 2011 9-reaction IRT radiolysis chemistry to 1 us.
//
// Follows public/irt-worker.js of allaunthefox/webgpu-dna (species and
// reaction tables :191-286, sampleIRT :116-184 with SamplePDC :91-113, erfcinv
// :31-39, erfcx :53-88, the per-primary event loop :470-667 and pairWithAlive
// :430-465).  The reference runs the primaries one after another on one CPU
// thread; here one warp owns one track (primary) at a time and the warps of a
// persistent grid pull tracks from a counter:
//
// * load: entries of the track (codes 4/7 skipped, 7 counted as initial H2)
//   are displaced in f64 with the thermalisation Gaussians, 32 at a time;
// * initial pairing: tiles of 32 particles held in lane registers, the partner
//   j broadcast to all lanes; one Philox block gives the acceptance draws of
//   four consecutive partners;
// * sort: the initial events of a track in (t, i, j) order, one block per
//   track, in shared memory;
// * events: the sorted initial events merged with a binary heap of product
//   events ordered by (t, i, j), kept by lane 0; the product re-pairing
//   (pairWithAlive) is spread over the 32 lanes.
//
// Random draws are keyed by what they are for (track, particle, pair), so the
// result does not depend on scheduling; the CPU oracle uses the same streams:
//   load of particle k            philox(blk, k, pid, 2), 53-bit doubles
//   acceptance of pair i<j         philox(j>>2, i, pid, 3), word j&3
//   SamplePDC trial t of (i, j)    philox(i, j, pid, 4 | t<<4)
//   product idx, partner jj        philox(idx, jj, pid, 5): Box-Muller radii
//                                  x,y,z + acceptance; philox(.., 5 | 1<<4):
//                                  Box-Muller angles.
#include <cstring>

#include "irt.cuh"
#include "dmath.cuh"

namespace wg {


__constant__ IrtConst c_irt;


constexpr int IB = 128;                  // threads per block (4 warps)

__device__ __forceinline__ double erfcinv_(double x) {                       // :31-39
    if (x <= 0 || x >= 2) return 0;
    double p = x > 1 ? 2 - x : x;
    double t = sqrt(-2 * log_(p / 2));
    double y = t - (2.515517 + 0.802853 * t + 0.010328 * t * t) /
                   (1 + 1.432788 * t + 0.189269 * t * t + 0.001308 * t * t * t);
    y *= 0.7071067811865475;
    return x > 1 ? -y : y;
}

__constant__ double c_erfcx[28] = {
    -1.3026537197817094, 6.4196979235649026e-1, 1.9476473204185836e-2, -9.561514786808631e-3,
    -9.46595344482036e-4, 3.66839497852761e-4, 4.2523324806907e-5, -2.0278578112534e-5,
    -1.624290004647e-6, 1.303655835580e-6, 1.5626441722e-8, -8.5238095915e-8,
    6.529054439e-9, 5.059343495e-9, -9.91364156e-10, -2.27365122e-10,
    9.6467911e-11, 2.394038e-12, -6.886027e-12, 8.94487e-13,
    3.13092e-13, -1.12708e-13, 3.81e-16, 7.106e-15,
    -1.523e-15, -9.4e-17, 1.21e-16, -2.8e-17};

__device__ double erfcx_pos(double x) {                                      // :53-88, x >= 0
    if (x >= 6) {
        double f = 0;
        for (int n = 30; n >= 1; --n) f = (0.5 * n) / (x + f);
        return 0.5641895835477563 / (x + f);
    }
    double t = 2.0 / (2.0 + x);
    double ty = 4 * t - 2;
    double d = 0, dd = 0;
    for (int j = 27; j > 0; --j) { double tmp = d; d = ty * d - dd + c_erfcx[j]; dd = tmp; }
    return t * exp_(0.5 * (c_erfcx[0] + ty * d) - dd);
}
__device__ __forceinline__ double erfcx_(double x) {
    if (x < 0) return 2 * exp_(x * x) - erfcx_pos(-x);
    return erfcx_pos(x);
}

// f32 erfcx for z >= 0, used only to bound the f64 value: the reference's
// Chebyshev form (first 14 coefficients) below 6, the asymptotic series
// (1 / (z sqrt(pi))) sum (-1)^k (2k-1)!! / (2 z^2)^k to k = 7 above.  Its
// largest relative error against the f64 form is 3.3e-7 (z on a 1e-5 grid
// to 200 and log-spaced to 1e8, with a 1-ulp expf).
__constant__ float c_erfcx_f[14] = {
    -1.3026537197817094f, 6.4196979235649026e-1f, 1.9476473204185836e-2f, -9.561514786808631e-3f,
    -9.46595344482036e-4f, 3.66839497852761e-4f, 4.2523324806907e-5f, -2.0278578112534e-5f,
    -1.624290004647e-6f, 1.303655835580e-6f, 1.5626441722e-8f, -8.5238095915e-8f,
    6.529054439e-9f, 5.059343495e-9f};

__device__ __forceinline__ float erfcx_f(float z) {
    if (z >= 6.0f) {
        float iz = __frcp_rn(z);
        float h = 0.5f * iz * iz;
        float s = 1.0f - 13.0f * h;
        s = 1.0f - 11.0f * h * s; s = 1.0f - 9.0f * h * s; s = 1.0f - 7.0f * h * s;
        s = 1.0f - 5.0f * h * s; s = 1.0f - 3.0f * h * s; s = 1.0f - h * s;
        return s * 0.5641895835f * iz;
    }
    float t = __fdividef(2.0f, 2.0f + z), ty = 4.0f * t - 2.0f, d = 0.0f, dd = 0.0f;
    for (int j = 13; j > 0; --j) { float tmp = d; d = ty * d - dd + c_erfcx_f[j]; dd = tmp; }
    return t * __expf(0.5f * (c_erfcx_f[0] + ty * d) - dd);
}

// SamplePDC (:91-113) for one pair, 32 trials at a time across the warp; the
// first accepted trial in trial order wins, as in the sequential loop.  Must
// be called by all 32 lanes with the same arguments.
//
// A trial is accepted when U2 <= lambdax (X <= 2b/a) or U2 M / X <= lambdax
// (X >= 2b/a), lambdax = e (1 - Q), e = exp(-b^2/X), Q = a sqrt(pi X)
// erfcx(b/sqrt(X) + a sqrt(X)).  Each trial first brackets the f64 lambdax
// with f32 arithmetic (the fast reciprocal, rsqrt, divide and exp2
// instructions, 2 ulp each; ex2 adds |x| 8.6e-8 for exp(x)):
//   X to 7e-7 relative, so b^2/X to 1.7e-6 and e to (4e-6 b^2/X + 2e-6);
//   z to 1e-6 relative, which moves erfcx by at most 1.2e-6 (|d ln erfcx/dz|
//   <= 1.13 and <= 1/z); with the 3.3e-7 of erfcx_f (8e-7 with the fast
//   exp) the prefactor Q is known to 4e-6, taken as 2e-5, 1 - Q to that
//   plus 1e-6;
//   for z >= 6 and b >= 0, where 1 - Q cancels, 1 - Q itself: with
//   beta = (b/sqrt(X))/z, Q = (1 - beta) S and erfcx(z) = S/(z sqrt(pi)),
//   S = 1 - h s (h = 1/(2z^2), s the asymptotic series of erfcx_f), so
//   1 - Q = beta + (1 - beta) h s, a sum of two non-negative terms known to
//   1.7e-6 and 4.2e-6 relative (1/z correctly rounded; the f32 series
//   within 2.2e-7 of h s); taken as 2e-5.  The f64 1 - Q it must bound
//   carries the rounding of Q near 1 (about 7 ulp, the continued fraction
//   of erfcx_pos within 2.2e-16), so 1e-14 is added on both sides;
// and decides when U2 (or U2 M against lambdax X) lies outside the bracket
// with a further 1e-6 (3e-6) margin.  Trials inside the bracket, near
// X = 2b/a, with e below exp(-80) in case B, z < 0, or a zero draw are
// evaluated exactly in f64; only the winner's X is computed in f64.
__device__ __noinline__ double pdc_warp(uint32_t i, uint32_t j, uint32_t pid, uint32_t k0, uint32_t k1, double a, double b,
                           int lane) {
    double p = 2.0 * sqrt(2.0 * b / a);
    double q = 2.0 / sqrt(2.0 * b / a);
    double M = fmax(1.0 / (a * a), 3.0 * b / a);
    const double pq = p + q * M, thr = p / pq, t2 = 2.0 * b / a;
    const float pqf = (float)pq, Mf = (float)M, t2f = (float)t2, bbf = (float)(b * b);
    const float af = (float)a, bf = (float)b;
    for (uint32_t t0 = 0; t0 < 10000; t0 += 32) {
        uint32_t trial = t0 + lane;
        int st = 0;                               // 0 rejected, 1 accepted, 2 undecided
        double U1 = 0, U2 = 0;
        if (trial < 10000) {
            u4 w = philox(i, j, pid, 4u | (trial << 4), k0, k1);
            U1 = u01d(w.x, w.y);
            U2 = u01d(w.z, w.w);
            st = 2;
            float xf;
            if (U1 < thr) { float h = (float)U1 * pqf * 0.5f; xf = h * h; }
            else { float h = __fdividef(2.0f * Mf, (float)(1.0 - U1) * pqf); xf = h * h; }
            const bool ca = xf < t2f * 0.99999f, cb = xf > t2f * 1.00001f;
            if (U2 > 0.0 && xf > 1e-30f && xf < 1.0e30f && (ca || cb)) {
                const float rs = rsqrtf(xf);
                const float argf = bbf * rs * rs;
                float elo = 0.0f, ehi = 1e-30f;
                if (argf <= 80.0f) {
                    const float ef = __expf(-argf), re = argf * 4e-6f + 2e-6f;
                    elo = ef * (1.0f - re); ehi = ef * (1.0f + re);
                }
                const float sx = xf * rs;
                const float zf = bf * rs + af * sx;
                if (zf >= 0.0f) {
                    float flo, fhi;
                    if (zf >= 6.0f && bf >= 0.0f) {
                        const float iz = __frcp_rn(zf), h = 0.5f * iz * iz;
                        float s = 1.0f - 13.0f * h;
                        s = 1.0f - 11.0f * h * s; s = 1.0f - 9.0f * h * s; s = 1.0f - 7.0f * h * s;
                        s = 1.0f - 5.0f * h * s; s = 1.0f - 3.0f * h * s;
                        const float omq = fmaf(af * sx * iz, h * s, bf * rs * iz);
                        flo = omq * 0.99998f - 1e-14f; fhi = omq * 1.00002f + 1e-14f;
                    } else {
                        const float Q = af * 1.7724539f * sx * erfcx_f(zf);
                        flo = 1.0f - Q * 1.00002f - 1e-6f; fhi = 1.0f - Q * 0.99998f + 1e-6f;
                    }
                    const double Llo = (double)(elo * fmaxf(flo, 0.0f)) * (1.0 - 1e-6);
                    const double Lhi = (double)(ehi * fmaxf(fhi, 0.0f)) * (1.0 + 1e-6) + 1e-37;
                    if (ca) st = U2 <= Llo ? 1 : (U2 > Lhi ? 0 : 2);
                    else {
                        const double lhs = U2 * M;
                        st = lhs <= Llo * (double)xf * (1.0 - 3e-6) ? 1 : (lhs > Lhi * (double)xf * (1.0 + 3e-6) ? 0 : 2);
                    }
                }
            }
        }
        if (__any_sync(0xffffffffu, st == 2) && st == 2) {
            double X;
            if (U1 < thr) { double h = U1 * pq / 2; X = h * h; }
            else { double h = 2 / ((1 - U1) * pq / M); X = h * h; }
            // lambdax <= e: a trial that fails against e alone is rejected
            // without evaluating erfcx (same decision as the full test)
            double e = exp_(-b * b / X);
            double v = U2 * M / X;
            st = 0;
            if ((X <= t2 && U2 <= e) || (X >= t2 && v <= e)) {
                double sqX = sqrt(X);
                double lambdax = e * (1.0 - a * sqrt(3.141592653589793 * X) * erfcx_(b / sqX + a * sqX));
                st = ((X <= t2 && U2 <= lambdax) || (X >= t2 && v <= lambdax)) ? 1 : 0;
            }
        }
        unsigned m = __ballot_sync(0xffffffffu, st == 1);
        if (m) {
            const int src = __ffs(m) - 1;
            double X = 0;
            if (lane == src) {
                if (U1 < thr) { double h = U1 * pq / 2; X = h * h; }
                else { double h = 2 / ((1 - U1) * pq / M); X = h * h; }
            }
            return __shfl_sync(0xffffffffu, X, src);
        }
    }
    return -1.0;
}

// sampleIRT (:116-184) with the acceptance draw U supplied.  Returns the
// reaction time t >= 0, -1 for no reaction, or -2 when SamplePDC must be run
// with (*pa, *pb); the caller then uses X / D for X > 0.
__device__ __forceinline__ double sample_pre(const IrtConst& C, double r0, int ri, double D, double U,
                                             double* pa, double* pb) {
    if (C.type[ri] == 0) {
        double sigma = C.sigma[ri], rc = C.rc[ri];
        if (sigma <= 0 || D <= 0) return -1;
        if (r0 <= sigma) return 0;
        double r0e = r0;
        if (rc != 0) r0e = -rc / (1 - exp_(rc / r0));
        if (r0e <= sigma) return 0;
        double Winf = sigma / r0e;
        if (U <= 0 || U >= Winf) return -1;
        double ei = erfcinv_(r0e * U / sigma);
        if (fabs(ei) < 1e-10) return -1;
        double dr = r0e - sigma;
        return 0.25 * dr * dr / (D * ei * ei);
    }
    double sigma_c = C.sigma[ri], rc = C.rc[ri];
    double b, sc_chk = sigma_c, r0_chk = r0;
    if (rc == 0) {
        b = (r0 - sigma_c) / 2;
    } else {
        double coth_r0 = 1.0 + 2.0 / expm1_(2.0 * (rc / (2 * r0)));
        b = rc / 4 * (coth_r0 - C.coth_sig[ri]);
        r0_chk = -rc / (1 - exp_(rc / r0));
        sc_chk = C.sigma_eff[ri];
    }
    if (sc_chk > r0_chk) return (C.prob[ri] > U) ? 0 : -1;
    double Winf = sc_chk / r0_chk * C.kobs[ri] / C.kdif[ri];
    if (Winf > U) { *pa = C.a_pdc[ri]; *pb = b; return -2; }
    return -1;
}

// Distance beyond which sample_pre certainly returns -1 for acceptance draw U:
//   TDC:  Winf = sigma / r0e and r0e >= r0 - max(rc,0)/2      -> r0 < sigma/U + rc/2
//   PDC:  contact needs r0 < sigma_x, Winf = sigma_x c / r0_chk with r0_chk >= r0
//         (c = kobs/kdif)                                     -> r0 < max(sigma_x, sigma_x c / U)
// with a relative and absolute safety margin for rounding.
__device__ __forceinline__ double r_acc(const IrtConst& C, int ri, double U) {
    double s = C.acc_s[ri];
    double R = fmax(s, s * C.acc_c[ri] / U) + C.acc_add[ri];
    return R * (1.0 + 1e-6) + 1e-6;
}

// event heap on (t, packed a<<16|b); nodes [0, HS) in shared memory, the rest in global memory
constexpr uint32_t HS = 512;
struct Heap {
    double* st; uint32_t* sab; double* gt; uint32_t* gab;
    __device__ __forceinline__ double t(uint32_t k) const { return k < HS ? st[k] : gt[k - HS]; }
    __device__ __forceinline__ uint32_t ab(uint32_t k) const { return k < HS ? sab[k] : gab[k - HS]; }
    __device__ __forceinline__ void set(uint32_t k, double tv, uint32_t abv) const {
        if (k < HS) { st[k] = tv; sab[k] = abv; } else { gt[k - HS] = tv; gab[k - HS] = abv; }
    }
};
__device__ __forceinline__ bool ev_less(double t1, uint32_t x, double t2, uint32_t y) {
    return t1 != t2 ? t1 < t2 : x < y;
}
__device__ void heap_push(const Heap& H, uint32_t& n, double t, uint32_t ab) {
    uint32_t c = n++;
    while (c > 0) {
        uint32_t p = (c - 1) >> 1;
        double tp = H.t(p);
        uint32_t ap = H.ab(p);
        if (!ev_less(t, ab, tp, ap)) break;
        H.set(c, tp, ap);
        c = p;
    }
    H.set(c, t, ab);
}
__device__ void heap_pop(const Heap& H, uint32_t& n) {
    n--;
    if (n == 0) return;
    double tp = H.t(n);
    uint32_t ap = H.ab(n);
    uint32_t p = 0;
    for (;;) {
        uint32_t l = 2 * p + 1;
        if (l >= n) break;
        uint32_t s = l;
        double ts = H.t(l);
        uint32_t as = H.ab(l);
        if (l + 1 < n) {
            double tr = H.t(l + 1);
            uint32_t ar = H.ab(l + 1);
            if (ev_less(tr, ar, ts, as)) { s = l + 1; ts = tr; as = ar; }
        }
        if (!ev_less(ts, as, tp, ap)) break;
        H.set(p, ts, as);
        p = s;
    }
    H.set(p, tp, ap);
}

constexpr uint32_t FULL = 0xffffffffu;
// checkpoint times of the reference timeline (:566-580), ns
__constant__ double c_cp[7] = {0.001, 0.01, 0.1, 1, 10, 100, 1000};

// Per-track storage (one track = one primary): particle slots at
// tbase(p) = 2*seg_off[p] + 64*p with capacity 2*len + 64 (len = the track's
// rad_buf entries; a track that outgrows it before the reference's CAP sets
// DERR_TRACK_SIZE), initial-event slots at ebase(p) = 16*seg_off[p] + 2048*p:
// up to ecap(p) = 8*len + 1024 events (DERR_HEAP beyond), twice that room for
// the power-of-two padding of the sort.
__device__ __forceinline__ unsigned long long tbase(const IArgs& A, uint32_t p) { return 2ull * A.seg_off[p] + 64ull * p; }
__device__ __forceinline__ uint32_t tcap(const IArgs& A, uint32_t p) { return (uint32_t)(2ull * (A.seg_off[p + 1] - A.seg_off[p]) + 64ull); }
__device__ __forceinline__ unsigned long long ebase(const IArgs& A, uint32_t p) { return 16ull * A.seg_off[p] + 2048ull * p; }
__device__ __forceinline__ uint32_t ecap(const IArgs& A, uint32_t p) { return (uint32_t)(8ull * (A.seg_off[p + 1] - A.seg_off[p]) + 1024ull); }

__device__ __forceinline__ void load_consts(IrtConst* dst, uint32_t* row) {
    for (int k = threadIdx.x; k < (int)(sizeof(IrtConst) / 4); k += blockDim.x)
        reinterpret_cast<uint32_t*>(dst)[k] = reinterpret_cast<const uint32_t*>(&c_irt)[k];
    __syncthreads();
    if (threadIdx.x < 6) {
        uint32_t r = 0;             // reaction index of (s, q) in 4-bit fields, 15 = none
        for (int q = 5; q >= 0; --q) r = (r << 4) | (uint32_t)(dst->map[threadIdx.x * 6 + q] & 15);
        row[threadIdx.x] = r;
    }
    __syncthreads();
}

// 1) load + thermalisation displacement (:475-537) and species lists; one warp per track
__global__ void __launch_bounds__(IB) k_irt_load(IArgs A) {
    __shared__ IrtConst s_c;
    __shared__ uint32_t s_row[6];
    load_consts(&s_c, s_row);
    const IrtConst& C = s_c;
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const uint32_t k0 = A.k0, k1 = A.k1;
    unsigned long long n_tracks = 0, n_part = 0;
    for (;;) {
        uint32_t p = 0;
        if (lane == 0) p = atomicAdd(&A.counters[0], 1u);
        p = __shfl_sync(FULL, p, 0);
        if (p >= A.nseg) break;
        unsigned long long s = A.seg_off[p], e = A.seg_off[p + 1];
        const uint32_t pid = A.pid_base + p;
        const uint32_t cap = tcap(A, p);
        const unsigned long long tb0 = tbase(A, p);
        double* px = A.px + tb0; double* py = A.py + tb0; double* pz = A.pz + tb0; double* tb = A.tb + tb0;
        int8_t* sp = A.sp + tb0; uint8_t* alive = A.alive + tb0;
        uint16_t* lst = A.lst + 6 * tb0; uint16_t* lpos = A.lpos + tb0;
        uint32_t n = 0, h2 = 0;
        float4* pf = A.pf + tb0;
        // origin of the track's f32 shadow coordinates: its first rad_buf entry
        const float4 r0 = A.rad[s];
        const double ox = r0.x, oy = r0.y, oz = r0.z;
        float mext = 0.0f;
        for (unsigned long long c = s; c < e; c += 32) {
            unsigned long long idx = c + lane;
            bool valid = idx < e;
            int code = -1;
            float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
            if (valid) { r = A.rad[idx]; code = (int)rintf(r.w) % 8; }
            bool keep = valid && code >= 0 && code != 4 && code != 7;
            h2 += __popc(__ballot_sync(FULL, valid && code == 7));
            unsigned m = __ballot_sync(FULL, keep);
            uint32_t k = n + __popc(m & lt);
            if (keep) {
                double x = r.x, y = r.y, z = r.z;
                int spc = code;
                double sigma = 0;
                int disp = 0;
                uint32_t blk = 0, wi = 4;
                u4 wb = {0, 0, 0, 0};
                auto nextd = [&]() -> double {
                    if (wi == 4) { wb = philox(blk++, k, pid, 2u, k0, k1); wi = 0; }
                    uint32_t a_ = wi == 0 ? wb.x : wb.z;
                    uint32_t b_ = wi == 0 ? wb.y : wb.w;
                    wi += 2;
                    return u01d(a_, b_);
                };
                if (code == 5) spc = 1;
                else if (code == 0 || code == 3) { if (nextd() < 0.5) { disp = 1; sigma = C.sig_oh; } }
                else if (code == 1) { disp = 1; sigma = C.sig_eaq; }
                else if (code == 2) { disp = 1; sigma = C.sig_h; }
                else if (code == 6) spc = 5;
                if (disp) {
                    double c6[3];
                    for (int ax = 0; ax < 3; ++ax) {
                        double r1 = nextd(), r2 = nextd(), r3 = nextd(), r4 = nextd(), r5 = nextd(), r6 = nextd();
                        c6[ax] = (r1 + r2 + r3 + r4 + r5 + r6 - 3) * 1.4142135623730951;
                    }
                    x += sigma * c6[0]; y += sigma * c6[1]; z += sigma * c6[2];
                }
                px[k] = x; py[k] = y; pz[k] = z; tb[k] = 0.0;
                sp[k] = (int8_t)spc; alive[k] = 1;
                float fx = (float)(x - ox), fy = (float)(y - oy), fz = (float)(z - oz);
                pf[k] = make_float4(fx, fy, fz, __int_as_float(spc));
                mext = fmaxf(mext, fmaxf(fabsf(fx), fmaxf(fabsf(fy), fabsf(fz))));
            }
            n += __popc(m);
        }
        for (int o = 16; o; o >>= 1) mext = fmaxf(mext, __shfl_xor_sync(FULL, mext, o));
        __syncwarp();
        __threadfence_block();
        uint32_t cnt[6] = {0, 0, 0, 0, 0, 0};
        float4* rec = A.rec + 6 * tb0;
        for (uint32_t c = 0; c < n; c += 32) {
            uint32_t k = c + lane;
            int spc = k < n ? sp[k] : -1;
            float4 sh = make_float4(0.f, 0.f, 0.f, 0.f);
            if (k < n) { sh = pf[k]; sh.w = 0.0f; }               // shadow and birth time 0
            for (int q = 0; q < 6; ++q) {
                unsigned m = __ballot_sync(FULL, spc == q);
                if (spc == q) {
                    uint32_t at = cnt[q] + __popc(m & lt);
                    lst[q * cap + at] = (uint16_t)k;
                    rec[q * cap + at] = sh;
                    lpos[k] = (uint16_t)at;
                }
                cnt[q] += __popc(m);
            }
        }
        if (lane < 6) A.tlc[6 * p + lane] = cnt[lane];
        if (lane == 0) {
            A.tn[p] = n;
            A.th2[p] = h2;
            // |f32 shadow distance - f64 distance| <= 3.1e-7 * extent; 1e-6 * extent + 1e-4 nm bounds it
            A.tdel[p] = mext * 1e-6f + 1e-4f;
            A.ttiles[p] = (n + 31) / 32;
            A.tev[p] = 0;
        }
        if (n) { n_tracks++; n_part += n; }
        if (lane == 0 && n) atomicMax(&A.counters[3], n);
    }
    if (lane == 0 && n_tracks) { atomicAdd(&A.acc[12], n_tracks); atomicAdd(&A.acc[13], n_part); }
}

// Cheap test that a pair may pass the exact acceptance-radius test r2 <= R^2
// of r_acc: f32 shadow distance r2f (error below del), acceptance word w
// with U = (w + 0.5) / 2^32 >= Uf.  Never false when the exact test is true:
//   R = max(s, s c / U) + add  (times 1 + 1e-6, plus 1e-6), so either
//   rf <= (s + add)(1+1e-6) + 1e-6 + del, or (rf - kb) U <= s c (1+1e-6)^2
//   with kb = add (1+1e-6) + 1e-6 + del, which holds for Uf <= U as well;
// both are squared, with a 1e-4 relative margin for the f32 arithmetic.
__device__ __forceinline__ bool pair_maybe(const IrtConst& C, int ri, float r2f, float del, uint32_t w) {
    float ta = (C.fa0[ri] + del) * 1.000001f;
    if (r2f <= ta * ta * 1.0001f) return true;
    float uf = __uint2float_rd(w) * 2.3283064365386963e-10f;
    float kb = (C.fkb0[ri] + del) * 1.000001f;
    float rhs = fmaf(kb, uf, C.fk[ri]);
    return r2f * uf * uf <= rhs * rhs * 1.0001f;
}

__device__ __forceinline__ u4 philox_accept(uint32_t blk, uint32_t i, uint32_t pid, const uint32_t* rk) {
    return philox_rk(blk, i, pid, 3u, rk);
}

// 2) initial pairing (:539-558): one warp per (track, tile of 32 particles).
//    The tile's particles sit in lane registers as f32 shadows; partners come
//    32 at a time through shared memory and are read as broadcasts.  The f32
//    distance settles the R_CUT test and the acceptance prefilter for almost
//    every pair; the rare candidates (and pairs within rounding of R_CUT) are
//    queued per warp and redone exactly in f64, 32 at a time, one per lane.
constexpr int IQ = 64;                   // candidate queue per warp

struct InitTrack {
    const double *px, *py, *pz;
    double* ET;
    uint32_t* EAB;
    uint32_t* tev;
    uint32_t ecp, pid;
};

// exact evaluation of queued candidates [0, cnt): one per lane; returns the
// reactive pairs inside R_CUT found among the near-R_CUT entries
__device__ __forceinline__ uint32_t init_batch(const IrtConst& C, const InitTrack& T, const uint32_t* qij,
                                               const uint32_t* qw, const uint16_t* qk, int cnt, int lane,
                                               uint32_t k0, uint32_t k1, bool& ev_over) {
    const unsigned lt = (1u << lane) - 1u;
    bool acc = false, pdcq = false;
    double t = 0, pa = 0, pb = 0, pD = 0;
    uint32_t i = 0, j = 0, np = 0;
    if (lane < cnt) {
        const uint32_t ij = qij[lane], k = qk[lane];
        uint32_t wd = qw[lane];
        i = ij >> 16; j = ij & 0xffffu;
        const int kind = (int)(k & 3u), ri = (int)((k >> 2) & 15u);
        const int si = (int)((k >> 6) & 7u), sj = (int)((k >> 9) & 7u);
        double dx = T.px[i] - T.px[j], dy = T.py[i] - T.py[j], dz = T.pz[i] - T.pz[j];
        double r2 = dx * dx + dy * dy + dz * dz;
        bool inside = true;
        if (kind == 2) {
            inside = r2 <= C.r_cut2;
            if (inside) {
                np = 1;
                u4 w4 = philox(j >> 2, i, T.pid, 3u, k0, k1);
                wd = (j & 3) == 0 ? w4.x : (j & 3) == 1 ? w4.y : (j & 3) == 2 ? w4.z : w4.w;
            }
        }
        if (inside) {
            double U = u01d32(wd);
            double R = r_acc(C, ri, U);
            if (r2 <= R * R) {
                double D = C.D[si] + C.D[sj];
                t = sample_pre(C, sqrt(r2), ri, D, U, &pa, &pb);
                if (t == -2.0) { pdcq = true; pD = D; }
                else acc = (t >= 0 && t < 1000);
            }
        }
    }
    unsigned pm = __ballot_sync(FULL, pdcq);
    while (pm) {
        int src = __ffs(pm) - 1;
        pm &= pm - 1;
        uint32_t qi = __shfl_sync(FULL, i, src), qj = __shfl_sync(FULL, j, src);
        double qa = __shfl_sync(FULL, pa, src), qb = __shfl_sync(FULL, pb, src);
        double X = pdc_warp(qi, qj, T.pid, k0, k1, qa, qb, lane);
        if (lane == src && X > 0) { t = X / pD; acc = t < 1000; }
    }
    unsigned m = __ballot_sync(FULL, acc);
    if (m) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(T.tev, (uint32_t)__popc(m));
        base = __shfl_sync(FULL, base, 0);
        uint32_t slot = base + __popc(m & lt);
        if (acc) {
            if (slot < T.ecp) { T.ET[slot] = t; T.EAB[slot] = (i << 16) | j; }
            else ev_over = true;
        }
    }
    return np;
}

// One out-of-line copy of the exact evaluation for the pairing kernel's two
// call sites (measured faster than two inlined copies: less code and fewer
// spills in the partner loop).
struct IbOut { uint32_t np; uint32_t over; };
__device__ __noinline__ IbOut init_batch_nc(const IrtConst& C, InitTrack T, const uint32_t* qij, const uint32_t* qw,
                                            const uint16_t* qk, int cnt, int lane, uint32_t k0, uint32_t k1) {
    bool over = false;
    const uint32_t np = init_batch(C, T, qij, qw, qk, cnt, lane, k0, k1, over);
    return IbOut{np, over ? 1u : 0u};
}

#ifndef WG_INIT_MINB
#define WG_INIT_MINB 7
#endif
__global__ void __launch_bounds__(IB, WG_INIT_MINB) k_irt_init(IArgs A) {
    __shared__ IrtConst s_c;
    __shared__ uint32_t s_row[6];
    __shared__ float4 s_pj[IB / 32][32];
    __shared__ uint32_t s_qij[IB / 32][IQ], s_qw[IB / 32][IQ];
    __shared__ uint16_t s_qk[IB / 32][IQ];
    load_consts(&s_c, s_row);
    const IrtConst& C = s_c;
    const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const unsigned long long nitems = A.toff[A.nseg];
    const float rcut = (float)sqrt(C.r_cut2);
    const uint32_t k0 = A.k0, k1 = A.k1;
    uint32_t* qij = s_qij[wl];
    uint32_t* qw = s_qw[wl];
    uint16_t* qk = s_qk[wl];
    unsigned long long n_pairs = 0;
    bool ev_over = false;
    for (;;) {
        unsigned long long item = 0;
        if (lane == 0) item = atomicAdd(&A.counters[1], 1u);
        item = __shfl_sync(FULL, item, 0);
        if (item >= nitems) break;
        uint32_t lo = 0, hi = A.nseg;                 // last p with toff[p] <= item
        while (hi - lo > 1) { uint32_t mid = (lo + hi) >> 1; if (A.toff[mid] <= item) lo = mid; else hi = mid; }
        const uint32_t p = lo;
        const uint32_t n = A.tn[p];
        const uint32_t i0 = 32u * (uint32_t)(item - A.toff[p]);
        const unsigned long long tb0 = tbase(A, p);
        const float4* pf = A.pf + tb0;
        const float del = A.tdel[p];
        const float clo = (rcut - del) * 0.99999f, chi = (rcut + del) * 1.00001f;
        const float lo2 = clo * clo, hi2 = chi * chi;
        InitTrack T{A.px + tb0, A.py + tb0, A.pz + tb0, A.ev_t + ebase(A, p), A.ev_ab + ebase(A, p), &A.tev[p],
                    ecap(A, p), A.pid_base + p};
        const uint32_t i = i0 + lane;
        const bool hi_ = i < n;
        float4 me = make_float4(0.f, 0.f, 0.f, 0.f);
        if (hi_) me = pf[i];
        const int si = hi_ ? __float_as_int(me.w) : 0;
        const uint32_t row = s_row[si];
        int qn = 0;
        for (uint32_t j0 = i0; j0 < n; j0 += 32) {
            __syncwarp();
            if (j0 + lane < n) s_pj[wl][lane] = pf[j0 + lane];
            __syncwarp();
            const uint32_t kmax = min(32u, n - j0);
            // partners in groups of 4 = one Philox block of acceptance words
            // (j0 is a multiple of 32): 4 distances, at most one Philox call
            for (uint32_t kk = 0; kk < kmax; kk += 4) {
                float r2[4];
                int rr[4], sv[4];
                bool ok[4];
                bool need = false;
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const uint32_t j = j0 + kk + u;
                    const float4 q = s_pj[wl][kk + u];
                    const bool in = kk + u < kmax;
                    sv[u] = in ? __float_as_int(q.w) : 0;
                    rr[u] = (int)((row >> (4 * sv[u])) & 15u);
                    ok[u] = in && hi_ && j > i && rr[u] != 15;
                    const float dx = me.x - q.x, dy = me.y - q.y, dz = me.z - q.z;
                    r2[u] = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                    need |= ok[u] && r2[u] < lo2;
                }
                u4 cw = {0, 0, 0, 0};
                if (need) cw = philox_accept((j0 + kk) >> 2, i, T.pid, A.rk);
                int kind[4];                            // 1: candidate, 2: near R_CUT
                bool any = false;
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const uint32_t wd = u == 0 ? cw.x : u == 1 ? cw.y : u == 2 ? cw.z : cw.w;
                    kind[u] = 0;
                    if (ok[u]) {
                        if (r2[u] < lo2) {
                            n_pairs++;
                            if (pair_maybe(C, rr[u], r2[u], del, wd)) kind[u] = 1;
                        } else if (r2[u] <= hi2) kind[u] = 2;
                    }
                    any |= kind[u] != 0;
                }
                if (!__any_sync(FULL, any)) continue;
                // queue entries of the four partners, 12 bits each (kind | rr << 2 | sv << 6);
                // the queueing loop is kept rolled (one copy of its code, fewer spills:
                // measured faster than four unrolled copies)
                uint64_t pk = 0;
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    pk |= (uint64_t)((uint32_t)kind[u] | ((uint32_t)rr[u] << 2) | ((uint32_t)sv[u] << 6)) << (12 * u);
#pragma unroll 1
                for (int u = 0; u < 4; ++u) {
                    const uint32_t f = (uint32_t)(pk >> (12 * u)) & 0xfffu;
                    const unsigned m = __ballot_sync(FULL, (f & 3u) != 0u);
                    if (!m) continue;
                    if (f & 3u) {
                        const int at = qn + __popc(m & lt);
                        qij[at] = (i << 16) | (j0 + kk + u);
                        qw[at] = u == 0 ? cw.x : u == 1 ? cw.y : u == 2 ? cw.z : cw.w;
                        qk[at] = (uint16_t)((f & 3u) | (((f >> 2) & 15u) << 2) | (si << 6) | ((f >> 6) << 9));
                    }
                    qn += __popc(m);
                    if (qn >= 32) {
                        __syncwarp();
                        const IbOut o = init_batch_nc(C, T, qij, qw, qk, 32, lane, k0, k1);
                        n_pairs += o.np;
                        ev_over |= o.over != 0u;
                        __syncwarp();
                        if (lane < qn - 32) { qij[lane] = qij[32 + lane]; qw[lane] = qw[32 + lane]; qk[lane] = qk[32 + lane]; }
                        qn -= 32;
                        __syncwarp();
                    }
                }
            }
        }
        if (qn) {
            __syncwarp();
            const IbOut o = init_batch_nc(C, T, qij, qw, qk, qn, lane, k0, k1);
            n_pairs += o.np;
            ev_over |= o.over != 0u;
            __syncwarp();
        }
    }
    if (__any_sync(FULL, ev_over) && lane == 0) atomicOr(A.err, DERR_HEAP);
    for (int o = 16; o; o >>= 1) n_pairs += __shfl_xor_sync(FULL, n_pairs, o);
    if (lane == 0 && n_pairs) atomicAdd(&A.acc[10], n_pairs);
}

__device__ __forceinline__ u4 philox_pair(uint32_t id, uint32_t jj, uint32_t pid, uint32_t k0, uint32_t k1) {
    return philox(id, jj, pid, 5u, k0, k1);
}
__device__ __forceinline__ u4 philox_pair_ang(uint32_t id, uint32_t jj, uint32_t pid, uint32_t k0, uint32_t k1) {
    return philox(id, jj, pid, 5u | (1u << 4), k0, k1);
}

__device__ __noinline__ double gauss_axis(uint32_t wa, uint32_t wb) {
    return sqrt(-2 * log_(u01d32(wa) + 1e-30)) * cos_(6.2831853 * u01d32(wb));
}

// the product being re-paired (uniform over the warp); its position and
// birth time are read back from its slot when a batch needs them
struct ProdCtx {
    const double *px, *py, *pz, *tb;
    double Di;
    uint32_t id, pid, k0, k1;
};

// Exact pairWithAlive step (:430-465) for queued partners [0, cnt), one per
// lane: Brownian sync of the partner by sqrt(2 D_j dt) (skipped when the
// Box-Muller radius bound shows it cannot come within r_acc), R_CUT, then
// sampleIRT; accepted events go to the warp's heap.  Returns true when the
// heap overflowed.
__device__ __forceinline__ bool prod_batch(const IrtConst& C, const ProdCtx& P, const uint32_t* pq, int cnt, int lane,
                                        const Heap& H, uint32_t& hn, uint32_t hcap) {
    bool acc = false, pdcq = false, over = false;
    double ta = 0, pa = 0, pb = 0, pD = 0;
    uint32_t jj = 0;
    const double pnx = P.px[P.id], pny = P.py[P.id], pnz = P.pz[P.id], pet = P.tb[P.id];
    if (lane < cnt) {
        const uint32_t e = pq[lane];
        jj = e & 0xffffu;
        const int r2i = (int)((e >> 16) & 15u), s2 = (int)(e >> 20);
        const double Dj = C.D[s2];
        const double dt = pet - P.tb[jj];
        double xj = P.px[jj], yj = P.py[jj], zj = P.pz[jj];
        const u4 q0 = philox(P.id, jj, P.pid, 5u, P.k0, P.k1);
        const double U = u01d32(q0.w);
        const double R = r_acc(C, r2i, U);
        bool need = true;
        if (dt > 0) {
            double sig = sqrt(2.0 * Dj * dt);
            // |gaussian 3-vector| <= sqrt(sum -2 ln u1_k) (Box-Muller radius), with margin
            float l0 = -2.0f * __logf(u01f32(q0.x));
            float l1 = -2.0f * __logf(u01f32(q0.y));
            float l2 = -2.0f * __logf(u01f32(q0.z));
            double B = (double)sqrtf((l0 + l1 + l2) * 1.0001f) + 1e-4;
            double ex = pnx - xj, ey = pny - yj, ez = pnz - zj;
            double dist = sqrt(ex * ex + ey * ey + ez * ez);
            if (dist - sig * B > R) need = false;
            if (need) {
                u4 q1 = philox(P.id, jj, P.pid, 5u | (1u << 4), P.k0, P.k1);
                double g0 = gauss_axis(q0.x, q1.x);
                double g1 = gauss_axis(q0.y, q1.y);
                double g2 = gauss_axis(q0.z, q1.z);
                xj += g0 * sig; yj += g1 * sig; zj += g2 * sig;
            }
        }
        if (need) {
            double dx = pnx - xj, dy = pny - yj, dz = pnz - zj;
            double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 <= C.r_cut2) {
                double D = P.Di + Dj;
                double t = sample_pre(C, sqrt(r2), r2i, D, U, &pa, &pb);
                if (t == -2.0) { pdcq = true; pD = D; }
                else if (t >= 0) { ta = pet + t; acc = ta < 1000; }
            }
        }
    }
    unsigned pm = __ballot_sync(FULL, pdcq);
    while (pm) {
        int src = __ffs(pm) - 1;
        pm &= pm - 1;
        uint32_t qj = __shfl_sync(FULL, jj, src);
        double qa = __shfl_sync(FULL, pa, src), qb = __shfl_sync(FULL, pb, src);
        double X = pdc_warp(P.id, qj, P.pid, P.k0, P.k1, qa, qb, lane);
        if (lane == src && X > 0) { ta = pet + X / pD; acc = ta < 1000; }
    }
    unsigned m = __ballot_sync(FULL, acc);
    while (m) {
        int src = __ffs(m) - 1;
        m &= m - 1;
        double tt = __shfl_sync(FULL, ta, src);
        uint32_t pj = __shfl_sync(FULL, jj, src);
        if (lane == 0) {
            if (hn < HS + hcap) {
                uint32_t a = pj < P.id ? pj : P.id, bq = pj < P.id ? P.id : pj;
                heap_push(H, hn, tt, (a << 16) | bq);
            } else over = true;
        }
    }
    hn = __shfl_sync(FULL, hn, 0);
    return __any_sync(FULL, over);
}

// 3) the initial events of each track in (t, i, j) order (:566): a block-wide
//     bitonic sort, in shared memory up to SORT_SM events (padded to a power
//     of two), in the track's own event slots beyond that (they hold 2 ecap).
//     Keys are unique, so the order is that of any other sort.
constexpr int SB = 256;
constexpr uint32_t SORT_SM = 4096;
__global__ void __launch_bounds__(SB) k_irt_sort(IArgs A) {
    __shared__ double st[SORT_SM];
    __shared__ uint32_t sab[SORT_SM];
    for (uint32_t k = blockIdx.x; k < A.nseg; k += gridDim.x) {
        const uint32_t p = A.order[k];                 // largest tracks first
        const uint32_t nev = A.tev[p];
        if (nev < 2 || nev > ecap(A, p)) continue;     // the event kernel reports the overflow
        double* T = A.ev_t + ebase(A, p);
        uint32_t* AB = A.ev_ab + ebase(A, p);
        uint32_t n2 = 2;
        while (n2 < nev) n2 <<= 1;
        const bool sm = n2 <= SORT_SM;
        double* t = sm ? st : T;
        uint32_t* ab = sm ? sab : AB;
        __syncthreads();                               // the previous track is written back
        for (uint32_t i = threadIdx.x; i < n2; i += SB) {
            if (i >= nev) { t[i] = 1e300; ab[i] = 0xffffffffu; }
            else if (sm) { st[i] = T[i]; sab[i] = AB[i]; }
        }
        __syncthreads();
        for (uint32_t kk = 2; kk <= n2; kk <<= 1) {
            for (uint32_t j = kk >> 1; j > 0; j >>= 1) {
                for (uint32_t q = threadIdx.x; q < (n2 >> 1); q += SB) {
                    const uint32_t i = ((q & ~(j - 1)) << 1) | (q & (j - 1)), l = i | j;   // bit j of i clear
                    const double ti = t[i], tl = t[l];
                    const uint32_t ai = ab[i], al = ab[l];
                    if (ev_less(tl, al, ti, ai) == ((i & kk) == 0)) { t[i] = tl; t[l] = ti; ab[i] = al; ab[l] = ai; }
                }
                __syncthreads();
            }
        }
        if (sm)
            for (uint32_t i = threadIdx.x; i < nev; i += SB) { T[i] = st[i]; AB[i] = sab[i]; }
    }
}

// 4) events (:566-660): pop the sorted initial events in (t, i, j) order
//    merged with a heap of product events; one warp per track
#ifndef WG_LOOP_MINB
#define WG_LOOP_MINB 4
#endif
__global__ void __launch_bounds__(IB, WG_LOOP_MINB) k_irt_loop(IArgs A) {
    __shared__ double s_tl[IB / 32][35];
    __shared__ double s_ht[IB / 32][HS];
    __shared__ uint32_t s_hab[IB / 32][HS];
    __shared__ int s_lc[IB / 32][6];
    __shared__ uint32_t s_pq[IB / 32][IQ];
    __shared__ IrtConst s_c;
    __shared__ uint32_t s_row[6];
    load_consts(&s_c, s_row);
    const IrtConst& C = s_c;
    const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
    const uint32_t gw = blockIdx.x * (IB / 32) + wl;
    uint32_t* pq = s_pq[wl];
    // CAP of the reference worker (:405): twice the largest track's species, plus 512
    const uint32_t capref = 2u * A.counters[3] + 512u;
    const uint32_t k0 = A.k0, k1 = A.k1;
    for (int k = lane; k < 35; k += 32) s_tl[wl][k] = 0.0;
    int* lc = s_lc[wl];
    Heap H{s_ht[wl], s_hab[wl], A.hov_t + (size_t)gw * A.hcap, A.hov_ab + (size_t)gw * A.hcap};
    // per-warp tallies in shared memory (lane 0): reactions 0..8, reacted, events, initial events
    __shared__ unsigned long long s_cnt[IB / 32][12];
    unsigned long long* tally = s_cnt[wl];
    for (int k = lane; k < 12; k += 32) tally[k] = 0;
    unsigned long long n_pairs = 0;
    __syncwarp();
    for (;;) {
        uint32_t k = 0;
        if (lane == 0) k = atomicAdd(&A.counters[2], 1u);
        k = __shfl_sync(FULL, k, 0);
        if (k >= A.nseg) break;
        const uint32_t p = A.order[k];                 // largest tracks first
        const uint32_t n = A.tn[p];
        if (n == 0) continue;
        const uint32_t pid = A.pid_base + p;
        const uint32_t cap = tcap(A, p);
        const unsigned long long tb0 = tbase(A, p);
        double* px = A.px + tb0; double* py = A.py + tb0; double* pz = A.pz + tb0; double* tb = A.tb + tb0;
        int8_t* sp = A.sp + tb0; uint8_t* alive = A.alive + tb0;
        uint16_t* lst = A.lst + 6 * tb0; uint16_t* lpos = A.lpos + tb0;
        float4* rec = A.rec + 6 * tb0;
        double* ET = A.ev_t + ebase(A, p);
        uint32_t* EAB = A.ev_ab + ebase(A, p);
        const uint32_t nev = A.tev[p];
        const float del = A.tdel[p];
        const float4 org = A.rad[A.seg_off[p]];
        const double ox = org.x, oy = org.y, oz = org.z;
        if (lane < 6) lc[lane] = (int)A.tlc[6 * p + lane];     // alive species of each kind
        if (nev > ecap(A, p)) { if (lane == 0) atomicOr(A.err, DERR_HEAP); continue; }
        if (lane == 0) tally[11] += nev;
        __syncwarp();
        uint32_t ip = 0, hn = 0;
        uint32_t ntot = n;
        double h2c = (double)A.th2[p];
        int cp = 0, c16 = 0;
        float* curve = A.curves ? A.curves + 80ull * p : nullptr;
        bool heap_over = false;
        for (;;) {
            double et = 0;
            uint32_t eab = 0;
            int have = 0, si = 0, sj = 0, ri = -1;
            if (lane == 0) {
                // pop until a reaction with products: stale events and reactions
                // without products change nothing the other lanes work on
                for (;;) {
                    const bool hi_ = ip < nev, hh = hn > 0;
                    if (!hi_ && !hh) break;
                    double ti = hi_ ? ET[ip] : 0.0, th = hh ? H.t(0) : 0.0;
                    uint32_t ai = hi_ ? EAB[ip] : 0u, ah = hh ? H.ab(0) : 0u;
                    if (hi_ && (!hh || ev_less(ti, ai, th, ah))) { et = ti; eab = ai; ip++; }
                    else { et = th; eab = ah; heap_pop(H, hn); }
                    tally[10]++;
                    while (cp < 7 && et >= c_cp[cp]) {
                        s_tl[wl][cp * 5 + 0] += lc[0]; s_tl[wl][cp * 5 + 1] += lc[1];
                        s_tl[wl][cp * 5 + 2] += lc[2]; s_tl[wl][cp * 5 + 3] += lc[4];
                        s_tl[wl][cp * 5 + 4] += h2c;
                        cp++;
                    }
                    while (curve && c16 < 16 && et >= C.t16[c16]) {
                        float* c = curve + 5 * c16;
                        c[0] = (float)lc[0]; c[1] = (float)lc[1]; c[2] = (float)lc[2]; c[3] = (float)lc[4];
                        c[4] = (float)h2c;
                        c16++;
                    }
                    const int ei = (int)(eab >> 16), ej = (int)(eab & 0xffffu);
                    if (!(alive[ei] && alive[ej])) continue;
                    const int a = sp[ei], b2 = sp[ej];
                    const int r = C.map[(a < b2 ? a : b2) * 6 + (a < b2 ? b2 : a)];
                    if (r < 0) continue;
                    alive[ei] = 0; alive[ej] = 0;
                    // rolled: one copy of the list update (fewer spills in the event kernel)
#pragma unroll 1
                    for (int w2 = 0; w2 < 2; ++w2) {
                        int k = w2 == 0 ? ei : ej, q = w2 == 0 ? a : b2;
                        uint32_t at = lpos[k];
                        uint16_t last = lst[q * cap + lc[q] - 1];
                        lst[q * cap + at] = last;
                        rec[q * cap + at] = rec[q * cap + lc[q] - 1];
                        lpos[last] = (uint16_t)at;
                        lc[q]--;
                    }
                    tally[9]++;
                    tally[r]++;
                    if (r == 3 || r == 4 || r == 6) h2c += 1;
                    if (C.nprod[r] == 0) continue;
                    have = 1; si = a; sj = b2; ri = r;
                    break;
                }
            }
            if (!__shfl_sync(FULL, have, 0)) break;
            et = __shfl_sync(FULL, et, 0);
            eab = __shfl_sync(FULL, eab, 0);
            const int ei = (int)(eab >> 16), ej = (int)(eab & 0xffffu);
            si = __shfl_sync(FULL, si, 0);
            sj = __shfl_sync(FULL, sj, 0);
            ri = __shfl_sync(FULL, ri, 0);
            const int np_ = C.nprod[ri];
            for (int pp = 0; pp < np_; ++pp) {
                int nsp = pp == 0 ? C.prod0[ri] : C.prod1[ri];
                uint32_t id = ntot;
                if (id >= capref) break;                 // the reference's CAP (:405, :621)
                if (id >= cap) { if (lane == 0) atomicOr(A.err, DERR_TRACK_SIZE); break; }
                double nx, ny, nz;
                if (np_ == 1) {                          // at the diffusion-weighted centre
                    const double sqDi = sqrt(C.D[si]), sqDj = sqrt(C.D[sj]);
                    const double ww = sqDi + sqDj;
                    const double xa = px[ei], ya = py[ei], za = pz[ei];
                    const double xb = px[ej], yb = py[ej], zb = pz[ej];
                    nx = (sqDj * xa + sqDi * xb) / ww;
                    ny = (sqDj * ya + sqDi * yb) / ww;
                    nz = (sqDj * za + sqDi * zb) / ww;
                } else {                                 // at the two reactants
                    const int e = pp == 0 ? ei : ej;
                    nx = px[e]; ny = py[e]; nz = pz[e];
                }
                const float nsx = (float)(nx - ox), nsy = (float)(ny - oy), nsz = (float)(nz - oz);
                if (lane == 0) {
                    px[id] = nx; py[id] = ny; pz[id] = nz; tb[id] = et;
                    sp[id] = (int8_t)nsp; alive[id] = 1;
                    lst[nsp * cap + lc[nsp]] = (uint16_t)id;
                    rec[nsp * cap + lc[nsp]] = make_float4(nsx, nsy, nsz, (float)et);
                    lpos[id] = (uint16_t)lc[nsp];
                    lc[nsp]++;
                }
                ntot++;
                __syncwarp();
                __threadfence_block();
                // pairWithAlive (:430-465) over the alive particles of the species that react with nsp.
                // f32 prefilter per partner; the partners it cannot rule out are queued and
                // evaluated exactly (ProdPair), 32 at a time, one per lane.
                const double Di = C.D[nsp];
                const uint32_t rowp = s_row[nsp];
                int qn = 0;
                const ProdCtx P{px, py, pz, tb, Di, id, pid, k0, k1};
                const float etf = (float)et, dtm = 1e-4f + 1e-6f * etf;
                const float rcut_hi = (float)sqrt(C.r_cut2) * 1.00001f;
                for (int s2 = 0; s2 < 6; ++s2) {
                    const int r2i = (int)((rowp >> (4 * s2)) & 15u);
                    if (r2i == 15) continue;
                    const uint32_t len = (uint32_t)lc[s2];
                    const float Djf2 = (float)(2.0 * C.D[s2]);
                    const float fs = C.fs[r2i], fsc = C.fsc[r2i], fadd = C.fadd[r2i];
                    const uint16_t* L2 = lst + s2 * cap;
                    const float4* R2 = rec + s2 * cap;
                    // chunks of 32 partners; the next chunk's list entry and record are
                    // loaded before this chunk is tested (the lists do not change here)
                    uint32_t jnext = lane < len ? L2[lane] : 0xffffu;
                    float4 rnext = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (lane < len) rnext = R2[lane];
                    for (uint32_t c0 = 0; c0 < len; c0 += 32) {
                        const uint32_t jj = jnext;
                        const float4 q = rnext;
                        {
                            const uint32_t li = c0 + 32u + lane;
                            jnext = li < len ? L2[li] : 0xffffu;
                            if (li < len) rnext = R2[li];
                        }
                        bool mv = false;
                        {
                            if (jj != 0xffffu && jj != id) {
                                n_pairs++;
                                const float ex = nsx - q.x, ey = nsy - q.y, ez = nsz - q.z;
                                const float dlo = (sqrtf(fmaf(ez, ez, fmaf(ey, ey, ex * ex))) - del) * 0.999998f;
                                // draw-free bound first: the displacement is at most the largest
                                // Box-Muller radius of 32-bit draws (sqrt(3 * 2 ln 2^33) = 11.72)
                                // times sqrt(2 D dt), and a partner beyond R_CUT after it is
                                // rejected by the exact path too
                                const float dth = etf - q.w + dtm;
                                if (dlo - (dth > 0.0f ? sqrtf(Djf2 * dth) * 11.8f : 0.0f) > rcut_hi) goto scored;
                                const u4 q0 = philox_pair(id, jj, pid, k0, k1);
                                // R of r_acc for U >= uf, rounded up
                                const float uf = __uint2float_rd(q0.w) * 2.3283064365386963e-10f;
                                const float rhi = (fmaxf(fs, __fdividef(fsc, uf)) + fadd) * 1.00002f + 1e-6f;
                                // dth: upper bound of dt = et - t_birth from the f32 birth time (error < dtm)
                                float reach = 0.0f, l0 = 0.0f, l1 = 0.0f, l2 = 0.0f, Bf = 0.0f;
                                if (dth > 0.0f) {
                                    l0 = -2.0f * __logf(u01f32(q0.x));
                                    l1 = -2.0f * __logf(u01f32(q0.y));
                                    l2 = -2.0f * __logf(u01f32(q0.z));
                                    Bf = sqrtf((l0 + l1 + l2) * 1.0001f);
                                    reach = sqrtf(Djf2 * dth) * 1.00001f * (Bf + 1e-4f);
                                }
                                mv = !(dlo - reach > rhi);
                                if (mv && dth > 0.0f) {
                                    // second stage: the partner displaced by the same Box-Muller draws in
                                    // f32.  Per axis |g_f - g| <= 2e-3 + 2e-5 |g| (sqrt of the log near 0,
                                    // fast log and cos, 2 ulp each), sigma within [sl, sh].
                                    const u4 q1 = philox_pair_ang(id, jj, pid, k0, k1);
                                    const float dtl = fmaxf(etf - q.w - dtm, 0.0f);
                                    const float sh = sqrtf(Djf2 * dth) * 1.00001f, sl = sqrtf(Djf2 * dtl) * 0.99999f;
                                    const float sm = 0.5f * (sh + sl), Bm = Bf + 1e-4f;
                                    // cos(2 pi u) = -cos(2 pi (u - 1/2)): the argument stays in [-pi, pi]
                                    const float g0 = -sqrtf(l0) * __cosf(6.2831853f * (u01f32(q1.x) - 0.5f));
                                    const float g1 = -sqrtf(l1) * __cosf(6.2831853f * (u01f32(q1.y) - 0.5f));
                                    const float g2 = -sqrtf(l2) * __cosf(6.2831853f * (u01f32(q1.z) - 0.5f));
                                    const float fx = ex - g0 * sm, fy = ey - g1 * sm, fz = ez - g2 * sm;
                                    const float d2 = sqrtf(fmaf(fz, fz, fmaf(fy, fy, fx * fx)));
                                    const float eg = 2e-3f + 2e-5f * Bm;
                                    const float err = 1.7320508f * (sh * eg + 0.5f * (Bm + eg) * (sh - sl)) + del;
                                    mv = !((d2 - err) * 0.99999f > rhi);
                                }
                            }
                        }
                    scored:
                        {
                            const unsigned m = __ballot_sync(FULL, mv);
                            if (m) {
                                if (mv) pq[qn + __popc(m & ((1u << lane) - 1u))] = jj | ((uint32_t)r2i << 16) | ((uint32_t)s2 << 20);
                                qn += __popc(m);
                                if (qn >= 32) {
                                    __syncwarp();
                                    heap_over |= prod_batch(C, P, pq, 32, lane, H, hn, A.hcap);
                                    __syncwarp();
                                    if (lane < qn - 32) pq[lane] = pq[32 + lane];
                                    qn -= 32;
                                    __syncwarp();
                                }
                            }
                        }
                    }
                }
                if (qn) {
                    __syncwarp();
                    heap_over |= prod_batch(C, P, pq, qn, lane, H, hn, A.hcap);
                }
                __syncwarp();
                __threadfence_block();
            }
        }
        if (lane == 0) {
            if (heap_over) atomicOr(A.err, DERR_HEAP);
            while (cp < 7) {
                s_tl[wl][cp * 5 + 0] += lc[0]; s_tl[wl][cp * 5 + 1] += lc[1];
                s_tl[wl][cp * 5 + 2] += lc[2]; s_tl[wl][cp * 5 + 3] += lc[4];
                s_tl[wl][cp * 5 + 4] += h2c;
                cp++;
            }
            while (curve && c16 < 16) {
                float* c = curve + 5 * c16;
                c[0] = (float)lc[0]; c[1] = (float)lc[1]; c[2] = (float)lc[2]; c[3] = (float)lc[4];
                c[4] = (float)h2c;
                c16++;
            }
        }
        __syncwarp();
    }
    for (int o = 16; o; o >>= 1) n_pairs += __shfl_xor_sync(FULL, n_pairs, o);
    __syncwarp();
    if (lane == 0) {
        for (int k = 0; k < 9; ++k) if (tally[k]) atomicAdd(&A.acc[k], tally[k]);
        if (tally[9]) atomicAdd(&A.acc[9], tally[9]);
        if (n_pairs) atomicAdd(&A.acc[10], n_pairs);
        if (tally[10]) atomicAdd(&A.acc[11], tally[10]);
        if (tally[11]) atomicAdd(&A.acc[14], tally[11]);
    }
    for (int k = lane; k < 35; k += 32)
        if (s_tl[wl][k] != 0.0) atomicAdd(&A.acc_tl[k], s_tl[wl][k]);
}

// codes -> grouping keys (pid << 34 | original index) for a caller's rad_buf
__global__ void k_group_keys(const float4* rad, unsigned long long n, unsigned long long* key, uint32_t* maxpid) {
    unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
    uint32_t mp = 0;
    if (i < n) {
        int w = (int)rintf(rad[i].w);
        uint32_t pid = w >= 0 ? (uint32_t)(w / 8) : 0u;
        key[i] = ((unsigned long long)pid << 34) | i;
        mp = pid;
    }
    for (int o = 16; o; o >>= 1) mp = max(mp, __shfl_xor_sync(0xffffffffu, mp, o));
    if ((threadIdx.x & 31) == 0) atomicMax(maxpid, mp);
}

// longest segment
__global__ void k_seg_max(const unsigned long long* off, uint32_t nseg, unsigned long long* out) {
    unsigned long long m = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nseg; i += gridDim.x * blockDim.x)
        m = max(m, off[i + 1] - off[i]);
    for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// ------------------------------------------------------------------ host side
cudaError_t irt_set_constants(const IrtConst& c) { return cudaMemcpyToSymbol(c_irt, &c, sizeof c); }

static int blocks_for(const void* k, int device, uint32_t limit = 0) {
    int sms = 0, per = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, IB, 0);
    if (per < 1) per = 1;
    if (limit && (int)limit < per) per = (int)limit;
    return sms * per;
}

// Order of the event kernel's tracks: by species count, largest first (a
// bucket sort in one block), so the longest event chains start early and the
// last wave holds the short ones.
__global__ void __launch_bounds__(1024) k_track_order(const uint32_t* tn, uint32_t nseg, uint32_t* order) {
    constexpr int NB = 512;
    __shared__ uint32_t cnt[NB], off[NB];
    __shared__ uint32_t smax;
    if (threadIdx.x == 0) smax = 0;
    for (int b = threadIdx.x; b < NB; b += blockDim.x) cnt[b] = 0;
    __syncthreads();
    uint32_t m = 0;
    for (uint32_t p = threadIdx.x; p < nseg; p += blockDim.x) m = max(m, tn[p]);
    atomicMax(&smax, m);
    __syncthreads();
    const uint32_t mx = smax > 0 ? smax : 1;
    for (uint32_t p = threadIdx.x; p < nseg; p += blockDim.x)
        atomicAdd(&cnt[(uint32_t)(((unsigned long long)(mx - min(tn[p], mx)) * (NB - 1)) / mx)], 1u);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t a = 0;
        for (int b = 0; b < NB; ++b) { off[b] = a; a += cnt[b]; }
    }
    __syncthreads();
    for (uint32_t p = threadIdx.x; p < nseg; p += blockDim.x) {
        const uint32_t b = (uint32_t)(((unsigned long long)(mx - min(tn[p], mx)) * (NB - 1)) / mx);
        order[atomicAdd(&off[b], 1u)] = p;
    }
}

int irt_warps(int device, const IrtShape& shape) {
    return blocks_for((const void*)k_irt_loop, device, shape.loop_per_sm) * (IB / 32);
}

// tile prefix: the scan of transport.cu
cudaError_t launch_scan_u32(const uint32_t* cnt, uint32_t n, unsigned long long* off, cudaStream_t s);

// timing events of the launch sequence: inside a stream capture they must be
// external event nodes, which a replay records like a plain cudaEventRecord
static cudaError_t irt_mark(cudaEvent_t e, cudaStream_t s) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t r = cudaStreamIsCapturing(s, &cs);
    if (r != cudaSuccess) return r;
    return cudaEventRecordWithFlags(e, s, cs == cudaStreamCaptureStatusActive ? cudaEventRecordExternal
                                                                              : cudaEventRecordDefault);
}

cudaError_t launch_irt(const IArgs& a, int device, const IrtShape& shape, cudaStream_t s, cudaEvent_t* ev) {
    { cudaError_t me_ = cudaMemsetAsync(a.counters, 0, 4 * sizeof(uint32_t), s); if (me_ != cudaSuccess) return me_; }
    k_irt_load<<<blocks_for((const void*)k_irt_load, device), IB, 0, s>>>(a);
    cudaError_t e = launch_scan_u32(a.ttiles, a.nseg, a.toff, s);
    if (e != cudaSuccess) return e;
    if (ev && (e = irt_mark(ev[0], s)) != cudaSuccess) return e;
    k_irt_init<<<blocks_for((const void*)k_irt_init, device, shape.init_per_sm), IB, 0, s>>>(a);
    if (ev && (e = irt_mark(ev[1], s)) != cudaSuccess) return e;
    k_track_order<<<1, 1024, 0, s>>>(a.tn, a.nseg, a.order);
    int sms = 0, per = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void*)k_irt_sort, SB, 0);
    const unsigned long long sgrid = (unsigned long long)sms * (unsigned long long)(per > 0 ? per : 1);
    k_irt_sort<<<(unsigned)(a.nseg < sgrid ? (a.nseg > 0 ? a.nseg : 1) : sgrid), SB, 0, s>>>(a);
    if (ev && (e = irt_mark(ev[2], s)) != cudaSuccess) return e;
    k_irt_loop<<<blocks_for((const void*)k_irt_loop, device, shape.loop_per_sm), IB, 0, s>>>(a);
    return cudaGetLastError();
}

// The IRT launch sequence as one CUDA graph, captured on a private stream and
// replayed on the caller's.  It is captured again when anything in the
// arguments (seed included) or the shapes changes; a repeated call on the same
// tracks and seed replays it.  If capturing fails the sequence runs as plain
// launches from then on.
cudaError_t irt_graph_run(const IArgs& a, int device, const IrtShape& shape, cudaStream_t s, cudaEvent_t* ev,
                          IrtGraph* g) {
    if (g->off) return launch_irt(a, device, shape, s, ev);
    IrtGraphKey want;
    memset(&want, 0, sizeof want);
    want.a = a;
    want.shape = shape;
    want.device = device;
    want.ev = ev;
    cudaError_t e;
    if (!g->exec || memcmp(&g->key, &want, sizeof want) != 0) {
        if (g->exec) { cudaGraphExecDestroy(g->exec); g->exec = nullptr; }
        cudaStream_t cs;
        if ((e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking)) != cudaSuccess) return e;
        cudaGraph_t gr = nullptr;
        e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            cudaError_t le = launch_irt(a, device, shape, cs, ev);
            e = cudaStreamEndCapture(cs, &gr);
            if (le != cudaSuccess) e = le;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&g->exec, gr, 0);
        if (gr) cudaGraphDestroy(gr);
        cudaStreamDestroy(cs);
        if (e != cudaSuccess) {
            cudaGetLastError();                  // clear the failed capture
            g->exec = nullptr;
            g->off = true;
            return launch_irt(a, device, shape, s, ev);
        }
        g->key = want;
    }
    return cudaGraphLaunch(g->exec, s);
}

cudaError_t launch_group_keys(const float4* rad, unsigned long long n, unsigned long long* key, uint32_t* maxpid,
                              cudaStream_t s) {
    { cudaError_t me_ = cudaMemsetAsync(maxpid, 0, 4, s); if (me_ != cudaSuccess) return me_; }
    if (n) k_group_keys<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(rad, n, key, maxpid);
    return cudaGetLastError();
}

cudaError_t launch_seg_max(const unsigned long long* off, uint32_t nseg, unsigned long long* out, cudaStream_t s) {
    { cudaError_t me_ = cudaMemsetAsync(out, 0, 8, s); if (me_ != cudaSuccess) return me_; }
    k_seg_max<<<148, 256, 0, s>>>(off, nseg, out);
    return cudaGetLastError();
}

}  // namespace wg
