/* oracle/transport.c -- CPU restatement of the reference's electron transport.
 *
 * TEST INFRASTRUCTURE ONLY (CPU oracle; see oracle.h).
 *
 * Follows, statement by statement and in the same floating-point evaluation
 * order, the WGSL of allaunthefox/webgpu-dna:
 *   src/shaders/helpers.wgsl:15-190   (xs_all, xs_shell_fracs, xs_exc_fracs,
 *                                      xs_el_cos, sample_W_sec, bsearch_cdf,
 *                                      xs_vib_total, sample_vib_mode, xs_dea, rn/rf)
 *   src/shaders/primary.wgsl:41-663   (dna_near, meesungnoen_sigma, deposit, main)
 *   src/shaders/secondary.wgsl:17-450 (the Phase B step, run up to MAX_SEC_STEPS
 *                                      times per secondary, dispatch.ts:137-139)
 *   src/gpu/buffers.ts:91-104         (seedPrimaryRNG, reference RNG mode)
 *
 * Processing order: primary pid, then its secondaries in emission order, then
 * pid+1.  Every particle owns its random stream (Philox key = seed, counter =
 * (block, secondary index, pid, 1)), so the results do not depend on the order
 * in which particles are processed; the rad_buf entries come out in canonical
 * order (pid, emitter, sequence), the same order the CUDA path canonicalises to.
 *
 * Must be compiled with -ffp-contract=off (no implicit FMA).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "om.h"
#include "oracle.h"
#include "internal.h"

#define T g_tab
static const float SB[5] = {10.79f, 13.39f, 16.05f, 32.30f, 539.0f};   /* helpers.wgsl:11 */
static const float EX[5] = {8.22f, 10.00f, 11.24f, 12.61f, 13.77f};    /* helpers.wgsl:13 */
static const float NWf = 33.4f;                                          /* helpers.wgsl:2 */
static const float TWO_PI_F = 6.28318530f;   /* 2.0*PI and 6.2831853 both round to this f32 */
static const float PI_F = 3.14159265f;
static const float DEA_E[14] = {0.0f, 4.2f, 4.3f, 5.8f, 6.0f, 6.2f, 6.4f, 7.0f, 7.5f, 7.7f,
                                8.4f, 10.2f, 11.2f, 12.3f};            /* helpers.wgsl:175 */
static const float DEA_S[14] = {0.0f, 0.0f, 0.0f, 2.5e-5f, 2.8e-4f, 6.0e-4f, 6.7e-4f, 3.7e-4f,
                                1.09e-4f, 7.0e-5f, 1.4e-4f, 2.0e-5f, 6.0e-5f, 0.0f};

/* ------------------------------------------------------------- random ---- */
typedef struct {
    int mode;               /* 0 philox, 1 reference xoshiro */
    uint32_t s[4];
    uint32_t k0, k1, c1, c2, c3, blk;
    uint32_t buf[4];
    int idx;
} rng_t;

static inline uint32_t rl(uint32_t x, int k) { return (x << k) | (x >> (32 - k)); }

static inline uint32_t rn(rng_t *r) {
    if (r->mode == 1) {      /* helpers.wgsl:189 */
        uint32_t *s = r->s;
        uint32_t res = rl(s[0] + s[3], 7) + s[0];
        uint32_t t = s[1] << 9;
        s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3]; s[2] ^= t; s[3] = rl(s[3], 11);
        return res;
    }
    if (r->idx == 4) {
        om_u4 o = om_philox(r->blk, r->c1, r->c2, r->c3, r->k0, r->k1);
        r->blk++;
        memcpy(r->buf, o.v, 16);
        r->idx = 0;
    }
    return r->buf[r->idx++];
}
static inline float rf(rng_t *r) { return om_u01f(rn(r)); }

static void rng_philox(rng_t *r, uint64_t seed, uint32_t pid, uint32_t sub) {
    memset(r, 0, sizeof *r);
    r->mode = 0;
    r->k0 = (uint32_t)seed; r->k1 = (uint32_t)(seed >> 32);
    r->c1 = sub; r->c2 = pid; r->c3 = 1u;
    r->idx = 4;
}
/* seedPrimaryRNG, buffers.ts:91-104 (all arithmetic mod 2^32) */
static void rng_reference(rng_t *r, uint32_t i, uint32_t seed) {
    memset(r, 0, sizeof *r);
    r->mode = 1;
    uint32_t s = (i + 1u) * 2654435761u + seed * 1013904223u;
    for (int j = 0; j < 4; ++j) {
        s ^= s >> 16;
        s *= 0x45d9f3bu;
        s ^= s >> 16;
        r->s[j] = s + (uint32_t)j * 0x9E3779B9u;
    }
}

/* ------------------------------------------------------------- tables ---- */
typedef struct { float x, y, z; } v3;

static void xs_all(float E, float *xi, float *xc, float *xl) {          /* helpers.wgsl:15-27 */
    if (E <= T.XE[0]) { *xi = 0.0f; *xc = 0.0f; *xl = T.XL[0]; return; }
    if (E >= T.XE[T.XN - 1]) { *xi = T.XI[T.XN - 1]; *xc = T.XC[T.XN - 1]; *xl = T.XL[T.XN - 1]; return; }
    float t = (om_logf(E) - T.LOG_XE0) * T.INV_LOG_XE_STEP;
    uint32_t i = (uint32_t)fminf(fmaxf(floorf(t), 0.0f), (float)(T.XN - 2));
    float f = t - (float)i;
    uint32_t j = i + 1;
    *xi = fmaxf(0.0f, T.XI[i] + (T.XI[j] - T.XI[i]) * f);
    *xc = fmaxf(0.0f, T.XC[i] + (T.XC[j] - T.XC[i]) * f);
    *xl = fmaxf(0.0f, T.XL[i] + (T.XL[j] - T.XL[i]) * f);
}

static void xs_shell_fracs(float E, float sf[5]) {                       /* helpers.wgsl:29-43 */
    if (E <= T.XE[0]) { for (int k = 0; k < 5; ++k) sf[k] = T.XSF[k][0]; return; }
    if (E >= T.XE[T.XN - 1]) { for (int k = 0; k < 5; ++k) sf[k] = T.XSF[k][T.XN - 1]; return; }
    float t = (om_logf(E) - T.LOG_XE0) * T.INV_LOG_XE_STEP;
    uint32_t i = (uint32_t)fminf(fmaxf(floorf(t), 0.0f), (float)(T.XN - 2));
    float f = t - (float)i;
    uint32_t j = i + 1;
    for (int k = 0; k < 5; ++k) sf[k] = fmaxf(0.0f, T.XSF[k][i] + (T.XSF[k][j] - T.XSF[k][i]) * f);
}

static void xs_exc_fracs(float E, float ef[5]) {                         /* helpers.wgsl:45-64 */
    if (E <= T.XE[0]) { for (int k = 0; k < 5; ++k) ef[k] = T.XEF[k][0]; return; }
    if (E >= T.XE[T.XN - 1]) { for (int k = 0; k < 5; ++k) ef[k] = T.XEF[k][85]; return; }
    float t = (om_logf(E) - T.LOG_XE0) * T.INV_LOG_XE_STEP;
    uint32_t i = (uint32_t)fminf(fmaxf(floorf(t), 0.0f), (float)(T.XN - 2));
    if (i > 85u) i = 85u;
    float f = (i == 85u) ? 0.0f : t - (float)i;
    uint32_t j = i + 1 < 85u ? i + 1 : 85u;
    for (int k = 0; k < 5; ++k) ef[k] = fmaxf(0.0f, T.XEF[k][i] + (T.XEF[k][j] - T.XEF[k][i]) * f);
}

static float xs_el_cos(float E, float r) {                               /* helpers.wgsl:66-82 */
    float rr = fminf(fmaxf(r, 0.0f), 1.0f);
    float jf = rr * (float)(T.N_AC - 1);
    uint32_t jlo = (uint32_t)floorf(jf);
    uint32_t jhi = jlo + 1 < T.N_AC - 1 ? jlo + 1 : T.N_AC - 1;
    float fj = jf - (float)jlo;
    float tE = (om_logf(fmaxf(E, T.XAE[0])) - T.LOG_XAE0) * T.INV_LOG_XAE_STEP;
    uint32_t iE = (uint32_t)fminf(fmaxf(floorf(tE), 0.0f), (float)(T.N_AE - 2));
    float fE = fminf(fmaxf(tE - (float)iE, 0.0f), 1.0f);
    uint32_t b0 = iE * T.N_AC, b1 = (iE + 1) * T.N_AC;
    float c00 = T.XAC[b0 + jlo], c01 = T.XAC[b0 + jhi];
    float c10 = T.XAC[b1 + jlo], c11 = T.XAC[b1 + jhi];
    float cE0 = c00 + (c01 - c00) * fj;
    float cE1 = c10 + (c11 - c10) * fj;
    return fminf(fmaxf(cE0 + (cE1 - cE0) * fE, -1.0f), 1.0f);
}

static float bsearch_cdf(uint32_t shell, uint32_t base, float r) {     /* helpers.wgsl:98-117 */
    const float *C = T.XWC[shell], *W = T.XWT[shell];
    uint32_t jlo = 0;
    for (uint32_t j = 0; j < T.N_WR - 1; ++j) {   /* linear scan, as the reference */
        if (C[base + j] <= r) jlo = j; else break;
    }
    uint32_t jhi = jlo + 1 < T.N_WR - 1 ? jlo + 1 : T.N_WR - 1;
    float c0 = C[base + jlo], c1 = C[base + jhi];
    float e0 = W[base + jlo], e1 = W[base + jhi];
    if (c1 <= c0) return e0;
    float f = fminf(fmaxf((r - c0) / (c1 - c0), 0.0f), 1.0f);
    return e0 + (e1 - e0) * f;
}

static float sample_W_sec(float E, uint32_t shell, float r) {          /* helpers.wgsl:88-96 */
    uint32_t lo = 0, hi = T.N_WE - 1;
    while (hi - lo > 1u) { uint32_t mid = (lo + hi) / 2u; if (T.XWE[mid] <= E) lo = mid; else hi = mid; }
    uint32_t iE = (fabsf(T.XWE[hi] - E) < fabsf(T.XWE[lo] - E)) ? hi : lo;
    return bsearch_cdf(shell, iE * T.N_WR, r);
}

static float xs_vib_total(float E) {                                    /* helpers.wgsl:135-144 */
    if (E < 2.0f || E > 100.0f) return 0.0f;
    for (uint32_t i = 0; i < T.N_VIB - 1; ++i) {
        if (E >= T.XVE[i] && E < T.XVE[i + 1]) {
            float f = (E - T.XVE[i]) / (T.XVE[i + 1] - T.XVE[i]);
            return fmaxf(0.0f, T.XVS[i] + (T.XVS[i + 1] - T.XVS[i]) * f);
        }
    }
    return 0.0f;
}

static uint32_t sample_vib_mode(float E, float r) {                     /* helpers.wgsl:148-170 */
    uint32_t bin = 0;
    for (uint32_t i = 0; i < T.N_VIB - 1; ++i) {
        if (E >= T.XVE[i] && E < T.XVE[i + 1]) { bin = i; break; }
    }
    uint32_t base = bin * 9u;
    float cumsum = 0.0f, cs[9];
    for (int k = 0; k < 9; ++k) {
        float frac = (T.VIB_LEV[k] > E) ? 0.0f : T.XVMF[base + k];
        cumsum = cumsum + frac;
        cs[k] = cumsum;
    }
    if (cumsum <= 0.0f) return 0u;
    float thr = r * cumsum;
    for (int k = 0; k < 9; ++k) if (thr < cs[k]) return (uint32_t)k;
    return 8u;
}

static float xs_dea(float E) {                                          /* helpers.wgsl:177-186 */
    if (E < 4.0f || E > 13.0f) return 0.0f;
    for (int i = 0; i < 13; ++i) {
        if (E >= DEA_E[i] && E < DEA_E[i + 1]) {
            float f = (E - DEA_E[i]) / (DEA_E[i + 1] - DEA_E[i]);
            return fmaxf(0.0f, DEA_S[i] + (DEA_S[i + 1] - DEA_S[i]) * f);
        }
    }
    return 0.0f;
}

static float meesungnoen_sigma(float k) {                               /* primary.wgsl:90-98 */
    if (k <= 0.1f) return 0.0f;
    float r = -4.06217193e-08f;
    r = r * k + 3.06848412e-06f; r = r * k - 9.93217814e-05f; r = r * k + 1.80172797e-03f;
    r = r * k - 2.01135480e-02f; r = r * k + 1.42939448e-01f; r = r * k - 6.48348714e-01f;
    r = r * k + 1.85227848e+00f; r = r * k - 3.36450378e+00f; r = r * k + 4.37785068e+00f;
    r = r * k - 4.20557339e+00f; r = r * k + 3.81679083e+00f; r = r * k - 2.34069784e-01f;
    return fmaxf(r, 0.0f) * 0.6267f;
}

/* ------------------------------------------------------------- sinks ----- */
typedef struct {
    float *rad; uint64_t *key; uint64_t n, cap;
    uint32_t *dose;
    uint64_t dep_units; double dep_f64;
    uint32_t counters[8], sec_stats[8], dbg[8];
    uint64_t steps;
} sink_t;

typedef struct {
    const orc_transport_params *p;
    sink_t *sk;
    uint32_t pid, sub, seq;
    float pidf;             /* f32(pid)*8.0 */
    uint32_t *sec_next;     /* the run's sec_buf index (counters[6] of primary.wgsl), shared */
} emit_t;

static void put(emit_t *e, float x, float y, float z, float code) {
    sink_t *s = e->sk;
    if (s->n == s->cap) {
        s->cap = s->cap ? s->cap * 2 : 4096;
        s->rad = (float *)realloc(s->rad, s->cap * 16);
        s->key = (uint64_t *)realloc(s->key, s->cap * 8);
    }
    float *d = s->rad + 4 * s->n;
    d[0] = x; d[1] = y; d[2] = z; d[3] = code + e->pidf;
    s->key[s->n] = ((uint64_t)(e->pid - e->p->pid_base) << 34) | ((uint64_t)e->sub << 17) | e->seq;
    e->seq++;
    s->n++;
}

static void deposit(emit_t *e, float px, float py, float pz, float dep) {  /* primary.wgsl:102-112 */
    if (dep <= 0.0f) return;
    const orc_transport_params *p = e->p;
    float box = p->box_nm;
    e->sk->dep_f64 += (double)dep;
    float vs = 2.0f * box / (float)p->vc;
    int ix = (int)floorf((px + box) / vs);
    int iy = (int)floorf((py + box) / vs);
    int iz = (int)floorf((pz + box) / vs);
    int n = (int)p->vc;
    if (ix < 0 || ix >= n || iy < 0 || iy >= n || iz < 0 || iz >= n) return;
    uint32_t u = (uint32_t)(dep * 100.0f);
    if (e->sk->dose) e->sk->dose[(uint32_t)((iz * n + iy) * n + ix)] += u;
    e->sk->dep_units += u;
    e->sk->dbg[5] += 1u;                 /* dose-grid updates (an instrumentation count) */
}

static uint32_t dna_near(const orc_transport_params *p, float px, float py, float pz) {
    /* primary.wgsl:41-86 */
    if (p->dna_enable == 0u) return 0u;
    const float r_damage = 0.29f;
    uint32_t N = p->dna_grid_n;
    float spacing = p->dna_spacing;
    float grid_off = -((float)(N - 1u) * spacing) * 0.5f;
    float inv_s = 1.0f / spacing;
    float fi_raw = (py - grid_off) * inv_s;
    float fj_raw = (pz - grid_off) * inv_s;
    int fi = (int)rintf(fi_raw);      /* WGSL round(): half to even */
    int fj = (int)rintf(fj_raw);
    if (fi < 0 || fi >= (int)N || fj < 0 || fj >= (int)N) return 0u;
    float fy = grid_off + (float)fi * spacing;
    float fz = grid_off + (float)fj * spacing;
    float y_rel = py - fy, z_rel = pz - fz;
    float r2 = y_rel * y_rel + z_rel * z_rel;
    float R_reach = p->dna_r_bb + r_damage;
    if (r2 > R_reach * R_reach) return 0u;
    int bp_est = (int)rintf((px - p->dna_x0) / p->dna_rise);
    int b0 = bp_est - 1 > 0 ? bp_est - 1 : 0;
    int b1 = bp_est + 1;
    const float d_phase = (float)(2.0 * 3.14159265 / 10.5);   /* WGSL abstract-float constant */
    float r_bb = p->dna_r_bb;
    for (int b = b0; b <= b1; ++b) {
        float bx = p->dna_x0 + (float)b * p->dna_rise;
        float phi = (float)b * d_phase;
        float s0z, s0y;
        om_sincosf(phi, &s0z, &s0y);
        s0y = r_bb * s0y; s0z = r_bb * s0z;
        float dx = px - bx;
        float dy0 = y_rel - s0y, dz0 = z_rel - s0z;
        if (dx * dx + dy0 * dy0 + dz0 * dz0 < r_damage * r_damage) return 1u;
        float s1z, s1y;
        om_sincosf(phi + PI_F, &s1z, &s1y);
        s1y = r_bb * s1y; s1z = r_bb * s1z;
        float dy1 = y_rel - s1y, dz1 = z_rel - s1z;
        if (dx * dx + dy1 * dy1 + dz1 * dz1 < r_damage * r_damage) return 1u;
    }
    return 0u;
}

/* Gaussian 3-D displacement: the (mu1..mu4) pattern of primary.wgsl:216-220 */
static v3 gauss3(rng_t *s, float sigma) {
    float u1 = fmaxf(rf(s), 1e-30f); float u2 = rf(s);
    float rr = sqrtf(-2.0f * om_logf(u1)) * sigma;
    float sn, cs; om_sincosf(TWO_PI_F * u2, &sn, &cs);
    v3 d;
    d.x = rr * cs; d.y = rr * sn;
    float u3 = fmaxf(rf(s), 1e-30f); float u4 = rf(s);
    d.z = sqrtf(-2.0f * om_logf(u3)) * sigma * om_cosf(TWO_PI_F * u4);
    return d;
}

/* H2O+ + eaq recombination -> H2Ovib dissociation channels (primary.wgsl:246-276) */
static void h2ovib(emit_t *e, rng_t *s, float x, float y, float z) {
    uint32_t *c = e->sk->counters;
    float r_vd = rf(s);
    if (r_vd < 0.1365f) {
        c[0] += 2u; c[5] += 1u; c[7] += 3u;
        put(e, x, y, z, 0.0f); put(e, x, y, z, 0.0f); put(e, x, y, z, 7.0f);
    } else if (r_vd < 0.494f) {
        c[0] += 1u; c[2] += 1u; c[7] += 2u;
        put(e, x, y, z, 0.0f); put(e, x, y, z, 2.0f);
    } else if (r_vd < 0.650f) {
        c[2] += 2u; c[7] += 2u;
        put(e, x, y, z, 2.0f); put(e, x, y, z, 2.0f);
    }
}

/* autoionisation of an excited level (primary.wgsl:473-536 / 560-619) */
static void autoionise(emit_t *e, rng_t *s, float px, float py, float pz) {
    uint32_t *c = e->sk->counters;
    v3 m = gauss3(s, 1.1547005f);
    float bpx = px + m.x, bpy = py + m.y, bpz = pz + m.z;
    float eaq_s = meesungnoen_sigma(1.7f);
    float aex = bpx, aey = bpy, aez = bpz;
    if (eaq_s > 0.0f) {
        v3 a = gauss3(s, eaq_s);
        aex = aex + a.x; aey = aey + a.y; aez = aez + a.z;
    }
    float dx = aex - bpx, dy = aey - bpy, dz = aez - bpz;
    float rsep = fmaxf(sqrtf(dx * dx + dy * dy + dz * dz), 1e-6f);
    float prec = 1.0f - om_expf(-0.711f / rsep);
    float rr = rf(s);
    if (rr < prec) {
        h2ovib(e, s, bpx, bpy, bpz);
    } else {
        c[0] += 1u; c[1] += 1u; c[3] += 1u; c[7] += 3u;
        put(e, bpx, bpy, bpz, 0.0f); put(e, aex, aey, aez, 1.0f); put(e, bpx, bpy, bpz, 3.0f);
    }
}

/* secondary record emitted by a primary (the Particle struct of primary.wgsl:14) */
typedef struct { float x, y, z, E, dx, dy, dz; rng_t r; } sec_t;
typedef struct { sec_t *v; uint32_t n, cap; } secvec_t;

/* Elastic rotation of (dx,dy,dz) by (cos_t, sin_t, cp, sp) (primary.wgsl:169-170) */
static void rotate(float *dx, float *dy, float *dz, float cos_t, float sin_t, float cp, float sp) {
    if (fabsf(*dz) > 0.99999f) {
        float sw = (*dz > 0.0f) ? 1.0f : -1.0f;
        *dx = sin_t * cp; *dy = sin_t * sp * sw; *dz = cos_t * sw;
    } else {
        float q = sqrtf(1.0f - *dz * *dz);
        float inv = 1.0f / q;
        float nx = *dx * cos_t + sin_t * (*dx * *dz * cp - *dy * sp) * inv;
        float ny = *dy * cos_t + sin_t * (*dy * *dz * cp + *dx * sp) * inv;
        float nz = *dz * cos_t - q * sin_t * cp;
        float len = sqrtf(nx * nx + ny * ny + nz * nz);
        *dx = nx / len; *dy = ny / len; *dz = nz / len;
    }
}

/* One interaction after the move (the r_type switch, primary.wgsl:180-649 and
 * secondary.wgsl:167-443). Returns 1 for an ionisation, 2 for an excitation. */
static int interact(emit_t *e, rng_t *s, float *pE, float px, float py, float pz,
                    float *dx, float *dy, float *dz, float xsi, float xsc, float svib,
                    float sdea, float s_tot, int primary, secvec_t *secs) {
    const orc_transport_params *p = e->p;
    uint32_t *c = e->sk->counters;
    float E = *pE;
    int kind = 0;
    float r_type = rf(s) * s_tot;
    if (r_type < xsi && E > SB[0]) {
        float sf[5];
        xs_shell_fracs(E, sf);
        float fsum = fmaxf(sf[0] + sf[1] + sf[2] + sf[3] + sf[4], 1e-12f);
        float r_sh = rf(s) * fsum;
        float bind; uint32_t shell;
        if (r_sh < sf[0]) { bind = SB[0]; shell = 0; }
        else if (r_sh < sf[0] + sf[1]) { bind = SB[1]; shell = 1; }
        else if (r_sh < sf[0] + sf[1] + sf[2]) { bind = SB[2]; shell = 2; }
        else if (r_sh < sf[0] + sf[1] + sf[2] + sf[3]) { bind = SB[3]; shell = 3; }
        else { bind = SB[4]; shell = 4; }
        if (E > bind) {
            float r_w = rf(s);
            float Wmax = (E + bind) * 0.5f;
            float W = sample_W_sec(E, shell, r_w);
            W = fminf(fmaxf(W, bind), Wmax);
            float W_sec = fmaxf(W - bind, 0.0f);
            E -= W;
            kind = 1;
            if (primary) {
                e->sk->dbg[4] += (uint32_t)(W * 10.0f);
                deposit(e, px, py, pz, bind);
                if (W_sec <= p->ce_eV) deposit(e, px, py, pz, W_sec);
                if (dna_near(p, px, py, pz) == 1u) c[4] += 1u;
                v3 m = gauss3(s, 1.1547005f);
                float mpx = px + m.x, mpy = py + m.y, mpz = pz + m.z;
                if (W_sec <= p->ce_eV) {
                    float eaq_s = meesungnoen_sigma(W_sec);
                    float epx = px, epy = py, epz = pz;
                    if (eaq_s > 0.0f) {
                        v3 a = gauss3(s, eaq_s);
                        epx = epx + a.x; epy = epy + a.y; epz = epz + a.z;
                    }
                    float rdx = epx - mpx, rdy = epy - mpy, rdz = epz - mpz;
                    float r_sep = fmaxf(sqrtf(rdx * rdx + rdy * rdy + rdz * rdz), 1e-6f);
                    float p_recomb = 1.0f - om_expf(-0.711f / r_sep);
                    float r_recomb = rf(s);
                    if (r_recomb < p_recomb) {
                        h2ovib(e, s, mpx, mpy, mpz);
                    } else {
                        c[0] += 1u; c[1] += 1u; c[3] += 1u; c[7] += 3u;
                        put(e, mpx, mpy, mpz, 0.0f); put(e, epx, epy, epz, 5.0f); put(e, mpx, mpy, mpz, 3.0f);
                    }
                } else {
                    float r_track = 0.04f * om_powf(W_sec, 1.3f);
                    float r_tail = meesungnoen_sigma(fminf(W_sec, 7.4f));
                    float r_sep_est = fmaxf(r_track + r_tail, 1e-3f);
                    float p_recomb_t = 1.0f - om_expf(-0.711f / r_sep_est);
                    float r_recomb_t = rf(s);
                    if (r_recomb_t < p_recomb_t) {
                        h2ovib(e, s, mpx, mpy, mpz);
                    } else {
                        c[0] += 1u; c[3] += 1u; c[7] += 2u;
                        put(e, mpx, mpy, mpz, 0.0f); put(e, mpx, mpy, mpz, 3.0f);
                    }
                }
                if (W_sec > p->ce_eV) {
                    /* primary.wgsl:363-364: every emission takes a sec_buf index;
                     * at or beyond max_sec the secondary is dropped together with
                     * its angle draws and the primary's momentum update.  Which
                     * emissions come last depends on the order the primaries run
                     * in, as in the reference. */
                    c[6]++;
                    uint32_t sec_idx = __atomic_fetch_add(e->sec_next, 1u, __ATOMIC_RELAXED);
                    if (sec_idx < p->max_sec) {
                        float E_before = E + bind + W_sec;
                        float cos_s;
                        if (W_sec < 50.0f) {
                            cos_s = 2.0f * rf(s) - 1.0f;
                        } else if (W_sec <= 200.0f) {
                            if (rf(s) <= 0.1f) cos_s = 2.0f * rf(s) - 1.0f;
                            else cos_s = rf(s) * 0.70710678f;
                        } else {
                            float sin2 = fminf(fmaxf((1.0f - W_sec / E_before) / (1.0f + W_sec / 1022000.0f), 0.0f), 1.0f);
                            cos_s = sqrtf(fmaxf(0.0f, 1.0f - sin2));
                        }
                        float sin_s = sqrtf(fmaxf(0.0f, 1.0f - cos_s * cos_s));
                        float sps, cps; om_sincosf(TWO_PI_F * rf(s), &sps, &cps);
                        float sdx = *dx, sdy = *dy, sdz = *dz;
                        rotate(&sdx, &sdy, &sdz, cos_s, sin_s, cps, sps);
                        float p_inc = sqrtf(E_before), p_sec = sqrtf(W_sec);
                        float pfx = p_inc * *dx - p_sec * sdx;
                        float pfy = p_inc * *dy - p_sec * sdy;
                        float pfz = p_inc * *dz - p_sec * sdz;
                        float pfl = sqrtf(pfx * pfx + pfy * pfy + pfz * pfz);
                        if (pfl > 1e-10f) { *dx = pfx / pfl; *dy = pfy / pfl; *dz = pfz / pfl; }
                        if (secs->n == secs->cap) {
                            secs->cap = secs->cap ? secs->cap * 2 : 256;
                            secs->v = (sec_t *)realloc(secs->v, secs->cap * sizeof(sec_t));
                        }
                        sec_t *q = &secs->v[secs->n++];
                        q->x = px; q->y = py; q->z = pz; q->E = W_sec;
                        q->dx = sdx; q->dy = sdy; q->dz = sdz;
                        if (s->mode == 1) {           /* child state = 4 parent draws */
                            memset(&q->r, 0, sizeof q->r);
                            q->r.mode = 1;
                            for (int j = 0; j < 4; ++j) q->r.s[j] = rn(s);
                        } else {
                            rng_philox(&q->r, p->seed, e->pid, secs->n);
                        }
                    }
                }
            } else {
                e->sk->sec_stats[4] += 1u;
                deposit(e, px, py, pz, W);
                v3 m = gauss3(s, 1.1547005f);
                float spx = px + m.x, spy = py + m.y, spz = pz + m.z;
                float eaq_s = meesungnoen_sigma(W_sec);
                float epx = px, epy = py, epz = pz;
                if (eaq_s > 0.0f) {
                    v3 a = gauss3(s, eaq_s);
                    epx = epx + a.x; epy = epy + a.y; epz = epz + a.z;
                }
                float rdx = epx - spx, rdy = epy - spy, rdz = epz - spz;
                float r_sep = fmaxf(sqrtf(rdx * rdx + rdy * rdy + rdz * rdz), 1e-6f);
                float p_recomb = 1.0f - om_expf(-0.711f / r_sep);
                float r_recomb = rf(s);
                if (r_recomb < p_recomb) {
                    h2ovib(e, s, spx, spy, spz);
                } else {
                    c[0] += 1u; c[1] += 1u; c[3] += 1u; c[7] += 3u;
                    put(e, spx, spy, spz, 0.0f); put(e, epx, epy, epz, 5.0f); put(e, spx, spy, spz, 3.0f);
                }
                if (dna_near(p, px, py, pz) == 1u) c[4] += 1u;
            }
        }
    } else if (r_type < xsi + xsc) {
        float ef[5];
        xs_exc_fracs(E, ef);
        float efsum = fmaxf(ef[0] + ef[1] + ef[2] + ef[3] + ef[4], 1e-12f);
        float r_ex = rf(s) * efsum;
        float exc_E; uint32_t lvl;
        if (r_ex < ef[0]) { exc_E = EX[0]; lvl = 0; }
        else if (r_ex < ef[0] + ef[1]) { exc_E = EX[1]; lvl = 1; }
        else if (r_ex < ef[0] + ef[1] + ef[2]) { exc_E = EX[2]; lvl = 2; }
        else if (r_ex < ef[0] + ef[1] + ef[2] + ef[3]) { exc_E = EX[3]; lvl = 3; }
        else { exc_E = EX[4]; lvl = 4; }
        float dep = fminf(exc_E, E);
        E -= dep;
        deposit(e, px, py, pz, dep);
        kind = 2;
        float r_ch = rf(s);
        if (lvl == 0u) {
            if (r_ch < 0.65f) {
                c[0] += 1u; c[2] += 1u; c[7] += 2u;
                put(e, px, py, pz, 0.0f); put(e, px, py, pz, 2.0f);
            }
        } else if (lvl == 1u) {
            if (r_ch < 0.175f) {
            } else if (r_ch < 0.2075f) {
                c[0] += 2u; c[5] += 1u; c[7] += 3u;
                put(e, px, py, pz, 0.0f); put(e, px, py, pz, 0.0f); put(e, px, py, pz, 7.0f);
            } else if (r_ch < 0.7075f) {
                autoionise(e, s, px, py, pz);
            } else if (r_ch < 0.961f) {
                c[0] += 1u; c[2] += 1u; c[7] += 2u;
                put(e, px, py, pz, 0.0f); put(e, px, py, pz, 2.0f);
            } else {
                c[2] += 2u; c[7] += 2u;
                put(e, px, py, pz, 2.0f); put(e, px, py, pz, 2.0f);
            }
        } else {
            if (r_ch < 0.50f) autoionise(e, s, px, py, pz);
        }
        if (dna_near(p, px, py, pz) == 1u) c[4] += 1u;
    } else if (r_type < xsi + xsc + svib) {
        uint32_t mode = sample_vib_mode(E, rf(s));
        float dep = fminf(T.VIB_LEV[mode], E);
        E -= dep;
        deposit(e, px, py, pz, dep);
    } else if (r_type < xsi + xsc + svib + sdea) {
        deposit(e, px, py, pz, E);
        c[0] += 1u; c[5] += 1u; c[7] += 3u;
        put(e, px, py, pz, 0.0f); put(e, px, py, pz, 6.0f); put(e, px, py, pz, 7.0f);
        E = 0.0f;
    }
    *pE = E;
    return kind;
}

/* Cross sections, free flight and elastic deflection shared by both phases
 * (primary.wgsl:155-172). Returns 0 when s_tot <= 0. */
static int fly(rng_t *s, float E, float *px, float *py, float *pz, float *dx, float *dy, float *dz,
               float *xsi, float *xsc, float *svib, float *sdea, float *s_tot, float *dist) {
    float xl;
    xs_all(E, xsi, xsc, &xl);
    *svib = xs_vib_total(E);
    *sdea = xs_dea(E);
    *s_tot = *xsi + *xsc + xl + *svib + *sdea;
    if (*s_tot <= 0.0f) return 0;
    float lambda = 1.0f / (NWf * *s_tot);
    *dist = -om_logf(fmaxf(rf(s), 1e-10f)) * lambda;
    float r_el = rf(s);
    float cos_el = xs_el_cos(E, r_el);
    float sin_el = sqrtf(fmaxf(0.0f, 1.0f - cos_el * cos_el));
    float sp, cp; om_sincosf(TWO_PI_F * rf(s), &sp, &cp);
    rotate(dx, dy, dz, cos_el, sin_el, cp, sp);
    *px += *dx * *dist; *py += *dy * *dist; *pz += *dz * *dist;
    return 1;
}

static void run_secondary(emit_t *e, sec_t *q) {                  /* secondary.wgsl:82-450 */
    const orc_transport_params *p = e->p;
    sink_t *sk = e->sk;
    float px = q->x, py = q->y, pz = q->z, E = q->E, dx = q->dx, dy = q->dy, dz = q->dz;
    rng_t *s = &q->r;
    for (uint32_t it = 0; it < p->sec_steps; ++it) {
        if (E < p->ce_eV) {
            deposit(e, px, py, pz, E);
            sk->counters[1] += 1u;
            float eaq_s = meesungnoen_sigma(E);
            float epx = px, epy = py, epz = pz;
            if (eaq_s > 0.0f) {
                v3 a = gauss3(s, eaq_s);
                epx = epx + a.x; epy = epy + a.y; epz = epz + a.z;
            }
            sk->counters[7] += 1u;
            put(e, epx, epy, epz, 5.0f);
            sk->sec_stats[1] += 1u;
            return;
        }
        if (fabsf(px) >= p->box_nm || fabsf(py) >= p->box_nm || fabsf(pz) >= p->box_nm) {
            sk->sec_stats[2] += 1u;
            return;
        }
        float xsi, xsc, svib, sdea, s_tot, dist;
        if (!fly(s, E, &px, &py, &pz, &dx, &dy, &dz, &xsi, &xsc, &svib, &sdea, &s_tot, &dist)) return;
        sk->sec_stats[3] += 1u;
        sk->steps++;
        interact(e, s, &E, px, py, pz, &dx, &dy, &dz, xsi, xsc, svib, sdea, s_tot, 0, NULL);
    }
}

static void run_primary(const orc_transport_params *p, uint32_t idx, sink_t *sk, float *res, uint32_t *sec_next) {
    uint32_t gid = p->pid_base + idx;
    emit_t e = {p, sk, gid, 0, 0, (float)gid * 8.0f, sec_next};
    rng_t s;
    if (p->rng_mode == 1) rng_reference(&s, gid, (uint32_t)p->seed);
    else rng_philox(&s, p->seed, gid, 0);
    float E = p->E_per_primary ? p->E_per_primary[idx] : p->E_eV;
    float px = 0.0f, py = 0.0f, pz = 0.0f;
    float sh = p->start_half;
    if (sh > 0.0f) {
        px = (rf(&s) * 2.0f - 1.0f) * sh;
        py = (rf(&s) * 2.0f - 1.0f) * sh;
        pz = (rf(&s) * 2.0f - 1.0f) * sh;
    }
    float spx = px, spy = py, spz = pz;
    float u1 = fmaxf(rf(&s), 1e-10f);
    float u2 = rf(&s);
    float cos_i = 1.0f - 2.0f * u1;
    float sin_i = sqrtf(fmaxf(0.0f, 1.0f - cos_i * cos_i));
    float spi, cpi; om_sincosf(TWO_PI_F * u2, &spi, &cpi);
    float dx = sin_i * cpi, dy = sin_i * spi, dz = cos_i;
    float total_path = 0.0f, productive_path = 0.0f, max_r = 0.0f;
    uint32_t n_ions = 0, n_exc = 0, escaped = 0;
    secvec_t secs = {0, 0, 0};
    for (uint32_t step = 0; step < p->max_steps; ++step) {
        if (E < p->ce_eV) break;
        if (fabsf(px) >= p->box_nm || fabsf(py) >= p->box_nm || fabsf(pz) >= p->box_nm) { escaped = 1; break; }
        int productive = E > 12.0f;
        float xsi, xsc, svib, sdea, s_tot, dist;
        if (!fly(&s, E, &px, &py, &pz, &dx, &dy, &dz, &xsi, &xsc, &svib, &sdea, &s_tot, &dist)) break;
        sk->steps++;
        total_path += dist;
        if (productive) productive_path += dist;
        float rdx = px - spx, rdy = py - spy, rdz = pz - spz;
        float r = sqrtf(rdx * rdx + rdy * rdy + rdz * rdz);
        if (r > max_r) max_r = r;
        if (fabsf(px) >= p->box_nm || fabsf(py) >= p->box_nm || fabsf(pz) >= p->box_nm) { escaped = 1; break; }
        int k = interact(&e, &s, &E, px, py, pz, &dx, &dy, &dz, xsi, xsc, svib, sdea, s_tot, 1, &secs);
        if (k == 1) n_ions++;
        else if (k == 2) n_exc++;
    }
    if (escaped == 0u && E > 0.0f) deposit(&e, px, py, pz, E);
    uint32_t *ru = (uint32_t *)res;
    res[0] = total_path; res[1] = productive_path; res[2] = E;
    ru[3] = n_ions; ru[4] = n_exc; ru[5] = escaped; res[6] = max_r; ru[7] = 0;
    sk->dbg[0] += n_ions; sk->dbg[1] += n_exc; sk->dbg[2] += escaped; sk->dbg[3] += 1u;
    /* Phase B for this primary's secondaries, in emission order */
    for (uint32_t k = 0; k < secs.n; ++k) {
        e.sub = k + 1;
        e.seq = 0;
        run_secondary(&e, &secs.v[k]);
    }
    free(secs.v);
}

int orc_transport(const orc_transport_params *p, orc_transport_out *o, int nthreads) {
    if (!g_tab.loaded) return -1;
    uint32_t np = p->np;
    size_t ngrid = (size_t)p->vc * p->vc * p->vc;
    if (nthreads < 1) nthreads = 1;
    /* per-primary sinks are merged in pid order, so the output order is
     * independent of the thread count */
    sink_t *sinks = (sink_t *)calloc(np ? np : 1, sizeof(sink_t));
    uint32_t **tdose = (uint32_t **)calloc((size_t)nthreads, sizeof(uint32_t *));
    if (!sinks || !tdose) return -2;
    if (o->dose) memset(o->dose, 0, ngrid * 4);
    uint32_t sec_next = 0;
#pragma omp parallel num_threads(nthreads)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        uint32_t *dl = NULL;
        if (o->dose) { dl = (uint32_t *)calloc(ngrid, 4); tdose[tid] = dl; }
#pragma omp for schedule(dynamic, 1)
        for (int64_t i = 0; i < (int64_t)np; ++i) {
            sinks[i].dose = dl;
            run_primary(p, (uint32_t)i, &sinks[i], o->results + 8 * i, &sec_next);
        }
    }
    memset(o->counters, 0, sizeof o->counters);
    memset(o->sec_stats, 0, sizeof o->sec_stats);
    memset(o->dbg, 0, sizeof o->dbg);
    uint64_t total = 0;
    for (uint32_t i = 0; i < np; ++i) total += sinks[i].n;
    o->rad = (float *)malloc((total ? total : 1) * 16);
    o->rad_key = (uint64_t *)malloc((total ? total : 1) * 8);
    o->rad_n = total;
    o->dep_units = 0; o->dep_eV_f64 = 0.0; o->steps = 0;
    uint64_t off = 0;
    for (uint32_t i = 0; i < np; ++i) {
        sink_t *s = &sinks[i];
        if (s->n) {
            memcpy(o->rad + 4 * off, s->rad, s->n * 16);
            memcpy(o->rad_key + off, s->key, s->n * 8);
        }
        off += s->n;
        for (int k = 0; k < 8; ++k) {
            o->counters[k] += s->counters[k];
            o->sec_stats[k] += s->sec_stats[k];
            o->dbg[k] += s->dbg[k];
        }
        o->dep_units += s->dep_units;
        o->dep_eV_f64 += s->dep_f64;
        o->steps += s->steps;
        free(s->rad); free(s->key);
    }
    o->sec_n = o->counters[6] < p->max_sec ? o->counters[6] : p->max_sec;
    if (o->dose) {
        for (int t = 0; t < nthreads; ++t) {
            if (!tdose[t]) continue;
            for (size_t v = 0; v < ngrid; ++v) o->dose[v] += tdose[t][v];
            free(tdose[t]);
        }
    }
    free(tdose);
    free(sinks);
    int rc = 0;
    if (o->counters[6] > p->max_sec) rc = 1;      /* a cap was reached: results not comparable */
    if (o->counters[7] > p->max_rad) rc = 1;
    return rc;
}
