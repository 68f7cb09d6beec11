/* oracle/scoring.c -- CPU restatement of the reference's DNA-damage scoring.
 *
 * TEST INFRASTRUCTURE ONLY (CPU oracle; see oracle.h).
 *
 * Follows allaunthefox/webgpu-dna:
 *   src/physics/dna-geometry.ts:16-68   buildDNATarget (f64 math, f32 storage)
 *   src/scoring/ssb-dsb.ts:43-121       scoreIndirectSSB
 *   src/scoring/ssb-dsb.ts:135-217      scoreDirectSSB_events
 *   src/scoring/ssb-dsb.ts:348-407      clusterDSB
 *   src/scoring/ssb-dsb.ts:421-427      makeSsbRng (LCG 1664525, 1013904223)
 * with JavaScript number semantics: every scalar is an IEEE double, typed
 * arrays round on store, Math.round rounds half-way cases up.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "oracle.h"

static double js_round(double x) {          /* Math.round: ties toward +inf */
    double f = floor(x);
    return (x - f >= 0.5) ? f + 1.0 : f;
}

int orc_build_dna(double L_nm, uint32_t grid_N, double spacing_nm, orc_dna *d) {
    memset(d, 0, sizeof *d);
    const double rise = 0.34, bp_per_turn = 10.5, r_bb = 1.0;
    uint32_t n_bp_per = (uint32_t)floor(L_nm / rise);
    double x0 = -((double)n_bp_per - 1) * rise * 0.5;
    double d_phase = (2 * M_PI) / bp_per_turn;
    uint32_t nf = grid_N * grid_N;
    d->grid_N = grid_N; d->n_bp_per = n_bp_per; d->n_fibers = nf; d->n_bp = nf * n_bp_per;
    d->rise = rise; d->r_bb = r_bb; d->spacing_nm = spacing_nm; d->x0 = x0; d->L_nm = L_nm;
    d->fy = (float *)malloc(nf * 4ull); d->fz = (float *)malloc(nf * 4ull);
    d->rbb0 = (float *)malloc(n_bp_per * 8ull); d->rbb1 = (float *)malloc(n_bp_per * 8ull);
    if (!d->fy || !d->fz || !d->rbb0 || !d->rbb1) return -1;
    double off = -(((double)grid_N - 1) * spacing_nm) * 0.5;
    for (uint32_t fi = 0; fi < grid_N; ++fi)
        for (uint32_t fj = 0; fj < grid_N; ++fj) {
            uint32_t idx = fi * grid_N + fj;
            d->fy[idx] = (float)(off + fi * spacing_nm);
            d->fz[idx] = (float)(off + fj * spacing_nm);
        }
    for (uint32_t i = 0; i < n_bp_per; ++i) {
        double phi = i * d_phase;
        d->rbb0[2 * i] = (float)(r_bb * cos(phi));
        d->rbb0[2 * i + 1] = (float)(r_bb * sin(phi));
        d->rbb1[2 * i] = (float)(r_bb * cos(phi + M_PI));
        d->rbb1[2 * i + 1] = (float)(r_bb * sin(phi + M_PI));
    }
    return 0;
}

void orc_free_dna(orc_dna *d) {
    free(d->fy); free(d->fz); free(d->rbb0); free(d->rbb1);
    memset(d, 0, sizeof *d);
}

static inline double lcg(uint32_t *s) {
    *s = *s * 1664525u + 1013904223u;
    return *s / 4294967296.0;
}

/* nearest backbone test shared by both scoring passes (ssb-dsb.ts:73-106);
 * returns 1 when in reach, with the hit byte index in *hidx and strand */
static int near_backbone(const orc_dna *d, double x, double y, double z, double r_d,
                         uint64_t *hidx, int *strand, int *cand) {
    double x_half = ((double)d->n_bp_per - 1) * d->rise * 0.5;
    double rise_inv = 1 / d->rise;
    double grid_off = -(((double)d->grid_N - 1) * d->spacing_nm) * 0.5;
    double inv_sp = 1 / d->spacing_nm;
    *cand = 0;
    if (x < -x_half - r_d || x > x_half + r_d) return 0;
    double fi = js_round((y - grid_off) * inv_sp);
    double fj = js_round((z - grid_off) * inv_sp);
    if (fi < 0 || fi >= d->grid_N || fj < 0 || fj >= d->grid_N) return 0;
    uint32_t fiber = (uint32_t)fi * d->grid_N + (uint32_t)fj;
    double y_rel = y - (double)d->fy[fiber];
    double z_rel = z - (double)d->fz[fiber];
    double r2 = y_rel * y_rel + z_rel * z_rel;
    double outer = d->r_bb + r_d;
    if (r2 > outer * outer) return 0;
    *cand = 1;
    double bp_est = js_round((x + x_half) * rise_inv);
    double b0 = bp_est - 2 > 0 ? bp_est - 2 : 0;
    double b1 = bp_est + 2 < (double)d->n_bp_per - 1 ? bp_est + 2 : (double)d->n_bp_per - 1;
    double best = INFINITY;
    int64_t best_bp = -1;
    int best_s = -1;
    for (double bb = b0; bb <= b1; bb += 1) {
        int64_t b = (int64_t)bb;
        double dx = x - (d->x0 + bb * d->rise);
        double dy0 = y_rel - (double)d->rbb0[2 * b], dz0 = z_rel - (double)d->rbb0[2 * b + 1];
        double d20 = dx * dx + dy0 * dy0 + dz0 * dz0;
        if (d20 < best) { best = d20; best_bp = b; best_s = 0; }
        double dy1 = y_rel - (double)d->rbb1[2 * b], dz1 = z_rel - (double)d->rbb1[2 * b + 1];
        double d21 = dx * dx + dy1 * dy1 + dz1 * dz1;
        if (d21 < best) { best = d21; best_bp = b; best_s = 1; }
    }
    if (!(best < r_d * r_d)) return 0;
    *hidx = (uint64_t)fiber * d->n_bp_per + (uint64_t)best_bp + (uint64_t)best_s * d->n_bp;
    *strand = best_s;
    return 1;
}

int orc_score_direct(const orc_dna *d, const float *rad, uint64_t rad_n, uint32_t lcg_state,
                     uint8_t *hits, orc_ssb_out *o) {
    memset(o, 0, sizeof *o);
    uint64_t i = 0;
    while (i < rad_n) {
        float x = rad[4 * i], y = rad[4 * i + 1], z = rad[4 * i + 2];
        uint64_t skip = 1;
        if (i + 1 < rad_n && rad[4 * (i + 1)] == x && rad[4 * (i + 1) + 1] == y && rad[4 * (i + 1) + 2] == z)
            skip = 2;
        i += skip;
        uint64_t h; int s, cand;
        int in = near_backbone(d, x, y, z, 0.29, &h, &s, &cand);
        o->candidates += (uint64_t)cand;
        if (!in) continue;
        o->in_reach++;
        if (lcg(&lcg_state) < 0.15) {
            if (hits[h] == 0) { hits[h] = 1; o->ssb++; if (s == 0) o->ssb0++; else o->ssb1++; }
        }
    }
    o->lcg_state = lcg_state;
    return 0;
}

int orc_score_indirect(const orc_dna *d, const float *pos, const uint32_t *alive, uint64_t n,
                       uint32_t lcg_state, uint8_t *hits, orc_ssb_out *o) {
    memset(o, 0, sizeof *o);
    for (uint64_t i = 0; i < n; ++i) {
        if (alive[i] == 0) continue;
        if (js_round(pos[4 * i + 3]) != 0.0) continue;
        uint64_t h; int s, cand;
        int in = near_backbone(d, pos[4 * i], pos[4 * i + 1], pos[4 * i + 2], 0.29, &h, &s, &cand);
        o->candidates += (uint64_t)cand;
        if (!in) continue;
        o->in_reach++;
        if (lcg(&lcg_state) < 0.4) {
            if (hits[h] == 0) { hits[h] = 1; o->ssb++; if (s == 0) o->ssb0++; else o->ssb1++; }
        }
    }
    o->lcg_state = lcg_state;
    return 0;
}

int orc_cluster_dsb(const orc_dna *d, const uint8_t *hits, uint64_t *dsb, double *dsb_expected,
                    uint64_t *ssb0, uint64_t *ssb1) {
    uint32_t n_per = d->n_bp_per;
    uint64_t n = d->n_bp;
    const int W = 10;
    double window_bp = 2 * W + 1;
    uint64_t di = 0, t0 = 0, t1 = 0;
    double de = 0;
    uint32_t *s0 = (uint32_t *)malloc(n_per * 4ull), *s1 = (uint32_t *)malloc(n_per * 4ull);
    uint8_t *used = (uint8_t *)malloc(n_per);
    for (uint32_t fi = 0; fi < d->n_fibers; ++fi) {
        uint64_t base = (uint64_t)fi * n_per;
        uint32_t k0 = 0, k1 = 0;
        for (uint32_t b = 0; b < n_per; ++b) {
            if (hits[base + b] == 1) s0[k0++] = b;
            if (hits[base + b + n] == 1) s1[k1++] = b;
        }
        if (k0 == 0 && k1 == 0) continue;
        t0 += k0; t1 += k1;
        memset(used, 0, k1);
        uint32_t jlo = 0;
        for (uint32_t a = 0; a < k0; ++a) {
            int64_t b0 = s0[a];
            while (jlo < k1 && (int64_t)s1[jlo] < b0 - W) jlo++;
            for (uint32_t j = jlo; j < k1 && (int64_t)s1[j] <= b0 + W; ++j)
                if (!used[j]) { used[j] = 1; di++; break; }
        }
        if (k0 > 0 && k1 > 0 && n_per > 0) {
            double p_pair = fmin(1, window_bp / n_per);
            double np = (double)k0 * (double)k1;
            de += 1 - pow(1 - p_pair, np);
        }
    }
    free(s0); free(s1); free(used);
    *dsb = di; *dsb_expected = de; *ssb0 = t0; *ssb1 = t1;
    return 0;
}

/* ---- dose-grid scoring (src/scoring/ssb-dsb.ts:227-334) and reductions
 * (src/scoring/dose.ts:13-85), JS number semantics: f64 arithmetic, f32 where
 * the reference stores into a Float32Array. */

/* scoreDirectSSB: expected direct SSBs from the voxel dose at each backbone
 * site.  lambda (2 * n_bp floats) receives the per-site expectations; strand
 * 1 divides the dose by 10 where strand 0 divides by 100, as the reference
 * does (ssb-dsb.ts:273-276). */
double orc_voxel_ssb(const orc_dna *d, const uint32_t *dose, uint32_t vc, double box_nm, float *lambda) {
    const double vox_nm = (2 * box_nm) / vc;
    const double vox_vol = vox_nm * vox_nm * vox_nm;
    const double half = box_nm;
    const double inv_vox = 1 / vox_nm;
    const double r = 0.29;                                       /* SSB_R_DAMAGE_NM */
    const double bb_vol_per_bp = (4.0 / 3) * M_PI * r * r * r;
    const double K = ((bb_vol_per_bp / vox_vol) * 0.15) / 22;   /* SSB_P_DIRECT, E_mean_ion */
    const uint64_t n = d->n_bp;
    double direct = 0;
    memset(lambda, 0, 2 * n * sizeof(float));
    for (uint32_t fi = 0; fi < d->n_fibers; ++fi) {
        const double fy = d->fy[fi], fz = d->fz[fi];
        const uint64_t base = (uint64_t)fi * d->n_bp_per;
        for (uint32_t b = 0; b < d->n_bp_per; ++b) {
            const double bx = d->x0 + b * d->rise;
            const double vx = floor((bx + half) * inv_vox);
            if (vx < 0 || vx >= vc) continue;
            const double y0 = fy + d->rbb0[2 * b], z0 = fz + d->rbb0[2 * b + 1];
            const double y1 = fy + d->rbb1[2 * b], z1 = fz + d->rbb1[2 * b + 1];
            const double vy0 = floor((y0 + half) * inv_vox), vz0 = floor((z0 + half) * inv_vox);
            const double vy1 = floor((y1 + half) * inv_vox), vz1 = floor((z1 + half) * inv_vox);
            if (vy0 >= 0 && vy0 < vc && vz0 >= 0 && vz0 < vc) {
                const double dd = dose[(uint64_t)((vz0 * vc + vy0) * vc + vx)] / 100.0;
                const double l = dd * K;
                lambda[base + b] = (float)l;
                direct += l;
            }
            if (vy1 >= 0 && vy1 < vc && vz1 >= 0 && vz1 < vc) {
                const double dd = dose[(uint64_t)((vz1 * vc + vy1) * vc + vx)] / 10.0;
                const double l = dd * K;
                lambda[n + base + b] = (float)l;
                direct += l;
            }
        }
    }
    return direct;
}

/* expectedDSBLocal: per fibre, strand-0 density times the strand-1 density
 * summed over +-DSB_WINDOW_BP, densities = lambda + indirect hit indicator. */
double orc_expected_dsb_local(const orc_dna *d, const float *lambda, const uint8_t *hits) {
    const int64_t W = 10, n_per = d->n_bp_per;
    const uint64_t n = d->n_bp;
    float *s0 = (float *)malloc(n_per * sizeof(float)), *s1 = (float *)malloc(n_per * sizeof(float));
    double e = 0;
    for (uint32_t fi = 0; fi < d->n_fibers; ++fi) {
        const uint64_t base = (uint64_t)fi * n_per;
        double sum0 = 0, sum1 = 0;
        for (int64_t b = 0; b < n_per; ++b) {
            const double v0 = (double)lambda[base + b] + ((hits && hits[base + b] == 1) ? 1 : 0);
            const double v1 = (double)lambda[n + base + b] + ((hits && hits[n + base + b] == 1) ? 1 : 0);
            s0[b] = (float)v0; s1[b] = (float)v1;
            sum0 += v0; sum1 += v1;
        }
        if (sum0 == 0 || sum1 == 0) continue;
        double win = 0;
        for (int64_t b = 0; b <= (W < n_per - 1 ? W : n_per - 1); ++b) win += s1[b];
        for (int64_t b = 0; b < n_per; ++b) {
            e += s0[b] * win;
            const int64_t lo = b - W, hi = b + 1 + W;
            if (hi < n_per) win += s1[hi];
            if (lo >= 0) win -= s1[lo];
        }
    }
    free(s0); free(s1);
    return e;
}

/* sumDoseEV (dose.ts:13-17): the exact integer sum / 100 */
double orc_dose_sum_ev(const uint32_t *dose, uint64_t n) {
    uint64_t s = 0;
    for (uint64_t i = 0; i < n; ++i) s += dose[i];
    return (double)s / 100.0;
}

/* projection sums of renderDoseProjection (dose.ts:61-85): axis 0 sums over z
 * into [y][x], axis 1 over x into [z][y]; stored as float like the reference */
void orc_dose_projection(const uint32_t *dose, uint32_t vc, int axis, float *proj) {
    for (uint32_t a = 0; a < vc; ++a)
        for (uint32_t b = 0; b < vc; ++b) {
            uint64_t s = 0;
            for (uint32_t c = 0; c < vc; ++c)
                s += axis == 0 ? dose[((uint64_t)c * vc + a) * vc + b] : dose[((uint64_t)a * vc + b) * vc + c];
            proj[(uint64_t)a * vc + b] = (float)(double)s;
        }
}
