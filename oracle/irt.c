/* oracle/irt.c -- CPU restatement of the reference's IRT chemistry worker.
 *
 * TEST INFRASTRUCTURE ONLY (CPU oracle; see oracle.h).
 *
 * Follows public/irt-worker.js of allaunthefox/webgpu-dna:
 *   :16-28    meesungnoen2002            :31-39   erfcinv
 *   :41-48    randn, clf6                :53-88   erfcx
 *   :91-113   SamplePDC                  :116-129 sampleIRT_type0 (TDC)
 *   :133-175  sampleIRT_type1 (PDC)      :191-286 species / reaction tables
 *   :289-346  MinHeap                    :430-465 pairWithAlive
 *   :370-698  onmessage (grouping, load + displacement, O(n^2) initial
 *             pairing, event loop with checkpoints, products, G values)
 *
 * Documented divergences (the reference is itself non-deterministic):
 *   1. Math.random() is replaced by Philox4x32-10 streams keyed by the track
 *      (pid) and the particle / pair indices, so that every draw is a function
 *      of what it is for, not of the order in which it is taken:
 *        load draws of particle k      counter (blk, k, pid, 2)
 *        acceptance draw of pair i<j   counter (j>>2, i, pid, 3), word j&3
 *        SamplePDC trial t of (i,j)    counter (i, j, pid, 4 | t<<4)
 *        product idx, partner jj       counter (idx, jj, pid, 5): words 0-2 are
 *                                      the Box-Muller radius draws of x, y, z,
 *                                      word 3 the acceptance draw; counter
 *                                      (idx, jj, pid, 5 | 1<<4): words 0-2 are
 *                                      the Box-Muller angle draws
 *      A 53-bit double is made from two words, a 32-bit one as (w+0.5)/2^32.
 *   2. Events with equal times leave the heap in (t, i, j) order (the
 *      reference's binary heap leaves ties in an arbitrary order).
 *   3. Elementary functions are the oracle's own (om.h); per-reaction
 *      constants use the C library, as the reference uses Math.*.
 *
 * Must be compiled with -ffp-contract=off.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "om.h"
#include "oracle.h"

#define NSP 6
#define NRX 9
static const double IRT_D[NSP] = {2.2, 4.9, 7.0, 9.46, 2.3, 5.3};
static const double VDW_R[NSP] = {0.22, 0.50, 0.19, 0.25, 0.21, 0.33};
static const int CHARGE[NSP] = {0, -1, 0, 1, 0, -1};
typedef struct { int a, b; double k; int prods[2]; int np; int type; } rxn_def;
static const rxn_def RXN[NRX] = {
    {0, 0, 0.55e10, {4, 0}, 1, 1},   /* OH+OH -> H2O2 */
    {0, 1, 2.95e10, {5, 0}, 1, 1},   /* eaq+OH -> OH- */
    {0, 2, 1.55e10, {0, 0}, 0, 1},   /* OH+H -> H2O */
    {1, 1, 0.636e10, {5, 5}, 2, 0},  /* eaq+eaq -> 2OH- + H2 */
    {1, 2, 2.50e10, {5, 0}, 1, 0},   /* eaq+H -> OH- + H2 */
    {1, 3, 2.11e10, {2, 0}, 1, 1},   /* eaq+H3O+ -> H */
    {2, 2, 0.503e10, {0, 0}, 0, 0},  /* H+H -> H2 */
    {1, 4, 1.10e10, {5, 0}, 2, 1},   /* eaq+H2O2 -> OH- + OH (prods 5, 0) */
    {3, 5, 1.13e11, {0, 0}, 0, 0},   /* H3O+ + OH- -> H2O */
};
static const double CHECKPOINTS[7] = {0.001, 0.01, 0.1, 1, 10, 100, 1000};

typedef struct {
    double sigma[NRX], sigma_eff[NRX], rc[NRX], kdif[NRX], kact[NRX], prob[NRX], kobs[NRX];
    double a_pdc[NRX];       /* SamplePDC 'a' (depends on the reaction only) */
    double coth_sig[NRX];    /* cosh/sinh(rc/(2 sigma_c)) for Coulomb PDC */
    int map[NSP * NSP];
    double sig_oh, sig_h, sig_eaq, r_cut2;
} irt_consts;

static irt_consts C;
static int C_ready;

static void init_consts(void) {                          /* irt-worker.js:204-286 */
    if (C_ready) return;
    const double ONS = 1.44 / (0.02527 * 80.1);
    const double Rs = 0.29;
    const double KC = 1e24 / (6.022e23 * 1e9);
    for (int r = 0; r < NRX; ++r) {
        int a = RXN[r].a, b = RXN[r].b;
        double Ds = IRT_D[a] + IRT_D[b];
        int self = (a == b);
        double rc = CHARGE[a] * CHARGE[b] * ONS;
        C.rc[r] = rc;
        double k = RXN[r].k * KC;
        C.kobs[r] = k;
        if (RXN[r].type == 0) {
            double sig = k / (4 * M_PI * Ds);
            if (self) sig *= 2;
            C.sigma[r] = sig; C.sigma_eff[r] = sig;
            C.kdif[r] = 0; C.kact[r] = 0; C.prob[r] = 1;
        } else {
            double sc = VDW_R[a] + VDW_R[b];
            C.sigma[r] = sc;
            double se, kd;
            if (rc == 0) { se = sc; kd = 4 * M_PI * Ds * sc; if (self) kd /= 2; }
            else { se = -rc / (1 - exp(rc / sc)); kd = 4 * M_PI * Ds * se; if (self) kd /= 2; }
            C.sigma_eff[r] = se; C.kdif[r] = kd;
            double ka = kd * k / (kd - k);
            C.kact[r] = ka;
            C.prob[r] = Rs / (Rs + (kd / ka) * (se + Rs));
            if (rc == 0) {
                C.a_pdc[r] = (1.0 / sc) * ka / k;
            } else {
                double v = ka / (4 * M_PI * sc * sc * exp(-rc / sc));
                double alpha = v + rc * Ds / (sc * sc * (1 - exp(-rc / sc)));
                double sh = sinh(rc / (2 * sc));
                C.a_pdc[r] = 4 * sc * sc * alpha / (Ds * rc * rc) * sh * sh;
                C.coth_sig[r] = cosh(rc / (2 * sc)) / sinh(rc / (2 * sc));
            }
        }
    }
    for (int i = 0; i < NSP * NSP; ++i) C.map[i] = -1;
    for (int r = 0; r < NRX; ++r) {
        C.map[RXN[r].a * NSP + RXN[r].b] = r;
        C.map[RXN[r].b * NSP + RXN[r].a] = r;
    }
    /* meesungnoen2002(1.7) * sqrt(pi)/2^(3/2)  (irt-worker.js:349-361) */
    static const double g[13] = {-4.06217193e-08, 3.06848412e-06, -9.93217814e-05, 1.80172797e-03,
                                 -2.01135480e-02, 1.42939448e-01, -6.48348714e-01, 1.85227848e+00,
                                 -3.36450378e+00, 4.37785068e+00, -4.20557339e+00, 3.81679083e+00,
                                 -2.34069784e-01};
    double rm = 0;
    for (int i = 12; i >= 0; --i) rm += g[12 - i] * pow(1.7, i);
    C.sig_eaq = rm * 0.62665706865775006;
    C.sig_oh = 0.8 / sqrt(3.0);
    C.sig_h = (17.0 / 18.0) * 2.4 / sqrt(3.0);
    double rcut = 1.45 + 2 * sqrt(8 * 9.46 * 1000);
    C.r_cut2 = rcut * rcut;
    C_ready = 1;
}

void orc_irt_rxn_table(double out[9][6]) {
    init_consts();
    for (int r = 0; r < NRX; ++r) {
        out[r][0] = C.sigma[r]; out[r][1] = C.sigma_eff[r]; out[r][2] = C.rc[r];
        out[r][3] = C.kdif[r]; out[r][4] = C.kact[r]; out[r][5] = C.prob[r];
    }
}

/* ------------------------------------------------------------ functions -- */
static double erfcinv_(double x) {                                   /* :31-39 */
    if (x <= 0 || x >= 2) return 0;
    double p = x > 1 ? 2 - x : x;
    double t = sqrt(-2 * om_log(p / 2));
    double y = t - (2.515517 + 0.802853 * t + 0.010328 * t * t) /
                   (1 + 1.432788 * t + 0.189269 * t * t + 0.001308 * t * t * t);
    y *= 0.7071067811865475;
    return x > 1 ? -y : y;
}

static const double ERFCX_C[28] = {
    -1.3026537197817094, 6.4196979235649026e-1, 1.9476473204185836e-2, -9.561514786808631e-3,
    -9.46595344482036e-4, 3.66839497852761e-4, 4.2523324806907e-5, -2.0278578112534e-5,
    -1.624290004647e-6, 1.303655835580e-6, 1.5626441722e-8, -8.5238095915e-8,
    6.529054439e-9, 5.059343495e-9, -9.91364156e-10, -2.27365122e-10,
    9.6467911e-11, 2.394038e-12, -6.886027e-12, 8.94487e-13,
    3.13092e-13, -1.12708e-13, 3.81e-16, 7.106e-15,
    -1.523e-15, -9.4e-17, 1.21e-16, -2.8e-17};

static double erfcx_(double x) {                                     /* :53-88 */
    if (x < 0) return 2 * om_exp(x * x) - erfcx_(-x);
    if (x >= 6) {
        double f = 0;
        for (int n = 30; n >= 1; --n) f = (0.5 * n) / (x + f);
        return 0.5641895835477563 / (x + f);
    }
    double t = 2.0 / (2.0 + x);
    double ty = 4 * t - 2;
    double d = 0, dd = 0;
    for (int j = 27; j > 0; --j) { double tmp = d; d = ty * d - dd + ERFCX_C[j]; dd = tmp; }
    return t * om_exp(0.5 * (ERFCX_C[0] + ty * d) - dd);
}

typedef struct { uint32_t k0, k1; uint32_t pid; } irt_rng;

static double pdc(const irt_rng *g, uint32_t i, uint32_t j, double a, double b) { /* :91-113 */
    double p = 2.0 * sqrt(2.0 * b / a);
    double q = 2.0 / sqrt(2.0 * b / a);
    double M = fmax(1.0 / (a * a), 3.0 * b / a);
    for (uint32_t trial = 0; trial < 10000; ++trial) {
        om_u4 w = om_philox(i, j, g->pid, 4u | (trial << 4), g->k0, g->k1);
        double U = om_u01d(w.v[0], w.v[1]);
        double X;
        if (U < p / (p + q * M)) { double h = U * (p + q * M) / 2; X = h * h; }
        else { double h = 2 / ((1 - U) * (p + q * M) / M); X = h * h; }
        U = om_u01d(w.v[2], w.v[3]);
        double sqX = sqrt(X);
        double lambdax = om_exp(-b * b / X) * (1.0 - a * sqrt(M_PI * X) * erfcx_(b / sqX + a * sqX));
        if ((X <= 2.0 * b / a && U <= lambdax) || (X >= 2.0 * b / a && U * M / X <= lambdax)) return X;
    }
    return -1.0;
}

/* sampleIRT (:116-184) with the acceptance draw U given */
static double sample_irt(const irt_rng *g, uint32_t i, uint32_t j, double r0, int ri, double D, double U) {
    if (RXN[ri].type == 0) {
        double sigma = C.sigma[ri], rc = C.rc[ri];
        if (sigma <= 0 || D <= 0) return -1;
        if (r0 <= sigma) return 0;
        double r0e = r0;
        if (rc != 0) r0e = -rc / (1 - om_exp(rc / r0));
        if (r0e <= sigma) return 0;
        double Winf = sigma / r0e;
        if (U <= 0 || U >= Winf) return -1;
        double ei = erfcinv_(r0e * U / sigma);
        if (fabs(ei) < 1e-10) return -1;
        double dr = r0e - sigma;
        return 0.25 * dr * dr / (D * ei * ei);
    }
    double sigma_c = C.sigma[ri], rc = C.rc[ri];
    double a, b, sc_chk = sigma_c, r0_chk = r0;
    a = C.a_pdc[ri];
    if (rc == 0) {
        b = (r0 - sigma_c) / 2;
    } else {
        double coth_r0 = 1.0 + 2.0 / om_expm1(2.0 * (rc / (2 * r0)));
        b = rc / 4 * (coth_r0 - C.coth_sig[ri]);
        r0_chk = -rc / (1 - om_exp(rc / r0));
        sc_chk = C.sigma_eff[ri];
    }
    if (sc_chk > r0_chk) return (C.prob[ri] > U) ? 0 : -1;
    double Winf = sc_chk / r0_chk * C.kobs[ri] / C.kdif[ri];
    if (Winf > U) {
        double X = pdc(g, i, j, a, b);
        if (X > 0) return X / D;
    }
    return -1;
}

/* ------------------------------------------------------------------ heap -- */
typedef struct { double t; int32_t a, b; } evt;
typedef struct { evt *v; size_t n, cap; } heap_t;

static inline int ev_less(const evt *x, const evt *y) {
    if (x->t != y->t) return x->t < y->t;
    if (x->a != y->a) return x->a < y->a;
    return x->b < y->b;
}
static void hpush(heap_t *h, double t, int a, int b) {
    if (h->n == h->cap) { h->cap = h->cap ? 2 * h->cap : 1024; h->v = (evt *)realloc(h->v, h->cap * sizeof(evt)); }
    size_t c = h->n++;
    h->v[c].t = t; h->v[c].a = a; h->v[c].b = b;
    while (c > 0) {
        size_t p = (c - 1) >> 1;
        if (!ev_less(&h->v[c], &h->v[p])) break;
        evt tmp = h->v[p]; h->v[p] = h->v[c]; h->v[c] = tmp; c = p;
    }
}
static evt hpop(heap_t *h) {
    evt top = h->v[0];
    h->n--;
    if (h->n > 0) {
        h->v[0] = h->v[h->n];
        size_t p = 0;
        for (;;) {
            size_t s = p, l = 2 * p + 1, r = 2 * p + 2;
            if (l < h->n && ev_less(&h->v[l], &h->v[s])) s = l;
            if (r < h->n && ev_less(&h->v[r], &h->v[s])) s = r;
            if (s == p) break;
            evt tmp = h->v[p]; h->v[p] = h->v[s]; h->v[s] = tmp; p = s;
        }
    }
    return top;
}

/* ------------------------------------------------------------ per track -- */
typedef struct {
    double *px, *py, *pz, *tb;
    int8_t *sp;
    uint8_t *alive;
    heap_t h;
} track_ws;

typedef struct {
    double tl[7][5];
    uint64_t rxn[NRX], reacted, pairs, events;
} track_acc;

/* the 16 log-spaced times of the per-track curves: 10^(-3 + 0.4 k) ns */
static double T16[16];

static void run_track(const float *rad, const uint64_t *idx, uint32_t n, uint32_t pid, uint32_t h2init,
                      uint32_t cap, const irt_rng *g0, track_ws *w, track_acc *acc, float *curve) {
    irt_rng g = *g0;
    g.pid = pid;
    uint32_t cnt[NSP] = {0};
    /* load + displacement (:475-537) */
    for (uint32_t k = 0; k < n; ++k) {
        const float *e = rad + 4 * idx[k];
        double x = e[0], y = e[1], z = e[2];
        int s = (int)lrintf(e[3]) % 8;
        w->alive[k] = 1;
        w->tb[k] = 0;
        uint32_t blk = 0, wi = 4;
        om_u4 wb = {{0, 0, 0, 0}};
        double sigma = 0;
        int disp = 0;
#define NEXTD(out) do { uint32_t a_, b_; if (wi == 4) { wb = om_philox(blk++, k, pid, 2u, g.k0, g.k1); wi = 0; } \
                        a_ = wb.v[wi++]; b_ = wb.v[wi++]; out = om_u01d(a_, b_); } while (0)
        if (s == 5) { w->sp[k] = 1; }
        else if (s == 0 || s == 3) {
            w->sp[k] = (int8_t)s;
            double u; NEXTD(u);
            if (u < 0.5) { disp = 1; sigma = C.sig_oh; }
        } else if (s == 1) { w->sp[k] = 1; disp = 1; sigma = C.sig_eaq; }
        else if (s == 2) { w->sp[k] = 2; disp = 1; sigma = C.sig_h; }
        else if (s == 6) { w->sp[k] = 5; }
        else { w->alive[k] = 0; w->sp[k] = (int8_t)s; }
        if (disp) {
            double c6[3];
            for (int ax = 0; ax < 3; ++ax) {
                double r1, r2, r3, r4, r5, r6;
                NEXTD(r1); NEXTD(r2); NEXTD(r3); NEXTD(r4); NEXTD(r5); NEXTD(r6);
                c6[ax] = (r1 + r2 + r3 + r4 + r5 + r6 - 3) * 1.4142135623730951;
            }
            x += sigma * c6[0]; y += sigma * c6[1]; z += sigma * c6[2];
        }
#undef NEXTD
        w->px[k] = x; w->py[k] = y; w->pz[k] = z;
        if (w->alive[k] && w->sp[k] >= 0 && w->sp[k] < NSP) cnt[w->sp[k]]++;
    }
    /* initial pairing (:539-558) */
    w->h.n = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (!w->alive[i]) continue;
        int si = w->sp[i];
        double Di = IRT_D[si];
        for (uint32_t j = i + 1; j < n; ++j) {
            if (!w->alive[j]) continue;
            int sj = w->sp[j];
            int ri = C.map[si * NSP + sj];
            if (ri < 0) continue;
            double dx = w->px[i] - w->px[j], dy = w->py[i] - w->py[j], dz = w->pz[i] - w->pz[j];
            double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 > C.r_cut2) continue;
            acc->pairs++;
            double r0 = sqrt(r2);
            om_u4 u4 = om_philox(j >> 2, i, pid, 3u, g.k0, g.k1);
            double U = om_u01d32(u4.v[j & 3]);
            double t = sample_irt(&g, i, j, r0, ri, Di + IRT_D[sj], U);
            if (t >= 0 && t < 1000) hpush(&w->h, t, (int)i, (int)j);
        }
    }
    /* event loop (:566-660) */
    uint32_t ntot = n;
    double h2 = (double)h2init;
    int cp = 0, c16 = 0;
    while (w->h.n > 0) {
        evt ev = hpop(&w->h);
        acc->events++;
        while (cp < 7 && ev.t >= CHECKPOINTS[cp]) {
            acc->tl[cp][0] += cnt[0]; acc->tl[cp][1] += cnt[1]; acc->tl[cp][2] += cnt[2];
            acc->tl[cp][3] += cnt[4]; acc->tl[cp][4] += h2;
            cp++;
        }
        while (curve && c16 < 16 && ev.t >= T16[c16]) {
            float *c = curve + 5 * c16;
            c[0] = (float)cnt[0]; c[1] = (float)cnt[1]; c[2] = (float)cnt[2]; c[3] = (float)cnt[4]; c[4] = (float)h2;
            c16++;
        }
        int i = ev.a, j = ev.b;
        if (!w->alive[i] || !w->alive[j]) continue;
        int si = w->sp[i], sj = w->sp[j];
        int ri = C.map[(si < sj ? si : sj) * NSP + (si < sj ? sj : si)];
        if (ri < 0) continue;
        w->alive[i] = 0; w->alive[j] = 0;
        cnt[si]--; cnt[sj]--;
        acc->reacted++;
        acc->rxn[ri]++;
        if (ri == 3 || ri == 4 || ri == 6) h2 += 1;
        int np = RXN[ri].np;
        if (np == 0) continue;
        double sqDi = sqrt(IRT_D[si]), sqDj = sqrt(IRT_D[sj]);
        double ww = sqDi + sqDj;
        double mx = (sqDj * w->px[i] + sqDi * w->px[j]) / ww;
        double my = (sqDj * w->py[i] + sqDi * w->py[j]) / ww;
        double mz = (sqDj * w->pz[i] + sqDi * w->pz[j]) / ww;
        for (int pp = 0; pp < np; ++pp) {
            int nsp = RXN[ri].prods[pp];
            uint32_t id = ntot;
            if (id >= cap) break;
            w->sp[id] = (int8_t)nsp; w->alive[id] = 1; w->tb[id] = ev.t;
            if (np == 1) { w->px[id] = mx; w->py[id] = my; w->pz[id] = mz; }
            else if (pp == 0) { w->px[id] = w->px[i]; w->py[id] = w->py[i]; w->pz[id] = w->pz[i]; }
            else { w->px[id] = w->px[j]; w->py[id] = w->py[j]; w->pz[id] = w->pz[j]; }
            cnt[nsp]++;
            ntot++;
            /* pairWithAlive (:430-465) */
            double Di = IRT_D[nsp];
            if (Di == 0) continue;
            for (uint32_t jj = 0; jj < ntot; ++jj) {
                if (jj == id || !w->alive[jj]) continue;
                int s2 = w->sp[jj];
                int r2i = C.map[nsp * NSP + s2];
                if (r2i < 0) continue;
                double Dj = IRT_D[s2];
                double dt = ev.t - w->tb[jj];
                acc->pairs++;
                double xj = w->px[jj], yj = w->py[jj], zj = w->pz[jj];
                om_u4 q0 = om_philox(id, jj, pid, 5u, g.k0, g.k1);
                if (dt > 0) {
                    double sig = sqrt(2.0 * Dj * dt);
                    om_u4 q1 = om_philox(id, jj, pid, 5u | (1u << 4), g.k0, g.k1);
                    double nrm[3];
                    for (int b = 0; b < 3; ++b) {
                        double u1 = om_u01d32(q0.v[b]), u2 = om_u01d32(q1.v[b]);
                        nrm[b] = sqrt(-2 * om_log(u1 + 1e-30)) * om_cos(6.2831853 * u2);
                    }
                    xj += nrm[0] * sig; yj += nrm[1] * sig; zj += nrm[2] * sig;
                }
                double dx = w->px[id] - xj, dy = w->py[id] - yj, dz = w->pz[id] - zj;
                double r2 = dx * dx + dy * dy + dz * dz;
                if (r2 > C.r_cut2) continue;
                double r0 = sqrt(r2);
                double U = om_u01d32(q0.v[3]);
                double t = sample_irt(&g, id, jj, r0, r2i, Di + Dj, U);
                if (t >= 0) {
                    double ta = ev.t + t;
                    if (ta < 1000) hpush(&w->h, ta, (int)(jj < id ? jj : id), (int)(jj < id ? id : jj));
                }
            }
        }
    }
    while (cp < 7) {
        acc->tl[cp][0] += cnt[0]; acc->tl[cp][1] += cnt[1]; acc->tl[cp][2] += cnt[2];
        acc->tl[cp][3] += cnt[4]; acc->tl[cp][4] += h2;
        cp++;
    }
    while (curve && c16 < 16) {
        float *c = curve + 5 * c16;
        c[0] = (float)cnt[0]; c[1] = (float)cnt[1]; c[2] = (float)cnt[2]; c[3] = (float)cnt[4]; c[4] = (float)h2;
        c16++;
    }
}

int orc_irt(const float *rad, uint64_t rad_n, uint32_t n_therm, double E_eV, uint64_t seed,
            orc_irt_out *o, int nthreads) {
    init_consts();
    float *curves = o->curves;
    uint64_t curves_cap = o->curves_cap;
    memset(o, 0, sizeof *o);
    o->curves = curves; o->curves_cap = curves_cap;
    if (curves) memset(curves, 0, curves_cap * 80 * sizeof(float));
    for (int k = 0; k < 16; ++k) T16[k] = pow(10.0, -3.0 + 0.4 * k);
    /* group by pid in order of first appearance (:380-394) */
    uint32_t maxpid = 0;
    for (uint64_t i = 0; i < rad_n; ++i) {
        int w = (int)lrintf(rad[4 * i + 3]);
        uint32_t pid = (uint32_t)(w / 8);
        if (pid > maxpid) maxpid = pid;
    }
    uint32_t npid = maxpid + 1;
    uint32_t *count = (uint32_t *)calloc(npid, 4), *h2 = (uint32_t *)calloc(npid, 4);
    uint64_t *first = (uint64_t *)malloc(npid * 8ull);
    for (uint32_t p = 0; p < npid; ++p) first[p] = UINT64_MAX;
    for (uint64_t i = 0; i < rad_n; ++i) {
        int w = (int)lrintf(rad[4 * i + 3]);
        int sp = w % 8;
        if (sp < 0 || sp == 4) continue;
        uint32_t pid = (uint32_t)(w / 8);
        if (sp == 7) { h2[pid]++; continue; }
        if (first[pid] == UINT64_MAX) first[pid] = i;
        count[pid]++;
    }
    uint64_t *off = (uint64_t *)malloc((npid + 1) * 8ull);
    off[0] = 0;
    uint32_t maxN = 0, ntr = 0;
    for (uint32_t p = 0; p < npid; ++p) {
        off[p + 1] = off[p] + count[p];
        if (count[p] > maxN) maxN = count[p];
        if (count[p]) ntr++;
    }
    uint64_t *idx = (uint64_t *)malloc((off[npid] ? off[npid] : 1) * 8);
    uint64_t *cur = (uint64_t *)malloc(npid * 8ull);
    memcpy(cur, off, npid * 8ull);
    for (uint64_t i = 0; i < rad_n; ++i) {
        int w = (int)lrintf(rad[4 * i + 3]);
        int sp = w % 8;
        if (sp < 0 || sp == 4 || sp == 7) continue;
        uint32_t pid = (uint32_t)(w / 8);
        idx[cur[pid]++] = i;
    }
    uint32_t cap = maxN * 2 + 512;
    irt_rng g = {(uint32_t)seed, (uint32_t)(seed >> 32), 0};
    if (nthreads < 1) nthreads = 1;
    track_acc *accs = (track_acc *)calloc((size_t)nthreads, sizeof(track_acc));
#pragma omp parallel num_threads(nthreads)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        track_ws w;
        memset(&w, 0, sizeof w);
        w.px = (double *)malloc(cap * 8ull); w.py = (double *)malloc(cap * 8ull);
        w.pz = (double *)malloc(cap * 8ull); w.tb = (double *)malloc(cap * 8ull);
        w.sp = (int8_t *)malloc(cap); w.alive = (uint8_t *)malloc(cap);
#pragma omp for schedule(dynamic, 1)
        for (int64_t p = 0; p < (int64_t)npid; ++p) {
            if (!count[p]) continue;
            float *curve = (o->curves && (uint64_t)p < o->curves_cap) ? o->curves + 80ull * (uint64_t)p : NULL;
            run_track(rad, idx + off[p], count[p], (uint32_t)p, h2[p], cap, &g, &w, &accs[tid], curve);
        }
        free(w.px); free(w.py); free(w.pz); free(w.tb); free(w.sp); free(w.alive); free(w.h.v);
    }
    for (int t = 0; t < nthreads; ++t) {
        for (int c = 0; c < 7; ++c) for (int s = 0; s < 5; ++s) o->tl[c][s] += accs[t].tl[c][s];
        for (int r = 0; r < NRX; ++r) o->rxn_counts[r] += accs[t].rxn[r];
        o->n_reacted += accs[t].reacted; o->n_pairs += accs[t].pairs; o->n_events += accs[t].events;
    }
    o->n_tracks = ntr;
    double dep = (double)n_therm * E_eV;
    double per100 = dep / 100;
    for (int c = 0; c < 7; ++c)
        for (int s = 0; s < 5; ++s) o->G[c][s] = per100 > 0 ? o->tl[c][s] / per100 : 0;
    free(accs); free(idx); free(cur); free(off); free(first); free(count); free(h2);
    return 0;
}
