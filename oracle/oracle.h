/* oracle/oracle.h -- CPU oracle of the electron-transport -> IRT -> scoring path.
 *
 * TEST INFRASTRUCTURE ONLY: a plain-C restatement of the reference's
 * algorithms, used by tests/, the smoke check and the benchmark's CPU-baseline
 * leg to check the CUDA product path.  Nothing in the product links it.
 *
 * Parity status: the cross-section tables are pinned bit for bit (SHA-256 of
 * every array against public/cross_sections.wgsl); geometry, constants, the
 * rad_buf encoding and the IRT known-answer smoke case are pinned by the
 * reference's own unit tests; transport and IRT statistics are pinned against
 * the reference's published 10 keV outputs (validation/webgpu-results.json)
 * within statistical error, because the reference's GPU shaders and JS worker
 * cannot run here (WebGPU is a graphics API; no Node).
 */
#ifndef WGDNA_ORACLE_H
#define WGDNA_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- tables (public/cross_sections.wgsl, loaded from the committed blob) */
int orc_load_tables(const char *blob_path);

/* ---- transport: Phase A (primary.wgsl:113-663) + Phase B (secondary.wgsl:82-450) */
typedef struct {
    uint32_t np;            /* P.n */
    float box_nm;           /* P.box  (half width) */
    float ce_eV;            /* P.ce   (cutoff) */
    uint32_t max_steps;     /* P.ms   (65536) */
    float E_eV;             /* P.be */
    uint32_t max_sec;       /* P.max_sec */
    uint32_t vc;            /* P.vc   (128) */
    uint32_t max_rad;       /* P.max_rad */
    float start_half;       /* P.start_half */
    uint32_t dna_enable;    /* P.dna_enable */
    uint32_t dna_grid_n;
    float dna_rise, dna_spacing, dna_x0, dna_r_bb;
    uint32_t sec_steps;     /* MAX_SEC_STEPS (2000), constants.ts:66 */
    uint32_t rng_mode;      /* 0 = Philox (build), 1 = reference xoshiro */
    uint64_t seed;          /* Philox key (mode 0) / floor(E) seed (mode 1) */
    uint32_t pid_base;      /* global id of primary 0 */
    const float *E_per_primary;  /* optional per-primary energy (NULL: E_eV) */
} orc_transport_params;

typedef struct {
    float *results;         /* np*8 words: path, prod, fE, ni(u32), nx(u32), esc(u32), mx, pad */
    uint32_t *dose;         /* vc^3 (may be NULL) */
    uint32_t counters[8];
    uint32_t sec_stats[8];
    uint32_t dbg[8];
    float *rad;             /* 4*rad_n floats, canonical order (malloc'd; orc_free) */
    uint64_t *rad_key;      /* rad_n keys (pid<<34 | sub<<17 | seq) */
    uint64_t rad_n;
    uint64_t dep_units;     /* sum of all in-grid u32(dep*100) deposits */
    double dep_eV_f64;      /* sum of every deposit (f64), in or out of the grid */
    uint64_t sec_n;         /* secondaries kept: min(counters[6] emitted, max_sec) */
    uint64_t steps;         /* electron steps taken (primary + secondary) */
} orc_transport_out;

int orc_transport(const orc_transport_params *p, orc_transport_out *o, int nthreads);
void orc_free(void *ptr);

/* ---- IRT chemistry worker (public/irt-worker.js:370-699) */
typedef struct {
    double tl[7][5];        /* counts at the 7 checkpoints: OH, eaq, H, H2O2, H2 */
    double G[7][5];         /* G values per 100 eV of n_therm*E_eV */
    uint64_t rxn_counts[9];
    uint64_t n_reacted;
    uint64_t n_pairs;       /* initial reactive pairs inside R_CUT + (product, partner) reactive pairs */
    uint64_t n_tracks;
    uint64_t n_events;      /* heap pops */
    float *curves;          /* optional, (max pid + 1) x 16 x 5: per-track counts of OH, eaq, H, H2O2, H2
                               at t_k = 10^(-3 + 0.4 k) ns, k = 0..15 (filled when not NULL) */
    uint64_t curves_cap;    /* tracks the curves buffer holds */
} orc_irt_out;

int orc_irt(const float *rad_buf, uint64_t rad_n, uint32_t n_therm, double E_eV,
            uint64_t seed, orc_irt_out *o, int nthreads);
/* per-reaction constants as computed at irt-worker.js:240-279 (sigma, sigma_eff,
 * rc, kdif, kact, prob) for tests */
void orc_irt_rxn_table(double out[9][6]);

/* ---- scoring (src/scoring/ssb-dsb.ts, src/physics/dna-geometry.ts) */
typedef struct {
    uint32_t grid_N, n_bp_per, n_fibers, n_bp;
    double rise, r_bb, spacing_nm, x0, L_nm;
    float *fy, *fz, *rbb0, *rbb1;
} orc_dna;

int orc_build_dna(double L_nm, uint32_t grid_N, double spacing_nm, orc_dna *d);
void orc_free_dna(orc_dna *d);

typedef struct {
    uint64_t ssb, ssb0, ssb1, candidates, in_reach;
    uint32_t lcg_state;     /* LCG state after the pass */
} orc_ssb_out;

/* scoreDirectSSB_events (ssb-dsb.ts:135-217); hits: 2*n_bp bytes, OR-ed into */
int orc_score_direct(const orc_dna *d, const float *rad, uint64_t rad_n, uint32_t lcg_state,
                     uint8_t *hits, orc_ssb_out *o);
/* scoreIndirectSSB (ssb-dsb.ts:43-121) */
int orc_score_indirect(const orc_dna *d, const float *pos, const uint32_t *alive, uint64_t n,
                       uint32_t lcg_state, uint8_t *hits, orc_ssb_out *o);
/* clusterDSB (ssb-dsb.ts:348-407) */
int orc_cluster_dsb(const orc_dna *d, const uint8_t *hits, uint64_t *dsb, double *dsb_expected,
                    uint64_t *ssb0, uint64_t *ssb1);

/* dose-grid scoring (ssb-dsb.ts:227-334) and dose reductions (dose.ts:13-85) */
double orc_voxel_ssb(const orc_dna *d, const uint32_t *dose, uint32_t vc, double box_nm, float *lambda);
double orc_expected_dsb_local(const orc_dna *d, const float *lambda, const uint8_t *hits);
double orc_dose_sum_ev(const uint32_t *dose, uint64_t n);
void orc_dose_projection(const uint32_t *dose, uint32_t vc, int axis, float *proj);

/* grid-hash chemistry backend (src/shaders/chemistry.wgsl, schedule.ts:38-46) on
 * the first n rad_buf entries: final pos (n x 4: x, y, z, kind) and alive,
 * counts[checkpoint][OH, eaq, H alive, H2O2 made, H2 made] at t = 0 and the
 * 7 checkpoints */
int orc_chem_grid(const float *rad, uint32_t n, uint64_t seed, float *pos, uint32_t *alive, uint32_t counts[8][5]);

/* elem.c: the elementary functions of om.h over a vector (fn codes in elem.c) */
int orc_elem(int fn, const double *x, double *y, uint64_t n);

#ifdef __cplusplus
}
#endif
#endif
