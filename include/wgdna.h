/* wgdna.h -- C ABI of the B200 path for allaunthefox/webgpu-dna's hot path:
 * electron transport in liquid water -> Karamitros 9-reaction IRT chemistry ->
 * SSB/DSB scoring on the 21x21 B-DNA fibre grid.
 *
 * Plain C types only (no CUDA or torch types).  Every function returns an int
 * status (WGDNA_OK = 0, negative on error) and wgdna_last_error() describes the
 * last error of the calling thread.  A context owns one CUDA stream and the
 * device buffers of one call at a time; it is not thread-safe.  Host buffers
 * are caller-owned.  Buffer overflows are not errors: they are counted in the
 * *_dropped fields, as the reference counts sec_dropped / rad_dropped
 * (src/gpu/dispatch.ts:124-126,190-192).  Device-side bounded waits that give
 * up set device_error and make the call return WGDNA_ERR_DEVICE.
 */
#ifndef WGDNA_H
#define WGDNA_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WGDNA_OK 0
#define WGDNA_ERR_ARG (-1)
#define WGDNA_ERR_CUDA (-2)
#define WGDNA_ERR_TABLES (-3)
#define WGDNA_ERR_CAPACITY (-4)
#define WGDNA_ERR_DEVICE (-5)
#define WGDNA_ERR_NOMEM (-6)
#define WGDNA_ERR_STATE (-7)

typedef struct wgdna_ctx wgdna_ctx;

/* Context configuration.  Replaces initGPU + allocateBuffers
 * (src/gpu/device.ts:11-33, src/gpu/buffers.ts:48-85): the buffer caps are the
 * reference's MAX_SEC / MAX_RAD / VC (src/physics/constants.ts:51-60). */
typedef struct {
    int device;                 /* CUDA device ordinal */
    const char *tables_path;    /* cross_sections.bin; NULL = next to the library */
    uint32_t max_primaries;     /* largest np per call */
    uint32_t max_sec;           /* MAX_SEC (5,000,000) */
    uint64_t max_rad;           /* MAX_RAD (16,000,000) */
    uint32_t vc;                /* dose grid edge VC (128) */
    uint32_t reserved;
} wgdna_cfg;

void wgdna_default_cfg(wgdna_cfg *cfg);
int wgdna_create(const wgdna_cfg *cfg, wgdna_ctx **out);      /* ensurePipelines, app.ts:65-84 */
void wgdna_destroy(wgdna_ctx *ctx);
const char *wgdna_last_error(void);
int wgdna_version(void);
/* Run the context's work on a caller's cudaStream_t (NULL = the context's own). */
int wgdna_set_stream(wgdna_ctx *ctx, void *cuda_stream);

/* Launch and scheduling shapes of the kernels.  No counterpart in the
 * reference (WebGPU picks none of these).  They change how work is spread over
 * the GPU, never the results: every particle, pair and track draws from its
 * own random stream.  wgdna_create reads them from data/tuning.txt next to the
 * library when that file exists (written by `python -m wgdna.autotune`, one
 * "key value" line per field below), else uses the defaults shown. */
typedef struct {
    uint32_t transport_ctas_per_sm;  /* resident transport CTAs per SM, 0 = as many as fit (2) */
    uint32_t prim_take;              /* primaries a transport warp may start per iteration (2), 1..32 */
    uint32_t stash_keep;             /* secondaries a warp keeps when its stash spills (16) */
    uint32_t stash_spill;            /* stash level that spills to the global queue (32), <= 48;
                                      * 0 = no stash: every secondary goes to the global queue */
    uint32_t queue_poll;             /* a busy warp polls the global queue every queue_poll iterations (8),
                                      * a power of two <= 1024 */
    uint32_t irt_init_blocks_per_sm; /* resident blocks of the IRT pairing kernel per SM, 0 = as many as fit */
    uint32_t irt_loop_blocks_per_sm; /* resident blocks of the IRT event kernel per SM, 0 = as many as fit */
} wgdna_tuning;
void wgdna_default_tuning(wgdna_tuning *t);
int wgdna_get_tuning(wgdna_ctx *ctx, wgdna_tuning *t);
int wgdna_set_tuning(wgdna_ctx *ctx, const wgdna_tuning *t);

/* Bounds of the device-side waits.  No counterpart in the reference (its
 * WebGPU queue has no device-side waits); for hosts that want a shorter
 * watchdog and for failure-detection tests.  queue_ns: a transport lane's wait
 * for a queued secondary to be published (default 2 s); idle_ns: a transport
 * warp's wait without work before the run ends (default 30 s); mma_ns: a
 * surrogate kernel's wait for its tensor-core step (default 1 s).  0 keeps the
 * default.  A wait that runs out sets a bit of the stage's device_error and the
 * call returns WGDNA_ERR_DEVICE; the context stays usable.  test_flags is 0 in
 * normal use; WGDNA_TEST_UNPUBLISHED makes the transport publish its queued
 * secondaries under an epoch that no consumer waits for (the queue wait runs
 * out), WGDNA_TEST_MMA_WAIT makes each surrogate tile give up its first
 * tensor-core wait before polling (the tile then waits, at most 1 s, for the
 * tensor cores to finish before it reads or frees tensor memory). */
#define WGDNA_TEST_UNPUBLISHED 1u
#define WGDNA_TEST_MMA_WAIT 2u
int wgdna_set_wait_limits(wgdna_ctx *ctx, uint64_t queue_ns, uint64_t idle_ns, uint64_t mma_ns,
                          uint32_t test_flags);

/* ---------------------------------------------------------------- Phase A+B */
/* The uniform structs P (src/gpu/dispatch.ts:13-42) and SP (dispatch.ts:45-70). */
typedef struct {
    uint32_t np;                /* P.n */
    float E_eV;                 /* P.be */
    float box_nm;               /* P.box (half width) */
    float ce_eV;                /* P.ce */
    uint32_t max_steps;         /* P.ms (65536) */
    uint32_t sec_steps;         /* MAX_SEC_STEPS (2000), constants.ts:66 */
    float start_half;           /* P.start_half */
    uint32_t dna_enable;        /* P.dna_enable */
    uint32_t dna_grid_n;
    float dna_rise, dna_spacing, dna_x0, dna_r_bb;
    uint32_t pid_base;          /* global id of primary 0 (sharding); w = (pid_base+i)*8 + code */
    uint64_t seed;              /* Philox key */
    const float *E_per_primary; /* optional host array of np energies (eV); NULL = E_eV for all */
} wgdna_transport_params;

typedef struct {
    uint32_t counters[8];       /* primary.wgsl:24-35: OH, eaq, H, H3O+, DNA hits, H2, sec idx, rad idx */
    uint32_t sec_stats[8];      /* [1] cutoff, [2] bounds, [3] steps, [4] tertiary ions */
    uint32_t dbg[8];            /* [0] ions, [1] exc, [2] escaped, [3] primaries, [4] sum W*10, [5] dose-grid atomics */
    uint64_t rad_n_raw, rad_n_stored, rad_dropped;
    uint64_t sec_n_raw, sec_n, sec_dropped;
    uint64_t dep_units;         /* sum of the dose grid (100 units per eV) */
    double dep_eV_f64;          /* every deposit summed in f64 */
    uint64_t steps;             /* electron steps */
    float ms_transport;         /* CUDA-event time of the transport kernel */
    float ms_canon;             /* CUDA-event time of rad_buf canonicalisation */
    uint32_t device_error;
    uint32_t n_therm;           /* primaries that did not escape */
} wgdna_transport_stats;

/* Phase A + Phase B (dispatch.ts:106-145) into device memory of the context.
 * rad_buf is left in canonical order: grouped by primary, the primary's own
 * entries first, then each secondary's, each in emission order. */
int wgdna_transport(wgdna_ctx *ctx, const wgdna_transport_params *p, wgdna_transport_stats *st);
/* Readbacks of the last transport (dispatch.ts:148-240).  Any pointer may be
 * NULL.  results: np*8 words (R struct, primary.wgsl:9); dose: vc^3 u32;
 * rad: 4 floats per entry, at most rad_cap entries. */
int wgdna_transport_copy_out(wgdna_ctx *ctx, float *results, uint32_t *dose, float *rad,
                             uint64_t rad_cap, uint64_t *rad_n);
/* Both of the above in one call: the device part of runAtEnergy (dispatch.ts:85-240). */
int wgdna_run_transport(wgdna_ctx *ctx, const wgdna_transport_params *p, float *results,
                        uint32_t *dose, float *rad, uint64_t rad_cap, uint64_t *rad_n,
                        wgdna_transport_stats *st);

/* ---------------------------------------------------------------- Phase C */
typedef struct {
    double counts[7][5];        /* alive OH, eaq, H, H2O2(+prod), H2 at 1,10,100 ps,1,10,100 ns,1 us */
    double G[7][5];             /* per 100 eV of n_therm * E_eV (irt-worker.js:670-682) */
    uint64_t rxn_counts[9];     /* irt-worker.js:685-694 order */
    uint64_t n_reacted, n_tracks, n_pairs, n_events;
    uint64_t n_particles, n_init_events;   /* tracked species loaded; events from the initial pairing */
    uint64_t chem_n;
    float ms;                   /* whole IRT on the device */
    float ms_load, ms_pairing, ms_events;   /* its kernels: load + displacement, initial pairing, event loop */
    uint32_t device_error;
    float ms_sort;              /* ordering of the tracks and sort of their initial events (before the event loop) */
} wgdna_irt_result;

/* runChemistryWorker (src/chemistry/worker.ts:32-87, public/irt-worker.js:370-699)
 * on a host rad_buf (4 floats per entry, w = pid*8 + species code). */
int wgdna_run_irt(wgdna_ctx *ctx, const float *rad_buf, uint64_t rad_n, uint32_t n_therm,
                  double E_eV, uint64_t seed, wgdna_irt_result *out);
/* The same on the rad_buf left in device memory by the last wgdna_transport. */
int wgdna_irt(wgdna_ctx *ctx, uint32_t n_therm, double E_eV, uint64_t seed, wgdna_irt_result *out);
/* Per-track G(t) curves (no reference counterpart: the surrogate chemistry
 * trains on them).  When enabled, every following IRT call records for each
 * track (primary id - pid_base) the counts of OH, eaq, H, H2O2 and H2 at the
 * 16 times t_k = 10^(-3 + 0.4 k) ns, k = 0..15, with the checkpoint rule of
 * irt-worker.js:566-580.  wgdna_irt_curves copies the last call's
 * n_tracks x 16 x 5 floats (NULL out: only report n_tracks). */
int wgdna_irt_record_curves(wgdna_ctx *ctx, int enable);
int wgdna_irt_curves(wgdna_ctx *ctx, float *out, uint64_t cap_tracks, uint64_t *n_tracks);
/* Per-reaction constants of the 9-reaction table (irt-worker.js:240-279), host
 * only: out[r] = {sigma, sigma_eff, rc, kdif, kact, prob} in nm / nm^3 ns^-1;
 * the worker reports sigma and rc in its rxn_info (irt-worker.js:690-694). */
int wgdna_reaction_table(double out[9][6]);

/* The reference's 'gpu' chemistry backend (src/shaders/chemistry.wgsl,
 * src/chemistry/schedule.ts:33-247): diffusion in fixed steps, a spatial hash
 * of 1.5 nm cells, contact reactions with compare-and-swap claims (so results
 * vary with thread timing, as in the reference), on the first
 * min(rad_n, 8,000,000) entries of rad (NULL: the last transport's rad_buf).
 * Checkpoints: t = 0 and 1 ps, 10 ps, 100 ps, 1 ns, 10 ns, 100 ns, 1 us.
 * pos (x, y, z, kind) and alive of the radicals when cap >= chem_n, for
 * scoreIndirectSSB (wgdna_score_indirect); either may be NULL. */
typedef struct {
    uint32_t counts[8][5];      /* alive OH, eaq, H; H2O2 and H2 made */
    double G[8][5];             /* per 100 eV of n_therm * E_eV * chem_n / rad_n */
    uint64_t chem_n;
    double deposited_eV;
    float ms;
} wgdna_chem_grid_result;
int wgdna_chem_grid(wgdna_ctx *ctx, const float *rad, uint64_t rad_n, uint32_t n_therm, double E_eV,
                    uint64_t seed, wgdna_chem_grid_result *out, float *pos, uint32_t *alive, uint64_t cap);

/* ---------------------------------------------------------------- scoring */
typedef struct {
    uint32_t grid_N, n_bp_per, n_fibers, n_bp;
    double rise, r_bb, spacing_nm, x0, L_nm;
} wgdna_dna_info;

/* buildDNATarget (src/physics/dna-geometry.ts:16-68), host only.  Array
 * pointers may be NULL; sizes: fy/fz grid_N^2, rbb0/rbb1 2*n_bp_per floats. */
int wgdna_build_dna_target(double L_nm, uint32_t grid_N, double spacing_nm, float *fy, float *fz,
                           float *rbb0, float *rbb1, wgdna_dna_info *info);
/* Upload the target used by the scoring entry points (default 3000 nm, 21, 150 nm). */
int wgdna_set_dna_target(wgdna_ctx *ctx, double L_nm, uint32_t grid_N, double spacing_nm);

typedef struct {
    uint64_t ssb, ssb0, ssb1, candidates, in_reach;
    uint32_t lcg_state;         /* makeSsbRng state after the pass */
    float ms;
} wgdna_ssb_result;

typedef struct {
    uint64_t dsb, ssb0, ssb1;
    double dsb_expected;
    float ms;
} wgdna_dsb_result;

/* scoreDirectSSB_events (src/scoring/ssb-dsb.ts:135-217).  hits (2*n_bp bytes)
 * is read and OR-ed into when not NULL, like the Uint8Array the reference
 * combines later (combineHits, ssb-dsb.ts:413-418). */
int wgdna_score_direct(wgdna_ctx *ctx, const float *rad, uint64_t rad_n, uint32_t lcg_state,
                       uint8_t *hits, wgdna_ssb_result *out);
/* scoreIndirectSSB (ssb-dsb.ts:43-121). */
int wgdna_score_indirect(wgdna_ctx *ctx, const float *pos, const uint32_t *alive, uint64_t n,
                         uint32_t lcg_state, uint8_t *hits, wgdna_ssb_result *out);
/* clusterDSB (ssb-dsb.ts:348-407). */
int wgdna_cluster_dsb(wgdna_ctx *ctx, const uint8_t *hits, wgdna_dsb_result *out);
/* Direct SSB + DSB clustering of the rad_buf left by the last wgdna_transport
 * (app.ts:182-185 with the worker backend, where indirect scoring is skipped). */
int wgdna_score(wgdna_ctx *ctx, uint32_t lcg_state, wgdna_ssb_result *ssb, wgdna_dsb_result *dsb);

/* Dose-grid reductions and dose-based scoring.  dose: a host vc^3 grid, or
 * NULL for the grid of the last wgdna_transport on the device. */
/* sumDoseEV (src/scoring/dose.ts:13-17): the grid's sum / 100. */
int wgdna_dose_sum(wgdna_ctx *ctx, const uint32_t *dose, double *eV);
/* The projection sums of renderDoseProjection (dose.ts:61-85): axis 0 sums over
 * z into proj[y][x], axis 1 over x into proj[z][y]; vc^2 floats. */
int wgdna_dose_projection(wgdna_ctx *ctx, const uint32_t *dose, int axis, float *proj);
/* scoreDirectSSB (ssb-dsb.ts:227-283): expected direct SSBs from the voxel dose
 * at the backbone sites of the context's DNA target; lambda (2 * n_bp floats,
 * may be NULL) receives the per-site expectations and stays on the device. */
int wgdna_score_voxel_ssb(wgdna_ctx *ctx, const uint32_t *dose, double box_nm, float *lambda,
                          double *direct_expected);
/* expectedDSBLocal (ssb-dsb.ts:285-334) on lambda (NULL: the last
 * wgdna_score_voxel_ssb) and indirect hit bytes (NULL: none). */
int wgdna_expected_dsb_local(wgdna_ctx *ctx, const float *lambda, const uint8_t *hits, double *dsb_expected);

/* ---------------------------------------------------------------- surrogate */
/* Learned chemistry (no reference counterpart): an MLP 64 -> 128 -> 128 ->
 * 128 -> 80 with GELU, bf16 weights and f32 accumulation on the tensor cores,
 * mapping a track descriptor to the track's G(t) (per 100 eV of the track's
 * energy) at the 16 curve times of wgdna_irt_curves, species-major within a
 * time: out[5 k + s], s = OH, eaq, H, H2O2, H2.  The IRT stays the reference
 * and the check: the model is trained on the IRT's own curves.
 *
 * Parameters (WGDNA_SG_NPARAM floats): W1 [128][64], b1 [128], W2 [128][128],
 * b2, W3 [128][128], b3, W4 [80][128], b4 [80].  Standardisation
 * (2*64 + 2*80 floats): input mean, input std, output mean, output std; the
 * network sees (x - mean) / std and predicts (G - mean) / std. */
#define WGDNA_SG_IN 64
#define WGDNA_SG_OUT 80
#define WGDNA_SG_NPARAM 51664
/* Descriptors of the tracks (primaries) of the last wgdna_transport, 64 floats
 * each (layout in webgpu-dna_b200/csrc/surrogate.cu); out may be NULL. */
int wgdna_track_descriptors(wgdna_ctx *ctx, float *out, uint64_t cap_tracks, uint64_t *n_tracks);
/* Random (Glorot, seeded) weights, identity standardisation, fresh Adam state. */
int wgdna_surrogate_init(wgdna_ctx *ctx, uint64_t seed);
/* Read and/or replace the f32 parameters (either pointer may be NULL). */
int wgdna_surrogate_params(wgdna_ctx *ctx, float *get, const float *set);
int wgdna_surrogate_norm(wgdna_ctx *ctx, float *get, const float *set);
/* Training data: n descriptors (n x 64) and IRT curves as G values (n x 80),
 * standardised with the current norm and kept on the device. */
int wgdna_surrogate_load(wgdna_ctx *ctx, const float *X, const float *G, uint64_t n);
/* Adam (beta 0.9 / 0.999) on the mean squared error of the standardised
 * outputs, shuffled full batches; losses[epoch] may be NULL. */
int wgdna_surrogate_train(wgdna_ctx *ctx, uint32_t epochs, uint32_t batch, float lr, uint64_t seed,
                          float *losses);
/* Loss and gradient over the first n loaded rows, without an update. */
int wgdna_surrogate_grad(wgdna_ctx *ctx, uint64_t n, float *grad, double *loss);
/* G for n host descriptors (X) or, X NULL, for the last descriptors; G n x 80 (may be NULL). */
int wgdna_surrogate_predict(wgdna_ctx *ctx, const float *X, uint64_t n, float *G);
/* Descriptors + prediction + energy-weighted sum for the last transport: the
 * surrogate's G(t) of the whole batch, G[16][5]; ms = device time. */
int wgdna_surrogate_chemistry(wgdna_ctx *ctx, double *G, float *ms);

/* ---------------------------------------------------------------- sharded runs */
/* One process per GPU, each with its block of primary ids (pid_base).  The
 * exchange steps need the context's device buffers: the dose grid (summed
 * over ranks), the hit bytes (OR-ed: MAX over ranks) and, for the exact
 * sharded direct-SSB scoring, a scoring pass that only reports its LCG draws
 * and leaves the hit bytes on the device, then clustering of the reduced
 * hits.  No reference counterpart: the reference runs on one device. */
typedef struct {
    uint32_t *dose;             /* vc^3 words */
    uint64_t dose_words;
    uint8_t *hits;              /* 2 * n_bp bytes (allocation rounded up to 4) */
    uint64_t hits_bytes;
    float *rad;                 /* canonical rad_buf of the last transport: rad_n x 4 */
    uint64_t rad_n;
    float *results;             /* n_primaries x 8 */
    uint32_t n_primaries;
    void *stream;               /* the context's cudaStream_t */
} wgdna_device_view;
int wgdna_device_views(wgdna_ctx *ctx, wgdna_device_view *v);
/* scoreDirectSSB_events of the last transport's rad_buf into zeroed device
 * hits: SSB counts, in_reach (= LCG draws) and the LCG state after them. */
int wgdna_score_draws(wgdna_ctx *ctx, uint32_t lcg_state, wgdna_ssb_result *ssb);
/* clusterDSB of the device hit bytes (after the caller's reduction). */
int wgdna_cluster_device(wgdna_ctx *ctx, wgdna_dsb_result *dsb);

/* Direct SSB scoring that allocates nothing.  No counterpart in the reference:
 * it serves callers that cannot call cudaMalloc (a host running under another
 * framework's memory pool or a fixed device-memory budget).  All pointers except
 * `dna` and `out` are device pointers owned by the caller: d_rad holds rad_n
 * entries (16-byte aligned), d_fy/d_fz/d_rbb0/d_rbb1 the target built by
 * wgdna_build_dna_target, and d_hits (4-byte aligned, 2*n_bp bytes rounded up
 * to a multiple of 4) is OR-ed into.  The scratch is a fixed 16.1 MB device
 * array that every GPU loading the library holds until exit; at most
 * 4,194,304 entries per call (larger lists fail with WGDNA_ERR_CAPACITY and
 * can be split where consecutive entries differ, chaining lcg_state and
 * hits).  The first call on a device looks up the array's device address, so
 * make it before any stream capture.  Calls share the array: calls that
 * overlap on the GPU race.  Runs on cuda_stream (NULL = the default stream)
 * and returns after the stream reaches the end of the call. */
int wgdna_score_direct_noalloc(const float *d_rad, uint64_t rad_n, const float *d_fy, const float *d_fz,
                               const float *d_rbb0, const float *d_rbb1, const wgdna_dna_info *dna,
                               uint32_t lcg_state, uint8_t *d_hits, void *cuda_stream, wgdna_ssb_result *out);

#ifdef __cplusplus
}
#endif
#endif
