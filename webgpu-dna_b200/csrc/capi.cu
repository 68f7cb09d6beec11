// capi.cu -- the C ABI (include/wgdna.h): context, buffers and entry points.
#include <dlfcn.h>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"

#include "chemgrid.cuh"
#include "dose.cuh"
#include "irt.cuh"
#include "scoring.cuh"
#include "surrogate_api.cuh"
#include "transport.cuh"

namespace wg {
int tables_load(const char* path, Tables* out, float** d_small, float2** d_xcw);
}

using namespace wg;

static thread_local char g_err[512];
void wg_set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}
extern "C" const char* wgdna_last_error(void) { return g_err; }
extern "C" int wgdna_version(void) { return 10000; }

struct wgdna_ctx {
    int device = 0;
    cudaStream_t stream = nullptr, own = nullptr;
    wgdna_cfg cfg{};
    Tables tab{};
    float* d_small = nullptr;
    float2* d_xcw = nullptr;
    // transport
    float* d_results = nullptr;
    uint32_t* d_dose = nullptr;
    float4* d_rad_raw = nullptr;
    unsigned long long* d_key = nullptr;
    float4* d_rad = nullptr;
    uint32_t* d_perm = nullptr;
    SecRec* d_secq = nullptr;
    DevState* d_st = nullptr;
    float* d_Eprim = nullptr;
    uint32_t seg_cap = 0;                 // entries of the pid arrays
    uint32_t* d_pid_cnt = nullptr;
    unsigned long long* d_pid_off = nullptr;
    uint32_t* d_pid_cur = nullptr;
    unsigned long long* d_red = nullptr;  // [0] dose sum [1] n_therm [2] seg max
    uint32_t* d_err = nullptr;            // canonicalisation / IRT / scoring error word
    uint32_t epoch = 0;
    int tblocks = 0;
    // bounds of the device-side waits (wgdna_set_wait_limits) and test switches
    unsigned long long wait_queue_ns = WG_QUEUE_WAIT_NS, wait_idle_ns = WG_IDLE_WAIT_NS, wait_mma_ns = WG_MMA_WAIT_NS;
    uint32_t test_flags = 0;
    wgdna_tuning tune{};                  // launch and scheduling shapes (wgdna_set_tuning)
    // last transport
    bool have_transport = false;
    uint32_t last_np = 0, last_nseg = 0, last_pid_base = 0, irt_pid_base = 0;
    float last_E = 0.0f;
    bool last_has_eprim = false;
    wg::SgState* sg = nullptr;           // surrogate chemistry (surrogate_api.cu)
    // dose-based scoring: an uploaded grid, per-site lambda, uploaded hits, f64 / u64 results
    uint32_t* d_dose_in = nullptr;
    float* d_lambda = nullptr;
    uint8_t* d_hits_in = nullptr;
    double* d_dres = nullptr;
    bool have_lambda = false;
    // grid-hash chemistry
    float4 *d_cg_pos = nullptr, *d_cg_rad = nullptr;
    uint32_t *d_cg_alive = nullptr, *d_cg_prod = nullptr, *d_cg_counts = nullptr;
    int *d_cg_head = nullptr, *d_cg_next = nullptr;
    wg::CgStep* d_cg_step = nullptr;
    size_t cg_cap = 0, cg_rad_cap = 0;
    cudaGraphExec_t cg_graph = nullptr;
    wg::CgGraphKey cg_key{};
    unsigned long long last_rad_n = 0;
    // DNA target + scoring
    wgdna_dna_info dna{};
    float *d_fy = nullptr, *d_fz = nullptr, *d_rbb0 = nullptr, *d_rbb1 = nullptr;
    uint8_t* d_hits = nullptr;
    uint32_t* d_alive = nullptr;
    unsigned long long alive_cap = 0;
    ScoreScratch sc{};
    unsigned long long sc_cap = 0;
    // IRT scratch
    bool irt_curves_on = false;
    float* d_curves = nullptr;
    size_t curves_cap = 0, curves_n = 0;
    size_t irt_slots = 0, irt_evslots = 0, irt_hov = 0, irt_pf_slots = 0;
    float4* d_pf = nullptr;
    float4* d_rec = nullptr;
    float* d_tdel = nullptr;
    uint32_t irt_tracks = 0, irt_hcap = 0;
    double *d_px = nullptr, *d_py = nullptr, *d_pz = nullptr, *d_tb = nullptr;
    int8_t* d_sp = nullptr;
    uint8_t* d_alive8 = nullptr;
    uint16_t *d_lst = nullptr, *d_lpos = nullptr;
    double* d_evt = nullptr;
    uint32_t* d_evab = nullptr;
    double* d_hov_t = nullptr;
    uint32_t* d_hov_ab = nullptr;
    uint32_t* d_track = nullptr;          // 11 per track: tn, th2, ttiles, tev, tlc[6], order
    unsigned long long* d_toff = nullptr;
    uint32_t* d_irt_cnt = nullptr;
    double* d_acc_tl = nullptr;
    unsigned long long* d_acc = nullptr;
    uint32_t* d_maxpid = nullptr;
    IrtGraph irt_graph;                   // the IRT launch sequence, captured once per argument set
    cudaEvent_t ev[11]{};
};

static std::string lib_dir() {
    Dl_info info;
    if (dladdr((void*)&wgdna_version, &info) && info.dli_fname) {
        std::string p(info.dli_fname);
        size_t k = p.find_last_of('/');
        if (k != std::string::npos) return p.substr(0, k);
    }
    return ".";
}

extern "C" void wgdna_default_tuning(wgdna_tuning* t) {
    if (!t) return;
    t->transport_ctas_per_sm = 0;
    t->prim_take = 2;
    t->stash_keep = 16;
    t->stash_spill = 32;
    t->queue_poll = 8;
    t->irt_init_blocks_per_sm = 0;
    t->irt_loop_blocks_per_sm = 0;
}

static bool tuning_ok(const wgdna_tuning& t) {
    const bool pow2 = t.queue_poll && (t.queue_poll & (t.queue_poll - 1)) == 0;
    const bool stash = t.stash_spill == 0 ? t.stash_keep == 0
                                          : (t.stash_spill <= TRANSPORT_STASH && t.stash_keep < t.stash_spill);
    return t.prim_take >= 1 && t.prim_take <= 32 && stash && pow2 && t.queue_poll <= 1024 &&
           t.transport_ctas_per_sm <= 8 && t.irt_init_blocks_per_sm <= 32 && t.irt_loop_blocks_per_sm <= 32;
}

// data/tuning.txt: "key value" lines (wgdna_tuning's field names), '#' comments;
// a missing file keeps the defaults, a malformed one is an error
static int tuning_load(const std::string& path, wgdna_tuning* t) {
    FILE* f = fopen(path.c_str(), "r");
    if (!f) return WGDNA_OK;
    char line[256];
    int rc = WGDNA_OK;
    while (rc == WGDNA_OK && fgets(line, sizeof line, f)) {
        char key[64];
        unsigned long v = 0;
        if (line[0] == '#' || sscanf(line, "%63s", key) != 1) continue;
        if (sscanf(line, "%63s %lu", key, &v) != 2) { rc = WGDNA_ERR_ARG; break; }
        uint32_t* dst = !strcmp(key, "transport_ctas_per_sm") ? &t->transport_ctas_per_sm
                      : !strcmp(key, "prim_take") ? &t->prim_take
                      : !strcmp(key, "stash_keep") ? &t->stash_keep
                      : !strcmp(key, "stash_spill") ? &t->stash_spill
                      : !strcmp(key, "queue_poll") ? &t->queue_poll
                      : !strcmp(key, "irt_init_blocks_per_sm") ? &t->irt_init_blocks_per_sm
                      : !strcmp(key, "irt_loop_blocks_per_sm") ? &t->irt_loop_blocks_per_sm : nullptr;
        if (!dst) { rc = WGDNA_ERR_ARG; break; }
        *dst = (uint32_t)v;
    }
    fclose(f);
    if (rc != WGDNA_OK || !tuning_ok(*t)) {
        wg_set_error("wgdna_create: malformed tuning table %s", path.c_str());
        return WGDNA_ERR_ARG;
    }
    return WGDNA_OK;
}

extern "C" int wgdna_get_tuning(wgdna_ctx* c, wgdna_tuning* t) {
    if (!c || !t) { wg_set_error("wgdna_get_tuning: NULL argument"); return WGDNA_ERR_ARG; }
    *t = c->tune;
    return WGDNA_OK;
}

extern "C" int wgdna_set_tuning(wgdna_ctx* c, const wgdna_tuning* t) {
    if (!c || !t) { wg_set_error("wgdna_set_tuning: NULL argument"); return WGDNA_ERR_ARG; }
    if (!tuning_ok(*t)) { wg_set_error("wgdna_set_tuning: a field is out of range"); return WGDNA_ERR_ARG; }
    WG_CUDA_OK(cudaSetDevice(c->device));
    c->tune = *t;
    c->tblocks = transport_blocks(c->device, t->transport_ctas_per_sm);
    return WGDNA_OK;
}

extern "C" void wgdna_default_cfg(wgdna_cfg* c) {
    if (!c) return;
    memset(c, 0, sizeof *c);
    c->device = 0;
    c->tables_path = nullptr;
    c->max_primaries = 4096;
    c->max_sec = 5000000u;
    c->max_rad = 16000000ull;
    c->vc = 128;
}

template <class T> static int dalloc(T** p, size_t n) {
    if (*p) { cudaFree(*p); *p = nullptr; }
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
    if (e != cudaSuccess) { wg_set_error("cudaMalloc(%zu bytes): %s", n * sizeof(T), cudaGetErrorString(e)); *p = nullptr; return WGDNA_ERR_NOMEM; }
    return WGDNA_OK;
}
#define TRY(x) do { int r_ = (x); if (r_ != WGDNA_OK) return r_; } while (0)

static int ensure_segments(wgdna_ctx* c, uint32_t nseg) {
    if (nseg <= c->seg_cap) return WGDNA_OK;
    uint32_t cap = nseg < 4096 ? 4096 : nseg;
    TRY(dalloc(&c->d_pid_cnt, cap));
    TRY(dalloc(&c->d_pid_cur, cap));
    TRY(dalloc(&c->d_pid_off, (size_t)cap + 1));
    c->seg_cap = cap;
    return WGDNA_OK;
}

extern "C" int wgdna_create(const wgdna_cfg* cfg, wgdna_ctx** out) {
    if (!out) { wg_set_error("wgdna_create: out is NULL"); return WGDNA_ERR_ARG; }
    *out = nullptr;
    wgdna_cfg c0;
    wgdna_default_cfg(&c0);
    if (cfg) c0 = *cfg;
    if (c0.max_primaries == 0 || c0.vc == 0 || c0.max_sec == 0 || c0.max_rad == 0) {
        wg_set_error("wgdna_create: capacities must be positive");
        return WGDNA_ERR_ARG;
    }
    if ((unsigned long long)c0.max_primaries > (1ull << 21)) {
        wg_set_error("wgdna_create: max_primaries %u exceeds 2097152 (w = pid*8 + code must stay exact in f32)",
                     c0.max_primaries);
        return WGDNA_ERR_ARG;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        wg_set_error("wgdna_create: no CUDA device");
        return WGDNA_ERR_CUDA;
    }
    if (c0.device < 0 || c0.device >= ndev) { wg_set_error("wgdna_create: bad device %d", c0.device); return WGDNA_ERR_ARG; }
    WG_CUDA_OK(cudaSetDevice(c0.device));
    wgdna_ctx* c = new wgdna_ctx();
    c->device = c0.device;
    c->cfg = c0;
    std::string tp = c0.tables_path ? std::string(c0.tables_path) : lib_dir() + "/data/cross_sections.bin";
    c->cfg.tables_path = nullptr;
    int rc = tables_load(tp.c_str(), &c->tab, &c->d_small, &c->d_xcw);
    if (rc != WGDNA_OK) { delete c; return rc; }
    cudaError_t e = cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking);
    if (e != cudaSuccess) { wg_set_error("cudaStreamCreate: %s", cudaGetErrorString(e)); delete c; return WGDNA_ERR_CUDA; }
    c->stream = c->own;
    for (auto& ev : c->ev) cudaEventCreate(&ev);
    size_t np = c0.max_primaries, nv = (size_t)c0.vc * c0.vc * c0.vc;
    int r = WGDNA_OK;
    if (r == WGDNA_OK) r = dalloc(&c->d_results, np * 8);
    if (r == WGDNA_OK) r = dalloc(&c->d_dose, nv);
    if (r == WGDNA_OK) r = dalloc(&c->d_rad_raw, c0.max_rad);
    if (r == WGDNA_OK) r = dalloc(&c->d_key, c0.max_rad);
    if (r == WGDNA_OK) r = dalloc(&c->d_rad, c0.max_rad);
    if (r == WGDNA_OK) r = dalloc(&c->d_perm, c0.max_rad);
    if (r == WGDNA_OK) r = dalloc(&c->d_secq, c0.max_sec);
    if (r == WGDNA_OK) r = dalloc(&c->d_st, 1);
    if (r == WGDNA_OK) r = dalloc(&c->d_Eprim, np);
    if (r == WGDNA_OK) r = dalloc(&c->d_red, 4);
    if (r == WGDNA_OK) r = dalloc(&c->d_err, 1);
    if (r == WGDNA_OK) r = ensure_segments(c, (uint32_t)np);
    if (r == WGDNA_OK && cudaMemset(c->d_secq, 0, sizeof(SecRec) * (size_t)c0.max_sec) != cudaSuccess) r = WGDNA_ERR_CUDA;
    if (r == WGDNA_OK) r = wgdna_set_dna_target(c, 3000.0, 21, 150.0);
    if (r != WGDNA_OK) { wgdna_destroy(c); return r; }
    wgdna_default_tuning(&c->tune);
    r = tuning_load(lib_dir() + "/data/tuning.txt", &c->tune);
    if (r != WGDNA_OK) { wgdna_destroy(c); return r; }
    c->tblocks = transport_blocks(c->device, c->tune.transport_ctas_per_sm);
    *out = c;
    return WGDNA_OK;
}

int ctx_view(wgdna_ctx* c, wg::CtxView* v) {
    v->device = c->device;
    v->stream = c->stream;
    v->rad = c->d_rad;
    v->seg_off = c->d_pid_off;
    v->nseg = c->last_nseg;
    v->have_transport = c->have_transport;
    v->Eprim = c->last_has_eprim ? c->d_Eprim : nullptr;
    v->E0 = c->last_E;
    v->sg = &c->sg;
    v->mma_ns = c->wait_mma_ns;
    v->mma_give_up_first = (c->test_flags & WGDNA_TEST_MMA_WAIT) != 0;
    return WGDNA_OK;
}

extern "C" int wgdna_set_wait_limits(wgdna_ctx* c, uint64_t queue_ns, uint64_t idle_ns, uint64_t mma_ns,
                                     uint32_t test_flags) {
    if (!c) { wg_set_error("wgdna_set_wait_limits: NULL context"); return WGDNA_ERR_ARG; }
    if (test_flags & ~(uint32_t)(WGDNA_TEST_UNPUBLISHED | WGDNA_TEST_MMA_WAIT)) {
        wg_set_error("wgdna_set_wait_limits: unknown test flags 0x%x", test_flags);
        return WGDNA_ERR_ARG;
    }
    c->wait_queue_ns = queue_ns ? queue_ns : WG_QUEUE_WAIT_NS;
    c->wait_idle_ns = idle_ns ? idle_ns : WG_IDLE_WAIT_NS;
    c->wait_mma_ns = mma_ns ? mma_ns : WG_MMA_WAIT_NS;
    c->test_flags = test_flags;
    return WGDNA_OK;
}

extern "C" void wgdna_destroy(wgdna_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    wg::sg_free(c->sg);
    void* ptrs[] = {c->d_small, c->d_xcw, c->d_results, c->d_dose, c->d_rad_raw, c->d_key, c->d_rad,
                    c->d_perm, c->d_secq, c->d_st, c->d_Eprim, c->d_pid_cnt, c->d_pid_off, c->d_pid_cur,
                    c->d_red, c->d_err, c->d_fy, c->d_fz, c->d_rbb0, c->d_rbb1, c->d_hits, c->d_alive,
                    c->sc.info, c->sc.last_brk, c->sc.cnt0, c->sc.cnt1, c->sc.cs_in, c->sc.base, c->sc.u64,
                    c->sc.fib, c->d_px, c->d_py, c->d_pz, c->d_tb, c->d_sp, c->d_alive8, c->d_lst, c->d_lpos, c->d_evt, c->d_evab,
                    c->d_hov_t, c->d_hov_ab, c->d_track, c->d_toff, c->d_irt_cnt, c->d_pf, c->d_rec, c->d_tdel, c->d_curves, c->d_acc_tl, c->d_acc, c->d_maxpid,
                    c->d_dose_in, c->d_lambda, c->d_hits_in, c->d_dres, c->d_cg_pos, c->d_cg_rad, c->d_cg_alive,
                    c->d_cg_prod, c->d_cg_counts, c->d_cg_head, c->d_cg_next, c->d_cg_step};
    if (c->cg_graph) cudaGraphExecDestroy(c->cg_graph);
    if (c->irt_graph.exec) cudaGraphExecDestroy(c->irt_graph.exec);
    for (void* p : ptrs) if (p) cudaFree(p);
    for (auto& ev : c->ev) if (ev) cudaEventDestroy(ev);
    if (c->own) cudaStreamDestroy(c->own);
    delete c;
}

static TArgs make_targs(wgdna_ctx* c, const wgdna_transport_params* p) {
    TArgs a;
    memset(&a, 0, sizeof a);
    a.np = p->np; a.box = p->box_nm; a.ce = p->ce_eV; a.ms = p->max_steps; a.be = p->E_eV;
    a.vc = c->cfg.vc; a.max_sec = c->cfg.max_sec; a.max_rad = c->cfg.max_rad;
    a.start_half = p->start_half; a.dna_enable = p->dna_enable; a.dna_grid_n = p->dna_grid_n;
    a.dna_rise = p->dna_rise; a.dna_spacing = p->dna_spacing; a.dna_x0 = p->dna_x0; a.dna_r_bb = p->dna_r_bb;
    a.sec_steps = p->sec_steps; a.k0 = (uint32_t)p->seed; a.k1 = (uint32_t)(p->seed >> 32); a.epoch = c->epoch;
    a.pid_base = p->pid_base;
    a.pub_epoch = (c->test_flags & WGDNA_TEST_UNPUBLISHED) ? c->epoch + 0x80000000u : c->epoch;
    a.ready_ns = c->wait_queue_ns;
    a.idle_ns = c->wait_idle_ns;
    a.prim_take = c->tune.prim_take;
    a.stash_keep = c->tune.stash_keep;
    a.stash_spill = c->tune.stash_spill;
    a.poll_mask = c->tune.queue_poll - 1;
    a.tab = c->tab;
    a.E_prim = p->E_per_primary ? c->d_Eprim : nullptr;
    a.results = c->d_results; a.dose = c->d_dose; a.rad = c->d_rad_raw; a.key = c->d_key;
    a.secq = c->d_secq; a.st = c->d_st;
    return a;
}

static IArgs make_iargs(wgdna_ctx* c, uint32_t nseg, uint64_t seed) {
    IArgs a;
    memset(&a, 0, sizeof a);
    a.rad = c->d_rad; a.seg_off = c->d_pid_off; a.nseg = nseg; a.pid_base = c->irt_pid_base;
    a.k0 = (uint32_t)seed; a.k1 = (uint32_t)(seed >> 32);
    philox_round_keys(a.k0, a.k1, a.rk);
    a.px = c->d_px; a.py = c->d_py; a.pz = c->d_pz; a.tb = c->d_tb; a.sp = c->d_sp; a.alive = c->d_alive8;
    a.lst = c->d_lst; a.lpos = c->d_lpos;
    a.ev_t = c->d_evt; a.ev_ab = c->d_evab;
    const size_t T = c->irt_tracks;
    a.tn = c->d_track; a.th2 = c->d_track + T; a.ttiles = c->d_track + 2 * T; a.tev = c->d_track + 3 * T;
    a.tlc = c->d_track + 4 * T;
    a.order = c->d_track + 10 * T;
    a.toff = c->d_toff;
    a.pf = c->d_pf; a.rec = c->d_rec; a.tdel = c->d_tdel;
    a.hov_t = c->d_hov_t; a.hov_ab = c->d_hov_ab; a.hcap = c->irt_hcap;
    a.counters = c->d_irt_cnt;
    a.acc_tl = c->d_acc_tl; a.acc = c->d_acc; a.err = c->d_err;
    return a;
}

extern "C" int wgdna_set_stream(wgdna_ctx* c, void* s) {
    if (!c) { wg_set_error("wgdna_set_stream: NULL context"); return WGDNA_ERR_ARG; }
    c->stream = s ? (cudaStream_t)s : c->own;
    return WGDNA_OK;
}

// ------------------------------------------------------------------ Phase A+B
extern "C" int wgdna_transport(wgdna_ctx* c, const wgdna_transport_params* p, wgdna_transport_stats* st) {
    if (!c || !p) { wg_set_error("wgdna_transport: NULL argument"); return WGDNA_ERR_ARG; }
    if (p->np == 0 || p->np > c->cfg.max_primaries) {
        wg_set_error("wgdna_transport: np=%u outside [1, %u]", p->np, c->cfg.max_primaries);
        return WGDNA_ERR_ARG;
    }
    if ((unsigned long long)p->pid_base + p->np > (1ull << 21)) {
        wg_set_error("wgdna_transport: pid_base + np exceeds 2097152 (w = pid*8 + code must stay exact in f32)");
        return WGDNA_ERR_ARG;
    }
    if (!(p->box_nm > 0.0f) || !(p->ce_eV > 0.0f) || !(p->E_eV >= 0.0f) || p->dna_grid_n == 0 ||
        !(p->dna_rise > 0.0f) || !(p->dna_spacing > 0.0f)) {
        wg_set_error("wgdna_transport: invalid physics parameters");
        return WGDNA_ERR_ARG;
    }
    WG_CUDA_OK(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    c->have_transport = false;
    size_t nv = (size_t)c->cfg.vc * c->cfg.vc * c->cfg.vc;
    WG_CUDA_OK(cudaMemsetAsync(c->d_st, 0, sizeof(DevState), s));
    WG_CUDA_OK(cudaMemsetAsync(c->d_dose, 0, nv * 4, s));
    WG_CUDA_OK(cudaMemsetAsync(c->d_err, 0, 4, s));
    if (p->E_per_primary)
        WG_CUDA_OK(cudaMemcpyAsync(c->d_Eprim, p->E_per_primary, (size_t)p->np * 4, cudaMemcpyHostToDevice, s));
    c->epoch++;
    if (c->epoch == 0) c->epoch = 1;
    TArgs a = make_targs(c, p);
    WG_CUDA_OK(cudaEventRecord(c->ev[0], s));
    WG_CUDA_OK(launch_transport(a, c->tblocks, s));
    WG_CUDA_OK(cudaEventRecord(c->ev[1], s));
    DevState hs;
    WG_CUDA_OK(cudaMemcpyAsync(&hs, c->d_st, sizeof hs, cudaMemcpyDeviceToHost, s));
    WG_CUDA_OK(cudaStreamSynchronize(s));
    unsigned long long stored = hs.rad_next.v < c->cfg.max_rad ? hs.rad_next.v : c->cfg.max_rad;
    WG_CUDA_OK(cudaEventRecord(c->ev[2], s));
    WG_CUDA_OK(launch_canon(c->d_key, c->d_rad_raw, stored, p->np, c->d_pid_cnt, c->d_pid_off, c->d_pid_cur,
                            c->d_perm, c->d_rad, c->d_err, s));
    WG_CUDA_OK(launch_reduce(c->d_results, p->np, c->d_dose, (uint32_t)nv, c->d_red, s));
    WG_CUDA_OK(cudaEventRecord(c->ev[3], s));
    unsigned long long red[2];
    uint32_t err2 = 0;
    WG_CUDA_OK(cudaMemcpyAsync(red, c->d_red, 16, cudaMemcpyDeviceToHost, s));
    WG_CUDA_OK(cudaMemcpyAsync(&err2, c->d_err, 4, cudaMemcpyDeviceToHost, s));
    WG_CUDA_OK(cudaStreamSynchronize(s));
    if (st) {
        memset(st, 0, sizeof *st);
        memcpy(st->counters, hs.counters, sizeof st->counters);
        memcpy(st->sec_stats, hs.sec_stats, sizeof st->sec_stats);
        memcpy(st->dbg, hs.dbg, sizeof st->dbg);
        st->counters[6] = hs.sec_tail.v;
        st->counters[7] = (uint32_t)hs.rad_next.v;
        st->rad_n_raw = hs.rad_next.v;
        st->rad_n_stored = stored;
        st->rad_dropped = hs.rad_next.v - stored;
        // dispatch.ts:125-126: emitted, kept (at most max_sec), dropped; the
        // global queue holds at most the kept ones, so sec_drop stays 0
        const uint32_t kept = hs.sec_tail.v < c->cfg.max_sec ? hs.sec_tail.v : c->cfg.max_sec;
        st->sec_n_raw = hs.sec_tail.v;
        st->sec_n = kept - (hs.sec_drop < kept ? hs.sec_drop : kept);
        st->sec_dropped = hs.sec_tail.v - st->sec_n;
        st->dep_units = red[0];
        st->dep_eV_f64 = hs.dep_f64;
        st->steps = hs.steps;
        st->n_therm = (uint32_t)red[1];
        st->ms_transport = elapsed_ms(c->ev[0], c->ev[1]);
        st->ms_canon = elapsed_ms(c->ev[2], c->ev[3]);
        st->device_error = hs.err | err2;
    }
    if (hs.err | err2) {
        wg_set_error("wgdna_transport: device error flags 0x%x", hs.err | err2);
        return WGDNA_ERR_DEVICE;
    }
    c->have_transport = true;
    c->last_np = p->np;
    c->last_nseg = p->np;
    c->last_pid_base = p->pid_base;
    c->last_rad_n = stored;
    c->last_E = p->E_eV;
    c->last_has_eprim = p->E_per_primary != nullptr;
    return WGDNA_OK;
}

extern "C" int wgdna_transport_copy_out(wgdna_ctx* c, float* results, uint32_t* dose, float* rad,
                                        uint64_t rad_cap, uint64_t* rad_n) {
    if (!c) { wg_set_error("wgdna_transport_copy_out: NULL context"); return WGDNA_ERR_ARG; }
    if (!c->have_transport) { wg_set_error("wgdna_transport_copy_out: no transport result"); return WGDNA_ERR_STATE; }
    cudaStream_t s = c->stream;
    size_t nv = (size_t)c->cfg.vc * c->cfg.vc * c->cfg.vc;
    if (results) WG_CUDA_OK(cudaMemcpyAsync(results, c->d_results, (size_t)c->last_np * 32, cudaMemcpyDeviceToHost, s));
    if (dose) WG_CUDA_OK(cudaMemcpyAsync(dose, c->d_dose, nv * 4, cudaMemcpyDeviceToHost, s));
    unsigned long long n = c->last_rad_n < rad_cap ? c->last_rad_n : rad_cap;
    if (rad && n) WG_CUDA_OK(cudaMemcpyAsync(rad, c->d_rad, n * 16, cudaMemcpyDeviceToHost, s));
    if (rad_n) *rad_n = c->last_rad_n;
    WG_CUDA_OK(cudaStreamSynchronize(s));
    return WGDNA_OK;
}

extern "C" int wgdna_run_transport(wgdna_ctx* c, const wgdna_transport_params* p, float* results,
                                   uint32_t* dose, float* rad, uint64_t rad_cap, uint64_t* rad_n,
                                   wgdna_transport_stats* st) {
    TRY(wgdna_transport(c, p, st));
    return wgdna_transport_copy_out(c, results, dose, rad, rad_cap, rad_n);
}

// ------------------------------------------------------------------ Phase C
static void irt_constants(IrtConst* C);

// Per-track particle slots 2*len + 64 and event slots 16*len + 2048 (the
// kernels' tbase / ebase), per-warp heap overflow hcap = 8*cap + 4096 with
// cap = 2*maxlen + 64 the largest track's particle slots.
static int irt_ensure(wgdna_ctx* c, uint32_t nseg, uint64_t rad_n, uint32_t cap) {
    size_t slots = 2 * (size_t)rad_n + 64 * (size_t)nseg;
    size_t evslots = 16 * (size_t)rad_n + 2048 * (size_t)nseg;
    uint32_t hcap = cap * 8u + 4096u;
    const IrtShape shape{c->tune.irt_init_blocks_per_sm, c->tune.irt_loop_blocks_per_sm};
    size_t hov = (size_t)irt_warps(c->device, shape) * hcap;
    if (slots > c->irt_slots) {
        TRY(dalloc(&c->d_px, slots)); TRY(dalloc(&c->d_py, slots)); TRY(dalloc(&c->d_pz, slots));
        TRY(dalloc(&c->d_tb, slots)); TRY(dalloc(&c->d_sp, slots)); TRY(dalloc(&c->d_alive8, slots));
        TRY(dalloc(&c->d_lst, 6 * slots)); TRY(dalloc(&c->d_lpos, slots));
        c->irt_slots = slots;
    }
    if (evslots > c->irt_evslots) {
        TRY(dalloc(&c->d_evt, evslots)); TRY(dalloc(&c->d_evab, evslots));
        c->irt_evslots = evslots;
    }
    if (hov > c->irt_hov) {
        TRY(dalloc(&c->d_hov_t, hov)); TRY(dalloc(&c->d_hov_ab, hov));
        c->irt_hov = hov;
    }
    c->irt_hcap = (uint32_t)(hov / irt_warps(c->device, shape));
    if (slots > c->irt_pf_slots) {
        TRY(dalloc(&c->d_pf, slots));
        TRY(dalloc(&c->d_rec, 6 * slots));
        c->irt_pf_slots = slots;
    }
    if (nseg > c->irt_tracks) {
        TRY(dalloc(&c->d_track, 11 * (size_t)nseg)); TRY(dalloc(&c->d_toff, (size_t)nseg + 1));
        TRY(dalloc(&c->d_tdel, (size_t)nseg));
        c->irt_tracks = nseg;
    }
    if (!c->d_irt_cnt) TRY(dalloc(&c->d_irt_cnt, 4));
    if (!c->d_acc_tl) TRY(dalloc(&c->d_acc_tl, 35));
    if (!c->d_acc) TRY(dalloc(&c->d_acc, 16));
    // the reaction constants live in __constant__ memory, which every device
    // holds separately: upload them once per device (the context's is current)
    static DeviceOnce consts;
    WG_CUDA_OK(consts.run([] {
        IrtConst C;
        irt_constants(&C);
        return irt_set_constants(C);
    }));
    return WGDNA_OK;
}

// run the IRT over nseg segments of c->d_rad (segment offsets in c->d_pid_off)
static int irt_run(wgdna_ctx* c, uint32_t nseg, uint32_t n_therm, double E_eV, uint64_t seed, uint64_t chem_n,
                   wgdna_irt_result* out) {
    cudaStream_t s = c->stream;
    WG_CUDA_OK(launch_seg_max(c->d_pid_off, nseg, c->d_red + 2, s));
    unsigned long long maxseg = 0;
    WG_CUDA_OK(cudaMemcpyAsync(&maxseg, c->d_red + 2, 8, cudaMemcpyDeviceToHost, s));
    WG_CUDA_OK(cudaStreamSynchronize(s));
    if (maxseg > (1ull << 24)) { wg_set_error("wgdna_irt: track of %llu entries is too large", maxseg); return WGDNA_ERR_CAPACITY; }
    uint32_t cap = (uint32_t)(2 * maxseg + 64);
    if (cap > 65535u) {
        wg_set_error("wgdna_irt: a track of %llu entries exceeds the 32,735-entry limit of the event encoding", maxseg);
        return WGDNA_ERR_CAPACITY;
    }
    TRY(irt_ensure(c, nseg, chem_n, cap));
    WG_CUDA_OK(cudaMemsetAsync(c->d_acc_tl, 0, 35 * 8, s));
    WG_CUDA_OK(cudaMemsetAsync(c->d_acc, 0, 16 * 8, s));
    WG_CUDA_OK(cudaMemsetAsync(c->d_err, 0, 4, s));
    IArgs a = make_iargs(c, nseg, seed);
    c->curves_n = 0;
    if (c->irt_curves_on) {
        if (nseg > c->curves_cap) {
            TRY(dalloc(&c->d_curves, (size_t)nseg * 80));
            c->curves_cap = nseg;
        }
        WG_CUDA_OK(cudaMemsetAsync(c->d_curves, 0, (size_t)nseg * 80 * sizeof(float), s));
        a.curves = c->d_curves;
        c->curves_n = nseg;
    }
    WG_CUDA_OK(cudaEventRecord(c->ev[4], s));
    WG_CUDA_OK(irt_graph_run(a, c->device, IrtShape{c->tune.irt_init_blocks_per_sm, c->tune.irt_loop_blocks_per_sm},
                             s, &c->ev[8], &c->irt_graph));
    WG_CUDA_OK(cudaEventRecord(c->ev[5], s));
    double tl[35];
    unsigned long long acc[16];
    uint32_t err = 0;
    WG_CUDA_OK(cudaMemcpyAsync(tl, c->d_acc_tl, sizeof tl, cudaMemcpyDeviceToHost, s));
    WG_CUDA_OK(cudaMemcpyAsync(acc, c->d_acc, sizeof acc, cudaMemcpyDeviceToHost, s));
    WG_CUDA_OK(cudaMemcpyAsync(&err, c->d_err, 4, cudaMemcpyDeviceToHost, s));
    WG_CUDA_OK(cudaStreamSynchronize(s));
    if (out) {
        memset(out, 0, sizeof *out);
        double per100 = ((double)n_therm * E_eV) / 100;
        for (int k = 0; k < 7; ++k)
            for (int q = 0; q < 5; ++q) {
                out->counts[k][q] = tl[k * 5 + q];
                out->G[k][q] = per100 > 0 ? tl[k * 5 + q] / per100 : 0;
            }
        for (int r = 0; r < 9; ++r) out->rxn_counts[r] = acc[r];
        out->n_reacted = acc[9]; out->n_pairs = acc[10]; out->n_events = acc[11]; out->n_tracks = acc[12];
        out->n_particles = acc[13]; out->n_init_events = acc[14];
        out->chem_n = chem_n;
        bool timed = true;
        out->ms = elapsed_ms(c->ev[4], c->ev[5]);
        out->ms_load = elapsed_ms(c->ev[4], c->ev[8], &timed);
        out->ms_pairing = elapsed_ms(c->ev[8], c->ev[9]);
        out->ms_sort = elapsed_ms(c->ev[9], c->ev[10]);
        out->ms_events = elapsed_ms(c->ev[10], c->ev[5]);
        // the per-kernel events inside a replayed graph could not be timed:
        // plain launches from the next call on, so that the times stay reported
        if (!timed && c->irt_graph.exec) c->irt_graph.off = true;
        out->device_error = err;
    }
    if (err) { wg_set_error("wgdna_irt: device error flags 0x%x", err); return WGDNA_ERR_DEVICE; }
    return WGDNA_OK;
}

extern "C" int wgdna_irt_record_curves(wgdna_ctx* c, int enable) {
    if (!c) { wg_set_error("wgdna_irt_record_curves: NULL context"); return WGDNA_ERR_ARG; }
    c->irt_curves_on = enable != 0;
    return WGDNA_OK;
}

extern "C" int wgdna_irt_curves(wgdna_ctx* c, float* out, uint64_t cap_tracks, uint64_t* n_tracks) {
    if (!c) { wg_set_error("wgdna_irt_curves: NULL context"); return WGDNA_ERR_ARG; }
    if (n_tracks) *n_tracks = c->curves_n;
    if (!out) return WGDNA_OK;
    if (cap_tracks < c->curves_n) {
        wg_set_error("wgdna_irt_curves: %zu tracks do not fit in %llu", c->curves_n, (unsigned long long)cap_tracks);
        return WGDNA_ERR_CAPACITY;
    }
    WG_CUDA_OK(cudaSetDevice(c->device));
    if (c->curves_n) {
        WG_CUDA_OK(cudaMemcpyAsync(out, c->d_curves, c->curves_n * 80 * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
        WG_CUDA_OK(cudaStreamSynchronize(c->stream));
    }
    return WGDNA_OK;
}

extern "C" int wgdna_irt(wgdna_ctx* c, uint32_t n_therm, double E_eV, uint64_t seed, wgdna_irt_result* out) {
    if (!c) { wg_set_error("wgdna_irt: NULL context"); return WGDNA_ERR_ARG; }
    if (!c->have_transport) { wg_set_error("wgdna_irt: no transport result in the context"); return WGDNA_ERR_STATE; }
    WG_CUDA_OK(cudaSetDevice(c->device));
    c->irt_pid_base = c->last_pid_base;
    return irt_run(c, c->last_nseg, n_therm, E_eV, seed, c->last_rad_n, out);
}

extern "C" int wgdna_run_irt(wgdna_ctx* c, const float* rad_buf, uint64_t rad_n, uint32_t n_therm, double E_eV,
                             uint64_t seed, wgdna_irt_result* out) {
    if (!c || (!rad_buf && rad_n)) { wg_set_error("wgdna_run_irt: NULL argument"); return WGDNA_ERR_ARG; }
    if (rad_n > c->cfg.max_rad) { wg_set_error("wgdna_run_irt: rad_n %llu exceeds max_rad", (unsigned long long)rad_n); return WGDNA_ERR_CAPACITY; }
    WG_CUDA_OK(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    c->have_transport = false;     // the rad_buf buffers are reused
    if (rad_n == 0) {
        if (out) { memset(out, 0, sizeof *out); }
        return WGDNA_OK;
    }
    WG_CUDA_OK(cudaMemcpyAsync(c->d_rad_raw, rad_buf, rad_n * 16, cudaMemcpyHostToDevice, s));
    if (!c->d_maxpid) TRY(dalloc(&c->d_maxpid, 1));
    WG_CUDA_OK(launch_group_keys(c->d_rad_raw, rad_n, c->d_key, c->d_maxpid, s));
    uint32_t maxpid = 0;
    WG_CUDA_OK(cudaMemcpyAsync(&maxpid, c->d_maxpid, 4, cudaMemcpyDeviceToHost, s));
    WG_CUDA_OK(cudaStreamSynchronize(s));
    uint32_t nseg = maxpid + 1;
    TRY(ensure_segments(c, nseg));
    WG_CUDA_OK(cudaMemsetAsync(c->d_err, 0, 4, s));
    WG_CUDA_OK(launch_canon(c->d_key, c->d_rad_raw, rad_n, nseg, c->d_pid_cnt, c->d_pid_off, c->d_pid_cur,
                            c->d_perm, c->d_rad, c->d_err, s));
    uint32_t err = 0;
    WG_CUDA_OK(cudaMemcpyAsync(&err, c->d_err, 4, cudaMemcpyDeviceToHost, s));
    WG_CUDA_OK(cudaStreamSynchronize(s));
    if (err) { wg_set_error("wgdna_run_irt: grouping error flags 0x%x", err); return WGDNA_ERR_DEVICE; }
    c->irt_pid_base = 0;
    return irt_run(c, nseg, n_therm, E_eV, seed, rad_n, out);
}

// IRT per-reaction constants, irt-worker.js:191-286 (C library functions,
// evaluated as the reference evaluates them with Math.*)
static void irt_constants(IrtConst* C) {
    memset(C, 0, sizeof *C);
    static const double D[6] = {2.2, 4.9, 7.0, 9.46, 2.3, 5.3};
    static const double VDW[6] = {0.22, 0.50, 0.19, 0.25, 0.21, 0.33};
    static const int Q[6] = {0, -1, 0, 1, 0, -1};
    struct R { int a, b; double k; int p0, p1, np, type; };
    static const R RX[9] = {{0, 0, 0.55e10, 4, 0, 1, 1}, {0, 1, 2.95e10, 5, 0, 1, 1}, {0, 2, 1.55e10, 0, 0, 0, 1},
                            {1, 1, 0.636e10, 5, 5, 2, 0}, {1, 2, 2.50e10, 5, 0, 1, 0}, {1, 3, 2.11e10, 2, 0, 1, 1},
                            {2, 2, 0.503e10, 0, 0, 0, 0}, {1, 4, 1.10e10, 5, 0, 2, 1}, {3, 5, 1.13e11, 0, 0, 0, 0}};
    const double ONS = 1.44 / (0.02527 * 80.1), Rs = 0.29, KC = 1e24 / (6.022e23 * 1e9);
    for (int i = 0; i < 6; ++i) C->D[i] = D[i];
    for (int r = 0; r < 9; ++r) {
        int a = RX[r].a, b = RX[r].b;
        double Ds = D[a] + D[b];
        int self = a == b;
        double rc = Q[a] * Q[b] * ONS;
        double k = RX[r].k * KC;
        C->rc[r] = rc; C->kobs[r] = k;
        C->type[r] = RX[r].type; C->nprod[r] = RX[r].np; C->prod0[r] = RX[r].p0; C->prod1[r] = RX[r].p1;
        if (RX[r].type == 0) {
            double sig = k / (4 * M_PI * Ds);
            if (self) sig *= 2;
            C->sigma[r] = sig; C->sigma_eff[r] = sig; C->kdif[r] = 0; C->prob[r] = 1;
            C->acc_s[r] = sig; C->acc_c[r] = 1.0; C->acc_add[r] = 0.5 * fabs(rc);
        } else {
            double sc = VDW[a] + VDW[b];
            C->sigma[r] = sc;
            double se, kd;
            if (rc == 0) { se = sc; kd = 4 * M_PI * Ds * sc; if (self) kd /= 2; }
            else { se = -rc / (1 - exp(rc / sc)); kd = 4 * M_PI * Ds * se; if (self) kd /= 2; }
            C->sigma_eff[r] = se; C->kdif[r] = kd;
            double ka = kd * k / (kd - k);
            C->kact[r] = ka;
            C->prob[r] = Rs / (Rs + (kd / ka) * (se + Rs));
            C->acc_s[r] = rc == 0 ? sc : se;
            C->acc_c[r] = k / kd;
            C->acc_add[r] = 0.5 * fabs(rc);
            if (rc == 0) {
                C->a_pdc[r] = (1.0 / sc) * ka / k;
            } else {
                double v = ka / (4 * M_PI * sc * sc * exp(-rc / sc));
                double alpha = v + rc * Ds / (sc * sc * (1 - exp(-rc / sc)));
                double sh = sinh(rc / (2 * sc));
                C->a_pdc[r] = 4 * sc * sc * alpha / (Ds * rc * rc) * sh * sh;
                C->coth_sig[r] = cosh(rc / (2 * sc)) / sinh(rc / (2 * sc));
            }
        }
    }
    for (int i = 0; i < 36; ++i) C->map[i] = -1;
    for (int r = 0; r < 9; ++r) { C->map[RX[r].a * 6 + RX[r].b] = r; C->map[RX[r].b * 6 + RX[r].a] = r; }
    static const double g[13] = {-4.06217193e-08, 3.06848412e-06, -9.93217814e-05, 1.80172797e-03,
                                 -2.01135480e-02, 1.42939448e-01, -6.48348714e-01, 1.85227848e+00,
                                 -3.36450378e+00, 4.37785068e+00, -4.20557339e+00, 3.81679083e+00,
                                 -2.34069784e-01};
    double rm = 0;
    for (int i = 12; i >= 0; --i) rm += g[12 - i] * pow(1.7, i);
    C->sig_eaq = rm * 0.62665706865775006;
    C->sig_oh = 0.8 / sqrt(3.0);
    C->sig_h = (17.0 / 18.0) * 2.4 / sqrt(3.0);
    double rcut = 1.45 + 2 * sqrt(8 * 9.46 * 1000);
    C->r_cut2 = rcut * rcut;
    for (int k = 0; k < 16; ++k) C->t16[k] = pow(10.0, -3.0 + 0.4 * k);
    for (int r = 0; r < 9; ++r) {
        double sr = C->acc_s[r], ad = C->acc_add[r];
        C->fa0[r] = (float)(((sr + ad) * (1.0 + 1e-6) + 1e-6) * (1.0 + 1e-7));
        C->fkb0[r] = (float)((ad * (1.0 + 1e-6) + 1e-6) * (1.0 + 1e-7));
        C->fk[r] = (float)(sr * C->acc_c[r] * (1.0 + 1e-6) * (1.0 + 1e-6) * (1.0 + 1e-7));
        C->fs[r] = (float)(sr * (1.0 + 1e-7));
        C->fsc[r] = (float)(sr * C->acc_c[r] * (1.0 + 1e-7));
        C->fadd[r] = (float)(ad * (1.0 + 1e-7));
    }
}

// ------------------------------------------------------------------ scoring
extern "C" int wgdna_build_dna_target(double L_nm, uint32_t grid_N, double spacing_nm, float* fy, float* fz,
                                      float* rbb0, float* rbb1, wgdna_dna_info* info) {
    // dna-geometry.ts:16-68 (f64 arithmetic, f32 storage)
    if (!(L_nm > 0) || grid_N == 0 || !(spacing_nm > 0)) { wg_set_error("wgdna_build_dna_target: invalid geometry"); return WGDNA_ERR_ARG; }
    const double rise = 0.34, bp_per_turn = 10.5, r_bb = 1.0;
    uint32_t n_bp_per = (uint32_t)floor(L_nm / rise);
    double x0 = -((double)n_bp_per - 1) * rise * 0.5;
    double d_phase = (2 * M_PI) / bp_per_turn;
    uint32_t nf = grid_N * grid_N;
    if (info) {
        info->grid_N = grid_N; info->n_bp_per = n_bp_per; info->n_fibers = nf; info->n_bp = nf * n_bp_per;
        info->rise = rise; info->r_bb = r_bb; info->spacing_nm = spacing_nm; info->x0 = x0; info->L_nm = L_nm;
    }
    double off = -(((double)grid_N - 1) * spacing_nm) * 0.5;
    for (uint32_t fi = 0; fi < grid_N; ++fi)
        for (uint32_t fj = 0; fj < grid_N; ++fj) {
            uint32_t idx = fi * grid_N + fj;
            if (fy) fy[idx] = (float)(off + fi * spacing_nm);
            if (fz) fz[idx] = (float)(off + fj * spacing_nm);
        }
    for (uint32_t i = 0; i < n_bp_per; ++i) {
        double phi = i * d_phase;
        if (rbb0) { rbb0[2 * i] = (float)(r_bb * cos(phi)); rbb0[2 * i + 1] = (float)(r_bb * sin(phi)); }
        if (rbb1) { rbb1[2 * i] = (float)(r_bb * cos(phi + M_PI)); rbb1[2 * i + 1] = (float)(r_bb * sin(phi + M_PI)); }
    }
    return WGDNA_OK;
}

extern "C" int wgdna_set_dna_target(wgdna_ctx* c, double L_nm, uint32_t grid_N, double spacing_nm) {
    if (!c) { wg_set_error("wgdna_set_dna_target: NULL context"); return WGDNA_ERR_ARG; }
    wgdna_dna_info info;
    TRY(wgdna_build_dna_target(L_nm, grid_N, spacing_nm, nullptr, nullptr, nullptr, nullptr, &info));
    if ((unsigned long long)info.n_bp * 2 >= (1ull << 29)) { wg_set_error("wgdna_set_dna_target: target too large"); return WGDNA_ERR_CAPACITY; }
    std::vector<float> fy(info.n_fibers), fz(info.n_fibers), r0(2 * info.n_bp_per), r1(2 * info.n_bp_per);
    TRY(wgdna_build_dna_target(L_nm, grid_N, spacing_nm, fy.data(), fz.data(), r0.data(), r1.data(), &info));
    WG_CUDA_OK(cudaSetDevice(c->device));
    TRY(dalloc(&c->d_fy, info.n_fibers)); TRY(dalloc(&c->d_fz, info.n_fibers));
    TRY(dalloc(&c->d_rbb0, 2 * info.n_bp_per)); TRY(dalloc(&c->d_rbb1, 2 * info.n_bp_per));
    size_t hb = ((size_t)info.n_bp * 2 + 3) & ~(size_t)3;
    TRY(dalloc(&c->d_hits, hb));
    TRY(dalloc(&c->sc.fib, 3 * (size_t)info.n_fibers));
    WG_CUDA_OK(cudaMemcpy(c->d_fy, fy.data(), fy.size() * 4, cudaMemcpyHostToDevice));
    WG_CUDA_OK(cudaMemcpy(c->d_fz, fz.data(), fz.size() * 4, cudaMemcpyHostToDevice));
    WG_CUDA_OK(cudaMemcpy(c->d_rbb0, r0.data(), r0.size() * 4, cudaMemcpyHostToDevice));
    WG_CUDA_OK(cudaMemcpy(c->d_rbb1, r1.data(), r1.size() * 4, cudaMemcpyHostToDevice));
    c->dna = info;
    return WGDNA_OK;
}

static DnaDev dna_dev(wgdna_ctx* c) {
    DnaDev d;
    d.fy = c->d_fy; d.fz = c->d_fz; d.rbb0 = c->d_rbb0; d.rbb1 = c->d_rbb1;
    d.x0 = c->dna.x0; d.rise = c->dna.rise; d.r_bb = c->dna.r_bb; d.spacing = c->dna.spacing_nm;
    d.grid_N = c->dna.grid_N; d.n_bp_per = c->dna.n_bp_per; d.n_bp = c->dna.n_bp;
    return d;
}

static int score_ensure(wgdna_ctx* c, unsigned long long n) {
    if (n <= c->sc_cap && c->sc.u64) return WGDNA_OK;
    unsigned long long cap = n < (1ull << 20) ? (1ull << 20) : n;
    unsigned long long nt = (cap + 1023) / 1024;
    TRY(dalloc(&c->sc.info, cap));
    TRY(dalloc(&c->sc.last_brk, nt)); TRY(dalloc(&c->sc.cnt0, nt)); TRY(dalloc(&c->sc.cnt1, nt));
    TRY(dalloc(&c->sc.cs_in, nt)); TRY(dalloc(&c->sc.base, nt));
    if (!c->sc.u64) TRY(dalloc(&c->sc.u64, 8));
    c->sc_cap = cap;
    return WGDNA_OK;
}

// score n entries of d_in (device) into c->d_hits
static int score_dev(wgdna_ctx* c, const float4* d_in, const uint32_t* d_alive, unsigned long long n, double p,
                     int dedupe, uint32_t lcg, wgdna_ssb_result* out) {
    TRY(score_ensure(c, n));
    cudaStream_t s = c->stream;
    DnaDev d = dna_dev(c);
    WG_CUDA_OK(cudaEventRecord(c->ev[6], s));
    WG_CUDA_OK(launch_score(d_in, d_alive, n, d, 0.29, p, dedupe, lcg, (uint32_t*)c->d_hits, c->sc, s));
    WG_CUDA_OK(cudaEventRecord(c->ev[7], s));
    unsigned long long u[8];
    WG_CUDA_OK(cudaMemcpyAsync(u, c->sc.u64, sizeof u, cudaMemcpyDeviceToHost, s));
    WG_CUDA_OK(cudaStreamSynchronize(s));
    if (out) {
        memset(out, 0, sizeof *out);
        out->ssb = u[0]; out->ssb0 = u[1]; out->ssb1 = u[2]; out->candidates = u[3];
        unsigned long long draws = n ? u[4] : 0;
        out->in_reach = draws;
        out->lcg_state = lcg_jump_host(lcg, draws);
        out->ms = elapsed_ms(c->ev[6], c->ev[7]);
    }
    return WGDNA_OK;
}

static int hits_in(wgdna_ctx* c, const uint8_t* hits) {
    size_t hb = (size_t)c->dna.n_bp * 2;
    if (hits) WG_CUDA_OK(cudaMemcpyAsync(c->d_hits, hits, hb, cudaMemcpyHostToDevice, c->stream));
    else WG_CUDA_OK(cudaMemsetAsync(c->d_hits, 0, (hb + 3) & ~(size_t)3, c->stream));
    return WGDNA_OK;
}

extern "C" int wgdna_score_direct(wgdna_ctx* c, const float* rad, uint64_t rad_n, uint32_t lcg_state,
                                  uint8_t* hits, wgdna_ssb_result* out) {
    if (!c || (!rad && rad_n)) { wg_set_error("wgdna_score_direct: NULL argument"); return WGDNA_ERR_ARG; }
    if (rad_n > c->cfg.max_rad) { wg_set_error("wgdna_score_direct: rad_n exceeds max_rad"); return WGDNA_ERR_CAPACITY; }
    WG_CUDA_OK(cudaSetDevice(c->device));
    c->have_transport = false;
    TRY(hits_in(c, hits));
    if (rad_n) WG_CUDA_OK(cudaMemcpyAsync(c->d_rad_raw, rad, rad_n * 16, cudaMemcpyHostToDevice, c->stream));
    TRY(score_dev(c, c->d_rad_raw, nullptr, rad_n, 0.15, 1, lcg_state, out));
    if (hits) WG_CUDA_OK(cudaMemcpy(hits, c->d_hits, (size_t)c->dna.n_bp * 2, cudaMemcpyDeviceToHost));
    return WGDNA_OK;
}

extern "C" int wgdna_score_indirect(wgdna_ctx* c, const float* pos, const uint32_t* alive, uint64_t n,
                                    uint32_t lcg_state, uint8_t* hits, wgdna_ssb_result* out) {
    if (!c || ((!pos || !alive) && n)) { wg_set_error("wgdna_score_indirect: NULL argument"); return WGDNA_ERR_ARG; }
    if (n > c->cfg.max_rad) { wg_set_error("wgdna_score_indirect: n exceeds max_rad"); return WGDNA_ERR_CAPACITY; }
    WG_CUDA_OK(cudaSetDevice(c->device));
    c->have_transport = false;
    TRY(hits_in(c, hits));
    if (n > c->alive_cap) { TRY(dalloc(&c->d_alive, n)); c->alive_cap = n; }
    if (n) {
        WG_CUDA_OK(cudaMemcpyAsync(c->d_rad_raw, pos, n * 16, cudaMemcpyHostToDevice, c->stream));
        WG_CUDA_OK(cudaMemcpyAsync(c->d_alive, alive, n * 4, cudaMemcpyHostToDevice, c->stream));
    }
    TRY(score_dev(c, c->d_rad_raw, c->d_alive, n, 0.4, 0, lcg_state, out));
    if (hits) WG_CUDA_OK(cudaMemcpy(hits, c->d_hits, (size_t)c->dna.n_bp * 2, cudaMemcpyDeviceToHost));
    return WGDNA_OK;
}

static int cluster_dev(wgdna_ctx* c, wgdna_dsb_result* out) {
    cudaStream_t s = c->stream;
    DnaDev d = dna_dev(c);
    WG_CUDA_OK(cudaEventRecord(c->ev[6], s));
    WG_CUDA_OK(launch_cluster(c->d_hits, d, c->dna.n_fibers, c->sc.fib, s));
    WG_CUDA_OK(cudaEventRecord(c->ev[7], s));
    std::vector<uint32_t> fib(3 * (size_t)c->dna.n_fibers);
    WG_CUDA_OK(cudaMemcpyAsync(fib.data(), c->sc.fib, fib.size() * 4, cudaMemcpyDeviceToHost, s));
    WG_CUDA_OK(cudaStreamSynchronize(s));
    if (out) {
        memset(out, 0, sizeof *out);
        double p_pair = fmin(1, (2.0 * 10 + 1) / c->dna.n_bp_per);
        for (uint32_t f = 0; f < c->dna.n_fibers; ++f) {
            uint32_t k0 = fib[3 * f + 1], k1 = fib[3 * f + 2];
            out->dsb += fib[3 * f]; out->ssb0 += k0; out->ssb1 += k1;
            if (k0 > 0 && k1 > 0) out->dsb_expected += 1 - pow(1 - p_pair, (double)k0 * (double)k1);
        }
        out->ms = elapsed_ms(c->ev[6], c->ev[7]);
    }
    return WGDNA_OK;
}

extern "C" int wgdna_cluster_dsb(wgdna_ctx* c, const uint8_t* hits, wgdna_dsb_result* out) {
    if (!c || !hits) { wg_set_error("wgdna_cluster_dsb: NULL argument"); return WGDNA_ERR_ARG; }
    WG_CUDA_OK(cudaSetDevice(c->device));
    TRY(hits_in(c, hits));
    return cluster_dev(c, out);
}

extern "C" int wgdna_score(wgdna_ctx* c, uint32_t lcg_state, wgdna_ssb_result* ssb, wgdna_dsb_result* dsb) {
    if (!c) { wg_set_error("wgdna_score: NULL context"); return WGDNA_ERR_ARG; }
    if (!c->have_transport) { wg_set_error("wgdna_score: no transport result in the context"); return WGDNA_ERR_STATE; }
    WG_CUDA_OK(cudaSetDevice(c->device));
    TRY(hits_in(c, nullptr));
    TRY(score_dev(c, c->d_rad, nullptr, c->last_rad_n, 0.15, 1, lcg_state, ssb));
    return cluster_dev(c, dsb);
}

extern "C" int wgdna_reaction_table(double out[9][6]) {
    if (!out) { wg_set_error("wgdna_reaction_table: NULL argument"); return WGDNA_ERR_ARG; }
    IrtConst C;
    irt_constants(&C);
    for (int r = 0; r < 9; ++r) {
        out[r][0] = C.sigma[r]; out[r][1] = C.sigma_eff[r]; out[r][2] = C.rc[r];
        out[r][3] = C.kdif[r]; out[r][4] = C.kact[r]; out[r][5] = C.prob[r];
    }
    return WGDNA_OK;
}

// ------------------------------------------------------------------ dose-grid scoring
// the grid to use: a host grid (uploaded) or the last transport's
static int dose_source(wgdna_ctx* c, const uint32_t* dose, const uint32_t** out) {
    const size_t nv = (size_t)c->cfg.vc * c->cfg.vc * c->cfg.vc;
    if (dose) {
        if (!c->d_dose_in) TRY(dalloc(&c->d_dose_in, nv));
        WG_CUDA_OK(cudaMemcpyAsync(c->d_dose_in, dose, nv * 4, cudaMemcpyHostToDevice, c->stream));
        *out = c->d_dose_in;
        return WGDNA_OK;
    }
    if (!c->have_transport) { wg_set_error("no dose grid: pass one or run wgdna_transport first"); return WGDNA_ERR_STATE; }
    *out = c->d_dose;
    return WGDNA_OK;
}

static wg::DoseDna dose_dna(wgdna_ctx* c) {
    wg::DoseDna d;
    d.fy = c->d_fy; d.fz = c->d_fz; d.rbb0 = c->d_rbb0; d.rbb1 = c->d_rbb1;
    d.n_fibers = c->dna.n_fibers; d.n_bp_per = c->dna.n_bp_per; d.x0 = c->dna.x0; d.rise = c->dna.rise;
    return d;
}

extern "C" int wgdna_dose_sum(wgdna_ctx* c, const uint32_t* dose, double* eV) {
    if (!c || !eV) { wg_set_error("wgdna_dose_sum: NULL argument"); return WGDNA_ERR_ARG; }
    WG_CUDA_OK(cudaSetDevice(c->device));
    const uint32_t* g = nullptr;
    TRY(dose_source(c, dose, &g));
    if (!c->d_dres) TRY(dalloc(&c->d_dres, 4));
    const size_t nv = (size_t)c->cfg.vc * c->cfg.vc * c->cfg.vc;
    WG_CUDA_OK(launch_dose_sum(g, nv, reinterpret_cast<unsigned long long*>(c->d_dres), c->stream));
    unsigned long long u = 0;
    WG_CUDA_OK(cudaMemcpyAsync(&u, c->d_dres, 8, cudaMemcpyDeviceToHost, c->stream));
    WG_CUDA_OK(cudaStreamSynchronize(c->stream));
    *eV = (double)u / 100.0;
    return WGDNA_OK;
}

extern "C" int wgdna_dose_projection(wgdna_ctx* c, const uint32_t* dose, int axis, float* proj) {
    if (!c || !proj || (axis != 0 && axis != 1)) { wg_set_error("wgdna_dose_projection: bad argument"); return WGDNA_ERR_ARG; }
    WG_CUDA_OK(cudaSetDevice(c->device));
    const uint32_t* g = nullptr;
    TRY(dose_source(c, dose, &g));
    const uint32_t vc = c->cfg.vc;
    float* d = nullptr;
    TRY(dalloc(&d, (size_t)vc * vc));
    WG_CUDA_OK(launch_dose_projection(g, vc, axis, d, c->stream));
    WG_CUDA_OK(cudaMemcpyAsync(proj, d, (size_t)vc * vc * 4, cudaMemcpyDeviceToHost, c->stream));
    WG_CUDA_OK(cudaStreamSynchronize(c->stream));
    cudaFree(d);
    return WGDNA_OK;
}

extern "C" int wgdna_score_voxel_ssb(wgdna_ctx* c, const uint32_t* dose, double box_nm, float* lambda,
                                     double* direct_expected) {
    if (!c) { wg_set_error("wgdna_score_voxel_ssb: NULL context"); return WGDNA_ERR_ARG; }
    WG_CUDA_OK(cudaSetDevice(c->device));
    const uint32_t* g = nullptr;
    TRY(dose_source(c, dose, &g));
    const size_t nl = 2 * (size_t)c->dna.n_bp;
    if (!c->d_lambda) TRY(dalloc(&c->d_lambda, nl));
    if (!c->d_dres) TRY(dalloc(&c->d_dres, 4));
    WG_CUDA_OK(launch_voxel_ssb(dose_dna(c), g, c->cfg.vc, box_nm, c->d_lambda, c->d_dres, c->stream));
    double e = 0;
    WG_CUDA_OK(cudaMemcpyAsync(&e, c->d_dres, 8, cudaMemcpyDeviceToHost, c->stream));
    if (lambda) WG_CUDA_OK(cudaMemcpyAsync(lambda, c->d_lambda, nl * 4, cudaMemcpyDeviceToHost, c->stream));
    WG_CUDA_OK(cudaStreamSynchronize(c->stream));
    c->have_lambda = true;
    if (direct_expected) *direct_expected = e;
    return WGDNA_OK;
}

extern "C" int wgdna_expected_dsb_local(wgdna_ctx* c, const float* lambda, const uint8_t* hits, double* dsb_expected) {
    if (!c || !dsb_expected) { wg_set_error("wgdna_expected_dsb_local: NULL argument"); return WGDNA_ERR_ARG; }
    WG_CUDA_OK(cudaSetDevice(c->device));
    const size_t nl = 2 * (size_t)c->dna.n_bp;
    if (!c->d_lambda) TRY(dalloc(&c->d_lambda, nl));
    if (lambda) WG_CUDA_OK(cudaMemcpyAsync(c->d_lambda, lambda, nl * 4, cudaMemcpyHostToDevice, c->stream));
    else if (!c->have_lambda) { wg_set_error("wgdna_expected_dsb_local: no lambda (run wgdna_score_voxel_ssb or pass one)"); return WGDNA_ERR_STATE; }
    const uint8_t* dh = nullptr;
    if (hits) {
        if (!c->d_hits_in) TRY(dalloc(&c->d_hits_in, nl));
        WG_CUDA_OK(cudaMemcpyAsync(c->d_hits_in, hits, nl, cudaMemcpyHostToDevice, c->stream));
        dh = c->d_hits_in;
    }
    if (!c->d_dres) TRY(dalloc(&c->d_dres, 4));
    WG_CUDA_OK(launch_expected_dsb(dose_dna(c), c->d_lambda, dh, c->d_dres, c->stream));
    WG_CUDA_OK(cudaMemcpyAsync(dsb_expected, c->d_dres, 8, cudaMemcpyDeviceToHost, c->stream));
    WG_CUDA_OK(cudaStreamSynchronize(c->stream));
    return WGDNA_OK;
}

// ------------------------------------------------------------------ grid-hash chemistry
extern "C" int wgdna_chem_grid(wgdna_ctx* c, const float* rad, uint64_t rad_n, uint32_t n_therm, double E_eV,
                               uint64_t seed, wgdna_chem_grid_result* out, float* pos, uint32_t* alive, uint64_t cap) {
    if (!c || !out) { wg_set_error("wgdna_chem_grid: NULL argument"); return WGDNA_ERR_ARG; }
    WG_CUDA_OK(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    const float4* src;
    uint64_t n_all;
    if (rad) {
        n_all = rad_n;
        if (rad_n > c->cg_rad_cap) { TRY(dalloc(&c->d_cg_rad, rad_n)); c->cg_rad_cap = rad_n; }
        WG_CUDA_OK(cudaMemcpyAsync(c->d_cg_rad, rad, rad_n * 16, cudaMemcpyHostToDevice, s));
        src = c->d_cg_rad;
    } else {
        if (!c->have_transport) { wg_set_error("wgdna_chem_grid: no rad_buf (pass one or run wgdna_transport)"); return WGDNA_ERR_STATE; }
        n_all = c->last_rad_n;
        src = c->d_rad;
    }
    const uint32_t n = (uint32_t)(n_all < wg::CG_CHEM_N ? n_all : wg::CG_CHEM_N);   // CHEM_N cap (schedule.ts:57)
    memset(out, 0, sizeof *out);
    if (n == 0) return WGDNA_OK;
    if (n > c->cg_cap) {
        TRY(dalloc(&c->d_cg_pos, n)); TRY(dalloc(&c->d_cg_alive, n)); TRY(dalloc(&c->d_cg_next, n));
        c->cg_cap = n;
    }
    if (!c->d_cg_head) {
        TRY(dalloc(&c->d_cg_head, wg::CG_HASH_SIZE)); TRY(dalloc(&c->d_cg_prod, 2));
        TRY(dalloc(&c->d_cg_counts, 40)); TRY(dalloc(&c->d_cg_step, 1));
    }
    wg::CgArgs a{src, n, (uint32_t)seed, (uint32_t)(seed >> 32), c->d_cg_pos, c->d_cg_alive, c->d_cg_head,
                 c->d_cg_next, c->d_cg_prod, c->d_cg_counts, c->d_cg_step};
    WG_CUDA_OK(cudaEventRecord(c->ev[4], s));
    WG_CUDA_OK(wg::cg_run(a, s, &c->cg_graph, &c->cg_key));
    WG_CUDA_OK(cudaEventRecord(c->ev[5], s));
    uint32_t counts[40];
    WG_CUDA_OK(cudaMemcpyAsync(counts, c->d_cg_counts, sizeof counts, cudaMemcpyDeviceToHost, s));
    if (pos && cap >= n) WG_CUDA_OK(cudaMemcpyAsync(pos, c->d_cg_pos, (size_t)n * 16, cudaMemcpyDeviceToHost, s));
    if (alive && cap >= n) WG_CUDA_OK(cudaMemcpyAsync(alive, c->d_cg_alive, (size_t)n * 4, cudaMemcpyDeviceToHost, s));
    WG_CUDA_OK(cudaStreamSynchronize(s));
    out->ms = elapsed_ms(c->ev[4], c->ev[5]);
    out->chem_n = n;
    // G per 100 eV of the deposited energy carried by the chem_n radicals (schedule.ts:218-227)
    out->deposited_eV = (double)n_therm * E_eV * ((double)n / (double)n_all);
    const double per100 = out->deposited_eV / 100;
    for (int k = 0; k < 8; ++k)
        for (int q = 0; q < 5; ++q) {
            out->counts[k][q] = counts[5 * k + q];
            out->G[k][q] = per100 > 0 ? counts[5 * k + q] / per100 : 0;
        }
    return WGDNA_OK;
}

// ------------------------------------------------------------------ sharded runs
extern "C" int wgdna_device_views(wgdna_ctx* c, wgdna_device_view* v) {
    if (!c || !v) { wg_set_error("wgdna_device_views: NULL argument"); return WGDNA_ERR_ARG; }
    memset(v, 0, sizeof *v);
    v->dose = c->d_dose;
    v->dose_words = (uint64_t)c->cfg.vc * c->cfg.vc * c->cfg.vc;
    v->hits = c->d_hits;
    v->hits_bytes = (uint64_t)c->dna.n_bp * 2;
    v->rad = reinterpret_cast<float*>(c->d_rad);
    v->rad_n = c->have_transport ? c->last_rad_n : 0;
    v->results = c->d_results;
    v->n_primaries = c->last_np;
    v->stream = c->stream;
    return WGDNA_OK;
}

extern "C" int wgdna_score_draws(wgdna_ctx* c, uint32_t lcg_state, wgdna_ssb_result* ssb) {
    if (!c) { wg_set_error("wgdna_score_draws: NULL context"); return WGDNA_ERR_ARG; }
    if (!c->have_transport) { wg_set_error("wgdna_score_draws: no transport result in the context"); return WGDNA_ERR_STATE; }
    WG_CUDA_OK(cudaSetDevice(c->device));
    TRY(hits_in(c, nullptr));
    return score_dev(c, c->d_rad, nullptr, c->last_rad_n, 0.15, 1, lcg_state, ssb);
}

extern "C" int wgdna_cluster_device(wgdna_ctx* c, wgdna_dsb_result* dsb) {
    if (!c) { wg_set_error("wgdna_cluster_device: NULL context"); return WGDNA_ERR_ARG; }
    WG_CUDA_OK(cudaSetDevice(c->device));
    return cluster_dev(c, dsb);
}
