// surrogate_api.cu -- C entry points of the surrogate chemistry (no reference
// counterpart): track descriptors, training of the MLP on IRT curves, and
// prediction of G(t) for the tracks of a transport.
#include <cmath>
#include <cstring>
#include <vector>

#include "wgdna.h"
#include "common.cuh"
#include "surrogate.cuh"
#include "surrogate_api.cuh"

using namespace wg;

namespace wg {

struct SgState {
    float *p = nullptr, *m = nullptr, *v = nullptr, *g = nullptr;
    __nv_bfloat16 *W = nullptr, *WT = nullptr;
    float *xmean = nullptr, *xinv = nullptr, *ymean = nullptr, *ystd = nullptr;
    float h_xmean[SG_IN], h_xstd[SG_IN], h_ymean[SG_OUT], h_ystd[SG_OUT];
    // training data (standardised) and batch buffers
    float *X = nullptr, *T = nullptr;
    uint64_t ndata = 0, data_cap = 0;
    uint32_t* rows = nullptr;
    float* Y = nullptr;
    __nv_bfloat16 *H0 = nullptr, *H1 = nullptr, *H2 = nullptr, *H3 = nullptr;
    float *Z1 = nullptr, *Z2 = nullptr, *Z3 = nullptr;
    uint64_t batch_cap = 0;
    double* loss = nullptr;
    uint32_t* err = nullptr;
    uint64_t step = 0;
    // descriptors / predictions of the last transport
    float *desc = nullptr, *xs = nullptr, *pred = nullptr;
    uint64_t desc_n = 0, desc_cap = 0;
    double* acc = nullptr;
    // bound of the kernels' tensor-core waits and the test switch (from the context)
    unsigned long long mma_ns = WG_MMA_WAIT_NS;
    uint32_t give_up_first = 0;
    cudaEvent_t ev[2] = {nullptr, nullptr};   // timing of wgdna_surrogate_chemistry
};

void sg_free(SgState* s) {
    if (!s) return;
    void* ptrs[] = {s->p, s->m, s->v, s->g, s->W, s->WT, s->xmean, s->xinv, s->ymean, s->ystd, s->X, s->T,
                    s->rows, s->Y, s->H0, s->H1, s->H2, s->H3, s->Z1, s->Z2, s->Z3, s->loss, s->err,
                    s->desc, s->xs, s->pred, s->acc};
    for (void* q : ptrs) if (q) cudaFree(q);
    for (cudaEvent_t e : s->ev) if (e) cudaEventDestroy(e);
    delete s;
}

}  // namespace wg

namespace {

template <class T> int salloc(T** p, size_t n) {
    if (*p) { cudaFree(*p); *p = nullptr; }
    cudaError_t e = cudaMalloc((void**)p, (n ? n : 1) * sizeof(T));
    if (e != cudaSuccess) {
        wg_set_error("cudaMalloc(%zu bytes): %s", n * sizeof(T), cudaGetErrorString(e));
        *p = nullptr;
        return WGDNA_ERR_NOMEM;
    }
    return WGDNA_OK;
}
#define STRY(x) do { int r_ = (x); if (r_ != WGDNA_OK) return r_; } while (0)

// splitmix64: seeds of the weight initialisation and the epoch shuffles
uint64_t smix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
double u01(uint64_t& s) { return (double)(smix(s) >> 11) * (1.0 / 9007199254740992.0); }

int ensure_state(wgdna_ctx* c, CtxView& v, SgState** out) {
    ctx_view(c, &v);
    WG_CUDA_OK(cudaSetDevice(v.device));
    if (*v.sg) {
        (*v.sg)->mma_ns = v.mma_ns;
        (*v.sg)->give_up_first = v.mma_give_up_first ? 1u : 0u;
        *out = *v.sg;
        return WGDNA_OK;
    }
    SgState* s = new SgState();
    *v.sg = s;
    s->mma_ns = v.mma_ns;
    s->give_up_first = v.mma_give_up_first ? 1u : 0u;
    STRY(salloc(&s->p, SG_NPARAM)); STRY(salloc(&s->m, SG_NPARAM)); STRY(salloc(&s->v, SG_NPARAM));
    STRY(salloc(&s->g, SG_NPARAM));
    STRY(salloc(&s->W, SG_WTOTAL)); STRY(salloc(&s->WT, SG_WTOTAL));
    STRY(salloc(&s->xmean, SG_IN)); STRY(salloc(&s->xinv, SG_IN));
    STRY(salloc(&s->ymean, SG_OUT)); STRY(salloc(&s->ystd, SG_OUT));
    STRY(salloc(&s->loss, 1)); STRY(salloc(&s->err, 1)); STRY(salloc(&s->acc, SG_OUT + 1));
    WG_CUDA_OK(cudaMemset(s->m, 0, SG_NPARAM * 4)); WG_CUDA_OK(cudaMemset(s->v, 0, SG_NPARAM * 4));
    WG_CUDA_OK(cudaMemset(s->g, 0, SG_NPARAM * 4)); WG_CUDA_OK(cudaMemset(s->p, 0, SG_NPARAM * 4));
    WG_CUDA_OK(cudaMemset(s->err, 0, 4));
    for (int k = 0; k < SG_IN; ++k) { s->h_xmean[k] = 0.0f; s->h_xstd[k] = 1.0f; }
    for (int k = 0; k < SG_OUT; ++k) { s->h_ymean[k] = 0.0f; s->h_ystd[k] = 1.0f; }
    *out = s;
    return WGDNA_OK;
}

int upload_norm(SgState* s, cudaStream_t st) {
    float xinv[SG_IN];
    for (int k = 0; k < SG_IN; ++k) xinv[k] = s->h_xstd[k] > 0 ? 1.0f / s->h_xstd[k] : 1.0f;
    WG_CUDA_OK(cudaMemcpyAsync(s->xmean, s->h_xmean, sizeof s->h_xmean, cudaMemcpyHostToDevice, st));
    WG_CUDA_OK(cudaMemcpyAsync(s->xinv, xinv, sizeof xinv, cudaMemcpyHostToDevice, st));
    WG_CUDA_OK(cudaMemcpyAsync(s->ymean, s->h_ymean, sizeof s->h_ymean, cudaMemcpyHostToDevice, st));
    WG_CUDA_OK(cudaMemcpyAsync(s->ystd, s->h_ystd, sizeof s->h_ystd, cudaMemcpyHostToDevice, st));
    return WGDNA_OK;
}

SgWeights weights(SgState* s) {
    SgWeights w;
    for (int l = 0; l < 4; ++l) { w.W[l] = s->W + SG_WOFF[l]; w.WT[l] = s->WT + SG_WOFF[l]; }
    w.p = s->p;
    return w;
}

int ensure_batch(SgState* s, uint64_t n) {
    if (n <= s->batch_cap) return WGDNA_OK;
    STRY(salloc(&s->rows, n)); STRY(salloc(&s->Y, n * SG_OUT));
    STRY(salloc(&s->H0, n * SG_IN)); STRY(salloc(&s->H1, n * SG_HID)); STRY(salloc(&s->H2, n * SG_HID));
    STRY(salloc(&s->H3, n * SG_HID)); STRY(salloc(&s->Z1, n * SG_HID)); STRY(salloc(&s->Z2, n * SG_HID));
    STRY(salloc(&s->Z3, n * SG_HID));
    s->batch_cap = n;
    return WGDNA_OK;
}

int check_err(SgState* s, cudaStream_t st, const char* who) {
    uint32_t e = 0;
    WG_CUDA_OK(cudaMemcpyAsync(&e, s->err, 4, cudaMemcpyDeviceToHost, st));
    WG_CUDA_OK(cudaStreamSynchronize(st));
    if (e) {
        wg_set_error("%s: device error flags 0x%x", who, e);
        cudaMemsetAsync(s->err, 0, 4, st);
        return WGDNA_ERR_DEVICE;
    }
    return WGDNA_OK;
}

// forward + backward over rows [rows] of the loaded data (n of them), gradients accumulated in s->g
int fwd_bwd(SgState* s, cudaStream_t st, const uint32_t* d_rows, uint32_t n) {
    SgFwdArgs f{};
    f.X = s->X; f.rows = d_rows; f.n = n; f.w = weights(s); f.Y = s->Y;
    f.H0 = s->H0; f.H1 = s->H1; f.H2 = s->H2; f.H3 = s->H3; f.Z1 = s->Z1; f.Z2 = s->Z2; f.Z3 = s->Z3;
    f.err = s->err; f.mma_ns = s->mma_ns; f.give_up_first = s->give_up_first;
    WG_CUDA_OK(launch_sg_forward(f, st));
    SgBwdArgs b{};
    b.T = s->T; b.rows = d_rows; b.n = n; b.w = f.w; b.Y = s->Y;
    b.H0 = s->H0; b.H1 = s->H1; b.H2 = s->H2; b.H3 = s->H3; b.Z1 = s->Z1; b.Z2 = s->Z2; b.Z3 = s->Z3;
    b.grad = s->g; b.loss = s->loss; b.err = s->err; b.mma_ns = s->mma_ns; b.give_up_first = s->give_up_first;
    WG_CUDA_OK(launch_sg_backward(b, st));
    return WGDNA_OK;
}

}  // namespace

extern "C" int wgdna_surrogate_init(wgdna_ctx* c, uint64_t seed) {
    if (!c) { wg_set_error("wgdna_surrogate_init: NULL context"); return WGDNA_ERR_ARG; }
    CtxView v;
    SgState* s;
    STRY(ensure_state(c, v, &s));
    std::vector<float> p(SG_NPARAM, 0.0f);
    uint64_t st = seed ^ 0x5EED5EEDull;
    const int woff[4] = {SG_OFF_W1, SG_OFF_W2, SG_OFF_W3, SG_OFF_W4};
    const int nin[4] = {SG_IN, SG_HID, SG_HID, SG_HID}, nout[4] = {SG_HID, SG_HID, SG_HID, SG_OUT};
    for (int l = 0; l < 4; ++l) {
        const double a = std::sqrt(6.0 / (nin[l] + nout[l]));          // Glorot uniform
        for (int i = 0; i < nin[l] * nout[l]; ++i) p[woff[l] + i] = (float)((2.0 * u01(st) - 1.0) * a);
    }
    WG_CUDA_OK(cudaMemcpyAsync(s->p, p.data(), SG_NPARAM * 4, cudaMemcpyHostToDevice, v.stream));
    WG_CUDA_OK(cudaMemsetAsync(s->m, 0, SG_NPARAM * 4, v.stream));
    WG_CUDA_OK(cudaMemsetAsync(s->v, 0, SG_NPARAM * 4, v.stream));
    WG_CUDA_OK(cudaMemsetAsync(s->g, 0, SG_NPARAM * 4, v.stream));
    s->step = 0;
    STRY(upload_norm(s, v.stream));
    WG_CUDA_OK(launch_sg_convert(s->p, s->W, s->WT, v.stream));
    WG_CUDA_OK(cudaStreamSynchronize(v.stream));
    return WGDNA_OK;
}

extern "C" int wgdna_surrogate_params(wgdna_ctx* c, float* get, const float* set) {
    if (!c) { wg_set_error("wgdna_surrogate_params: NULL context"); return WGDNA_ERR_ARG; }
    CtxView v;
    SgState* s;
    STRY(ensure_state(c, v, &s));
    if (set) {
        WG_CUDA_OK(cudaMemcpyAsync(s->p, set, SG_NPARAM * 4, cudaMemcpyHostToDevice, v.stream));
        WG_CUDA_OK(launch_sg_convert(s->p, s->W, s->WT, v.stream));
    }
    if (get) WG_CUDA_OK(cudaMemcpyAsync(get, s->p, SG_NPARAM * 4, cudaMemcpyDeviceToHost, v.stream));
    WG_CUDA_OK(cudaStreamSynchronize(v.stream));
    return WGDNA_OK;
}

extern "C" int wgdna_surrogate_norm(wgdna_ctx* c, float* get, const float* set) {
    if (!c) { wg_set_error("wgdna_surrogate_norm: NULL context"); return WGDNA_ERR_ARG; }
    CtxView v;
    SgState* s;
    STRY(ensure_state(c, v, &s));
    if (set) {
        memcpy(s->h_xmean, set, sizeof s->h_xmean);
        memcpy(s->h_xstd, set + SG_IN, sizeof s->h_xstd);
        memcpy(s->h_ymean, set + 2 * SG_IN, sizeof s->h_ymean);
        memcpy(s->h_ystd, set + 2 * SG_IN + SG_OUT, sizeof s->h_ystd);
        STRY(upload_norm(s, v.stream));
        WG_CUDA_OK(cudaStreamSynchronize(v.stream));
    }
    if (get) {
        memcpy(get, s->h_xmean, sizeof s->h_xmean);
        memcpy(get + SG_IN, s->h_xstd, sizeof s->h_xstd);
        memcpy(get + 2 * SG_IN, s->h_ymean, sizeof s->h_ymean);
        memcpy(get + 2 * SG_IN + SG_OUT, s->h_ystd, sizeof s->h_ystd);
    }
    return WGDNA_OK;
}

extern "C" int wgdna_surrogate_load(wgdna_ctx* c, const float* X, const float* G, uint64_t n) {
    if (!c || (n && (!X || !G))) { wg_set_error("wgdna_surrogate_load: NULL argument"); return WGDNA_ERR_ARG; }
    CtxView v;
    SgState* s;
    STRY(ensure_state(c, v, &s));
    if (n > s->data_cap) {
        STRY(salloc(&s->X, n * SG_IN)); STRY(salloc(&s->T, n * SG_OUT));
        s->data_cap = n;
    }
    float* tmp = nullptr;
    STRY(salloc(&tmp, n * SG_OUT > n * SG_IN ? n * SG_OUT : n * SG_IN));
    WG_CUDA_OK(cudaMemcpyAsync(tmp, X, n * SG_IN * 4, cudaMemcpyHostToDevice, v.stream));
    WG_CUDA_OK(launch_sg_standardise(tmp, s->X, n, SG_IN, s->xmean, s->xinv, v.stream));
    // targets: (G - mean) / std
    std::vector<float> yinv(SG_OUT);
    for (int k = 0; k < SG_OUT; ++k) yinv[k] = s->h_ystd[k] > 0 ? 1.0f / s->h_ystd[k] : 1.0f;
    float* d_yinv = nullptr;
    STRY(salloc(&d_yinv, SG_OUT));
    WG_CUDA_OK(cudaMemcpyAsync(d_yinv, yinv.data(), SG_OUT * 4, cudaMemcpyHostToDevice, v.stream));
    WG_CUDA_OK(cudaMemcpyAsync(tmp, G, n * SG_OUT * 4, cudaMemcpyHostToDevice, v.stream));
    WG_CUDA_OK(launch_sg_standardise(tmp, s->T, n, SG_OUT, s->ymean, d_yinv, v.stream));
    WG_CUDA_OK(cudaStreamSynchronize(v.stream));
    cudaFree(tmp);
    cudaFree(d_yinv);
    s->ndata = n;
    return WGDNA_OK;
}

extern "C" int wgdna_surrogate_grad(wgdna_ctx* c, uint64_t n, float* grad, double* loss) {
    if (!c) { wg_set_error("wgdna_surrogate_grad: NULL context"); return WGDNA_ERR_ARG; }
    CtxView v;
    SgState* s;
    STRY(ensure_state(c, v, &s));
    if (n == 0 || n > s->ndata || n > 0xffffffffull) { wg_set_error("wgdna_surrogate_grad: bad row count"); return WGDNA_ERR_ARG; }
    STRY(ensure_batch(s, n));
    WG_CUDA_OK(cudaMemsetAsync(s->g, 0, SG_NPARAM * 4, v.stream));
    WG_CUDA_OK(cudaMemsetAsync(s->loss, 0, 8, v.stream));
    STRY(fwd_bwd(s, v.stream, nullptr, (uint32_t)n));
    STRY(check_err(s, v.stream, "wgdna_surrogate_grad"));
    if (grad) WG_CUDA_OK(cudaMemcpyAsync(grad, s->g, SG_NPARAM * 4, cudaMemcpyDeviceToHost, v.stream));
    double l = 0;
    WG_CUDA_OK(cudaMemcpyAsync(&l, s->loss, 8, cudaMemcpyDeviceToHost, v.stream));
    WG_CUDA_OK(cudaMemsetAsync(s->g, 0, SG_NPARAM * 4, v.stream));
    WG_CUDA_OK(cudaStreamSynchronize(v.stream));
    if (loss) *loss = l / ((double)n * SG_OUT);
    return WGDNA_OK;
}

extern "C" int wgdna_surrogate_train(wgdna_ctx* c, uint32_t epochs, uint32_t batch, float lr, uint64_t seed,
                                     float* losses) {
    if (!c || batch == 0) { wg_set_error("wgdna_surrogate_train: bad argument"); return WGDNA_ERR_ARG; }
    CtxView v;
    SgState* s;
    STRY(ensure_state(c, v, &s));
    if (s->ndata == 0) { wg_set_error("wgdna_surrogate_train: no data loaded"); return WGDNA_ERR_STATE; }
    const uint64_t n = s->ndata;
    const uint32_t B = (uint32_t)(batch < n ? batch : n);
    STRY(ensure_batch(s, B));
    uint32_t* d_perm = nullptr;
    STRY(salloc(&d_perm, n));
    std::vector<uint32_t> perm(n);
    uint64_t st = seed ^ 0xA5A5A5A5ull;
    for (uint32_t e = 0; e < epochs; ++e) {
        for (uint64_t i = 0; i < n; ++i) perm[i] = (uint32_t)i;
        for (uint64_t i = n - 1; i > 0; --i) {                     // Fisher-Yates
            uint64_t j = smix(st) % (i + 1);
            uint32_t t = perm[i]; perm[i] = perm[j]; perm[j] = t;
        }
        WG_CUDA_OK(cudaMemcpyAsync(d_perm, perm.data(), n * 4, cudaMemcpyHostToDevice, v.stream));
        WG_CUDA_OK(cudaMemsetAsync(s->loss, 0, 8, v.stream));
        const uint64_t nb = n / B;                                   // full batches
        for (uint64_t b = 0; b < nb; ++b) {
            STRY(fwd_bwd(s, v.stream, d_perm + b * B, B));
            s->step++;
            const float b1t = (float)std::pow(0.9, (double)s->step), b2t = (float)std::pow(0.999, (double)s->step);
            WG_CUDA_OK(launch_sg_adam(s->p, s->m, s->v, s->g, lr, b1t, b2t, s->W, s->WT, v.stream));
        }
        double l = 0;
        WG_CUDA_OK(cudaMemcpyAsync(&l, s->loss, 8, cudaMemcpyDeviceToHost, v.stream));
        STRY(check_err(s, v.stream, "wgdna_surrogate_train"));
        if (losses) losses[e] = (float)(l / ((double)nb * B * SG_OUT));
    }
    cudaFree(d_perm);
    return WGDNA_OK;
}

// predictions on host inputs (X not NULL) or on the descriptors of the last
// wgdna_track_descriptors call (X NULL); G is n x 80, per 100 eV
extern "C" int wgdna_surrogate_predict(wgdna_ctx* c, const float* X, uint64_t n, float* G) {
    if (!c) { wg_set_error("wgdna_surrogate_predict: NULL context"); return WGDNA_ERR_ARG; }
    CtxView v;
    SgState* s;
    STRY(ensure_state(c, v, &s));
    const float* src = s->desc;
    if (X) {
        if (n > s->desc_cap) {
            STRY(salloc(&s->desc, n * SG_IN)); STRY(salloc(&s->xs, n * SG_IN)); STRY(salloc(&s->pred, n * SG_OUT));
            s->desc_cap = n;
        }
        WG_CUDA_OK(cudaMemcpyAsync(s->desc, X, n * SG_IN * 4, cudaMemcpyHostToDevice, v.stream));
        s->desc_n = n;
        src = s->desc;
    } else {
        n = s->desc_n;
    }
    if (n == 0) return WGDNA_OK;
    if (n > 0xffffffffull) { wg_set_error("wgdna_surrogate_predict: too many rows"); return WGDNA_ERR_ARG; }
    WG_CUDA_OK(launch_sg_standardise(src, s->xs, n, SG_IN, s->xmean, s->xinv, v.stream));
    SgFwdArgs f{};
    f.X = s->xs; f.n = (uint32_t)n; f.w = weights(s); f.Y = s->pred; f.err = s->err;
    f.mma_ns = s->mma_ns; f.give_up_first = s->give_up_first;
    WG_CUDA_OK(launch_sg_forward(f, v.stream));
    STRY(check_err(s, v.stream, "wgdna_surrogate_predict"));
    if (G) {
        std::vector<float> y(n * SG_OUT);
        WG_CUDA_OK(cudaMemcpyAsync(y.data(), s->pred, n * SG_OUT * 4, cudaMemcpyDeviceToHost, v.stream));
        WG_CUDA_OK(cudaStreamSynchronize(v.stream));
        for (uint64_t i = 0; i < n; ++i)
            for (int k = 0; k < SG_OUT; ++k) G[i * SG_OUT + k] = y[i * SG_OUT + k] * s->h_ystd[k] + s->h_ymean[k];
    }
    return WGDNA_OK;
}

extern "C" int wgdna_track_descriptors(wgdna_ctx* c, float* out, uint64_t cap, uint64_t* n_tracks) {
    if (!c) { wg_set_error("wgdna_track_descriptors: NULL context"); return WGDNA_ERR_ARG; }
    CtxView v;
    SgState* s;
    STRY(ensure_state(c, v, &s));
    if (!v.have_transport) { wg_set_error("wgdna_track_descriptors: no transport result in the context"); return WGDNA_ERR_STATE; }
    const uint64_t n = v.nseg;
    if (n > s->desc_cap) {
        STRY(salloc(&s->desc, n * SG_IN)); STRY(salloc(&s->xs, n * SG_IN)); STRY(salloc(&s->pred, n * SG_OUT));
        s->desc_cap = n;
    }
    DescArgs a{v.rad, v.seg_off, v.nseg, v.Eprim, v.E0, s->desc};
    WG_CUDA_OK(launch_descriptors(a, v.stream));
    s->desc_n = n;
    if (n_tracks) *n_tracks = n;
    if (out) {
        if (cap < n) { wg_set_error("wgdna_track_descriptors: %llu tracks do not fit", (unsigned long long)n); return WGDNA_ERR_CAPACITY; }
        WG_CUDA_OK(cudaMemcpyAsync(out, s->desc, n * SG_IN * 4, cudaMemcpyDeviceToHost, v.stream));
    }
    WG_CUDA_OK(cudaStreamSynchronize(v.stream));
    return WGDNA_OK;
}

// the surrogate's G(t) for all tracks of the last transport, energy-weighted
// like the IRT's (counts over n_therm * E / 100): G[16][5].  Three launches
// and one host synchronisation: the descriptors, the forward pass (inputs
// standardised on load, the energy-weighted sums of its de-standardised
// outputs added in its last epilogue), and the read-back of those sums.
extern "C" int wgdna_surrogate_chemistry(wgdna_ctx* c, double* G, float* ms) {
    if (!c || !G) { wg_set_error("wgdna_surrogate_chemistry: NULL argument"); return WGDNA_ERR_ARG; }
    CtxView v;
    SgState* s;
    STRY(ensure_state(c, v, &s));
    if (!v.have_transport) { wg_set_error("wgdna_surrogate_chemistry: no transport result in the context"); return WGDNA_ERR_STATE; }
    const uint64_t n = v.nseg;
    if (n > s->desc_cap) {
        STRY(salloc(&s->desc, n * SG_IN)); STRY(salloc(&s->xs, n * SG_IN)); STRY(salloc(&s->pred, n * SG_OUT));
        s->desc_cap = n;
    }
    if (!s->ev[0]) {
        WG_CUDA_OK(cudaEventCreate(&s->ev[0]));
        WG_CUDA_OK(cudaEventCreate(&s->ev[1]));
    }
    WG_CUDA_OK(cudaEventRecord(s->ev[0], v.stream));
    WG_CUDA_OK(cudaMemsetAsync(s->acc, 0, (SG_OUT + 1) * sizeof(double), v.stream));
    DescArgs da{v.rad, v.seg_off, v.nseg, v.Eprim, v.E0, s->desc};
    WG_CUDA_OK(launch_descriptors(da, v.stream));
    s->desc_n = n;
    SgFwdArgs f{};
    f.X = s->desc; f.n = (uint32_t)n; f.w = weights(s); f.Y = nullptr; f.err = s->err;
    f.mma_ns = s->mma_ns; f.give_up_first = s->give_up_first;
    f.xmean = s->xmean; f.xinv = s->xinv; f.ymean = s->ymean; f.ystd = s->ystd;
    f.E = v.Eprim; f.E0 = v.E0; f.acc = s->acc;
    WG_CUDA_OK(launch_sg_forward(f, v.stream));
    WG_CUDA_OK(cudaEventRecord(s->ev[1], v.stream));
    double acc[SG_OUT + 1];
    uint32_t err = 0;
    WG_CUDA_OK(cudaMemcpyAsync(acc, s->acc, sizeof acc, cudaMemcpyDeviceToHost, v.stream));
    WG_CUDA_OK(cudaMemcpyAsync(&err, s->err, 4, cudaMemcpyDeviceToHost, v.stream));
    WG_CUDA_OK(cudaStreamSynchronize(v.stream));
    if (err) {
        wg_set_error("wgdna_surrogate_chemistry: device error flags 0x%x", err);
        cudaMemsetAsync(s->err, 0, 4, v.stream);
        return WGDNA_ERR_DEVICE;
    }
    if (ms) *ms = elapsed_ms(s->ev[0], s->ev[1]);
    for (int k = 0; k < SG_OUT; ++k) G[k] = acc[SG_OUT] > 0 ? acc[k] / acc[SG_OUT] : 0.0;
    return WGDNA_OK;
}
