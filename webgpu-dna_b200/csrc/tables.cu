// tables.cu -- loads the cross-section table blob into device memory.
//
// The blob is the float32 image of public/cross_sections.wgsl:9-72 written by
// webgpu-dna_b200/data/gen_tables.py (layout documented there).  Small tables
// are packed in the order of common.cuh's S_* offsets so the transport kernel
// can copy them to shared memory in one pass; the Born CDF / energy-transfer
// tables (2 x 5 x 58 x 250 floats) stay in global memory (L2 resident).
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"

namespace wg {

struct Entry { std::string name; uint32_t dtype, count, off; };

static bool find(const std::vector<Entry>& es, const char* name, uint32_t count, uint32_t* off) {
    for (const auto& e : es)
        if (e.name == name) {
            if (count && e.count != count) return false;
            *off = e.off;
            return true;
        }
    return false;
}

int tables_load(const char* path, Tables* out, float** d_small, float2** d_xcw) {
    FILE* f = fopen(path, "rb");
    if (!f) { wg_set_error("cannot open cross-section blob %s", path); return WGDNA_ERR_TABLES; }
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    std::vector<unsigned char> b((size_t)sz);
    size_t got = fread(b.data(), 1, (size_t)sz, f);
    fclose(f);
    if (got != (size_t)sz || sz < 16 || memcmp(b.data(), "WGDNAXS1", 8) != 0) {
        wg_set_error("%s is not a cross-section blob", path);
        return WGDNA_ERR_TABLES;
    }
    uint32_t n, dbytes;
    memcpy(&n, b.data() + 8, 4);
    memcpy(&dbytes, b.data() + 12, 4);
    size_t hsz = (16 + 40 * (size_t)n + 15) & ~(size_t)15;
    if (hsz + dbytes != (size_t)sz) { wg_set_error("cross-section blob %s is truncated", path); return WGDNA_ERR_TABLES; }
    std::vector<Entry> es;
    for (uint32_t i = 0; i < n; ++i) {
        const unsigned char* e = b.data() + 16 + 40 * i;
        Entry x;
        x.name.assign((const char*)e, strnlen((const char*)e, 24));
        memcpy(&x.dtype, e + 24, 4);
        memcpy(&x.count, e + 28, 4);
        memcpy(&x.off, e + 32, 4);
        es.push_back(x);
    }
    const unsigned char* data = b.data() + hsz;
    auto u32 = [&](const char* nm, uint32_t* v) {
        uint32_t off;
        if (!find(es, nm, 1, &off)) return false;
        memcpy(v, data + off, 4);
        return true;
    };
    auto f32 = [&](const char* nm, float* v) {
        uint32_t off;
        if (!find(es, nm, 1, &off)) return false;
        memcpy(v, data + off, 4);
        return true;
    };
    Tables t{};
    bool ok = u32("XN", &t.xn) && u32("N_AE", &t.n_ae) && u32("N_AC", &t.n_ac) && u32("N_WE", &t.n_we) &&
              u32("N_WR", &t.n_wr) && u32("N_VIB", &t.n_vib) && f32("LOG_XE0", &t.log_xe0) &&
              f32("INV_LOG_XE_STEP", &t.inv_log_xe_step) && f32("LOG_XAE0", &t.log_xae0) &&
              f32("INV_LOG_XAE_STEP", &t.inv_log_xae_step);
    if (!ok || t.xn != (uint32_t)XN_ || t.n_ae != (uint32_t)NAE_ || t.n_ac != (uint32_t)NAC_ ||
        t.n_we != (uint32_t)NWE_ || t.n_wr != (uint32_t)NWR_ || t.n_vib != (uint32_t)NVIB_) {
        wg_set_error("cross-section blob %s has unexpected table sizes", path);
        return WGDNA_ERR_TABLES;
    }
    std::vector<float> small(S_TOTAL_PAD, 0.0f);
    auto put = [&](const char* nm, int dst, uint32_t count) {
        uint32_t off;
        if (!find(es, nm, count, &off)) return false;
        memcpy(small.data() + dst, data + off, 4ull * count);
        return true;
    };
    ok = put("XE", S_XE, XN_) && put("XI", S_XI, XN_) && put("XC", S_XC, XN_) && put("XL", S_XL, XN_);
    char nm[16];
    for (int k = 0; k < 5 && ok; ++k) {
        snprintf(nm, sizeof nm, "XSF%d", k); ok = ok && put(nm, S_XSF + k * XN_, XN_);
        snprintf(nm, sizeof nm, "XEF%d", k); ok = ok && put(nm, S_XEF + k * XN_, XN_);
    }
    ok = ok && put("XAE", S_XAE, NAE_) && put("XAC", S_XAC, NAE_ * NAC_) && put("XWE", S_XWE, NWE_) &&
         put("XVE", S_XVE, NVIB_) && put("XVS", S_XVS, NVIB_) && put("XVMF", S_XVMF, NVIB_ * 9) &&
         put("VIB_LEV", S_VIB, 9);
    std::vector<float> xwc(5 * NWE_ * NWR_), xwt(5 * NWE_ * NWR_);
    std::vector<float2> xcw(5 * NWE_ * NWR_);
    for (int k = 0; k < 5 && ok; ++k) {
        uint32_t off;
        snprintf(nm, sizeof nm, "XWC%d", k);
        ok = ok && find(es, nm, NWE_ * NWR_, &off);
        if (ok) memcpy(xwc.data() + k * NWE_ * NWR_, data + off, 4ull * NWE_ * NWR_);
        snprintf(nm, sizeof nm, "XWT%d", k);
        ok = ok && find(es, nm, NWE_ * NWR_, &off);
        if (ok) memcpy(xwt.data() + k * NWE_ * NWR_, data + off, 4ull * NWE_ * NWR_);
    }
    if (!ok) { wg_set_error("cross-section blob %s is missing an array", path); return WGDNA_ERR_TABLES; }
    for (size_t i = 0; i < xcw.size(); ++i) xcw[i] = make_float2(xwc[i], xwt[i]);
    // guide table: the CDF at breakpoints 0, 16, ..., 240 of every (shell, energy) row
    for (int k = 0; k < 5; ++k)
        for (int r = 0; r < NWE_; ++r)
            for (int m = 0; m < GUIDES; ++m)
                small[S_GUIDE + (k * NWE_ + r) * GUIDES + m] = xwc[(size_t)k * NWE_ * NWR_ + r * NWR_ + 16 * m];
    WG_CUDA_OK(cudaMalloc(d_small, small.size() * 4));
    WG_CUDA_OK(cudaMalloc(d_xcw, xcw.size() * sizeof(float2)));
    WG_CUDA_OK(cudaMemcpy(*d_small, small.data(), small.size() * 4, cudaMemcpyHostToDevice));
    WG_CUDA_OK(cudaMemcpy(*d_xcw, xcw.data(), xcw.size() * sizeof(float2), cudaMemcpyHostToDevice));
    t.small = *d_small;
    t.xcw = *d_xcw;
    *out = t;
    return WGDNA_OK;
}

}  // namespace wg
