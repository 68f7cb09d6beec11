/* oracle/tables.c -- loads the cross-section blob into the oracle.
 * TEST INFRASTRUCTURE ONLY (CPU oracle).
 *
 * The blob is the float32 image of public/cross_sections.wgsl:9-72 written by
 * webgpu-dna_b200/data/gen_tables.py; its layout is documented there.  This
 * loader is independent of the product's loader (webgpu-dna_b200/csrc/tables.cu).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "oracle.h"
#include "internal.h"

orc_tables g_tab;
static unsigned char *g_blob;

static const void *find(const unsigned char *head, uint32_t n, const unsigned char *data,
                        const char *name, uint32_t want_count) {
    for (uint32_t i = 0; i < n; ++i) {
        const unsigned char *e = head + 16 + 40 * i;
        if (strncmp((const char *)e, name, 24) == 0) {
            uint32_t cnt, off;
            memcpy(&cnt, e + 28, 4);
            memcpy(&off, e + 32, 4);
            if (want_count && cnt != want_count) return NULL;
            return data + off;
        }
    }
    return NULL;
}

int orc_load_tables(const char *path) {
    FILE *f = fopen(path, "rb");
    if (!f) return -1;
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    unsigned char *b = (unsigned char *)malloc((size_t)sz);
    if (!b || fread(b, 1, (size_t)sz, f) != (size_t)sz) { fclose(f); free(b); return -2; }
    fclose(f);
    if (memcmp(b, "WGDNAXS1", 8) != 0) { free(b); return -3; }
    uint32_t n, dbytes;
    memcpy(&n, b + 8, 4);
    memcpy(&dbytes, b + 12, 4);
    size_t hsz = 16 + 40 * (size_t)n;
    hsz = (hsz + 15) & ~(size_t)15;
    if (hsz + dbytes != (size_t)sz) { free(b); return -4; }
    const unsigned char *data = b + hsz;
    orc_tables t;
    memset(&t, 0, sizeof t);
#define U32(nm) do { const void *p_ = find(b, n, data, #nm, 1); if (!p_) { free(b); return -5; } memcpy(&t.nm, p_, 4); } while (0)
#define F32S(nm) do { const void *p_ = find(b, n, data, #nm, 1); if (!p_) { free(b); return -5; } memcpy(&t.nm, p_, 4); } while (0)
    U32(XN); U32(N_AE); U32(N_AC); U32(N_WE); U32(N_WR); U32(N_VIB);
    F32S(LOG_XE0); F32S(INV_LOG_XE_STEP); F32S(LOG_XAE0); F32S(INV_LOG_XAE_STEP);
    F32S(LOG_XWE0); F32S(INV_LOG_XWE_STEP);
#define ARR(dst, nm, cnt) do { dst = (const float *)find(b, n, data, nm, cnt); if (!dst) { free(b); return -6; } } while (0)
    ARR(t.XE, "XE", t.XN); ARR(t.XI, "XI", t.XN); ARR(t.XC, "XC", t.XN); ARR(t.XL, "XL", t.XN);
    char nm[16];
    for (int k = 0; k < 5; ++k) {
        snprintf(nm, sizeof nm, "XSF%d", k); ARR(t.XSF[k], nm, t.XN);
        snprintf(nm, sizeof nm, "XEF%d", k); ARR(t.XEF[k], nm, t.XN);
        snprintf(nm, sizeof nm, "XWC%d", k); ARR(t.XWC[k], nm, t.N_WE * t.N_WR);
        snprintf(nm, sizeof nm, "XWT%d", k); ARR(t.XWT[k], nm, t.N_WE * t.N_WR);
    }
    ARR(t.XAE, "XAE", t.N_AE); ARR(t.XAC, "XAC", t.N_AE * t.N_AC);
    ARR(t.XWE, "XWE", t.N_WE);
    ARR(t.XVE, "XVE", t.N_VIB); ARR(t.XVS, "XVS", t.N_VIB);
    ARR(t.XVMF, "XVMF", t.N_VIB * 9); ARR(t.VIB_LEV, "VIB_LEV", 9);
    free(g_blob);
    g_blob = b;
    t.loaded = 1;
    g_tab = t;
    return 0;
}

void orc_free(void *p) { free(p); }
