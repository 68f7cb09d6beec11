/* oracle/internal.h -- shared state of the CPU oracle (test infrastructure). */
#ifndef WGDNA_ORACLE_INTERNAL_H
#define WGDNA_ORACLE_INTERNAL_H
#include <stdint.h>

/* The cross-section table set of public/cross_sections.wgsl:9-72. */
typedef struct {
    const float *XE, *XI, *XC, *XL;
    const float *XSF[5], *XEF[5];
    const float *XAE, *XAC;
    const float *XWE, *XWC[5], *XWT[5];
    const float *XVE, *XVS, *XVMF, *VIB_LEV;
    uint32_t XN, N_AE, N_AC, N_WE, N_WR, N_VIB;
    float LOG_XE0, INV_LOG_XE_STEP, LOG_XAE0, INV_LOG_XAE_STEP, LOG_XWE0, INV_LOG_XWE_STEP;
    int loaded;
} orc_tables;

extern orc_tables g_tab;

#endif
