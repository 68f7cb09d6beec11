/* chemgrid.c -- CPU restatement of the grid-hash chemistry backend
 * (src/shaders/chemistry.wgsl:1-334 with the schedule of
 * src/chemistry/schedule.ts:38-46) for tests: sequential, so the claims of
 * competing pairs resolve in radical order and the hash chains hold the
 * radicals in descending index order.  Random streams and arithmetic are
 * those of webgpu-dna_b200/csrc/chemgrid.cu, so every diffusion step matches
 * the CUDA path bit for bit; only the order of competing claims differs. */
#include <stdlib.h>
#include <string.h>

#include "oracle.h"
#include "om.h"

#define CG_HASH 8388608u
#define CG_CELL 1.5f

static uint32_t cg_hash(int ix, int iy, int iz) {
    uint32_t h = (uint32_t)(ix * 73856093) ^ (uint32_t)(iy * 19349663) ^ (uint32_t)(iz * 83492791);
    return h % CG_HASH;
}

static float cg_sigma(int a, int b) {
    if (a > b) { int t = a; a = b; b = t; }
    if (a == 0 && b == 0) return 0.44f;
    if (a == 0 && b == 1) return 0.57f;
    if (a == 0 && b == 2) return 0.45f;
    if (a == 1 && b == 1) return 0.54f;
    if (a == 1 && b == 2) return 0.61f;
    if (a == 1 && b == 3) return 0.47f;
    if (a == 2 && b == 2) return 0.34f;
    return 0.0f;
}

static float cg_pc(int a, int b) {
    if (a > b) { int t = a; a = b; b = t; }
    if (a == 0 && b == 0) return 0.376f;
    if (a == 0 && b == 1) return 0.980f;
    if (a == 0 && b == 2) return 0.511f;
    if (a == 1 && b == 1) return 0.125f;
    if (a == 1 && b == 2) return 0.455f;
    if (a == 1 && b == 3) return 0.538f;
    if (a == 2 && b == 2) return 0.216f;
    return 0.0f;
}

static int cg_prod(int a, int b) {
    if (a > b) { int t = a; a = b; b = t; }
    if (a == 0 && b == 0) return 1;
    if (a == 1 && b == 1) return 2;
    if (a == 1 && b == 2) return 2;
    if (a == 1 && b == 3) return 3;
    if (a == 2 && b == 2) return 2;
    return 0;
}

static void gauss2(float u1, float u2, float *g0, float *g1) {
    u1 = fmaxf(u1, 1e-10f);
    float r = sqrtf(-2.0f * om_logf(u1));
    float s, c;
    om_sincosf(6.28318530f * u2, &s, &c);
    *g0 = r * c;
    *g1 = r * s;
}

static int cg_cell(float x) { return (int)floorf(x / CG_CELL); }

static void count(const float *pos, const uint32_t *alive, uint32_t n, const uint32_t *prod, uint32_t *out) {
    memset(out, 0, 5 * sizeof(uint32_t));
    for (uint32_t i = 0; i < n; ++i) {
        if (!alive[i]) continue;
        int k = (int)rintf(pos[4 * i + 3]);
        if (k >= 0 && k <= 2) out[k]++;
    }
    out[3] = prod[0]; out[4] = prod[1];
}

int orc_chem_grid(const float *rad, uint32_t n, uint64_t seed, float *pos, uint32_t *alive, uint32_t counts[8][5]) {
    static const float DT[7] = {0.0001f, 0.001f, 0.005f, 0.05f, 0.5f, 3.0f, 30.0f};
    static const int NS[7] = {10, 9, 18, 18, 18, 30, 30};
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    int *head = (int *)malloc(CG_HASH * sizeof(int));
    int *next = (int *)malloc((n ? n : 1) * sizeof(int));
    if (!head || !next) { free(head); free(next); return -1; }
    uint32_t prod[2] = {0, 0};
    for (uint32_t i = 0; i < n; ++i) {
        const float *r = rad + 4 * i;
        int kind = (int)(lrintf(r[3]) % 8);
        float *p = pos + 4 * i;
        p[0] = r[0]; p[1] = r[1]; p[2] = r[2]; p[3] = (float)kind;
        alive[i] = 1;
        om_u4 w = om_philox(i, 0xffffffffu, 0u, 6u, k0, k1);
        float sigma = 0.0f;
        int disp = 1;
        if (kind == 0) sigma = 0.462f;
        else if (kind == 1) sigma = 1.764f;
        else if (kind == 2) sigma = 1.309f;
        else if (kind == 3) sigma = om_u01f(w.v[3]) < 0.5f ? 0.462f : 0.0f;
        else if (kind == 5) { kind = 1; sigma = 0.0f; }
        else disp = 0;
        if (disp) {
            float g0, g1, g2, g3;
            gauss2(om_u01f(w.v[0]), om_u01f(w.v[1]), &g0, &g1);
            om_u4 w2 = om_philox(i, 0xfffffffeu, 0u, 6u, k0, k1);
            gauss2(om_u01f(w2.v[0]), om_u01f(w2.v[1]), &g2, &g3);
            p[0] = p[0] + sigma * g0;
            p[1] = p[1] + sigma * g1;
            p[2] = p[2] + sigma * g2;
            p[3] = (float)kind;
        }
    }
    count(pos, alive, n, prod, counts[0]);
    uint32_t step = 0;
    for (int stage = 0; stage < 7; ++stage) {
        for (int k = 0; k < NS[stage]; ++k) {
            ++step;
            const float dt = DT[stage];
            for (uint32_t i = 0; i < n; ++i) {                                    /* diffuse */
                if (!alive[i]) continue;
                float *p = pos + 4 * i;
                int kind = (int)rintf(p[3]);
                float D;
                if (kind == 0) D = 2.2f; else if (kind == 1) D = 4.9f; else if (kind == 2) D = 7.0f;
                else if (kind == 3) D = 9.0f; else continue;
                float sigma = sqrtf(2.0f * D * dt);
                om_u4 w = om_philox(i, step, 0u, 6u, k0, k1);
                float g0, g1, g2, g3;
                gauss2(om_u01f(w.v[0]), om_u01f(w.v[1]), &g0, &g1);
                gauss2(om_u01f(w.v[2]), om_u01f(w.v[3]), &g2, &g3);
                p[0] += sigma * g0; p[1] += sigma * g1; p[2] += sigma * g2;
            }
            for (uint32_t h = 0; h < CG_HASH; ++h) head[h] = -1;                  /* clear + build */
            for (uint32_t i = 0; i < n; ++i) {
                if (!alive[i]) { next[i] = -1; continue; }
                const float *p = pos + 4 * i;
                uint32_t h = cg_hash(cg_cell(p[0]), cg_cell(p[1]), cg_cell(p[2]));
                next[i] = head[h];
                head[h] = (int)i;
            }
            for (uint32_t i = 0; i < n; ++i) {                                    /* react */
                if (!alive[i]) continue;
                const float *pi = pos + 4 * i;
                const int ki = (int)rintf(pi[3]);
                if (ki < 0 || ki > 3) continue;
                const int ix = cg_cell(pi[0]), iy = cg_cell(pi[1]), iz = cg_cell(pi[2]);
                uint32_t draw = 0;
                om_u4 w = {{0, 0, 0, 0}};
                int done = 0;
                for (int dz = -1; dz <= 1 && !done; ++dz)
                    for (int dy = -1; dy <= 1 && !done; ++dy)
                        for (int dx = -1; dx <= 1 && !done; ++dx) {
                            int j = head[cg_hash(ix + dx, iy + dy, iz + dz)];
                            for (uint32_t it = 0; it < 1024u && j >= 0 && !done; ++it) {
                                const uint32_t ju = (uint32_t)j;
                                const int jn = next[ju];
                                if (ju <= i || !alive[ju]) { j = jn; continue; }
                                const float *pj = pos + 4 * ju;
                                const int kj = (int)rintf(pj[3]);
                                if (kj < 0 || kj > 3) { j = jn; continue; }
                                const float R = cg_sigma(ki, kj);
                                if (R <= 0.0f) { j = jn; continue; }
                                const float ddx = pi[0] - pj[0], ddy = pi[1] - pj[1], ddz = pi[2] - pj[2];
                                if (ddx * ddx + ddy * ddy + ddz * ddz > R * R) { j = jn; continue; }
                                if ((draw & 3u) == 0u) w = om_philox(i, step, 1u + (draw >> 2), 6u, k0, k1);
                                const uint32_t word = w.v[draw & 3u];
                                draw++;
                                if (om_u01f(word) >= cg_pc(ki, kj)) { j = jn; continue; }
                                alive[i] = 0; alive[ju] = 0;
                                const int pr = cg_prod(ki, kj);
                                if (pr == 1) prod[0]++;
                                else if (pr == 2) prod[1]++;
                                else if (pr == 3) {
                                    const uint32_t e = ki == 1 ? i : ju;
                                    pos[4 * e + 3] = 2.0f;
                                    alive[e] = 1;
                                }
                                done = 1;
                            }
                        }
            }
        }
        count(pos, alive, n, prod, counts[stage + 1]);
    }
    free(head); free(next);
    return 0;
}
