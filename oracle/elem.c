/* oracle/elem.c -- vector evaluation of the oracle's elementary functions.
 *
 * TEST INFRASTRUCTURE ONLY.  Exposes the functions of om.h (the arithmetic the
 * CUDA path defines in csrc/dmath.cuh and the oracle restates) to the tests,
 * which bound their error against high-precision references in ulps.
 */
#include "om.h"

/* fn: 0 logf  1 expf  2 sinf  3 cosf  4 powf(x, 1.3)  5 log  6 exp  7 expm1  8 cos.
 * The f32 functions take x rounded to f32 and return their f32 result widened. */
int orc_elem(int fn, const double *x, double *y, uint64_t n) {
    for (uint64_t i = 0; i < n; ++i) {
        const float xf = (float)x[i];
        switch (fn) {
        case 0: y[i] = om_logf(xf); break;
        case 1: y[i] = om_expf(xf); break;
        case 2: y[i] = om_sinf(xf); break;
        case 3: y[i] = om_cosf(xf); break;
        case 4: y[i] = om_powf(xf, 1.3f); break;
        case 5: y[i] = om_log(x[i]); break;
        case 6: y[i] = om_exp(x[i]); break;
        case 7: y[i] = om_expm1(x[i]); break;
        case 8: y[i] = om_cos(x[i]); break;
        default: return -1;
        }
    }
    return 0;
}
