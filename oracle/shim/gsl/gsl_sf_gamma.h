/* Stand-in for GSL's gsl_sf_lnfact, used by the reference's calc_sum_fact
 * (dragonfly/src/iterate.c:101,107). Test infrastructure only.
 *
 * GSL is not vendored with the reference and its version is not pinned, so the
 * exact table GSL uses is not reproduced: ln(n!) = lgamma(n + 1). The product
 * computes sum_fact the same way, so oracle and product agree; the value only
 * shifts each frame's reported log-likelihood by a constant.
 */
#ifndef DFG_ORACLE_SHIM_GSL_SF_GAMMA_H
#define DFG_ORACLE_SHIM_GSL_SF_GAMMA_H

#include <math.h>

static inline double gsl_sf_lnfact(unsigned int n) { return lgamma((double)n + 1.0); }

#endif
