/* Empty stand-in for <gsl/gsl_sf_bessel.h>. The legacy engine's max_emc.c
 * includes it but calls none of its functions. Test infrastructure only. */
#ifndef DFG_ORACLE_SHIM_GSL_SF_BESSEL_H
#define DFG_ORACLE_SHIM_GSL_SF_BESSEL_H
#endif
