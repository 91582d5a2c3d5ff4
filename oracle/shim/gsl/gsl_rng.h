/* Empty stand-in for <gsl/gsl_rng.h>. The legacy engine's iterate.h includes
 * it; the parts of the legacy engine the oracle recipe compiles (max_emc.c,
 * interp.c) draw no random numbers. Test infrastructure only. */
#ifndef DFG_ORACLE_SHIM_GSL_RNG_H
#define DFG_ORACLE_SHIM_GSL_RNG_H
#endif
