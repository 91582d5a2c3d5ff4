/* Empty stand-in for <hdf5.h>. The reference's emcfile.h includes it, but the
 * oracle build leaves out emcfile.c (the only HDF5 user) and parses the binary
 * .emc format itself. Test infrastructure only. */
#ifndef DFG_ORACLE_SHIM_HDF5_H
#define DFG_ORACLE_SHIM_HDF5_H
#endif
