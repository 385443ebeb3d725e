/*
 * Empty placeholder for <hdf5.h>.  src/dataio.h includes it but declares no
 * HDF5 types in its prototypes; src/dataio.c (the only file that uses HDF5)
 * is replaced by synth_dataio.c in the oracle build.  Test infrastructure.
 */
#ifndef SSG_REF_HDF5_PLACEHOLDER_H
#define SSG_REF_HDF5_PLACEHOLDER_H
#endif
