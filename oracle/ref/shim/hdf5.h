/*
 * Type-only stand-in for hdf5.h, written for this project: the oracle build
 * of the reference compiles none of the HDF5 output/resume sources, but some
 * headers name these types in prototypes.  Test infrastructure only.
 */
#ifndef PVOF_SHIM_HDF5_H
#define PVOF_SHIM_HDF5_H
typedef long hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;
typedef long long hssize_t;
#endif
