/* Empty stand-in: the HDF5 writer (src/phdf5.cpp) is not part of the solve
 * path and is not compiled; only the types its header names are declared.
 * TEST INFRASTRUCTURE ONLY (oracle/_ref). */
#ifndef PP_SHIM_HDF5_H
#define PP_SHIM_HDF5_H
typedef long long hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;
typedef long long hssize_t;
#endif
