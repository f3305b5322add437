/*
 * No-op stand-in for the HDF5 calls of the reference's particle dump
 * (src/RW_IO.cpp:376-461), so the unmodified driver compiles without HDF5.
 * Nothing is written. TEST INFRASTRUCTURE ONLY.
 */
#ifndef SPB_TEST_HDF5_STUB_H
#define SPB_TEST_HDF5_STUB_H
#include "mpi.h"   /* parallel HDF5 builds bring MPI in through this header */
typedef long long hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;
#define H5F_ACC_TRUNC 0
#define H5P_DEFAULT 0
#define H5S_SCALAR 0
#define H5S_ALL 0
#define H5T_NATIVE_INT 0
#define H5T_NATIVE_FLOAT 0
#define H5T_IEEE_F32BE 0
static inline hid_t H5Fcreate(const char *, unsigned, hid_t, hid_t) { return 1; }
static inline hid_t H5Screate(int) { return 1; }
static inline hid_t H5Screate_simple(int, const hsize_t *, const hsize_t *) { return 1; }
static inline hid_t H5Acreate(hid_t, const char *, hid_t, hid_t, hid_t, hid_t) { return 1; }
static inline herr_t H5Awrite(hid_t, hid_t, const void *) { return 0; }
static inline hid_t H5Gcreate(hid_t, const char *, hid_t, hid_t, hid_t) { return 1; }
static inline hid_t H5Dcreate(hid_t, const char *, hid_t, hid_t, hid_t, hid_t, hid_t) { return 1; }
static inline herr_t H5Dwrite(hid_t, hid_t, hid_t, hid_t, hid_t, const void *) { return 0; }
static inline herr_t H5Aclose(hid_t) { return 0; }
static inline herr_t H5Sclose(hid_t) { return 0; }
static inline herr_t H5Dclose(hid_t) { return 0; }
static inline herr_t H5Gclose(hid_t) { return 0; }
static inline herr_t H5Fclose(hid_t) { return 0; }
#endif
