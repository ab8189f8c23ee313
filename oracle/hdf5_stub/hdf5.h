/*
 * Stand-in for <hdf5.h> used only to compile the reference's OpenMP driver
 * as the timed CPU baseline (HDF5 is not installed on these machines).  The
 * driver's HDF5 output (testDensitySubGrid_omp.cpp:453-495) becomes a no-op;
 * the transport and balance being timed are untouched.
 */
#ifndef CMI_HDF5_STUB_H
#define CMI_HDF5_STUB_H
typedef long hid_t;
typedef unsigned long long hsize_t;
enum { H5F_ACC_TRUNC = 0, H5P_DEFAULT = 0, H5S_SIMPLE = 0, H5S_SELECT_SET = 0,
       H5T_NATIVE_DOUBLE = 0 };
static inline hid_t H5Fcreate(const char *, int, int, int) { return 1; }
static inline hid_t H5Gcreate(hid_t, const char *, int, int, int) { return 1; }
static inline hid_t H5Screate(int) { return 1; }
static inline int H5Sset_extent_simple(hid_t, int, const hsize_t *, const hsize_t *) { return 0; }
static inline hid_t H5Dcreate(hid_t, const char *, int, hid_t, int, int, int) { return 1; }
static inline int H5Sselect_hyperslab(hid_t, int, const hsize_t *, const void *,
                                      const hsize_t *, const void *) { return 0; }
static inline int H5Dwrite(hid_t, int, hid_t, hid_t, int, const void *) { return 0; }
static inline int H5Sclose(hid_t) { return 0; }
static inline int H5Dclose(hid_t) { return 0; }
static inline int H5Gclose(hid_t) { return 0; }
static inline int H5Fclose(hid_t) { return 0; }
#endif
