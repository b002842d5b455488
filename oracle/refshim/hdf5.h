// Test infrastructure only: HDF5 declarations the reference's table reader
// names.  No test reads an HDF5 file; every call aborts.
#ifndef AXREF_SHIM_HDF5_H
#define AXREF_SHIM_HDF5_H
#include <cstdlib>
typedef long long hid_t;
typedef int herr_t;
typedef int H5T_class_t;
#define H5P_DEFAULT 0
#define H5P_FILE_ACCESS 1
#define H5P_DATASET_XFER 2
#define H5F_ACC_RDONLY 0
#define H5S_ALL 0
#define H5T_NATIVE_INT 1
#define H5T_NATIVE_DOUBLE 2
#define H5T_INTEGER 0
#define H5T_FLOAT 1
[[noreturn]] inline void axref_no_hdf5() { std::abort(); }
inline hid_t H5Pcreate(int) { axref_no_hdf5(); }
inline herr_t H5Pclose(hid_t) { axref_no_hdf5(); }
inline hid_t H5Fopen(const char *, int, hid_t) { axref_no_hdf5(); }
inline herr_t H5Fclose(hid_t) { axref_no_hdf5(); }
inline hid_t H5Dopen(hid_t, const char *, hid_t) { axref_no_hdf5(); }
inline herr_t H5Dclose(hid_t) { axref_no_hdf5(); }
inline hid_t H5Dget_type(hid_t) { axref_no_hdf5(); }
inline H5T_class_t H5Tget_class(hid_t) { axref_no_hdf5(); }
inline herr_t H5Tclose(hid_t) { axref_no_hdf5(); }
inline herr_t H5Dread(hid_t, int, int, int, hid_t, void *) { axref_no_hdf5(); }
#endif
