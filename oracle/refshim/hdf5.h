// Test infrastructure only: the HDF5 calls the reference's table reader
// makes (EOSX/src/utils/eos_utils.hxx get_hdf5_*_dset,
// EOSX/src/eos_3p_tabulated3d/eos_3p_tabulated3d.hxx init), served from an
// in-memory set of named datasets that a test registers through the
// harness (ora_h5_put_*).  No file is read: any file name opens that set.
#ifndef AXREF_SHIM_HDF5_H
#define AXREF_SHIM_HDF5_H
#include <cstring>
#include <map>
#include <string>
#include <vector>
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

struct axref_h5_dset {
  bool is_int = false;
  std::vector<double> d;
  std::vector<int> i;
};
inline std::map<std::string, axref_h5_dset> &axref_h5_store() {
  static std::map<std::string, axref_h5_dset> s;
  return s;
}
// open dataset handles: handle h (>= 1) names axref_h5_handles()[h - 1]
inline std::vector<std::string> &axref_h5_handles() {
  static std::vector<std::string> h;
  return h;
}
inline hid_t H5Pcreate(int) { return 1; }
inline herr_t H5Pclose(hid_t) { return 0; }
inline hid_t H5Fopen(const char *, int, hid_t) {
  return axref_h5_store().empty() ? -1 : 1;
}
inline herr_t H5Fclose(hid_t) { return 0; }
inline hid_t H5Dopen(hid_t, const char *name, hid_t) {
  if (!axref_h5_store().count(name))
    return -1;
  axref_h5_handles().push_back(name);
  return hid_t(axref_h5_handles().size());
}
inline herr_t H5Dclose(hid_t) { return 0; }
inline hid_t H5Dget_type(hid_t dset) { return dset; }
inline H5T_class_t H5Tget_class(hid_t dset) {
  return axref_h5_store()[axref_h5_handles()[dset - 1]].is_int ? H5T_INTEGER : H5T_FLOAT;
}
inline herr_t H5Tclose(hid_t) { return 0; }
inline herr_t H5Dread(hid_t dset, int memtype, int, int, hid_t, void *buf) {
  const axref_h5_dset &s = axref_h5_store()[axref_h5_handles()[dset - 1]];
  if (memtype == H5T_NATIVE_INT) {
    if (!s.is_int)
      return -1;
    std::memcpy(buf, s.i.data(), s.i.size() * sizeof(int));
  } else {
    if (s.is_int)
      return -1;
    std::memcpy(buf, s.d.data(), s.d.size() * sizeof(double));
  }
  return 0;
}
#endif
