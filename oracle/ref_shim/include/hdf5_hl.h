/* The HDF5 high-level (H5LT) calls that appear in the reference's reionization sources; see
   hdf5.h.  Test infrastructure for oracle/_ref only. */
#ifndef RG_SHIM_HDF5_HL_H
#define RG_SHIM_HDF5_HL_H
#include "hdf5.h"
#ifdef __cplusplus
extern "C" {
#endif

herr_t H5LTset_attribute_double(hid_t loc, const char* obj, const char* attr, const double* buf, size_t size);
herr_t H5LTget_attribute_double(hid_t loc, const char* obj, const char* attr, double* buf);
herr_t H5LTmake_dataset_double(hid_t loc, const char* name, int rank, const hsize_t* dims, const double* buf);
herr_t H5LTread_dataset_double(hid_t loc, const char* name, double* buf);
herr_t H5LTget_dataset_ndims(hid_t loc, const char* name, int* rank);
herr_t H5LTget_dataset_info(hid_t loc, const char* name, hsize_t* dims, H5T_class_t* cls, size_t* size);

#ifdef __cplusplus
}
#endif
#endif
