/* Types, constants and prototypes of the HDF5 calls that appear in the reference's reionization
   sources (HDF5 1.10 API names).  The step itself reads and writes no HDF5 file; ref_stubs.c
   makes every one of these calls abort.  Test infrastructure for oracle/_ref only. */
#ifndef RG_SHIM_HDF5_H
#define RG_SHIM_HDF5_H
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef int64_t hid_t;
typedef int herr_t;
typedef int htri_t;
typedef unsigned long long hsize_t;
typedef long long hssize_t;
typedef enum H5T_class_t { H5T_NO_CLASS = -1, H5T_INTEGER = 0, H5T_FLOAT = 1 } H5T_class_t;
typedef enum H5S_seloper_t { H5S_SELECT_SET = 0 } H5S_seloper_t;
typedef enum H5FD_mpio_xfer_t { H5FD_MPIO_INDEPENDENT = 0, H5FD_MPIO_COLLECTIVE = 1 } H5FD_mpio_xfer_t;

#define H5P_DEFAULT ((hid_t)0)
#define H5E_DEFAULT ((hid_t)0)
#define H5S_ALL ((hid_t)0)
#define H5P_DATASET_XFER ((hid_t)101)
#define H5P_DATASET_CREATE ((hid_t)102)
#define H5P_FILE_ACCESS ((hid_t)103)
#define H5T_NATIVE_FLOAT ((hid_t)201)
#define H5T_NATIVE_DOUBLE ((hid_t)202)
#define H5T_NATIVE_INT ((hid_t)203)
#define H5T_NATIVE_LLONG ((hid_t)204)
#define H5F_ACC_RDONLY 0u
#define H5F_ACC_RDWR 1u
#define H5F_ACC_TRUNC 2u

hid_t H5Fopen(const char* name, unsigned flags, hid_t fapl);
hid_t H5Fcreate(const char* name, unsigned flags, hid_t fcpl, hid_t fapl);
herr_t H5Fclose(hid_t f);
hid_t H5Pcreate(hid_t cls);
herr_t H5Pclose(hid_t p);
herr_t H5Pset_dxpl_mpio(hid_t p, H5FD_mpio_xfer_t mode);
herr_t H5Pset_fapl_mpio(hid_t p, int comm, int info);
herr_t H5Pset_chunk(hid_t p, int ndims, const hsize_t* dims);
hid_t H5Screate_simple(int rank, const hsize_t* dims, const hsize_t* maxdims);
herr_t H5Sclose(hid_t s);
herr_t H5Sselect_hyperslab(hid_t s, H5S_seloper_t op, const hsize_t* start, const hsize_t* stride,
                           const hsize_t* count, const hsize_t* block);
herr_t H5Sselect_none(hid_t s);
hid_t H5Dcreate(hid_t loc, const char* name, hid_t type, hid_t space, hid_t lcpl, hid_t dcpl, hid_t dapl);
herr_t H5Dwrite(hid_t d, hid_t mtype, hid_t mspace, hid_t fspace, hid_t xfer, const void* buf);
herr_t H5Dclose(hid_t d);
htri_t H5Lexists(hid_t loc, const char* name, hid_t lapl);
typedef herr_t (*H5E_auto2_t)(hid_t estack, void* client_data);
herr_t H5Eget_auto2(hid_t estack_id, H5E_auto2_t* func, void** client_data);
herr_t H5Eset_auto2(hid_t estack_id, H5E_auto2_t func, void* client_data);
#define H5Eget_auto H5Eget_auto2
#define H5Eset_auto H5Eset_auto2

#ifdef __cplusplus
}
#endif
#endif
