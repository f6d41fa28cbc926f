/*
 * TEST INFRASTRUCTURE ONLY.  Declaration-only stand-in for the HDF5 C API so
 * that LibAPR's headers (which include the .apr file IO through
 * numerics/APRReconstruction.hpp -> LazyData.hpp -> io/APRFile.hpp) compile
 * for the CPU oracle build in oracle/_ref.  No IO entry point is ever called:
 * every function returns a failure value.  HDF5 itself is not installed.
 */
#ifndef APRB_ORACLE_HDF5_STUB_H
#define APRB_ORACLE_HDF5_STUB_H
#include <stdint.h>
#include <stddef.h>
#include <sys/types.h>
typedef int64_t hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;
typedef long long hssize_t;
typedef int htri_t;
typedef struct { hsize_t nlinks; int storage_type; int64_t max_corder; int mounted; } H5G_info_t;
typedef enum { H5S_SELECT_SET = 0 } H5S_seloper_t;
typedef enum { H5T_DIR_DEFAULT = 0 } H5T_direction_t;
typedef enum { H5G_GROUP = 0, H5G_DATASET = 1 } H5G_obj_t;
typedef enum { H5S_SCALAR = 0 } H5S_class_t;
typedef herr_t (*H5E_auto1_t)(void *);
#define H5P_DEFAULT ((hid_t)0)
#define H5P_FILE_ACCESS ((hid_t)0)
#define H5F_ACC_TRUNC 0u
#define H5F_ACC_RDWR 1u
#define H5F_ACC_RDONLY 0u
#define H5T_NATIVE_UINT64 ((hid_t)1)
#define H5T_NATIVE_FLOAT ((hid_t)2)
#define H5T_NATIVE_UINT16 ((hid_t)3)
#define H5T_NATIVE_UINT8 ((hid_t)4)
#define H5T_NATIVE_INT16 ((hid_t)5)
#define H5T_NATIVE_INT ((hid_t)6)
#define H5T_NATIVE_UINT ((hid_t)7)
#define H5T_NATIVE_INT8 ((hid_t)8)
#define H5T_NATIVE_INT64 ((hid_t)9)
#define H5T_NATIVE_DOUBLE ((hid_t)10)
#define H5T_C_S1 ((hid_t)11)
static inline herr_t H5Gclose(hid_t) { return -1; }
static inline hid_t H5Gopen2(hid_t, const char *, hid_t) { return -1; }
static inline hid_t H5Gcreate2(hid_t, const char *, hid_t, hid_t, hid_t) { return -1; }
static inline herr_t H5Gget_num_objs(hid_t, hsize_t *n) { if (n) *n = 0; return -1; }
static inline int H5Gget_objtype_by_idx(hid_t, hsize_t) { return -1; }
static inline ssize_t H5Gget_objname_by_idx(hid_t, hsize_t, char *, size_t) { return -1; }
static inline herr_t H5Gget_info_by_name(hid_t, const char *, H5G_info_t *, hid_t) { return -1; }
static inline herr_t H5Sclose(hid_t) { return -1; }
static inline hid_t H5Screate_simple(int, const hsize_t *, const hsize_t *) { return -1; }
static inline hid_t H5Screate(H5S_class_t) { return -1; }
static inline herr_t H5Sselect_hyperslab(hid_t, H5S_seloper_t, const hsize_t *, const hsize_t *, const hsize_t *, const hsize_t *) { return -1; }
static inline int H5Sget_simple_extent_dims(hid_t, hsize_t *, hsize_t *) { return -1; }
static inline int H5Sget_simple_extent_ndims(hid_t) { return -1; }
static inline herr_t H5Aclose(hid_t) { return -1; }
static inline herr_t H5Aread(hid_t, hid_t, void *) { return -1; }
static inline herr_t H5Awrite(hid_t, hid_t, const void *) { return -1; }
static inline hid_t H5Aopen(hid_t, const char *, hid_t) { return -1; }
static inline hid_t H5Acreate2(hid_t, const char *, hid_t, hid_t, hid_t, hid_t) { return -1; }
static inline hid_t H5Aget_type(hid_t) { return -1; }
static inline ssize_t H5Iget_name(hid_t, char *, size_t) { return -1; }
static inline herr_t H5Fclose(hid_t) { return -1; }
static inline hid_t H5Fopen(const char *, unsigned, hid_t) { return -1; }
static inline hid_t H5Fcreate(const char *, unsigned, hid_t, hid_t) { return -1; }
static inline herr_t H5Fget_filesize(hid_t, hsize_t *s) { if (s) *s = 0; return -1; }
static inline herr_t H5Eset_auto1(H5E_auto1_t, void *) { return -1; }
static inline herr_t H5Eget_auto1(H5E_auto1_t *, void **) { return -1; }
static inline hid_t H5Dopen2(hid_t, const char *, hid_t) { return -1; }
static inline hid_t H5Dget_space(hid_t) { return -1; }
static inline hid_t H5Dget_type(hid_t) { return -1; }
static inline herr_t H5Dclose(hid_t) { return -1; }
static inline herr_t H5Dread(hid_t, hid_t, hid_t, hid_t, hid_t, void *) { return -1; }
static inline herr_t H5Dwrite(hid_t, hid_t, hid_t, hid_t, hid_t, const void *) { return -1; }
static inline htri_t H5Tequal(hid_t, hid_t) { return 0; }
static inline herr_t H5Tclose(hid_t) { return -1; }
static inline hid_t H5Tcopy(hid_t) { return -1; }
static inline herr_t H5Tset_size(hid_t, size_t) { return -1; }
static inline hid_t H5Tget_native_type(hid_t, H5T_direction_t) { return -1; }
static inline hid_t H5Pcreate(hid_t) { return -1; }
static inline herr_t H5Pset_cache(hid_t, int, size_t, size_t, double) { return -1; }
static inline herr_t H5Pget_cache(hid_t, int *, size_t *, size_t *, double *) { return -1; }
static inline htri_t H5Lexists(hid_t, const char *, hid_t) { return 0; }
#endif
