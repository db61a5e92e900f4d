/*
 * TEST INFRASTRUCTURE ONLY — an in-memory stand-in for the subset of the
 * HDF5 C API that the reference program calls.  libhdf5 is not installed in
 * this image, so the reference's inverse-p path (which passes the angular
 * up-weight histograms between stages through HDF5 files) is linked against
 * this header and hdf5_stub.cpp when it is built as the parity oracle.
 *
 * Only the calls made by the reference are provided (src/hist.cpp:115-220,
 * src/io.cpp:418-593, src/io.cpp:654-720).  "Files" live in a process-wide
 * map keyed by file name; nothing touches the disk.  Datasets and attributes
 * keep their stored element type and are converted on read, as libhdf5 does
 * (the reference writes histogram min/max/base as float attributes and reads
 * them back as double, src/hist.cpp:141-151 vs :189-191).
 */
#pragma once
#include <cstdint>
#include <cstddef>

typedef int64_t hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;
typedef long long hssize_t;

#define H5P_DEFAULT ((hid_t)0)
#define H5S_ALL ((hid_t)0)
#define H5F_ACC_RDONLY 0u
#define H5F_ACC_TRUNC 2u

typedef enum { H5S_SCALAR = 0, H5S_SIMPLE = 1 } H5S_class_t;
typedef enum { H5T_ORDER_LE = 0, H5T_ORDER_BE = 1 } H5T_order_t;

extern const hid_t H5T_NATIVE_DOUBLE;
extern const hid_t H5T_NATIVE_FLOAT;
extern const hid_t H5T_NATIVE_INT;
extern const hid_t H5T_NATIVE_LONG;
extern const hid_t H5T_C_S1;

hid_t H5Fopen(const char *name, unsigned flags, hid_t fapl);
hid_t H5Fcreate(const char *name, unsigned flags, hid_t fcpl, hid_t fapl);
herr_t H5Fclose(hid_t file);

hid_t H5Gopen(hid_t loc, const char *name, hid_t gapl);
hid_t H5Gcreate2(hid_t loc, const char *name, hid_t lcpl, hid_t gcpl, hid_t gapl);
herr_t H5Gclose(hid_t group);

hid_t H5Dopen2(hid_t loc, const char *name, hid_t dapl);
hid_t H5Dcreate2(hid_t loc, const char *name, hid_t type, hid_t space, hid_t lcpl, hid_t dcpl, hid_t dapl);
herr_t H5Dread(hid_t dset, hid_t mem_type, hid_t mem_space, hid_t file_space, hid_t plist, void *buf);
herr_t H5Dwrite(hid_t dset, hid_t mem_type, hid_t mem_space, hid_t file_space, hid_t plist, const void *buf);
hid_t H5Dget_space(hid_t dset);
herr_t H5Dclose(hid_t dset);

hid_t H5Screate(H5S_class_t type);
hid_t H5Screate_simple(int rank, const hsize_t *dims, const hsize_t *maxdims);
hssize_t H5Sget_simple_extent_npoints(hid_t space);
herr_t H5Sclose(hid_t space);

hid_t H5Aopen(hid_t obj, const char *name, hid_t aapl);
hid_t H5Acreate2(hid_t loc, const char *name, hid_t type, hid_t space, hid_t acpl, hid_t aapl);
herr_t H5Aread(hid_t attr, hid_t mem_type, void *buf);
herr_t H5Awrite(hid_t attr, hid_t mem_type, const void *buf);
herr_t H5Aclose(hid_t attr);

hid_t H5Tcopy(hid_t type);
herr_t H5Tset_order(hid_t type, H5T_order_t order);

/* Harness helpers (not HDF5 API): drop every in-memory file. */
void h5stub_reset(void);
