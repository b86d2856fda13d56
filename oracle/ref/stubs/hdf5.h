/*
 * Minimal HDF5 type/constant stub used ONLY to compile the reference's
 * unity build (pardiso/i3mg.c sources) for the CPU oracle.  The oracle
 * never calls the reference's loader()/saver() (pardiso/load3mg.c:724-1766),
 * which are the only users of these symbols; the functions below are
 * link-time stand-ins that report failure (-1) if ever reached.
 *
 * Test infrastructure only: nothing in the product links this header.
 */
#ifndef P2_HDF5_STUB_H
#define P2_HDF5_STUB_H

typedef long long hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;

#define H5P_DEFAULT 0
#define H5S_ALL 0
#define H5S_SELECT_SET 0
#define H5F_ACC_TRUNC 0
#define H5F_ACC_RDONLY 0
#define H5T_NATIVE_FLOAT 0
#define H5T_NATIVE_LONG 0
#define H5T_NATIVE_INT 0
#define H5T_NATIVE_DOUBLE 0
#define H5T_NATIVE_CHAR 0

static hid_t p2_h5_fail(void) { return -1; }
#define H5Fcreate(...) p2_h5_fail()
#define H5Fopen(...) p2_h5_fail()
#define H5Fclose(...) ((herr_t)p2_h5_fail())
#define H5Gcreate(...) p2_h5_fail()
#define H5Gopen(...) p2_h5_fail()
#define H5Gclose(...) ((herr_t)p2_h5_fail())
#define H5Screate_simple(...) p2_h5_fail()
#define H5Sclose(...) ((herr_t)p2_h5_fail())
#define H5Sselect_hyperslab(...) ((herr_t)p2_h5_fail())
#define H5Sget_simple_extent_npoints(...) p2_h5_fail()
#define H5Dcreate(...) p2_h5_fail()
#define H5Dopen(...) p2_h5_fail()
#define H5Dclose(...) ((herr_t)p2_h5_fail())
#define H5Dwrite(...) ((herr_t)p2_h5_fail())
#define H5Dread(...) ((herr_t)p2_h5_fail())
#define H5Dget_space(...) p2_h5_fail()
#define H5Acreate(...) p2_h5_fail()
#define H5Aopen_by_name(...) p2_h5_fail()
#define H5Awrite(...) ((herr_t)p2_h5_fail())
#define H5Aread(...) ((herr_t)p2_h5_fail())
#define H5Aclose(...) ((herr_t)p2_h5_fail())

#endif
