// Oracle build shim: Fortran-to-C scalar types for the LAPACK/CBLAS
// declarations the reference sources include (src_util/clapack.h, cblas.h).
//
// Test infrastructure only. The reference's own copy declares `integer` as a
// 64-bit `long`, while the LAPACK in this image (OpenBLAS 0.3.15, LP64) takes
// 32-bit Fortran integers. Declaring `integer` as `int` here makes the
// reference's dstev_ call pass and receive 32-bit values, so `info` is exact.
#pragma once

typedef int integer;
typedef unsigned int uinteger;
typedef char *address;
typedef short int shortint;
typedef float f2c_real;
typedef double doublereal;
typedef struct { f2c_real r, i; } f2c_complex;
typedef struct { doublereal r, i; } doublecomplex;
typedef int logical;
typedef short int shortlogical;
typedef char logical1;
typedef char integer1;
typedef int ftnlen;
typedef int ftnint;
typedef int flag;

typedef logical (*L_fp)(...);
typedef int (*U_fp)(...);
typedef doublereal (*D_fp)(...);
typedef doublereal (*E_fp)(...);
typedef void (*C_fp)(...);
typedef void (*Z_fp)(...);
typedef int (*I_fp)(...);
typedef int (*S_fp)(...);
typedef f2c_real (*R_fp)(...);
typedef shortint (*J_fp)(...);
typedef void (*H_fp)(...);
typedef doublereal E_f;
