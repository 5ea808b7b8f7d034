/*
 * mkl.h -- the MKL types the reference's common.h (common.h:9) needs when its
 * hot path runs on the B200 library: the drop-in headers make no MKL call, so
 * only MKL_Complex16 and the integer types remain.  Put this directory before
 * any Intel MKL include directory (or drop MKL from the build entirely).
 */
#ifndef VIE_DROPIN_MKL_H
#define VIE_DROPIN_MKL_H
typedef struct { double real, imag; } MKL_Complex16;
typedef int MKL_INT;
typedef long MKL_LONG;
#endif
