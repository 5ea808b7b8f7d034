/*
 * mkl.h -- minimal stand-in for the ten Intel MKL entry points that the
 * reference VIE_FFT code calls (test infrastructure only; Intel MKL is not
 * installed on this image and cannot be installed).
 *
 * DFTI (3D double complex, in place, unnormalised):
 *   DftiCreateDescriptor / DftiCommitDescriptor / DftiComputeForward /
 *   DftiComputeBackward / DftiFreeDescriptor
 *   call sites: GreenFunction.h:132-139, fft.h:65-126, 154-218, 246-308, 334-396
 * CBLAS level 1 (double complex, MKL_INT = int under the LP64 interface the
 * reference links, README.md:37):
 *   cblas_zcopy, cblas_zscal, cblas_zaxpy, cblas_zdotc_sub, cblas_zdotu_sub
 *   call sites: CG_Iteration.h (all five Krylov drivers)
 *
 * The transforms are computed by oracle/vo_fft.c.  MKL's own rounding is not
 * reproducible here; the shim's transform agrees with numpy.fft to ~1e-15.
 */
#ifndef VIE_MKL_SHIM_H
#define VIE_MKL_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double real, imag; } MKL_Complex16;
typedef int MKL_INT;
typedef long MKL_LONG;

enum DFTI_CONFIG_VALUE { DFTI_SINGLE = 35, DFTI_DOUBLE = 36, DFTI_COMPLEX = 32, DFTI_REAL = 33 };

typedef struct vie_dfti_desc* DFTI_DESCRIPTOR_HANDLE;

MKL_LONG DftiCreateDescriptor(DFTI_DESCRIPTOR_HANDLE* h, enum DFTI_CONFIG_VALUE prec,
                              enum DFTI_CONFIG_VALUE domain, MKL_LONG dim, ...);
MKL_LONG DftiCommitDescriptor(DFTI_DESCRIPTOR_HANDLE h);
MKL_LONG DftiComputeForward(DFTI_DESCRIPTOR_HANDLE h, void* x);
MKL_LONG DftiComputeBackward(DFTI_DESCRIPTOR_HANDLE h, void* x);
MKL_LONG DftiFreeDescriptor(DFTI_DESCRIPTOR_HANDLE* h);

void cblas_zcopy(const MKL_INT n, const void* x, const MKL_INT incx, void* y, const MKL_INT incy);
void cblas_zscal(const MKL_INT n, const void* a, void* x, const MKL_INT incx);
void cblas_zaxpy(const MKL_INT n, const void* a, const void* x, const MKL_INT incx, void* y,
                 const MKL_INT incy);
void cblas_zdotc_sub(const MKL_INT n, const void* x, const MKL_INT incx, const void* y,
                     const MKL_INT incy, void* dotc);
void cblas_zdotu_sub(const MKL_INT n, const void* x, const MKL_INT incx, const void* y,
                     const MKL_INT incy, void* dotu);

#ifdef __cplusplus
}
#endif
#endif
