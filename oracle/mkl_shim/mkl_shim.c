/*
 * mkl_shim.c -- implementation of the MKL stand-in declared in mkl.h
 * (test infrastructure only).  Semantics follow the MKL reference manual for
 * the calls the VIE_FFT reference makes: a 3D DFTI_COMPLEX/DFTI_DOUBLE
 * descriptor with default (unit) forward and backward scales, in-place
 * placement, row-major dense strides; CBLAS zdotc = sum conj(x_i) y_i and
 * zdotu = sum x_i y_i.
 */
#include "mkl.h"
#include "../vo_fft.h"

#include <stdarg.h>
#include <stdlib.h>

struct vie_dfti_desc { int dim; long n[3]; };

MKL_LONG DftiCreateDescriptor(DFTI_DESCRIPTOR_HANDLE* h, enum DFTI_CONFIG_VALUE prec,
                              enum DFTI_CONFIG_VALUE domain, MKL_LONG dim, ...) {
    if (!h || prec != DFTI_DOUBLE || domain != DFTI_COMPLEX || dim < 1 || dim > 3) return 1;
    struct vie_dfti_desc* d = (struct vie_dfti_desc*)calloc(1, sizeof(*d));
    if (!d) return 1;
    va_list ap;
    va_start(ap, dim);
    if (dim == 1) {
        d->n[0] = va_arg(ap, MKL_LONG);
    } else {
        const MKL_LONG* l = va_arg(ap, const MKL_LONG*);
        for (int i = 0; i < dim; i++) d->n[i] = l[i];
    }
    va_end(ap);
    d->dim = (int)dim;
    *h = d;
    return 0;
}

MKL_LONG DftiCommitDescriptor(DFTI_DESCRIPTOR_HANDLE h) { return h ? 0 : 1; }

static MKL_LONG run(DFTI_DESCRIPTOR_HANDLE h, void* x, int sign) {
    if (!h || !x) return 1;
    long n0 = 1, n1 = 1, n2 = 1;
    if (h->dim == 1) n2 = h->n[0];
    else if (h->dim == 2) { n1 = h->n[0]; n2 = h->n[1]; }
    else { n0 = h->n[0]; n1 = h->n[1]; n2 = h->n[2]; }
    return vo_fft3d((vo_cplx*)x, (int)n0, (int)n1, (int)n2, sign) == 0 ? 0 : 1;
}

MKL_LONG DftiComputeForward(DFTI_DESCRIPTOR_HANDLE h, void* x) { return run(h, x, -1); }
MKL_LONG DftiComputeBackward(DFTI_DESCRIPTOR_HANDLE h, void* x) { return run(h, x, +1); }

MKL_LONG DftiFreeDescriptor(DFTI_DESCRIPTOR_HANDLE* h) {
    if (!h) return 1;
    free(*h);
    *h = NULL;
    return 0;
}

typedef struct { double re, im; } zc;

void cblas_zcopy(const MKL_INT n, const void* x, const MKL_INT incx, void* y, const MKL_INT incy) {
    const zc* a = (const zc*)x;
    zc* b = (zc*)y;
    for (MKL_INT i = 0; i < n; i++) b[(long)i * incy] = a[(long)i * incx];
}

void cblas_zscal(const MKL_INT n, const void* a, void* x, const MKL_INT incx) {
    const zc s = *(const zc*)a;
    zc* v = (zc*)x;
    for (MKL_INT i = 0; i < n; i++) {
        zc t = v[(long)i * incx];
        v[(long)i * incx].re = s.re * t.re - s.im * t.im;
        v[(long)i * incx].im = s.re * t.im + s.im * t.re;
    }
}

void cblas_zaxpy(const MKL_INT n, const void* a, const void* x, const MKL_INT incx, void* y,
                 const MKL_INT incy) {
    const zc s = *(const zc*)a;
    const zc* u = (const zc*)x;
    zc* v = (zc*)y;
    for (MKL_INT i = 0; i < n; i++) {
        zc t = u[(long)i * incx];
        v[(long)i * incy].re += s.re * t.re - s.im * t.im;
        v[(long)i * incy].im += s.re * t.im + s.im * t.re;
    }
}

static void dot(const MKL_INT n, const zc* x, MKL_INT incx, const zc* y, MKL_INT incy, int conj,
                zc* out) {
    double sr = 0.0, si = 0.0;
    for (MKL_INT i = 0; i < n; i++) {
        zc a = x[(long)i * incx], b = y[(long)i * incy];
        if (conj) a.im = -a.im;
        sr += a.re * b.re - a.im * b.im;
        si += a.re * b.im + a.im * b.re;
    }
    out->re = sr;
    out->im = si;
}

void cblas_zdotc_sub(const MKL_INT n, const void* x, const MKL_INT incx, const void* y,
                     const MKL_INT incy, void* dotc) {
    dot(n, (const zc*)x, incx, (const zc*)y, incy, 1, (zc*)dotc);
}

void cblas_zdotu_sub(const MKL_INT n, const void* x, const MKL_INT incx, const void* y,
                     const MKL_INT incy, void* dotu) {
    dot(n, (const zc*)x, incx, (const zc*)y, incy, 0, (zc*)dotu);
}
