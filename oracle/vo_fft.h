/*
 * vo_fft.h -- CPU double-complex FFT used ONLY as test infrastructure.
 *
 * This file is part of the oracle (the CPU checker of the CUDA path). It is
 * never linked into the product library. Two things use it:
 *   1. the MKL shim (oracle/mkl_shim/), so that the reference's unchanged
 *      DFTI call sites (GreenFunction.h:131-139, fft.h:64-126 and the other
 *      L_* functions) compile and run here without Intel MKL;
 *   2. the C restatement of the hot path (oracle/vie_oracle.c).
 *
 * Definition (the MKL DFTI default for a DFTI_COMPLEX/DFTI_DOUBLE descriptor
 * with no scale set): forward X[k] = sum_n x[n] exp(-2 pi i k n / N),
 * backward x[n] = sum_k X[k] exp(+2 pi i k n / N), both unnormalised,
 * multi-dimensional transforms row-major (last index fastest).
 *
 * Algorithm: in-place mixed-radix decimation-in-frequency with radices
 * 4, 2, 3, 5 and a generic O(p^2) butterfly for any other prime factor,
 * followed by a digit-reversal gather.  Twiddles are tabulated once per
 * length in double precision from sin/cos of exactly reduced angles.
 */
#ifndef VO_FFT_H
#define VO_FFT_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double re, im; } vo_cplx;

typedef struct vo_plan1d vo_plan1d;

/* Plan for a 1D transform of length n (any n >= 1). NULL on allocation failure. */
vo_plan1d* vo_plan1d_create(int n);
void vo_plan1d_destroy(vo_plan1d* p);

/* In-place 1D transform of x (contiguous). sign = -1 forward, +1 backward. */
void vo_fft1d(const vo_plan1d* p, vo_cplx* x, int sign);

/* In-place 3D transform of a row-major (n0, n1, n2) array. Returns 0 on success. */
int vo_fft3d(vo_cplx* x, int n0, int n1, int n2, int sign);

#ifdef __cplusplus
}
#endif
#endif
