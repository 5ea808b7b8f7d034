/*
 * vo_fft.c -- CPU double-complex FFT for the oracle (test infrastructure only).
 * See vo_fft.h for the transform definition.  This is the stand-in for the
 * MKL DFTI 3D double-complex transform that the reference calls at
 * GreenFunction.h:131-139 and fft.h:64-126 (and in every other L_* function).
 */
#include "vo_fft.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define VO_MAXF 64

struct vo_plan1d {
    int n;
    int nf;
    int fac[VO_MAXF];
    vo_cplx* tw;   /* tw[t] = exp(-2 pi i t / n), t in [0, n) */
    int* perm;     /* natural index k -> storage position after DIF stages */
};

static int factorize(int n, int* fac) {
    int nf = 0;
    while (n % 4 == 0) { fac[nf++] = 4; n /= 4; }
    while (n % 2 == 0) { fac[nf++] = 2; n /= 2; }
    for (int p = 3; p * p <= n; p += 2)
        while (n % p == 0) { fac[nf++] = p; n /= p; }
    if (n > 1) fac[nf++] = n;
    return nf;
}

vo_plan1d* vo_plan1d_create(int n) {
    if (n < 1) return NULL;
    vo_plan1d* p = (vo_plan1d*)calloc(1, sizeof(vo_plan1d));
    if (!p) return NULL;
    p->n = n;
    p->nf = factorize(n, p->fac);
    p->tw = (vo_cplx*)malloc(sizeof(vo_cplx) * (size_t)n);
    p->perm = (int*)malloc(sizeof(int) * (size_t)n);
    if (!p->tw || !p->perm) { vo_plan1d_destroy(p); return NULL; }
    for (int t = 0; t < n; t++) {
        /* angle reduced in long double to keep the table accurate to ~1 ulp */
        long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)t / (long double)n;
        p->tw[t].re = (double)cosl(a);
        p->tw[t].im = (double)sinl(a);
    }
    /* DIF with radices R1..Rk (in plan order) leaves X[q1 + R1 q2 + R1 R2 q3 + ...]
       at position q1 (n/R1) + q2 (n/(R1 R2)) + ... + qk. */
    for (int k = 0; k < n; k++) {
        int rem = k, pos = 0, span = n;
        for (int s = 0; s < p->nf; s++) {
            int R = p->fac[s];
            int q = rem % R;
            rem /= R;
            span /= R;
            pos += q * span;
        }
        p->perm[k] = pos;
    }
    return p;
}

void vo_plan1d_destroy(vo_plan1d* p) {
    if (!p) return;
    free(p->tw);
    free(p->perm);
    free(p);
}

static inline vo_cplx cmul(vo_cplx a, vo_cplx b) {
    vo_cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
    return r;
}

/* twiddle exp(sign * 2 pi i t / n) from the forward table */
static inline vo_cplx twid(const vo_plan1d* p, long t, int sign) {
    vo_cplx w = p->tw[t % p->n];
    if (sign > 0) w.im = -w.im;
    return w;
}

void vo_fft1d(const vo_plan1d* p, vo_cplx* x, int sign) {
    const int n = p->n;
    if (n == 1) return;
    vo_cplx v[VO_MAXF > 64 ? VO_MAXF : 64];
    vo_cplx* vbig = NULL;
    vo_cplx* ybig = NULL;
    int L = n;
    for (int s = 0; s < p->nf; s++) {
        const int R = p->fac[s];
        const int m = L / R;
        const int stride_tw = n / L; /* W_L^e = W_n^(e * n / L) */
        vo_cplx* vv = v;
        vo_cplx* yy = NULL;
        if (R > 64) {
            vbig = (vo_cplx*)realloc(vbig, sizeof(vo_cplx) * (size_t)R);
            ybig = (vo_cplx*)realloc(ybig, sizeof(vo_cplx) * (size_t)R);
            vv = vbig;
            yy = ybig;
        }
        vo_cplx ysmall[64];
        if (!yy) yy = ysmall;
        for (int b = 0; b < n / L; b++) {
            vo_cplx* base = x + (size_t)b * L;
            for (int j = 0; j < m; j++) {
                for (int r = 0; r < R; r++) vv[r] = base[j + r * m];
                if (R == 2) {
                    yy[0].re = vv[0].re + vv[1].re; yy[0].im = vv[0].im + vv[1].im;
                    yy[1].re = vv[0].re - vv[1].re; yy[1].im = vv[0].im - vv[1].im;
                } else if (R == 4) {
                    vo_cplx a0 = {vv[0].re + vv[2].re, vv[0].im + vv[2].im};
                    vo_cplx a1 = {vv[0].re - vv[2].re, vv[0].im - vv[2].im};
                    vo_cplx b0 = {vv[1].re + vv[3].re, vv[1].im + vv[3].im};
                    vo_cplx b1 = {vv[1].re - vv[3].re, vv[1].im - vv[3].im};
                    /* multiply b1 by sign*i: forward (-i), backward (+i) */
                    vo_cplx jb1;
                    if (sign < 0) { jb1.re = b1.im; jb1.im = -b1.re; }
                    else { jb1.re = -b1.im; jb1.im = b1.re; }
                    yy[0].re = a0.re + b0.re; yy[0].im = a0.im + b0.im;
                    yy[2].re = a0.re - b0.re; yy[2].im = a0.im - b0.im;
                    yy[1].re = a1.re + jb1.re; yy[1].im = a1.im + jb1.im;
                    yy[3].re = a1.re - jb1.re; yy[3].im = a1.im - jb1.im;
                } else {
                    const int sR = n / R;
                    for (int q = 0; q < R; q++) {
                        double sr = 0.0, si = 0.0;
                        for (int r = 0; r < R; r++) {
                            vo_cplx w = twid(p, (long)((r * (long)q) % R) * sR, sign);
                            sr += vv[r].re * w.re - vv[r].im * w.im;
                            si += vv[r].re * w.im + vv[r].im * w.re;
                        }
                        yy[q].re = sr;
                        yy[q].im = si;
                    }
                }
                for (int q = 0; q < R; q++) {
                    vo_cplx y = yy[q];
                    if (j != 0 && q != 0) y = cmul(y, twid(p, (long)j * q * stride_tw, sign));
                    base[j + q * m] = y;
                }
            }
        }
        L = m;
    }
    free(vbig);
    free(ybig);
    /* digit-reversal gather into natural order */
    vo_cplx* tmp = (vo_cplx*)malloc(sizeof(vo_cplx) * (size_t)n);
    if (!tmp) abort();
    for (int k = 0; k < n; k++) tmp[k] = x[p->perm[k]];
    memcpy(x, tmp, sizeof(vo_cplx) * (size_t)n);
    free(tmp);
}

int vo_fft3d(vo_cplx* x, int n0, int n1, int n2, int sign) {
    enum { B = 16 };
    vo_plan1d* p0 = vo_plan1d_create(n0);
    vo_plan1d* p1 = vo_plan1d_create(n1);
    vo_plan1d* p2 = vo_plan1d_create(n2);
    int nmax = n0 > n1 ? n0 : n1;
    vo_cplx* buf = (vo_cplx*)malloc(sizeof(vo_cplx) * (size_t)B * (size_t)nmax);
    if (!p0 || !p1 || !p2 || !buf) {
        vo_plan1d_destroy(p0); vo_plan1d_destroy(p1); vo_plan1d_destroy(p2); free(buf);
        return -1;
    }
    const size_t s0 = (size_t)n1 * n2, s1 = (size_t)n2;
    /* axis 2: contiguous rows */
    for (size_t r = 0; r < (size_t)n0 * n1; r++) vo_fft1d(p2, x + r * n2, sign);
    /* axis 1: blocks of B adjacent columns gathered into rows */
    for (int i = 0; i < n0; i++) {
        for (int k0 = 0; k0 < n2; k0 += B) {
            int nb = (n2 - k0) < B ? (n2 - k0) : B;
            for (int j = 0; j < n1; j++)
                for (int t = 0; t < nb; t++) buf[(size_t)t * n1 + j] = x[i * s0 + j * s1 + k0 + t];
            for (int t = 0; t < nb; t++) vo_fft1d(p1, buf + (size_t)t * n1, sign);
            for (int j = 0; j < n1; j++)
                for (int t = 0; t < nb; t++) x[i * s0 + j * s1 + k0 + t] = buf[(size_t)t * n1 + j];
        }
    }
    /* axis 0 */
    for (int j = 0; j < n1; j++) {
        for (int k0 = 0; k0 < n2; k0 += B) {
            int nb = (n2 - k0) < B ? (n2 - k0) : B;
            for (int i = 0; i < n0; i++)
                for (int t = 0; t < nb; t++) buf[(size_t)t * n0 + i] = x[i * s0 + j * s1 + k0 + t];
            for (int t = 0; t < nb; t++) vo_fft1d(p0, buf + (size_t)t * n0, sign);
            for (int i = 0; i < n0; i++)
                for (int t = 0; t < nb; t++) x[i * s0 + j * s1 + k0 + t] = buf[(size_t)t * n0 + i];
        }
    }
    free(buf);
    vo_plan1d_destroy(p0); vo_plan1d_destroy(p1); vo_plan1d_destroy(p2);
    return 0;
}
