/*
 * vie_oracle.c -- CPU restatement of the VIE_FFT hot path (see vie_oracle.h).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA library, never the
 * product.  It restates, in plain C and in the reference's own operation
 * order, the functions of GreenFunction.h, fft.h, CG_Iteration.h and the
 * absorption / extinction sums of NearFar.h.  Each function cites the lines
 * it follows.  The 3D transforms come from vo_fft.c (the same unnormalised
 * DFT definition as the reference's MKL DFTI calls).
 */
#include "vie_oracle.h"
#include "vo_fft.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* constants of common.h:15-19 */
static const double PI = 3.1415926535897932384626433832795;
#define Z0 (120 * PI)
static const double EPSC = 1.0e-7;

typedef vo_cplx cx;

static inline cx mk(double r, double i) { cx c = {r, i}; return c; }
static inline cx add(cx a, cx b) { return mk(a.re + b.re, a.im + b.im); }
static inline cx sub(cx a, cx b) { return mk(a.re - b.re, a.im - b.im); }
static inline cx mul(cx a, cx b) { return mk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
static inline cx scl(cx a, double s) { return mk(a.re * s, a.im * s); }
static inline cx cj(cx a) { return mk(a.re, -a.im); }
static inline cx cdiv(cx a, cx b) {
    /* C99 complex division: the same library routine as std::complex<double>
       operator/ in the reference, so the quotients agree bit for bit */
    double complex r = CMPLX(a.re, a.im) / CMPLX(b.re, b.im);
    return mk(creal(r), cimag(r));
}
static inline cx cexpi(double t) { return mk(cos(t), sin(t)); } /* exp(i t) */

/* ------------------------------------------------------------------------ */
/* Green_Function_Compute, GreenFunction.h:8-141                            */
/* ------------------------------------------------------------------------ */
int vo_green(const vo_grid* g, double* out) {
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const int Lx = 2 * nx, Ly = 2 * ny, Lz = 2 * nz;
    const double dV = g->dx * g->dy * g->dz;                      /* :23 */
    const double D = 2 * pow(dV / (4.0 / 3.0 * PI), 1.0 / 3.0);   /* :24 */
    const double p = 0.5 * g->k0 * D;                             /* :25 */
    const double k0 = g->k0;
    /* octant values on offsets [0..nx] x [0..ny] x [0..nz] (:53-88) */
    const size_t ox = (size_t)(ny + 1) * (nz + 1), oy = (size_t)(nz + 1);
    cx* oct = (cx*)malloc(sizeof(cx) * (size_t)(nx + 1) * ox);
    if (!oct) return 1;
    /* sinh(-ip)/(-ip) - cosh(-ip) = sin(p)/p - cos(p), a real number */
    const double shape = sin(p) / p - cos(p);
    for (int i = 0; i <= nx; i++)
        for (int j = 0; j <= ny; j++)
            for (int k = 0; k <= nz; k++) {
                cx v;
                if (i + j + k != 0) {
                    double r = sqrt(pow(i * g->dx, 2.0) + pow(j * g->dy, 2.0) + pow(k * g->dz, 2.0));
                    cx e = cexpi(-k0 * r);
                    double den = 1.0 / 3.0 * PI * k0 * k0 * pow(D, 2.0) * r; /* :68 */
                    v = mk(e.re * shape / den * dV, e.im * shape / den * dV);
                } else {
                    /* singular self cell: ((1 + i p) e^{-i p} - 1) / (pi k0^2 D^3 / 6) * dV (:77-84) */
                    cx t = sub(mul(mk(1.0, p), cexpi(-p)), mk(1.0, 0.0));
                    double den = 1.0 / 6.0 * PI * k0 * k0 * pow(D, 3.0);
                    v = mk(t.re / den * dV, t.im / den * dV);
                }
                oct[i * ox + j * oy + k] = v;
            }
    /* even periodic extension: index i >= n maps to 2n - i (:92-129) */
    cx* G = (cx*)out;
    for (int i = 0; i < Lx; i++) {
        int ii = i >= nx ? Lx - i : i;
        for (int j = 0; j < Ly; j++) {
            int jj = j >= ny ? Ly - j : j;
            for (int k = 0; k < Lz; k++) {
                int kk = k >= nz ? Lz - k : k;
                G[((size_t)i * Ly + j) * Lz + k] = oct[ii * ox + jj * oy + kk];
            }
        }
    }
    free(oct);
    /* unnormalised forward transform (:131-139) */
    return vo_fft3d(G, Lx, Ly, Lz, -1) == 0 ? 0 : 2;
}

/* ------------------------------------------------------------------------ */
/* Incident_Wave, GreenFunction.h:144-248                                   */
/* ------------------------------------------------------------------------ */
/* edge integral of exp(-i k s) over a cell of length d, times the point phase,
   in the reference's complex arithmetic (GreenFunction.h:182-194) */
static cx edge_phase(double phase, double kk, double d) {
    double complex V1 = CMPLX(0.0, -phase);
    double complex V4;
    if (fabs(kk) < EPSC) {
        V4 = cexp(V1) * d;                                  /* :187-190 */
    } else {
        double complex V2 = CMPLX(0.0, -(kk * d / 2.0));
        double complex V3 = CMPLX(0.0, (kk * d / 2.0));
        V4 = cexp(V1) * (cexp(V2) - cexp(V3)) / CMPLX(0.0, -kk);   /* :193 */
    }
    return mk(creal(V4), cimag(V4));
}

int vo_incident(const vo_grid* g, double theta, double phi, double psi, double* e) {
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const size_t a = (size_t)nx * ny * nz;
    const double th = PI * theta / 180.0, ph = PI * phi / 180.0, ps = PI * psi / 180.0;
    const double kx = g->k0 * sin(th) * cos(ph);   /* :162-164 */
    const double ky = g->k0 * sin(th) * sin(ph);
    const double kz = g->k0 * cos(th);
    const double px = cos(th) * cos(ph) * cos(ps) - sin(ph) * sin(ps);  /* :196-199 */
    const double py = cos(th) * sin(ph) * cos(ps) + cos(ph) * sin(ps);  /* :219-222 */
    cx* ex = (cx*)e;
    cx* ey = ex + a;
    cx* ez = ey + a;
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                size_t v = ((size_t)i * ny + j) * nz + k;
                double xm, ym, zm;
                xm = (i + 1) * g->dx; ym = (j + 0.5) * g->dy; zm = (k + 0.5) * g->dz;
                ex[v] = scl(edge_phase(kx * xm + ky * ym + kz * zm, kx, g->dx), px);
                xm = (i + 0.5) * g->dx; ym = (j + 1) * g->dy; zm = (k + 0.5) * g->dz;
                ey[v] = scl(edge_phase(kx * xm + ky * ym + kz * zm, ky, g->dy), py);
                xm = (i + 0.5) * g->dx; ym = (j + 0.5) * g->dy; zm = (k + 1) * g->dz;
                /* -real(V4)*sin(theta)*cos(psi), evaluated left to right as :243-244 */
                cx vz = edge_phase(kx * xm + ky * ym + kz * zm, kz, g->dz);
                ez[v] = mk(-vz.re * sin(th) * cos(ps), -vz.im * sin(th) * cos(ps));
            }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Operator: Current_Expansion (CG_Iteration.h:50-83), L_DC_Dq (fft.h:41-127),
   L_Dq (fft.h:224-309), L??_DO (fft.h:405-624), their _Conjugate twins, and
   Current_Reset (fft.h:13-35), assembled like X/Y/Z_FFT (CG_Iteration.h:86-173). */
/* ------------------------------------------------------------------------ */
typedef struct {
    const vo_grid* g;
    const cx* green;
    const cx* eps;
    const unsigned char* flags;
    int L[3];
    double d[3];
    double* cs[3]; /* cos(2 pi k / L_a) */
    double* sn[3]; /* sin(2 pi k / L_a) */
    cx* tmp;       /* (2N)^3 scratch, Temp_Current */
} op_ctx;

static int op_init(op_ctx* o, const vo_grid* g, const double* green, const double* eps,
                   const unsigned char* flags) {
    memset(o, 0, sizeof(*o));
    o->g = g;
    o->green = (const cx*)green;
    o->eps = (const cx*)eps;
    o->flags = flags;
    o->L[0] = 2 * g->nx; o->L[1] = 2 * g->ny; o->L[2] = 2 * g->nz;
    o->d[0] = g->dx; o->d[1] = g->dy; o->d[2] = g->dz;
    for (int ax = 0; ax < 3; ax++) {
        o->cs[ax] = (double*)malloc(sizeof(double) * o->L[ax]);
        o->sn[ax] = (double*)malloc(sizeof(double) * o->L[ax]);
        if (!o->cs[ax] || !o->sn[ax]) return 1;
        for (int k = 0; k < o->L[ax]; k++) {
            /* same argument as fft.h:95-99: 2*PI*index/double(L) */
            o->cs[ax][k] = cos(2 * PI * k / (double)o->L[ax]);
            o->sn[ax][k] = sin(2 * PI * k / (double)o->L[ax]);
        }
    }
    o->tmp = (cx*)malloc(sizeof(cx) * (size_t)o->L[0] * o->L[1] * o->L[2]);
    return o->tmp ? 0 : 1;
}

static void op_free(op_ctx* o) {
    for (int ax = 0; ax < 3; ax++) { free(o->cs[ax]); free(o->sn[ax]); }
    free(o->tmp);
}

/* Current_Expansion: zero (2N)^3, copy the valid block of component s
   (Jx: i < nx-1; Jy: j < ny-1; Jz: k < nz-1). */
static void expand(op_ctx* o, const cx* J, int s) {
    const int nx = o->g->nx, ny = o->g->ny, nz = o->g->nz;
    const int Ly = o->L[1], Lz = o->L[2];
    memset(o->tmp, 0, sizeof(cx) * (size_t)o->L[0] * Ly * Lz);
    int lim[3] = {nx, ny, nz};
    lim[s] -= 1;
    for (int i = 0; i < lim[0]; i++)
        for (int j = 0; j < lim[1]; j++)
            for (int k = 0; k < lim[2]; k++)
                o->tmp[((size_t)i * Ly + j) * Lz + k] = J[((size_t)i * ny + j) * nz + k];
}

/* spectral multiply of one block: self (src == fld) or cross */
static void spectral(op_ctx* o, int src, int fld, int conj) {
    const double k0 = o->g->k0;
    const int Lx = o->L[0], Ly = o->L[1], Lz = o->L[2];
    const double d_src = o->d[src], d_fld = o->d[fld];
    cx V5, V6;
    if (src == fld) {
        /* fft.h:76-77 (forward), :167-168 (conjugate) */
        double s = conj ? -1.0 : 1.0;
        V5 = mk(0, s * k0 * Z0 * d_src / Lx / Ly / Lz);
        V6 = mk(0, s * Z0 / k0 / d_src / Lx / Ly / Lz);
    } else {
        /* fft.h:256 uses delta of the source; :344 (conjugate) delta of the field */
        V5 = conj ? mk(0, -Z0 / k0 / d_fld / Lx / Ly / Lz) : mk(0, Z0 / k0 / d_src / Lx / Ly / Lz);
        V6 = mk(0, 0);
    }
    for (int i = 0; i < Lx; i++)
        for (int j = 0; j < Ly; j++)
            for (int k = 0; k < Lz; k++) {
                size_t v = ((size_t)i * Ly + j) * Lz + k;
                int idx[3] = {i, j, k};
                cx V1 = o->tmp[v];
                cx V2 = conj ? cj(o->green[v]) : o->green[v];
                double cs = o->cs[src][idx[src]], sn = o->sn[src][idx[src]];
                double cf = o->cs[fld][idx[fld]], sf = o->sn[fld][idx[fld]];
                cx r;
                if (src == fld) {
                    /* V3 = 1 - e^{-i theta}, V4 = e^{i theta} - 1 (fft.h:95-99); conjugated in :186-190 */
                    cx V3 = conj ? mk(1.0 - cs, -sn) : mk(1.0 - cs, sn);
                    cx V4 = conj ? mk(cs - 1.0, -sn) : mk(cs - 1.0, sn);
                    r = mul(mul(V1, V2), add(V5, mul(mul(V6, V3), V4)));   /* :100 */
                } else if (!conj) {
                    cx V3 = mk(1.0 - cs, sn);       /* source, fft.h:276-277 */
                    cx V4 = mk(cf - 1.0, sf);       /* field,  fft.h:279-280 */
                    r = mul(mul(mul(mul(V5, V1), V2), V3), V4);            /* :281 */
                } else {
                    cx V3 = mk(1.0 - cf, -sf);      /* field,  fft.h:365-366 */
                    cx V4 = mk(cs - 1.0, -sn);      /* source, fft.h:368-369 */
                    r = mul(mul(mul(mul(V5, V1), V2), V3), V4);            /* :370 */
                }
                o->tmp[v] = r;
            }
}

/* FFT block: forward transform of tmp, multiply, backward, add the
   (nx, ny, nz) corner to F (fft.h:113-123). */
static int fft_block(op_ctx* o, cx* F, int src, int fld, int conj) {
    const int nx = o->g->nx, ny = o->g->ny, nz = o->g->nz;
    const int Ly = o->L[1], Lz = o->L[2];
    if (vo_fft3d(o->tmp, o->L[0], Ly, Lz, -1)) return 1;
    spectral(o, src, fld, conj);
    if (vo_fft3d(o->tmp, o->L[0], Ly, Lz, +1)) return 1;
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                size_t v = ((size_t)i * ny + j) * nz + k;
                F[v] = add(F[v], o->tmp[((size_t)i * Ly + j) * Lz + k]);
            }
    return 0;
}

/* L??_DO: F += -i d Z0 / (2 k0) (1/(eps_b - 1) + 1/(eps_a - 1)) J on the valid
   block of component f, reading the expanded current (fft.h:405-438 etc.). */
static void diag_term(op_ctx* o, cx* F, int f, int conj) {
    const int nx = o->g->nx, ny = o->g->ny, nz = o->g->nz;
    const int Ly = o->L[1], Lz = o->L[2];
    const double k0 = o->g->k0;
    cx V4 = conj ? mk(0.0, o->d[f] / 2.0 * Z0 / k0) : mk(0.0, -o->d[f] / 2.0 * Z0 / k0);
    cx one = mk(1.0, 0.0);
    int lim[3] = {nx, ny, nz};
    lim[f] -= 1;
    int step[3] = {ny * nz, nz, 1};
    for (int i = 0; i < lim[0]; i++)
        for (int j = 0; j < lim[1]; j++)
            for (int k = 0; k < lim[2]; k++) {
                size_t v = ((size_t)i * ny + j) * nz + k;
                cx ea = o->eps[v + step[f]], eb = o->eps[v];
                cx V2 = conj ? mk(ea.re - 1.0, -ea.im) : mk(ea.re - 1.0, ea.im);
                cx V3 = conj ? mk(eb.re - 1.0, -eb.im) : mk(eb.re - 1.0, eb.im);
                cx V1 = o->tmp[((size_t)i * Ly + j) * Lz + k];
                V1 = mul(mul(V4, add(cdiv(one, V2), cdiv(one, V3))), V1);
                F[v] = add(F[v], V1);
            }
}

static int apply_op(op_ctx* o, const cx* in, cx* out, int conj) {
    const size_t a = (size_t)o->g->nx * o->g->ny * o->g->nz;
    /* source order of X_FFT/Y_FFT/Z_FFT: self first, then the other two ascending */
    static const int order[3][3] = {{0, 1, 2}, {1, 0, 2}, {2, 0, 1}};
    for (int f = 0; f < 3; f++) {
        cx* F = out + f * a;
        memset(F, 0, sizeof(cx) * a);
        for (int t = 0; t < 3; t++) {
            int s = order[f][t];
            expand(o, in + s * a, s);
            if (t == 0) diag_term(o, F, f, conj);
            if (fft_block(o, F, s, f, conj)) return 1;
        }
        const unsigned char* fl = o->flags + f * a;
        for (size_t v = 0; v < a; v++) F[v] = scl(F[v], (double)fl[v]);   /* Current_Reset */
    }
    return 0;
}

int vo_matvec(const vo_grid* g, const double* green, const double* eps,
              const unsigned char* flags, const double* in, double* out, int conj) {
    op_ctx o;
    if (op_init(&o, g, green, eps, flags)) { op_free(&o); return 1; }
    int rc = apply_op(&o, (const cx*)in, (cx*)out, conj);
    op_free(&o);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* Krylov drivers, CG_Iteration.h:176-1362                                   */
/* ------------------------------------------------------------------------ */
typedef struct { cx* c; } vec3; /* 3*a complex */

static cx dotc3(const cx* x, const cx* y, size_t a) {
    /* three zdotc_sub calls summed x + y + z (e.g. CG_Iteration.h:573-577) */
    cx tot = mk(0, 0);
    for (int c = 0; c < 3; c++) {
        double sr = 0.0, si = 0.0;
        for (size_t i = 0; i < a; i++) {
            cx u = x[c * a + i], w = y[c * a + i];
            sr += u.re * w.re + u.im * w.im;
            si += u.re * w.im - u.im * w.re;
        }
        tot.re += sr; tot.im += si;
    }
    return tot;
}

static cx dotu3(const cx* x, const cx* y, size_t a) {
    cx tot = mk(0, 0);
    for (int c = 0; c < 3; c++) {
        double sr = 0.0, si = 0.0;
        for (size_t i = 0; i < a; i++) {
            cx u = x[c * a + i], w = y[c * a + i];
            sr += u.re * w.re - u.im * w.im;
            si += u.re * w.im + u.im * w.re;
        }
        tot.re += sr; tot.im += si;
    }
    return tot;
}

static void axpy(cx al, const cx* x, cx* y, size_t n) {
    for (size_t i = 0; i < n; i++) y[i] = add(y[i], mul(al, x[i]));
}
static void scal(cx al, cx* x, size_t n) {
    for (size_t i = 0; i < n; i++) x[i] = mul(al, x[i]);
}

int vo_solve(const vo_grid* g, const double* green, const double* eps,
             const unsigned char* flags, const double* einc, int solver, double thr,
             int maxit, double* xout, int* steps_out, double* err_out) {
    const size_t a = (size_t)g->nx * g->ny * g->nz;
    const size_t n = 3 * a;
    if (maxit <= 0) maxit = (int)a; /* loop bound m < Total_inc */
    op_ctx o;
    if (op_init(&o, g, green, eps, flags)) { op_free(&o); return 1; }
    cx* b = (cx*)malloc(sizeof(cx) * n);
    cx* x = (cx*)xout;
    cx* r = (cx*)calloc(n, sizeof(cx));
    cx* p = (cx*)calloc(n, sizeof(cx));
    cx* q = (cx*)calloc(n, sizeof(cx));
    cx* Ap = (cx*)calloc(n, sizeof(cx));
    cx* Aq = (cx*)calloc(n, sizeof(cx));
    cx* rc = (cx*)calloc(n, sizeof(cx));
    cx* pc = (cx*)calloc(n, sizeof(cx));
    cx* qc = (cx*)calloc(n, sizeof(cx));
    int rcode = 0, steps = maxit;
    double Error = -1.0;
    if (!b || !r || !p || !q || !Ap || !Aq || !rc || !pc || !qc) { rcode = 1; goto done; }
    memcpy(b, einc, sizeof(cx) * n);
    for (size_t i = 0; i < n; i++) b[i] = scl(b[i], (double)flags[i]);   /* E_inc reset */
    memset(x, 0, sizeof(cx) * n);

    if (solver == 3) {
        /* BICGSTAB_FFT, CG_Iteration.h:531-776 */
        memcpy(r, b, sizeof(cx) * n);
        cx bnrm2 = dotc3(b, b, a);
        cx alpha = mk(0, 0), omega = mk(1, 0), rho, rho_1 = mk(0, 0);
        for (int m = 0; m < maxit; m++) {
            rho = dotc3(b, r, a);                                   /* :594-598 */
            if (m > 0) {
                cx beta = mul(cdiv(rho, rho_1), cdiv(alpha, omega)); /* :603-609 */
                axpy(mk(-omega.re, -omega.im), Ap, p, n);           /* :612-616 */
                scal(beta, p, n);                                   /* :618-620 */
                axpy(mk(1, 0), r, p, n);                            /* :622-626 */
            } else {
                memcpy(p, r, sizeof(cx) * n);
            }
            if (apply_op(&o, p, Ap, 0)) { rcode = 1; goto done; }  /* :639-649 */
            alpha = cdiv(rho, dotc3(b, Ap, a));                     /* :652-662 */
            memcpy(q, r, sizeof(cx) * n);                           /* :665-672 */
            axpy(mk(-alpha.re, -alpha.im), Ap, q, n);
            if (apply_op(&o, q, Aq, 0)) { rcode = 1; goto done; }  /* :677-687 */
            omega = cdiv(dotc3(Aq, q, a), dotc3(Aq, Aq, a));        /* :690-706 */
            axpy(alpha, p, x, n);                                   /* :709-714 */
            axpy(omega, q, x, n);
            memcpy(r, q, sizeof(cx) * n);                           /* :717-724 */
            axpy(mk(-omega.re, -omega.im), Aq, r, n);
            Error = sqrt(dotc3(r, r, a).re / bnrm2.re);             /* :727-734 */
            if (Error < thr) { steps = m; break; }
            rho_1 = rho;
        }
    } else if (solver == 4) {
        /* CORS_FFT, CG_Iteration.h:780-1073 */
        memcpy(r, b, sizeof(cx) * n);
        cx bnrm2 = dotc3(b, b, a);
        cx alpha = mk(0, 0), rho, rho_1 = mk(0, 0);
        for (int m = 0; m < maxit; m++) {
            if (apply_op(&o, r, Ap, 0)) { rcode = 1; goto done; }  /* :853-863 */
            rho = dotc3(b, Ap, a);                                  /* :865-869 */
            if (m > 0) {
                cx beta = cdiv(rho, rho_1);                         /* :874-878 */
                memcpy(p, r, sizeof(cx) * n);                       /* :883-888 */
                axpy(beta, pc, p, n);
                memcpy(qc, Ap, sizeof(cx) * n);                     /* :891-896 */
                axpy(beta, rc, qc, n);
                scal(beta, q, n);                                   /* :899-915 */
                axpy(mk(1, 0), rc, q, n);
                scal(beta, q, n);
                axpy(mk(1, 0), qc, q, n);
            } else {
                memcpy(p, r, sizeof(cx) * n);                       /* :920-932 */
                memcpy(qc, Ap, sizeof(cx) * n);
                memcpy(q, Ap, sizeof(cx) * n);
            }
            if (apply_op(&o, q, Aq, 0)) { rcode = 1; goto done; }  /* :938-948 */
            alpha = cdiv(rho, dotc3(b, Aq, a));                     /* :951-962 */
            cx na = mk(-alpha.re, -alpha.im);
            memcpy(pc, p, sizeof(cx) * n);                          /* :965-972 */
            axpy(na, q, pc, n);
            memcpy(rc, qc, sizeof(cx) * n);                         /* :975-981 */
            axpy(na, Aq, rc, n);
            axpy(mk(2 * alpha.re, 2 * alpha.im), p, x, n);          /* :984-988 */
            cx a2 = mul(mul(alpha, alpha), mk(-1.0, 0.0));          /* :990-997 */
            axpy(a2, q, x, n);
            axpy(mk(-2.0 * alpha.re, -2.0 * alpha.im), qc, r, n);   /* :1000-1004 */
            axpy(mul(alpha, alpha), Aq, r, n);                      /* :1006-1012 */
            Error = sqrt(dotc3(r, r, a).re / bnrm2.re);             /* :1015-1022 */
            if (Error < thr) { steps = m; break; }
            rho_1 = rho;
        }
    } else if (solver == 5) {
        /* BICORSTAB_FFT, CG_Iteration.h:1076-1362 */
        memcpy(r, b, sizeof(cx) * n);
        cx bnrm2 = dotc3(b, b, a);
        cx alpha = mk(0, 0), omega = mk(0, 0), rho, rho_1 = mk(0, 0);
        for (int m = 0; m < maxit; m++) {
            if (apply_op(&o, r, Ap, 0)) { rcode = 1; goto done; }  /* :1145-1155 */
            rho = dotc3(b, Ap, a);                                  /* :1158-1162 */
            if (m > 0) {
                cx beta = mul(cdiv(rho, rho_1), cdiv(alpha, omega)); /* :1167-1173 */
                cx no = mk(-omega.re, -omega.im);
                axpy(no, q, p, n);                                  /* :1176-1190 */
                scal(beta, p, n);
                axpy(mk(1, 0), r, p, n);
                axpy(no, Aq, q, n);                                 /* :1193-1207 */
                scal(beta, q, n);
                axpy(mk(1, 0), Ap, q, n);
            } else {
                memcpy(p, r, sizeof(cx) * n);                       /* :1212-1218 */
                memcpy(q, Ap, sizeof(cx) * n);
            }
            if (apply_op(&o, q, Aq, 0)) { rcode = 1; goto done; }  /* :1224-1234 */
            alpha = cdiv(rho, dotc3(b, Aq, a));                     /* :1237-1248 */
            cx na = mk(-alpha.re, -alpha.im);
            memcpy(pc, r, sizeof(cx) * n);                          /* :1251-1258 */
            axpy(na, q, pc, n);
            memcpy(qc, Ap, sizeof(cx) * n);                         /* :1261-1268 */
            axpy(na, Aq, qc, n);
            omega = cdiv(dotc3(qc, pc, a), dotc3(qc, qc, a));       /* :1271-1287 */
            axpy(alpha, p, x, n);                                   /* :1290-1295 */
            axpy(omega, pc, x, n);
            memcpy(r, pc, sizeof(cx) * n);                          /* :1298-1305 */
            axpy(mk(-omega.re, -omega.im), qc, r, n);
            Error = sqrt(dotc3(r, r, a).re / bnrm2.re);             /* :1308-1315 */
            if (Error < thr) { steps = m; break; }
            rho_1 = rho;
        }
    } else if (solver == 1) {
        /* CG_FFT (CGNR), CG_Iteration.h:176-357 */
        memcpy(r, b, sizeof(cx) * n);
        scal(mk(-1.0, 0.0), r, n);                                  /* :208-216 */
        if (apply_op(&o, b, p, 1)) { rcode = 1; goto done; }       /* :219-229 */
        double v3 = dotc3(p, p, a).re;                              /* :234-237 */
        double vx = dotc3(b, b, a).re;                              /* :239-242 */
        for (int m = 0; m < maxit; m++) {
            double v1 = v3;
            if (apply_op(&o, p, Ap, 0)) { rcode = 1; goto done; }  /* :253-263 */
            double v2 = dotc3(Ap, Ap, a).re;                        /* :265-268 */
            double alpha = v1 / v2;                                 /* :271 */
            axpy(mk(alpha, 0.0), p, x, n);                          /* :273-277 */
            axpy(mk(alpha, 0.0), Ap, r, n);                         /* :279-281 */
            double v4 = dotc3(r, r, a).re;                          /* :283-286 */
            if (apply_op(&o, r, q, 1)) { rcode = 1; goto done; }   /* :291-301 */
            v3 = dotc3(q, q, a).re;                                 /* :303-306 */
            double beta = v3 / v1;                                  /* :309 */
            scal(mk(beta, 0.0), p, n);                              /* :311-320 */
            axpy(mk(-1.0, 0.0), q, p, n);
            Error = v4 / vx;                                        /* :323 */
            if (Error < thr) { steps = m; break; }
        }
    } else if (solver == 2) {
        /* BICG_FFT (complex symmetric), CG_Iteration.h:360-528 */
        memcpy(r, b, sizeof(cx) * n);
        cx v1 = dotu3(r, r, a);                                     /* :402-406 */
        memcpy(p, r, sizeof(cx) * n);                               /* :413-424 */
        scal(cdiv(mk(1, 0), v1), p, n);
        cx vx = v1;
        for (int m = 0; m < maxit; m++) {
            if (apply_op(&o, p, Ap, 0)) { rcode = 1; goto done; }  /* :437-447 */
            v1 = dotu3(Ap, p, a);                                   /* :449-453 */
            cx alpha = cdiv(mk(1, 0), v1);                          /* :456-460 */
            axpy(alpha, p, x, n);                                   /* :463-465 */
            axpy(mk(-alpha.re, -alpha.im), Ap, r, n);               /* :467-473 */
            cx v2 = dotu3(r, r, a);                                 /* :475-479 */
            cx beta = cdiv(mk(1, 0), v2);                           /* :482-486 */
            axpy(beta, r, p, n);                                    /* :489-491 */
            Error = sqrt((v2.re * v2.re + v2.im * v2.im) / (vx.re * vx.re + vx.im * vx.im));
            if (Error < thr) { steps = m; break; }
        }
    } else {
        rcode = 2;
    }
done:
    if (steps_out) *steps_out = steps;
    if (err_out) *err_out = Error;
    free(b); free(r); free(p); free(q); free(Ap); free(Aq); free(rc); free(pc); free(qc);
    op_free(&o);
    return rcode;
}

/* ------------------------------------------------------------------------ */
/* Post-processing sums of NearFar.h                                          */
/* ------------------------------------------------------------------------ */
double vo_farfield1(const vo_grid* g, const double* xin, double theta, double phi, double psi) {
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const size_t a = (size_t)nx * ny * nz;
    const cx* J = (const cx*)xin;
    const double Volume = g->dx * g->dy * g->dz;
    const double v1 = cos(PI * theta / 180.0), v2 = sin(PI * theta / 180.0);   /* :44-47 */
    const double v3 = cos(PI * phi / 180.0), v4 = sin(PI * phi / 180.0);
    const double vx = v2 * v3, vy = v2 * v4, vz = v1;
    cx S[3] = {{0, 0}, {0, 0}, {0, 0}};
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                double xm = (i + 0.5) * g->dx, ym = (j + 0.5) * g->dy, zm = (k + 0.5) * g->dz;
                cx ph = cexpi(g->k0 * (xm * vx + ym * vy + zm * vz));    /* :71-72 */
                size_t v = ((size_t)i * ny + j) * nz + k;
                for (int c = 0; c < 3; c++) S[c] = add(S[c], mul(ph, J[c * a + v]));
            }
    S[0] = scl(mul(cexpi(g->k0 * 0.5 * g->dx * vx), S[0]), Volume);        /* :89-96 */
    S[1] = scl(mul(cexpi(g->k0 * 0.5 * g->dy * vy), S[1]), Volume);
    S[2] = scl(mul(cexpi(g->k0 * 0.5 * g->dz * vz), S[2]), Volume);
    double tm = Z0 * (S[0].re * v1 * v3 + S[1].re * v1 * v4 - S[2].re * v2);   /* :99-100 */
    double te = Z0 * (S[0].re * v4 - S[1].re * v3);                            /* :103-104 */
    return cos(PI * psi / 180.0) * tm - sin(PI * psi / 180.0) * te;            /* :107 */
}

int vo_absorption(const vo_grid* g, const double* xin, const double* eps_in,
                  const unsigned char* mat, int metal_label, int active_label,
                  double* metal_abs, double* active_abs, double* active_volume) {
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const size_t a = (size_t)nx * ny * nz;
    const cx* J = (const cx*)xin;
    const cx* eps = (const cx*)eps_in;
    const double k0 = g->k0;
    const cx V5 = mk(0.0, -1.0 / 2.0 * Z0 / k0), V6 = mk(1.0, 0.0), V7 = mk(2.0, 0.0); /* :125-127 */
    const double dV = g->dx * g->dy * g->dz;
    double em = 0.0, ea = 0.0, av = 0.0;
    const size_t step[3] = {(size_t)ny * nz, (size_t)nz, 1};
    for (int i = 0; i < nx - 1; i++)                                       /* :186-190 */
        for (int j = 0; j < ny - 1; j++)
            for (int k = 0; k < nz - 1; k++) {
                size_t v = ((size_t)i * ny + j) * nz + k;
                for (int c = 0; c < 3; c++) {
                    cx Jc = J[c * a + v];
                    double absJ = sqrt(Jc.re * Jc.re + Jc.im * Jc.im);
                    cx e2 = eps[v + step[c]], e3 = eps[v];
                    cx V2 = mk(e2.re - 1.0, e2.im), V3 = mk(e3.re - 1.0, e3.im);
                    V2 = add(cdiv(V6, V2), cdiv(V6, V3));
                    cx V1 = mul(V2, V5);
                    cx V4 = add(cdiv(V7, V2), V6);
                    double absE = absJ * sqrt(V1.re * V1.re + V1.im * V1.im);
                    unsigned char m2 = mat[v + step[c]], m3 = mat[v];
                    double contrib = k0 / Z0 * (-V4.im) * absE * absE * dV;
                    if (m2 == metal_label && m3 == metal_label) em += contrib;
                    if (m2 == active_label && m3 == active_label) { ea += contrib; av += dV; }
                }
            }
    if (metal_abs) *metal_abs = em;
    if (active_abs) *active_abs = ea;
    if (active_volume) *active_volume = av;
    return 0;
}

/* One self-term block exactly as L_DC_Dq (fft.h:41-127) does it on an already
   expanded (2N)^3 current: forward FFT, spectral multiply, backward FFT,
   field += crop.  Used to time the CPU baseline per block. */
int vo_block(const vo_grid* g, const double* green, double* padded, double* field) {
    op_ctx o;
    if (op_init(&o, g, green, NULL, NULL)) { op_free(&o); return 1; }
    free(o.tmp);
    o.tmp = (cx*)padded;
    int rc = fft_block(&o, (cx*)field, 0, 0, 0);
    o.tmp = NULL;
    op_free(&o);
    return rc;
}

