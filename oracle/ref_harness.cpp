/*
 * ref_harness.cpp -- builds the REFERENCE's own hot-path code into
 * oracle/_ref/libvieref.so (test infrastructure only: it is the checker,
 * never the product).
 *
 * The reference headers are included from where they lie (the Makefile puts
 * the reference's vie_fft/ directory on the include path).  The only change
 * is a build-time copy of CG_Iteration.h written to oracle/_ref/gen/ in which
 * line 46 `const double CG_THR=0.001;` becomes a mutable global, so that a
 * caller can pick the relative-residual threshold (1e-6, 1e-8 ...) exactly as
 * a maintainer would by editing that constant.
 *
 * The harness replaces the reference's driver-level glue:
 *   - Parameter_Input (Model.h:88-213) derives the grid from PPW and
 *     staircase rules; here the caller gives Nx, Ny, Nz, the cell sizes, k0,
 *     the 4-entry permittivity table and the angles directly, and the arrays
 *     are allocated the way Model.h:172-201 does (Memory3D + memset 0).
 *   - printf from the Krylov drivers (CG_Iteration.h:326-331 etc.) is
 *     captured to record the step count and the last error.
 *   - fopen/fprintf/fclose in NearFar.h are captured so that the extinction
 *     and absorption numbers written to ../result/*.txt come back to the
 *     caller instead of the file system.
 */
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <cmath>
#include <memory.h>
#include <assert.h>
#include "mkl.h"

/* ---- printf / file capture ------------------------------------------------ */
static int g_quiet = 1;
static int g_steps = -1;
static double g_err = -1.0;
static int g_nprint = 0;

extern "C" int ref_printf(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    if (strncmp(fmt, "CG Error", 8) == 0) {
        g_err = va_arg(ap, double);
        g_nprint++;
    } else if (strncmp(fmt, "Steps", 5) == 0) {
        g_steps = va_arg(ap, int);
    } else if (strstr(fmt, "%d\n\n") != NULL && strstr(fmt, "%lf") == NULL) {
        /* BICORSTAB_FFT prints its step count with a non-ASCII label
           (CG_Iteration.h:1318); it is the only "%d\n\n" line there. */
        g_steps = va_arg(ap, int);
    }
    va_end(ap);
    if (!g_quiet) {
        va_start(ap, fmt);
        vprintf(fmt, ap);
        va_end(ap);
    }
    return 0;
}

enum { F_METAL = 1, F_ACTIVE, F_GRID, F_FIELD, F_RCS, F_OTHER };
static char g_file_tokens[8];
static double g_ext_over_cs = 0.0, g_metal_abs = 0.0, g_active_abs = 0.0;
static double g_rcs_theta[181], g_rcs_phi[181];
static int g_rcs_row = 0;

extern "C" FILE* ref_fopen(const char* name, const char* mode) {
    (void)mode;
    int t = F_OTHER;
    if (strstr(name, "Ene_Metal")) t = F_METAL;
    else if (strstr(name, "Ene_Active")) t = F_ACTIVE;
    else if (strstr(name, "Grid")) t = F_GRID;
    else if (strstr(name, "Field")) t = F_FIELD;
    else if (strstr(name, "RCS")) { t = F_RCS; g_rcs_row = 0; }
    return (FILE*)&g_file_tokens[t];
}

extern "C" int ref_fprintf(FILE* f, const char* fmt, ...) {
    int t = (int)((char*)f - g_file_tokens);
    va_list ap;
    va_start(ap, fmt);
    if (t == F_METAL) {
        (void)va_arg(ap, int);
        g_ext_over_cs = va_arg(ap, double);
        g_metal_abs = va_arg(ap, double);
    } else if (t == F_ACTIVE) {
        (void)va_arg(ap, int);
        g_active_abs = va_arg(ap, double);
    } else if (t == F_RCS && g_rcs_row < 181) {
        g_rcs_theta[g_rcs_row] = va_arg(ap, double);
        g_rcs_phi[g_rcs_row] = va_arg(ap, double);
        g_rcs_row++;
    }
    va_end(ap);
    return 0;
}

extern "C" int ref_fclose(FILE* f) { (void)f; return 0; }

#define printf ref_printf
#define fopen ref_fopen
#define fprintf ref_fprintf
#define fclose ref_fclose

#include "Model.h"
#include "GreenFunction.h"
#include "CG_Iteration.h" /* build-time copy with a mutable CG_THR */
#include "NearFar.h"

#undef printf
#undef fopen
#undef fprintf
#undef fclose

/* ---- state ---------------------------------------------------------------- */
static int g_alloc = 0;        /* model arrays allocated */
static int g_inputs_live = 0;  /* Ex/Ey/Ez_inc, Green_Function, Flag_* live (drivers free them) */
static int g_current_live = 0; /* Current_*, Material live (NearField frees them) */

static void free_all() {
    if (g_inputs_live) {
        RMemory3D(Ex_inc); RMemory3D(Ey_inc); RMemory3D(Ez_inc);
        RMemory3D(Green_Function);
        RMemory3D(Flag_X); RMemory3D(Flag_Y); RMemory3D(Flag_Z);
        g_inputs_live = 0;
    }
    if (g_current_live) {
        RMemory3D(Current_X); RMemory3D(Current_Y); RMemory3D(Current_Z);
        RMemory3D(Material);
        g_current_live = 0;
    }
    g_alloc = 0;
}

extern "C" {

void ref_set_verbose(int v) { g_quiet = v ? 0 : 1; }

/* Allocate and zero every model array the way Model.h:172-201 does. */
int ref_setup(int nx, int ny, int nz, double dx, double dy, double dz, double k0_in,
              const double* eps_re4, const double* eps_im4, double theta, double phi,
              double psi) {
    if (nx < 2 || ny < 2 || nz < 2) return 1;
    free_all();
    Nx = nx; Ny = ny; Nz = nz;
    NNx = 2 * Nx; NNy = 2 * Ny; NNz = 2 * Nz;
    delta_x = dx; delta_y = dy; delta_z = dz;
    k0 = k0_in;
    for (int m = 0; m < NUM_DIE; m++) { Real_EPR[m] = eps_re4[m]; Imag_EPR[m] = eps_im4[m]; }
    Theta = theta; Phi = phi; Psi = psi;
    Current_X = Memory3D(Current_X, Nx, Ny, Nz);
    Current_Y = Memory3D(Current_Y, Nx, Ny, Nz);
    Current_Z = Memory3D(Current_Z, Nx, Ny, Nz);
    Green_Function = Memory3D(Green_Function, NNx, NNy, NNz);
    Material = Memory3D(Material, Nx, Ny, Nz);
    Ex_inc = Memory3D(Ex_inc, Nx, Ny, Nz);
    Ey_inc = Memory3D(Ey_inc, Nx, Ny, Nz);
    Ez_inc = Memory3D(Ez_inc, Nx, Ny, Nz);
    Flag_X = Memory3D(Flag_X, Nx, Ny, Nz);
    Flag_Y = Memory3D(Flag_Y, Nx, Ny, Nz);
    Flag_Z = Memory3D(Flag_Z, Nx, Ny, Nz);
    size_t a = (size_t)Nx * Ny * Nz, m = (size_t)NNx * NNy * NNz;
    memset(Current_X[0][0], 0, a * sizeof(MKL_Complex16));
    memset(Current_Y[0][0], 0, a * sizeof(MKL_Complex16));
    memset(Current_Z[0][0], 0, a * sizeof(MKL_Complex16));
    memset(Green_Function[0][0], 0, m * sizeof(MKL_Complex16));
    memset(Ex_inc[0][0], 0, a * sizeof(MKL_Complex16));
    memset(Ey_inc[0][0], 0, a * sizeof(MKL_Complex16));
    memset(Ez_inc[0][0], 0, a * sizeof(MKL_Complex16));
    memset(Material[0][0], 0, a);
    memset(Flag_X[0][0], 0, a);
    memset(Flag_Y[0][0], 0, a);
    memset(Flag_Z[0][0], 0, a);
    g_alloc = g_inputs_live = g_current_live = 1;
    return 0;
}

/* Material index and the three edge flags from the caller (row-major Nx*Ny*Nz). */
int ref_set_geometry(const unsigned char* material, const unsigned char* fx,
                     const unsigned char* fy, const unsigned char* fz) {
    if (!g_inputs_live || !g_current_live) return 1;
    size_t a = (size_t)Nx * Ny * Nz;
    memcpy(Material[0][0], material, a);
    memcpy(Flag_X[0][0], fx, a);
    memcpy(Flag_Y[0][0], fy, a);
    memcpy(Flag_Z[0][0], fz, a);
    return 0;
}

/* The reference's own single-sphere geometry: Model_Identifier (Model.h:216-236)
   through GetMaterial (Model.h:305-332) and GetFlag (Model.h:335-398). */
int ref_sphere_geometry(double dia, double box_l, double box_w, double box_h) {
    if (!g_inputs_live || !g_current_live) return 1;
    Dia = dia; Box_L = box_l; Box_W = box_w; Box_H = box_h;
    Cross_Section = PI * Dia * Dia / 4.0;
    GetMaterial();
    GetFlag();
    return 0;
}

int ref_get_geometry(unsigned char* material, unsigned char* fx, unsigned char* fy,
                     unsigned char* fz) {
    if (!g_inputs_live || !g_current_live) return 1;
    size_t a = (size_t)Nx * Ny * Nz;
    memcpy(material, Material[0][0], a);
    memcpy(fx, Flag_X[0][0], a);
    memcpy(fy, Flag_Y[0][0], a);
    memcpy(fz, Flag_Z[0][0], a);
    return 0;
}

void ref_set_cross_section(double cs) { Cross_Section = cs; }

/* Green_Function_Compute (GreenFunction.h:8-141); out gets the (2Nx,2Ny,2Nz) spectrum. */
int ref_green(double* out) {
    if (!g_inputs_live) return 1;
    Green_Function_Compute();
    if (out) memcpy(out, Green_Function[0][0], sizeof(MKL_Complex16) * (size_t)NNx * NNy * NNz);
    return 0;
}

/* Overwrite the stored Green spectrum (e.g. with one computed elsewhere). */
int ref_set_green(const double* in) {
    if (!g_inputs_live) return 1;
    memcpy(Green_Function[0][0], in, sizeof(MKL_Complex16) * (size_t)NNx * NNy * NNz);
    return 0;
}

/* Incident_Wave (GreenFunction.h:144-248). */
int ref_incident(double* ex, double* ey, double* ez) {
    if (!g_inputs_live) return 1;
    Incident_Wave();
    size_t a = sizeof(MKL_Complex16) * (size_t)Nx * Ny * Nz;
    if (ex) memcpy(ex, Ex_inc[0][0], a);
    if (ey) memcpy(ey, Ey_inc[0][0], a);
    if (ez) memcpy(ez, Ez_inc[0][0], a);
    return 0;
}

int ref_set_incident(const double* ex, const double* ey, const double* ez) {
    if (!g_inputs_live) return 1;
    size_t a = sizeof(MKL_Complex16) * (size_t)Nx * Ny * Nz;
    memcpy(Ex_inc[0][0], ex, a);
    memcpy(Ey_inc[0][0], ey, a);
    memcpy(Ez_inc[0][0], ez, a);
    return 0;
}

/* One operator application exactly as the drivers do it: zero the field,
   X_FFT/Y_FFT/Z_FFT (CG_Iteration.h:131-173) or their _Conjugate twins
   (:86-128), then Current_Reset (fft.h:13-35).  in/out: 3 x Nx*Ny*Nz complex. */
int ref_matvec(const double* in, double* out, int conj) {
    if (!g_inputs_live || !g_current_live) return 1;
    int Dim[3] = {Nx, Ny, Nz};
    size_t a = (size_t)Nx * Ny * Nz;
    MKL_Complex16*** sx = NULL; MKL_Complex16*** sy = NULL; MKL_Complex16*** sz = NULL;
    MKL_Complex16*** fx = NULL; MKL_Complex16*** fy = NULL; MKL_Complex16*** fz = NULL;
    MKL_Complex16*** tmp = NULL;
    sx = Memory3D(sx, Nx, Ny, Nz); sy = Memory3D(sy, Nx, Ny, Nz); sz = Memory3D(sz, Nx, Ny, Nz);
    fx = Memory3D(fx, Nx, Ny, Nz); fy = Memory3D(fy, Nx, Ny, Nz); fz = Memory3D(fz, Nx, Ny, Nz);
    tmp = Memory3D(tmp, NNx, NNy, NNz);
    memcpy(sx[0][0], in, a * sizeof(MKL_Complex16));
    memcpy(sy[0][0], in + 2 * a, a * sizeof(MKL_Complex16));
    memcpy(sz[0][0], in + 4 * a, a * sizeof(MKL_Complex16));
    memset(fx[0][0], 0, a * sizeof(MKL_Complex16));
    memset(fy[0][0], 0, a * sizeof(MKL_Complex16));
    memset(fz[0][0], 0, a * sizeof(MKL_Complex16));
    if (conj) {
        X_FFT_Conjugate(fx, sx, sy, sz, tmp, Green_Function, Dim);
        Y_FFT_Conjugate(fy, sx, sy, sz, tmp, Green_Function, Dim);
        Z_FFT_Conjugate(fz, sx, sy, sz, tmp, Green_Function, Dim);
    } else {
        X_FFT(fx, sx, sy, sz, tmp, Green_Function, Dim);
        Y_FFT(fy, sx, sy, sz, tmp, Green_Function, Dim);
        Z_FFT(fz, sx, sy, sz, tmp, Green_Function, Dim);
    }
    Current_Reset(fx, 0, Dim);
    Current_Reset(fy, 1, Dim);
    Current_Reset(fz, 2, Dim);
    memcpy(out, fx[0][0], a * sizeof(MKL_Complex16));
    memcpy(out + 2 * a, fy[0][0], a * sizeof(MKL_Complex16));
    memcpy(out + 4 * a, fz[0][0], a * sizeof(MKL_Complex16));
    RMemory3D(sx); RMemory3D(sy); RMemory3D(sz);
    RMemory3D(fx); RMemory3D(fy); RMemory3D(fz);
    RMemory3D(tmp);
    return 0;
}

/* Per-function parity of the operator pieces.  `which`:
   0..2  X_FFT / Y_FFT / Z_FFT (CG_Iteration.h:131-173) on (in) -> field
   3..5  the _Conjugate twins (:86-128)
   Field starts at zero, no Current_Reset (the drivers reset afterwards). */
int ref_row(int which, const double* in, double* out) {
    if (!g_inputs_live || !g_current_live) return 1;
    int Dim[3] = {Nx, Ny, Nz};
    size_t a = (size_t)Nx * Ny * Nz;
    MKL_Complex16*** sx = NULL; MKL_Complex16*** sy = NULL; MKL_Complex16*** sz = NULL;
    MKL_Complex16*** f = NULL; MKL_Complex16*** tmp = NULL;
    sx = Memory3D(sx, Nx, Ny, Nz); sy = Memory3D(sy, Nx, Ny, Nz); sz = Memory3D(sz, Nx, Ny, Nz);
    f = Memory3D(f, Nx, Ny, Nz); tmp = Memory3D(tmp, NNx, NNy, NNz);
    memcpy(sx[0][0], in, a * 16); memcpy(sy[0][0], in + 2 * a, a * 16); memcpy(sz[0][0], in + 4 * a, a * 16);
    memset(f[0][0], 0, a * 16);
    switch (which) {
        case 0: X_FFT(f, sx, sy, sz, tmp, Green_Function, Dim); break;
        case 1: Y_FFT(f, sx, sy, sz, tmp, Green_Function, Dim); break;
        case 2: Z_FFT(f, sx, sy, sz, tmp, Green_Function, Dim); break;
        case 3: X_FFT_Conjugate(f, sx, sy, sz, tmp, Green_Function, Dim); break;
        case 4: Y_FFT_Conjugate(f, sx, sy, sz, tmp, Green_Function, Dim); break;
        case 5: Z_FFT_Conjugate(f, sx, sy, sz, tmp, Green_Function, Dim); break;
        default: return 2;
    }
    memcpy(out, f[0][0], a * 16);
    RMemory3D(sx); RMemory3D(sy); RMemory3D(sz); RMemory3D(f); RMemory3D(tmp);
    return 0;
}

/* One block on component `src` of (in) after Current_Expansion (CG_Iteration.h:50-83):
   kind 0 L_DC_Dq (fld = src), 1 L_Dq, 2 L??_DO of src; conj selects the
   _Conjugate twin.  Field starts at zero. */
int ref_block(int kind, int src, int fld, int conj, const double* in, double* out) {
    if (!g_inputs_live || !g_current_live) return 1;
    int Dim[3] = {Nx, Ny, Nz};
    size_t a = (size_t)Nx * Ny * Nz;
    MKL_Complex16*** J = NULL; MKL_Complex16*** f = NULL; MKL_Complex16*** tmp = NULL;
    J = Memory3D(J, Nx, Ny, Nz); f = Memory3D(f, Nx, Ny, Nz); tmp = Memory3D(tmp, NNx, NNy, NNz);
    memcpy(J[0][0], in + 2 * a * src, a * 16);
    memset(f[0][0], 0, a * 16);
    Current_Expansion(tmp, J, src, Dim);
    const double d[3] = {delta_x, delta_y, delta_z};
    if (kind == 0) {
        if (conj) L_DC_Dq_Conjugate(f, tmp, Green_Function, d[src], src, Dim);
        else L_DC_Dq(f, tmp, Green_Function, d[src], src, Dim);
    } else if (kind == 1) {
        if (conj) L_Dq_Conjugate(f, tmp, Green_Function, src, fld, d[fld], Dim);
        else L_Dq(f, tmp, Green_Function, src, fld, d[src], Dim);
    } else {
        if (src == 0) { if (conj) LXX_DO_Conjugate(f, tmp, Dim); else LXX_DO(f, tmp, Dim); }
        if (src == 1) { if (conj) LYY_DO_Conjugate(f, tmp, Dim); else LYY_DO(f, tmp, Dim); }
        if (src == 2) { if (conj) LZZ_DO_Conjugate(f, tmp, Dim); else LZZ_DO(f, tmp, Dim); }
    }
    memcpy(out, f[0][0], a * 16);
    RMemory3D(J); RMemory3D(f); RMemory3D(tmp);
    return 0;
}

/* Current_Reset (fft.h:13-35) on a copy. */
int ref_reset(double* v, int flag) {
    if (!g_inputs_live) return 1;
    int Dim[3] = {Nx, Ny, Nz};
    size_t a = (size_t)Nx * Ny * Nz;
    MKL_Complex16*** J = NULL;
    J = Memory3D(J, Nx, Ny, Nz);
    memcpy(J[0][0], v, a * 16);
    Current_Reset(J, flag, Dim);
    memcpy(v, J[0][0], a * 16);
    RMemory3D(J);
    return 0;
}

/* One self-term block L_DC_Dq (fft.h:41-127) on a pre-expanded (2N)^3 array,
   for per-function timing of the reference (the unit of one matvec is nine of
   these blocks plus cheap O(N^3) work). */
int ref_time_block(double* padded, double* field) {
    if (!g_inputs_live) return 1;
    int Dim[3] = {Nx, Ny, Nz};
    MKL_Complex16*** tmp = NULL;
    MKL_Complex16*** fld = NULL;
    tmp = (MKL_Complex16***)malloc(sizeof(MKL_Complex16**) * NNx);
    tmp[0] = (MKL_Complex16**)malloc(sizeof(MKL_Complex16*) * (size_t)NNx * NNy);
    for (int i = 0; i < NNx; i++) tmp[i] = tmp[0] + (size_t)NNy * i;
    tmp[0][0] = (MKL_Complex16*)padded;
    for (int i = 0; i < NNx; i++)
        for (int j = 0; j < NNy; j++) tmp[i][j] = tmp[0][0] + ((size_t)i * NNy + j) * NNz;
    fld = (MKL_Complex16***)malloc(sizeof(MKL_Complex16**) * Nx);
    fld[0] = (MKL_Complex16**)malloc(sizeof(MKL_Complex16*) * (size_t)Nx * Ny);
    for (int i = 0; i < Nx; i++) fld[i] = fld[0] + (size_t)Ny * i;
    fld[0][0] = (MKL_Complex16*)field;
    for (int i = 0; i < Nx; i++)
        for (int j = 0; j < Ny; j++) fld[i][j] = fld[0][0] + ((size_t)i * Ny + j) * Nz;
    L_DC_Dq(fld, tmp, Green_Function, delta_x, 0, Dim);
    free(tmp[0]); free(tmp); free(fld[0]); free(fld);
    return 0;
}

/* Run one of the reference Krylov drivers (CG_Iteration.h): 1 CG_FFT, 2 BICG_FFT,
   3 BICGSTAB_FFT, 4 CORS_FFT, 5 BICORSTAB_FFT, with threshold thr.  x: 3 x a
   complex solution (Current_X/Y/Z).  The drivers free Ex/Ey/Ez_inc,
   Green_Function and Flag_* (CG_Iteration.h:769-775); the harness records that. */
int ref_solve(int solver, double thr, double* x, int* steps, double* last_err) {
    if (!g_inputs_live || !g_current_live) return 1;
    CG_THR = thr;
    size_t a = (size_t)Nx * Ny * Nz;
    memset(Current_X[0][0], 0, a * sizeof(MKL_Complex16));
    memset(Current_Y[0][0], 0, a * sizeof(MKL_Complex16));
    memset(Current_Z[0][0], 0, a * sizeof(MKL_Complex16));
    g_steps = -1; g_err = -1.0; g_nprint = 0;
    switch (solver) {
        case 1: CG_FFT(); break;
        case 2: BICG_FFT(); break;
        case 3: BICGSTAB_FFT(); break;
        case 4: CORS_FFT(); break;
        case 5: BICORSTAB_FFT(); break;
        default: return 2;
    }
    g_inputs_live = 0; /* freed by the driver */
    if (x) {
        memcpy(x, Current_X[0][0], a * sizeof(MKL_Complex16));
        memcpy(x + 2 * a, Current_Y[0][0], a * sizeof(MKL_Complex16));
        memcpy(x + 4 * a, Current_Z[0][0], a * sizeof(MKL_Complex16));
    }
    if (steps) *steps = g_steps;
    if (last_err) *last_err = g_err;
    return 0;
}

/* Overwrite Current_X/Y/Z (e.g. with a solution computed elsewhere) before the
   post-processing calls below. */
int ref_set_current(const double* x) {
    if (!g_current_live) return 1;
    size_t a = (size_t)Nx * Ny * Nz;
    memcpy(Current_X[0][0], x, a * sizeof(MKL_Complex16));
    memcpy(Current_Y[0][0], x + 2 * a, a * sizeof(MKL_Complex16));
    memcpy(Current_Z[0][0], x + 4 * a, a * sizeof(MKL_Complex16));
    return 0;
}

/* FarField1 (NearFar.h:16-109): forward scattering amplitude Forward_RCS. */
int ref_farfield1(double* forward_rcs) {
    if (!g_current_live) return 1;
    FarField1();
    if (forward_rcs) *forward_rcs = Forward_RCS;
    return 0;
}

/* FarField2 (NearFar.h:302-477): 181 E-plane and 181 H-plane RCS values (dB). */
int ref_farfield2(double* rcs_theta, double* rcs_phi) {
    if (!g_current_live) return 1;
    FarField2();
    if (rcs_theta) memcpy(rcs_theta, g_rcs_theta, sizeof(g_rcs_theta));
    if (rcs_phi) memcpy(rcs_phi, g_rcs_phi, sizeof(g_rcs_phi));
    return 0;
}

/* NearField (NearFar.h:113-298): returns the three numbers it writes,
   extinction/Cross_Section, Ene_Metal*Z0/Cross_Section and
   3*Ene_Active/Absorb_Volume.  NearField frees Current_* and Material. */
int ref_nearfield(double* ext_over_cs, double* metal_abs, double* active_abs) {
    if (!g_current_live) return 1;
    NearField();
    g_current_live = 0;
    if (ext_over_cs) *ext_over_cs = g_ext_over_cs;
    if (metal_abs) *metal_abs = g_metal_abs;
    if (active_abs) *active_abs = g_active_abs;
    return 0;
}

void ref_release(void) { free_all(); }

} /* extern "C" */
