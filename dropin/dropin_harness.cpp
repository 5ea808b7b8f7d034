/*
 * dropin_harness.cpp -- test harness for the drop-in headers (not part of the
 * drop-in itself): the same entry points as oracle/ref_harness.cpp, but every
 * reference function here is the drop-in one, so the parity tests feed both
 * harnesses the same inputs.  Built by dropin/Makefile into
 * dropin/_build/libvie_dropin_harness.so.
 */
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "GreenFunction.h"
#include "fft.h"
#include "CG_Iteration.h"

static int g_live = 0;

extern "C" {

int dh_setup(int nx, int ny, int nz, double dx, double dy, double dz, double k0_in, const double* eps_re4,
             const double* eps_im4, double theta, double phi, double psi) {
    Nx = nx; Ny = ny; Nz = nz;
    NNx = 2 * Nx; NNy = 2 * Ny; NNz = 2 * Nz;
    delta_x = dx; delta_y = dy; delta_z = dz;
    k0 = k0_in;
    for (int m = 0; m < NUM_DIE; m++) { Real_EPR[m] = eps_re4[m]; Imag_EPR[m] = eps_im4[m]; }
    Theta = theta; Phi = phi; Psi = psi;
    if (g_live) {
        RMemory3D(Current_X); RMemory3D(Current_Y); RMemory3D(Current_Z); RMemory3D(Green_Function);
        RMemory3D(Material); RMemory3D(Ex_inc); RMemory3D(Ey_inc); RMemory3D(Ez_inc);
        RMemory3D(Flag_X); RMemory3D(Flag_Y); RMemory3D(Flag_Z);
    }
    Current_X = Memory3D(Current_X, Nx, Ny, Nz); Current_Y = Memory3D(Current_Y, Nx, Ny, Nz);
    Current_Z = Memory3D(Current_Z, Nx, Ny, Nz); Green_Function = Memory3D(Green_Function, NNx, NNy, NNz);
    Material = Memory3D(Material, Nx, Ny, Nz); Ex_inc = Memory3D(Ex_inc, Nx, Ny, Nz);
    Ey_inc = Memory3D(Ey_inc, Nx, Ny, Nz); Ez_inc = Memory3D(Ez_inc, Nx, Ny, Nz);
    Flag_X = Memory3D(Flag_X, Nx, Ny, Nz); Flag_Y = Memory3D(Flag_Y, Nx, Ny, Nz); Flag_Z = Memory3D(Flag_Z, Nx, Ny, Nz);
    g_live = 1;
    return 0;
}

int dh_set_geometry(const unsigned char* material, const unsigned char* fx, const unsigned char* fy,
                    const unsigned char* fz) {
    size_t a = (size_t)Nx * Ny * Nz;
    memcpy(Material[0][0], material, a); memcpy(Flag_X[0][0], fx, a);
    memcpy(Flag_Y[0][0], fy, a); memcpy(Flag_Z[0][0], fz, a);
    return 0;
}

int dh_green(double* out) {
    Green_Function_Compute();
    if (out) memcpy(out, Green_Function[0][0], 16 * (size_t)NNx * NNy * NNz);
    return 0;
}

int dh_incident(double* ex, double* ey, double* ez) {
    Incident_Wave();
    size_t a = 16 * (size_t)Nx * Ny * Nz;
    memcpy(ex, Ex_inc[0][0], a); memcpy(ey, Ey_inc[0][0], a); memcpy(ez, Ez_inc[0][0], a);
    return 0;
}

int dh_row(int which, const double* in, double* out) {
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

int dh_block(int kind, int src, int fld, int conj, const double* in, double* out) {
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

int dh_reset(double* v, int flag) {
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

/* one driver through FFT_Program-style dispatch: 1 CG .. 5 BICORSTAB; x: 3a solution */
int dh_solve(int solver, double* x) {
    switch (solver) {
        case 1: CG_FFT(); break;
        case 2: BICG_FFT(); break;
        case 3: BICGSTAB_FFT(); break;
        case 4: CORS_FFT(); break;
        case 5: BICORSTAB_FFT(); break;
        default: return 2;
    }
    size_t a = 16 * (size_t)Nx * Ny * Nz;
    memcpy(x, Current_X[0][0], a); memcpy(x + a / 8, Current_Y[0][0], a); memcpy(x + a / 4, Current_Z[0][0], a);
    // the driver released Ex/Ey/Ez_inc, Green_Function and Flag_*: allocate fresh ones for later calls
    Ex_inc = Memory3D(Ex_inc, Nx, Ny, Nz); Ey_inc = Memory3D(Ey_inc, Nx, Ny, Nz); Ez_inc = Memory3D(Ez_inc, Nx, Ny, Nz);
    Green_Function = Memory3D(Green_Function, NNx, NNy, NNz);
    Flag_X = Memory3D(Flag_X, Nx, Ny, Nz); Flag_Y = Memory3D(Flag_Y, Nx, Ny, Nz); Flag_Z = Memory3D(Flag_Z, Nx, Ny, Nz);
    return 0;
}

}  // extern "C"
