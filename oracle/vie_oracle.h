/*
 * vie_oracle.h -- CPU restatement of the VIE_FFT hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker for the CUDA library: only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * it.  The product library (vie_fft_b200/) never links or calls it.
 *
 * Every array is row-major (C order, last index fastest) like the
 * reference's Memory3D buffers (common.h:68-94); complex numbers are
 * interleaved (re, im) doubles like MKL_Complex16.  Permittivities use the
 * reference's e^{+j omega t} sign convention (lossy media have a NEGATIVE
 * imaginary part, data/Au_epr.txt).
 *
 * Vector layout for the three current / field components: one contiguous
 * block of 3*a complex numbers, x then y then z, a = nx*ny*nz.
 */
#ifndef VIE_ORACLE_H
#define VIE_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int nx, ny, nz;     /* grid size (Nx, Ny, Nz in Model.h:32-34) */
    double dx, dy, dz;  /* cell sizes (delta_x/y/z, Model.h:28-30), units of 100 nm */
    double k0;          /* free-space wavenumber (Model.h:25) */
} vo_grid;

/* Green_Function_Compute (GreenFunction.h:8-141): scalar Green's function on
   (2nx,2ny,2nz), even periodic extension, forward FFT.  out: (2nx*2ny*2nz) complex. */
int vo_green(const vo_grid* g, double* out);

/* Incident_Wave (GreenFunction.h:144-248). e: 3*a complex (Ex_inc, Ey_inc, Ez_inc). */
int vo_incident(const vo_grid* g, double theta, double phi, double psi, double* e);

/* One operator application as the Krylov drivers perform it: zero field,
   X/Y/Z_FFT (CG_Iteration.h:131-173) or X/Y/Z_FFT_Conjugate (:86-128), then
   Current_Reset (fft.h:13-35).
   green: full (2N)^3 spectrum from vo_green; eps: a complex per-voxel
   permittivity (Real_EPR/Imag_EPR[Material], Model.h:82-83); flags: 3*a bytes
   (Flag_X, Flag_Y, Flag_Z); in/out: 3*a complex. */
int vo_matvec(const vo_grid* g, const double* green, const double* eps,
              const unsigned char* flags, const double* in, double* out, int conj);

/* Krylov drivers (CG_Iteration.h): solver 1 CG_FFT (:176-357), 2 BICG_FFT
   (:360-528), 3 BICGSTAB_FFT (:531-776), 4 CORS_FFT (:780-1073),
   5 BICORSTAB_FFT (:1076-1362).  einc: 3*a incident field (masked in place
   copy, the input is not modified); x: 3*a solution; maxit <= 0 means the
   reference cap nx*ny*nz.  steps: the step index m printed by the reference
   at convergence ("Steps: m"), or the number of iterations run if the cap is
   reached; err: the last error value. */
int vo_solve(const vo_grid* g, const double* green, const double* eps,
             const unsigned char* flags, const double* einc, int solver, double thr,
             int maxit, double* x, int* steps, double* err);

/* FarField1 (NearFar.h:16-109): Forward_RCS for incidence (theta, phi, psi). */
double vo_farfield1(const vo_grid* g, const double* x, double theta, double phi, double psi);

/* Absorption sums of NearField (NearFar.h:180-250): metal_abs = Ene_Metal,
   active_abs = Ene_Active, active_volume = Absorb_Volume, for material labels
   (0 air, 2 metal, 3 active in the reference model) and eps per voxel. */
int vo_absorption(const vo_grid* g, const double* x, const double* eps,
                  const unsigned char* material, int metal_label, int active_label,
                  double* metal_abs, double* active_abs, double* active_volume);

/* One L_DC_Dq block (fft.h:41-127) on an expanded (2nx,2ny,2nz) current
   (modified in place) accumulating into field (a complex); for timing. */
int vo_block(const vo_grid* g, const double* green, double* padded, double* field);

#ifdef __cplusplus
}
#endif
#endif
