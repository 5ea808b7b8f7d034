/*
 * vie_b200.h -- C ABI of the B200 VIE-FFT library (libvie_b200.so).
 *
 * Plain pointers and sizes only.  Host arrays follow the reference layout:
 * C order (last index fastest) over (nx, ny, nz) like Memory3D buffers
 * (common.h:68-94); complex values are interleaved (re, im) doubles like
 * MKL_Complex16; a vector of the three current / field components is one
 * block of 3*a complex values (x, then y, then z), a = nx*ny*nz.
 * Permittivities use the reference's exp(+j omega t) sign convention: lossy
 * media have a NEGATIVE imaginary part (data/Au_epr.txt).
 *
 * Every function returns a status code (VIE_OK = 0) and leaves a message for
 * vie_last_error().  The reference checks no status at all; the drop-in
 * headers (dropin/*.h) turn a non-zero status into a message on stderr and
 * exit(1).
 *
 * One context = one grid on one GPU with one CUDA stream.  Contexts are
 * independent; a single context is not safe for concurrent calls.
 */
#ifndef VIE_B200_H
#define VIE_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define VIE_API __attribute__((visibility("default")))
#else
#define VIE_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define VIE_OK 0
#define VIE_ERR_ARG 1        /* bad argument or size */
#define VIE_ERR_ALLOC 2      /* device or host allocation failed */
#define VIE_ERR_CUDA 3       /* CUDA runtime error */
#define VIE_ERR_BREAKDOWN 4  /* Krylov breakdown (zero denominator) */
#define VIE_ERR_MAXIT 5      /* iteration cap reached before the tolerance */
#define VIE_ERR_NAN 6        /* NaN / Inf in the iteration */
#define VIE_ERR_STATE 7      /* call order (e.g. solve before vie_green) */
#define VIE_ERR_TIMEOUT 8    /* a bounded device wait expired */
#define VIE_ERR_NODEVICE 9   /* no CUDA device */

/* solvers: the reference's Iteration_Type values (CG_Iteration.h:47) */
#define VIE_SOLVER_CG 1         /* CGNR, CG_FFT (CG_Iteration.h:176-357) */
#define VIE_SOLVER_BICG 2       /* complex-symmetric BiCG, BICG_FFT (:360-528) */
#define VIE_SOLVER_BICGSTAB 3   /* BICGSTAB_FFT (:531-776), the reference default */
#define VIE_SOLVER_CORS 4       /* CORS_FFT (:780-1073) */
#define VIE_SOLVER_BICORSTAB 5  /* BICORSTAB_FFT (:1076-1362) */

/* arithmetic of a solve */
#define VIE_PREC_FP64 0   /* every operation in FP64 complex */
#define VIE_PREC_MIXED 1  /* FP32-complex Krylov with FP64 defect correction: BiCGSTAB
                             folds in FP64 true residuals (reliable updates), the other
                             drivers restart an FP32 inner solve per FP64 refinement */

typedef struct vie_ctx vie_ctx;

typedef struct {
    int nx, ny, nz;      /* grid, Nx/Ny/Nz of Model.h:32-34 (each >= 2) */
    double dx, dy, dz;   /* cell sizes delta_x/y/z (Model.h:28-30), in the reference's 100 nm unit */
    double k0;           /* free-space wavenumber (Model.h:25) */
    int device;          /* CUDA device ordinal */
} vie_grid;

/* Create a context for one grid.  Replaces the allocation part of
   Parameter_Input (Model.h:172-201) for the arrays the hot path owns. */
VIE_API int vie_create(const vie_grid* g, vie_ctx** out);
VIE_API void vie_destroy(vie_ctx* ctx);
VIE_API const char* vie_last_error(const vie_ctx* ctx);
VIE_API const char* vie_status_string(int status);

/* Geometry.  material: a bytes of indices into a permittivity table of
   n_materials entries (the reference's Material with Real_EPR / Imag_EPR,
   Model.h:17, 81-83; index 0 is the air dummy 1.1).  Equivalent per-voxel
   form: vie_set_eps with a complex values. */
VIE_API int vie_set_material(vie_ctx* ctx, const uint8_t* material, const double* eps_re, const double* eps_im,
                     int n_materials);
VIE_API int vie_set_eps(vie_ctx* ctx, const double* eps);
/* Edge flags Flag_X, Flag_Y, Flag_Z (Model.h:21-23, GetFlag Model.h:335-398), a bytes each. */
VIE_API int vie_set_flags(vie_ctx* ctx, const uint8_t* fx, const uint8_t* fy, const uint8_t* fz);

/* Green_Function_Compute (GreenFunction.h:8-141), on the GPU in FP64.  The
   spectrum is kept as its (nx+1)(ny+1)(nz+1) even-symmetric octant. */
VIE_API int vie_green(vie_ctx* ctx);
/* The natural-order (2nx, 2ny, 2nz) spectrum the reference stores in
   Green_Function after Green_Function_Compute. out: 8a complex. */
VIE_API int vie_green_spectrum(vie_ctx* ctx, double* out);

/* Incident_Wave (GreenFunction.h:144-248), on the GPU in FP64.  The field
   becomes the right-hand side of the next solve; out (3a complex) may be NULL. */
VIE_API int vie_incident(vie_ctx* ctx, double theta, double phi, double psi, double* out);
/* Right-hand side from the host (Ex_inc, Ey_inc, Ez_inc; 3a complex). */
VIE_API int vie_set_rhs(vie_ctx* ctx, const double* e);

/* One operator application y = A x, or y = A^H x when conj != 0, with host
   buffers (3a complex each), exactly as the drivers compose it: zeroed field,
   X_FFT/Y_FFT/Z_FFT (CG_Iteration.h:131-173) or the _Conjugate twins
   (:86-128), then Current_Reset (fft.h:13-35). */
VIE_API int vie_matvec(vie_ctx* ctx, const double* x, double* y, int conj);
/* Same as vie_matvec (FP64, host buffers), but it allocates no device memory.
   No counterpart in the reference.  For callers that must not allocate while
   they apply the operator: code that calls it inside a long loop, where the
   cudaMalloc/cudaFree pair of vie_matvec would synchronise the whole device
   each time, or a process whose free device memory is held by another
   allocator, where a new cudaMalloc can fail.  The device copies of x and y
   and the pass scratch live in one static 64 MiB device array per GPU, so the
   grid may have at most 174762 voxels (VIE_ERR_ARG beyond that).  All calls on
   a GPU share that array: calls that overlap on one GPU race and must be
   serialised by the caller.  The first call on a device looks up the array's
   device address; make it before any stream capture. */
VIE_API int vie_matvec_static(vie_ctx* ctx, const double* x, double* y, int conj);
/* Parts of one operator application, for the reference's block functions:
   VIE_PART_GREEN  the FFT blocks L_DC_Dq / L_Dq (fft.h:41-127, 224-309)
   VIE_PART_DIAG   the diagonal terms LXX_DO / LYY_DO / LZZ_DO (fft.h:405-588)
   VIE_PART_MASK   Current_Reset of the output (fft.h:13-35)
   vie_matvec is vie_apply with VIE_PART_ALL; X_FFT etc. are GREEN | DIAG. */
#define VIE_PART_GREEN 1
#define VIE_PART_DIAG 2
#define VIE_PART_MASK 4
#define VIE_PART_ALL 7
VIE_API int vie_apply(vie_ctx* ctx, const double* x, double* y, int conj, int parts);
/* Current_Reset (fft.h:13-35): v (a complex, host) *= Flag of component comp (0 x, 1 y, 2 z). */
VIE_API int vie_reset(vie_ctx* ctx, double* v, int comp);
/* Same on device buffers of the context's GPU.  precision VIE_PREC_FP64:
   x, y are 3a double2; VIE_PREC_MIXED: 3a float2 (the FP32 operator).
   Runs on the context stream; returns after the launch (no sync). */
VIE_API int vie_matvec_dev(vie_ctx* ctx, const void* x, void* y, int conj, int precision);

typedef struct {
    int solver;         /* VIE_SOLVER_* */
    int precision;      /* VIE_PREC_FP64 or VIE_PREC_MIXED */
    double tol;         /* relative-residual threshold (CG_THR, CG_Iteration.h:46) */
    int max_iter;       /* iteration cap; <= 0 means nx*ny*nz like the reference */
    double inner_tol;   /* mixed: residual reduction per FP64 refinement step
                           (<= 0: 0.03 for BiCGSTAB's reliable updates, 5e-5 for the
                           restarted inner solves of the other drivers, whose last
                           one stops at 0.9 of the reduction still needed) */
    int max_outer;      /* mixed: refinement cap (<= 0: 30) */
    int verbose;        /* print "CG Error" per iteration like the reference */
    int true_residual;  /* FP64 solves: evaluate ||b - A x|| / ||b|| at exit (one more
                           operator application); mixed solves always report it */
} vie_solve_params;

typedef struct {
    int steps;          /* index m of the converged iteration ("Steps: m"), as the reference prints */
    int iterations;     /* Krylov iterations executed (sum of inner ones when mixed) */
    int outer;          /* refinement steps (mixed) */
    int matvecs_fp64;   /* operator applications in FP64 */
    int matvecs_fp32;   /* operator applications in FP32 */
    double relres;      /* the solver's own residual estimate at exit */
    double true_relres; /* ||b - A x|| / ||b|| in FP64 at exit (-1 when not evaluated) */
    double seconds;     /* device time of the solve */
    int graph_loops;    /* iteration loops of the solve that ran as one CUDA graph launch (a device-side
                           WHILE loop over the captured iteration body); 0: iterated from the host */
    int status;         /* this solve's own status (VIE_OK, VIE_ERR_MAXIT, VIE_ERR_BREAKDOWN, ...) */
} vie_solve_info;

/* Solve A x = b for the current right-hand side from x0 = 0.  Replaces
   FFT_Program (CG_Iteration.h:1365-1388) and the driver it dispatches to.
   x (3a complex) may be NULL; the solution also stays on the device. */
VIE_API int vie_solve(vie_ctx* ctx, const vie_solve_params* p, double* x, vie_solve_info* info);
/* Batched solve (no reference counterpart: the reference runs one wavelength
   per process, main.cpp:27-36).  Solves the systems of n distinct contexts on
   the same GPU (each with its own grid, material, Green's function and
   right-hand side: wavelength x polarisation sweeps, uneven particle grids) in
   ONE CUDA graph launch: a device-side WHILE loop whose every pass runs each
   still-unconverged instance's iteration body as a parallel branch; converged
   instances launch nothing.  Same parameters for all instances; precision FP64
   with any solver, or VIE_PREC_MIXED with BiCGSTAB.  Solutions stay in the
   contexts (vie_get_solution); infos (n entries, may be NULL) receive each
   instance's counts, `seconds` being the time of the whole batch.  Returns
   the first non-OK instance status (VIE_ERR_MAXIT if any instance hit its cap). */
VIE_API int vie_solve_batch(vie_ctx* const* ctxs, int n, const vie_solve_params* p, vie_solve_info* infos);
/* Absorbed power in a set of edges and its gradient with respect to the
   per-voxel complex permittivity (no reference counterpart; the objective is
   the absorption sum of NearField, NearFar.h:186-250, restricted to the
   edges whose bit is set in edge_mask: bit f of byte v selects the f-edge of
   voxel v, e.g. Ene_Active = edges whose two voxels are both active, with
   i, j, k < N - 1).  Runs the forward solve with p (J), *power = P, and, if
   grad != NULL, one adjoint solve with the same driver and precision on the
   conjugated source (the operator is complex-symmetric for cubic voxels,
   which this requires) and grad[v] = dP/dRe(eps_v) + i dP/dIm(eps_v) for the
   permittivity in the convention of vie_set_eps (a complex).  The context
   keeps its right-hand side; its solution is the forward field afterwards.
   info_fwd / info_adj (may be NULL) receive the two solves' counts. */
VIE_API int vie_power_grad(vie_ctx* ctx, const unsigned char* edge_mask, const vie_solve_params* p, double* power,
                           double* grad, vie_solve_info* info_fwd, vie_solve_info* info_adj);
/* Geometry on the GPU (GetMaterial / GetFlag, Model.h:305-398, without host
   label evaluation).  A scene is a list of primitives in priority order: the
   label of a point is that of the first primitive holding it whose parent
   (another primitive of the list, or -1) holds it too, else 0 (air): e.g. the
   reference's layered model lists its spheres first with the spacer box as
   parent, then the spacer box, then the active box.  The primitive
   tests are the reference's forms of Model_Identifier (Model.h:215-300):
   VIE_PRIM_SPHERE sqrt(|p - c|^2) <= r (its one-sphere model), VIE_PRIM_SPHERE_F32
   float(|p - c|^2) < float(r^2) (the sphere loop of its layered model) and
   VIE_PRIM_BOX |p_i - c_i| < h_i on every axis (its layers).  Coordinates in
   the grid's units, origin at the grid corner.  Sets the edge flags and the
   permittivity from the table (as vie_set_flags + vie_set_material) and, when
   material_out != NULL, returns the labels (a bytes).  At most 256 primitives. */
#define VIE_PRIM_SPHERE 1
#define VIE_PRIM_SPHERE_F32 2
#define VIE_PRIM_BOX 3
typedef struct {
    int kind;     /* VIE_PRIM_* */
    int label;    /* material index 0..255 */
    int parent;   /* index of another primitive that must also hold the point, or -1 */
    int pad;
    double c[3];  /* centre */
    double r;     /* sphere radius */
    double h[3];  /* box half-widths */
} vie_primitive;
VIE_API int vie_set_geometry_scene(vie_ctx* ctx, const vie_primitive* prims, int n, const double* eps_re,
                                   const double* eps_im, int n_materials, uint8_t* material_out);

/* Post-processing of the last solution on the GPU (the field stays on the
   device).  vie_farfield1 replaces FarField1 (NearFar.h:16-109): Forward_RCS
   for the incidence angles theta, phi, psi (degrees).  vie_farfield2 replaces
   FarField2 (NearFar.h:302-477): the 181 E-plane (phi) and 181 H-plane
   (phi + 90) RCS values in dB, theta = 0..180.  vie_nearfield replaces the
   absorption sums of NearField (NearFar.h:186-250): Ene_Metal, Ene_Active and
   Absorb_Volume from the material labels (2 metal, 3 active; a bytes). */
VIE_API int vie_farfield1(vie_ctx* ctx, double theta, double phi, double psi, double* forward_rcs);
VIE_API int vie_farfield2(vie_ctx* ctx, double phi, double* rcs_theta, double* rcs_phi);
VIE_API int vie_nearfield(vie_ctx* ctx, const uint8_t* material, double* ene_metal, double* ene_active,
                          double* absorb_volume);

/* Autotuner of the FFT schedule (no reference counterpart).  Times, for this
   context's grid, the candidate schedules of each axis (register four-step
   kernels where the length has them; generic shared-memory kernels with the
   default, reversed and 16 -> 4x4 / 8x2 radix orders and pencil tiles around
   the default) and rebuilds the operators with the fastest.  flags: 1 FP64,
   2 FP32 (0: both), 4 tune again even when the process already has a choice
   for this grid.  Choices are shared by every later context with the same
   grid and device in the process, and kept in the text file named by the
   environment variable VIE_TUNE_CACHE when set; VIE_AUTOTUNE=1 tunes each new
   grid automatically.  report (may be NULL) receives a one-line summary.
   Needs vie_set_flags first; results do not depend on the schedule beyond
   rounding. */
VIE_API int vie_autotune(vie_ctx* ctx, int flags, char* report, int report_len);
/* ||b - A x|| / ||b|| of the last solution for the current right-hand side,
   evaluated in FP64 (one operator application). */
VIE_API int vie_residual(vie_ctx* ctx, double* relres);
/* Copy the last solution (Current_X/Y/Z) to the host, 3a complex. */
VIE_API int vie_get_solution(vie_ctx* ctx, double* x);
/* Replace the solution by a given current (3a complex, the layout of
   Current_X/Y/Z), e.g. to post-process a field computed elsewhere. */
VIE_API int vie_set_solution(vie_ctx* ctx, const double* x);
/* Device pointer of the last solution (3a double2), valid until the next solve. */
VIE_API int vie_solution_device(vie_ctx* ctx, const void** x);

/* Device pointers and byte sizes of the context's FP64 right-hand side and
   solution, for callers that keep data on the GPU. */
VIE_API int vie_rhs_device(vie_ctx* ctx, void** rhs);

/* Synchronise the context stream. */
VIE_API int vie_sync(vie_ctx* ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that order their
   own work or record timing events on it. */
VIE_API int vie_stream(vie_ctx* ctx, void** stream);

/* Number of CUDA kernels this library has launched in this process. */
VIE_API long long vie_launch_count(void);

/* Library version string. */
VIE_API const char* vie_version(void);

#ifdef __cplusplus
}
#endif
#endif
