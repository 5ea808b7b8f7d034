/*
 * CG_Iteration.h -- drop-in replacement of the reference's vie_fft/CG_Iteration.h
 * (same include guard, globals, constants, names and signatures) running on the
 * B200 library (include/vie_b200.h).
 *
 *   Current_Expansion (CG_Iteration.h:50-83)  zero (2N)^3, copy the valid block
 *   X/Y/Z_FFT[_Conjugate] (:86-173)           one row block of A (or A^H), no reset
 *   CG_FFT, BICG_FFT, BICGSTAB_FFT, CORS_FFT, BICORSTAB_FFT (:176-1362)
 *                                            the solve on the GPU (vie_solve)
 *   FFT_Program (:1365-1388)                  dispatch on Iteration_Type
 *
 * The drivers keep the reference's contract: x0 = 0, right-hand side E_inc
 * masked by the edge flags, the threshold CG_THR on the same error measure,
 * "CG Error" / "Steps" lines on stdout, the solution in Current_X/Y/Z, and
 * Ex/Ey/Ez_inc, Green_Function and Flag_X/Y/Z released at the end
 * (CG_Iteration.h:769-775).  Differences: the iteration cap nx*ny*nz ends the
 * solve with a warning on stderr (the reference stops silently there), and a
 * Krylov breakdown (a zero or non-finite scalar, which the reference would
 * carry as NaN up to the cap) stops the program with a message.
 * VIE_PRECISION=mixed in the environment selects the FP32/FP64 solve.
 */
#ifndef CG_ITERATION
#define CG_ITERATION

#include "fft.h"

// iterative variables of the reference (CG_Iteration.h:11-43); the GPU solve
// keeps its vectors on the device, these stay unallocated
MKL_Complex16*** Temp_Current;
MKL_Complex16 ***Apx, ***Apy, ***Apz, ***Aqx, ***Aqy, ***Aqz;
MKL_Complex16 ***q1x, ***q1y, ***q1z, ***p1x, ***p1y, ***p1z, ***r0x, ***r0y, ***r0z;
MKL_Complex16 ***q1x_c, ***q1y_c, ***q1z_c, ***p1x_c, ***p1y_c, ***p1z_c, ***r0x_c, ***r0y_c, ***r0z_c;
unsigned char*** Pre_Flag;   // preconditioner flag (unused, as in the reference)
const double CG_THR = 0.001;  // threshold (CG_Iteration.h:46)
const int Iteration_Type = 3; // 1 CG, 2 BICG, 3 BICGSTAB, 4 CORS, 5 BICORSTAB (CG_Iteration.h:47)

// expand currents (CG_Iteration.h:50-83): data staging only
void Current_Expansion(MKL_Complex16*** Temp_Current_V, MKL_Complex16*** const Current, int Flag, const int* Dim) {
    std::memset(Temp_Current_V[0][0], 0, sizeof(MKL_Complex16) * 8 * (size_t)Dim[0] * Dim[1] * Dim[2]);
    int lim[3] = {Dim[0], Dim[1], Dim[2]};
    lim[Flag] -= 1;
    for (int i = 0; i < lim[0]; i++)
        for (int j = 0; j < lim[1]; j++)
            std::memcpy(Temp_Current_V[i][j], Current[i][j], sizeof(MKL_Complex16) * (size_t)lim[2]);
}

namespace vie_dropin {

inline void row_block(MKL_Complex16*** Field, MKL_Complex16*** Sx, MKL_Complex16*** Sy, MKL_Complex16*** Sz,
                      int row, int conj) {
    vie_ctx* c = context();
    std::vector<double> x, y(6 * (size_t)voxels());
    gather(x, Sx, Sy, Sz);
    check(vie_apply(c, x.data(), y.data(), conj, VIE_PART_GREEN | VIE_PART_DIAG), "vie_apply");
    add_component(Field, y, row);
}

inline void run_driver(int solver) {
    vie_ctx* c = context();
    upload_geometry(c);
    std::vector<double> e, x(6 * (size_t)voxels());
    gather(e, Ex_inc, Ey_inc, Ez_inc);
    check(vie_set_rhs(c, e.data()), "vie_set_rhs");
    vie_solve_params p;
    std::memset(&p, 0, sizeof(p));
    p.solver = solver;
    const char* prec = std::getenv("VIE_PRECISION");
    p.precision = (prec && std::strcmp(prec, "mixed") == 0) ? VIE_PREC_MIXED : VIE_PREC_FP64;
    p.tol = CG_THR;
    p.max_iter = 0;
    p.verbose = std::getenv("VIE_QUIET") ? 0 : 1;
    vie_solve_info info;
    int rc = vie_solve(c, &p, x.data(), &info);
    if (rc == VIE_ERR_MAXIT)
        std::fprintf(stderr, "vie_b200: iteration cap reached (relative residual %g)\n", info.relres);
    else
        check(rc, "vie_solve");
    scatter(x, Current_X, Current_Y, Current_Z);
    // the drivers release these (CG_Iteration.h:769-775)
    RMemory3D(Ex_inc);
    RMemory3D(Ey_inc);
    RMemory3D(Ez_inc);
    RMemory3D(Green_Function);
    RMemory3D(Flag_X);
    RMemory3D(Flag_Y);
    RMemory3D(Flag_Z);
}

}  // namespace vie_dropin

#define VIE_DROPIN_ROW(NAME, ROW, CONJ)                                                                         \
    void NAME(MKL_Complex16*** Field, MKL_Complex16*** const Sourx, MKL_Complex16*** const Soury,              \
              MKL_Complex16*** const Sourz, MKL_Complex16*** temp, MKL_Complex16*** const Green, const int* Dim) { \
        (void)temp; (void)Green; (void)Dim;                                                                     \
        vie_dropin::row_block(Field, Sourx, Soury, Sourz, ROW, CONJ);                                           \
    }
VIE_DROPIN_ROW(X_FFT_Conjugate, 0, 1)
VIE_DROPIN_ROW(Y_FFT_Conjugate, 1, 1)
VIE_DROPIN_ROW(Z_FFT_Conjugate, 2, 1)
VIE_DROPIN_ROW(X_FFT, 0, 0)
VIE_DROPIN_ROW(Y_FFT, 1, 0)
VIE_DROPIN_ROW(Z_FFT, 2, 0)
#undef VIE_DROPIN_ROW

void CG_FFT() { vie_dropin::run_driver(VIE_SOLVER_CG); }
void BICG_FFT() { vie_dropin::run_driver(VIE_SOLVER_BICG); }
void BICGSTAB_FFT() { vie_dropin::run_driver(VIE_SOLVER_BICGSTAB); }
void CORS_FFT() { vie_dropin::run_driver(VIE_SOLVER_CORS); }
void BICORSTAB_FFT() { vie_dropin::run_driver(VIE_SOLVER_BICORSTAB); }

// VIE-FFT program (CG_Iteration.h:1365-1388)
void FFT_Program() {
    if (Iteration_Type == 1) CG_FFT();
    else if (Iteration_Type == 2) BICG_FFT();
    else if (Iteration_Type == 3) BICGSTAB_FFT();
    else if (Iteration_Type == 4) CORS_FFT();
    else BICORSTAB_FFT();
}

#endif
