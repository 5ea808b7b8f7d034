/*
 * fft.h -- drop-in replacement of the reference's vie_fft/fft.h (same include
 * guard, names and signatures).  Every block runs on the B200 library; the
 * Green argument is not read because the library keeps the spectrum computed
 * by Green_Function_Compute on the GPU.
 *
 *   Current_Reset        (fft.h:13-35)    vie_reset
 *   L_DC_Dq[_Conjugate]  (fft.h:41-219)   vie_apply, Green part, one source
 *   L_Dq[_Conjugate]     (fft.h:224-397)  vie_apply, Green part, one source
 *   LXX/LYY/LZZ_DO[_Conjugate] (fft.h:405-624) vie_apply, diagonal part
 *
 * The reference calls the FFT blocks on an expanded current (Current_Expansion,
 * CG_Iteration.h:50-83): only its (Nx, Ny, Nz) corner can be non-zero, and the
 * block leaves the transformed array in `current_xyz` as scratch that no caller
 * reads.  The replacements read that corner and leave `current_xyz` unchanged.
 */
#ifndef FFT_SW
#define FFT_SW

#include "Model.h"
#include "vie_dropin.h"

namespace vie_dropin {

// the (Nx, Ny, Nz) corner of a (2Nx, 2Ny, 2Nz) array as component `comp` of a 3-vector
inline void corner_as_component(std::vector<double>& v, MKL_Complex16*** padded, int comp) {
    const size_t a = (size_t)voxels();
    v.assign(6 * a, 0.0);
    double* d = v.data() + 2 * a * comp;
    for (int i = 0; i < Nx; i++)
        for (int j = 0; j < Ny; j++)
            std::memcpy(d + 2 * ((size_t)i * Ny + j) * Nz, padded[i][j], 16 * (size_t)Nz);
}

inline void block(MKL_Complex16*** field, MKL_Complex16*** padded, int src, int fld, int conj, int parts) {
    vie_ctx* c = context();
    std::vector<double> x, y(6 * (size_t)voxels());
    corner_as_component(x, padded, src);
    check(vie_apply(c, x.data(), y.data(), conj, parts), "vie_apply");
    add_component(field, y, fld);
}

}  // namespace vie_dropin

void Current_Reset(MKL_Complex16*** Current, const int Flag, const int* Dim) {
    (void)Dim;
    vie_dropin::check(vie_reset(vie_dropin::context(), reinterpret_cast<double*>(Current[0][0]), Flag), "vie_reset");
}

void L_DC_Dq(MKL_Complex16*** temp_xyz, MKL_Complex16*** current_xyz, MKL_Complex16*** const Green,
             const double delta_xyz, const int Index_Source, const int* Dim) {
    (void)Green; (void)delta_xyz; (void)Dim;
    vie_dropin::block(temp_xyz, current_xyz, Index_Source, Index_Source, 0, VIE_PART_GREEN);
}

void L_DC_Dq_Conjugate(MKL_Complex16*** temp_xyz, MKL_Complex16*** current_xyz, MKL_Complex16*** const Green,
                       const double delta_xyz, const int Index_Source, const int* Dim) {
    (void)Green; (void)delta_xyz; (void)Dim;
    vie_dropin::block(temp_xyz, current_xyz, Index_Source, Index_Source, 1, VIE_PART_GREEN);
}

void L_Dq(MKL_Complex16*** temp_xyz, MKL_Complex16*** current_xyz, MKL_Complex16*** const Green,
          const int Index_Source, const int Index_Field, const double delta_xyz_source, const int* Dim) {
    (void)Green; (void)delta_xyz_source; (void)Dim;
    vie_dropin::block(temp_xyz, current_xyz, Index_Source, Index_Field, 0, VIE_PART_GREEN);
}

void L_Dq_Conjugate(MKL_Complex16*** temp_xyz, MKL_Complex16*** current_xyz, MKL_Complex16*** const Green,
                    const int Index_Source, const int Index_Field, const double delta_xyz_field, const int* Dim) {
    (void)Green; (void)delta_xyz_field; (void)Dim;
    vie_dropin::block(temp_xyz, current_xyz, Index_Source, Index_Field, 1, VIE_PART_GREEN);
}

// diagonal (non-FFT) terms of one component, on the expanded current
#define VIE_DROPIN_DIAG(NAME, COMP, CONJ)                                                     \
    void NAME(MKL_Complex16*** temp, MKL_Complex16*** current, const int* Dim) {             \
        (void)Dim;                                                                            \
        vie_dropin::block(temp, current, COMP, COMP, CONJ, VIE_PART_DIAG);                    \
    }
VIE_DROPIN_DIAG(LXX_DO, 0, 0)
VIE_DROPIN_DIAG(LXX_DO_Conjugate, 0, 1)
VIE_DROPIN_DIAG(LYY_DO, 1, 0)
VIE_DROPIN_DIAG(LYY_DO_Conjugate, 1, 1)
VIE_DROPIN_DIAG(LZZ_DO, 2, 0)
VIE_DROPIN_DIAG(LZZ_DO_Conjugate, 2, 1)
#undef VIE_DROPIN_DIAG

#endif
