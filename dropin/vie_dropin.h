/*
 * vie_dropin.h -- shared state of the drop-in headers GreenFunction.h, fft.h and
 * CG_Iteration.h: one library context for the current grid of the reference's
 * globals (Model.h:13-46), rebuilt when the grid, the cell sizes or k0 change.
 *
 * Status handling: the reference checks no status; here any failing library
 * call prints its message to stderr and exits with status 1.
 */
#ifndef VIE_DROPIN_H
#define VIE_DROPIN_H

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "Model.h"
#include "vie_b200.h"

namespace vie_dropin {

inline vie_ctx*& ctx_ref() {
    static vie_ctx* c = nullptr;
    return c;
}

inline void check(int rc, const char* what) {
    if (rc != VIE_OK) {
        std::fprintf(stderr, "vie_b200: %s failed: %s (%s)\n", what, vie_status_string(rc),
                     ctx_ref() ? vie_last_error(ctx_ref()) : "");
        std::exit(1);
    }
}

// The context for the current globals; geometry and materials are uploaded on
// every call because GetMaterial / GetFlag may have changed them.
inline vie_ctx* context() {
    static int gx = 0, gy = 0, gz = 0;
    static double gdx = 0, gdy = 0, gdz = 0, gk0 = 0;
    vie_ctx*& c = ctx_ref();
    if (!c || gx != Nx || gy != Ny || gz != Nz || gdx != delta_x || gdy != delta_y || gdz != delta_z || gk0 != k0) {
        if (c) vie_destroy(c);
        c = nullptr;
        vie_grid g;
        g.nx = Nx; g.ny = Ny; g.nz = Nz;
        g.dx = delta_x; g.dy = delta_y; g.dz = delta_z;
        g.k0 = k0;
        g.device = std::getenv("VIE_DEVICE") ? std::atoi(std::getenv("VIE_DEVICE")) : 0;
        check(vie_create(&g, &c), "vie_create");
        gx = Nx; gy = Ny; gz = Nz; gdx = delta_x; gdy = delta_y; gdz = delta_z; gk0 = k0;
    }
    return c;
}

// Flags and materials from the reference's globals (Model.h:17, 21-23, 81-83).
inline void upload_geometry(vie_ctx* c) {
    check(vie_set_flags(c, Flag_X[0][0], Flag_Y[0][0], Flag_Z[0][0]), "vie_set_flags");
    check(vie_set_material(c, Material[0][0], Real_EPR, Imag_EPR, NUM_DIE), "vie_set_material");
}

inline long long voxels() { return (long long)Nx * Ny * Nz; }

// 3-component vector <-> three Memory3D arrays
inline void gather(std::vector<double>& v, MKL_Complex16*** x, MKL_Complex16*** y, MKL_Complex16*** z) {
    const size_t a = (size_t)voxels();
    v.resize(6 * a);
    std::memcpy(v.data(), x[0][0], 16 * a);
    std::memcpy(v.data() + 2 * a, y[0][0], 16 * a);
    std::memcpy(v.data() + 4 * a, z[0][0], 16 * a);
}

inline void scatter(const std::vector<double>& v, MKL_Complex16*** x, MKL_Complex16*** y, MKL_Complex16*** z) {
    const size_t a = (size_t)voxels();
    std::memcpy(x[0][0], v.data(), 16 * a);
    std::memcpy(y[0][0], v.data() + 2 * a, 16 * a);
    std::memcpy(z[0][0], v.data() + 4 * a, 16 * a);
}

// component `comp` of y added to field (the blocks accumulate, fft.h:113-123)
inline void add_component(MKL_Complex16*** field, const std::vector<double>& y, int comp) {
    const size_t a = (size_t)voxels();
    double* f = reinterpret_cast<double*>(field[0][0]);
    const double* s = y.data() + 2 * a * comp;
    for (size_t i = 0; i < 2 * a; i++) f[i] += s[i];
}

}  // namespace vie_dropin

#endif
