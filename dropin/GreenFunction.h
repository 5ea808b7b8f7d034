/*
 * GreenFunction.h -- drop-in replacement of the reference's vie_fft/GreenFunction.h
 * (same include guard, same functions, same globals contract) running on the
 * B200 library (include/vie_b200.h).
 *
 *   Green_Function_Compute (GreenFunction.h:8-141): the scalar Green's
 *     function with its singular self term, the even extension and the forward
 *     transform, computed on the GPU in FP64; the (2Nx, 2Ny, 2Nz) spectrum is
 *     copied into the global Green_Function as the reference leaves it.
 *   Incident_Wave (GreenFunction.h:144-248): the edge-integrated plane wave on
 *     the staggered grids, computed on the GPU in FP64, into Ex/Ey/Ez_inc.
 */
#ifndef GREENFUNCTION
#define GREENFUNCTION

#include "Model.h"
#include "vie_dropin.h"

void Green_Function_Compute() {
    vie_ctx* c = vie_dropin::context();
    vie_dropin::upload_geometry(c);
    vie_dropin::check(vie_green(c), "vie_green");
    vie_dropin::check(vie_green_spectrum(c, reinterpret_cast<double*>(Green_Function[0][0])), "vie_green_spectrum");
}

void Incident_Wave() {
    vie_ctx* c = vie_dropin::context();
    std::vector<double> e(6 * (size_t)vie_dropin::voxels());
    vie_dropin::check(vie_incident(c, Theta, Phi, Psi, e.data()), "vie_incident");
    vie_dropin::scatter(e, Ex_inc, Ey_inc, Ez_inc);
}

#endif
