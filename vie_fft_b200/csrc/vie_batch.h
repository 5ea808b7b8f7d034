// vie_batch.h -- the persistent multi-instance loop of batched mixed-precision
// BiCGSTAB solves (vie_solve_batch), host side.
#pragma once
#include <vector>

#include "vie_internal.h"

namespace vie {

// One instance of a batch after its set-up (solve_bicgstab_mixed with a plan):
// the device vectors, scalars, reduction partials and control block of its
// context, and copies of its two operators' device views.
struct FusedInstance {
    vie_ctx* ctx = nullptr;
    OpDev<float2> op32{};
    OpDev<double2> op64{};
    long long a = 0;
    float2 *r = nullptr, *p = nullptr, *v = nullptr, *sv = nullptr, *t = nullptr, *x32 = nullptr, *b32 = nullptr;
    double2 *r64 = nullptr, *b64 = nullptr, *x64 = nullptr;
    double2* S = nullptr;
    double2* partial = nullptr;
    KCtl* ctl = nullptr;
    double2* hist = nullptr;
};

// both operators of the context run every axis on the register kernels
bool batch_fused_eligible(const vie_ctx* ctx);

// Runs the iterations of every instance to its own stop in one graph launch on
// stream S.  launched is false when the graph could not be built (nothing ran).
// Each instance's control block holds its outcome afterwards.
int batch_fused_loop(std::vector<FusedInstance>& inst, cudaStream_t S, vie_ctx* ectx, bool& launched);

}  // namespace vie
