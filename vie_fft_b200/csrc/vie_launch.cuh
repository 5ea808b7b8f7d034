// vie_launch.cuh -- launch of the five operator passes with fused prologue/epilogue.
#pragma once
#include <mutex>
#include <unordered_map>

#include "vie_internal.h"

namespace vie {

// Raise the dynamic shared-memory cap of one kernel once per larger size
// (cudaFuncSetAttribute is per function; the cache is keyed by the kernel's
// address and device).
inline cudaError_t ensure_smem(const void* kernel, size_t bytes) {
    static std::mutex mu;
    static std::unordered_map<const void*, size_t> set_bytes[64];
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    size_t& cur = set_bytes[dev & 63][kernel];
    if (bytes <= cur) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}
template <typename K> inline cudaError_t ensure_smem(K* kernel, size_t bytes) {
    return ensure_smem(reinterpret_cast<const void*>(kernel), bytes);
}

inline unsigned ceil_div(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

// Number of blocks of the last pass (rows of the reduction partials).
template <typename T> inline long long epilogue_blocks(const Operator<T>& op) {
    return (long long)ceil_div((long long)op.dev.nx * op.dev.ny, op.dev.tz) * 3;
}

// y = A x (or A^H x) with a prologue producing the source values and an
// epilogue consuming the outputs.  xdiag is the source vector the diagonal
// term reads (the same values the prologue returns where valid).
template <typename T, class Pro, class Epi>
int launch_operator(Operator<T>& op, Pro pro, Epi epi, const cplx_t<T>* xdiag, bool conj, double2* partial,
                    cudaStream_t st, Error& err) {
    using C = cplx_t<T>;
    const OpDev<C>& d = op.dev;
    const long long nrows = (long long)d.nx * d.ny;
    const int Lz = 2 * d.nz, Ly = 2 * d.ny;
    {
        auto kf = k_fwd_z<C, Pro>;
        VIE_CUDA_TRY(ensure_smem(kf, op.smem_z), err);
        kf<<<dim3(ceil_div(nrows, d.tz), 3), kThreads, op.smem_z, st>>>(d, pro);
        count_launch();
    }
    {
        auto kf = k_fwd_y<C>;
        VIE_CUDA_TRY(ensure_smem(kf, op.smem_y), err);
        kf<<<dim3(ceil_div(Lz, d.tc), d.nx, 3), kThreads, op.smem_y, st>>>(d);
        count_launch();
    }
    if (conj) {
        auto kf = k_x_spectral<C, true>;
        VIE_CUDA_TRY(ensure_smem(kf, op.smem_x), err);
        kf<<<dim3(ceil_div(Lz, d.tx), Ly), kThreads, op.smem_x, st>>>(d);
        count_launch();
    } else {
        auto kf = k_x_spectral<C, false>;
        VIE_CUDA_TRY(ensure_smem(kf, op.smem_x), err);
        kf<<<dim3(ceil_div(Lz, d.tx), Ly), kThreads, op.smem_x, st>>>(d);
        count_launch();
    }
    {
        auto kf = k_inv_y<C>;
        VIE_CUDA_TRY(ensure_smem(kf, op.smem_y), err);
        kf<<<dim3(ceil_div(Lz, d.tc), d.nx, 3), kThreads, op.smem_y, st>>>(d);
        count_launch();
    }
    if (conj) {
        auto kf = k_inv_z<C, true, Epi>;
        VIE_CUDA_TRY(ensure_smem(kf, op.smem_z), err);
        kf<<<dim3(ceil_div(nrows, d.tz), 3), kThreads, op.smem_z, st>>>(d, xdiag, epi, partial);
        count_launch();
    } else {
        auto kf = k_inv_z<C, false, Epi>;
        VIE_CUDA_TRY(ensure_smem(kf, op.smem_z), err);
        kf<<<dim3(ceil_div(nrows, d.tz), 3), kThreads, op.smem_z, st>>>(d, xdiag, epi, partial);
        count_launch();
    }
    VIE_CUDA_TRY(cudaGetLastError(), err);
    return VIE_OK;
}

}  // namespace vie
