// vie_launch.cuh -- launch of the five operator passes with fused prologue/epilogue.
#pragma once
#include <mutex>
#include <unordered_map>

#include "vie_fast.cuh"
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
    if (bytes <= cur && cur > 0) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    // prefer the largest shared-memory carveout so several CTAs of the pencil passes fit per SM
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    if (e == cudaSuccess) cur = bytes;
    return e;
}
template <typename K> inline cudaError_t ensure_smem(K* kernel, size_t bytes) {
    return ensure_smem(reinterpret_cast<const void*>(kernel), bytes);
}

inline unsigned ceil_div(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

// Number of blocks of the last pass (rows of the reduction partials).
template <typename T> inline long long epilogue_blocks(const Operator<T>& op) {
    using C = cplx_t<T>;
    const long long nrows = (long long)op.dev.nx * op.dev.ny;
    int rows = op.dev.tz;
    if (op.dev.fast[2]) {
        switch (op.dev.nz) {
#define VIE_ROWS_CASE(NN) case NN: rows = fast_rows<C, NN>(); break;
            VIE_FAST_LENGTHS(VIE_ROWS_CASE)
#undef VIE_ROWS_CASE
        }
    }
    return (long long)ceil_div(nrows, rows) * 3;
}

// fast z passes for a compile-time N
template <typename T, int N, class Pro, class Epi>
int launch_fast_z(Operator<T>& op, bool forward, Pro pro, Epi epi, const cplx_t<T>* xdiag, bool conj,
                  double2* partial, cudaStream_t st, Error& err) {
    using C = cplx_t<T>;
    constexpr int ROWS = fast_rows<C, N>(), L = fast_lanes<C, N>();
    constexpr size_t smem = fast_smem_row<C, N>();
    const long long nrows = (long long)op.dev.nx * op.dev.ny;
    dim3 grid(ceil_div(nrows, ROWS), 3);
    if (forward) {
        auto kf = kf_fwd_z<C, N, Pro>;
        VIE_CUDA_TRY(ensure_smem(kf, smem), err);
        kf<<<grid, L * ROWS, smem, st>>>(op.dev, pro);
        count_launch();
    } else {
        auto kf = kf_inv_z<C, N, Epi>;
        VIE_CUDA_TRY(ensure_smem(kf, smem), err);
        kf<<<grid, L * ROWS, smem, st>>>(op.dev, xdiag, epi, partial, conj ? 1 : 0);
        count_launch();
    }
    return VIE_OK;
}

template <typename T, int N>
int launch_fast_y(Operator<T>& op, bool forward, cudaStream_t st, Error& err) {
    using C = cplx_t<T>;
    constexpr int TP = FastTiles<C>::TP_Y, L = fast_lanes<C, N>();
    constexpr size_t smem = fast_smem_col<C, N>();
    dim3 grid(ceil_div(2 * op.dev.nz, TP), op.dev.nx, 3);
    if (op.use_ytma && op.dev.b == op.tm_b_addr && op.dev.c == op.tm_c_addr) {
        // tiles staged by TMA (default; the autotuner may switch it off); 128 more
        // bytes of shared memory to align the destination
        auto kt = forward ? kf_fwd_y_tma<C, N> : kf_inv_y_tma<C, N>;
        VIE_CUDA_TRY(ensure_smem(kt, smem + 128), err);
        kt<<<grid, TP * L, smem + 128, st>>>(op.dev, forward ? op.tm_b : op.tm_c);
        count_launch();
        return VIE_OK;
    }
    auto kf = forward ? kf_fwd_y<C, N> : kf_inv_y<C, N>;
    VIE_CUDA_TRY(ensure_smem(kf, smem), err);
    kf<<<grid, TP * L, smem, st>>>(op.dev);
    count_launch();
    return VIE_OK;
}

template <typename T, int N, int TP>
int launch_fast_x_tp(Operator<T>& op, bool conj, cudaStream_t st, Error& err) {
    using C = cplx_t<T>;
    constexpr size_t smem = fast_smem_x<C, N, TP>();
    dim3 grid(ceil_div(2 * op.dev.nz, TP), 2 * op.dev.ny);
    auto kf = kf_x_spectral<C, N, TP>;
    VIE_CUDA_TRY(ensure_smem(kf, smem), err);
    kf<<<grid, fast_x_threads<C, N, TP>(), smem, st>>>(op.dev, conj ? 1 : 0);
    count_launch();
    return VIE_OK;
}
// the x pass with the operator's tile choice (OpDev::xalt: 0 default, 1 half)
template <typename T, int N>
int launch_fast_x(Operator<T>& op, bool conj, cudaStream_t st, Error& err) {
    using C = cplx_t<T>;
    if (op.dev.xalt) return launch_fast_x_tp<T, N, FastTiles<C>::TP_X / 2>(op, conj, st, err);
    return launch_fast_x_tp<T, N, FastTiles<C>::TP_X>(op, conj, st, err);
}

#define VIE_FAST_SWITCH(n, CALL)                                   \
    switch (n) {                                                    \
        case 256: { constexpr int NN = 256; CALL; } break;          \
        case 192: { constexpr int NN = 192; CALL; } break;          \
        case 176: { constexpr int NN = 176; CALL; } break;          \
        case 160: { constexpr int NN = 160; CALL; } break;          \
        case 144: { constexpr int NN = 144; CALL; } break;          \
        case 128: { constexpr int NN = 128; CALL; } break;          \
        case 120: { constexpr int NN = 120; CALL; } break;          \
        case 112: { constexpr int NN = 112; CALL; } break;          \
        case 96: { constexpr int NN = 96; CALL; } break;            \
        case 88: { constexpr int NN = 88; CALL; } break;            \
        case 80: { constexpr int NN = 80; CALL; } break;            \
        case 72: { constexpr int NN = 72; CALL; } break;            \
        case 64: { constexpr int NN = 64; CALL; } break;            \
        case 56: { constexpr int NN = 56; CALL; } break;            \
        case 48: { constexpr int NN = 48; CALL; } break;            \
        case 40: { constexpr int NN = 40; CALL; } break;            \
        case 32: { constexpr int NN = 32; CALL; } break;            \
        case 24: { constexpr int NN = 24; CALL; } break;            \
        case 16: { constexpr int NN = 16; CALL; } break;            \
        default: break;                                             \
    }

// y = A x (or A^H x) with a prologue producing the source values and an
// epilogue consuming the outputs.  xdiag is the source vector the diagonal
// term reads (the same values the prologue returns where valid).  Each axis
// runs the register four-step kernels when its length is one of the
// compile-time lengths, the generic shared-memory kernels otherwise.
template <typename T, class Pro, class Epi>
int launch_operator(Operator<T>& op, Pro pro, Epi epi, const cplx_t<T>* xdiag, bool conj, double2* partial,
                    cudaStream_t st, Error& err) {
    using C = cplx_t<T>;
    const OpDev<C>& d = op.dev;
    const long long nrows = (long long)d.nx * d.ny;
    const int Lz = 2 * d.nz, Ly = 2 * d.ny;
    int rc = VIE_OK;
    // F1
    if (d.fast[2]) {
        VIE_FAST_SWITCH(d.nz, rc = (launch_fast_z<T, NN, Pro, Epi>(op, true, pro, epi, xdiag, conj, partial, st, err)));
    } else {
        auto kf = k_fwd_z<C, Pro>;
        VIE_CUDA_TRY(ensure_smem(kf, op.smem_z), err);
        kf<<<dim3(ceil_div(nrows, d.tz), 3), kThreads, op.smem_z, st>>>(d, pro);
        count_launch();
    }
    if (rc) return rc;
    // F2
    if (d.fast[1]) {
        VIE_FAST_SWITCH(d.ny, rc = (launch_fast_y<T, NN>(op, true, st, err)));
    } else {
        auto kf = k_fwd_y<C>;
        VIE_CUDA_TRY(ensure_smem(kf, op.smem_y), err);
        kf<<<dim3(ceil_div(Lz, d.tc), d.nx, 3), kThreads, op.smem_y, st>>>(d);
        count_launch();
    }
    if (rc) return rc;
    // F3
    if (d.fast[0]) {
        VIE_FAST_SWITCH(d.nx, rc = (launch_fast_x<T, NN>(op, conj, st, err)));
    } else if (conj) {
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
    if (rc) return rc;
    // I2
    if (d.fast[1]) {
        VIE_FAST_SWITCH(d.ny, rc = (launch_fast_y<T, NN>(op, false, st, err)));
    } else {
        auto kf = k_inv_y<C>;
        VIE_CUDA_TRY(ensure_smem(kf, op.smem_y), err);
        kf<<<dim3(ceil_div(Lz, d.tc), d.nx, 3), kThreads, op.smem_y, st>>>(d);
        count_launch();
    }
    if (rc) return rc;
    // I1
    if (d.fast[2]) {
        VIE_FAST_SWITCH(d.nz, rc = (launch_fast_z<T, NN, Pro, Epi>(op, false, pro, epi, xdiag, conj, partial, st, err)));
    } else if (conj) {
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
    if (rc) return rc;
    VIE_CUDA_TRY(cudaGetLastError(), err);
    return VIE_OK;
}

}  // namespace vie
