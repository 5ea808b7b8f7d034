// vie_static_scratch.cu -- an operator application that allocates no device memory.
//
// vie_matvec allocates device copies of its input and output on every call and
// the operator's five passes use the context's scratch spectra.  Some callers
// must not allocate device memory while they apply the operator: a host program
// that applies it inside a long outer loop cannot afford the cudaMalloc/cudaFree
// pair per call (cudaFree synchronises the whole device and stalls every other
// stream), and a process whose free device memory is held by another allocator
// (PyTorch's caching allocator, or a solve that sized its Krylov workspace to the
// card) can see a fresh cudaMalloc fail.  vie_matvec_static serves them: the
// device copies of x and y and the b/c scratch spectra all live in one
// file-scope __device__ array of kStaticBytes (64 MiB) that every GPU which
// loads this library holds until the process exits.
//
// Limits and sharing:
//   * the grid must fit: 384 bytes per voxel (x, y: 48 each; b: 96; c: 192),
//     i.e. at most 174762 voxels (about 55^3); larger grids get VIE_ERR_ARG;
//   * every call on a device uses the same array and leaves the last call's data
//     in it.  Nothing needs to start at zero: the input copy, both scratch
//     spectra and the output are overwritten entirely by each call.  Calls that
//     overlap on one GPU (two host threads with contexts on the same device)
//     race on the array and must be serialised by the caller;
//   * the first call on a device looks up the device address of the array
//     (cudaGetSymbolAddress, with that device current); make that first call
//     before any stream capture that might include later calls.
#include <mutex>

#include "vie_launch.cuh"

namespace {

constexpr size_t kStaticBytes = 64ull << 20;
constexpr int kMaxDevices = 128;

__device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];

// Device address of g_static_scratch per device.  In host code the symbol name
// is only a host-side stand-in: passing it to a kernel would fault (or silently
// use host memory), so kernels get the address looked up here.
std::mutex g_addr_mu;
void* g_addr[kMaxDevices] = {};

int static_scratch_address(vie_ctx* ctx, void** out) {
    if (ctx->device < 0 || ctx->device >= kMaxDevices)
        return ctx->set_error(VIE_ERR_ARG, "vie_matvec_static: device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_addr_mu);
    if (!g_addr[ctx->device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);  // device is current (set by the caller)
        if (e != cudaSuccess || !p)
            return ctx->set_error(VIE_ERR_CUDA, std::string("vie_matvec_static: cudaGetSymbolAddress: ") +
                                                    cudaGetErrorString(e));
        g_addr[ctx->device] = p;
    }
    *out = g_addr[ctx->device];
    return VIE_OK;
}

}  // namespace

extern "C" int vie_matvec_static(vie_ctx* ctx, const double* x, double* y, int conj) {
    using namespace vie;
    if (!ctx || !x || !y) return VIE_ERR_ARG;
    if (int u = ctx->check_usable()) return u;
    if (!ctx->have_flags) return ctx->set_error(VIE_ERR_STATE, "edge flags not set (vie_set_flags)");
    if (!ctx->have_eps) return ctx->set_error(VIE_ERR_STATE, "permittivity not set (vie_set_material / vie_set_eps)");
    if (!ctx->have_green) return ctx->set_error(VIE_ERR_STATE, "Green's function not computed (vie_green)");
    const long long a = ctx->a;
    const size_t vec = align_up(sizeof(double2) * 3 * (size_t)a, 256);
    const size_t bb = align_up(sizeof(double2) * 3 * (size_t)ctx->nx * ctx->ny * 2 * ctx->nz, 256);
    const size_t cb = align_up(sizeof(double2) * 3 * (size_t)ctx->nx * 2 * ctx->ny * 2 * ctx->nz, 256);
    const size_t need = 2 * vec + bb + cb;
    if (need > kStaticBytes)
        return ctx->set_error(VIE_ERR_ARG, "vie_matvec_static: a grid of " + std::to_string(a) + " voxels needs " +
                                               std::to_string(need) + " bytes; the static scratch holds " +
                                               std::to_string(kStaticBytes) + " bytes (at most " +
                                               std::to_string(kStaticBytes / 384) + " voxels)");
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return ctx->set_error(VIE_ERR_CUDA, cudaGetErrorString(e));
    void* base = nullptr;
    int rc = static_scratch_address(ctx, &base);
    if (rc) return rc;
    unsigned char* p = static_cast<unsigned char*>(base);
    double2* dx = reinterpret_cast<double2*>(p);
    double2* dy = reinterpret_cast<double2*>(p + vec);
    // the context's FP64 operator with its b/c scratch redirected into the array
    Operator<double> op = ctx->op64;
    op.owns_scratch = false;
    op.d_b = reinterpret_cast<double2*>(p + 2 * vec);
    op.d_c = reinterpret_cast<double2*>(p + 2 * vec + bb);
    op.dev.b = op.d_b;
    op.dev.c = op.d_c;
    const size_t bytes = sizeof(double2) * 3 * (size_t)a;
    e = cudaMemcpyAsync(dx, x, bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) return ctx->set_error(VIE_ERR_CUDA, cudaGetErrorString(e));
    rc = launch_operator<double>(op, ProCopy<double2>{dx, a}, EpiStore<double2>{dy, a}, dx, conj != 0, nullptr,
                                 ctx->stream, ctx->err);
    if (!rc) {
        e = cudaMemcpyAsync(y, dy, bytes, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = ctx->set_error(VIE_ERR_CUDA, cudaGetErrorString(e));
    } else {
        cudaStreamSynchronize(ctx->stream);  // the passes already enqueued finish before the status word is read
    }
    // the z passes stage their rows on bounded waits that report through the
    // FP64 operator's status word (shared with this copy of the operator): a
    // wait that ran out left part of y undone, which is an error of this call
    return ctx->check_waits(rc);
}
