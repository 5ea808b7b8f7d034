// vie_internal.h -- host-side structures of the VIE library (not part of the ABI).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/vie_b200.h"
#include "vie_operator.cuh"

namespace vie {

// Kernel launches issued by this library in this process (every <<<>>> site
// adds to it right after the launch).
extern std::atomic<long long> g_launches;
inline void count_launch(long long n = 1) { g_launches.fetch_add(n, std::memory_order_relaxed); }

constexpr double kPI = 3.1415926535897932384626433832795;  // common.h:17
constexpr double kZ0 = 120 * kPI;                            // common.h:18

struct Error {
    int code = VIE_OK;
    std::string msg;
};

#define VIE_CUDA_TRY(expr, errobj)                                                        \
    do {                                                                                  \
        cudaError_t e__ = (expr);                                                         \
        if (e__ != cudaSuccess) {                                                         \
            (errobj).code = VIE_ERR_CUDA;                                                 \
            (errobj).msg = std::string(#expr) + ": " + cudaGetErrorString(e__);          \
            return VIE_ERR_CUDA;                                                          \
        }                                                                                 \
    } while (0)

// Radix plan for a length-n transform; an empty override means the default
// greedy factorisation (16, 8, 4, 2, 3, 5, 7, then any prime).
AxisPlan make_axis_plan(int n, const std::vector<int>& override_radices = {});
// DIF output position of every index (perm[m]) for a plan.
std::vector<int> axis_perm(const AxisPlan& pl);

// Tile sizes of the five passes for one precision.
struct TileCfg {
    int tz = 0, tc = 0, tx = 0;
    int fast[3] = {-1, -1, -1};  // per axis: 1 register four-step kernels, 0 generic, -1 automatic
    int xalt = 0;                // register x pass with the half pencil tile
    int ytma = 1;                // register y passes with their tiles staged by TMA (0: plain loads)
    int zstage = 1;              // register z passes stage their rows with bulk copies (0: element loads)
    int wait_test = 0;           // 1: staged tiles' waits run out on purpose (timeout-path tests)
};

// Operator state for one arithmetic precision.  Owns its tables, the Green
// octant and per-voxel contrast in that precision, and the b/c scratch.
template <typename T> struct Operator {
    using C = cplx_t<T>;
    bool ready = false;
    OpDev<C> dev{};
    size_t smem_z = 0, smem_y = 0, smem_x = 0;
    // owned device allocations
    void* d_tables = nullptr;
    C* d_Gs = nullptr;
    C* d_w = nullptr;
    C* d_b = nullptr;
    C* d_c = nullptr;
    bool owns_scratch = true;
    // TMA view of the b scratch for the forward y pass (2D: 2 Lz reals x 3 nx ny rows)
    CUtensorMap tm_b{};
    bool tm_b_ok = false;
    bool use_ytma = false;
    const void* tm_b_addr = nullptr;  // the buffer tm_b was encoded for
    CUtensorMap tm_c{};          // TMA view of the c spectra for the inverse y pass
    bool tm_c_ok = false;
    const void* tm_c_addr = nullptr;
    // two words of mapped pinned host memory (h_status), so the host reads them
    // after a synchronisation without a copy: [0] set by a kernel whose bounded
    // wait ran out, [1] set when its copy had still not landed when it left
    int* h_status = nullptr;
    int* d_status = nullptr;

    int init(int nx, int ny, int nz, const double d[3], double k0, const TileCfg& tiles,
             const AxisPlan plans[3], const unsigned char* d_flags, Error& err);
    // upload the Green octant (FP64, unscaled, on device) scaled by i Z0/(k0 M) in precision T
    int set_green(const double2* d_oct64, double k0, cudaStream_t st, Error& err);
    // per-voxel 1/(eps-1) from host doubles (interleaved complex)
    int set_contrast(const double* w_host, cudaStream_t st, Error& err);
    void release();
    // y = A x (conj: A^H), plain store
    int apply(const C* x, C* y, bool conj, cudaStream_t st, Error& err);
    size_t scratch_bytes() const;
    // since the last call: 0 no bounded device wait ran out, 1 one ran out (its
    // tile left undone), 2 a copy was also still in flight when its block left;
    // the words are cleared
    int take_timeout() {
        if (!h_status) return 0;
        volatile int* s = h_status;
        const int r = s[1] ? 2 : (s[0] ? 1 : 0);
        s[0] = s[1] = 0;
        return r;
    }
};

// Device-resident Krylov scalars (FP64 complex), one block per solve.
enum ScalarSlot {
    S_RHO = 0, S_RHO1, S_ALPHA, S_OMEGA, S_BETA, S_BNRM2, S_RR, S_ERR,
    S_T0, S_T1, S_T2, S_T3, S_T4, S_T5, S_DONE, S_NAN, S_COUNT
};

// Device-resident control block of one iterative solve.  The decision at the
// end of every iteration (converged, breakdown, cap, reliable update) is taken
// on the device and written to `state`; the kernels of the next iteration are
// gated on it (Gate), and a captured iteration graph loops while the state is
// not terminal.
enum KrylovState { KS_RUN = 0, KS_UPDATE = 1, KS_DONE = 2, KS_BREAKDOWN = 3, KS_MAXIT = 4, KS_RESET = 5 };
struct KCtl {
    int state;
    int iter;      // iterations completed
    int maxit;
    int steps;     // step index of convergence (the reference's "Steps")
    int updates;   // reliable updates
    int loops;     // executions of the iteration body
    int hist_cap;  // entries of the history array
    int pad;
    double thr;    // threshold on the solver's error measure
    double delta;  // reliable-update trigger (mixed BiCGSTAB)
    double rmax2;  // largest ||r||^2 since the last reliable update
    double bn2;    // FP64 ||b||^2 (mixed BiCGSTAB)
    double last;   // last error (true residual after an update)
};

}  // namespace vie

// The opaque context of the C ABI.
struct vie_ctx {
    int device = 0;
    int nx = 0, ny = 0, nz = 0;
    long long a = 0;
    double d[3] = {0, 0, 0};
    double k0 = 0;
    cudaStream_t stream = nullptr;
    vie::Error err;

    // geometry / material (device)
    unsigned char* d_flags = nullptr;     // packed Flag_X | Flag_Y<<1 | Flag_Z<<2
    std::vector<double> w_host;           // 1/(eps-1) per voxel, interleaved
    bool have_flags = false, have_eps = false;

    // Green octant (FP64, unscaled) and operators
    double2* d_green = nullptr;           // (nx+1)(ny+1)(nz+1)
    bool have_green = false;
    vie::AxisPlan plans[3];
    // FFT schedule of each precision (autotuner choice or defaults)
    vie::TileCfg sched64, sched32;
    vie::AxisPlan plans64[3], plans32[3];
    bool sched_set = false;
    std::string tune_report;
    vie::Operator<double> op64;
    vie::Operator<float> op32;

    // right-hand side and solution (FP64, 3a each)
    double2* d_rhs = nullptr;
    double2* d_x = nullptr;
    bool have_rhs = false, have_x = false;

    // Krylov workspace (allocated on first solve)
    std::vector<void*> work;
    double2* d_scal = nullptr;            // vie::S_COUNT scalars
    double2* d_partial = nullptr;         // reduction partials
    size_t partial_cap = 0;               // entries
    double2* h_scal = nullptr;            // pinned mirror
    vie::KCtl* d_ctl = nullptr;           // solve control block (device)
    vie::KCtl* h_ctl = nullptr;           // pinned mirror
    double2* d_hist = nullptr;            // per iteration: (error, true residual of a reliable update or -1)
    int hist_cap = 0;
    vie::Gate gate{nullptr, 0};           // gate applied to launches while an iteration body is enqueued
    int use_graphs = 1;                   // capture the iteration body in a CUDA graph with a device-side loop
    long long graph_launches = 0;         // solve loops run as one graph launch
    int capturing = 0;                    // an iteration body is being captured
    cudaStream_t stream_aux = nullptr;    // capture stream of conditional (IF) bodies
    cudaStream_t stream_parent = nullptr; // ctx->stream while an IF body is captured on stream_aux

    // set when a staged copy was still in flight as its block left: shared
    // memory of that SM may still be written, so nothing more is launched
    bool unusable = false;

    int set_error(int code, const std::string& m) {
        err.code = code;
        err.msg = m;
        return code;
    }
    // after a synchronisation: VIE_ERR_TIMEOUT when a kernel's bounded wait on
    // its staged tile ran out since the last check (its pass was left undone)
    int check_waits(int rc) {
        const int t64 = op64.take_timeout(), t32 = op32.take_timeout();
        if (t64 == 2 || t32 == 2) {
            unusable = true;
            return set_error(VIE_ERR_TIMEOUT, "a TMA copy was still in flight when its bounded waits ran out; "
                                              "this context launches nothing more (destroy it)");
        }
        if (t64 || t32) return set_error(VIE_ERR_TIMEOUT, "a TMA tile load did not complete within its bounded wait");
        return rc;
    }
    // VIE_ERR_TIMEOUT once check_waits has marked the context unusable
    int check_usable() {
        if (!unusable) return VIE_OK;
        return set_error(VIE_ERR_TIMEOUT, "context unusable: an earlier call left a TMA copy in flight (destroy it)");
    }
};
