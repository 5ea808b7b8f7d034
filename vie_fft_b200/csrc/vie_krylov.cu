// vie_krylov.cu -- Krylov drivers of CG_Iteration.h on the GPU.
//
// All scalars (rho, alpha, omega, beta, norms) live in device memory as FP64
// complex and are produced by one-block finalize kernels from per-block
// partial sums (fixed summation order, so runs are deterministic).  Dot
// products always accumulate in FP64, also when the vectors are FP32.  The
// stop decision of every iteration (the reference's printf/break,
// CG_Iteration.h:733-747) is also taken on the device, into a control block
// (KCtl); every kernel of an iteration is gated on the control state, so the
// iteration body is captured once into a CUDA graph whose conditional WHILE
// node repeats it until the state is terminal: one graph launch per solve, no
// host round trip per iteration.  The per-iteration errors are kept in a
// device history and printed after the solve.
//
// BiCGSTAB fuses its vector updates into the operator passes:
//   p = r + beta (p - omega v)    in the first pass of A p  (CG_Iteration.h:611-633)
//   b^H v                         in the last pass of A p   (:652-662)
//   s = r - alpha v               in the first pass of A s  (:664-672)
//   t^H s, t^H t                  in the last pass of A s   (:689-706)
//   x += alpha p + omega s, r = s - omega t, r^H r, b^H r   one vector pass (:708-731, :594-598)
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <initializer_list>
#include <string>
#include <vector>

#include "vie_batch.h"
#include "vie_krylov.cuh"

namespace vie {

// end of one iteration body: count it and set the WHILE condition of the graph
__global__ void k_loop_cond(KCtl* ctl, cudaGraphConditionalHandle h) {
    ctl->loops++;
    const int s = ctl->state;
    cudaGraphSetConditional(h, (s == KS_RUN || s == KS_UPDATE || s == KS_RESET) ? 1u : 0u);
}
__global__ void k_loop_count(KCtl* ctl) { ctl->loops++; }
// condition of an IF node: the control state equals `when`
__global__ void k_set_if(const KCtl* ctl, cudaGraphConditionalHandle h, int when) {
    cudaGraphSetConditional(h, ctl->state == when ? 1u : 0u);
}

// y32 = float(x64)
__global__ void k_to_f32(float2* __restrict__ y, const double2* __restrict__ x, long long n, Gate gate) {
    if (gate_closed(gate)) return;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] = make_float2((float)x[i].x, (float)x[i].y);
}

// x64 += x32; x32 = 0 (the FP64 solution update of a reliable-update step)
__global__ void k_fold_correction(double2* __restrict__ x64, float2* __restrict__ x32, long long n, Gate gate) {
    if (gate_closed(gate)) return;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float2 d = x32[i];
        double2 v = x64[i];
        v.x += (double)d.x;
        v.y += (double)d.y;
        x64[i] = v;
        x32[i] = make_float2(0.f, 0.f);
    }
}

// ---------------------------------------------------------------------------
// workspace helpers
// ---------------------------------------------------------------------------

static int ensure_scalars(vie_ctx* ctx) {
    if (!ctx->d_scal) {
        VIE_CUDA_TRY(cudaMalloc(&ctx->d_scal, sizeof(double2) * S_COUNT * 4), ctx->err);
        VIE_CUDA_TRY(cudaMallocHost(&ctx->h_scal, sizeof(double2) * S_COUNT), ctx->err);
    }
    const long long need = std::max<long long>(kVecBlocks, 3LL * ((long long)ctx->nx * ctx->ny + 1)) * 4;
    if ((long long)ctx->partial_cap < need) {
        if (ctx->d_partial) cudaFree(ctx->d_partial);
        VIE_CUDA_TRY(cudaMalloc(&ctx->d_partial, sizeof(double2) * need), ctx->err);
        ctx->partial_cap = need;
    }
    return VIE_OK;
}

// pool of 3a-vectors by byte size
static void* work_vec(vie_ctx* ctx, int idx, size_t elem, int* rc) {
    const size_t bytes = elem * 3 * (size_t)ctx->a;
    // slot layout: ctx->work holds pairs (ptr, size) encoded as two entries
    const size_t need = 2 * (size_t)(idx + 1);
    while (ctx->work.size() < need) ctx->work.push_back(nullptr);
    void*& p = ctx->work[2 * idx];
    size_t sz = (size_t)(uintptr_t)ctx->work[2 * idx + 1];
    if (p && sz >= bytes) return p;
    if (p) cudaFree(p);
    p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        *rc = ctx->set_error(VIE_ERR_ALLOC, "device allocation of a Krylov vector failed");
        ctx->work[2 * idx + 1] = nullptr;
        return nullptr;
    }
    ctx->work[2 * idx + 1] = (void*)(uintptr_t)bytes;
    return p;
}

template <int K, class Fin>
static int finalize(vie_ctx* ctx, long long nblk, Fin fin) {
    k_finalize<K, Fin><<<1, 256, 0, ctx->stream>>>(ctx->d_partial, nblk, ctx->d_scal, fin, ctx->gate);
    count_launch();
    VIE_CUDA_TRY(cudaGetLastError(), ctx->err);
    return VIE_OK;
}

// blocks of a k_lin launch (and reduction partials it writes): one wave of
// resident blocks, at most kVecBlocks.  Instances with 40 registers hold 6
// blocks per SM; with kVecBlocks they would run a second wave a third full.
template <typename C, int NT, int K> static long long lin_blocks() {
    return std::min<int>(kVecBlocks, persistent_grid(k_lin<C, NT, K>, 256, 0));
}

template <typename C, int NT, int K>
static int lin(vie_ctx* ctx, const LinArgs<C, NT, K>& g) {
    k_lin<C, NT, K><<<(int)lin_blocks<C, NT, K>(), 256, 0, ctx->stream>>>(g, 3 * ctx->a, ctx->d_scal, ctx->d_partial,
                                                                         ctx->gate);
    count_launch();
    VIE_CUDA_TRY(cudaGetLastError(), ctx->err);
    return VIE_OK;
}

template <typename C, int K>
static int dots(vie_ctx* ctx, const DotArgs<C, K>& g) {
    k_dots<C, K><<<kVecBlocks, 256, 0, ctx->stream>>>(g, 3 * ctx->a, ctx->d_partial, ctx->gate);
    count_launch();
    VIE_CUDA_TRY(cudaGetLastError(), ctx->err);
    return VIE_OK;
}

static CoefSpec cs(int slot, double re = 1.0, double im = 0.0) { return CoefSpec{slot, re, im}; }

// read err and nan flags
static int read_scalars(vie_ctx* ctx) {
    VIE_CUDA_TRY(cudaMemcpyAsync(ctx->h_scal, ctx->d_scal, sizeof(double2) * S_COUNT, cudaMemcpyDeviceToHost,
                                 ctx->stream),
                 ctx->err);
    VIE_CUDA_TRY(cudaStreamSynchronize(ctx->stream), ctx->err);
    return VIE_OK;
}

// Reliable-update trigger of the mixed BiCGSTAB: the FP32 residual has fallen
// by this factor below its maximum since the last update.  Measured at 256^3
// (two right-hand sides): 0.1 -> 4.94 s, 0.03 -> 4.77 s, 0.01 -> 4.81 s,
// 0.003 -> 5.01 s per solve; at 128^3 the smaller values save updates.
constexpr double kReliableDelta = 0.03;

struct KrylovResult {
    int steps = -1;
    int iterations = 0;
    int matvecs = 0;
    double err = -1;
    int status = VIE_OK;
};

// matvec with generic prologue/epilogue on operator op, under the current gate
template <typename T, class Pro, class Epi>
static int opmv(vie_ctx* ctx, Operator<T>& op, Pro pro, Epi epi, const cplx_t<T>* xdiag, bool conj) {
    op.dev.gate = ctx->gate;
    const int rc = launch_operator<T>(op, pro, epi, xdiag, conj, ctx->d_partial, ctx->stream, ctx->err);
    op.dev.gate = Gate{nullptr, 0};
    return rc;
}

// ---------------------------------------------------------------------------
// control block and the iteration loop
// ---------------------------------------------------------------------------
__global__ void k_ctl_init(KCtl* c, double thr, int maxit, double delta, int cap) {
    KCtl v;
    v.state = KS_RUN;
    v.iter = 0;
    v.maxit = maxit;
    v.steps = -1;
    v.updates = 0;
    v.loops = 0;
    v.hist_cap = cap;
    v.pad = 0;
    v.thr = thr;
    v.delta = delta;
    v.rmax2 = 0.0;
    v.bn2 = 0.0;
    v.last = -1.0;
    *c = v;
}

// state RUN, counters zero; the history holds up to 2^20 iterations
static int ctl_init(vie_ctx* ctx, double thr, int maxit, double delta) {
    if (!ctx->d_ctl) {
        VIE_CUDA_TRY(cudaMalloc(&ctx->d_ctl, sizeof(KCtl)), ctx->err);
        VIE_CUDA_TRY(cudaMallocHost(&ctx->h_ctl, sizeof(KCtl)), ctx->err);
    }
    const int cap = (int)std::min<long long>(std::max(maxit, 1), 1LL << 20);
    if (ctx->hist_cap < cap) {
        if (ctx->d_hist) cudaFree(ctx->d_hist);
        ctx->d_hist = nullptr;
        ctx->hist_cap = 0;
        VIE_CUDA_TRY(cudaMalloc(&ctx->d_hist, sizeof(double2) * cap), ctx->err);
        ctx->hist_cap = cap;
    }
    k_ctl_init<<<1, 1, 0, ctx->stream>>>(ctx->d_ctl, thr, maxit, delta, ctx->hist_cap);
    count_launch();
    VIE_CUDA_TRY(cudaGetLastError(), ctx->err);
    return VIE_OK;
}

static int ctl_read(vie_ctx* ctx) {
    VIE_CUDA_TRY(cudaMemcpyAsync(ctx->h_ctl, ctx->d_ctl, sizeof(KCtl), cudaMemcpyDeviceToHost, ctx->stream), ctx->err);
    VIE_CUDA_TRY(cudaStreamSynchronize(ctx->stream), ctx->err);
    return VIE_OK;
}

static bool ks_live(int s) { return s == KS_RUN || s == KS_UPDATE || s == KS_RESET; }

// Launches enqueued between cond_begin(when) and cond_end run only while the
// control state equals `when`.  Inside a captured body they become the child
// graph of a conditional IF node, so they are not launched at all otherwise;
// outside a capture their gates alone skip them.
static int cond_begin(vie_ctx* ctx, int when) {
    if (!ctx->capturing) return VIE_OK;
    cudaStream_t st = ctx->stream;
    cudaStreamCaptureStatus cst;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    VIE_CUDA_TRY(cudaStreamGetCaptureInfo(st, &cst, nullptr, &g, &deps, &nd), ctx->err);
    cudaGraphConditionalHandle h;
    VIE_CUDA_TRY(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault), ctx->err);
    k_set_if<<<1, 1, 0, st>>>(ctx->d_ctl, h, when);
    count_launch();
    VIE_CUDA_TRY(cudaGetLastError(), ctx->err);
    VIE_CUDA_TRY(cudaStreamGetCaptureInfo(st, &cst, nullptr, &g, &deps, &nd), ctx->err);
    cudaGraphNodeParams np = {cudaGraphNodeTypeConditional};
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeIf;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    VIE_CUDA_TRY(cudaGraphAddNode(&node, g, deps, nd, &np), ctx->err);
    VIE_CUDA_TRY(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies), ctx->err);
    if (!ctx->stream_aux)
        VIE_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->stream_aux, cudaStreamNonBlocking), ctx->err);
    VIE_CUDA_TRY(cudaStreamBeginCaptureToGraph(ctx->stream_aux, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                               cudaStreamCaptureModeRelaxed),
                 ctx->err);
    ctx->stream_parent = st;
    ctx->stream = ctx->stream_aux;
    return VIE_OK;
}
static int cond_end(vie_ctx* ctx) {
    if (!ctx->capturing || !ctx->stream_parent) return VIE_OK;
    cudaGraph_t g = nullptr;
    ctx->stream = ctx->stream_parent;
    ctx->stream_parent = nullptr;
    VIE_CUDA_TRY(cudaStreamEndCapture(ctx->stream_aux, &g), ctx->err);
    return VIE_OK;
}

// Graph form of the loop: the body is captured once as the child graph of a
// conditional WHILE node whose condition k_loop_cond sets from the control
// state after every pass, so the whole solve is one graph launch.  Returns
// an error with launched == false when the graph could not be built (nothing
// of the body ran then).
template <class Body>
static int run_loop_graph(vie_ctx* ctx, Body& body, bool& launched) {
    cudaStream_t st = ctx->stream;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int rc = VIE_OK;
    launched = false;
    do {
        cudaGraphConditionalHandle h;
        if (cudaGraphCreate(&graph, 0) != cudaSuccess ||
            cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
            rc = ctx->set_error(VIE_ERR_CUDA, "conditional graph handle");
            break;
        }
        cudaGraphNodeParams np = {cudaGraphNodeTypeConditional};
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        if (cudaGraphAddNode(&node, graph, nullptr, 0, &np) != cudaSuccess) {
            rc = ctx->set_error(VIE_ERR_CUDA, "conditional WHILE node");
            break;
        }
        cudaGraph_t bodyg = np.conditional.phGraph_out[0];
        if (cudaStreamBeginCaptureToGraph(st, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
            rc = ctx->set_error(VIE_ERR_CUDA, "stream capture into the loop body");
            break;
        }
        const long long n0 = g_launches.load();
        ctx->capturing = 1;
        int brc = body();
        if (ctx->stream_parent) {  // an IF body left open by an error
            cudaGraph_t tmp = nullptr;
            cudaStreamEndCapture(ctx->stream_aux, &tmp);
            ctx->stream = ctx->stream_parent;
            ctx->stream_parent = nullptr;
        }
        ctx->capturing = 0;
        k_loop_cond<<<1, 1, 0, st>>>(ctx->d_ctl, h);
        count_launch();
        cudaGraph_t captured = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(st, &captured);
        const long long per = g_launches.load() - n0;
        count_launch(-per);  // counted again below, once per executed pass
        if (brc) { rc = brc; break; }
        if (ce != cudaSuccess) {
            rc = ctx->set_error(VIE_ERR_CUDA, std::string("stream capture of the loop body: ") + cudaGetErrorString(ce));
            break;
        }
        if (cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
            rc = ctx->set_error(VIE_ERR_CUDA, "graph instantiation");
            break;
        }
        launched = true;
        VIE_CUDA_TRY(cudaGraphLaunch(exec, st), ctx->err);
        if ((rc = ctl_read(ctx))) break;
        count_launch(per * ctx->h_ctl->loops);
        ctx->graph_launches++;
    } while (0);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (rc && !launched) (void)cudaGetLastError();  // clear a non-sticky build error
    return rc;
}

// Runs the iteration body until the control state is terminal: as one graph
// launch (default), or, with VIE_GRAPH=0 or where the graph cannot be built,
// launched from the host with the state read back after every pass.
template <class Body>
static int run_loop(vie_ctx* ctx, Body body) {
    if (ctx->use_graphs) {
        bool launched = false;
        const int rc = run_loop_graph(ctx, body, launched);
        if (launched || rc == VIE_OK) return rc;
        // the graph could not be built (nothing ran): the same body from the host
        std::fprintf(stderr, "vie_b200: %s; iterating without graphs\n", ctx->err.msg.c_str());
        ctx->err.code = VIE_OK;
        ctx->use_graphs = 0;
    }
    cudaStream_t st = ctx->stream;
    while (true) {
        int rc = body();
        if (rc) return rc;
        k_loop_count<<<1, 1, 0, st>>>(ctx->d_ctl);
        count_launch();
        VIE_CUDA_TRY(cudaGetLastError(), ctx->err);
        if ((rc = ctl_read(ctx))) return rc;
        if (!ks_live(ctx->h_ctl->state)) return VIE_OK;
    }
}

// ---------------------------------------------------------------------------
// several solves in one graph loop
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool ks_live_dev(int s) { return s == KS_RUN || s == KS_UPDATE || s == KS_RESET; }

// start of a batch pass: open the IF node of every instance that is still live
__global__ void k_batch_live(KCtl* const* __restrict__ ctls, const cudaGraphConditionalHandle* __restrict__ hs, int n) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const bool live = ks_live_dev(ctls[i]->state);
        if (live) ctls[i]->loops++;
        cudaGraphSetConditional(hs[i], live ? 1u : 0u);
    }
}
// end of a batch pass: loop again while any instance is live
__global__ void k_batch_cond(KCtl* const* __restrict__ ctls, int n, cudaGraphConditionalHandle h, int* passes) {
    int any = 0;
    for (int i = threadIdx.x; i < n; i += 32) any |= ks_live_dev(ctls[i]->state) ? 1 : 0;
    any = __any_sync(0xffffffffu, any);
    if (threadIdx.x == 0) {
        (*passes)++;
        cudaGraphSetConditional(h, any ? 1u : 0u);
    }
}

template <class PlanT>
static int run_loop_batch_graph(std::vector<PlanT*>& plans, cudaStream_t S, vie_ctx* ectx, bool& launched) {
    const int n = (int)plans.size();
    launched = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    void* dmem = nullptr;
    int rc = VIE_OK;
    std::vector<long long> per(n, 0);
    do {
        // device arrays: control-block pointers, IF handles, pass counter
        const size_t off_h = align_up(sizeof(KCtl*) * n, 64), off_p = align_up(off_h + sizeof(cudaGraphConditionalHandle) * n, 64);
        if (cudaMalloc(&dmem, off_p + 64) != cudaSuccess) { rc = ectx->set_error(VIE_ERR_ALLOC, "batch control arrays"); break; }
        KCtl** d_ctls = (KCtl**)dmem;
        cudaGraphConditionalHandle* d_hs = (cudaGraphConditionalHandle*)((char*)dmem + off_h);
        int* d_passes = (int*)((char*)dmem + off_p);
        cudaGraphConditionalHandle hw;
        if (cudaGraphCreate(&graph, 0) != cudaSuccess ||
            cudaGraphConditionalHandleCreate(&hw, graph, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
            rc = ectx->set_error(VIE_ERR_CUDA, "batch graph / WHILE handle");
            break;
        }
        cudaGraphNodeParams wp = {cudaGraphNodeTypeConditional};
        wp.conditional.handle = hw;
        wp.conditional.type = cudaGraphCondTypeWhile;
        wp.conditional.size = 1;
        cudaGraphNode_t wnode;
        if (cudaGraphAddNode(&wnode, graph, nullptr, 0, &wp) != cudaSuccess) {
            rc = ectx->set_error(VIE_ERR_CUDA, "batch WHILE node");
            break;
        }
        cudaGraph_t bodyg = wp.conditional.phGraph_out[0];
        std::vector<cudaGraphConditionalHandle> hs(n);
        std::vector<KCtl*> ctls(n);
        bool ok = true;
        for (int i = 0; i < n && ok; i++) {
            ok = cudaGraphConditionalHandleCreate(&hs[i], bodyg, 0, cudaGraphCondAssignDefault) == cudaSuccess;
            ctls[i] = plans[i]->ctx->d_ctl;
        }
        if (!ok || cudaMemcpy(d_ctls, ctls.data(), sizeof(KCtl*) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(d_hs, hs.data(), sizeof(cudaGraphConditionalHandle) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemset(d_passes, 0, sizeof(int)) != cudaSuccess) {
            rc = ectx->set_error(VIE_ERR_CUDA, "batch IF handles");
            break;
        }
        if (cudaStreamBeginCaptureToGraph(S, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
            rc = ectx->set_error(VIE_ERR_CUDA, "stream capture of the batch body");
            break;
        }
        k_batch_live<<<1, 256, 0, S>>>(d_ctls, d_hs, n);
        cudaStreamCaptureStatus cst;
        cudaGraph_t g2 = nullptr;
        const cudaGraphNode_t* dp = nullptr;
        size_t nd = 0;
        std::vector<cudaGraphNode_t> deps, ifs(n);
        if (cudaStreamGetCaptureInfo(S, &cst, nullptr, &g2, &dp, &nd) == cudaSuccess) deps.assign(dp, dp + nd);
        else ok = false;
        for (int i = 0; i < n && ok && !rc; i++) {
            vie_ctx* c = plans[i]->ctx;
            cudaGraphNodeParams ip = {cudaGraphNodeTypeConditional};
            ip.conditional.handle = hs[i];
            ip.conditional.type = cudaGraphCondTypeIf;
            ip.conditional.size = 1;
            if (cudaGraphAddNode(&ifs[i], bodyg, deps.data(), deps.size(), &ip) != cudaSuccess ||
                cudaStreamBeginCaptureToGraph(c->stream, ip.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                              cudaStreamCaptureModeRelaxed) != cudaSuccess) {
                ok = false;
                break;
            }
            const long long n0 = g_launches.load();
            c->capturing = 1;
            const int brc = plans[i]->body();
            if (c->stream_parent) {
                cudaGraph_t tmp = nullptr;
                cudaStreamEndCapture(c->stream_aux, &tmp);
                c->stream = c->stream_parent;
                c->stream_parent = nullptr;
            }
            c->capturing = 0;
            c->gate = Gate{nullptr, 0};
            cudaGraph_t tmp = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(c->stream, &tmp);
            per[i] = g_launches.load() - n0;
            count_launch(-per[i]);
            if (brc) rc = brc;
            else if (ce != cudaSuccess) ok = false;
        }
        if (ok && !rc)
            ok = cudaStreamUpdateCaptureDependencies(S, ifs.data(), n, cudaStreamSetCaptureDependencies) == cudaSuccess;
        k_batch_cond<<<1, 32, 0, S>>>(d_ctls, n, hw, d_passes);
        cudaGraph_t captured = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(S, &captured);
        if (rc) break;
        if (!ok || ce != cudaSuccess) {
            rc = ectx->set_error(VIE_ERR_CUDA, "capture of the batch body");
            break;
        }
        if (cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
            rc = ectx->set_error(VIE_ERR_CUDA, "batch graph instantiation");
            break;
        }
        launched = true;
        if (cudaGraphLaunch(exec, S) != cudaSuccess || cudaStreamSynchronize(S) != cudaSuccess) {
            rc = ectx->set_error(VIE_ERR_CUDA, std::string("batch graph: ") + cudaGetErrorString(cudaGetLastError()));
            break;
        }
        int passes = 0;
        if (cudaMemcpy(&passes, d_passes, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
            rc = ectx->set_error(VIE_ERR_CUDA, "batch pass count");
            break;
        }
        count_launch(2LL * passes);
        for (int i = 0; i < n && !rc; i++) {
            vie_ctx* c = plans[i]->ctx;
            if ((rc = ctl_read(c))) break;
            count_launch(per[i] * c->h_ctl->loops);
            c->graph_launches++;
        }
    } while (0);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (dmem) cudaFree(dmem);
    if (rc && !launched) (void)cudaGetLastError();
    return rc;
}

// the drivers' console output, replayed from the device history:
// "CG Error" per step, "Steps" at convergence (CG_Iteration.h:323-331 etc.);
// BiCORSTAB prints only "Steps" at convergence (:1315-1327); the mixed solve
// prints the true residual of every reliable update
enum PrintStyle { PS_ERR_STEPS = 0, PS_STEPS_ONLY = 1, PS_RELIABLE = 2 };
static int print_history(vie_ctx* ctx, const KCtl& c, int style) {
    const int n = std::min(c.iter, c.hist_cap);
    if (n <= 0) return VIE_OK;
    std::vector<double2> h((size_t)n);
    VIE_CUDA_TRY(cudaMemcpy(h.data(), ctx->d_hist, sizeof(double2) * n, cudaMemcpyDeviceToHost), ctx->err);
    for (int m = 0; m < n; m++) {
        if (style == PS_RELIABLE) {
            if (h[m].y >= 0.0) printf("CG Error: %lf (true residual)\n", h[m].y);
            else printf("CG Error: %lf\n", h[m].x);
        } else if (c.state == KS_DONE && m == c.steps) {
            if (style == PS_ERR_STEPS) printf("CG Error: %lf\nSteps: %d\n\n", h[m].x, m);
            else printf("Steps: %d\n\n", m);
        } else {
            printf("CG Error: %lf\n", h[m].x);
        }
    }
    fflush(stdout);
    return VIE_OK;
}

// outcome of a loop from the control block (already read back)
static int finish(vie_ctx* ctx, KrylovResult& res, int mv_setup, int mv_per_iter, int style, int verbose,
                  const char* name) {
    const KCtl c = *ctx->h_ctl;
    if (verbose) {
        const int rc = print_history(ctx, c, style);
        if (rc) return rc;
    }
    res.iterations = c.iter;
    res.matvecs = mv_setup + mv_per_iter * c.iter;
    res.err = c.last;
    if (c.state == KS_DONE) {
        res.steps = c.steps;
        return VIE_OK;
    }
    if (c.state == KS_MAXIT) {
        res.status = VIE_ERR_MAXIT;
        return VIE_OK;
    }
    res.status = VIE_ERR_BREAKDOWN;
    return ctx->set_error(VIE_ERR_BREAKDOWN, std::string(name) + " breakdown (zero or non-finite scalar) at step " +
                                                 std::to_string(c.iter - 1));
}

// A solve split into its set-up (already enqueued on the context stream), an
// iteration body and a completion step, so that several solves can share one
// graph loop (vie_solve_batch).
struct SolvePlan {
    vie_ctx* ctx = nullptr;
    std::function<int()> body;
    std::function<int()> finish;
};

// run the loop now (plan == nullptr) or hand body and completion to a batch
static int launch_or_plan(vie_ctx* ctx, SolvePlan* plan, std::function<int()> body, std::function<int()> fin) {
    if (plan) {
        plan->ctx = ctx;
        plan->body = std::move(body);
        plan->finish = std::move(fin);
        return VIE_OK;
    }
    int rc = run_loop(ctx, body);
    ctx->gate = Gate{nullptr, 0};
    if (rc) return rc;
    return fin();
}

static int zero_vecs(vie_ctx* ctx, size_t bytes, std::initializer_list<void*> vs) {
    for (void* v : vs) VIE_CUDA_TRY(cudaMemsetAsync(v, 0, bytes, ctx->stream), ctx->err);
    return VIE_OK;
}

// ---------------------------------------------------------------------------
// solvers on C-precision vectors.  b: masked right-hand side, x: solution
// (zeroed here), thr: threshold on the solver's own error measure.  Each one
// is a set-up followed by an iteration body whose first pass equals the
// reference's first step because the direction vectors start at zero and
// beta at 0.
// ---------------------------------------------------------------------------
template <typename T>
static int solve_bicgstab(vie_ctx* ctx, Operator<T>& op, const cplx_t<T>* b, cplx_t<T>* x, double thr, int maxit,
                          int verbose, int vbase, KrylovResult& res, SolvePlan* plan = nullptr) {
    using C = cplx_t<T>;
    int rc = VIE_OK;
    const long long a = ctx->a, n = 3 * a;
    C* r = (C*)work_vec(ctx, vbase + 0, sizeof(C), &rc);
    C* p = (C*)work_vec(ctx, vbase + 1, sizeof(C), &rc);
    C* v = (C*)work_vec(ctx, vbase + 2, sizeof(C), &rc);
    C* sv = (C*)work_vec(ctx, vbase + 3, sizeof(C), &rc);
    C* t = (C*)work_vec(ctx, vbase + 4, sizeof(C), &rc);
    if (rc) return rc;
    cudaStream_t st = ctx->stream;
    if ((rc = zero_vecs(ctx, sizeof(C) * n, {x, p, v}))) return rc;
    VIE_CUDA_TRY(cudaMemcpyAsync(r, b, sizeof(C) * n, cudaMemcpyDeviceToDevice, st), ctx->err);  // :565-567
    {
        DotArgs<C, 2> g{{b, b}, {b, r}, {1, 1}};
        if ((rc = dots(ctx, g))) return rc;
        if ((rc = finalize<2>(ctx, kVecBlocks, FinBicgstabInit{}))) return rc;
    }
    if ((rc = ctl_init(ctx, thr, maxit, 0.0))) return rc;
    KCtl* ctl = ctx->d_ctl;
    double2* hist = ctx->d_hist;
    const long long nblk = epilogue_blocks(op);
    auto body = [=, &op]() -> int {
        int rc2;
        ctx->gate = Gate{&ctl->state, KS_RUN};
        // p = r + beta (p - omega v) (:611-633); v = A p; b^H v (:652-662)
        if ((rc2 = opmv(ctx, op, ProBicgP<C>{r, p, v, ctx->d_scal, a}, EpiDotB<C>{v, b, a}, p, false))) return rc2;
        if ((rc2 = finalize<1>(ctx, nblk, FinAlpha{}))) return rc2;
        // s = r - alpha v (:664-672); t = A s; t^H s, t^H t (:689-706)
        if ((rc2 = opmv(ctx, op, ProBicgS<C>{r, v, sv, ctx->d_scal, a}, EpiDotTS<C>{t, sv, a}, sv, false))) return rc2;
        if ((rc2 = finalize<2>(ctx, nblk, FinOmega{}))) return rc2;
        k_bicgstab_update<C><<<kVecBlocks, 256, 0, ctx->stream>>>(x, p, sv, t, r, b, n, ctx->d_scal, ctx->d_partial,
                                                                   ctx->gate);
        count_launch();
        VIE_CUDA_TRY(cudaGetLastError(), ctx->err);
        return finalize<2>(ctx, kVecBlocks, then(FinBicgstabUpdate{}, DecideErr{ctl, hist}));
    };
    auto fin = [ctx, &res, verbose]() { return finish(ctx, res, 0, 2, PS_ERR_STEPS, verbose, "BiCGSTAB"); };
    return launch_or_plan(ctx, plan, body, fin);
}

template <typename T>
static int solve_cors(vie_ctx* ctx, Operator<T>& op, const cplx_t<T>* b, cplx_t<T>* x, double thr, int maxit,
                      int verbose, int vbase, KrylovResult& res, SolvePlan* plan = nullptr) {
    using C = cplx_t<T>;
    int rc = VIE_OK;
    const long long a = ctx->a, n = 3 * a;
    C* r = (C*)work_vec(ctx, vbase + 0, sizeof(C), &rc);
    C* p = (C*)work_vec(ctx, vbase + 1, sizeof(C), &rc);
    C* q = (C*)work_vec(ctx, vbase + 2, sizeof(C), &rc);
    C* Ap = (C*)work_vec(ctx, vbase + 3, sizeof(C), &rc);
    C* Aq = (C*)work_vec(ctx, vbase + 4, sizeof(C), &rc);
    C* rc_ = (C*)work_vec(ctx, vbase + 5, sizeof(C), &rc);
    C* pc = (C*)work_vec(ctx, vbase + 6, sizeof(C), &rc);
    C* qc = (C*)work_vec(ctx, vbase + 7, sizeof(C), &rc);
    if (rc) return rc;
    cudaStream_t st = ctx->stream;
    if ((rc = zero_vecs(ctx, sizeof(C) * n, {x, q, rc_, pc}))) return rc;
    VIE_CUDA_TRY(cudaMemcpyAsync(r, b, sizeof(C) * n, cudaMemcpyDeviceToDevice, st), ctx->err);  // :826-828
    {
        DotArgs<C, 1> g{{b}, {b}, {1}};
        if ((rc = dots(ctx, g))) return rc;
        if ((rc = finalize<1>(ctx, kVecBlocks, FinStore1{S_BNRM2}))) return rc;
    }
    if ((rc = ctl_init(ctx, thr, maxit, 0.0))) return rc;
    KCtl* ctl = ctx->d_ctl;
    double2* hist = ctx->d_hist;
    const long long nblk = epilogue_blocks(op);
    // the update kernel in one wave of resident blocks: k_cors_update<float2>
    // holds 6 blocks per SM, and a grid of kVecBlocks (8 per SM) would leave a
    // second wave a third full (256^3: 0.79 ms against 0.65 ms in one wave)
    const int ncu = std::min<int>(kVecBlocks, persistent_grid(k_cors_update<C>, 256, 0));
    auto body = [=, &op]() -> int {
        int rc2;
        ctx->gate = Gate{&ctl->state, KS_RUN};
        // Ap = A r; rho = b^H Ap (:853-869)
        if ((rc2 = opmv(ctx, op, ProCopy<C>{r, a}, EpiDotB<C>{Ap, b, a}, r, false))) return rc2;
        if ((rc2 = finalize<1>(ctx, nblk, FinCorsRho{ctl}))) return rc2;
        // p = r + beta pc; qc = Ap + beta rc; q = qc + beta rc + beta^2 q (:880-915)
        // in the first pass of Aq = A q; alpha = rho / (b^H Aq) (:938-962).  On the
        // first step beta = 0 and pc = rc = q = 0: p = r, qc = q = Ap (:843-851)
        if ((rc2 = opmv(ctx, op, ProCorsQ<C>{r, p, pc, Ap, qc, rc_, q, ctx->d_scal, a}, EpiDotB<C>{Aq, b, a}, q,
                        false)))
            return rc2;
        if ((rc2 = finalize<1>(ctx, nblk, FinCorsAlpha{}))) return rc2;
        // pc = p - alpha q; rc = qc - alpha Aq (:964-981); x += 2 alpha p - alpha^2 q
        // (:983-997); r += -2 alpha qc + alpha^2 Aq (:999-1012); r^H r: one pass
        k_cors_update<C><<<ncu, 256, 0, ctx->stream>>>(pc, rc_, x, r, p, q, qc, Aq, n, ctx->d_scal, ctx->d_partial,
                                                        ctx->gate);
        count_launch();
        VIE_CUDA_TRY(cudaGetLastError(), ctx->err);
        return finalize<1>(ctx, ncu, then(FinErr{}, DecideErr{ctl, hist}));
    };
    auto fin = [ctx, &res, verbose]() { return finish(ctx, res, 0, 2, PS_ERR_STEPS, verbose, "CORS"); };
    return launch_or_plan(ctx, plan, body, fin);
}

template <typename T>
static int solve_bicorstab(vie_ctx* ctx, Operator<T>& op, const cplx_t<T>* b, cplx_t<T>* x, double thr, int maxit,
                           int verbose, int vbase, KrylovResult& res, SolvePlan* plan = nullptr) {
    using C = cplx_t<T>;
    int rc = VIE_OK;
    const long long a = ctx->a, n = 3 * a;
    C* r = (C*)work_vec(ctx, vbase + 0, sizeof(C), &rc);
    C* p = (C*)work_vec(ctx, vbase + 1, sizeof(C), &rc);
    C* q = (C*)work_vec(ctx, vbase + 2, sizeof(C), &rc);
    C* Ap = (C*)work_vec(ctx, vbase + 3, sizeof(C), &rc);
    C* Aq = (C*)work_vec(ctx, vbase + 4, sizeof(C), &rc);
    C* pc = (C*)work_vec(ctx, vbase + 5, sizeof(C), &rc);
    C* qc = (C*)work_vec(ctx, vbase + 6, sizeof(C), &rc);
    if (rc) return rc;
    cudaStream_t st = ctx->stream;
    if ((rc = zero_vecs(ctx, sizeof(C) * n, {x, p, q, Aq}))) return rc;
    VIE_CUDA_TRY(cudaMemcpyAsync(r, b, sizeof(C) * n, cudaMemcpyDeviceToDevice, st), ctx->err);  // :1118-1120
    {
        DotArgs<C, 1> g{{b}, {b}, {1}};
        if ((rc = dots(ctx, g))) return rc;
        if ((rc = finalize<1>(ctx, kVecBlocks, FinStore1{S_BNRM2}))) return rc;
    }
    if ((rc = ctl_init(ctx, thr, maxit, 0.0))) return rc;
    KCtl* ctl = ctx->d_ctl;
    double2* hist = ctx->d_hist;
    const long long nblk = epilogue_blocks(op);
    auto body = [=, &op]() -> int {
        int rc2;
        ctx->gate = Gate{&ctl->state, KS_RUN};
        if ((rc2 = opmv(ctx, op, ProCopy<C>{r, a}, EpiDotB<C>{Ap, b, a}, r, false))) return rc2;   // :1145-1162
        if ((rc2 = finalize<1>(ctx, nblk, FinBicorRho{ctl}))) return rc2;
        // p = r + beta (p - omega q); q = Ap + beta (q - omega Aq)  (:1175-1207);
        // first step: beta = 0 and p = q = Aq = 0 give p = r, q = Ap (:1134-1143)
        if ((rc2 = lin(ctx, LinArgs<C, 3, 0>{p, 0, {{p, cs(S_BETA)}, {q, cs(S_T2, -1.0)}, {r, cs(-1)}}, {}})))
            return rc2;
        if ((rc2 = lin(ctx, LinArgs<C, 3, 0>{q, 0, {{q, cs(S_BETA)}, {Aq, cs(S_T2, -1.0)}, {Ap, cs(-1)}}, {}})))
            return rc2;
        if ((rc2 = opmv(ctx, op, ProCopy<C>{q, a}, EpiDotB<C>{Aq, b, a}, q, false))) return rc2;   // :1224-1248
        if ((rc2 = finalize<1>(ctx, nblk, FinAlpha{}))) return rc2;
        // pc = r - alpha q; qc = Ap - alpha Aq; omega = qc^H pc / qc^H qc  (:1250-1287)
        if ((rc2 = lin(ctx, LinArgs<C, 2, 0>{pc, 0, {{r, cs(-1)}, {q, cs(S_ALPHA, -1.0)}}, {}}))) return rc2;
        if ((rc2 = lin(ctx, LinArgs<C, 2, 2>{qc, 0, {{Ap, cs(-1)}, {Aq, cs(S_ALPHA, -1.0)}}, {{pc, 1}, {nullptr, 1}}})))
            return rc2;
        // d0 = conj(pc).qc, so qc^H pc = conj(d0)
        if ((rc2 = finalize<2>(ctx, lin_blocks<C, 2, 2>(), FinBicorOmega{}))) return rc2;
        // x += alpha p + omega pc; r = pc - omega qc; r^H r  (:1289-1315)
        if ((rc2 = lin(ctx, LinArgs<C, 2, 0>{x, 1, {{p, cs(S_ALPHA)}, {pc, cs(S_OMEGA)}}, {}}))) return rc2;
        if ((rc2 = lin(ctx, LinArgs<C, 2, 1>{r, 0, {{pc, cs(-1)}, {qc, cs(S_OMEGA, -1.0)}}, {{nullptr, 1}}})))
            return rc2;
        return finalize<1>(ctx, lin_blocks<C, 2, 1>(), then(FinErr{}, DecideErr{ctl, hist}));
    };
    auto fin = [ctx, &res, verbose]() { return finish(ctx, res, 0, 2, PS_STEPS_ONLY, verbose, "BiCORSTAB"); };
    return launch_or_plan(ctx, plan, body, fin);
}

template <typename T>
static int solve_cg(vie_ctx* ctx, Operator<T>& op, const cplx_t<T>* b, cplx_t<T>* x, double thr, int maxit,
                    int verbose, int vbase, KrylovResult& res, SolvePlan* plan = nullptr) {
    using C = cplx_t<T>;
    int rc = VIE_OK;
    const long long a = ctx->a, n = 3 * a;
    C* r = (C*)work_vec(ctx, vbase + 0, sizeof(C), &rc);
    C* p = (C*)work_vec(ctx, vbase + 1, sizeof(C), &rc);
    C* q = (C*)work_vec(ctx, vbase + 2, sizeof(C), &rc);
    C* Ap = (C*)work_vec(ctx, vbase + 3, sizeof(C), &rc);
    if (rc) return rc;
    if ((rc = zero_vecs(ctx, sizeof(C) * n, {x}))) return rc;
    // r = -b (:208-216); p = A^H b (:219-229)
    if ((rc = lin(ctx, LinArgs<C, 1, 0>{r, 0, {{b, cs(-1, -1.0)}}, {}}))) return rc;
    if ((rc = opmv(ctx, op, ProCopy<C>{b, a}, EpiNorm<C>{p, a}, b, true))) return rc;
    const long long nblk = epilogue_blocks(op);
    if ((rc = finalize<1>(ctx, nblk, FinStore1{S_T0}))) return rc;  // v3 = ||p||^2
    {
        DotArgs<C, 1> g{{b}, {b}, {1}};
        if ((rc = dots(ctx, g))) return rc;
        if ((rc = finalize<1>(ctx, kVecBlocks, FinStore1{S_BNRM2}))) return rc;  // vx
    }
    if ((rc = ctl_init(ctx, thr, maxit, 0.0))) return rc;
    KCtl* ctl = ctx->d_ctl;
    double2* hist = ctx->d_hist;
    auto body = [=, &op]() -> int {
        int rc2;
        ctx->gate = Gate{&ctl->state, KS_RUN};
        if ((rc2 = opmv(ctx, op, ProCopy<C>{p, a}, EpiNorm<C>{Ap, a}, p, false))) return rc2;  // :253-268
        if ((rc2 = finalize<1>(ctx, nblk, FinCgAlpha{}))) return rc2;
        // x += alpha p; r += alpha Ap; v4 = ||r||^2 (:273-286)
        if ((rc2 = lin(ctx, LinArgs<C, 1, 0>{x, 1, {{p, cs(S_ALPHA)}}, {}}))) return rc2;
        if ((rc2 = lin(ctx, LinArgs<C, 1, 1>{r, 1, {{Ap, cs(S_ALPHA)}}, {{nullptr, 1}}}))) return rc2;
        if ((rc2 = finalize<1>(ctx, lin_blocks<C, 1, 1>(), FinCgErr{}))) return rc2;
        // q = A^H r; v3 = ||q||^2; beta = v3 / v1 (:291-309)
        if ((rc2 = opmv(ctx, op, ProCopy<C>{r, a}, EpiNorm<C>{q, a}, r, true))) return rc2;
        if ((rc2 = finalize<1>(ctx, nblk, FinCgBeta{}))) return rc2;
        // p = beta p - q (:311-320); then the stop rule on v4 / vx (:323-331)
        if ((rc2 = lin(ctx, LinArgs<C, 2, 0>{p, 0, {{p, cs(S_BETA)}, {q, cs(-1, -1.0)}}, {}}))) return rc2;
        return finalize<1>(ctx, 1, then(FinNone{}, DecideErr{ctl, hist}));
    };
    auto fin = [ctx, &res, verbose]() { return finish(ctx, res, 1, 2, PS_ERR_STEPS, verbose, "CG"); };
    return launch_or_plan(ctx, plan, body, fin);
}

template <typename T>
static int solve_bicg(vie_ctx* ctx, Operator<T>& op, const cplx_t<T>* b, cplx_t<T>* x, double thr, int maxit,
                      int verbose, int vbase, KrylovResult& res, SolvePlan* plan = nullptr) {
    using C = cplx_t<T>;
    int rc = VIE_OK;
    const long long a = ctx->a, n = 3 * a;
    C* r = (C*)work_vec(ctx, vbase + 0, sizeof(C), &rc);
    C* p = (C*)work_vec(ctx, vbase + 1, sizeof(C), &rc);
    C* Ap = (C*)work_vec(ctx, vbase + 2, sizeof(C), &rc);
    if (rc) return rc;
    cudaStream_t st = ctx->stream;
    if ((rc = zero_vecs(ctx, sizeof(C) * n, {x}))) return rc;
    VIE_CUDA_TRY(cudaMemcpyAsync(r, b, sizeof(C) * n, cudaMemcpyDeviceToDevice, st), ctx->err);  // :398-400
    {
        DotArgs<C, 1> g{{r}, {r}, {0}};
        if ((rc = dots(ctx, g))) return rc;
        if ((rc = finalize<1>(ctx, kVecBlocks, FinBicgInit{}))) return rc;  // v1 = r^T r (:402-406)
    }
    // p = r / v1 (:413-424)
    if ((rc = lin(ctx, LinArgs<C, 1, 0>{p, 0, {{r, cs(S_T0)}}, {}}))) return rc;
    if ((rc = ctl_init(ctx, thr, maxit, 0.0))) return rc;
    KCtl* ctl = ctx->d_ctl;
    double2* hist = ctx->d_hist;
    const long long nblk = epilogue_blocks(op);
    auto body = [=, &op]() -> int {
        int rc2;
        ctx->gate = Gate{&ctl->state, KS_RUN};
        if ((rc2 = opmv(ctx, op, ProCopy<C>{p, a}, EpiDotU<C>{Ap, p, a}, p, false))) return rc2;  // :437-453
        if ((rc2 = finalize<1>(ctx, nblk, FinBicgAlpha{}))) return rc2;
        // x += alpha p; r -= alpha Ap; v2 = r^T r (:463-479)
        if ((rc2 = lin(ctx, LinArgs<C, 1, 0>{x, 1, {{p, cs(S_ALPHA)}}, {}}))) return rc2;
        if ((rc2 = lin(ctx, LinArgs<C, 1, 1>{r, 1, {{Ap, cs(S_ALPHA, -1.0)}}, {{nullptr, 0}}}))) return rc2;
        if ((rc2 = finalize<1>(ctx, lin_blocks<C, 1, 1>(), FinBicgBeta{}))) return rc2;
        // p += beta r (:489-491); then the stop rule (:497-505)
        if ((rc2 = lin(ctx, LinArgs<C, 1, 0>{p, 1, {{r, cs(S_BETA)}}, {}}))) return rc2;
        return finalize<1>(ctx, 1, then(FinNone{}, DecideErr{ctl, hist}));
    };
    auto fin = [ctx, &res, verbose]() { return finish(ctx, res, 0, 1, PS_ERR_STEPS, verbose, "BiCG"); };
    return launch_or_plan(ctx, plan, body, fin);
}

template <typename T>
static int run_solver(vie_ctx* ctx, Operator<T>& op, int solver, const cplx_t<T>* b, cplx_t<T>* x, double thr,
                      int maxit, int verbose, int vbase, KrylovResult& res, SolvePlan* plan = nullptr) {
    VIE_CUDA_TRY(cudaMemsetAsync(ctx->d_scal, 0, sizeof(double2) * S_COUNT, ctx->stream), ctx->err);
    switch (solver) {
        case VIE_SOLVER_BICGSTAB: return solve_bicgstab<T>(ctx, op, b, x, thr, maxit, verbose, vbase, res, plan);
        case VIE_SOLVER_CORS: return solve_cors<T>(ctx, op, b, x, thr, maxit, verbose, vbase, res, plan);
        case VIE_SOLVER_CG: return solve_cg<T>(ctx, op, b, x, thr, maxit, verbose, vbase, res, plan);
        case VIE_SOLVER_BICG: return solve_bicg<T>(ctx, op, b, x, thr, maxit, verbose, vbase, res, plan);
        case VIE_SOLVER_BICORSTAB: return solve_bicorstab<T>(ctx, op, b, x, thr, maxit, verbose, vbase, res, plan);
        default: return ctx->set_error(VIE_ERR_ARG, "unknown solver " + std::to_string(solver));
    }
}

// ||b - A x|| / ||b|| in FP64; r64 and the scalar slots S_T5 (||r||^2), S_BNRM2 are overwritten
static int true_residual(vie_ctx* ctx, const double2* b, const double2* x, double2* r, double* relres,
                         double2* bn2_slot_value) {
    int rc;
    const long long a = ctx->a;
    if ((rc = opmv(ctx, ctx->op64, ProCopy<double2>{x, a}, EpiResidual<double2>{r, b, a}, x, false))) return rc;
    if ((rc = finalize<1>(ctx, epilogue_blocks(ctx->op64), FinNorm{S_T5}))) return rc;
    if ((rc = read_scalars(ctx))) return rc;
    *relres = std::sqrt(ctx->h_scal[S_T5].x / bn2_slot_value->x);
    return VIE_OK;
}

// BiCGSTAB in FP32 with reliable updates in FP64 (mixed precision).
//
// The recurrences of BICGSTAB_FFT (CG_Iteration.h:591-748) run on FP32 vectors
// with the fused FP32 operator; scalars and inner products stay FP64.  When
// the recursive residual has fallen by `delta` below its largest value since
// the last update (or below the tolerance), the FP32 correction is folded into
// the FP64 solution, r = b - A x is recomputed with the FP64 operator, and that
// true residual replaces the FP32 one (rho and beta follow it).  The Krylov
// directions p, v are kept, so no subspace is lost as in a restart.  The solve
// stops only on the FP64 true residual.  The three phases (FP32 step, FP64
// update, residual replacement) are gated on the control state, so one
// captured body covers all of them.
static int solve_bicgstab_mixed(vie_ctx* ctx, const double2* b64, double2* x64, double tol, double delta,
                                int maxit, int verbose, KrylovResult& res, int& updates, int& mv64,
                                SolvePlan* plan = nullptr) {
    using C = float2;
    int rc = VIE_OK;
    const long long a = ctx->a, n = 3 * a;
    Operator<float>& op = ctx->op32;
    C* r = (C*)work_vec(ctx, 8, sizeof(C), &rc);
    C* p = (C*)work_vec(ctx, 9, sizeof(C), &rc);
    C* v = (C*)work_vec(ctx, 10, sizeof(C), &rc);
    C* sv = (C*)work_vec(ctx, 11, sizeof(C), &rc);
    C* t = (C*)work_vec(ctx, 12, sizeof(C), &rc);
    C* x32 = (C*)work_vec(ctx, 13, sizeof(C), &rc);
    C* b32 = (C*)work_vec(ctx, 14, sizeof(C), &rc);
    double2* r64 = (double2*)work_vec(ctx, 21, sizeof(double2), &rc);
    if (rc) return rc;
    cudaStream_t st = ctx->stream;
    VIE_CUDA_TRY(cudaMemsetAsync(ctx->d_scal, 0, sizeof(double2) * S_COUNT, st), ctx->err);
    VIE_CUDA_TRY(cudaMemsetAsync(x64, 0, sizeof(double2) * n, st), ctx->err);
    if ((rc = zero_vecs(ctx, sizeof(C) * n, {x32, p, v}))) return rc;
    k_to_f32<<<kVecBlocks, 256, 0, st>>>(b32, b64, n, Gate{nullptr, 0});
    count_launch();
    VIE_CUDA_TRY(cudaMemcpyAsync(r, b32, sizeof(C) * n, cudaMemcpyDeviceToDevice, st), ctx->err);
    if ((rc = ctl_init(ctx, tol, maxit, delta))) return rc;
    KCtl* ctl = ctx->d_ctl;
    double2* hist = ctx->d_hist;
    {
        // ||b||^2 from the FP64 right-hand side, rho = b^H r in FP32 data
        DotArgs<double2, 1> g{{b64}, {b64}, {1}};
        if ((rc = dots(ctx, g))) return rc;
        if ((rc = finalize<1>(ctx, kVecBlocks, FinCtlBn2{ctl}))) return rc;
        DotArgs<C, 2> g2{{b32, b32}, {b32, r}, {1, 1}};
        if ((rc = dots(ctx, g2))) return rc;
        if ((rc = finalize<2>(ctx, kVecBlocks, FinBicgstabInit{}))) return rc;
    }
    const long long nblk = epilogue_blocks(op);
    const long long nblk64 = epilogue_blocks(ctx->op64);
    auto body = [=, &op]() -> int {
        int rc2;
        // FP32 BiCGSTAB step
        ctx->gate = Gate{&ctl->state, KS_RUN};
        if ((rc2 = opmv(ctx, op, ProBicgP<C>{r, p, v, ctx->d_scal, a}, EpiDotB<C>{v, b32, a}, p, false))) return rc2;
        if ((rc2 = finalize<1>(ctx, nblk, FinAlpha{}))) return rc2;
        if ((rc2 = opmv(ctx, op, ProBicgS<C>{r, v, sv, ctx->d_scal, a}, EpiDotTS<C>{t, sv, a}, sv, false))) return rc2;
        if ((rc2 = finalize<2>(ctx, nblk, FinOmega{}))) return rc2;
        k_bicgstab_update<C><<<kVecBlocks, 256, 0, ctx->stream>>>(x32, p, sv, t, r, b32, n, ctx->d_scal,
                                                                   ctx->d_partial, ctx->gate);
        count_launch();
        VIE_CUDA_TRY(cudaGetLastError(), ctx->err);
        if ((rc2 = finalize<2>(ctx, kVecBlocks, then(FinBicgstabUpdate{}, DecideReliable{ctl, hist})))) return rc2;
        // reliable update (only when requested): x += x32 in FP64, r64 = b - A x in FP64
        if ((rc2 = cond_begin(ctx, KS_UPDATE))) return rc2;
        ctx->gate = Gate{&ctl->state, KS_UPDATE};
        k_fold_correction<<<kVecBlocks, 256, 0, ctx->stream>>>(x64, x32, n, ctx->gate);
        count_launch();
        VIE_CUDA_TRY(cudaGetLastError(), ctx->err);
        if ((rc2 = opmv(ctx, ctx->op64, ProCopy<double2>{x64, a}, EpiResidual<double2>{r64, b64, a}, x64, false)))
            return rc2;
        if ((rc2 = finalize<1>(ctx, nblk64, then(FinNorm{S_T5}, DecideTrue{ctl, hist})))) return rc2;
        // residual replacement: r32 = float(r64); rho = b^H r and the next beta
        ctx->gate = Gate{&ctl->state, KS_RESET};
        k_to_f32<<<kVecBlocks, 256, 0, ctx->stream>>>(r, r64, n, ctx->gate);
        count_launch();
        VIE_CUDA_TRY(cudaGetLastError(), ctx->err);
        DotArgs<C, 1> g{{b32}, {r}, {1}};
        if ((rc2 = dots(ctx, g))) return rc2;
        if ((rc2 = finalize<1>(ctx, kVecBlocks, then(FinRhoReset{}, DecideResume{ctl})))) return rc2;
        return cond_end(ctx);
    };
    auto fin = [ctx, &res, &updates, &mv64, verbose]() {
        const int rc2 = finish(ctx, res, 0, 2, PS_RELIABLE, verbose, "mixed BiCGSTAB");
        updates = ctx->h_ctl->updates;
        mv64 = updates;
        return rc2;
    };
    return launch_or_plan(ctx, plan, body, fin);
}

// masked FP64 right-hand side b = E_inc . Flag (work slot 20) and ||b||^2
static int prepare_rhs(vie_ctx* ctx, double2** b64_out, double2* bn2_out) {
    int rc = VIE_OK;
    const long long a = ctx->a;
    double2* b64 = (double2*)work_vec(ctx, 20, sizeof(double2), &rc);
    if (rc) return rc;
    k_mask_rhs<double2><<<kVecBlocks, 256, 0, ctx->stream>>>(ctx->d_rhs, ctx->d_flags, b64, a, 1.0);
    count_launch();
    VIE_CUDA_TRY(cudaGetLastError(), ctx->err);
    DotArgs<double2, 1> g{{b64}, {b64}, {1}};
    if ((rc = dots(ctx, g))) return rc;
    if ((rc = finalize<1>(ctx, kVecBlocks, FinNorm{S_BNRM2}))) return rc;
    if ((rc = read_scalars(ctx))) return rc;
    *bn2_out = ctx->h_scal[S_BNRM2];
    *b64_out = b64;
    if (!(bn2_out->x > 0.0)) return ctx->set_error(VIE_ERR_ARG, "right-hand side is zero on every flagged edge");
    return VIE_OK;
}

int solve_driver(vie_ctx* ctx, const vie_solve_params* prm, vie_solve_info* info) {
    int rc = ensure_scalars(ctx);
    if (rc) return rc;
    const long long a = ctx->a, n = 3 * a;
    const int maxit = prm->max_iter > 0 ? prm->max_iter : (int)std::min<long long>(a, 2000000000LL);
    cudaStream_t st = ctx->stream;
    cudaEvent_t e0, e1;
    VIE_CUDA_TRY(cudaEventCreate(&e0), ctx->err);
    VIE_CUDA_TRY(cudaEventCreate(&e1), ctx->err);
    VIE_CUDA_TRY(cudaEventRecord(e0, st), ctx->err);
    vie_solve_info out{};
    out.steps = -1;
    const long long graphs0 = ctx->graph_launches;
    // masked right-hand side b (FP64) in work slot 20, ||b||^2
    double2* b64 = nullptr;
    double2 bn2;
    if ((rc = prepare_rhs(ctx, &b64, &bn2))) return rc;
    int status = VIE_OK;
    if (prm->precision == VIE_PREC_FP64) {
        KrylovResult res;
        rc = run_solver<double>(ctx, ctx->op64, prm->solver, b64, ctx->d_x, prm->tol, maxit, prm->verbose, 0, res);
        if (rc) return rc;
        status = res.status;
        out.steps = res.steps;
        out.iterations = res.iterations;
        out.matvecs_fp64 = res.matvecs;
        out.relres = res.err;
    } else if (prm->precision == VIE_PREC_MIXED && prm->solver == VIE_SOLVER_BICGSTAB) {
        KrylovResult res;
        int updates = 0, mv64 = 0;
        const double delta = prm->inner_tol > 0 ? prm->inner_tol : kReliableDelta;
        rc = solve_bicgstab_mixed(ctx, b64, ctx->d_x, prm->tol, delta, maxit, prm->verbose, res, updates, mv64);
        if (rc && rc != VIE_ERR_BREAKDOWN) return rc;
        status = rc == VIE_ERR_BREAKDOWN ? VIE_ERR_BREAKDOWN : res.status;
        out.steps = res.steps;
        out.iterations = res.iterations;
        out.outer = updates;
        out.matvecs_fp32 = res.matvecs;
        out.matvecs_fp64 = mv64;
        out.relres = res.err;
        ctx->err.code = VIE_OK;
    } else if (prm->precision == VIE_PREC_MIXED) {
        // FP32 inner Krylov inside FP64 defect correction:
        //   r = b - A x (FP64);  solve A d = r / ||r|| in FP32;  x += ||r|| d (FP64)
        // Default inner reduction 5e-5: two refinement steps reach 1e-8.
        // Measured on the 256^3 solar cell with CORS to 1e-8: 2e-4 -> 3 steps,
        // 285 FP32 iterations, 2.30 s; 1e-4 -> 3 steps, 293, 2.37 s; 5e-5, 3e-5
        // and 2e-5 -> 2 steps, 282, 2.27 s.
        const double inner_tol = prm->inner_tol > 0 ? prm->inner_tol : 5e-5;
        const int max_outer = prm->max_outer > 0 ? prm->max_outer : 30;
        double2* r64 = (double2*)work_vec(ctx, 21, sizeof(double2), &rc);
        float2* b32 = (float2*)work_vec(ctx, 22, sizeof(float2), &rc);
        float2* d32 = (float2*)work_vec(ctx, 23, sizeof(float2), &rc);
        if (rc) return rc;
        VIE_CUDA_TRY(cudaMemsetAsync(ctx->d_x, 0, sizeof(double2) * n, st), ctx->err);
        VIE_CUDA_TRY(cudaMemcpyAsync(r64, b64, sizeof(double2) * n, cudaMemcpyDeviceToDevice, st), ctx->err);
        double relres = 1.0;
        double2 rr = bn2;
        int outer = 0;
        while (true) {
            relres = std::sqrt(rr.x / bn2.x);
            if (relres < prm->tol) break;
            if (outer >= max_outer) { status = VIE_ERR_MAXIT; break; }
            if (out.iterations >= maxit) { status = VIE_ERR_MAXIT; break; }
            // r32 = r64 / ||r||
            {
                // put ||r||^2 in S_T5 for the scaling kernels
                VIE_CUDA_TRY(cudaMemcpyAsync(ctx->d_scal + S_T5, &rr, sizeof(double2), cudaMemcpyHostToDevice, st),
                             ctx->err);
                VIE_CUDA_TRY(cudaStreamSynchronize(st), ctx->err);
                k_scale_to<float2><<<kVecBlocks, 256, 0, st>>>(b32, r64, n, ctx->d_scal, S_T5);
                count_launch();
                VIE_CUDA_TRY(cudaGetLastError(), ctx->err);
            }
            KrylovResult res;
            // the last inner solve aims at 0.9 of the reduction still needed: the
            // FP32 recursive residual tracks the true one closely at that depth,
            // and a miss costs one short extra step, not a wrong result (the loop
            // stops only on the FP64 true residual)
            const double itol = std::max(inner_tol, 0.9 * prm->tol / relres);
            rc = run_solver<float>(ctx, ctx->op32, prm->solver, b32, d32, itol, maxit - out.iterations, prm->verbose,
                                   8, res);
            if (rc && rc != VIE_ERR_BREAKDOWN) return rc;
            out.iterations += res.iterations;
            out.matvecs_fp32 += res.matvecs;
            // x += ||r|| d  (scale from S_T5 = ||r||^2 saved before the inner solve overwrote slots)
            VIE_CUDA_TRY(cudaMemcpyAsync(ctx->d_scal + S_T5, &rr, sizeof(double2), cudaMemcpyHostToDevice, st),
                         ctx->err);
            k_accum_d<float2><<<kVecBlocks, 256, 0, st>>>(ctx->d_x, d32, n, ctx->d_scal, S_T5, 1);
            count_launch();
            VIE_CUDA_TRY(cudaGetLastError(), ctx->err);
            // r = b - A x in FP64
            double rel;
            if ((rc = true_residual(ctx, b64, ctx->d_x, r64, &rel, &bn2))) return rc;
            out.matvecs_fp64 += 1;
            rr = ctx->h_scal[S_T5];
            outer++;
            if (res.status == VIE_ERR_BREAKDOWN && rel >= relres) {
                status = VIE_ERR_BREAKDOWN;
                relres = rel;
                break;
            }
        }
        ctx->err.code = VIE_OK;
        out.outer = outer;
        out.relres = std::sqrt(rr.x / bn2.x);
        out.steps = out.iterations > 0 ? out.iterations - 1 : 0;
    } else {
        return ctx->set_error(VIE_ERR_ARG, "unknown precision mode");
    }
    VIE_CUDA_TRY(cudaEventRecord(e1, st), ctx->err);
    VIE_CUDA_TRY(cudaEventSynchronize(e1), ctx->err);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    out.seconds = ms * 1e-3;
    out.graph_loops = (int)(ctx->graph_launches - graphs0);
    // true residual in FP64 (after the timed region): the mixed loop already
    // holds it; an FP64 solve evaluates it on request
    if (prm->precision == VIE_PREC_MIXED) {
        out.true_relres = out.relres;
    } else if (prm->true_residual) {
        double2* r64 = (double2*)work_vec(ctx, 21, sizeof(double2), &rc);
        if (rc) return rc;
        double rel;
        if ((rc = true_residual(ctx, b64, ctx->d_x, r64, &rel, &bn2))) return rc;
        out.true_relres = rel;
    } else {
        out.true_relres = -1.0;
    }
    ctx->have_x = true;
    out.status = status;
    if (info) *info = out;
    if (status == VIE_ERR_MAXIT)
        return ctx->set_error(VIE_ERR_MAXIT, "iteration cap reached before the tolerance");
    if (status == VIE_ERR_BREAKDOWN)
        return ctx->set_error(VIE_ERR_BREAKDOWN, "Krylov breakdown before the tolerance");
    return VIE_OK;
}

// Several solves (one per context, all on one GPU) in one graph launch.  Each
// instance is prepared on its own stream (masked right-hand side, set-up of
// its driver); then one WHILE loop runs, per pass, every live instance's
// iteration body as a parallel IF branch, until every instance has converged,
// broken down or reached its cap.  Supported: FP64 with any driver, mixed
// precision with BiCGSTAB (reliable updates).
int solve_batch_driver(vie_ctx* const* ctxs, int n, const vie_solve_params* prm, vie_solve_info* infos) {
    struct Job {
        vie_ctx* ctx = nullptr;
        double2* b64 = nullptr;
        double2 bn2;
        KrylovResult res;
        int updates = 0, mv64 = 0;
        SolvePlan plan;
        cudaEvent_t ready = nullptr;
    };
    vie_ctx* c0 = ctxs[0];
    const bool mixed = prm->precision == VIE_PREC_MIXED;
    if (mixed && prm->solver != VIE_SOLVER_BICGSTAB)
        return c0->set_error(VIE_ERR_ARG, "batched mixed precision is BiCGSTAB only");
    if (!mixed && prm->precision != VIE_PREC_FP64) return c0->set_error(VIE_ERR_ARG, "unknown precision mode");
    std::vector<Job> jobs((size_t)n);
    cudaStream_t S = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = VIE_OK;
    auto cleanup = [&]() {
        for (auto& j : jobs)
            if (j.ready) cudaEventDestroy(j.ready);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (S) cudaStreamDestroy(S);
    };
    if (cudaStreamCreateWithFlags(&S, cudaStreamNonBlocking) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
        cudaEventCreate(&e1) != cudaSuccess) {
        cleanup();
        return c0->set_error(VIE_ERR_CUDA, "batch stream / events");
    }
    cudaEventRecord(e0, S);
    // prepare every instance on its own stream (after e0, for the timing)
    for (int i = 0; i < n && !rc; i++) {
        Job& j = jobs[i];
        vie_ctx* ctx = j.ctx = ctxs[i];
        if ((rc = ensure_scalars(ctx))) break;
        if (cudaStreamWaitEvent(ctx->stream, e0, 0) != cudaSuccess) { rc = ctx->set_error(VIE_ERR_CUDA, "wait"); break; }
        if ((rc = prepare_rhs(ctx, &j.b64, &j.bn2))) break;
        const int maxit = prm->max_iter > 0 ? prm->max_iter : (int)std::min<long long>(ctx->a, 2000000000LL);
        if (mixed) {
            const double delta = prm->inner_tol > 0 ? prm->inner_tol : kReliableDelta;
            rc = solve_bicgstab_mixed(ctx, j.b64, ctx->d_x, prm->tol, delta, maxit, prm->verbose, j.res, j.updates,
                                      j.mv64, &j.plan);
        } else {
            rc = run_solver<double>(ctx, ctx->op64, prm->solver, j.b64, ctx->d_x, prm->tol, maxit, prm->verbose, 0,
                                    j.res, &j.plan);
        }
        if (rc) break;
        if (cudaEventCreate(&j.ready) != cudaSuccess || cudaEventRecord(j.ready, ctx->stream) != cudaSuccess ||
            cudaStreamWaitEvent(S, j.ready, 0) != cudaSuccess) {
            rc = ctx->set_error(VIE_ERR_CUDA, "batch set-up events");
            break;
        }
    }
    if (rc) {
        if (c0->err.code == VIE_OK && rc) c0->set_error(rc, "batch set-up failed");
        cleanup();
        return rc;
    }
    std::vector<SolvePlan*> plans;
    for (auto& j : jobs) plans.push_back(&j.plan);
    bool launched = false;
    // Each instance's iteration body is a branch of the graph pass.  With
    // VIE_BATCH_FUSED=1, a mixed BiCGSTAB batch on the register kernels runs
    // every pass as one persistent kernel per group of a size class instead
    // (vie_batch.cu): the same bits, a fixed set of kernels per group and pass,
    // but about 10% fewer instances/s on the 176-instance C4 batch, where the
    // branches' short blocks overlap the instances' phases better.
    const char* bf = std::getenv("VIE_BATCH_FUSED");
    bool fused = mixed && c0->use_graphs && bf && bf[0] == '1';
    for (auto& j : jobs) fused = fused && batch_fused_eligible(j.ctx);
    if (fused) {
        std::vector<FusedInstance> fi((size_t)n);
        for (int i = 0; i < n && !rc; i++) {
            vie_ctx* c = jobs[i].ctx;
            FusedInstance& f = fi[i];
            f.ctx = c;
            f.op32 = c->op32.dev;
            f.op64 = c->op64.dev;
            f.a = c->a;
            // the vectors solve_bicgstab_mixed set up (work slots 8-14, 21; b in 20, x the solution)
            f.r = (float2*)work_vec(c, 8, sizeof(float2), &rc);
            f.p = (float2*)work_vec(c, 9, sizeof(float2), &rc);
            f.v = (float2*)work_vec(c, 10, sizeof(float2), &rc);
            f.sv = (float2*)work_vec(c, 11, sizeof(float2), &rc);
            f.t = (float2*)work_vec(c, 12, sizeof(float2), &rc);
            f.x32 = (float2*)work_vec(c, 13, sizeof(float2), &rc);
            f.b32 = (float2*)work_vec(c, 14, sizeof(float2), &rc);
            f.r64 = (double2*)work_vec(c, 21, sizeof(double2), &rc);
            f.b64 = jobs[i].b64;
            f.x64 = c->d_x;
            f.S = c->d_scal;
            f.partial = c->d_partial;
            f.ctl = c->d_ctl;
            f.hist = c->d_hist;
        }
        if (!rc) rc = batch_fused_loop(fi, S, c0, launched);
        for (int i = 0; i < n && launched && !rc; i++) {
            vie_ctx* c = jobs[i].ctx;
            if ((rc = ctl_read(c))) break;
            c->graph_launches++;
        }
    } else if (c0->use_graphs) {
        rc = run_loop_batch_graph(plans, S, c0, launched);
    }
    if (!launched) {
        // the graph could not be built (nothing ran) or graphs are off: the
        // same bodies round-robin from the host, states read back every pass
        if (rc) std::fprintf(stderr, "vie_b200: %s; batch iterating without graphs\n", c0->err.msg.c_str());
        rc = VIE_OK;
        c0->err.code = VIE_OK;
        cudaStreamSynchronize(S);
        std::vector<char> live((size_t)n, 1);
        for (bool any = true; any && !rc;) {
            any = false;
            for (int i = 0; i < n && !rc; i++) {
                if (!live[i]) continue;
                vie_ctx* c = jobs[i].ctx;
                if ((rc = plans[i]->body())) break;
                c->gate = Gate{nullptr, 0};
                k_loop_count<<<1, 1, 0, c->stream>>>(c->d_ctl);
                count_launch();
            }
            for (int i = 0; i < n && !rc; i++) {
                if (!live[i]) continue;
                if ((rc = ctl_read(jobs[i].ctx))) break;
                live[i] = ks_live(jobs[i].ctx->h_ctl->state);
                any = any || live[i];
            }
        }
        for (auto& j : jobs) cudaEventRecord(j.ready, j.ctx->stream), cudaStreamWaitEvent(S, j.ready, 0);
    }
    if (rc) {
        cleanup();
        return rc;
    }
    cudaEventRecord(e1, S);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    int first_err = VIE_OK;
    for (int i = 0; i < n; i++) {
        Job& j = jobs[i];
        vie_ctx* ctx = j.ctx;
        int frc = j.plan.finish();
        vie_solve_info out{};
        out.steps = j.res.steps;
        out.iterations = j.res.iterations;
        out.relres = j.res.err;
        if (mixed) {
            out.outer = j.updates;
            out.matvecs_fp32 = j.res.matvecs;
            out.matvecs_fp64 = j.mv64;
            out.true_relres = j.res.err;
        } else {
            out.matvecs_fp64 = j.res.matvecs;
            out.true_relres = -1.0;
        }
        out.seconds = ms * 1e-3;
        out.graph_loops = launched ? 1 : 0;
        ctx->have_x = true;
        int status = frc;
        if (!status && j.res.status == VIE_ERR_MAXIT)
            status = ctx->set_error(VIE_ERR_MAXIT, "iteration cap reached before the tolerance");
        out.status = status;
        if (infos) infos[i] = out;
        if (status && !first_err) first_err = status;
    }
    cleanup();
    return first_err;
}

// ||b - A x|| / ||b|| of the current solution in FP64 (one operator application)
int residual_driver(vie_ctx* ctx, double* relres) {
    int rc = ensure_scalars(ctx);
    if (rc) return rc;
    const long long a = ctx->a;
    cudaStream_t st = ctx->stream;
    double2* b64 = (double2*)work_vec(ctx, 20, sizeof(double2), &rc);
    double2* r64 = (double2*)work_vec(ctx, 21, sizeof(double2), &rc);
    if (rc) return rc;
    k_mask_rhs<double2><<<kVecBlocks, 256, 0, st>>>(ctx->d_rhs, ctx->d_flags, b64, a, 1.0);
    count_launch();
    VIE_CUDA_TRY(cudaGetLastError(), ctx->err);
    DotArgs<double2, 1> g{{b64}, {b64}, {1}};
    if ((rc = dots(ctx, g))) return rc;
    if ((rc = finalize<1>(ctx, kVecBlocks, FinNorm{S_BNRM2}))) return rc;
    if ((rc = read_scalars(ctx))) return rc;
    double2 bn2 = ctx->h_scal[S_BNRM2];
    if (!(bn2.x > 0.0)) return ctx->set_error(VIE_ERR_ARG, "right-hand side is zero on every flagged edge");
    return true_residual(ctx, b64, ctx->d_x, r64, relres, &bn2);
}

// v *= Flag of component comp (Current_Reset, fft.h:13-35)
__global__ void k_mask_component(double2* __restrict__ v, const unsigned char* __restrict__ flags, long long a,
                                 int comp) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a; i += (long long)gridDim.x * blockDim.x)
        if (!((flags[i] >> comp) & 1)) v[i] = make_double2(0.0, 0.0);
}

void mask_component(double2* v, const unsigned char* flags, long long a, int comp, cudaStream_t st) {
    k_mask_component<<<kVecBlocks, 256, 0, st>>>(v, flags, a, comp);
    count_launch();
}

}  // namespace vie
