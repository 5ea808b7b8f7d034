// vie_batch.cu -- batched mixed-precision BiCGSTAB as persistent multi-instance
// kernels.
//
// The instances of a batch are grouped into size classes (same grid and FFT
// schedule).  Every pass of an iteration is ONE kernel for a whole class: a
// persistent grid-stride loop over the virtual blocks of the instances of the
// class that are in the pass's phase, each virtual block running the same block
// body as the single solve's kernel (vie_fast.cuh *_blk) on that instance's
// descriptor (its operator view, fused prologue / epilogue, vectors, scalars and
// reduction partials).  A list kernel rebuilds, per phase, the instances in it
// from their control blocks: the FP32 step (state RUN), the FP64 reliable update
// (UPDATE) and the residual replacement (RESET), so an instance that has
// converged costs no block at all.  The iteration body of all classes is
// captured once as the child graph of a conditional WHILE node: a whole batch is
// one graph launch.
//
// Every instance computes what its own single solve computes, bit for bit: the
// same block bodies on the same block coordinates (the z rows and y tiles with
// plain loads, which give the staged kernels' results bit for bit), the same
// per-block partial sums of the vector kernels, the same fixed-order finalize
// and the same decisions on its own control block.
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <unordered_map>

#include "vie_batch.h"
#include "vie_krylov.cuh"

namespace vie {
namespace {

// ---------------------------------------------------------------------------
// descriptors
// ---------------------------------------------------------------------------
// one operator application of an instance with its fused prologue / epilogue
template <typename C, class Pro, class Epi> struct OpInst {
    OpDev<C> op;  // first member: the y and x passes read it through a byte stride
    Pro pro;
    Epi epi;
    const C* xdiag;
    double2* partial;
};
template <int K, class Fin> struct FinInst {
    const double2* partial;
    double2* S;
    long long nblk;
    Fin fin;
};
template <typename C> struct UpdInst {  // x += alpha p + omega s; r = s - omega t
    C* x;
    const C* p;
    const C* sv;
    const C* t;
    C* r;
    const C* b;
    long long n;
    const double2* S;
    double2* partial;
};
struct FoldInst {  // x64 += x32; x32 = 0
    double2* x64;
    float2* x32;
    long long n;
};
struct ToInst {  // r32 = float(r64); b^H r32
    float2* r;
    const double2* r64;
    const float2* b;
    long long n;
    double2* partial;
};

// ---------------------------------------------------------------------------
// persistent pass kernels: virtual block vb -> (instance idx[vb / per], rest)
// ---------------------------------------------------------------------------
template <typename C> __device__ __forceinline__ const OpDev<C>& op_at(const char* base, size_t stride, int i) {
    return *reinterpret_cast<const OpDev<C>*>(base + stride * (size_t)i);
}

// F1: per instance 3 components x gx row blocks
template <typename C, int N, class Pro, class Epi>
__global__ void __launch_bounds__(FastLB<C, N>::ROW, FastLB<C, N>::ROW_MIN)
    kb_fwd_z(const OpInst<C, Pro, Epi>* __restrict__ d, const int* __restrict__ idx, const int* __restrict__ cnt, int gx) {
    const long long per = 3LL * gx, total = (long long)(*cnt) * per;
    for (long long vb = blockIdx.x; vb < total; vb += gridDim.x) {
        const OpInst<C, Pro, Epi>& q = d[idx[vb / per]];
        const int rem = (int)(vb % per);
        kf_fwd_z_blk<C, N, Pro>(q.op, q.pro, rem % gx, rem / gx);
        __syncthreads();
    }
}
// I1: the same blocks; reduction partials of the instance at s gx + bx.  The
// operator mode (conj) is a run-time argument as in the single solve's kernel,
// so that the compiler contracts the block body's arithmetic the same way.
template <typename C, int N, class Pro, class Epi>
__global__ void __launch_bounds__(FastLB<C, N>::ROW, FastLB<C, N>::ROW_MIN)
    kb_inv_z(const OpInst<C, Pro, Epi>* __restrict__ d, const int* __restrict__ idx, const int* __restrict__ cnt, int gx,
             int conj) {
    const long long per = 3LL * gx, total = (long long)(*cnt) * per;
    for (long long vb = blockIdx.x; vb < total; vb += gridDim.x) {
        const OpInst<C, Pro, Epi>& q = d[idx[vb / per]];
        const int rem = (int)(vb % per);
        kf_inv_z_blk<C, N, Epi>(q.op, q.xdiag, q.epi, q.partial, conj, rem % gx, rem / gx, gx);
        __syncthreads();
    }
}
// F2 / I2: per instance 3 components x nx x gx kz tiles
template <typename C, int N, bool FWD>
__global__ void __launch_bounds__(FastLB<C, N>::COL, FastLB<C, N>::COL_MIN)
    kb_y(const char* __restrict__ base, size_t stride, const int* __restrict__ idx, const int* __restrict__ cnt, int gx,
         int nx) {
    const long long per = 3LL * nx * gx, total = (long long)(*cnt) * per;
    for (long long vb = blockIdx.x; vb < total; vb += gridDim.x) {
        const OpDev<C>& op = op_at<C>(base, stride, idx[vb / per]);
        const int rem = (int)(vb % per), t = rem / gx;
        if (FWD) kf_fwd_y_blk<C, N>(op, rem % gx, t % nx, t / nx);
        else kf_inv_y_blk<C, N>(op, rem % gx, t % nx, t / nx);
        __syncthreads();
    }
}
// F3: per instance 2 ny x gx kz tiles (conj a run-time argument, as for I1)
template <typename C, int N, int TP>
__global__ void __launch_bounds__(FastXLB<C, TP>::XT, FastXLB<C, TP>::X_MIN)
    kb_x(const char* __restrict__ base, size_t stride, const int* __restrict__ idx, const int* __restrict__ cnt, int gx,
         int ly, int conj) {
    const long long per = (long long)ly * gx, total = (long long)(*cnt) * per;
    for (long long vb = blockIdx.x; vb < total; vb += gridDim.x) {
        const OpDev<C>& op = op_at<C>(base, stride, idx[vb / per]);
        const int rem = (int)(vb % per);
        kf_x_spectral_blk<C, N, TP>(op, conj, rem % gx, rem / gx);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// persistent vector kernels: virtual block bx of kVecBlocks per instance, the
// elements bx * 256 + tid + k * kVecBlocks * 256 (the single solve's blocks)
// ---------------------------------------------------------------------------
template <typename C>
__global__ void __launch_bounds__(256) kb_update(const UpdInst<C>* __restrict__ d, const int* __restrict__ idx,
                                                 const int* __restrict__ cnt) {
    const long long total = (long long)(*cnt) * kVecBlocks;
    const long long stride = (long long)kVecBlocks * 256;
    for (long long vb = blockIdx.x; vb < total; vb += gridDim.x) {
        const UpdInst<C>& q = d[idx[vb / kVecBlocks]];
        const int bx = (int)(vb % kVecBlocks);
        const C alpha = from_d2<C>(q.S[S_ALPHA]), omega = from_d2<C>(q.S[S_OMEGA]);
        double2 acc[2] = {make_double2(0, 0), make_double2(0, 0)};
        for (long long i = (long long)bx * 256 + threadIdx.x; i < q.n; i += stride) {
            const C si = q.sv[i];
            q.x[i] = cadd(cadd(q.x[i], cmul(alpha, q.p[i])), cmul(omega, si));
            const C ri = csub(si, cmul(omega, q.t[i]));
            q.r[i] = ri;
            acc_dotc(acc[0], ri, ri);
            acc_dotc(acc[1], q.b[i], ri);
        }
        block_reduce_store<2>(acc, q.partial, bx);
        __syncthreads();
    }
}
__global__ void __launch_bounds__(256) kb_fold(const FoldInst* __restrict__ d, const int* __restrict__ idx,
                                               const int* __restrict__ cnt) {
    const long long total = (long long)(*cnt) * kVecBlocks;
    const long long stride = (long long)kVecBlocks * 256;
    for (long long vb = blockIdx.x; vb < total; vb += gridDim.x) {
        const FoldInst& q = d[idx[vb / kVecBlocks]];
        const int bx = (int)(vb % kVecBlocks);
        for (long long i = (long long)bx * 256 + threadIdx.x; i < q.n; i += stride) {
            const float2 dv = q.x32[i];
            double2 v = q.x64[i];
            v.x += (double)dv.x;
            v.y += (double)dv.y;
            q.x64[i] = v;
            q.x32[i] = make_float2(0.f, 0.f);
        }
    }
}
// r32 = float(r64), then conj(b) . r32 into the partials (the single solve's
// k_to_f32 and k_dots: the same elements per block)
__global__ void __launch_bounds__(256) kb_to_f32_dot(const ToInst* __restrict__ d, const int* __restrict__ idx,
                                                     const int* __restrict__ cnt) {
    const long long total = (long long)(*cnt) * kVecBlocks;
    const long long stride = (long long)kVecBlocks * 256;
    for (long long vb = blockIdx.x; vb < total; vb += gridDim.x) {
        const ToInst& q = d[idx[vb / kVecBlocks]];
        const int bx = (int)(vb % kVecBlocks);
        double2 acc[1] = {make_double2(0, 0)};
        for (long long i = (long long)bx * 256 + threadIdx.x; i < q.n; i += stride) {
            const float2 ri = make_float2((float)q.r64[i].x, (float)q.r64[i].y);
            q.r[i] = ri;
            acc_dotc(acc[0], q.b[i], ri);
        }
        block_reduce_store<1>(acc, q.partial, bx);
        __syncthreads();
    }
}

// finalize of every listed instance: the fixed-order sum of k_finalize
template <int K, class Fin>
__global__ void __launch_bounds__(256) kb_finalize(const FinInst<K, Fin>* __restrict__ d, const int* __restrict__ idx,
                                                   const int* __restrict__ cnt) {
    __shared__ double2 red[K][256];
    const int n = *cnt;
    for (int j = blockIdx.x; j < n; j += gridDim.x) {
        const FinInst<K, Fin>& q = d[idx[j]];
        for (int k = 0; k < K; k++) {
            double rx = 0, ry = 0;
            for (long long b = threadIdx.x; b < q.nblk; b += blockDim.x) {
                const double2 v = q.partial[b * K + k];
                rx += v.x;
                ry += v.y;
            }
            red[k][threadIdx.x] = make_double2(rx, ry);
        }
        __syncthreads();
        for (int h = 128; h > 0; h >>= 1) {
            if (threadIdx.x < h)
                for (int k = 0; k < K; k++) {
                    red[k][threadIdx.x].x += red[k][threadIdx.x + h].x;
                    red[k][threadIdx.x].y += red[k][threadIdx.x + h].y;
                }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            double2 dd[K];
            for (int k = 0; k < K; k++) dd[k] = red[k][0];
            q.fin(q.S, dd);
        }
        __syncthreads();
    }
}

// the instances of a class in `state`, in batch order; the RUN list also counts
// one executed iteration body for each instance in it
__global__ void kb_list(KCtl* const* __restrict__ ctls, int n, int state, int* __restrict__ idx, int* __restrict__ cnt,
                        int count_loop) {
    if (threadIdx.x != 0) return;
    int m = 0;
    for (int i = 0; i < n; i++) {
        KCtl* c = ctls[i];
        if (c->state == state) {
            idx[m++] = i;
            if (count_loop) c->loops++;
        }
    }
    *cnt = m;
}
// end of a pass: loop again while any instance of the batch is live
__global__ void kb_cond(KCtl* const* __restrict__ ctls, int n, cudaGraphConditionalHandle h, int* passes) {
    int any = 0;
    for (int i = threadIdx.x; i < n; i += 32) {
        const int s = ctls[i]->state;
        any |= (s == KS_RUN || s == KS_UPDATE || s == KS_RESET) ? 1 : 0;
    }
    any = __any_sync(0xffffffffu, any);
    if (threadIdx.x == 0) {
        (*passes)++;
        cudaGraphSetConditional(h, any ? 1u : 0u);
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
// the passes of one operator application for the listed instances of a class,
// each with the block shape and shared memory of the single solve's kernel
template <typename C, int N, class Pro, class Epi>
int lb_fwd_z(const OpInst<C, Pro, Epi>* d, const int* idx, const int* cnt, long long nrows, cudaStream_t st, Error& err) {
    constexpr int ROWS = fast_rows<C, N>(), L = fast_lanes<C, N>();
    constexpr size_t smem = fast_smem_row<C, N>();
    auto k = kb_fwd_z<C, N, Pro, Epi>;
    VIE_CUDA_TRY(ensure_smem(k, smem), err);
    k<<<persistent_grid(k, L * ROWS, smem), L * ROWS, smem, st>>>(d, idx, cnt, (int)ceil_div(nrows, ROWS));
    count_launch();
    return VIE_OK;
}
template <typename C, int N, class Pro, class Epi>
int lb_inv_z(const OpInst<C, Pro, Epi>* d, const int* idx, const int* cnt, long long nrows, cudaStream_t st, Error& err) {
    constexpr int ROWS = fast_rows<C, N>(), L = fast_lanes<C, N>();
    constexpr size_t smem = fast_smem_row<C, N>();
    auto k = kb_inv_z<C, N, Pro, Epi>;
    VIE_CUDA_TRY(ensure_smem(k, smem), err);
    k<<<persistent_grid(k, L * ROWS, smem), L * ROWS, smem, st>>>(d, idx, cnt, (int)ceil_div(nrows, ROWS), 0);
    count_launch();
    return VIE_OK;
}
template <typename C, int N, bool FWD>
int lb_y(const char* base, size_t stride, const int* idx, const int* cnt, int nx, int nz, cudaStream_t st, Error& err) {
    constexpr int TP = FastTiles<C>::TP_Y, L = fast_lanes<C, N>();
    constexpr size_t smem = fast_smem_col<C, N>();
    auto k = kb_y<C, N, FWD>;
    VIE_CUDA_TRY(ensure_smem(k, smem), err);
    k<<<persistent_grid(k, TP * L, smem), TP * L, smem, st>>>(base, stride, idx, cnt, (int)ceil_div(2 * nz, TP), nx);
    count_launch();
    return VIE_OK;
}
template <typename C, int N, int TP>
int lb_x_tp(const char* base, size_t stride, const int* idx, const int* cnt, int ny, int nz, cudaStream_t st,
            Error& err) {
    constexpr size_t smem = fast_smem_x<C, N, TP>();
    constexpr int th = fast_x_threads<C, N, TP>();
    auto k = kb_x<C, N, TP>;
    VIE_CUDA_TRY(ensure_smem(k, smem), err);
    k<<<persistent_grid(k, th, smem), th, smem, st>>>(base, stride, idx, cnt, (int)ceil_div(2 * nz, TP), 2 * ny, 0);
    count_launch();
    return VIE_OK;
}
template <typename C, int N>
int lb_x(const char* base, size_t stride, const int* idx, const int* cnt, int ny, int nz, int xalt, cudaStream_t st,
         Error& err) {
    if (xalt) return lb_x_tp<C, N, FastTiles<C>::TP_X / 2>(base, stride, idx, cnt, ny, nz, st, err);
    return lb_x_tp<C, N, FastTiles<C>::TP_X>(base, stride, idx, cnt, ny, nz, st, err);
}

template <typename C, class Pro, class Epi>
int launch_op_batch(const OpInst<C, Pro, Epi>* d, const int* idx, const int* cnt, int nx, int ny, int nz, int xalt,
                    cudaStream_t st, Error& err) {
    using I = OpInst<C, Pro, Epi>;
    const char* base = reinterpret_cast<const char*>(d);
    const long long nrows = (long long)nx * ny;
    int rc = VIE_ERR_ARG;
    VIE_FAST_SWITCH(nz, rc = (lb_fwd_z<C, NN, Pro, Epi>(d, idx, cnt, nrows, st, err)));
    if (rc) return rc;
    rc = VIE_ERR_ARG;
    VIE_FAST_SWITCH(ny, rc = (lb_y<C, NN, true>(base, sizeof(I), idx, cnt, nx, nz, st, err)));
    if (rc) return rc;
    rc = VIE_ERR_ARG;
    VIE_FAST_SWITCH(nx, rc = (lb_x<C, NN>(base, sizeof(I), idx, cnt, ny, nz, xalt, st, err)));
    if (rc) return rc;
    rc = VIE_ERR_ARG;
    VIE_FAST_SWITCH(ny, rc = (lb_y<C, NN, false>(base, sizeof(I), idx, cnt, nx, nz, st, err)));
    if (rc) return rc;
    rc = VIE_ERR_ARG;
    VIE_FAST_SWITCH(nz, rc = (lb_inv_z<C, NN, Pro, Epi>(d, idx, cnt, nrows, st, err)));
    if (rc) return rc;  // (a length without a register plan is rejected by batch_fused_eligible)
    VIE_CUDA_TRY(cudaGetLastError(), err);
    return VIE_OK;
}

template <int K, class Fin>
int launch_fin_batch(const FinInst<K, Fin>* d, const int* idx, const int* cnt, int n, cudaStream_t st, Error& err) {
    kb_finalize<K, Fin><<<n, 256, 0, st>>>(d, idx, cnt);
    count_launch();
    VIE_CUDA_TRY(cudaGetLastError(), err);
    return VIE_OK;
}

// device arena of one batch: descriptors of every class, lists, control pointers
struct Arena {
    std::vector<unsigned char> host;
    size_t put(const void* p, size_t bytes) {
        const size_t off = align_up(host.size(), 256);
        host.resize(off + bytes);
        if (p) std::memcpy(host.data() + off, p, bytes);
        return off;
    }
};

using InstP = OpInst<float2, ProBicgP<float2>, EpiDotB<float2>>;
using InstS = OpInst<float2, ProBicgS<float2>, EpiDotTS<float2>>;
using InstR = OpInst<double2, ProCopy<double2>, EpiResidual<double2>>;
using FinA = FinInst<1, FinAlpha>;
using FinO = FinInst<2, FinOmega>;
using FinU = FinInst<2, FinThen<FinBicgstabUpdate, DecideReliable>>;
using FinT = FinInst<1, FinThen<FinNorm, DecideTrue>>;
using FinR = FinInst<1, FinThen<FinRhoReset, DecideResume>>;

struct ClassPlan {
    int nx, ny, nz, xalt32, xalt64;
    std::vector<int> members;  // indices into the batch
    // arena offsets
    size_t ip, is, ir, fa, fo, fu, ft, fr, upd, fold, to, ctls, run, upd_l, rst;
};

}  // namespace

bool batch_fused_eligible(const vie_ctx* ctx) {
    for (int ax = 0; ax < 3; ax++)
        if (!ctx->op32.dev.fast[ax] || !ctx->op64.dev.fast[ax]) return false;
    return ctx->op32.ready && ctx->op64.ready;
}

int batch_fused_loop(std::vector<FusedInstance>& inst, cudaStream_t S, vie_ctx* ectx, bool& launched) {
    launched = false;
    const int n = (int)inst.size();
    // size classes (grid and x-pass tiles of both operators), cut into groups of
    // at most `chunk` instances: each group is one branch of the graph pass, so
    // the groups' compute-bound x passes overlap other groups' memory-bound
    // passes, while the kernels per pass stay independent of the instance count
    // within a group.  VIE_BATCH_CHUNK sets the group size (default 16).
    int chunk = 16;
    if (const char* cv = std::getenv("VIE_BATCH_CHUNK")) chunk = std::max(1, std::atoi(cv));
    std::map<std::tuple<int, int, int, int, int>, int> key_to_class;
    std::vector<ClassPlan> classes;
    for (int i = 0; i < n; i++) {
        const FusedInstance& f = inst[i];
        const auto key = std::make_tuple(f.op32.nx, f.op32.ny, f.op32.nz, f.op32.xalt, f.op64.xalt);
        auto it = key_to_class.find(key);
        if (it == key_to_class.end() || (int)classes[it->second].members.size() >= chunk) {
            ClassPlan cp{};
            cp.nx = f.op32.nx; cp.ny = f.op32.ny; cp.nz = f.op32.nz; cp.xalt32 = f.op32.xalt; cp.xalt64 = f.op64.xalt;
            classes.push_back(cp);
            key_to_class[key] = (int)classes.size() - 1;
            it = key_to_class.find(key);
        }
        classes[it->second].members.push_back(i);
    }
    // descriptors
    Arena ar;
    std::vector<KCtl*> all_ctls((size_t)n);
    for (int i = 0; i < n; i++) all_ctls[i] = inst[i].ctl;
    const size_t off_all = ar.put(all_ctls.data(), sizeof(KCtl*) * n);
    const size_t off_passes = ar.put(nullptr, sizeof(int));
    for (ClassPlan& cp : classes) {
        const int m = (int)cp.members.size();
        std::vector<InstP> ip(m);
        std::vector<InstS> is(m);
        std::vector<InstR> ir(m);
        std::vector<FinA> fa(m);
        std::vector<FinO> fo(m);
        std::vector<FinU> fu(m);
        std::vector<FinT> ft(m);
        std::vector<FinR> fr(m);
        std::vector<UpdInst<float2>> up(m);
        std::vector<FoldInst> fold(m);
        std::vector<ToInst> to(m);
        std::vector<KCtl*> ctls(m);
        for (int j = 0; j < m; j++) {
            FusedInstance& f = inst[cp.members[j]];
            vie_ctx* c = f.ctx;
            const long long a = f.a, nn = 3 * a;
            // the operator views with plain loads and no gate (the lists select the instances)
            OpDev<float2> o32 = f.op32;
            o32.gate = Gate{nullptr, 0};
            o32.zstage = 0;
            OpDev<double2> o64 = f.op64;
            o64.gate = Gate{nullptr, 0};
            o64.zstage = 0;
            const long long nb32 = epilogue_blocks(c->op32), nb64 = epilogue_blocks(c->op64);
            ip[j] = InstP{o32, ProBicgP<float2>{f.r, f.p, f.v, f.S, a}, EpiDotB<float2>{f.v, f.b32, a}, f.p, f.partial};
            is[j] = InstS{o32, ProBicgS<float2>{f.r, f.v, f.sv, f.S, a}, EpiDotTS<float2>{f.t, f.sv, a}, f.sv, f.partial};
            ir[j] = InstR{o64, ProCopy<double2>{f.x64, a}, EpiResidual<double2>{f.r64, f.b64, a}, f.x64, f.partial};
            fa[j] = FinA{f.partial, f.S, nb32, FinAlpha{}};
            fo[j] = FinO{f.partial, f.S, nb32, FinOmega{}};
            fu[j] = FinU{f.partial, f.S, (long long)kVecBlocks, then(FinBicgstabUpdate{}, DecideReliable{f.ctl, f.hist})};
            ft[j] = FinT{f.partial, f.S, nb64, then(FinNorm{S_T5}, DecideTrue{f.ctl, f.hist})};
            fr[j] = FinR{f.partial, f.S, (long long)kVecBlocks, then(FinRhoReset{}, DecideResume{f.ctl})};
            up[j] = UpdInst<float2>{f.x32, f.p, f.sv, f.t, f.r, f.b32, nn, f.S, f.partial};
            fold[j] = FoldInst{f.x64, f.x32, nn};
            to[j] = ToInst{f.r, f.r64, f.b32, nn, f.partial};
            ctls[j] = f.ctl;
        }
        cp.ip = ar.put(ip.data(), sizeof(InstP) * m);
        cp.is = ar.put(is.data(), sizeof(InstS) * m);
        cp.ir = ar.put(ir.data(), sizeof(InstR) * m);
        cp.fa = ar.put(fa.data(), sizeof(FinA) * m);
        cp.fo = ar.put(fo.data(), sizeof(FinO) * m);
        cp.fu = ar.put(fu.data(), sizeof(FinU) * m);
        cp.ft = ar.put(ft.data(), sizeof(FinT) * m);
        cp.fr = ar.put(fr.data(), sizeof(FinR) * m);
        cp.upd = ar.put(up.data(), sizeof(UpdInst<float2>) * m);
        cp.fold = ar.put(fold.data(), sizeof(FoldInst) * m);
        cp.to = ar.put(to.data(), sizeof(ToInst) * m);
        cp.ctls = ar.put(ctls.data(), sizeof(KCtl*) * m);
        cp.run = ar.put(nullptr, sizeof(int) * (m + 1));  // [count, idx...]
        cp.upd_l = ar.put(nullptr, sizeof(int) * (m + 1));
        cp.rst = ar.put(nullptr, sizeof(int) * (m + 1));
    }
    unsigned char* dmem = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<cudaStream_t> cs(classes.size(), nullptr);
    std::vector<cudaEvent_t> join(classes.size(), nullptr);
    cudaEvent_t fork = nullptr;
    int rc = VIE_OK;
    long long per = 0;
    Error& err = ectx->err;
    do {
        if (cudaMalloc(&dmem, ar.host.size()) != cudaSuccess) { rc = ectx->set_error(VIE_ERR_ALLOC, "batch descriptors"); break; }
        if (cudaMemcpy(dmem, ar.host.data(), ar.host.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
            rc = ectx->set_error(VIE_ERR_CUDA, "batch descriptor upload");
            break;
        }
        bool ok = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming) == cudaSuccess;
        for (size_t k = 0; k < classes.size() && ok; k++)
            ok = cudaStreamCreateWithFlags(&cs[k], cudaStreamNonBlocking) == cudaSuccess &&
                 cudaEventCreateWithFlags(&join[k], cudaEventDisableTiming) == cudaSuccess;
        if (!ok) { rc = ectx->set_error(VIE_ERR_CUDA, "batch streams / events"); break; }
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
        if (cudaStreamBeginCaptureToGraph(S, wp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                          cudaStreamCaptureModeRelaxed) != cudaSuccess) {
            rc = ectx->set_error(VIE_ERR_CUDA, "stream capture of the batch body");
            break;
        }
        const long long n0 = g_launches.load();
        cudaEventRecord(fork, S);
        int brc = VIE_OK;
        for (size_t k = 0; k < classes.size() && !brc; k++) {
            const ClassPlan& cp = classes[k];
            const int m = (int)cp.members.size();
            cudaStream_t st = cs[k];
            auto P = [&](size_t off) { return dmem + off; };
            int* run = reinterpret_cast<int*>(P(cp.run));
            int* updl = reinterpret_cast<int*>(P(cp.upd_l));
            int* rst = reinterpret_cast<int*>(P(cp.rst));
            KCtl* const* ctls = reinterpret_cast<KCtl* const*>(P(cp.ctls));
            cudaStreamWaitEvent(st, fork, 0);
            // FP32 BiCGSTAB step of the instances in RUN
            kb_list<<<1, 32, 0, st>>>(ctls, m, KS_RUN, run + 1, run, 1);
            count_launch();
            if ((brc = launch_op_batch(reinterpret_cast<const InstP*>(P(cp.ip)), run + 1, run, cp.nx, cp.ny, cp.nz,
                                       cp.xalt32, st, err))) break;
            if ((brc = launch_fin_batch(reinterpret_cast<const FinA*>(P(cp.fa)), run + 1, run, m, st, err))) break;
            if ((brc = launch_op_batch(reinterpret_cast<const InstS*>(P(cp.is)), run + 1, run, cp.nx, cp.ny, cp.nz,
                                       cp.xalt32, st, err))) break;
            if ((brc = launch_fin_batch(reinterpret_cast<const FinO*>(P(cp.fo)), run + 1, run, m, st, err))) break;
            kb_update<float2><<<persistent_grid(kb_update<float2>, 256, 0), 256, 0, st>>>(
                reinterpret_cast<const UpdInst<float2>*>(P(cp.upd)), run + 1, run);
            count_launch();
            if ((brc = launch_fin_batch(reinterpret_cast<const FinU*>(P(cp.fu)), run + 1, run, m, st, err))) break;
            // reliable update of the instances that asked for one: x += x32, r64 = b - A x in FP64
            kb_list<<<1, 32, 0, st>>>(ctls, m, KS_UPDATE, updl + 1, updl, 0);
            count_launch();
            kb_fold<<<persistent_grid(kb_fold, 256, 0), 256, 0, st>>>(reinterpret_cast<const FoldInst*>(P(cp.fold)),
                                                                        updl + 1, updl);
            count_launch();
            if ((brc = launch_op_batch(reinterpret_cast<const InstR*>(P(cp.ir)), updl + 1, updl, cp.nx, cp.ny, cp.nz,
                                       cp.xalt64, st, err))) break;
            if ((brc = launch_fin_batch(reinterpret_cast<const FinT*>(P(cp.ft)), updl + 1, updl, m, st, err))) break;
            // residual replacement: r32 = float(r64), rho = b^H r
            kb_list<<<1, 32, 0, st>>>(ctls, m, KS_RESET, rst + 1, rst, 0);
            count_launch();
            kb_to_f32_dot<<<persistent_grid(kb_to_f32_dot, 256, 0), 256, 0, st>>>(
                reinterpret_cast<const ToInst*>(P(cp.to)), rst + 1, rst);
            count_launch();
            if ((brc = launch_fin_batch(reinterpret_cast<const FinR*>(P(cp.fr)), rst + 1, rst, m, st, err))) break;
            cudaEventRecord(join[k], st);
            cudaStreamWaitEvent(S, join[k], 0);
        }
        kb_cond<<<1, 32, 0, S>>>(reinterpret_cast<KCtl* const*>(dmem + off_all), n, hw,
                                 reinterpret_cast<int*>(dmem + off_passes));
        count_launch();
        cudaGraph_t captured = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(S, &captured);
        per = g_launches.load() - n0;
        count_launch(-per);
        if (brc) { rc = brc; break; }
        if (ce != cudaSuccess) {
            rc = ectx->set_error(VIE_ERR_CUDA, std::string("capture of the batch body: ") + cudaGetErrorString(ce));
            break;
        }
        if (cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
            rc = ectx->set_error(VIE_ERR_CUDA, "batch graph instantiation");
            break;
        }
        if (cudaMemsetAsync(dmem + off_passes, 0, sizeof(int), S) != cudaSuccess) {
            rc = ectx->set_error(VIE_ERR_CUDA, "batch pass counter");
            break;
        }
        launched = true;
        if (cudaGraphLaunch(exec, S) != cudaSuccess || cudaStreamSynchronize(S) != cudaSuccess) {
            rc = ectx->set_error(VIE_ERR_CUDA, std::string("batch graph: ") + cudaGetErrorString(cudaGetLastError()));
            break;
        }
        int passes = 0;
        if (cudaMemcpy(&passes, dmem + off_passes, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
            rc = ectx->set_error(VIE_ERR_CUDA, "batch pass count");
            break;
        }
        count_launch(per * passes);
    } while (0);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (auto e : join)
        if (e) cudaEventDestroy(e);
    for (auto st : cs)
        if (st) cudaStreamDestroy(st);
    if (fork) cudaEventDestroy(fork);
    if (dmem) cudaFree(dmem);
    if (rc && !launched) (void)cudaGetLastError();
    return rc;
}

}  // namespace vie
