// vie_krylov.cuh -- device side of the Krylov drivers shared by the single and the
// batched solves: FP64 complex helpers, the fixed-order finalize reduction, the
// scalar programs and stop decisions, the fused prologue / epilogue functors of
// the operator passes and the grid-stride vector kernels.
#pragma once
#include "vie_launch.cuh"

namespace vie {

// ---------------------------------------------------------------------------
// device complex helpers on double2
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 ddiv(double2 a, double2 b) {
    // Smith's scaled division
    if (fabs(b.x) >= fabs(b.y)) {
        const double r = b.y / b.x, d = b.x + b.y * r;
        return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
    }
    const double r = b.x / b.y, d = b.x * r + b.y;
    return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
}
__device__ __forceinline__ double2 dmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ bool dfinite(double2 a) { return isfinite(a.x) && isfinite(a.y); }

template <typename C> __device__ __forceinline__ C coef_c(double2 v) { return from_d2<C>(v); }

// conj(u) * v accumulated in FP64
template <typename C> __device__ __forceinline__ void acc_dotc(double2& acc, C u, C v) {
    const double ux = u.x, uy = u.y, vx = v.x, vy = v.y;
    acc.x += ux * vx + uy * vy;
    acc.y += ux * vy - uy * vx;
}
template <typename C> __device__ __forceinline__ void acc_dotu(double2& acc, C u, C v) {
    const double ux = u.x, uy = u.y, vx = v.x, vy = v.y;
    acc.x += ux * vx - uy * vy;
    acc.y += ux * vy + uy * vx;
}

// ---------------------------------------------------------------------------
// finalize: fixed-order sum of the partials, then a scalar update on thread 0
// ---------------------------------------------------------------------------
template <int K, class Fin>
__global__ void __launch_bounds__(256) k_finalize(const double2* __restrict__ partial, long long nblk, double2* S,
                                                  Fin fin, Gate gate) {
    if (gate_closed(gate)) return;
    __shared__ double2 red[K][256];
    for (int k = 0; k < K; k++) {
        double rx = 0, ry = 0;
        for (long long b = threadIdx.x; b < nblk; b += blockDim.x) {
            const double2 v = partial[b * K + k];
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
        double2 d[K];
        for (int k = 0; k < K; k++) d[k] = red[k][0];
        fin(S, d);
    }
}

// scalar programs -----------------------------------------------------------
struct FinStore1 {  // S[slot] = d0
    int slot;
    __device__ void operator()(double2* S, const double2* d) const { S[slot] = d[0]; }
};
struct FinStore2 {
    int s0, s1;
    __device__ void operator()(double2* S, const double2* d) const { S[s0] = d[0]; S[s1] = d[1]; }
};
// BiCGSTAB -------------------------------------------------------------------
struct FinBicgstabInit {  // d0 = b^H b, d1 = b^H r
    __device__ void operator()(double2* S, const double2* d) const {
        S[S_BNRM2] = d[0];
        S[S_RHO] = d[1];
        S[S_OMEGA] = make_double2(1.0, 0.0);  // :587-588
        S[S_ALPHA] = make_double2(0.0, 0.0);
        S[S_NAN] = make_double2(0.0, 0.0);
    }
};
struct FinAlpha {  // alpha = rho / d0
    __device__ void operator()(double2* S, const double2* d) const {
        S[S_ALPHA] = ddiv(S[S_RHO], d[0]);
        if (!dfinite(S[S_ALPHA])) S[S_NAN] = make_double2(1.0, 0.0);
    }
};
struct FinOmega {  // omega = (t^H s) / (t^H t)
    __device__ void operator()(double2* S, const double2* d) const {
        S[S_OMEGA] = ddiv(d[0], d[1]);
        if (!dfinite(S[S_OMEGA])) S[S_NAN] = make_double2(1.0, 0.0);
    }
};
struct FinBicgstabUpdate {  // d0 = r^H r, d1 = b^H r(new)
    __device__ void operator()(double2* S, const double2* d) const {
        S[S_RR] = d[0];
        S[S_ERR] = make_double2(sqrt(d[0].x / S[S_BNRM2].x), 0.0);  // :734
        const double2 rho_new = d[1];
        // beta = (rho / rho_1) (alpha / omega)  (:603-609), for the next iteration
        S[S_BETA] = dmul(ddiv(rho_new, S[S_RHO]), ddiv(S[S_ALPHA], S[S_OMEGA]));
        S[S_RHO1] = S[S_RHO];
        S[S_RHO] = rho_new;
        if (!dfinite(S[S_ERR]) || !dfinite(S[S_BETA])) S[S_NAN] = make_double2(1.0, 0.0);
    }
};
// CORS -----------------------------------------------------------------------
struct FinCorsRho {  // d0 = b^H A r
    const KCtl* ctl;
    __device__ void operator()(double2* S, const double2* d) const {
        S[S_RHO] = d[0];
        if (ctl->iter > 0) {
            const double2 beta = ddiv(d[0], S[S_RHO1]);  // :874-878
            S[S_BETA] = beta;
            S[S_T0] = dmul(beta, beta);
        }
        if (!dfinite(S[S_RHO]) || !dfinite(S[S_BETA])) S[S_NAN] = make_double2(1.0, 0.0);
    }
};
struct FinCorsAlpha {  // d0 = b^H A q
    __device__ void operator()(double2* S, const double2* d) const {
        const double2 al = ddiv(S[S_RHO], d[0]);  // :951-962
        S[S_ALPHA] = al;
        S[S_T1] = dmul(al, al);
        if (!dfinite(al)) S[S_NAN] = make_double2(1.0, 0.0);
    }
};
struct FinErr {  // d0 = r^H r; err = sqrt(rr / bnrm2); rho_1 = rho
    __device__ void operator()(double2* S, const double2* d) const {
        S[S_RR] = d[0];
        S[S_ERR] = make_double2(sqrt(d[0].x / S[S_BNRM2].x), 0.0);
        S[S_RHO1] = S[S_RHO];
        if (!dfinite(S[S_ERR])) S[S_NAN] = make_double2(1.0, 0.0);
    }
};
// BiCORSTAB ------------------------------------------------------------------
struct FinBicorRho {  // d0 = b^H A r
    const KCtl* ctl;
    __device__ void operator()(double2* S, const double2* d) const {
        S[S_RHO] = d[0];
        if (ctl->iter > 0) {
            S[S_BETA] = dmul(ddiv(d[0], S[S_RHO1]), ddiv(S[S_ALPHA], S[S_OMEGA]));  // :1167-1173
            S[S_T2] = dmul(S[S_BETA], S[S_OMEGA]);  // beta * omega of the previous step
        }
        if (!dfinite(S[S_RHO]) || !dfinite(S[S_BETA])) S[S_NAN] = make_double2(1.0, 0.0);
    }
};
struct FinBicorOmega {  // S_T3 = conj(pc)^T qc, S_T4 = qc^H qc  ->  omega = conj(S_T3) / S_T4
    __device__ void operator()(double2* S, const double2* d) const {
        const double2 num = make_double2(d[0].x, -d[0].y);
        S[S_OMEGA] = ddiv(num, d[1]);
        if (!dfinite(S[S_OMEGA])) S[S_NAN] = make_double2(1.0, 0.0);
    }
};
// CG (CGNR) ------------------------------------------------------------------
struct FinCgInit {  // d0 = ||p||^2 (v3), d1 = ||b||^2 (vx)
    __device__ void operator()(double2* S, const double2* d) const {
        S[S_T0] = d[0];
        S[S_BNRM2] = d[1];
        S[S_NAN] = make_double2(0.0, 0.0);
    }
};
struct FinCgAlpha {  // d0 = ||Ap||^2 (v2); alpha = v1 / v2 with v1 = v3
    __device__ void operator()(double2* S, const double2* d) const {
        S[S_T1] = S[S_T0];  // v1 = v3
        S[S_ALPHA] = make_double2(S[S_T1].x / d[0].x, 0.0);
        if (!dfinite(S[S_ALPHA])) S[S_NAN] = make_double2(1.0, 0.0);
    }
};
struct FinCgBeta {  // d0 = ||q||^2 (v3); beta = v3 / v1
    __device__ void operator()(double2* S, const double2* d) const {
        S[S_T0] = d[0];
        S[S_BETA] = make_double2(d[0].x / S[S_T1].x, 0.0);
        if (!dfinite(S[S_BETA])) S[S_NAN] = make_double2(1.0, 0.0);
    }
};
struct FinCgErr {  // d0 = ||r||^2 (v4); err = v4 / vx (not rooted, :323)
    __device__ void operator()(double2* S, const double2* d) const {
        S[S_RR] = d[0];
        S[S_ERR] = make_double2(d[0].x / S[S_BNRM2].x, 0.0);
        if (!dfinite(S[S_ERR])) S[S_NAN] = make_double2(1.0, 0.0);
    }
};
// BiCG -------------------------------------------------------------------------
struct FinBicgInit {  // d0 = r^T r
    __device__ void operator()(double2* S, const double2* d) const {
        S[S_BNRM2] = d[0];  // vx
        S[S_T0] = ddiv(make_double2(1.0, 0.0), d[0]);  // 1/v1
        S[S_NAN] = make_double2(0.0, 0.0);
    }
};
struct FinBicgAlpha {  // d0 = Ap^T p; alpha = 1/v1
    __device__ void operator()(double2* S, const double2* d) const {
        S[S_ALPHA] = ddiv(make_double2(1.0, 0.0), d[0]);
        if (!dfinite(S[S_ALPHA])) S[S_NAN] = make_double2(1.0, 0.0);
    }
};
struct FinBicgBeta {  // d0 = r^T r (v2); beta = 1/v2; err = sqrt(|v2|^2/|vx|^2)
    __device__ void operator()(double2* S, const double2* d) const {
        const double2 v2 = d[0], vx = S[S_BNRM2];
        S[S_BETA] = ddiv(make_double2(1.0, 0.0), v2);
        S[S_ERR] = make_double2(sqrt((v2.x * v2.x + v2.y * v2.y) / (vx.x * vx.x + vx.y * vx.y)), 0.0);
        if (!dfinite(S[S_ERR]) || !dfinite(S[S_BETA])) S[S_NAN] = make_double2(1.0, 0.0);
    }
};
// reliable update: rho := b^H r for the replaced residual and the beta of the next step
struct FinRhoReset {  // d0 = b^H r(true)
    __device__ void operator()(double2* S, const double2* d) const {
        S[S_RHO] = d[0];
        S[S_BETA] = dmul(ddiv(d[0], S[S_RHO1]), ddiv(S[S_ALPHA], S[S_OMEGA]));
        if (!dfinite(S[S_BETA])) S[S_NAN] = make_double2(1.0, 0.0);
    }
};
// refinement -------------------------------------------------------------------
struct FinNorm {  // S[slot] = d0 (a squared norm)
    int slot;
    __device__ void operator()(double2* S, const double2* d) const { S[slot] = d[0]; }
};
struct FinNone {  // decision only (the scalars are already in place)
    __device__ void operator()(double2*, const double2*) const {}
};
struct FinCtlBn2 {  // FP64 ||b||^2 of the mixed solve into the control block (also the first residual maximum)
    KCtl* ctl;
    __device__ void operator()(double2* S, const double2* d) const {
        ctl->bn2 = d[0].x;
        ctl->rmax2 = d[0].x;
    }
};

// stop decisions ------------------------------------------------------------------
// a finalize step followed by a decision on the control block
template <class F, class D> struct FinThen {
    F f;
    D dec;
    __device__ void operator()(double2* S, const double2* d) const {
        f(S, d);
        dec(S);
    }
};
template <class F, class D> static FinThen<F, D> then(F f, D dec) { return FinThen<F, D>{f, dec}; }

// the drivers' rule: stop when err < CG_THR (CG_Iteration.h:323-331, 497-505,
// 733-747, 1022-1035, 1315-1327); a non-finite scalar without convergence is a
// breakdown; the iteration cap ends the solve
struct DecideErr {
    KCtl* ctl;
    double2* hist;
    __device__ void operator()(double2* S) const {
        const double err = S[S_ERR].x;
        const int m = ctl->iter;
        if (m < ctl->hist_cap) hist[m] = make_double2(err, -1.0);
        ctl->iter = m + 1;
        ctl->last = err;
        if (err < ctl->thr) {
            ctl->state = KS_DONE;
            ctl->steps = m;
        } else if (S[S_NAN].x != 0.0) {
            ctl->state = KS_BREAKDOWN;
        } else if (m + 1 >= ctl->maxit) {
            ctl->state = KS_MAXIT;
        }
    }
};
// mixed BiCGSTAB after the FP32 step: request a reliable update when the
// recursive residual fell by delta below its running maximum, or below the
// tolerance
struct DecideReliable {
    KCtl* ctl;
    double2* hist;
    __device__ void operator()(double2* S) const {
        const double err = S[S_ERR].x, rr = S[S_RR].x;
        const int m = ctl->iter;
        if (m < ctl->hist_cap) hist[m] = make_double2(err, -1.0);
        ctl->iter = m + 1;
        ctl->last = err;
        if (S[S_NAN].x != 0.0 && !(err < ctl->thr)) {
            ctl->state = KS_BREAKDOWN;
        } else if (rr < ctl->delta * ctl->delta * ctl->rmax2 || err < ctl->thr) {
            ctl->state = KS_UPDATE;
        } else {
            ctl->rmax2 = fmax(ctl->rmax2, rr);
            if (m + 1 >= ctl->maxit) ctl->state = KS_MAXIT;
        }
    }
};
// after r = b - A x in FP64 (S_T5 = ||r||^2): stop on the true residual, else
// replace the FP32 residual by it
struct DecideTrue {
    KCtl* ctl;
    double2* hist;
    __device__ void operator()(double2* S) const {
        const double rel = sqrt(S[S_T5].x / ctl->bn2);
        const int m = ctl->iter - 1;
        if (m >= 0 && m < ctl->hist_cap) hist[m].y = rel;
        ctl->updates++;
        ctl->last = rel;
        if (rel < ctl->thr) {
            ctl->state = KS_DONE;
            ctl->steps = m;
        } else if (ctl->iter >= ctl->maxit) {
            ctl->state = KS_MAXIT;
        } else {
            ctl->state = KS_RESET;
            ctl->rmax2 = rel * rel * ctl->bn2;
        }
    }
};
struct DecideResume {  // residual replaced: iterate again
    KCtl* ctl;
    __device__ void operator()(double2*) const { ctl->state = KS_RUN; }
};


// ---------------------------------------------------------------------------
// generic fused vector kernel:  y = sum_i c_i x_i  (+ y if acc), c_i from slots;
// optional dots conj(u_k) . y_new (or plain u_k . y_new)
// ---------------------------------------------------------------------------
struct CoefSpec {
    int slot;       // -1: constant
    double re, im;  // multiplier
};
template <typename C> struct LinTerm {
    const C* x;
    CoefSpec c;
};
template <typename C> struct DotSpec {
    const C* u;  // nullptr: u = y_new
    int conj;
};
template <typename C, int NT, int K> struct LinArgs {
    C* y;
    int acc;
    LinTerm<C> t[NT];
    DotSpec<C> d[K > 0 ? K : 1];
};

__device__ __forceinline__ double2 eval_coef(const CoefSpec& c, const double2* S) {
    const double2 base = c.slot >= 0 ? S[c.slot] : make_double2(1.0, 0.0);
    return dmul(base, make_double2(c.re, c.im));
}

template <typename C, int NT, int K>
__global__ void __launch_bounds__(256) k_lin(LinArgs<C, NT, K> g, long long n, const double2* __restrict__ S,
                                             double2* __restrict__ partial, Gate gate) {
    if (gate_closed(gate)) return;
    C cf[NT];
#pragma unroll
    for (int i = 0; i < NT; i++) cf[i] = coef_c<C>(eval_coef(g.t[i].c, S));
    constexpr int KA = K > 0 ? K : 1;
    double2 acc[KA];
#pragma unroll
    for (int k = 0; k < KA; k++) acc[k] = make_double2(0, 0);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        C v = g.acc ? g.y[i] : czero<C>();
#pragma unroll
        for (int t = 0; t < NT; t++) v = cadd(v, cmul(cf[t], g.t[t].x[i]));
        g.y[i] = v;
#pragma unroll
        for (int k = 0; k < K; k++) {
            const C u = g.d[k].u ? g.d[k].u[i] : v;
            if (g.d[k].conj) acc_dotc(acc[k], u, v);
            else acc_dotu(acc[k], u, v);
        }
    }
    if constexpr (K > 0) block_reduce_store<KA>(acc, partial, blockIdx.x);
}

// dots only
template <typename C, int K> struct DotArgs {
    const C* u[K];
    const C* v[K];
    int conj[K];
};
template <typename C, int K>
__global__ void __launch_bounds__(256) k_dots(DotArgs<C, K> g, long long n, double2* __restrict__ partial,
                                              Gate gate) {
    if (gate_closed(gate)) return;
    double2 acc[K];
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] = make_double2(0, 0);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int k = 0; k < K; k++) {
            if (g.conj[k]) acc_dotc(acc[k], g.u[k][i], g.v[k][i]);
            else acc_dotu(acc[k], g.u[k][i], g.v[k][i]);
        }
    }
    block_reduce_store<K>(acc, partial, blockIdx.x);
}

// b = e . flag (Current_Reset on E_inc, CG_Iteration.h:560-562), converted to C
template <typename C>
__global__ void k_mask_rhs(const double2* __restrict__ e, const unsigned char* __restrict__ flags, C* __restrict__ b,
                           long long a, double scale) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 3 * a;
         i += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(i / a);
        const long long v = i - s * a;
        const double f = ((flags[v] >> s) & 1) ? scale : 0.0;
        b[i] = from_d2<C>(make_double2(e[i].x * f, e[i].y * f));
    }
}

// y64 (+)= scale * x (C precision)
template <typename C>
__global__ void k_accum_d(double2* __restrict__ y, const C* __restrict__ x, long long n, const double2* S, int slot,
                          int accumulate) {
    const double s = slot >= 0 ? sqrt(S[slot].x) : 1.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double2 v = as_d2(x[i]);
        double2 o = accumulate ? y[i] : make_double2(0, 0);
        o.x += s * v.x;
        o.y += s * v.y;
        y[i] = o;
    }
}

// y32 = x64 / sqrt(S[slot])
template <typename C>
__global__ void k_scale_to(C* __restrict__ y, const double2* __restrict__ x, long long n, const double2* S, int slot) {
    const double s = 1.0 / sqrt(S[slot].x);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] = from_d2<C>(make_double2(x[i].x * s, x[i].y * s));
}


// ---------------------------------------------------------------------------
// prologue / epilogue functors of the fused BiCGSTAB and refinement
// ---------------------------------------------------------------------------
// Each prologue has load(s, idx) (every global read of one element, issued
// before any store so a chunk of elements can be loaded together) and
// apply(s, idx, loaded) (arithmetic and stores); each epilogue has pre(s, idx)
// (the vector it reads) and put(s, idx, y, acc, pre).  operator() chains them
// for kernels that work element by element.
template <typename C> struct ProCopyWrite {  // p = r
    const C* __restrict__ r;
    C* __restrict__ p;
    long long a;
    struct L { C r; };
    __device__ __forceinline__ L load(int s, long long idx) const { return L{r[s * a + idx]}; }
    __device__ __forceinline__ C apply(int s, long long idx, const L& l) const {
        p[s * a + idx] = l.r;
        return l.r;
    }
    __device__ __forceinline__ C operator()(int s, long long idx, bool) const { return apply(s, idx, load(s, idx)); }
};
template <typename C> struct ProBicgP {  // p = r + beta (p - omega v)
    const C* __restrict__ r;
    C* __restrict__ p;
    const C* __restrict__ v;
    const double2* __restrict__ S;
    long long a;
    struct L { C r, p, v, beta, omega; };
    __device__ __forceinline__ L load(int s, long long idx) const {
        const long long o = s * a + idx;
        return L{r[o], p[o], v[o], from_d2<C>(S[S_BETA]), from_d2<C>(S[S_OMEGA])};
    }
    // r and v staged by the forward z pass (p is also written here, so it is read per element)
    static constexpr int NSTAGE = 2;
    __device__ __forceinline__ const C* stage_src(int k) const { return k ? v : r; }
    __device__ __forceinline__ L load_staged(int s, long long idx, const C* sv) const {
        return L{sv[0], p[s * a + idx], sv[1], from_d2<C>(S[S_BETA]), from_d2<C>(S[S_OMEGA])};
    }
    __device__ __forceinline__ C apply(int s, long long idx, const L& l) const {
        const C pv = cadd(l.r, cmul(l.beta, csub(l.p, cmul(l.omega, l.v))));
        p[s * a + idx] = pv;
        return pv;
    }
    __device__ __forceinline__ C operator()(int s, long long idx, bool) const { return apply(s, idx, load(s, idx)); }
};
template <typename C> struct ProBicgS {  // s = r - alpha v
    const C* __restrict__ r;
    const C* __restrict__ v;
    C* __restrict__ sv;
    const double2* __restrict__ S;
    long long a;
    struct L { C r, v, alpha; };
    __device__ __forceinline__ L load(int s, long long idx) const {
        const long long o = s * a + idx;
        return L{r[o], v[o], from_d2<C>(S[S_ALPHA])};
    }
    static constexpr int NSTAGE = 2;
    __device__ __forceinline__ const C* stage_src(int k) const { return k ? v : r; }
    __device__ __forceinline__ L load_staged(int, long long, const C* sv) const {
        return L{sv[0], sv[1], from_d2<C>(S[S_ALPHA])};
    }
    __device__ __forceinline__ C apply(int s, long long idx, const L& l) const {
        const C x = csub(l.r, cmul(l.alpha, l.v));
        sv[s * a + idx] = x;
        return x;
    }
    __device__ __forceinline__ C operator()(int s, long long idx, bool) const { return apply(s, idx, load(s, idx)); }
};
template <typename C> struct EpiDotB {  // store y; acc conj(b) y
    static constexpr int K = 1;
    C* __restrict__ y;
    const C* __restrict__ b;
    long long a;
    __device__ __forceinline__ C pre(int s, long long idx) const { return b[s * a + idx]; }
    __device__ __forceinline__ void put(int s, long long idx, C v, double2* acc, C bv) const {
        y[s * a + idx] = v;
        acc_dotc(acc[0], bv, v);
    }
    __device__ __forceinline__ void operator()(int s, long long idx, C v, double2* acc) const {
        put(s, idx, v, acc, pre(s, idx));
    }
};
template <typename C> struct EpiDotTS {  // store t; acc conj(t) s, conj(t) t
    static constexpr int K = 2;
    C* __restrict__ y;
    const C* __restrict__ sv;
    long long a;
    __device__ __forceinline__ C pre(int s, long long idx) const { return sv[s * a + idx]; }
    __device__ __forceinline__ void put(int s, long long idx, C v, double2* acc, C svv) const {
        y[s * a + idx] = v;
        acc_dotc(acc[0], v, svv);
        acc_dotc(acc[1], v, v);
    }
    __device__ __forceinline__ void operator()(int s, long long idx, C v, double2* acc) const {
        put(s, idx, v, acc, pre(s, idx));
    }
};
template <typename C> struct EpiNorm {  // store y; acc ||y||^2
    static constexpr int K = 1;
    C* __restrict__ y;
    long long a;
    __device__ __forceinline__ C pre(int, long long) const { return czero<C>(); }
    __device__ __forceinline__ void put(int s, long long idx, C v, double2* acc, C) const {
        y[s * a + idx] = v;
        acc_dotc(acc[0], v, v);
    }
    __device__ __forceinline__ void operator()(int s, long long idx, C v, double2* acc) const {
        put(s, idx, v, acc, czero<C>());
    }
};
template <typename C> struct EpiDotU {  // store y; acc y^T u (unconjugated)
    static constexpr int K = 1;
    C* __restrict__ y;
    const C* __restrict__ u;
    long long a;
    __device__ __forceinline__ C pre(int s, long long idx) const { return u[s * a + idx]; }
    __device__ __forceinline__ void put(int s, long long idx, C v, double2* acc, C uv) const {
        y[s * a + idx] = v;
        acc_dotu(acc[0], v, uv);
    }
    __device__ __forceinline__ void operator()(int s, long long idx, C v, double2* acc) const {
        put(s, idx, v, acc, pre(s, idx));
    }
};
template <typename C> struct EpiResidual {  // r = b - y; acc ||r||^2
    static constexpr int K = 1;
    C* __restrict__ r;
    const C* __restrict__ b;
    long long a;
    __device__ __forceinline__ C pre(int s, long long idx) const { return b[s * a + idx]; }
    __device__ __forceinline__ void put(int s, long long idx, C v, double2* acc, C bv) const {
        const C rv = csub(bv, v);
        r[s * a + idx] = rv;
        acc_dotc(acc[0], rv, rv);
    }
    __device__ __forceinline__ void operator()(int s, long long idx, C v, double2* acc) const {
        put(s, idx, v, acc, pre(s, idx));
    }
};

// CORS: the three vector updates after beta (CG_Iteration.h:880-915) as the
// prologue of the forward z pass of A q, element by element exactly as the
// separate passes compute them (k_lin: zero, then each term added in order):
//   p = r + beta pc;  qc = Ap + beta rc;  q = beta^2 q + beta rc + qc (new qc)
// and q (new) is the operator's source.  r and Ap are staged with the rows.
template <typename C> struct ProCorsQ {
    const C* __restrict__ r;
    C* __restrict__ p;
    const C* __restrict__ pc;
    const C* __restrict__ Ap;
    C* __restrict__ qc;
    const C* __restrict__ rc;
    C* __restrict__ q;
    const double2* __restrict__ S;
    long long a;
    struct L { C r, pc, Ap, rc, q, one, beta, t0; };
    __device__ __forceinline__ L coefs(C rv, C pcv, C apv, C rcv, C qv) const {
        return L{rv, pcv, apv, rcv, qv, coef_c<C>(eval_coef(CoefSpec{-1, 1.0, 0.0}, S)),
                 coef_c<C>(eval_coef(CoefSpec{S_BETA, 1.0, 0.0}, S)), coef_c<C>(eval_coef(CoefSpec{S_T0, 1.0, 0.0}, S))};
    }
    __device__ __forceinline__ L load(int s, long long idx) const {
        const long long o = s * a + idx;
        return coefs(r[o], pc[o], Ap[o], rc[o], q[o]);
    }
    static constexpr int NSTAGE = 2;
    __device__ __forceinline__ const C* stage_src(int k) const { return k ? Ap : r; }
    __device__ __forceinline__ L load_staged(int s, long long idx, const C* sv) const {
        const long long o = s * a + idx;
        return coefs(sv[0], pc[o], sv[1], rc[o], q[o]);
    }
    __device__ __forceinline__ C apply(int s, long long idx, const L& l) const {
        const long long o = s * a + idx;
        const C pv = cadd(cadd(czero<C>(), cmul(l.one, l.r)), cmul(l.beta, l.pc));
        const C qcv = cadd(cadd(czero<C>(), cmul(l.one, l.Ap)), cmul(l.beta, l.rc));
        const C qv = cadd(cadd(cadd(czero<C>(), cmul(l.t0, l.q)), cmul(l.beta, l.rc)), cmul(l.one, qcv));
        p[o] = pv;
        qc[o] = qcv;
        q[o] = qv;
        return qv;
    }
    __device__ __forceinline__ C operator()(int s, long long idx, bool) const { return apply(s, idx, load(s, idx)); }
};

// CORS: the four vector updates after alpha (CG_Iteration.h:964-1012) in one
// pass, each output as its separate pass computes it, with r^H r of the new r:
//   pc = p - alpha q;  rc = qc - alpha Aq;  x += 2 alpha p - alpha^2 q;
//   r += -2 alpha qc + alpha^2 Aq
template <typename C>
__global__ void __launch_bounds__(256) k_cors_update(C* __restrict__ pc, C* __restrict__ rc, C* __restrict__ x,
                                                     C* __restrict__ r, const C* __restrict__ p,
                                                     const C* __restrict__ q, const C* __restrict__ qc,
                                                     const C* __restrict__ Aq, long long n,
                                                     const double2* __restrict__ S, double2* __restrict__ partial,
                                                     Gate gate) {
    if (gate_closed(gate)) return;
    const C one = coef_c<C>(eval_coef(CoefSpec{-1, 1.0, 0.0}, S));
    const C mal = coef_c<C>(eval_coef(CoefSpec{S_ALPHA, -1.0, 0.0}, S));
    const C al2 = coef_c<C>(eval_coef(CoefSpec{S_ALPHA, 2.0, 0.0}, S));
    const C mt1 = coef_c<C>(eval_coef(CoefSpec{S_T1, -1.0, 0.0}, S));
    const C mal2 = coef_c<C>(eval_coef(CoefSpec{S_ALPHA, -2.0, 0.0}, S));
    const C t1 = coef_c<C>(eval_coef(CoefSpec{S_T1, 1.0, 0.0}, S));
    double2 acc[1] = {make_double2(0, 0)};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const C pi = p[i], qi = q[i], qci = qc[i], aqi = Aq[i];
        pc[i] = cadd(cadd(czero<C>(), cmul(one, pi)), cmul(mal, qi));
        rc[i] = cadd(cadd(czero<C>(), cmul(one, qci)), cmul(mal, aqi));
        x[i] = cadd(cadd(x[i], cmul(al2, pi)), cmul(mt1, qi));
        const C rv = cadd(cadd(r[i], cmul(mal2, qci)), cmul(t1, aqi));
        r[i] = rv;
        acc_dotc(acc[0], rv, rv);
    }
    block_reduce_store<1>(acc, partial, blockIdx.x);
}

// x += alpha p + omega s; r = s - omega t; acc r^H r, b^H r
template <typename C>
__global__ void __launch_bounds__(256) k_bicgstab_update(C* __restrict__ x, const C* __restrict__ p,
                                                         const C* __restrict__ sv, const C* __restrict__ t,
                                                         C* __restrict__ r, const C* __restrict__ b, long long n,
                                                         const double2* __restrict__ S, double2* __restrict__ partial,
                                                         Gate gate) {
    if (gate_closed(gate)) return;
    const C alpha = from_d2<C>(S[S_ALPHA]), omega = from_d2<C>(S[S_OMEGA]);
    double2 acc[2] = {make_double2(0, 0), make_double2(0, 0)};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const C si = sv[i];
        x[i] = cadd(cadd(x[i], cmul(alpha, p[i])), cmul(omega, si));
        const C ri = csub(si, cmul(omega, t[i]));
        r[i] = ri;
        acc_dotc(acc[0], ri, ri);
        acc_dotc(acc[1], b[i], ri);
    }
    block_reduce_store<2>(acc, partial, blockIdx.x);
}


// blocks of the grid-stride vector kernels (8 per SM of a B200)
constexpr int kVecBlocks = 148 * 8;

}  // namespace vie
