// vie_operator.cuh -- the discretised VIE operator as five pruned FFT passes.
//
// The reference applies one row block of the operator as nine zero-padded
// (2Nx,2Ny,2Nz) FFT pairs (CG_Iteration.h:131-173 -> fft.h:41-127, 224-309).
// Here the whole operator y = A x (three field components from three source
// components) is
//
//   F1  forward z: pad fused at load (rows of Nz -> 2Nz spectral, natural order)
//   F2  forward y: columns of Ny -> 2Ny (digit-reversed halves)
//   F3  forward x, spectral multiply with the dyadic Green symbol, inverse x,
//       crop to Nx (all three components of one (ky, kz-tile) column together)
//   I2  inverse y, crop to Ny
//   I1  inverse z, crop to Nz, diagonal inverse-contrast term (fft.h:405-624),
//       edge mask (Current_Reset, fft.h:13-35), optional fused Krylov work
//
// Every padded axis of length 2N is split exactly into two length-N FFTs:
//   X[2m]   = DFT_N(x)[m],   X[2m+1] = DFT_N(x . W_2N^n)[m]
//   y[n<N]  = IDFT_N(E)[n] + W_2N^{-n} IDFT_N(O)[n]
// so the zero half of the padding is never stored or read.
//
// Spectral symbol (derived from fft.h:76-100 and 256-281; M = 8 Nx Ny Nz):
//   rho   = sum_s P_s J_s
//   E_f   = Gs (kappa_f J_f + Q_f rho)
// forward:   P_s = d+_s / delta_s,  Q_f = d-_f,  Gs = (i Z0 / (k0 M)) Gtilde
// conjugate: P_s = conj(d-_s),  Q_f = conj(d+_f) / delta_f,  Gs -> conj(Gs)
// (fft.h:167-190, 344-370); kappa_f = k0^2 delta_f, d+ = 1 - e^{-i theta},
// d- = e^{i theta} - 1, theta = 2 pi k / (2N).
#pragma once
#include "vie_fft_core.cuh"

namespace vie {

constexpr int kThreads = 256;

// per-axis device tables, in the slot order the passes store spectra in
template <typename C> struct AxisTables {
    const C* tw;               // tw[u] = exp(-2 pi i u / 2N), u in [0, 2N)
    const unsigned short* perm;  // perm[m] = DIF output position of index m, m in [0, N)
    const C* P[2];             // [fwd, conj] slot -> P
    const C* Q[2];             // [fwd, conj] slot -> Q
    const int* gfold;          // slot -> folded index into the Green octant, [0, N]
};

// Device-side control of an iterative solve.  Every kernel of a captured
// iteration carries a gate and returns at once unless the solve's state word
// equals the state the kernel belongs to, so one iteration body can be
// replayed (CUDA graph) without host decisions in between.
struct Gate {
    const int* state;  // nullptr: always open
    int when;
};
__device__ __forceinline__ bool gate_closed(const Gate& g) { return g.state != nullptr && *g.state != g.when; }

template <typename C> struct OpDev {
    int nx, ny, nz;
    long long a;               // nx*ny*nz
    int tz, tc, tx;            // pencils per tile: z passes, y passes, x pass
    AxisPlan plan[3];
    AxisTables<C> ax[3];
    const C* Gs;               // (nx+1)(ny+1)(nz+1) octant, scaled
    const C* w;                // per voxel 1/(eps-1)
    const unsigned char* flags;  // bit0 Flag_X, bit1 Flag_Y, bit2 Flag_Z
    int fast[3];               // axis uses the register four-step kernels (half-natural slots)
    int xalt;                  // register x pass with the alternative (half) pencil tile
    int parts;                 // VIE_PART_* bits: Green blocks, diagonal term, edge mask
    typename real_of<C>::type kappa[3];   // k0^2 delta_f
    typename real_of<C>::type dcoef[3];   // -delta_f Z0 / (2 k0)
    C* b;                      // 3 * nx*ny*2nz scratch
    C* c;                      // 3 * nx*2ny*2nz scratch
    Gate gate;                 // launch gate of the current solve (state == nullptr: always run)
    int* status;               // device word set by a kernel whose bounded wait ran out (TMA staging)
    int zstage;                // register z passes stage their rows with bulk copies (0: element loads)
    int wait_test;             // 1: every staged tile's wait runs out on purpose (tests of the timeout path)
};

__host__ __device__ inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// dynamic shared memory: [tw 2N][perm N u16][pad][buf nsets*N*TP]
template <typename C>
__host__ __device__ inline size_t pass_smem_bytes(int N, int nsets, int TP) {
    size_t s = sizeof(C) * 2 * (size_t)N;
    s += sizeof(unsigned short) * (size_t)N;
    s = align_up(s, 16);
    s += sizeof(C) * (size_t)nsets * N * TP;
    return s;
}

template <typename C>
__device__ __forceinline__ void load_axis_tables(const AxisTables<C>& t, int N, C*& tw, unsigned short*& perm,
                                                 C*& buf) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    tw = reinterpret_cast<C*>(smem_raw);
    perm = reinterpret_cast<unsigned short*>(tw + 2 * N);
    size_t off = align_up(sizeof(C) * 2 * (size_t)N + sizeof(unsigned short) * (size_t)N, 16);
    buf = reinterpret_cast<C*>(smem_raw + off);
    for (int u = threadIdx.x; u < 2 * N; u += blockDim.x) tw[u] = t.tw[u];
    for (int u = threadIdx.x; u < N; u += blockDim.x) perm[u] = t.perm[u];
}

// ---------------------------------------------------------------------------
// block reduction of K complex FP64 accumulators -> partial[blockLinear*K + k]
// ---------------------------------------------------------------------------
template <int K>
__device__ __forceinline__ void block_reduce_store(double2 (&acc)[K], double2* __restrict__ partial,
                                                   long long blin) {
    __shared__ double2 red[K][kThreads / 32];
#pragma unroll
    for (int k = 0; k < K; k++) {
        double rx = acc[k].x, ry = acc[k].y;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            rx += __shfl_down_sync(0xffffffffu, rx, o);
            ry += __shfl_down_sync(0xffffffffu, ry, o);
        }
        if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = make_double2(rx, ry);
    }
    __syncthreads();
    if (threadIdx.x < K) {
        const int k = threadIdx.x;
        double rx = 0, ry = 0;
        for (int wi = 0; wi < (int)(blockDim.x >> 5); wi++) { rx += red[k][wi].x; ry += red[k][wi].y; }
        partial[blin * K + k] = make_double2(rx, ry);
    }
}

// ---------------------------------------------------------------------------
// F1: forward z with the zero padding fused into the load.
//   pro(s, idx, valid) returns the source value of component s at voxel idx
//   (and may write Krylov vectors); the value is used only where valid.
// ---------------------------------------------------------------------------
template <typename C, class Pro>
__global__ void __launch_bounds__(kThreads) k_fwd_z(OpDev<C> op, Pro pro) {
    if (gate_closed(op.gate)) return;
    const int N = op.nz, T = op.tz, TP = T + 1;
    C* tw; unsigned short* perm; C* buf;
    load_axis_tables(op.ax[2], N, tw, perm, buf);
    const int s = blockIdx.y;
    const long long nrows = (long long)op.nx * op.ny;
    const long long row0 = (long long)blockIdx.x * T;
    const int fs = N * TP;
    __syncthreads();
    for (int e = threadIdx.x; e < T * N; e += blockDim.x) {
        const int t = e / N, n = e - t * N;
        const long long row = row0 + t;
        C x = czero<C>();
        if (row < nrows) {
            const int i = (int)(row / op.ny), j = (int)(row - (long long)i * op.ny);
            const bool valid = (s != 0 || i < op.nx - 1) && (s != 1 || j < op.ny - 1) && (s != 2 || n < N - 1);
            x = pro(s, row * N + n, valid);
            if (!valid) x = czero<C>();
        }
        buf[n * TP + t] = x;
        buf[fs + n * TP + t] = cmul(x, tw[n]);
    }
    __syncthreads();
    smem_fft_fwd(buf, 2, fs, T, TP, op.plan[2], tw);
    const int L = 2 * N;
    for (int e = threadIdx.x; e < T * L; e += blockDim.x) {
        const int t = e / L, k = e - t * L;
        const long long row = row0 + t;
        if (row < nrows) op.b[((long long)s * nrows + row) * L + k] = buf[(k & 1) * fs + perm[k >> 1] * TP + t];
    }
}

// F2: forward y.  grid (kz tiles, nx, 3)
template <typename C>
__global__ void __launch_bounds__(kThreads) k_fwd_y(OpDev<C> op) {
    if (gate_closed(op.gate)) return;
    const int N = op.ny, T = op.tc, TP = T;
    C* tw; unsigned short* perm; C* buf;
    load_axis_tables(op.ax[1], N, tw, perm, buf);
    const int Lz = 2 * op.nz;
    const int kz0 = blockIdx.x * T, i = blockIdx.y, s = blockIdx.z;
    const int fs = N * TP;
    const C* src = op.b + ((long long)s * op.nx + i) * (long long)op.ny * Lz;
    __syncthreads();
    for (int e = threadIdx.x; e < T * N; e += blockDim.x) {
        const int t = e % T, j = e / T;
        C x = czero<C>();
        if (kz0 + t < Lz) x = src[(long long)j * Lz + kz0 + t];
        buf[j * TP + t] = x;
        buf[fs + j * TP + t] = cmul(x, tw[j]);
    }
    __syncthreads();
    smem_fft_fwd(buf, 2, fs, T, TP, op.plan[1], tw);
    C* dst = op.c + ((long long)s * op.nx + i) * (long long)(2 * N) * Lz;
    for (int e = threadIdx.x; e < T * 2 * N; e += blockDim.x) {
        const int t = e % T, slot = e / T;
        if (kz0 + t < Lz) {
            const int h = slot >= N, p = slot - h * N;
            dst[(long long)slot * Lz + kz0 + t] = buf[h * fs + p * TP + t];
        }
    }
}

// F3: forward x, spectral multiply, inverse x, crop.  grid (kz tiles, 2ny)
template <typename C, bool CONJ>
__global__ void __launch_bounds__(kThreads) k_x_spectral(OpDev<C> op) {
    if (gate_closed(op.gate)) return;
    using R = typename real_of<C>::type;
    const int N = op.nx, T = op.tx, TP = T;
    C* tw; unsigned short* perm; C* buf;
    load_axis_tables(op.ax[0], N, tw, perm, buf);
    const int Lz = 2 * op.nz, Ly = 2 * op.ny;
    const int kz0 = blockIdx.x * T, ky = blockIdx.y;
    const int fs = N * TP;                 // set (s, h) at buf[(2 s + h) * fs]
    const long long cs = (long long)Ly * Lz;  // stride of i in c
    __syncthreads();
    for (int e = threadIdx.x; e < 3 * T * N; e += blockDim.x) {
        const int t = e % T, rest = e / T, i = rest % N, s = rest / N;
        C x = czero<C>();
        if (kz0 + t < Lz) x = op.c[((long long)s * N + i) * cs + (long long)ky * Lz + kz0 + t];
        buf[(2 * s) * fs + i * TP + t] = x;
        buf[(2 * s + 1) * fs + i * TP + t] = cmul(x, tw[i]);
    }
    __syncthreads();
    smem_fft_fwd(buf, 6, fs, T, TP, op.plan[0], tw);
    {
        const int md = CONJ ? 1 : 0;
        const C Py = op.ax[1].P[md][ky], Qy = op.ax[1].Q[md][ky];
        const int gy = op.ax[1].gfold[ky];
        const R kx_ = op.kappa[0], ky_ = op.kappa[1], kz_ = op.kappa[2];
        for (int e = threadIdx.x; e < 2 * N * T; e += blockDim.x) {
            const int t = e % T, sx = e / T;
            const int kz = kz0 + t;
            if (kz >= Lz) continue;
            const int h = sx >= N, p = sx - h * N;
            const C Px = op.ax[0].P[md][sx], Qx = op.ax[0].Q[md][sx];
            const C Pz = op.ax[2].P[md][kz], Qz = op.ax[2].Q[md][kz];
            const int gx = op.ax[0].gfold[sx], gz = op.ax[2].gfold[kz];
            C G = op.Gs[((long long)gx * (op.ny + 1) + gy) * (op.nz + 1) + gz];
            if (CONJ) G = cconj(G);
            const int o = h * fs + p * TP + t;
            const C Jx = buf[o], Jy = buf[2 * fs + o], Jz = buf[4 * fs + o];
            const C rho = cadd(cadd(cmul(Px, Jx), cmul(Py, Jy)), cmul(Pz, Jz));
            buf[o] = cmul(G, cadd(cscale(Jx, kx_), cmul(Qx, rho)));
            buf[2 * fs + o] = cmul(G, cadd(cscale(Jy, ky_), cmul(Qy, rho)));
            buf[4 * fs + o] = cmul(G, cadd(cscale(Jz, kz_), cmul(Qz, rho)));
        }
    }
    __syncthreads();
    smem_fft_inv(buf, 6, fs, T, TP, op.plan[0], tw);
    for (int e = threadIdx.x; e < 3 * T * N; e += blockDim.x) {
        const int t = e % T, rest = e / T, i = rest % N, s = rest / N;
        if (kz0 + t < Lz) {
            const C y = cadd(buf[(2 * s) * fs + i * TP + t], cmulc(buf[(2 * s + 1) * fs + i * TP + t], tw[i]));
            op.c[((long long)s * N + i) * cs + (long long)ky * Lz + kz0 + t] = y;
        }
    }
}

// I2: inverse y, crop.  grid (kz tiles, nx, 3)
template <typename C>
__global__ void __launch_bounds__(kThreads) k_inv_y(OpDev<C> op) {
    if (gate_closed(op.gate)) return;
    const int N = op.ny, T = op.tc, TP = T;
    C* tw; unsigned short* perm; C* buf;
    load_axis_tables(op.ax[1], N, tw, perm, buf);
    const int Lz = 2 * op.nz;
    const int kz0 = blockIdx.x * T, i = blockIdx.y, s = blockIdx.z;
    const int fs = N * TP;
    const C* src = op.c + ((long long)s * op.nx + i) * (long long)(2 * N) * Lz;
    __syncthreads();
    for (int e = threadIdx.x; e < T * 2 * N; e += blockDim.x) {
        const int t = e % T, slot = e / T;
        const int h = slot >= N, p = slot - h * N;
        C x = czero<C>();
        if (kz0 + t < Lz) x = src[(long long)slot * Lz + kz0 + t];
        buf[h * fs + p * TP + t] = x;
    }
    __syncthreads();
    smem_fft_inv(buf, 2, fs, T, TP, op.plan[1], tw);
    C* dst = op.b + ((long long)s * op.nx + i) * (long long)N * Lz;
    for (int e = threadIdx.x; e < T * N; e += blockDim.x) {
        const int t = e % T, j = e / T;
        if (kz0 + t < Lz) {
            const C y = cadd(buf[j * TP + t], cmulc(buf[fs + j * TP + t], tw[j]));
            dst[(long long)j * Lz + kz0 + t] = y;
        }
    }
}

// I1: inverse z, crop, diagonal term, mask, epilogue.  grid (row tiles, 3)
//   epi(s, idx, y, acc) receives the finished operator output of component s
//   at voxel idx and stores / accumulates it.
template <typename C, bool CONJ, class Epi>
__global__ void __launch_bounds__(kThreads) k_inv_z(OpDev<C> op, const C* __restrict__ xin, Epi epi,
                                                     double2* __restrict__ partial) {
    if (gate_closed(op.gate)) return;
    using R = typename real_of<C>::type;
    const int N = op.nz, T = op.tz, TP = T + 1;
    C* tw; unsigned short* perm; C* buf;
    load_axis_tables(op.ax[2], N, tw, perm, buf);
    const int s = blockIdx.y;
    const long long nrows = (long long)op.nx * op.ny;
    const long long row0 = (long long)blockIdx.x * T;
    const int fs = N * TP, L = 2 * N;
    __syncthreads();
    for (int e = threadIdx.x; e < T * L; e += blockDim.x) {
        const int t = e / L, k = e - t * L;
        const long long row = row0 + t;
        C x = czero<C>();
        if (row < nrows) x = op.b[((long long)s * nrows + row) * L + k];
        buf[(k & 1) * fs + perm[k >> 1] * TP + t] = x;
    }
    __syncthreads();
    smem_fft_inv(buf, 2, fs, T, TP, op.plan[2], tw);
    constexpr int KA = Epi::K > 0 ? Epi::K : 1;
    double2 acc[KA];
#pragma unroll
    for (int k = 0; k < KA; k++) acc[k] = make_double2(0.0, 0.0);
    const long long sstep = s == 0 ? (long long)op.ny * N : (s == 1 ? (long long)N : 1LL);
    const R dc = op.dcoef[s];
    const bool use_green = op.parts & 1, use_diag = op.parts & 2, use_mask = op.parts & 4;
    // four elements per thread and step: all their global reads (flags, contrast
    // pair, diagonal source, the epilogue's vector) first, then the arithmetic
    // and stores; the selections give the branchy form's results bit for bit
    constexpr int CH = 4;
    const int total = T * N, stride = blockDim.x;
    for (int e0 = threadIdx.x; e0 < total; e0 += CH * stride) {
        long long idx[CH];
        bool ok[CH], dv[CH];
        unsigned char fl[CH];
        C wa[CH], wb[CH], xv[CH], pv[CH];
#pragma unroll
        for (int q = 0; q < CH; q++) {
            const int e = e0 + q * stride;
            const int t = e / N, n = e - t * N;
            const long long row = row0 + t;
            ok[q] = e < total && row < nrows;
            idx[q] = ok[q] ? row * N + n : 0;
            const int i = (int)(row / op.ny), j = (int)(row - (long long)i * op.ny);
            dv[q] = ok[q] && (s != 0 || i < op.nx - 1) && (s != 1 || j < op.ny - 1) && (s != 2 || n < N - 1);
            fl[q] = op.flags[idx[q]];
            wa[q] = op.w[idx[q]];
            wb[q] = op.w[dv[q] ? idx[q] + sstep : idx[q]];
            xv[q] = xin[(long long)s * op.a + idx[q]];
            pv[q] = epi.pre(s, idx[q]);
        }
#pragma unroll
        for (int q = 0; q < CH; q++) {
            if (!ok[q]) continue;
            const int e = e0 + q * stride;
            const int t = e / N, n = e - t * N;
            C y = use_green ? cadd(buf[n * TP + t], cmulc(buf[fs + n * TP + t], tw[n])) : czero<C>();
            // -i delta Z0/(2 k0) (w_a + w_b) J   (fft.h:419-433); conjugate twin :455-469
            const C ws = cadd(wb[q], wa[q]);
            C coef = mkc(-dc * ws.y, dc * ws.x);  // i * dc * ws with dc = -delta Z0/(2 k0)
            if (CONJ) coef = cconj(coef);
            const C yd = cadd(y, cmul(coef, xv[q]));
            y = (use_diag && dv[q]) ? yd : y;
            y = (!use_mask || ((fl[q] >> s) & 1)) ? y : czero<C>();
            epi.put(s, idx[q], y, acc, pv[q]);
        }
    }
    if constexpr (Epi::K > 0) block_reduce_store<KA>(acc, partial, (long long)blockIdx.y * gridDim.x + blockIdx.x);
}

// ---------------------------------------------------------------------------
// prologue / epilogue functors
// ---------------------------------------------------------------------------
// prologue / epilogue interface: load/apply and pre/put split the global
// reads from the arithmetic and the stores (see the Krylov functors)
template <typename C> struct ProCopy {
    const C* __restrict__ x;
    long long a;
    struct L { C x; };
    static constexpr int NSTAGE = 1;
    __device__ __forceinline__ const C* stage_src(int) const { return x; }
    __device__ __forceinline__ L load_staged(int, long long, const C* v) const { return L{v[0]}; }
    __device__ __forceinline__ L load(int s, long long idx) const { return L{x[s * a + idx]}; }
    __device__ __forceinline__ C apply(int, long long, const L& l) const { return l.x; }
    __device__ __forceinline__ C operator()(int s, long long idx, bool) const { return x[s * a + idx]; }
};

template <typename C> struct EpiStore {
    static constexpr int K = 0;
    C* __restrict__ y;
    long long a;
    __device__ __forceinline__ C pre(int, long long) const { return czero<C>(); }
    __device__ __forceinline__ void put(int s, long long idx, C v, double2*, C) const { y[s * a + idx] = v; }
    __device__ __forceinline__ void operator()(int s, long long idx, C v, double2*) const { y[s * a + idx] = v; }
};

}  // namespace vie
