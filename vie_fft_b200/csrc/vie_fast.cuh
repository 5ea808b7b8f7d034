// vie_fast.cuh -- register-resident four-step pencil FFT passes for the common
// axis lengths (compile-time N = R1 * R2).
//
// Each length-N transform is done as
//     X[k1 + R1 k2] = sum_n2 W_R2^{n2 k2} W_N^{n2 k1} sum_n1 x[n2 + R2 n1] W_R1^{n1 k1}
// step A: thread "n2" loads its R1 inputs (stride R2), DFT_R1 in registers,
//         twiddles W_N^{n2 k1}, one shared-memory transpose;
// step B: thread "k1" reads its R2 values, DFT_R2 in registers and holds
//         X[k1 + R1 k2], k2 < R2: a natural-order spectrum, strided over threads.
// The inverse runs the same two steps backwards with conjugate twiddles.
// Padding split as in vie_operator.cuh: the even half transforms x, the odd
// half x . W_2N^n; the inverse crop combines y = y_even + W_2N^{-n} y_odd.
//
// Spectral slot orders these kernels use: z natural (slot = k); x and y
// "half-natural" (slot = h N + m for spectral index k = 2m + h).
//
// All index arithmetic is compile-time except the tile origins; thread roles:
//   column passes (pencils contiguous in memory): tid = lane * TP + tx,
//   row passes (pencils are contiguous rows):     tid = row * L + lane.
#pragma once
#include <cuda.h>
#include <type_traits>

#include "vie_operator.cuh"

namespace vie {

template <int N> struct FastPlan { static constexpr bool ok = false; static constexpr int R1 = 1, R2 = 1; };
#define VIE_FAST_PLAN(NN, A, B) \
    template <> struct FastPlan<NN> { static constexpr bool ok = true; static constexpr int R1 = A, R2 = B; };
VIE_FAST_PLAN(256, 16, 16)
VIE_FAST_PLAN(192, 16, 12)
VIE_FAST_PLAN(176, 16, 11)
VIE_FAST_PLAN(160, 16, 10)
VIE_FAST_PLAN(144, 16, 9)
VIE_FAST_PLAN(128, 16, 8)
VIE_FAST_PLAN(120, 8, 15)
VIE_FAST_PLAN(112, 16, 7)
VIE_FAST_PLAN(96, 16, 6)
VIE_FAST_PLAN(88, 8, 11)
VIE_FAST_PLAN(80, 16, 5)
VIE_FAST_PLAN(72, 8, 9)
VIE_FAST_PLAN(64, 8, 8)
VIE_FAST_PLAN(56, 8, 7)
VIE_FAST_PLAN(48, 8, 6)
VIE_FAST_PLAN(40, 8, 5)
VIE_FAST_PLAN(32, 8, 4)
VIE_FAST_PLAN(24, 8, 3)
VIE_FAST_PLAN(16, 4, 4)
#undef VIE_FAST_PLAN
// the axis lengths with register four-step kernels (one case per FastPlan above)
#define VIE_FAST_LENGTHS(X) \
    X(256) X(192) X(176) X(160) X(144) X(128) X(120) X(112) X(96) X(88) X(80) X(72) X(64) X(56) X(48) X(40) X(32) \
    X(24) X(16)

inline bool fast_length(int n) {
#define VIE_FL_CASE(NN) if (n == NN) return true;
    VIE_FAST_LENGTHS(VIE_FL_CASE)
#undef VIE_FL_CASE
    return false;
}

template <int R, bool INV, typename C> __device__ __forceinline__ void dft_reg(C* v) { dft_reg_any<R, INV>(v); }

// pencils per CTA of the column passes (one row segment of TP * sizeof(C) bytes)
template <typename C> struct FastTiles;
template <> struct FastTiles<float2> { static constexpr int TP_Y = 16, TP_X = 8, ROWS_DIV = 1; };
template <> struct FastTiles<double2> { static constexpr int TP_Y = 8, TP_X = 4, ROWS_DIV = 2; };

// shared memory layout: [tw 2N][buffer]
template <typename C, int N> __device__ __forceinline__ C* fast_smem(const C* gtw, C*& tw) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    tw = reinterpret_cast<C*>(smem_raw);
    for (int u = threadIdx.x; u < 2 * N; u += blockDim.x) tw[u] = gtw[u];
    return tw + 2 * N;
}

template <typename C, int N> __host__ __device__ constexpr int fast_lanes() {
    return FastPlan<N>::R1 > FastPlan<N>::R2 ? FastPlan<N>::R1 : FastPlan<N>::R2;
}
template <typename C, int N> __host__ __device__ constexpr int fast_rows() {
    return (256 / fast_lanes<C, N>()) / FastTiles<C>::ROWS_DIV;
}

template <typename C, int N> __host__ __device__ constexpr size_t fast_smem_row() {
    // E[2][ROWS][R][R'+1]: rows outermost, padded inner rows (bank-conflict free)
    constexpr int R1 = FastPlan<N>::R1, R2 = FastPlan<N>::R2;
    constexpr int A = R1 * (R2 + 1) > R2 * (R1 + 1) ? R1 * (R2 + 1) : R2 * (R1 + 1);
    return sizeof(C) * (2 * (size_t)N + 2 * (size_t)A * fast_rows<C, N>());
}
// x pass: E[3][2][R1][R2*TP + TP] (each k1 block padded by TP entries).  The
// pencil tile TP of the x pass has two instantiations per precision (the
// default TP_X and TP_X / 2, chosen per grid by the autotuner).
template <typename C> __host__ __device__ constexpr int fast_x_tile(int alt) {
    return alt ? FastTiles<C>::TP_X / 2 : FastTiles<C>::TP_X;
}
template <typename C, int N, int TP = FastTiles<C>::TP_X> __host__ __device__ constexpr int fast_x_kstride() {
    return FastPlan<N>::R2 * TP + TP;
}
template <typename C, int N> __host__ __device__ constexpr size_t fast_smem_col() {
    return sizeof(C) * (2 * (size_t)N + 2 * (size_t)N * FastTiles<C>::TP_Y);
}
template <typename C, int N, int TP = FastTiles<C>::TP_X> __host__ __device__ constexpr size_t fast_smem_x() {
    return sizeof(C) * (2 * (size_t)N + 6 * (size_t)FastPlan<N>::R1 * fast_x_kstride<C, N, TP>());
}

// launch bounds: threads per CTA and the CTAs per SM the register allocation must allow
template <typename C, int N> struct FastLB;
// (x pass: 3 * 16 * TP threads, and as many CTAs per SM as keep the register
// cap of the default tile: 2 * TP_X / TP)
template <int N> struct FastLB<float2, N> {
    static constexpr int ROW = 256, COL = 256, ROW_MIN = 3, COL_MIN = 3;
};
template <int N> struct FastLB<double2, N> {
    static constexpr int ROW = 128, COL = 128, ROW_MIN = 3, COL_MIN = 3;
};
template <typename C, int TP> struct FastXLB {
    static constexpr int XT = 3 * 16 * TP, X_MIN = 2 * FastTiles<C>::TP_X / TP;
};

// ---------------------------------------------------------------------------
// Asynchronous staging into shared memory (TMA unit).  Every wait on an
// mbarrier is bounded: after kTmaWaitIters polls the block records the failure
// in op.status[0] (mapped host memory, read by the host after the call), waits
// once more (bounded) for the copy still in flight and leaves its tile undone.
// If that second wait runs out too, the copy may still write into shared
// memory after the block has left, so the block also sets op.status[1]; the
// host then marks the context unusable.
// op.wait_test makes that path run on purpose: the first wait then polls a
// second mbarrier that nothing completes, kTestWaitIters times.
constexpr int kTmaWaitIters = 1 << 22;
constexpr int kTestWaitIters = 1 << 10;

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool mbar_wait_bounded(unsigned bar, unsigned phase, int limit = kTmaWaitIters) {
    for (int it = 0; it < limit; it++) {
        unsigned ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(bar), "r"(phase)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// bars[0]: the staged tile's barrier; bars[1]: the one nothing completes (wait test)
__device__ __forceinline__ void stage_init(unsigned long long* bars) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bars)) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bars + 1)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// the block's wait for its staged tile; false (for the whole block alike) when it
// ran out, after the status word is set and the copy in flight is waited for
__device__ __forceinline__ bool stage_ready(unsigned long long* bars, int wait_test, int* status) {
    const bool ok = wait_test ? mbar_wait_bounded(smem_u32(bars + 1), 0, kTestWaitIters)
                              : mbar_wait_bounded(smem_u32(bars), 0);
    if (!__syncthreads_or(!ok)) return true;
    if (threadIdx.x == 0 && status) *(volatile int*)status = 1;
    const bool landed = mbar_wait_bounded(smem_u32(bars), 0);
    if (threadIdx.x == 0 && status && !landed) *(volatile int*)(status + 1) = 1;
    return false;
}
__device__ __forceinline__ void mbar_expect(unsigned bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// contiguous global -> shared copy; both addresses 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}
__device__ __forceinline__ bool aligned16(const void* p) { return ((unsigned long long)p & 15ull) == 0; }
// two consecutive complex values (16-byte aligned pair address for float2)
template <typename C> __device__ __forceinline__ void st_pair(C* p, C a, C b) {
    p[0] = a;
    p[1] = b;
}
template <> __device__ __forceinline__ void st_pair<float2>(float2* p, float2 a, float2 b) {
    *reinterpret_cast<float4*>(p) = make_float4(a.x, a.y, b.x, b.y);
}

// Prologues whose source vectors the forward z pass stages whole rows of:
// Pro::NSTAGE vectors (layout s a + idx) returned by stage_src(k), and
// load_staged() building the prologue's operands from the staged values (any
// other operand it still reads from global memory).  Prologues without
// NSTAGE read everything element by element.
template <class P, class = void> struct stage_count { static constexpr int value = 0; };
template <class P> struct stage_count<P, std::void_t<decltype(P::NSTAGE)>> { static constexpr int value = P::NSTAGE; };

// ---------------------------------------------------------------------------
// F1 (row pass): forward z with padding fused into the load.
// E layout: E[h][row][k1][n2], k1 stride R2 + 1 (conflict-free transposed reads).
// ---------------------------------------------------------------------------
// The pass bodies take their block coordinates as arguments: the kernels below
// pass blockIdx, the persistent batch kernels (vie_batch.cu) the coordinates of
// the virtual block they are at.  Every early return is taken by the whole block.
template <typename C, int N, class Pro>
__device__ __forceinline__ void kf_fwd_z_blk(const OpDev<C>& op, const Pro& pro, const int bx, const int s) {
    if (gate_closed(op.gate)) return;
    constexpr int R1 = FastPlan<N>::R1, R2 = FastPlan<N>::R2, L = fast_lanes<C, N>(), ROWS = fast_rows<C, N>();
    constexpr int SR = R2 + 1;                 // padded row of E
    constexpr int HS = R1 * ROWS * SR;         // one half: [ROWS][R1][SR]
    C* tw;
    C* E = fast_smem<C, N>(op.ax[2].tw, tw);
    const int lane = threadIdx.x % L, r = threadIdx.x / L;
    const long long nrows = (long long)op.nx * op.ny;
    const long long row = (long long)bx * ROWS + r;
    const bool live = row < nrows;
    // the prologue's source rows of this block staged whole into E (when they fit
    // and are 16-byte aligned), then read from shared memory
    constexpr int NS = stage_count<Pro>::value;
    constexpr int ESZ = 2 * (R1 * (R2 + 1) > R2 * (R1 + 1) ? R1 * (R2 + 1) : R2 * (R1 + 1)) * ROWS;
    constexpr bool kCanStage = NS > 0 && NS * ROWS * N <= ESZ;
    __shared__ __align__(8) unsigned long long zbar[2];
    bool staged = false;
    const long long row0 = (long long)bx * ROWS;
    const int nr = (int)(nrows - row0 < ROWS ? nrows - row0 : ROWS);
    if constexpr (kCanStage) {
        staged = op.zstage != 0;
#pragma unroll
        for (int k = 0; k < NS; k++) staged = staged && aligned16(pro.stage_src(k) + s * op.a + row0 * N);
        if (staged && threadIdx.x == 0) stage_init(zbar);
    }
    __syncthreads();
    if constexpr (kCanStage) {
        if (staged) {
            const unsigned b = smem_u32(zbar);
            if (threadIdx.x == 0) {
                const unsigned bytes = (unsigned)(sizeof(C) * N) * (unsigned)nr;
                mbar_expect(b, bytes * NS);
#pragma unroll
                for (int k = 0; k < NS; k++) bulk_load(E + k * ROWS * N, pro.stage_src(k) + s * op.a + row0 * N, bytes, b);
            }
            if (!stage_ready(zbar, op.wait_test, op.status)) return;
        }
    }
    C v[R1];
    if (lane < R2 && live) {
        const int n2 = lane;
        const int i = (int)(row / op.ny), j = (int)(row - (long long)i * op.ny);
        const bool vrow = (s != 0 || i < op.nx - 1) && (s != 1 || j < op.ny - 1);
        // the prologue's reads of a chunk of elements first, then its arithmetic and stores
        constexpr int CH = R1 % 4 == 0 ? 4 : 1;
#pragma unroll
        for (int c0 = 0; c0 < R1; c0 += CH) {
            typename Pro::L ld[CH];
#pragma unroll
            for (int q = 0; q < CH; q++) {
                const int n = n2 + R2 * (c0 + q);
                if constexpr (kCanStage) {
                    if (staged) {
                        C sv[NS > 0 ? NS : 1];
#pragma unroll
                        for (int k = 0; k < NS; k++) sv[k] = E[k * ROWS * N + r * N + n];
                        ld[q] = pro.load_staged(s, row * N + n, sv);
                        continue;
                    }
                }
                ld[q] = pro.load(s, row * N + n);
            }
#pragma unroll
            for (int q = 0; q < CH; q++) {
                const int n = n2 + R2 * (c0 + q);
                const bool valid = vrow && (s != 2 || n < N - 1);
                const C x = pro.apply(s, row * N + n, ld[q]);
                v[c0 + q] = valid ? x : czero<C>();
            }
        }
    }
    if constexpr (kCanStage) {
        if (staged) __syncthreads();  // the staged rows are overwritten below
    }
    if (lane < R2 && live) {
        const int n2 = lane;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            C a[R1];
#pragma unroll
            for (int n1 = 0; n1 < R1; n1++) a[n1] = h ? cmul(v[n1], tw[n2 + R2 * n1]) : v[n1];
            dft_reg<R1, false>(a);
#pragma unroll
            for (int k1 = 0; k1 < R1; k1++) {
                const C t = k1 ? cmul(a[k1], tw[2 * n2 * k1]) : a[k1];
                E[h * HS + (r * R1 + k1) * SR + n2] = t;
            }
        }
    }
    __syncthreads();
    C X[2][R2];
    if (lane < R1 && live) {
        const int k1 = lane;
#pragma unroll
        for (int h = 0; h < 2; h++) {
#pragma unroll
            for (int n2 = 0; n2 < R2; n2++) X[h][n2] = E[h * HS + (r * R1 + k1) * SR + n2];
            dft_reg<R2, false>(X[h]);
        }
    }
    // the block's output rows are contiguous: gathered in E in their global
    // order and written by one bulk copy (when 16-byte aligned)
    C* bdst = op.b + ((long long)s * nrows + row0) * (2 * N);
    if (op.zstage && aligned16(bdst)) {
        __syncthreads();  // every read of E is done
        if (lane < R1 && live) {
            const int k1 = lane;
#pragma unroll
            for (int k2 = 0; k2 < R2; k2++) {
                const int m = k1 + R1 * k2;
                st_pair(E + r * (2 * N) + 2 * m, X[0][k2], X[1][k2]);
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            const unsigned bytes = (unsigned)(sizeof(C) * 2 * N) * (unsigned)nr;
            asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(bdst), "r"(smem_u32(E)),
                         "r"(bytes)
                         : "memory");
            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
            asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
        }
        return;
    }
    if (lane < R1 && live) {
        const int k1 = lane;
        C* dst = op.b + ((long long)s * nrows + row) * (2 * N);
#pragma unroll
        for (int k2 = 0; k2 < R2; k2++) {
            const int m = k1 + R1 * k2;
            dst[2 * m] = X[0][k2];
            dst[2 * m + 1] = X[1][k2];
        }
    }
}
template <typename C, int N, class Pro>
__global__ void __launch_bounds__(FastLB<C, N>::ROW, FastLB<C, N>::ROW_MIN) kf_fwd_z(OpDev<C> op, Pro pro) {
    kf_fwd_z_blk<C, N, Pro>(op, pro, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// I1 (row pass): inverse z, crop, diagonal term, mask, epilogue.
// E layout: E[h][row][n2][k1], n2 stride R1 + 1.
// ---------------------------------------------------------------------------
// (conj: the adjoint operator's diagonal coefficient; a run-time flag, the
// two modes differ by one conjugation)
// (gdx: the row blocks of a component, the stride of the reduction partials)
template <typename C, int N, class Epi>
__device__ __forceinline__ void kf_inv_z_blk(const OpDev<C>& op, const C* __restrict__ xin, const Epi& epi,
                                             double2* __restrict__ partial, const int conj, const int bx, const int s,
                                             const int gdx) {
    if (gate_closed(op.gate)) return;
    using R = typename real_of<C>::type;
    constexpr int R1 = FastPlan<N>::R1, R2 = FastPlan<N>::R2, L = fast_lanes<C, N>(), ROWS = fast_rows<C, N>();
    constexpr int SR = R1 + 1;
    constexpr int HS = R2 * ROWS * SR;
    C* tw;
    C* E = fast_smem<C, N>(op.ax[2].tw, tw);
    const int lane = threadIdx.x % L, r = threadIdx.x / L;
    const long long nrows = (long long)op.nx * op.ny;
    const long long row = (long long)bx * ROWS + r;
    const bool live = row < nrows;
    // the block's spectra rows (contiguous) staged whole into E by one bulk copy
    __shared__ __align__(8) unsigned long long zbar[2];
    const long long row0 = (long long)bx * ROWS;
    const int nr = (int)(nrows - row0 < ROWS ? nrows - row0 : ROWS);
    const C* bsrc = op.b + ((long long)s * nrows + row0) * (2 * N);
    const bool staged = op.zstage != 0 && aligned16(bsrc);
    if (staged && threadIdx.x == 0) stage_init(zbar);
    __syncthreads();
    if (staged) {
        if (threadIdx.x == 0) {
            const unsigned bytes = (unsigned)(sizeof(C) * 2 * N) * (unsigned)nr;
            mbar_expect(smem_u32(zbar), bytes);
            bulk_load(E, bsrc, bytes, smem_u32(zbar));
        }
        if (!stage_ready(zbar, op.wait_test, op.status)) return;
    }
    C X[2][R2];
    if (lane < R1 && live) {
        const int k1 = lane;
        if (staged) {
            const C* src = E + r * (2 * N);
#pragma unroll
            for (int k2 = 0; k2 < R2; k2++) {
                const int m = k1 + R1 * k2;
                X[0][k2] = src[2 * m];
                X[1][k2] = src[2 * m + 1];
            }
        } else {
            const C* src = op.b + ((long long)s * nrows + row) * (2 * N);
#pragma unroll
            for (int k2 = 0; k2 < R2; k2++) {
                const int m = k1 + R1 * k2;
                X[0][k2] = src[2 * m];
                X[1][k2] = src[2 * m + 1];
            }
        }
    }
    if (staged) __syncthreads();  // the staged rows are overwritten below
    if (lane < R1 && live) {
        const int k1 = lane;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            dft_reg<R2, true>(X[h]);
#pragma unroll
            for (int n2 = 0; n2 < R2; n2++) {
                const C t = n2 ? cmulc(X[h][n2], tw[2 * n2 * k1]) : X[h][n2];
                E[h * HS + (r * R2 + n2) * SR + k1] = t;
            }
        }
    }
    __syncthreads();
    constexpr int KA = Epi::K > 0 ? Epi::K : 1;
    double2 acc[KA];
#pragma unroll
    for (int k = 0; k < KA; k++) acc[k] = make_double2(0.0, 0.0);
    if (lane < R2 && live) {
        const int n2 = lane;
        C y0[R1], y1[R1];
#pragma unroll
        for (int k1 = 0; k1 < R1; k1++) {
            y0[k1] = E[(r * R2 + n2) * SR + k1];
            y1[k1] = E[HS + (r * R2 + n2) * SR + k1];
        }
        dft_reg<R1, true>(y0);
        dft_reg<R1, true>(y1);
        const int i = (int)(row / op.ny), j = (int)(row - (long long)i * op.ny);
        const bool vrow = (s != 0 || i < op.nx - 1) && (s != 1 || j < op.ny - 1);
        const long long sstep = s == 0 ? (long long)op.ny * N : (s == 1 ? (long long)N : 1LL);
        const R dc = op.dcoef[s];
        const bool use_green = op.parts & 1, use_diag = op.parts & 2, use_mask = op.parts & 4;
        // crop: the Green part y0 + W_2N^{-n} y1 of every element (frees the two halves)
        C g[R1];
#pragma unroll
        for (int n1 = 0; n1 < R1; n1++)
            g[n1] = use_green ? cadd(y0[n1], cmulc(y1[n1], tw[n2 + R2 * n1])) : czero<C>();
        // all reads of a chunk of elements (flags, contrast pair, diagonal source,
        // the epilogue's vector) are issued before its arithmetic and stores;
        // the selections below give the results of the branchy form bit for bit
        constexpr int CH = R1 % 4 == 0 ? 4 : 1;
#pragma unroll
        for (int c0 = 0; c0 < R1; c0 += CH) {
            unsigned char fl[CH];
            C wa[CH], wb[CH], xv[CH], pv[CH];
#pragma unroll
            for (int q = 0; q < CH; q++) {
                const int n = n2 + R2 * (c0 + q);
                const long long idx = row * N + n;
                const bool dv = vrow && (s != 2 || n < N - 1);
                fl[q] = op.flags[idx];
                wa[q] = op.w[idx];
                wb[q] = op.w[dv ? idx + sstep : idx];
                xv[q] = xin[(long long)s * op.a + idx];
                pv[q] = epi.pre(s, idx);
            }
#pragma unroll
            for (int q = 0; q < CH; q++) {
                const int n1 = c0 + q;
                const int n = n2 + R2 * n1;
                const long long idx = row * N + n;
                const bool dv = use_diag && vrow && (s != 2 || n < N - 1);
                C y = g[n1];
                const C ws = cadd(wb[q], wa[q]);
                C coef = mkc(-dc * ws.y, dc * ws.x);
                if (conj) coef = cconj(coef);
                const C yd = cadd(y, cmul(coef, xv[q]));
                y = dv ? yd : y;
                y = (!use_mask || ((fl[q] >> s) & 1)) ? y : czero<C>();
                epi.put(s, idx, y, acc, pv[q]);
            }
        }
    }
    if constexpr (Epi::K > 0) block_reduce_store<KA>(acc, partial, (long long)s * gdx + bx);
}
template <typename C, int N, class Epi>
__global__ void __launch_bounds__(FastLB<C, N>::ROW, FastLB<C, N>::ROW_MIN) kf_inv_z(OpDev<C> op, const C* __restrict__ xin, Epi epi,
                                                double2* __restrict__ partial, int conj) {
    kf_inv_z_blk<C, N, Epi>(op, xin, epi, partial, conj, blockIdx.x, blockIdx.y, gridDim.x);
}

// ---------------------------------------------------------------------------
// F2 (column pass): forward y.  grid (kz tiles of TP, nx, 3).
// E layout: E[h][k1][n2][tx].
// ---------------------------------------------------------------------------
template <typename C, int N>
__device__ __forceinline__ void kf_fwd_y_blk(const OpDev<C>& op, const int bx, const int i, const int s) {
    if (gate_closed(op.gate)) return;
    constexpr int R1 = FastPlan<N>::R1, R2 = FastPlan<N>::R2, TP = FastTiles<C>::TP_Y;
    constexpr int HS = N * TP;
    C* tw;
    C* E = fast_smem<C, N>(op.ax[1].tw, tw);
    const int tx = threadIdx.x % TP, lane = threadIdx.x / TP;
    const int Lz = 2 * op.nz;
    const int kz = bx * TP + tx;
    const bool live = kz < Lz;
    const C* src = op.b + ((long long)s * op.nx + i) * (long long)N * Lz;
    __syncthreads();
    if (lane < R2 && live) {
        const int n2 = lane;
        C v[R1];
#pragma unroll
        for (int n1 = 0; n1 < R1; n1++) v[n1] = src[(long long)(n2 + R2 * n1) * Lz + kz];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            C a[R1];
#pragma unroll
            for (int n1 = 0; n1 < R1; n1++) a[n1] = h ? cmul(v[n1], tw[n2 + R2 * n1]) : v[n1];
            dft_reg<R1, false>(a);
#pragma unroll
            for (int k1 = 0; k1 < R1; k1++)
                E[h * HS + (k1 * R2 + n2) * TP + tx] = k1 ? cmul(a[k1], tw[2 * n2 * k1]) : a[k1];
        }
    }
    __syncthreads();
    if (lane < R1 && live) {
        const int k1 = lane;
        C* dst = op.c + ((long long)s * op.nx + i) * (long long)(2 * N) * Lz;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            C X[R2];
#pragma unroll
            for (int n2 = 0; n2 < R2; n2++) X[n2] = E[h * HS + (k1 * R2 + n2) * TP + tx];
            dft_reg<R2, false>(X);
#pragma unroll
            for (int k2 = 0; k2 < R2; k2++) dst[(long long)(h * N + k1 + R1 * k2) * Lz + kz] = X[k2];
        }
    }
}
template <typename C, int N>
__global__ void __launch_bounds__(FastLB<C, N>::COL, FastLB<C, N>::COL_MIN) kf_fwd_y(OpDev<C> op) {
    kf_fwd_y_blk<C, N>(op, blockIdx.x, blockIdx.y, blockIdx.z);
}

// F2 with its pencil tile staged by TMA: one cp.async.bulk.tensor load of the
// [N rows x TP columns] slab tile into the front of E (the shared buffer the
// pass transposes through), completion on an mbarrier, then the same
// arithmetic as kf_fwd_y reading its inputs from shared memory.  The tensor
// map views b as 2D (columns: 2 Lz reals, rows: 3 nx N).  The x coordinate,
// 2 kz0 reals = 8 kz0 (FP32) or 16 kz0 (FP64) bytes with kz0 a multiple of TP,
// is always a multiple of 128 bytes; no multicast.  The wait is bounded (see
// mbar_wait_bounded).

template <typename C, int N>
__global__ void __launch_bounds__(FastLB<C, N>::COL, FastLB<C, N>::COL_MIN)
    kf_fwd_y_tma(OpDev<C> op, const __grid_constant__ CUtensorMap tm) {
    if (gate_closed(op.gate)) return;
    constexpr int R1 = FastPlan<N>::R1, R2 = FastPlan<N>::R2, TP = FastTiles<C>::TP_Y;
    constexpr int HS = N * TP;
    __shared__ __align__(8) unsigned long long bar[2];
    C* tw;
    C* E = fast_smem<C, N>(op.ax[1].tw, tw);
    // the TMA destination 128-byte aligned (the launch reserves 128 more bytes)
    E = reinterpret_cast<C*>(reinterpret_cast<char*>(E) + ((128u - (smem_u32(E) & 127u)) & 127u));
    const int tx = threadIdx.x % TP, lane = threadIdx.x / TP;
    const int Lz = 2 * op.nz;
    const int kz = blockIdx.x * TP + tx, i = blockIdx.y, s = blockIdx.z;
    const bool live = kz < Lz;
    const unsigned b = smem_u32(bar);
    if (threadIdx.x == 0) stage_init(bar);
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_expect(b, (unsigned)(sizeof(C) * N * TP));
        const int x = 2 * (int)blockIdx.x * TP;                    // reals
        const int y = ((int)blockIdx.z * op.nx + (int)blockIdx.y) * N;  // rows
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
            ::"r"(smem_u32(E)), "l"(&tm), "r"(x), "r"(y), "r"(b)
            : "memory");
    }
    if (!stage_ready(bar, op.wait_test, op.status)) return;
    // inputs of this thread from the staged tile (row n = n2 + R2 n1, column tx)
    C v[R1];
    const int n2 = lane;
    if (lane < R2 && live) {
#pragma unroll
        for (int n1 = 0; n1 < R1; n1++) v[n1] = E[(n2 + R2 * n1) * TP + tx];
    }
    __syncthreads();  // the tile is overwritten below
    if (lane < R2 && live) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
            C a[R1];
#pragma unroll
            for (int n1 = 0; n1 < R1; n1++) a[n1] = h ? cmul(v[n1], tw[n2 + R2 * n1]) : v[n1];
            dft_reg<R1, false>(a);
#pragma unroll
            for (int k1 = 0; k1 < R1; k1++)
                E[h * HS + (k1 * R2 + n2) * TP + tx] = k1 ? cmul(a[k1], tw[2 * n2 * k1]) : a[k1];
        }
    }
    __syncthreads();
    if (lane < R1 && live) {
        const int k1 = lane;
        C* dst = op.c + ((long long)s * op.nx + i) * (long long)(2 * N) * Lz;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            C X[R2];
#pragma unroll
            for (int n2b = 0; n2b < R2; n2b++) X[n2b] = E[h * HS + (k1 * R2 + n2b) * TP + tx];
            dft_reg<R2, false>(X);
#pragma unroll
            for (int k2 = 0; k2 < R2; k2++) dst[(long long)(h * N + k1 + R1 * k2) * Lz + kz] = X[k2];
        }
    }
}

// I2 (column pass): inverse y, crop.  E layout: E[h][n2][k1][tx].
template <typename C, int N>
__device__ __forceinline__ void kf_inv_y_blk(const OpDev<C>& op, const int bx, const int i, const int s) {
    if (gate_closed(op.gate)) return;
    constexpr int R1 = FastPlan<N>::R1, R2 = FastPlan<N>::R2, TP = FastTiles<C>::TP_Y;
    constexpr int HS = N * TP;
    C* tw;
    C* E = fast_smem<C, N>(op.ax[1].tw, tw);
    const int tx = threadIdx.x % TP, lane = threadIdx.x / TP;
    const int Lz = 2 * op.nz;
    const int kz = bx * TP + tx;
    const bool live = kz < Lz;
    const C* src = op.c + ((long long)s * op.nx + i) * (long long)(2 * N) * Lz;
    __syncthreads();
    if (lane < R1 && live) {
        const int k1 = lane;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            C X[R2];
#pragma unroll
            for (int k2 = 0; k2 < R2; k2++) X[k2] = src[(long long)(h * N + k1 + R1 * k2) * Lz + kz];
            dft_reg<R2, true>(X);
#pragma unroll
            for (int n2 = 0; n2 < R2; n2++)
                E[h * HS + (n2 * R1 + k1) * TP + tx] = n2 ? cmulc(X[n2], tw[2 * n2 * k1]) : X[n2];
        }
    }
    __syncthreads();
    if (lane < R2 && live) {
        const int n2 = lane;
        C y0[R1], y1[R1];
#pragma unroll
        for (int k1 = 0; k1 < R1; k1++) {
            y0[k1] = E[(n2 * R1 + k1) * TP + tx];
            y1[k1] = E[HS + (n2 * R1 + k1) * TP + tx];
        }
        dft_reg<R1, true>(y0);
        dft_reg<R1, true>(y1);
        C* dst = op.b + ((long long)s * op.nx + i) * (long long)N * Lz;
#pragma unroll
        for (int n1 = 0; n1 < R1; n1++) {
            const int n = n2 + R2 * n1;
            dst[(long long)n * Lz + kz] = cadd(y0[n1], cmulc(y1[n1], tw[n]));
        }
    }
}
template <typename C, int N>
__global__ void __launch_bounds__(FastLB<C, N>::COL, FastLB<C, N>::COL_MIN) kf_inv_y(OpDev<C> op) {
    kf_inv_y_blk<C, N>(op, blockIdx.x, blockIdx.y, blockIdx.z);
}

// I2 with its tile staged by TMA: the [2N rows x TP columns] spectra tile as two
// boxes of N rows (the box height limit is 256) into E, one mbarrier; the same
// alignment, bounded wait and arithmetic rules as kf_fwd_y_tma.  Each half is
// read into registers before its results overwrite its part of E.
template <typename C, int N>
__global__ void __launch_bounds__(FastLB<C, N>::COL, FastLB<C, N>::COL_MIN)
    kf_inv_y_tma(OpDev<C> op, const __grid_constant__ CUtensorMap tm) {
    if (gate_closed(op.gate)) return;
    constexpr int R1 = FastPlan<N>::R1, R2 = FastPlan<N>::R2, TP = FastTiles<C>::TP_Y;
    constexpr int HS = N * TP;
    __shared__ __align__(8) unsigned long long bar[2];
    C* tw;
    C* E = fast_smem<C, N>(op.ax[1].tw, tw);
    E = reinterpret_cast<C*>(reinterpret_cast<char*>(E) + ((128u - (smem_u32(E) & 127u)) & 127u));
    const int tx = threadIdx.x % TP, lane = threadIdx.x / TP;
    const int Lz = 2 * op.nz;
    const int kz = blockIdx.x * TP + tx, i = blockIdx.y, s = blockIdx.z;
    const bool live = kz < Lz;
    const unsigned b = smem_u32(bar);
    if (threadIdx.x == 0) stage_init(bar);
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_expect(b, (unsigned)(sizeof(C) * 2 * N * TP));
        const int x = 2 * (int)blockIdx.x * TP;
        const int y = ((int)blockIdx.z * op.nx + (int)blockIdx.y) * 2 * N;
#pragma unroll
        for (int h = 0; h < 2; h++)
            asm volatile(
                "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
                "[%4];" ::"r"(smem_u32(E + h * HS)),
                "l"(&tm), "r"(x), "r"(y + h * N), "r"(b)
                : "memory");
    }
    if (!stage_ready(bar, op.wait_test, op.status)) return;
    const int k1 = lane;
#pragma unroll
    for (int h = 0; h < 2; h++) {
        C X[R2];
        if (lane < R1 && live) {
#pragma unroll
            for (int k2 = 0; k2 < R2; k2++) X[k2] = E[h * HS + (k1 + R1 * k2) * TP + tx];
        }
        __syncthreads();  // this half of the tile is overwritten below
        if (lane < R1 && live) {
            dft_reg<R2, true>(X);
#pragma unroll
            for (int n2 = 0; n2 < R2; n2++)
                E[h * HS + (n2 * R1 + k1) * TP + tx] = n2 ? cmulc(X[n2], tw[2 * n2 * k1]) : X[n2];
        }
    }
    __syncthreads();
    if (lane < R2 && live) {
        const int n2 = lane;
        C y0[R1], y1[R1];
#pragma unroll
        for (int q = 0; q < R1; q++) {
            y0[q] = E[(n2 * R1 + q) * TP + tx];
            y1[q] = E[HS + (n2 * R1 + q) * TP + tx];
        }
        dft_reg<R1, true>(y0);
        dft_reg<R1, true>(y1);
        C* dst = op.b + ((long long)s * op.nx + i) * (long long)N * Lz;
#pragma unroll
        for (int n1 = 0; n1 < R1; n1++) {
            const int n = n2 + R2 * n1;
            dst[(long long)n * Lz + kz] = cadd(y0[n1], cmulc(y1[n1], tw[n]));
        }
    }
}

// ---------------------------------------------------------------------------
// F3 (column pass, three components): forward x, spectral multiply, inverse x,
// crop.  grid (kz tiles of TP, 2ny).  E layout: E[s][h][k1][n2][tx], k1 blocks
// padded by TP entries (forward)
// then E[s][h][k1][k2][tx] (spectra) then E[s][h][k1][n2][tx] (inverse).
// Thread roles: steps A/A' (tx, s, n2); step B / multiply / B' (tx, h, k1).
// ---------------------------------------------------------------------------
// (conj: the adjoint operator's tables and conj(Gs); a run-time flag)
template <typename C, int N, int TP>
__device__ __forceinline__ void kf_x_spectral_blk(const OpDev<C>& op, const int conj, const int bx, const int ky) {
    if (gate_closed(op.gate)) return;
    using R = typename real_of<C>::type;
    constexpr int R1 = FastPlan<N>::R1, R2 = FastPlan<N>::R2;
    constexpr int L = R1 > R2 ? R1 : R2;
    constexpr int KS = fast_x_kstride<C, N, TP>();  // stride of k1 (R2*TP + TP padding)
    constexpr int HS = R1 * KS, SS = 2 * HS;
    C* tw;
    C* E = fast_smem<C, N>(op.ax[0].tw, tw);
    const int Lz = 2 * op.nz, Ly = 2 * op.ny;
    const long long cs = (long long)Ly * Lz;
    const int tx = threadIdx.x % TP;
    const int kz = bx * TP + tx;
    const bool live = kz < Lz;
    __syncthreads();
    // step A: thread (tx, s, n2)
    {
        const int q = threadIdx.x / TP;  // 0 .. 3L-1
        const int s = q / L, n2 = q % L;
        if (s < 3 && n2 < R2 && live) {
            C v[R1];
#pragma unroll
            for (int n1 = 0; n1 < R1; n1++)
                v[n1] = op.c[((long long)s * N + n2 + R2 * n1) * cs + (long long)ky * Lz + kz];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                C a[R1];
#pragma unroll
                for (int n1 = 0; n1 < R1; n1++) a[n1] = h ? cmul(v[n1], tw[n2 + R2 * n1]) : v[n1];
                dft_reg<R1, false>(a);
#pragma unroll
                for (int k1 = 0; k1 < R1; k1++)
                    E[s * SS + h * HS + k1 * KS + n2 * TP + tx] = k1 ? cmul(a[k1], tw[2 * n2 * k1]) : a[k1];
            }
        }
    }
    __syncthreads();
    // step B, multiply, step B': thread (tx, h, k1); every element it touches is its own
    {
        const int q = threadIdx.x / TP;
        const int h = q / R1, k1 = q % R1;
        if (h < 2 && live) {
            const int md = conj ? 1 : 0;
            C* base = E + h * HS + k1 * KS + tx;  // + s*SS + k2*TP
#pragma unroll
            for (int s = 0; s < 3; s++) {
                C X[R2];
#pragma unroll
                for (int n2 = 0; n2 < R2; n2++) X[n2] = base[s * SS + n2 * TP];
                dft_reg<R2, false>(X);
#pragma unroll
                for (int k2 = 0; k2 < R2; k2++) base[s * SS + k2 * TP] = X[k2];
            }
            const C Py = op.ax[1].P[md][ky], Qy = op.ax[1].Q[md][ky];
            const int gy = op.ax[1].gfold[ky];
            const C Pz = op.ax[2].P[md][kz], Qz = op.ax[2].Q[md][kz];
            const int gz = op.ax[2].gfold[kz];
            const R kx_ = op.kappa[0], ky_ = op.kappa[1], kz_ = op.kappa[2];
#pragma unroll 4
            for (int k2 = 0; k2 < R2; k2++) {
                const int sx = h * N + k1 + R1 * k2;
                const C Px = op.ax[0].P[md][sx], Qx = op.ax[0].Q[md][sx];
                // slot h N + m holds frequency k = 2m + h; its octant index folds k > N
                const int kx = 2 * (k1 + R1 * k2) + h;
                const int gx = kx <= N ? kx : 2 * N - kx;
                C G = op.Gs[((long long)gx * (op.ny + 1) + gy) * (op.nz + 1) + gz];
                if (conj) G = cconj(G);
                C* e = base + k2 * TP;
                const C Jx = e[0], Jy = e[SS], Jz = e[2 * SS];
                const C rho = cadd(cadd(cmul(Px, Jx), cmul(Py, Jy)), cmul(Pz, Jz));
                e[0] = cmul(G, cadd(cscale(Jx, kx_), cmul(Qx, rho)));
                e[SS] = cmul(G, cadd(cscale(Jy, ky_), cmul(Qy, rho)));
                e[2 * SS] = cmul(G, cadd(cscale(Jz, kz_), cmul(Qz, rho)));
            }
#pragma unroll
            for (int s = 0; s < 3; s++) {
                C X[R2];
#pragma unroll
                for (int k2 = 0; k2 < R2; k2++) X[k2] = base[s * SS + k2 * TP];
                dft_reg<R2, true>(X);
#pragma unroll
                for (int n2 = 0; n2 < R2; n2++) base[s * SS + n2 * TP] = n2 ? cmulc(X[n2], tw[2 * n2 * k1]) : X[n2];
            }
        }
    }
    __syncthreads();
    // step A': thread (tx, s, n2)
    {
        const int q = threadIdx.x / TP;
        const int s = q / L, n2 = q % L;
        if (s < 3 && n2 < R2 && live) {
            C y0[R1], y1[R1];
#pragma unroll
            for (int k1 = 0; k1 < R1; k1++) {
                y0[k1] = E[s * SS + k1 * KS + n2 * TP + tx];
                y1[k1] = E[s * SS + HS + k1 * KS + n2 * TP + tx];
            }
            dft_reg<R1, true>(y0);
            dft_reg<R1, true>(y1);
#pragma unroll
            for (int n1 = 0; n1 < R1; n1++) {
                const int n = n2 + R2 * n1;
                op.c[((long long)s * N + n) * cs + (long long)ky * Lz + kz] = cadd(y0[n1], cmulc(y1[n1], tw[n]));
            }
        }
    }
}
template <typename C, int N, int TP>
__global__ void __launch_bounds__(FastXLB<C, TP>::XT, FastXLB<C, TP>::X_MIN) kf_x_spectral(OpDev<C> op, int conj) {
    kf_x_spectral_blk<C, N, TP>(op, conj, blockIdx.x, blockIdx.y);
}

template <typename C, int N, int TP = FastTiles<C>::TP_X> constexpr int fast_x_threads() {
    return 3 * (FastPlan<N>::R1 > FastPlan<N>::R2 ? FastPlan<N>::R1 : FastPlan<N>::R2) * TP;
}

}  // namespace vie
