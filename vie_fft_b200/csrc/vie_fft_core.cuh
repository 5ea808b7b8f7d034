// vie_fft_core.cuh -- batched in-shared-memory FFT stages for the VIE operator.
//
// A batch of pencils of length N lives in shared memory in "pencil-minor"
// layout: element n of pencil t of set f sits at buf[f*fstride + n*TP + t].
// Threads are mapped pencil-fastest, so every stage touches contiguous words
// for consecutive threads.
//
// Forward: in-place mixed-radix decimation in frequency.  Natural-order input,
// digit-reversed output: with radices R1..Rk, position
//     p = q1*(N/R1) + q2*(N/(R1 R2)) + ... + qk
// holds X[q1 + R1 q2 + R1 R2 q3 + ...].
// Inverse: the exact transpose (decimation in time, conjugate twiddles),
// digit-reversed input, natural-order output, unnormalised.
//
// Twiddles come from a table tw[u] = exp(-2 pi i u / (2N)), u in [0, 2N)
// (the half-length twiddles exp(-2 pi i t / N) are tw[2t]); the same table
// provides the exp(-2 pi i n / 2N) factors of the zero-padding split.
#pragma once
#include <type_traits>
#include "vie_complex.cuh"

namespace vie {

constexpr int kMaxStages = 12;
constexpr int kMaxGenericRadix = 64;

struct AxisPlan {
    int n;                    // transform length (unpadded axis length)
    int nst;                  // number of stages
    int rad[kMaxStages];      // radices in DIF order
};

// ---------------------------------------------------------------------------
// radix codelets: y[q] = sum_r v[r] W_R^{r q}, W_R = exp(-/+ 2 pi i / R)
// ---------------------------------------------------------------------------
template <bool INV, typename C> __host__ __device__ __forceinline__ C mul_mi_dir(C a) {
    // forward: multiply by -i; inverse: by +i
    return INV ? cmul_pi(a) : cmul_mi(a);
}

template <bool INV, typename C> __host__ __device__ __forceinline__ void dft2(C& a, C& b) {
    C t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

template <bool INV, typename C> __host__ __device__ __forceinline__ void dft4(C& v0, C& v1, C& v2, C& v3) {
    C a0 = cadd(v0, v2), a1 = csub(v0, v2);
    C b0 = cadd(v1, v3), b1 = mul_mi_dir<INV>(csub(v1, v3));
    v0 = cadd(a0, b0);
    v2 = csub(a0, b0);
    v1 = cadd(a1, b1);
    v3 = csub(a1, b1);
}

template <typename C> struct RealT { using R = typename real_of<C>::type; };

// multiply by exp(-/+ i pi/4), exp(-/+ i 3pi/4)
template <bool INV, typename C> __host__ __device__ __forceinline__ C w8_1(C x) {
    using R = typename real_of<C>::type;
    const R h = (R)0.70710678118654752440084436210485;
    return INV ? mkc(h * (x.x - x.y), h * (x.y + x.x)) : mkc(h * (x.x + x.y), h * (x.y - x.x));
}
template <bool INV, typename C> __host__ __device__ __forceinline__ C w8_3(C x) {
    using R = typename real_of<C>::type;
    const R h = (R)0.70710678118654752440084436210485;
    return INV ? mkc(h * (-x.x - x.y), h * (x.x - x.y)) : mkc(h * (-x.x + x.y), h * (-x.y - x.x));
}

template <bool INV, typename C> __host__ __device__ __forceinline__ void dft8(C* v) {
    C u0 = cadd(v[0], v[4]), u1 = cadd(v[1], v[5]), u2 = cadd(v[2], v[6]), u3 = cadd(v[3], v[7]);
    C w0 = csub(v[0], v[4]);
    C w1 = w8_1<INV>(csub(v[1], v[5]));
    C w2 = mul_mi_dir<INV>(csub(v[2], v[6]));
    C w3 = w8_3<INV>(csub(v[3], v[7]));
    dft4<INV>(u0, u1, u2, u3);
    dft4<INV>(w0, w1, w2, w3);
    v[0] = u0; v[2] = u1; v[4] = u2; v[6] = u3;
    v[1] = w0; v[3] = w1; v[5] = w2; v[7] = w3;
}

template <bool INV, typename C> __host__ __device__ __forceinline__ void dft16(C* v) {
    using R = typename real_of<C>::type;
    const R c1 = (R)0.92387953251128675612818318939679;  // cos(pi/8)
    const R s1 = (R)0.38268343236508977172845998403040;  // sin(pi/8)
    const R h = (R)0.70710678118654752440084436210485;
    const R sg = INV ? (R)1 : (R)-1;                       // sign of the imaginary part
    C u[8], w[8];
#pragma unroll
    for (int r = 0; r < 8; r++) {
        u[r] = cadd(v[r], v[r + 8]);
        w[r] = csub(v[r], v[r + 8]);
    }
    // w[r] *= exp(sg * i * 2 pi r / 16)
    w[1] = cmul(w[1], mkc(c1, sg * s1));
    w[2] = cmul(w[2], mkc(h, sg * h));
    w[3] = cmul(w[3], mkc(s1, sg * c1));
    w[4] = mul_mi_dir<INV>(w[4]);
    w[5] = cmul(w[5], mkc(-s1, sg * c1));
    w[6] = cmul(w[6], mkc(-h, sg * h));
    w[7] = cmul(w[7], mkc(-c1, sg * s1));
    dft8<INV>(u);
    dft8<INV>(w);
#pragma unroll
    for (int q = 0; q < 8; q++) {
        v[2 * q] = u[q];
        v[2 * q + 1] = w[q];
    }
}

template <bool INV, typename C> __host__ __device__ __forceinline__ void dft3(C* v) {
    using R = typename real_of<C>::type;
    const R s3 = (R)0.86602540378443864676372317075294;
    C t1 = cadd(v[1], v[2]);
    C t2 = csub(v[0], cscale(t1, (R)0.5));
    C t3 = cscale(csub(v[1], v[2]), s3);
    C jt3 = mul_mi_dir<INV>(t3);  // forward: -i t3
    v[0] = cadd(v[0], t1);
    v[1] = cadd(t2, jt3);
    v[2] = csub(t2, jt3);
}

template <bool INV, typename C> __host__ __device__ __forceinline__ void dft5(C* v) {
    using R = typename real_of<C>::type;
    const R c1 = (R)0.30901699437494742410229341718282;   // cos(2pi/5)
    const R c2 = (R)-0.80901699437494742410229341718282;  // cos(4pi/5)
    const R s1 = (R)0.95105651629515357211643933337938;   // sin(2pi/5)
    const R s2 = (R)0.58778525229247312916870595463907;   // sin(4pi/5)
    C a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
    C a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
    C x0 = v[0];
    C p1 = cadd(x0, cadd(cscale(a1, c1), cscale(a2, c2)));
    C p2 = cadd(x0, cadd(cscale(a1, c2), cscale(a2, c1)));
    C q1 = mul_mi_dir<INV>(cadd(cscale(b1, s1), cscale(b2, s2)));
    C q2 = mul_mi_dir<INV>(csub(cscale(b1, s2), cscale(b2, s1)));
    v[0] = cadd(x0, cadd(a1, a2));
    v[1] = cadd(p1, q1);
    v[4] = csub(p1, q1);
    v[2] = cadd(p2, q2);
    v[3] = csub(p2, q2);
}

// ---------------------------------------------------------------------------
// compile-time twiddles W_R^e = exp(-2 pi i e / R) for the register codelets
// of radices 6, 7, 9, 10, 11, 12.  cos/sin come from Taylor series evaluated
// by the compiler after reduction of the angle to |r| <= pi/4 around the
// nearest quarter turn (exact integer reduction; 12 terms leave < 1e-20).
// ---------------------------------------------------------------------------
struct CtCS {
    double c, s;
};
__host__ __device__ constexpr CtCS ct_cos_sin_2pi(long long p, long long q) {
    constexpr double two_pi = 6.283185307179586476925286766559;
    p %= q;
    if (p < 0) p += q;
    const long long k = (4 * p + q / 2) / q;             // nearest quarter turn
    const double r = two_pi * (double)(4 * p - k * q) / (double)(4 * q);
    double sn = r, cs = 1.0, ts = r, tc = 1.0;
    for (int n = 1; n < 12; n++) {
        ts *= -r * r / (double)((2 * n) * (2 * n + 1));
        tc *= -r * r / (double)((2 * n - 1) * (2 * n));
        sn += ts;
        cs += tc;
    }
    switch (k & 3) {
        case 0: return CtCS{cs, sn};
        case 1: return CtCS{-sn, cs};
        case 2: return CtCS{-cs, -sn};
        default: return CtCS{sn, -cs};
    }
}
template <int E, int R> struct CtW {
    static constexpr CtCS v = ct_cos_sin_2pi(E, R);
    static constexpr double c = v.c, s = v.s;   // W_R^E = c - i s
};

template <int B, int E, class F> __host__ __device__ __forceinline__ void static_for(F&& f) {
    if constexpr (B < E) {
        f(std::integral_constant<int, B>{});
        static_for<B + 1, E>(f);
    }
}

// x * W_R^E (forward) or x * conj(W_R^E) (inverse)
template <int R, int E, bool INV, typename C> __host__ __device__ __forceinline__ C ct_twiddle(C x) {
    using Rl = typename real_of<C>::type;
    constexpr int e = ((E % R) + R) % R;
    if constexpr (e == 0) {
        return x;
    } else {
        constexpr double c = CtW<e, R>::c, sn = INV ? -CtW<e, R>::s : CtW<e, R>::s;
        // (c - i sn) x
        return mkc((Rl)c * x.x + (Rl)sn * x.y, (Rl)c * x.y - (Rl)sn * x.x);
    }
}

template <int R, bool INV, typename C> __host__ __device__ __forceinline__ void dft_reg_any(C* v);

// odd R: pairs r, R-r folded, X_k = x0 + sum a_r cos - i sum b_r sin (forward)
template <int R, bool INV, typename C> __host__ __device__ __forceinline__ void dft_odd(C* v) {
    using Rl = typename real_of<C>::type;
    constexpr int H = (R - 1) / 2;
    C a[H], b[H];
    const C x0 = v[0];
    C sum = x0;
#pragma unroll
    for (int j = 0; j < H; j++) {
        a[j] = cadd(v[j + 1], v[R - 1 - j]);
        b[j] = csub(v[j + 1], v[R - 1 - j]);
        sum = cadd(sum, a[j]);
    }
    v[0] = sum;
    static_for<1, H + 1>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        C re = x0, im = czero<C>();
        static_for<0, H>([&](auto jc) {
            constexpr int j = decltype(jc)::value;
            constexpr int e = ((j + 1) * k) % R;
            re = cadd(re, cscale(a[j], (Rl)CtW<e, R>::c));
            im = cadd(im, cscale(b[j], (Rl)CtW<e, R>::s));
        });
        const C jim = INV ? cmul_pi(im) : cmul_mi(im);
        v[k] = cadd(re, jim);
        v[R - k] = csub(re, jim);
    });
}

// R = P Q in registers: DFT_P over stride-Q subsequences, twiddles W_R^{n2 k1},
// DFT_Q; natural order in and out
template <int P, int Q, bool INV, typename C> __host__ __device__ __forceinline__ void dft_pq(C* v) {
    constexpr int R = P * Q;
    C t[R];
    static_for<0, Q>([&](auto n2c) {
        constexpr int n2 = decltype(n2c)::value;
        C u[P];
#pragma unroll
        for (int n1 = 0; n1 < P; n1++) u[n1] = v[n2 + Q * n1];
        dft_reg_any<P, INV>(u);
        static_for<0, P>([&](auto k1c) {
            constexpr int k1 = decltype(k1c)::value;
            t[n2 * P + k1] = ct_twiddle<R, n2 * k1, INV>(u[k1]);
        });
    });
#pragma unroll
    for (int k1 = 0; k1 < P; k1++) {
        C w[Q];
#pragma unroll
        for (int n2 = 0; n2 < Q; n2++) w[n2] = t[n2 * P + k1];
        dft_reg_any<Q, INV>(w);
#pragma unroll
        for (int k2 = 0; k2 < Q; k2++) v[k1 + P * k2] = w[k2];
    }
}

// register DFT of a compile-time radix
template <int R, bool INV, typename C> __host__ __device__ __forceinline__ void dft_reg_any(C* v) {
    if constexpr (R == 1) {
    } else if constexpr (R == 2) dft2<INV>(v[0], v[1]);
    else if constexpr (R == 3) dft3<INV>(v);
    else if constexpr (R == 4) dft4<INV>(v[0], v[1], v[2], v[3]);
    else if constexpr (R == 5) dft5<INV>(v);
    else if constexpr (R == 6) dft_pq<2, 3, INV>(v);
    else if constexpr (R == 8) dft8<INV>(v);
    else if constexpr (R == 9) dft_pq<3, 3, INV>(v);
    else if constexpr (R == 10) dft_pq<2, 5, INV>(v);
    else if constexpr (R == 12) dft_pq<4, 3, INV>(v);
    else if constexpr (R == 15) dft_pq<3, 5, INV>(v);
    else if constexpr (R == 16) dft16<INV>(v);
    else if constexpr (R % 2 == 1) dft_odd<R, INV>(v);
    else static_assert(R == 2, "unsupported register radix");
}

// direct O(R^2) DFT for any other radix; W_R^e = tw[2 e (N/R)] (tw has 2N entries)
template <bool INV, int RMAX, typename C>
__host__ __device__ __forceinline__ void dft_generic(C* v, int R, const C* tw, int N) {
    C y[RMAX];
    const int st = 2 * (N / R);
    for (int q = 0; q < R; q++) {
        C acc = v[0];
        int e = 0;
        for (int r = 1; r < R; r++) {
            e += q;
            if (e >= R) e -= R;
            C w = tw[e * st];
            acc = cadd(acc, INV ? cmulc(v[r], w) : cmul(v[r], w));
        }
        y[q] = acc;
    }
    for (int q = 0; q < R; q++) v[q] = y[q];
}

template <int R, bool INV, typename C>
__host__ __device__ __forceinline__ void dft_fixed(C* v, const C* tw, int N) {
    if constexpr (R == 2) dft2<INV>(v[0], v[1]);
    else if constexpr (R == 3) dft3<INV>(v);
    else if constexpr (R == 4) dft4<INV>(v[0], v[1], v[2], v[3]);
    else if constexpr (R == 5) dft5<INV>(v);
    else if constexpr (R == 8) dft8<INV>(v);
    else if constexpr (R == 16) dft16<INV>(v);
    else dft_generic<INV, R>(v, R, tw, N);
}

// ---------------------------------------------------------------------------
// one stage over every (set, pencil, butterfly) work item
// ---------------------------------------------------------------------------
template <int R, bool INV, typename C>
__host__ __device__ __forceinline__ void fft_stage(C* __restrict__ buf, int nsets, int fstride, int T, int TP,
                                                   int N, int L, const C* __restrict__ tw, int tid, int nthr) {
    const int m = L / R;
    const int nb = N / R;
    const int total = nsets * T * nb;
    const int tws = 2 * (N / L);  // W_L^e = tw[e * tws]
    for (int w = tid; w < total; w += nthr) {
        const int t = w % T;
        const int rest = w / T;
        const int bj = rest % nb;
        const int f = rest / nb;
        const int b = bj / m;
        const int j = bj - b * m;
        C* base = buf + f * fstride + t + (b * L + j) * TP;
        C v[R];
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = base[r * m * TP];
        if (INV) {
            if (j != 0) {
#pragma unroll
                for (int q = 1; q < R; q++) v[q] = cmulc(v[q], tw[j * q * tws]);
            }
            dft_fixed<R, true>(v, tw, N);
        } else {
            dft_fixed<R, false>(v, tw, N);
            if (j != 0) {
#pragma unroll
                for (int q = 1; q < R; q++) v[q] = cmul(v[q], tw[j * q * tws]);
            }
        }
#pragma unroll
        for (int r = 0; r < R; r++) base[r * m * TP] = v[r];
    }
}

template <bool INV, typename C>
__host__ __device__ __noinline__ void fft_stage_runtime(C* __restrict__ buf, int nsets, int fstride, int T, int TP,
                                                        int N, int L, int R, const C* __restrict__ tw, int tid,
                                                        int nthr) {
    const int m = L / R;
    const int nb = N / R;
    const int total = nsets * T * nb;
    const int tws = 2 * (N / L);
    for (int w = tid; w < total; w += nthr) {
        const int t = w % T;
        const int rest = w / T;
        const int bj = rest % nb;
        const int f = rest / nb;
        const int b = bj / m;
        const int j = bj - b * m;
        C* base = buf + f * fstride + t + (b * L + j) * TP;
        C v[kMaxGenericRadix];
        for (int r = 0; r < R; r++) v[r] = base[r * m * TP];
        if (INV) {
            if (j != 0)
                for (int q = 1; q < R; q++) v[q] = cmulc(v[q], tw[j * q * tws]);
            dft_generic<true, kMaxGenericRadix>(v, R, tw, N);
        } else {
            dft_generic<false, kMaxGenericRadix>(v, R, tw, N);
            if (j != 0)
                for (int q = 1; q < R; q++) v[q] = cmul(v[q], tw[j * q * tws]);
        }
        for (int r = 0; r < R; r++) base[r * m * TP] = v[r];
    }
}

template <bool INV, typename C>
__host__ __device__ __forceinline__ void fft_stage_dispatch(C* buf, int nsets, int fstride, int T, int TP, int N,
                                                            int L, int R, const C* tw, int tid, int nthr) {
    switch (R) {
        case 2: fft_stage<2, INV>(buf, nsets, fstride, T, TP, N, L, tw, tid, nthr); break;
        case 3: fft_stage<3, INV>(buf, nsets, fstride, T, TP, N, L, tw, tid, nthr); break;
        case 4: fft_stage<4, INV>(buf, nsets, fstride, T, TP, N, L, tw, tid, nthr); break;
        case 5: fft_stage<5, INV>(buf, nsets, fstride, T, TP, N, L, tw, tid, nthr); break;
        case 7: fft_stage<7, INV>(buf, nsets, fstride, T, TP, N, L, tw, tid, nthr); break;
        case 8: fft_stage<8, INV>(buf, nsets, fstride, T, TP, N, L, tw, tid, nthr); break;
        case 16: fft_stage<16, INV>(buf, nsets, fstride, T, TP, N, L, tw, tid, nthr); break;
        default: fft_stage_runtime<INV>(buf, nsets, fstride, T, TP, N, L, R, tw, tid, nthr); break;
    }
}

// Forward DIF over all stages.  Caller syncs before; this syncs after each stage.
template <typename C>
__device__ __forceinline__ void smem_fft_fwd(C* buf, int nsets, int fstride, int T, int TP,
                                             const AxisPlan& pl, const C* tw) {
    int L = pl.n;
    for (int s = 0; s < pl.nst; s++) {
        const int R = pl.rad[s];
        fft_stage_dispatch<false>(buf, nsets, fstride, T, TP, pl.n, L, R, tw, threadIdx.x, blockDim.x);
        L /= R;
        __syncthreads();
    }
}

// Inverse DIT over all stages (reverse order).  Caller syncs before; syncs after each stage.
template <typename C>
__device__ __forceinline__ void smem_fft_inv(C* buf, int nsets, int fstride, int T, int TP,
                                             const AxisPlan& pl, const C* tw) {
    int m = 1;
    for (int s = pl.nst - 1; s >= 0; s--) {
        const int R = pl.rad[s];
        const int L = m * R;
        fft_stage_dispatch<true>(buf, nsets, fstride, T, TP, pl.n, L, R, tw, threadIdx.x, blockDim.x);
        m = L;
        __syncthreads();
    }
}

}  // namespace vie
