// vie_complex.cuh -- complex arithmetic on float2 / double2 for the VIE kernels.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace vie {

template <typename T> struct cplx_of;
template <> struct cplx_of<float> { using type = float2; };
template <> struct cplx_of<double> { using type = double2; };
template <typename T> using cplx_t = typename cplx_of<T>::type;

template <typename T> struct real_of;
template <> struct real_of<float2> { using type = float; };
template <> struct real_of<double2> { using type = double; };

__host__ __device__ __forceinline__ float2 mkc(float r, float i) { return make_float2(r, i); }
__host__ __device__ __forceinline__ double2 mkc(double r, double i) { return make_double2(r, i); }

template <typename C> __host__ __device__ __forceinline__ C czero() {
    C z; z.x = 0; z.y = 0; return z;
}

template <typename C> __host__ __device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename C> __host__ __device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
    C r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}
// a * conj(b)
template <typename C> __host__ __device__ __forceinline__ C cmulc(C a, C b) {
    C r;
    r.x = a.x * b.x + a.y * b.y;
    r.y = a.y * b.x - a.x * b.y;
    return r;
}
template <typename C> __host__ __device__ __forceinline__ C cconj(C a) { C r; r.x = a.x; r.y = -a.y; return r; }
template <typename C, typename R> __host__ __device__ __forceinline__ C cscale(C a, R s) { C r; r.x = a.x * s; r.y = a.y * s; return r; }
// multiply by +i (s=+1) or -i (s=-1)
template <typename C> __host__ __device__ __forceinline__ C cmul_pi(C a) { C r; r.x = -a.y; r.y = a.x; return r; }
template <typename C> __host__ __device__ __forceinline__ C cmul_mi(C a) { C r; r.x = a.y; r.y = -a.x; return r; }

// float2 complex add / subtract / scale with the paired FP32 instructions of
// sm_100 (one instruction per complex operation instead of two)
#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 1000)
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return __fmul2_rn(a, make_float2(s, s)); }
#endif

// conversions between precisions
__host__ __device__ __forceinline__ float2 to_f2(double2 a) { return make_float2((float)a.x, (float)a.y); }
__host__ __device__ __forceinline__ double2 to_d2(float2 a) { return make_double2((double)a.x, (double)a.y); }
template <typename C> __host__ __device__ __forceinline__ C from_d2(double2 a);
template <> __host__ __device__ __forceinline__ float2 from_d2<float2>(double2 a) { return to_f2(a); }
template <> __host__ __device__ __forceinline__ double2 from_d2<double2>(double2 a) { return a; }
template <typename C> __host__ __device__ __forceinline__ double2 as_d2(C a) { return make_double2((double)a.x, (double)a.y); }

}  // namespace vie
