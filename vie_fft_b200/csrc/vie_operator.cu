// vie_operator.cu -- host setup of the operator: radix plans, per-axis tables,
// Green octant scaling, contrast upload, scratch, and the plain matvec.
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "vie_launch.cuh"

namespace vie {

AxisPlan make_axis_plan(int n, const std::vector<int>& override_radices) {
    AxisPlan pl{};
    pl.n = n;
    pl.nst = 0;
    if (!override_radices.empty()) {
        int prod = 1;
        for (int r : override_radices) {
            if (pl.nst >= kMaxStages) break;
            pl.rad[pl.nst++] = r;
            prod *= r;
        }
        if (prod == n) return pl;
        pl.nst = 0;  // invalid override: fall back to the default
    }
    int m = n;
    while (m % 16 == 0 && pl.nst < kMaxStages) { pl.rad[pl.nst++] = 16; m /= 16; }
    if (m % 8 == 0) { pl.rad[pl.nst++] = 8; m /= 8; }
    else if (m % 4 == 0) { pl.rad[pl.nst++] = 4; m /= 4; }
    else if (m % 2 == 0) { pl.rad[pl.nst++] = 2; m /= 2; }
    for (int p = 3; m > 1 && pl.nst < kMaxStages; p += 2) {
        if (p * p > m) { pl.rad[pl.nst++] = m; m = 1; break; }
        while (m % p == 0 && pl.nst < kMaxStages) { pl.rad[pl.nst++] = p; m /= p; }
    }
    if (m > 1 && pl.nst < kMaxStages) pl.rad[pl.nst++] = m;
    return pl;
}

std::vector<int> axis_perm(const AxisPlan& pl) {
    std::vector<int> perm(pl.n);
    for (int m = 0; m < pl.n; m++) {
        int rem = m, pos = 0, span = pl.n;
        for (int s = 0; s < pl.nst; s++) {
            const int R = pl.rad[s];
            const int q = rem % R;
            rem /= R;
            span /= R;
            pos += q * span;
        }
        perm[m] = pos;
    }
    return perm;
}

// cuTensorMapEncodeTiled from the driver, through the runtime (no link to libcuda)
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

template <typename C> static C to_c(double re, double im);
template <> float2 to_c<float2>(double re, double im) { return make_float2((float)re, (float)im); }
template <> double2 to_c<double2>(double re, double im) { return make_double2(re, im); }

// Tile sizes: start from the defaults and halve while the pass does not fit
// in the shared-memory budget (two CTAs per SM where possible).
template <typename C> static int fit_tile(int t, int N, int nsets, int pad) {
    const size_t budget = 113 * 1024;
    while (t > 1 && pass_smem_bytes<C>(N, nsets, t + pad) > budget) t /= 2;
    return t;
}

template <typename T>
int Operator<T>::init(int nx, int ny, int nz, const double d[3], double k0, const TileCfg& tiles,
                      const AxisPlan plans[3], const unsigned char* d_flags, Error& err) {
    release();
    for (int ax = 0; ax < 3; ax++) {
        const AxisPlan& pl = plans[ax];
        for (int s = 0; s < pl.nst; s++)
            if (pl.rad[s] > kMaxGenericRadix) {
                err.code = VIE_ERR_ARG;
                err.msg = "axis length " + std::to_string(pl.n) + " has a prime factor above " +
                          std::to_string(kMaxGenericRadix);
                return VIE_ERR_ARG;
            }
    }
    OpDev<C>& o = dev;
    o = OpDev<C>{};
    o.nx = nx; o.ny = ny; o.nz = nz;
    o.a = (long long)nx * ny * nz;
    o.parts = VIE_PART_ALL;
    const bool dbl = sizeof(T) == 8;
    o.tz = fit_tile<C>(tiles.tz > 0 ? tiles.tz : (dbl ? 8 : 16), nz, 2, 1);
    o.tc = fit_tile<C>(tiles.tc > 0 ? tiles.tc : (dbl ? 8 : 16), ny, 2, 0);
    o.tx = fit_tile<C>(tiles.tx > 0 ? tiles.tx : (dbl ? 4 : 8), nx, 6, 0);
    smem_z = pass_smem_bytes<C>(nz, 2, o.tz + 1);
    smem_y = pass_smem_bytes<C>(ny, 2, o.tc);
    smem_x = pass_smem_bytes<C>(nx, 6, o.tx);
    if (smem_z > 227 * 1024 || smem_y > 227 * 1024 || smem_x > 227 * 1024) {
        err.code = VIE_ERR_ARG;
        err.msg = "grid axis too long for the shared-memory pencil passes";
        return VIE_ERR_ARG;
    }
    const int n[3] = {nx, ny, nz};
    for (int ax = 0; ax < 3; ax++) o.plan[ax] = plans[ax];
    // register four-step kernels for the compile-time lengths (VIE_FAST=0 forces the generic ones)
    const char* fe = std::getenv("VIE_FAST");
    const bool allow_fast = !(fe && fe[0] == '0');
    for (int ax = 0; ax < 3; ax++)
        o.fast[ax] = (allow_fast && fast_length(n[ax]) && tiles.fast[ax] != 0) ? 1 : 0;
    o.xalt = tiles.xalt ? 1 : 0;
    o.zstage = tiles.zstage ? 1 : 0;
    o.wait_test = tiles.wait_test ? 1 : 0;

    // ---- tables: per axis tw[2N], perm[N] (u16), P[2][2N], Q[2][2N], gfold[2N]
    size_t bytes = 0;
    size_t off_tw[3], off_perm[3], off_P[3][2], off_Q[3][2], off_g[3];
    for (int ax = 0; ax < 3; ax++) {
        const size_t L = 2 * (size_t)n[ax];
        off_tw[ax] = bytes; bytes = align_up(bytes + sizeof(C) * L, 256);
        off_perm[ax] = bytes; bytes = align_up(bytes + sizeof(unsigned short) * n[ax], 256);
        for (int md = 0; md < 2; md++) {
            off_P[ax][md] = bytes; bytes = align_up(bytes + sizeof(C) * L, 256);
            off_Q[ax][md] = bytes; bytes = align_up(bytes + sizeof(C) * L, 256);
        }
        off_g[ax] = bytes; bytes = align_up(bytes + sizeof(int) * L, 256);
    }
    std::vector<unsigned char> h(bytes, 0);
    for (int ax = 0; ax < 3; ax++) {
        const int N = n[ax];
        const int L = 2 * N;
        const double delta = d[ax];
        C* tw = reinterpret_cast<C*>(h.data() + off_tw[ax]);
        for (int u = 0; u < L; u++) {
            const long double ang = -2.0L * 3.14159265358979323846264338327950288L * u / (long double)L;
            tw[u] = to_c<C>((double)cosl(ang), (double)sinl(ang));
        }
        std::vector<int> perm = axis_perm(plans[ax]);
        std::vector<int> dr(N);
        for (int m = 0; m < N; m++) dr[perm[m]] = m;
        unsigned short* pp = reinterpret_cast<unsigned short*>(h.data() + off_perm[ax]);
        for (int m = 0; m < N; m++) pp[m] = (unsigned short)perm[m];
        int* gf = reinterpret_cast<int*>(h.data() + off_g[ax]);
        C* Pf = reinterpret_cast<C*>(h.data() + off_P[ax][0]);
        C* Qf = reinterpret_cast<C*>(h.data() + off_Q[ax][0]);
        C* Pc = reinterpret_cast<C*>(h.data() + off_P[ax][1]);
        C* Qc = reinterpret_cast<C*>(h.data() + off_Q[ax][1]);
        for (int slot = 0; slot < L; slot++) {
            int k;
            if (ax == 2) {
                k = slot;  // z spectra are stored in natural order
            } else if (o.fast[ax]) {
                const int hh = slot >= N ? 1 : 0;
                k = 2 * (slot - hh * N) + hh;  // half-natural: slot = h N + m, k = 2m + h
            } else {
                const int hh = slot >= N ? 1 : 0;
                k = 2 * dr[slot - hh * N] + hh;
            }
            gf[slot] = k <= N ? k : L - k;
            // theta = 2 pi k / L, as fft.h:95-99
            const double c = std::cos(2 * kPI * k / (double)L), s = std::sin(2 * kPI * k / (double)L);
            const double dpr = 1.0 - c, dpi = s;   // d+ = 1 - e^{-i theta}
            const double dmr = c - 1.0, dmi = s;   // d- = e^{i theta} - 1
            Pf[slot] = to_c<C>(dpr / delta, dpi / delta);
            Qf[slot] = to_c<C>(dmr, dmi);
            Pc[slot] = to_c<C>(dmr, -dmi);
            Qc[slot] = to_c<C>(dpr / delta, -dpi / delta);
        }
    }
    VIE_CUDA_TRY(cudaMalloc(&d_tables, bytes), err);
    VIE_CUDA_TRY(cudaMemcpy(d_tables, h.data(), bytes, cudaMemcpyHostToDevice), err);
    unsigned char* base = static_cast<unsigned char*>(d_tables);
    for (int ax = 0; ax < 3; ax++) {
        o.ax[ax].tw = reinterpret_cast<const C*>(base + off_tw[ax]);
        o.ax[ax].perm = reinterpret_cast<const unsigned short*>(base + off_perm[ax]);
        for (int md = 0; md < 2; md++) {
            o.ax[ax].P[md] = reinterpret_cast<const C*>(base + off_P[ax][md]);
            o.ax[ax].Q[md] = reinterpret_cast<const C*>(base + off_Q[ax][md]);
        }
        o.ax[ax].gfold = reinterpret_cast<const int*>(base + off_g[ax]);
        o.kappa[ax] = (T)(k0 * k0 * d[ax]);
        o.dcoef[ax] = (T)(-d[ax] * kZ0 / (2.0 * k0));
    }
    const size_t goct = (size_t)(nx + 1) * (ny + 1) * (nz + 1);
    VIE_CUDA_TRY(cudaMalloc(&d_Gs, sizeof(C) * goct), err);
    VIE_CUDA_TRY(cudaMalloc(&d_w, sizeof(C) * (size_t)o.a), err);
    VIE_CUDA_TRY(cudaMemset(d_w, 0, sizeof(C) * (size_t)o.a), err);
    if (owns_scratch) {
        VIE_CUDA_TRY(cudaMalloc(&d_b, sizeof(C) * 3 * (size_t)nx * ny * 2 * nz), err);
        VIE_CUDA_TRY(cudaMalloc(&d_c, sizeof(C) * 3 * (size_t)nx * 2 * ny * 2 * nz), err);
    }
    o.Gs = d_Gs;
    o.w = d_w;
    o.flags = d_flags;
    o.b = d_b;
    o.c = d_c;
    // status word of the bounded waits, and the TMA view of b for the forward y pass
    if (!h_status) {
        VIE_CUDA_TRY(cudaHostAlloc(&h_status, 2 * sizeof(int), cudaHostAllocMapped), err);
        h_status[0] = h_status[1] = 0;
        VIE_CUDA_TRY(cudaHostGetDevicePointer(&d_status, h_status, 0), err);
    }
    o.status = d_status;
    use_ytma = tm_b_ok = tm_c_ok = false;
    tm_b_addr = tm_c_addr = nullptr;
    if (o.fast[1] && tiles.ytma && d_b && d_c && ny <= 256) {
        if (EncodeTiledFn enc = encode_tiled()) {
            constexpr int TPY = FastTiles<C>::TP_Y;
            const cuuint64_t dims[2] = {(cuuint64_t)4 * nz, (cuuint64_t)3 * nx * ny};  // reals, rows
            const cuuint64_t strides[1] = {(cuuint64_t)4 * nz * sizeof(T)};             // bytes per row
            const cuuint32_t box[2] = {(cuuint32_t)2 * TPY, (cuuint32_t)ny};
            const cuuint32_t estr[2] = {1, 1};
            const CUresult r = enc(&tm_b, sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                                   2, d_b, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            tm_b_ok = r == CUDA_SUCCESS;
            tm_b_addr = d_b;
            // c: 2 Lz reals x 3 nx 2ny rows, boxes of ny rows (one half of a y line)
            const cuuint64_t dims_c[2] = {(cuuint64_t)4 * nz, (cuuint64_t)6 * nx * ny};
            const CUresult rc2 = enc(&tm_c, sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                                     2, d_c, dims_c, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            tm_c_ok = rc2 == CUDA_SUCCESS;
            tm_c_addr = d_c;
            use_ytma = tm_b_ok && tm_c_ok;
        }
    }
    ready = true;
    return VIE_OK;
}

template <typename T> size_t Operator<T>::scratch_bytes() const {
    const size_t nx = dev.nx, ny = dev.ny, nz = dev.nz;
    return sizeof(C) * 3 * (nx * ny * 2 * nz + nx * 2 * ny * 2 * nz);
}

template <typename C>
__global__ void k_scale_green(const double2* __restrict__ oct, C* __restrict__ out, size_t n, double sr,
                              double si) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double2 g = oct[i];
        out[i] = from_d2<C>(make_double2(sr * g.x - si * g.y, sr * g.y + si * g.x));
    }
}

template <typename T>
int Operator<T>::set_green(const double2* d_oct64, double k0, cudaStream_t st, Error& err) {
    const size_t goct = (size_t)(dev.nx + 1) * (dev.ny + 1) * (dev.nz + 1);
    const double M = 8.0 * (double)dev.nx * dev.ny * dev.nz;
    // c = i Z0 / (k0 M): the 1/M and i Z0/k0 factors of V5/V6 (fft.h:76-77, 256)
    k_scale_green<C><<<592, 256, 0, st>>>(d_oct64, d_Gs, goct, 0.0, kZ0 / (k0 * M));
    count_launch();
    VIE_CUDA_TRY(cudaGetLastError(), err);
    return VIE_OK;
}

template <typename T>
int Operator<T>::set_contrast(const double* w_host, cudaStream_t st, Error& err) {
    const size_t a = (size_t)dev.a;
    std::vector<C> hw(a);
    for (size_t i = 0; i < a; i++) hw[i] = to_c<C>(w_host[2 * i], w_host[2 * i + 1]);
    VIE_CUDA_TRY(cudaMemcpyAsync(d_w, hw.data(), sizeof(C) * a, cudaMemcpyHostToDevice, st), err);
    VIE_CUDA_TRY(cudaStreamSynchronize(st), err);
    return VIE_OK;
}

template <typename T> void Operator<T>::release() {
    if (d_tables) cudaFree(d_tables);
    if (d_Gs) cudaFree(d_Gs);
    if (d_w) cudaFree(d_w);
    if (owns_scratch) {
        if (d_b) cudaFree(d_b);
        if (d_c) cudaFree(d_c);
    }
    if (h_status) cudaFreeHost(h_status);
    d_tables = nullptr; d_Gs = nullptr; d_w = nullptr; d_b = nullptr; d_c = nullptr;
    h_status = d_status = nullptr;
    dev.status = nullptr;
    use_ytma = tm_b_ok = tm_c_ok = false;
    ready = false;
}

template <typename T>
int Operator<T>::apply(const C* x, C* y, bool conj, cudaStream_t st, Error& err) {
    ProCopy<C> pro{x, dev.a};
    EpiStore<C> epi{y, dev.a};
    return launch_operator<T>(*this, pro, epi, x, conj, nullptr, st, err);
}

template struct Operator<float>;
template struct Operator<double>;

}  // namespace vie
