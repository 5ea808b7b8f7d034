// vie_green.cu -- Green's-function spectrum and incident field on the GPU (FP64).
//
// Green_Function_Compute (GreenFunction.h:8-141) evaluates the scalar Green's
// function on offsets [0..nx] x [0..ny] x [0..nz], extends it evenly to the
// (2nx, 2ny, 2nz) circulant (index i >= n maps to 2n - i, :92-129) and takes
// an unnormalised forward FFT (:131-139).  For an even-extended sequence that
// FFT is separable into one DCT-I per axis on the octant:
//   Gt(k) = G(0) + (-1)^k G(N) + 2 sum_{n=1}^{N-1} G(n) cos(pi k n / N),
// so the spectrum is computed directly on the (nx+1)(ny+1)(nz+1) octant that
// the operator reads, in FP64, with exactly reduced cosine arguments.
#include <cmath>

#include "vie_internal.h"

namespace vie {

// spatial octant, GreenFunction.h:53-88
__global__ void k_green_spatial(double2* __restrict__ g, int nx, int ny, int nz, double dx, double dy, double dz,
                                double k0, double amp, double2 self) {
    const long long n = (long long)(nx + 1) * (ny + 1) * (nz + 1);
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n;
         v += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(v % (nz + 1));
        const long long r1 = v / (nz + 1);
        const int j = (int)(r1 % (ny + 1));
        const int i = (int)(r1 / (ny + 1));
        if (i + j + k == 0) {
            g[v] = self;
        } else {
            const double x = i * dx, y = j * dy, z = k * dz;
            const double r = sqrt(x * x + y * y + z * z);
            double s, c;
            sincos(-k0 * r, &s, &c);
            // exp(-i k0 r) (sin p / p - cos p) / (pi k0^2 D^2 r / 3) * dV
            const double f = amp / r;
            g[v] = make_double2(c * f, s * f);
        }
    }
}

// One DCT-I along an axis of an array viewed as [outer][len][inner], in place.
// A block owns W columns of one outer index (all len entries), so blocks
// never touch each other's data.  cosT[u] = cos(pi u / (len-1)), u < 2(len-1).
constexpr int kDctW = 16;
constexpr int kDctKB = 4;

__global__ void __launch_bounds__(256) k_dct1_axis(double2* __restrict__ g, int len, long long inner,
                                                   long long outer, const double* __restrict__ cosT) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* tile = reinterpret_cast<double2*>(smem_raw);  // [len][W]
    const int N = len - 1;
    const int twoN = 2 * N;
    const bool rows = inner == 1;  // transform along the contiguous axis
    // column block decomposition
    const long long ncolblk = rows ? (outer + kDctW - 1) / kDctW : outer * ((inner + kDctW - 1) / kDctW);
    for (long long cb = blockIdx.x; cb < ncolblk; cb += gridDim.x) {
        long long o0, in0;
        int W;
        if (rows) {
            o0 = cb * kDctW;
            in0 = 0;
            W = (int)min((long long)kDctW, outer - o0);
        } else {
            const long long nib = (inner + kDctW - 1) / kDctW;
            o0 = cb / nib;
            in0 = (cb % nib) * kDctW;
            W = (int)min((long long)kDctW, inner - in0);
        }
        // element (n, w) address
        auto addr = [&](int n, int w) -> long long {
            return rows ? (o0 + w) * (long long)len + n : (o0 * len + n) * inner + in0 + w;
        };
        __syncthreads();
        for (int e = threadIdx.x; e < len * kDctW; e += blockDim.x) {
            int n, w;
            if (rows) { w = e / len; n = e % len; } else { w = e % kDctW; n = e / kDctW; }
            double2 v = make_double2(0, 0);
            if (w < W) v = g[addr(n, w)];
            tile[n * kDctW + w] = v;
        }
        __syncthreads();
        const int nkb = (len + kDctKB - 1) / kDctKB;
        for (int e = threadIdx.x; e < nkb * kDctW; e += blockDim.x) {
            const int w = e % kDctW, kb = e / kDctW;
            double2 acc[kDctKB];
            int kk[kDctKB];
#pragma unroll
            for (int q = 0; q < kDctKB; q++) { acc[q] = make_double2(0, 0); kk[q] = kb * kDctKB + q; }
            for (int n = 0; n <= N; n++) {
                const double2 v = tile[n * kDctW + w];
                const double wn = (n == 0 || n == N) ? 1.0 : 2.0;
#pragma unroll
                for (int q = 0; q < kDctKB; q++) {
                    const int u = (int)(((long long)kk[q] * n) % twoN);
                    const double c = wn * cosT[u];
                    acc[q].x = fma(c, v.x, acc[q].x);
                    acc[q].y = fma(c, v.y, acc[q].y);
                }
            }
            if (w < W) {
#pragma unroll
                for (int q = 0; q < kDctKB; q++)
                    if (kk[q] <= N) g[addr(kk[q], w)] = acc[q];
            }
        }
    }
}

// natural-order (2nx, 2ny, 2nz) spectrum from the octant
__global__ void k_green_expand(const double2* __restrict__ oct, double2* __restrict__ out, int nx, int ny, int nz) {
    const long long Lx = 2 * nx, Ly = 2 * ny, Lz = 2 * nz;
    const long long n = Lx * Ly * Lz;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n;
         v += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(v % Lz);
        const long long r1 = v / Lz;
        const int j = (int)(r1 % Ly);
        const int i = (int)(r1 / Ly);
        const int fi = i <= nx ? i : (int)Lx - i, fj = j <= ny ? j : (int)Ly - j, fk = k <= nz ? k : (int)Lz - k;
        out[v] = oct[((long long)fi * (ny + 1) + fj) * (nz + 1) + fk];
    }
}

// Incident_Wave (GreenFunction.h:144-248): edge-integrated plane wave on the
// three staggered grids.
__global__ void k_incident(double2* __restrict__ e, int nx, int ny, int nz, double dx, double dy, double dz, double kx,
                           double ky, double kz, double px, double py, double pz, double eps_small) {
    const long long a = (long long)nx * ny * nz;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < a;
         v += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(v % nz);
        const long long r1 = v / nz;
        const int j = (int)(r1 % ny);
        const int i = (int)(r1 / ny);
        const double kk[3] = {kx, ky, kz};
        const double dd[3] = {dx, dy, dz};
        const double pol[3] = {px, py, pz};
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const double xm = (i + (c == 0 ? 1.0 : 0.5)) * dx;
            const double ym = (j + (c == 1 ? 1.0 : 0.5)) * dy;
            const double zm = (k + (c == 2 ? 1.0 : 0.5)) * dz;
            double s, co;
            sincos(-(kx * xm + ky * ym + kz * zm), &s, &co);
            // (exp(-i k d/2) - exp(i k d/2)) / (-i k) = 2 sin(k d / 2) / k; d when |k| < EPS (:187-193)
            const double len = fabs(kk[c]) < eps_small ? dd[c] : 2.0 * sin(kk[c] * dd[c] / 2.0) / kk[c];
            e[c * a + v] = make_double2(co * len * pol[c], s * len * pol[c]);
        }
    }
}

int green_compute(vie_ctx* ctx) {
    Error& err = ctx->err;
    const int nx = ctx->nx, ny = ctx->ny, nz = ctx->nz;
    const double dx = ctx->d[0], dy = ctx->d[1], dz = ctx->d[2], k0 = ctx->k0;
    const long long goct = (long long)(nx + 1) * (ny + 1) * (nz + 1);
    if (!ctx->d_green) VIE_CUDA_TRY(cudaMalloc(&ctx->d_green, sizeof(double2) * goct), err);
    const double dV = dx * dy * dz;                                   // :23
    const double D = 2 * std::pow(dV / (4.0 / 3.0 * kPI), 1.0 / 3.0);  // :24
    const double p = 0.5 * k0 * D;                                    // :25
    // sinh(-ip)/(-ip) - cosh(-ip) = sin(p)/p - cos(p)
    const double shape = std::sin(p) / p - std::cos(p);
    const double amp = shape / (1.0 / 3.0 * kPI * k0 * k0 * std::pow(D, 2.0)) * dV;
    // ((1 + i p) e^{-i p} - 1) / (pi k0^2 D^3 / 6) * dV   (:77-84)
    const double den = 1.0 / 6.0 * kPI * k0 * k0 * std::pow(D, 3.0);
    const double sr = (std::cos(p) + p * std::sin(p)) - 1.0;  // Re((1+ip)(cos p - i sin p)) - 1
    const double si = p * std::cos(p) - std::sin(p);          // Im((1+ip)(cos p - i sin p))
    const double2 self = make_double2(sr / den * dV, si / den * dV);
    k_green_spatial<<<1184, 256, 0, ctx->stream>>>(ctx->d_green, nx, ny, nz, dx, dy, dz, k0, amp, self);
    count_launch();
    VIE_CUDA_TRY(cudaGetLastError(), err);
    const int n3[3] = {nx, ny, nz};
    const long long E[3] = {nx + 1, ny + 1, nz + 1};
    int maxN = std::max(nx, std::max(ny, nz));
    double* d_cos = nullptr;
    VIE_CUDA_TRY(cudaMalloc(&d_cos, sizeof(double) * 2 * maxN * 3), err);
    std::vector<double> hc(2 * (size_t)maxN * 3, 0.0);
    for (int ax = 0; ax < 3; ax++)
        for (int u = 0; u < 2 * n3[ax]; u++)
            hc[ax * 2 * maxN + u] =
                (double)cosl(3.14159265358979323846264338327950288L * u / (long double)n3[ax]);
    VIE_CUDA_TRY(cudaMemcpyAsync(d_cos, hc.data(), sizeof(double) * hc.size(), cudaMemcpyHostToDevice, ctx->stream),
                 err);
    for (int ax = 2; ax >= 0; ax--) {
        const long long len = E[ax];
        long long inner = 1, outer = 1;
        for (int b = ax + 1; b < 3; b++) inner *= E[b];
        for (int b = 0; b < ax; b++) outer *= E[b];
        const size_t smem = sizeof(double2) * (size_t)len * kDctW;
        if (smem > 227 * 1024) {
            cudaFree(d_cos);
            err.code = VIE_ERR_ARG;
            err.msg = "grid axis too long for the Green's-function transform";
            return VIE_ERR_ARG;
        }
        VIE_CUDA_TRY(cudaFuncSetAttribute(k_dct1_axis, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), err);
        k_dct1_axis<<<148 * 8, 256, smem, ctx->stream>>>(ctx->d_green, (int)len, inner, outer, d_cos + ax * 2 * maxN);
        count_launch();
        VIE_CUDA_TRY(cudaGetLastError(), err);
    }
    VIE_CUDA_TRY(cudaStreamSynchronize(ctx->stream), err);
    cudaFree(d_cos);
    return VIE_OK;
}

int green_expand(vie_ctx* ctx, double2* d_out) {
    k_green_expand<<<1184, 256, 0, ctx->stream>>>(ctx->d_green, d_out, ctx->nx, ctx->ny, ctx->nz);
    count_launch();
    VIE_CUDA_TRY(cudaGetLastError(), ctx->err);
    return VIE_OK;
}

int incident_compute(vie_ctx* ctx, double theta, double phi, double psi, double2* d_e) {
    const double th = kPI * theta / 180.0, ph = kPI * phi / 180.0, ps = kPI * psi / 180.0;
    const double kx = ctx->k0 * std::sin(th) * std::cos(ph);  // :162-164
    const double ky = ctx->k0 * std::sin(th) * std::sin(ph);
    const double kz = ctx->k0 * std::cos(th);
    const double px = std::cos(th) * std::cos(ph) * std::cos(ps) - std::sin(ph) * std::sin(ps);  // :196-199
    const double py = std::cos(th) * std::sin(ph) * std::cos(ps) + std::cos(ph) * std::sin(ps);  // :219-222
    const double pz = -std::sin(th) * std::cos(ps);                                              // :243-244
    k_incident<<<1184, 256, 0, ctx->stream>>>(d_e, ctx->nx, ctx->ny, ctx->nz, ctx->d[0], ctx->d[1], ctx->d[2], kx, ky,
                                              kz, px, py, pz, 1.0e-7);
    count_launch();
    VIE_CUDA_TRY(cudaGetLastError(), ctx->err);
    return VIE_OK;
}

}  // namespace vie
