// vie_post.cu -- post-processing of the solution on the GPU: the radiated
// far field of the current (FarField1's forward scattering, NearFar.h:16-109;
// FarField2's E- and H-plane RCS, NearFar.h:302-477) and NearField's
// absorption sums (NearFar.h:186-250), without copying the field to the host.
//
// Far field: for a direction v the reference sums, per component c,
//     S_c(v) = sum_{i,j,k} exp(i k0 (x_i vx + y_j vy + z_k vz)) J_c[i,j,k],
//     x_i = (i + 1/2) dx, ...
// The phase factors per axis, so k_radiation computes for one (i, j) row
//     T_c(v) = sum_k ez_v(k) J_c[i,j,k]   and adds ex_v(i) ey_v(j) T_c(v).
// A block stages rows of J (three components) in shared memory once and
// reuses them for up to 256 directions, one direction per thread; the phase
// tables are [axis index][direction] so a warp reads them coalesced.  The
// block partials are summed in a fixed order (deterministic).
#include <cmath>
#include <vector>

#include "vie_internal.h"

namespace vie {

namespace {

constexpr int kRowsPerStage = 2;     // (i, j) rows staged per step
constexpr int kPostBlocks = 148 * 2;

// ez[k * M + d] = exp(i k0 (k + 1/2) dz vz_d), likewise ex, ey
__global__ void k_phase_tables(const double3* __restrict__ dirs, int M, int nx, int ny, int nz, double3 kd,
                               double2* __restrict__ ex, double2* __restrict__ ey, double2* __restrict__ ez) {
    const int total = M * (nx + ny + nz);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const int d = t % M, q = t / M;
        double ph;
        double2* out;
        if (q < nx) {
            ph = kd.x * (q + 0.5) * dirs[d].x;
            out = ex + q * M + d;
        } else if (q < nx + ny) {
            ph = kd.y * (q - nx + 0.5) * dirs[d].y;
            out = ey + (q - nx) * M + d;
        } else {
            ph = kd.z * (q - nx - ny + 0.5) * dirs[d].z;
            out = ez + (q - nx - ny) * M + d;
        }
        double s, c;
        sincos(ph, &s, &c);
        *out = make_double2(c, s);
    }
}

__device__ __forceinline__ void cmac(double2& acc, double2 a, double2 b) {
    acc.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x));
    acc.y = fma(a.x, b.y, fma(a.y, b.x, acc.y));
}
__device__ __forceinline__ double2 cmul2(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// partial[(blockIdx.x * M + d) * 3 + c] = this block's share of S_c(v_d)
__global__ void __launch_bounds__(256) k_radiation(const double2* __restrict__ J, int nx, int ny, int nz, int M,
                                                   const double2* __restrict__ ex, const double2* __restrict__ ey,
                                                   const double2* __restrict__ ez, double2* __restrict__ partial) {
    extern __shared__ double2 rowbuf[];  // [kRowsPerStage][3][nz]
    const long long a = (long long)nx * ny * nz;
    const int nrows = nx * ny;
    const int d = blockIdx.y * blockDim.x + threadIdx.x;
    const bool live = d < M;
    double2 acc[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
    for (int r0 = blockIdx.x * kRowsPerStage; r0 < nrows; r0 += gridDim.x * kRowsPerStage) {
        const int nr = min(kRowsPerStage, nrows - r0);
        __syncthreads();
        for (int u = threadIdx.x; u < nr * 3 * nz; u += blockDim.x) {
            const int rr = u / (3 * nz), rem = u - rr * 3 * nz, c = rem / nz, k = rem - c * nz;
            rowbuf[u] = J[c * a + (long long)(r0 + rr) * nz + k];
        }
        __syncthreads();
        if (!live) continue;
        for (int rr = 0; rr < nr; rr++) {
            const int row = r0 + rr, i = row / ny, j = row - i * ny;
            double2 t[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
            const double2* src = rowbuf + rr * 3 * nz;
            for (int k = 0; k < nz; k++) {
                const double2 e = ez[k * M + d];
                cmac(t[0], e, src[k]);
                cmac(t[1], e, src[nz + k]);
                cmac(t[2], e, src[2 * nz + k]);
            }
            const double2 exy = cmul2(ex[i * M + d], ey[j * M + d]);
#pragma unroll
            for (int c = 0; c < 3; c++) cmac(acc[c], exy, t[c]);
        }
    }
    if (live)
        for (int c = 0; c < 3; c++) partial[((long long)blockIdx.x * M + d) * 3 + c] = acc[c];
}

__global__ void k_radiation_sum(const double2* __restrict__ partial, int nblk, int M, double2* __restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * M) return;
    double sx = 0.0, sy = 0.0;
    for (int b = 0; b < nblk; b++) {
        const double2 v = partial[(long long)b * 3 * M + t];
        sx += v.x;
        sy += v.y;
    }
    out[t] = make_double2(sx, sy);
}

// NearField sums over edges with i, j, k < N - 1 (NearFar.h:186-250):
// part[b * 3 + 0] Ene_Metal, + 1 Ene_Active, + 2 Absorb_Volume
__global__ void __launch_bounds__(256) k_nearfield(const double2* __restrict__ J, const double2* __restrict__ w,
                                                   const unsigned char* __restrict__ mat, int nx, int ny, int nz,
                                                   double k0, double dvol, double* __restrict__ part) {
    const long long a = (long long)nx * ny * nz;
    const long long step[3] = {(long long)ny * nz, (long long)nz, 1LL};
    double em = 0.0, ea = 0.0, av = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 3 * a; t += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(t / a);
        const long long v = t - c * a;
        const int i = (int)(v / step[0]), j = (int)((v / nz) % ny), k = (int)(v % nz);
        if (i >= nx - 1 || j >= ny - 1 || k >= nz - 1) continue;
        const long long vb = v + step[c];
        const int m2 = mat[vb], m3 = mat[v];
        const bool metal = m2 == 2 && m3 == 2, active = m2 == 3 && m3 == 3;
        if (!metal && !active) continue;
        // V2 = 1/(eps_b - 1) + 1/(eps_a - 1); V1 = V2 (-i Z0/(2 k0)); V4 = 2/V2 + 1
        const double2 V2 = make_double2(w[vb].x + w[v].x, w[vb].y + w[v].y);
        const double h = 0.5 * kZ0 / k0;
        const double2 V1 = make_double2(V2.y * h, -V2.x * h);
        const double den = V2.x * V2.x + V2.y * V2.y;
        const double imV4 = -2.0 * V2.y / den;  // Im(2 / V2)
        const double2 jv = J[t];
        const double absE2 = (jv.x * jv.x + jv.y * jv.y) * (V1.x * V1.x + V1.y * V1.y);
        const double contrib = k0 / kZ0 * (-imV4) * absE2 * dvol;
        if (metal) em += contrib;
        if (active) {
            ea += contrib;
            av += dvol;
        }
    }
    __shared__ double red[3][256];
    red[0][threadIdx.x] = em;
    red[1][threadIdx.x] = ea;
    red[2][threadIdx.x] = av;
    __syncthreads();
    for (int hh = 128; hh > 0; hh >>= 1) {
        if (threadIdx.x < hh)
            for (int q = 0; q < 3; q++) red[q][threadIdx.x] += red[q][threadIdx.x + hh];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < 3; q++) part[blockIdx.x * 3 + q] = red[q][0];
}

// S_c(v) for M directions of the current solution (3M complex, host)
int radiation_sums(vie_ctx* ctx, const std::vector<double3>& dirs, std::vector<double2>& out) {
    const int M = (int)dirs.size();
    const int nx = ctx->nx, ny = ctx->ny, nz = ctx->nz;
    cudaStream_t st = ctx->stream;
    const size_t smem = sizeof(double2) * kRowsPerStage * 3 * (size_t)nz;
    if (smem > 200 * 1024) return ctx->set_error(VIE_ERR_ARG, "z axis too long for the far-field kernel");
    const int threads = 256;
    const int dchunks = (M + threads - 1) / threads;
    const int nblk = kPostBlocks;
    double3* d_dirs = nullptr;
    double2 *ex = nullptr, *ey = nullptr, *ez = nullptr, *part = nullptr, *sum = nullptr;
    const size_t ntab = (size_t)M * (nx + ny + nz);
    auto release = [&]() {
        cudaFree(d_dirs);
        cudaFree(ex);
        cudaFree(part);
        cudaFree(sum);
    };
    if (cudaMalloc(&d_dirs, sizeof(double3) * M) != cudaSuccess || cudaMalloc(&ex, sizeof(double2) * ntab) != cudaSuccess ||
        cudaMalloc(&part, sizeof(double2) * 3 * (size_t)M * nblk) != cudaSuccess ||
        cudaMalloc(&sum, sizeof(double2) * 3 * (size_t)M) != cudaSuccess) {
        release();
        return ctx->set_error(VIE_ERR_ALLOC, "far-field buffers");
    }
    ey = ex + (size_t)M * nx;
    ez = ey + (size_t)M * ny;
    cudaError_t e = cudaMemcpyAsync(d_dirs, dirs.data(), sizeof(double3) * M, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        const double3 kd = make_double3(ctx->k0 * ctx->d[0], ctx->k0 * ctx->d[1], ctx->k0 * ctx->d[2]);
        k_phase_tables<<<kPostBlocks, 256, 0, st>>>(d_dirs, M, nx, ny, nz, kd, ex, ey, ez);
        count_launch();
        if (smem > 48 * 1024) e = cudaFuncSetAttribute(k_radiation, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    }
    if (e == cudaSuccess) {
        k_radiation<<<dim3(nblk, dchunks), threads, smem, st>>>(ctx->d_x, nx, ny, nz, M, ex, ey, ez, part);
        count_launch();
        k_radiation_sum<<<(3 * M + 255) / 256, 256, 0, st>>>(part, nblk, M, sum);
        count_launch();
        e = cudaGetLastError();
    }
    out.assign(3 * (size_t)M, make_double2(0, 0));
    if (e == cudaSuccess) e = cudaMemcpyAsync(out.data(), sum, sizeof(double2) * 3 * M, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    release();
    if (e != cudaSuccess) return ctx->set_error(VIE_ERR_CUDA, cudaGetErrorString(e));
    return VIE_OK;
}

double3 direction(double theta_deg, double phi_deg) {
    const double th = kPI * theta_deg / 180.0, ph = kPI * phi_deg / 180.0;
    return make_double3(std::sin(th) * std::cos(ph), std::sin(th) * std::sin(ph), std::cos(th));
}

// the projection factor exp(i k0 delta/2 v) and the cell volume (NearFar.h:88-99)
void project(vie_ctx* ctx, const double3& v, double2* S) {
    const double vol = ctx->d[0] * ctx->d[1] * ctx->d[2];
    const double ph[3] = {ctx->k0 * 0.5 * ctx->d[0] * v.x, ctx->k0 * 0.5 * ctx->d[1] * v.y,
                          ctx->k0 * 0.5 * ctx->d[2] * v.z};
    for (int c = 0; c < 3; c++) {
        const double cr = std::cos(ph[c]), ci = std::sin(ph[c]);
        S[c] = make_double2((cr * S[c].x - ci * S[c].y) * vol, (cr * S[c].y + ci * S[c].x) * vol);
    }
}

}  // namespace

// FarField1 (NearFar.h:16-109): Forward_RCS in the incident direction
int farfield1_driver(vie_ctx* ctx, double theta, double phi, double psi, double* fwd) {
    std::vector<double2> S;
    const double3 v = direction(theta, phi);
    int rc = radiation_sums(ctx, {v}, S);
    if (rc) return rc;
    project(ctx, v, S.data());
    const double th = kPI * theta / 180.0, ph = kPI * phi / 180.0;
    const double v1 = std::cos(th), v2 = std::sin(th), v3 = std::cos(ph), v4 = std::sin(ph);
    const double tm = kZ0 * (S[0].x * v1 * v3 + S[1].x * v1 * v4 - S[2].x * v2);
    const double te = kZ0 * (S[0].x * v4 - S[1].x * v3);
    *fwd = std::cos(kPI * psi / 180.0) * tm - std::sin(kPI * psi / 180.0) * te;
    return VIE_OK;
}

// FarField2 (NearFar.h:302-477): E plane (phi) and H plane (phi + 90), theta 0..180, dB
int farfield2_driver(vie_ctx* ctx, double phi, double* rcs_theta, double* rcs_phi) {
    std::vector<double3> dirs;
    for (int plane = 0; plane < 2; plane++)
        for (int ang = 0; ang <= 180; ang++) dirs.push_back(direction((double)ang, plane ? phi + 90.0 : phi));
    std::vector<double2> S;
    int rc = radiation_sums(ctx, dirs, S);
    if (rc) return rc;
    const double k0 = ctx->k0, norm = (2 * kPI / k0) * (2 * kPI / k0);
    for (int plane = 0; plane < 2; plane++) {
        const double pd = plane ? phi + 90.0 : phi;
        const double v3 = std::cos(kPI * pd / 180.0), v4 = std::sin(kPI * pd / 180.0);
        for (int ang = 0; ang <= 180; ang++) {
            const int m = plane * 181 + ang;
            double2* s = S.data() + 3 * (size_t)m;
            project(ctx, dirs[m], s);
            const double v1 = std::cos(kPI * ang / 180.0), v2 = std::sin(kPI * ang / 180.0);
            double m1, m2;
            if (!plane) {
                m1 = s[0].x * v1 * v3 + s[1].x * v1 * v4 - s[2].x * v2;
                m2 = s[0].y * v1 * v3 + s[1].y * v1 * v4 - s[2].y * v2;
            } else {
                m1 = s[0].x * v4 - s[1].x * v3;
                m2 = s[0].y * v4 - s[1].y * v3;
            }
            const double rcs = k0 * k0 * kZ0 * kZ0 * (m1 * m1 + m2 * m2) / (4.0 * kPI);
            (plane ? rcs_phi : rcs_theta)[ang] = 10.0 * std::log10(rcs / norm);
        }
    }
    return VIE_OK;
}

// NearField (NearFar.h:186-250): Ene_Metal, Ene_Active, Absorb_Volume
int nearfield_driver(vie_ctx* ctx, const unsigned char* material, double* out3) {
    cudaStream_t st = ctx->stream;
    unsigned char* d_mat = nullptr;
    double* d_part = nullptr;
    if (cudaMalloc(&d_mat, (size_t)ctx->a) != cudaSuccess ||
        cudaMalloc(&d_part, sizeof(double) * 3 * kPostBlocks) != cudaSuccess) {
        cudaFree(d_mat);
        return ctx->set_error(VIE_ERR_ALLOC, "near-field buffers");
    }
    std::vector<double> part(3 * kPostBlocks);
    cudaError_t e = cudaMemcpyAsync(d_mat, material, (size_t)ctx->a, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        k_nearfield<<<kPostBlocks, 256, 0, st>>>(ctx->d_x, ctx->op64.dev.w, d_mat, ctx->nx, ctx->ny, ctx->nz, ctx->k0,
                                                 ctx->d[0] * ctx->d[1] * ctx->d[2], d_part);
        count_launch();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(part.data(), d_part, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d_mat);
    cudaFree(d_part);
    if (e != cudaSuccess) return ctx->set_error(VIE_ERR_CUDA, cudaGetErrorString(e));
    out3[0] = out3[1] = out3[2] = 0.0;
    for (int b = 0; b < kPostBlocks; b++)
        for (int q = 0; q < 3; q++) out3[q] += part[3 * b + q];
    return VIE_OK;
}

}  // namespace vie
