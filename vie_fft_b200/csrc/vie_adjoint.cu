// vie_adjoint.cu -- absorbed power in a set of edges and its gradient with
// respect to the per-voxel complex permittivity (adjoint method).
//
// Objective: the absorption sum of NearField (NearFar.h:186-250) over a caller
// chosen set of edges E (for Ene_Active: edges whose two voxels both hold the
// active material, i, j, k < N - 1):
//     P = sum_{e in E} k0/Z0 Im(-V4_e) |V1_e J_e|^2 dV,
//     V2 = w_a + w_b, V1 = -i Z0/(2 k0) V2, V4 = 2/V2 + 1, w = 1/(eps - 1),
// which is exactly  P = sum_{e in E} C0 Im(w_a + w_b) |J_e|^2,  C0 = Z0 dV / (2 k0).
//
// J solves A(w) J = b.  With g_e = C0 Im(V2_e) J_e (e in E), dP through J is
// -2 Re(lambda^H dA J), A^H lambda = g.  The operator is complex-symmetric for
// cubic voxels (A^T = A), so lambda = conj(mu) with A mu = conj(g): the
// adjoint solve reuses the forward operator and driver with the conjugated
// source.  A depends on w only through its diagonal term, i dcoef_f (w_a + w_b)
// on the flagged edge e = (a, b) (fft.h:419-433), so per voxel v
//     S_v = sum_{flagged e touching v} mu_e i dcoef_f J_e
//     R_v = sum_{e in E touching v} C0 |J_e|^2
//     dP/dRe eps_v + i dP/dIm eps_v = conj( w_v^2 (2 S_v + i R_v) )
// (dw/deps = -w^2; the first term is the implicit part, the second the
// explicit Im(w) of the objective).  Only the two converged fields J and mu
// are kept; no Krylov history is stored.
#include <cmath>
#include <vector>

#include "vie_internal.h"

namespace vie {

int solve_driver(vie_ctx* ctx, const vie_solve_params* prm, vie_solve_info* info);

namespace {

constexpr int kAdjBlocks = 148 * 4;

struct EdgeGeom {
    int nx, ny, nz;
    long long a;
    long long step[3];  // voxel-index stride of each axis
};

__device__ __forceinline__ bool edge_valid(const EdgeGeom& g, long long v, int f) {
    // the edge (v, f) has its second voxel inside the grid
    const int i = (int)(v / ((long long)g.ny * g.nz));
    const int j = (int)((v / g.nz) % g.ny);
    const int k = (int)(v % g.nz);
    return f == 0 ? i < g.nx - 1 : (f == 1 ? j < g.ny - 1 : k < g.nz - 1);
}

// P partials and the adjoint source src_e = conj(g_e) = C0 Im(V2_e) conj(J_e) on E
__global__ void __launch_bounds__(256) k_power_source(const double2* __restrict__ J, const double2* __restrict__ w,
                                                      const unsigned char* __restrict__ mask, EdgeGeom g, double c0,
                                                      double2* __restrict__ src, double* __restrict__ partial) {
    double acc = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 3 * g.a;
         t += (long long)gridDim.x * blockDim.x) {
        const int f = (int)(t / g.a);
        const long long v = t - f * g.a;
        double2 s = make_double2(0.0, 0.0);
        if (((mask[v] >> f) & 1) && edge_valid(g, v, f)) {
            const double q = c0 * (w[v].y + w[v + g.step[f]].y);
            const double2 j = J[t];
            acc += q * (j.x * j.x + j.y * j.y);
            s = make_double2(q * j.x, -q * j.y);
        }
        src[t] = s;
    }
    __shared__ double red[256];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

__global__ void k_sum_partials(const double* __restrict__ partial, int n, double* __restrict__ out) {
    __shared__ double red[256];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += partial[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

// gradient per voxel from the forward field J and the adjoint field mu
__global__ void __launch_bounds__(256) k_adjoint_grad(const double2* __restrict__ J, const double2* __restrict__ mu,
                                                      const double2* __restrict__ w,
                                                      const unsigned char* __restrict__ flags,
                                                      const unsigned char* __restrict__ mask, EdgeGeom g, double c0,
                                                      double3 dcoef, double2* __restrict__ grad) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < g.a;
         v += (long long)gridDim.x * blockDim.x) {
        double sx = 0.0, sy = 0.0, r = 0.0;
#pragma unroll
        for (int f = 0; f < 3; f++) {
            const double dc = f == 0 ? dcoef.x : (f == 1 ? dcoef.y : dcoef.z);
            // the edge (v, f) and the edge (v - e_f, f) both touch voxel v
#pragma unroll
            for (int side = 0; side < 2; side++) {
                long long e = v;
                if (side == 1) {
                    const bool has = f == 0 ? v >= g.step[0] : (f == 1 ? ((v / g.nz) % g.ny) > 0 : (v % g.nz) > 0);
                    if (!has) continue;
                    e = v - g.step[f];
                }
                if (!edge_valid(g, e, f)) continue;
                const double2 j = J[f * g.a + e];
                if ((flags[e] >> f) & 1) {
                    // mu_e * (i dc) * J_e
                    const double2 m = mu[f * g.a + e];
                    const double pr = m.x * j.x - m.y * j.y, pi = m.x * j.y + m.y * j.x;
                    sx += -dc * pi;
                    sy += dc * pr;
                }
                if ((mask[e] >> f) & 1) r += c0 * (j.x * j.x + j.y * j.y);
            }
        }
        // conj( w^2 (2 S + i R) )
        const double2 wv = w[v];
        const double w2x = wv.x * wv.x - wv.y * wv.y, w2y = 2.0 * wv.x * wv.y;
        const double tx = 2.0 * sx, ty = 2.0 * sy + r;
        grad[v] = make_double2(w2x * tx - w2y * ty, -(w2x * ty + w2y * tx));
    }
}

}  // namespace

// see include/vie_b200.h (vie_power_grad)
int power_grad_driver(vie_ctx* ctx, const unsigned char* edge_mask, const vie_solve_params* prm, double* power,
                      double* grad, vie_solve_info* info_fwd, vie_solve_info* info_adj) {
    const long long a = ctx->a, n3 = 3 * a;
    cudaStream_t st = ctx->stream;
    EdgeGeom g{ctx->nx, ctx->ny, ctx->nz, a, {(long long)ctx->ny * ctx->nz, (long long)ctx->nz, 1LL}};
    const double c0 = kZ0 * ctx->d[0] * ctx->d[1] * ctx->d[2] / (2.0 * ctx->k0);
    // device buffers: mask, saved incident field, saved forward field, partials, P, gradient
    unsigned char* d_mask = nullptr;
    double2 *d_rhs_bak = nullptr, *d_J = nullptr, *d_grad = nullptr;
    double* d_part = nullptr;
    int rc = VIE_OK;
    auto release = [&]() {
        cudaFree(d_mask);
        cudaFree(d_rhs_bak);
        cudaFree(d_J);
        cudaFree(d_grad);
        cudaFree(d_part);
    };
    if (cudaMalloc(&d_mask, (size_t)a) != cudaSuccess || cudaMalloc(&d_rhs_bak, sizeof(double2) * n3) != cudaSuccess ||
        cudaMalloc(&d_J, sizeof(double2) * n3) != cudaSuccess ||
        cudaMalloc(&d_part, sizeof(double) * (kAdjBlocks + 1)) != cudaSuccess ||
        (grad && cudaMalloc(&d_grad, sizeof(double2) * a) != cudaSuccess)) {
        release();
        return ctx->set_error(VIE_ERR_ALLOC, "device buffers of the adjoint gradient");
    }
    auto cuda_fail = [&](cudaError_t e) {
        release();
        return ctx->set_error(VIE_ERR_CUDA, cudaGetErrorString(e));
    };
    cudaError_t e = cudaMemcpyAsync(d_mask, edge_mask, (size_t)a, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_rhs_bak, ctx->d_rhs, sizeof(double2) * n3, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return cuda_fail(e);
    // forward solve: J
    vie_solve_info fi{};
    rc = solve_driver(ctx, prm, &fi);
    if (info_fwd) *info_fwd = fi;
    if (rc) {
        cudaMemcpyAsync(ctx->d_rhs, d_rhs_bak, sizeof(double2) * n3, cudaMemcpyDeviceToDevice, st);
        cudaStreamSynchronize(st);
        release();
        return rc;
    }
    e = cudaMemcpyAsync(d_J, ctx->d_x, sizeof(double2) * n3, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return cuda_fail(e);
    const double2* w = ctx->op64.dev.w;  // per-voxel 1/(eps - 1), FP64 (uploaded by the solve at the latest)
    if (!w) {
        release();
        return ctx->set_error(VIE_ERR_STATE, "permittivity not uploaded");
    }
    // P and the adjoint source (written over the right-hand side)
    k_power_source<<<kAdjBlocks, 256, 0, st>>>(d_J, w, d_mask, g, c0, ctx->d_rhs, d_part);
    count_launch();
    k_sum_partials<<<1, 256, 0, st>>>(d_part, kAdjBlocks, d_part + kAdjBlocks);
    count_launch();
    double P = 0.0;
    e = cudaMemcpyAsync(&P, d_part + kAdjBlocks, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e);
    if (power) *power = P;
    vie_solve_info ai{};
    ai.steps = -1;
    if (grad) {
        bool src_zero = !(P != 0.0);
        if (!src_zero) {
            // adjoint: A mu = conj(g) (A complex-symmetric), same driver and precision
            rc = solve_driver(ctx, prm, &ai);
            if (rc) {
                cudaMemcpyAsync(ctx->d_rhs, d_rhs_bak, sizeof(double2) * n3, cudaMemcpyDeviceToDevice, st);
                cudaMemcpyAsync(ctx->d_x, d_J, sizeof(double2) * n3, cudaMemcpyDeviceToDevice, st);
                cudaStreamSynchronize(st);
                if (info_adj) *info_adj = ai;
                release();
                return rc;
            }
        } else {
            // P = 0: no field on the objective edges, the gradient is zero
            e = cudaMemsetAsync(ctx->d_x, 0, sizeof(double2) * n3, st);
            if (e != cudaSuccess) return cuda_fail(e);
        }
        const double3 dcoef = make_double3(-ctx->d[0] * kZ0 / (2.0 * ctx->k0), -ctx->d[1] * kZ0 / (2.0 * ctx->k0),
                                           -ctx->d[2] * kZ0 / (2.0 * ctx->k0));
        k_adjoint_grad<<<kAdjBlocks, 256, 0, st>>>(d_J, ctx->d_x, w, ctx->d_flags, d_mask, g, c0, dcoef, d_grad);
        count_launch();
        e = cudaMemcpyAsync(grad, d_grad, sizeof(double2) * a, cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) return cuda_fail(e);
    }
    if (info_adj) *info_adj = ai;
    // the context keeps its incident field and the forward solution
    e = cudaMemcpyAsync(ctx->d_rhs, d_rhs_bak, sizeof(double2) * n3, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->d_x, d_J, sizeof(double2) * n3, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e);
    release();
    return VIE_OK;
}

}  // namespace vie
