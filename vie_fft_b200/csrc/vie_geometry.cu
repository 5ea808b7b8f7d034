// vie_geometry.cu -- material labels and edge flags on the GPU (GetMaterial
// and GetFlag, Model.h:305-398) from an analytic scene.
//
// The label of a point is that of the first primitive of the scene that holds
// it and whose parent (any other primitive, or none) holds it too, else 0
// (air).  The primitive
// tests are the reference's own forms of Model_Identifier (Model.h:215-300):
//   VIE_PRIM_SPHERE      sqrt((x-cx)^2 + (y-cy)^2 + (z-cz)^2) <= r   (one sphere)
//   VIE_PRIM_SPHERE_F32  float(squared distance) < float(r^2)        (the sphere
//                        loop of the layered solar-cell model)
//   VIE_PRIM_BOX         |x-cx| < hx && |y-cy| < hy && |z-cz| < hz    (its layers)
// Material[i][j][k] is the label at the voxel centre; Flag_f is set when the
// rooftop point and both neighbouring voxel centres along f are non-air
// (Model.h:352-394).
#include <cmath>
#include <vector>

#include "vie_internal.h"

namespace vie {

namespace {

constexpr int kMaxPrims = 256;

__device__ __forceinline__ bool prim_holds(const vie_primitive& p, double x, double y, double z) {
    const double dx = x - p.c[0], dy = y - p.c[1], dz = z - p.c[2];
    if (p.kind == VIE_PRIM_SPHERE) return sqrt(dx * dx + dy * dy + dz * dz) <= p.r;
    if (p.kind == VIE_PRIM_SPHERE_F32) return (float)(dx * dx + dy * dy + dz * dz) < (float)(p.r * p.r);
    return fabs(dx) < p.h[0] && fabs(dy) < p.h[1] && fabs(dz) < p.h[2];
}

__device__ __forceinline__ int scene_label(const vie_primitive* P, int n, double x, double y, double z) {
    for (int q = 0; q < n; q++) {
        if (!prim_holds(P[q], x, y, z)) continue;
        const int par = P[q].parent;
        if (par >= 0 && !prim_holds(P[par], x, y, z)) continue;
        return P[q].label;
    }
    return 0;
}

__global__ void __launch_bounds__(256) k_scene(const vie_primitive* __restrict__ prims, int n, int nx, int ny, int nz,
                                               double dx, double dy, double dz, unsigned char* __restrict__ material,
                                               unsigned char* __restrict__ flags) {
    __shared__ vie_primitive P[kMaxPrims];
    for (int q = threadIdx.x; q < n; q += blockDim.x) P[q] = prims[q];
    __syncthreads();
    const long long a = (long long)nx * ny * nz;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < a; v += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(v / ((long long)ny * nz)), j = (int)((v / nz) % ny), k = (int)(v % nz);
        // GetMaterial (Model.h:319-324)
        material[v] = (unsigned char)scene_label(P, n, i * dx + 0.5 * dx, j * dy + 0.5 * dy, k * dz + 0.5 * dz);
        unsigned char f = 0;
        {   // x rooftop (Model.h:352-364)
            const double px = (i + 1) * dx, py = (j + 0.5) * dy, pz = (k + 0.5) * dz;
            if (scene_label(P, n, px, py, pz) != 0 && scene_label(P, n, px - 0.5 * dx, py, pz) != 0 &&
                scene_label(P, n, px + 0.5 * dx, py, pz) != 0)
                f |= 1;
        }
        {   // y rooftop (:367-379)
            const double px = (i + 0.5) * dx, py = (j + 1) * dy, pz = (k + 0.5) * dz;
            if (scene_label(P, n, px, py, pz) != 0 && scene_label(P, n, px, py - 0.5 * dy, pz) != 0 &&
                scene_label(P, n, px, py + 0.5 * dy, pz) != 0)
                f |= 2;
        }
        {   // z rooftop (:382-394)
            const double px = (i + 0.5) * dx, py = (j + 0.5) * dy, pz = (k + 1) * dz;
            if (scene_label(P, n, px, py, pz) != 0 && scene_label(P, n, px, py, pz - 0.5 * dz) != 0 &&
                scene_label(P, n, px, py, pz + 0.5 * dz) != 0)
                f |= 4;
        }
        flags[v] = f;
    }
}

}  // namespace

// labels and flags of the scene into material_out (host, a bytes) and ctx->d_flags
int scene_driver(vie_ctx* ctx, const vie_primitive* prims, int n, unsigned char* material_out) {
    cudaStream_t st = ctx->stream;
    vie_primitive* d_prims = nullptr;
    unsigned char* d_mat = nullptr;
    if (cudaMalloc(&d_prims, sizeof(vie_primitive) * (n > 0 ? n : 1)) != cudaSuccess ||
        cudaMalloc(&d_mat, (size_t)ctx->a) != cudaSuccess) {
        cudaFree(d_prims);
        return ctx->set_error(VIE_ERR_ALLOC, "scene buffers");
    }
    cudaError_t e = cudaSuccess;
    if (n > 0) e = cudaMemcpyAsync(d_prims, prims, sizeof(vie_primitive) * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        k_scene<<<148 * 8, 256, 0, st>>>(d_prims, n, ctx->nx, ctx->ny, ctx->nz, ctx->d[0], ctx->d[1], ctx->d[2], d_mat,
                                         ctx->d_flags);
        count_launch();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(material_out, d_mat, (size_t)ctx->a, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d_prims);
    cudaFree(d_mat);
    if (e != cudaSuccess) return ctx->set_error(VIE_ERR_CUDA, cudaGetErrorString(e));
    return VIE_OK;
}

int scene_check(const vie_primitive* prims, int n) {
    if (n < 0 || n > kMaxPrims || (n > 0 && !prims)) return VIE_ERR_ARG;
    for (int q = 0; q < n; q++) {
        const vie_primitive& p = prims[q];
        if (p.kind != VIE_PRIM_SPHERE && p.kind != VIE_PRIM_SPHERE_F32 && p.kind != VIE_PRIM_BOX) return VIE_ERR_ARG;
        if (p.label < 0 || p.label > 255 || p.parent >= n || p.parent < -1 || p.parent == q) return VIE_ERR_ARG;
    }
    return VIE_OK;
}

}  // namespace vie
