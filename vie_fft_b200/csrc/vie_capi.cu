// vie_capi.cu -- the extern "C" entry points declared in include/vie_b200.h.
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>

#include "vie_internal.h"

namespace vie {
int green_compute(vie_ctx* ctx);
int green_expand(vie_ctx* ctx, double2* d_out);
int incident_compute(vie_ctx* ctx, double theta, double phi, double psi, double2* d_e);
int solve_driver(vie_ctx* ctx, const vie_solve_params* prm, vie_solve_info* info);
int solve_batch_driver(vie_ctx* const* ctxs, int n, const vie_solve_params* prm, vie_solve_info* infos);
void tune_apply_cached(vie_ctx* ctx);
int scene_driver(vie_ctx* ctx, const vie_primitive* prims, int n, unsigned char* material_out);
int scene_check(const vie_primitive* prims, int n);
int farfield1_driver(vie_ctx* ctx, double theta, double phi, double psi, double* fwd);
int farfield2_driver(vie_ctx* ctx, double phi, double* rcs_theta, double* rcs_phi);
int nearfield_driver(vie_ctx* ctx, const unsigned char* material, double* out3);
int autotune_driver(vie_ctx* ctx, int flags);
int power_grad_driver(vie_ctx* ctx, const unsigned char* edge_mask, const vie_solve_params* prm, double* power,
                      double* grad, vie_solve_info* info_fwd, vie_solve_info* info_adj);
int residual_driver(vie_ctx* ctx, double* relres);
void mask_component(double2* v, const unsigned char* flags, long long a, int comp, cudaStream_t st);
}  // namespace vie

using namespace vie;

std::atomic<long long> vie::g_launches{0};

namespace {

int check_ctx(vie_ctx* ctx) { return ctx ? VIE_OK : VIE_ERR_ARG; }

#define CTX_CUDA(expr)                                                                     \
    do {                                                                                   \
        cudaError_t e__ = (expr);                                                          \
        if (e__ != cudaSuccess) return ctx->set_error(VIE_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e__)); \
    } while (0)

// (Re)build both operators once flags exist (tables do not depend on eps or Green).
// Tile sizes: defaults chosen per precision by Operator::init; the
// environment variable VIE_TILES="tz,tc,tx" overrides them (tuning runs).
TileCfg tiles_from_env() {
    TileCfg t{};
    if (const char* s = std::getenv("VIE_TILES")) {
        int a = 0, b = 0, c = 0;
        if (std::sscanf(s, "%d,%d,%d", &a, &b, &c) == 3) { t.tz = a; t.tc = b; t.tx = c; }
    }
    // VIE_XTILE=1: the register x pass with the half pencil tile (otherwise the autotuner decides)
    if (const char* x = std::getenv("VIE_XTILE")) t.xalt = std::atoi(x) == 1 ? 1 : 0;
    // VIE_TMA=0: the y passes with plain loads instead of TMA-staged tiles
    if (const char* x = std::getenv("VIE_TMA")) t.ytma = std::atoi(x) == 0 ? 0 : 1;
    // VIE_ZSTAGE=0: the z passes with element loads instead of rows staged by bulk copies
    if (const char* x = std::getenv("VIE_ZSTAGE")) t.zstage = std::atoi(x) == 0 ? 0 : 1;
    // VIE_WAIT_TEST=1: every staged tile's wait runs out (tests of VIE_ERR_TIMEOUT)
    if (const char* x = std::getenv("VIE_WAIT_TEST")) t.wait_test = std::atoi(x) == 1 ? 1 : 0;
    return t;
}

int ensure_operators(vie_ctx* ctx) {
    if (ctx->op64.ready && ctx->op32.ready) return VIE_OK;
    if (!ctx->sched_set) {
        // defaults (VIE_TILES), replaced by a tuned schedule of this grid when
        // the process has one (vie_autotune, VIE_TUNE_CACHE); VIE_AUTOTUNE=1
        // tunes every new grid shape on first use
        ctx->sched64 = ctx->sched32 = tiles_from_env();
        for (int ax = 0; ax < 3; ax++) ctx->plans64[ax] = ctx->plans32[ax] = ctx->plans[ax];
        ctx->sched_set = true;
        tune_apply_cached(ctx);
    }
    int rc = ctx->op64.init(ctx->nx, ctx->ny, ctx->nz, ctx->d, ctx->k0, ctx->sched64, ctx->plans64, ctx->d_flags,
                            ctx->err);
    if (rc) return rc;
    rc = ctx->op32.init(ctx->nx, ctx->ny, ctx->nz, ctx->d, ctx->k0, ctx->sched32, ctx->plans32, ctx->d_flags,
                        ctx->err);
    if (rc) return rc;
    if (const char* at = std::getenv("VIE_AUTOTUNE"))
        if (at[0] == '1' && ctx->tune_report.empty()) rc = autotune_driver(ctx, 0);
    return rc;
}

int ready_for_operator(vie_ctx* ctx) {
    if (int rc = ctx->check_usable()) return rc;
    if (!ctx->have_flags) return ctx->set_error(VIE_ERR_STATE, "edge flags not set (vie_set_flags)");
    if (!ctx->have_eps) return ctx->set_error(VIE_ERR_STATE, "permittivity not set (vie_set_material / vie_set_eps)");
    if (!ctx->have_green) return ctx->set_error(VIE_ERR_STATE, "Green's function not computed (vie_green)");
    return VIE_OK;
}

int upload_contrast(vie_ctx* ctx) {
    int rc = ensure_operators(ctx);
    if (rc) return rc;
    rc = ctx->op64.set_contrast(ctx->w_host.data(), ctx->stream, ctx->err);
    if (rc) return rc;
    return ctx->op32.set_contrast(ctx->w_host.data(), ctx->stream, ctx->err);
}

}  // namespace

extern "C" {

long long vie_launch_count(void) { return g_launches.load(); }

const char* vie_version(void) { return "vie_b200 0.1 (sm_100a)"; }

const char* vie_status_string(int s) {
    switch (s) {
        case VIE_OK: return "ok";
        case VIE_ERR_ARG: return "invalid argument";
        case VIE_ERR_ALLOC: return "allocation failed";
        case VIE_ERR_CUDA: return "CUDA error";
        case VIE_ERR_BREAKDOWN: return "Krylov breakdown";
        case VIE_ERR_MAXIT: return "iteration cap reached";
        case VIE_ERR_NAN: return "non-finite value";
        case VIE_ERR_STATE: return "call order";
        case VIE_ERR_TIMEOUT: return "device wait timed out";
        case VIE_ERR_NODEVICE: return "no CUDA device";
        default: return "unknown status";
    }
}

const char* vie_last_error(const vie_ctx* ctx) { return ctx ? ctx->err.msg.c_str() : "null context"; }

int vie_create(const vie_grid* g, vie_ctx** out) {
    if (!g || !out) return VIE_ERR_ARG;
    *out = nullptr;
    if (g->nx < 2 || g->ny < 2 || g->nz < 2 || !(g->dx > 0) || !(g->dy > 0) || !(g->dz > 0) || !(g->k0 > 0))
        return VIE_ERR_ARG;
    if (g->nx > 65535 || g->ny > 32767 || g->nz > 65535) return VIE_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return VIE_ERR_NODEVICE;
    if (g->device < 0 || g->device >= ndev) return VIE_ERR_ARG;
    vie_ctx* ctx = new (std::nothrow) vie_ctx();
    if (!ctx) return VIE_ERR_ALLOC;
    ctx->device = g->device;
    ctx->nx = g->nx; ctx->ny = g->ny; ctx->nz = g->nz;
    ctx->a = (long long)g->nx * g->ny * g->nz;
    ctx->d[0] = g->dx; ctx->d[1] = g->dy; ctx->d[2] = g->dz;
    ctx->k0 = g->k0;
    const int n3[3] = {g->nx, g->ny, g->nz};
    for (int ax = 0; ax < 3; ax++) ctx->plans[ax] = make_axis_plan(n3[ax]);
    if (cudaSetDevice(g->device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&ctx->d_flags, (size_t)ctx->a) != cudaSuccess ||
        cudaMalloc(&ctx->d_rhs, sizeof(double2) * 3 * (size_t)ctx->a) != cudaSuccess ||
        cudaMalloc(&ctx->d_x, sizeof(double2) * 3 * (size_t)ctx->a) != cudaSuccess) {
        vie_destroy(ctx);
        return VIE_ERR_ALLOC;
    }
    cudaMemset(ctx->d_flags, 0, (size_t)ctx->a);
    cudaMemset(ctx->d_x, 0, sizeof(double2) * 3 * (size_t)ctx->a);
    ctx->w_host.assign(2 * (size_t)ctx->a, 0.0);
    if (const char* gv = std::getenv("VIE_GRAPH")) ctx->use_graphs = std::atoi(gv) != 0;
    *out = ctx;
    return VIE_OK;
}

void vie_destroy(vie_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    ctx->op64.release();
    ctx->op32.release();
    if (ctx->d_flags) cudaFree(ctx->d_flags);
    if (ctx->d_green) cudaFree(ctx->d_green);
    if (ctx->d_rhs) cudaFree(ctx->d_rhs);
    if (ctx->d_x) cudaFree(ctx->d_x);
    for (size_t i = 0; i < ctx->work.size(); i += 2)
        if (ctx->work[i]) cudaFree(ctx->work[i]);
    if (ctx->d_scal) cudaFree(ctx->d_scal);
    if (ctx->d_partial) cudaFree(ctx->d_partial);
    if (ctx->h_scal) cudaFreeHost(ctx->h_scal);
    if (ctx->d_ctl) cudaFree(ctx->d_ctl);
    if (ctx->h_ctl) cudaFreeHost(ctx->h_ctl);
    if (ctx->d_hist) cudaFree(ctx->d_hist);
    if (ctx->stream_aux) cudaStreamDestroy(ctx->stream_aux);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

int vie_set_eps(vie_ctx* ctx, const double* eps) {
    if (check_ctx(ctx) || !eps) return VIE_ERR_ARG;
    if (int u = ctx->check_usable()) return u;
    cudaSetDevice(ctx->device);
    // w = 1/(eps - 1), the per-voxel factor of the diagonal term (fft.h:430-432)
    for (long long v = 0; v < ctx->a; v++) {
        const std::complex<double> e(eps[2 * v] - 1.0, eps[2 * v + 1]);
        if (e == std::complex<double>(0.0, 0.0))
            return ctx->set_error(VIE_ERR_ARG, "permittivity equal to 1 (zero contrast) at voxel " + std::to_string(v));
        const std::complex<double> w = 1.0 / e;
        ctx->w_host[2 * v] = w.real();
        ctx->w_host[2 * v + 1] = w.imag();
    }
    ctx->have_eps = true;
    if (!ctx->have_flags) return VIE_OK;
    return upload_contrast(ctx);
}

int vie_set_material(vie_ctx* ctx, const uint8_t* material, const double* eps_re, const double* eps_im,
                     int n_materials) {
    if (check_ctx(ctx) || !material || !eps_re || !eps_im || n_materials < 1 || n_materials > 256)
        return VIE_ERR_ARG;
    if (int u = ctx->check_usable()) return u;
    std::vector<double> eps(2 * (size_t)ctx->a);
    for (long long v = 0; v < ctx->a; v++) {
        const int m = material[v];
        if (m >= n_materials) return ctx->set_error(VIE_ERR_ARG, "material index outside the permittivity table");
        eps[2 * v] = eps_re[m];
        eps[2 * v + 1] = eps_im[m];
    }
    return vie_set_eps(ctx, eps.data());
}

int vie_set_geometry_scene(vie_ctx* ctx, const vie_primitive* prims, int n, const double* eps_re,
                           const double* eps_im, int n_materials, uint8_t* material_out) {
    if (check_ctx(ctx) || !eps_re || !eps_im || n_materials < 1 || n_materials > 256) return VIE_ERR_ARG;
    if (int u = ctx->check_usable()) return u;
    if (scene_check(prims, n)) return ctx->set_error(VIE_ERR_ARG, "invalid scene primitive (kind, label or parent)");
    for (int q = 0; q < n; q++)
        if (prims[q].label >= n_materials) return ctx->set_error(VIE_ERR_ARG, "scene label outside the table");
    cudaSetDevice(ctx->device);
    std::vector<uint8_t> mat((size_t)ctx->a);
    int rc = scene_driver(ctx, prims, n, mat.data());
    if (rc) return rc;
    ctx->have_flags = true;
    if ((rc = vie_set_material(ctx, mat.data(), eps_re, eps_im, n_materials))) return rc;
    if ((rc = ensure_operators(ctx))) return rc;
    if (ctx->have_green) {
        rc = ctx->op64.set_green(ctx->d_green, ctx->k0, ctx->stream, ctx->err);
        if (!rc) rc = ctx->op32.set_green(ctx->d_green, ctx->k0, ctx->stream, ctx->err);
    }
    if (!rc && material_out) std::memcpy(material_out, mat.data(), (size_t)ctx->a);
    return rc;
}

int vie_set_flags(vie_ctx* ctx, const uint8_t* fx, const uint8_t* fy, const uint8_t* fz) {
    if (check_ctx(ctx) || !fx || !fy || !fz) return VIE_ERR_ARG;
    if (int u = ctx->check_usable()) return u;
    cudaSetDevice(ctx->device);
    std::vector<uint8_t> packed((size_t)ctx->a);
    for (long long v = 0; v < ctx->a; v++)
        packed[v] = (uint8_t)((fx[v] ? 1 : 0) | (fy[v] ? 2 : 0) | (fz[v] ? 4 : 0));
    CTX_CUDA(cudaMemcpy(ctx->d_flags, packed.data(), (size_t)ctx->a, cudaMemcpyHostToDevice));
    ctx->have_flags = true;
    int rc = ensure_operators(ctx);
    if (rc) return rc;
    if (ctx->have_eps) rc = upload_contrast(ctx);
    if (!rc && ctx->have_green) {
        rc = ctx->op64.set_green(ctx->d_green, ctx->k0, ctx->stream, ctx->err);
        if (!rc) rc = ctx->op32.set_green(ctx->d_green, ctx->k0, ctx->stream, ctx->err);
    }
    return rc;
}

int vie_green(vie_ctx* ctx) {
    if (check_ctx(ctx)) return VIE_ERR_ARG;
    if (int u = ctx->check_usable()) return u;
    cudaSetDevice(ctx->device);
    int rc = green_compute(ctx);
    if (rc) return rc;
    ctx->have_green = true;
    if (ctx->op64.ready) {
        rc = ctx->op64.set_green(ctx->d_green, ctx->k0, ctx->stream, ctx->err);
        if (!rc) rc = ctx->op32.set_green(ctx->d_green, ctx->k0, ctx->stream, ctx->err);
        if (rc) return rc;
    }
    CTX_CUDA(cudaStreamSynchronize(ctx->stream));
    return VIE_OK;
}

int vie_green_spectrum(vie_ctx* ctx, double* out) {
    if (check_ctx(ctx) || !out) return VIE_ERR_ARG;
    if (int u = ctx->check_usable()) return u;
    if (!ctx->have_green) return ctx->set_error(VIE_ERR_STATE, "Green's function not computed (vie_green)");
    cudaSetDevice(ctx->device);
    const size_t m = 8 * (size_t)ctx->a;
    double2* d = nullptr;
    CTX_CUDA(cudaMalloc(&d, sizeof(double2) * m));
    int rc = green_expand(ctx, d);
    if (!rc) {
        cudaError_t e = cudaMemcpyAsync(out, d, sizeof(double2) * m, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = ctx->set_error(VIE_ERR_CUDA, cudaGetErrorString(e));
    }
    cudaFree(d);
    return rc;
}

int vie_incident(vie_ctx* ctx, double theta, double phi, double psi, double* out) {
    if (check_ctx(ctx)) return VIE_ERR_ARG;
    if (int u = ctx->check_usable()) return u;
    cudaSetDevice(ctx->device);
    int rc = incident_compute(ctx, theta, phi, psi, ctx->d_rhs);
    if (rc) return rc;
    ctx->have_rhs = true;
    if (out) {
        CTX_CUDA(cudaMemcpyAsync(out, ctx->d_rhs, sizeof(double2) * 3 * (size_t)ctx->a, cudaMemcpyDeviceToHost,
                                 ctx->stream));
    }
    CTX_CUDA(cudaStreamSynchronize(ctx->stream));
    return VIE_OK;
}

int vie_set_rhs(vie_ctx* ctx, const double* e) {
    if (check_ctx(ctx) || !e) return VIE_ERR_ARG;
    if (int u = ctx->check_usable()) return u;
    cudaSetDevice(ctx->device);
    CTX_CUDA(cudaMemcpyAsync(ctx->d_rhs, e, sizeof(double2) * 3 * (size_t)ctx->a, cudaMemcpyHostToDevice, ctx->stream));
    CTX_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->have_rhs = true;
    return VIE_OK;
}

int vie_rhs_device(vie_ctx* ctx, void** rhs) {
    if (check_ctx(ctx) || !rhs) return VIE_ERR_ARG;
    if (int u = ctx->check_usable()) return u;
    *rhs = ctx->d_rhs;
    ctx->have_rhs = true;
    return VIE_OK;
}

int vie_matvec_dev(vie_ctx* ctx, const void* x, void* y, int conj, int precision) {
    if (check_ctx(ctx) || !x || !y) return VIE_ERR_ARG;
    int rc = ready_for_operator(ctx);
    if (rc) return rc;
    cudaSetDevice(ctx->device);
    if (precision == VIE_PREC_FP64)
        return ctx->op64.apply((const double2*)x, (double2*)y, conj != 0, ctx->stream, ctx->err);
    if (precision == VIE_PREC_MIXED)
        return ctx->op32.apply((const float2*)x, (float2*)y, conj != 0, ctx->stream, ctx->err);
    return ctx->set_error(VIE_ERR_ARG, "precision must be VIE_PREC_FP64 or VIE_PREC_MIXED");
}

int vie_matvec(vie_ctx* ctx, const double* x, double* y, int conj) { return vie_apply(ctx, x, y, conj, VIE_PART_ALL); }

int vie_apply(vie_ctx* ctx, const double* x, double* y, int conj, int parts) {
    if (check_ctx(ctx) || !x || !y || (parts & ~VIE_PART_ALL)) return VIE_ERR_ARG;
    int rc = ready_for_operator(ctx);
    if (rc) return rc;
    cudaSetDevice(ctx->device);
    const size_t bytes = sizeof(double2) * 3 * (size_t)ctx->a;
    double2 *dx = nullptr, *dy = nullptr;
    CTX_CUDA(cudaMalloc(&dx, bytes));
    if (cudaMalloc(&dy, bytes) != cudaSuccess) {
        cudaFree(dx);
        return ctx->set_error(VIE_ERR_ALLOC, "device allocation failed");
    }
    cudaError_t e = cudaMemcpyAsync(dx, x, bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) {
        vie::Operator<double> op = ctx->op64;  // same tables and scratch, selected parts
        op.dev.parts = parts;
        rc = op.apply(dx, dy, conj != 0, ctx->stream, ctx->err);
        if (!rc) {
            e = cudaMemcpyAsync(y, dy, bytes, cudaMemcpyDeviceToHost, ctx->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        }
    }
    if (e != cudaSuccess) rc = ctx->set_error(VIE_ERR_CUDA, cudaGetErrorString(e));
    cudaFree(dx);
    cudaFree(dy);
    return ctx->check_waits(rc);
}

int vie_reset(vie_ctx* ctx, double* v, int comp) {
    if (check_ctx(ctx) || !v || comp < 0 || comp > 2) return VIE_ERR_ARG;
    if (int u = ctx->check_usable()) return u;
    if (!ctx->have_flags) return ctx->set_error(VIE_ERR_STATE, "edge flags not set (vie_set_flags)");
    cudaSetDevice(ctx->device);
    const size_t bytes = sizeof(double2) * (size_t)ctx->a;
    double2* d = nullptr;
    CTX_CUDA(cudaMalloc(&d, bytes));
    cudaError_t e = cudaMemcpyAsync(d, v, bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) {
        mask_component(d, ctx->d_flags, ctx->a, comp, ctx->stream);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(v, d, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d);
    if (e != cudaSuccess) return ctx->set_error(VIE_ERR_CUDA, cudaGetErrorString(e));
    return VIE_OK;
}

int vie_solve(vie_ctx* ctx, const vie_solve_params* p, double* x, vie_solve_info* info) {
    if (check_ctx(ctx) || !p) return VIE_ERR_ARG;
    int rc = ready_for_operator(ctx);
    if (rc) return rc;
    if (!ctx->have_rhs) return ctx->set_error(VIE_ERR_STATE, "no right-hand side (vie_incident / vie_set_rhs)");
    if (!(p->tol > 0)) return ctx->set_error(VIE_ERR_ARG, "tolerance must be positive");
    cudaSetDevice(ctx->device);
    ctx->err.code = VIE_OK;
    ctx->err.msg.clear();
    rc = solve_driver(ctx, p, info);
    if (x && ctx->have_x) {
        cudaError_t e = cudaMemcpyAsync(x, ctx->d_x, sizeof(double2) * 3 * (size_t)ctx->a, cudaMemcpyDeviceToHost,
                                        ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess && !rc) rc = ctx->set_error(VIE_ERR_CUDA, cudaGetErrorString(e));
    }
    return ctx->check_waits(rc);
}

int vie_solve_batch(vie_ctx* const* ctxs, int n, const vie_solve_params* p, vie_solve_info* infos) {
    if (!ctxs || n < 1 || !p) return VIE_ERR_ARG;
    for (int i = 0; i < n; i++) {
        vie_ctx* c = ctxs[i];
        if (check_ctx(c)) return VIE_ERR_ARG;
        for (int k = 0; k < i; k++)
            if (ctxs[k] == c) return c->set_error(VIE_ERR_ARG, "a context appears twice in the batch");
        if (c->device != ctxs[0]->device) return c->set_error(VIE_ERR_ARG, "batch contexts on different devices");
        int rc = ready_for_operator(c);
        if (rc) return rc;
        if (!c->have_rhs) return c->set_error(VIE_ERR_STATE, "no right-hand side (vie_incident / vie_set_rhs)");
        c->err.code = VIE_OK;
        c->err.msg.clear();
    }
    if (!(p->tol > 0)) return ctxs[0]->set_error(VIE_ERR_ARG, "tolerance must be positive");
    cudaSetDevice(ctxs[0]->device);
    int rc = solve_batch_driver(ctxs, n, p, infos);
    cudaStreamSynchronize(ctxs[0]->stream);
    for (int i = 0; i < n; i++) {
        const int w = ctxs[i]->check_waits(VIE_OK);
        if (w && !rc) rc = w;
    }
    return rc;
}

int vie_power_grad(vie_ctx* ctx, const unsigned char* edge_mask, const vie_solve_params* p, double* power,
                   double* grad, vie_solve_info* info_fwd, vie_solve_info* info_adj) {
    if (check_ctx(ctx) || !edge_mask || !p || !power) return VIE_ERR_ARG;
    int rc = ready_for_operator(ctx);
    if (rc) return rc;
    if (!ctx->have_rhs) return ctx->set_error(VIE_ERR_STATE, "no right-hand side (vie_incident / vie_set_rhs)");
    if (!(p->tol > 0)) return ctx->set_error(VIE_ERR_ARG, "tolerance must be positive");
    if (grad && !(ctx->d[0] == ctx->d[1] && ctx->d[1] == ctx->d[2]))
        return ctx->set_error(VIE_ERR_ARG, "the adjoint gradient needs cubic voxels (complex-symmetric operator)");
    cudaSetDevice(ctx->device);
    ctx->err.code = VIE_OK;
    ctx->err.msg.clear();
    rc = power_grad_driver(ctx, edge_mask, p, power, grad, info_fwd, info_adj);
    rc = ctx->check_waits(rc);
    if (!rc) ctx->have_x = true;
    return rc;
}

static int ready_for_post(vie_ctx* ctx) {
    if (check_ctx(ctx)) return VIE_ERR_ARG;
    if (int u = ctx->check_usable()) return u;
    if (!ctx->have_x) return ctx->set_error(VIE_ERR_STATE, "no solution yet (vie_solve)");
    cudaSetDevice(ctx->device);
    return VIE_OK;
}

int vie_farfield1(vie_ctx* ctx, double theta, double phi, double psi, double* forward_rcs) {
    int rc = ready_for_post(ctx);
    if (rc) return rc;
    if (!forward_rcs) return ctx->set_error(VIE_ERR_ARG, "null output");
    return farfield1_driver(ctx, theta, phi, psi, forward_rcs);
}

int vie_farfield2(vie_ctx* ctx, double phi, double* rcs_theta, double* rcs_phi) {
    int rc = ready_for_post(ctx);
    if (rc) return rc;
    if (!rcs_theta || !rcs_phi) return ctx->set_error(VIE_ERR_ARG, "null output");
    return farfield2_driver(ctx, phi, rcs_theta, rcs_phi);
}

int vie_nearfield(vie_ctx* ctx, const uint8_t* material, double* ene_metal, double* ene_active,
                  double* absorb_volume) {
    int rc = ready_for_post(ctx);
    if (rc) return rc;
    if (!material) return ctx->set_error(VIE_ERR_ARG, "null material");
    if (!ctx->have_eps || !ctx->op64.ready) return ctx->set_error(VIE_ERR_STATE, "permittivity not set");
    double o[3];
    rc = nearfield_driver(ctx, material, o);
    if (rc) return rc;
    if (ene_metal) *ene_metal = o[0];
    if (ene_active) *ene_active = o[1];
    if (absorb_volume) *absorb_volume = o[2];
    return VIE_OK;
}

int vie_autotune(vie_ctx* ctx, int flags, char* report, int report_len) {
    if (check_ctx(ctx)) return VIE_ERR_ARG;
    if (int u = ctx->check_usable()) return u;
    if (!ctx->have_flags) return ctx->set_error(VIE_ERR_STATE, "edge flags not set (vie_set_flags)");
    cudaSetDevice(ctx->device);
    int rc = ensure_operators(ctx);
    if (!rc) rc = autotune_driver(ctx, flags);
    if (report && report_len > 0) {
        std::snprintf(report, (size_t)report_len, "%s", ctx->tune_report.c_str());
    }
    return rc;
}

int vie_residual(vie_ctx* ctx, double* relres) {
    if (check_ctx(ctx) || !relres) return VIE_ERR_ARG;
    int rc = ready_for_operator(ctx);
    if (rc) return rc;
    if (!ctx->have_rhs || !ctx->have_x) return ctx->set_error(VIE_ERR_STATE, "no solution yet (vie_solve)");
    cudaSetDevice(ctx->device);
    return residual_driver(ctx, relres);
}

int vie_get_solution(vie_ctx* ctx, double* x) {
    if (check_ctx(ctx) || !x) return VIE_ERR_ARG;
    if (!ctx->have_x) return ctx->set_error(VIE_ERR_STATE, "no solution yet (vie_solve)");
    cudaSetDevice(ctx->device);
    CTX_CUDA(cudaMemcpyAsync(x, ctx->d_x, sizeof(double2) * 3 * (size_t)ctx->a, cudaMemcpyDeviceToHost, ctx->stream));
    CTX_CUDA(cudaStreamSynchronize(ctx->stream));
    return VIE_OK;
}

int vie_set_solution(vie_ctx* ctx, const double* x) {
    if (check_ctx(ctx) || !x) return VIE_ERR_ARG;
    cudaSetDevice(ctx->device);
    CTX_CUDA(cudaMemcpyAsync(ctx->d_x, x, sizeof(double2) * 3 * (size_t)ctx->a, cudaMemcpyHostToDevice, ctx->stream));
    CTX_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->have_x = true;
    return VIE_OK;
}

int vie_solution_device(vie_ctx* ctx, const void** x) {
    if (check_ctx(ctx) || !x) return VIE_ERR_ARG;
    *x = ctx->d_x;
    return VIE_OK;
}

int vie_stream(vie_ctx* ctx, void** stream) {
    if (check_ctx(ctx) || !stream) return VIE_ERR_ARG;
    *stream = (void*)ctx->stream;
    return VIE_OK;
}

int vie_sync(vie_ctx* ctx) {
    if (check_ctx(ctx)) return VIE_ERR_ARG;
    CTX_CUDA(cudaStreamSynchronize(ctx->stream));
    return ctx->check_waits(VIE_OK);
}

}  // extern "C"
