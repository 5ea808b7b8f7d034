// vie_tune.cu -- autotuner of the FFT schedule of one grid.
//
// Per axis the operator can run the register four-step kernels (lengths with a
// compile-time plan) or the generic shared-memory kernels with any radix order
// and pencil tile.  The three axes are separable: z decides F1/I1, y F2/I2, x
// the spectral pass F3.  The tuner therefore walks the axes one at a time
// (z, y, x), times whole operator applications for every candidate of that
// axis with the others fixed at their current best, and keeps the fastest:
//   1. register kernels (when the length has them), else
//   2. generic kernels, radix orders: the default greedy one, its reverse,
//      16 -> 4x4 and 16 -> 8x2 splits (at the default tile), then
//   3. the pencil tile of the best generic order.
// Choices are cached per (device, grid, precision) for the process, so later
// contexts of the same grid (a batch) reuse them, and in the text file named
// by VIE_TUNE_CACHE when that is set.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "vie_launch.cuh"

namespace vie {

namespace {

struct Sched {
    TileCfg t;
    AxisPlan plan[3];
    float ms = 0.f;
};

std::mutex g_mu;
std::map<std::string, Sched> g_cache;
bool g_loaded = false;

std::string cache_key(int dev, int nx, int ny, int nz, int bytes) {
    std::ostringstream o;
    o << dev << ' ' << nx << ' ' << ny << ' ' << nz << ' ' << bytes;
    return o.str();
}

std::string plan_str(const AxisPlan& p) {
    std::string s;
    for (int i = 0; i < p.nst; i++) s += (i ? "x" : "") + std::to_string(p.rad[i]);
    return s;
}

// one line per entry: key(5 ints) then per axis: fast tile nst radices..., then
// xalt, ms and ytma (absent in older files: TMA staging on)
std::string serialize(const std::string& key, const Sched& s) {
    std::ostringstream o;
    o << key;
    const int tile[3] = {s.t.tx, s.t.tc, s.t.tz};
    for (int ax = 0; ax < 3; ax++) {
        o << ' ' << s.t.fast[ax] << ' ' << tile[ax] << ' ' << s.plan[ax].nst;
        for (int i = 0; i < s.plan[ax].nst; i++) o << ' ' << s.plan[ax].rad[i];
    }
    o << ' ' << s.t.xalt << ' ' << s.ms << ' ' << s.t.ytma;
    return o.str();
}

void load_file_locked() {
    if (g_loaded) return;
    g_loaded = true;
    const char* path = std::getenv("VIE_TUNE_CACHE");
    if (!path) return;
    FILE* f = std::fopen(path, "r");
    if (!f) return;
    char line[1024];
    while (std::fgets(line, sizeof line, f)) {
        std::istringstream in(line);
        int k[5];
        Sched s;
        bool ok = true;
        for (int& v : k) ok = ok && (in >> v);
        int tile[3];
        for (int ax = 0; ax < 3 && ok; ax++) {
            ok = ok && (in >> s.t.fast[ax] >> tile[ax] >> s.plan[ax].nst) && s.plan[ax].nst >= 0 &&
                 s.plan[ax].nst <= kMaxStages;
            int prod = 1;
            for (int i = 0; ok && i < s.plan[ax].nst; i++) {
                ok = ok && (in >> s.plan[ax].rad[i]) && s.plan[ax].rad[i] >= 2 &&
                     s.plan[ax].rad[i] <= kMaxGenericRadix;
                if (ok) prod *= s.plan[ax].rad[i];
            }
            s.plan[ax].n = prod;
            ok = ok && prod == k[1 + ax];
        }
        ok = ok && (in >> s.t.xalt >> s.ms) && (s.t.xalt == 0 || s.t.xalt == 1);
        if (!ok) continue;
        int ytma = 1;
        if (in >> ytma) s.t.ytma = ytma == 0 ? 0 : 1;
        s.t.tx = tile[0];
        s.t.tc = tile[1];
        s.t.tz = tile[2];
        g_cache[cache_key(k[0], k[1], k[2], k[3], k[4])] = s;
    }
    std::fclose(f);
}

void store_locked(const std::string& key, const Sched& s) {
    g_cache[key] = s;
    const char* path = std::getenv("VIE_TUNE_CACHE");
    if (!path) return;
    if (FILE* f = std::fopen(path, "a")) {
        std::fprintf(f, "%s\n", serialize(key, s).c_str());
        std::fclose(f);
    }
}

std::vector<AxisPlan> generic_orders(int n) {
    std::vector<AxisPlan> out;
    auto add = [&](const std::vector<int>& r) {
        if (r.empty() || (int)r.size() > kMaxStages) return;
        AxisPlan p = make_axis_plan(n, r);
        for (const AxisPlan& q : out)
            if (q.nst == p.nst && std::equal(q.rad, q.rad + q.nst, p.rad)) return;
        out.push_back(p);
    };
    const AxisPlan d = make_axis_plan(n);
    std::vector<int> base(d.rad, d.rad + d.nst);
    add(base);
    add(std::vector<int>(base.rbegin(), base.rend()));
    std::vector<int> s44, s82;
    for (int r : base) {
        if (r == 16) {
            s44.insert(s44.end(), {4, 4});
            s82.insert(s82.end(), {8, 2});
        } else {
            s44.push_back(r);
            s82.push_back(r);
        }
    }
    add(s44);
    add(s82);
    return out;
}

template <typename T>
int time_apply(vie_ctx* ctx, Operator<T>& op, const cplx_t<T>* x, cplx_t<T>* y, float* ms) {
    cudaStream_t st = ctx->stream;
    int rc = op.apply(x, y, false, st, ctx->err);
    if (rc) return rc;
    cudaEvent_t e0, e1;
    VIE_CUDA_TRY(cudaEventCreate(&e0), ctx->err);
    VIE_CUDA_TRY(cudaEventCreate(&e1), ctx->err);
    constexpr int reps = 3;
    cudaEventRecord(e0, st);
    for (int i = 0; i < reps && !rc; i++) rc = op.apply(x, y, false, st, ctx->err);
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = t / reps;
    // a schedule whose staged waits ran out was timed with tiles left undone:
    // the tuning fails rather than pick it (the status words are cleared here)
    if (const int w = op.take_timeout()) {
        if (w == 2) ctx->unusable = true;
        return ctx->set_error(VIE_ERR_TIMEOUT, "autotuner: a staged tile's bounded wait ran out while timing a schedule");
    }
    return rc;
}

template <typename T> int tune_one(vie_ctx* ctx, Operator<T>& op, Sched& best, std::string& report) {
    using C = cplx_t<T>;
    const int n[3] = {ctx->nx, ctx->ny, ctx->nz};
    const bool dbl = sizeof(T) == 8;
    C *x = nullptr, *y = nullptr;
    VIE_CUDA_TRY(cudaMalloc(&x, sizeof(C) * 3 * (size_t)ctx->a), ctx->err);
    if (cudaMalloc(&y, sizeof(C) * 3 * (size_t)ctx->a) != cudaSuccess) {
        cudaFree(x);
        return ctx->set_error(VIE_ERR_ALLOC, "autotuner vectors");
    }
    cudaMemsetAsync(x, 0, sizeof(C) * 3 * (size_t)ctx->a, ctx->stream);
    int rc = VIE_OK;
    auto measure = [&](const Sched& s, float* ms) -> int {
        int r = op.init(ctx->nx, ctx->ny, ctx->nz, ctx->d, ctx->k0, s.t, s.plan, ctx->d_flags, ctx->err);
        if (r) return r;
        return time_apply<T>(ctx, op, x, y, ms);
    };
    // start: the current schedule
    if ((rc = measure(best, &best.ms))) goto done;
    for (int ax : {2, 1, 0}) {
        int* tile = ax == 2 ? &best.t.tz : (ax == 1 ? &best.t.tc : &best.t.tx);
        const int deft = ax == 0 ? (dbl ? 4 : 8) : (dbl ? 8 : 16);
        std::vector<Sched> cands;
        if (fast_length(n[ax])) {
            Sched s = best;
            s.t.fast[ax] = 1;
            s.ms = 0.f;  // measured below
            cands.push_back(s);
            if (ax == 0) {  // the register x pass with the half pencil tile
                s.t.xalt = 1;
                cands.push_back(s);
            }
            if (ax == 1) {  // the register y passes with TMA staging switched the other way
                s.t.ytma = 1 - s.t.ytma;
                cands.push_back(s);
            }
        }
        Sched bestg;
        float bestg_ms = 1e30f;
        for (const AxisPlan& p : generic_orders(n[ax])) {
            Sched s = best;
            s.t.fast[ax] = 0;
            s.plan[ax] = p;
            int* st = ax == 2 ? &s.t.tz : (ax == 1 ? &s.t.tc : &s.t.tx);
            *st = deft;
            float ms;
            int r = measure(s, &ms);
            if (r == VIE_ERR_ARG) { ctx->err.code = VIE_OK; continue; }  // schedule does not fit
            if (r) { rc = r; goto done; }
            s.ms = ms;
            if (ms < bestg_ms) { bestg_ms = ms; bestg = s; }
        }
        if (bestg_ms < 1e30f) {
            for (int t : {deft / 2, deft * 2, deft * 4}) {
                if (t < 1) continue;
                Sched s = bestg;
                int* st = ax == 2 ? &s.t.tz : (ax == 1 ? &s.t.tc : &s.t.tx);
                *st = t;
                float ms;
                int r = measure(s, &ms);
                if (r == VIE_ERR_ARG) { ctx->err.code = VIE_OK; continue; }
                if (r) { rc = r; goto done; }
                s.ms = ms;
                if (ms < bestg_ms) { bestg_ms = ms; bestg = s; }
            }
            cands.push_back(bestg);
        }
        for (Sched& s : cands) {
            if (s.ms == 0.f) {
                int r = measure(s, &s.ms);
                if (r) { rc = r; goto done; }
            }
            if (s.ms < best.ms) best = s;
        }
        (void)tile;
    }
    {
        std::ostringstream o;
        o << (dbl ? "fp64" : "fp32") << " " << best.ms << " ms:";
        const char* nm[3] = {"x", "y", "z"};
        const int tl[3] = {best.t.tx, best.t.tc, best.t.tz};
        for (int ax = 0; ax < 3; ax++) {
            o << ' ' << nm[ax] << '=';
            if (best.t.fast[ax] == 1 || (best.t.fast[ax] < 0 && fast_length(n[ax])))
                o << "fast" << (ax == 0 && best.t.xalt ? "/half-tile" : "") << (ax == 1 && best.t.ytma ? "/tma" : "");
            else o << "generic[" << plan_str(best.plan[ax]) << "]/t" << tl[ax];
        }
        report = o.str();
    }
done:
    cudaFree(x);
    cudaFree(y);
    return rc;
}

// rebuild an operator with a schedule and restore its Green octant and contrast
template <typename T> int rebuild(vie_ctx* ctx, Operator<T>& op, const Sched& s) {
    int rc = op.init(ctx->nx, ctx->ny, ctx->nz, ctx->d, ctx->k0, s.t, s.plan, ctx->d_flags, ctx->err);
    if (!rc && ctx->have_green) rc = op.set_green(ctx->d_green, ctx->k0, ctx->stream, ctx->err);
    if (!rc && ctx->have_eps) rc = op.set_contrast(ctx->w_host.data(), ctx->stream, ctx->err);
    if (!rc) VIE_CUDA_TRY(cudaStreamSynchronize(ctx->stream), ctx->err);
    return rc;
}

}  // namespace

// the cached schedules of this grid, if the process has them
void tune_apply_cached(vie_ctx* ctx) {
    std::lock_guard<std::mutex> lk(g_mu);
    load_file_locked();
    auto it = g_cache.find(cache_key(ctx->device, ctx->nx, ctx->ny, ctx->nz, 16));
    if (it != g_cache.end()) {
        ctx->sched64 = it->second.t;
        for (int ax = 0; ax < 3; ax++) ctx->plans64[ax] = it->second.plan[ax];
    }
    it = g_cache.find(cache_key(ctx->device, ctx->nx, ctx->ny, ctx->nz, 8));
    if (it != g_cache.end()) {
        ctx->sched32 = it->second.t;
        for (int ax = 0; ax < 3; ax++) ctx->plans32[ax] = it->second.plan[ax];
    }
}

// flags: 1 FP64, 2 FP32 (0: both), 4 tune again even if cached
int autotune_driver(vie_ctx* ctx, int flags) {
    const int which = (flags & 3) ? (flags & 3) : 3;
    std::string rep;
    for (int prec : {1, 2}) {
        if (!(which & prec)) continue;
        const int bytes = prec == 1 ? 16 : 8;
        const std::string key = cache_key(ctx->device, ctx->nx, ctx->ny, ctx->nz, bytes);
        Sched s;
        bool cached = false;
        {
            std::lock_guard<std::mutex> lk(g_mu);
            load_file_locked();
            auto it = g_cache.find(key);
            if (it != g_cache.end() && !(flags & 4)) {
                s = it->second;
                cached = true;
            }
        }
        std::string r;
        int rc = VIE_OK;
        if (!cached) {
            s.t = prec == 1 ? ctx->sched64 : ctx->sched32;
            for (int ax = 0; ax < 3; ax++) s.plan[ax] = prec == 1 ? ctx->plans64[ax] : ctx->plans32[ax];
            rc = prec == 1 ? tune_one<double>(ctx, ctx->op64, s, r) : tune_one<float>(ctx, ctx->op32, s, r);
            if (rc) return rc;
            std::lock_guard<std::mutex> lk(g_mu);
            store_locked(key, s);
        } else {
            r = std::string(prec == 1 ? "fp64" : "fp32") + " cached " + serialize(key, s);
        }
        if (prec == 1) {
            ctx->sched64 = s.t;
            for (int ax = 0; ax < 3; ax++) ctx->plans64[ax] = s.plan[ax];
            rc = rebuild<double>(ctx, ctx->op64, s);
        } else {
            ctx->sched32 = s.t;
            for (int ax = 0; ax < 3; ax++) ctx->plans32[ax] = s.plan[ax];
            rc = rebuild<float>(ctx, ctx->op32, s);
        }
        if (rc) return rc;
        rep += (rep.empty() ? "" : "; ") + r;
    }
    ctx->tune_report = rep;
    return VIE_OK;
}

}  // namespace vie
