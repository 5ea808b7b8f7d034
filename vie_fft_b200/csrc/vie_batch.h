// vie_batch.h -- the persistent multi-instance loop of batched mixed-precision
// BiCGSTAB solves (vie_solve_batch), host side.
#pragma once
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "vie_internal.h"

namespace vie {

// One instance of a batch after its set-up (solve_bicgstab_mixed with a plan):
// the device vectors, scalars, reduction partials and control block of its
// context, and copies of its two operators' device views.
struct FusedInstance {
    vie_ctx* ctx = nullptr;
    OpDev<float2> op32{};
    OpDev<double2> op64{};
    long long a = 0;
    float2 *r = nullptr, *p = nullptr, *v = nullptr, *sv = nullptr, *t = nullptr, *x32 = nullptr, *b32 = nullptr;
    double2 *r64 = nullptr, *b64 = nullptr, *x64 = nullptr;
    double2* S = nullptr;
    double2* partial = nullptr;
    KCtl* ctl = nullptr;
    double2* hist = nullptr;
};

inline int sms_of_device() {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1) n = 1;
    return n;
}
// blocks of a persistent kernel on the current device: as many as fit on every
// SM at once (one wave)
template <typename K> int persistent_grid(K kernel, int threads, size_t smem) {
    static std::mutex mu;
    static std::map<std::tuple<const void*, int, int, size_t>, int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    const auto key = std::make_tuple(reinterpret_cast<const void*>(kernel), dev, threads, smem);
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(key);
    if (it == cache.end()) {
        int nb = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, threads, smem) != cudaSuccess || nb < 1) nb = 1;
        it = cache.emplace(key, nb * sms_of_device()).first;
    }
    return it->second;
}

// both operators of the context run every axis on the register kernels
bool batch_fused_eligible(const vie_ctx* ctx);

// Runs the iterations of every instance to its own stop in one graph launch on
// stream S.  launched is false when the graph could not be built (nothing ran).
// Each instance's control block holds its outcome afterwards.
int batch_fused_loop(std::vector<FusedInstance>& inst, cudaStream_t S, vie_ctx* ectx, bool& launched);

}  // namespace vie
