// Library-wide C ABI entry points: version, last error, launch counter.
#include <atomic>
#include <mutex>
#include <set>
#include <string>

#include "common.cuh"

namespace demsph {

std::atomic<long long> g_launches{0};
static thread_local std::string t_last_error;

void set_last_error(const std::string& s) { t_last_error = s; }

// Devices whose pool retention is settled (by default or by the caller).
static std::mutex g_pool_m;
static std::set<int> g_pool_set;
constexpr unsigned long long kDefaultRetainBytes = 8ull << 30;

static void set_retention(int dev, unsigned long long bytes) {
    cudaMemPool_t pool;
    DEMSPH_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
    unsigned long long v = bytes;  // the attribute is a 64-bit unsigned value
    DEMSPH_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &v));
}

// A tuning setting: without a device (scenes built on the host only) or
// when the pool refuses, the stock behaviour stays and nothing is reported.
void default_pool_retention() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        (void)cudaGetLastError();
        return;
    }
    std::lock_guard<std::mutex> lk(g_pool_m);
    if (!g_pool_set.insert(dev).second) return;
    cudaMemPool_t pool;
    unsigned long long v = kDefaultRetainBytes;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess ||
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &v) != cudaSuccess)
        (void)cudaGetLastError();
}

}  // namespace demsph

extern "C" {

const char* demsph_last_error(void) { return demsph::t_last_error.c_str(); }
const char* demsph_version(void) { return "demsph-b200 0.1 (sm_100a)"; }
long long demsph_kernel_launches(void) { return demsph::g_launches.load(); }

int demsph_retain_device_memory(unsigned long long bytes) {
    return demsph::guarded([&] {
        int dev = 0;
        DEMSPH_CUDA(cudaGetDevice(&dev));
        std::lock_guard<std::mutex> lk(demsph::g_pool_m);
        demsph::g_pool_set.insert(dev);  // the caller's choice stands
        demsph::set_retention(dev, bytes);
    });
}

}  // extern "C"
