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

int demsph_device_alloc(void** ptr, size_t bytes, void* stream) {
    return demsph::guarded([&] {
        if (!ptr) throw demsph::Status(DEMSPH_ERR_INVALID, "null output pointer");
        *ptr = nullptr;
        if (bytes == 0) return;
        DEMSPH_CUDA(cudaMallocAsync(ptr, bytes, (cudaStream_t)stream));
    });
}

int demsph_device_free(void* ptr, void* stream) {
    return demsph::guarded([&] {
        if (ptr) DEMSPH_CUDA(cudaFreeAsync(ptr, (cudaStream_t)stream));
    });
}

int demsph_memcpy(void* dst, const void* src, size_t bytes, int kind, void* stream) {
    return demsph::guarded([&] {
        if (bytes == 0) return;
        if (!dst || !src) throw demsph::Status(DEMSPH_ERR_INVALID, "null pointer");
        cudaMemcpyKind k = kind == 0 ? cudaMemcpyHostToDevice
                                     : (kind == 1 ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice);
        if (kind < 0 || kind > 2) throw demsph::Status(DEMSPH_ERR_INVALID, "memcpy kind must be 0, 1 or 2");
        DEMSPH_CUDA(cudaMemcpyAsync(dst, src, bytes, k, (cudaStream_t)stream));
        DEMSPH_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    });
}

}  // extern "C"
