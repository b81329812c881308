// Library-wide C ABI entry points: version, last error, launch counter.
#include <atomic>
#include <string>

#include "common.cuh"

namespace demsph {

std::atomic<long long> g_launches{0};
static thread_local std::string t_last_error;

void set_last_error(const std::string& s) { t_last_error = s; }

}  // namespace demsph

extern "C" {

const char* demsph_last_error(void) { return demsph::t_last_error.c_str(); }
const char* demsph_version(void) { return "demsph-b200 0.1 (sm_100a)"; }
long long demsph_kernel_launches(void) { return demsph::g_launches.load(); }

int demsph_retain_device_memory(unsigned long long bytes) {
    return demsph::guarded([&] {
        int dev = 0;
        DEMSPH_CUDA(cudaGetDevice(&dev));
        cudaMemPool_t pool;
        DEMSPH_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
        unsigned long long v = bytes;  // the attribute is a 64-bit unsigned value
        DEMSPH_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &v));
    });
}

}  // extern "C"
