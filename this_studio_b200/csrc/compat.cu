// The reference's sort / scan launchers with their exact C signatures
// (DEMSPH/kernel/buildHashStartEnd.cuh:5-19), so code written against the
// reference's C ABI links against this library unchanged.  Behaviour follows
// DEMSPH/kernel/buildHashStartEnd.cu:
//   buildHashStartEnd  hashIndex[i] = i; stable sort of (hashValue, hashIndex)
//                      by hashValue (ascending, in place); for every sorted
//                      position with 0 <= h < startEndSize, start[h] = first
//                      position of key h, end[h] = last + 1.  Entries of
//                      start / end for absent keys are left untouched, as in
//                      the reference (the callers memset them to -1).
//   buildPrefixSum     inclusive scan of count[0..size) into prefixSum.
// The grid / block arguments are accepted and ignored: launch geometry is
// chosen here.  Like the reference these return void; a failure is recorded
// for demsph_last_error().
#include <atomic>
#include <climits>

#include "radix.cuh"

namespace demsph {

extern std::atomic<long long> g_launches;

// setHashIndex (buildHashStartEnd.cu:6-12) + the order-preserving map of the
// int32 keys onto uint32 (flip the sign bit) for the radix sort.
static __global__ void k_hb_prep(const int* __restrict__ hashValue, int n, unsigned* __restrict__ keys,
                                 int* __restrict__ hashIndex) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    keys[i] = (unsigned)hashValue[i] ^ 0x80000000u;
    hashIndex[i] = i;
}

// Writes the sorted keys back and runs findStartAndEnd (buildHashStartEnd.cu:14-34).
static __global__ void k_hb_finish(const unsigned* __restrict__ keys, int n, int startEndSize, int* __restrict__ hashValue,
                                   int* __restrict__ start, int* __restrict__ end) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int h = (int)(keys[i] ^ 0x80000000u);
    hashValue[i] = h;
    if (h < 0 || h >= startEndSize) return;
    if (i == 0 || (int)(keys[i - 1] ^ 0x80000000u) != h) start[h] = i;
    if (i == n - 1 || (int)(keys[i + 1] ^ 0x80000000u) != h) end[h] = i + 1;
}

// Words of scratch buildHashStartEnd needs for n keys: the radix sort's plus
// one key array.
static constexpr size_t hash_sort_scratch_words(int n) { return rx_scratch_words(n) + (size_t)n + 64; }

// The sort behind buildHashStartEnd on caller-provided scratch (words from
// hash_sort_scratch_words).
void hash_sort_start_end(int* start, int* end, int* hashIndex, int* hashValue, int startEndSize, int n, int* scratch,
                         cudaStream_t s) {
    if (n <= 0) return;
    unsigned* keys = (unsigned*)scratch;
    RadixScratch rs = rx_carve(scratch + n + 32, n);
    k_hb_prep<<<grid_for(n, 256), 256, 0, s>>>(hashValue, n, keys, hashIndex);
    int launches = 2 + rx_sort(keys, hashIndex, n, 32, rs, s);
    k_hb_finish<<<grid_for(n, 256), 256, 0, s>>>(keys, n, startEndSize, hashValue, start, end);
    g_launches += launches;
    DEMSPH_LAUNCH_CHECK();
}

// ------------------------------------------------ non-allocating variant --
// Scratch for demsph_build_hash_start_end_noalloc: one fixed array in the
// module image, sized for DEMSPH_NOALLOC_MAX_KEYS keys (3.3 MB).  Each GPU that
// loads the library holds it until the process exits.  Every word a call
// reads is written earlier in the same call (histograms, scan tiles and key
// buffers are fully overwritten), so nothing needs clearing between calls;
// calls that overlap on the GPU share it and race.
static __device__ __align__(256) int g_hash_sort_scratch[hash_sort_scratch_words(DEMSPH_NOALLOC_MAX_KEYS)];

// Device address of the array on the current device.  Host code cannot use
// the symbol itself (in host code it names a host-side stand-in), so the
// address is looked up on every call: the lookup is cheap after the first
// one on a device (which may load the module), and a cached pointer would go
// stale if the device's primary context were reset and the module reloaded.
static int* noalloc_scratch() {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_hash_sort_scratch);
    if (e != cudaSuccess) throw CudaError(e, "cudaGetSymbolAddress of the sort scratch array failed");
    return (int*)p;
}

}  // namespace demsph

using namespace demsph;

extern "C" {

void buildHashStartEnd(int* start, int* end, int* hashIndex, int* hashValue, const size_t startEndSize,
                       const size_t hashListSize, const size_t gridD_GPU, const size_t blockD_GPU,
                       cudaStream_t stream_GPU) {
    (void)gridD_GPU;
    (void)blockD_GPU;
    guarded([&] {
        if (hashListSize == 0) return;
        if (hashListSize > (size_t)(1 << 30) || startEndSize > (size_t)0x7fffffff)
            throw Status(DEMSPH_ERR_INVALID, "buildHashStartEnd: sizes exceed the int32 range");
        int n = (int)hashListSize;
        int* scratch = nullptr;
        DEMSPH_CUDA(cudaMallocAsync((void**)&scratch, hash_sort_scratch_words(n) * sizeof(int), stream_GPU));
        hash_sort_start_end(start, end, hashIndex, hashValue, (int)startEndSize, n, scratch, stream_GPU);
        DEMSPH_CUDA(cudaFreeAsync(scratch, stream_GPU));
    });
}

int demsph_build_hash_start_end_noalloc(int* start, int* end, int* hashIndex, int* hashValue, size_t startEndSize,
                                        size_t hashListSize, cudaStream_t stream) {
    return guarded([&] {
        if (hashListSize == 0) return;
        if (hashListSize > (size_t)DEMSPH_NOALLOC_MAX_KEYS)
            throw Status(DEMSPH_ERR_INVALID, "demsph_build_hash_start_end_noalloc: " + std::to_string(hashListSize) +
                                                 " keys exceed the fixed scratch for " +
                                                 std::to_string(DEMSPH_NOALLOC_MAX_KEYS) + " keys");
        if (startEndSize > (size_t)INT_MAX) throw Status(DEMSPH_ERR_INVALID, "startEndSize exceeds the int32 range");
        int* scratch = noalloc_scratch();
        hash_sort_start_end(start, end, hashIndex, hashValue, (int)startEndSize, (int)hashListSize, scratch, stream);
    });
}

void buildPrefixSum(int* prefixSum, int* count, const size_t size, cudaStream_t stream) {
    guarded([&] {
        if (size == 0) return;
        if (size > (size_t)4096 * 4096) throw Status(DEMSPH_ERR_INVALID, "buildPrefixSum: size above 16,777,216");
        int n = (int)size;
        int nt = (n + 4095) / 4096;
        int* scratch = nullptr;
        if (nt > 1) DEMSPH_CUDA(cudaMallocAsync((void**)&scratch, (2 * (size_t)nt + 2) * sizeof(int), stream));
        g_launches += rx_scan(count, prefixSum, n, scratch, scratch ? scratch + nt : nullptr, 1, stream);
        DEMSPH_LAUNCH_CHECK();
        if (scratch) DEMSPH_CUDA(cudaFreeAsync(scratch, stream));
    });
}

}  // extern "C"
