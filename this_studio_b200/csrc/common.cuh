// Shared device math, status codes and device-buffer ownership for the
// DEMSPH B200 library.
#pragma once
#include <cstring>
#include <mutex>
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>
#include <memory>
#include <thread>
#include <atomic>
#include <condition_variable>
#include <deque>
#include <pthread.h>
#include <utility>
#include <algorithm>

#include "../../include/demsph.h"

namespace demsph {

// ----------------------------------------------------------------- errors --
struct CudaError : std::runtime_error {
    cudaError_t code;
    CudaError(cudaError_t c, const char* what) : std::runtime_error(what), code(c) {}
};
struct Status : std::runtime_error {
    int code;
    Status(int c, const std::string& what) : std::runtime_error(what), code(c) {}
};

#define DEMSPH_CUDA(call)                                                                  \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            char b_[512];                                                                  \
            snprintf(b_, sizeof b_, "%s:%d %s: %s", __FILE__, __LINE__, #call,             \
                     cudaGetErrorString(e_));                                              \
            throw ::demsph::CudaError(e_, b_);                                             \
        }                                                                                  \
    } while (0)

#define DEMSPH_LAUNCH_CHECK() DEMSPH_CUDA(cudaGetLastError())

// Last error text, per thread, readable through demsph_last_error().
void set_last_error(const std::string& s);

// Runs f, converting exceptions into the C-ABI status convention.
template <class F>
static inline int guarded(F&& f) {
    try {
        f();
        return DEMSPH_OK;
    } catch (const Status& s) {
        set_last_error(s.what());
        return s.code;
    } catch (const CudaError& e) {
        set_last_error(e.what());
        return DEMSPH_ERR_CUDA;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return DEMSPH_ERR_ALLOC;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return DEMSPH_ERR_INVALID;
    }
}

// ---------------------------------------------------------- device buffer --
// Owns a device allocation made with cudaMallocAsync on the owner's stream.
// std::allocator that leaves trivially constructible elements uninitialised
// on resize, so host staging arrays are first touched by the (parallel) code
// that fills them rather than by a serial zero fill.
template <class T>
struct DefaultInitAlloc : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = DefaultInitAlloc<U>;
    };
    DefaultInitAlloc() = default;
    template <class U>
    DefaultInitAlloc(const DefaultInitAlloc<U>&) {}
    template <class U>
    void construct(U* p) {
        ::new ((void*)p) U;
    }
    template <class U, class... Args>
    void construct(U* p, Args&&... args) {
        ::new ((void*)p) U(std::forward<Args>(args)...);
    }
};
template <class T>
using HostVec = std::vector<T, DefaultInitAlloc<T>>;

// Host worker threads kept for the life of the process.  host_parallel hands
// its chunks to them instead of starting threads per call: starting and
// joining a thread costs tens of microseconds, and a scene's set-up and
// read-back make dozens of parallel calls.  Several callers may submit at
// once; a caller runs chunks of its own job until none is left and then
// waits for the chunks the workers took, so every job completes, also one
// submitted from inside a chunk (a worker that waits there runs its own
// job's chunks first).  The pool is never destroyed (no join at exit); a
// child process made by fork() starts its own on first use (the parent's
// workers do not exist there, and its lock may have been held at the fork).
class HostPool {
  public:
    static HostPool& get() {
        static std::atomic<HostPool*> cur{nullptr};
        static std::once_flag hook;
        std::call_once(hook, [] { pthread_atfork(nullptr, nullptr, [] { cur.store(nullptr); }); });
        HostPool* p = cur.load();
        if (!p) {
            static std::mutex make;
            std::lock_guard<std::mutex> lk(make);
            p = cur.load();
            if (!p) {
                p = new HostPool();
                cur.store(p);
            }
        }
        return *p;
    }
    // f(i) for every i in [0, k), on the workers and the calling thread.
    template <class F>
    void run(int k, F& f) {
        Job j;
        j.k = k;
        j.ctx = &f;
        j.call = [](void* c, int i) { (*static_cast<F*>(c))(i); };
        {
            std::lock_guard<std::mutex> lk(m_);
            q_.push_back(&j);
        }
        work_.notify_all();
        for (int i = j.next.fetch_add(1); i < k; i = j.next.fetch_add(1)) {
            j.call(j.ctx, i);
            j.done.fetch_add(1, std::memory_order_acq_rel);
        }
        std::unique_lock<std::mutex> lk(m_);
        auto it = std::find(q_.begin(), q_.end(), &j);
        if (it != q_.end()) q_.erase(it);
        done_.wait(lk, [&] { return j.done.load(std::memory_order_acquire) == k; });
    }

  private:
    struct Job {
        int k = 0;
        std::atomic<int> next{0}, done{0};
        void* ctx = nullptr;
        void (*call)(void*, int) = nullptr;
    };
    HostPool() {
        const unsigned hw = std::thread::hardware_concurrency();
        const int workers = (int)std::min(7u, hw > 1 ? hw - 1 : 1u);
        for (int t = 0; t < workers; t++) std::thread([this] { loop(); }).detach();
    }
    void loop() {
        for (;;) {
            Job* j = nullptr;
            int i = 0;
            {
                std::unique_lock<std::mutex> lk(m_);
                work_.wait(lk, [&] { return !q_.empty(); });
                j = q_.front();
                i = j->next.fetch_add(1);
                if (i >= j->k) {  // every chunk of the front job is taken
                    q_.pop_front();
                    continue;
                }
            }
            j->call(j->ctx, i);
            // after this increment the job may be gone: only the pool is touched
            j->done.fetch_add(1, std::memory_order_acq_rel);
            std::lock_guard<std::mutex> lk(m_);
            done_.notify_all();
        }
    }
    std::mutex m_;
    std::condition_variable work_, done_;
    std::deque<Job*> q_;
};

// Runs f(begin, end) over [0, n) in up to `threads` chunks on the host pool
// (one, on the calling thread, when n is small).
template <class F>
static void host_parallel(long n, F&& f, int threads = 8) {
    const long minChunk = 32768;
    int k = (int)std::min<long>(threads, std::max<long>(1, n / minChunk));
    if (k <= 1) {
        f(0L, n);
        return;
    }
    const long step = (n + k - 1) / k;
    auto chunk = [&](int t) {
        const long b = t * step, e = std::min(n, b + step);
        if (b < e) f(b, e);
    };
    HostPool::get().run(k, chunk);
}

// Many device-to-device copies in one launch: a scene's snapshot is some
// forty buffers, and one copy call each costs a few microseconds of launch
// latency on the stream even when the buffers are small.  Buffers are the
// library's own allocations (256-byte aligned), copied in 16-byte words; a
// copy's last partial word goes byte by byte.  Buffers of kCopyKernelMax bytes
// or more still go to the copy engines (cudaMemcpyAsync): there the call's
// latency is small beside the transfer, and the engines leave the SMs to
// whatever else runs (a kernel copy of a large batch scene's snapshot took SMs
// from the scene stepped beside it).
constexpr int kCopyMax = 48;
constexpr size_t kCopyKernelMax = (size_t)1 << 20;
struct CopyList {
    const char* src[kCopyMax];
    char* dst[kCopyMax];
    unsigned long long bytes[kCopyMax];
    unsigned long long first[kCopyMax + 1];  // first 16-byte word of each copy
    int n;
};
static __global__ void k_copy_list(CopyList c) {
    const unsigned long long total = c.first[c.n];
    for (unsigned long long w = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; w < total;
         w += (unsigned long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = c.n - 1;
        while (lo < hi) {  // the last copy whose first word is <= w
            const int mid = (lo + hi + 1) >> 1;
            if (c.first[mid] <= w) lo = mid;
            else hi = mid - 1;
        }
        const unsigned long long o = (w - c.first[lo]) * 16;
        const unsigned long long len = c.bytes[lo] - o;
        if (len >= 16) {
            *reinterpret_cast<int4*>(c.dst[lo] + o) = *reinterpret_cast<const int4*>(c.src[lo] + o);
        } else {
            for (unsigned long long b = 0; b < len; b++) c.dst[lo][o + b] = c.src[lo][o + b];
        }
    }
}
struct CopyItem {
    void* dst;
    const void* src;
    size_t bytes;
};
// Issues the copies on stream s: the small ones kCopyMax per kernel launch,
// the large ones as copy-engine transfers.  Returns the kernel launches.
static inline int copy_list(const std::vector<CopyItem>& items, cudaStream_t s) {
    int launches = 0;
    CopyList c{};
    auto flush = [&] {
        if (c.n == 0) return;
        const unsigned long long words = c.first[c.n];
        const unsigned grid = (unsigned)std::min<unsigned long long>((words + 255) / 256, 148ull * 8);
        k_copy_list<<<grid, 256, 0, s>>>(c);
        launches++;
        c = CopyList{};
    };
    for (const CopyItem& it : items) {
        if (it.bytes == 0) continue;
        if (it.bytes >= kCopyKernelMax) {
            DEMSPH_CUDA(cudaMemcpyAsync(it.dst, it.src, it.bytes, cudaMemcpyDeviceToDevice, s));
            continue;
        }
        c.src[c.n] = (const char*)it.src;
        c.dst[c.n] = (char*)it.dst;
        c.bytes[c.n] = it.bytes;
        c.first[c.n + 1] = c.first[c.n] + (it.bytes + 15) / 16;
        c.n++;
        if (c.n == kCopyMax) flush();
    }
    flush();
    return launches;
}

// Process-wide page-locked staging for bulk host <-> device copies of scene
// records: copies from (or to) pageable memory run at a fraction of the
// link's speed, so the records are copied into this buffer by several host
// threads and moved by one DMA.  Grown on demand and kept; one user at a
// time (lock() while filling, copying and waiting for the copy).
struct PinnedStage {
    std::mutex m;
    char* p = nullptr;
    size_t n = 0;
    static PinnedStage& get() {
        static PinnedStage s;
        return s;
    }
    // A buffer of at least `bytes`; call with m held.
    char* reserve(size_t bytes) {
        if (n < bytes) {
            if (p) cudaFreeHost(p);
            p = nullptr;
            n = 0;
            const size_t want = bytes + bytes / 4;
            if (cudaHostAlloc((void**)&p, want, cudaHostAllocDefault) != cudaSuccess) {
                (void)cudaGetLastError();
                p = nullptr;
                return nullptr;  // the caller copies from pageable memory instead
            }
            n = want;
        }
        return p;
    }
};
// memcpy of `bytes` in up to 8 host threads (one below 64 KB).
static inline void host_copy(void* dst, const void* src, size_t bytes) {
    host_parallel((long)bytes, [&](long a, long b) {
        if (b > a) std::memcpy((char*)dst + a, (const char*)src + a, (size_t)(b - a));
    });
}

template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaStream_t s = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    void release() {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count, cudaStream_t stream, bool zero = true) {
        release();
        s = stream;
        n = count;
        if (count == 0) return;
        DEMSPH_CUDA(cudaMallocAsync((void**)&p, count * sizeof(T), stream));
        if (zero) DEMSPH_CUDA(cudaMemsetAsync(p, 0, count * sizeof(T), stream));
    }
    // Grows to at least count elements, keeping the first n elements.
    void grow(size_t count, cudaStream_t stream) {
        if (count <= n) return;
        T* q = nullptr;
        DEMSPH_CUDA(cudaMallocAsync((void**)&q, count * sizeof(T), stream));
        DEMSPH_CUDA(cudaMemsetAsync(q, 0, count * sizeof(T), stream));
        if (p && n) DEMSPH_CUDA(cudaMemcpyAsync(q, p, n * sizeof(T), cudaMemcpyDeviceToDevice, stream));
        if (p) cudaFreeAsync(p, s);
        p = q;
        n = count;
        s = stream;
    }
    template <class A>
    void upload(const std::vector<T, A>& h, cudaStream_t stream) {
        alloc(h.size(), stream, false);
        if (!h.empty()) DEMSPH_CUDA(cudaMemcpyAsync(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, stream));
    }
    void download(std::vector<T>& h, cudaStream_t stream) const {
        h.resize(n);
        if (n) DEMSPH_CUDA(cudaMemcpyAsync(h.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost, stream));
    }
    size_t bytes() const { return n * sizeof(T); }
};

static inline unsigned grid_for(size_t n, unsigned block) { return (unsigned)((n + block - 1) / block); }

// Chained launches (programmatic dependent launch): a kernel launched with
// launch_chained may be scheduled while the kernel before it on the stream
// is still draining, so its launch and block dispatch overlap that kernel's
// tail instead of following its completion.  Such a kernel calls
// chain_enter() first, before any access to global memory and before any
// early return: griddepcontrol.wait returns once every kernel it depends on
// has completed and its writes are visible, and since every block of every
// chained kernel waits there, each chained kernel completes after the one
// before it, so the ordering stays transitive along the stream.
// griddepcontrol.launch_dependents then lets the next chained kernel be
// scheduled as soon as every block of this one has started.  Launched
// without the attribute (chain = false), such a kernel runs after the one
// before it as usual and its wait returns at once.
__device__ __forceinline__ void chain_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
template <class... P, class... A>
inline void launch_chained(void (*kernel)(P...), unsigned grid, unsigned block, cudaStream_t s, bool chain,
                           A&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = chain ? 1 : 0;
    DEMSPH_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...));
}
// Keeps up to 8 GiB of freed memory in the current device's default pool,
// once per device, unless the caller set a limit (demsph_retain_device_memory).
void default_pool_retention();
// SMs of the current device (asked once per device and host thread).
static inline int device_sms() {
    thread_local int dev = -1, sms = 1;
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess) return sms;
    if (d != dev && cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d) == cudaSuccess) dev = d;
    return sms > 0 ? sms : 1;
}

// Zero-fill as a kernel: inside captured step loops every node is a kernel,
// so a pooled graph of the same shape can be updated to another scene's
// sizes (memset nodes cannot change their size in an update).
static __global__ void k_zero_ints(int* __restrict__ a, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = 0;
}

// ------------------------------------------------------------ vector math --
// double3 algebra in the form the reference uses (myVec.h:25-176).
__host__ __device__ __forceinline__ double3 mk3(double x, double y, double z) { return make_double3(x, y, z); }
__host__ __device__ __forceinline__ double3 operator+(double3 a, double3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ __forceinline__ double3 operator-(double3 a, double3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ __forceinline__ double3 operator-(double3 a) { return mk3(-a.x, -a.y, -a.z); }
__host__ __device__ __forceinline__ double3 operator*(double3 a, double s) { return mk3(a.x * s, a.y * s, a.z * s); }
__host__ __device__ __forceinline__ double3 operator*(double s, double3 a) { return mk3(a.x * s, a.y * s, a.z * s); }
__host__ __device__ __forceinline__ double3 operator/(double3 a, double s) { double i = 1.0 / s; return mk3(a.x * i, a.y * i, a.z * i); }
__host__ __device__ __forceinline__ double3& operator+=(double3& a, double3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
__host__ __device__ __forceinline__ double3& operator-=(double3& a, double3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; return a; }
__host__ __device__ __forceinline__ double3& operator*=(double3& a, double s) { a.x *= s; a.y *= s; a.z *= s; return a; }
__host__ __device__ __forceinline__ double dot(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ double3 cross(double3 a, double3 b) {
    return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__host__ __device__ __forceinline__ double len2(double3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
__host__ __device__ __forceinline__ double len(double3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
__host__ __device__ __forceinline__ double3 normalize(double3 v) {
    double l2 = v.x * v.x + v.y * v.y + v.z * v.z;
    if (l2 < 1.0e-20) return mk3(0, 0, 0);
    double inv = 1.0 / sqrt(l2);
    return mk3(v.x * inv, v.y * inv, v.z * inv);
}
__host__ __device__ __forceinline__ double3 xyz(double4 a) { return mk3(a.x, a.y, a.z); }
__host__ __device__ __forceinline__ double4 d4(double3 a, double w) { return make_double4(a.x, a.y, a.z, w); }

// float3 algebra for the mixed-precision force laws.
__host__ __device__ __forceinline__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ __forceinline__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ __forceinline__ float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
__host__ __device__ __forceinline__ float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__host__ __device__ __forceinline__ float3 operator*(float s, float3 a) { return make_float3(a.x * s, a.y * s, a.z * s); }
__host__ __device__ __forceinline__ float3& operator+=(float3& a, float3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
__host__ __device__ __forceinline__ float3& operator-=(float3& a, float3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; return a; }
__host__ __device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ float3 cross(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__host__ __device__ __forceinline__ float len(float3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }

// Precision traits: V<double> = double3, V<float> = float3.
template <class R> struct VecOf;
template <> struct VecOf<double> { using T = double3; };
template <> struct VecOf<float> { using T = float3; };
template <class R> using V = typename VecOf<R>::T;

template <class R> __host__ __device__ __forceinline__ V<R> cvt(double3 a);
template <> __host__ __device__ __forceinline__ double3 cvt<double>(double3 a) { return a; }
template <> __host__ __device__ __forceinline__ float3 cvt<float>(double3 a) { return make_float3((float)a.x, (float)a.y, (float)a.z); }
__host__ __device__ __forceinline__ double3 up(double3 a) { return a; }
__host__ __device__ __forceinline__ double3 up(float3 a) { return mk3(a.x, a.y, a.z); }
template <class R> __host__ __device__ __forceinline__ V<R> v3r(R x, R y, R z);
template <> __host__ __device__ __forceinline__ double3 v3r<double>(double x, double y, double z) { return mk3(x, y, z); }
template <> __host__ __device__ __forceinline__ float3 v3r<float>(float x, float y, float z) { return make_float3(x, y, z); }
__host__ __device__ __forceinline__ double rsq(double x) { return sqrt(x); }
__host__ __device__ __forceinline__ float rsq(float x) { return sqrtf(x); }
__host__ __device__ __forceinline__ double rlen(double3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
__host__ __device__ __forceinline__ float rlen(float3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }

static constexpr double kPi = 3.14159265358979323846;

// ----------------------------------------------------------------- grid ---
// spatialGrid (DEMSPH/kernel/boundary.h:70-94): cells of at least the
// requested size tiling [mn, mx); keys z*ny*nx + y*nx + x.
struct GridDesc {
    double3 mn, mx, cs;
    int nx, ny, nz;
    int ncell() const { return nx * ny * nz; }
};
static inline bool grid_set(GridDesc& g, double3 mn, double3 mx, double cell) {
    if (mx.x <= mn.x || mx.y <= mn.y || mx.z <= mn.z || cell < 1.e-20) return false;
    g.mn = mn;
    g.mx = mx;
    double3 d = mx - mn;
    g.nx = d.x > cell ? int(d.x / cell) : 1;
    g.ny = d.y > cell ? int(d.y / cell) : 1;
    g.nz = d.z > cell ? int(d.z / cell) : 1;
    g.cs = mk3(d.x / double(g.nx), d.y / double(g.ny), d.z / double(g.nz));
    return true;
}
// calculateGridPosition (neighborSearchKernel.cuh:4-9): truncation toward zero.
__host__ __device__ __forceinline__ int3 cell_of(double3 p, const GridDesc& g) {
    return make_int3(int((p.x - g.mn.x) / g.cs.x), int((p.y - g.mn.y) / g.cs.y), int((p.z - g.mn.z) / g.cs.z));
}
__host__ __device__ __forceinline__ int key_of(int3 c, const GridDesc& g) { return c.z * g.ny * g.nx + c.y * g.nx + c.x; }
// calculateHash kernel (neighborSearchKernel.cu:6-27): clamp into the domain first.
__host__ __device__ __forceinline__ int clamped_key(double3 p, const GridDesc& g) {
    if (p.x < g.mn.x) p.x = g.mn.x; else if (p.x >= g.mx.x) p.x = g.mx.x - 0.5 * g.cs.x;
    if (p.y < g.mn.y) p.y = g.mn.y; else if (p.y >= g.mx.y) p.y = g.mx.y - 0.5 * g.cs.y;
    if (p.z < g.mn.z) p.z = g.mn.z; else if (p.z >= g.mx.z) p.z = g.mx.z - 0.5 * g.cs.z;
    int3 c = cell_of(p, g);
    // A coordinate within an ulp below the max face can round up to index n
    // (and NaN converts to an arbitrary int); keep the key inside the table.
    c.x = c.x < 0 ? 0 : (c.x > g.nx - 1 ? g.nx - 1 : c.x);
    c.y = c.y < 0 ? 0 : (c.y > g.ny - 1 ? g.ny - 1 : c.y);
    c.z = c.z < 0 ? 0 : (c.z > g.nz - 1 ? g.nz - 1 : c.z);
    return key_of(c, g);
}
// The 27-cell stencil with the reference's index clamping
// (ballNeighborSearchKernel.cu:25-46).  The three x-neighbours of a row are
// consecutive keys, so each (y, z) row is ONE contiguous range of the
// cell-sorted index list: nine ranges instead of 27 lookups, visited in the
// reference's (z, y, x) order.
struct Stencil {
    int3 c, s, e;
};
__device__ __forceinline__ Stencil stencil_of_cell3(int3 c, const GridDesc& g);
__device__ __forceinline__ Stencil stencil_of(double3 p, const GridDesc& g) { return stencil_of_cell3(cell_of(p, g), g); }
// The stencil of cell `key` (the cell an object was sorted into, wherever it
// has moved since).
__device__ __forceinline__ Stencil stencil_of_cell(int key, const GridDesc& g) {
    return stencil_of_cell3(make_int3(key % g.nx, (key / g.nx) % g.ny, key / (g.nx * g.ny)), g);
}
__device__ __forceinline__ Stencil stencil_of_cell3(int3 c, const GridDesc& g) {
    Stencil st;
    st.c = c;
    st.s = make_int3(-1, -1, -1);
    st.e = make_int3(1, 1, 1);
    if (st.c.x <= 0) { st.c.x = 0; st.s.x = 0; }
    if (st.c.x >= g.nx - 1) { st.c.x = g.nx - 1; st.e.x = 0; }
    if (st.c.y <= 0) { st.c.y = 0; st.s.y = 0; }
    if (st.c.y >= g.ny - 1) { st.c.y = g.ny - 1; st.e.y = 0; }
    if (st.c.z <= 0) { st.c.z = 0; st.s.z = 0; }
    if (st.c.z >= g.nz - 1) { st.c.z = g.nz - 1; st.e.z = 0; }
    return st;
}
// Calls f(begin, end) for each stencil row range of the sorted list.
// cellStart has ncell+1 entries (exclusive scan of the cell counts).
template <class F>
__device__ __forceinline__ void for_stencil_rows(const Stencil& st, const GridDesc& g, const int* __restrict__ cellStart, F&& f) {
    for (int zz = st.s.z; zz <= st.e.z; zz++)
        for (int yy = st.s.y; yy <= st.e.y; yy++) {
            int k0 = key_of(make_int3(st.c.x + st.s.x, st.c.y + yy, st.c.z + zz), g);
            int k1 = key_of(make_int3(st.c.x + st.e.x, st.c.y + yy, st.c.z + zz), g);
            int b = __ldg(cellStart + k0), e = __ldg(cellStart + k1 + 1);
            if (b < e) f(b, e);
        }
}

// Device status word shared by the kernels of one scene.  Kernels record
// capacity overflows here instead of writing out of bounds.
struct DevStatus {
    int overflow;      // nonzero: a list overflowed its capacity
    int need_pairs;    // largest per-row count seen for the ball/fluid list
    int need_rev;      // largest reverse-list count
    int need_aux;      // largest per-row count for the secondary list
    int bad_index;     // nonzero: a remapped index fell outside its array
    int need_mark;     // largest per-row count for the fluid-marker list
    int need_mrev;     // largest per-row count for the marker-fluid list
};

}  // namespace demsph
