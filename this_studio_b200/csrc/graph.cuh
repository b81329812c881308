// CUDA-graph capture of a scene's step loop.  The steps of a scene are pure
// device work with fixed buffers between reallocations, so a block of steps is
// captured once (on a private capture stream) and replayed with one
// cudaGraphLaunch per block on the scene's stream.  Any reallocation of a
// buffer the captured kernels use drops the graph; the next run captures anew.
//
// Instantiated graphs are not destroyed when dropped: destroying one can wait
// on unrelated work of other streams for tens of milliseconds.  They go to a
// process-wide pool, and a new capture first tries to update a pooled graph
// of the same shape in place (cudaGraphExecUpdate: same kernels, new
// arguments and launch sizes) -- the batched form re-creates scenes of the
// same shape at every membership change.
#pragma once
#include <atomic>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace demsph {

extern std::atomic<long long> g_launches;

class ExecPool {
  public:
    static ExecPool& get() {
        static ExecPool pool;
        return pool;
    }
    // A pooled graph updated to `g`, or nullptr when none of this device fits.
    cudaGraphExec_t take(int dev, cudaGraph_t g) {
        std::lock_guard<std::mutex> lk(m_);
        for (size_t k = 0; k < spare_.size(); k++) {
            if (spare_[k].first != dev) continue;
            cudaGraphExecUpdateResultInfo info;
            if (cudaGraphExecUpdate(spare_[k].second, g, &info) == cudaSuccess) {
                cudaGraphExec_t e = spare_[k].second;
                spare_.erase(spare_.begin() + k);
                return e;
            }
            (void)cudaGetLastError();  // a shape mismatch is not an error here
        }
        return nullptr;
    }
    void put(int dev, cudaGraphExec_t e) {
        std::lock_guard<std::mutex> lk(m_);
        if (spare_.size() >= kMax) {  // keep the pool bounded: retire the oldest
            cudaGraphExecDestroy(spare_.front().second);
            spare_.erase(spare_.begin());
        }
        spare_.push_back({dev, e});
    }

  private:
    static constexpr size_t kMax = 32;
    std::mutex m_;
    std::vector<std::pair<int, cudaGraphExec_t>> spare_;
};

struct StepGraph {
    cudaGraphExec_t exec = nullptr;
    cudaStream_t cap = nullptr;
    cudaStream_t last = nullptr;  // the stream of the last replay
    int dev = 0;
    long long launches = 0;  // kernels per replay
    int steps = 0;           // steps per replay
    StepGraph() = default;
    StepGraph(const StepGraph&) = delete;
    StepGraph& operator=(const StepGraph&) = delete;
    ~StepGraph() {
        reset();
        if (cap) cudaStreamDestroy(cap);
    }
    // Hands the instantiated graph to the pool once its last replay is done.
    void reset() {
        if (exec) {
            if (last) cudaStreamSynchronize(last);
            ExecPool::get().put(dev, exec);
        }
        exec = nullptr;
        last = nullptr;
        steps = 0;
    }
    bool ready() const { return exec != nullptr; }
    // Captures body() -- nsteps steps issued on `stream` -- with `stream`
    // pointing at the capture stream meanwhile.
    template <class F>
    void capture(int nsteps, cudaStream_t& stream, F&& body) {
        reset();
        if (!cap) DEMSPH_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        const cudaStream_t keep = stream;
        const long long l0 = g_launches.load();
        cudaGraph_t g = nullptr;
        DEMSPH_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        stream = cap;
        try {
            body();
        } catch (...) {
            stream = keep;
            cudaStreamEndCapture(cap, &g);
            if (g) cudaGraphDestroy(g);
            g_launches = l0;
            throw;
        }
        stream = keep;
        DEMSPH_CUDA(cudaStreamEndCapture(cap, &g));
        launches = g_launches.load() - l0;
        g_launches = l0;
        DEMSPH_CUDA(cudaGetDevice(&dev));
        exec = ExecPool::get().take(dev, g);
        cudaError_t e = cudaSuccess;
        if (!exec) e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            exec = nullptr;
            DEMSPH_CUDA(e);
        }
        steps = nsteps;
    }
    void launch(cudaStream_t stream) {
        DEMSPH_CUDA(cudaGraphLaunch(exec, stream));
        last = stream;
        g_launches += launches;
    }
};

// Graphs of one scene keyed by the host-side buffer indices at capture time
// (which of each pair of ping-pong buffers is current): a block replayed from
// a different index state would use the wrong buffers.
struct GraphSet {
    std::map<int, std::unique_ptr<StepGraph>> byKey;
    long epoch = 0;  // counts resets: graphs built on this scene's buffers elsewhere check it
    void reset() {
        byKey.clear();
        epoch++;
    }
    StepGraph& at(int key) {
        auto& p = byKey[key];
        if (!p) p = std::make_unique<StepGraph>();
        return *p;
    }
};

}  // namespace demsph
