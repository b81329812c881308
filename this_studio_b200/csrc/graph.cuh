// CUDA-graph capture of a scene's step loop.  The steps of a scene are pure
// device work with fixed buffers between reallocations, so a block of steps is
// captured once (on a private capture stream) and replayed with one
// cudaGraphLaunch per block on the scene's stream.  Any reallocation of a
// buffer the captured kernels use drops the graph; the next run captures anew.
#pragma once
#include <atomic>
#include <map>
#include <memory>

#include "common.cuh"

namespace demsph {

extern std::atomic<long long> g_launches;

struct StepGraph {
    cudaGraphExec_t exec = nullptr;
    cudaStream_t cap = nullptr;
    long long launches = 0;  // kernels per replay
    int steps = 0;           // steps per replay
    StepGraph() = default;
    StepGraph(const StepGraph&) = delete;
    StepGraph& operator=(const StepGraph&) = delete;
    ~StepGraph() {
        reset();
        if (cap) cudaStreamDestroy(cap);
    }
    void reset() {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
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
        const cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            exec = nullptr;
            DEMSPH_CUDA(e);
        }
        steps = nsteps;
    }
    void launch(cudaStream_t stream) {
        DEMSPH_CUDA(cudaGraphLaunch(exec, stream));
        g_launches += launches;
    }
};

// Graphs of one scene keyed by the host-side buffer indices at capture time
// (which of each pair of ping-pong buffers is current): a block replayed from
// a different index state would use the wrong buffers.
struct GraphSet {
    std::map<int, std::unique_ptr<StepGraph>> byKey;
    void reset() { byKey.clear(); }
    StepGraph& at(int key) {
        auto& p = byKey[key];
        if (!p) p = std::make_unique<StepGraph>();
        return *p;
    }
};

}  // namespace demsph
