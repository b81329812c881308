// FP64 conservation diagnostics: a deterministic two-level reduction of K
// per-object terms.  The grid is fixed (kDiagBlocks blocks striding over the
// objects) and both levels add in a fixed order, so a state gives the same
// bits every time.  Term is a functor `void operator()(int i, double* v)`
// writing object i's K terms.
#pragma once
#include <atomic>

#include "common.cuh"

namespace demsph {

extern std::atomic<long long> g_launches;

constexpr int kDiagThreads = 256;
constexpr int kDiagBlocks = 296;  // two per SM

template <int K, class Term>
__global__ void __launch_bounds__(kDiagThreads) k_diag_partial(Term term, int n, double* __restrict__ partial) {
    __shared__ double sh[K][kDiagThreads];
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] = 0.0;
    for (int i = blockIdx.x * kDiagThreads + threadIdx.x; i < n; i += kDiagBlocks * kDiagThreads) {
        double v[K];
        term(i, v);
#pragma unroll
        for (int k = 0; k < K; k++) acc[k] += v[k];
    }
#pragma unroll
    for (int k = 0; k < K; k++) sh[k][threadIdx.x] = acc[k];
    __syncthreads();
    for (int w = kDiagThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
#pragma unroll
            for (int k = 0; k < K; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x < K) partial[(size_t)blockIdx.x * K + threadIdx.x] = sh[threadIdx.x][0];
}

template <int K>
__global__ void k_diag_final(const double* __restrict__ partial, double* __restrict__ out) {
    const int k = threadIdx.x;
    if (k >= K) return;
    double s = 0.0;
    for (int b = 0; b < kDiagBlocks; b++) s += partial[(size_t)b * K + k];
    out[k] = s;
}

// Sums the K terms of objects [0, n) into out_host (K doubles); `scratch`
// holds the partial sums and the result.  Synchronises the stream.
template <int K, class Term>
void diag_reduce(const Term& term, int n, double* out_host, DBuf<double>& scratch, cudaStream_t s) {
    static_assert(K <= kDiagThreads, "too many terms");
    const size_t need = (size_t)kDiagBlocks * K + K;
    if (scratch.n < need) scratch.alloc(need, s, false);
    k_diag_partial<K, Term><<<kDiagBlocks, kDiagThreads, 0, s>>>(term, n, scratch.p);
    k_diag_final<K><<<1, 32, 0, s>>>(scratch.p, scratch.p + (size_t)kDiagBlocks * K);
    g_launches += 2;
    DEMSPH_LAUNCH_CHECK();
    DEMSPH_CUDA(cudaMemcpyAsync(out_host, scratch.p + (size_t)kDiagBlocks * K, K * sizeof(double),
                                cudaMemcpyDeviceToHost, s));
    DEMSPH_CUDA(cudaStreamSynchronize(s));
}

}  // namespace demsph
