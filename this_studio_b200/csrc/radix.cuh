// Stable LSD radix sort of (uint32 key, int value) pairs, 8-bit digits,
// replacing thrust::sort_by_key in the reference's hash sort
// (DEMSPH/kernel/buildHashStartEnd.cu:60).
//
// Each pass: per-tile digit histograms -> exclusive scan of the
// digit-major histogram -> stable scatter.  Inside a tile the scatter ranks
// items with __match_any_sync / __popc within a warp and a per-warp digit
// count table in shared memory across warps, visiting items in index order,
// so equal keys keep their input order (the property the reference relies
// on: thrust's radix sort is stable).
//
// All scratch comes from a caller-provided RadixScratch, so the same kernels
// serve an allocating and a non-allocating entry point.
#pragma once
#include "common.cuh"

namespace demsph {

constexpr int kRxThreads = 256;
constexpr int kRxItems = 8;
constexpr int kRxTile = kRxThreads * kRxItems;  // 2048 items per tile
constexpr int kRxBins = 256;

static __global__ void __launch_bounds__(kRxThreads) k_rx_hist(const unsigned* __restrict__ keys, int n, int shift,
                                                               int* __restrict__ hist, int ntiles) {
    __shared__ int h[kRxBins];
    h[threadIdx.x] = 0;
    __syncthreads();
    int base = blockIdx.x * kRxTile;
#pragma unroll
    for (int r = 0; r < kRxItems; r++) {
        int i = base + r * kRxThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255u], 1);
    }
    __syncthreads();
    hist[threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// Exclusive scan of one 4096-element tile (1024 threads x 4 items); with a
// tile offset it finishes a multi-tile scan, with tileSum it produces the
// per-tile totals of the first level.
// `in` and `out` may be the same array (the sort scans its histogram in
// place): each thread reads its four words before the first barrier and
// writes them after the last, so they carry no __restrict__.
static __global__ void __launch_bounds__(1024) k_rx_scan(const int* in, int* out, int n,
                                                         const int* __restrict__ tileOffset, int* __restrict__ tileSum,
                                                         int inclusive) {
    __shared__ int ws[32];
    int base = blockIdx.x * 4096 + threadIdx.x * 4;
    int v[4], s = 0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        v[i] = (base + i < n) ? in[base + i] : 0;
        s += v[i];
    }
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    if (w == 0) {
        int a = ws[lane], xs = a;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, xs, o);
            if (lane >= o) xs += y;
        }
        ws[lane] = xs - a;
        if (lane == 31 && tileSum) tileSum[blockIdx.x] = xs;
    }
    __syncthreads();
    if (!out) return;
    int e = x - s + ws[w] + (tileOffset ? tileOffset[blockIdx.x] : 0);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        if (inclusive) e += v[i];
        if (base + i < n) out[base + i] = e;
        if (!inclusive) e += v[i];
    }
}

static __global__ void __launch_bounds__(kRxThreads) k_rx_scatter(const unsigned* __restrict__ kin,
                                                                  const int* __restrict__ vin,
                                                                  unsigned* __restrict__ kout, int* __restrict__ vout,
                                                                  int n, int shift, const int* __restrict__ offs,
                                                                  int ntiles) {
    __shared__ int running[kRxBins];
    __shared__ int warpCnt[kRxThreads / 32][kRxBins];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    running[t] = offs[t * ntiles + blockIdx.x];
    const int base = blockIdx.x * kRxTile;
    for (int r = 0; r < kRxItems; r++) {
#pragma unroll
        for (int k = 0; k < kRxThreads / 32; k++) warpCnt[k][t] = 0;
        __syncthreads();
        const int i = base + r * kRxThreads + t;
        const bool valid = i < n;
        const unsigned key = valid ? kin[i] : 0u;
        const int d = valid ? (int)((key >> shift) & 255u) : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int lrank = __popc(peers & ((1u << lane) - 1u));
        if (valid && lrank == 0) warpCnt[w][d] = __popc(peers);
        __syncthreads();
        if (valid) {
            int pre = 0;
            for (int k = 0; k < w; k++) pre += warpCnt[k][d];
            int pos = running[d] + pre + lrank;
            kout[pos] = key;
            vout[pos] = vin[i];
        }
        __syncthreads();
        int sum = 0;
#pragma unroll
        for (int k = 0; k < kRxThreads / 32; k++) sum += warpCnt[k][t];
        running[t] += sum;
        __syncthreads();
    }
}

// Raw scratch for a sort of up to `cap` items.
struct RadixScratch {
    unsigned* keysB;  // cap
    int* valsB;       // cap
    int* hist;        // 256 * tiles(cap)
    int* scanSums;    // tiles of the histogram scan
    int* scanOffs;    // tiles + 1
};

static constexpr inline int rx_tiles(int n) { return (n + kRxTile - 1) / kRxTile; }
// Number of int-sized words of scratch a sort of n items needs.
static constexpr inline size_t rx_scratch_words(int n) {
    return 2 * (size_t)n + 256 * (size_t)rx_tiles(n > 0 ? n : 1) +
           2 * ((256 * (size_t)rx_tiles(n > 0 ? n : 1) + 4095) / 4096) + 1 + 64;
}
static inline RadixScratch rx_carve(int* base, int n) {
    RadixScratch s;
    size_t t = (size_t)rx_tiles(n > 0 ? n : 1);
    size_t h = 256 * t;
    size_t st = (h + 4095) / 4096;
    s.keysB = (unsigned*)base;
    s.valsB = base + n;
    s.hist = base + 2 * (size_t)n;
    s.scanSums = s.hist + h;
    s.scanOffs = s.scanSums + st;
    return s;
}

// Exclusive (or inclusive) scan of n ints where n <= 4096 * 4096, using the
// given tile-sum / tile-offset scratch.  Returns the number of launches.
static inline int rx_scan(const int* in, int* out, int n, int* sums, int* offs, int inclusive, cudaStream_t s) {
    if (n <= 4096) {
        k_rx_scan<<<1, 1024, 0, s>>>(in, out, n, nullptr, nullptr, inclusive);
        return 1;
    }
    int nt = (n + 4095) / 4096;
    k_rx_scan<<<nt, 1024, 0, s>>>(in, nullptr, n, nullptr, sums, 0);
    k_rx_scan<<<1, 1024, 0, s>>>(sums, offs, nt, nullptr, nullptr, 0);
    k_rx_scan<<<nt, 1024, 0, s>>>(in, out, n, offs, nullptr, inclusive);
    return 3;
}

// Sorts (keys, vals) in place by the low `bits` bits of the keys, stably.
// keys/vals hold the input and receive the result.  Returns launches issued.
static inline int rx_sort(unsigned* keys, int* vals, int n, int bits, const RadixScratch& sc, cudaStream_t s) {
    if (n <= 1) return 0;
    const int nt = rx_tiles(n);
    int launches = 0;
    unsigned* ka = keys;
    int* va = vals;
    unsigned* kb = sc.keysB;
    int* vb = sc.valsB;
    const int passes = bits <= 0 ? 1 : (bits + 7) / 8;
    for (int p = 0; p < passes; p++) {
        int shift = 8 * p;
        k_rx_hist<<<nt, kRxThreads, 0, s>>>(ka, n, shift, sc.hist, nt);
        launches += 1 + rx_scan(sc.hist, sc.hist, 256 * nt, sc.scanSums, sc.scanOffs, 0, s);
        k_rx_scatter<<<nt, kRxThreads, 0, s>>>(ka, va, kb, vb, n, shift, sc.hist, nt);
        launches++;
        unsigned* tk = ka; ka = kb; kb = tk;
        int* tv = va; va = vb; vb = tv;
    }
    if (ka != keys) {
        DEMSPH_CUDA(cudaMemcpyAsync(keys, ka, (size_t)n * sizeof(unsigned), cudaMemcpyDeviceToDevice, s));
        DEMSPH_CUDA(cudaMemcpyAsync(vals, va, (size_t)n * sizeof(int), cudaMemcpyDeviceToDevice, s));
    }
    return launches;
}

}  // namespace demsph
