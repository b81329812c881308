// Counting sort of objects into a dense cell grid, replacing the reference's
// thrust::sort_by_key + findStartAndEnd (DEMSPH/kernel/buildHashStartEnd.cu:
// 6-83) and its thrust::inclusive_scan (buildHashStartEnd.cu:85-117).
//
// The number of cells is known, so a histogram + exclusive scan + scatter
// gives the sorted index list and every cell's [start, start+1) range in
// O(N + C) with no comparison sort.  The scatter uses atomics, so a ranking
// pass inside each cell restores the reference's stable (key, index) order and
// makes the result deterministic.
#pragma once
#include "common.cuh"

namespace demsph {

constexpr int kScanBlock = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanBlock * kScanItems;

// Histogram: key[i] = clamped cell key of object i; cnt[key]++.  With
// outsideOnly, objects inside the domain get key -1 and stay out of the table
// (calculateDummyHash, neighborSearchKernel.cu:29-55).
// A non-null gate makes every kernel of a build return at once while *gate is
// zero, so a build can sit in a captured step and run only when the device
// decides to (the skin lists of the fluid).
static __global__ void k_cell_count(const double4* __restrict__ p, int n, GridDesc g, int* __restrict__ key,
                             int* __restrict__ cnt, int outsideOnly, const int* __restrict__ gate) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (gate && *gate == 0)) return;
    double4 q = p[i];
    if (outsideOnly && q.x >= g.mn.x && q.x < g.mx.x && q.y >= g.mn.y && q.y < g.mx.y && q.z >= g.mn.z &&
        q.z < g.mx.z) {
        key[i] = -1;
        return;
    }
    int k = clamped_key(mk3(q.x, q.y, q.z), g);
    key[i] = k;
    atomicAdd(cnt + k, 1);
}

// One tile of an exclusive scan.  Optionally reads a per-tile offset, writes
// the tile total, and writes the scanned values (out[n] = grand total).
static __global__ void __launch_bounds__(kScanBlock) k_scan_tile(const int* __restrict__ in, int* __restrict__ out, int n,
                                                          const int* __restrict__ tileOffset,
                                                          int* __restrict__ tileSum, const int* __restrict__ gate) {
    if (gate && *gate == 0) return;
    __shared__ int warpSums[kScanBlock / 32];
    int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    int v[kScanItems];
    int s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
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
    if (lane == 31) warpSums[w] = x;
    __syncthreads();
    if (w == 0) {
        int ws = warpSums[lane];
        int xs = ws;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, xs, o);
            if (lane >= o) xs += y;
        }
        warpSums[lane] = xs - ws;
        if (lane == 31 && tileSum) tileSum[blockIdx.x] = xs;
    }
    __syncthreads();
    if (!out) return;
    int e = x - s + warpSums[w] + (tileOffset ? tileOffset[blockIdx.x] : 0);
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        if (base + i < n) out[base + i] = e;
        e += v[i];
        if (base + i == n - 1) out[n] = e;
    }
}

// Scatter into cell order: the atomic decrement returns the counters to zero
// for the next rebuild, so no memset is needed between rebuilds.
static __global__ void k_cell_scatter(const int* __restrict__ key, int n, const int* __restrict__ start, int* __restrict__ cnt,
                               int* __restrict__ sorted, const int* __restrict__ gate) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (gate && *gate == 0)) return;
    int k = key[i];
    if (k < 0) return;
    int slot = start[k] + atomicSub(cnt + k, 1) - 1;
    sorted[slot] = i;
}

// Restores ascending order inside each cell by orderKey[value] (by the value
// itself when orderKey is null): the stable order of the reference sort.  One
// thread per object counts the cell members that precede it, so a crowded
// cell costs O(members) per thread instead of a serial insertion sort.
static __global__ void k_cell_rank(int n, const int* __restrict__ key, const int* __restrict__ start,
                                   const int* __restrict__ unordered, int* __restrict__ sorted,
                                   const int* __restrict__ orderKey, int ncell, const int* __restrict__ gate) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n || (gate && *gate == 0)) return;
    if (s >= start[ncell]) return;  // start[ncell] = objects in the table
    int v = unordered[s];
    int c = key[v];
    int b = start[c], e = start[c + 1];
    int kv = orderKey ? orderKey[v] : v;
    int r = 0;
    for (int q = b; q < e; q++) {
        int u = unordered[q];
        int ku = orderKey ? orderKey[u] : u;
        r += ku < kv;
    }
    sorted[b + r] = v;
}

// Host side: owns the cell arrays of one grid and builds them on a stream.
struct CellTable {
    GridDesc g{};
    int ncell = 0;
    DBuf<int> key, cnt, start, sorted, unordered;
    std::vector<DBuf<int>*> scanTmp;  // per-level tile sums / offsets
    int launches = 0;                 // kernels issued by the last build

    ~CellTable() {
        for (auto* b : scanTmp) delete b;
    }
    void setup(const GridDesc& grid, int nobj, cudaStream_t s) {
        g = grid;
        ncell = g.ncell();
        key.alloc(nobj > 0 ? nobj : 1, s, false);
        sorted.alloc(nobj > 0 ? nobj : 1, s, false);
        unordered.alloc(nobj > 0 ? nobj : 1, s, false);
        cnt.alloc(ncell, s, true);
        start.alloc((size_t)ncell + 1, s, true);
        for (auto* b : scanTmp) delete b;
        scanTmp.clear();
        int m = ncell;
        while (m > kScanTile) {
            int nt = (m + kScanTile - 1) / kScanTile;
            auto* sums = new DBuf<int>();
            sums->alloc(nt, s, true);
            auto* offs = new DBuf<int>();
            offs->alloc((size_t)nt + 1, s, true);
            scanTmp.push_back(sums);
            scanTmp.push_back(offs);
            m = nt;
        }
    }
    // Exclusive scan of in[0..n) into out[0..n], recursing over tile sums.
    void scan(const int* in, int* out, int n, int level, cudaStream_t s, const int* gate) {
        if (n <= kScanTile) {
            k_scan_tile<<<1, kScanBlock, 0, s>>>(in, out, n, nullptr, nullptr, gate);
            launches++;
            return;
        }
        int nt = (n + kScanTile - 1) / kScanTile;
        int* sums = scanTmp[2 * level]->p;
        int* offs = scanTmp[2 * level + 1]->p;
        k_scan_tile<<<nt, kScanBlock, 0, s>>>(in, nullptr, n, nullptr, sums, gate);
        launches++;
        scan(sums, offs, nt, level + 1, s, gate);
        k_scan_tile<<<nt, kScanBlock, 0, s>>>(in, out, n, offs, nullptr, gate);
        launches++;
    }
    // Sorts objects p[0..n) (positions in .xyz) into cells.
    // outsideOnly: only objects outside the domain enter the table.
    // gate: device word; the build happens only where it is nonzero.
    void build(const double4* p, int n, cudaStream_t s, const int* orderKey = nullptr, bool outsideOnly = false,
               const int* gate = nullptr) {
        launches = 0;
        if (n > 0) {
            k_cell_count<<<grid_for(n, 256), 256, 0, s>>>(p, n, g, key.p, cnt.p, outsideOnly ? 1 : 0, gate);
            launches++;
        }
        scan(cnt.p, start.p, ncell, 0, s, gate);
        if (n > 0) {
            k_cell_scatter<<<grid_for(n, 256), 256, 0, s>>>(key.p, n, start.p, cnt.p, unordered.p, gate);
            k_cell_rank<<<grid_for(n, 256), 256, 0, s>>>(n, key.p, start.p, unordered.p, sorted.p, orderKey, ncell,
                                                         gate);
            launches += 2;
        }
        DEMSPH_LAUNCH_CHECK();
    }
};

}  // namespace demsph
