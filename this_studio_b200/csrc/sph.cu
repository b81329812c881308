// WCSPH path of the DEMSPH B200 library: per-step cell sort with physical
// reordering of the fluid state, fluid-fluid and fluid-dummy neighbour lists,
// Riemann momentum and continuity (Wendland C2), the linear equation of
// state, and the scene runtime behind the demsph_sph_* C ABI.
//
// Layout in HBM (one scene):
//   fluid  pos (x,y,z,h) | vel (vx,vy,vz,m) | st (rho,p,c,nu) : double4,
//          rho0, drho : double, id : int (caller's index).  Every step the
//          fluid is counting-sorted into cells and the arrays are permuted into
//          cell order (double-buffered), so a cell's particles are contiguous
//          and neighbour gathers stay in L1/L2.
//   dummy  pos | vel | st (c,nu,rho0,-) | normal : double4, sorted once.
//   lists  ELL rows, entry k of object i at row_at(i, k, K): the rows of 8
//          consecutive objects interleaved 4 entries at a time.
#include <array>
#include <map>
#include <algorithm>
#include <climits>
#include <atomic>
#include <cmath>
#include <memory>
#include <type_traits>

#include "cells.cuh"
#include "coupling.hpp"
#include "graph.cuh"
#include "vtu.hpp"
#include "diag.cuh"

namespace demsph {

extern std::atomic<long long> g_launches;

// Constants of the mixed-precision passes specialised for scenes whose fluid
// particles share h, m, c and nu and whose dummies share m, c, nu and rho0
// (with the fluid's h): every benchmark scene, and the reference's examples.
// Lengths in the pair terms stay in position quanta (r' = r / q, the exact
// integer difference of the fixed-point positions), so no per-pair rescaling
// is needed: grad W = K dq(q_n) r'/|r'| with K = 21 / (16 pi h^4) and
// q_n = |r'| q / h.
struct UniK {
    float invhq;   // q / h
    float K;       // 21 / (16 pi h^4)
    float c2q;     // (2 h / q)^2, the cutoff in quanta squared
    float cF;      // fluid sound speed
    float mF2;     // 2 m (fluid)
    float bF;      // 2 nu m (fluid-fluid viscosity factor)
    float mF, mD;  // particle masses (continuity)
    float mD2;     // 2 m_dummy
    float bD;      // 2 (nu + nu_dummy) / 2 m_dummy
    float cbarD;   // (c + c_dummy) / 2
    float invcD2;  // 1 / c_dummy^2
    float rho0D;   // dummy rest density
    float3 gq;     // gravity times q
};

struct SphDev {
    int N, ND, KF, KD;
    GridDesc g;
    const int* fStart;   // fluid cell start (new order)
    const int* dStart;   // dummy cell start (dummies stored in cell order)
    const double4* pos;  // current fluid pos
    const double4* lpos; // fluid pos when this step's lists were built (same slot order)
    const double4* vel;
    const double4* st;
    const double* rho0;
    double* drho;
    double4* posOut;
    double4* velOut;
    double4* stOut;
    double4* acc;
    const double4* dpos;
    const double4* dvel;
    const double4* dst;
    const double4* dnorm;
    // FP32 shadows of the fluid (v, m) and (rho, p, c, nu) records and of
    // the dummies' (v, m), (c, nu, rho0, -) and normals: what the
    // mixed-precision passes gather (the FP32 values those passes would
    // round the FP64 records to anyway).  Each kernel that writes an FP64
    // record writes its shadow too.
    const float4* velf;
    const float4* stf;
    float4* velfOut;
    float4* stfOut;
    const float4* dvelf;
    const float4* dstf;
    const float4* dnormf;
    // Fixed-point fluid / dummy positions for the mixed-precision passes:
    // (x - grid min) / q rounded to an integer, kept modulo 2^32, with h's
    // FP32 bits in w.  q is a power of two small enough that neighbours
    // (|r| < 2 h, plus a step's drift) differ by less than 2^30 quanta, so
    // the wrapped 32-bit difference of two positions is exact; r_ij is that
    // difference times q, rounded once to FP32.
    const int4* posq;
    int4* posqOut;
    const int4* dposq;
    float q;
    double invq;
    const float4* posf;   // fluid (x, y, z) - grid min and h, FP32, this step's order
    const float4* dposf;  // dummies, same form
    float eps;            // bound on |float coordinate - exact coordinate|
    int* nbF;
    int* cntF;
    int* nbD;
    int* cntD;
    // Skin lists: rows of every candidate within the cutoff plus a skin at
    // the last rebuild, rebuilt only when some particle has drifted half the
    // skin; the first momentum pass of each step evaluates them with the
    // exact cutoff test and writes the pairs it kept into nbF / nbD (the
    // reference's per-step pair set) for the step's later passes.
    float skin;        // added to the cutoff by the list build (0: exact lists)
    const int* gate;   // device word: nonzero when this step rebuilds
    int* nbV;
    int* cntV;
    int* nbVD;
    int* cntVD;
    const double4* xb;  // positions at the last rebuild
    unsigned* maxd2;    // largest squared drifts since the rebuild (float bits)
    // Moving boundary particles ("markers") that sample the DEM balls coupled
    // to the fluid, in this step's cell order, with the dummies' record
    // layout; mid maps a slot to the marker's index in body order, where
    // mforce collects the reaction of the fluid on each marker.
    int NM, KM;
    const int* mStart;
    const double4* mpos;
    const double4* mvel;
    const double4* mst;
    const double4* mnorm;
    const float4* mposf;
    const float4* mvelf;
    const float4* mstf;
    const float4* mnormf;
    const int4* mposq;
    const int* mid;
    int* nbM;
    int* cntM;
    int KR;          // the transposed list: fluid partners of each marker slot
    int* nbR;
    int* cntR;
    // Skin rows of the fluid-marker pairs (fluid rows and transposed rows),
    // built at a skin rebuild; a step's first momentum pass and first
    // reaction keep the pairs within the exact cutoff into nbM / nbR.
    int* nbMV;
    int* cntMV;
    int* nbRV;
    int* cntRV;
    double4* mforce;
    double3 gravity;
    DevStatus* status;
    UniK uk;  // set when the scene qualifies for the specialised passes
};

// A boundary set (dummies or markers) as the fluid passes read it.
struct BView {
    const double4* pos;
    const double4* vel;
    const double4* st;
    const double4* norm;
    const float4* velf;
    const float4* stf;
    const float4* normf;
    const int4* posq;
};
__device__ __forceinline__ BView dummy_view(const SphDev& d) {
    return BView{d.dpos, d.dvel, d.dst, d.dnorm, d.dvelf, d.dstf, d.dnormf, d.dposq};
}
__device__ __forceinline__ BView marker_view(const SphDev& d) {
    return BView{d.mpos, d.mvel, d.mst, d.mnorm, d.mvelf, d.mstf, d.mnormf, d.mposq};
}

// Wendland C2 kernel gradient (WCSPHIntegrationKernel.cuh:15-32), with the
// powers written as products.  Returns the factor f with gradW = f * r_ij.
template <class R>
__device__ __forceinline__ R gradw_factor(R r, R h) {
    if (r < (R)1.e-20 || r >= (R)2.0 * h) return (R)0;
    R q = r / h;
    R sigma = (R)21.0 / ((R)16.0 * (R)kPi * h * h * h);
    R t = (R)1.0 - (R)0.5 * q;
    R t3 = t * t * t;
    R dq = -(R)2.0 * t3 * ((R)1.0 + (R)2.0 * q) + (R)2.0 * (t3 * t);
    R dWdr = sigma * dq / h;
    return dWdr / r;
}

// The same factor with the per-particle constants of h hoisted out of the
// pair loop: invh = 1/h, sig = 21 / (16 pi h^3) and the pair's 1/r.  Only when
// the neighbour's h differs from the particle's are they formed per pair.
template <class R>
struct HConst {
    R h, invh, sig;
};
template <class R>
__device__ __forceinline__ HConst<R> hconst(R h) {
    return HConst<R>{h, (R)1.0 / h, (R)21.0 / ((R)16.0 * (R)kPi * h * h * h)};
}
template <class R>
__device__ __forceinline__ R gradw_fast(R r, R inv_r, const HConst<R>& hi, R hj) {
    HConst<R> k = hi;
    if (hj != hi.h) k = hconst<R>((R)0.5 * (hi.h + hj));
    if (r < (R)1.e-20 || r >= (R)2.0 * k.h) return (R)0;
    R q = r * k.invh;
    R t = (R)1.0 - (R)0.5 * q;
    R t3 = t * t * t;
    R dq = -(R)2.0 * t3 * ((R)1.0 + (R)2.0 * q) + (R)2.0 * (t3 * t);
    return k.sig * dq * k.invh * inv_r;
}
__device__ __forceinline__ double rsqrt_r(double x) { return rsqrt(x); }
__device__ __forceinline__ float rsqrt_r(float x) { return rsqrtf(x); }

// Four lanes cooperate on one fluid particle: neighbour loops are split
// across the lane quad and the partial sums are combined with shuffles, so a
// 128-thread block holds 32 particles and four times as many gathers are in
// flight per particle as with one thread each.
constexpr int kQuad = 4;
constexpr int kSphBlock = 128;
constexpr int kSphPerBlock = kSphBlock / kQuad;
__device__ __forceinline__ unsigned quad_mask() { return 0xFu << ((threadIdx.x & 31) & ~3u); }
template <class T>
__device__ __forceinline__ T quad_sum(T v, unsigned m) {
    v += __shfl_xor_sync(m, v, 1);
    v += __shfl_xor_sync(m, v, 2);
    return v;
}

__device__ __forceinline__ float4 f4(double4 a) { return make_float4((float)a.x, (float)a.y, (float)a.z, (float)a.w); }

__device__ __forceinline__ int4 fixq(double4 p, double3 o, double invq) {
    const unsigned long long x = (unsigned long long)__double2ll_rn((p.x - o.x) * invq);
    const unsigned long long y = (unsigned long long)__double2ll_rn((p.y - o.y) * invq);
    const unsigned long long z = (unsigned long long)__double2ll_rn((p.z - o.z) * invq);
    return make_int4((int)(unsigned)x, (int)(unsigned)y, (int)(unsigned)z, __float_as_int((float)p.w));
}
// a - b for two fixed-point coordinates of nearby particles, exact.
__device__ __forceinline__ float fixdiff(int a, int b, float q) {
    return (float)(int)((unsigned)a - (unsigned)b) * q;
}
__global__ void k_sph_fix(int n, const double4* __restrict__ pos, double3 o, double invq, int4* __restrict__ posq) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) posq[t] = fixq(pos[t], o, invq);
}
// Packed fluid shadows (scenes on the uniform-constant passes, whose h and m
// are the scene's constants): the fixed-point position carries rho in w and
// the FP32 velocity carries p in w, so a neighbour is two 16-byte gathers.
__device__ __forceinline__ int4 fixq_rho(double4 p, double4 st, double3 o, double invq) {
    int4 a = fixq(p, o, invq);
    a.w = __float_as_int((float)st.x);
    return a;
}
__device__ __forceinline__ float4 velf_p(double4 v, double4 st) {
    return make_float4((float)v.x, (float)v.y, (float)v.z, (float)st.y);
}
// Sets the w components of the fluid shadows for the packed (rho, p) or the
// general (h, m) layout.
__global__ void k_sph_pack(int n, const double4* __restrict__ pos, const double4* __restrict__ vel,
                           const double4* __restrict__ st, int4* __restrict__ posq, float4* __restrict__ velf,
                           int packed) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const double4 q = st[t];
    posq[t].w = __float_as_int(packed ? (float)q.x : (float)pos[t].w);
    velf[t].w = packed ? (float)q.y : (float)vel[t].w;
}

// Rewrites the FP32 shadows from the FP64 records (after a host-side change).
__global__ void k_sph_shadow(int n, const double4* __restrict__ a, const double4* __restrict__ b,
                             const double4* __restrict__ c, float4* __restrict__ af, float4* __restrict__ bf,
                             float4* __restrict__ cf) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    af[t] = f4(a[t]);
    bf[t] = f4(b[t]);
    if (c) cf[t] = f4(c[t]);
}

__global__ void k_iota(int n, int* __restrict__ a) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) a[t] = t;
}
// Copies one batch member's particles to [start, start + n) of the batch
// arrays, translated by off: (pos, vel, st) records and, for fluid, rho0 and
// a zero density change; for dummies `extra` is the dummy density.
__global__ void k_sph_place(int n, int start, double3 off, const double4* __restrict__ pos,
                            const double4* __restrict__ vel, const double4* __restrict__ st,
                            const double* __restrict__ extra, double4* __restrict__ pos2, double4* __restrict__ vel2,
                            double4* __restrict__ st2, double* __restrict__ extra2, double* __restrict__ zero2) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const double4 p = pos[t];
    pos2[start + t] = make_double4(p.x + off.x, p.y + off.y, p.z + off.z, p.w);
    vel2[start + t] = vel[t];
    st2[start + t] = st[t];
    extra2[start + t] = extra[t];
    if (zero2) zero2[start + t] = 0.0;
}
// getSPH on the device: the fluid records back into the caller's order
// (slot t holds caller index id[t]), in the host arrays' layout (3 doubles
// per vector), so each requested field is one contiguous copy to the host.
__global__ void k_sph_unpermute(int n, const int* __restrict__ id, const double4* __restrict__ pos,
                                const double4* __restrict__ vel, const double4* __restrict__ acc,
                                const double4* __restrict__ st, const double* __restrict__ drho,
                                double* __restrict__ oPos, double* __restrict__ oVel, double* __restrict__ oAcc,
                                double* __restrict__ oRho, double* __restrict__ oP, double* __restrict__ oDrho) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const long o = id[t];
    if (oPos) { const double4 a = pos[t]; oPos[3 * o] = a.x; oPos[3 * o + 1] = a.y; oPos[3 * o + 2] = a.z; }
    if (oVel) { const double4 a = vel[t]; oVel[3 * o] = a.x; oVel[3 * o + 1] = a.y; oVel[3 * o + 2] = a.z; }
    if (oAcc) { const double4 a = acc[t]; oAcc[3 * o] = a.x; oAcc[3 * o + 1] = a.y; oAcc[3 * o + 2] = a.z; }
    if (oRho || oP) {
        const double4 q = st[t];
        if (oRho) oRho[o] = q.x;
        if (oP) oP[o] = q.y;
    }
    if (oDrho) oDrho[o] = drho[t];
}

// Skin-list rebuild of a step: copies the records the gated permute wrote
// into the scratch halves of the ping-pong pairs back into the current
// halves (so the host's buffer indices do not depend on the device's
// decision) and records the rebuild positions.
__global__ void k_sph_copy_back(int n, const int* __restrict__ gate, const double4* __restrict__ pos2,
                                const double4* __restrict__ vel2, const double4* __restrict__ st2,
                                const double* __restrict__ rho02, const double* __restrict__ drho2,
                                const int* __restrict__ id2, const float4* __restrict__ velf2,
                                const float4* __restrict__ stf2, const int4* __restrict__ posq2,
                                double4* __restrict__ pos, double4* __restrict__ vel, double4* __restrict__ st,
                                double* __restrict__ rho0, double* __restrict__ drho, int* __restrict__ id,
                                float4* __restrict__ velf, float4* __restrict__ stf, int4* __restrict__ posq,
                                double4* __restrict__ xb) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n || *gate == 0) return;
    const double4 p = pos2[t];
    pos[t] = p;
    xb[t] = p;
    vel[t] = vel2[t];
    st[t] = st2[t];
    rho0[t] = rho02[t];
    drho[t] = drho2[t];
    id[t] = id2[t];
    velf[t] = velf2[t];
    stf[t] = stf2[t];
    posq[t] = posq2[t];
}

// Skin-list state of a scene, on the device.
constexpr int kSkinSlots = 256;
struct SkinState {
    int rebuild;                 // this step rebuilds (read by the gated kernels)
    int force;                   // set by the host after any change of the particle state
    int rebuilds;                // rebuilds so far (statistics)
    int pad;
    unsigned maxd2[kSkinSlots];  // largest squared drifts since the rebuild, as float bits
};
// Start of a step (one block of kSkinSlots threads): rebuild when forced or
// when some particle has drifted more than half the skin since the last
// rebuild (then no pair within the cutoff now was beyond cutoff + skin at
// the rebuild).
// Inside a captured step the decision also sets the condition of the graph's
// IF node around the rebuild (setCond = 1), so a step that keeps its lists
// launches none of the rebuild's kernels.
__global__ void __launch_bounds__(kSkinSlots) k_sph_skin_decide(SkinState* st, float half2,
                                                                 cudaGraphConditionalHandle cond, int setCond) {
    __shared__ unsigned m[kSkinSlots];
    const int t = threadIdx.x;
    m[t] = st->maxd2[t];
    __syncthreads();
    for (int h = kSkinSlots / 2; h > 0; h >>= 1) {
        if (t < h) m[t] = max(m[t], m[t + h]);
        __syncthreads();
    }
    const bool r = st->force != 0 || m[0] > __float_as_uint(half2);  // unsigned: a NaN drift rebuilds
    __syncthreads();
    if (r) st->maxd2[t] = 0u;
    if (t == 0) {
        st->rebuild = r ? 1 : 0;
        if (r) {
            st->force = 0;
            st->rebuilds++;
        }
        if (setCond) cudaGraphSetConditional(cond, r ? 1u : 0u);
    }
}

// World position of marker k (body order): its ball's centre plus the
// marker's offset, with h in w.
// With skin lists (maxd2 set) each marker's drift from its position at the
// last rebuild (xbM, body order) goes into the fluid's drift maxima, so
// that the rebuild decision covers both sides of a fluid-marker pair.
__global__ void k_sph_marker_place(int nm, const int* __restrict__ mb, const double4* __restrict__ moff,
                                   const double4* __restrict__ bpos, double4* __restrict__ tmp,
                                   const double4* __restrict__ xbM, unsigned* __restrict__ maxd2) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nm) return;
    const double4 o = moff[k];
    const double3 p = xyz(bpos[mb[k]]) + xyz(o);
    tmp[k] = d4(p, o.w);
    if (maxd2) {
        const double3 dd = p - xyz(xbM[k]);
        atomicMax(maxd2 + (blockIdx.x & (kSkinSlots - 1)), __float_as_uint((float)dot(dd, dd)));
    }
}
// Puts the markers into cell order (sorted[t] = body-order index of slot t)
// with their ball's rigid-body velocity v + omega x offset, the outward
// normal offset / |offset|, the record (c, nu, rho0, 0) and the mass in
// vel.w from mrec = (c, nu, rho0, m),
// and the FP32 and fixed-point copies the mixed-precision passes read.
__global__ void k_sph_marker_gather(int nm, const int* __restrict__ sorted, const double4* __restrict__ tmp,
                                    const int* __restrict__ mb, const double4* __restrict__ moff,
                                    const double4* __restrict__ mrec, const double4* __restrict__ bvel,
                                    const double4* __restrict__ bangv, double3 origin, double invq,
                                    double4* __restrict__ mpos,
                                    double4* __restrict__ mvel, double4* __restrict__ mst,
                                    double4* __restrict__ mnorm, float4* __restrict__ mposf,
                                    float4* __restrict__ mvelf, float4* __restrict__ mstf,
                                    float4* __restrict__ mnormf, int4* __restrict__ mposq, int* __restrict__ mid,
                                    const int* __restrict__ gate, double4* __restrict__ xbM) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nm) return;
    const int k = sorted[t];
    const double4 p = tmp[k];
    if (xbM && *gate) xbM[k] = p;  // a skin rebuild: the drift is measured from here
    const int b = mb[k];
    const double3 off = xyz(moff[k]);
    const double3 v = xyz(bvel[b]) + cross(xyz(bangv[b]), off);
    const double l2 = dot(off, off);
    const double3 n = l2 > 0.0 ? off * (1.0 / sqrt(l2)) : mk3(0, 0, 0);
    const double4 r4 = mrec[k];
    const double4 rec = make_double4(r4.x, r4.y, r4.z, 0);
    const double4 v4 = d4(v, r4.w), n4 = d4(n, 0);
    mpos[t] = p;
    mvel[t] = v4;
    mst[t] = rec;
    mnorm[t] = n4;
    mposf[t] = make_float4((float)(p.x - origin.x), (float)(p.y - origin.y), (float)(p.z - origin.z), (float)p.w);
    mvelf[t] = f4(v4);
    mstf[t] = f4(rec);
    mnormf[t] = f4(n4);
    mposq[t] = fixq(p, origin, invq);
    mid[t] = k;
}
// Coupling force and torque of each coupled ball: the sum of its markers'
// reactions (body order, markers [start[b], start[b+1])), and of offset x
// reaction, written at the ball's index.
// Balls with at most a few markers each (small balls: one marker at the
// centre): one thread per ball, the markers in order.
__global__ void k_sph_body_force_thread(int nb, const int* __restrict__ start, const int* __restrict__ ball,
                                        const double4* __restrict__ mforce, const double4* __restrict__ moff,
                                        double4* __restrict__ force, double4* __restrict__ torque) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    double3 F = mk3(0, 0, 0), T = mk3(0, 0, 0);
    for (int k = start[b]; k < start[b + 1]; k++) {
        const double3 f = xyz(mforce[k]);
        F += f;
        T += cross(xyz(moff[k]), f);
    }
    force[ball[b]] = d4(F, 0);
    torque[ball[b]] = d4(T, 0);
}
// Larger balls: one warp per ball, each lane sums a strided share of the
// ball's markers, then a fixed butterfly over the warp (the same sums every run).
constexpr int kBodyBlock = 256;
__global__ void __launch_bounds__(kBodyBlock) k_sph_body_force(int nb, const int* __restrict__ start,
                                                               const int* __restrict__ ball,
                                                               const double4* __restrict__ mforce,
                                                               const double4* __restrict__ moff,
                                                               double4* __restrict__ force,
                                                               double4* __restrict__ torque) {
    const int b = blockIdx.x * (kBodyBlock / 32) + (threadIdx.x >> 5);
    if (b >= nb) return;  // whole warps
    const int lane = threadIdx.x & 31;
    double3 F = mk3(0, 0, 0), T = mk3(0, 0, 0);
    for (int k = start[b] + lane; k < start[b + 1]; k += 32) {
        const double3 f = xyz(mforce[k]);
        F += f;
        T += cross(xyz(moff[k]), f);
    }
    for (int o = 16; o > 0; o >>= 1) {
        F.x += __shfl_xor_sync(0xffffffffu, F.x, o);
        F.y += __shfl_xor_sync(0xffffffffu, F.y, o);
        F.z += __shfl_xor_sync(0xffffffffu, F.z, o);
        T.x += __shfl_xor_sync(0xffffffffu, T.x, o);
        T.y += __shfl_xor_sync(0xffffffffu, T.y, o);
        T.z += __shfl_xor_sync(0xffffffffu, T.z, o);
    }
    if (lane == 0) {
        force[ball[b]] = d4(F, 0);
        torque[ball[b]] = d4(T, 0);
    }
}
// The same with one block per ball, for balls with hundreds of markers: each
// thread sums a strided share, then a fixed-order tree over the warps.
__global__ void __launch_bounds__(kBodyBlock) k_sph_body_force_block(const int* __restrict__ start,
                                                                     const int* __restrict__ ball,
                                                                     const double4* __restrict__ mforce,
                                                                     const double4* __restrict__ moff,
                                                                     double4* __restrict__ force,
                                                                     double4* __restrict__ torque) {
    __shared__ double sh[kBodyBlock / 32][6];
    const int b = blockIdx.x;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double3 F = mk3(0, 0, 0), T = mk3(0, 0, 0);
    for (int k = start[b] + threadIdx.x; k < start[b + 1]; k += kBodyBlock) {
        const double3 f = xyz(mforce[k]);
        F += f;
        T += cross(xyz(moff[k]), f);
    }
    for (int o = 16; o > 0; o >>= 1) {
        F.x += __shfl_xor_sync(0xffffffffu, F.x, o);
        F.y += __shfl_xor_sync(0xffffffffu, F.y, o);
        F.z += __shfl_xor_sync(0xffffffffu, F.z, o);
        T.x += __shfl_xor_sync(0xffffffffu, T.x, o);
        T.y += __shfl_xor_sync(0xffffffffu, T.y, o);
        T.z += __shfl_xor_sync(0xffffffffu, T.z, o);
    }
    if (lane == 0) {
        sh[w][0] = F.x; sh[w][1] = F.y; sh[w][2] = F.z;
        sh[w][3] = T.x; sh[w][4] = T.y; sh[w][5] = T.z;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        F = mk3(0, 0, 0);
        T = mk3(0, 0, 0);
        for (int v = 0; v < kBodyBlock / 32; v++) {
            F += mk3(sh[v][0], sh[v][1], sh[v][2]);
            T += mk3(sh[v][3], sh[v][4], sh[v][5]);
        }
        force[ball[b]] = d4(F, 0);
        torque[ball[b]] = d4(T, 0);
    }
}
// Puts the dummies into cell order (sorted[t] = caller index of slot t).
__global__ void k_sph_dummy_gather(int nd, const int* __restrict__ sorted, const double4* __restrict__ tp,
                                   const double4* __restrict__ tv, const double4* __restrict__ ts,
                                   const double* __restrict__ trh, double3 origin, double4* __restrict__ dpos,
                                   double4* __restrict__ dvel, double4* __restrict__ dst, double* __restrict__ drh,
                                   float4* __restrict__ dposf, int* __restrict__ did) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nd) return;
    const int o = sorted[t];
    const double4 p = tp[o];
    dpos[t] = p;
    dvel[t] = tv[o];
    dst[t] = ts[o];
    drh[t] = trh[o];
    dposf[t] = make_float4((float)(p.x - origin.x), (float)(p.y - origin.y), (float)(p.z - origin.z), (float)p.w);
    did[t] = o;
}

// Permutes the fluid into this step's cell order.
__global__ void k_sph_permute(int n, const int* __restrict__ sorted, const double4* __restrict__ pos,
                              const double4* __restrict__ vel, const double4* __restrict__ st,
                              const double* __restrict__ rho0, const double* __restrict__ drho,
                              const int* __restrict__ id, double4* __restrict__ pos2, double4* __restrict__ vel2,
                              double4* __restrict__ st2, double* __restrict__ rho02, double* __restrict__ drho2,
                              int* __restrict__ id2, float4* __restrict__ posf, float4* __restrict__ velf2,
                              float4* __restrict__ stf2, int4* __restrict__ posq2, double3 origin, double invq,
                              const int* __restrict__ gate, int packed) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n || (gate && *gate == 0)) return;
    int o = sorted[t];
    double4 p = pos[o];
    pos2[t] = p;
    const double4 v = vel[o], q = st[o];
    posq2[t] = packed ? fixq_rho(p, q, origin, invq) : fixq(p, origin, invq);
    posf[t] = make_float4((float)(p.x - origin.x), (float)(p.y - origin.y), (float)(p.z - origin.z), (float)p.w);
    vel2[t] = v;
    st2[t] = q;
    velf2[t] = packed ? velf_p(v, q) : f4(v);
    stf2[t] = f4(q);
    rho02[t] = rho0[o];
    drho2[t] = drho[o];
    id2[t] = id[o];
}

// countSPHInteractionsKernel / writeSPHInteractionsKernel and the dummy pair
// kernels (SPHNeighborSearchKernel.cu:6-228) in one pass: j != i,
// |r_ij| <= 2 max(h_i, h_j), rows in the reference's stencil order.
//
// Built one warp per cell (the warps stride over the cells with a grid of a
// few blocks per SM, so that a launch gated off by the skin decision, or the
// empty cells of a mostly empty domain, cost little).  All particles of a
// cell share the cell's 27-cell stencil (the reference clamps positions and
// cell indices the same way for
// every particle of a cell), so the warp stages the stencil's candidates --
// nine rows of three contiguous cells, in row order -- once in shared memory
// (coalesced loads), then sweeps them for each of the cell's particles in
// turn, one candidate per lane: a ballot of the hits and a popcount prefix
// give every hit its slot, so the row keeps the candidates' order, which is
// the reference's.  A stencil with more candidates than the stage holds is
// swept in consecutive chunks with the running count carried over.
//
// The test runs on FP32 coordinates relative to the grid minimum.  Each is
// within eps of the exact value, so |r|^2 is within `band` of the exact
// |r|^2; only candidates inside that band take the reference's FP64 test, so
// the pair set is the reference's exactly.
// Block shapes of the list build the autotuner chooses from: warps per
// block, candidates staged per warp (a multiple of 32), and the resident
// blocks per SM the register budget is fitted to.
struct ListShape {
    int warps, stage, minBlocks;
};
constexpr ListShape kListShapes[] = {{4, 512, 6}, {4, 384, 8}, {8, 256, 4}, {2, 512, 12}};
constexpr int kNumListShapes = 4;

// Layout of the neighbour rows (every list of this file: fluid-fluid,
// fluid-dummy, fluid-marker, the transposed marker rows, their skin rows).
// A pass gives each object a quad of lanes, lane `sub` taking entries sub,
// sub + 4, ...; a warp holds the quads of 8 consecutive objects.  The rows of
// 8 consecutive objects are therefore interleaved 4 entries at a time: the 32
// entries a warp reads in one iteration of a pair loop (entries 4m .. 4m + 3
// of its 8 objects) are one 128-byte line, instead of 16 bytes from each of 8
// rows.  Entry k of object i is at row_base(i, K) + 32 (k / 4) + k % 4; an
// array of n rows of capacity K holds row_words(n, K) entries.
__host__ __device__ __forceinline__ size_t row_base(int i, int K) {
    return (size_t)(i >> 3) * (size_t)((K + 3) & ~3) * 8 + (size_t)(i & 7) * 4;
}
__host__ __device__ __forceinline__ size_t row_at(int i, int k, int K) {
    return row_base(i, K) + (size_t)(k >> 2) * 32 + (k & 3);
}
static inline size_t row_words(size_t n, int K) {
    return ((n + 7) & ~(size_t)7) * (size_t)((std::max(K, 1) + 3) & ~3);
}


__device__ __forceinline__ float list_band(float cut, float eps) {
    return 4.0f * eps * (cut + 2.0f * eps) * 1.7321f + 4.0e-6f * cut * cut;
}

// Staged candidate: (x, y, z) relative to the grid minimum and, when every
// particle has the same h, the candidate's index in w (its bits); otherwise
// w = h and the index is staged separately.  Padding entries sit far away.
template <bool kUniformH>
struct ListStage {
    float4* pos;
    int* idx;
    __device__ __forceinline__ void put(int v, float4 q, int j) const {
        if (kUniformH) q.w = __int_as_float(j);
        else idx[v] = j;
        pos[v] = q;
    }
    __device__ __forceinline__ void pad(int v) const {
        pos[v] = make_float4(1.0e18f, 1.0e18f, 1.0e18f, kUniformH ? __int_as_float(-1) : 0.0f);
        if (!kUniformH) idx[v] = -1;
    }
    __device__ __forceinline__ int index(int v, float4 q) const { return kUniformH ? __float_as_int(q.w) : idx[v]; }
};

// One own particle against one staged batch: hit / band flags for this lane.
template <bool kUniformH>
__device__ __forceinline__ void list_test(const float4& pf, const float4& q, float loI, float hiI, float eps,
                                          float skin, bool& in, bool& band) {
    float lo = loI, hi = hiI;
    if (!kUniformH && q.w > pf.w) {
        const float cut = 2.0f * q.w + skin, c2 = cut * cut, bd = list_band(cut, eps);
        lo = c2 - bd;
        hi = c2 + bd;
    }
    const float dx = pf.x - q.x, dy = pf.y - q.y, dz = pf.z - q.z;
    const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    in = d2 < lo;
    band = !in && d2 <= hi;
}

__device__ __forceinline__ bool list_exact(const double4* __restrict__ own, const double4* __restrict__ other, int i,
                                           int j) {
    const double4 pi = own[i], pj = other[j];
    const double cd = 2.0 * fmax(pi.w, pj.w);
    const double3 r = xyz(pi) - xyz(pj);
    return (cd * cd - dot(r, r)) >= 0.;
}

template <bool kUniformH, int kStage>
__device__ __forceinline__ void cell_lists(int ps, int pe, const Stencil& st, const GridDesc& g,
                                           const int* __restrict__ cellStart, const double4* __restrict__ own,
                                           const float4* __restrict__ ownf, const double4* __restrict__ other,
                                           const float4* __restrict__ otherf, float eps, bool same, int K, int N,
                                           int* __restrict__ nb, int* __restrict__ cnt, int* needMax, int* overflow,
                                           const ListStage<kUniformH>& sg, float skin = 0.0f) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    int total = 0;
    for_stencil_rows(st, g, cellStart, [&](int b, int e) { total += e - b; });
    if (total == 0) {
        for (int i = ps + lane; i < pe; i += 32) cnt[i] = 0;
        return;
    }
    const int nchunk = (total + kStage - 1) / kStage;
    for (int ch = 0; ch < nchunk; ch++) {
        const int c0 = ch * kStage, c1 = min(total, c0 + kStage);
        const int m = c1 - c0, mp = (m + 31) & ~31;
        __syncwarp();
        int off = 0;
        for_stencil_rows(st, g, cellStart, [&](int b, int e) {
            const int lo = max(b, b + (c0 - off)), hi = min(e, b + (c1 - off));
            for (int j = lo + lane; j < hi; j += 32) sg.put(off + (j - b) - c0, otherf[j], j);
            off += e - b;
        });
        if (m + lane < mp) sg.pad(m + lane);
        __syncwarp();
        // two own particles per sweep share each staged load
        for (int i0 = ps; i0 < pe; i0 += 2) {
            const int i1 = min(i0 + 1, pe - 1);
            const bool two = i0 + 1 < pe;
            const float4 pa = ownf[i0], pb = ownf[i1];
            const float cA = 2.0f * pa.w + skin, cB = 2.0f * pb.w + skin;
            const float bA = list_band(cA, eps), bB = list_band(cB, eps);
            const float loA = cA * cA - bA, hiA = cA * cA + bA, loB = cB * cB - bB, hiB = cB * cB + bB;
            int na = ch == 0 ? 0 : cnt[i0];
            int nbc = (ch == 0 || !two) ? 0 : cnt[i1];
            for (int v0 = 0; v0 < mp; v0 += 32) {
                const int v = v0 + lane;
                const float4 q = sg.pos[v];
                const int j = sg.index(v, q);
                bool inA, bandA, inB, bandB;
                list_test<kUniformH>(pa, q, loA, hiA, eps, skin, inA, bandA);
                list_test<kUniformH>(pb, q, loB, hiB, eps, skin, inB, bandB);
                if (skin > 0.0f) {  // a skin row only has to hold every pair within the cutoff
                    inA = inA || bandA;
                    inB = inB || bandB;
                    bandA = bandB = false;
                }
                if (same) {
                    if (j == i0) inA = bandA = false;
                    if (j == i1) inB = bandB = false;
                }
                if (!two) inB = bandB = false;
                if (__any_sync(0xffffffffu, bandA || bandB)) {
                    if (bandA) inA = list_exact(own, other, i0, j);
                    if (bandB) inB = list_exact(own, other, i1, j);
                }
                const unsigned hA = __ballot_sync(0xffffffffu, inA);
                const unsigned hB = __ballot_sync(0xffffffffu, inB);
                if (hA) {
                    const int k = na + __popc(hA & lt);
                    if (inA && k < K) nb[row_at(i0, k, K)] = j;
                    na += __popc(hA);
                }
                if (hB) {
                    const int k = nbc + __popc(hB & lt);
                    if (inB && k < K) nb[row_at(i1, k, K)] = j;
                    nbc += __popc(hB);
                }
            }
            if (lane < 2 && (lane == 0 || two)) {
                const int i = lane == 0 ? i0 : i1;
                const int c = lane == 0 ? na : nbc;
                if (ch + 1 < nchunk) {
                    cnt[i] = c;
                } else if (c > K) {  // the passes walk this particle's stencil instead
                    atomicMax(needMax, c);
                    atomicExch(overflow, 1);
                    cnt[i] = -1;
                } else {
                    cnt[i] = c;
                }
            }
            __syncwarp();
        }
    }
}

template <bool kUniformH, int kShape, bool kMarkers>
__global__ void __launch_bounds__(32 * kListShapes[kShape].warps, kListShapes[kShape].minBlocks)
    k_sph_lists_cell(SphDev d, int ncell) {
    constexpr int kListWarps = kListShapes[kShape].warps, kStage = kListShapes[kShape].stage;
    __shared__ float4 sPos[kListWarps][kStage];
    __shared__ int sIdx[kUniformH ? 1 : kListWarps][kUniformH ? 1 : kStage];
    const int w = threadIdx.x >> 5;
    if (d.gate && *d.gate == 0) return;
    ListStage<kUniformH> sg{sPos[w], kUniformH ? nullptr : sIdx[kUniformH ? 0 : w]};
    for (int cell = blockIdx.x * kListWarps + w; cell < ncell; cell += gridDim.x * kListWarps) {
        const int ps = d.fStart[cell], pe = d.fStart[cell + 1];
        if (ps == pe) continue;
        // stencil of the cell: the one every particle of the cell computes
        const double4 p0 = d.pos[ps];
        Stencil st = stencil_of(xyz(p0), d.g);
        cell_lists<kUniformH, kStage>(ps, pe, st, d.g, d.fStart, d.pos, d.posf, d.pos, d.posf, d.eps, true, d.KF, d.N,
                                      d.nbF, d.cntF, &d.status->need_pairs, &d.status->overflow, sg, d.skin);
        if (d.ND > 0)
            cell_lists<kUniformH, kStage>(ps, pe, st, d.g, d.dStart, d.pos, d.posf, d.dpos, d.dposf, d.eps, false,
                                          d.KD, d.N, d.nbD, d.cntD, &d.status->need_aux, &d.status->overflow, sg,
                                          d.skin);
        else
            for (int i = ps + (threadIdx.x & 31); i < pe; i += 32) d.cntD[i] = 0;
        if (kMarkers)
            cell_lists<kUniformH, kStage>(ps, pe, st, d.g, d.mStart, d.pos, d.posf, d.mpos, d.mposf, d.eps, false,
                                          d.KM, d.N, d.nbM, d.cntM, &d.status->need_mark, &d.status->overflow, sg);
    }
}

// The transposed fluid-marker list: for each marker slot, the fluid
// particles within the list cutoff, one warp per marker cell (the fluid
// list build with the roles swapped; the FP64 test is symmetric, so the
// pairs are exactly those of the fluid rows).  With skin lists (d.skin > 0,
// gated on the rebuild decision) the rows are skin rows.
template <bool kUniformH, int kShape>
__global__ void __launch_bounds__(32 * kListShapes[kShape].warps, kListShapes[kShape].minBlocks)
    k_sph_marker_lists(SphDev d, int ncell) {
    constexpr int kListWarps = kListShapes[kShape].warps, kStage = kListShapes[kShape].stage;
    __shared__ float4 sPos[kListWarps][kStage];
    __shared__ int sIdx[kUniformH ? 1 : kListWarps][kUniformH ? 1 : kStage];
    const int w = threadIdx.x >> 5;
    if (d.gate && *d.gate == 0) return;
    ListStage<kUniformH> sg{sPos[w], kUniformH ? nullptr : sIdx[kUniformH ? 0 : w]};
    for (int cell = blockIdx.x * kListWarps + w; cell < ncell; cell += gridDim.x * kListWarps) {
        const int ps = d.mStart[cell], pe = d.mStart[cell + 1];
        if (ps == pe) continue;
        Stencil st = stencil_of(xyz(d.mpos[ps]), d.g);
        cell_lists<kUniformH, kStage>(ps, pe, st, d.g, d.fStart, d.mpos, d.mposf, d.pos, d.posf, d.eps, false, d.KR,
                                      d.NM, d.nbR, d.cntR, &d.status->need_mrev, &d.status->overflow, sg, d.skin);
    }
}

// The fluid-marker skin rows: k_sph_lists_cell's marker row alone, at a skin
// rebuild (gated), within the cutoff plus the skin.
template <bool kUniformH, int kShape>
__global__ void __launch_bounds__(32 * kListShapes[kShape].warps, kListShapes[kShape].minBlocks)
    k_sph_marker_rows(SphDev d, int ncell) {
    constexpr int kListWarps = kListShapes[kShape].warps, kStage = kListShapes[kShape].stage;
    __shared__ float4 sPos[kListWarps][kStage];
    __shared__ int sIdx[kUniformH ? 1 : kListWarps][kUniformH ? 1 : kStage];
    const int w = threadIdx.x >> 5;
    if (d.gate && *d.gate == 0) return;
    ListStage<kUniformH> sg{sPos[w], kUniformH ? nullptr : sIdx[kUniformH ? 0 : w]};
    for (int cell = blockIdx.x * kListWarps + w; cell < ncell; cell += gridDim.x * kListWarps) {
        const int ps = d.fStart[cell], pe = d.fStart[cell + 1];
        if (ps == pe) continue;
        Stencil st = stencil_of_cell(cell, d.g);
        cell_lists<kUniformH, kStage>(ps, pe, st, d.g, d.mStart, d.pos, d.posf, d.mpos, d.mposf, d.eps, false, d.KM,
                                      d.N, d.nbM, d.cntM, &d.status->need_mark, &d.status->overflow, sg, d.skin);
    }
}

// Calls f(j) for this lane's share of particle i's neighbours: from the ELL
// row when it fitted (cnt >= 0), otherwise (a row that overflowed its
// capacity) by walking the cell stencil of pi with the list's cutoff test
// against `other`.  With pi and `other` the positions the lists were built
// from this yields the list's pair set; the fluid passes after the step's
// drift pass the drifted positions (see k_sph_accel).
// A row's count word: a count c >= 0 of a dense row (lane `sub` of the quad
// takes entries sub, sub + 4, ... below c), or, with kLaneRows set, four lane
// counts of 7 bits (lane `sub` takes entries sub, sub + 4, ... of its own
// count: the rows the first pass on skin lists writes), or -1 (overflowed).
constexpr int kLaneRows = 1 << 30;
__host__ __device__ __forceinline__ int lane_count(int cnt, int sub) {
    if (cnt >= kLaneRows) return (cnt >> (7 * sub)) & 127;
    return cnt > sub ? (cnt - sub + 3) >> 2 : 0;
}

template <class F>
__device__ __forceinline__ void quad_neighbors(int cnt, const int* __restrict__ nb, int K, int i, int self,
                                               const double4 pi, const GridDesc& g,
                                               const int* __restrict__ cellStart,
                                               const double4* __restrict__ other, F&& f) {
    const int sub = threadIdx.x & 3;
    if (cnt >= 0) {
        // two neighbours per iteration, their row entries loaded one
        // iteration ahead so the index load is off the gather's critical path
        // (this lane's m-th entry, 4m + sub, sits at row[32 m])
        const int* __restrict__ row = nb + row_base(i, K) + sub;
        const int mend = lane_count(cnt, sub);
        int m = 0;
        int j0 = m < mend ? __ldg(row) : -1;
        int j1 = m + 1 < mend ? __ldg(row + 32) : -1;
        for (; m < mend; m += 2) {
            const int a = j0, b = j1;
            const int mn = m + 2;
            j0 = mn < mend ? __ldg(row + 32 * mn) : -1;
            j1 = mn + 1 < mend ? __ldg(row + 32 * (mn + 1)) : -1;
            f(a);
            if (b >= 0) f(b);
        }
        return;
    }
    const double3 ri = xyz(pi);
    Stencil st = stencil_of(ri, g);
    for_stencil_rows(st, g, cellStart, [&](int b, int e) {
        for (int j = b + sub; j < e; j += kQuad) {
            if (j == self) continue;
            double4 pj = other[j];
            double cut = 2.0 * fmax(pi.w, pj.w);
            double3 r = ri - xyz(pj);
            if ((cut * cut - dot(r, r)) >= 0.) f(j);
        }
    });
}

// updateWCSPHAccelerationKernel (WCSPHIntegrationKernel.cu:42-148) fused with
// the half kick (SPHVelocityIntegrationKernel, :150-159) and, in the first
// half, the drift (SPHPositionIntegrationKernel, :161-170).  Reads the state
// arrays and writes the integrated particle into separate output arrays, so
// no thread sees a neighbour's updated state.
// r_ij = r_i - r_j and h_j: from the FP64 positions in the FP64 passes, from
// the fixed-point positions in the mixed-precision ones.
template <class R>
struct OwnPos {
    double3 r;
    int4 q;
};
template <class R>
__device__ __forceinline__ void pair_r(const OwnPos<R>& o, const double4* __restrict__ pos,
                                       const int4* __restrict__ posq, float q, int j, V<R>& rij, R& hj) {
    if constexpr (std::is_same<R, float>::value) {
        const int4 b = posq[j];
        rij = make_float3(fixdiff(o.q.x, b.x, q), fixdiff(o.q.y, b.y, q), fixdiff(o.q.z, b.z, q));
        hj = __int_as_float(b.w);
    } else {
        const double4 b = pos[j];
        rij = o.r - xyz(b);
        hj = b.w;
    }
}
// a / b: IEEE division in the FP64 passes, the fast reciprocal-based divide
// (a couple of ulp) in the mixed-precision ones.
__device__ __forceinline__ double div_r(double a, double b) { return a / b; }
__device__ __forceinline__ float div_r(float a, float b) { return __fdividef(a, b); }

// Neighbour records in the precision of the pass: the FP64 records for the
// FP64 passes, their FP32 shadows for the mixed-precision ones (the same
// values those passes would compute by rounding the FP64 records).
template <class R>
__device__ __forceinline__ void load_fluid(const SphDev& d, int j, V<R>& vj, R& mj, R& rhoj, R& PR, R& cj, R& nuj) {
    if constexpr (std::is_same<R, float>::value) {
        const float4 v = d.velf[j], q = d.stf[j];
        vj = make_float3(v.x, v.y, v.z);
        mj = v.w;
        rhoj = q.x; PR = q.y; cj = q.z; nuj = q.w;
    } else {
        const double4 v = d.vel[j], q = d.st[j];
        vj = xyz(v);
        mj = v.w;
        rhoj = q.x; PR = q.y; cj = q.z; nuj = q.w;
    }
}
template <class R>
__device__ __forceinline__ void load_dummy(const BView& b, int j, V<R>& nw, V<R>& vj, R& mj, R& cj, R& nuj, R& rho0j) {
    if constexpr (std::is_same<R, float>::value) {
        const float4 n = b.normf[j], v = b.velf[j], q = b.stf[j];
        nw = make_float3(n.x, n.y, n.z);
        vj = make_float3(v.x, v.y, v.z);
        mj = v.w;
        cj = q.x; nuj = q.y; rho0j = q.z;
    } else {
        const double4 n = b.norm[j], v = b.vel[j], q = b.st[j];
        nw = xyz(n);
        vj = xyz(v);
        mj = v.w;
        cj = q.x; nuj = q.y; rho0j = q.z;
    }
}

// A fluid particle's own values as the passes use them.
template <class R>
struct FluidOwn {
    OwnPos<R> op;
    V<R> vi;
    R rhoi, PL, ci, nui;
    HConst<R> hk;
};
template <class R>
__device__ __forceinline__ FluidOwn<R> fluid_own(const SphDev& d, int i, const double4& pi4, const double4& vi4,
                                                 const double4& s4) {
    return FluidOwn<R>{OwnPos<R>{xyz(pi4), std::is_same<R, float>::value ? d.posq[i] : make_int4(0, 0, 0, 0)},
                       cvt<R>(xyz(vi4)),
                       (R)s4.x,
                       (R)s4.y,
                       (R)s4.z,
                       (R)s4.w,
                       hconst<R>((R)pi4.w)};
}

// Fluid-boundary term of updateWCSPHAccelerationKernel
// (WCSPHIntegrationKernel.cu:110-143): the boundary particle j takes the
// mirrored normal velocity and the hydrostatically extrapolated pressure
// PR = PL + rho_i max(0, -g . r_ij), rho_j = PR / c_j^2 + rho0_j.
template <class R>
__device__ __forceinline__ void boundary_acc_r(const SphDev& d, const FluidOwn<R>& o, const BView& bv, int j,
                                               const V<R>& rij, R hj, const V<R>& g, V<R>& acc) {
    using VR = V<R>;
    VR nw, vj;
    R cj, nuj, rho0j, mj;
    load_dummy<R>(bv, j, nw, vj, mj, cj, nuj, rho0j);
    R UL = dot(-nw, o.vi);
    R UR = -UL + (R)2.0 * dot(-nw, vj);
    R grj = -dot(g, rij);
    if (grj < (R)0.) grj = (R)0.;
    R PR = o.PL + o.rhoi * grj;
    R rhoj = div_r(PR, cj * cj) + rho0j;
    R r2 = dot(rij, rij);
    R inv_r = r2 < (R)1.0e-20 ? (R)0 : rsqrt_r(r2);
    R r = r2 * inv_r;
    VR dW = gradw_fast<R>(r, inv_r, o.hk, hj) * rij;
    R cbar = (R)0.5 * (o.ci + cj), rbar = (R)0.5 * (o.rhoi + rhoj);
    R beta = fmin((R)3.0 * fmax(UL - UR, (R)0.0), cbar);
    R Ps = (R)0.5 * (o.PL + PR) + (R)0.5 * beta * rbar * (UL - UR);
    R inv_rr = div_r((R)1.0, o.rhoi * rhoj);
    acc -= (R)2.0 * mj * (Ps * inv_rr) * dW;
    R nuij = (R)0.5 * (o.nui + nuj);
    acc += (R)2.0 * nuij * dot(rij * inv_r, dW) * (o.vi - vj) * mj * inv_rr;
}
template <class R>
__device__ __forceinline__ void boundary_acc(const SphDev& d, const FluidOwn<R>& o, const BView& bv, int j,
                                             const V<R>& g, V<R>& acc) {
    V<R> rij;
    R hj;
    pair_r<R>(o.op, bv.pos, bv.posq, d.q, j, rij, hj);
    boundary_acc_r<R>(d, o, bv, j, rij, hj, g, acc);
}

// Fluid-fluid term of updateWCSPHAccelerationKernel
// (WCSPHIntegrationKernel.cu:70-109) given r_ij and h_j, accumulated into acc.
template <class R>
__device__ __forceinline__ void fluid_acc_r(const SphDev& d, const FluidOwn<R>& o, int j, const V<R>& rij, R hj,
                                            V<R>& acc) {
    using VR = V<R>;
    VR vj;
    R rhoj, PR, cj, nuj, mj;
    load_fluid<R>(d, j, vj, mj, rhoj, PR, cj, nuj);
    R r2 = dot(rij, rij);
    // -normalize(r_ij) and |r_ij| from one reciprocal square root, as the
    // reference's normalize does (myVec.h:112-128)
    R inv_r = r2 < (R)1.0e-20 ? (R)0 : rsqrt_r(r2);
    R r = r2 * inv_r;
    VR e = rij * (-inv_r);
    R UL = dot(o.vi, e), UR = dot(vj, e);
    VR dW = gradw_fast<R>(r, inv_r, o.hk, hj) * rij;
    R cbar = (R)0.5 * (o.ci + cj), rbar = (R)0.5 * (o.rhoi + rhoj);
    R beta = fmin((R)3.0 * fmax(UL - UR, (R)0.0), cbar);
    R Ps = (R)0.5 * (o.PL + PR) + (R)0.5 * beta * rbar * (UL - UR);
    R inv_rr = div_r((R)1.0, o.rhoi * rhoj);
    acc -= (R)2.0 * mj * (Ps * inv_rr) * dW;
    R nuij = (R)0.5 * (o.nui + nuj);
    // Q5: r_hat . gradW without 1/r, as the reference (WCSPHIntegrationKernel.cu:108)
    acc += (R)2.0 * nuij * dot(-e, dW) * (o.vi - vj) * mj * inv_rr;
}
template <class R>
__device__ __forceinline__ void fluid_acc(const SphDev& d, const FluidOwn<R>& o, int j, V<R>& acc) {
    V<R> rij;
    R hj;
    pair_r<R>(o.op, d.pos, d.posq, d.q, j, rij, hj);
    fluid_acc_r<R>(d, o, j, rij, hj, acc);
}

// The reference list's cutoff test (countSPHInteractionsKernel,
// SPHNeighborSearchKernel.cu:6-60): (cut^2 - |r|^2) >= 0, cut = 2 max(h_i, h_j),
// on the FP64 positions, given the pass's r_ij and h_j.  In FP64 that r_ij is
// the reference's.  The mixed passes test the FP32 square of the fixed-point
// difference (the pair term's own |r|^2) and take the FP64 test only in a
// band of 2e-6 cut^2 around the cutoff, which covers that square's rounding
// (< 5e-7 relative) and the positions' quantisation (< 3e-8 relative).
// pi_of() gives the FP64 position of i when the band needs it (the reaction
// on the markers loads it only then); the fluid passes pass what they hold.
template <class PI>
__device__ __forceinline__ bool cutoff_f(const float3& rij, float hi, float hj, PI&& pi_of,
                                         const double4* __restrict__ other, int j) {
    const float d2 = dot(rij, rij);
    const float cut = 2.0f * fmaxf(hi, hj);
    const float c2 = cut * cut, band = 2.0e-6f * c2;
    if (d2 < c2 - band) return true;
    if (d2 > c2 + band) return false;
    const double4 pi = pi_of();
    const double4 pj = other[j];
    const double cd = 2.0 * fmax(pi.w, pj.w);
    const double3 r = xyz(pi) - xyz(pj);
    return (cd * cd - dot(r, r)) >= 0.;
}
template <class R>
__device__ __forceinline__ bool cutoff_r(const V<R>& rij, R hj, const double4& pi, const double4* __restrict__ other,
                                         int j) {
    if constexpr (std::is_same<R, float>::value) {
        return cutoff_f(rij, (float)pi.w, hj, [&] { return pi; }, other, j);
    } else {
        const double cd = 2.0 * fmax(pi.w, hj);
        return (cd * cd - dot(rij, rij)) >= 0.;
    }
}

// One skin row of particle i in the first pass of a step: fn(j) tests the
// exact cutoff, adds the pair's term when it holds, and returns the test.
// Each lane of the quad takes entries sub, sub + 4, ... of the skin row and
// writes the ones it keeps to sub, sub + 4, ... of the exact row nbOut (in
// place of its own candidates, so never past them); cntOut gets the four
// lane counts (kLaneRows), which the step's later passes read.  A skin row
// that overflowed its capacity (cnt < 0) is replaced by the cell-stencil
// walk, and the exact row is marked overflowed (-1: the later passes walk as
// well); so is a row with more than 127 pairs in one lane.
template <class F>
__device__ __forceinline__ void skin_loop(int cnt, const int* __restrict__ nbV, int K, int i, int* __restrict__ nbOut,
                                          int* __restrict__ cntOut, const double4& pi, const GridDesc& g,
                                          const int* __restrict__ cellStart, const double4* __restrict__ other,
                                          int self, F&& fn) {
    const int sub = threadIdx.x & 3;
    if (cnt < 0) {
        if (sub == 0) cntOut[i] = -1;
        Stencil st = stencil_of(xyz(pi), g);
        for_stencil_rows(st, g, cellStart, [&](int b, int e) {
            for (int j = b + sub; j < e; j += kQuad)
                if (j != self) fn(j);
        });
        return;
    }
    // this lane's entries of the dense skin row (4m + sub at row[32 m]); the
    // kept ones become its lane row of this step (w-th kept at out[32 w])
    const int* __restrict__ row = nbV + row_base(i, K) + sub;
    int* __restrict__ out = nbOut + row_base(i, K) + sub;
    int w = 0;  // pairs this lane kept
    const int mend = lane_count(cnt, sub);
    int m = 0;
    int j0 = m < mend ? __ldg(row) : -1;
    int j1 = m + 1 < mend ? __ldg(row + 32) : -1;
    for (; m < mend; m += 2) {
        const int a = j0, b = j1;
        const int mn = m + 2;
        j0 = mn < mend ? __ldg(row + 32 * mn) : -1;
        j1 = mn + 1 < mend ? __ldg(row + 32 * (mn + 1)) : -1;
        if (fn(a)) out[32 * w++] = a;
        if (b >= 0 && fn(b)) out[32 * w++] = b;
    }
    const unsigned gm = quad_mask();
    const int over = quad_sum(w > 127 ? 1 : 0, gm);
    const int packed = quad_sum(w << (7 * sub), gm);
    if (sub == 0) cntOut[i] = over ? -1 : (kLaneRows | packed);
}

// Fluid-boundary term of updateWCSPHDensityChangeKernel
// (WCSPHIntegrationKernel.cu:240-270), before the factor 2 rho_i.
template <class R>
__device__ __forceinline__ void boundary_drho(const SphDev& d, const FluidOwn<R>& o, const BView& bv, int j,
                                              const V<R>& g, R& dRho) {
    using VR = V<R>;
    VR rij, nw, vj;
    R hj, cj, nuj, rho0j, mj;
    pair_r<R>(o.op, bv.pos, bv.posq, d.q, j, rij, hj);
    load_dummy<R>(bv, j, nw, vj, mj, cj, nuj, rho0j);
    R grj = -dot(g, rij);
    if (grj < (R)0.) grj = (R)0.;
    R PR = o.PL + o.rhoi * grj;
    R rhoj = div_r(PR, cj * cj) + rho0j;
    R r2 = dot(rij, rij);
    R inv_r = r2 < (R)1.0e-20 ? (R)0 : rsqrt_r(r2);
    R r = r2 * inv_r;
    VR dW = gradw_fast<R>(r, inv_r, o.hk, hj) * rij;
    VR e = rij * (-inv_r);
    R cbar = (R)0.5 * (o.ci + cj), rbar = (R)0.5 * (o.rhoi + rhoj);
    VR vs = (R)0.5 * (o.vi + vj);
    vs += (R)0.5 * div_r(o.PL - PR, rbar * cbar) * e;
    dRho += div_r(mj, rhoj) * dot(o.vi - vs, dW);
}

// Resident blocks per SM the passes' register budgets are fitted to (FP32 /
// FP64 arithmetic): what the measured-fastest register allocations gave.
template <class R>
constexpr int kAccelBlocks = std::is_same<R, float>::value ? 7 : 4;
template <class R>
constexpr int kDensityBlocks = std::is_same<R, float>::value ? 8 : 5;

// kSkin: the first pass of a step on skin lists (first = 1).  The quad walks
// the particle's skin rows, keeps the pairs within the exact cutoff (their
// terms are the pass's sum, and they are written as this step's exact rows
// for the continuity and second momentum passes), and the pass records the
// particle's drift from its rebuild position.
template <class R, bool kMarkers, bool kSkin = false>
__global__ void __launch_bounds__(kSphBlock, kAccelBlocks<R>) k_sph_accel(SphDev d, double hdt, double dt, int first) {
    const int i = blockIdx.x * kSphPerBlock + threadIdx.x / kQuad;
    if (i >= d.N) return;
    const int sub = threadIdx.x & 3;
    const unsigned gm = quad_mask();
    using VR = V<R>;
    const double4 pi4 = d.pos[i];
    const double3 ri = xyz(pi4);
    const double4 vi4 = d.vel[i];
    const FluidOwn<R> o = fluid_own<R>(d, i, pi4, vi4, d.st[i]);
    VR acc = v3r<R>(0, 0, 0);
    const VR g = cvt<R>(d.gravity);
    if constexpr (kSkin) {
        skin_loop(d.cntV[i], d.nbV, d.KF, i, d.nbF, d.cntF, pi4, d.g, d.fStart, d.pos, i, [&](int j) {
            VR rij;
            R hj;
            pair_r<R>(o.op, d.pos, d.posq, d.q, j, rij, hj);
            if (!cutoff_r<R>(rij, hj, pi4, d.pos, j)) return false;
            fluid_acc_r<R>(d, o, j, rij, hj, acc);
            return true;
        });
        if (d.ND > 0) {
            const BView dv = dummy_view(d);
            skin_loop(d.cntVD[i], d.nbVD, d.KD, i, d.nbD, d.cntD, pi4, d.g, d.dStart, d.dpos, -1, [&](int j) {
                VR rij;
                R hj;
                pair_r<R>(o.op, d.dpos, d.dposq, d.q, j, rij, hj);
                if (!cutoff_r<R>(rij, hj, pi4, d.dpos, j)) return false;
                boundary_acc_r<R>(d, o, dv, j, rij, hj, g, acc);
                return true;
            });
        }
    } else {
        quad_neighbors(d.cntF[i], d.nbF, d.KF, i, i, pi4, d.g, d.fStart, d.pos,
                       [&](int j) { fluid_acc<R>(d, o, j, acc); });
        if (d.ND > 0) {
            const BView dv = dummy_view(d);
            quad_neighbors(d.cntD[i], d.nbD, d.KD, i, -1, pi4, d.g, d.dStart, d.dpos,
                           [&](int j) { boundary_acc<R>(d, o, dv, j, g, acc); });
        }
    }
    if constexpr (kMarkers) {
        const BView mv = marker_view(d);
        if constexpr (kSkin) {
            // the fluid-marker skin row, with the same exact test the reaction
            // on the markers applies to its transposed row (cutoff_r from the
            // fluid's side of the pair, on the same positions)
            skin_loop(d.cntMV[i], d.nbMV, d.KM, i, d.nbM, d.cntM, pi4, d.g, d.mStart, d.mpos, -1, [&](int j) {
                VR rij;
                R hj;
                pair_r<R>(o.op, mv.pos, mv.posq, d.q, j, rij, hj);
                if (!cutoff_r<R>(rij, hj, pi4, d.mpos, j)) return false;
                boundary_acc_r<R>(d, o, mv, j, rij, hj, g, acc);
                return true;
            });
        } else {
            // the markers' terms, from this step's fluid-marker rows; an
            // overflowed row walks the marker cells at the rows' build
            // positions, so the pairs are exactly the ones the reaction on
            // the markers uses
            const int cM = d.cntM[i];
            quad_neighbors(cM, d.nbM, d.KM, i, -1, cM < 0 ? d.lpos[i] : pi4, d.g, d.mStart, d.mpos,
                           [&](int j) { boundary_acc<R>(d, o, mv, j, g, acc); });
        }
    }
    double3 a = up(acc);
    a.x = quad_sum(a.x, gm);
    a.y = quad_sum(a.y, gm);
    a.z = quad_sum(a.z, gm);
    if (sub != 0) return;
    a += d.gravity;
    d.acc[i] = d4(a, 0);
    double3 v = xyz(vi4) + hdt * a;
    const double4 v4 = d4(v, vi4.w);
    d.velOut[i] = v4;
    d.velfOut[i] = f4(v4);
    if (first) {
        const double4 pn = d4(ri + dt * v, pi4.w);
        d.posOut[i] = pn;
        d.posqOut[i] = fixq(pn, d.g.mn, d.invq);
        if constexpr (kSkin) {
            // drift since the rebuild, into one of kSkinSlots maxima (spread so
            // that the atomics of different blocks do not queue on one address)
            const double3 dd = xyz(pn) - xyz(d.xb[i]);
            atomicMax(d.maxd2 + (blockIdx.x & (kSkinSlots - 1)), __float_as_uint((float)dot(dd, dd)));
        }
    }
}

// updateWCSPHDensityChangeKernel + SPHDensityPressureIntegrationKernel
// (WCSPHIntegrationKernel.cu:172-282): drho += dt * 2 rho_i sum m_j/rho_j
// (v_i - v*) . gradW; clamp drho >= -0.1 rho0; rho = rho0 + drho; p = c^2 drho.
template <class R, bool kMarkers>
__global__ void __launch_bounds__(kSphBlock, kDensityBlocks<R>) k_sph_density(SphDev d, double dt) {
    const int i = blockIdx.x * kSphPerBlock + threadIdx.x / kQuad;
    if (i >= d.N) return;
    const int sub = threadIdx.x & 3;
    const unsigned gm = quad_mask();
    using VR = V<R>;
    const double4 pi4 = d.pos[i];
    const double4 s4 = d.st[i];
    const FluidOwn<R> o = fluid_own<R>(d, i, pi4, d.vel[i], s4);
    R dRho = (R)0;
    quad_neighbors(d.cntF[i], d.nbF, d.KF, i, i, pi4, d.g, d.fStart, d.pos, [&](int j) {
        VR rij, vj;
        R hj, rhoj, PR, cj, nuj, mj;
        pair_r<R>(o.op, d.pos, d.posq, d.q, j, rij, hj);
        load_fluid<R>(d, j, vj, mj, rhoj, PR, cj, nuj);
        R r2 = dot(rij, rij);
        R inv_r = r2 < (R)1.0e-20 ? (R)0 : rsqrt_r(r2);
        R r = r2 * inv_r;
        VR dW = gradw_fast<R>(r, inv_r, o.hk, hj) * rij;
        VR e = rij * (-inv_r);
        R cbar = (R)0.5 * (o.ci + cj), rbar = (R)0.5 * (o.rhoi + rhoj);
        VR vs = (R)0.5 * (o.vi + vj);
        vs += (R)0.5 * div_r(o.PL - PR, rbar * cbar) * e;
        dRho += div_r(mj, rhoj) * dot(o.vi - vs, dW);
    });
    const VR g = cvt<R>(d.gravity);
    if (d.ND > 0) {
        const BView dv = dummy_view(d);
        quad_neighbors(d.cntD[i], d.nbD, d.KD, i, -1, pi4, d.g, d.dStart, d.dpos,
                       [&](int j) { boundary_drho<R>(d, o, dv, j, g, dRho); });
    }
    if constexpr (kMarkers) {
        const BView mv = marker_view(d);
        const int cM = d.cntM[i];
        quad_neighbors(cM, d.nbM, d.KM, i, -1, cM < 0 ? d.lpos[i] : pi4, d.g, d.mStart, d.mpos,
                       [&](int j) { boundary_drho<R>(d, o, mv, j, g, dRho); });
    }
    double dsum = quad_sum((double)dRho, gm);
    if (sub != 0) return;
    double dr = dsum * (2.0 * (double)o.rhoi);
    double ch = d.drho[i] + dr * dt;
    d.drho[i] = ch;
    double r0 = d.rho0[i];
    if (ch < -0.1 * r0) ch = -0.1 * r0;
    const double4 so = make_double4(ch + r0, s4.z * s4.z * ch, s4.z, s4.w);
    d.stOut[i] = so;
    d.stfOut[i] = f4(so);
}

// ---------------------------------------------------------------------------
// Mixed-precision passes for scenes with uniform particle constants (UniK);
// with markers (kMarkers) the shadows stay unpacked and the markers' terms
// come from the general boundary functions.  Same pair sets, same formulas as k_sph_accel /
// k_sph_density (updateWCSPHAccelerationKernel and
// updateWCSPHDensityChangeKernel, WCSPHIntegrationKernel.cu:42-282), with
// the constants hoisted and the terms regrouped:
//   grad W_ij = K dq r'/|r'|,  dq = 2 t^3 (t - 1 - 2 q_n),  t = max(1 - q_n/2, 0);
//   U_L - U_R = -(v_i - v_j) . r'/|r'|;
//   r_hat . grad W = K dq (the reference's viscosity factor, Q5);
//   momentum:   a_i += s [2 nu m (v_i - v_j) - 2 m P* r'/|r'|],  s = K dq / (rho_i rho_j);
//   continuity: (v_i - v*) . grad W = K dq [(v_i - v_j) . r'/|r'| + (P_L - P_R) / (rho_bar c_bar)] / 2.
// The fluid shadows are packed (k_sph_pack): the fixed-point position
// carries rho in w and the FP32 velocity carries p, so a fluid neighbour is
// two 16-byte gathers (the general passes gather a third record, the FP32
// state); a dummy is three (position, velocity, normal).  Each pass writes
// the packed shadows of the records it writes; the continuity pass, which
// changes rho and p, writes the next position / velocity buffers.

struct PairGeom {
    float3 r;   // r_i - r_j in quanta
    float inv_r;
    float Kdq;  // K dq(q_n)
};
__device__ __forceinline__ PairGeom pair_geom(const int4& qi, const int4& qj, const UniK& u) {
    PairGeom p;
    p.r = make_float3((float)(int)((unsigned)qi.x - (unsigned)qj.x), (float)(int)((unsigned)qi.y - (unsigned)qj.y),
                      (float)(int)((unsigned)qi.z - (unsigned)qj.z));
    const float r2 = dot(p.r, p.r);
    p.inv_r = rsqrtf(fmaxf(r2, 1e-30f));
    const float qn = r2 * p.inv_r * u.invhq;
    const float t = fmaxf(1.0f - 0.5f * qn, 0.0f);
    const float t3 = t * t * t;
    p.Kdq = u.K * (2.0f * t3 * (t - 1.0f - 2.0f * qn));
    return p;
}
// The reference's cutoff test for a skin candidate, from the quanta
// difference: FP32 outside a band of 2e-6 cut^2, the FP64 test on the FP64
// positions inside it (as cutoff_f).
__device__ __forceinline__ bool cutoff_u(const float3& r, const UniK& u, const double4& pi,
                                         const double4* __restrict__ other, int j) {
    const float d2 = dot(r, r);
    const float band = 2.0e-6f * u.c2q;
    if (d2 < u.c2q - band) return true;
    if (d2 > u.c2q + band) return false;
    const double4 pj = other[j];
    const double cd = 2.0 * fmax(pi.w, pj.w);
    const double3 dr = xyz(pi) - xyz(pj);
    return (cd * cd - dot(dr, dr)) >= 0.;
}

struct OwnU {
    int4 q;
    float3 v;
    float rho, PL;
};
// The own particle as the pair loops use it (fixed-point position with rho,
// FP32 velocity, rho and p).  The FP64 velocity and state records are read
// again after the loops rather than kept, so they hold no registers there.
__device__ __forceinline__ OwnU own_u(const SphDev& d, int i) {
    const double4 v = d.vel[i];
    const double4 st = d.st[i];
    return OwnU{d.posq[i], make_float3((float)v.x, (float)v.y, (float)v.z), (float)st.x, (float)st.y};
}
// A fluid neighbour's (v, p) and rho: from the packed shadows, or in a scene
// with markers, whose reaction kernel reads the shadows' usual w components
// (h, m), from the velocity shadow and the FP32 state (a third gather).
template <bool kUnpacked>
__device__ __forceinline__ float4 nb_vp(const SphDev& d, int j, const int4& qj, float& rhoj) {
    const float4 v = d.velf[j];
    if constexpr (kUnpacked) {
        const float4 sj = d.stf[j];
        rhoj = sj.x;
        return make_float4(v.x, v.y, v.z, sj.y);
    } else {
        rhoj = __int_as_float(qj.w);
        return v;
    }
}
// vj = (v_j, p_j), rhoj from the packed shadows
__device__ __forceinline__ void acc_fluid_u(const OwnU& o, const PairGeom& p, const float4& vj, float rhoj,
                                            const UniK& u, float3& acc) {
    const float3 dv = o.v - make_float3(vj.x, vj.y, vj.z);
    const float dU = -dot(dv, p.r) * p.inv_r;
    const float beta = fminf(3.0f * fmaxf(dU, 0.0f), u.cF);
    const float Ps = 0.5f * (o.PL + vj.w) + 0.5f * beta * (0.5f * (o.rho + rhoj)) * dU;
    const float s = p.Kdq * __fdividef(1.0f, o.rho * rhoj);
    const float sw = s * u.mF2 * Ps * p.inv_r;
    const float sb = s * u.bF;
    acc += sb * dv - sw * p.r;
}
// The dummy's extrapolated pressure and density (WCSPHIntegrationKernel.cu:
// 110-143): P_R = P_L + rho_i max(-g . r_ij, 0), rho_j = P_R / c_j^2 + rho0_j.
__device__ __forceinline__ void dummy_state_u(const OwnU& o, const PairGeom& p, const UniK& u, float& PR, float& rhoj) {
    const float grj = fmaxf(-dot(u.gq, p.r), 0.0f);
    PR = o.PL + o.rho * grj;
    rhoj = PR * u.invcD2 + u.rho0D;
}
__device__ __forceinline__ void acc_dummy_u(const OwnU& o, const PairGeom& p, const float4& vj, const float4& nj,
                                            const UniK& u, float3& acc) {
    const float3 vd = make_float3(vj.x, vj.y, vj.z), nw = make_float3(nj.x, nj.y, nj.z);
    const float UL = -dot(nw, o.v);
    const float UR = -UL - 2.0f * dot(nw, vd);
    float PR, rhoj;
    dummy_state_u(o, p, u, PR, rhoj);
    const float dU = UL - UR;
    const float beta = fminf(3.0f * fmaxf(dU, 0.0f), u.cbarD);
    const float Ps = 0.5f * (o.PL + PR) + 0.5f * beta * (0.5f * (o.rho + rhoj)) * dU;
    const float s = p.Kdq * __fdividef(1.0f, o.rho * rhoj);
    const float sw = s * u.mD2 * Ps * p.inv_r;
    const float sb = s * u.bD;
    acc += sb * (o.v - vd) - sw * p.r;
}

// Resident blocks: the first pass (skin rows) fits 48 registers without
// spilling and gains from the extra warps (10 blocks: 70 -> 66 us at 128k);
// the second pass keeps 64 (at 48 it spills).  kMarkers: a coupled scene
// (unpacked shadows; the markers' terms by the general boundary functions,
// the same pairs and terms as the general passes and the reaction kernel),
// at 8 blocks despite a few spills (ice sheet 5.4-5.6 ms per coupled step at
// 7 blocks, 5.1-5.2 at 8; 6 and 9 blocks no better).
template <bool kSkin, bool kMarkers>
constexpr int kUniAccelBlocks = kMarkers ? 8 : (kSkin ? 10 : 8);
template <bool kSkin, bool kMarkers = false>
__global__ void __launch_bounds__(kSphBlock, kUniAccelBlocks<kSkin, kMarkers>)
    k_sph_accel_u(SphDev d, double hdt, double dt, int first) {
    const int i = blockIdx.x * kSphPerBlock + threadIdx.x / kQuad;
    if (i >= d.N) return;
    const int sub = threadIdx.x & 3;
    const unsigned gm = quad_mask();
    const UniK& u = d.uk;
    const double4 pi4 = d.pos[i];
    const OwnU o = own_u(d, i);
    float3 acc = make_float3(0.f, 0.f, 0.f);
    if constexpr (kSkin) {
        skin_loop(d.cntV[i], d.nbV, d.KF, i, d.nbF, d.cntF, pi4, d.g, d.fStart, d.pos, i, [&](int j) {
            const int4 qj = d.posq[j];
            const PairGeom p = pair_geom(o.q, qj, u);
            if (!cutoff_u(p.r, u, pi4, d.pos, j)) return false;
            float rhoj;
            const float4 vj = nb_vp<kMarkers>(d, j, qj, rhoj);
            acc_fluid_u(o, p, vj, rhoj, u, acc);
            return true;
        });
        if (d.ND > 0) {
            skin_loop(d.cntVD[i], d.nbVD, d.KD, i, d.nbD, d.cntD, pi4, d.g, d.dStart, d.dpos, -1, [&](int j) {
                const PairGeom p = pair_geom(o.q, d.dposq[j], u);
                if (!cutoff_u(p.r, u, pi4, d.dpos, j)) return false;
                acc_dummy_u(o, p, d.dvelf[j], d.dnormf[j], u, acc);
                return true;
            });
        }
    } else {
        quad_neighbors(d.cntF[i], d.nbF, d.KF, i, i, pi4, d.g, d.fStart, d.pos, [&](int j) {
            const int4 qj = d.posq[j];
            const PairGeom p = pair_geom(o.q, qj, u);
            float rhoj;
            const float4 vj = nb_vp<kMarkers>(d, j, qj, rhoj);
            acc_fluid_u(o, p, vj, rhoj, u, acc);
        });
        if (d.ND > 0) {
            quad_neighbors(d.cntD[i], d.nbD, d.KD, i, -1, pi4, d.g, d.dStart, d.dpos, [&](int j) {
                const PairGeom p = pair_geom(o.q, d.dposq[j], u);
                acc_dummy_u(o, p, d.dvelf[j], d.dnormf[j], u, acc);
            });
        }
    }
    if constexpr (kMarkers) {
        // as k_sph_accel: the fluid-marker skin row with the exact test the
        // reaction on the markers applies, or this step's rows (an overflowed
        // row walks the marker cells at the rows' build positions)
        const FluidOwn<float> fo = fluid_own<float>(d, i, pi4, d.vel[i], d.st[i]);
        const BView mv = marker_view(d);
        const float3 g = cvt<float>(d.gravity);
        if constexpr (kSkin) {
            skin_loop(d.cntMV[i], d.nbMV, d.KM, i, d.nbM, d.cntM, pi4, d.g, d.mStart, d.mpos, -1, [&](int j) {
                float3 rij;
                float hj;
                pair_r<float>(fo.op, mv.pos, mv.posq, d.q, j, rij, hj);
                if (!cutoff_r<float>(rij, hj, pi4, d.mpos, j)) return false;
                boundary_acc_r<float>(d, fo, mv, j, rij, hj, g, acc);
                return true;
            });
        } else {
            const int cM = d.cntM[i];
            quad_neighbors(cM, d.nbM, d.KM, i, -1, cM < 0 ? d.lpos[i] : pi4, d.g, d.mStart, d.mpos,
                           [&](int j) { boundary_acc<float>(d, fo, mv, j, g, acc); });
        }
    }
    double3 a = up(acc);
    a.x = quad_sum(a.x, gm);
    a.y = quad_sum(a.y, gm);
    a.z = quad_sum(a.z, gm);
    if (sub != 0) return;
    const double4 vi4 = d.vel[i];
    const double4 s4 = d.st[i];
    a += d.gravity;
    d.acc[i] = d4(a, 0);
    const double3 v = xyz(vi4) + hdt * a;
    const double4 v4 = d4(v, vi4.w);
    d.velOut[i] = v4;
    d.velfOut[i] = kMarkers ? f4(v4) : velf_p(v4, s4);
    if (first) {
        const double4 pn = d4(xyz(pi4) + dt * v, pi4.w);
        d.posOut[i] = pn;
        d.posqOut[i] = kMarkers ? fixq(pn, d.g.mn, d.invq) : fixq_rho(pn, s4, d.g.mn, d.invq);
        if constexpr (kSkin) {
            const double3 dd = xyz(pn) - xyz(d.xb[i]);
            atomicMax(d.maxd2 + (blockIdx.x & (kSkinSlots - 1)), __float_as_uint((float)dot(dd, dd)));
        }
    }
}

template <bool kMarkers = false>
__global__ void __launch_bounds__(kSphBlock, 8) k_sph_density_u(SphDev d, double dt) {
    const int i = blockIdx.x * kSphPerBlock + threadIdx.x / kQuad;
    if (i >= d.N) return;
    const int sub = threadIdx.x & 3;
    const unsigned gm = quad_mask();
    const UniK& u = d.uk;
    const double4 pi4 = d.pos[i];
    const OwnU o = own_u(d, i);
    float sumF = 0.f, sumD = 0.f;  // sum of (1 / rho_j) (v_i - v*) . grad W / (1/2), per kind of neighbour
    quad_neighbors(d.cntF[i], d.nbF, d.KF, i, i, pi4, d.g, d.fStart, d.pos, [&](int j) {
        const int4 qj = d.posq[j];
        const PairGeom p = pair_geom(o.q, qj, u);
        float rhoj;
        const float4 vj = nb_vp<kMarkers>(d, j, qj, rhoj);  // (v_j, p_j)
        const float3 dv = o.v - make_float3(vj.x, vj.y, vj.z);
        const float rbar = 0.5f * (o.rho + rhoj);
        const float X = __fdividef(o.PL - vj.w, rbar * u.cF);
        sumF += __fdividef(p.Kdq * (dot(dv, p.r) * p.inv_r + X), rhoj);
    });
    if (d.ND > 0) {
        quad_neighbors(d.cntD[i], d.nbD, d.KD, i, -1, pi4, d.g, d.dStart, d.dpos, [&](int j) {
            const PairGeom p = pair_geom(o.q, d.dposq[j], u);
            const float4 vj = d.dvelf[j];
            float PR, rhoj;
            dummy_state_u(o, p, u, PR, rhoj);
            const float3 dv = o.v - make_float3(vj.x, vj.y, vj.z);
            const float rbar = 0.5f * (o.rho + rhoj);
            const float X = __fdividef(o.PL - PR, rbar * u.cbarD);
            sumD += __fdividef(p.Kdq * (dot(dv, p.r) * p.inv_r + X), rhoj);
        });
    }
    float dRhoM = 0.f;  // the markers' terms, as k_sph_density
    if constexpr (kMarkers) {
        const FluidOwn<float> fo = fluid_own<float>(d, i, pi4, d.vel[i], d.st[i]);
        const BView mv = marker_view(d);
        const float3 g = cvt<float>(d.gravity);
        const int cM = d.cntM[i];
        quad_neighbors(cM, d.nbM, d.KM, i, -1, cM < 0 ? d.lpos[i] : pi4, d.g, d.mStart, d.mpos,
                       [&](int j) { boundary_drho<float>(d, fo, mv, j, g, dRhoM); });
    }
    const double dsum =
        quad_sum(0.5 * ((double)u.mF * (double)sumF + (double)u.mD * (double)sumD) + (double)dRhoM, gm);
    if (sub != 0) return;
    const double4 vi4 = d.vel[i];
    const double4 s4 = d.st[i];
    const double dr = dsum * (2.0 * (double)o.rho);
    double ch = d.drho[i] + dr * dt;
    d.drho[i] = ch;
    const double r0 = d.rho0[i];
    if (ch < -0.1 * r0) ch = -0.1 * r0;
    const double4 so = make_double4(ch + r0, s4.z * s4.z * ch, s4.z, s4.w);
    d.stOut[i] = so;
    d.stfOut[i] = f4(so);
    if constexpr (kMarkers) return;  // unpacked shadows: the state records alone change
    // the next position / velocity buffers: the same records, their packed
    // shadows with the new rho and p
    d.posOut[i] = pi4;
    d.velOut[i] = vi4;
    d.posqOut[i] = make_int4(o.q.x, o.q.y, o.q.z, __float_as_int((float)so.x));
    d.velfOut[i] = velf_p(vi4, so);
}

// Reaction of the fluid on the markers: for marker t, minus the sum over
// the fluid particles a whose list rows hold t of m_a times marker t's term
// in a's acceleration, evaluated by the same function from the same state as
// the fluid's pass (so the pair set and the terms are the fluid's own).  Four
// lanes share the marker's transposed list row; the result, times w, is
// written (add = 0) or added (add = 1) at the marker's body-order index.
// kSkinRows: the first reaction of a step on skin lists walks the transposed
// skin row, keeps the pairs the fluid's first pass keeps (cutoff_r from the
// fluid's side, on the same positions: the test is the pass's own) and
// writes them as this step's transposed rows for the second reaction.
template <class R>
constexpr int kMarkerForceBlocks = std::is_same<R, float>::value ? 8 : 4;
template <class R, bool kSkinRows>
__global__ void __launch_bounds__(kSphBlock, kMarkerForceBlocks<R>) k_sph_marker_force(SphDev d, double w, int add) {
    const int t = blockIdx.x * kSphPerBlock + threadIdx.x / kQuad;
    if (t >= d.NM) return;
    const int sub = threadIdx.x & 3;
    const unsigned gm = quad_mask();
    using VR = V<R>;
    const double4 pm = d.mpos[t];
    const double3 rm = xyz(pm);
    const BView mv = marker_view(d);
    const VR g = cvt<R>(d.gravity);
    double3 F = mk3(0, 0, 0);
    // the pair (a, t) from the fluid's side: false when outside the exact
    // cutoff (tested only for skin rows), else its term is added
    auto term = [&](int a, bool test) {
        VR acc = v3r<R>(0, 0, 0);
        if constexpr (std::is_same<R, float>::value) {
            // the FP32 shadows hold what fluid_own rounds the FP64 records to;
            // the mass is the shadow's FP32 rounding (relative 6e-8)
            const int4 qa = d.posq[a];
            const float ha = __int_as_float(qa.w);
            const OwnPos<float> op{mk3(0, 0, 0), qa};
            float3 rij;
            float hj;
            pair_r<float>(op, mv.pos, mv.posq, d.q, t, rij, hj);
            if (test && !cutoff_f(rij, ha, hj, [&] { return d.pos[a]; }, d.mpos, t)) return false;
            const float4 va = d.velf[a], sa = d.stf[a];
            const FluidOwn<float> o{op, make_float3(va.x, va.y, va.z), sa.x, sa.y, sa.z, sa.w, hconst<float>(ha)};
            boundary_acc_r<R>(d, o, mv, t, rij, hj, g, acc);
            F -= (double)va.w * up(acc);
        } else {
            const double4 pa = d.pos[a];
            const OwnPos<double> op{xyz(pa), make_int4(0, 0, 0, 0)};
            double3 rij;
            double hj;
            pair_r<double>(op, mv.pos, mv.posq, d.q, t, rij, hj);
            if (test && !cutoff_r<double>(rij, hj, pa, d.mpos, t)) return false;
            const double4 va = d.vel[a];
            const FluidOwn<R> o = fluid_own<R>(d, a, pa, va, d.st[a]);
            boundary_acc_r<R>(d, o, mv, t, rij, hj, g, acc);
            F -= va.w * up(acc);
        }
        return true;
    };
    if constexpr (kSkinRows) {
        skin_loop(d.cntRV[t], d.nbRV, d.KR, t, d.nbR, d.cntR, pm, d.g, d.fStart, d.pos, -1,
                  [&](int a) { return term(a, true); });
    } else {
        const int cnt = d.cntR[t];
        if (cnt >= 0) {
            // the transposed list (k_sph_marker_lists, or the first reaction's
            // exact rows on skin lists): the fluid rows' pair set
            const int* __restrict__ row = d.nbR + row_base(t, d.KR) + sub;
            const int c = lane_count(cnt, sub);
            for (int k = 0; k < c; k++) term(__ldg(row + 32 * k), false);
        } else {
            // an overflowed row: the same pairs from the cell stencil, with the
            // cutoff test on the build-time positions
            Stencil st = stencil_of(rm, d.g);
            for_stencil_rows(st, d.g, d.fStart, [&](int b, int e) {
                for (int a = b + sub; a < e; a += kQuad) {
                    const double4 la = d.lpos[a];
                    const double cut = 2.0 * fmax(la.w, pm.w);
                    const double3 r = xyz(la) - rm;
                    if ((cut * cut - dot(r, r)) >= 0.) term(a, false);
                }
            });
        }
    }
    F.x = quad_sum(F.x, gm);
    F.y = quad_sum(F.y, gm);
    F.z = quad_sum(F.z, gm);
    if (sub != 0) return;
    const int k = d.mid[t];
    const double3 prev = add ? xyz(d.mforce[k]) : mk3(0, 0, 0);
    d.mforce[k] = d4(prev + w * F, 0);
}

// calDummyParticleNormalKernel (WCSPHIntegrationKernel.cu:4-40) over the
// dummy-dummy pairs (j != i within 2 max(h)), walked in stencil order; the
// pairs are also written out as an ELL list for inspection.
__global__ void k_sph_dummy_normals(int nd, GridDesc g, const int* __restrict__ dStart, const double4* __restrict__ dpos,
                                    const double4* __restrict__ dvel, const double* __restrict__ drho,
                                    double4* __restrict__ dnorm, int K, int* __restrict__ nb, int* __restrict__ cnt,
                                    DevStatus* status) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nd) return;
    double4 pi = dpos[i];
    double3 ri = xyz(pi);
    double3 th = mk3(0, 0, 0);
    int c = 0;
    Stencil st = stencil_of(ri, g);
    for_stencil_rows(st, g, dStart, [&](int b, int e) {
        for (int j = b; j < e; j++) {
            if (j == i) continue;
            double4 pj = dpos[j];
            double cut = 2.0 * fmax(pi.w, pj.w);
            double3 r = ri - xyz(pj);
            if ((cut * cut - dot(r, r)) >= 0.) {
                if (c < K) nb[(size_t)c * nd + i] = j;
                c++;
                double rl = len(r);
                double f = gradw_factor<double>(rl, 0.5 * (pi.w + pj.w));
                th -= dvel[j].w / drho[j] * (f * r);
            }
        }
    });
    if (c > K) {
        atomicMax(&status->need_rev, c);
        atomicExch(&status->overflow, 1);
        c = K;
    }
    cnt[i] = c;
    dnorm[i] = (len2(th) > 1.e-10) ? d4(th / len(th), 0) : make_double4(0, 0, 0, 0);
}

// Copies continuing batch members' fluid state from another scene.  Member k
// holds caller ids [srcStart[k], srcStart[k] + num[k]) there (the table is
// sorted by srcStart) and [dstStart[k], ...) here; for the source particle at
// sorted slot t, dstSlot maps its destination id to its current slot here.
// Positions are translated by the member's shift.
__global__ void k_sph_copy_members(int nsrc, const int* __restrict__ srcId, const double4* __restrict__ spos,
                                   const double4* __restrict__ svel, const double4* __restrict__ sst,
                                   const double* __restrict__ sdrho, int count, const int* __restrict__ srcStart,
                                   const int* __restrict__ dstStart, const int* __restrict__ num,
                                   const double4* __restrict__ shift, const int* __restrict__ dstSlot,
                                   double4* __restrict__ dpos, double4* __restrict__ dvel, double4* __restrict__ dst,
                                   double* __restrict__ ddrho) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nsrc) return;
    const int id = srcId[t];
    // last member starting at or before id
    int lo = 0, hi = count - 1, k = -1;
    while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        if (srcStart[mid] <= id) {
            k = mid;
            lo = mid + 1;
        } else {
            hi = mid - 1;
        }
    }
    if (k < 0 || id >= srcStart[k] + num[k]) return;  // not carried
    const int u = dstSlot[dstStart[k] + (id - srcStart[k])];
    const double4 p = spos[t];
    const double4 sh = shift[k];
    dpos[u] = make_double4(p.x + sh.x, p.y + sh.y, p.z + sh.z, p.w);
    dvel[u] = svel[t];
    dst[u] = sst[t];
    ddrho[u] = sdrho[t];
}
__global__ void k_sph_slot_of(int n, const int* __restrict__ id, int* __restrict__ slot) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) slot[id[t]] = t;
}

// ================================================================ host =====
// Marker offsets of a ball of radius R: shells l = 0, 1, ... at radius
// r_l = R - (l + 1/2) dx while l dx < 2 h and r_l > dx / 4 (the layers a
// fluid particle outside the surface can reach), shell l carrying
// n_l = max(1, round(4 pi r_l^2 / dx^2)) points on the golden-angle spiral
// z_k = 1 - (2k + 1) / n_l, phi_k = k pi (3 - sqrt 5).  A ball too small
// for any shell gets one marker at its centre.
static void marker_offsets(double R, double dx, double h, std::vector<double3>& out) {
    const double ga = kPi * (3.0 - std::sqrt(5.0));
    for (int l = 0; l * dx < 2.0 * h; l++) {
        const double r = R - (l + 0.5) * dx;
        if (!(r > 0.25 * dx)) break;
        const long nl = std::max(1L, std::lround(4.0 * kPi * r * r / (dx * dx)));
        for (long k = 0; k < nl; k++) {
            const double z = 1.0 - (2.0 * k + 1.0) / (double)nl;
            const double rho = std::sqrt(std::max(0.0, 1.0 - z * z));
            const double phi = ga * (double)k;
            out.push_back(mk3(r * rho * std::cos(phi), r * rho * std::sin(phi), r * z));
        }
    }
    if (out.empty()) out.push_back(mk3(0, 0, 0));
}

// FP64 conservation diagnostics of the fluid, per particle, summed by
// diag_reduce: 0 mass, 1-3 momentum sum m v, 4 kinetic energy, 5 potential
// energy -sum m g.x, 6 sum of the density changes (Delta rho), 7 volume
// sum m / rho.
struct SphDiagTerm {
    const double4* pos;
    const double4* vel;
    const double4* st;
    const double* drho;
    double3 g;
    __device__ void operator()(int i, double* v) const {
        const double4 p = pos[i], u = vel[i];
        const double m = u.w;
        v[0] = m;
        v[1] = m * u.x; v[2] = m * u.y; v[3] = m * u.z;
        v[4] = 0.5 * m * (u.x * u.x + u.y * u.y + u.z * u.z);
        v[5] = -m * (g.x * p.x + g.y * p.y + g.z * p.z);
        v[6] = drho[i];
        v[7] = m / st[i].x;
    }
};

struct SphScene {
    cudaStream_t s = 0;
    int precision = DEMSPH_PRECISION_FP64;
    bool ready = false;
    // host staging: fluid and dummy particles in caller order
    struct HostSet {
        HostVec<double4> pos, vel, st;  // st = (rho, p, c, nu)
        HostVec<double> rho0, drho;
        size_t size() const { return pos.size(); }
    } hf, hd;
    double3 gravity{0, 0, 0};
    double dt = 0;
    long iStep = 0;
    double time = 0;
    int KF = 96, KD = 64, KDD = 96;
    double listHeadroom = 0.125;  // row capacity above the initial longest row (autotuner)
    CellTable fCells, dCells;
    DBuf<double4> pos[2], vel[2], st[2];
    DBuf<double> rho0[2], drho[2];
    DBuf<int> id[2];
    DBuf<double4> acc;
    DBuf<float4> posf, dposf;
    DBuf<float4> velf[2], stf[2], dvelf, dstf, dnormf;  // FP32 shadows
    DBuf<int4> posq[2], dposq;                           // fixed-point positions
    float q = 0;
    double invq = 0;
    float eps = 0;
    int P = 0, Vv = 0, S = 0, R0 = 0, D = 0, ID = 0;
    int L = 0;  // pos buffer the current lists were built from
    DBuf<double4> dpos, dvel, dst, dnorm;
    DBuf<double> drhoD;  // dummy densities (normals only)
    DBuf<int> did;
    DBuf<int> nbF, cntF, nbD, cntD, nbDD, cntDD;
    DBuf<DevStatus> status;
    DBuf<double> diagScratch;
    bool haveLists = false;

    // Skin lists (coupled scenes too, with the markers' rows): rows hold every candidate
    // within cutoff + skin at the last rebuild; a step rebuilds them (cell
    // sort, reorder, list build, all gated on the device) only when some
    // particle has drifted half the skin, and its first momentum pass keeps
    // the pairs within the exact cutoff.  The grid's cells are
    // 2 h_max (1 + skinMax) wide so that the 27-cell stencil covers the skin.
    float skinMax = 0.04f;   // fraction of 2 h_max the grid allows (fixed at initialisation)
    float skinFrac = 0.04f;  // fraction in use (0: exact lists every step)
    double cellFactor = 1.0;  // grid cell = cellFactor x 2 h_max (1 + skin) (autotuner)
    double hmaxGrid = 0;
    DBuf<int> nbV, cntV, nbVD, cntVD;
    DBuf<double4> xb;
    DBuf<SkinState> skinState;
    bool skin_on() const { return skinFrac > 0; }
    float skin_abs() const { return (float)(2.0 * hmaxGrid * skinFrac); }
    // The next step rebuilds the skin lists (after any host-side change).
    void skin_force() {
        if (skinState.p) DEMSPH_CUDA(cudaMemsetAsync(&skinState.p->force, 1, 1, s));
    }

    int nF = 0, nD = 0;  // fluid / dummy counts (the host sets before initialisation)
    int N() const { return nF; }
    int ND() const { return nD; }
    float hUni = 0;      // the common h when uniformH
    // Uniform particle constants (fluid h, m, c, nu; dummy m, c, nu, rho0,
    // dummy h = fluid h): the mixed-precision passes then run
    // k_sph_accel_u / k_sph_density_u.  uniKernels = false keeps the general
    // passes (for comparisons).
    struct Uniform {
        bool on = false;
        double h = 0, mF = 0, cF = 0, nuF = 0, mD = 0, cD = 0, nuD = 0, rho0D = 0;
        bool operator==(const Uniform& o) const {
            return on == o.on && h == o.h && mF == o.mF && cF == o.cF && nuF == o.nuF && mD == o.mD && cD == o.cD &&
                   nuD == o.nuD && rho0D == o.rho0D;
        }
    } uni;
    bool uniKernels = true;
    static Uniform uniform_of(const HostSet& f, const HostSet& dm) {
        Uniform u;
        if (f.size() == 0) return u;
        u.h = f.pos[0].w; u.mF = f.vel[0].w; u.cF = f.st[0].z; u.nuF = f.st[0].w;
        bool ok = true;
        for (size_t k = 0; k < f.size() && ok; k++)
            ok = f.pos[k].w == u.h && f.vel[k].w == u.mF && f.st[k].z == u.cF && f.st[k].w == u.nuF;
        if (dm.size()) {
            u.mD = dm.vel[0].w; u.cD = dm.st[0].z; u.nuD = dm.st[0].w; u.rho0D = dm.rho0[0];
            for (size_t k = 0; k < dm.size() && ok; k++)
                ok = dm.pos[k].w == u.h && dm.vel[k].w == u.mD && dm.st[k].z == u.cD && dm.st[k].w == u.nuD &&
                     dm.rho0[k] == u.rho0D;
        }
        u.on = ok;
        return u;
    }
    // The uniform-constant passes (mixed precision); with markers they read
    // the unpacked shadows (packed only when nM == 0).
    bool uni_path() const { return uni.on && uniKernels && precision != DEMSPH_PRECISION_FP64; }
    UniK uni_consts() const {
        UniK k{};
        const double h = uni.h, qd = (double)q;
        k.invhq = (float)(qd / h);
        k.K = (float)(21.0 / (16.0 * kPi * h * h * h * h));
        k.c2q = (float)((2.0 * h / qd) * (2.0 * h / qd));
        k.cF = (float)uni.cF;
        k.mF2 = (float)(2.0 * uni.mF);
        k.bF = (float)(2.0 * uni.nuF * uni.mF);
        k.mF = (float)uni.mF;
        k.mD = (float)uni.mD;
        k.mD2 = (float)(2.0 * uni.mD);
        k.bD = (float)(2.0 * (0.5 * (uni.nuF + uni.nuD)) * uni.mD);
        k.cbarD = (float)(0.5 * (uni.cF + uni.cD));
        k.invcD2 = uni.cD > 0 ? (float)(1.0 / (uni.cD * uni.cD)) : 0.0f;
        k.rho0D = (float)uni.rho0D;
        k.gq = make_float3((float)(gravity.x * qd), (float)(gravity.y * qd), (float)(gravity.z * qd));
        return k;
    }

    // Coupled DEM balls.  Each is sampled by markers (moving boundary
    // particles) on shells inside its surface; body b owns the markers
    // [hBStart[b], hBStart[b+1]) of the body-order arrays.  The markers are
    // placed from the balls' state at the start of each coupled step and stay
    // where they are when the fluid is stepped alone.
    int nM = 0, KM = 48, KR = 96, nBody = 0;
    std::vector<int> hBall, hBStart{0}, hMb;
    int maxMarkersPerBody = 0;
    std::vector<double4> hMoff, hMrec;  // offset (x, y, z, h); (c, nu, rho0, m)
    demsph_dem_t coupledDem = nullptr;
    DBuf<int> mb, mid, bBall, bStart;
    DBuf<double4> moff, mrec, mtmp, mpos, mvel, mst, mnorm, mforce;
    DBuf<float4> mposf, mvelf, mstf, mnormf;
    DBuf<int4> mposq;
    DBuf<int> nbM, cntM, nbR, cntR;
    DBuf<int> nbMV, cntMV, nbRV, cntRV;  // skin rows of the fluid-marker pairs
    DBuf<double4> xbM;                   // marker positions at the last skin rebuild (body order)
    CellTable mCells;
    DemBodies bodies{};
    bool coupling = false;  // inside a coupled block: place markers, compute reactions
    // Graphs of kCoupledSteps coupled steps, keyed by both scenes' buffer
    // state; dropped when either scene drops its own graphs (buffers or
    // kernel arguments changed) or the DEM substep count changes.
    static constexpr int kCoupledSteps = 10;
    GraphSet cgraph;
    long cgSphEpoch = -1, cgDemEpoch = -1;
    int cgSub = 0;

    SphDev dev() {
        SphDev d{};
        d.N = N(); d.ND = ND(); d.KF = KF; d.KD = KD;
        d.g = fCells.g;
        d.fStart = fCells.start.p;
        d.dStart = dCells.start.p;
        d.pos = pos[P].p; d.lpos = pos[L].p; d.vel = vel[Vv].p; d.st = st[S].p; d.rho0 = rho0[R0].p; d.drho = drho[D].p;
        d.acc = acc.p;
        d.dpos = dpos.p; d.dvel = dvel.p; d.dst = dst.p; d.dnorm = dnorm.p;
        d.velf = velf[Vv].p; d.stf = stf[S].p;
        d.posq = posq[P].p; d.dposq = dposq.p; d.q = q; d.invq = invq;
        d.dvelf = dvelf.p; d.dstf = dstf.p; d.dnormf = dnormf.p;
        d.nbF = nbF.p; d.cntF = cntF.p; d.nbD = nbD.p; d.cntD = cntD.p;
        d.posf = posf.p; d.dposf = dposf.p; d.eps = eps;
        d.gravity = gravity;
        d.status = status.p;
        d.NM = nM; d.KM = KM;
        d.mStart = mCells.start.p;
        d.mpos = mpos.p; d.mvel = mvel.p; d.mst = mst.p; d.mnorm = mnorm.p;
        d.mposf = mposf.p; d.mvelf = mvelf.p; d.mstf = mstf.p; d.mnormf = mnormf.p; d.mposq = mposq.p;
        d.mid = mid.p; d.nbM = nbM.p; d.cntM = cntM.p; d.mforce = mforce.p;
        d.KR = KR; d.nbR = nbR.p; d.cntR = cntR.p;
        d.nbMV = nbMV.p; d.cntMV = cntMV.p; d.nbRV = nbRV.p; d.cntRV = cntRV.p;
        d.skin = 0.0f; d.gate = nullptr;
        d.nbV = nbV.p; d.cntV = cntV.p; d.nbVD = nbVD.p; d.cntVD = cntVD.p;
        d.xb = xb.p; d.maxd2 = skinState.p ? skinState.p->maxd2 : nullptr;
        if (uni.on) d.uk = uni_consts();
        return d;
    }

    void alloc_lists() {
        graph.reset();  // the captured kernels hold the old list buffers
        size_t n = (size_t)N();
        nbF.alloc(row_words(n, KF), s, false);
        cntF.alloc(n, s, true);
        nbD.alloc(row_words(n, std::max(KD, 1)), s, false);
        cntD.alloc(n, s, true);
        if (nM > 0) {
            nbM.alloc(row_words(n, KM), s, false);
            cntM.alloc(n, s, true);
            nbR.alloc(row_words((size_t)nM, KR), s, false);
            cntR.alloc(nM, s, true);
        }
        if (skinMax > 0) {
            nbV.alloc(row_words(n, KF), s, false);
            cntV.alloc(n, s, true);
            nbVD.alloc(row_words(n, std::max(KD, 1)), s, false);
            cntVD.alloc(n, s, true);
            if (xb.n < n) xb.alloc(n, s, true);
            if (nM > 0) {
                nbMV.alloc(row_words(n, KM), s, false);
                cntMV.alloc(n, s, true);
                nbRV.alloc(row_words((size_t)nM, KR), s, false);
                cntRV.alloc(nM, s, true);
                if (xbM.n < (size_t)nM) xbM.alloc(nM, s, true);
            }
            if (!skinState.p) skinState.alloc(1, s, true);
            skin_force();
        }
    }

    // WCSPHSolver::neighborSearch (WCSPHSolver.h:150-285): fluid cell sort,
    // reorder, neighbour lists.
    // all fluid and dummy particles share one h: the list build keeps the
    // candidate index in the staged record
    bool uniformH = false;
    int listShape = 0;  // index into kListShapes (autotuned)
    // Blocks of a list build over ncell cells: one warp per cell up to eight
    // waves of the shape's resident blocks, the warps striding beyond.
    template <int kShape>
    static unsigned list_grid(int ncell) {
        const unsigned cap = (unsigned)(device_sms() * kListShapes[kShape].minBlocks * 8);
        return std::min(grid_for(ncell, kListShapes[kShape].warps), cap);
    }
    template <int S>
    void launch_lists_shape(const SphDev& d, bool withMarkers) {
        constexpr int W = kListShapes[S].warps;
        const unsigned grid = list_grid<S>(fCells.ncell);
        if (withMarkers && nM > 0) {
            if (uniformH) k_sph_lists_cell<true, S, true><<<grid, 32 * W, 0, s>>>(d, fCells.ncell);
            else k_sph_lists_cell<false, S, true><<<grid, 32 * W, 0, s>>>(d, fCells.ncell);
            if (coupling) {  // the transposed rows the reaction reads
                if (uniformH) k_sph_marker_lists<true, S><<<grid, 32 * W, 0, s>>>(d, fCells.ncell);
                else k_sph_marker_lists<false, S><<<grid, 32 * W, 0, s>>>(d, fCells.ncell);
                g_launches += 1;
            }
        } else {
            if (uniformH) k_sph_lists_cell<true, S, false><<<grid, 32 * W, 0, s>>>(d, fCells.ncell);
            else k_sph_lists_cell<false, S, false><<<grid, 32 * W, 0, s>>>(d, fCells.ncell);
        }
    }
    // withMarkers: the fluid-marker rows (and, inside a coupled step, the
    // transposed rows) come out of the same build (exact lists every step).
    void launch_lists(const SphDev& d, bool withMarkers = true) {
        switch (listShape) {
            case 0: launch_lists_shape<0>(d, withMarkers); break;
            case 1: launch_lists_shape<1>(d, withMarkers); break;
            case 2: launch_lists_shape<2>(d, withMarkers); break;
            default: launch_lists_shape<3>(d, withMarkers); break;
        }
    }
    // Skin lists with markers: the fluid-marker skin rows and the transposed
    // skin rows, at a (gated) skin rebuild.
    template <int S>
    void launch_marker_rows_shape(const SphDev& d) {
        constexpr int W = kListShapes[S].warps;
        const unsigned grid = list_grid<S>(fCells.ncell);
        if (uniformH) k_sph_marker_rows<true, S><<<grid, 32 * W, 0, s>>>(d, fCells.ncell);
        else k_sph_marker_rows<false, S><<<grid, 32 * W, 0, s>>>(d, fCells.ncell);
        const unsigned mgrid = list_grid<S>(mCells.ncell);
        if (uniformH) k_sph_marker_lists<true, S><<<mgrid, 32 * W, 0, s>>>(d, mCells.ncell);
        else k_sph_marker_lists<false, S><<<mgrid, 32 * W, 0, s>>>(d, mCells.ncell);
        g_launches += 2;
    }
    void launch_marker_rows(const SphDev& d) {
        switch (listShape) {
            case 0: launch_marker_rows_shape<0>(d); break;
            case 1: launch_marker_rows_shape<1>(d); break;
            case 2: launch_marker_rows_shape<2>(d); break;
            default: launch_marker_rows_shape<3>(d); break;
        }
    }
    // Moves the fluid records (and their FP32 shadows) into this step's cell order.
    void permute(const int* gate = nullptr) {
        const int n = N();
        k_sph_permute<<<grid_for(n, 256), 256, 0, s>>>(n, fCells.sorted.p, pos[P].p, vel[Vv].p, st[S].p, rho0[R0].p,
                                                       drho[D].p, id[ID].p, pos[P ^ 1].p, vel[Vv ^ 1].p, st[S ^ 1].p,
                                                       rho0[R0 ^ 1].p, drho[D ^ 1].p, id[ID ^ 1].p, posf.p,
                                                       velf[Vv ^ 1].p, stf[S ^ 1].p, posq[P ^ 1].p, fCells.g.mn,
                                                       invq, gate, packed ? 1 : 0);
        if (gate) {  // a device-side decision: copy back instead of flipping the indices
            k_sph_copy_back<<<grid_for(n, 256), 256, 0, s>>>(
                n, gate, pos[P ^ 1].p, vel[Vv ^ 1].p, st[S ^ 1].p, rho0[R0 ^ 1].p, drho[D ^ 1].p, id[ID ^ 1].p,
                velf[Vv ^ 1].p, stf[S ^ 1].p, posq[P ^ 1].p, pos[P].p, vel[Vv].p, st[S].p, rho0[R0].p, drho[D].p,
                id[ID].p, velf[Vv].p, stf[S].p, posq[P].p, xb.p);
            g_launches += 1;
        } else {
            P ^= 1; Vv ^= 1; S ^= 1; R0 ^= 1; D ^= 1; ID ^= 1;
        }
        L = P;
    }
    // Rewrites the fluid shadows after a host-side change of the records.
    void refresh_shadows() {
        const int n = N();
        k_sph_shadow<<<grid_for(n, 256), 256, 0, s>>>(n, vel[Vv].p, st[S].p, nullptr, velf[Vv].p, stf[S].p, nullptr);
        k_sph_fix<<<grid_for(n, 256), 256, 0, s>>>(n, pos[P].p, fCells.g.mn, invq, posq[P].p);
        g_launches += 2;
        if (packed) {
            k_sph_pack<<<grid_for(n, 256), 256, 0, s>>>(n, pos[P].p, vel[Vv].p, st[S].p, posq[P].p, velf[Vv].p, 1);
            g_launches += 1;
        }
        DEMSPH_LAUNCH_CHECK();
        skin_force();
    }
    // The fluid shadows' layout follows whether the uniform-constant passes
    // run (packed) or the general ones; called at the entry of every call
    // that launches the passes, outside any stream capture.
    bool packed = false;
    void sync_mode() {
        const bool want = ready && uni_path() && nM == 0;
        if (want == packed) return;
        packed = want;
        graph.reset();          // captured launches carry the layout
        oneStepAfter.clear();   // and the packed passes move the buffer indices differently
        const int n = N();
        k_sph_pack<<<grid_for(n, 256), 256, 0, s>>>(n, pos[P].p, vel[Vv].p, st[S].p, posq[P].p, velf[Vv].p,
                                                    packed ? 1 : 0);
        g_launches += 1;
        DEMSPH_LAUNCH_CHECK();
    }
    // Markers from the coupled balls' current state, in cell order.
    void place_markers() {
        marker_place(false);
        marker_sort(nullptr);
    }
    // The markers' positions in body order; with skin lists (drift) each
    // marker's drift since the last rebuild joins the rebuild decision.
    void marker_place(bool drift) {
        k_sph_marker_place<<<grid_for(nM, 256), 256, 0, s>>>(nM, mb.p, moff.p, bodies.pos, mtmp.p, xbM.p,
                                                             drift ? skinState.p->maxd2 : nullptr);
        g_launches += 1;
    }
    // Cell sort (gated on a skin rebuild: otherwise the slots keep the order
    // of the last rebuild, which the skin rows index) and the records in slot
    // order; a skin rebuild also re-anchors the drift.
    void marker_sort(const int* gate) {
        mCells.build(mtmp.p, nM, s, nullptr, false, gate);
        k_sph_marker_gather<<<grid_for(nM, 256), 256, 0, s>>>(
            nM, mCells.sorted.p, mtmp.p, mb.p, moff.p, mrec.p, bodies.vel, bodies.angv, fCells.g.mn, invq, mpos.p,
            mvel.p, mst.p, mnorm.p, mposf.p, mvelf.p, mstf.p, mnormf.p, mposq.p, mid.p, gate,
            gate ? xbM.p : nullptr);
        g_launches += 1 + mCells.launches;
        DEMSPH_LAUNCH_CHECK();
    }
    void neighbor_search() {
        const int n = N();
        if (coupling && nM > 0) place_markers();
        fCells.build(pos[P].p, n, s, id[ID].p);
        g_launches += fCells.launches;
        permute();
        SphDev d = dev();
        launch_lists(d);
        g_launches += 2;
        DEMSPH_LAUNCH_CHECK();
        haveLists = true;
        skin_force();  // the particles moved in memory: the skin rows are stale
    }
    // The step's rebuild of the skin lists, gated on the device's decision.
    void skin_rebuild() {
        if (condCapture) {
            skin_rebuild_conditional();
            return;
        }
        skin_rebuild_sort();
        skin_rebuild_lists();
    }
    // The decision and the gated cell sorts (in a coupled step the markers
    // are placed first: their drift joins the decision).
    void skin_rebuild_sort() {
        const int* gate = &skinState.p->rebuild;
        const bool move = coupling && nM > 0;
        if (move) marker_place(true);
        k_sph_skin_decide<<<1, kSkinSlots, 0, s>>>(skinState.p, (float)(0.25 * skin_abs() * skin_abs()),
                                                   cudaGraphConditionalHandle(), 0);
        if (move) marker_sort(gate);
        fCells.build(pos[P].p, N(), s, id[ID].p, false, gate);
        g_launches += 1 + fCells.launches;
    }

    // Conditional rebuild (a scene without markers, inside a stream capture):
    // the decision kernel, then an IF node whose body -- captured into the
    // node's graph on a helper stream -- is the cell sort, the reorder and the
    // skin-list build.  The body's kernels keep their device-side gate, so the
    // body does the same work as the gated launches outside graphs; they are
    // counted when a rebuild runs them, not per replay.
    bool condOK = true;         // the runtime took conditional capture so far
    bool condEnabled = false;   // demsph_sph_set_conditional_rebuild (off: profilers skip such graphs' kernels)
    bool condCapture = false;   // set while a block of steps is captured
    long long condBodyLaunches = 0;
    cudaStream_t condStream = nullptr;
    bool cond_wanted() const { return condOK && condEnabled && nM == 0 && skin_on(); }
    ~SphScene() {
        if (condStream) cudaStreamDestroy(condStream);
        if (statusEv) {
            cudaEventSynchronize(statusEv);
            cudaEventDestroy(statusEv);
        }
        if (hostStatus) cudaFreeHost(hostStatus);
    }
    void skin_rebuild_conditional() {
        cudaStreamCaptureStatus cs;
        cudaGraph_t g = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        DEMSPH_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
        cudaGraphConditionalHandle h;
        DEMSPH_CUDA(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
        k_sph_skin_decide<<<1, kSkinSlots, 0, s>>>(skinState.p, (float)(0.25 * skin_abs() * skin_abs()), h, 1);
        g_launches += 1;
        DEMSPH_LAUNCH_CHECK();
        DEMSPH_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
        cudaGraphNodeParams p{};
        p.type = cudaGraphNodeTypeConditional;
        p.conditional.handle = h;
        p.conditional.type = cudaGraphCondTypeIf;
        p.conditional.size = 1;
        cudaGraphNode_t node;
        DEMSPH_CUDA(cudaGraphAddNode(&node, g, deps, nd, &p));
        cudaGraph_t body = p.conditional.phGraph_out[0];
        if (!condStream) DEMSPH_CUDA(cudaStreamCreateWithFlags(&condStream, cudaStreamNonBlocking));
        DEMSPH_CUDA(cudaStreamBeginCaptureToGraph(condStream, body, nullptr, nullptr, 0,
                                                  cudaStreamCaptureModeThreadLocal));
        const cudaStream_t keep = s;
        const long long l0 = g_launches.load();
        s = condStream;
        try {
            const int* gate = &skinState.p->rebuild;
            fCells.build(pos[P].p, N(), s, id[ID].p, false, gate);
            g_launches += fCells.launches;
            skin_rebuild_lists();
        } catch (...) {
            s = keep;
            cudaGraph_t tmp = nullptr;
            cudaStreamEndCapture(condStream, &tmp);
            g_launches = l0;
            throw;
        }
        s = keep;
        condBodyLaunches = g_launches.load() - l0;
        g_launches = l0;
        cudaGraph_t out = nullptr;
        DEMSPH_CUDA(cudaStreamEndCapture(condStream, &out));
        DEMSPH_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    }
    // Captures a block of steps, with conditional rebuilds when they apply; a
    // runtime that refuses them leaves the block captured with the gated
    // launches (and later blocks too).
    template <class F>
    void capture_steps(StepGraph& gr, int nsteps, F&& body) {
        if (cond_wanted()) {
            const std::array<int, 7> idx = {P, Vv, S, R0, D, ID, L};
            const bool lists0 = haveLists;
            condCapture = true;
            try {
                gr.capture(nsteps, s, body);
                condCapture = false;
                return;
            } catch (const Status&) {
                condCapture = false;
                condOK = false;
                (void)cudaGetLastError();
                P = idx[0]; Vv = idx[1]; S = idx[2]; R0 = idx[3]; D = idx[4]; ID = idx[5]; L = idx[6];
                haveLists = lists0;
            }
        }
        gr.capture(nsteps, s, body);
    }
    // The gated reorder and skin-list build (with markers: the fluid-marker
    // skin rows and their transposed rows too).
    void skin_rebuild_lists() {
        const int* gate = &skinState.p->rebuild;
        permute(gate);
        launch_lists(skin_view(gate), false);
        g_launches += 2;
        if (nM > 0) {
            SphDev d = skin_view(gate);
            d.nbM = nbMV.p; d.cntM = cntMV.p; d.nbR = nbRV.p; d.cntR = cntRV.p;
            launch_marker_rows(d);
        }
        DEMSPH_LAUNCH_CHECK();
        haveLists = true;
    }
    // The device view the skin-list build writes through.
    SphDev skin_view(const int* gate) {
        SphDev d = dev();
        d.skin = skin_abs();
        d.gate = gate;
        d.nbF = nbV.p; d.cntF = cntV.p; d.nbD = nbVD.p; d.cntD = cntVD.p;
        return d;
    }
    // The first momentum pass of a step on the skin lists.
    void accel_skin() {
        SphDev d = dev();
        d.posOut = pos[P ^ 1].p;
        d.velOut = vel[Vv ^ 1].p;
        d.velfOut = velf[Vv ^ 1].p;
        d.posqOut = posq[P ^ 1].p;
        launch_accel(d, 0.5 * dt, dt, 1, coupling, true);
        P ^= 1;
        Vv ^= 1;
    }
    // The momentum pass (k_sph_accel) on the state d reads (with the markers'
    // terms when there are markers), preceded inside a coupled step by the
    // reaction on the markers (half of it from each of a step's two passes:
    // first = 1 writes, first = 0 adds).
    // skin: the first pass of a step on skin lists (first = 1).
    void launch_accel(const SphDev& d, double hdt, double tstep, int first, bool reaction, bool skin = false) {
        const int n = N();
        const unsigned grid = grid_for(n, kSphPerBlock);
        const bool fp64 = precision == DEMSPH_PRECISION_FP64;
        if (nM > 0) {
            if (reaction) {
                const unsigned mg = grid_for(nM, kSphPerBlock);
                if (skin) {
                    if (fp64) k_sph_marker_force<double, true><<<mg, kSphBlock, 0, s>>>(d, 0.5, 0);
                    else k_sph_marker_force<float, true><<<mg, kSphBlock, 0, s>>>(d, 0.5, 0);
                } else {
                    if (fp64) k_sph_marker_force<double, false><<<mg, kSphBlock, 0, s>>>(d, 0.5, first ? 0 : 1);
                    else k_sph_marker_force<float, false><<<mg, kSphBlock, 0, s>>>(d, 0.5, first ? 0 : 1);
                }
                g_launches += 1;
            }
            if (uni_path()) {
                if (skin) k_sph_accel_u<true, true><<<grid, kSphBlock, 0, s>>>(d, hdt, tstep, first);
                else k_sph_accel_u<false, true><<<grid, kSphBlock, 0, s>>>(d, hdt, tstep, first);
            } else if (skin) {
                if (fp64) k_sph_accel<double, true, true><<<grid, kSphBlock, 0, s>>>(d, hdt, tstep, first);
                else k_sph_accel<float, true, true><<<grid, kSphBlock, 0, s>>>(d, hdt, tstep, first);
            } else {
                if (fp64) k_sph_accel<double, true><<<grid, kSphBlock, 0, s>>>(d, hdt, tstep, first);
                else k_sph_accel<float, true><<<grid, kSphBlock, 0, s>>>(d, hdt, tstep, first);
            }
            g_launches += 1;
        } else if (packed) {
            if (skin) k_sph_accel_u<true><<<grid, kSphBlock, 0, s>>>(d, hdt, tstep, first);
            else k_sph_accel_u<false><<<grid, kSphBlock, 0, s>>>(d, hdt, tstep, first);
            g_launches += 1;
        } else {
            if (skin) {
                if (fp64) k_sph_accel<double, false, true><<<grid, kSphBlock, 0, s>>>(d, hdt, tstep, first);
                else k_sph_accel<float, false, true><<<grid, kSphBlock, 0, s>>>(d, hdt, tstep, first);
            } else {
                if (fp64) k_sph_accel<double, false><<<grid, kSphBlock, 0, s>>>(d, hdt, tstep, first);
                else k_sph_accel<float, false><<<grid, kSphBlock, 0, s>>>(d, hdt, tstep, first);
            }
            g_launches += 1;
        }
        DEMSPH_LAUNCH_CHECK();
    }
    void accel(int first) {
        SphDev d = dev();
        d.posOut = pos[P ^ 1].p;
        d.velOut = vel[Vv ^ 1].p;
        d.velfOut = velf[Vv ^ 1].p;
        d.posqOut = posq[P ^ 1].p;
        launch_accel(d, 0.5 * dt, dt, first, coupling);
        if (first) P ^= 1;
        Vv ^= 1;
    }
    void density() {
        SphDev d = dev();
        const int n = N();
        d.stOut = st[S ^ 1].p;
        d.stfOut = stf[S ^ 1].p;
        const unsigned grid = grid_for(n, kSphPerBlock);
        const bool fp64 = precision == DEMSPH_PRECISION_FP64;
        if (nM > 0) {
            if (uni_path()) k_sph_density_u<true><<<grid, kSphBlock, 0, s>>>(d, dt);
            else if (fp64) k_sph_density<double, true><<<grid, kSphBlock, 0, s>>>(d, dt);
            else k_sph_density<float, true><<<grid, kSphBlock, 0, s>>>(d, dt);
            g_launches += 1;
        } else if (packed) {
            // the packed shadows carry rho and p: the pass writes the next
            // buffers of positions and velocities (copies of the records, with
            // the new rho / p in their shadows) as well
            d.posOut = pos[P ^ 1].p;
            d.velOut = vel[Vv ^ 1].p;
            d.posqOut = posq[P ^ 1].p;
            d.velfOut = velf[Vv ^ 1].p;
            k_sph_density_u<false><<<grid, kSphBlock, 0, s>>>(d, dt);
            g_launches += 1;
            P ^= 1;
            Vv ^= 1;
        } else {
            if (fp64) k_sph_density<double, false><<<grid, kSphBlock, 0, s>>>(d, dt);
            else k_sph_density<float, false><<<grid, kSphBlock, 0, s>>>(d, dt);
            g_launches += 1;
        }
        DEMSPH_LAUNCH_CHECK();
        S ^= 1;
    }
    // One pass of the WCSPHSolver::solve loop (WCSPHSolver.h:607-621).
    void step_body() {
        if (skin_on()) {
            skin_rebuild();
            accel_skin();
        } else {
            neighbor_search();
            accel(1);
        }
        density();
        accel(0);
    }
    void step_once() {
        iStep++;
        time += dt;
        step_body();
    }
    // Two steps per graph: every ping-pong index is back to its parity.
    GraphSet graph;
    bool useGraphs = true;
    int index_key() const { return P | Vv << 1 | S << 2 | R0 << 3 | D << 4 | ID << 5; }

    // One step with a CUDA event after every phase, on the scene stream:
    // 0 cell sort, 1 permute + lists, 2 accel + kick + drift, 3 continuity + EOS,
    // 4 accel + kick.  Adds each phase's milliseconds into ms[0..4].
    void step_profiled(double* ms) {
        cudaEvent_t ev[6];
        for (auto& e : ev) DEMSPH_CUDA(cudaEventCreate(&e));
        iStep++;
        time += dt;
        const int n = N();
        DEMSPH_CUDA(cudaEventRecord(ev[0], s));
        if (skin_on()) {
            // 0 decision + gated cell sort, 1 gated reorder + skin lists, 2 first pass on the skin rows
            skin_rebuild_sort();
            DEMSPH_CUDA(cudaEventRecord(ev[1], s));
            skin_rebuild_lists();
            DEMSPH_CUDA(cudaEventRecord(ev[2], s));
            accel_skin();
        } else {
            fCells.build(pos[P].p, n, s, id[ID].p);
            g_launches += fCells.launches;
            DEMSPH_CUDA(cudaEventRecord(ev[1], s));
            permute();
            SphDev d = dev();
            launch_lists(d);
            g_launches += 2;
            haveLists = true;
            DEMSPH_CUDA(cudaEventRecord(ev[2], s));
            accel(1);
        }
        DEMSPH_CUDA(cudaEventRecord(ev[3], s));
        density();
        DEMSPH_CUDA(cudaEventRecord(ev[4], s));
        accel(0);
        DEMSPH_CUDA(cudaEventRecord(ev[5], s));
        DEMSPH_CUDA(cudaEventSynchronize(ev[5]));
        for (int k = 0; k < 5; k++) {
            float t = 0;
            DEMSPH_CUDA(cudaEventElapsedTime(&t, ev[k], ev[k + 1]));
            ms[k] += t;
        }
        for (auto& e : ev) cudaEventDestroy(e);
    }

    DevStatus read_status() {
        DevStatus h{};
        DEMSPH_CUDA(cudaMemcpyAsync(&h, status.p, sizeof h, cudaMemcpyDeviceToHost, s));
        DEMSPH_CUDA(cudaStreamSynchronize(s));
        return h;
    }
    void clear_status() { DEMSPH_CUDA(cudaMemsetAsync(status.p, 0, sizeof(DevStatus), s)); }
    void grow(const DevStatus& st2) {
        if (st2.need_pairs > KF) KF = st2.need_pairs + st2.need_pairs / 4 + 1;
        if (st2.need_aux > KD) KD = st2.need_aux + st2.need_aux / 4 + 1;
        if (st2.need_mark > KM) KM = st2.need_mark + st2.need_mark / 4 + 1;
        if (st2.need_mrev > KR) KR = st2.need_mrev + st2.need_mrev / 4 + 1;
        alloc_lists();
        haveLists = false;  // rebuilt by the next neighbour search
    }

    // Saved dynamic state for overflow replay.
    struct Snap {
        std::vector<std::unique_ptr<DBuf<char>>> bufs;
        std::vector<void*> dst;
        std::vector<size_t> bytes;
        long iStep;
        double time;
        int P, Vv, S, R0, D, ID, L;
        // with the skin lists (rows, rebuild positions, rebuild state), so
        // that the steps after a restore use the rows the steps after the
        // snapshot used; valid while the list capacities are unchanged
        bool lists = false;
        int KF = 0, KD = 0;
        bool haveLists = false;
    };
    // The copies are collected and issued as copy_list launches at the end of
    // take() (and of restore()).
    std::vector<CopyItem> snapCopies;
    template <class T>
    void snap_add(Snap& sn, DBuf<T>& b) {
        if (!b.p || b.n == 0) return;
        auto c = std::make_unique<DBuf<char>>();
        c->alloc(b.bytes(), s, false);
        snapCopies.push_back({c->p, b.p, b.bytes()});
        sn.dst.push_back((void*)b.p);
        sn.bytes.push_back(b.bytes());
        sn.bufs.push_back(std::move(c));
    }
    void take(Snap& sn, bool withLists = false) {
        snapCopies.clear();
        take_buffers(sn, withLists);
        g_launches += copy_list(snapCopies, s);
        DEMSPH_LAUNCH_CHECK();
    }
    void take_buffers(Snap& sn, bool withLists) {
        sn.iStep = iStep; sn.time = time; sn.P = P; sn.Vv = Vv; sn.S = S; sn.R0 = R0; sn.D = D; sn.ID = ID; sn.L = L;
        snap_add(sn, pos[P]); snap_add(sn, vel[Vv]); snap_add(sn, st[S]); snap_add(sn, rho0[R0]);
        snap_add(sn, drho[D]); snap_add(sn, id[ID]);
        sn.lists = withLists && skin_on() && nM == 0 && skinState.p;
        if (sn.lists) {
            sn.KF = KF; sn.KD = KD; sn.haveLists = haveLists;
            snap_add(sn, nbV); snap_add(sn, cntV); snap_add(sn, nbVD); snap_add(sn, cntVD); snap_add(sn, xb);
            snap_add(sn, skinState);
            snap_add(sn, posf);
        }
    }
    void restore(Snap& sn) {
        const bool lists = sn.lists && sn.KF == KF && sn.KD == KD;
        snapCopies.clear();
        for (size_t k = 0; k < sn.bufs.size(); k++) {
            if (!lists && k >= 6) break;  // the state records come first
            snapCopies.push_back({sn.dst[k], sn.bufs[k]->p, sn.bytes[k]});
        }
        g_launches += copy_list(snapCopies, s);
        DEMSPH_LAUNCH_CHECK();
        iStep = sn.iStep; time = sn.time; P = sn.P; Vv = sn.Vv; S = sn.S; R0 = sn.R0; D = sn.D; ID = sn.ID; L = sn.L;
        refresh_shadows();  // the FP32 / fixed-point copies follow the restored records (and force a skin rebuild)
        if (lists) {
            // the restored rows and rebuild state stand: no forced rebuild
            DEMSPH_CUDA(cudaMemsetAsync(&skinState.p->force, 0, 1, s));
            haveLists = sn.haveLists;
        }
    }
    // Steps without a state snapshot: a list row that overflows its capacity
    // is walked from the cell table by the passes (same neighbours), so an
    // overflow never changes results; the lists are regrown for later calls.
    // The status of a run's steps is copied to pinned host memory when they
    // are queued and looked at by the next call, so step() returns without
    // waiting for the device.  Nothing in a step depends on it: a list row
    // that overflows is walked from the cell table by the passes (same
    // neighbours), and the lists are regrown before the next steps.  The
    // device status keeps its flags until they are consumed, so a later
    // copy carries every earlier overflow.
    DevStatus* hostStatus = nullptr;
    cudaEvent_t statusEv = nullptr;
    bool statusPending = false;
    void status_async() {
        if (!hostStatus) {
            DEMSPH_CUDA(cudaHostAlloc((void**)&hostStatus, sizeof(DevStatus), cudaHostAllocDefault));
            DEMSPH_CUDA(cudaEventCreateWithFlags(&statusEv, cudaEventDisableTiming));
        }
        DEMSPH_CUDA(cudaMemcpyAsync(hostStatus, status.p, sizeof(DevStatus), cudaMemcpyDeviceToHost, s));
        DEMSPH_CUDA(cudaEventRecord(statusEv, s));
        statusPending = true;
    }
    // Acts on the last queued status once the device has written it (wait:
    // block until then); an overflow regrows the lists and clears the flags.
    void consume_status(bool wait) {
        if (!statusPending) return;
        if (wait) {
            DEMSPH_CUDA(cudaEventSynchronize(statusEv));
        } else {
            const cudaError_t q = cudaEventQuery(statusEv);
            if (q == cudaErrorNotReady) {  // still queued: a later call looks
                if (cudaPeekAtLastError() == cudaErrorNotReady) (void)cudaGetLastError();
                return;
            }
            DEMSPH_CUDA(q);
        }
        statusPending = false;
        const DevStatus st2 = *hostStatus;
        if (st2.overflow) {
            grow(st2);
            clear_status();
        }
    }
    void run(long n) {
        if (!ready) throw Status(DEMSPH_ERR_NOT_READY, "scene not initialised");
        if (n <= 0) return;
        sync_mode();
        consume_status(false);
        long k = 0;
        if (useGraphs && n >= 2) {
            StepGraph& gr = graph.at(index_key());
            if (!gr.ready()) capture_steps(gr, 2, [&] { step_body(); step_body(); });
            for (; k + 2 <= n; k += 2) {
                gr.launch(s);
                iStep += 2;
                time += 2 * dt;
            }
        }
        // a single step (step(1), or the odd one): a one-step graph per
        // ping-pong state, with the host's indices set to the state it leaves
        for (; k < n && useGraphs; k++) {
            const int key = index_key() | kOneStepKey;
            StepGraph& gr = graph.at(key);
            if (!gr.ready()) {
                capture_steps(gr, 1, [&] { step_body(); });  // moves the host's indices on
                oneStepAfter[key] = {P, Vv, S, R0, D, ID, L};
            } else {
                const auto& a = oneStepAfter.at(key);
                P = a[0]; Vv = a[1]; S = a[2]; R0 = a[3]; D = a[4]; ID = a[5]; L = a[6];
            }
            gr.launch(s);
            iStep += 1;
            time += dt;
        }
        for (; k < n; k++) step_once();
        status_async();
    }
    static constexpr int kOneStepKey = 1 << 10;
    std::map<int, std::array<int, 7>> oneStepAfter;  // one-step graph key -> indices after the step

    // ------------------------------------------------ coupled DEM balls ----
    // Samples balls[0..n) of the DEM scene (radii read from its device
    // state) with markers of spacing dx and smoothing length hm, sound speed
    // c, viscosity nu and rest density rho0 (mass rho0 dx^3), and places them
    // at the balls' current positions.
    void add_bodies(demsph_dem_t dem, long n, const int* balls, double dx, double hm, double c, double nu,
                    double rho0) {
        if (!ready) throw Status(DEMSPH_ERR_NOT_READY, "scene not initialised");
        if (coupledDem && coupledDem != dem) throw Status(DEMSPH_ERR_INVALID, "scene is coupled to another DEM scene");
        if (n <= 0 || !balls) throw Status(DEMSPH_ERR_INVALID, "no balls");
        if (!(dx > 0) || !(hm > 0) || !(c > 0) || !(rho0 > 0) || !(nu >= 0))
            throw Status(DEMSPH_ERR_INVALID, "marker spacing, h, sound speed and density must be positive");
        const GridDesc& g = fCells.g;
        if (2.0 * hm > std::min(g.cs.x, std::min(g.cs.y, g.cs.z)) * (1.0 + 1e-12))
            throw Status(DEMSPH_ERR_INVALID, "marker h above the fluid's largest h");
        const DemBodies B = dem_bodies(dem);
        std::vector<double4> bp(B.n);
        DEMSPH_CUDA(cudaMemcpyAsync(bp.data(), B.pos, B.n * sizeof(double4), cudaMemcpyDeviceToHost, s));
        DEMSPH_CUDA(cudaStreamSynchronize(s));
        std::vector<int> seen(B.n, 0);
        for (int b : hBall) seen[b] = 1;
        for (long k = 0; k < n; k++) {
            const int b = balls[k];
            if (b < 0 || b >= B.n) throw Status(DEMSPH_ERR_INVALID, "ball index out of range");
            if (seen[b]) throw Status(DEMSPH_ERR_INVALID, "ball coupled twice");
            seen[b] = 1;
        }
        const double mass = rho0 * dx * dx * dx;
        for (long k = 0; k < n; k++) {
            const int b = balls[k];
            std::vector<double3> off;
            marker_offsets(bp[b].w, dx, hm, off);
            for (const double3& o : off) {
                hMb.push_back(b);
                hMoff.push_back(make_double4(o.x, o.y, o.z, hm));
                hMrec.push_back(make_double4(c, nu, rho0, mass));
            }
            hBall.push_back(b);
            hBStart.push_back((int)hMb.size());
            maxMarkersPerBody = std::max(maxMarkersPerBody, (int)off.size());
        }
        if (hMb.size() > (size_t)INT_MAX / 2) throw Status(DEMSPH_ERR_INVALID, "too many markers");
        coupledDem = dem;
        nBody = (int)hBall.size();
        nM = (int)hMb.size();
        if (uniformH && (float)hm != hUni) uniformH = false;
        mb.upload(hMb, s); moff.upload(hMoff, s); mrec.upload(hMrec, s);
        bBall.upload(hBall, s); bStart.upload(hBStart, s);
        mtmp.alloc(nM, s, false); mpos.alloc(nM, s, false); mvel.alloc(nM, s, false); mst.alloc(nM, s, false);
        mnorm.alloc(nM, s, false); mposf.alloc(nM, s, false); mvelf.alloc(nM, s, false); mstf.alloc(nM, s, false);
        mnormf.alloc(nM, s, false); mposq.alloc(nM, s, false); mid.alloc(nM, s, false);
        mforce.alloc(nM, s, true);
        mCells.setup(g, nM, s);
        alloc_lists();  // resets the graphs
        bodies = B;
        coupling = true;
        place_markers();
        coupling = false;
        haveLists = false;
        DEMSPH_CUDA(cudaStreamSynchronize(s));
    }

    // n coupled steps: per step the markers follow the balls, the fluid takes
    // one step (WCSPHSolver::solve's loop body) with the markers as moving
    // boundary particles, the balls receive the mean of the reactions of the
    // step's two acceleration passes, and the DEM takes demSub steps of
    // dt / demSub with that force held.  A DEM list overflow replays the
    // whole call after regrowth.
    void coupled_run(demsph_dem_t dem, long n, int demSub) {
        if (!ready) throw Status(DEMSPH_ERR_NOT_READY, "scene not initialised");
        if (!coupledDem || dem != coupledDem) throw Status(DEMSPH_ERR_INVALID, "scene is not coupled to this DEM scene");
        if (demSub < 1) throw Status(DEMSPH_ERR_INVALID, "DEM substeps must be at least 1");
        if (n <= 0) return;
        const DemBodies B = dem_bodies(dem);
        if (std::fabs(B.dt * demSub - dt) > 1e-9 * dt)
            throw Status(DEMSPH_ERR_INVALID, "DEM time step times substeps differs from the fluid time step");
        // one coupled step, issued on s (the scene stream, or a capture stream)
        auto one = [&] {
            iStep++;
            time += dt;
            step_body();
            if (maxMarkersPerBody <= 8)
                k_sph_body_force_thread<<<grid_for(nBody, 256), 256, 0, s>>>(nBody, bStart.p, bBall.p, mforce.p, moff.p,
                                                                             B.force, B.torque);
            else if (maxMarkersPerBody > 256)
                k_sph_body_force_block<<<nBody, kBodyBlock, 0, s>>>(bStart.p, bBall.p, mforce.p, moff.p, B.force,
                                                                    B.torque);
            else
                k_sph_body_force<<<grid_for(nBody, kBodyBlock / 32), kBodyBlock, 0, s>>>(nBody, bStart.p, bBall.p,
                                                                                       mforce.p, moff.p, B.force,
                                                                                       B.torque);
            g_launches += 1;
            DEMSPH_LAUNCH_CHECK();
            dem_block_steps(dem, demSub, s);
        };
        for (int attempt = 0; attempt < 8; attempt++) {
            Snap sn;
            take(sn);
            clear_status();
            // the markers' drift is measured from the rebuild that placed them:
            // steps of the fluid alone may have rebuilt without them
            skin_force();
            dem_block_begin(dem, s);
            bodies = B;
            coupling = true;
            long k = 0;
            try {
                if (useGraphs && dem_graphable(dem)) {
                    // blocks of kCoupledSteps coupled steps start where a DEM
                    // re-sort just happened, so that each block holds the same
                    // launches (an even number of fluid steps and of DEM
                    // re-sorts: every ping-pong index is back to its parity)
                    for (long di; k < n; k++) {
                        double dtm;
                        dem_clock(dem, &di, &dtm);
                        if (di % 5 == 0) break;
                        one();
                    }
                    if (cgSphEpoch != graph.epoch || cgDemEpoch != dem_graph_epoch(dem) || cgSub != demSub) {
                        cgraph.reset();
                        cgSphEpoch = graph.epoch;
                        cgDemEpoch = dem_graph_epoch(dem);
                        cgSub = demSub;
                    }
                    for (; k + kCoupledSteps <= n; k += kCoupledSteps) {
                        StepGraph& gr = cgraph.at(index_key() | dem_graph_key(dem) << 6);
                        if (!gr.ready()) {
                            const long i0 = iStep;
                            const double t0 = time;
                            long di;
                            double dtm;
                            dem_clock(dem, &di, &dtm);
                            gr.capture(kCoupledSteps, s, [&] {
                                for (int j = 0; j < kCoupledSteps; j++) one();
                            });
                            iStep = i0;
                            time = t0;
                            dem_set_clock(dem, di, dtm);
                        }
                        gr.launch(s);
                        iStep += kCoupledSteps;
                        time += kCoupledSteps * dt;
                        dem_advance_clock(dem, (long)kCoupledSteps * demSub);
                    }
                }
                for (; k < n; k++) one();
            } catch (...) {
                coupling = false;
                dem_block_end(dem);
                throw;
            }
            coupling = false;
            const bool ok = dem_block_end(dem);
            DevStatus st2 = read_status();
            if (st2.overflow) grow(st2);
            if (ok) return;
            restore(sn);
        }
        throw Status(DEMSPH_ERR_OVERFLOW, "DEM lists kept overflowing during coupled steps");
    }

    // Host particle sets -> device scene (WCSPHSolver::initialize, WCSPHSolver.h:578-612).
    // One pass over a particle set in host threads: any non-finite position
    // or non-positive h, the largest h, whether every h has the FP32 value h0,
    // and whether every particle has the first one's constants (h, m, c, nu
    // and, for dummies, rho0).
    struct SetScan {
        bool bad = false, sameH = true, sameConst = true;
        double hmax = 0;
    };
    static SetScan scan_set(const HostSet& t, float h0, bool dummies) {
        SetScan r;
        const long n = (long)t.size();
        if (n == 0) return r;
        const double4 p0 = t.pos[0], v0 = t.vel[0], s0 = t.st[0];
        const double r0 = t.rho0[0];
        std::mutex mu;
        host_parallel(n, [&](long a, long b) {
            SetScan c;
            for (long k = a; k < b; k++) {
                const double4 p = t.pos[k];
                if (!std::isfinite(p.x) || !std::isfinite(p.y) || !std::isfinite(p.z) || !(p.w > 0)) c.bad = true;
                c.hmax = std::max(c.hmax, p.w);
                c.sameH = c.sameH && (float)p.w == h0;
                c.sameConst = c.sameConst && p.w == p0.w && t.vel[k].w == v0.w && t.st[k].z == s0.z &&
                              t.st[k].w == s0.w && (!dummies || t.rho0[k] == r0);
            }
            std::lock_guard<std::mutex> lk(mu);
            r.bad = r.bad || c.bad;
            r.hmax = std::max(r.hmax, c.hmax);
            r.sameH = r.sameH && c.sameH;
            r.sameConst = r.sameConst && c.sameConst;
        });
        return r;
    }
    void initialize(double3 mn, double3 mx, double3 g, double timeStep, int prec) {
        if (hf.size() == 0) throw Status(DEMSPH_ERR_SCENE, "the number of fluid particles is equal to 0");
        // the same h everywhere, as the list build sees it (FP32)
        const float h0 = (float)hf.pos[0].w;
        const SetScan sf = scan_set(hf, h0, false), sd = scan_set(hd, h0, true);
        if (sf.bad) throw Status(DEMSPH_ERR_SCENE, "fluid particle with non-finite position or non-positive h");
        const double hmax = std::max(sf.hmax, sd.hmax);
        const bool uniH = sf.sameH && sd.sameH;
        nF = (int)hf.size();
        nD = (int)hd.size();
        init_grid(mn, mx, g, timeStep, prec, hmax, uniH);
        hUni = h0;
        // uniform constants (uniform_of): the fluid's and the dummies' own
        // constants the same throughout, and the dummies' h the fluid's
        Uniform u;
        u.h = hf.pos[0].w; u.mF = hf.vel[0].w; u.cF = hf.st[0].z; u.nuF = hf.st[0].w;
        bool on = sf.sameConst;
        if (hd.size()) {
            u.mD = hd.vel[0].w; u.cD = hd.st[0].z; u.nuD = hd.st[0].w; u.rho0D = hd.rho0[0];
            on = on && sd.sameConst && hd.pos[0].w == u.h;
        }
        u.on = on;
        this->uni = u;
        const int n = N(), nd = ND();
        // the records through the pinned staging: fluid pos, vel, st, rho0,
        // drho; dummies in caller order (pos, vel), (c, nu, rho0, 0), rho
        DBuf<double4> tp, tv, ts;
        DBuf<double> trh;
        if (nd > 0) {
            tp.alloc(nd, s, false); tv.alloc(nd, s, false); ts.alloc(nd, s, false); trh.alloc(nd, s, false);
        }
        const size_t f4 = (size_t)n * sizeof(double4), f1 = (size_t)n * sizeof(double);
        const size_t d4 = (size_t)nd * sizeof(double4), d1 = (size_t)nd * sizeof(double);
        const size_t total = 3 * f4 + 2 * f1 + 3 * d4 + d1;
        std::vector<double4> dst4;
        std::vector<double> rh;
        {
            PinnedStage& ps = PinnedStage::get();
            std::lock_guard<std::mutex> lk(ps.m);
            char* st0 = ps.reserve(total);
            auto up = [&](void* dev, const void* host, size_t bytes, size_t& off) {
                if (bytes == 0) return;
                if (st0) {
                    host_copy(st0 + off, host, bytes);
                    DEMSPH_CUDA(cudaMemcpyAsync(dev, st0 + off, bytes, cudaMemcpyHostToDevice, s));
                    off += bytes;
                } else {
                    DEMSPH_CUDA(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, s));
                }
            };
            size_t off = 0;
            up(pos[0].p, hf.pos.data(), f4, off); up(vel[0].p, hf.vel.data(), f4, off); up(st[0].p, hf.st.data(), f4, off);
            up(rho0[0].p, hf.rho0.data(), f1, off); up(drho[0].p, hf.drho.data(), f1, off);
            if (nd > 0) {
                up(tp.p, hd.pos.data(), d4, off); up(tv.p, hd.vel.data(), d4, off);
                // the dummies' (c, nu, rho0, 0) and rho, written straight into the staging
                double4* sst = st0 ? (double4*)(st0 + off) : nullptr;
                double* srh = st0 ? (double*)(st0 + off + d4) : nullptr;
                if (!st0) { dst4.resize(nd); rh.resize(nd); sst = dst4.data(); srh = rh.data(); }
                host_parallel(nd, [&](long a, long b) {
                    for (long i = a; i < b; i++) {
                        sst[i] = make_double4(hd.st[i].z, hd.st[i].w, hd.rho0[i], 0);
                        srh[i] = hd.st[i].x;
                    }
                });
                DEMSPH_CUDA(cudaMemcpyAsync(ts.p, sst, d4, cudaMemcpyHostToDevice, s));
                DEMSPH_CUDA(cudaMemcpyAsync(trh.p, srh, d1, cudaMemcpyHostToDevice, s));
            }
            DEMSPH_CUDA(cudaStreamSynchronize(s));  // the staging is free again
        }
        init_finish(tp, tv, ts, trh);
    }

    // Grid, buffers and the precision constants of a scene of nF fluid and
    // nD dummy particles (no particle data yet).
    void init_grid(double3 mn, double3 mx, double3 g, double timeStep, int prec, double hmax, bool uni) {
        if (nF == 0) throw Status(DEMSPH_ERR_SCENE, "the number of fluid particles is equal to 0");
        if (!(timeStep > 0)) throw Status(DEMSPH_ERR_INVALID, "time step must be positive");
        if (!(hmax > 0)) throw Status(DEMSPH_ERR_SCENE, "non-positive smoothing length");
        graph.reset();
        precision = prec;
        gravity = g;
        dt = timeStep;
        uniformH = uni;
        hmaxGrid = hmax;
        const double cell = 2.0 * hmax * (1.0 + skinMax) * cellFactor;
        GridDesc gd{};
        if (!grid_set(gd, mn, mx, cell)) throw Status(DEMSPH_ERR_SCENE, "invalid domain or cell size");
        status.alloc(1, s, true);
        const int n = N(), nd = ND();
        fCells.setup(gd, n, s);
        dCells.setup(gd, std::max(nd, 1), s);
        for (int b = 0; b < 2; b++) {
            pos[b].alloc(n, s, false); vel[b].alloc(n, s, false); st[b].alloc(n, s, false);
            velf[b].alloc(n, s, false); stf[b].alloc(n, s, false); posq[b].alloc(n, s, false);
            rho0[b].alloc(n, s, false); drho[b].alloc(n, s, false); id[b].alloc(n, s, false);
        }
        P = Vv = S = R0 = D = ID = L = 0;
        k_iota<<<grid_for(n, 256), 256, 0, s>>>(n, id[0].p);
        g_launches += 1;
        acc.alloc(n, s, true);
        posf.alloc(n, s, true);
        // FP32 prefilter bound: coordinates are stored relative to the grid
        // minimum; a float within |x| <= L has error <= L * 2^-24.  Positions
        // outside the domain by up to a domain length are still covered.
        {
            double L = std::max(gd.mx.x - gd.mn.x, std::max(gd.mx.y - gd.mn.y, gd.mx.z - gd.mn.z));
            eps = (float)(2.0 * L * std::ldexp(1.0, -24));
        }
        // fixed-point quantum: the largest power of two with 8 h_max below 2^30 quanta
        {
            const int k = (int)std::floor(std::log2(std::ldexp(1.0, 30) / (8.0 * hmax)));
            q = (float)std::ldexp(1.0, -k);
            invq = std::ldexp(1.0, k);
        }
    }

    // With the fluid in pos[0].. and the dummies in caller order in tp/tv/ts/trh:
    // dummies into cell order (initializeBoundaryCondition, WCSPHSolver.h:29-110),
    // wall normals, FP32 shadows, list capacities.
    void init_finish(DBuf<double4>& tp, DBuf<double4>& tv, DBuf<double4>& ts, DBuf<double>& trh) {
        const int nd = ND();
        const GridDesc gd = fCells.g;
        if (nd > 0) {
            dCells.build(tp.p, nd, s);
            g_launches += dCells.launches;
            dpos.alloc(nd, s, false); dvel.alloc(nd, s, false); dst.alloc(nd, s, false); drhoD.alloc(nd, s, false);
            dposf.alloc(nd, s, false); did.alloc(nd, s, false);
            k_sph_dummy_gather<<<grid_for(nd, 256), 256, 0, s>>>(nd, dCells.sorted.p, tp.p, tv.p, ts.p, trh.p, gd.mn,
                                                                 dpos.p, dvel.p, dst.p, drhoD.p, dposf.p, did.p);
            g_launches += 1;
            dnorm.alloc(nd, s, true);
            for (int attempt = 0; attempt < 8; attempt++) {
                nbDD.alloc((size_t)nd * KDD, s, false);
                cntDD.alloc(nd, s, true);
                clear_status();
                k_sph_dummy_normals<<<grid_for(nd, 128), 128, 0, s>>>(nd, gd, dCells.start.p, dpos.p, dvel.p, drhoD.p,
                                                                      dnorm.p, KDD, nbDD.p, cntDD.p, status.p);
                g_launches += 1;
                DEMSPH_LAUNCH_CHECK();
                DevStatus st2 = read_status();
                if (!st2.overflow) break;
                KDD = st2.need_rev + st2.need_rev / 4 + 1;
            }
            dvelf.alloc(nd, s, false); dstf.alloc(nd, s, false); dnormf.alloc(nd, s, false);
            k_sph_shadow<<<grid_for(nd, 256), 256, 0, s>>>(nd, dvel.p, dst.p, dnorm.p, dvelf.p, dstf.p, dnormf.p);
            dposq.alloc(nd, s, false);
            k_sph_fix<<<grid_for(nd, 256), 256, 0, s>>>(nd, dpos.p, gd.mn, invq, dposq.p);
            g_launches += 2;
            DEMSPH_LAUNCH_CHECK();
        } else {
            dCells.build(nullptr, 0, s);
            g_launches += dCells.launches;
        }
        // size the neighbour lists on the initial configuration (sorting the
        // fluid into cell order, which any later step does anyway): one build
        // with no room in the rows records the longest row of each list
        KF = 0;
        KD = 0;
        alloc_lists();
        clear_status();
        neighbor_search();
        if (skinMax > 0 && skinFrac > 0) launch_lists(skin_view(nullptr), false);  // the skin rows are longer
        const DevStatus st2 = read_status();
        KF = std::max(st2.need_pairs, 1);
        KD = std::max(st2.need_aux, 1);
        // headroom for compression during the run
        KF = KF + (int)std::ceil(KF * listHeadroom);
        KD = KD + (int)std::ceil(KD * listHeadroom);
        alloc_lists();
        haveLists = false;
        iStep = 0;
        time = 0;
        ready = true;
        sync_mode();
        DEMSPH_CUDA(cudaStreamSynchronize(s));
    }
};

}  // namespace demsph

// ================================================================ C ABI ====
using namespace demsph;

struct demsph_sph_scene {
    SphScene sc;
};

static inline double3 sld3(const double* a, long i) { return mk3(a[3 * i], a[3 * i + 1], a[3 * i + 2]); }
static inline void sst3(double* a, long i, double3 v) { a[3 * i] = v.x; a[3 * i + 1] = v.y; a[3 * i + 2] = v.z; }

#define SPH_CHECK(h) \
    if (!(h)) throw Status(DEMSPH_ERR_INVALID, "null scene handle")

extern "C" {

int demsph_sph_create(demsph_sph_t* out, void* stream) {
    return guarded([&] {
        if (!out) throw Status(DEMSPH_ERR_INVALID, "null output pointer");
        default_pool_retention();
        auto* h = new demsph_sph_scene();
        h->sc.s = (cudaStream_t)stream;
        *out = h;
    });
}
int demsph_sph_destroy(demsph_sph_t h) {
    return guarded([&] {
        if (!h) return;
        cudaStream_t s = h->sc.s;
        delete h;
        DEMSPH_CUDA(cudaStreamSynchronize(s));
    });
}
// addSPH / addDummy (WCSPHSolver.h:520-560): h = 1.3 spacing, m = spacing^3 rho.
// addSPH / addDummy (WCSPHSolver.h:523-541) for n particles: records in
// the caller's order, skipping those with density or sound speed <= 0 as the
// reference does.  Filled by several host threads (each first-touching its
// own part of the new arrays): count the kept particles per chunk, then write.
static void add_particles(SphScene::HostSet& t, long n, const double* pos, const double* vel, const double* c,
                          const double* spacing, const double* dens, const double* visc) {
    if (n <= 0) return;
    const int kThreads = 8;
    const long step = (n + kThreads - 1) / kThreads;
    std::vector<long> kept(kThreads + 1, 0);
    host_parallel(kThreads, [&](long a, long b) {
        for (long ch = a; ch < b; ch++) {
            long cnt = 0;
            for (long i = ch * step; i < std::min(n, (ch + 1) * step); i++) cnt += (dens[i] > 0. && c[i] > 0.);
            kept[ch + 1] = cnt;
        }
    }, 1);
    for (int ch = 0; ch < kThreads; ch++) kept[ch + 1] += kept[ch];
    const size_t b0 = t.pos.size(), m = (size_t)kept[kThreads];
    t.pos.resize(b0 + m); t.vel.resize(b0 + m); t.st.resize(b0 + m); t.rho0.resize(b0 + m); t.drho.resize(b0 + m);
    auto fill = [&](int ch) {
        const long lo = ch * step, hi = std::min(n, (ch + 1) * step);
        size_t k = b0 + kept[ch];
        for (long i = lo; i < hi; i++) {
            const double rho = dens[i], cc = c[i], sp = spacing[i];
            if (rho <= 0. || cc <= 0.) continue;  // WCSPHSolver.h:525-526
            const double mass = sp * sp * sp * rho;
            t.pos[k] = make_double4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], 1.3 * sp);
            t.vel[k] = vel ? make_double4(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2], mass)
                           : make_double4(0, 0, 0, mass);
            t.st[k] = make_double4(rho, 0.0, cc, visc[i]);
            t.rho0[k] = rho;
            t.drho[k] = 0.0;
            k++;
        }
    };
    if (n < 65536) {
        for (int ch = 0; ch < kThreads; ch++) fill(ch);
    } else {
        HostPool::get().run(kThreads, fill);
    }
}
int demsph_sph_add(demsph_sph_t h, int dummy, long n, const double* pos, const double* vel, const double* c,
                   const double* spacing, const double* dens, const double* visc) {
    return guarded([&] {
        SPH_CHECK(h);
        SphScene& s = h->sc;
        if (s.ready) throw Status(DEMSPH_ERR_INVALID, "particles must be added before initialisation");
        add_particles(dummy ? s.hd : s.hf, n, pos, vel, c, spacing, dens, visc);
        s.nF = (int)s.hf.size();
        s.nD = (int)s.hd.size();
    });
}

// ------------------------------------------------------ batch members ----
// A scene uploaded once to the device in the library's record layout, from
// which batch scenes are assembled on the device.
struct demsph_sph_member {
    cudaStream_t s = 0;
    SphScene::HostSet hf, hd;  // staging until sealed
    bool sealed = false;
    int nf = 0, nd = 0;
    double hmax = 0;
    float h0 = 0;
    bool uni = true;
    SphScene::Uniform un;  // uniform constants, recorded at sealing
    DBuf<double4> fpos, fvel, fst, dpos, dvel, dst;
    DBuf<double> frho0, drh;
};
int demsph_sph_member_create(demsph_sph_member_t* out, void* stream) {
    return guarded([&] {
        if (!out) throw Status(DEMSPH_ERR_INVALID, "null output pointer");
        auto* m = new demsph_sph_member();
        m->s = (cudaStream_t)stream;
        *out = m;
    });
}
int demsph_sph_member_destroy(demsph_sph_member_t m) {
    return guarded([&] {
        if (!m) return;
        cudaStream_t s = m->s;
        delete m;
        DEMSPH_CUDA(cudaStreamSynchronize(s));
    });
}
int demsph_sph_member_add(demsph_sph_member_t m, int dummy, long n, const double* pos, const double* vel,
                          const double* c, const double* spacing, const double* dens, const double* visc) {
    return guarded([&] {
        if (!m) throw Status(DEMSPH_ERR_INVALID, "null member handle");
        if (m->sealed) throw Status(DEMSPH_ERR_INVALID, "member already sealed");
        add_particles(dummy ? m->hd : m->hf, n, pos, vel, c, spacing, dens, visc);
    });
}
int demsph_sph_member_seal(demsph_sph_member_t m) {
    return guarded([&] {
        if (!m) throw Status(DEMSPH_ERR_INVALID, "null member handle");
        if (m->sealed) return;
        if (m->hf.size() == 0) throw Status(DEMSPH_ERR_SCENE, "the number of fluid particles is equal to 0");
        for (auto& p : m->hf.pos)
            if (!std::isfinite(p.x) || !std::isfinite(p.y) || !std::isfinite(p.z) || !(p.w > 0))
                throw Status(DEMSPH_ERR_SCENE, "fluid particle with non-finite position or non-positive h");
        m->h0 = (float)m->hf.pos[0].w;
        for (auto* set : {&m->hf, &m->hd})
            for (auto& p : set->pos) {
                m->hmax = std::max(m->hmax, p.w);
                m->uni = m->uni && (float)p.w == m->h0;
            }
        m->nf = (int)m->hf.size();
        m->nd = (int)m->hd.size();
        m->un = SphScene::uniform_of(m->hf, m->hd);
        m->fpos.upload(m->hf.pos, m->s); m->fvel.upload(m->hf.vel, m->s); m->fst.upload(m->hf.st, m->s);
        m->frho0.upload(m->hf.rho0, m->s);
        if (m->nd > 0) {
            std::vector<double4> dst4(m->nd);
            std::vector<double> rh(m->nd);
            for (int i = 0; i < m->nd; i++) {
                dst4[i] = make_double4(m->hd.st[i].z, m->hd.st[i].w, m->hd.rho0[i], 0);
                rh[i] = m->hd.st[i].x;
            }
            m->dpos.upload(m->hd.pos, m->s); m->dvel.upload(m->hd.vel, m->s);
            m->dst.upload(dst4, m->s); m->drh.upload(rh, m->s);
        }
        DEMSPH_CUDA(cudaStreamSynchronize(m->s));
        m->hf = SphScene::HostSet{};
        m->hd = SphScene::HostSet{};
        m->sealed = true;
    });
}
int demsph_sph_member_count(demsph_sph_member_t m, int dummy, long* n) {
    return guarded([&] {
        if (!m || !n) throw Status(DEMSPH_ERR_INVALID, "null argument");
        *n = m->sealed ? (dummy ? m->nd : m->nf) : (long)(dummy ? m->hd.size() : m->hf.size());
    });
}
int demsph_sph_assemble(demsph_sph_t h, int count, const demsph_sph_member_t* members, const double* offsets,
                        const double* mn, const double* mx, const double* g, double dt, int prec) {
    return guarded([&] {
        SPH_CHECK(h);
        SphScene& s = h->sc;
        if (s.ready || s.hf.size() || s.hd.size()) throw Status(DEMSPH_ERR_INVALID, "assemble needs an empty scene");
        if (prec != DEMSPH_PRECISION_FP64 && prec != DEMSPH_PRECISION_MIXED)
            throw Status(DEMSPH_ERR_INVALID, "unknown precision mode");
        if (count < 1 || !members || !offsets) throw Status(DEMSPH_ERR_INVALID, "no members");
        long nf = 0, nd = 0;
        double hmax = 0;
        bool uni = true;
        for (int k = 0; k < count; k++) {
            const demsph_sph_member* m = members[k];
            if (!m || !m->sealed) throw Status(DEMSPH_ERR_NOT_READY, "member not sealed");
            nf += m->nf;
            nd += m->nd;
            hmax = std::max(hmax, m->hmax);
            uni = uni && m->uni && m->h0 == members[0]->h0;
        }
        if (nf + nd > INT_MAX / 2) throw Status(DEMSPH_ERR_INVALID, "batch too large");
        s.nF = (int)nf;
        s.nD = (int)nd;
        s.init_grid(sld3(mn, 0), sld3(mx, 0), sld3(g, 0), dt, prec, hmax, uni);
        s.hUni = (float)members[0]->h0;
        // uniform constants: the members' fluid constants agree, and so do the
        // dummy constants of the members that have dummies
        SphScene::Uniform un = members[0]->un;
        bool haveD = members[0]->nd > 0;
        for (int k = 1; k < count && un.on; k++) {
            const SphScene::Uniform& v = members[k]->un;
            un.on = v.on && v.h == un.h && v.mF == un.mF && v.cF == un.cF && v.nuF == un.nuF;
            if (members[k]->nd > 0) {
                if (!haveD) {
                    un.mD = v.mD; un.cD = v.cD; un.nuD = v.nuD; un.rho0D = v.rho0D;
                    haveD = true;
                } else {
                    un.on = un.on && v.mD == un.mD && v.cD == un.cD && v.nuD == un.nuD && v.rho0D == un.rho0D;
                }
            }
        }
        s.uni = un;
        DBuf<double4> tp, tv, ts;
        DBuf<double> trh;
        if (nd > 0) {
            tp.alloc(nd, s.s, false); tv.alloc(nd, s.s, false); ts.alloc(nd, s.s, false); trh.alloc(nd, s.s, false);
        }
        int f0 = 0, d0 = 0;
        for (int k = 0; k < count; k++) {
            const demsph_sph_member* m = members[k];
            const double3 off = sld3(offsets, k);
            k_sph_place<<<grid_for(m->nf, 256), 256, 0, s.s>>>(m->nf, f0, off, m->fpos.p, m->fvel.p, m->fst.p,
                                                               m->frho0.p, s.pos[0].p, s.vel[0].p, s.st[0].p,
                                                               s.rho0[0].p, s.drho[0].p);
            if (m->nd > 0)
                k_sph_place<<<grid_for(m->nd, 256), 256, 0, s.s>>>(m->nd, d0, off, m->dpos.p, m->dvel.p, m->dst.p,
                                                                   m->drh.p, tp.p, tv.p, ts.p, trh.p, nullptr);
            g_launches += m->nd > 0 ? 2 : 1;
            f0 += m->nf;
            d0 += m->nd;
        }
        DEMSPH_LAUNCH_CHECK();
        s.init_finish(tp, tv, ts, trh);
    });
}
int demsph_sph_initialize(demsph_sph_t h, const double* mn, const double* mx, const double* g, double dt, int prec) {
    return guarded([&] {
        SPH_CHECK(h);
        if (prec != DEMSPH_PRECISION_FP64 && prec != DEMSPH_PRECISION_MIXED)
            throw Status(DEMSPH_ERR_INVALID, "unknown precision mode");
        h->sc.initialize(sld3(mn, 0), sld3(mx, 0), sld3(g, 0), dt, prec);
    });
}
int demsph_sph_step(demsph_sph_t h, long n) {
    return guarded([&] {
        SPH_CHECK(h);
        h->sc.run(n);
    });
}
int demsph_sph_synchronize(demsph_sph_t h) {
    return guarded([&] {
        SPH_CHECK(h);
        DEMSPH_CUDA(cudaStreamSynchronize(h->sc.s));
        h->sc.consume_status(true);
    });
}
int demsph_sph_neighbor_search(demsph_sph_t h) {
    return guarded([&] {
        SPH_CHECK(h);
        SphScene& s = h->sc;
        if (!s.ready) throw Status(DEMSPH_ERR_NOT_READY, "scene not initialised");
        s.sync_mode();
        s.clear_status();
        s.neighbor_search();
        DevStatus st2 = s.read_status();
        if (st2.overflow) {  // rebuild with room so that the lists are complete
            s.grow(st2);
            SphDev d = s.dev();
            s.launch_lists(d);
            g_launches += 1;
            DEMSPH_LAUNCH_CHECK();
        }
    });
}
int demsph_sph_eval_accel(demsph_sph_t h) {
    return guarded([&] {
        SPH_CHECK(h);
        SphScene& s = h->sc;
        if (!s.ready || !s.haveLists) throw Status(DEMSPH_ERR_NOT_READY, "no neighbour lists");
        s.sync_mode();
        // acceleration only: kick / drift go to the scratch buffers, the state is unchanged
        SphDev d = s.dev();
        d.posOut = s.pos[s.P ^ 1].p;
        d.velOut = s.vel[s.Vv ^ 1].p;
        d.velfOut = s.velf[s.Vv ^ 1].p;
        d.posqOut = s.posq[s.P ^ 1].p;
        s.launch_accel(d, 0.0, 0.0, 0, false);
        DEMSPH_CUDA(cudaStreamSynchronize(s.s));
    });
}
int demsph_sph_profile_steps(demsph_sph_t h, long n, double* phaseMs) {
    return guarded([&] {
        SPH_CHECK(h);
        SphScene& s = h->sc;
        if (!s.ready) throw Status(DEMSPH_ERR_NOT_READY, "scene not initialised");
        for (int k = 0; k < 5; k++) phaseMs[k] = 0.0;
        s.sync_mode();
        s.clear_status();
        for (long k = 0; k < n; k++) s.step_profiled(phaseMs);
        DevStatus st2 = s.read_status();
        if (st2.overflow) throw Status(DEMSPH_ERR_OVERFLOW, "neighbour lists overflowed during profiling");
        for (int k = 0; k < 5; k++) phaseMs[k] /= (double)(n > 0 ? n : 1);
    });
}
int demsph_sph_tune(demsph_sph_t h, int trials, int* chosen, double* msPerShape) {
    return guarded([&] {
        SPH_CHECK(h);
        SphScene& s = h->sc;
        if (!s.ready) throw Status(DEMSPH_ERR_NOT_READY, "scene not initialised");
        if (trials < 1) throw Status(DEMSPH_ERR_INVALID, "trials must be positive");
        // one full neighbour search sorts the fluid and sizes the lists for
        // the current state; then each block shape rebuilds the same lists
        s.clear_status();
        s.neighbor_search();
        DevStatus st0 = s.read_status();
        if (st0.overflow) {
            s.grow(st0);
            s.clear_status();
            s.neighbor_search();
        }
        cudaEvent_t e0, e1;
        DEMSPH_CUDA(cudaEventCreate(&e0));
        DEMSPH_CUDA(cudaEventCreate(&e1));
        const int keep = s.listShape;
        int best = keep;
        double bestMs = 1e300;
        for (int v = 0; v < kNumListShapes; v++) {
            s.listShape = v;
            SphDev d = s.dev();
            s.launch_lists(d);  // warm-up
            DEMSPH_CUDA(cudaEventRecord(e0, s.s));
            for (int t = 0; t < trials; t++) s.launch_lists(d);
            DEMSPH_CUDA(cudaEventRecord(e1, s.s));
            DEMSPH_CUDA(cudaEventSynchronize(e1));
            float ms = 0;
            DEMSPH_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            const double per = ms / trials;
            if (msPerShape) msPerShape[v] = per;
            if (per < bestMs) {
                bestMs = per;
                best = v;
            }
        }
        g_launches += (long long)kNumListShapes * (trials + 1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        s.listShape = best;
        s.graph.reset();
        // leave lists built by the chosen shape
        s.launch_lists(s.dev());
        g_launches += 1;
        DEMSPH_LAUNCH_CHECK();
        DEMSPH_CUDA(cudaStreamSynchronize(s.s));
        if (chosen) *chosen = best;
        (void)keep;
    });
}
int demsph_sph_tune_skin(demsph_sph_t h, int steps, double* chosen, double* msPerStep) {
    return guarded([&] {
        SPH_CHECK(h);
        SphScene& s = h->sc;
        if (!s.ready) throw Status(DEMSPH_ERR_NOT_READY, "scene not initialised");
        if (steps < 2) throw Status(DEMSPH_ERR_INVALID, "steps must be at least 2");
        // no skin, half the grid's skin, the grid's skin: each timed over the
        // same steps from the same saved state
        const double cand[3] = {0.0, 0.5 * s.skinMax, (double)s.skinMax};
        const int nc = s.skinMax > 0 ? 3 : 1;
        SphScene::Snap sn;
        s.take(sn);
        cudaEvent_t e0, e1;
        DEMSPH_CUDA(cudaEventCreate(&e0));
        DEMSPH_CUDA(cudaEventCreate(&e1));
        double bestMs = 1e300, best = s.skinFrac;
        for (int k = 0; k < nc; k++) {
            s.skinFrac = (float)cand[k];
            s.graph.reset();
            s.skin_force();
            s.run(2);  // captures the step graphs, rebuilds the lists
            DEMSPH_CUDA(cudaEventRecord(e0, s.s));
            s.run(steps);
            DEMSPH_CUDA(cudaEventRecord(e1, s.s));
            DEMSPH_CUDA(cudaEventSynchronize(e1));
            float ms = 0;
            DEMSPH_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            const double per = ms / steps;
            if (msPerStep) msPerStep[k] = per;
            if (per < bestMs) {
                bestMs = per;
                best = cand[k];
            }
            s.restore(sn);
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        s.skinFrac = (float)best;
        s.graph.reset();
        s.skin_force();
        DEMSPH_CUDA(cudaStreamSynchronize(s.s));
        if (chosen) *chosen = best;
    });
}
int demsph_sph_num_list_shapes(void) { return kNumListShapes; }
int demsph_sph_set_graphs(demsph_sph_t h, int enable) {
    return guarded([&] {
        SPH_CHECK(h);
        h->sc.useGraphs = enable != 0;
        h->sc.graph.reset();
    });
}
int demsph_sph_set_skin(demsph_sph_t h, double fraction) {
    return guarded([&] {
        SPH_CHECK(h);
        SphScene& s = h->sc;
        if (!(fraction >= 0) || fraction > 1.0) throw Status(DEMSPH_ERR_INVALID, "skin fraction must be in [0, 1]");
        if (s.ready && (float)fraction > s.skinMax)  // the grid's value is stored as FP32
            throw Status(DEMSPH_ERR_INVALID, "skin above the one the grid was built for");
        if (!s.ready) s.skinMax = (float)fraction;
        s.skinFrac = (float)fraction;
        s.graph.reset();  // the captured launches carry the skin
        s.skin_force();
    });
}
int demsph_sph_set_uniform_kernels(demsph_sph_t h, int enable) {
    return guarded([&] {
        SPH_CHECK(h);
        h->sc.uniKernels = enable != 0;
        h->sc.graph.reset();  // captured launches name the kernels
        if (h->sc.ready) h->sc.sync_mode();
    });
}
int demsph_sph_uniform_kernels(demsph_sph_t h, int* active) {
    return guarded([&] {
        SPH_CHECK(h);
        if (!active) throw Status(DEMSPH_ERR_INVALID, "null output pointer");
        h->sc.sync_mode();
        *active = h->sc.ready && h->sc.uni_path() ? 1 : 0;
    });
}
struct demsph_sph_snapshot {
    demsph_sph_t scene = nullptr;
    SphScene::Snap snap;
};
int demsph_sph_snapshot(demsph_sph_t h, demsph_sph_snapshot_t* out) {
    return guarded([&] {
        SPH_CHECK(h);
        if (!out) throw Status(DEMSPH_ERR_INVALID, "null output pointer");
        SphScene& s = h->sc;
        if (!s.ready) throw Status(DEMSPH_ERR_NOT_READY, "scene not initialised");
        auto* sn = new struct demsph_sph_snapshot();
        sn->scene = h;
        try {
            s.take(sn->snap, true);
            DEMSPH_CUDA(cudaStreamSynchronize(s.s));
        } catch (...) {
            delete sn;
            throw;
        }
        *out = sn;
    });
}
int demsph_sph_restore(demsph_sph_t h, demsph_sph_snapshot_t sn) {
    return guarded([&] {
        SPH_CHECK(h);
        if (!sn) throw Status(DEMSPH_ERR_INVALID, "null snapshot");
        if (sn->scene != h) throw Status(DEMSPH_ERR_INVALID, "the snapshot belongs to another scene");
        SphScene& s = h->sc;
        s.sync_mode();
        s.restore(sn->snap);
        DEMSPH_CUDA(cudaStreamSynchronize(s.s));
    });
}
int demsph_sph_snapshot_destroy(demsph_sph_snapshot_t sn) {
    return guarded([&] {
        if (!sn) return;
        cudaStream_t st = sn->scene ? sn->scene->sc.s : 0;
        delete sn;
        DEMSPH_CUDA(cudaStreamSynchronize(st));
    });
}
int demsph_sph_diagnostics(demsph_sph_t h, double* out) {
    return guarded([&] {
        SPH_CHECK(h);
        if (!out) throw Status(DEMSPH_ERR_INVALID, "null output pointer");
        SphScene& s = h->sc;
        if (!s.ready) throw Status(DEMSPH_ERR_NOT_READY, "scene not initialised");
        SphDiagTerm t{s.pos[s.P].p, s.vel[s.Vv].p, s.st[s.S].p, s.drho[s.D].p, s.gravity};
        diag_reduce<8>(t, s.N(), out, s.diagScratch, s.s);
    });
}
int demsph_sph_skin_stats(demsph_sph_t h, double* fraction, long* rebuilds) {
    return guarded([&] {
        SPH_CHECK(h);
        SphScene& s = h->sc;
        if (fraction) *fraction = s.skin_on() ? s.skinFrac : 0.0;
        if (rebuilds) {
            *rebuilds = 0;
            if (s.skinState.p) {
                SkinState st{};
                DEMSPH_CUDA(cudaMemcpyAsync(&st, s.skinState.p, sizeof st, cudaMemcpyDeviceToHost, s.s));
                DEMSPH_CUDA(cudaStreamSynchronize(s.s));
                *rebuilds = st.rebuilds;
            }
        }
    });
}
int demsph_sph_set_conditional_rebuild(demsph_sph_t h, int enable) {
    return guarded([&] {
        SPH_CHECK(h);
        h->sc.condEnabled = enable != 0;
        h->sc.graph.reset();
        h->sc.oneStepAfter.clear();
    });
}
int demsph_sph_conditional_rebuild(demsph_sph_t h, int* active, long* launchesPerRebuild) {
    return guarded([&] {
        SPH_CHECK(h);
        const SphScene& s = h->sc;
        const bool on = s.cond_wanted() && s.useGraphs;
        if (active) *active = on ? 1 : 0;
        if (launchesPerRebuild) *launchesPerRebuild = on ? (long)s.condBodyLaunches : 0;
    });
}
int demsph_sph_set_cell_factor(demsph_sph_t h, double factor) {
    return guarded([&] {
        SPH_CHECK(h);
        SphScene& s = h->sc;
        if (s.ready) throw Status(DEMSPH_ERR_INVALID, "the cell size is set before initialisation");
        if (!(factor >= 1.0 && factor <= 4.0)) throw Status(DEMSPH_ERR_INVALID, "cell factor must be in [1, 4]");
        s.cellFactor = factor;
    });
}
int demsph_sph_set_list_headroom(demsph_sph_t h, double fraction) {
    return guarded([&] {
        SPH_CHECK(h);
        SphScene& s = h->sc;
        if (s.ready) throw Status(DEMSPH_ERR_INVALID, "the list headroom is set before initialisation");
        if (!(fraction >= 0.0 && fraction <= 4.0)) throw Status(DEMSPH_ERR_INVALID, "headroom must be in [0, 4]");
        s.listHeadroom = fraction;
    });
}
int demsph_sph_list_capacity(demsph_sph_t h, int* fluidRow, int* dummyRow) {
    return guarded([&] {
        SPH_CHECK(h);
        if (fluidRow) *fluidRow = h->sc.KF;
        if (dummyRow) *dummyRow = h->sc.KD;
    });
}
int demsph_sph_set_list_shape(demsph_sph_t h, int shape) {
    return guarded([&] {
        SPH_CHECK(h);
        if (shape < 0 || shape >= kNumListShapes) throw Status(DEMSPH_ERR_INVALID, "unknown list block shape");
        h->sc.listShape = shape;
        h->sc.graph.reset();
    });
}
int demsph_sph_copy_members(demsph_sph_t dsth, demsph_sph_t srch, int count, const int* srcStart,
                            const int* dstStart, const int* num, const double* shift) {
    return guarded([&] {
        SPH_CHECK(dsth);
        SPH_CHECK(srch);
        SphScene& d = dsth->sc;
        SphScene& s = srch->sc;
        if (!d.ready || !s.ready) throw Status(DEMSPH_ERR_NOT_READY, "scenes not initialised");
        if (count < 0 || (count > 0 && (!srcStart || !dstStart || !num || !shift)))
            throw Status(DEMSPH_ERR_INVALID, "missing member tables");
        const int ns = s.N(), nd = d.N();
        std::vector<int> ord(count);
        for (int k = 0; k < count; k++) {
            ord[k] = k;
            if (num[k] < 0 || srcStart[k] < 0 || dstStart[k] < 0 || srcStart[k] + num[k] > ns ||
                dstStart[k] + num[k] > nd)
                throw Status(DEMSPH_ERR_INVALID, "member range out of bounds");
        }
        std::sort(ord.begin(), ord.end(), [&](int a, int b) { return srcStart[a] < srcStart[b]; });
        std::vector<int> ss(count), ds(count), nn(count);
        std::vector<double4> sh(count);
        for (int k = 0; k < count; k++) {
            const int o = ord[k];
            ss[k] = srcStart[o]; ds[k] = dstStart[o]; nn[k] = num[o];
            sh[k] = make_double4(shift[3 * o], shift[3 * o + 1], shift[3 * o + 2], 0);
            if (k > 0 && ss[k] < ss[k - 1] + nn[k - 1]) throw Status(DEMSPH_ERR_INVALID, "member ranges overlap");
        }
        if (count == 0) return;
        DBuf<int> dss, dds, dnn, slot;
        DBuf<double4> dsh;
        dss.upload(ss, d.s); dds.upload(ds, d.s); dnn.upload(nn, d.s); dsh.upload(sh, d.s);
        slot.alloc(nd, d.s, false);
        DEMSPH_CUDA(cudaStreamSynchronize(s.s));
        k_sph_slot_of<<<grid_for(nd, 256), 256, 0, d.s>>>(nd, d.id[d.ID].p, slot.p);
        k_sph_copy_members<<<grid_for(ns, 256), 256, 0, d.s>>>(ns, s.id[s.ID].p, s.pos[s.P].p, s.vel[s.Vv].p,
                                                              s.st[s.S].p, s.drho[s.D].p, count, dss.p, dds.p, dnn.p,
                                                              dsh.p, slot.p, d.pos[d.P].p, d.vel[d.Vv].p, d.st[d.S].p,
                                                              d.drho[d.D].p);
        g_launches += 2;
        DEMSPH_LAUNCH_CHECK();
        d.refresh_shadows();
        DEMSPH_CUDA(cudaStreamSynchronize(d.s));
        d.haveLists = false;
    });
}
int demsph_sph_num(demsph_sph_t h, int dummy, long* n) {
    return guarded([&] {
        SPH_CHECK(h);
        *n = dummy ? h->sc.ND() : h->sc.N();
    });
}
int demsph_sph_step_index(demsph_sph_t h, long* step, double* time) {
    return guarded([&] {
        SPH_CHECK(h);
        if (step) *step = h->sc.iStep;
        if (time) *time = h->sc.time;
    });
}
int demsph_sph_get(demsph_sph_t h, int dummy, double* pos, double* vel, double* accel, double* rho, double* p,
                   double* drho, double* normal) {
    return guarded([&] {
        SPH_CHECK(h);
        SphScene& s = h->sc;
        if (!s.ready) throw Status(DEMSPH_ERR_NOT_READY, "scene not initialised");
        if (dummy) {
            int nd = s.ND();
            if (nd == 0) return;
            std::vector<double4> P4, V4, S4, N4;
            std::vector<int> ID;
            std::vector<double> RH;
            s.dpos.download(P4, s.s); s.dvel.download(V4, s.s); s.dnorm.download(N4, s.s); s.did.download(ID, s.s);
            s.drhoD.download(RH, s.s);
            DEMSPH_CUDA(cudaStreamSynchronize(s.s));
            for (int t = 0; t < nd; t++) {
                int o = ID[t];
                if (pos) sst3(pos, o, xyz(P4[t]));
                if (vel) sst3(vel, o, xyz(V4[t]));
                if (accel) sst3(accel, o, mk3(0, 0, 0));
                if (rho) rho[o] = RH[t];
                if (p) p[o] = 0.0;
                if (drho) drho[o] = 0.0;
                if (normal) sst3(normal, o, xyz(N4[t]));
            }
            return;
        }
        const int n = s.N();
        // all fields share the order of the last permutation: put them back into
        // the caller's order on the device, then one copy per field
        const size_t w3 = (size_t)3 * n;
        const size_t words = (pos ? w3 : 0) + (vel ? w3 : 0) + (accel ? w3 : 0) + (rho ? n : 0) + (p ? n : 0) +
                             (drho ? n : 0);
        if (words > 0) {
            DBuf<double> out;
            out.alloc(words, s.s, false);
            double* q = out.p;
            auto take = [&](double* host, size_t len) -> double* {
                if (!host) return nullptr;
                double* d = q;
                q += len;
                return d;
            };
            double* dPos = take(pos, w3);
            double* dVel = take(vel, w3);
            double* dAcc = take(accel, w3);
            double* dRho = take(rho, n);
            double* dP = take(p, n);
            double* dDr = take(drho, n);
            k_sph_unpermute<<<grid_for(n, 256), 256, 0, s.s>>>(n, s.id[s.ID].p, s.pos[s.P].p, s.vel[s.Vv].p, s.acc.p,
                                                              s.st[s.S].p, s.drho[s.D].p, dPos, dVel, dAcc, dRho, dP,
                                                              dDr);
            g_launches += 1;
            DEMSPH_LAUNCH_CHECK();
            // one copy into the pinned staging, then host threads to the caller's arrays
            PinnedStage& ps = PinnedStage::get();
            std::lock_guard<std::mutex> lk(ps.m);
            char* st0 = ps.reserve(words * sizeof(double));
            if (st0) {
                DEMSPH_CUDA(cudaMemcpyAsync(st0, out.p, words * sizeof(double), cudaMemcpyDeviceToHost, s.s));
                DEMSPH_CUDA(cudaStreamSynchronize(s.s));
                const double* hq = (const double*)st0;
                auto back = [&](double* host, size_t len) {
                    if (!host) return;
                    host_copy(host, hq, len * sizeof(double));
                    hq += len;
                };
                back(pos, w3); back(vel, w3); back(accel, w3); back(rho, n); back(p, n); back(drho, n);
            } else {
                auto back = [&](double* host, const double* dev, size_t len) {
                    if (host) DEMSPH_CUDA(cudaMemcpyAsync(host, dev, len * sizeof(double), cudaMemcpyDeviceToHost, s.s));
                };
                back(pos, dPos, w3); back(vel, dVel, w3); back(accel, dAcc, w3);
                back(rho, dRho, n); back(p, dP, n); back(drho, dDr, n);
                DEMSPH_CUDA(cudaStreamSynchronize(s.s));
            }
        }
        if (normal) std::fill(normal, normal + w3, 0.0);
    });
}
// outputWCSPHVTU / outputDummyVTU (WCSPHSolver.h:360-520): <dir>/SPH_NNNN.vtu
// and <dir>/dummy_NNNN.vtu in the reference's layout, particles in caller order.
int demsph_sph_write_vtu(demsph_sph_t h, const char* dir, long frame, int what) {
    return guarded([&] {
        SPH_CHECK(h);
        if (!dir) throw Status(DEMSPH_ERR_INVALID, "null directory");
        SphScene& s = h->sc;
        if (!s.ready) throw Status(DEMSPH_ERR_NOT_READY, "scene not initialised");
        const std::string d(dir);
        if (what & DEMSPH_VTU_FLUID) {
            const int n = s.N();
            std::vector<double4> P4, V4, S4;
            std::vector<int> ID;
            s.pos[s.P].download(P4, s.s); s.vel[s.Vv].download(V4, s.s); s.st[s.S].download(S4, s.s);
            s.id[s.ID].download(ID, s.s);
            DEMSPH_CUDA(cudaStreamSynchronize(s.s));
            std::vector<double3> p(n), v(n);
            std::vector<double> hh(n), rho(n), pr(n);
            for (int t = 0; t < n; t++) {
                const int o = ID[t];
                p[o] = xyz(P4[t]); v[o] = xyz(V4[t]); hh[o] = P4[t].w; rho[o] = S4[t].x; pr[o] = S4[t].y;
            }
            vtu::File f(d, "SPH", frame);
            f.head(s.time, s.iStep, n, n);
            f.points(p);
            f.vertex_cells(n);
            f.begin_data("PointData", "smoothLength");
            f.floats("smoothLength", hh);
            f.floats("density", rho);
            f.floats("pressure", pr);
            f.vectors("velocity", v);
            f.end_data("PointData");
        }
        if (what & DEMSPH_VTU_DUMMIES) {
            const int nd = s.ND();
            std::vector<double4> P4, V4, N4;
            std::vector<int> ID;
            if (nd > 0) {
                s.dpos.download(P4, s.s); s.dvel.download(V4, s.s); s.dnorm.download(N4, s.s); s.did.download(ID, s.s);
                DEMSPH_CUDA(cudaStreamSynchronize(s.s));
            }
            std::vector<double3> p(nd), v(nd), nn(nd);
            std::vector<double> hh(nd);
            for (int t = 0; t < nd; t++) {
                const int o = ID[t];
                p[o] = xyz(P4[t]); v[o] = xyz(V4[t]); nn[o] = xyz(N4[t]); hh[o] = P4[t].w;
            }
            vtu::File f(d, "dummy", frame);
            f.head(s.time, s.iStep, nd, nd);
            f.points(p);
            f.vertex_cells(nd);
            f.begin_data("PointData", "smoothLength");
            f.floats("smoothLength", hh);
            f.vectors("velocity", v);
            f.vectors("normal", nn);
            f.end_data("PointData");
        }
    });
}
int demsph_sph_set(demsph_sph_t h, const double* pos, const double* vel, const double* rho, const double* p,
                   const double* drho) {
    return guarded([&] {
        SPH_CHECK(h);
        SphScene& s = h->sc;
        int n = s.N();
        if (!s.ready) {
            for (int i = 0; i < n; i++) {
                if (pos) { double3 q = sld3(pos, i); s.hf.pos[i].x = q.x; s.hf.pos[i].y = q.y; s.hf.pos[i].z = q.z; }
                if (vel) { double3 q = sld3(vel, i); s.hf.vel[i].x = q.x; s.hf.vel[i].y = q.y; s.hf.vel[i].z = q.z; }
                if (rho) s.hf.st[i].x = rho[i];
                if (p) s.hf.st[i].y = p[i];
                if (drho) s.hf.drho[i] = drho[i];
            }
            return;
        }
        std::vector<double4> P4, V4, S4;
        std::vector<double> DR;
        std::vector<int> ID;
        s.pos[s.P].download(P4, s.s); s.vel[s.Vv].download(V4, s.s); s.st[s.S].download(S4, s.s);
        s.drho[s.D].download(DR, s.s); s.id[s.ID].download(ID, s.s);
        DEMSPH_CUDA(cudaStreamSynchronize(s.s));
        for (int t = 0; t < n; t++) {
            int o = ID[t];
            if (pos) { double3 q = sld3(pos, o); P4[t].x = q.x; P4[t].y = q.y; P4[t].z = q.z; }
            if (vel) { double3 q = sld3(vel, o); V4[t].x = q.x; V4[t].y = q.y; V4[t].z = q.z; }
            if (rho) S4[t].x = rho[o];
            if (p) S4[t].y = p[o];
            if (drho) DR[t] = drho[o];
        }
        DEMSPH_CUDA(cudaMemcpyAsync(s.pos[s.P].p, P4.data(), n * sizeof(double4), cudaMemcpyHostToDevice, s.s));
        DEMSPH_CUDA(cudaMemcpyAsync(s.vel[s.Vv].p, V4.data(), n * sizeof(double4), cudaMemcpyHostToDevice, s.s));
        DEMSPH_CUDA(cudaMemcpyAsync(s.st[s.S].p, S4.data(), n * sizeof(double4), cudaMemcpyHostToDevice, s.s));
        DEMSPH_CUDA(cudaMemcpyAsync(s.drho[s.D].p, DR.data(), n * sizeof(double), cudaMemcpyHostToDevice, s.s));
        s.refresh_shadows();
        DEMSPH_CUDA(cudaStreamSynchronize(s.s));
        s.haveLists = false;
    });
}
int demsph_sph_num_pairs(demsph_sph_t h, int which, long* n) {
    return guarded([&] {
        SPH_CHECK(h);
        SphScene& s = h->sc;
        std::vector<int> cnt;
        if (which == 2) s.cntDD.download(cnt, s.s);
        else {
            if (!s.haveLists) throw Status(DEMSPH_ERR_NOT_READY, "no neighbour lists");
            (which == 0 ? s.cntF : s.cntD).download(cnt, s.s);
        }
        DEMSPH_CUDA(cudaStreamSynchronize(s.s));
        long t = 0;
        for (int c : cnt) {
            if (c < 0) throw Status(DEMSPH_ERR_OVERFLOW, "a list row overflowed; call neighborSearch to rebuild");
            if (which == 2) t += c;
            else
                for (int sub = 0; sub < kQuad; sub++) t += lane_count(c, sub);
        }
        *n = t;
    });
}
int demsph_sph_get_pairs(demsph_sph_t h, int which, int* a, int* b) {
    return guarded([&] {
        SPH_CHECK(h);
        SphScene& s = h->sc;
        std::vector<int> cnt, nb, rowId, colId;
        int rows, K = 0;
        if (which == 2) {
            s.cntDD.download(cnt, s.s); s.nbDD.download(nb, s.s);
            s.did.download(rowId, s.s);
            colId = std::vector<int>();
            rows = s.ND(); K = s.KDD;
        } else {
            if (!s.haveLists) throw Status(DEMSPH_ERR_NOT_READY, "no neighbour lists");
            (which == 0 ? s.cntF : s.cntD).download(cnt, s.s);
            (which == 0 ? s.nbF : s.nbD).download(nb, s.s);
            s.id[s.ID].download(rowId, s.s);
            rows = s.N(); K = which == 0 ? s.KF : s.KD;
        }
        std::vector<int> didv;
        s.did.download(didv, s.s);
        // the neighbours' positions when the lists were built
        std::vector<double4> colPos;
        if (which == 0) s.pos[s.L].download(colPos, s.s);
        else s.dpos.download(colPos, s.s);
        DEMSPH_CUDA(cudaStreamSynchronize(s.s));
        const std::vector<int>& col = (which == 0) ? rowId : didv;
        // The reference's row order: its stencil visits cells in ascending key
        // on a grid of 2 h_max cells, each cell in ascending original index.
        // This library's cells are wider (they cover the skin of the skin
        // lists), so each row is put into that order here.
        GridDesc gref{};
        grid_set(gref, s.fCells.g.mn, s.fCells.g.mx, 2.0 * s.hmaxGrid);
        std::vector<long long> colKey(colPos.size());
        for (size_t j = 0; j < colPos.size(); j++)
            colKey[j] = (long long)clamped_key(xyz(colPos[j]), gref) * (1LL << 31) + col[j];
        // rows emitted in the caller's original order
        std::vector<int> rowOf(rows);
        for (int t = 0; t < rows; t++) rowOf[rowId[t]] = t;
        for (int c : cnt)
            if (c < 0) throw Status(DEMSPH_ERR_OVERFLOW, "a list row overflowed; call neighborSearch to rebuild");
        long w = 0;
        std::vector<int> slots;
        for (int o = 0; o < rows; o++) {
            int t = rowOf[o];
            slots.clear();
            if (which == 2) {
                for (int k = 0; k < cnt[t]; k++) slots.push_back(nb[(size_t)k * rows + t]);
            } else {
                for (int sub = 0; sub < kQuad; sub++)
                    for (int m = 0; m < lane_count(cnt[t], sub); m++) slots.push_back(nb[row_at(t, sub + kQuad * m, K)]);
            }
            std::sort(slots.begin(), slots.end(), [&](int x, int y) { return colKey[x] < colKey[y]; });
            for (int j : slots) {
                a[w] = o;
                b[w] = col[j];
                w++;
            }
        }
    });
}

// ------------------------------------------------ coupled DEM balls ----
int demsph_sph_couple_balls(demsph_sph_t h, demsph_dem_t dem, long n, const int* balls, double spacing,
                            double smoothingLength, double soundSpeed, double viscosity, double density) {
    return guarded([&] {
        SPH_CHECK(h);
        if (!dem) throw Status(DEMSPH_ERR_INVALID, "null DEM scene handle");
        h->sc.add_bodies(dem, n, balls, spacing, smoothingLength, soundSpeed, viscosity, density);
        h->sc.sync_mode();  // scenes with markers keep the shadows unpacked
    });
}
int demsph_sph_couple_step(demsph_sph_t h, demsph_dem_t dem, long n, int demSubsteps) {
    return guarded([&] {
        SPH_CHECK(h);
        h->sc.sync_mode();
        h->sc.coupled_run(dem, n, demSubsteps);
    });
}
int demsph_sph_num_markers(demsph_sph_t h, long* n, long* bodies) {
    return guarded([&] {
        SPH_CHECK(h);
        if (n) *n = h->sc.nM;
        if (bodies) *bodies = h->sc.nBody;
    });
}
int demsph_sph_get_markers(demsph_sph_t h, double* pos, double* vel, double* normal, double* force, int* ball) {
    return guarded([&] {
        SPH_CHECK(h);
        SphScene& s = h->sc;
        const int nm = s.nM;
        if (nm == 0) return;
        std::vector<double4> p, v, nr, f;
        std::vector<int> slot;
        s.mpos.download(p, s.s); s.mvel.download(v, s.s); s.mnorm.download(nr, s.s); s.mforce.download(f, s.s);
        s.mid.download(slot, s.s);
        DEMSPH_CUDA(cudaStreamSynchronize(s.s));
        for (int t = 0; t < nm; t++) {
            const int k = slot[t];
            if (k < 0 || k >= nm) throw Status(DEMSPH_ERR_INVALID, "marker order corrupted");
            if (pos) sst3(pos, k, xyz(p[t]));
            if (vel) sst3(vel, k, xyz(v[t]));
            if (normal) sst3(normal, k, xyz(nr[t]));
        }
        for (int k = 0; k < nm; k++) {
            if (force) sst3(force, k, xyz(f[k]));
            if (ball) ball[k] = s.hMb[k];
        }
    });
}
int demsph_sph_get_coupling(demsph_sph_t h, int* ball, double* force, double* torque) {
    return guarded([&] {
        SPH_CHECK(h);
        SphScene& s = h->sc;
        if (!s.coupledDem) return;
        const DemBodies B = dem_bodies(s.coupledDem);
        std::vector<double4> F(B.n), T(B.n);
        DEMSPH_CUDA(cudaMemcpyAsync(F.data(), B.force, B.n * sizeof(double4), cudaMemcpyDeviceToHost, s.s));
        DEMSPH_CUDA(cudaMemcpyAsync(T.data(), B.torque, B.n * sizeof(double4), cudaMemcpyDeviceToHost, s.s));
        DEMSPH_CUDA(cudaStreamSynchronize(s.s));
        for (int b = 0; b < s.nBody; b++) {
            const int i = s.hBall[b];
            if (ball) ball[b] = i;
            if (force) sst3(force, b, xyz(F[i]));
            if (torque) sst3(torque, b, xyz(T[i]));
        }
    });
}

}  // extern "C"
