// DEM path of the DEMSPH B200 library: neighbour search with contact-history
// carry, contact / bond forces, mesh-wall contact, clump and sphere
// integration, and the scene runtime behind the demsph_dem_* C ABI.
//
// Layout in HBM (one scene):
//   balls   pos (x,y,z,r) | vel (vx,vy,vz,1/m) | angv (wx,wy,wz,-) : double4 SoA
//   pairs   ELL, column-major: slot(k, A) = k*N + A for the k-th partner B>A of
//           ball A; ids int32, springs double4, per-slot force / B-side torque.
//           Double-buffered across rebuilds so history carries old -> new.
//   reverse per-ball list of the slots in which the ball is the B side.
//   walls   triangle (i0,i1,i2,wall) int4, vertices double4, per-ball ELL of
//           candidate triangles with their springs (double-buffered per call).
// Kernels walk balls in cell order (the order array of the last rebuild) so
// that neighbouring threads touch neighbouring memory.
#include <algorithm>
#include <climits>
#include <array>
#include <atomic>
#include <cmath>
#include <map>
#include <memory>
#include <unordered_map>

#include "cells.cuh"
#include "graph.cuh"
#include "vtu.hpp"
#include "dem_physics.cuh"
#include "coupling.hpp"
#include "external.cuh"
#include "diag.cuh"

namespace demsph {

extern std::atomic<long long> g_launches;

// Everything a DEM kernel needs, passed by value.
struct DemDev {
    int N, K, KR, KT;
    int nBond, nTri, nVert, nWall, nClump;
    int nMat, cap;
    int roll, tors;
    GridDesc bg, tg;
    const MatPair* mats;
    double4* pos;
    double4* vel;
    double4* angv;
    double4* force;
    double4* torque;
    double4* forceA;
    double4* torqueA;
    const int* mat;
    const int* clump;
    const int* order;      // cell-sorted candidate list (balls, or periodic ghosts)
    const int* qorder;     // the balls that query the lists, in cell order
    const int* cellStart;  // candidate grid
    // current / previous pair lists
    int* pj;
    int* pcnt;
    double4* spS;
    double4* spR;
    double4* spT;
    const int* pjOld;
    const int* pcntOld;
    const double4* spSOld;
    const double4* spROld;
    const double4* spTOld;
    double4* pF;
    double4* pTB;
    int* rcnt;
    int* rslot;
    // bonds
    const int2* bab;
    int* bok;
    double4* bpoint;
    double4* bnormal;
    double4* bFs;
    double4* bTb;
    double* bFn;
    double* bTt;
    double* bsmax;
    double* btmax;
    double4* bF;
    double4* bTA;
    double4* bTB;
    int* bpair;  // 1 when the bond's balls are a pair of the current list
    const int* bincStart;
    const int* binc;
    // mesh walls
    double4* wpos;
    double4* wvel;
    double4* wangv;
    double4* wq;
    const int* wmat;
    const double4* vlocal;
    double4* vglobal;
    const int* vwall;
    const int4* tris;
    double4* tcenter;
    const int* triOrder;
    const int* triCellStart;
    double4* wbox;  // [min, max] corners of the mesh vertices' box
    int* wtj;
    int* wcnt;
    double4* wS;
    double4* wR;
    double4* wT;
    const int* wtjOld;
    const int* wcntOld;
    const double4* wSOld;
    const double4* wROld;
    const double4* wTOld;
    // clumps
    double4* cpos;
    double4* cvel;
    double4* cangv;
    double4* cforce;
    double4* ctorque;
    double4* cq;
    const double4* cinvIa;
    const double4* cinvIb;
    const double* cinvm;
    const int2* cpeb;
    // external force hook
    const double4* fconst;
    // force and torque of a coupled fluid on each ball (or null)
    const double4* cplF;
    const double4* cplT;
    double framp;
    double damp;
    int buoy;
    double brho, bcd, blevel;
    double3 bg3, bu;
    double3 gravity;
    DevStatus* status;
};

// ------------------------------------------------------------ rebuild ------
// countBallInteractionsKernel + writeBallInteractionsKernel
// (ballNeighborSearchKernel.cu:6-151) as one pass: candidate B > A, not both
// fixed, not the same clump, |r_AB| <= 1.1 (r_A + r_B); rows in the
// reference's stencil order; springs carried from A's previous row.
__global__ void k_dem_build_pairs(DemDev d) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= d.N) return;
    const int A = d.qorder[t];
    const double4 pa = d.pos[A];
    const double3 ra = xyz(pa);
    const double imA = d.vel[A].w;
    const int clA = d.clump[A];
    const int oldCnt = d.pcntOld ? d.pcntOld[A] : 0;
    int cnt = 0;
    Stencil st = stencil_of(ra, d.bg);
    for_stencil_rows(st, d.bg, d.cellStart, [&](int b, int e) {
        for (int k = b; k < e; k++) {
            const int B = d.order[k];
            if (A >= B) continue;
            const double imB = d.vel[B].w;
            if (imA == 0 && imB == 0) continue;
            const int clB = d.clump[B];
            if (clB >= 0 && clA == clB) continue;
            const double4 pb = d.pos[B];
            double cut = 1.1 * (pa.w + pb.w);
            double3 r = ra - xyz(pb);
            if ((cut * cut - dot(r, r)) >= 0.) {
                if (cnt < d.K) {
                    size_t slot = (size_t)cnt * d.N + A;
                    d.pj[slot] = B;
                    double4 s = make_double4(0, 0, 0, 0), rr = s, tt = s;
                    for (int q = 0; q < oldCnt; q++) {
                        size_t os = (size_t)q * d.N + A;
                        if (d.pjOld[os] == B) {
                            s = d.spSOld[os];
                            if (d.roll) rr = d.spROld[os];
                            if (d.tors) tt = d.spTOld[os];
                            break;
                        }
                    }
                    d.spS[slot] = s;
                    if (d.roll) d.spR[slot] = rr;
                    if (d.tors) d.spT[slot] = tt;
                }
                cnt++;
            }
        }
    });
    if (cnt > d.K) {
        atomicMax(&d.status->need_pairs, cnt);
        atomicExch(&d.status->overflow, 1);
        cnt = d.K;
    }
    d.pcnt[A] = cnt;
}

// Reverse incidence: for each pair slot, record it in the B ball's list.
__global__ void k_dem_reverse(DemDev d) {
    int A = blockIdx.x * blockDim.x + threadIdx.x;
    if (A >= d.N) return;
    int c = d.pcnt[A];
    for (int k = 0; k < c; k++) {
        int slot = k * d.N + A;
        int B = d.pj[slot];
        int r = atomicAdd(d.rcnt + B, 1);
        if (r < d.KR) {
            d.rslot[(size_t)r * d.N + B] = slot;
        } else {
            atomicMax(&d.status->need_rev, r + 1);
            atomicExch(&d.status->overflow, 1);
        }
    }
}
// Orders each reverse list by the A ball (the reference's stable sort of the
// pairs by objectPointing, DEMSolver.h:59-78), for a deterministic sum.
__global__ void k_dem_reverse_order(DemDev d) {
    int B = blockIdx.x * blockDim.x + threadIdx.x;
    if (B >= d.N) return;
    int c = d.rcnt[B];
    if (c > d.KR) { c = d.KR; d.rcnt[B] = c; }
    for (int i = 1; i < c; i++) {
        int v = d.rslot[(size_t)i * d.N + B];
        int kv = v % d.N;
        int j = i - 1;
        while (j >= 0) {
            int u = d.rslot[(size_t)j * d.N + B];
            if (u % d.N <= kv) break;
            d.rslot[(size_t)(j + 1) * d.N + B] = u;
            j--;
        }
        d.rslot[(size_t)(j + 1) * d.N + B] = v;
    }
}

// ------------------------------------------------------- force evaluation --
// updateBallContactKernel + calBallContactForceTorqueKernel
// (contactKernel.cu:135-259) for every pair in ball A's row, fused with the
// A-side sum of sumObjectPointedForceTorqueFromInteractionKernel
// (contactKernel.cu:657-681).  The pair force and the B-side torque
// contribution -(T_c + (r_c - r_B) x F_c) are stored for the B side.
template <class R>
__device__ __forceinline__ void pair_forces_ball(const DemDev& d, int A, double dt) {
    const double4 pa = d.pos[A];
    const double3 ra = xyz(pa);
    const double4 va4 = d.vel[A];
    const double3 va = xyz(va4);
    const double3 wa = xyz(d.angv[A]);
    const int matA = d.mat[A];
    const int c = d.pcnt[A];
    double3 FA = mk3(0, 0, 0), TA = mk3(0, 0, 0);
    for (int k = 0; k < c; k++) {
        size_t slot = (size_t)k * d.N + A;
        int B = d.pj[slot];
        double4 pb = d.pos[B];
        double3 rb = xyz(pb);
        double4 vb4 = d.vel[B];
        double3 wb = xyz(d.angv[B]);
        double3 rij = ra - rb;
        double3 n = normalize(rij);
        double delta = pa.w + pb.w - len(rij);
        double3 rc = rb + (pb.w - 0.5 * delta) * n;
        double Rad = pa.w * pb.w / (pa.w + pb.w);
        double m = 1. / (va4.w + vb4.w);
        double3 vc = va + cross(wa, rc - ra) - (xyz(vb4) + cross(wb, rc - rb));
        double3 wij = wa - wb;
        const MatPair mp = d.mats[pair_param_index(matA, d.mat[B], d.nMat, d.cap)];
        double4 s4 = d.spS[slot];
        double3 es = xyz(s4), er = mk3(0, 0, 0), et = mk3(0, 0, 0);
        if (d.roll) er = xyz(d.spR[slot]);
        if (d.tors) et = xyz(d.spT[slot]);
        V<R> F, T;
        contact_law<R>(mp, F, T, es, er, et, vc, wij, n, delta, m, Rad, dt, d.roll, d.tors);
        d.spS[slot] = d4(es, 0);
        if (d.roll) d.spR[slot] = d4(er, 0);
        if (d.tors) d.spT[slot] = d4(et, 0);
        double3 Fd = up(F), Td = up(T);
        d.pF[slot] = d4(Fd, 0);
        d.pTB[slot] = d4(-Td - cross(rc - rb, Fd), 0);
        FA += Fd;
        TA += Td + cross(rc - ra, Fd);
    }
    d.forceA[A] = d4(FA, 0);
    d.torqueA[A] = d4(TA, 0);
}
template <class R>
__global__ void __launch_bounds__(128, 4) k_dem_pair_forces(DemDev d, double dt) {
    chain_enter();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < d.N) pair_forces_ball<R>(d, d.qorder[t], dt);
}

// calBondedForceTorqueKernel (contactKernel.cu:535-655).  Instead of adding
// into the pair (bond with a contact pair) or FP64 atomics (without), each
// bond stores its contributions to both balls; the per-ball pass sums them
// over a static incidence list, so the result is deterministic.
__global__ void k_dem_bonds(DemDev d, double dt) {
    chain_enter();
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= d.nBond) return;
    if (d.bok[b] == 0) {
        d.bFn[b] = 0;
        d.bTt[b] = 0;
        d.bFs[b] = make_double4(0, 0, 0, 0);
        d.bTb[b] = make_double4(0, 0, 0, 0);
        d.bF[b] = make_double4(0, 0, 0, 0);
        d.bTA[b] = make_double4(0, 0, 0, 0);
        d.bTB[b] = make_double4(0, 0, 0, 0);
        return;
    }
    int2 ab = d.bab[b];
    int i = ab.x, j = ab.y;
    double4 pi4 = d.pos[i], pj4 = d.pos[j];
    double3 ri = xyz(pi4), rj = xyz(pj4);
    double3 n0 = xyz(d.bnormal[b]);
    double3 n = normalize(ri - rj);
    double delta = pi4.w + pj4.w - len(ri - rj);
    double3 rc = rj + (pj4.w - 0.5 * delta) * n;
    // The reference takes r_c and n from the matching contact pair when one
    // exists; that pair computed them with these same expressions.
    const bool found = d.bpair[b] != 0;
    d.bpoint[b] = d4(rc, 0);
    d.bnormal[b] = d4(n, 0);
    double3 wi = xyz(d.angv[i]), wj = xyz(d.angv[j]);
    double3 vc = xyz(d.vel[i]) + cross(wi, rc - ri) - (xyz(d.vel[j]) + cross(wj, rc - rj));
    const MatPair mp = d.mats[pair_param_index(d.mat[i], d.mat[j], d.nMat, d.cap)];
    double Fn = d.bFn[b], Tt = d.bTt[b];
    double3 Fs = xyz(d.bFs[b]), Tb = xyz(d.bTb[b]);
    double smax = d.bsmax[b], tmax = d.btmax[b];
    d.bok[b] = parallel_bond(Fn, Tt, Fs, Tb, smax, tmax, n0, n, vc, wi, wj, pi4.w, pj4.w, dt, mp);
    d.bFn[b] = Fn;
    d.bTt[b] = Tt;
    d.bFs[b] = d4(Fs, 0);
    d.bTb[b] = d4(Tb, 0);
    d.bsmax[b] = smax;
    d.btmax[b] = tmax;
    double3 Fb = Fn * n + Fs;
    double3 Tn = Tt * n + Tb;
    d.bF[b] = d4(Fb, 0);
    if (!found) {
        d.bTA[b] = d4(Tn + cross(rc - ri, Fs), 0);
        d.bTB[b] = d4(-Tt * n - Tb + cross(rc - rj, -Fs), 0);
    } else {
        d.bTA[b] = d4(Tn + cross(rc - ri, Fb), 0);
        d.bTB[b] = d4(-Tn - cross(rc - rj, Fb), 0);
    }
}

// Whether each bond's balls (A, B) are a pair of the current list: the
// per-bond search of A's row in calBondedForceTorqueKernel
// (contactKernel.cu:595-611), done once per list rebuild instead of in every
// force evaluation (the list only changes at a rebuild).
__global__ void k_dem_bond_pairs(DemDev d) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= d.nBond) return;
    const int2 ab = d.bab[b];
    const int c = d.pcnt[ab.x];
    int found = 0;
    for (int k = 0; k < c; k++) {
        if (d.pj[(size_t)k * d.N + ab.x] == ab.y) { found = 1; break; }
    }
    d.bpair[b] = found;
}

// The box of all mesh vertices (a triangle's box lies inside it): a ball
// farther than its radius from it has no candidate triangle.
constexpr int kBoxThreads = 256;
__global__ void __launch_bounds__(kBoxThreads) k_dem_wall_box(DemDev d) {
    __shared__ double3 lo[kBoxThreads], hi[kBoxThreads];
    const int t = threadIdx.x;
    double3 a = mk3(1e300, 1e300, 1e300), b = mk3(-1e300, -1e300, -1e300);
    for (int v = t; v < d.nVert; v += kBoxThreads) {
        const double3 p = xyz(d.vglobal[v]);
        a = mk3(fmin(a.x, p.x), fmin(a.y, p.y), fmin(a.z, p.z));
        b = mk3(fmax(b.x, p.x), fmax(b.y, p.y), fmax(b.z, p.z));
    }
    lo[t] = a;
    hi[t] = b;
    __syncthreads();
    for (int h = kBoxThreads / 2; h > 0; h >>= 1) {
        if (t < h) {
            lo[t] = mk3(fmin(lo[t].x, lo[t + h].x), fmin(lo[t].y, lo[t + h].y), fmin(lo[t].z, lo[t + h].z));
            hi[t] = mk3(fmax(hi[t].x, hi[t + h].x), fmax(hi[t].y, hi[t + h].y), fmax(hi[t].z, hi[t + h].z));
        }
        __syncthreads();
    }
    if (t == 0) {
        d.wbox[0] = d4(lo[0], 0);
        d.wbox[1] = d4(hi[0], 0);
    }
}

// Mesh-wall contacts of one force evaluation, per ball: candidate triangles
// by AABB over the triangle grid with spring carry
// (count/writeBallTriangleInteractionsKernel, ballNeighborSearchKernel.cu:153-338),
// edge/vertex de-duplication (updateBallTriangleContact, contactKernel.cu:261-418)
// and the wall law (calBallWallContactForceTorqueKernel, contactKernel.cu:420-533),
// added into the ball's A-side accumulators before k_dem_finalize sums them.
// (A kernel of its own: the candidate arrays and the law would otherwise set
// the register budget of every ball's finish.)
constexpr int kMaxTriPerBall = 32;
template <class R>
__device__ __forceinline__ void walls_ball(const DemDev& d, int i, double dtWall) {
    const double4 p4 = d.pos[i];
    const double3 ri = xyz(p4);
    {
        // outside the mesh box by more than r (with a relative margin that
        // covers rounding): no triangle passes the candidate test below
        const double3 lo = xyz(d.wbox[0]), hi = xyz(d.wbox[1]);
        const double cx = fmin(fmax(ri.x, lo.x), hi.x), cy = fmin(fmax(ri.y, lo.y), hi.y),
                     cz = fmin(fmax(ri.z, lo.z), hi.z);
        const double dx = ri.x - cx, dy = ri.y - cy, dz = ri.z - cz;
        if (dx * dx + dy * dy + dz * dz > 1.000001 * p4.w * p4.w) {
            d.wcnt[i] = 0;
            return;
        }
    }
    double3 F = mk3(0, 0, 0), T = mk3(0, 0, 0);
    bool any = false;
    // candidate triangles in the reference's stencil order
    int tri[kMaxTriPerBall];
    int cnt = 0;
    Stencil st = stencil_of(ri, d.tg);
    const double r2 = p4.w * p4.w;
    for_stencil_rows(st, d.tg, d.triCellStart, [&](int b, int e) {
        for (int k = b; k < e; k++) {
            int tj = d.triOrder[k];
            int4 tv = d.tris[tj];
            double3 a = xyz(d.vglobal[tv.x]), bb = xyz(d.vglobal[tv.y]), c = xyz(d.vglobal[tv.z]);
            double cx = fmin(fmax(ri.x, fmin(a.x, fmin(bb.x, c.x))), fmax(a.x, fmax(bb.x, c.x)));
            double cy = fmin(fmax(ri.y, fmin(a.y, fmin(bb.y, c.y))), fmax(a.y, fmax(bb.y, c.y)));
            double cz = fmin(fmax(ri.z, fmin(a.z, fmin(bb.z, c.z))), fmax(a.z, fmax(bb.z, c.z)));
            double dx = ri.x - cx, dy = ri.y - cy, dz = ri.z - cz;
            if (dx * dx + dy * dy + dz * dz <= r2) {
                if (cnt < d.KT && cnt < kMaxTriPerBall) tri[cnt] = tj;
                cnt++;
            }
        }
    });
    if (cnt > d.KT || cnt > kMaxTriPerBall) {
        atomicMax(&d.status->need_aux, cnt);
        atomicExch(&d.status->overflow, 1);
        cnt = min(d.KT, kMaxTriPerBall);
    }
    // springs: carry from this ball's previous candidate row
    double3 sS[kMaxTriPerBall], sR[kMaxTriPerBall], sT[kMaxTriPerBall];
    double3 cp[kMaxTriPerBall];
    int type[kMaxTriPerBall];
    const int oc = d.wcntOld ? d.wcntOld[i] : 0;
    for (int c = 0; c < cnt; c++) {
        sS[c] = sR[c] = sT[c] = mk3(0, 0, 0);
        for (int q = 0; q < oc; q++) {
            size_t os = (size_t)q * d.N + i;
            if (d.wtjOld[os] == tri[c]) {
                sS[c] = xyz(d.wSOld[os]);
                if (d.roll) sR[c] = xyz(d.wROld[os]);
                if (d.tors) sT[c] = xyz(d.wTOld[os]);
                break;
            }
        }
        int4 tv = d.tris[tri[c]];
        cp[c] = mk3(0, 0, 0);
        type[c] = classify_sphere_triangle(ri, p4.w, xyz(d.vglobal[tv.x]), xyz(d.vglobal[tv.y]),
                                           xyz(d.vglobal[tv.z]), cp[c]);
    }
    // de-duplication, sequential as in the reference thread
    unsigned cancel = 0;
    for (int c = 0; c < cnt; c++) {
        if (type[c] == kCtNone) {
            sS[c] = sR[c] = sT[c] = mk3(0, 0, 0);
            cancel |= 1u << c;
            continue;
        }
        if (type[c] == kCtFace) continue;
        for (int c1 = 0; c1 < cnt; c1++) {
            if (c1 == c) continue;
            int t1 = type[c1];
            bool copy = false;
            if (t1 == kCtNone) continue;
            if (t1 == kCtFace) {
                int4 tv = d.tris[tri[c1]];
                double3 q0 = xyz(d.vglobal[tv.x]), q1 = xyz(d.vglobal[tv.y]), q2 = xyz(d.vglobal[tv.z]);
                if (len2(cross(cp[c] - q0, q1 - q0)) < 1.e-20) copy = true;
                else if (len2(cross(cp[c] - q1, q2 - q1)) < 1.e-20) copy = true;
                else if (len2(cross(cp[c] - q0, q2 - q0)) < 1.e-20) copy = true;
            } else if (t1 == kCtEdge) {
                if (type[c] == t1) { if (c1 < c && len2(cp[c] - cp[c1]) < 1.e-20) copy = true; }
                else if (len2(cp[c] - cp[c1]) < 1.e-20) copy = true;
            } else {
                if (type[c] == t1 && c1 < c && len2(cp[c] - cp[c1]) < 1.e-20) copy = true;
            }
            if (copy) {
                sS[c] = sS[c1]; sR[c] = sR[c1]; sT[c] = sT[c1];
                cancel |= 1u << c;
                break;
            }
        }
    }
    // wall law (fixed balls skip it, as calBallWallContactForceTorqueKernel returns early)
    const double4 v4 = cnt ? d.vel[i] : make_double4(0, 0, 0, 0);
    if (cnt && !(v4.w < 1.e-20)) {
        const double3 vi = xyz(v4), wi = xyz(d.angv[i]);
        const double m = 1. / v4.w;
        const int mi = d.mat[i];
        for (int c = 0; c < cnt; c++) {
            if (cancel & (1u << c)) continue;
            int wj = d.tris[tri[c]].w;
            double3 n = normalize(ri - cp[c]);
            double delta = p4.w - len(ri - cp[c]);
            double3 rj = xyz(d.wpos[wj]), vj = xyz(d.wvel[wj]), wwj = xyz(d.wangv[wj]);
            double3 vc = vi + cross(wi, cp[c] - ri) - (vj + cross(wwj, cp[c] - rj));
            double3 wij = wi - wwj;
            const MatPair mp = d.mats[pair_param_index(mi, d.wmat[wj], d.nMat, d.cap)];
            V<R> Fc, Tc;
            contact_law<R>(mp, Fc, Tc, sS[c], sR[c], sT[c], vc, wij, n, delta, m, p4.w, dtWall, d.roll, d.tors);
            double3 Fd = up(Fc);
            F += Fd;
            T += up(Tc) + cross(cp[c] - ri, Fd);
            any = true;
        }
    }
    for (int c = 0; c < cnt; c++) {
        size_t s = (size_t)c * d.N + i;
        d.wtj[s] = tri[c];
        d.wS[s] = d4(sS[c], 0);
        if (d.roll) d.wR[s] = d4(sR[c], 0);
        if (d.tors) d.wT[s] = d4(sT[c], 0);
    }
    d.wcnt[i] = cnt;
    if (any) {
        d.forceA[i] = d4(xyz(d.forceA[i]) + F, 0);
        d.torqueA[i] = d4(xyz(d.torqueA[i]) + T, 0);
    }
}
template <class R>
__global__ void __launch_bounds__(128) k_dem_walls(DemDev d, double dtWall) {
    chain_enter();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < d.N) walls_ball<R>(d, d.order[t], dtWall);
}
// Small scenes, whose steps are bound by the latency of each launch's chain
// of loads: a ball's pair forces and then its wall contacts in one thread
// (the wall terms are added to the A-side sums the pair forces just wrote, as
// the separate kernels do, so the result is the same).
template <class R>
__global__ void __launch_bounds__(128) k_dem_pair_walls(DemDev d, double dt, double dtWall) {
    chain_enter();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= d.N) return;
    const int A = d.qorder[t];
    pair_forces_ball<R>(d, A, dt);
    walls_ball<R>(d, A, dtWall);
}

// Per-ball finish of one force evaluation:
//  * the A-side sums (pairs, periodic ghosts, mesh walls), the B-side pair
//    sum (sumObjectPointingForceTorqueFromInteractionKernel,
//    contactKernel.cu:683-714) and bond contributions;
//  * the external force hook (externalForceTorque.cu);
//  * optionally the half-kick (+ drift) of ballIntegrationKernel.cu:30-56,112-121.
template <class R>
__global__ void __launch_bounds__(128, 8) k_dem_finalize(DemDev d, double extTime, int ext, int integ, double hdt) {
    chain_enter();
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= d.N) return;
    const int i = d.order[t];
    double3 F = xyz(d.forceA[i]), T = xyz(d.torqueA[i]);
    const int rc = d.rcnt[i];
    for (int r = 0; r < rc; r++) {
        int slot = d.rslot[(size_t)r * d.N + i];
        F -= xyz(d.pF[slot]);
        T += xyz(d.pTB[slot]);
    }
    if (d.nBond) {
        for (int q = d.bincStart[i]; q < d.bincStart[i + 1]; q++) {
            int e = d.binc[q];
            int b = e >> 1;
            if (e & 1) { F -= xyz(d.bF[b]); T += xyz(d.bTB[b]); }
            else { F += xyz(d.bF[b]); T += xyz(d.bTA[b]); }
        }
    }
    const double4 p4 = d.pos[i];
    const double3 ri = xyz(p4);
    const double4 v4 = d.vel[i];
    if (ext) {
        // launchAddConstantForce (externalForceTorque.cu:4-24)
        if (d.fconst) {
            double c = 1.0;
            if (d.framp > 0) { c = extTime / d.framp; if (c > 1.0) c = 1.0; }
            F += xyz(d.fconst[i]) * c;
        }
        if (d.cplF) {
            F += xyz(d.cplF[i]);
            T += xyz(d.cplT[i]);
        }
        // launchAddGlobalDampingForceTorque (externalForceTorque.cu:26-57)
        if (d.damp != 0) {
            double3 f0 = F, t0 = T;
            F -= d.damp * len(f0) * normalize(xyz(v4));
            T -= d.damp * len(t0) * normalize(xyz(d.angv[i]));
        }
        // addBuoyancyDragKernel (externalForceTorque.cu:66-133)
        if (d.buoy && !(v4.w <= 0.0)) {
            double3 Fbd = buoyancy_drag(ri, xyz(v4), p4.w, d.brho, d.bcd, d.bg3, d.bu, d.blevel);
            F.x += Fbd.x;
            F.y += Fbd.y;
            F.z += Fbd.z;
        }
    }
    // integ = 1 is the first evaluation of a step with no clumps and no hook:
    // nothing reads its force and torque before the second evaluation
    // overwrites them, so only the second stores them (64 B per sphere less)
    if (integ != 1) {
        d.force[i] = d4(F, 0);
        d.torque[i] = d4(T, 0);
    }
    if (integ) {
        // ballVelocityAngularVelocityIntegrationKernel (ballIntegrationKernel.cu:30-56)
        double3 v = xyz(v4);
        double im = v4.w;
        if (d.clump[i] < 0 && !(im < 1.e-20)) {
            v += (F * im + d.gravity) * hdt;
            d.vel[i] = d4(v, im);
            if (!(p4.w < 1.e-20)) {
                double I = 0.4 * p4.w * p4.w / im;
                double3 w = xyz(d.angv[i]) + T / I * hdt;
                d.angv[i] = d4(w, 0);
            }
        }
        // positionIntegrationKernel (ballIntegrationKernel.cu:112-121), first half only
        if (integ == 1) d.pos[i] = d4(ri + (2.0 * hdt) * v, p4.w);
    }
}

// ----------------------------------------------------------- integration --
// sumClumpForceTorqueKernel (ballIntegrationKernel.cu:3-28, Q1 corrected: the
// pebble forces are summed) + clumpVelocityAngularVelocityIntegrationKernel
// (:58-79) + in the first half the clump drift and quaternion update (:101-121).
__global__ void k_dem_clumps(DemDev d, double hdt, int first) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= d.nClump) return;
    int2 pe = d.cpeb[c];
    double3 cp = xyz(d.cpos[c]);
    double3 Fc = mk3(0, 0, 0), Tc = mk3(0, 0, 0);
    for (int i = pe.x; i < pe.y; i++) {
        double3 Fi = xyz(d.force[i]);
        Fc += Fi;
        Tc += xyz(d.torque[i]) + cross(xyz(d.pos[i]) - cp, Fi);
    }
    d.cforce[c] = d4(Fc, 0);
    d.ctorque[c] = d4(Tc, 0);
    double im = d.cinvm[c];
    double3 v = xyz(d.cvel[c]), w = xyz(d.cangv[c]);
    double4 q = d.cq[c];
    if (im > 1.e-20) {
        v += (Fc * im + d.gravity) * hdt;
        w += rot_inv_inertia_apply(q, d.cinvIa[c], d.cinvIb[c], Tc) * hdt;
        d.cvel[c] = d4(v, 0);
        d.cangv[c] = d4(w, 0);
    }
    if (first) {
        d.cpos[c] = d4(cp + (2.0 * hdt) * v, 0);
        d.cq[c] = quat_rotate(q, w, 2.0 * hdt);
    }
}
// setPebbleVelocityAngularVelocityKernel (ballIntegrationKernel.cu:81-99)
__global__ void k_dem_pebbles(DemDev d) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.N) return;
    int c = d.clump[i];
    if (c < 0) return;
    double3 w = xyz(d.cangv[c]);
    d.angv[i] = d4(w, 0);
    double4 v4 = d.vel[i];
    d.vel[i] = d4(xyz(d.cvel[c]) + cross(w, xyz(d.pos[i]) - xyz(d.cpos[c])), v4.w);
}
// ballVelocityAngularVelocityIntegrationKernel + positionIntegrationKernel
// (ballIntegrationKernel.cu:30-56,112-121) for scenes with clumps.
__global__ void k_dem_integrate(DemDev d, double hdt, int first) {
    chain_enter();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.N) return;
    double4 v4 = d.vel[i];
    double3 v = xyz(v4);
    double im = v4.w;
    if (d.clump[i] < 0 && !(im < 1.e-20)) {
        v += (xyz(d.force[i]) * im + d.gravity) * hdt;
        d.vel[i] = d4(v, im);
        double r = d.pos[i].w;
        if (!(r < 1.e-20)) {
            double I = 0.4 * r * r / im;
            d.angv[i] = d4(xyz(d.angv[i]) + xyz(d.torque[i]) / I * hdt, 0);
        }
    }
    if (first) {
        double4 p = d.pos[i];
        d.pos[i] = d4(xyz(p) + (2.0 * hdt) * v, p.w);
    }
}
// The ball arrays in the reference's layout (ball_ of particle.h: double3
// position, velocity, angular velocity, force, torque; double radius and
// inverse mass), written before an addExternalForceTorque callback and read
// back after it, so the callback's kernels see and change the state as the
// reference's hooks do.
struct HookArrays {
    double3* pos;
    double3* vel;
    double3* angv;
    double3* force;
    double3* torque;
    double* rad;
    double* invm;
};
__global__ void k_dem_hook_out(DemDev d, HookArrays h) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.N) return;
    const double4 p = d.pos[i], v = d.vel[i];
    h.pos[i] = xyz(p);
    h.rad[i] = p.w;
    h.vel[i] = xyz(v);
    h.invm[i] = v.w;
    h.angv[i] = xyz(d.angv[i]);
    h.force[i] = xyz(d.force[i]);
    h.torque[i] = xyz(d.torque[i]);
}
__global__ void k_dem_hook_in(DemDev d, HookArrays h) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.N) return;
    d.pos[i] = d4(h.pos[i], h.rad[i]);
    d.vel[i] = d4(h.vel[i], h.invm[i]);
    d.angv[i] = d4(h.angv[i], 0);
    d.force[i] = d4(h.force[i], 0);
    d.torque[i] = d4(h.torque[i], 0);
}
// FP64 conservation diagnostics of a DEM scene, per object (the balls, then
// the clumps), summed by diag_reduce:
//   0-2  linear momentum  sum m v            (moving bodies: free spheres and
//   3-5  angular momentum sum x x m v + I w   clumps; pebbles count through
//   6    translational kinetic energy         their clump; fixed balls, with
//   7    rotational kinetic energy            inverse mass 0, not at all)
//   8    mass
//   9-11 sum of the ball forces of the last force evaluation (all balls: the
//        contact and bond forces cancel pairwise, so this is the sum of the
//        external and wall forces)
struct DemDiagTerm {
    DemDev d;
    __device__ void operator()(int i, double* v) const {
#pragma unroll
        for (int k = 0; k < 12; k++) v[k] = 0.0;
        double3 x, u, w, L;
        double m;
        if (i < d.N) {
            const double3 F = xyz(d.force[i]);
            v[9] = F.x; v[10] = F.y; v[11] = F.z;
            const double4 v4 = d.vel[i];
            if (!(v4.w > 0.0) || d.clump[i] >= 0) return;
            const double4 p4 = d.pos[i];
            m = 1.0 / v4.w;
            x = xyz(p4); u = xyz(v4); w = xyz(d.angv[i]);
            L = (0.4 * m * p4.w * p4.w) * w;
        } else {
            const int c = i - d.N;
            const double im = d.cinvm[c];
            if (!(im > 1.e-20)) return;
            m = 1.0 / im;
            x = xyz(d.cpos[c]); u = xyz(d.cvel[c]); w = xyz(d.cangv[c]);
            // world inverse inertia R I^-1 R^T by columns, then I_world w by Cramer's rule
            const double4 q = d.cq[c], Ia = d.cinvIa[c], Ib = d.cinvIb[c];
            const double3 c0 = rot_inv_inertia_apply(q, Ia, Ib, mk3(1, 0, 0));
            const double3 c1 = rot_inv_inertia_apply(q, Ia, Ib, mk3(0, 1, 0));
            const double3 c2 = rot_inv_inertia_apply(q, Ia, Ib, mk3(0, 0, 1));
            const double det = dot(c0, cross(c1, c2));
            L = (fabs(det) > 0.0) ? mk3(dot(w, cross(c1, c2)), dot(c0, cross(w, c2)), dot(c0, cross(c1, w))) / det
                                  : mk3(0, 0, 0);
        }
        const double3 P = m * u;
        const double3 Lx = cross(x, P) + L;
        v[0] = P.x; v[1] = P.y; v[2] = P.z;
        v[3] = Lx.x; v[4] = Lx.y; v[5] = Lx.z;
        v[6] = 0.5 * m * dot(u, u);
        v[7] = 0.5 * dot(w, L);
        v[8] = m;
    }
};

// wallPositionIntegrationKernel + wallOrientationIntegrationKernel (wallIntegrationKernel.cu:3-23)
__global__ void k_dem_wall_move(DemDev d, double dt) {
    int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= d.nWall) return;
    d.wpos[w] = d4(xyz(d.wpos[w]) + dt * xyz(d.wvel[w]), 0);
    d.wq[w] = quat_rotate(d.wq[w], xyz(d.wangv[w]), dt);
}
// updateWallVertexGlobalPosition (wallIntegrationKernel.cu:25-37)
__global__ void k_dem_vertices(DemDev d) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= d.nVert) return;
    int w = d.vwall[v];
    d.vglobal[v] = d4(xyz(d.wpos[w]) + quat_apply(d.wq[w], xyz(d.vlocal[v])), 0);
}
// updateTriangleCircumcenter (wallIntegrationKernel.cu:39-53)
__global__ void k_dem_circumcenters(DemDev d) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= d.nTri) return;
    int4 tv = d.tris[t];
    d.tcenter[t] = d4(circumcenter(xyz(d.vglobal[tv.x]), xyz(d.vglobal[tv.y]), xyz(d.vglobal[tv.z])), 0);
}

// -------------------------------------------------------- periodic ghosts --
// buildDummyPosition (neighborSearchKernel.cu:57-77): every ball, shifted by
// the domain length along each flagged axis where it lies within one cell of
// the lower face.
__global__ void k_dem_ghost_pos(int n, const double4* __restrict__ pos, double4* __restrict__ gpos, GridDesc g,
                                int3 dir) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 p = pos[i];
    const double3 L = g.mx - g.mn;
    if (dir.x == 1 && p.x - g.mn.x < g.cs.x) p.x += L.x;
    if (dir.y == 1 && p.y - g.mn.y < g.cs.y) p.y += L.y;
    if (dir.z == 1 && p.z - g.mn.z < g.cs.z) p.z += L.z;
    gpos[i] = p;
}
// Adds one ghost pass's pair forces into the A-side accumulators: the
// pointed-side sums (written by k_dem_pair_forces into FA / TA) and the
// pointing-side sums over the ghost reverse lists
// (sumObjectPointed / sumObjectPointingForceTorqueFromInteractionKernel,
// contactKernel.cu:657-714, with the ghost positions as torque arms).
__global__ void k_dem_ghost_sum(int n, const double4* __restrict__ FA, const double4* __restrict__ TA,
                                const int* __restrict__ rcnt, const int* __restrict__ rslot, int KR,
                                const double4* __restrict__ pF, const double4* __restrict__ pTB,
                                double4* __restrict__ forceA, double4* __restrict__ torqueA) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double3 F = xyz(FA[i]), T = xyz(TA[i]);
    const int c = min(rcnt[i], KR);
    for (int r = 0; r < c; r++) {
        const int slot = rslot[(size_t)r * n + i];
        F -= xyz(pF[slot]);
        T += xyz(pTB[slot]);
    }
    forceA[i] = d4(xyz(forceA[i]) + F, 0);
    torqueA[i] = d4(xyz(torqueA[i]) + T, 0);
}

// ------------------------------------------------------------ batching ----
// Places one batch member's balls at [start, start + n) of the batch arrays,
// translated by off, with material ids shifted by matOff and the member's
// clump ids (clumpLocal, -1 for a free ball; may be null) by clumpOff.
__global__ void k_dem_place(int n, int start, double3 off, int matOff, int clumpOff, const double4* __restrict__ pos,
                            const double4* __restrict__ vel, const double4* __restrict__ angv,
                            const int* __restrict__ mat, const int* __restrict__ clumpLocal,
                            double4* __restrict__ pos2, double4* __restrict__ vel2, double4* __restrict__ angv2,
                            int* __restrict__ mat2, int* __restrict__ clump2) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const double4 p = pos[t];
    pos2[start + t] = make_double4(p.x + off.x, p.y + off.y, p.z + off.z, p.w);
    vel2[start + t] = vel[t];
    angv2[start + t] = angv[t];
    mat2[start + t] = mat[t] + matOff;
    const int c = clumpLocal ? clumpLocal[t] : -1;
    clump2[start + t] = c >= 0 ? c + clumpOff : -1;
}

// Carries the bodies of continuing batch members from another scene: clumps
// [srcC, srcC + nC) there become [dstC, ...) here (centroid translated by
// shift, velocity, angular velocity, orientation), bonds [srcB, srcB + nB)
// become [dstB, ...) (intact flag, contact point translated by shift,
// normal, the accumulated normal / shear forces and torques and the peak
// stresses).  The pebbles and the bonds' end balls move with the member's
// balls (k_dem_copy_member).
__global__ void k_dem_copy_bodies(DemDev dst, DemDev src, int srcC, int dstC, int nC, int srcB, int dstB, int nB,
                                  double3 shift) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nC) {
        const int a = dstC + t, b = srcC + t;
        const double4 c = src.cpos[b];
        dst.cpos[a] = make_double4(c.x + shift.x, c.y + shift.y, c.z + shift.z, c.w);
        dst.cvel[a] = src.cvel[b];
        dst.cangv[a] = src.cangv[b];
        dst.cq[a] = src.cq[b];
    }
    if (t < nB) {
        const int a = dstB + t, b = srcB + t;
        dst.bok[a] = src.bok[b];
        const double4 p = src.bpoint[b];
        dst.bpoint[a] = make_double4(p.x + shift.x, p.y + shift.y, p.z + shift.z, p.w);
        dst.bnormal[a] = src.bnormal[b];
        dst.bFs[a] = src.bFs[b];
        dst.bTb[a] = src.bTb[b];
        dst.bFn[a] = src.bFn[b];
        dst.bTt[a] = src.bTt[b];
        dst.bsmax[a] = src.bsmax[b];
        dst.btmax[a] = src.btmax[b];
    }
}

// Copies the state of one continuing batch member from another scene: its n
// balls at [srcStart, srcStart + n) there go to [dstStart, dstStart + n) here
// -- kinematics translated by shift, pair rows with partner indices moved by
// dstStart - srcStart, ball-triangle rows with triangle indices moved by
// triDelta.  A partner outside the member's range means inconsistent maps:
// the entry is dropped and bad_index set.
__global__ void k_dem_copy_member(DemDev dst, DemDev src, int n, int srcStart, int dstStart, int triDelta,
                                  double3 shift) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int s = srcStart + t, a = dstStart + t;
    const int bd = dstStart - srcStart;
    double4 p = src.pos[s];
    dst.pos[a] = make_double4(p.x + shift.x, p.y + shift.y, p.z + shift.z, p.w);
    dst.vel[a] = src.vel[s];
    dst.angv[a] = src.angv[s];
    dst.force[a] = src.force[s];
    dst.torque[a] = src.torque[s];
    int c = src.pcnt[s];
    int kept = 0;
    for (int k = 0; k < c; k++) {
        size_t so = (size_t)k * src.N + s, dO = (size_t)kept * dst.N + a;
        int j = src.pj[so] + bd;
        if (j < dstStart || j >= dstStart + n) {
            atomicExch(&dst.status->bad_index, 1);
            continue;
        }
        dst.pj[dO] = j;
        dst.spS[dO] = src.spS[so];
        if (dst.roll) dst.spR[dO] = src.spR[so];
        if (dst.tors) dst.spT[dO] = src.spT[so];
        kept++;
    }
    dst.pcnt[a] = kept;
    if (dst.nTri && src.nTri && src.wcnt) {
        int cw = src.wcnt[s];
        kept = 0;
        for (int k = 0; k < cw; k++) {
            size_t so = (size_t)k * src.N + s, dO = (size_t)kept * dst.N + a;
            int tr = src.wtj[so] + triDelta;
            if (tr < 0 || tr >= dst.nTri) {
                atomicExch(&dst.status->bad_index, 1);
                continue;
            }
            dst.wtj[dO] = tr;
            dst.wS[dO] = src.wS[so];
            if (dst.roll) dst.wR[dO] = src.wR[so];
            if (dst.tors) dst.wT[dO] = src.wT[so];
            kept++;
        }
        dst.wcnt[a] = kept;
    }
}

// ================================================================ host =====
struct HostMatRows {
    struct Row { int a, b; double v[11]; };
    std::vector<Row> h, l, bd;
};

struct DemScene {
    cudaStream_t s = 0;
    int precision = DEMSPH_PRECISION_MIXED;
    bool ready = false;
    // host staging (the reference's host halves of HostDeviceArray1D)
    std::vector<double4> hPos, hVel, hAngv;
    std::vector<int> hMat, hClump;
    HostMatRows rows;
    std::vector<MatPair> hMatTab;  // the pair-parameter table (host copy of `mats`)
    std::vector<double4> hCpos, hCvel, hCangv, hCq, hCinvIa, hCinvIb;
    std::vector<double> hCinvm;
    std::vector<int2> hCpeb;
    std::vector<double4> hWpos, hWvel, hWangv, hWq;
    std::vector<int> hWmat;
    std::vector<double4> hVlocal;
    std::vector<int> hVwall;
    std::vector<int4> hTris;
    std::vector<int2> hBab;
    std::vector<double4> hBpoint, hBnormal;
    std::vector<double4> hFconst;
    double framp = 0, damp = 0;
    int buoy = 0;
    double brho = 0, bcd = 0, blevel = 0;
    double3 bg3{0, 0, 0}, bu{0, 0, 0};
    // parameters
    double3 gmin{0, 0, 0}, gmax{0, 0, 0}, gravity{0, 0, 0};
    double dt = 0;
    long iStep = 0;
    double time = 0;
    int K = 16, KR = 16, KT = 8;
    int nMat = 0, cap = 0, roll = 0, tors = 0;
    bool wallsMove = false;
    // device
    DBuf<MatPair> mats;
    DBuf<double4> pos, vel, angv, force, torque, forceA, torqueA;
    DBuf<int> mat, clump;
    CellTable ballCells, triCells;
    DBuf<int> pj[2], pcnt[2];
    DBuf<double4> spS[2], spR[2], spT[2];
    int cur = 0;
    bool havePairs = false;
    DBuf<double4> pF, pTB;
    DBuf<int> rcnt, rslot;
    DBuf<int2> bab;
    DBuf<int> bok;
    DBuf<double4> bpoint, bnormal, bFs, bTb, bF, bTA, bTB;
    DBuf<double> bFn, bTt, bsmax, btmax;
    DBuf<int> bincStart, binc;
    DBuf<int> bpair;
    bool bondPairsStale = true;  // bpair does not describe the current pair list
    DBuf<double4> wpos, wvel, wangv, wq, vlocal, vglobal, tcenter;
    DBuf<double4> wbox;
    DBuf<int> wmat, vwall;
    DBuf<int4> tris;
    DBuf<int> wtj[2], wcnt[2];
    DBuf<double4> wS[2], wR[2], wT[2];
    int wcur = 0;
    bool haveWallRows = false;
    DBuf<double4> cpos, cvel, cangv, cforce, ctorque, cq, cinvIa, cinvIb;
    DBuf<double> cinvm;
    DBuf<int2> cpeb;
    DBuf<double4> fconst;
    DBuf<double4> cplF, cplT;  // fluid coupling force / torque per ball (allocated by a coupling)
    // inside a coupled block: the DEM launches on the block's stream; its own is kept here
    cudaStream_t blockOwn = 0;
    bool inBlock = false;
    DBuf<DevStatus> status;
    DBuf<double> diagScratch;
    static constexpr int kMergedWallBalls = 65536;  // up to this size k_dem_pair_walls
    // Up to this size the force-evaluation kernels are chained launches: the
    // 4,096-sphere bounce 23.4 -> 21.4 us per step in FP64, 19.9 -> 19.6
    // mixed, the touching pack 53.9 -> 52.5; the 220k beam was 0.8% slower.
    static constexpr int kChainBalls = 65536;

    // Periodic boundaries (setPeriodicBoundary, DEMSolver.h:1944-1959): one
    // ghost set per active direction, passed in the reference's order X, Y,
    // Z, XY, YZ, XZ, XYZ (DEMSolver.h:1416-1422).  Each force evaluation of a
    // step rebuilds the set's ghost positions, its table of ghosts that left
    // the domain, its ghost pair list (springs carried from the previous
    // evaluation's list) and adds the ghost pair forces
    // (addDummyContactForceTorque, DEMSolver.h:279-426).
    struct GhostSet {
        int3 dir;
        DBuf<double4> gpos;
        CellTable cells;
        DBuf<int> pj[2], pcnt[2];
        DBuf<double4> spS[2], spR[2], spT[2];
        int cur = 0;
        bool have = false;
        DBuf<double4> pF, pTB, FA, TA;
        DBuf<int> rcnt, rslot;
        int K = 8, KR = 8;
    };
    bool perX = false, perY = false, perZ = false;
    std::vector<std::unique_ptr<GhostSet>> ghosts;
    DBuf<DevStatus> gstatus;

    int nB = 0;                // balls (the host arrays' size until a batch assembly)
    bool assembled = false;    // balls placed on the device from member records
    double assembledRmax = 0;  // their largest radius
    double cellFactor = 1.0;   // ball grid cell = cellFactor x 2 r_max (autotuner; 1 = the reference's)
    int N() const { return nB; }

    DemDev dev(bool withOld) {
        DemDev d{};
        d.N = N(); d.K = K; d.KR = KR; d.KT = KT;
        d.nBond = (int)hBab.size(); d.nTri = (int)hTris.size(); d.nVert = (int)hVlocal.size();
        d.nWall = (int)hWpos.size(); d.nClump = (int)hCpos.size();
        d.nMat = nMat; d.cap = cap; d.roll = roll; d.tors = tors;
        d.bg = ballCells.g; d.tg = triCells.g;
        d.mats = mats.p;
        d.pos = pos.p; d.vel = vel.p; d.angv = angv.p; d.force = force.p; d.torque = torque.p;
        d.forceA = forceA.p; d.torqueA = torqueA.p; d.mat = mat.p; d.clump = clump.p;
        d.order = ballCells.sorted.p; d.qorder = ballCells.sorted.p; d.cellStart = ballCells.start.p;
        int o = cur ^ 1;
        d.pj = pj[cur].p; d.pcnt = pcnt[cur].p; d.spS = spS[cur].p; d.spR = spR[cur].p; d.spT = spT[cur].p;
        if (withOld && havePairs) {
            d.pjOld = pj[o].p; d.pcntOld = pcnt[o].p; d.spSOld = spS[o].p; d.spROld = spR[o].p; d.spTOld = spT[o].p;
        }
        d.pF = pF.p; d.pTB = pTB.p; d.rcnt = rcnt.p; d.rslot = rslot.p;
        d.bab = bab.p; d.bok = bok.p; d.bpoint = bpoint.p; d.bnormal = bnormal.p; d.bFs = bFs.p; d.bTb = bTb.p;
        d.bFn = bFn.p; d.bTt = bTt.p; d.bsmax = bsmax.p; d.btmax = btmax.p; d.bF = bF.p; d.bTA = bTA.p; d.bTB = bTB.p;
        d.bpair = bpair.p;
        d.bincStart = bincStart.p; d.binc = binc.p;
        d.wpos = wpos.p; d.wvel = wvel.p; d.wangv = wangv.p; d.wq = wq.p; d.wmat = wmat.p;
        d.vlocal = vlocal.p; d.vglobal = vglobal.p; d.vwall = vwall.p; d.tris = tris.p; d.tcenter = tcenter.p;
        d.triOrder = triCells.sorted.p; d.triCellStart = triCells.start.p; d.wbox = wbox.p;
        int wo = wcur ^ 1;
        d.wtj = wtj[wcur].p; d.wcnt = wcnt[wcur].p; d.wS = wS[wcur].p; d.wR = wR[wcur].p; d.wT = wT[wcur].p;
        if (haveWallRows) {
            d.wtjOld = wtj[wo].p; d.wcntOld = wcnt[wo].p; d.wSOld = wS[wo].p; d.wROld = wR[wo].p; d.wTOld = wT[wo].p;
        }
        d.cpos = cpos.p; d.cvel = cvel.p; d.cangv = cangv.p; d.cforce = cforce.p; d.ctorque = ctorque.p; d.cq = cq.p;
        d.cinvIa = cinvIa.p; d.cinvIb = cinvIb.p; d.cinvm = cinvm.p; d.cpeb = cpeb.p;
        d.fconst = hFconst.empty() ? nullptr : fconst.p;
        d.cplF = cplF.p;
        d.cplT = cplT.p;
        d.framp = framp; d.damp = damp; d.buoy = buoy; d.brho = brho; d.bcd = bcd; d.blevel = blevel;
        d.bg3 = bg3; d.bu = bu; d.gravity = gravity;
        d.status = status.p;
        return d;
    }

    // ------------------------------------------------------- set-up ------
    void build_materials() {
        int mx = -1;
        for (auto& r : rows.h) mx = std::max(mx, std::max(r.a, r.b));
        for (auto& r : rows.l) mx = std::max(mx, std::max(r.a, r.b));
        for (auto& r : rows.bd) mx = std::max(mx, std::max(r.a, r.b));
        nMat = mx < 0 ? 0 : mx + 1;
        cap = nMat > 0 ? nMat * (nMat + 1) / 2 + 1 : 0;
        // defaults of buildFromTables (contactKernel.cu:18-31)
        MatPair def{};
        def.linear = 0; def.D = 0.0;  // e = 1 -> ln e = 0
        def.gamma = 1.0; def.knks = 1.0;
        std::vector<MatPair> tab(std::max(cap, 1), def);
        std::vector<double> res(std::max(cap, 1), 1.0);
        for (auto& r : rows.h) {
            int ip = pair_param_index(r.a, r.b, nMat, cap);
            MatPair& m = tab[ip];
            m.E = r.v[0]; m.G = r.v[1]; res[ip] = r.v[2]; m.krks = r.v[3]; m.ktks = r.v[4];
        }
        std::vector<std::array<double, 3>> hmu(std::max(cap, 1), {0, 0, 0});
        for (auto& r : rows.h) {
            int ip = pair_param_index(r.a, r.b, nMat, cap);
            hmu[ip] = {r.v[5], r.v[6], r.v[7]};
        }
        std::vector<std::array<double, 11>> lin(std::max(cap, 1));
        for (auto& x : lin) x.fill(0.0);
        for (auto& r : rows.l) {
            int ip = pair_param_index(r.a, r.b, nMat, cap);
            for (int k = 0; k < 11; k++) lin[ip][k] = r.v[k];
        }
        for (auto& r : rows.bd) {
            int ip = pair_param_index(r.a, r.b, nMat, cap);
            MatPair& m = tab[ip];
            m.gamma = r.v[0]; m.Eb = r.v[1]; m.knks = r.v[2]; m.sigma = r.v[3]; m.C = r.v[4]; m.mu = r.v[5];
        }
        roll = tors = 0;
        for (int ip = 0; ip < (int)tab.size(); ip++) {
            MatPair& m = tab[ip];
            double logR = std::log(res[ip]);
            m.D = -logR / std::sqrt(logR * logR + kPi * kPi);
            if (lin[ip][0] > 1.e-20) {
                m.linear = 1;
                m.kn = lin[ip][0]; m.ks = lin[ip][1]; m.kr = lin[ip][2]; m.kt = lin[ip][3];
                m.dn = lin[ip][4]; m.ds = lin[ip][5]; m.dr = lin[ip][6]; m.dt = lin[ip][7];
                m.mus = lin[ip][8]; m.mur = lin[ip][9]; m.mut = lin[ip][10];
                if (m.kr > 0) roll = 1;
                if (m.kt > 0) tors = 1;
            } else {
                m.linear = 0;
                m.mus = hmu[ip][0]; m.mur = hmu[ip][1]; m.mut = hmu[ip][2];
                if (m.krks > 0 && m.G > 0) roll = 1;
                if (m.ktks > 0 && m.G > 0) tors = 1;
            }
        }
        hMatTab.assign(tab.begin(), tab.end());
        mats.upload(hMatTab, s);
    }

    void upload_bonds() {
        int nb = (int)hBab.size();
        std::vector<int> ok(nb, 1);
        std::vector<double> zero(nb, 0.0);
        std::vector<double4> z4(nb, make_double4(0, 0, 0, 0));
        bab.upload(hBab, s);
        bok.upload(ok, s);
        bpoint.upload(hBpoint, s);
        bnormal.upload(hBnormal, s);
        bFs.upload(z4, s); bTb.upload(z4, s); bF.upload(z4, s); bTA.upload(z4, s); bTB.upload(z4, s);
        bFn.upload(zero, s); bTt.upload(zero, s); bsmax.upload(zero, s); btmax.upload(zero, s);
        // static incidence list per ball, bonds in order (deterministic sum)
        std::vector<int> cnt(N() + 1, 0);
        for (auto& e : hBab) { cnt[e.x + 1]++; cnt[e.y + 1]++; }
        for (int i = 0; i < N(); i++) cnt[i + 1] += cnt[i];
        std::vector<int> inc(std::max(2 * nb, 1)), fill(cnt.begin(), cnt.end() - 1);
        for (int b = 0; b < nb; b++) {
            inc[fill[hBab[b].x]++] = 2 * b;
            inc[fill[hBab[b].y]++] = 2 * b + 1;
        }
        bincStart.upload(cnt, s);
        binc.upload(inc, s);
        bpair.alloc(std::max(nb, 1), s, true);
        bondPairsStale = true;
    }

    void alloc_pairs() {
        graph.reset();  // captured kernels hold the old buffers
        size_t n = (size_t)N();
        for (int b = 0; b < 2; b++) {
            pj[b].alloc(n * K, s, true);
            pcnt[b].alloc(n, s, true);
            spS[b].alloc(n * K, s, true);
            spR[b].alloc(roll ? n * K : 1, s, true);
            spT[b].alloc(tors ? n * K : 1, s, true);
        }
        pF.alloc(n * K, s, true);
        pTB.alloc(n * K, s, true);
        rcnt.alloc(n, s, true);
        rslot.alloc(n * KR, s, true);
    }
    void alloc_wall_rows() {
        graph.reset();
        size_t n = (size_t)N();
        for (int b = 0; b < 2; b++) {
            wtj[b].alloc(n * KT, s, true);
            wcnt[b].alloc(n, s, true);
            wS[b].alloc(n * KT, s, true);
            wR[b].alloc(roll ? n * KT : 1, s, true);
            wT[b].alloc(tors ? n * KT : 1, s, true);
        }
    }
    // Capacity growth keeps the k*N + A layout, so the first planes stay valid.
    void grow(int needPairs, int needRev, int needTri) {
        if (needPairs > K || needRev > KR || needTri > KT) graph.reset();
        bondPairsStale = true;
        size_t n = (size_t)N();
        if (needPairs > K) {
            int nk = needPairs + needPairs / 4 + 1;
            for (int b = 0; b < 2; b++) {
                pj[b].grow(n * nk, s);
                spS[b].grow(n * nk, s);
                if (roll) spR[b].grow(n * nk, s);
                if (tors) spT[b].grow(n * nk, s);
            }
            pF.alloc(n * nk, s, true);
            pTB.alloc(n * nk, s, true);
            K = nk;
        }
        if (needRev > KR) {
            int nk = needRev + needRev / 4 + 1;
            rslot.alloc(n * nk, s, true);
            KR = nk;
        }
        if (needTri > KT) {
            int nk = std::min(needTri + needTri / 4 + 1, kMaxTriPerBall);
            if (needTri > kMaxTriPerBall)
                throw Status(DEMSPH_ERR_OVERFLOW, "a ball touches more than 32 candidate triangles");
            for (int b = 0; b < 2; b++) {
                wtj[b].grow(n * nk, s);
                wS[b].grow(n * nk, s);
                if (roll) wR[b].grow(n * nk, s);
                if (tors) wT[b].grow(n * nk, s);
            }
            KT = nk;
        }
    }

    void launch_count(int k) { g_launches += k; }

    // ------------------------------------------------- periodic ghosts -----
    void ghost_alloc(GhostSet& g) {
        const size_t n = (size_t)N();
        for (int b = 0; b < 2; b++) {
            g.pj[b].alloc(n * g.K, s, true);
            g.pcnt[b].alloc(n, s, true);
            g.spS[b].alloc(n * g.K, s, true);
            g.spR[b].alloc(roll ? n * g.K : 1, s, true);
            g.spT[b].alloc(tors ? n * g.K : 1, s, true);
        }
        g.pF.alloc(n * g.K, s, true);
        g.pTB.alloc(n * g.K, s, true);
        g.FA.alloc(n, s, true);
        g.TA.alloc(n, s, true);
        g.rcnt.alloc(n, s, true);
        g.rslot.alloc(n * g.KR, s, true);
    }
    void ghost_setup() {
        ghosts.clear();
        auto add = [&](int x, int y, int z) {
            auto g = std::make_unique<GhostSet>();
            g->dir = make_int3(x, y, z);
            ghosts.push_back(std::move(g));
        };
        if (perX) add(1, 0, 0);
        if (perY) add(0, 1, 0);
        if (perZ) add(0, 0, 1);
        if (perX && perY) add(1, 1, 0);
        if (perY && perZ) add(0, 1, 1);
        if (perX && perZ) add(1, 0, 1);
        if (perX && perY && perZ) add(1, 1, 1);
        for (auto& g : ghosts) {
            g->gpos.alloc(N(), s, false);
            g->cells.setup(ballCells.g, N(), s);
            ghost_alloc(*g);
        }
        gstatus.alloc(1, s, true);
    }
    // Capacity growth keeps the k*N + A layout, as for the main lists.
    void ghost_grow(int needPairs, int needRev) {
        const size_t n = (size_t)N();
        for (auto& gp : ghosts) {
            GhostSet& g = *gp;
            if (needPairs > g.K) {
                graph.reset();
                const int nk = needPairs + needPairs / 4 + 1;
                for (int b = 0; b < 2; b++) {
                    g.pj[b].grow(n * nk, s);
                    g.spS[b].grow(n * nk, s);
                    if (roll) g.spR[b].grow(n * nk, s);
                    if (tors) g.spT[b].grow(n * nk, s);
                }
                g.pF.alloc(n * nk, s, true);
                g.pTB.alloc(n * nk, s, true);
                g.K = nk;
            }
            if (needRev > g.KR) {
                graph.reset();
                const int nk = needRev + needRev / 4 + 1;
                g.rslot.alloc(n * nk, s, true);
                g.KR = nk;
            }
        }
    }
    DemDev ghost_view(GhostSet& g) {
        DemDev d = dev(false);
        d.pos = g.gpos.p;
        d.order = g.cells.sorted.p;
        d.cellStart = g.cells.start.p;
        d.K = g.K;
        d.KR = g.KR;
        const int o = g.cur ^ 1;
        d.pj = g.pj[g.cur].p; d.pcnt = g.pcnt[g.cur].p;
        d.spS = g.spS[g.cur].p; d.spR = g.spR[g.cur].p; d.spT = g.spT[g.cur].p;
        if (g.have) {
            d.pjOld = g.pj[o].p; d.pcntOld = g.pcnt[o].p;
            d.spSOld = g.spS[o].p; d.spROld = g.spR[o].p; d.spTOld = g.spT[o].p;
        } else {
            d.pjOld = nullptr; d.pcntOld = nullptr; d.spSOld = nullptr; d.spROld = nullptr; d.spTOld = nullptr;
        }
        d.pF = g.pF.p; d.pTB = g.pTB.p;
        d.forceA = g.FA.p; d.torqueA = g.TA.p;
        d.rcnt = g.rcnt.p; d.rslot = g.rslot.p;
        d.status = gstatus.p;
        d.nBond = 0;
        d.nTri = 0;
        return d;
    }
    // addDummyContactForceTorque (DEMSolver.h:279-426) of every active set,
    // added into the pointed-side accumulators of this force evaluation.
    void ghost_passes(double dt) {
        const int n = N();
        for (auto& gp : ghosts) {
            GhostSet& g = *gp;
            k_dem_ghost_pos<<<grid_for(n, 256), 256, 0, s>>>(n, pos.p, g.gpos.p, ballCells.g, g.dir);
            g.cells.build(g.gpos.p, n, s, nullptr, true);
            launch_count(1 + g.cells.launches);
            g.cur ^= 1;
            DemDev d = ghost_view(g);
            k_dem_build_pairs<<<grid_for(n, 128), 128, 0, s>>>(d);
            k_zero_ints<<<grid_for(n, 256), 256, 0, s>>>(g.rcnt.p, n);
            k_dem_reverse<<<grid_for(n, 256), 256, 0, s>>>(d);
            k_dem_reverse_order<<<grid_for(n, 256), 256, 0, s>>>(d);
            if (precision == DEMSPH_PRECISION_FP64) k_dem_pair_forces<double><<<grid_for(n, 128), 128, 0, s>>>(d, dt);
            else k_dem_pair_forces<float><<<grid_for(n, 128), 128, 0, s>>>(d, dt);
            k_dem_ghost_sum<<<grid_for(n, 256), 256, 0, s>>>(n, g.FA.p, g.TA.p, g.rcnt.p, g.rslot.p, g.KR, g.pF.p,
                                                             g.pTB.p, forceA.p, torqueA.p);
            launch_count(6);
            DEMSPH_LAUNCH_CHECK();
            g.have = true;
        }
    }

    // ------------------------------------------------------- pieces ------
    void neighbor_search() {
        ballCells.build(pos.p, N(), s);
        launch_count(ballCells.launches);
        cur ^= 1;
        DemDev d = dev(true);
        k_dem_build_pairs<<<grid_for(N(), 128), 128, 0, s>>>(d);
        k_zero_ints<<<grid_for(N(), 256), 256, 0, s>>>(rcnt.p, N());
        k_dem_reverse<<<grid_for(N(), 256), 256, 0, s>>>(d);
        k_dem_reverse_order<<<grid_for(N(), 256), 256, 0, s>>>(d);
        launch_count(4);
        DEMSPH_LAUNCH_CHECK();
        havePairs = true;
        bondPairsStale = true;
    }
    void tri_grid() {
        if (hTris.empty()) return;
        triCells.build(tcenter.p, (int)hTris.size(), s);
        if (wbox.n < 2) wbox.alloc(2, s, false);
        DemDev d = dev(false);
        k_dem_wall_box<<<1, kBoxThreads, 0, s>>>(d);
        launch_count(1 + triCells.launches);
    }
    // calculateBallContactForceTorque(dt) [+ addTriangleContactForceTorque(dtWall)]
    // [+ external hook at extTime] [+ half-step integration]
    void force_eval(double dt, bool walls, double dtWall, bool ext, double extTime, int integ, double hdt,
                    bool ghostPass = false) {
        DemDev d = dev(false);
        const int n = N();
        // small scenes: each kernel is launched while the one before it drains
        // (launch_chained); on large ones the early launch gained nothing
        const bool chain = n <= kChainBalls;
        // small scenes without periodic ghosts: wall contacts in the pair kernel
        const bool merged = walls && !hTris.empty() && n <= kMergedWallBalls && ghosts.empty();
        if (merged) {
            if (wallsMove || !haveWallRows) tri_grid();
            wcur ^= 1;
            d = dev(false);
            if (precision == DEMSPH_PRECISION_FP64)
                launch_chained(k_dem_pair_walls<double>, grid_for(n, 128), 128, s, chain, d, dt, dtWall);
            else
                launch_chained(k_dem_pair_walls<float>, grid_for(n, 128), 128, s, chain, d, dt, dtWall);
        } else {
            if (precision == DEMSPH_PRECISION_FP64) launch_chained(k_dem_pair_forces<double>, grid_for(n, 128), 128, s, chain, d, dt);
            else launch_chained(k_dem_pair_forces<float>, grid_for(n, 128), 128, s, chain, d, dt);
        }
        launch_count(1);
        if (ghostPass && !ghosts.empty()) ghost_passes(dt);
        if (d.nBond) {
            if (bondPairsStale) {
                k_dem_bond_pairs<<<grid_for(d.nBond, 256), 256, 0, s>>>(d);
                launch_count(1);
                bondPairsStale = false;
            }
            launch_chained(k_dem_bonds, grid_for(d.nBond, 128), 128, s, chain, d, dt);
            launch_count(1);
        }
        bool doWalls = walls && !hTris.empty();
        if (doWalls && !merged) {
            if (wallsMove || !haveWallRows) tri_grid();
            wcur ^= 1;
            d = dev(false);
        } else if (!doWalls) {
            d.nTri = 0;
        }
        if (doWalls && !merged) {
            if (precision == DEMSPH_PRECISION_FP64) launch_chained(k_dem_walls<double>, grid_for(n, 128), 128, s, chain, d, dtWall);
            else launch_chained(k_dem_walls<float>, grid_for(n, 128), 128, s, chain, d, dtWall);
            launch_count(1);
        }
        bool clumps = !hCpos.empty();
        const bool hook = ext && hookFn != nullptr;
        int fin = (clumps || hook) ? 0 : integ;
        if (precision == DEMSPH_PRECISION_FP64)
            launch_chained(k_dem_finalize<double>, grid_for(n, 128), 128, s, chain, d, extTime, ext ? 1 : 0, fin, hdt);
        else
            launch_chained(k_dem_finalize<float>, grid_for(n, 128), 128, s, chain, d, extTime, ext ? 1 : 0, fin, hdt);
        launch_count(1);
        if (doWalls) {
            haveWallRows = true;
            if (wallsMove) {
                k_dem_wall_move<<<grid_for(d.nWall, 64), 64, 0, s>>>(d, dtWall);
                k_dem_vertices<<<grid_for(d.nVert, 256), 256, 0, s>>>(d);
                k_dem_circumcenters<<<grid_for(d.nTri, 256), 256, 0, s>>>(d);
                launch_count(3);
            }
        }
        if (hook) run_hook(extTime);
        if ((clumps || hook) && integ) {
            if (clumps) {
                k_dem_clumps<<<grid_for(d.nClump, 128), 128, 0, s>>>(d, hdt, integ == 1);
                k_dem_pebbles<<<grid_for(n, 256), 256, 0, s>>>(d);
                launch_count(2);
            }
            launch_chained(k_dem_integrate, grid_for(n, 256), 256, s, chain, d, hdt, integ == 1 ? 1 : 0);
            launch_count(1);
        }
        DEMSPH_LAUNCH_CHECK();
    }

    // addExternalForceTorque (virtual, DEMSolver.h:1372; called after each
    // force evaluation of a step, :1464,1470): a caller's callback between
    // the force evaluation and the half-step integration.  The ball state is
    // copied into arrays of the reference's layout before the call and read
    // back after it; the callback's device work must be ordered on the
    // scene's stream or the legacy default stream.
    demsph_dem_hook_fn hookFn = nullptr;
    void* hookUser = nullptr;
    DBuf<double3> hkPos, hkVel, hkAngv, hkForce, hkTorque;
    DBuf<double> hkRad, hkInvm;
    HookArrays hook_arrays() {
        const size_t n = (size_t)N();
        if (hkPos.n < n) {
            hkPos.alloc(n, s, true); hkVel.alloc(n, s, true); hkAngv.alloc(n, s, true);
            hkForce.alloc(n, s, true); hkTorque.alloc(n, s, true);
            hkRad.alloc(n, s, true); hkInvm.alloc(n, s, true);
        }
        return HookArrays{hkPos.p, hkVel.p, hkAngv.p, hkForce.p, hkTorque.p, hkRad.p, hkInvm.p};
    }
    static void order_after(cudaStream_t waiter, cudaStream_t done) {
        cudaEvent_t ev;
        DEMSPH_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        DEMSPH_CUDA(cudaEventRecord(ev, done));
        DEMSPH_CUDA(cudaStreamWaitEvent(waiter, ev, 0));
        DEMSPH_CUDA(cudaEventDestroy(ev));
    }
    void run_hook(double t) {
        const HookArrays h = hook_arrays();
        DemDev d = dev(false);
        k_dem_hook_out<<<grid_for(N(), 256), 256, 0, s>>>(d, h);
        launch_count(1);
        DEMSPH_LAUNCH_CHECK();
        const bool legacy = (s == 0 || s == cudaStreamLegacy);
        if (!legacy) order_after(cudaStreamLegacy, s);
        demsph_dem_hook_fn fn = hookFn;
        if (fn) fn(hookUser, iStep, t);
        if (!legacy) order_after(s, cudaStreamLegacy);
        k_dem_hook_in<<<grid_for(N(), 256), 256, 0, s>>>(d, h);
        launch_count(1);
        DEMSPH_LAUNCH_CHECK();
    }
    // One pass of loop_ball / loop_ball_wall (DEMSolver.h:1376-1485).
    void step_once() {
        const double hdt = 0.5 * dt;
        iStep++;
        time += dt;
        if (iStep % 5 == 0) neighbor_search();
        bool walls = !hTris.empty();
        force_eval(hdt, walls, dt, true, time - hdt, 1, hdt, true);
        force_eval(hdt, walls, dt, true, time, 2, hdt, true);
    }
    // Ten steps per graph, starting one step after a re-sort: two re-sorts
    // per replay, so the pair and wall-row buffer indices are back to their
    // parity.  Only scenes whose step does not depend on the time (no force
    // ramp) are captured, since the hook time is a kernel argument.
    GraphSet graph;
    bool useGraphs = true;
    static constexpr int kGraphSteps = 10;
    int index_key() const {
        int k = cur | wcur << 1;
        for (size_t g = 0; g < ghosts.size(); g++) k |= (ghosts[g]->cur | (ghosts[g]->have ? 2 : 0)) << (2 + 2 * g);
        return k;
    }
    bool graphable() const { return useGraphs && !(framp > 0) && ready && !hookFn; }

    DevStatus read_status() {
        DevStatus h{};
        DEMSPH_CUDA(cudaMemcpyAsync(&h, status.p, sizeof h, cudaMemcpyDeviceToHost, s));
        DEMSPH_CUDA(cudaStreamSynchronize(s));
        return h;
    }
    void clear_status() { DEMSPH_CUDA(cudaMemsetAsync(status.p, 0, sizeof(DevStatus), s)); }

    // ---------------------------------------------------- snapshots ------
    // Dynamic state copied before a batch of steps so that a capacity
    // overflow can be undone, the lists regrown and the steps replayed.
    struct Snap {
        std::vector<std::unique_ptr<DBuf<char>>> bufs;
        std::vector<std::pair<void*, size_t>> src;
        long iStep;
        double time;
        int cur, wcur;
        bool havePairs, haveWallRows;
        int K, KT;
        std::vector<std::pair<int, bool>> ghost;  // (cur, have) per ghost set
    };
    // The snapshot's device copies are kept between calls and reused while
    // they are large enough, so a step() call allocates nothing after the first.
    // The copies are collected and issued as one copy_list launch at the end
    // of take().
    std::vector<CopyItem> snapCopies;
    template <class T>
    void snap_add(Snap& sn, DBuf<T>& b) {
        if (!b.p || b.n == 0) return;
        const size_t k = sn.src.size();
        if (k == sn.bufs.size()) sn.bufs.push_back(std::make_unique<DBuf<char>>());
        DBuf<char>& c = *sn.bufs[k];
        if (c.n < b.bytes()) c.alloc(b.bytes(), s, false);
        snapCopies.push_back({c.p, b.p, b.bytes()});
        sn.src.push_back({(void*)&b, b.bytes()});
    }
    void take(Snap& sn) {
        snapCopies.clear();
        sn.src.clear();
        sn.iStep = iStep; sn.time = time; sn.cur = cur; sn.wcur = wcur; sn.havePairs = havePairs;
        sn.haveWallRows = haveWallRows; sn.K = K; sn.KT = KT;
        snap_add(sn, pos); snap_add(sn, vel); snap_add(sn, angv); snap_add(sn, force); snap_add(sn, torque);
        for (int b = 0; b < 2; b++) {
            snap_add(sn, pj[b]); snap_add(sn, pcnt[b]); snap_add(sn, spS[b]);
            if (roll) snap_add(sn, spR[b]);
            if (tors) snap_add(sn, spT[b]);
            snap_add(sn, wtj[b]); snap_add(sn, wcnt[b]); snap_add(sn, wS[b]);
            if (roll) snap_add(sn, wR[b]);
            if (tors) snap_add(sn, wT[b]);
        }
        snap_add(sn, ballCells.sorted); snap_add(sn, ballCells.start);
        snap_add(sn, rcnt); snap_add(sn, rslot);
        snap_add(sn, bok); snap_add(sn, bpoint); snap_add(sn, bnormal); snap_add(sn, bFs); snap_add(sn, bTb);
        snap_add(sn, bFn); snap_add(sn, bTt); snap_add(sn, bsmax); snap_add(sn, btmax);
        snap_add(sn, wpos); snap_add(sn, wq); snap_add(sn, vglobal); snap_add(sn, tcenter);
        snap_add(sn, cpos); snap_add(sn, cvel); snap_add(sn, cangv); snap_add(sn, cq);
        sn.ghost.clear();
        for (auto& gp : ghosts) {
            GhostSet& g = *gp;
            sn.ghost.push_back({g.cur, g.have});
            for (int b = 0; b < 2; b++) {
                snap_add(sn, g.pj[b]); snap_add(sn, g.pcnt[b]); snap_add(sn, g.spS[b]);
                if (roll) snap_add(sn, g.spR[b]);
                if (tors) snap_add(sn, g.spT[b]);
            }
        }
        launch_count(copy_list(snapCopies, s));
        DEMSPH_LAUNCH_CHECK();
    }
    Snap snap;
    void restore(Snap& sn) {
        // pair / reverse rows were regrown in place (layout k*N + A), so the
        // saved prefix is copied back into the start of each buffer.
        snapCopies.clear();
        for (size_t k = 0; k < sn.src.size(); k++) {
            DBuf<char>* dst = (DBuf<char>*)sn.src[k].first;
            snapCopies.push_back({dst->p, sn.bufs[k]->p, sn.src[k].second});
        }
        launch_count(copy_list(snapCopies, s));
        DEMSPH_LAUNCH_CHECK();
        iStep = sn.iStep; time = sn.time; cur = sn.cur; wcur = sn.wcur; havePairs = sn.havePairs;
        haveWallRows = sn.haveWallRows;
        bondPairsStale = true;
        for (size_t g = 0; g < ghosts.size() && g < sn.ghost.size(); g++) {
            ghosts[g]->cur = sn.ghost[g].first;
            ghosts[g]->have = sn.ghost[g].second;
        }
    }

    void steps_graph(long n) {
        long k = 0;
        if (graphable()) {
            for (; k < n && iStep % 5 != 0; k++) step_once();
            // the buffer-state key is taken per block: the first block after
            // initialisation also switches ghost lists to spring carry
            for (; k + kGraphSteps <= n; k += kGraphSteps) {
                StepGraph& gr = graph.at(index_key());
                if (!gr.ready()) {
                    const long i0 = iStep;
                    const double t0 = time;
                    gr.capture(kGraphSteps, s, [&] {
                        for (int j = 0; j < kGraphSteps; j++) step_once();
                    });
                    iStep = i0;
                    time = t0;
                }
                gr.launch(s);
                iStep += kGraphSteps;
                time += kGraphSteps * dt;
            }
        }
        for (; k < n; k++) step_once();
    }

    void run(long n) {
        if (!ready) throw Status(DEMSPH_ERR_NOT_READY, "scene not initialised");
        if (n <= 0) return;
        for (int attempt = 0; attempt < 8; attempt++) {
            Snap& sn = snap;
            take(sn);
            clear_status();
            if (!ghosts.empty()) DEMSPH_CUDA(cudaMemsetAsync(gstatus.p, 0, sizeof(DevStatus), s));
            steps_graph(n);
            DevStatus st = read_status();
            DevStatus gs{};
            if (!ghosts.empty()) {
                DEMSPH_CUDA(cudaMemcpyAsync(&gs, gstatus.p, sizeof gs, cudaMemcpyDeviceToHost, s));
                DEMSPH_CUDA(cudaStreamSynchronize(s));
            }
            if (!st.overflow && !gs.overflow) return;
            if (st.overflow) grow(st.need_pairs, st.need_rev, st.need_aux);
            if (gs.overflow) ghost_grow(gs.need_pairs, gs.need_rev);
            restore(sn);
            // rows past the old capacity hold stale data; the rebuild rewrites them.
        }
        throw Status(DEMSPH_ERR_OVERFLOW, "pair lists kept overflowing after regrowth");
    }

    void initialize(double3 mn, double3 mx, double3 g, double timeStep, int prec) {
        graph.reset();
        if (N() == 0) throw Status(DEMSPH_ERR_SCENE, "the number of particles is equal to 0");
        if (!(timeStep > 0)) throw Status(DEMSPH_ERR_INVALID, "time step must be positive");
        double cell = 0;
        if (!assembled) {
            for (auto& p : hPos) {
                if (!std::isfinite(p.x) || !std::isfinite(p.y) || !std::isfinite(p.z) || !(p.w > 0))
                    throw Status(DEMSPH_ERR_SCENE, "ball with non-finite position or non-positive radius");
            }
            pos.upload(hPos, s); vel.upload(hVel, s); angv.upload(hAngv, s);
            mat.upload(hMat, s); clump.upload(hClump, s);
            for (auto& p : hPos) cell = std::max(cell, p.w * 2.0);
        } else {
            cell = 2.0 * assembledRmax;
        }
        cell *= cellFactor;
        precision = prec;
        gmin = mn; gmax = mx; gravity = g; dt = timeStep;
        build_materials();
        int n = N();
        force.alloc(n, s, true); torque.alloc(n, s, true); forceA.alloc(n, s, true); torqueA.alloc(n, s, true);
        status.alloc(1, s, true);
        // grids (DEMSolver.h:245-263)
        GridDesc bg{};
        if (!grid_set(bg, mn, mx, cell)) throw Status(DEMSPH_ERR_SCENE, "invalid domain or cell size");
        ballCells.setup(bg, n, s);
        double tcell = cell;
        std::vector<double4> cent(hTris.size());
        for (size_t t = 0; t < hTris.size(); t++) {
            double3 a = xyz(hVlocal[hTris[t].x]), b = xyz(hVlocal[hTris[t].y]), c = xyz(hVlocal[hTris[t].z]);
            double3 cc = circumcenter(a, b, c);
            tcell = std::max(tcell, 2.0 * len(a - cc));
            tcell = std::max(tcell, 2.0 * len(b - cc));
            tcell = std::max(tcell, 2.0 * len(c - cc));
            int w = hTris[t].w;
            double3 o = xyz(hWpos[w]);
            cent[t] = d4(circumcenter(a + o, b + o, c + o), 0);
        }
        GridDesc tg{};
        grid_set(tg, mn, mx, tcell);
        if (!hTris.empty()) triCells.setup(tg, (int)hTris.size(), s);
        else triCells.g = tg;
        // bodies
        clump_upload();
        wpos.upload(hWpos, s); wvel.upload(hWvel, s); wangv.upload(hWangv, s); wq.upload(hWq, s);
        wmat.upload(hWmat, s);
        vlocal.upload(hVlocal, s);
        std::vector<double4> vg(hVlocal.size());
        for (size_t v = 0; v < hVlocal.size(); v++) vg[v] = d4(xyz(hVlocal[v]) + xyz(hWpos[hVwall[v]]), 0);
        vglobal.upload(vg, s);
        vwall.upload(hVwall, s);
        tris.upload(hTris, s);
        tcenter.upload(cent, s);
        wallsMove = false;
        for (size_t w = 0; w < hWpos.size(); w++)
            if (len2(xyz(hWvel[w])) > 0 || len2(xyz(hWangv[w])) > 0) wallsMove = true;
        fconst.upload(hFconst, s);
        upload_bonds();
        // lists
        alloc_pairs();
        alloc_wall_rows();
        ghost_setup();
        cur = 0; wcur = 0; havePairs = false; haveWallRows = false;
        // neighbour search + one dt = 0 force evaluation (DEMSolver.h:1995-1997);
        // grow and redo when a first guess of a capacity was too small.
        for (int attempt = 0; attempt < 8; attempt++) {
            clear_status();
            neighbor_search();
            force_eval(0.0, !hTris.empty(), 0.0, false, 0.0, 0, 0.0);
            DevStatus st = read_status();
            if (!st.overflow) break;
            grow(st.need_pairs, st.need_rev, st.need_aux);
            havePairs = false;
            haveWallRows = false;
            if (attempt == 7) throw Status(DEMSPH_ERR_OVERFLOW, "initial pair lists overflow");
        }
        iStep = 0;
        time = 0;
        ready = true;
        DEMSPH_CUDA(cudaStreamSynchronize(s));
    }
    void clump_upload() {
        cpos.upload(hCpos, s); cvel.upload(hCvel, s); cangv.upload(hCangv, s); cq.upload(hCq, s);
        cinvIa.upload(hCinvIa, s); cinvIb.upload(hCinvIb, s); cinvm.upload(hCinvm, s); cpeb.upload(hCpeb, s);
        std::vector<double4> z(hCpos.size(), make_double4(0, 0, 0, 0));
        cforce.upload(z, s); ctorque.upload(z, s);
    }
};

}  // namespace demsph

// ================================================================ C ABI ====
using namespace demsph;

struct demsph_dem_scene {
    DemScene sc;
};

static inline double3 ld3(const double* a, long i) { return mk3(a[3 * i], a[3 * i + 1], a[3 * i + 2]); }
static inline void st3(double* a, long i, double3 v) { a[3 * i] = v.x; a[3 * i + 1] = v.y; a[3 * i + 2] = v.z; }

#define SCENE_CHECK(h) \
    if (!(h)) throw Status(DEMSPH_ERR_INVALID, "null scene handle")

// ------------------------------------------- coupled DEM-SPH stepping ----
namespace demsph {

DemBodies dem_bodies(demsph_dem_t h) {
    DemScene& sc = h->sc;
    if (!sc.ready) throw Status(DEMSPH_ERR_NOT_READY, "DEM scene not initialised");
    const int n = sc.N();
    DEMSPH_CUDA(cudaStreamSynchronize(sc.s));  // the ball state is read on another stream
    if (sc.cplF.n < (size_t)n) {
        sc.cplF.alloc(n, sc.s, true);
        sc.cplT.alloc(n, sc.s, true);
        sc.graph.reset();  // captured finalize launches lack the hook
    }
    return DemBodies{n, sc.pos.p, sc.vel.p, sc.angv.p, sc.cplF.p, sc.cplT.p, sc.dt};
}

static void stream_after(cudaStream_t waiter, cudaStream_t done) {
    if (waiter == done) return;
    cudaEvent_t ev;
    DEMSPH_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    DEMSPH_CUDA(cudaEventRecord(ev, done));
    DEMSPH_CUDA(cudaStreamWaitEvent(waiter, ev, 0));
    DEMSPH_CUDA(cudaEventDestroy(ev));
}

void dem_block_begin(demsph_dem_t h, cudaStream_t s) {
    DemScene& sc = h->sc;
    if (!sc.ready) throw Status(DEMSPH_ERR_NOT_READY, "DEM scene not initialised");
    if (sc.inBlock) throw Status(DEMSPH_ERR_INVALID, "DEM scene already in a coupled block");
    stream_after(s, sc.s);
    sc.blockOwn = sc.s;
    sc.inBlock = true;
    sc.s = s;
    sc.take(sc.snap);
    sc.clear_status();
    if (!sc.ghosts.empty()) DEMSPH_CUDA(cudaMemsetAsync(sc.gstatus.p, 0, sizeof(DevStatus), s));
}

void dem_block_steps(demsph_dem_t h, int n, cudaStream_t s) {
    DemScene& sc = h->sc;
    const cudaStream_t keep = sc.s;
    sc.s = s;
    try {
        for (int k = 0; k < n; k++) sc.step_once();
    } catch (...) {
        sc.s = keep;
        throw;
    }
    sc.s = keep;
}

bool dem_graphable(demsph_dem_t h) { return h->sc.graphable(); }
void dem_clock(demsph_dem_t h, long* iStep, double* time) {
    *iStep = h->sc.iStep;
    *time = h->sc.time;
}
void dem_set_clock(demsph_dem_t h, long iStep, double time) {
    h->sc.iStep = iStep;
    h->sc.time = time;
}
void dem_advance_clock(demsph_dem_t h, long steps) {
    h->sc.iStep += steps;
    h->sc.time += steps * h->sc.dt;
}
int dem_graph_key(demsph_dem_t h) { return h->sc.index_key(); }
long dem_graph_epoch(demsph_dem_t h) { return h->sc.graph.epoch; }

bool dem_block_end(demsph_dem_t h) {
    DemScene& sc = h->sc;
    if (!sc.inBlock) throw Status(DEMSPH_ERR_INVALID, "no coupled block in progress");
    DevStatus st = sc.read_status();
    DevStatus gs{};
    if (!sc.ghosts.empty()) {
        DEMSPH_CUDA(cudaMemcpyAsync(&gs, sc.gstatus.p, sizeof gs, cudaMemcpyDeviceToHost, sc.s));
        DEMSPH_CUDA(cudaStreamSynchronize(sc.s));
    }
    bool ok = !st.overflow && !gs.overflow;
    if (!ok) {
        if (st.overflow) sc.grow(st.need_pairs, st.need_rev, st.need_aux);
        if (gs.overflow) sc.ghost_grow(gs.need_pairs, gs.need_rev);
        sc.restore(sc.snap);
        DEMSPH_CUDA(cudaStreamSynchronize(sc.s));
    }
    sc.s = sc.blockOwn;
    sc.inBlock = false;
    return ok;
}


}  // namespace demsph

// Appends the pebbles and the clump record of addClump (DEMSolver.h:1796-1845)
// to the host tables of T (a scene or a batch member, both with the same
// vectors): pebbles take the clump's mean density for their masses and its
// rigid-body velocity; the clump keeps its centroid, velocity, angular
// velocity, unit orientation and the inverse of its inertia tensor (the
// symmetric inverse of myMat.h:163-179).  Clump cid, pebbles [ps, ps + np).
template <class T>
static void append_clump(T& s, int cid, int ps, long np, const double* pts, const double* rad,
                         const double* centroid, const double* vel, const double* w, double mass, const double* I6,
                         int mat) {
    const int pe = ps + (int)np;
    double3 c = ld3(centroid, 0), v = ld3(vel, 0), ww = ld3(w, 0);
    std::vector<double3> pv(np, v);
    double vol = 0., im = 0.;
    if (mass > 1.e-20) {
        im = 1.0 / mass;
        for (long i = 0; i < np; i++) {
            vol += 4.0 / 3.0 * kPi * std::pow(rad[i], 3.0);
            pv[i] += cross(ww, ld3(pts, i) - c);
        }
    }
    double dave = vol > 0. ? mass / vol : 0.;
    for (long i = 0; i < np; i++) {
        double r = rad[i];
        double m = 4. / 3. * r * r * r * kPi * dave;
        double pim = m > 0.0 ? 1.0 / m : 0.0;
        s.hPos.push_back(d4(ld3(pts, i), r));
        s.hVel.push_back(d4(pv[i], pim));
        s.hAngv.push_back(d4(ww, 0));
        s.hMat.push_back(mat);
        s.hClump.push_back(cid);
    }
    double xx = I6[0], yy = I6[1], zz = I6[2], xy = I6[3], xz = I6[4], yz = I6[5];
    double di = 1.0 / (xx * (yy * zz - yz * yz) + xy * (yz * xz - xy * zz) + xz * (xy * yz - yy * xz));
    double ixx = (yy * zz - yz * yz) * di, iyy = (xx * zz - xz * xz) * di, izz = (xx * yy - xy * xy) * di;
    double ixy = -(xy * zz - xz * yz) * di, ixz = (xy * yz - xz * yy) * di, iyz = -(xx * yz - xz * xy) * di;
    s.hCpos.push_back(d4(c, 0));
    s.hCvel.push_back(d4(v, 0));
    s.hCangv.push_back(d4(ww, 0));
    s.hCq.push_back(make_double4(1, 0, 0, 0));
    s.hCinvIa.push_back(make_double4(ixx, iyy, izz, ixy));
    s.hCinvIb.push_back(make_double4(ixz, iyz, 0, 0));
    s.hCinvm.push_back(im);
    s.hCpeb.push_back(make_int2(ps, pe));
}
extern "C" {

int demsph_dem_create(demsph_dem_t* out, void* stream) {
    return guarded([&] {
        if (!out) throw Status(DEMSPH_ERR_INVALID, "null output pointer");
        default_pool_retention();
        auto* h = new demsph_dem_scene();
        h->sc.s = (cudaStream_t)stream;
        *out = h;
    });
}
int demsph_dem_destroy(demsph_dem_t h) {
    return guarded([&] {
        if (!h) return;
        cudaStream_t s = h->sc.s;
        delete h;
        DEMSPH_CUDA(cudaStreamSynchronize(s));
    });
}
int demsph_dem_set_hertzian_pair(demsph_dem_t h, int a, int b, double E, double G, double e, double krks, double ktks,
                                 double mus, double mur, double mut) {
    return guarded([&] {
        SCENE_CHECK(h);
        h->sc.rows.h.push_back({a, b, {E, G, e, krks, ktks, mus, mur, mut, 0, 0, 0}});
    });
}
int demsph_dem_set_linear_pair(demsph_dem_t h, int a, int b, double kn, double ks, double kr, double kt, double dn,
                               double ds, double dr, double dtt, double mus, double mur, double mut) {
    return guarded([&] {
        SCENE_CHECK(h);
        h->sc.rows.l.push_back({a, b, {kn, ks, kr, kt, dn, ds, dr, dtt, mus, mur, mut}});
    });
}
int demsph_dem_set_bonded_pair(demsph_dem_t h, int a, int b, double gamma, double Eb, double knks, double sigma,
                               double C, double mu) {
    return guarded([&] {
        SCENE_CHECK(h);
        h->sc.rows.bd.push_back({a, b, {gamma, Eb, knks, sigma, C, mu, 0, 0, 0, 0, 0}});
    });
}
int demsph_dem_add_balls(demsph_dem_t h, long n, const double* pos, const double* vel, const double* w,
                         const double* rad, const double* dens, const int* mat, const int* clump, int fixed) {
    return guarded([&] {
        SCENE_CHECK(h);
        DemScene& s = h->sc;
        if (s.ready || s.assembled) throw Status(DEMSPH_ERR_INVALID, "balls must be added before initialisation");
        if (n < 0 || (n > 0 && (!pos || !rad || !mat))) throw Status(DEMSPH_ERR_INVALID, "missing ball arrays");
        for (long i = 0; i < n; i++) {
            double r = rad[i];
            double im = 0.0;
            if (!fixed) {
                double mass = 4. / 3. * r * r * r * kPi * (dens ? dens[i] : 0.0);
                if (mass > 0.0) im = 1.0 / mass;
            }
            s.hPos.push_back(d4(ld3(pos, i), r));
            s.hVel.push_back(d4(fixed || !vel ? mk3(0, 0, 0) : ld3(vel, i), im));
            s.hAngv.push_back(d4(fixed || !w ? mk3(0, 0, 0) : ld3(w, i), 0));
            s.hMat.push_back(mat[i]);
            s.hClump.push_back(clump ? clump[i] : -1);
        }
        s.nB = (int)s.hPos.size();
    });
}
// ------------------------------------------------------ batch members ----
// One scene's balls uploaded once to the device in the library's record
// layout, from which batch scenes are assembled on the device.
struct demsph_dem_member {
    cudaStream_t s = 0;
    std::vector<double4> hPos, hVel, hAngv;  // staging until sealed
    std::vector<int> hMat, hClump;           // hClump: member-local clump id, -1 for a free ball
    // the member's clumps (kept on the host: assembly appends them to the
    // scene's clump table, translated and renumbered)
    std::vector<double4> hCpos, hCvel, hCangv, hCq, hCinvIa, hCinvIb;
    std::vector<double> hCinvm;
    std::vector<int2> hCpeb;
    bool sealed = false;
    int n = 0, matMax = -1;
    double rmax = 0;
    DBuf<double4> pos, vel, angv;
    DBuf<int> mat, clump;
};
int demsph_dem_member_create(demsph_dem_member_t* out, void* stream) {
    return guarded([&] {
        if (!out) throw Status(DEMSPH_ERR_INVALID, "null output pointer");
        auto* m = new demsph_dem_member();
        m->s = (cudaStream_t)stream;
        *out = m;
    });
}
int demsph_dem_member_destroy(demsph_dem_member_t m) {
    return guarded([&] {
        if (!m) return;
        cudaStream_t s = m->s;
        delete m;
        DEMSPH_CUDA(cudaStreamSynchronize(s));
    });
}
int demsph_dem_member_add_balls(demsph_dem_member_t m, long n, const double* pos, const double* vel, const double* w,
                                const double* rad, const double* dens, const int* mat, int fixed) {
    return guarded([&] {
        if (!m) throw Status(DEMSPH_ERR_INVALID, "null member handle");
        if (m->sealed) throw Status(DEMSPH_ERR_INVALID, "member already sealed");
        if (n < 0 || (n > 0 && (!pos || !rad || !mat))) throw Status(DEMSPH_ERR_INVALID, "missing ball arrays");
        for (long i = 0; i < n; i++) {
            double r = rad[i];
            double im = 0.0;
            if (!fixed) {
                double mass = 4. / 3. * r * r * r * kPi * (dens ? dens[i] : 0.0);
                if (mass > 0.0) im = 1.0 / mass;
            }
            m->hPos.push_back(d4(ld3(pos, i), r));
            m->hVel.push_back(d4(fixed || !vel ? mk3(0, 0, 0) : ld3(vel, i), im));
            m->hAngv.push_back(d4(fixed || !w ? mk3(0, 0, 0) : ld3(w, i), 0));
            m->hMat.push_back(mat[i]);
            m->hClump.push_back(-1);
        }
    });
}
int demsph_dem_member_add_clump(demsph_dem_member_t m, long np, const double* pts, const double* rad,
                                const double* centroid, const double* vel, const double* w, double mass,
                                const double* I6, int mat) {
    return guarded([&] {
        if (!m) throw Status(DEMSPH_ERR_INVALID, "null member handle");
        if (m->sealed) throw Status(DEMSPH_ERR_INVALID, "member already sealed");
        if (np < 0 || (np > 0 && (!pts || !rad)) || !centroid || !vel || !w || !I6)
            throw Status(DEMSPH_ERR_INVALID, "missing clump arrays");
        append_clump(*m, (int)m->hCpos.size(), (int)m->hPos.size(), np, pts, rad, centroid, vel, w, mass, I6, mat);
    });
}
int demsph_dem_member_num_clumps(demsph_dem_member_t m, long* n) {
    return guarded([&] {
        if (!m || !n) throw Status(DEMSPH_ERR_INVALID, "null argument");
        *n = (long)m->hCpos.size();
    });
}
int demsph_dem_member_seal(demsph_dem_member_t m) {
    return guarded([&] {
        if (!m) throw Status(DEMSPH_ERR_INVALID, "null member handle");
        if (m->sealed) return;
        if (m->hPos.empty()) throw Status(DEMSPH_ERR_SCENE, "the number of particles is equal to 0");
        for (auto& p : m->hPos) {
            if (!std::isfinite(p.x) || !std::isfinite(p.y) || !std::isfinite(p.z) || !(p.w > 0))
                throw Status(DEMSPH_ERR_SCENE, "ball with non-finite position or non-positive radius");
            m->rmax = std::max(m->rmax, p.w);
        }
        for (int v : m->hMat) {
            if (v < 0) throw Status(DEMSPH_ERR_SCENE, "negative material index");
            m->matMax = std::max(m->matMax, v);
        }
        m->n = (int)m->hPos.size();
        m->pos.upload(m->hPos, m->s); m->vel.upload(m->hVel, m->s); m->angv.upload(m->hAngv, m->s);
        m->mat.upload(m->hMat, m->s);
        if (!m->hCpos.empty()) m->clump.upload(m->hClump, m->s);
        DEMSPH_CUDA(cudaStreamSynchronize(m->s));
        m->hPos = {}; m->hVel = {}; m->hAngv = {}; m->hMat = {}; m->hClump = {};
        m->sealed = true;
    });
}
int demsph_dem_member_count(demsph_dem_member_t m, long* n) {
    return guarded([&] {
        if (!m || !n) throw Status(DEMSPH_ERR_INVALID, "null argument");
        *n = m->sealed ? m->n : (long)m->hPos.size();
    });
}
int demsph_dem_assemble_balls(demsph_dem_t h, int count, const demsph_dem_member_t* members, const double* offsets,
                              const int* matOffset) {
    return guarded([&] {
        SCENE_CHECK(h);
        DemScene& s = h->sc;
        if (s.ready || s.assembled || !s.hPos.empty())
            throw Status(DEMSPH_ERR_INVALID, "assemble needs a scene without balls");
        if (count < 1 || !members || !offsets || !matOffset) throw Status(DEMSPH_ERR_INVALID, "no members");
        long n = 0;
        double rmax = 0;
        for (int k = 0; k < count; k++) {
            const demsph_dem_member* m = members[k];
            if (!m || !m->sealed) throw Status(DEMSPH_ERR_NOT_READY, "member not sealed");
            if (matOffset[k] < 0) throw Status(DEMSPH_ERR_INVALID, "negative material offset");
            n += m->n;
            rmax = std::max(rmax, m->rmax);
        }
        if (n > INT_MAX / 64) throw Status(DEMSPH_ERR_INVALID, "batch too large");
        s.nB = (int)n;
        s.pos.alloc(n, s.s, false); s.vel.alloc(n, s.s, false); s.angv.alloc(n, s.s, false);
        s.mat.alloc(n, s.s, false); s.clump.alloc(n, s.s, false);
        int b0 = 0;
        for (int k = 0; k < count; k++) {
            const demsph_dem_member* m = members[k];
            const int c0 = (int)s.hCpos.size();
            k_dem_place<<<grid_for(m->n, 256), 256, 0, s.s>>>(m->n, b0, ld3(offsets, k), matOffset[k], c0, m->pos.p,
                                                             m->vel.p, m->angv.p, m->mat.p,
                                                             m->hCpos.empty() ? nullptr : m->clump.p, s.pos.p,
                                                             s.vel.p, s.angv.p, s.mat.p, s.clump.p);
            const double3 off = ld3(offsets, k);
            for (size_t c = 0; c < m->hCpos.size(); c++) {
                const double4 p = m->hCpos[c];
                s.hCpos.push_back(make_double4(p.x + off.x, p.y + off.y, p.z + off.z, p.w));
                s.hCvel.push_back(m->hCvel[c]);
                s.hCangv.push_back(m->hCangv[c]);
                s.hCq.push_back(m->hCq[c]);
                s.hCinvIa.push_back(m->hCinvIa[c]);
                s.hCinvIb.push_back(m->hCinvIb[c]);
                s.hCinvm.push_back(m->hCinvm[c]);
                s.hCpeb.push_back(make_int2(m->hCpeb[c].x + b0, m->hCpeb[c].y + b0));
            }
            b0 += m->n;
        }
        g_launches += count;
        DEMSPH_LAUNCH_CHECK();
        s.assembled = true;
        s.assembledRmax = rmax;
    });
}
int demsph_dem_add_clump(demsph_dem_t h, long np, const double* pts, const double* rad, const double* centroid,
                         const double* vel, const double* w, double mass, const double* I6, int mat) {
    return guarded([&] {
        SCENE_CHECK(h);
        DemScene& s = h->sc;
        if (s.ready || s.assembled) throw Status(DEMSPH_ERR_INVALID, "clumps must be added before initialisation");
        if (np < 0 || (np > 0 && (!pts || !rad)) || !centroid || !vel || !w || !I6)
            throw Status(DEMSPH_ERR_INVALID, "missing clump arrays");
        append_clump(s, (int)s.hCpos.size(), s.N(), np, pts, rad, centroid, vel, w, mass, I6, mat);
        s.nB = (int)s.hPos.size();
    });
}
int demsph_dem_add_mesh_wall(demsph_dem_t h, long nv, const double* verts, long nt, const int* i0, const int* i1,
                             const int* i2, const double* position, int mat) {
    return guarded([&] {
        SCENE_CHECK(h);
        DemScene& s = h->sc;
        if (s.ready) throw Status(DEMSPH_ERR_INVALID, "walls must be added before initialisation");
        int mxi = -1;
        for (long t = 0; t < nt; t++) mxi = std::max(mxi, std::max(i0[t], std::max(i1[t], i2[t])));
        if (mxi >= nv) return;  // the reference returns silently (DEMSolver.h:1897)
        int vs = (int)s.hVlocal.size();
        int wi = (int)s.hWpos.size();
        double3 p = ld3(position, 0);
        s.hWpos.push_back(d4(p, 0));
        s.hWvel.push_back(make_double4(0, 0, 0, 0));
        s.hWangv.push_back(make_double4(0, 0, 0, 0));
        s.hWq.push_back(make_double4(1, 0, 0, 0));
        s.hWmat.push_back(mat);
        for (long v = 0; v < nv; v++) {
            s.hVlocal.push_back(d4(ld3(verts, v), 0));
            s.hVwall.push_back(wi);
        }
        for (long t = 0; t < nt; t++) s.hTris.push_back(make_int4(vs + i0[t], vs + i1[t], vs + i2[t], wi));
    });
}
int demsph_dem_set_wall_motion(demsph_dem_t h, int wall, const double* vel, const double* w) {
    return guarded([&] {
        SCENE_CHECK(h);
        DemScene& s = h->sc;
        if (wall < 0 || wall >= (int)s.hWpos.size()) throw Status(DEMSPH_ERR_INVALID, "wall index out of range");
        if (s.ready) throw Status(DEMSPH_ERR_INVALID, "wall motion must be set before initialisation");
        s.hWvel[wall] = d4(ld3(vel, 0), 0);
        s.hWangv[wall] = d4(ld3(w, 0), 0);
    });
}
int demsph_dem_add_bonds(demsph_dem_t h, long n, const int* a0, const int* b0, const double* posHost, long npos) {
    return guarded([&] {
        SCENE_CHECK(h);
        h->sc.graph.reset();  // kernel arguments or buffers change
        DemScene& s = h->sc;
        std::map<std::pair<int, int>, int> have;
        for (auto& e : s.hBab) have[{e.x, e.y}] = 1;
        for (long k = 0; k < n; k++) {
            int i0 = a0[k], i1 = b0[k];
            if (i0 < 0 || i1 < 0 || i0 >= npos || i1 >= npos || i0 == i1) continue;
            int a = std::min(i0, i1), b = std::max(i0, i1);
            if (have.count({a, b})) continue;
            have[{a, b}] = 1;
            double3 pa = ld3(posHost, a), pb = ld3(posHost, b);
            s.hBab.push_back(make_int2(a, b));
            s.hBpoint.push_back(d4(0.5 * (pa + pb), 0));
            s.hBnormal.push_back(d4(normalize(pa - pb), 0));
        }
        if (s.ready) {
            // the reference re-runs initialize() after addInitialCondition (DEMSolver.h:1998)
            s.upload_bonds();
            DEMSPH_CUDA(cudaStreamSynchronize(s.s));
        }
    });
}
int demsph_dem_set_constant_force(demsph_dem_t h, long n, const double* f, double ramp) {
    return guarded([&] {
        SCENE_CHECK(h);
        h->sc.graph.reset();  // kernel arguments or buffers change
        DemScene& s = h->sc;
        s.hFconst.assign(std::max<long>(n, 0), make_double4(0, 0, 0, 0));
        for (long i = 0; i < n; i++) s.hFconst[i] = d4(ld3(f, i), 0);
        if (s.ready) {
            s.hFconst.resize(s.N(), make_double4(0, 0, 0, 0));
            s.fconst.upload(s.hFconst, s.s);
        }
        s.framp = ramp;
    });
}
int demsph_dem_set_global_damping(demsph_dem_t h, double c) {
    return guarded([&] {
        SCENE_CHECK(h);
        h->sc.graph.reset();  // kernel arguments or buffers change
        h->sc.damp = c;
    });
}
int demsph_dem_set_buoyancy_drag(demsph_dem_t h, double rho, double cd, const double* g, const double* u, double lvl) {
    return guarded([&] {
        SCENE_CHECK(h);
        h->sc.graph.reset();  // kernel arguments or buffers change
        DemScene& s = h->sc;
        s.buoy = 1; s.brho = rho; s.bcd = cd; s.bg3 = ld3(g, 0); s.bu = ld3(u, 0); s.blevel = lvl;
    });
}
int demsph_dem_set_external_hook(demsph_dem_t h, demsph_dem_hook_fn fn, void* user) {
    return guarded([&] {
        SCENE_CHECK(h);
        DemScene& s = h->sc;
        if (s.inBlock) throw Status(DEMSPH_ERR_INVALID, "set_external_hook inside a coupled block");
        s.hookFn = fn;
        s.hookUser = fn ? user : nullptr;
    });
}
int demsph_dem_hook_arrays(demsph_dem_t h, demsph_ball_arrays* out) {
    return guarded([&] {
        SCENE_CHECK(h);
        if (!out) throw Status(DEMSPH_ERR_INVALID, "null output pointer");
        DemScene& s = h->sc;
        if (!s.ready) throw Status(DEMSPH_ERR_NOT_READY, "scene not initialised");
        const HookArrays a = s.hook_arrays();
        out->position = (double*)a.pos;
        out->velocity = (double*)a.vel;
        out->angularVelocity = (double*)a.angv;
        out->force = (double*)a.force;
        out->torque = (double*)a.torque;
        out->radius = a.rad;
        out->inverseMass = a.invm;
        out->materialID = s.mat.p;
        out->clumpID = s.clump.p;
        out->n = s.N();
    });
}
int demsph_dem_reserve(demsph_dem_t h, int pairsPerBall, int reversePerBall, int trianglesPerBall) {
    return guarded([&] {
        SCENE_CHECK(h);
        DemScene& s = h->sc;
        if (s.ready) throw Status(DEMSPH_ERR_INVALID, "capacities must be reserved before initialisation");
        if (pairsPerBall < 0 || reversePerBall < 0 || trianglesPerBall < 0)
            throw Status(DEMSPH_ERR_INVALID, "negative capacity");
        s.K = std::max(s.K, pairsPerBall);
        s.KR = std::max(s.KR, reversePerBall);
        s.KT = std::max(s.KT, std::min(trianglesPerBall, kMaxTriPerBall));
    });
}
int demsph_dem_set_cell_factor(demsph_dem_t h, double factor) {
    return guarded([&] {
        SCENE_CHECK(h);
        DemScene& s = h->sc;
        if (s.ready) throw Status(DEMSPH_ERR_INVALID, "the cell size is set before initialisation");
        if (!(factor >= 1.0 && factor <= 4.0)) throw Status(DEMSPH_ERR_INVALID, "cell factor must be in [1, 4]");
        s.cellFactor = factor;
    });
}
int demsph_dem_capacity(demsph_dem_t h, int* pairsPerBall, int* reversePerBall, int* trianglesPerBall) {
    return guarded([&] {
        SCENE_CHECK(h);
        if (pairsPerBall) *pairsPerBall = h->sc.K;
        if (reversePerBall) *reversePerBall = h->sc.KR;
        if (trianglesPerBall) *trianglesPerBall = h->sc.KT;
    });
}
int demsph_dem_set_periodic(demsph_dem_t h, int x, int y, int z) {
    return guarded([&] {
        SCENE_CHECK(h);
        DemScene& s = h->sc;
        if (s.ready) throw Status(DEMSPH_ERR_INVALID, "periodic boundaries must be set before initialisation");
        // setPeriodicBoundary (DEMSolver.h:1944-1959): flags accumulate
        if (x) s.perX = true;
        if (y) s.perY = true;
        if (z) s.perZ = true;
    });
}
int demsph_dem_initialize(demsph_dem_t h, const double* mn, const double* mx, const double* g, double dt, int prec) {
    return guarded([&] {
        SCENE_CHECK(h);
        if (prec != DEMSPH_PRECISION_FP64 && prec != DEMSPH_PRECISION_MIXED)
            throw Status(DEMSPH_ERR_INVALID, "unknown precision mode");
        DemScene& s = h->sc;
        if (!s.hFconst.empty()) s.hFconst.resize(s.N(), make_double4(0, 0, 0, 0));
        s.initialize(ld3(mn, 0), ld3(mx, 0), ld3(g, 0), dt, prec);
    });
}
int demsph_dem_step(demsph_dem_t h, long n) {
    return guarded([&] {
        SCENE_CHECK(h);
        h->sc.run(n);
    });
}
int demsph_dem_neighbor_search(demsph_dem_t h) {
    return guarded([&] {
        SCENE_CHECK(h);
        DemScene& s = h->sc;
        if (!s.ready) throw Status(DEMSPH_ERR_NOT_READY, "scene not initialised");
        s.clear_status();
        s.neighbor_search();
        DevStatus st = s.read_status();
        if (st.overflow) {
            s.grow(st.need_pairs, st.need_rev, 0);
            s.cur ^= 1;  // rebuild from the same previous list
            s.neighbor_search();
        }
    });
}
int demsph_dem_eval_forces(demsph_dem_t h, double dt, int walls, double dtWall) {
    return guarded([&] {
        SCENE_CHECK(h);
        DemScene& s = h->sc;
        if (!s.ready) throw Status(DEMSPH_ERR_NOT_READY, "scene not initialised");
        s.graph.reset();  // the ghost passes flip list buffers outside a graph
        s.force_eval(dt, (walls & 1) != 0, dtWall, (walls & 4) != 0, s.time, 0, 0.0, (walls & 2) != 0);
        DEMSPH_CUDA(cudaStreamSynchronize(s.s));
    });
}
int demsph_dem_set_graphs(demsph_dem_t h, int enable) {
    return guarded([&] {
        SCENE_CHECK(h);
        h->sc.useGraphs = enable != 0;
        h->sc.graph.reset();
    });
}
int demsph_dem_num_balls(demsph_dem_t h, long* n) {
    return guarded([&] { SCENE_CHECK(h); *n = h->sc.N(); });
}
int demsph_dem_num_bonds(demsph_dem_t h, long* n) {
    return guarded([&] { SCENE_CHECK(h); *n = (long)h->sc.hBab.size(); });
}
int demsph_dem_num_clumps(demsph_dem_t h, long* n) {
    return guarded([&] { SCENE_CHECK(h); *n = (long)h->sc.hCpos.size(); });
}
int demsph_dem_step_index(demsph_dem_t h, long* step, double* time) {
    return guarded([&] {
        SCENE_CHECK(h);
        if (step) *step = h->sc.iStep;
        if (time) *time = h->sc.time;
    });
}
int demsph_dem_get_balls(demsph_dem_t h, double* pos, double* vel, double* w, double* force, double* torque) {
    return guarded([&] {
        SCENE_CHECK(h);
        DemScene& s = h->sc;
        if (!s.ready && !s.assembled) {
            for (int i = 0; i < s.N(); i++) {
                if (pos) st3(pos, i, xyz(s.hPos[i]));
                if (vel) st3(vel, i, xyz(s.hVel[i]));
                if (w) st3(w, i, xyz(s.hAngv[i]));
                if (force) st3(force, i, mk3(0, 0, 0));
                if (torque) st3(torque, i, mk3(0, 0, 0));
            }
            return;
        }
        std::vector<double4> a;
        auto get = [&](DBuf<double4>& b, double* o) {
            if (!o) return;
            b.download(a, s.s);
            DEMSPH_CUDA(cudaStreamSynchronize(s.s));
            for (int i = 0; i < s.N(); i++) st3(o, i, xyz(a[i]));
        };
        get(s.pos, pos); get(s.vel, vel); get(s.angv, w);
        if (s.ready) {
            get(s.force, force); get(s.torque, torque);
        } else {
            for (int i = 0; i < s.N(); i++) {
                if (force) st3(force, i, mk3(0, 0, 0));
                if (torque) st3(torque, i, mk3(0, 0, 0));
            }
        }
    });
}
int demsph_dem_set_balls(demsph_dem_t h, const double* pos, const double* vel, const double* w) {
    return guarded([&] {
        SCENE_CHECK(h);
        DemScene& s = h->sc;
        if (!s.ready && !s.assembled) {
            for (int i = 0; i < s.N(); i++) {
                if (pos) { double3 p = ld3(pos, i); s.hPos[i].x = p.x; s.hPos[i].y = p.y; s.hPos[i].z = p.z; }
                if (vel) { double3 p = ld3(vel, i); s.hVel[i].x = p.x; s.hVel[i].y = p.y; s.hVel[i].z = p.z; }
                if (w) { double3 p = ld3(w, i); s.hAngv[i].x = p.x; s.hAngv[i].y = p.y; s.hAngv[i].z = p.z; }
            }
            return;
        }
        // on the device: replace xyz, keep w (radius / inverse mass)
        std::vector<double4> a;
        auto put = [&](DBuf<double4>& b, const double* in) {
            if (!in) return;
            b.download(a, s.s);
            DEMSPH_CUDA(cudaStreamSynchronize(s.s));
            for (int i = 0; i < s.N(); i++) {
                double3 p = ld3(in, i);
                a[i].x = p.x; a[i].y = p.y; a[i].z = p.z;
            }
            DEMSPH_CUDA(cudaMemcpyAsync(b.p, a.data(), a.size() * sizeof(double4), cudaMemcpyHostToDevice, s.s));
            DEMSPH_CUDA(cudaStreamSynchronize(s.s));
        };
        put(s.pos, pos); put(s.vel, vel); put(s.angv, w);
    });
}

// Pair rows flattened into the reference's CSR order.
static void collect_rows(DemScene& s, int which, std::vector<int>& A, std::vector<int>& B, std::vector<size_t>& slot) {
    int n = s.N();
    std::vector<int> cnt, ids;
    if (which >= 2) {  // periodic ghost set which - 2
        const size_t g = (size_t)(which - 2);
        if (g >= s.ghosts.size()) throw Status(DEMSPH_ERR_INVALID, "no such periodic ghost set");
        DemScene::GhostSet& gs = *s.ghosts[g];
        if (!gs.have) return;
        gs.pcnt[gs.cur].download(cnt, s.s);
        gs.pj[gs.cur].download(ids, s.s);
    } else if (which == 0) {
        if (!s.havePairs) return;
        s.pcnt[s.cur].download(cnt, s.s);
        s.pj[s.cur].download(ids, s.s);
    } else {
        if (!s.haveWallRows) return;
        s.wcnt[s.wcur].download(cnt, s.s);
        s.wtj[s.wcur].download(ids, s.s);
    }
    DEMSPH_CUDA(cudaStreamSynchronize(s.s));
    for (int a = 0; a < n; a++)
        for (int k = 0; k < cnt[a]; k++) {
            size_t sl = (size_t)k * n + a;
            A.push_back(a);
            B.push_back(ids[sl]);
            slot.push_back(sl);
        }
}
int demsph_dem_num_pairs(demsph_dem_t h, int which, long* n) {
    return guarded([&] {
        SCENE_CHECK(h);
        std::vector<int> A, B;
        std::vector<size_t> sl;
        collect_rows(h->sc, which, A, B, sl);
        *n = (long)A.size();
    });
}
int demsph_dem_get_pairs(demsph_dem_t h, int which, int* a, int* b, double* sliding, double* rolling, double* torsion,
                         double* force, double* torque) {
    return guarded([&] {
        SCENE_CHECK(h);
        DemScene& s = h->sc;
        std::vector<int> A, B;
        std::vector<size_t> sl;
        collect_rows(s, which, A, B, sl);
        std::vector<double4> S, Rr, T, F, TB;
        if (which >= 2) {
            DemScene::GhostSet& g = *s.ghosts[which - 2];
            if (!A.empty()) {
                if (sliding) g.spS[g.cur].download(S, s.s);
                if (rolling && s.roll) g.spR[g.cur].download(Rr, s.s);
                if (torsion && s.tors) g.spT[g.cur].download(T, s.s);
                if (force) g.pF.download(F, s.s);
                if (torque) g.pTB.download(TB, s.s);
            }
        } else {
            int c = which == 0 ? s.cur : s.wcur;
            if (sliding) (which == 0 ? s.spS[c] : s.wS[c]).download(S, s.s);
            if (rolling && s.roll) (which == 0 ? s.spR[c] : s.wR[c]).download(Rr, s.s);
            if (torsion && s.tors) (which == 0 ? s.spT[c] : s.wT[c]).download(T, s.s);
            if (which == 0 && force) s.pF.download(F, s.s);
            if (which == 0 && torque) s.pTB.download(TB, s.s);
        }
        DEMSPH_CUDA(cudaStreamSynchronize(s.s));
        std::vector<double4> P;
        if (which == 0 && torque) s.pos.download(P, s.s);
        DEMSPH_CUDA(cudaStreamSynchronize(s.s));
        for (size_t k = 0; k < A.size(); k++) {
            if (a) a[k] = A[k];
            if (b) b[k] = B[k];
            if (sliding) st3(sliding, k, xyz(S[sl[k]]));
            if (rolling) st3(rolling, k, s.roll ? xyz(Rr[sl[k]]) : mk3(0, 0, 0));
            if (torsion) st3(torsion, k, s.tors ? xyz(T[sl[k]]) : mk3(0, 0, 0));
            if (force) st3(force, k, which != 1 ? xyz(F[sl[k]]) : mk3(0, 0, 0));
            if (torque) st3(torque, k, which != 1 ? xyz(TB[sl[k]]) : mk3(0, 0, 0));
        }
    });
}
// Sets the springs of the current rows (which = 0: ball-ball pair list,
// 1: ball-triangle candidate rows) from a list keyed by (ball, partner).
static void import_rows(DemScene& s, int which, long n, const int* a, const int* b, const double* sl, const double* ro,
                        const double* to) {
    if (which == 0 && !s.havePairs) throw Status(DEMSPH_ERR_NOT_READY, "no pair list");
    if (which == 1 && !s.haveWallRows) throw Status(DEMSPH_ERR_NOT_READY, "no wall contact rows");
    std::unordered_map<long long, long> idx;
    idx.reserve((size_t)n * 2 + 1);
    for (long k = 0; k < n; k++) idx[((long long)a[k] << 32) | (unsigned)b[k]] = k;
    int N = s.N();
    int c = which == 0 ? s.cur : s.wcur;
    DBuf<int>& CNT = which == 0 ? s.pcnt[c] : s.wcnt[c];
    DBuf<int>& IDS = which == 0 ? s.pj[c] : s.wtj[c];
    DBuf<double4>& BS = which == 0 ? s.spS[c] : s.wS[c];
    DBuf<double4>& BR = which == 0 ? s.spR[c] : s.wR[c];
    DBuf<double4>& BT = which == 0 ? s.spT[c] : s.wT[c];
    std::vector<int> cnt, ids;
    std::vector<double4> S, Rr, T;
    CNT.download(cnt, s.s);
    IDS.download(ids, s.s);
    BS.download(S, s.s);
    if (s.roll) BR.download(Rr, s.s);
    if (s.tors) BT.download(T, s.s);
    DEMSPH_CUDA(cudaStreamSynchronize(s.s));
    for (int A = 0; A < N; A++)
        for (int k = 0; k < cnt[A]; k++) {
            size_t slot = (size_t)k * N + A;
            auto it = idx.find(((long long)A << 32) | (unsigned)ids[slot]);
            if (it == idx.end()) continue;
            S[slot] = d4(ld3(sl, it->second), 0);
            if (s.roll && ro) Rr[slot] = d4(ld3(ro, it->second), 0);
            if (s.tors && to) T[slot] = d4(ld3(to, it->second), 0);
        }
    DEMSPH_CUDA(cudaMemcpyAsync(BS.p, S.data(), S.size() * sizeof(double4), cudaMemcpyHostToDevice, s.s));
    if (s.roll) DEMSPH_CUDA(cudaMemcpyAsync(BR.p, Rr.data(), Rr.size() * sizeof(double4), cudaMemcpyHostToDevice, s.s));
    if (s.tors) DEMSPH_CUDA(cudaMemcpyAsync(BT.p, T.data(), T.size() * sizeof(double4), cudaMemcpyHostToDevice, s.s));
    DEMSPH_CUDA(cudaStreamSynchronize(s.s));
}
int demsph_dem_import_springs(demsph_dem_t h, long n, const int* a, const int* b, const double* sl, const double* ro,
                              const double* to) {
    return guarded([&] {
        SCENE_CHECK(h);
        h->sc.graph.reset();  // kernel arguments or buffers change
        import_rows(h->sc, 0, n, a, b, sl, ro, to);
    });
}
int demsph_dem_import_wall_springs(demsph_dem_t h, long n, const int* ball, const int* tri, const double* sl,
                                   const double* ro, const double* to) {
    return guarded([&] {
        SCENE_CHECK(h);
        h->sc.graph.reset();  // kernel arguments or buffers change
        import_rows(h->sc, 1, n, ball, tri, sl, ro, to);
    });
}
int demsph_dem_copy_members(demsph_dem_t dst, demsph_dem_t src, int count, const int* srcStart, const int* dstStart,
                            const int* num, const int* triDelta, const double* shift) {
    return guarded([&] {
        SCENE_CHECK(dst);
        SCENE_CHECK(src);
        DemScene& d = dst->sc;
        DemScene& s = src->sc;
        if (!d.ready || !s.ready) throw Status(DEMSPH_ERR_NOT_READY, "scenes not initialised");
        if (!s.havePairs || !d.havePairs) throw Status(DEMSPH_ERR_NOT_READY, "scene has no pair list");
        if (d.roll != s.roll || d.tors != s.tors)
            throw Status(DEMSPH_ERR_INVALID, "source and destination differ in rolling / torsion springs");
        if (count < 0 || (count > 0 && (!srcStart || !dstStart || !num || !triDelta || !shift)))
            throw Status(DEMSPH_ERR_INVALID, "missing member tables");
        for (int k = 0; k < count; k++)
            if (num[k] < 0 || srcStart[k] < 0 || dstStart[k] < 0 || srcStart[k] + num[k] > s.N() ||
                dstStart[k] + num[k] > d.N())
                throw Status(DEMSPH_ERR_INVALID, "member range out of bounds");
        // the rows keep their counts, so give the destination at least the source's capacities
        d.grow(s.K, 0, s.haveWallRows ? s.KT : 0);
        // the source's work must be finished before the destination reads it
        DEMSPH_CUDA(cudaStreamSynchronize(s.s));
        d.clear_status();
        DemDev dd = d.dev(false);
        if (!d.haveWallRows || d.hTris.empty()) dd.nTri = 0;
        DemDev sd = s.dev(false);
        if (!s.haveWallRows) sd.wcnt = nullptr;
        for (int k = 0; k < count; k++) {
            if (num[k] == 0) continue;
            k_dem_copy_member<<<grid_for(num[k], 128), 128, 0, d.s>>>(dd, sd, num[k], srcStart[k], dstStart[k],
                                                                     triDelta[k], ld3(shift, k));
            d.launch_count(1);
        }
        DEMSPH_LAUNCH_CHECK();
        DevStatus cs = d.read_status();
        if (cs.bad_index) throw Status(DEMSPH_ERR_INVALID, "a carried pair partner or triangle left its member");
        d.bondPairsStale = true;  // bonds look their pairs up in the carried rows
        // reverse lists for the copied rows
        const int n = d.N();
        DEMSPH_CUDA(cudaMemsetAsync(d.rcnt.p, 0, sizeof(int) * n, d.s));
        DemDev dr = d.dev(false);
        k_dem_reverse<<<grid_for(n, 256), 256, 0, d.s>>>(dr);
        k_dem_reverse_order<<<grid_for(n, 256), 256, 0, d.s>>>(dr);
        d.launch_count(2);
        DevStatus st = d.read_status();
        if (st.overflow) {
            d.grow(0, st.need_rev, 0);
            DEMSPH_CUDA(cudaMemsetAsync(d.rcnt.p, 0, sizeof(int) * n, d.s));
            dr = d.dev(false);
            k_dem_reverse<<<grid_for(n, 256), 256, 0, d.s>>>(dr);
            k_dem_reverse_order<<<grid_for(n, 256), 256, 0, d.s>>>(dr);
            d.launch_count(2);
        }
        DEMSPH_CUDA(cudaStreamSynchronize(d.s));
    });
}
int demsph_dem_copy_member_bodies(demsph_dem_t dst, demsph_dem_t src, int count, const int* srcClump,
                                  const int* dstClump, const int* numClumps, const int* srcBond, const int* dstBond,
                                  const int* numBonds, const double* shift) {
    return guarded([&] {
        SCENE_CHECK(dst);
        SCENE_CHECK(src);
        DemScene& d = dst->sc;
        DemScene& s = src->sc;
        if (!d.ready || !s.ready) throw Status(DEMSPH_ERR_NOT_READY, "scenes not initialised");
        if (count < 0 || (count > 0 && (!srcClump || !dstClump || !numClumps || !srcBond || !dstBond || !numBonds ||
                                        !shift)))
            throw Status(DEMSPH_ERR_INVALID, "missing member tables");
        const long sc = (long)s.hCpos.size(), dc = (long)d.hCpos.size();
        const long sb = (long)s.hBab.size(), db = (long)d.hBab.size();
        for (int k = 0; k < count; k++) {
            if (numClumps[k] < 0 || srcClump[k] < 0 || dstClump[k] < 0 || srcClump[k] + (long)numClumps[k] > sc ||
                dstClump[k] + (long)numClumps[k] > dc)
                throw Status(DEMSPH_ERR_INVALID, "member clump range out of bounds");
            if (numBonds[k] < 0 || srcBond[k] < 0 || dstBond[k] < 0 || srcBond[k] + (long)numBonds[k] > sb ||
                dstBond[k] + (long)numBonds[k] > db)
                throw Status(DEMSPH_ERR_INVALID, "member bond range out of bounds");
            // a carried bond must join the same two member balls on both sides
            for (int j = 0; j < numBonds[k]; j++) {
                const int2 a = s.hBab[srcBond[k] + j], b = d.hBab[dstBond[k] + j];
                if (a.x - s.hBab[srcBond[k]].x != b.x - d.hBab[dstBond[k]].x ||
                    a.y - s.hBab[srcBond[k]].x != b.y - d.hBab[dstBond[k]].x)
                    throw Status(DEMSPH_ERR_INVALID, "carried bonds differ between the scenes");
            }
        }
        DEMSPH_CUDA(cudaStreamSynchronize(s.s));
        d.graph.reset();  // bond pairs are looked up again
        DemDev dd = d.dev(false), sd = s.dev(false);
        for (int k = 0; k < count; k++) {
            const int n = std::max(numClumps[k], numBonds[k]);
            if (n == 0) continue;
            k_dem_copy_bodies<<<grid_for(n, 128), 128, 0, d.s>>>(dd, sd, srcClump[k], dstClump[k], numClumps[k],
                                                                srcBond[k], dstBond[k], numBonds[k], ld3(shift, k));
            d.launch_count(1);
        }
        DEMSPH_LAUNCH_CHECK();
        d.bondPairsStale = true;
        DEMSPH_CUDA(cudaStreamSynchronize(d.s));
    });
}
int demsph_dem_get_bonds(demsph_dem_t h, int* a, int* b, int* ok, double* fn, double* tt, double* fs, double* tb,
                         double* normal, double* point) {
    return guarded([&] {
        SCENE_CHECK(h);
        DemScene& s = h->sc;
        int nb = (int)s.hBab.size();
        if (!s.ready) throw Status(DEMSPH_ERR_NOT_READY, "scene not initialised");
        std::vector<int> OK;
        std::vector<double> FN, TT;
        std::vector<double4> FS, TB, NO, PO;
        s.bok.download(OK, s.s); s.bFn.download(FN, s.s); s.bTt.download(TT, s.s); s.bFs.download(FS, s.s);
        s.bTb.download(TB, s.s); s.bnormal.download(NO, s.s); s.bpoint.download(PO, s.s);
        DEMSPH_CUDA(cudaStreamSynchronize(s.s));
        for (int k = 0; k < nb; k++) {
            if (a) a[k] = s.hBab[k].x;
            if (b) b[k] = s.hBab[k].y;
            if (ok) ok[k] = OK[k];
            if (fn) fn[k] = FN[k];
            if (tt) tt[k] = TT[k];
            if (fs) st3(fs, k, xyz(FS[k]));
            if (tb) st3(tb, k, xyz(TB[k]));
            if (normal) st3(normal, k, xyz(NO[k]));
            if (point) st3(point, k, xyz(PO[k]));
        }
    });
}
struct demsph_dem_snapshot {
    demsph_dem_t scene = nullptr;
    DemScene::Snap snap;
};
int demsph_dem_snapshot(demsph_dem_t h, demsph_dem_snapshot_t* out) {
    return guarded([&] {
        SCENE_CHECK(h);
        if (!out) throw Status(DEMSPH_ERR_INVALID, "null output pointer");
        DemScene& s = h->sc;
        if (!s.ready) throw Status(DEMSPH_ERR_NOT_READY, "scene not initialised");
        if (s.inBlock) throw Status(DEMSPH_ERR_INVALID, "snapshot inside a coupled block");
        auto* sn = new struct demsph_dem_snapshot();
        sn->scene = h;
        try {
            s.take(sn->snap);
            DEMSPH_CUDA(cudaStreamSynchronize(s.s));
        } catch (...) {
            delete sn;
            throw;
        }
        *out = sn;
    });
}
int demsph_dem_restore(demsph_dem_t h, demsph_dem_snapshot_t sn) {
    return guarded([&] {
        SCENE_CHECK(h);
        if (!sn) throw Status(DEMSPH_ERR_INVALID, "null snapshot");
        if (sn->scene != h) throw Status(DEMSPH_ERR_INVALID, "the snapshot belongs to another scene");
        DemScene& s = h->sc;
        if (s.inBlock) throw Status(DEMSPH_ERR_INVALID, "restore inside a coupled block");
        s.restore(sn->snap);
        DEMSPH_CUDA(cudaStreamSynchronize(s.s));
    });
}
int demsph_dem_snapshot_destroy(demsph_dem_snapshot_t sn) {
    return guarded([&] {
        if (!sn) return;
        cudaStream_t st = sn->scene ? sn->scene->sc.s : 0;
        delete sn;
        DEMSPH_CUDA(cudaStreamSynchronize(st));
    });
}
int demsph_dem_diagnostics(demsph_dem_t h, double* out) {
    return guarded([&] {
        SCENE_CHECK(h);
        if (!out) throw Status(DEMSPH_ERR_INVALID, "null output pointer");
        DemScene& s = h->sc;
        if (!s.ready) throw Status(DEMSPH_ERR_NOT_READY, "scene not initialised");
        DemDiagTerm t{s.dev(false)};
        diag_reduce<12>(t, s.N() + (int)s.hCpos.size(), out, s.diagScratch, s.s);
    });
}
int demsph_dem_set_bonds(demsph_dem_t h, long n, const int* ok, const double* fn, const double* tt, const double* fs,
                         const double* tb, const double* normal, const double* point) {
    return guarded([&] {
        SCENE_CHECK(h);
        DemScene& s = h->sc;
        if (!s.ready) throw Status(DEMSPH_ERR_NOT_READY, "scene not initialised");
        const long nb = (long)s.hBab.size();
        if (n != nb) throw Status(DEMSPH_ERR_INVALID, "set_bonds: n must equal the number of bonds");
        if (nb == 0) return;
        s.graph.reset();  // buffers change under captured launches
        if (ok) {
            std::vector<int> v(ok, ok + nb);
            s.bok.upload(v, s.s);
            DEMSPH_CUDA(cudaStreamSynchronize(s.s));
        }
        auto scalars = [&](DBuf<double>& b, const double* src) {
            if (!src) return;
            std::vector<double> v(src, src + nb);
            b.upload(v, s.s);
            DEMSPH_CUDA(cudaStreamSynchronize(s.s));
        };
        auto vectors = [&](DBuf<double4>& b, const double* src) {
            if (!src) return;
            std::vector<double4> v(nb);
            for (long k = 0; k < nb; k++) v[k] = d4(ld3(src, k), 0);
            b.upload(v, s.s);
            DEMSPH_CUDA(cudaStreamSynchronize(s.s));
        };
        scalars(s.bFn, fn);
        scalars(s.bTt, tt);
        vectors(s.bFs, fs);
        vectors(s.bTb, tb);
        vectors(s.bnormal, normal);
        vectors(s.bpoint, point);
    });
}
// ------------------------------------------------------------ VTU frames --
// outputBallVTU, outputMeshWallVTU, outputBallInteractionVTU,
// outputBondedInteractionVTU, outputBallTriangleInteractionVTU
// (DEMSolver.h:908-1370), same files and arrays.  The interaction frames
// evaluate each listed contact on the current state (geometry from the
// current positions, the contact law with a zero time increment on copies of
// the stored springs); the reference writes the values of its last force
// evaluation, half a drift earlier.
static void ball_arrays(DemScene& s, std::vector<double4>& P, std::vector<double4>& V, std::vector<double4>& W,
                        std::vector<int>& M, std::vector<int>& Cl) {
    if (!s.ready && !s.assembled) {
        P = s.hPos; V = s.hVel; W = s.hAngv; M = s.hMat; Cl = s.hClump;
        return;
    }
    s.pos.download(P, s.s); s.vel.download(V, s.s); s.angv.download(W, s.s);
    s.mat.download(M, s.s); s.clump.download(Cl, s.s);
    DEMSPH_CUDA(cudaStreamSynchronize(s.s));
}
static std::vector<double3> xyz_of(const std::vector<double4>& a) {
    std::vector<double3> o(a.size());
    for (size_t i = 0; i < a.size(); i++) o[i] = xyz(a[i]);
    return o;
}
int demsph_dem_write_vtu(demsph_dem_t h, const char* dir, long frame, int what) {
    return guarded([&] {
        SCENE_CHECK(h);
        if (!dir) throw Status(DEMSPH_ERR_INVALID, "null directory");
        DemScene& s = h->sc;
        const std::string d(dir);
        const int n = s.N();
        std::vector<double4> P, V, W;
        std::vector<int> M, Cl;
        ball_arrays(s, P, V, W, M, Cl);
        if (what & DEMSPH_VTU_BALLS) {
            vtu::File f(d, "ball", frame);
            f.head(s.time, s.iStep, n, n);
            f.points(xyz_of(P));
            f.vertex_cells(n);
            f.begin_data("PointData", "radius");
            std::vector<double> r(n);
            for (int i = 0; i < n; i++) r[i] = P[i].w;
            f.floats("radius", r);
            f.ints("materialID", M);
            f.ints("clumpID", Cl);
            f.vectors("velocity", xyz_of(V));
            f.vectors("angularVelocity", xyz_of(W));
            f.end_data("PointData");
        }
        if ((what & DEMSPH_VTU_MESH_WALLS) && !s.hTris.empty()) {
            std::vector<double4> VG;
            if (s.ready) {
                s.vglobal.download(VG, s.s);
                DEMSPH_CUDA(cudaStreamSynchronize(s.s));
            } else {
                VG.resize(s.hVlocal.size());
                for (size_t v = 0; v < s.hVlocal.size(); v++)
                    VG[v] = d4(xyz(s.hVlocal[v]) + xyz(s.hWpos[s.hVwall[v]]), 0);
            }
            vtu::File f(d, "triangleWall", frame);
            f.head(s.time, s.iStep, VG.size(), s.hTris.size());
            f.points(xyz_of(VG));
            f.triangle_cells(s.hTris);
            f.begin_data("CellData", "materialID");
            std::vector<int> wid(s.hTris.size()), tm(s.hTris.size());
            for (size_t t = 0; t < s.hTris.size(); t++) {
                wid[t] = s.hTris[t].w;
                tm[t] = s.hWmat[s.hTris[t].w];
            }
            f.ints("wallID", wid);
            f.ints("materialID", tm);
            f.end_data("CellData");
        }
        auto contact_frame = [&](int which, const char* stem) {
            std::vector<int> A, B;
            std::vector<size_t> sl;
            if (s.ready) collect_rows(s, which, A, B, sl);
            std::vector<double4> S, R, T, VG;
            const int c = which == 0 ? s.cur : s.wcur;
            if (!A.empty()) {
                (which == 0 ? s.spS[c] : s.wS[c]).download(S, s.s);
                if (s.roll) (which == 0 ? s.spR[c] : s.wR[c]).download(R, s.s);
                if (s.tors) (which == 0 ? s.spT[c] : s.wT[c]).download(T, s.s);
                if (which == 1) s.vglobal.download(VG, s.s);
                DEMSPH_CUDA(cudaStreamSynchronize(s.s));
            }
            const size_t m = A.size();
            std::vector<double3> pt(m), nrm(m), fc(m), tc(m), es(m), er(m), et(m);
            std::vector<double> ov(m);
            for (size_t k = 0; k < m; k++) {
                const int a = A[k];
                const double3 ra = xyz(P[a]);
                es[k] = xyz(S[sl[k]]);
                er[k] = s.roll ? xyz(R[sl[k]]) : mk3(0, 0, 0);
                et[k] = s.tors ? xyz(T[sl[k]]) : mk3(0, 0, 0);
                double3 rc, n, vc, wij;
                double delta, mass, Rad;
                int mb;
                if (which == 0) {
                    const int b = B[k];
                    const double3 rb = xyz(P[b]);
                    n = normalize(ra - rb);
                    delta = P[a].w + P[b].w - len(ra - rb);
                    rc = rb + (P[b].w - 0.5 * delta) * n;
                    vc = xyz(V[a]) + cross(xyz(W[a]), rc - ra) - (xyz(V[b]) + cross(xyz(W[b]), rc - rb));
                    wij = xyz(W[a]) - xyz(W[b]);
                    mass = 1. / (V[a].w + V[b].w);
                    Rad = P[a].w * P[b].w / (P[a].w + P[b].w);
                    mb = M[b];
                } else {
                    const int4 tv = s.hTris[B[k]];
                    rc = mk3(0, 0, 0);
                    classify_sphere_triangle(ra, P[a].w, xyz(VG[tv.x]), xyz(VG[tv.y]), xyz(VG[tv.z]), rc);
                    n = normalize(ra - rc);
                    delta = P[a].w - len(ra - rc);
                    const int wj = tv.w;
                    const double3 rw = xyz(s.hWpos[wj]);
                    vc = xyz(V[a]) + cross(xyz(W[a]), rc - ra) - (xyz(s.hWvel[wj]) + cross(xyz(s.hWangv[wj]), rc - rw));
                    wij = xyz(W[a]) - xyz(s.hWangv[wj]);
                    mass = V[a].w > 0 ? 1. / V[a].w : 0.0;
                    Rad = P[a].w;
                    mb = s.hWmat[wj];
                }
                pt[k] = rc;
                nrm[k] = n;
                ov[k] = delta;
                double3 F = mk3(0, 0, 0), Tq = mk3(0, 0, 0);
                if (delta > 0 && s.cap > 0 && mass > 0) {
                    double3 s0 = es[k], r0 = er[k], t0 = et[k];
                    const MatPair& mp = s.hMatTab[pair_param_index(M[a], mb, s.nMat, s.cap)];
                    contact_law<double>(mp, F, Tq, s0, r0, t0, vc, wij, n, delta, mass, Rad, 0.0, s.roll, s.tors);
                }
                fc[k] = F;
                tc[k] = Tq;
            }
            vtu::File f(d, stem, frame);
            f.head(s.time, s.iStep, m, m);
            f.points(pt);
            f.vertex_cells(m);
            f.begin_data("PointData", "overlap");
            f.floats("overlap", ov);
            f.vectors("contact normal", nrm);
            f.vectors("contact force", fc);
            f.vectors("contact torque", tc);
            f.vectors("sliding spring", es);
            f.vectors("rolling spring", er);
            f.vectors("torsion spring", et);
            f.end_data("PointData");
        };
        if (what & DEMSPH_VTU_BALL_INTERACTIONS) contact_frame(0, "ballInteraction");
        if ((what & DEMSPH_VTU_BALL_TRIANGLE_INTERACTIONS) && !s.hTris.empty())
            contact_frame(1, "ballTriangleInteraction");
        if (what & DEMSPH_VTU_BONDED_INTERACTIONS) {
            const int nb = (int)s.hBab.size();
            std::vector<int> OK(nb, 1);
            std::vector<double> FN(nb, 0.0), TT(nb, 0.0), SM(nb, 0.0), TM(nb, 0.0);
            std::vector<double4> FS(nb), TB(nb), NO(s.hBnormal), PO(s.hBpoint);
            if (s.ready && nb > 0) {
                s.bok.download(OK, s.s); s.bFn.download(FN, s.s); s.bTt.download(TT, s.s); s.bFs.download(FS, s.s);
                s.bTb.download(TB, s.s); s.bnormal.download(NO, s.s); s.bpoint.download(PO, s.s);
                s.bsmax.download(SM, s.s); s.btmax.download(TM, s.s);
                DEMSPH_CUDA(cudaStreamSynchronize(s.s));
            } else {
                for (int k = 0; k < nb; k++) FS[k] = TB[k] = make_double4(0, 0, 0, 0);
            }
            vtu::File f(d, "bondedInteraction", frame);
            f.head(s.time, s.iStep, nb, nb);
            f.points(xyz_of(PO));
            f.vertex_cells(nb);
            f.begin_data("PointData", "overlap");
            f.ints("is bonded", OK);
            f.floats("normal force", FN);
            f.floats("torsion torque", TT);
            f.floats("maximum normal stress", SM);
            f.floats("maximum shear stress", TM);
            f.vectors("contact normal", xyz_of(NO));
            f.vectors("shearing force", xyz_of(FS));
            f.vectors("bending torque", xyz_of(TB));
            f.end_data("PointData");
        }
    });
}
int demsph_dem_get_clumps(demsph_dem_t h, double* pos, double* vel, double* w, double* q) {
    return guarded([&] {
        SCENE_CHECK(h);
        DemScene& s = h->sc;
        if (!s.ready) throw Status(DEMSPH_ERR_NOT_READY, "scene not initialised");
        std::vector<double4> P, Vv, W, Q;
        s.cpos.download(P, s.s); s.cvel.download(Vv, s.s); s.cangv.download(W, s.s); s.cq.download(Q, s.s);
        DEMSPH_CUDA(cudaStreamSynchronize(s.s));
        for (size_t c = 0; c < P.size(); c++) {
            if (pos) st3(pos, c, xyz(P[c]));
            if (vel) st3(vel, c, xyz(Vv[c]));
            if (w) st3(w, c, xyz(W[c]));
            if (q) { q[4 * c] = Q[c].x; q[4 * c + 1] = Q[c].y; q[4 * c + 2] = Q[c].z; q[4 * c + 3] = Q[c].w; }
        }
    });
}
int demsph_dem_get_walls(demsph_dem_t h, double* pos, double* q, double* vglobal) {
    return guarded([&] {
        SCENE_CHECK(h);
        DemScene& s = h->sc;
        if (!s.ready) throw Status(DEMSPH_ERR_NOT_READY, "scene not initialised");
        std::vector<double4> P, Q, VG;
        s.wpos.download(P, s.s); s.wq.download(Q, s.s); s.vglobal.download(VG, s.s);
        DEMSPH_CUDA(cudaStreamSynchronize(s.s));
        for (size_t c = 0; c < P.size(); c++) {
            if (pos) st3(pos, c, xyz(P[c]));
            if (q) { q[4 * c] = Q[c].x; q[4 * c + 1] = Q[c].y; q[4 * c + 2] = Q[c].z; q[4 * c + 3] = Q[c].w; }
        }
        if (vglobal) for (size_t v = 0; v < VG.size(); v++) st3(vglobal, v, xyz(VG[v]));
    });
}

}  // extern "C"
