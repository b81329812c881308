// demsph_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// FP64 CPU restatement of the DEMSPH per-step particle-interaction path
// (DEMSPH/kernel in kaiqideng/this_studio).  It exists to check the CUDA
// library, never to stand in for it: only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg may load it.
//
// Every function cites the reference file:line it restates.  Arithmetic is
// IEEE double, evaluated in the same order as the reference device code,
// except that normalize() uses 1/sqrt where the device code uses rsqrt
// (DEMSPH/kernel/myUtility/myVec.h:119-125) and that FP64 atomics become
// sequential adds in bond order (DEMSPH/kernel/contactKernel.cu:644-650).
//
// Reference quirks (the oracle follows the corrected form; each is listed so
// a reader can map behaviour back to the reference):
//   Q1 sumClumpForceTorqueKernel reads force_c[i] with a pebble index
//      (ballIntegrationKernel.cu:20): an out-of-bounds read, undefined, so the
//      oracle sums pebble forces force_p[i] as the kernel clearly intends.
//   Q2 addTriangleContactForceTorque(dt) runs twice per step and drifts the
//      wall by a full dt each time (DEMSolver.h:556-564,1463,1469): kept.
//   Q5 SPH viscosity uses r_hat.gradW without 1/r (WCSPHIntegrationKernel.cu:
//      108,144): kept.
//   Q6 pebble positions are drifted with their velocity, never re-placed from
//      the clump quaternion (ballIntegrationKernel.cu:81-99): kept.
//   Q7 objectPointing::interactionStart/End are set to -1 only at allocation
//      (interaction.h:212-221) and never reset before a rebuild
//      (DEMSolver.h:59-78), so an object that loses all incoming pairs keeps a
//      stale range.  The oracle resets them to -1 before every rebuild.
//   Q8 addMeshWall ignores its velocity / angularVelocity arguments
//      (DEMSolver.h:1901-1911): kept; oracle_dem_set_wall_motion sets them.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <unordered_set>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace ora {

// ---------------------------------------------------------------- vectors --
// myVec.h:25-128
struct V3 { double x, y, z; };
static inline V3 v3(double x, double y, double z) { return V3{x, y, z}; }
static inline V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 operator*(V3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
static inline V3 operator*(double s, V3 a) { return v3(a.x * s, a.y * s, a.z * s); }
static inline V3 operator/(V3 a, double s) { double inv = 1.0 / s; return v3(a.x * inv, a.y * inv, a.z * inv); }
static inline V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
static inline V3& operator+=(V3& a, V3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
static inline V3& operator-=(V3& a, V3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; return a; }
static inline V3& operator*=(V3& a, double s) { a.x *= s; a.y *= s; a.z *= s; return a; }
static inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 cross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline double lengthSquared(V3 v) { return v.x * v.x + v.y * v.y + v.z * v.z; }
static inline double length(V3 v) { return std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }
static inline V3 normalize(V3 v) {
    double l2 = v.x * v.x + v.y * v.y + v.z * v.z;
    if (l2 < 1.0e-20) return v3(0, 0, 0);
    double inv = 1.0 / std::sqrt(l2);
    return v3(v.x * inv, v.y * inv, v.z * inv);
}
static const double PI = 3.14159265358979323846;

// Rodrigues rotation, myVec.h:134-176
static inline V3 rotateVector(V3 v, V3 ang) {
    double a2 = dot(ang, ang);
    if (a2 < 1.0e-20) return v;
    double a = std::sqrt(a2);
    double s = std::sin(a), c = std::cos(a);
    double inv = 1.0 / a;
    V3 k = v3(ang.x * inv, ang.y * inv, ang.z * inv);
    double kv = k.x * v.x + k.y * v.y + k.z * v.z;
    V3 kxv = v3(k.y * v.z - k.z * v.y, k.z * v.x - k.x * v.z, k.x * v.y - k.y * v.x);
    double t3 = kv * (1.0 - c);
    return v3(v.x * c + kxv.x * s + k.x * t3, v.y * c + kxv.y * s + k.y * t3, v.z * c + kxv.z * s + k.z * t3);
}

// ------------------------------------------------------------ quaternions --
struct Quat { double q0, q1, q2, q3; };
// myQua.h:51-62
static inline Quat qnormalize(Quat q) {
    double l2 = q.q0 * q.q0 + q.q1 * q.q1 + q.q2 * q.q2 + q.q3 * q.q3;
    if (l2 < 1.0e-20) return q;
    double inv = 1.0 / std::sqrt(l2);
    return Quat{q.q0 * inv, q.q1 * inv, q.q2 * inv, q.q3 * inv};
}
// myQua.h:77-92: q <- normalize(q + q (x) (0, w dt/2))
static inline Quat quaternionRotate(Quat q, V3 w, double dt) {
    V3 v = w * (0.5 * dt);
    Quat d;
    d.q0 = -q.q1 * v.x - q.q2 * v.y - q.q3 * v.z;
    d.q1 = q.q0 * v.x + q.q3 * v.y - q.q2 * v.z;
    d.q2 = -q.q3 * v.x + q.q0 * v.y + q.q1 * v.z;
    d.q3 = q.q2 * v.x - q.q1 * v.y + q.q0 * v.z;
    return qnormalize(Quat{q.q0 + d.q0, q.q1 + d.q1, q.q2 + d.q2, q.q3 + d.q3});
}
// myQua.h:103-113
static inline V3 rotateVectorByQuaternion(Quat q, V3 v) {
    V3 qv = v3(q.q1, q.q2, q.q3);
    V3 t = cross(qv, v) * 2.0;
    return v + (t * q.q0) + cross(qv, t);
}

// ------------------------------------------------------- symmetric 3x3 ---
struct SymM { double xx, yy, zz, xy, xz, yz; };
static inline V3 operator*(SymM m, V3 v) {
    return v3(m.xx * v.x + m.xy * v.y + m.xz * v.z, m.xy * v.x + m.yy * v.y + m.yz * v.z,
              m.xz * v.x + m.yz * v.y + m.zz * v.z);
}
// myMat.h:107-158: R invI R^T
static inline SymM rotateInverseInertiaTensor(Quat q, SymM I) {
    double q0 = q.q0, q1 = q.q1, q2 = q.q2, q3 = q.q3;
    double q11 = 2 * q1 * q1, q22 = 2 * q2 * q2, q33 = 2 * q3 * q3;
    double a = 1.0 - q22 - q33, b = 2 * (q1 * q2 - q0 * q3), c = 2 * (q1 * q3 + q0 * q2);
    double d = 2 * (q1 * q2 + q0 * q3), e = 1.0 - q11 - q33, f = 2 * (q2 * q3 - q0 * q1);
    double g = 2 * (q1 * q3 - q0 * q2), h = 2 * (q2 * q3 + q0 * q1), i = 1.0 - q11 - q22;
    double r0x = I.xx * a + I.xy * b + I.xz * c, r0y = I.xy * a + I.yy * b + I.yz * c, r0z = I.xz * a + I.yz * b + I.zz * c;
    double r1x = I.xx * d + I.xy * e + I.xz * f, r1y = I.xy * d + I.yy * e + I.yz * f, r1z = I.xz * d + I.yz * e + I.zz * f;
    double r2x = I.xx * g + I.xy * h + I.xz * i, r2y = I.xy * g + I.yy * h + I.yz * i, r2z = I.xz * g + I.yz * h + I.zz * i;
    return SymM{r0x * a + r0y * b + r0z * c, r1x * d + r1y * e + r1z * f, r2x * g + r2y * h + r2z * i,
                r0x * d + r0y * e + r0z * f, r0x * g + r0y * h + r0z * i, r1x * g + r1y * h + r1z * i};
}
// myMat.h:163-179
static inline SymM inverse(SymM A) {
    double di = 1.0 / (A.xx * (A.yy * A.zz - A.yz * A.yz) + A.xy * (A.yz * A.xz - A.xy * A.zz) +
                       A.xz * (A.xy * A.yz - A.yy * A.xz));
    return SymM{(A.yy * A.zz - A.yz * A.yz) * di, (A.xx * A.zz - A.xz * A.xz) * di, (A.xx * A.yy - A.xy * A.xy) * di,
                -(A.xy * A.zz - A.xz * A.yz) * di, (A.xy * A.yz - A.xz * A.yy) * di, -(A.xx * A.yz - A.xz * A.xy) * di};
}

// wallIntegrationKernel.cuh:4-29
static inline V3 triangleCircumcenter(V3 a, V3 b, V3 c) {
    V3 ab = b - a, ac = c - a;
    V3 n = cross(ab, ac);
    double n2 = dot(n, n);
    if (n2 < 1e-30) return (a + b + c) / 3.0;
    V3 t1 = cross(n, ab) * dot(ac, ac);
    V3 t2 = cross(ac, n) * dot(ab, ab);
    double inv = 1.0 / (2.0 * n2);
    return a + (t1 + t2) * inv;
}

// ------------------------------------------------------ material tables ---
// contactParameters.h:62-100 (param-major packing) and :123-141 (pair index)
enum { H_E = 0, H_G, H_RES, H_KRKS, H_KTKS, H_MUS, H_MUR, H_MUT, H_COUNT };
enum { L_KN = 0, L_KS, L_KR, L_KT, L_DN, L_DS, L_DR, L_DT, L_MUS, L_MUR, L_MUT, L_COUNT };
enum { B_GAMMA = 0, B_E, B_KNKS, B_SIGMA, B_C, B_MU, B_COUNT };

struct Row { int a, b; double v[11]; };

static inline int pairParamIndex(int a, int b, int nMat, int cap) {
    if (nMat <= 0 || cap <= 0) return 0;
    if (a < 0 || b < 0 || a >= nMat || b >= nMat) return cap - 1;
    int i = a, j = b;
    if (i > j) std::swap(i, j);
    long long idx = ((long long)i * (2LL * nMat - i + 1LL)) / 2LL + (long long)(j - i);
    if (idx < 0) idx = 0;
    if (idx >= cap) idx = cap - 1;
    return (int)idx;
}

struct Materials {
    std::vector<Row> hrows, lrows, brows;
    int nMat = 0, cap = 0;
    std::vector<double> H, L, B;
    // contactKernel.cu:6-104 (buildFromTables)
    void build() {
        int mx = -1;
        for (auto& r : hrows) mx = std::max(mx, std::max(r.a, r.b));
        for (auto& r : lrows) mx = std::max(mx, std::max(r.a, r.b));
        for (auto& r : brows) mx = std::max(mx, std::max(r.a, r.b));
        nMat = mx < 0 ? 0 : mx + 1;
        if (nMat <= 0) { cap = 0; return; }
        cap = nMat * (nMat + 1) / 2 + 1;
        H.assign((size_t)H_COUNT * cap, 0.0);
        L.assign((size_t)L_COUNT * cap, 0.0);
        B.assign((size_t)B_COUNT * cap, 0.0);
        for (int i = 0; i < cap; i++) H[(size_t)H_RES * cap + i] = 1.0;
        for (int i = 0; i < cap; i++) { B[(size_t)B_GAMMA * cap + i] = 1.0; B[(size_t)B_KNKS * cap + i] = 1.0; }
        for (auto& r : hrows) { int ip = pairParamIndex(r.a, r.b, nMat, cap); for (int p = 0; p < H_COUNT; p++) H[(size_t)p * cap + ip] = r.v[p]; }
        for (auto& r : lrows) { int ip = pairParamIndex(r.a, r.b, nMat, cap); for (int p = 0; p < L_COUNT; p++) L[(size_t)p * cap + ip] = r.v[p]; }
        for (auto& r : brows) { int ip = pairParamIndex(r.a, r.b, nMat, cap); for (int p = 0; p < B_COUNT; p++) B[(size_t)p * cap + ip] = r.v[p]; }
    }
    int index(int a, int b) const { return pairParamIndex(a, b, nMat, cap); }
    // The reference reads through a null table when no row was ever set; the
    // oracle returns zeros then (reads of an unset table never happen in a
    // valid scene).
    double h(int ip, int p) const { return cap ? H[(size_t)p * cap + ip] : (p == H_RES ? 1.0 : 0.0); }
    double l(int ip, int p) const { return cap ? L[(size_t)p * cap + ip] : 0.0; }
    double b(int ip, int p) const { return cap ? B[(size_t)p * cap + ip] : ((p == B_GAMMA || p == B_KNKS) ? 1.0 : 0.0); }
};

// ------------------------------------------------------------ spatial grid -
struct I3 { int x, y, z; };
struct Grid {
    V3 mn{0, 0, 0}, mx{0, 0, 0}, cs{0, 0, 0};
    I3 n{0, 0, 0};
    bool valid = false;
    std::vector<int> start, end;
    size_t ncell() const { return (size_t)n.x * (size_t)n.y * (size_t)n.z; }
};
// boundary.h:70-94
static void gridSet(Grid& g, V3 mn, V3 mx, double cell) {
    if (mx.x <= mn.x || mx.y <= mn.y || mx.z <= mn.z || cell < 1.e-20) return;
    g.mn = mn; g.mx = mx;
    V3 d = mx - mn;
    g.n.x = d.x > cell ? int(d.x / cell) : 1;
    g.n.y = d.y > cell ? int(d.y / cell) : 1;
    g.n.z = d.z > cell ? int(d.z / cell) : 1;
    g.cs = v3(d.x / double(g.n.x), d.y / double(g.n.y), d.z / double(g.n.z));
    g.valid = true;
    g.start.assign(g.ncell(), -1);
    g.end.assign(g.ncell(), -1);
}
// neighborSearchKernel.cuh:4-14
static inline I3 gridPosition(V3 p, const Grid& g) {
    return I3{int((p.x - g.mn.x) / g.cs.x), int((p.y - g.mn.y) / g.cs.y), int((p.z - g.mn.z) / g.cs.z)};
}
static inline int hashOf(I3 q, const Grid& g) { return q.z * g.n.y * g.n.x + q.y * g.n.x + q.x; }
// neighborSearchKernel.cu:6-27 (clamped key)
static inline int clampedHash(V3 p, const Grid& g) {
    if (p.x < g.mn.x) p.x = g.mn.x; else if (p.x >= g.mx.x) p.x = g.mx.x - 0.5 * g.cs.x;
    if (p.y < g.mn.y) p.y = g.mn.y; else if (p.y >= g.mx.y) p.y = g.mx.y - 0.5 * g.cs.y;
    if (p.z < g.mn.z) p.z = g.mn.z; else if (p.z >= g.mx.z) p.z = g.mx.z - 0.5 * g.cs.z;
    return hashOf(gridPosition(p, g), g);
}
// Stable (key, index) sort + cell start/end:
// neighborSearchKernel.cu:79-106 and buildHashStartEnd.cu:6-83.
static void buildCellTable(Grid& g, const std::vector<V3>& p, std::vector<int>& hashIndex, std::vector<int>& hashValue) {
    size_t n = p.size();
    hashValue.resize(n);
    hashIndex.resize(n);
    for (size_t i = 0; i < n; i++) hashValue[i] = clampedHash(p[i], g);
    std::iota(hashIndex.begin(), hashIndex.end(), 0);
    std::stable_sort(hashIndex.begin(), hashIndex.end(), [&](int a, int b) { return hashValue[a] < hashValue[b]; });
    std::vector<int> sortedKey(n);
    for (size_t i = 0; i < n; i++) sortedKey[i] = hashValue[hashIndex[i]];
    hashValue.swap(sortedKey);  // the reference sorts hashValue in place
    std::fill(g.start.begin(), g.start.end(), -1);
    std::fill(g.end.begin(), g.end.end(), -1);
    for (size_t i = 0; i < n; i++) {
        int h = hashValue[i];
        if (h < 0 || (size_t)h >= g.ncell()) continue;
        if (i == 0 || hashValue[i - 1] != h) g.start[h] = (int)i;
        if (i == n - 1 || hashValue[i + 1] != h) g.end[h] = (int)(i + 1);
    }
}
// The 27-cell walk with the reference's cell clamping (ballNeighborSearchKernel.cu:25-46).
template <class F>
static inline void forEachStencilCell(V3 p, const Grid& g, F&& f) {
    I3 q = gridPosition(p, g);
    I3 s{-1, -1, -1}, e{1, 1, 1};
    if (q.x <= 0) { q.x = 0; s.x = 0; }
    if (q.x >= g.n.x - 1) { q.x = g.n.x - 1; e.x = 0; }
    if (q.y <= 0) { q.y = 0; s.y = 0; }
    if (q.y >= g.n.y - 1) { q.y = g.n.y - 1; e.y = 0; }
    if (q.z <= 0) { q.z = 0; s.z = 0; }
    if (q.z >= g.n.z - 1) { q.z = g.n.z - 1; e.z = 0; }
    for (int zz = s.z; zz <= e.z; zz++)
        for (int yy = s.y; yy <= e.y; yy++)
            for (int xx = s.x; xx <= e.x; xx++) {
                int h = hashOf(I3{q.x + xx, q.y + yy, q.z + zz}, g);
                int st = g.start[h];
                if (st == -1) continue;
                f(st, g.end[h]);
            }
}

// -------------------------------------------------------------- contact ---
// contactKernel.cuh:64-97
static inline V3 integrateSlidingOrRollingSpring(V3 sp, V3 sv, V3 n, V3 Fn, double mu, double k, double c, double dt) {
    V3 s = v3(0, 0, 0);
    if (k > 0.) {
        V3 s1 = sp - dot(sp, n) * n;
        double a1 = length(s1);
        if (a1 > 1.e-10) s1 *= length(sp) / a1;
        s = s1 + sv * dt;
        if (mu > 0.) {
            V3 fs = -k * s - c * sv;
            double af = length(fs), an = length(Fn);
            if (af > mu * an) {
                double ratio = mu * an / af;
                fs *= ratio;
                s = -(fs + c * sv) / k;
            }
        }
    }
    return s;
}
// contactKernel.cuh:99-126
static inline V3 integrateTorsionSpring(V3 sp, V3 tv, V3 n, V3 Fn, double mu, double k, double c, double dt) {
    V3 s = v3(0, 0, 0);
    if (k > 0.) {
        s = dot(sp + tv * dt, n) * n;
        if (mu > 0.) {
            V3 fs = -k * s - c * tv;
            double af = length(fs), an = length(Fn);
            if (af > mu * an) {
                double ratio = mu * an / af;
                fs *= ratio;
                s = -(fs + c * tv) / k;
            }
        }
    }
    return s;
}
// Shared tail of LinearContact / HertzianMindlinContact (contactKernel.cuh:128-290).
static inline void contactLaw(V3& F, V3& T, V3& es, V3& er, V3& et, V3 vc, V3 wij, V3 n, double delta, double m, double R,
                              double dt, double kn, double ks, double kr, double kt, double cn, double cs, double cr,
                              double ct, double mus, double mur, double mut) {
    V3 vn = dot(vc, n) * n;
    V3 Fn = kn * delta * n - vn * cn;
    V3 vs = vc - vn;
    es = integrateSlidingOrRollingSpring(es, vs, n, Fn, mus, ks, cs, dt);
    V3 Fs = -ks * es - cs * vs;
    V3 vr = -R * cross(n, wij);
    er = integrateSlidingOrRollingSpring(er, vr, n, Fn, mur, kr, cr, dt);
    V3 Fr = -kr * er - cr * vr;
    V3 Tr = R * cross(n, Fr);
    double D2 = 2 * R;
    V3 vt = D2 * dot(wij, n) * n;
    et = integrateTorsionSpring(et, vt, n, Fn, mut, kt, ct, dt);
    V3 Ft = -kt * et - ct * vt;
    V3 Tt = D2 * Ft;
    F = Fn + Fs;
    T = Tr + Tt;
}
// calBallContactForceTorqueKernel body (contactKernel.cu:218-252) selecting
// LinearContact (contactKernel.cuh:128-207) or HertzianMindlinContact (:209-290).
static inline void pairLaw(const Materials& M, int ip, V3& F, V3& T, V3& es, V3& er, V3& et, V3 vc, V3 wij, V3 n,
                           double delta, double m, double R, double dt) {
    F = v3(0, 0, 0);
    T = v3(0, 0, 0);
    double kn = M.l(ip, L_KN);
    if (kn > 1.e-20) {
        if (delta > 0) {
            double ks = M.l(ip, L_KS), kr = M.l(ip, L_KR), kt = M.l(ip, L_KT);
            double dn = M.l(ip, L_DN), ds = M.l(ip, L_DS), dr = M.l(ip, L_DR), dtt = M.l(ip, L_DT);
            double cn = 2. * dn * std::sqrt(m * kn), cs = 2. * ds * std::sqrt(m * ks);
            double cr = 2. * dr * std::sqrt(m * kr), ct = 2. * dtt * std::sqrt(m * kt);
            contactLaw(F, T, es, er, et, vc, wij, n, delta, m, R, dt, kn, ks, kr, kt, cn, cs, cr, ct, M.l(ip, L_MUS),
                       M.l(ip, L_MUR), M.l(ip, L_MUT));
        } else {
            es = er = et = v3(0, 0, 0);
        }
    } else {
        double logR = std::log(M.h(ip, H_RES));
        double D = -logR / std::sqrt(logR * logR + PI * PI);
        if (delta > 0) {
            double E = M.h(ip, H_E), G = M.h(ip, H_G);
            double kn2 = 4. / 3. * E * std::sqrt(R * delta);
            double ks = 8. * G * std::sqrt(R * delta);
            double s56 = std::sqrt(5. / 6.);
            double cn = 2. * s56 * D * std::sqrt(m * kn2);
            double cs = 2. * s56 * D * std::sqrt(m * ks);
            double kr = ks * M.h(ip, H_KRKS), kt = ks * M.h(ip, H_KTKS);
            double cr = 2. * s56 * D * std::sqrt(m * kr);
            double ct = 2. * s56 * D * std::sqrt(m * kt);
            contactLaw(F, T, es, er, et, vc, wij, n, delta, m, R, dt, kn2, ks, kr, kt, cn, cs, cr, ct, M.h(ip, H_MUS),
                       M.h(ip, H_MUR), M.h(ip, H_MUT));
        } else {
            es = er = et = v3(0, 0, 0);
        }
    }
}

// contactKernel.cuh:4-62
static inline int parallelBondedContact(double& Fn, double& Tt, V3& Fs, V3& Tb, double& smax, double& tmax, V3 n0, V3 n,
                                        V3 vc, V3 wA, V3 wB, double rA, double rB, double dt, double gamma, double Eb,
                                        double knks, double sigma, double C, double mu) {
    V3 th1 = cross(n0, n);
    Fs = rotateVector(Fs, th1);
    Tb = rotateVector(Tb, th1);
    V3 th2 = dot(0.5 * (wA + wB) * dt, n) * n;
    Fs = rotateVector(Fs, th2);
    Tb = rotateVector(Tb, th2);
    double rmin = rA < rB ? rA : rB;
    double Rb = gamma * rmin;
    double A = Rb * Rb * PI;
    double I = Rb * Rb * Rb * Rb / 4. * PI;
    double J = 2 * I;
    double knA = Eb / (rA + rB);
    double ksA = knA / knks;
    V3 dn = dot(vc, n) * n * dt;
    V3 dtr = vc * dt - dn;
    Fn -= dot(dn * knA * A, n);
    Fs -= dtr * ksA * A;
    V3 wr = wA - wB;
    V3 rn = dot(wr, n) * n * dt;
    V3 rt = wr * dt - rn;
    Tt -= dot(rn * ksA * J, n);
    Tb -= rt * knA * I;
    smax = -Fn / A + length(Tb) / I * Rb;
    tmax = length(Fs) / A + std::fabs(Tt) / J * Rb;
    int ok = 1;
    if (sigma > 0 && smax > sigma) ok = 0;
    else if (C > 0 && tmax > C - mu * smax) ok = 0;
    return ok;
}

// -------------------------------------------------- sphere vs triangle ---
enum { CT_NONE = 0, CT_FACE, CT_EDGE, CT_VERTEX };
static inline double clamp01(double x) { return x < 0.0 ? 0.0 : (x > 1.0 ? 1.0 : x); }
static inline double dist2(V3 a, V3 b) { V3 d = a - b; return dot(d, d); }
// contactKernel.cuh:315-330
static inline V3 closestPointOnSegment(V3 a, V3 b, V3 p, double& t) {
    V3 ab = b - a;
    double ab2 = dot(ab, ab);
    if (ab2 <= 1e-30) { t = 0.0; return a; }
    t = clamp01(dot(p - a, ab) / ab2);
    return a + ab * t;
}
// contactKernel.cuh:367-501
static inline int classifySphereTriangle(V3 c, double r, V3 v0, V3 v1, V3 v2, V3& cp) {
    double r2 = r * r;
    double eps2 = 1e-12 * std::fmax(1.0, r2);
    V3 ab = v1 - v0, ac = v2 - v0;
    V3 n = cross(ab, ac);
    double area2 = dot(n, n);
    if (area2 <= 1e-20) {
        double t01, t02, t12;
        V3 q01 = closestPointOnSegment(v0, v1, c, t01);
        V3 q02 = closestPointOnSegment(v0, v2, c, t02);
        V3 q12 = closestPointOnSegment(v1, v2, c, t12);
        double dmin = dist2(c, q01);
        cp = q01;
        int type = (t01 > 0.0 && t01 < 1.0) ? CT_EDGE : CT_VERTEX;
        double d02 = dist2(c, q02);
        if (d02 < dmin) { dmin = d02; cp = q02; type = (t02 > 0.0 && t02 < 1.0) ? CT_EDGE : CT_VERTEX; }
        double d12 = dist2(c, q12);
        if (d12 < dmin) { dmin = d12; cp = q12; type = (t12 > 0.0 && t12 < 1.0) ? CT_EDGE : CT_VERTEX; }
        return (dmin <= r2 + eps2) ? type : CT_NONE;
    }
    V3 ap = c - v0;
    double d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) { cp = v0; return dist2(c, v0) <= r2 + eps2 ? CT_VERTEX : CT_NONE; }
    V3 bp = c - v1;
    double d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0 && d4 <= d3) { cp = v1; return dist2(c, v1) <= r2 + eps2 ? CT_VERTEX : CT_NONE; }
    double vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
        double t = d1 / (d1 - d3);
        cp = v0 + ab * t;
        return dist2(c, cp) <= r2 + eps2 ? CT_EDGE : CT_NONE;
    }
    V3 cpv = c - v2;
    double d5 = dot(ab, cpv), d6 = dot(ac, cpv);
    if (d6 >= 0.0 && d5 <= d6) { cp = v2; return dist2(c, v2) <= r2 + eps2 ? CT_VERTEX : CT_NONE; }
    double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
        double t = d2 / (d2 - d6);
        cp = v0 + ac * t;
        return dist2(c, cp) <= r2 + eps2 ? CT_EDGE : CT_NONE;
    }
    double va = d3 * d6 - d5 * d4;
    if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
        double t = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        cp = v1 + (v2 - v1) * t;
        return dist2(c, cp) <= r2 + eps2 ? CT_EDGE : CT_NONE;
    }
    double sum = va + vb + vc;
    if (std::fabs(sum) <= 1e-30) return CT_NONE;  // cp left as passed in
    double inv = 1.0 / sum;
    double v = vb * inv, w = vc * inv;
    cp = v0 + ab * v + ac * w;
    return dist2(c, cp) <= r2 + eps2 ? CT_FACE : CT_NONE;
}

// ------------------------------------------------------------ DEM scene ---
struct Body {  // clump or mesh-wall rigid body (particle.h:274, DEMSolver.h:137-142)
    std::vector<V3> pos, vel, w, force, torque;
    std::vector<Quat> q;
    std::vector<SymM> invI;
    std::vector<double> invMass;
    std::vector<int> mat, start, end;
    size_t size() const { return pos.size(); }
    void add(V3 p, V3 v, V3 ww, Quat qq, SymM I, double im, int m, int s, int e) {
        pos.push_back(p); vel.push_back(v); w.push_back(ww); force.push_back(v3(0, 0, 0)); torque.push_back(v3(0, 0, 0));
        q.push_back(qq); invI.push_back(I); invMass.push_back(im); mat.push_back(m); start.push_back(s); end.push_back(e);
    }
};

struct Pairs {  // pair + spring + contact + objectPointed + objectPointing (interaction.h)
    size_t n = 0;
    std::vector<int> pointed, pointing, hashIndex, cancel;
    std::vector<V3> sl, ro, to, cpoint, cnormal, cforce, ctorque;
    std::vector<double> overlap;
    std::vector<int> prefix;          // per pointed object (inclusive scan of counts)
    std::vector<int> iStart, iEnd;    // per pointing object: range in hashIndex
    void resize(size_t m) {
        n = m;
        pointed.assign(m, 0); pointing.assign(m, 0); hashIndex.assign(m, 0); cancel.assign(m, 0);
        sl.assign(m, v3(0, 0, 0)); ro.assign(m, v3(0, 0, 0)); to.assign(m, v3(0, 0, 0));
        cpoint.assign(m, v3(0, 0, 0)); cnormal.assign(m, v3(0, 0, 0)); cforce.assign(m, v3(0, 0, 0));
        ctorque.assign(m, v3(0, 0, 0)); overlap.assign(m, 0.0);
    }
    // DEMSolver.h:59-78: sort pairs by pointing (stable), start/end per object.
    void buildPointing(size_t nObj) {
        iStart.assign(nObj, -1);  // Q7 corrected: reset every build
        iEnd.assign(nObj, -1);
        hashIndex.resize(n);
        std::iota(hashIndex.begin(), hashIndex.end(), 0);
        std::stable_sort(hashIndex.begin(), hashIndex.end(), [&](int a, int b) { return pointing[a] < pointing[b]; });
        for (size_t k = 0; k < n; k++) {
            int h = pointing[hashIndex[k]];
            if (k == 0 || pointing[hashIndex[k - 1]] != h) iStart[h] = (int)k;
            if (k == n - 1 || pointing[hashIndex[k + 1]] != h) iEnd[h] = (int)(k + 1);
        }
    }
    int rowStart(int i) const { return i > 0 ? prefix[i - 1] : 0; }
};

struct DEM {
    Materials M;
    // balls (particle.h:6-272)
    std::vector<V3> pos, vel, w, force, torque;
    std::vector<double> rad, invMass;
    std::vector<int> mat, clump;
    Body clumps, walls;
    // mesh (wall.h)
    std::vector<int> t0, t1, t2, tWall;
    std::vector<V3> tCenter;
    std::vector<V3> vLocal, vGlobal;
    std::vector<int> vWall;
    // bonds (DEMSolver.h:88-135, interaction.h:371-509)
    std::vector<int> bA, bB, bOk;
    std::vector<V3> bPoint, bNormal, bFs, bTb;
    std::vector<double> bFn, bTt, bSmax, bTmax;
    Grid ballGrid, triGrid;
    std::vector<int> ballHashIndex, ballHashValue, triHashIndex, triHashValue;
    Pairs bb, bt;
    // external force hook (externalForceTorque.cu)
    bool hasBuoy = false;
    double buoyRho = 0, buoyCd = 0, buoyLevel = 0;
    V3 buoyG{0, 0, 0}, buoyU{0, 0, 0};
    double dampCoeff = 0;
    std::vector<V3> constForce;
    double constRamp = 0;
    // force / torque of a coupled fluid per ball (particle-level coupling)
    std::vector<V3> cplF, cplT;
    V3 gravity{0, 0, 0};
    double dt = 0;
    long iStep = 0;
    double time = 0;
    bool initialized = false;
    // periodic ghost sets (DEMSolver.h:81-86,1944-1959)
    struct Ghost {
        int dx, dy, dz;
        std::vector<V3> gpos;
        Grid grid;
        std::vector<int> hashIndex, hashValue;
        Pairs p;
    };
    bool perX = false, perY = false, perZ = false;
    std::vector<Ghost> ghosts;
    size_t nb() const { return pos.size(); }
};

// DEMSolver.h:698-777 + ballNeighborSearchKernel.cu:6-151
static void demNeighborSearch(DEM& s) {
    const size_t N = s.nb();
    if (!s.ballGrid.valid || N == 0) return;
    buildCellTable(s.ballGrid, s.pos, s.ballHashIndex, s.ballHashValue);
    Pairs old = s.bb;  // updateOldPairOldSpring + the not-yet-rebuilt pointing ranges
    std::vector<int> cnt(N, 0);
    auto accept = [&](int A, int B) -> bool {
        if (A >= B) return false;
        if (s.invMass[A] == 0 && s.invMass[B] == 0) return false;
        if (s.clump[B] >= 0 && s.clump[A] == s.clump[B]) return false;
        double cut = 1.1 * (s.rad[A] + s.rad[B]);
        V3 r = s.pos[A] - s.pos[B];
        return (cut * cut - dot(r, r)) >= 0.;
    };
#pragma omp parallel for schedule(dynamic, 256)
    for (long A = 0; A < (long)N; A++) {
        int c = 0;
        forEachStencilCell(s.pos[A], s.ballGrid, [&](int st, int en) {
            for (int k = st; k < en; k++) if (accept((int)A, s.ballHashIndex[k])) c++;
        });
        cnt[A] = c;
    }
    std::vector<int> prefix(N);
    std::partial_sum(cnt.begin(), cnt.end(), prefix.begin());
    size_t P = N ? (size_t)prefix[N - 1] : 0;
    s.bb.resize(P);
    s.bb.prefix = prefix;
#pragma omp parallel for schedule(dynamic, 256)
    for (long A = 0; A < (long)N; A++) {
        int w = A > 0 ? prefix[A - 1] : 0;
        forEachStencilCell(s.pos[A], s.ballGrid, [&](int st, int en) {
            for (int k = st; k < en; k++) {
                int B = s.ballHashIndex[k];
                if (!accept((int)A, B)) continue;
                s.bb.pointed[w] = (int)A;
                s.bb.pointing[w] = B;
                if (B < (int)old.iStart.size() && old.iStart[B] != -1) {
                    for (int j = old.iStart[B]; j < old.iEnd[B]; j++) {
                        int j1 = old.hashIndex[j];
                        if (old.pointed[j1] == (int)A) {
                            s.bb.sl[w] = old.sl[j1]; s.bb.ro[w] = old.ro[j1]; s.bb.to[w] = old.to[j1];
                            break;
                        }
                    }
                }
                w++;
            }
        });
    }
    s.bb.buildPointing(N);
}

// DEMSolver.h:599-695 + contactKernel.cu:135-259,535-714
static void demBallForces(DEM& s, double dt) {
    const size_t N = s.nb();
    std::fill(s.force.begin(), s.force.end(), v3(0, 0, 0));
    std::fill(s.torque.begin(), s.torque.end(), v3(0, 0, 0));
    Pairs& p = s.bb;
#pragma omp parallel for schedule(static)
    for (long k = 0; k < (long)p.n; k++) {
        int i = p.pointed[k], j = p.pointing[k];
        // updateBallContactKernel (contactKernel.cu:135-163)
        V3 rij = s.pos[i] - s.pos[j];
        V3 n = normalize(rij);
        double delta = s.rad[i] + s.rad[j] - length(rij);
        V3 rc = s.pos[j] + (s.rad[j] - 0.5 * delta) * n;
        p.cpoint[k] = rc; p.cnormal[k] = n; p.overlap[k] = delta;
        // calBallContactForceTorqueKernel (contactKernel.cu:165-259)
        double R = s.rad[i] * s.rad[j] / (s.rad[i] + s.rad[j]);
        double m = 1. / (s.invMass[i] + s.invMass[j]);
        V3 vc = s.vel[i] + cross(s.w[i], rc - s.pos[i]) - (s.vel[j] + cross(s.w[j], rc - s.pos[j]));
        V3 wij = s.w[i] - s.w[j];
        int ip = s.M.index(s.mat[i], s.mat[j]);
        V3 F, T;
        pairLaw(s.M, ip, F, T, p.sl[k], p.ro[k], p.to[k], vc, wij, n, delta, m, R, dt);
        p.cforce[k] = F; p.ctorque[k] = T;
    }
    // calBondedForceTorqueKernel (contactKernel.cu:535-655), sequential in bond order
    for (size_t b = 0; b < s.bA.size(); b++) {
        if (s.bOk[b] == 0) {
            s.bFn[b] = 0; s.bTt[b] = 0; s.bFs[b] = v3(0, 0, 0); s.bTb[b] = v3(0, 0, 0);
            continue;
        }
        int i = s.bA[b], j = s.bB[b];
        V3 ri = s.pos[i], rj = s.pos[j];
        V3 n0 = s.bNormal[b];
        V3 n = normalize(ri - rj);
        double delta = s.rad[i] + s.rad[j] - length(ri - rj);
        V3 rc = rj + (s.rad[j] - 0.5 * delta) * n;
        s.bPoint[b] = rc; s.bNormal[b] = n;
        bool found = false;
        int kc = 0;
        if (p.n > 0 && !p.prefix.empty()) {
            for (int k = p.rowStart(i); k < p.prefix[i]; k++) {
                if (p.pointing[k] == j) {
                    found = true; kc = k; rc = p.cpoint[k]; n = p.cnormal[k];
                    s.bPoint[b] = rc; s.bNormal[b] = n;
                    break;
                }
            }
        }
        V3 vc = s.vel[i] + cross(s.w[i], rc - ri) - (s.vel[j] + cross(s.w[j], rc - rj));
        int ip = s.M.index(s.mat[i], s.mat[j]);
        s.bOk[b] = parallelBondedContact(s.bFn[b], s.bTt[b], s.bFs[b], s.bTb[b], s.bSmax[b], s.bTmax[b], n0, n, vc,
                                         s.w[i], s.w[j], s.rad[i], s.rad[j], dt, s.M.b(ip, B_GAMMA), s.M.b(ip, B_E),
                                         s.M.b(ip, B_KNKS), s.M.b(ip, B_SIGMA), s.M.b(ip, B_C), s.M.b(ip, B_MU));
        double Fn = s.bFn[b], Tt = s.bTt[b];
        V3 Fs = s.bFs[b], Tb = s.bTb[b];
        if (!found) {
            s.force[i] += Fn * n + Fs;
            s.torque[i] += Tt * n + Tb + cross(rc - ri, Fs);
            s.force[j] += -Fn * n - Fs;
            s.torque[j] += -Tt * n - Tb + cross(rc - rj, -Fs);
        } else {
            p.cforce[kc] += Fn * n + Fs;
            p.ctorque[kc] += Tt * n + Tb;
        }
    }
    // sumObjectPointed / sumObjectPointing (contactKernel.cu:657-714)
    if (p.prefix.size() == N) {
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)N; i++) {
            V3 Fi = v3(0, 0, 0), Ti = v3(0, 0, 0);
            for (int k = p.rowStart((int)i); k < p.prefix[i]; k++) {
                Fi += p.cforce[k];
                Ti += p.ctorque[k] + cross(p.cpoint[k] - s.pos[i], p.cforce[k]);
            }
            s.force[i] += Fi;
            s.torque[i] += Ti;
        }
    }
    if (p.iStart.size() == N) {
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)N; i++) {
            V3 Fi = v3(0, 0, 0), Ti = v3(0, 0, 0);
            if (p.iStart[i] != -1) {
                for (int k = p.iStart[i]; k < p.iEnd[i]; k++) {
                    int k1 = p.hashIndex[k];
                    Fi -= p.cforce[k1];
                    Ti -= p.ctorque[k1];
                    Ti -= cross(p.cpoint[k1] - s.pos[i], p.cforce[k1]);
                }
            }
            s.force[i] += Fi;
            s.torque[i] += Ti;
        }
    }
}

// addDummyContactForceTorque (DEMSolver.h:279-426): ghost positions
// (buildDummyPosition, neighborSearchKernel.cu:57-77), a cell table of the
// ghosts that left the domain (calculateDummyHash, neighborSearchKernel.cu:
// 29-55, then the stable sort of buildHashStartEnd), the pair rule of
// count/writeBallInteractionsKernel on the ghost positions with springs
// carried from the previous ghost list, the contact law, and the pointed /
// pointing sums with the ghost positions as torque arms.
static void demGhostForces(DEM& s, DEM::Ghost& g, double dt) {
    const size_t N = s.nb();
    const Grid& bg = s.ballGrid;
    const V3 L = bg.mx - bg.mn;
    g.gpos.resize(N);
    for (size_t i = 0; i < N; i++) {
        V3 p = s.pos[i];
        if (g.dx == 1 && p.x - bg.mn.x < bg.cs.x) p.x += L.x;
        if (g.dy == 1 && p.y - bg.mn.y < bg.cs.y) p.y += L.y;
        if (g.dz == 1 && p.z - bg.mn.z < bg.cs.z) p.z += L.z;
        g.gpos[i] = p;
    }
    g.hashValue.assign(N, -1);
    g.hashIndex.resize(N);
    for (size_t i = 0; i < N; i++) {
        V3 p = g.gpos[i];
        bool out = p.x < bg.mn.x || p.x >= bg.mx.x || p.y < bg.mn.y || p.y >= bg.mx.y || p.z < bg.mn.z ||
                   p.z >= bg.mx.z;
        if (out) g.hashValue[i] = clampedHash(p, bg);
    }
    std::iota(g.hashIndex.begin(), g.hashIndex.end(), 0);
    std::stable_sort(g.hashIndex.begin(), g.hashIndex.end(),
                     [&](int a, int b) { return g.hashValue[a] < g.hashValue[b]; });
    std::vector<int> sortedKey(N);
    for (size_t i = 0; i < N; i++) sortedKey[i] = g.hashValue[g.hashIndex[i]];
    g.grid = bg;
    std::fill(g.grid.start.begin(), g.grid.start.end(), -1);
    std::fill(g.grid.end.begin(), g.grid.end.end(), -1);
    for (size_t i = 0; i < N; i++) {
        int h = sortedKey[i];
        if (h < 0) continue;
        if (i == 0 || sortedKey[i - 1] != h) g.grid.start[h] = (int)i;
        if (i == N - 1 || sortedKey[i + 1] != h) g.grid.end[h] = (int)(i + 1);
    }
    Pairs old = g.p;
    auto accept = [&](int A, int B) -> bool {
        if (A >= B) return false;
        if (s.invMass[A] == 0 && s.invMass[B] == 0) return false;
        if (s.clump[B] >= 0 && s.clump[A] == s.clump[B]) return false;
        double cut = 1.1 * (s.rad[A] + s.rad[B]);
        V3 r = g.gpos[A] - g.gpos[B];
        return (cut * cut - dot(r, r)) >= 0.;
    };
    std::vector<int> cnt(N, 0);
    for (size_t A = 0; A < N; A++) {
        int c = 0;
        forEachStencilCell(g.gpos[A], g.grid, [&](int st, int en) {
            for (int k = st; k < en; k++) if (accept((int)A, g.hashIndex[k])) c++;
        });
        cnt[A] = c;
    }
    std::vector<int> prefix(N);
    std::partial_sum(cnt.begin(), cnt.end(), prefix.begin());
    size_t P = N ? (size_t)prefix[N - 1] : 0;
    g.p.resize(P);
    g.p.prefix = prefix;
    for (size_t A = 0; A < N; A++) {
        int w = A > 0 ? prefix[A - 1] : 0;
        forEachStencilCell(g.gpos[A], g.grid, [&](int st, int en) {
            for (int k = st; k < en; k++) {
                int B = g.hashIndex[k];
                if (!accept((int)A, B)) continue;
                g.p.pointed[w] = (int)A;
                g.p.pointing[w] = B;
                if (B < (int)old.iStart.size() && old.iStart[B] != -1) {
                    for (int j = old.iStart[B]; j < old.iEnd[B]; j++) {
                        int j1 = old.hashIndex[j];
                        if (old.pointed[j1] == (int)A) {
                            g.p.sl[w] = old.sl[j1]; g.p.ro[w] = old.ro[j1]; g.p.to[w] = old.to[j1];
                            break;
                        }
                    }
                }
                w++;
            }
        });
    }
    g.p.buildPointing(N);
    Pairs& p = g.p;
    for (size_t k = 0; k < p.n; k++) {
        int i = p.pointed[k], j = p.pointing[k];
        V3 rij = g.gpos[i] - g.gpos[j];
        V3 n = normalize(rij);
        double delta = s.rad[i] + s.rad[j] - length(rij);
        V3 rc = g.gpos[j] + (s.rad[j] - 0.5 * delta) * n;
        p.cpoint[k] = rc; p.cnormal[k] = n; p.overlap[k] = delta;
        double R = s.rad[i] * s.rad[j] / (s.rad[i] + s.rad[j]);
        double m = 1. / (s.invMass[i] + s.invMass[j]);
        V3 vc = s.vel[i] + cross(s.w[i], rc - g.gpos[i]) - (s.vel[j] + cross(s.w[j], rc - g.gpos[j]));
        V3 wij = s.w[i] - s.w[j];
        int ip = s.M.index(s.mat[i], s.mat[j]);
        V3 F, T;
        pairLaw(s.M, ip, F, T, p.sl[k], p.ro[k], p.to[k], vc, wij, n, delta, m, R, dt);
        p.cforce[k] = F; p.ctorque[k] = T;
    }
    for (size_t i = 0; i < N; i++) {
        V3 Fi = v3(0, 0, 0), Ti = v3(0, 0, 0);
        for (int k = p.rowStart((int)i); k < p.prefix[i]; k++) {
            Fi += p.cforce[k];
            Ti += p.ctorque[k] + cross(p.cpoint[k] - g.gpos[i], p.cforce[k]);
        }
        s.force[i] += Fi;
        s.torque[i] += Ti;
    }
    for (size_t i = 0; i < N; i++) {
        V3 Fi = v3(0, 0, 0), Ti = v3(0, 0, 0);
        if (p.iStart[i] != -1) {
            for (int k = p.iStart[i]; k < p.iEnd[i]; k++) {
                int k1 = p.hashIndex[k];
                Fi -= p.cforce[k1];
                Ti -= p.ctorque[k1];
                Ti -= cross(p.cpoint[k1] - g.gpos[i], p.cforce[k1]);
            }
        }
        s.force[i] += Fi;
        s.torque[i] += Ti;
    }
}

// DEMSolver.h:428-597 with ballNeighborSearchKernel.cu:153-338 and
// contactKernel.cu:261-533; wallIntegrationKernel.cu:3-53.
static void demTriangleForces(DEM& s, double dt) {
    const size_t T = s.t0.size();
    if (T == 0) return;
    const size_t N = s.nb();
    buildCellTable(s.triGrid, s.tCenter, s.triHashIndex, s.triHashValue);
    Pairs old = s.bt;
    auto aabbHit = [&](int A, int tri) -> bool {
        V3 p = s.pos[A];
        V3 a = s.vGlobal[s.t0[tri]], b = s.vGlobal[s.t1[tri]], c = s.vGlobal[s.t2[tri]];
        double mnx = std::fmin(a.x, std::fmin(b.x, c.x)), mny = std::fmin(a.y, std::fmin(b.y, c.y)),
               mnz = std::fmin(a.z, std::fmin(b.z, c.z));
        double mxx = std::fmax(a.x, std::fmax(b.x, c.x)), mxy = std::fmax(a.y, std::fmax(b.y, c.y)),
               mxz = std::fmax(a.z, std::fmax(b.z, c.z));
        double cx = std::fmin(std::fmax(p.x, mnx), mxx), cy = std::fmin(std::fmax(p.y, mny), mxy),
               cz = std::fmin(std::fmax(p.z, mnz), mxz);
        double dx = p.x - cx, dy = p.y - cy, dz = p.z - cz;
        return dx * dx + dy * dy + dz * dz <= s.rad[A] * s.rad[A];
    };
    std::vector<int> cnt(N, 0);
#pragma omp parallel for schedule(dynamic, 256)
    for (long A = 0; A < (long)N; A++) {
        int c = 0;
        forEachStencilCell(s.pos[A], s.triGrid, [&](int st, int en) {
            for (int k = st; k < en; k++) if (aabbHit((int)A, s.triHashIndex[k])) c++;
        });
        cnt[A] = c;
    }
    std::vector<int> prefix(N);
    std::partial_sum(cnt.begin(), cnt.end(), prefix.begin());
    size_t P = N ? (size_t)prefix[N - 1] : 0;
    s.bt.resize(P);
    s.bt.prefix = prefix;
#pragma omp parallel for schedule(dynamic, 256)
    for (long A = 0; A < (long)N; A++) {
        int wpos = A > 0 ? prefix[A - 1] : 0;
        forEachStencilCell(s.pos[A], s.triGrid, [&](int st, int en) {
            for (int k = st; k < en; k++) {
                int B = s.triHashIndex[k];
                if (!aabbHit((int)A, B)) continue;
                s.bt.pointed[wpos] = (int)A;
                s.bt.pointing[wpos] = B;
                if (B < (int)old.iStart.size() && old.iStart[B] != -1) {
                    for (int j = old.iStart[B]; j < old.iEnd[B]; j++) {
                        int j1 = old.hashIndex[j];
                        if (old.pointed[j1] == (int)A) {
                            s.bt.sl[wpos] = old.sl[j1]; s.bt.ro[wpos] = old.ro[j1]; s.bt.to[wpos] = old.to[j1];
                            break;
                        }
                    }
                }
                wpos++;
            }
        });
    }
    s.bt.buildPointing(T);
    Pairs& p = s.bt;
    if (p.n > 0) {
#pragma omp parallel for schedule(dynamic, 64)
        for (long i = 0; i < (long)N; i++) {
            // updateBallTriangleContact (contactKernel.cu:261-418)
            int st = p.rowStart((int)i), en = p.prefix[i];
            for (int c = st; c < en; c++) {
                p.cancel[c] = 0;
                int tj = p.pointing[c];
                double ri = s.rad[i];
                V3 pi = s.pos[i];
                V3 p0 = s.vGlobal[s.t0[tj]], p1 = s.vGlobal[s.t1[tj]], p2 = s.vGlobal[s.t2[tj]];
                V3 rc = v3(0, 0, 0);
                int type = classifySphereTriangle(pi, ri, p0, p1, p2, rc);
                p.cpoint[c] = rc;
                p.cnormal[c] = normalize(pi - rc);
                p.overlap[c] = ri - length(pi - rc);
                if (type == CT_NONE) {
                    p.sl[c] = p.ro[c] = p.to[c] = v3(0, 0, 0);
                    p.cancel[c] = 1;
                    continue;
                }
                if (type != CT_FACE) {
                    for (int c1 = st; c1 < en; c1++) {
                        if (c1 == c) continue;
                        int tj1 = p.pointing[c1];
                        V3 q0 = s.vGlobal[s.t0[tj1]], q1 = s.vGlobal[s.t1[tj1]], q2 = s.vGlobal[s.t2[tj1]];
                        V3 rc1 = v3(0, 0, 0);
                        int type1 = classifySphereTriangle(pi, ri, q0, q1, q2, rc1);
                        bool copy = false;
                        if (type1 == CT_NONE) continue;
                        else if (type1 == CT_FACE) {
                            if (lengthSquared(cross(rc - q0, q1 - q0)) < 1.e-20) copy = true;
                            else if (lengthSquared(cross(rc - q1, q2 - q1)) < 1.e-20) copy = true;
                            else if (lengthSquared(cross(rc - q0, q2 - q0)) < 1.e-20) copy = true;
                        } else if (type1 == CT_EDGE) {
                            if (type == type1) { if (c1 < c && lengthSquared(rc - rc1) < 1.e-20) copy = true; }
                            else if (lengthSquared(rc - rc1) < 1.e-20) copy = true;
                        } else {
                            if (type == type1 && c1 < c && lengthSquared(rc - rc1) < 1.e-20) copy = true;
                        }
                        if (copy) {
                            p.sl[c] = p.sl[c1]; p.ro[c] = p.ro[c1]; p.to[c] = p.to[c1];
                            p.cancel[c] = 1;
                            break;
                        }
                    }
                }
            }
            // calBallWallContactForceTorqueKernel (contactKernel.cu:420-533)
            if (s.invMass[i] < 1.e-20) continue;
            V3 ri = s.pos[i], vi = s.vel[i], wi = s.w[i];
            double R = s.rad[i];
            double m = 1. / s.invMass[i];
            for (int c = st; c < en; c++) {
                p.cforce[c] = v3(0, 0, 0);
                p.ctorque[c] = v3(0, 0, 0);
                if (p.cancel[c] == 1) continue;
                int wj = s.tWall[p.pointing[c]];
                V3 rc = p.cpoint[c], n = p.cnormal[c];
                double delta = p.overlap[c];
                V3 rj = s.walls.pos[wj], vj = s.walls.vel[wj], wwj = s.walls.w[wj];
                V3 vc = vi + cross(wi, rc - ri) - (vj + cross(wwj, rc - rj));
                V3 wij = wi - wwj;
                int ip = s.M.index(s.mat[i], s.walls.mat[wj]);
                V3 F, Tq;
                pairLaw(s.M, ip, F, Tq, p.sl[c], p.ro[c], p.to[c], vc, wij, n, delta, m, R, dt);
                p.cforce[c] = F; p.ctorque[c] = Tq;
                s.force[i] += F;
                s.torque[i] += Tq + cross(rc - ri, F);
            }
        }
    }
    // launchWallIntegration / vertex / circumcenter (wallIntegrationKernel.cu:3-53)
    for (size_t wi = 0; wi < s.walls.size(); wi++) {
        s.walls.pos[wi] += dt * s.walls.vel[wi];
        s.walls.q[wi] = quaternionRotate(s.walls.q[wi], s.walls.w[wi], dt);
    }
    for (size_t v = 0; v < s.vLocal.size(); v++) {
        int wi = s.vWall[v];
        s.vGlobal[v] = s.walls.pos[wi] + rotateVectorByQuaternion(s.walls.q[wi], s.vLocal[v]);
    }
    for (size_t t = 0; t < T; t++) s.tCenter[t] = triangleCircumcenter(s.vGlobal[s.t0[t]], s.vGlobal[s.t1[t]], s.vGlobal[s.t2[t]]);
}

// externalForceTorque.cu:4-133 (user hook as configured by the scene)
static void demExternal(DEM& s, double time) {
    const size_t N = s.nb();
    if (!s.constForce.empty()) {
        double c = 1.0;
        if (s.constRamp > 0) { c = time / s.constRamp; if (c > 1.0) c = 1.0; }
        for (size_t i = 0; i < N && i < s.constForce.size(); i++) s.force[i] += s.constForce[i] * c;
    }
    for (size_t i = 0; i < N && i < s.cplF.size(); i++) {
        s.force[i] += s.cplF[i];
        s.torque[i] += s.cplT[i];
    }
    if (s.dampCoeff != 0) {
        for (size_t i = 0; i < N; i++) {
            V3 f = s.force[i], t = s.torque[i];
            s.force[i] -= s.dampCoeff * length(f) * normalize(s.vel[i]);
            s.torque[i] -= s.dampCoeff * length(t) * normalize(s.w[i]);
        }
    }
    if (s.hasBuoy) {
        for (size_t i = 0; i < N; i++) {
            if (s.invMass[i] <= 0.0) continue;
            double r = s.rad[i];
            double d = s.buoyLevel - s.pos[i].z;
            double Vsub;
            if (d <= -r) Vsub = 0.0;
            else if (d >= r) Vsub = (4.0 / 3.0) * PI * r * r * r;
            else { double h = d + r; Vsub = (PI * h * h * (3.0 * r - h)) / 3.0; }
            if (Vsub <= 0.0) continue;
            V3 Fb = v3(-s.buoyRho * Vsub * s.buoyG.x, -s.buoyRho * Vsub * s.buoyG.y, -s.buoyRho * Vsub * s.buoyG.z);
            double Vs = (4.0 / 3.0) * PI * r * r * r;
            double alpha = (Vs > 1.e-30) ? (Vsub / Vs) : 0.0;
            V3 vr = s.vel[i] - s.buoyU;
            double v2 = dot(vr, vr);
            V3 Fd = v3(0, 0, 0);
            if (v2 > 1.e-30 && s.buoyCd > 0.0) {
                double vm = std::sqrt(v2);
                double Aeff = alpha * (PI * r * r);
                double k = 0.5 * s.buoyRho * s.buoyCd * Aeff * vm;
                Fd = v3(-k * vr.x, -k * vr.y, -k * vr.z);
            }
            s.force[i].x += Fb.x + Fd.x;
            s.force[i].y += Fb.y + Fd.y;
            s.force[i].z += Fb.z + Fd.z;
        }
    }
}

// ballIntegrationKernel.cu:3-121,123-309; DEMSolver.h:779-906
static void demClumpGather(DEM& s) {
    for (size_t c = 0; c < s.clumps.size(); c++) {
        V3 F = v3(0, 0, 0), T = v3(0, 0, 0);
        for (int i = s.clumps.start[c]; i < s.clumps.end[c]; i++) {
            V3 Fi = s.force[i];  // Q1 corrected (reference reads force_c[i])
            F += Fi;
            T += s.torque[i] + cross(s.pos[i] - s.clumps.pos[c], Fi);
        }
        s.clumps.force[c] = F;
        s.clumps.torque[c] = T;
    }
}
static void demClumpKick(DEM& s, double hdt) {
    for (size_t c = 0; c < s.clumps.size(); c++) {
        double im = s.clumps.invMass[c];
        if (im > 1.e-20) {
            s.clumps.vel[c] += (s.clumps.force[c] * im + s.gravity) * hdt;
            s.clumps.w[c] += (rotateInverseInertiaTensor(s.clumps.q[c], s.clumps.invI[c]) * s.clumps.torque[c]) * hdt;
        }
    }
}
static void demPebbleVelocity(DEM& s) {
    for (size_t i = 0; i < s.nb(); i++) {
        int c = s.clump[i];
        if (c < 0) continue;
        V3 w = s.clumps.w[c];
        s.w[i] = w;
        s.vel[i] = s.clumps.vel[c] + cross(w, s.pos[i] - s.clumps.pos[c]);
    }
}
static void demBallKick(DEM& s, double hdt) {
    for (size_t i = 0; i < s.nb(); i++) {
        if (s.clump[i] >= 0) continue;
        double im = s.invMass[i];
        if (im < 1.e-20) continue;
        s.vel[i] += (s.force[i] * im + s.gravity) * hdt;
        double r = s.rad[i];
        if (r < 1.e-20) continue;
        double I = 0.4 * r * r / im;
        s.w[i] += s.torque[i] / I * hdt;
    }
}
static void demFirstHalf(DEM& s, double hdt) {
    if (s.clumps.size() > 0) {
        demClumpGather(s);
        demClumpKick(s, hdt);
        for (size_t c = 0; c < s.clumps.size(); c++) {
            s.clumps.pos[c] += 2.0 * hdt * s.clumps.vel[c];
            s.clumps.q[c] = quaternionRotate(s.clumps.q[c], s.clumps.w[c], 2.0 * hdt);
        }
        demPebbleVelocity(s);
    }
    demBallKick(s, hdt);
    for (size_t i = 0; i < s.nb(); i++) s.pos[i] += 2.0 * hdt * s.vel[i];
}
static void demSecondHalf(DEM& s, double hdt) {
    if (s.clumps.size() > 0) {
        demClumpGather(s);
        demClumpKick(s, hdt);
        demPebbleVelocity(s);
    }
    demBallKick(s, hdt);
}

// One pass of loop_ball / loop_ball_wall (DEMSolver.h:1376-1485).
static void demStep(DEM& s) {
    const double dt = s.dt, hdt = 0.5 * dt;
    s.iStep++;
    s.time += dt;
    if (s.iStep % 5 == 0) demNeighborSearch(s);
    demBallForces(s, hdt);
    demTriangleForces(s, dt);
    for (auto& g : s.ghosts) demGhostForces(s, g, hdt);
    demExternal(s, s.time - hdt);
    demFirstHalf(s, hdt);
    demBallForces(s, hdt);
    demTriangleForces(s, dt);
    for (auto& g : s.ghosts) demGhostForces(s, g, hdt);
    demExternal(s, s.time);
    demSecondHalf(s, hdt);
}

// ------------------------------------------------------------ WCSPH ------
// WCSPHIntegrationKernel.cuh:15-32
static inline V3 gradW(V3 rij, double h) {
    double r = length(rij);
    if (r < 1.e-20 || r >= 2.0 * h) return v3(0, 0, 0);
    double q = r / h;
    double sigma = 21.0 / (16.0 * PI * h * h * h);
    double t = 1.0 - 0.5 * q;
    double dq = (-2.0 * std::pow(t, 3) * (1.0 + 2.0 * q) + 2.0 * std::pow(t, 4));
    double dWdr = sigma * dq / h;
    return (dWdr / r) * rij;
}

struct SPHSet {  // particle.h:552-837
    std::vector<V3> pos, vel, acc, normal;
    std::vector<double> drho, rho, p, rho0, h, m, c, nu;
    size_t size() const { return pos.size(); }
    void add(V3 x, V3 v, double cc, double spacing, double dens, double visc) {
        if (dens <= 0. || cc <= 0.) return;  // WCSPHSolver.h:523-541
        pos.push_back(x); vel.push_back(v); acc.push_back(v3(0, 0, 0)); normal.push_back(v3(0, 0, 0));
        drho.push_back(0.0); rho.push_back(dens); p.push_back(0.0); rho0.push_back(dens);
        h.push_back(1.3 * spacing); m.push_back(spacing * spacing * spacing * dens); c.push_back(cc); nu.push_back(visc);
    }
};
struct CSR { std::vector<int> prefix, pointed, pointing; };

struct SPH {
    SPHSet f, d;
    Grid grid;
    std::vector<int> fHashIndex, fHashValue, dHashIndex, dHashValue;
    CSR ff, fd, dd;
    // Particle-level coupling to DEM balls (no reference counterpart): the
    // markers sampling each coupled ball, in body order, act on the fluid as
    // dummies; mkF collects the fluid's reaction on each marker.
    SPHSet mk;
    std::vector<int> mkBall, body, bodyStart{0};
    std::vector<V3> mkOff, mkF;
    std::vector<int> mHashIndex, mHashValue;
    CSR fm;
    bool coupling = false;
    V3 gravity{0, 0, 0};
    double dt = 0;
    long iStep = 0;
    double time = 0;
    bool initialized = false;
};

// countSPHInteractionsKernel / writeSPHInteractionsKernel and the dummy
// variants (SPHNeighborSearchKernel.cu:6-228).
static void sphPairs(const SPHSet& a, const SPHSet& b, const Grid& g, const std::vector<int>& bHashIndex, bool same, CSR& out) {
    size_t N = a.size();
    std::vector<int> cnt(N, 0);
    auto accept = [&](int A, int B) -> bool {
        if (same && A == B) return false;
        double cut = 2.0 * std::fmax(a.h[A], b.h[B]);
        V3 r = a.pos[A] - b.pos[B];
        return (cut * cut - dot(r, r)) >= 0.;
    };
#pragma omp parallel for schedule(dynamic, 256)
    for (long A = 0; A < (long)N; A++) {
        int c = 0;
        forEachStencilCell(a.pos[A], g, [&](int st, int en) {
            for (int k = st; k < en; k++) if (accept((int)A, bHashIndex[k])) c++;
        });
        cnt[A] = c;
    }
    out.prefix.resize(N);
    std::partial_sum(cnt.begin(), cnt.end(), out.prefix.begin());
    size_t P = N ? (size_t)out.prefix[N - 1] : 0;
    out.pointed.assign(P, 0);
    out.pointing.assign(P, 0);
#pragma omp parallel for schedule(dynamic, 256)
    for (long A = 0; A < (long)N; A++) {
        int w = A > 0 ? out.prefix[A - 1] : 0;
        forEachStencilCell(a.pos[A], g, [&](int st, int en) {
            for (int k = st; k < en; k++) {
                int B = bHashIndex[k];
                if (!accept((int)A, B)) continue;
                out.pointed[w] = (int)A;
                out.pointing[w] = B;
                w++;
            }
        });
    }
}

// WCSPHSolver.h:29-110 + calDummyParticleNormalKernel (WCSPHIntegrationKernel.cu:4-40)
static void sphInitBoundary(SPH& s) {
    size_t Nd = s.d.size();
    if (Nd == 0) return;
    buildCellTable(s.grid, s.d.pos, s.dHashIndex, s.dHashValue);
    sphPairs(s.d, s.d, s.grid, s.dHashIndex, true, s.dd);
    for (size_t i = 0; i < Nd; i++) {
        s.d.normal[i] = v3(0, 0, 0);
        V3 ri = s.d.pos[i];
        double hi = s.d.h[i];
        V3 th = v3(0, 0, 0);
        for (int k = i > 0 ? s.dd.prefix[i - 1] : 0; k < s.dd.prefix[i]; k++) {
            int j = s.dd.pointing[k];
            V3 dW = gradW(ri - s.d.pos[j], 0.5 * (hi + s.d.h[j]));
            th -= s.d.m[j] / s.d.rho[j] * dW;
        }
        if (lengthSquared(th) > 1.e-10) s.d.normal[i] = th / length(th);
    }
}

// WCSPHSolver.h:150-285
static void sphNeighborSearch(SPH& s) {
    buildCellTable(s.grid, s.f.pos, s.fHashIndex, s.fHashValue);
    sphPairs(s.f, s.f, s.grid, s.fHashIndex, true, s.ff);
    if (s.d.size() == 0) {
        s.fd.prefix.assign(s.f.size(), 0); s.fd.pointed.clear(); s.fd.pointing.clear();
    } else {
        buildCellTable(s.grid, s.d.pos, s.dHashIndex, s.dHashValue);
        sphPairs(s.f, s.d, s.grid, s.dHashIndex, false, s.fd);
    }
    if (s.mk.size() == 0) {
        s.fm.prefix.assign(s.f.size(), 0); s.fm.pointed.clear(); s.fm.pointing.clear();
    } else {
        buildCellTable(s.grid, s.mk.pos, s.mHashIndex, s.mHashValue);
        sphPairs(s.f, s.mk, s.grid, s.mHashIndex, false, s.fm);
    }
}

// The fluid-dummy term of updateWCSPHAccelerationKernel
// (WCSPHIntegrationKernel.cu:110-143) for fluid i and boundary particle j of
// set d, accumulated into acc in the reference's order.
static inline void sphBoundaryAcc(const SPH& s, const SPHSet& d, long i, int j, V3& acc) {
    const SPHSet& f = s.f;
    V3 g = s.gravity;
    V3 ri = f.pos[i], vi = f.vel[i];
    double ci = f.c[i], hi = f.h[i], nui = f.nu[i], rhoi = f.rho[i], PL = f.p[i];
    V3 rj = d.pos[j], vj = d.vel[j];
    double cj = d.c[j], hj = d.h[j], nuj = d.nu[j], mj = d.m[j];
    V3 nw = d.normal[j];
    double UL = dot(-nw, vi);
    double UR = -UL + 2.0 * dot(-nw, vj);
    double grj = dot(g, rj - ri);
    if (grj < 0.) grj = 0.;
    double PR = PL + rhoi * grj;
    double rhoj = PR / (cj * cj) + d.rho0[j];
    V3 rij = ri - rj;
    V3 dW = gradW(rij, 0.5 * (hi + hj));
    double cbar = 0.5 * (ci + cj), rbar = 0.5 * (rhoi + rhoj);
    double beta = std::fmin(3.0 * std::fmax(UL - UR, 0.0), cbar);
    double Ps = 0.5 * (PL + PR) + 0.5 * beta * rbar * (UL - UR);
    acc -= 2.0 * mj * (Ps / (rhoi * rhoj)) * dW;
    double nuij = 0.5 * (nui + nuj);
    acc += 2.0 * nuij * dot(normalize(rij), dW) * (vi - vj) * mj / (rhoi * rhoj);
}
// The fluid-dummy term of updateWCSPHDensityChangeKernel
// (WCSPHIntegrationKernel.cu:240-270), before the factor 2 rho_i.
static inline double sphBoundaryDrho(const SPH& s, const SPHSet& d, long i, int j) {
    const SPHSet& f = s.f;
    V3 g = s.gravity;
    V3 ri = f.pos[i], vi = f.vel[i];
    double ci = f.c[i], hi = f.h[i], rhoi = f.rho[i], PL = f.p[i];
    V3 rj = d.pos[j], vj = d.vel[j];
    double cj = d.c[j], hj = d.h[j], mj = d.m[j];
    double grj = dot(g, rj - ri);
    if (grj < 0.) grj = 0.;
    double PR = PL + rhoi * grj;
    double rhoj = PR / (cj * cj) + d.rho0[j];
    V3 rij = ri - rj;
    V3 dW = gradW(rij, 0.5 * (hi + hj));
    V3 e = -normalize(rij);
    double cbar = 0.5 * (ci + cj), rbar = 0.5 * (rhoi + rhoj);
    V3 vs = 0.5 * (vi + vj);
    vs += 0.5 * ((PL - PR) / (rbar * cbar)) * e;
    return mj / rhoj * dot(vi - vs, dW);
}

// updateWCSPHAccelerationKernel (WCSPHIntegrationKernel.cu:42-148)
static void sphAccel(SPH& s, double reactionWeight = 0.0, bool resetReaction = false) {
    const SPHSet& f = s.f;
    V3 g = s.gravity;
    size_t N = f.size();
    // per fluid-marker pair: the marker's term in the fluid acceleration
    std::vector<V3> pairAcc(s.coupling ? s.fm.pointing.size() : 0);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)N; i++) {
        V3 ri = f.pos[i], vi = f.vel[i];
        double ci = f.c[i], hi = f.h[i], nui = f.nu[i], rhoi = f.rho[i], PL = f.p[i];
        V3 acc = v3(0, 0, 0);
        for (int k = i > 0 ? s.ff.prefix[i - 1] : 0; k < s.ff.prefix[i]; k++) {
            int j = s.ff.pointing[k];
            V3 rj = f.pos[j], vj = f.vel[j];
            double cj = f.c[j], hj = f.h[j], nuj = f.nu[j], rhoj = f.rho[j], PR = f.p[j], mj = f.m[j];
            V3 rij = ri - rj;
            V3 e = -normalize(rij);
            double UL = dot(vi, e), UR = dot(vj, e);
            V3 dW = gradW(rij, 0.5 * (hi + hj));
            double cbar = 0.5 * (ci + cj), rbar = 0.5 * (rhoi + rhoj);
            double beta = std::fmin(3.0 * std::fmax(UL - UR, 0.0), cbar);
            double Ps = 0.5 * (PL + PR) + 0.5 * beta * rbar * (UL - UR);
            acc -= 2.0 * mj * (Ps / (rhoi * rhoj)) * dW;
            double nuij = 0.5 * (nui + nuj);
            acc += 2.0 * nuij * dot(normalize(rij), dW) * (vi - vj) * mj / (rhoi * rhoj);
        }
        if (!s.fd.prefix.empty())
            for (int k = i > 0 ? s.fd.prefix[i - 1] : 0; k < s.fd.prefix[i]; k++)
                sphBoundaryAcc(s, s.d, i, s.fd.pointing[k], acc);
        if (!s.fm.prefix.empty())
            for (int k = i > 0 ? s.fm.prefix[i - 1] : 0; k < s.fm.prefix[i]; k++) {
                if (s.coupling) {
                    V3 a = v3(0, 0, 0);
                    sphBoundaryAcc(s, s.mk, i, s.fm.pointing[k], a);
                    pairAcc[k] = a;
                }
                sphBoundaryAcc(s, s.mk, i, s.fm.pointing[k], acc);
            }
        s.f.acc[i] = acc + g;
    }
    if (!s.coupling) return;
    // reaction on each marker: minus m_a times its term in a_a
    if (resetReaction) s.mkF.assign(s.mk.size(), v3(0, 0, 0));
    std::vector<V3> r(s.mk.size(), v3(0, 0, 0));
    for (size_t k = 0; k < pairAcc.size(); k++) r[s.fm.pointing[k]] -= f.m[s.fm.pointed[k]] * pairAcc[k];
    for (size_t j = 0; j < r.size(); j++) s.mkF[j] += reactionWeight * r[j];
}

// updateWCSPHDensityChangeKernel + SPHDensityPressureIntegrationKernel
// (WCSPHIntegrationKernel.cu:172-282)
static void sphDensity(SPH& s, double dt) {
    const SPHSet& f = s.f;
    size_t N = f.size();
    std::vector<double> dr(N);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)N; i++) {
        V3 ri = f.pos[i], vi = f.vel[i];
        double ci = f.c[i], hi = f.h[i], rhoi = f.rho[i], PL = f.p[i];
        double dRho = 0.0;
        for (int k = i > 0 ? s.ff.prefix[i - 1] : 0; k < s.ff.prefix[i]; k++) {
            int j = s.ff.pointing[k];
            V3 rj = f.pos[j], vj = f.vel[j];
            double cj = f.c[j], hj = f.h[j], rhoj = f.rho[j], PR = f.p[j], mj = f.m[j];
            V3 rij = ri - rj;
            V3 dW = gradW(rij, 0.5 * (hi + hj));
            V3 e = -normalize(rij);
            double cbar = 0.5 * (ci + cj), rbar = 0.5 * (rhoi + rhoj);
            V3 vs = 0.5 * (vi + vj);
            vs += 0.5 * ((PL - PR) / (rbar * cbar)) * e;
            dRho += mj / rhoj * dot(vi - vs, dW);
        }
        if (!s.fd.prefix.empty())
            for (int k = i > 0 ? s.fd.prefix[i - 1] : 0; k < s.fd.prefix[i]; k++)
                dRho += sphBoundaryDrho(s, s.d, i, s.fd.pointing[k]);
        if (!s.fm.prefix.empty())
            for (int k = i > 0 ? s.fm.prefix[i - 1] : 0; k < s.fm.prefix[i]; k++)
                dRho += sphBoundaryDrho(s, s.mk, i, s.fm.pointing[k]);
        dRho *= 2.0 * rhoi;
        dr[i] = dRho;
    }
    for (size_t i = 0; i < N; i++) {
        s.f.drho[i] += dr[i] * dt;
        double ch = s.f.drho[i], r0 = s.f.rho0[i];
        if (ch < -0.1 * r0) ch = -0.1 * r0;
        s.f.rho[i] = ch + r0;
        s.f.p[i] = s.f.c[i] * s.f.c[i] * ch;
    }
}

// WCSPHSolver.h:607-621 loop body + launchWCSPH1st/2ndHalfIntegration
// (WCSPHIntegrationKernel.cu:308-472)
static void sphStep(SPH& s) {
    double dt = s.dt;
    s.iStep++;
    s.time += dt;
    sphNeighborSearch(s);
    size_t N = s.f.size();
    sphAccel(s, 0.5, true);
    for (size_t i = 0; i < N; i++) s.f.vel[i] += (0.5 * dt) * s.f.acc[i];
    for (size_t i = 0; i < N; i++) s.f.pos[i] += dt * s.f.vel[i];
    sphDensity(s, dt);
    sphAccel(s, 0.5, false);
    for (size_t i = 0; i < N; i++) s.f.vel[i] += (0.5 * dt) * s.f.acc[i];
}

// ------------------------------------------- particle-level coupling ----
// Marker offsets of a ball of radius R: shells l = 0, 1, ... at radius
// r_l = R - (l + 1/2) dx while l dx < 2 h and r_l > dx / 4, shell l carrying
// n_l = max(1, round(4 pi r_l^2 / dx^2)) points on the golden-angle spiral
// z_k = 1 - (2k + 1) / n_l, phi_k = k pi (3 - sqrt 5); a ball too small for
// any shell gets one marker at its centre.
static std::vector<V3> markerOffsets(double R, double dx, double h) {
    std::vector<V3> out;
    const double ga = PI * (3.0 - std::sqrt(5.0));
    for (int l = 0; l * dx < 2.0 * h; l++) {
        const double r = R - (l + 0.5) * dx;
        if (!(r > 0.25 * dx)) break;
        const long nl = std::max(1L, std::lround(4.0 * PI * r * r / (dx * dx)));
        for (long k = 0; k < nl; k++) {
            const double z = 1.0 - (2.0 * k + 1.0) / (double)nl;
            const double rho = std::sqrt(std::max(0.0, 1.0 - z * z));
            const double phi = ga * (double)k;
            out.push_back(v3(r * rho * std::cos(phi), r * rho * std::sin(phi), r * z));
        }
    }
    if (out.empty()) out.push_back(v3(0, 0, 0));
    return out;
}

// Markers at their balls' state: centre + offset, rigid velocity
// v + omega x offset, outward normal offset / |offset|.
static void placeMarkers(SPH& s, const DEM& d) {
    for (size_t k = 0; k < s.mk.size(); k++) {
        const int b = s.mkBall[k];
        const V3 o = s.mkOff[k];
        s.mk.pos[k] = d.pos[b] + o;
        s.mk.vel[k] = d.vel[b] + cross(d.w[b], o);
        const double l2 = dot(o, o);
        s.mk.normal[k] = l2 > 0.0 ? o * (1.0 / std::sqrt(l2)) : v3(0, 0, 0);
    }
}

// One coupled step: markers follow the balls, one fluid step with them,
// each ball's coupling force / torque = the sum of its markers' reactions
// (mean of the step's two acceleration passes), then `sub` DEM steps.
static void coupledStep(SPH& s, DEM& d, int sub) {
    placeMarkers(s, d);
    s.coupling = true;
    sphStep(s);
    s.coupling = false;
    d.cplF.assign(d.nb(), v3(0, 0, 0));
    d.cplT.assign(d.nb(), v3(0, 0, 0));
    for (size_t b = 0; b < s.body.size(); b++) {
        V3 F = v3(0, 0, 0), T = v3(0, 0, 0);
        for (int k = s.bodyStart[b]; k < s.bodyStart[b + 1]; k++) {
            F += s.mkF[k];
            T += cross(s.mkOff[k], s.mkF[k]);
        }
        d.cplF[s.body[b]] = F;
        d.cplT[s.body[b]] = T;
    }
    for (int k = 0; k < sub; k++) demStep(d);
}

static inline V3 ld3(const double* a, size_t i) { return v3(a[3 * i], a[3 * i + 1], a[3 * i + 2]); }
static inline void st3(double* a, size_t i, V3 v) { a[3 * i] = v.x; a[3 * i + 1] = v.y; a[3 * i + 2] = v.z; }

}  // namespace ora

using namespace ora;

extern "C" {

int oracle_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

// ------------------------------------------------------------------ DEM --
void* oracle_dem_create() { return new DEM(); }
void oracle_dem_destroy(void* h) { delete (DEM*)h; }

// DEMSolver.h:1637-1662
void oracle_dem_set_hertzian_pair(void* h, int a, int b, double E, double G, double e, double krks, double ktks,
                                  double mus, double mur, double mut) {
    Row r{a, b, {E, G, e, krks, ktks, mus, mur, mut, 0, 0, 0}};
    ((DEM*)h)->M.hrows.push_back(r);
}
// DEMSolver.h:1667-1700
void oracle_dem_set_linear_pair(void* h, int a, int b, double kn, double ks, double kr, double kt, double dn, double ds,
                                double dr, double dtt, double mus, double mur, double mut) {
    Row r{a, b, {kn, ks, kr, kt, dn, ds, dr, dtt, mus, mur, mut}};
    ((DEM*)h)->M.lrows.push_back(r);
}
// DEMSolver.h:1705-1726
void oracle_dem_set_bonded_pair(void* h, int a, int b, double gamma, double Eb, double knks, double sigma, double C,
                                double mu) {
    Row r{a, b, {gamma, Eb, knks, sigma, C, mu, 0, 0, 0, 0, 0}};
    ((DEM*)h)->M.brows.push_back(r);
}
// DEMSolver.h:1728-1768 (addBall / addFixedBall); density <= 0 with fixed=1 marks a fixed ball.
void oracle_dem_add_balls(void* h, long n, const double* pos, const double* vel, const double* w, const double* rad,
                          const double* dens, const int* mat, const int* clump, int fixed) {
    DEM& s = *(DEM*)h;
    for (long i = 0; i < n; i++) {
        s.pos.push_back(ld3(pos, i));
        s.vel.push_back(fixed ? v3(0, 0, 0) : ld3(vel, i));
        s.w.push_back(fixed ? v3(0, 0, 0) : ld3(w, i));
        s.force.push_back(v3(0, 0, 0));
        s.torque.push_back(v3(0, 0, 0));
        s.rad.push_back(rad[i]);
        double im = 0.0;
        if (!fixed) {
            double mass = 4. / 3. * rad[i] * rad[i] * rad[i] * PI * dens[i];
            if (mass > 0.0) im = 1.0 / mass;
        }
        s.invMass.push_back(im);
        s.mat.push_back(mat[i]);
        s.clump.push_back(clump ? clump[i] : -1);
    }
}
// DEMSolver.h:1796-1845
void oracle_dem_add_clump(void* h, long np, const double* pts, const double* rad, const double* centroid,
                          const double* vel, const double* w, double mass, const double* inertia, int mat) {
    DEM& s = *(DEM*)h;
    int cid = (int)s.clumps.size();
    int ps = (int)s.nb(), pe = ps + (int)np;
    V3 c = ld3(centroid, 0), v = ld3(vel, 0), ww = ld3(w, 0);
    std::vector<V3> pv(np, v);
    double vol = 0., im = 0.;
    if (mass > 1.e-20) {
        im = 1.0 / mass;
        for (long i = 0; i < np; i++) {
            vol += 4.0 / 3.0 * PI * std::pow(rad[i], 3.0);
            pv[i] += cross(ww, ld3(pts, i) - c);
        }
    }
    double dave = vol > 0. ? mass / vol : 0.;
    for (long i = 0; i < np; i++) {
        double d = dave;
        int cc = cid;
        oracle_dem_add_balls(h, 1, pts + 3 * i, &pv[i].x, &ww.x, rad + i, &d, &mat, &cc, 0);
    }
    SymM I{inertia[0], inertia[1], inertia[2], inertia[3], inertia[4], inertia[5]};
    s.clumps.add(c, v, ww, Quat{1, 0, 0, 0}, inverse(I), im, mat, ps, pe);
}
// DEMSolver.h:1882-1935 (Q8: velocity / angularVelocity ignored)
void oracle_dem_add_mesh_wall(void* h, long nv, const double* verts, long nt, const int* i0, const int* i1,
                              const int* i2, const double* pos, int mat) {
    DEM& s = *(DEM*)h;
    int vs = (int)s.vLocal.size();
    int wi = (int)s.walls.size();
    V3 p = ld3(pos, 0);
    s.walls.add(p, v3(0, 0, 0), v3(0, 0, 0), Quat{1, 0, 0, 0}, SymM{0, 0, 0, 0, 0, 0}, 0.0, mat, vs, vs + (int)nv);
    for (long i = 0; i < nv; i++) {
        s.vLocal.push_back(ld3(verts, i));
        s.vGlobal.push_back(ld3(verts, i) + p);
        s.vWall.push_back(wi);
    }
    for (long t = 0; t < nt; t++) {
        s.t0.push_back(vs + i0[t]); s.t1.push_back(vs + i1[t]); s.t2.push_back(vs + i2[t]);
        s.tWall.push_back(wi);
        s.tCenter.push_back(triangleCircumcenter(ld3(verts, i0[t]) + p, ld3(verts, i1[t]) + p, ld3(verts, i2[t]) + p));
    }
}
void oracle_dem_set_wall_motion(void* h, int wall, const double* vel, const double* w) {
    DEM& s = *(DEM*)h;
    s.walls.vel[wall] = ld3(vel, 0);
    s.walls.w[wall] = ld3(w, 0);
}
// DEMSolver.h:93-135 (bondedInteraction::add)
void oracle_dem_add_bonds(void* h, long n, const int* a0, const int* b0, const double* posHost, long npos) {
    DEM& s = *(DEM*)h;
    // bondedInteraction::add (DEMSolver.h:93-135) skips a pair that is already
    // bonded; its linear search is a set lookup here (same result)
    std::unordered_set<long long> have;
    for (size_t j = 0; j < s.bA.size(); j++) have.insert(((long long)s.bA[j] << 32) | (unsigned)s.bB[j]);
    for (long k = 0; k < n; k++) {
        int i0 = a0[k], i1 = b0[k];
        if (i0 < 0 || i1 < 0 || i0 >= npos || i1 >= npos || i0 == i1) continue;
        int a = std::min(i0, i1), b = std::max(i0, i1);
        if (!have.insert(((long long)a << 32) | (unsigned)b).second) continue;
        V3 pa = ld3(posHost, a), pb = ld3(posHost, b);
        s.bA.push_back(a); s.bB.push_back(b); s.bOk.push_back(1);
        s.bPoint.push_back(0.5 * (pa + pb)); s.bNormal.push_back(normalize(pa - pb));
        s.bFs.push_back(v3(0, 0, 0)); s.bTb.push_back(v3(0, 0, 0));
        s.bFn.push_back(0); s.bTt.push_back(0); s.bSmax.push_back(0); s.bTmax.push_back(0);
    }
}
void oracle_dem_set_buoyancy_drag(void* h, double rho, double Cd, const double* g, const double* u, double level) {
    DEM& s = *(DEM*)h;
    s.hasBuoy = true; s.buoyRho = rho; s.buoyCd = Cd; s.buoyG = ld3(g, 0); s.buoyU = ld3(u, 0); s.buoyLevel = level;
}
void oracle_dem_set_global_damping(void* h, double c) { ((DEM*)h)->dampCoeff = c; }
void oracle_dem_set_constant_force(void* h, long n, const double* f, double ramp) {
    DEM& s = *(DEM*)h;
    s.constForce.resize(n);
    for (long i = 0; i < n; i++) s.constForce[i] = ld3(f, i);
    s.constRamp = ramp;
}
// DEMSolver.h:245-276 + solve() initialisation (:1994-1997)
int oracle_dem_initialize(void* h, const double* mn, const double* mx, const double* g, double dt) {
    DEM& s = *(DEM*)h;
    s.M.build();
    s.gravity = ld3(g, 0);
    s.dt = dt;
    double cell = 0.0;
    for (double r : s.rad) cell = std::max(cell, r * 2.0);
    gridSet(s.ballGrid, ld3(mn, 0), ld3(mx, 0), cell);
    for (size_t t = 0; t < s.t0.size(); t++) {
        V3 a = s.vLocal[s.t0[t]], b = s.vLocal[s.t1[t]], c = s.vLocal[s.t2[t]];
        V3 cc = triangleCircumcenter(a, b, c);
        cell = std::max(cell, 2.0 * length(a - cc));
        cell = std::max(cell, 2.0 * length(b - cc));
        cell = std::max(cell, 2.0 * length(c - cc));
    }
    gridSet(s.triGrid, ld3(mn, 0), ld3(mx, 0), cell);
    if (!s.ballGrid.valid || s.nb() == 0) return 2;
    s.bb = Pairs();
    s.bt = Pairs();
    s.ghosts.clear();
    auto addGhost = [&](int x, int y, int z) {
        DEM::Ghost g;
        g.dx = x; g.dy = y; g.dz = z;
        s.ghosts.push_back(g);
    };
    if (s.perX) addGhost(1, 0, 0);
    if (s.perY) addGhost(0, 1, 0);
    if (s.perZ) addGhost(0, 0, 1);
    if (s.perX && s.perY) addGhost(1, 1, 0);
    if (s.perY && s.perZ) addGhost(0, 1, 1);
    if (s.perX && s.perZ) addGhost(1, 0, 1);
    if (s.perX && s.perY && s.perZ) addGhost(1, 1, 1);
    demNeighborSearch(s);
    demBallForces(s, 0.0);
    demTriangleForces(s, 0.0);
    s.iStep = 0;
    s.time = 0;
    s.initialized = true;
    return 0;
}
int oracle_dem_step(void* h, long n) {
    DEM& s = *(DEM*)h;
    if (!s.initialized) return 5;
    for (long k = 0; k < n; k++) demStep(s);
    return 0;
}
void oracle_dem_neighbor_search(void* h) { demNeighborSearch(*(DEM*)h); }
// calculateBallContactForceTorque(dt) then optionally addTriangleContactForceTorque(dtWall)
void oracle_dem_eval_forces(void* h, double dt, int walls, double dtWall) {
    DEM& s = *(DEM*)h;
    demBallForces(s, dt);
    if (walls) demTriangleForces(s, dtWall);
}
long oracle_dem_num_balls(void* h) { return (long)((DEM*)h)->nb(); }
void oracle_dem_set_periodic(void* h, int x, int y, int z) {
    DEM& s = *(DEM*)h;
    if (x) s.perX = true;
    if (y) s.perY = true;
    if (z) s.perZ = true;
}
long oracle_dem_num_ghost_pairs(void* h, int set) {
    DEM& s = *(DEM*)h;
    return set >= 0 && set < (int)s.ghosts.size() ? (long)s.ghosts[set].p.n : 0;
}
void oracle_dem_get_ghost_pairs(void* h, int set, int* a, int* b, double* sl, double* force) {
    DEM& s = *(DEM*)h;
    if (set < 0 || set >= (int)s.ghosts.size()) return;
    Pairs& p = s.ghosts[set].p;
    for (size_t k = 0; k < p.n; k++) {
        if (a) a[k] = p.pointed[k];
        if (b) b[k] = p.pointing[k];
        if (sl) st3(sl, k, p.sl[k]);
        if (force) st3(force, k, p.cforce[k]);
    }
}
long oracle_dem_num_pairs(void* h) { return (long)((DEM*)h)->bb.n; }
long oracle_dem_num_wall_pairs(void* h) { return (long)((DEM*)h)->bt.n; }
long oracle_dem_num_bonds(void* h) { return (long)((DEM*)h)->bA.size(); }
long oracle_dem_step_index(void* h) { return ((DEM*)h)->iStep; }
void oracle_dem_get_balls(void* h, double* pos, double* vel, double* w, double* force, double* torque) {
    DEM& s = *(DEM*)h;
    for (size_t i = 0; i < s.nb(); i++) {
        if (pos) st3(pos, i, s.pos[i]);
        if (vel) st3(vel, i, s.vel[i]);
        if (w) st3(w, i, s.w[i]);
        if (force) st3(force, i, s.force[i]);
        if (torque) st3(torque, i, s.torque[i]);
    }
}
void oracle_dem_set_balls(void* h, const double* pos, const double* vel, const double* w) {
    DEM& s = *(DEM*)h;
    for (size_t i = 0; i < s.nb(); i++) {
        if (pos) s.pos[i] = ld3(pos, i);
        if (vel) s.vel[i] = ld3(vel, i);
        if (w) s.w[i] = ld3(w, i);
    }
}
// which: 0 ball-ball, 1 ball-triangle
void oracle_dem_get_pairs(void* h, int which, int* a, int* b, double* sl, double* ro, double* to, double* force,
                          double* torque, double* point, double* overlap) {
    DEM& s = *(DEM*)h;
    Pairs& p = which ? s.bt : s.bb;
    for (size_t k = 0; k < p.n; k++) {
        if (a) a[k] = p.pointed[k];
        if (b) b[k] = p.pointing[k];
        if (sl) st3(sl, k, p.sl[k]);
        if (ro) st3(ro, k, p.ro[k]);
        if (to) st3(to, k, p.to[k]);
        if (force) st3(force, k, p.cforce[k]);
        if (torque) st3(torque, k, p.ctorque[k]);
        if (point) st3(point, k, p.cpoint[k]);
        if (overlap) overlap[k] = p.overlap[k];
    }
}
// Carry springs from a caller-supplied pair list into the current ball-ball
// list (the writeBallInteractionsKernel carry rule, ballNeighborSearchKernel.cu:130-143).
void oracle_dem_import_springs(void* h, long n, const int* a, const int* b, const double* sl, const double* ro,
                               const double* to) {
    DEM& s = *(DEM*)h;
    Pairs& p = s.bb;
    for (size_t k = 0; k < p.n; k++) {
        for (long j = 0; j < n; j++) {
            if (a[j] == p.pointed[k] && b[j] == p.pointing[k]) {
                p.sl[k] = ld3(sl, j); p.ro[k] = ld3(ro, j); p.to[k] = ld3(to, j);
                break;
            }
        }
    }
}
void oracle_dem_get_bonds(void* h, int* a, int* b, int* ok, double* fn, double* tt, double* fs, double* tb,
                          double* normal, double* point) {
    DEM& s = *(DEM*)h;
    for (size_t k = 0; k < s.bA.size(); k++) {
        if (a) a[k] = s.bA[k];
        if (b) b[k] = s.bB[k];
        if (ok) ok[k] = s.bOk[k];
        if (fn) fn[k] = s.bFn[k];
        if (tt) tt[k] = s.bTt[k];
        if (fs) st3(fs, k, s.bFs[k]);
        if (tb) st3(tb, k, s.bTb[k]);
        if (normal) st3(normal, k, s.bNormal[k]);
        if (point) st3(point, k, s.bPoint[k]);
    }
}
long oracle_dem_num_clumps(void* h) { return (long)((DEM*)h)->clumps.size(); }
void oracle_dem_get_clumps(void* h, double* pos, double* vel, double* w, double* q) {
    DEM& s = *(DEM*)h;
    for (size_t c = 0; c < s.clumps.size(); c++) {
        if (pos) st3(pos, c, s.clumps.pos[c]);
        if (vel) st3(vel, c, s.clumps.vel[c]);
        if (w) st3(w, c, s.clumps.w[c]);
        if (q) { q[4 * c] = s.clumps.q[c].q0; q[4 * c + 1] = s.clumps.q[c].q1; q[4 * c + 2] = s.clumps.q[c].q2; q[4 * c + 3] = s.clumps.q[c].q3; }
    }
}
long oracle_dem_num_walls(void* h) { return (long)((DEM*)h)->walls.size(); }
void oracle_dem_get_walls(void* h, double* pos, double* q, double* vglobal) {
    DEM& s = *(DEM*)h;
    for (size_t c = 0; c < s.walls.size(); c++) {
        if (pos) st3(pos, c, s.walls.pos[c]);
        if (q) { q[4 * c] = s.walls.q[c].q0; q[4 * c + 1] = s.walls.q[c].q1; q[4 * c + 2] = s.walls.q[c].q2; q[4 * c + 3] = s.walls.q[c].q3; }
    }
    if (vglobal) for (size_t v = 0; v < s.vGlobal.size(); v++) st3(vglobal, v, s.vGlobal[v]);
}

// ---------------------------------------------------------------- WCSPH --
void* oracle_sph_create() { return new SPH(); }
void oracle_sph_destroy(void* h) { delete (SPH*)h; }
// WCSPHSolver.h:523-541 (addSPH / addDummy)
void oracle_sph_add(void* h, int dummy, long n, const double* pos, const double* vel, const double* c,
                    const double* spacing, const double* dens, const double* visc) {
    SPH& s = *(SPH*)h;
    SPHSet& t = dummy ? s.d : s.f;
    for (long i = 0; i < n; i++) t.add(ld3(pos, i), ld3(vel, i), c[i], spacing[i], dens[i], visc[i]);
}
// WCSPHSolver.h:127-147
int oracle_sph_initialize(void* h, const double* mn, const double* mx, const double* g, double dt) {
    SPH& s = *(SPH*)h;
    s.gravity = ld3(g, 0);
    s.dt = dt;
    double cell = 0.0;
    for (double x : s.f.h) cell = std::max(cell, x * 2.0);
    for (double x : s.d.h) cell = std::max(cell, x * 2.0);
    gridSet(s.grid, ld3(mn, 0), ld3(mx, 0), cell);
    if (!s.grid.valid) return 2;
    sphInitBoundary(s);
    s.initialized = true;
    return 0;
}
int oracle_sph_step(void* h, long n) {
    SPH& s = *(SPH*)h;
    if (!s.initialized) return 5;
    for (long k = 0; k < n; k++) sphStep(s);
    return 0;
}
void oracle_sph_neighbor_search(void* h) { sphNeighborSearch(*(SPH*)h); }
void oracle_sph_eval_accel(void* h) { sphAccel(*(SPH*)h); }
void oracle_sph_eval_density(void* h, double dt) { sphDensity(*(SPH*)h, dt); }
long oracle_sph_num(void* h, int dummy) { SPH& s = *(SPH*)h; return (long)(dummy ? s.d.size() : s.f.size()); }
long oracle_sph_num_pairs(void* h, int which) {
    SPH& s = *(SPH*)h;
    const CSR& c = which == 0 ? s.ff : (which == 1 ? s.fd : s.dd);
    return (long)c.pointing.size();
}
void oracle_sph_get_pairs(void* h, int which, int* a, int* b) {
    SPH& s = *(SPH*)h;
    const CSR& c = which == 0 ? s.ff : (which == 1 ? s.fd : s.dd);
    for (size_t k = 0; k < c.pointing.size(); k++) { a[k] = c.pointed[k]; b[k] = c.pointing[k]; }
}
void oracle_sph_get(void* h, int dummy, double* pos, double* vel, double* acc, double* rho, double* p, double* drho,
                    double* normal) {
    SPH& s = *(SPH*)h;
    SPHSet& t = dummy ? s.d : s.f;
    for (size_t i = 0; i < t.size(); i++) {
        if (pos) st3(pos, i, t.pos[i]);
        if (vel) st3(vel, i, t.vel[i]);
        if (acc) st3(acc, i, t.acc[i]);
        if (rho) rho[i] = t.rho[i];
        if (p) p[i] = t.p[i];
        if (drho) drho[i] = t.drho[i];
        if (normal) st3(normal, i, t.normal[i]);
    }
}
// Particle-level coupling (no reference counterpart): markers for balls[0..n)
// of the DEM scene, placed at the balls' current state.
int oracle_sph_couple_balls(void* h, void* dem, long n, const int* balls, double dx, double hm, double c, double nu,
                            double rho0) {
    SPH& s = *(SPH*)h;
    DEM& d = *(DEM*)dem;
    for (long k = 0; k < n; k++) {
        const int b = balls[k];
        if (b < 0 || (size_t)b >= d.nb()) return 1;
        for (const V3& o : markerOffsets(d.rad[b], dx, hm)) {
            s.mk.pos.push_back(v3(0, 0, 0)); s.mk.vel.push_back(v3(0, 0, 0));
            s.mk.acc.push_back(v3(0, 0, 0)); s.mk.normal.push_back(v3(0, 0, 0));
            s.mk.drho.push_back(0.0); s.mk.rho.push_back(rho0); s.mk.p.push_back(0.0); s.mk.rho0.push_back(rho0);
            s.mk.h.push_back(hm); s.mk.m.push_back(rho0 * dx * dx * dx); s.mk.c.push_back(c); s.mk.nu.push_back(nu);
            s.mkBall.push_back(b);
            s.mkOff.push_back(o);
        }
        s.body.push_back(b);
        s.bodyStart.push_back((int)s.mkBall.size());
    }
    s.mkF.assign(s.mk.size(), v3(0, 0, 0));
    placeMarkers(s, d);
    return 0;
}
int oracle_couple_step(void* h, void* dem, long n, int sub) {
    SPH& s = *(SPH*)h;
    DEM& d = *(DEM*)dem;
    if (!s.initialized || !d.initialized) return 5;
    for (long k = 0; k < n; k++) coupledStep(s, d, sub);
    return 0;
}
long oracle_sph_num_markers(void* h) { return (long)((SPH*)h)->mk.size(); }
void oracle_sph_get_markers(void* h, double* pos, double* vel, double* normal, double* force, int* ball) {
    SPH& s = *(SPH*)h;
    for (size_t k = 0; k < s.mk.size(); k++) {
        if (pos) st3(pos, k, s.mk.pos[k]);
        if (vel) st3(vel, k, s.mk.vel[k]);
        if (normal) st3(normal, k, s.mk.normal[k]);
        if (force) st3(force, k, s.mkF[k]);
        if (ball) ball[k] = s.mkBall[k];
    }
}
void oracle_sph_get_coupling(void* h, void* dem, int* ball, double* force, double* torque) {
    SPH& s = *(SPH*)h;
    DEM& d = *(DEM*)dem;
    for (size_t b = 0; b < s.body.size(); b++) {
        const int i = s.body[b];
        if (ball) ball[b] = i;
        if (force) st3(force, b, i < (int)d.cplF.size() ? d.cplF[i] : v3(0, 0, 0));
        if (torque) st3(torque, b, i < (int)d.cplT.size() ? d.cplT[i] : v3(0, 0, 0));
    }
}
void oracle_sph_set(void* h, const double* pos, const double* vel, const double* rho, const double* p,
                    const double* drho) {
    SPH& s = *(SPH*)h;
    for (size_t i = 0; i < s.f.size(); i++) {
        if (pos) s.f.pos[i] = ld3(pos, i);
        if (vel) s.f.vel[i] = ld3(vel, i);
        if (rho) s.f.rho[i] = rho[i];
        if (p) s.f.p[i] = p[i];
        if (drho) s.f.drho[i] = drho[i];
    }
}

}  // extern "C"
