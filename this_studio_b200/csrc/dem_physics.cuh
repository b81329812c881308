// Device physics of the DEM path: material table, contact laws (linear,
// Hertz-Mindlin), parallel bond, sphere-triangle classification and rigid
// body helpers.  Each function states the reference lines it restates.
#pragma once
#include "common.cuh"

namespace demsph {

// --------------------------------------------------------- material table --
// One entry per symmetric material pair, indexed like the reference's packed
// tables (contactParameters.h:123-141).  The entry carries the model choice
// (linear when k_n > 1e-20, else Hertz-Mindlin: contactKernel.cu:218-252) and
// the Hertz damping ratio D = -ln e / sqrt(ln^2 e + pi^2) (contactKernel.cu:239-240),
// precomputed once instead of per pair.
struct MatPair {
    int linear;
    int pad;
    // linear (contactParameters.h:75-89)
    double kn, ks, kr, kt, dn, ds, dr, dt;
    // Hertz-Mindlin (contactParameters.h:62-73)
    double E, G, D, krks, ktks;
    // friction (the active model's)
    double mus, mur, mut;
    // parallel bond (contactParameters.h:91-100)
    double gamma, Eb, knks, sigma, C, mu;
};

__host__ __device__ __forceinline__ int pair_param_index(int a, int b, int nMat, int cap) {
    if (nMat <= 0 || cap <= 0) return 0;
    if (a < 0 || b < 0 || a >= nMat || b >= nMat) return cap - 1;
    int i = a, j = b;
    if (i > j) { int t = i; i = j; j = t; }
    long long idx = ((long long)i * (2LL * nMat - i + 1LL)) / 2LL + (long long)(j - i);
    if (idx < 0) idx = 0;
    if (idx >= cap) idx = cap - 1;
    return (int)idx;
}

// --------------------------------------------------------------- springs ---
// integrateSlidingOrRollingSpring (contactKernel.cuh:64-97).  The spring is
// accumulated in FP64; the trial force for the Coulomb cap uses R.
template <class R>
__host__ __device__ __forceinline__ double3 spring_slide(double3 sp, V<R> sv, double3 n, V<R> Fn, R mu, R k, R c, double dt) {
    double3 s = mk3(0, 0, 0);
    if (k > (R)0) {
        double3 s1 = sp - dot(sp, n) * n;
        double a1 = len(s1);
        if (a1 > 1.e-10) s1 *= len(sp) / a1;
        s = s1 + up(sv) * dt;
        if (mu > (R)0) {
            V<R> fs = -(cvt<R>(s) * k) - sv * c;
            R af = rlen(fs), an = rlen(Fn);
            if (af > mu * an) {
                R ratio = mu * an / af;
                fs = fs * ratio;
                s = -(up(fs) + up(sv * c)) / (double)k;
            }
        }
    }
    return s;
}
// integrateTorsionSpring (contactKernel.cuh:99-126)
template <class R>
__host__ __device__ __forceinline__ double3 spring_torsion(double3 sp, V<R> tv, double3 n, V<R> Fn, R mu, R k, R c, double dt) {
    double3 s = mk3(0, 0, 0);
    if (k > (R)0) {
        s = dot(sp + up(tv) * dt, n) * n;
        if (mu > (R)0) {
            V<R> fs = -(cvt<R>(s) * k) - tv * c;
            R af = rlen(fs), an = rlen(Fn);
            if (af > mu * an) {
                R ratio = mu * an / af;
                fs = fs * ratio;
                s = -(up(fs) + up(tv * c)) / (double)k;
            }
        }
    }
    return s;
}

// LinearContact / HertzianMindlinContact (contactKernel.cuh:128-290) after
// the model's stiffness and damping have been formed.  Geometry (n, delta)
// and relative velocities arrive in FP64; R is the arithmetic of the law.
template <class R>
__host__ __device__ __forceinline__ void law_tail(V<R>& F, V<R>& T, double3& es, double3& er, double3& et, double3 vc,
                                         double3 wij, double3 n, R delta, R Rad, double dt, R kn, R ks, R kr, R kt,
                                         R cn, R cs, R cr, R ct, R mus, R mur, R mut, bool roll, bool tors) {
    V<R> nr = cvt<R>(n);
    V<R> vcr = cvt<R>(vc);
    V<R> vn = dot(vcr, nr) * nr;
    V<R> Fn = kn * delta * nr - vn * cn;
    V<R> vs = vcr - vn;
    es = spring_slide<R>(es, vs, n, Fn, mus, ks, cs, dt);
    V<R> Fs = -(ks * cvt<R>(es)) - cs * vs;
    F = Fn + Fs;
    T = v3r<R>(0, 0, 0);
    if (roll) {
        V<R> wr = cvt<R>(wij);
        V<R> vr = -Rad * cross(nr, wr);
        er = spring_slide<R>(er, vr, n, Fn, mur, kr, cr, dt);
        V<R> Fr = -(kr * cvt<R>(er)) - cr * vr;
        T = Rad * cross(nr, Fr);
    }
    if (tors) {
        V<R> wr = cvt<R>(wij);
        R D2 = (R)2 * Rad;
        V<R> vt = D2 * dot(wr, nr) * nr;
        et = spring_torsion<R>(et, vt, n, Fn, mut, kt, ct, dt);
        V<R> Ft = -(kt * cvt<R>(et)) - ct * vt;
        T += D2 * Ft;
    }
}

// calBallContactForceTorqueKernel's law selection (contactKernel.cu:218-252)
// with LinearContact (contactKernel.cuh:128-207) / HertzianMindlinContact (:209-290).
// roll / tors skip the rolling and torsion springs when no material pair of
// the scene has a rolling / torsion stiffness (their springs then stay zero,
// which is what the reference computes for k = 0).
template <class R>
__host__ __device__ __forceinline__ void contact_law(const MatPair& mp, V<R>& F, V<R>& T, double3& es, double3& er, double3& et,
                                            double3 vc, double3 wij, double3 n, double delta, double m, double Rad,
                                            double dt, bool roll, bool tors) {
    F = v3r<R>(0, 0, 0);
    T = v3r<R>(0, 0, 0);
    if (!(delta > 0)) {
        es = er = et = mk3(0, 0, 0);
        return;
    }
    if (mp.linear) {
        R kn = (R)mp.kn, ks = (R)mp.ks, kr = (R)mp.kr, kt = (R)mp.kt, mr = (R)m;
        R cn = (R)2 * (R)mp.dn * rsq(mr * kn);
        R cs = (R)2 * (R)mp.ds * rsq(mr * ks);
        R cr = (R)2 * (R)mp.dr * rsq(mr * kr);
        R ct = (R)2 * (R)mp.dt * rsq(mr * kt);
        law_tail<R>(F, T, es, er, et, vc, wij, n, (R)delta, (R)Rad, dt, kn, ks, kr, kt, cn, cs, cr, ct, (R)mp.mus,
                    (R)mp.mur, (R)mp.mut, roll, tors);
    } else {
        R sq = rsq((R)Rad * (R)delta);
        R kn = (R)(4. / 3.) * (R)mp.E * sq;
        R ks = (R)8 * (R)mp.G * sq;
        R s56 = rsq((R)(5. / 6.));
        R mr = (R)m, D = (R)mp.D;
        R cn = (R)2 * s56 * D * rsq(mr * kn);
        R cs = (R)2 * s56 * D * rsq(mr * ks);
        R kr = ks * (R)mp.krks, kt = ks * (R)mp.ktks;
        R cr = (R)2 * s56 * D * rsq(mr * kr);
        R ct = (R)2 * s56 * D * rsq(mr * kt);
        law_tail<R>(F, T, es, er, et, vc, wij, n, (R)delta, (R)Rad, dt, kn, ks, kr, kt, cn, cs, cr, ct, (R)mp.mus,
                    (R)mp.mur, (R)mp.mut, roll, tors);
    }
}

// Rodrigues rotation (myVec.h:134-176)
__device__ __forceinline__ double3 rotate_vector(double3 v, double3 ang) {
    double a2 = dot(ang, ang);
    if (a2 < 1.0e-20) return v;
    double a = sqrt(a2);
    double s, c;
    sincos(a, &s, &c);
    double inv = 1.0 / a;
    double3 k = mk3(ang.x * inv, ang.y * inv, ang.z * inv);
    double kv = k.x * v.x + k.y * v.y + k.z * v.z;
    double3 kxv = mk3(k.y * v.z - k.z * v.y, k.z * v.x - k.x * v.z, k.x * v.y - k.y * v.x);
    double t3 = kv * (1.0 - c);
    return mk3(v.x * c + kxv.x * s + k.x * t3, v.y * c + kxv.y * s + k.y * t3, v.z * c + kxv.z * s + k.z * t3);
}

// ParallelBondedContact (contactKernel.cuh:4-62); bond state stays FP64.
__device__ __forceinline__ int parallel_bond(double& Fn, double& Tt, double3& Fs, double3& Tb, double& smax,
                                             double& tmax, double3 n0, double3 n, double3 vc, double3 wA, double3 wB,
                                             double rA, double rB, double dt, const MatPair& mp) {
    double3 th1 = cross(n0, n);
    Fs = rotate_vector(Fs, th1);
    Tb = rotate_vector(Tb, th1);
    double3 th2 = dot(0.5 * (wA + wB) * dt, n) * n;
    Fs = rotate_vector(Fs, th2);
    Tb = rotate_vector(Tb, th2);
    double rmin = rA < rB ? rA : rB;
    double Rb = mp.gamma * rmin;
    double A = Rb * Rb * kPi;
    double I = Rb * Rb * Rb * Rb / 4. * kPi;
    double J = 2 * I;
    double knA = mp.Eb / (rA + rB);
    double ksA = knA / mp.knks;
    double3 dn = dot(vc, n) * n * dt;
    double3 dtr = vc * dt - dn;
    Fn -= dot(dn * knA * A, n);
    Fs -= dtr * ksA * A;
    double3 wr = wA - wB;
    double3 rn = dot(wr, n) * n * dt;
    double3 rt = wr * dt - rn;
    Tt -= dot(rn * ksA * J, n);
    Tb -= rt * knA * I;
    smax = -Fn / A + len(Tb) / I * Rb;
    tmax = len(Fs) / A + fabs(Tt) / J * Rb;
    int ok = 1;
    if (mp.sigma > 0 && smax > mp.sigma) ok = 0;
    else if (mp.C > 0 && tmax > mp.C - mp.mu * smax) ok = 0;
    return ok;
}

// ------------------------------------------------------ sphere/triangle ---
enum : int { kCtNone = 0, kCtFace = 1, kCtEdge = 2, kCtVertex = 3 };
__host__ __device__ __forceinline__ double clamp01(double x) { return x < 0.0 ? 0.0 : (x > 1.0 ? 1.0 : x); }
__host__ __device__ __forceinline__ double dist2(double3 a, double3 b) { double3 d = a - b; return dot(d, d); }
// closestPointOnSegment (contactKernel.cuh:315-330)
__host__ __device__ __forceinline__ double3 closest_on_segment(double3 a, double3 b, double3 p, double& t) {
    double3 ab = b - a;
    double ab2 = dot(ab, ab);
    if (ab2 <= 1e-30) { t = 0.0; return a; }
    t = clamp01(dot(p - a, ab) / ab2);
    return a + ab * t;
}
// classifySphereTriangleContact (contactKernel.cuh:367-501): Ericson's
// Voronoi-region closest point; degenerate triangles as three segments.
__host__ __device__ __forceinline__ int classify_sphere_triangle(double3 c, double r, double3 v0, double3 v1, double3 v2,
                                                        double3& cp) {
    double r2 = r * r;
    double eps2 = 1e-12 * fmax(1.0, r2);
    double3 ab = v1 - v0, ac = v2 - v0;
    double3 nn = cross(ab, ac);
    if (dot(nn, nn) <= 1e-20) {
        double t01, t02, t12;
        double3 q01 = closest_on_segment(v0, v1, c, t01);
        double3 q02 = closest_on_segment(v0, v2, c, t02);
        double3 q12 = closest_on_segment(v1, v2, c, t12);
        double dmin = dist2(c, q01);
        cp = q01;
        int type = (t01 > 0.0 && t01 < 1.0) ? kCtEdge : kCtVertex;
        double d02 = dist2(c, q02);
        if (d02 < dmin) { dmin = d02; cp = q02; type = (t02 > 0.0 && t02 < 1.0) ? kCtEdge : kCtVertex; }
        double d12 = dist2(c, q12);
        if (d12 < dmin) { dmin = d12; cp = q12; type = (t12 > 0.0 && t12 < 1.0) ? kCtEdge : kCtVertex; }
        return (dmin <= r2 + eps2) ? type : kCtNone;
    }
    double3 ap = c - v0;
    double d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) { cp = v0; return dist2(c, v0) <= r2 + eps2 ? kCtVertex : kCtNone; }
    double3 bp = c - v1;
    double d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0 && d4 <= d3) { cp = v1; return dist2(c, v1) <= r2 + eps2 ? kCtVertex : kCtNone; }
    double vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
        double t = d1 / (d1 - d3);
        cp = v0 + ab * t;
        return dist2(c, cp) <= r2 + eps2 ? kCtEdge : kCtNone;
    }
    double3 cpv = c - v2;
    double d5 = dot(ab, cpv), d6 = dot(ac, cpv);
    if (d6 >= 0.0 && d5 <= d6) { cp = v2; return dist2(c, v2) <= r2 + eps2 ? kCtVertex : kCtNone; }
    double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
        double t = d2 / (d2 - d6);
        cp = v0 + ac * t;
        return dist2(c, cp) <= r2 + eps2 ? kCtEdge : kCtNone;
    }
    double va = d3 * d6 - d5 * d4;
    if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
        double t = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        cp = v1 + (v2 - v1) * t;
        return dist2(c, cp) <= r2 + eps2 ? kCtEdge : kCtNone;
    }
    double sum = va + vb + vc;
    if (fabs(sum) <= 1e-30) return kCtNone;
    double inv = 1.0 / sum;
    double v = vb * inv, w = vc * inv;
    cp = v0 + ab * v + ac * w;
    return dist2(c, cp) <= r2 + eps2 ? kCtFace : kCtNone;
}

// ------------------------------------------------------------ rigid body ---
// quaternionRotate (myQua.h:77-92); q stored as double4 (q0, q1, q2, q3).
__host__ __device__ __forceinline__ double4 quat_rotate(double4 q, double3 w, double dt) {
    double3 v = w * (0.5 * dt);
    double d0 = -q.y * v.x - q.z * v.y - q.w * v.z;
    double d1 = q.x * v.x + q.w * v.y - q.z * v.z;
    double d2 = -q.w * v.x + q.x * v.y + q.y * v.z;
    double d3 = q.z * v.x - q.y * v.y + q.x * v.z;
    double4 r = make_double4(q.x + d0, q.y + d1, q.z + d2, q.w + d3);
    double l2 = r.x * r.x + r.y * r.y + r.z * r.z + r.w * r.w;
    if (l2 < 1.0e-20) return r;
    double inv = 1.0 / sqrt(l2);
    return make_double4(r.x * inv, r.y * inv, r.z * inv, r.w * inv);
}
// rotateVectorByQuaternion (myQua.h:103-113)
__host__ __device__ __forceinline__ double3 quat_apply(double4 q, double3 v) {
    double3 qv = mk3(q.y, q.z, q.w);
    double3 t = cross(qv, v) * 2.0;
    return v + (t * q.x) + cross(qv, t);
}
// triangleCircumcenter (wallIntegrationKernel.cuh:4-29)
__host__ __device__ __forceinline__ double3 circumcenter(double3 a, double3 b, double3 c) {
    double3 ab = b - a, ac = c - a;
    double3 n = cross(ab, ac);
    double n2 = dot(n, n);
    if (n2 < 1e-30) return (a + b + c) / 3.0;
    double3 t1 = cross(n, ab) * dot(ac, ac);
    double3 t2 = cross(ac, n) * dot(ab, ab);
    double inv = 1.0 / (2.0 * n2);
    return a + (t1 + t2) * inv;
}
// rotateInverseInertiaTensor (myMat.h:107-158) applied to a vector:
// (R invI R^T) T with invI given as (xx, yy, zz, xy) + (xz, yz).
__device__ __forceinline__ double3 rot_inv_inertia_apply(double4 q, double4 Ia, double4 Ib, double3 t) {
    double q0 = q.x, q1 = q.y, q2 = q.z, q3 = q.w;
    double xx = Ia.x, yy = Ia.y, zz = Ia.z, xy = Ia.w, xz = Ib.x, yz = Ib.y;
    double q11 = 2 * q1 * q1, q22 = 2 * q2 * q2, q33 = 2 * q3 * q3;
    double a = 1.0 - q22 - q33, b = 2 * (q1 * q2 - q0 * q3), c = 2 * (q1 * q3 + q0 * q2);
    double d = 2 * (q1 * q2 + q0 * q3), e = 1.0 - q11 - q33, f = 2 * (q2 * q3 - q0 * q1);
    double g = 2 * (q1 * q3 - q0 * q2), h = 2 * (q2 * q3 + q0 * q1), i = 1.0 - q11 - q22;
    double r0x = xx * a + xy * b + xz * c, r0y = xy * a + yy * b + yz * c, r0z = xz * a + yz * b + zz * c;
    double r1x = xx * d + xy * e + xz * f, r1y = xy * d + yy * e + yz * f, r1z = xz * d + yz * e + zz * f;
    double r2x = xx * g + xy * h + xz * i, r2y = xy * g + yy * h + yz * i, r2z = xz * g + yz * h + zz * i;
    double mxx = r0x * a + r0y * b + r0z * c, myy = r1x * d + r1y * e + r1z * f, mzz = r2x * g + r2y * h + r2z * i;
    double mxy = r0x * d + r0y * e + r0z * f, mxz = r0x * g + r0y * h + r0z * i, myz = r1x * g + r1y * h + r1z * i;
    return mk3(mxx * t.x + mxy * t.y + mxz * t.z, mxy * t.x + myy * t.y + myz * t.z, mxz * t.x + myz * t.y + mzz * t.z);
}

}  // namespace demsph
