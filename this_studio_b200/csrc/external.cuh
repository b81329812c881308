// Force terms of the reference's user hooks (DEMSPH/externalForceTorque.cu),
// shared by the fused per-ball finish of a force evaluation (dem.cu) and the
// reference-signature launchers (external.cu).
#pragma once
#include "common.cuh"

namespace demsph {

// addBuoyancyDragKernel (externalForceTorque.cu:79-133) for one sphere:
// buoyancy of the volume below the plane z = level (spherical cap,
// sphereSubmergedVolumePlaneZ, :66-77) plus quadratic drag against a uniform
// current, scaled by the submerged fraction.  Returns the force to add; zero
// when the sphere is dry.
__host__ __device__ __forceinline__ double3 buoyancy_drag(double3 ri, double3 vi, double r, double rho, double cd,
                                                          double3 g, double3 u, double level) {
    double dd = level - ri.z;
    double Vsub;
    if (dd <= -r) Vsub = 0.0;
    else if (dd >= r) Vsub = (4.0 / 3.0) * kPi * r * r * r;
    else { double h = dd + r; Vsub = (kPi * h * h * (3.0 * r - h)) / 3.0; }
    if (!(Vsub > 0.0)) return mk3(0, 0, 0);
    double3 Fb = mk3(-rho * Vsub * g.x, -rho * Vsub * g.y, -rho * Vsub * g.z);
    double Vs = (4.0 / 3.0) * kPi * r * r * r;
    double alpha = (Vs > 1.e-30) ? (Vsub / Vs) : 0.0;
    double3 vr = vi - u;
    double v2 = dot(vr, vr);
    double3 Fdr = mk3(0, 0, 0);
    if (v2 > 1.e-30 && cd > 0.0) {
        double vm = sqrt(v2);
        double Aeff = alpha * (kPi * r * r);
        double kk = 0.5 * rho * cd * Aeff * vm;
        Fdr = mk3(-kk * vr.x, -kk * vr.y, -kk * vr.z);
    }
    return mk3(Fb.x + Fdr.x, Fb.y + Fdr.y, Fb.z + Fdr.z);
}

}  // namespace demsph
