// The reference's user-force launchers with their exact C signatures
// (DEMSPH/externalForceTorque.h:6-36), so addExternalForceTorque hooks
// written for the reference call them unchanged.  They work on ball arrays in
// the reference's layout (one double3 per ball for force, torque, position,
// velocity, angular velocity; one double per ball for radius and inverse
// mass): the arrays an external-force callback of this library receives
// (demsph_dem_hook_arrays), or any caller's arrays of that layout.  Behaviour
// follows DEMSPH/externalForceTorque.cu:
//   launchAddConstantForce             force[i] += force_external[i]      (:4-24)
//   launchAddGlobalDampingForceTorque  force[i] -= c |force[i]| v_hat,
//                                      torque[i] -= c |torque[i]| w_hat   (:26-57)
//   launchAddBuoyancyDrag              buoyancy below the plane z = waterLevel
//                                      plus quadratic drag; balls with inverse
//                                      mass <= 0 are skipped             (:59-160)
// The launch geometry is chosen here (gridD / blockD are accepted and
// ignored).  Like the reference they return void; a launch failure is
// recorded for demsph_last_error().
#include <atomic>

#include "external.cuh"

namespace demsph {

extern std::atomic<long long> g_launches;

static __global__ void k_ext_constant(double3* __restrict__ force, const double3* __restrict__ fe, size_t n) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    force[i] = force[i] + fe[i];
}

static __global__ void k_ext_damping(double3* __restrict__ force, double3* __restrict__ torque,
                                     const double3* __restrict__ v, const double3* __restrict__ w, double c,
                                     size_t n) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double3 f = force[i], t = torque[i];
    force[i] = f - c * len(f) * normalize(v[i]);
    torque[i] = t - c * len(t) * normalize(w[i]);
}

static __global__ void k_ext_buoyancy(double3* __restrict__ force, const double3* __restrict__ pos,
                                      const double3* __restrict__ vel, const double* __restrict__ rad,
                                      const double* __restrict__ invm, double rho, double cd, double3 g, double3 u,
                                      double level, size_t n) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (invm && invm[i] <= 0.0) return;
    const double3 F = buoyancy_drag(pos[i], vel[i], rad[i], rho, cd, g, u, level);
    double3 f = force[i];
    f.x += F.x;
    f.y += F.y;
    f.z += F.z;
    force[i] = f;
}

static void after_launch() {
    g_launches += 1;
    DEMSPH_LAUNCH_CHECK();
}

}  // namespace demsph

using namespace demsph;

extern "C" {

void launchAddConstantForce(double3* force, const double3* force_external, const size_t num, const size_t gridD,
                            const size_t blockD, cudaStream_t stream) {
    (void)gridD;
    (void)blockD;
    guarded([&] {
        if (num == 0) return;
        if (!force || !force_external) throw Status(DEMSPH_ERR_INVALID, "launchAddConstantForce: null array");
        k_ext_constant<<<grid_for(num, 256), 256, 0, stream>>>(force, force_external, num);
        after_launch();
    });
}

void launchAddGlobalDampingForceTorque(double3* force, double3* torque, const double3* velocity,
                                       const double3* angularVelocity, const double dampCoeff, const size_t num,
                                       const size_t gridD, const size_t blockD, cudaStream_t stream) {
    (void)gridD;
    (void)blockD;
    guarded([&] {
        if (num == 0) return;
        if (!force || !torque || !velocity || !angularVelocity)
            throw Status(DEMSPH_ERR_INVALID, "launchAddGlobalDampingForceTorque: null array");
        k_ext_damping<<<grid_for(num, 256), 256, 0, stream>>>(force, torque, velocity, angularVelocity, dampCoeff,
                                                               num);
        after_launch();
    });
}

void launchAddBuoyancyDrag(double3* force, double3* position, double3* velocity, double* radius, double* inverseMass,
                           const double rhoFluid, const double Cd, const double3 gravity, const double3 fluidVelocity,
                           const double waterLevel, const size_t numBall, const size_t gridD, const size_t blockD,
                           cudaStream_t stream) {
    (void)gridD;
    (void)blockD;
    guarded([&] {
        if (numBall == 0) return;
        if (!force || !position || !velocity || !radius)
            throw Status(DEMSPH_ERR_INVALID, "launchAddBuoyancyDrag: null array");
        k_ext_buoyancy<<<grid_for(numBall, 256), 256, 0, stream>>>(force, position, velocity, radius, inverseMass,
                                                                    rhoFluid, Cd, gravity, fluidVelocity, waterLevel,
                                                                    numBall);
        after_launch();
    });
}

}  // extern "C"
