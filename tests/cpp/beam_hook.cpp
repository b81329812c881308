// A bonded cantilever written as the reference's scene main()s are: a
// DEMSolver subclass whose addExternalForceTorque ramps a tip load and adds
// global damping through the reference's launchers on getBall()'s arrays,
// and whose addInitialCondition bonds the initial contacts.  Compiled against
// include/demsph_compat (the reference's include names) and run by
// tests/test_gpu_reference_scenes.py, which compares the printed final state
// with the FP64 oracle.  Arguments: maximum time (s), precision (0 FP64,
// 1 mixed).
#include <cstdio>
#include <cstdlib>

#include "externalForceTorque.h"
#include "kernel/DEMSolver.h"

class problem : public DEMSolver {
public:
    const double3 f_c = make_double3(0, 0, 100.e3);
    const double L_beam = 4.0;
    const size_t n_bond = 10;
    const double c_d = 0.1;
    const double dt = 1.e-5;
    HostDeviceArray1D<double3> f_e;
    long hookCalls = 0;

    problem() : DEMSolver(0) {}

    void addExternalForceTorque(const size_t iStep, const double time) override {
        (void)iStep;
        double c = time;
        if (c > 1.0) c = 1.0;
        std::vector<double3> f(n_bond + 1, make_double3(0., 0., 0.));
        f[n_bond] = f_c * c;
        f_e.setHost(f);
        f_e.copyHostToDevice(0);
        launchAddConstantForce(getBall().force(), f_e.d_ptr, getBall().deviceSize(), getBall().gridDim(),
                               getBall().blockDim(), 0);
        launchAddGlobalDampingForceTorque(getBall().force(), getBall().torque(), getBall().velocity(),
                                          getBall().angularVelocity(), c_d, getBall().deviceSize(),
                                          getBall().gridDim(), getBall().blockDim(), 0);
        hookCalls++;
    }

    bool addInitialCondition() override {
        std::vector<int> obj0 = getBallPairPointed();
        std::vector<int> obj1 = getBallPairPointing();
        std::vector<double3> pos = getBall().positionHostCopy();
        addBondedInteraction(obj0, obj1, pos);
        return true;
    }
};

int main(int argc, char** argv) {
    const double tMax = argc > 1 ? std::atof(argv[1]) : 0.05;
    problem test;
    if (argc > 2) test.setPrecision(std::atoi(argv[2]));
    test.setBondedPair(0, 0, 1.0, 200e9, 2.6, 0.0, 0.0, 0.0);
    const double r = test.L_beam / double(test.n_bond) / 2.0;
    test.addFixedBall(make_double3(0., 0., 0.), r, 0);
    for (size_t i = 0; i < test.n_bond; i++)
        test.addBall(make_double3((i + 1) * 2. * r, 0., 0.), make_double3(0., 0., 0.), make_double3(0., 0., 0.), r,
                     7800, 0);
    test.solve(make_double3(0., -r, -r), make_double3(test.L_beam, r, r), make_double3(0., 0., 0.), test.dt, tMax, 0,
               "");
    std::vector<double3> p = test.getBall().positionHostCopy();
    std::printf("hook_calls %ld\n", test.hookCalls);
    for (const double3& q : p) std::printf("pos %.17g %.17g %.17g\n", q.x, q.y, q.z);
    return 0;
}
