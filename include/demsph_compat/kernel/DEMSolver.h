// Stand-in for DEMSPH/kernel/DEMSolver.h: a scene written for the reference
// (`#include "kernel/DEMSolver.h"`, a DEMSolver subclass overriding
// addExternalForceTorque / addInitialCondition, the launchers of
// externalForceTorque.h on getBall()'s arrays) compiles unchanged with
// `-I <this library>/include/demsph_compat` and runs on the B200 library.
// The class, HostDeviceArray1D and the double3 helpers come from
// include/demsph; symMatrix / make_symMatrix name the facade's SymMatrix.
#pragma once
#include "../../demsph/solvers.hpp"
#include "../../demsph/vec.hpp"

using demsph::BallArrays;
using demsph::DEMSolver;
using demsph::HostDeviceArray1D;
using symMatrix = demsph::SymMatrix;

// make_symMatrix (myMat.h): components in the order xx, yy, zz, xy, xz, yz
inline symMatrix make_symMatrix(double xx, double yy, double zz, double xy, double xz, double yz) {
    return symMatrix{xx, yy, zz, xy, xz, yz};
}
