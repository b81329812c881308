// Stand-in for DEMSPH/externalForceTorque.h: the reference's user-force
// launchers (launchAddConstantForce, launchAddGlobalDampingForceTorque,
// launchAddBuoyancyDrag) with its signatures, exported by the B200 library
// and declared in include/demsph.h.
#pragma once
#include <cstddef>
#include <driver_types.h>
#include <vector_types.h>

#include "../demsph.h"
