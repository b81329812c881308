// Stand-in for DEMSPH/kernel/WCSPHSolver.h: a scene written for the
// reference (a WCSPHSolver subclass calling addSPH / addDummy / solve)
// compiles unchanged with `-I <this library>/include/demsph_compat`.
#pragma once
#include "../../demsph/solvers.hpp"
#include "../../demsph/vec.hpp"

using demsph::WCSPHSolver;
