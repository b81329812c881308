// Internal interface between the coupled DEM-SPH stepper (sph.cu) and the
// DEM scene (dem.cu).  The stepper runs both solvers on one stream: it reads
// the balls' state to place the markers that sample them in the fluid, writes
// the fluid's force and torque on each ball into the DEM's coupling buffers
// (added to the contact forces in the DEM's external-force hook), and runs
// DEM steps between fluid steps without a host synchronisation.
#pragma once
#include <cuda_runtime.h>

#include "../../include/demsph.h"

namespace demsph {

struct DemBodies {
    int n;                // balls
    const double4* pos;   // (x, y, z, radius), caller order
    const double4* vel;   // (v, 1/m)
    const double4* angv;  // (omega, -)
    double4* force;       // coupling force per ball
    double4* torque;      // coupling torque per ball
    double dt;            // DEM time step
};

// The DEM scene's ball state and coupling buffers (allocated, zero, on the
// first call).  The scene must be initialised.
DemBodies dem_bodies(demsph_dem_t h);
// Starts a block of coupled steps on stream s: s waits for the DEM's own
// stream, the DEM launches on s until dem_block_end, and its dynamic state
// is saved for a replay.
void dem_block_begin(demsph_dem_t h, cudaStream_t s);
// n DEM steps (DEMSolver::solve's loop body) issued on stream s (the
// block's stream, or the stream capturing it).
void dem_block_steps(demsph_dem_t h, int n, cudaStream_t s);
// For capturing coupled steps in a CUDA graph: whether the DEM step can be
// replayed (no time-dependent kernel arguments), its step counter and clock
// (saved around a capture, advanced after a replay), the key of its
// ping-pong buffer state, and a counter of its graph resets (a change means
// its buffers or kernel arguments changed).
bool dem_graphable(demsph_dem_t h);
void dem_clock(demsph_dem_t h, long* iStep, double* time);
void dem_set_clock(demsph_dem_t h, long iStep, double time);
void dem_advance_clock(demsph_dem_t h, long steps);
int dem_graph_key(demsph_dem_t h);
long dem_graph_epoch(demsph_dem_t h);
// Ends the block (synchronising its stream).  Returns false when a DEM
// list overflowed: the lists were regrown and the DEM state restored to the
// block's start, and the block must be replayed.
bool dem_block_end(demsph_dem_t h);

}  // namespace demsph
