/*
 * demsph.h -- C ABI of the B200-native DEMSPH particle-interaction library
 * (libdemsph_b200.so).
 *
 * The reference (kaiqideng/this_studio, DEMSPH/kernel) exposes its per-step
 * path as two C++ solver classes whose public methods set up a scene and run
 * the step loop (DEMSolver, DEMSPH/kernel/DEMSolver.h:1633-2049; WCSPHSolver,
 * DEMSPH/kernel/WCSPHSolver.h:522-624), on top of extern "C" kernel launchers.
 * This header is the flat C form of that scene-setup / solver-step interface:
 * one function per public method, plain pointers and sizes, no C++ or torch
 * types, so cgo / JNI / ctypes / N-API bind it directly.  The C++ facade in
 * include/demsph/solvers.hpp restores the reference class and method names.
 *
 * Conventions
 *  - Every function returns an int status: DEMSPH_OK (0) or a DEMSPH_ERR_*
 *    code; nothing exits the process (the reference calls exit(1) when
 *    cudaSetDevice fails, DEMSolver.h:1974-1981).  demsph_last_error() gives
 *    the message of the last failure on the calling thread.
 *  - Vectors are arrays of 3 doubles (x, y, z) per object, packed: n objects
 *    take 3n doubles.  Quaternions are (q0, q1, q2, q3); symmetric matrices are
 *    (xx, yy, zz, xy, xz, yz) as in the reference (myQua.h:10-15, myMat.h:15-27).
 *  - Host arrays are read during the call only.  Getters write into caller
 *    buffers sized from the matching demsph_*_num_* query.
 *  - `stream` is a cudaStream_t passed as void*; 0 means the legacy stream.
 *    All device work of a scene is ordered on its stream.  Getters
 *    synchronise that stream.
 *  - A scene owns all device memory it allocates; demsph_*_destroy frees it.
 */
#ifndef DEMSPH_H
#define DEMSPH_H

#include <stddef.h>

/* CUDA's stream handle (cudaStream_t is struct CUstream_st*) and double3,
 * named without including the CUDA headers */
struct CUstream_st;
struct double3;

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define DEMSPH_OK 0
#define DEMSPH_ERR_INVALID 1     /* bad argument or call order               */
#define DEMSPH_ERR_SCENE 2       /* malformed scene (empty, NaN, bad sizes)  */
#define DEMSPH_ERR_OVERFLOW 3    /* a list overflowed and could not regrow   */
#define DEMSPH_ERR_CUDA 4        /* CUDA runtime error                       */
#define DEMSPH_ERR_NOT_READY 5   /* scene not initialised                    */
#define DEMSPH_ERR_TIMEOUT 6     /* a bounded device wait gave up            */
#define DEMSPH_ERR_ALLOC 7       /* host or device allocation failed         */

/* arithmetic of the force laws (positions, velocities and springs are FP64
 * in both modes) */
#define DEMSPH_PRECISION_FP64 0  /* reference arithmetic throughout         */
#define DEMSPH_PRECISION_MIXED 1 /* FP32 force laws, FP64 state            */

typedef struct demsph_dem_scene* demsph_dem_t;
typedef struct demsph_dem_member* demsph_dem_member_t;
typedef struct demsph_sph_scene* demsph_sph_t;
typedef struct demsph_sph_member* demsph_sph_member_t;
typedef struct demsph_dem_snapshot* demsph_dem_snapshot_t;
typedef struct demsph_sph_snapshot* demsph_sph_snapshot_t;

const char* demsph_last_error(void);
const char* demsph_version(void);
/* Number of CUDA kernels this library has launched since load (instrumentation). */
long long demsph_kernel_launches(void);
/* No counterpart in the reference.  Scene buffers come from the current
 * device's default stream-ordered memory pool, whose stock setting hands
 * freed memory back to the driver at every synchronisation (re-mapping it on
 * the next allocation costs milliseconds per scene, and more on a busy GPU).
 * The first scene created on a device sets the pool to keep up to 8 GiB of
 * freed memory in this process; this call sets another limit (0: the stock
 * behaviour), and a limit set here is never overridden.  Affects only this
 * process. */
int demsph_retain_device_memory(unsigned long long bytes);
/* No counterpart in the reference (its HostDeviceArray1D calls the CUDA
 * runtime directly, myHostDeviceArray.h:99-186).  Device memory for callers
 * that do not link the CUDA runtime themselves, such as the header-only C++
 * facade's HostDeviceArray1D: stream-ordered allocation from the current
 * device's default pool, its release, and a copy (kind 0 host to device, 1
 * device to host, 2 device to device) that returns once the copy is done. */
int demsph_device_alloc(void** ptr, size_t bytes, void* stream);
int demsph_device_free(void* ptr, void* stream);
int demsph_memcpy(void* dst, const void* src, size_t bytes, int kind, void* stream);

/* ======================================================================= */
/* DEM: spheres, clumps, triangle-mesh walls, contact + parallel bonds      */
/* ======================================================================= */

/* DEMSolver::DEMSolver(cudaStream_t)  -- DEMSolver.h:147 */
int demsph_dem_create(demsph_dem_t* out, void* stream);
/* DEMSolver::~DEMSolver -- DEMSolver.h:153 */
int demsph_dem_destroy(demsph_dem_t s);

/* DEMSolver::setHertzianPair -- DEMSolver.h:1637-1662 */
int demsph_dem_set_hertzian_pair(demsph_dem_t s, int materialA, int materialB, double effectiveYoungsModulus,
                                 double effectiveShearModulus, double restitution, double rollingToShearStiffness,
                                 double torsionToShearStiffness, double slidingFriction, double rollingFriction,
                                 double torsionFriction);
/* DEMSolver::setLinearPair -- DEMSolver.h:1667-1700 */
int demsph_dem_set_linear_pair(demsph_dem_t s, int materialA, int materialB, double kn, double ks, double kr,
                               double kt, double dn, double ds, double dr, double dt, double slidingFriction,
                               double rollingFriction, double torsionFriction);
/* DEMSolver::setBondedPair -- DEMSolver.h:1705-1726 */
int demsph_dem_set_bonded_pair(demsph_dem_t s, int materialA, int materialB, double bondRadiusMultiplier,
                               double bondYoungsModulus, double normalToShearStiffness, double tensileStrength,
                               double cohesion, double friction);

/* DEMSolver::addBall (density > 0) / addFixedBall (fixed != 0), n at once --
 * DEMSolver.h:1728-1768.  clumpID may be NULL (all -1). */
int demsph_dem_add_balls(demsph_dem_t s, long n, const double* position, const double* velocity,
                         const double* angularVelocity, const double* radius, const double* density,
                         const int* materialID, const int* clumpID, int fixed);
/* DEMSolver::addClump -- DEMSolver.h:1796-1845 */
int demsph_dem_add_clump(demsph_dem_t s, long numPebbles, const double* pebblePosition, const double* pebbleRadius,
                         const double* centroid, const double* velocity, const double* angularVelocity, double mass,
                         const double* inertiaTensor6, int materialID);
/* DEMSolver::addMeshWall -- DEMSolver.h:1882-1935.  Like the reference, the
 * wall starts at rest; use demsph_dem_set_wall_motion to move it. */
int demsph_dem_add_mesh_wall(demsph_dem_t s, long numVertices, const double* vertexLocal, long numTriangles,
                             const int* tri0, const int* tri1, const int* tri2, const double* position,
                             int materialID);
/* Sets a mesh wall's velocity and angular velocity (the reference writes the
 * wall body arrays through getMeshWallBody(), DEMSolver.h:1545). */
int demsph_dem_set_wall_motion(demsph_dem_t s, int wall, const double* velocity, const double* angularVelocity);
/* DEMSolver::addBondedInteraction -- DEMSolver.h:1937-1942 (bondedInteraction::add, :93-135).
 * Callable before or after initialisation (the reference's addInitialCondition hook, :1998). */
int demsph_dem_add_bonds(demsph_dem_t s, long n, const int* objectPointed, const int* objectPointing,
                         const double* ballPosition, long numBallPositions);

/* The reference's external force hook (virtual addExternalForceTorque,
 * DEMSolver.h:1372) runs user kernels from DEMSPH/externalForceTorque.cu.
 * These three configure the same kernels, applied in this order each call:
 * constant force (launchAddConstantForce, externalForceTorque.cu:14-24; the
 * force is scaled by min(time/ramp, 1) when ramp > 0), global damping
 * (launchAddGlobalDampingForceTorque, :41-57), buoyancy + drag against the
 * plane z = waterLevel (launchAddBuoyancyDrag, :135-160). */
int demsph_dem_set_constant_force(demsph_dem_t s, long n, const double* force, double rampTime);
int demsph_dem_set_global_damping(demsph_dem_t s, double dampingCoefficient);
int demsph_dem_set_buoyancy_drag(demsph_dem_t s, double fluidDensity, double dragCoefficient, const double* gravity,
                                 const double* fluidVelocity, double waterLevel);

/* DEMSolver::addExternalForceTorque (virtual, DEMSolver.h:1372), as a
 * callback: when set, every force evaluation of a step (two per step, the
 * reference's calls at DEMSolver.h:1464,1470 and in the periodic loops)
 * calls fn(user, iStep, time) after the contact, bond and wall forces and
 * the configured hooks above are summed, and before the half-step
 * integration; iStep is 1-based and time is t - dt/2, then t, as in the
 * reference.  Around the call the ball state sits in arrays of the
 * reference's layout (demsph_dem_hook_arrays); whatever the callback's
 * kernels write there (force and torque, or also position, velocity,
 * angular velocity, radius, inverse mass) is taken back before the
 * integration.  The callback's device work must be ordered on the scene's
 * stream or on the legacy default stream (stream 0), as the reference's
 * hooks launch on stream 0.  It runs on the host thread that called
 * demsph_dem_step; it may call demsph_dem_hook_arrays, demsph_dem_num_balls
 * and demsph_dem_set_external_hook (to remove itself) but no other function
 * of this scene.  A scene with a callback
 * launches every kernel directly (no CUDA graphs), and steps replayed after
 * a list overflow call it again.  fn = NULL removes it.
 *
 * demsph_dem_hook_arrays: device pointers to those arrays (3 doubles per
 * ball for position, velocity, angularVelocity, force, torque; one double per
 * ball for radius and inverseMass; the scene's int materialID and clumpID;
 * n balls), allocated on first request.  Their contents are current only
 * while a callback runs. */
typedef void (*demsph_dem_hook_fn)(void* user, long iStep, double time);
typedef struct demsph_ball_arrays {
    double* position;
    double* velocity;
    double* angularVelocity;
    double* force;
    double* torque;
    double* radius;
    double* inverseMass;
    int* materialID;
    int* clumpID;
    long n;
} demsph_ball_arrays;
int demsph_dem_set_external_hook(demsph_dem_t s, demsph_dem_hook_fn fn, void* user);
int demsph_dem_hook_arrays(demsph_dem_t s, demsph_ball_arrays* out);

/* The initialisation part of DEMSolver::solve (DEMSolver.h:1961-1997):
 * upload, grids (cell = 2 r_max; triangle cell >= 2 circumradius),
 * neighbour search, one force evaluation with dt = 0.  precision is
 * DEMSPH_PRECISION_*. */
/* setPeriodicBoundary (DEMSolver.h:1944-1959), before initialize: periodic
 * ghost passes along the flagged axes and their combinations, as the
 * reference runs them (DEMSolver.h:279-426,1407-1534).  demsph_dem_get_pairs
 * with which = 2 + k returns the pairs of the k-th active ghost set (order X,
 * Y, Z, XY, YZ, XZ, XYZ over the active ones). */
int demsph_dem_set_periodic(demsph_dem_t s, int x, int y, int z);
/* No counterpart in the reference.  List capacities per ball (pair rows,
 * reverse rows, candidate triangles): reserve raises the initial capacities
 * before initialize (they still grow on demand), capacity reads the current
 * ones. */
int demsph_dem_reserve(demsph_dem_t s, int pairsPerBall, int reversePerBall, int trianglesPerBall);
/* No counterpart in the reference (autotuner).  The ball grid's cell edge as a
 * multiple (1 to 4) of the reference's 2 r_max (DEMSolver.h:245-263); set
 * before initialisation.  Any factor gives the same pairs (a 27-cell stencil
 * still covers every contact); rows come in another order, so sums differ by
 * rounding. */
int demsph_dem_set_cell_factor(demsph_dem_t s, double factor);
int demsph_dem_capacity(demsph_dem_t s, int* pairsPerBall, int* reversePerBall, int* trianglesPerBall);
int demsph_dem_initialize(demsph_dem_t s, const double* minBoundary, const double* maxBoundary,
                          const double* gravity, double timeStep, int precision);
/* numSteps passes of the step loop (loop_ball / loop_ball_wall,
 * DEMSolver.h:1376-1485): neighbour search every 5th step, two force
 * evaluations and the kick-drift-kick integration per step. */
int demsph_dem_step(demsph_dem_t s, long numSteps);
/* No counterpart in the reference.  step() replays the scene's step loop as
 * CUDA graphs (blocks of 10 steps aligned to the re-sort cadence, captured on
 * first use and whenever buffers were reallocated); enable = 0 launches every
 * kernel directly instead.  Both give identical results.  Scenes with a force
 * ramp (setConstantForce with rampTime > 0) always launch directly. */
int demsph_dem_set_graphs(demsph_dem_t s, int enable);
/* Protected step pieces of DEMSolver, exposed for parity checks:
 * neighborSearch (DEMSolver.h:698-777) and calculateBallContactForceTorque
 * (:599-695) followed, when walls & 1, by addTriangleContactForceTorque(dtWall)
 * (:428-597), when walls & 2, by the periodic ghost passes
 * addDummyContactForceTorque(dt) (:279-426), and when walls & 4, by the
 * external forces (the configured hooks and a callback) at the scene's
 * current time, as addExternalForceTorque (:1372) after a force evaluation. */
int demsph_dem_neighbor_search(demsph_dem_t s);
int demsph_dem_eval_forces(demsph_dem_t s, double dt, int walls, double dtWall);

/* No counterpart in the reference (which keeps its state in host-device
 * arrays that a caller copies by hand).  A device copy of a scene's
 * dynamic state -- balls, clumps, walls, pair and triangle rows with their
 * springs, bonds, periodic ghost lists, the step counter -- and its
 * restoration into the same scene, for checkpoints kept in device memory,
 * what-if branches and replays: steps from a restored state repeat the steps
 * after the snapshot bit for bit.  A snapshot holds device memory until
 * destroyed; it restores only into the scene it was taken from. */
int demsph_dem_snapshot(demsph_dem_t s, demsph_dem_snapshot_t* out);
int demsph_dem_restore(demsph_dem_t s, demsph_dem_snapshot_t snapshot);
int demsph_dem_snapshot_destroy(demsph_dem_snapshot_t snapshot);
/* No counterpart in the reference (which has no diagnostics).  FP64
 * conservation diagnostics of the current state, summed on the device in a
 * fixed order (the same bits for the same state), 12 doubles: linear
 * momentum (3), angular momentum about the origin (3, x cross m v plus I w),
 * translational and rotational kinetic energy, mass -- over the moving
 * bodies (free spheres and clumps; pebbles count through their clump) --
 * and the sum of the ball forces of the last force evaluation (3; contact
 * and bond forces cancel pairwise). */
int demsph_dem_diagnostics(demsph_dem_t s, double* out);
int demsph_dem_num_balls(demsph_dem_t s, long* n);
int demsph_dem_num_pairs(demsph_dem_t s, int which /*0 ball-ball, 1 ball-triangle*/, long* n);
int demsph_dem_num_bonds(demsph_dem_t s, long* n);
int demsph_dem_num_clumps(demsph_dem_t s, long* n);
int demsph_dem_step_index(demsph_dem_t s, long* step, double* time);
/* ball_ getters (DEMSolver::getBall, DEMSolver.h:1541); any pointer may be NULL. */
int demsph_dem_get_balls(demsph_dem_t s, double* position, double* velocity, double* angularVelocity, double* force,
                         double* torque);
int demsph_dem_set_balls(demsph_dem_t s, const double* position, const double* velocity,
                         const double* angularVelocity);
/* getBallPair* / getBallTrianglePair* (DEMSolver.h:1549-1631), in the
 * reference's CSR order (rows by objectPointed, stencil order inside a row). */
int demsph_dem_get_pairs(demsph_dem_t s, int which, int* objectPointed, int* objectPointing, double* sliding,
                         double* rolling, double* torsion, double* force, double* torque);
/* Seeds contact history: springs of matching (pointed, pointing) pairs of the
 * current ball-ball list are set from the given list (the carry rule of
 * writeBallInteractionsKernel, ballNeighborSearchKernel.cu:130-143). */
int demsph_dem_import_springs(demsph_dem_t s, long n, const int* objectPointed, const int* objectPointing,
                              const double* sliding, const double* rolling, const double* torsion);
/* Same for the ball-triangle contact rows, keyed by (ball, triangle).  No
 * counterpart in the reference: used to carry wall contact history when a
 * scene's state moves between device scenes (batching). */
int demsph_dem_import_wall_springs(demsph_dem_t s, long n, const int* ball, const int* triangle,
                                   const double* sliding, const double* rolling, const double* torsion);
/* No counterpart in the reference (batching).  Copies the state of the
 * continuing members of a batch from scene src into scene dst on the device.
 * Member k's balls [srcStart[k], srcStart[k] + num[k]) in src become
 * [dstStart[k], ...) in dst: positions (plus shift[3k..3k+2]), velocities,
 * angular velocities, pair rows (partners moved by dstStart[k] - srcStart[k];
 * partners must lie in the member's own range) and ball-triangle rows
 * (triangle indices plus triDelta[k]).  dst must have been initialised with
 * the same material / spring configuration. */
int demsph_dem_copy_members(demsph_dem_t dst, demsph_dem_t src, int count, const int* srcStart, const int* dstStart,
                            const int* num, const int* triDelta, const double* shift);
/* No counterpart in the reference (batching).  Carries the clumps and bonds
 * of continuing members from scene src into scene dst, after
 * demsph_dem_copy_members has carried their balls: member k's clumps
 * [srcClump[k], +numClumps[k]) in src become [dstClump[k], ...) in dst
 * (centroid plus shift[3k..3k+2], velocity, angular velocity, orientation)
 * and its bonds [srcBond[k], +numBonds[k]) become [dstBond[k], ...) (intact
 * flag, contact point plus shift, normal, accumulated forces and torques,
 * peak stresses).  The bonds of a member must join the same member balls, in
 * the same order, in both scenes. */
int demsph_dem_copy_member_bodies(demsph_dem_t dst, demsph_dem_t src, int count, const int* srcClump,
                                  const int* dstClump, const int* numClumps, const int* srcBond, const int* dstBond,
                                  const int* numBonds, const double* shift);
/* Batch members (no counterpart in the reference).  A member is one scene's
 * balls uploaded once to the device: create, add balls exactly as
 * demsph_dem_add_balls and clumps as demsph_dem_add_clump, seal (validates,
 * uploads, drops the host copy of the balls).  demsph_dem_assemble_balls places `count` sealed members' balls into
 * a scene that has none yet -- member k translated by offsets[3k..3k+2], its
 * material ids shifted by matOffset[k], member order kept -- as
 * demsph_dem_add_balls would from the same balls; walls, materials and the
 * rest are added as usual, then demsph_dem_initialize. */
int demsph_dem_member_create(demsph_dem_member_t* out, void* stream);
int demsph_dem_member_destroy(demsph_dem_member_t m);
int demsph_dem_member_add_balls(demsph_dem_member_t m, long n, const double* position, const double* velocity,
                                const double* angularVelocity, const double* radius, const double* density,
                                const int* materialID, int fixed);
/* addClump (DEMSolver.h:1796-1845) into a member: its pebbles follow the
 * member's balls added so far (member-local indices), the clump keeps its
 * centroid, velocity, angular velocity and inverse inertia.  Assembly
 * appends the clumps of each member, in member order, to the scene's clump
 * table (centroids translated, pebble ranges and clump ids renumbered). */
int demsph_dem_member_add_clump(demsph_dem_member_t m, long np, const double* point, const double* radius,
                                const double* centroid, const double* velocity, const double* angularVelocity,
                                double mass, const double* inertia, int materialID);
int demsph_dem_member_num_clumps(demsph_dem_member_t m, long* n);
int demsph_dem_member_seal(demsph_dem_member_t m);
int demsph_dem_member_count(demsph_dem_member_t m, long* n);
int demsph_dem_assemble_balls(demsph_dem_t s, int count, const demsph_dem_member_t* members, const double* offsets,
                              const int* matOffset);
/* getBondedInteraction (DEMSolver.h:1547) fields */
int demsph_dem_get_bonds(demsph_dem_t s, int* objectPointed, int* objectPointing, int* isBonded, double* normalForce,
                         double* torsionTorque, double* shearForce, double* bendingTorque, double* normal,
                         double* point);
/* Writes the bond state, in the order demsph_dem_get_bonds returns it (n =
 * the number of bonds); any array may be NULL to keep that field.  No
 * counterpart in the reference, whose bond arrays callers write through
 * getBondedInteraction() (DEMSolver.h:1547): used to start a force
 * evaluation from a given bond state. */
int demsph_dem_set_bonds(demsph_dem_t s, long n, const int* isBonded, const double* normalForce,
                         const double* torsionTorque, const double* shearForce, const double* bendingTorque,
                         const double* normal, const double* point);
/* getClump (DEMSolver.h:1543) */
/* outputBallVTU / outputMeshWallVTU / outputBallInteractionVTU /
 * outputBondedInteractionVTU / outputBallTriangleInteractionVTU
 * (DEMSolver.h:908-1370): writes <dir>/ball_NNNN.vtu, triangleWall_NNNN.vtu,
 * ballInteraction_NNNN.vtu, bondedInteraction_NNNN.vtu and
 * ballTriangleInteraction_NNNN.vtu (NNNN = frame) for the parts selected in
 * `what` (DEMSPH_VTU_* bits), in the reference's layout.  Interaction frames
 * evaluate each listed contact on the current state (zero time increment). */
#define DEMSPH_VTU_BALLS 1
#define DEMSPH_VTU_MESH_WALLS 2
#define DEMSPH_VTU_BALL_INTERACTIONS 4
#define DEMSPH_VTU_BONDED_INTERACTIONS 8
#define DEMSPH_VTU_BALL_TRIANGLE_INTERACTIONS 16
#define DEMSPH_VTU_FLUID 1
#define DEMSPH_VTU_DUMMIES 2
int demsph_dem_write_vtu(demsph_dem_t s, const char* dir, long frame, int what);
int demsph_dem_get_clumps(demsph_dem_t s, double* position, double* velocity, double* angularVelocity,
                          double* orientation);
/* getMeshWallBody (DEMSolver.h:1545) and vertex global positions */
int demsph_dem_get_walls(demsph_dem_t s, double* position, double* orientation, double* vertexGlobal);

/* ======================================================================= */
/* WCSPH: weakly compressible SPH with fixed dummy wall particles           */
/* ======================================================================= */

/* WCSPHSolver::WCSPHSolver(cudaStream_t) -- WCSPHSolver.h:21 */
int demsph_sph_create(demsph_sph_t* out, void* stream);
int demsph_sph_destroy(demsph_sph_t s);
/* WCSPHSolver::addSPH / addDummy, n at once -- WCSPHSolver.h:523-541
 * (m = spacing^3 rho, h = 1.3 spacing; particles with rho <= 0 or c <= 0 are skipped). */
int demsph_sph_add(demsph_sph_t s, int dummy, long n, const double* position, const double* velocity,
                   const double* soundSpeed, const double* spacing, const double* density, const double* viscosity);
/* Initialisation part of WCSPHSolver::solve (WCSPHSolver.h:567-600):
 * grid (cell = 2 h_max), dummy-dummy pairs and dummy wall normals. */
int demsph_sph_initialize(demsph_sph_t s, const double* minBoundary, const double* maxBoundary, const double* gravity,
                          double timeStep, int precision);
/* numSteps passes of the WCSPHSolver::solve loop (WCSPHSolver.h:607-621),
 * queued on the scene's stream: the call returns without waiting for the
 * device (getters, snapshots and demsph_sph_synchronize wait).  A neighbour
 * row that overflows during the steps is walked from the cell table (same
 * pairs); the lists are regrown at the next call. */
int demsph_sph_step(demsph_sph_t s, long numSteps);
/* No counterpart in the reference.  Waits for the scene's queued work. */
int demsph_sph_synchronize(demsph_sph_t s);
/* No counterpart in the reference.  step() replays the step loop as CUDA
 * graphs of two steps; enable = 0 launches every kernel directly.  Both give
 * identical results. */
int demsph_sph_set_graphs(demsph_sph_t s, int enable);
/* Protected step pieces (WCSPHSolver.h:150-358), for parity checks. */
int demsph_sph_neighbor_search(demsph_sph_t s);
int demsph_sph_eval_accel(demsph_sph_t s);

/* Instrumentation (no counterpart in the reference, which has no timers):
 * runs numSteps steps with a CUDA event after each phase on the scene stream
 * and returns the mean milliseconds per step of the 5 phases: cell sort,
 * reorder + neighbour lists, momentum + kick + drift, continuity + EOS,
 * momentum + kick. */
int demsph_sph_profile_steps(demsph_sph_t s, long numSteps, double* phaseMs);
/* No counterpart in the reference (autotuner).  Rebuilds the neighbour lists
 * of the current state `trials` times with each compiled block shape of the
 * list build (warps per block x candidates staged per warp), times them with
 * CUDA events on the scene's stream, and keeps the fastest for later steps.
 * Writes the chosen shape to *chosen and each shape's milliseconds per build
 * to msPerShape[0 .. demsph_sph_num_list_shapes()-1] (either may be NULL).
 * The lists are unchanged by the choice (same pairs, same order). */
int demsph_sph_tune(demsph_sph_t s, int trials, int* chosen, double* msPerShape);
int demsph_sph_num_list_shapes(void);
/* No counterpart in the reference (autotuner).  The grid's cell edge as a
 * multiple (1 to 4) of 2 h_max (1 + skin); set before initialisation.  Any
 * factor gives the same pairs; rows come in another order. */
int demsph_sph_set_cell_factor(demsph_sph_t s, double factor);
/* No counterpart in the reference.  enable = 1: in CUDA-graph steps of a
 * scene with skin lists (and no coupled balls), the list rebuild -- cell
 * sort, reorder, skin rows -- is the body of a conditional graph node whose
 * condition the rebuild decision sets on the device, so steps that keep their
 * lists launch none of its kernels (2% off the 128k dam break's step).  Off by
 * default: the rebuild's kernels are then launched every step and return at
 * once when the decision says so (results are identical), because Nsight
 * Compute does not profile the kernel nodes of graphs that hold conditional
 * nodes.
 * conditional_rebuild reports whether it is in use and how many kernels one
 * rebuild runs (the library's launch counter counts them only when they run,
 * which the host does not see: add rebuilds x launchesPerRebuild). */
int demsph_sph_set_conditional_rebuild(demsph_sph_t s, int enable);
int demsph_sph_conditional_rebuild(demsph_sph_t s, int* active, long* launchesPerRebuild);
/* No counterpart in the reference (autotuner).  The neighbour rows are sized at
 * initialisation to the longest row of one build times (1 + fraction)
 * (default 0.125) and regrown by a quarter when a later build overflows
 * (the step is then replayed); set before initialisation.  list_capacity
 * reports the current row capacities of the fluid-fluid and fluid-dummy
 * lists. */
int demsph_sph_set_list_headroom(demsph_sph_t s, double fraction);
int demsph_sph_list_capacity(demsph_sph_t s, int* fluidRow, int* dummyRow);
/* Selects a list-build block shape by index (what demsph_sph_tune picks). */
int demsph_sph_set_list_shape(demsph_sph_t s, int shape);

/* No counterpart in the reference (batching).  Copies the fluid state of
 * the continuing members of a batch from scene src into scene dst on the
 * device: member k's particles with caller ids [srcStart[k], srcStart[k] +
 * num[k]) in src are ids [dstStart[k], ...) in dst; positions (plus
 * shift[3k..3k+2]), velocities, density, pressure and density change are
 * copied.  Source ranges must not overlap.  dst's neighbour lists are rebuilt
 * at its next step. */
int demsph_sph_copy_members(demsph_sph_t dst, demsph_sph_t src, int count, const int* srcStart, const int* dstStart,
                            const int* num, const double* shift);

/* Batch members (no counterpart in the reference).  A member is one scene's
 * particles uploaded once to the device in the library's record layout:
 * create, add fluid / dummy particles exactly as demsph_sph_add, seal
 * (validates, uploads, drops the host copy).  demsph_sph_assemble then
 * initialises an empty scene from `count` sealed members on the device --
 * member k's fluid and dummies translated by offsets[3k..3k+2], fluid in
 * member order (member 0's particles first) -- as demsph_sph_initialize
 * would from the same particles added in that order.  Members stay valid and
 * can be assembled again. */
int demsph_sph_member_create(demsph_sph_member_t* out, void* stream);
int demsph_sph_member_destroy(demsph_sph_member_t m);
int demsph_sph_member_add(demsph_sph_member_t m, int dummy, long n, const double* position, const double* velocity,
                          const double* soundSpeed, const double* spacing, const double* density,
                          const double* viscosity);
int demsph_sph_member_seal(demsph_sph_member_t m);
int demsph_sph_member_count(demsph_sph_member_t m, int dummy, long* n);
int demsph_sph_assemble(demsph_sph_t s, int count, const demsph_sph_member_t* members, const double* offsets,
                        const double* minBoundary, const double* maxBoundary, const double* gravity, double timeStep,
                        int precision);

/* outputWCSPHVTU / outputDummyVTU (WCSPHSolver.h:360-520): writes
 * <dir>/SPH_NNNN.vtu and/or <dir>/dummy_NNNN.vtu (what: DEMSPH_VTU_FLUID,
 * DEMSPH_VTU_DUMMIES) in the reference's layout. */
int demsph_sph_write_vtu(demsph_sph_t s, const char* dir, long frame, int what);

/* Skin lists (no counterpart in the reference, which rebuilds its lists every
 * step: WCSPHSolver::neighborSearch, WCSPHSolver.h:150-285).  The fluid's
 * neighbour rows hold every candidate within the cutoff plus a skin of
 * `fraction` x 2 h_max at their last rebuild; a step rebuilds them (cell sort,
 * reorder, list build) only when some particle has drifted half the skin, and
 * its first momentum pass keeps the pairs that pass the reference's exact
 * cutoff test on that step's positions, so every step uses the reference's
 * pair set.  Default 0.04; 0 rebuilds exact lists every step.  Before
 * initialisation the value also sizes the grid's cells (2 h_max (1 +
 * fraction)); afterwards it may only be lowered.  With coupled balls the
 * fluid-marker rows are skin rows too, and a marker's drift joins the
 * rebuild decision.  skin_stats: the fraction in use (0 when off) and the
 * rebuilds so far. */
int demsph_sph_set_skin(demsph_sph_t s, double fraction);
/* Autotunes the skin (and with it the share of steps that rebuild lists and
 * the length of the rows): times `steps` steps with no skin, half the grid's
 * skin and the grid's skin, each from the same saved state (restored after),
 * and keeps the fastest.  msPerStep (3 doubles, or NULL) gets the times. */
int demsph_sph_tune_skin(demsph_sph_t s, int steps, double* chosen, double* msPerStep);
int demsph_sph_skin_stats(demsph_sph_t s, double* fraction, long* rebuilds);

/* No counterpart in the reference.  The fluid's state (positions,
 * velocities, density, pressure, density change, order, the step counter)
 * copied on the device and restored into the same scene; the neighbour
 * lists are rebuilt at the next step, which then repeats the steps after
 * the snapshot bit for bit.  A snapshot restores only into its own scene. */
int demsph_sph_snapshot(demsph_sph_t s, demsph_sph_snapshot_t* out);
int demsph_sph_restore(demsph_sph_t s, demsph_sph_snapshot_t snapshot);
int demsph_sph_snapshot_destroy(demsph_sph_snapshot_t snapshot);
/* No counterpart in the reference.  In mixed precision, a scene whose fluid
 * particles share h, m, c and nu and whose dummies share m, c, nu and rest
 * density (with the fluid's h) runs momentum and continuity passes
 * specialised for it (constants hoisted, terms regrouped; same pairs, same
 * formulas), coupled scenes included (the markers' terms as in the general
 * passes); enable = 0 keeps the general passes.  uniform_kernels reports
 * whether the specialised passes are in use. */
int demsph_sph_set_uniform_kernels(demsph_sph_t s, int enable);
int demsph_sph_uniform_kernels(demsph_sph_t s, int* active);
/* No counterpart in the reference.  FP64 conservation diagnostics of the
 * fluid, summed on the device in a fixed order, 8 doubles: mass, momentum
 * (3), kinetic energy, potential energy -sum m g.x, sum of the density
 * changes Delta rho, volume sum m / rho. */
int demsph_sph_diagnostics(demsph_sph_t s, double* out);
int demsph_sph_num(demsph_sph_t s, int dummy, long* n);
int demsph_sph_num_pairs(demsph_sph_t s, int which /*0 fluid-fluid, 1 fluid-dummy, 2 dummy-dummy*/, long* n);
int demsph_sph_step_index(demsph_sph_t s, long* step, double* time);
/* getSPH / getDummy (WCSPHSolver.h:563-565), in the caller's original order. */
int demsph_sph_get(demsph_sph_t s, int dummy, double* position, double* velocity, double* acceleration,
                   double* density, double* pressure, double* densityChange, double* normal);
int demsph_sph_set(demsph_sph_t s, const double* position, const double* velocity, const double* density,
                   const double* pressure, const double* densityChange);
/* Pair lists in the reference's CSR order (countSPHInteractionsKernel and friends,
 * SPHNeighborSearchKernel.cu:6-228), indices in the caller's original order. */
int demsph_sph_get_pairs(demsph_sph_t s, int which, int* objectPointed, int* objectPointing);

/* ======================================================================= */
/* Particle-level DEM-SPH coupling                                          */
/* ======================================================================= */
/* The reference couples DEM balls to a fluid only through a buoyancy-drag
 * plane (addBuoyancyDragKernel, externalForceTorque.cu:66-133, kept as
 * demsph_dem_set_buoyancy_drag).  These calls couple balls of an initialised
 * DEM scene to the fluid of an initialised SPH scene particle by particle.
 *
 * Each coupled ball is sampled by markers: moving boundary particles on
 * shells r_l = R - (l + 1/2) spacing inside its surface (l spacing < 2 h,
 * r_l > spacing / 4), max(1, round(4 pi r_l^2 / spacing^2)) per shell on a
 * golden-angle spiral (one marker at the centre of a ball too small for a
 * shell).  A marker carries its ball's rigid velocity v + omega x offset,
 * the outward normal, mass density * spacing^3, and acts on the fluid
 * exactly as a dummy particle does (the fluid-dummy terms of
 * updateWCSPHAccelerationKernel and updateWCSPHDensityChangeKernel,
 * WCSPHIntegrationKernel.cu:110-143,240-270).  The ball receives minus the
 * sum of m_a times its markers' terms in the fluid accelerations (force, and
 * offset x force as torque), so momentum is exchanged exactly.
 *
 * couple_balls: couples balls[0..n) (DEM indices) with markers of the given
 * spacing, h (at most the fluid's largest h), sound speed, viscosity and
 * rest density, placed at the balls' current state.  One SPH scene couples
 * to one DEM scene; calls add balls.
 * couple_step: n coupled steps.  Per step the markers follow the balls, the
 * fluid takes one step with them, each ball's coupling force and torque
 * are set to the mean of the reactions of the step's two acceleration
 * passes, and the DEM takes demSubsteps steps (its time step times
 * demSubsteps must equal the fluid's) with them held.  Both scenes run on
 * the SPH scene's stream during the call; a DEM list overflow replays the
 * call.  Stepping either scene alone keeps the markers and the coupling
 * force where the last coupled step left them.
 * get_markers: per marker in body order (balls in the order coupled):
 * position, velocity, outward normal, last reaction on it (3 doubles each),
 * and its ball.  get_coupling: per coupled ball its index, force, torque. */
int demsph_sph_couple_balls(demsph_sph_t s, demsph_dem_t dem, long n, const int* balls, double spacing,
                            double smoothingLength, double soundSpeed, double viscosity, double density);
int demsph_sph_couple_step(demsph_sph_t s, demsph_dem_t dem, long n, int demSubsteps);
int demsph_sph_num_markers(demsph_sph_t s, long* markers, long* balls);
int demsph_sph_get_markers(demsph_sph_t s, double* position, double* velocity, double* normal, double* force,
                           int* ball);
int demsph_sph_get_coupling(demsph_sph_t s, int* ball, double* force, double* torque);

/* ======================================================================= */
/* Reference launcher compatibility                                          */
/* ======================================================================= */
/* The reference's sort / scan launchers with their exact signatures
 * (DEMSPH/kernel/buildHashStartEnd.cuh:5-19; `struct CUstream_st*` is
 * cudaStream_t).  They return void like the reference; a failure is
 * recorded for demsph_last_error().  gridD / blockD are ignored.
 *
 * buildHashStartEnd: hashIndex[i] = i, stable sort of (hashValue, hashIndex)
 * by hashValue in place (a hand-written LSD radix sort instead of
 * thrust::sort_by_key), then start[h] / end[h] for every key 0 <= h <
 * startEndSize that occurs (buildHashStartEnd.cu:6-83).  Scratch of about
 * 3 * hashListSize ints is taken with cudaMallocAsync on the stream.
 * buildPrefixSum: inclusive scan (buildHashStartEnd.cu:85-117), size <= 2^24. */
void buildHashStartEnd(int* start, int* end, int* hashIndex, int* hashValue, const size_t startEndSize,
                       const size_t hashListSize, const size_t gridD_GPU, const size_t blockD_GPU,
                       struct CUstream_st* stream_GPU);
void buildPrefixSum(int* prefixSum, int* count, const size_t size, struct CUstream_st* stream);

/* No counterpart in the reference.  The same sort and start / end table as
 * buildHashStartEnd, for callers that cannot allocate device memory: a host
 * loop that reserved its whole memory budget up front, or code issuing work
 * where a cudaMalloc (which may synchronise the device, or fail under memory
 * pressure) is not allowed.  It calls no allocator: its scratch is a fixed
 * array inside the library, sized for DEMSPH_NOALLOC_MAX_KEYS keys (3.3 MB,
 * held on every GPU that loads the library until the process exits).  Each
 * call looks up that array's device address on the current device; the
 * first lookup on a device may load the library's module, so make the first
 * call on a device before any stream capture.  All calls share the one array, so
 * calls that overlap on the GPU (other streams, other host threads) race;
 * calls ordered on one stream are safe.  Returns DEMSPH_OK,
 * DEMSPH_ERR_INVALID when hashListSize > DEMSPH_NOALLOC_MAX_KEYS (with a
 * message in demsph_last_error), or DEMSPH_ERR_CUDA. */
/* The reference's user-force launchers with its exact signatures
 * (DEMSPH/externalForceTorque.h:6-36; `struct double3` is CUDA's double3):
 * on ball arrays of the reference's layout, such as those an external-force
 * callback receives (demsph_dem_hook_arrays).  They return void like the
 * reference; a failure is recorded for demsph_last_error().  gridD / blockD
 * are ignored.
 * launchAddConstantForce: force[i] += force_external[i] (externalForceTorque.cu:4-24).
 * launchAddGlobalDampingForceTorque: force[i] -= c |force[i]| v_i / |v_i|,
 *   torque[i] -= c |torque[i]| w_i / |w_i| (:26-57).
 * launchAddBuoyancyDrag: buoyancy of the part of each ball below the plane
 *   z = waterLevel plus quadratic drag against fluidVelocity; balls with
 *   inverseMass <= 0 are skipped (:59-160). */
void launchAddConstantForce(struct double3* force, const struct double3* force_external, const size_t num,
                            const size_t gridD, const size_t blockD, struct CUstream_st* stream);
void launchAddGlobalDampingForceTorque(struct double3* force, struct double3* torque, const struct double3* velocity,
                                       const struct double3* angularVelocity, const double dampCoeff, const size_t num,
                                       const size_t gridD, const size_t blockD, struct CUstream_st* stream);
void launchAddBuoyancyDrag(struct double3* force, struct double3* position, struct double3* velocity, double* radius,
                           double* inverseMass, const double rhoFluid, const double Cd, const struct double3 gravity,
                           const struct double3 fluidVelocity, const double waterLevel, const size_t numBall,
                           const size_t gridD, const size_t blockD, struct CUstream_st* stream);

#define DEMSPH_NOALLOC_MAX_KEYS 262144
int demsph_build_hash_start_end_noalloc(int* start, int* end, int* hashIndex, int* hashValue, size_t startEndSize,
                                        size_t hashListSize, struct CUstream_st* stream);

#ifdef __cplusplus
}
#endif
#endif /* DEMSPH_H */
