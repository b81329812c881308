// solvers.hpp -- C++ facade over include/demsph.h with the reference's class
// and method names (DEMSolver, DEMSPH/kernel/DEMSolver.h:144-2078;
// WCSPHSolver, DEMSPH/kernel/WCSPHSolver.h:18-635), header-only.
//
// Differences from the reference: failures throw demsph::Error instead of
// exiting; the virtual hooks are configuration
// (setConstantForce / setGlobalDamping / setBuoyancyDrag, and
// addBondedInteraction after initialize() for bonded initial contacts).
#pragma once
#include <driver_types.h>
#include <vector_functions.h>
#include <vector_types.h>

#include <array>
#include <stdexcept>
#include <string>
#include <vector>

#include "../demsph.h"

namespace demsph {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& w) : std::runtime_error(w), code(c) {}
};

inline void check(int rc, const char* what) {
    if (rc != DEMSPH_OK) throw Error(rc, std::string(what) + ": " + demsph_last_error());
}

// Symmetric 3x3 matrix in the reference's order (myMat.h:15-27).
struct SymMatrix {
    double xx, yy, zz, xy, xz, yz;
};

// size_t(maximumTime / timeStep) + 1 passes of `while (iStep <= numStep)`
// (DEMSolver.h:1988,1380) run numStep + 1 steps.
inline long solveSteps(double timeStep, double maximumTime) {
    return (long)(size_t)(maximumTime / timeStep) + 2;
}

// The reference's frame cadence (DEMSolver.h:1984-2046, WCSPHSolver.h:587-621):
// frame 0 after initialisation; numStep = total - 1, frameInterval = numStep /
// numFrame (numStep when numFrame is 0, at least 1); after step iStep
// (1-based) a frame whenever iStep % frameInterval == 0.
template <class Step, class Write>
inline void runFrames(long total, size_t numFrame, Step step, Write write) {
    long numStep = total - 1;
    long interval = numFrame > 0 ? numStep / (long)numFrame : numStep;
    if (interval < 1) interval = 1;
    write(0);
    long done = 0, frame = 0;
    while (done < total) {
        long next = (done / interval + 1) * interval;
        if (next > total) next = total;
        step(next - done);
        done = next;
        if (done % interval == 0) write(++frame);
    }
}

class DEMSolver {
public:
    explicit DEMSolver(cudaStream_t s = nullptr) { check(demsph_dem_create(&h_, (void*)s), "DEMSolver"); }
    ~DEMSolver() { demsph_dem_destroy(h_); }
    DEMSolver(const DEMSolver&) = delete;
    DEMSolver& operator=(const DEMSolver&) = delete;

    void setHertzianPair(int a, int b, double E, double G, double e, double krks, double ktks, double mus,
                         double mur, double mut) {
        check(demsph_dem_set_hertzian_pair(h_, a, b, E, G, e, krks, ktks, mus, mur, mut), "setHertzianPair");
    }
    void setLinearPair(int a, int b, double kn, double ks, double kr, double kt, double dn, double ds, double dr,
                       double dt, double mus, double mur, double mut) {
        check(demsph_dem_set_linear_pair(h_, a, b, kn, ks, kr, kt, dn, ds, dr, dt, mus, mur, mut), "setLinearPair");
    }
    void setBondedPair(int a, int b, double gamma, double Eb, double knks, double sigma, double C, double mu) {
        check(demsph_dem_set_bonded_pair(h_, a, b, gamma, Eb, knks, sigma, C, mu), "setBondedPair");
    }
    void addBall(double3 p, double3 v, double3 w, double r, double density, int mat, int clumpID = -1) {
        check(demsph_dem_add_balls(h_, 1, &p.x, &v.x, &w.x, &r, &density, &mat, &clumpID, 0), "addBall");
        ++numBalls_;
    }
    void addFixedBall(double3 p, double r, int mat, int clumpID = -1) {
        check(demsph_dem_add_balls(h_, 1, &p.x, nullptr, nullptr, &r, nullptr, &mat, &clumpID, 1), "addFixedBall");
        ++numBalls_;
    }
    void addClump(std::vector<double3> point, std::vector<double> radius, double3 centroid, double3 v, double3 w,
                  double mass, SymMatrix I, int mat) {
        double I6[6] = {I.xx, I.yy, I.zz, I.xy, I.xz, I.yz};
        check(demsph_dem_add_clump(h_, (long)point.size(), &point[0].x, radius.data(), &centroid.x, &v.x, &w.x, mass,
                                   I6, mat),
              "addClump");
        numBalls_ += (long)point.size();
    }
    void addMeshWall(const std::vector<double3>& vertices, const std::vector<int>& tri0,
                     const std::vector<int>& tri1, const std::vector<int>& tri2, const double3& position,
                     const double3& velocity, const double3& angularVelocity, int mat) {
        (void)velocity;
        (void)angularVelocity;  // not applied, as in the reference (DEMSolver.h:1901-1911)
        check(demsph_dem_add_mesh_wall(h_, (long)vertices.size(), &vertices[0].x, (long)tri0.size(), tri0.data(),
                                       tri1.data(), tri2.data(), &position.x, mat),
              "addMeshWall");
        walls_ += tri0.empty() ? 0 : 1;
    }
    void setMeshWallMotion(int wall, double3 v, double3 w) {
        check(demsph_dem_set_wall_motion(h_, wall, &v.x, &w.x), "setMeshWallMotion");
    }
    void addBondedInteraction(const std::vector<int>& a, const std::vector<int>& b,
                              const std::vector<double3>& ballPosition) {
        check(demsph_dem_add_bonds(h_, (long)a.size(), a.data(), b.data(), &ballPosition[0].x,
                                   (long)ballPosition.size()),
              "addBondedInteraction");
    }
    void setConstantForce(const std::vector<double3>& f, double rampTime = 0.0) {
        check(demsph_dem_set_constant_force(h_, (long)f.size(), &f[0].x, rampTime), "setConstantForce");
    }
    void setGlobalDamping(double c) { check(demsph_dem_set_global_damping(h_, c), "setGlobalDamping"); }
    void setBuoyancyDrag(double rho, double Cd, double3 g, double3 u, double level) {
        check(demsph_dem_set_buoyancy_drag(h_, rho, Cd, &g.x, &u.x, level), "setBuoyancyDrag");
    }
    void initialize(double3 mn, double3 mx, double3 g, double dt, int precision = DEMSPH_PRECISION_MIXED) {
        check(demsph_dem_initialize(h_, &mn.x, &mx.x, &g.x, dt, precision), "initialize");
    }
    void step(long n) { check(demsph_dem_step(h_, n), "step"); }
    // DEMSolver::solve (DEMSolver.h:1961-2049); VTU frames in `dir` (none when empty).
    void solve(double3 mn, double3 mx, double3 g, double dt, double maximumTime, size_t numFrame,
               const std::string& dir, size_t deviceID = 0, size_t maximumThread = 256) {
        (void)deviceID; (void)maximumThread;
        initialize(mn, mx, g, dt);
        const long total = solveSteps(dt, maximumTime);
        if (dir.empty()) {
            step(total);
            return;
        }
        const int what = DEMSPH_VTU_BALLS | DEMSPH_VTU_BONDED_INTERACTIONS | DEMSPH_VTU_BALL_INTERACTIONS |
                         (walls_ ? DEMSPH_VTU_MESH_WALLS | DEMSPH_VTU_BALL_TRIANGLE_INTERACTIONS : 0);
        runFrames(total, numFrame, [&](long n) { step(n); },
                  [&](long f) { check(demsph_dem_write_vtu(h_, dir.c_str(), f, what), "writeVTU"); });
    }
    std::vector<double3> getBallPosition() {
        std::vector<double3> p(numBalls_);
        check(demsph_dem_get_balls(h_, &p[0].x, nullptr, nullptr, nullptr, nullptr), "getBall");
        return p;
    }
    std::vector<int> getBallPairPointed() { return pairs(0).first; }
    std::vector<int> getBallPairPointing() { return pairs(0).second; }
    demsph_dem_t handle() { return h_; }

private:
    std::pair<std::vector<int>, std::vector<int>> pairs(int which) {
        long n = 0;
        check(demsph_dem_num_pairs(h_, which, &n), "numPairs");
        std::vector<int> a(n), b(n);
        if (n) check(demsph_dem_get_pairs(h_, which, a.data(), b.data(), nullptr, nullptr, nullptr, nullptr, nullptr),
                     "getPairs");
        return {a, b};
    }
    demsph_dem_t h_ = nullptr;
    long numBalls_ = 0;
    int walls_ = 0;
};

class WCSPHSolver {
public:
    explicit WCSPHSolver(cudaStream_t s = nullptr) { check(demsph_sph_create(&h_, (void*)s), "WCSPHSolver"); }
    ~WCSPHSolver() { demsph_sph_destroy(h_); }
    WCSPHSolver(const WCSPHSolver&) = delete;
    WCSPHSolver& operator=(const WCSPHSolver&) = delete;

    void addSPH(double3 p, double3 v, double c, double spacing, double density, double viscosity) {
        check(demsph_sph_add(h_, 0, 1, &p.x, &v.x, &c, &spacing, &density, &viscosity), "addSPH");
    }
    void addDummy(double3 p, double3 v, double c, double spacing, double density, double viscosity) {
        check(demsph_sph_add(h_, 1, 1, &p.x, &v.x, &c, &spacing, &density, &viscosity), "addDummy");
    }
    void initialize(double3 mn, double3 mx, double3 g, double dt, int precision = DEMSPH_PRECISION_FP64) {
        check(demsph_sph_initialize(h_, &mn.x, &mx.x, &g.x, dt, precision), "initialize");
    }
    void step(long n) { check(demsph_sph_step(h_, n), "step"); }
    // WCSPHSolver::solve (WCSPHSolver.h:567-624); VTU frames in `dir` (none when empty).
    void solve(double3 mn, double3 mx, double3 g, double dt, double maximumTime, size_t numFrame,
               const std::string& dir, size_t deviceID = 0, size_t maximumThread = 256) {
        (void)deviceID; (void)maximumThread;
        initialize(mn, mx, g, dt);
        const long total = solveSteps(dt, maximumTime);
        if (dir.empty()) {
            step(total);
            return;
        }
        runFrames(total, numFrame, [&](long n) { step(n); }, [&](long f) {
            check(demsph_sph_write_vtu(h_, dir.c_str(), f, DEMSPH_VTU_FLUID | DEMSPH_VTU_DUMMIES), "writeVTU");
        });
    }
    std::vector<double3> getSPHPosition() {
        long n = 0;
        check(demsph_sph_num(h_, 0, &n), "num");
        std::vector<double3> p(n);
        if (n) check(demsph_sph_get(h_, 0, &p[0].x, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr), "getSPH");
        return p;
    }
    demsph_sph_t handle() { return h_; }

private:
    demsph_sph_t h_ = nullptr;
};

}  // namespace demsph
