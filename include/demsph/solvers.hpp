// solvers.hpp -- C++ facade over include/demsph.h with the reference's class
// and method names (DEMSolver, DEMSPH/kernel/DEMSolver.h:144-2078;
// WCSPHSolver, DEMSPH/kernel/WCSPHSolver.h:18-635), header-only.
//
// The reference's virtual hooks are virtual here too: a subclass overriding
// addExternalForceTorque(iStep, time) has it called after each force
// evaluation of a step (DEMSolver.h:1372, called at :1464,1470), with
// getBall() giving the ball arrays in the reference's layout for the
// reference's launchers (launchAddConstantForce and the others, declared in
// demsph.h); addInitialCondition() is called once after initialisation
// (DEMSolver.h:1998).  The same forces can also be configured without a
// subclass (setConstantForce / setGlobalDamping / setBuoyancyDrag).
// Failures throw demsph::Error instead of exiting.
#pragma once
#include <driver_types.h>
#include <vector_functions.h>
#include <vector_types.h>

#include <array>
#include <exception>
#include <stdexcept>
#include <string>
#include <utility>
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

// A device array with a host staging copy, as the reference's
// HostDeviceArray1D (myHostDeviceArray.h:99-186) that hook code uses to pass
// its own per-ball data to a launcher: setHost / pushHost, then
// copyHostToDevice, then d_ptr on the device.  Memory comes from the
// library (stream-ordered allocation), so no CUDA runtime link is needed.
template <class T>
class HostDeviceArray1D {
public:
    T* d_ptr = nullptr;

    HostDeviceArray1D() = default;
    ~HostDeviceArray1D() { release(); }
    HostDeviceArray1D(const HostDeviceArray1D&) = delete;
    HostDeviceArray1D& operator=(const HostDeviceArray1D&) = delete;
    HostDeviceArray1D(HostDeviceArray1D&& o) noexcept { *this = std::move(o); }
    HostDeviceArray1D& operator=(HostDeviceArray1D&& o) noexcept {
        if (this != &o) {
            release();
            d_ptr = o.d_ptr; n_ = o.n_; s_ = o.s_; host_ = std::move(o.host_);
            o.d_ptr = nullptr; o.n_ = 0;
        }
        return *this;
    }

    size_t hostSize() const { return host_.size(); }
    size_t deviceSize() const { return n_; }
    void setHost(const std::vector<T>& h) { host_ = h; }
    void pushHost(const T& v) { host_.push_back(v); }
    const std::vector<T>& hostRef() const { return host_; }
    void allocateDevice(size_t n, cudaStream_t s, bool zeroFill = true) {
        release();
        s_ = s;
        check(demsph_device_alloc((void**)&d_ptr, n * sizeof(T), (void*)s), "HostDeviceArray1D::allocateDevice");
        n_ = n;
        if (zeroFill && n) {
            std::vector<T> z(n, T{});
            check(demsph_memcpy(d_ptr, z.data(), n * sizeof(T), 0, (void*)s), "HostDeviceArray1D::allocateDevice");
        }
    }
    void copyHostToDevice(cudaStream_t s) {
        if (n_ != host_.size()) allocateDevice(host_.size(), s, false);
        if (n_) check(demsph_memcpy(d_ptr, host_.data(), n_ * sizeof(T), 0, (void*)s), "copyHostToDevice");
    }
    void copyDeviceToHost(cudaStream_t s) {
        host_.resize(n_);
        if (n_) check(demsph_memcpy(host_.data(), d_ptr, n_ * sizeof(T), 1, (void*)s), "copyDeviceToHost");
    }
    std::vector<T> getHostCopy() {
        copyDeviceToHost(s_);
        return host_;
    }

private:
    void release() {
        if (d_ptr) demsph_device_free(d_ptr, (void*)s_);
        d_ptr = nullptr;
        n_ = 0;
    }
    size_t n_ = 0;
    cudaStream_t s_ = nullptr;
    std::vector<T> host_;
};

// What DEMSolver::getBall() returns (the reference's ball_, particle.h):
// device pointers to the ball arrays in the reference's layout, current
// while addExternalForceTorque runs, the launch geometry of the reference
// (blockDim = min(maximumThread, n), gridDim to cover n), and host copies.
class BallArrays {
public:
    explicit BallArrays(demsph_dem_t h) : h_(h) {}
    double3* position() { return (double3*)arrays().position; }
    double3* velocity() { return (double3*)arrays().velocity; }
    double3* angularVelocity() { return (double3*)arrays().angularVelocity; }
    double3* force() { return (double3*)arrays().force; }
    double3* torque() { return (double3*)arrays().torque; }
    double* radius() { return arrays().radius; }
    double* inverseMass() { return arrays().inverseMass; }
    int* materialID() { return arrays().materialID; }
    int* clumpID() { return arrays().clumpID; }
    size_t deviceSize() const {
        long n = 0;
        check(demsph_dem_num_balls(h_, &n), "getBall");
        return (size_t)n;
    }
    size_t hostSize() const { return deviceSize(); }
    size_t blockDim() const {
        size_t n = deviceSize();
        size_t b = n < maxThread_ ? n : maxThread_;
        return b ? b : 1;
    }
    size_t gridDim() const { return (deviceSize() + blockDim() - 1) / blockDim(); }
    std::vector<double3> positionHostCopy() { return copy(0); }
    std::vector<double3> velocityHostCopy() { return copy(1); }
    std::vector<double3> angularVelocityHostCopy() { return copy(2); }
    std::vector<double3> forceHostCopy() { return copy(3); }
    std::vector<double3> torqueHostCopy() { return copy(4); }
    size_t maxThread_ = 256;

private:
    demsph_ball_arrays arrays() {
        demsph_ball_arrays a{};
        check(demsph_dem_hook_arrays(h_, &a), "getBall");
        return a;
    }
    std::vector<double3> copy(int which) {
        std::vector<double3> v(deviceSize());
        double* p[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
        if (!v.empty()) {
            p[which] = &v[0].x;
            check(demsph_dem_get_balls(h_, p[0], p[1], p[2], p[3], p[4]), "getBall");
        }
        return v;
    }
    demsph_dem_t h_;
};

class DEMSolver {
public:
    explicit DEMSolver(cudaStream_t s = nullptr) {
        check(demsph_dem_create(&h_, (void*)s), "DEMSolver");
        ball_ = BallArrays(h_);
    }
    virtual ~DEMSolver() { demsph_dem_destroy(h_); }
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
    // The precision solve() initialises with (DEMSPH_PRECISION_*; mixed by default).
    void setPrecision(int precision) { precision_ = precision; }
    void initialize(double3 mn, double3 mx, double3 g, double dt, int precision) {
        check(demsph_dem_initialize(h_, &mn.x, &mx.x, &g.x, dt, precision), "initialize");
    }
    void initialize(double3 mn, double3 mx, double3 g, double dt) { initialize(mn, mx, g, dt, precision_); }
    void step(long n) {
        const int rc = demsph_dem_step(h_, n);
        rethrowHookError();
        check(rc, "step");
    }
    // DEMSolver::solve (DEMSolver.h:1961-2049): initialisation (upload,
    // grids, neighbour search, one force evaluation with dt = 0), then
    // addInitialCondition(), then the step loop with addExternalForceTorque
    // after each force evaluation; VTU frames in `dir` on the reference's
    // cadence (none when `dir` is empty).
    void solve(double3 mn, double3 mx, double3 g, double dt, double maximumTime, size_t numFrame,
               const std::string& dir, size_t deviceID = 0, size_t maximumThread = 256) {
        (void)deviceID;
        ball_.maxThread_ = maximumThread ? maximumThread : 256;
        initialize(mn, mx, g, dt);
        addInitialCondition();
        check(demsph_dem_set_external_hook(h_, &DEMSolver::hookTrampoline, this), "solve");
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
    // ball_ (DEMSolver::getBall, DEMSolver.h:1541)
    BallArrays& getBall() { return ball_; }
    std::vector<double3> getBallPosition() {
        std::vector<double3> p(numBalls_);
        check(demsph_dem_get_balls(h_, &p[0].x, nullptr, nullptr, nullptr, nullptr), "getBall");
        return p;
    }
    std::vector<int> getBallPairPointed() { return pairs(0).first; }
    std::vector<int> getBallPairPointing() { return pairs(0).second; }
    demsph_dem_t handle() { return h_; }

protected:
    // DEMSolver::addExternalForceTorque (virtual, DEMSolver.h:1372): called
    // after each force evaluation of a step, at time t - dt/2 and t.  This
    // default adds nothing and takes the callback away, so a solver that
    // does not override it steps as one without hooks (CUDA graphs on).
    virtual void addExternalForceTorque(const size_t iStep, const double time) {
        (void)iStep;
        (void)time;
        demsph_dem_set_external_hook(h_, nullptr, nullptr);
    }
    // DEMSolver::addInitialCondition (virtual, DEMSolver.h:1536), called once
    // after initialisation; returns whether it changed the scene.
    virtual bool addInitialCondition() { return false; }

private:
    static void hookTrampoline(void* self, long iStep, double time) {
        DEMSolver* s = static_cast<DEMSolver*>(self);
        if (s->hookError_) return;
        try {
            s->addExternalForceTorque((size_t)iStep, time);
        } catch (...) {
            s->hookError_ = std::current_exception();
            demsph_dem_set_external_hook(s->h_, nullptr, nullptr);
        }
    }
    void rethrowHookError() {
        if (hookError_) {
            std::exception_ptr e = hookError_;
            hookError_ = nullptr;
            std::rethrow_exception(e);
        }
    }
    std::pair<std::vector<int>, std::vector<int>> pairs(int which) {
        long n = 0;
        check(demsph_dem_num_pairs(h_, which, &n), "numPairs");
        std::vector<int> a(n), b(n);
        if (n) check(demsph_dem_get_pairs(h_, which, a.data(), b.data(), nullptr, nullptr, nullptr, nullptr, nullptr),
                     "getPairs");
        return {a, b};
    }
    demsph_dem_t h_ = nullptr;
    BallArrays ball_{nullptr};
    std::exception_ptr hookError_;
    int precision_ = DEMSPH_PRECISION_MIXED;
    long numBalls_ = 0;
    int walls_ = 0;
};

class WCSPHSolver {
public:
    explicit WCSPHSolver(cudaStream_t s = nullptr) { check(demsph_sph_create(&h_, (void*)s), "WCSPHSolver"); }
    virtual ~WCSPHSolver() { demsph_sph_destroy(h_); }
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
