// Stand-in for DEMSPH/pointCloudGeneration.h: the scene generators the
// reference's examples call, with its signatures and its operation order (so
// the points come out bit for bit; the same generators in Python are
// this_studio_b200/scenes.py).
//   generateUniformPointCloud  inclusive-endpoint lattice, x fastest      (:7-58)
//   HexPBC2D / makeHexPBC2D    periodic cell of a hexagonal x-y packing   (:60-150)
//   generateHexPointCloud      hexagonal layer, odd rows shifted by dx/2  (:152-195)
//   TriangleMesh / makeCylinderMesh  side quads as two triangles, capped  (:197-327)
#pragma once
#include <algorithm>
#include <cmath>
#include <vector>

#include "../demsph/vec.hpp"

inline std::vector<double3> generateUniformPointCloud(const double3 minBound, const double3 maxBound, const double dx) {
    std::vector<double3> pts;
    if (dx <= 0.0) return pts;
    const double eps = 1e-12;
    const double lo[3] = {std::min(minBound.x, maxBound.x), std::min(minBound.y, maxBound.y),
                          std::min(minBound.z, maxBound.z)};
    const double hi[3] = {std::max(minBound.x, maxBound.x), std::max(minBound.y, maxBound.y),
                          std::max(minBound.z, maxBound.z)};
    std::vector<double> axis[3];
    for (int k = 0; k < 3; k++) {
        const long n = std::max(0L, (long)std::floor((hi[k] - lo[k]) / dx + eps) + 1);
        for (long i = 0; i < n; i++) {
            const double v = lo[k] + i * dx;
            if (v <= hi[k] + eps) axis[k].push_back(v);
        }
    }
    pts.reserve(axis[0].size() * axis[1].size() * axis[2].size());
    for (double z : axis[2])
        for (double y : axis[1])
            for (double x : axis[0]) pts.push_back(make_double3(x, y, z));
    return pts;
}

struct HexPBC2D {
    double3 min{0.0, 0.0, 0.0};  // periodic cell, half-open [min, max)
    double3 max{0.0, 0.0, 0.0};
    double Lx{0.0};
    double Ly{0.0};
    double shearX{0.0};  // x shift that goes with a wrap in y (odd row count)
    int nx{0};
    int ny{0};
    bool periodicX{false};
    bool periodicY{false};
};

// Rows dy = a sqrt(3)/2 apart; a periodic axis is snapped up to a whole
// number of steps (ceil(L/step - 1e-12)), a bounded one holds
// floor(L/step + 1e-12) steps.
inline HexPBC2D makeHexPBC2D(const double3 minBound, const double3 maxBound, const double spacing,
                             const bool periodicX, const bool periodicY) {
    HexPBC2D pbc;
    pbc.periodicX = periodicX;
    pbc.periodicY = periodicY;
    if (spacing <= 0.0) return pbc;
    const double dx = spacing;
    const double dy = spacing * std::sqrt(3.0) * 0.5;
    const double lx = std::max(0.0, maxBound.x - minBound.x);
    const double ly = std::max(0.0, maxBound.y - minBound.y);
    const int nx = periodicX ? std::max(1, (int)std::ceil(lx / dx - 1e-12)) : std::max(1, (int)std::floor(lx / dx + 1e-12));
    const int ny = periodicY ? std::max(1, (int)std::ceil(ly / dy - 1e-12)) : std::max(1, (int)std::floor(ly / dy + 1e-12));
    pbc.nx = nx;
    pbc.ny = ny;
    pbc.min = minBound;
    pbc.Lx = nx * dx;
    pbc.Ly = ny * dy;
    pbc.max = make_double3(periodicX ? minBound.x + pbc.Lx : maxBound.x, periodicY ? minBound.y + pbc.Ly : maxBound.y,
                           maxBound.z);
    pbc.shearX = (periodicY && (ny & 1)) ? 0.5 * dx : 0.0;
    return pbc;
}

// Rows along x, odd rows shifted by dx/2, at z = min z; a bounded axis
// stops at its max.
inline void generateHexPointCloud(const double3 minBound, const double3 maxBound, const double spacing,
                                  const bool periodicX, const bool periodicY, std::vector<double3>& points,
                                  HexPBC2D& pbc) {
    points.clear();
    pbc = makeHexPBC2D(minBound, maxBound, spacing, periodicX, periodicY);
    if (pbc.nx <= 0 || pbc.ny <= 0 || spacing <= 0.0) return;
    const double dx = spacing;
    const double dy = spacing * std::sqrt(3.0) * 0.5;
    for (int j = 0; j < pbc.ny; j++) {
        const double y = pbc.min.y + j * dy;
        if (!periodicY && y >= maxBound.y) break;
        const double shift = (j & 1) ? 0.5 * dx : 0.0;
        for (int i = 0; i < pbc.nx; i++) {
            const double x = pbc.min.x + i * dx + shift;
            if (!periodicX && x >= maxBound.x) break;
            points.push_back(make_double3(x, y, pbc.min.z));
        }
    }
}

struct TriangleMesh {
    std::vector<double3> vertices;
    std::vector<int> tri0;
    std::vector<int> tri1;
    std::vector<int> tri2;
    void reserveTriangles(size_t n) {
        tri0.reserve(n);
        tri1.reserve(n);
        tri2.reserve(n);
    }
    void addTriangle(int i0, int i1, int i2) {
        tri0.push_back(i0);
        tri1.push_back(i1);
        tri2.push_back(i2);
    }
    size_t numTriangles() const { return tri0.size(); }
};

// u, v spanning the plane normal to the unit axis a, {u, v, a} right-handed.
inline void buildOrthonormalBasis(const double3& a, double3& u, double3& v) {
    const double3 tmp = (std::fabs(a.z) < 0.9) ? make_double3(0, 0, 1) : make_double3(0, 1, 0);
    u = normalize(cross(tmp, a));
    v = normalize(cross(a, u));
}

// nHeight + 1 rings of nAround vertices from -height/2 to +height/2 along
// the axis through `center`, two triangles per side quad, and with caps a
// centre vertex and a triangle fan at each end.
inline TriangleMesh makeCylinderMesh(const double3& center, const double3& axis, double radius, double height,
                                     int nAround, int nHeight, bool caps = true) {
    TriangleMesh m;
    if (nAround < 3 || nHeight < 1 || !(radius > 0.0) || !(height > 0.0)) return m;
    const double3 w = normalize(axis);
    double3 u, v;
    buildOrthonormalBasis(w, u, v);
    for (int iz = 0; iz <= nHeight; iz++) {
        const double t = (double)iz / (double)nHeight;
        const double z = (t - 0.5) * height;
        const double3 c = make_double3(center.x + z * w.x, center.y + z * w.y, center.z + z * w.z);
        for (int ia = 0; ia < nAround; ia++) {
            const double ang = (2.0 * pi()) * ((double)ia / (double)nAround);
            const double ca = std::cos(ang), sa = std::sin(ang);
            m.vertices.push_back(make_double3(c.x + radius * (ca * u.x + sa * v.x), c.y + radius * (ca * u.y + sa * v.y),
                                              c.z + radius * (ca * u.z + sa * v.z)));
        }
    }
    auto vid = [&](int iz, int ia) { return iz * nAround + ia % nAround; };
    m.reserveTriangles((size_t)2 * nAround * nHeight + (caps ? 2 * nAround : 0));
    for (int iz = 0; iz < nHeight; iz++)
        for (int ia = 0; ia < nAround; ia++) {
            const int i00 = vid(iz, ia), i01 = vid(iz, ia + 1), i10 = vid(iz + 1, ia), i11 = vid(iz + 1, ia + 1);
            m.addTriangle(i00, i10, i11);
            m.addTriangle(i00, i11, i01);
        }
    if (caps) {
        const int bottom = (int)m.vertices.size();
        m.vertices.push_back(make_double3(center.x + (-0.5 * height) * w.x, center.y + (-0.5 * height) * w.y,
                                          center.z + (-0.5 * height) * w.z));
        const int top = (int)m.vertices.size();
        m.vertices.push_back(make_double3(center.x + (0.5 * height) * w.x, center.y + (0.5 * height) * w.y,
                                          center.z + (0.5 * height) * w.z));
        for (int ia = 0; ia < nAround; ia++) m.addTriangle(bottom, vid(0, ia + 1), vid(0, ia));
        for (int ia = 0; ia < nAround; ia++) m.addTriangle(top, vid(nHeight, ia), vid(nHeight, ia + 1));
    }
    return m;
}
