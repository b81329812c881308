// ASCII VTK UnstructuredGrid (.vtu) frames in the layout the reference's
// solvers write (DEMSolver.h:908-1370, WCSPHSolver.h:360-520): FieldData TIME
// and STEP, one Piece of points (vertex cells) or triangles, then named point
// or cell arrays, numbers in fixed notation with 10 decimals.  Host code.
#pragma once
#include <sys/stat.h>
#include <cerrno>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <string>
#include <vector>

#include "common.cuh"

namespace demsph {
namespace vtu {

// mkdir -p
static inline void make_dirs(const std::string& dir) {
    std::string cur;
    std::stringstream ss(dir);
    std::string part;
    if (!dir.empty() && dir[0] == '/') cur = "/";
    while (std::getline(ss, part, '/')) {
        if (part.empty()) continue;
        cur += part + "/";
        if (mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST)
            throw Status(DEMSPH_ERR_INVALID, "cannot create directory " + cur);
    }
}

class File {
  public:
    File(const std::string& dir, const char* stem, long frame) {
        make_dirs(dir);
        std::ostringstream name;
        name << dir << "/" << stem << "_" << std::setw(4) << std::setfill('0') << frame << ".vtu";
        path_ = name.str();
        out_.open(path_.c_str());
        if (!out_) throw Status(DEMSPH_ERR_INVALID, "cannot open " + path_);
        out_ << std::fixed << std::setprecision(10);
    }
    ~File() {
        if (out_.is_open()) out_.close();
    }
    void head(double time, long step, size_t npoints, size_t ncells) {
        out_ << "<?xml version=\"1.0\"?>\n"
                "<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
                "  <UnstructuredGrid>\n"
                "    <FieldData>\n"
                "      <DataArray type=\"Float32\" Name=\"TIME\"  NumberOfTuples=\"1\" format=\"ascii\"> "
             << time
             << " </DataArray>\n"
                "      <DataArray type=\"Int32\"   Name=\"STEP\"  NumberOfTuples=\"1\" format=\"ascii\"> "
             << step
             << " </DataArray>\n"
                "    </FieldData>\n"
                "    <Piece NumberOfPoints=\""
             << npoints << "\" NumberOfCells=\"" << ncells << "\">\n";
    }
    void points(const std::vector<double3>& p) {
        out_ << "      <Points>\n"
                "        <DataArray type=\"Float32\" NumberOfComponents=\"3\" format=\"ascii\">\n";
        for (const double3& q : p) out_ << ' ' << q.x << ' ' << q.y << ' ' << q.z;
        out_ << "\n        </DataArray>\n"
                "      </Points>\n";
    }
    // one VTK_VERTEX cell per point
    void vertex_cells(size_t n) {
        out_ << "      <Cells>\n"
                "        <DataArray type=\"Int32\" Name=\"connectivity\" format=\"ascii\">\n";
        for (size_t i = 0; i < n; ++i) out_ << ' ' << i;
        out_ << "\n        </DataArray>\n"
                "        <DataArray type=\"Int32\" Name=\"offsets\" format=\"ascii\">\n";
        for (size_t i = 1; i <= n; ++i) out_ << ' ' << i;
        out_ << "\n        </DataArray>\n"
                "        <DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n";
        for (size_t i = 0; i < n; ++i) out_ << " 1";
        out_ << "\n        </DataArray>\n"
                "      </Cells>\n";
    }
    // one VTK_TRIANGLE cell per (i0, i1, i2)
    void triangle_cells(const std::vector<int4>& t) {
        out_ << "      <Cells>\n"
                "        <DataArray type=\"Int32\" Name=\"connectivity\" format=\"ascii\">\n";
        for (const int4& q : t) out_ << ' ' << q.x << ' ' << q.y << ' ' << q.z;
        out_ << "\n        </DataArray>\n"
                "        <DataArray type=\"Int32\" Name=\"offsets\" format=\"ascii\">\n";
        for (size_t i = 1; i <= t.size(); ++i) out_ << ' ' << (3 * i);
        out_ << "\n        </DataArray>\n"
                "        <DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n";
        for (size_t i = 0; i < t.size(); ++i) out_ << " 5";
        out_ << "\n        </DataArray>\n"
                "      </Cells>\n";
    }
    void begin_data(const char* section, const char* scalars) {
        out_ << "      <" << section << " Scalars=\"" << scalars << "\">\n";
    }
    void floats(const char* name, const std::vector<double>& v) {
        out_ << "        <DataArray type=\"Float32\" Name=\"" << name << "\" format=\"ascii\">\n";
        for (double x : v) out_ << ' ' << x;
        out_ << "\n        </DataArray>\n";
    }
    void ints(const char* name, const std::vector<int>& v) {
        out_ << "        <DataArray type=\"Int32\" Name=\"" << name << "\" format=\"ascii\">\n";
        for (int x : v) out_ << ' ' << x;
        out_ << "\n        </DataArray>\n";
    }
    void vectors(const char* name, const std::vector<double3>& v) {
        out_ << "        <DataArray type=\"Float32\" Name=\"" << name << "\" NumberOfComponents=\"3\" format=\"ascii\">\n";
        for (const double3& q : v) out_ << ' ' << q.x << ' ' << q.y << ' ' << q.z;
        out_ << "\n        </DataArray>\n";
    }
    void end_data(const char* section) {
        out_ << "      </" << section << ">\n"
                "    </Piece>\n"
                "  </UnstructuredGrid>\n"
                "</VTKFile>\n";
        out_.flush();
        if (!out_) throw Status(DEMSPH_ERR_INVALID, "write failed: " + path_);
    }

  private:
    std::string path_;
    std::ofstream out_;
};

}  // namespace vtu
}  // namespace demsph
