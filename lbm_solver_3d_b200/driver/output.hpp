// ============================================================================
//  output.hpp -- the host driver's result files. Formats are those of the
//  reference (src/utils/io.cpp:44-97, src/utils/analytic.cpp:27-64) so that
//  its post-processing and tests read them unchanged:
//    <prefix>_final.vtk / <prefix>_<t>.vtk   legacy binary big-endian VTK
//    <prefix>_traj.dat                        15 columns per traj_every steps
//    <prefix>_squirmer.dat                    final rigid-body state
//    <prefix>_profile_{y,z}.dat               Poiseuille profiles (no squirmer)
//    <prefix>_summary.txt                     key value diagnostics
// ============================================================================
#pragma once
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/lbmgpu.h"

namespace lbmdrv {

// The fields the writers read, wherever they live.
struct FieldsView {
    int nx = 0, ny = 0, nz = 0;
    const uint8_t* flag = nullptr;
    const double* rho = nullptr;
    const double* u = nullptr;   // interleaved (ux, uy, uz)
    size_t size() const { return (size_t)nx * ny * nz; }
};

// Host copy of the fields the writers need.
struct Fields {
    int nx = 0, ny = 0, nz = 0;
    std::vector<uint8_t> flag;
    std::vector<double> rho, u;  // u interleaved (ux, uy, uz)
    size_t size() const { return (size_t)nx * ny * nz; }
    FieldsView view() const { return FieldsView{nx, ny, nz, flag.data(), rho.data(), u.data()}; }
};

void makeDirectory(const std::string& dir);                  // throws std::runtime_error
void writeVtk(const FieldsView& F, const std::string& path); // throws std::runtime_error
inline void writeVtk(const Fields& F, const std::string& path) { writeVtk(F.view(), path); }

class TrajectoryFile {
public:
    explicit TrajectoryFile(const std::string& path, bool append = false);
    ~TrajectoryFile();
    void append(const double* row);   // 15 values (see lbmgpu_traj_rows)
    void flush();
private:
    std::FILE* fp_ = nullptr;
};

void writeSquirmerState(const lbmgpu_squirmer& s, double nu, int t, const std::string& path);

// Exact solutions (analytic.cpp:11-25) and the relative L2 error of u_x over
// the cross-section x = 0, with the centre-line profile files. Returns a
// negative value without walls.
double ductSeries(double y, double z, double a, double b, double G, double mu);
double planeProfile(double y, double a, double G, double mu);
double poiseuilleL2(const Fields& F, bool wallsY, bool wallsZ, double G, double mu, const std::string& base);

}  // namespace lbmdrv
