// ============================================================================
//  output.cpp -- result files in the reference's formats.
// ============================================================================
#include "output.hpp"

#include <cmath>
#include <cstring>
#include <filesystem>
#include <stdexcept>

namespace lbmdrv {

namespace {

constexpr double kPi = 3.14159265358979323846;

// legacy VTK binary data is big-endian
void putBigEndian(std::FILE* fp, const double* v, size_t n) {
    std::vector<unsigned char> buf(8 * n);
    for (size_t k = 0; k < n; ++k) {
        uint64_t bits;
        std::memcpy(&bits, &v[k], 8);
        for (int b = 0; b < 8; ++b) buf[8 * k + b] = (unsigned char)(bits >> (56 - 8 * b));
    }
    std::fwrite(buf.data(), 1, buf.size(), fp);
}

}  // namespace

void makeDirectory(const std::string& dir) {
    if (dir.empty()) return;
    std::error_code ec;
    std::filesystem::create_directories(dir, ec);
    if (ec) throw std::runtime_error("cannot create output directory '" + dir + "': " + ec.message());
}

// io.cpp:44-67: flag (u8), density (f64; 1 on solid nodes), velocity
// (3 x f64; 0 on solid nodes), STRUCTURED_POINTS with unit spacing.
void writeVtk(const FieldsView& F, const std::string& path) {
    std::FILE* fp = std::fopen(path.c_str(), "wb");
    if (!fp) throw std::runtime_error("cannot write '" + path + "'");
    const size_t N = F.size();
    std::fprintf(fp, "# vtk DataFile Version 3.0\nlbm-squirmer\nBINARY\nDATASET STRUCTURED_POINTS\n");
    std::fprintf(fp, "DIMENSIONS %d %d %d\nORIGIN 0 0 0\nSPACING 1 1 1\nPOINT_DATA %zu\n", F.nx, F.ny, F.nz, N);
    std::fprintf(fp, "SCALARS flag unsigned_char 1\nLOOKUP_TABLE default\n");
    std::fwrite(F.flag, 1, N, fp);
    std::fprintf(fp, "\n");
    std::vector<double> d(N);
    for (size_t n = 0; n < N; ++n) d[n] = F.flag[n] == LBMGPU_FLUID ? F.rho[n] : 1.0;
    std::fprintf(fp, "SCALARS density double 1\nLOOKUP_TABLE default\n");
    putBigEndian(fp, d.data(), N);
    std::fprintf(fp, "\n");
    std::vector<double> v(3 * N, 0.0);
    for (size_t n = 0; n < N; ++n)
        if (F.flag[n] == LBMGPU_FLUID) { v[3 * n] = F.u[3 * n]; v[3 * n + 1] = F.u[3 * n + 1]; v[3 * n + 2] = F.u[3 * n + 2]; }
    std::fprintf(fp, "VECTORS velocity double\n");
    putBigEndian(fp, v.data(), 3 * N);
    std::fprintf(fp, "\n");
    std::fclose(fp);
}

// io.cpp:72-83
TrajectoryFile::TrajectoryFile(const std::string& path, bool append) {
    fp_ = std::fopen(path.c_str(), append ? "a" : "w");
    if (!fp_) throw std::runtime_error("cannot write '" + path + "'");
    if (!append) std::fprintf(fp_, "# t X Y Z ex ey ez Ux Uy Uz Wx Wy Wz Fwall_y Fwall_z\n");
}
TrajectoryFile::~TrajectoryFile() {
    if (fp_) std::fclose(fp_);
}
void TrajectoryFile::flush() {
    if (fp_) std::fflush(fp_);
}
void TrajectoryFile::append(const double* r) {
    std::fprintf(fp_, "%d %.6f %.6f %.6f %.6f %.6f %.6f %.6e %.6e %.6e %.6e %.6e %.6e %.6e %.6e\n", (int)r[0], r[1],
                 r[2], r[3], r[4], r[5], r[6], r[7], r[8], r[9], r[10], r[11], r[12], r[13], r[14]);
}

// io.cpp:87-97
void writeSquirmerState(const lbmgpu_squirmer& s, double nu, int t, const std::string& path) {
    std::FILE* fp = std::fopen(path.c_str(), "w");
    if (!fp) throw std::runtime_error("cannot write '" + path + "'");
    std::fprintf(fp, "t %d\nR %.10g\nB1 %.10g\nbeta %.10g\nU0 %.10g\nnu %.10g\nFS %.10g\n", t, s.R, s.B1, s.beta,
                 s.U0, nu, s.FS);
    std::fprintf(fp, "X %.10g %.10g %.10g\ne %.10g %.10g %.10g\n", s.X[0], s.X[1], s.X[2], s.e[0], s.e[1], s.e[2]);
    std::fprintf(fp, "U %.10g %.10g %.10g\nW %.10g %.10g %.10g\ncontacts %lld\n", s.U[0], s.U[1], s.U[2], s.W[0],
                 s.W[1], s.W[2], s.contacts);
    std::fclose(fp);
}

// Rectangular duct -a<y<a, -b<z<b driven by G: series over odd n < 400 with
// cosh(k|z|)/cosh(kb) evaluated without overflow (analytic.cpp:11-21).
double ductSeries(double y, double z, double a, double b, double G, double mu) {
    double sum = 0.0;
    for (int n = 1; n < 400; n += 2) {
        const double k = n * kPi / (2.0 * a), A = k * std::fabs(z), B = k * b;
        const double ratio = std::exp(A - B) * (1.0 + std::exp(-2.0 * A)) / (1.0 + std::exp(-2.0 * B));
        const double sign = ((n - 1) / 2) % 2 == 0 ? 1.0 : -1.0;
        sum += sign * (1.0 - ratio) * std::cos(k * y) / ((double)n * n * n);
    }
    return 16.0 * a * a * G / (mu * kPi * kPi * kPi) * sum;
}

double planeProfile(double y, double a, double G, double mu) { return G / (2.0 * mu) * (a * a - y * y); }

// analytic.cpp:27-64
double poiseuilleL2(const Fields& F, bool wallsY, bool wallsZ, double G, double mu, const std::string& base) {
    if (!wallsY && !wallsZ) return -1.0;
    const double yc = 0.5 * (F.ny - 1), zc = 0.5 * (F.nz - 1);
    const double a = 0.5 * (F.ny - 2), b = 0.5 * (F.nz - 2);
    auto exact = [&](int y, int z) {
        if (wallsY && wallsZ) return ductSeries(y - yc, z - zc, a, b, G, mu);
        if (wallsY) return planeProfile(y - yc, a, G, mu);
        return planeProfile(z - zc, b, G, mu);
    };
    auto at = [&](int y, int z) { return (size_t)F.nx * ((size_t)y + (size_t)F.ny * z); };
    double num = 0, den = 0;
    for (int z = 0; z < F.nz; ++z)
        for (int y = 0; y < F.ny; ++y) {
            const size_t n = at(y, z);
            if (F.flag[n] != LBMGPU_FLUID) continue;
            const double ue = exact(y, z), ux = F.u[3 * n];
            num += (ux - ue) * (ux - ue);
            den += ue * ue;
        }
    const int zm = F.nz / 2, ym = F.ny / 2;
    if (std::FILE* fp = std::fopen((base + "_profile_y.dat").c_str(), "w")) {
        std::fprintf(fp, "# y-yc  ux_lbm  ux_exact   (z = %d)\n", zm);
        for (int y = 0; y < F.ny; ++y)
            if (F.flag[at(y, zm)] == LBMGPU_FLUID)
                std::fprintf(fp, "%9.3f %.10e %.10e\n", y - yc, F.u[3 * at(y, zm)], exact(y, zm));
        std::fclose(fp);
    }
    if (std::FILE* fp = std::fopen((base + "_profile_z.dat").c_str(), "w")) {
        std::fprintf(fp, "# z-zc  ux_lbm  ux_exact   (y = %d)\n", ym);
        for (int z = 0; z < F.nz; ++z)
            if (F.flag[at(ym, z)] == LBMGPU_FLUID)
                std::fprintf(fp, "%9.3f %.10e %.10e\n", z - zc, F.u[3 * at(ym, z)], exact(ym, z));
        std::fclose(fp);
    }
    return den > 0 ? std::sqrt(num / den) : -1.0;
}

}  // namespace lbmdrv
