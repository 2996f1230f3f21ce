// ============================================================================
//  params.cpp -- key = value parsing for the host driver (behaviour of
//  src/utils/params.cpp:37-157: keys, aliases, booleans, messages).
// ============================================================================
#include "params.hpp"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <fstream>
#include <functional>
#include <map>
#include <stdexcept>

namespace lbmdrv {

namespace {

std::string strip(const std::string& s) {
    size_t b = 0, e = s.size();
    while (b < e && std::isspace((unsigned char)s[b])) ++b;
    while (e > b && std::isspace((unsigned char)s[e - 1])) --e;
    return s.substr(b, e - b);
}

std::string lowercase(std::string s) {
    for (char& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

bool parseBool(const std::string& v) {
    static const std::map<std::string, bool> words = {{"1", true},  {"true", true},   {"yes", true}, {"on", true},
                                                      {"0", false}, {"false", false}, {"no", false}, {"off", false}};
    auto it = words.find(lowercase(v));
    if (it == words.end()) throw std::runtime_error("cannot interpret '" + v + "' as a boolean");
    return it->second;
}

using Setter = std::function<void(Params&, const std::string&)>;

Setter asInt(int Params::*m) { return [m](Params& p, const std::string& v) { p.*m = std::stoi(v); }; }
Setter asReal(double Params::*m) { return [m](Params& p, const std::string& v) { p.*m = std::stod(v); }; }
Setter asFlag(bool Params::*m) { return [m](Params& p, const std::string& v) { p.*m = parseBool(v); }; }
Setter asText(std::string Params::*m) { return [m](Params& p, const std::string& v) { p.*m = v; }; }
Setter asAxis(double Params::*m) {
    return [m](Params& p, const std::string& v) { p.*m = std::stod(v); p.useOrientation = true; };
}

// every accepted key, aliases included (params.cpp:40-70, plus additions)
const std::map<std::string, Setter>& keyTable() {
    static const std::map<std::string, Setter> t = {
        {"nx", asInt(&Params::NX)}, {"ny", asInt(&Params::NY)}, {"nz", asInt(&Params::NZ)},
        {"tau", asReal(&Params::tau)}, {"lambda", asReal(&Params::Lambda)},
        {"fx", asReal(&Params::Fx)}, {"fy", asReal(&Params::Fy)}, {"fz", asReal(&Params::Fz)},
        {"walls_y", asFlag(&Params::wallsY)}, {"wallsy", asFlag(&Params::wallsY)},
        {"walls_z", asFlag(&Params::wallsZ)}, {"wallsz", asFlag(&Params::wallsZ)},
        {"steps", asInt(&Params::steps)},
        {"print_every", asInt(&Params::printEvery)}, {"print", asInt(&Params::printEvery)},
        {"vtk_every", asInt(&Params::vtkEvery)}, {"vtk", asInt(&Params::vtkEvery)},
        {"traj_every", asInt(&Params::trajEvery)}, {"traj", asInt(&Params::trajEvery)},
        {"tol", asReal(&Params::tol)},
        {"mass_correction_every", asInt(&Params::massCorrectionEvery)},
        {"output_dir", asText(&Params::outputDir)}, {"prefix", asText(&Params::prefix)},
        {"squirmer", asFlag(&Params::squirmer)}, {"sq", asFlag(&Params::squirmer)},
        {"radius", asReal(&Params::R)}, {"r", asReal(&Params::R)},
        {"b1", asReal(&Params::B1)}, {"beta", asReal(&Params::beta)},
        {"rho_p", asReal(&Params::rhoP)}, {"rhop", asReal(&Params::rhoP)},
        {"x0", asReal(&Params::x0)}, {"y0", asReal(&Params::y0)}, {"z0", asReal(&Params::z0)},
        {"angle", asReal(&Params::angle)}, {"planar", asFlag(&Params::planar)},
        {"eps", asReal(&Params::eps)}, {"hc", asReal(&Params::hc)}, {"hmin", asReal(&Params::hmin)},
        {"ex", asAxis(&Params::ex)}, {"ey", asAxis(&Params::ey)}, {"ez", asAxis(&Params::ez)},
        {"device", asInt(&Params::device)},
        {"checkpoint_every", asInt(&Params::checkpointEvery)},
        {"restart", asText(&Params::restart)},
        {"precision",
         [](Params& p, const std::string& v) {
             const std::string l = lowercase(strip(v));
             if (l == "fp64") p.precision = LBMGPU_FP64;
             else if (l == "fp32") p.precision = LBMGPU_FP32;
             else if (l == "fp16") p.precision = LBMGPU_FP16;
             else throw std::runtime_error("precision must be one of fp64, fp32, fp16");
         }},
    };
    return t;
}

}  // namespace

void Params::set(const std::string& keyIn, const std::string& value) {
    const std::string key = lowercase(strip(keyIn));
    const auto& t = keyTable();
    auto it = t.find(key);
    if (it == t.end()) throw std::runtime_error("unknown parameter '" + key + "'");
    try {
        it->second(*this, value);
    } catch (const std::invalid_argument&) {
        throw std::runtime_error("invalid value '" + value + "' for parameter '" + key + "'");
    }
}

void Params::loadFile(const std::string& path) {
    std::ifstream in(path);
    if (!in) throw std::runtime_error("cannot open input file '" + path + "'");
    std::string line;
    for (int lineNo = 1; std::getline(in, line); ++lineNo) {
        line = strip(line.substr(0, line.find('#')));
        if (line.empty()) continue;
        const size_t eq = line.find('=');
        if (eq == std::string::npos)
            throw std::runtime_error(path + ":" + std::to_string(lineNo) + ": expected 'key = value'");
        try {
            set(line.substr(0, eq), strip(line.substr(eq + 1)));
        } catch (const std::runtime_error& e) {
            throw std::runtime_error(path + ":" + std::to_string(lineNo) + ": " + e.what());
        }
    }
}

void Params::parseCommandLine(int argc, char** argv) {
    for (int k = 1; k < argc; ++k) {
        const std::string a = argv[k];
        const size_t eq = a.find('=');
        if (eq == std::string::npos) loadFile(a);
        else set(a.substr(0, eq), a.substr(eq + 1));
    }
}

void Params::validate() const {
    // The rules of params.cpp:120-140 live in the library (lbmgpu_validate);
    // steps and print_every are host-loop settings checked here, in the
    // reference's order: lattice and fluid, then steps, then the intervals,
    // then the squirmer.
    char msg[256];
    lbmgpu_params c = toC();
    c.squirmer = 0;
    c.traj_every = 1;
    if (lbmgpu_validate(&c, msg, sizeof msg) != LBMGPU_OK) throw std::runtime_error(msg);
    if (steps < 0) throw std::runtime_error("steps must be >= 0");
    if (printEvery < 1 || trajEvery < 1) throw std::runtime_error("print_every and traj_every must be >= 1");
    c = toC();
    if (lbmgpu_validate(&c, msg, sizeof msg) != LBMGPU_OK) throw std::runtime_error(msg);
}

// Startup banner, the layout of params.cpp:145-157.
void Params::print(std::FILE* fp) const {
    std::fprintf(fp, "grid        : %d x %d x %d\n", NX, NY, NZ);
    std::fprintf(fp, "fluid       : tau = %.4f (nu = %.5f), TRT Lambda = %.4f, F = (%.3e, %.3e, %.3e)\n", tau,
                 (tau - 0.5) / 3.0, Lambda, Fx, Fy, Fz);
    std::fprintf(fp, "walls       : y %s, z %s (x periodic)\n", wallsY ? "on" : "off", wallsZ ? "on" : "off");
    std::fprintf(fp, "run         : %d steps, output '%s/%s_*'\n", steps, outputDir.c_str(), prefix.c_str());
    if (!squirmer) return;
    const double U0 = 2.0 * B1 / 3.0, nu = (tau - 0.5) / 3.0;
    std::fprintf(fp, "squirmer    : R = %.2f, B1 = %.4f, beta = %+.2f (%s), U0 = %.5f, Re = 2RU0/nu = %.3f\n", R, B1,
                 beta, beta < 0 ? "pusher" : (beta > 0 ? "puller" : "neutral"), U0, 2 * R * U0 / nu);
    std::fprintf(fp, "              angle = %.1f deg, rho_p = %.2f, planar = %d\n", angle, rhoP, (int)planar);
    std::fprintf(fp, "wall pot.   : eps = %.3f (F_max = eps F_S), hc = %.2f, hmin = %.2f\n", eps, hc, hmin);
}

lbmgpu_params Params::toC() const {
    lbmgpu_params c;
    lbmgpu_params_default(&c);
    c.nx = NX; c.ny = NY; c.nz = NZ;
    c.tau = tau; c.lambda = Lambda; c.fx = Fx; c.fy = Fy; c.fz = Fz;
    c.walls_y = wallsY; c.walls_z = wallsZ;
    c.traj_every = trajEvery; c.mass_correction_every = massCorrectionEvery;
    c.squirmer = squirmer;
    c.radius = R; c.b1 = B1; c.beta = beta; c.rho_p = rhoP;
    c.x0 = x0; c.y0 = y0; c.z0 = z0; c.angle = angle; c.planar = planar;
    c.eps = eps; c.hc = hc; c.hmin = hmin;
    c.use_orientation = useOrientation; c.ex = ex; c.ey = ey; c.ez = ez;
    c.precision = precision; c.device = device;
    return c;
}

}  // namespace lbmdrv
