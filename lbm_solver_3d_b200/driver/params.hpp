// ============================================================================
//  params.hpp -- the host driver's parameter set.
//
//  The same keys, aliases, defaults, file syntax, command-line override order,
//  validation rules and messages as lbm::Params (src/utils/params.hpp:14-63,
//  src/utils/params.cpp:37-157), so existing input decks and command lines run
//  unchanged. Added keys: precision (fp64 | fp32 | fp16), ex/ey/ez (a 3-D
//  initial orientation instead of `angle`), device, checkpoint_every and
//  restart (checkpoint / restart of the whole device state).
// ============================================================================
#pragma once
#include <cstdio>
#include <string>

#include "../../include/lbmgpu.h"

namespace lbmdrv {

struct Params {
    int NX = 64, NY = 34, NZ = 32;
    double tau = 1.0, Lambda = 3.0 / 16.0, Fx = 0.0, Fy = 0.0, Fz = 0.0;
    bool wallsY = true, wallsZ = false;
    int steps = 10000, printEvery = 1000, vtkEvery = 0, trajEvery = 50;
    double tol = 0.0;
    int massCorrectionEvery = 10;
    std::string outputDir = "outputs", prefix = "run";
    bool squirmer = false;
    double R = 4.0, B1 = 0.015, beta = 0.0, rhoP = 1.0;
    double x0 = -1, y0 = -1, z0 = -1, angle = 30.0;
    bool planar = true;
    double eps = 0.2, hc = 2.0, hmin = 0.5;
    // additions
    int precision = LBMGPU_FP64;
    bool useOrientation = false;
    double ex = 0.0, ey = 0.0, ez = 0.0;
    int device = 0;
    int checkpointEvery = 0;          // write <prefix>_checkpoint.bin every this many steps (0: never)
    std::string restart;              // continue from this checkpoint file

    void set(const std::string& key, const std::string& value);  // throws std::runtime_error
    void loadFile(const std::string& path);
    void parseCommandLine(int argc, char** argv);
    void validate() const;
    void print(std::FILE* fp) const;
    lbmgpu_params toC() const;
};

}  // namespace lbmdrv
