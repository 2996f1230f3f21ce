// ============================================================================
//  lbm_squirmer_gpu -- drop-in replacement of the reference's lbm_squirmer
//  executable (src/main.cpp) running the time loop on a B200 through the C
//  ABI of include/lbmgpu.h.
//
//  Usage:  lbm_squirmer_gpu <input_file> [key=value ...]
//
//  Same input files, overrides, console lines and result files as the
//  reference. The device runs the steps between two host events (print,
//  VTK, end, or a full trajectory ring) without a host round trip; trajectory
//  rows recorded on the device are written after each such stretch.
// ============================================================================
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <future>
#include <iterator>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "output.hpp"
#include "params.hpp"

using namespace lbmdrv;

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr long long kTrajRing = 4096;  // rows the device ring holds (lbmgpu_traj_rows)

struct Device {
    lbmgpu_handle* h = nullptr;
    ~Device() { if (h) lbmgpu_destroy(h); }
    void check(int rc) const {
        if (rc != LBMGPU_OK) throw std::runtime_error(std::string("device: ") + lbmgpu_last_error(h));
    }
    Fields fields(const Params& p) const {
        Fields F;
        F.nx = p.NX; F.ny = p.NY; F.nz = p.NZ;
        F.flag.resize(F.size()); F.rho.resize(F.size()); F.u.resize(3 * F.size());
        check(lbmgpu_fields(h, F.flag.data(), F.rho.data(), F.u.data()));
        return F;
    }
    lbmgpu_diagnostics diag() const {
        lbmgpu_diagnostics d;
        check(lbmgpu_diag(h, &d));
        return d;
    }
    lbmgpu_squirmer squirmer() const {
        lbmgpu_squirmer s;
        check(lbmgpu_squirmer_state(h, &s));
        return s;
    }
};

// VTK snapshots written beside the time loop: the device packs the fields of
// the snapshot step into a buffer of its own (lbmgpu_snapshot_begin) and the
// loop goes on; a writer thread copies them into page-locked host buffers
// (lbmgpu_snapshot_read) and writes the file. One snapshot is in flight at a
// time: the next one first waits for the previous file.
class SnapshotWriter {
public:
    SnapshotWriter(const Device& dev, const Params& p) : dev_(dev) {
        view_.nx = p.NX; view_.ny = p.NY; view_.nz = p.NZ;
        const size_t N = view_.size();
        flag_ = static_cast<uint8_t*>(lbmgpu_host_alloc(N));
        rho_ = static_cast<double*>(lbmgpu_host_alloc(N * sizeof(double)));
        u_ = static_cast<double*>(lbmgpu_host_alloc(3 * N * sizeof(double)));
        if (!flag_ || !rho_ || !u_) throw std::runtime_error("cannot allocate page-locked snapshot buffers");
        view_.flag = flag_; view_.rho = rho_; view_.u = u_;
    }
    ~SnapshotWriter() {
        if (pending_.valid()) pending_.wait();
        lbmgpu_host_free(flag_); lbmgpu_host_free(rho_); lbmgpu_host_free(u_);
    }
    void write(const std::string& path) {
        finish();
        dev_.check(lbmgpu_snapshot_begin(dev_.h));
        pending_ = std::async(std::launch::async, [this, path] {
            if (lbmgpu_snapshot_read(dev_.h, flag_, rho_, u_) != LBMGPU_OK)
                throw std::runtime_error(std::string("device: ") + lbmgpu_snapshot_last_error(dev_.h));
            writeVtk(view_, path);
        });
    }
    void finish() {   // rethrows a failure of the previous write
        if (pending_.valid()) pending_.get();
    }
private:
    const Device& dev_;
    FieldsView view_;
    uint8_t* flag_ = nullptr;
    double* rho_ = nullptr;
    double* u_ = nullptr;
    std::future<void> pending_;
};

void drainTrajectory(const Device& dev, TrajectoryFile& traj) {
    static double rows[1024 * 15];
    for (;;) {
        int n = 0;
        long long dropped = 0;
        dev.check(lbmgpu_traj_rows(dev.h, rows, 1024, &n, &dropped));
        if (dropped) throw std::runtime_error("trajectory rows were overwritten before being written");
        for (int k = 0; k < n; ++k) traj.append(rows + 15 * k);
        if (n < 1024) return;
    }
}

int runSimulation(const Params& p) {
    const std::string base = p.outputDir + "/" + p.prefix;
    std::printf("================ lbm-squirmer ================\n");
    p.print(stdout);
    std::printf("==============================================\n");

    Device dev;
    const lbmgpu_params cp = p.toC();
    if (lbmgpu_create(&cp, &dev.h) != LBMGPU_OK)
        throw std::runtime_error(std::string("device: ") + lbmgpu_last_error(nullptr));
    int t = 0;
    if (!p.restart.empty()) {   // continue a checkpointed run: same parameters, state from the file
        std::ifstream in(p.restart, std::ios::binary);
        if (!in) throw std::runtime_error("cannot read '" + p.restart + "'");
        const std::vector<char> buf((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
        dev.check(lbmgpu_checkpoint_load(dev.h, buf.data(), buf.size()));
        long long t0 = 0;
        dev.check(lbmgpu_time(dev.h, &t0));
        t = (int)t0;
        std::printf("restarted from %s at t=%d\n", p.restart.c_str(), t);
    }
    std::unique_ptr<TrajectoryFile> traj;
    if (p.squirmer) traj = std::make_unique<TrajectoryFile>(base + "_traj.dat", !p.restart.empty());
    const double nu = (p.tau - 0.5) / 3.0;

    std::unique_ptr<SnapshotWriter> snaps;
    if (p.vtkEvery > 0) snaps = std::make_unique<SnapshotWriter>(dev, p);

    const auto t0 = std::chrono::steady_clock::now();
    double prevSum = 0.0;
    bool converged = false;
    while (t < p.steps) {
        // the next step at which the host has something to do (main.cpp:60-87)
        long long next = std::min<long long>(p.steps, (long long)(t / p.printEvery + 1) * p.printEvery);
        if (p.vtkEvery > 0) next = std::min<long long>(next, (long long)(t / p.vtkEvery + 1) * p.vtkEvery);
        if (p.squirmer) next = std::min<long long>(next, t + kTrajRing * p.trajEvery);
        if (p.checkpointEvery > 0)
            next = std::min<long long>(next, (long long)(t / p.checkpointEvery + 1) * p.checkpointEvery);
        dev.check(lbmgpu_run(dev.h, (int)(next - t)));
        t = (int)next;
        if (p.squirmer) drainTrajectory(dev, *traj);
        if (snaps && t % p.vtkEvery == 0) snaps->write(base + "_" + std::to_string(t) + ".vtk");
        if (p.checkpointEvery > 0 && t % p.checkpointEvery == 0) {
            if (traj) traj->flush();
            size_t n = 0;
            dev.check(lbmgpu_checkpoint_size(dev.h, &n));
            std::vector<char> buf(n);
            dev.check(lbmgpu_checkpoint_save(dev.h, buf.data(), n));
            const std::string path = base + "_checkpoint.bin", tmp = path + ".tmp";
            std::ofstream out(tmp, std::ios::binary);
            out.write(buf.data(), (std::streamsize)n);
            out.close();
            if (!out || std::rename(tmp.c_str(), path.c_str()) != 0)
                throw std::runtime_error("cannot write '" + path + "'");
        }
        if (t % p.printEvery == 0) {
            if (p.squirmer) {
                const lbmgpu_squirmer s = dev.squirmer();
                const double U0 = 2.0 * s.B1 / 3.0;
                std::printf("t=%8d  X=(%9.2f,%7.2f,%7.2f)  angle=%7.2f deg  |U|/U0=%.3f  <rho>=%.6f\n", t, s.X[0], s.X[1],
                            s.X[2], std::atan2(s.e[1], s.e[0]) * 180.0 / kPi,
                            std::sqrt(s.U[0] * s.U[0] + s.U[1] * s.U[1] + s.U[2] * s.U[2]) / U0,
                            dev.diag().mean_density);
                traj->flush();
            } else {
                const lbmgpu_diagnostics d = dev.diag();
                const double change = std::fabs(d.sum_ux - prevSum) / (std::fabs(d.sum_ux) + 1e-30);
                prevSum = d.sum_ux;
                std::printf("t=%8d  u_max=%.6e  F_wall_x=%.6e  rel.change=%.3e\n", t, d.max_speed, d.wall_force[0], change);
                if (p.tol > 0 && change < p.tol) { converged = true; std::fflush(stdout); break; }
            }
            std::fflush(stdout);
        }
    }
    if (snaps) snaps->finish();
    const int done = converged ? t : p.steps;
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    const double ncell = (double)p.NX * p.NY * p.NZ;
    std::printf("%d steps in %.1f s (%.2f MLUPS)\n", done, sec, sec > 0 ? 1e-6 * ncell * done / sec : 0.0);

    // final output (main.cpp:93-112)
    const Fields F = dev.fields(p);
    writeVtk(F, base + "_final.vtk");
    const lbmgpu_diagnostics d = dev.diag();
    std::FILE* sum = std::fopen((base + "_summary.txt").c_str(), "w");
    if (!sum) throw std::runtime_error("cannot write '" + base + "_summary.txt'");
    std::fprintf(sum, "steps %d\nconverged %d\nnu %.10g\nmean_density %.10g\nmax_speed %.10g\n", done, (int)converged,
                 nu, d.mean_density, d.max_speed);
    std::fprintf(sum, "wall_force %.10g %.10g %.10g\n", d.wall_force[0], d.wall_force[1], d.wall_force[2]);
    const double nf = (double)d.n_fluid;
    std::fprintf(sum, "body_force_total %.10g %.10g %.10g\n", p.Fx * nf, p.Fy * nf, p.Fz * nf);
    if (p.squirmer) {
        const lbmgpu_squirmer s = dev.squirmer();
        writeSquirmerState(s, nu, done, base + "_squirmer.dat");
        std::printf("hard-gap safety activations: %lld steps\n", s.contacts);
        std::fprintf(sum, "contacts %lld\n", s.contacts);
    } else {
        const double err = poiseuilleL2(F, p.wallsY, p.wallsZ, p.Fx, nu, base);
        if (err >= 0) {
            std::printf("relative L2 error vs exact Poiseuille solution: %.4e\n", err);
            std::fprintf(sum, "l2_error %.10g\n", err);
        }
    }
    std::fclose(sum);
    std::printf("output written to %s_*\n", base.c_str());
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <input_file> [key=value ...]\n", argv[0]);
        return 1;
    }
    Params p;
    try {
        p.parseCommandLine(argc, argv);
        p.validate();
        makeDirectory(p.outputDir);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    try {
        return runSimulation(p);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
}
