// ============================================================================
//  ref_harness.cpp -- TEST INFRASTRUCTURE ONLY (the oracle checker).
//
//  C entry points around the reference solver's own public C++ API
//  (class lbm::LBM, src/utils/lbm.hpp:19-84, whose data members are public
//  "for I/O and tests", lbm.hpp:64-78). The recipe in oracle/Makefile compiles
//  this file together with the reference's unmodified sources into
//  oracle/_ref/libref_harness.so. Nothing in the product links it: only the
//  tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
//
//  What the harness adds over the reference CLI (src/main.cpp):
//    * a 3-D initial orientation (the CLI only sets e from an in-plane angle,
//      src/utils/squirmer.cpp:26-27), written into the public sq.e after the
//      constructor -- the initial flag map does not depend on e;
//    * raw FP64 access to f, rho, u, flag and the squirmer state.
// ============================================================================
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <stdexcept>
#include <string>

#include "analytic.hpp"
#include "io.hpp"
#include "lbm.hpp"
#include "params.hpp"

namespace {
struct RefHandle {
    lbm::Params p;
    lbm::LBM* L = nullptr;
    long t = 0;
};
void put_err(char* err, int n, const char* msg) {
    if (err && n > 0) { std::snprintf(err, (size_t)n, "%s", msg); }
}
}  // namespace

extern "C" {

// kv: nargs strings "key=value" (the reference's own key set, params.cpp:37-75).
void* ref_create(int nargs, const char* const* kv, char* err, int errlen) {
    RefHandle* h = new RefHandle();
    try {
        for (int k = 0; k < nargs; ++k) {
            std::string a = kv[k];
            const auto eq = a.find('=');
            if (eq == std::string::npos) throw std::runtime_error("expected key=value: " + a);
            h->p.set(a.substr(0, eq), a.substr(eq + 1));
        }
        h->p.validate();
        h->L = new lbm::LBM(h->p);
    } catch (const std::exception& e) {
        put_err(err, errlen, e.what());
        delete h;
        return nullptr;
    }
    return h;
}

void ref_destroy(void* hp) {
    RefHandle* h = (RefHandle*)hp;
    if (!h) return;
    delete h->L;
    delete h;
}

void ref_set_orientation(void* hp, double ex, double ey, double ez) {
    RefHandle* h = (RefHandle*)hp;
    const double n = std::sqrt(ex * ex + ey * ey + ez * ez);
    h->L->sq.e[0] = ex / n; h->L->sq.e[1] = ey / n; h->L->sq.e[2] = ez / n;
}

void ref_step(void* hp) { ((RefHandle*)hp)->L->step(); }
void ref_advance_squirmer(void* hp) { ((RefHandle*)hp)->L->advanceSquirmer(); }
void ref_correct_mass(void* hp) { ((RefHandle*)hp)->L->correctMass(); }

// The time loop of src/main.cpp:60-64 without I/O: step, advanceSquirmer,
// correctMass every mass_correction_every steps (squirmer runs only).
// traj (optional, may be null): rows of 15 doubles every traj_every steps,
// laid out as the trajectory file columns (src/utils/io.cpp:79-83).
int ref_run(void* hp, int nsteps, double* traj, int max_rows) {
    RefHandle* h = (RefHandle*)hp;
    lbm::LBM& L = *h->L;
    int rows = 0;
    for (int k = 0; k < nsteps; ++k) {
        const long t = ++h->t;
        L.step();
        if (L.hasSquirmer) {
            L.advanceSquirmer();
            if (h->p.massCorrectionEvery > 0 && t % h->p.massCorrectionEvery == 0) L.correctMass();
            if (traj && t % h->p.trajEvery == 0 && rows < max_rows) {
                const lbm::Squirmer& s = L.sq;
                double* r = traj + 15 * rows;
                r[0] = (double)t;
                for (int d = 0; d < 3; ++d) {
                    r[1 + d] = s.X[d]; r[4 + d] = s.e[d]; r[7 + d] = s.U[d]; r[10 + d] = s.W[d];
                }
                r[13] = s.Fw[1]; r[14] = s.Fw[2];
                ++rows;
            }
        }
    }
    return rows;
}

long ref_time(void* hp) { return ((RefHandle*)hp)->t; }
long ref_ncells(void* hp) { return (long)((RefHandle*)hp)->L->N; }

void ref_get_f(void* hp, double* out) {
    const lbm::LBM& L = *((RefHandle*)hp)->L;
    std::memcpy(out, L.f.data(), L.f.size() * sizeof(double));
}
void ref_set_f(void* hp, const double* in) {
    lbm::LBM& L = *((RefHandle*)hp)->L;
    std::memcpy(L.f.data(), in, L.f.size() * sizeof(double));
}
void ref_get_fields(void* hp, unsigned char* flag, double* rho, double* u3) {
    const lbm::LBM& L = *((RefHandle*)hp)->L;
    for (size_t n = 0; n < L.N; ++n) {
        if (flag) flag[n] = L.flag[n];
        if (rho) rho[n] = L.rho[n];
        if (u3) { u3[3 * n] = L.ux[n]; u3[3 * n + 1] = L.uy[n]; u3[3 * n + 2] = L.uz[n]; }
    }
}
// Squirmer state: X[3] e[3] U[3] W[3] Fh[3] Th[3] Fc[3] Tc[3] Fw[3] contacts M I FS
void ref_squirmer_state(void* hp, double* o) {
    const lbm::Squirmer& s = ((RefHandle*)hp)->L->sq;
    for (int d = 0; d < 3; ++d) {
        o[d] = s.X[d]; o[3 + d] = s.e[d]; o[6 + d] = s.U[d]; o[9 + d] = s.W[d];
        o[12 + d] = s.Fh[d]; o[15 + d] = s.Th[d]; o[18 + d] = s.Fc[d]; o[21 + d] = s.Tc[d];
        o[24 + d] = s.Fw[d];
    }
    o[27] = (double)s.contacts; o[28] = s.M; o[29] = s.I; o[30] = s.FS;
}
// Overwrite the mutable rigid-body state (X, e, U, W) -- used to start
// single-step parity cases from a seeded state.
void ref_set_squirmer_state(void* hp, const double* X, const double* e, const double* U, const double* W) {
    lbm::Squirmer& s = ((RefHandle*)hp)->L->sq;
    for (int d = 0; d < 3; ++d) { s.X[d] = X[d]; s.e[d] = e[d]; s.U[d] = U[d]; s.W[d] = W[d]; }
}
void ref_wall_force(void* hp, double* o) {
    const lbm::LBM& L = *((RefHandle*)hp)->L;
    o[0] = L.wallForce[0]; o[1] = L.wallForce[1]; o[2] = L.wallForce[2];
}
// countFluid, meanDensity, maxSpeed, sumUx (src/utils/lbm.cpp:342-364)
void ref_diag(void* hp, double* o) {
    const lbm::LBM& L = *((RefHandle*)hp)->L;
    o[0] = (double)L.countFluid(); o[1] = L.meanDensity(); o[2] = L.maxSpeed(); o[3] = L.sumUx();
}
// Relative L2 error against the exact Poiseuille/duct solution, and the
// profile files <base>_profile_{y,z}.dat (src/utils/analytic.cpp:27-64).
double ref_poiseuille_error(void* hp, const char* base) {
    return lbm::poiseuilleError(*((RefHandle*)hp)->L, base);
}
double ref_duct_velocity(double y, double z, double a, double b, double G, double mu) {
    return lbm::ductVelocity(y, z, a, b, G, mu);
}
void ref_write_vtk(void* hp, const char* path) { lbm::writeVTK(*((RefHandle*)hp)->L, path); }

}  // extern "C"
