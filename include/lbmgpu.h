/* ============================================================================
 *  lbmgpu.h -- C ABI of the B200 (sm_100a) D3Q19 TRT + squirmer solver.
 *
 *  This is the drop-in boundary for the per-step hot path of the lbm-squirmer
 *  solver. In the reference the boundary is the C++ class lbm::LBM
 *  (src/utils/lbm.hpp:19-84): constructor, step(), advanceSquirmer(),
 *  correctMass(), the const diagnostics and the public host arrays read by the
 *  output writers. Here the same operations are plain C functions over an
 *  opaque handle; the library owns all device memory, no C++ exception crosses
 *  the boundary, and every function returns an int status (LBMGPU_OK = 0,
 *  negative on failure; lbmgpu_last_error() gives the message).
 *
 *  Threading: a handle is used by one host thread at a time. Distinct handles
 *  are independent and may run on different streams or devices.
 * ==========================================================================*/
#ifndef LBMGPU_H
#define LBMGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBMGPU_ABI_VERSION 1

/* ---- status codes -------------------------------------------------------
 * The reference reports failures as std::runtime_error caught once in main
 * (src/main.cpp:38-45). Here they are return codes. */
#define LBMGPU_OK            0
#define LBMGPU_ERR_INVALID  -1  /* invalid parameters or arguments (params.cpp:120-140 rules) */
#define LBMGPU_ERR_CUDA     -2  /* a CUDA runtime call failed */
#define LBMGPU_ERR_NAN      -3  /* non-finite force, torque or rigid-body state on the device */
#define LBMGPU_ERR_DEVICE   -4  /* a device-side consistency check failed (see message) */
#define LBMGPU_ERR_NOMEM    -5  /* device allocation failed */
#define LBMGPU_ERR_WATCHDOG -6  /* a bounded device wait gave up */

/* ---- population storage ("precision forms") ----------------------------- */
#define LBMGPU_FP64  0  /* f_i stored and computed in FP64 (the plain method)          */
#define LBMGPU_FP32  1  /* f_i - w_i rho0 stored in FP32, FP32 arithmetic               */
#define LBMGPU_FP16  2  /* f_i - w_i rho0 stored as scaled FP16, FP32 arithmetic        */

/* ---- node types (src/utils/lattice.hpp:36) ------------------------------- */
#define LBMGPU_FLUID    0
#define LBMGPU_WALL     1
#define LBMGPU_PARTICLE 2

/* POD mirror of lbm::Params (src/utils/params.hpp:14-56) restricted to what
 * the device needs, plus the additions of this library (last block). Fill it
 * with lbmgpu_params_default() first: the defaults are the reference's. */
typedef struct lbmgpu_params {
    /* grid (params.hpp:16) */
    int nx, ny, nz;
    /* fluid (params.hpp:20-22) */
    double tau, lambda, fx, fy, fz;
    /* boundaries, x always periodic (params.hpp:26-27) */
    int walls_y, walls_z;
    /* run control that the device loop needs (params.hpp:34, :36) */
    int traj_every, mass_correction_every;
    /* squirmer (params.hpp:42-50) */
    int squirmer;
    double radius, b1, beta, rho_p, x0, y0, z0, angle;
    int planar;
    /* soft wall potential (params.hpp:54-56) */
    double eps, hc, hmin;
    /* --- additions --- */
    int use_orientation;      /* 1: initial orientation (ex,ey,ez) instead of `angle` */
    double ex, ey, ez;
    int precision;            /* LBMGPU_FP64 / LBMGPU_FP32 / LBMGPU_FP16 */
    int device;               /* CUDA device ordinal */
} lbmgpu_params;

/* Squirmer state (src/utils/squirmer.hpp:16-37). */
typedef struct lbmgpu_squirmer {
    double X[3], e[3], U[3], W[3];
    double Fh[3], Th[3];      /* momentum-exchange force/torque of the last step */
    double Fc[3], Tc[3];      /* cover/uncover momentum pending for the next integrate */
    double Fw[3];             /* soft wall force of the last update */
    double R, B1, beta, M, I, FS, U0;
    long long contacts;       /* hard-gap activations (lbm.cpp:248-249) */
} lbmgpu_squirmer;

/* Diagnostics (src/utils/lbm.cpp:342-364) plus the wall force (lbm.hpp:74). */
typedef struct lbmgpu_diagnostics {
    long long n_fluid;        /* countFluid */
    double mean_density;      /* meanDensity: mean of rho over fluid nodes */
    double max_speed;         /* maxSpeed */
    double sum_ux;            /* sumUx */
    double wall_force[3];     /* momentum exchange with WALL nodes in the last step */
} lbmgpu_diagnostics;

typedef struct lbmgpu_handle lbmgpu_handle;

/* Reference defaults (params.hpp:16-56); precision FP64, device 0. */
void lbmgpu_params_default(lbmgpu_params* p);

/* Validation with the reference's rules and messages (params.cpp:120-140),
 * plus checks of the additions. Returns LBMGPU_OK or LBMGPU_ERR_INVALID and
 * writes the message into msg (may be NULL). Replaces Params::validate. */
int lbmgpu_validate(const lbmgpu_params* p, char* msg, size_t msg_len);

/* Replaces LBM::LBM(const Params&) (lbm.cpp:60-94): allocates the lattice on
 * the device, sets flags, f = w_i (rho = 1, u = 0) and maps the squirmer.
 * On failure *out is NULL; the message is available from
 * lbmgpu_last_error(NULL) on the calling thread. */
int lbmgpu_create(const lbmgpu_params* p, lbmgpu_handle** out);
int lbmgpu_destroy(lbmgpu_handle* h);

/* nsteps iterations of the reference time loop body (src/main.cpp:60-64):
 * LBM::step, then with a squirmer LBM::advanceSquirmer and LBM::correctMass
 * every mass_correction_every steps. Runs on the device without host
 * synchronisation inside (CUDA graphs); returns after queuing and checking
 * the device status word once at the end. Trajectory rows are recorded on
 * the device every traj_every steps (read them with lbmgpu_traj_rows). */
int lbmgpu_run(lbmgpu_handle* h, int nsteps);

/* The three reference calls one at a time, for callers that drive the loop
 * themselves: LBM::step (lbm.cpp:128-224), LBM::advanceSquirmer
 * (lbm.cpp:257-263) and LBM::correctMass (lbm.cpp:324-339). */
int lbmgpu_step(lbmgpu_handle* h);
int lbmgpu_advance_squirmer(lbmgpu_handle* h);
int lbmgpu_correct_mass(lbmgpu_handle* h);

/* Completed time steps. */
int lbmgpu_time(const lbmgpu_handle* h, long long* t);

/* Squirmer state (replaces reading lbm::LBM::sq, lbm.hpp:77). */
int lbmgpu_squirmer_state(lbmgpu_handle* h, lbmgpu_squirmer* s);

/* Host copies of the fields the output writers read (lbm.hpp:70-72): node
 * type per node (N bytes), rho (N doubles) and u as interleaved (ux,uy,uz)
 * (3N doubles), N = nx*ny*nz, node index n = x + nx*(y + ny*z). rho/u have
 * the reference's meaning: the pre-collision moments of the last step, with
 * uncovered nodes overridden by the refill. Any pointer may be NULL. */
int lbmgpu_fields(lbmgpu_handle* h, uint8_t* flag, double* rho, double* u3);

/* Diagnostics replacing countFluid/meanDensity/maxSpeed/sumUx and wallForce. */
int lbmgpu_diag(lbmgpu_handle* h, lbmgpu_diagnostics* d);

/* Trajectory rows recorded since the last call (15 doubles each, the columns
 * of src/utils/io.cpp:79-83: t X Y Z ex ey ez Ux Uy Uz Wx Wy Wz Fwall_y
 * Fwall_z). Writes at most max_rows rows; *nrows gets the number written.
 * The device ring holds 4096 rows; older unread rows are dropped and
 * counted in *dropped (may be NULL). */
int lbmgpu_traj_rows(lbmgpu_handle* h, double* rows, int max_rows, int* nrows, long long* dropped);

/* Populations in the reference layout f[i*N + n] as FP64 (lbm.hpp:58-59,
 * :69), whatever the storage precision. get reads the logical (post-stream)
 * populations including any pending mass correction; set overwrites them
 * (used for restart and for seeded parity cases). */
int lbmgpu_get_populations(lbmgpu_handle* h, double* f);
int lbmgpu_set_populations(lbmgpu_handle* h, const double* f);

/* Overwrite the rigid-body state X, e, U, W (seeded parity cases, restart).
 * The lattice mapping is not changed. */
int lbmgpu_set_squirmer_state(lbmgpu_handle* h, const double X[3], const double e[3],
                              const double U[3], const double W[3]);

/* Run all work of this handle on the given cudaStream_t (NULL: the library's
 * own stream). The stream must stay valid until reset or destroy. */
int lbmgpu_set_stream(lbmgpu_handle* h, void* cuda_stream);

/* Number of kernel launches this handle has issued (graph launches count
 * every kernel node they run). */
int lbmgpu_launch_count(const lbmgpu_handle* h, long long* n);

/* Measurement aid (no counterpart in the reference): times the kernels of one
 * time step separately with CUDA events on the handle's stream, `reps`
 * launches each (reps is rounded up to an even number so the AA parity is
 * preserved). ms[0] = bulk collide-stream kernel, ms[1] = boundary/zone
 * kernel (0 if there is none), ms[2] = squirmer kernel (0 without a squirmer);
 * averages per launch. The populations advance `reps` steps without the
 * sphere update in between, so the physical state is no longer meaningful
 * afterwards: use it on a handle kept for measurement. */
int lbmgpu_time_kernels(lbmgpu_handle* h, int reps, double ms[3]);

/* Message of the last failure on this handle (or of lbmgpu_create on the
 * calling thread when h is NULL). Never NULL. */
const char* lbmgpu_last_error(const lbmgpu_handle* h);

int lbmgpu_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* LBMGPU_H */
