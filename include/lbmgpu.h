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

/* Asynchronous snapshot of the same fields, for writers that run beside the
 * time loop (replaces the reference's writeVTK reading the solver's host
 * arrays between two steps, io.cpp:44-67 called from main.cpp:67).
 * lbmgpu_snapshot_begin queues, after the work already issued on the
 * handle's stream, a device-side copy of the node types, rho and u of the
 * last step into a snapshot buffer of the handle (allocated on the first
 * call, 33 bytes per node) and returns at once: the time loop may continue.
 * lbmgpu_snapshot_read waits for that copy only (not for steps queued after
 * it) and copies the snapshot into the host buffers, laid out as for
 * lbmgpu_fields, on a stream of its own, so the copy overlaps the steps
 * running meanwhile. It may be called from another host thread while the
 * owning thread keeps advancing the lattice (it touches only the snapshot);
 * its failures are reported by lbmgpu_snapshot_last_error. One snapshot at a
 * time: _begin returns LBMGPU_ERR_INVALID while the previous one is unread.
 * Host buffers from lbmgpu_host_alloc make the copies faster. */
int lbmgpu_snapshot_begin(lbmgpu_handle* h);
int lbmgpu_snapshot_read(lbmgpu_handle* h, uint8_t* flag, double* rho, double* u3);
const char* lbmgpu_snapshot_last_error(const lbmgpu_handle* h);

/* Page-locked host memory (cudaHostAlloc) for buffers that receive fields or
 * snapshots: the device copies into it directly instead of through a staging
 * buffer. NULL on failure; free with lbmgpu_host_free. */
void* lbmgpu_host_alloc(size_t bytes);
int lbmgpu_host_free(void* p);

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

/* Checkpoint / restart (no counterpart in the reference, which cannot resume
 * a run). A checkpoint is the complete device state of a lattice in a host
 * buffer: the stored populations (storage form and AA parity as they are),
 * flags, rho/u of the last step, the squirmer state with its zones, pending
 * mass correction and counters, the boundary-link list and the trajectory
 * ring, behind a header that records the deck the state belongs to (sizes,
 * storage form, walls, tau, lambda, body force, cadences, squirmer model).
 * Loading it into a lattice created with the same parameters continues the
 * run bit for bit. _size gives the bytes _save needs. _load validates the
 * whole buffer on the host before anything reaches the device: the header
 * against the lattice's parameters, every link node index (inside the
 * lattice, ascending, a fluid node next to the sphere), the zone boxes, the
 * counters and the node types against the wall layers. A mismatch or a
 * corrupt buffer returns LBMGPU_ERR_INVALID and leaves the lattice as it was.
 * _check runs the same validation against parameters alone (no device, no
 * handle), e.g. to reject a restart file before creating the lattice. */
int lbmgpu_checkpoint_size(lbmgpu_handle* h, size_t* bytes);
int lbmgpu_checkpoint_save(lbmgpu_handle* h, void* buf, size_t len);
int lbmgpu_checkpoint_load(lbmgpu_handle* h, const void* buf, size_t len);
int lbmgpu_checkpoint_check(const lbmgpu_params* p, const void* buf, size_t len, char* msg, size_t msg_len);

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

/* Failure detection without a fault: runs the bounded wait the device kernels
 * use on an mbarrier that nothing arrives at, giving up after `limit` tries
 * (1 .. 2^22; the kernels themselves use 2^22). *status receives the device
 * status bits (16 = the watchdog gave up); the call returns
 * LBMGPU_ERR_WATCHDOG in that case, as lbmgpu_run and lbmgpu_batch_run do
 * when a wait of theirs gives up, and the device stays usable. No
 * counterpart in the reference (its CPU loop has no waits to bound). */
int lbmgpu_watchdog_selftest(int device, long long limit, int* status);

/* Message of the last failure on this handle (or of lbmgpu_create on the
 * calling thread when h is NULL). Never NULL. */
const char* lbmgpu_last_error(const lbmgpu_handle* h);

int lbmgpu_abi_version(void);

/* ---------------------------------------------------------------------------
 * Swimmer surrogate network (no counterpart in the reference).
 *
 * A multilayer perceptron 4 -> 64 -> 64 -> 64 -> 3 with SiLU after each
 * hidden layer, trained and evaluated by the library's own kernels: one CTA
 * runs the whole network forward and backward on a tile of 32 samples, and a
 * second kernel sums the tiles' gradients in a fixed order and takes one
 * Adam step on the FP32 master parameters. With bf16 = 1 every matrix product
 * uses BF16 operands on the tensor cores with FP32 accumulation; with bf16 = 0
 * it is computed in FP32.
 * Parameters (LBMGPU_MLP_NPARAMS floats): W1[64][4] b1[64] W2[64][64] b2[64]
 * W3[64][64] b3[64] W4[3][64] b4[3], each W[out][in]. Loss: mean over samples
 * and outputs of the squared error. Inputs x[n][4], targets/outputs y[n][3],
 * FP32, row-major. Errors: lbmgpu_mlp_last_error.
 * ------------------------------------------------------------------------- */
#define LBMGPU_MLP_IN 4
#define LBMGPU_MLP_HIDDEN 64
#define LBMGPU_MLP_OUT 3
#define LBMGPU_MLP_NPARAMS (64 * 4 + 64 + 64 * 64 + 64 + 64 * 64 + 64 + 3 * 64 + 3)
typedef struct lbmgpu_mlp lbmgpu_mlp;
int lbmgpu_mlp_create(int device, int bf16, lbmgpu_mlp** out);   /* parameters 0 */
int lbmgpu_mlp_destroy(lbmgpu_mlp* m);
int lbmgpu_mlp_set_params(lbmgpu_mlp* m, const float* params, int reset_optimizer);
int lbmgpu_mlp_get_params(lbmgpu_mlp* m, float* params);
/* Adam hyper-parameters (defaults 0.9, 0.999, 1e-8). */
int lbmgpu_mlp_set_adam(lbmgpu_mlp* m, float beta1, float beta2, float eps);
/* Training set, copied to the device. */
int lbmgpu_mlp_set_data(lbmgpu_mlp* m, const float* x, const float* y, int n);
/* Adam steps over consecutive minibatches of `batch` samples taken from the
 * training set in the given order (indices into the training set); returns
 * the mean of the minibatch losses in *mean_loss (may be NULL). */
int lbmgpu_mlp_train_epoch(lbmgpu_mlp* m, const int* order, int n_order, int batch, float lr, float* mean_loss);
/* Loss and gradient (LBMGPU_MLP_NPARAMS floats, may be NULL) over the whole
 * training set at the current parameters; no update. */
int lbmgpu_mlp_loss_grad(lbmgpu_mlp* m, float* loss, float* grad);
/* Inference: y[n][3] = net(x[n][4]). BF16 networks run on the tensor cores
 * through tensor memory (tcgen05.mma, 128 samples per CTA, FP32
 * accumulators in TMEM); FP32 networks on the warp-tiled FP32 kernel.
 * lbmgpu_mlp_forward_ex chooses the path: LBMGPU_MLP_PATH_AUTO (as above),
 * LBMGPU_MLP_PATH_WARP (the warp-tiled training kernel's forward: mma.sync
 * for BF16, FMA for FP32) or LBMGPU_MLP_PATH_TCGEN05 (BF16 networks only). */
#define LBMGPU_MLP_PATH_AUTO 0
#define LBMGPU_MLP_PATH_WARP 1
#define LBMGPU_MLP_PATH_TCGEN05 2
int lbmgpu_mlp_forward(lbmgpu_mlp* m, const float* x, int n, float* y);
int lbmgpu_mlp_forward_ex(lbmgpu_mlp* m, const float* x, int n, float* y, int path);
const char* lbmgpu_mlp_last_error(const lbmgpu_mlp* m);

/* ---------------------------------------------------------------------------
 * Allocation-free diagnostics (no counterpart in the reference: its
 * diagnostics, lbm.cpp:342-364, read the solver's own host arrays).
 *
 * lbmgpu_field_stats_static computes what lbmgpu_diag reports (count of FLUID
 * nodes, mean density, max |u| and sum of u_x over FLUID nodes) for fields
 * that live in the CALLER's device memory: flag (N bytes, LBMGPU_FLUID = 0 in
 * the low two bits), rho, ux, uy, uz (N doubles each), all on the current
 * device. wall_force is not computed and is returned as 0.
 *
 * Who needs it: callers that keep their own lattice fields on the GPU and
 * cannot allocate when they want the statistics. Creating a handle allocates
 * about 100 bytes per node. cudaMalloc/cudaFree may synchronise the whole
 * device and fail once HBM is committed to the populations. Code that must not
 * stall other streams, or that runs with the memory already spoken for (a
 * monitor polling a running time loop, a caller near the memory limit),
 * therefore uses this entry point. It allocates no device memory: its reduction
 * scratch is a static device array of the library (512 KB per device).
 *
 * Limit: 1 <= n_nodes <= LBMGPU_STATIC_STATS_MAX_NODES (2^25 nodes, e.g.
 * 256^3 x 2); larger sizes return LBMGPU_ERR_INVALID with a message.
 * Set-up: the first call on each device looks up the scratch's address
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * The lookup is repeated when the device's context has been recreated
 * (cudaDeviceReset), whose module load may place the array elsewhere.
 * Concurrency: the scratch is one per device and shared by all callers, so
 * calls that overlap on a device (from several host threads, or on several
 * streams) race and corrupt each other's results: serialise them.
 * The call queues its work on cuda_stream (NULL: the legacy default stream)
 * and returns after that stream has finished it. Errors are reported by
 * lbmgpu_last_error(NULL) on the calling thread. */
#define LBMGPU_STATIC_STATS_MAX_NODES 33554432LL
int lbmgpu_field_stats_static(const uint8_t* flag, const double* rho, const double* ux, const double* uy,
                              const double* uz, long long n_nodes, void* cuda_stream, lbmgpu_diagnostics* out);

/* ---------------------------------------------------------------------------
 * Ensembles (no counterpart in the reference, whose executable runs one
 * lattice per process; parameter studies there launch the binary once per
 * case, e.g. postprocessing/lbm_post.py:39-56 driving src/main.cpp).
 *
 * An ensemble advances n independent lattices ("members") together: one
 * persistent bulk launch per step covers the rows of every member, one launch
 * the zones around all squirmers and one the squirmer updates (a CTA per
 * member), captured in CUDA graphs. Each member follows exactly the same
 * arithmetic as a lattice created alone with lbmgpu_create, so its results
 * are those of lbmgpu_run on that lattice.
 * Members may differ in size (nx, ny, nz), squirmer geometry, swimming
 * parameters, initial orientation and output cadence; they must share tau,
 * lambda, the body force, the walls, precision, mass_correction_every,
 * squirmer (on/off) and device.
 * ------------------------------------------------------------------------- */
typedef struct lbmgpu_batch lbmgpu_batch;

/* Creates the n members from ps[0..n-1]. On failure *out is NULL and the
 * message is available from lbmgpu_batch_last_error(NULL). */
int lbmgpu_batch_create(const lbmgpu_params* ps, int n, lbmgpu_batch** out);
int lbmgpu_batch_destroy(lbmgpu_batch* b);

/* nsteps time steps of every member (the loop body of lbmgpu_run). */
int lbmgpu_batch_run(lbmgpu_batch* b, int nsteps);

/* The handle of member i, for the read-only calls: lbmgpu_time,
 * lbmgpu_squirmer_state, lbmgpu_fields, lbmgpu_diag, lbmgpu_traj_rows,
 * lbmgpu_get_populations, lbmgpu_launch_count, lbmgpu_last_error. Calls that
 * advance or modify a member on its own return LBMGPU_ERR_INVALID. The handle
 * is owned by the ensemble (do not destroy it). */
int lbmgpu_batch_member(lbmgpu_batch* b, int i, lbmgpu_handle** h);

/* Number of members and total lattice nodes (either pointer may be NULL). */
int lbmgpu_batch_size(const lbmgpu_batch* b, int* members, long long* cells);

/* Tiling of the bulk launch.
 *   tile = 32, 64 or 128: every CTA walks rows with that many threads per
 *     x-row, loading populations straight from global memory;
 *   tile = LBMGPU_TILE_ROWCTA: one CTA of 128 threads per row (grid = rows,
 *     ctas_per_sm unused);
 *   tile = LBMGPU_TILE_CHUNK: one warp per 32 consecutive nodes of a row
 *     (grid = chunks / 4, ctas_per_sm unused);
 *   tile = LBMGPU_TILE_CHUNKP: the same chunks walked by persistent warps
 *     (grid = ctas_per_sm x SMs, 4 warps per CTA);
 *   tile = LBMGPU_TILE_RUNS: on steps without sums, runs of consecutive rows
 *     of one member's z-plane (contiguous in memory) are copied into
 *     shared memory by bulk asynchronous copies, several runs deep, while
 *     eight warps per CTA update the runs already staged (grid = ctas_per_sm
 *     x SMs, persistent); steps with sums use the persistent chunks;
 *   tile = LBMGPU_TILE_STAGED3 / _STAGED4: each CTA owns a contiguous range
 *     of rows (equal node counts); a producer warp stages every row's
 *     populations and flags in shared memory with bulk asynchronous copies,
 *     3 or 4 rows deep, while four warps update the rows already staged.
 * ctas_per_sm (1..16): the grid is that many CTAs per SM. */
#define LBMGPU_TILE_ROWCTA 1
#define LBMGPU_TILE_CHUNK 2
#define LBMGPU_TILE_CHUNKP 3
#define LBMGPU_TILE_RUNS 4
#define LBMGPU_TILE_STAGED3 (-3)
#define LBMGPU_TILE_STAGED4 (-4)
int lbmgpu_batch_set_tiling(lbmgpu_batch* b, int tile, int ctas_per_sm);

/* Times the bulk launch for every tiling candidate, `reps` pairs of launches
 * each, and keeps the fastest. The populations are saved to a temporary
 * device buffer before and restored after, so the ensemble's state is
 * unchanged. Outputs (may be NULL): the chosen tiling and its time per launch. */
int lbmgpu_batch_autotune(lbmgpu_batch* b, int reps, int* tile, int* ctas_per_sm, double* best_ms);

/* Measurement aid: average device time of one bulk launch over all members
 * with the current tiling (2*reps launches; the populations advance without
 * the sphere update, as in lbmgpu_time_kernels). */
int lbmgpu_batch_time_bulk(lbmgpu_batch* b, int reps, double* ms_per_launch);

/* Runs the ensemble's caller-facing work on this cudaStream_t (NULL: the
 * ensemble's own stream). The stream stays the caller's: it is not destroyed
 * with the ensemble. */
int lbmgpu_batch_set_stream(lbmgpu_batch* b, void* cuda_stream);
int lbmgpu_batch_launch_count(const lbmgpu_batch* b, long long* n);
const char* lbmgpu_batch_last_error(const lbmgpu_batch* b);

#ifdef __cplusplus
}
#endif
#endif /* LBMGPU_H */
