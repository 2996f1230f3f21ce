// ============================================================================
//  lbm_common.cuh -- lattice constants, node-flag bits, storage forms and the
//  device-side records shared by the kernels of liblbmgpu.
// ============================================================================
#pragma once
#include <cmath>
#include <cstdint>
#include <cuda_fp16.h>

namespace lbmgpu {

// ---- D3Q19, in the reference's order (src/utils/lattice.hpp:18-30) --------
// Opposite pairs (1,2)(3,4)...(17,18); the order fixes the summation order of
// the moments, which the FP64 path keeps identical to the reference's.
constexpr int Q = 19;

__host__ __device__ constexpr int CX(int i) {
    constexpr int t[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
    return t[i];
}
__host__ __device__ constexpr int CY(int i) {
    constexpr int t[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
    return t[i];
}
__host__ __device__ constexpr int CZ(int i) {
    constexpr int t[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
    return t[i];
}
__host__ __device__ constexpr int OPP(int i) { return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1); }
__host__ __device__ constexpr double WD(int i) { return i == 0 ? 1.0 / 3.0 : (i <= 6 ? 1.0 / 18 : 1.0 / 36); }
__host__ __device__ constexpr float WF(int i) { return i == 0 ? 1.0f / 3.0f : (i <= 6 ? 1.0f / 18 : 1.0f / 36); }

// ---- node flag byte ---------------------------------------------------------
// bits 0-1: node type, same values as the reference's NodeType
//           (lattice.hpp:36) so the byte's low bits are what the VTK writes;
// bit 2   : FLUID node with at least one WALL neighbour (static);
// bit 3   : FLUID node with at least one PARTICLE neighbour (rebuilt with the
//           boundary-link list whenever the sphere's mapping changes).
// A FLUID node with bits 2-3 clear streams all 19 populations without a
// single neighbour-type lookup.
constexpr uint8_t T_FLUID = 0, T_WALL = 1, T_PARTICLE = 2;
constexpr uint8_t TYPE_MASK = 3, NEAR_WALL = 4, NEAR_PARTICLE = 8;

// ---- status bits (device error word) --------------------------------------
constexpr int ST_NAN = 1;            // non-finite force/torque/state
constexpr int ST_REMAP_RANGE = 2;    // squirmer moved >= 1 cell in one step
constexpr int ST_LINK_OVERFLOW = 4;  // boundary-link list exceeded its capacity
constexpr int ST_REMAP_OVERFLOW = 8; // more changed nodes than the remap can order
constexpr int ST_WATCHDOG = 16;      // a bounded wait for staged data gave up

// ---- storage forms ----------------------------------------------------------
// FP64: f_i itself. FP32 / FP16: the deviation f_i - w_i rho0 (rho0 = 1), FP16
// scaled by 2^12 so that typical deviations (1e-8 .. 0.05) stay normal.
// The stream kernels work in storage units: ld/st/rt move the stored number
// as it is (for FP16 the scaled deviation), and SC / INV convert between
// storage units and deviations (1 for FP32, so its arithmetic is unchanged).
// T2 is the 2-element vector of the stored type (two x-adjacent nodes).
// A is the arithmetic of the collision in each form. FP32 storage computes in
// FP64: the moments of the stored numbers and the TRT update are then exact
// enough that the collision conserves mass and momentum to FP64 rounding, and
// the only FP32 rounding left is the store. (In FP32 arithmetic the moments'
// rounding is re-injected into the flow every step; over the 10000 steps of the
// 256x128x128 squirmer lattice that left u 1e-4 away from the FP64 form, against
// 1e-8 with FP64 arithmetic.) FP16 storage keeps FP32 arithmetic: its storage
// rounding (2^-11) dominates either way.
struct StoreF64 {
    using T = double;
    using T2 = double2;
    using A = double;
    static constexpr bool shifted = false;
    static constexpr float SC = 1.0f, INV = 1.0f;
    __device__ static double ld(const T* p) { return *p; }
    __device__ static void st(T* p, double v) { *p = v; }
    // streaming store (evict first): the bulk's stores, read again only next step
    __device__ static void st_cs(T* p, double v) { __stcs(p, v); }
    __device__ static double rt(double v) { return v; }  // value as it will be stored
};
struct StoreF32 {
    using T = float;
    using T2 = float2;
    using A = double;
    static constexpr bool shifted = true;
    static constexpr float SC = 1.0f, INV = 1.0f;
    __device__ static float ld(const T* p) { return *p; }
    __device__ static void st(T* p, float v) { *p = v; }
    __device__ static void st_cs(T* p, float v) { __stcs(p, v); }
    __device__ static float rt(float v) { return v; }
    __device__ static float2 ld2(const T* p) { return *reinterpret_cast<const float2*>(p); }
    __device__ static void st2(T* p, float a, float b) { *reinterpret_cast<float2*>(p) = make_float2(a, b); }
    __device__ static void st2_cs(T* p, float a, float b) { __stcs(reinterpret_cast<float2*>(p), make_float2(a, b)); }
};
constexpr float FP16_SCALE = 4096.0f, FP16_INV_SCALE = 1.0f / 4096.0f;
struct StoreF16 {
    using T = __half;
    using T2 = __half2;
    using A = float;
    static constexpr bool shifted = true;
    static constexpr float SC = FP16_SCALE, INV = FP16_INV_SCALE;
    __device__ static float ld(const T* p) { return __half2float(*p); }
    __device__ static void st(T* p, float v) { *p = __float2half_rn(v); }
    __device__ static void st_cs(T* p, float v) {
        __stcs(reinterpret_cast<unsigned short*>(p), __half_as_ushort(__float2half_rn(v)));
    }
    __device__ static float rt(float v) { return __half2float(__float2half_rn(v)); }
    __device__ static float2 ld2(const T* p) { return __half22float2(*reinterpret_cast<const __half2*>(p)); }
    __device__ static void st2(T* p, float a, float b) {
        *reinterpret_cast<__half2*>(p) = __floats2half2_rn(a, b);
    }
    __device__ static void st2_cs(T* p, float a, float b) {
        const __half2 h = __floats2half2_rn(a, b);
        __stcs(reinterpret_cast<unsigned int*>(p), *reinterpret_cast<const unsigned int*>(&h));
    }
};

// ---- lattice description (kernel argument, fixed per handle) ---------------
struct Lattice {
    int nx, ny, nz;
    unsigned N;            // nx*ny*nz (< 2^31)
    unsigned nxy;
    int walls_y, walls_z;
    double omP, omM, gP, gM, F[3];  // TRT rates and Guo factors (lbm.cpp:65-69, :129)
    // FP32 copies and per-direction forcing constants of the shifted forms:
    // cF[i] = c_i . F and cm[i] = gM * 3 w_i (c_i . F) for the odd i of each pair
    float omPf, omMf, gPf, gMf, Ff[3], uFh[3];
    // gP w per weight class (0: rest, 1: axes, 2: diagonals), formed once here
    // so that every kernel's FP32 Guo term rounds the same way
    float gPw[3];
    float cF[Q], cm[Q];
    int force_free;        // F = 0: the Guo source terms vanish (FP32 arithmetic skips them)
    // 1 and -0, held in the kernel argument so that the compiler cannot see
    // their values: the two-node FP32 arithmetic forms every operation as an
    // FMA with one of them (k_stream.cuh, Paired)
    float one, mzero;
};

// ---- the zone around the sphere ----------------------------------------------
// A box of fixed width around the sphere. Its fluid nodes are updated by the
// zone kernel, which runs after the squirmer update of the previous step; the
// bulk kernel skips them and so need not wait for that update. lo is the
// lower corner (unwrapped along y/z walls, wrapped into [0, n) along periodic
// axes); w the width actually covered (at most the lattice extent). Zones are
// kept for three consecutive steps (slot = step mod 3): the squirmer update of
// step s writes the zone of step s + 2 while steps s + 1 read theirs.
struct ZoneBox {
    int lo[3], w[3];
};
constexpr int ZONE_SLOTS = 3;
// Cells around the remap box. The zone of step s + 2 is laid out around the
// box of the position after step s; it must hold (a) every node whose flags
// the squirmer update after step s + 1 changes (inside the box of the next
// position) and (b) every node whose density that update's refill reads
// (inside that box too), whose densities the zone kernel of step s + 1 stored
// from the zone laid out one step earlier. The centre moves less than one cell
// per step (checked: ST_REMAP_RANGE), so across two steps each box bound
// shifts by at most 2 cells.
constexpr int ZONE_MARGIN = 2;

// Zone width along an axis: the remap box (lbm.cpp:273-275) is at most
// 2*ceil(R) + 6 cells wide; the zone adds ZONE_MARGIN cells on each side.
__host__ __device__ inline int zone_width(double R, int n, bool wall_axis) {
    const int w = 2 * (int)ceil(R) + 6 + 2 * ZONE_MARGIN;
    return wall_axis ? w : (w < n ? w : n);
}

// The zone around remap box [blo, blo + bw) along one axis.
__host__ __device__ inline void zone_axis(int blo, int n, int w, bool wall_axis, int& lo) {
    lo = blo - ZONE_MARGIN;
    if (!wall_axis) lo = w >= n ? 0 : ((lo % n) + n) % n;
}

__host__ __device__ inline bool in_zone_axis(int c, int lo, int w, int n, bool wall_axis) {
    int d = c - lo;
    if (!wall_axis && d < 0) d += n;
    return d >= 0 && d < w;
}

// ---- squirmer / run state on the device ------------------------------------
// Everything the per-step kernels need to decide and compute without a host
// round trip. FP64 throughout.
struct SqState {
    // model (squirmer.hpp:16-18, :35-36)
    double R, B1, beta, M, I, eps, hc, hmin, FS;
    int planar, present;
    // rigid-body state (squirmer.hpp:22-31)
    double X[3], e[3], U[3], W[3];
    double Fh[3], Th[3], Fc[3], Tc[3], Fw[3];
    long long contacts;
    // step bookkeeping
    long long t;                 // completed squirmer updates (= time steps in run mode)
    long long n_fluid;           // number of FLUID nodes
    int mass_every, traj_every;
    int corr_pending;            // apply f_i += w_i * corr_d on the next load
    double corr_d;
    // zones of the next steps (slot = step mod 3)
    ZoneBox zone[ZONE_SLOTS];
    // boundary-link list
    int n_links;
    // last wall force (written on macro steps)
    double wall_force[3];
    // trajectory ring
    long long traj_count;
    int status;
};

// The shell of remap candidates (nodes whose distance to a reference centre
// is within R +- (1.05 + SHELL_SLACK)), kept between squirmer updates. While
// the centre stays within SHELL_SLACK of the reference centre, every node that
// can change type lies in it.
struct ShellCache {
    double X[3];   // reference centre (unwrapped, like SqState::X)
    int n;         // candidates in the list
    int valid;     // 0: rebuild on the next remap
};
constexpr double SHELL_SLACK = 0.75;

constexpr int TRAJ_RING = 4096;
constexpr int TRAJ_COLS = 15;

// Per-node partial sums written by the stream kernel for boundary-link nodes:
// F (3), T (3), and two spare slots.
constexpr int LINK_PART = 8;
// Per-block partials of the stream kernel on reduction steps: wall force (3), mass (1).
constexpr int BLOCK_PART = 4;

struct StreamArgs {
    void* f;                      // populations, SoA f[i*N + n]
    uint8_t* flag;
    double* rho;                  // pre-collision moments (FP64)
    double* ux; double* uy; double* uz;
    double* link_part;            // [n_links][LINK_PART], one row per near-particle node
    const int* linkslot;          // node -> its row of link_part
    double* block_part;           // bulk kernel: [blocks][BLOCK_PART]
    double* block_part_b;         // zone kernel: [blocks][BLOCK_PART]
    const int* wallrows;          // (y, z) of the fluid rows next to a wall
    int n_wallrows;
    int zone_cells;               // cells of the zone grid (zone width product bound)
    int zw[3];                    // zone grid extents (fixed per lattice)
    SqState* sq;
    // per-step settings, fixed at launch (hence in a captured graph):
    int zslot;                    // zone slot of this step
    int do_mass;                  // sum the stored populations (a correction step)
    int apply_corr;               // add the pending correction on load (after one)
    int* row_claim;               // staged-row bulk: row counter and CTAs done (RowsWork)
};

// ---- ensembles (k_batch.cuh) -------------------------------------------------
constexpr int BATCH_MAX_NX = 256;   // longest x-row of an ensemble member

// Programmatic dependent launch. A kernel launched with programmatic stream
// serialisation may start before its predecessor in the stream has finished;
// pdl_wait() blocks until that predecessor has completed and its writes are
// visible, so it comes before the first read of anything the predecessor
// writes. pdl_launch_dependents() lets the successor start early. Both are
// no-ops for an ordinary launch.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

struct RowRef {
    int m, y, z;       // member, row coordinates
    int part;          // entry of the row's partial sums (member base + y + ny*z)
};
struct RunRef {        // nrow consecutive rows [y0, y0 + nrow) of one member's plane z: contiguous nodes
    int m, y0, z, nrow;
};
struct ChunkRef {      // 32 consecutive nodes [x0, x0 + 32) of one row (the last may be short)
    int m, y, z, x0;
};
struct RowChunks {     // the chunks of one row, and where its partial sums go
    int first, count, part, pad;
};
struct BatchStep {     // per-step settings shared by all members
    int zslot, do_mass, apply_corr;
};
struct SqStep {        // per-step settings of the members' squirmer updates
    int parity, stages, corr_step, zslot_a, zslot_b;
};
struct MemberParts {   // where a member's partial sums live
    int row0, nrow, nzb;  // ny*nz row entries from row0 (wall layers stay 0), zone blocks
};

}  // namespace lbmgpu
