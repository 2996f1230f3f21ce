// ============================================================================
//  lbmgpu.cu -- the C ABI (include/lbmgpu.h): handle, device memory, set-up
//  of the initial state, the CUDA-graph time loop and the host-facing
//  accessors.
//
//  Time loop (lbmgpu_run). Step s runs three kernels:
//    B(s)  k_bulk     every fluid node outside the zone (two launches when
//                     there are walls: the rows next to a wall are a launch
//                     of their own, on stream b ahead of Z(s), or on stream
//                     a after the rest of B(s) when the bulk is short and a
//                     squirmer's chain Z -> S is the longer path)
//    Z(s)  k_zone     the zone around the sphere
//    S(s)  k_squirmer rigid body, remap, link list, bookkeeping
//  on two streams, with exactly the dependencies the data needs:
//    B(s) after B(s-1), Z(s-1)          [+ S(s-1) if step s-1 was a mass-
//                                         correction step: B applies it]
//    Z(s) after B(s-1), Z(s-1), S(s-1)
//    S(s) after Z(s)                    [+ B(s) on correction steps: mass sums]
//  so S(s) overlaps B(s+1). Runs of steps are captured once into a CUDA graph
//  (the pattern repeats with period lcm(2, 3, k): AA parity, zone slot, mass
//  correction every k steps) and replayed.
// ============================================================================
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/lbmgpu.h"
#include "k_aux.cuh"
#include "k_batch.cuh"
#include "k_squirmer.cuh"
#include "launch.h"

using namespace lbmgpu;

namespace {

constexpr double PI = 3.14159265358979323846;
constexpr int DIAG_GRID = 296;
constexpr int MAX_PERIOD = 240;   // longest correction period captured in one graph pattern
constexpr int MIN_GRAPH = 48;     // steps per captured graph, at least

thread_local std::string g_create_error;

struct Graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int steps = 0;
};

}  // namespace

struct lbmgpu_handle {
    lbmgpu_params p{};
    Lattice L{};
    const Launchers* lz = nullptr;
    size_t esize = 8;
    int has_sq = 0;
    cudaStream_t own = nullptr, stream = nullptr;  // the caller-facing stream
    cudaStream_t zs = nullptr;                     // zone/squirmer stream (high priority)
    cudaStream_t cap = nullptr, cap2 = nullptr;    // graph capture streams
    cudaEvent_t ev_b[2] = {nullptr, nullptr}, ev_z = nullptr, ev_s = nullptr, ev_fork = nullptr, ev_join = nullptr;

    // device memory
    void* f = nullptr;
    uint8_t* flag = nullptr;
    double *rho = nullptr, *ux = nullptr, *uy = nullptr, *uz = nullptr;
    int* wallrows = nullptr;     // (y, z) pairs of rows next to a wall
    int* links = nullptr;
    int* linkslot = nullptr;
    int link_cap = 0;
    double* link_part = nullptr;
    double* block_part = nullptr;
    unsigned nblocks = 0;
    double* block_part_b = nullptr;
    unsigned nblocks_b = 0;
    int* row_claim = nullptr;      // staged-row bulk: row counter, CTAs done
    int* ordermap = nullptr;
    int* chg_node = nullptr;
    int* chg_key = nullptr;
    int* cand = nullptr;
    int* shell = nullptr;          // cached remap candidates
    ShellCache* shell_hdr = nullptr;
    uint8_t* mark = nullptr;
    int chg_cap = 0;
    double* traj = nullptr;
    SqState* sq = nullptr;
    double* scratch = nullptr;   // N doubles
    double* small = nullptr;     // reduction partials / results

    // launch geometry
    StreamGeom geom{};
    int zone_cells = 0, zw[3] = {0, 0, 0};
    int period = 6;              // steps after which the launch pattern repeats
    bool corr_in_graph = false;  // correction steps are part of the captured pattern
    bool wallrows_on_a = false;  // wall rows follow the bulk on stream a (short bulk, squirmer chain)

    // host mirrors
    long long t_main = 0;        // time steps issued (AA parity; step s = t_main + 1)
    long long traj_read = 0;
    long long launches = 0;
    bool pending_corr = false;   // a correction computed by the last step is still to be applied
    // captured step patterns; index 1: the first step applies the mass
    // correction computed by the step before the pattern
    Graph g[2];
    std::string err;
    // ensemble member: populations and flags live in the ensemble's pools,
    // work is issued by the ensemble on its streams
    bool member = false;

    // packed fields for the host (allocated on first use): rho (N doubles),
    // u interleaved (3N doubles), node types (N bytes) -- one buffer for
    // lbmgpu_fields, one for the asynchronous snapshot
    unsigned char* packed = nullptr;
    unsigned char* snap = nullptr;
    cudaStream_t snap_stream = nullptr;   // the snapshot's copies to the host
    cudaEvent_t snap_ready = nullptr;     // the snapshot's packing is done
    std::atomic<bool> snap_pending{false};
    std::string snap_err;
};

// ---------------------------------------------------------------------------
namespace {

int fail(lbmgpu_handle* h, int code, const std::string& msg) {
    if (h) h->err = msg; else g_create_error = msg;
    return code;
}

#define CUDA_TRY(h, call)                                                                          \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return fail(h, e_ == cudaErrorMemoryAllocation ? LBMGPU_ERR_NOMEM : LBMGPU_ERR_CUDA,    \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                       \
    } while (0)

const Launchers* launchers_for(int prec) {
    switch (prec) {
        case LBMGPU_FP64: return &launchers_f64();
        case LBMGPU_FP32: return &launchers_f32();
        case LBMGPU_FP16: return &launchers_f16();
        default: return nullptr;
    }
}

size_t esize_for(int prec) { return prec == LBMGPU_FP64 ? 8 : (prec == LBMGPU_FP32 ? 4 : 2); }

// The bulk kernel of steps without sums, where the lattice allows a choice:
// LBMGPU_BULK=rows (rows staged in shared memory, the default: two nodes per
// update thread in FP16 storage, one otherwise), rows1 (staged, one node per
// thread in every form), pair (two nodes per thread loaded from global memory,
// shifted forms) or node (one node per thread). The results are the same bit
// for bit; the variable exists to compare their speed.
int bulk_kind() {
    const char* e = std::getenv("LBMGPU_BULK");
    if (!e || !*e || !std::strcmp(e, "rows")) return 2;
    if (!std::strcmp(e, "rows1")) return 3;
    if (!std::strcmp(e, "pair")) return 1;
    return 0;
}

// SMs the persistent staged-row bulk leaves to the squirmer update of the
// second stream, whose CTA needs an SM to itself (a zone CTA fits beside the
// bulk's CTAs on any SM): LBMGPU_ROWS_RESERVE, else ROWS_RESERVE with a
// squirmer and none without one.
constexpr int ROWS_RESERVE = 2;
int rows_reserve(bool squirmer, int sms) {
    const char* e = std::getenv("LBMGPU_ROWS_RESERVE");
    int r = squirmer ? ROWS_RESERVE : 0;
    if (e && *e) r = std::atoi(e);
    return std::max(0, std::min(r, sms / 2));
}

// Capacity of the boundary-link list of a lattice with these parameters (the
// links lie inside the sphere's box, so the box volume bounds them).
int link_capacity(const lbmgpu_params& p) {
    const int box = p.squirmer ? 2 * (int)std::ceil(p.radius) + 8 : 1;
    return (int)((long long)box * box * box);
}

// Settings of time step s (1-based).
struct StepPlan {
    long long s;
    int par, zslot;
    bool corr;        // s is a mass-correction step
    bool apply;       // s applies the correction computed by step s - 1
    bool macro;       // s stores all macroscopic fields and the wall force
};

bool is_corr_step(const lbmgpu_handle* h, long long s) {
    const int k = h->p.mass_correction_every;
    return h->has_sq && k > 0 && s % k == 0;
}

StreamArgs stream_args(lbmgpu_handle* h, const StepPlan& sp) {
    StreamArgs a;
    a.f = h->f; a.flag = h->flag; a.rho = h->rho; a.ux = h->ux; a.uy = h->uy; a.uz = h->uz;
    a.link_part = h->link_part; a.linkslot = h->linkslot;
    a.block_part = h->block_part; a.block_part_b = h->block_part_b;
    a.wallrows = h->wallrows; a.n_wallrows = (int)h->geom.nwallrows;
    a.zone_cells = h->zone_cells;
    for (int d = 0; d < 3; ++d) a.zw[d] = h->zw[d];
    a.sq = h->sq;
    a.zslot = sp.zslot; a.do_mass = sp.corr ? 1 : 0; a.apply_corr = sp.apply ? 1 : 0;
    a.row_claim = h->row_claim;
    return a;
}

SqArgs squirmer_args(lbmgpu_handle* h, int parity, int stages, int corr_step, int za, int zb) {
    SqArgs a;
    a.f = h->f; a.flag = h->flag; a.rho = h->rho; a.ux = h->ux; a.uy = h->uy; a.uz = h->uz;
    a.links = h->links; a.linkslot = h->linkslot; a.link_cap = h->link_cap;
    a.link_part = h->link_part; a.block_part = h->block_part; a.nblocks = (int)h->nblocks;
    a.block_part_b = h->block_part_b; a.nblocks_b = (int)h->nblocks_b;
    a.block_part_w = nullptr; a.nblocks_w = 0;
    a.ordermap = h->ordermap; a.chg_node = h->chg_node; a.chg_key = h->chg_key; a.cand = h->cand; a.mark = h->mark;
    a.chg_cap = h->chg_cap; a.shell = h->shell; a.shell_hdr = h->shell_hdr;
    a.traj = h->traj; a.sq = h->sq; a.parity = parity; a.stages = stages;
    a.corr_step = corr_step; a.zslot_a = za; a.zslot_b = zb;
    return a;
}

// ---- small non-templated kernels -------------------------------------------
__global__ void k_fill_d(double* p, size_t n, double v) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) p[k] = v;
}
__global__ void k_fill_i(int* p, size_t n, int v) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) p[k] = v;
}
__global__ void k_scatter_slots(const int* links, int n, int* linkslot) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) linkslot[links[k]] = k;
}

// wall force of a macro step: fixed-order sum of both kernels' block partials
__global__ void k_finalize(const double* bp, unsigned nb, const double* bpz, unsigned nbz, SqState* sq) {
    __shared__ double red[8][3];
    double a0 = 0, a1 = 0, a2 = 0;
    for (unsigned b = threadIdx.x; b < nb + nbz; b += blockDim.x) {
        const double* q = b < nb ? bp + (size_t)b * BLOCK_PART : bpz + (size_t)(b - nb) * BLOCK_PART;
        a0 += q[0]; a1 += q[1]; a2 += q[2];
    }
    for (int o = 16; o > 0; o >>= 1) {
        a0 += __shfl_down_sync(0xffffffffu, a0, o);
        a1 += __shfl_down_sync(0xffffffffu, a1, o);
        a2 += __shfl_down_sync(0xffffffffu, a2, o);
    }
    if ((threadIdx.x & 31) == 0) { red[threadIdx.x >> 5][0] = a0; red[threadIdx.x >> 5][1] = a1; red[threadIdx.x >> 5][2] = a2; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0, s1 = 0, s2 = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { s0 += red[w][0]; s1 += red[w][1]; s2 += red[w][2]; }
        sq->wall_force[0] = s0; sq->wall_force[1] = s1; sq->wall_force[2] = s2;
    }
}

__global__ void k_clear_pending(SqState* sq) {
    if (threadIdx.x == 0) sq->corr_pending = 0;
}

// diagnostics (lbm.cpp:342-364): count, sum rho, max |u|, sum ux over fluid nodes
__global__ void k_diag_partial(unsigned N, const uint8_t* flag, const double* rho, const double* ux, const double* uy,
                               const double* uz, double* part) {
    __shared__ double red[8][4];
    double c = 0, m = 0, mx = 0, sx = 0;
    for (unsigned n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += gridDim.x * blockDim.x) {
        if ((flag[n] & TYPE_MASK) != T_FLUID) continue;
        c += 1.0; m += rho[n]; sx += ux[n];
        const double sp = sqrt(ux[n] * ux[n] + uy[n] * uy[n] + uz[n] * uz[n]);
        mx = fmax(mx, sp);
    }
    for (int o = 16; o > 0; o >>= 1) {
        c += __shfl_down_sync(0xffffffffu, c, o);
        m += __shfl_down_sync(0xffffffffu, m, o);
        mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
        sx += __shfl_down_sync(0xffffffffu, sx, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { red[w][0] = c; red[w][1] = m; red[w][2] = mx; red[w][3] = sx; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0, d = 0, e = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { a += red[k][0]; b += red[k][1]; d = fmax(d, red[k][2]); e += red[k][3]; }
        part[4 * blockIdx.x] = a; part[4 * blockIdx.x + 1] = b; part[4 * blockIdx.x + 2] = d; part[4 * blockIdx.x + 3] = e;
    }
}
__global__ void k_diag_final(const double* part, int nparts, double* out) {
    if (threadIdx.x != 0) return;
    double a = 0, b = 0, d = 0, e = 0;
    for (int k = 0; k < nparts; ++k) { a += part[4 * k]; b += part[4 * k + 1]; d = fmax(d, part[4 * k + 2]); e += part[4 * k + 3]; }
    out[0] = a; out[1] = b; out[2] = d; out[3] = e;
}

// The fields the writers read, packed for one copy each to the host: rho,
// u interleaved as (ux, uy, uz) per node, and the node type (low two flag bits).
__global__ void k_pack_fields(unsigned N, const uint8_t* __restrict__ flag, const double* __restrict__ rho,
                              const double* __restrict__ ux, const double* __restrict__ uy,
                              const double* __restrict__ uz, double* __restrict__ prho, double* __restrict__ pu,
                              uint8_t* __restrict__ pflag) {
    for (unsigned n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += gridDim.x * blockDim.x) {
        prho[n] = rho[n];
        pu[3 * (size_t)n] = ux[n];
        pu[3 * (size_t)n + 1] = uy[n];
        pu[3 * (size_t)n + 2] = uz[n];
        pflag[n] = flag[n] & TYPE_MASK;
    }
}

// ---- host-side restatement of the initial state ----------------------------
struct HostInit {
    std::vector<uint8_t> flag;
    std::vector<int> links;
    std::vector<int> wallrows;
    SqState s{};
};

size_t hidx(const lbmgpu_params& p, int x, int y, int z) { return (size_t)x + (size_t)p.nx * ((size_t)y + (size_t)p.ny * z); }

// LBM::offsetFromSquirmer (lbm.cpp:100-104)
void h_offset(const lbmgpu_params& p, const SqState& s, double px, double py, double pz, double r[3]) {
    r[0] = px - s.X[0]; r[0] -= p.nx * std::round(r[0] / p.nx);
    r[1] = py - s.X[1]; if (!p.walls_y) r[1] -= p.ny * std::round(r[1] / p.ny);
    r[2] = pz - s.X[2]; if (!p.walls_z) r[2] -= p.nz * std::round(r[2] / p.nz);
}

// the sphere's bounding box (lbm.cpp:272-276)
void h_box(const lbmgpu_params& p, const SqState& s, int lo[3], int w[3]) {
    const double R = s.R;
    int x0 = (int)std::floor(s.X[0] - R) - 2, x1 = (int)std::ceil(s.X[0] + R) + 2;
    int y0 = (int)std::floor(s.X[1] - R) - 2, y1 = (int)std::ceil(s.X[1] + R) + 2;
    int z0 = (int)std::floor(s.X[2] - R) - 2, z1 = (int)std::ceil(s.X[2] + R) + 2;
    if (p.walls_y) { y0 = std::max(0, y0); y1 = std::min(p.ny - 1, y1); }
    lo[0] = x0; lo[1] = y0; lo[2] = z0;
    w[0] = x1 - x0 + 1; w[1] = y1 - y0 + 1; w[2] = z1 - z0 + 1;
}

void set_zones(const lbmgpu_params& p, SqState& s) {
    int lo[3], w[3];
    h_box(p, s, lo, w);
    const int nd[3] = {p.nx, p.ny, p.nz};
    const bool wall_axis[3] = {false, p.walls_y != 0, p.walls_z != 0};
    for (int k = 0; k < ZONE_SLOTS; ++k)
        for (int d = 0; d < 3; ++d) {
            s.zone[k].w[d] = zone_width(s.R, nd[d], wall_axis[d]);
            zone_axis(lo[d], nd[d], s.zone[k].w[d], wall_axis[d], s.zone[k].lo[d]);
        }
}

bool near_wall(const lbmgpu_params& p, int y, int z) {
    return (p.walls_y && (y == 1 || y == p.ny - 2)) || (p.walls_z && (z == 1 || z == p.nz - 2));
}
bool is_wall(const lbmgpu_params& p, int y, int z) {
    return (p.walls_y && (y == 0 || y == p.ny - 1)) || (p.walls_z && (z == 0 || z == p.nz - 1));
}

void build_initial(const lbmgpu_params& p, HostInit& hi) {
    const size_t N = (size_t)p.nx * p.ny * p.nz;
    hi.flag.assign(N, T_FLUID);
    // WALL layers (lbm.cpp:72-78), near-wall bits and the static wall list:
    // a whole x-row shares its (y, z) classification.
    long long nf = 0;
    for (int z = 0; z < p.nz; ++z)
        for (int y = 0; y < p.ny; ++y) {
            const uint8_t v = is_wall(p, y, z) ? T_WALL : (near_wall(p, y, z) ? (uint8_t)(T_FLUID | NEAR_WALL) : T_FLUID);
            std::memset(hi.flag.data() + hidx(p, 0, y, z), v, p.nx);
            if (v != T_WALL) nf += p.nx;
            if (v == (T_FLUID | NEAR_WALL)) { hi.wallrows.push_back(y); hi.wallrows.push_back(z); }
        }
    SqState& s = hi.s;
    std::memset(&s, 0, sizeof(s));
    s.present = p.squirmer;
    s.mass_every = p.mass_correction_every;
    s.traj_every = p.traj_every;
    const double nu = (p.tau - 0.5) / 3.0;
    if (p.squirmer) {
        // Squirmer::init (squirmer.cpp:20-30)
        s.R = p.radius; s.B1 = p.b1; s.beta = p.beta; s.planar = p.planar;
        s.M = p.rho_p * 4.0 / 3.0 * PI * s.R * s.R * s.R;
        s.I = 0.4 * s.M * s.R * s.R;
        s.X[0] = p.x0 >= 0 ? p.x0 : 0.5 * (p.nx - 1);
        s.X[1] = p.y0 >= 0 ? p.y0 : 0.5 * (p.ny - 1);
        s.X[2] = p.z0 >= 0 ? p.z0 : 0.5 * (p.nz - 1);
        if (p.use_orientation) {
            const double n = std::sqrt(p.ex * p.ex + p.ey * p.ey + p.ez * p.ez);
            s.e[0] = p.ex / n; s.e[1] = p.ey / n; s.e[2] = p.ez / n;
        } else {
            const double a = p.angle * PI / 180.0;
            s.e[0] = std::cos(a); s.e[1] = std::sin(a); s.e[2] = 0.0;
        }
        s.eps = p.eps; s.hc = p.hc; s.hmin = p.hmin;
        s.FS = 6.0 * PI * nu * s.R * (2.0 * s.B1 / 3.0);
        // updateParticleFlags(true) (lbm.cpp:271-291)
        int lo[3], w[3];
        h_box(p, s, lo, w);
        for (int zz = lo[2]; zz < lo[2] + w[2]; ++zz)
            for (int yy = lo[1]; yy < lo[1] + w[1]; ++yy)
                for (int xx = lo[0]; xx < lo[0] + w[0]; ++xx) {
                    const int x = ((xx % p.nx) + p.nx) % p.nx, y = ((yy % p.ny) + p.ny) % p.ny, z = ((zz % p.nz) + p.nz) % p.nz;
                    const size_t n = hidx(p, x, y, z);
                    if ((hi.flag[n] & TYPE_MASK) == T_WALL) continue;
                    double r[3];
                    h_offset(p, s, x, y, z, r);
                    const bool inside = r[0] * r[0] + r[1] * r[1] + r[2] * r[2] < s.R * s.R;
                    if (inside && (hi.flag[n] & TYPE_MASK) != T_PARTICLE) { hi.flag[n] = T_PARTICLE; --nf; }
                }
        // near-particle bits and the boundary-link list (ascending node order):
        // fluid nodes with a PARTICLE neighbour lie within the box
        std::vector<int> cand;
        for (int zz = lo[2] - 1; zz <= lo[2] + w[2]; ++zz)
            for (int yy = lo[1] - 1; yy <= lo[1] + w[1]; ++yy)
                for (int xx = lo[0] - 1; xx <= lo[0] + w[0]; ++xx) {
                    const int x = ((xx % p.nx) + p.nx) % p.nx, y = ((yy % p.ny) + p.ny) % p.ny, z = ((zz % p.nz) + p.nz) % p.nz;
                    const size_t n = hidx(p, x, y, z);
                    if ((hi.flag[n] & TYPE_MASK) != T_FLUID) continue;
                    bool np = false;
                    for (int i = 1; i < Q && !np; ++i) {
                        const int xn = (x + CX(i) + p.nx) % p.nx, yn = (y + CY(i) + p.ny) % p.ny, zn = (z + CZ(i) + p.nz) % p.nz;
                        np = (hi.flag[hidx(p, xn, yn, zn)] & TYPE_MASK) == T_PARTICLE;
                    }
                    if (np) cand.push_back((int)n);
                }
        std::sort(cand.begin(), cand.end());
        cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
        for (int n : cand) { hi.flag[n] |= NEAR_PARTICLE; hi.links.push_back(n); }
        set_zones(p, s);
    }
    s.n_fluid = nf;
    s.n_links = (int)hi.links.size();
}

int validate_impl(const lbmgpu_params* p, std::string& m) {
    auto bad = [&](const char* s) { m = s; return LBMGPU_ERR_INVALID; };
    if (!p) return bad("null parameters");
    // Params::validate (params.cpp:120-140)
    if (p->nx < 1 || p->ny < 1 || p->nz < 1) return bad("grid dimensions must be positive");
    if (p->walls_y && p->ny < 4) return bad("ny must be >= 4 with walls in y");
    if (p->walls_z && p->nz < 4) return bad("nz must be >= 4 with walls in z");
    if (p->tau <= 0.5) return bad("tau must be > 0.5");
    if (p->lambda <= 0.0) return bad("lambda must be > 0");
    if (p->traj_every < 1) return bad("print_every and traj_every must be >= 1");
    // additions
    if ((double)p->nx * p->ny * p->nz >= 2147483648.0) return bad("lattice too large: nx*ny*nz must be < 2^31");
    if (p->ny > 65535 || p->nz > 65535) return bad("ny and nz must be <= 65535");
    if (p->precision < LBMGPU_FP64 || p->precision > LBMGPU_FP16) return bad("precision must be FP64, FP32 or FP16");
    if (p->mass_correction_every < 0) return bad("mass_correction_every must be >= 0");
    if (p->use_orientation && std::sqrt(p->ex * p->ex + p->ey * p->ey + p->ez * p->ez) == 0.0)
        return bad("orientation (ex, ey, ez) must be non-zero");
    if (!p->squirmer) return LBMGPU_OK;
    if (p->radius <= 1.0) return bad("squirmer radius must be > 1 lattice unit");
    if (std::fabs(p->angle) >= 45.0) return bad("initial angle must satisfy |angle| < 45 deg from the x-axis");
    if (p->rho_p <= 0.0) return bad("rho_p must be > 0");
    if (p->eps < 0.0 || p->hc <= 0.0 || p->hmin < 0.0) return bad("eps >= 0, hc > 0, hmin >= 0 required");
    const double y = p->y0 >= 0 ? p->y0 : 0.5 * (p->ny - 1);
    if (p->walls_y && (y - p->radius - 0.5 < p->hmin || (p->ny - 1.5) - y - p->radius < p->hmin))
        return bad("squirmer initially overlaps (or is too close to) a y-wall");
    if (2.0 * p->radius + 2.0 > p->nx || (!p->walls_y && 2.0 * p->radius + 2.0 > p->ny) || 2.0 * p->radius + 2.0 > p->nz)
        return bad("domain too small for the squirmer");
    if (2.0 * p->b1 / 3.0 > 0.05) return bad("swimming speed U0 = 2 B1 / 3 too large (Mach number); keep U0 < 0.05");
    if (p->radius > 200.0) return bad("squirmer radius must be <= 200 lattice units");
    return LBMGPU_OK;
}

void drop_graph(lbmgpu_handle* h) {
    for (Graph& g : h->g) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.graph) cudaGraphDestroy(g.graph);
        g = Graph{};
    }
}

void free_all(lbmgpu_handle* h) {
    drop_graph(h);
    if (h->member) { h->f = nullptr; h->flag = nullptr; }
    void* ptrs[] = {h->f, h->flag, h->rho, h->ux, h->uy, h->uz, h->wallrows, h->links, h->linkslot,
                    h->link_part, h->block_part, h->block_part_b, h->row_claim, h->ordermap, h->chg_node, h->chg_key,
                    h->cand, h->mark, h->traj, h->sq, h->scratch, h->small, h->shell, h->shell_hdr,
                    h->packed, h->snap};
    for (void* q : ptrs) if (q) cudaFree(q);
    for (cudaEvent_t e : {h->ev_b[0], h->ev_b[1], h->ev_z, h->ev_s, h->ev_fork, h->ev_join, h->snap_ready})
        if (e) cudaEventDestroy(e);
    for (cudaStream_t s : {h->own, h->zs, h->cap, h->cap2, h->snap_stream})
        if (s) cudaStreamDestroy(s);
}

StepPlan plan_step(lbmgpu_handle* h, long long s, bool macro, bool apply) {
    StepPlan sp;
    sp.s = s;
    sp.par = (int)((s - 1) & 1);
    sp.zslot = (int)(s % ZONE_SLOTS);
    sp.corr = is_corr_step(h, s);
    sp.apply = apply;
    sp.macro = macro;
    return sp;
}

// One time step of the time loop, B on stream a, Z and S on stream b (see the
// dependency list at the top of this file). When called for step s, ev_b[s&1]
// marks B(s-1)... precisely: ev_b[(s-1)&1] marks B(s-1), ev_z marks Z(s-1) and
// ev_s marks S(s-1).
void issue_fused(lbmgpu_handle* h, cudaStream_t sa, cudaStream_t sb, const StepPlan& sp) {
    const StreamArgs a = stream_args(h, sp);
    const int par = sp.par;
    cudaStreamWaitEvent(sa, h->ev_z, 0);
    if (sp.apply) cudaStreamWaitEvent(sa, h->ev_s, 0);
    h->lz->bulk(par, h->has_sq != 0, sp.macro, h->L, a, h->geom, sa);
    int k = 1;
    if (h->geom.nwallrows && h->wallrows_on_a) { h->lz->wallrows(par, h->has_sq != 0, sp.macro, h->L, a, h->geom, sa); ++k; }
    cudaEventRecord(h->ev_b[sp.s & 1], sa);
    cudaStreamWaitEvent(sb, h->ev_b[(sp.s - 1) & 1], 0);
    if (h->geom.nwallrows && !h->wallrows_on_a) { h->lz->wallrows(par, h->has_sq != 0, sp.macro, h->L, a, h->geom, sb); ++k; }
    if (h->geom.bgrid) { h->lz->zone(par, h->has_sq != 0, sp.macro, h->L, a, h->geom, sb); ++k; }
    cudaEventRecord(h->ev_z, sb);
    if (sp.macro) {
        cudaStreamWaitEvent(sb, h->ev_b[sp.s & 1], 0);
        k_finalize<<<1, 256, 0, sb>>>(h->block_part, h->nblocks, h->block_part_b, h->geom.bgrid ? h->nblocks_b : 0, h->sq);
        ++k;
    }
    if (h->has_sq) {
        if (sp.corr) cudaStreamWaitEvent(sb, h->ev_b[sp.s & 1], 0);
        const int za = (int)((sp.s + 2) % ZONE_SLOTS);
        h->lz->squirmer(h->L, squirmer_args(h, par ^ 1, STAGE_FORCE | STAGE_BODY | STAGE_REMAP | STAGE_LOOP,
                                            sp.corr ? 1 : 0, za, -1), sb);
        cudaEventRecord(h->ev_s, sb);
        ++k;
    }
    h->launches += k;
}

// Make the events describe "everything issued so far on stream sa" before a
// sequence of fused steps on (sa, sb), and join sb back into sa after it.
void fused_begin(lbmgpu_handle* h, cudaStream_t sa, cudaStream_t sb) {
    cudaEventRecord(h->ev_fork, sa);
    cudaStreamWaitEvent(sb, h->ev_fork, 0);
    for (cudaEvent_t e : {h->ev_b[0], h->ev_b[1], h->ev_z, h->ev_s}) cudaEventRecord(e, sa);
}
void fused_end(lbmgpu_handle* h, cudaStream_t sa, cudaStream_t sb) {
    cudaEventRecord(h->ev_join, sb);
    cudaStreamWaitEvent(sa, h->ev_join, 0);
}

// The captured pattern of `steps` steps. It starts at a step s with
// (s - 1) % period == 0; apply0 says whether its first step applies a
// correction computed by the step before (the usual case once the run is
// under way: the period is a multiple of the correction interval, so the
// step before a pattern is a correction step). Without corrections in the
// pattern, the graph is only launched over stretches that contain no
// correction step.
int ensure_graph(lbmgpu_handle* h, int steps, bool apply0) {
    Graph& g = h->g[apply0 ? 1 : 0];
    if (g.exec && g.steps == steps) return LBMGPU_OK;
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
    g = Graph{};
    CUDA_TRY(h, cudaStreamBeginCapture(h->cap, cudaStreamCaptureModeThreadLocal));
    const long long saved = h->launches;
    fused_begin(h, h->cap, h->cap2);
    for (int k = 0; k < steps; ++k) {
        const long long s = 1 + k;
        const bool apply = k == 0 ? apply0 : h->corr_in_graph && is_corr_step(h, s - 1);
        StepPlan sp = plan_step(h, s, false, apply);
        if (!h->corr_in_graph) sp.corr = false;
        issue_fused(h, h->cap, h->cap2, sp);
    }
    fused_end(h, h->cap, h->cap2);
    h->launches = saved;
    CUDA_TRY(h, cudaStreamEndCapture(h->cap, &g.graph));
    CUDA_TRY(h, cudaGraphInstantiate(&g.exec, g.graph, 0));
    g.steps = steps;
    return LBMGPU_OK;
}

// Packed fields (k_pack_fields): rho, u interleaved, node types.
struct PackedView {
    double* rho;
    double* u;
    uint8_t* flag;
};
PackedView packed_view(const lbmgpu_handle* h, unsigned char* base) {
    const size_t N = h->L.N;
    return PackedView{reinterpret_cast<double*>(base), reinterpret_cast<double*>(base) + N,
                      reinterpret_cast<uint8_t*>(base + 4 * N * sizeof(double))};
}
cudaError_t ensure_packed(lbmgpu_handle* h, unsigned char** buf) {
    if (*buf) return cudaSuccess;
    return cudaMalloc(reinterpret_cast<void**>(buf), (size_t)h->L.N * (4 * sizeof(double) + 1));
}
void pack_fields(lbmgpu_handle* h, unsigned char* buf, cudaStream_t st) {
    const PackedView v = packed_view(h, buf);
    k_pack_fields<<<1184, 256, 0, st>>>(h->L.N, h->flag, h->rho, h->ux, h->uy, h->uz, v.rho, v.u, v.flag);
    ++h->launches;
}

int check_status(lbmgpu_handle* h) {
    CUDA_TRY(h, cudaGetLastError());
    int st = 0;
    CUDA_TRY(h, cudaMemcpyAsync(&st, &h->sq->status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    if (st & ST_NAN) return fail(h, LBMGPU_ERR_NAN, "non-finite squirmer force, torque or state");
    if (st & ST_REMAP_RANGE)
        return fail(h, LBMGPU_ERR_DEVICE, "squirmer moved one lattice cell or more in a single step");
    if (st & ST_LINK_OVERFLOW) return fail(h, LBMGPU_ERR_DEVICE, "boundary-link list capacity exceeded");
    if (st & ST_REMAP_OVERFLOW) return fail(h, LBMGPU_ERR_DEVICE, "remap changed-node list capacity exceeded");
    if (st & ST_WATCHDOG) return fail(h, LBMGPU_ERR_WATCHDOG, "a bounded device wait gave up");
    return LBMGPU_OK;
}

}  // namespace

// ============================================================================
//  C ABI
// ============================================================================
extern "C" {

int lbmgpu_abi_version(void) { return LBMGPU_ABI_VERSION; }

void lbmgpu_params_default(lbmgpu_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    // lbm::Params defaults (params.hpp:16-56)
    p->nx = 64; p->ny = 34; p->nz = 32;
    p->tau = 1.0; p->lambda = 3.0 / 16.0; p->fx = p->fy = p->fz = 0.0;
    p->walls_y = 1; p->walls_z = 0;
    p->traj_every = 50; p->mass_correction_every = 10;
    p->squirmer = 0;
    p->radius = 4.0; p->b1 = 0.015; p->beta = 0.0; p->rho_p = 1.0;
    p->x0 = p->y0 = p->z0 = -1.0; p->angle = 30.0; p->planar = 1;
    p->eps = 0.2; p->hc = 2.0; p->hmin = 0.5;
    p->use_orientation = 0; p->ex = 0.0; p->ey = 0.0; p->ez = 0.0;
    p->precision = LBMGPU_FP64; p->device = 0;
}

int lbmgpu_validate(const lbmgpu_params* p, char* msg, size_t msg_len) {
    std::string m;
    const int rc = validate_impl(p, m);
    if (msg && msg_len) std::snprintf(msg, msg_len, "%s", m.c_str());
    return rc;
}

}  // extern "C"

namespace {
// Ensemble members: no streams of their own, populations and flags carved
// from the ensemble's pools.
struct MemberOpts {
    cudaStream_t stream;
    void* f;
    uint8_t* flag;
};

int create_impl(const lbmgpu_params* p, const MemberOpts* mo, lbmgpu_handle** out) {
    if (!out) return fail(nullptr, LBMGPU_ERR_INVALID, "null output pointer");
    *out = nullptr;
    std::string m;
    if (validate_impl(p, m) != LBMGPU_OK) return fail(nullptr, LBMGPU_ERR_INVALID, m);
    lbmgpu_handle* h = new lbmgpu_handle();
    h->p = *p;
    h->member = mo != nullptr;
    h->lz = launchers_for(p->precision);
    h->esize = esize_for(p->precision);
    h->has_sq = p->squirmer;
    auto bail = [&](int rc) {
        g_create_error = h->err;
        free_all(h);
        delete h;
        return rc;
    };
#define CTRY(call)                                                                                  \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) {                                                                    \
            h->err = std::string(#call) + ": " + cudaGetErrorString(e_);                            \
            return bail(e_ == cudaErrorMemoryAllocation ? LBMGPU_ERR_NOMEM : LBMGPU_ERR_CUDA);      \
        }                                                                                           \
    } while (0)
    CTRY(cudaSetDevice(p->device));
    CTRY(h->lz->prepare());
    if (mo) {
        h->stream = mo->stream;
    } else {
        int prio_lo = 0, prio_hi = 0;
        CTRY(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
        CTRY(cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking));
        CTRY(cudaStreamCreateWithPriority(&h->zs, cudaStreamNonBlocking, prio_hi));
        CTRY(cudaStreamCreateWithFlags(&h->cap, cudaStreamNonBlocking));
        CTRY(cudaStreamCreateWithPriority(&h->cap2, cudaStreamNonBlocking, prio_hi));
        for (cudaEvent_t* e : {&h->ev_b[0], &h->ev_b[1], &h->ev_z, &h->ev_s, &h->ev_fork, &h->ev_join})
            CTRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
        h->stream = h->own;
    }

    Lattice& L = h->L;
    L.nx = p->nx; L.ny = p->ny; L.nz = p->nz;
    L.N = (unsigned)((size_t)p->nx * p->ny * p->nz);
    L.nxy = (unsigned)((size_t)p->nx * p->ny);
    L.walls_y = p->walls_y; L.walls_z = p->walls_z;
    // TRT rates (lbm.cpp:65-69) and Guo factors (lbm.cpp:129)
    L.omP = 1.0 / p->tau;
    L.omM = 1.0 / (0.5 + p->lambda / (p->tau - 0.5));
    L.gP = 1.0 - 0.5 * L.omP;
    L.gM = 1.0 - 0.5 * L.omM;
    L.F[0] = p->fx; L.F[1] = p->fy; L.F[2] = p->fz;
    L.omPf = (float)L.omP; L.omMf = (float)L.omM; L.gPf = (float)L.gP; L.gMf = (float)L.gM;
    for (int c = 0; c < 3; ++c) L.gPw[c] = (float)(L.gP * (c == 0 ? WD(0) : (c == 1 ? WD(1) : WD(7))));
    for (int d = 0; d < 3; ++d) { L.Ff[d] = (float)L.F[d]; L.uFh[d] = 0.0f; }
    L.force_free = L.F[0] == 0.0 && L.F[1] == 0.0 && L.F[2] == 0.0;
    L.one = 1.0f;
    L.mzero = -0.0f;
    for (int i = 0; i < Q; ++i) {
        const double cF = CX(i) * L.F[0] + CY(i) * L.F[1] + CZ(i) * L.F[2];
        L.cF[i] = (float)cF;
        L.cm[i] = (float)(L.gM * 3.0 * WD(i) * cF);
    }
    const size_t N = L.N;

    HostInit hi;
    build_initial(*p, hi);
    h->geom.nwallrows = (unsigned)(hi.wallrows.size() / 2);
    // Wall rows and zone nodes are disjoint and the wall rows need only what
    // the bulk of the same step needs, so they may go on either stream. On
    // stream b they overlap the bulk but lengthen the chain wall rows -> zone ->
    // squirmer; when the bulk moves less than ~200 MB (about 40 us) that chain
    // is the step, and they go after the bulk on stream a instead.
    h->wallrows_on_a = h->has_sq && (double)Q * 2.0 * h->esize * (double)N <= 200e6;
    // FP64: a long bulk runs denser (3 CTAs/SM); a short one keeps 2, which
    // leaves room on the SMs for the zone and squirmer chain beside it
    h->geom.dense = (double)Q * 2.0 * h->esize * (double)N > 200e6;
    // nx not a multiple of 32: on steps without sums the bulk runs over each
    // plane's rows away from walls as one range of nodes (no idle lanes)
    {
        const int rows = p->walls_y ? p->ny - 4 : p->ny, planes = p->walls_z ? p->nz - 4 : p->nz;
        const long long range = (long long)rows * p->nx;
        h->geom.flat = dim3(0, 0, 0);
        if (p->nx % 32 != 0 && rows > 0 && planes > 0)
            h->geom.flat = dim3((unsigned)((range + 255) / 256), (unsigned)planes, 1);
        // shifted forms, nx a multiple of 64: on steps without sums the bulk
        // updates two x-adjacent nodes per thread (k_bulk_pair); the block is
        // the largest multiple of 32 up to 128 threads that divides nx / 2
        h->geom.pair = dim3(0, 0, 0);
        if (p->precision != LBMGPU_FP64 && p->nx % 64 == 0 && bulk_kind() == 1) {
            const int pairs = p->nx / 2;
            int tb = 32;
            for (int b = 128; b >= 32; b -= 32)
                if (pairs % b == 0) { tb = b; break; }
            h->geom.pair_block = dim3((unsigned)tb, 1, 1);
            h->geom.pair = dim3((unsigned)(pairs / tb), (unsigned)p->ny, (unsigned)p->nz);
        }
        // nx a multiple of 32 up to 256: rows staged in shared memory
        // (k_bulk_rows), a persistent grid of the CTAs that fit on the SMs
        h->geom.rows_grid = 0;
        if (p->nx % 32 == 0 && p->nx <= ROWS_MAX_NX && rows > 0 && planes > 0 && bulk_kind() >= 2) {
            int sms = 0, dev = p->device;
            h->geom.rows_pairs = p->precision == LBMGPU_FP16 && p->nx % 64 == 0 && bulk_kind() == 2;
            const int per_sm = h->lz->rows_ctas_per_sm(p->nx, h->geom.rows_pairs);
            if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && per_sm > 0) {
                h->geom.rows_nry = rows;
                h->geom.rows_n = rows * planes;
                h->geom.rows_ylo = p->walls_y ? 2 : 0;
                h->geom.rows_zlo = p->walls_z ? 2 : 0;
                h->geom.rows_grid = (unsigned)std::min<long long>((long long)sms * per_sm, (long long)rows * planes);
                h->geom.rows_reserve = rows_reserve(h->has_sq != 0, sms);
            }
        }
    }
    h->link_cap = link_capacity(*p);
    h->chg_cap = h->link_cap;
    if ((long long)hi.links.size() >= h->link_cap) {
        h->err = "boundary-link list of the initial state exceeds its capacity";
        return bail(LBMGPU_ERR_DEVICE);
    }
    {
        const int tx = p->nx >= 256 ? 256 : ((p->nx + 31) / 32) * 32;
        h->geom.block = dim3(tx, 1, 1);
        h->geom.grid = dim3((p->nx + tx - 1) / tx, p->ny, p->nz);
        h->nblocks = h->geom.grid.x * h->geom.grid.y * h->geom.grid.z;
        if (h->has_sq) {
            h->zw[0] = zone_width(p->radius, p->nx, false);
            h->zw[1] = zone_width(p->radius, p->ny, p->walls_y != 0);
            h->zw[2] = zone_width(p->radius, p->nz, p->walls_z != 0);
            h->zone_cells = h->zw[0] * h->zw[1] * h->zw[2];
        }
        const long long nb = (long long)h->zone_cells;
        h->geom.bgrid = (unsigned)((nb + BOUNDARY_BLOCK - 1) / BOUNDARY_BLOCK);
        h->nblocks_b = std::max(1u, h->geom.bgrid);
        // period of the launch pattern: AA parity (2), zone slots (3), mass correction (k)
        const int k = p->mass_correction_every;
        const int base = std::lcm(2, ZONE_SLOTS);
        h->corr_in_graph = h->has_sq && k > 0 && std::lcm(base, k) <= MAX_PERIOD;
        h->period = h->corr_in_graph ? std::lcm(base, k) : base;
    }

    if (mo) {
        h->f = mo->f;
        h->flag = mo->flag;
    } else {
        CTRY(cudaMalloc(&h->f, (size_t)Q * N * h->esize));
        CTRY(cudaMalloc(&h->flag, N));
    }
    CTRY(cudaMalloc(&h->rho, N * sizeof(double)));
    CTRY(cudaMalloc(&h->ux, N * sizeof(double)));
    CTRY(cudaMalloc(&h->uy, N * sizeof(double)));
    CTRY(cudaMalloc(&h->uz, N * sizeof(double)));
    CTRY(cudaMalloc(&h->scratch, N * sizeof(double)));
    CTRY(cudaMalloc(&h->block_part, (size_t)h->nblocks * BLOCK_PART * sizeof(double)));
    CTRY(cudaMalloc(&h->block_part_b, (size_t)h->nblocks_b * BLOCK_PART * sizeof(double)));
    CTRY(cudaMalloc(&h->row_claim, 2 * sizeof(int)));
    CTRY(cudaMalloc(&h->wallrows, std::max<size_t>(2, hi.wallrows.size()) * sizeof(int)));
    CTRY(cudaMalloc(&h->sq, sizeof(SqState)));
    CTRY(cudaMalloc(&h->small, (2 * MASS_GRID + 4 * DIAG_GRID + 16) * sizeof(double)));
    CTRY(cudaMalloc(&h->links, (size_t)h->link_cap * sizeof(int)));
    CTRY(cudaMalloc(&h->link_part, (size_t)h->link_cap * LINK_PART * sizeof(double)));
    if (h->has_sq) {
        CTRY(cudaMalloc(&h->linkslot, N * sizeof(int)));
        CTRY(cudaMalloc(&h->ordermap, N * sizeof(int)));
        CTRY(cudaMalloc(&h->chg_node, (size_t)h->chg_cap * sizeof(int)));
        CTRY(cudaMalloc(&h->chg_key, (size_t)h->chg_cap * sizeof(int)));
        CTRY(cudaMalloc(&h->mark, (size_t)h->chg_cap));
        CTRY(cudaMalloc(&h->cand, (size_t)h->chg_cap * sizeof(int)));
        CTRY(cudaMalloc(&h->shell, (size_t)h->chg_cap * sizeof(int)));
        CTRY(cudaMalloc(&h->shell_hdr, sizeof(ShellCache)));
        CTRY(cudaMalloc(&h->traj, (size_t)TRAJ_RING * TRAJ_COLS * sizeof(double)));
    }
    cudaStream_t st = h->stream;
    h->lz->fill_rest(L, h->f, st);
    k_fill_d<<<592, 256, 0, st>>>(h->rho, N, 1.0);
    k_fill_d<<<592, 256, 0, st>>>(h->ux, N, 0.0);
    k_fill_d<<<592, 256, 0, st>>>(h->uy, N, 0.0);
    k_fill_d<<<592, 256, 0, st>>>(h->uz, N, 0.0);
    h->launches += 5;
    CTRY(cudaMemsetAsync(h->block_part, 0, (size_t)h->nblocks * BLOCK_PART * sizeof(double), st));
    CTRY(cudaMemsetAsync(h->block_part_b, 0, (size_t)h->nblocks_b * BLOCK_PART * sizeof(double), st));
    CTRY(cudaMemsetAsync(h->row_claim, 0, 2 * sizeof(int), st));
    if (!hi.wallrows.empty())
        CTRY(cudaMemcpyAsync(h->wallrows, hi.wallrows.data(), hi.wallrows.size() * sizeof(int),
                             cudaMemcpyHostToDevice, st));
    CTRY(cudaMemsetAsync(h->link_part, 0, (size_t)h->link_cap * LINK_PART * sizeof(double), st));
    CTRY(cudaMemcpyAsync(h->flag, hi.flag.data(), N, cudaMemcpyHostToDevice, st));
    if (h->has_sq) {
        k_fill_i<<<592, 256, 0, st>>>(h->ordermap, N, -1);
        CTRY(cudaMemsetAsync(h->shell_hdr, 0, sizeof(ShellCache), st));   // no shell yet
        CTRY(cudaMemsetAsync(h->linkslot, 0, N * sizeof(int), st));
        if (!hi.links.empty()) {
            CTRY(cudaMemcpyAsync(h->links, hi.links.data(), hi.links.size() * sizeof(int), cudaMemcpyHostToDevice, st));
            k_scatter_slots<<<64, 256, 0, st>>>(h->links, (int)hi.links.size(), h->linkslot);
        }
        h->launches += 2;
        CTRY(cudaMemsetAsync(h->traj, 0, (size_t)TRAJ_RING * TRAJ_COLS * sizeof(double), st));
    }
    CTRY(cudaMemcpyAsync(h->sq, &hi.s, sizeof(SqState), cudaMemcpyHostToDevice, st));
    CTRY(cudaStreamSynchronize(st));  // host vectors go out of scope
    CTRY(cudaGetLastError());
#undef CTRY
    *out = h;
    return LBMGPU_OK;
}
}  // namespace

extern "C" {

int lbmgpu_create(const lbmgpu_params* p, lbmgpu_handle** out) { return create_impl(p, nullptr, out); }

int lbmgpu_destroy(lbmgpu_handle* h) {
    if (!h) return LBMGPU_OK;
    if (h->member) return fail(h, LBMGPU_ERR_INVALID, "handle belongs to an ensemble: destroy the ensemble");
    cudaSetDevice(h->p.device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->zs) cudaStreamSynchronize(h->zs);
    free_all(h);
    delete h;
    return LBMGPU_OK;
}

int lbmgpu_run(lbmgpu_handle* h, int nsteps) {
    if (!h) return LBMGPU_ERR_INVALID;
    if (h->member) return fail(h, LBMGPU_ERR_INVALID, "handle belongs to an ensemble: advance it with lbmgpu_batch_run");
    if (nsteps < 0) return fail(h, LBMGPU_ERR_INVALID, "nsteps must be >= 0");
    if (nsteps == 0) return LBMGPU_OK;
    CUDA_TRY(h, cudaSetDevice(h->p.device));
    cudaStream_t sa = h->stream, sb = h->zs;
    const int per_step = 1 + (h->geom.nwallrows ? 1 : 0) + (h->geom.bgrid ? 1 : 0) + (h->has_sq ? 1 : 0);
    const int gsteps = h->period * ((MIN_GRAPH + h->period - 1) / h->period);
    fused_begin(h, sa, sb);
    long long rem = nsteps;
    while (rem > 0) {
        const long long s = h->t_main + 1;
        const bool last = rem == 1;
        // A captured graph starts at a pattern boundary, ends before the last
        // step (which stores the macroscopic fields), and contains correction
        // steps only if the pattern period includes them.
        bool graph_ok = !last && h->t_main % h->period == 0 && rem - 1 >= gsteps;
        if (graph_ok && h->has_sq && h->p.mass_correction_every > 0 && !h->corr_in_graph) {
            const int k = h->p.mass_correction_every;
            graph_ok = (h->t_main / k) == ((h->t_main + gsteps) / k);  // no correction step inside
        }
        if (graph_ok) {
            // the graph carries its own fork and join on the caller's stream
            fused_end(h, sa, sb);
            int rc = ensure_graph(h, gsteps, h->pending_corr);
            if (rc) return rc;
            CUDA_TRY(h, cudaGraphLaunch(h->g[h->pending_corr ? 1 : 0].exec, sa));
            h->launches += (long long)gsteps * per_step;
            h->t_main += gsteps;
            rem -= gsteps;
            h->pending_corr = is_corr_step(h, h->t_main);
            fused_begin(h, sa, sb);
            continue;
        }
        issue_fused(h, sa, sb, plan_step(h, s, last, h->pending_corr));
        h->t_main = s;
        h->pending_corr = is_corr_step(h, s);
        --rem;
    }
    fused_end(h, sa, sb);
    return check_status(h);
}

// LBM::step alone: both collide-stream kernels, then the sphere force of the
// step (lbm.cpp:219-223), all on the caller's stream.
int lbmgpu_step(lbmgpu_handle* h) {
    if (!h) return LBMGPU_ERR_INVALID;
    if (h->member) return fail(h, LBMGPU_ERR_INVALID, "handle belongs to an ensemble: advance it with lbmgpu_batch_run");
    CUDA_TRY(h, cudaSetDevice(h->p.device));
    StepPlan sp = plan_step(h, h->t_main + 1, true, h->pending_corr);
    sp.corr = false;
    const StreamArgs a = stream_args(h, sp);
    cudaStream_t st = h->stream;
    h->lz->bulk(sp.par, h->has_sq != 0, true, h->L, a, h->geom, st);
    if (h->geom.nwallrows) { h->lz->wallrows(sp.par, h->has_sq != 0, true, h->L, a, h->geom, st); ++h->launches; }
    if (h->geom.bgrid) { h->lz->zone(sp.par, h->has_sq != 0, true, h->L, a, h->geom, st); ++h->launches; }
    k_finalize<<<1, 256, 0, st>>>(h->block_part, h->nblocks, h->block_part_b, h->geom.bgrid ? h->nblocks_b : 0, h->sq);
    h->launches += 2;
    if (h->has_sq) {
        h->lz->squirmer(h->L, squirmer_args(h, sp.par ^ 1, STAGE_FORCE, 0, -1, -1), st);
        k_clear_pending<<<1, 32, 0, st>>>(h->sq);
        h->launches += 2;
    }
    h->pending_corr = false;
    ++h->t_main;
    return check_status(h);
}

int lbmgpu_advance_squirmer(lbmgpu_handle* h) {
    if (!h) return LBMGPU_ERR_INVALID;
    if (h->member) return fail(h, LBMGPU_ERR_INVALID, "handle belongs to an ensemble: advance it with lbmgpu_batch_run");
    if (!h->has_sq) return LBMGPU_OK;  // LBM::advanceSquirmer returns without a squirmer (lbm.cpp:258)
    CUDA_TRY(h, cudaSetDevice(h->p.device));
    const long long s = h->t_main;  // the step just done
    h->lz->squirmer(h->L, squirmer_args(h, (int)(h->t_main & 1), STAGE_BODY | STAGE_REMAP, 0,
                                        (int)((s + 1) % ZONE_SLOTS), (int)((s + 2) % ZONE_SLOTS)), h->stream);
    ++h->launches;
    return check_status(h);
}

int lbmgpu_correct_mass(lbmgpu_handle* h) {
    if (!h) return LBMGPU_ERR_INVALID;
    if (h->member) return fail(h, LBMGPU_ERR_INVALID, "handle belongs to an ensemble: advance it with lbmgpu_batch_run");
    CUDA_TRY(h, cudaSetDevice(h->p.device));
    // a correction still pending from lbmgpu_run is folded in and applied now
    double* part = h->small;
    double* dflag = h->small + 2 * MASS_GRID;
    h->lz->correct_mass(h->L, h->f, h->flag, (int)(h->t_main & 1), h->sq, part, dflag, h->stream);
    h->launches += 3;
    h->pending_corr = false;
    return check_status(h);
}

int lbmgpu_time(const lbmgpu_handle* h, long long* t) {
    if (!h || !t) return LBMGPU_ERR_INVALID;
    *t = h->t_main;
    return LBMGPU_OK;
}

int lbmgpu_squirmer_state(lbmgpu_handle* h, lbmgpu_squirmer* o) {
    if (!h || !o) return LBMGPU_ERR_INVALID;
    CUDA_TRY(h, cudaSetDevice(h->p.device));
    SqState s;
    CUDA_TRY(h, cudaMemcpyAsync(&s, h->sq, sizeof(s), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    for (int d = 0; d < 3; ++d) {
        o->X[d] = s.X[d]; o->e[d] = s.e[d]; o->U[d] = s.U[d]; o->W[d] = s.W[d];
        o->Fh[d] = s.Fh[d]; o->Th[d] = s.Th[d]; o->Fc[d] = s.Fc[d]; o->Tc[d] = s.Tc[d]; o->Fw[d] = s.Fw[d];
    }
    o->R = s.R; o->B1 = s.B1; o->beta = s.beta; o->M = s.M; o->I = s.I; o->FS = s.FS;
    o->U0 = 2.0 * s.B1 / 3.0;
    o->contacts = s.contacts;
    return LBMGPU_OK;
}

int lbmgpu_set_squirmer_state(lbmgpu_handle* h, const double X[3], const double e[3], const double U[3],
                              const double W[3]) {
    if (!h || !X || !e || !U || !W) return LBMGPU_ERR_INVALID;
    if (h->member) return fail(h, LBMGPU_ERR_INVALID, "handle belongs to an ensemble: advance it with lbmgpu_batch_run");
    if (!h->has_sq) return fail(h, LBMGPU_ERR_INVALID, "no squirmer in this lattice");
    CUDA_TRY(h, cudaSetDevice(h->p.device));
    SqState s;
    CUDA_TRY(h, cudaMemcpyAsync(&s, h->sq, sizeof(s), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    for (int d = 0; d < 3; ++d) { s.X[d] = X[d]; s.e[d] = e[d]; s.U[d] = U[d]; s.W[d] = W[d]; }
    set_zones(h->p, s);
    CUDA_TRY(h, cudaMemcpyAsync(h->sq, &s, sizeof(s), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return LBMGPU_OK;
}

int lbmgpu_fields(lbmgpu_handle* h, uint8_t* flag, double* rho, double* u3) {
    if (!h) return LBMGPU_ERR_INVALID;
    CUDA_TRY(h, cudaSetDevice(h->p.device));
    const size_t N = h->L.N;
    cudaStream_t st = h->stream;
    CUDA_TRY(h, ensure_packed(h, &h->packed));
    pack_fields(h, h->packed, st);
    const PackedView v = packed_view(h, h->packed);
    if (rho) CUDA_TRY(h, cudaMemcpyAsync(rho, v.rho, N * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (u3) CUDA_TRY(h, cudaMemcpyAsync(u3, v.u, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (flag) CUDA_TRY(h, cudaMemcpyAsync(flag, v.flag, N, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(h, cudaStreamSynchronize(st));
    return LBMGPU_OK;
}

int lbmgpu_snapshot_begin(lbmgpu_handle* h) {
    if (!h) return LBMGPU_ERR_INVALID;
    if (h->snap_pending.load()) return fail(h, LBMGPU_ERR_INVALID, "the previous snapshot has not been read");
    CUDA_TRY(h, cudaSetDevice(h->p.device));
    CUDA_TRY(h, ensure_packed(h, &h->snap));
    if (!h->snap_stream) {
        CUDA_TRY(h, cudaStreamCreateWithFlags(&h->snap_stream, cudaStreamNonBlocking));
        CUDA_TRY(h, cudaEventCreateWithFlags(&h->snap_ready, cudaEventDisableTiming));
    }
    pack_fields(h, h->snap, h->stream);   // after everything issued on the handle's stream so far
    CUDA_TRY(h, cudaEventRecord(h->snap_ready, h->stream));
    CUDA_TRY(h, cudaGetLastError());
    h->snap_pending.store(true);
    return LBMGPU_OK;
}

int lbmgpu_snapshot_read(lbmgpu_handle* h, uint8_t* flag, double* rho, double* u3) {
    if (!h) return LBMGPU_ERR_INVALID;
    if (!h->snap_pending.load()) { h->snap_err = "no snapshot taken (lbmgpu_snapshot_begin)"; return LBMGPU_ERR_INVALID; }
    const size_t N = h->L.N;
    const PackedView v = packed_view(h, h->snap);
    cudaStream_t st = h->snap_stream;
    cudaError_t e = cudaSetDevice(h->p.device);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, h->snap_ready, 0);
    if (e == cudaSuccess && rho) e = cudaMemcpyAsync(rho, v.rho, N * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && u3) e = cudaMemcpyAsync(u3, v.u, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && flag) e = cudaMemcpyAsync(flag, v.flag, N, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    h->snap_pending.store(false);
    if (e != cudaSuccess) {
        h->snap_err = std::string("lbmgpu_snapshot_read: ") + cudaGetErrorString(e);
        return LBMGPU_ERR_CUDA;
    }
    return LBMGPU_OK;
}

const char* lbmgpu_snapshot_last_error(const lbmgpu_handle* h) { return h ? h->snap_err.c_str() : ""; }

void* lbmgpu_host_alloc(size_t bytes) {
    void* p = nullptr;
    if (bytes == 0 || cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) return nullptr;
    return p;
}

int lbmgpu_host_free(void* p) {
    if (p && cudaFreeHost(p) != cudaSuccess) return LBMGPU_ERR_CUDA;
    return LBMGPU_OK;
}

int lbmgpu_diag(lbmgpu_handle* h, lbmgpu_diagnostics* d) {
    if (!h || !d) return LBMGPU_ERR_INVALID;
    CUDA_TRY(h, cudaSetDevice(h->p.device));
    double* part = h->small + 2 * MASS_GRID + 8;
    double* res = part + 4 * DIAG_GRID;
    k_diag_partial<<<DIAG_GRID, 256, 0, h->stream>>>(h->L.N, h->flag, h->rho, h->ux, h->uy, h->uz, part);
    k_diag_final<<<1, 32, 0, h->stream>>>(part, DIAG_GRID, res);
    h->launches += 2;
    double r[4];
    SqState s;
    CUDA_TRY(h, cudaMemcpyAsync(r, res, sizeof(r), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(&s, h->sq, sizeof(s), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    d->n_fluid = (long long)r[0];
    d->mean_density = r[0] > 0 ? r[1] / r[0] : 0.0;
    d->max_speed = r[2];
    d->sum_ux = r[3];
    for (int k = 0; k < 3; ++k) d->wall_force[k] = s.wall_force[k];
    return LBMGPU_OK;
}

int lbmgpu_traj_rows(lbmgpu_handle* h, double* rows, int max_rows, int* nrows, long long* dropped) {
    if (!h || !nrows || (max_rows > 0 && !rows)) return LBMGPU_ERR_INVALID;
    *nrows = 0;
    if (dropped) *dropped = 0;
    if (!h->has_sq) return LBMGPU_OK;
    CUDA_TRY(h, cudaSetDevice(h->p.device));
    long long cnt = 0;
    CUDA_TRY(h, cudaMemcpyAsync(&cnt, &h->sq->traj_count, sizeof(cnt), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    long long first = h->traj_read;
    if (cnt - first > TRAJ_RING) {
        if (dropped) *dropped = cnt - first - TRAJ_RING;
        first = cnt - TRAJ_RING;
    }
    const long long avail = cnt - first;
    const int take = (int)std::min<long long>(avail, max_rows);
    if (take > 0) {
        std::vector<double> ring((size_t)TRAJ_RING * TRAJ_COLS);
        CUDA_TRY(h, cudaMemcpyAsync(ring.data(), h->traj, ring.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
        for (int k = 0; k < take; ++k) {
            const long long idx = (first + k) % TRAJ_RING;
            std::memcpy(rows + (size_t)k * TRAJ_COLS, ring.data() + idx * TRAJ_COLS, TRAJ_COLS * sizeof(double));
        }
    }
    h->traj_read = first + take;
    *nrows = take;
    return LBMGPU_OK;
}

// ---- checkpoint / restart --------------------------------------------------
// A checkpoint is the complete device state of a lattice as stored: the
// populations in their storage form and AA parity, flags, the moments of the
// last step, the squirmer state (with its zones, pending mass correction and
// trajectory counters), the boundary-link list and the trajectory ring. A
// lattice created with the same parameters and loaded from it continues bit
// for bit as the saved one would have.
//
// The header records every parameter the stored state depends on (sizes,
// storage form, walls, the TRT and forcing constants, the squirmer model and
// the cadences). Loading checks them against the lattice's own parameters and
// checks every index in the payload on the host (link nodes, zone boxes,
// counters, node types against the wall layers) before anything is copied to
// the device, so a checkpoint of another deck or a corrupt file is rejected
// with LBMGPU_ERR_INVALID instead of reaching a kernel.
namespace {
struct CkptHeader {
    char magic[8];
    uint32_t version, precision;
    int32_t nx, ny, nz, has_sq;
    int64_t t_main, traj_read;
    int32_t pending_corr, n_links;
    uint64_t f_bytes, sq_bytes;
    // the deck of the stored state (version 2)
    int32_t walls_y, walls_z, planar, mass_correction_every, traj_every, reserved;
    double tau, lambda, fx, fy, fz, radius, b1, beta, rho_p, eps, hc, hmin;
};
constexpr char CKPT_MAGIC[8] = {'L', 'B', 'M', 'G', 'P', 'U', 'C', 'K'};
constexpr uint32_t CKPT_VERSION = 2;

size_t ckpt_payload(const lbmgpu_params& p, int n_links) {
    const size_t N = (size_t)p.nx * p.ny * p.nz;
    size_t b = sizeof(CkptHeader) + (size_t)Q * N * esize_for(p.precision) + N + 4 * N * sizeof(double) + sizeof(SqState);
    if (p.squirmer) b += (size_t)n_links * sizeof(int) + (size_t)TRAJ_RING * TRAJ_COLS * sizeof(double);
    return b;
}
size_t ckpt_bytes(const lbmgpu_handle* h, int n_links) { return ckpt_payload(h->p, n_links); }

void ckpt_fill_deck(CkptHeader& hd, const lbmgpu_params& p) {
    hd.walls_y = p.walls_y; hd.walls_z = p.walls_z; hd.planar = p.planar;
    hd.mass_correction_every = p.mass_correction_every; hd.traj_every = p.traj_every; hd.reserved = 0;
    hd.tau = p.tau; hd.lambda = p.lambda; hd.fx = p.fx; hd.fy = p.fy; hd.fz = p.fz;
    hd.radius = p.radius; hd.b1 = p.b1; hd.beta = p.beta; hd.rho_p = p.rho_p;
    hd.eps = p.eps; hd.hc = p.hc; hd.hmin = p.hmin;
}

// Every check of a checkpoint against the parameters of the lattice it is to
// be loaded into, on the host. Returns an empty string when it may be loaded.
std::string ckpt_check(const lbmgpu_params& p, const void* buf, size_t len) {
    if (!buf) return "null checkpoint buffer";
    if (len < sizeof(CkptHeader)) return "not a checkpoint (too short)";
    CkptHeader hd;
    std::memcpy(&hd, buf, sizeof(hd));
    if (std::memcmp(hd.magic, CKPT_MAGIC, 8) != 0 || hd.version != CKPT_VERSION)
        return "not a checkpoint of this library (magic/version)";
    const size_t N = (size_t)p.nx * p.ny * p.nz;
    if (hd.nx != p.nx || hd.ny != p.ny || hd.nz != p.nz || (int)hd.precision != p.precision ||
        hd.has_sq != p.squirmer || hd.sq_bytes != sizeof(SqState) || hd.f_bytes != (uint64_t)Q * N * esize_for(p.precision))
        return "checkpoint of another lattice (sizes, precision or squirmer differ)";
    CkptHeader mine{};
    ckpt_fill_deck(mine, p);
    const bool same_deck = hd.walls_y == mine.walls_y && hd.walls_z == mine.walls_z &&
                           hd.mass_correction_every == mine.mass_correction_every && hd.traj_every == mine.traj_every &&
                           std::memcmp(&hd.tau, &mine.tau, 5 * sizeof(double)) == 0 &&
                           (!p.squirmer || (hd.planar == mine.planar &&
                                            std::memcmp(&hd.radius, &mine.radius, 7 * sizeof(double)) == 0));
    if (!same_deck)
        return "checkpoint of another deck (walls, tau, lambda, body force, cadences or squirmer model differ)";
    if (hd.t_main < 0 || hd.traj_read < 0 || (hd.pending_corr != 0 && hd.pending_corr != 1))
        return "checkpoint header corrupt (counters)";
    if (hd.n_links < 0 || hd.n_links > (p.squirmer ? link_capacity(p) : 0))
        return "checkpoint link list too long";
    if (len < ckpt_payload(p, hd.n_links)) return "checkpoint truncated";
    // payload: node types against the lattice's wall layers
    const char* q = static_cast<const char*>(buf) + sizeof(hd) + hd.f_bytes;
    const uint8_t* flag = reinterpret_cast<const uint8_t*>(q);
    for (int z = 0; z < p.nz; ++z)
        for (int y = 0; y < p.ny; ++y) {
            const bool wall = is_wall(p, y, z), nw = !wall && near_wall(p, y, z);
            const uint8_t* row = flag + hidx(p, 0, y, z);
            for (int x = 0; x < p.nx; ++x) {
                const uint8_t t = row[x] & TYPE_MASK;
                if (row[x] & ~(uint8_t)(TYPE_MASK | NEAR_WALL | NEAR_PARTICLE) || t > T_PARTICLE)
                    return "checkpoint corrupt: invalid node flag";
                if ((t == T_WALL) != wall || ((row[x] & NEAR_WALL) != 0) != nw || (t == T_PARTICLE && !p.squirmer))
                    return "checkpoint corrupt: node types disagree with the lattice's walls";
            }
        }
    q += N + 4 * N * sizeof(double);
    SqState s;
    std::memcpy(&s, q, sizeof(s));
    q += sizeof(SqState);
    if (s.status != 0) return "checkpoint of a failed run (device status set)";
    if (s.t < 0 || s.traj_count < 0 || s.n_fluid < 0 || s.n_fluid > (long long)N)
        return "checkpoint corrupt: squirmer counters";
    if (!p.squirmer) return std::string();
    if (s.n_links != hd.n_links) return "checkpoint corrupt: link count differs between header and state";
    if (s.R != p.radius || s.B1 != p.b1 || s.beta != p.beta || s.planar != p.planar || s.present != 1)
        return "checkpoint of another deck (squirmer model differs)";
    for (int d = 0; d < 3; ++d)
        if (!std::isfinite(s.X[d]) || !std::isfinite(s.e[d]) || !std::isfinite(s.U[d]) || !std::isfinite(s.W[d]))
            return "checkpoint corrupt: non-finite squirmer state";
    // the centre: unwrapped along x (bounded well inside int range), inside
    // the channel along a walled axis
    if (std::fabs(s.X[0]) > 1e9 || std::fabs(s.X[1]) > 1e9 || std::fabs(s.X[2]) > 1e9 ||
        (p.walls_y && (s.X[1] < 0.0 || s.X[1] > p.ny - 1)) || (p.walls_z && (s.X[2] < 0.0 || s.X[2] > p.nz - 1)))
        return "checkpoint corrupt: squirmer centre outside the lattice";
    // zone boxes: the widths of this lattice, corners inside the ranges the
    // zone kernel indexes from (wrapped along periodic axes)
    const int nd[3] = {p.nx, p.ny, p.nz};
    const bool wall_axis[3] = {false, p.walls_y != 0, p.walls_z != 0};
    for (int k = 0; k < ZONE_SLOTS; ++k)
        for (int d = 0; d < 3; ++d) {
            const int w = s.zone[k].w[d], lo = s.zone[k].lo[d];
            if (w != zone_width(p.radius, nd[d], wall_axis[d])) return "checkpoint corrupt: zone width";
            if (wall_axis[d] ? (lo < -w || lo > nd[d]) : (lo < 0 || lo >= nd[d])) return "checkpoint corrupt: zone corner";
        }
    // link nodes: ascending, inside the lattice, FLUID with the near-particle bit
    const int* links = reinterpret_cast<const int*>(q);
    for (int k = 0; k < hd.n_links; ++k) {
        const int n = links[k];
        if (n < 0 || (size_t)n >= N || (k > 0 && n <= links[k - 1]))
            return "checkpoint corrupt: link node index out of range or out of order";
        if (flag[n] != (T_FLUID | NEAR_PARTICLE) && flag[n] != (T_FLUID | NEAR_PARTICLE | NEAR_WALL))
            return "checkpoint corrupt: link node is not a fluid node next to the sphere";
    }
    return std::string();
}

int ckpt_links(lbmgpu_handle* h, int* n_links) {
    SqState s;
    CUDA_TRY(h, cudaMemcpyAsync(&s, h->sq, sizeof(s), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    *n_links = h->has_sq ? std::max(0, s.n_links) : 0;
    return LBMGPU_OK;
}
}  // namespace

int lbmgpu_checkpoint_size(lbmgpu_handle* h, size_t* bytes) {
    if (!h || !bytes) return LBMGPU_ERR_INVALID;
    CUDA_TRY(h, cudaSetDevice(h->p.device));
    int nl = 0;
    const int rc = ckpt_links(h, &nl);
    if (rc) return rc;
    *bytes = ckpt_bytes(h, nl);
    return LBMGPU_OK;
}

int lbmgpu_checkpoint_save(lbmgpu_handle* h, void* buf, size_t len) {
    if (!h || !buf) return LBMGPU_ERR_INVALID;
    CUDA_TRY(h, cudaSetDevice(h->p.device));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    if (h->zs) CUDA_TRY(h, cudaStreamSynchronize(h->zs));
    int nl = 0;
    int rc = ckpt_links(h, &nl);
    if (rc) return rc;
    if (len < ckpt_bytes(h, nl)) return fail(h, LBMGPU_ERR_INVALID, "checkpoint buffer too small (lbmgpu_checkpoint_size)");
    const size_t N = h->L.N;
    CkptHeader hd{};
    std::memcpy(hd.magic, CKPT_MAGIC, 8);
    hd.version = CKPT_VERSION; hd.precision = (uint32_t)h->p.precision;
    hd.nx = h->p.nx; hd.ny = h->p.ny; hd.nz = h->p.nz; hd.has_sq = h->has_sq;
    hd.t_main = h->t_main; hd.traj_read = h->traj_read; hd.pending_corr = h->pending_corr ? 1 : 0;
    hd.n_links = nl;
    hd.f_bytes = (uint64_t)Q * N * h->esize; hd.sq_bytes = sizeof(SqState);
    ckpt_fill_deck(hd, h->p);
    char* p = static_cast<char*>(buf);
    std::memcpy(p, &hd, sizeof(hd)); p += sizeof(hd);
    cudaStream_t st = h->stream;
    auto d2h = [&](const void* src, size_t n) {
        const cudaError_t e = cudaMemcpyAsync(p, src, n, cudaMemcpyDeviceToHost, st);
        p += n;
        return e;
    };
    CUDA_TRY(h, d2h(h->f, hd.f_bytes));
    CUDA_TRY(h, d2h(h->flag, N));
    CUDA_TRY(h, d2h(h->rho, N * sizeof(double)));
    CUDA_TRY(h, d2h(h->ux, N * sizeof(double)));
    CUDA_TRY(h, d2h(h->uy, N * sizeof(double)));
    CUDA_TRY(h, d2h(h->uz, N * sizeof(double)));
    CUDA_TRY(h, d2h(h->sq, sizeof(SqState)));
    if (h->has_sq) {
        if (nl) CUDA_TRY(h, d2h(h->links, (size_t)nl * sizeof(int)));
        CUDA_TRY(h, d2h(h->traj, (size_t)TRAJ_RING * TRAJ_COLS * sizeof(double)));
    }
    CUDA_TRY(h, cudaStreamSynchronize(st));
    return LBMGPU_OK;
}

int lbmgpu_checkpoint_load(lbmgpu_handle* h, const void* buf, size_t len) {
    if (!h || !buf) return LBMGPU_ERR_INVALID;
    if (h->member) return fail(h, LBMGPU_ERR_INVALID, "handle belongs to an ensemble: advance it with lbmgpu_batch_run");
    const std::string why = ckpt_check(h->p, buf, len);
    if (!why.empty()) return fail(h, LBMGPU_ERR_INVALID, why);
    CkptHeader hd;
    std::memcpy(&hd, buf, sizeof(hd));
    CUDA_TRY(h, cudaSetDevice(h->p.device));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    if (h->zs) CUDA_TRY(h, cudaStreamSynchronize(h->zs));
    const size_t N = h->L.N;
    const char* p = static_cast<const char*>(buf) + sizeof(hd);
    cudaStream_t st = h->stream;
    auto h2d = [&](void* dst, size_t n) {
        const cudaError_t e = cudaMemcpyAsync(dst, p, n, cudaMemcpyHostToDevice, st);
        p += n;
        return e;
    };
    CUDA_TRY(h, h2d(h->f, hd.f_bytes));
    CUDA_TRY(h, h2d(h->flag, N));
    CUDA_TRY(h, h2d(h->rho, N * sizeof(double)));
    CUDA_TRY(h, h2d(h->ux, N * sizeof(double)));
    CUDA_TRY(h, h2d(h->uy, N * sizeof(double)));
    CUDA_TRY(h, h2d(h->uz, N * sizeof(double)));
    CUDA_TRY(h, h2d(h->sq, sizeof(SqState)));
    if (h->has_sq) {
        if (hd.n_links) {
            CUDA_TRY(h, h2d(h->links, (size_t)hd.n_links * sizeof(int)));
            k_scatter_slots<<<64, 256, 0, st>>>(h->links, hd.n_links, h->linkslot);
            ++h->launches;
        }
        CUDA_TRY(h, h2d(h->traj, (size_t)TRAJ_RING * TRAJ_COLS * sizeof(double)));
        // the cached remap shell belongs to this handle's earlier state: rebuild
        // it from the loaded centre (its content never changes results, only
        // which candidates are tested)
        CUDA_TRY(h, cudaMemsetAsync(h->shell_hdr, 0, sizeof(ShellCache), st));
    }
    CUDA_TRY(h, cudaStreamSynchronize(st));
    CUDA_TRY(h, cudaGetLastError());
    h->t_main = hd.t_main;
    h->traj_read = hd.traj_read;
    h->pending_corr = hd.pending_corr != 0;
    return LBMGPU_OK;
}

int lbmgpu_checkpoint_check(const lbmgpu_params* p, const void* buf, size_t len, char* msg, size_t msg_len) {
    std::string m;
    int rc = validate_impl(p, m);
    if (rc == LBMGPU_OK) {
        m = ckpt_check(*p, buf, len);
        rc = m.empty() ? LBMGPU_OK : LBMGPU_ERR_INVALID;
    }
    if (msg && msg_len) std::snprintf(msg, msg_len, "%s", m.c_str());
    return rc;
}

int lbmgpu_get_populations(lbmgpu_handle* h, double* f) {
    if (!h || !f) return LBMGPU_ERR_INVALID;
    CUDA_TRY(h, cudaSetDevice(h->p.device));
    const size_t N = h->L.N;
    const int P = (int)(h->t_main & 1);
    for (int i = 0; i < Q; ++i) {
        h->lz->get_pop(h->L, h->f, h->flag, h->sq, P, i, h->scratch, h->stream);
        ++h->launches;
        CUDA_TRY(h, cudaMemcpyAsync(f + (size_t)i * N, h->scratch, N * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    }
    return check_status(h);
}

int lbmgpu_set_populations(lbmgpu_handle* h, const double* f) {
    if (!h || !f) return LBMGPU_ERR_INVALID;
    if (h->member) return fail(h, LBMGPU_ERR_INVALID, "handle belongs to an ensemble: advance it with lbmgpu_batch_run");
    CUDA_TRY(h, cudaSetDevice(h->p.device));
    const size_t N = h->L.N;
    const int P = (int)(h->t_main & 1);
    for (int i = 0; i < Q; ++i) {
        CUDA_TRY(h, cudaMemcpyAsync(h->scratch, f + (size_t)i * N, N * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        h->lz->set_pop(h->L, h->f, P, i, h->scratch, h->stream);
        ++h->launches;
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    }
    k_clear_pending<<<1, 32, 0, h->stream>>>(h->sq);
    ++h->launches;
    h->pending_corr = false;
    return check_status(h);
}

int lbmgpu_set_stream(lbmgpu_handle* h, void* cuda_stream) {
    if (!h) return LBMGPU_ERR_INVALID;
    if (h->member) return fail(h, LBMGPU_ERR_INVALID, "handle belongs to an ensemble: advance it with lbmgpu_batch_run");
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    h->stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : h->own;
    return LBMGPU_OK;
}

int lbmgpu_time_kernels(lbmgpu_handle* h, int reps, double ms[3]) {
    if (!h || !ms || reps < 1) return LBMGPU_ERR_INVALID;
    if (h->member) return fail(h, LBMGPU_ERR_INVALID, "handle belongs to an ensemble: advance it with lbmgpu_batch_run");
    CUDA_TRY(h, cudaSetDevice(h->p.device));
    reps += reps & 1;
    cudaEvent_t e0, e1;
    CUDA_TRY(h, cudaEventCreate(&e0));
    CUDA_TRY(h, cudaEventCreate(&e1));
    cudaStream_t st = h->stream;
    float t = 0.f;
    auto plan = [&](int k) { return plan_step(h, h->t_main + 1 + k, false, false); };
    // bulk kernel alone
    CUDA_TRY(h, cudaEventRecord(e0, st));
    for (int k = 0; k < reps; ++k) {
        const StepPlan sp = plan(k);
        h->lz->bulk(sp.par, h->has_sq != 0, false, h->L, stream_args(h, sp), h->geom, st);
    }
    CUDA_TRY(h, cudaEventRecord(e1, st));
    CUDA_TRY(h, cudaEventSynchronize(e1));
    CUDA_TRY(h, cudaEventElapsedTime(&t, e0, e1));
    ms[0] = t / reps;
    h->launches += reps;
    // zone kernel alone
    ms[1] = 0.0;
    if (h->geom.bgrid) {
        CUDA_TRY(h, cudaEventRecord(e0, st));
        for (int k = 0; k < reps; ++k) {
            const StepPlan sp = plan(k);
            h->lz->zone(sp.par, h->has_sq != 0, false, h->L, stream_args(h, sp), h->geom, st);
        }
        CUDA_TRY(h, cudaEventRecord(e1, st));
        CUDA_TRY(h, cudaEventSynchronize(e1));
        CUDA_TRY(h, cudaEventElapsedTime(&t, e0, e1));
        ms[1] = t / reps;
        h->launches += reps;
    }
    ms[2] = 0.0;
    if (h->has_sq) {
        CUDA_TRY(h, cudaEventRecord(e0, st));
        for (int k = 0; k < reps; ++k)
            h->lz->squirmer(h->L, squirmer_args(h, (int)(h->t_main & 1), STAGE_FORCE | STAGE_BODY | STAGE_REMAP, 0, -1, -1), st);
        CUDA_TRY(h, cudaEventRecord(e1, st));
        CUDA_TRY(h, cudaEventSynchronize(e1));
        CUDA_TRY(h, cudaEventElapsedTime(&t, e0, e1));
        ms[2] = t / reps;
        h->launches += reps;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return check_status(h);
}

int lbmgpu_launch_count(const lbmgpu_handle* h, long long* n) {
    if (!h || !n) return LBMGPU_ERR_INVALID;
    *n = h->launches;
    return LBMGPU_OK;
}

const char* lbmgpu_last_error(const lbmgpu_handle* h) {
    if (!h) return g_create_error.c_str();
    return h->err.c_str();
}

}  // extern "C"

// ============================================================================
//  Ensembles (lbmgpu_batch_*): many independent lattices advanced together
//  by the batch kernels of k_batch.cuh.
// ============================================================================
namespace {

// Wall force of every member on a macro step (one CTA per member): its row
// entries, then its zone blocks, in the order and with the thread count of
// k_finalize, so the result equals that of the lattice run alone.
__global__ void k_finalize_batch(const MemberParts* __restrict__ mp, const double* row_part, const double* zone_part,
                                 int gzmax, const StreamArgs* __restrict__ args) {
    __shared__ double red[8][3];
    const int m = blockIdx.x;
    const MemberParts q = mp[m];
    double a0 = 0, a1 = 0, a2 = 0;
    for (int k = threadIdx.x; k < q.nrow + q.nzb; k += blockDim.x) {
        const double* p = k < q.nrow ? row_part + (size_t)(q.row0 + k) * BLOCK_PART
                                     : zone_part + ((size_t)m * gzmax + (k - q.nrow)) * BLOCK_PART;
        a0 += p[0]; a1 += p[1]; a2 += p[2];
    }
    for (int o = 16; o > 0; o >>= 1) {
        a0 += __shfl_down_sync(0xffffffffu, a0, o);
        a1 += __shfl_down_sync(0xffffffffu, a1, o);
        a2 += __shfl_down_sync(0xffffffffu, a2, o);
    }
    if ((threadIdx.x & 31) == 0) { red[threadIdx.x >> 5][0] = a0; red[threadIdx.x >> 5][1] = a1; red[threadIdx.x >> 5][2] = a2; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0, s1 = 0, s2 = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { s0 += red[w][0]; s1 += red[w][1]; s2 += red[w][2]; }
        SqState* sq = args[m].sq;
        sq->wall_force[0] = s0; sq->wall_force[1] = s1; sq->wall_force[2] = s2;
    }
}

// status words of all members, OR-ed
__global__ void k_batch_status(const StreamArgs* args, int n, int* out) {
    int st = 0;
    for (int m = threadIdx.x; m < n; m += blockDim.x) st |= args[m].sq->status;
    for (int o = 16; o > 0; o >>= 1) st |= __shfl_down_sync(0xffffffffu, st, o);
    __shared__ int red[8];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = st;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t |= red[w];
        *out = t;
    }
}

}  // namespace

struct lbmgpu_batch {
    std::vector<lbmgpu_handle*> m;
    lbmgpu_params p0{};
    const Launchers* lz = nullptr;
    int has_sq = 0, period = 6, sms = 148;
    bool corr_in_graph = false;
    cudaStream_t own = nullptr;    // the ensemble's own caller-facing stream
    cudaStream_t sa = nullptr;     // the caller-facing stream in use (own or the caller's)
    cudaStream_t sb = nullptr, cap = nullptr, cap2 = nullptr;
    cudaEvent_t ev_b[2] = {nullptr, nullptr}, ev_z = nullptr, ev_s = nullptr, ev_fork = nullptr, ev_join = nullptr;
    void* fpool = nullptr;
    uint8_t* flagpool = nullptr;
    Lattice* d_lat = nullptr;
    StreamArgs* d_args = nullptr;
    SqArgs* d_sqargs = nullptr;
    RowRef* d_rows = nullptr;
    RowRef* d_wrows = nullptr;
    MemberParts* d_parts = nullptr;
    int2* d_zblocks = nullptr;     // (member, block) of every zone block
    int4* d_runs = nullptr;        // staged-run kernel: runs of interior rows
    double *row_part = nullptr, *zone_part = nullptr;
    int* d_status = nullptr;
    BatchArgs ba{};
    // tiling of the bulk launch (autotuned): tile > 0 is k_bulk_batch with that
    // many threads per row, tile < 0 is k_bulk_staged with -tile stages;
    // the grid is bps CTAs per SM
    int tile = LBMGPU_TILE_CHUNKP, bps = 4;   // bps: resident CTAs per SM, set at creation
    int* d_bounds = nullptr;       // staged kernel: row range of each CTA
    ChunkRef* d_chunks = nullptr;  // chunk kernel
    ChunkRef* d_flat = nullptr;    // persistent chunk kernel, steps without sums
    RowChunks* d_rowchunks = nullptr;
    double* chunk_part = nullptr;
    int bounds_cap = 0, bounds_grid = 0;
    std::vector<long long> row_prefix;   // nodes in the rows before row r (rows away from walls)
    long long cells = 0, t = 0, launches = 0;
    bool pending_corr = false;
    Graph g[2];   // captured patterns; index 1: the first step applies a pending correction
    std::string err;
};

namespace {

int bfail(lbmgpu_batch* b, int code, const std::string& msg) {
    if (b) b->err = msg; else g_create_error = msg;
    return code;
}

#define BTRY(b, call)                                                                              \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return bfail(b, e_ == cudaErrorMemoryAllocation ? LBMGPU_ERR_NOMEM : LBMGPU_ERR_CUDA,   \
                         std::string(#call) + ": " + cudaGetErrorString(e_));                      \
    } while (0)

void batch_drop_graphs(lbmgpu_batch* b);

void batch_free(lbmgpu_batch* b) {
    batch_drop_graphs(b);
    for (lbmgpu_handle* h : b->m) {
        h->member = true;
        free_all(h);
        delete h;
    }
    b->m.clear();
    void* ptrs[] = {b->fpool, b->flagpool, b->d_lat, b->d_args, b->d_sqargs, b->d_rows, b->d_wrows, b->d_parts, b->d_zblocks, b->d_runs,
                    b->row_part, b->zone_part, b->d_status, b->d_bounds, b->d_chunks, b->d_rowchunks,
                    b->chunk_part, b->d_flat};
    for (void* q : ptrs) if (q) cudaFree(q);
    for (cudaEvent_t e : {b->ev_b[0], b->ev_b[1], b->ev_z, b->ev_s, b->ev_fork, b->ev_join})
        if (e) cudaEventDestroy(e);
    for (cudaStream_t s : {b->own, b->sb, b->cap, b->cap2})
        if (s) cudaStreamDestroy(s);
}

bool is_corr_batch(const lbmgpu_batch* b, long long s) {
    const int k = b->p0.mass_correction_every;
    return b->has_sq && k > 0 && s % k == 0;
}

// Row ranges of the staged kernel's CTAs: contiguous, with equal node counts.
int set_bounds(lbmgpu_batch* b, int grid) {
    if (b->bounds_grid == grid && b->d_bounds) return LBMGPU_OK;
    if (grid + 1 > b->bounds_cap) {
        if (b->d_bounds) cudaFree(b->d_bounds);
        b->d_bounds = nullptr;
        b->bounds_cap = 0;
        BTRY(b, cudaMalloc(&b->d_bounds, (size_t)(grid + 1) * sizeof(int)));
        b->bounds_cap = grid + 1;
        b->ba.bounds = b->d_bounds;
    }
    const std::vector<long long>& pre = b->row_prefix;   // size nrows + 1
    const int nrows = (int)pre.size() - 1;
    std::vector<int> bd(grid + 1);
    bd[0] = 0;
    int r = 0;
    for (int c = 1; c < grid; ++c) {
        const long long target = pre[nrows] * c / grid;
        while (r < nrows && pre[r] < target) ++r;
        bd[c] = r;
    }
    bd[grid] = nrows;
    BTRY(b, cudaMemcpy(b->d_bounds, bd.data(), (size_t)(grid + 1) * sizeof(int), cudaMemcpyHostToDevice));
    b->bounds_grid = grid;
    return LBMGPU_OK;
}

// the bulk launch (rows away from walls) with a given tiling
void launch_bulk(lbmgpu_batch* b, int tile, int grid, int par, bool macro, BatchStep bst, cudaStream_t s) {
    if (tile < 0) b->lz->batch_staged(par, macro, -tile, grid, b->ba, bst, s);
    else if (tile == LBMGPU_TILE_ROWCTA) b->lz->batch_rowcta(par, macro, false, b->ba, bst, s);
    else if (tile == LBMGPU_TILE_CHUNK) b->lz->batch_chunk(par, macro, macro || bst.do_mass, 0, b->ba, bst, s);
    else if (tile == LBMGPU_TILE_CHUNKP) b->lz->batch_chunk(par, macro, macro || bst.do_mass, grid, b->ba, bst, s);
    else if (tile == LBMGPU_TILE_RUNS) {
        if (macro || bst.do_mass)   // sums in k_bulk's row order: the persistent chunks, one wave
            b->lz->batch_chunk(par, macro, true, b->sms * std::min(16, b->lz->chunkp_ctas_per_sm()), b->ba, bst, s);
        else
            b->lz->batch_runs(par, grid, b->ba, bst, s);
    }
    else b->lz->batch_bulk(par, macro, false, tile, grid, b->ba, bst, s);
}

void issue_batch(lbmgpu_batch* b, cudaStream_t sa, cudaStream_t sb, long long s, bool macro, bool apply,
                 bool capture = false) {
    const int par = (int)((s - 1) & 1);
    const bool corr = is_corr_batch(b, s) && (!capture || b->corr_in_graph);
    const BatchStep bst{(int)(s % ZONE_SLOTS), corr ? 1 : 0, apply ? 1 : 0};
    const int grid = b->sms * b->bps;
    cudaStreamWaitEvent(sa, b->ev_z, 0);
    if (apply) cudaStreamWaitEvent(sa, b->ev_s, 0);
    launch_bulk(b, b->tile, grid, par, macro, bst, sa);
    cudaEventRecord(b->ev_b[s & 1], sa);
    cudaStreamWaitEvent(sb, b->ev_b[(s - 1) & 1], 0);
    int k = 1;
    if (b->ba.nwrows) {
        b->lz->batch_rowcta(par, macro, true, b->ba, bst, sb);   // one CTA per wall row
        ++k;
    }
    if (b->has_sq) { b->lz->batch_zone(par, macro, b->ba, bst, sb); ++k; }
    cudaEventRecord(b->ev_z, sb);
    if (macro) {
        cudaStreamWaitEvent(sb, b->ev_b[s & 1], 0);
        k_finalize_batch<<<(unsigned)b->m.size(), 256, 0, sb>>>(b->d_parts, b->row_part, b->zone_part, b->ba.gzmax,
                                                               b->d_args);
        ++k;
    }
    if (b->has_sq) {
        if (corr) cudaStreamWaitEvent(sb, b->ev_b[s & 1], 0);
        const SqStep sst{par ^ 1, STAGE_FORCE | STAGE_BODY | STAGE_REMAP | STAGE_LOOP, corr ? 1 : 0,
                         (int)((s + 2) % ZONE_SLOTS), -1};
        b->lz->batch_squirmer(b->ba, sst, sb);
        cudaEventRecord(b->ev_s, sb);
        ++k;
    }
    b->launches += k;
}

void batch_begin(lbmgpu_batch* b, cudaStream_t sa, cudaStream_t sb) {
    cudaEventRecord(b->ev_fork, sa);
    cudaStreamWaitEvent(sb, b->ev_fork, 0);
    for (cudaEvent_t e : {b->ev_b[0], b->ev_b[1], b->ev_z, b->ev_s}) cudaEventRecord(e, sa);
}
void batch_end(lbmgpu_batch* b, cudaStream_t sa, cudaStream_t sb) {
    cudaEventRecord(b->ev_join, sb);
    cudaStreamWaitEvent(sa, b->ev_join, 0);
}

// The ensemble's captured pattern (see ensure_graph): apply0 = its first
// step applies the correction of the step before the pattern.
int batch_graph(lbmgpu_batch* b, int steps, bool apply0) {
    Graph& g = b->g[apply0 ? 1 : 0];
    if (g.exec && g.steps == steps) return LBMGPU_OK;
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
    g = Graph{};
    BTRY(b, cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
    const long long saved = b->launches;
    batch_begin(b, b->cap, b->cap2);
    for (int k = 0; k < steps; ++k) {
        const long long s = 1 + k;
        const bool apply = k == 0 ? apply0 : b->corr_in_graph && is_corr_batch(b, s - 1);
        issue_batch(b, b->cap, b->cap2, s, false, apply, true);
    }
    batch_end(b, b->cap, b->cap2);
    b->launches = saved;
    BTRY(b, cudaStreamEndCapture(b->cap, &g.graph));
    BTRY(b, cudaGraphInstantiate(&g.exec, g.graph, 0));
    g.steps = steps;
    return LBMGPU_OK;
}

void batch_drop_graphs(lbmgpu_batch* b) {
    for (Graph& g : b->g) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.graph) cudaGraphDestroy(g.graph);
        g = Graph{};
    }
}

int batch_status(lbmgpu_batch* b) {
    BTRY(b, cudaGetLastError());
    k_batch_status<<<1, 256, 0, b->sa>>>(b->d_args, (int)b->m.size(), b->d_status);
    int st = 0;
    BTRY(b, cudaMemcpyAsync(&st, b->d_status, sizeof(int), cudaMemcpyDeviceToHost, b->sa));
    BTRY(b, cudaStreamSynchronize(b->sa));
    if (st & ST_NAN) return bfail(b, LBMGPU_ERR_NAN, "non-finite squirmer force, torque or state in a member");
    if (st & ST_WATCHDOG) return bfail(b, LBMGPU_ERR_WATCHDOG, "a staged row did not arrive in shared memory in time");
    if (st & (ST_REMAP_RANGE | ST_LINK_OVERFLOW | ST_REMAP_OVERFLOW))
        return bfail(b, LBMGPU_ERR_DEVICE, "a member's squirmer update failed a consistency check");
    return LBMGPU_OK;
}

}  // namespace

extern "C" {

int lbmgpu_batch_create(const lbmgpu_params* ps, int n, lbmgpu_batch** out) {
    if (!out || !ps || n < 1) return bfail(nullptr, LBMGPU_ERR_INVALID, "need at least one member");
    *out = nullptr;
    const lbmgpu_params& p0 = ps[0];
    for (int i = 0; i < n; ++i) {
        std::string m;
        if (validate_impl(&ps[i], m) != LBMGPU_OK)
            return bfail(nullptr, LBMGPU_ERR_INVALID, "member " + std::to_string(i) + ": " + m);
        const lbmgpu_params& q = ps[i];
        if (q.tau != p0.tau || q.lambda != p0.lambda || q.fx != p0.fx || q.fy != p0.fy || q.fz != p0.fz ||
            q.walls_y != p0.walls_y || q.walls_z != p0.walls_z || q.precision != p0.precision ||
            q.mass_correction_every != p0.mass_correction_every || q.squirmer != p0.squirmer || q.device != p0.device)
            return bfail(nullptr, LBMGPU_ERR_INVALID,
                         "member " + std::to_string(i) + ": members must share tau, lambda, body force, walls, "
                         "precision, mass_correction_every, squirmer and device");
        if (q.nx > BATCH_MAX_NX)
            return bfail(nullptr, LBMGPU_ERR_INVALID,
                         "member " + std::to_string(i) + ": nx must be <= " + std::to_string(BATCH_MAX_NX) + " in an ensemble");
    }
    lbmgpu_batch* b = new lbmgpu_batch();
    b->p0 = p0;
    b->lz = launchers_for(p0.precision);
    b->has_sq = p0.squirmer;
    auto bail = [&](int rc) {
        g_create_error = b->err;
        batch_free(b);
        delete b;
        return rc;
    };
#define CB(call)                                                                                    \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) {                                                                    \
            b->err = std::string(#call) + ": " + cudaGetErrorString(e_);                            \
            return bail(e_ == cudaErrorMemoryAllocation ? LBMGPU_ERR_NOMEM : LBMGPU_ERR_CUDA);      \
        }                                                                                           \
    } while (0)
    CB(cudaSetDevice(p0.device));
    CB(b->lz->prepare());
    CB(cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, p0.device));
    int prio_lo = 0, prio_hi = 0;
    CB(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
    CB(cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking));
    b->sa = b->own;
    CB(cudaStreamCreateWithPriority(&b->sb, cudaStreamNonBlocking, prio_hi));
    CB(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
    CB(cudaStreamCreateWithPriority(&b->cap2, cudaStreamNonBlocking, prio_hi));
    for (cudaEvent_t* e : {&b->ev_b[0], &b->ev_b[1], &b->ev_z, &b->ev_s, &b->ev_fork, &b->ev_join})
        CB(cudaEventCreateWithFlags(e, cudaEventDisableTiming));

    // the packed pools: every member's populations back to back, then flags
    const size_t es = esize_for(p0.precision);
    std::vector<size_t> foff(n), goff(n);
    size_t ftot = 0, gtot = 0;
    for (int i = 0; i < n; ++i) {
        const size_t N = (size_t)ps[i].nx * ps[i].ny * ps[i].nz;
        foff[i] = ftot; ftot += ((size_t)Q * N * es + 255) / 256 * 256;
        goff[i] = gtot; gtot += (N + 255) / 256 * 256;
        b->cells += (long long)N;
    }
    CB(cudaMalloc(&b->fpool, ftot));
    CB(cudaMalloc(&b->flagpool, gtot));
    for (int i = 0; i < n; ++i) {
        MemberOpts mo{b->sa, static_cast<char*>(b->fpool) + foff[i], b->flagpool + goff[i]};
        lbmgpu_handle* h = nullptr;
        const int rc = create_impl(&ps[i], &mo, &h);
        if (rc != LBMGPU_OK) {
            b->err = "member " + std::to_string(i) + ": " + g_create_error;
            return bail(rc);
        }
        b->m.push_back(h);
    }

    // rows (away from walls / next to a wall) and the partial-sum layout: each
    // member owns ny*nz row entries indexed y + ny*z (the wall layers' stay 0)
    // and gzmax zone-block entries, as a lattice run alone lays out its blocks
    std::vector<RowRef> rows, wrows;
    std::vector<MemberParts> parts(n);
    int gzmax = 1;
    size_t nparts = 0;
    for (int i = 0; i < n; ++i) {
        const lbmgpu_params& q = ps[i];
        parts[i].row0 = (int)nparts;
        parts[i].nrow = q.ny * q.nz;
        for (int z = 0; z < q.nz; ++z)
            for (int y = 0; y < q.ny; ++y) {
                if (is_wall(q, y, z)) continue;
                (near_wall(q, y, z) ? wrows : rows).push_back(RowRef{i, y, z, (int)nparts + y + q.ny * z});
            }
        nparts += (size_t)q.ny * q.nz;
        parts[i].nzb = b->has_sq ? (int)b->m[i]->geom.bgrid : 0;
        gzmax = std::max(gzmax, parts[i].nzb);
    }
    // runs of consecutive interior rows of a plane for the staged-run kernel:
    // rows 0 and ny-1 (interior only without walls in y) stay single, so an
    // odd step's source rows y - c_y of a longer run never wrap
    std::vector<int4> runs;
    {
        const int maxn = b->lz->runs_max_nodes;
        for (int i = 0; i < n; ++i) {
            const lbmgpu_params& q = ps[i];
            const int R = std::max(1, maxn / q.nx);
            for (int z = 0; z < q.nz; ++z) {
                int y = 0;
                while (y < q.ny) {
                    if (is_wall(q, y, z) || near_wall(q, y, z)) { ++y; continue; }
                    int len = 1;
                    if (y > 0 && y < q.ny - 1)
                        while (len < R && y + len < q.ny - 1 && !is_wall(q, y + len, z) && !near_wall(q, y + len, z))
                            ++len;
                    runs.push_back(make_int4(i, y, z, len));
                    y += len;
                }
            }
        }
    }
    CB(cudaMalloc(&b->d_runs, std::max<size_t>(1, runs.size()) * sizeof(int4)));
    if (!runs.empty())
        CB(cudaMemcpy(b->d_runs, runs.data(), runs.size() * sizeof(int4), cudaMemcpyHostToDevice));
    CB(cudaMalloc(&b->d_rows, std::max<size_t>(1, rows.size()) * sizeof(RowRef)));
    CB(cudaMalloc(&b->d_wrows, std::max<size_t>(1, wrows.size()) * sizeof(RowRef)));
    CB(cudaMalloc(&b->row_part, nparts * BLOCK_PART * sizeof(double)));
    CB(cudaMalloc(&b->zone_part, (size_t)n * gzmax * BLOCK_PART * sizeof(double)));
    CB(cudaMalloc(&b->d_parts, (size_t)n * sizeof(MemberParts)));
    std::vector<int2> zblocks;
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < parts[i].nzb; ++k) zblocks.push_back(make_int2(i, k));
    CB(cudaMalloc(&b->d_zblocks, std::max<size_t>(1, zblocks.size()) * sizeof(int2)));
    if (!zblocks.empty())
        CB(cudaMemcpy(b->d_zblocks, zblocks.data(), zblocks.size() * sizeof(int2), cudaMemcpyHostToDevice));
    CB(cudaMalloc(&b->d_lat, (size_t)n * sizeof(Lattice)));
    CB(cudaMalloc(&b->d_args, (size_t)n * sizeof(StreamArgs)));
    CB(cudaMalloc(&b->d_sqargs, (size_t)n * sizeof(SqArgs)));
    CB(cudaMalloc(&b->d_status, sizeof(int)));
    std::vector<Lattice> lat(n);
    std::vector<StreamArgs> args(n);
    std::vector<SqArgs> sqa(n);
    for (int i = 0; i < n; ++i) {
        lbmgpu_handle* h = b->m[i];
        lat[i] = h->L;
        args[i] = stream_args(h, plan_step(h, 1, false, false));
        sqa[i] = squirmer_args(h, 0, 0, 0, -1, -1);
        sqa[i].block_part = b->row_part + (size_t)parts[i].row0 * BLOCK_PART;
        sqa[i].nblocks = parts[i].nrow;
        sqa[i].block_part_b = b->zone_part + (size_t)i * gzmax * BLOCK_PART;
        sqa[i].nblocks_b = parts[i].nzb;
        sqa[i].block_part_w = nullptr;
        sqa[i].nblocks_w = 0;
    }
    // 32-node chunks of the rows away from walls, and each row's chunk range
    std::vector<ChunkRef> chunks;
    std::vector<RowChunks> rowchunks(rows.size());
    for (size_t r = 0; r < rows.size(); ++r) {
        const int nx = ps[rows[r].m].nx;
        rowchunks[r] = RowChunks{(int)chunks.size(), (nx + 31) / 32, rows[r].part, 0};
        for (int x0 = 0; x0 < nx; x0 += 32) chunks.push_back(ChunkRef{rows[r].m, rows[r].y, rows[r].z, x0});
    }
    // Runs of consecutive rows away from walls in one z-plane of one member are
    // contiguous in memory; on steps without sums the persistent chunk kernel
    // walks them in full 32-node pieces ([x0, x0 + len) from row y, continuing
    // into the next rows), so no lane idles at a row's end.
    std::vector<ChunkRef> flat;
    for (size_t r = 0; r < rows.size();) {
        size_t e = r + 1;
        while (e < rows.size() && rows[e].m == rows[r].m && rows[e].z == rows[r].z &&
               rows[e].y == rows[e - 1].y + 1)
            ++e;
        const int nx = ps[rows[r].m].nx;
        const long long total = (long long)(e - r) * nx;
        for (long long o = 0; o < total; o += 32) {
            const int len = (int)std::min<long long>(32, total - o);
            const int y = rows[r].y + (int)(o / nx), x0 = (int)(o % nx);
            flat.push_back(ChunkRef{rows[r].m, y, rows[r].z, x0 | (len << 16)});
        }
        r = e;
    }
    CB(cudaMalloc(&b->d_flat, std::max<size_t>(1, flat.size()) * sizeof(ChunkRef)));
    if (!flat.empty())
        CB(cudaMemcpyAsync(b->d_flat, flat.data(), flat.size() * sizeof(ChunkRef), cudaMemcpyHostToDevice, b->sa));
    b->ba.flat = b->d_flat; b->ba.nflat = (int)flat.size();
    CB(cudaMalloc(&b->d_chunks, std::max<size_t>(1, chunks.size()) * sizeof(ChunkRef)));
    CB(cudaMalloc(&b->d_rowchunks, std::max<size_t>(1, rowchunks.size()) * sizeof(RowChunks)));
    CB(cudaMalloc(&b->chunk_part, std::max<size_t>(1, chunks.size()) * BLOCK_PART * sizeof(double)));
    cudaStream_t st = b->sa;
    if (!chunks.empty()) {
        CB(cudaMemcpyAsync(b->d_chunks, chunks.data(), chunks.size() * sizeof(ChunkRef), cudaMemcpyHostToDevice, st));
        CB(cudaMemcpyAsync(b->d_rowchunks, rowchunks.data(), rowchunks.size() * sizeof(RowChunks),
                           cudaMemcpyHostToDevice, st));
    }
    b->ba.chunks = b->d_chunks; b->ba.nchunks = (int)chunks.size();
    b->ba.rowchunks = b->d_rowchunks; b->ba.chunk_part = b->chunk_part;
    CB(cudaMemcpyAsync(b->d_rows, rows.data(), rows.size() * sizeof(RowRef), cudaMemcpyHostToDevice, st));
    if (!wrows.empty())
        CB(cudaMemcpyAsync(b->d_wrows, wrows.data(), wrows.size() * sizeof(RowRef), cudaMemcpyHostToDevice, st));
    CB(cudaMemcpyAsync(b->d_parts, parts.data(), n * sizeof(MemberParts), cudaMemcpyHostToDevice, st));
    CB(cudaMemcpyAsync(b->d_lat, lat.data(), n * sizeof(Lattice), cudaMemcpyHostToDevice, st));
    CB(cudaMemcpyAsync(b->d_args, args.data(), n * sizeof(StreamArgs), cudaMemcpyHostToDevice, st));
    CB(cudaMemcpyAsync(b->d_sqargs, sqa.data(), n * sizeof(SqArgs), cudaMemcpyHostToDevice, st));
    CB(cudaMemsetAsync(b->row_part, 0, nparts * BLOCK_PART * sizeof(double), st));
    CB(cudaMemsetAsync(b->zone_part, 0, (size_t)n * gzmax * BLOCK_PART * sizeof(double), st));
    CB(cudaStreamSynchronize(st));
    b->ba.lat = b->d_lat; b->ba.args = b->d_args; b->ba.sqargs = b->d_sqargs;
    b->ba.rows = b->d_rows; b->ba.nrows = (int)rows.size();
    b->ba.wrows = b->d_wrows; b->ba.nwrows = (int)wrows.size();
    b->ba.row_part = b->row_part; b->ba.zone_part = b->zone_part;
    b->ba.gzmax = gzmax; b->ba.nmembers = n; b->ba.parts = b->d_parts;
    b->ba.zblocks = b->d_zblocks; b->ba.nzblocks = (int)zblocks.size();
    b->ba.runs = b->d_runs; b->ba.nruns = (int)runs.size();
    {
        int nxmax = 1;
        for (int i = 0; i < n; ++i) nxmax = std::max(nxmax, ps[i].nx);
        const size_t es = b->lz->esize;
        b->ba.cap = (int)(((size_t)nxmax * es + 32 + 15) / 16 * 16 / es);
        b->ba.fcap = (nxmax + 32 + 15) / 16 * 16;
        b->row_prefix.assign(rows.size() + 1, 0);
        for (size_t r = 0; r < rows.size(); ++r) b->row_prefix[r + 1] = b->row_prefix[r] + ps[rows[r].m].nx;
    }
    const int k = p0.mass_correction_every;
    const int base = std::lcm(2, ZONE_SLOTS);
    b->corr_in_graph = b->has_sq && k > 0 && std::lcm(base, k) <= MAX_PERIOD;
    b->period = b->corr_in_graph ? std::lcm(base, k) : base;
    b->bps = std::min(16, b->lz->chunkp_ctas_per_sm());   // one wave of the persistent chunk kernel
    if (set_bounds(b, b->sms * b->bps) != LBMGPU_OK) return bail(LBMGPU_ERR_CUDA);
#undef CB
    *out = b;
    return LBMGPU_OK;
}

int lbmgpu_batch_destroy(lbmgpu_batch* b) {
    if (!b) return LBMGPU_OK;
    cudaSetDevice(b->p0.device);
    if (b->sa) cudaStreamSynchronize(b->sa);
    if (b->sb) cudaStreamSynchronize(b->sb);
    batch_free(b);
    delete b;
    return LBMGPU_OK;
}

int lbmgpu_batch_size(const lbmgpu_batch* b, int* members, long long* cells) {
    if (!b) return LBMGPU_ERR_INVALID;
    if (members) *members = (int)b->m.size();
    if (cells) *cells = b->cells;
    return LBMGPU_OK;
}

int lbmgpu_batch_member(lbmgpu_batch* b, int i, lbmgpu_handle** h) {
    if (!b || !h || i < 0 || i >= (int)b->m.size()) return bfail(b, LBMGPU_ERR_INVALID, "no such member");
    *h = b->m[i];
    return LBMGPU_OK;
}

int lbmgpu_batch_run(lbmgpu_batch* b, int nsteps) {
    if (!b) return LBMGPU_ERR_INVALID;
    if (nsteps < 0) return bfail(b, LBMGPU_ERR_INVALID, "nsteps must be >= 0");
    if (nsteps == 0) return LBMGPU_OK;
    BTRY(b, cudaSetDevice(b->p0.device));
    cudaStream_t sa = b->sa, sb = b->sb;
    const int per_step = 1 + (b->ba.nwrows ? 1 : 0) + (b->has_sq ? 2 : 0);
    const int gsteps = b->period * ((MIN_GRAPH + b->period - 1) / b->period);
    batch_begin(b, sa, sb);
    long long rem = nsteps;
    while (rem > 0) {
        const bool last = rem == 1;
        bool graph_ok = !last && b->t % b->period == 0 && rem - 1 >= gsteps;
        if (graph_ok && b->has_sq && b->p0.mass_correction_every > 0 && !b->corr_in_graph) {
            const int k = b->p0.mass_correction_every;
            graph_ok = (b->t / k) == ((b->t + gsteps) / k);
        }
        if (graph_ok) {
            batch_end(b, sa, sb);
            int rc = batch_graph(b, gsteps, b->pending_corr);
            if (rc) return rc;
            BTRY(b, cudaGraphLaunch(b->g[b->pending_corr ? 1 : 0].exec, sa));
            b->launches += (long long)gsteps * per_step;
            b->t += gsteps;
            rem -= gsteps;
            b->pending_corr = is_corr_batch(b, b->t);
            batch_begin(b, sa, sb);
            continue;
        }
        const long long s = b->t + 1;
        issue_batch(b, sa, sb, s, last, b->pending_corr);
        b->t = s;
        b->pending_corr = is_corr_batch(b, s);
        --rem;
    }
    batch_end(b, sa, sb);
    for (lbmgpu_handle* h : b->m) { h->t_main = b->t; h->pending_corr = b->pending_corr; }
    return batch_status(b);
}

int lbmgpu_batch_set_tiling(lbmgpu_batch* b, int tile, int ctas_per_sm) {
    if (!b) return LBMGPU_ERR_INVALID;
    if ((tile != 32 && tile != 64 && tile != 128 && tile != LBMGPU_TILE_STAGED3 && tile != LBMGPU_TILE_STAGED4 &&
         tile != LBMGPU_TILE_ROWCTA && tile != LBMGPU_TILE_CHUNK && tile != LBMGPU_TILE_CHUNKP &&
         tile != LBMGPU_TILE_RUNS) ||
        ctas_per_sm < 1 || ctas_per_sm > 16)
        return bfail(b, LBMGPU_ERR_INVALID, "tile must be 32, 64, 128 (threads per row), LBMGPU_TILE_ROWCTA, "
                                            "LBMGPU_TILE_CHUNK(P), LBMGPU_TILE_RUNS or "
                                            "LBMGPU_TILE_STAGED3/4, and ctas_per_sm 1..16");
    BTRY(b, cudaSetDevice(b->p0.device));
    BTRY(b, cudaStreamSynchronize(b->sa));
    BTRY(b, cudaStreamSynchronize(b->sb));
    const int rc = set_bounds(b, b->sms * ctas_per_sm);
    if (rc) return rc;
    b->tile = tile;
    b->bps = ctas_per_sm;
    batch_drop_graphs(b);
    return LBMGPU_OK;
}

int lbmgpu_batch_autotune(lbmgpu_batch* b, int reps, int* threads_per_row, int* ctas_per_sm, double* best_ms) {
    if (!b || reps < 1) return LBMGPU_ERR_INVALID;
    BTRY(b, cudaSetDevice(b->p0.device));
    cudaStream_t st = b->sa;
    BTRY(b, cudaStreamSynchronize(b->sb));
    // the candidates run real steps (without the sphere update); the
    // populations are saved first and restored afterwards
    size_t bytes = 0;
    for (lbmgpu_handle* h : b->m) bytes += ((size_t)Q * h->L.N * h->esize + 255) / 256 * 256;
    void* save = nullptr;
    BTRY(b, cudaMalloc(&save, bytes));
    BTRY(b, cudaMemcpyAsync(save, b->fpool, bytes, cudaMemcpyDeviceToDevice, st));
    cudaEvent_t e0, e1;
    BTRY(b, cudaEventCreate(&e0));
    BTRY(b, cudaEventCreate(&e1));
    const int tiles[9] = {LBMGPU_TILE_CHUNK, LBMGPU_TILE_CHUNKP, LBMGPU_TILE_ROWCTA, 32, 64, 128,
                          LBMGPU_TILE_STAGED3, LBMGPU_TILE_STAGED4, LBMGPU_TILE_RUNS};
    const int bpss[8] = {1, 2, 3, 4, 5, 6, 7, 8};
    double best = 1e30;
    int btx = b->tile, bbps = b->bps;
    const BatchStep bst{(int)((b->t + 1) % ZONE_SLOTS), 0, 0};
    for (int tx : tiles)
        for (int bps : bpss) {
            if ((tx == LBMGPU_TILE_ROWCTA || tx == LBMGPU_TILE_CHUNK) && bps != 1) continue;   // grid = rows / chunks
            if (tx == LBMGPU_TILE_RUNS && bps > 3) continue;   // shared memory holds at most 2 resident
            const int grid = b->sms * bps;
            if (tx < 0) {
                const int rc = set_bounds(b, grid);
                if (rc) return rc;
            }
            launch_bulk(b, tx, grid, 0, false, bst, st);  // warm-up
            launch_bulk(b, tx, grid, 1, false, bst, st);
            BTRY(b, cudaEventRecord(e0, st));
            for (int r = 0; r < reps; ++r) {
                launch_bulk(b, tx, grid, 0, false, bst, st);
                launch_bulk(b, tx, grid, 1, false, bst, st);
            }
            BTRY(b, cudaEventRecord(e1, st));
            BTRY(b, cudaEventSynchronize(e1));
            float ms = 0.f;
            BTRY(b, cudaEventElapsedTime(&ms, e0, e1));
            b->launches += 2 * reps + 2;
            const double per = ms / (2.0 * reps);
            if (per < best) { best = per; btx = tx; bbps = bps; }
        }
    BTRY(b, cudaMemcpyAsync(b->fpool, save, bytes, cudaMemcpyDeviceToDevice, st));
    BTRY(b, cudaStreamSynchronize(st));
    cudaFree(save);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const int rc = lbmgpu_batch_set_tiling(b, btx, bbps);
    if (rc) return rc;
    if (threads_per_row) *threads_per_row = btx;
    if (ctas_per_sm) *ctas_per_sm = bbps;
    if (best_ms) *best_ms = best;
    return batch_status(b);
}

int lbmgpu_batch_time_bulk(lbmgpu_batch* b, int reps, double* ms_per_launch) {
    if (!b || reps < 1 || !ms_per_launch) return LBMGPU_ERR_INVALID;
    BTRY(b, cudaSetDevice(b->p0.device));
    cudaStream_t st = b->sa;
    BTRY(b, cudaStreamSynchronize(b->sb));
    cudaEvent_t e0, e1;
    BTRY(b, cudaEventCreate(&e0));
    BTRY(b, cudaEventCreate(&e1));
    const BatchStep bst{(int)((b->t + 1) % ZONE_SLOTS), 0, 0};
    const int grid = b->sms * b->bps;
    BTRY(b, cudaEventRecord(e0, st));
    for (int r = 0; r < reps; ++r) {
        launch_bulk(b, b->tile, grid, (int)((b->t + 2 * r) & 1), false, bst, st);
        launch_bulk(b, b->tile, grid, (int)((b->t + 2 * r + 1) & 1), false, bst, st);
    }
    BTRY(b, cudaEventRecord(e1, st));
    BTRY(b, cudaEventSynchronize(e1));
    float ms = 0.f;
    BTRY(b, cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->launches += 2 * reps;
    *ms_per_launch = ms / (2.0 * reps);
    return batch_status(b);
}

int lbmgpu_batch_set_stream(lbmgpu_batch* b, void* cuda_stream) {
    if (!b) return LBMGPU_ERR_INVALID;
    BTRY(b, cudaStreamSynchronize(b->sa));
    b->sa = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : b->own;
    for (lbmgpu_handle* h : b->m) h->stream = b->sa;
    return LBMGPU_OK;
}

int lbmgpu_batch_launch_count(const lbmgpu_batch* b, long long* n) {
    if (!b || !n) return LBMGPU_ERR_INVALID;
    *n = b->launches;
    return LBMGPU_OK;
}

const char* lbmgpu_batch_last_error(const lbmgpu_batch* b) {
    if (!b) return g_create_error.c_str();
    return b->err.c_str();
}

}  // extern "C"

// ============================================================================
//  lbmgpu_watchdog_selftest: the bounded-wait path of the device kernels,
//  exercised without a fault. One CTA waits on a shared-memory mbarrier that
//  nothing arrives at, with the given try limit; when the wait gives up the
//  kernel sets ST_WATCHDOG in a status word and returns, as the staged bulk
//  kernel does, and the host turns that into LBMGPU_ERR_WATCHDOG.
// ============================================================================
namespace {
__global__ void k_watchdog_selftest(long long limit, int* status) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) *status = mbar_wait_n(&bar, 0u, limit) ? 0 : ST_WATCHDOG;
}
}  // namespace

extern "C" int lbmgpu_watchdog_selftest(int device, long long limit, int* status) {
    if (!status || limit < 1 || limit > MBAR_WAIT_LIMIT)
        return fail(nullptr, LBMGPU_ERR_INVALID, "lbmgpu_watchdog_selftest: limit must be 1..2^22 tries");
    int* d = nullptr;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaMalloc(&d, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(d, 0, sizeof(int));
    if (e == cudaSuccess) {
        k_watchdog_selftest<<<1, 32>>>(limit, d);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(status, d, sizeof(int), cudaMemcpyDeviceToHost);
    if (d) cudaFree(d);
    if (e != cudaSuccess) return fail(nullptr, LBMGPU_ERR_CUDA, std::string("lbmgpu_watchdog_selftest: ") + cudaGetErrorString(e));
    if (*status & ST_WATCHDOG) return fail(nullptr, LBMGPU_ERR_WATCHDOG, "a bounded device wait gave up");
    return LBMGPU_OK;
}

// ============================================================================
//  lbmgpu_field_stats_static: the diagnostics of lbmgpu_diag over fields in the
//  caller's own device memory, with no allocation. Its reduction scratch is a
//  file-scope device array (one per device, shared by every caller), not a
//  handle buffer and not cudaMalloc.
// ============================================================================
namespace {

constexpr int STATS_BLOCK = 256;
constexpr int STATS_TILE = 2048;                                  // nodes per CTA (8 per thread)
constexpr long long STATS_MAX_TILES = LBMGPU_STATIC_STATS_MAX_NODES / STATS_TILE;
static_assert(LBMGPU_STATIC_STATS_MAX_NODES % STATS_TILE == 0, "tile count");

// [0, 4*MAX_TILES)  per-tile partials (count, sum rho, max |u|, sum ux)
// [4*MAX_TILES, +4) the result
// then one unsigned completion counter (must be 0 at launch)
struct StatsScratch {
    double part[4 * STATS_MAX_TILES];
    double result[4];
    unsigned done;
};
static __device__ __align__(256) unsigned char g_stats_scratch[sizeof(StatsScratch)];   // 512 KB + 40 B per device

// One CTA per tile of STATS_TILE nodes; the last CTA to finish sums the tile
// partials in tile order, so the result does not depend on which CTAs ran first.
__global__ void __launch_bounds__(STATS_BLOCK) k_field_stats_static(unsigned long long N, const uint8_t* flag,
                                                                   const double* rho, const double* ux,
                                                                   const double* uy, const double* uz,
                                                                   StatsScratch* sc) {
    __shared__ double red[STATS_BLOCK / 32][4];
    __shared__ bool last;
    double c = 0, m = 0, mx = 0, sx = 0;
    const unsigned long long base = (unsigned long long)blockIdx.x * STATS_TILE;
    for (int k = threadIdx.x; k < STATS_TILE; k += STATS_BLOCK) {
        const unsigned long long n = base + k;
        if (n >= N || (flag[n] & TYPE_MASK) != T_FLUID) continue;
        c += 1.0; m += rho[n]; sx += ux[n];
        mx = fmax(mx, sqrt(ux[n] * ux[n] + uy[n] * uy[n] + uz[n] * uz[n]));
    }
    for (int o = 16; o > 0; o >>= 1) {
        c += __shfl_down_sync(0xffffffffu, c, o);
        m += __shfl_down_sync(0xffffffffu, m, o);
        mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
        sx += __shfl_down_sync(0xffffffffu, sx, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { red[w][0] = c; red[w][1] = m; red[w][2] = mx; red[w][3] = sx; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0, d = 0, e = 0;
        for (int k = 0; k < STATS_BLOCK / 32; ++k) { a += red[k][0]; b += red[k][1]; d = fmax(d, red[k][2]); e += red[k][3]; }
        double* p = sc->part + 4 * (size_t)blockIdx.x;
        p[0] = a; p[1] = b; p[2] = d; p[3] = e;
        __threadfence();
        last = atomicAdd(&sc->done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // the last CTA: strided sums over the tiles, then the same tree as above
    c = m = mx = sx = 0;
    for (unsigned t = threadIdx.x; t < gridDim.x; t += STATS_BLOCK) {
        const volatile double* p = sc->part + 4 * (size_t)t;
        c += p[0]; m += p[1]; mx = fmax(mx, p[2]); sx += p[3];
    }
    for (int o = 16; o > 0; o >>= 1) {
        c += __shfl_down_sync(0xffffffffu, c, o);
        m += __shfl_down_sync(0xffffffffu, m, o);
        mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
        sx += __shfl_down_sync(0xffffffffu, sx, o);
    }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) { red[w][0] = c; red[w][1] = m; red[w][2] = mx; red[w][3] = sx; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0, d = 0, e = 0;
        for (int k = 0; k < STATS_BLOCK / 32; ++k) { a += red[k][0]; b += red[k][1]; d = fmax(d, red[k][2]); e += red[k][3]; }
        sc->result[0] = a; sc->result[1] = b; sc->result[2] = d; sc->result[3] = e;
    }
}

// Device address of g_stats_scratch, looked up once per device and context.
// The address belongs to the device's (primary) context: after the context is
// destroyed and recreated (cudaDeviceReset) the module is loaded again and the
// array may live elsewhere, so the cache entry is keyed by the context that
// was current at the lookup (the driver's cuCtxGetCurrent, reached through
// the runtime's cudaGetDriverEntryPoint, so no link against libcuda is needed).
constexpr int STATS_MAX_DEVICES = 64;
std::mutex g_stats_mu;
struct StatsAddr {
    void* ctx;
    StatsScratch* addr;
};
StatsAddr g_stats_addr[STATS_MAX_DEVICES] = {};

using CtxGetCurrentFn = int (*)(void**);   // CUresult cuCtxGetCurrent(CUcontext*)
void* current_context() {
    static CtxGetCurrentFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<CtxGetCurrentFn>(f);
    }();
    void* ctx = nullptr;
    if (!fn || fn(&ctx) != 0) return nullptr;
    return ctx;
}

cudaError_t stats_scratch(int dev, StatsScratch** out) {
    std::lock_guard<std::mutex> lk(g_stats_mu);
    StatsAddr& c = g_stats_addr[dev];
    void* ctx = current_context();
    if (!c.addr || !ctx || ctx != c.ctx) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_stats_scratch);   // binds the device's context
        if (e != cudaSuccess) return e;
        c.addr = static_cast<StatsScratch*>(p);
        c.ctx = current_context();
    }
    *out = c.addr;
    return cudaSuccess;
}

}  // namespace

extern "C" int lbmgpu_field_stats_static(const uint8_t* flag, const double* rho, const double* ux, const double* uy,
                                         const double* uz, long long n_nodes, void* cuda_stream,
                                         lbmgpu_diagnostics* out) {
    if (!out || !flag || !rho || !ux || !uy || !uz)
        return fail(nullptr, LBMGPU_ERR_INVALID, "lbmgpu_field_stats_static: null pointer argument");
    if (n_nodes < 1 || n_nodes > LBMGPU_STATIC_STATS_MAX_NODES)
        return fail(nullptr, LBMGPU_ERR_INVALID,
                    "lbmgpu_field_stats_static: n_nodes = " + std::to_string(n_nodes) + " is outside 1.." +
                        std::to_string(LBMGPU_STATIC_STATS_MAX_NODES) + ", the capacity of its static scratch");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess && (dev < 0 || dev >= STATS_MAX_DEVICES)) e = cudaErrorInvalidDevice;
    StatsScratch* sc = nullptr;
    if (e == cudaSuccess) e = stats_scratch(dev, &sc);
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(&sc->done, 0, sizeof(unsigned), st);
    const unsigned tiles = (unsigned)((n_nodes + STATS_TILE - 1) / STATS_TILE);
    if (e == cudaSuccess) {
        k_field_stats_static<<<tiles, STATS_BLOCK, 0, st>>>((unsigned long long)n_nodes, flag, rho, ux, uy, uz, sc);
        e = cudaGetLastError();
    }
    double r[4] = {0, 0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(r, sc->result, sizeof(r), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return fail(nullptr, LBMGPU_ERR_CUDA, std::string("lbmgpu_field_stats_static: ") + cudaGetErrorString(e));
    out->n_fluid = (long long)r[0];
    out->mean_density = r[0] > 0 ? r[1] / r[0] : 0.0;
    out->max_speed = r[2];
    out->sum_ux = r[3];
    out->wall_force[0] = out->wall_force[1] = out->wall_force[2] = 0.0;
    return LBMGPU_OK;
}
