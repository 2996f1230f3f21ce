// ============================================================================
//  lbmgpu.cu -- the C ABI (include/lbmgpu.h): handle, device memory, set-up
//  of the initial state, the CUDA-graph time loop and the host-facing
//  accessors.
// ============================================================================
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/lbmgpu.h"
#include "k_aux.cuh"
#include "k_squirmer.cuh"
#include "launch.h"

using namespace lbmgpu;

namespace {

constexpr double PI = 3.14159265358979323846;
constexpr int GRAPH_LONG = 64;   // steps in the long captured graph (even)
constexpr int DIAG_GRID = 296;

thread_local std::string g_create_error;

struct GraphSlot {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

}  // namespace

struct lbmgpu_handle {
    lbmgpu_params p{};
    Lattice L{};
    const Launchers* lz = nullptr;
    size_t esize = 8;
    int has_sq = 0;
    cudaStream_t own = nullptr, stream = nullptr, cap = nullptr;

    // device memory
    void* f = nullptr;
    uint8_t* flag = nullptr;
    double *rho = nullptr, *ux = nullptr, *uy = nullptr, *uz = nullptr;
    int* wall_nodes = nullptr;
    int n_wall = 0;
    int* links = nullptr;
    int link_cap = 0;
    double* link_part = nullptr;
    double* block_part = nullptr;
    unsigned nblocks = 0;
    double* block_part_b = nullptr;
    unsigned nblocks_b = 0;
    StreamGeom geom{};
    int* ordermap = nullptr;
    int* chg_node = nullptr;
    int* chg_key = nullptr;
    int* cand = nullptr;
    uint8_t* mark = nullptr;
    int chg_cap = 0;
    double* traj = nullptr;
    SqState* sq = nullptr;
    double* scratch = nullptr;   // N doubles
    double* small = nullptr;     // reduction partials / results (2*MASS_GRID + DIAG_GRID*4 + 16)

    // host mirrors
    long long t_main = 0;        // stream-kernel steps issued (AA parity)
    long long traj_read = 0;
    long long launches = 0;
    GraphSlot g_short, g_long;
    std::string err;
};

// ---------------------------------------------------------------------------
namespace {

int fail(lbmgpu_handle* h, int code, const std::string& msg) {
    if (h) h->err = msg; else g_create_error = msg;
    return code;
}

#define CUDA_TRY(h, call)                                                              \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess)                                                         \
            return fail(h, e_ == cudaErrorMemoryAllocation ? LBMGPU_ERR_NOMEM : LBMGPU_ERR_CUDA, \
                        std::string(#call) + ": " + cudaGetErrorString(e_));           \
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

StreamArgs stream_args(lbmgpu_handle* h, int fused) {
    StreamArgs a;
    a.f = h->f; a.flag = h->flag; a.rho = h->rho; a.ux = h->ux; a.uy = h->uy; a.uz = h->uz;
    a.link_part = h->link_part; a.block_part = h->block_part; a.block_part_b = h->block_part_b;
    a.wall_nodes = h->wall_nodes; a.n_wall = h->n_wall; a.links = h->links; a.sq = h->sq;
    a.fused = fused;
    return a;
}

SqArgs squirmer_args(lbmgpu_handle* h, int parity, int stages) {
    SqArgs a;
    a.f = h->f; a.flag = h->flag; a.rho = h->rho; a.ux = h->ux; a.uy = h->uy; a.uz = h->uz;
    a.links = h->links; a.link_cap = h->link_cap;
    a.link_part = h->link_part; a.block_part = h->block_part; a.nblocks = (int)h->nblocks;
    a.block_part_b = h->block_part_b; a.nblocks_b = (int)h->nblocks_b;
    a.ordermap = h->ordermap; a.chg_node = h->chg_node; a.chg_key = h->chg_key; a.cand = h->cand; a.mark = h->mark; a.chg_cap = h->chg_cap;
    a.traj = h->traj; a.sq = h->sq; a.parity = parity; a.stages = stages;
    return a;
}

// ---- small non-templated kernels -------------------------------------------
__global__ void k_fill_d(double* p, size_t n, double v) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) p[k] = v;
}
__global__ void k_fill_i(int* p, size_t n, int v) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) p[k] = v;
}

// wall force of a macro step: fixed-order sum of the stream kernel's block partials
__global__ void k_finalize(const double* block_part, unsigned nblocks, SqState* sq) {
    __shared__ double red[8][3];
    double a0 = 0, a1 = 0, a2 = 0;
    for (unsigned b = threadIdx.x; b < nblocks; b += blockDim.x) {
        a0 += block_part[(size_t)b * BLOCK_PART + 0];
        a1 += block_part[(size_t)b * BLOCK_PART + 1];
        a2 += block_part[(size_t)b * BLOCK_PART + 2];
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

// ---- host-side restatement of the initial state ----------------------------
struct HostInit {
    std::vector<uint8_t> flag;
    std::vector<int> links;
    std::vector<int> wall_nodes;
    SqState s{};
};

size_t hidx(const lbmgpu_params& p, int x, int y, int z) { return (size_t)x + (size_t)p.nx * ((size_t)y + (size_t)p.ny * z); }

// LBM::offsetFromSquirmer (lbm.cpp:100-104)
void h_offset(const lbmgpu_params& p, const SqState& s, double px, double py, double pz, double r[3]) {
    r[0] = px - s.X[0]; r[0] -= p.nx * std::round(r[0] / p.nx);
    r[1] = py - s.X[1]; if (!p.walls_y) r[1] -= p.ny * std::round(r[1] / p.ny);
    r[2] = pz - s.X[2]; if (!p.walls_z) r[2] -= p.nz * std::round(r[2] / p.nz);
}

void h_box(const lbmgpu_params& p, const SqState& s, int lo[3], int w[3]) {
    const double R = s.R;
    int x0 = (int)std::floor(s.X[0] - R) - 2, x1 = (int)std::ceil(s.X[0] + R) + 2;
    int y0 = (int)std::floor(s.X[1] - R) - 2, y1 = (int)std::ceil(s.X[1] + R) + 2;
    int z0 = (int)std::floor(s.X[2] - R) - 2, z1 = (int)std::ceil(s.X[2] + R) + 2;
    if (p.walls_y) { y0 = std::max(0, y0); y1 = std::min(p.ny - 1, y1); }
    lo[0] = x0; lo[1] = y0; lo[2] = z0;
    w[0] = x1 - x0 + 1; w[1] = y1 - y0 + 1; w[2] = z1 - z0 + 1;
}

void build_initial(const lbmgpu_params& p, const Lattice& L, HostInit& hi) {
    const size_t N = (size_t)p.nx * p.ny * p.nz;
    hi.flag.assign(N, T_FLUID);
    // WALL layers (lbm.cpp:72-78)
    for (int z = 0; z < p.nz; ++z)
        for (int y = 0; y < p.ny; ++y)
            for (int x = 0; x < p.nx; ++x) {
                const bool wall = (p.walls_y && (y == 0 || y == p.ny - 1)) || (p.walls_z && (z == 0 || z == p.nz - 1));
                hi.flag[hidx(p, x, y, z)] = wall ? T_WALL : T_FLUID;
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
                    if (hi.flag[n] == T_WALL) continue;
                    double r[3];
                    h_offset(p, s, x, y, z, r);
                    const bool inside = r[0] * r[0] + r[1] * r[1] + r[2] * r[2] < s.R * s.R;
                    hi.flag[n] = inside ? T_PARTICLE : T_FLUID;
                }
        const int nd[3] = {p.nx, p.ny, p.nz};
        for (int d = 0; d < 3; ++d) {
            const int ww = w[d] + 4;
            s.rb_w[d] = std::min(ww, nd[d]);
            s.rb_lo[d] = ww >= nd[d] ? 0 : (((lo[d] - 2) % nd[d]) + nd[d]) % nd[d];
        }
        s.rb_valid = 1;
    }
    // near-wall / near-particle bits, boundary-link list in node order, fluid count
    long long nf = 0;
    std::vector<uint8_t> base(hi.flag);
    for (int z = 0; z < p.nz; ++z)
        for (int y = 0; y < p.ny; ++y)
            for (int x = 0; x < p.nx; ++x) {
                const size_t n = hidx(p, x, y, z);
                if (base[n] != T_FLUID) continue;
                ++nf;
                bool nw = false, np = false;
                for (int i = 1; i < Q; ++i) {
                    const int xn = (x + CX(i) + p.nx) % p.nx, yn = (y + CY(i) + p.ny) % p.ny, zn = (z + CZ(i) + p.nz) % p.nz;
                    const uint8_t t = base[hidx(p, xn, yn, zn)];
                    nw |= t == T_WALL; np |= t == T_PARTICLE;
                }
                hi.flag[n] = T_FLUID | (nw ? NEAR_WALL : 0) | (np ? NEAR_PARTICLE : 0);
                if (np) hi.links.push_back((int)n);
            }
    // positions next to a wall (static; whatever their type becomes later)
    for (int z = 0; z < p.nz; ++z)
        for (int y = 0; y < p.ny; ++y)
            for (int x = 0; x < p.nx; ++x) {
                const size_t n = hidx(p, x, y, z);
                if (base[n] == T_WALL) continue;
                bool nw = false;
                for (int i = 1; i < Q; ++i) {
                    const int xn = (x + CX(i) + p.nx) % p.nx, yn = (y + CY(i) + p.ny) % p.ny, zn = (z + CZ(i) + p.nz) % p.nz;
                    nw |= base[hidx(p, xn, yn, zn)] == T_WALL;
                }
                if (nw) hi.wall_nodes.push_back((int)n);
            }
    s.n_fluid = nf;
    s.n_links = (int)hi.links.size();
    (void)L;
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
    return LBMGPU_OK;
}

void free_all(lbmgpu_handle* h) {
    for (GraphSlot* g : {&h->g_short, &h->g_long}) {
        if (g->exec) cudaGraphExecDestroy(g->exec);
        if (g->graph) cudaGraphDestroy(g->graph);
        g->exec = nullptr; g->graph = nullptr;
    }
    void* ptrs[] = {h->f, h->flag, h->rho, h->ux, h->uy, h->uz, h->wall_nodes, h->links, h->link_part, h->block_part, h->block_part_b,
                    h->ordermap, h->chg_node, h->chg_key, h->cand, h->mark, h->traj, h->sq, h->scratch, h->small};
    for (void* q : ptrs) if (q) cudaFree(q);
    if (h->own) cudaStreamDestroy(h->own);
    if (h->cap) cudaStreamDestroy(h->cap);
}

// ---- one time step ---------------------------------------------------------
// fused = 1: the time-loop body of main.cpp:60-64; fused = 0: LBM::step only.
void issue_step(lbmgpu_handle* h, cudaStream_t st, int par, bool macro, int fused) {
    const StreamArgs a = stream_args(h, fused);
    h->lz->stream(par, h->has_sq != 0, macro, h->L, a, h->geom, st);
    int k = h->geom.bgrid ? 2 : 1;
    if (macro) { k_finalize<<<1, 256, 0, st>>>(h->block_part_b, h->nblocks_b, h->sq); ++k; }
    if (h->has_sq && fused) {
        h->lz->squirmer(h->L, squirmer_args(h, par ^ 1, STAGE_FORCE | STAGE_BODY | STAGE_REMAP | STAGE_LOOP), st);
        ++k;
    }
    h->launches += k;
}

int ensure_graph(lbmgpu_handle* h, GraphSlot& g, int steps) {
    if (g.exec) return LBMGPU_OK;
    CUDA_TRY(h, cudaStreamBeginCapture(h->cap, cudaStreamCaptureModeThreadLocal));
    const long long saved = h->launches;
    for (int k = 0; k < steps; ++k) issue_step(h, h->cap, k & 1, false, 1);
    h->launches = saved;
    CUDA_TRY(h, cudaStreamEndCapture(h->cap, &g.graph));
    CUDA_TRY(h, cudaGraphInstantiate(&g.exec, g.graph, 0));
    return LBMGPU_OK;
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

int lbmgpu_create(const lbmgpu_params* p, lbmgpu_handle** out) {
    if (!out) return fail(nullptr, LBMGPU_ERR_INVALID, "null output pointer");
    *out = nullptr;
    std::string m;
    if (validate_impl(p, m) != LBMGPU_OK) return fail(nullptr, LBMGPU_ERR_INVALID, m);
    lbmgpu_handle* h = new lbmgpu_handle();
    h->p = *p;
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
    CTRY(cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking));
    CTRY(cudaStreamCreateWithFlags(&h->cap, cudaStreamNonBlocking));
    h->stream = h->own;

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
    for (int d = 0; d < 3; ++d) { L.Ff[d] = (float)L.F[d]; L.uFh[d] = 0.0f; }
    for (int i = 0; i < Q; ++i) {
        const double cF = CX(i) * L.F[0] + CY(i) * L.F[1] + CZ(i) * L.F[2];
        L.cF[i] = (float)cF;
        L.cm[i] = (float)(L.gM * 3.0 * WD(i) * cF);
    }
    const size_t N = L.N;

    HostInit hi;
    build_initial(*p, L, hi);
    h->n_wall = (int)hi.wall_nodes.size();
    const int box = h->has_sq ? 2 * (int)std::ceil(p->radius) + 8 : 1;
    const long long boxvol = (long long)box * box * box;
    h->link_cap = (int)std::max<long long>(boxvol, (long long)hi.links.size() + 1);
    h->chg_cap = (int)boxvol;
    {
        const int tx = p->nx >= 256 ? 256 : ((p->nx + 31) / 32) * 32;
        h->geom.block = dim3(tx, 1, 1);
        h->geom.grid = dim3((p->nx + tx - 1) / tx, p->ny, p->nz);
        h->nblocks = h->geom.grid.x * h->geom.grid.y * h->geom.grid.z;
        const long long nb = (long long)h->n_wall + (h->has_sq ? h->link_cap : 0);
        h->geom.bgrid = (unsigned)((nb + BOUNDARY_BLOCK - 1) / BOUNDARY_BLOCK);
        h->nblocks_b = std::max(1u, h->geom.bgrid);
    }

    CTRY(cudaMalloc(&h->f, (size_t)Q * N * h->esize));
    CTRY(cudaMalloc(&h->flag, N));
    CTRY(cudaMalloc(&h->rho, N * sizeof(double)));
    CTRY(cudaMalloc(&h->ux, N * sizeof(double)));
    CTRY(cudaMalloc(&h->uy, N * sizeof(double)));
    CTRY(cudaMalloc(&h->uz, N * sizeof(double)));
    CTRY(cudaMalloc(&h->scratch, N * sizeof(double)));
    CTRY(cudaMalloc(&h->block_part, (size_t)h->nblocks * BLOCK_PART * sizeof(double)));
    CTRY(cudaMalloc(&h->block_part_b, (size_t)h->nblocks_b * BLOCK_PART * sizeof(double)));
    CTRY(cudaMalloc(&h->wall_nodes, std::max<size_t>(1, hi.wall_nodes.size()) * sizeof(int)));
    CTRY(cudaMalloc(&h->sq, sizeof(SqState)));
    CTRY(cudaMalloc(&h->small, (2 * MASS_GRID + 4 * DIAG_GRID + 16) * sizeof(double)));
    CTRY(cudaMalloc(&h->links, (size_t)h->link_cap * sizeof(int)));
    CTRY(cudaMalloc(&h->link_part, (size_t)h->link_cap * LINK_PART * sizeof(double)));
    if (h->has_sq) {
        CTRY(cudaMalloc(&h->ordermap, N * sizeof(int)));
        CTRY(cudaMalloc(&h->chg_node, (size_t)h->chg_cap * sizeof(int)));
        CTRY(cudaMalloc(&h->chg_key, (size_t)h->chg_cap * sizeof(int)));
        CTRY(cudaMalloc(&h->mark, (size_t)h->chg_cap));
        CTRY(cudaMalloc(&h->cand, (size_t)h->chg_cap * sizeof(int)));
        CTRY(cudaMalloc(&h->traj, (size_t)TRAJ_RING * TRAJ_COLS * sizeof(double)));
    }
    cudaStream_t st = h->stream;
    h->lz->fill_rest(L, h->f, st);
    k_fill_d<<<592, 256, 0, st>>>(h->rho, N, 1.0);
    k_fill_d<<<592, 256, 0, st>>>(h->ux, N, 0.0);
    k_fill_d<<<592, 256, 0, st>>>(h->uy, N, 0.0);
    k_fill_d<<<592, 256, 0, st>>>(h->uz, N, 0.0);
    CTRY(cudaMemsetAsync(h->block_part, 0, (size_t)h->nblocks * BLOCK_PART * sizeof(double), st));
    CTRY(cudaMemsetAsync(h->block_part_b, 0, (size_t)h->nblocks_b * BLOCK_PART * sizeof(double), st));
    if (!hi.wall_nodes.empty())
        CTRY(cudaMemcpyAsync(h->wall_nodes, hi.wall_nodes.data(), hi.wall_nodes.size() * sizeof(int),
                             cudaMemcpyHostToDevice, st));
    CTRY(cudaMemsetAsync(h->link_part, 0, (size_t)h->link_cap * LINK_PART * sizeof(double), st));
    CTRY(cudaMemcpyAsync(h->flag, hi.flag.data(), N, cudaMemcpyHostToDevice, st));
    if (h->has_sq) {
        k_fill_i<<<592, 256, 0, st>>>(h->ordermap, N, -1);
        if (!hi.links.empty())
            CTRY(cudaMemcpyAsync(h->links, hi.links.data(), hi.links.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        CTRY(cudaMemsetAsync(h->traj, 0, (size_t)TRAJ_RING * TRAJ_COLS * sizeof(double), st));
    }
    CTRY(cudaStreamSynchronize(st));  // host vectors go out of scope
    CTRY(cudaMemcpyAsync(h->sq, &hi.s, sizeof(SqState), cudaMemcpyHostToDevice, st));
    CTRY(cudaStreamSynchronize(st));
    CTRY(cudaGetLastError());
    h->launches += 5 + (h->has_sq ? 1 : 0);
#undef CTRY
    *out = h;
    return LBMGPU_OK;
}

int lbmgpu_destroy(lbmgpu_handle* h) {
    if (!h) return LBMGPU_OK;
    cudaSetDevice(h->p.device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_all(h);
    delete h;
    return LBMGPU_OK;
}

int lbmgpu_run(lbmgpu_handle* h, int nsteps) {
    if (!h) return LBMGPU_ERR_INVALID;
    if (nsteps < 0) return fail(h, LBMGPU_ERR_INVALID, "nsteps must be >= 0");
    if (nsteps == 0) return LBMGPU_OK;
    CUDA_TRY(h, cudaSetDevice(h->p.device));
    const int per_step = (h->geom.bgrid ? 2 : 1) + (h->has_sq ? 1 : 0);
    int rem = nsteps;
    while (rem > 1) {
        if (h->t_main & 1) {
            issue_step(h, h->stream, 1, false, 1);
            ++h->t_main; --rem;
        } else if (rem - 1 >= GRAPH_LONG) {
            int rc = ensure_graph(h, h->g_long, GRAPH_LONG);
            if (rc) return rc;
            CUDA_TRY(h, cudaGraphLaunch(h->g_long.exec, h->stream));
            h->launches += (long long)GRAPH_LONG * per_step;
            h->t_main += GRAPH_LONG; rem -= GRAPH_LONG;
        } else if (rem - 1 >= 2) {
            int rc = ensure_graph(h, h->g_short, 2);
            if (rc) return rc;
            CUDA_TRY(h, cudaGraphLaunch(h->g_short.exec, h->stream));
            h->launches += 2 * per_step;
            h->t_main += 2; rem -= 2;
        } else {
            issue_step(h, h->stream, (int)(h->t_main & 1), false, 1);
            ++h->t_main; --rem;
        }
    }
    issue_step(h, h->stream, (int)(h->t_main & 1), true, 1);  // last step: macro fields + wall force
    ++h->t_main;
    return check_status(h);
}

int lbmgpu_step(lbmgpu_handle* h) {
    if (!h) return LBMGPU_ERR_INVALID;
    CUDA_TRY(h, cudaSetDevice(h->p.device));
    issue_step(h, h->stream, (int)(h->t_main & 1), true, 0);
    if (h->has_sq) {
        // the tail of LBM::step: Fh, Th of this step (lbm.cpp:220-223)
        h->lz->squirmer(h->L, squirmer_args(h, (int)((h->t_main + 1) & 1), STAGE_FORCE), h->stream);
        k_clear_pending<<<1, 32, 0, h->stream>>>(h->sq);
        h->launches += 2;
    }
    ++h->t_main;
    return check_status(h);
}

int lbmgpu_advance_squirmer(lbmgpu_handle* h) {
    if (!h) return LBMGPU_ERR_INVALID;
    if (!h->has_sq) return LBMGPU_OK;  // LBM::advanceSquirmer returns without a squirmer (lbm.cpp:258)
    CUDA_TRY(h, cudaSetDevice(h->p.device));
    h->lz->squirmer(h->L, squirmer_args(h, (int)(h->t_main & 1), STAGE_BODY | STAGE_REMAP), h->stream);
    ++h->launches;
    return check_status(h);
}

int lbmgpu_correct_mass(lbmgpu_handle* h) {
    if (!h) return LBMGPU_ERR_INVALID;
    CUDA_TRY(h, cudaSetDevice(h->p.device));
    // a correction still pending from lbmgpu_run is applied first
    double* part = h->small;
    double* dflag = h->small + 2 * MASS_GRID;
    h->lz->correct_mass(h->L, h->f, h->flag, (int)(h->t_main & 1), h->sq, part, dflag, h->stream);
    h->launches += 3;
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
    if (!h->has_sq) return fail(h, LBMGPU_ERR_INVALID, "no squirmer in this lattice");
    CUDA_TRY(h, cudaSetDevice(h->p.device));
    SqState s;
    CUDA_TRY(h, cudaMemcpyAsync(&s, h->sq, sizeof(s), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    for (int d = 0; d < 3; ++d) { s.X[d] = X[d]; s.e[d] = e[d]; s.U[d] = U[d]; s.W[d] = W[d]; }
    int lo[3], w[3];
    h_box(h->p, s, lo, w);
    const int nd[3] = {h->p.nx, h->p.ny, h->p.nz};
    for (int d = 0; d < 3; ++d) {
        const int ww = w[d] + 4;
        s.rb_w[d] = std::min(ww, nd[d]);
        s.rb_lo[d] = ww >= nd[d] ? 0 : (((lo[d] - 2) % nd[d]) + nd[d]) % nd[d];
    }
    CUDA_TRY(h, cudaMemcpyAsync(h->sq, &s, sizeof(s), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return LBMGPU_OK;
}

int lbmgpu_fields(lbmgpu_handle* h, uint8_t* flag, double* rho, double* u3) {
    if (!h) return LBMGPU_ERR_INVALID;
    CUDA_TRY(h, cudaSetDevice(h->p.device));
    const size_t N = h->L.N;
    cudaStream_t st = h->stream;
    if (flag) {
        CUDA_TRY(h, cudaMemcpyAsync(flag, h->flag, N, cudaMemcpyDeviceToHost, st));
    }
    if (rho) CUDA_TRY(h, cudaMemcpyAsync(rho, h->rho, N * sizeof(double), cudaMemcpyDeviceToHost, st));
    std::vector<double> tmp;
    if (u3) {
        tmp.resize(3 * N);
        CUDA_TRY(h, cudaMemcpyAsync(tmp.data(), h->ux, N * sizeof(double), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(h, cudaMemcpyAsync(tmp.data() + N, h->uy, N * sizeof(double), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(h, cudaMemcpyAsync(tmp.data() + 2 * N, h->uz, N * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    CUDA_TRY(h, cudaStreamSynchronize(st));
    if (flag) for (size_t n = 0; n < N; ++n) flag[n] &= TYPE_MASK;
    if (u3)
        for (size_t n = 0; n < N; ++n) { u3[3 * n] = tmp[n]; u3[3 * n + 1] = tmp[N + n]; u3[3 * n + 2] = tmp[2 * N + n]; }
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
    std::vector<double> ring((size_t)TRAJ_RING * TRAJ_COLS);
    if (take > 0) {
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
    return check_status(h);
}

int lbmgpu_set_stream(lbmgpu_handle* h, void* cuda_stream) {
    if (!h) return LBMGPU_ERR_INVALID;
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    h->stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : h->own;
    return LBMGPU_OK;
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
