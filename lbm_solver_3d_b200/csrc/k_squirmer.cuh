// ============================================================================
//  k_squirmer.cuh -- the per-step squirmer update on the device, one CTA:
//
//   stage FORCE: sum the boundary-link partials of the step into Fh, Th
//                (fixed order, deterministic) -- the tail of LBM::step
//                (lbm.cpp:219-223).
//   stage BODY : LBM::applyWallPotential, Squirmer::integrate and
//                LBM::enforceMinimumGap (lbm.cpp:231-253,
//                squirmer.cpp:52-77), FP64.
//   stage REMAP: LBM::updateParticleFlags(false) (lbm.cpp:271-320) with the
//                reference's order-dependent semantics, then a rebuild of the
//                boundary-link list (fluid nodes next to the sphere, in
//                ascending node order) and of the near-particle flag bits.
//   stage LOOP : time-loop bookkeeping of src/main.cpp:60-64: schedule the
//                mass correction of correction steps (applied by the next
//                stream kernel on load), record the trajectory row, and set
//                the region whose densities the next step must store.
//
//  Remap ordering. The reference walks the sphere's bounding box in z, y, x
//  order and updates flags, f and rho in place, so an uncovered node sees
//  the new state of nodes visited before it and the old state of the rest.
//  Here the changed nodes are found in parallel and compacted in box order
//  (their order key is the box index of their first visit); each changed
//  node's neighbour data (old flag, old rho, change order) is gathered in
//  parallel into shared memory; one thread then replays the changes in box
//  order, resolving neighbours that changed earlier from shared memory; the
//  writes go out in parallel. Batches of BATCH changed nodes keep the shared
//  memory bounded; a batch sees the global writes of the batches before it.
// ============================================================================
#pragma once
#include <cub/block/block_scan.cuh>

#include "k_logical.cuh"
#include "k_stream.cuh"

namespace lbmgpu {

constexpr int SQ_THREADS = 512;
constexpr int SQ_BATCH = 256;
constexpr int SQ_SORT_CAP = 2048;
constexpr int SQ_GROUP = 4;         // remap candidates tested per thread with their loads in flight together   // changes ordered in shared memory (3 ints each)
constexpr int STAGE_BODY = 1, STAGE_REMAP = 2, STAGE_LOOP = 4, STAGE_FORCE = 8;

struct SqArgs {
    void* f;
    uint8_t* flag;
    double* rho; double* ux; double* uy; double* uz;
    int* links;
    int* linkslot;            // node -> row of its boundary-link entry
    int link_cap;
    const double* link_part;
    const double* block_part;     // bulk kernel partials (mass in column 3)
    int nblocks;
    const double* block_part_b;   // zone kernel partials
    int nblocks_b;
    const double* block_part_w;   // wall-row partials of an ensemble member (else unused)
    int nblocks_w;
    int* ordermap;            // N entries, -1 when idle
    int* chg_node;            // changed-node list (capacity chg_cap)
    int* chg_key;
    int* cand;                // candidate nodes of the remap / link scans (chg_cap)
    uint8_t* mark;            // chg_cap bytes: one verdict per candidate
    int chg_cap;
    int* shell;               // cached remap candidates (chg_cap entries)
    ShellCache* shell_hdr;
    double* traj;             // TRAJ_RING x TRAJ_COLS
    SqState* sq;
    int parity;               // parity of the state being remapped
    int stages;
    int corr_step;            // this step is a mass-correction step (time-loop mode)
    int zslot_a, zslot_b;     // zone slots to (re)write from the new position, -1: none
};

struct ChgSh {
    double r[3];
    double p[3];
    double mass;
    double rr, ub[3];
    double nbrho[18];
    int nbord[18];
    int node, kind;           // kind: 1 covered, 2 uncovered
    uint8_t nbfl[18];
};

// softWallForce (squirmer.cpp:73-77)
__device__ __forceinline__ double soft_wall_force(double h, double eps, double FS, double hc) {
    if (h >= hc) return 0.0;
    const double s = 1.0 - fmax(h, 0.0) / hc;
    return eps * FS * s * s;
}

// Deterministic block sum of ncols (<= 8) columns over rows of a strided array.
template <int NC>
__device__ void block_sum_rows(const double* base, int rows, int stride, int col0, double* out_sh) {
    __shared__ double red[SQ_THREADS / 32][8];
    double acc[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) acc[c] = 0.0;
    for (int k = threadIdx.x; k < rows; k += SQ_THREADS) {
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[c] += base[(size_t)k * stride + col0 + c];
    }
#pragma unroll
    for (int c = 0; c < NC; ++c)
        for (int o = 16; o > 0; o >>= 1) acc[c] += __shfl_down_sync(0xffffffffu, acc[c], o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int c = 0; c < NC; ++c) red[wid][c] = acc[c];
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            double s = 0.0;
            for (int w = 0; w < SQ_THREADS / 32; ++w) s += red[w][c];
            out_sh[c] = s;
        }
    }
    __syncthreads();
}

// Coordinates along one axis of a box, visited in ascending wrapped order.
struct AxisRange {
    int start, width, n, wrap;
    __device__ void init(int lo_unwrapped, int w, int nd) {
        if (w >= nd) { start = 0; width = nd; wrap = 0; n = nd; return; }
        start = ((lo_unwrapped % nd) + nd) % nd;
        width = w; n = nd;
        wrap = start + w > nd ? start + w - nd : 0;
    }
    __device__ int at(int b) const { return b < wrap ? b : start + (b - wrap); }
};

static_assert(3 * SQ_SORT_CAP * sizeof(int) <= SQ_BATCH * sizeof(ChgSh), "the change sort fits the batch stage");

template <class S>
__device__ void squirmer_update(const Lattice& L, const SqArgs& a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ChgSh* ch = reinterpret_cast<ChgSh*>(smem_raw);
    __shared__ SqState s;
    __shared__ double sums[8];
    __shared__ int sh_total, sh_box[6], sh_rebuild, sh_ncand;
    __shared__ double sh_mass_delta;
    __shared__ long long sh_dfluid;
    typedef cub::BlockScan<int, SQ_THREADS> Scan;
    __shared__ typename Scan::TempStorage scan_tmp;

    const int tid = threadIdx.x;
    {   // the state, one word per thread
        constexpr int NS = (int)(sizeof(SqState) / 4);
        static_assert(sizeof(SqState) % 4 == 0 && NS <= SQ_THREADS, "one word per thread");
        if (tid < NS) reinterpret_cast<uint32_t*>(&s)[tid] = reinterpret_cast<const uint32_t*>(a.sq)[tid];
    }
    if (tid == 0) {
        sh_mass_delta = 0.0;
        sh_dfluid = 0;
    }
    __syncthreads();
    if (s.status & (ST_NAN | ST_REMAP_RANGE | ST_LINK_OVERFLOW)) return;  // invalid already; the host reports it

    const long long t_now = s.t + 1;
    const bool loop = (a.stages & STAGE_LOOP) != 0;
    const bool corr_step = loop && a.corr_step;

    // ---------------- stage BODY ----------------
    if (a.stages & STAGE_FORCE) {
        block_sum_rows<6>(a.link_part, s.n_links, LINK_PART, 0, sums);
        if (tid == 0)
            for (int d = 0; d < 3; ++d) { s.Fh[d] = sums[d]; s.Th[d] = sums[3 + d]; }
        __syncthreads();
    }
    if (a.stages & STAGE_BODY) {
        if (tid == 0) {
            // LBM::applyWallPotential (lbm.cpp:231-241)
            s.Fw[0] = s.Fw[1] = s.Fw[2] = 0.0;
            if (L.walls_y) {
                s.Fw[1] += soft_wall_force(s.X[1] - s.R - 0.5, s.eps, s.FS, s.hc);
                s.Fw[1] -= soft_wall_force((L.ny - 1.5) - s.X[1] - s.R, s.eps, s.FS, s.hc);
            }
            if (L.walls_z) {
                s.Fw[2] += soft_wall_force(s.X[2] - s.R - 0.5, s.eps, s.FS, s.hc);
                s.Fw[2] -= soft_wall_force((L.nz - 1.5) - s.X[2] - s.R, s.eps, s.FS, s.hc);
            }
            // Squirmer::integrate (squirmer.cpp:52-68)
            for (int d = 0; d < 3; ++d) {
                s.U[d] += (s.Fh[d] + s.Fc[d] + s.Fw[d]) / s.M;
                s.W[d] += (s.Th[d] + s.Tc[d]) / s.I;
                s.Fc[d] = s.Tc[d] = 0.0;
            }
            if (s.planar) { s.U[2] = 0.0; s.W[0] = 0.0; s.W[1] = 0.0; }
            const double Xold[3] = {s.X[0], s.X[1], s.X[2]};
            for (int d = 0; d < 3; ++d) s.X[d] += s.U[d];
            const double we0 = s.W[1] * s.e[2] - s.W[2] * s.e[1];
            const double we1 = s.W[2] * s.e[0] - s.W[0] * s.e[2];
            const double we2 = s.W[0] * s.e[1] - s.W[1] * s.e[0];
            s.e[0] += we0; s.e[1] += we1; s.e[2] += we2;
            if (s.planar) s.e[2] = 0.0;
            const double nrm = sqrt(s.e[0] * s.e[0] + s.e[1] * s.e[1] + s.e[2] * s.e[2]);
            for (int d = 0; d < 3; ++d) s.e[d] /= nrm;
            // LBM::enforceMinimumGap (lbm.cpp:245-253)
            for (int d = 1; d <= 2; ++d) {
                if ((d == 1 && !L.walls_y) || (d == 2 && !L.walls_z)) continue;
                const int Nd = d == 1 ? L.ny : L.nz;
                const double lo = 0.5 + s.R + s.hmin, hi = (Nd - 1.5) - s.R - s.hmin;
                if (s.X[d] < lo) { s.X[d] = lo; if (s.U[d] < 0) s.U[d] = 0; ++s.contacts; }
                if (s.X[d] > hi) { s.X[d] = hi; if (s.U[d] > 0) s.U[d] = 0; ++s.contacts; }
            }
            s.t = t_now;
            bool ok = true;
            for (int d = 0; d < 3; ++d)
                ok = ok && isfinite(s.X[d]) && isfinite(s.U[d]) && isfinite(s.W[d]) && isfinite(s.e[d]) &&
                     isfinite(s.Fh[d]) && isfinite(s.Th[d]);
            if (!ok) s.status |= ST_NAN;
            // The densities the refill reads were stored for the box of the
            // previous position widened by 2; that covers this step's box
            // widened by 1 only if the centre moved less than one cell.
            else if (fabs(s.X[0] - Xold[0]) >= 1.0 || fabs(s.X[1] - Xold[1]) >= 1.0 || fabs(s.X[2] - Xold[2]) >= 1.0)
                s.status |= ST_REMAP_RANGE;
        }
        __syncthreads();
    }
    if (s.status & (ST_NAN | ST_REMAP_RANGE)) {
        if (tid == 0) *a.sq = s;
        return;
    }

    // the sphere's bounding box (lbm.cpp:272-276)
    if (tid == 0) {
        const double R = s.R;
        int x0 = (int)floor(s.X[0] - R) - 2, x1 = (int)ceil(s.X[0] + R) + 2;
        int y0 = (int)floor(s.X[1] - R) - 2, y1 = (int)ceil(s.X[1] + R) + 2;
        int z0 = (int)floor(s.X[2] - R) - 2, z1 = (int)ceil(s.X[2] + R) + 2;
        if (L.walls_y) { y0 = max(0, y0); y1 = min(L.ny - 1, y1); }
        sh_box[0] = x0; sh_box[1] = y0; sh_box[2] = z0;
        sh_box[3] = x1 - x0 + 1; sh_box[4] = y1 - y0 + 1; sh_box[5] = z1 - z0 + 1;
    }
    __syncthreads();
    const int bx0 = sh_box[0], by0 = sh_box[1], bz0 = sh_box[2];
    const int bw = sh_box[3], bh = sh_box[4], bd = sh_box[5];
    const int V = bw * bh * bd;
    const double R2 = s.R * s.R;

    // ---------------- stage REMAP ----------------
    if (a.stages & STAGE_REMAP) {
        // Wrapped centre for the cheap distance filters (X[0] is kept unwrapped).
        const double cxw = s.X[0] - L.nx * floor(s.X[0] / L.nx);
        const double cyw = L.walls_y ? s.X[1] : s.X[1] - L.ny * floor(s.X[1] / L.ny);
        const double czw = L.walls_z ? s.X[2] : s.X[2] - L.nz * floor(s.X[2] / L.nz);
        auto approx_r2 = [&](int x, int y, int z) -> double {
            double dx = x - cxw, dy = y - cyw, dz = z - czw;
            if (dx > 0.5 * L.nx) dx -= L.nx; else if (dx < -0.5 * L.nx) dx += L.nx;
            if (!L.walls_y) { if (dy > 0.5 * L.ny) dy -= L.ny; else if (dy < -0.5 * L.ny) dy += L.ny; }
            if (!L.walls_z) { if (dz > 0.5 * L.nz) dz -= L.nz; else if (dz < -0.5 * L.nz) dz += L.nz; }
            return dx * dx + dy * dy + dz * dz;
        };
        // Only nodes within one cell of the sphere's surface can change: the
        // centre moved less than a cell since the last remap (checked in stage
        // BODY), so nodes deeper than that were and stay PARTICLE and nodes
        // farther out were and stay FLUID. The candidates are the nodes within
        // R +- 1.05 of the centre (0.05 covers the cheap distance against the
        // reference's exact offset, which makes the decision). The shell list
        // widens that by SHELL_SLACK around a reference centre, so it holds
        // every candidate while the centre stays within SHELL_SLACK of it
        // (triangle inequality), and the box walk that builds it runs only
        // when the centre leaves that ball.

        // (1) candidates: the cached shell, rebuilt in box order (z, y, x of
        // the first visit) when the centre has left the slack around the
        // reference centre of the list. A cached list that yields more than
        // SQ_SORT_CAP changes is rebuilt at once (second pass).
        if (tid == 0) {
            const ShellCache hc = *a.shell_hdr;
            const double d0 = s.X[0] - hc.X[0], d1 = s.X[1] - hc.X[1], d2 = s.X[2] - hc.X[2];
            sh_rebuild = !(hc.valid && d0 * d0 + d1 * d1 + d2 * d2 < SHELL_SLACK * SHELL_SLACK);
            sh_ncand = hc.n;
        }
        __syncthreads();
        for (int pass = 0; pass < 2; ++pass) {
            if (pass == 1) {
                if (!(!sh_rebuild && sh_total > SQ_SORT_CAP)) break;   // uniform
                __syncthreads();
                if (tid == 0) sh_rebuild = 1;
                __syncthreads();
            }
            const int chunk = (V + SQ_THREADS - 1) / SQ_THREADS;
            const int k0 = min(V, tid * chunk), k1 = min(V, k0 + chunk);
            auto box_walk = [&](auto&& visit) {
                if (k0 >= k1) return;
                int bx = k0 % bw, by = (k0 / bw) % bh, bz = k0 / (bw * bh);
                int x = (((bx0 + bx) % L.nx) + L.nx) % L.nx;
                int y = (((by0 + by) % L.ny) + L.ny) % L.ny;
                int z = (((bz0 + bz) % L.nz) + L.nz) % L.nz;
                for (int k = k0; k < k1; ++k) {
                    // a box wider than the lattice revisits nodes; the first visit counts
                    if (bx < L.nx && by < L.ny && bz < L.nz) visit(k, x, y, z);
                    if (++bx == bw) {
                        bx = 0; x = (((bx0) % L.nx) + L.nx) % L.nx;
                        if (++by == bh) { by = 0; y = (((by0) % L.ny) + L.ny) % L.ny; ++bz; if (++z == L.nz) z = 0; }
                        else if (++y == L.ny) y = 0;
                    } else if (++x == L.nx) x = 0;
                }
            };
            if (sh_rebuild) {   // uniform
                const double Sin = fmax(s.R - 1.05 - SHELL_SLACK, 0.0), Sout = s.R + 1.05 + SHELL_SLACK;
                const double Sin2 = Sin * Sin, Sout2 = Sout * Sout;
                int cnt = 0;
                box_walk([&](int, int x, int y, int z) {
                    const double r2 = approx_r2(x, y, z);
                    cnt += (r2 >= Sin2 && r2 < Sout2);
                });
                int off = 0;
                Scan(scan_tmp).ExclusiveSum(cnt, off, sh_total);
                __syncthreads();
                box_walk([&](int, int x, int y, int z) {
                    const double r2 = approx_r2(x, y, z);
                    if (r2 >= Sin2 && r2 < Sout2) {
                        if (off < a.chg_cap) a.shell[off] = x + L.nx * (y + L.ny * z);
                        ++off;
                    }
                });
                if (tid == 0) {
                    sh_ncand = min(sh_total, a.chg_cap);
                    ShellCache hc;
                    for (int d = 0; d < 3; ++d) hc.X[d] = s.X[d];
                    hc.n = sh_ncand;
                    hc.valid = 1;
                    *a.shell_hdr = hc;
                }
                __syncthreads();
            }
            const int ncand = sh_ncand;
            // (2) exact test of each candidate (flag load + the reference's
            // offset), SQ_GROUP candidates per thread at a time: their node
            // indices and flags are all loaded before the first test
            for (int c0 = tid; c0 < ncand; c0 += SQ_GROUP * SQ_THREADS) {
                unsigned nn[SQ_GROUP];
                uint8_t ty[SQ_GROUP];
#pragma unroll
                for (int g = 0; g < SQ_GROUP; ++g) {
                    const int c = c0 + g * SQ_THREADS;
                    nn[g] = c < ncand ? (unsigned)a.shell[c] : 0u;
                }
#pragma unroll
                for (int g = 0; g < SQ_GROUP; ++g)
                    ty[g] = c0 + g * SQ_THREADS < ncand ? (uint8_t)(a.flag[nn[g]] & TYPE_MASK) : (uint8_t)T_WALL;
#pragma unroll
                for (int g = 0; g < SQ_GROUP; ++g) {
                    const int c = c0 + g * SQ_THREADS;
                    if (c >= ncand) break;
                    const unsigned n = nn[g];
                    uint8_t mk = 0;
                    if (ty[g] != T_WALL) {
                        const int x = (int)(n % (unsigned)L.nx), y = (int)((n / (unsigned)L.nx) % (unsigned)L.ny),
                                  z = (int)(n / L.nxy);
                        double r[3];
                        offset_from_squirmer(L, &s, x, y, z, r);
                        const bool inside = r[0] * r[0] + r[1] * r[1] + r[2] * r[2] < R2;
                        if (inside != (ty[g] == T_PARTICLE)) mk = inside ? 1 : 2;
                    }
                    a.mark[c] = mk;
                }
            }
            __syncthreads();
            // (3) changed nodes in list order
            {
                const int ch2 = (ncand + SQ_THREADS - 1) / SQ_THREADS;
                const int c0 = min(ncand, tid * ch2), c1 = min(ncand, c0 + ch2);
                int cnt = 0;
                for (int c = c0; c < c1; ++c) cnt += a.mark[c] != 0;
                int off = 0;
                Scan(scan_tmp).ExclusiveSum(cnt, off, sh_total);
                __syncthreads();
                for (int c = c0; c < c1; ++c) {
                    const uint8_t mk = a.mark[c];
                    if (!mk) continue;
                    a.chg_node[off] = a.shell[c];
                    a.chg_key[off] = mk;
                    ++off;
                }
            }
            __syncthreads();
        }
        // A list cached under an earlier box is in that box's order: put the
        // changes in the order of their first visit in this box (rank sort on
        // the visit index; distinct nodes have distinct indices).
        if (!sh_rebuild && sh_total > 1) {   // uniform
            const int nchg = sh_total;
            int* keys = reinterpret_cast<int*>(smem_raw);
            int* nodes = keys + SQ_SORT_CAP;
            int* kinds = nodes + SQ_SORT_CAP;
            for (int e = tid; e < nchg; e += SQ_THREADS) {
                const unsigned n = (unsigned)a.chg_node[e];
                const int x = (int)(n % (unsigned)L.nx), y = (int)((n / (unsigned)L.nx) % (unsigned)L.ny),
                          z = (int)(n / L.nxy);
                const int kx = ((x - bx0) % L.nx + L.nx) % L.nx;
                const int ky = ((y - by0) % L.ny + L.ny) % L.ny;
                const int kz = ((z - bz0) % L.nz + L.nz) % L.nz;
                keys[e] = (kz * bh + ky) * bw + kx;
                nodes[e] = (int)n;
                kinds[e] = a.chg_key[e];
            }
            __syncthreads();
            for (int e = tid; e < nchg; e += SQ_THREADS) {
                const int ke = keys[e];
                int rank = 0;
                for (int j = 0; j < nchg; ++j) rank += keys[j] < ke;
                a.chg_node[rank] = nodes[e];
                a.chg_key[rank] = kinds[e];
            }
            __syncthreads();
        }
        const int total = sh_total;
        for (int k = tid; k < total; k += SQ_THREADS) a.ordermap[a.chg_node[k]] = k;
        __syncthreads();

        // (4) batches: gather, ordered replay, scatter
        for (int b0 = 0; b0 < total; b0 += SQ_BATCH) {
            const int nb = min(SQ_BATCH, total - b0);
            for (int e = tid; e < nb; e += SQ_THREADS) {
                ChgSh& c = ch[e];
                const unsigned n = (unsigned)a.chg_node[b0 + e];
                c.node = (int)n;
                c.kind = a.chg_key[b0 + e];
                const int x = (int)(n % (unsigned)L.nx), y = (int)((n / (unsigned)L.nx) % (unsigned)L.ny),
                          z = (int)(n / L.nxy);
                offset_from_squirmer(L, &s, x, y, z, c.r);
                if (c.kind == 1) {
                    // covered: momentum of the node's populations (lbm.cpp:294-298)
                    double p0 = 0, p1 = 0, p2 = 0, m = 0;
                    for (int i = 0; i < Q; ++i) {
                        const size_t k = logical_slot(L, a.parity, i, n, x, y, z);
                        const double fv = Pop<S>::get(a.f, k, i);
                        p0 += fv * c_cx[i]; p1 += fv * c_cy[i]; p2 += fv * c_cz[i];
                        m += Pop<S>::raw(a.f, k);
                    }
                    c.p[0] = p0; c.p[1] = p1; c.p[2] = p2; c.mass = m;
                }
            }
            __syncthreads();
            for (int q = tid; q < nb * 18; q += SQ_THREADS) {
                const int e = q / 18, j = q % 18 + 1;
                ChgSh& c = ch[e];
                if (c.kind != 2) continue;
                const unsigned n = (unsigned)c.node;
                const int x = (int)(n % (unsigned)L.nx), y = (int)((n / (unsigned)L.nx) % (unsigned)L.ny),
                          z = (int)(n / L.nxy);
                // lbm.cpp:305: neighbour with wrap in every axis
                const int xn = (x + c_cx[j] + L.nx) % L.nx, yn = (y + c_cy[j] + L.ny) % L.ny,
                          zn = (z + c_cz[j] + L.nz) % L.nz;
                const unsigned m = (unsigned)xn + (unsigned)L.nx * ((unsigned)yn + (unsigned)L.ny * (unsigned)zn);
                c.nbfl[j - 1] = a.flag[m] & TYPE_MASK;
                c.nbrho[j - 1] = a.rho[m];
                c.nbord[j - 1] = a.ordermap[m];
            }
            __syncthreads();
            if (tid == 0) {
                for (int e = 0; e < nb; ++e) {
                    ChgSh& c = ch[e];
                    if (c.kind == 1) {
                        const double t0 = c.r[1] * c.p[2] - c.r[2] * c.p[1];
                        const double t1 = c.r[2] * c.p[0] - c.r[0] * c.p[2];
                        const double t2 = c.r[0] * c.p[1] - c.r[1] * c.p[0];
                        s.Fc[0] += c.p[0]; s.Tc[0] += t0;
                        s.Fc[1] += c.p[1]; s.Tc[1] += t1;
                        s.Fc[2] += c.p[2]; s.Tc[2] += t2;
                        if (corr_step) sh_mass_delta -= c.mass;
                        sh_dfluid -= 1;
                        continue;
                    }
                    // uncovered: refill (lbm.cpp:302-317)
                    double rs = 0; int cntf = 0;
                    const int k_me = b0 + e;
                    for (int j = 0; j < 18; ++j) {
                        const int o = c.nbord[j];
                        uint8_t ty = c.nbfl[j];
                        double rv = c.nbrho[j];
                        if (o >= b0 && o < k_me) {  // changed earlier in this batch
                            const ChgSh& cc = ch[o - b0];
                            ty = cc.kind == 1 ? T_PARTICLE : T_FLUID;
                            if (cc.kind == 2) rv = cc.rr;
                        }
                        if (ty == T_FLUID) { rs += rv; ++cntf; }
                    }
                    const double rr = cntf ? rs / cntf : 1.0;
                    double ub[3];
                    surface_velocity(&s, c.r, ub, false);
                    c.rr = rr; c.ub[0] = ub[0]; c.ub[1] = ub[1]; c.ub[2] = ub[2];
                    const double p0 = rr * ub[0], p1 = rr * ub[1], p2 = rr * ub[2];
                    const double t0 = c.r[1] * p2 - c.r[2] * p1;
                    const double t1 = c.r[2] * p0 - c.r[0] * p2;
                    const double t2 = c.r[0] * p1 - c.r[1] * p0;
                    s.Fc[0] -= p0; s.Tc[0] -= t0;
                    s.Fc[1] -= p1; s.Tc[1] -= t1;
                    s.Fc[2] -= p2; s.Tc[2] -= t2;
                    sh_dfluid += 1;
                    if (corr_step) {
                        const double usq = ub[0] * ub[0] + ub[1] * ub[1] + ub[2] * ub[2];
                        for (int i = 0; i < Q; ++i) {
                            const double cu = c_cx[i] * ub[0] + c_cy[i] * ub[1] + c_cz[i] * ub[2];
                            const double feq = c_w[i] * rr * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * usq);
                            sh_mass_delta += Pop<S>::stored_raw(feq, i);
                        }
                    }
                }
            }
            __syncthreads();
            // scatter: flags, refilled populations, rho/u of uncovered nodes
            for (int q = tid; q < nb * Q; q += SQ_THREADS) {
                const int e = q / Q, i = q % Q;
                const ChgSh& c = ch[e];
                const unsigned n = (unsigned)c.node;
                const int x = (int)(n % (unsigned)L.nx), y = (int)((n / (unsigned)L.nx) % (unsigned)L.ny),
                          z = (int)(n / L.nxy);
                if (i == 0) {
                    uint8_t nf = T_PARTICLE;
                    if (c.kind == 2) {
                        const bool nw = (L.walls_y && (y == 1 || y == L.ny - 2)) || (L.walls_z && (z == 1 || z == L.nz - 2));
                        nf = T_FLUID | (nw ? NEAR_WALL : 0);
                        a.rho[n] = c.rr; a.ux[n] = c.ub[0]; a.uy[n] = c.ub[1]; a.uz[n] = c.ub[2];
                    }
                    a.flag[n] = nf;
                }
                if (c.kind == 2) {
                    // equilibrium() (lattice.hpp:42-47) at (rr, U + W x r)
                    const double cu = c_cx[i] * c.ub[0] + c_cy[i] * c.ub[1] + c_cz[i] * c.ub[2];
                    const double usq = c.ub[0] * c.ub[0] + c.ub[1] * c.ub[1] + c.ub[2] * c.ub[2];
                    const double feq = c_w[i] * c.rr * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * usq);
                    Pop<S>::put(a.f, logical_slot(L, a.parity, i, n, x, y, z), i, feq);
                }
            }
            __syncthreads();
        }
        for (int k = tid; k < total; k += SQ_THREADS) a.ordermap[a.chg_node[k]] = -1;

        // (5) boundary-link list: FLUID nodes with a PARTICLE neighbour, in
        // ascending node order over the sphere's box.
        if (total > 0 || s.n_links < 0) {
            const int old = max(0, s.n_links);
            for (int k = tid; k < old; k += SQ_THREADS) {
                const int n = a.links[k];
                a.flag[n] &= (uint8_t)~NEAR_PARTICLE;
            }
            __syncthreads();
            AxisRange ax, ay, az;
            ax.init(bx0, bw, L.nx); ay.init(by0, bh, L.ny); az.init(bz0, bd, L.nz);
            const int V2 = ax.width * ay.width * az.width;
            // after the remap FLUID means r >= R; PARTICLE neighbours lie within sqrt(2)
            const double Lin = fmax(s.R - 0.05, 0.0), Lout = s.R + 1.5;
            const double Lin2 = Lin * Lin, Lout2 = Lout * Lout;
            const int chk = (V2 + SQ_THREADS - 1) / SQ_THREADS;
            const int q0 = min(V2, tid * chk), q1 = min(V2, q0 + chk);
            auto region_walk = [&](auto&& visit) {
                for (int k = q0; k < q1; ++k) {
                    const int x = ax.at(k % ax.width), y = ay.at((k / ax.width) % ay.width),
                              z = az.at(k / (ax.width * ay.width));
                    visit(x, y, z);
                }
            };
            {
                int cnt = 0;
                region_walk([&](int x, int y, int z) {
                    const double r2 = approx_r2(x, y, z);
                    cnt += (r2 >= Lin2 && r2 < Lout2);
                });
                int off = 0;
                Scan(scan_tmp).ExclusiveSum(cnt, off, sh_total);
                __syncthreads();
                region_walk([&](int x, int y, int z) {
                    const double r2 = approx_r2(x, y, z);
                    if (r2 >= Lin2 && r2 < Lout2) {
                        if (off < a.chg_cap) a.cand[off] = x + L.nx * (y + L.ny * z);
                        ++off;
                    }
                });
            }
            __syncthreads();
            const int nc2 = min(sh_total, a.chg_cap);
            for (int c = tid; c < nc2; c += SQ_THREADS) {
                const unsigned n = (unsigned)a.cand[c];
                uint8_t mk = 0;
                if ((a.flag[n] & TYPE_MASK) == T_FLUID) {
                    const int x = (int)(n % (unsigned)L.nx), y = (int)((n / (unsigned)L.nx) % (unsigned)L.ny),
                              z = (int)(n / L.nxy);
                    const Nbr nbh(L, x, y, z);
                    bool near = false;
#pragma unroll
                    for (int j = 1; j < Q; ++j) near |= (a.flag[nbh.of(n, j)] & TYPE_MASK) == T_PARTICLE;
                    mk = near;
                }
                a.mark[c] = mk;
            }
            __syncthreads();
            {
                const int ch2 = (nc2 + SQ_THREADS - 1) / SQ_THREADS;
                const int c0 = min(nc2, tid * ch2), c1 = min(nc2, c0 + ch2);
                int cnt = 0;
                for (int c = c0; c < c1; ++c) cnt += a.mark[c];
                int off = 0;
                Scan(scan_tmp).ExclusiveSum(cnt, off, sh_total);
                __syncthreads();
                for (int c = c0; c < c1; ++c) {
                    if (!a.mark[c]) continue;
                    const int n = a.cand[c];
                    if (off < a.link_cap) {
                        a.links[off] = n;
                        a.linkslot[n] = off;
                        a.flag[n] |= NEAR_PARTICLE;
                    }
                    ++off;
                }
            }
            __syncthreads();
            if (tid == 0) {
                s.n_links = min(sh_total, a.link_cap);
                if (sh_total > a.link_cap) s.status |= ST_LINK_OVERFLOW;
            }
        }
        if (tid == 0) s.n_fluid += sh_dfluid;
    }

    // ---------------- stage LOOP ----------------
    double mstep = 0.0;
    if (corr_step) {
        block_sum_rows<1>(a.block_part, a.nblocks, BLOCK_PART, 3, sums);
        mstep = sums[0];
        block_sum_rows<1>(a.block_part_b, a.nblocks_b, BLOCK_PART, 3, sums);
        mstep += sums[0];
        if (a.nblocks_w > 0) {
            block_sum_rows<1>(a.block_part_w, a.nblocks_w, BLOCK_PART, 3, sums);
            mstep += sums[0];
        }
    }
    if (tid == 0) {
        if (loop) {
            s.corr_pending = 0;
            if (corr_step && s.n_fluid > 0) {
                // LBM::correctMass (lbm.cpp:324-339): d = 1 - m / n_fluid, with m
                // the populations summed after this step and its remap.
                const double m = mstep + sh_mass_delta;
                s.corr_d = S::shifted ? -(m / (double)s.n_fluid) : 1.0 - m / (double)s.n_fluid;
                s.corr_pending = 1;
            }
            if (s.traj_every > 0 && s.t % s.traj_every == 0) {
                double* row = a.traj + (size_t)(s.traj_count % TRAJ_RING) * TRAJ_COLS;
                row[0] = (double)s.t;
                for (int d = 0; d < 3; ++d) {
                    row[1 + d] = s.X[d]; row[4 + d] = s.e[d]; row[7 + d] = s.U[d]; row[10 + d] = s.W[d];
                }
                row[13] = s.Fw[1]; row[14] = s.Fw[2];
                s.traj_count += 1;
            }
        } else {
            s.corr_pending = 0;
        }
        // zones of the coming steps, from this box (see ZoneBox)
        const int blo[3] = {bx0, by0, bz0};
        const int nd[3] = {L.nx, L.ny, L.nz};
        const bool wall_axis[3] = {false, L.walls_y != 0, L.walls_z != 0};
        for (int slot : {a.zslot_a, a.zslot_b}) {
            if (slot < 0) continue;
            for (int d = 0; d < 3; ++d) {
                s.zone[slot].w[d] = zone_width(s.R, nd[d], wall_axis[d]);
                zone_axis(blo[d], nd[d], s.zone[slot].w[d], wall_axis[d], s.zone[slot].lo[d]);
            }
        }
        *a.sq = s;
    }
}

template <class S>
__global__ void __launch_bounds__(SQ_THREADS) k_squirmer(const Lattice L, const SqArgs a) {
    pdl_wait();
    pdl_launch_dependents();
    squirmer_update<S>(L, a);
}

// Ensemble: one CTA per member, each with its own lattice and arguments; the
// per-step settings are the same for all members.
template <class S>
__global__ void __launch_bounds__(SQ_THREADS) k_squirmer_batch(const Lattice* lat, const SqArgs* args, SqStep st) {
    __shared__ __align__(16) Lattice L;
    __shared__ __align__(16) SqArgs A;
    {   // the member's records, one word per thread, with this step's settings
        constexpr int NL = (int)(sizeof(Lattice) / 4), NA = (int)(sizeof(SqArgs) / 4);
        static_assert(NL <= SQ_THREADS && NA <= SQ_THREADS, "one word per thread");
        const int t = threadIdx.x;
        if (t < NL) reinterpret_cast<uint32_t*>(&L)[t] = reinterpret_cast<const uint32_t*>(lat + blockIdx.x)[t];
        if (t < NA) {
            uint32_t w = reinterpret_cast<const uint32_t*>(args + blockIdx.x)[t];
            if (t == (int)(offsetof(SqArgs, parity) / 4)) w = (uint32_t)st.parity;
            if (t == (int)(offsetof(SqArgs, stages) / 4)) w = (uint32_t)st.stages;
            if (t == (int)(offsetof(SqArgs, corr_step) / 4)) w = (uint32_t)st.corr_step;
            if (t == (int)(offsetof(SqArgs, zslot_a) / 4)) w = (uint32_t)st.zslot_a;
            if (t == (int)(offsetof(SqArgs, zslot_b) / 4)) w = (uint32_t)st.zslot_b;
            reinterpret_cast<uint32_t*>(&A)[t] = w;
        }
    }
    __syncthreads();
    squirmer_update<S>(L, A);
}

}  // namespace lbmgpu
