// ============================================================================
//  k_stream.cuh -- one time step of LBM::step (src/utils/lbm.cpp:128-224)
//  over the in-place AA access pattern, as two kernels over disjoint node sets:
//
//    k_bulk      every FLUID node with no WALL or PARTICLE neighbour (flag byte
//                exactly 0). A 3-D grid, threads along x: no integer division,
//                no neighbour-type lookup, no branch per direction.
//    k_boundary  the FLUID nodes next to a wall (a static list) and next to the
//                sphere (the boundary-link list the squirmer kernel rebuilds):
//                halfway bounce-back with the moving-boundary correction and the
//                momentum exchange, reduced per node (sphere) or per block
//                (walls).
//
//  Layout: one population array A[i][n] = A[i*N + n] (structure of arrays,
//  n = x + nx*(y + ny*z)), no second buffer.
//
//  AA pattern. Let P = completed steps mod 2 be the parity of the state.
//    P = 0 ("natural"):  logical f_i(n) is A[i][n].
//    P = 1 ("swapped"):  logical f_i(n) is A[opp(i)][n - c_i].
//  An even step (P 0 -> 1) reads A[i][n] and writes the post-collision value
//  of direction i to A[opp(i)][n]: it touches only its own node. An odd step
//  (P 1 -> 0) reads A[opp(i)][n - c_i] and writes A[i][n + c_i]. In both, the
//  slots a node reads are the slots it writes, so the update is in place,
//  race free, and any partition of the fluid nodes into kernels is valid.
//  Halfway bounce-back (lbm.cpp:188-199): when n + c_i is solid, the reflected
//  value becomes logical f_opp(i)(n) of the next state, i.e. A[i][n + c_i]
//  after an even step (a slot of the solid node, read back by the next odd
//  step) and A[opp(i)][n] after an odd step:
//      local  = A[opp(i)][n],   remote = A[i][n + c_i]
//      even:  fluid target -> local,  solid target -> remote
//      odd:   fluid target -> remote, solid target -> local
//  The logical mapping depends only on P, never on the flags, so the sphere
//  may cover/uncover nodes between steps (the remap reads and writes logical
//  slots through the same mapping).
//
//  FP64 form: the arithmetic of the reference, operation for operation and in
//  the same order, compiled without FMA contraction: one step reproduces the
//  reference's populations bit for bit.
//  FP32 / FP16 forms: deviations d_i = f_i - w_i are stored; moments and the
//  TRT update run in FP32 in deviation form, one opposite pair at a time
//  (f+_i, feq+_i and S+_i are shared by i and opp(i), the odd parts change
//  sign); boundary-link velocities, the momentum exchange and all sums are FP64.
// ============================================================================
#pragma once
#include "lbm_common.cuh"

namespace lbmgpu {

constexpr int BOUNDARY_BLOCK = 128;

// LBM::offsetFromSquirmer (lbm.cpp:100-104): minimum image in x always, in
// y/z only where there is no wall.
__device__ __forceinline__ void offset_from_squirmer(const Lattice& L, const SqState* s, double px,
                                                     double py, double pz, double r[3]) {
    r[0] = px - s->X[0]; r[0] -= L.nx * round(r[0] / L.nx);
    r[1] = py - s->X[1]; if (!L.walls_y) r[1] -= L.ny * round(r[1] / L.ny);
    r[2] = pz - s->X[2]; if (!L.walls_z) r[2] -= L.nz * round(r[2] / L.nz);
}

// Squirmer::surfaceVelocity (squirmer.cpp:35-46): U + W x r, plus the Blake
// two-mode slip B1 (1 + beta cos th)(cos th r^ - e) when with_slip.
__device__ __forceinline__ void surface_velocity(const SqState* s, const double r[3], double ub[3],
                                                 bool with_slip) {
    const double wr0 = s->W[1] * r[2] - s->W[2] * r[1];
    const double wr1 = s->W[2] * r[0] - s->W[0] * r[2];
    const double wr2 = s->W[0] * r[1] - s->W[1] * r[0];
    ub[0] = s->U[0] + wr0; ub[1] = s->U[1] + wr1; ub[2] = s->U[2] + wr2;
    if (!with_slip) return;
    const double rn = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    if (rn < 1e-12) return;
    const double rh[3] = {r[0] / rn, r[1] / rn, r[2] / rn};
    const double ct = s->e[0] * rh[0] + s->e[1] * rh[1] + s->e[2] * rh[2];
    const double amp = s->B1 * (1.0 + s->beta * ct);
    for (int d = 0; d < 3; ++d) ub[d] += amp * (ct * rh[d] - s->e[d]);
}

// Neighbour offsets with periodic wrap in every axis (lbm.cpp:180-184). Walls
// are solid node layers, so wrapping across them never reaches a fluid node.
struct Nbr {
    int xp, xm, yp, ym, zp, zm;
    __device__ __forceinline__ Nbr(const Lattice& L, int x, int y, int z) {
        xp = (x == L.nx - 1) ? 1 - L.nx : 1;
        xm = (x == 0) ? L.nx - 1 : -1;
        yp = (y == L.ny - 1) ? (1 - L.ny) * L.nx : L.nx;
        ym = (y == 0) ? (L.ny - 1) * L.nx : -L.nx;
        zp = (z == L.nz - 1) ? (1 - L.nz) * (int)L.nxy : (int)L.nxy;
        zm = (z == 0) ? (L.nz - 1) * (int)L.nxy : -(int)L.nxy;
    }
    // n + c_i
    __device__ __forceinline__ unsigned of(unsigned n, int i) const {
        int o = 0;
        if (CX(i) > 0) o += xp; else if (CX(i) < 0) o += xm;
        if (CY(i) > 0) o += yp; else if (CY(i) < 0) o += ym;
        if (CZ(i) > 0) o += zp; else if (CZ(i) < 0) o += zm;
        return (unsigned)((int)n + o);
    }
};

// Deterministic block reduction of 4 doubles into out[0..3] (thread 0 writes).
// BLOCK bounds the block size; the warps actually present are counted.
template <int BLOCK>
__device__ __forceinline__ void block_reduce4(double v0, double v1, double v2, double v3, double* out) {
    __shared__ double red[BLOCK / 32][4];
    const int nwarps = (int)((blockDim.x * blockDim.y * blockDim.z + 31) >> 5);
    const unsigned full = 0xffffffffu;
    for (int o = 16; o > 0; o >>= 1) {
        v0 += __shfl_down_sync(full, v0, o);
        v1 += __shfl_down_sync(full, v1, o);
        v2 += __shfl_down_sync(full, v2, o);
        v3 += __shfl_down_sync(full, v3, o);
    }
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int lane = tid & 31, wid = tid >> 5;
    if (lane == 0) { red[wid][0] = v0; red[wid][1] = v1; red[wid][2] = v2; red[wid][3] = v3; }
    __syncthreads();
    if (tid == 0) {
        double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
        for (int w = 0; w < nwarps; ++w) { s0 += red[w][0]; s1 += red[w][1]; s2 += red[w][2]; s3 += red[w][3]; }
        out[0] = s0; out[1] = s1; out[2] = s2; out[3] = s3;
    }
}

// Loads of the 19 logical populations of node n in a state of parity PAR.
template <class S, int PAR, class V>
__device__ __forceinline__ void load_node(const typename S::T* __restrict__ f, unsigned N, unsigned n,
                                          const Nbr& nb, V* v) {
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const typename S::T* p = PAR == 0 ? f + (size_t)i * N + n : f + (size_t)OPP(i) * N + nb.of(n, OPP(i));
        v[i] = (V)S::ld(p);
    }
}

// The per-step settings every thread reads from the device state.
struct StepFlags {
    bool do_mass;
    int corr_on;
    double corr;
};
template <bool SQ>
__device__ __forceinline__ StepFlags step_flags(const StreamArgs& a) {
    StepFlags s{false, 0, 0.0};
    if (SQ) {
        const SqState* sq = a.sq;
        s.corr_on = sq->corr_pending;
        s.corr = sq->corr_d;
        if (a.fused && sq->mass_every > 0) s.do_mass = ((sq->t + 1) % sq->mass_every) == 0;
    }
    return s;
}

__device__ __forceinline__ bool in_rho_box(const Lattice& L, const SqState* sq, int x, int y, int z) {
    int dx = x - sq->rb_lo[0]; if (dx < 0) dx += L.nx;
    int dy = y - sq->rb_lo[1]; if (dy < 0) dy += L.ny;
    int dz = z - sq->rb_lo[2]; if (dz < 0) dz += L.nz;
    return dx < sq->rb_w[0] && dy < sq->rb_w[1] && dz < sq->rb_w[2];
}

// ---------------------------------------------------------------------------
//  k_bulk<S, PAR, SQ, MACRO>: nodes whose flag byte is 0.
//    SQ    the lattice has a squirmer: store rho inside the refill region,
//          apply a pending mass correction, sum the mass on correction steps
//    MACRO store rho and u of every node (the last step of every host call)
//  grid (ceil(nx/blockDim.x), ny, nz); block (TX, 1, 1) with TX = 32..256.
// ---------------------------------------------------------------------------
template <class S, int PAR, bool SQ, bool MACRO>
__global__ void __launch_bounds__(256) k_bulk(const Lattice L, const StreamArgs a) {
    using T = typename S::T;
    T* __restrict__ f = static_cast<T*>(a.f);
    const unsigned N = L.N;
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, z = blockIdx.z;
    const unsigned n = (unsigned)x + (unsigned)L.nx * ((unsigned)y + (unsigned)L.ny * (unsigned)z);
    const bool active = x < L.nx && a.flag[n] == 0;
    const StepFlags sf = step_flags<SQ>(a);
    double msum = 0.0;

    if (active) {
        const Nbr nb(L, x, y, z);
        const bool store_rho = MACRO || (SQ && in_rho_box(L, a.sq, x, y, z));
        if constexpr (!S::shifted) {
            // ---------------- FP64: the reference's arithmetic ----------------
            double fv[Q];
            load_node<S, PAR>(f, N, n, nb, fv);
            if (SQ && sf.corr_on) {
#pragma unroll
                for (int i = 0; i < Q; ++i) fv[i] += WD(i) * sf.corr;  // LBM::correctMass (lbm.cpp:337)
            }
            // moments, Guo half-force velocity (lbm.cpp:143-152)
            double r = 0, mx = 0, my = 0, mz = 0;
#pragma unroll
            for (int i = 0; i < Q; ++i) {
                r += fv[i];
                if (CX(i) > 0) mx += fv[i]; else if (CX(i) < 0) mx -= fv[i];
                if (CY(i) > 0) my += fv[i]; else if (CY(i) < 0) my -= fv[i];
                if (CZ(i) > 0) mz += fv[i]; else if (CZ(i) < 0) mz -= fv[i];
            }
            const double Fx = L.F[0], Fy = L.F[1], Fz = L.F[2];
            const double u = (mx + 0.5 * Fx) / r, v = (my + 0.5 * Fy) / r, wz = (mz + 0.5 * Fz) / r;
            if (store_rho) a.rho[n] = r;
            if (MACRO) { a.ux[n] = u; a.uy[n] = v; a.uz[n] = wz; }
            const double usq = u * u + v * v + wz * wz, uF = u * Fx + v * Fy + wz * Fz;
#pragma unroll
            for (int i = 0; i < Q; ++i) {
                // TRT + Guo forcing (lbm.cpp:162-172)
                const int io = OPP(i);
                const double cu = CX(i) * u + CY(i) * v + CZ(i) * wz;
                const double cF = CX(i) * Fx + CY(i) * Fy + CZ(i) * Fz;
                const double feqP = WD(i) * r * (1.0 + 4.5 * cu * cu - 1.5 * usq);
                const double feqM = WD(i) * r * 3.0 * cu;
                const double fP = 0.5 * (fv[i] + fv[io]), fM = 0.5 * (fv[i] - fv[io]);
                const double SP = WD(i) * (9.0 * cu * cF - 3.0 * uF), SM = WD(i) * 3.0 * cF;
                const double fpost = fv[i] - L.omP * (fP - feqP) - L.omM * (fM - feqM) + L.gP * SP + L.gM * SM;
                S::st(PAR == 0 ? f + (size_t)io * N + n : f + (size_t)i * N + nb.of(n, i), fpost);
                if (SQ && sf.do_mass) msum += fpost;
            }
        } else {
            // ------------- FP32 arithmetic on stored deviations ---------------
            float d[Q];
            load_node<S, PAR>(f, N, n, nb, d);
            if (SQ && sf.corr_on) {
#pragma unroll
                for (int i = 0; i < Q; ++i) d[i] += (float)(WD(i) * sf.corr);
            }
            float dr = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
            for (int i = 0; i < Q; ++i) {
                dr += d[i];
                if (CX(i) > 0) jx += d[i]; else if (CX(i) < 0) jx -= d[i];
                if (CY(i) > 0) jy += d[i]; else if (CY(i) < 0) jy -= d[i];
                if (CZ(i) > 0) jz += d[i]; else if (CZ(i) < 0) jz -= d[i];
            }
            const float rho = 1.0f + dr;
            const float inv = 1.0f / rho;
            const float u = (jx + 0.5f * L.Ff[0]) * inv, v = (jy + 0.5f * L.Ff[1]) * inv, wz = (jz + 0.5f * L.Ff[2]) * inv;
            if (store_rho) a.rho[n] = 1.0 + (double)dr;
            if (MACRO) { a.ux[n] = u; a.uy[n] = v; a.uz[n] = wz; }
            const float usq = u * u + v * v + wz * wz;
            const float uF = u * L.Ff[0] + v * L.Ff[1] + wz * L.Ff[2];
            const float omP = L.omPf, omM = L.omMf, gP = L.gPf;
            const float k15 = 1.5f * usq;
            {   // rest population: c = 0
                const float eP = WF(0) * (dr - rho * k15);
                const float out = d[0] - omP * (d[0] - eP) - gP * WF(0) * 3.0f * uF;
                S::st(f + n, out);
                if (SQ && sf.do_mass) msum += (double)S::rt(out);
            }
#pragma unroll
            for (int i = 1; i < Q; i += 2) {
                const int io = i + 1;
                const float cu = CX(i) * u + CY(i) * v + CZ(i) * wz;
                const float w = WF(i);
                const float eP = w * (dr + rho * (4.5f * cu * cu - k15));  // feq+ - w
                const float eM = 3.0f * w * rho * cu;                       // feq-
                const float fP = 0.5f * (d[i] + d[io]), fM = 0.5f * (d[i] - d[io]);
                const float A = gP * w * (9.0f * cu * L.cF[i] - 3.0f * uF) - omP * (fP - eP);
                const float B = L.cm[i] - omM * (fM - eM);
                const float oi = d[i] + A + B, oo = d[io] + A - B;
                if (PAR == 0) {
                    S::st(f + (size_t)io * N + n, oi);
                    S::st(f + (size_t)i * N + n, oo);
                } else {
                    S::st(f + (size_t)i * N + nb.of(n, i), oi);
                    S::st(f + (size_t)io * N + nb.of(n, io), oo);
                }
                if (SQ && sf.do_mass) msum += (double)S::rt(oi) + (double)S::rt(oo);
            }
        }
    }
    if (SQ && sf.do_mass) {
        const unsigned bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
        block_reduce4<256>(0.0, 0.0, 0.0, msum, a.block_part + (size_t)bid * BLOCK_PART);
    }
}

// ---------------------------------------------------------------------------
//  k_boundary<S, PAR, SQ, MACRO>: thread k handles wall_nodes[k] (k < n_wall;
//  skipped unless FLUID without PARTICLE neighbour) or links[k - n_wall]
//  (k - n_wall < n_links, the row of link_part it writes).
// ---------------------------------------------------------------------------
template <class S, int PAR, bool SQ, bool MACRO>
__global__ void __launch_bounds__(BOUNDARY_BLOCK) k_boundary(const Lattice L, const StreamArgs a) {
    using T = typename S::T;
    T* __restrict__ f = static_cast<T*>(a.f);
    const unsigned N = L.N;
    const SqState* __restrict__ sq = a.sq;
    const int k = blockIdx.x * BOUNDARY_BLOCK + threadIdx.x;
    const int n_links = SQ ? sq->n_links : 0;
    int link = -1;
    unsigned n = 0;
    bool active = false;
    if (k < a.n_wall) {
        n = (unsigned)a.wall_nodes[k];
        const uint8_t fl = a.flag[n];
        active = (fl & TYPE_MASK) == T_FLUID && !(fl & NEAR_PARTICLE);
    } else if (SQ && k - a.n_wall < n_links) {
        link = k - a.n_wall;
        n = (unsigned)a.links[link];
        active = true;
    }
    const StepFlags sf = step_flags<SQ>(a);
    const bool do_red = MACRO || sf.do_mass;
    double fw0 = 0.0, fw1 = 0.0, fw2 = 0.0, msum = 0.0;

    if (active) {
        const int x = (int)(n % (unsigned)L.nx);
        const unsigned yz = n / (unsigned)L.nx;
        const int y = (int)(yz % (unsigned)L.ny);
        const int z = (int)(yz / (unsigned)L.ny);
        const Nbr nb(L, x, y, z);
        const bool store_rho = MACRO || (SQ && in_rho_box(L, sq, x, y, z));
        double fp0 = 0.0, fp1 = 0.0, fp2 = 0.0, tp0 = 0.0, tp1 = 0.0, tp2 = 0.0;

        if constexpr (!S::shifted) {
            double fv[Q];
            load_node<S, PAR>(f, N, n, nb, fv);
            if (SQ && sf.corr_on) {
#pragma unroll
                for (int i = 0; i < Q; ++i) fv[i] += WD(i) * sf.corr;
            }
            double r = 0, mx = 0, my = 0, mz = 0;
#pragma unroll
            for (int i = 0; i < Q; ++i) {
                r += fv[i];
                if (CX(i) > 0) mx += fv[i]; else if (CX(i) < 0) mx -= fv[i];
                if (CY(i) > 0) my += fv[i]; else if (CY(i) < 0) my -= fv[i];
                if (CZ(i) > 0) mz += fv[i]; else if (CZ(i) < 0) mz -= fv[i];
            }
            const double Fx = L.F[0], Fy = L.F[1], Fz = L.F[2];
            const double u = (mx + 0.5 * Fx) / r, v = (my + 0.5 * Fy) / r, wz = (mz + 0.5 * Fz) / r;
            if (store_rho) a.rho[n] = r;
            if (MACRO) { a.ux[n] = u; a.uy[n] = v; a.uz[n] = wz; }
            const double usq = u * u + v * v + wz * wz, uF = u * Fx + v * Fy + wz * Fz;
#pragma unroll
            for (int i = 0; i < Q; ++i) {
                const int io = OPP(i);
                const double cu = CX(i) * u + CY(i) * v + CZ(i) * wz;
                const double cF = CX(i) * Fx + CY(i) * Fy + CZ(i) * Fz;
                const double feqP = WD(i) * r * (1.0 + 4.5 * cu * cu - 1.5 * usq);
                const double feqM = WD(i) * r * 3.0 * cu;
                const double fP = 0.5 * (fv[i] + fv[io]), fM = 0.5 * (fv[i] - fv[io]);
                const double SP = WD(i) * (9.0 * cu * cF - 3.0 * uF), SM = WD(i) * 3.0 * cF;
                const double fpost = fv[i] - L.omP * (fP - feqP) - L.omM * (fM - feqM) + L.gP * SP + L.gM * SM;
                const unsigned nbi = nb.of(n, i);
                T* local = f + (size_t)io * N + n;
                T* remote = f + (size_t)i * N + nbi;
                const uint8_t tt = i == 0 ? T_FLUID : (a.flag[nbi] & TYPE_MASK);
                if (tt == T_FLUID) {  // push (lbm.cpp:186)
                    S::st(PAR == 0 ? local : remote, fpost);
                    if (sf.do_mass) msum += fpost;
                    continue;
                }
                // halfway bounce-back with moving-boundary correction (lbm.cpp:189-199)
                double ub[3] = {0, 0, 0}, rb[3] = {0, 0, 0};
                if (SQ && tt == T_PARTICLE) {
                    offset_from_squirmer(L, sq, x + 0.5 * CX(i), y + 0.5 * CY(i), z + 0.5 * CZ(i), rb);
                    surface_velocity(sq, rb, ub, true);
                }
                const double cub = CX(i) * ub[0] + CY(i) * ub[1] + CZ(i) * ub[2];
                const double fb = fpost - 6.0 * WD(i) * r * cub;
                S::st(PAR == 0 ? remote : local, fb);
                if (sf.do_mass) msum += fb;
                // Galilean-invariant momentum exchange (lbm.cpp:202-215)
                const double sm = fpost + fb, dl = fpost - fb;
                const double dpx = sm * CX(i) - dl * ub[0];
                const double dpy = sm * CY(i) - dl * ub[1];
                const double dpz = sm * CZ(i) - dl * ub[2];
                if (tt == T_WALL) { fw0 += dpx; fw1 += dpy; fw2 += dpz; }
                else {
                    fp0 += dpx; fp1 += dpy; fp2 += dpz;
                    tp0 += rb[1] * dpz - rb[2] * dpy;
                    tp1 += rb[2] * dpx - rb[0] * dpz;
                    tp2 += rb[0] * dpy - rb[1] * dpx;
                }
            }
        } else {
            float d[Q];
            load_node<S, PAR>(f, N, n, nb, d);
            if (SQ && sf.corr_on) {
#pragma unroll
                for (int i = 0; i < Q; ++i) d[i] += (float)(WD(i) * sf.corr);
            }
            float dr = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
            for (int i = 0; i < Q; ++i) {
                dr += d[i];
                if (CX(i) > 0) jx += d[i]; else if (CX(i) < 0) jx -= d[i];
                if (CY(i) > 0) jy += d[i]; else if (CY(i) < 0) jy -= d[i];
                if (CZ(i) > 0) jz += d[i]; else if (CZ(i) < 0) jz -= d[i];
            }
            const float rho = 1.0f + dr;
            const float inv = 1.0f / rho;
            const float u = (jx + 0.5f * L.Ff[0]) * inv, v = (jy + 0.5f * L.Ff[1]) * inv, wz = (jz + 0.5f * L.Ff[2]) * inv;
            if (store_rho) a.rho[n] = 1.0 + (double)dr;
            if (MACRO) { a.ux[n] = u; a.uy[n] = v; a.uz[n] = wz; }
            const float usq = u * u + v * v + wz * wz;
            const float uF = u * L.Ff[0] + v * L.Ff[1] + wz * L.Ff[2];
            const float omP = L.omPf, omM = L.omMf, gP = L.gPf;
            const float k15 = 1.5f * usq;
            float post[Q];
            post[0] = d[0] - omP * (d[0] - WF(0) * (dr - rho * k15)) - gP * WF(0) * 3.0f * uF;
#pragma unroll
            for (int i = 1; i < Q; i += 2) {
                const int io = i + 1;
                const float cu = CX(i) * u + CY(i) * v + CZ(i) * wz;
                const float w = WF(i);
                const float eP = w * (dr + rho * (4.5f * cu * cu - k15));
                const float eM = 3.0f * w * rho * cu;
                const float fP = 0.5f * (d[i] + d[io]), fM = 0.5f * (d[i] - d[io]);
                const float A = gP * w * (9.0f * cu * L.cF[i] - 3.0f * uF) - omP * (fP - eP);
                const float B = L.cm[i] - omM * (fM - eM);
                post[i] = d[i] + A + B;
                post[io] = d[io] + A - B;
            }
#pragma unroll
            for (int i = 0; i < Q; ++i) {
                const float dpost = post[i];
                const unsigned nbi = nb.of(n, i);
                T* local = f + (size_t)OPP(i) * N + n;
                T* remote = f + (size_t)i * N + nbi;
                const uint8_t tt = i == 0 ? T_FLUID : (a.flag[nbi] & TYPE_MASK);
                if (tt == T_FLUID) {
                    S::st(PAR == 0 ? local : remote, dpost);
                    if (sf.do_mass) msum += (double)S::rt(dpost);
                    continue;
                }
                double ub[3] = {0, 0, 0}, rb[3] = {0, 0, 0};
                if (SQ && tt == T_PARTICLE) {
                    offset_from_squirmer(L, sq, x + 0.5 * CX(i), y + 0.5 * CY(i), z + 0.5 * CZ(i), rb);
                    surface_velocity(sq, rb, ub, true);
                }
                const double cub = CX(i) * ub[0] + CY(i) * ub[1] + CZ(i) * ub[2];
                const double dl = 6.0 * WD(i) * (double)rho * cub;   // fpost - fb
                const float dfb = (float)((double)dpost - dl);
                S::st(PAR == 0 ? remote : local, dfb);
                if (sf.do_mass) msum += (double)S::rt(dfb);
                const double fpost = WD(i) + (double)dpost;
                const double sm = 2.0 * fpost - dl;                   // fpost + fb
                const double dpx = sm * CX(i) - dl * ub[0];
                const double dpy = sm * CY(i) - dl * ub[1];
                const double dpz = sm * CZ(i) - dl * ub[2];
                if (tt == T_WALL) { fw0 += dpx; fw1 += dpy; fw2 += dpz; }
                else {
                    fp0 += dpx; fp1 += dpy; fp2 += dpz;
                    tp0 += rb[1] * dpz - rb[2] * dpy;
                    tp1 += rb[2] * dpx - rb[0] * dpz;
                    tp2 += rb[0] * dpy - rb[1] * dpx;
                }
            }
        }
        if (SQ && link >= 0) {
            double* lp = a.link_part + (size_t)link * LINK_PART;
            lp[0] = fp0; lp[1] = fp1; lp[2] = fp2; lp[3] = tp0; lp[4] = tp1; lp[5] = tp2;
        }
    }
    if (do_red) block_reduce4<BOUNDARY_BLOCK>(fw0, fw1, fw2, msum, a.block_part_b + (size_t)blockIdx.x * BLOCK_PART);
}

}  // namespace lbmgpu
