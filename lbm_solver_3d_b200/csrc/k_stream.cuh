// ============================================================================
//  k_stream.cuh -- one time step of LBM::step (src/utils/lbm.cpp:128-224)
//  over the in-place AA access pattern, as two kernels over disjoint node sets:
//
//    k_bulk  every FLUID node without a PARTICLE neighbour outside the zone
//            around the sphere. A 3-D grid, threads along x: no integer
//            division, no neighbour-type lookup, nothing read from the
//            squirmer update. Wall layers are whole x-rows, so a row next to a
//            wall knows its solid directions from (y, z) alone (halfway
//            bounce-back, momentum exchange on the wall).
//    k_zone  the FLUID nodes of the zone (a box of fixed width around the
//            sphere, see ZoneBox): halfway bounce-back with the moving-boundary
//            correction and the momentum exchange, reduced per node (sphere)
//            or per block (walls).
//  Because k_bulk never touches the zone, it may run while the squirmer update
//  of the previous step is still remapping the sphere.
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
#include <type_traits>

#include "k_logical.cuh"
#include "lbm_common.cuh"

namespace lbmgpu {

// Threads of a zone CTA, and the registers the single-lattice zone kernel may
// use. Sized so that a zone CTA fits on an SM beside the staged-row bulk
// kernel's two CTAs: those are 18 warps of 96 registers, spread 5/5/4/4 over
// the SM's four 16,384-register partitions, which leaves 4,096 registers in
// two of them -- one warp of 128 registers each. The zone of the next step
// then runs while the bulk of this one does instead of after it.
constexpr int BOUNDARY_BLOCK = 64;
constexpr int ZONE_MAX_REGS = 128;

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

__device__ __forceinline__ bool in_zone(const Lattice& L, const ZoneBox& z, int x, int y, int zc) {
    return in_zone_axis(x, z.lo[0], z.w[0], L.nx, false) && in_zone_axis(y, z.lo[1], z.w[1], L.ny, L.walls_y) &&
           in_zone_axis(zc, z.lo[2], z.w[2], L.nz, L.walls_z);
}

// Partial sums a node contributes: wall force, stored mass (correction steps),
// sphere force and torque.
struct NodeSums {
    double fw[3] = {0, 0, 0};
    double mass = 0;
    double fp[3] = {0, 0, 0}, tp[3] = {0, 0, 0};
    unsigned pmask = 0;   // GENERAL: directions of the node's particle links, left for zone_particle_links
    double rho = 0;       // GENERAL: the node's density, for zone_particle_links
};

// Post-collision values of a zone block's particle links, [direction][thread]:
// the population itself (FP64) or its deviation (shifted forms).
template <class S>
using LinkStash = typename S::A;

// ---------------------------------------------------------------------------
//  update_node: the whole LBM::step body for one fluid node n.
//    GENERAL = false: every neighbour is fluid (flag byte 0): plain push.
//    GENERAL = true : neighbour types are read for nodes whose flag has a
//                     near-wall / near-particle bit: bounce-back, momentum
//                     exchange.
//    STORE_RHO: keep rho (and u if MACRO) for this node.
// ---------------------------------------------------------------------------
// Wall-adjacent rows, for the bulk kernel: bit 0 the y-1 layer is a wall,
// bit 1 the y+1 layer, bit 2 z-1, bit 3 z+1 (a whole x-row shares them).
__device__ __forceinline__ uint8_t wall_row(const Lattice& L, int y, int z) {
    uint8_t w = 0;
    if (L.walls_y) { if (y == 1) w |= 1; if (y == L.ny - 2) w |= 2; }
    if (L.walls_z) { if (z == 1) w |= 4; if (z == L.nz - 2) w |= 8; }
    return w;
}
__device__ __forceinline__ bool wall_dir(int i, uint8_t wr) {
    return (CY(i) < 0 && (wr & 1)) || (CY(i) > 0 && (wr & 2)) || (CZ(i) < 0 && (wr & 4)) || (CZ(i) > 0 && (wr & 8));
}

// Types of the 18 neighbours n + c_i, 2 bits each at bit 2i (the loads are
// independent and go out together).
__device__ __forceinline__ uint64_t neighbour_types(const Lattice& L, const uint8_t* __restrict__ flag, unsigned n,
                                                    const Nbr& nb) {
    uint64_t m = 0;
#pragma unroll
    for (int i = 1; i < Q; ++i) m |= (uint64_t)(flag[nb.of(n, i)] & TYPE_MASK) << (2 * i);
    return m;
}

// Where update_node reads the 19 logical populations from: the population
// array itself (GlobalSrc), or a copy staged in shared memory (StagedSrc in
// k_batch.cuh). Either returns the stored values converted by S::ld.
struct GlobalSrc {
    template <class S, int PAR, class V>
    __device__ __forceinline__ void load(const typename S::T* __restrict__ f, unsigned N, unsigned n, const Nbr& nb,
                                         V* v) const {
        load_node<S, PAR>(f, N, n, nb, v);
    }
};

// Constants of the collision in the arithmetic A of a storage form (A = float:
// the FP32 copies kept in Lattice; A = double: the FP64 values themselves).
template <class A> struct Coll;
template <> struct Coll<float> {
    __device__ static float omP(const Lattice& L) { return L.omPf; }
    __device__ static float omM(const Lattice& L) { return L.omMf; }
    __device__ static float gP(const Lattice& L) { return L.gPf; }
    __device__ static float F(const Lattice& L, int d) { return L.Ff[d]; }
    __device__ static float cF(const Lattice& L, int i) { return L.cF[i]; }
    __device__ static float cm(const Lattice& L, int i) { return L.cm[i]; }
    __host__ __device__ static constexpr float w(int i) { return WF(i); }
};
template <> struct Coll<double> {
    __device__ static double omP(const Lattice& L) { return L.omP; }
    __device__ static double omM(const Lattice& L) { return L.omM; }
    __device__ static double gP(const Lattice& L) { return L.gP; }
    __device__ static double F(const Lattice& L, int d) { return L.F[d]; }
    __device__ static double cF(const Lattice& L, int i) { return CX(i) * L.F[0] + CY(i) * L.F[1] + CZ(i) * L.F[2]; }
    __device__ static double cm(const Lattice& L, int i) { return L.gM * 3.0 * WD(i) * cF(L, i); }
    __host__ __device__ static constexpr double w(int i) { return WD(i); }
};

// Moments of a node in the shifted forms, from its 19 stored numbers d (storage
// units: the deviation times S::SC), in the form's arithmetic A: dr = sum of d,
// rho, and the Guo half-force velocity (lbm.cpp:143-152).
template <class S, class A = typename S::A>
__device__ __forceinline__ void shifted_moments(const Lattice& L, const float* d, A& dr, A& rho, A& u, A& v, A& wz) {
    A jx = 0, jy = 0, jz = 0;
    dr = 0;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const A di = (A)d[i];
        dr += di;
        if (CX(i) > 0) jx += di; else if (CX(i) < 0) jx -= di;
        if (CY(i) > 0) jy += di; else if (CY(i) < 0) jy -= di;
        if (CZ(i) > 0) jz += di; else if (CZ(i) < 0) jz -= di;
    }
    if constexpr (sizeof(A) == 4) {   // every operation spelled out: no kernel contracts it differently
        rho = __fmaf_rn(dr, S::INV, 1.0f);
        const float inv = __fdiv_rn(1.0f, rho);
        u = __fmul_rn(__fmaf_rn(jx, S::INV, __fmul_rn(0.5f, L.Ff[0])), inv);
        v = __fmul_rn(__fmaf_rn(jy, S::INV, __fmul_rn(0.5f, L.Ff[1])), inv);
        wz = __fmul_rn(__fmaf_rn(jz, S::INV, __fmul_rn(0.5f, L.Ff[2])), inv);
    } else {
        rho = A(1) + dr * (A)S::INV;
        const A inv = A(1) / rho;
        u = (jx * (A)S::INV + A(0.5) * Coll<A>::F(L, 0)) * inv;
        v = (jy * (A)S::INV + A(0.5) * Coll<A>::F(L, 1)) * inv;
        wz = (jz * (A)S::INV + A(0.5) * Coll<A>::F(L, 2)) * inv;
    }
}

// The per-node terms of the collision: k15 = 1.5 |u|^2, uF = u . F and
// srho = S::SC * rho (FP32: explicit operations, as in shifted_moments).
template <class S, class A = typename S::A>
__device__ __forceinline__ void shifted_terms(const Lattice& L, A rho, A u, A v, A wz, A& k15, A& uF, A& srho) {
    if constexpr (sizeof(A) == 4) {
        k15 = __fmul_rn(1.5f, __fmaf_rn(wz, wz, __fmaf_rn(v, v, __fmul_rn(u, u))));
        uF = __fmaf_rn(wz, L.Ff[2], __fmaf_rn(v, L.Ff[1], __fmul_rn(u, L.Ff[0])));
        srho = __fmul_rn(S::SC, rho);   // a power of two: exact
    } else {
        k15 = A(1.5) * (u * u + v * v + wz * wz);
        uF = u * Coll<A>::F(L, 0) + v * Coll<A>::F(L, 1) + wz * Coll<A>::F(L, 2);
        srho = (A)S::SC * rho;
    }
}

// weight class of direction i: 0 rest, 1 axes, 2 diagonals
__host__ __device__ constexpr int wclass(int i) { return i == 0 ? 0 : (i <= 6 ? 1 : 2); }

// Two nodes' FP32 numbers side by side (element 0: the first node, element 1:
// the second) and the sm_100 paired FP32 FMA on them (PTX fma.rn.f32x2: each
// element rounded once, as __fmaf_rn rounds it).
__device__ __forceinline__ float2 bc2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
    unsigned long long r, pa, pb, pc;
    asm("mov.b64 %0, {%1, %2};" : "=l"(pa) : "f"(a.x), "f"(a.y));
    asm("mov.b64 %0, {%1, %2};" : "=l"(pb) : "f"(b.x), "f"(b.y));
    asm("mov.b64 %0, {%1, %2};" : "=l"(pc) : "f"(c.x), "f"(c.y));
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(pa), "l"(pb), "l"(pc));
    float2 o;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(o.x), "=f"(o.y) : "l"(r));
    return o;
}

// Paired adds, subtracts and multiplies, each written as that FMA with a
// constant the compiler cannot see (Lattice::one = 1, Lattice::mzero = -0):
//   a + b = fma(a, 1, b),  a - b = fma(b, -1, a),  a * b = fma(a, b, -0).
// x * 1 and x * -1 are exact and p + (-0) = p for every p, signed zeros
// included, so each is the IEEE result of the scalar __fadd_rn / __fsub_rn /
// __fmul_rn bit for bit; and as FMAs with unknown operands they are neither
// fused with their neighbours nor reordered. (Written as the plain paired add
// and multiply instructions instead, the two-node results were measured to
// differ from the one-node ones in the last place.)
struct Paired {
    float2 one, mone, mz;
    __device__ __forceinline__ explicit Paired(const Lattice& L)
        : one(bc2(L.one)), mone(bc2(-L.one)), mz(bc2(L.mzero)) {}
    __device__ __forceinline__ float2 add(float2 a, float2 b) const { return fma2(a, one, b); }
    __device__ __forceinline__ float2 sub(float2 a, float2 b) const { return fma2(b, mone, a); }
    __device__ __forceinline__ float2 mul(float2 a, float2 b) const { return fma2(a, b, mz); }
};

// c_i . u in FP32 for a moving direction (one or two nonzero components, each
// -1 or 1): the terms in x, y, z order and one explicit rounded sum, formed the
// same way by the one-node (V = float) and the two-node (V = float2) code.
__device__ __forceinline__ float cdot_neg(float a) { return -a; }
__device__ __forceinline__ float2 cdot_neg(float2 a) { return neg2(a); }
struct ScalarAdd {
    __device__ __forceinline__ float add(float a, float b) const { return __fadd_rn(a, b); }
};
template <class V, class Ops>
__device__ __forceinline__ V cdot_f(int i, V u, V v, V wz, const Ops& op) {
    V t[3];
    int k = 0;
    if (CX(i) != 0) t[k++] = CX(i) > 0 ? u : cdot_neg(u);
    if (CY(i) != 0) t[k++] = CY(i) > 0 ? v : cdot_neg(v);
    if (CZ(i) != 0) t[k++] = CZ(i) > 0 ? wz : cdot_neg(wz);
    return k == 1 ? t[0] : op.add(t[0], t[1]);
}

// TRT + Guo post-collision values in storage units (lbm.cpp:162-172, deviation
// form), in the form's arithmetic A: the rest population, and one opposite pair
// (i, i+1). srho = S::SC * rho, k15 = 1.5 |u|^2, uF = u . F. FORCE = false
// drops the Guo source terms, which vanish for F = 0.
//
// f+, feq+ and S+ are shared by the pair and the odd parts have opposite signs.
// In FP32 arithmetic every operation is an explicit intrinsic (and the
// constants are formed once on the host), so that every kernel rounds the same
// way: left to the compiler, a*b + c*d may be contracted into an FMA either way
// round, and differently in different kernels.
template <class S, bool FORCE, class A = typename S::A>
__device__ __forceinline__ A rest_post(const Lattice& L, A d0, A dr, A srho, A k15, A uF) {
    using C = Coll<A>;
    if constexpr (sizeof(A) == 4) {
        const float eP = __fmul_rn(C::w(0), __fmaf_rn(-srho, k15, dr));
        const float o = __fmaf_rn(-L.omPf, __fsub_rn(d0, eP), d0);
        return FORCE ? __fmaf_rn(-3.0f * S::SC * L.gPw[0], uF, o) : o;
    } else {
        const A eP = C::w(0) * (dr - srho * k15);
        const A o = d0 - C::omP(L) * (d0 - eP);
        return FORCE ? o - (A)S::SC * C::gP(L) * C::w(0) * A(3) * uF : o;
    }
}
template <class S, bool FORCE, class A = typename S::A>
__device__ __forceinline__ void pair_post(const Lattice& L, int i, A di, A dio, A u, A v, A wz, A dr, A srho, A k15,
                                          A uF, A& oi, A& oo) {
    using C = Coll<A>;
    const A w = C::w(i);
    if constexpr (sizeof(A) == 4) {
        const float cu = cdot_f<float>(i, u, v, wz, ScalarAdd());
        // every operation spelled out, so that no kernel contracts it differently
        const int c = wclass(i);
        const float eP = __fmul_rn(C::w(i), __fmaf_rn(srho, __fmaf_rn(__fmul_rn(4.5f, cu), cu, -k15), dr));
        const float eM = __fmul_rn(__fmul_rn(3.0f * C::w(i), srho), cu);
        const float fP = __fmul_rn(0.5f, __fadd_rn(di, dio)), fM = __fmul_rn(0.5f, __fsub_rn(di, dio));
        float a = __fmul_rn(-L.omPf, __fsub_rn(fP, eP));
        float b = __fmul_rn(-L.omMf, __fsub_rn(fM, eM));
        if (FORCE) {
            a = __fmaf_rn(S::SC * L.gPw[c], __fmaf_rn(__fmul_rn(9.0f, cu), L.cF[i], __fmul_rn(-3.0f, uF)), a);
            b = __fadd_rn(b, S::SC * L.cm[i]);
        }
        oi = __fadd_rn(__fadd_rn(di, a), b);
        oo = __fsub_rn(__fadd_rn(dio, a), b);
    } else {
        const A cu = CX(i) * u + CY(i) * v + CZ(i) * wz;
        const A eP = w * (dr + srho * (A(4.5) * cu * cu - k15));   // feq+ - w, storage units
        const A eM = A(3) * w * srho * cu;                          // feq-
        const A fP = A(0.5) * (di + dio), fM = A(0.5) * (di - dio);
        A a, b;
        if (FORCE) {
            a = (A)S::SC * C::gP(L) * w * (A(9) * cu * C::cF(L, i) - A(3) * uF) - C::omP(L) * (fP - eP);
            b = (A)S::SC * C::cm(L, i) - C::omM(L) * (fM - eM);
        } else {
            a = -C::omP(L) * (fP - eP);
            b = -C::omM(L) * (fM - eM);
        }
        oi = di + a + b;
        oo = dio + a - b;
    }
}

template <class S, bool STREAM, class V>
__device__ __forceinline__ void put_st(typename S::T* p, V v) {
    if constexpr (STREAM) S::st_cs(p, v);
    else S::st(p, v);
}

// Collide and push of a node with only fluid neighbours, in the form's
// arithmetic on its stored numbers: the rest population, then one opposite
// pair at a time; each value is rounded to the storage type once, as stored.
// STREAM: streaming stores (the bulk's nodes, read again only next step, so
// they need not displace the zone's and the squirmer update's data in L2).
template <class S, int PAR, bool FORCE, bool STREAM = false, class A = typename S::A>
__device__ __forceinline__ void plain_pairs(const Lattice& L, typename S::T* __restrict__ f, unsigned N, unsigned n,
                                            const Nbr& nb, const float* d, A dr, A srho, A u, A v, A wz, A uF, A k15,
                                            bool do_mass, NodeSums& out) {
    {   // rest population: c = 0
        const float o0 = (float)rest_post<S, FORCE>(L, (A)d[0], dr, srho, k15, uF);
        put_st<S, STREAM>(f + n, o0);
        if (do_mass) out.mass += (double)S::rt(o0) * S::INV;
    }
#pragma unroll
    for (int i = 1; i < Q; i += 2) {
        const int io = i + 1;
        A ai, ao;
        pair_post<S, FORCE>(L, i, (A)d[i], (A)d[io], u, v, wz, dr, srho, k15, uF, ai, ao);
        const float oi = (float)ai, oo = (float)ao;
        if (PAR == 0) {
            put_st<S, STREAM>(f + (size_t)io * N + n, oi);
            put_st<S, STREAM>(f + (size_t)i * N + n, oo);
        } else {
            put_st<S, STREAM>(f + (size_t)i * N + nb.of(n, i), oi);
            put_st<S, STREAM>(f + (size_t)io * N + nb.of(n, io), oo);
        }
        if (do_mass) out.mass += (double)S::rt(oi) * S::INV + (double)S::rt(oo) * S::INV;
    }
}

// GENERAL: the particle links are not computed here. Their post-collision
// values go to link_stash[i * BOUNDARY_BLOCK + threadIdx.x], their directions
// to out.pmask, and zone_particle_links finishes them with the whole warp.
// FP64 collide and push of a node with only fluid neighbours, in the
// reference's arithmetic (lbm.cpp:162-172, every operation in its order, no
// contraction), one opposite pair (i, i+1) at a time. The terms of i+1 are
// those of i with c -> -c: cu, c.F, feq-, f-, S- change sign exactly and feq+,
// f+, S+ are equal, so they are formed once; fpost_{i+1} adds the negated odd
// terms in the reference's order. The results are the reference's bits
// (where a term is +-0 its sign may differ, which leaves a nonzero sum as it
// is). FORCE = false drops the Guo terms: for F = 0 they are +-0.
template <class S, int PAR, bool FORCE, bool STREAM = false>
__device__ __forceinline__ void plain_pairs_fp64(const Lattice& L, typename S::T* __restrict__ f, unsigned N, unsigned n,
                                                 const Nbr& nb, const double* fv, double r, double u, double v,
                                                 double wz, double usq, double uF, bool do_mass, NodeSums& out) {
    const double Fx = L.F[0], Fy = L.F[1], Fz = L.F[2];
    {   // rest population
        const double cu = CX(0) * u + CY(0) * v + CZ(0) * wz;
        const double cF = CX(0) * Fx + CY(0) * Fy + CZ(0) * Fz;
        const double feqP = WD(0) * r * (1.0 + 4.5 * cu * cu - 1.5 * usq);
        const double feqM = WD(0) * r * 3.0 * cu;
        const double fP = 0.5 * (fv[0] + fv[0]), fM = 0.5 * (fv[0] - fv[0]);
        const double SP = WD(0) * (9.0 * cu * cF - 3.0 * uF), SM = WD(0) * 3.0 * cF;
        const double fpost = FORCE ? fv[0] - L.omP * (fP - feqP) - L.omM * (fM - feqM) + L.gP * SP + L.gM * SM
                                   : fv[0] - L.omP * (fP - feqP) - L.omM * (fM - feqM);
        put_st<S, STREAM>(f + n, fpost);
        if (do_mass) out.mass += fpost;
    }
#pragma unroll
    for (int i = 1; i < Q; i += 2) {
        const int io = i + 1;
        const double cu = CX(i) * u + CY(i) * v + CZ(i) * wz;
        const double feqP = WD(i) * r * (1.0 + 4.5 * cu * cu - 1.5 * usq);
        const double feqM = WD(i) * r * 3.0 * cu;
        const double fP = 0.5 * (fv[i] + fv[io]), fM = 0.5 * (fv[i] - fv[io]);
        const double A = L.omP * (fP - feqP), B = L.omM * (fM - feqM);
        double fi, fo;
        if (FORCE) {
            const double cF = CX(i) * Fx + CY(i) * Fy + CZ(i) * Fz;
            const double SP = WD(i) * (9.0 * cu * cF - 3.0 * uF), SM = WD(i) * 3.0 * cF;
            const double C = L.gP * SP, D = L.gM * SM;
            fi = fv[i] - A - B + C + D;
            fo = fv[io] - A + B + C - D;
        } else {
            fi = fv[i] - A - B;
            fo = fv[io] - A + B;
        }
        if (PAR == 0) {
            put_st<S, STREAM>(f + (size_t)io * N + n, fi);
            put_st<S, STREAM>(f + (size_t)i * N + n, fo);
        } else {
            put_st<S, STREAM>(f + (size_t)i * N + nb.of(n, i), fi);
            put_st<S, STREAM>(f + (size_t)io * N + nb.of(n, io), fo);
        }
        if (do_mass) { out.mass += fi; out.mass += fo; }
    }
}

// The post-collision populations of all 19 directions in the pair form of
// plain_pairs_fp64 (the reference's bits), for the boundary path. The bulk
// keeps its own copy of these lines, which stores each pair as soon as it is
// formed: written through this helper it spills more at 3 CTAs/SM.
template <bool FORCE>
__device__ __forceinline__ void collide_pairs_fp64(const Lattice& L, const double* fv, double r, double u, double v,
                                                   double wz, double usq, double uF, double* post) {
    const double Fx = L.F[0], Fy = L.F[1], Fz = L.F[2];
    {
        const double cu = CX(0) * u + CY(0) * v + CZ(0) * wz;
        const double cF = CX(0) * Fx + CY(0) * Fy + CZ(0) * Fz;
        const double feqP = WD(0) * r * (1.0 + 4.5 * cu * cu - 1.5 * usq);
        const double feqM = WD(0) * r * 3.0 * cu;
        const double fP = 0.5 * (fv[0] + fv[0]), fM = 0.5 * (fv[0] - fv[0]);
        const double SP = WD(0) * (9.0 * cu * cF - 3.0 * uF), SM = WD(0) * 3.0 * cF;
        post[0] = FORCE ? fv[0] - L.omP * (fP - feqP) - L.omM * (fM - feqM) + L.gP * SP + L.gM * SM
                        : fv[0] - L.omP * (fP - feqP) - L.omM * (fM - feqM);
    }
#pragma unroll
    for (int i = 1; i < Q; i += 2) {
        const int io = i + 1;
        const double cu = CX(i) * u + CY(i) * v + CZ(i) * wz;
        const double feqP = WD(i) * r * (1.0 + 4.5 * cu * cu - 1.5 * usq);
        const double feqM = WD(i) * r * 3.0 * cu;
        const double fP = 0.5 * (fv[i] + fv[io]), fM = 0.5 * (fv[i] - fv[io]);
        const double A = L.omP * (fP - feqP), B = L.omM * (fM - feqM);
        if (FORCE) {
            const double cF = CX(i) * Fx + CY(i) * Fy + CZ(i) * Fz;
            const double SP = WD(i) * (9.0 * cu * cF - 3.0 * uF), SM = WD(i) * 3.0 * cF;
            const double C = L.gP * SP, D = L.gM * SM;
            post[i] = fv[i] - A - B + C + D;
            post[io] = fv[io] - A + B + C - D;
        } else {
            post[i] = fv[i] - A - B;
            post[io] = fv[io] - A + B;
        }
    }
}

// STREAM: the plain nodes' stores are streaming stores (plain_pairs).
template <class S, int PAR, bool GENERAL, bool MACRO, bool STREAM = !GENERAL, class Src = GlobalSrc>
__device__ __forceinline__ void update_node(const Lattice& L, const StreamArgs& a, unsigned n, int x, int y, int z,
                                            uint8_t fl, uint8_t wallrow, bool store_rho, NodeSums& out,
                                            const Src& src = Src(), LinkStash<S>* link_stash = nullptr) {
    using T = typename S::T;
    T* __restrict__ f = static_cast<T*>(a.f);
    const unsigned N = L.N;
    const Nbr nb(L, x, y, z);
    // GENERAL: neighbour types from the flag bytes; otherwise only whole wall
    // layers next to the row (wallrow) can be solid.
    const bool boundary = GENERAL ? (fl & (NEAR_WALL | NEAR_PARTICLE)) != 0 : wallrow != 0;
    // GENERAL: the neighbours' types, 2 bits per direction, all read before the
    // first population store (a byte load may alias the stores, so a load
    // inside the direction loop would wait for the stores before it)
    const uint64_t ntypes = GENERAL && boundary ? neighbour_types(L, a.flag, n, nb) : 0ull;
    const SqState* __restrict__ sq = a.sq;
    const bool do_mass = a.do_mass != 0;

    if constexpr (!S::shifted) {
        // ---------------- FP64: the reference's arithmetic ----------------
        double fv[Q];
        src.template load<S, PAR>(f, N, n, nb, fv);
        if (a.apply_corr) {
            const double corr = sq->corr_d;
#pragma unroll
            for (int i = 0; i < Q; ++i) fv[i] += WD(i) * corr;  // LBM::correctMass (lbm.cpp:337)
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
        if (GENERAL) out.rho = r;
        const double usq = u * u + v * v + wz * wz, uF = u * Fx + v * Fy + wz * Fz;
        if (!boundary) {   // every neighbour fluid: the pair form, same bits
            if (L.force_free)
                plain_pairs_fp64<S, PAR, false, STREAM>(L, f, N, n, nb, fv, r, u, v, wz, usq, uF, do_mass, out);
            else
                plain_pairs_fp64<S, PAR, true, STREAM>(L, f, N, n, nb, fv, r, u, v, wz, usq, uF, do_mass, out);
            return;
        }
        // TRT + Guo forcing (lbm.cpp:162-172), in the pair form
        double post[Q];
        if (L.force_free) collide_pairs_fp64<false>(L, fv, r, u, v, wz, usq, uF, post);
        else collide_pairs_fp64<true>(L, fv, r, u, v, wz, usq, uF, post);
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const int io = OPP(i);
            const double fpost = post[i];
            const unsigned nbi = nb.of(n, i);
            T* local = f + (size_t)io * N + n;
            T* remote = f + (size_t)i * N + nbi;
            uint8_t tt = T_FLUID;
            if (boundary && i != 0)
                tt = GENERAL ? (uint8_t)((ntypes >> (2 * i)) & 3u) : (wall_dir(i, wallrow) ? T_WALL : T_FLUID);
            if (tt == T_FLUID) {  // push (lbm.cpp:186)
                S::st(PAR == 0 ? local : remote, fpost);
                if (do_mass) out.mass += fpost;
                continue;
            }
            if (GENERAL && tt == T_PARTICLE) {   // finished by zone_particle_links
                link_stash[i * BOUNDARY_BLOCK + threadIdx.x] = fpost;
                out.pmask |= 1u << i;
                continue;
            }
            // halfway bounce-back at a wall (lbm.cpp:189-199, u_b = 0)
            const double ub[3] = {0, 0, 0};
            const double cub = CX(i) * ub[0] + CY(i) * ub[1] + CZ(i) * ub[2];
            const double fb = fpost - 6.0 * WD(i) * r * cub;
            S::st(PAR == 0 ? remote : local, fb);
            if (do_mass) out.mass += fb;
            // Galilean-invariant momentum exchange (lbm.cpp:202-215)
            const double sm = fpost + fb, dl = fpost - fb;
            const double dpx = sm * CX(i) - dl * ub[0];
            const double dpy = sm * CY(i) - dl * ub[1];
            const double dpz = sm * CZ(i) - dl * ub[2];
            out.fw[0] += dpx; out.fw[1] += dpy; out.fw[2] += dpz;   // only wall links reach here
        }
    } else {
        // ---- shifted forms: stored deviations (storage units), arithmetic S::A ----
        using AR = typename S::A;
        float d[Q];
        src.template load<S, PAR>(f, N, n, nb, d);
        if (a.apply_corr) {
            const double corr = sq->corr_d;
#pragma unroll
            for (int i = 0; i < Q; ++i) d[i] += (float)(WD(i) * corr * S::SC);
        }
        AR dr, rho, u, v, wz;
        shifted_moments<S>(L, d, dr, rho, u, v, wz);
        if (GENERAL) out.rho = (double)rho;
        if (store_rho) a.rho[n] = 1.0 + (double)dr * S::INV;
        if (MACRO) { a.ux[n] = u; a.uy[n] = v; a.uz[n] = wz; }
        AR k15, uF, srho;
        shifted_terms<S>(L, rho, u, v, wz, k15, uF, srho);
        if (!boundary) {
            if (L.force_free)   // uniform: the Guo source terms are exactly zero
                plain_pairs<S, PAR, false, STREAM>(L, f, N, n, nb, d, dr, srho, u, v, wz, uF, k15, do_mass, out);
            else
                plain_pairs<S, PAR, true, STREAM>(L, f, N, n, nb, d, dr, srho, u, v, wz, uF, k15, do_mass, out);
        } else {
            AR post[Q];
            post[0] = rest_post<S, true>(L, (AR)d[0], dr, srho, k15, uF);
#pragma unroll
            for (int i = 1; i < Q; i += 2)
                pair_post<S, true>(L, i, (AR)d[i], (AR)d[i + 1], u, v, wz, dr, srho, k15, uF, post[i], post[i + 1]);
#pragma unroll
            for (int i = 0; i < Q; ++i) {
                const AR dpost = post[i];
                const unsigned nbi = nb.of(n, i);
                T* local = f + (size_t)OPP(i) * N + n;
                T* remote = f + (size_t)i * N + nbi;
                const uint8_t tt = i == 0 ? T_FLUID
                                   : GENERAL ? (uint8_t)((ntypes >> (2 * i)) & 3u)
                                             : (wall_dir(i, wallrow) ? T_WALL : T_FLUID);
                if (tt == T_FLUID) {
                    const float o = (float)dpost;
                    S::st(PAR == 0 ? local : remote, o);
                    if (do_mass) out.mass += (double)S::rt(o) * S::INV;
                    continue;
                }
                if (GENERAL && tt == T_PARTICLE) {   // finished by zone_particle_links
                    link_stash[i * BOUNDARY_BLOCK + threadIdx.x] = dpost;
                    out.pmask |= 1u << i;
                    continue;
                }
                const double ub[3] = {0, 0, 0};   // wall: u_b = 0
                const double cub = CX(i) * ub[0] + CY(i) * ub[1] + CZ(i) * ub[2];
                const double dl = 6.0 * WD(i) * (double)rho * cub;   // fpost - fb (deviation units)
                const float dfb = (float)((double)dpost - dl * S::SC);
                S::st(PAR == 0 ? remote : local, dfb);
                if (do_mass) out.mass += (double)S::rt(dfb) * S::INV;
                const double fpost = WD(i) + (double)dpost * S::INV;
                const double sm = 2.0 * fpost - dl;                   // fpost + fb
                const double dpx = sm * CX(i) - dl * ub[0];
                const double dpy = sm * CY(i) - dl * ub[1];
                const double dpz = sm * CZ(i) - dl * ub[2];
                out.fw[0] += dpx; out.fw[1] += dpy; out.fw[2] += dpz;   // only wall links reach here
            }
        }
    }
}

// Resident 256-thread CTAs per SM the bulk kernels are compiled for: FP32
// arithmetic on stored deviations fits 64 registers (4); FP64 arithmetic on
// FP32 storage spills at 80 and gets 128 (2); the FP64 form keeps 2 unless the
// bulk is long (DENSE, see k_bulk).
template <class S>
__host__ __device__ constexpr int bulk_min_blocks(bool dense) {
    return !S::shifted ? (dense ? 3 : 2) : (sizeof(typename S::A) == 8 ? 2 : 4);
}

// ---------------------------------------------------------------------------
//  k_bulk<S, PAR, SQ, MACRO, WR>: fluid nodes without a PARTICLE neighbour,
//  outside the zone.
//    SQ    the lattice has a squirmer (and hence a zone to skip)
//    MACRO store rho and u of every node (the last step of every host call)
//    WR    false: grid (ceil(nx/TX), ny, nz), rows next to a wall skipped;
//          true : grid (ceil(nx/TX), n_wallrows), only those rows, whose
//                 solid directions follow from (y, z) (bounce-back and the
//                 wall's momentum exchange compiled in only here)
//  block (TX, 1, 1) with TX = 32..256. Block partials are indexed by the row,
//  so the two launches fill disjoint entries of one array. Reads nothing the
//  squirmer update writes (except the correction value on the step after a
//  correction step, when the launch waits for it).
// ---------------------------------------------------------------------------
//    DENSE (FP64 only) 3 CTAs/SM instead of 2 (80 registers, a few spills): for
//          long bulks; a short one leaves room for the zone and squirmer chain
template <class S, int PAR, bool SQ, bool MACRO, bool WR, bool DENSE = false>
__global__ void __launch_bounds__(256, bulk_min_blocks<S>(DENSE)) k_bulk(const Lattice L, const StreamArgs a) {
    pdl_wait();
    pdl_launch_dependents();
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y, z;
    if (WR) { y = a.wallrows[2 * blockIdx.y]; z = a.wallrows[2 * blockIdx.y + 1]; }
    else { y = blockIdx.y; z = blockIdx.z; }
    const uint8_t wr = wall_row(L, y, z);
    if (!WR && wr) return;  // block-uniform: the wall-row launch owns this row and its partials
    const unsigned n = (unsigned)x + (unsigned)L.nx * ((unsigned)y + (unsigned)L.ny * (unsigned)z);
    // FLUID with no PARTICLE neighbour; wall neighbours are whole layers
    bool active = x < L.nx && (a.flag[n] & (uint8_t)~NEAR_WALL) == 0;
    if (SQ && active) active = !in_zone(L, a.sq->zone[a.zslot], x, y, z);
    NodeSums sums;
    if (active) update_node<S, PAR, false, MACRO>(L, a, n, x, y, z, 0, WR ? wr : (uint8_t)0, MACRO, sums);
    if (a.do_mass || MACRO) {
        const unsigned bid = blockIdx.x + gridDim.x * ((unsigned)y + (unsigned)L.ny * (unsigned)z);
        block_reduce4<256>(sums.fw[0], sums.fw[1], sums.fw[2], sums.mass, a.block_part + (size_t)bid * BLOCK_PART);
    }
}

// k_bulk_flat<S, PAR, SQ, DENSE>: the nodes of k_bulk on a step without sums
// (no mass correction, no macroscopic output), for lattices whose nx is not a
// multiple of 32. The rows away from walls of one z-plane are one contiguous
// range of nodes; 256 threads take 256 consecutive nodes of it, so no lane
// idles at a row's end. Grid (ceil(range / 256), planes away from z walls).
template <class S, int PAR, bool SQ, bool DENSE = false>
__global__ void __launch_bounds__(256, bulk_min_blocks<S>(DENSE)) k_bulk_flat(const Lattice L, const StreamArgs a) {
    pdl_wait();
    pdl_launch_dependents();
    const int ylo = L.walls_y ? 2 : 0, rows = L.walls_y ? L.ny - 4 : L.ny;
    const int z = (L.walls_z ? 2 : 0) + (int)blockIdx.y;
    const int o = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (o >= rows * L.nx) return;
    const int dy = o / L.nx;
    const int x = o - dy * L.nx, y = ylo + dy;
    const unsigned n = (unsigned)x + (unsigned)L.nx * ((unsigned)y + (unsigned)L.ny * (unsigned)z);
    bool active = (a.flag[n] & (uint8_t)~NEAR_WALL) == 0;
    if (SQ && active) active = !in_zone(L, a.sq->zone[a.zslot], x, y, z);
    NodeSums sums;
    if (active) update_node<S, PAR, false, false>(L, a, n, x, y, z, 0, 0, false, sums);
}

// ---------------------------------------------------------------------------
//  k_bulk_pair<S, PAR, SQ, FORCE>: the nodes of k_bulk on a step without sums
//  (no mass correction, no macroscopic output) in the shifted forms, two
//  x-adjacent nodes (x0, x0 + 1) per thread, x0 even. Every direction moves
//  both nodes' values with one 2-element load and one 2-element store (8 B in
//  FP32, 4 B in FP16), so a warp touches 64 consecutive nodes of a direction
//  row per instruction. Requires nx a multiple of 64 (whole warps of pairs,
//  aligned vectors); blockDim.x divides nx / 2 (a multiple of 32, at most
//  PAIR_BLOCK), grid (nx / 2 / blockDim.x, ny, nz), rows next to a wall
//  skipped (their own launch).
//
//  Even steps read and write the node's own slots A[i][n], A[opp(i)][n]: both
//  aligned pairs. Odd steps read A[opp(i)][n - c_i] and write A[i][n + c_i],
//  one cell off in x for the directions with c_x != 0. Such a direction is
//  moved as aligned pairs all the same and the x shift made across lanes:
//    load, source x - 1: node x0 takes the previous lane's upper element,
//      x0 + 1 its own lower one; source x + 1: node x0 its own upper element,
//      x0 + 1 the next lane's lower one;
//    store, target x + 1: the aligned pair (x0, x0 + 1) holds the previous
//      lane's x0 - 1 value and this lane's x0 value; target x - 1: this lane's
//      x0 + 1 value and the next lane's x0 + 2 value.
//  A lane whose neighbour in that direction is in another warp, or across the
//  periodic x boundary, loads or stores that element alone. A node that the
//  bulk does not update (the zone, a node next to the sphere) is neither read
//  into nor written by a vector: the pair is split into single elements.
//  The per-node arithmetic is that of update_node's force-free / forced
//  branches (shifted_moments, rest_post, pair_post), so results are those of
//  k_bulk bit for bit.
// ---------------------------------------------------------------------------
constexpr int PAIR_BLOCK = 128;

// A thread's pair of nodes (x0, x0 + 1) in row (y, z), with its neighbours in
// the warp along x: has_prev / has_next = the lane before / after holds the
// pair before / after in the same row (not across a warp or the periodic
// boundary), prev_act1 / next_act0 = that lane's adjacent node is updated by
// the bulk; xm / xp = x0 - 1 and x0 + 2 wrapped.
struct PairRow {
    unsigned row, n0;
    int x0, xm, xp, y, z;
    int yp, ym, zp, zm;   // row offsets of the y/z neighbours (periodic wrap as in Nbr)
    bool act0, act1, prev_act1, next_act0, has_prev, has_next;
    __device__ __forceinline__ PairRow(const Lattice& L, int x0_, int y_, int z_, int lane, bool a0, bool a1)
        : x0(x0_), y(y_), z(z_), act0(a0), act1(a1) {
        row = (unsigned)L.nx * ((unsigned)y + (unsigned)L.ny * (unsigned)z);
        n0 = row + (unsigned)x0;
        has_prev = lane > 0 && x0 > 0;
        has_next = lane < 31 && x0 + 2 < L.nx;
        prev_act1 = __shfl_up_sync(0xffffffffu, act1, 1) && has_prev;
        next_act0 = __shfl_down_sync(0xffffffffu, act0, 1) && has_next;
        xm = x0 == 0 ? L.nx - 1 : x0 - 1;
        xp = x0 + 2 == L.nx ? 0 : x0 + 2;
        yp = (y == L.ny - 1) ? (1 - L.ny) * L.nx : L.nx;
        ym = (y == 0) ? (L.ny - 1) * L.nx : -L.nx;
        zp = (z == L.nz - 1) ? (1 - L.nz) * (int)L.nxy : (int)L.nxy;
        zm = (z == 0) ? (L.nz - 1) * (int)L.nxy : -(int)L.nxy;
    }
    __device__ __forceinline__ int ryz(int i) const {   // row offset of n + c_i in y and z
        return (CY(i) > 0 ? yp : (CY(i) < 0 ? ym : 0)) + (CZ(i) > 0 ? zp : (CZ(i) < 0 ? zm : 0));
    }
};

// Collision of a thread's two nodes x0, x0 + 1 from their 19 logical stored
// numbers d0, d1; put(i, a0, a1) receives the post-collision values of
// direction i of both nodes, rounded to the FP32 they are stored through.
template <class S, int PAR, bool FORCE, class Put>
__device__ __forceinline__ void pair_collide(const Lattice& L, const StreamArgs& a, float* d0, float* d1, Put&& put) {
    if (a.apply_corr) {
        const double corr = a.sq->corr_d;
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const float c = (float)(WD(i) * corr * S::SC);
            d0[i] += c; d1[i] += c;
        }
    }
    using AR = typename S::A;
    if constexpr (sizeof(AR) == 4) {
        // FP32 arithmetic: the moments and per-node terms node by node, then
        // the collision of both nodes at once in paired FMAs (Paired), the
        // operations of rest_post and pair_post<float> in their order, so
        // each node's values are those of the one-node kernels bit for bit.
        float dr0, rho0, u0, v0, w0, dr1, rho1, u1, v1, w1;
        shifted_moments<S>(L, d0, dr0, rho0, u0, v0, w0);
        shifted_moments<S>(L, d1, dr1, rho1, u1, v1, w1);
        float k0, k1, uF0, uF1, sr0, sr1;
        shifted_terms<S>(L, rho0, u0, v0, w0, k0, uF0, sr0);
        shifted_terms<S>(L, rho1, u1, v1, w1, k1, uF1, sr1);
        const Paired op(L);
        const float2 dr = make_float2(dr0, dr1), u = make_float2(u0, u1), v = make_float2(v0, v1),
                     wz = make_float2(w0, w1), k15 = make_float2(k0, k1), uF = make_float2(uF0, uF1),
                     srho = make_float2(sr0, sr1);
        {   // rest population
            const float2 d = make_float2(d0[0], d1[0]);
            const float2 eP = op.mul(bc2(WF(0)), fma2(neg2(srho), k15, dr));
            float2 o = fma2(bc2(-L.omPf), op.sub(d, eP), d);
            if (FORCE) o = fma2(bc2(-3.0f * S::SC * L.gPw[0]), uF, o);
            put(0, o.x, o.y);
        }
#pragma unroll
        for (int i = 1; i < Q; i += 2) {
            const float2 di = make_float2(d0[i], d1[i]), dio = make_float2(d0[i + 1], d1[i + 1]);
            const float2 cu = cdot_f<float2>(i, u, v, wz, op);
            const float2 eP = op.mul(bc2(WF(i)), fma2(srho, fma2(op.mul(bc2(4.5f), cu), cu, neg2(k15)), dr));
            const float2 eM = op.mul(op.mul(bc2(3.0f * WF(i)), srho), cu);
            const float2 fP = op.mul(bc2(0.5f), op.add(di, dio));
            const float2 fM = op.mul(bc2(0.5f), op.sub(di, dio));
            float2 ta = op.mul(bc2(-L.omPf), op.sub(fP, eP));
            float2 tb = op.mul(bc2(-L.omMf), op.sub(fM, eM));
            if (FORCE) {
                ta = fma2(bc2(S::SC * L.gPw[wclass(i)]),
                          fma2(op.mul(bc2(9.0f), cu), bc2(L.cF[i]), op.mul(bc2(-3.0f), uF)), ta);
                tb = op.add(tb, bc2(S::SC * L.cm[i]));
            }
            const float2 oi = op.add(op.add(di, ta), tb);
            const float2 oo = op.sub(op.add(dio, ta), tb);
            put(i, oi.x, oi.y);
            put(i + 1, oo.x, oo.y);
        }
        return;
    }
    AR dr0, rho0, u0, v0, w0, dr1, rho1, u1, v1, w1;
    shifted_moments<S>(L, d0, dr0, rho0, u0, v0, w0);
    shifted_moments<S>(L, d1, dr1, rho1, u1, v1, w1);
    AR k0, k1, uF0, uF1, sr0, sr1;
    shifted_terms<S>(L, rho0, u0, v0, w0, k0, uF0, sr0);
    shifted_terms<S>(L, rho1, u1, v1, w1, k1, uF1, sr1);
    put(0, (float)rest_post<S, FORCE>(L, (AR)d0[0], dr0, sr0, k0, uF0),
        (float)rest_post<S, FORCE>(L, (AR)d1[0], dr1, sr1, k1, uF1));
#pragma unroll
    for (int i = 1; i < Q; i += 2) {
        AR a0i, a0o, a1i, a1o;
        pair_post<S, FORCE>(L, i, (AR)d0[i], (AR)d0[i + 1], u0, v0, w0, dr0, sr0, k0, uF0, a0i, a0o);
        pair_post<S, FORCE>(L, i, (AR)d1[i], (AR)d1[i + 1], u1, v1, w1, dr1, sr1, k1, uF1, a1i, a1o);
        // direction i's post value goes where the next state reads logical
        // f_i: even step -> A[opp(i)][n]; odd step -> A[i][n + c_i]
        put(i, (float)a0i, (float)a1i);
        put(i + 1, (float)a0o, (float)a1o);
    }
}

// Collide and store of a thread's two nodes (the second half of k_bulk_pair,
// shared with the staged two-node kernel): d0, d1 are the 19 logical stored
// numbers of x0 and x0 + 1. Every lane of the warp calls it (the stores
// shuffle the x-shifted values between lanes).
template <class S, int PAR, bool FORCE>
__device__ __forceinline__ void pair_collide_store(const Lattice& L, const StreamArgs& a, typename S::T* __restrict__ f,
                                                   const PairRow& pr, float* d0, float* d1) {
    using T = typename S::T;
    const unsigned N = L.N;
    const int x0 = pr.x0;
    const bool act0 = pr.act0, act1 = pr.act1;

    // post-collision value of direction i to its slot; (a0, a1) = the values
    // of nodes x0, x0 + 1, already rounded to the FP32 they are stored through
    auto put = [&](int i, float a0, float a1) {
        if (PAR == 0) {                                        // A[opp(i)][n]
            T* p = f + (size_t)OPP(i) * N + pr.n0;
            if (act0 && act1) S::st2_cs(p, a0, a1);
            else { if (act0) S::st_cs(p, a0); if (act1) S::st_cs(p + 1, a1); }
            return;
        }
        T* rowp = f + (size_t)i * N + (size_t)((int)pr.row + pr.ryz(i));   // A[i][n + c_i]
        if (CX(i) == 0) {
            if (act0 && act1) S::st2_cs(rowp + x0, a0, a1);
            else { if (act0) S::st_cs(rowp + x0, a0); if (act1) S::st_cs(rowp + x0 + 1, a1); }
        } else if (CX(i) > 0) {                                // targets x0 + 1, x0 + 2
            const float pv = __shfl_up_sync(0xffffffffu, a1, 1);
            if (pr.prev_act1 && act0) S::st2_cs(rowp + x0, pv, a0);
            else { if (pr.prev_act1) S::st_cs(rowp + x0, pv); if (act0) S::st_cs(rowp + x0 + 1, a0); }
            if (!pr.has_next && act1) S::st_cs(rowp + pr.xp, a1);
        } else {                                               // targets x0 - 1, x0
            const float nv = __shfl_down_sync(0xffffffffu, a0, 1);
            if (act1 && pr.next_act0) S::st2_cs(rowp + x0, a1, nv);
            else { if (act1) S::st_cs(rowp + x0, a1); if (pr.next_act0) S::st_cs(rowp + x0 + 1, nv); }
            if (!pr.has_prev && act0) S::st_cs(rowp + pr.xm, a0);
        }
    };
    pair_collide<S, PAR, FORCE>(L, a, d0, d1, put);
}

template <class S, int PAR, bool SQ, bool FORCE>
__global__ void __launch_bounds__(PAIR_BLOCK, 4) k_bulk_pair(const Lattice L, const StreamArgs a) {
    using T = typename S::T;
    pdl_wait();
    pdl_launch_dependents();
    const int y = blockIdx.y, z = blockIdx.z;
    if (wall_row(L, y, z)) return;   // block-uniform: the wall-row launch owns this row
    T* __restrict__ f = static_cast<T*>(a.f);
    const unsigned N = L.N;
    const int lane = threadIdx.x & 31;
    const int x0 = 2 * (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const unsigned n0 = (unsigned)L.nx * ((unsigned)y + (unsigned)L.ny * (unsigned)z) + (unsigned)x0;
    bool act0 = (a.flag[n0] & (uint8_t)~NEAR_WALL) == 0;
    bool act1 = (a.flag[n0 + 1] & (uint8_t)~NEAR_WALL) == 0;
    if (SQ) {
        const ZoneBox zb = a.sq->zone[a.zslot];
        act0 = act0 && !in_zone(L, zb, x0, y, z);
        act1 = act1 && !in_zone(L, zb, x0 + 1, y, z);
    }
    const PairRow pr(L, x0, y, z, lane, act0, act1);

    // ---- loads: logical f_i of both nodes ----
    float d0[Q], d1[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        if (PAR == 0) {
            const float2 q = S::ld2(f + (size_t)i * N + n0);
            d0[i] = q.x; d1[i] = q.y;
        } else {
            const int o = OPP(i);                              // read A[o][n + c_o]
            const T* rowp = f + (size_t)o * N + (size_t)((int)pr.row + pr.ryz(o));
            const float2 q = S::ld2(rowp + x0);
            if (CX(o) == 0) {
                d0[i] = q.x; d1[i] = q.y;
            } else if (CX(o) < 0) {                            // source x - 1
                const float up = __shfl_up_sync(0xffffffffu, q.y, 1);
                d0[i] = pr.has_prev ? up : S::ld(rowp + pr.xm);
                d1[i] = q.x;
            } else {                                           // source x + 1
                const float dn = __shfl_down_sync(0xffffffffu, q.x, 1);
                d0[i] = q.y;
                d1[i] = pr.has_next ? dn : S::ld(rowp + pr.xp);
            }
        }
    }
    pair_collide_store<S, PAR, FORCE>(L, a, f, pr, d0, d1);
}

// ---------------------------------------------------------------------------
//  k_zone<S, PAR, SQ, MACRO>: thread k updates the fluid node at cell k of the
//  zone (row-major, x fastest). Zone nodes store rho every step (the refill of
//  the next remap reads it) and write one row of link_part per near-particle
//  node; wall force and mass go to block partials.
// ---------------------------------------------------------------------------
// The particle links left by update_node<GENERAL> (lbm.cpp:189-215 with u_b
// = U + W x r_b + slip, r_b at the link midpoint), finished by the whole warp
// (every lane calls it): in round k each lane takes its k-th link in
// ascending direction order, so the warp runs as many rounds as its busiest
// lane has links instead of one pass per direction that any lane needs. The
// arithmetic and the order of the per-node sums are those of the direction
// loop in update_node.
template <class S, int PAR>
__device__ __forceinline__ void zone_particle_links(const Lattice& L, const StreamArgs& a, const SqState* sq,
                                                    unsigned n, int x, int y, int z, bool do_mass,
                                                    const LinkStash<S>* stash, NodeSums& out) {
    using T = typename S::T;
    T* __restrict__ f = static_cast<T*>(a.f);
    unsigned m = out.pmask;
    const int rounds = __reduce_max_sync(0xffffffffu, (unsigned)__popc(m));
    for (int k = 0; k < rounds; ++k) {
        if (!m) continue;
        const int i = __ffs(m) - 1;
        m &= m - 1;
        const int cx = c_cx[i], cy = c_cy[i], cz = c_cz[i];
        const double w = c_w[i];
        T* local = f + (size_t)opp_rt(i) * L.N + n;
        T* remote = f + (size_t)i * L.N + nbr_rt(L, x, y, z, cx, cy, cz);
        double rb[3], ub[3];
        offset_from_squirmer(L, sq, x + 0.5 * cx, y + 0.5 * cy, z + 0.5 * cz, rb);
        surface_velocity(sq, rb, ub, true);
        const double cub = cx * ub[0] + cy * ub[1] + cz * ub[2];
        double sm, dl;
        if constexpr (!S::shifted) {
            const double fpost = stash[i * BOUNDARY_BLOCK + threadIdx.x];
            const double fb = fpost - 6.0 * w * out.rho * cub;
            S::st(PAR == 0 ? remote : local, fb);
            if (do_mass) out.mass += fb;
            sm = fpost + fb;
            dl = fpost - fb;
        } else {
            const float dpost = stash[i * BOUNDARY_BLOCK + threadIdx.x];   // storage units
            dl = 6.0 * w * out.rho * cub;   // fpost - fb (deviation units)
            const float dfb = (float)((double)dpost - dl * S::SC);
            S::st(PAR == 0 ? remote : local, dfb);
            if (do_mass) out.mass += (double)S::rt(dfb) * S::INV;
            const double fpost = w + (double)dpost * S::INV;
            sm = 2.0 * fpost - dl;            // fpost + fb
        }
        const double dpx = sm * cx - dl * ub[0];
        const double dpy = sm * cy - dl * ub[1];
        const double dpz = sm * cz - dl * ub[2];
        out.fp[0] += dpx; out.fp[1] += dpy; out.fp[2] += dpz;
        out.tp[0] += rb[1] * dpz - rb[2] * dpy;
        out.tp[1] += rb[2] * dpx - rb[0] * dpz;
        out.tp[2] += rb[0] * dpy - rb[1] * dpx;
    }
}

// Cell k of the zone, one per thread (every thread of the block calls it);
// returns the sums for the block reduction. sq is the block's copy of the
// squirmer state, stash the block's particle-link values.
template <class S, int PAR, bool SQ, bool MACRO>
__device__ __forceinline__ void zone_cell(const Lattice& L, const StreamArgs& a, int k, NodeSums& sums,
                                          const SqState* sq, LinkStash<S>* stash) {
    bool active = false;
    unsigned n = 0;
    int x = 0, y = 0, z = 0;
    if (SQ && k < a.zone_cells) {
        const ZoneBox* zb = &sq->zone[a.zslot];
        const int bx = k % a.zw[0], by = (k / a.zw[0]) % a.zw[1], bz = k / (a.zw[0] * a.zw[1]);
        x = zb->lo[0] + bx; if (x >= L.nx) x -= L.nx;
        y = zb->lo[1] + by; z = zb->lo[2] + bz;
        if (L.walls_y) active = y >= 0 && y < L.ny; else { if (y >= L.ny) y -= L.ny; active = true; }
        if (L.walls_z) active = active && z >= 0 && z < L.nz; else if (z >= L.nz) z -= L.nz;
        if (active) {
            n = (unsigned)x + (unsigned)L.nx * ((unsigned)y + (unsigned)L.ny * (unsigned)z);
            active = (a.flag[n] & TYPE_MASK) == T_FLUID;
        }
    }
    uint8_t fl = 0;
    if (active) {
        fl = a.flag[n];
        update_node<S, PAR, true, MACRO>(L, a, n, x, y, z, fl, 0, SQ || MACRO, sums, GlobalSrc(), stash);
    }
    if (SQ) {
        zone_particle_links<S, PAR>(L, a, sq, n, x, y, z, a.do_mass != 0, stash, sums);
        if (active && (fl & NEAR_PARTICLE)) {
            double* lp = a.link_part + (size_t)a.linkslot[n] * LINK_PART;
            lp[0] = sums.fp[0]; lp[1] = sums.fp[1]; lp[2] = sums.fp[2];
            lp[3] = sums.tp[0]; lp[4] = sums.tp[1]; lp[5] = sums.tp[2];
        }
    }
}

// The squirmer state, word by word, into a block's shared copy.
__device__ __forceinline__ void copy_sq_state(SqState* dst, const SqState* src) {
    constexpr int NS = (int)(sizeof(SqState) / 4);
    static_assert(sizeof(SqState) % 4 == 0, "whole words");
    for (int k = (int)threadIdx.x; k < NS; k += (int)blockDim.x)
        reinterpret_cast<uint32_t*>(dst)[k] = reinterpret_cast<const uint32_t*>(src)[k];
}

template <class S, int PAR, bool SQ, bool MACRO>
__global__ void __maxnreg__(ZONE_MAX_REGS) k_zone(const Lattice L, const StreamArgs a) {
    pdl_wait();
    pdl_launch_dependents();
    __shared__ __align__(16) SqState zsq;
    __shared__ LinkStash<S> stash[Q * BOUNDARY_BLOCK];
    if (SQ) copy_sq_state(&zsq, a.sq);
    __syncthreads();
    NodeSums sums;
    zone_cell<S, PAR, SQ, MACRO>(L, a, blockIdx.x * BOUNDARY_BLOCK + threadIdx.x, sums, &zsq, stash);
    if (MACRO || a.do_mass)
        block_reduce4<BOUNDARY_BLOCK>(sums.fw[0], sums.fw[1], sums.fw[2], sums.mass,
                                      a.block_part_b + (size_t)blockIdx.x * BLOCK_PART);
}

}  // namespace lbmgpu
