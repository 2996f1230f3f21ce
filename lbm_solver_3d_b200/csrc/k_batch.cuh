// ============================================================================
//  k_batch.cuh -- the time step of an ensemble of independent lattices
//  ("members": slit channels of uneven sizes, each with its own squirmer),
//  advanced together. The populations of all members live in one packed pool;
//  each member has its own lattice record and arguments in device tables.
//
//    k_bulk_batch  one persistent launch over the x-rows of every member.
//                  TX threads cover a row (cells per thread = ceil(nx/TX)),
//                  256/TX rows are in flight per CTA, the grid is a multiple
//                  of the SM count; TX and the CTAs per SM are chosen by the
//                  autotuner (lbmgpu_batch_autotune). Per-row partial sums
//                  (wall force, mass) keep every member's reductions separate
//                  and in a fixed order.
//    k_zone_batch  the zones of all members, grid (zone blocks, members).
//    k_squirmer_batch (k_squirmer.cuh) one CTA per member.
//  The members share the fluid parameters (tau, Lambda, body force, walls,
//  storage form, mass-correction interval); geometry and squirmer differ.
// ============================================================================
#pragma once
#include "k_stream.cuh"

namespace lbmgpu {


// Rows of at most BATCH_MAX_NX nodes: the partial sums of a row are formed
// exactly as k_bulk forms them for a row held by one block of ceil32(nx)
// threads (one node per thread, a shuffle tree per 32 nodes, the warps' sums
// added in order), so a member's mass correction and wall force equal those of
// the same lattice run alone, bit for bit.
constexpr int BATCH_CHUNKS = BATCH_MAX_NX / 32;

__device__ __forceinline__ void chunk_reduce(NodeSums& s) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s.fw[0] += __shfl_down_sync(0xffffffffu, s.fw[0], o);
        s.fw[1] += __shfl_down_sync(0xffffffffu, s.fw[1], o);
        s.fw[2] += __shfl_down_sync(0xffffffffu, s.fw[2], o);
        s.mass += __shfl_down_sync(0xffffffffu, s.mass, o);
    }
}

template <class S, int PAR, bool MACRO, bool WR, int TX>
__global__ void __launch_bounds__(256) k_bulk_batch(const Lattice* __restrict__ lat, const StreamArgs* __restrict__ args,
                                                    const RowRef* __restrict__ rows, int nrows,
                                                    double* __restrict__ row_part, BatchStep st) {
    constexpr int RB = 256 / TX;
    __shared__ Lattice sL[RB];
    __shared__ StreamArgs sA[RB];
    __shared__ ZoneBox sZ[RB];
    __shared__ int sY[RB], sZc[RB], sP[RB];
    __shared__ double red[RB][BATCH_CHUNKS][4];
    const int slot = threadIdx.x / TX, lane = threadIdx.x % TX;
    const bool sums_on = st.do_mass || MACRO;
    int cur_m = -1;   // member whose records the slot holds (rows come grouped by member)
    for (int base = blockIdx.x * RB; base < nrows; base += gridDim.x * RB) {
        const int r = base + slot;
        if (lane == 0 && r < nrows) {
            const RowRef rr = rows[r];
            if (rr.m != cur_m) {
                cur_m = rr.m;
                sL[slot] = lat[rr.m];
                StreamArgs a = args[rr.m];
                a.zslot = st.zslot; a.do_mass = st.do_mass; a.apply_corr = st.apply_corr;
                sA[slot] = a;
                sZ[slot] = a.sq->zone[st.zslot];
            }
            sY[slot] = rr.y; sZc[slot] = rr.z; sP[slot] = rr.part;
        }
        __syncthreads();
        if (r < nrows) {   // uniform over the row's warps
            const Lattice& L = sL[slot];
            const StreamArgs& a = sA[slot];
            const int y = sY[slot], z = sZc[slot];
            const uint8_t wr = WR ? wall_row(L, y, z) : (uint8_t)0;
            const int nxr = (L.nx + 31) & ~31;
            for (int x = lane; x < nxr; x += TX) {
                NodeSums sums;
                if (x < L.nx) {
                    const unsigned n = (unsigned)x + (unsigned)L.nx * ((unsigned)y + (unsigned)L.ny * (unsigned)z);
                    const bool active = (a.flag[n] & (uint8_t)~NEAR_WALL) == 0 && !in_zone(L, sZ[slot], x, y, z);
                    if (active) update_node<S, PAR, false, MACRO>(L, a, n, x, y, z, 0, wr, MACRO, sums);
                }
                if (sums_on) {
                    chunk_reduce(sums);
                    if ((x & 31) == 0) {
                        double* c = red[slot][x >> 5];
                        c[0] = sums.fw[0]; c[1] = sums.fw[1]; c[2] = sums.fw[2]; c[3] = sums.mass;
                    }
                }
            }
        }
        __syncthreads();
        if (sums_on && lane == 0 && r < nrows) {
            const int nch = (sL[slot].nx + 31) >> 5;
            double t0 = 0, t1 = 0, t2 = 0, t3 = 0;
            for (int k = 0; k < nch; ++k) {
                t0 += red[slot][k][0]; t1 += red[slot][k][1]; t2 += red[slot][k][2]; t3 += red[slot][k][3];
            }
            double* out = row_part + (size_t)sP[slot] * BLOCK_PART;
            out[0] = t0; out[1] = t1; out[2] = t2; out[3] = t3;
        }
        __syncthreads();   // the shared row records are rewritten next iteration
    }
}

template <class S, int PAR, bool MACRO>
__global__ void __launch_bounds__(BOUNDARY_BLOCK) k_zone_batch(const Lattice* __restrict__ lat,
                                                               const StreamArgs* __restrict__ args,
                                                               double* __restrict__ zone_part, int gzmax, BatchStep st) {
    __shared__ Lattice L;
    __shared__ StreamArgs A;
    const int m = blockIdx.y;
    if (threadIdx.x == 0) {
        L = lat[m];
        StreamArgs a = args[m];
        a.zslot = st.zslot; a.do_mass = st.do_mass; a.apply_corr = st.apply_corr;
        A = a;
    }
    __syncthreads();
    if ((int)(blockIdx.x * BOUNDARY_BLOCK) >= A.zone_cells) return;  // block-uniform
    NodeSums sums;
    zone_cell<S, PAR, true, MACRO>(L, A, blockIdx.x * BOUNDARY_BLOCK + threadIdx.x, sums);
    if (MACRO || st.do_mass)
        block_reduce4<BOUNDARY_BLOCK>(sums.fw[0], sums.fw[1], sums.fw[2], sums.mass,
                                      zone_part + ((size_t)m * gzmax + blockIdx.x) * BLOCK_PART);
}

}  // namespace lbmgpu
