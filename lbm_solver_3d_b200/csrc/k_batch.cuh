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

// ---------------------------------------------------------------------------
//  k_bulk_rowcta<S, PAR, MACRO>: the rows away from walls, one CTA of
//  ROWCTA_THREADS threads per row (grid = rows; the hardware scheduler keeps
//  the SMs full, as for k_bulk on a single lattice). Warp 0 copies the row's
//  member records into shared memory; nodes x = tid, tid + ROWCTA_THREADS.
//  Row partial sums are formed as in k_bulk_batch.
// ---------------------------------------------------------------------------
constexpr int ROWCTA_THREADS = 128;

template <class S, int PAR, bool MACRO>
__global__ void __launch_bounds__(ROWCTA_THREADS) k_bulk_rowcta(const Lattice* __restrict__ lat,
                                                                const StreamArgs* __restrict__ args,
                                                                const RowRef* __restrict__ rows,
                                                                double* __restrict__ row_part, BatchStep st) {
    __shared__ __align__(16) Lattice sL;
    __shared__ __align__(16) StreamArgs sA;
    __shared__ ZoneBox sZ;
    __shared__ double red[BATCH_CHUNKS][4];
    const int tid = threadIdx.x, lane = tid & 31;
    const RowRef rr = rows[blockIdx.x];   // uniform: one row per CTA
    if (tid < 32) {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(lat + rr.m);
        uint32_t* dst = reinterpret_cast<uint32_t*>(&sL);
        for (int k = lane; k < (int)(sizeof(Lattice) / 4); k += 32) dst[k] = src[k];
        const uint32_t* srca = reinterpret_cast<const uint32_t*>(args + rr.m);
        uint32_t* dsta = reinterpret_cast<uint32_t*>(&sA);
        for (int k = lane; k < (int)(sizeof(StreamArgs) / 4); k += 32) dsta[k] = srca[k];
        if (lane == 0) sZ = args[rr.m].sq->zone[st.zslot];
        __syncwarp();
        if (lane == 0) { sA.zslot = st.zslot; sA.do_mass = st.do_mass; sA.apply_corr = st.apply_corr; }
    }
    __syncthreads();
    const bool sums_on = st.do_mass || MACRO;
    const Lattice& L = sL;
    const int y = rr.y, z = rr.z;
    const int nxr = (L.nx + 31) & ~31;
    for (int x = tid; x < nxr; x += ROWCTA_THREADS) {
        NodeSums sums;
        if (x < L.nx) {
            const unsigned n = (unsigned)x + (unsigned)L.nx * ((unsigned)y + (unsigned)L.ny * (unsigned)z);
            const bool active = (sA.flag[n] & (uint8_t)~NEAR_WALL) == 0 && !in_zone(L, sZ, x, y, z);
            if (active) update_node<S, PAR, false, MACRO>(L, sA, n, x, y, z, 0, 0, MACRO, sums);
        }
        if (sums_on) {
            chunk_reduce(sums);
            if (lane == 0) {
                double* c = red[x >> 5];
                c[0] = sums.fw[0]; c[1] = sums.fw[1]; c[2] = sums.fw[2]; c[3] = sums.mass;
            }
        }
    }
    if (sums_on) {
        __syncthreads();
        if (tid == 0) {
            const int nch = nxr >> 5;
            double t0 = 0, t1 = 0, t2 = 0, t3 = 0;
            for (int c = 0; c < nch; ++c) { t0 += red[c][0]; t1 += red[c][1]; t2 += red[c][2]; t3 += red[c][3]; }
            double* out = row_part + (size_t)rr.part * BLOCK_PART;
            out[0] = t0; out[1] = t1; out[2] = t2; out[3] = t3;
        }
    }
}

// ---------------------------------------------------------------------------
//  k_bulk_staged<S, PAR, MACRO, NST>: the rows away from walls, like
//  k_bulk_batch, with the populations staged through shared memory.
//
//  CTA c owns the contiguous rows [bounds[c], bounds[c+1]) of the row list
//  (balanced by node count on the host) and walks them in order through NST
//  stages. A stage holds the 19 direction-rows one row reads: for an even
//  step A[i] of the row itself, for an odd step A[opp(i)] of the row
//  (y - cy_i, z - cz_i), each a whole x-row. Thread 0 fills a stage with 19
//  bulk asynchronous copies (cp.async.bulk, global -> shared, no multicast)
//  that complete on the stage's mbarrier; the copy of each direction-row
//  starts at the 16-byte boundary below it and is rounded up to 16 bytes, so
//  it may read up to 15 bytes either side of the row (inside the population
//  allocation, whose size is a multiple of 256 bytes). While a row is updated
//  from its stage, the next NST - 1 rows are in flight, so the bytes in
//  flight per SM sit in shared memory rather than in registers.
//  Results are stored straight to global memory. Row partial sums are formed
//  as in k_bulk_batch (bit-identical to a lattice run alone).
//  Waits are bounded: a stage that does not arrive sets ST_WATCHDOG in the
//  member's status word and the CTA stops.
// ---------------------------------------------------------------------------
constexpr int STAGED_THREADS = 128;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* m, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* m, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(m)), "r"(bytes) : "memory");
}
// true once the phase with the given parity has completed; false after the
// iteration limit (each try_wait also suspends for a while in hardware)
__device__ __forceinline__ bool mbar_wait(uint64_t* m, uint32_t parity) {
    const uint32_t a = smem_u32(m);
    for (int it = 0; it < (1 << 22); ++it) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* m) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(m))
                 : "memory");
}

// populations of node x from a stage (see update_node's Src parameter)
template <class T>
struct StagedSrc {
    const T* sb;        // the stage: Q direction-rows of cap elements
    const int* off;     // element offset of each direction-row in its slot
    int cap, x, nx;
    template <class S, int PAR, class V>
    __device__ __forceinline__ void load(const T*, unsigned, unsigned, const Nbr&, V* v) const {
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            int xs = x;
            if (PAR == 1) {
                xs = x - CX(i);
                if (xs < 0) xs += nx; else if (xs >= nx) xs -= nx;
            }
            v[i] = (V)S::ld(sb + i * cap + off[i] + xs);
        }
    }
};

template <class S, int PAR>
__device__ __forceinline__ void stage_issue(typename S::T* sb, uint64_t* mbar, int* off, const Lattice& L,
                                            const StreamArgs& a, int y, int z, int cap) {
    using T = typename S::T;
    const T* f = static_cast<const T*>(a.f);
    uintptr_t start[Q];
    unsigned bytes[Q], total = 0;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        int ys = y, zs = z, arr = i;
        if (PAR == 1) {
            arr = OPP(i);
            ys = y - CY(i); if (ys < 0) ys += L.ny; else if (ys >= L.ny) ys -= L.ny;
            zs = z - CZ(i); if (zs < 0) zs += L.nz; else if (zs >= L.nz) zs -= L.nz;
        }
        const uintptr_t src = reinterpret_cast<uintptr_t>(f + (size_t)arr * L.N + (size_t)L.nx * (ys + (size_t)L.ny * zs));
        start[i] = src & ~(uintptr_t)15;
        off[i] = (int)((src - start[i]) / sizeof(T));
        bytes[i] = (unsigned)(((src + (uintptr_t)L.nx * sizeof(T) - start[i]) + 15) & ~(uintptr_t)15);
        total += bytes[i];
    }
    mbar_expect_tx(mbar, total);
#pragma unroll
    for (int i = 0; i < Q; ++i) bulk_g2s(sb + (size_t)i * cap, reinterpret_cast<const void*>(start[i]), bytes[i], mbar);
}

template <class S, int PAR, bool MACRO, int NST>
__global__ void __launch_bounds__(STAGED_THREADS) k_bulk_staged(const Lattice* __restrict__ lat,
                                                                const StreamArgs* __restrict__ args,
                                                                const RowRef* __restrict__ rows,
                                                                const int* __restrict__ bounds,
                                                                double* __restrict__ row_part, BatchStep st, int cap) {
    using T = typename S::T;
    extern __shared__ __align__(128) unsigned char staged_raw[];
    T* const buf = reinterpret_cast<T*>(staged_raw);
    __shared__ __align__(8) uint64_t mbar[NST];
    __shared__ Lattice sL[NST];
    __shared__ StreamArgs sA[NST];
    __shared__ ZoneBox sZ[NST];
    __shared__ int sY[NST], sZc[NST], sP[NST], sOff[NST][Q];
    __shared__ double red[2][BATCH_CHUNKS][4];
    __shared__ int s_abort;
    const int tid = threadIdx.x, lane = tid & 31;
    const int r0 = bounds[blockIdx.x], r1 = bounds[blockIdx.x + 1];
    const bool sums_on = st.do_mass || MACRO;

    auto issue = [&](int r, int s) {   // thread 0 only
        const RowRef rr = rows[r];
        sL[s] = lat[rr.m];
        StreamArgs a = args[rr.m];
        a.zslot = st.zslot; a.do_mass = st.do_mass; a.apply_corr = st.apply_corr;
        sA[s] = a;
        sZ[s] = a.sq->zone[st.zslot];
        sY[s] = rr.y; sZc[s] = rr.z; sP[s] = rr.part;
        stage_issue<S, PAR>(buf + (size_t)s * Q * cap, &mbar[s], sOff[s], sL[s], a, rr.y, rr.z, cap);
    };

    if (tid == 0) {
        for (int s = 0; s < NST; ++s) mbar_init(&mbar[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
    }
    __syncthreads();
    if (tid == 0)
        for (int k = 0; k < NST && r0 + k < r1; ++k) issue(r0 + k, k);

    uint32_t parity = 0;   // bit s: parity of the next phase of stage s
    for (int r = r0, k = 0; r < r1; ++r, ++k) {
        const int s = k % NST;
        const bool ok = mbar_wait(&mbar[s], (parity >> s) & 1u);
        parity ^= 1u << s;
        if (!ok) {
            s_abort = 1;
        } else {
            const Lattice& L = sL[s];
            const StreamArgs& a = sA[s];
            const int y = sY[s], z = sZc[s];
            const T* sb = buf + (size_t)s * Q * cap;
            const int nxr = (L.nx + 31) & ~31;
            for (int x = tid; x < nxr; x += STAGED_THREADS) {
                NodeSums sums;
                if (x < L.nx) {
                    const unsigned n = (unsigned)x + (unsigned)L.nx * ((unsigned)y + (unsigned)L.ny * (unsigned)z);
                    const bool active = (a.flag[n] & (uint8_t)~NEAR_WALL) == 0 && !in_zone(L, sZ[s], x, y, z);
                    if (active)
                        update_node<S, PAR, false, MACRO>(L, a, n, x, y, z, 0, 0, MACRO, sums,
                                                          StagedSrc<T>{sb, sOff[s], cap, x, L.nx});
                }
                if (sums_on) {
                    chunk_reduce(sums);
                    if (lane == 0) {
                        double* c = red[k & 1][x >> 5];
                        c[0] = sums.fw[0]; c[1] = sums.fw[1]; c[2] = sums.fw[2]; c[3] = sums.mass;
                    }
                }
            }
        }
        __syncthreads();   // stage s and the records of row r are no longer read
        if (s_abort) {
            if (tid == 0) {
                atomicOr(&sA[s].sq->status, ST_WATCHDOG);
                for (int q = 0; q < NST; ++q) mbar_wait(&mbar[q], (parity >> q) & 1u);   // bounded
            }
            return;
        }
        if (tid == 0) {
            if (sums_on) {
                const int nch = (sL[s].nx + 31) >> 5;
                double t0 = 0, t1 = 0, t2 = 0, t3 = 0;
                for (int c = 0; c < nch; ++c) {
                    t0 += red[k & 1][c][0]; t1 += red[k & 1][c][1]; t2 += red[k & 1][c][2]; t3 += red[k & 1][c][3];
                }
                double* out = row_part + (size_t)sP[s] * BLOCK_PART;
                out[0] = t0; out[1] = t1; out[2] = t2; out[3] = t3;
            }
            if (r + NST < r1) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                issue(r + NST, s);
            }
        }
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
