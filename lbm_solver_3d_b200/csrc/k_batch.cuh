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

// Streaming stores in the ensemble's bulk kernels: FP16 storage only. In FP32
// storage they made the chunk kernel slower (5.18 -> 5.61 ms for 256 members),
// its partly written lines leaving L2 before the neighbouring warps fill them.
template <class S>
constexpr bool ens_stream() { return sizeof(typename S::T) == 2; }



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

// Resident 128-thread CTAs per SM the ensemble's row and chunk kernels are
// compiled for: 7 (72 registers) with FP32 arithmetic, 4 (128) with FP64
// arithmetic (the FP64 form and FP32 storage), which spills at 72.
template <class S>
__host__ __device__ constexpr int batch_min_blocks() {
    return S::shifted && sizeof(typename S::A) == 4 ? 7 : 4;
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
                    if (active) update_node<S, PAR, false, MACRO, ens_stream<S>()>(L, a, n, x, y, z, 0, wr, MACRO, sums);
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
//  k_bulk_rowcta<S, PAR, MACRO, WR>: the rows away from walls (WR: the rows
//  next to a wall, with their bounce-back and wall momentum), one CTA of
//  ROWCTA_THREADS threads per row (grid = rows; the hardware scheduler keeps
//  the SMs full, as for k_bulk on a single lattice). Warp 0 copies the row's
//  member records into shared memory; nodes x = tid, tid + ROWCTA_THREADS.
//  Row partial sums are formed as in k_bulk_batch.
// ---------------------------------------------------------------------------
constexpr int ROWCTA_THREADS = 128;

template <class S, int PAR, bool MACRO, bool WR>
__global__ void __launch_bounds__(ROWCTA_THREADS, batch_min_blocks<S>()) k_bulk_rowcta(const Lattice* __restrict__ lat,
                                                                const StreamArgs* __restrict__ args,
                                                                const RowRef* __restrict__ rows,
                                                                double* __restrict__ row_part, BatchStep st) {
    __shared__ __align__(16) Lattice sL;
    __shared__ __align__(16) StreamArgs sA;
    __shared__ ZoneBox sZ;
    __shared__ double red[BATCH_CHUNKS][4];
    const int tid = threadIdx.x, lane = tid & 31;
    const RowRef rr = rows[blockIdx.x];   // uniform: one row per CTA
    {   // the member's records, one word per thread, with this step's settings
        constexpr int NL = (int)(sizeof(Lattice) / 4), NA = (int)(sizeof(StreamArgs) / 4);
        static_assert(NL <= ROWCTA_THREADS && NA <= ROWCTA_THREADS, "one word per thread");
        if (tid < NL) reinterpret_cast<uint32_t*>(&sL)[tid] = reinterpret_cast<const uint32_t*>(lat + rr.m)[tid];
        if (tid < NA) {
            uint32_t w = reinterpret_cast<const uint32_t*>(args + rr.m)[tid];
            if (tid == (int)(offsetof(StreamArgs, zslot) / 4)) w = (uint32_t)st.zslot;
            if (tid == (int)(offsetof(StreamArgs, do_mass) / 4)) w = (uint32_t)st.do_mass;
            if (tid == (int)(offsetof(StreamArgs, apply_corr) / 4)) w = (uint32_t)st.apply_corr;
            reinterpret_cast<uint32_t*>(&sA)[tid] = w;
        }
        if (tid == ROWCTA_THREADS - 1) sZ = args[rr.m].sq->zone[st.zslot];
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
            if (active) update_node<S, PAR, false, MACRO, ens_stream<S>()>(L, sA, n, x, y, z, 0, WR ? wall_row(L, y, z) : (uint8_t)0, MACRO, sums);
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
//  k_bulk_chunk<S, PAR, MACRO>: the rows away from walls cut into chunks of 32
//  consecutive nodes; every warp owns one chunk (4 warps per CTA, grid =
//  chunks / 4) and runs on its own: it copies its member's records into its
//  shared slot (one word per lane), with no CTA-wide barrier, and its lanes
//  update x0 + lane. Lanes are idle only past the end of a row, in its last
//  chunk. On steps that sum, each chunk's partial (the shuffle tree over its
//  32 nodes) goes to chunk_part, and k_fold_chunks adds a row's chunks in
//  order: the row partial is bit-identical to k_bulk's (0 + c0 + c1 + ...).
// ---------------------------------------------------------------------------
constexpr int CHUNK_WARPS = 4;

template <class S, int PAR, bool MACRO>
__global__ void __launch_bounds__(32 * CHUNK_WARPS, batch_min_blocks<S>()) k_bulk_chunk(
    const Lattice* __restrict__ lat, const StreamArgs* __restrict__ args, const ChunkRef* __restrict__ chunks,
    int nchunks, double* __restrict__ chunk_part, BatchStep st) {
    __shared__ __align__(16) Lattice sL[CHUNK_WARPS];
    __shared__ __align__(16) StreamArgs sA[CHUNK_WARPS];
    __shared__ ZoneBox sZ[CHUNK_WARPS];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * CHUNK_WARPS + w;
    if (c >= nchunks) return;   // warp-uniform
    const ChunkRef cr = chunks[c];
    {
        constexpr int NL = (int)(sizeof(Lattice) / 4), NA = (int)(sizeof(StreamArgs) / 4);
        const uint32_t* srcl = reinterpret_cast<const uint32_t*>(lat + cr.m);
        uint32_t* dstl = reinterpret_cast<uint32_t*>(&sL[w]);
        for (int k = lane; k < NL; k += 32) dstl[k] = srcl[k];
        const uint32_t* srca = reinterpret_cast<const uint32_t*>(args + cr.m);
        uint32_t* dsta = reinterpret_cast<uint32_t*>(&sA[w]);
        for (int k = lane; k < NA; k += 32) {
            uint32_t v = srca[k];
            if (k == (int)(offsetof(StreamArgs, zslot) / 4)) v = (uint32_t)st.zslot;
            if (k == (int)(offsetof(StreamArgs, do_mass) / 4)) v = (uint32_t)st.do_mass;
            if (k == (int)(offsetof(StreamArgs, apply_corr) / 4)) v = (uint32_t)st.apply_corr;
            dsta[k] = v;
        }
        if (lane == 0) sZ[w] = args[cr.m].sq->zone[st.zslot];
        __syncwarp();
    }
    const Lattice& L = sL[w];
    const StreamArgs& a = sA[w];
    NodeSums sums;
    const int x = cr.x0 + lane;
    if (x < L.nx) {
        const unsigned n = (unsigned)x + (unsigned)L.nx * ((unsigned)cr.y + (unsigned)L.ny * (unsigned)cr.z);
        const bool active = (a.flag[n] & (uint8_t)~NEAR_WALL) == 0 && !in_zone(L, sZ[w], x, cr.y, cr.z);
        if (active) update_node<S, PAR, false, MACRO, ens_stream<S>()>(L, a, n, x, cr.y, cr.z, 0, 0, MACRO, sums);
    }
    if (st.do_mass || MACRO) {
        chunk_reduce(sums);
        if (lane == 0) {
            double* o = chunk_part + (size_t)c * BLOCK_PART;
            o[0] = sums.fw[0]; o[1] = sums.fw[1]; o[2] = sums.fw[2]; o[3] = sums.mass;
        }
    }
}

// k_bulk_chunkp<S, PAR, MACRO>: the chunks of k_bulk_chunk walked by persistent
// warps (grid = SMs x CTAs per SM, 4 warps per CTA): warp g takes chunks
// g, g + G, g + 2G, ... (G = all warps). The member records are copied only
// when the member changes, and the next chunk's descriptor is loaded while
// the current chunk is updated, so a warp's start-up latency is paid once.
// FLAT (steps without sums): the chunks are 32-node pieces of runs of rows,
// x0 in the low 16 bits of ChunkRef::x0 and the length above; a piece starts
// at (x0, y) and continues into the next rows of the same z-plane, and no
// partials are written.
template <class S, int PAR, bool MACRO, bool FLAT = false>
__global__ void __launch_bounds__(32 * CHUNK_WARPS, batch_min_blocks<S>()) k_bulk_chunkp(
    const Lattice* __restrict__ lat, const StreamArgs* __restrict__ args, const ChunkRef* __restrict__ chunks,
    int nchunks, double* __restrict__ chunk_part, BatchStep st) {
    __shared__ __align__(16) Lattice sL[CHUNK_WARPS];
    __shared__ __align__(16) StreamArgs sA[CHUNK_WARPS];
    __shared__ ZoneBox sZ[CHUNK_WARPS];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int G = gridDim.x * CHUNK_WARPS;
    int c = blockIdx.x * CHUNK_WARPS + w;
    int cur_m = -1;
    ChunkRef next{};
    if (c < nchunks) next = chunks[c];
    for (; c < nchunks; c += G) {
        const ChunkRef cr = next;
        if (c + G < nchunks) next = chunks[c + G];   // in flight while this chunk is updated
        if (cr.m != cur_m) {                          // warp-uniform
            __syncwarp();
            constexpr int NL = (int)(sizeof(Lattice) / 4), NA = (int)(sizeof(StreamArgs) / 4);
            const uint32_t* srcl = reinterpret_cast<const uint32_t*>(lat + cr.m);
            uint32_t* dstl = reinterpret_cast<uint32_t*>(&sL[w]);
            for (int k = lane; k < NL; k += 32) dstl[k] = srcl[k];
            const uint32_t* srca = reinterpret_cast<const uint32_t*>(args + cr.m);
            uint32_t* dsta = reinterpret_cast<uint32_t*>(&sA[w]);
            for (int k = lane; k < NA; k += 32) {
                uint32_t v = srca[k];
                if (k == (int)(offsetof(StreamArgs, zslot) / 4)) v = (uint32_t)st.zslot;
                if (k == (int)(offsetof(StreamArgs, do_mass) / 4)) v = (uint32_t)st.do_mass;
                if (k == (int)(offsetof(StreamArgs, apply_corr) / 4)) v = (uint32_t)st.apply_corr;
                dsta[k] = v;
            }
            if (lane == 0) sZ[w] = args[cr.m].sq->zone[st.zslot];
            __syncwarp();
            cur_m = cr.m;
        }
        const Lattice& L = sL[w];
        const StreamArgs& a = sA[w];
        NodeSums sums;
        int x, y = cr.y;
        bool on;
        if (FLAT) {
            x = (cr.x0 & 0xffff) + lane;
            on = lane < (cr.x0 >> 16);
            while (x >= L.nx) { x -= L.nx; ++y; }
        } else {
            x = cr.x0 + lane;
            on = x < L.nx;
        }
        if (on) {
            const unsigned n = (unsigned)x + (unsigned)L.nx * ((unsigned)y + (unsigned)L.ny * (unsigned)cr.z);
            const bool active = (a.flag[n] & (uint8_t)~NEAR_WALL) == 0 && !in_zone(L, sZ[w], x, y, cr.z);
            if (active) update_node<S, PAR, false, MACRO, ens_stream<S>()>(L, a, n, x, y, cr.z, 0, 0, MACRO, sums);
        }
        if (!FLAT && (st.do_mass || MACRO)) {
            chunk_reduce(sums);
            if (lane == 0) {
                double* o = chunk_part + (size_t)c * BLOCK_PART;
                o[0] = sums.fw[0]; o[1] = sums.fw[1]; o[2] = sums.fw[2]; o[3] = sums.mass;
            }
        }
    }
}

// row partial = its chunk partials added in order, from 0 (one thread per row)
static __global__ void k_fold_chunks(const RowChunks* __restrict__ rc, int nrows, const double* __restrict__ chunk_part,
                              double* __restrict__ row_part) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrows) return;
    const RowChunks q = rc[r];
    double t0 = 0, t1 = 0, t2 = 0, t3 = 0;
    for (int k = 0; k < q.count; ++k) {
        const double* p = chunk_part + (size_t)(q.first + k) * BLOCK_PART;
        t0 += p[0]; t1 += p[1]; t2 += p[2]; t3 += p[3];
    }
    double* o = row_part + (size_t)q.part * BLOCK_PART;
    o[0] = t0; o[1] = t1; o[2] = t2; o[3] = t3;
}

// ---------------------------------------------------------------------------
//  k_bulk_staged<S, PAR, MACRO, NST>: the rows away from walls, like
//  k_bulk_batch, with every row's populations staged in shared memory by bulk
//  asynchronous copies and a producer warp that runs ahead of the consumers.
//
//  CTA c owns the contiguous rows [bounds[c], bounds[c+1]) of the row list
//  (balanced by node count on the host). A stage holds what one row reads:
//  the 19 direction-rows (an even step reads A[i] of the row itself, an odd
//  step A[opp(i)] of the row (y - cy_i, z - cz_i); each a whole x-row) and
//  the row's flag bytes.
//    warp 0 (producer)   for each row: wait until its stage is free (empty
//                        barrier), copy the member's records into a member
//                        slot if the member changed, and fill the stage with
//                        20 cp.async.bulk copies (global -> shared, no
//                        multicast) that complete on the stage's full barrier.
//                        Each copy starts at the 16-byte boundary below its
//                        row and is rounded up to 16 bytes, so it may read up
//                        to 15 bytes either side of the row, always inside the
//                        allocation (sizes are multiples of 256 bytes).
//    warps 1-4 (update)  wait for the stage (full barrier), update the row's
//                        nodes from it (stores go straight to global memory),
//                        release the stage (empty barrier).
//  NST - 1 rows are in flight while one is updated, so the bytes in flight per
//  SM sit in shared memory rather than in registers. Row partial sums are
//  formed as in k_bulk_batch (bit-identical to a lattice run alone).
//  Every wait is bounded: on a timeout ST_WATCHDOG is set in the member's
//  status word and the CTA stops. The only CTA-wide barrier after the start
//  is the last one, which every warp reaches once its own loop has ended (all
//  its waits are bounded). Behind it, after an abort, one thread waits
//  (bounded) for the last copy the producer issued into each stage, so no bulk
//  copy is still landing in this CTA's shared memory when it exits.
// ---------------------------------------------------------------------------
constexpr int STAGED_UPDATE_WARPS = 4;
constexpr int STAGED_THREADS = 32 * (1 + STAGED_UPDATE_WARPS);

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* m, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* m, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(m)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* m) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(m)) : "memory");
}
// true once the phase with the given parity has completed; false after
// `limit` tries (each try_wait also suspends for a while in hardware)
__device__ __forceinline__ bool mbar_wait_n(uint64_t* m, uint32_t parity, long long limit) {
    const uint32_t a = smem_u32(m);
    for (long long it = 0; it < limit; ++it) {
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
constexpr long long MBAR_WAIT_LIMIT = 1ll << 22;
__device__ __forceinline__ bool mbar_wait(uint64_t* m, uint32_t parity) { return mbar_wait_n(m, parity, MBAR_WAIT_LIMIT); }
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* m) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(m))
                 : "memory");
}
// An L2 policy that evicts first: for the bulk's own traffic, read once per
// step, so that it does not displace the zone's and the squirmer update's data.
__device__ __forceinline__ uint64_t l2_evict_first() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
// global -> shared bulk copy with an L2 policy
__device__ __forceinline__ void bulk_g2s_hint(void* dst, const void* src, unsigned bytes, uint64_t* m, uint64_t pol) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(m)), "l"(pol)
                 : "memory");
}
// shared -> global bulk copy with an L2 policy (this thread's bulk group)
__device__ __forceinline__ void bulk_s2g_hint(void* dst, const void* src, unsigned bytes, uint64_t pol) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group.L2::cache_hint [%0], [%1], %2, %3;"
                 ::"l"(dst), "r"(smem_u32(src)), "r"(bytes), "l"(pol)
                 : "memory");
}
// shared -> global bulk copy (this thread's bulk group); both addresses 16-byte
// aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_s2g(void* dst, const void* src, unsigned bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;"
                 ::"l"(dst), "r"(smem_u32(src)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// this thread's bulk groups have finished reading their shared-memory sources
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// ... and have completed
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// this thread's shared-memory writes become visible to later bulk copies
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// named barrier `id` over `n` threads (a multiple of 32) that also returns the
// AND of p over them: the same value in every participating thread
__device__ __forceinline__ bool bar_and(int id, int n, bool p) {
    unsigned r;
    asm volatile("{\n\t.reg .pred pi, po;\n\tsetp.ne.u32 pi, %1, 0;\n\t"
                 "bar.red.and.pred po, %2, %3, pi;\n\tselp.u32 %0, 1, 0, po;\n\t}"
                 : "=r"(r) : "r"((unsigned)p), "r"(id), "r"(n) : "memory");
    return r != 0;
}
__device__ __forceinline__ void bar_sync_n(int id, int n) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }

// 16-byte aligned start and rounded-up length of the copy of [p, p + bytes)
__device__ __forceinline__ void span16(const void* p, size_t bytes, uintptr_t& start, unsigned& len, int& off) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    start = a & ~(uintptr_t)15;
    off = (int)(a - start);
    len = (unsigned)((a + bytes - start + 15) & ~(uintptr_t)15);
}

// velocity set by a runtime index (lanes of the producer take one direction each)
__device__ __forceinline__ int c_opp_rt(int i) { return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1); }
__device__ __forceinline__ int c_cx_rt(int i) {
    int v = 0;
#pragma unroll
    for (int k = 0; k < Q; ++k) if (k == i) v = CX(k);
    return v;
}
__device__ __forceinline__ int c_cy_rt(int i) {
    int v = 0;
#pragma unroll
    for (int k = 0; k < Q; ++k) if (k == i) v = CY(k);
    return v;
}
__device__ __forceinline__ int c_cz_rt(int i) {
    int v = 0;
#pragma unroll
    for (int k = 0; k < Q; ++k) if (k == i) v = CZ(k);
    return v;
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

template <class S, int PAR, bool MACRO, int NST>
__global__ void __launch_bounds__(STAGED_THREADS) k_bulk_staged(const Lattice* __restrict__ lat,
                                                                const StreamArgs* __restrict__ args,
                                                                const RowRef* __restrict__ rows,
                                                                const int* __restrict__ bounds,
                                                                double* __restrict__ row_part, BatchStep st, int cap,
                                                                int fcap) {
    using T = typename S::T;
    constexpr int MS = NST + 1;   // member slots: a slot is reused NST + 1 member changes later
    extern __shared__ __align__(128) unsigned char staged_raw[];
    T* const buf = reinterpret_cast<T*>(staged_raw);                                   // NST x Q x cap
    uint8_t* const fbuf = staged_raw + (size_t)NST * Q * cap * sizeof(T);             // NST x fcap
    __shared__ __align__(8) uint64_t full[NST], empty[NST];
    __shared__ __align__(16) Lattice recL[MS];
    __shared__ __align__(16) StreamArgs recA[MS];
    __shared__ ZoneBox recZ[MS];
    __shared__ int sSlot[NST], sY[NST], sZc[NST], sP[NST], sOff[NST][Q], sFoff[NST];
    __shared__ double red[NST][BATCH_CHUNKS][4];   // chunk sums of the row in stage q
    __shared__ int cnt[NST];                        // update warps done with the row in stage q
    __shared__ volatile int s_abort;
    __shared__ int s_issued;                        // stages armed by the producer
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int r0 = bounds[blockIdx.x], r1 = bounds[blockIdx.x + 1];
    const bool sums_on = st.do_mass || MACRO;

    if (tid == 0) {
        for (int q = 0; q < NST; ++q) {
            mbar_init(&full[q], 1);
            mbar_init(&empty[q], STAGED_UPDATE_WARPS);
            cnt[q] = 0;
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
        s_issued = 0;
    }
    __syncthreads();

    if (warp == 0) {
        // ---------------- producer ----------------
        int last_m = -1, slot = -1;
        RowRef batch{};   // lane j holds rows[base + j]: one load per 32 rows
        for (int k = 0; r0 + k < r1; ++k) {
            const int q = k % NST;
            if ((k & 31) == 0 && r0 + k + lane < r1) batch = rows[r0 + k + lane];
            if (k >= NST) {
                int go = 1;   // decided by lane 0 for the whole warp
                if (lane == 0) go = mbar_wait(&empty[q], (uint32_t)((k / NST - 1) & 1)) && !s_abort;
                go = __shfl_sync(0xffffffffu, go, 0);
                if (!go) { if (lane == 0) s_abort = 1; break; }
            }
            const int src_lane = k & 31;
            const RowRef rr{__shfl_sync(0xffffffffu, batch.m, src_lane), __shfl_sync(0xffffffffu, batch.y, src_lane),
                            __shfl_sync(0xffffffffu, batch.z, src_lane), __shfl_sync(0xffffffffu, batch.part, src_lane)};
            if (rr.m != last_m) {
                slot = (slot + 1) % MS;
                const uint32_t* srcl = reinterpret_cast<const uint32_t*>(lat + rr.m);
                uint32_t* dstl = reinterpret_cast<uint32_t*>(&recL[slot]);
                for (int w = lane; w < (int)(sizeof(Lattice) / 4); w += 32) dstl[w] = srcl[w];
                const uint32_t* srca = reinterpret_cast<const uint32_t*>(args + rr.m);
                uint32_t* dsta = reinterpret_cast<uint32_t*>(&recA[slot]);
                for (int w = lane; w < (int)(sizeof(StreamArgs) / 4); w += 32) dsta[w] = srca[w];
                if (lane == 0) recZ[slot] = args[rr.m].sq->zone[st.zslot];
                __syncwarp();
                if (lane == 0) {
                    recA[slot].zslot = st.zslot; recA[slot].do_mass = st.do_mass; recA[slot].apply_corr = st.apply_corr;
                }
                last_m = rr.m;
                __syncwarp();
            }
            // lane i < Q copies direction-row i, lane Q the flag row
            const Lattice& L = recL[slot];
            uintptr_t start = 0;
            unsigned len = 0;
            int ob = 0;
            if (lane < Q) {
                const int i = lane;
                int ys = rr.y, zs = rr.z, arr = i;
                if (PAR == 1) {
                    arr = c_opp_rt(i);
                    ys = rr.y - c_cy_rt(i); if (ys < 0) ys += L.ny; else if (ys >= L.ny) ys -= L.ny;
                    zs = rr.z - c_cz_rt(i); if (zs < 0) zs += L.nz; else if (zs >= L.nz) zs -= L.nz;
                }
                const T* f = static_cast<const T*>(recA[slot].f);
                span16(f + (size_t)arr * L.N + (size_t)L.nx * (ys + (size_t)L.ny * zs), (size_t)L.nx * sizeof(T), start,
                       len, ob);
                sOff[q][i] = ob / (int)sizeof(T);
            } else if (lane == Q) {
                span16(recA[slot].flag + (size_t)L.nx * (rr.y + (size_t)L.ny * rr.z), (size_t)L.nx, start, len, ob);
                sFoff[q] = ob;
            }
            unsigned total = len;
            for (int o = 16; o > 0; o >>= 1) total += __shfl_down_sync(0xffffffffu, total, o);
            if (lane == 0) {
                sSlot[q] = slot; sY[q] = rr.y; sZc[q] = rr.z; sP[q] = rr.part;
                mbar_expect_tx(&full[q], total);   // releases the records written above
            }
            __syncwarp();
            if (lane < Q)
                bulk_g2s(buf + ((size_t)q * Q + lane) * cap, reinterpret_cast<const void*>(start), len, &full[q]);
            else if (lane == Q)
                bulk_g2s(fbuf + (size_t)q * fcap, reinterpret_cast<const void*>(start), len, &full[q]);
            if (lane == 0) s_issued = k + 1;
            __syncwarp();
        }
    } else {
    // ---------------- update warps ----------------
    const int ut = tid - 32;   // 0 .. 32 * STAGED_UPDATE_WARPS - 1
    for (int k = 0; r0 + k < r1; ++k) {
        const int q = k % NST;
        int go = 1;   // decided by lane 0 for the whole warp
        if (lane == 0) {
            const bool ok = mbar_wait(&full[q], (uint32_t)((k / NST) & 1));
            if (!ok && !s_abort) { s_abort = 1; atomicOr(&recA[sSlot[q]].sq->status, ST_WATCHDOG); }
            go = ok && !s_abort;
        }
        go = __shfl_sync(0xffffffffu, go, 0);
        if (!go) break;
        const int slot = sSlot[q];
        const Lattice& L = recL[slot];
        const StreamArgs& a = recA[slot];
        const int y = sY[q], z = sZc[q];
        const T* sb = buf + (size_t)q * Q * cap;
        const uint8_t* sf = fbuf + (size_t)q * fcap + sFoff[q];
        const int nxr = (L.nx + 31) & ~31;
        for (int x = ut; x < nxr; x += 32 * STAGED_UPDATE_WARPS) {
            NodeSums sums;
            if (x < L.nx) {
                const unsigned n = (unsigned)x + (unsigned)L.nx * ((unsigned)y + (unsigned)L.ny * (unsigned)z);
                const bool active = (sf[x] & (uint8_t)~NEAR_WALL) == 0 && !in_zone(L, recZ[slot], x, y, z);
                if (active)
                    update_node<S, PAR, false, MACRO, ens_stream<S>()>(L, a, n, x, y, z, 0, 0, MACRO, sums,
                                                      StagedSrc<T>{sb, sOff[q], cap, x, L.nx});
            }
            if (sums_on) {
                chunk_reduce(sums);
                if (lane == 0) {
                    double* c = red[q][x >> 5];
                    c[0] = sums.fw[0]; c[1] = sums.fw[1]; c[2] = sums.fw[2]; c[3] = sums.mass;
                }
            }
        }
        __syncwarp();
        if (lane == 0) {
            if (sums_on) {
                // the last update warp to finish the row adds its chunk sums in order
                __threadfence_block();
                if (atomicAdd(&cnt[q], 1) == STAGED_UPDATE_WARPS - 1) {
                    __threadfence_block();
                    const int nch = nxr >> 5;
                    double t0 = 0, t1 = 0, t2 = 0, t3 = 0;
                    for (int c = 0; c < nch; ++c) {
                        t0 += red[q][c][0]; t1 += red[q][c][1]; t2 += red[q][c][2]; t3 += red[q][c][3];
                    }
                    double* out = row_part + (size_t)sP[q] * BLOCK_PART;
                    out[0] = t0; out[1] = t1; out[2] = t2; out[3] = t3;
                    cnt[q] = 0;
                }
            }
            mbar_arrive(&empty[q]);   // the stage (and red[q]) may be refilled
        }
    }
    }
    // After an abort, stage q may still receive the copies of its last arming
    // (the update warps stopped waiting for them): wait for that phase to
    // complete before the CTA's shared memory is released.
    __syncthreads();
    if (tid == 0 && s_abort) {
        const int issued = s_issued;
        for (int q = 0; q < NST && q < issued; ++q) {
            const int arms = (issued - q + NST - 1) / NST;   // times stage q was armed
            mbar_wait(&full[q], (uint32_t)((arms - 1) & 1));
        }
    }
}

// ---------------------------------------------------------------------------
//  k_bulk_runs<S, PAR>: the rows away from walls of every member on a step
//  without sums, staged through shared memory in runs: a run is up to
//  RunsCfg<S>::NODES nodes of consecutive interior rows of one member's z-plane,
//  which are consecutive in memory for every direction (odd steps read the rows
//  of the plane shifted by the direction's (c_y, c_z), again consecutive;
//  walls in y keep y - c_y inside the plane, and a run that would wrap in y is
//  a single row). One producer warp copies the 19 ranges and the flags of a
//  run with bulk asynchronous copies (from the 16-byte boundary below each
//  range, rounded up: never outside the member's padded slice) into one of NST
//  stages; eight update warps update the run's nodes from the stage with
//  update_node's arithmetic and release it. Persistent CTAs take runs
//  blockIdx.x + k * gridDim.x. Bounded waits and the drain on exit as in
//  k_bulk_staged. The populations do not depend on how rows are grouped, so
//  members stay bit-identical to lattices run alone; steps with sums use the
//  chunk kernels, which form the row partials in k_bulk's order.
// ---------------------------------------------------------------------------
constexpr int RUNS_UPDATE_WARPS = 8;
constexpr int RUNS_THREADS = 32 * (1 + RUNS_UPDATE_WARPS);
template <class S> struct RunsCfg;
template <> struct RunsCfg<StoreF64> { static constexpr int NST = 2, NODES = 256; };
template <> struct RunsCfg<StoreF32> { static constexpr int NST = 3, NODES = 384; };
template <> struct RunsCfg<StoreF16> { static constexpr int NST = 4, NODES = 512; };
static_assert(RunsCfg<StoreF64>::NODES >= BATCH_MAX_NX, "a run holds at least one row of every member");
// elements per staged direction range (a run plus the 16-byte rounding at both
// ends), flag bytes per stage, bytes per stage (all multiples of 16)
template <class S> __host__ __device__ constexpr int runs_cap() {
    return RunsCfg<S>::NODES + 32 / (int)sizeof(typename S::T);
}
template <class S> __host__ __device__ constexpr int runs_fcap() { return RunsCfg<S>::NODES + 32; }
template <class S> __host__ __device__ constexpr size_t runs_stage_bytes() {
    return (size_t)Q * runs_cap<S>() * sizeof(typename S::T) + runs_fcap<S>();
}

// populations of node (row, x) of a staged run
template <class T>
struct RunSrc {
    const T* sb;
    const int* off;     // element offset of each direction's range in its slot
    int cap, x, nx, row;
    template <class S, int PAR, class V>
    __device__ __forceinline__ void load(const T*, unsigned, unsigned, const Nbr&, V* v) const {
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            int xs = x;
            if (PAR == 1) {
                xs = x - CX(i);
                if (xs < 0) xs += nx; else if (xs >= nx) xs -= nx;
            }
            v[i] = (V)S::ld(sb + i * cap + off[i] + row * nx + xs);
        }
    }
};

template <class S, int PAR>
__global__ void __launch_bounds__(RUNS_THREADS, 2) k_bulk_runs(const Lattice* __restrict__ lat,
                                                            const StreamArgs* __restrict__ args,
                                                            const int4* __restrict__ runs, int nruns, BatchStep st) {
    using T = typename S::T;
    constexpr int NST = RunsCfg<S>::NST, MS = NST + 1, CAP = runs_cap<S>(), FCAP = runs_fcap<S>();
    constexpr size_t STAGE = runs_stage_bytes<S>();
    extern __shared__ __align__(128) unsigned char runs_raw[];
    __shared__ __align__(8) uint64_t full[NST], empty[NST];
    __shared__ __align__(16) Lattice recL[MS];
    __shared__ __align__(16) StreamArgs recA[MS];
    __shared__ ZoneBox recZ[MS];
    __shared__ int sSlot[NST], sOff[NST][Q], sFoff[NST];
    __shared__ int4 sRun[NST];
    __shared__ volatile int s_abort;
    __shared__ int s_issued;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        for (int q = 0; q < NST; ++q) {
            mbar_init(&full[q], 1);
            mbar_init(&empty[q], RUNS_UPDATE_WARPS);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
        s_issued = 0;
    }
    __syncthreads();

    if (warp == 0) {
        // ---------------- producer ----------------
        int last_m = -1, slot = -1;
        for (int k = 0; (int)blockIdx.x + k * (int)gridDim.x < nruns; ++k) {
            const int q = k % NST;
            if (k >= NST) {
                int go = 1;
                if (lane == 0) {
                    const bool ok = mbar_wait(&empty[q], (uint32_t)((k / NST - 1) & 1));
                    if (!ok && !s_abort) { s_abort = 1; atomicOr(&args[0].sq->status, ST_WATCHDOG); }
                    go = ok && !s_abort;
                }
                if (!__shfl_sync(0xffffffffu, go, 0)) break;
            }
            const int4 run = runs[blockIdx.x + k * gridDim.x];   // (m, y0, z, nrow)
            if (run.x != last_m) {
                slot = (slot + 1) % MS;
                const uint32_t* srcl = reinterpret_cast<const uint32_t*>(lat + run.x);
                uint32_t* dstl = reinterpret_cast<uint32_t*>(&recL[slot]);
                for (int w = lane; w < (int)(sizeof(Lattice) / 4); w += 32) dstl[w] = srcl[w];
                const uint32_t* srca = reinterpret_cast<const uint32_t*>(args + run.x);
                uint32_t* dsta = reinterpret_cast<uint32_t*>(&recA[slot]);
                for (int w = lane; w < (int)(sizeof(StreamArgs) / 4); w += 32) dsta[w] = srca[w];
                if (lane == 0) recZ[slot] = args[run.x].sq->zone[st.zslot];
                __syncwarp();
                if (lane == 0) {
                    recA[slot].zslot = st.zslot; recA[slot].do_mass = st.do_mass; recA[slot].apply_corr = st.apply_corr;
                }
                last_m = run.x;
                __syncwarp();
            }
            const Lattice& L = recL[slot];
            const size_t cnt = (size_t)run.w * L.nx;
            unsigned char* sb = runs_raw + (size_t)q * STAGE;
            uintptr_t start = 0;
            unsigned len = 0;
            int ob = 0;
            if (lane < Q) {
                const int i = lane;
                int ys = run.y, zs = run.z, arr = i;
                if (PAR == 1) {
                    arr = c_opp_rt(i);
                    ys = run.y - c_cy_rt(i); if (ys < 0) ys += L.ny; else if (ys >= L.ny) ys -= L.ny;
                    zs = run.z - c_cz_rt(i); if (zs < 0) zs += L.nz; else if (zs >= L.nz) zs -= L.nz;
                }
                const T* f = static_cast<const T*>(recA[slot].f);
                span16(f + (size_t)arr * L.N + (size_t)L.nx * (ys + (size_t)L.ny * zs), cnt * sizeof(T), start, len, ob);
                sOff[q][i] = ob / (int)sizeof(T);
            } else if (lane == Q) {
                span16(recA[slot].flag + (size_t)L.nx * (run.y + (size_t)L.ny * run.z), cnt, start, len, ob);
                sFoff[q] = ob;
            }
            unsigned total = len;
            for (int o = 16; o > 0; o >>= 1) total += __shfl_down_sync(0xffffffffu, total, o);
            if (lane == 0) {
                sSlot[q] = slot; sRun[q] = run;
                mbar_expect_tx(&full[q], total);   // releases the records written above
            }
            __syncwarp();
            if (lane < Q)
                bulk_g2s(sb + (size_t)lane * CAP * sizeof(T), reinterpret_cast<const void*>(start), len, &full[q]);
            else if (lane == Q)
                bulk_g2s(sb + (size_t)Q * CAP * sizeof(T), reinterpret_cast<const void*>(start), len, &full[q]);
            if (lane == 0) s_issued = k + 1;
            __syncwarp();
        }
    } else {
        // ---------------- update warps ----------------
        const int ut = tid - 32;
        for (int k = 0; (int)blockIdx.x + k * (int)gridDim.x < nruns; ++k) {
            const int q = k % NST;
            const bool ok = mbar_wait(&full[q], (uint32_t)((k / NST) & 1));
            if (!__all_sync(0xffffffffu, ok)) {
                if (lane == 0 && !s_abort) { s_abort = 1; atomicOr(&args[0].sq->status, ST_WATCHDOG); }
                break;
            }
            if (__shfl_sync(0xffffffffu, s_abort, 0)) break;
            const int slot = sSlot[q];
            const Lattice& L = recL[slot];
            const StreamArgs& a = recA[slot];
            const int4 run = sRun[q];
            const T* sb = reinterpret_cast<const T*>(runs_raw + (size_t)q * STAGE);
            const uint8_t* sf = runs_raw + (size_t)q * STAGE + (size_t)Q * CAP * sizeof(T) + sFoff[q];
            const int cnt = run.w * L.nx;
            const unsigned n0 = (unsigned)L.nx * ((unsigned)run.y + (unsigned)L.ny * (unsigned)run.z);
            for (int j = ut; j < cnt; j += 32 * RUNS_UPDATE_WARPS) {
                const int row = j / L.nx, x = j - row * L.nx, y = run.y + row;
                const bool active = (sf[j] & (uint8_t)~NEAR_WALL) == 0 && !in_zone(L, recZ[slot], x, y, run.z);
                if (active) {
                    NodeSums sums;
                    update_node<S, PAR, false, false, ens_stream<S>()>(L, a, n0 + (unsigned)j, x, y, run.z, 0, 0, false, sums,
                                                      RunSrc<T>{sb, sOff[q], CAP, x, L.nx, row});
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[q]);
        }
    }
    __syncthreads();
    if (tid == 0 && s_abort) {
        const int issued = s_issued;
        for (int q = 0; q < NST && q < issued; ++q) mbar_wait(&full[q], (uint32_t)(((issued - q + NST - 1) / NST - 1) & 1));
    }
}

// ---------------------------------------------------------------------------
//  k_bulk_rows<S, PAR, SQ>: the rows away from walls of a single lattice on a
//  step without sums, staged through shared memory by the bulk-copy engine.
//
//  A bulk kernel that loads its populations into registers is bound by how
//  many bytes each SM keeps in flight: 19 loads per thread in flight at the
//  occupancy the registers allow (measured on the 256x128x128 lattice: ~117 KB
//  per SM -> 0.90 of the copy rate, ~78 KB -> 0.80, ~39 KB -> 0.50). Here the
//  loads do not occupy registers: each CTA keeps RowsCfg<S>::NST whole x-rows
//  of all 19 directions (plus the row's flags) in flight in shared memory.
//
//  CTA = one producer warp + nx update threads (nx a multiple of 32, at most
//  ROWS_MAX_NX), persistent over the interior rows (y = ylo + r % nry,
//  z = zlo + r / nry), which the producers claim one at a time from a counter
//  (RowsWork): a CTA that starts late, or shares its SM with other kernels,
//  takes fewer rows instead of ending late. CTAs that land on one of the
//  `reserve` lowest-numbered SMs leave at once (rows_idle).
//    producer   per row: claims the row, waits for the stage to be free
//               (empty barrier), publishes the row number, then
//               lane i < 19 copies direction-row i of the state -- A[i] of row
//               (y, z) on an even step, A[opp(i)] of row (y - c_iy, z - c_iz)
//               on an odd step, always a whole row, 16-byte aligned -- and
//               lane 19 the row's flags, completing on the full barrier;
//               when the rows are used up it publishes -1 (a plain arrive);
//    update     thread x waits for the row (full barrier), reads its 19
//               logical populations from the stage (odd step: x - c_ix,
//               wrapped, inside the staged row), updates the node with the
//               same arithmetic as k_bulk and stores straight to global
//               memory, then releases the stage.
//  Every wait is bounded; on a timeout ST_WATCHDOG is set, all warps leave
//  their loops, and after the CTA's last barrier one thread waits (bounded)
//  for the last copy armed into each stage before the CTA exits.
// ---------------------------------------------------------------------------
constexpr int ROWS_MAX_NX = 256;
template <class S> struct RowsCfg;
template <> struct RowsCfg<StoreF64> { static constexpr int NST = 2, MINB = 2; };
template <> struct RowsCfg<StoreF32> { static constexpr int NST = 4, MINB = 2; };
template <> struct RowsCfg<StoreF16> { static constexpr int NST = 6, MINB = 3; };

template <class S>
__host__ __device__ constexpr size_t rows_stage_bytes(int nx) {
    return (size_t)Q * nx * sizeof(typename S::T) + (size_t)nx;   // nx % 32 == 0: every part 16-byte aligned
}

// The interior rows of one launch and how CTAs share them. claim[0] is the
// next unclaimed row, claim[1] the CTAs that have finished; the last CTA to
// finish sets both back to 0 for the next launch, which stream order keeps
// after this one.
struct RowsWork {
    int nry, nrows, ylo, zlo;   // rows nry x (nrows / nry) from (ylo, zlo)
    int reserve;                // CTAs on SMs with %smid < reserve take no rows
    int* claim;
};

__device__ __forceinline__ unsigned sm_id() {
    unsigned r;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(r));
    return r;
}

// A CTA on one of the reserved SMs takes no rows, so that the squirmer update
// (one CTA of 512 threads, which needs an SM to itself) finds one free while
// the persistent grid runs -- except the grid's last CTA, so that the rows are
// done whatever the placement (the claim counter lets one CTA finish them
// all). Uniform over the CTA.
__device__ __forceinline__ bool rows_idle(const RowsWork& w) {
    return (int)sm_id() < w.reserve && blockIdx.x + 1 < gridDim.x;
}

// Populations of node x from a staged row (whole direction-rows of nx elements;
// odd steps read x - c_x, wrapped inside the row).
template <class S>
struct RowSrc {
    const typename S::T* sb;
    int nx, x;
    template <class S_, int PAR, class V>
    __device__ __forceinline__ void load(const typename S::T*, unsigned, unsigned, const Nbr&, V* v) const {
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            int xs = x;
            if (PAR == 1) {
                xs = x - CX(i);
                if (xs < 0) xs += nx; else if (xs >= nx) xs -= nx;
            }
            v[i] = (V)S::ld(sb + i * nx + xs);
        }
    }
};

// The producer warp's copies of one row into a stage (k_bulk_rows, _rows2):
// lane i < 19 the direction-row of the state that the row's nodes read as
// logical f_i (even step: A[i] of row (y, z); odd step: A[opp(i)] of row
// (y - c_iy, z - c_iz), wrapped), lane 19 the row's flags; all whole rows.
template <class S, int PAR>
__device__ __forceinline__ void stage_row(const Lattice& L, const StreamArgs& a, int y, int z, unsigned char* sb,
                                          uint64_t* full, int lane) {
    using T = typename S::T;
    const int nx = L.nx;
    if (lane < Q) {
        const int i = lane;
        int ys = y, zs = z, arr = i;
        if (PAR == 1) {
            arr = c_opp_rt(i);
            ys = y - c_cy_rt(i); if (ys < 0) ys += L.ny; else if (ys >= L.ny) ys -= L.ny;
            zs = z - c_cz_rt(i); if (zs < 0) zs += L.nz; else if (zs >= L.nz) zs -= L.nz;
        }
        const T* f = static_cast<const T*>(a.f);
        bulk_g2s_hint(sb + (size_t)i * nx * sizeof(T), f + (size_t)arr * L.N + (size_t)nx * (ys + (size_t)L.ny * zs),
                      (unsigned)(nx * sizeof(T)), full, l2_evict_first());
    } else if (lane == Q) {
        bulk_g2s(sb + (size_t)Q * nx * sizeof(T), a.flag + (size_t)nx * (y + (size_t)L.ny * z), (unsigned)nx, full);
    }
}

// The producer loop shared by k_bulk_rows and k_bulk_rows2 (warp 0): claim a
// row, wait for its stage, publish it in rowid[q] and stage it; -1 ends the
// consumers' loop. Returns with s_issued = stages armed with copies.
template <class S, int PAR, int NST>
__device__ __forceinline__ void rows_produce(const Lattice& L, const StreamArgs& a, const RowsWork& w,
                                             unsigned char* raw, size_t stage, uint64_t* full, uint64_t* empty,
                                             int* rowid, volatile int& s_abort, int& s_issued, int lane) {
    for (int k = 0;; ++k) {
        const int q = k % NST;
        int r = 0;
        if (lane == 0) r = atomicAdd(w.claim, 1);   // before the wait: its latency overlaps it
        r = __shfl_sync(0xffffffffu, r, 0);
        if (k >= NST) {
            int go = 1;
            if (lane == 0) {
                const bool ok = mbar_wait(&empty[q], (uint32_t)((k / NST - 1) & 1));
                if (!ok && !s_abort) { s_abort = 1; atomicOr(&a.sq->status, ST_WATCHDOG); }
                go = ok && !s_abort;
            }
            if (!__shfl_sync(0xffffffffu, go, 0)) return;
        }
        if (r >= w.nrows) {   // no rows left: the consumers stop at this stage
            if (lane == 0) { rowid[q] = -1; mbar_arrive(&full[q]); }
            return;
        }
        unsigned char* sb = raw + (size_t)q * stage;
        if (lane == 0) { rowid[q] = r; mbar_expect_tx(&full[q], (unsigned)stage); }   // the arrive releases rowid[q]
        __syncwarp();
        stage_row<S, PAR>(L, a, w.ylo + r % w.nry, w.zlo + r / w.nry, sb, &full[q], lane);
        if (lane == 0) s_issued = k + 1;
        __syncwarp();
    }
}

// The consumers' wait for stage k: the row staged there, or -1 to leave (no
// rows left, or an abort, whose watchdog status this sets).
template <int NST>
__device__ __forceinline__ int rows_next(const StreamArgs& a, uint64_t* full, const int* rowid,
                                         volatile int& s_abort, int k, int lane) {
    const int q = k % NST;
    const bool ok = mbar_wait(&full[q], (uint32_t)((k / NST) & 1));
    if (!__all_sync(0xffffffffu, ok)) {
        if (lane == 0 && !s_abort) { s_abort = 1; atomicOr(&a.sq->status, ST_WATCHDOG); }
        return -1;
    }
    if (__shfl_sync(0xffffffffu, s_abort, 0)) return -1;   // lane 0's view, so the warp leaves together
    return __shfl_sync(0xffffffffu, rowid[q], 0);
}

// The end of a rows kernel: after an abort one thread waits (bounded) for the
// last copy armed into each stage, then the CTA counts itself done; the last
// one resets the claim counter.
template <int NST>
__device__ __forceinline__ void rows_finish(const RowsWork& w, uint64_t* full, volatile int& s_abort, int s_issued,
                                            int tid) {
    __syncthreads();
    if (tid == 0) {
        if (s_abort) {
            const int issued = s_issued;
            for (int q = 0; q < NST && q < issued; ++q)
                mbar_wait(&full[q], (uint32_t)(((issued - q + NST - 1) / NST - 1) & 1));
        }
        __threadfence();
        if (atomicAdd(w.claim + 1, 1) == (int)gridDim.x - 1) {
            w.claim[0] = 0;
            w.claim[1] = 0;
            __threadfence();
        }
    }
}

// SUMS: the step forms the rows' partial sums (a mass-correction step, or
// MACRO); steps without sums run an instantiation without that code.
template <class S, int PAR, bool SQ, bool MACRO, bool SUMS>
__global__ void __launch_bounds__(32 + ROWS_MAX_NX, RowsCfg<S>::MINB) k_bulk_rows(const Lattice L, const StreamArgs a,
                                                                                 const RowsWork w) {
    using T = typename S::T;
    constexpr int NST = RowsCfg<S>::NST;
    extern __shared__ __align__(128) unsigned char rows_raw[];
    __shared__ __align__(8) uint64_t full[NST], empty[NST];
    __shared__ ZoneBox zb;
    __shared__ double red[SUMS ? NST : 1][ROWS_MAX_NX / 32][4];   // the row's warp sums (summing steps)
    __shared__ int cnt[NST];                                       // update warps done with the row in stage q
    __shared__ int rowid[NST];                                     // the row in stage q (-1: none left)
    __shared__ volatile int s_abort;
    __shared__ int s_issued;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nx = L.nx, nupd = nx >> 5;
    const size_t stage = rows_stage_bytes<S>(nx);
    if (tid == 0) {
        for (int q = 0; q < NST; ++q) {
            mbar_init(&full[q], 1);
            mbar_init(&empty[q], nupd);
            cnt[q] = 0;
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
        s_issued = 0;
        if (SQ) zb = a.sq->zone[a.zslot];
    }
    __syncthreads();

    if (rows_idle(w)) {
    } else if (warp == 0) {
        rows_produce<S, PAR, NST>(L, a, w, rows_raw, stage, full, empty, rowid, s_abort, s_issued, lane);
    } else {
        // ---------------- update threads ----------------
        const int x = tid - 32, uw = warp - 1;
        for (int k = 0;; ++k) {
            const int r = rows_next<NST>(a, full, rowid, s_abort, k, lane);
            if (r < 0) break;
            const int q = k % NST;
            const int y = w.ylo + r % w.nry, z = w.zlo + r / w.nry;
            const unsigned char* sb = rows_raw + (size_t)q * stage;
            const uint8_t fl = sb[(size_t)Q * nx * sizeof(T) + x];
            bool active = (fl & (uint8_t)~NEAR_WALL) == 0;
            // the zone test: y and z are the row's (uniform), x the node's
            if (SQ && active && in_zone_axis(y, zb.lo[1], zb.w[1], L.ny, L.walls_y) &&
                in_zone_axis(z, zb.lo[2], zb.w[2], L.nz, L.walls_z))
                active = !in_zone_axis(x, zb.lo[0], zb.w[0], L.nx, false);
            NodeSums sums;
            if (active) {
                const unsigned n = (unsigned)x + (unsigned)nx * ((unsigned)y + (unsigned)L.ny * (unsigned)z);
                update_node<S, PAR, false, MACRO>(L, a, n, x, y, z, 0, 0, MACRO, sums,
                                                  RowSrc<S>{reinterpret_cast<const T*>(sb), nx, x});
            }
            if constexpr (SUMS) {
                // the row's partial sums in k_bulk's order (a block of nx threads
                // per row: each warp's shuffle tree, then the warps in order)
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    sums.fw[0] += __shfl_down_sync(0xffffffffu, sums.fw[0], o);
                    sums.fw[1] += __shfl_down_sync(0xffffffffu, sums.fw[1], o);
                    sums.fw[2] += __shfl_down_sync(0xffffffffu, sums.fw[2], o);
                    sums.mass += __shfl_down_sync(0xffffffffu, sums.mass, o);
                }
                if (lane == 0) {
                    double* c = red[q][uw];
                    c[0] = sums.fw[0]; c[1] = sums.fw[1]; c[2] = sums.fw[2]; c[3] = sums.mass;
                    __threadfence_block();
                    if (atomicAdd(&cnt[q], 1) == nupd - 1) {   // the last warp done adds them up in order
                        __threadfence_block();
                        double t0 = 0, t1 = 0, t2 = 0, t3 = 0;
                        for (int v = 0; v < nupd; ++v) {
                            t0 += red[q][v][0]; t1 += red[q][v][1]; t2 += red[q][v][2]; t3 += red[q][v][3];
                        }
                        double* out = a.block_part + ((size_t)y + (size_t)L.ny * z) * BLOCK_PART;
                        out[0] = t0; out[1] = t1; out[2] = t2; out[3] = t3;
                        cnt[q] = 0;
                    }
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[q]);   // this warp is done with the stage (and red[q])
        }
    }
    rows_finish<NST>(w, full, s_abort, s_issued, tid);
}

// ---------------------------------------------------------------------------
//  k_bulk_rows2<S, PAR, SQ>: k_bulk_rows with two x-adjacent nodes per update
//  thread (nx a multiple of 64), for the FP16 form, whose one-node kernel is
//  bound by instruction issue rather than memory: the directions without an x
//  shift are read from the stage as one 4-byte pair, and the results leave
//  through one of two paths, chosen per row by a vote of the update warps:
//    whole row  every node of the row is updated here (no zone, solid or
//               wall node): each direction's results form one whole row of
//               the next state (even step: A[opp(i)] of row (y, z) at x; odd
//               step: A[i] of row (y + c_iy, z + c_iz) at x + c_ix, wrapped),
//               so they are written over the stage (every read of it is done
//               by then) and leave as 19 bulk copies shared -> global, issued
//               by the first update warp, which releases the stage once the
//               copies have read it;
//    otherwise  pair_collide_store (paired conversions and 4-byte stores, the
//               x-shifted directions exchanged between lanes), the second
//               half of k_bulk_pair.
//  The update warps meet at named barrier 1 (a timed-out wait or an abort is
//  folded into the barrier's AND, so they leave the loop together and none
//  waits for a warp that has left). Same staging, claiming, bounded waits and
//  drain as k_bulk_rows.
// ---------------------------------------------------------------------------
template <class S> struct Rows2Cfg;
template <> struct Rows2Cfg<StoreF16> { static constexpr int NST = 5, MINB = 4; };
template <> struct Rows2Cfg<StoreF32> { static constexpr int NST = 3, MINB = 2; };

template <class S, int PAR, bool SQ>
__global__ void __launch_bounds__(32 + ROWS_MAX_NX / 2, Rows2Cfg<S>::MINB) k_bulk_rows2(const Lattice L,
                                                                                       const StreamArgs a,
                                                                                       const RowsWork w) {
    using T = typename S::T;
    constexpr int NST = Rows2Cfg<S>::NST;
    extern __shared__ __align__(128) unsigned char rows_raw[];
    __shared__ __align__(8) uint64_t full[NST], empty[NST];
    __shared__ ZoneBox zb;
    __shared__ int rowid[NST];
    __shared__ volatile int s_abort;
    __shared__ int s_issued;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nx = L.nx, nupd = nx >> 6;
    const size_t stage = rows_stage_bytes<S>(nx);
    if (tid == 0) {
        for (int q = 0; q < NST; ++q) {
            mbar_init(&full[q], 1);
            mbar_init(&empty[q], nupd);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
        s_issued = 0;
        if (SQ) zb = a.sq->zone[a.zslot];
    }
    __syncthreads();

    if (rows_idle(w)) {
    } else if (warp == 0) {
        rows_produce<S, PAR, NST>(L, a, w, rows_raw, stage, full, empty, rowid, s_abort, s_issued, lane);
    } else {
        // ---------------- update threads: nodes x0 = 2 t, x0 + 1 ----------------
        T* __restrict__ fw = static_cast<T*>(a.f);
        const int x0 = 2 * (tid - 32), nthr = nupd * 32;
        bool stored = false;   // this thread issued bulk stores (waits for them before it exits)
        for (int k = 0;; ++k) {
            const int q = k % NST;
            bool ok = mbar_wait(&full[q], (uint32_t)((k / NST) & 1));
            ok = __all_sync(0xffffffffu, ok);
            // one verdict for all update warps (named barrier 1): no warp may
            // leave the loop while another waits at that barrier
            if (!bar_and(1, nthr, ok && !s_abort)) {
                if (lane == 0 && !ok && !s_abort) { s_abort = 1; atomicOr(&a.sq->status, ST_WATCHDOG); }
                break;
            }
            const int r = rowid[q];
            if (r < 0) break;   // the same stage entry for every warp
            const int y = w.ylo + r % w.nry, z = w.zlo + r / w.nry;
            T* sb = reinterpret_cast<T*>(rows_raw + (size_t)q * stage);
            const uint8_t* sf = rows_raw + (size_t)q * stage + (size_t)Q * nx * sizeof(T);
            bool act0 = (sf[x0] & (uint8_t)~NEAR_WALL) == 0, act1 = (sf[x0 + 1] & (uint8_t)~NEAR_WALL) == 0;
            if (SQ && in_zone_axis(y, zb.lo[1], zb.w[1], L.ny, L.walls_y) &&
                in_zone_axis(z, zb.lo[2], zb.w[2], L.nz, L.walls_z)) {
                act0 = act0 && !in_zone_axis(x0, zb.lo[0], zb.w[0], nx, false);
                act1 = act1 && !in_zone_axis(x0 + 1, zb.lo[0], zb.w[0], nx, false);
            }
            float d0[Q], d1[Q];
#pragma unroll
            for (int i = 0; i < Q; ++i) {
                const T* rowi = sb + i * nx;
                if (PAR == 0 || CX(i) == 0) {           // x0, x0 + 1: one aligned pair
                    const float2 v = S::ld2(rowi + x0);
                    d0[i] = v.x; d1[i] = v.y;
                } else if (CX(i) > 0) {                 // x0 - 1 (wrapped), x0
                    d0[i] = S::ld(rowi + (x0 == 0 ? nx - 1 : x0 - 1));
                    d1[i] = S::ld(rowi + x0);
                } else {                                // x0 + 1, x0 + 2 (wrapped)
                    d0[i] = S::ld(rowi + x0 + 1);
                    d1[i] = S::ld(rowi + (x0 + 2 == nx ? 0 : x0 + 2));
                }
            }
            // every read of the stage is done; is every node of the row updated here?
            if (bar_and(1, nthr, act0 && act1)) {
                // Whole row: each direction's results form one whole row of the
                // next state (even step: A[opp(i)] of row (y, z) at x; odd step:
                // A[i] of row (y + c_iy, z + c_iz) at x + c_ix, wrapped), so they
                // are written over the stage and leave as 19 bulk copies.
                auto put = [&](int i, float v0, float v1) {
                    if (PAR == 0) {
                        S::st2(sb + OPP(i) * nx + x0, v0, v1);
                    } else if (CX(i) == 0) {
                        S::st2(sb + i * nx + x0, v0, v1);
                    } else if (CX(i) > 0) {
                        S::st(sb + i * nx + x0 + 1, v0);
                        S::st(sb + i * nx + (x0 + 2 == nx ? 0 : x0 + 2), v1);
                    } else {
                        S::st(sb + i * nx + (x0 == 0 ? nx - 1 : x0 - 1), v0);
                        S::st(sb + i * nx + x0, v1);
                    }
                };
                if (L.force_free) pair_collide<S, PAR, false>(L, a, d0, d1, put);
                else pair_collide<S, PAR, true>(L, a, d0, d1, put);
                fence_async_smem();
                bar_sync_n(1, nthr);
                if (warp == 1 && lane < Q) {
                    const int i = lane;
                    int yd = y, zd = z;
                    if (PAR == 1) {
                        yd = y + c_cy_rt(i); if (yd < 0) yd += L.ny; else if (yd >= L.ny) yd -= L.ny;
                        zd = z + c_cz_rt(i); if (zd < 0) zd += L.nz; else if (zd >= L.nz) zd -= L.nz;
                    }
                    bulk_s2g_hint(fw + (size_t)i * L.N + (size_t)nx * (yd + (size_t)L.ny * zd), sb + (size_t)i * nx,
                                  (unsigned)(nx * sizeof(T)), l2_evict_first());
                    bulk_commit();
                    bulk_wait_read();   // the stage may be refilled once the copy has read it
                    stored = true;
                }
            } else {
                const PairRow pr(L, x0, y, z, lane, act0, act1);
                if (L.force_free) pair_collide_store<S, PAR, false>(L, a, fw, pr, d0, d1);
                else pair_collide_store<S, PAR, true>(L, a, fw, pr, d0, d1);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[q]);
        }
        if (stored) bulk_wait_all();
    }
    rows_finish<NST>(w, full, s_abort, s_issued, tid);
}

// One CTA per zone block of every member: zblocks lists the (member, block)
// pairs that exist (members' zones differ in size), so no CTA is launched for
// a block beyond its member's zone.
template <class S, int PAR, bool MACRO>
__global__ void __launch_bounds__(BOUNDARY_BLOCK) k_zone_batch(const Lattice* __restrict__ lat,
                                                               const StreamArgs* __restrict__ args,
                                                               const int2* __restrict__ zblocks,
                                                               double* __restrict__ zone_part, int gzmax, BatchStep st) {
    __shared__ Lattice L;
    __shared__ StreamArgs A;
    const int2 mb = zblocks[blockIdx.x];
    const int m = mb.x, blk = mb.y;
    if (threadIdx.x == 0) {
        L = lat[m];
        StreamArgs a = args[m];
        a.zslot = st.zslot; a.do_mass = st.do_mass; a.apply_corr = st.apply_corr;
        A = a;
    }
    __syncthreads();
    __shared__ __align__(16) SqState zsq;
    __shared__ LinkStash<S> stash[Q * BOUNDARY_BLOCK];
    copy_sq_state(&zsq, A.sq);
    __syncthreads();
    NodeSums sums;
    zone_cell<S, PAR, true, MACRO>(L, A, blk * BOUNDARY_BLOCK + threadIdx.x, sums, &zsq, stash);
    if (MACRO || st.do_mass)
        block_reduce4<BOUNDARY_BLOCK>(sums.fw[0], sums.fw[1], sums.fw[2], sums.mass,
                                      zone_part + ((size_t)m * gzmax + blk) * BLOCK_PART);
}

}  // namespace lbmgpu
