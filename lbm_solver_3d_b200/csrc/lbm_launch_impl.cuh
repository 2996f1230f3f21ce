// ============================================================================
//  lbm_launch_impl.cuh -- launcher table for one storage form (included by
//  exactly one translation unit per form).
// ============================================================================
#pragma once
#include "k_aux.cuh"
#include "k_batch.cuh"
#include "k_squirmer.cuh"
#include "k_stream.cuh"
#include "launch.h"

namespace lbmgpu {

template <class F>
static cudaError_t max_shared_split(F* fn) {
    return cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
}

template <class S>
static size_t rows_smem(int nx) { return (size_t)RowsCfg<S>::NST * rows_stage_bytes<S>(nx); }
template <class S>
static size_t rows2_smem(int nx) {
    if constexpr (S::shifted) return (size_t)Rows2Cfg<S>::NST * rows_stage_bytes<S>(nx);
    else return 0;
}

template <class S, int PAR, bool SQ, bool MACRO>
static void bulk_one(const Lattice& L, const StreamArgs& a, const StreamGeom& g, cudaStream_t st) {
    if (g.rows_grid) {   // rows staged in shared memory (every step; sums in k_bulk's order)
        const RowsWork w{g.rows_nry, g.rows_n, g.rows_ylo, g.rows_zlo, g.rows_reserve, a.row_claim};
        if constexpr (S::shifted && !MACRO) {
            if (g.rows_pairs && !a.do_mass) {   // no sums this step: two nodes per update thread
                k_bulk_rows2<S, PAR, SQ><<<g.rows_grid, 32 + L.nx / 2, rows2_smem<S>(L.nx), st>>>(L, a, w);
                return;
            }
        }
        if (MACRO || a.do_mass)
            k_bulk_rows<S, PAR, SQ, MACRO, true><<<g.rows_grid, 32 + L.nx, rows_smem<S>(L.nx), st>>>(L, a, w);
        else
            k_bulk_rows<S, PAR, SQ, false, false><<<g.rows_grid, 32 + L.nx, rows_smem<S>(L.nx), st>>>(L, a, w);
        return;
    }
    if constexpr (S::shifted && !MACRO) {
        if (!a.do_mass && g.pair.x) {   // no sums this step: two x-adjacent nodes per thread
            if (L.force_free) k_bulk_pair<S, PAR, SQ, false><<<g.pair, g.pair_block, 0, st>>>(L, a);
            else k_bulk_pair<S, PAR, SQ, true><<<g.pair, g.pair_block, 0, st>>>(L, a);
            return;
        }
    }
    if (!MACRO && !a.do_mass && g.flat.x) {   // no sums this step: whole rows of nodes per block
        if (!S::shifted && g.dense) k_bulk_flat<S, PAR, SQ, true><<<g.flat, 256, 0, st>>>(L, a);
        else k_bulk_flat<S, PAR, SQ><<<g.flat, 256, 0, st>>>(L, a);
        return;
    }
    if constexpr (!S::shifted) {
        if (g.dense) {
            k_bulk<S, PAR, SQ, MACRO, false, true><<<g.grid, g.block, 0, st>>>(L, a);
            return;
        }
    }
    k_bulk<S, PAR, SQ, MACRO, false><<<g.grid, g.block, 0, st>>>(L, a);
}
// Launch with programmatic stream serialisation: the kernel may be scheduled
// while its predecessor in the stream finishes, and waits for it in pdl_wait().
// Used on the stream of the chain wall rows -> zone -> squirmer update, whose
// kernels follow one another step after step.
template <class... KArgs, class... Args>
static void launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kern, args...);
}

template <class S, int PAR, bool SQ, bool MACRO>
static void wallrows_one(const Lattice& L, const StreamArgs& a, const StreamGeom& g, cudaStream_t st) {
    if (g.nwallrows) launch_pdl(k_bulk<S, PAR, SQ, MACRO, true>, dim3(g.grid.x, g.nwallrows, 1), g.block, 0, st, L, a);
}
template <class S, int PAR, bool SQ, bool MACRO>
static void zone_one(const Lattice& L, const StreamArgs& a, const StreamGeom& g, cudaStream_t st) {
    if (g.bgrid) launch_pdl(k_zone<S, PAR, SQ, MACRO>, dim3(g.bgrid), dim3(BOUNDARY_BLOCK), 0, st, L, a);
}

#define LBMGPU_DISPATCH(FN)                                                                                  \
    template <class S>                                                                                       \
    static void FN##_dispatch(int par, bool sq, bool macro, const Lattice& L, const StreamArgs& a,          \
                              const StreamGeom& g, cudaStream_t st) {                                        \
        switch ((par ? 4 : 0) | (sq ? 2 : 0) | (macro ? 1 : 0)) {                                            \
            case 0: FN##_one<S, 0, false, false>(L, a, g, st); break;                                        \
            case 1: FN##_one<S, 0, false, true>(L, a, g, st); break;                                         \
            case 2: FN##_one<S, 0, true, false>(L, a, g, st); break;                                         \
            case 3: FN##_one<S, 0, true, true>(L, a, g, st); break;                                          \
            case 4: FN##_one<S, 1, false, false>(L, a, g, st); break;                                        \
            case 5: FN##_one<S, 1, false, true>(L, a, g, st); break;                                         \
            case 6: FN##_one<S, 1, true, false>(L, a, g, st); break;                                         \
            default: FN##_one<S, 1, true, true>(L, a, g, st); break;                                         \
        }                                                                                                    \
    }
LBMGPU_DISPATCH(bulk)
LBMGPU_DISPATCH(wallrows)
LBMGPU_DISPATCH(zone)
#undef LBMGPU_DISPATCH

inline size_t squirmer_smem() { return sizeof(ChgSh) * SQ_BATCH; }

template <class S>
static void squirmer_launch(const Lattice& L, const SqArgs& a, cudaStream_t st) {
    launch_pdl(k_squirmer<S>, dim3(1), dim3(SQ_THREADS), squirmer_smem(), st, L, a);
}

template <class S>
static void fill_launch(const Lattice& L, void* f, cudaStream_t st) {
    k_fill_rest<S><<<1184, AUX_BLOCK, 0, st>>>(L, f);
}

template <class S>
static void get_pop_launch(const Lattice& L, const void* f, const uint8_t* flag, const SqState* sq, int P, int i,
                           double* out, cudaStream_t st) {
    k_get_pop<S><<<1184, AUX_BLOCK, 0, st>>>(L, f, flag, sq, P, i, out);
}

template <class S>
static void set_pop_launch(const Lattice& L, void* f, int P, int i, const double* in, cudaStream_t st) {
    k_set_pop<S><<<1184, AUX_BLOCK, 0, st>>>(L, f, P, i, in);
}

template <class S>
static void correct_mass_launch(const Lattice& L, void* f, const uint8_t* flag, int P, SqState* sq, double* part,
                                double* dflag, cudaStream_t st) {
    k_mass_partial<S><<<MASS_GRID, AUX_BLOCK, 0, st>>>(L, f, flag, P, part);
    k_mass_final<S><<<1, 32, 0, st>>>(part, MASS_GRID, sq, dflag);
    k_mass_apply<S><<<1184, AUX_BLOCK, 0, st>>>(L, f, flag, P, sq, dflag);
}

template <class S, int PAR, bool MACRO, bool WR>
static void batch_bulk_tx(int tx, int grid, const BatchArgs& b, BatchStep st, cudaStream_t s) {
    const RowRef* rows = WR ? b.wrows : b.rows;
    const int n = WR ? b.nwrows : b.nrows;
    double* part = b.row_part;
    if (n == 0) return;
    switch (tx) {
        case 32: k_bulk_batch<S, PAR, MACRO, WR, 32><<<grid, 256, 0, s>>>(b.lat, b.args, rows, n, part, st); break;
        case 64: k_bulk_batch<S, PAR, MACRO, WR, 64><<<grid, 256, 0, s>>>(b.lat, b.args, rows, n, part, st); break;
        default: k_bulk_batch<S, PAR, MACRO, WR, 128><<<grid, 256, 0, s>>>(b.lat, b.args, rows, n, part, st); break;
    }
}

template <class S>
static void batch_bulk_launch(int par, bool macro, bool wr, int tx, int grid, const BatchArgs& b, BatchStep st,
                              cudaStream_t s) {
    switch ((par ? 4 : 0) | (macro ? 2 : 0) | (wr ? 1 : 0)) {
        case 0: batch_bulk_tx<S, 0, false, false>(tx, grid, b, st, s); break;
        case 1: batch_bulk_tx<S, 0, false, true>(tx, grid, b, st, s); break;
        case 2: batch_bulk_tx<S, 0, true, false>(tx, grid, b, st, s); break;
        case 3: batch_bulk_tx<S, 0, true, true>(tx, grid, b, st, s); break;
        case 4: batch_bulk_tx<S, 1, false, false>(tx, grid, b, st, s); break;
        case 5: batch_bulk_tx<S, 1, false, true>(tx, grid, b, st, s); break;
        case 6: batch_bulk_tx<S, 1, true, false>(tx, grid, b, st, s); break;
        default: batch_bulk_tx<S, 1, true, true>(tx, grid, b, st, s); break;
    }
}

template <class S, int PAR, bool MACRO, bool WR>
static void rowcta_one(const BatchArgs& b, BatchStep st, cudaStream_t s) {
    const RowRef* rows = WR ? b.wrows : b.rows;
    const int n = WR ? b.nwrows : b.nrows;
    if (n) k_bulk_rowcta<S, PAR, MACRO, WR><<<n, ROWCTA_THREADS, 0, s>>>(b.lat, b.args, rows, b.row_part, st);
}

template <class S>
static void batch_rowcta_launch(int par, bool macro, bool wr, const BatchArgs& b, BatchStep st, cudaStream_t s) {
    switch ((par ? 4 : 0) | (macro ? 2 : 0) | (wr ? 1 : 0)) {
        case 0: rowcta_one<S, 0, false, false>(b, st, s); break;
        case 1: rowcta_one<S, 0, false, true>(b, st, s); break;
        case 2: rowcta_one<S, 0, true, false>(b, st, s); break;
        case 3: rowcta_one<S, 0, true, true>(b, st, s); break;
        case 4: rowcta_one<S, 1, false, false>(b, st, s); break;
        case 5: rowcta_one<S, 1, false, true>(b, st, s); break;
        case 6: rowcta_one<S, 1, true, false>(b, st, s); break;
        default: rowcta_one<S, 1, true, true>(b, st, s); break;
    }
}

template <class S, int PAR, bool MACRO>
static void chunk_one(bool sums, const BatchArgs& b, BatchStep st, cudaStream_t s) {
    if (b.nchunks == 0) return;
    k_bulk_chunk<S, PAR, MACRO><<<(b.nchunks + CHUNK_WARPS - 1) / CHUNK_WARPS, 32 * CHUNK_WARPS, 0, s>>>(
        b.lat, b.args, b.chunks, b.nchunks, b.chunk_part, st);
    if (sums) k_fold_chunks<<<(b.nrows + 255) / 256, 256, 0, s>>>(b.rowchunks, b.nrows, b.chunk_part, b.row_part);
}

template <class S, int PAR, bool MACRO>
static void chunkp_one(int grid, bool sums, const BatchArgs& b, BatchStep st, cudaStream_t s) {
    if (b.nchunks == 0) return;
    if (!sums && b.nflat > 0) {   // no partial sums this step: the run pieces
        k_bulk_chunkp<S, PAR, MACRO, true><<<grid, 32 * CHUNK_WARPS, 0, s>>>(b.lat, b.args, b.flat, b.nflat, nullptr, st);
        return;
    }
    k_bulk_chunkp<S, PAR, MACRO><<<grid, 32 * CHUNK_WARPS, 0, s>>>(b.lat, b.args, b.chunks, b.nchunks, b.chunk_part, st);
    if (sums) k_fold_chunks<<<(b.nrows + 255) / 256, 256, 0, s>>>(b.rowchunks, b.nrows, b.chunk_part, b.row_part);
}

template <class S>
static int chunkp_occupancy() {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_bulk_chunkp<S, 1, false>, 32 * CHUNK_WARPS, 0) != cudaSuccess)
        return 4;
    return n > 0 ? n : 1;
}

// grid > 0: the persistent variant with that many CTAs
template <class S>
static void batch_chunk_launch(int par, bool macro, bool sums, int grid, const BatchArgs& b, BatchStep st,
                               cudaStream_t s) {
    switch ((grid > 0 ? 4 : 0) | (par ? 2 : 0) | (macro ? 1 : 0)) {
        case 0: chunk_one<S, 0, false>(sums, b, st, s); break;
        case 1: chunk_one<S, 0, true>(sums, b, st, s); break;
        case 2: chunk_one<S, 1, false>(sums, b, st, s); break;
        case 3: chunk_one<S, 1, true>(sums, b, st, s); break;
        case 4: chunkp_one<S, 0, false>(grid, sums, b, st, s); break;
        case 5: chunkp_one<S, 0, true>(grid, sums, b, st, s); break;
        case 6: chunkp_one<S, 1, false>(grid, sums, b, st, s); break;
        default: chunkp_one<S, 1, true>(grid, sums, b, st, s); break;
    }
}

template <class S, int PAR, bool MACRO, int NST>
static void staged_one(int grid, const BatchArgs& b, BatchStep st, cudaStream_t s) {
    const size_t smem = (size_t)NST * ((size_t)Q * b.cap * sizeof(typename S::T) + b.fcap);
    k_bulk_staged<S, PAR, MACRO, NST><<<grid, STAGED_THREADS, smem, s>>>(b.lat, b.args, b.rows, b.bounds, b.row_part,
                                                                        st, b.cap, b.fcap);
}

template <class S>
static void batch_staged_launch(int par, bool macro, int nst, int grid, const BatchArgs& b, BatchStep st,
                                cudaStream_t s) {
    if (b.nrows == 0) return;
    const int sel = (par ? 4 : 0) | (macro ? 2 : 0) | (nst == 4 ? 1 : 0);
    switch (sel) {
        case 0: staged_one<S, 0, false, 3>(grid, b, st, s); break;
        case 1: staged_one<S, 0, false, 4>(grid, b, st, s); break;
        case 2: staged_one<S, 0, true, 3>(grid, b, st, s); break;
        case 3: staged_one<S, 0, true, 4>(grid, b, st, s); break;
        case 4: staged_one<S, 1, false, 3>(grid, b, st, s); break;
        case 5: staged_one<S, 1, false, 4>(grid, b, st, s); break;
        case 6: staged_one<S, 1, true, 3>(grid, b, st, s); break;
        default: staged_one<S, 1, true, 4>(grid, b, st, s); break;
    }
}

template <class S, int PAR, bool MACRO, int NST>
static cudaError_t staged_attr() {
    return cudaFuncSetAttribute(k_bulk_staged<S, PAR, MACRO, NST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                200 * 1024);
}

template <class S>
static void batch_zone_launch(int par, bool macro, const BatchArgs& b, BatchStep st, cudaStream_t s) {
    if (b.nzblocks == 0) return;
    const dim3 grid(b.nzblocks);
    switch ((par ? 2 : 0) | (macro ? 1 : 0)) {
        case 0: k_zone_batch<S, 0, false><<<grid, BOUNDARY_BLOCK, 0, s>>>(b.lat, b.args, b.zblocks, b.zone_part, b.gzmax, st); break;
        case 1: k_zone_batch<S, 0, true><<<grid, BOUNDARY_BLOCK, 0, s>>>(b.lat, b.args, b.zblocks, b.zone_part, b.gzmax, st); break;
        case 2: k_zone_batch<S, 1, false><<<grid, BOUNDARY_BLOCK, 0, s>>>(b.lat, b.args, b.zblocks, b.zone_part, b.gzmax, st); break;
        default: k_zone_batch<S, 1, true><<<grid, BOUNDARY_BLOCK, 0, s>>>(b.lat, b.args, b.zblocks, b.zone_part, b.gzmax, st); break;
    }
}

template <class S>
static void batch_squirmer_launch(const BatchArgs& b, SqStep st, cudaStream_t s) {
    k_squirmer_batch<S><<<b.nmembers, SQ_THREADS, squirmer_smem(), s>>>(b.lat, b.sqargs, st);
}

template <class S>
static void batch_runs_launch(int par, int grid, const BatchArgs& b, BatchStep st, cudaStream_t s) {
    if (b.nruns == 0) return;
    const size_t smem = (size_t)RunsCfg<S>::NST * runs_stage_bytes<S>();
    if (par) k_bulk_runs<S, 1><<<grid, RUNS_THREADS, smem, s>>>(b.lat, b.args, b.runs, b.nruns, st);
    else k_bulk_runs<S, 0><<<grid, RUNS_THREADS, smem, s>>>(b.lat, b.args, b.runs, b.nruns, st);
}

template <class S>
static int rows_occupancy(int nx, bool pairs) {
    int n = 0;
    cudaError_t e;
    if constexpr (S::shifted) {
        if (pairs) {
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_bulk_rows2<S, 0, true>, 32 + nx / 2, rows2_smem<S>(nx));
            return e == cudaSuccess ? n : 0;
        }
    }
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_bulk_rows<S, 0, true, false, false>, 32 + nx, rows_smem<S>(nx));
    return e == cudaSuccess ? n : 0;
}

template <class S>
static cudaError_t prepare_launch() {
    cudaError_t e = cudaFuncSetAttribute(k_squirmer<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)squirmer_smem());
    if (e != cudaSuccess) return e;
    const int runs_smem = (int)((size_t)RunsCfg<S>::NST * runs_stage_bytes<S>());
    for (auto fn : {k_bulk_runs<S, 0>, k_bulk_runs<S, 1>}) {
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, runs_smem);
        if (e != cudaSuccess) return e;
    }
    if constexpr (S::shifted) {
        const int r2 = (int)rows2_smem<S>(ROWS_MAX_NX);
        for (auto fn : {k_bulk_rows2<S, 0, false>, k_bulk_rows2<S, 0, true>, k_bulk_rows2<S, 1, false>,
                        k_bulk_rows2<S, 1, true>}) {
            e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, r2);
            if (e != cudaSuccess) return e;
        }
    }
    const int rs = (int)rows_smem<S>(ROWS_MAX_NX);
    for (auto fn : {k_bulk_rows<S, 0, false, false, false>, k_bulk_rows<S, 0, true, false, false>,
                    k_bulk_rows<S, 1, false, false, false>, k_bulk_rows<S, 1, true, false, false>,
                    k_bulk_rows<S, 0, false, false, true>, k_bulk_rows<S, 0, true, false, true>,
                    k_bulk_rows<S, 1, false, false, true>, k_bulk_rows<S, 1, true, false, true>,
                    k_bulk_rows<S, 0, false, true, true>, k_bulk_rows<S, 0, true, true, true>,
                    k_bulk_rows<S, 1, false, true, true>, k_bulk_rows<S, 1, true, true, true>}) {
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, rs);
        if (e != cudaSuccess) return e;
    }
    e = cudaFuncSetAttribute(k_squirmer_batch<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)squirmer_smem());
    if (e != cudaSuccess) return e;
    // The staged-row bulk and the kernels of the second stream that should run
    // beside it (zone, squirmer update, wall rows) ask for the largest shared
    // memory split. Left to the default, two bulk CTAs (2 x 77 KB) get the
    // 164 KB split, whose 7 KB left over holds no zone CTA (11 KB), and the
    // zone of the next step then waits for the bulk to end.
    for (auto fn : {k_bulk_rows<S, 0, false, false, false>, k_bulk_rows<S, 0, true, false, false>,
                    k_bulk_rows<S, 1, false, false, false>, k_bulk_rows<S, 1, true, false, false>,
                    k_bulk_rows<S, 0, false, false, true>, k_bulk_rows<S, 0, true, false, true>,
                    k_bulk_rows<S, 1, false, false, true>, k_bulk_rows<S, 1, true, false, true>,
                    k_bulk_rows<S, 0, false, true, true>, k_bulk_rows<S, 0, true, true, true>,
                    k_bulk_rows<S, 1, false, true, true>, k_bulk_rows<S, 1, true, true, true>}) {
        e = max_shared_split(fn);
        if (e != cudaSuccess) return e;
    }
    if constexpr (S::shifted) {
        for (auto fn : {k_bulk_rows2<S, 0, false>, k_bulk_rows2<S, 0, true>, k_bulk_rows2<S, 1, false>,
                        k_bulk_rows2<S, 1, true>}) {
            e = max_shared_split(fn);
            if (e != cudaSuccess) return e;
        }
    }
    for (auto fn : {k_zone<S, 0, false, false>, k_zone<S, 0, false, true>, k_zone<S, 0, true, false>,
                    k_zone<S, 0, true, true>, k_zone<S, 1, false, false>, k_zone<S, 1, false, true>,
                    k_zone<S, 1, true, false>, k_zone<S, 1, true, true>}) {
        e = max_shared_split(fn);
        if (e != cudaSuccess) return e;
    }
    for (auto fn : {k_bulk<S, 0, false, false, true>, k_bulk<S, 0, false, true, true>, k_bulk<S, 0, true, false, true>,
                    k_bulk<S, 0, true, true, true>, k_bulk<S, 1, false, false, true>, k_bulk<S, 1, false, true, true>,
                    k_bulk<S, 1, true, false, true>, k_bulk<S, 1, true, true, true>}) {
        e = max_shared_split(fn);
        if (e != cudaSuccess) return e;
    }
    e = max_shared_split(k_squirmer<S>);
    if (e != cudaSuccess) return e;
    cudaError_t es[8] = {staged_attr<S, 0, false, 3>(), staged_attr<S, 0, false, 4>(), staged_attr<S, 0, true, 3>(),
                         staged_attr<S, 0, true, 4>(),  staged_attr<S, 1, false, 3>(), staged_attr<S, 1, false, 4>(),
                         staged_attr<S, 1, true, 3>(),  staged_attr<S, 1, true, 4>()};
    for (cudaError_t x : es)
        if (x != cudaSuccess) return x;
    return cudaSuccess;
}

template <class S>
static Launchers make_launchers() {
    Launchers l;
    l.bulk = &bulk_dispatch<S>;
    l.wallrows = &wallrows_dispatch<S>;
    l.zone = &zone_dispatch<S>;
    l.squirmer = &squirmer_launch<S>;
    l.fill_rest = &fill_launch<S>;
    l.get_pop = &get_pop_launch<S>;
    l.set_pop = &set_pop_launch<S>;
    l.correct_mass = &correct_mass_launch<S>;
    l.prepare = &prepare_launch<S>;
    l.batch_bulk = &batch_bulk_launch<S>;
    l.batch_zone = &batch_zone_launch<S>;
    l.batch_squirmer = &batch_squirmer_launch<S>;
    l.batch_staged = &batch_staged_launch<S>;
    l.batch_rowcta = &batch_rowcta_launch<S>;
    l.batch_chunk = &batch_chunk_launch<S>;
    l.chunkp_ctas_per_sm = &chunkp_occupancy<S>;
    l.rows_ctas_per_sm = &rows_occupancy<S>;
    l.batch_runs = &batch_runs_launch<S>;
    l.runs_max_nodes = RunsCfg<S>::NODES;
    l.esize = sizeof(typename S::T);
    return l;
}

}  // namespace lbmgpu
