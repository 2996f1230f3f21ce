// ============================================================================
//  launch.h -- host-side launchers exported by the per-precision translation
//  units (lbm_f64.cu is compiled without FMA contraction so its FP64
//  arithmetic matches the reference's; lbm_lp.cu holds the FP32/FP16 forms).
// ============================================================================
#pragma once
#include <cuda_runtime.h>

#include "lbm_common.cuh"

namespace lbmgpu {

struct SqArgs;

// launch geometry of one step: the bulk kernel's 3-D grid and the zone
// kernel's 1-D grid (0: no zone and no wall nodes)
struct StreamGeom {
    dim3 grid, block;
    unsigned bgrid;
    unsigned nwallrows;  // rows next to a wall (0: none)
    bool dense;          // FP64: the bulk at 3 CTAs/SM (a long bulk)
    dim3 flat;           // k_bulk_flat's grid for steps without sums (x = 0: not used)
    dim3 pair, pair_block;   // k_bulk_pair's grid and block for steps without sums (x = 0: not used)
    // k_bulk_rows (rows staged in shared memory) for steps without sums: grid
    // (rows_grid = 0: not used), interior rows nry x (rows_n / nry) from (ylo, zlo)
    unsigned rows_grid = 0;
    int rows_nry = 0, rows_n = 0, rows_ylo = 0, rows_zlo = 0;
    bool rows_pairs = false;   // two nodes per update thread (k_bulk_rows2)
    int rows_reserve = 0;      // SMs (lowest %smid) the rows grid leaves to the squirmer update
};

struct SqArgs;

// device tables of an ensemble
struct BatchArgs {
    const Lattice* lat;
    const StreamArgs* args;
    const SqArgs* sqargs;
    const RowRef* rows;  int nrows;    // rows away from walls
    const RowRef* wrows; int nwrows;   // rows next to a wall
    double* row_part;                  // one entry per (member, y, z) row, both row kinds
    double* zone_part;
    int gzmax;                         // zone-block entries per member in zone_part
    const int2* zblocks; int nzblocks; // (member, block) of every zone block that exists
    int nmembers;
    const MemberParts* parts;
    const int* bounds;                 // staged kernel: row range of each CTA (grid + 1 entries)
    const ChunkRef* chunks; int nchunks;   // chunk kernel: 32-node pieces of the rows away from walls
    const RowChunks* rowchunks;        // chunk kernel: each row's chunks
    const ChunkRef* flat; int nflat;   // persistent chunk kernel, steps without sums: 32-node pieces of row runs
    const int4* runs; int nruns;       // staged-run kernel: (member, y0, z, rows) of consecutive interior rows
    double* chunk_part;                // chunk kernel: partial sums per chunk
    int cap;                           // staged kernel: elements per staged direction-row
    int fcap;                          // staged kernel: bytes per staged flag row
};

struct Launchers {
    // the two collide-stream kernels of one time step
    void (*bulk)(int par, bool sq, bool macro, const Lattice& L, const StreamArgs& a, const StreamGeom& g,
                 cudaStream_t st);
    void (*wallrows)(int par, bool sq, bool macro, const Lattice& L, const StreamArgs& a, const StreamGeom& g,
                     cudaStream_t st);
    void (*zone)(int par, bool sq, bool macro, const Lattice& L, const StreamArgs& a, const StreamGeom& g,
                 cudaStream_t st);
    // the squirmer update (stages: STAGE_* bits)
    void (*squirmer)(const Lattice& L, const SqArgs& a, cudaStream_t st);
    void (*fill_rest)(const Lattice& L, void* f, cudaStream_t st);
    void (*get_pop)(const Lattice& L, const void* f, const uint8_t* flag, const SqState* sq, int P, int i,
                    double* out, cudaStream_t st);
    void (*set_pop)(const Lattice& L, void* f, int P, int i, const double* in, cudaStream_t st);
    // explicit mass correction: partial sums, final, apply
    void (*correct_mass)(const Lattice& L, void* f, const uint8_t* flag, int P, SqState* sq, double* part,
                         double* dflag, cudaStream_t st);
    cudaError_t (*prepare)();  // one-time function attributes
    // ensembles: the bulk rows (tx threads per row, grid CTAs), the zones,
    // the squirmer updates and the wall forces of all members
    void (*batch_bulk)(int par, bool macro, bool wallrows, int tx, int grid, const BatchArgs& b, BatchStep st,
                       cudaStream_t s);
    void (*batch_zone)(int par, bool macro, const BatchArgs& b, BatchStep st, cudaStream_t s);
    // the rows away from walls through shared-memory stages (k_bulk_staged)
    void (*batch_staged)(int par, bool macro, int nst, int grid, const BatchArgs& b, BatchStep st, cudaStream_t s);
    // one warp per 32-node chunk (k_bulk_chunk, then k_fold_chunks when summing)
    void (*batch_chunk)(int par, bool macro, bool sums, int grid, const BatchArgs& b, BatchStep st, cudaStream_t s);
    int (*chunkp_ctas_per_sm)();   // resident CTAs per SM of the persistent chunk kernel
    int (*rows_ctas_per_sm)(int nx, bool pairs);   // resident CTAs per SM of k_bulk_rows(2) for rows of nx nodes
    // rows away from walls in runs staged through shared memory (k_bulk_runs, steps without sums)
    void (*batch_runs)(int par, int grid, const BatchArgs& b, BatchStep st, cudaStream_t s);
    int runs_max_nodes;                // nodes per run
    // one CTA per row (k_bulk_rowcta): rows away from walls, or next to one
    void (*batch_rowcta)(int par, bool macro, bool wallrows, const BatchArgs& b, BatchStep st, cudaStream_t s);
    size_t esize;
    void (*batch_squirmer)(const BatchArgs& b, SqStep st, cudaStream_t s);
};

const Launchers& launchers_f64();
const Launchers& launchers_f32();
const Launchers& launchers_f16();

size_t squirmer_smem_bytes();

}  // namespace lbmgpu
