// ============================================================================
//  k_aux.cuh -- kernels off the per-step path, templated on the storage form:
//  initial fill, logical population export/import, and the explicit
//  LBM::correctMass of the step-by-step interface.
// ============================================================================
#pragma once
#include "k_logical.cuh"

namespace lbmgpu {

constexpr int AUX_BLOCK = 256;
constexpr int MASS_GRID = 592;  // 4 x 148 SMs; fixed so the reduction order is fixed

// f = w_i everywhere (rho = 1, u = 0; lbm.cpp:82-84): w_i in FP64, 0 as deviation.
template <class S>
__global__ void k_fill_rest(const Lattice L, void* f) {
    const size_t total = (size_t)Q * L.N;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(k / L.N);
        Pop<S>::put(f, k, i, c_w[i]);
    }
}

// out[n] = logical f_i(n) as FP64 (+ pending mass correction on fluid nodes).
template <class S>
__global__ void k_get_pop(const Lattice L, const void* f, const uint8_t* flag, const SqState* sq, int P, int i,
                          double* out) {
    const int pend = sq->corr_pending;
    const double add = pend ? c_w[i] * sq->corr_d : 0.0;
    for (unsigned n = blockIdx.x * blockDim.x + threadIdx.x; n < L.N; n += gridDim.x * blockDim.x) {
        const int x = (int)(n % (unsigned)L.nx), y = (int)((n / (unsigned)L.nx) % (unsigned)L.ny), z = (int)(n / L.nxy);
        double v = Pop<S>::get(f, logical_slot(L, P, i, n, x, y, z), i);
        if (pend && (flag[n] & TYPE_MASK) == T_FLUID) v += add;
        out[n] = v;
    }
}

template <class S>
__global__ void k_set_pop(const Lattice L, void* f, int P, int i, const double* in) {
    for (unsigned n = blockIdx.x * blockDim.x + threadIdx.x; n < L.N; n += gridDim.x * blockDim.x) {
        const int x = (int)(n % (unsigned)L.nx), y = (int)((n / (unsigned)L.nx) % (unsigned)L.ny), z = (int)(n / L.nxy);
        Pop<S>::put(f, logical_slot(L, P, i, n, x, y, z), i, in[n]);
    }
}

// LBM::correctMass (lbm.cpp:324-339), first pass: per-block sums of the stored
// populations over fluid nodes and the fluid count.
template <class S>
__global__ void __launch_bounds__(AUX_BLOCK) k_mass_partial(const Lattice L, const void* f, const uint8_t* flag,
                                                            int P, double* part) {
    __shared__ double sm[AUX_BLOCK / 32][2];
    double m = 0.0, c = 0.0;
    for (unsigned n = blockIdx.x * blockDim.x + threadIdx.x; n < L.N; n += gridDim.x * blockDim.x) {
        if ((flag[n] & TYPE_MASK) != T_FLUID) continue;
        const int x = (int)(n % (unsigned)L.nx), y = (int)((n / (unsigned)L.nx) % (unsigned)L.ny), z = (int)(n / L.nxy);
        for (int i = 0; i < Q; ++i) m += Pop<S>::raw(f, logical_slot(L, P, i, n, x, y, z));
        c += 1.0;
    }
    for (int o = 16; o > 0; o >>= 1) {
        m += __shfl_down_sync(0xffffffffu, m, o);
        c += __shfl_down_sync(0xffffffffu, c, o);
    }
    if ((threadIdx.x & 31) == 0) { sm[threadIdx.x >> 5][0] = m; sm[threadIdx.x >> 5][1] = c; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0;
        for (int w = 0; w < AUX_BLOCK / 32; ++w) { a += sm[w][0]; b += sm[w][1]; }
        part[2 * blockIdx.x] = a; part[2 * blockIdx.x + 1] = b;
    }
}

// second pass: d = 1 - m / nf (as a deviation sum for the shifted forms). A
// correction still pending from the time loop (applied on the next load) is
// folded in: it would add w_i*d_p to every population of every fluid node,
// i.e. nf*d_p to m. The total is applied at once and nothing stays pending.
template <class S>
__global__ void k_mass_final(const double* part, int nparts, SqState* sq, double* dflag) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double m = 0, c = 0;
    for (int b = 0; b < nparts; ++b) { m += part[2 * b]; c += part[2 * b + 1]; }
    if (c == 0.0) { *dflag = 0.0; return; }
    const double dp = sq->corr_pending ? sq->corr_d : 0.0;
    m += c * dp;
    const double dn = S::shifted ? -(m / c) : 1.0 - m / c;
    sq->corr_d = dn + dp;
    sq->corr_pending = 0;
    *dflag = 1.0;
}

template <class S>
__global__ void k_mass_apply(const Lattice L, void* f, const uint8_t* flag, int P, const SqState* sq,
                             const double* dflag) {
    if (*dflag == 0.0) return;
    const double d = sq->corr_d;
    for (unsigned n = blockIdx.x * blockDim.x + threadIdx.x; n < L.N; n += gridDim.x * blockDim.x) {
        if ((flag[n] & TYPE_MASK) != T_FLUID) continue;
        const int x = (int)(n % (unsigned)L.nx), y = (int)((n / (unsigned)L.nx) % (unsigned)L.ny), z = (int)(n / L.nxy);
        for (int i = 0; i < Q; ++i) {
            const size_t k = logical_slot(L, P, i, n, x, y, z);
            Pop<S>::put(f, k, i, Pop<S>::get(f, k, i) + c_w[i] * d);
        }
    }
}

}  // namespace lbmgpu
