// ============================================================================
//  k_logical.cuh -- access to logical populations f_i(n) of the AA state
//  (see k_stream.cuh for the mapping), and their FP64 values in every
//  storage form. Used off the hot loop: remap, population export/import,
//  explicit mass correction.
// ============================================================================
#pragma once
#include "lbm_common.cuh"

namespace lbmgpu {

// Wrapped neighbour n + c_i for runtime i (lbm.cpp:180-184 / :305).
__device__ __forceinline__ unsigned nbr_rt(const Lattice& L, int x, int y, int z, int cx, int cy, int cz) {
    int xn = x + cx, yn = y + cy, zn = z + cz;
    if (xn < 0) xn += L.nx; else if (xn >= L.nx) xn -= L.nx;
    if (yn < 0) yn += L.ny; else if (yn >= L.ny) yn -= L.ny;
    if (zn < 0) zn += L.nz; else if (zn >= L.nz) zn -= L.nz;
    return (unsigned)xn + (unsigned)L.nx * ((unsigned)yn + (unsigned)L.ny * (unsigned)zn);
}

// Runtime velocity table (device), same order as lattice.hpp:18-23.
static __device__ __constant__ int c_cx[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
static __device__ __constant__ int c_cy[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
static __device__ __constant__ int c_cz[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
static __device__ __constant__ double c_w[Q] = {1.0 / 3.0,
                                         1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 18,
                                         1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36,
                                         1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36};

__device__ __forceinline__ int opp_rt(int i) { return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1); }

// Index of the storage slot holding logical f_i(n) in a state of parity P.
__device__ __forceinline__ size_t logical_slot(const Lattice& L, int P, int i, unsigned n, int x, int y, int z) {
    if (P == 0 || i == 0) return (size_t)i * L.N + n;
    const int o = opp_rt(i);  // n - c_i = n + c_opp(i)
    return (size_t)o * L.N + nbr_rt(L, x, y, z, c_cx[o], c_cy[o], c_cz[o]);
}

// Stored number <-> FP64 population for each storage form. raw() is the stored
// number as a double (f itself for FP64, the deviation f - w_i otherwise);
// get() is the population; put() stores a population; stored_raw() is what
// put() would store, as a double (used by the mass balance).
template <class S> struct Pop;
template <> struct Pop<StoreF64> {
    __device__ static double raw(const void* f, size_t k) { return static_cast<const double*>(f)[k]; }
    __device__ static double get(const void* f, size_t k, int) { return raw(f, k); }
    __device__ static void put(void* f, size_t k, int, double v) { static_cast<double*>(f)[k] = v; }
    __device__ static double stored_raw(double v, int) { return v; }
};
template <> struct Pop<StoreF32> {
    __device__ static double raw(const void* f, size_t k) { return (double)static_cast<const float*>(f)[k]; }
    __device__ static double get(const void* f, size_t k, int i) { return c_w[i] + raw(f, k); }
    __device__ static void put(void* f, size_t k, int i, double v) { static_cast<float*>(f)[k] = (float)(v - c_w[i]); }
    __device__ static double stored_raw(double v, int i) { return (double)(float)(v - c_w[i]); }
};
template <> struct Pop<StoreF16> {
    __device__ static double raw(const void* f, size_t k) {
        return (double)(__half2float(static_cast<const __half*>(f)[k]) * FP16_INV_SCALE);
    }
    __device__ static double get(const void* f, size_t k, int i) { return c_w[i] + raw(f, k); }
    __device__ static void put(void* f, size_t k, int i, double v) {
        static_cast<__half*>(f)[k] = __float2half_rn((float)(v - c_w[i]) * FP16_SCALE);
    }
    __device__ static double stored_raw(double v, int i) {
        return (double)(__half2float(__float2half_rn((float)(v - c_w[i]) * FP16_SCALE)) * FP16_INV_SCALE);
    }
};

}  // namespace lbmgpu
