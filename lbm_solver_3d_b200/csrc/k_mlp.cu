// ============================================================================
//  k_mlp.cu -- the swimmer surrogate network: a 4 -> 64 -> 64 -> 64 -> 3
//  multilayer perceptron with SiLU after each hidden layer, trained and
//  evaluated by the kernels below (no library GEMM, no autograd).
//
//  One CTA owns a tile of MLP_T = 32 samples and runs the whole network on it
//  from shared memory: forward through the four layers, the mean-squared loss,
//  and backward to the weight and bias gradients of the tile, which it writes
//  to its own row of a partials array. k_mlp_adam then sums the rows in a
//  fixed order (deterministic) and applies one Adam step to the FP32 master
//  parameters.
//
//  Every product is a warp-tiled GEMM on 16 x 8 output tiles:
//    BF16 = true   mma.sync m16n8k16 with BF16 operands (rounded from the FP32
//                  values in shared memory) and FP32 accumulation;
//    BF16 = false  the same tiles with FP32 FMAs (k in ascending order).
//  The layer shapes are padded to multiples of the tile (inputs 4 -> 16,
//  outputs 3 -> 16) with zeros.
//
//  Parameter layout (FP32, the order of the C ABI): W1[64][4] b1[64]
//  W2[64][64] b2[64] W3[64][64] b3[64] W4[3][64] b4[3], W[out][in].
// ============================================================================
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/lbmgpu.h"

namespace {

constexpr int NI = LBMGPU_MLP_IN, NH = LBMGPU_MLP_HIDDEN, NO = LBMGPU_MLP_OUT;
constexpr int NP = LBMGPU_MLP_NPARAMS;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + NH * NI, OFF_W2 = OFF_B1 + NH, OFF_B2 = OFF_W2 + NH * NH,
              OFF_W3 = OFF_B2 + NH, OFF_B3 = OFF_W3 + NH * NH, OFF_W4 = OFF_B3 + NH, OFF_B4 = OFF_W4 + NO * NH;
static_assert(OFF_B4 + NO == NP, "parameter layout");

constexpr int MLP_T = 32;        // samples per CTA
constexpr int MLP_THREADS = 256; // 8 warps
constexpr int PI_ = 16;          // padded input width
constexpr int PO = 16;           // padded output width

// shared-memory layout (floats)
struct Smem {
    float W1[NH * PI_], W2[NH * NH], W3[NH * NH], W4[PO * NH];
    float b1[NH], b2[NH], b3[NH], b4[PO];
    float H0[MLP_T * PI_];
    float Z1[MLP_T * NH], H1[MLP_T * NH], Z2[MLP_T * NH], H2[MLP_T * NH], Z3[MLP_T * NH], H3[MLP_T * NH];
    float Y[MLP_T * PO];
    float dA[MLP_T * NH], dB[MLP_T * NH];
    float red[MLP_THREADS / 32];
};

__device__ __forceinline__ float sigmoid(float z) { return 1.0f / (1.0f + expf(-z)); }
__device__ __forceinline__ float silu(float z) { return z * sigmoid(z); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = sigmoid(z);
    return s * (1.0f + z * (1.0f - s));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);   // .x (low half) = lo
    uint32_t u;
    memcpy(&u, &v, 4);
    return u;
}

// C(m, n) = sum_k A(m, k) B(k, n) for an M x N output (multiples of 16 and 8),
// K a multiple of 16. A(m, k) = A[m*as0 + k*as1], B(k, n) = B[k*bs0 + n*bs1].
// Each warp takes 16 x 8 tiles in turn; out(m, n, value) receives every element.
template <bool BF16, class Out>
__device__ __forceinline__ void gemm(int M, int N, int K, const float* A, int as0, int as1, const float* B, int bs0,
                                     int bs1, Out out) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, tq = lane & 3;
    const int tn_count = N / 8, tiles = (M / 16) * tn_count;
    for (int t = warp; t < tiles; t += MLP_THREADS / 32) {
        const int m0 = (t / tn_count) * 16, n0 = (t % tn_count) * 8;
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        if constexpr (BF16) {
            for (int k0 = 0; k0 < K; k0 += 16) {
                auto a = [&](int r, int k) { return A[(m0 + r) * as0 + (k0 + k) * as1]; };
                auto b = [&](int k, int n) { return B[(k0 + k) * bs0 + (n0 + n) * bs1]; };
                const uint32_t a0 = pack_bf16(a(g, 2 * tq), a(g, 2 * tq + 1));
                const uint32_t a1 = pack_bf16(a(g + 8, 2 * tq), a(g + 8, 2 * tq + 1));
                const uint32_t a2 = pack_bf16(a(g, 2 * tq + 8), a(g, 2 * tq + 9));
                const uint32_t a3 = pack_bf16(a(g + 8, 2 * tq + 8), a(g + 8, 2 * tq + 9));
                const uint32_t b0 = pack_bf16(b(2 * tq, g), b(2 * tq + 1, g));
                const uint32_t b1 = pack_bf16(b(2 * tq + 8, g), b(2 * tq + 9, g));
                asm volatile(
                    "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                    "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
                    : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                    : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
            }
        } else {
            const int r0 = m0 + g, r1 = m0 + g + 8, q0 = n0 + 2 * tq, q1 = q0 + 1;
            for (int k = 0; k < K; ++k) {
                const float x0 = A[r0 * as0 + k * as1], x1 = A[r1 * as0 + k * as1];
                const float y0 = B[k * bs0 + q0 * bs1], y1 = B[k * bs0 + q1 * bs1];
                c[0] = fmaf(x0, y0, c[0]); c[1] = fmaf(x0, y1, c[1]);
                c[2] = fmaf(x1, y0, c[2]); c[3] = fmaf(x1, y1, c[3]);
            }
        }
        out(m0 + g, n0 + 2 * tq, c[0]);
        out(m0 + g, n0 + 2 * tq + 1, c[1]);
        out(m0 + g + 8, n0 + 2 * tq, c[2]);
        out(m0 + g + 8, n0 + 2 * tq + 1, c[3]);
    }
}

// Forward (and, when TRAIN, backward) of one tile of MLP_T samples.
//   X [n][4], Yt [n][3] (targets, TRAIN), idx: sample order (NULL: identity);
//   TRAIN: grad_part[blockIdx.x][NP] and loss_part[blockIdx.x] = sum of
//          squared errors of the tile; dL/dY = 2 (Y - Yt) * inv_count;
//   else:  Yout [n][3].
template <bool BF16, bool TRAIN>
__global__ void __launch_bounds__(MLP_THREADS) k_mlp_tile(const float* __restrict__ params, const float* __restrict__ X,
                                                          const float* __restrict__ Yt, const int* __restrict__ idx,
                                                          int base, int n, float inv_count, float* __restrict__ grad_part,
                                                          float* __restrict__ loss_part, float* __restrict__ Yout) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem& S = *reinterpret_cast<Smem*>(smem_raw);
    const int tid = threadIdx.x;
    const int t0 = base + blockIdx.x * MLP_T;   // first sample slot of this tile

    // parameters, padded
    for (int e = tid; e < NH * PI_; e += MLP_THREADS) {
        const int j = e / PI_, k = e % PI_;
        S.W1[e] = k < NI ? params[OFF_W1 + j * NI + k] : 0.f;
    }
    for (int e = tid; e < NH * NH; e += MLP_THREADS) {
        S.W2[e] = params[OFF_W2 + e];
        S.W3[e] = params[OFF_W3 + e];
    }
    for (int e = tid; e < PO * NH; e += MLP_THREADS) {
        const int j = e / NH;
        S.W4[e] = j < NO ? params[OFF_W4 + e] : 0.f;
    }
    for (int e = tid; e < NH; e += MLP_THREADS) {
        S.b1[e] = params[OFF_B1 + e]; S.b2[e] = params[OFF_B2 + e]; S.b3[e] = params[OFF_B3 + e];
    }
    if (tid < PO) S.b4[tid] = tid < NO ? params[OFF_B4 + tid] : 0.f;
    // inputs
    for (int e = tid; e < MLP_T * PI_; e += MLP_THREADS) {
        const int s = e / PI_, k = e % PI_;
        const int slot = t0 + s;
        float v = 0.f;
        if (k < NI && slot < n) v = X[(size_t)(idx ? idx[slot] : slot) * NI + k];
        S.H0[e] = v;
    }
    __syncthreads();

    // ---- forward ----
    gemm<BF16>(MLP_T, NH, PI_, S.H0, PI_, 1, S.W1, 1, PI_, [&](int m, int j, float v) {
        const float z = v + S.b1[j];
        S.Z1[m * NH + j] = z; S.H1[m * NH + j] = silu(z);
    });
    __syncthreads();
    gemm<BF16>(MLP_T, NH, NH, S.H1, NH, 1, S.W2, 1, NH, [&](int m, int j, float v) {
        const float z = v + S.b2[j];
        S.Z2[m * NH + j] = z; S.H2[m * NH + j] = silu(z);
    });
    __syncthreads();
    gemm<BF16>(MLP_T, NH, NH, S.H2, NH, 1, S.W3, 1, NH, [&](int m, int j, float v) {
        const float z = v + S.b3[j];
        S.Z3[m * NH + j] = z; S.H3[m * NH + j] = silu(z);
    });
    __syncthreads();
    gemm<BF16>(MLP_T, PO, NH, S.H3, NH, 1, S.W4, 1, NH, [&](int m, int j, float v) { S.Y[m * PO + j] = v + S.b4[j]; });
    __syncthreads();

    if constexpr (!TRAIN) {
        for (int e = tid; e < MLP_T * NO; e += MLP_THREADS) {
            const int s = e / NO, o = e % NO;
            if (t0 + s < n) Yout[(size_t)(t0 + s) * NO + o] = S.Y[s * PO + o];
        }
        return;
    } else {
        // ---- loss and dL/dY (kept in dA as [T][PO]) ----
        float se = 0.f;
        for (int e = tid; e < MLP_T * PO; e += MLP_THREADS) {
            const int s = e / PO, o = e % PO;
            const int slot = t0 + s;
            float d = 0.f;
            if (o < NO && slot < n) {
                const float r = S.Y[e] - Yt[(size_t)(idx ? idx[slot] : slot) * NO + o];
                se += r * r;
                d = 2.f * r * inv_count;
            }
            S.dA[e] = d;
        }
        for (int o = 16; o > 0; o >>= 1) se += __shfl_down_sync(0xffffffffu, se, o);
        if ((tid & 31) == 0) S.red[tid >> 5] = se;
        __syncthreads();
        float* gp = grad_part + (size_t)blockIdx.x * NP;
        if (tid == 0) {
            float tot = 0.f;
            for (int w = 0; w < MLP_THREADS / 32; ++w) tot += S.red[w];
            loss_part[blockIdx.x] = tot;
        }
        // ---- layer 4 ----
        gemm<BF16>(PO, NH, MLP_T, S.dA, 1, PO, S.H3, NH, 1, [&](int j, int k, float v) {
            if (j < NO) gp[OFF_W4 + j * NH + k] = v;
        });
        if (tid < NO) {
            float b = 0.f;
            for (int s = 0; s < MLP_T; ++s) b += S.dA[s * PO + tid];
            gp[OFF_B4 + tid] = b;
        }
        gemm<BF16>(MLP_T, NH, PO, S.dA, PO, 1, S.W4, NH, 1, [&](int m, int k, float v) {
            S.dB[m * NH + k] = v * dsilu(S.Z3[m * NH + k]);
        });
        __syncthreads();
        // ---- layer 3 (dZ3 in dB) ----
        gemm<BF16>(NH, NH, MLP_T, S.dB, 1, NH, S.H2, NH, 1, [&](int j, int k, float v) { gp[OFF_W3 + j * NH + k] = v; });
        if (tid < NH) {
            float b = 0.f;
            for (int s = 0; s < MLP_T; ++s) b += S.dB[s * NH + tid];
            gp[OFF_B3 + tid] = b;
        }
        gemm<BF16>(MLP_T, NH, NH, S.dB, NH, 1, S.W3, NH, 1, [&](int m, int k, float v) {
            S.dA[m * NH + k] = v * dsilu(S.Z2[m * NH + k]);
        });
        __syncthreads();
        // ---- layer 2 (dZ2 in dA) ----
        gemm<BF16>(NH, NH, MLP_T, S.dA, 1, NH, S.H1, NH, 1, [&](int j, int k, float v) { gp[OFF_W2 + j * NH + k] = v; });
        if (tid < NH) {
            float b = 0.f;
            for (int s = 0; s < MLP_T; ++s) b += S.dA[s * NH + tid];
            gp[OFF_B2 + tid] = b;
        }
        gemm<BF16>(MLP_T, NH, NH, S.dA, NH, 1, S.W2, NH, 1, [&](int m, int k, float v) {
            S.dB[m * NH + k] = v * dsilu(S.Z1[m * NH + k]);
        });
        __syncthreads();
        // ---- layer 1 (dZ1 in dB) ----
        gemm<BF16>(NH, PI_, MLP_T, S.dB, 1, NH, S.H0, PI_, 1, [&](int j, int k, float v) {
            if (k < NI) gp[OFF_W1 + j * NI + k] = v;
        });
        if (tid < NH) {
            float b = 0.f;
            for (int s = 0; s < MLP_T; ++s) b += S.dB[s * NH + tid];
            gp[OFF_B1 + tid] = b;
        }
    }
}

// Sum of the tile partials (tile order) and one Adam step. With lr = 0 only
// the gradient (and loss) is produced.
__global__ void k_mlp_adam(float* __restrict__ params, float* __restrict__ m1, float* __restrict__ m2,
                           const float* __restrict__ grad_part, int nparts, const float* __restrict__ loss_part,
                           float inv_count, float lr, float beta1, float beta2, float eps, float bc1, float bc2,
                           float* __restrict__ grad_out, float* __restrict__ loss_out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p == 0 && loss_out) {
        float l = 0.f;
        for (int c = 0; c < nparts; ++c) l += loss_part[c];
        *loss_out = l * inv_count;
    }
    if (p >= NP) return;
    float g = 0.f;
    for (int c = 0; c < nparts; ++c) g += grad_part[(size_t)c * NP + p];
    if (grad_out) grad_out[p] = g;
    if (lr == 0.f) return;
    const float a = beta1 * m1[p] + (1.f - beta1) * g;
    const float b = beta2 * m2[p] + (1.f - beta2) * g * g;
    m1[p] = a; m2[p] = b;
    params[p] -= lr * (a / bc1) / (sqrtf(b / bc2) + eps);
}

// ---------------------------------------------------------------------------
//  k_mlp_fwd_tc: BF16 inference on the fifth-generation tensor cores.
//
//  One CTA of 128 threads owns 128 samples: thread i is sample i, and row i
//  of every product. Each layer is D[128 x N] = A[128 x K] . W^T with A (the
//  activations) and W (the weights, [out][in]) in shared memory as BF16 and D
//  in tensor memory (FP32, 64 columns allocated per CTA):
//    thread 0 issues tcgen05.mma (kind::f16, cta_group::1, M = 128,
//    N = 64 or 16, K = 16 per instruction) and tcgen05.commit to an mbarrier;
//    every warp then reads its 32 rows of D with tcgen05.ld (32x32b), adds the
//    bias, applies SiLU and writes the next layer's A in BF16.
//  Operand layout in shared memory: K-major with no swizzle. The 8 x 8 BF16
//  core matrices are 128 contiguous bytes (8 rows of 16 bytes). Row r, column k
//  of an R-row operand is at byte ((k / 8) * R + r) * 16 + (k % 8) * 2, so the
//  stride between 8-row groups (SBO) is 128 bytes and the stride between the
//  two 8-column halves of a K = 16 step (LBO) is R * 16 bytes.
//  Waits on the mbarrier are bounded; a timeout sets *err, and the tensor
//  memory is released on every path.
// ---------------------------------------------------------------------------
constexpr int TC_M = 128;              // samples per CTA
constexpr int TC_COLS = 64;            // tensor-memory columns (FP32 accumulators)

struct TcSmem {
    alignas(128) __nv_bfloat16 A[NH / 8][TC_M][8];       // activations, K-major core matrices
    alignas(128) __nv_bfloat16 W1[PI_ / 8][NH][8];
    alignas(128) __nv_bfloat16 W2[NH / 8][NH][8];
    alignas(128) __nv_bfloat16 W3[NH / 8][NH][8];
    alignas(128) __nv_bfloat16 W4[NH / 8][PO][8];
    float b1[NH], b2[NH], b3[NH], b4[PO];
    alignas(8) uint64_t mbar;
    uint32_t tmem_base;
};

__device__ __forceinline__ uint64_t umma_desc(const void* smem, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(smem);
    uint64_t d = 0;
    d |= (uint64_t)((a >> 4) & 0x3FFFu);                     // start address
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;       // leading dimension byte offset
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;       // stride dimension byte offset
    d |= (uint64_t)1 << 46;                                  // descriptor version (sm_100)
    return d;                                                // base offset 0, no swizzle
}

// BF16 x BF16 -> FP32, both operands K-major, M = 128
__host__ __device__ constexpr uint32_t umma_idesc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);
}

__device__ __forceinline__ bool tc_wait(uint64_t* m, uint32_t parity) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(m);
    for (int it = 0; it < (1 << 22); ++it) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(ok) : "r"(a), "r"(parity) : "memory");
        if (ok) return true;
    }
    return false;
}

// D[tmem] = A . W^T over K (multiple of 16), issued by one thread, completion on mbar
__device__ __forceinline__ void tc_layer(uint32_t tmem, const void* A, const void* W, int K, int N, uint64_t* mbar) {
    const uint32_t idesc = umma_idesc(N);
    for (int k16 = 0; k16 < K / 16; ++k16) {
        const uint64_t da = umma_desc((const char*)A + (size_t)k16 * 2 * TC_M * 16, TC_M * 16, 128);
        const uint64_t db = umma_desc((const char*)W + (size_t)k16 * 2 * N * 16, N * 16, 128);
        const uint32_t acc = k16 > 0;
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}"
            :: "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0)
            : "memory");
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"((uint32_t)__cvta_generic_to_shared(mbar)) : "memory");
}

// 16 FP32 columns of this thread's row of D
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

// W[out][in] (FP32, global) -> BF16 K-major core matrices with R rows (outputs)
// and KP columns (inputs, zero-padded), rows >= rows_valid zero
__device__ __forceinline__ void tc_load_w(__nv_bfloat16* dst, const float* w, int R, int rows_valid, int KP, int kin) {
    for (int e = threadIdx.x; e < R * KP; e += blockDim.x) {
        const int r = e / KP, k = e % KP;
        const float v = (r < rows_valid && k < kin) ? w[r * kin + k] : 0.f;
        dst[((size_t)(k / 8) * R + r) * 8 + (k % 8)] = __float2bfloat16_rn(v);
    }
}

__global__ void __launch_bounds__(TC_M) k_mlp_fwd_tc(const float* __restrict__ params, const float* __restrict__ X,
                                                     int n, float* __restrict__ Yout, int* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char tc_raw[];
    TcSmem& S = *reinterpret_cast<TcSmem*>(tc_raw);
    const int tid = threadIdx.x, warp = tid >> 5;
    const int row = blockIdx.x * TC_M + tid;

    if (warp == 0) {   // tensor memory: one warp allocates, the same warp frees
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"((uint32_t)__cvta_generic_to_shared(&S.tmem_base)), "r"(TC_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"((uint32_t)__cvta_generic_to_shared(&S.mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_load_w(&S.W1[0][0][0], params + OFF_W1, NH, NH, PI_, NI);
    tc_load_w(&S.W2[0][0][0], params + OFF_W2, NH, NH, NH, NH);
    tc_load_w(&S.W3[0][0][0], params + OFF_W3, NH, NH, NH, NH);
    tc_load_w(&S.W4[0][0][0], params + OFF_W4, PO, NO, NH, NH);
    for (int e = tid; e < NH; e += TC_M) { S.b1[e] = params[OFF_B1 + e]; S.b2[e] = params[OFF_B2 + e]; S.b3[e] = params[OFF_B3 + e]; }
    if (tid < PO) S.b4[tid] = tid < NO ? params[OFF_B4 + tid] : 0.f;
    {   // this thread's input row, padded to 16
        float xv[PI_];
#pragma unroll
        for (int k = 0; k < PI_; ++k) xv[k] = (k < NI && row < n) ? X[(size_t)row * NI + k] : 0.f;
#pragma unroll
        for (int c = 0; c < PI_ / 8; ++c)
#pragma unroll
            for (int j = 0; j < 8; ++j) S.A[c][tid][j] = __float2bfloat16_rn(xv[c * 8 + j]);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // operands visible to the tensor cores
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = S.tmem_base;
    const uint32_t my_lanes = tmem + ((uint32_t)(warp * 32) << 16);

    bool ok = true;
    uint32_t phase = 0, last = 0;   // last: the phase of the most recent commit
    const void* Ws[3] = {&S.W1[0][0][0], &S.W2[0][0][0], &S.W3[0][0][0]};
    const float* bs[3] = {S.b1, S.b2, S.b3};
    for (int l = 0; l < 3 && ok; ++l) {
        if (tid == 0) tc_layer(tmem, &S.A[0][0][0], Ws[l], l == 0 ? PI_ : NH, NH, &S.mbar);
        last = phase;
        ok = __all_sync(0xffffffffu, tc_wait(&S.mbar, phase));   // warp-uniform: tcgen05.ld is .sync.aligned
        phase ^= 1;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (ok) {
            float h[NH];
#pragma unroll
            for (int q = 0; q < NH / 16; ++q) tc_ld16(my_lanes + q * 16, h + q * 16);
#pragma unroll
            for (int j = 0; j < NH; ++j) h[j] = silu(h[j] + bs[l][j]);
#pragma unroll
            for (int c = 0; c < NH / 8; ++c)
#pragma unroll
                for (int j = 0; j < 8; ++j) S.A[c][tid][j] = __float2bfloat16_rn(h[c * 8 + j]);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        ok = __syncthreads_and(ok);
    }
    if (ok) {
        if (tid == 0) tc_layer(tmem, &S.A[0][0][0], &S.W4[0][0][0], NH, PO, &S.mbar);
        last = phase;
        ok = __all_sync(0xffffffffu, tc_wait(&S.mbar, phase));
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (ok) {
            float y[16];
            tc_ld16(my_lanes, y);
            if (row < n)
#pragma unroll
                for (int o = 0; o < NO; ++o) Yout[(size_t)row * NO + o] = y[o] + S.b4[o];
        }
    }
    ok = __syncthreads_and(ok);   // the same verdict in every warp
    if (!ok) {
        // A wait gave up while the last layer's MMAs may still be writing
        // tensor memory: wait (bounded) for their commit before the columns
        // are freed.
        if (tid == 0) {
            atomicExch(err, 1);
            tc_wait(&S.mbar, last);
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(TC_COLS));
}

template <bool BF16, bool TRAIN>
cudaError_t prepare_tile() {
    return cudaFuncSetAttribute(k_mlp_tile<BF16, TRAIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem));
}

thread_local std::string g_mlp_error;

}  // namespace

struct lbmgpu_mlp {
    int device = 0, bf16 = 0;
    cudaStream_t stream = nullptr;
    float *params = nullptr, *m1 = nullptr, *m2 = nullptr;
    float *X = nullptr, *Y = nullptr;   // training set
    int n = 0, cap = 0;
    int* idx = nullptr;
    int idx_cap = 0;
    float* grad_part = nullptr;
    float* loss_part = nullptr;
    int part_cap = 0;                   // tiles
    float *xin = nullptr, *yout = nullptr;
    int xin_cap = 0, yout_cap = 0;      // floats
    float* small = nullptr;             // [0] loss, [1..NP] gradient
    int* d_err = nullptr;               // tensor-core forward: a bounded wait gave up
    long long t = 0;                    // Adam steps taken
    float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
    std::string err;
};

namespace {

int mfail(lbmgpu_mlp* m, int code, const std::string& msg) {
    if (m) m->err = msg; else g_mlp_error = msg;
    return code;
}

#define MTRY(m, call)                                                                               \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            return mfail(m, e_ == cudaErrorMemoryAllocation ? LBMGPU_ERR_NOMEM : LBMGPU_ERR_CUDA,     \
                         std::string(#call) + ": " + cudaGetErrorString(e_));                       \
    } while (0)

cudaError_t grow(float** p, int* cap, long long need_elems) {
    if (need_elems <= *cap) return cudaSuccess;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    cudaError_t e = cudaMalloc(p, (size_t)need_elems * sizeof(float));
    if (e == cudaSuccess) *cap = (int)need_elems;
    return e;
}

int ensure_parts(lbmgpu_mlp* m, int tiles) {
    if (tiles <= m->part_cap) return LBMGPU_OK;
    if (m->grad_part) cudaFree(m->grad_part);
    if (m->loss_part) cudaFree(m->loss_part);
    m->grad_part = m->loss_part = nullptr;
    m->part_cap = 0;
    MTRY(m, cudaMalloc(&m->grad_part, (size_t)tiles * NP * sizeof(float)));
    MTRY(m, cudaMalloc(&m->loss_part, (size_t)tiles * sizeof(float)));
    m->part_cap = tiles;
    return LBMGPU_OK;
}

// fwd + bwd over samples [0, count) of the order `idx` (or identity), then
// the reduction (and Adam step when lr > 0)
int train_batch(lbmgpu_mlp* m, const int* idx, int base, int count, float lr, float* d_grad, float* d_loss) {
    const int tiles = (count + MLP_T - 1) / MLP_T;
    int rc = ensure_parts(m, tiles);
    if (rc) return rc;
    const float inv = 1.0f / (float)(count * NO);
    const size_t sm = sizeof(Smem);
    // the tile kernel sees slots [base, base + count) of idx as its samples
    if (m->bf16)
        k_mlp_tile<true, true><<<tiles, MLP_THREADS, sm, m->stream>>>(m->params, m->X, m->Y, idx, base, base + count,
                                                                      inv, m->grad_part, m->loss_part, nullptr);
    else
        k_mlp_tile<false, true><<<tiles, MLP_THREADS, sm, m->stream>>>(m->params, m->X, m->Y, idx, base, base + count,
                                                                       inv, m->grad_part, m->loss_part, nullptr);
    float bc1 = 1.f, bc2 = 1.f;
    if (lr > 0.f) {
        m->t += 1;
        bc1 = 1.f - powf(m->beta1, (float)m->t);
        bc2 = 1.f - powf(m->beta2, (float)m->t);
    }
    k_mlp_adam<<<(NP + 255) / 256, 256, 0, m->stream>>>(m->params, m->m1, m->m2, m->grad_part, tiles, m->loss_part, inv,
                                                        lr, m->beta1, m->beta2, m->eps, bc1, bc2, d_grad, d_loss);
    MTRY(m, cudaGetLastError());
    return LBMGPU_OK;
}

}  // namespace

extern "C" {

int lbmgpu_mlp_create(int device, int bf16, lbmgpu_mlp** out) {
    if (!out) return mfail(nullptr, LBMGPU_ERR_INVALID, "null output pointer");
    *out = nullptr;
    lbmgpu_mlp* m = new lbmgpu_mlp();
    m->device = device;
    m->bf16 = bf16 ? 1 : 0;
    auto bail = [&](cudaError_t e, const char* what) {
        g_mlp_error = std::string(what) + ": " + cudaGetErrorString(e);
        lbmgpu_mlp_destroy(m);
        return e == cudaErrorMemoryAllocation ? LBMGPU_ERR_NOMEM : LBMGPU_ERR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaSetDevice(device)) != cudaSuccess) return bail(e, "cudaSetDevice");
    if ((e = prepare_tile<true, true>()) != cudaSuccess) return bail(e, "smem attribute");
    if ((e = prepare_tile<false, true>()) != cudaSuccess) return bail(e, "smem attribute");
    if ((e = prepare_tile<true, false>()) != cudaSuccess) return bail(e, "smem attribute");
    if ((e = prepare_tile<false, false>()) != cudaSuccess) return bail(e, "smem attribute");
    if ((e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking)) != cudaSuccess) return bail(e, "stream");
    if ((e = cudaMalloc(&m->params, NP * sizeof(float))) != cudaSuccess) return bail(e, "cudaMalloc");
    if ((e = cudaMalloc(&m->m1, NP * sizeof(float))) != cudaSuccess) return bail(e, "cudaMalloc");
    if ((e = cudaMalloc(&m->m2, NP * sizeof(float))) != cudaSuccess) return bail(e, "cudaMalloc");
    if ((e = cudaMalloc(&m->small, (NP + 1) * sizeof(float))) != cudaSuccess) return bail(e, "cudaMalloc");
    if ((e = cudaMalloc(&m->d_err, sizeof(int))) != cudaSuccess) return bail(e, "cudaMalloc");
    if ((e = cudaMemsetAsync(m->d_err, 0, sizeof(int), m->stream)) != cudaSuccess) return bail(e, "memset");
    if ((e = cudaMemsetAsync(m->params, 0, NP * sizeof(float), m->stream)) != cudaSuccess) return bail(e, "memset");
    if ((e = cudaMemsetAsync(m->m1, 0, NP * sizeof(float), m->stream)) != cudaSuccess) return bail(e, "memset");
    if ((e = cudaMemsetAsync(m->m2, 0, NP * sizeof(float), m->stream)) != cudaSuccess) return bail(e, "memset");
    if ((e = cudaStreamSynchronize(m->stream)) != cudaSuccess) return bail(e, "sync");
    *out = m;
    return LBMGPU_OK;
}

int lbmgpu_mlp_destroy(lbmgpu_mlp* m) {
    if (!m) return LBMGPU_OK;
    cudaSetDevice(m->device);
    if (m->stream) cudaStreamSynchronize(m->stream);
    void* ptrs[] = {m->params, m->m1, m->m2, m->X, m->Y, m->idx, m->grad_part, m->loss_part, m->xin, m->yout, m->small,
                    m->d_err};
    for (void* p : ptrs) if (p) cudaFree(p);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
    return LBMGPU_OK;
}

int lbmgpu_mlp_set_params(lbmgpu_mlp* m, const float* params, int reset_optimizer) {
    if (!m || !params) return LBMGPU_ERR_INVALID;
    MTRY(m, cudaSetDevice(m->device));
    MTRY(m, cudaMemcpyAsync(m->params, params, NP * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    if (reset_optimizer) {
        MTRY(m, cudaMemsetAsync(m->m1, 0, NP * sizeof(float), m->stream));
        MTRY(m, cudaMemsetAsync(m->m2, 0, NP * sizeof(float), m->stream));
        m->t = 0;
    }
    MTRY(m, cudaStreamSynchronize(m->stream));
    return LBMGPU_OK;
}

int lbmgpu_mlp_get_params(lbmgpu_mlp* m, float* params) {
    if (!m || !params) return LBMGPU_ERR_INVALID;
    MTRY(m, cudaSetDevice(m->device));
    MTRY(m, cudaMemcpyAsync(params, m->params, NP * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    MTRY(m, cudaStreamSynchronize(m->stream));
    return LBMGPU_OK;
}

int lbmgpu_mlp_set_adam(lbmgpu_mlp* m, float beta1, float beta2, float eps) {
    if (!m || !(beta1 >= 0.f && beta1 < 1.f) || !(beta2 >= 0.f && beta2 < 1.f) || !(eps > 0.f))
        return mfail(m, LBMGPU_ERR_INVALID, "Adam needs 0 <= beta1, beta2 < 1 and eps > 0");
    m->beta1 = beta1; m->beta2 = beta2; m->eps = eps;
    return LBMGPU_OK;
}

int lbmgpu_mlp_set_data(lbmgpu_mlp* m, const float* x, const float* y, int n) {
    if (!m || !x || !y || n < 1) return mfail(m, LBMGPU_ERR_INVALID, "need n >= 1 samples");
    MTRY(m, cudaSetDevice(m->device));
    if (n > m->cap) {
        if (m->X) cudaFree(m->X);
        if (m->Y) cudaFree(m->Y);
        m->X = m->Y = nullptr;
        m->cap = 0;
        MTRY(m, cudaMalloc(&m->X, (size_t)n * NI * sizeof(float)));
        MTRY(m, cudaMalloc(&m->Y, (size_t)n * NO * sizeof(float)));
        m->cap = n;
    }
    MTRY(m, cudaMemcpyAsync(m->X, x, (size_t)n * NI * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    MTRY(m, cudaMemcpyAsync(m->Y, y, (size_t)n * NO * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    MTRY(m, cudaStreamSynchronize(m->stream));
    m->n = n;
    return LBMGPU_OK;
}

int lbmgpu_mlp_train_epoch(lbmgpu_mlp* m, const int* order, int n_order, int batch, float lr, float* mean_loss) {
    if (!m || !order || n_order < 1 || batch < 1 || !(lr > 0.f))
        return mfail(m, LBMGPU_ERR_INVALID, "need an order of >= 1 samples, batch >= 1 and lr > 0");
    if (m->n < 1) return mfail(m, LBMGPU_ERR_INVALID, "no training data (lbmgpu_mlp_set_data)");
    for (int k = 0; k < n_order; ++k)
        if (order[k] < 0 || order[k] >= m->n) return mfail(m, LBMGPU_ERR_INVALID, "order holds an index out of range");
    MTRY(m, cudaSetDevice(m->device));
    if (n_order > m->idx_cap) {
        if (m->idx) cudaFree(m->idx);
        m->idx = nullptr;
        m->idx_cap = 0;
        MTRY(m, cudaMalloc(&m->idx, (size_t)n_order * sizeof(int)));
        m->idx_cap = n_order;
    }
    MTRY(m, cudaMemcpyAsync(m->idx, order, (size_t)n_order * sizeof(int), cudaMemcpyHostToDevice, m->stream));
    const int steps = (n_order + batch - 1) / batch;
    std::vector<float> losses(steps);
    float* d_losses = nullptr;
    MTRY(m, cudaMalloc(&d_losses, (size_t)steps * sizeof(float)));
    for (int s = 0; s < steps; ++s) {
        const int base = s * batch, count = std::min(batch, n_order - base);
        const int rc = train_batch(m, m->idx, base, count, lr, nullptr, d_losses + s);
        if (rc) { cudaFree(d_losses); return rc; }
    }
    cudaError_t e = cudaMemcpyAsync(losses.data(), d_losses, (size_t)steps * sizeof(float), cudaMemcpyDeviceToHost,
                                    m->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
    cudaFree(d_losses);
    MTRY(m, e);
    if (mean_loss) {
        double acc = 0;
        for (float l : losses) acc += l;
        *mean_loss = (float)(acc / steps);
    }
    return LBMGPU_OK;
}

int lbmgpu_mlp_loss_grad(lbmgpu_mlp* m, float* loss, float* grad) {
    if (!m || !loss) return LBMGPU_ERR_INVALID;
    if (m->n < 1) return mfail(m, LBMGPU_ERR_INVALID, "no training data (lbmgpu_mlp_set_data)");
    MTRY(m, cudaSetDevice(m->device));
    const int rc = train_batch(m, nullptr, 0, m->n, 0.f, m->small + 1, m->small);
    if (rc) return rc;
    MTRY(m, cudaMemcpyAsync(loss, m->small, sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    if (grad) MTRY(m, cudaMemcpyAsync(grad, m->small + 1, NP * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    MTRY(m, cudaStreamSynchronize(m->stream));
    return LBMGPU_OK;
}

int lbmgpu_mlp_forward_ex(lbmgpu_mlp* m, const float* x, int n, float* y, int path) {
    if (!m || !x || !y || n < 1) return mfail(m, LBMGPU_ERR_INVALID, "need n >= 1 inputs");
    if (path != LBMGPU_MLP_PATH_AUTO && path != LBMGPU_MLP_PATH_WARP && path != LBMGPU_MLP_PATH_TCGEN05)
        return mfail(m, LBMGPU_ERR_INVALID, "unknown forward path");
    if (path == LBMGPU_MLP_PATH_TCGEN05 && !m->bf16)
        return mfail(m, LBMGPU_ERR_INVALID, "the tensor-memory path computes in BF16: create the network with bf16 = 1");
    MTRY(m, cudaSetDevice(m->device));
    MTRY(m, grow(&m->xin, &m->xin_cap, (long long)n * NI));
    MTRY(m, grow(&m->yout, &m->yout_cap, (long long)n * NO));
    MTRY(m, cudaMemcpyAsync(m->xin, x, (size_t)n * NI * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    const bool tc = m->bf16 && path != LBMGPU_MLP_PATH_WARP;
    if (tc) {
        k_mlp_fwd_tc<<<(n + TC_M - 1) / TC_M, TC_M, sizeof(TcSmem), m->stream>>>(m->params, m->xin, n, m->yout, m->d_err);
    } else {
        const int tiles = (n + MLP_T - 1) / MLP_T;
        const size_t sm = sizeof(Smem);
        if (m->bf16)
            k_mlp_tile<true, false><<<tiles, MLP_THREADS, sm, m->stream>>>(m->params, m->xin, nullptr, nullptr, 0, n,
                                                                           0.f, nullptr, nullptr, m->yout);
        else
            k_mlp_tile<false, false><<<tiles, MLP_THREADS, sm, m->stream>>>(m->params, m->xin, nullptr, nullptr, 0, n,
                                                                            0.f, nullptr, nullptr, m->yout);
    }
    MTRY(m, cudaGetLastError());
    int err = 0;
    MTRY(m, cudaMemcpyAsync(y, m->yout, (size_t)n * NO * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    if (tc) MTRY(m, cudaMemcpyAsync(&err, m->d_err, sizeof(int), cudaMemcpyDeviceToHost, m->stream));
    MTRY(m, cudaStreamSynchronize(m->stream));
    if (err) return mfail(m, LBMGPU_ERR_WATCHDOG, "a tensor-core layer did not complete in time");
    return LBMGPU_OK;
}

int lbmgpu_mlp_forward(lbmgpu_mlp* m, const float* x, int n, float* y) {
    return lbmgpu_mlp_forward_ex(m, x, n, y, LBMGPU_MLP_PATH_AUTO);
}

const char* lbmgpu_mlp_last_error(const lbmgpu_mlp* m) { return m ? m->err.c_str() : g_mlp_error.c_str(); }

}  // extern "C"
