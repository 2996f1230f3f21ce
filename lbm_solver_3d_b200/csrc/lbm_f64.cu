// FP64 storage form. Compiled with --fmad=false: the FP64 arithmetic of the
// stream, squirmer and refill kernels then rounds exactly like the reference's
// (which GCC compiles without FMA contraction in ISO C++ mode).
#include "lbm_launch_impl.cuh"

namespace lbmgpu {
const Launchers& launchers_f64() {
    static const Launchers l = make_launchers<StoreF64>();
    return l;
}
size_t squirmer_smem_bytes() { return squirmer_smem(); }
}  // namespace lbmgpu
