// FP32-shifted and FP16-storage forms (deviations f_i - w_i stored; FP64
// arithmetic for FP32 storage and FP32 arithmetic for FP16 storage; FP64
// boundary-link sums and rigid body).
#include "lbm_launch_impl.cuh"

namespace lbmgpu {
const Launchers& launchers_f32() {
    static const Launchers l = make_launchers<StoreF32>();
    return l;
}
const Launchers& launchers_f16() {
    static const Launchers l = make_launchers<StoreF16>();
    return l;
}
}  // namespace lbmgpu
