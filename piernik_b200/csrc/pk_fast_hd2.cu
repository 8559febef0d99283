// pk_fast_hd2.cu -- tolerance-mode fused and batched sweeps for neutral + dust (hydro).
// Compiled with --fmad=true (multiply-add contraction), unlike every other
// unit; it instantiates only the FAST kernels (pk_fast.cuh arithmetic).
#include "pk_launch.cuh"

namespace pk {
const FastOps* fast_ops_hd2() { return make_fast_ops<Phys<K_NEU, K_DST, K_NONE, false>>(); }
}  // namespace pk
