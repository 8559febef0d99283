// pk_fast_hd1.cu -- tolerance-mode fused and batched sweeps for neutral fluid (hydro).
// Compiled with --fmad=true (multiply-add contraction), unlike every other
// unit; it instantiates only the FAST kernels (pk_fast.cuh arithmetic).
#include "pk_launch.cuh"

namespace pk {
const FastOps* fast_ops_hd1() { return make_fast_ops<Phys<K_NEU, K_NONE, K_NONE, false>>(); }
}  // namespace pk
