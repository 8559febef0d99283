// pk_fast_mhd1.cu -- tolerance-mode fused and batched sweeps for ionized fluid + B + psi.
// Compiled with --fmad=true (multiply-add contraction), unlike every other
// unit; it instantiates only the FAST kernels (pk_fast.cuh arithmetic).
#include "pk_launch.cuh"

namespace pk {
const FastOps* fast_ops_mhd1() { return make_fast_ops<Phys<K_ION, K_NONE, K_NONE, true>>(); }
}  // namespace pk
