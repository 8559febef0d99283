// pk_fast_mhd3.cu -- tolerance-mode fused and batched sweeps for ionized + neutral + dust + B + psi.
// Compiled with --fmad=true (multiply-add contraction), unlike every other
// unit; it instantiates only the FAST kernels (pk_fast.cuh arithmetic).
#include "pk_launch.cuh"

namespace pk {
const FastOps* fast_ops_mhd3() { return make_fast_ops<Phys<K_ION, K_NEU, K_DST, true>>(); }
}  // namespace pk
