// pk_phys_mhd3.cu -- kernels and launches for ionized + neutral + dust + B + psi.
#include "pk_launch.cuh"

namespace pk {
const PhysOps* ops_mhd3() { return make_ops<Phys<K_ION, K_NEU, K_DST, true>>(); }
}  // namespace pk
