// pk_phys_mhd2.cu -- kernels and launches for ionized + neutral fluid + B + psi.
#include "pk_launch.cuh"

namespace pk {
const PhysOps* ops_mhd2() { return make_ops<Phys<K_ION, K_NEU, K_NONE, true>>(); }
}  // namespace pk
