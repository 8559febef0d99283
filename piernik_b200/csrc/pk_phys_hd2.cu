// pk_phys_hd2.cu -- kernels and launches for a fluid with energy plus pressureless dust, no B.
#include "pk_launch.cuh"

namespace pk {
const PhysOps* ops_hd2() { return make_ops<Phys<K_NEU, K_DST, K_NONE, false>>(); }
}  // namespace pk
