// pk_phys_hd1.cu -- kernels and launches for one fluid with energy, no B (solve_cg_u).
#include "pk_launch.cuh"

namespace pk {
const PhysOps* ops_hd1() { return make_ops<Phys<K_NEU, K_NONE, K_NONE, false>>(); }
}  // namespace pk
